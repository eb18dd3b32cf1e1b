// ORACLE — test infrastructure only (the checker, never the product).
//
// C entry points around the reference's own psp::DistHelmholtz on one
// process (include/psp/dist_helmholtz.hpp and dist_helmholtz/*.hpp,
// compiled unchanged from the reference tree against clique_shim.hpp):
//   the constructor (main.hpp:12-441): panel geometry (PanelV, PanelDepth,
//     PanelPadding, main.hpp:728-790) and the global nested-dissection
//     ordering (localToNaturalMap_, main.hpp:1423-1477);
//   the global sparse rows exactly as Initialize forms them
//     (initialize_finalize.hpp:340-375): GetGlobalVelocity, then
//     FormGlobalRow (527-587) for every row in the reference's order;
//   the PML stretches s1Inv, s2Inv, s3Inv and s3InvArtificial (415-525).
// Clique's symbolic analysis, which the constructor also calls, is not
// reproduced (a no-op here), so nothing that needs the frontal structure is
// exposed.  The members are private in the reference; this translation unit
// opens them to call them as a test harness.
#include "clique_shim.hpp"
#include "psp/discretization.hpp"
#include "psp/dist_uniform_grid.hpp"
#define private public
#include "psp/dist_helmholtz.hpp"
#undef private

#include <complex>
#include <memory>
#include <string>

namespace {
std::string g_error;
typedef psp::DistHelmholtz<double> DH;

template <typename F>
int Guard(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}
}  // namespace

extern "C" {

const char* ref_dh_error() { return g_error.c_str(); }

// bcs: front, right, back, left, top (0 PML, 1 Dirichlet).
int ref_dh_create(double omega, int nx, int ny, int nz, double wx, double wy, double wz, const int* bcs, int bx,
                  int by, int bz, double sigmax, double sigmay, double sigmaz, double damping, int planes, int cutoff,
                  void** out) {
    return Guard([&] {
        psp::Discretization<double> disc(omega, nx, ny, nz, wx, wy, wz, (psp::Boundary)bcs[0],
                                         (psp::Boundary)bcs[1], (psp::Boundary)bcs[2], (psp::Boundary)bcs[3],
                                         (psp::Boundary)bcs[4], bx, by, bz);
        disc.sigmax = sigmax;
        disc.sigmay = sigmay;
        disc.sigmaz = sigmaz;
        psp::cliq::RecordedTrees().clear();
        *out = new DH(disc, 0, damping, planes, cutoff);
    });
}

// Elimination tree t (0 bottom, then the leftover inner panel's if there
// is one, then the top) that the last ref_dh_create built: per node (off,
// size, parent, number of original lower-structure entries), then the
// lower-structure entries of all nodes, concatenated.  Either output may be
// null (counts only).
int ref_dh_tree(int t, int* numNodes, int* numLower, int* info, int* lower) {
    return Guard([&] {
        const auto& trees = psp::cliq::RecordedTrees();
        if (t < 0 || t >= (int)trees.size()) throw std::logic_error("no such elimination tree");
        const auto& T = trees[t];
        *numNodes = (int)T.size();
        int nl = 0;
        for (size_t i = 0; i < T.size(); ++i) {
            if (info) {
                info[4 * i + 0] = T[i].off;
                info[4 * i + 1] = T[i].size;
                info[4 * i + 2] = T[i].parent;
                info[4 * i + 3] = (int)T[i].lowerStruct.size();
            }
            if (lower) std::copy(T[i].lowerStruct.begin(), T[i].lowerStruct.end(), lower + nl);
            nl += (int)T[i].lowerStruct.size();
        }
        *numLower = nl;
    });
}

void ref_dh_destroy(void* h) { delete static_cast<DH*>(h); }

// Per panel: lowest v, depth, padding (v = nz - 1 - z).
int ref_dh_geometry(void* h, int* numPanels, int* info) {
    return Guard([&] {
        const DH& H = *static_cast<DH*>(h);
        *numPanels = H.numPanels_;
        if (info)
            for (int p = 0; p < H.numPanels_; ++p) {
                info[3 * p + 0] = H.PanelV(p);
                info[3 * p + 1] = H.PanelDepth(p);
                info[3 * p + 2] = H.PanelPadding(p);
            }
    });
}

// The reference's row order: natural index of every row.
int ref_dh_local_to_natural(void* h, int* out) {
    return Guard([&] {
        const DH& H = *static_cast<DH*>(h);
        std::copy(H.localToNaturalMap_.begin(), H.localToNaturalMap_.end(), out);
    });
}

// Global rows for a natural-order velocity: rowOffsets (N + 1 entries) and
// the complex entries of every row (center, then the -x, +x, -y, +y, -v, +v
// neighbours that exist), as Initialize forms them.  With entries null only
// *nnz is set.
int ref_dh_rows(void* h, const double* velocity, int* nnz, int* rowOffsets, double* entries) {
    return Guard([&] {
        DH& H = *static_cast<DH*>(h);
        const int nx = H.disc_.nx, ny = H.disc_.ny, nz = H.disc_.nz;
        *nnz = H.localRowOffsets_.back();
        if (!entries) return;
        psp::DistUniformGrid<double> vel(nx, ny, nz, 0, 1);
        std::copy(velocity, velocity + (size_t)nx * ny * nz, vel.Buffer());
        std::vector<double> myGlobalVelocity;
        std::vector<int> offsets;
        H.GetGlobalVelocity(vel, myGlobalVelocity, offsets);
        H.localEntries_.resize(H.localRowOffsets_.back());
        for (int iLocal = 0; iLocal < H.localSize_; ++iLocal) {
            const int naturalIndex = H.localToNaturalMap_[iLocal];
            const int x = naturalIndex % nx, y = (naturalIndex / nx) % ny, z = naturalIndex / (nx * ny);
            const int proc = vel.OwningProcess(x, y, z);
            const double alpha = myGlobalVelocity[offsets[proc]++];
            H.FormGlobalRow(alpha, x, y, (nz - 1) - z, H.localRowOffsets_[iLocal]);
        }
        std::copy(H.localRowOffsets_.begin(), H.localRowOffsets_.end(), rowOffsets);
        std::copy(H.localEntries_.begin(), H.localEntries_.end(), reinterpret_cast<std::complex<double>*>(entries));
    });
}

// PML stretch `which` (1 s1Inv, 2 s2Inv, 3 s3Inv, 4 s3InvArtificial with
// vOffset) at n indices.
int ref_dh_stretch(void* h, int which, int n, const int* idx, int vOffset, double* out) {
    return Guard([&] {
        const DH& H = *static_cast<DH*>(h);
        std::complex<double>* o = reinterpret_cast<std::complex<double>*>(out);
        for (int i = 0; i < n; ++i)
            o[i] = which == 1 ? H.s1Inv(idx[i])
                 : which == 2 ? H.s2Inv(idx[i])
                 : which == 3 ? H.s3Inv(idx[i])
                              : H.s3InvArtificial(idx[i], vOffset);
    });
}

}  // extern "C"
