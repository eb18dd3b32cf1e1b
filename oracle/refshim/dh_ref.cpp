// ORACLE — test infrastructure only (the checker, never the product).
//
// C entry points around the reference's own psp::DistHelmholtz on one
// process (include/psp/dist_helmholtz.hpp and dist_helmholtz/*.hpp,
// compiled unchanged from the reference tree with its psp.hpp, against the
// stand-in for Clique and Elemental in clique.hpp):
//   the constructor (main.hpp:12-441): panel geometry (PanelV, PanelDepth,
//     PanelPadding, main.hpp:728-790) and the global nested-dissection
//     ordering (localToNaturalMap_, main.hpp:1423-1477);
//   the global sparse rows exactly as Initialize forms them
//     (initialize_finalize.hpp:340-375): GetGlobalVelocity, then
//     FormGlobalRow (527-587) for every row in the reference's order;
//   the PML stretches s1Inv, s2Inv, s3Inv and s3InvArtificial (415-525);
//   the panel fronts as Initialize fills them (FillPanelFronts with
//   FormLowerColumnOfNode, 589-806, 1284-1394), on node structures from
//   the stand-in's symbolic analysis;
// Clique's symbolic analysis, which the constructor also calls, is not
// reproduced (a no-op here), so nothing that needs the frontal structure is
// exposed.  The members are private in the reference; this translation unit
// opens them to call them as a test harness.
#include "clique.hpp"
#define private public
#include "psp.hpp"
#undef private

#include <complex>
#include <memory>
#include <string>

// The oracle's panel solve (oracle/psp_oracle.cpp): B := T_p B on panel p's
// planes of a natural-order grid of k interleaved right-hand sides.
extern "C" int oracle_solve_panel(void* h, double* grid, int k, int p);

namespace {
std::string g_error, g_log;
typedef psp::DistHelmholtz<double> DH;
typedef std::complex<double> Cd;

// The global rows exactly as Initialize forms them (initialize_finalize.hpp:
// 340-375) for a natural-order velocity.
void FormRows(DH& H, const double* velocity) {
    const int nx = H.disc_.nx, ny = H.disc_.ny, nz = H.disc_.nz;
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
}

// T_i applied to the right-hand sides of panel i, laid out as the
// reference's SolvePanel hands them to Clique (solve.hpp:736-822): node by
// node of the panel's elimination order, each node's padding rows first
// (zero), then its physical rows, which are the reference's rows
// LocalPanelOffset(i) onwards.  The physical rows go through a natural-order
// grid to the oracle's panel solve and come back the same way.
void OraclePanelSolve(const DH& H, void* oracle, int i, cliq::DistNodalMultiVec<Cd>& X) {
    const cliq::DistSymmInfo& info = H.PanelAnalysis(i);
    const int padding = H.PanelPadding(i), depth = H.PanelDepth(i);
    const int k = X.localNodes.empty() ? 0 : X.localNodes[0].Width();
    const size_t N = (size_t)H.disc_.nx * H.disc_.ny * H.disc_.nz;
    std::vector<Cd> grid(N * k, Cd(0));
    for (int pass = 0; pass < 2; ++pass) {
        int bOff = H.LocalPanelOffset(i);
        for (size_t t = 0; t < info.localNodes.size(); ++t) {
            const int size = info.localNodes[t].size;
            const int paddingSize = (size / (padding + depth)) * padding;
            elem::Matrix<Cd>& mat = X.localNodes[t];
            for (int r = 0; r < size - paddingSize; ++r) {
                Cd* g = &grid[(size_t)H.localToNaturalMap_[bOff + r] * k];
                for (int c = 0; c < k; ++c) {
                    if (pass == 0) g[c] = mat.Get(paddingSize + r, c);
                    else mat.Set(paddingSize + r, c, g[c]);
                }
            }
            bOff += size - paddingSize;
        }
        if (pass == 0 && oracle_solve_panel(oracle, reinterpret_cast<double*>(grid.data()), k, i))
            throw std::runtime_error("oracle panel solve failed");
    }
}

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
        cliq::RecordedTrees().clear();
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
        const auto& trees = cliq::RecordedTrees();
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

void ref_dh_destroy(void* h) {
    DH* H = static_cast<DH*>(h);
    for (auto* f : H->fullInnerFacts_) delete f;
    H->fullInnerFacts_.clear();
    delete H;
}

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

// The reference's own Solve (solve.hpp:12-611: pull, GMRES(m) with its
// sweep Precondition, Multiply and Givens updates, push) of the k
// right-hand sides in `grid` (natural order, interleaved), in place, with
// the global rows formed from `velocity` and Clique's panel solves replaced
// by those of `oracle` (an initialized oracle handle of the same problem).
// What the reference prints goes to ref_dh_log().
int ref_dh_solve(void* h, void* oracle, const double* velocity, double* grid, int k, int m, double relTol) {
    return Guard([&] {
        DH& H = *static_cast<DH*>(h);
        FormRows(H, velocity);
        // Initialize allocates one front tree per full inner panel; the
        // panel solver tells panels apart by these objects.
        std::map<const void*, int> panelOf;
        if ((int)H.fullInnerFacts_.size() != H.numFullInnerPanels_) {
            H.fullInnerFacts_.clear();
            for (int j = 0; j < H.numFullInnerPanels_; ++j)
                H.fullInnerFacts_.push_back(new cliq::DistSymmFrontTree<Cd>);
        }
        for (int i = H.numPanels_ - 1; i >= 0; --i) panelOf[&H.PanelFactorization(i)] = i;
        cliq::InstalledPanelSolver() = [&](const void* fact, cliq::DistNodalMultiVec<Cd>& X) {
            OraclePanelSolve(H, oracle, panelOf.at(fact), X);
        };
        const int nx = H.disc_.nx, ny = H.disc_.ny, nz = H.disc_.nz;
        psp::DistUniformGrid<Cd> B(nx, ny, nz, 0, k);
        const size_t n = (size_t)nx * ny * nz * k;
        std::copy(reinterpret_cast<const Cd*>(grid), reinterpret_cast<const Cd*>(grid) + n, B.Buffer());
        std::ostringstream log;
        std::streambuf* old = std::cout.rdbuf(log.rdbuf());
        try {
            H.Solve(B, m, relTol);
        } catch (...) {
            std::cout.rdbuf(old);
            g_log = log.str();
            cliq::InstalledPanelSolver() = nullptr;
            throw;
        }
        std::cout.rdbuf(old);
        g_log = log.str();
        cliq::InstalledPanelSolver() = nullptr;
        std::copy(B.LockedBuffer(), B.LockedBuffer() + n, reinterpret_cast<Cd*>(grid));
    });
}

const char* ref_dh_log() { return g_log.c_str(); }

// One of the reference's operators on the k right-hand sides in `grid`
// (natural order, interleaved), in place: op 0 Multiply (B := A B,
// solve.hpp:613-679), op 1 Precondition (the sweep, 681-734, around the
// oracle's panel solves), op 2 SolvePanel of panel `panel` alone
// (736-882), each between the reference's own PullRightHandSides and
// PushRightHandSides (58-239); the rows come from `velocity`.
int ref_dh_apply(void* h, void* oracle, const double* velocity, double* grid, int k, int op, int panel) {
    return Guard([&] {
        DH& H = *static_cast<DH*>(h);
        FormRows(H, velocity);
        std::map<const void*, int> panelOf;
        if ((int)H.fullInnerFacts_.size() != H.numFullInnerPanels_) {
            H.fullInnerFacts_.clear();
            for (int j = 0; j < H.numFullInnerPanels_; ++j)
                H.fullInnerFacts_.push_back(new cliq::DistSymmFrontTree<Cd>);
        }
        for (int i = H.numPanels_ - 1; i >= 0; --i) panelOf[&H.PanelFactorization(i)] = i;
        cliq::InstalledPanelSolver() = [&](const void* fact, cliq::DistNodalMultiVec<Cd>& X) {
            OraclePanelSolve(H, oracle, panelOf.at(fact), X);
        };
        const int nx = H.disc_.nx, ny = H.disc_.ny, nz = H.disc_.nz;
        psp::DistUniformGrid<Cd> G(nx, ny, nz, 0, k);
        const size_t n = (size_t)nx * ny * nz * k;
        std::copy(reinterpret_cast<const Cd*>(grid), reinterpret_cast<const Cd*>(grid) + n, G.Buffer());
        elem::Matrix<Cd> B;
        std::ostringstream log;
        std::streambuf* old = std::cout.rdbuf(log.rdbuf());
        try {
            H.PullRightHandSides(G, B);
            if (op == 0) H.Multiply(B);
            else if (op == 1) H.Precondition(B);
            else H.SolvePanel(B, panel);
            H.PushRightHandSides(G, B);
        } catch (...) {
            std::cout.rdbuf(old);
            cliq::InstalledPanelSolver() = nullptr;
            throw;
        }
        std::cout.rdbuf(old);
        cliq::InstalledPanelSolver() = nullptr;
        std::copy(G.LockedBuffer(), G.LockedBuffer() + n, reinterpret_cast<Cd*>(grid));
    });
}

// Global rows for a natural-order velocity: rowOffsets (N + 1 entries) and
// the complex entries of every row (center, then the -x, +x, -y, +y, -v, +v
// neighbours that exist), as Initialize forms them.  With entries null only
// *nnz is set.
int ref_dh_rows(void* h, const double* velocity, int* nnz, int* rowOffsets, double* entries) {
    return Guard([&] {
        DH& H = *static_cast<DH*>(h);
        *nnz = H.localRowOffsets_.back();
        if (!entries) return;
        FormRows(H, velocity);
        std::copy(H.localRowOffsets_.begin(), H.localRowOffsets_.end(), rowOffsets);
        std::copy(H.localEntries_.begin(), H.localEntries_.end(), reinterpret_cast<std::complex<double>*>(entries));
    });
}

// Node t of panel p's front as the reference's Initialize fills it
// (GetPanelVelocity then FillPanelFronts, initialize_finalize.hpp:123-136,
// 884-1044, 1284-1394): pivot count *s, structure size *u and, with out
// non-null, the (s + u) x s column-major frontal columns as (re, im) pairs.
int ref_dh_panel_front(void* h, const double* velocity, int p, int t, int* s, int* u, double* out) {
    return Guard([&] {
        const DH& H = *static_cast<DH*>(h);
        if (p < 0 || p >= H.numPanels_) throw std::logic_error("no such panel");
        const cliq::DistSymmInfo& info = H.PanelAnalysis(p);
        if (t < 0 || t >= (int)info.localNodes.size()) throw std::logic_error("no such node");
        *s = info.localNodes[t].size;
        *u = (int)info.localNodes[t].lowerStruct.size();
        if (!out) return;
        const int nx = H.disc_.nx, ny = H.disc_.ny, nz = H.disc_.nz;
        psp::DistUniformGrid<double> vel(nx, ny, nz, 0, 1);
        std::copy(velocity, velocity + (size_t)nx * ny * nz, vel.Buffer());
        const int vOffset = H.PanelV(p) - H.PanelPadding(p);
        const int vSize = H.PanelDepth(p) + H.PanelPadding(p);
        std::vector<double> myPanelVelocity;
        std::vector<int> offsets;
        std::map<int, int> nestedToNatural, naturalToNested;
        H.GetPanelVelocity(vOffset, vSize, info, vel, myPanelVelocity, offsets, nestedToNatural, naturalToNested);
        cliq::DistSymmFrontTree<Cd> fact;
        H.FillPanelFronts(vOffset, vSize, info, fact, vel, myPanelVelocity, offsets, nestedToNatural,
                          naturalToNested);
        const elem::Matrix<Cd>& F = fact.localFronts[t].frontL;
        Cd* o = reinterpret_cast<Cd*>(out);
        for (int j = 0; j < F.Width(); ++j)
            for (int i = 0; i < F.Height(); ++i) o[(size_t)j * F.Height() + i] = F.Get(i, j);
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
