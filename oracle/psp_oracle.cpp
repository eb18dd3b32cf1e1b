// ORACLE — test infrastructure only. Nothing in the product links or calls this file.
//
// FP64 CPU restatement of PSP's sweeping-preconditioned Helmholtz solve
// (poulson/PSP, include/psp/dist_helmholtz/*.hpp), used by tests/, by
// __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the checker.
//
// Parity status: the panel factorization in PSP is a call into Clique
// (cliq::LDL / cliq::Solve, source absent from the reference tree, revision not
// recorded).  This file replaces it by the textbook no-pivot complex-symmetric
// multifrontal LDL^T on the same elimination tree; the reference holds no golden
// vectors, so the Clique part is "parity unpinned".  The whole-solve output is
// independently pinned against an FP64 sparse direct solve of the assembled
// global operator (scipy) in tests/test_oracle.py.
//
// Every function cites the reference lines it restates.  One MPI rank is
// assumed (distDepth = 0, teamSize = 1), which is the only configuration the
// single-GPU product replaces.
//
// Vector layouts follow the reference: the solver works on column-major
// N x k matrices in the global nested-dissection ("ND") order; user grids are
// natural x-fastest order with the k right-hand sides interleaved per point
// (DistUniformGrid with one process, dist_uniform_grid.hpp:292-342).

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

typedef std::complex<double> C;

enum { BC_PML = 0, BC_DIRICHLET = 1 };

struct Disc {
    double omega;
    int nx, ny, nz;
    double wx, wy, wz;
    int frontBC, rightBC, backBC, leftBC, topBC;
    int bx, by, bz;
    double sigmax, sigmay, sigmaz;
};

// One node of a panel's elimination tree (main.hpp:1709-1900) plus the
// symbolic fill structure Clique's SymmetricAnalysis would produce.
struct Node {
    int off = 0, size = 0;
    int xOff = 0, yOff = 0, bnx = 0, bny = 0;
    bool leaf = false;
    int parent = -1;
    int children[2] = {-1, -1};
    int numChildren = 0;
    std::vector<int> origLower;  // sorted original (stencil) lower structure
    std::vector<int> lower;      // sorted fill structure
    std::vector<int> relInds;    // position of each lower[] entry in parent's front
};

struct PanelTree {
    int vSize = 0;
    std::vector<Node> nodes;     // postorder: left subtree, right subtree, node
    std::vector<int> ndToNat;    // panel ND index -> x + y*nx + vLocal*nx*ny
};

struct Front {
    int s = 0, u = 0;
    std::vector<C> L;  // (s+u) x s column-major: strict lower of L11, D on diag, L21 below
};

struct Solver {
    Disc disc;
    double damping;
    int P, cutoff;
    double hx, hy, hz;
    int bottomDepth, topOrigDepth, innerDepth, leftoverInnerDepth;
    bool haveLeftover;
    int numFullInnerPanels, numPanels;
    int N;
    // Global operator (initialize_finalize.hpp:340-376) in global ND order.
    std::vector<int> ndToNat, natToNd;
    std::vector<int> rowPtr, cols;  // cols are global ND indices
    std::vector<C> vals;
    // Panel classes: 0 = bottom/full inner, 1 = leftover, 2 = top (main.hpp:705-726)
    PanelTree trees[3];
    std::vector<std::vector<Front>> fronts;  // per panel
    bool initialized = false;
    // HListCopy of the last solve (solve.hpp:257-261, 391-395, 422-426):
    // the unrotated first-cycle Hessenberg matrices, m x m column-major per
    // right-hand side, and the cycle's inner-step count.
    std::vector<C> firstH;
    int firstCount = 0, firstM = 0, firstK = 0;
};

// ---------------------------------------------------------------- geometry

// main.hpp:12-57
void Geometry(Solver& S) {
    const Disc& d = S.disc;
    S.hx = d.wx / (d.nx + 1);
    S.hy = d.wy / (d.ny + 1);
    S.hz = d.wz / (d.nz + 1);
    const bool topHasPML = (d.topBC == BC_PML);
    S.bottomDepth = d.bz + S.P;
    S.topOrigDepth = topHasPML ? d.bz + S.P : S.P;
    if (d.nz <= S.bottomDepth + S.topOrigDepth)
        throw std::logic_error(
            "The domain is very shallow. Please run a sparse-direct factorization instead.");
    S.innerDepth = d.nz - (S.bottomDepth + S.topOrigDepth);
    S.leftoverInnerDepth = S.innerDepth % S.P;
    S.haveLeftover = (S.leftoverInnerDepth != 0);
    S.numFullInnerPanels = S.innerDepth / S.P;
    S.numPanels = 1 + S.numFullInnerPanels + (S.haveLeftover ? 1 : 0) + 1;
    S.N = d.nx * d.ny * d.nz;
}

// main.hpp:728-738
int PanelPadding(const Solver& S, int p) { return p == 0 ? 0 : S.disc.bz; }

// main.hpp:740-752
int PanelDepth(const Solver& S, int p) {
    if (p == 0) return S.bottomDepth;
    if (p < 1 + S.numFullInnerPanels) return S.P;
    if (S.haveLeftover && p == 1 + S.numFullInnerPanels) return S.leftoverInnerDepth;
    return S.topOrigDepth;
}

// main.hpp:779-793
int PanelV(const Solver& S, int p) {
    if (p == 0) return 0;
    if (p < S.numFullInnerPanels + 1) return S.bottomDepth + S.P * (p - 1);
    if (S.haveLeftover && p == S.numFullInnerPanels + 1)
        return S.bottomDepth + S.P * S.numFullInnerPanels;
    return S.bottomDepth + S.P * S.numFullInnerPanels + S.leftoverInnerDepth;
}

// main.hpp:705-726 (which analysis a panel uses)
int PanelClass(const Solver& S, int p) {
    if (p < 1 + S.numFullInnerPanels) return 0;
    if (S.haveLeftover && p == 1 + S.numFullInnerPanels) return 1;
    return 2;
}

// main.hpp:1431-1477 with depthTilSerial = 0 (one rank)
int ReorderedIndexRecursion(int x, int y, int vLocal, int xSize, int ySize, int vSize,
                            int cutoff, int offset) {
    if (xSize * ySize <= cutoff) return offset + (x + y * xSize + vLocal * xSize * ySize);
    if (xSize >= ySize) {
        const int middle = (xSize - 1) / 2;
        if (x < middle)
            return ReorderedIndexRecursion(x, y, vLocal, middle, ySize, vSize, cutoff, offset);
        if (x == middle) return offset + std::max(xSize - 1, 0) * ySize * vSize + (y + vLocal * ySize);
        return ReorderedIndexRecursion(x - middle - 1, y, vLocal, std::max(xSize - middle - 1, 0),
                                       ySize, vSize, cutoff, offset + middle * ySize * vSize);
    } else {
        const int middle = (ySize - 1) / 2;
        if (y < middle)
            return ReorderedIndexRecursion(x, y, vLocal, xSize, middle, vSize, cutoff, offset);
        if (y == middle) return offset + xSize * std::max(ySize - 1, 0) * vSize + (x + vLocal * xSize);
        return ReorderedIndexRecursion(x, y - middle - 1, vLocal, xSize, std::max(ySize - middle - 1, 0),
                                       vSize, cutoff, offset + xSize * middle * vSize);
    }
}

int RI(const Solver& S, int x, int y, int vLocal, int vSize) {
    return ReorderedIndexRecursion(x, y, vLocal, S.disc.nx, S.disc.ny, vSize, S.cutoff, 0);
}

// main.hpp:1709-1900: build the tree in postorder, with the original lower
// structure of every node.
int BuildTree(const Solver& S, PanelTree& T, int xOff, int yOff, int bnx, int bny, int parent) {
    const int nx = S.disc.nx, ny = S.disc.ny, vSize = T.vSize;
    Node node;
    node.xOff = xOff; node.yOff = yOff; node.bnx = bnx; node.bny = bny;
    node.parent = parent;
    if (bnx * bny <= S.cutoff) {
        node.leaf = true;
        node.size = bnx * bny * vSize;
        node.off = RI(S, xOff, yOff, 0, vSize);
        if (xOff > 0)
            for (int i = 0; i < vSize; ++i)
                for (int j = 0; j < bny; ++j) node.origLower.push_back(RI(S, xOff - 1, yOff + j, i, vSize));
        if (xOff + bnx < nx)
            for (int i = 0; i < vSize; ++i)
                for (int j = 0; j < bny; ++j) node.origLower.push_back(RI(S, xOff + bnx, yOff + j, i, vSize));
        if (yOff > 0)
            for (int i = 0; i < vSize; ++i)
                for (int j = 0; j < bnx; ++j) node.origLower.push_back(RI(S, xOff + j, yOff - 1, i, vSize));
        if (yOff + bny < ny)
            for (int i = 0; i < vSize; ++i)
                for (int j = 0; j < bnx; ++j) node.origLower.push_back(RI(S, xOff + j, yOff + bny, i, vSize));
        std::sort(node.origLower.begin(), node.origLower.end());
        T.nodes.push_back(node);
        return (int)T.nodes.size() - 1;
    }
    int left, right;
    if (bnx >= bny) {
        const int middle = (bnx - 1) / 2;
        // children first (postorder); parent index patched below
        left = BuildTree(S, T, xOff, yOff, middle, bny, -2);
        right = BuildTree(S, T, xOff + middle + 1, yOff, std::max(bnx - middle - 1, 0), bny, -2);
        node.size = bny * vSize;
        node.off = RI(S, xOff + middle, yOff, 0, vSize);
        if (yOff > 0)
            for (int i = 0; i < vSize; ++i) node.origLower.push_back(RI(S, xOff + middle, yOff - 1, i, vSize));
        if (yOff + bny < ny)
            for (int i = 0; i < vSize; ++i) node.origLower.push_back(RI(S, xOff + middle, yOff + bny, i, vSize));
    } else {
        const int middle = (bny - 1) / 2;
        left = BuildTree(S, T, xOff, yOff, bnx, middle, -2);
        right = BuildTree(S, T, xOff, yOff + middle + 1, bnx, std::max(bny - middle - 1, 0), -2);
        node.size = bnx * vSize;
        node.off = RI(S, xOff, yOff + middle, 0, vSize);
        if (xOff > 0)
            for (int i = 0; i < vSize; ++i) node.origLower.push_back(RI(S, xOff - 1, yOff + middle, i, vSize));
        if (xOff + bnx < nx)
            for (int i = 0; i < vSize; ++i) node.origLower.push_back(RI(S, xOff + bnx, yOff + middle, i, vSize));
    }
    std::sort(node.origLower.begin(), node.origLower.end());
    node.children[0] = left;
    node.children[1] = right;
    node.numChildren = 2;
    T.nodes.push_back(node);
    const int me = (int)T.nodes.size() - 1;
    T.nodes[left].parent = me;
    T.nodes[right].parent = me;
    return me;
}

// The fill structure a symmetric analysis yields (what cliq::SymmetricAnalysis
// computes at main.hpp:432-435): lower(node) = (origLower U children's lower)
// restricted to indices past the node; plus the relative indices of each child
// structure inside the parent's front.
void SymbolicAnalysis(PanelTree& T) {
    for (size_t t = 0; t < T.nodes.size(); ++t) {
        Node& n = T.nodes[t];
        std::vector<int> all = n.origLower;
        for (int c = 0; c < n.numChildren; ++c) {
            const Node& ch = T.nodes[n.children[c]];
            all.insert(all.end(), ch.lower.begin(), ch.lower.end());
        }
        std::sort(all.begin(), all.end());
        all.erase(std::unique(all.begin(), all.end()), all.end());
        n.lower.clear();
        for (int idx : all)
            if (idx >= n.off + n.size) n.lower.push_back(idx);
        for (int c = 0; c < n.numChildren; ++c) {
            Node& ch = T.nodes[n.children[c]];
            ch.relInds.resize(ch.lower.size());
            for (size_t a = 0; a < ch.lower.size(); ++a) {
                const int idx = ch.lower[a];
                if (idx < n.off + n.size)
                    ch.relInds[a] = idx - n.off;
                else
                    ch.relInds[a] = n.size + int(std::lower_bound(n.lower.begin(), n.lower.end(), idx) -
                                                 n.lower.begin());
            }
        }
    }
}

// initialize_finalize.hpp:1173-1282 (LocalReorderingRecursion, one rank):
// panel ND index -> panel-natural index.
void LocalReorderingRecursion(std::vector<int>& reordering, int offset, int xOffset, int yOffset,
                              int xSize, int ySize, int vSize, int nx, int ny, int cutoff) {
    if (xSize * ySize <= cutoff) {
        for (int v = 0; v < vSize; ++v)
            for (int yd = 0; yd < ySize; ++yd)
                for (int xd = 0; xd < xSize; ++xd)
                    reordering[offset++] = (xOffset + xd) + (yOffset + yd) * nx + v * nx * ny;
    } else if (xSize >= ySize) {
        const int xLeftSize = (xSize - 1) / 2;
        const int xRightSize = std::max(xSize - xLeftSize - 1, 0);
        LocalReorderingRecursion(reordering, offset, xOffset, yOffset, xLeftSize, ySize, vSize, nx, ny, cutoff);
        offset += xLeftSize * ySize * vSize;
        LocalReorderingRecursion(reordering, offset, xOffset + xLeftSize + 1, yOffset, xRightSize, ySize,
                                 vSize, nx, ny, cutoff);
        offset += xRightSize * ySize * vSize;
        const int x = xOffset + xLeftSize;
        for (int v = 0; v < vSize; ++v)
            for (int yd = 0; yd < ySize; ++yd) reordering[offset++] = x + (yOffset + yd) * nx + v * nx * ny;
    } else {
        const int yLeftSize = (ySize - 1) / 2;
        const int yRightSize = std::max(ySize - yLeftSize - 1, 0);
        LocalReorderingRecursion(reordering, offset, xOffset, yOffset, xSize, yLeftSize, vSize, nx, ny, cutoff);
        offset += xSize * yLeftSize * vSize;
        LocalReorderingRecursion(reordering, offset, xOffset, yOffset + yLeftSize + 1, xSize, yRightSize,
                                 vSize, nx, ny, cutoff);
        offset += xSize * yRightSize * vSize;
        const int y = yOffset + yLeftSize;
        for (int v = 0; v < vSize; ++v)
            for (int xd = 0; xd < xSize; ++xd) reordering[offset++] = (xOffset + xd) + y * nx + v * nx * ny;
    }
}

void BuildPanelTree(const Solver& S, PanelTree& T, int vSize) {
    T.vSize = vSize;
    T.nodes.clear();
    BuildTree(S, T, 0, 0, S.disc.nx, S.disc.ny, -1);
    T.nodes.back().parent = -1;
    SymbolicAnalysis(T);
    T.ndToNat.assign((size_t)S.disc.nx * S.disc.ny * vSize, 0);
    LocalReorderingRecursion(T.ndToNat, 0, 0, 0, S.disc.nx, S.disc.ny, vSize, S.disc.nx, S.disc.ny, S.cutoff);
}

// ---------------------------------------------------------------- PML

// initialize_finalize.hpp:415-441
C s1Inv(const Solver& S, int x) {
    const Disc& d = S.disc;
    const double etax = d.bx * S.hx;
    if (x < (d.bx - 1) && d.frontBC == BC_PML) {
        const double delta = (d.bx - 1) - x;
        return C(1, (d.sigmax / etax) * (delta / d.bx) * (delta / d.bx) * (2 * M_PI / d.omega));
    } else if (x > (d.nx - d.bx) && d.backBC == BC_PML) {
        const double delta = x - (d.nx - d.bx);
        return C(1, (d.sigmax / etax) * (delta / d.bx) * (delta / d.bx) * (2 * M_PI / d.omega));
    }
    return C(1, 0);
}

// initialize_finalize.hpp:443-469
C s2Inv(const Solver& S, int y) {
    const Disc& d = S.disc;
    const double etay = d.by * S.hy;
    if (y < (d.by - 1) && d.leftBC == BC_PML) {
        const double delta = (d.by - 1) - y;
        return C(1, (d.sigmay / etay) * (delta / d.by) * (delta / d.by) * (2 * M_PI / d.omega));
    } else if (y > (d.ny - d.by) && d.rightBC == BC_PML) {
        const double delta = y - (d.ny - d.by);
        return C(1, (d.sigmay / etay) * (delta / d.by) * (delta / d.by) * (2 * M_PI / d.omega));
    }
    return C(1, 0);
}

// initialize_finalize.hpp:471-497
C s3Inv(const Solver& S, int v) {
    const Disc& d = S.disc;
    const double etaz = d.bz * S.hz;
    if (v < d.bz - 1) {
        const double delta = (d.bz - 1) - v;
        return C(1, (d.sigmaz / etaz) * (delta / d.bz) * (delta / d.bz) * (2 * M_PI / d.omega));
    } else if (v > (d.nz - d.bz) && d.topBC == BC_PML) {
        const double delta = v - (d.nz - d.bz);
        return C(1, (d.sigmaz / etaz) * (delta / d.bz) * (delta / d.bz) * (2 * M_PI / d.omega));
    }
    return C(1, 0);
}

// initialize_finalize.hpp:499-525
C s3InvArtificial(const Solver& S, int v, int vOffset) {
    const Disc& d = S.disc;
    const double etaz = d.bz * S.hz;
    if (v < vOffset + d.bz - 1) {
        const double delta = (vOffset + d.bz - 1) - v;
        return C(1, (d.sigmaz / etaz) * (delta / d.bz) * (delta / d.bz) * (2 * M_PI / d.omega));
    } else if (v > (d.nz - d.bz) && d.topBC == BC_PML) {
        const double delta = v - (d.nz - d.bz);
        return C(1, (d.sigmaz / etaz) * (delta / d.bz) * (delta / d.bz) * (2 * M_PI / d.omega));
    }
    return C(1, 0);
}

struct Stencil { C center, xL, xR, yL, yR, vL, vR; };

// Shared arithmetic of FormGlobalRow (initialize_finalize.hpp:527-587) and
// FormLowerColumnOfNode (589-651): the six face terms and the centre term.
Stencil StencilTerms(const Solver& S, double alpha, int x, int y, C s3L, C s3M, C s3R, C omegaC) {
    const C s1InvL = s1Inv(S, x - 1), s1InvM = s1Inv(S, x), s1InvR = s1Inv(S, x + 1);
    const C s2InvL = s2Inv(S, y - 1), s2InvM = s2Inv(S, y), s2InvR = s2Inv(S, y + 1);
    const double hx = S.hx, hy = S.hy, hz = S.hz;
    const C xTop = s2InvM * s3M;
    const C xTermL = (xTop / s1InvL + xTop / s1InvM) / (2 * hx * hx);
    const C xTermR = (xTop / s1InvR + xTop / s1InvM) / (2 * hx * hx);
    const C yTop = s1InvM * s3M;
    const C yTermL = (yTop / s2InvL + yTop / s2InvM) / (2 * hy * hy);
    const C yTermR = (yTop / s2InvR + yTop / s2InvM) / (2 * hy * hy);
    const C zTop = s1InvM * s2InvM;
    const C vTermL = (zTop / s3L + zTop / s3M) / (2 * hz * hz);
    const C vTermR = (zTop / s3R + zTop / s3M) / (2 * hz * hz);
    Stencil st;
    st.center = (xTermL + xTermR + yTermL + yTermR + vTermL + vTermR) -
                (omegaC / alpha) * (omegaC / alpha) * s1InvM * s2InvM * s3M;
    st.xL = xTermL; st.xR = xTermR; st.yL = yTermL; st.yR = yTermR; st.vL = vTermL; st.vR = vTermR;
    return st;
}

inline double Velocity(const Solver& S, const double* vel, int x, int y, int v) {
    const int z = (S.disc.nz - 1) - v;
    return vel[x + y * S.disc.nx + (size_t)z * S.disc.nx * S.disc.ny];
}

// ---------------------------------------------------------------- global operator

// Global ND ordering: panel p occupies [nx*ny*PanelV(p), nx*ny*(PanelV(p)+depth)),
// ordered by ReorderedIndex(x,y,vLocal,depth) (main.hpp:1406-1427, 823-1059).
void BuildGlobalOrdering(Solver& S) {
    const int nx = S.disc.nx, ny = S.disc.ny, nz = S.disc.nz;
    S.ndToNat.assign(S.N, 0);
    S.natToNd.assign(S.N, 0);
    for (int p = 0; p < S.numPanels; ++p) {
        const int depth = PanelDepth(S, p), vPanel = PanelV(S, p);
        std::vector<int> reord((size_t)nx * ny * depth);
        LocalReorderingRecursion(reord, 0, 0, 0, nx, ny, depth, nx, ny, S.cutoff);
        const int base = nx * ny * vPanel;
        for (size_t i = 0; i < reord.size(); ++i) {
            const int pn = reord[i];
            const int x = pn % nx, y = (pn / nx) % ny, vLocal = pn / (nx * ny);
            const int v = vPanel + vLocal;
            const int z = (nz - 1) - v;
            const int nat = x + y * nx + z * nx * ny;
            S.ndToNat[base + i] = nat;
            S.natToNd[nat] = base + (int)i;
        }
    }
}

// MapLocalPanelIndices/MapLocalConnectionIndices (main.hpp:823-1273) and
// FormGlobalRow (initialize_finalize.hpp:527-587, 340-376).
void FormGlobalOperator(Solver& S, const double* vel) {
    const int nx = S.disc.nx, ny = S.disc.ny, nz = S.disc.nz;
    S.rowPtr.assign(S.N + 1, 0);
    for (int i = 0; i < S.N; ++i) {
        const int nat = S.ndToNat[i];
        const int x = nat % nx, y = (nat / nx) % ny, z = nat / (nx * ny), v = (nz - 1) - z;
        int c = 1 + (x > 0) + (x + 1 < nx) + (y > 0) + (y + 1 < ny) + (v > 0) + (v + 1 < nz);
        S.rowPtr[i + 1] = S.rowPtr[i] + c;
    }
    S.cols.assign(S.rowPtr.back(), 0);
    S.vals.assign(S.rowPtr.back(), C(0));
#pragma omp parallel for schedule(static)
    for (int i = 0; i < S.N; ++i) {
        const int nat = S.ndToNat[i];
        const int x = nat % nx, y = (nat / nx) % ny, z = nat / (nx * ny), v = (nz - 1) - z;
        const double alpha = vel[nat];
        const Stencil st = StencilTerms(S, alpha, x, y, s3Inv(S, v - 1), s3Inv(S, v), s3Inv(S, v + 1),
                                        C(S.disc.omega, 0));
        int o = S.rowPtr[i];
        S.cols[o] = i; S.vals[o++] = st.center;
        if (x > 0) { S.cols[o] = S.natToNd[nat - 1]; S.vals[o++] = -st.xL; }
        if (x + 1 < nx) { S.cols[o] = S.natToNd[nat + 1]; S.vals[o++] = -st.xR; }
        if (y > 0) { S.cols[o] = S.natToNd[nat - nx]; S.vals[o++] = -st.yL; }
        if (y + 1 < ny) { S.cols[o] = S.natToNd[nat + nx]; S.vals[o++] = -st.yR; }
        if (v > 0) { S.cols[o] = S.natToNd[nat + nx * ny]; S.vals[o++] = -st.vL; }
        if (v + 1 < nz) { S.cols[o] = S.natToNd[nat - nx * ny]; S.vals[o++] = -st.vR; }
    }
}

// ---------------------------------------------------------------- panel fronts

// Dense partial LDL^T (no pivoting, transpose not conjugate: isHermitian=false,
// initialize_finalize.hpp:1299) of an n x n front, eliminating its first s
// columns; the trailing (n-s) x (n-s) block becomes the Schur complement.  F is
// column-major, only the lower triangle is referenced.  Textbook blocked
// right-looking elimination standing in for cliq::LDL.
void PartialLDL(C* F, int n, int s) {
    const int nb = 48;
    std::vector<C> w(n);
    for (int j0 = 0; j0 < s; j0 += nb) {
        const int jb = std::min(nb, s - j0);
        for (int j = j0; j < j0 + jb; ++j) {
            C* colj = F + (size_t)j * n;
            const C d = colj[j];
            if (d == C(0)) throw std::runtime_error("zero pivot in panel factorization");
            const C dinv = C(1) / d;
            for (int i = j + 1; i < n; ++i) { w[i] = colj[i]; colj[i] *= dinv; }
            for (int k = j + 1; k < j0 + jb; ++k) {
                const C coef = w[k];
                C* colk = F + (size_t)k * n;
                for (int i = k; i < n; ++i) colk[i] -= colj[i] * coef;
            }
        }
        const int kStart = j0 + jb;
        // Threads over trailing columns when not already inside a parallel
        // region (the full factorization parallelises over panels instead).
#pragma omp parallel for schedule(dynamic, 8) if (!omp_in_parallel() && (n - kStart) > 64)
        for (int k = kStart; k < n; ++k) {
            C* colk = F + (size_t)k * n;
            for (int j = j0; j < j0 + jb; ++j) {
                const C* colj = F + (size_t)j * n;
                const C coef = colj[j] * colj[k];  // d_j * L(k,j)
                for (int i = k; i < n; ++i) colk[i] -= colj[i] * coef;
            }
        }
    }
}

// FillPanelFronts (initialize_finalize.hpp:1284-1394) with
// The first s columns of node t's front of panel p as FillPanelFronts
// forms them (initialize_finalize.hpp:1284-1340 with FormLowerColumnOfNode,
// 589-806): the padded panel's operator with the damped frequency and the
// artificial PML, on and below the diagonal; column j at F + j ld.
void AssembleFront(const Solver& S, int p, size_t t, const double* vel, C* F, int ld) {
    const int nx = S.disc.nx, ny = S.disc.ny;
    const PanelTree& T = S.trees[PanelClass(S, p)];
    const int vSize = T.vSize;
    const int vOffset = PanelV(S, p) - PanelPadding(S, p);
    const C shiftedOmega(S.disc.omega, S.damping);
    const Node& node = T.nodes[t];
    const int s = node.size;
    {
        const int n = ld;
        for (int j = 0; j < s; ++j) {
            const int pn = T.ndToNat[node.off + j];
            const int x = pn % nx, y = (pn / nx) % ny, vLocal = pn / (nx * ny);
            const int v = vOffset + vLocal;
            const double alpha = Velocity(S, vel, x, y, v);
            const Stencil st = StencilTerms(S, alpha, x, y, s3InvArtificial(S, v - 1, vOffset),
                                            s3InvArtificial(S, v, vOffset), s3InvArtificial(S, v + 1, vOffset),
                                            shiftedOmega);
            C* col = F + (size_t)j * n;
            col[j] = st.center;
            auto put = [&](int xx, int yy, int vl, C val) {
                const int nested = RI(S, xx, yy, vl, vSize);
                if (nested <= node.off + j) return;
                int row;
                if (nested < node.off + s)
                    row = nested - node.off;
                else
                    row = s + int(std::lower_bound(node.lower.begin(), node.lower.end(), nested) -
                                  node.lower.begin());
                col[row] = val;
            };
            if (x > 0) put(x - 1, y, vLocal, -st.xL);
            if (x + 1 < nx) put(x + 1, y, vLocal, -st.xR);
            if (y > 0) put(x, y - 1, vLocal, -st.yL);
            if (y + 1 < ny) put(x, y + 1, vLocal, -st.yR);
            if (vLocal > 0) put(x, y, vLocal - 1, -st.vL);
            if (vLocal + 1 < vSize) put(x, y, vLocal + 1, -st.vR);
        }
    }
}

// FillPanelFronts (above), then the multifrontal factorization that
// cliq::LDL performs (initialize_finalize.hpp:145-150).
void FactorPanel(Solver& S, int p, const double* vel) {
    const PanelTree& T = S.trees[PanelClass(S, p)];
    std::vector<Front>& fr = S.fronts[p];
    fr.assign(T.nodes.size(), Front());
    std::vector<std::vector<C>> updates(T.nodes.size());
    for (size_t t = 0; t < T.nodes.size(); ++t) {
        const Node& node = T.nodes[t];
        const int s = node.size, u = (int)node.lower.size(), n = s + u;
        std::vector<C> F((size_t)n * n, C(0));
        AssembleFront(S, p, t, vel, F.data(), n);
        // extend-add of the children's Schur complements
        for (int c = 0; c < node.numChildren; ++c) {
            const int ch = node.children[c];
            const Node& cn = T.nodes[ch];
            const int uc = (int)cn.lower.size();
            const std::vector<C>& U = updates[ch];
            for (int b = 0; b < uc; ++b) {
                const int rb = cn.relInds[b];
                for (int a = b; a < uc; ++a) F[(size_t)rb * n + cn.relInds[a]] += U[(size_t)b * uc + a];
            }
            std::vector<C>().swap(updates[ch]);
        }
        PartialLDL(F.data(), n, s);
        Front& f = fr[t];
        f.s = s; f.u = u;
        f.L.assign(F.begin(), F.begin() + (size_t)n * s);
        if (u > 0) {
            std::vector<C>& U = updates[t];
            U.assign((size_t)u * u, C(0));
            for (int b = 0; b < u; ++b)
                for (int a = b; a < u; ++a) U[(size_t)b * u + a] = F[(size_t)(s + b) * n + (s + a)];
        }
    }
}

// cliq::Solve (solve.hpp:822) on one RHS column of a panel-subproblem vector
// xp (ND order of the padded panel): forward with L, D^{-1}, backward with L^T.
void SolvePanelColumn(const Solver& S, int p, C* xp) {
    const PanelTree& T = S.trees[PanelClass(S, p)];
    const std::vector<Front>& fr = S.fronts[p];
    const size_t numNodes = T.nodes.size();
    std::vector<std::vector<C>> upd(numNodes);
    std::vector<C> r;
    for (size_t t = 0; t < numNodes; ++t) {
        const Node& node = T.nodes[t];
        const Front& f = fr[t];
        const int s = f.s, u = f.u, n = s + u;
        r.assign(n, C(0));
        for (int i = 0; i < s; ++i) r[i] = xp[node.off + i];
        for (int c = 0; c < node.numChildren; ++c) {
            const int ch = node.children[c];
            const Node& cn = T.nodes[ch];
            for (size_t a = 0; a < cn.lower.size(); ++a) r[cn.relInds[a]] += upd[ch][a];
            std::vector<C>().swap(upd[ch]);
        }
        for (int j = 0; j < s; ++j) {
            const C* col = f.L.data() + (size_t)j * n;
            const C rj = r[j];
            for (int i = j + 1; i < n; ++i) r[i] -= col[i] * rj;
        }
        for (int i = 0; i < s; ++i) xp[node.off + i] = r[i];
        upd[t].assign(r.begin() + s, r.end());
    }
    for (size_t t = 0; t < numNodes; ++t) {
        const Node& node = T.nodes[t];
        const Front& f = fr[t];
        const int n = f.s + f.u;
        for (int j = 0; j < f.s; ++j) xp[node.off + j] /= f.L[(size_t)j * n + j];
    }
    for (size_t tt = numNodes; tt-- > 0;) {
        const Node& node = T.nodes[tt];
        const Front& f = fr[tt];
        const int s = f.s, u = f.u, n = s + u;
        r.assign(n, C(0));
        for (int i = 0; i < s; ++i) r[i] = xp[node.off + i];
        for (int a = 0; a < u; ++a) r[s + a] = xp[node.lower[a]];
        for (int j = s - 1; j >= 0; --j) {
            const C* col = f.L.data() + (size_t)j * n;
            C acc = r[j];
            for (int i = j + 1; i < n; ++i) acc -= col[i] * r[i];
            r[j] = acc;
        }
        for (int i = 0; i < s; ++i) xp[node.off + i] = r[i];
    }
}

// SolvePanel (solve.hpp:736-882): B_i := T_i B_i on the global ND matrix B
// (column-major, N x k).  Padding rows (first xySize*padding of every node)
// enter as zero and are dropped.
void SolvePanel(const Solver& S, C* B, int k, int p) {
    const PanelTree& T = S.trees[PanelClass(S, p)];
    const int padding = PanelPadding(S, p), depth = PanelDepth(S, p);
    const size_t nSub = T.ndToNat.size();
    const int panelOff = S.disc.nx * S.disc.ny * PanelV(S, p);
#pragma omp parallel for schedule(dynamic, 1)
    for (int r = 0; r < k; ++r) {
        std::vector<C> xp(nSub, C(0));
        C* Bcol = B + (size_t)r * S.N;
        int bOff = panelOff;
        for (const Node& node : T.nodes) {
            const int xySize = node.size / (padding + depth);
            const int pad = xySize * padding, rem = node.size - pad;
            for (int i = 0; i < rem; ++i) xp[node.off + pad + i] = Bcol[bOff + i];
            bOff += rem;
        }
        SolvePanelColumn(S, p, xp.data());
        bOff = panelOff;
        for (const Node& node : T.nodes) {
            const int xySize = node.size / (padding + depth);
            const int pad = xySize * padding, rem = node.size - pad;
            for (int i = 0; i < rem; ++i) Bcol[bOff + i] = xp[node.off + pad + i];
            bOff += rem;
        }
    }
}

// Value of the global-operator entry (row, col) (localEntries_ lookup as in
// main.hpp:318-328 / 350-362).
C Entry(const Solver& S, int row, int col) {
    for (int o = S.rowPtr[row]; o < S.rowPtr[row + 1]; ++o)
        if (S.cols[o] == col) return S.vals[o];
    throw std::logic_error("did not find panel connection");
}

// SubdiagonalUpdate (solve.hpp:884-948): B_{i+1} -= A_{i+1,i} B_i, through
// the z-couplings of the first plane of panel i+1.
void SubdiagonalUpdate(const Solver& S, C* B, int k, int i) {
    const int nx = S.disc.nx, ny = S.disc.ny, nz = S.disc.nz;
    const int v = PanelV(S, i + 1);
    const int z = (nz - 1) - v;
#pragma omp parallel for schedule(static)
    for (int xy = 0; xy < nx * ny; ++xy) {
        const int row = S.natToNd[xy + z * nx * ny];
        const int col = S.natToNd[xy + (z + 1) * nx * ny];
        const C a = Entry(S, row, col);
        for (int r = 0; r < k; ++r) B[row + (size_t)r * S.N] -= a * B[col + (size_t)r * S.N];
    }
}

// ExtractPanel + MultiplySuperdiagonal (solve.hpp:950-1047): Z := B_i,
// B_i := -A_{i,i+1} B_{i+1}.
void ExtractAndMultiplySuperdiagonal(const Solver& S, C* B, int k, int i, std::vector<C>& Z) {
    const int nx = S.disc.nx, ny = S.disc.ny, nz = S.disc.nz;
    const int off = nx * ny * PanelV(S, i), size = nx * ny * PanelDepth(S, i);
    Z.resize((size_t)size * k);
    for (int r = 0; r < k; ++r) {
        std::memcpy(&Z[(size_t)r * size], B + off + (size_t)r * S.N, sizeof(C) * size);
        std::fill(B + off + (size_t)r * S.N, B + off + size + (size_t)r * S.N, C(0));
    }
    const int v = PanelV(S, i) + PanelDepth(S, i) - 1;
    const int z = (nz - 1) - v;
#pragma omp parallel for schedule(static)
    for (int xy = 0; xy < nx * ny; ++xy) {
        const int row = S.natToNd[xy + z * nx * ny];
        const int col = S.natToNd[xy + (z - 1) * nx * ny];
        const C a = Entry(S, row, col);
        for (int r = 0; r < k; ++r) B[row + (size_t)r * S.N] = -a * B[col + (size_t)r * S.N];
    }
}

// UpdatePanel (solve.hpp:1049-1061): B_i += Z.
void UpdatePanel(const Solver& S, C* B, int k, int i, const std::vector<C>& Z) {
    const int off = S.disc.nx * S.disc.ny * PanelV(S, i), size = S.disc.nx * S.disc.ny * PanelDepth(S, i);
    for (int r = 0; r < k; ++r)
        for (int s = 0; s < size; ++s) B[off + s + (size_t)r * S.N] += Z[(size_t)r * size + s];
}

// Precondition (solve.hpp:681-734).
void Precondition(const Solver& S, C* B, int k) {
    for (int i = 0; i < S.numPanels - 1; ++i) {
        SolvePanel(S, B, k, i);
        SubdiagonalUpdate(S, B, k, i);
    }
    SolvePanel(S, B, k, S.numPanels - 1);
    std::vector<C> Z;
    for (int i = S.numPanels - 2; i >= 0; --i) {
        ExtractAndMultiplySuperdiagonal(S, B, k, i, Z);
        SolvePanel(S, B, k, i);
        UpdatePanel(S, B, k, i, Z);
    }
}

// Multiply (solve.hpp:613-679): B := A B.
void Multiply(const Solver& S, C* B, int k) {
    std::vector<C> X(B, B + (size_t)S.N * k);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < S.N; ++i) {
        for (int r = 0; r < k; ++r) {
            const C* x = X.data() + (size_t)r * S.N;
            C acc = S.vals[S.rowPtr[i]] * x[i];
            for (int o = S.rowPtr[i] + 1; o < S.rowPtr[i + 1]; ++o) acc += S.vals[o] * x[S.cols[o]];
            B[i + (size_t)r * S.N] = acc;
        }
    }
}

// ---------------------------------------------------------------- GMRES helpers

// Norms / InnerProducts / DivideColumns / SubtractScaledColumns
// (environment.hpp:177-257); blas::Dot is the conjugated dot v^H w.
void Norms(const C* X, int n, int k, double* out) {
    for (int r = 0; r < k; ++r) {
        double acc = 0;
        const C* x = X + (size_t)r * n;
#pragma omp parallel for reduction(+ : acc) schedule(static)
        for (int i = 0; i < n; ++i) acc += std::norm(x[i]);
        out[r] = std::sqrt(acc);
    }
}

void InnerProducts(const C* V, const C* W, int n, int k, C* out) {
    for (int r = 0; r < k; ++r) {
        double re = 0, im = 0;
        const C* v = V + (size_t)r * n;
        const C* w = W + (size_t)r * n;
#pragma omp parallel for reduction(+ : re, im) schedule(static)
        for (int i = 0; i < n; ++i) {
            const C t = std::conj(v[i]) * w[i];
            re += t.real(); im += t.imag();
        }
        out[r] = C(re, im);
    }
}

// lapack::ComputeGivens (solve.hpp:486-487): [c s; -conj(s) c] [f; g] = [rho; 0].
void ComputeGivens(C f, C g, double* c, C* s, C* rho) {
    const double af = std::abs(f), ag = std::abs(g);
    if (ag == 0) { *c = 1; *s = 0; *rho = f; return; }
    if (af == 0) { *c = 0; *s = std::conj(g) / ag; *rho = ag; return; }
    const double nrm = std::hypot(af, ag);
    *c = af / nrm;
    *s = (f / af) * std::conj(g) / nrm;
    *rho = (f / af) * nrm;
}

}  // namespace

// ---------------------------------------------------------------- C interface

extern "C" {

struct oracle_disc {
    double omega;
    int nx, ny, nz;
    double wx, wy, wz;
    int frontBC, rightBC, backBC, leftBC, topBC;
    int bx, by, bz;
    double sigmax, sigmay, sigmaz;
};

struct oracle_stats {
    int iterations;
    int converged;
    int lucky_breakdown;
    double final_max_rel_resid;
    double setup_seconds;
    double solve_seconds;
};

static std::string g_err;
const char* oracle_last_error() { return g_err.c_str(); }

int oracle_create(const oracle_disc* d, double damping, int planesPerPanel, int cutoff, void** out) {
    try {
        Solver* S = new Solver;
        std::memcpy(&S->disc, d, sizeof(Disc));
        S->damping = damping;
        S->P = planesPerPanel;
        S->cutoff = cutoff;
        Geometry(*S);
        BuildGlobalOrdering(*S);
        BuildPanelTree(*S, S->trees[0], S->bottomDepth);
        if (S->haveLeftover) BuildPanelTree(*S, S->trees[1], S->leftoverInnerDepth + d->bz);
        BuildPanelTree(*S, S->trees[2], S->topOrigDepth + d->bz);
        *out = S;
        return 0;
    } catch (std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

void oracle_destroy(void* h) { delete (Solver*)h; }

// Geometry summary: numPanels, then per panel (vLow, depth, padding, class).
// PML stretch `which` (1 s1Inv, 2 s2Inv, 3 s3Inv, 4 s3InvArtificial with
// vOffset) at n indices, as (re, im) pairs.
int oracle_stretch(void* h, int which, int n, const int* idx, int vOffset, double* out) {
    const Solver& S = *(const Solver*)h;
    for (int i = 0; i < n; ++i) {
        const C c = which == 1 ? s1Inv(S, idx[i])
                  : which == 2 ? s2Inv(S, idx[i])
                  : which == 3 ? s3Inv(S, idx[i])
                               : s3InvArtificial(S, idx[i], vOffset);
        out[2 * i] = c.real();
        out[2 * i + 1] = c.imag();
    }
    return 0;
}

// Node t of panel p: its pivot count *s and structure size *u, and (out
// non-null) the first s columns of its front, (s + u) x s column-major as
// (re, im) pairs, as assembled from `velocity` before any update is added.
int oracle_panel_front(void* h, const double* velocity, int p, int t, int* s, int* u, double* out) {
    const Solver& S = *(const Solver*)h;
    if (p < 0 || p >= S.numPanels) return 1;
    const PanelTree& T = S.trees[PanelClass(S, p)];
    if (t < 0 || t >= (int)T.nodes.size()) return 1;
    const Node& node = T.nodes[t];
    *s = node.size;
    *u = (int)node.lower.size();
    if (out) {
        const int n = *s + *u;
        std::vector<C> F((size_t)n * n, C(0));
        AssembleFront(S, p, (size_t)t, velocity, F.data(), n);
        std::memcpy(out, F.data(), sizeof(C) * (size_t)n * *s);
    }
    return 0;
}

int oracle_geometry(void* h, int* numPanels, int* panelInfo) {
    Solver& S = *(Solver*)h;
    *numPanels = S.numPanels;
    if (panelInfo)
        for (int p = 0; p < S.numPanels; ++p) {
            panelInfo[4 * p + 0] = PanelV(S, p);
            panelInfo[4 * p + 1] = PanelDepth(S, p);
            panelInfo[4 * p + 2] = PanelPadding(S, p);
            panelInfo[4 * p + 3] = PanelClass(S, p);
        }
    return 0;
}

// Global ND order -> natural index map (length N).
int oracle_nd_to_natural(void* h, int* out) {
    Solver& S = *(Solver*)h;
    std::memcpy(out, S.ndToNat.data(), sizeof(int) * S.N);
    return 0;
}

// Tree summary of panel class c: number of nodes, then per node
// (off, size, lowerSize, parent).
int oracle_tree(void* h, int c, int* numNodes, int* info) {
    Solver& S = *(Solver*)h;
    const PanelTree& T = S.trees[c];
    *numNodes = (int)T.nodes.size();
    if (info)
        for (size_t t = 0; t < T.nodes.size(); ++t) {
            info[4 * t + 0] = T.nodes[t].off;
            info[4 * t + 1] = T.nodes[t].size;
            info[4 * t + 2] = (int)T.nodes[t].lower.size();
            info[4 * t + 3] = T.nodes[t].parent;
        }
    return 0;
}

int oracle_initialize(void* h, const double* velocity) {
    Solver& S = *(Solver*)h;
    try {
        if (S.disc.omega == 0) throw std::logic_error("PML does not work at zero frequency");
        FormGlobalOperator(S, velocity);
        S.fronts.assign(S.numPanels, std::vector<Front>());
#pragma omp parallel for schedule(dynamic, 1)
        for (int p = 0; p < S.numPanels; ++p) FactorPanel(S, p, velocity);
        S.initialized = true;
        return 0;
    } catch (std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// Global operator in ND order: nnz, then rowPtr (N+1), cols (nnz), vals (2*nnz doubles).
int oracle_global_operator(void* h, int* nnz, int* rowPtr, int* cols, double* vals) {
    Solver& S = *(Solver*)h;
    *nnz = S.rowPtr.back();
    if (rowPtr) std::memcpy(rowPtr, S.rowPtr.data(), sizeof(int) * (S.N + 1));
    if (cols) std::memcpy(cols, S.cols.data(), sizeof(int) * S.rowPtr.back());
    if (vals) std::memcpy(vals, S.vals.data(), sizeof(C) * S.rowPtr.back());
    return 0;
}

// PullRightHandSides / PushRightHandSides (solve.hpp:58-239) for one process:
// grid is natural order with k interleaved scalars per point.
static void Pull(const Solver& S, const C* grid, int k, std::vector<C>& B) {
    B.resize((size_t)S.N * k);
    for (int i = 0; i < S.N; ++i)
        for (int r = 0; r < k; ++r) B[i + (size_t)r * S.N] = grid[(size_t)S.ndToNat[i] * k + r];
}
static void Push(const Solver& S, C* grid, int k, const std::vector<C>& B) {
    for (int i = 0; i < S.N; ++i)
        for (int r = 0; r < k; ++r) grid[(size_t)S.ndToNat[i] * k + r] = B[i + (size_t)r * S.N];
}

// Forms the global operator only (FormGlobalRow for every row).
int oracle_form_operator(void* h, const double* velocity) {
    Solver& S = *(Solver*)h;
    FormGlobalOperator(S, velocity);
    return 0;
}

// B := A B on a natural-order interleaved grid (complex as 2 doubles).
int oracle_multiply(void* h, double* grid, int k) {
    Solver& S = *(Solver*)h;
    if (S.rowPtr.empty()) { g_err = "global operator not formed"; return 1; }
    std::vector<C> B;
    Pull(S, (C*)grid, k, B);
    Multiply(S, B.data(), k);
    Push(S, (C*)grid, k, B);
    return 0;
}

// B := M^{-1} B (sweeping preconditioner) on a natural-order interleaved grid.
int oracle_precondition(void* h, double* grid, int k) {
    Solver& S = *(Solver*)h;
    if (!S.initialized) { g_err = "not initialized"; return 1; }
    std::vector<C> B;
    Pull(S, (C*)grid, k, B);
    Precondition(S, B.data(), k);
    Push(S, (C*)grid, k, B);
    return 0;
}

// B := T_p B restricted to panel p (one SolvePanel), natural-order grid.
int oracle_solve_panel(void* h, double* grid, int k, int p) {
    Solver& S = *(Solver*)h;
    std::vector<C> B;
    Pull(S, (C*)grid, k, B);
    SolvePanel(S, B.data(), k, p);
    Push(S, (C*)grid, k, B);
    return 0;
}

// InternalSolveWithGMRES (solve.hpp:241-611) wrapped by Solve (12-56).
// resid_history (may be null) receives the max relative residual of every
// inner step, up to max_history entries.
int oracle_solve(void* h, double* grid, int k, int m, double relTol, int maxIts, oracle_stats* stats,
                 double* resid_history, int max_history) {
    Solver& S = *(Solver*)h;
    try {
        if (!S.initialized) throw std::logic_error("not initialized");
        const int n = S.N;
        std::vector<C> bList;
        Pull(S, (C*)grid, k, bList);
        std::vector<C> V((size_t)n * k * m), x0((size_t)n * k), x((size_t)n * k, C(0)), w(bList);
        std::vector<C> z((size_t)(m + 1) * k), H((size_t)m * m * k);
        std::vector<double> cs((size_t)m * k);
        std::vector<C> sn((size_t)m * k);
        std::vector<C> alpha(k);
        std::vector<double> beta(k), delta(k), origResid(k), resid(k);
        Norms(w.data(), n, k, origResid.data());
        for (double v : origResid)
            if (v != v) throw std::runtime_error("Original residual norms had a NaN");
        int it = 0;
        bool converged = false;
        stats->lucky_breakdown = 0;
        double maxRel = 0;
        bool firstBatch = true;
        S.firstH.assign((size_t)m * m * k, C(0));
        S.firstCount = 0;
        S.firstM = m;
        S.firstK = k;
        while (!converged) {
            x0 = x;
            Precondition(S, w.data(), k);
            Norms(w.data(), n, k, beta.data());
            for (double v : beta)
                if (v != v) throw std::runtime_error("beta list had a NaN");
            for (int r = 0; r < k; ++r)
                for (int i = 0; i < n; ++i) V[(size_t)r * n + i] = w[(size_t)r * n + i] / beta[r];
            std::fill(z.begin(), z.end(), C(0));
            for (int r = 0; r < k; ++r) z[(size_t)r * (m + 1)] = beta[r];
            for (int j = 0; j < m; ++j) {
                std::memcpy(w.data(), &V[(size_t)j * n * k], sizeof(C) * n * k);
                Multiply(S, w.data(), k);
                Precondition(S, w.data(), k);
                for (int i = 0; i <= j; ++i) {
                    const C* vi = &V[(size_t)i * n * k];
                    InnerProducts(vi, w.data(), n, k, alpha.data());
                    for (int r = 0; r < k; ++r) H[(size_t)r * m * m + (size_t)j * m + i] = alpha[r];
                    if (firstBatch)
                        for (int r = 0; r < k; ++r) S.firstH[(size_t)r * m * m + (size_t)j * m + i] = alpha[r];
                    for (int r = 0; r < k; ++r) {
                        const C a = alpha[r];
                        C* wr = w.data() + (size_t)r * n;
                        const C* vr = vi + (size_t)r * n;
#pragma omp parallel for schedule(static)
                        for (int q = 0; q < n; ++q) wr[q] -= a * vr[q];
                    }
                }
                Norms(w.data(), n, k, delta.data());
                for (double v : delta)
                    if (v != v) throw std::runtime_error("delta list had a NaN");
                bool zero = false;
                for (double v : delta)
                    if (v == 0) zero = true;
                if (zero) {
                    // solve.hpp:405-414: returns before bList = xList, so the
                    // grid keeps the right-hand sides.
                    stats->lucky_breakdown = 1;
                    stats->iterations = it;
                    stats->converged = 0;
                    stats->final_max_rel_resid = maxRel;
                    return 0;
                }
                if (j + 1 != m) {
                    for (int r = 0; r < k; ++r)
                        for (int q = 0; q < n; ++q)
                            V[(size_t)(j + 1) * n * k + (size_t)r * n + q] = w[(size_t)r * n + q] / delta[r];
                    if (firstBatch)
                        for (int r = 0; r < k; ++r) S.firstH[(size_t)r * m * m + (size_t)j * m + j + 1] = delta[r];
                }
                for (int r = 0; r < k; ++r) {
                    C* Hr = &H[(size_t)r * m * m];  // column-major m x m, H(i,j) = Hr[j*m+i]
                    for (int i = 0; i < j; ++i) {
                        const double c = cs[(size_t)r * m + i];
                        const C s = sn[(size_t)r * m + i];
                        const C a = Hr[(size_t)j * m + i], b = Hr[(size_t)j * m + i + 1];
                        Hr[(size_t)j * m + i] = c * a + s * b;
                        Hr[(size_t)j * m + i + 1] = -std::conj(s) * a + c * b;
                    }
                }
                for (int r = 0; r < k; ++r) {
                    C* Hr = &H[(size_t)r * m * m];
                    const C etajj = Hr[(size_t)j * m + j];
                    const C etajp1j = delta[r];
                    double c;
                    C s, rho;
                    ComputeGivens(etajj, etajp1j, &c, &s, &rho);
                    if (c != c || s != s || rho != rho) throw std::runtime_error("Givens was NaN");
                    Hr[(size_t)j * m + j] = rho;
                    cs[(size_t)r * m + j] = c;
                    sn[(size_t)r * m + j] = s;
                    C* zr = &z[(size_t)r * (m + 1)];
                    const C zj = zr[j], zj1 = zr[j + 1];
                    zr[j] = c * zj + s * zj1;
                    zr[j + 1] = -std::conj(s) * zj + c * zj1;
                    // y = triu(H)^{-1} z (elem::Trsv, UPPER, NORMAL, NON_UNIT)
                    std::vector<C> y(zr, zr + j + 1);
                    for (int i = j; i >= 0; --i) {
                        C acc = y[i];
                        for (int q = i + 1; q <= j; ++q) acc -= Hr[(size_t)q * m + i] * y[q];
                        y[i] = acc / Hr[(size_t)i * m + i];
                    }
                    C* xr = x.data() + (size_t)r * n;
                    const C* x0r = x0.data() + (size_t)r * n;
#pragma omp parallel for schedule(static)
                    for (int q = 0; q < n; ++q) {
                        C acc = x0r[q];
                        for (int i = 0; i <= j; ++i) acc += y[i] * V[(size_t)i * n * k + (size_t)r * n + q];
                        xr[q] = acc;
                    }
                }
                // w := b - A x
                for (size_t q = 0; q < w.size(); ++q) w[q] = -x[q];
                Multiply(S, w.data(), k);
                for (size_t q = 0; q < w.size(); ++q) w[q] += bList[q];
                Norms(w.data(), n, k, resid.data());
                for (double v : resid)
                    if (v != v) throw std::runtime_error("resid norm list has NaN");
                maxRel = 0;
                for (int r = 0; r < k; ++r) maxRel = std::max(maxRel, resid[r] / origResid[r]);
                if (resid_history && it < max_history) resid_history[it] = maxRel;
                ++it;
                if (firstBatch) S.firstCount = it;
                if (maxRel < relTol) {
                    converged = true;
                    break;
                }
                if (maxIts > 0 && it >= maxIts) {
                    Push(S, (C*)grid, k, x);
                    stats->iterations = it;
                    stats->converged = 0;
                    stats->final_max_rel_resid = maxRel;
                    return 0;
                }
            }
            firstBatch = false;
        }
        Push(S, (C*)grid, k, x);
        stats->iterations = it;
        stats->converged = 1;
        stats->final_max_rel_resid = maxRel;
        return 0;
    } catch (std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// The first-cycle Hessenberg matrices of the last oracle_solve (the
// reference's HListCopy under PRINT_RITZ_VALUES, solve.hpp:589-608): *count
// inner steps, *m and *k; out (may be null) receives k blocks of m x m
// complex column-major values.  The Ritz values are the eigenvalues of the
// leading count x count block of each.
int oracle_first_cycle_hessenberg(void* h, int* count, int* m, int* k, double* out) {
    Solver& S = *(Solver*)h;
    *count = S.firstCount;
    *m = S.firstM;
    *k = S.firstK;
    if (out && !S.firstH.empty()) std::memcpy(out, S.firstH.data(), S.firstH.size() * sizeof(C));
    return 0;
}

// Bounded timing sample of the full-size workload for the CPU baseline:
// out[0] global operator formation, out[1+c] factorization of one panel of
// class c (threads inside the fronts), out[4+c] one SolvePanel of that panel
// with k right-hand sides, out[7] one Multiply with k right-hand sides.
// Classes absent from the geometry report -1.
int oracle_sample(void* h, const double* velocity, int k, int reps, double* out) {
    Solver& S = *(Solver*)h;
    try {
        auto now = [] { return omp_get_wtime(); };
        double t = now();
        FormGlobalOperator(S, velocity);
        out[0] = now() - t;
        S.fronts.assign(S.numPanels, std::vector<Front>());
        int rep[3] = {-1, -1, -1};
        for (int p = S.numPanels - 1; p >= 0; --p) rep[PanelClass(S, p)] = p;
        std::vector<C> B((size_t)S.N * k);
        uint64_t seed = 12345;
        for (auto& v : B) {
            seed = seed * 6364136223846793005ULL + 1442695040888963407ULL;
            const double a = ((seed >> 11) & 0xFFFFF) / double(0xFFFFF) - 0.5;
            const double b = ((seed >> 33) & 0xFFFFF) / double(0xFFFFF) - 0.5;
            v = C(a, b);
        }
        for (int c = 0; c < 3; ++c) {
            out[1 + c] = -1;
            out[4 + c] = -1;
            if (rep[c] < 0) continue;
            t = now();
            FactorPanel(S, rep[c], velocity);
            out[1 + c] = now() - t;
            t = now();
            for (int r = 0; r < reps; ++r) SolvePanel(S, B.data(), k, rep[c]);
            out[4 + c] = (now() - t) / std::max(reps, 1);
            std::vector<Front>().swap(S.fronts[rep[c]]);
        }
        t = now();
        Multiply(S, B.data(), k);
        out[7] = now() - t;
        return 0;
    } catch (std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// Bounded timing pieces for workloads too large for a whole CPU solve.
// Each returns the wall seconds of one piece of Initialize or Solve on the
// handle's own problem (threads as for the full solve).
//
// Factors panel p (FactorPanel, the cliq::LDL stand-in) and keeps its fronts.
int oracle_time_factor_panel(void* h, const double* velocity, int p, double* seconds) {
    Solver& S = *(Solver*)h;
    try {
        if (p < 0 || p >= S.numPanels) throw std::runtime_error("panel index out of range");
        if ((int)S.fronts.size() != S.numPanels) S.fronts.assign(S.numPanels, std::vector<Front>());
        const double t = omp_get_wtime();
        FactorPanel(S, p, velocity);
        *seconds = omp_get_wtime() - t;
        return 0;
    } catch (std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// SolvePanel of panel p (solve.hpp:736-882) on k seeded right-hand sides.
// When panel p holds no factors, fronts of its structure are allocated with
// a unit diagonal and zeros elsewhere: the solve then streams exactly the
// bytes and does exactly the operations it does on real factors (operand
// values do not change the cost of FP64 arithmetic away from denormals),
// without a factorization first.
int oracle_time_panel_solve(void* h, int p, int k, double* seconds) {
    Solver& S = *(Solver*)h;
    try {
        if (p < 0 || p >= S.numPanels) throw std::runtime_error("panel index out of range");
        if ((int)S.fronts.size() != S.numPanels) S.fronts.assign(S.numPanels, std::vector<Front>());
        std::vector<Front>& fr = S.fronts[p];
        if (fr.empty()) {
            const PanelTree& T = S.trees[PanelClass(S, p)];
            fr.assign(T.nodes.size(), Front());
            for (size_t t = 0; t < T.nodes.size(); ++t) {
                Front& f = fr[t];
                f.s = T.nodes[t].size;
                f.u = (int)T.nodes[t].lower.size();
                f.L.assign((size_t)(f.s + f.u) * f.s, C(0));
                for (int j = 0; j < f.s; ++j) f.L[(size_t)j * (f.s + f.u) + j] = C(1);
            }
        }
        std::vector<C> B((size_t)S.N * k);
        uint64_t seed = 2024;
        for (auto& v : B) {
            seed = seed * 6364136223846793005ULL + 1442695040888963407ULL;
            v = C(((seed >> 11) & 0xFFFFF) / double(0xFFFFF) - 0.5, ((seed >> 33) & 0xFFFFF) / double(0xFFFFF) - 0.5);
        }
        const double t = omp_get_wtime();
        SolvePanel(S, B.data(), k, p);
        *seconds = omp_get_wtime() - t;
        return 0;
    } catch (std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// Frees the fronts of panel p.
int oracle_release_panel(void* h, int p) {
    Solver& S = *(Solver*)h;
    if (p >= 0 && p < (int)S.fronts.size()) std::vector<Front>().swap(S.fronts[p]);
    return 0;
}

// Multiply (solve.hpp:613-679) of k seeded right-hand sides; the global
// operator must have been formed (oracle_form_operator).
int oracle_time_multiply(void* h, int k, double* seconds) {
    Solver& S = *(Solver*)h;
    try {
        if (S.vals.empty()) throw std::runtime_error("the global operator has not been formed");
        std::vector<C> B((size_t)S.N * k, C(0.25, -0.5));
        const double t = omp_get_wtime();
        Multiply(S, B.data(), k);
        *seconds = omp_get_wtime() - t;
        return 0;
    } catch (std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

int oracle_num_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
