// Device kernels of the sweeping-preconditioned Helmholtz solve and the
// descriptors the host orchestration fills for them.  Every batched kernel
// walks a task list, so one launch covers all fronts of one elimination-tree
// depth across every panel (and every problem) in flight.
#pragma once
#include <vector>

#include "common.cuh"

namespace psp_b200 {

// ------------------------------------------------------------------ stencil

// 1-D PML tables live on the device with one guard entry on each side:
// table[i+1] holds the value at grid index i, i in [-1, n].
struct StencilParams {
    int nx, ny, nz;
    double ihx2, ihy2, ihz2;  // 1/(2 h^2) per axis
    double omega;
    const z64* s1; const z64* is1;  // s1Inv and its reciprocal (initialize_finalize.hpp:415-441)
    const z64* s2; const z64* is2;  // s2Inv (443-469)
    const z64* s3; const z64* is3;  // s3Inv on the global sweep coordinate v (471-497)
};

// y := A x, or y := b - A x when b != nullptr, for natural-order grids with
// k interleaved right-hand sides (Multiply, solve.hpp:613-679; the operator is
// FormGlobalRow, initialize_finalize.hpp:527-587, evaluated on the fly).
void LaunchHelmholtzApply(const z64* x, z64* y, const z64* b, const double* vel, const StencilParams& sp, int k,
                          cudaStream_t st);
// The same on planes [zFirst, zFirst + zCount) of slabs whose first stored
// plane is zSlab (x must hold the existing planes next to the range).
void LaunchHelmholtzApplyPlanes(const z64* x, z64* y, const z64* b, const double* vel, const StencilParams& sp,
                                int k, int zFirst, int zCount, int zSlab, cudaStream_t st);

// grad[i] (+)= -Re( dA_ii/dvel_i * sum_r Z[i,r] U[i,r] ) for natural-order
// [N][k] grids: the velocity gradient of a real misfit whose forward fields
// are U and whose adjoint fields (A Z = conj of the misfit's field gradient)
// are Z.  dA_ii/dvel_i = 2 omega^2 / vel_i^3 * s1 s2 s3 differentiates the
// centre term of FormGlobalRow (initialize_finalize.hpp:567-568); the
// operator is complex symmetric, so Z reuses the forward factors.
void LaunchVelocityGradient(const z64* U, const z64* Z, const double* vel, const StencilParams& sp, int k,
                            double* grad, int accumulate, cudaStream_t st);

// ------------------------------------------------------------------ batched GEMM

// C = alpha * op(A) * diag(d) * op(B) + beta * C, complex, no conjugation.
// lowerC restricts the update to row >= col.  triA/triB describe structural
// zeros: triA 1 -> op(A)[r][k] = 0 for k > r, 2 -> for k < r;
// triB 1 -> op(B)[k][c] = 0 for k < c, 2 -> for k > c.
template <typename R>
struct GemmOp {
    const cpx<R>* A;
    const cpx<R>* B;
    cpx<R>* C;
    const cpx<R>* d;
    int64_t lda, ldb, ldc;
    int M, N, K;
    int transA, transB, lowerC, triA, triB;
    R alpha_re, alpha_im, beta_re, beta_im;
};
struct GemmTile {
    int op, tm, tn;
};

enum GemmShape { kGemmSquare = 0, kGemmSkinny = 1 };
int GemmTileM(GemmShape s);
int GemmTileN(GemmShape s);
// Appends the output tiles of `op` (index opIndex) to `tiles`.
template <typename R>
void AppendGemmTiles(const GemmOp<R>& op, int opIndex, GemmShape shape, std::vector<GemmTile>& tiles);
template <typename R>
void LaunchGemm(const GemmOp<R>* ops, const GemmTile* tiles, int numTiles, GemmShape shape, cudaStream_t st);

// Tensor-core (tcgen05, split TF32) form of the complex-single batched GEMM
// (factor_tc.cu) for ops with real alpha and beta: same op semantics, 128 x
// 64 output tiles, each a self-contained record (operand pointers at the
// tile's origin and the start of its K range), so the kernel reads one
// record per tile and no op table.  A pipeline wait that times out sets the
// value 2 in *status and leaves its tile unwritten.
constexpr int kGemmTcRows = 128, kGemmTcCols = 64;
struct GemmTcTile {
    const c32* A;  // op(A)(row0, kb)
    const c32* B;  // op(B)(kb, col0)
    const c32* d;  // d + kb, or null
    c32* C;        // C(row0, col0)
    int lda, ldb, ldc;
    int m, n, nk;  // rows and columns of the tile inside the op, K extent
    int diag;      // lowerC: only tile-relative r - c >= diag is written
    int flags;     // bit 0 transA, bit 1 transB
    float alpha, beta;
};
// Whether `op` can take tensor-core tiles (real alpha and beta).
bool GemmTcEligible(const GemmOp<float>& op);
void PrepareFactorTcKernels();
void AppendGemmTilesTc(const GemmOp<float>& op, std::vector<GemmTcTile>& tiles);
void LaunchGemmTc(const GemmTcTile* tiles, int numTiles, int* status, cudaStream_t st);

// ------------------------------------------------------------------ factorization

constexpr int kNB = 32;  // column block of the frontal LDL^T

// Leading dimension of a front's persistent factor G: s + u rounded up to
// even, so that every column starts on a 16-byte boundary for bulk copies
// (the padding row is zero).
__host__ __device__ inline int GLeadingDim(int s, int u) { return (s + u + 1) & ~1; }

// One front of one panel during the factorization (cliq::LDL replacement).
template <typename R>
struct FactorFront {
    cpx<R>* L;      // transient (s+u) x s frontal columns, ld = s+u
    cpx<R>* G;      // persistent (s+u) x s: [inv(L11); -L21 inv(L11)], ld = ldg
    cpx<R>* D;      // persistent pivots, s entries
    cpx<R>* U;      // u x u Schur complement (update matrix), ld = u
    cpx<R>* T;      // inversion scratch
    const int* rel; // u entries: row of each structure index in the parent front
    int s, u;
    int ldg;        // leading dimension of G: s+u rounded up to even (16-byte aligned columns)
    int parent;     // index of the parent in the same descriptor array (-1 for a root)
    int cls;        // panel class (tables below)
    int ndOff;      // first ND index of the node in its class ordering
    int vOffset;    // global sweep coordinate of the padded subproblem's first plane
    int s3aOff;     // offset of the panel's artificial-PML table
};

struct ClassTables {
    const int* ndToNat[3];
    const int* nbrRows[3];
};

struct AssemblyParams {
    StencilParams sp;
    const double* vel;    // natural-order velocity
    const z64* s3a;       // artificial s3Inv per panel, vSize+2 entries each
    const z64* is3a;
    double damping;
    ClassTables tabs;
};

template <typename R>
void LaunchAssemble(const FactorFront<R>* fronts, const int* list, int n, const AssemblyParams& ap,
                    cudaStream_t st);
// tasks: (child front, first update column)
template <typename R>
void LaunchExtendAdd(const FactorFront<R>* fronts, const int2* tasks, int n, cudaStream_t st);
template <typename R>
void LaunchLdlDiag(const FactorFront<R>* fronts, const int* list, int n, int J, int* status, cudaStream_t st);
// tasks: (front, first row of a kTrsmRows-row tile below the diagonal block)
constexpr int kTrsmRows = 32;
template <typename R>
void LaunchLdlTrsm(const FactorFront<R>* fronts, const int2* tasks, int n, int J, cudaStream_t st);

// ------------------------------------------------------------------ panel solves

// One front of the panel being solved (cliq::Solve replacement, sweep.cu).
template <typename R>
struct SweepFront {
    const cpx<R>* G;      // (s+u) x s selectively inverted factor, ld = ldg
    const cpx<R>* D;      // pivots
    cpx<R>* Rb;           // [s+u][3][k]: natural rhs, child 0 update, child 1 update
    cpx<R>* parentRb;     // the parent's Rb (null for a root)
    cpx<R>* Y;            // [s][k] forward result
    cpx<R>* Z;            // [s+u][k] backward input
    const int* lower;     // u ND indices of the front's structure
    const int* rel;       // u rows of the structure in the parent front
    int s, u, ndOff, childSlot;
    int ldg;              // leading dimension of G (even)
    const void* tmap;     // complex single: TMA maps of G (forward, backward; 128 bytes each)
};

// One CTA of a sweep launch: kSweepRows output rows from row0, kSweepCols
// right-hand sides from col0, the K-chunk [k0, k1); split `split` of `nsplit`
// whose partials live at slot+split and whose arrival counter is `counter`.
struct SweepTile {
    int front, row0, col0, k0, k1, split, nsplit, slot, counter;
};

constexpr int kSweepRows = 64;     // output rows per CTA (one per thread of a slice)
constexpr int kSweepSlices = 4;    // K-slices per CTA, one warp pair each
constexpr int kSweepThreads = kSweepRows * kSweepSlices;
constexpr int kSweepCols = 16;
constexpr size_t kSweepSmemBytes = 32 * 1024;  // staged right-hand-side chunk

constexpr int kTcRows = 128;       // rows per CTA of the tensor-core sweep kernels (UMMA M)

// Device scratch of the sweep: split-K partials (rows-per-tile * kSweepCols
// complex entries per slot), arrival counters (zero between launches), the
// panel's ND-ordered solution vector [ND index][k] and a status word (bit 2:
// a tensor-core pipeline wait timed out).
struct SweepWork {
    void* partials;
    int* counters;
    void* xnd;
    int* status;
};

struct PanelIO {
    const int* ndToNat;
    int nxy, nx, nz;
    int ldk;         // row stride (complex entries per point) of the natural-order grid
    int padding;     // leading planes of the subproblem that are artificial padding
    int vOffset;     // global v of the subproblem's first plane
    int lowV, highV; // global v range of the panel's own planes
    int inMode;      // 0: B_i; 1: B_i - A_{i,i-1} B_{i-1}; 2: -A_{i,i+1} B_{i+1} only
    int outAccumulate;
    StencilParams sp;
};

// Largest K-chunk a sweep CTA can stage.
template <typename R>
int SweepMaxChunk();
// Sets kernel attributes the sweep kernels need (call before any graph capture).
template <typename R>
void PrepareSweepKernels();
// tasks: (front, first row), kSweepRows rows each.  `pdl`: launch as a
// programmatic dependent of the preceding kernel (the tensor-core sweep).
template <typename R>
void LaunchSweepPregather(const SweepFront<R>* fr, const int2* tasks, int n, const z64* B, int k, const PanelIO& io,
                          cudaStream_t st, bool pdl = false);
template <typename R>
void LaunchSweepForward(const SweepFront<R>* fr, const SweepTile* tiles, int n, int maxChunk, int k,
                        const SweepWork& w, cudaStream_t st);
template <typename R>
void LaunchSweepBackwardGather(const SweepFront<R>* fr, const int2* tasks, int n, int k, const SweepWork& w,
                               cudaStream_t st, bool pdl = false);
template <typename R>
void LaunchSweepBackward(const SweepFront<R>* fr, const SweepTile* tiles, int n, int maxChunk, z64* B, int k,
                         const PanelIO& io, const SweepWork& w, cudaStream_t st);

// Tensor-core (tcgen05, split TF32) forms for complex-single factors
// (sweep_tc.cu); tiles of kTcRows rows, any K-chunk length, and `cols` (16
// or 32) right-hand sides per tile: the tile list's col0 steps by `cols`,
// and a split tile's partial slots and counters are per 16-column sub-tile
// (slot (t.slot + split) * cols / 16 + h, counter t.counter * cols / 16 + h).
void PrepareSweepTcKernels();
// Bytes of the two TMA maps of one front, and their encoding (host) into
// out (64-byte aligned host memory) for the front's G, s, u and ldg.
constexpr size_t kSweepTcMapBytes = 256;
void EncodeSweepTcMaps(const SweepFront<float>& f, void* out);
void LaunchSweepForwardTc(const SweepFront<float>* fr, const SweepTile* tiles, int n, int k, int cols,
                          const SweepWork& w, cudaStream_t st);
void LaunchSweepBackwardTc(const SweepFront<float>* fr, const SweepTile* tiles, int n, z64* B, int k, int cols,
                           const PanelIO& io, const SweepWork& w, cudaStream_t st);

// ------------------------------------------------------------------ GMRES vectors

// Per-RHS reductions over natural-order [N][k] vectors; partial sums per block
// land in `partial` (gridDim x k) and a second pass sums them in fixed order.
int ReduceBlocks(int64_t npoints, int k);
void LaunchNormsPartial(const z64* w, int64_t npoints, int k, double* partial, cudaStream_t st);
void LaunchSumPartialReal(const double* partial, int nblocks, int k, double* out, int sqrtOut, cudaStream_t st);
// w -= h_prev (.) v_prev (if v_prev) and partial dots conj(v_next) . w
void LaunchMgsStep(z64* w, const z64* v_prev, const z64* h_prev, const z64* v_next, int64_t npoints, int k,
                   z64* partial, cudaStream_t st);
void LaunchSumPartialComplex(const z64* partial, int nblocks, int k, z64* out, cudaStream_t st);
// v := w / s (per RHS, s real)
void LaunchScaleColumns(const z64* w, const double* s, z64* v, int64_t npoints, int k, cudaStream_t st);
// x := x0 + sum_i y[i,r] V_i[:,r]
void LaunchCombine(const z64* x0, const z64* V, int64_t vstride, const z64* y, int j1, z64* x, int64_t npoints,
                   int k, cudaStream_t st);
// w := w - h (.) v   (final MGS axpy)
void LaunchAxpyColumns(z64* w, const z64* v, const z64* h, int64_t npoints, int k, cudaStream_t st);

}  // namespace psp_b200
