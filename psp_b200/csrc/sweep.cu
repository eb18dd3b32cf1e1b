// Multi-RHS frontal solves of the sweep (cliq::Solve replacement) on the
// selectively inverted factors G = [inv(L11); -L21 inv(L11)].
//
// Forward, per front:  [Y; U] = G * R_s + [0; R_u]
// Backward, per front: X_s = G^T * [inv(D) Y; X_u]
//
// Data flow of one panel solve (all buffers are dense, k right-hand sides
// contiguous per row):
//   * pre-gather: every front row's right-hand side from the natural-order
//     grid (with the sweep's panel coupling folded in) lands in plane 0 of the
//     front's R buffer; planes 1 and 2 (one per child) start at zero;
//   * forward, one launch per tree depth from the leaves: a CTA stages the sum
//     of the three planes for its K-chunk, streams its rows of G once, and the
//     tile's final CTA writes Y, or pushes U into the parent's plane reserved
//     for this child (no two writers share an address, so no atomics);
//   * backward, per depth from the root: a gather writes Z = [inv(D) Y; X_u]
//     (X_u read from the panel's ND-ordered solution vector), then a GEMM
//     launch streams G^T and writes X_s to that vector and to the grid.
// One CTA owns kSweepRows output rows (one per thread) and kSweepCols right-
// hand sides; long K ranges are split over CTAs and the partials reduced in
// fixed order by the tile's last CTA, so results are deterministic.
#include "kernels.cuh"

namespace psp_b200 {

namespace {

constexpr int kGatherThreads = 256;

// Read-only cached load of one complex entry.
__device__ __forceinline__ cpx<float> LdgC(const cpx<float>* p) {
    const float2 v = __ldg(reinterpret_cast<const float2*>(p));
    return mk(v.x, v.y);
}
__device__ __forceinline__ cpx<double> LdgC(const cpx<double>* p) {
    const double2 v = __ldg(reinterpret_cast<const double2*>(p));
    return mk(v.x, v.y);
}

template <typename R>
__device__ __forceinline__ cpx<R> NaturalRhs(const PanelIO& io, const z64* __restrict__ B, int col, int r) {
    const int pn = io.ndToNat[col];
    const int xy = pn % io.nxy, vl = pn / io.nxy;
    if (vl < io.padding) return mk<R>(0, 0);
    const int v = io.vOffset + vl;
    const int64_t nat = xy + (int64_t)(io.nz - 1 - v) * io.nxy;
    const int x = xy % io.nx, y = xy / io.nx;
    const StencilParams& sp = io.sp;
    if (io.inMode == 2) {
        if (v != io.highV) return mk<R>(0, 0);
        const z64 cz = sp.s1[x + 1] * sp.s2[y + 1];
        const z64 coef = sp.ihz2 * (cz * (sp.is3[v + 2] + sp.is3[v + 1]));
        return ccast<R>(coef * B[(nat - io.nxy) * io.ldk + r]);
    }
    z64 val = B[nat * io.ldk + r];
    if (io.inMode == 1 && v == io.lowV) {
        const z64 cz = sp.s1[x + 1] * sp.s2[y + 1];
        const z64 coef = sp.ihz2 * (cz * (sp.is3[v] + sp.is3[v + 1]));
        val += coef * B[(nat + io.nxy) * io.ldk + r];
    }
    return ccast<R>(val);
}

// Adds the accumulators of K-slices 1.. into slice 0 through shared memory
// `red` (which may alias the staged chunk: the first barrier retires it).
template <typename R>
__device__ __forceinline__ void ReduceSlices(cpx<R>* red, cpx<R> (&acc)[kSweepCols]) {
    const int slice = threadIdx.x / kSweepRows, row = threadIdx.x % kSweepRows;
    __syncthreads();
    if (slice > 0) {
#pragma unroll
        for (int n = 0; n < kSweepCols; ++n) red[((slice - 1) * kSweepCols + n) * kSweepRows + row] = acc[n];
    }
    __syncthreads();
    if (slice == 0) {
        for (int s = 1; s < kSweepSlices; ++s) {
#pragma unroll
            for (int n = 0; n < kSweepCols; ++n) acc[n] += red[((s - 1) * kSweepCols + n) * kSweepRows + row];
        }
    }
}

// Split-K over CTAs: slice 0 stores this CTA's partial; returns true in the
// CTA that must finish the tile, whose slice-0 threads then hold the
// fixed-order sum of all partials.
template <typename R>
__device__ __forceinline__ bool ReduceSplits(const SweepTile& t, const SweepWork& w, cpx<R> (&acc)[kSweepCols]) {
    if (t.nsplit <= 1) return true;
    __shared__ int isLast;
    cpx<R>* part = reinterpret_cast<cpx<R>*>(w.partials);
    const int tid = threadIdx.x;
    const bool owner = tid < kSweepRows;
    if (owner) {
        cpx<R>* mine = part + ((int64_t)(t.slot + t.split) * kSweepCols) * kSweepRows;
#pragma unroll
        for (int n = 0; n < kSweepCols; ++n) mine[n * kSweepRows + tid] = acc[n];
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) {
        const int prev = atomicAdd(w.counters + t.counter, 1);
        isLast = (prev == t.nsplit - 1);
    }
    __syncthreads();
    if (!isLast) return false;
    __threadfence();
    if (owner) {
#pragma unroll
        for (int n = 0; n < kSweepCols; ++n) acc[n] = mk<R>(0, 0);
        for (int s = 0; s < t.nsplit; ++s) {
            const cpx<R>* p = part + ((int64_t)(t.slot + s) * kSweepCols) * kSweepRows;
#pragma unroll
            for (int n = 0; n < kSweepCols; ++n) acc[n] += p[n * kSweepRows + tid];
        }
    }
    if (tid == 0) w.counters[t.counter] = 0;  // ready for the next launch
    return true;
}

// K range of this thread's slice inside the CTA's chunk [k0, k1).
__device__ __forceinline__ void SliceRange(int k0, int k1, int& sb, int& se) {
    const int slice = threadIdx.x / kSweepRows;
    const int q = (k1 - k0 + kSweepSlices - 1) / kSweepSlices;
    sb = k0 + slice * q;
    se = min(k1, sb + q);
}

// acc[n] += sum_{kk in [kb, ke)} A(kk) * S[kk - k0][n], A(kk) = ap[kk * astep].
// Loads run one batch ahead of the arithmetic so each warp keeps a batch of
// G in flight while it computes on the previous one.
template <typename R>
__device__ __forceinline__ void StreamRow(const cpx<R>* __restrict__ ap, int64_t astep, int kb, int ke, int k0,
                                          const cpx<R>* S, cpx<R> (&acc)[kSweepCols]) {
    constexpr int U = sizeof(R) == 4 ? 8 : 2;
    const int nb = (ke - kb) / U;
    const cpx<R>* p = ap + (int64_t)kb * astep;
    cpx<R> cur[U], nxt[U];
    if (nb > 0) {
#pragma unroll
        for (int u = 0; u < U; ++u) cur[u] = LdgC(p + u * astep);
    }
    for (int b = 0; b < nb; ++b) {
        const bool more = b + 1 < nb;
        if (more) {
            const cpx<R>* q = p + (int64_t)(b + 1) * U * astep;
#pragma unroll
            for (int u = 0; u < U; ++u) nxt[u] = LdgC(q + u * astep);
        }
        const cpx<R>* s0 = S + (kb + b * U - k0) * kSweepCols;
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const cpx<R>* s = s0 + u * kSweepCols;
#pragma unroll
            for (int n = 0; n < kSweepCols; ++n) cfma(acc[n], cur[u], s[n]);
        }
        if (more) {
#pragma unroll
            for (int u = 0; u < U; ++u) cur[u] = nxt[u];
        }
    }
    for (int kk = kb + nb * U; kk < ke; ++kk) {
        const cpx<R> a = ap[kk * astep];
        const cpx<R>* s = S + (kk - k0) * kSweepCols;
#pragma unroll
        for (int n = 0; n < kSweepCols; ++n) cfma(acc[n], a, s[n]);
    }
}

// Plane 0 of every front row := natural right-hand side (zero below the
// front's pivots), planes 1-2 := 0.  tasks: (front, first row).
template <typename R>
__global__ void __launch_bounds__(kGatherThreads) sweep_pregather_kernel(const SweepFront<R>* __restrict__ fr,
                                                                         const int2* __restrict__ tasks,
                                                                         const z64* __restrict__ B, int k,
                                                                         PanelIO io) {
    PdlTrigger();
    PdlWait();
    const int2 task = tasks[blockIdx.x];
    const SweepFront<R> f = fr[task.x];
    const int rows = min(kSweepRows, f.s + f.u - task.y);
    for (int e = threadIdx.x; e < rows * k; e += blockDim.x) {
        const int i = task.y + e / k, n = e % k;
        cpx<R>* dst = f.Rb + (int64_t)i * 3 * k + n;
        dst[0] = i < f.s ? NaturalRhs<R>(io, B, f.ndOff + i, n) : mk<R>(0, 0);
        dst[k] = mk<R>(0, 0);
        dst[2 * k] = mk<R>(0, 0);
    }
}

template <typename R>
__global__ void __launch_bounds__(kSweepThreads, 2) sweep_forward_kernel(const SweepFront<R>* __restrict__ fr,
                                                                      const SweepTile* __restrict__ tiles, int k,
                                                                      SweepWork work) {
    extern __shared__ unsigned char smem_raw[];
    cpx<R>* Bs = reinterpret_cast<cpx<R>*>(smem_raw);  // [kc][kSweepCols]
    const SweepTile t = tiles[blockIdx.x];
    const SweepFront<R> f = fr[t.front];
    const int tid = threadIdx.x;
    const int kc = t.k1 - t.k0;
    const int ncol = min(kSweepCols, k - t.col0);
    for (int e = tid; e < kc * kSweepCols; e += blockDim.x) {
        const int kk = e / kSweepCols, n = e % kSweepCols;
        cpx<R> v = mk<R>(0, 0);
        if (n < ncol) {
            const cpx<R>* src = f.Rb + (int64_t)(t.k0 + kk) * 3 * k + t.col0 + n;
            v = src[0] + src[k] + src[2 * k];
        }
        Bs[e] = v;
    }
    __syncthreads();
    const int r = t.row0 + tid % kSweepRows;
    const int M = f.s + f.u;
    cpx<R> acc[kSweepCols];
#pragma unroll
    for (int n = 0; n < kSweepCols; ++n) acc[n] = mk<R>(0, 0);
    int sb, se;
    SliceRange(t.k0, t.k1, sb, se);
    if (r < M) StreamRow<R>(f.G + r, f.ldg, sb, min(se, r + 1), t.k0, Bs, acc);  // inv(L11) lower triangular
    ReduceSlices<R>(Bs, acc);
    if (!ReduceSplits<R>(t, work, acc)) return;
    if (tid >= kSweepRows || r >= M) return;
    if (r < f.s) {
        cpx<R>* dst = f.Y + (int64_t)r * k + t.col0;
#pragma unroll
        for (int n = 0; n < kSweepCols; ++n)
            if (n < ncol) dst[n] = acc[n];
    } else if (f.parentRb) {
        const cpx<R>* src = f.Rb + (int64_t)r * 3 * k + t.col0;
        cpx<R>* dst = f.parentRb + ((int64_t)f.rel[r - f.s] * 3 + 1 + f.childSlot) * k + t.col0;
#pragma unroll
        for (int n = 0; n < kSweepCols; ++n)
            if (n < ncol) dst[n] = acc[n] + src[n] + src[k + n] + src[2 * k + n];
    }
}

// Z := [inv(D) Y; X_u] for the fronts of one depth.  tasks: (front, first row).
template <typename R>
__global__ void __launch_bounds__(kGatherThreads) sweep_bgather_kernel(const SweepFront<R>* __restrict__ fr,
                                                                       const int2* __restrict__ tasks, int k,
                                                                       SweepWork work) {
    PdlTrigger();
    PdlWait();
    const int2 task = tasks[blockIdx.x];
    const SweepFront<R> f = fr[task.x];
    const cpx<R>* X = reinterpret_cast<const cpx<R>*>(work.xnd);
    const int rows = min(kSweepRows, f.s + f.u - task.y);
    for (int e = threadIdx.x; e < rows * k; e += blockDim.x) {
        const int i = task.y + e / k, n = e % k;
        f.Z[(int64_t)i * k + n] = i < f.s ? cdiv(f.Y[(int64_t)i * k + n], f.D[i])
                                          : X[(int64_t)f.lower[i - f.s] * k + n];
    }
}

template <typename R>
__global__ void __launch_bounds__(kSweepThreads, 2) sweep_backward_kernel(const SweepFront<R>* __restrict__ fr,
                                                                       const SweepTile* __restrict__ tiles,
                                                                       z64* __restrict__ B, int k, PanelIO io,
                                                                       SweepWork work) {
    extern __shared__ unsigned char smem_raw[];
    cpx<R>* Zs = reinterpret_cast<cpx<R>*>(smem_raw);
    cpx<R>* X = reinterpret_cast<cpx<R>*>(work.xnd);  // [ND index][k]
    const SweepTile t = tiles[blockIdx.x];
    const SweepFront<R> f = fr[t.front];
    const int tid = threadIdx.x;
    const int kc = t.k1 - t.k0;
    const int ncol = min(kSweepCols, k - t.col0);
    const int64_t ld = f.ldg;
    for (int e = tid; e < kc * kSweepCols; e += blockDim.x) {
        const int kk = e / kSweepCols, n = e % kSweepCols;
        Zs[e] = n < ncol ? f.Z[(int64_t)(t.k0 + kk) * k + t.col0 + n] : mk<R>(0, 0);
    }
    __syncthreads();
    const int r = t.row0 + tid % kSweepRows;
    cpx<R> acc[kSweepCols];
#pragma unroll
    for (int n = 0; n < kSweepCols; ++n) acc[n] = mk<R>(0, 0);
    int sb, se;
    SliceRange(t.k0, t.k1, sb, se);
    if (r < f.s) StreamRow<R>(f.G + r * ld, 1, max(sb, r), se, t.k0, Zs, acc);  // G^T upper triangular
    ReduceSlices<R>(Zs, acc);
    if (!ReduceSplits<R>(t, work, acc)) return;
    if (tid >= kSweepRows || r >= f.s) return;
    const int col = f.ndOff + r;
    cpx<R>* xd = X + (int64_t)col * k + t.col0;
#pragma unroll
    for (int n = 0; n < kSweepCols; ++n)
        if (n < ncol) xd[n] = acc[n];
    const int pn = io.ndToNat[col];
    const int xy = pn % io.nxy, vl = pn / io.nxy;
    if (vl < io.padding) return;
    const int v = io.vOffset + vl;
    z64* dst = B + (xy + (int64_t)(io.nz - 1 - v) * io.nxy) * io.ldk + t.col0;
#pragma unroll
    for (int n = 0; n < kSweepCols; ++n) {
        if (n >= ncol) break;
        const z64 val = ccast<double>(acc[n]);
        dst[n] = io.outAccumulate ? dst[n] + val : val;
    }
}

}  // namespace

template <typename R>
int SweepMaxChunk() {
    return (int)(kSweepSmemBytes / (sizeof(cpx<R>) * kSweepCols));
}

// Dynamic shared memory of a sweep CTA: the staged chunk, reused for the
// slice reduction.
template <typename R>
size_t SweepSmem(int chunk) {
    const size_t staged = sizeof(cpx<R>) * kSweepCols * chunk;
    const size_t red = sizeof(cpx<R>) * kSweepCols * kSweepRows * (kSweepSlices - 1);
    return staged > red ? staged : red;
}

template <typename R>
void PrepareSweepKernels() {
    const int bytes = (int)SweepSmem<R>(SweepMaxChunk<R>());
    CUDA_CHECK(cudaFuncSetAttribute(sweep_forward_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    CUDA_CHECK(cudaFuncSetAttribute(sweep_backward_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
}

template <typename R>
void LaunchSweepPregather(const SweepFront<R>* fr, const int2* tasks, int n, const z64* B, int k, const PanelIO& io,
                          cudaStream_t st, bool pdl) {
    if (n <= 0) return;
    if (pdl) {
        LaunchPdl(sweep_pregather_kernel<R>, dim3(n), dim3(kGatherThreads), 0, st, fr, tasks, B, k, io);
        return;
    }
    sweep_pregather_kernel<R><<<n, kGatherThreads, 0, st>>>(fr, tasks, B, k, io);
    CUDA_LAUNCH_CHECK();
}

template <typename R>
void LaunchSweepForward(const SweepFront<R>* fr, const SweepTile* tiles, int n, int maxChunk, int k,
                        const SweepWork& w, cudaStream_t st) {
    if (n <= 0) return;
    sweep_forward_kernel<R><<<n, kSweepThreads, SweepSmem<R>(maxChunk), st>>>(fr, tiles, k, w);
    CUDA_LAUNCH_CHECK();
}

template <typename R>
void LaunchSweepBackwardGather(const SweepFront<R>* fr, const int2* tasks, int n, int k, const SweepWork& w,
                               cudaStream_t st, bool pdl) {
    if (n <= 0) return;
    if (pdl) {
        LaunchPdl(sweep_bgather_kernel<R>, dim3(n), dim3(kGatherThreads), 0, st, fr, tasks, k, w);
        return;
    }
    sweep_bgather_kernel<R><<<n, kGatherThreads, 0, st>>>(fr, tasks, k, w);
    CUDA_LAUNCH_CHECK();
}

template <typename R>
void LaunchSweepBackward(const SweepFront<R>* fr, const SweepTile* tiles, int n, int maxChunk, z64* B, int k,
                         const PanelIO& io, const SweepWork& w, cudaStream_t st) {
    if (n <= 0) return;
    sweep_backward_kernel<R><<<n, kSweepThreads, SweepSmem<R>(maxChunk), st>>>(fr, tiles, B, k, io, w);
    CUDA_LAUNCH_CHECK();
}

#define PSP_SWEEP_INSTANTIATE(R)                                                                                  \
    template int SweepMaxChunk<R>();                                                                              \
    template void PrepareSweepKernels<R>();                                                                       \
    template void LaunchSweepPregather<R>(const SweepFront<R>*, const int2*, int, const z64*, int, const PanelIO&, \
                                          cudaStream_t, bool);                                                    \
    template void LaunchSweepForward<R>(const SweepFront<R>*, const SweepTile*, int, int, int, const SweepWork&,  \
                                        cudaStream_t);                                                            \
    template void LaunchSweepBackwardGather<R>(const SweepFront<R>*, const int2*, int, int, const SweepWork&,     \
                                               cudaStream_t, bool);                                               \
    template void LaunchSweepBackward<R>(const SweepFront<R>*, const SweepTile*, int, int, z64*, int,           \
                                         const PanelIO&, const SweepWork&, cudaStream_t);

PSP_SWEEP_INSTANTIATE(double)
PSP_SWEEP_INSTANTIATE(float)

}  // namespace psp_b200
