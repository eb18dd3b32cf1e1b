// Tensor-core (tcgen05) versions of the sweep's frontal products for complex-
// single factors, with the same data flow as sweep.cu:
//   forward  [Y; U] = G R_s + [0; R_u]      backward  X_s = G^T [inv(D) Y; X_u]
//
// A complex product C = A B (A: rows x K, B: K x 16 right-hand sides) runs as
// one real product on the tensor core: A's rows read as interleaved
// (re, im) pairs form a rows x 2K real matrix, and every complex entry b of
// B becomes the 2x2 real block [[re b, im b], [-im b, re b]] of a 2K x 32
// real matrix, so the 32 real accumulator columns are C's interleaved
// (re, im) pairs.  Each operand is split into tf32 head and tail
// (x = hi + lo) and the products hi*hi + hi*lo + lo*hi are accumulated in
// FP32 in tensor memory: about FP32 accuracy from TF32 inputs.
//
// One CTA (128 threads) owns 128 rows (one UMMA M=128 tile) and 16 right-
// hand sides over one K-chunk; it stages 16 complex K-columns at a time into
// two shared-memory buffers while the tensor core consumes the previous one.
// Every wait on an mbarrier is bounded; a timeout sets bit 2 of the status
// word, releases tensor memory and leaves the tile unwritten.
#include "kernels.cuh"
#include "umma.cuh"

namespace psp_b200 {

namespace {

using umma::KMajorOffset;

constexpr int kTcThreads = 128;
constexpr int kStageK = 16;                                      // complex K per stage
constexpr uint32_t kSbo = (2 * kStageK / 4) * umma::kChunkBytes;  // 8-row group stride (1 KB)
constexpr uint32_t kAPlane = kTcRows * 2 * kStageK * 4;           // 16 KB
constexpr uint32_t kBPlane = 2 * kSweepCols * 2 * kStageK * 4;    // 4 KB
constexpr uint32_t kStageBytes = 2 * kAPlane + 2 * kBPlane;
constexpr int kStages = 2;
constexpr uint32_t kTmemCols = 32;
constexpr uint32_t kIdesc = umma::InstrDescTf32(kTcRows, 2 * kSweepCols);

__device__ __forceinline__ void StoreSplitPair(unsigned char* hi, unsigned char* lo, uint32_t off, float a, float b) {
    float ah, al, bh, bl;
    umma::SplitTf32(a, ah, al);
    umma::SplitTf32(b, bh, bl);
    *reinterpret_cast<float2*>(hi + off) = make_float2(ah, bh);
    *reinterpret_cast<float2*>(lo + off) = make_float2(al, bl);
}

// B' rows 2n, 2n+1 for complex entry b at (kc, n): the 2x2 real block.
__device__ __forceinline__ void StoreBBlock(unsigned char* S, int kc, int n, c32 b) {
    unsigned char* hi = S + 2 * kAPlane;
    unsigned char* lo = hi + kBPlane;
    StoreSplitPair(hi, lo, KMajorOffset(2 * n, 2 * kc, kSbo), b.re, -b.im);
    StoreSplitPair(hi, lo, KMajorOffset(2 * n + 1, 2 * kc, kSbo), b.im, b.re);
}

// One stage's operands held in registers between the global loads and the
// split/store into shared memory, so the loads of stage st+1 are in flight
// while stage st is handed to the tensor core.
constexpr int kBPerThread = kStageK * kSweepCols / kTcThreads;  // 2
struct StageRegs {
    c32 a[kStageK];
    c32 b[kBPerThread];
};

__device__ __forceinline__ c32 LdgC32(const c32* p) {
    const float2 v = __ldg(reinterpret_cast<const float2*>(p));
    return mk(v.x, v.y);
}

__device__ __forceinline__ void StoreStage(unsigned char* S, const StageRegs& R, bool rowMajorA) {
    const int tid = threadIdx.x;
#pragma unroll
    for (int i = 0; i < kStageK; ++i) {
        // forward: this thread's row, K-column i; backward: element tid + 128 i
        const int m = rowMajorA ? (tid + i * kTcThreads) / kStageK : tid;
        const int kc = rowMajorA ? (tid + i * kTcThreads) % kStageK : i;
        StoreSplitPair(S, S + kAPlane, KMajorOffset(m, 2 * kc, kSbo), R.a[i].re, R.a[i].im);
    }
#pragma unroll
    for (int j = 0; j < kBPerThread; ++j) {
        const int e = tid + j * kTcThreads;
        StoreBBlock(S, e / kSweepCols, e % kSweepCols, R.b[j]);
    }
}

__device__ __forceinline__ void IssueStage(unsigned char* S, uint32_t tmem, bool first) {
    const uint32_t aHi = umma::SmemAddr(S), aLo = aHi + kAPlane;
    const uint32_t bHi = aHi + 2 * kAPlane, bLo = bHi + kBPlane;
#pragma unroll
    for (int s = 0; s < 2 * kStageK / 8; ++s) {
        const uint32_t o = s * 2 * umma::kChunkBytes;
        const uint64_t ah = umma::SmemDesc(aHi + o, umma::kChunkBytes, kSbo);
        const uint64_t al = umma::SmemDesc(aLo + o, umma::kChunkBytes, kSbo);
        const uint64_t bh = umma::SmemDesc(bHi + o, umma::kChunkBytes, kSbo);
        const uint64_t bl = umma::SmemDesc(bLo + o, umma::kChunkBytes, kSbo);
        umma::MmaTf32(tmem, ah, bh, kIdesc, (first && s == 0) ? 0u : 1u);
        umma::MmaTf32(tmem, ah, bl, kIdesc, 1u);
        umma::MmaTf32(tmem, al, bh, kIdesc, 1u);
    }
}

// Split-K over CTAs for 128-row tiles (every thread owns one row).
__device__ __forceinline__ bool ReduceSplitsTc(const SweepTile& t, const SweepWork& w, c32 (&acc)[kSweepCols]) {
    if (t.nsplit <= 1) return true;
    __shared__ int isLast;
    c32* part = reinterpret_cast<c32*>(w.partials);
    const int tid = threadIdx.x;
    c32* mine = part + ((int64_t)(t.slot + t.split) * kSweepCols) * kTcRows;
#pragma unroll
    for (int n = 0; n < kSweepCols; ++n) mine[n * kTcRows + tid] = acc[n];
    __threadfence();
    __syncthreads();
    if (tid == 0) isLast = (atomicAdd(w.counters + t.counter, 1) == t.nsplit - 1);
    __syncthreads();
    if (!isLast) return false;
    __threadfence();
#pragma unroll
    for (int n = 0; n < kSweepCols; ++n) acc[n] = mk<float>(0, 0);
    for (int s = 0; s < t.nsplit; ++s) {
        const c32* p = part + ((int64_t)(t.slot + s) * kSweepCols) * kTcRows;
#pragma unroll
        for (int n = 0; n < kSweepCols; ++n) acc[n] += p[n * kTcRows + tid];
    }
    if (tid == 0) w.counters[t.counter] = 0;
    return true;
}

// Shared prologue: mbarriers and TMEM; returns the TMEM base column address.
__device__ __forceinline__ uint32_t TcSetup(uint64_t* mbar, uint32_t* slot) {
    const int warp = threadIdx.x / 32;
    if (threadIdx.x == 0) {
        for (int i = 0; i <= kStages; ++i) umma::MbarInit(&mbar[i], 1);
        umma::FenceMbarInit();
    }
    if (warp == 0) umma::TmemAlloc(slot, kTmemCols);
    umma::FenceBeforeSync();
    __syncthreads();
    umma::FenceAfterSync();
    return *slot;
}

// Waits for every issued MMA, reads this thread's accumulator row and frees
// TMEM.  Returns false (status set) if the tensor-core pipeline timed out.
__device__ __forceinline__ bool TcFinish(uint64_t* mbar, uint32_t tmem, int nst, bool ok, int* status,
                                         c32 (&acc)[kSweepCols]) {
    const int warp = threadIdx.x / 32;
    if (nst > 0) {
        if (threadIdx.x == 0) umma::CommitTo(&mbar[kStages]);
        if (!umma::MbarWaitBounded(&mbar[kStages], 0, status)) ok = false;
    }
    ok = !__syncthreads_or(!ok);
    umma::FenceAfterSync();
#pragma unroll
    for (int n = 0; n < kSweepCols; ++n) acc[n] = mk<float>(0, 0);
    if (nst > 0 && ok) {
        float v[32];
        umma::TmemLoad32(tmem + ((uint32_t)(warp * 32) << 16), v);
#pragma unroll
        for (int n = 0; n < kSweepCols; ++n) acc[n] = mk(v[2 * n], v[2 * n + 1]);
    }
    umma::FenceBeforeSync();
    __syncthreads();
    if (warp == 0) umma::TmemDealloc(tmem, kTmemCols);
    return ok;
}

__global__ void __launch_bounds__(kTcThreads) sweep_tc_forward_kernel(const SweepFront<float>* __restrict__ fr,
                                                                      const SweepTile* __restrict__ tiles, int k,
                                                                      SweepWork work) {
    extern __shared__ unsigned char smem_raw[];
    __shared__ uint64_t mbar[kStages + 1];
    __shared__ uint32_t tmemSlot;
    unsigned char* smem = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const SweepTile t = tiles[blockIdx.x];
    const SweepFront<float> f = fr[t.front];
    const int tid = threadIdx.x;
    const int M = f.s + f.u;
    const int64_t ld = M;
    const int ncol = min(kSweepCols, k - t.col0);
    const int kb = t.k0, ke = min(t.k1, t.row0 + kTcRows);  // inv(L11) is lower triangular
    const int nst = ke > kb ? (ke - kb + kStageK - 1) / kStageK : 0;
    const uint32_t tmem = TcSetup(mbar, &tmemSlot);
    bool ok = true;
    const int r = t.row0 + tid;
    // rows of G are strided (column-major): thread = row, loop over K
    auto load = [&](StageRegs& R, int st) {
        const int kBase = kb + st * kStageK;
#pragma unroll
        for (int kc = 0; kc < kStageK; ++kc) {
            const int kk = kBase + kc;
            R.a[kc] = (r < M && kk < ke) ? LdgC32(f.G + r + kk * ld) : mk<float>(0, 0);
        }
#pragma unroll
        for (int j = 0; j < kBPerThread; ++j) {
            const int e = tid + j * kTcThreads;
            const int kk = kBase + e / kSweepCols, n = e % kSweepCols;
            c32 b = mk<float>(0, 0);
            if (kk < ke && n < ncol) {
                const c32* src = f.Rb + (int64_t)kk * 3 * k + t.col0 + n;
                b = src[0] + src[k] + src[2 * k];
            }
            R.b[j] = b;
        }
    };
    StageRegs cur, nxt;
    if (nst > 0) load(cur, 0);
    for (int st = 0; st < nst; ++st) {
        const int buf = st & 1;
        if (st >= kStages && !umma::MbarWaitBounded(&mbar[buf], ((st >> 1) - 1) & 1, work.status)) ok = false;
        if (__syncthreads_or(!ok)) { ok = false; break; }
        unsigned char* S = smem + buf * kStageBytes;
        StoreStage(S, cur, false);
        if (st + 1 < nst) load(nxt, st + 1);
        umma::FenceProxyAsync();
        __syncthreads();
        if (tid == 0) {
            umma::FenceAfterSync();
            IssueStage(S, tmem, st == 0);
            umma::CommitTo(&mbar[buf]);
        }
        cur = nxt;
    }
    c32 acc[kSweepCols];
    if (!TcFinish(mbar, tmem, nst, ok, work.status, acc)) return;
    if (!ReduceSplitsTc(t, work, acc)) return;
    if (r >= M) return;
    if (r < f.s) {
        c32* dst = f.Y + (int64_t)r * k + t.col0;
#pragma unroll
        for (int n = 0; n < kSweepCols; ++n)
            if (n < ncol) dst[n] = acc[n];
    } else if (f.parentRb) {
        const c32* src = f.Rb + (int64_t)r * 3 * k + t.col0;
        c32* dst = f.parentRb + ((int64_t)f.rel[r - f.s] * 3 + 1 + f.childSlot) * k + t.col0;
#pragma unroll
        for (int n = 0; n < kSweepCols; ++n)
            if (n < ncol) dst[n] = acc[n] + src[n] + src[k + n] + src[2 * k + n];
    }
}

__global__ void __launch_bounds__(kTcThreads) sweep_tc_backward_kernel(const SweepFront<float>* __restrict__ fr,
                                                                       const SweepTile* __restrict__ tiles,
                                                                       z64* __restrict__ B, int k, PanelIO io,
                                                                       SweepWork work) {
    extern __shared__ unsigned char smem_raw[];
    __shared__ uint64_t mbar[kStages + 1];
    __shared__ uint32_t tmemSlot;
    unsigned char* smem = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    c32* X = reinterpret_cast<c32*>(work.xnd);
    const SweepTile t = tiles[blockIdx.x];
    const SweepFront<float> f = fr[t.front];
    const int tid = threadIdx.x;
    const int64_t ld = f.s + f.u;
    const int ncol = min(kSweepCols, k - t.col0);
    const int kb = max(t.k0, t.row0), ke = t.k1;  // G^T is upper triangular in its first s columns
    const int nst = ke > kb ? (ke - kb + kStageK - 1) / kStageK : 0;
    const uint32_t tmem = TcSetup(mbar, &tmemSlot);
    bool ok = true;
    // rows of G^T are contiguous: consecutive threads read consecutive K
    auto load = [&](StageRegs& R, int st) {
        const int kBase = kb + st * kStageK;
#pragma unroll
        for (int i = 0; i < kStageK; ++i) {
            const int e = tid + i * kTcThreads;
            const int rr = t.row0 + e / kStageK, kk = kBase + e % kStageK;
            R.a[i] = (rr < f.s && kk < ke) ? LdgC32(f.G + kk + rr * ld) : mk<float>(0, 0);
        }
#pragma unroll
        for (int j = 0; j < kBPerThread; ++j) {
            const int e = tid + j * kTcThreads;
            const int kk = kBase + e / kSweepCols, n = e % kSweepCols;
            R.b[j] = (kk < ke && n < ncol) ? f.Z[(int64_t)kk * k + t.col0 + n] : mk<float>(0, 0);
        }
    };
    StageRegs cur, nxt;
    if (nst > 0) load(cur, 0);
    for (int st = 0; st < nst; ++st) {
        const int buf = st & 1;
        if (st >= kStages && !umma::MbarWaitBounded(&mbar[buf], ((st >> 1) - 1) & 1, work.status)) ok = false;
        if (__syncthreads_or(!ok)) { ok = false; break; }
        unsigned char* S = smem + buf * kStageBytes;
        StoreStage(S, cur, true);
        if (st + 1 < nst) load(nxt, st + 1);
        umma::FenceProxyAsync();
        __syncthreads();
        if (tid == 0) {
            umma::FenceAfterSync();
            IssueStage(S, tmem, st == 0);
            umma::CommitTo(&mbar[buf]);
        }
        cur = nxt;
    }
    c32 acc[kSweepCols];
    if (!TcFinish(mbar, tmem, nst, ok, work.status, acc)) return;
    if (!ReduceSplitsTc(t, work, acc)) return;
    const int r = t.row0 + tid;
    if (r >= f.s) return;
    const int col = f.ndOff + r;
    c32* xd = X + (int64_t)col * k + t.col0;
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

constexpr size_t kTcSmem = kStages * kStageBytes + 1024;

}  // namespace

void PrepareSweepTcKernels() {
    CUDA_CHECK(cudaFuncSetAttribute(sweep_tc_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)kTcSmem));
    CUDA_CHECK(cudaFuncSetAttribute(sweep_tc_backward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)kTcSmem));
}

void LaunchSweepForwardTc(const SweepFront<float>* fr, const SweepTile* tiles, int n, int k, const SweepWork& w,
                          cudaStream_t st) {
    if (n <= 0) return;
    sweep_tc_forward_kernel<<<n, kTcThreads, kTcSmem, st>>>(fr, tiles, k, w);
    CUDA_LAUNCH_CHECK();
}

void LaunchSweepBackwardTc(const SweepFront<float>* fr, const SweepTile* tiles, int n, z64* B, int k,
                           const PanelIO& io, const SweepWork& w, cudaStream_t st) {
    if (n <= 0) return;
    sweep_tc_backward_kernel<<<n, kTcThreads, kTcSmem, st>>>(fr, tiles, B, k, io, w);
    CUDA_LAUNCH_CHECK();
}

}  // namespace psp_b200
