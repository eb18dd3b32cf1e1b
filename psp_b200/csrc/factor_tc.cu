// Tensor-core (tcgen05) form of the factorization's batched complex-single
// GEMM, with gemm_kernel's semantics (kernels.cu) for real alpha and beta:
//   C = alpha op(A) diag(d) op(B) + beta C over a list of output tiles,
//   only r >= c when lowerC, the K range narrowed by the structural-zero
//   flags (entries inside the range are read as stored).
//
// As in sweep_tc.cu, the complex product is one real product (A's rows as
// interleaved (re, im) pairs, every B entry a 2x2 real block) and both
// operands are split into tf32 head and tail; per 8-value K step
//   A_hi B_hi + A_hi B_lo + A_lo B_hi   (three N = 128 MMAs, one accumulator)
// about FP32 accuracy.  A's split stage lives in tensor memory (the MMA
// reads A from TMEM), so only B's planes take shared memory.
//
// Persistent and warp-specialized: CTA b takes tiles b, b + grid, ... (each
// a 128 x 64 complex block described by one GemmTcTile record) and streams
// their K stages (8 complex columns) through three roles:
//   converters (8 warps)  asynchronous copies of operand stages into a
//                         kRaw-slot ring kAhead stages ahead (zero-filled
//                         outside the operands, any transposition), then the
//                         split: A into TMEM (one lane per row), B into
//                         one of two 64-byte-swizzled plane sets (d scales
//                         B's rows here);
//   MMA (one thread)      the split MMAs of a stage into one of two
//                         128-column TMEM accumulators; stage flags mark
//                         a tile's first and last stage;
//   epilogue (4 warps)    one accumulator row per thread: alpha acc + beta C,
//                         C staged in shared memory by copies issued while
//                         the tile's MMAs run; coalesced column stores.
// Every wait is bounded; a timeout sets the value 2 in the status word and
// ends all roles, leaving unfinished tiles unwritten.
#include <climits>

#include "kernels.cuh"
#include "umma.cuh"

namespace psp_b200 {

namespace {

constexpr int kBM = kGemmTcRows, kBN = kGemmTcCols;
constexpr int kSK = 8;  // complex K per stage: one 64-byte plane row
constexpr int kEpiThreads = 128, kConvThreads = 256;
constexpr int kConv0 = kEpiThreads, kMma0 = kConv0 + kConvThreads;
constexpr int kFThreads = kMma0 + 32;
constexpr int kRaw = 6, kAhead = kRaw - 1;  // raw slots; stages in flight ahead of the conversion
constexpr int kPlaneSets = 2, kAccs = 2;

constexpr uint32_t kBPl = 2 * kBN * 64;  // 8 KB: B' has 2 kBN rows of 16 tf32
constexpr uint32_t kPlSet = 2 * kBPl;     // B hi, B lo
// TMEM columns: two accumulators of 2 kBN columns, then per plane set the
// split A stage (head, then tail: 2 kSK columns each, lane = row)
constexpr uint32_t kAccCols = 2 * kBN;
constexpr uint32_t kACol0 = kAccs * kAccCols;
constexpr uint32_t kACols = 2 * kSK;
__host__ __device__ constexpr uint32_t ACol(int p) { return kACol0 + (uint32_t)p * 2 * kACols; }

constexpr int kApad = kBM + 1, kBpad = kBN + 1;  // raw A [kc][row], raw B [kc][col]
constexpr uint32_t kRawA = kSK * kApad * 8, kRawB = kSK * kBpad * 8;
constexpr uint32_t kRawSlot = kRawA + kRawB + kSK * 8;  // + d
constexpr uint32_t kRawOff = kPlaneSets * kPlSet;
constexpr uint32_t kStageOff = kRawOff + kRaw * kRawSlot;  // C staging [col][row]
constexpr size_t kFactorTcSmem = kStageOff + (size_t)kBN * kBM * 8 + 1024;
constexpr uint32_t kTmemCols = 512;
constexpr uint32_t kIdesc = umma::InstrDescTf32(kBM, 2 * kBN);
constexpr int kFirst = 1, kLast = 2;  // stage flags: a tile's first and last stage
// The tensor core adds each MMA's products into its FP32 accumulator with
// truncation, so an accumulator holds at most kChainStages stages (64
// complex K); the epilogue sums a tile's chains in FP32 (round to nearest)
// in a TMEM sum region and adds the last chain on the way out.
constexpr int kChainStages = 8;
constexpr int kChainFirst = 4, kChainLast = 8;  // stage flags: a chain's first and last stage
constexpr uint32_t kSumCol = ACol(kPlaneSets);   // 2 kBN columns

static_assert(kRawSlot % 16 == 0 && kStageOff % 16 == 0, "copy targets stay 16-byte aligned");
static_assert(kPlSet % 1024 == 0 && kBPl % 512 == 0, "swizzle atoms stay aligned");
static_assert(kSumCol + kAccCols <= kTmemCols, "accumulators, A stages and the chain sum fit in TMEM");
static_assert(kFactorTcSmem <= 232448, "shared memory per CTA");
static_assert(kConvThreads == 2 * kBM && kConvThreads == 4 * kBN, "converter thread mapping");

struct Sync {
    uint64_t planeFull[kPlaneSets], planeEmpty[kPlaneSets];
    uint64_t accFull[kAccs], accEmpty[kAccs];
    uint64_t mmaDrain;           // the MMA thread's last commit when a role gave up
    int rawFlags[kRaw];          // written and read by converter thread 0
    int planeFlags[kPlaneSets];  // converter thread 0 -> MMA thread
    uint32_t tmem;
    int abort;
};

// Bounded wait (umma::kWaitLimitNs); false once this or another role gave up.
__device__ __forceinline__ bool Wait(uint64_t* mbar, uint32_t parity, Sync& S, int* status) {
    if (umma::MbarTryWait(mbar, parity)) return true;
    const uint64_t t0 = umma::GlobalTimerNs();
    for (;;) {
        if (umma::MbarTryWait(mbar, parity)) return true;
        if (*reinterpret_cast<volatile int*>(&S.abort)) return false;
        if (umma::GlobalTimerNs() - t0 > umma::kWaitLimitNs) break;
    }
    *reinterpret_cast<volatile int*>(&S.abort) = 1;
    atomicOr(status, 2);
    return false;
}

// An empty K range still takes one zero-filled stage, so every tile produces
// an accumulator.
__device__ __forceinline__ int StagesOf(const GemmTcTile& t) { return t.nk > 0 ? (t.nk + kSK - 1) / kSK : 1; }

__device__ __forceinline__ void Split2(c32 x, float2& hi, float2& lo) {
    umma::SplitTf32Fast(x.re, hi.x, lo.x);
    umma::SplitTf32Fast(x.im, hi.y, lo.y);
}

// ------------------------------------------------------------------ converters

// This thread's copies of stage st of tile T into raw slot `raw`.
__device__ __forceinline__ void IssueStage(const GemmTcTile& T, int st, unsigned char* raw, int ct) {
    const int kBase = st * kSK;
    const bool tA = T.flags & 1, tB = T.flags & 2;
    c32* ra = reinterpret_cast<c32*>(raw);
    c32* rb = reinterpret_cast<c32*>(raw + kRawA);
    c32* rd = reinterpret_cast<c32*>(raw + kRawA + kRawB);
#pragma unroll
    for (int i = 0; i < kSK * kBM / kConvThreads; ++i) {
        const int e = ct + i * kConvThreads;
        const int r = tA ? e / kSK : e % kBM;
        const int kc = tA ? e % kSK : e / kBM;
        const int k = kBase + kc;
        const bool ok = r < T.m && k < T.nk;
        const c32* src = tA ? T.A + k + (int64_t)r * T.lda : T.A + r + (int64_t)k * T.lda;
        umma::CpAsync8(ra + kc * kApad + r, ok ? src : T.A, ok ? 8u : 0u);
    }
#pragma unroll
    for (int i = 0; i < kSK * kBN / kConvThreads; ++i) {
        const int e = ct + i * kConvThreads;
        const int c = tB ? e % kBN : e / kSK;
        const int kc = tB ? e / kBN : e % kSK;
        const int k = kBase + kc;
        const bool ok = c < T.n && k < T.nk;
        const c32* src = tB ? T.B + c + (int64_t)k * T.ldb : T.B + k + (int64_t)c * T.ldb;
        umma::CpAsync8(rb + kc * kBpad + c, ok ? src : T.B, ok ? 8u : 0u);
    }
    if (ct < kSK) {
        if (T.d) {
            const bool ok = kBase + ct < T.nk;
            umma::CpAsync8(rd + ct, ok ? T.d + kBase + ct : T.d, ok ? 8u : 0u);
        } else {
            rd[ct] = mk(1.f, 0.f);
        }
    }
}

// Splits raw slot `raw` into plane set P.  A: thread = row, 2 chunks (4
// complex K).  B: thread = (column c, chunk q): rows 2c, 2c+1 of B' hold the
// 2x2 real blocks of complex K 2q, 2q+1; the first of the two stores goes to
// row 2c or 2c+1 by bit 2 of c, so each store wave covers all banks.
__device__ __forceinline__ void ConvertStage(const unsigned char* raw, unsigned char* P, uint32_t tmemA, int ct) {
    const c32* ra = reinterpret_cast<const c32*>(raw);
    const c32* rb = reinterpret_cast<const c32*>(raw + kRawA);
    const c32* rd = reinterpret_cast<const c32*>(raw + kRawA + kRawB);
    {
        // row = this warp's TMEM lane quarter + lane; half h of the stage's K
        const int row = ct & (kBM - 1), h = ct / kBM;
        float hi[8], lo[8];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            float2 hv, lv;
            Split2(ra[(4 * h + j) * kApad + row], hv, lv);
            hi[2 * j] = hv.x;
            hi[2 * j + 1] = hv.y;
            lo[2 * j] = lv.x;
            lo[2 * j + 1] = lv.y;
        }
        const uint32_t at = tmemA + ((uint32_t)(row & ~31) << 16) + 8 * h;
        umma::TmemStore8(at, hi);
        umma::TmemStore8(at + kACols, lo);
    }
    {
        unsigned char* bHi = P;
        unsigned char* bLo = bHi + kBPl;
        const int c = ct >> 2, q = ct & 3;
        const c32 b0 = rb[(2 * q) * kBpad + c] * rd[2 * q];
        const c32 b1 = rb[(2 * q + 1) * kBpad + c] * rd[2 * q + 1];
        float2 h0, l0, h1, l1;
        Split2(b0, h0, l0);
        Split2(b1, h1, l1);
        const float4 hr = make_float4(h0.x, -h0.y, h1.x, -h1.y), hi = make_float4(h0.y, h0.x, h1.y, h1.x);
        const float4 lr = make_float4(l0.x, -l0.y, l1.x, -l1.y), li = make_float4(l0.y, l0.x, l1.y, l1.x);
        const uint32_t o0 = umma::Sw64Offset(2 * c, q), o1 = umma::Sw64Offset(2 * c + 1, q);
        if ((c >> 2) & 1) {
            *reinterpret_cast<float4*>(bHi + o1) = hi;
            *reinterpret_cast<float4*>(bHi + o0) = hr;
            *reinterpret_cast<float4*>(bLo + o1) = li;
            *reinterpret_cast<float4*>(bLo + o0) = lr;
        } else {
            *reinterpret_cast<float4*>(bHi + o0) = hr;
            *reinterpret_cast<float4*>(bHi + o1) = hi;
            *reinterpret_cast<float4*>(bLo + o0) = lr;
            *reinterpret_cast<float4*>(bLo + o1) = li;
        }
    }
}

__device__ void ConverterRole(const GemmTcTile* tiles, int n, unsigned char* smem, Sync& S, int* status) {
    const int ct = threadIdx.x - kConv0;
    const int G = gridDim.x;
    unsigned char* raw = smem + kRawOff;
    // load cursor: tile t (record cur), stage st of nst; the next record is
    // read a tile ahead
    int t = blockIdx.x, st = 0;
    bool more = t < n;
    GemmTcTile cur, nxt;
    if (more) cur = tiles[t];
    if (t + G < n) nxt = tiles[t + G];
    int nst = more ? StagesOf(cur) : 0;
    int issued = 0;
    // one committed copy group per stage slot, empty past the stream's end
    auto issueNext = [&]() {
        if (more) {
            const int slot = issued % kRaw;
            IssueStage(cur, st, raw + slot * kRawSlot, ct);
            if (ct == 0)
                S.rawFlags[slot] = (st == 0 ? kFirst : 0) | (st == nst - 1 ? kLast : 0) |
                                   (st % kChainStages == 0 ? kChainFirst : 0) |
                                   (st % kChainStages == kChainStages - 1 || st == nst - 1 ? kChainLast : 0);
            ++issued;
            if (++st == nst) {
                t += G;
                st = 0;
                more = t < n;
                if (more) {
                    cur = nxt;
                    nst = StagesOf(cur);
                    if (t + G < n) nxt = tiles[t + G];
                }
            }
        }
        umma::CpAsyncCommit();
    };
    for (int i = 0; i < kAhead; ++i) issueNext();
    for (int g = 0; g < issued; ++g) {
        const int p = g % kPlaneSets;
        umma::CpAsyncWait<kAhead - 1>();
        bool ok = true;
        if (ct == 0 && g >= kPlaneSets) ok = Wait(&S.planeEmpty[p], ((g / kPlaneSets) - 1) & 1, S, status);
        // stage g's copies are visible to every converter, stage g-1's slot
        // is free, and plane set p is free (its MMAs completed)
        if (umma::NamedBarrierOr(1, kConvThreads, !ok)) break;
        const int slot = g % kRaw;
        if (ct == 0) S.planeFlags[p] = S.rawFlags[slot];
        issueNext();
        ConvertStage(raw + slot * kRawSlot, smem + p * kPlSet, S.tmem + ACol(p), ct);
        umma::TmemStoreWait();
        umma::FenceProxyAsync();
        umma::FenceBeforeSync();
        umma::MbarArrive(&S.planeFull[p]);
    }
    umma::CpAsyncWaitAll();
}

// ------------------------------------------------------------------ MMA

__device__ void MmaRole(int n, unsigned char* smem, Sync& S, int* status) {
    const int G = gridDim.x;
    const int ntiles = (int)blockIdx.x < n ? (n - (int)blockIdx.x + G - 1) / G : 0;
    int g = 0, q = 0;  // stages and chains issued
    for (int i = 0; i < ntiles; ++g) {
        const int p = g % kPlaneSets, a = q % kAccs;
        if (!Wait(&S.planeFull[p], (g / kPlaneSets) & 1, S, status)) return;
        const int flags = *reinterpret_cast<volatile int*>(&S.planeFlags[p]);
        const bool first = flags & kChainFirst;
        if (first && q >= kAccs && !Wait(&S.accEmpty[a], ((q / kAccs) - 1) & 1, S, status)) return;
        umma::FenceAfterSync();
        const uint32_t acc = S.tmem + a * kAccCols, aHi = S.tmem + ACol(p), aLo = aHi + kACols;
        const uint32_t bHi = umma::SmemAddr(smem + p * kPlSet), bLo = bHi + kBPl;
#pragma unroll
        for (int s = 0; s < 2 * kSK / 8; ++s) {
            const uint64_t bh = umma::SmemDescSw64(bHi + 32 * s), bl = umma::SmemDescSw64(bLo + 32 * s);
            umma::MmaTf32TmemA(acc, aHi + 8 * s, bh, kIdesc, (first && s == 0) ? 0u : 1u);
            umma::MmaTf32TmemA(acc, aHi + 8 * s, bl, kIdesc, 1u);
            umma::MmaTf32TmemA(acc, aLo + 8 * s, bh, kIdesc, 1u);
        }
        umma::CommitTo(&S.planeEmpty[p]);
        if (flags & kChainLast) {
            umma::CommitTo(&S.accFull[a]);
            ++q;
        }
        if (flags & kLast) ++i;
    }
}

// ------------------------------------------------------------------ epilogue

// This thread's copies of its row of the C tile into the staging tile
// ([col][row]), where the tile writes and beta is nonzero.
__device__ __forceinline__ void IssueC(const GemmTcTile& T, c32* stage) {
    const int r = threadIdx.x;
    if (T.beta == 0.f || r >= T.m) return;
    const int ncol = min(T.n, r - T.diag + 1);  // r - c >= diag
    const c32* src = T.C + r;
    for (int c = 0; c < ncol; ++c, src += T.ldc) umma::CpAsync8(stage + c * kBM + r, src, 8u);
}

// alpha acc + beta C for this thread's row of 16 columns from column j0.
template <bool kFull>
__device__ __forceinline__ void StoreCols(const GemmTcTile& T, const float (&v)[32], const c32* stage, int j0) {
    const int r = threadIdx.x;
    c32* dst = T.C + r + (int64_t)j0 * T.ldc;
    const float al = T.alpha, be = T.beta;
#pragma unroll
    for (int q = 0; q < 16; ++q, dst += T.ldc) {
        const int c = j0 + q;
        if (!kFull && (r >= T.m || c >= T.n || r - c < T.diag)) continue;
        c32 out = mk(al * v[2 * q], al * v[2 * q + 1]);
        if (be != 0.f) {
            const c32 cv = stage[c * kBM + r];
            out.re = fmaf(be, cv.re, out.re);
            out.im = fmaf(be, cv.im, out.im);
        }
        *dst = out;
    }
}

__device__ void EpilogueRole(const GemmTcTile* tiles, int n, c32* stage, Sync& S, int* status) {
    const int tid = threadIdx.x, warp = tid / 32;
    const int G = gridDim.x;
    const uint32_t lane = (uint32_t)(warp * 32) << 16;
    GemmTcTile cur;
    if ((int)blockIdx.x < n) {
        cur = tiles[blockIdx.x];
        IssueC(cur, stage);
    }
    umma::CpAsyncCommit();
    const uint32_t tsum = S.tmem + lane + kSumCol;
    int q = 0;  // chains drained
    for (int t = blockIdx.x; t < n; t += G) {
        GemmTcTile nxt;
        if (t + G < n) nxt = tiles[t + G];
        // every chain but the last goes into the sum region; every epilogue
        // thread takes the same branches (they share named barriers)
        const int nch = (StagesOf(cur) + kChainStages - 1) / kChainStages;
        bool quit = false;  // the same on every epilogue thread
        for (int c = 0; c + 1 < nch && !quit; ++c, ++q) {
            const int a = q % kAccs;
            const bool ok = Wait(&S.accFull[a], (q / kAccs) & 1, S, status);
            quit = umma::NamedBarrierOr(2, kEpiThreads, !ok);
            if (quit) break;
            umma::FenceAfterSync();
            const uint32_t acc = S.tmem + lane + a * kAccCols;
#pragma unroll 1
            for (int j = 0; j < kBN / 16; ++j) {
                float v[32];
                umma::TmemLoad32(acc + 32 * j, v);
                if (c > 0) {
                    float w[32];
                    umma::TmemLoad32(tsum + 32 * j, w);
#pragma unroll
                    for (int e = 0; e < 32; ++e) v[e] += w[e];
                }
                umma::TmemStore32NoWait(tsum + 32 * j, v);
            }
            umma::TmemStoreWait();
            umma::FenceBeforeSync();
            umma::MbarArrive(&S.accEmpty[a]);
        }
        if (quit) break;
        const int a = q % kAccs;
        const bool ok = Wait(&S.accFull[a], (q / kAccs) & 1, S, status);
        ++q;
        umma::CpAsyncWaitAll();
        if (umma::NamedBarrierOr(2, kEpiThreads, !ok)) break;  // the staged C is visible
        umma::FenceAfterSync();
        const bool full = cur.m == kBM && cur.n == kBN && cur.diag <= 1 - kBN;
        const uint32_t acc = S.tmem + lane + a * kAccCols;
#pragma unroll 1
        for (int j = 0; j < kBN / 16; ++j) {
            float v[32];
            umma::TmemLoad32(acc + 32 * j, v);
            if (nch > 1) {
                float w[32];
                umma::TmemLoad32(tsum + 32 * j, w);
#pragma unroll
                for (int e = 0; e < 32; ++e) v[e] += w[e];
            }
            if (full)
                StoreCols<true>(cur, v, stage, 16 * j);
            else
                StoreCols<false>(cur, v, stage, 16 * j);
        }
        umma::FenceBeforeSync();
        umma::MbarArrive(&S.accEmpty[a]);
        umma::NamedBarrier(2, kEpiThreads);  // the staging tile is rewritten next
        if (t + G < n) {
            cur = nxt;
            IssueC(cur, stage);
        }
        umma::CpAsyncCommit();
    }
    umma::CpAsyncWaitAll();
}

// ------------------------------------------------------------------ kernel

__global__ void __launch_bounds__(kFThreads, 1)
    factor_gemm_tc_kernel(const GemmTcTile* __restrict__ tiles, int n, int* status) {
    extern __shared__ unsigned char smem_raw[];
    __shared__ Sync S;
    unsigned char* smem = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int i = 0; i < kPlaneSets; ++i) {
            umma::MbarInit(&S.planeFull[i], kConvThreads);
            umma::MbarInit(&S.planeEmpty[i], 1);
        }
        for (int i = 0; i < kAccs; ++i) {
            umma::MbarInit(&S.accFull[i], 1);
            umma::MbarInit(&S.accEmpty[i], kEpiThreads);
        }
        umma::MbarInit(&S.mmaDrain, 1);
        S.abort = 0;
        umma::FenceMbarInit();
    }
    if (tid / 32 == 0) umma::TmemAlloc(&S.tmem, kTmemCols);
    umma::FenceBeforeSync();
    __syncthreads();
    umma::FenceAfterSync();
    if (tid < kConv0) {
        EpilogueRole(tiles, n, reinterpret_cast<c32*>(smem + kStageOff), S, status);
    } else if (tid < kMma0) {
        ConverterRole(tiles, n, smem, S, status);
    } else if (tid == kMma0) {
        MmaRole(n, smem, S, status);
    }
    umma::FenceBeforeSync();
    __syncthreads();
    // when a role gave up, the MMA thread waits (bounded) for the tensor-core
    // operations it issued before tensor memory is freed (S.abort is no
    // longer written, so every thread takes the same branch; the converters
    // have waited for their own copies)
    if (*reinterpret_cast<volatile int*>(&S.abort)) {
        if (tid == kMma0) {
            umma::CommitTo(&S.mmaDrain);
            umma::MbarWaitBounded(&S.mmaDrain, 0, nullptr);
        }
        umma::FenceBeforeSync();
        __syncthreads();
    }
    if (tid / 32 == 0) {
        umma::FenceAfterSync();
        umma::TmemDealloc(S.tmem, kTmemCols);
    }
}

int g_factorSMs = 0;

}  // namespace

bool GemmTcEligible(const GemmOp<float>& op) { return op.alpha_im == 0.f && op.beta_im == 0.f; }

void PrepareFactorTcKernels() {
    CUDA_CHECK(cudaFuncSetAttribute(factor_gemm_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)kFactorTcSmem));
    int dev = 0;
    CUDA_CHECK(cudaGetDevice(&dev));
    CUDA_CHECK(cudaDeviceGetAttribute(&g_factorSMs, cudaDevAttrMultiProcessorCount, dev));
}

void AppendGemmTilesTc(const GemmOp<float>& op, std::vector<GemmTcTile>& tiles) {
    if (op.M <= 0 || op.N <= 0) return;
    const int tmN = (op.M + kBM - 1) / kBM, tnN = (op.N + kBN - 1) / kBN;
    for (int tn = 0; tn < tnN; ++tn)
        for (int tm = 0; tm < tmN; ++tm) {
            const int row0 = tm * kBM, col0 = tn * kBN;
            if (op.lowerC && row0 + kBM - 1 < col0) continue;
            // K range of the tile (gemm_kernel's structural-zero rules)
            int kb = 0, ke = op.K;
            if (op.triA == 1) ke = std::min(ke, row0 + kBM);
            if (op.triA == 2) kb = std::max(kb, row0);
            if (op.triB == 1) kb = std::max(kb, col0);
            if (op.triB == 2) ke = std::min(ke, col0 + kBN);
            GemmTcTile t;
            t.A = op.transA ? op.A + kb + (int64_t)row0 * op.lda : op.A + row0 + (int64_t)kb * op.lda;
            t.B = op.transB ? op.B + col0 + (int64_t)kb * op.ldb : op.B + kb + (int64_t)col0 * op.ldb;
            t.d = op.d ? op.d + kb : nullptr;
            t.C = op.C + row0 + (int64_t)col0 * op.ldc;
            t.lda = (int)op.lda;
            t.ldb = (int)op.ldb;
            t.ldc = (int)op.ldc;
            t.m = std::min(kBM, op.M - row0);
            t.n = std::min(kBN, op.N - col0);
            t.nk = std::max(0, ke - kb);
            t.diag = op.lowerC ? col0 - row0 : INT_MIN / 2;
            t.flags = (op.transA ? 1 : 0) | (op.transB ? 2 : 0);
            t.alpha = op.alpha_re;
            t.beta = op.beta_re;
            tiles.push_back(t);
        }
}

void LaunchGemmTc(const GemmTcTile* tiles, int numTiles, int* status, cudaStream_t st) {
    if (numTiles <= 0) return;
    const int grid = numTiles < g_factorSMs ? numTiles : g_factorSMs;
    factor_gemm_tc_kernel<<<grid, kFThreads, kFactorTcSmem, st>>>(tiles, numTiles, status);
    CUDA_LAUNCH_CHECK();
}

}  // namespace psp_b200
