// Tensor-core (tcgen05) versions of the sweep's frontal products for complex-
// single factors, with the same data flow as sweep.cu:
//   forward  [Y; U] = G R_s + [0; R_u]      backward  X_s = G^T [inv(D) Y; X_u]
//
// A complex product C = A B (A: rows x K, B: K x 16 right-hand sides) runs as
// one real product on the tensor core: A's rows read as interleaved
// (re, im) pairs form a rows x 2K real matrix, and every complex entry b of
// B becomes the 2x2 real block [[re b, im b], [-im b, re b]] of a 2K x 32
// real matrix, so the 2 NC real accumulator columns are C's interleaved
// (re, im) pairs.  Each operand is split into tf32 head and tail
// (x = hi + lo) and hi*hi + hi*lo + lo*hi is accumulated in FP32 in tensor
// memory (about FP32 accuracy from TF32 inputs) with two MMAs per 8-value K
// step: A_hi [B_hi | B_lo] (N = 4 NC) and A_lo B_hi (N = 2 NC, onto the first
// 2 NC columns); the epilogue adds the two halves.
//
// A tile is 128 rows (one UMMA M=128 accumulator) x NC right-hand sides
// (NC = 16, or 32 when a launch has more than 16: every G stage is then split
// once for twice the right-hand sides) over one K-chunk, consumed in stages
// of 16 complex K-columns.  The kernels are
// persistent (one CTA per SM walks the tiles blockIdx.x, blockIdx.x + grid,
// ...) and warp-specialized, with mbarriers between the roles:
//   producer (1 thread) one tiled TMA copy per stage of G's 128 x 16 box
//                       (forward) or G^T's (backward), from two tensor maps
//                       per front, into a ring of raw stages (completion by
//                       transaction bytes)
//   converters (8 warps) split raw stage g into tf32 head/tail: forward A
//                       into TMEM (the MMA reads A from tensor memory),
//                       backward A and both B's into 128-byte swizzled
//                       K-major planes (kPlaneSets buffers); each also
//                       copies its own right-hand-side entries kAhead
//                       stages ahead
//   MMA (1 thread)      tcgen05.mma per stage into one of kAccs TMEM
//                       accumulators (round robin by chain: a tile's stages
//                       in runs of kChainStages)
//   epilogue (4 warps)  TMEM -> registers: the chains of a tile summed in
//                       FP32, split-K reduction, and the result through
//                       shared memory so that its global accesses are
//                       coalesced; what the write-out reads from global
//                       memory is loaded before the accumulator is ready.
// Every wait on an mbarrier is bounded; a timeout sets bit 2 of the status
// word and a shared abort flag that ends every role's loop; the CTA then
// frees tensor memory and returns, leaving unfinished tiles unwritten.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "kernels.cuh"
#include "umma.cuh"

namespace psp_b200 {

namespace {

constexpr int kEpiWarps = 4, kLoadWarps = 8;
constexpr int kEpiThreads = 32 * kEpiWarps;
constexpr int kLoadThreads = 32 * kLoadWarps;
constexpr int kLoad0 = kEpiThreads;                   // first converter thread
constexpr int kMma0 = kLoad0 + kLoadThreads;          // the MMA thread
constexpr int kProd0 = kMma0 + 32;                    // the producer warp
constexpr int kTcThreads = kProd0 + 32;               // 448
constexpr int kGroups = 2;                            // converter groups, alternating stages
constexpr int kGroupThreads = kLoadThreads / kGroups; // 128

constexpr int kStageK = 16;                            // complex K per stage (one 128-byte swizzle row)
constexpr uint32_t kAPlane = kTcRows * 128;            // 16 KB
constexpr int kPlaneSets = kGroups;                    // one per converter group
// The forward kernel keeps each plane set's split A stage in TMEM after the
// accumulators (head then tail, 2 kStageK columns each, lane = row): the MMA
// reads A from tensor memory and only B's planes go through shared memory.
constexpr uint32_t kAStageCols = 2 * kStageK;
constexpr uint32_t kTmemCols = 512;
constexpr uint32_t kRawA = kStageK * kTcRows * 8;      // 16 KB
constexpr int kRawMax = 8;
constexpr int kAccMax = 4, kOwnMax = 3;
// The tensor core adds each MMA's products into its FP32 accumulator with
// truncation, so long accumulation chains in TMEM lose accuracy (a K-chunk of
// 512 columns left the large layered model's preconditioner 9e-5 away from
// FP32 CUDA-core arithmetic, and GMRES took 21 steps instead of 9).  Each
// accumulator therefore holds at most kChainStages stages (64 complex K);
// the epilogue sums the chains of a tile in FP32 (round to nearest) into a
// TMEM sum region, and adds the last chain on the way out.
constexpr int kChainStages = 4;

// The result passes through shared memory 16 right-hand sides (one sub-tile)
// at a time, with row stride kOutPad.
constexpr int kOutPad = kSweepCols + 1;
constexpr uint32_t kStaging = kTcRows * kOutPad * 8;
constexpr int kOutRowsPerPass = kEpiThreads / kSweepCols;  // 8
constexpr int kOutPerThread = kTcRows / kOutRowsPerPass;   // 16

// Shapes of the kernels with NC right-hand sides per tile.
//   B planes: 2 NC rows of B' (hi, then lo right after it).
//   Accumulators: 4 NC f32 columns each ([A_hi B_hi + A_lo B_hi | A_hi B_lo]),
//   kAccs of them (chains in flight per CTA), then the tile's chain sum
//   (2 NC columns).
//   Raw data of the stages in flight: A arrives by one tiled TMA copy per
//   stage into a ring of RawSlots(fwd) slots shared by both groups (forward
//   G's 128-row x 16-column box, [kc][row]; backward G^T's 128 x 16 box,
//   [row][kc]); the forward keeps A in TMEM, so its last four slots reuse
//   the A planes of the plane sets.  Each group has a ring of kOwn slots of
//   its own copies of B (forward [plane][kc][n], backward [kc][n]), every
//   entry read back by the thread that copied it (OwnEntry).
template <int NC>
struct Cfg {
    static constexpr int kCols = NC;
    static constexpr int kSubs = NC / kSweepCols;                    // 16-column sub-tiles
    static constexpr uint32_t kBPlane = 2 * NC * 128;
    static constexpr uint32_t kPlaneSet = 2 * kAPlane + 2 * kBPlane;  // A hi, A lo, B hi, B lo
    static constexpr uint32_t kAccCols = 4 * NC;
    static constexpr int kAccs = NC == 16 ? 4 : 2;
    static constexpr uint32_t kIdescHi = umma::InstrDescTf32(kTcRows, 4 * NC);
    static constexpr uint32_t kIdescLo = umma::InstrDescTf32(kTcRows, 2 * NC);
    static constexpr int kAheadOwn = NC == 16 ? 2 : 1;              // own stages in flight per group
    static constexpr int kOwn = kAheadOwn + 1;
    __host__ __device__ static constexpr int RawSlots(bool fwd) { return NC == 16 ? (fwd ? 8 : 6) : (fwd ? 7 : 5); }
    __host__ __device__ static constexpr int RawInRegion(bool fwd) {
        return NC == 16 ? (fwd ? 4 : 6) : (fwd ? 3 : 5);
    }
    __host__ __device__ static constexpr uint32_t OwnSlot(bool fwd) {
        return fwd ? 3 * kStageK * NC * 8 : kStageK * NC * 8;
    }
    __host__ __device__ static constexpr uint32_t OwnBase(bool fwd) { return RawInRegion(fwd) * kRawA; }
    __host__ __device__ static constexpr uint32_t RegionBytes(bool fwd) {
        return OwnBase(fwd) + kGroups * kOwn * OwnSlot(fwd);
    }
    static constexpr uint32_t kRegionOff = kPlaneSets * kPlaneSet;
    static constexpr uint32_t kRegion = RegionBytes(true) > RegionBytes(false) ? RegionBytes(true) : RegionBytes(false);
    static constexpr uint32_t kStagingOff = kRegionOff + kRegion;
    static constexpr size_t kSmem = kStagingOff + kStaging + 1024;
    __host__ __device__ static constexpr uint32_t ACol(int ps) {
        return kAccs * kAccCols + (uint32_t)ps * 2 * kAStageCols;
    }
    // the running sum of a tile's finished chains: NC complex per lane
    static constexpr uint32_t kSumCol = kAccs * kAccCols + kPlaneSets * 2 * kAStageCols;
    static_assert(RawSlots(true) - RawInRegion(true) == 2 * kPlaneSets && kRawA == kAPlane,
                  "the forward's extra raw slots are the plane sets' A planes");
    static_assert(RawSlots(true) <= kRawMax && RawSlots(false) <= kRawMax, "raw ring");
    static_assert(kAccs <= kAccMax && kOwn <= kOwnMax, "sync arrays");
    static_assert(kSumCol + 2 * NC <= kTmemCols, "accumulators, A stages and the chain sum fit in TMEM");
    static_assert(kSmem <= 232448, "shared memory per CTA");
};

// Raw A slot `slot` (shared-memory base `smem`, 1 KB aligned).
template <int NC, bool kFwd>
__device__ __forceinline__ unsigned char* RawSlotPtr(unsigned char* smem, int slot) {
    using C = Cfg<NC>;
    if (slot < C::RawInRegion(kFwd)) return smem + C::kRegionOff + slot * kRawA;
    const int e = slot - C::RawInRegion(kFwd);
    return smem + (e / 2) * C::kPlaneSet + (e % 2) * kAPlane;
}

// Stage description handed from the loaders to the MMA thread.
struct StageHdr {
    int valid, st, nst, j;
};

struct Sync {
    uint64_t planeFull[kPlaneSets], planeEmpty[kPlaneSets];
    uint64_t accFull[kAccMax], accEmpty[kAccMax];
    uint64_t rawFull[kRawMax], rawEmpty[kRawMax];
    uint64_t mmaDrain;           // the MMA thread's last commit when a role gave up
    StageHdr hdr[kPlaneSets];
    int ownInfo[kGroups][kOwnMax];  // stage place, packed (see InfoSt); written and read by a group's first thread
    int rawK[kRawMax][2];        // stage's first K index and the tile's K end
    uint32_t tmem;
    int abort;
    int isLast;
    int rawIssued;  // raw A copies the producer issued
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

__device__ __forceinline__ void TileRange(const SweepTile& t, bool fwd, int& kb, int& ke, int& nst) {
    // inv(L11) is lower triangular: the forward K range ends at the tile's
    // last row, the backward (G^T) range starts at its first
    kb = fwd ? t.k0 : max(t.k0, t.row0);
    ke = fwd ? min(t.k1, t.row0 + kTcRows) : t.k1;
    // an empty range still takes one (zero-filled) stage, so every tile
    // produces an accumulator
    nst = ke > kb ? (ke - kb + kStageK - 1) / kStageK : 1;
}

// Zero, or the entry at p when `pred`: a predicated load whose destination
// is not read until its consumer needs it, so several stay in flight.
__device__ __forceinline__ c32 LdgC32If(const c32* p, bool pred) {
    float x, y;
    asm volatile(
        "{\n\t.reg .pred q;\n\t"
        "setp.ne.b32 q, %3, 0;\n\t"
        "mov.f32 %0, 0f00000000;\n\t"
        "mov.f32 %1, 0f00000000;\n\t"
        "@q ld.global.nc.v2.f32 {%0, %1}, [%2];\n\t}\n"
        : "=f"(x), "=f"(y)
        : "l"(p), "r"((int)pred));
    return mk(x, y);
}

// ------------------------------------------------------------------ loaders

// A stage's place in the tile sequence, packed as
// (j << 20) | (nst << 10) | st.
__device__ __forceinline__ int InfoSt(int info) { return info & 1023; }
__device__ __forceinline__ int InfoNst(int info) { return (info >> 10) & 1023; }
__device__ __forceinline__ int InfoJ(int info) { return info >> 20; }

// Stages between fetching the next tile's descriptor and its front.
constexpr int kFrontLag = 2;

// What the copies of one tile need.
struct LoadMeta {
    const c32* G;
    const c32* B;  // forward: Rb; backward: Z
    const void* tmap;  // forward map of the front (the backward map follows it)
    int ld, rows, row0, col0, kb, ke, nst;
};

// Walks this CTA's (tile, stage) sequence.  The next tile's descriptor is
// fetched when a tile starts and its front a few stages later (once the
// descriptor has arrived), so that neither load stalls the copies.
template <bool kFwd>
struct LoadCursor {
    const SweepFront<float>* fr;
    const SweepTile* tiles;
    int n, k;
    int ti, st, j, gl, total;  // gl: stages issued; total: stages in all (-1 until known)
    LoadMeta m;
    int nFront, nRow0, nCol0, nK0, nK1;  // next tile
    const c32 *nG, *nB;                  // its front
    const void* nMap;
    int ns, nu, haveNt, haveNf;

    __device__ __forceinline__ void SetMeta(int row0, int col0, int k0, int k1, const c32* G, const c32* B, int s,
                                            int u, const void* tmap) {
        m.G = G;
        m.B = B;
        m.tmap = tmap;
        m.ld = GLeadingDim(s, u);
        m.rows = kFwd ? s + u : s;
        m.row0 = row0;
        m.col0 = col0;
        SweepTile t;
        t.row0 = row0; t.k0 = k0; t.k1 = k1;
        TileRange(t, kFwd, m.kb, m.ke, m.nst);
    }
    __device__ __forceinline__ void Start(const SweepFront<float>* fr_, const SweepTile* tiles_, int n_, int k_) {
        fr = fr_; tiles = tiles_; n = n_; k = k_;
        ti = blockIdx.x; j = 0; st = 0; gl = 0;
        total = ti >= n ? 0 : -1;
        haveNt = haveNf = 0;
        if (total == 0) return;
        const SweepTile t = tiles[ti];
        const SweepFront<float>& f = fr[t.front];
        SetMeta(t.row0, t.col0, t.k0, t.k1, f.G, kFwd ? f.Rb : f.Z, f.s, f.u, f.tmap);
        PrefetchTile();
    }
    __device__ __forceinline__ void PrefetchTile() {
        haveNt = ti + (int)gridDim.x < n;
        haveNf = 0;
        if (haveNt) {
            const SweepTile& t = tiles[ti + gridDim.x];
            nFront = t.front; nRow0 = t.row0; nCol0 = t.col0; nK0 = t.k0; nK1 = t.k1;
        }
    }
    __device__ __forceinline__ void PrefetchFront() {
        if (haveNt && !haveNf) {
            const SweepFront<float>& f = fr[nFront];
            nG = f.G;
            nB = kFwd ? f.Rb : f.Z;
            nMap = f.tmap;
            ns = f.s;
            nu = f.u;
            haveNf = 1;
        }
    }
    __device__ __forceinline__ bool Valid(int g) const { return total < 0 || g < total; }
    __device__ __forceinline__ int Info() const { return (j << 20) | (m.nst << 10) | st; }
    __device__ __forceinline__ int KBase() const { return m.kb + st * kStageK; }

    // Moves to the next stage.
    __device__ __forceinline__ void Advance() {
        ++gl;
        if (++st < m.nst) {
            if (st == kFrontLag) PrefetchFront();
            return;
        }
        ti += gridDim.x;
        ++j;
        st = 0;
        if (ti >= n) { total = gl; return; }
        PrefetchFront();
        SetMeta(nRow0, nCol0, nK0, nK1, nG, nB, ns, nu, nMap);
        PrefetchTile();
    }
};

// ------------------------------------------------------------------ producer

// Lane 0 of one warp copies each stage's A operand with one tiled TMA copy of
// the front's map: forward the 128-row x 16-column box of G at (row0,
// kBase), backward the 16 x 128 box of G at (kBase, row0), i.e. 128 rows of
// G^T.  Rows or columns outside G arrive as zeros; K columns past the tile's
// range are masked by the converters.
template <int NC, bool kFwd>
__device__ void ProducerRole(const SweepFront<float>* __restrict__ fr, const SweepTile* __restrict__ tiles, int n,
                             int k, unsigned char* smem, Sync& S, int* status) {
    using C = Cfg<NC>;
    if ((threadIdx.x & 31) != 0) return;
    LoadCursor<kFwd> cur;
    cur.Start(fr, tiles, n, k);
    int g = 0;
    for (; cur.Valid(g); ++g) {
        const int slot = g % C::RawSlots(kFwd);
        if (g >= C::RawSlots(kFwd) && !Wait(&S.rawEmpty[slot], ((g / C::RawSlots(kFwd)) - 1) & 1, S, status)) break;
        const LoadMeta& m = cur.m;
        const int kBase = cur.KBase();
        S.rawK[slot][0] = kBase;
        S.rawK[slot][1] = m.ke;
        umma::MbarArriveExpectTx(&S.rawFull[slot], kRawA);
        const unsigned char* map = reinterpret_cast<const unsigned char*>(m.tmap) + (kFwd ? 0 : 128);
        if (kFwd)
            umma::TmaLoad2D(RawSlotPtr<NC, kFwd>(smem, slot), map, m.row0, kBase, &S.rawFull[slot]);
        else
            umma::TmaLoad2D(RawSlotPtr<NC, kFwd>(smem, slot), map, kBase, m.row0, &S.rawFull[slot]);
        cur.Advance();
    }
    S.rawIssued = g;
}

// After a role gave up: waits (bounded) until the last copy into every raw
// slot has landed, so none is in flight when the CTA exits.  Copy g of the
// ring fills slot g % R in its phase g / R.
template <int NC, bool kFwd>
__device__ __forceinline__ void DrainRaw(Sync& S) {
    constexpr int R = Cfg<NC>::RawSlots(kFwd);
    const int G = S.rawIssued;
    for (int s = 0; s < R && s < G; ++s) umma::MbarWaitBounded(&S.rawFull[s], ((G - 1 - s) / R) & 1, nullptr);
}

// ------------------------------------------------------------------ converters

// Splits x into tf32 head and tail.
__device__ __forceinline__ void Split2(c32 x, float2& hi, float2& lo) {
    umma::SplitTf32Fast(x.re, hi.x, lo.x);
    umma::SplitTf32Fast(x.im, hi.y, lo.y);
}

// The right-hand-side entry (kc, nn) of a stage that converter thread ct
// copies and converts in its j-th slot: consecutive threads take
// consecutive columns, and columns 8-15 of every 16 take the neighbouring
// K row, so that a warp's B' stores use both 8-byte halves of a 16-byte
// chunk as well as all eight swizzle phases (two wavefronts per store, the
// least for 256 bytes); its copies still read whole 32-byte sectors.  The
// entry sits at kc NC + nn in the group's copy slot.
template <int NC>
__device__ __forceinline__ void OwnEntry(int ct, int j, int& kc, int& nn) {
    const int e = ct + j * kGroupThreads;
    nn = e % NC;
    kc = (e / NC) ^ ((nn >> 3) & 1);
}

// Issues this converter thread's own copies of the cursor's stage (its two
// B entries; backward also its eight 16-byte A chunks, zero-filled outside
// the tile), commits one copy group and moves the cursor to the group's
// next stage.
template <int NC, bool kFwd>
__device__ __forceinline__ void IssueOwn(LoadCursor<kFwd>& cur, unsigned char* own, int gr, Sync& S) {
    using C = Cfg<NC>;
    if (cur.total >= 0) {
        umma::CpAsyncCommit();
        return;
    }
    const int slot = (cur.gl / kGroups) % C::kOwn;
    const LoadMeta& m = cur.m;
    const int ct = (threadIdx.x - kLoad0) % kGroupThreads;
    if (ct == 0) S.ownInfo[gr][slot] = cur.Info();
    unsigned char* base = own + slot * C::OwnSlot(kFwd);
    c32* rb = reinterpret_cast<c32*>(base);
    const int ncol = min(NC, cur.k - m.col0);
    const int kBase = cur.KBase();
#pragma unroll
    for (int j = 0; j < kStageK * NC / kGroupThreads; ++j) {
        int kc, nn;
        OwnEntry<NC>(ct, j, kc, nn);
        const int e = kc * NC + nn;
        const int kk = kBase + kc;
        const bool ok = kk < m.ke && nn < ncol;
        if (kFwd) {
            const c32* src = m.B + (int64_t)kk * 3 * cur.k + m.col0 + nn;
#pragma unroll
            for (int p = 0; p < 3; ++p)
                umma::CpAsync8(rb + p * kStageK * NC + e, ok ? src + p * cur.k : m.B, ok ? 8u : 0u);
        } else {
            umma::CpAsync8(rb + e, ok ? m.B + (int64_t)kk * cur.k + m.col0 + nn : m.B, ok ? 8u : 0u);
        }
    }
    umma::CpAsyncCommit();
#pragma unroll
    for (int i = 0; i < kGroups; ++i) cur.Advance();
}

// Converts one raw stage into plane set P (thread ct of a group); forward
// K-columns at or beyond kValid are taken as zero.
template <int NC, bool kFwd>
__device__ __forceinline__ void ConvertStage(unsigned char* P, const unsigned char* rawA, const unsigned char* own,
                                             int kValid, int ct, uint32_t tmemA) {
    using C = Cfg<NC>;
    unsigned char* aHi = P;
    unsigned char* aLo = P + kAPlane;
    const c32 zero = mk<float>(0, 0);
    if (kFwd) {
        // thread ct = row = TMEM lane ct of this warp's lane quarter
        const c32* ra = reinterpret_cast<const c32*>(rawA);
        const int row = ct;
        float hi[2 * kStageK], lo[2 * kStageK];
#pragma unroll
        for (int kc = 0; kc < kStageK; ++kc) {
            float2 h, l;
            Split2(kc < kValid ? ra[kc * kTcRows + row] : zero, h, l);
            hi[2 * kc] = h.x;
            hi[2 * kc + 1] = h.y;
            lo[2 * kc] = l.x;
            lo[2 * kc + 1] = l.y;
        }
        const uint32_t at = tmemA + ((uint32_t)(row & ~31) << 16);
        umma::TmemStore32NoWait(at, hi);
        umma::TmemStore32NoWait(at + kAStageCols, lo);
    } else {
        // G^T rows from the raw ring ([row][kc]); K past the tile's range is zero
        const c32* ra = reinterpret_cast<const c32*>(rawA);
#pragma unroll
        for (int i = 0; i < kStageK * kTcRows / 2 / kGroupThreads; ++i) {
            const int c = ct + i * kGroupThreads;
            const int m = c / (kStageK / 2), q = c % (kStageK / 2);
            float2 h0, l0, h1, l1;
            Split2(2 * q < kValid ? ra[m * kStageK + 2 * q] : zero, h0, l0);
            Split2(2 * q + 1 < kValid ? ra[m * kStageK + 2 * q + 1] : zero, h1, l1);
            const uint32_t off = umma::Sw128Offset(m, q);
            *reinterpret_cast<float4*>(aHi + off) = make_float4(h0.x, h0.y, h1.x, h1.y);
            *reinterpret_cast<float4*>(aLo + off) = make_float4(l0.x, l0.y, l1.x, l1.y);
        }
    }
    // B: entry (kc, n) becomes rows 2n, 2n+1 of B' at K positions 2kc, 2kc+1
    const c32* rb = reinterpret_cast<const c32*>(own);
    unsigned char* bHi = P + 2 * kAPlane;
    unsigned char* bLo = bHi + C::kBPlane;
#pragma unroll
    for (int j = 0; j < kStageK * NC / kGroupThreads; ++j) {
        int kc, nn;
        OwnEntry<NC>(ct, j, kc, nn);
        const int e = kc * NC + nn;
        const c32 b = kFwd ? rb[e] + rb[kStageK * NC + e] + rb[2 * kStageK * NC + e] : rb[e];
        float2 h, l;
        Split2(b, h, l);
        const uint32_t o0 = umma::Sw128Offset(2 * nn, kc >> 1) + (kc & 1) * 8;
        const uint32_t o1 = umma::Sw128Offset(2 * nn + 1, kc >> 1) + (kc & 1) * 8;
        // lanes with bit 2 of n set store their odd row first, so each store
        // instruction covers all eight swizzle phases of a row group
        const bool odd = (nn >> 2) & 1;
        const float2 hr = make_float2(h.x, -h.y), hi = make_float2(h.y, h.x);
        const float2 lr = make_float2(l.x, -l.y), li = make_float2(l.y, l.x);
        *reinterpret_cast<float2*>(bHi + (odd ? o1 : o0)) = odd ? hi : hr;
        *reinterpret_cast<float2*>(bHi + (odd ? o0 : o1)) = odd ? hr : hi;
        *reinterpret_cast<float2*>(bLo + (odd ? o1 : o0)) = odd ? li : lr;
        *reinterpret_cast<float2*>(bLo + (odd ? o0 : o1)) = odd ? lr : li;
    }
}

// Converts stage g (a stage of this thread's group, plane set g % 2) or
// ends the stream; false when the role is done.
template <int NC, bool kFwd>
__device__ __forceinline__ bool ConverterStep(unsigned char* smem, unsigned char* own, const LoadCursor<kFwd>& cur,
                                              int g, int gr, int ct, Sync& S, int* status) {
    using C = Cfg<NC>;
    const int ps = gr, slot = g % C::RawSlots(kFwd), oslot = (g / kGroups) % C::kOwn;
    const bool valid = cur.Valid(g);
    if (valid && !Wait(&S.rawFull[slot], (g / C::RawSlots(kFwd)) & 1, S, status)) return false;
    if (g >= kGroups && !Wait(&S.planeEmpty[ps], ((g / kGroups) - 1) & 1, S, status)) return false;
    umma::CpAsyncWait<C::kAheadOwn>();  // this thread's own copies of stage g have landed
    if (valid) {
        const int kValid = S.rawK[slot][1] - S.rawK[slot][0];
        ConvertStage<NC, kFwd>(smem + ps * C::kPlaneSet, RawSlotPtr<NC, kFwd>(smem, slot),
                               own + oslot * C::OwnSlot(kFwd), kValid, ct, S.tmem + C::ACol(ps));
    }
    if (kFwd) {
        umma::TmemStoreWait();
        umma::FenceBeforeSync();
    }
    umma::FenceProxyAsync();
    if (ct == 0) {
        const int info = S.ownInfo[gr][oslot];
        S.hdr[ps] = valid ? StageHdr{1, InfoSt(info), InfoNst(info), InfoJ(info)} : StageHdr{0, 0, 0, 0};
    }
    umma::MbarArrive(&S.planeFull[ps]);
    if (valid) umma::MbarArrive(&S.rawEmpty[slot]);
    return valid;
}

template <int NC, bool kFwd>
__device__ void ConverterRole(const SweepFront<float>* __restrict__ fr, const SweepTile* __restrict__ tiles, int n,
                              int k, unsigned char* smem, Sync& S, int* status) {
    using C = Cfg<NC>;
    const int lt = threadIdx.x - kLoad0;
    const int gr = lt / kGroupThreads, ct = lt % kGroupThreads;
    unsigned char* own = smem + C::kRegionOff + C::OwnBase(kFwd) + gr * C::kOwn * C::OwnSlot(kFwd);
    LoadCursor<kFwd> cur;
    cur.Start(fr, tiles, n, k);
    for (int i = 0; i < gr; ++i) cur.Advance();
    PdlWait();  // right-hand sides come from the preceding kernels
#pragma unroll
    for (int a = 0; a < C::kAheadOwn; ++a) IssueOwn<NC>(cur, own, gr, S);
    for (int g = gr;; g += kGroups) {
        IssueOwn<NC>(cur, own, gr, S);
        if (!ConverterStep<NC, kFwd>(smem, own, cur, g, gr, ct, S, status)) break;
    }
    umma::CpAsyncWaitAll();
}

// ------------------------------------------------------------------ MMA

// `init`: accumulate onto the accumulator's contents (every stage of a tile
// but its first); otherwise the MMA overwrites it.
// Forward: A's split stage is read from TMEM at tmemA (head, then tail).
template <int NC, bool kFwd>
__device__ __forceinline__ void IssueStage(const unsigned char* P, uint32_t tmem, uint32_t tmemA, bool init) {
    using C = Cfg<NC>;
    const uint32_t aHi = umma::SmemAddr(P), aLo = aHi + kAPlane, bHi = aHi + 2 * kAPlane;
#pragma unroll
    for (int s = 0; s < 2 * kStageK / 8; ++s) {
        const uint32_t o = s * 32;
        const uint64_t bd = umma::SmemDescSw128(bHi + o);
        if (kFwd) {
            umma::MmaTf32TmemA(tmem, tmemA + 8 * s, bd, C::kIdescHi, (init || s > 0) ? 1u : 0u);
            umma::MmaTf32TmemA(tmem, tmemA + kAStageCols + 8 * s, bd, C::kIdescLo, 1u);
        } else {
            umma::MmaTf32(tmem, umma::SmemDescSw128(aHi + o), bd, C::kIdescHi, (init || s > 0) ? 1u : 0u);
            umma::MmaTf32(tmem, umma::SmemDescSw128(aLo + o), bd, C::kIdescLo, 1u);
        }
    }
}

// A tile's stages form chains of kChainStages; chain q (counted over the
// CTA's tiles) accumulates in accumulator q % kAccs.
__device__ __forceinline__ bool ChainFirst(int st) { return st % kChainStages == 0; }
__device__ __forceinline__ bool ChainLast(int st, int nst) { return st % kChainStages == kChainStages - 1 || st == nst - 1; }
__device__ __forceinline__ int NumChains(int nst) { return (nst + kChainStages - 1) / kChainStages; }

template <int NC, bool kFwd>
__device__ void MmaRole(const unsigned char* planes, Sync& S, int* status) {
    using C = Cfg<NC>;
    int q = 0;  // chains finished
    for (int g = 0;; ++g) {
        const int ps = g % kPlaneSets;
        if (!Wait(&S.planeFull[ps], (g / kPlaneSets) & 1, S, status)) return;
        const StageHdr h = S.hdr[ps];
        if (!h.valid) return;  // the epilogue counts its own tiles
        const int b = q % C::kAccs;
        const bool first = ChainFirst(h.st);
        if (first && !Wait(&S.accEmpty[b], (q / C::kAccs) & 1, S, status)) return;
        umma::FenceAfterSync();
        IssueStage<NC, kFwd>(planes + ps * C::kPlaneSet, S.tmem + b * C::kAccCols, S.tmem + C::ACol(ps), !first);
        umma::CommitTo(&S.planeEmpty[ps]);
        if (ChainLast(h.st, h.nst)) {
            umma::CommitTo(&S.accFull[b]);
            ++q;
        }
    }
}

// ------------------------------------------------------------------ epilogue

// Split-K over CTAs: partial tiles [slot][column][row]; the last CTA to arrive
// sums them in split order.  Epilogue threads only (named barrier 1).
__device__ __forceinline__ bool ReduceSplitsTc(const SweepTile& t, const SweepWork& w, Sync& S,
                                               c32 (&acc)[kSweepCols], int subs, int h) {
    if (t.nsplit <= 1) return true;
    c32* part = reinterpret_cast<c32*>(w.partials);
    const int row = threadIdx.x;
    const int counter = t.counter * subs + h;
    c32* mine = part + ((int64_t)((t.slot + t.split) * subs + h) * kSweepCols) * kTcRows;
#pragma unroll
    for (int n = 0; n < kSweepCols; ++n) mine[n * kTcRows + row] = acc[n];
    __threadfence();
    umma::NamedBarrier(1, kEpiThreads);
    if (row == 0) S.isLast = (atomicAdd(w.counters + counter, 1) == t.nsplit - 1);
    umma::NamedBarrier(1, kEpiThreads);
    const bool last = S.isLast;
    umma::NamedBarrier(1, kEpiThreads);  // isLast is rewritten by the next tile
    if (!last) return false;
    __threadfence();
#pragma unroll
    for (int n = 0; n < kSweepCols; ++n) acc[n] = mk<float>(0, 0);
    for (int s = 0; s < t.nsplit; ++s) {
        const c32* p = part + ((int64_t)((t.slot + s) * subs + h) * kSweepCols) * kTcRows;
#pragma unroll
        for (int n = 0; n < kSweepCols; ++n) acc[n] += p[n * kTcRows + row];
    }
    if (row == 0) w.counters[counter] = 0;
    return true;
}

// The epilogue drains one accumulator per tile while the MMAs of the next
// kAccs - 1 tiles run: it loads the accumulator (lane = row), releases it at
// once (the tile's first MMA overwrites it), and writes the result through a
// shared-memory staging tile so that its global accesses are coalesced:
// thread e handles column e % 16 of rows e / 16 + 8 i there.  A tile of NC
// right-hand sides is written as NC / 16 sub-tiles of 16 (columns coff ..
// coff + 15).  What a sub-tile's write-out reads from global memory (the
// forward's carried right-hand sides of the update rows, which are added to
// the product on the way to the parent; each row's parent row or natural
// index) is loaded before its accumulator is ready.

__device__ __forceinline__ bool TileOf(const SweepTile* tiles, int n, int j, int& ti) {
    ti = blockIdx.x + j * gridDim.x;
    return ti < n;
}

__device__ __forceinline__ int LdgIntIf(const int* p, bool pred) {
    int x;
    asm volatile(
        "{\n\t.reg .pred q;\n\t"
        "setp.ne.b32 q, %2, 0;\n\t"
        "mov.b32 %0, -1;\n\t"
        "@q ld.global.nc.b32 %0, [%1];\n\t}\n"
        : "=r"(x)
        : "l"(p), "r"((int)pred));
    return x;
}

struct SubPrefetch {
    c32 carry[kOutPerThread];  // forward: right-hand side of update row (sum of its three planes)
    int idx[kOutPerThread];    // forward: the update row's row in the parent; backward: natural index
};

template <bool kFwd>
__device__ __forceinline__ void PrefetchSub(const SweepFront<float>& f, const SweepTile& t, int k, int coff,
                                            const PanelIO& io, SubPrefetch& pf) {
    const int e = threadIdx.x, n = e % kSweepCols;
    const int col = t.col0 + coff + n;
#pragma unroll
    for (int i = 0; i < kOutPerThread; ++i) {
        const int r = t.row0 + e / kSweepCols + i * kOutRowsPerPass;
        if (kFwd) {
            const bool upd = r >= f.s && r < f.s + f.u;
            pf.idx[i] = LdgIntIf(f.rel + (upd ? r - f.s : 0), upd);
            const bool ok = upd && f.parentRb && col < k;
            const c32* src = f.Rb + (int64_t)r * 3 * k + col;
            pf.carry[i] = LdgC32If(src, ok) + LdgC32If(src + k, ok) + LdgC32If(src + 2 * k, ok);
        } else {
            const bool in = r < f.s;
            pf.idx[i] = LdgIntIf(io.ndToNat + f.ndOff + (in ? r : 0), in);
        }
    }
}

// Sub-tile h of accumulator b (TMEM address taddr of this warp's lanes):
// its columns of the first half plus the same columns of the second half.
template <int NC>
__device__ __forceinline__ void LoadAccumulator(uint32_t taddr, int h, c32 (&acc)[kSweepCols]) {
    float v[kSweepCols];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        umma::TmemLoad16(taddr + 2 * kSweepCols * h + kSweepCols * q, v);
#pragma unroll
        for (int c = 0; c < kSweepCols / 2; ++c) acc[8 * q + c] = mk(v[2 * c], v[2 * c + 1]);
    }
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        umma::TmemLoad16(taddr + 2 * NC + 2 * kSweepCols * h + kSweepCols * q, v);
#pragma unroll
        for (int c = 0; c < kSweepCols / 2; ++c) acc[8 * q + c] += mk(v[2 * c], v[2 * c + 1]);
    }
}

// Sub-tile h of a tile's chain sum (TMEM address tsum of this warp's lanes,
// 16 complex columns at 32 h): acc += sum, or sum := acc.
__device__ __forceinline__ void AddSum(uint32_t tsum, int h, c32 (&acc)[kSweepCols]) {
    float v[kSweepCols];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        umma::TmemLoad16(tsum + 2 * kSweepCols * h + kSweepCols * q, v);
#pragma unroll
        for (int c = 0; c < kSweepCols / 2; ++c) acc[8 * q + c] += mk(v[2 * c], v[2 * c + 1]);
    }
}
__device__ __forceinline__ void StoreSum(uint32_t tsum, int h, const c32 (&acc)[kSweepCols]) {
    float v[2 * kSweepCols];
#pragma unroll
    for (int c = 0; c < kSweepCols; ++c) {
        v[2 * c] = acc[c].re;
        v[2 * c + 1] = acc[c].im;
    }
    umma::TmemStore32NoWait(tsum + 2 * kSweepCols * h, v);
}

// Coalesced write-out of a sub-tile from the staging tile.
template <bool kFwd>
__device__ __forceinline__ void StoreTile(const SweepFront<float>& f, const SweepTile& t, int k, int coff,
                                          const c32* stage, const SubPrefetch& pf, z64* B, c32* X,
                                          const PanelIO& io) {
    const int e = threadIdx.x, n = e % kSweepCols;
    const int col = t.col0 + coff + n;
    if (col >= k) return;
    const int rows = kFwd ? f.s + f.u : f.s;
#pragma unroll
    for (int i = 0; i < kOutPerThread; ++i) {
        const int row = e / kSweepCols + i * kOutRowsPerPass;
        const int r = t.row0 + row;
        if (r >= rows) continue;
        const c32 v = stage[row * kOutPad + n];
        if (kFwd) {
            if (r < f.s) f.Y[(int64_t)r * k + col] = v;
            else if (f.parentRb) f.parentRb[((int64_t)pf.idx[i] * 3 + 1 + f.childSlot) * k + col] = v + pf.carry[i];
        } else {
            X[(int64_t)(f.ndOff + r) * k + col] = v;
            const int pn = pf.idx[i];
            const int xy = pn % io.nxy, vl = pn / io.nxy;
            if (vl < io.padding) continue;
            z64* dst = B + (xy + (int64_t)(io.nz - 1 - (io.vOffset + vl)) * io.nxy) * io.ldk + col;
            const z64 val = ccast<double>(v);
            *dst = io.outAccumulate ? *dst + val : val;
        }
    }
}

template <int NC, bool kFwd>
__device__ void EpilogueRole(const SweepFront<float>* __restrict__ fr, const SweepTile* __restrict__ tiles, int n,
                             int k, const SweepWork& w, c32* staging, Sync& S, z64* B, const PanelIO& io) {
    using C = Cfg<NC>;
    const int warp = threadIdx.x / 32, row = threadIdx.x;
    c32* X = reinterpret_cast<c32*>(w.xnd);
    int ti;
    PdlWait();  // carries, split-K scratch and outputs are shared with the preceding kernels
    for (int q = 0; q < C::kAccs; ++q) umma::MbarArrive(&S.accEmpty[q]);  // every accumulator starts free
    const uint32_t lanes = (uint32_t)(warp * 32) << 16;
    const uint32_t tsum = S.tmem + C::kSumCol + lanes;
    int q = 0;  // chains drained
    for (int j = 0; TileOf(tiles, n, j, ti); ++j) {
        const SweepTile t = tiles[ti];
        const SweepFront<float> f = fr[t.front];
        int kb, ke, nst;
        TileRange(t, kFwd, kb, ke, nst);
        const int nch = NumChains(nst);
        // every chain but the last goes into the sum region; every epilogue
        // thread takes the same branches (they share named barriers)
        for (int c = 0; c + 1 < nch; ++c, ++q) {
            const int b = q % C::kAccs;
            const bool ok = Wait(&S.accFull[b], (q / C::kAccs) & 1, S, w.status);
            if (umma::NamedBarrierOr(1, kEpiThreads, !ok)) return;
            umma::FenceAfterSync();
            const uint32_t taddr = S.tmem + b * C::kAccCols + lanes;
#pragma unroll 1
            for (int h = 0; h < C::kSubs; ++h) {
                c32 acc[kSweepCols];
                LoadAccumulator<NC>(taddr, h, acc);
                if (c > 0) AddSum(tsum, h, acc);
                StoreSum(tsum, h, acc);
            }
            umma::TmemStoreWait();
            umma::FenceBeforeSync();
            umma::MbarArrive(&S.accEmpty[b]);
        }
        // the write-out's global reads overlap the last chain's MMAs
        SubPrefetch pf;
        PrefetchSub<kFwd>(f, t, k, 0, io, pf);
        const int b = q % C::kAccs;
        const bool ok = Wait(&S.accFull[b], (q / C::kAccs) & 1, S, w.status);
        ++q;
        if (umma::NamedBarrierOr(1, kEpiThreads, !ok)) return;
        umma::FenceAfterSync();
        const uint32_t taddr = S.tmem + b * C::kAccCols + lanes;
#pragma unroll
        for (int h = 0; h < C::kSubs; ++h) {
            if (h > 0) PrefetchSub<kFwd>(f, t, k, h * kSweepCols, io, pf);
            c32 acc[kSweepCols];
            LoadAccumulator<NC>(taddr, h, acc);
            if (nch > 1) AddSum(tsum, h, acc);
            if (h == C::kSubs - 1) {
                umma::FenceBeforeSync();
                umma::MbarArrive(&S.accEmpty[b]);
            }
            if (!ReduceSplitsTc(t, w, S, acc, C::kSubs, h)) continue;
#pragma unroll
            for (int c = 0; c < kSweepCols; ++c) staging[row * kOutPad + c] = acc[c];
            umma::NamedBarrier(1, kEpiThreads);
            StoreTile<kFwd>(f, t, k, h * kSweepCols, staging, pf, B, X, io);
            umma::NamedBarrier(1, kEpiThreads);  // staging is rewritten next
        }
    }
}

// ------------------------------------------------------------------ kernels

template <int NC>
__device__ __forceinline__ void InitSync(Sync& S) {
    if (threadIdx.x == 0) {
        for (int i = 0; i < kPlaneSets; ++i) {
            umma::MbarInit(&S.planeFull[i], kGroupThreads);
            umma::MbarInit(&S.planeEmpty[i], 1);
        }
        for (int i = 0; i < Cfg<NC>::kAccs; ++i) {
            umma::MbarInit(&S.accFull[i], 1);
            umma::MbarInit(&S.accEmpty[i], kEpiThreads);
        }
        for (int i = 0; i < kRawMax; ++i) {
            umma::MbarInit(&S.rawFull[i], 1);
            umma::MbarInit(&S.rawEmpty[i], kGroupThreads);
        }
        umma::MbarInit(&S.mmaDrain, 1);
        S.abort = 0;
        S.rawIssued = 0;
        umma::FenceMbarInit();
    }
    if (threadIdx.x / 32 == 0) umma::TmemAlloc(&S.tmem, kTmemCols);
    umma::FenceBeforeSync();
    __syncthreads();
    umma::FenceAfterSync();
}

// Every role has returned.  When one gave up, the others may have left
// asynchronous work behind: the MMA thread waits (bounded) for its
// tensor-core operations, the producer for its copies, before the CTA frees
// tensor memory and exits.  S.abort is no longer written, so every thread
// takes the same branch.
template <int NC, bool kFwd>
__device__ __forceinline__ void Teardown(Sync& S) {
    umma::FenceBeforeSync();
    __syncthreads();
    if (*reinterpret_cast<volatile int*>(&S.abort)) {
        if (threadIdx.x == kMma0) {
            umma::CommitTo(&S.mmaDrain);
            umma::MbarWaitBounded(&S.mmaDrain, 0, nullptr);
        }
        if (threadIdx.x == kProd0) DrainRaw<NC, kFwd>(S);
        umma::FenceBeforeSync();
        __syncthreads();
    }
    if (threadIdx.x / 32 == 0) {
        umma::FenceAfterSync();
        umma::TmemDealloc(S.tmem, kTmemCols);
    }
}

__device__ __forceinline__ unsigned char* SmemBase() {
    extern __shared__ unsigned char smem_raw[];
    return reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
}

template <int NC>
__global__ void __launch_bounds__(kTcThreads, 1) sweep_tc_forward_kernel(const SweepFront<float>* __restrict__ fr,
                                                                         const SweepTile* __restrict__ tiles, int n,
                                                                         int k, SweepWork work) {
    __shared__ Sync S;
    unsigned char* smem = SmemBase();
    PdlTrigger();
    InitSync<NC>(S);
    const int tid = threadIdx.x;
    if (tid < kLoad0) {
        EpilogueRole<NC, true>(fr, tiles, n, k, work, reinterpret_cast<c32*>(smem + Cfg<NC>::kStagingOff), S,
                               nullptr, PanelIO{});
    } else if (tid < kMma0) {
        ConverterRole<NC, true>(fr, tiles, n, k, smem, S, work.status);
    } else if (tid == kMma0) {
        MmaRole<NC, true>(smem, S, work.status);
    } else if (tid >= kProd0) {
        ProducerRole<NC, true>(fr, tiles, n, k, smem, S, work.status);
    }
    Teardown<NC, true>(S);
}

template <int NC>
__global__ void __launch_bounds__(kTcThreads, 1) sweep_tc_backward_kernel(const SweepFront<float>* __restrict__ fr,
                                                                          const SweepTile* __restrict__ tiles, int n,
                                                                          z64* __restrict__ B, int k, PanelIO io,
                                                                          SweepWork work) {
    __shared__ Sync S;
    unsigned char* smem = SmemBase();
    PdlTrigger();
    InitSync<NC>(S);
    const int tid = threadIdx.x;
    if (tid < kLoad0) {
        EpilogueRole<NC, false>(fr, tiles, n, k, work, reinterpret_cast<c32*>(smem + Cfg<NC>::kStagingOff), S, B,
                                io);
    } else if (tid < kMma0) {
        ConverterRole<NC, false>(fr, tiles, n, k, smem, S, work.status);
    } else if (tid == kMma0) {
        MmaRole<NC, false>(smem, S, work.status);
    } else if (tid >= kProd0) {
        ProducerRole<NC, false>(fr, tiles, n, k, smem, S, work.status);
    }
    Teardown<NC, false>(S);
}

int g_numSMs = 0;

int GridFor(int n) { return n < g_numSMs ? n : g_numSMs; }

// A CTA's tile count travels in the upper bits of a stage's packed place
// (InfoSt: 11 bits for the tile, 10 each for the stage and the stage count).
void CheckTilesPerCta(int n) {
    const int g = GridFor(n);
    if (g > 0 && (n + g - 1) / g >= (1 << 11))
        throw PspError(kRuntimeError, "a sweep launch has more than 2047 tiles per CTA (" + std::to_string(n) +
                                          " tiles); the problem is too large for one GPU's sweep tiling");
}

}  // namespace

namespace {
PFN_cuTensorMapEncodeTiled_v12000 g_encodeTiled = nullptr;
}

void EncodeSweepTcMaps(const SweepFront<float>& f, void* out) {
    if (!g_encodeTiled) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        CUDA_CHECK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !fn) throw PspError(kCudaError, "cuTensorMapEncodeTiled is unavailable");
        g_encodeTiled = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    // G as a (s+u) x s array of 8-byte complex-single entries, column stride
    // ldg (even, so every column starts on a 16-byte boundary)
    const cuuint64_t dims[2] = {(cuuint64_t)(f.s + f.u), (cuuint64_t)f.s};
    const cuuint64_t strides[1] = {(cuuint64_t)f.ldg * sizeof(c32)};
    const cuuint32_t unit[2] = {1, 1};
    const cuuint32_t boxes[2][2] = {{(cuuint32_t)kTcRows, (cuuint32_t)kStageK}, {(cuuint32_t)kStageK, (cuuint32_t)kTcRows}};
    CUtensorMap* maps = static_cast<CUtensorMap*>(out);
    for (int b = 0; b < 2; ++b) {
        const CUresult r = g_encodeTiled(&maps[b], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<c32*>(f.G), dims,
                                         strides, boxes[b], unit, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) throw PspError(kCudaError, "cuTensorMapEncodeTiled failed for a sweep front");
    }
}

void PrepareSweepTcKernels() {
    int dev = 0;
    CUDA_CHECK(cudaGetDevice(&dev));
    CUDA_CHECK(cudaDeviceGetAttribute(&g_numSMs, cudaDevAttrMultiProcessorCount, dev));
    CUDA_CHECK(cudaFuncSetAttribute(sweep_tc_forward_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)Cfg<16>::kSmem));
    CUDA_CHECK(cudaFuncSetAttribute(sweep_tc_backward_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)Cfg<16>::kSmem));
    CUDA_CHECK(cudaFuncSetAttribute(sweep_tc_forward_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)Cfg<32>::kSmem));
    CUDA_CHECK(cudaFuncSetAttribute(sweep_tc_backward_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)Cfg<32>::kSmem));
}

void LaunchSweepForwardTc(const SweepFront<float>* fr, const SweepTile* tiles, int n, int k, int cols,
                          const SweepWork& w, cudaStream_t st) {
    if (n <= 0) return;
    CheckTilesPerCta(n);
    if (cols == 32)
        LaunchPdl(sweep_tc_forward_kernel<32>, dim3(GridFor(n)), dim3(kTcThreads), Cfg<32>::kSmem, st, fr, tiles, n,
                  k, w);
    else
        LaunchPdl(sweep_tc_forward_kernel<16>, dim3(GridFor(n)), dim3(kTcThreads), Cfg<16>::kSmem, st, fr, tiles, n,
                  k, w);
    CUDA_LAUNCH_CHECK();
}

void LaunchSweepBackwardTc(const SweepFront<float>* fr, const SweepTile* tiles, int n, z64* B, int k, int cols,
                           const PanelIO& io, const SweepWork& w, cudaStream_t st) {
    if (n <= 0) return;
    CheckTilesPerCta(n);
    if (cols == 32)
        LaunchPdl(sweep_tc_backward_kernel<32>, dim3(GridFor(n)), dim3(kTcThreads), Cfg<32>::kSmem, st, fr, tiles,
                  n, B, k, io, w);
    else
        LaunchPdl(sweep_tc_backward_kernel<16>, dim3(GridFor(n)), dim3(kTcThreads), Cfg<16>::kSmem, st, fr, tiles,
                  n, B, k, io, w);
    CUDA_LAUNCH_CHECK();
}

}  // namespace psp_b200
