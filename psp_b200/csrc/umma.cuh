// Minimal sm_100a tensor-core toolkit: tcgen05 MMA with operands in shared
// memory and the accumulator in tensor memory (TMEM), completion through
// mbarriers.  Layout and descriptor encodings follow the sm100 UMMA
// definitions (SWIZZLE_NONE, K-major canonical layout):
//   a K-major operand tile of R rows x K tf32 values is stored as 8-row x
//   16-byte "core matrices" (rows 16 B apart); the K-chunks of one 8-row
//   group are kChunkBytes apart (the descriptor's leading byte offset) and
//   consecutive 8-row groups are sbo bytes apart (its stride byte offset).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace psp_b200 {
namespace umma {

constexpr uint32_t kChunkBytes = 128;  // one core matrix: 8 rows x 16 bytes

// Byte offset of element (row, k) of a K-major tile whose 8-row groups are
// `sbo` bytes apart.
__device__ __forceinline__ uint32_t KMajorOffset(int row, int k, uint32_t sbo) {
    return (uint32_t)(row >> 3) * sbo + (uint32_t)(k >> 2) * kChunkBytes + (uint32_t)(row & 7) * 16u +
           (uint32_t)(k & 3) * 4u;
}

__device__ __forceinline__ uint32_t SmemAddr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: start address, leading byte offset (between
// the two 16-byte K-chunks an MMA consumes), stride byte offset (between
// 8-row groups), version 1, no swizzle.
__device__ __forceinline__ uint64_t SmemDesc(uint32_t smemAddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((smemAddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version for sm100
    return d;
}

// Descriptor of a K-major operand in the 128-byte-swizzle layout: rows of
// 128 bytes (32 tf32 K values), 8-row atoms of 1 KB (1 KB aligned), and the
// 16-byte chunk c of row r stored at chunk position c ^ (r % 8).  Advancing
// the start address by 32 bytes selects the next 8-value K step.
__device__ __forceinline__ uint64_t SmemDescSw128(uint32_t smemAddr) {
    uint64_t d = 0;
    d |= (uint64_t)((smemAddr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;             // leading byte offset (unused by swizzled K-major)
    d |= (uint64_t)(1024 >> 4) << 32;   // stride byte offset: one 8-row atom
    d |= (uint64_t)1 << 46;             // descriptor version for sm100
    d |= (uint64_t)2 << 61;             // SWIZZLE_128B
    return d;
}

// Byte offset of the 16-byte chunk `chunk` of row `row` in that layout.
__device__ __forceinline__ uint32_t Sw128Offset(int row, int chunk) {
    return (uint32_t)(row >> 3) * 1024u + (uint32_t)(row & 7) * 128u + (uint32_t)((chunk ^ (row & 7)) & 7) * 16u;
}

// The same in the 64-byte-swizzle layout: rows of 64 bytes (16 tf32 K
// values), 8-row atoms of 512 bytes (512-byte aligned), chunk c of row r at
// chunk position c ^ ((r / 2) % 4); +32 bytes selects the second K step.
__device__ __forceinline__ uint64_t SmemDescSw64(uint32_t smemAddr) {
    uint64_t d = 0;
    d |= (uint64_t)((smemAddr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;            // leading byte offset (unused by swizzled K-major)
    d |= (uint64_t)(512 >> 4) << 32;   // stride byte offset: one 8-row atom
    d |= (uint64_t)1 << 46;            // descriptor version for sm100
    d |= (uint64_t)4 << 61;            // SWIZZLE_64B
    return d;
}
__device__ __forceinline__ uint32_t Sw64Offset(int row, int chunk) {
    return (uint32_t)(row >> 3) * 512u + (uint32_t)(row & 7) * 64u + (uint32_t)((chunk ^ (row >> 1)) & 3) * 16u;
}

// Instruction descriptor: D f32, A and B tf32, both K-major, M x N.
__host__ __device__ constexpr uint32_t InstrDescTf32(int M, int N) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void MmaTf32(uint32_t tmemD, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n"
        :
        : "r"(tmemD), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// The same with A read from tensor memory: M rows in TMEM lanes 0..M-1, one
// tf32 K value per 32-bit column starting at column address tmemA.
__device__ __forceinline__ void MmaTf32TmemA(uint32_t tmemD, uint32_t tmemA, uint64_t bdesc, uint32_t idesc,
                                             uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}\n"
        :
        : "r"(tmemD), "r"(tmemA), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// Arrive on `mbar` once every tcgen05 operation issued so far by this thread
// has completed.
__device__ __forceinline__ void CommitTo(uint64_t* mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(SmemAddr(mbar))
                 : "memory");
}

__device__ __forceinline__ void FenceBeforeSync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void FenceAfterSync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Generic-proxy shared-memory writes become visible to the tensor core.
__device__ __forceinline__ void FenceProxyAsync() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void MbarInit(uint64_t* mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(SmemAddr(mbar)), "r"(count) : "memory");
}
__device__ __forceinline__ void FenceMbarInit() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// One bounded test of a phase; the hardware may suspend the thread (up to
// about a microsecond) until the phase completes instead of spinning.
__device__ __forceinline__ bool MbarTryWait(uint64_t* mbar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2, %3;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(ok)
        : "r"(SmemAddr(mbar)), "r"(phase), "r"(1000u)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t GlobalTimerNs() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Longest wait on one mbarrier phase before a kernel gives up (ns).
constexpr uint64_t kWaitLimitNs = 1000000000ull;

// Bounded wait for the phase of parity `phase` of `mbar` to complete; false
// (and *status set) after kWaitLimitNs.
__device__ __forceinline__ bool MbarWaitBounded(uint64_t* mbar, uint32_t phase, int* status) {
    if (MbarTryWait(mbar, phase)) return true;
    const uint64_t t0 = GlobalTimerNs();
    for (;;) {
        if (MbarTryWait(mbar, phase)) return true;
        if (GlobalTimerNs() - t0 > kWaitLimitNs) break;
    }
    if (status) atomicOr(status, 2);
    return false;
}

// TMEM allocation by one full warp; the column address lands in *slot.
__device__ __forceinline__ void TmemAlloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(SmemAddr(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void TmemDealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 32 consecutive f32 columns of this thread's TMEM lane (lane = row of D).
__device__ __forceinline__ void TmemLoad32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// 8-byte asynchronous global->shared copy (no register staging); bytes past
// `srcBytes` (0 or 8) are zero-filled and not read.
__device__ __forceinline__ void CpAsync8(void* dst, const void* src, uint32_t srcBytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(SmemAddr(dst)), "l"(src), "r"(srcBytes)
                 : "memory");
}
// 16-byte asynchronous global->shared copy (both addresses 16-byte aligned);
// bytes past `srcBytes` (0, 8 or 16) are zero-filled and not read.
__device__ __forceinline__ void CpAsync16(void* dst, const void* src, uint32_t srcBytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(SmemAddr(dst)), "l"(src), "r"(srcBytes)
                 : "memory");
}
__device__ __forceinline__ void CpAsyncCommit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// Waits until at most N of this thread's committed copy groups are pending.
template <int N>
__device__ __forceinline__ void CpAsyncWait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void CpAsyncWaitAll() { asm volatile("cp.async.wait_all;" ::: "memory"); }
// Arrive on `mbar` once all prior cp.async copies of this thread have landed;
// the arrival counts against the barrier's initial count.
__device__ __forceinline__ void CpAsyncArrive(uint64_t* mbar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(SmemAddr(mbar)) : "memory");
}
// Bulk asynchronous copy of `bytes` (a multiple of 16; both addresses 16-byte
// aligned) from global to this CTA's shared memory, completing as
// transaction bytes on `mbar`.
__device__ __forceinline__ void BulkCopy(void* dst, const void* src, uint32_t bytes, uint64_t* mbar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(SmemAddr(dst)),
        "l"(src), "r"(bytes), "r"(SmemAddr(mbar))
        : "memory");
}
// Tiled 2-D tensor copy (no multicast) of the box at coordinates (x, y) of
// the tensor map at `tmap` (global memory, 64-byte aligned) into this CTA's
// shared memory (128-byte aligned), completing as transaction bytes on
// `mbar`; elements outside the tensor are zero-filled.  x * element size
// must be a multiple of 16 bytes.
__device__ __forceinline__ void TmaLoad2D(void* dst, const void* tmap, int x, int y, uint64_t* mbar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(SmemAddr(dst)),
        "l"(tmap), "r"(x), "r"(y), "r"(SmemAddr(mbar))
        : "memory");
}

// Arrive on `mbar` and add `bytes` to the transaction bytes its phase waits for.
__device__ __forceinline__ void MbarArriveExpectTx(uint64_t* mbar, uint32_t bytes) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(
                     SmemAddr(mbar)),
                 "r"(bytes)
                 : "memory");
}

// Plain arrive (release semantics at CTA scope).
__device__ __forceinline__ void MbarArrive(uint64_t* mbar) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(SmemAddr(mbar))
                 : "memory");
}
// Named barrier over `nthreads` threads (a multiple of 32).
__device__ __forceinline__ void NamedBarrier(int id, int nthreads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}
// Named barrier that also ORs `pred` over the participating threads.
__device__ __forceinline__ bool NamedBarrierOr(int id, int nthreads, bool pred) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 q, %1, 0;\n\t"
        "bar.red.or.pred p, %2, %3, q;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(r)
        : "r"((uint32_t)pred), "r"(id), "r"(nthreads)
        : "memory");
    return r != 0;
}

// Writes 32 consecutive f32 columns of this thread's TMEM lane without
// waiting (TmemStoreWait() waits for all of this thread's TMEM stores).
__device__ __forceinline__ void TmemStore32NoWait(uint32_t taddr, const float (&v)[32]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], "
        "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
        "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};\n"
        ::"r"(taddr),
        "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])), "r"(__float_as_uint(v[3])),
        "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])), "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])),
        "r"(__float_as_uint(v[8])), "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
        "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])), "r"(__float_as_uint(v[15])),
        "r"(__float_as_uint(v[16])), "r"(__float_as_uint(v[17])), "r"(__float_as_uint(v[18])), "r"(__float_as_uint(v[19])),
        "r"(__float_as_uint(v[20])), "r"(__float_as_uint(v[21])), "r"(__float_as_uint(v[22])), "r"(__float_as_uint(v[23])),
        "r"(__float_as_uint(v[24])), "r"(__float_as_uint(v[25])), "r"(__float_as_uint(v[26])), "r"(__float_as_uint(v[27])),
        "r"(__float_as_uint(v[28])), "r"(__float_as_uint(v[29])), "r"(__float_as_uint(v[30])), "r"(__float_as_uint(v[31]))
        : "memory");
}

// Writes 32 consecutive f32 columns of this thread's TMEM lane and waits
// for the write.
__device__ __forceinline__ void TmemStore32(uint32_t taddr, const float (&v)[32]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], "
        "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
        "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};\n"
        ::"r"(taddr),
        "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])), "r"(__float_as_uint(v[3])),
        "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])), "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])),
        "r"(__float_as_uint(v[8])), "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
        "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])), "r"(__float_as_uint(v[15])),
        "r"(__float_as_uint(v[16])), "r"(__float_as_uint(v[17])), "r"(__float_as_uint(v[18])), "r"(__float_as_uint(v[19])),
        "r"(__float_as_uint(v[20])), "r"(__float_as_uint(v[21])), "r"(__float_as_uint(v[22])), "r"(__float_as_uint(v[23])),
        "r"(__float_as_uint(v[24])), "r"(__float_as_uint(v[25])), "r"(__float_as_uint(v[26])), "r"(__float_as_uint(v[27])),
        "r"(__float_as_uint(v[28])), "r"(__float_as_uint(v[29])), "r"(__float_as_uint(v[30])), "r"(__float_as_uint(v[31]))
        : "memory");
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// Writes 8 consecutive 32-bit columns of this thread's TMEM lane without
// waiting; TmemStoreWait() waits for all of this thread's TMEM stores.
__device__ __forceinline__ void TmemStore8(uint32_t taddr, const float (&v)[8]) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};\n" ::"r"(taddr),
                 "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
                 "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
                 "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7]))
                 : "memory");
}
__device__ __forceinline__ void TmemStoreWait() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// 16 consecutive f32 columns of this thread's TMEM lane.
__device__ __forceinline__ void TmemLoad16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Split x into a tf32 head rounded by integer arithmetic on the bit pattern
// (11 significant bits, ties away from zero) and the exact fp32 tail x - hi,
// of which the MMA reads the top 11 bits: x ~= hi + lo to ~2^-21 relative,
// in three integer/FP32 operations (no conversion instructions).
__device__ __forceinline__ void SplitTf32Fast(float x, float& hi, float& lo) {
    hi = __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
    lo = x - hi;
}

// Split x into a tf32 head and a tf32 tail: x ~= hi + lo to ~2^-22 relative.
__device__ __forceinline__ void SplitTf32(float x, float& hi, float& lo) {
    uint32_t h;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(x));
    hi = __uint_as_float(h);
    uint32_t l;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(l) : "f"(x - hi));
    lo = __uint_as_float(l);
}

}  // namespace umma
}  // namespace psp_b200
