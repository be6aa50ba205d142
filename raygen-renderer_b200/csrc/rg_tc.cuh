// rg_tc.cuh - 5th-generation tensor-core (tcgen05) building blocks for sm_100a.
//
// One CTA of 128 threads computes D[128 x N] (+)= A[128 x K] * B[N x K]^T with
// BF16 operands in shared memory and the FP32 accumulator in tensor memory:
//  * operands are stored K-major without swizzle, in 8-row x 16-byte core
//    matrices: element (r, k) at (r / 8) * SBO + (k / 8) * 128 + (r % 8) * 16
//    + (k % 8) * 2 bytes, SBO = K / 8 * 128 (the K chunks of an 8-row group
//    are contiguous, LBO = 128 bytes);
//  * one elected thread issues K / 16 MMAs of M = 128 and commits them to an
//    mbarrier; every thread waits on it (bounded), then each warp reads its 32
//    accumulator lanes (rows) with tcgen05.ld.
// Descriptor bit layouts follow the PTX ISA (shared-memory matrix descriptor:
// start >> 4 in [0,14), LBO >> 4 in [16,30), SBO >> 4 in [32,46), version 1 in
// [46,48), layout type in [61,64); instruction descriptor for kind::f16: FP32
// accumulator [4,6) = 1, BF16 A [7,10) = 1 and B [10,13) = 1, K-major A/B,
// N >> 3 in [17,23), M >> 4 in [24,29)).
#pragma once

#include <cstdint>

namespace rg {
namespace tc {

constexpr uint32_t kWaitLimit = 1u << 26;  // mbarrier polls before a kernel gives up
constexpr int kErrTcTimeout = 0x7c01;      // error word value: a tensor-core wait ran out

__device__ __forceinline__ uint32_t smemAddr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t smemDesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1u << 46;  // descriptor version for this architecture
  return d;                 // base offset 0, no swizzle
}

// K-major operand in the 64-byte swizzled layout TMA writes with a 64-byte
// swizzle: rows of 64 bytes, 8-row groups 512 bytes apart (SBO), and the
// 16-byte chunk c of row r stored at chunk c ^ ((r >> 1) & 3).  The swizzle
// follows the shared-memory address, so a start moved by whole rows or by a
// 32-byte K step within the row still reads the data TMA placed (the buffer is
// 1024-byte aligned).
__device__ __forceinline__ uint64_t smemDescSw64(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)1u << 16;           // leading byte offset: unused for a swizzled K-major operand
  d |= (uint64_t)(512u >> 4) << 32;  // 8 rows x 64 bytes
  d |= (uint64_t)1u << 46;           // descriptor version for this architecture
  d |= (uint64_t)4u << 61;           // layout type: 64-byte swizzle
  return d;
}

// The same for rows of 32 bytes (16 BF16 channels) in the 32-byte swizzled
// layout: 8-row groups 256 bytes apart, chunk c of row r at c ^ ((r >> 2) & 1).
__device__ __forceinline__ uint64_t smemDescSw32(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)1u << 16;           // leading byte offset: unused for a swizzled K-major operand
  d |= (uint64_t)(256u >> 4) << 32;  // 8 rows x 32 bytes
  d |= (uint64_t)1u << 46;           // descriptor version for this architecture
  d |= (uint64_t)6u << 61;           // layout type: 32-byte swizzle
  return d;
}

__host__ __device__ constexpr uint32_t instrDescBf16(int M, int N) {
  return (1u << 4)                       // FP32 accumulator
         | (1u << 7)                     // A: BF16
         | (1u << 10)                    // B: BF16
         | ((uint32_t)(N >> 3) << 17)    // N
         | ((uint32_t)(M >> 4) << 24);   // M
}

__device__ __forceinline__ void tmemAlloc(uint32_t* dstSmem, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smemAddr(dstSmem)), "r"(cols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmemFree(uint32_t taddr, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}

__device__ __forceinline__ void mbarInit(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smemAddr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbarTryWait(uint64_t* bar, uint32_t phase) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smemAddr(bar)), "r"(phase)
      : "memory");
  return done != 0;
}

// Bounded wait: false when `limit` polls ran out.
__device__ __forceinline__ bool mbarWait(uint64_t* bar, uint32_t phase, uint32_t limit = kWaitLimit) {
  for (uint32_t i = 0; i < limit; ++i)
    if (mbarTryWait(bar, phase)) return true;
  return false;
}

// 16-byte asynchronous global -> shared copy; with `valid` false nothing is
// read and the 16 destination bytes are zero-filled.
__device__ __forceinline__ void cpAsync16(uint32_t dst, const void* src, bool valid) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(valid ? 16u : 0u)
               : "memory");
}
__device__ __forceinline__ void cpAsyncCommit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// Wait until at most N of this thread's committed copy groups are still in flight.
template <int N>
__device__ __forceinline__ void cpAsyncWait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// The barrier expects `bytes` more transaction bytes in its current phase; this thread arrives.
__device__ __forceinline__ void mbarArriveExpectTx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smemAddr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbarArrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smemAddr(bar)) : "memory");
}
// Make initialised barriers visible to the asynchronous proxy (TMA, tensor cores).
__device__ __forceinline__ void fenceBarrierInit() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// TMA tile load (no multicast) of a 4-D box at (c0, c1, c2, c3) into this CTA's
// shared memory; completes `bytes` of transactions on `bar`.  c0 is the
// innermost coordinate and must address a 16-byte boundary; the others may be
// negative or past the end (those elements are zero-filled).
__device__ __forceinline__ void tmaLoad4d(uint32_t dst, const void* tmap, int c0, int c1, int c2, int c3,
                                          uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(dst),
      "l"(tmap), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smemAddr(bar))
      : "memory");
}

__device__ __forceinline__ void fenceProxyAsync() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fenceAfterSync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fenceBeforeSync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

// D (tmem) (+)= A * B^T for one K step of 16 (descriptors point at the step's
// first core matrices).  Issued by one thread.
__device__ __forceinline__ void mmaBf16(uint32_t tmemD, uint64_t descA, uint64_t descB, uint32_t idesc,
                                        bool accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      :
      : "r"(tmemD), "l"(descA), "l"(descB), "r"(idesc), "r"((uint32_t)accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}

// Arrive on `bar` when every MMA issued so far by this thread has completed.
__device__ __forceinline__ void commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smemAddr(bar))
               : "memory");
}

// 32 consecutive FP32 accumulator columns of this thread's lane.
__device__ __forceinline__ void tmemLoad32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Byte offset of the 16-byte chunk (row r, K chunk kc) in a K-major operand of K columns.
__host__ __device__ __forceinline__ uint32_t chunkOffset(int r, int kc, int K) {
  return (uint32_t)((r >> 3) * (K / 8) * 128 + kc * 128 + (r & 7) * 16);
}

}  // namespace tc
}  // namespace rg
