// cb2_tc.cuh -- building blocks of the tcgen05 kernels (sm_100a): mbarriers
// with bounded waits, TMA loads, the f16 / bf16 MMA with its descriptors,
// tensor-memory loads and the 64-byte-swizzled K-major shared-memory layout.
#pragma once

#include <cuda.h>
#include <cstdint>

namespace cb2 {
namespace tc {

constexpr unsigned long long kWaitNs = 200ull * 1000 * 1000;   // 200 ms per wait

__device__ inline uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ inline unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ inline void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ inline void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// wait for the phase with the given parity to complete; false after
// budget_ns (0: one try).  The pipelines' waits take the context's budget;
// the drains after an abort (copies and MMAs still in flight) take kWaitNs.
__device__ inline bool mbar_wait(uint64_t *bar, uint32_t parity, unsigned long long budget_ns = kWaitNs) {
  const uint32_t addr = smem_u32(bar);
  unsigned long long t0 = 0;
  for (uint32_t it = 0;; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
    if (budget_ns == 0) return false;
    if (it == 64) t0 = globaltimer();
    if (it > 64) {
      if (globaltimer() - t0 > budget_ns) return false;
      __nanosleep(32);
    }
  }
}

// L2 policies: the B tables are re-read by every CTA of an order (keep
// them), the raw operand rows are read once (let them go first)
__device__ inline uint64_t policy_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ inline uint64_t policy_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}

__device__ inline void tma_load_2d_hint(void *dst, const CUtensorMap *tm, uint64_t *bar, int c0, int c1,
                                        uint64_t policy) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
      " [%0], [%1, {%3, %4}], [%2], %5;"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(tm)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "l"(policy)
      : "memory");
}


// instruction descriptor: D f32, A and B f16, both K-major, M x N
__device__ inline uint32_t idesc_f16_f32(int M, int N) {
  return (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ inline void mma_f16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc));
}

__device__ inline void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ inline void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ inline void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ inline void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// two 32-column loads (columns ta.. and tb..) behind one wait
__device__ inline void tmem_ld32x2(uint32_t ta, uint32_t tb, float va[32], float vb[32]) {
  uint32_t r[64];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%64];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47,%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%65];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]), "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]), "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]), "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]), "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
      : "r"(ta), "r"(tb)
      : "memory");
#pragma unroll
  for (int i = 0; i < 32; i++) { va[i] = __uint_as_float(r[i]); vb[i] = __uint_as_float(r[32 + i]); }
}

// tcgen05.ld 16x256b, two loads behind one wait: thread t receives columns
// 2 (t & 3) and 2 (t & 3) + 1 of lanes (t >> 2) and (t >> 2) + 8 of the 16
// lanes addressed (va[0..1]: lane t >> 2, va[2..3]: lane (t >> 2) + 8)
__device__ inline void tmem_ld_16x256b_pair(uint32_t ta, uint32_t tb, float va[4], float vb[4]) {
  uint32_t r[8];
  asm volatile(
      "tcgen05.ld.sync.aligned.16x256b.x1.b32 {%0,%1,%2,%3}, [%8];\n\t"
      "tcgen05.ld.sync.aligned.16x256b.x1.b32 {%4,%5,%6,%7}, [%9];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
      : "r"(ta), "r"(tb)
      : "memory");
#pragma unroll
  for (int i = 0; i < 4; i++) { va[i] = __uint_as_float(r[i]); vb[i] = __uint_as_float(r[4 + i]); }
}

// four 16x256b loads (layout as above) behind one wait
__device__ inline void tmem_ld_16x256b_quad(uint32_t ta, uint32_t tb, uint32_t tc, uint32_t td, float va[4],
                                            float vb[4], float vc[4], float vd[4]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.16x256b.x1.b32 {%0,%1,%2,%3}, [%16];\n\t"
      "tcgen05.ld.sync.aligned.16x256b.x1.b32 {%4,%5,%6,%7}, [%17];\n\t"
      "tcgen05.ld.sync.aligned.16x256b.x1.b32 {%8,%9,%10,%11}, [%18];\n\t"
      "tcgen05.ld.sync.aligned.16x256b.x1.b32 {%12,%13,%14,%15}, [%19];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(ta), "r"(tb), "r"(tc), "r"(td)
      : "memory");
#pragma unroll
  for (int i = 0; i < 4; i++) {
    va[i] = __uint_as_float(r[i]); vb[i] = __uint_as_float(r[4 + i]);
    vc[i] = __uint_as_float(r[8 + i]); vd[i] = __uint_as_float(r[12 + i]);
  }
}

__device__ inline unsigned char *smem_base_1024(unsigned char *raw) {
  return (unsigned char *)(((uintptr_t)raw + 1023) & ~(uintptr_t)1023);
}

// shared-memory descriptor, K-major, 64-byte swizzle (8-row groups 512 bytes apart)
__device__ inline uint64_t smem_desc_sw64(const void *p) {
  uint64_t d = (uint64_t)((smem_u32(p) & 0x3FFFF) >> 4);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(512 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)4 << 61;                 // 64-byte swizzle
  return d;
}

__device__ inline uint32_t sw64_chunk(int row, int c) {
  return (uint32_t)row * 64u + ((uint32_t)(c ^ ((row >> 1) & 3)) << 4);
}

__device__ inline void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// instruction descriptor of kind::f16 with bf16 operands: D f32, A and B
// bf16, both K-major, M x N
__device__ inline uint32_t idesc_bf16_f32(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// TMEM columns (a power of two >= 32) for one warp of the CTA; the address
// lands in *slot (shared memory)
__device__ inline void tmem_alloc(uint32_t *slot, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(cols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ inline void tmem_dealloc(uint32_t addr, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(addr), "r"(cols));
}

}  // namespace tc
}  // namespace cb2
