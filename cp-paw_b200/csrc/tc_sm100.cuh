// Blackwell (sm_100a) tensor-core primitives as inline PTX: mbarriers, named
// barriers, TMEM allocation, tcgen05.mma of kind::tf32 with shared-memory
// operand descriptors, tcgen05.commit and TMEM loads.  Used by the
// mixed-precision contractions.
//
// Operand tiles live in shared memory in the K-major layout without swizzle:
// element (row r, k) of a tile with R rows sits at byte
//     (k / 4) * (R * 16) + r * 16 + (k % 4) * 4            (fp32 / tf32)
// i.e. groups of four K values form 16-byte rows, eight consecutive rows form
// one 128-byte core matrix (stride-byte offset 128), and the next group of four
// K values starts R*16 bytes further (leading-byte offset R*16).  One MMA of
// kind::tf32 consumes K = 8, i.e. two such groups.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace cuw {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ---- mbarrier ---------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for the phase of the given parity to complete; gives up (false) after
// max_cycles SM clocks so that a logic error can never hang the GPU.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long max_cycles) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > max_cycles) return false;
  }
  return true;
}
// one arrival (of the count given at init) on *bar
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// ---- named barriers ------------------------------------------------------------
// barrier among `nthreads` threads (a multiple of 32) on hardware barrier `id`
// (1..15; 0 is __syncthreads), returning whether any of them passed pred
__device__ __forceinline__ bool bar_or(int id, int nthreads, bool pred) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.or.pred q, %2, %3, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)pred), "r"(id), "r"(nthreads)
      : "memory");
  return r != 0;
}
__device__ __forceinline__ void bar_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// generic-proxy writes to shared memory become visible to the tensor core
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// ---- tensor memory ------------------------------------------------------------
// executed by one full warp; the TMEM address is written to *dst
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// ---- descriptors ----------------------------------------------------------------
// shared-memory matrix descriptor: K-major, no swizzle, version 1 (sm_100)
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// instruction descriptor of kind::tf32: D fp32, A and B tf32, both K-major
__host__ __device__ constexpr uint32_t idesc_tf32(int m, int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// ---- MMA ------------------------------------------------------------------------------
// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread
__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// D[tmem] (+)= A[tmem] * B[smem]^T: A held in tensor memory (lane = row,
// one 32-bit column per K value), issued by one thread
__device__ __forceinline__ void mma_tf32_ta(uint32_t d_tmem, uint32_t a_tmem, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d_tmem),
      "r"(a_tmem), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// arrives once on *bar when every MMA issued so far by this thread has completed
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// ---- TMEM -> registers ---------------------------------------------------------------------
// warp w (w % 4 = q) reads TMEM lanes 32q..32q+31; lane t gets row 32q+t,
// columns [col, col+16) of the 32-bit accumulator
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
// registers -> TMEM: lane t of warp w (w % 4 = q) writes row 32q+t, columns
// [col, col+8) of the 32-bit TMEM address taddr
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t (&r)[8]) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr), "r"(r[0]),
               "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
               : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// ---- split precision ------------------------------------------------------------------------
// x = hi + lo with hi a tf32 value (10 explicit mantissa bits, rounded to
// nearest) and lo = fp32(x) - hi, exact in fp32; the tensor core reads lo as
// tf32 too, so hi*hi + hi*lo + lo*hi carries about 21 significant bits (the
// bits of x beyond fp32 lie far below lo's tf32 precision).  One conversion
// per value: float/double conversions are a low-throughput operation.
__device__ __forceinline__ void split_tf32f(float xf, float& hi, float& lo) {
  const uint32_t u = (__float_as_uint(xf) + 0x1000u) & 0xFFFFE000u;
  hi = __uint_as_float(u);
  lo = xf - hi;
}
__device__ __forceinline__ void split_tf32(double x, float& hi, float& lo) { split_tf32f((float)x, hi, lo); }

// ---- asynchronous global -> shared copies (cp.async) -------------------------------------
// 16 bytes from gmem to smem; bytes beyond src_bytes (0..16) are zero-filled
// and not read.  Both addresses are 16-byte aligned.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(smem)), "l"(gmem), "r"(src_bytes)
               : "memory");
}
// 8 bytes (8-byte aligned addresses), zero-filled beyond src_bytes (0 or 8)
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, int src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(smem_u32(smem)), "l"(gmem), "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// the mbarrier receives one arrival (counted in addition to the ones it was
// initialised for) once every prior cp.async of this thread has completed
__device__ __forceinline__ void cp_async_mbar_arrive(uint64_t* bar) {
  asm volatile("cp.async.mbarrier.arrive.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// bulk copy of `bytes` (a multiple of 16; both addresses 16-byte aligned) from
// global to this CTA's shared memory, completing `bytes` transactions on *bar
__device__ __forceinline__ void bulk_g2s(void* smem, const void* gmem, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(smem)),
               "l"(gmem), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
// 2-D tiled TMA load (no multicast): the box of tensor map *tm at element
// coordinates (x, y) into this CTA's shared memory, completing its bytes on
// *bar.  x times the element size is a multiple of 16 bytes; elements outside
// the tensor read as zero.
__device__ __forceinline__ void tma_load_2d(void* smem, const CUtensorMap* tm, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(smem_u32(smem)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}
// one arrival on *bar that also announces `tx` bytes of copies to complete
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t tx) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(tx) : "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// ---- packed fp32 ------------------------------------------------------------------------
// (a0, a1) += (b0, b1) with one add.rn.f32x2 (round to nearest)
__device__ __forceinline__ void add2(float& a0, float& a1, uint32_t b0, uint32_t b1) {
  asm("{\n\t.reg .b64 p, q;\n\t"
      "mov.b64 p, {%0, %1};\n\t"
      "mov.b64 q, {%2, %3};\n\t"
      "add.rn.f32x2 p, p, q;\n\t"
      "mov.b64 {%0, %1}, p;\n\t}"
      : "+f"(a0), "+f"(a1)
      : "r"(b0), "r"(b1));
}

}  // namespace tc
}  // namespace cuw
