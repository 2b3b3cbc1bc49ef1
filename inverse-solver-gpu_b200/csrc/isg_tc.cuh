// Thin wrappers over the sm_100a PTX used by the tensor-core engine:
// mbarriers, bulk async copies, tcgen05 (TMEM allocation, MMA, commit, loads)
// and the shared-memory matrix descriptor.  Every wait is bounded: on expiry
// it raises a flag in global memory and returns false instead of spinning on.
#pragma once

#include <cstdint>
#include <cuda_fp16.h>

namespace isg {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes));
}
__device__ __forceinline__ bool mbar_test(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for the phase with the given parity to complete; gives up after
// `limit` polls, records `code` in *err and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *err, int code,
                                          long limit = 20000000L) {
  for (long i = 0; i < limit; i++) {
    if (mbar_test(bar, parity)) return true;
    if (i > 64) __nanosleep(32);
  }
  if (err) atomicExch(err, code);
  return false;
}

// The same wait, also giving up (without raising the flag again) once another
// role of the CTA has set *abort; on expiry it sets *abort itself.
__device__ __forceinline__ bool mbar_wait_or(uint64_t *bar, uint32_t parity, volatile int *abort, int *err, int code,
                                             long limit = 20000000L) {
  for (long i = 0; i < limit; i++) {
    if (mbar_test(bar, parity)) return true;
    if (*abort) return false;
    if (i > 64) __nanosleep(32);
  }
  *abort = 1;
  if (err) atomicExch(err, code);
  return false;
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}

// 16-byte asynchronous global -> shared copy; zero-fills when !valid.
__device__ __forceinline__ void cp_async16z(void *smem, const void *gmem, bool valid) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(smem)), "l"(gmem),
               "r"(valid ? 16 : 0));
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }

// 1-D bulk copy global -> shared, completion counted on an mbarrier.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// Tiled 5-D tensor load global -> shared (no multicast), completion counted on
// an mbarrier.  c0 is the innermost coordinate; it must address a 16-byte
// boundary.  Coordinates outside the tensor read as zero.
__device__ __forceinline__ void tma_load_5d(void *dst, const void *tmap, int c0, int c1, int c2, int c3, int c4,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], "
      "[%7];\n" ::"r"(smem_u32(dst)),
      "l"(tmap), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar))
      : "memory");
}

// Tiled 4-D tensor load global -> shared (no multicast); c0 (innermost) must
// address a 16-byte boundary.  Coordinates outside the tensor read as zero.
__device__ __forceinline__ void tma_load_4d(void *dst, const void *tmap, int c0, int c1, int c2, int c3,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];\n" ::"r"(smem_u32(dst)),
      "l"(tmap), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}

// Bulk prefetch of a contiguous global range into L2 (16-byte aligned, size a
// multiple of 16).
__device__ __forceinline__ void bulk_prefetch_l2(const void *src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(src), "r"(bytes) : "memory");
}

// ---- tcgen05 ----
__device__ __forceinline__ void tmem_alloc(uint32_t *dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(dst_smem)),
               "r"(ncols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols));
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// Shared-memory matrix descriptor, no swizzle (core matrices of 8 rows x 16
// bytes, rows 16 bytes apart): lbo = bytes between core matrices adjacent in
// K, sbo = bytes between core matrices adjacent in M/N.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for tcgen05
  return d;                // base offset 0, relative LBO, swizzle none
}

// The descriptor of the same matrix layout `bytes` further on (bytes a multiple
// of 16, the start address staying below 256 KB): only the start field moves.
__device__ __forceinline__ uint64_t desc_add(uint64_t d, uint32_t bytes) { return d + (bytes >> 4); }

// Instruction descriptor of kind::f16 with F16 A and B, F32 accumulation,
// both operands K-major.
__host__ __device__ constexpr uint32_t idesc_f16_f32(int M, int N) {
  return (1u << 4)                       // D format F32
         | (0u << 7) | (0u << 10)        // A, B format F16
         | ((uint32_t)(N >> 3) << 17)    // N / 8
         | ((uint32_t)(M >> 4) << 24);   // M / 16
}

__device__ __forceinline__ void mma_f16(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, int accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}
// Arrives on the mbarrier once every MMA issued so far by this thread is done.
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(bar))
               : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// 8 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float *v) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; i++) v[i] = __uint_as_float(r[i]);
}

// 32 consecutive FP32 columns of this thread's TMEM lane (one wait).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// Splits v (already scaled into the FP16 range) into hi + lo with
// hi = fp16(v) and lo = fp16(v - hi).
__device__ __forceinline__ void split_f16(float v, __half &hi, __half &lo) {
  hi = __float2half_rn(v);
  lo = __float2half_rn(v - __half2float(hi));
}

// Power-of-two scale that maps max|v| to about 2^14 (exact in FP32).
__device__ __forceinline__ float pow2_scale(float maxabs) {
  if (!(maxabs > 0.f) || !isfinite(maxabs)) return 1.f;
  int e;
  frexpf(maxabs, &e);  // maxabs = m * 2^e, m in [0.5, 1)
  return ldexpf(1.f, 14 - e);
}

// Splits (a, b), already scaled into the FP16 range, into packed hi and lo halves.
__device__ __forceinline__ void split2(float a, float b, __half2 &hi, __half2 &lo) {
  hi = __floats2half2_rn(a, b);
  const float2 h = __half22float2(hi);
  lo = __floats2half2_rn(a - h.x, b - h.y);
}

// The same split as packed 32-bit words (lo half = first value).
__device__ __forceinline__ void split2u(float a, float b, uint32_t &hi, uint32_t &lo) {
  __half2 h, l;
  split2(a, b, h, l);
  hi = *(uint32_t *)&h;
  lo = *(uint32_t *)&l;
}
__device__ __forceinline__ void st_shared_v4(void *p, const uint32_t (&v)[4]) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};\n" ::"r"(smem_u32(p)), "r"(v[0]), "r"(v[1]), "r"(v[2]),
               "r"(v[3])
               : "memory");
}

constexpr int kPipeThreads = 512;

// Named barrier 1..15 (0 is __syncthreads) over `count` threads.
__device__ __forceinline__ void named_sync(int id, int count) {
  asm volatile("bar.sync %0, %1;\n" ::"r"(id), "r"(count) : "memory");
}

// The persistent pipelined tensor-core kernels (P2M, M2M, L2L) run items (a
// tile of leaves, or a group of consecutive parents, of one RHS) through three
// roles, each item's buffers alternating between two sets: converter warps
// turn the item's input into the FP16 hi/lo data operand [b] while the MMA
// warp multiplies the previous item's operand [1-b] into TMEM accumulator 1-b
// and the epilogue warps drain the accumulator of the item before that.
// Hand-offs are mbarriers: zfull (the item's input landed), bfull / bfree
// (operand written / consumed by the MMAs), tfull / tfree (accumulator
// written / read out).  Every wait is bounded and gives up once any role has
// given up.  The weight operand stays resident in shared memory.
// A role split: CONV converter warps (0 .. CONV-1), one MMA warp (CONV), EPI
// epilogue warps after it (a multiple of 4; the TMEM lane quarter of warp w is
// w % 4, and the epilogue warps of one quarter split the columns in EPI / 4
// groups).
template <int CONV, int EPI>
struct PipeRoles {
  static constexpr int conv_warps = CONV, mma_warp = CONV, epi_warp0 = CONV + 1;
  static constexpr int threads = 32 * (CONV + 1 + EPI), conv = 32 * CONV, epi = 32 * EPI, epi_groups = EPI / 4;
};

constexpr int kPipeConvWarps = 11;  // warps 0..10
constexpr int kPipeMmaWarp = 11;    // warp 11
constexpr int kPipeEpiWarp0 = 12;   // warps 12..15, one per TMEM lane quarter
constexpr int kPipeConv = 32 * kPipeConvWarps;
constexpr int kPipeEpi = kPipeThreads - 32 * kPipeEpiWarp0;
constexpr int kPipeEpiGroups = kPipeEpi / 128;  // column groups of the accumulator

// Barrier slots: A, zfull[2], bfull[2], bfree[2], tfull[2], tfree[2]; then
// the TMEM base and the abort flag.
struct PipeBars {
  uint64_t *abar, *zfull, *bfull, *bfree, *tfull, *tfree;
  uint32_t *tslot;
  volatile int *abort;
  __device__ explicit PipeBars(char *p) {
    uint64_t *b = (uint64_t *)p;
    abar = b;
    zfull = b + 1;
    bfull = b + 3;
    bfree = b + 5;
    tfull = b + 7;
    tfree = b + 9;
    tslot = (uint32_t *)(b + 11);
    abort = (volatile int *)(b + 12);
  }
};

}  // namespace tc
}  // namespace isg
