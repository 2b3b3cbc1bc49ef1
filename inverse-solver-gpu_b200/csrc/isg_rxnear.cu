// Near-field receivers: the dense receiver operator of the reference's
// commented near-field form (setup_born.cpp:52-60),
//     go[m][n] = integrate(rx_m, pos_n),   gh[n][m] = conj(go[m][n]),
// for numrx receivers rx_m = radius (cos 2 pi m / numrx, sin 2 pi m / numrx)
// (the directions of mom.cpp:149-154 at a finite radius), applied as complex
// GEMMs on the tcgen05 tensor cores:
//     forward  r[j][m] = sum_n go[m][n] x[j][n]   (M = receivers, K = pixels)
//     adjoint  x[j][n] = sum_m gh[n][m] r[j][m]   (M = pixels, K = receivers)
//
// Both tables are built once on the device (FP64 integrate, split into FP16
// hi/lo after a power-of-two scale) as 32 KB blocks of 128 rows x 32 K: the
// real parts (hi, lo), then the imaginary parts.  A CTA multiplies one such
// row tile by the batch: the right-hand sides' real parts as B rows 0..R-1 and
// their imaginary parts as rows R..2R-1 (N = 2R <= 256), so one MMA pair gives
// D_re = Re(G) B and D_im = Im(G) B, and the epilogue combines
//     forward  re = D_re[j] - D_im[R + j],  im = D_re[R + j] + D_im[j]
//     adjoint  re = D_re[j] + D_im[R + j],  im = D_re[R + j] - D_im[j]
// (the adjoint table stores Re and Im of go, not of its conjugate).  Each
// K-block is converted from FP32 by all threads into the FP16 hi/lo B operand
// while the previous block's MMAs run (double-buffered A and B).  The forward
// GEMM has K = numunk and is split over CTAs; the partial products are summed
// in split order by a second kernel, so results do not depend on timing.
#include <cmath>
#include <cstring>

#include "isg_context.hpp"
#include "isg_green.cuh"
#include "isg_tc.cuh"

namespace isg {

struct RxPlan {
  double radius = 0;
  int nrx = 0, U = 0;
  int mt_f = 0, kb_f = 0;  // forward: row tiles of receivers, K-blocks of pixels
  int mt_a = 0, kb_a = 0;  // adjoint: row tiles of pixels, K-blocks of receivers
  int nsplit = 1, kb_per = 1;  // forward K split over CTAs: splits, K-blocks per split
  uint8_t *Af = nullptr, *Aa = nullptr;  // [mt][kb] 32 KB blocks
  float ainv = 1;          // 1 / the tables' power-of-two scale
  unsigned *rowmax = nullptr;  // [max_rhs] max |re|, |im| of the batch's inputs (FP32 bits)
  float2 *part = nullptr;      // [nsplit][max_rhs][nrx] forward partial products
  int *err = nullptr;
};

namespace {

using namespace tc;

constexpr int kRxKB = 32;                 // K per block
constexpr int kRxBlock = 4 * 128 * kRxKB * 2;  // 32 KB: re hi, re lo, im hi, im lo
constexpr int kRxSplit = 128 * kRxKB * 2;      // 8 KB: one FP16 split of 128 rows
constexpr int kRxMaxN = 256;                   // 2 x 128 right-hand sides
constexpr int kRxBBuf = kRxMaxN * kRxKB * 2 * 2;  // 32 KB: B hi then lo for N = 256
constexpr int kRxThreads = 256;
constexpr int kErrRx = 131;
struct RxSmem {
  static constexpr int a = 0;                     // 2 A blocks
  static constexpr int b = 2 * kRxBlock;          // 2 B operands
  static constexpr int bars = b + 2 * kRxBBuf;    // afull[2], mdone[2], fin
  static constexpr int misc = bars + 8 * 8;
  static constexpr int total = misc + 16;
};

// Offset of element (row, k) of a 128 x 32 (or N x 32) K-major FP16 block in
// the no-swizzle core-matrix layout: core matrix (row / 8, k / 8), 8 rows x 16 bytes.
__host__ __device__ __forceinline__ int rx_core_off(int row, int k) {
  return (((row >> 3) * 4 + (k >> 3)) * 64 + (row & 7) * 8 + (k & 7)) * 2;
}

__device__ __forceinline__ double2 rx_point(double radius, int m, int nrx) {
  const double ang = 360.0 / nrx * m;
  return make_double2(radius * cos(ang / 360 * 2 * kPiD), radius * sin(ang / 360 * 2 * kPiD));
}

// Pixel centre of blocked index n (leaves in raster order, row-major inside a leaf).
__device__ __forceinline__ double2 rx_pixel(int n, int nleaf, double res) {
  const int leaf = n / kBB, p = n % kBB;
  const int Y = (leaf / nleaf) * kBox + p / kBox, X = (leaf % nleaf) * kBox + p % kBox;
  const double D = (double)nleaf * kBox * res;
  return make_double2(-D / 2 + (X + 0.5) * res, D / 2 - (Y + 0.5) * res);
}

struct RxBuild {
  double k0, res, radius;
  int nrx, U, nleaf;
};

__device__ __forceinline__ double2 rx_entry(const RxBuild &B, int m, int n) {
  const double2 r = rx_point(B.radius, m, B.nrx), p = rx_pixel(n, B.nleaf, B.res);
  return green_entry_d(B.k0, B.res, p.x - r.x, p.y - r.y);
}

// Largest |re|, |im| of the table (FP32 bits, atomicMax on non-negative floats).
__global__ void k_rx_max(RxBuild B, unsigned *mx) {
  float m = 0.f;
  const size_t total = (size_t)B.nrx * B.U;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const double2 g = rx_entry(B, (int)(e / B.U), (int)(e % B.U));
    m = fmaxf(m, (float)fmax(fabs(g.x), fabs(g.y)));
  }
  const unsigned bits = __reduce_max_sync(0xffffffffu, __float_as_uint(m));
  if ((threadIdx.x & 31) == 0 && bits) atomicMax(mx, bits);
}

// One block per (row tile, K-block) of a table: forward rows = receivers and
// K = pixels, adjoint rows = pixels and K = receivers; rows or K beyond the
// operator are zero.
__global__ void k_rx_pack(RxBuild B, int adjoint, int kb_total, const unsigned *mx, uint8_t *A) {
  const int mt = blockIdx.y, kb = blockIdx.x;
  const float s = pow2_scale(__uint_as_float(*mx));
  __half *blk = (__half *)(A + ((size_t)mt * kb_total + kb) * kRxBlock);
  const int rows = adjoint ? B.U : B.nrx, kdim = adjoint ? B.nrx : B.U;
  for (int e = threadIdx.x; e < 128 * kRxKB; e += blockDim.x) {
    const int row = e / kRxKB, k = e % kRxKB;
    const int R = mt * 128 + row, K = kb * kRxKB + k;
    double2 g = make_double2(0.0, 0.0);
    if (R < rows && K < kdim) g = adjoint ? rx_entry(B, K, R) : rx_entry(B, R, K);
    __half rh, rl, ih, il;
    split_f16((float)g.x * s, rh, rl);
    split_f16((float)g.y * s, ih, il);
    const int o = rx_core_off(row, k) / 2;
    blk[o] = rh;
    blk[kRxSplit / 2 + o] = rl;
    blk[2 * kRxSplit / 2 + o] = ih;
    blk[3 * kRxSplit / 2 + o] = il;
  }
}

// max |re|, |im| per right-hand side of [R][ld] complex rows (first kvalid elements)
__global__ void k_rx_rowmax(const float2 *x, int64_t ld, int kvalid, unsigned *rowmax) {
  const int j = blockIdx.y;
  float m = 0.f;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < kvalid; k += gridDim.x * blockDim.x) {
    const float2 v = x[(size_t)j * ld + k];
    m = fmaxf(m, fmaxf(fabsf(v.x), fabsf(v.y)));
  }
  const unsigned bits = __reduce_max_sync(0xffffffffu, __float_as_uint(m));
  if ((threadIdx.x & 31) == 0 && bits) atomicMax(&rowmax[j], bits);
}

struct RxGemmArgs {
  const uint8_t *A;   // table blocks [mt][kb_total]
  int kb_total, kb_per;  // K-blocks per row tile, per CTA (split)
  const float2 *x;    // B source: [R][ldx] complex, K index = element
  int64_t ldx;
  int kvalid, R, npad;  // valid K, right-hand sides, N = 2R padded to 16
  const unsigned *rowmax;
  float ainv;
  int adjoint;
  float2 *out;        // [split][R][ldo] complex; rows of the output = table rows
  int64_t ldo;
  size_t split_stride;
  int mvalid;
  int *err;
};

__global__ void __launch_bounds__(kRxThreads, 1) k_rx_gemm(RxGemmArgs A) {
  extern __shared__ __align__(1024) char sm[];
  uint64_t *afull = (uint64_t *)(sm + RxSmem::bars), *mdone = afull + 2, *fin = afull + 4;
  uint32_t *tslot = (uint32_t *)(sm + RxSmem::misc);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int mt = blockIdx.x, split = blockIdx.y;
  const int kb0 = split * A.kb_per, kb1 = min(kb0 + A.kb_per, A.kb_total);
  if (threadIdx.x == 0) {
    for (int i = 0; i < 5; i++) mbar_init(afull + i, 1);
    fence_mbar_init();
  }
  if (warp == 0) tmem_alloc(tslot, 512);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;  // D_re in columns [0, npad), D_im in [256, 256 + npad)
  const uint32_t idesc = idesc_f16_f32(128, A.npad), sbase = smem_u32(sm);
  const int R = A.R;
  bool ok = true;
  for (int kb = kb0, it = 0; kb < kb1; kb++, it++) {
    const int b = it & 1;
    // buffers b (A and B) are free once the MMAs of block it - 2 are done
    if (it >= 2) ok = mbar_wait(mdone + b, ((it >> 1) - 1) & 1, A.err, kErrRx) && ok;
    if (threadIdx.x == 0 && ok) {
      mbar_expect_tx(afull + b, kRxBlock);
      bulk_g2s(sm + RxSmem::a + b * kRxBlock, A.A + ((size_t)mt * A.kb_total + kb) * kRxBlock, kRxBlock, afull + b);
    }
    // B operand: row j = Re x_j, row R + j = Im x_j over K = kb * 32 .. + 32, scaled per RHS
    __half *bh = (__half *)(sm + RxSmem::b + b * kRxBBuf), *bl = bh + A.npad * kRxKB;
    for (int e = threadIdx.x; e < R * (kRxKB / 8); e += kRxThreads) {
      const int j = e / (kRxKB / 8), c = e % (kRxKB / 8);  // 8 K-elements of RHS j
      const float s = pow2_scale(__uint_as_float(A.rowmax[j]));
      __align__(16) __half rh[8], rl[8], ih[8], il[8];
#pragma unroll
      for (int q = 0; q < 8; q++) {
        const int K = kb * kRxKB + c * 8 + q;
        const float2 v = K < A.kvalid ? A.x[(size_t)j * A.ldx + K] : make_float2(0.f, 0.f);
        split_f16(v.x * s, rh[q], rl[q]);
        split_f16(v.y * s, ih[q], il[q]);
      }
      const int o0 = rx_core_off(j, c * 8) / 2, o1 = rx_core_off(R + j, c * 8) / 2;
      *(uint4 *)(bh + o0) = *(uint4 *)rh;
      *(uint4 *)(bl + o0) = *(uint4 *)rl;
      *(uint4 *)(bh + o1) = *(uint4 *)ih;
      *(uint4 *)(bl + o1) = *(uint4 *)il;
    }
    // rows 2R .. npad - 1 stay zero
    for (int e = threadIdx.x; e < (A.npad - 2 * R) * (kRxKB / 8); e += kRxThreads) {
      const int r = 2 * R + e / (kRxKB / 8), c = e % (kRxKB / 8);
      const int o = rx_core_off(r, c * 8) / 2;
      *(uint4 *)(bh + o) = make_uint4(0, 0, 0, 0);
      *(uint4 *)(bl + o) = make_uint4(0, 0, 0, 0);
    }
    fence_proxy_async();
    __syncthreads();
    if (threadIdx.x == 0) {
      ok = mbar_wait(afull + b, (it >> 1) & 1, A.err, kErrRx) && ok;
      tc_fence_after();
      if (ok) {
        const uint32_t ab = sbase + RxSmem::a + b * kRxBlock, bb = sbase + RxSmem::b + b * kRxBBuf;
        const uint64_t brh = smem_desc(bb, 128, 512), brl = smem_desc(bb + A.npad * kRxKB * 2, 128, 512);
#pragma unroll
        for (int part = 0; part < 2; part++) {  // re, im of the table
          const uint64_t ah = smem_desc(ab + part * 2 * kRxSplit, 128, 512);
          const uint64_t al = smem_desc(ab + part * 2 * kRxSplit + kRxSplit, 128, 512);
          const uint32_t d = tmem + (uint32_t)(part * 256);
#pragma unroll
          for (int ks = 0; ks < kRxKB / 16; ks++) {
            const int acc = (kb > kb0 || ks > 0) ? 1 : 0;
            mma_f16(d, desc_add(ah, ks * 256), desc_add(brh, ks * 256), idesc, acc);
            mma_f16(d, desc_add(ah, ks * 256), desc_add(brl, ks * 256), idesc, 1);
            mma_f16(d, desc_add(al, ks * 256), desc_add(brh, ks * 256), idesc, 1);
          }
        }
      }
      mma_commit(mdone + b);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) mma_commit(fin);
  ok = mbar_wait(fin, 0, A.err, kErrRx) && ok && kb1 > kb0;
  tc_fence_after();
  // epilogue: lane = table row, columns = right-hand sides; warps 0..3 and 4..7
  // take alternate groups of 16 right-hand sides
  const int qd = warp & 3, half = warp >> 2;
  const int row = mt * 128 + 32 * qd + lane;
  float2 *out = A.out + (size_t)split * A.split_stride;
  for (int j0 = 16 * half; j0 < R; j0 += 32) {
    __syncwarp();
    float dre[16], dre2[16], dim[16], dim2[16];
    tmem_ld16(tmem + ((uint32_t)(32 * qd) << 16) + (uint32_t)j0, dre);
    tmem_ld16(tmem + ((uint32_t)(32 * qd) << 16) + (uint32_t)(R + j0), dre2);
    tmem_ld16(tmem + ((uint32_t)(32 * qd) << 16) + (uint32_t)(256 + j0), dim);
    tmem_ld16(tmem + ((uint32_t)(32 * qd) << 16) + (uint32_t)(256 + R + j0), dim2);
    if (ok && row < A.mvalid) {
#pragma unroll
      for (int q = 0; q < 16; q++) {
        const int j = j0 + q;
        if (j >= R) break;
        const float inv = A.ainv / pow2_scale(__uint_as_float(A.rowmax[j]));
        const float re = A.adjoint ? dre[q] + dim2[q] : dre[q] - dim2[q];
        const float im = A.adjoint ? dre2[q] - dim[q] : dre2[q] + dim[q];
        out[(size_t)j * A.ldo + row] = make_float2(re * inv, im * inv);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, 512);
}

// r[j][m] = sum over splits of part[s][j][m], in split order
__global__ void k_rx_sum(const float2 *part, int nsplit, size_t stride, int R, int nrx, float2 *r) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= R * nrx) return;
  float2 s = make_float2(0.f, 0.f);
  for (int q = 0; q < nsplit; q++) {
    const float2 v = part[q * stride + e];
    s.x += v.x;
    s.y += v.y;
  }
  r[e] = s;
}

}  // namespace

void rxnear_destroy(isg_ctx *c) {
  if (!c->rx) return;
  cudaFree(c->rx->Af);
  cudaFree(c->rx->Aa);
  cudaFree(c->rx->rowmax);
  cudaFree(c->rx->part);
  cudaFree(c->rx->err);
  delete c->rx;
  c->rx = nullptr;
}

bool rxnear_active(const isg_ctx *c) { return c->rx != nullptr; }

isg_status rxnear_setup(isg_ctx *c, double radius) {
  rxnear_destroy(c);
  if (radius == 0) return ISG_OK;
  const HostTables &T = c->T;
  const double half_diag = std::sqrt(2.0) * T.side * T.res / 2;
  if (!(radius > half_diag + T.res)) {
    c->err = "near-field receivers must lie outside the domain (radius > half its diagonal)";
    return ISG_BAD_ARG;
  }
  RxPlan *P = new RxPlan();
  c->rx = P;
  P->radius = radius;
  P->nrx = T.numrx;
  P->U = T.U;
  P->mt_f = (P->nrx + 127) / 128;
  P->kb_f = (P->U + kRxKB - 1) / kRxKB;
  P->mt_a = (P->U + 127) / 128;
  P->kb_a = (P->nrx + kRxKB - 1) / kRxKB;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->opts.device);
  // K-blocks per split first, then the number of (non-empty) splits
  const int target = std::max(1, std::min(P->kb_f, sms / P->mt_f));
  P->kb_per = (P->kb_f + target - 1) / target;
  P->nsplit = (P->kb_f + P->kb_per - 1) / P->kb_per;
  const size_t R = (size_t)std::min(c->opts.max_rhs, kRxMaxN / 2);
  isg_status e;
  unsigned *mx = nullptr;
  if ((e = cuda_check(c, cudaMalloc(&P->Af, (size_t)P->mt_f * P->kb_f * kRxBlock), "receiver tables")) ||
      (e = cuda_check(c, cudaMalloc(&P->Aa, (size_t)P->mt_a * P->kb_a * kRxBlock), "receiver tables")) ||
      (e = cuda_check(c, cudaMalloc(&P->rowmax, R * sizeof(unsigned)), "receiver tables")) ||
      (e = cuda_check(c, cudaMalloc(&P->part, (size_t)P->nsplit * R * P->nrx * sizeof(float2)), "receiver tables")) ||
      (e = cuda_check(c, cudaMalloc(&P->err, sizeof(int)), "receiver tables")) ||
      (e = cuda_check(c, cudaMalloc(&mx, sizeof(unsigned)), "receiver tables"))) {
    cudaFree(mx);
    rxnear_destroy(c);
    return e;
  }
  cudaMemset(P->err, 0, sizeof(int));
  cudaMemset(mx, 0, sizeof(unsigned));
  RxBuild B{T.k0, T.res, radius, P->nrx, P->U, T.nleaf};
  count_launch(3);
  k_rx_max<<<4 * sms, 256>>>(B, mx);
  k_rx_pack<<<dim3(P->kb_f, P->mt_f), 256>>>(B, 0, P->kb_f, mx, P->Af);
  k_rx_pack<<<dim3(P->kb_a, P->mt_a), 256>>>(B, 1, P->kb_a, mx, P->Aa);
  unsigned hm = 0;
  cudaMemcpy(&hm, mx, sizeof(unsigned), cudaMemcpyDeviceToHost);
  cudaFree(mx);
  float fm;
  std::memcpy(&fm, &hm, sizeof(float));
  int ex = 0;
  std::frexp((double)fm, &ex);
  P->ainv = (float)std::ldexp(1.0, ex - 14);  // 1 / pow2_scale(fm)
  cudaFuncSetAttribute(k_rx_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, RxSmem::total);
  if ((e = cuda_check(c, cudaDeviceSynchronize(), "receiver tables")) != ISG_OK) {
    rxnear_destroy(c);
    return e;
  }
  return ISG_OK;
}

// Forward (r = go x) or adjoint (x = gh r) on blocked vectors, in batches of
// at most 128 right-hand sides.
isg_status rxnear_apply(isg_ctx *c, const float2 *in, float2 *out, int nrhs, int adjoint, cudaStream_t st) {
  RxPlan &P = *c->rx;
  const int Rmax = std::min(c->opts.max_rhs, kRxMaxN / 2);
  for (int j0 = 0; j0 < nrhs; j0 += Rmax) {
    const int R = std::min(Rmax, nrhs - j0);
    const int64_t ldin = adjoint ? P.nrx : P.U, ldout = adjoint ? P.U : P.nrx;
    RxGemmArgs A;
    A.A = adjoint ? P.Aa : P.Af;
    A.kb_total = adjoint ? P.kb_a : P.kb_f;
    const int nsplit = adjoint ? 1 : P.nsplit;
    A.kb_per = adjoint ? A.kb_total : P.kb_per;
    A.x = in + (size_t)j0 * ldin;
    A.ldx = ldin;
    A.kvalid = (int)ldin;
    A.R = R;
    A.npad = std::max(16, (2 * R + 15) / 16 * 16);
    A.rowmax = P.rowmax;
    A.ainv = P.ainv;
    A.adjoint = adjoint;
    A.ldo = ldout;
    A.mvalid = (int)ldout;
    A.err = P.err;
    if (adjoint) {
      A.out = out + (size_t)j0 * ldout;
      A.split_stride = 0;
    } else {
      A.out = P.part;
      A.split_stride = (size_t)R * P.nrx;
    }
    cudaMemsetAsync(P.rowmax, 0, (size_t)R * sizeof(unsigned), st);
    count_launch(2);
    k_rx_rowmax<<<dim3(std::max(1, std::min(64, (int)((ldin + 255) / 256))), R), 256, 0, st>>>(A.x, ldin, A.kvalid,
                                                                                              P.rowmax);
    k_rx_gemm<<<dim3(adjoint ? P.mt_a : P.mt_f, nsplit), kRxThreads, RxSmem::total, st>>>(A);
    if (!adjoint) {
      count_launch();
      k_rx_sum<<<(R * P.nrx + 255) / 256, 256, 0, st>>>(P.part, nsplit, A.split_stride, R, P.nrx,
                                                        out + (size_t)j0 * P.nrx);
    }
  }
  return cuda_check(c, cudaGetLastError(), "receiver GEMM");
}

int rxnear_error(isg_ctx *c) {
  if (!c->rx) return 0;
  int h = 0;
  cudaMemcpy(&h, c->rx->err, sizeof(int), cudaMemcpyDeviceToHost);
  return h;
}

}  // namespace isg
