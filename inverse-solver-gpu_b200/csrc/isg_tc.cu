// Tensor-core engine for the dense leaf stages of the MLFMA matvec on sm_100a.
//
// Near field + L2P (kernels.cu:32-81, 292-319; solve.cpp:170-216) and P2M
// (kernels.cu:6-30; solve.cpp:80-92) are complex GEMMs with a shared,
// translation-invariant operand.  Each runs as a real GEMM through the
// embedding [re, im] x [[re, -im], [im, re]] on tcgen05 (kind::f16, FP32
// accumulation in TMEM).  FP32 accuracy comes from splitting both operands
// into FP16 pairs, v = hi + lo, after a power-of-two scaling of each tile into
// the FP16 range, and summing hi*hi + hi*lo + lo*hi (the lo*lo term is below
// FP32 rounding).
//
// Near-field CTA: a tile of 16 x 8 leaves of one RHS.  Its 18 x 10 halo of
// leaves is stored once in shared memory in the K-major core-matrix layout
// [halo row][16-byte K chunk][halo column], so the operand of each of the nine
// neighbour slots is the same halo seen through a descriptor shifted by one
// halo row / column.  The weights (9 slots x 128 x 128 reals, then the
// L2P basis) stream through a 4-deep ring of 16 KB stages filled by bulk
// async copies.  Warp 1 is the copy producer, thread 0 issues the MMAs, the
// other warps load and convert operands and all warps run the epilogue.
#include <cmath>
#include <cstring>
#include <vector>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "isg_context.hpp"
#include "isg_tc.cuh"

namespace isg {

namespace {

using namespace tc;

constexpr int kTY = 16, kTX = 8;                 // leaves per tile (one 128-row MMA)
constexpr int kPair = 2;                         // tiles per CTA, stacked in y, sharing every weight stage
constexpr int kHR = kPair * kTY + 2, kHC = kTX + 2;  // 34 x 10 halo of the pair
constexpr int kLboA = kHC * 16;                  // 160
constexpr int kSboA = 16 * kLboA;                // 2560 (one halo row: 16 K-chunks)
constexpr int kRegion = kHR * kSboA;             // 87040 bytes per FP16 split
constexpr int kStageBytes = 16384;               // hi [128 x 32] + lo [128 x 32]
constexpr int kStageHalf = 8192;
constexpr int kNB = 3;                           // ring depth
constexpr int kNearStages = 36;                  // 9 slots x 4 K-chunks of 32 reals
constexpr int kLocChunksMax = 20;                // K chunks (8 reals each) of the L2P operand
constexpr int kSboL = kLocChunksMax * 128;       // 2560
constexpr int kL2pTile = 16 * kSboL;             // 40960: one tile's L2P operand per split
constexpr int kLoaders = 224;                    // warps 0, 2..7
constexpr int kErrNearFull = 101, kErrNearEmpty = 102, kErrNearDone = 103, kErrP2m = 111;

struct NearSmem {
  static constexpr int hi = 0, lo = kRegion, stages = 2 * kRegion, bars = stages + kNB * kStageBytes;
  static constexpr int misc = bars + 16 * 8;
  static constexpr int total = misc + 256;
};
static_assert(kPair * kL2pTile <= kRegion, "the L2P operands reuse the halo region");
static_assert(kPair * 128 * 66 * 8 <= 2 * kRegion, "the epilogue tiles reuse the halo region");

__device__ __forceinline__ int loader_id() {
  const int w = threadIdx.x >> 5;
  return w == 0 ? threadIdx.x : threadIdx.x - 32;
}
__device__ __forceinline__ void loaders_bar() { asm volatile("bar.sync 1, %0;\n" ::"n"(kLoaders)); }

// max over the loader threads (named barrier 1)
__device__ float loaders_max(float v, float *scratch) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) scratch[w] = v;
  loaders_bar();
  float m = 0.f;
  for (int q = 0; q < 8; q++)
    if (q != 1) m = fmaxf(m, scratch[q]);
  loaders_bar();
  return m;
}

__device__ __forceinline__ float2 transform(float2 v, float2 g, int mode) {
  if (mode == IN_G) return cmul(g, v);
  if (mode == IN_CONJ) return cconj(v);
  return v;
}

__device__ __forceinline__ float cabs1(float2 v) { return fmaxf(fabsf(v.x), fabsf(v.y)); }

// Stores 4 complex values as one 16-byte chunk of hi and one of lo.
__device__ __forceinline__ void store_chunk(char *smem, int off, const float2 *v, float s) {
  __align__(16) __half h[8], l[8];
#pragma unroll
  for (int p = 0; p < 4; p++) {
    split_f16(v[p].x * s, h[2 * p], l[2 * p]);
    split_f16(v[p].y * s, h[2 * p + 1], l[2 * p + 1]);
  }
  *(uint4 *)(smem + NearSmem::hi + off) = *(uint4 *)h;
  *(uint4 *)(smem + NearSmem::lo + off) = *(uint4 *)l;
}

struct TcNearArgs {
  const float2 *x, *g;  // operator input (transformed by mode)
  const float2 *xe;     // x of the `x - ...` epilogue
  int64_t gstride;
  int mode;
  const int *active;
  const float2 *loc_leaf;  // per-RHS stride mp
  size_t mp;
  int ns;
  const uint8_t *B;  // stages: 36 near + nl2p basis
  int nl2p;          // L2P stages
  float inv_w, inv_b;  // 1 / weight scales
  float2 *y;
  int epi, red;
  const float2 *dot_a;
  double *part;
  int nleaf, U, tiles_x, tiles;
  int loc_vec;  // leaf locals can be copied in 16-byte chunks (ns % 4 == 0, aligned)
  int pair;     // tiles per CTA: kPair, or 1 when the launch is too small to fill the GPU
  const unsigned *locmax;  // when set: [R][kMaxLevels] maxima of the locals (written by M2L), the L2P scale
  int lvl_leaf;
  int tma_x;    // the halo comes by two tensor loads (map tmx)
  int tma_loc;  // the leaf locals come by tensor loads (map tml)
  int *err;
};

// tmx views the input as [RHS][leaf row][4-pixel chunk][leaf column][8 floats]
// and tml the leaf locals as [RHS][leaf row][4-sample chunk][leaf column][8
// floats]: a box of either lands in the staging layout below (first 16 bytes
// of every chunk in the hi slots, the second 16 in the lo slots).
__global__ void __launch_bounds__(256, 1) k_tc_near(TcNearArgs A, const __grid_constant__ CUtensorMap tmx,
                                                    const __grid_constant__ CUtensorMap tml) {
  extern __shared__ __align__(1024) char sm[];
  const int rhs = blockIdx.y;
  if (A.active && !A.active[rhs]) return;
  uint64_t *full = (uint64_t *)(sm + NearSmem::bars);
  uint64_t *empty = full + kNB;
  uint64_t *done = empty + kNB;
  uint64_t *hbar = done + 1, *lbar = done + 2;  // halo, leaf locals landed
  uint32_t *tslot = (uint32_t *)(sm + NearSmem::misc);
  float *fscr = (float *)(sm + NearSmem::misc + 16);      // [8]
  float *scales = (float *)(sm + NearSmem::misc + 48);    // [2]
  double *dscr = (double *)(sm + NearSmem::misc + 64);    // [8][3]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int pair = blockIdx.x;
  const int pty = pair / A.tiles_x, ptx = pair % A.tiles_x;
  const int ty0 = pty * A.pair * kTY, tx0 = ptx * kTX;
  const int tiles_y = (A.nleaf + kTY - 1) / kTY;
  const int ntile = min(A.pair, tiles_y - pty * A.pair);
  const size_t rbase = (size_t)rhs * A.U;
  const float2 *gr = A.g ? A.g + rhs * A.gstride : nullptr;
  const int nstages = kNearStages + A.nl2p;

  if (threadIdx.x == 0) {
    for (int b = 0; b < kNB; b++) {
      mbar_init(&full[b], 1);
      mbar_init(&empty[b], 1);
    }
    mbar_init(done, 1);
    mbar_init(hbar, 1);
    mbar_init(lbar, 1);
    fence_mbar_init();
  }
  if (warp == 0) tmem_alloc(tslot, 512);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;  // near field of tile u in columns [128 u, +128), L2P in [256 + 128 u, +128)

  // ---- halo of the input: every thread stages x as FP32 with cp.async where its
  // FP16 halves will go (first two pixels of a 4-pixel chunk in the hi slot,
  // last two in the lo slot); the loaders then form g x and its max in place,
  // and convert to hi/lo once the pair's scale is known ----
  // (halo row, 4-pixel chunk, halo column): consecutive items are consecutive
  // 16-byte slots, free of bank conflicts
  const int kItems = (A.pair * kTY + 2) * kHC * 16;
  if (threadIdx.x == 32) {
    // the epilogue's x and dot vector rows of the pair, into L2 while the MMAs run
    const uint32_t run = (uint32_t)min(kTX, A.nleaf - tx0) * kBB * 8;
    for (int r = 0; r < ntile * kTY; r++) {
      const int ly = ty0 + r;
      if (ly >= A.nleaf) break;
      const size_t at = rbase + (size_t)(ly * A.nleaf + tx0) * kBB;
      if (A.epi == EPI_FWD || A.epi == EPI_ADJ || A.red == RED_TS) bulk_prefetch_l2(A.xe + at, run);
      if (A.red == RED_DOT) bulk_prefetch_l2(A.dot_a + at, run);
    }
  }
  if (A.tma_x) {
    // two tensor loads: pixels 0, 1 of every chunk to the hi slots, 2, 3 to the lo slots
    if (threadIdx.x == 0) {
      mbar_expect_tx(hbar, 2 * kItems * 16);
      tma_load_5d(sm + NearSmem::hi, &tmx, 0, tx0 - 1, 0, ty0 - 1, rhs, hbar);
      tma_load_5d(sm + NearSmem::lo, &tmx, 4, tx0 - 1, 0, ty0 - 1, rhs, hbar);
    }
    mbar_wait(hbar, 0, A.err, kErrNearFull);
  } else {
    for (int it = threadIdx.x; it < kItems; it += blockDim.x) {
      const int hc = it % kHC, c = (it / kHC) & 15, hr = it / (kHC * 16);
      const int ly = ty0 - 1 + hr, lx = tx0 - 1 + hc;
      const bool in = ly >= 0 && ly < A.nleaf && lx >= 0 && lx < A.nleaf;
      const size_t i = in ? (size_t)(ly * A.nleaf + lx) * kBB + 4 * c : 0;
      const int off = hr * kSboA + c * kLboA + hc * 16;
      cp_async16z(sm + NearSmem::hi + off, A.x + rbase + i, in);
      cp_async16z(sm + NearSmem::lo + off, A.x + rbase + i + 2, in);
    }
    cp_async_wait_all();
  }
  __syncthreads();

  if (warp == 1) {
    // ---- producer: weight stages through the ring ----
    if (lane == 0) {
      for (int t = 0; t < nstages; t++) {
        const int b = t % kNB;
        if (t >= kNB && !mbar_wait(&empty[b], ((t / kNB) - 1) & 1, A.err, kErrNearEmpty)) break;
        mbar_expect_tx(&full[b], kStageBytes);
        bulk_g2s(sm + NearSmem::stages + b * kStageBytes, A.B + (size_t)t * kStageBytes, kStageBytes, &full[b]);
      }
    }
  } else {
    const int li = loader_id();
    float mx = 0.f;
#pragma unroll 8
    for (int it = li; it < kItems; it += kLoaders) {
      const int hc = it % kHC, c = (it / kHC) & 15, hr = it / (kHC * 16);
      const int off = hr * kSboA + c * kLboA + hc * 16;
      float4 *ph = (float4 *)(sm + NearSmem::hi + off), *pl = (float4 *)(sm + NearSmem::lo + off);
      float4 g0 = make_float4(0.f, 0.f, 0.f, 0.f), g1 = g0;
      if (A.mode == IN_G) {
        const int ly = ty0 - 1 + hr, lx = tx0 - 1 + hc;
        if (ly >= 0 && ly < A.nleaf && lx >= 0 && lx < A.nleaf) {
          const size_t i = (size_t)(ly * A.nleaf + lx) * kBB + 4 * c;
          g0 = *(const float4 *)(gr + i);
          g1 = *(const float4 *)(gr + i + 2);
        }
      }
      const float4 a0 = *ph, a1 = *pl;
      const float2 v0 = transform(make_float2(a0.x, a0.y), make_float2(g0.x, g0.y), A.mode);
      const float2 v1 = transform(make_float2(a0.z, a0.w), make_float2(g0.z, g0.w), A.mode);
      const float2 v2 = transform(make_float2(a1.x, a1.y), make_float2(g1.x, g1.y), A.mode);
      const float2 v3 = transform(make_float2(a1.z, a1.w), make_float2(g1.z, g1.w), A.mode);
      mx = fmaxf(mx, fmaxf(fmaxf(cabs1(v0), cabs1(v1)), fmaxf(cabs1(v2), cabs1(v3))));
      *ph = make_float4(v0.x, v0.y, v1.x, v1.y);
      *pl = make_float4(v2.x, v2.y, v3.x, v3.y);
    }
    const float s1 = pow2_scale(loaders_max(mx, fscr));
    for (int it = li; it < kItems; it += kLoaders) {
      const int hc = it % kHC, c = (it / kHC) & 15, hr = it / (kHC * 16);
      const int off = hr * kSboA + c * kLboA + hc * 16;
      const float4 q0 = *(const float4 *)(sm + NearSmem::hi + off), q1 = *(const float4 *)(sm + NearSmem::lo + off);
      const float2 v[4] = {make_float2(q0.x, q0.y), make_float2(q0.z, q0.w), make_float2(q1.x, q1.y),
                           make_float2(q1.z, q1.w)};
      store_chunk(sm, off, v, s1);
    }
    if (li == 0) scales[0] = s1;
    fence_proxy_async();
    loaders_bar();

    // ---- MMA issue: every weight stage serves both tiles of the pair ----
    const uint32_t idesc = idesc_f16_f32(128, 128);
    const uint32_t sbase = smem_u32(sm);
    if (threadIdx.x == 0) {
      tc_fence_after();
      const uint64_t ah0 = smem_desc(sbase + NearSmem::hi, kLboA, kSboA);
      const uint64_t al0 = smem_desc(sbase + NearSmem::lo, kLboA, kSboA);
      const uint64_t bh0 = smem_desc(sbase + NearSmem::stages, 128, 512);
      const uint64_t bl0 = smem_desc(sbase + NearSmem::stages + kStageHalf, 128, 512);
      for (int t = 0; t < kNearStages; t++) {
        const int b = t % kNB;
        if (!mbar_wait(&full[b], (t / kNB) & 1, A.err, kErrNearFull)) break;
        const int s = t >> 2, c = t & 3, dr = s / 3 - 1, dc = s % 3 - 1;
#pragma unroll
        for (int ks = 0; ks < 2; ks++) {
          const uint32_t boff = b * kStageBytes + ks * 256;
          for (int u = 0; u < ntile; u++) {
            const uint32_t aoff = (u * kTY + 1 + dr) * kSboA + (1 + dc) * 16 + (uint32_t)(c * 4 + ks * 2) * kLboA;
            const uint32_t d = tmem + 128 * u;
            mma_f16(d, desc_add(ah0, aoff), desc_add(bh0, boff), idesc, (t | ks) ? 1 : 0);
            mma_f16(d, desc_add(ah0, aoff), desc_add(bl0, boff), idesc, 1);
            mma_f16(d, desc_add(al0, aoff), desc_add(bh0, boff), idesc, 1);
          }
        }
        mma_commit(&empty[b]);
      }
      mma_commit(done);
    }

    // ---- L2P operands: the tiles' leaf locals, staged with cp.async into the
    // halo region once the near-field MMAs are done, then scaled and converted ----
    const int nchunk = (A.ns + 3) / 4;
    const bool vec_ok = A.loc_vec != 0;
    const int kL = ntile * 128 * kLocChunksMax;
    const float2 *lr = A.loc_leaf + (size_t)rhs * A.mp;
    const bool near_ok = mbar_wait(done, 0, A.err, kErrNearDone);
    float s2 = 1.f;
    if (near_ok && A.tma_loc) {
      // one tensor load per tile and slot: samples 0, 1 of every chunk to hi, 2, 3 to lo
      if (li == 0) {
        mbar_expect_tx(lbar, ntile * 2 * kL2pTile);
        for (int u = 0; u < ntile; u++) {
          tma_load_5d(sm + NearSmem::hi + u * kL2pTile, &tml, 0, tx0, 0, ty0 + u * kTY, rhs, lbar);
          tma_load_5d(sm + NearSmem::lo + u * kL2pTile, &tml, 4, tx0, 0, ty0 + u * kTY, rhs, lbar);
        }
      }
      mbar_wait(lbar, 0, A.err, kErrNearFull);
    }
    if (near_ok) {
      for (int it = li; it < kL && !A.tma_loc; it += kLoaders) {
        // (tile, row group, chunk, row in group): consecutive 16-byte slots
        const int m7 = it & 7, c = (it >> 3) % kLocChunksMax, mg = (it >> 3) / kLocChunksMax;
        const int u = mg >> 4, m = ((mg & 15) << 3) | m7;
        const int ly = ty0 + u * kTY + m / kTX, lx = tx0 + m % kTX;
        const bool valid = c < nchunk && ly < A.nleaf && lx < A.nleaf;
        const int off = u * kL2pTile + (m >> 3) * kSboL + c * 128 + (m & 7) * 16;
        const float2 *src = lr + (valid ? (size_t)(ly * A.nleaf + lx) * A.ns + 4 * c : 0);
        if (vec_ok) {
          cp_async16z(sm + NearSmem::hi + off, src, valid);
          cp_async16z(sm + NearSmem::lo + off, src + 2, valid);
        } else {
          float2 v[4];
#pragma unroll
          for (int p = 0; p < 4; p++) v[p] = (valid && 4 * c + p < A.ns) ? src[p] : make_float2(0.f, 0.f);
          *(float4 *)(sm + NearSmem::hi + off) = make_float4(v[0].x, v[0].y, v[1].x, v[1].y);
          *(float4 *)(sm + NearSmem::lo + off) = make_float4(v[2].x, v[2].y, v[3].x, v[3].y);
        }
      }
      cp_async_wait_all();
      loaders_bar();
      if (A.locmax) {  // the leaf level's maximum per RHS, from M2L
        s2 = pow2_scale(__uint_as_float(A.locmax[rhs * kMaxLevels + A.lvl_leaf]));
      } else {
        float mx2 = 0.f;
        for (int it = li; it < kL; it += kLoaders) {
          // (tile, row group, chunk, row in group): consecutive 16-byte slots
          const int m7 = it & 7, c = (it >> 3) % kLocChunksMax, mg = (it >> 3) / kLocChunksMax;
          const int u = mg >> 4, m = ((mg & 15) << 3) | m7;
          const int off = u * kL2pTile + (m >> 3) * kSboL + c * 128 + (m & 7) * 16;
          const float4 q0 = *(const float4 *)(sm + NearSmem::hi + off),
                       q1 = *(const float4 *)(sm + NearSmem::lo + off);
          mx2 = fmaxf(mx2, fmaxf(fmaxf(fabsf(q0.x), fabsf(q0.y)), fmaxf(fabsf(q0.z), fabsf(q0.w))));
          mx2 = fmaxf(mx2, fmaxf(fmaxf(fabsf(q1.x), fabsf(q1.y)), fmaxf(fabsf(q1.z), fabsf(q1.w))));
        }
        s2 = pow2_scale(loaders_max(mx2, fscr));
      }
      for (int it = li; it < kL; it += kLoaders) {
        // (tile, row group, chunk, row in group): consecutive 16-byte slots
        const int m7 = it & 7, c = (it >> 3) % kLocChunksMax, mg = (it >> 3) / kLocChunksMax;
        const int u = mg >> 4, m = ((mg & 15) << 3) | m7;
        const int off = u * kL2pTile + (m >> 3) * kSboL + c * 128 + (m & 7) * 16;
        const float4 q0 = *(const float4 *)(sm + NearSmem::hi + off), q1 = *(const float4 *)(sm + NearSmem::lo + off);
        const float2 v[4] = {make_float2(q0.x, q0.y), make_float2(q0.z, q0.w), make_float2(q1.x, q1.y),
                             make_float2(q1.z, q1.w)};
        store_chunk(sm, off, v, s2);
      }
    } else {
      loaders_bar();  // keeps the named-barrier count of the loaders the same on this path
      if (!A.locmax) (void)loaders_max(0.f, fscr);
    }
    if (li == 0) scales[1] = s2;
    fence_proxy_async();
    loaders_bar();
    if (threadIdx.x == 0) {
      tc_fence_after();
      const uint64_t ah0 = smem_desc(sbase + NearSmem::hi, 128, kSboL);
      const uint64_t al0 = smem_desc(sbase + NearSmem::lo, 128, kSboL);
      const uint64_t bh0 = smem_desc(sbase + NearSmem::stages, 128, 512);
      const uint64_t bl0 = smem_desc(sbase + NearSmem::stages + kStageHalf, 128, 512);
      for (int t = kNearStages; t < nstages; t++) {
        const int b = t % kNB;
        if (!mbar_wait(&full[b], (t / kNB) & 1, A.err, kErrNearFull)) break;
        const int c = t - kNearStages;
#pragma unroll
        for (int ks = 0; ks < 2; ks++) {
          const uint32_t boff = b * kStageBytes + ks * 256;
          for (int u = 0; u < ntile; u++) {
            const uint32_t aoff = u * kL2pTile + (uint32_t)(c * 4 + ks * 2) * 128;
            const uint32_t d = tmem + 256 + 128 * u;
            mma_f16(d, desc_add(ah0, aoff), desc_add(bh0, boff), idesc, (c | ks) ? 1 : 0);
            mma_f16(d, desc_add(ah0, aoff), desc_add(bl0, boff), idesc, 1);
            mma_f16(d, desc_add(al0, aoff), desc_add(bh0, boff), idesc, 1);
          }
        }
        mma_commit(&empty[b]);
      }
      mma_commit(done);
    }
  }

  // ---- epilogue (all warps), in two passes per tile: (1) each thread takes its
  // leaf's 32 pixels out of TMEM (near field and L2P, scaled back) into a padded
  // shared tile [leaf][66 float2] in the halo region, free once the L2P MMAs are
  // done; (2) each warp then takes one leaf at a time, so x, the dot vector and
  // y move as 512 contiguous bytes per warp access ----
  constexpr int kOutLd = 66;  // float2 per leaf row: 16-byte aligned rows, 2-way bank spread
  const int q = warp & 3, hh = warp >> 2;
  const int m = 32 * q + lane;
  const bool need_x = A.epi == EPI_FWD || A.epi == EPI_ADJ || A.red == RED_TS;
  const bool ok = mbar_wait(done, 1, A.err, kErrNearDone);
  __syncthreads();
  tc_fence_after();
  const float inv1 = A.inv_w / scales[0], inv2 = A.inv_b / scales[1];
  for (int u = 0; u < ntile; u++) {
    float2 *ot = (float2 *)(sm + NearSmem::hi) + (size_t)u * 128 * kOutLd;
#pragma unroll
    for (int ch = 0; ch < 4; ch++) {
      const int col = 64 * hh + 16 * ch;
      float d1[16], d2[16];
      tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + 128 * u + col, d1);
      tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + 256 + 128 * u + col, d2);
#pragma unroll
      for (int p = 0; p < 8; p++)
        ot[m * kOutLd + col / 2 + p] =
            make_float2(d1[2 * p] * inv1 + d2[2 * p] * inv2, d1[2 * p + 1] * inv1 + d2[2 * p + 1] * inv2);
    }
  }
  __syncthreads();
  for (int u = 0; u < ntile; u++) {
    const float2 *ot = (const float2 *)(sm + NearSmem::hi) + (size_t)u * 128 * kOutLd;
    double r0 = 0, r1 = 0, r2 = 0;
    // every load of the tile first (one round trip), then the arithmetic and stores
    float4 xv[16], av[16];
    size_t idx[16];
    bool live[16];
#pragma unroll
    for (int r = 0; r < 16; r++) {
      const int e = threadIdx.x + 256 * r, lm = e >> 5, pp = e & 31;  // leaf, pixel pair
      const int ly = ty0 + u * kTY + lm / kTX, lx = tx0 + lm % kTX;
      live[r] = ok && ly < A.nleaf && lx < A.nleaf;
      idx[r] = live[r] ? rbase + (size_t)(ly * A.nleaf + lx) * kBB + 2 * pp : rbase;
      xv[r] = (need_x && live[r]) ? *(const float4 *)(A.xe + idx[r]) : make_float4(0.f, 0.f, 0.f, 0.f);
      av[r] = (A.red == RED_DOT && live[r]) ? *(const float4 *)(A.dot_a + idx[r]) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
#pragma unroll
    for (int r = 0; r < 16; r++) {
      if (!live[r]) continue;
      const int e = threadIdx.x + 256 * r, lm = e >> 5, pp = e & 31;
      const size_t i = idx[r];
      const float4 ov = *(const float4 *)(ot + lm * kOutLd + 2 * pp);
      float2 o[2] = {make_float2(ov.x, ov.y), make_float2(ov.z, ov.w)};
      const float2 xin[2] = {make_float2(xv[r].x, xv[r].y), make_float2(xv[r].z, xv[r].w)};
      if (A.epi == EPI_FWD) {
        o[0] = csub(xin[0], o[0]);
        o[1] = csub(xin[1], o[1]);
      } else if (A.epi == EPI_ADJ) {
        const float4 gv = *(const float4 *)(gr + (i - rbase));
        o[0] = csub(xin[0], cconj(cmul(make_float2(gv.x, gv.y), o[0])));
        o[1] = csub(xin[1], cconj(cmul(make_float2(gv.z, gv.w), o[1])));
      } else if (A.epi == EPI_CONJ) {
        o[0] = cconj(o[0]);
        o[1] = cconj(o[1]);
      }
      *(float4 *)(A.y + i) = make_float4(o[0].x, o[0].y, o[1].x, o[1].y);
      if (A.red == RED_DOT) {
        const float2 a0 = make_float2(av[r].x, av[r].y), a1 = make_float2(av[r].z, av[r].w);
        r0 += (double)a0.x * o[0].x + (double)a0.y * o[0].y + (double)a1.x * o[1].x + (double)a1.y * o[1].y;
        r1 += (double)a0.x * o[0].y - (double)a0.y * o[0].x + (double)a1.x * o[1].y - (double)a1.y * o[1].x;
      } else if (A.red == RED_TS) {
#pragma unroll
        for (int e2 = 0; e2 < 2; e2++) {
          r0 += (double)o[e2].x * xin[e2].x + (double)o[e2].y * xin[e2].y;
          r1 += (double)o[e2].x * xin[e2].y - (double)o[e2].y * xin[e2].x;
          r2 += (double)o[e2].x * o[e2].x + (double)o[e2].y * o[e2].y;
        }
      }
    }
    if (A.red != RED_NONE) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        r0 += __shfl_xor_sync(0xffffffffu, r0, o);
        r1 += __shfl_xor_sync(0xffffffffu, r1, o);
        r2 += __shfl_xor_sync(0xffffffffu, r2, o);
      }
      if (lane == 0) {
        dscr[warp * 3 + 0] = r0;
        dscr[warp * 3 + 1] = r1;
        dscr[warp * 3 + 2] = r2;
      }
    }
    __syncthreads();
    if (A.red != RED_NONE && threadIdx.x == 0) {
      double s0 = 0, s1v = 0, s2v = 0;
      for (int w2 = 0; w2 < 8; w2++) {
        s0 += dscr[w2 * 3 + 0];
        s1v += dscr[w2 * 3 + 1];
        s2v += dscr[w2 * 3 + 2];
      }
      const int tile = (pty * A.pair + u) * A.tiles_x + ptx;
      double *p = A.part + ((size_t)rhs * A.tiles + tile) * 4;
      p[0] = s0;
      p[1] = s1v;
      p[2] = s2v;
      p[3] = 0;
    }
    __syncthreads();  // dscr is reused by the next tile
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, 512);
}

// ---- near field + L2P, persistent and pipelined ----
// Items are pairs of vertically adjacent 16 x 8-leaf tiles of one RHS; a
// persistent CTA walks them in steps of gridDim.x.  An item's K dimension (9
// neighbour slots x 128 source reals of the halo, then 2 ns reals of the leaf
// locals for L2P) is staged in shared memory one A-stage at a time: a halo
// K-group (32 source reals of every leaf of the pair's 34 x 10-leaf halo)
// feeds the nine weight stages of its K range; an L2P stage (32 reals of the
// locals of the pair's 256 leaves) feeds one.  Stage order: H0 H1 H2 H3 L0 ..
// L4; the weights are packed in the same order.  An A-stage arrives as FP32 by
// one tensor load whose rows are a leaf's 32 reals (128 contiguous bytes) into
// a staging buffer, and the converters write it as FP16 hi/lo in the MMA's
// core-matrix layout into an operand buffer.  The whole halo is never
// resident, so two staging buffers, two operand buffers and a three-deep
// weight ring fit in shared memory and the roles overlap:
//   warp 0      tensor loads of the A-stages (4-D maps, no multicast)
//   warp 1      bulk copies of the weight stages
//   warp 2      MMA issue (one thread)
//   warps 3..6  A-stage conversion to FP16 hi/lo
//   warps 7..14 epilogue, two per TMEM lane quarter (columns 0..63, 64..127)
// Near field and L2P accumulate into one TMEM accumulator per tile: the input
// is scaled by the power of two that P2M's per-RHS maximum gives and the
// locals by M2L's, each lowered until both products carry the same power of
// two.  Two accumulator sets (two tiles x 128 columns each) alternate between
// items, so an item's epilogue runs under the next item's MMAs.
constexpr int kNpKC = 4;                                       // 8-real K-chunks per A-stage
constexpr int kNpHaloSplit = kHR * kNpKC * kHC * 16;           // 21760: one FP16 split of a halo K-group
constexpr int kNpL2pSplit = kPair * kTY * kNpKC * kTX * 16;    // 16384: one FP16 split of an L2P stage
constexpr int kNpBuf = 2 * kNpHaloSplit;                       // 43520: an operand (hi, lo) or a staged A-stage
constexpr int kNpHaloBytes = kHR * kHC * 32 * 4;               // 43520: a halo K-group as FP32
constexpr int kNpL2pBytes = kPair * kTY * kTX * 32 * 4;        // 32768: an L2P stage as FP32
constexpr int kNpNS = 2, kNpNO = 2, kNpNB = 3;                 // staging, operand buffers, weight ring depth
constexpr int kNpConvWarp0 = 3, kNpConvWarps = 4, kNpEpiWarp0 = 7, kNpEpiWarps = 8;
constexpr int kNpThreads = 32 * (kNpEpiWarp0 + kNpEpiWarps);  // 480
constexpr int kNpConv = 32 * kNpConvWarps, kNpEpi = 32 * kNpEpiWarps;
constexpr int kInMaxSlot = kMaxLevels - 1;                     // levmax slot of P2M's input maximum
constexpr int kErrNp = 121;
struct NpSmem {
  static constexpr int s = 0;                                  // kNpNS FP32 staging buffers
  static constexpr int o = kNpNS * kNpBuf;                     // kNpNO FP16 hi/lo operand buffers
  static constexpr int b = o + kNpNO * kNpBuf;                 // kNpNB weight stages
  static constexpr int bars = b + kNpNB * kStageBytes;         // 19 mbarriers
  static constexpr int misc = bars + 24 * 8;                   // TMEM base, abort flag
  static constexpr int dscr = misc + 16;                       // [2][kNpEpiWarps][3] double
  static constexpr int total = dscr + 2 * kNpEpiWarps * 3 * 8;
};
static_assert(kNpBuf % 128 == 0 && NpSmem::o % 128 == 0, "tensor-load destinations are 128-byte aligned");
static_assert(kNpHaloBytes <= kNpBuf && kNpL2pBytes <= kNpBuf && 2 * kNpL2pSplit <= kNpBuf, "buffer sizes");
static_assert(NpSmem::total <= 227 * 1024, "shared memory of one CTA");

// A-stage a of an item: returns 0 (halo K-group a, a < 4) or 1 (L2P stage
// a - 4) and its index.  The L2P stages come last: tensor-core accumulation
// rounds each step against the running sum, and interleaving the L2P terms
// into the near-field sum measured 2x the operator error (5.5e-6 against
// 2.5e-6 relative to FP64 on random inputs).
__host__ __device__ inline int np_stage(int a, int nl2p, int &idx) {
  (void)nl2p;
  if (a < 4) {
    idx = a;
    return 0;
  }
  idx = a - 4;
  return 1;
}

// A dot product's terms over one epilogue chunk at FP32 instruction cost:
// each product a b is split exactly into its rounded value p and its rounding
// error fma(a, b, -p) (Dekker's TwoProduct); the p go round-robin into four
// independent FP32 partial sums (short dependency chains), the errors into a
// fifth, and the five are added into the FP64 sum once per chunk.  Each
// partial sum rounds three times over a 16-term chunk, below the rounding of
// the complex64 vectors themselves; the _rn intrinsics keep the compiler from
// contracting the exact split.  (Converting every product to FP64 cost 1.75
// ms of a 4.4 ms 256-RHS launch; Kahan compensation, a four-add dependency
// chain per term, cost more than that.)
struct Acc32 {
  float p[4] = {0.f, 0.f, 0.f, 0.f}, e = 0.f;
  __device__ __forceinline__ void add_prod(int j, float a, float b) {
    const float q = __fmul_rn(a, b);
    e = __fadd_rn(e, fmaf(a, b, -q));
    p[j & 3] = __fadd_rn(p[j & 3], q);
  }
  __device__ __forceinline__ double take() {
    const double v = (((double)p[0] + (double)p[1]) + ((double)p[2] + (double)p[3])) + (double)e;
    p[0] = p[1] = p[2] = p[3] = e = 0.f;
    return v;
  }
};

struct TcNearPipeArgs {
  const float2 *x, *g;  // operator input (transformed by mode)
  const float2 *xe;     // x of the `x - ...` epilogue
  int64_t gstride;
  int mode;
  const int *active;
  const uint8_t *B;  // weight stages in A-stage order
  int nl2p;
  float sw, sb;      // power-of-two scales of the near-field weights and the L2P basis
  const unsigned *levmax, *locmax;  // [R][kMaxLevels]: P2M's input maximum (slot kInMaxSlot), M2L's locals
  int lvl_leaf;
  float2 *y;
  int epi, red;
  const float2 *dot_a;
  double *part;
  int nleaf, U, tiles_x, tiles_y, tiles, ppr, nitems;
  int *err;
};

// The item's operand scales: input s1 and locals s2 lowered to a common product scale p = s1 sw = s2 sb.
// A zero maximum (an all-zero input or locals) leaves the other operand's scale alone.
__device__ __forceinline__ void np_scales(const TcNearPipeArgs &A, int rhs, float &s1, float &s2, float &p) {
  const float mx = __uint_as_float(A.levmax[rhs * kMaxLevels + kInMaxSlot]);
  const float ml = __uint_as_float(A.locmax[rhs * kMaxLevels + A.lvl_leaf]);
  const float a = mx > 0.f ? pow2_scale(mx) * A.sw : INFINITY;
  const float b = ml > 0.f ? pow2_scale(ml) * A.sb : INFINITY;
  p = fminf(a, b);
  if (!(p < INFINITY)) p = A.sw;
  s1 = p / A.sw;
  s2 = p / A.sb;
}

__global__ void __launch_bounds__(kNpThreads, 1) k_tc_near_pipe(TcNearPipeArgs A, const __grid_constant__ CUtensorMap tmh,
                                                                const __grid_constant__ CUtensorMap tml) {
  extern __shared__ __align__(1024) char sm[];
  uint64_t *sfull = (uint64_t *)(sm + NpSmem::bars);  // staging landed / read out
  uint64_t *sfree = sfull + kNpNS;
  uint64_t *ofull = sfree + kNpNS, *ofree = ofull + kNpNO;  // operand converted / consumed by the MMAs
  uint64_t *bfull = ofree + kNpNO, *bempty = bfull + kNpNB;
  uint64_t *tfull = bempty + kNpNB, *tfree = tfull + 2, *mdone = tfree + 2;
  uint32_t *tslot = (uint32_t *)(sm + NpSmem::misc);
  volatile int *abort = (volatile int *)(sm + NpSmem::misc + 4);
  double *dscr = (double *)(sm + NpSmem::dscr);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int i = 0; i < 2 * kNpNS + 2 * kNpNO + 2 * kNpNB + 5; i++) mbar_init(sfull + i, 1);
    *abort = 0;
    fence_mbar_init();
  }
  if (warp == 0) tmem_alloc(tslot, 512);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;  // set s, tile u: columns [256 s + 128 u, +128)
  const int na = 4 + A.nl2p;     // A-stages per item
  const int nb = 36 + A.nl2p;    // weight stages per item
  auto next_item = [&](int w) {
    do w += gridDim.x;
    while (w < A.nitems && A.active && !A.active[w / A.ppr]);
    return w;
  };
  const int first = (A.active && blockIdx.x < A.nitems && !A.active[blockIdx.x / A.ppr]) ? next_item(blockIdx.x)
                                                                                           : blockIdx.x;
  auto geom = [&](int w, int &rhs, int &ty0, int &tx0, int &ntile) {
    rhs = w / A.ppr;
    const int pr = w % A.ppr, pty = pr / A.tiles_x, ptx = pr % A.tiles_x;
    ty0 = pty * kPair * kTY;
    tx0 = ptx * kTX;
    ntile = min(kPair, A.tiles_y - pty * kPair);
  };

  if (warp == 0) {
    // ---- A-stage tensor loads into the staging buffers: rows of 32 reals ----
    if (lane == 0) {
      int ka = 0;
      const bool pre_x = A.epi == EPI_FWD || A.epi == EPI_ADJ || A.red == RED_TS;
      for (int w = first; w < A.nitems && !*abort; w = next_item(w)) {
        int rhs, ty0, tx0, ntile;
        geom(w, rhs, ty0, tx0, ntile);
        // the rows the epilogue will read for this item (x, the dot vector, g), into L2
        // about one item ahead of it: its loads then wait on L2, not on HBM
        {
          const uint32_t run = (uint32_t)min(kTX, A.nleaf - tx0) * kBB * 8;
          const size_t rb = (size_t)rhs * A.U;
          for (int r = 0; r < ntile * kTY && ty0 + r < A.nleaf; r++) {
            const size_t at = (size_t)((ty0 + r) * A.nleaf + tx0) * kBB;
            if (pre_x) bulk_prefetch_l2(A.xe + rb + at, run);
            if (A.red == RED_DOT) bulk_prefetch_l2(A.dot_a + rb + at, run);
            if (A.epi == EPI_ADJ) bulk_prefetch_l2(A.g + rhs * A.gstride + at, run);
          }
        }
        for (int a = 0; a < na; a++, ka++) {
          const int i = ka % kNpNS;
          if (!mbar_wait_or(sfree + i, ((ka / kNpNS) & 1) ^ 1, abort, A.err, kErrNp)) break;
          char *dst = sm + NpSmem::s + i * kNpBuf;
          int idx;
          if (np_stage(a, A.nl2p, idx) == 0) {
            mbar_expect_tx(sfull + i, kNpHaloBytes);
            tma_load_4d(dst, &tmh, 32 * idx, tx0 - 1, ty0 - 1, rhs, sfull + i);
          } else {
            mbar_expect_tx(sfull + i, kNpL2pBytes);
            tma_load_4d(dst, &tml, 32 * idx, tx0, ty0, rhs, sfull + i);
          }
        }
      }
      // every load issued has landed before the CTA exits (bounded waits)
      for (int j = 1; j <= kNpNS && j <= ka; j++) {
        const int kk = ka - j;
        mbar_wait(sfull + kk % kNpNS, (kk / kNpNS) & 1, A.err, kErrNp);
      }
    }
  } else if (warp == 1) {
    // ---- weight stages through the ring, in A-stage order ----
    if (lane == 0) {
      int kb = 0;
      for (int w = first; w < A.nitems && !*abort; w = next_item(w)) {
        for (int t = 0; t < nb; t++, kb++) {
          const int b = kb % kNpNB;
          if (!mbar_wait_or(bempty + b, ((kb / kNpNB) & 1) ^ 1, abort, A.err, kErrNp)) break;
          mbar_expect_tx(bfull + b, kStageBytes);
          bulk_g2s(sm + NpSmem::b + b * kStageBytes, A.B + (size_t)t * kStageBytes, kStageBytes, bfull + b);
        }
      }
      for (int j = 1; j <= kNpNB && j <= kb; j++) {
        const int kk = kb - j;
        mbar_wait(bfull + kk % kNpNB, (kk / kNpNB) & 1, A.err, kErrNp);
      }
    }
  } else if (warp == 2) {
    // ---- MMA issue (one thread): D[128 target reals][256 leaves of the pair] +=
    // weights (A, M = 128) x data (B, N = 256): both tiles in one instruction, so
    // each weight stage is 2 K-steps x 3 split products ----
    if (lane == 0) {
      const uint32_t idesc = idesc_f16_f32(128, 2 * 128), sbase = smem_u32(sm);
      int ka = 0, kb = 0, it = 0;
      bool ok = true;
      for (int w = first; w < A.nitems && ok; w = next_item(w), it++) {
        const int set = it & 1;
        const uint32_t d = tmem + (uint32_t)(set * 256);
        ok = mbar_wait_or(tfree + set, ((it >> 1) & 1) ^ 1, abort, A.err, kErrNp);
        for (int a = 0; a < na && ok; a++, ka++) {
          const int i = ka % kNpNO;
          ok = mbar_wait_or(ofull + i, (ka / kNpNO) & 1, abort, A.err, kErrNp);
          int idx;
          const int kind = np_stage(a, A.nl2p, idx);
          const uint32_t obase = sbase + NpSmem::o + i * kNpBuf;
          const uint32_t lbo = kind == 0 ? kHC * 16 : kTX * 16;  // K-adjacent core matrices
          const uint64_t dh0 = smem_desc(obase, lbo, kNpKC * lbo);
          const uint64_t dl0 = smem_desc(obase + (kind == 0 ? kNpHaloSplit : kNpL2pSplit), lbo, kNpKC * lbo);
          const int nq = kind == 0 ? 9 : 1;
          for (int q = 0; q < nq && ok; q++, kb++) {
            const int b = kb % kNpNB;
            ok = mbar_wait_or(bfull + b, (kb / kNpNB) & 1, abort, A.err, kErrNp);
            tc_fence_after();
            if (!ok) break;
            const uint32_t bb = sbase + NpSmem::b + b * kStageBytes;
            const uint64_t wh0 = smem_desc(bb, 128, 512), wl0 = smem_desc(bb + kStageHalf, 128, 512);
            // neighbour slot q: the pair's 32 leaf rows start at halo row 1 + dr, column 1 + dc
            const uint32_t doff0 = kind == 0 ? (uint32_t)((q / 3) * (kNpKC * kHC * 16) + (q % 3) * 16) : 0u;
#pragma unroll
            for (int ks = 0; ks < 2; ks++) {
              const uint32_t doff = doff0 + (uint32_t)ks * 2 * lbo;
              const int acc = (a | q | ks) ? 1 : 0;
              mma_f16(d, desc_add(wh0, ks * 256), desc_add(dh0, doff), idesc, acc);
              mma_f16(d, desc_add(wh0, ks * 256), desc_add(dl0, doff), idesc, 1);
              mma_f16(d, desc_add(wl0, ks * 256), desc_add(dh0, doff), idesc, 1);
            }
            mma_commit(bempty + b);
          }
          if (ok) mma_commit(ofree + i);
        }
        if (ok) mma_commit(tfull + set);
      }
      // every MMA issued is complete before the CTA frees TMEM (bounded wait)
      mma_commit(mdone);
      mbar_wait(mdone, 0, A.err, kErrNp);
    }
  } else if (warp < kNpEpiWarp0) {
    // ---- converters: a staged FP32 A-stage becomes the FP16 hi/lo operand.  One
    // unit is a 4-complex chunk (32 bytes) of one leaf: staging [row][col][32 reals]
    // to operand [row][chunk][col][16 bytes], hi then lo ----
    const int ct = threadIdx.x - 32 * kNpConvWarp0;
    int ka = 0;
    for (int w = first; w < A.nitems; w = next_item(w)) {
      int rhs, ty0, tx0, ntile;
      geom(w, rhs, ty0, tx0, ntile);
      float s1, s2, p;
      np_scales(A, rhs, s1, s2, p);
      const float2 *gr = A.g ? A.g + rhs * A.gstride : nullptr;
      for (int a = 0; a < na; a++, ka++) {
        const int i = ka % kNpNS, o = ka % kNpNO;
        const bool ok = mbar_wait_or(sfull + i, (ka / kNpNS) & 1, abort, A.err, kErrNp) &&
                        mbar_wait_or(ofree + o, ((ka / kNpNO) & 1) ^ 1, abort, A.err, kErrNp);
        const float4 *st = (const float4 *)(sm + NpSmem::s + i * kNpBuf);
        char *hi = sm + NpSmem::o + o * kNpBuf;
        int idx;
        if (np_stage(a, A.nl2p, idx) == 0) {
          char *lo = hi + kNpHaloSplit;
          for (int e = ct; e < kHR * kHC * kNpKC && ok; e += kNpConv) {
            const int c = e & 3, hc = (e >> 2) % kHC, hr = (e >> 2) / kHC;
            const float4 a0 = st[2 * e], a1 = st[2 * e + 1];  // staging offset ((hr * 10 + hc) * 32 + 8 c) reals
            float4 g0 = make_float4(0.f, 0.f, 0.f, 0.f), g1 = g0;
            if (A.mode == IN_G) {
              const int ly = ty0 - 1 + hr, lx = tx0 - 1 + hc;
              if (ly >= 0 && ly < A.nleaf && lx >= 0 && lx < A.nleaf) {
                const size_t gi = (size_t)(ly * A.nleaf + lx) * kBB + 16 * idx + 4 * c;
                g0 = *(const float4 *)(gr + gi);
                g1 = *(const float4 *)(gr + gi + 2);
              }
            }
            const float2 v0 = transform(make_float2(a0.x, a0.y), make_float2(g0.x, g0.y), A.mode);
            const float2 v1 = transform(make_float2(a0.z, a0.w), make_float2(g0.z, g0.w), A.mode);
            const float2 v2 = transform(make_float2(a1.x, a1.y), make_float2(g1.x, g1.y), A.mode);
            const float2 v3 = transform(make_float2(a1.z, a1.w), make_float2(g1.z, g1.w), A.mode);
            uint32_t h[4], l[4];
            split2u(v0.x * s1, v0.y * s1, h[0], l[0]);
            split2u(v1.x * s1, v1.y * s1, h[1], l[1]);
            split2u(v2.x * s1, v2.y * s1, h[2], l[2]);
            split2u(v3.x * s1, v3.y * s1, h[3], l[3]);
            const int off = ((hr * kNpKC + c) * kHC + hc) * 16;
            st_shared_v4(hi + off, h);
            st_shared_v4(lo + off, l);
          }
        } else {
          char *lo = hi + kNpL2pSplit;
          for (int e = ct; e < kPair * kTY * kTX * kNpKC && ok; e += kNpConv) {
            const int c = e & 3, col = (e >> 2) & (kTX - 1), row = e >> 5;
            const float4 a0 = st[2 * e], a1 = st[2 * e + 1];  // staging offset ((row * 8 + col) * 32 + 8 c) reals
            uint32_t h[4], l[4];
            split2u(a0.x * s2, a0.y * s2, h[0], l[0]);
            split2u(a0.z * s2, a0.w * s2, h[1], l[1]);
            split2u(a1.x * s2, a1.y * s2, h[2], l[2]);
            split2u(a1.z * s2, a1.w * s2, h[3], l[3]);
            const int off = ((row * kNpKC + c) * kTX + col) * 16;
            st_shared_v4(hi + off, h);
            st_shared_v4(lo + off, l);
          }
        }
        fence_proxy_async();
        named_sync(1, kNpConv);
        if (ct == 0) {
          mbar_arrive(sfree + i);
          mbar_arrive(ofull + o);
        }
      }
    }
  } else {
    // ---- epilogue: TMEM lane = target real (pixel 16 qd + lane / 2, real part on
    // even lanes), column = leaf of the pair; the warp's 32 lanes are 128 contiguous
    // bytes of one leaf's output, so every load and store is one coalesced row.
    // Warps 7..10 take the pair's first tile (columns 0..127), 11..14 the second ----
    const int ew = warp - kNpEpiWarp0, qd = warp & 3, hh = ew >> 2;
    const bool odd = lane & 1;
    const bool need_x = A.epi == EPI_FWD || A.epi == EPI_ADJ || A.red == RED_TS;
    const float *xf = (const float *)A.xe, *af = (const float *)A.dot_a;
    float *yf = (float *)A.y;
    int it = 0;
    for (int w = first; w < A.nitems; w = next_item(w), it++) {
      int rhs, ty0, tx0, ntile;
      geom(w, rhs, ty0, tx0, ntile);
      const int set = it & 1;
      float s1, s2, p;
      np_scales(A, rhs, s1, s2, p);
      const float inv = 1.f / p;
      const bool ok = mbar_wait_or(tfull + set, (it >> 1) & 1, abort, A.err, kErrNp);
      tc_fence_after();
      const size_t rbase = (size_t)rhs * A.U;
      const float *gf = A.g ? (const float *)(A.g + rhs * A.gstride) : nullptr;
      const float *xr = xf + 2 * rbase, *ar = af + 2 * rbase;
      float *yr = yf + 2 * rbase;
      double r0 = 0, r1 = 0, r2 = 0;
      Acc32 q0, q1, q2;
      if (hh < ntile) {  // warp-uniform
        // chunks of 8 leaves (one leaf row of the tile); the loads of chunk ch + 1 are in
        // flight while chunk ch is computed and stored
        const int lyb = ty0 + hh * kTY;
        auto fidx = [&](int ch, int j) { return 2 * ((lyb + ch) * A.nleaf + tx0 + j) * kBB + 32 * qd + lane; };
        auto load = [&](int ch, float (&xv)[8], float (&av)[8], float (&gv)[8], unsigned &live) {
          live = 0;
#pragma unroll
          for (int j = 0; j < 8; j++) {
            const bool lv = ok && lyb + ch < A.nleaf && tx0 + j < A.nleaf;
            live |= lv ? 1u << j : 0u;
            const int fi = fidx(ch, j);
            xv[j] = (need_x && lv) ? xr[fi] : 0.f;
            av[j] = (A.red == RED_DOT && lv) ? ar[fi] : 0.f;
            gv[j] = (A.epi == EPI_ADJ && lv) ? gf[fi] : 0.f;
          }
        };
        auto process = [&](int ch, const float (&xv)[8], const float (&av)[8], const float (&gv)[8], unsigned live) {
          float d[8];
          tmem_ld8(tmem + ((uint32_t)(32 * qd) << 16) + (uint32_t)(set * 256 + 128 * hh + 8 * ch), d);
#pragma unroll
          for (int j = 0; j < 8; j++) {
            if (!((live >> j) & 1)) continue;  // warp-uniform
            const float o = d[j] * inv;
            float v = o;
            if (A.epi == EPI_FWD) {
              v = xv[j] - o;
            } else if (A.epi == EPI_ADJ) {  // x - conj(g o)
              const float op = __shfl_xor_sync(0xffffffffu, o, 1), gp = __shfl_xor_sync(0xffffffffu, gv[j], 1);
              v = odd ? xv[j] + (gp * o + gv[j] * op) : xv[j] - (gv[j] * o - gp * op);
            } else if (A.epi == EPI_CONJ) {
              v = odd ? -o : o;
            }
            yr[fidx(ch, j)] = v;
            if (A.red == RED_DOT) {  // conj(a) y
              const float vp = __shfl_xor_sync(0xffffffffu, v, 1);
              q0.add_prod(j, av[j], v);
              q1.add_prod(j, odd ? -av[j] : av[j], vp);
            } else if (A.red == RED_TS) {  // conj(y) x and |y|^2
              const float xp = __shfl_xor_sync(0xffffffffu, xv[j], 1);
              q0.add_prod(j, v, xv[j]);
              q1.add_prod(j, odd ? -v : v, xp);
              q2.add_prod(j, v, v);
            }
          }
          if (A.red != RED_NONE && (ch & 1)) {  // two chunks' FP32 partial sums into the FP64 ones
            r0 += q0.take();
            r1 += q1.take();
            r2 += q2.take();
          }
        };
        float xa[8], aa[8], ga[8], xb[8], ab[8], gb[8];
        unsigned la, lb;
        load(0, xa, aa, ga, la);
#pragma unroll 1
        for (int ch = 0; ch < 16; ch += 2) {
          load(ch + 1, xb, ab, gb, lb);
          process(ch, xa, aa, ga, la);
          if (ch + 2 < 16) load(ch + 2, xa, aa, ga, la);
          process(ch + 1, xb, ab, gb, lb);
        }
      }
      if (A.red != RED_NONE) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          r0 += __shfl_xor_sync(0xffffffffu, r0, o);
          r1 += __shfl_xor_sync(0xffffffffu, r1, o);
          r2 += __shfl_xor_sync(0xffffffffu, r2, o);
        }
        if (lane == 0) {
          double *ds = dscr + (set * kNpEpiWarps + ew) * 3;
          ds[0] = r0;
          ds[1] = r1;
          ds[2] = r2;
        }
      }
      tc_fence_before();
      named_sync(2, kNpEpi);  // the accumulator set is read out, the warps' sums are in dscr
      if (ew == 0 && lane == 0) {
        mbar_arrive(tfree + set);
        if (A.red != RED_NONE && ok) {
          double s0 = 0, s1v = 0, s2v = 0;
          for (int k = 0; k < kNpEpiWarps; k++) {
            const double *ds = dscr + (set * kNpEpiWarps + k) * 3;
            s0 += ds[0];
            s1v += ds[1];
            s2v += ds[2];
          }
          // the pair's sum goes to its first tile's slot, zero to the second's
          const int pr = w % A.ppr, pty = pr / A.tiles_x, ptx = pr % A.tiles_x;
          for (int u = 0; u < ntile; u++) {
            double *pp = A.part + ((size_t)rhs * A.tiles + (pty * kPair + u) * A.tiles_x + ptx) * 4;
            pp[0] = u ? 0.0 : s0;
            pp[1] = u ? 0.0 : s1v;
            pp[2] = u ? 0.0 : s2v;
            pp[3] = 0.0;
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, 512);
}

// ---- P2M: persistent CTAs over (RHS, 128-leaf tile) items, N = 2 ns padded to 16 ----
// The coefficient matrix is loaded once per CTA; each item's input is loaded
// into registers while the previous item's outputs are written, converted to
// FP16 hi/lo, multiplied, and its multipoles go back through shared memory so
// that the 128 consecutive leaf rings are written as one contiguous block.
constexpr int kP2mA = 16 * 2048;  // one FP16 split of the [128 x 128] operand
struct P2mSmem {
  static constexpr int hi = 0, lo = kP2mA, b = 2 * kP2mA;
  // then: B (4 stages), output tile [128][ns + 1] float2, barriers
  __host__ __device__ static size_t out(int stage_bytes) { return (size_t)b + 4 * (size_t)stage_bytes; }
  __host__ __device__ static size_t bars(int stage_bytes, int ns) { return (out(stage_bytes) + (size_t)128 * (ns + 1) * 8 + 15) & ~(size_t)15; }
  __host__ __device__ static size_t total(int stage_bytes, int ns) { return bars(stage_bytes, ns) + 64; }
};

struct TcP2mArgs {
  const float2 *x, *g;
  int64_t gstride;
  int mode;
  const int *active;
  const uint8_t *B;  // 4 stages of [npad x 32] hi then lo
  int npad, stage_bytes;
  float inv_c;
  float2 *mul_leaf;
  size_t mp;
  int ns, nleaves, U, tiles, nitems;
  int *err;
  unsigned *levmax;  // [R][kMaxLevels]: this level's max |re|, |im| per RHS (FP32 bits)
  int lvl;
};

__global__ void __launch_bounds__(256, 1) k_tc_p2m(TcP2mArgs A) {
  extern __shared__ __align__(1024) char sm[];
  float2 *osm = (float2 *)(sm + P2mSmem::out(A.stage_bytes));
  uint64_t *bar = (uint64_t *)(sm + P2mSmem::bars(A.stage_bytes, A.ns));
  uint64_t *done = bar + 1;
  uint32_t *tslot = (uint32_t *)(bar + 2);
  float *fscr = (float *)(bar + 3);  // [8]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    mbar_init(done, 1);
    fence_mbar_init();
  }
  if (warp == 0) tmem_alloc(tslot, 256);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const int bbytes = 4 * A.stage_bytes;
  if (threadIdx.x == 0) {
    mbar_expect_tx(bar, bbytes);
    for (int c = 0; c < 4; c++)
      bulk_g2s(sm + P2mSmem::b + c * A.stage_bytes, A.B + (size_t)c * A.stage_bytes, A.stage_bytes, bar);
  }
  auto active_item = [&](int w) {
    while (w < A.nitems && A.active && !A.active[w / A.tiles]) w += gridDim.x;
    return w;
  };
  // one item's input: 128 leaves x 16 chunks of 4 pixels, 8 chunks per thread;
  // chunk r of thread t is (row group, chunk, row in group) = it >> 7, (it >> 3) & 15, it & 7
  constexpr int kPer = 128 * 16 / 256;
  float2 v[kPer][4];
  auto load = [&](int w, float &mx) {
    const int rhs = w / A.tiles, leaf0 = (w % A.tiles) * 128;
    const size_t rbase = (size_t)rhs * A.U;
    const float2 *gr = A.g ? A.g + rhs * A.gstride : nullptr;
    mx = 0.f;
#pragma unroll
    for (int r = 0; r < kPer; r++) {
      const int it = threadIdx.x + r * 256;
      const int m = ((it >> 7) << 3) | (it & 7), c = (it >> 3) & 15, leaf = leaf0 + m;
#pragma unroll
      for (int p = 0; p < 4; p++) v[r][p] = make_float2(0.f, 0.f);
      if (leaf < A.nleaves) {
        const size_t i = (size_t)leaf * kBB + 4 * c;
        const float4 a0 = *(const float4 *)(A.x + rbase + i), a1 = *(const float4 *)(A.x + rbase + i + 2);
        float4 g0 = make_float4(0.f, 0.f, 0.f, 0.f), g1 = g0;
        if (A.mode == IN_G) {
          g0 = *(const float4 *)(gr + i);
          g1 = *(const float4 *)(gr + i + 2);
        }
        v[r][0] = transform(make_float2(a0.x, a0.y), make_float2(g0.x, g0.y), A.mode);
        v[r][1] = transform(make_float2(a0.z, a0.w), make_float2(g0.z, g0.w), A.mode);
        v[r][2] = transform(make_float2(a1.x, a1.y), make_float2(g1.x, g1.y), A.mode);
        v[r][3] = transform(make_float2(a1.z, a1.w), make_float2(g1.z, g1.w), A.mode);
#pragma unroll
        for (int p = 0; p < 4; p++) mx = fmaxf(mx, cabs1(v[r][p]));
      }
    }
  };
  const uint32_t sbase = smem_u32(sm);
  const uint32_t idesc = idesc_f16_f32(128, A.npad);
  const int nchunks = A.npad / 16;
  const int q = warp & 3, hh = warp >> 2;
  const int c0 = hh ? (nchunks + 1) / 2 : 0, c1 = hh ? nchunks : (nchunks + 1) / 2;
  bool ok = mbar_wait(bar, 0, A.err, kErrP2m);  // the coefficients
  int parity = 0;
  int w = active_item(blockIdx.x);
  float mx = 0.f;
  if (w < A.nitems) load(w, mx);
  while (w < A.nitems) {
    // scale, convert and store this item's operand; the previous item's MMAs are done
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) fscr[warp] = mx;
    __syncthreads();
    float m2 = 0.f;
    for (int k = 0; k < 8; k++) m2 = fmaxf(m2, fscr[k]);
    const float s = pow2_scale(m2);
    // the input's maximum per RHS: the near-field kernel's scale for the same input
    if (threadIdx.x == 0 && m2 > 0.f && A.lvl < kInMaxSlot)
      atomicMax(&A.levmax[(w / A.tiles) * kMaxLevels + kInMaxSlot], __float_as_uint(m2));
#pragma unroll
    for (int r = 0; r < kPer; r++) {
      const int it = threadIdx.x + r * 256;
      __align__(16) __half h[8], l[8];
#pragma unroll
      for (int p = 0; p < 4; p++) {
        split_f16(v[r][p].x * s, h[2 * p], l[2 * p]);
        split_f16(v[r][p].y * s, h[2 * p + 1], l[2 * p + 1]);
      }
      const int off = it * 16;  // (it >> 7) * 2048 + ((it >> 3) & 15) * 128 + (it & 7) * 16
      *(uint4 *)(sm + P2mSmem::hi + off) = *(uint4 *)h;
      *(uint4 *)(sm + P2mSmem::lo + off) = *(uint4 *)l;
    }
    fence_proxy_async();
    __syncthreads();
    if (threadIdx.x == 0) {
      tc_fence_after();
      if (ok) {
        const uint64_t ah0 = smem_desc(sbase + P2mSmem::hi, 128, 2048);
        const uint64_t al0 = smem_desc(sbase + P2mSmem::lo, 128, 2048);
        const uint64_t bh0 = smem_desc(sbase + P2mSmem::b, 128, 512);
        const uint64_t bl0 = smem_desc(sbase + P2mSmem::b + A.stage_bytes / 2, 128, 512);
        for (int c = 0; c < 4; c++)
#pragma unroll
          for (int ks = 0; ks < 2; ks++) {
            const uint32_t aoff = (uint32_t)(c * 4 + ks * 2) * 128, boff = c * A.stage_bytes + ks * 256;
            mma_f16(tmem, desc_add(ah0, aoff), desc_add(bh0, boff), idesc, (c | ks) ? 1 : 0);
            mma_f16(tmem, desc_add(ah0, aoff), desc_add(bl0, boff), idesc, 1);
            mma_f16(tmem, desc_add(al0, aoff), desc_add(bh0, boff), idesc, 1);
          }
      }
      mma_commit(done);
    }
    // the next item's input, in flight while this one is multiplied and written
    const int rhs = w / A.tiles, leaf0 = (w % A.tiles) * 128;
    const int nxt = active_item(w + gridDim.x);
    float mxn = 0.f;
    if (nxt < A.nitems) load(nxt, mxn);
    ok = mbar_wait(done, parity, A.err, kErrP2m) && ok;
    parity ^= 1;
    tc_fence_after();
    const float inv = A.inv_c / s;
    const int m = 32 * q + lane;
    float omx = 0.f;
    for (int ch = c0; ch < c1; ch++) {
      float d[16];
      tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + 16 * ch, d);
#pragma unroll
      for (int p = 0; p < 8; p++) {
        const int k = 8 * ch + p;
        if (k < A.ns) {
          const float2 o = make_float2(d[2 * p] * inv, d[2 * p + 1] * inv);
          osm[m * (A.ns + 1) + k] = o;
          if (leaf0 + m < A.nleaves) omx = fmaxf(omx, fmaxf(fabsf(o.x), fabsf(o.y)));
        }
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) omx = fmaxf(omx, __shfl_xor_sync(0xffffffffu, omx, o));
    if (lane == 0 && ok) atomicMax(&A.levmax[rhs * kMaxLevels + A.lvl], __float_as_uint(omx));
    tc_fence_before();
    __syncthreads();
    if (ok) {
      const int nl = min(128, A.nleaves - leaf0);
      float2 *out = A.mul_leaf + (size_t)rhs * A.mp + (size_t)leaf0 * A.ns;
      for (int e = threadIdx.x; e < nl * A.ns; e += blockDim.x) {
        const int mm = e / A.ns, k = e - mm * A.ns;
        out[e] = osm[mm * (A.ns + 1) + k];
      }
    }
    __syncthreads();  // the output tile and fscr are reused by the next item
    w = nxt;
    mx = mxn;
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, 256);
}

// ---- P2M, pipelined: converter, MMA and epilogue roles over double-buffered
// A operands (128 leaves x 64 pixels x re, im, FP16 hi/lo) and TMEM
// accumulators; the coefficients (B, 4 stages) stay resident.  The converters
// load an item's pixels straight from global memory (every leaf is 512
// contiguous bytes), apply the input transform, take the item's maximum among
// themselves, and split.  The epilogue reads each leaf's ring from its TMEM
// lane and turns lanes into contiguous runs through a small per-warp tile;
// it keeps the level maximum for the M2M above. ----
struct P2mPipeSmem {
  __host__ __device__ static size_t a(int b) { return (size_t)b * 2 * kP2mA; }  // hi, then lo kP2mA on
  __host__ __device__ static size_t bst() { return 4 * (size_t)kP2mA; }
  // per epilogue warp: 32 leaves x 8 complex (+1 pad)
  __host__ __device__ static size_t epi(int stage_bytes) { return bst() + 4 * (size_t)stage_bytes; }
  __host__ __device__ static size_t bar(int stage_bytes) { return epi(stage_bytes) + 8 * 32 * 9 * 8; }
  __host__ __device__ static size_t total(int stage_bytes) { return bar(stage_bytes) + 256; }
};
// Roles: converters warps 0..7, MMA warp 8, epilogue warps 9..16 (two per
// TMEM lane quarter warp % 4, each taking every other 16-column chunk).
constexpr int kP2mConvWarps = 8, kP2mMmaWarp = 8, kP2mEpiWarp0 = 9, kP2mThreads = 17 * 32;
constexpr int kP2mConv = 32 * kP2mConvWarps, kP2mEpi = kP2mThreads - 32 * kP2mEpiWarp0;
constexpr int kP2mUnits = 128 * 16;                             // (leaf, 4-pixel chunk) per item
constexpr int kP2mPer = (kP2mUnits + kP2mConv - 1) / kP2mConv;  // units per converter thread

__global__ void __launch_bounds__(kP2mThreads, 1) k_tc_p2m_pipe(TcP2mArgs A) {
  extern __shared__ __align__(1024) char sm[];
  const PipeBars Bq(sm + P2mPipeSmem::bar(A.stage_bytes));
  float *fscr = (float *)(Bq.abar + 16);  // [kP2mConvWarps] converter maxima
  float *sval = fscr + 16;                // [2] the scale of the item in buffer b
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int i = 0; i < 11; i++) mbar_init(Bq.abar + i, 1);
    *Bq.abort = 0;
    fence_mbar_init();
  }
  if (warp == 0) tmem_alloc(Bq.tslot, 512);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *Bq.tslot;
  auto next_item = [&](int w) {
    do w += gridDim.x;
    while (w < A.nitems && A.active && !A.active[w / A.tiles]);
    return w;
  };
  const int first = (A.active && !A.active[blockIdx.x / A.tiles]) ? next_item(blockIdx.x) : blockIdx.x;
  // an item's pixels (its leaves are one contiguous run) into operand buffer b, as FP32
  auto stage = [&](int w, int b) {
    const int rhs = w / A.tiles, leaf0 = (w % A.tiles) * 128;
    const uint32_t bytes = (uint32_t)min(128, A.nleaves - leaf0) * kBB * 8;
    mbar_expect_tx(Bq.zfull + b, bytes);
    bulk_g2s(sm + P2mPipeSmem::a(b), A.x + (size_t)rhs * A.U + (size_t)leaf0 * kBB, bytes, Bq.zfull + b);
  };

  if (warp < kP2mConvWarps) {
    // ---- converters ----
    if (threadIdx.x == 0) {
      mbar_expect_tx(Bq.abar, 4 * A.stage_bytes);
      for (int c = 0; c < 4; c++)
        bulk_g2s(sm + P2mPipeSmem::bst() + c * A.stage_bytes, A.B + (size_t)c * A.stage_bytes, A.stage_bytes,
                 Bq.abar);
      if (first < A.nitems) {
        stage(first, 0);
        const int second = next_item(first);
        if (second < A.nitems) stage(second, 1);
      }
    }
    int w = first;
    for (int it = 0; w < A.nitems; it++) {
      const int b = it & 1, ph = (it >> 1) & 1;
      // the staged pixels, and the scale slot (free once the epilogue of item it - 2 is done)
      const bool fok = mbar_wait_or(Bq.zfull + b, ph, Bq.abort, A.err, kErrP2m) &&
                       mbar_wait_or(Bq.tfree + b, ph ^ 1, Bq.abort, A.err, kErrP2m);
      const int leaf0 = (w % A.tiles) * 128;
      const float4 *zst = (const float4 *)(sm + P2mPipeSmem::a(b));  // [leaf][32 float4]
      float2 v[kP2mPer][4];
      float mx = 0.f;
#pragma unroll
      for (int r = 0; r < kP2mPer; r++) {
        const int u = threadIdx.x + r * kP2mConv;
        const int m = ((u >> 7) << 3) | (u & 7), c = (u >> 3) & 15;
#pragma unroll
        for (int p = 0; p < 4; p++) v[r][p] = make_float2(0.f, 0.f);
        if (u < kP2mUnits && leaf0 + m < A.nleaves) {
          // odd leaves read their two halves in the other order: the 16-byte loads of a
          // warp then fall on 8 distinct bank groups
          const int odd = m & 1;
          const float4 x0 = zst[m * 32 + 2 * c + odd], x1 = zst[m * 32 + 2 * c + 1 - odd];
          const float4 a0 = odd ? x1 : x0, a1 = odd ? x0 : x1;
          const float2 g0 = make_float2(0.f, 0.f);
          v[r][0] = transform(make_float2(a0.x, a0.y), g0, A.mode);
          v[r][1] = transform(make_float2(a0.z, a0.w), g0, A.mode);
          v[r][2] = transform(make_float2(a1.x, a1.y), g0, A.mode);
          v[r][3] = transform(make_float2(a1.z, a1.w), g0, A.mode);
#pragma unroll
          for (int p = 0; p < 4; p++) mx = fmaxf(mx, cabs1(v[r][p]));
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      if (lane == 0) fscr[warp] = mx;
      named_sync(1, kP2mConv);  // every staged value is in registers: the buffer is rewritten in place
      float m2 = 0.f;
      for (int k = 0; k < kP2mConvWarps; k++) m2 = fmaxf(m2, fscr[k]);
      const float s = pow2_scale(m2);
      // the input's maximum per RHS: the near-field kernel's scale for the same input
      if (threadIdx.x == 0 && fok && m2 > 0.f && A.lvl < kInMaxSlot)
        atomicMax(&A.levmax[(w / A.tiles) * kMaxLevels + kInMaxSlot], __float_as_uint(m2));
      char *ahi = sm + P2mPipeSmem::a(b), *alo = ahi + kP2mA;
      if (fok) {
#pragma unroll
        for (int r = 0; r < kP2mPer; r++) {
          const int u = threadIdx.x + r * kP2mConv;
          if (u >= kP2mUnits) continue;
          uint32_t h[4], l[4];
#pragma unroll
          for (int p = 0; p < 4; p++) split2u(v[r][p].x * s, v[r][p].y * s, h[p], l[p]);
          st_shared_v4(ahi + u * 16, h);  // u * 16 = (m >> 3) * 2048 + c * 128 + (m & 7) * 16
          st_shared_v4(alo + u * 16, l);
        }
      }
      if (threadIdx.x == 0) sval[b] = s;
      fence_proxy_async();
      named_sync(1, kP2mConv);  // the operand is written; fscr may be reused
      if (threadIdx.x == 0) mbar_arrive(Bq.bfull + b);
      w = next_item(w);
    }
  } else if (warp == kP2mMmaWarp) {
    // ---- MMA issue: D[128 leaves][npad] = A[b] (hi/lo) x coefficients (hi/lo) ----
    const uint32_t idesc = idesc_f16_f32(128, A.npad), sbase = smem_u32(sm);
    const uint64_t bh0 = smem_desc(sbase + (uint32_t)P2mPipeSmem::bst(), 128, 512);
    const uint64_t bl0 = smem_desc(sbase + (uint32_t)P2mPipeSmem::bst() + A.stage_bytes / 2, 128, 512);
    const bool aok = mbar_wait_or(Bq.abar, 0, Bq.abort, A.err, kErrP2m);
    int w = first;
    for (int it = 0; w < A.nitems; it++) {
      const int b = it & 1, ph = (it >> 1) & 1;
      const bool ok = mbar_wait_or(Bq.bfull + b, ph, Bq.abort, A.err, kErrP2m) && aok;
      if (lane == 0) {
        tc_fence_after();
        if (ok) {
          const uint64_t ah0 = smem_desc(sbase + (uint32_t)P2mPipeSmem::a(b), 128, 2048);
          const uint64_t al0 = smem_desc(sbase + (uint32_t)P2mPipeSmem::a(b) + kP2mA, 128, 2048);
          const uint32_t d = tmem + (uint32_t)(b * 256);
          for (int c = 0; c < 4; c++)
#pragma unroll
            for (int ks = 0; ks < 2; ks++) {
              const uint32_t aoff = (uint32_t)(c * 4 + ks * 2) * 128, boff = c * A.stage_bytes + ks * 256;
              mma_f16(d, desc_add(ah0, aoff), desc_add(bh0, boff), idesc, (c | ks) ? 1 : 0);
              mma_f16(d, desc_add(ah0, aoff), desc_add(bl0, boff), idesc, 1);
              mma_f16(d, desc_add(al0, aoff), desc_add(bh0, boff), idesc, 1);
            }
        }
        mma_commit(Bq.tfull + b);
      }
      __syncwarp();
      w = next_item(w);
    }
  } else {
    // ---- epilogue: lane = leaf, columns 2k (re), 2k + 1 (im).  Each 16-column chunk
    // (8 samples of the warp's 32 consecutive leaves) goes through a padded
    // shared tile so that 8 lanes write one leaf's 64 contiguous bytes ----
    const int ew = warp - kP2mEpiWarp0, qd = warp & 3, eg = ew >> 2;  // lane quarter, chunk parity
    float2 *tile = (float2 *)(sm + P2mPipeSmem::epi(A.stage_bytes)) + ew * 32 * 9;
    int w = first, w2 = first < A.nitems ? next_item(next_item(first)) : A.nitems;
    for (int it = 0; w < A.nitems; it++) {
      const int b = it & 1, ph = (it >> 1) & 1;
      // tfull: the accumulator; bfull (already complete): the item's scale is visible
      const bool ok = mbar_wait_or(Bq.tfull + b, ph, Bq.abort, A.err, kErrP2m) &&
                      mbar_wait_or(Bq.bfull + b, ph, Bq.abort, A.err, kErrP2m);
      tc_fence_after();
      // the MMAs are done with operand buffer b: item it + 2's pixels go there now
      if (ew == 0 && lane == 0 && w2 < A.nitems) stage(w2, b);
      w2 = w2 < A.nitems ? next_item(w2) : A.nitems;
      const int rhs = w / A.tiles, leafw = (w % A.tiles) * 128 + 32 * qd;  // the warp's first leaf
      const float inv = A.inv_c / sval[b];
      float2 *outw = A.mul_leaf + (size_t)rhs * A.mp + (size_t)leafw * A.ns;
      float omx = 0.f;
      const uint32_t taddr = tmem + ((uint32_t)(32 * qd) << 16) + (uint32_t)(b * 256);
      for (int c0 = 16 * eg; c0 < A.npad; c0 += 32) {
        float d[16];
        tmem_ld16(taddr + c0, d);
        const int k0 = c0 / 2, nk = min(8, A.ns - k0);
#pragma unroll
        for (int j = 0; j < 8; j++)
          if (j < nk) tile[lane * 9 + j] = make_float2(d[2 * j] * inv, d[2 * j + 1] * inv);
        __syncwarp();
        if (ok) {
#pragma unroll
          for (int r = 0; r < 8; r++) {  // element r * 32 + lane: leaf e / 8, sample e % 8
            const int e = r * 32 + lane, lf = e >> 3, j = e & 7;
            if (j < nk && leafw + lf < A.nleaves) {
              const float2 o = tile[lf * 9 + j];
              outw[(size_t)lf * A.ns + k0 + j] = o;
              omx = fmaxf(omx, fmaxf(fabsf(o.x), fabsf(o.y)));
            }
          }
        }
        __syncwarp();
      }
      tc_fence_before();
      named_sync(2, kP2mEpi);  // the accumulator is read out
      if (ew == 0 && lane == 0) mbar_arrive(Bq.tfree + b);
      const unsigned mbits = __reduce_max_sync(0xffffffffu, __float_as_uint(omx));  // omx >= 0
      if (lane == 0 && ok && mbits) atomicMax(&A.levmax[rhs * kMaxLevels + A.lvl], mbits);
      w = next_item(w);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, 512);
}

// ---- host: operand construction ----

inline double pow2_scale_host(double maxabs) {
  if (!(maxabs > 0)) return 1.0;
  int e;
  std::frexp(maxabs, &e);
  return std::ldexp(1.0, 14 - e);
}

// Writes the [nrows x 32] K-major FP16 core-matrix block of reals(row, k0..k0+31)
// as hi then lo (each nrows/8 groups x 4 chunks x 8 rows x 8 halves).
template <class F>
void pack_stage(std::vector<uint8_t> &buf, size_t at, int nrows, int k0, double scale, F real_at) {
  const size_t half = (size_t)nrows * 32 * 2;
  __half *hi = (__half *)(buf.data() + at), *lo = (__half *)(buf.data() + at + half);
  for (int n = 0; n < nrows; n++)
    for (int k = 0; k < 32; k++) {
      const double v = real_at(n, k0 + k) * scale;
      const __half h = __double2half(v);
      const __half l = __double2half(v - (double)__half2float(h));
      const size_t idx = ((size_t)(n / 8) * 4 + k / 8) * 64 + (n % 8) * 8 + (k % 8);
      hi[idx] = h;
      lo[idx] = l;
    }
}

}  // namespace

struct TcPlan {
  uint8_t *nearB = nullptr;
  uint8_t *nearNp = nullptr;  // the same stages in the pipelined kernel's A-stage order
  int nl2p = 0;
  float inv_w = 1, inv_b = 1;
  float sw = 1, sb = 1;
  uint8_t *p2mB = nullptr;
  int npad = 0, p2m_stage = 0;
  float inv_c = 1;
  int *err = nullptr;
  bool ok = false;
  int near_pair = 0;  // tiles per near-field CTA picked by isg_autotune (0: built-in choice)
};

bool tc_available(const isg_ctx *c) { return c->tc && c->tc->ok; }
void tc_set_near_pair(isg_ctx *c, int pair) {
  if (tc_available(c)) c->tc->near_pair = pair;
}
int tc_near_pair(const isg_ctx *c) { return tc_available(c) ? c->tc->near_pair : 0; }

}  // namespace isg

int *isg_ctx::tc_err_flag() const { return tc ? tc->err : nullptr; }

namespace isg {

isg_status tc_setup(isg_ctx *c) {
  int dev = 0, major = 0, minor = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
  const HostTables &T = c->T;
  const int ns = T.nsamp[T.L - 1];
  c->tc = new TcPlan();
  TcPlan &P = *c->tc;
  if (major != 10 || ns > 4 * kLocChunksMax || T.nleaf < 1) return ISG_OK;  // engine unavailable, SIMT remains
  // near field: real embedding of near[slot][t][b]; row n = 2t + d, K = 2b + e
  auto wreal = [&](int s, int n, int k) {
    const cd w = T.near[((size_t)s * kBB + n / 2) * kBB + k / 2];
    const int d = n & 1, e = k & 1;
    return d == 0 ? (e == 0 ? w.real() : -w.imag()) : (e == 0 ? w.imag() : w.real());
  };
  auto breal = [&](int n, int k) {
    if (k / 2 >= ns) return 0.0;
    const cd w = T.basis[(size_t)(n / 2) * ns + k / 2];
    const int d = n & 1, e = k & 1;
    return d == 0 ? (e == 0 ? w.real() : -w.imag()) : (e == 0 ? w.imag() : w.real());
  };
  double mw = 0, mb = 0, mc = 0;
  for (const cd &v : T.near) mw = std::max(mw, std::max(std::abs(v.real()), std::abs(v.imag())));
  for (const cd &v : T.basis) mb = std::max(mb, std::max(std::abs(v.real()), std::abs(v.imag())));
  for (const cd &v : T.coeff) mc = std::max(mc, std::max(std::abs(v.real()), std::abs(v.imag())));
  const double sw = pow2_scale_host(mw), sb = pow2_scale_host(mb), sc = pow2_scale_host(mc);
  const int kl = ((2 * ns + 31) / 32) * 32;  // L2P K padded to whole stages
  P.nl2p = kl / 32;
  std::vector<uint8_t> nb((size_t)(kNearStages + P.nl2p) * kStageBytes, 0);
  for (int t = 0; t < kNearStages; t++)
    pack_stage(nb, (size_t)t * kStageBytes, 128, (t & 3) * 32, sw, [&](int n, int k) { return wreal(t >> 2, n, k); });
  for (int c2 = 0; c2 < P.nl2p; c2++)
    pack_stage(nb, (size_t)(kNearStages + c2) * kStageBytes, 128, c2 * 32, sb, breal);
  P.inv_w = (float)(1.0 / sw);
  P.inv_b = (float)(1.0 / sb);
  P.sw = (float)sw;
  P.sb = (float)sb;
  // pipelined kernel: per A-stage, a halo K-group's nine slots or one L2P stage
  std::vector<uint8_t> np((size_t)(kNearStages + P.nl2p) * kStageBytes, 0);
  {
    size_t t = 0;
    for (int a = 0; a < 4 + P.nl2p; a++) {
      int idx;
      if (np_stage(a, P.nl2p, idx) == 0) {
        for (int q = 0; q < 9; q++, t++)
          pack_stage(np, t * kStageBytes, 128, idx * 32, sw, [&](int n, int k) { return wreal(q, n, k); });
      } else {
        pack_stage(np, (t++) * kStageBytes, 128, idx * 32, sb, breal);
      }
    }
  }
  // P2M: row n = 2k + d over samples (padded to a multiple of 16), K = 2 pixel + e
  P.npad = ((2 * ns + 15) / 16) * 16;
  P.p2m_stage = P.npad * 32 * 2 * 2;
  auto creal = [&](int n, int k) {
    if (n / 2 >= ns) return 0.0;
    const cd w = T.coeff[(size_t)(n / 2) * kBB + k / 2];
    const int d = n & 1, e = k & 1;
    return d == 0 ? (e == 0 ? w.real() : -w.imag()) : (e == 0 ? w.imag() : w.real());
  };
  std::vector<uint8_t> pb((size_t)4 * P.p2m_stage, 0);
  for (int c2 = 0; c2 < 4; c2++) pack_stage(pb, (size_t)c2 * P.p2m_stage, P.npad, c2 * 32, sc, creal);
  P.inv_c = (float)(1.0 / sc);
  isg_status e;
  if ((e = cuda_check(c, cudaMalloc(&P.nearB, nb.size()), "tc alloc")) != ISG_OK) return e;
  if ((e = cuda_check(c, cudaMalloc(&P.nearNp, np.size()), "tc alloc")) != ISG_OK) return e;
  if ((e = cuda_check(c, cudaMalloc(&P.p2mB, pb.size()), "tc alloc")) != ISG_OK) return e;
  if ((e = cuda_check(c, cudaMalloc(&P.err, sizeof(int)), "tc alloc")) != ISG_OK) return e;
  cudaMemcpy(P.nearB, nb.data(), nb.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(P.nearNp, np.data(), np.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(P.p2mB, pb.data(), pb.size(), cudaMemcpyHostToDevice);
  cudaMemset(P.err, 0, sizeof(int));
  cudaFuncSetAttribute(k_tc_near, cudaFuncAttributeMaxDynamicSharedMemorySize, NearSmem::total);
  cudaFuncSetAttribute(k_tc_near_pipe, cudaFuncAttributeMaxDynamicSharedMemorySize, NpSmem::total);
  cudaFuncSetAttribute(k_tc_p2m, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)P2mSmem::total(P.p2m_stage, ns));
  cudaFuncSetAttribute(k_tc_p2m_pipe, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)P2mPipeSmem::total(P.p2m_stage));
  if ((e = cuda_check(c, cudaGetLastError(), "tc setup")) != ISG_OK) return e;
  P.ok = true;
  return ISG_OK;
}

void tc_destroy(isg_ctx *c) {
  if (!c->tc) return;
  cudaFree(c->tc->nearB);
  cudaFree(c->tc->nearNp);
  cudaFree(c->tc->p2mB);
  cudaFree(c->tc->err);
  delete c->tc;
  c->tc = nullptr;
}

int tc_near_blocks(const isg_ctx *c) {
  const int tx = (c->P.nleaf + kTX - 1) / kTX, ty = (c->P.nleaf + kTY - 1) / kTY;
  return tx * ty;
}

int tc_error(isg_ctx *c) {
  if (!tc_available(c)) return 0;
  int h = 0;
  cudaMemcpy(&h, c->tc->err, sizeof(int), cudaMemcpyDeviceToHost);
  return h;
}

static bool aligned16(const void *p) { return ((uintptr_t)p & 15) == 0; }

// cuTensorMapEncodeTiled through the runtime's driver entry-point query, so
// that the library does not link the driver library (it still loads where
// there is no driver, for the checks that need none); null when unavailable.
// The lookup runs once per process; C++11 makes the static's initialisation
// thread-safe, so contexts on several host threads may race to it.
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = []() -> PFN_cuTensorMapEncodeTiled_v12000 {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      return (PFN_cuTensorMapEncodeTiled_v12000)p;
    return nullptr;
  }();
  return fn;
}

// The pipelined near-field kernel; returns false (launching nothing) when the
// call does not meet its conditions: P2M's input maximum known (N.inmax), leaf
// rings of a multiple of 4 samples (<= 80), 16-byte aligned vectors and both
// tensor maps encoded.
static bool tc_near_pipe(isg_ctx *c, const NearArgs &N, cudaStream_t st, isg_status *e) {
  const DevPlan &P = c->P;
  const TcPlan &T = *c->tc;
  const float2 *loc_leaf = N.loc + P.lv[P.L - 1].off;
  if (!N.inmax || !N.locmax || !T.nearNp || P.ns_leaf % 4 || P.ns_leaf > 4 * kLocChunksMax || P.mp % 2 ||
      !aligned16(loc_leaf) || P.L - 1 >= kInMaxSlot)
    return false;
  const PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
  if (!encode) return false;
  TcNearPipeArgs A;
  A.x = N.in.x;
  A.xe = N.x_epi ? N.x_epi : N.in.x;
  A.g = N.in.g;
  A.gstride = N.in.gstride;
  A.mode = N.in.mode;
  A.active = N.in.active;
  A.B = T.nearNp;
  A.nl2p = T.nl2p;
  A.sw = T.sw;
  A.sb = T.sb;
  A.levmax = N.inmax;
  A.locmax = N.locmax;
  A.lvl_leaf = P.L - 1;
  A.y = N.y;
  A.epi = N.epi;
  A.red = N.red;
  A.dot_a = N.dot_a;
  A.part = N.part;
  A.nleaf = P.nleaf;
  A.U = P.U;
  A.tiles_x = (P.nleaf + kTX - 1) / kTX;
  A.tiles_y = (P.nleaf + kTY - 1) / kTY;
  A.tiles = A.tiles_x * A.tiles_y;
  A.ppr = A.tiles_x * ((A.tiles_y + kPair - 1) / kPair);
  A.nitems = A.ppr * N.in.nrhs;
  A.err = T.err;
  // tmh: the input as [RHS][leaf row][leaf column][128 reals], a box is one halo
  // K-group (32 reals) of the pair's 34 x 10 halo; tml: the leaf locals as
  // [RHS][leaf row][leaf column][2 ns reals], a box is one L2P stage of the pair
  CUtensorMap tmh, tml;
  memset(&tmh, 0, sizeof(tmh));
  memset(&tml, 0, sizeof(tml));
  const cuuint32_t one[4] = {1, 1, 1, 1};
  const cuuint64_t hd[4] = {2 * kBB, (cuuint64_t)P.nleaf, (cuuint64_t)P.nleaf, (cuuint64_t)N.in.nrhs};
  const cuuint64_t hs[3] = {(cuuint64_t)kBB * 8, (cuuint64_t)P.nleaf * kBB * 8, (cuuint64_t)P.U * 8};
  const cuuint32_t hb[4] = {32, (cuuint32_t)kHC, (cuuint32_t)kHR, 1};
  const cuuint64_t ld[4] = {(cuuint64_t)(2 * P.ns_leaf), (cuuint64_t)P.nleaf, (cuuint64_t)P.nleaf,
                            (cuuint64_t)N.in.nrhs};
  const cuuint64_t ls[3] = {(cuuint64_t)P.ns_leaf * 8, (cuuint64_t)P.nleaf * P.ns_leaf * 8, (cuuint64_t)P.mp * 8};
  const cuuint32_t lb[4] = {32, (cuuint32_t)kTX, (cuuint32_t)(kPair * kTY), 1};
  if (encode(&tmh, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, (void *)A.x, hd, hs, hb, one, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS ||
      encode(&tml, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, (void *)loc_leaf, ld, ls, lb, one,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->opts.device);
  count_launch();
  k_tc_near_pipe<<<std::min(A.nitems, sms), kNpThreads, NpSmem::total, st>>>(A, tmh, tml);
  *e = cuda_check(c, cudaGetLastError(), "tc near launch");
  return true;
}

isg_status tc_near(isg_ctx *c, const NearArgs &N, cudaStream_t st) {
  const DevPlan &P = c->P;
  const TcPlan &T = *c->tc;
  if (!aligned16(N.in.x) || (N.x_epi && !aligned16(N.x_epi)) || (N.in.g && !aligned16(N.in.g)) || !aligned16(N.y) ||
      (N.dot_a && !aligned16(N.dot_a)) ||
      (N.in.gstride % 2) || N.epi == EPI_L2P_ONLY)
    return ISG_UNSUPPORTED;
  isg_status pe = ISG_OK;
  if (tc_near_pipe(c, N, st, &pe)) return pe;
  TcNearArgs A;
  A.x = N.in.x;
  A.xe = N.x_epi ? N.x_epi : N.in.x;
  A.g = N.in.g;
  A.gstride = N.in.gstride;
  A.mode = N.in.mode;
  A.active = N.in.active;
  A.loc_leaf = N.loc + P.lv[P.L - 1].off;
  A.mp = P.mp;
  A.ns = P.ns_leaf;
  A.B = T.nearB;
  A.nl2p = T.nl2p;
  A.inv_w = T.inv_w;
  A.inv_b = T.inv_b;
  A.y = N.y;
  A.epi = N.epi;
  A.red = N.red;
  A.dot_a = N.dot_a;
  A.part = N.part;
  A.nleaf = P.nleaf;
  A.U = P.U;
  A.tiles_x = (P.nleaf + kTX - 1) / kTX;
  const int tiles_y = (P.nleaf + kTY - 1) / kTY;
  A.tiles = A.tiles_x * tiles_y;
  A.loc_vec = (P.ns_leaf % 4 == 0) && aligned16(A.loc_leaf) && (P.mp % 2 == 0);
  A.err = T.err;
  A.locmax = N.locmax;
  A.lvl_leaf = P.L - 1;
  count_launch();
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->opts.device);
  A.pair = (A.tiles * N.in.nrhs >= 2 * kPair * sms) ? kPair : 1;
  if (T.near_pair > 0 && 4 * N.in.nrhs >= P.tuned_nrhs) A.pair = std::min(T.near_pair, kPair);
  const int pairs = A.tiles_x * ((tiles_y + A.pair - 1) / A.pair);
  // tensor maps (see k_tc_near); a map that does not encode keeps its 16-byte copies
  CUtensorMap tmx, tml;
  memset(&tmx, 0, sizeof(tmx));
  memset(&tml, 0, sizeof(tml));
  const cuuint32_t one[5] = {1, 1, 1, 1, 1};
  const PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
  A.tma_x = 0;
  if (encode) {
    const cuuint64_t dims[5] = {8, (cuuint64_t)P.nleaf, 16, (cuuint64_t)P.nleaf, (cuuint64_t)N.in.nrhs};
    const cuuint64_t strides[4] = {(cuuint64_t)kBB * 8, 32, (cuuint64_t)P.nleaf * kBB * 8, (cuuint64_t)P.U * 8};
    const cuuint32_t box[5] = {4, (cuuint32_t)kHC, 16, (cuuint32_t)(A.pair * kTY + 2), 1};
    A.tma_x = encode(&tmx, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5, (void *)A.x, dims, strides, box, one,
                                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                     CU_TENSOR_MAP_L2_PROMOTION_NONE,
                                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
  }
  A.tma_loc = 0;
  if (A.loc_vec && encode) {
    const cuuint64_t dims[5] = {8, (cuuint64_t)P.nleaf, (cuuint64_t)(P.ns_leaf / 4), (cuuint64_t)P.nleaf,
                                (cuuint64_t)N.in.nrhs};
    const cuuint64_t strides[4] = {(cuuint64_t)P.ns_leaf * 8, 32, (cuuint64_t)P.nleaf * P.ns_leaf * 8,
                                   (cuuint64_t)P.mp * 8};
    const cuuint32_t box[5] = {4, (cuuint32_t)kTX, (cuuint32_t)kLocChunksMax, (cuuint32_t)kTY, 1};
    A.tma_loc = P.ns_leaf / 4 <= kLocChunksMax &&
                encode(&tml, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5, (void *)A.loc_leaf, dims, strides,
                                       box, one, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                       CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
  }
  k_tc_near<<<dim3(pairs, N.in.nrhs), 256, NearSmem::total, st>>>(A, tmx, tml);
  return cuda_check(c, cudaGetLastError(), "tc near launch");
}

isg_status tc_p2m(isg_ctx *c, const BatchArgs &B, float2 *mul, cudaStream_t st) {
  const DevPlan &P = c->P;
  const TcPlan &T = *c->tc;
  if (!aligned16(B.x) || (B.g && !aligned16(B.g)) || (B.gstride % 2)) return ISG_UNSUPPORTED;
  TcP2mArgs A;
  A.x = B.x;
  A.g = B.g;
  A.gstride = B.gstride;
  A.mode = B.mode;
  A.active = B.active;
  A.B = T.p2mB;
  A.npad = T.npad;
  A.stage_bytes = T.p2m_stage;
  A.inv_c = T.inv_c;
  A.mul_leaf = mul + P.lv[P.L - 1].off;
  A.mp = P.mp;
  A.ns = P.ns_leaf;
  A.nleaves = P.nleaf * P.nleaf;
  A.U = P.U;
  A.tiles = (A.nleaves + 127) / 128;
  A.nitems = A.tiles * B.nrhs;
  A.err = T.err;
  A.levmax = c->levmax;
  A.lvl = P.L - 1;
  count_launch();
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->opts.device);
  if (B.mode == IN_G)  // the pipelined kernel stages x alone
    k_tc_p2m<<<std::min(A.nitems, sms), 256, P2mSmem::total(T.p2m_stage, A.ns), st>>>(A);
  else
    k_tc_p2m_pipe<<<std::min(A.nitems, sms), kP2mThreads, P2mPipeSmem::total(T.p2m_stage), st>>>(A);
  return cuda_check(c, cudaGetLastError(), "tc p2m launch");
}

}  // namespace isg
