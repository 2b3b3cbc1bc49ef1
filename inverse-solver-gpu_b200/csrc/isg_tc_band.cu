// M2M on the tensor cores as a banded GEMM over every ring of a level.
//
// Interpolation (M2M, kernels.cu:83-136, solve.cpp:93-112) applies one real
// banded matrix per level to complex rings: D[sample][ring] = sum_j W[sample][j]
// ring[j].
// Output samples are tiled by 128 (the MMA M); for each tile the weights are
// restricted to the circular window of input samples its rows touch (a few
// dozen more than 128 x the rate ratio), precomputed on the host as FP16 hi/lo
// K-chunks of 64 in the core-matrix layout and brought in by bulk copies.  The
// CTA's 128 MMA columns are 16 parents x 4 children x (re, im) of one level of
// one or more RHS (64 KB of shared memory and 128 TMEM columns, so three CTAs
// share an SM: each CTA's load, MMA and epilogue phases run one after another,
// and the SM overlaps them across CTAs); ring values are split into FP16
// hi/lo after a power-of-two scale per CTA (3 products, FP32 accumulation in
// TMEM).  The child shift
// phases are folded into the epilogue (sum over the four children), exactly as
// in the reference.
//
// L2L (kernels.cu:138-190, solve.cpp:150-168) on the tensor cores, for the
// levels whose rings have at most 128 samples (the leaves and their parents,
// most of the tree's samples): persistent CTAs keep the level's whole
// anterpolation matrix (128 child samples x the parent ring, FP16 hi/lo) in
// shared memory and walk items of 32 (or 16) parents.  An item's parent rings
// arrive by cp.async while the previous item is multiplied and written; each
// CTA forms the four shifted copies shl[q][j] z[j] of every ring directly in
// the FP16 hi/lo operand layout (256 MMA columns = 32 parents x 4 children x
// re, im), and the epilogue writes each child ring from TMEM with the child
// sample on the lane, so every store is coalesced.  Coarser levels keep the
// SIMT tiled kernel.
#include <algorithm>
#include <cmath>
#include <vector>

#include "isg_context.hpp"
#include "isg_tc.cuh"

namespace isg {

namespace {

using namespace tc;

constexpr int kCols = 128;        // MMA N: 16 parents x 4 children x (re, im)
constexpr int kParents = 16;
constexpr int kKC = 64;           // K chunk
constexpr int kAHalf = 128 * kKC * 2;    // 16 KB: one FP16 split of an A chunk
constexpr int kBHalf = kCols * kKC * 2;  // 16 KB
constexpr int kSmem = 2 * kAHalf + 2 * kBHalf + 256 + 4 * kParents;  // + barriers, TMEM slot, scratch, per-parent maxima and flags
constexpr int kErrBand = 121;

struct BandArgs {
  const float2 *src;  // child-level multipoles (level base)
  float2 *dst;        // parent-level multipoles (level base)
  size_t mp;
  int n_p, ns_in, ns_out;
  const float2 *shift;  // shiftmul of the parent level, [4][ns_p]
  const uint8_t *A;     // K-chunks of this transition (hi then lo, 32 KB each)
  const int *kw0, *nchunk, *chunk0;  // per M-tile: window start (-1: whole ring), chunks, first chunk
  float inv_a;
  int nparents, ncols;  // ncols = parents x RHS
  const int *active;
  int *err;
  unsigned *levmax;        // [R][kMaxLevels] max |re|, |im| per RHS and level (FP32 bits)
  int lvl_in, lvl_out;
};

// One ring of the CTA: its base pointer, or none.
struct RingRef {
  const float2 *p;
};

__device__ __forceinline__ RingRef ring_ref(const BandArgs &A, int ring) {
  const int pl = ring >> 2, q = ring & 3, gp = blockIdx.x * kParents + pl;
  RingRef r{nullptr};
  if (gp >= A.ncols) return r;
  const int rhs = gp / A.nparents, P = gp % A.nparents;
  if (A.active && !A.active[rhs]) return r;
  const float2 *base = A.src + (size_t)rhs * A.mp;
  const int py = P / A.n_p, px = P % A.n_p, nc = 2 * A.n_p;
  r.p = base + (size_t)((2 * py + (q >> 1)) * nc + 2 * px + (q & 1)) * A.ns_in;
  return r;
}

// Eight consecutive window samples kk0 .. kk0+7 of a ring (zero outside).
__device__ __forceinline__ void ring_load8(const BandArgs &A, const RingRef &r, int kk0, int kw0, float2 *v) {
  int j0;
  if (kw0 < 0) {
    j0 = kk0;
  } else {
    j0 = (kw0 + kk0) % A.ns_in;  // the window may be longer than the ring; weights past it are zero
  }
  if (r.p && !(j0 & 1) && j0 + 8 <= A.ns_in) {  // eight samples inside the ring, 16-byte aligned
    const float4 *q4 = (const float4 *)(r.p + j0);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const float4 t = q4[k];
      v[2 * k] = make_float2(t.x, t.y);
      v[2 * k + 1] = make_float2(t.z, t.w);
    }
    return;
  }
#pragma unroll
  for (int k = 0; k < 8; k++) {
    int j = j0 + k;
    bool ok = r.p != nullptr;
    if (kw0 < 0) {
      ok = ok && j < A.ns_in;
    } else if (j >= A.ns_in) {
      j -= A.ns_in;
    }
    float2 x = make_float2(0.f, 0.f);
    if (ok) x = r.p[j];
    v[k] = x;
  }
}

__global__ void __launch_bounds__(256, 3) k_tc_band(BandArgs A) {
  extern __shared__ __align__(1024) char sm[];
  char *ahi = sm, *bhi = sm + 2 * kAHalf, *blo = bhi + kBHalf;
  uint64_t *abar = (uint64_t *)(blo + kBHalf);
  uint64_t *mbar = abar + 1;
  uint32_t *tslot = (uint32_t *)(abar + 2);
  float *fscr = (float *)(abar + 3);  // [8]
  unsigned *pmax = (unsigned *)(abar + 16);  // [kParents] output maxima (FP32 bits)
  if (threadIdx.x < kParents) pmax[threadIdx.x] = 0u;
  int *pvalid = (int *)(pmax + kParents);  // [kParents] the parent exists and its RHS is active
  if (threadIdx.x < kParents) {
    const int gp = blockIdx.x * kParents + threadIdx.x;
    pvalid[threadIdx.x] = gp < A.ncols && !(A.active && !A.active[gp / A.nparents]);
  }
  // no parent of this CTA exists with an active RHS (converged RHS at the end
  // of a batch): nothing to load, multiply or write
  if (!__syncthreads_or(threadIdx.x < kParents && pvalid[threadIdx.x])) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int mt = blockIdx.y, m0 = mt * 128;
  const int kw0 = A.kw0[mt], nch = A.nchunk[mt];
  const uint8_t *Achunks = A.A + (size_t)A.chunk0[mt] * 2 * kAHalf;

  // power-of-two scale from the input level's maximum over the CTA's RHS
  // (written by the kernel that produced that level)
  float mx = 0.f;
  if (threadIdx.x == 0) {
    const int g0 = blockIdx.x * kParents, g1 = min(A.ncols, g0 + kParents) - 1;
    for (int r = g0 / A.nparents; r <= g1 / A.nparents; r++)
      mx = fmaxf(mx, __uint_as_float(A.levmax[r * kMaxLevels + A.lvl_in]));
  }
  if (lane == 0) fscr[warp] = mx;
  if (threadIdx.x == 0) {
    mbar_init(abar, 1);
    mbar_init(mbar, 1);
    fence_mbar_init();
  }
  if (warp == 0) tmem_alloc(tslot, kCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  float m2 = 0.f;
  for (int w = 0; w < 8; w++) m2 = fmaxf(m2, fscr[w]);
  const float s = pow2_scale(m2);
  const uint32_t idesc = idesc_f16_f32(128, kCols);
  const uint32_t sbase = smem_u32(sm);
  bool ok = true;

  for (int ch = 0; ch < nch; ch++) {
    if (threadIdx.x == 0) {
      mbar_expect_tx(abar, 2 * kAHalf);
      bulk_g2s(ahi, Achunks + (size_t)ch * 2 * kAHalf, 2 * kAHalf, abar);
    }
    // B chunk: ring r gives rows 2r (re) and 2r + 1 (im); item = (ring, 8-sample group)
#pragma unroll 2
    for (int it = threadIdx.x; it < 4 * kParents * (kKC / 8); it += blockDim.x) {
      const int r = it >> 3, g8 = it & 7;
      __align__(16) __half hr[8], lr[8], hi8[8], li8[8];
      float2 v[8];
      ring_load8(A, ring_ref(A, r), ch * kKC + g8 * 8, kw0, v);
#pragma unroll
      for (int k = 0; k < 8; k++) {
        split_f16(v[k].x * s, hr[k], lr[k]);
        split_f16(v[k].y * s, hi8[k], li8[k]);
      }
      const int n0 = 2 * r, n1 = 2 * r + 1;
      const int o0 = ((n0 >> 3) * (kKC / 8) + g8) * 128 + (n0 & 7) * 16;
      const int o1 = ((n1 >> 3) * (kKC / 8) + g8) * 128 + (n1 & 7) * 16;
      *(uint4 *)(bhi + o0) = *(uint4 *)hr;
      *(uint4 *)(blo + o0) = *(uint4 *)lr;
      *(uint4 *)(bhi + o1) = *(uint4 *)hi8;
      *(uint4 *)(blo + o1) = *(uint4 *)li8;
    }
    fence_proxy_async();
    __syncthreads();
    if (threadIdx.x == 0) {
      tc_fence_after();
      if (mbar_wait(abar, ch & 1, A.err, kErrBand)) {
        const uint64_t ah = smem_desc(sbase, 128, (kKC / 8) * 128);
        const uint64_t al = smem_desc(sbase + kAHalf, 128, (kKC / 8) * 128);
        const uint64_t bh = smem_desc(sbase + 2 * kAHalf, 128, (kKC / 8) * 128);
        const uint64_t bl = smem_desc(sbase + 2 * kAHalf + kBHalf, 128, (kKC / 8) * 128);
#pragma unroll
        for (int ks = 0; ks < kKC / 16; ks++) {
          const uint32_t k = ks * 256;
          mma_f16(tmem, desc_add(ah, k), desc_add(bh, k), idesc, (ch | ks) ? 1 : 0);
          mma_f16(tmem, desc_add(ah, k), desc_add(bl, k), idesc, 1);
          mma_f16(tmem, desc_add(al, k), desc_add(bh, k), idesc, 1);
        }
      }
      mma_commit(mbar);
    }
    ok = mbar_wait(mbar, ch & 1, A.err, kErrBand) && ok;
    __syncthreads();
  }

  // ---- epilogue ----
  tc_fence_after();
  const float inv = A.inv_a / s;
  const int qd = warp & 3, h = warp >> 2;
  const int km = m0 + 32 * qd + lane;
  const bool row_ok = ok && km < A.ns_out;
  float2 sh[4];  // the row's four child shift phases, the same for every parent
#pragma unroll
  for (int q = 0; q < 4; q++) sh[q] = row_ok ? __ldg(&A.shift[q * A.ns_out + km]) : make_float2(0.f, 0.f);
  for (int pp = 0; pp < kCols / 32; pp++) {
    float d[16];
    tmem_ld16(tmem + ((uint32_t)(32 * qd) << 16) + (kCols / 2) * h + 16 * pp, d);
#pragma unroll
    for (int u = 0; u < 2; u++) {
      // the parent is the same for every lane of the warp
      const int pl = (kParents / 2) * h + 2 * pp + u, gp = blockIdx.x * kParents + pl;
      if (!pvalid[pl]) continue;
      const int rhs = gp / A.nparents, P = gp % A.nparents;
      unsigned mbits = 0u;
      if (row_ok) {
        float2 *base = A.dst + (size_t)rhs * A.mp;
        const float *dv = d + 8 * u;
        float2 acc = make_float2(0.f, 0.f);
#pragma unroll
        for (int q = 0; q < 4; q++) cfma(acc, sh[q], make_float2(dv[2 * q] * inv, dv[2 * q + 1] * inv));
        base[(size_t)P * A.ns_out + km] = acc;
        mbits = __float_as_uint(fmaxf(fabsf(acc.x), fabsf(acc.y)));
      }
      mbits = __reduce_max_sync(0xffffffffu, mbits);
      if (lane == 0 && mbits) atomicMax(&pmax[pl], mbits);
    }
  }
  tc_fence_before();
  __syncthreads();
  // the parent level's maximum per RHS, read by the next coarser M2M
  if (threadIdx.x < kParents) {
    const int gp = blockIdx.x * kParents + threadIdx.x;
    if (gp < A.ncols && pmax[threadIdx.x])
      atomicMax(&A.levmax[(gp / A.nparents) * kMaxLevels + A.lvl_out], pmax[threadIdx.x]);
  }
  if (warp == 0) tmem_dealloc(tmem, kCols);
}

// ---- L2L ----
constexpr int kErrL2l = 122;

struct L2lArgs {
  float2 *loc;  // every level's locals; parent rings at off_in, child rings at off_out
  size_t mp, off_in, off_out;
  int lg_np, ns_in, ns_out, Kp, ppi;  // log2 parents per side, padded K, parents per item
  unsigned kc_magic;                  // ceil(2^32 / (Kp / 8)): division by Kp / 8 as a high multiply
  const uint8_t *A;                   // [128 x Kp] FP16 hi then lo, K-major core matrices
  const float2 *shl;                  // [ns_in][4] local shifts of the parent level
  float inv_a, shl_max;
  int nparents, items_per_rhs, nitems;
  const int *active;
  int *err;
  const unsigned *locmax;  // [R][kMaxLevels] max |re|, |im| of the locals per level (written by M2L)
  int lvl_in;
};

using L2lRoles = PipeRoles<8, 8>;
using M2mRoles = PipeRoles<11, 4>;

// L2L layout: A hi/lo; B[2] hi/lo; the shifts [4][Kp + 2] (child-major,
// padded against bank conflicts); two staging buffers, each the item's ppi
// consecutive parent rings (one contiguous run) and Kp zero samples; barriers.
struct L2lSmem {
  size_t a, b, bbuf, sh, z, zbuf, bar, total;
  __host__ __device__ L2lSmem(int Kp, int ppi, int ns) {
    a = 0;
    b = a + (size_t)512 * Kp;
    bbuf = (size_t)32 * ppi * Kp;
    sh = b + 2 * bbuf;
    z = sh + (((size_t)32 * (Kp + 2) + 127) & ~(size_t)127);
    zbuf = ((size_t)(ppi * ns + Kp) * 8 + 127) & ~(size_t)127;
    bar = z + 2 * zbuf;
    total = bar + 256;
  }
};

template <class R>
__global__ void __launch_bounds__(R::threads, 1) k_tc_l2l(L2lArgs A) {
  extern __shared__ __align__(1024) char sm[];
  const L2lSmem L(A.Kp, A.ppi, A.ns_in);
  const int N = 8 * A.ppi, Kp = A.Kp, kc = Kp / 8, zs = A.ns_in;
  const PipeBars Bq(sm + L.bar);
  float2 *shs = (float2 *)(sm + L.sh);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  auto bbuf = [&](int b) { return sm + L.b + b * L.bbuf; };  // hi, then lo N * Kp * 2 bytes on
  auto zbuf = [&](int b) { return (float2 *)(sm + L.z + b * L.zbuf); };
  if (threadIdx.x == 0) {
    for (int i = 0; i < 11; i++) mbar_init(Bq.abar + i, 1);
    *Bq.abort = 0;
    fence_mbar_init();
  }
  if (warp == 0) tmem_alloc(Bq.tslot, 2 * N);
  for (int e = threadIdx.x; e < 4 * (Kp + 2); e += blockDim.x) {
    const int q = e / (Kp + 2), j = e - q * (Kp + 2);
    shs[e] = j < A.ns_in ? __ldg(A.shl + 4 * j + q) : make_float2(0.f, 0.f);
  }
  // zero both staging buffers: the tail past the last ring is read (against zero weights)
  for (int e = threadIdx.x; e < (int)(2 * L.zbuf / 4); e += blockDim.x) ((float *)zbuf(0))[e] = 0.f;
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *Bq.tslot;
  auto next_item = [&](int w) {
    do w += gridDim.x;
    while (w < A.nitems && A.active && !A.active[w / A.items_per_rhs]);
    return w;
  };
  const int first = (A.active && !A.active[blockIdx.x / A.items_per_rhs]) ? next_item(blockIdx.x) : blockIdx.x;
  auto scale_of = [&](int w) {
    return pow2_scale(1.5f * A.shl_max * __uint_as_float(A.locmax[(w / A.items_per_rhs) * kMaxLevels + A.lvl_in]));
  };
  // an item's ppi consecutive parent rings: one bulk copy
  const uint32_t run = (uint32_t)A.ppi * A.ns_in * 8;
  auto stage = [&](int w, int b) {
    if (lane != 0) return;
    const int rhs = w / A.items_per_rhs, p0 = (w % A.items_per_rhs) * A.ppi;
    mbar_expect_tx(Bq.zfull + b, run);
    bulk_g2s(zbuf(b), A.loc + (size_t)rhs * A.mp + A.off_in + (size_t)p0 * A.ns_in, run, Bq.zfull + b);
  };
  const int ngroups = A.ppi * kc;

  if (warp < R::conv_warps) {
    // ---- converters: B[b] rows 8 parent + 2 q + (re, im) = shl[q][j] z[j] s ----
    if (warp == 0) {
      if (lane == 0) {
        mbar_expect_tx(Bq.abar, 512 * Kp);
        bulk_g2s(sm + L.a, A.A, 512 * Kp, Bq.abar);
      }
      if (first < A.nitems) stage(first, 0);
      const int second = first < A.nitems ? next_item(first) : A.nitems;
      if (second < A.nitems) stage(second, 1);
    }
    int w = first, w2 = first < A.nitems ? next_item(next_item(first)) : A.nitems;
    for (int it = 0; w < A.nitems; it++) {
      const int b = it & 1, ph = (it >> 1) & 1;
      const bool zok = mbar_wait_or(Bq.zfull + b, ph, Bq.abort, A.err, kErrL2l);
      const bool bok = mbar_wait_or(Bq.bfree + b, ph ^ 1, Bq.abort, A.err, kErrL2l);
      const float s = scale_of(w);
      const float2 *zst = zbuf(b);
      char *bhi = bbuf(b), *blo = bhi + (size_t)N * Kp * 2;
      if (zok && bok) {
        // a unit is one child q of one core-matrix group (8 samples of one parent):
        // both rows, hi and lo
#pragma unroll 2
        for (int u = threadIdx.x; u < 4 * ngroups; u += R::conv) {
          const int q = u & 3, cm = u >> 2;
          const int pl = (int)__umulhi((unsigned)cm, A.kc_magic), j0 = 8 * (cm - pl * kc);
          const float4 *zp = (const float4 *)(zst + pl * zs + j0);
          const float4 *sp = (const float4 *)(shs + q * (Kp + 2) + j0);
          uint32_t hr[4], lr[4], hm[4], lm[4];
#pragma unroll
          for (int i = 0; i < 4; i++) {
            const float4 z = zp[i], sh = sp[i];
            const float re0 = fmaf(sh.x, z.x, -sh.y * z.y) * s, im0 = fmaf(sh.x, z.y, sh.y * z.x) * s;
            const float re1 = fmaf(sh.z, z.z, -sh.w * z.w) * s, im1 = fmaf(sh.z, z.w, sh.w * z.z) * s;
            split2u(re0, re1, hr[i], lr[i]);
            split2u(im0, im1, hm[i], lm[i]);
          }
          const uint32_t o = (uint32_t)cm * 128 + q * 32;
          st_shared_v4(bhi + o, hr);
          st_shared_v4(bhi + o + 16, hm);
          st_shared_v4(blo + o, lr);
          st_shared_v4(blo + o + 16, lm);
        }
      }
      fence_proxy_async();
      named_sync(1, R::conv);  // every converter is done with zbuf(b) and B[b]
      if (threadIdx.x == 0) mbar_arrive(Bq.bfull + b);
      if (warp == 0 && w2 < A.nitems) stage(w2, b);
      w = next_item(w);
      w2 = w2 < A.nitems ? next_item(w2) : A.nitems;
    }
  } else if (warp == R::mma_warp) {
    // ---- MMA issue ----
    const uint32_t idesc = idesc_f16_f32(128, N);
    const uint32_t sbo = (uint32_t)kc * 128, sbase = smem_u32(sm);
    const uint64_t ah = smem_desc(sbase + (uint32_t)L.a, 128, sbo);
    const uint64_t al = smem_desc(sbase + (uint32_t)L.a + 256 * Kp, 128, sbo);
    const bool aok = mbar_wait_or(Bq.abar, 0, Bq.abort, A.err, kErrL2l);
    int w = first;
    for (int it = 0; w < A.nitems; it++) {
      const int b = it & 1, ph = (it >> 1) & 1;
      const bool ok = mbar_wait_or(Bq.bfull + b, ph, Bq.abort, A.err, kErrL2l) &&
                      mbar_wait_or(Bq.tfree + b, ph ^ 1, Bq.abort, A.err, kErrL2l) && aok;
      if (lane == 0) {
        tc_fence_after();
        if (ok) {
          const uint64_t bh = smem_desc(smem_u32(bbuf(b)), 128, sbo);
          const uint64_t bl = smem_desc(smem_u32(bbuf(b)) + N * Kp * 2, 128, sbo);
          const uint32_t d = tmem + (uint32_t)(b * N);
          for (int ks = 0; ks < Kp / 16; ks++) {
            const uint32_t k = ks * 256;
            mma_f16(d, desc_add(ah, k), desc_add(bh, k), idesc, ks ? 1 : 0);
            mma_f16(d, desc_add(ah, k), desc_add(bl, k), idesc, 1);
            mma_f16(d, desc_add(al, k), desc_add(bh, k), idesc, 1);
          }
        }
        mma_commit(Bq.bfree + b);
        mma_commit(Bq.tfull + b);
      }
      __syncwarp();
      w = next_item(w);
    }
  } else {
    // ---- epilogue: lane = child sample, 16 columns = 2 parents x 4 children x (re, im) ----
    const int ew = warp - R::epi_warp0, qd = warp & 3, ch0 = ew >> 2;  // lane quarter, column group
    const int km = 32 * qd + lane;
    const int nc = 2 << A.lg_np, npm = (1 << A.lg_np) - 1;
    const int so = A.ns_out, qoff[4] = {0, so, nc * so, nc * so + so};
    int w = first;
    for (int it = 0; w < A.nitems; it++) {
      const int b = it & 1, ph = (it >> 1) & 1;
      const bool ok = mbar_wait_or(Bq.tfull + b, ph, Bq.abort, A.err, kErrL2l);
      tc_fence_after();
      const int rhs = w / A.items_per_rhs, p0 = (w % A.items_per_rhs) * A.ppi;
      const float inv = A.inv_a / scale_of(w);
      // the item's parents share a row: parent p0 + pl's first child is 2 pl clusters on
      float2 *ob = A.loc + (size_t)rhs * A.mp + A.off_out + km +
                   (size_t)(2 * (p0 >> A.lg_np) * nc + 2 * (p0 & npm)) * so;
      for (int cg = 0; cg < N / (32 * R::epi_groups); cg++) {  // 32 columns = 4 parents
        const int col0 = ch0 * (N / R::epi_groups) + 32 * cg;
        float d[32];
        tmem_ld32(tmem + ((uint32_t)(32 * qd) << 16) + (uint32_t)(b * N + col0), d);
        if (!ok || km >= A.ns_out) continue;
#pragma unroll
        for (int u = 0; u < 4; u++) {
          float2 *o = ob + (size_t)2 * (col0 / 8 + u) * so;
#pragma unroll
          for (int q = 0; q < 4; q++) o[qoff[q]] = make_float2(d[8 * u + 2 * q] * inv, d[8 * u + 2 * q + 1] * inv);
        }
      }
      tc_fence_before();
      named_sync(2, R::epi);  // the accumulator is read out
      if (ew == 0 && lane == 0) mbar_arrive(Bq.tfree + b);
      w = next_item(w);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, 2 * N);
}

// ---- M2M, persistent, for parents of at most 128 samples ----
// The same shape as the L2L kernel, transposed roles: A = the interpolation
// matrix [128 parent samples x Kp child samples] resident in shared memory;
// an item is 32 (or 16) parents of one RHS, B rows 8 parent + 2 q + (re, im)
// hold child q's ring (the children's own samples, no shift before the
// product), and the epilogue forms sum_q shm[q][k] D_q[k] for each parent
// sample k on its lane.  The operand scale comes from the child level's
// maximum per RHS (written by the kernel that produced the children), and the
// kernel writes the parent level's maximum for the next transition.
constexpr int kErrM2m = 123;

struct M2mArgs {
  float2 *mul;  // every level's multipoles; children at off_in, parents at off_out
  size_t mp, off_in, off_out;
  int lg_np, ns_in, ns_out, Kp, ppi, mt;  // mt: 128-sample tiles of the parent ring (1 or 2)
  unsigned kc_magic;
  const uint8_t *A;    // per tile, [128 x Kp] FP16 hi then lo
  const float2 *shm;   // [4][ns_out] multipole shifts of the parent level
  float inv_a;
  int nparents, items_per_rhs, nitems;
  const int *active;
  int *err;
  unsigned *levmax;
  int lvl_in, lvl_out;
};

// A hi/lo; B[2] hi/lo; staged child rings [2][2 rows][2 ppi clusters][ns]
// (the item's parents are consecutive in one row, so each child row is one
// contiguous run), each buffer followed by Kp zero samples; barriers and flags.
struct M2mSmem {
  size_t a, b, bbuf, z, zbuf, bar, total;
  __host__ __device__ M2mSmem(int Kp, int ppi, int ns, int mt) {
    a = 0;
    b = a + (size_t)512 * Kp * mt;
    bbuf = (size_t)32 * ppi * Kp;
    z = b + 2 * bbuf;
    zbuf = ((size_t)(4 * ppi * ns + Kp) * 8 + 127) & ~(size_t)127;
    bar = z + 2 * zbuf;
    total = bar + 256;
  }
};

template <class R>
__global__ void __launch_bounds__(R::threads, 1) k_tc_m2m(M2mArgs A) {
  extern __shared__ __align__(1024) char sm[];
  const M2mSmem L(A.Kp, A.ppi, A.ns_in, A.mt);
  const int N = 8 * A.ppi, Kp = A.Kp, kc = Kp / 8, zs = A.ns_in;
  uint64_t *bars = (uint64_t *)(sm + L.bar);
  uint64_t *abar = bars, *zfull = bars + 1, *bfull = bars + 3, *bfree = bars + 5, *tfull = bars + 7,
           *tfree = bars + 9;
  uint32_t *tslot = (uint32_t *)(bars + 11);
  volatile int *abort = (volatile int *)(bars + 12);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  auto bbuf = [&](int b) { return sm + L.b + b * L.bbuf; };  // hi, then lo N * Kp * 2 bytes on
  auto zbuf = [&](int b) { return (float2 *)(sm + L.z + b * L.zbuf); };
  if (threadIdx.x == 0) {
    for (int i = 0; i < 11; i++) mbar_init(bars + i, 1);
    *abort = 0;
    fence_mbar_init();
  }
  if (warp == 0) tmem_alloc(tslot, 2 * A.mt * N);
  // zero both buffers: the tails past the last ring are read (against zero weights) and stay 0
  for (int e = threadIdx.x; e < (int)(2 * L.zbuf / 4); e += blockDim.x) ((float *)zbuf(0))[e] = 0.f;
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  auto next_item = [&](int w) {
    do w += gridDim.x;
    while (w < A.nitems && A.active && !A.active[w / A.items_per_rhs]);
    return w;
  };
  const int first = (A.active && !A.active[blockIdx.x / A.items_per_rhs]) ? next_item(blockIdx.x) : blockIdx.x;
  auto scale_of = [&](int w) {
    return pow2_scale(__uint_as_float(A.levmax[(w / A.items_per_rhs) * kMaxLevels + A.lvl_in]));
  };
  const int nc = 2 << A.lg_np, npm = (1 << A.lg_np) - 1;
  const uint32_t ring_bytes = (uint32_t)A.ns_in * 8;
  // an item's children: two contiguous runs of 2 ppi rings (child rows 2 py, 2 py + 1)
  auto stage = [&](int w, int b) {
    if (lane != 0) return;
    const int rhs = w / A.items_per_rhs, P = (w % A.items_per_rhs) * A.ppi;
    const int py = P >> A.lg_np, px = P & npm;
    const float2 *base = A.mul + (size_t)rhs * A.mp + A.off_in;
    const uint32_t run = 2 * A.ppi * ring_bytes;
    mbar_expect_tx(zfull + b, 2 * run);
    for (int qy = 0; qy < 2; qy++)
      bulk_g2s(zbuf(b) + qy * 2 * A.ppi * zs, base + ((size_t)(2 * py + qy) * nc + 2 * px) * A.ns_in, run, zfull + b);
  };
  const int ngroups = A.ppi * kc;  // core-matrix groups of B (8 rows x 8 samples)

  if (warp < R::conv_warps) {
    // ---- converters: B[b] rows 8 parent + 2 q + (re, im) = child q's samples times s ----
    if (warp == 0) {
      if (lane == 0) {
        mbar_expect_tx(abar, 512 * Kp * A.mt);
        bulk_g2s(sm + L.a, A.A, 512 * Kp * A.mt, abar);
      }
      __syncwarp();
      if (first < A.nitems) stage(first, 0);
      const int second = first < A.nitems ? next_item(first) : A.nitems;
      if (second < A.nitems) stage(second, 1);
    }
    int w = first, w2 = first < A.nitems ? next_item(next_item(first)) : A.nitems;
    for (int it = 0; w < A.nitems; it++) {
      const int b = it & 1, ph = (it >> 1) & 1;
      const bool zok = mbar_wait_or(zfull + b, ph, abort, A.err, kErrM2m);
      const bool bok = mbar_wait_or(bfree + b, ph ^ 1, abort, A.err, kErrM2m);
      const float s = scale_of(w);
      const float2 *zst = zbuf(b);
      char *bhi = bbuf(b), *blo = bhi + (size_t)N * Kp * 2;
      if (zok && bok) {
#pragma unroll 2
        for (int u = threadIdx.x; u < 4 * ngroups; u += R::conv) {
          const int q = u & 3, cm = u >> 2;
          const int pl = (int)__umulhi((unsigned)cm, A.kc_magic), j8 = cm - pl * kc;
          const int slot = (q >> 1) * 2 * A.ppi + 2 * pl + (q & 1);
          const float4 *zp = (const float4 *)(zst + slot * zs + 8 * j8);
          uint32_t hr[4], lr[4], hm[4], lm[4];
#pragma unroll
          for (int i = 0; i < 4; i++) {
            const float4 z = zp[i];
            split2u(z.x * s, z.z * s, hr[i], lr[i]);
            split2u(z.y * s, z.w * s, hm[i], lm[i]);
          }
          const uint32_t o = (uint32_t)cm * 128 + q * 32;
          st_shared_v4(bhi + o, hr);
          st_shared_v4(bhi + o + 16, hm);
          st_shared_v4(blo + o, lr);
          st_shared_v4(blo + o + 16, lm);
        }
      }
      fence_proxy_async();
      named_sync(1, R::conv);  // every converter is done with zbuf(b) and B[b]
      if (threadIdx.x == 0) mbar_arrive(bfull + b);
      if (warp == 0 && w2 < A.nitems) stage(w2, b);
      w = next_item(w);
      w2 = w2 < A.nitems ? next_item(w2) : A.nitems;
    }
  } else if (warp == R::mma_warp) {
    // ---- MMA issue ----
    const uint32_t idesc = idesc_f16_f32(128, N);
    const uint32_t sbo = (uint32_t)kc * 128, sbase = smem_u32(sm);
    const uint64_t ah = smem_desc(sbase + (uint32_t)L.a, 128, sbo);
    const uint64_t al = smem_desc(sbase + (uint32_t)L.a + 256 * Kp, 128, sbo);
    const uint32_t tile_bytes = 512 * Kp;  // hi and lo of one 128-sample tile
    const bool aok = mbar_wait_or(abar, 0, abort, A.err, kErrM2m);
    int w = first;
    for (int it = 0; w < A.nitems; it++) {
      const int b = it & 1, ph = (it >> 1) & 1;
      const bool ok = mbar_wait_or(bfull + b, ph, abort, A.err, kErrM2m) &&
                      mbar_wait_or(tfree + b, ph ^ 1, abort, A.err, kErrM2m) && aok;
      if (lane == 0) {
        tc_fence_after();
        if (ok) {
          const uint64_t bh = smem_desc(smem_u32(bbuf(b)), 128, sbo);
          const uint64_t bl = smem_desc(smem_u32(bbuf(b)) + N * Kp * 2, 128, sbo);
          for (int t = 0; t < A.mt; t++) {
            const uint32_t d = tmem + (uint32_t)((b * A.mt + t) * N), ta = t * tile_bytes;
            for (int ks = 0; ks < Kp / 16; ks++) {
              const uint32_t k = ks * 256;
              mma_f16(d, desc_add(ah, ta + k), desc_add(bh, k), idesc, ks ? 1 : 0);
              mma_f16(d, desc_add(ah, ta + k), desc_add(bl, k), idesc, 1);
              mma_f16(d, desc_add(al, ta + k), desc_add(bh, k), idesc, 1);
            }
          }
        }
        mma_commit(bfree + b);
        mma_commit(tfull + b);
      }
      __syncwarp();
      w = next_item(w);
    }
  } else {
    // ---- epilogue: lane = parent sample (of tile t), 32 columns = 4 parents x 4 children x (re, im) ----
    const int ew = warp - R::epi_warp0, qd = warp & 3, ch0 = ew >> 2;  // lane quarter, column group
    float2 shq[2][4];
#pragma unroll
    for (int t = 0; t < 2; t++)
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int km = 128 * t + 32 * qd + lane;
        shq[t][q] = t < A.mt && km < A.ns_out ? __ldg(A.shm + q * A.ns_out + km) : make_float2(0.f, 0.f);
      }
    int w = first;
    for (int it = 0; w < A.nitems; it++) {
      const int b = it & 1, ph = (it >> 1) & 1;
      const bool ok = mbar_wait_or(tfull + b, ph, abort, A.err, kErrM2m);
      tc_fence_after();
      const int rhs = w / A.items_per_rhs, p0 = (w % A.items_per_rhs) * A.ppi;
      const float inv = A.inv_a / scale_of(w);
      float omx = 0.f;
#pragma unroll
      for (int t = 0; t < 2; t++) {
        if (t >= A.mt) break;
        const int km = 128 * t + 32 * qd + lane;
        float2 *obase = A.mul + (size_t)rhs * A.mp + A.off_out + km;
        for (int cg = 0; cg < N / (32 * R::epi_groups); cg++) {  // 32 columns = 4 parents
          const int col0 = ch0 * (N / R::epi_groups) + 32 * cg;
          float d[32];
          tmem_ld32(tmem + ((uint32_t)(32 * qd) << 16) + (uint32_t)((b * A.mt + t) * N + col0), d);
          if (!ok || km >= A.ns_out) continue;
#pragma unroll
          for (int u = 0; u < 4; u++) {
            const int P = p0 + col0 / 8 + u;
            float2 acc = make_float2(0.f, 0.f);
#pragma unroll
            for (int q = 0; q < 4; q++)
              cfma(acc, shq[t][q], make_float2(d[8 * u + 2 * q] * inv, d[8 * u + 2 * q + 1] * inv));
            obase[(size_t)P * A.ns_out] = acc;
            omx = fmaxf(omx, fmaxf(fabsf(acc.x), fabsf(acc.y)));
          }
        }
      }
      tc_fence_before();
      named_sync(2, R::epi);  // the accumulator is read out
      if (ew == 0 && lane == 0) mbar_arrive(tfree + b);
      // the parent level's maximum for the next transition (omx >= 0: bits order as values)
      const unsigned mbits = __reduce_max_sync(0xffffffffu, __float_as_uint(omx));
      if (lane == 0 && ok && mbits) atomicMax(&A.levmax[rhs * kMaxLevels + A.lvl_out], mbits);
      w = next_item(w);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, 2 * A.mt * N);
}

struct M2mPlan {
  uint8_t *A = nullptr;  // device
  int Kp = 0, ppi = 0, mt = 1;
  unsigned kc_magic = 0;
  float inv_a = 1;
  bool ok = false;
};

// One L2L transition on the tensor cores (child level `lvl`).
struct L2lPlan {
  uint8_t *A = nullptr;  // device
  int Kp = 0, ppi = 0;
  unsigned kc_magic = 0;
  float inv_a = 1, shl_max = 1;
  bool ok = false;
};

// One level transition: weight chunks and per-tile windows.
struct Transition {
  int mtiles = 0;
  int *kw0 = nullptr, *nchunk = nullptr, *chunk0 = nullptr;  // device
  uint8_t *A = nullptr;                                      // device
  float inv_a = 1;
  bool ok = false;
};

// Packs reals(row, k0 .. k0+63) of a [128 x K] block as FP16 hi then lo in the
// K-major core-matrix layout (SBO = 8 chunks x 128 B, LBO = 128 B).
template <class F>
void pack_chunk(std::vector<uint8_t> &buf, size_t at, int k0, double scale, F real_at) {
  __half *hi = (__half *)(buf.data() + at), *lo = (__half *)(buf.data() + at + kAHalf);
  for (int n = 0; n < 128; n++)
    for (int k = 0; k < kKC; k++) {
      const double v = real_at(n, k0 + k) * scale;
      const __half h = __double2half(v);
      const __half l = __double2half(v - (double)__half2float(h));
      const size_t idx = ((size_t)(n / 8) * (kKC / 8) + k / 8) * 64 + (n % 8) * 8 + (k % 8);
      hi[idx] = h;
      lo[idx] = l;
    }
}

}  // namespace

struct BandPlan {
  Transition m2m[kMaxLevels];  // indexed by parent level
  M2mPlan pm2m[kMaxLevels];    // persistent M2M, indexed by parent level
  L2lPlan l2l[kMaxLevels];     // indexed by child level
  std::vector<void *> allocs;
  int sms = 148;
};

// Packs a dense [128 x Kp] real matrix as FP16 hi then lo (K-major core
// matrices) after a power-of-two scale; returns the inverse of the scale.
static double pack_resident(const std::vector<double> &dense, int Kp, std::vector<uint8_t> &buf, int tiles = 1) {
  double mw = 0;
  for (double v : dense) mw = std::max(mw, std::abs(v));
  int e2;
  std::frexp(mw > 0 ? mw : 1.0, &e2);
  const double sa = std::ldexp(1.0, 14 - e2);
  buf.assign((size_t)512 * Kp * tiles, 0);
  for (int t = 0; t < tiles; t++) {  // tile t: rows 128 t .. 128 t + 127, hi then lo
    __half *hi = (__half *)(buf.data() + (size_t)512 * Kp * t), *lo = hi + (size_t)128 * Kp;
    for (int m = 0; m < 128; m++)
      for (int k = 0; k < Kp; k++) {
        const double v = dense[(size_t)(128 * t + m) * Kp + k] * sa;
        const __half h = __double2half(v);
        const __half l = __double2half(v - (double)__half2float(h));
        const size_t idx = ((size_t)(m / 8) * (Kp / 8) + k / 8) * 64 + (m % 8) * 8 + (k % 8);
        hi[idx] = h;
        lo[idx] = l;
      }
  }
  return 1.0 / sa;
}

// ceil(2^32 / kc), if it divides exactly for every group index below `count`.
static bool kc_magic(unsigned kc, unsigned count, unsigned *magic) {
  const unsigned m = (unsigned)((((unsigned long long)1 << 32) + kc - 1) / kc);
  for (unsigned cm = 0; cm < count; cm++)
    if ((unsigned)(((unsigned long long)cm * m) >> 32) != cm / kc) return false;
  *magic = m;
  return true;
}

// The persistent M2M into parent level i (ns_i <= 128): the interpolation
// matrix [parent sample x child sample] resident in shared memory.
static isg_status build_m2m(isg_ctx *c, int i, size_t smem_cap) {
  const HostTables &H = c->T;
  const int ns_out = H.nsamp[i], ns_in = H.nsamp[i + 1], ni = H.ninter;
  M2mPlan &T = c->band->pm2m[i];
  if (ns_out > 256) return ISG_OK;
  const int Kp = (ns_in + 15) / 16 * 16, mt = (ns_out + 127) / 128;
  int ppi = 0;
  for (int cand : {32, 16, 8})
    if (M2mSmem(Kp, cand, ns_in, mt).total <= smem_cap && (1 << i) >= cand) {
      ppi = cand;
      break;
    }
  const int nparents = 1 << (2 * i);
  if (!ppi || nparents % ppi || !kc_magic(Kp / 8, (unsigned)(ppi * Kp / 8), &T.kc_magic)) return ISG_OK;
  std::vector<double> dense((size_t)128 * mt * Kp, 0.0);
  for (int k = 0; k < ns_out; k++)
    for (int t = 0; t < ni; t++) dense[(size_t)k * Kp + H.intind[i][(size_t)k * ni + t]] += H.interp[i][(size_t)k * ni + t];
  std::vector<uint8_t> buf;
  T.inv_a = (float)pack_resident(dense, Kp, buf, mt);
  isg_status e;
  if ((e = cuda_check(c, cudaMalloc(&T.A, buf.size()), "m2m alloc")) != ISG_OK) return e;
  if ((e = cuda_check(c, cudaMemcpy(T.A, buf.data(), buf.size(), cudaMemcpyHostToDevice), "m2m upload")) != ISG_OK)
    return e;
  T.Kp = Kp;
  T.ppi = ppi;
  T.mt = mt;
  T.ok = true;
  return ISG_OK;
}

// The [128 x Kp] anterpolation matrix of child level i (rows: child samples,
// columns: parent samples) as FP16 hi then lo in the K-major core-matrix
// layout, after a power-of-two scale; shl_max = max |shiftloc| of the parent.
static isg_status build_l2l(isg_ctx *c, int i, size_t smem_cap) {
  const HostTables &H = c->T;
  const int ns_out = H.nsamp[i], ns_in = H.nsamp[i - 1], W = 2 * H.ninter, taps = H.antcount[i];
  L2lPlan &T = c->band->l2l[i];
  if (ns_out > 128) return ISG_OK;
  const int Kp = (ns_in + 15) / 16 * 16;
  int ppi = 0;
  for (int cand : {32, 16, 8})
    if (L2lSmem(Kp, cand, ns_in).total <= smem_cap) {
      ppi = cand;
      break;
    }
  const int nparents = 1 << (2 * (i - 1));
  if (!ppi || nparents % ppi || (1 << (i - 1)) < ppi) return ISG_OK;  // an item's parents share a row
  std::vector<double> dense((size_t)128 * Kp, 0.0);
  for (int k = 0; k < ns_out; k++)
    for (int t = 0; t < taps; t++) {
      const int j = H.antind[i][(size_t)k * W + t];
      dense[(size_t)k * Kp + j] += H.anterp[i][(size_t)k * W + t];
    }
  if (!kc_magic(Kp / 8, (unsigned)(ppi * Kp / 8), &T.kc_magic)) return ISG_OK;
  std::vector<uint8_t> buf;
  T.inv_a = (float)pack_resident(dense, Kp, buf);
  double smax = 0;
  for (const cd &z : H.shiftloc[i - 1]) smax = std::max(smax, std::abs(z));
  isg_status e;
  if ((e = cuda_check(c, cudaMalloc(&T.A, buf.size()), "l2l alloc")) != ISG_OK) return e;
  if ((e = cuda_check(c, cudaMemcpy(T.A, buf.data(), buf.size(), cudaMemcpyHostToDevice), "l2l upload")) != ISG_OK)
    return e;
  T.Kp = Kp;
  T.ppi = ppi;
  T.shl_max = (float)std::max(smax, 1e-30);
  T.ok = true;
  return ISG_OK;
}

// Builds one transition from rows of taps (index into the input ring, weight).
static isg_status build_transition(isg_ctx *c, Transition &T, int ns_out, int ns_in,
                                   const std::vector<std::vector<std::pair<int, double>>> &rows) {
  double mw = 0;
  for (auto &r : rows)
    for (auto &t : r) mw = std::max(mw, std::abs(t.second));
  int e2;
  std::frexp(mw > 0 ? mw : 1.0, &e2);
  const double sa = std::ldexp(1.0, 14 - e2);
  T.mtiles = (ns_out + 127) / 128;
  std::vector<int> kw0(T.mtiles), nch(T.mtiles), ch0(T.mtiles);
  std::vector<uint8_t> buf;
  int chunks = 0;
  for (int mt = 0; mt < T.mtiles; mt++) {
    std::vector<char> used(ns_in, 0);
    for (int m = mt * 128; m < std::min(ns_out, mt * 128 + 128); m++)
      for (auto &t : rows[m])
        if (t.second != 0.0) used[t.first] = 1;
    // shortest circular arc covering every used sample
    int start = 0, len = ns_in, best_gap = 0, nused = 0;
    for (int j = 0; j < ns_in; j++) nused += used[j];
    if (nused > 0 && nused < ns_in) {
      int first = -1;
      for (int j = 0; j < ns_in; j++)
        if (used[j]) {
          first = j;
          break;
        }
      int prev = first;
      for (int step = 1; step <= ns_in; step++) {
        const int j = (first + step) % ns_in;
        if (!used[j]) continue;
        const int gap = (j - prev + ns_in) % ns_in - 1;
        if (gap > best_gap) {
          best_gap = gap;
          start = j;
        }
        prev = j;
        if (j == first) break;
      }
      len = ns_in - best_gap;
    }
    const bool whole = len >= ns_in - 8;
    kw0[mt] = whole ? -1 : start;
    const int span = whole ? ns_in : len;
    nch[mt] = (span + kKC - 1) / kKC;
    ch0[mt] = chunks;
    std::vector<double> dense((size_t)128 * nch[mt] * kKC, 0.0);
    for (int m = mt * 128; m < std::min(ns_out, mt * 128 + 128); m++)
      for (auto &t : rows[m]) {
        const int kk = whole ? t.first : (t.first - start + ns_in) % ns_in;
        if (kk < nch[mt] * kKC) dense[(size_t)(m - mt * 128) * nch[mt] * kKC + kk] += t.second;
      }
    buf.resize(buf.size() + (size_t)nch[mt] * 2 * kAHalf, 0);
    for (int ch = 0; ch < nch[mt]; ch++)
      pack_chunk(buf, (size_t)(chunks + ch) * 2 * kAHalf, ch * kKC, sa,
                 [&](int n, int k) { return dense[(size_t)n * nch[mt] * kKC + k]; });
    chunks += nch[mt];
  }
  isg_status e;
  if ((e = cuda_check(c, cudaMalloc(&T.A, buf.size()), "band alloc")) != ISG_OK) return e;
  if ((e = cuda_check(c, cudaMalloc(&T.kw0, T.mtiles * sizeof(int)), "band alloc")) != ISG_OK) return e;
  if ((e = cuda_check(c, cudaMalloc(&T.nchunk, T.mtiles * sizeof(int)), "band alloc")) != ISG_OK) return e;
  if ((e = cuda_check(c, cudaMalloc(&T.chunk0, T.mtiles * sizeof(int)), "band alloc")) != ISG_OK) return e;
  cudaMemcpy(T.A, buf.data(), buf.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(T.kw0, kw0.data(), T.mtiles * sizeof(int), cudaMemcpyHostToDevice);
  cudaMemcpy(T.nchunk, nch.data(), T.mtiles * sizeof(int), cudaMemcpyHostToDevice);
  cudaMemcpy(T.chunk0, ch0.data(), T.mtiles * sizeof(int), cudaMemcpyHostToDevice);
  T.inv_a = (float)(1.0 / sa);
  T.ok = true;
  return ISG_OK;
}

isg_status band_setup(isg_ctx *c) {
  c->band = new BandPlan();
  if (!tc_available(c)) return ISG_OK;
  const HostTables &H = c->T;
  const int L = H.L, ni = H.ninter;
  isg_status e;
  for (int i = 2; i <= L - 2; i++) {  // M2M into parent level i
    const int nsp = H.nsamp[i], nsc = H.nsamp[i + 1];
    std::vector<std::vector<std::pair<int, double>>> rows(nsp);
    for (int k = 0; k < nsp; k++)
      for (int t = 0; t < ni; t++)
        rows[k].push_back({H.intind[i][(size_t)k * ni + t], H.interp[i][(size_t)k * ni + t]});
    if ((e = build_transition(c, c->band->m2m[i], nsp, nsc, rows)) != ISG_OK) return e;
  }
  int dev = 0, optin = 0;
  cudaFuncAttributes fa;
  if ((e = cuda_check(c, cudaGetDevice(&dev), "device")) != ISG_OK ||
      (e = cuda_check(c, cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev), "attr")) !=
          ISG_OK ||
      (e = cuda_check(c, cudaDeviceGetAttribute(&c->band->sms, cudaDevAttrMultiProcessorCount, dev), "attr")) !=
          ISG_OK ||
      (e = cuda_check(c, cudaFuncGetAttributes(&fa, k_tc_l2l<L2lRoles>), "l2l attr")) != ISG_OK)
    return e;
  const size_t cap = (size_t)optin - fa.sharedSizeBytes;
  for (int i = 3; i < L; i++)  // L2L into child level i
    if ((e = build_l2l(c, i, cap)) != ISG_OK) return e;
  for (int i = 2; i <= L - 2; i++)  // persistent M2M into parent level i
    if ((e = build_m2m(c, i, cap)) != ISG_OK) return e;
  if ((e = cuda_check(c, cudaFuncSetAttribute(k_tc_m2m<M2mRoles>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cap),
                      "m2m attr")) != ISG_OK)
    return e;
  if ((e = cuda_check(c, cudaFuncSetAttribute(k_tc_l2l<L2lRoles>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cap),
                      "l2l attr")) != ISG_OK)
    return e;
  return cuda_check(c, cudaFuncSetAttribute(k_tc_band, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmem),
                    "band attr");
}

void band_destroy(isg_ctx *c) {
  if (!c->band) return;
  for (int i = 0; i < kMaxLevels; i++)
  {
    Transition *T = &c->band->m2m[i];
    cudaFree(T->A);
    cudaFree(T->kw0);
    cudaFree(T->nchunk);
    cudaFree(T->chunk0);
    cudaFree(c->band->l2l[i].A);
    cudaFree(c->band->pm2m[i].A);
  }
  delete c->band;
  c->band = nullptr;
}

static isg_status band_launch(isg_ctx *c, int lvl, const Transition &T, const float2 *src, float2 *dst, int n_p,
                              int ns_in, int ns_out, const float2 *shift, int nrhs, const int *active,
                              cudaStream_t st) {
  BandArgs A;
  A.src = src;
  A.dst = dst;
  A.mp = c->P.mp;
  A.n_p = n_p;
  A.ns_in = ns_in;
  A.ns_out = ns_out;
  A.shift = shift;
  A.A = T.A;
  A.kw0 = T.kw0;
  A.nchunk = T.nchunk;
  A.chunk0 = T.chunk0;
  A.inv_a = T.inv_a;
  A.nparents = n_p * n_p;
  A.ncols = A.nparents * nrhs;
  A.active = active;
  A.err = c->tc_err_flag();
  A.levmax = c->levmax;
  A.lvl_in = lvl + 1;
  A.lvl_out = lvl;
  count_launch();
  k_tc_band<<<dim3((A.ncols + kParents - 1) / kParents, T.mtiles), 256, kSmem, st>>>(A);
  return cuda_check(c, cudaGetLastError(), "band launch");
}

bool band_m2m(isg_ctx *c, int lvl, float2 *mul, int nrhs, const int *active, cudaStream_t st, isg_status *e) {
  if (!c->band || lvl >= kMaxLevels) return false;
  const DevLevel &p = c->P.lv[lvl], &ch = c->P.lv[lvl + 1];
  if (c->band->pm2m[lvl].ok) {
    const M2mPlan &T = c->band->pm2m[lvl];
    M2mArgs A;
    A.mul = mul;
    A.mp = c->P.mp;
    A.off_in = ch.off;
    A.off_out = p.off;
    A.lg_np = 0;
    while ((1 << A.lg_np) < p.n) A.lg_np++;
    A.ns_in = ch.ns;
    A.ns_out = p.ns;
    A.Kp = T.Kp;
    A.ppi = T.ppi;
    A.mt = T.mt;
    A.kc_magic = T.kc_magic;
    A.A = T.A;
    A.shm = p.shm;
    A.inv_a = T.inv_a;
    A.nparents = p.n * p.n;
    A.items_per_rhs = A.nparents / T.ppi;
    A.nitems = A.items_per_rhs * nrhs;
    A.active = active;
    A.err = c->tc_err_flag();
    A.levmax = c->levmax;
    A.lvl_in = lvl + 1;
    A.lvl_out = lvl;
    count_launch();
    k_tc_m2m<M2mRoles><<<std::min(A.nitems, c->band->sms), M2mRoles::threads, M2mSmem(T.Kp, T.ppi, ch.ns, T.mt).total, st>>>(A);
    *e = cuda_check(c, cudaGetLastError(), "m2m launch");
    return true;
  }
  if (!c->band->m2m[lvl].ok) return false;
  *e = band_launch(c, lvl, c->band->m2m[lvl], mul + ch.off, mul + p.off, p.n, ch.ns, p.ns, p.shm, nrhs, active,
                   st);
  return true;
}


bool band_l2l(isg_ctx *c, int lvl, float2 *loc, int nrhs, const int *active, cudaStream_t st, isg_status *e) {
  if (!c->band || lvl >= kMaxLevels || !c->band->l2l[lvl].ok) return false;
  const L2lPlan &T = c->band->l2l[lvl];
  const DevLevel &p = c->P.lv[lvl - 1], &ch = c->P.lv[lvl];
  L2lArgs A;
  A.loc = loc;
  A.mp = c->P.mp;
  A.off_in = p.off;
  A.off_out = ch.off;
  A.lg_np = 0;
  while ((1 << A.lg_np) < p.n) A.lg_np++;
  A.ns_in = p.ns;
  A.ns_out = ch.ns;
  A.Kp = T.Kp;
  A.kc_magic = T.kc_magic;
  A.ppi = T.ppi;
  A.A = T.A;
  A.shl = p.shlT;
  A.inv_a = T.inv_a;
  A.shl_max = T.shl_max;
  A.locmax = c->locmax;
  A.lvl_in = lvl - 1;
  A.nparents = p.n * p.n;
  A.items_per_rhs = A.nparents / T.ppi;
  A.nitems = A.items_per_rhs * nrhs;
  A.active = active;
  A.err = c->tc_err_flag();
  count_launch();
  k_tc_l2l<L2lRoles><<<std::min(A.nitems, c->band->sms), L2lRoles::threads, L2lSmem(T.Kp, T.ppi, p.ns).total, st>>>(A);
  *e = cuda_check(c, cudaGetLastError(), "l2l launch");
  return true;
}

}  // namespace isg
