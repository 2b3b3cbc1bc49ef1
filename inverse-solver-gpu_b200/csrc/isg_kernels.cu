// Complex-FP32 SIMT kernels of the MLFMA matvec (the reference's kernels.cu
// P2M/M2M/M2L/L2L/L2P/P2P stages, re-designed for a batched, RHS-major layout
// and raster cluster numbering).  The tensor-core leaf kernels live in
// isg_tc.cu.
#include <algorithm>
#include <atomic>

#include "isg_device.cuh"

namespace isg {

static std::atomic<int64_t> g_launches{0};
void count_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
int64_t launch_count() { return g_launches.load(std::memory_order_relaxed); }

namespace {

constexpr int kNearTY = 4;  // near-field tile: 4 x 8 leaves per block
constexpr int kNearTX = 8;
constexpr int kHaloLeaves = (kNearTY + 2) * (kNearTX + 2);

__device__ __forceinline__ bool inactive(const int *active, int rhs) { return active && !active[rhs]; }

// P2M (kernels.cu:6-30, solve.cpp:80-92): leaf multipoles
// mul[leaf][k] = sum_n coeff[k][n] * in[leaf*64 + n], 32 leaves per block.
__global__ void __launch_bounds__(128) k_p2m(const float2 *__restrict__ x, const float2 *__restrict__ g,
                                             int64_t gstride, int mode, const int *__restrict__ active,
                                             const float2 *__restrict__ coeffT, int ns, int nleaves, int U,
                                             float2 *__restrict__ mul_leaf, size_t mp) {
  const int rhs = blockIdx.y;
  if (inactive(active, rhs)) return;
  __shared__ float2 xs[32][kBB];
  const int leaf0 = blockIdx.x * 32;
  const float2 *xr = x + (size_t)rhs * U;
  const float2 *gr = g ? g + rhs * gstride : nullptr;
  for (int e = threadIdx.x; e < 32 * kBB; e += blockDim.x) {
    const int leaf = leaf0 + e / kBB;
    float2 v = make_float2(0.f, 0.f);
    if (leaf < nleaves) {
      const size_t i = (size_t)leaf * kBB + e % kBB;
      v = load_in(xr, gr, mode, i, i);
    }
    xs[e / kBB][e % kBB] = v;
  }
  __syncthreads();
  float2 *out = mul_leaf + (size_t)rhs * mp;
  for (int u = threadIdx.x; u < 8 * ns; u += blockDim.x) {
    const int k = u % ns, lg = u / ns;
    float2 acc[4] = {};
#pragma unroll 8
    for (int n = 0; n < kBB; n++) {
      const float2 c = __ldg(&coeffT[n * ns + k]);
#pragma unroll
      for (int j = 0; j < 4; j++) cfma(acc[j], c, xs[lg * 4 + j][n]);
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int leaf = leaf0 + lg * 4 + j;
      if (leaf < nleaves) out[(size_t)leaf * ns + k] = acc[j];
    }
  }
}

constexpr int kSmemStage = 200 * 1024;  // largest ring staged in shared memory
constexpr int kStageBudget = 32 * 1024;  // per-block staging target for the small levels

__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(valid ? 8 : 0));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::); }
// Block-wide barrier usable from warp-uniform divergent paths (every warp
// reaches it the same number of times).
__device__ __forceinline__ void block_bar1() { asm volatile("bar.sync 1, %0;\n" ::"r"(blockDim.x)); }

// M2M (kernels.cu:83-136, solve.cpp:93-112): parent sample km gathers the
// 30-tap interpolation of each of its four children, shifts it to the parent
// centre and sums.  A block covers `npb` parents whose children's rings are
// staged in shared memory (STAGE), or reads through L1 when one parent's
// children are too large to stage (top levels only).
template <bool STAGE>
__global__ void __launch_bounds__(256) k_m2m(float2 *__restrict__ mul, size_t mp, size_t off_p, size_t off_c, int n_p,
                                             int ns_p, int ns_c, int npb, int chunks, const int *__restrict__ ifirst,
                                             const float *__restrict__ iw, const float2 *__restrict__ shm,
                                             int ninter, const int *__restrict__ active) {
  extern __shared__ float2 chs[];
  const int rhs = blockIdx.y;
  if (inactive(active, rhs)) return;
  const int nparent = n_p * n_p, n_c = 2 * n_p;
  const int pb = blockIdx.x / chunks, chunk = blockIdx.x % chunks;
  const int p0 = pb * npb, np_here = min(npb, nparent - p0);
  const float2 *base = mul + (size_t)rhs * mp + off_c;
  auto child = [&](int pc, int q) {
    return (size_t)((2 * (pc / n_p) + (q >> 1)) * n_c + 2 * (pc % n_p) + (q & 1)) * ns_c;
  };
  if (STAGE) {
    for (int e = threadIdx.x; e < np_here * 4 * ns_c; e += blockDim.x) {
      const int j = e % ns_c, q = (e / ns_c) & 3, pl = e / (4 * ns_c);
      chs[e] = base[child(p0 + pl, q) + j];
    }
    __syncthreads();
  }
  const int per = (np_here * ns_p + chunks - 1) / chunks, u_hi = min(np_here * ns_p, (chunk + 1) * per);
  for (int u = chunk * per + threadIdx.x; u < u_hi; u += blockDim.x) {
    const int pl = u / ns_p, km = u % ns_p, pc = p0 + pl;
    int idx = ifirst[km];
    float2 acc[4] = {};
    for (int t = 0; t < ninter; t++) {
      const float w = __ldg(&iw[t * ns_p + km]);
#pragma unroll
      for (int q = 0; q < 4; q++) rfma(acc[q], w, STAGE ? chs[(pl * 4 + q) * ns_c + idx] : base[child(pc, q) + idx]);
      if (++idx == ns_c) idx = 0;
    }
    float2 res = make_float2(0.f, 0.f);
#pragma unroll
    for (int q = 0; q < 4; q++) cfma(res, __ldg(&shm[q * ns_p + km]), acc[q]);
    mul[(size_t)rhs * mp + off_p + (size_t)pc * ns_p + km] = res;
  }
}

// M2L (kernels.cu:239-266, solve.cpp:133-148) as a 2-D stencil per sample.
// The far list of a cluster is the 6x6 block of its parent's neighbours'
// children minus its own 3x3 neighbourhood, clipped to the grid, so for a
// cluster of parity (OY, OX) at row 2a+OY the sources are rows 2a-2 .. 2a+3
// of a six-column window, and the 27 translation weights depend only on the
// parity and the sample.  A block owns one chunk of 32 samples: each thread
// keeps its 27 weights in registers for the whole launch and walks a list of
// (tile of 16 x 4 clusters, RHS) items, sliding a 6x6 register window of
// multipoles down a column of eight same-parity clusters.  The (16+4) x (4+4)
// halo of the next item is fetched with cp.async while the current one is
// computed.
constexpr int kM2lRows = 16, kM2lCols = 4, kM2lKC = 32;
constexpr int kM2lHR = kM2lRows + 4, kM2lHC = kM2lCols + 4;
constexpr int kM2lHalo = kM2lHR * kM2lHC * kM2lKC;

struct M2lArgs {
  const float2 *mul;
  float2 *loc;
  size_t mp, off;
  int n, ns, tiles_x, tiles, nitems;
  const float2 *T;
  const int *active;
};

__device__ __forceinline__ void m2l_issue(const M2lArgs &A, int item, int k0, float2 *buf) {
  const int tile = item % A.tiles, rhs = item / A.tiles;
  const int cy0 = (tile / A.tiles_x) * kM2lRows, cx0 = (tile % A.tiles_x) * kM2lCols;
  const float2 *m = A.mul + (size_t)rhs * A.mp + A.off;
  for (int e = threadIdx.x; e < kM2lHalo; e += blockDim.x) {
    const int kk = e % kM2lKC, hc = (e / kM2lKC) % kM2lHC, hr = e / (kM2lKC * kM2lHC);
    const int cy = cy0 - 2 + hr, cx = cx0 - 2 + hc, k = k0 + kk;
    const bool ok = cy >= 0 && cy < A.n && cx >= 0 && cx < A.n && k < A.ns;
    cp_async8(&buf[e], ok ? (const void *)&m[(size_t)(cy * A.n + cx) * A.ns + k] : (const void *)A.mul, ok);
  }
}

// One window step: rows of the 6x6 window live in six register slots that
// rotate by two per step (ROT = step mod 3), so no registers are moved.
template <int OY, int OX, int ROT>
__device__ __forceinline__ void m2l_step(const float2 (*hs)[kM2lHC][kM2lKC], float2 (&w)[6][6],
                                         const float2 (&tw)[6][6], int a, int b, int kk, int cy0, int cx0,
                                         bool live, const M2lArgs &A, int k, float2 *out) {
  constexpr int NR0 = OY + 1, NC0 = OX + 1;  // first near row/column inside the window
#pragma unroll
  for (int j = 0; j < 6; j++) {
    w[(4 + 2 * ROT) % 6][j] = hs[2 * a + 4][2 * b + j][kk];
    w[(5 + 2 * ROT) % 6][j] = hs[2 * a + 5][2 * b + j][kk];
  }
  float2 acc[3] = {};
  int term = 0;
#pragma unroll
  for (int i = 0; i < 6; i++)
#pragma unroll
    for (int j = 0; j < 6; j++) {
      const bool nearby = (i >= NR0 && i < NR0 + 3 && j >= NC0 && j < NC0 + 3);
      if (nearby) continue;
      cfma(acc[term % 3], tw[i][j], w[(i + 2 * ROT) % 6][j]);
      term++;
    }
  const int cy = cy0 + 2 * a + OY, cx = cx0 + 2 * b + OX;
  if (live && cy < A.n && cx < A.n && k < A.ns)
    out[(size_t)(cy * A.n + cx) * A.ns + k] = cadd(acc[0], cadd(acc[1], acc[2]));
}

template <int OY, int OX>
__device__ __forceinline__ void m2l_worker(const M2lArgs &A, float2 *hbuf) {
  constexpr int NR0 = OY + 1, NC0 = OX + 1;
  const int kk = threadIdx.x & 31, b = threadIdx.x >> 7;
  const int k0 = blockIdx.x * kM2lKC, k = k0 + kk;
  float2 tw[6][6];
#pragma unroll
  for (int i = 0; i < 6; i++)
#pragma unroll
    for (int j = 0; j < 6; j++) {
      const bool nearby = (i >= NR0 && i < NR0 + 3 && j >= NC0 && j < NC0 + 3);
      tw[i][j] = (!nearby && k < A.ns) ? __ldg(&A.T[((i + 1 - OY) * 7 + (j + 1 - OX)) * A.ns + k])
                                       : make_float2(0.f, 0.f);
    }
  int buf = 0;
  const int G = gridDim.y;
  for (int item = blockIdx.y; item < A.nitems; item += G) {
    if (item + G < A.nitems) m2l_issue(A, item + G, k0, hbuf + (buf ^ 1) * kM2lHalo);
    cp_async_commit();
    cp_async_wait1();
    block_bar1();
    const float2(*hs)[kM2lHC][kM2lKC] = (const float2(*)[kM2lHC][kM2lKC])(hbuf + buf * kM2lHalo);
    const int tile = item % A.tiles, rhs = item / A.tiles;
    const bool live = !(A.active && !A.active[rhs]);
    const int cy0 = (tile / A.tiles_x) * kM2lRows, cx0 = (tile % A.tiles_x) * kM2lCols;
    float2 *out = A.loc + (size_t)rhs * A.mp + A.off;
    float2 w[6][6];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int j = 0; j < 6; j++) w[i][j] = hs[i][2 * b + j][kk];
    static_assert(kM2lRows / 2 == 8, "window walk is unrolled for eight steps");
#pragma unroll 1
    for (int a = 0; a < 6; a += 3) {
      m2l_step<OY, OX, 0>(hs, w, tw, a, b, kk, cy0, cx0, live, A, k, out);
      m2l_step<OY, OX, 1>(hs, w, tw, a + 1, b, kk, cy0, cx0, live, A, k, out);
      m2l_step<OY, OX, 2>(hs, w, tw, a + 2, b, kk, cy0, cx0, live, A, k, out);
    }
    m2l_step<OY, OX, 0>(hs, w, tw, 6, b, kk, cy0, cx0, live, A, k, out);
    m2l_step<OY, OX, 1>(hs, w, tw, 7, b, kk, cy0, cx0, live, A, k, out);
    block_bar1();
    buf ^= 1;
  }
}

__global__ void __launch_bounds__(256, 1) k_m2l(M2lArgs A) {
  extern __shared__ float2 hbuf[];
  if (blockIdx.y < A.nitems) m2l_issue(A, blockIdx.y, blockIdx.x * kM2lKC, hbuf);
  cp_async_commit();
  switch ((threadIdx.x >> 5) & 3) {
    case 0: m2l_worker<0, 0>(A, hbuf); break;
    case 1: m2l_worker<0, 1>(A, hbuf); break;
    case 2: m2l_worker<1, 0>(A, hbuf); break;
    default: m2l_worker<1, 1>(A, hbuf); break;
  }
}

// L2L (kernels.cu:137-238, solve.cpp:149-169 and 389-429): the parent's local
// expansion, shifted to each child centre, anterpolated to the child rate and
// added to (or written over) the child's local expansion.  A block covers `npb`
// parents whose four shifted rings are staged in shared memory, or reads
// through L1 when one parent's rings are too large (top levels only).
template <bool STAGE>
__global__ void __launch_bounds__(256) k_l2l(float2 *__restrict__ loc, size_t mp, size_t off_p, size_t off_c, int n_p,
                                             int ns_p, int ns_c, int npb, int chunks, const int *__restrict__ afirst,
                                             const float *__restrict__ aw, int awidth,
                                             const float2 *__restrict__ shl_p, int accumulate,
                                             const int *__restrict__ active) {
  extern __shared__ float2 tmp[];
  const int rhs = blockIdx.y;
  if (inactive(active, rhs)) return;
  const int nparent = n_p * n_p, n_c = 2 * n_p;
  const int pb = blockIdx.x / chunks, chunk = blockIdx.x % chunks;
  const int p0 = pb * npb, np_here = min(npb, nparent - p0);
  const float2 *lp0 = loc + (size_t)rhs * mp + off_p;
  if (STAGE) {
    for (int e = threadIdx.x; e < np_here * 4 * ns_p; e += blockDim.x) {
      const int j = e % ns_p, q = (e / ns_p) & 3, pl = e / (4 * ns_p);
      tmp[e] = cmul(__ldg(&shl_p[q * ns_p + j]), lp0[(size_t)(p0 + pl) * ns_p + j]);
    }
    __syncthreads();
  }
  float2 *lc = loc + (size_t)rhs * mp + off_c;
  const int per = (np_here * ns_c + chunks - 1) / chunks, u_hi = min(np_here * ns_c, (chunk + 1) * per);
  for (int u = chunk * per + threadIdx.x; u < u_hi; u += blockDim.x) {
    const int pl = u / ns_c, km = u % ns_c, pc = p0 + pl;
    const float2 *lp = lp0 + (size_t)pc * ns_p;
    int idx = afirst[km];
    float2 acc[4] = {};
    for (int t = 0; t < awidth; t++) {
      const float w = __ldg(&aw[t * ns_c + km]);
      if (STAGE) {
#pragma unroll
        for (int q = 0; q < 4; q++) rfma(acc[q], w, tmp[(pl * 4 + q) * ns_p + idx]);
      } else {
        const float2 v = lp[idx];
#pragma unroll
        for (int q = 0; q < 4; q++) rfma(acc[q], w, cmul(__ldg(&shl_p[q * ns_p + idx]), v));
      }
      if (++idx == ns_p) idx = 0;
    }
    const int py = pc / n_p, px = pc % n_p;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      float2 *d = lc + (size_t)((2 * py + (q >> 1)) * n_c + 2 * px + (q & 1)) * ns_c + km;
      *d = accumulate ? cadd(*d, acc[q]) : acc[q];
    }
  }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// L2P (kernels.cu:32-81, solve.cpp:170-182) + near field (kernels.cu:292-319,
// solve.cpp:199-216) + matvec epilogue (kernels.cu:402-409) + BiCGSTAB partial
// dot products, for a tile of 4 x 8 leaves of one RHS.  The 6 x 10 halo of
// leaves sits in shared memory; thread (t, row) owns pixel t of the 8 leaves of
// one tile row.
__global__ void __launch_bounds__(256) k_near(const float2 *__restrict__ x, const float2 *__restrict__ g,
                                              int64_t gstride, int mode, const int *__restrict__ active,
                                              const float2 *__restrict__ loc_leaf, size_t mp, int ns,
                                              const float2 *__restrict__ nearW, const float2 *__restrict__ basisT,
                                              float2 *__restrict__ y, int epi, int red,
                                              const float2 *__restrict__ dot_a, double *__restrict__ part, int nleaf,
                                              int U, int tiles_x, int tiles_total) {
  const int rhs = blockIdx.y;
  if (inactive(active, rhs)) return;
  extern __shared__ float2 sm[];
  float2 *hx = sm;                          // [60 leaves][64]
  float2 *ls = sm + kHaloLeaves * kBB;      // [32 leaves][ns]
  const int tile = blockIdx.x;
  const int ty0 = (tile / tiles_x) * kNearTY, tx0 = (tile % tiles_x) * kNearTX;
  const size_t rbase = (size_t)rhs * U;
  const float2 *gr = g ? g + rhs * gstride : nullptr;
  const bool do_near = (epi != EPI_L2P_ONLY);
  if (do_near) {
    for (int e = threadIdx.x; e < kHaloLeaves * kBB; e += blockDim.x) {
      const int h = e / kBB, p = e % kBB;
      const int ly = ty0 - 1 + h / (kNearTX + 2), lx = tx0 - 1 + h % (kNearTX + 2);
      float2 v = make_float2(0.f, 0.f);
      if (ly >= 0 && ly < nleaf && lx >= 0 && lx < nleaf) {
        const size_t i = (size_t)(ly * nleaf + lx) * kBB + p;
        v = load_in(x + rbase, gr, mode, i, i);
      }
      hx[e] = v;
    }
  }
  const float2 *lr = loc_leaf + (size_t)rhs * mp;
  for (int e = threadIdx.x; e < kNearTY * kNearTX * ns; e += blockDim.x) {
    const int j = e / ns, k = e % ns;
    const int ly = ty0 + j / kNearTX, lx = tx0 + j % kNearTX;
    float2 v = make_float2(0.f, 0.f);
    if (ly < nleaf && lx < nleaf) v = lr[(size_t)(ly * nleaf + lx) * ns + k];
    ls[e] = v;
  }
  __syncthreads();

  const int t = threadIdx.x & (kBB - 1), row = threadIdx.x >> 6;
  float2 acc[kNearTX];
#pragma unroll
  for (int j = 0; j < kNearTX; j++) acc[j] = make_float2(0.f, 0.f);
  if (do_near) {
    for (int s = 0; s < 9; s++) {
      const int dr = s / 3 - 1, dc = s % 3 - 1;
      const float2 *W = nearW + s * kBB * kBB + t;
      const float2 *hrow = hx + ((row + 1 + dr) * (kNearTX + 2) + 1 + dc) * kBB;
#pragma unroll 4
      for (int b = 0; b < kBB; b++) {
        const float2 w = __ldg(&W[b * kBB]);
#pragma unroll
        for (int j = 0; j < kNearTX; j++) cfma(acc[j], w, hrow[j * kBB + b]);
      }
    }
  }
  {
    const float2 *lrow = ls + row * kNearTX * ns;
#pragma unroll 4
    for (int k = 0; k < ns; k++) {
      const float2 bv = __ldg(&basisT[k * kBB + t]);
#pragma unroll
      for (int j = 0; j < kNearTX; j++) cfma(acc[j], bv, lrow[j * ns + k]);
    }
  }

  double r0 = 0, r1 = 0, r2 = 0;
  const int ly = ty0 + row;
#pragma unroll
  for (int j = 0; j < kNearTX; j++) {
    const int lx = tx0 + j;
    if (ly >= nleaf || lx >= nleaf) continue;
    const size_t i = (size_t)(ly * nleaf + lx) * kBB + t;
    float2 out = acc[j];
    if (epi == EPI_FWD) {
      out = csub(x[rbase + i], acc[j]);
    } else if (epi == EPI_ADJ) {
      out = csub(x[rbase + i], cconj(cmul(gr[i], acc[j])));
    } else if (epi == EPI_CONJ) {
      out = cconj(acc[j]);
    }
    y[rbase + i] = out;
    if (red == RED_DOT) {
      const float2 a = dot_a[rbase + i];
      r0 += (double)a.x * out.x + (double)a.y * out.y;
      r1 += (double)a.x * out.y - (double)a.y * out.x;
    } else if (red == RED_TS) {
      const float2 s = x[rbase + i];
      r0 += (double)out.x * s.x + (double)out.y * s.y;
      r1 += (double)out.x * s.y - (double)out.y * s.x;
      r2 += (double)out.x * out.x + (double)out.y * out.y;
    }
  }
  if (red != RED_NONE) {
    __shared__ double wsum[8][3];
    r0 = warp_sum(r0);
    r1 = warp_sum(r1);
    r2 = warp_sum(r2);
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
      wsum[w][0] = r0;
      wsum[w][1] = r1;
      wsum[w][2] = r2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double s0 = 0, s1 = 0, s2 = 0;
      for (int q = 0; q < 8; q++) {
        s0 += wsum[q][0];
        s1 += wsum[q][1];
        s2 += wsum[q][2];
      }
      double *p = part + ((size_t)rhs * tiles_total + tile) * 4;
      p[0] = s0;
      p[1] = s1;
      p[2] = s2;
      p[3] = 0;
    }
  }
}

// Receiver interpolation of the root pattern (solve.cpp:330-337).
__global__ void k_rx_interp(const float2 *__restrict__ mul0, size_t mp, float2 *__restrict__ rx, int numrx, int ns0,
                            const int *__restrict__ hfirst, const float *__restrict__ hw, int ninter) {
  const int rhs = blockIdx.y;
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= numrx) return;
  const float2 *src = mul0 + (size_t)rhs * mp;
  float2 acc = make_float2(0.f, 0.f);
  int idx = hfirst[m];
  for (int t = 0; t < ninter; t++) {
    rfma(acc, hw[t * numrx + m], src[idx]);
    if (++idx == ns0) idx = 0;
  }
  rx[(size_t)rhs * numrx + m] = acc;
}

// Receiver anterpolation onto the root local expansion, times
// (-4i) numrx res^2 (solve.cpp:381-387).
__global__ void k_rx_anterp(const float2 *__restrict__ rx, float2 *__restrict__ loc0, size_t mp, int numrx, int ns0,
                            const int *__restrict__ hind, const float *__restrict__ haw, int width, float2 scale) {
  const int rhs = blockIdx.y;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ns0) return;
  const float2 *src = rx + (size_t)rhs * numrx;
  float2 acc = make_float2(0.f, 0.f);
  for (int t = 0; t < width; t++) rfma(acc, haw[(size_t)k * width + t], src[hind[(size_t)k * width + t]]);
  loc0[(size_t)rhs * mp + k] = cmul(acc, scale);
}

__global__ void k_permute(const int *__restrict__ perm, const float2 *__restrict__ in, float2 *__restrict__ out, int U,
                          int gather) {
  const size_t r = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < U; i += gridDim.x * blockDim.x) {
    if (gather)
      out[r * U + i] = in[r * U + perm[i]];
    else
      out[r * U + perm[i]] = in[r * U + i];
  }
}

}  // namespace

void launch_p2m(const DevPlan &P, const BatchArgs &B, float2 *mul, cudaStream_t st) {
  const int nleaves = P.nleaf * P.nleaf;
  dim3 grid((nleaves + 31) / 32, B.nrhs);
  count_launch();
  k_p2m<<<grid, 128, 0, st>>>(B.x, B.g, B.gstride, B.mode, B.active, P.coeffT, P.ns_leaf, nleaves, P.U,
                              mul + P.lv[P.L - 1].off, P.mp);
}

// Parents per block so that the staged rings stay near kStageBudget.
static int parents_per_block(size_t ring_bytes, int nparent) {
  const int npb = (int)std::max<size_t>(1, kStageBudget / std::max<size_t>(1, ring_bytes));
  return std::min(npb, std::max(1, nparent));
}

// Splits each block's outputs over several blocks when the level has too few
// parents to fill the GPU (the top levels, and any level at small batches).
static int output_chunks(int blocks, int nrhs, int npb, int ns_out) {
  const int want = 2 * 148;
  if (npb != 1 || blocks * nrhs >= want) return 1;
  return std::max(1, std::min((ns_out + 127) / 128, (want + blocks * nrhs - 1) / (blocks * nrhs)));
}

void launch_m2m(const DevPlan &P, int lvl, float2 *mul, int nrhs, const int *active, cudaStream_t st) {
  const DevLevel &p = P.lv[lvl], &c = P.lv[lvl + 1];
  const size_t ring = (size_t)4 * c.ns * sizeof(float2);
  const int nparent = p.n * p.n;
  count_launch();
  if (ring <= (size_t)kSmemStage) {
    const int npb = parents_per_block(ring, nparent), blocks = (nparent + npb - 1) / npb;
    const int chunks = output_chunks(blocks, nrhs, npb, p.ns);
    const size_t smem = ring * npb;
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_m2m<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    dim3 grid(blocks * chunks, nrhs);
    k_m2m<true><<<grid, 256, smem, st>>>(mul, P.mp, p.off, c.off, p.n, p.ns, c.ns, npb, chunks, p.ifirst, p.iw,
                                         p.shm, P.ninter, active);
  } else {
    const int chunks = output_chunks(nparent, nrhs, 1, p.ns);
    dim3 grid(nparent * chunks, nrhs);
    k_m2m<false><<<grid, 256, 0, st>>>(mul, P.mp, p.off, c.off, p.n, p.ns, c.ns, 1, chunks, p.ifirst, p.iw, p.shm,
                                       P.ninter, active);
  }
}

void launch_m2l(const DevPlan &P, int lvl, const float2 *mul, float2 *loc, int nrhs, const int *active,
                cudaStream_t st) {
  const DevLevel &c = P.lv[lvl];
  M2lArgs A;
  A.mul = mul;
  A.loc = loc;
  A.mp = P.mp;
  A.off = c.off;
  A.n = c.n;
  A.ns = c.ns;
  A.tiles_x = (c.n + kM2lCols - 1) / kM2lCols;
  A.tiles = A.tiles_x * ((c.n + kM2lRows - 1) / kM2lRows);
  A.nitems = A.tiles * nrhs;
  A.T = c.T;
  A.active = active;
  const int nkc = (c.ns + kM2lKC - 1) / kM2lKC;
  // one resident block per SM: spread the items so every SM has a sample chunk
  const int groups = std::max(1, std::min(A.nitems, (2 * 148 + nkc - 1) / nkc));
  const size_t smem = 2 * (size_t)kM2lHalo * sizeof(float2);
  cudaFuncSetAttribute(k_m2l, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  count_launch();
  k_m2l<<<dim3(nkc, groups), 256, smem, st>>>(A);
}

void launch_l2l(const DevPlan &P, int lvl, float2 *loc, int nrhs, const int *active, bool accumulate,
                cudaStream_t st) {
  const DevLevel &c = P.lv[lvl], &p = P.lv[lvl - 1];
  const size_t ring = (size_t)4 * p.ns * sizeof(float2);
  const int nparent = p.n * p.n;
  count_launch();
  if (ring <= (size_t)kSmemStage) {
    const int npb = parents_per_block(ring, nparent), blocks = (nparent + npb - 1) / npb;
    const int chunks = output_chunks(blocks, nrhs, npb, c.ns);
    const size_t smem = ring * npb;
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_l2l<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    dim3 grid(blocks * chunks, nrhs);
    k_l2l<true><<<grid, 256, smem, st>>>(loc, P.mp, p.off, c.off, p.n, p.ns, c.ns, npb, chunks, c.afirst, c.aw,
                                         c.awidth, p.shl, accumulate ? 1 : 0, active);
  } else {
    const int chunks = output_chunks(nparent, nrhs, 1, c.ns);
    dim3 grid(nparent * chunks, nrhs);
    k_l2l<false><<<grid, 256, 0, st>>>(loc, P.mp, p.off, c.off, p.n, p.ns, c.ns, 1, chunks, c.afirst, c.aw,
                                       c.awidth, p.shl, accumulate ? 1 : 0, active);
  }
}

int near_blocks_per_rhs(const DevPlan &P) {
  const int ty = (P.nleaf + kNearTY - 1) / kNearTY, tx = (P.nleaf + kNearTX - 1) / kNearTX;
  return ty * tx;
}

void launch_near(const DevPlan &P, const NearArgs &A, cudaStream_t st) {
  const int tiles_x = (P.nleaf + kNearTX - 1) / kNearTX;
  const int tiles = near_blocks_per_rhs(P);
  const size_t smem = (size_t)(kHaloLeaves * kBB + kNearTY * kNearTX * P.ns_leaf) * sizeof(float2);
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_near, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  dim3 grid(tiles, A.in.nrhs);
  count_launch();
  k_near<<<grid, 256, smem, st>>>(A.in.x, A.in.g, A.in.gstride, A.in.mode, A.in.active, A.loc + P.lv[P.L - 1].off,
                                  P.mp, P.ns_leaf, P.nearW, P.basisT, A.y, A.epi, A.red, A.dot_a, A.part, P.nleaf,
                                  P.U, tiles_x, tiles);
}

void launch_rx_interp(const DevPlan &P, const float2 *mul, float2 *rx, int nrhs, cudaStream_t st) {
  dim3 grid((P.numrx + 127) / 128, nrhs);
  count_launch();
  k_rx_interp<<<grid, 128, 0, st>>>(mul + P.lv[0].off, P.mp, rx, P.numrx, P.lv[0].ns, P.hfirst, P.hw, P.ninter);
}

void launch_rx_anterp(const DevPlan &P, const float2 *rx, float2 *loc, int nrhs, float2 scale, cudaStream_t st) {
  dim3 grid((P.lv[0].ns + 127) / 128, nrhs);
  count_launch();
  k_rx_anterp<<<grid, 128, 0, st>>>(rx, loc + P.lv[0].off, P.mp, P.numrx, P.lv[0].ns, P.hind, P.haw, P.hwidth, scale);
}

void launch_permute(const int *perm, const float2 *in, float2 *out, int U, int nrhs, bool gather, cudaStream_t st) {
  dim3 grid(std::min((U + 255) / 256, 1184), nrhs);
  count_launch();
  k_permute<<<grid, 256, 0, st>>>(perm, in, out, U, gather ? 1 : 0);
}

}  // namespace isg
