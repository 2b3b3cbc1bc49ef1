// Complex-FP32 SIMT kernels of the MLFMA matvec (the reference's kernels.cu
// P2M/M2M/M2L/L2L/L2P/P2P stages, re-designed for a batched, RHS-major layout
// and raster cluster numbering).  The tensor-core leaf kernels live in
// isg_tc.cu.
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

// M2M (kernels.cu:83-136, solve.cpp:93-112): parent sample km gathers the
// 30-tap interpolation of each child, shifts it to the parent centre and sums.
__global__ void __launch_bounds__(128) k_m2m(float2 *__restrict__ mul, size_t mp, size_t off_p, size_t off_c, int n_p,
                                             int ns_p, int ns_c, const int *__restrict__ ifirst,
                                             const float *__restrict__ iw, const float2 *__restrict__ shm,
                                             int ninter, const int *__restrict__ active) {
  const int rhs = blockIdx.z;
  if (inactive(active, rhs)) return;
  const int km = blockIdx.x * blockDim.x + threadIdx.x;
  if (km >= ns_p) return;
  const int pc = blockIdx.y, py = pc / n_p, px = pc % n_p, n_c = 2 * n_p;
  const float2 *base = mul + (size_t)rhs * mp + off_c;
  const int f = ifirst[km];
  float2 res = make_float2(0.f, 0.f);
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const float2 *ch = base + (size_t)((2 * py + (q >> 1)) * n_c + 2 * px + (q & 1)) * ns_c;
    float2 acc = make_float2(0.f, 0.f);
    int idx = f;
    for (int t = 0; t < ninter; t++) {
      rfma(acc, __ldg(&iw[t * ns_p + km]), ch[idx]);
      if (++idx == ns_c) idx = 0;
    }
    cfma(res, __ldg(&shm[q * ns_p + km]), acc);
  }
  mul[(size_t)rhs * mp + off_p + (size_t)pc * ns_p + km] = res;
}

// M2L (kernels.cu:239-266, solve.cpp:133-148) fused with L2L from the parent
// level (kernels.cu:137-238, solve.cpp:149-169).  The far list of a cluster is
// the 6x6 block of its parent's neighbours' children minus its own 3x3
// neighbourhood, clipped to the grid; T is indexed by the source offset.
__global__ void __launch_bounds__(128) k_m2l_l2l(const float2 *__restrict__ mul, float2 *__restrict__ loc, size_t mp,
                                                 size_t off_c, size_t off_p, int n, int ns, int ns_p,
                                                 const float2 *__restrict__ T, const int *__restrict__ afirst,
                                                 const float *__restrict__ aw, int awidth,
                                                 const float2 *__restrict__ shl_p, int do_m2l, int do_l2l,
                                                 const int *__restrict__ active) {
  const int rhs = blockIdx.z;
  if (inactive(active, rhs)) return;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ns) return;
  const int c = blockIdx.y, cy = c / n, cx = c % n;
  float2 acc = make_float2(0.f, 0.f);
  if (do_m2l) {
    const float2 *m = mul + (size_t)rhs * mp + off_c;
    const int oy = cy & 1, ox = cx & 1;
    for (int dy = -2 - oy; dy <= 3 - oy; dy++) {
      const int yy = cy + dy;
      if (yy < 0 || yy >= n) continue;
      for (int dx = -2 - ox; dx <= 3 - ox; dx++) {
        const int xx = cx + dx;
        if (xx < 0 || xx >= n) continue;
        if (dy >= -1 && dy <= 1 && dx >= -1 && dx <= 1) continue;
        cfma(acc, __ldg(&T[((dy + 3) * 7 + dx + 3) * ns + k]), m[(size_t)(yy * n + xx) * ns + k]);
      }
    }
  }
  if (do_l2l) {
    const int np = n >> 1;
    const float2 *lp = loc + (size_t)rhs * mp + off_p + (size_t)((cy >> 1) * np + (cx >> 1)) * ns_p;
    const float2 *sh = shl_p + ((cy & 1) * 2 + (cx & 1)) * ns_p;
    int idx = afirst[k];
    float2 a2 = make_float2(0.f, 0.f);
    for (int t = 0; t < awidth; t++) {
      rfma(a2, __ldg(&aw[t * ns + k]), cmul(__ldg(&sh[idx]), lp[idx]));
      if (++idx == ns_p) idx = 0;
    }
    acc = cadd(acc, a2);
  }
  loc[(size_t)rhs * mp + off_c + (size_t)c * ns + k] = acc;
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

void launch_m2m(const DevPlan &P, int lvl, float2 *mul, int nrhs, const int *active, cudaStream_t st) {
  const DevLevel &p = P.lv[lvl], &c = P.lv[lvl + 1];
  dim3 grid((p.ns + 127) / 128, p.n * p.n, nrhs);
  count_launch();
  k_m2m<<<grid, 128, 0, st>>>(mul, P.mp, p.off, c.off, p.n, p.ns, c.ns, p.ifirst, p.iw, p.shm, P.ninter, active);
}

void launch_m2l_l2l(const DevPlan &P, int lvl, const float2 *mul, float2 *loc, int nrhs, const int *active,
                    bool do_m2l, bool do_l2l, cudaStream_t st) {
  const DevLevel &c = P.lv[lvl];
  const DevLevel *p = lvl > 0 ? &P.lv[lvl - 1] : nullptr;
  dim3 grid((c.ns + 127) / 128, c.n * c.n, nrhs);
  count_launch();
  k_m2l_l2l<<<grid, 128, 0, st>>>(mul, loc, P.mp, c.off, p ? p->off : 0, c.n, c.ns, p ? p->ns : 1, c.T, c.afirst,
                                  c.aw, c.awidth, p ? p->shl : nullptr, do_m2l ? 1 : 0, (do_l2l && p) ? 1 : 0,
                                  active);
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
