// Complex-FP32 SIMT kernels of the MLFMA matvec (the reference's kernels.cu
// P2M/M2M/M2L/L2L/L2P/P2P stages, re-designed for a batched, RHS-major layout
// and raster cluster numbering).  The tensor-core leaf kernels live in
// isg_tc.cu.
#include <algorithm>
#include <atomic>

#include "isg_device.cuh"

namespace isg {

static std::atomic<int64_t> g_launches{0};
// While this thread captures a CUDA graph its launches are tallied here
// instead; each replay of the graph then counts them again.
static thread_local int64_t *t_capture_sink = nullptr;
void count_launch(int n) {
  if (t_capture_sink)
    *t_capture_sink += n;
  else
    g_launches.fetch_add(n, std::memory_order_relaxed);
}
int64_t launch_count() { return g_launches.load(std::memory_order_relaxed); }
void capture_launches(int64_t *sink) { t_capture_sink = sink; }

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


__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(valid ? 8 : 0));
}
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// M2L (kernels.cu:239-266, solve.cpp:133-148) as a 2-D stencil per sample.
// The far list of a cluster is the 6x6 block of its parent's neighbours'
// children minus its own 3x3 neighbourhood, clipped to the grid, so the four
// siblings of a 2x2 group at rows 2a, 2a+1 all draw on rows 2a-2 .. 2a+3 of
// the same six-column window, each with 27 of the 40 translation weights
// T[(dy+3)*7+dx+3][k] whose offset is not inside the 3x3.  A thread owns one
// sample k of one column of sibling groups: it keeps the 40 weights in
// registers and slides the window down `ty` groups, two new rows per step.
// The window lives in a private ring of kM2lRing row slots in shared memory
// (slot-major, thread-minor, so every access is conflict-free), filled by
// 8-byte cp.async copies kM2lAhead steps ahead of the step being computed,
// one commit group per step.  Each thread waits only for its own copies
// (cp.async.wait_group), so there is no block barrier, and the loads in
// flight hold no registers (one column per thread: 157 registers, three blocks
// and 12 warps per SM; two columns: 204 registers, two blocks).
// Rows outside the grid are the same for the whole block and copy as zeros; a
// column outside the grid copies zeros by a zero source size.  Consecutive
// threads take consecutive samples, so every load and store is coalesced.
struct M2lArgs {
  const float2 *mul;
  float2 *loc;
  size_t mp, off;
  int n, ns, ty;
  const float2 *T;
  const int *active;
  const float2 *zeros;  // at least ns zeros
  unsigned *locmax;     // optional [R][kMaxLevels]: max |re|, |im| of the level's locals (FP32 bits)
  int lvl;
};

constexpr int kM2lAhead = 2;                 // steps of window rows in flight ahead of the computing step
constexpr int kM2lRing = 6 + 2 * kM2lAhead;  // row slots per thread
constexpr int kM2lThreads = 128;
// window columns per ring row for NC sibling-group columns per thread (6 or 8)
__host__ __device__ constexpr int m2l_cols(int nc) { return 4 + 2 * nc; }
__host__ __device__ constexpr size_t m2l_smem(int nc) {  // 60 KB (NC = 1), 80 KB (NC = 2)
  return (size_t)kM2lRing * m2l_cols(nc) * kM2lThreads * sizeof(float2);
}

__device__ __forceinline__ void cp_async8z(void *smem, const void *gmem, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(valid ? 8 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// NC sibling-group columns per thread: groups 2 bp .. 2 bp + NC - 1 of the
// thread's column pair bp read window columns 2 b0 - 2 .. 2 b0 + 2 NC + 1
// (b0 = NC bp), so with NC = 2 one 6 x 8 window feeds 8 outputs (216 complex
// FMAs) where two NC = 1 threads read 6 x 6 windows each: a third fewer ring
// loads and cp.async issues per FMA, at 8 instead of 12 warps per SM.
// Each complex multiply-add is two packed FP32 pair FMAs (fma.rn.f32x2) on
// two accumulators per output, one for the window value's real part and one
// for its imaginary part, combined once per step: half the FMA instructions
// of the scalar form, with the weights kept as their natural (re, im) pairs.
template <bool ACC, int NC>
__global__ void __launch_bounds__(kM2lThreads, NC == 1 ? 3 : 2) k_m2l(M2lArgs A) {
  constexpr int NW = m2l_cols(NC);
  extern __shared__ __align__(16) float2 m2l_ring[];  // [kM2lRing][NW][kM2lThreads]
  const int rhs = blockIdx.z;
  if (A.active && !A.active[rhs]) return;
  const int half = A.n >> 1, ns = A.ns, ncp = half / NC;
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= ncp * ns) return;  // no block barrier below
  const int bp = f / ns, k = f - bp * ns, b0 = NC * bp;
  const int a0 = blockIdx.y * A.ty, a1 = min(a0 + A.ty, half);
  f32x2 tw[7][7];  // (re, im) of each translation weight as one packed pair
#pragma unroll
  for (int dy = 0; dy < 7; dy++)
#pragma unroll
    for (int dx = 0; dx < 7; dx++)
      tw[dy][dx] = (dy >= 2 && dy <= 4 && dx >= 2 && dx <= 4)
                       ? 0ull
                       : __ldg((const unsigned long long *)&A.T[(dy * 7 + dx) * ns + k]);
  const float2 *m = A.mul + (size_t)rhs * A.mp + A.off + k;
  float2 *out = A.loc + (size_t)rhs * A.mp + A.off + k;
  const size_t row_stride = (size_t)A.n * ns;
  // the window columns 2 b0 - 2 .. 2 b0 + NW - 3: element offsets within a row, and which are inside the grid
  int coff[NW];
  unsigned cin = 0;
#pragma unroll
  for (int j = 0; j < NW; j++) {
    const int col = 2 * b0 - 2 + j;
    const bool ok = col >= 0 && col < A.n;
    coff[j] = ok ? col * ns : 0;
    cin |= ok ? 1u << j : 0u;
  }
  float2 *ring = m2l_ring + threadIdx.x;
  const int r0 = 2 * a0 - 2;  // window row of slot 0
  auto issue_row = [&](int r) {
    const bool rok = r >= 0 && r < A.n;  // the same for the whole block
    float2 *dst = ring + (size_t)((r - r0) % kM2lRing) * NW * kM2lThreads;
    const float2 *src = m + (rok ? (size_t)r * row_stride : 0);
#pragma unroll
    for (int j = 0; j < NW; j++) cp_async8z(dst + j * kM2lThreads, src + coff[j], rok && ((cin >> j) & 1));
  };
  // groups: the first step's six rows, then two rows per step
  for (int i = 0; i < 6; i++) issue_row(r0 + i);
  cp_async_commit();
#pragma unroll
  for (int s = 1; s < kM2lAhead; s++) {
    if (a0 + s < a1) {
      issue_row(2 * (a0 + s) + 2);
      issue_row(2 * (a0 + s) + 3);
    }
    cp_async_commit();
  }
  float2 ob[NC][2][2];
  auto old = [&](int a, float2(&dst)[NC][2][2]) {
#pragma unroll
    for (int gx = 0; gx < NC; gx++)
#pragma unroll
      for (int oy = 0; oy < 2; oy++)
#pragma unroll
        for (int ox = 0; ox < 2; ox++)
          dst[gx][oy][ox] = ACC ? out[(size_t)(2 * a + oy) * row_stride + (size_t)(2 * (b0 + gx) + ox) * ns]
                                : make_float2(0.f, 0.f);
  };
  old(a0, ob);
  float mx = 0.f;
#pragma unroll 1
  for (int a = a0; a < a1; a++) {
    if (a + kM2lAhead < a1) {
      issue_row(2 * (a + kM2lAhead) + 2);
      issue_row(2 * (a + kM2lAhead) + 3);
    }
    cp_async_commit();
    // complex products on packed pairs: ax += (w.x, w.x) * (t.x, t.y) and
    // ay += (w.y, w.y) * (t.x, t.y), so that t w = (ax.x - ay.y, ax.y + ay.x)
    f32x2 ax[NC][2][2], ay[NC][2][2];
#pragma unroll
    for (int gx = 0; gx < NC; gx++)
#pragma unroll
      for (int oy = 0; oy < 2; oy++)
#pragma unroll
        for (int ox = 0; ox < 2; ox++) {
          ax[gx][oy][ox] = pk2(ob[gx][oy][ox].x, ob[gx][oy][ox].y);
          ay[gx][oy][ox] = 0ull;
        }
    if (a + 1 < a1) old(a + 1, ob);  // the next step's old locals, in flight during this one
    cp_async_wait_group<kM2lAhead>();  // this step's rows have landed
#pragma unroll
    for (int i = 0; i < 6; i++) {
      const float2 *src = ring + (size_t)((2 * a - 2 + i - r0) % kM2lRing) * NW * kM2lThreads;
#pragma unroll
      for (int j = 0; j < NW; j++) {
        const float2 w = src[j * kM2lThreads];
        const f32x2 wx = pk2(w.x, w.x), wy = pk2(w.y, w.y);
#pragma unroll
        for (int gx = 0; gx < NC; gx++) {
          const int jj = j - 2 * gx;
          if (jj < 0 || jj >= 6) continue;
#pragma unroll
          for (int oy = 0; oy < 2; oy++)
#pragma unroll
            for (int ox = 0; ox < 2; ox++) {
              const int dy = i - 2 - oy, dx = jj - 2 - ox;  // source minus target
              if (dy >= -1 && dy <= 1 && dx >= -1 && dx <= 1) continue;
              ax[gx][oy][ox] = fma2(wx, tw[dy + 3][dx + 3], ax[gx][oy][ox]);
              ay[gx][oy][ox] = fma2(wy, tw[dy + 3][dx + 3], ay[gx][oy][ox]);
            }
        }
      }
    }
#pragma unroll
    for (int gx = 0; gx < NC; gx++)
#pragma unroll
      for (int oy = 0; oy < 2; oy++)
#pragma unroll
        for (int ox = 0; ox < 2; ox++) {
          const float2 px = upk2(ax[gx][oy][ox]), py = upk2(ay[gx][oy][ox]);
          const float2 r = make_float2(px.x - py.y, px.y + py.x);
          out[(size_t)(2 * a + oy) * row_stride + (size_t)(2 * (b0 + gx) + ox) * ns] = r;
          mx = fmaxf(mx, fmaxf(fabsf(r.x), fabsf(r.y)));
        }
  }
  cp_async_wait_group<0>();
  if (A.locmax) {  // the level's maximum, for the power-of-two scale of the tensor-core L2L below it
    const unsigned mm = __activemask(), bits = __reduce_max_sync(mm, __float_as_uint(mx));
    if ((threadIdx.x & 31) == __ffs(mm) - 1 && bits) atomicMax(&A.locmax[rhs * kMaxLevels + A.lvl], bits);
  }
}

// Tiled M2M / L2L.  A column is one (RHS, parent) pair.  A block takes `cols`
// columns and one tile of tb.out output samples; tb.out / kTileOut threads per
// column each accumulate kTileOut of them.  The block stages the tile's input
// window of every ring it reads in shared memory ([window sample][ring],
// padded against bank conflicts) with cp.async, after one thread per ring has
// worked out the ring's address.  Each thread then walks the window once with
// its kTileOut x 4 accumulators live: the band weights (and the L2L shift
// phases) are the same for every thread of the block, so each staged value
// feeds 32 (M2M) or 36 (L2L) FMAs from registers.  Outputs go back through
// shared memory so that every ring is written in runs of tb.out samples.
struct TileArgs {
  const float2 *src;
  float2 *dst;
  size_t mp, off_in, off_out;
  int n_p, ns_in, ns_out, nparent, ncols, cols;
  TileBand tb;
  const float2 *shT;  // [ns][4]: L2L shiftloc of the parent level, M2M shiftmul of the parent level
  const int *active;
};

// Shared-memory carve-up of one tiled block (float2 units, 16-byte aligned parts).
// With dup, the weights are stored as (w, w) pairs and each shift phase s as
// (s.x, s.x, -s.y, s.y), the operands of packed FP32 pair arithmetic.
struct TileSmem {
  size_t win, w, sh, src, dst, total;
  __host__ __device__ TileSmem(int wmax, int ld, int out, int nsrc, int ndst, size_t out_tile, bool dup = false) {
    auto up2 = [](size_t x) { return (x + 1) & ~(size_t)1; };
    win = 0;
    w = up2(((size_t)wmax * ld > out_tile ? (size_t)wmax * ld : out_tile));
    sh = w + up2((size_t)wmax * out / (dup ? 1 : 2));
    src = sh + (size_t)wmax * (dup ? 8 : 4);
    dst = src + nsrc;
    total = dst + ndst;
  }
};

__device__ __forceinline__ const float2 *ring_ptr(const TileArgs &A, const float2 *base, size_t off, int gc, int q,
                                                  int level_n, int ns) {
  if (gc >= A.ncols) return nullptr;
  const int rhs = gc / A.nparent, P = gc - rhs * A.nparent;
  if (inactive(A.active, rhs)) return nullptr;
  size_t cl = P;
  if (q >= 0) {
    const int py = P / A.n_p, px = P - py * A.n_p;
    cl = (size_t)(2 * py + (q >> 1)) * level_n + 2 * px + (q & 1);
  }
  return base + (size_t)rhs * A.mp + off + cl * ns;
}

// Whether some column c0 .. c0 + cols - 1 of a tiled block exists and belongs
// to an active RHS; the same answer in every thread of the block (block size
// >= cols).  A block without one returns before it loads anything: in the last
// iterations of a batch most RHS have converged, and their columns would
// otherwise still be staged and multiplied as zeros.
__device__ __forceinline__ bool any_active_column(const TileArgs &A, int c0) {
  const int gc = c0 + (int)threadIdx.x;
  return __syncthreads_or(threadIdx.x < (unsigned)A.cols && gc < A.ncols && !inactive(A.active, gc / A.nparent));
}

// L2L into the children of each column's parent: z = parent local, four
// shifted copies shl[q][j] z[j], anterpolated by the tile's band weights and
// written over the children's locals.
__global__ void __launch_bounds__(128) k_l2l_tile(TileArgs A) {
  extern __shared__ float2 sm[];
  const int cols = A.cols, TO = A.tb.out, tile = blockIdx.y, c0 = blockIdx.x * cols;
  if (!any_active_column(A, c0)) return;
  const int a0 = A.tb.a0[tile], wl = A.tb.wl[tile], ld = cols + 1;
  const TileSmem L(A.tb.wmax, ld, TO, cols, 4 * cols, (size_t)4 * TO * ld, true);
  const float2 **sp = (const float2 **)(sm + L.src);
  float2 **dp = (float2 **)(sm + L.dst);
  float4 *sw = (float4 *)(sm + L.w);   // [wl][TO / 2]: (w, w, w', w') pairs
  float4 *ss = (float4 *)(sm + L.sh);  // [wl][4]: (s.x, s.x, -s.y, s.y) per child
  for (int t = threadIdx.x; t < 4 * cols; t += blockDim.x) {
    if (t < cols) sp[t] = ring_ptr(A, A.src, A.off_in, c0 + t, -1, A.n_p, A.ns_in);
    dp[t] = (float2 *)ring_ptr(A, A.dst, A.off_out, c0 + (t >> 2), t & 3, 2 * A.n_p, A.ns_out);
  }
  {
    const float4 *wt = (const float4 *)(A.tb.w + (size_t)tile * A.tb.wmax * TO);
    for (int e = threadIdx.x; e < wl * TO / 4; e += blockDim.x) {
      const float4 w = __ldg(wt + e);
      sw[2 * e] = make_float4(w.x, w.x, w.y, w.y);
      sw[2 * e + 1] = make_float4(w.z, w.z, w.w, w.w);
    }
    for (int e = threadIdx.x; e < 4 * wl; e += blockDim.x) {
      int j = a0 + (e >> 2);
      if (j >= A.ns_in) j -= A.ns_in;
      const float2 v = __ldg(A.shT + 4 * j + (e & 3));
      ss[e] = make_float4(v.x, v.x, -v.y, v.y);
    }
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int r = warp; r < cols; r += nw) {
    const float2 *ring = sp[r];
    for (int jj = lane; jj < wl; jj += 32) {
      int j = a0 + jj;
      if (j >= A.ns_in) j -= A.ns_in;
      cp_async8(&sm[jj * ld + r], ring ? ring + j : A.src, ring != nullptr);
    }
  }
  cp_async_wait_all();
  __syncthreads();
  const int col = threadIdx.x % cols, sub = threadIdx.x / cols;
  f32x2 acc[kTileOut][4];
#pragma unroll
  for (int i = 0; i < kTileOut; i++)
#pragma unroll
    for (int q = 0; q < 4; q++) acc[i][q] = 0ull;
  const int wstep = TO / 2;
  const int2 span = A.tb.span[tile * (TO / kTileOut) + sub];
#pragma unroll 2
  for (int jj = span.x; jj < span.y; jj++) {
    const float2 z = sm[jj * ld + col];
    const f32x2 zz = pk2(z.x, z.y), zs = pk2(z.y, z.x);
    f32x2 v[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {  // shl[q] z as packed pairs
      const float4 sq = ss[4 * jj + q];
      v[q] = fma2(pk2(sq.z, sq.w), zs, mul2(pk2(sq.x, sq.y), zz));
    }
#pragma unroll
    for (int i2 = 0; i2 < kTileOut / 2; i2++) {
      const float4 w = sw[jj * wstep + sub * (kTileOut / 2) + i2];
      const f32x2 wa = pk2(w.x, w.y), wb = pk2(w.z, w.w);
#pragma unroll
      for (int q = 0; q < 4; q++) {
        acc[2 * i2][q] = fma2(wa, v[q], acc[2 * i2][q]);
        acc[2 * i2 + 1][q] = fma2(wb, v[q], acc[2 * i2 + 1][q]);
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 4; q++)
#pragma unroll
    for (int i = 0; i < kTileOut; i++) sm[(q * TO + sub * kTileOut + i) * ld + col] = upk2(acc[i][q]);
  __syncthreads();
  for (int e = threadIdx.x; e < cols * 4 * TO; e += blockDim.x) {
    const int i = e % TO, cq = e / TO, km = tile * TO + i;
    float2 *d = dp[cq];
    if (d && km < A.ns_out) d[km] = sm[((cq & 3) * TO + i) * ld + (cq >> 2)];
  }
}

// M2M into each column's parent: the four children's rings interpolated by the
// tile's band weights, then shifted by shm[q][k] and summed.
__global__ void __launch_bounds__(128) k_m2m_tile(TileArgs A) {
  extern __shared__ float2 sm[];
  const int cols = A.cols, TO = A.tb.out, tile = blockIdx.y, c0 = blockIdx.x * cols;
  if (!any_active_column(A, c0)) return;
  const int a0 = A.tb.a0[tile], wl = A.tb.wl[tile], ld = 4 * cols + 1;
  const TileSmem L(A.tb.wmax, ld, TO, 4 * cols, cols, (size_t)TO * (cols + 1));
  const float2 **sp = (const float2 **)(sm + L.src);
  float2 **dp = (float2 **)(sm + L.dst);
  float4 *sw = (float4 *)(sm + L.w);
  const int n_c = 2 * A.n_p;
  for (int t = threadIdx.x; t < 4 * cols; t += blockDim.x) {
    sp[t] = ring_ptr(A, A.src, A.off_in, c0 + (t >> 2), t & 3, n_c, A.ns_in);
    if (t < cols) dp[t] = (float2 *)ring_ptr(A, A.dst, A.off_out, c0 + t, -1, A.n_p, A.ns_out);
  }
  {
    const float4 *wt = (const float4 *)(A.tb.w + (size_t)tile * A.tb.wmax * TO);
    for (int e = threadIdx.x; e < wl * TO / 4; e += blockDim.x) cp_async16(sw + e, wt + e);
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int r = warp; r < 4 * cols; r += nw) {
    const float2 *ring = sp[r];
    float2 *dst = sm + (r & 3) * cols + (r >> 2);
    for (int jj = lane; jj < wl; jj += 32) {
      int j = a0 + jj;
      if (j >= A.ns_in) j -= A.ns_in;
      cp_async8(dst + jj * ld, ring ? ring + j : A.src, ring != nullptr);
    }
  }
  cp_async_wait_all();
  __syncthreads();
  const int col = threadIdx.x % cols, sub = threadIdx.x / cols;
  float2 acc[kTileOut][4] = {};
  const int wstep = TO / 4;
  const int2 span = A.tb.span[tile * (TO / kTileOut) + sub];
#pragma unroll 2
  for (int jj = span.x; jj < span.y; jj++) {
    float2 v[4];
#pragma unroll
    for (int q = 0; q < 4; q++) v[q] = sm[jj * ld + q * cols + col];
    const float4 w0 = sw[jj * wstep + 2 * sub], w1 = sw[jj * wstep + 2 * sub + 1];
    const float wv[kTileOut] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
#pragma unroll
    for (int i = 0; i < kTileOut; i++)
#pragma unroll
      for (int q = 0; q < 4; q++) rfma(acc[i][q], wv[i], v[q]);
  }
  const float4 *sh = (const float4 *)A.shT;
  float2 res[kTileOut];
#pragma unroll
  for (int i = 0; i < kTileOut; i++) {
    const int k = min(tile * TO + sub * kTileOut + i, A.ns_out - 1);
    const float4 s01 = __ldg(sh + 2 * k), s23 = __ldg(sh + 2 * k + 1);
    res[i] = make_float2(0.f, 0.f);
    cfma(res[i], make_float2(s01.x, s01.y), acc[i][0]);
    cfma(res[i], make_float2(s01.z, s01.w), acc[i][1]);
    cfma(res[i], make_float2(s23.x, s23.y), acc[i][2]);
    cfma(res[i], make_float2(s23.z, s23.w), acc[i][3]);
  }
  __syncthreads();
  const int ldo = cols + 1;
#pragma unroll
  for (int i = 0; i < kTileOut; i++) sm[(sub * kTileOut + i) * ldo + col] = res[i];
  __syncthreads();
  for (int e = threadIdx.x; e < cols * TO; e += blockDim.x) {
    const int i = e % TO, cl = e / TO, kp = tile * TO + i;
    float2 *d = dp[cl];
    if (d && kp < A.ns_out) d[kp] = sm[i * ldo + cl];
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

static TileArgs tile_args(const float2 *src, float2 *dst, size_t mp, size_t off_in, size_t off_out, int n_p,
                          int ns_in, int ns_out, int nrhs, const TileBand &tb, const float2 *shT, int cap,
                          const int *active) {
  TileArgs A;
  A.src = src;
  A.dst = dst;
  A.mp = mp;
  A.off_in = off_in;
  A.off_out = off_out;
  A.n_p = n_p;
  A.ns_in = ns_in;
  A.ns_out = ns_out;
  A.nparent = n_p * n_p;
  A.ncols = A.nparent * nrhs;
  A.cols = std::min(cap, std::max(32, (A.ncols + 31) / 32 * 32));
  A.tb = tb;
  A.shT = shT;
  A.active = active;
  return A;
}

void launch_m2m(const DevPlan &P, int lvl, float2 *mul, int nrhs, const int *active, cudaStream_t st) {
  const DevLevel &p = P.lv[lvl], &c = P.lv[lvl + 1];
  const int cap = (p.m2m_cols > 0 && 4 * nrhs >= P.tuned_nrhs) ? p.m2m_cols : 32;
  const TileArgs A = tile_args(mul, mul, P.mp, c.off, p.off, p.n, c.ns, p.ns, nrhs, p.mt, p.shmT, cap, active);
  const TileSmem L(p.mt.wmax, 4 * A.cols + 1, p.mt.out, 4 * A.cols, A.cols, (size_t)p.mt.out * (A.cols + 1));
  const size_t smem = L.total * sizeof(float2);
  count_launch();
  k_m2m_tile<<<dim3((A.ncols + A.cols - 1) / A.cols, p.mt.tiles), A.cols * (p.mt.out / kTileOut), smem, st>>>(A);
}

void launch_m2l(const DevPlan &P, int lvl, const float2 *mul, float2 *loc, int nrhs, const int *active, bool accumulate,
                cudaStream_t st,
                unsigned *locmax) {
  const DevLevel &c = P.lv[lvl];
  M2lArgs A;
  A.mul = mul;
  A.loc = loc;
  A.mp = P.mp;
  A.off = c.off;
  A.n = c.n;
  A.ns = c.ns;
  A.T = c.T;
  A.active = active;
  A.zeros = P.zeros;
  A.locmax = locmax;
  A.lvl = lvl;
  // two sibling-group columns per thread where the level has at least four
  const int half = c.n / 2, nc = half >= 4 ? 2 : 1, bx = (half / nc * c.ns + 127) / 128;
  // eight groups per thread when the grid stays large, fewer for small batches
  int ty = std::min(8, half);
  while (ty > 1 && (size_t)bx * ((half + ty - 1) / ty) * nrhs < 4 * 148) ty /= 2;
  if (c.m2l_ty > 0 && 4 * nrhs >= P.tuned_nrhs) ty = std::min(c.m2l_ty, std::max(1, half));
  A.ty = ty;
  count_launch();
  const dim3 grid(bx, (half + ty - 1) / ty, nrhs);
  if (nc == 2) {
    if (accumulate)
      k_m2l<true, 2><<<grid, kM2lThreads, m2l_smem(2), st>>>(A);
    else
      k_m2l<false, 2><<<grid, kM2lThreads, m2l_smem(2), st>>>(A);
  } else {
    if (accumulate)
      k_m2l<true, 1><<<grid, kM2lThreads, m2l_smem(1), st>>>(A);
    else
      k_m2l<false, 1><<<grid, kM2lThreads, m2l_smem(1), st>>>(A);
  }
}

void launch_l2l(const DevPlan &P, int lvl, float2 *loc, int nrhs, const int *active, cudaStream_t st) {
  const DevLevel &c = P.lv[lvl], &p = P.lv[lvl - 1];
  const int cap = (c.l2l_cols > 0 && 4 * nrhs >= P.tuned_nrhs) ? c.l2l_cols : 64;
  const TileArgs A = tile_args(loc, loc, P.mp, p.off, c.off, p.n, p.ns, c.ns, nrhs, c.at, p.shlT, cap, active);
  const TileSmem L(c.at.wmax, A.cols + 1, c.at.out, A.cols, 4 * A.cols, (size_t)4 * c.at.out * (A.cols + 1), true);
  const size_t smem = L.total * sizeof(float2);
  count_launch();
  k_l2l_tile<<<dim3((A.ncols + A.cols - 1) / A.cols, c.at.tiles), A.cols * (c.at.out / kTileOut), smem, st>>>(A);
}

int near_blocks_per_rhs(const DevPlan &P) {
  const int ty = (P.nleaf + kNearTY - 1) / kNearTY, tx = (P.nleaf + kNearTX - 1) / kNearTX;
  return ty * tx;
}

void launch_near(const DevPlan &P, const NearArgs &A, cudaStream_t st) {
  const int tiles_x = (P.nleaf + kNearTX - 1) / kNearTX;
  const int tiles = near_blocks_per_rhs(P);
  const size_t smem = (size_t)(kHaloLeaves * kBB + kNearTY * kNearTX * P.ns_leaf) * sizeof(float2);
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

namespace isg {
// Opt-in shared memory for the kernels whose size depends on the level, set
// once per device so that no launch (and no graph capture) needs it.
template <class K>
static cudaError_t allow_max_smem(K kernel, int optin) {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, kernel);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
}

cudaError_t kernels_setup() {
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e == cudaSuccess) e = allow_max_smem(k_m2m_tile, optin);
  if (e == cudaSuccess) e = allow_max_smem(k_l2l_tile, optin);
  if (e == cudaSuccess) e = allow_max_smem(k_near, optin);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_m2l<true, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)m2l_smem(1));
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_m2l<false, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)m2l_smem(1));
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_m2l<true, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)m2l_smem(2));
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_m2l<false, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)m2l_smem(2));
  return e;
}

cudaError_t aggregate_kernels_load() {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, k_permute);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_p2m);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_m2m_tile);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_rx_interp);
  return e;
}
}  // namespace isg
