// Learned warm start: a Fourier neural operator on the pixel grid that maps a
// contrast g and an incident field b to an estimate of the total field u of
// (I - G diag(g)) u = b.  It has no counterpart in the reference (whose solves
// start from zero); BiCGSTAB still runs to the same true residual from it.
//
// Network, per sample (raster order, P = N x N pixels, width C, L layers,
// M x 2M retained Fourier modes):
//   s1  = G (g b)                  first Born scattered field (one MLFMA matvec)
//   in  = [chi, b, chi b, s1, chi s1] as (Re, Im) pairs          (chi = g / k0^2)
//   v0  = Wl in + bl                                            (10 -> C, per pixel)
//   h_l = W_l v_l + bw_l + S_l(v_l),  v_{l+1} = GELU(h_l)          (last layer: no GELU)
//   S_l(v) = Re iDFT_x iDFT_y [ R_l(k) . DFT_y DFT_x v ]   (kx < M, ky in [0,M) u [N-M,N))
//   u0  = b + (Wp v_L + Ws in + bp)                             (C + 10 -> 2, per pixel)
// The truncated transforms are dense products with cos/sin tables, so every
// stage is an FP32 GEMM (k_gemm), a small complex contraction along y
// (k_fy_*), a per-mode channel mix (k_mix_*) or an elementwise kernel.  The
// backward pass applies the exact transposes of the same real-linear maps;
// Adam updates the FP32 parameters.  Everything runs in this file's kernels.
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "isg_context.hpp"
#include "isg_tc.cuh"

namespace isg {

constexpr int kFnoIn = 10;  // input channels

struct FnoModel {
  int C = 32, M = 12, L = 4, S = 4, KY = 24, NM = 288, N = 0, P = 0;
  size_t nparam = 0, off_Wl = 0, off_bl = 0, off_Wp = 0, off_Ws = 0, off_bp = 0;
  std::vector<size_t> off_R, off_W, off_bw;
  float *param = nullptr, *grad = nullptr, *am = nullptr, *av = nullptr;
  int adam_t = 0;
  bool tensor = true;  // products as BF16 tcgen05 MMAs (FP32 accumulation); false: FP32 k_gemm
  int *err = nullptr;  // wait-limit flag of the tensor-core GEMM
  float *Ex = nullptr, *Ix = nullptr;  // [N][2M], [2M][N]
  float2 *Fy = nullptr;                // [KY][N]
  float *in = nullptr, *spec = nullptr, *out = nullptr, *dout = nullptr, *dva = nullptr, *dvb = nullptr;
  std::vector<float *> v, h;  // v[0..L], h[0..L-1]
  float *T = nullptr, *Z = nullptr;  // [S C N][2M]
  std::vector<float2 *> X;           // [L][S][C][NM]
  float2 *Y = nullptr;               // [S][C][NM]
  float2 *gr = nullptr, *br = nullptr, *ur = nullptr, *xr = nullptr;  // raster complex [S][P]
  float2 *gb = nullptr, *bb = nullptr, *xb = nullptr, *yb = nullptr;  // blocked complex [S][P]
  float2 *sr = nullptr;                                               // raster Born field [S][P]
  double *red = nullptr;             // per-sample sums [S][2] + loss
  std::vector<void *> allocs;
  ~FnoModel() {
    for (void *p : allocs) cudaFree(p);
  }
  template <class T_>
  cudaError_t alloc(T_ **p, size_t n) {
    cudaError_t e = cudaMalloc((void **)p, std::max<size_t>(1, n) * sizeof(T_));
    if (e == cudaSuccess) allocs.push_back(*p);
    return e;
  }
};

namespace {

// ---------------- batched strided FP32 GEMM ----------------
// C[b][m][n] (=, +=, or atomically +=) alpha * sum_k A[b][m][k] B[b][k][n]
struct GemmArgs {
  const float *A, *B;
  float *C;
  int M, N, K, ksplit, mode;  // mode 0: store, 1: add, 2: atomic add
  long long sAm, sAk, sBk, sBn, sCm, sCn, bA, bB, bC;
  float alpha;
};
constexpr int kGT = 64, kGK = 16;

__global__ void __launch_bounds__(256) k_gemm(GemmArgs g) {
  __shared__ float As[kGK][kGT + 4];
  __shared__ float Bs[kGK][kGT + 4];
  const int batch = blockIdx.z / g.ksplit, ks = blockIdx.z % g.ksplit;
  const float *A = g.A + batch * g.bA, *B = g.B + batch * g.bB;
  float *C = g.C + batch * g.bC;
  const int m0 = blockIdx.y * kGT, n0 = blockIdx.x * kGT;
  const int kper = ((g.K + g.ksplit - 1) / g.ksplit + kGK - 1) / kGK * kGK;
  const int kbeg = ks * kper, kend = min(g.K, kbeg + kper);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  float acc[4][4] = {};
  for (int k0 = kbeg; k0 < kend; k0 += kGK) {
    for (int e = threadIdx.x; e < kGT * kGK; e += 256) {
      int mm, kk;
      if (g.sAk == 1) {
        kk = e % kGK;
        mm = e / kGK;
      } else {
        mm = e % kGT;
        kk = e / kGT;
      }
      const int m = m0 + mm, k = k0 + kk;
      As[kk][mm] = (m < g.M && k < kend) ? A[m * g.sAm + k * g.sAk] : 0.f;
    }
    for (int e = threadIdx.x; e < kGT * kGK; e += 256) {
      int nn, kk;
      if (g.sBk == 1) {
        kk = e % kGK;
        nn = e / kGK;
      } else {
        nn = e % kGT;
        kk = e / kGT;
      }
      const int n = n0 + nn, k = k0 + kk;
      Bs[kk][nn] = (n < g.N && k < kend) ? B[k * g.sBk + n * g.sBn] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kGK; kk++) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; i++) a[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; j++) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int m = m0 + ty + 16 * i, n = n0 + tx + 16 * j;
      if (m >= g.M || n >= g.N) continue;
      float *c = C + m * g.sCm + n * g.sCn;
      const float v = g.alpha * acc[i][j];
      if (g.mode == 2)
        atomicAdd(c, v);
      else
        *c = g.mode == 1 ? *c + v : v;
    }
}

// ---------------- truncated DFT along y and the mode mix ----------------
// out[b][r][kx] = sum_y F[r][y] in[b][y][kx]
__global__ void k_fy_fwd(const float2 *__restrict__ in, float2 *__restrict__ out, const float2 *__restrict__ F, int NB,
                         int N, int M, int KY) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)NB * KY * M) return;
  const int kx = idx % M, r = (idx / M) % KY;
  const long long b = idx / ((long long)M * KY);
  const float2 *src = in + b * N * M + kx;
  const float2 *f = F + (size_t)r * N;
  float2 acc = make_float2(0.f, 0.f);
  for (int y = 0; y < N; y++) cfma(acc, __ldg(&f[y]), src[(size_t)y * M]);
  out[(b * KY + r) * M + kx] = acc;
}

// out[b][y][kx] = sum_r conj(F[r][y]) in[b][r][kx]
__global__ void k_fy_inv(const float2 *__restrict__ in, float2 *__restrict__ out, const float2 *__restrict__ F, int NB,
                         int N, int M, int KY) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)NB * N * M) return;
  const int kx = idx % M, y = (idx / M) % N;
  const long long b = idx / ((long long)M * N);
  const float2 *src = in + b * KY * M + kx;
  float2 acc = make_float2(0.f, 0.f);
  for (int r = 0; r < KY; r++) cfma(acc, cconj(__ldg(&F[(size_t)r * N + y])), src[(size_t)r * M]);
  out[(b * N + y) * M + kx] = acc;
}

// The weight as the products use it: rounded to BF16 in the tensor-core
// model (whose GEMMs see BF16 weights), unchanged in the FP32 model.
__device__ __forceinline__ float2 wround(float2 w, int bf16) {
  return bf16 ? make_float2(__bfloat162float(__float2bfloat16_rn(w.x)), __bfloat162float(__float2bfloat16_rn(w.y)))
              : w;
}

// Y[s][o][k] = sum_c R[k][o][c] X[s][c][k]
__global__ void k_mix_fwd(const float2 *__restrict__ X, const float2 *__restrict__ R, float2 *__restrict__ Y, int S,
                          int C, int NM, int bf16) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= S * C * NM) return;
  const int k = idx % NM, o = (idx / NM) % C, s = idx / (NM * C);
  float2 acc = make_float2(0.f, 0.f);
  for (int c = 0; c < C; c++)
    cfma(acc, wround(__ldg(&R[((size_t)k * C + o) * C + c]), bf16), X[((size_t)s * C + c) * NM + k]);
  Y[((size_t)s * C + o) * NM + k] = acc;
}

// dX[s][c][k] = sum_o conj(R[k][o][c]) dY[s][o][k]
__global__ void k_mix_bwd_x(const float2 *__restrict__ dY, const float2 *__restrict__ R, float2 *__restrict__ dX, int S,
                            int C, int NM, int bf16) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= S * C * NM) return;
  const int k = idx % NM, c = (idx / NM) % C, s = idx / (NM * C);
  float2 acc = make_float2(0.f, 0.f);
  for (int o = 0; o < C; o++)
    cfma(acc, cconj(wround(__ldg(&R[((size_t)k * C + o) * C + c]), bf16)), dY[((size_t)s * C + o) * NM + k]);
  dX[((size_t)s * C + c) * NM + k] = acc;
}

// dR[k][o][c] += sum_s dY[s][o][k] conj(X[s][c][k])
__global__ void k_mix_bwd_r(const float2 *__restrict__ dY, const float2 *__restrict__ X, float2 *__restrict__ dR, int S,
                            int C, int NM) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= NM * C * C) return;
  const int c = idx % C, o = (idx / C) % C, k = idx / (C * C);
  float2 acc = dR[idx];
  for (int s = 0; s < S; s++) cfma(acc, dY[((size_t)s * C + o) * NM + k], cconj(X[((size_t)s * C + c) * NM + k]));
  dR[idx] = acc;
}

// ---------------- elementwise ----------------
__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d(float x) {
  return 0.5f * (1.f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

// in[s][10][p] from raster complex g (per sample or shared), b and s1
__global__ void k_fno_prep(const float2 *__restrict__ g, int g_per_sample, const float2 *__restrict__ b,
                           const float2 *__restrict__ s1, float *__restrict__ in, int S, int P, float chi_scale) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)S * P) return;
  const int p = idx % P, s = idx / P;
  const float2 gv = g[(g_per_sample ? (size_t)s * P : 0) + p];
  const float2 chi = make_float2(gv.x * chi_scale, gv.y * chi_scale);
  const float2 f[5] = {chi, b[idx], cmul(chi, b[idx]), s1[idx], cmul(chi, s1[idx])};
  float *o = in + (size_t)s * kFnoIn * P + p;
#pragma unroll
  for (int q = 0; q < 5; q++) {
    o[(size_t)(2 * q) * P] = f[q].x;
    o[(size_t)(2 * q + 1) * P] = f[q].y;
  }
}

// s1 = b - y (blocked; y = A b = b - G(g b))
__global__ void k_fno_born(const float2 *__restrict__ b, const float2 *__restrict__ y, float2 *__restrict__ s1,
                           long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) s1[i] = make_float2(b[i].x - y[i].x, b[i].y - y[i].y);
}

// h[s][o][p] += bias[o] (+ spec[s][o][p]); v = act ? GELU(h) : h
__global__ void k_act_fwd(float *__restrict__ h, const float *__restrict__ bias, const float *__restrict__ spec,
                          float *__restrict__ v, int S, int C, int P, int act) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)S * C * P) return;
  const int o = (idx / P) % C;
  float x = h[idx] + bias[o] + (spec ? spec[idx] : 0.f);
  h[idx] = x;
  v[idx] = act ? gelu(x) : x;
}

// dh = act ? dv * GELU'(h) : dv   (in place)
__global__ void k_act_bwd(float *__restrict__ dv, const float *__restrict__ h, long long n) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx < n) dv[idx] *= gelu_d(h[idx]);
}

// db[o] += sum_{s,p} d[s][o][p]; grid (C, blocks over S*P)
__global__ void k_bias_grad(const float *__restrict__ d, float *__restrict__ db, int S, int C, int P) {
  const int o = blockIdx.x;
  float acc = 0.f;
  for (long long e = (long long)blockIdx.y * blockDim.x + threadIdx.x; e < (long long)S * P;
       e += (long long)gridDim.y * blockDim.x) {
    const int s = e / P, p = e % P;
    acc += d[((size_t)s * C + o) * P + p];
  }
  for (int w = 16; w > 0; w >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, w);
  __shared__ float red[8];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
    atomicAdd(&db[o], t);
  }
}

// x[s][p] = b[s][p] + out[s][0..1][p]
__global__ void k_fno_combine(const float2 *__restrict__ b, const float *__restrict__ out, float2 *__restrict__ x,
                              int S, int P) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)S * P) return;
  const int p = idx % P, s = idx / P;
  const float *o = out + (size_t)s * 2 * P + p;
  x[idx] = make_float2(b[idx].x + o[0], b[idx].y + o[P]);
}

// red[2s] += |u|^2, red[2s+1] += |b + out - u|^2
__global__ void k_fno_sums(const float2 *__restrict__ b, const float *__restrict__ out, const float2 *__restrict__ u,
                           double *__restrict__ red, int P) {
  const int s = blockIdx.y;
  double uu = 0.0, ee = 0.0;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
    const size_t i = (size_t)s * P + p;
    const float *o = out + (size_t)s * 2 * P + p;
    const float2 uv = u[i];
    const float ex = b[i].x + o[0] - uv.x, ey = b[i].y + o[P] - uv.y;
    uu += (double)uv.x * uv.x + (double)uv.y * uv.y;
    ee += (double)ex * ex + (double)ey * ey;
  }
  for (int w = 16; w > 0; w >>= 1) {
    uu += __shfl_xor_sync(0xffffffffu, uu, w);
    ee += __shfl_xor_sync(0xffffffffu, ee, w);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&red[2 * s], uu);
    atomicAdd(&red[2 * s + 1], ee);
  }
}

// dout[s][0..1][p] = 2 (b + out - u) / (|u_s|^2 nsamples)
__global__ void k_fno_dout(const float2 *__restrict__ b, const float *__restrict__ out, const float2 *__restrict__ u,
                           const double *__restrict__ red, float *__restrict__ dout, int S, int P, int nsamples) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)S * P) return;
  const int p = idx % P, s = idx / P;
  const float scale = (float)(2.0 / (fmax(red[2 * s], 1e-30) * nsamples));
  const float *o = out + (size_t)s * 2 * P + p;
  float *d = dout + (size_t)s * 2 * P + p;
  d[0] = scale * (b[idx].x + o[0] - u[idx].x);
  d[P] = scale * (b[idx].y + o[P] - u[idx].y);
}

// blocked: r = y - b; red[2s] += |b|^2, red[2s+1] += |r|^2 (r written over y)
__global__ void k_fno_resid(float2 *__restrict__ y, const float2 *__restrict__ b, double *__restrict__ red, int P) {
  const int s = blockIdx.y;
  double bb = 0.0, rr = 0.0;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
    const size_t i = (size_t)s * P + p;
    const float2 bv = b[i], r = make_float2(y[i].x - bv.x, y[i].y - bv.y);
    y[i] = r;
    bb += (double)bv.x * bv.x + (double)bv.y * bv.y;
    rr += (double)r.x * r.x + (double)r.y * r.y;
  }
  for (int w = 16; w > 0; w >>= 1) {
    bb += __shfl_xor_sync(0xffffffffu, bb, w);
    rr += __shfl_xor_sync(0xffffffffu, rr, w);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&red[2 * s], bb);
    atomicAdd(&red[2 * s + 1], rr);
  }
}

// dout[s][0..1][p] = 2 d[s][p] / (|b_s|^2 nsamples), d in raster order
__global__ void k_fno_dout_resid(const float2 *__restrict__ d, const double *__restrict__ red, float *__restrict__ dout,
                                 int S, int P, int nsamples) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)S * P) return;
  const int p = idx % P, s = idx / P;
  const float scale = (float)(2.0 / (fmax(red[2 * s], 1e-30) * nsamples));
  float *o = dout + (size_t)s * 2 * P + p;
  o[0] = scale * d[idx].x;
  o[P] = scale * d[idx].y;
}

__global__ void k_adam(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m, float *__restrict__ v,
                       long long n, float lr, float b1, float b2, float eps, float c1, float c2) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

inline unsigned blocks(long long n, int t = 256) { return (unsigned)((n + t - 1) / t); }

// ---------------- batched strided GEMM on the tcgen05 tensor cores ----------------
// The same product as k_gemm with BF16 operands and FP32 accumulation: each
// CTA computes a 128 x NT tile of C (NT = BfArgs::nt, a multiple of 16, at
// most 256) in TMEM.  Per K-stage of 64 all 256 threads read the FP32 A and B
// tiles through their strides (consecutive threads along whichever of the two
// indices is contiguous), round them to BF16 and store them in the K-major
// no-swizzle core-matrix layout (8 rows x 16 bytes per core matrix); one
// thread issues the stage's four K = 16 MMAs while the threads fill the other
// stage buffer.  Shared memory and TMEM are sized to the tile (one stage
// buffer when K fits in one, TMEM columns rounded up from NT), so the skinny
// products of the network (K and N of 32) run many CTAs per SM.  The epilogue reads TMEM lane = row of the tile, column = n.
// Rows, columns and K beyond the problem are zero-filled, so any M, N, K work.
namespace bf {
using namespace tc;
constexpr int KC = 64;                 // K per stage
constexpr int kA = 128 * KC * 2;       // 16 KB: A tile
constexpr int kB = 256 * KC * 2;       // 32 KB: B tile at NT = 256
constexpr int kSmem = 2 * (kA + kB) + 64;  // at most: two stages at NT = 256, mbarriers, TMEM slot
constexpr int kThreads = 256;
constexpr int kErr = 151;

__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N) {
  return (1u << 4)                      // D format F32
         | (1u << 7) | (1u << 10)       // A, B format BF16
         | ((uint32_t)(N >> 3) << 17)   // N / 8
         | ((uint32_t)(M >> 4) << 24);  // M / 16
}

__device__ __forceinline__ void mma_bf16(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, int acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

// byte offset of element (row, k) in a K-major tile of KC columns
__device__ __forceinline__ int core_off(int row, int k) {
  return (((row >> 3) * (KC / 8) + (k >> 3)) * 64 + (row & 7) * 8 + (k & 7)) * 2;
}

__device__ __forceinline__ uint32_t pack(float a, float b) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);  // a in the low half
  return *reinterpret_cast<const uint32_t *>(&h);
}

// rows [r0, r0 + nrows) x K [k0, k0 + KC) of X (element (r, k) at r sr + k sk)
// as BF16 into dst; rows >= rvalid and k >= kend read as zero
__device__ __forceinline__ void stage(char *dst, const float *X, long long sr, long long sk, int r0, int nrows,
                                      int rvalid, int k0, int kend) {
  const bool kcontig = sk == 1;
  // 16-byte loads where a row's K run is contiguous and 16-byte aligned (kb is a multiple of 8)
  const bool vec = kcontig && (sr & 3) == 0 && (reinterpret_cast<uintptr_t>(X) & 15) == 0;
  for (int e = threadIdx.x; e < nrows * (KC / 8); e += kThreads) {
    const int row = kcontig ? e / (KC / 8) : e % nrows, kc = kcontig ? e % (KC / 8) : e / nrows;
    const int r = r0 + row, kb = k0 + kc * 8;
    float v[8];
    if (vec && r < rvalid && kb + 8 <= kend) {
      const float4 a = *(const float4 *)(X + (long long)r * sr + kb), b = *(const float4 *)(X + (long long)r * sr + kb + 4);
      v[0] = a.x, v[1] = a.y, v[2] = a.z, v[3] = a.w, v[4] = b.x, v[5] = b.y, v[6] = b.z, v[7] = b.w;
    } else {
#pragma unroll
      for (int q = 0; q < 8; q++)
        v[q] = (r < rvalid && kb + q < kend) ? X[(long long)r * sr + (long long)(kb + q) * sk] : 0.f;
    }
    *(uint4 *)(dst + core_off(row, kc * 8)) = make_uint4(pack(v[0], v[1]), pack(v[2], v[3]), pack(v[4], v[5]),
                                                         pack(v[6], v[7]));
  }
}

struct Args {
  const float *A, *B;
  float *C;
  int M, N, K, ksplit, mode, nt;
  int stage, tcols;  // bytes of one stage buffer (A tile + nt B rows); TMEM columns (power of two >= nt, >= 32)
  long long sAm, sAk, sBk, sBn, sCm, sCn, bA, bB, bC;
  float alpha;
  int *err;
};

__global__ void __launch_bounds__(kThreads, 1) k_gemm_bf16(Args g) {
  extern __shared__ __align__(1024) char sm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int batch = blockIdx.z / g.ksplit, ks = blockIdx.z % g.ksplit;
  const float *A = g.A + batch * g.bA, *B = g.B + batch * g.bB;
  float *C = g.C + batch * g.bC;
  const int m0 = blockIdx.y * 128, n0 = blockIdx.x * g.nt;
  const int kper = ((g.K + g.ksplit - 1) / g.ksplit + KC - 1) / KC * KC;
  const int kbeg = ks * kper, kend = min(g.K, kbeg + kper);
  const int nbuf = kper > KC ? 2 : 1;  // one stage buffer when the split's K fits in one
  uint64_t *mdone = (uint64_t *)(sm + nbuf * g.stage), *fin = mdone + 2;
  uint32_t *tslot = (uint32_t *)(mdone + 4);
  if (threadIdx.x == 0) {
    for (int i = 0; i < 3; i++) mbar_init(mdone + i, 1);
    fence_mbar_init();
  }
  if (warp == 0) tmem_alloc(tslot, g.tcols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot, idesc = idesc_bf16_f32(128, g.nt), sbase = smem_u32(sm);
  bool ok = true;
  int it = 0;
  for (int k0 = kbeg; k0 < kend; k0 += KC, it++) {
    const int b = it & 1;
    // stage buffer b is free once the MMAs of stage it - 2 are done
    if (it >= 2) ok = mbar_wait(mdone + b, ((it >> 1) - 1) & 1, g.err, kErr) && ok;
    char *sa = sm + b * g.stage;
    stage(sa, A, g.sAm, g.sAk, m0, 128, g.M, k0, kend);
    stage(sa + kA, B, g.sBn, g.sBk, n0, g.nt, g.N, k0, kend);
    fence_proxy_async();
    __syncthreads();
    if (threadIdx.x == 0) {
      tc_fence_after();
      if (ok) {
        const uint64_t ad = smem_desc(sbase + b * g.stage, 128, KC / 8 * 128);
        const uint64_t bd = smem_desc(sbase + b * g.stage + kA, 128, KC / 8 * 128);
#pragma unroll
        for (int q = 0; q < KC / 16; q++)
          mma_bf16(tmem, desc_add(ad, q * 256), desc_add(bd, q * 256), idesc, (it > 0 || q > 0) ? 1 : 0);
      }
      mma_commit(mdone + b);
    }
  }
  if (threadIdx.x == 0) mma_commit(fin);
  ok = mbar_wait(fin, 0, g.err, kErr) && ok && kend > kbeg;
  tc_fence_after();
  // epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31, column groups of 16 alternating between w < 4 and w >= 4
  const int qd = warp & 3, half = warp >> 2, row = m0 + 32 * qd + lane;
  const int nvalid = min(g.nt, g.N - n0);
  // Row-major C (consecutive columns contiguous): each warp turns its 32 x 16 block around in shared
  // memory (the stage buffers, free once the MMAs are done) so that 16 lanes write one row's 64 bytes.
  const bool rowmajor = g.sCn == 1 && g.mode != 2;
  float *tile = reinterpret_cast<float *>(sm) + warp * (32 * 17);
  for (int c0 = 16 * half; c0 < g.nt; c0 += 32) {
    __syncwarp();
    float d[16];
    tmem_ld16(tmem + ((uint32_t)(32 * qd) << 16) + (uint32_t)c0, d);
    if (rowmajor) {
#pragma unroll
      for (int q = 0; q < 16; q++) tile[lane * 17 + q] = d[q];
      __syncwarp();
      const int cq = lane & 15;
      if (ok && c0 + cq < nvalid) {
#pragma unroll 4
        for (int rr = lane >> 4; rr < 32; rr += 2) {
          const int r = m0 + 32 * qd + rr;
          if (r >= g.M) break;
          float *c = C + (long long)r * g.sCm + (n0 + c0 + cq);
          const float v = g.alpha * tile[rr * 17 + cq];
          *c = g.mode == 1 ? *c + v : v;
        }
      }
      continue;
    }
    if (!ok || row >= g.M) continue;
#pragma unroll
    for (int q = 0; q < 16; q++) {
      if (c0 + q >= nvalid) break;
      float *c = C + (long long)row * g.sCm + (long long)(n0 + c0 + q) * g.sCn;
      const float v = g.alpha * d[q];
      if (g.mode == 2)
        atomicAdd(c, v);
      else
        *c = g.mode == 1 ? *c + v : v;
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, g.tcols);
}
}  // namespace bf

void gemm_bf16(cudaStream_t st, int *err, int batch, int M, int N, int K, const float *A, long long sAm, long long sAk,
               long long bA, const float *B, long long sBk, long long sBn, long long bB, float *C, long long sCm,
               long long sCn, long long bC, int mode, int ksplit, float alpha) {
  // rows of the tile come from the larger of M and N: C^T = B^T A^T when M is the small side
  if (M < 128 && N > M) {
    std::swap(M, N);
    std::swap(A, B);
    std::swap(bA, bB);
    std::swap(sCm, sCn);
    const long long am = sBn, ak = sBk, bk = sAk, bn = sAm;
    sAm = am, sAk = ak, sBk = bk, sBn = bn;
  }
  const int nt = std::min(256, (N + 15) / 16 * 16);
  int tcols = 32;
  while (tcols < nt) tcols *= 2;
  const int stage = bf::kA + nt * bf::KC * 2;
  const int kper = ((K + ksplit - 1) / ksplit + bf::KC - 1) / bf::KC * bf::KC;
  // at most 512 / tcols CTAs may share an SM's 512 TMEM columns: ask for enough shared memory that no
  // more fit (228 KB per SM, 1 KB of it reserved per CTA), so no CTA waits inside tcgen05.alloc
  const int ctas = 512 / tcols;
  const int smem = std::max((kper > bf::KC ? 2 : 1) * stage + 64, 233472 / (ctas + 1) - 1024 + 16);
  bf::Args g{A, B, C, M, N, K, ksplit, mode, nt, stage, tcols, sAm, sAk, sBk, sBn, sCm, sCn, bA, bB, bC, alpha, err};
  count_launch();
  bf::k_gemm_bf16<<<dim3((N + nt - 1) / nt, (M + 127) / 128, batch * ksplit), bf::kThreads, smem, st>>>(g);
}

// The model's GEMMs: BF16 tcgen05 (the default) or FP32 k_gemm.
void gemm(const FnoModel &F, cudaStream_t st, int batch, int M, int N, int K, const float *A, long long sAm, long long sAk, long long bA,
          const float *B, long long sBk, long long sBn, long long bB, float *C, long long sCm, long long sCn,
          long long bC, int mode, int ksplit = 1, float alpha = 1.f) {
  if (F.tensor) {
    gemm_bf16(st, F.err, batch, M, N, K, A, sAm, sAk, bA, B, sBk, sBn, bB, C, sCm, sCn, bC, mode, ksplit,
              alpha);
    return;
  }
  GemmArgs g{A, B, C, M, N, K, ksplit, mode, sAm, sAk, sBk, sBn, sCm, sCn, bA, bB, bC, alpha};
  count_launch();
  k_gemm<<<dim3((N + kGT - 1) / kGT, (M + kGT - 1) / kGT, batch * ksplit), 256, 0, st>>>(g);
}

int ksplit_for(long long K) { return (int)std::max<long long>(1, std::min<long long>(256, K / 4096)); }

uint64_t mix64(uint64_t &s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
double unif(uint64_t &s) { return (mix64(s) >> 11) * (1.0 / 9007199254740992.0); }

}  // namespace

// ---- model set-up ----
isg_status fno_create(isg_ctx *c, const isg_fno_opts *o) {
  if (!c->gpu_ready) return ISG_BAD_ARG;
  const int N = c->T.side;
  if (o->width < 1 || o->width > 128 || o->layers < 1 || o->layers > 8 || o->modes < 1 || 2 * o->modes > N ||
      o->batch < 1 || o->batch > 64) {
    c->err = "fno options out of range (width 1..128, layers 1..8, 1 <= modes <= side/2, batch 1..64)";
    return ISG_BAD_ARG;
  }
  fno_destroy(c);
  FnoModel *F = new FnoModel();
  c->fno = F;
  F->C = o->width;
  F->M = o->modes;
  F->L = o->layers;
  F->S = o->batch;
  F->KY = 2 * F->M;
  F->NM = F->KY * F->M;
  F->N = N;
  F->P = N * N;
  F->tensor = o->tensor != 0;
  if (F->tensor && !tc_available(c)) {
    c->err = "fno: BF16 tensor-core products need an sm_100 device (set tensor = 0 for FP32)";
    return ISG_UNSUPPORTED;
  }
  const int C = F->C, M = F->M, L = F->L, S = F->S, KY = F->KY, NM = F->NM, P = F->P;
  // parameter layout, each block on a 4-float boundary
  size_t off = 0;
  auto take = [&](size_t n) {
    const size_t r = off;
    off += (n + 3) / 4 * 4;
    return r;
  };
  F->off_Wl = take((size_t)C * kFnoIn);
  F->off_bl = take(C);
  for (int l = 0; l < L; l++) {
    F->off_R.push_back(take((size_t)2 * NM * C * C));
    F->off_W.push_back(take((size_t)C * C));
    F->off_bw.push_back(take(C));
  }
  F->off_Wp = take((size_t)2 * C);
  F->off_Ws = take((size_t)2 * kFnoIn);
  F->off_bp = take(2);
  F->nparam = off;
  // seeded initialisation
  std::vector<float> h(F->nparam, 0.f);
  uint64_t seed = 0x5EEDull ^ (uint64_t)o->seed * 0x9E3779B97F4A7C15ull;
  auto fill = [&](size_t at, size_t n, double lim) {
    for (size_t i = 0; i < n; i++) h[at + i] = (float)((2.0 * unif(seed) - 1.0) * lim);
  };
  fill(F->off_Wl, (size_t)C * kFnoIn, 1.0 / std::sqrt((double)kFnoIn));
  for (int l = 0; l < L; l++) {
    for (size_t i = 0; i < (size_t)2 * NM * C * C; i++) h[F->off_R[l] + i] = (float)(unif(seed) / ((double)C * C));
    fill(F->off_W[l], (size_t)C * C, 1.0 / std::sqrt((double)C));
  }
  fill(F->off_Wp, (size_t)2 * C, 0.1 / std::sqrt((double)C));
  // transform tables
  const double th = 2.0 * M_PI / N;
  std::vector<float> ex((size_t)N * 2 * M), ix((size_t)2 * M * N);
  for (int x = 0; x < N; x++)
    for (int k = 0; k < M; k++) {
      const double a = th * (double)((long long)k * x % N), w = (k == 0 ? 1.0 : 2.0) / ((double)N * N);
      ex[(size_t)x * 2 * M + 2 * k] = (float)std::cos(a);
      ex[(size_t)x * 2 * M + 2 * k + 1] = (float)-std::sin(a);
      ix[(size_t)(2 * k) * N + x] = (float)(w * std::cos(a));
      ix[(size_t)(2 * k + 1) * N + x] = (float)(-w * std::sin(a));
    }
  std::vector<float2> fy((size_t)KY * N);
  for (int r = 0; r < KY; r++) {
    const long long f = r < M ? r : N - KY + r;
    for (int y = 0; y < N; y++) {
      const double a = th * (double)(f * y % N);
      fy[(size_t)r * N + y] = make_float2((float)std::cos(a), (float)-std::sin(a));
    }
  }
  auto ck = [&](cudaError_t e) { return cuda_check(c, e, "fno alloc"); };
  isg_status e;
  if ((e = ck(F->alloc(&F->param, F->nparam))) || (e = ck(F->alloc(&F->grad, F->nparam))) ||
      (e = ck(F->alloc(&F->am, F->nparam))) || (e = ck(F->alloc(&F->av, F->nparam))) ||
      (e = ck(F->alloc(&F->Ex, ex.size()))) || (e = ck(F->alloc(&F->Ix, ix.size()))) ||
      (e = ck(F->alloc(&F->Fy, fy.size()))) || (e = ck(F->alloc(&F->err, 1))) ||
      (e = ck(cudaMemset(F->err, 0, sizeof(int)))))
    return e;
  if (F->tensor &&
      (e = ck(cudaFuncSetAttribute(bf::k_gemm_bf16, cudaFuncAttributeMaxDynamicSharedMemorySize, bf::kSmem))))
    return e;
  const size_t act = (size_t)S * C * P;
  F->v.assign(L + 1, nullptr);
  F->h.assign(L, nullptr);
  F->X.assign(L, nullptr);
  for (int l = 0; l <= L; l++)
    if ((e = ck(F->alloc(&F->v[l], act)))) return e;
  for (int l = 0; l < L; l++)
    if ((e = ck(F->alloc(&F->h[l], act))) || (e = ck(F->alloc(&F->X[l], (size_t)S * C * NM)))) return e;
  if ((e = ck(F->alloc(&F->in, (size_t)S * kFnoIn * P))) || (e = ck(F->alloc(&F->spec, act))) ||
      (e = ck(F->alloc(&F->out, (size_t)S * 2 * P))) || (e = ck(F->alloc(&F->dout, (size_t)S * 2 * P))) ||
      (e = ck(F->alloc(&F->dva, act))) || (e = ck(F->alloc(&F->dvb, act))) ||
      (e = ck(F->alloc(&F->T, (size_t)S * C * N * 2 * M))) || (e = ck(F->alloc(&F->Z, (size_t)S * C * N * 2 * M))) ||
      (e = ck(F->alloc(&F->Y, (size_t)S * C * NM))) || (e = ck(F->alloc(&F->gr, (size_t)S * P))) ||
      (e = ck(F->alloc(&F->br, (size_t)S * P))) || (e = ck(F->alloc(&F->ur, (size_t)S * P))) ||
      (e = ck(F->alloc(&F->xr, (size_t)S * P))) || (e = ck(F->alloc(&F->red, (size_t)2 * S + 2))) ||
      (e = ck(F->alloc(&F->gb, (size_t)S * P))) || (e = ck(F->alloc(&F->bb, (size_t)S * P))) ||
      (e = ck(F->alloc(&F->xb, (size_t)S * P))) || (e = ck(F->alloc(&F->yb, (size_t)S * P))) ||
      (e = ck(F->alloc(&F->sr, (size_t)S * P))))
    return e;
  if ((e = ck(cudaMemcpy(F->param, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice))) ||
      (e = ck(cudaMemset(F->grad, 0, F->nparam * sizeof(float)))) ||
      (e = ck(cudaMemset(F->am, 0, F->nparam * sizeof(float)))) ||
      (e = ck(cudaMemset(F->av, 0, F->nparam * sizeof(float)))) ||
      (e = ck(cudaMemcpy(F->Ex, ex.data(), ex.size() * sizeof(float), cudaMemcpyHostToDevice))) ||
      (e = ck(cudaMemcpy(F->Ix, ix.data(), ix.size() * sizeof(float), cudaMemcpyHostToDevice))) ||
      (e = ck(cudaMemcpy(F->Fy, fy.data(), fy.size() * sizeof(float2), cudaMemcpyHostToDevice))))
    return e;
  return ISG_OK;
}

void fno_destroy(isg_ctx *c) {
  delete c->fno;
  c->fno = nullptr;
}

namespace {

// Forward pass of n <= S samples whose raster inputs are in F.gr (per sample
// when g_per_sample) and F.br; leaves every activation for the backward pass.
void fno_forward(isg_ctx *c, int n, int g_per_sample, cudaStream_t st) {
  FnoModel &F = *c->fno;
  const int C = F.C, M = F.M, N = F.N, P = F.P, KY = F.KY, NM = F.NM;
  const float *W = F.param;
  const float chi = (float)(1.0 / (c->T.k0 * c->T.k0));
  k_fno_prep<<<blocks((long long)n * P), 256, 0, st>>>(F.gr, g_per_sample, F.br, F.sr, F.in, n, P, chi);
  count_launch();
  const long long IP = (long long)kFnoIn * P;
  // lift
  gemm(F, st, n, C, P, kFnoIn, W + F.off_Wl, kFnoIn, 1, 0, F.in, P, 1, IP, F.v[0], P, 1, (long long)C * P, 0);
  k_act_fwd<<<blocks((long long)n * C * P), 256, 0, st>>>(F.v[0], W + F.off_bl, nullptr, F.v[0], n, C, P, 0);
  count_launch();
  for (int l = 0; l < F.L; l++) {
    const int rows = n * C * N;
    gemm(F, st, 1, rows, 2 * M, N, F.v[l], N, 1, 0, F.Ex, 2 * M, 1, 0, F.T, 2 * M, 1, 0, 0);
    k_fy_fwd<<<blocks((long long)n * C * KY * M), 256, 0, st>>>((const float2 *)F.T, F.X[l], F.Fy, n * C, N, M, KY);
    k_mix_fwd<<<blocks((long long)n * C * NM), 256, 0, st>>>(F.X[l], (const float2 *)(W + F.off_R[l]), F.Y, n, C, NM,
                                                             F.tensor);
    k_fy_inv<<<blocks((long long)n * C * N * M), 256, 0, st>>>(F.Y, (float2 *)F.Z, F.Fy, n * C, N, M, KY);
    count_launch(3);
    gemm(F, st, 1, rows, N, 2 * M, F.Z, 2 * M, 1, 0, F.Ix, N, 1, 0, F.spec, N, 1, 0, 0);
    gemm(F, st, n, C, P, C, W + F.off_W[l], C, 1, 0, F.v[l], P, 1, (long long)C * P, F.h[l], P, 1, (long long)C * P, 0);
    k_act_fwd<<<blocks((long long)n * C * P), 256, 0, st>>>(F.h[l], W + F.off_bw[l], F.spec, F.v[l + 1], n, C, P,
                                                            l + 1 < F.L);
    count_launch();
  }
  gemm(F, st, n, 2, P, C, W + F.off_Wp, C, 1, 0, F.v[F.L], P, 1, (long long)C * P, F.out, P, 1, 2LL * P, 0);
  gemm(F, st, n, 2, P, kFnoIn, W + F.off_Ws, kFnoIn, 1, 0, F.in, P, 1, IP, F.out, P, 1, 2LL * P, 1);
  k_act_fwd<<<blocks((long long)n * 2 * P), 256, 0, st>>>(F.out, W + F.off_bp, nullptr, F.out, n, 2, P, 0);
  count_launch();
}

// Backward pass from F.dout, accumulating into F.grad.
void fno_backward(isg_ctx *c, int n, cudaStream_t st) {
  FnoModel &F = *c->fno;
  const int C = F.C, M = F.M, N = F.N, P = F.P, KY = F.KY, NM = F.NM;
  const float *W = F.param;
  float *G = F.grad;
  const long long CP = (long long)C * P;
  const int ks = ksplit_for(P);
  // projection
  const long long IP = (long long)kFnoIn * P;
  gemm(F, st, n, 2, C, P, F.dout, P, 1, 2LL * P, F.v[F.L], 1, P, CP, G + F.off_Wp, C, 1, 0, 2, ks);
  gemm(F, st, n, 2, kFnoIn, P, F.dout, P, 1, 2LL * P, F.in, 1, P, IP, G + F.off_Ws, kFnoIn, 1, 0, 2, ks);
  k_bias_grad<<<dim3(2, 64), 256, 0, st>>>(F.dout, G + F.off_bp, n, 2, P);
  count_launch();
  float *dv = F.dva, *dn = F.dvb;
  gemm(F, st, n, C, P, 2, W + F.off_Wp, 1, C, 0, F.dout, P, 1, 2LL * P, dv, P, 1, CP, 0);
  for (int l = F.L - 1; l >= 0; l--) {
    if (l + 1 < F.L) {
      k_act_bwd<<<blocks((long long)n * CP), 256, 0, st>>>(dv, F.h[l], (long long)n * CP);
      count_launch();
    }
    // dv now holds dh
    k_bias_grad<<<dim3(C, 64), 256, 0, st>>>(dv, G + F.off_bw[l], n, C, P);
    count_launch();
    gemm(F, st, n, C, C, P, dv, P, 1, CP, F.v[l], 1, P, CP, G + F.off_W[l], C, 1, 0, 2, ks);
    const int rows = n * C * N;
    gemm(F, st, 1, rows, 2 * M, N, dv, N, 1, 0, F.Ix, 1, N, 0, F.Z, 2 * M, 1, 0, 0);
    k_fy_fwd<<<blocks((long long)n * C * KY * M), 256, 0, st>>>((const float2 *)F.Z, F.Y, F.Fy, n * C, N, M, KY);
    k_mix_bwd_r<<<blocks((long long)NM * C * C), 256, 0, st>>>(F.Y, F.X[l], (float2 *)(G + F.off_R[l]), n, C, NM);
    // dX into the (free) layer-l spectrum buffer of the next pass: reuse T as scratch for dX
    k_mix_bwd_x<<<blocks((long long)n * C * NM), 256, 0, st>>>(F.Y, (const float2 *)(W + F.off_R[l]),
                                                               (float2 *)F.T, n, C, NM, F.tensor);
    k_fy_inv<<<blocks((long long)n * C * N * M), 256, 0, st>>>((const float2 *)F.T, (float2 *)F.Z, F.Fy, n * C, N, M,
                                                               KY);
    count_launch(4);
    gemm(F, st, 1, rows, N, 2 * M, F.Z, 2 * M, 1, 0, F.Ex, 1, 2 * M, 0, dn, N, 1, 0, 0);
    gemm(F, st, n, C, P, C, W + F.off_W[l], 1, C, 0, dv, P, 1, CP, dn, P, 1, CP, 1);
    std::swap(dv, dn);
  }
  // lift
  gemm(F, st, n, C, kFnoIn, P, dv, P, 1, CP, F.in, 1, P, IP, G + F.off_Wl, kFnoIn, 1, 0, 2, ks);
  k_bias_grad<<<dim3(C, 64), 256, 0, st>>>(dv, G + F.off_bl, n, C, P);
  count_launch();
}

// Chunk [s0, s0 + n) of the caller's vectors (g shared when gs == 0): blocked
// copies of g and b (gb, bb), raster copies (gr, br, ur) and the raster Born
// field s1 = G(g b) (sr).  Leaves x0's buffers free.
isg_status fno_gather(isg_ctx *c, const float2 *g, int64_t gs, const float2 *b, const float2 *u, int s0, int n,
                      int order, cudaStream_t st) {
  FnoModel &F = *c->fno;
  const int U = (int)c->P.U;
  auto to_blocked = [&](const float2 *src, float2 *dst, int cnt) {
    if (order == ISG_ORDER_BLOCKED)
      cudaMemcpyAsync(dst, src, (size_t)cnt * U * sizeof(float2), cudaMemcpyDeviceToDevice, st);
    else
      launch_permute(order_perm(c, order), src, dst, U, cnt, true, st);
  };
  to_blocked(b + (size_t)s0 * U, F.bb, n);
  to_blocked(g + (gs ? (size_t)s0 * gs : 0), F.gb, gs ? n : 1);
  launch_permute(c->P.perm_raster, F.bb, F.br, U, n, false, st);
  launch_permute(c->P.perm_raster, F.gb, F.gr, U, gs ? n : 1, false, st);
  if (u) {
    to_blocked(u + (size_t)s0 * U, F.xb, n);
    launch_permute(c->P.perm_raster, F.xb, F.ur, U, n, false, st);
  }
  const int engine = tc_available(c) ? ISG_ENGINE_TENSOR : ISG_ENGINE_SIMT;
  isg_status e = run_matvec(c, F.bb, F.gb, gs ? U : 0, F.yb, n, OP_FWD, engine, RED_NONE, nullptr, nullptr, st);
  if (e != ISG_OK) return e;
  k_fno_born<<<blocks((long long)n * U), 256, 0, st>>>(F.bb, F.yb, F.xb, (long long)n * U);
  count_launch();
  launch_permute(c->P.perm_raster, F.xb, F.sr, U, n, false, st);
  return ISG_OK;
}

}  // namespace

// ISG_TIMEOUT once a tensor-core GEMM of the model has hit its wait limit
// (synchronises the stream).
isg_status fno_status(isg_ctx *c, cudaStream_t st) {
  int h = 0;
  isg_status e = cuda_check(c, cudaMemcpyAsync(&h, c->fno->err, sizeof(int), cudaMemcpyDeviceToHost, st), "fno status");
  if (e == ISG_OK) e = cuda_check(c, cudaStreamSynchronize(st), "fno status");
  if (e == ISG_OK && h) {
    c->err = "a tensor-core GEMM of the warm-start network hit its wait limit";
    return ISG_TIMEOUT;
  }
  return e;
}

// x0 = b + N(g, b) for nrhs samples, all vectors in the caller's order.
isg_status fno_apply(isg_ctx *c, const float2 *g, int64_t gs, const float2 *b, float2 *x, int nrhs, int order,
                     cudaStream_t st) {
  FnoModel &F = *c->fno;
  const size_t U = c->P.U;
  const int chunk = std::min(F.S, c->opts.max_rhs);
  for (int s0 = 0; s0 < nrhs; s0 += chunk) {
    const int n = std::min(chunk, nrhs - s0);
    isg_status e = fno_gather(c, g, gs, b, nullptr, s0, n, order, st);
    if (e != ISG_OK) return e;
    fno_forward(c, n, gs != 0, st);
    k_fno_combine<<<blocks((long long)n * F.P), 256, 0, st>>>(F.br, F.out, F.ur, n, F.P);
    count_launch();
    float2 *dst = x + (size_t)s0 * U;
    if (order == ISG_ORDER_RASTER) {
      cudaMemcpyAsync(dst, F.ur, (size_t)n * U * sizeof(float2), cudaMemcpyDeviceToDevice, st);
    } else if (order == ISG_ORDER_BLOCKED) {
      launch_permute(c->P.perm_raster, F.ur, dst, (int)U, n, true, st);
    } else {
      launch_permute(c->P.perm_raster, F.ur, F.xr, (int)U, n, true, st);
      launch_permute(c->P.perm_tree, F.xr, dst, (int)U, n, false, st);
    }
  }
  isg_status e = cuda_check(c, cudaGetLastError(), "fno apply");
  return e == ISG_OK ? fno_status(c, st) : e;
}

// Gradient of the mean loss over nrhs samples into F.grad (zeroed first); the
// loss goes to *loss.  With reference fields u: relative squared field error
// |x0 - u|^2 / |u|^2.  Without (u null): relative squared initial residual
// |b - A x0|^2 / |b|^2 of the forward system, A = I - G diag(g), whose
// gradient 2 A^H (A x0 - b) / |b|^2 takes one forward and one adjoint matvec.
isg_status fno_gradient(isg_ctx *c, const float2 *g, int64_t gs, const float2 *b, const float2 *u, int nrhs, int order,
                        double *loss, cudaStream_t st) {
  FnoModel &F = *c->fno;
  cudaMemsetAsync(F.grad, 0, F.nparam * sizeof(float), st);
  double total = 0.0;
  const int chunk = std::min(F.S, c->opts.max_rhs);
  const int engine = tc_available(c) ? ISG_ENGINE_TENSOR : ISG_ENGINE_SIMT;
  const int U = (int)c->P.U;
  for (int s0 = 0; s0 < nrhs; s0 += chunk) {
    const int n = std::min(chunk, nrhs - s0);
    isg_status ge = fno_gather(c, g, gs, b, u, s0, n, order, st);
    if (ge != ISG_OK) return ge;
    fno_forward(c, n, gs != 0, st);
    cudaMemsetAsync(F.red, 0, (size_t)(2 * F.S + 2) * sizeof(double), st);
    if (u) {
      k_fno_sums<<<dim3(64, n), 256, 0, st>>>(F.br, F.out, F.ur, F.red, F.P);
      k_fno_dout<<<blocks((long long)n * F.P), 256, 0, st>>>(F.br, F.out, F.ur, F.red, F.dout, n, F.P, nrhs);
      count_launch(2);
    } else {
      // x0 and the inputs in the blocked layout, r = A x0 - b, d = A^H r
      k_fno_combine<<<blocks((long long)n * F.P), 256, 0, st>>>(F.br, F.out, F.ur, n, F.P);
      count_launch();
      launch_permute(c->P.perm_raster, F.ur, F.xb, U, n, true, st);
      isg_status e = run_matvec(c, F.xb, F.gb, gs ? U : 0, F.yb, n, OP_FWD, engine, RED_NONE, nullptr, nullptr, st);
      if (e != ISG_OK) return e;
      k_fno_resid<<<dim3(64, n), 256, 0, st>>>(F.yb, F.bb, F.red, U);
      count_launch();
      if ((e = run_matvec(c, F.yb, F.gb, gs ? U : 0, F.xb, n, OP_ADJ, engine, RED_NONE, nullptr, nullptr, st)) !=
          ISG_OK)
        return e;
      launch_permute(c->P.perm_raster, F.xb, F.ur, U, n, false, st);
      k_fno_dout_resid<<<blocks((long long)n * F.P), 256, 0, st>>>(F.ur, F.red, F.dout, n, F.P, nrhs);
      count_launch();
    }
    fno_backward(c, n, st);
    std::vector<double> h((size_t)2 * n);
    cudaMemcpyAsync(h.data(), F.red, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st);
    isg_status e = cuda_check(c, cudaStreamSynchronize(st), "fno gradient");
    if (e != ISG_OK) return e;
    for (int s = 0; s < n; s++) total += h[2 * s + 1] / std::max(h[2 * s], 1e-30);
  }
  if (loss) *loss = total / nrhs;
  isg_status e = cuda_check(c, cudaGetLastError(), "fno gradient");
  return e == ISG_OK ? fno_status(c, st) : e;
}

isg_status fno_adam(isg_ctx *c, float lr, cudaStream_t st) {
  FnoModel &F = *c->fno;
  F.adam_t++;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - std::pow(b1, (float)F.adam_t), c2 = 1.f - std::pow(b2, (float)F.adam_t);
  k_adam<<<blocks((long long)F.nparam), 256, 0, st>>>(F.param, F.grad, F.am, F.av, (long long)F.nparam, lr, b1, b2,
                                                      1e-8f, c1, c2);
  count_launch();
  return cuda_check(c, cudaGetLastError(), "fno adam");
}

size_t fno_param_count(const isg_ctx *c) { return c->fno ? c->fno->nparam : 0; }
float *fno_param_ptr(isg_ctx *c, int which) {
  if (!c->fno) return nullptr;
  return which == 0 ? c->fno->param : c->fno->grad;
}

}  // namespace isg

// ---------------- C ABI ----------------
using namespace isg;

namespace {
isg_status fno_ready(isg_ctx *c) {
  if (!c) return ISG_BAD_ARG;
  if (!c->fno) {
    c->err = "no warm-start network: call isg_fno_create first";
    return ISG_UNSUPPORTED;
  }
  return cuda_check(c, cudaSetDevice(c->opts.device), "cudaSetDevice");
}
bool fno_bad(isg_ctx *c, const void *g, int64_t gs, const void *b, int nrhs, int order) {
  if (!g || !b || nrhs < 1 || order < ISG_ORDER_TREE || order > ISG_ORDER_BLOCKED || (gs != 0 && gs != c->P.U)) {
    c->err = "fno: null pointer, nrhs < 1, bad order or g_stride not in {0, numunk}";
    return true;
  }
  return false;
}
}  // namespace

extern "C" {

void isg_default_fno_opts(isg_fno_opts *o) {
  if (!o) return;
  o->width = 32;
  o->modes = 12;
  o->layers = 4;
  o->batch = 4;
  o->seed = 1;
  o->tensor = 1;
}

isg_status isg_fno_create(isg_ctx *c, const isg_fno_opts *o) {
  if (!c || !o) return ISG_BAD_ARG;
  if (!c->gpu_ready) {
    isg_status e = isg_setup_gpu(c);
    if (e != ISG_OK) return e;
  }
  isg_status e = cuda_check(c, cudaSetDevice(c->opts.device), "cudaSetDevice");
  if (e != ISG_OK) return e;
  e = fno_create(c, o);
  if (e != ISG_OK) fno_destroy(c);
  return e;
}

int64_t isg_fno_param_count(const isg_ctx *c) { return c ? (int64_t)fno_param_count(c) : 0; }

isg_status isg_fno_params(isg_ctx *c, float *host, int64_t n, int which, int set) {
  isg_status e = fno_ready(c);
  if (e != ISG_OK) return e;
  if (!host || n != (int64_t)fno_param_count(c) || which < 0 || which > 1 || (set && which != 0)) {
    c->err = "fno params: n must equal isg_fno_param_count; only parameters (which 0) can be set";
    return ISG_BAD_ARG;
  }
  float *d = fno_param_ptr(c, which);
  return cuda_check(c,
                    set ? cudaMemcpy(d, host, (size_t)n * sizeof(float), cudaMemcpyHostToDevice)
                        : cudaMemcpy(host, d, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost),
                    "fno params");
}

isg_status isg_fno_apply(isg_ctx *c, const void *g, int64_t gs, const void *b, void *x, int nrhs, int order,
                         isg_stream stream) {
  isg_status e = fno_ready(c);
  if (e != ISG_OK) return e;
  if (!x || fno_bad(c, g, gs, b, nrhs, order)) return ISG_BAD_ARG;
  return fno_apply(c, (const float2 *)g, gs, (const float2 *)b, (float2 *)x, nrhs, order, (cudaStream_t)stream);
}

isg_status isg_fno_grad(isg_ctx *c, const void *g, int64_t gs, const void *b, const void *u, int nrhs, int order,
                        double *loss, isg_stream stream) {
  isg_status e = fno_ready(c);
  if (e != ISG_OK) return e;
  if (fno_bad(c, g, gs, b, nrhs, order)) return ISG_BAD_ARG;
  return fno_gradient(c, (const float2 *)g, gs, (const float2 *)b, (const float2 *)u, nrhs, order, loss,
                      (cudaStream_t)stream);
}

isg_status isg_fno_train_step(isg_ctx *c, const void *g, int64_t gs, const void *b, const void *u, int nrhs,
                              int order, float lr, double *loss, isg_stream stream) {
  isg_status e = isg_fno_grad(c, g, gs, b, u, nrhs, order, loss, stream);
  if (e != ISG_OK) return e;
  if (!(lr > 0.f)) {
    c->err = "fno: learning rate must be positive";
    return ISG_BAD_ARG;
  }
  return fno_adam(c, lr, (cudaStream_t)stream);
}

}  // extern "C"
