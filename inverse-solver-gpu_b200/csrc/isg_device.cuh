// Device-side plan of one MLFMA operator: FP32 tables in the layouts the
// kernels read, plus per-call launch helpers.  Everything here is built from
// the FP64 HostTables by isg_context.cu.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace isg {

constexpr int kMaxLevels = 12;
constexpr int kBox = 8;
constexpr int kBB = 64;  // pixels per leaf
// Kernels put one RHS per grid row (gridDim.y or .z), so no batch may exceed this.
constexpr int kMaxGridY = 65535;

// A banded resampling (interpolation or anterpolation) cut into tiles of `out`
// consecutive output samples (a multiple of kTileOut, the outputs one thread
// accumulates): tile t reads the circular window of wl[t] input samples
// starting at a0[t], with weights w[t][jj][i] (jj < wmax, zero padded)
// relative to that window.
constexpr int kTileOut = 8;
struct TileBand {
  float *w = nullptr;  // [tiles][wmax][out]
  int *a0 = nullptr, *wl = nullptr;
  int2 *span = nullptr;  // [tiles][out / kTileOut]: window rows [x, y) where a thread's kTileOut outputs have taps
  int tiles = 0, wmax = 0, out = kTileOut;
};

// Per-level device tables.  Level numbering is the reference's (0 = root).
struct DevLevel {
  int n = 0;        // clusters per side (2^level)
  int ns = 0;       // angular samples
  size_t off = 0;   // element offset of this level inside one RHS's multipole block
  // interpolation from level+1 (children) into this level: taps (first + t) mod ns_{level+1}
  int *ifirst = nullptr;   // [ns]
  float *iw = nullptr;     // [ninter][ns]
  float2 *shm = nullptr;   // [4][ns] multipole shift child -> this level
  float2 *shl = nullptr;   // [4][ns] local shift this level -> child
  // anterpolation from level-1 (parent) into this level: taps (first + t) mod ns_{level-1}
  int *afirst = nullptr;   // [ns]
  float *aw = nullptr;     // [awidth][ns]
  int awidth = 0;
  float2 *T = nullptr;     // [49][ns] translation operators (level >= 2)
  TileBand mt;             // interpolation into this level (M2M), tiled
  TileBand at;             // anterpolation into this level (L2L), tiled
  float2 *shmT = nullptr;  // [ns][4] shm transposed
  float2 *shlT = nullptr;  // [ns][4] shl transposed
  // launch shapes picked by isg_autotune (0: the built-in choice)
  int m2l_ty = 0;    // sibling-group rows per M2L thread
  int l2l_cols = 0;  // columns per L2L tile block
  int m2m_cols = 0;  // columns per M2M tile block
};

struct DevPlan {
  int L = 0, side = 0, nleaf = 0, U = 0, ninter = 0, numrx = 0;
  int ns_leaf = 0;
  double res = 0.1;
  float2 *nearW = nullptr;   // [9][64 basis][64 testing]
  float2 *coeffT = nullptr;  // [64 pixel][ns_leaf]
  float2 *basisT = nullptr;  // [ns_leaf][64 pixel]
  DevLevel lv[kMaxLevels];
  size_t mp = 0;             // multipole elements per RHS over all levels
  int *hfirst = nullptr;     // [numrx]
  float *hw = nullptr;       // [ninter][numrx]
  int *hind = nullptr;       // [ns_0][hwidth]
  float *haw = nullptr;      // [ns_0][hwidth]
  int hwidth = 0;
  int tuned_nrhs = 0;         // batch the tuned shapes were timed on; they apply from a quarter of it
  float2 *zeros = nullptr;    // [max ns] zeros: what a clipped M2L column reads
  int *perm_tree = nullptr;   // blocked index -> tree index
  int *perm_raster = nullptr; // blocked index -> raster index
};

// How the operator input is formed from the caller's vector.
enum InMode { IN_PLAIN = 0, IN_G = 1, IN_CONJ = 2 };
// What the near-field kernel writes.
enum EpiMode { EPI_G = 0, EPI_FWD = 1, EPI_ADJ = 2, EPI_L2P_ONLY = 3, EPI_CONJ = 4 };
// Which FP64 partial sums the near-field kernel emits per RHS.
enum RedMode { RED_NONE = 0, RED_DOT = 1, RED_TS = 2 };

__host__ __device__ inline float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ inline float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ inline float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ inline float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
// acc += a * b
__device__ __forceinline__ void cfma(float2 &acc, float2 a, float2 b) {
  acc.x = fmaf(a.x, b.x, acc.x);
  acc.x = fmaf(-a.y, b.y, acc.x);
  acc.y = fmaf(a.x, b.y, acc.y);
  acc.y = fmaf(a.y, b.x, acc.y);
}
// Packed FP32 pairs (fma/mul .f32x2, sm_100): one instruction does both halves.
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 pk2(float a, float b) {
  f32x2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ float2 upk2(f32x2 r) {
  float2 a;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
  return a;
}
__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c) {
  f32x2 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ f32x2 mul2(f32x2 a, f32x2 b) {
  f32x2 d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
// acc += w * b (real weight)
__device__ __forceinline__ void rfma(float2 &acc, float w, float2 b) {
  acc.x = fmaf(w, b.x, acc.x);
  acc.y = fmaf(w, b.y, acc.y);
}

__device__ __forceinline__ float2 load_in(const float2 *__restrict__ x, const float2 *__restrict__ g, int mode,
                                          size_t i, size_t gi) {
  float2 v = x[i];
  if (mode == IN_G) return cmul(g[gi], v);
  if (mode == IN_CONJ) return cconj(v);
  return v;
}

// Arguments shared by the leaf kernels for one batch.
struct BatchArgs {
  const float2 *x = nullptr;   // [R][U] blocked
  const float2 *g = nullptr;   // contrast (may be null for IN_PLAIN)
  int64_t gstride = 0;         // elements between consecutive RHS contrasts
  int mode = IN_PLAIN;
  int nrhs = 0;
  const int *active = nullptr; // per-RHS mask (null = all active)
};

// Process-wide count of kernel launches issued by this library.
void count_launch(int n = 1);
int64_t launch_count();
// Non-null: this thread's launches go to *sink (graph capture); null: back to the count.
void capture_launches(int64_t *sink);
// Per-device kernel attributes (isg_kernels.cu), called by isg_setup_gpu.
cudaError_t kernels_setup();
// Loads the kernels of the receiver projection (permute, P2M, M2M, receiver
// interpolation) into the current device's context now, not at their first launch.
cudaError_t aggregate_kernels_load();

// ---- launchers (isg_kernels.cu) ----
void launch_p2m(const DevPlan &P, const BatchArgs &B, float2 *mul, cudaStream_t st);
void launch_m2m(const DevPlan &P, int lvl, float2 *mul, int nrhs, const int *active, cudaStream_t st);
// M2L into level lvl: written over its local expansions, or added to them.
void launch_m2l(const DevPlan &P, int lvl, const float2 *mul, float2 *loc, int nrhs, const int *active, bool accumulate,
                cudaStream_t st,
                unsigned *locmax = nullptr);
// L2L from level lvl-1 into level lvl, written over its locals.
void launch_l2l(const DevPlan &P, int lvl, float2 *loc, int nrhs, const int *active, cudaStream_t st);
// y = epilogue(L2P(loc_leaf) + near(x)); optional FP64 partials per block.
struct NearArgs {
  BatchArgs in;
  const float2 *loc = nullptr;  // leaf-level locals base (per-RHS stride P.mp)
  float2 *y = nullptr;          // [R][U]
  int epi = EPI_G;
  int red = RED_NONE;
  const float2 *dot_a = nullptr;  // RED_DOT: partial of sum conj(a) * y
  double *part = nullptr;         // [R][nblocks][4]
  const float2 *x_epi = nullptr;  // x of the `x - ...` epilogue when in.x already holds g x (else in.x)
  const unsigned *locmax = nullptr;  // tensor engine: per-RHS level maxima of the locals, written by M2L
  const unsigned *inmax = nullptr;   // tensor engine: [R][kMaxLevels] whose last slot holds the input's
                                     // maximum per RHS, written by the tensor-core P2M of the same matvec
};
int near_blocks_per_rhs(const DevPlan &P);
void launch_near(const DevPlan &P, const NearArgs &A, cudaStream_t st);
void launch_rx_interp(const DevPlan &P, const float2 *mul, float2 *rx, int nrhs, cudaStream_t st);
void launch_rx_anterp(const DevPlan &P, const float2 *rx, float2 *loc, int nrhs, float2 scale, cudaStream_t st);
void launch_permute(const int *perm, const float2 *in, float2 *out, int U, int nrhs, bool gather, cudaStream_t st);

}  // namespace isg
