// Batched BiCGSTAB (bicgs_gpu.cu:116-224, bicgs.cpp:88-179) with every scalar
// kept on the device in FP64, per-RHS convergence masks, and the dot products
// fused into the producing kernels.  The host only polls an active-RHS counter
// every `check_every` iterations.
#include <algorithm>
#include <cmath>
#include <vector>

#include "isg_context.hpp"

namespace isg {

namespace {

__device__ __forceinline__ bool inactive(const int *active, int rhs) { return active && !active[rhs]; }

__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  const double d = b.x * b.x + b.y * b.y;
  return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}
__device__ __forceinline__ double2 dmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 f2(double2 a) { return make_float2((float)a.x, (float)a.y); }
__device__ __forceinline__ double2 ld2(const double *p) { return make_double2(p[0], p[1]); }
__device__ __forceinline__ void st2(double *p, double2 v) {
  p[0] = v.x;
  p[1] = v.y;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sums up to three partials per thread over a 256-thread block into s[0..2]
// in a fixed order; thread 0 gets the block totals.
__device__ void block_sum3(double a, double b, double c, double *out) {
  __shared__ double ws[8][3];
  a = warp_sum(a);
  b = warp_sum(b);
  c = warp_sum(c);
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    ws[w][0] = a;
    ws[w][1] = b;
    ws[w][2] = c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s0 = 0, s1 = 0, s2 = 0;
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) {
      s0 += ws[q][0];
      s1 += ws[q][1];
      s2 += ws[q][2];
    }
    out[0] = s0;
    out[1] = s1;
    out[2] = s2;
  }
  __syncthreads();
}

// Per-RHS total of `nb` block partials (4 doubles each), deterministic.
__device__ void sum_partials(const double *part, int rhs, int nb, double *tot) {
  double a = 0, b = 0, c = 0;
  const double *p = part + (size_t)rhs * nb * 4;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) {
    a += p[i * 4 + 0];
    b += p[i * 4 + 1];
    c += p[i * 4 + 2];
  }
  __shared__ double t[3];
  block_sum3(a, b, c, t);
  tot[0] = t[0];
  tot[1] = t[1];
  tot[2] = t[2];
}

__device__ void write_part(double *part, int rhs, int nb, double a, double b, double c) {
  __shared__ double t[3];
  block_sum3(a, b, c, t);
  if (threadIdx.x == 0) {
    double *p = part + ((size_t)rhs * nb + blockIdx.x) * 4;
    p[0] = t[0];
    p[1] = t[1];
    p[2] = t[2];
    p[3] = 0;
  }
}

// Initial residual: r = b (zero guess) or r = b - Ax (Ax in t); r~ = r.
// Partials: ||b||^2, ||r||^2.
__global__ void __launch_bounds__(256) k_init(const float2 *__restrict__ b, const float2 *__restrict__ t,
                                              float2 *__restrict__ x, float2 *__restrict__ r, float2 *__restrict__ rt,
                                              int U, int zero_guess, double *part) {
  const int rhs = blockIdx.y;
  const size_t base = (size_t)rhs * U;
  double bb = 0, rr = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < U; i += gridDim.x * blockDim.x) {
    const float2 bv = b[base + i];
    float2 rv = bv;
    if (zero_guess)
      x[base + i] = make_float2(0.f, 0.f);
    else
      rv = csub(bv, t[base + i]);
    r[base + i] = rv;
    rt[base + i] = rv;
    bb += (double)bv.x * bv.x + (double)bv.y * bv.y;
    rr += (double)rv.x * rv.x + (double)rv.y * rv.y;
  }
  write_part(part, rhs, gridDim.x, bb, rr, 0);
}

__global__ void __launch_bounds__(256) k_fin_init(RhsState *st, int *active, int *count, const double *part, int nb,
                                                  int zero_guess, double tol) {
  const int rhs = blockIdx.x;
  double tot[3];
  sum_partials(part, rhs, nb, tot);
  if (threadIdx.x) return;
  RhsState &s = st[rhs];
  double bn = sqrt(tot[0]);
  if (bn < 1e-20) bn = 1;
  s.bn = bn;
  s.err = sqrt(tot[1]) / bn;
  s.tres = -1;
  s.target = tol;
  s.rho[0] = tot[1];
  s.rho[1] = 0;
  s.rho1[0] = s.rho1[1] = 0;
  s.alpha[0] = s.alpha[1] = 0;
  s.omega[0] = s.omega[1] = 0;
  s.iter = 0;
  s.matvecs = zero_guess ? 0 : 1;
  s.fresh = 1;
  s.restarts = 0;
  if (!isfinite(s.err)) {
    s.status = ISG_NONFINITE;
    s.active = 0;
  } else if (s.err > tol) {
    s.status = ISG_NOT_CONVERGED;
    s.active = 1;
  } else {
    s.status = ISG_OK;
    s.active = 0;
  }
  active[rhs] = s.active;
  if (s.active) atomicAdd(count, 1);
}

// p = r (first iteration) or p = r + beta (p - omega v), beta = (rho/rho1)(alpha/omega)
// (bicgs.cpp:132-139).
// With gp: also gp = g p, the input of the forward matvec that follows.
__global__ void __launch_bounds__(256) k_update_p(const RhsState *st, const int *active, const float2 *__restrict__ r,
                                                  float2 *__restrict__ p, const float2 *__restrict__ v, int U,
                                                  const float2 *__restrict__ g, int64_t gstride,
                                                  float2 *__restrict__ gp) {
  const int rhs = blockIdx.y;
  if (inactive(active, rhs)) return;
  const RhsState &s = st[rhs];
  const size_t base = (size_t)rhs * U;
  const float2 *gr = g + rhs * gstride;
  const bool fresh = s.fresh;
  const double2 beta = fresh ? make_double2(0.0, 0.0) : dmul(cdiv(ld2(s.rho), ld2(s.rho1)), cdiv(ld2(s.alpha), ld2(s.omega)));
  const float2 bf = f2(beta), of = fresh ? make_float2(0.f, 0.f) : f2(ld2(s.omega));
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < U; i += gridDim.x * blockDim.x) {
    float2 pn = r[base + i];
    if (!fresh) pn = cadd(pn, cmul(bf, csub(p[base + i], cmul(of, v[base + i]))));
    p[base + i] = pn;
    if (gp) gp[base + i] = cmul(gr[i], pn);
  }
}

// alpha = rho / <r~, v> (bicgs.cpp:145).
__global__ void __launch_bounds__(256) k_fin_alpha(RhsState *st, int *active, const double *part, int nb) {
  const int rhs = blockIdx.x;
  if (!active[rhs]) return;
  double tot[3];
  sum_partials(part, rhs, nb, tot);
  if (threadIdx.x) return;
  RhsState &s = st[rhs];
  const double2 a = cdiv(ld2(s.rho), make_double2(tot[0], tot[1]));
  st2(s.alpha, a);
  s.matvecs++;
  s.fresh = 0;
  if (!isfinite(a.x) || !isfinite(a.y)) {
    s.status = ISG_NONFINITE;
    s.active = 0;
    active[rhs] = 0;
  }
}

// s = r - alpha v (bicgs.cpp:146).
// With gsv: also gsv = g s, the input of the forward matvec that follows.
__global__ void __launch_bounds__(256) k_update_s(const RhsState *st, const int *active, const float2 *__restrict__ r,
                                                  const float2 *__restrict__ v, float2 *__restrict__ s, int U,
                                                  const float2 *__restrict__ g, int64_t gstride,
                                                  float2 *__restrict__ gsv) {
  const int rhs = blockIdx.y;
  if (inactive(active, rhs)) return;
  const float2 a = f2(ld2(st[rhs].alpha));
  const size_t base = (size_t)rhs * U;
  const float2 *gr = g + rhs * gstride;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < U; i += gridDim.x * blockDim.x) {
    const float2 sv = csub(r[base + i], cmul(a, v[base + i]));
    s[base + i] = sv;
    if (gsv) gsv[base + i] = cmul(gr[i], sv);
  }
}

// omega = <t, s> / ||t||^2 (bicgs.cpp:153); zero when t vanishes, which only
// happens when s itself is zero (bicgs_gpu.cu:197 guards the same case).
__global__ void __launch_bounds__(256) k_fin_omega(RhsState *st, const int *active, const double *part, int nb) {
  const int rhs = blockIdx.x;
  if (!active[rhs]) return;
  double tot[3];
  sum_partials(part, rhs, nb, tot);
  if (threadIdx.x) return;
  RhsState &s = st[rhs];
  s.matvecs++;
  if (tot[2] > 0) {
    s.omega[0] = tot[0] / tot[2];
    s.omega[1] = tot[1] / tot[2];
  } else {
    s.omega[0] = s.omega[1] = 0;
  }
}

// x += alpha p + omega s; r = s - omega t (bicgs.cpp:155-159); partials
// ||r||^2 and <r~, r> for the convergence test and the next rho.
__global__ void __launch_bounds__(256) k_update_xr(const RhsState *st, const int *active, float2 *__restrict__ x,
                                                   float2 *__restrict__ r, const float2 *__restrict__ rt,
                                                   const float2 *__restrict__ p, const float2 *__restrict__ s,
                                                   const float2 *__restrict__ t, int U, double *part) {
  const int rhs = blockIdx.y;
  if (inactive(active, rhs)) return;
  const float2 a = f2(ld2(st[rhs].alpha)), o = f2(ld2(st[rhs].omega));
  const size_t base = (size_t)rhs * U;
  double rr = 0, dr = 0, di = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < U; i += gridDim.x * blockDim.x) {
    const float2 sv = s[base + i];
    x[base + i] = cadd(x[base + i], cadd(cmul(a, p[base + i]), cmul(o, sv)));
    const float2 rv = csub(sv, cmul(o, t[base + i]));
    r[base + i] = rv;
    const float2 q = rt[base + i];
    rr += (double)rv.x * rv.x + (double)rv.y * rv.y;
    dr += (double)q.x * rv.x + (double)q.y * rv.y;
    di += (double)q.x * rv.y - (double)q.y * rv.x;
  }
  write_part(part, rhs, gridDim.x, rr, dr, di);
}

// Convergence and breakdown tests of one iteration (bicgs.cpp:160-169, 127-131).
__global__ void __launch_bounds__(256) k_fin_iter(RhsState *st, int *active, int *count, const double *part, int nb,
                                                  double tol, int maxit) {
  const int rhs = blockIdx.x;
  if (!active[rhs]) return;
  double tot[3];
  sum_partials(part, rhs, nb, tot);
  if (threadIdx.x) return;
  RhsState &s = st[rhs];
  s.iter++;
  s.err = sqrt(tot[0]) / s.bn;
  const double om = hypot(s.omega[0], s.omega[1]);
  const double rho_new = hypot(tot[1], tot[2]);
  int stop = 0;
  if (!isfinite(s.err)) {
    s.status = ISG_NONFINITE;
    stop = 1;
  } else if (s.err < s.target) {
    s.status = ISG_OK;
    stop = 1;
  } else if (om < 1e-20) {
    s.status = ISG_BREAKDOWN;
    stop = 1;
  } else if (s.iter >= maxit) {
    s.status = ISG_NOT_CONVERGED;
    stop = 1;
  } else if (rho_new < 1e-20) {
    s.status = ISG_BREAKDOWN;
    stop = 1;
  }
  s.rho1[0] = s.rho[0];
  s.rho1[1] = s.rho[1];
  s.rho[0] = tot[1];
  s.rho[1] = tot[2];
  if (stop) {
    s.active = 0;
    active[rhs] = 0;
  } else {
    atomicAdd(count, 1);
  }
}

// True residual b - A x (A x in t) into r and r~, partial ||.||^2.
__global__ void __launch_bounds__(256) k_true_res(const float2 *__restrict__ b, const float2 *__restrict__ t,
                                                  float2 *__restrict__ r, float2 *__restrict__ rt, int U,
                                                  double *part) {
  const int rhs = blockIdx.y;
  const size_t base = (size_t)rhs * U;
  double rr = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < U; i += gridDim.x * blockDim.x) {
    const float2 rv = csub(b[base + i], t[base + i]);
    r[base + i] = rv;
    rt[base + i] = rv;
    rr += (double)rv.x * rv.x + (double)rv.y * rv.y;
  }
  write_part(part, rhs, gridDim.x, rr, 0, 0);
}

// Records the true residual and restarts (r = r~ = b - Ax, p = r) every RHS
// that stopped on the recursive residual but misses tol on the true one.  The
// restarted RHS then stops at half its previous recursive target: the FP32
// recurrence drifts from b - Ax by about the same amount again, so stopping
// at tol a second time would land on the same miss.
__global__ void __launch_bounds__(256) k_fin_true(RhsState *st, int *active, int *count, const double *part, int nb,
                                                  double tol, int max_restarts, int maxit) {
  const int rhs = blockIdx.x;
  double tot[3];
  sum_partials(part, rhs, nb, tot);
  if (threadIdx.x) return;
  RhsState &s = st[rhs];
  s.matvecs++;
  s.tres = sqrt(tot[0]) / s.bn;
  if (s.status == ISG_OK && !(s.tres <= tol) && s.restarts < max_restarts && s.iter < maxit) {
    s.restarts++;
    s.target *= 0.5;
    s.status = ISG_NOT_CONVERGED;
    s.active = 1;
    s.fresh = 1;
    s.rho[0] = tot[0];
    s.rho[1] = 0;
    s.err = s.tres;
    active[rhs] = 1;
    atomicAdd(count, 1);
  }
}

}  // namespace

isg_status run_matvec(isg_ctx *c, const float2 *x, const float2 *g, int64_t gs, float2 *y, int nrhs, int kind,
                      int engine, int red, const float2 *dot_a, const int *active, cudaStream_t st,
                      const float2 *gx) {
  const DevPlan &P = c->P;
  BatchArgs B;
  B.x = x;
  B.g = g;
  B.gstride = gs;
  B.nrhs = nrhs;
  B.active = active;
  B.mode = (kind == OP_FWD) ? IN_G : (kind == OP_G ? IN_PLAIN : IN_CONJ);
  const bool tc = (engine == ISG_ENGINE_TENSOR) && tc_available(c);
  if (engine == ISG_ENGINE_TENSOR && !tc) return ISG_UNSUPPORTED;
  // the tensor leaf kernels read g x directly when the caller already formed it
  BatchArgs Bg = B;
  const bool pre = tc && gx && kind == OP_FWD;
  if (pre) {
    Bg.x = gx;
    Bg.g = nullptr;
    Bg.gstride = 0;
    Bg.mode = IN_PLAIN;
  }
  if (tc) {
    cudaMemsetAsync(c->levmax, 0, (size_t)nrhs * kMaxLevels * sizeof(unsigned), st);
    cudaMemsetAsync(c->locmax, 0, (size_t)nrhs * kMaxLevels * sizeof(unsigned), st);
    isg_status e = tc_p2m(c, Bg, c->mul, st);
    if (e != ISG_OK) return e;
  } else {
    launch_p2m(P, B, c->mul, st);
  }
  isg_status be = ISG_OK;
  for (int i = P.L - 2; i >= 2; i--)
    if (!(tc && band_m2m(c, i, c->mul, nrhs, active, st, &be))) launch_m2m(P, i, c->mul, nrhs, active, st);
  if (be != ISG_OK) return be;
  // level by level: the parent's locals anterpolated over the level (L2L),
  // then the level's own far-field translations added (M2L)
  for (int i = 2; i < P.L; i++) {
    if (i >= 3 && !(tc && band_l2l(c, i, c->loc, nrhs, active, st, &be))) launch_l2l(P, i, c->loc, nrhs, active, st);
    launch_m2l(P, i, c->mul, c->loc, nrhs, active, i >= 3, st, tc ? c->locmax : nullptr);
  }
  if (be != ISG_OK) return be;
  NearArgs A;
  A.in = pre ? Bg : B;
  A.x_epi = pre ? x : nullptr;
  A.locmax = tc ? c->locmax : nullptr;  // M2L of the leaves wrote it above
  A.inmax = tc ? c->levmax : nullptr;   // and P2M the input's maximum
  A.loc = c->loc;
  A.y = y;
  A.epi = (kind == OP_FWD) ? EPI_FWD : (kind == OP_ADJ ? EPI_ADJ : (kind == OP_GCONJ ? EPI_CONJ : EPI_G));
  A.red = red;
  A.dot_a = dot_a;
  A.part = c->part;
  if (tc) return tc_near(c, A, st);
  launch_near(P, A, st);
  return cuda_check(c, cudaGetLastError(), "matvec launch");
}

namespace {

// One context's batch in a BiCGSTAB solve (bicgs_gpu.cu:116-224,
// bicgs.cpp:88-179): set-up, the block of `check` iterations, the
// true-residual check and the results.  isg_bicgs drives one run;
// isg_bicgs_group drives several contexts' runs together.
struct BicgsRun {
  isg_ctx *c;
  float2 *x;
  const float2 *g, *b;
  int64_t gs;
  int R, kind, engine, nbv, nbn, check, zero_guess;
  const isg_solve_opts *o;
  float2 *gx;  // forward solves on the tensor engine: the updates also write g p and g s

  BicgsRun(isg_ctx *c_, float2 *x_, const float2 *g_, int64_t gs_, const float2 *b_, int R_, int hermitian,
           const isg_solve_opts *o_)
      : c(c_), x(x_), g(g_), b(b_), gs(gs_), R(R_), o(o_) {
    kind = hermitian ? OP_ADJ : OP_FWD;
    engine = o->engine;
    nbv = c->vec_blocks;
    nbn = (engine == ISG_ENGINE_TENSOR && tc_available(c)) ? tc_near_blocks(c) : near_blocks_per_rhs(c->P);
    check = std::max(1, o->check_every);
    zero_guess = o->guess == ISG_GUESS_ZERO;
    gx = (kind == OP_FWD && engine == ISG_ENGINE_TENSOR && tc_available(c)) ? c->vgx : nullptr;
  }
  dim3 vgrid() const { return dim3(nbv, R); }
  long host_cap() const { return (long)(o->maxit + 2) * (o->max_restarts + 1) + 8; }

  isg_status init(cudaStream_t st) {
    if (!zero_guess) {
      isg_status e = run_matvec(c, x, g, gs, c->vt, R, kind, engine, RED_NONE, nullptr, nullptr, st);
      if (e != ISG_OK) return e;
    }
    count_launch();
    k_init<<<vgrid(), 256, 0, st>>>(b, c->vt, x, c->vr, c->vrt, c->P.U, zero_guess, c->part);
    cudaMemsetAsync(c->count, 0, sizeof(int), st);
    count_launch();
    k_fin_init<<<R, 256, 0, st>>>(c->state, c->active, c->count, c->part, nbv, zero_guess, o->tol);
    return cuda_check(c, cudaGetLastError(), "bicgs init");
  }
  // `check` iterations of every active RHS (bicgs.cpp:120-177); inactive ones return at once
  isg_status block(cudaStream_t st) {
    const int U = c->P.U;
    for (int k = 0; k < check; k++) {
      count_launch();
      k_update_p<<<vgrid(), 256, 0, st>>>(c->state, c->active, c->vr, c->vp, c->vv, U, g, gs, gx);
      isg_status be = run_matvec(c, c->vp, g, gs, c->vv, R, kind, engine, RED_DOT, c->vrt, c->active, st, gx);
      if (be != ISG_OK) return be;
      count_launch();
      k_fin_alpha<<<R, 256, 0, st>>>(c->state, c->active, c->part, nbn);
      count_launch();
      k_update_s<<<vgrid(), 256, 0, st>>>(c->state, c->active, c->vr, c->vv, c->vs, U, g, gs, gx);
      be = run_matvec(c, c->vs, g, gs, c->vt, R, kind, engine, RED_TS, nullptr, c->active, st, gx);
      if (be != ISG_OK) return be;
      count_launch();
      k_fin_omega<<<R, 256, 0, st>>>(c->state, c->active, c->part, nbn);
      count_launch();
      k_update_xr<<<vgrid(), 256, 0, st>>>(c->state, c->active, x, c->vr, c->vrt, c->vp, c->vs, c->vt, U, c->part);
      cudaMemsetAsync(c->count, 0, sizeof(int), st);
      count_launch();
      k_fin_iter<<<R, 256, 0, st>>>(c->state, c->active, c->count, c->part, nbv, o->tol, o->maxit);
    }
    return cuda_check(c, cudaGetLastError(), "bicgs iteration");
  }
  void read_count(cudaStream_t st) {
    cudaMemcpyAsync(c->h_count, c->count, sizeof(int), cudaMemcpyDeviceToHost, st);
  }
  // True residual b - A x of every RHS; restarts any that stopped early (k_fin_true).
  isg_status true_residual(cudaStream_t st) {
    isg_status e = run_matvec(c, x, g, gs, c->vt, R, kind, engine, RED_NONE, nullptr, nullptr, st);
    if (e != ISG_OK) return e;
    count_launch();
    k_true_res<<<vgrid(), 256, 0, st>>>(b, c->vt, c->vr, c->vrt, c->P.U, c->part);
    cudaMemsetAsync(c->count, 0, sizeof(int), st);
    count_launch();
    k_fin_true<<<R, 256, 0, st>>>(c->state, c->active, c->count, c->part, nbv, o->tol, o->max_restarts, o->maxit);
    read_count(st);
    return ISG_OK;
  }
  isg_status results(isg_solve_info *info, cudaStream_t st) {
    std::vector<RhsState> hs(R);
    cudaMemcpyAsync(hs.data(), c->state, R * sizeof(RhsState), cudaMemcpyDeviceToHost, st);
    isg_status e = cuda_check(c, cudaStreamSynchronize(st), "bicgs results");
    if (e != ISG_OK) return e;
    if (engine == ISG_ENGINE_TENSOR && tc_error(c)) {
      c->err = "a tensor-core kernel hit its wait limit";
      return ISG_TIMEOUT;
    }
    isg_status worst = ISG_OK;
    for (int r = 0; r < R; r++) {
      if (info) {
        info[r].iterations = hs[r].iter;
        info[r].matvecs = hs[r].matvecs;
        info[r].status = hs[r].status;
        info[r].restarts = hs[r].restarts;
        info[r].residual = hs[r].err;
        info[r].true_residual = hs[r].tres;
      }
      if (hs[r].status != ISG_OK && (worst == ISG_OK || hs[r].status > worst)) worst = (isg_status)hs[r].status;
    }
    return worst;
  }
};

bool capturable(const isg_solve_opts *o, cudaStream_t st) {
  return o->graph && st != nullptr && st != cudaStreamLegacy && st != cudaStreamPerThread;
}

}  // namespace

isg_status run_bicgs(isg_ctx *c, float2 *x, const float2 *g, int64_t gs, const float2 *b, int R, int hermitian,
                     const isg_solve_opts *o, isg_solve_info *info, cudaStream_t st) {
  BicgsRun run(c, x, g, gs, b, R, hermitian, o);
  isg_status e = run.init(st);
  if (e != ISG_OK) return e;
  const long host_cap = run.host_cap();
  long host_iters = 0;
  // The block's launches depend only on the pointers and sizes below, so it is
  // captured once and replayed (not on the legacy default stream, which cannot
  // be captured); the executable graph is cached in the context.
  isg_ctx::GraphKey key;
  key.x = x;
  key.g = g;
  key.gs = gs;
  key.R = R;
  key.kind = run.kind;
  key.engine = run.engine;
  key.check = run.check;
  key.maxit = o->maxit;
  key.tol = o->tol;
  auto replay = [&]() -> isg_status {
    if (!(c->graph_exec && c->graph_key == key)) {
      if (c->graph_exec) cudaGraphExecDestroy((cudaGraphExec_t)c->graph_exec);
      c->graph_exec = nullptr;
      int64_t captured = 0;
      isg_status ce = cuda_check(c, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "graph capture");
      if (ce != ISG_OK) return ce;
      capture_launches(&captured);
      isg_status be = run.block(st);
      capture_launches(nullptr);
      cudaGraph_t gr = nullptr;
      ce = cuda_check(c, cudaStreamEndCapture(st, &gr), "graph capture end");
      if (be != ISG_OK || ce != ISG_OK) {
        if (gr) cudaGraphDestroy(gr);
        return be != ISG_OK ? be : ce;
      }
      cudaGraphExec_t ex = nullptr;
      ce = cuda_check(c, cudaGraphInstantiate(&ex, gr, 0), "graph instantiate");
      cudaGraphDestroy(gr);
      if (ce != ISG_OK) return ce;
      c->graph_exec = ex;
      c->graph_key = key;
      c->graph_launches = captured;
    }
    count_launch((int)c->graph_launches);
    return cuda_check(c, cudaGraphLaunch((cudaGraphExec_t)c->graph_exec, st), "graph launch");
  };
  const bool want_graph = capturable(o, st);
  for (;;) {
    run.read_count(st);
    if ((e = cuda_check(c, cudaStreamSynchronize(st), "bicgs poll")) != ISG_OK) return e;
    if (*c->h_count > 0 && host_iters < host_cap) {
      if ((e = want_graph ? replay() : run.block(st)) != ISG_OK) return e;
      host_iters += run.check;
      continue;
    }
    if (!o->true_residual) break;
    if ((e = run.true_residual(st)) != ISG_OK) return e;
    if ((e = cuda_check(c, cudaStreamSynchronize(st), "bicgs true residual")) != ISG_OK) return e;
    if (*c->h_count == 0 || host_iters >= host_cap) break;
  }
  return run.results(info, st);
}

// Several contexts' batches solved together (same device, same options).  One
// host poll reads every member's active count; each block of `check`
// iterations of all members is one CUDA graph whose branches are the members'
// iteration blocks on forked streams (joined back on st), captured once per
// call and launched once per poll.  The true-residual checks run member after
// member on st.  Results go to each member's info; returns the worst status.
isg_status run_bicgs_group(int n, isg_ctx *const *cs, float2 *const *xs, const float2 *const *gs_, const int64_t *gss,
                           const float2 *const *bs, const int *Rs, int hermitian, const isg_solve_opts *o,
                           isg_solve_info *const *infos, cudaStream_t st) {
  std::vector<BicgsRun> runs;
  runs.reserve(n);
  for (int i = 0; i < n; i++) runs.emplace_back(cs[i], xs[i], gs_[i], gss[i], bs[i], Rs[i], hermitian, o);
  isg_ctx *c0 = cs[0];
  isg_status e = ISG_OK;
  for (auto &r : runs)
    if ((e = r.init(st)) != ISG_OK) return e;
  long host_cap = 0;
  for (auto &r : runs) host_cap = std::max(host_cap, r.host_cap());
  long host_iters = 0;
  std::vector<cudaStream_t> side(n, nullptr);
  std::vector<cudaEvent_t> join(n, nullptr);
  cudaEvent_t fork = nullptr;
  cudaGraphExec_t exec = nullptr;
  int64_t captured = 0;
  auto cleanup = [&]() {
    if (exec) cudaGraphExecDestroy(exec);
    for (int i = 0; i < n; i++) {
      if (join[i]) cudaEventDestroy(join[i]);
      if (side[i]) cudaStreamDestroy(side[i]);
    }
    if (fork) cudaEventDestroy(fork);
  };
  const bool want_graph = capturable(o, st);
  auto step = [&]() -> isg_status {
    if (!want_graph) {
      for (auto &r : runs)
        if ((e = r.block(st)) != ISG_OK) return e;
      return ISG_OK;
    }
    if (!exec) {
      isg_status ce = cuda_check(c0, cudaEventCreateWithFlags(&fork, cudaEventDisableTiming), "group event");
      for (int i = 0; i < n && ce == ISG_OK; i++) {
        ce = cuda_check(c0, cudaStreamCreateWithFlags(&side[i], cudaStreamNonBlocking), "group stream");
        if (ce == ISG_OK) ce = cuda_check(c0, cudaEventCreateWithFlags(&join[i], cudaEventDisableTiming), "group event");
      }
      if (ce != ISG_OK) return ce;
      if ((ce = cuda_check(c0, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "group capture")) != ISG_OK)
        return ce;
      capture_launches(&captured);
      isg_status be = cuda_check(c0, cudaEventRecord(fork, st), "group fork");
      for (int i = 0; i < n && be == ISG_OK; i++) {
        be = cuda_check(c0, cudaStreamWaitEvent(side[i], fork, 0), "group fork");
        if (be == ISG_OK) be = runs[i].block(side[i]);
        if (be == ISG_OK) be = cuda_check(c0, cudaEventRecord(join[i], side[i]), "group join");
        if (be == ISG_OK) be = cuda_check(c0, cudaStreamWaitEvent(st, join[i], 0), "group join");
      }
      capture_launches(nullptr);
      cudaGraph_t gr = nullptr;
      ce = cuda_check(c0, cudaStreamEndCapture(st, &gr), "group capture end");
      if (be != ISG_OK || ce != ISG_OK) {
        if (gr) cudaGraphDestroy(gr);
        return be != ISG_OK ? be : ce;
      }
      ce = cuda_check(c0, cudaGraphInstantiate(&exec, gr, 0), "group instantiate");
      cudaGraphDestroy(gr);
      if (ce != ISG_OK) return ce;
    }
    count_launch((int)captured);
    return cuda_check(c0, cudaGraphLaunch(exec, st), "group graph launch");
  };
  auto active = [&]() {
    long t = 0;
    for (auto &r : runs) t += *r.c->h_count;
    return t;
  };
  for (;;) {
    for (auto &r : runs) r.read_count(st);
    if ((e = cuda_check(c0, cudaStreamSynchronize(st), "group poll")) != ISG_OK) break;
    if (active() > 0 && host_iters < host_cap) {
      if ((e = step()) != ISG_OK) break;
      host_iters += runs[0].check;
      continue;
    }
    if (!o->true_residual) break;
    for (auto &r : runs)
      if ((e = r.true_residual(st)) != ISG_OK) break;
    if (e != ISG_OK) break;
    if ((e = cuda_check(c0, cudaStreamSynchronize(st), "group true residual")) != ISG_OK) break;
    if (active() == 0 || host_iters >= host_cap) break;
  }
  cleanup();
  if (e != ISG_OK) return e;
  isg_status worst = ISG_OK;
  for (int i = 0; i < n; i++) {
    const isg_status ri = runs[i].results(infos ? infos[i] : nullptr, st);
    if (ri == ISG_CUDA_ERROR || ri == ISG_TIMEOUT) return ri;
    if (ri != ISG_OK && (worst == ISG_OK || ri > worst)) worst = ri;
  }
  return worst;
}

}  // namespace isg
