// The inversion loop of the reference driver (mom.cpp:222-399, with the
// measurement synthesis of setup_born.cpp:139-168 and the metrics of
// write_error, setup_born.cpp:171-242), device-resident and batched over
// transmitters.  The contrast, gradient and search direction are complex128;
// the per-transmitter fields are complex64; every reduction is FP64.  The
// small receiver-side arrays (numrx per transmitter) are reduced on the host.
#include <algorithm>
#include <cmath>
#include <complex>
#include <random>
#include <vector>

#include <cstdio>
#include <string>

#include "isg_context.hpp"

namespace isg {

namespace {

using zd = std::complex<double>;

__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__global__ void k_permute_z(const int *__restrict__ perm, const double2 *__restrict__ in, double2 *__restrict__ out,
                            int U, int gather) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < U; i += gridDim.x * blockDim.x) {
    if (gather)
      out[i] = in[perm[i]];
    else
      out[perm[i]] = in[i];
  }
}

// g = k0^2 chi (mom.cpp:289)
__global__ void k_g_of_chi(const double2 *__restrict__ o, double k2, float2 *__restrict__ g, int U) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < U; i += gridDim.x * blockDim.x)
    g[i] = make_float2((float)(o[i].x * k2), (float)(o[i].y * k2));
}

// C = conj(g) Y (mom.cpp:253)
__global__ void k_conj_g_mul(const float2 *__restrict__ g, const float2 *__restrict__ Y, float2 *__restrict__ C, int U) {
  const size_t r = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < U; i += gridDim.x * blockDim.x)
    C[r * U + i] = cmul(cconj(g[i]), Y[r * U + i]);
}

// x = conj(y) per RHS
__global__ void k_conj_copy(const float2 *__restrict__ y, float2 *__restrict__ x, int U) {
  const size_t r = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < U; i += gridDim.x * blockDim.x) x[r * U + i] = cconj(y[r * U + i]);
}

// x = conj(g x) per RHS
__global__ void k_conj_g_times(const float2 *__restrict__ g, float2 *__restrict__ x, int U) {
  const size_t r = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < U; i += gridDim.x * blockDim.x)
    x[r * U + i] = cconj(cmul(g[i], x[r * U + i]));
}

// Y += C (mom.cpp:262)
__global__ void k_add(float2 *__restrict__ Y, const float2 *__restrict__ C, int U) {
  const size_t r = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < U; i += gridDim.x * blockDim.x)
    Y[r * U + i] = cadd(Y[r * U + i], C[r * U + i]);
}

// od += sum_r conj(tot_r) Y_r + R regular^2 o (mom.cpp:263-269)
__global__ void k_grad_accum(const float2 *__restrict__ tot, const float2 *__restrict__ Y, const double2 *__restrict__ o,
                             double reg2, double2 *__restrict__ od, int U, int R) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < U; i += gridDim.x * blockDim.x) {
    double2 acc = od[i];
    for (int r = 0; r < R; r++) {
      const float2 t = tot[(size_t)r * U + i], y = Y[(size_t)r * U + i];
      acc.x += (double)t.x * y.x + (double)t.y * y.y;
      acc.y += (double)t.x * y.y - (double)t.y * y.x;
      acc.x += reg2 * o[i].x;
      acc.y += reg2 * o[i].y;
    }
    od[i] = acc;
  }
}

// Y = tot ot k0^2 (mom.cpp:284)
__global__ void k_born(const float2 *__restrict__ tot, const double2 *__restrict__ ot, double k2,
                       float2 *__restrict__ Y, int U) {
  const size_t r = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < U; i += gridDim.x * blockDim.x) {
    const float2 t = tot[r * U + i];
    const float2 s = make_float2((float)(ot[i].x * k2), (float)(ot[i].y * k2));
    Y[r * U + i] = cmul(t, s);
  }
}

// Y = Y + g X (mom.cpp:301), or Y = g X when overwrite (mom.cpp:331, setup_born.cpp:146)
__global__ void k_gx(float2 *__restrict__ Y, const float2 *__restrict__ g, const float2 *__restrict__ X, int U,
                     int overwrite) {
  const size_t r = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < U; i += gridDim.x * blockDim.x) {
    const float2 v = cmul(g[i], X[r * U + i]);
    Y[r * U + i] = overwrite ? v : cadd(Y[r * U + i], v);
  }
}

// o -= alpha ot (mom.cpp:320); ot = od + beta ot (mom.cpp:399)
__global__ void k_axpy_z(double2 *__restrict__ y, const double2 *__restrict__ x, double2 a, int U, int mode) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < U; i += gridDim.x * blockDim.x) {
    if (mode == 0) {
      const double2 v = zmul(a, x[i]);
      y[i] = make_double2(y[i].x - v.x, y[i].y - v.y);
    } else {
      const double2 v = zmul(a, y[i]);
      y[i] = make_double2(x[i].x + v.x, x[i].y + v.y);
    }
  }
}

// FP64 sums over U: mode 0 (write_error): |a|^2, |b|^2, |b - c|^2 (c may be null);
// mode 1 (Polak-Ribiere, mom.cpp:388-391): a conj(a - b) (re, im), |b|^2.
__global__ void __launch_bounds__(256) k_sums(const double2 *__restrict__ a, const double2 *__restrict__ b,
                                              const double2 *__restrict__ c, int U, int mode, double *part) {
  double s0 = 0, s1 = 0, s2 = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < U; i += gridDim.x * blockDim.x) {
    const double2 av = a[i], bv = b[i];
    if (mode == 0) {
      s0 += av.x * av.x + av.y * av.y;
      s1 += bv.x * bv.x + bv.y * bv.y;
      if (c) {
        const double dx = bv.x - c[i].x, dy = bv.y - c[i].y;
        s2 += dx * dx + dy * dy;
      }
    } else {
      const double dx = av.x - bv.x, dy = av.y - bv.y;
      s0 += av.x * dx + av.y * dy;
      s1 += av.y * dx - av.x * dy;
      s2 += bv.x * bv.x + bv.y * bv.y;
    }
  }
  __shared__ double ws[8][3];
  for (int o = 16; o > 0; o >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  if ((threadIdx.x & 31) == 0) {
    ws[threadIdx.x >> 5][0] = s0;
    ws[threadIdx.x >> 5][1] = s1;
    ws[threadIdx.x >> 5][2] = s2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t0 = 0, t1 = 0, t2 = 0;
    for (int w = 0; w < 8; w++) {
      t0 += ws[w][0];
      t1 += ws[w][1];
      t2 += ws[w][2];
    }
    part[blockIdx.x * 3 + 0] = t0;
    part[blockIdx.x * 3 + 1] = t1;
    part[blockIdx.x * 3 + 2] = t2;
  }
}

// Device buffers of one inversion call.
struct Dbim {
  isg_ctx *c;
  cudaStream_t st;
  int ntx, U, nrx, R;
  double k2;
  std::vector<void *> allocs;
  float2 *incb = nullptr, *tot = nullptr, *X = nullptr, *Y = nullptr, *C = nullptr, *g = nullptr;
  float2 *rxd = nullptr;  // ntx x nrx receiver-side scratch
  float2 *adj = nullptr;  // ntx x U previous adjoint fields (warm start only)
  bool warm = false;
  double2 *o = nullptr, *od = nullptr, *ot = nullptr, *save = nullptr, *otrue = nullptr;
  double *part = nullptr;
  std::vector<zd> mes, mesd, rhs;
  int64_t solves = 0, iters = 0;
  isg_solve_opts so;

  template <class T>
  isg_status alloc(T **p, size_t n) {
    void *q = nullptr;
    isg_status e = cuda_check(c, cudaMalloc(&q, std::max<size_t>(1, n) * sizeof(T)), "dbim alloc");
    if (e == ISG_OK) {
      allocs.push_back(q);
      *p = (T *)q;
    }
    return e;
  }
  ~Dbim() {
    for (void *p : allocs) cudaFree(p);
  }
  dim3 vgrid(int r = 1) const { return dim3(std::min((U + 255) / 256, 1184), r); }
  int chunk(int k) const { return std::min(R, ntx - k * R); }
  int nchunks() const { return (ntx + R - 1) / R; }

  // guess: ISG_GUESS_ZERO, or ISG_GUESS_CALLER with x holding the start
  isg_status solve(float2 *x, const float2 *b, int n, int hermitian, int guess = ISG_GUESS_ZERO) {
    std::vector<isg_solve_info> info(n);
    isg_solve_opts o = so;
    o.guess = guess;
    if (so.guess == ISG_GUESS_LEARNED && !hermitian && guess == ISG_GUESS_ZERO && c->fno) {
      isg_status e = fno_apply(c, g, 0, b, x, n, ISG_ORDER_BLOCKED, st);
      if (e != ISG_OK) return e;
      o.guess = ISG_GUESS_CALLER;
    }
    isg_status e = run_bicgs(c, x, g, 0, b, n, hermitian, &o, info.data(), st);
    if (e == ISG_CUDA_ERROR || e == ISG_BAD_ARG || e == ISG_UNSUPPORTED || e == ISG_TIMEOUT) return e;
    solves += n;
    for (auto &i : info) iters += i.iterations;
    return ISG_OK;
  }
  // far-field samples of X for transmitters [k R, k R + n), to the host
  isg_status far_field(const float2 *Xs, int k, int n, std::vector<zd> &out) {
    isg_status e = run_receive(c, Xs, rxd, n, st);
    if (e != ISG_OK) return e;
    std::vector<float2> h((size_t)n * nrx);
    cudaMemcpyAsync(h.data(), rxd, h.size() * sizeof(float2), cudaMemcpyDeviceToHost, st);
    if ((e = cuda_check(c, cudaStreamSynchronize(st), "dbim far field")) != ISG_OK) return e;
    for (size_t q = 0; q < h.size(); q++) out[(size_t)k * R * nrx + q] = zd(h[q].x, h[q].y);
    return ISG_OK;
  }
  isg_status set_g() {
    k_g_of_chi<<<vgrid(), 256, 0, st>>>(o, k2, g, U);
    count_launch();
    return cuda_check(c, cudaGetLastError(), "dbim g");
  }
  // mom.cpp:247-271: od = sum over transmitters of conj(tot) (y + mlfmah(x))
  // with y = aggregateh(mesd) and x the adjoint solve with rhs conj(g) y.
  bool warm_ready = false;  // adj holds a previous iteration's adjoint fields
  isg_status gradient(double regular) {
    isg_status e;
    cudaMemsetAsync(od, 0, (size_t)U * sizeof(double2), st);
    std::vector<float2> hm((size_t)R * nrx);
    for (int k = 0; k < nchunks(); k++) {
      const int n = chunk(k);
      for (size_t q = 0; q < (size_t)n * nrx; q++) {
        const zd v = mesd[(size_t)k * R * nrx + q];
        hm[q] = make_float2((float)v.real(), (float)v.imag());
      }
      cudaMemcpyAsync(rxd, hm.data(), (size_t)n * nrx * sizeof(float2), cudaMemcpyHostToDevice, st);
      if ((e = run_receiveh(c, Y, rxd, n, st)) != ISG_OK) return e;
      k_conj_g_mul<<<vgrid(n), 256, 0, st>>>(g, Y, C, U);
      count_launch();
      float2 *xa = warm ? adj + (size_t)k * R * U : X;  // the previous adjoint fields, when kept
      int guess = warm && warm_ready ? ISG_GUESS_CALLER : ISG_GUESS_ZERO;
      if (guess == ISG_GUESS_ZERO && so.guess == ISG_GUESS_LEARNED && c->fno) {
        // The adjoint system x - conj(g G conj(x)) = conj(g) y (the adjoint matvec of bicgs.cpp:62-87)
        // is the forward one in disguise: with z = conj(x) it reads z = g (conj(y) + G z), so
        // x = conj(g w) with (I - G g) w = conj(y), a forward solve whose incident field conj(y) is
        // radiated by sources at the receivers.  The forward network's w0 = N(g, conj(y)) therefore
        // seeds it: x0 = conj(g w0).
        k_conj_copy<<<vgrid(n), 256, 0, st>>>(Y, xa, U);
        count_launch();
        if ((e = fno_apply(c, g, 0, xa, xa, n, ISG_ORDER_BLOCKED, st)) != ISG_OK) return e;
        k_conj_g_times<<<vgrid(n), 256, 0, st>>>(g, xa, U);
        count_launch();
        guess = ISG_GUESS_CALLER;
      }
      if ((e = solve(xa, C, n, 1, guess)) != ISG_OK) return e;
      if (warm) cudaMemcpyAsync(X, xa, (size_t)n * U * sizeof(float2), cudaMemcpyDeviceToDevice, st);
      if ((e = run_matvec(c, X, nullptr, 0, C, n, OP_GCONJ, so.engine, RED_NONE, nullptr, nullptr, st)) != ISG_OK)
        return e;
      k_add<<<vgrid(n), 256, 0, st>>>(Y, C, U);
      k_grad_accum<<<vgrid(), 256, 0, st>>>(tot + (size_t)k * R * U, Y, o, regular * regular, od, U, n);
      count_launch(2);
      if ((e = cuda_check(c, cudaStreamSynchronize(st), "dbim gradient")) != ISG_OK) return e;
    }
    warm_ready = warm;
    return ISG_OK;
  }
  isg_status sums(const double2 *a, const double2 *b, const double2 *cc, int mode, double *out) {
    const int nb = 256;
    k_sums<<<nb, 256, 0, st>>>(a, b, cc, U, mode, part);
    count_launch();
    std::vector<double> h(nb * 3);
    cudaMemcpyAsync(h.data(), part, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st);
    isg_status e = cuda_check(c, cudaStreamSynchronize(st), "dbim sums");
    out[0] = out[1] = out[2] = 0;
    for (int i = 0; i < nb; i++)
      for (int j = 0; j < 3; j++) out[j] += h[i * 3 + j];
    return e;
  }
};

}  // namespace

}  // namespace isg

using namespace isg;

extern "C" {

void isg_default_dbim_opts(isg_dbim_opts *o) {
  if (!o) return;
  o->iterations = 3;
  o->regular = 0.0;
  o->start_from_chi = 0;
  isg_default_solve_opts(&o->solve);
  o->solve.tol = 1e-4;
  o->warm_start = 0;
  o->checkpoint = nullptr;
}

isg_status isg_measure(isg_ctx *c, int ntx, const void *inc, const double *chi, int order, double noise,
                       uint64_t seed, const isg_solve_opts *solve, void *mes, isg_stream stream) {
  if (!c || !inc || !chi || !mes || ntx < 1 || order < 0 || order > 2) return ISG_BAD_ARG;
  isg_status e = c->gpu_ready ? ISG_OK : isg_setup_gpu(c);
  if (e != ISG_OK) return e;
  Dbim D;
  D.c = c;
  D.st = (cudaStream_t)stream;
  D.ntx = ntx;
  D.U = c->P.U;
  D.nrx = c->P.numrx;
  D.R = std::min(ntx, c->opts.max_rhs);
  D.k2 = c->T.k0 * c->T.k0;
  isg_default_solve_opts(&D.so);
  if (solve) D.so = *solve;
  D.so.guess = ISG_GUESS_ZERO;
  const size_t U = D.U;
  if ((e = D.alloc(&D.X, (size_t)D.R * U)) || (e = D.alloc(&D.Y, (size_t)D.R * U)) || (e = D.alloc(&D.g, U)) ||
      (e = D.alloc(&D.o, U)) || (e = D.alloc(&D.rxd, (size_t)D.R * D.nrx)))
    return e;
  const int *perm = order_perm(c, order);
  if (perm) {
    k_permute_z<<<D.vgrid(), 256, 0, D.st>>>(perm, (const double2 *)chi, D.o, D.U, 1);
    count_launch();
  } else {
    cudaMemcpyAsync(D.o, chi, U * sizeof(double2), cudaMemcpyDeviceToDevice, D.st);
  }
  if ((e = D.set_g()) != ISG_OK) return e;
  std::vector<zd> out((size_t)ntx * D.nrx);
  for (int k = 0; k < D.nchunks(); k++) {
    const int n = D.chunk(k);
    const float2 *src = (const float2 *)inc + (size_t)k * D.R * U;
    if (perm) {
      launch_permute(perm, src, D.Y, D.U, n, true, D.st);
      src = D.Y;
    }
    if ((e = D.solve(D.X, src, n, 0)) != ISG_OK) return e;
    k_gx<<<D.vgrid(n), 256, 0, D.st>>>(D.X, D.g, D.X, D.U, 1);
    count_launch();
    if ((e = D.far_field(D.X, k, n, out)) != ISG_OK) return e;
  }
  if (noise > 0) {
    double nrm = 0;
    for (auto &v : out) nrm += std::norm(v);
    const double sigma = noise * std::sqrt(nrm) / std::sqrt(2.0 * out.size());
    std::mt19937_64 gen(seed);
    std::normal_distribution<double> nd(0.0, sigma);
    for (auto &v : out) v += zd(nd(gen), nd(gen));
  }
  std::vector<float2> h(out.size());
  for (size_t q = 0; q < out.size(); q++) h[q] = make_float2((float)out[q].real(), (float)out[q].imag());
  cudaMemcpyAsync(mes, h.data(), h.size() * sizeof(float2), cudaMemcpyHostToDevice, D.st);
  return cuda_check(c, cudaStreamSynchronize(D.st), "measure");
}

isg_status isg_dbim(isg_ctx *c, int ntx, const void *inc, const void *mes, const double *chi_true, double *chi,
                    int order, const isg_dbim_opts *opts, isg_dbim_record *hist, isg_stream stream) {
  if (!c || !inc || !mes || !chi || ntx < 1 || order < 0 || order > 2) return ISG_BAD_ARG;
  isg_status e = c->gpu_ready ? ISG_OK : isg_setup_gpu(c);
  if (e != ISG_OK) return e;
  isg_dbim_opts O;
  isg_default_dbim_opts(&O);
  if (opts) O = *opts;
  if (O.iterations < 0) return ISG_BAD_ARG;
  Dbim D;
  D.c = c;
  D.st = (cudaStream_t)stream;
  D.ntx = ntx;
  D.U = c->P.U;
  D.nrx = c->P.numrx;
  D.R = std::min(ntx, c->opts.max_rhs);
  D.k2 = c->T.k0 * c->T.k0;
  D.so = O.solve;
  if (D.so.guess == ISG_GUESS_CALLER) D.so.guess = ISG_GUESS_ZERO;  // every reference solve starts at 0
  if (D.so.guess == ISG_GUESS_LEARNED && !c->fno) {
    c->err = "ISG_GUESS_LEARNED needs a warm-start network (isg_fno_create)";
    return ISG_UNSUPPORTED;
  }
  D.warm = O.warm_start != 0;
  bool wrote_hist = false;
  const size_t U = D.U, nm = (size_t)ntx * D.nrx;
  if ((e = D.alloc(&D.incb, (size_t)ntx * U)) || (e = D.alloc(&D.tot, (size_t)ntx * U)) ||
      (e = D.alloc(&D.X, (size_t)D.R * U)) || (e = D.alloc(&D.Y, (size_t)D.R * U)) ||
      (e = D.alloc(&D.C, (size_t)D.R * U)) || (e = D.alloc(&D.g, U)) || (e = D.alloc(&D.o, U)) ||
      (e = D.alloc(&D.od, U)) || (e = D.alloc(&D.ot, U)) || (e = D.alloc(&D.save, U)) ||
      (e = D.alloc(&D.rxd, (size_t)D.R * D.nrx)) || (e = D.alloc(&D.part, 256 * 3)))
    return e;
  if (chi_true && (e = D.alloc(&D.otrue, U))) return e;
  if (D.warm && (e = D.alloc(&D.adj, (size_t)ntx * U))) return e;
  const int *perm = order_perm(c, order);
  cudaStream_t st = D.st;
  // inputs into the blocked layout
  if (perm) {
    launch_permute(perm, (const float2 *)inc, D.incb, D.U, ntx, true, st);
    if (chi_true) k_permute_z<<<D.vgrid(), 256, 0, st>>>(perm, (const double2 *)chi_true, D.otrue, D.U, 1);
    k_permute_z<<<D.vgrid(), 256, 0, st>>>(perm, (const double2 *)chi, D.o, D.U, 1);
    count_launch(chi_true ? 2 : 1);
  } else {
    cudaMemcpyAsync(D.incb, inc, (size_t)ntx * U * sizeof(float2), cudaMemcpyDeviceToDevice, st);
    if (chi_true) cudaMemcpyAsync(D.otrue, chi_true, U * sizeof(double2), cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(D.o, chi, U * sizeof(double2), cudaMemcpyDeviceToDevice, st);
  }
  {
    std::vector<float2> hm(nm);
    cudaMemcpyAsync(hm.data(), mes, nm * sizeof(float2), cudaMemcpyDeviceToHost, st);
    if ((e = cuda_check(c, cudaStreamSynchronize(st), "dbim inputs")) != ISG_OK) return e;
    D.mes.resize(nm);
    for (size_t q = 0; q < nm; q++) D.mes[q] = zd(hm[q].x, hm[q].y);
  }
  D.mesd.assign(nm, zd(0, 0));
  D.rhs.assign(nm, zd(0, 0));
  double mesnorm = 0, objnorm = 0;
  for (auto &v : D.mes) mesnorm += std::norm(v);
  if (chi_true) {
    double t[3];
    if ((e = D.sums(D.otrue, D.otrue, nullptr, 0, t)) != ISG_OK) return e;
    objnorm = t[0];
  }
  if (!O.start_from_chi) {
    // mom.cpp:225-229: no object, total field = incident, mesd = -mes
    cudaMemsetAsync(D.o, 0, U * sizeof(double2), st);
    cudaMemcpyAsync(D.tot, D.incb, (size_t)ntx * U * sizeof(float2), cudaMemcpyDeviceToDevice, st);
    for (size_t q = 0; q < nm; q++) D.mesd[q] = -D.mes[q];
    if ((e = D.set_g()) != ISG_OK) return e;
  } else {
    // mom.cpp:230-245 (commented restart): solve the total fields of the given contrast
    if ((e = D.set_g()) != ISG_OK) return e;
    for (int k = 0; k < D.nchunks(); k++) {
      const int n = D.chunk(k);
      float2 *tk = D.tot + (size_t)k * D.R * U;
      if ((e = D.solve(tk, D.incb + (size_t)k * D.R * U, n, 0)) != ISG_OK) return e;
      k_gx<<<D.vgrid(n), 256, 0, st>>>(D.X, D.g, tk, D.U, 1);
      count_launch();
      if ((e = D.far_field(D.X, k, n, D.rhs)) != ISG_OK) return e;
    }
    for (size_t q = 0; q < nm; q++) D.mesd[q] = D.rhs[q] - D.mes[q];
  }
  // setup_born.cpp:171-242 (write_error): the contrast in raster order as
  // cg_<iteration>.bin (complex128) and one line of hist.txt per record
  auto checkpoint = [&](int file_iter, const isg_dbim_record &r) -> isg_status {
    std::vector<double2> h(U), raster(U);
    cudaMemcpyAsync(h.data(), D.o, U * sizeof(double2), cudaMemcpyDeviceToHost, st);
    isg_status e2 = cuda_check(c, cudaStreamSynchronize(st), "dbim checkpoint");
    if (e2 != ISG_OK) return e2;
    for (size_t n = 0; n < U; n++) raster[c->T.raster_of_blocked[n]] = h[n];
    const std::string dir(O.checkpoint);
    const std::string cg = dir + "/cg_" + std::to_string(file_iter) + ".bin";
    FILE *f = std::fopen(cg.c_str(), "wb");
    FILE *hf = std::fopen((dir + "/hist.txt").c_str(), wrote_hist ? "a" : "w");
    const bool ok = f && hf && std::fwrite(raster.data(), sizeof(double2), U, f) == U &&
                    std::fprintf(hf, "%e %e %e %e %e\n", r.misfit, r.object_error, r.reg_cost, r.grad_norm,
                                 r.object_norm) > 0;
    if (f) std::fclose(f);
    if (hf) std::fclose(hf);
    wrote_hist = true;
    if (!ok) {
      c->err = "dbim checkpoint: cannot write " + cg + " or hist.txt";
      return ISG_BAD_ARG;
    }
    return ISG_OK;
  };
  auto record = [&](int idx, double alpha, zd beta) -> isg_status {
    if (!hist && !O.checkpoint) return ISG_OK;
    double t[3];
    isg_status e2 = D.sums(D.od, D.o, D.otrue, 0, t);
    if (e2 != ISG_OK) return e2;
    double err = 0;
    for (auto &v : D.mesd) err += std::norm(v);
    isg_dbim_record local{};
    isg_dbim_record &r = hist ? hist[idx] : local;
    r.misfit = err / mesnorm;
    r.object_error = chi_true ? t[2] / objnorm : -1.0;
    r.reg_cost = O.regular * O.regular * t[1] / mesnorm;
    r.grad_norm = t[0];
    r.object_norm = t[1];
    r.alpha = alpha;
    r.beta_re = beta.real();
    r.beta_im = beta.imag();
    r.solves = D.solves;
    r.iterations = D.iters;
    // write_error(0) after the first gradient, write_error(iter) after each iteration
    if (O.checkpoint) return checkpoint(idx == 0 ? 0 : idx - 1, r);
    return ISG_OK;
  };
  if ((e = D.gradient(O.regular)) != ISG_OK) return e;
  if ((e = record(0, 0.0, zd(0, 0))) != ISG_OK) return e;
  cudaMemcpyAsync(D.ot, D.od, U * sizeof(double2), cudaMemcpyDeviceToDevice, st);
  for (int it = 0; it < O.iterations; it++) {
    // mom.cpp:280-316: Born-linearised step length alpha = Re<mesd, J ot> / |J ot|^2
    for (int k = 0; k < D.nchunks(); k++) {
      const int n = D.chunk(k);
      k_born<<<D.vgrid(n), 256, 0, st>>>(D.tot + (size_t)k * D.R * U, D.ot, D.k2, D.Y, D.U);
      count_launch();
      if ((e = run_matvec(c, D.Y, nullptr, 0, D.C, n, OP_G, D.so.engine, RED_NONE, nullptr, nullptr, st)) != ISG_OK)
        return e;
      if ((e = D.solve(D.X, D.C, n, 0)) != ISG_OK) return e;
      k_gx<<<D.vgrid(n), 256, 0, st>>>(D.Y, D.g, D.X, D.U, 0);
      count_launch();
      if ((e = D.far_field(D.Y, k, n, D.rhs)) != ISG_OK) return e;
    }
    zd t1(0, 0);
    double t2 = 0;
    for (size_t q = 0; q < nm; q++) {
      t1 += std::conj(D.mesd[q]) * D.rhs[q];
      t2 += std::norm(D.rhs[q]);
    }
    const double alpha = t1.real() / t2;
    // mom.cpp:318-336: step, then re-solve the total fields
    k_axpy_z<<<D.vgrid(), 256, 0, st>>>(D.o, D.ot, make_double2(alpha, 0.0), D.U, 0);
    count_launch();
    if ((e = D.set_g()) != ISG_OK) return e;
    for (int k = 0; k < D.nchunks(); k++) {
      const int n = D.chunk(k);
      float2 *tk = D.tot + (size_t)k * D.R * U;
      // warm: tk still holds this transmitter's total field of the previous contrast
      if ((e = D.solve(tk, D.incb + (size_t)k * D.R * U, n, 0, D.warm ? ISG_GUESS_CALLER : ISG_GUESS_ZERO)) !=
          ISG_OK)
        return e;
      k_gx<<<D.vgrid(n), 256, 0, st>>>(D.X, D.g, tk, D.U, 1);
      count_launch();
      if ((e = D.far_field(D.X, k, n, D.rhs)) != ISG_OK) return e;
    }
    for (size_t q = 0; q < nm; q++) D.mesd[q] = D.rhs[q] - D.mes[q];
    cudaMemcpyAsync(D.save, D.od, U * sizeof(double2), cudaMemcpyDeviceToDevice, st);
    if ((e = D.gradient(O.regular)) != ISG_OK) return e;
    // mom.cpp:383-399: Polak-Ribiere beta = <od, od - save> / |save|^2
    double t[3];
    if ((e = D.sums(D.od, D.save, nullptr, 1, t)) != ISG_OK) return e;
    const zd beta = zd(t[0], t[1]) / t[2];
    if ((e = record(it + 1, alpha, beta)) != ISG_OK) return e;
    k_axpy_z<<<D.vgrid(), 256, 0, st>>>(D.ot, D.od, make_double2(beta.real(), beta.imag()), D.U, 1);
    count_launch();
  }
  if (perm) {
    k_permute_z<<<D.vgrid(), 256, 0, st>>>(perm, D.o, (double2 *)chi, D.U, 0);
    count_launch();
  } else {
    cudaMemcpyAsync(chi, D.o, U * sizeof(double2), cudaMemcpyDeviceToDevice, st);
  }
  return cuda_check(c, cudaStreamSynchronize(st), "dbim");
}

}  // extern "C"
