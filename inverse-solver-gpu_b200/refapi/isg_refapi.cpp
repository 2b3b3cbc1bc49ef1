// libisg_ref.so: the reference's routine names and globals (include/isg_refapi.h)
// on top of the C ABI of libisg.so.  Host code only.
#include "../../include/isg_refapi.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/isg.h"

using cdouble = std::complex<double>;

// ---- globals owned by the caller's driver (mom.cpp:4-69) ----
extern double res;
extern int box;
extern int level;
extern double k0;
extern int numunk;
extern int numrx;
extern double toli;
extern int iti;
extern cdouble *pos;
extern int *unkmap;
extern double bicgst, innert, outert;
extern int matvecin, matvecout;

namespace {

isg_ctx *g_ctx = nullptr;
float2 *d_x = nullptr, *d_o = nullptr, *d_b = nullptr, *d_r = nullptr;  // device vectors
float2 *h_stage = nullptr;                                           // pinned staging, numunk
int g_device = 0;

void fail(const char *what, isg_status s) {
  fprintf(stderr, "isg_refapi: %s failed: %s (%s)\n", what, isg_status_string(s), isg_last_error(g_ctx));
  exit(1);
}

void check(const char *what, isg_status s) {
  if (s != ISG_OK) fail(what, s);
}

void cuda(const char *what, cudaError_t e) {
  if (e != cudaSuccess) {
    fprintf(stderr, "isg_refapi: %s: %s\n", what, cudaGetErrorString(e));
    exit(1);
  }
}

void to_device(float2 *dst, const cdouble *src, int n) {
  for (int i = 0; i < n; i++) h_stage[i] = make_float2((float)src[i].real(), (float)src[i].imag());
  cuda("H2D", cudaMemcpy(dst, h_stage, (size_t)n * sizeof(float2), cudaMemcpyHostToDevice));
}

void to_host(cdouble *dst, const float2 *src, int n) {
  cuda("D2H", cudaMemcpy(h_stage, src, (size_t)n * sizeof(float2), cudaMemcpyDeviceToHost));
  for (int i = 0; i < n; i++) dst[i] = cdouble(h_stage[i].x, h_stage[i].y);
}

double now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

void setup_mlfma() {
  isg_opts o;
  isg_default_opts(&o);
  o.level = level;
  o.box = box;
  o.res = res;
  o.k0 = k0;
  o.numrx = numrx;
  o.max_rhs = 1;
  if (const char *d = getenv("ISG_DEVICE")) o.device = atoi(d);
  g_device = o.device;
  check("setup_mlfma", isg_create(&o, &g_ctx));
  if (numunk != isg_numunk(g_ctx)) {
    fprintf(stderr, "isg_refapi: numunk %d does not match the grid of level %d\n", numunk, level);
    exit(1);
  }
  const void *p = nullptr;
  int64_t n = 0;
  pos = new cdouble[numunk];
  unkmap = new int[numunk];
  check("pos", isg_host_table(g_ctx, "pos", 0, &p, &n));
  memcpy(pos, p, (size_t)numunk * sizeof(cdouble));
  check("unkmap", isg_host_table(g_ctx, "unkmap", 0, &p, &n));
  memcpy(unkmap, p, (size_t)numunk * sizeof(int));
}

void setup_gpu() {
  check("setup_gpu", isg_setup_gpu(g_ctx));
  const size_t bytes = (size_t)(numunk > numrx ? numunk : numrx) * sizeof(float2);
  cuda("alloc", cudaMalloc(&d_x, bytes));
  cuda("alloc", cudaMalloc(&d_o, bytes));
  cuda("alloc", cudaMalloc(&d_b, bytes));
  cuda("alloc", cudaMalloc(&d_r, bytes));
  cuda("alloc", cudaMallocHost(&h_stage, bytes));
}

void setup_bicgs() {}

void bicgs(cdouble *x, cdouble *o, cdouble *b, bool ishermitian) {
  const double t0 = now();
  to_device(d_o, o, numunk);
  to_device(d_b, b, numunk);
  to_device(d_x, x, numunk);
  isg_solve_opts so;
  isg_default_solve_opts(&so);
  so.tol = toli;
  so.maxit = iti;
  so.guess = ISG_GUESS_CALLER;
  if (const char *e = getenv("ISG_ENGINE")) so.engine = atoi(e);
  isg_solve_info info;
  const isg_status s = isg_bicgs(g_ctx, d_x, d_o, 0, d_b, 1, ishermitian ? 1 : 0, ISG_ORDER_TREE, &so, &info, nullptr);
  if (s == ISG_CUDA_ERROR || s == ISG_BAD_ARG || s == ISG_UNSUPPORTED || s == ISG_TIMEOUT || s == ISG_NO_DEVICE)
    fail("bicgs", s);
  if (info.status != ISG_OK)
    printf("NOT CONVERGED! **************************** iter: %d proc: %d\n", info.iterations, 0);
  printf("NUMBER OF %d ITERATIONS: %d (%d)\n", ishermitian ? 1 : 0, info.iterations, info.matvecs);
  matvecin += info.matvecs;
  to_host(x, d_x, numunk);
  bicgst += now() - t0;
}

void matvec(cdouble *x, cdouble *o, cdouble *r, bool ishermitian) {
  to_device(d_x, x, numunk);
  to_device(d_o, o, numunk);
  check("matvec", isg_matvec(g_ctx, d_x, d_o, 0, d_r, 1, ishermitian ? 1 : 0, ISG_ORDER_TREE, ISG_ENGINE_SIMT,
                             nullptr));
  matvecin++;
  to_host(r, d_r, numunk);
}

static void mlfma_impl(cdouble *x, cdouble *r, int conj) {
  const double t0 = now();
  to_device(d_x, x, numunk);
  check("mlfma", isg_mlfma(g_ctx, d_x, d_r, 1, conj, ISG_ORDER_TREE, ISG_ENGINE_SIMT, nullptr));
  matvecin++;
  to_host(r, d_r, numunk);
  innert += now() - t0;
}

void mlfma(cdouble *x, cdouble *r) { mlfma_impl(x, r, 0); }
void mlfmah(cdouble *x, cdouble *r) { mlfma_impl(x, r, 1); }

void aggregate(cdouble *x, cdouble *rx) {
  const double t0 = now();
  to_device(d_x, x, numunk);
  check("aggregate", isg_aggregate(g_ctx, d_x, d_r, 1, ISG_ORDER_TREE, nullptr));
  matvecout++;
  to_host(rx, d_r, numrx);
  outert += now() - t0;
}

void aggregateh(cdouble *x, cdouble *rx) {
  const double t0 = now();
  to_device(d_r, rx, numrx);
  check("aggregateh", isg_aggregateh(g_ctx, d_x, d_r, 1, ISG_ORDER_TREE, nullptr));
  matvecout++;
  to_host(x, d_x, numunk);
  outert += now() - t0;
}
