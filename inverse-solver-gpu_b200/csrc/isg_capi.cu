// C ABI of libisg.so (include/isg.h): context lifecycle, table upload
// (the reference's setup_gpu, gpu.cu:69-260, and setup_bicgs,
// bicgs_gpu.cu:89-113), operator, solver and receiver entry points.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "isg_context.hpp"

using namespace isg;

namespace isg {

isg_status cuda_check(isg_ctx *c, cudaError_t e, const char *what) {
  if (e == cudaSuccess) return ISG_OK;
  if (c) c->err = std::string(what) + ": " + cudaGetErrorString(e);
  return ISG_CUDA_ERROR;
}

const int *order_perm(const isg_ctx *c, int order) {
  return order == ISG_ORDER_TREE ? c->P.perm_tree : (order == ISG_ORDER_RASTER ? c->P.perm_raster : nullptr);
}

// solve.cpp:249-355: P2M, M2M up to the root, interpolation to the receivers.
isg_status run_aggregate(isg_ctx *c, const float2 *xb, float2 *rx, int nrhs, cudaStream_t st) {
  BatchArgs B;
  B.x = xb;
  B.nrhs = nrhs;
  launch_p2m(c->P, B, c->mul, st);
  for (int i = c->P.L - 2; i >= 0; i--) launch_m2m(c->P, i, c->mul, nrhs, nullptr, st);
  launch_rx_interp(c->P, c->mul, rx, nrhs, st);
  return cuda_check(c, cudaGetLastError(), "aggregate");
}

// solve.cpp:356-456: anterpolation from the receivers times (-4i) numrx res^2,
// L2L down to the leaves (overwriting), L2P.
isg_status run_aggregateh(isg_ctx *c, float2 *xb, const float2 *rx, int nrhs, cudaStream_t st) {
  const float scale = (float)(-4.0 * c->T.numrx * c->T.res * c->T.res);
  launch_rx_anterp(c->P, rx, c->loc, nrhs, make_float2(0.f, scale), st);
  for (int i = 1; i < c->P.L; i++) launch_l2l(c->P, i, c->loc, nrhs, nullptr, st);
  NearArgs A;
  A.in.nrhs = nrhs;
  A.loc = c->loc;
  A.y = xb;
  A.epi = EPI_L2P_ONLY;
  launch_near(c->P, A, st);
  return cuda_check(c, cudaGetLastError(), "aggregateh");
}

isg_status run_receive(isg_ctx *c, const float2 *xb, float2 *rx, int nrhs, cudaStream_t st) {
  return rxnear_active(c) ? rxnear_apply(c, xb, rx, nrhs, 0, st) : run_aggregate(c, xb, rx, nrhs, st);
}

isg_status run_receiveh(isg_ctx *c, float2 *xb, const float2 *rx, int nrhs, cudaStream_t st) {
  return rxnear_active(c) ? rxnear_apply(c, rx, xb, nrhs, 1, st) : run_aggregateh(c, xb, rx, nrhs, st);
}

}  // namespace isg

namespace {

template <class T>
isg_status upload(isg_ctx *c, T **dst, const std::vector<T> &src) {
  void *p = nullptr;
  isg_status e = cuda_check(c, cudaMalloc(&p, std::max<size_t>(1, src.size()) * sizeof(T)), "cudaMalloc table");
  if (e != ISG_OK) return e;
  c->dev_allocs.push_back(p);
  *dst = (T *)p;
  if (!src.empty()) e = cuda_check(c, cudaMemcpy(p, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice), "upload");
  return e;
}

// Tiles of `out` output samples of a banded resampling whose output sample k
// reads input (idx[k * stride] + t) mod ns_in with weight wt[k * stride + t],
// t < width (the kernels' circular tap walk).
isg_status upload_tile_band(isg_ctx *c, TileBand *tb, const std::vector<int> &idx, const std::vector<double> &wt,
                            int stride, int width, int ns_out, int ns_in, int out) {
  const int tiles = (ns_out + out - 1) / out;
  std::vector<int> a0(tiles), wl(tiles);
  auto rel = [&](int t, int k, int u) { return ((idx[(size_t)k * stride] + u - a0[t]) % ns_in + ns_in) % ns_in; };
  int wmax = 1;
  for (int t = 0; t < tiles; t++) {
    a0[t] = idx[(size_t)t * out * stride];
    int len = 1;
    for (int k = t * out; k < std::min(ns_out, (t + 1) * out); k++)
      for (int u = 0; u < width; u++) len = std::max(len, rel(t, k, u) + 1);
    wl[t] = len;
    wmax = std::max(wmax, len);
  }
  std::vector<float> w((size_t)tiles * wmax * out, 0.f);
  for (int t = 0; t < tiles; t++)
    for (int k = t * out; k < std::min(ns_out, (t + 1) * out); k++)
      for (int u = 0; u < width; u++)
        w[((size_t)t * wmax + rel(t, k, u)) * out + (k - t * out)] += (float)wt[(size_t)k * stride + u];
  // per group of kTileOut outputs, the window rows that carry any of its weights
  const int subs = out / kTileOut;
  std::vector<int2> span((size_t)tiles * subs);
  for (int t = 0; t < tiles; t++)
    for (int b = 0; b < subs; b++) {
      int lo = wl[t], hi = 0;
      for (int jj = 0; jj < wl[t]; jj++)
        for (int i = b * kTileOut; i < (b + 1) * kTileOut; i++)
          if (w[((size_t)t * wmax + jj) * out + i] != 0.f) {
            lo = std::min(lo, jj);
            hi = std::max(hi, jj + 1);
          }
      span[(size_t)t * subs + b] = make_int2(std::min(lo, hi), hi);
    }
  tb->tiles = tiles;
  tb->wmax = wmax;
  tb->out = out;
  isg_status e;
  if ((e = upload(c, &tb->w, w)) || (e = upload(c, &tb->a0, a0)) || (e = upload(c, &tb->wl, wl)) ||
      (e = upload(c, &tb->span, span)))
    return e;
  return ISG_OK;
}

// [4][ns] -> [ns][4]
std::vector<float2> transpose4(const std::vector<cd> &v, int ns) {
  std::vector<float2> o((size_t)4 * ns);
  for (int q = 0; q < 4; q++)
    for (int k = 0; k < ns; k++) {
      const cd z = v[(size_t)q * ns + k];
      o[(size_t)k * 4 + q] = make_float2((float)z.real(), (float)z.imag());
    }
  return o;
}

template <class T>
isg_status dalloc(isg_ctx *c, T **dst, size_t n) {
  void *p = nullptr;
  isg_status e = cuda_check(c, cudaMalloc(&p, std::max<size_t>(1, n) * sizeof(T)), "cudaMalloc workspace");
  if (e != ISG_OK) return e;
  c->dev_allocs.push_back(p);
  *dst = (T *)p;
  return ISG_OK;
}

float2 to_f2(const cd &v) { return make_float2((float)v.real(), (float)v.imag()); }

isg_status need_gpu(isg_ctx *c) {
  if (!c) return ISG_BAD_ARG;
  if (!c->gpu_ready) {
    isg_status e = isg_setup_gpu(c);
    if (e != ISG_OK) return e;
  }
  return cuda_check(c, cudaSetDevice(c->opts.device), "cudaSetDevice");
}

cudaStream_t pick(isg_ctx *, isg_stream s) { return (cudaStream_t)s; }

const int *perm_for(const isg_ctx *c, int order) {
  return order == ISG_ORDER_TREE ? c->P.perm_tree : (order == ISG_ORDER_RASTER ? c->P.perm_raster : nullptr);
}

bool bad_order(int order) { return order < ISG_ORDER_TREE || order > ISG_ORDER_BLOCKED; }

// Brings nrhs caller vectors into the blocked layout (dst) unless they are already.
const float2 *to_blocked(isg_ctx *c, const void *src, float2 *dst, int nrhs, int order, cudaStream_t st) {
  if (order == ISG_ORDER_BLOCKED) return (const float2 *)src;
  launch_permute(perm_for(c, order), (const float2 *)src, dst, c->P.U, nrhs, true, st);
  return dst;
}

void from_blocked(isg_ctx *c, const float2 *src, void *dst, int nrhs, int order, cudaStream_t st) {
  if (order == ISG_ORDER_BLOCKED) {
    if ((const void *)src != dst) cudaMemcpyAsync(dst, src, (size_t)nrhs * c->P.U * sizeof(float2), cudaMemcpyDeviceToDevice, st);
    return;
  }
  launch_permute(perm_for(c, order), src, (float2 *)dst, c->P.U, nrhs, false, st);
}

isg_status check_batch(isg_ctx *c, int nrhs) {
  if (nrhs < 1 || nrhs > c->opts.max_rhs) {
    c->err = "nrhs must be in [1, max_rhs]";
    return ISG_BAD_ARG;
  }
  return ISG_OK;
}

// Contrast in blocked order: shared (g_stride 0) or one per RHS (g_stride U).
isg_status contrast(isg_ctx *c, const void *g, int64_t gs, int nrhs, int order, cudaStream_t st, const float2 **out) {
  if (!g) {
    c->err = "contrast pointer is null";
    return ISG_BAD_ARG;
  }
  if (gs != 0 && gs != c->P.U && order != ISG_ORDER_BLOCKED) {
    c->err = "g_stride must be 0 or numunk when reordering";
    return ISG_BAD_ARG;
  }
  *out = to_blocked(c, g, c->wg, gs ? nrhs : 1, order, st);
  return ISG_OK;
}

uint64_t splitmix(uint64_t &s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
double uniform(uint64_t &s) { return (splitmix(s) >> 11) * (1.0 / 9007199254740992.0); }

}  // namespace

extern "C" {

void isg_default_opts(isg_opts *o) {
  if (!o) return;
  o->level = 5;
  o->box = 8;
  o->res = 0.1;
  o->k0 = 2 * M_PI;
  o->beta = 5;
  o->ninter = 30;
  o->numrx = 32;
  o->max_rhs = 1;
  o->device = 0;
}

void isg_default_solve_opts(isg_solve_opts *o) {
  if (!o) return;
  o->tol = 1e-5;
  o->maxit = 300;
  o->guess = ISG_GUESS_ZERO;
  o->check_every = 1;
  o->true_residual = 1;
  o->max_restarts = 2;
  o->graph = 1;
  o->engine = ISG_ENGINE_SIMT;
}

const char *isg_status_string(isg_status s) {
  switch (s) {
    case ISG_OK: return "ok";
    case ISG_NOT_CONVERGED: return "not converged";
    case ISG_BREAKDOWN: return "breakdown";
    case ISG_NONFINITE: return "non-finite residual";
    case ISG_CUDA_ERROR: return "CUDA error";
    case ISG_BAD_ARG: return "bad argument";
    case ISG_TIMEOUT: return "timeout";
    case ISG_NO_DEVICE: return "no CUDA device";
    case ISG_UNSUPPORTED: return "unsupported";
  }
  return "unknown";
}

const char *isg_last_error(const isg_ctx *c) { return c ? c->err.c_str() : "null context"; }

isg_status isg_create(const isg_opts *opts, isg_ctx **out) {
  if (!opts || !out) return ISG_BAD_ARG;
  *out = nullptr;
  if (opts->max_rhs < 1 || opts->max_rhs > kMaxGridY) return ISG_BAD_ARG;
  isg_ctx *c = new isg_ctx();
  c->opts = *opts;
  // the near-field blocks and translation operators wait for the device (set-up)
  // or for a table query, whichever comes first
  std::string err =
      build_tables(opts->level, opts->box, opts->res, opts->k0, opts->beta, opts->ninter, opts->numrx, c->T, false);
  if (!err.empty()) {
    delete c;
    return ISG_BAD_ARG;
  }
  *out = c;
  return ISG_OK;
}

isg_status isg_setup_gpu(isg_ctx *c) {
  if (!c) return ISG_BAD_ARG;
  if (c->gpu_ready) return ISG_OK;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= c->opts.device) {
    cudaGetLastError();
    c->err = "no CUDA device";
    return ISG_NO_DEVICE;
  }
  isg_status e;
  if ((e = cuda_check(c, cudaSetDevice(c->opts.device), "cudaSetDevice")) != ISG_OK) return e;
  if ((e = cuda_check(c, cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "stream")) != ISG_OK) return e;
  if (!c->T.green_ready && (e = green_tables_gpu(c)) != ISG_OK) return e;
  const HostTables &T = c->T;
  DevPlan &P = c->P;
  const int L = T.L, ns = T.nsamp[L - 1], ni = T.ninter, W = 2 * ni;
  P.L = L;
  P.side = T.side;
  P.nleaf = T.nleaf;
  P.U = T.U;
  P.ninter = ni;
  P.numrx = T.numrx;
  P.ns_leaf = ns;
  P.res = T.res;
  {
    std::vector<float2> w((size_t)9 * kBB * kBB), co((size_t)kBB * ns), ba((size_t)kBB * ns);
    for (int s = 0; s < 9; s++)
      for (int t = 0; t < kBB; t++)
        for (int b = 0; b < kBB; b++) w[((size_t)s * kBB + b) * kBB + t] = to_f2(T.near[((size_t)s * kBB + t) * kBB + b]);
    for (int k = 0; k < ns; k++)
      for (int n = 0; n < kBB; n++) {
        co[(size_t)n * ns + k] = to_f2(T.coeff[(size_t)k * kBB + n]);
        ba[(size_t)k * kBB + n] = to_f2(T.basis[(size_t)n * ns + k]);
      }
    if ((e = upload(c, &P.nearW, w)) || (e = upload(c, &P.coeffT, co)) || (e = upload(c, &P.basisT, ba))) return e;
  }
  size_t off = 0;
  for (int i = 0; i < L; i++) {
    DevLevel &d = P.lv[i];
    d.n = 1 << i;
    d.ns = T.nsamp[i];
    d.off = off;
    off += (size_t)d.n * d.n * d.ns;
    if (i < L - 1) {
      std::vector<int> f(d.ns);
      std::vector<float> w((size_t)ni * d.ns);
      std::vector<float2> sm((size_t)4 * d.ns), sl((size_t)4 * d.ns);
      for (int k = 0; k < d.ns; k++) {
        f[k] = T.intind[i][(size_t)k * ni];
        for (int t = 0; t < ni; t++) w[(size_t)t * d.ns + k] = (float)T.interp[i][(size_t)k * ni + t];
      }
      for (size_t q = 0; q < sm.size(); q++) {
        sm[q] = to_f2(T.shiftmul[i][q]);
        sl[q] = to_f2(T.shiftloc[i][q]);
      }
      if ((e = upload(c, &d.ifirst, f)) || (e = upload(c, &d.iw, w)) || (e = upload(c, &d.shm, sm)) ||
          (e = upload(c, &d.shl, sl)))
        return e;
      if ((e = upload_tile_band(c, &d.mt, T.intind[i], T.interp[i], ni, ni, d.ns, T.nsamp[i + 1], 2 * kTileOut)) ||
          (e = upload(c, &d.shmT, transpose4(T.shiftmul[i], d.ns))) ||
          (e = upload(c, &d.shlT, transpose4(T.shiftloc[i], d.ns))))
        return e;
    }
    if (i >= 1) {
      d.awidth = T.antcount[i];
      std::vector<int> f(d.ns);
      std::vector<float> w((size_t)d.awidth * d.ns);
      for (int k = 0; k < d.ns; k++) {
        f[k] = T.antind[i][(size_t)k * W];
        for (int t = 0; t < d.awidth; t++) w[(size_t)t * d.ns + k] = (float)T.anterp[i][(size_t)k * W + t];
      }
      if ((e = upload(c, &d.afirst, f)) || (e = upload(c, &d.aw, w))) return e;
      if ((e = upload_tile_band(c, &d.at, T.antind[i], T.anterp[i], W, d.awidth, d.ns, T.nsamp[i - 1], 2 * kTileOut)))
        return e;
    }
    if (i >= 2) {
      std::vector<float2> tr(T.trans[i].size());
      for (size_t q = 0; q < tr.size(); q++) tr[q] = to_f2(T.trans[i][q]);
      if ((e = upload(c, &d.T, tr))) return e;
    }
  }
  P.mp = off;
  {
    const int nr = T.numrx, ns0 = T.nsamp[0];
    std::vector<int> hf(nr);
    std::vector<float> hw((size_t)ni * nr);
    for (int m = 0; m < nr; m++) {
      hf[m] = T.intindh[(size_t)m * ni];
      for (int t = 0; t < ni; t++) hw[(size_t)t * nr + m] = (float)T.interph[(size_t)m * ni + t];
    }
    std::vector<float> haw((size_t)ns0 * W);
    for (size_t q = 0; q < haw.size(); q++) haw[q] = (float)T.anterph[q];
    P.hwidth = W;
    if ((e = upload(c, &P.hfirst, hf)) || (e = upload(c, &P.hw, hw)) || (e = upload(c, &P.hind, T.antindh)) ||
        (e = upload(c, &P.haw, haw)))
      return e;
  }
  if ((e = upload(c, &P.perm_tree, T.tree_of_blocked)) || (e = upload(c, &P.perm_raster, T.raster_of_blocked))) return e;

  const size_t R = c->opts.max_rhs, U = T.U;
  c->vec_blocks = (int)std::min<size_t>(512, std::max<size_t>(1, U / 2048));
  c->part_blocks = std::max(c->vec_blocks, near_blocks_per_rhs(P));
  if ((e = dalloc(c, &c->mul, R * P.mp)) || (e = dalloc(c, &c->loc, R * P.mp)) || (e = dalloc(c, &c->wx, R * U)) ||
      (e = dalloc(c, &c->wy, R * U)) || (e = dalloc(c, &c->wg, R * U)) || (e = dalloc(c, &c->vr, R * U)) ||
      (e = dalloc(c, &c->vrt, R * U)) || (e = dalloc(c, &c->vp, R * U)) || (e = dalloc(c, &c->vv, R * U)) ||
      (e = dalloc(c, &c->vs, R * U)) || (e = dalloc(c, &c->vt, R * U)) || (e = dalloc(c, &c->vgx, R * U)) || (e = dalloc(c, &c->levmax, 2 * R * kMaxLevels)) ||
      (e = dalloc(c, &c->part, R * (size_t)c->part_blocks * 4 + 64)) || (e = dalloc(c, &c->state, R)) ||
      (e = dalloc(c, &c->active, R)) || (e = dalloc(c, &c->count, 1)))
    return e;
  c->locmax = c->levmax + R * kMaxLevels;
  if ((e = cuda_check(c, cudaMallocHost(&c->h_count, sizeof(int)), "cudaMallocHost"))) return e;
  if ((e = cuda_check(c, cudaMemset(c->mul, 0, R * P.mp * sizeof(float2)), "memset"))) return e;
  if ((e = cuda_check(c, cudaMemset(c->loc, 0, R * P.mp * sizeof(float2)), "memset"))) return e;
  {
    int nsmax = 1;
    for (int i = 0; i < L; i++) nsmax = std::max(nsmax, T.nsamp[i]);
    if ((e = dalloc(c, &P.zeros, (size_t)nsmax)) ||
        (e = cuda_check(c, cudaMemset(P.zeros, 0, (size_t)nsmax * sizeof(float2)), "memset")))
      return e;
  }
  if ((e = cuda_check(c, kernels_setup(), "kernel attributes")) != ISG_OK) return e;
  if ((e = tc_setup(c)) != ISG_OK) return e;
  if ((e = band_setup(c)) != ISG_OK) return e;
  if ((e = noalloc_prepare(c)) != ISG_OK) return e;
  c->gpu_ready = true;
  return cuda_check(c, cudaDeviceSynchronize(), "setup sync");
}

void isg_destroy(isg_ctx *c) {
  if (!c) return;
  if (c->gpu_ready || !c->dev_allocs.empty()) {
    cudaSetDevice(c->opts.device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->graph_exec) cudaGraphExecDestroy((cudaGraphExec_t)c->graph_exec);
    fno_destroy(c);
    rxnear_destroy(c);
    band_destroy(c);
    tc_destroy(c);
    for (void *p : c->dev_allocs) cudaFree(p);
    if (c->h_count) cudaFreeHost(c->h_count);
    if (c->stream) cudaStreamDestroy(c->stream);
  }
  delete c;
}

int isg_numunk(const isg_ctx *c) { return c ? c->T.U : 0; }
int isg_side(const isg_ctx *c) { return c ? c->T.side : 0; }
int isg_levels(const isg_ctx *c) { return c ? c->T.L : 0; }
int isg_numsamp(const isg_ctx *c, int lvl) { return (c && lvl >= 0 && lvl < c->T.L) ? c->T.nsamp[lvl] : 0; }

isg_status isg_host_table(const isg_ctx *c, const char *name, int lvl, const void **data, int64_t *count) {
  if (!c || !name || !data || !count) return ISG_BAD_ARG;
  const HostTables &T = c->T;
  std::string n(name);
  auto put = [&](const auto &v) {
    *data = v.data();
    *count = (int64_t)v.size();
    return ISG_OK;
  };
  const bool lv_ok = lvl >= 0 && lvl < T.L;
  if ((n == "near" || n == "trans") && !T.green_ready) build_green_tables(const_cast<HostTables &>(T));
  if (n == "numsamp") return put(T.nsamp);
  if (n == "numterm") return put(T.nterm);
  if (n == "clusize") return put(T.csize);
  if (n == "near") return put(T.near);
  if (n == "coeff_multi") return put(T.coeff);
  if (n == "basis_local") return put(T.basis);
  if (n == "interph") return put(T.interph);
  if (n == "intindh") return put(T.intindh);
  if (n == "anterph") return put(T.anterph);
  if (n == "antindh") return put(T.antindh);
  if (n == "pos") return put(T.pos_tree);
  if (n == "unkmap") return put(T.unkmap);
  if (n == "tree_of_blocked") return put(T.tree_of_blocked);
  if (n == "raster_of_blocked") return put(T.raster_of_blocked);
  if (!lv_ok) return ISG_BAD_ARG;
  if (n == "interp") return put(T.interp[lvl]);
  if (n == "intind") return put(T.intind[lvl]);
  if (n == "anterp") return put(T.anterp[lvl]);
  if (n == "antind") return put(T.antind[lvl]);
  if (n == "shiftmul") return put(T.shiftmul[lvl]);
  if (n == "shiftloc") return put(T.shiftloc[lvl]);
  if (n == "trans") return put(T.trans[lvl]);
  return ISG_BAD_ARG;
}

isg_status isg_reorder(isg_ctx *c, const void *in, void *out, int nrhs, int from, int to, isg_stream stream) {
  isg_status e = need_gpu(c);
  if (e != ISG_OK) return e;
  if (bad_order(from) || bad_order(to) || !in || !out || (e = check_batch(c, nrhs)) != ISG_OK) return ISG_BAD_ARG;
  cudaStream_t st = pick(c, stream);
  if (from == to) {
    if (in != out) cudaMemcpyAsync(out, in, (size_t)nrhs * c->P.U * sizeof(float2), cudaMemcpyDeviceToDevice, st);
  } else if (from == ISG_ORDER_BLOCKED) {
    from_blocked(c, (const float2 *)in, out, nrhs, to, st);
  } else if (to == ISG_ORDER_BLOCKED) {
    launch_permute(perm_for(c, from), (const float2 *)in, (float2 *)out, c->P.U, nrhs, true, st);
  } else {
    launch_permute(perm_for(c, from), (const float2 *)in, c->wx, c->P.U, nrhs, true, st);
    from_blocked(c, c->wx, out, nrhs, to, st);
  }
  return cuda_check(c, cudaGetLastError(), "reorder");
}

isg_status isg_mlfma(isg_ctx *c, const void *x, void *r, int nrhs, int conj, int order, int engine, isg_stream stream) {
  isg_status e = need_gpu(c);
  if (e != ISG_OK) return e;
  if (!x || !r || bad_order(order) || (e = check_batch(c, nrhs)) != ISG_OK) return ISG_BAD_ARG;
  cudaStream_t st = pick(c, stream);
  const float2 *xb = to_blocked(c, x, c->wx, nrhs, order, st);
  float2 *yb = order == ISG_ORDER_BLOCKED ? (float2 *)r : c->wy;
  e = run_matvec(c, xb, nullptr, 0, yb, nrhs, conj ? OP_GCONJ : OP_G, engine, RED_NONE, nullptr, nullptr, st);
  if (e != ISG_OK) return e;
  from_blocked(c, yb, r, nrhs, order, st);
  return cuda_check(c, cudaGetLastError(), "mlfma");
}

isg_status isg_matvec(isg_ctx *c, const void *x, const void *g, int64_t g_stride, void *y, int nrhs, int hermitian,
                      int order, int engine, isg_stream stream) {
  isg_status e = need_gpu(c);
  if (e != ISG_OK) return e;
  if (!x || !y || bad_order(order) || (e = check_batch(c, nrhs)) != ISG_OK) return ISG_BAD_ARG;
  cudaStream_t st = pick(c, stream);
  const float2 *gb = nullptr;
  if ((e = contrast(c, g, g_stride, nrhs, order, st, &gb)) != ISG_OK) return e;
  const int64_t gs = (g_stride && order != ISG_ORDER_BLOCKED) ? c->P.U : g_stride;
  const float2 *xb = to_blocked(c, x, c->wx, nrhs, order, st);
  float2 *yb = order == ISG_ORDER_BLOCKED ? (float2 *)y : c->wy;
  e = run_matvec(c, xb, gb, gs, yb, nrhs, hermitian ? OP_ADJ : OP_FWD, engine, RED_NONE, nullptr, nullptr, st);
  if (e != ISG_OK) return e;
  from_blocked(c, yb, y, nrhs, order, st);
  return cuda_check(c, cudaGetLastError(), "matvec");
}

isg_status isg_bicgs(isg_ctx *c, void *x, const void *g, int64_t g_stride, const void *b, int nrhs, int hermitian,
                     int order, const isg_solve_opts *opts, isg_solve_info *info, isg_stream stream) {
  isg_status e = need_gpu(c);
  if (e != ISG_OK) return e;
  if (!x || !b || bad_order(order) || (e = check_batch(c, nrhs)) != ISG_OK) return ISG_BAD_ARG;
  isg_solve_opts o;
  isg_default_solve_opts(&o);
  if (opts) o = *opts;
  if (!(o.tol > 0) || o.maxit < 0 || o.guess < 0 || o.guess > ISG_GUESS_LEARNED) {
    c->err = "bad solve options";
    return ISG_BAD_ARG;
  }
  cudaStream_t st = pick(c, stream);
  if (o.guess == ISG_GUESS_LEARNED) {
    if (hermitian) {
      o.guess = ISG_GUESS_ZERO;  // the network is trained on forward solves
    } else {
      if (!c->fno || (g_stride != 0 && g_stride != c->P.U)) {
        c->err = "ISG_GUESS_LEARNED needs a warm-start network (isg_fno_create) and g_stride 0 or numunk";
        return ISG_UNSUPPORTED;
      }
      if ((e = fno_apply(c, (const float2 *)g, g_stride, (const float2 *)b, (float2 *)x, nrhs, order, st)) != ISG_OK)
        return e;
      o.guess = ISG_GUESS_CALLER;
    }
  }
  const float2 *gb = nullptr;
  if ((e = contrast(c, g, g_stride, nrhs, order, st, &gb)) != ISG_OK) return e;
  const int64_t gs = (g_stride && order != ISG_ORDER_BLOCKED) ? c->P.U : g_stride;
  const float2 *bb = to_blocked(c, b, c->wy, nrhs, order, st);
  float2 *xb = (float2 *)x;
  if (order != ISG_ORDER_BLOCKED) {
    xb = c->wx;
    if (o.guess == ISG_GUESS_CALLER) launch_permute(perm_for(c, order), (const float2 *)x, xb, c->P.U, nrhs, true, st);
  }
  isg_status rs = run_bicgs(c, xb, gb, gs, bb, nrhs, hermitian, &o, info, st);
  if (rs == ISG_CUDA_ERROR || rs == ISG_BAD_ARG || rs == ISG_UNSUPPORTED) return rs;
  from_blocked(c, xb, x, nrhs, order, st);
  if ((e = cuda_check(c, cudaStreamSynchronize(st), "bicgs")) != ISG_OK) return e;
  return rs;
}

isg_status isg_bicgs_group(int n, const isg_group_member *m, int hermitian, int order, const isg_solve_opts *opts,
                           isg_stream stream) {
  if (n < 1 || !m) return ISG_BAD_ARG;
  isg_ctx *c0 = m[0].ctx;
  if (!c0) return ISG_BAD_ARG;
  isg_solve_opts o;
  isg_default_solve_opts(&o);
  if (opts) o = *opts;
  if (!(o.tol > 0) || o.maxit < 0 || o.guess < 0 || o.guess > ISG_GUESS_LEARNED) {
    c0->err = "bad solve options";
    return ISG_BAD_ARG;
  }
  for (int i = 0; i < n; i++) {
    isg_ctx *c = m[i].ctx;
    isg_status e = c ? need_gpu(c) : ISG_BAD_ARG;
    if (e != ISG_OK) return e;
    if (!m[i].x || !m[i].b || bad_order(order) || (e = check_batch(c, m[i].nrhs)) != ISG_OK) return ISG_BAD_ARG;
    for (int j = 0; j < i; j++)
      if (m[j].ctx == c || m[j].ctx->opts.device != c->opts.device) {
        c0->err = "isg_bicgs_group: members need distinct contexts on one device";
        return ISG_BAD_ARG;
      }
    if (o.guess == ISG_GUESS_LEARNED && !hermitian &&
        (!c->fno || (m[i].g_stride != 0 && m[i].g_stride != c->P.U))) {
      c->err = "ISG_GUESS_LEARNED needs a warm-start network (isg_fno_create) and g_stride 0 or numunk";
      return ISG_UNSUPPORTED;
    }
  }
  cudaStream_t st = pick(c0, stream);
  isg_solve_opts om = o;
  if (om.guess == ISG_GUESS_LEARNED) om.guess = hermitian ? ISG_GUESS_ZERO : ISG_GUESS_CALLER;
  std::vector<isg_ctx *> cs(n);
  std::vector<float2 *> xs(n);
  std::vector<const float2 *> gs(n), bs(n);
  std::vector<int64_t> gss(n);
  std::vector<int> Rs(n);
  std::vector<isg_solve_info *> infos(n);
  for (int i = 0; i < n; i++) {
    isg_ctx *c = m[i].ctx;
    isg_status e;
    if (o.guess == ISG_GUESS_LEARNED && !hermitian &&
        (e = fno_apply(c, (const float2 *)m[i].g, m[i].g_stride, (const float2 *)m[i].b, (float2 *)m[i].x, m[i].nrhs,
                       order, st)) != ISG_OK)
      return e;
    if ((e = contrast(c, m[i].g, m[i].g_stride, m[i].nrhs, order, st, &gs[i])) != ISG_OK) return e;
    gss[i] = (m[i].g_stride && order != ISG_ORDER_BLOCKED) ? c->P.U : m[i].g_stride;
    bs[i] = to_blocked(c, m[i].b, c->wy, m[i].nrhs, order, st);
    xs[i] = (float2 *)m[i].x;
    if (order != ISG_ORDER_BLOCKED) {
      xs[i] = c->wx;
      if (om.guess == ISG_GUESS_CALLER)
        launch_permute(perm_for(c, order), (const float2 *)m[i].x, xs[i], c->P.U, m[i].nrhs, true, st);
    }
    cs[i] = c;
    Rs[i] = m[i].nrhs;
    infos[i] = m[i].info;
  }
  isg_status rs = run_bicgs_group(n, cs.data(), xs.data(), gs.data(), gss.data(), bs.data(), Rs.data(), hermitian, &om,
                                  infos.data(), st);
  if (rs == ISG_CUDA_ERROR || rs == ISG_BAD_ARG || rs == ISG_UNSUPPORTED) return rs;
  for (int i = 0; i < n; i++) from_blocked(cs[i], xs[i], m[i].x, m[i].nrhs, order, st);
  isg_status e = cuda_check(c0, cudaStreamSynchronize(st), "bicgs group");
  return e != ISG_OK ? e : rs;
}

isg_status isg_aggregate(isg_ctx *c, const void *x, void *rx, int nrhs, int order, isg_stream stream) {
  isg_status e = need_gpu(c);
  if (e != ISG_OK) return e;
  if (!x || !rx || bad_order(order) || (e = check_batch(c, nrhs)) != ISG_OK) return ISG_BAD_ARG;
  cudaStream_t st = pick(c, stream);
  return run_aggregate(c, to_blocked(c, x, c->wx, nrhs, order, st), (float2 *)rx, nrhs, st);
}

isg_status isg_aggregateh(isg_ctx *c, void *x, const void *rx, int nrhs, int order, isg_stream stream) {
  isg_status e = need_gpu(c);
  if (e != ISG_OK) return e;
  if (!x || !rx || bad_order(order) || (e = check_batch(c, nrhs)) != ISG_OK) return ISG_BAD_ARG;
  cudaStream_t st = pick(c, stream);
  float2 *y = order == ISG_ORDER_BLOCKED ? (float2 *)x : c->wy;
  if ((e = run_aggregateh(c, y, (const float2 *)rx, nrhs, st)) != ISG_OK) return e;
  from_blocked(c, y, x, nrhs, order, st);
  return cuda_check(c, cudaGetLastError(), "aggregateh");
}

isg_status isg_set_nearfield_receivers(isg_ctx *c, double radius) {
  isg_status e = need_gpu(c);
  if (e != ISG_OK) return e;
  if (!(radius >= 0)) {
    c->err = "receiver radius must be >= 0";
    return ISG_BAD_ARG;
  }
  return rxnear_setup(c, radius);
}

isg_status isg_receive(isg_ctx *c, const void *x, void *rx, int nrhs, int order, isg_stream stream) {
  isg_status e = need_gpu(c);
  if (e != ISG_OK) return e;
  if (!x || !rx || bad_order(order) || (e = check_batch(c, nrhs)) != ISG_OK) return ISG_BAD_ARG;
  cudaStream_t st = pick(c, stream);
  return run_receive(c, to_blocked(c, x, c->wx, nrhs, order, st), (float2 *)rx, nrhs, st);
}

isg_status isg_receiveh(isg_ctx *c, void *x, const void *rx, int nrhs, int order, isg_stream stream) {
  isg_status e = need_gpu(c);
  if (e != ISG_OK) return e;
  if (!x || !rx || bad_order(order) || (e = check_batch(c, nrhs)) != ISG_OK) return ISG_BAD_ARG;
  cudaStream_t st = pick(c, stream);
  float2 *y = order == ISG_ORDER_BLOCKED ? (float2 *)x : c->wy;
  if ((e = run_receiveh(c, y, (const float2 *)rx, nrhs, st)) != ISG_OK) return e;
  from_blocked(c, y, x, nrhs, order, st);
  return cuda_check(c, cudaGetLastError(), "receiveh");
}

int64_t isg_kernel_launches(void) { return launch_count(); }

isg_status isg_time_stages(isg_ctx *c, int nrhs, int engine, int reps, double *ms) {
  isg_status e = need_gpu(c);
  if (e != ISG_OK) return e;
  if (!ms || reps < 1 || (e = check_batch(c, nrhs)) != ISG_OK) return ISG_BAD_ARG;
  if (engine == ISG_ENGINE_TENSOR && !tc_available(c)) return ISG_UNSUPPORTED;
  cudaStream_t st = c->stream;
  const DevPlan &P = c->P;
  const size_t n = (size_t)nrhs * P.U;
  cudaMemsetAsync(c->wx, 0, n * sizeof(float2), st);
  cudaMemsetAsync(c->wg, 0, (size_t)P.U * sizeof(float2), st);
  cudaEvent_t ev[5];
  for (auto &v : ev) cudaEventCreate(&v);
  double acc[5] = {0, 0, 0, 0, 0};
  BatchArgs B;
  B.x = c->wx;
  B.g = c->wg;
  B.mode = IN_G;
  B.nrhs = nrhs;
  NearArgs A;
  A.in = B;
  A.loc = c->loc;
  A.y = c->wy;
  A.epi = EPI_FWD;
  A.red = RED_DOT;
  A.dot_a = c->wx;
  A.part = c->part;
  const bool tc = engine == ISG_ENGINE_TENSOR;
  if (tc) {
    // as in a forward tensor-engine solve: the vector updates already formed g x
    // (wx stands in for it), so P2M and the near field read it plainly and the
    // epilogue takes x separately
    B.g = nullptr;
    B.gstride = 0;
    B.mode = IN_PLAIN;
    A.in = B;
    A.x_epi = c->wx;
    A.locmax = c->locmax;
    A.inmax = c->levmax;
  }
  for (int r = -1; r < reps; r++) {
    cudaEventRecord(ev[0], st);
    if (tc) {
      cudaMemsetAsync(c->levmax, 0, (size_t)nrhs * kMaxLevels * sizeof(unsigned), st);
      cudaMemsetAsync(c->locmax, 0, (size_t)nrhs * kMaxLevels * sizeof(unsigned), st);
      tc_p2m(c, B, c->mul, st);
    } else {
      launch_p2m(P, B, c->mul, st);
    }
    cudaEventRecord(ev[1], st);
    isg_status be = ISG_OK;
    for (int i = P.L - 2; i >= 2; i--)
      if (!(tc && band_m2m(c, i, c->mul, nrhs, nullptr, st, &be))) launch_m2m(P, i, c->mul, nrhs, nullptr, st);
    cudaEventRecord(ev[2], st);
    for (int i = 2; i < P.L; i++) {
      if (i >= 3 && !(tc && band_l2l(c, i, c->loc, nrhs, nullptr, st, &be))) launch_l2l(P, i, c->loc, nrhs, nullptr, st);
      launch_m2l(P, i, c->mul, c->loc, nrhs, nullptr, i >= 3, st, tc ? c->locmax : nullptr);
    }
    cudaEventRecord(ev[3], st);
    if (tc) tc_near(c, A, st); else launch_near(P, A, st);
    cudaEventRecord(ev[4], st);
    if ((e = cuda_check(c, cudaEventSynchronize(ev[4]), "time_stages")) != ISG_OK) break;
    if (r < 0) continue;  // warm-up pass
    float t;
    for (int q = 0; q < 4; q++) {
      cudaEventElapsedTime(&t, ev[q], ev[q + 1]);
      acc[q] += t;
    }
    cudaEventElapsedTime(&t, ev[0], ev[4]);
    acc[4] += t;
  }
  for (auto &v : ev) cudaEventDestroy(v);
  for (int q = 0; q < 5; q++) ms[q] = acc[q] / reps;
  return e;
}

isg_status isg_make_phantom(const isg_ctx *c, const isg_phantom *ph, double *chi) {
  if (!c || !ph || !chi) return ISG_BAD_ARG;
  const HostTables &T = c->T;
  const int S = T.side;
  const double D = S * T.res;
  uint64_t s = ph->seed * 0x2545F4914F6CDD1Dull + 0x1234567ull;
  std::fill(chi, chi + 2 * (size_t)T.U, 0.0);
  if (ph->kind == 0) {
    for (int e = 0; e < ph->count; e++) {
      const double a = ph->axis_min + (ph->axis_max - ph->axis_min) * uniform(s);
      const double b = ph->axis_min + (ph->axis_max - ph->axis_min) * uniform(s);
      const double m = std::min(std::max(a, b), D / 2);
      const double cx = (-D / 2 + m) + (D - 2 * m) * uniform(s);
      const double cy = (-D / 2 + m) + (D - 2 * m) * uniform(s);
      const double th = M_PI * uniform(s);
      const double eps = ph->eps_min + (ph->eps_max - ph->eps_min) * uniform(s);
      const double tand = ph->tand_max * uniform(s);
      const double ct = std::cos(th), st = std::sin(th);
      for (int Y = 0; Y < S; Y++)
        for (int X = 0; X < S; X++) {
          const double px = -D / 2 + (X + 0.5) * T.res - cx, py = D / 2 - (Y + 0.5) * T.res - cy;
          const double u = (ct * px + st * py) / a, v = (-st * px + ct * py) / b;
          if (u * u + v * v <= 1.0) {
            chi[2 * ((size_t)Y * S + X)] = eps - 1.0;
            chi[2 * ((size_t)Y * S + X) + 1] = eps * tand;
          }
        }
    }
    return ISG_OK;
  }
  if (ph->kind == 1) {
    // Gaussian random field: white noise smoothed by a separable Gaussian of
    // standard deviation corr_len, mapped affinely onto [eps_min, eps_max].
    std::mt19937_64 gen(s);
    std::normal_distribution<double> nd(0.0, 1.0);
    std::vector<double> f((size_t)T.U), tmp((size_t)T.U);
    for (auto &v : f) v = nd(gen);
    const double sig = ph->corr_len / T.res;
    const int rad = std::max(1, (int)std::ceil(3 * sig));
    std::vector<double> ker(2 * rad + 1);
    for (int k = -rad; k <= rad; k++) ker[k + rad] = std::exp(-0.5 * k * k / (sig * sig));
    for (int Y = 0; Y < S; Y++)
      for (int X = 0; X < S; X++) {
        double acc = 0;
        for (int k = -rad; k <= rad; k++) {
          const int xx = X + k;
          if (xx >= 0 && xx < S) acc += ker[k + rad] * f[(size_t)Y * S + xx];
        }
        tmp[(size_t)Y * S + X] = acc;
      }
    for (int Y = 0; Y < S; Y++)
      for (int X = 0; X < S; X++) {
        double acc = 0;
        for (int k = -rad; k <= rad; k++) {
          const int yy = Y + k;
          if (yy >= 0 && yy < S) acc += ker[k + rad] * tmp[(size_t)yy * S + X];
        }
        f[(size_t)Y * S + X] = acc;
      }
    const auto mm = std::minmax_element(f.begin(), f.end());
    const double lo = *mm.first, hi = *mm.second, span = hi > lo ? hi - lo : 1.0;
    for (size_t i = 0; i < f.size(); i++) {
      const double eps = ph->eps_min + (ph->eps_max - ph->eps_min) * (f[i] - lo) / span;
      chi[2 * i] = eps - 1.0;
      chi[2 * i + 1] = 0.0;
    }
    return ISG_OK;
  }
  return ISG_BAD_ARG;
}

isg_status isg_make_plane_waves(const isg_ctx *c, int ntx, int first, int count, int order, double *inc) {
  if (!c || !inc || ntx < 1 || count < 0 || bad_order(order)) return ISG_BAD_ARG;
  const HostTables &T = c->T;
  for (int j = 0; j < count; j++) {
    const double ang = 2 * M_PI * (first + j) / ntx;
    const double dx = std::cos(ang), dy = std::sin(ang);
    for (int b = 0; b < T.U; b++) {
      const int r = T.raster_of_blocked[b];
      const int dst = order == ISG_ORDER_RASTER ? r : (order == ISG_ORDER_TREE ? T.unkmap[r] : b);
      const cd p = T.pos_raster[r];
      const cd v = std::exp(cd(0, T.k0 * (dx * p.real() + dy * p.imag())));
      inc[2 * ((size_t)j * T.U + dst)] = v.real();
      inc[2 * ((size_t)j * T.U + dst) + 1] = v.imag();
    }
  }
  return ISG_OK;
}

isg_status isg_make_line_sources(const isg_ctx *c, int ntx, int first, int count, double radius, int order,
                                 double *inc) {
  if (!c || !inc || ntx < 1 || count < 0 || bad_order(order)) return ISG_BAD_ARG;
  const HostTables &T = c->T;
  for (int j = 0; j < count; j++) {
    const double ang = 2 * M_PI * (first + j) / ntx;
    const double sx = radius * std::cos(ang), sy = radius * std::sin(ang);
    for (int b = 0; b < T.U; b++) {
      const int r = T.raster_of_blocked[b];
      const int dst = order == ISG_ORDER_RASTER ? r : (order == ISG_ORDER_TREE ? T.unkmap[r] : b);
      const cd p = T.pos_raster[r];
      const cd v = green_entry(T.k0, T.res, p.real() - sx, p.imag() - sy) / (T.res * T.res);
      inc[2 * ((size_t)j * T.U + dst)] = v.real();
      inc[2 * ((size_t)j * T.U + dst) + 1] = v.imag();
    }
  }
  return ISG_OK;
}

}  // extern "C"
