// Launch-shape autotuner: times the candidate shapes of the level-dependent
// kernels on this context's own buffers and keeps the fastest per level.
//   M2L   sibling-group rows per thread          1, 2, 4, ..., 64
//   L2L   columns (RHS x parent) per tile block  32, 64
//   M2M   columns per tile block (SIMT path)     32, 64
//   near  16x8-leaf tiles per tensor-core CTA    1, 2
// Every candidate computes the same outputs in the same order per output, so
// the choice changes only the time.  The shapes apply to launches of at least
// a quarter of the tuned batch; smaller batches keep the built-in choices.
#include <cfloat>

#include "isg_context.hpp"

using namespace isg;

namespace {

template <class F>
float time_launch(cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1, F launch) {
  launch();  // warm-up
  cudaEventRecord(e0, st);
  for (int r = 0; r < 3; r++) launch();
  cudaEventRecord(e1, st);
  if (cudaEventSynchronize(e1) != cudaSuccess) return FLT_MAX;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  return ms / 3;
}

}  // namespace

extern "C" {

isg_status isg_autotune(isg_ctx *c, int nrhs, int engine, isg_stream stream) {
  if (!c) return ISG_BAD_ARG;
  isg_status e;
  if (!c->gpu_ready && (e = isg_setup_gpu(c)) != ISG_OK) return e;
  if ((e = cuda_check(c, cudaSetDevice(c->opts.device), "cudaSetDevice")) != ISG_OK) return e;
  if (nrhs < 1 || nrhs > c->opts.max_rhs || (engine != ISG_ENGINE_SIMT && engine != ISG_ENGINE_TENSOR)) {
    c->err = "autotune: nrhs must be in [1, max_rhs] and engine an isg_engine";
    return ISG_BAD_ARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  DevPlan &P = c->P;
  P.tuned_nrhs = nrhs;  // candidates below are applied at this batch
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (int i = 2; i < P.L; i++) {  // M2L, accumulating from level 3 on as in the matvec
    DevLevel &d = P.lv[i];
    int best = 0;
    float tbest = FLT_MAX;
    for (int ty : {1, 2, 4, 8, 16, 32, 64}) {
      if (ty > std::max(1, d.n / 2)) break;
      d.m2l_ty = ty;
      const float t = time_launch(st, e0, e1, [&] { launch_m2l(P, i, c->mul, c->loc, nrhs, nullptr, i >= 3, st); });
      if (t < tbest) tbest = t, best = ty;
    }
    d.m2l_ty = best;
  }
  for (int i = 3; i < P.L; i++) {  // L2L into level i
    DevLevel &d = P.lv[i];
    int best = 0;
    float tbest = FLT_MAX;
    for (int cols : {32, 64}) {
      d.l2l_cols = cols;
      const float t = time_launch(st, e0, e1, [&] { launch_l2l(P, i, c->loc, nrhs, nullptr, st); });
      if (t < tbest) tbest = t, best = cols;
    }
    d.l2l_cols = best;
  }
  for (int i = 2; i <= P.L - 2; i++) {  // SIMT M2M into parent level i
    DevLevel &d = P.lv[i];
    int best = 0;
    float tbest = FLT_MAX;
    for (int cols : {32, 64}) {
      d.m2m_cols = cols;
      const float t = time_launch(st, e0, e1, [&] { launch_m2m(P, i, c->mul, nrhs, nullptr, st); });
      if (t < tbest) tbest = t, best = cols;
    }
    d.m2m_cols = best;
  }
  if (engine == ISG_ENGINE_TENSOR && tc_available(c)) {
    NearArgs A;
    A.in.x = c->wx;
    A.in.nrhs = nrhs;
    A.in.mode = IN_PLAIN;
    A.loc = c->loc;
    A.y = c->wy;
    A.epi = EPI_G;
    A.red = RED_NONE;
    A.part = c->part;
    int best = 0;
    float tbest = FLT_MAX;
    for (int pair : {1, 2}) {
      tc_set_near_pair(c, pair);
      const float t = time_launch(st, e0, e1, [&] { tc_near(c, A, st); });
      if (t < tbest) tbest = t, best = pair;
    }
    tc_set_near_pair(c, best);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  // a captured iteration graph holds the old shapes
  if (c->graph_exec) {
    cudaGraphExecDestroy((cudaGraphExec_t)c->graph_exec);
    c->graph_exec = nullptr;
  }
  return cuda_check(c, cudaGetLastError(), "autotune");
}

isg_status isg_tuned(const isg_ctx *c, int what, int level, int *value) {
  if (!c || !value || what < 0 || what > 3 || level < 0 || level >= c->P.L) return ISG_BAD_ARG;
  const DevLevel &d = c->P.lv[level];
  *value = what == 0 ? d.m2l_ty : what == 1 ? d.l2l_cols : what == 2 ? d.m2m_cols : tc_near_pair(c);
  return ISG_OK;
}

}  // extern "C"
