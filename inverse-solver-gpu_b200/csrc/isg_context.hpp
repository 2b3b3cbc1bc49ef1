// The opaque isg_ctx behind the C ABI: host tables, device plan, workspaces.
#pragma once

#include <string>
#include <vector>

#include "../../include/isg.h"
#include "isg_device.cuh"
#include "isg_tables.hpp"

namespace isg {

// Per-RHS BiCGSTAB scalars, kept on the device (FP64, bicgs.cpp:100-110).
struct RhsState {
  double bn;          // ||b|| (1 when ||b|| < 1e-20, bicgs.cpp:111-113)
  double err;         // recursive ||r|| / ||b||
  double tres;        // true residual after the final check, -1 if not computed
  double target;      // recursive-residual stopping target: tol, halved at each true-residual restart
  double rho[2];      // current <r~, r>
  double rho1[2];     // previous rho
  double alpha[2];
  double omega[2];
  int iter, matvecs, status, active, fresh, restarts;
};

struct TcPlan;    // tensor-core leaf stage tables (isg_tc.cu)
struct FnoModel;  // learned warm start (isg_fno.cu)
struct BandPlan;  // tensor-core M2M tables (isg_tc_band.cu)
struct RxPlan;    // near-field receiver tables (isg_rxnear.cu)

}  // namespace isg

struct isg_ctx {
  isg_opts opts{};
  isg::HostTables T;
  isg::DevPlan P;
  bool gpu_ready = false;
  cudaStream_t stream = nullptr;
  std::string err;
  std::vector<void *> dev_allocs;

  // workspaces sized for opts.max_rhs
  float2 *mul = nullptr, *loc = nullptr;  // [R][P.mp]
  float2 *wx = nullptr, *wy = nullptr;    // [R][U] reorder scratch
  float2 *wg = nullptr;                   // [R][U] contrast in blocked order
  float2 *vr = nullptr, *vrt = nullptr, *vp = nullptr, *vv = nullptr, *vs = nullptr, *vt = nullptr;
  float2 *vgx = nullptr;  // [R][U] g times the next matvec's input, written by the update kernels
  unsigned *levmax = nullptr;  // [R][kMaxLevels] per-level max |re|, |im| of the multipoles (FP32 bits)
  unsigned *locmax = nullptr;  // [R][kMaxLevels] the same for the locals (written by M2L)
  double *part = nullptr;  // [R][part_blocks][4]
  int part_blocks = 0;
  isg::RhsState *state = nullptr;  // [R]
  int *active = nullptr;           // [R]
  int *count = nullptr;            // active-RHS counter
  int *h_count = nullptr;          // pinned host mirror
  int vec_blocks = 0;
  isg::TcPlan *tc = nullptr;
  isg::BandPlan *band = nullptr;
  isg::FnoModel *fno = nullptr;
  isg::RxPlan *rx = nullptr;  // near-field receivers, when set
  // device address of isg_aggregate_noalloc's static array, resolved by isg_setup_gpu
  float2 *static_scratch = nullptr;
  // BiCGSTAB iteration block captured as a CUDA graph, and what it was captured for
  void *graph_exec = nullptr;
  int64_t graph_launches = 0;
  struct GraphKey {
    const void *x = nullptr, *g = nullptr;
    int64_t gs = 0;
    int R = 0, kind = 0, engine = 0, check = 0, maxit = 0;
    double tol = 0;
    bool operator==(const GraphKey &o) const {
      return x == o.x && g == o.g && gs == o.gs && R == o.R && kind == o.kind && engine == o.engine &&
             check == o.check && maxit == o.maxit && tol == o.tol;
    }
  } graph_key;
  int *tc_err_flag() const;
};

namespace isg {
// Internal operator entry points shared by the C ABI and the solver.
enum OpKind { OP_G = 0, OP_GCONJ = 1, OP_FWD = 2, OP_ADJ = 3 };
isg_status run_matvec(isg_ctx *c, const float2 *x, const float2 *g, int64_t gs, float2 *y, int nrhs, int kind,
                      int engine, int red, const float2 *dot_a, const int *active, cudaStream_t st,
                      const float2 *gx = nullptr);
isg_status run_bicgs(isg_ctx *c, float2 *x, const float2 *g, int64_t gs, const float2 *b, int nrhs, int hermitian,
                     const isg_solve_opts *o, isg_solve_info *info, cudaStream_t st);
isg_status run_bicgs_group(int n, isg_ctx *const *cs, float2 *const *xs, const float2 *const *gs, const int64_t *gss,
                           const float2 *const *bs, const int *Rs, int hermitian, const isg_solve_opts *o,
                           isg_solve_info *const *infos, cudaStream_t st);
isg_status cuda_check(isg_ctx *c, cudaError_t e, const char *what);
// Receiver projection and back-projection on blocked vectors (isg_capi.cu).
isg_status run_aggregate(isg_ctx *c, const float2 *xb, float2 *rx, int nrhs, cudaStream_t st);
isg_status run_aggregateh(isg_ctx *c, float2 *xb, const float2 *rx, int nrhs, cudaStream_t st);
const int *order_perm(const isg_ctx *c, int order);
// The receiver operators of the inversion loop: near-field receivers (dense
// GEMMs, isg_rxnear.cu) when set, else the far-field aggregate / aggregateh.
isg_status run_receive(isg_ctx *c, const float2 *xb, float2 *rx, int nrhs, cudaStream_t st);
isg_status run_receiveh(isg_ctx *c, float2 *xb, const float2 *rx, int nrhs, cudaStream_t st);
isg_status rxnear_setup(isg_ctx *c, double radius);
void rxnear_destroy(isg_ctx *c);
bool rxnear_active(const isg_ctx *c);
isg_status rxnear_apply(isg_ctx *c, const float2 *in, float2 *out, int nrhs, int adjoint, cudaStream_t st);
int rxnear_error(isg_ctx *c);
// Tensor-core engine (isg_tc.cu).
isg_status tc_setup(isg_ctx *c);
void tc_destroy(isg_ctx *c);
bool tc_available(const isg_ctx *c);
// Tiles per near-field CTA chosen by isg_autotune (0: built-in choice).
void tc_set_near_pair(isg_ctx *c, int pair);
int tc_near_pair(const isg_ctx *c);
isg_status tc_p2m(isg_ctx *c, const BatchArgs &B, float2 *mul, cudaStream_t st);
isg_status tc_near(isg_ctx *c, const NearArgs &A, cudaStream_t st);
// Per-RHS partial sums written by tc_near (one per tile).
int tc_near_blocks(const isg_ctx *c);
// Nonzero when a bounded wait inside a tensor-core kernel gave up.
int tc_error(isg_ctx *c);
// Tensor-core M2M into parent level lvl; false when
// the transition has no tensor-core tables (the caller uses the SIMT kernel).
isg_status band_setup(isg_ctx *c);
void band_destroy(isg_ctx *c);
bool band_m2m(isg_ctx *c, int lvl, float2 *mul, int nrhs, const int *active, cudaStream_t st, isg_status *e);
// L2L into child level lvl on the tensor cores (overwrites its locals); false
// when the level is not covered (its rings have more than 128 samples).
bool band_l2l(isg_ctx *c, int lvl, float2 *loc, int nrhs, const int *active, cudaStream_t st, isg_status *e);
// The near-field blocks and translation operators computed on the device into
// the host tables (isg_tables_gpu.cu); called by isg_setup_gpu.
isg_status green_tables_gpu(isg_ctx *c);
// Static scratch of isg_aggregate_noalloc (isg_noalloc.cu): resolves its
// address and loads its kernels; called by isg_setup_gpu.
isg_status noalloc_prepare(isg_ctx *c);
// Learned warm start (isg_fno.cu).
isg_status fno_create(isg_ctx *c, const isg_fno_opts *o);
void fno_destroy(isg_ctx *c);
isg_status fno_apply(isg_ctx *c, const float2 *g, int64_t gs, const float2 *b, float2 *x, int nrhs, int order,
                     cudaStream_t st);
isg_status fno_gradient(isg_ctx *c, const float2 *g, int64_t gs, const float2 *b, const float2 *u, int nrhs, int order,
                        double *loss, cudaStream_t st);
isg_status fno_adam(isg_ctx *c, float lr, cudaStream_t st);
size_t fno_param_count(const isg_ctx *c);
float *fno_param_ptr(isg_ctx *c, int which);
}  // namespace isg
