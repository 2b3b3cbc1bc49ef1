// isg_aggregate_noalloc: the receiver projection of isg_aggregate (P2M, M2M up
// to the root, interpolation to the receivers; solve.cpp:249-355) with its
// multipole tree and its reordered input in a fixed device array of this file
// instead of the context's workspaces.  It calls no allocator.
//
// Scratch layout for nrhs right-hand sides: [nrhs][mp] multipoles, then
// [nrhs][U] blocked input when the caller's order is not ISG_ORDER_BLOCKED.
// Every element the kernels read was written earlier in the same call (P2M
// writes every leaf sample, each M2M every parent sample), so nothing has to
// be cleared between calls.
//
// The array lives in this file's own device module.  CUDA loads modules
// lazily (the default since CUDA 12.2), and loading this one is what
// allocates the array's 64 MiB, so isg_setup_gpu calls noalloc_prepare: the
// address lookup below loads the module there, together with the kernels the
// entry point launches, and the entry point itself only reads the address the
// context keeps.
#include "isg_context.hpp"

namespace isg {
namespace {

constexpr size_t kScratchElems = (size_t)ISG_STATIC_SCRATCH_BYTES / sizeof(float2);
static __device__ __align__(256) float2 g_scratch[kScratchElems];

}  // namespace

// Called by isg_setup_gpu with the context's device current: the device
// address of g_scratch (host code cannot use the symbol itself as a device
// pointer), and the kernels of the entry point loaded now rather than on its
// first call.
isg_status noalloc_prepare(isg_ctx *c) {
  void *p = nullptr;
  isg_status e = cuda_check(c, cudaGetSymbolAddress(&p, g_scratch), "cudaGetSymbolAddress(static scratch)");
  if (e != ISG_OK) return e;
  if ((e = cuda_check(c, aggregate_kernels_load(), "loading the receiver-projection kernels")) != ISG_OK) return e;
  c->static_scratch = (float2 *)p;
  return ISG_OK;
}

}  // namespace isg

using namespace isg;

extern "C" isg_status isg_aggregate_noalloc(isg_ctx *c, const void *x, void *rx, int nrhs, int order,
                                            isg_stream stream) {
  if (!c) return ISG_BAD_ARG;
  if (!c->gpu_ready || !c->static_scratch) {
    c->err = "isg_aggregate_noalloc needs isg_setup_gpu first (it allocates nothing itself)";
    return ISG_BAD_ARG;
  }
  if (!x || !rx || order < ISG_ORDER_TREE || order > ISG_ORDER_BLOCKED || nrhs < 1) {
    c->err = "isg_aggregate_noalloc: null pointer, bad order or nrhs < 1";
    return ISG_BAD_ARG;
  }
  if (nrhs > kMaxGridY) {
    c->err = "isg_aggregate_noalloc: nrhs=" + std::to_string(nrhs) + " exceeds " + std::to_string(kMaxGridY) +
             " RHS per call (one grid row per RHS)";
    return ISG_BAD_ARG;
  }
  const size_t per_rhs = c->P.mp + (order == ISG_ORDER_BLOCKED ? 0 : (size_t)c->P.U);
  if ((size_t)nrhs * per_rhs > kScratchElems) {
    c->err = "isg_aggregate_noalloc: nrhs=" + std::to_string(nrhs) + " needs " +
             std::to_string((size_t)nrhs * per_rhs * sizeof(float2)) + " bytes of scratch; the static array holds " +
             std::to_string((size_t)ISG_STATIC_SCRATCH_BYTES) + " (at most " +
             std::to_string(kScratchElems / per_rhs) + " RHS per call at this level and order)";
    return ISG_BAD_ARG;
  }
  isg_status e = cuda_check(c, cudaSetDevice(c->opts.device), "cudaSetDevice");
  if (e != ISG_OK) return e;
  cudaStream_t st = (cudaStream_t)stream;
  float2 *mul = c->static_scratch;
  const float2 *xb = (const float2 *)x;
  if (order != ISG_ORDER_BLOCKED) {
    float2 *wx = c->static_scratch + (size_t)nrhs * c->P.mp;
    launch_permute(order_perm(c, order), (const float2 *)x, wx, c->P.U, nrhs, true, st);
    xb = wx;
  }
  BatchArgs B;
  B.x = xb;
  B.nrhs = nrhs;
  launch_p2m(c->P, B, mul, st);
  for (int i = c->P.L - 2; i >= 0; i--) launch_m2m(c->P, i, mul, nrhs, nullptr, st);
  launch_rx_interp(c->P, mul, (float2 *)rx, nrhs, st);
  return cuda_check(c, cudaGetLastError(), "aggregate_noalloc");
}
