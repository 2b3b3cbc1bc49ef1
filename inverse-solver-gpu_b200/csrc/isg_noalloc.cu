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
#include <mutex>

#include "isg_context.hpp"

namespace isg {
namespace {

constexpr size_t kScratchElems = (size_t)ISG_STATIC_SCRATCH_BYTES / sizeof(float2);
static __device__ __align__(256) float2 g_scratch[kScratchElems];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
float2 *g_scratch_ptr[kMaxDevices] = {};

// Device address of g_scratch on the current device (ctx->opts.device), looked
// up once per device.
isg_status scratch_address(isg_ctx *c, float2 **out) {
  const int dev = c->opts.device;
  if (dev < 0 || dev >= kMaxDevices) {
    c->err = "device ordinal out of range for the static scratch";
    return ISG_BAD_ARG;
  }
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    void *p = nullptr;
    isg_status e = cuda_check(c, cudaGetSymbolAddress(&p, g_scratch), "cudaGetSymbolAddress(static scratch)");
    if (e != ISG_OK) return e;
    g_scratch_ptr[dev] = (float2 *)p;
  }
  *out = g_scratch_ptr[dev];
  return ISG_OK;
}

}  // namespace
}  // namespace isg

using namespace isg;

extern "C" isg_status isg_aggregate_noalloc(isg_ctx *c, const void *x, void *rx, int nrhs, int order,
                                            isg_stream stream) {
  if (!c) return ISG_BAD_ARG;
  if (!c->gpu_ready) {
    c->err = "isg_aggregate_noalloc needs isg_setup_gpu first (it allocates nothing itself)";
    return ISG_BAD_ARG;
  }
  if (!x || !rx || order < ISG_ORDER_TREE || order > ISG_ORDER_BLOCKED || nrhs < 1) {
    c->err = "isg_aggregate_noalloc: null pointer, bad order or nrhs < 1";
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
  float2 *scratch = nullptr;
  if ((e = scratch_address(c, &scratch)) != ISG_OK) return e;
  cudaStream_t st = (cudaStream_t)stream;
  float2 *mul = scratch;
  const float2 *xb = (const float2 *)x;
  if (order != ISG_ORDER_BLOCKED) {
    float2 *wx = scratch + (size_t)nrhs * c->P.mp;
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
