// The Green's-function tables of the MLFMA operator built on the device at
// set-up: the near-field blocks (setup_mlfma.cpp:492-505 over integrate.cpp:
// 15-41) and the diagonal translation operators (setup_mlfma.cpp:506-543).
// They are the only tables that evaluate Bessel functions, and the host's cost
// grows with the square of the coarsest level's sample count (seconds at
// 4096 x 4096 pixels); here one thread per (level, offset) computes the Hankel
// functions H_p = J_p + i Y_p, p = 0..P, and one thread per (level, offset,
// sample) sums the translation series.  Everything is FP64; the results are
// copied back into the host tables, from which set-up continues as before.
//
// Bessel functions of integer order (x > 0):
//  - J_p by Miller's backward recurrence (J. C. P. Miller, 1952; Abramowitz &
//    Stegun 9.12): start at an even order N well above max(P, x) with
//    J_{N+1} = 0, J_N = 1, recur J_{p-1} = (2p / x) J_p - J_{p+1} downwards
//    (rescaling if the values grow past 1e250), and normalise with
//    J_0 + 2 sum_{k >= 1} J_{2k} = 1 (A&S 9.1.46).  Above the turning point
//    p ~ x, J_p decays like Ai((p - x) (2 / x)^(1/3)); N = max(P, x) +
//    15 max(P, x)^(1/3) + 30 puts the start where J_N is below 1e-24 of the
//    largest values.
//  - Y_p by the forward recurrence Y_{p+1} = (2p / x) Y_p - Y_{p-1}
//    (A&S 9.1.27), which is stable for increasing order, from Y_0 and Y_1 of
//    the CUDA math library.
#include <cmath>

#include "isg_context.hpp"
#include "isg_green.cuh"

namespace isg {
namespace {

// near[s][t][b]: testing pixel t of a leaf, basis pixel b of the leaf in neighbour slot s
__global__ void k_green_near(double k0, double res, double2 *near) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 9 * kBB * kBB) return;
  const int s = e / (kBB * kBB), ti = (e / kBB) % kBB, bi = e % kBB;
  const int dr = s / 3 - 1, dc = s % 3 - 1;
  const int ty = ti / kBox, tx = ti % kBox, by = bi / kBox, bx = bi % kBox;
  const double dx = (dc * kBox + bx - tx) * res;
  const double dy = -(dr * kBox + by - ty) * res;
  near[e] = green_entry_d(k0, res, dx, dy);
}

struct GreenLevel {
  int ns, P;
  double a;  // cluster side
  size_t hoff, toff;  // offsets of the level's Hankel block [49][pstride] and translation block [49][ns]
};

// The offset (cm, cn) of the 7 x 7 stencil, observation minus source centre
// (setup_mlfma.cpp:526-527); far when |r| > a sqrt(3).
__device__ __forceinline__ bool green_offset(int o, double a, double &rx, double &ry) {
  const int cm = o / 7, cn = o % 7;
  rx = -(-3 * a + cn * a);
  ry = -(3 * a - cm * a);
  return hypot(rx, ry) > a * sqrt(3.0);
}

// One thread per (level, offset): H_p(k0 |r|), p = 0..P.
__global__ void k_green_hankel(const GreenLevel *lv, int nlev, double k0, int pstride, double2 *H) {
  const int o = blockIdx.x, l = blockIdx.y;
  if (threadIdx.x != 0 || l >= nlev) return;
  const GreenLevel G = lv[l];
  double rx, ry;
  if (!green_offset(o, G.a, rx, ry)) return;
  const double x = k0 * hypot(rx, ry);
  const int P = G.P;
  double2 *h = H + G.hoff + (size_t)o * pstride;
  const double m = fmax((double)P, x);
  int N = (int)(m + 15.0 * cbrt(m) + 30.0);
  N += N & 1;
  double jp1 = 0.0, jp = 1.0, sum = 0.0;  // J_{p+1}, J_p (unnormalised), 2 sum of even orders >= 2
  for (int p = N; p >= 1; p--) {
    if (p <= P) h[p].x = jp;
    if ((p & 1) == 0) sum += 2.0 * jp;
    const double jm1 = (2.0 * p / x) * jp - jp1;
    jp1 = jp;
    jp = jm1;
    if (fabs(jp) > 1e250) {
      jp *= 1e-250;
      jp1 *= 1e-250;
      sum *= 1e-250;
      for (int q = p; q <= P; q++) h[q].x *= 1e-250;
    }
  }
  h[0].x = jp;
  sum += jp;
  const double inv = 1.0 / sum;
  for (int p = 0; p <= P; p++) h[p].x *= inv;
  h[0].y = y0(x);
  if (P >= 1) h[1].y = y1(x);
  for (int p = 1; p < P; p++) h[p + 1].y = (2.0 * p / x) * h[p].y - h[p - 1].y;
}

// One thread per (offset, sample) of a level: T(k) = H_0 + sum_p 2 cos(p (2 pi k / ns - phi)) H_p i^p
// (setup_mlfma.cpp:528-541).
__global__ void k_green_trans(GreenLevel G, int pstride, const double2 *H, double2 *T) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x, o = blockIdx.y;
  if (k >= G.ns) return;
  double2 *out = T + G.toff + (size_t)o * G.ns + k;
  double rx, ry;
  if (!green_offset(o, G.a, rx, ry)) {
    *out = make_double2(0.0, 0.0);
    return;
  }
  const double phi = atan2(ry, rx);
  const double2 *h = H + G.hoff + (size_t)o * pstride;
  const double th = 2 * kPiD * k / G.ns - phi;
  double sr = h[0].x, si = h[0].y;
  for (int p = 1; p <= G.P; p++) {
    const double c = 2 * cos(p * th);
    const double2 v = h[p];
    double tr, ti;  // v i^p
    switch (p & 3) {
      case 0: tr = v.x, ti = v.y; break;
      case 1: tr = -v.y, ti = v.x; break;
      case 2: tr = -v.x, ti = -v.y; break;
      default: tr = v.y, ti = -v.x; break;
    }
    sr += c * tr;
    si += c * ti;
  }
  *out = make_double2(sr, si);
}

}  // namespace

isg_status green_tables_gpu(isg_ctx *c) {
  HostTables &T = c->T;
  const int L = T.L;
  std::vector<GreenLevel> lv;
  int pstride = 1;
  size_t hsize = 0, tsize = 0;
  for (int i = 2; i < L; i++) pstride = std::max(pstride, T.nterm[i] + 1);
  for (int i = 2; i < L; i++) {
    GreenLevel G;
    G.ns = T.nsamp[i];
    G.P = T.nterm[i];
    G.a = T.csize[i];
    G.hoff = hsize;
    G.toff = tsize;
    hsize += (size_t)49 * pstride;
    tsize += (size_t)49 * G.ns;
    lv.push_back(G);
  }
  const size_t nnear = (size_t)9 * kBB * kBB;
  double2 *dnear = nullptr, *dH = nullptr, *dT = nullptr;
  GreenLevel *dlv = nullptr;
  isg_status e = ISG_OK;
  auto fail = [&](cudaError_t r, const char *what) { return e == ISG_OK ? (e = cuda_check(c, r, what)) : e; };
  fail(cudaMalloc(&dnear, nnear * sizeof(double2)), "green tables alloc");
  if (!lv.empty()) {
    fail(cudaMalloc(&dH, std::max<size_t>(hsize, 1) * sizeof(double2)), "green tables alloc");
    fail(cudaMalloc(&dT, std::max<size_t>(tsize, 1) * sizeof(double2)), "green tables alloc");
    fail(cudaMalloc(&dlv, lv.size() * sizeof(GreenLevel)), "green tables alloc");
  }
  if (e == ISG_OK) {
    count_launch();
    k_green_near<<<(int)((nnear + 127) / 128), 128>>>(T.k0, T.res, dnear);
    if (!lv.empty()) {
      fail(cudaMemcpy(dlv, lv.data(), lv.size() * sizeof(GreenLevel), cudaMemcpyHostToDevice), "green tables copy");
      count_launch();
      k_green_hankel<<<dim3(49, (unsigned)lv.size()), 32>>>(dlv, (int)lv.size(), T.k0, pstride, dH);
      for (const GreenLevel &G : lv) {
        count_launch();
        k_green_trans<<<dim3((G.ns + 127) / 128, 49), 128>>>(G, pstride, dH, dT);
      }
    }
    fail(cudaGetLastError(), "green tables launch");
  }
  std::vector<double2> hnear(nnear), htr(tsize);
  if (e == ISG_OK) fail(cudaMemcpy(hnear.data(), dnear, nnear * sizeof(double2), cudaMemcpyDeviceToHost), "green near");
  if (e == ISG_OK && tsize)
    fail(cudaMemcpy(htr.data(), dT, tsize * sizeof(double2), cudaMemcpyDeviceToHost), "green trans");
  cudaFree(dnear);
  cudaFree(dH);
  cudaFree(dT);
  cudaFree(dlv);
  if (e != ISG_OK) return e;
  T.near.resize(nnear);
  for (size_t q = 0; q < nnear; q++) T.near[q] = cd(hnear[q].x, hnear[q].y);
  T.trans.assign(L, {});
  for (int i = 2; i < L; i++) {
    const GreenLevel &G = lv[i - 2];
    T.trans[i].resize((size_t)49 * G.ns);
    for (size_t q = 0; q < T.trans[i].size(); q++) T.trans[i][q] = cd(htr[G.toff + q].x, htr[G.toff + q].y);
  }
  T.green_ready = true;
  return ISG_OK;
}

}  // namespace isg
