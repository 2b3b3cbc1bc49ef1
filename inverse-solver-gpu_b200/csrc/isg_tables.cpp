// FP64 host setup of the MLFMA tables.  Formulas follow the reference's
// setup_mlfma.cpp and integrate.cpp (cited per table); the code is organised
// around the library's raster cluster numbering, in which near and far lists
// are stencils and every leaf-level table is computed once from integer pixel
// offsets.
#include "isg_tables.hpp"

#include <cmath>
#include <cstdio>

namespace isg {

static const double kPi = 3.14159265358979323846;

// Antiderivative of log(x^2 + y^2) used by the analytic self term
// (integrate.cpp:11-13).
static double log_rect(double x, double y) {
  return -3 * x * y + x * y * std::log(x * x + y * y) + x * x * std::atan(y / x) + y * y * std::atan(x / y);
}

cd green_entry(double k0, double res, double dx, double dy) {
  // integrate.cpp:15-41: (i/4) res^2 (J0 + i Y0)(k0 d); for the pixel's own
  // centre the log singularity of Y0 is integrated analytically over the square.
  const double dist = std::hypot(dx, dy);
  cd value(j0(k0 * dist), 0.0);
  cd self(0.0, 0.0);
  if (dist < res / 8) {
    value += cd(0.0, 0.5772156649015329 * 2 / kPi + 2 / kPi * std::log(0.5));
    const double x0 = dx - res / 2, x1 = dx + res / 2, y0v = dy - res / 2, y1 = dy + res / 2;
    const double area_log = log_rect(x1, y1) - log_rect(x0, y1) - log_rect(x1, y0v) + log_rect(x0, y0v);
    self = cd(0.0, (area_log / 2 + std::log(k0) * res * res) * 2 / kPi);
  } else {
    value += cd(0.0, y0(k0 * dist));
  }
  value *= res * res;
  return (value + self) * cd(0.0, 0.25);
}

// Lagrange interpolation row (setup_mlfma.cpp:573-599, 653-677): weights of
// the ninter taps of a ring of nin samples that reproduce sample m of a ring of
// nout samples, and the tap indices modulo nin.
static void lagrange(int m, int nout, int nin, int ninter, double *w, int *idx) {
  const double ratio = (double)nin / nout;
  const int c0 = (ninter % 2 == 0) ? (int)std::ceil(m * ratio) : (int)std::lround(m * ratio);
  const double xm = (double)m / nout;
  for (int n = 0; n < ninter; n++) {
    const int ind = c0 + n - ninter / 2;
    const double xn = (double)ind / nin;
    double prod = 1;
    for (int k = 0; k < ninter; k++) {
      if (k == n) continue;
      const double xk = (double)(c0 + k - ninter / 2) / nin;
      prod = prod * (xm - xk) / (xn - xk);
    }
    w[n] = prod;
    idx[n] = ((ind % nin) + nin) % nin;
  }
}

// Transpose of an interpolator (setup_mlfma.cpp:600-631, 678-693): row k of
// the result lists every (source sample, weight * scale) whose taps reach k.
// With `rotate`, each row is rotated so its indices run contiguously modulo
// the source ring (setup_mlfma.cpp:619-630).
static std::string transpose_interp(const std::vector<double> &w, const std::vector<int> &idx, int nsrc, int ndst,
                                    int ninter, double scale, bool rotate, std::vector<double> &tw,
                                    std::vector<int> &tidx, int &longest) {
  const int width = 2 * ninter;
  tw.assign((size_t)ndst * width, 0.0);
  tidx.assign((size_t)ndst * width, 0);
  std::vector<int> fill(ndst, 0);
  for (int m = 0; m < nsrc; m++)
    for (int n = 0; n < ninter; n++) {
      const int k = idx[(size_t)m * ninter + n];
      if (fill[k] >= width) return "interpolator transpose overflows 2*ninter taps (sample rates too far apart)";
      tidx[(size_t)k * width + fill[k]] = m;
      tw[(size_t)k * width + fill[k]] = w[(size_t)m * ninter + n] * scale;
      fill[k]++;
    }
  longest = 0;
  for (int k = 0; k < ndst; k++) {
    longest = std::max(longest, fill[k]);
    if (!rotate) continue;
    int *ri = &tidx[(size_t)k * width];
    double *rw = &tw[(size_t)k * width];
    for (int n = 1; n < fill[k]; n++)
      if (ri[n] != ri[n - 1] + 1) {
        std::vector<int> ti(ri + n, ri + fill[k]);
        std::vector<double> td(rw + n, rw + fill[k]);
        ti.insert(ti.end(), ri, ri + n);
        td.insert(td.end(), rw, rw + n);
        std::copy(ti.begin(), ti.end(), ri);
        std::copy(td.begin(), td.end(), rw);
        break;
      }
  }
  return "";
}

void build_green_tables(HostTables &t) {
  const int L = t.L, box = t.box, bb = t.bb;
  const double res = t.res, k0 = t.k0;
  // Near-field blocks (setup_mlfma.cpp:492-505): testing pixel t of a leaf,
  // basis pixel b of the neighbour leaf in slot s; translation-invariant.
  t.near.assign((size_t)9 * bb * bb, cd(0, 0));
  for (int s = 0; s < 9; s++) {
    const int dr = s / 3 - 1, dc = s % 3 - 1;
    for (int ti = 0; ti < bb; ti++)
      for (int bi = 0; bi < bb; bi++) {
        const int ty = ti / box, tx = ti % box, by = bi / box, bx = bi % box;
        const double dx = (dc * box + bx - tx) * res;
        const double dy = -(dr * box + by - ty) * res;
        t.near[((size_t)s * bb + ti) * bb + bi] = green_entry(k0, res, dx, dy);
      }
  }

  // Diagonal translation operators for the 7x7 offsets (setup_mlfma.cpp:506-543).
  t.trans.assign(L, {});
  {
    std::vector<cd> hank, ipow;
    for (int p = 0; p < t.nterm[0]; p++) ipow.push_back(std::exp(cd(0, (p + 1) * kPi / 2)));
    for (int i = 2; i < L; i++) {
      const int ns = t.nsamp[i], P = t.nterm[i];
      const double a = t.csize[i];
      t.trans[i].assign((size_t)49 * ns, cd(0, 0));
      hank.assign(P + 1, cd(0, 0));
      for (int cm = 0; cm < 7; cm++)
        for (int cn = 0; cn < 7; cn++) {
          const cd r = -cd(-3 * a + cn * a, 3 * a - cm * a);  // observation minus source centre
          if (!(std::abs(r) > a * std::sqrt(3.0))) continue;
          const double kr = k0 * std::abs(r), phi = std::arg(r);
          for (int p = 0; p <= P; p++) hank[p] = cd(jn(p, kr), yn(p, kr));
          for (int k = 0; k < ns; k++) {
            cd sum = hank[0];
            for (int p = 1; p <= P; p++) sum = sum + 2 * std::cos(p * (2 * kPi * k / ns - phi)) * hank[p] * ipow[p - 1];
            t.trans[i][(size_t)(cm * 7 + cn) * ns + k] = sum;
          }
        }
    }
  }

  t.green_ready = true;
}

std::string build_tables(int level, int box, double res, double k0, int beta, int ninter, int numrx, HostTables &t,
                         bool with_green) {
  if (level < 3 || level > 12) return "level must be in [3, 12]";
  if (box != 8) return "only 8x8-pixel leaves are supported";
  if (ninter < 2 || ninter % 2) return "ninter must be even and >= 2";
  if (numrx < 1) return "numrx must be >= 1";
  if (!(res > 0) || !(k0 > 0)) return "res and k0 must be positive";
  t = HostTables();
  t.L = level;
  t.box = box;
  t.bb = box * box;
  t.side = box << (level - 1);
  t.nleaf = 1 << (level - 1);
  t.U = t.side * t.side;
  t.ninter = ninter;
  t.beta = beta;
  t.numrx = numrx;
  t.k0 = k0;
  t.res = res;
  const int L = level, bb = t.bb;

  // Sample counts (setup_mlfma.cpp:75-85).
  t.nclus.resize(L);
  t.nsamp.resize(L);
  t.nterm.resize(L);
  t.csize.resize(L);
  for (int i = 0; i < L; i++) {
    t.nclus[i] = 1 << (2 * i);
    t.csize[i] = res * box * std::pow(2.0, L - i - 1);
    const double kr = std::sqrt(2.0) * k0 * t.csize[i];
    t.nterm[i] = (int)std::floor(kr + 1.8 * std::pow((double)beta, 2.0 / 3) * std::pow(kr, 1.0 / 3));
    t.nsamp[i] = 4 * t.nterm[i];
  }
  const int nsl = t.nsamp[L - 1];

  // Plane-wave P2M coefficients and L2P basis about the leaf centre
  // (setup_mlfma.cpp:544-553, integrate.cpp:43-69).
  t.coeff.resize((size_t)nsl * bb);
  t.basis.resize((size_t)nsl * bb);
  {
    const double half = t.csize[L - 1] / 2 - res / 2;
    for (int n = 0; n < bb; n++) {
      const double px = -half + (n % box) * res, py = half - (n / box) * res;
      for (int k = 0; k < nsl; k++) {
        const double ang = 2 * kPi * k / nsl;
        const double ph = k0 * (std::cos(ang) * px + std::sin(ang) * py);
        t.coeff[(size_t)k * bb + n] = std::exp(cd(0, -ph)) * (res * res);
        t.basis[(size_t)n * nsl + k] = std::exp(cd(0, ph)) / cd(nsl) * cd(0, 0.25);
      }
    }
  }

  if (with_green) build_green_tables(t);

  // Shift phases to the four children (setup_mlfma.cpp:554-570); child
  // q = row*2 + col, rho = parent centre - child centre.
  t.shiftmul.assign(L, {});
  t.shiftloc.assign(L, {});
  for (int i = 0; i < L - 1; i++) {
    const int ns = t.nsamp[i];
    const double sc = t.csize[i + 1];
    t.shiftmul[i].resize((size_t)4 * ns);
    t.shiftloc[i].resize((size_t)4 * ns);
    for (int q = 0; q < 4; q++) {
      const double rx = (0.5 - (q & 1)) * sc, ry = ((q >> 1) - 0.5) * sc;
      for (int k = 0; k < ns; k++) {
        const double ang = 2 * kPi * k / ns;
        const double ph = k0 * std::cos(ang) * rx + k0 * std::sin(ang) * ry;
        t.shiftmul[i][(size_t)q * ns + k] = std::exp(cd(0, ph));
        t.shiftloc[i][(size_t)q * ns + k] = std::exp(cd(0, -ph));
      }
    }
  }

  // Interpolators child rate -> parent rate, and their rotated transposes
  // (setup_mlfma.cpp:571-631).
  t.interp.assign(L, {});
  t.intind.assign(L, {});
  t.anterp.assign(L, {});
  t.antind.assign(L, {});
  t.antcount.assign(L, 0);
  for (int i = 0; i < L - 1; i++) {
    const int ns = t.nsamp[i];
    t.interp[i].resize((size_t)ns * ninter);
    t.intind[i].resize((size_t)ns * ninter);
    for (int m = 0; m < ns; m++)
      lagrange(m, ns, t.nsamp[i + 1], ninter, &t.interp[i][(size_t)m * ninter], &t.intind[i][(size_t)m * ninter]);
  }
  for (int i = 1; i < L; i++) {
    // Scale by the rate ratio as (w * ns_i) / ns_{i-1}, the reference's order of
    // operations (setup_mlfma.cpp:616), so both agree to the last bit.
    std::vector<double> scaled(t.interp[i - 1].size());
    for (size_t e = 0; e < scaled.size(); e++) scaled[e] = t.interp[i - 1][e] * t.nsamp[i] / t.nsamp[i - 1];
    std::string err = transpose_interp(scaled, t.intind[i - 1], t.nsamp[i - 1], t.nsamp[i], ninter, 1.0, true,
                                       t.anterp[i], t.antind[i], t.antcount[i]);
    if (!err.empty()) return err;
    // The device kernels read each row as a contiguous run from its first index.
    const int w = 2 * ninter, nsp = t.nsamp[i - 1];
    for (int k = 0; k < t.nsamp[i]; k++)
      for (int n = 0; n < w; n++) {
        if (t.anterp[i][(size_t)k * w + n] == 0.0) continue;
        if (t.antind[i][(size_t)k * w + n] != (t.antind[i][(size_t)k * w] + n) % nsp)
          return "anterpolation row is not contiguous";
      }
  }

  // Receiver ring (setup_mlfma.cpp:642-695).
  {
    const int ns0 = t.nsamp[0];
    t.interph.resize((size_t)numrx * ninter);
    t.intindh.resize((size_t)numrx * ninter);
    for (int m = 0; m < numrx; m++)
      lagrange(m, numrx, ns0, ninter, &t.interph[(size_t)m * ninter], &t.intindh[(size_t)m * ninter]);
    std::vector<double> scaled(t.interph.size());
    for (size_t e = 0; e < scaled.size(); e++) scaled[e] = t.interph[e] * ns0 / numrx;
    int cnt = 0;
    std::string err = transpose_interp(scaled, t.intindh, numrx, ns0, ninter, 1.0, false, t.anterph, t.antindh, cnt);
    if (!err.empty()) return "receiver " + err;
  }

  // Orderings and pixel centres (setup_mlfma.cpp:156-185).
  {
    const int S = t.side, nl = t.nleaf;
    const double D = S * res;
    t.pos_raster.resize(t.U);
    t.pos_tree.resize(t.U);
    t.unkmap.resize(t.U);
    t.tree_of_blocked.resize(t.U);
    t.raster_of_blocked.resize(t.U);
    for (int Y = 0; Y < S; Y++)
      for (int X = 0; X < S; X++) {
        const int r = Y * S + X;
        const int ly = Y / box, lx = X / box, py = Y % box, px = X % box;
        const int blocked = (ly * nl + lx) * bb + py * box + px;
        const int tree = tree_index(ly, lx, L - 1) * bb + py * box + px;
        const cd p(-D / 2 + (X + 0.5) * res, D / 2 - (Y + 0.5) * res);
        t.pos_raster[r] = p;
        t.pos_tree[tree] = p;
        t.unkmap[r] = tree;
        t.tree_of_blocked[blocked] = tree;
        t.raster_of_blocked[blocked] = r;
      }
  }
  return "";
}

}  // namespace isg
