/* Restated FP64 oracle of the reference's MLFMA forward/adjoint solve path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path, never the product.
 * Every routine restates the reference's arithmetic step by step, in FP64 and
 * in the reference's tree order, citing the file:line it follows.  It is pinned
 * against the reference's own compiled CPU path (oracle/_ref) and the golden
 * fixtures in tests/golden/.
 */
#define _DEFAULT_SOURCE /* jn, yn, j0, y0 from libm */
#include "isg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

struct orc_ctx {
  int L, box, bb, beta, ninter, numrx, U;
  double k0, res;
  int *nclus, *nsamp, *nterm;
  double *csize;
  double complex **cen;
  int **par;
  int **nearl, **farl, **traid;
  double complex *pos;
  int *unkmap;
  double complex *nearT; /* [9][bb][bb]: near[slot][testing][basis] */
  double complex *coeff; /* [ns_leaf][bb] */
  double complex *basis; /* [bb][ns_leaf] */
  double **interp;
  int **intind;          /* level i < L-1: [ns_i][ninter] */
  double **anterp;
  int **antind;          /* level i >= 1: [ns_i][2 ninter] */
  double complex **shm, **shl; /* level i < L-1: [4][ns_i] */
  double complex **trans;      /* level i >= 2: [49][ns_i] */
  double *interph;
  int *intindh; /* [numrx][ninter] */
  double *anterph;
  int *antindh; /* [ns_0][2 ninter] */
  double complex **mul, **loc;
  double complex *buf;
  double complex *go; /* near-field receivers: [numrx][U] integrate(rx_m, pos_n), or NULL */
};

/* integrate.cpp:7-9 */
static double complex hn(int order, double x) { return jn(order, x) + I * yn(order, x); }

/* integrate.cpp:11-13: antiderivative of log(x^2+y^2) over a rectangle corner. */
static double integ(double x, double y) {
  return -3 * x * y + x * y * log(x * x + y * y) + x * x * atan(y / x) + y * y * atan(x / y);
}

/* integrate.cpp:15-41 */
double complex orc_integrate(const orc_ctx *c, double complex post, double complex posb) {
  double res = c->res, k0 = c->k0;
  double dist = cabs(post - posb);
  double complex numer = j0(k0 * dist);
  double complex anal = 0;
  if (dist < res / 8) {
    numer += I * (0.5772156649015329 * 2 / M_PI + 2 / M_PI * log(0.5));
    double xcen = creal(posb - post), ycen = cimag(posb - post);
    double xmin = xcen - res / 2, xmax = xcen + res / 2;
    double ymin = ycen - res / 2, ymax = ycen + res / 2;
    double analt = integ(xmax, ymax) - integ(xmin, ymax) - integ(xmax, ymin) + integ(xmin, ymin);
    anal = I * ((analt / 2 + log(k0) * res * res) * 2 / M_PI);
  } else {
    numer += I * y0(k0 * dist);
  }
  numer *= res * res;
  return (numer + anal) * (0.25 * I);
}

/* integrate.cpp:43-56 (sign -1) and :58-69 (sign +1, without res^2). */
static double complex plane_wave(const orc_ctx *c, double complex center, double complex p, int order, int sign) {
  int numang = c->nsamp[c->L - 1];
  double angle = 2 * M_PI * order / numang;
  double ux = cos(angle), uy = sin(angle);
  double complex d = p - center;
  double ph = c->k0 * (ux * creal(d) + uy * cimag(d));
  if (sign < 0) return cexp(-I * ph) * (c->res * c->res);
  return cexp(I * ph);
}

/* Lagrange weights of setup_mlfma.cpp:573-599 and :653-677: sample m of a
 * ring of nout samples from ninter taps of a ring of nin samples. */
static void lagrange_row(int m, int nout, int nin, int ninter, double *w, int *idx) {
  double ratio = (double)nin / nout;
  int center = (ninter % 2 == 0) ? (int)ceil(m * ratio) : (int)round(m * ratio);
  double xm = (double)m / nout;
  for (int n = 0; n < ninter; n++) {
    int ind = center + n - ninter / 2;
    double mul = 1, xn = (double)ind / nin;
    for (int k = 0; k < ninter; k++)
      if (k != n) {
        double xk = (double)(center + k - ninter / 2) / nin;
        mul = mul * (xm - xk) / (xn - xk);
      }
    w[n] = mul;
    ind = ind % nin;
    if (ind < 0) ind += nin;
    idx[n] = ind;
  }
}

orc_ctx *orc_create(int level, double k0, double res, int box, int beta, int ninter, int numrx) {
  if (level < 3 || box < 1 || ninter < 2) return NULL;
  orc_ctx *c = calloc(1, sizeof *c);
  int L = level;
  c->L = L;
  c->box = box;
  c->bb = box * box;
  c->beta = beta;
  c->ninter = ninter;
  c->numrx = numrx;
  c->k0 = k0;
  c->res = res;
  int side = box << (L - 1);
  c->U = side * side;
  int bb = c->bb, U = c->U;

  /* setup_mlfma.cpp:70-85 */
  c->nclus = malloc(L * sizeof(int));
  c->nsamp = malloc(L * sizeof(int));
  c->nterm = malloc(L * sizeof(int));
  c->csize = malloc(L * sizeof(double));
  for (int i = 0; i < L; i++) {
    c->nclus[i] = 1 << (2 * i);
    c->csize[i] = res * box * pow(2, L - i - 1);
    double kr = sqrt(2) * k0 * c->csize[i];
    double term = kr + 1.8 * pow(beta, 2.0 / 3) * pow(kr, 1.0 / 3);
    c->nterm[i] = (int)floor(term);
    c->nsamp[i] = 4 * c->nterm[i];
  }

  /* setup_mlfma.cpp:105-153: children of cluster p at level i are 4p..4p+3
   * (k*2+l, k = row from the top, l = column); pixels of leaf p are p*bb.. */
  c->cen = calloc(L, sizeof(double complex *));
  c->par = calloc(L, sizeof(int *));
  c->nearl = calloc(L, sizeof(int *));
  c->farl = calloc(L, sizeof(int *));
  c->traid = calloc(L, sizeof(int *));
  for (int i = 0; i < L; i++) {
    c->cen[i] = calloc(c->nclus[i], sizeof(double complex));
    c->par[i] = malloc(c->nclus[i] * sizeof(int));
    c->nearl[i] = malloc(9 * c->nclus[i] * sizeof(int));
    c->farl[i] = malloc(27 * c->nclus[i] * sizeof(int));
    c->traid[i] = malloc(27 * c->nclus[i] * sizeof(int));
    for (int m = 0; m < 27 * c->nclus[i]; m++) c->traid[i][m] = -1;
  }
  c->par[0][0] = -1;
  for (int i = 1; i < L; i++)
    for (int ch = 0; ch < c->nclus[i]; ch++) c->par[i][ch] = ch / 4;

  /* setup_mlfma.cpp:156-175 */
  c->pos = malloc(U * sizeof(double complex));
  c->cen[0][0] = 0;
  for (int i = 0; i < L; i++)
    for (int m = 0; m < c->nclus[i]; m++) {
      if (i < L - 1) {
        double complex cor = c->cen[i][m] + c->csize[i] / 4 * (-1 + I);
        for (int k = 0; k < 2; k++)
          for (int l = 0; l < 2; l++)
            c->cen[i + 1][m * 4 + k * 2 + l] = cor + (l * c->csize[i + 1] - I * (k * c->csize[i + 1]));
      } else {
        double complex cor = c->cen[i][m] + (c->csize[i] / 2 - res / 2) * (-1 + I);
        for (int k = 0; k < box; k++)
          for (int l = 0; l < box; l++) c->pos[m * bb + k * box + l] = cor + (l * res - I * (k * res));
      }
    }

  /* setup_mlfma.cpp:177-185 */
  c->unkmap = malloc(U * sizeof(int));
  {
    double complex cor = c->csize[0] / 2 * (-1 + I);
    for (int n = 0; n < U; n++) {
      int l = (int)floor((creal(c->pos[n]) - creal(cor)) / res);
      int k = (int)floor((cimag(cor) - cimag(c->pos[n])) / res);
      c->unkmap[k * side + l] = n;
    }
  }

  /* setup_mlfma.cpp:186-223 */
  for (int i = 0; i < L; i++) {
    for (int m = 0; m < 9 * c->nclus[i]; m++) c->nearl[i][m] = -1;
    for (int m = 0; m < 27 * c->nclus[i]; m++) c->farl[i][m] = -1;
  }
  c->nearl[0][0] = 0;
  for (int i = 1; i < L; i++) {
    double dim = c->csize[i];
    for (int m = 0; m < c->nclus[i]; m++) {
      int nid = 0, fid = 0, p = c->par[i][m];
      for (int ind = 0; ind < 9; ind++) {
        int uncle = c->nearl[i - 1][p * 9 + ind];
        if (uncle == -1) continue;
        for (int q = 0; q < 4; q++) {
          int n = uncle * 4 + q;
          if (cabs(c->cen[i][n] - c->cen[i][m]) < dim * sqrt(3))
            c->nearl[i][m * 9 + nid++] = n;
          else
            c->farl[i][m * 27 + fid++] = n;
        }
      }
    }
  }

  /* setup_mlfma.cpp:459-484: leaf near lists re-sorted into 3x3 slots
   * (slot = (row offset + 1) * 3 + (column offset + 1), rows downward). */
  {
    int i = L - 1;
    double a = c->csize[i];
    for (int m = 0; m < c->nclus[i]; m++) {
      int slot[9];
      for (int s = 0; s < 9; s++) slot[s] = -1;
      for (int s = 0; s < 9; s++) {
        int n = c->nearl[i][m * 9 + s];
        if (n == -1) continue;
        double complex d = c->cen[i][m] - c->cen[i][n];
        int mm = (int)round(cimag(d) / a) + 1, nn = (int)round(-creal(d) / a) + 1;
        slot[mm * 3 + nn] = n;
      }
      memcpy(&c->nearl[i][m * 9], slot, sizeof slot);
    }
  }

  /* setup_mlfma.cpp:492-505: nine translation-invariant bb x bb near blocks,
   * each filled from the first leaf that has that slot. */
  c->nearT = calloc(9 * (size_t)bb * bb, sizeof(double complex));
  {
    int i = L - 1;
    for (int s = 0; s < 9; s++) {
      int m = -1, n = -1;
      for (int q = 0; q < c->nclus[i]; q++)
        if (c->nearl[i][q * 9 + s] != -1) {
          m = q;
          n = c->nearl[i][q * 9 + s];
          break;
        }
      if (m < 0) continue;
      for (int k = 0; k < bb; k++)
        for (int l = 0; l < bb; l++)
          c->nearT[(size_t)s * bb * bb + k * bb + l] = orc_integrate(c, c->pos[m * bb + k], c->pos[n * bb + l]);
    }
  }

  /* setup_mlfma.cpp:506-543: diagonal translation operators. */
  c->trans = calloc(L, sizeof(double complex *));
  {
    int P0 = c->nterm[0];
    double complex *hank = malloc((2 * P0 + 1) * sizeof(double complex));
    double complex *expn = malloc((P0 + 1) * sizeof(double complex));
    for (int p = 0; p < P0; p++) expn[p] = cexp(I * ((p + 1) * M_PI / 2));
    for (int i = 2; i < L; i++) {
      int ns = c->nsamp[i];
      double a = c->csize[i];
      c->trans[i] = calloc(49 * (size_t)ns, sizeof(double complex));
      for (int m = 0; m < c->nclus[i]; m++)
        for (int q = 0; q < 27; q++) {
          int n = c->farl[i][m * 27 + q];
          if (n == -1) continue;
          double complex d = c->cen[i][n] - c->cen[i][m];
          int nn = (int)round(creal(d) / a) + 3, mm = (int)round(-cimag(d) / a) + 3;
          c->traid[i][m * 27 + q] = mm * 7 + nn;
        }
      for (int cm = 0; cm < 7; cm++)
        for (int cn = 0; cn < 7; cn++) {
          double complex r = -((-3 * a + cn * a) + I * (3 * a - cm * a));
          if (!(cabs(r) > a * sqrt(3))) continue;
          for (int p = 0; p < c->nterm[i] + 1; p++) hank[p] = hn(p, c->k0 * cabs(r));
          for (int k = 0; k < ns; k++) {
            double complex red = hank[0];
            for (int p = 1; p < c->nterm[i] + 1; p++)
              red += 2 * cos(p * (2 * M_PI * k / ns - carg(r))) * hank[p] * expn[p - 1];
            c->trans[i][(cm * 7 + cn) * (size_t)ns + k] = red;
          }
        }
    }
    free(hank);
    free(expn);
  }

  /* setup_mlfma.cpp:544-553 */
  {
    int ns = c->nsamp[L - 1];
    c->coeff = malloc((size_t)ns * bb * sizeof(double complex));
    c->basis = malloc((size_t)ns * bb * sizeof(double complex));
    for (int n = 0; n < bb; n++)
      for (int k = 0; k < ns; k++) {
        c->coeff[k * bb + n] = plane_wave(c, c->cen[L - 1][0], c->pos[n], k, -1);
        c->basis[n * ns + k] = plane_wave(c, c->cen[L - 1][0], c->pos[n], k, +1) / (double complex)ns * (0.25 * I);
      }
  }

  /* setup_mlfma.cpp:554-570 */
  c->shm = calloc(L, sizeof(double complex *));
  c->shl = calloc(L, sizeof(double complex *));
  for (int i = 0; i < L - 1; i++) {
    int ns = c->nsamp[i];
    c->shm[i] = malloc(4 * (size_t)ns * sizeof(double complex));
    c->shl[i] = malloc(4 * (size_t)ns * sizeof(double complex));
    for (int q = 0; q < 4; q++) {
      double complex rho = c->cen[i][0] - c->cen[i + 1][q];
      for (int k = 0; k < ns; k++) {
        double ang = 2 * M_PI * k / ns;
        double kx = k0 * cos(ang), ky = k0 * sin(ang);
        double prod = kx * creal(rho) + ky * cimag(rho);
        c->shm[i][q * ns + k] = cexp(I * prod);
        c->shl[i][q * ns + k] = cexp(-I * prod);
      }
    }
  }

  /* setup_mlfma.cpp:571-599 */
  c->interp = calloc(L, sizeof(double *));
  c->intind = calloc(L, sizeof(int *));
  for (int i = 0; i < L - 1; i++) {
    int ns = c->nsamp[i];
    c->interp[i] = malloc((size_t)ns * ninter * sizeof(double));
    c->intind[i] = malloc((size_t)ns * ninter * sizeof(int));
    for (int m = 0; m < ns; m++)
      lagrange_row(m, ns, c->nsamp[i + 1], ninter, &c->interp[i][m * ninter], &c->intind[i][m * ninter]);
  }

  /* setup_mlfma.cpp:600-631: transposed interpolators, scaled by the rate
   * ratio and rotated so that each row's taps are contiguous modulo Q. */
  c->anterp = calloc(L, sizeof(double *));
  c->antind = calloc(L, sizeof(int *));
  {
    int w = 2 * ninter;
    int *tmpi = malloc(w * sizeof(int));
    double *tmpd = malloc(w * sizeof(double));
    for (int i = 1; i < L; i++) {
      int ns = c->nsamp[i], nsp = c->nsamp[i - 1];
      int *list = calloc(ns, sizeof(int));
      c->anterp[i] = calloc((size_t)ns * w, sizeof(double));
      c->antind[i] = calloc((size_t)ns * w, sizeof(int));
      for (int m = 0; m < nsp; m++)
        for (int n = 0; n < ninter; n++) {
          int ind = c->intind[i - 1][m * ninter + n];
          if (list[ind] >= w) abort();
          c->antind[i][ind * w + list[ind]] = m;
          c->anterp[i][ind * w + list[ind]] = c->interp[i - 1][m * ninter + n] * ns / nsp;
          list[ind]++;
        }
      for (int m = 0; m < ns; m++) {
        int *ai = &c->antind[i][m * w];
        double *ad = &c->anterp[i][m * w];
        for (int n = 1; n < list[m]; n++)
          if (ai[n] != ai[n - 1] + 1) {
            int cnt = list[m];
            memcpy(tmpi, ai + n, (cnt - n) * sizeof(int));
            memcpy(tmpd, ad + n, (cnt - n) * sizeof(double));
            memcpy(tmpi + cnt - n, ai, n * sizeof(int));
            memcpy(tmpd + cnt - n, ad, n * sizeof(double));
            memcpy(ai, tmpi, cnt * sizeof(int));
            memcpy(ad, tmpd, cnt * sizeof(double));
            break;
          }
      }
      free(list);
    }
    free(tmpi);
    free(tmpd);
  }

  /* setup_mlfma.cpp:642-695: receiver ring interpolation and its transpose. */
  {
    int ns0 = c->nsamp[0], w = 2 * ninter;
    c->interph = malloc((size_t)numrx * ninter * sizeof(double));
    c->intindh = malloc((size_t)numrx * ninter * sizeof(int));
    c->anterph = calloc((size_t)ns0 * w, sizeof(double));
    c->antindh = calloc((size_t)ns0 * w, sizeof(int));
    for (int m = 0; m < numrx; m++) lagrange_row(m, numrx, ns0, ninter, &c->interph[m * ninter], &c->intindh[m * ninter]);
    int *list = calloc(ns0, sizeof(int));
    for (int m = 0; m < numrx; m++)
      for (int n = 0; n < ninter; n++) {
        int ind = c->intindh[m * ninter + n];
        if (list[ind] >= w) abort();
        c->antindh[ind * w + list[ind]] = m;
        c->anterph[ind * w + list[ind]] = c->interph[m * ninter + n] * ns0 / numrx;
        list[ind]++;
      }
    free(list);
  }

  c->mul = calloc(L, sizeof(double complex *));
  c->loc = calloc(L, sizeof(double complex *));
  for (int i = 0; i < L; i++) {
    c->mul[i] = calloc((size_t)c->nclus[i] * c->nsamp[i], sizeof(double complex));
    c->loc[i] = calloc((size_t)c->nclus[i] * c->nsamp[i], sizeof(double complex));
  }
  c->buf = calloc(U, sizeof(double complex));
  return c;
}

void orc_destroy(orc_ctx *c) {
  if (!c) return;
  free(c->go);
  for (int i = 0; i < c->L; i++) {
    free(c->cen[i]);
    free(c->par[i]);
    free(c->nearl[i]);
    free(c->farl[i]);
    free(c->traid[i]);
    free(c->trans[i]);
    free(c->interp[i]);
    free(c->intind[i]);
    free(c->anterp[i]);
    free(c->antind[i]);
    free(c->shm[i]);
    free(c->shl[i]);
    free(c->mul[i]);
    free(c->loc[i]);
  }
  free(c->cen);
  free(c->par);
  free(c->nearl);
  free(c->farl);
  free(c->traid);
  free(c->trans);
  free(c->interp);
  free(c->intind);
  free(c->anterp);
  free(c->antind);
  free(c->shm);
  free(c->shl);
  free(c->mul);
  free(c->loc);
  free(c->nclus);
  free(c->nsamp);
  free(c->nterm);
  free(c->csize);
  free(c->pos);
  free(c->unkmap);
  free(c->nearT);
  free(c->coeff);
  free(c->basis);
  free(c->interph);
  free(c->intindh);
  free(c->anterph);
  free(c->antindh);
  free(c->buf);
  free(c);
}

int orc_numunk(const orc_ctx *c) { return c->U; }
int orc_numsamp(const orc_ctx *c, int lvl) { return c->nsamp[lvl]; }

const void *orc_table(const orc_ctx *c, const char *name, int lvl) {
#define T(nm, expr) \
  if (!strcmp(name, nm)) return (const void *)(expr);
  T("numclus", c->nclus)
  T("numsamp", c->nsamp)
  T("numterm", c->nterm)
  T("clusize", c->csize)
  T("clusc", c->cen[lvl])
  T("clusnear", c->nearl[lvl])
  T("clusfar", c->farl[lvl])
  T("traid", c->traid[lvl])
  T("near", c->nearT)
  T("coeff_multi", c->coeff)
  T("basis_local", c->basis)
  T("interp", c->interp[lvl])
  T("intind", c->intind[lvl])
  T("anterp", c->anterp[lvl])
  T("antind", c->antind[lvl])
  T("shiftmul", c->shm[lvl])
  T("shiftloc", c->shl[lvl])
  T("trans", c->trans[lvl])
  T("interph", c->interph)
  T("intindh", c->intindh)
  T("anterph", c->anterph)
  T("antindh", c->antindh)
  T("pos", c->pos)
  T("unkmap", c->unkmap)
#undef T
  return NULL;
}

/* solve.cpp:80-92 */
static void p2m(orc_ctx *c, const double complex *x) {
  int L = c->L, bb = c->bb, ns = c->nsamp[L - 1];
#pragma omp parallel for
  for (int m = 0; m < c->nclus[L - 1]; m++)
    for (int k = 0; k < ns; k++) {
      double complex red = 0;
      for (int n = 0; n < bb; n++) red += c->coeff[k * bb + n] * x[m * bb + n];
      c->mul[L - 1][(size_t)m * ns + k] = red;
    }
}

/* solve.cpp:93-112: interpolate the four children to the parent rate, shift
 * to the parent centre and sum. */
static void m2m(orc_ctx *c, int i) {
  int ns = c->nsamp[i], nsc = c->nsamp[i + 1], ni = c->ninter;
#pragma omp parallel for
  for (int m = 0; m < c->nclus[i]; m++)
    for (int km = 0; km < ns; km++) {
      double complex t1 = 0;
      for (int q = 0; q < 4; q++) {
        const double complex *ch = &c->mul[i + 1][(size_t)(m * 4 + q) * nsc];
        double complex red = 0;
        for (int k = 0; k < ni; k++) red += c->interp[i][km * ni + k] * ch[c->intind[i][km * ni + k]];
        t1 += red * c->shm[i][q * ns + km];
      }
      c->mul[i][(size_t)m * ns + km] = t1;
    }
}

/* solve.cpp:133-148 */
static void m2l(orc_ctx *c, int i) {
  int ns = c->nsamp[i];
#pragma omp parallel for
  for (int m = 0; m < c->nclus[i]; m++)
    for (int q = 0; q < 27; q++) {
      int n = c->farl[i][m * 27 + q];
      if (n == -1) continue;
      const double complex *t = &c->trans[i][(size_t)c->traid[i][m * 27 + q] * ns];
      for (int k = 0; k < ns; k++) c->loc[i][(size_t)m * ns + k] += t[k] * c->mul[i][(size_t)n * ns + k];
    }
}

/* solve.cpp:149-169 (accumulate) and :389-429 (overwrite): shift the parent's
 * local expansion to each child centre and anterpolate to the child rate. */
static void l2l(orc_ctx *c, int i, int overwrite) {
  int ns = c->nsamp[i], nsc = c->nsamp[i + 1], w = 2 * c->ninter;
#pragma omp parallel
  {
    double complex *tmp = malloc(ns * sizeof(double complex));
#pragma omp for
    for (int n = 0; n < c->nclus[i]; n++)
      for (int q = 0; q < 4; q++) {
        for (int kn = 0; kn < ns; kn++) tmp[kn] = c->shl[i][q * ns + kn] * c->loc[i][(size_t)n * ns + kn];
        double complex *dst = &c->loc[i + 1][(size_t)(n * 4 + q) * nsc];
        for (int km = 0; km < nsc; km++) {
          double complex red = 0;
          for (int k = 0; k < w; k++) red += c->anterp[i + 1][km * w + k] * tmp[c->antind[i + 1][km * w + k]];
          dst[km] = overwrite ? red : dst[km] + red;
        }
      }
    free(tmp);
  }
}

/* solve.cpp:170-182 (and :430-442) */
static void l2p(orc_ctx *c, double complex *r) {
  int L = c->L, bb = c->bb, ns = c->nsamp[L - 1];
#pragma omp parallel for
  for (int m = 0; m < c->nclus[L - 1]; m++)
    for (int n = 0; n < bb; n++) {
      double complex red = 0;
      for (int k = 0; k < ns; k++) red += c->basis[n * ns + k] * c->loc[L - 1][(size_t)m * ns + k];
      r[m * bb + n] = red;
    }
}

/* solve.cpp:199-216 */
static void p2p(orc_ctx *c, const double complex *x, double complex *r) {
  int L = c->L, bb = c->bb;
#pragma omp parallel for
  for (int m = 0; m < c->nclus[L - 1]; m++)
    for (int t = 0; t < bb; t++) {
      double complex red = 0;
      for (int s = 0; s < 9; s++) {
        int n = c->nearl[L - 1][m * 9 + s];
        if (n == -1) continue;
        const double complex *blk = &c->nearT[(size_t)s * bb * bb + t * bb];
        for (int q = 0; q < bb; q++) red += x[n * bb + q] * blk[q];
      }
      r[m * bb + t] += red;
    }
}

/* solve.cpp:25-248 */
void orc_mlfma(orc_ctx *c, const double complex *x, double complex *r) {
  int L = c->L;
  for (int i = 0; i < L; i++) memset(c->loc[i], 0, (size_t)c->nclus[i] * c->nsamp[i] * sizeof(double complex));
  p2m(c, x);
  for (int i = L - 2; i > 1; i--) m2m(c, i);
  for (int i = 2; i < L; i++) m2l(c, i);
  for (int i = 2; i < L - 1; i++) l2l(c, i, 0);
  l2p(c, r);
  p2p(c, x, r);
}

/* solve.cpp:8-24 */
void orc_mlfmah(orc_ctx *c, const double complex *x, double complex *r) {
  for (int n = 0; n < c->U; n++) c->buf[n] = conj(x[n]);
  double complex *tmp = malloc(c->U * sizeof(double complex));
  memcpy(tmp, c->buf, c->U * sizeof(double complex));
  orc_mlfma(c, tmp, r);
  free(tmp);
  for (int n = 0; n < c->U; n++) r[n] = conj(r[n]);
}

void orc_dense_matvec(const orc_ctx *c, const double complex *x, double complex *r) {
#pragma omp parallel for schedule(dynamic, 16)
  for (int m = 0; m < c->U; m++) {
    double complex red = 0;
    for (int n = 0; n < c->U; n++) red += orc_integrate(c, c->pos[m], c->pos[n]) * x[n];
    r[m] = red;
  }
}

/* bicgs.cpp:62-87 */
void orc_matvec(orc_ctx *c, const double complex *x, const double complex *g, double complex *y, int hermitian) {
  int U = c->U;
  double complex *in = malloc(U * sizeof(double complex));
  if (hermitian)
    for (int n = 0; n < U; n++) in[n] = conj(x[n]);
  else
    for (int n = 0; n < U; n++) in[n] = g[n] * x[n];
  orc_mlfma(c, in, y);
  if (hermitian)
    for (int n = 0; n < U; n++) y[n] = x[n] - conj(g[n] * y[n]);
  else
    for (int n = 0; n < U; n++) y[n] = x[n] - y[n];
  free(in);
}

static double norm2(const double complex *a, int U) {
  double s = 0;
  for (int m = 0; m < U; m++) s += creal(a[m]) * creal(a[m]) + cimag(a[m]) * cimag(a[m]);
  return s;
}

static double complex inner(const double complex *a, const double complex *b, int U) {
  double complex s = 0;
  for (int m = 0; m < U; m++) s += conj(a[m]) * b[m];
  return s;
}

/* bicgs.cpp:88-179 */
int orc_bicgs(orc_ctx *c, double complex *x, const double complex *g, const double complex *b, int hermitian,
              double tol, int maxit, double *err) {
  int U = c->U;
  size_t bytes = U * sizeof(double complex);
  double complex *r = malloc(bytes), *rt = malloc(bytes), *p = malloc(bytes), *v = malloc(bytes);
  double complex *s = malloc(bytes), *t = malloc(bytes);
  double complex alpha = 0, beta, omega = 0, rho, rho1 = 0;
  int iter = 0;
  double bn = sqrt(norm2(b, U));
  if (bn < 1e-20) bn = 1;
  orc_matvec(c, x, g, r, hermitian);
  for (int n = 0; n < U; n++) r[n] = b[n] - r[n];
  double error = sqrt(norm2(r, U)) / bn;
  if (error > tol) {
    memcpy(rt, r, bytes);
    while (iter < maxit) {
      iter++;
      rho = inner(rt, r, U);
      if (cabs(rho) < 1e-20) break;
      if (iter == 1)
        memcpy(p, r, bytes);
      else {
        beta = (rho / rho1) * (alpha / omega);
        for (int n = 0; n < U; n++) p[n] = r[n] + beta * (p[n] - omega * v[n]);
      }
      orc_matvec(c, p, g, v, hermitian);
      alpha = rho / inner(rt, v, U);
      for (int n = 0; n < U; n++) s[n] = r[n] - alpha * v[n];
      orc_matvec(c, s, g, t, hermitian);
      /* bicgs.cpp:153, with the guard of the linked GPU solver (bicgs_gpu.cu:
       * 373-376) for t = s = 0, which the reference's -ffast-math CPU build
       * also resolves to a finite omega */
      double complex ts = inner(t, s, U);
      double tt = norm2(t, U);
      omega = (cabs(ts) < 1e-200 && tt < 1e-200) ? 1.0 : ts / tt;
      for (int n = 0; n < U; n++) {
        x[n] = x[n] + alpha * p[n] + omega * s[n];
        r[n] = s[n] - omega * t[n];
      }
      error = sqrt(norm2(r, U)) / bn;
      if (error < tol) break;
      if (cabs(omega) < 1e-20) break;
      rho1 = rho;
    }
  }
  if (err) *err = error;
  free(r);
  free(rt);
  free(p);
  free(v);
  free(s);
  free(t);
  return iter;
}

/* solve.cpp:249-355 */
void orc_aggregate(orc_ctx *c, const double complex *x, double complex *rx) {
  int L = c->L, ni = c->ninter;
  p2m(c, x);
  for (int i = L - 2; i > 1; i--) m2m(c, i);
  for (int i = 1; i > -1; i--) m2m(c, i);
  for (int m = 0; m < c->numrx; m++) {
    double complex red = 0;
    for (int k = 0; k < ni; k++) red += c->interph[m * ni + k] * c->mul[0][c->intindh[m * ni + k]];
    rx[m] = red;
  }
}

/* solve.cpp:356-456 */
void orc_aggregateh(orc_ctx *c, double complex *x, const double complex *rx) {
  int L = c->L, w = 2 * c->ninter;
  for (int m = 0; m < c->nsamp[0]; m++) {
    double complex red = 0;
    for (int k = 0; k < w; k++) red += c->anterph[m * w + k] * rx[c->antindh[m * w + k]];
    c->loc[0][m] = red * (-4 * I) * (double complex)(c->numrx * c->res * c->res);
  }
  for (int i = 0; i < L - 1; i++) l2l(c, i, 1);
  l2p(c, x);
}

/* Near-field receivers (the reference's commented dense form, setup_born.cpp:52-60):
 * numrx points at radius (cos, sin)(360 / numrx m degrees) (mom.cpp:149-154 at a
 * finite radius), go[m][n] = integrate(rx_m, pos_n).  radius 0 removes them. */
void orc_set_nearfield(orc_ctx *c, double radius) {
  free(c->go);
  c->go = NULL;
  if (radius == 0) return;
  c->go = malloc((size_t)c->numrx * c->U * sizeof(double complex));
  for (int m = 0; m < c->numrx; m++) {
    double ang = 360.0 / c->numrx * m;
    double complex r = radius * (cos(ang / 360 * 2 * M_PI) + I * sin(ang / 360 * 2 * M_PI));
    for (int n = 0; n < c->U; n++) c->go[(size_t)m * c->U + n] = orc_integrate(c, r, c->pos[n]);
  }
}

/* rx = go x with near-field receivers, else the far-field aggregate. */
void orc_receive(orc_ctx *c, const double complex *x, double complex *rx) {
  if (!c->go) {
    orc_aggregate(c, x, rx);
    return;
  }
  for (int m = 0; m < c->numrx; m++) {
    double complex s = 0;
    for (int n = 0; n < c->U; n++) s += c->go[(size_t)m * c->U + n] * x[n];
    rx[m] = s;
  }
}

/* x = gh rx, gh = conj(go)^T (setup_born.cpp:57-59), else the far-field aggregateh. */
void orc_receiveh(orc_ctx *c, double complex *x, const double complex *rx) {
  if (!c->go) {
    orc_aggregateh(c, x, rx);
    return;
  }
  for (int n = 0; n < c->U; n++) x[n] = 0;
  for (int m = 0; m < c->numrx; m++)
    for (int n = 0; n < c->U; n++) x[n] += conj(c->go[(size_t)m * c->U + n]) * rx[m];
}

/* One write_error record (setup_born.cpp:171-242). */
static void dbim_record(const orc_ctx *c, int ntx, const double complex *mesd, const double complex *od,
                        const double complex *o, const double complex *otrue, double regular, double mesnorm,
                        double objnorm, double *rec) {
  int U = c->U;
  double err = 0, errd = 0, obj = 0, objn = 0, errm = 0;
  for (int m = 0; m < ntx * c->numrx; m++) err += creal(mesd[m] * conj(mesd[m]));
  for (int n = 0; n < U; n++) {
    errd += creal(od[n] * conj(od[n]));
    double complex ro = regular * o[n];
    obj += creal(ro * conj(ro));
    objn += creal(o[n] * conj(o[n]));
    double complex d = o[n] - otrue[n];
    errm += creal(d * conj(d));
  }
  rec[0] = err / mesnorm;
  rec[1] = errm / objnorm;
  rec[2] = obj / mesnorm;
  rec[3] = errd;
  rec[4] = objn;
}

/* mom.cpp:247-271 (and 338-362): gradient od of the misfit at contrast o. */
static void dbim_gradient(orc_ctx *c, int ntx, const double complex *o, const double complex *tot,
                          const double complex *mesd, double regular, double tol, int maxit, double complex *od) {
  int U = c->U;
  double k2 = c->k0 * c->k0;
  double complex *y = malloc(U * sizeof(double complex)), *cc = malloc(U * sizeof(double complex));
  double complex *g = malloc(U * sizeof(double complex)), *x = malloc(U * sizeof(double complex));
  for (int n = 0; n < U; n++) od[n] = 0;
  for (int i = 0; i < ntx; i++) {
    orc_receiveh(c, y, &mesd[i * c->numrx]);
    for (int n = 0; n < U; n++) {
      cc[n] = conj(o[n] * k2) * y[n];
      g[n] = o[n] * k2;
      x[n] = 0;
    }
    orc_bicgs(c, x, g, cc, 1, tol, maxit, NULL);
    orc_mlfmah(c, x, cc);
    for (int n = 0; n < U; n++) {
      y[n] += cc[n];
      od[n] += conj(tot[(size_t)i * U + n]) * y[n];
      od[n] += regular * regular * o[n];
    }
  }
  free(y);
  free(cc);
  free(g);
  free(x);
}

int orc_dbim(orc_ctx *c, int ntx, const double complex *inc, const double complex *chi_true, int iterations,
             double regular, double tol, int maxit, double complex *o, double *hist, double *alpha,
             double complex *beta) {
  int U = c->U, nr = c->numrx;
  double k2 = c->k0 * c->k0;
  size_t fb = (size_t)ntx * U * sizeof(double complex), mb = (size_t)ntx * nr * sizeof(double complex);
  double complex *tot = malloc(fb), *mes = malloc(mb), *mesd = malloc(mb), *rhs = malloc(mb);
  double complex *od = malloc(U * sizeof(double complex)), *ot = malloc(U * sizeof(double complex));
  double complex *save = malloc(U * sizeof(double complex)), *g = malloc(U * sizeof(double complex));
  double complex *x = malloc(U * sizeof(double complex)), *y = malloc(U * sizeof(double complex));
  double complex *cc = malloc(U * sizeof(double complex));
  /* setup_born.cpp:139-149: measurements of the true contrast */
  for (int n = 0; n < U; n++) g[n] = chi_true[n] * k2;
  for (int i = 0; i < ntx; i++) {
    for (int n = 0; n < U; n++) x[n] = 0;
    orc_bicgs(c, x, g, &inc[(size_t)i * U], 0, tol, maxit, NULL);
    for (int n = 0; n < U; n++) x[n] *= g[n];
    orc_receive(c, x, &mes[i * nr]);
  }
  double objnorm = 0, mesnorm = 0;
  for (int n = 0; n < U; n++) objnorm += creal(chi_true[n] * conj(chi_true[n]));
  for (int m = 0; m < ntx * nr; m++) mesnorm += creal(mes[m] * conj(mes[m]));
  /* mom.cpp:224-229: no object, total field = incident */
  for (int n = 0; n < U; n++) o[n] = 0;
  memcpy(tot, inc, fb);
  for (int m = 0; m < ntx * nr; m++) mesd[m] = -mes[m];
  dbim_gradient(c, ntx, o, tot, mesd, regular, tol, maxit, od);
  dbim_record(c, ntx, mesd, od, o, chi_true, regular, mesnorm, objnorm, &hist[0]);
  memcpy(ot, od, U * sizeof(double complex));
  for (int it = 0; it < iterations; it++) {
    /* mom.cpp:280-316: Born-linearised step length */
    for (int i = 0; i < ntx; i++) {
      for (int n = 0; n < U; n++) y[n] = tot[(size_t)i * U + n] * ot[n] * k2;
      orc_mlfma(c, y, cc);
      for (int n = 0; n < U; n++) {
        x[n] = 0;
        g[n] = o[n] * k2;
      }
      orc_bicgs(c, x, g, cc, 0, tol, maxit, NULL);
      for (int n = 0; n < U; n++) y[n] += o[n] * k2 * x[n];
      orc_receive(c, y, &rhs[i * nr]);
    }
    double complex t1 = 0;
    double t2 = 0;
    for (int m = 0; m < ntx * nr; m++) {
      t1 += conj(mesd[m]) * rhs[m];
      t2 += creal(rhs[m] * conj(rhs[m]));
    }
    double a = creal(t1) / t2;
    alpha[it] = a;
    /* mom.cpp:318-336: step, then re-solve the total fields */
    for (int n = 0; n < U; n++) o[n] -= a * ot[n];
    for (int n = 0; n < U; n++) g[n] = o[n] * k2;
    for (int i = 0; i < ntx; i++) {
      double complex *ti = &tot[(size_t)i * U];
      for (int n = 0; n < U; n++) ti[n] = 0;
      orc_bicgs(c, ti, g, &inc[(size_t)i * U], 0, tol, maxit, NULL);
      for (int n = 0; n < U; n++) x[n] = ti[n] * o[n] * k2;
      orc_receive(c, x, &rhs[i * nr]);
      for (int m = 0; m < nr; m++) mesd[i * nr + m] = rhs[i * nr + m] - mes[i * nr + m];
    }
    memcpy(save, od, U * sizeof(double complex));
    dbim_gradient(c, ntx, o, tot, mesd, regular, tol, maxit, od);
    dbim_record(c, ntx, mesd, od, o, chi_true, regular, mesnorm, objnorm, &hist[5 * (it + 1)]);
    /* mom.cpp:383-399: Polak-Ribiere direction */
    double complex n1 = 0;
    double n2 = 0;
    for (int n = 0; n < U; n++) {
      n1 += od[n] * conj(od[n] - save[n]);
      n2 += creal(save[n] * conj(save[n]));
    }
    double complex b = n1 / n2;
    beta[it] = b;
    for (int n = 0; n < U; n++) ot[n] = od[n] + b * ot[n];
  }
  free(tot);
  free(mes);
  free(mesd);
  free(rhs);
  free(od);
  free(ot);
  free(save);
  free(g);
  free(x);
  free(y);
  free(cc);
  return 0;
}
