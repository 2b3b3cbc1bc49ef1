/* Seeded synthetic inputs of the benchmark workloads: the random-ellipse
 * contrast and the plane-wave incident fields that the product library's
 * isg_make_phantom (kind 0) and isg_make_plane_waves write, restated with the
 * same arithmetic in the same order, so that the reference's side of a
 * comparison gets bit-identical inputs without loading the product library.
 *
 * Test and benchmark infrastructure only (part of liboracle.so): tests/ and
 * bench.py's reference arm call it; nothing in the product links it.
 *
 * The reference itself reads its contrast from a phantom file
 * (setup_born.cpp:103-113) and builds plane waves exp(i k0 d.r) over its pixel
 * centres (setup_born.cpp:62-65); the file does not exist, so seeded ellipses
 * stand in for it. */
#define _DEFAULT_SOURCE /* M_PI, as the library takes it from <cmath> */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "isg_oracle.h"

static uint64_t splitmix(uint64_t *s) {
  uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static double uniform(uint64_t *s) { return (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0); }

static double dmin(double a, double b) { return b < a ? b : a; }
static double dmax(double a, double b) { return a < b ? b : a; }

void orc_in_ellipses(int side, double res, int count, double axis_min, double axis_max, double eps_min,
                     double eps_max, double tand_max, uint64_t seed, double complex *chi) {
  const int S = side;
  const double D = S * res;
  uint64_t s = seed * 0x2545F4914F6CDD1Dull + 0x1234567ull;
  memset(chi, 0, sizeof(double complex) * (size_t)S * S);
  for (int e = 0; e < count; e++) {
    const double a = axis_min + (axis_max - axis_min) * uniform(&s);
    const double b = axis_min + (axis_max - axis_min) * uniform(&s);
    const double m = dmin(dmax(a, b), D / 2);
    const double cx = (-D / 2 + m) + (D - 2 * m) * uniform(&s);
    const double cy = (-D / 2 + m) + (D - 2 * m) * uniform(&s);
    const double th = M_PI * uniform(&s);
    const double eps = eps_min + (eps_max - eps_min) * uniform(&s);
    const double tand = tand_max * uniform(&s);
    const double ct = cos(th), st = sin(th);
    for (int Y = 0; Y < S; Y++)
      for (int X = 0; X < S; X++) {
        const double px = -D / 2 + (X + 0.5) * res - cx, py = D / 2 - (Y + 0.5) * res - cy;
        const double u = (ct * px + st * py) / a, v = (-st * px + ct * py) / b;
        if (u * u + v * v <= 1.0) chi[(size_t)Y * S + X] = CMPLX(eps - 1.0, eps * tand);
      }
  }
}

void orc_in_plane_waves(int side, double res, double k0, int ntx, int first, int count, const int *unkmap,
                        double complex *inc) {
  const int S = side;
  const double D = S * res;
  const size_t U = (size_t)S * S;
  for (int j = 0; j < count; j++) {
    const double ang = 2 * M_PI * (first + j) / ntx;
    const double dx = cos(ang), dy = sin(ang);
    for (int Y = 0; Y < S; Y++)
      for (int X = 0; X < S; X++) {
        const int r = Y * S + X;
        const double pr = -D / 2 + (X + 0.5) * res, pi = D / 2 - (Y + 0.5) * res;
        inc[(size_t)j * U + (unkmap ? (size_t)unkmap[r] : (size_t)r)] = cexp(CMPLX(0.0, k0 * (dx * pr + dy * pi)));
      }
  }
}
