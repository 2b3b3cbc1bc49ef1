// The reference's integrate (integrate.cpp:15-41) as a device function, FP64:
// the Green's function entry (i/4) res^2 H_0(k0 d) between two pixel centres
// (point approximation), and for a pixel's own centre the log singularity of
// Y_0 integrated analytically over the square (the antiderivative of
// integrate.cpp:11-13).  J_0 and Y_0 come from the CUDA math library.
#pragma once

#include <cmath>

namespace isg {

constexpr double kPiD = 3.14159265358979323846;

__device__ inline double log_rect_d(double x, double y) {
  return -3 * x * y + x * y * log(x * x + y * y) + x * x * atan(y / x) + y * y * atan(x / y);
}

// Entry for the displacement (basis point - testing point) = (dx, dy).
__device__ inline double2 green_entry_d(double k0, double res, double dx, double dy) {
  const double dist = hypot(dx, dy);
  double vr = j0(k0 * dist), vi, si = 0.0;
  if (dist < res / 8) {
    vi = 0.5772156649015329 * 2 / kPiD + 2 / kPiD * log(0.5);
    const double x0 = dx - res / 2, x1 = dx + res / 2, y0v = dy - res / 2, y1v = dy + res / 2;
    const double area_log = log_rect_d(x1, y1v) - log_rect_d(x0, y1v) - log_rect_d(x1, y0v) + log_rect_d(x0, y0v);
    si = (area_log / 2 + log(k0) * res * res) * 2 / kPiD;
  } else {
    vi = y0(k0 * dist);
  }
  vr *= res * res;
  vi *= res * res;
  // (value + i si) * i / 4
  return make_double2(-(vi + si) * 0.25, vr * 0.25);
}

}  // namespace isg
