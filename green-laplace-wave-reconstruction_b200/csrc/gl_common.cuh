// Shared device helpers for the Green--Laplace engine: complex arithmetic,
// spectral boxes, per-bin finite-depth geometry and the FFT conventions.
//
// Layout conventions (all device buffers):
//   * complex values are interleaved (re, im) doubles (double2);
//   * a spectral "box" is the rectangle [x0, x0+w) x [y0, y0+h) of signed mode
//     numbers (mx, my) that contains a spectrum's support; box arrays are
//     row-major [h][w] (row = y), matching the reference's [iy, ix] layout;
//   * spectra are N^2-scaled like numpy.fft.fft2 of the reference grid, so a
//     physical value is (1/(Nx Ny)) sum_k S_k e^{i k x}.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define GL_HD __host__ __device__ __forceinline__
#define GL_D __device__ __forceinline__

namespace gl {

typedef double2 cplx;

GL_HD cplx cmk(double r, double i) { return make_double2(r, i); }
GL_HD cplx cadd(cplx a, cplx b) { return cmk(a.x + b.x, a.y + b.y); }
GL_HD cplx csub(cplx a, cplx b) { return cmk(a.x - b.x, a.y - b.y); }
GL_HD cplx cmul(cplx a, cplx b) { return cmk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
GL_HD cplx cscale(double s, cplx a) { return cmk(s * a.x, s * a.y); }
// multiply by i and by -i
GL_HD cplx cmuli(cplx a) { return cmk(-a.y, a.x); }
GL_HD cplx cmulmi(cplx a) { return cmk(a.y, -a.x); }
GL_HD cplx csq(cplx a) { return cmul(a, a); }
GL_HD cplx czero() { return cmk(0.0, 0.0); }
GL_HD cplx cconj(cplx a) { return cmk(a.x, -a.y); }

// |z| as numpy computes it (hypot).
GL_D double cabs_(cplx a) { return hypot(a.x, a.y); }

// hypot(v) < t, numpy's |z| comparison (a squared-magnitude shortcut that
// skips hypot away from t measured slower in the accumulation kernels).
GL_D bool abs_below(cplx v, double t) { return cabs_(v) < t; }

// Running max of |v| = hypot(v) with NaN propagation.
GL_D double keep_max_abs(double cur, cplx v) {
  const double m = cabs_(v);
  return (m > cur || m != m) ? m : cur;
}

// Max of non-negative doubles through the integer order of their bit patterns.
// NaN patterns order above +inf, so a NaN input propagates to the result.
GL_D void atomic_max_nonneg(unsigned long long* slot, double v) {
  atomicMax(slot, (unsigned long long)__double_as_longlong(v));
}
GL_D double as_double(unsigned long long bits) { return __longlong_as_double((long long)bits); }

// Index of signed mode number m on a periodic grid of length n (power of two).
GL_HD int wrap(int m, int n) { return m & (n - 1); }

// The same for any length n > 0 (column grids of length 16 m, m not a power
// of two); the power-of-two test is uniform across a launch.
GL_HD int wrap_any(int m, int n) {
  if ((n & (n - 1)) == 0) return m & (n - 1);
  if (m < 0) m += n;  // callers pass -n <= m < 2n: no division
  else if (m >= n) m -= n;
  if (m >= 0 && m < n) return m;
  const int r = m % n;
  return r < 0 ? r + n : r;
}

struct Box {
  int x0, y0, w, h;  // signed mode origin, width (x) and height (y)
};

// Per-bin finite-depth geometry of a box, stored as separate planes of
// length w*h: qx, qy, q, nu (= sqrt(q tanh q)), A (= q tanh q), sqrtA.
struct GeoPlanes {
  const double* qx;
  const double* qy;
  const double* q;
  const double* nu;
  const double* a;
  const double* sqrt_a;
};

GL_D double safe_nu(double nu) { return nu > 2.2250738585072014e-308 ? nu : 2.2250738585072014e-308; }

// sinh(sqrt(A) tau)/sqrt(A) with its tau limit at A = 0.
GL_D double sinh_over_root(double sqrt_a, double tau) {
  return sqrt_a > 0.0 ? sinh(sqrt_a * tau) / sqrt_a : tau;
}

}  // namespace gl
