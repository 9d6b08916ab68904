/*
 * fftw3_shim.c -- this project's implementation of the FFTW3 subset in
 * fftw3.h, for building the reference's order-4 executor
 * (paper/order4/cpp/gl_eta44_fftw.cpp) from its own source as a parity
 * oracle.  Test infrastructure only.
 *
 * A 2-D transform is a pass of 1-D transforms over the rows, then one over
 * the columns (each column gathered into a contiguous buffer).  Power-of-two
 * lengths use an iterative radix-2 Cooley-Tukey transform (bit-reversed
 * input order, in place); other lengths a direct O(n^2) sum with exact
 * (j k mod n) twiddle indexing.  Twiddles exp(sign 2 pi i k / n) are
 * evaluated in long double and rounded once.  The row and column passes are
 * spread over OpenMP threads (fftw_plan_with_nthreads).
 */
#include "fftw3.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

struct gl_fftw_plan_s {
  int n0, n1, sign;
  fftw_complex *in, *out;
  double* tw0; /* n0 twiddles (re, im) */
  double* tw1; /* n1 twiddles */
  int nthreads;
};

static int g_nthreads = 1;

void* fftw_malloc(size_t bytes) {
  void* p = NULL;
  if (posix_memalign(&p, 64, bytes ? bytes : 1) != 0) return NULL;
  return p;
}

void fftw_free(void* p) { free(p); }

int fftw_init_threads(void) { return 1; }

void fftw_plan_with_nthreads(int nthreads) { g_nthreads = nthreads > 0 ? nthreads : 1; }

void fftw_cleanup_threads(void) {}

static double* twiddles(int n, int sign) {
  double* w = (double*)malloc(sizeof(double) * 2 * (size_t)n);
  if (!w) return NULL;
  const long double two_pi = 6.283185307179586476925286766559005768L;
  for (int k = 0; k < n; ++k) {
    const long double a = two_pi * (long double)k / (long double)n;
    w[2 * k] = (double)cosl(a);
    w[2 * k + 1] = (double)(sign * sinl(a));
  }
  return w;
}

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

/* In-place length-n transform of x (n complex values) with twiddle table w
 * (w[k] = exp(sign 2 pi i k / n)); tmp holds n complex values of scratch. */
static void dft1(double* x, int n, const double* w, double* tmp) {
  if (n <= 1) return;
  if (is_pow2(n)) {
    /* bit-reversal permutation */
    for (int i = 1, j = 0; i < n; ++i) {
      int bit = n >> 1;
      for (; j & bit; bit >>= 1) j ^= bit;
      j ^= bit;
      if (i < j) {
        double t0 = x[2 * i], t1 = x[2 * i + 1];
        x[2 * i] = x[2 * j];
        x[2 * i + 1] = x[2 * j + 1];
        x[2 * j] = t0;
        x[2 * j + 1] = t1;
      }
    }
    for (int len = 2; len <= n; len <<= 1) {
      const int half = len >> 1, step = n / len;
      for (int s = 0; s < n; s += len) {
        for (int k = 0; k < half; ++k) {
          const double wr = w[2 * (k * step)], wi = w[2 * (k * step) + 1];
          double* a = x + 2 * (s + k);
          double* b = x + 2 * (s + k + half);
          const double br = b[0] * wr - b[1] * wi;
          const double bi = b[0] * wi + b[1] * wr;
          b[0] = a[0] - br;
          b[1] = a[1] - bi;
          a[0] += br;
          a[1] += bi;
        }
      }
    }
    return;
  }
  for (int k = 0; k < n; ++k) {
    double sr = 0.0, si = 0.0;
    long long idx = 0;
    for (int j = 0; j < n; ++j) {
      const double wr = w[2 * idx], wi = w[2 * idx + 1];
      sr += x[2 * j] * wr - x[2 * j + 1] * wi;
      si += x[2 * j] * wi + x[2 * j + 1] * wr;
      idx += k;
      if (idx >= n) idx -= n;
    }
    tmp[2 * k] = sr;
    tmp[2 * k + 1] = si;
  }
  memcpy(x, tmp, sizeof(double) * 2 * (size_t)n);
}

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex* in, fftw_complex* out, int sign,
                           unsigned flags) {
  (void)flags;
  if (n0 < 1 || n1 < 1 || !in || !out || (sign != FFTW_FORWARD && sign != FFTW_BACKWARD)) return NULL;
  fftw_plan p = (fftw_plan)calloc(1, sizeof(*p));
  if (!p) return NULL;
  p->n0 = n0;
  p->n1 = n1;
  p->sign = sign;
  p->in = in;
  p->out = out;
  p->tw0 = twiddles(n0, sign);
  p->tw1 = twiddles(n1, sign);
  p->nthreads = g_nthreads;
  if (!p->tw0 || !p->tw1) {
    fftw_destroy_plan(p);
    return NULL;
  }
  return p;
}

void fftw_execute(const fftw_plan p) {
  const int n0 = p->n0, n1 = p->n1;
  double* o = (double*)p->out;
  if (p->out != p->in) memcpy(o, p->in, sizeof(fftw_complex) * (size_t)n0 * n1);
  const int nmax = n0 > n1 ? n0 : n1;
#pragma omp parallel num_threads(p->nthreads)
  {
    double* col = (double*)malloc(sizeof(double) * 2 * (size_t)nmax);
    double* tmp = (double*)malloc(sizeof(double) * 2 * (size_t)nmax);
#pragma omp for schedule(static)
    for (int r = 0; r < n0; ++r) dft1(o + 2 * (size_t)r * n1, n1, p->tw1, tmp);
#pragma omp for schedule(static)
    for (int c = 0; c < n1; ++c) {
      for (int r = 0; r < n0; ++r) {
        col[2 * r] = o[2 * ((size_t)r * n1 + c)];
        col[2 * r + 1] = o[2 * ((size_t)r * n1 + c) + 1];
      }
      dft1(col, n0, p->tw0, tmp);
      for (int r = 0; r < n0; ++r) {
        o[2 * ((size_t)r * n1 + c)] = col[2 * r];
        o[2 * ((size_t)r * n1 + c) + 1] = col[2 * r + 1];
      }
    }
    free(col);
    free(tmp);
  }
}

void fftw_destroy_plan(fftw_plan p) {
  if (!p) return;
  free(p->tw0);
  free(p->tw1);
  free(p);
}
