// Register-resident power-of-two FFTs for lengths 16..4096.
//
// A length-n transform is run by a group of T = n/16 threads that each hold
// 16 complex values per pass.  Passes are Stockham autosort steps of radix 16
// (the last one radix 2, 4 or 8 when log2 n is not a multiple of 4), so a
// 256-point transform is two passes and a 1024-point one three, with one
// shared-memory round trip between passes instead of one per radix-4 stage.
// The first pass reads its inputs through a caller functor (global memory,
// on-the-fly multipliers, zero outside a spectral box) and the last pass
// hands its outputs to a caller functor (kept columns only, physical
// scaling), so intermediate rows never exist in global memory.
//
// Shared rows use a padded layout, element i at i + i/16, which keeps the
// stride-16 stores of the first pass free of bank conflicts.  Groups of at
// most 32 threads synchronise with __syncwarp; larger groups use one named
// barrier per group.
#pragma once
#include "gl_fft.cuh"

namespace gl {

GL_HD int phys(int i) { return i + (i >> 4); }
GL_HD int padded_len(int n) { return n + (n >> 4) + 1; }  // +1: odd stride between rows

// cos(pi/8), sin(pi/8), sqrt(2)/2
constexpr double FC8 = 0.92387953251128675613;
constexpr double FS8 = 0.38268343236508977173;
constexpr double FH2 = 0.70710678118654752440;

template <int SIGN>
GL_D cplx wconst(double re, double im_fwd) {  // forward constant (re, im); inverse: conjugate
  return cmk(re, SIGN < 0 ? im_fwd : -im_fwd);
}

template <int SIGN>
GL_D void dft2(cplx* v) {
  const cplx a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <int SIGN>
GL_D void dft4v(cplx* v) {
  cplx a = v[0], b = v[1], c = v[2], d = v[3];
  dft4<SIGN>(a, b, c, d);
  v[0] = a;
  v[1] = b;
  v[2] = c;
  v[3] = d;
}

// 8 = 2 x 4: X[k2 + 4 k1] = A[k2] + (-1)^k1 W8^k2 B[k2]
template <int SIGN>
GL_D void dft8(cplx* v) {
  cplx a0 = v[0], a1 = v[2], a2 = v[4], a3 = v[6];
  cplx b0 = v[1], b1 = v[3], b2 = v[5], b3 = v[7];
  dft4<SIGN>(a0, a1, a2, a3);
  dft4<SIGN>(b0, b1, b2, b3);
  b1 = cmul(b1, wconst<SIGN>(FH2, -FH2));
  b2 = SIGN < 0 ? cmulmi(b2) : cmuli(b2);
  b3 = cmul(b3, wconst<SIGN>(-FH2, -FH2));
  v[0] = cadd(a0, b0);
  v[4] = csub(a0, b0);
  v[1] = cadd(a1, b1);
  v[5] = csub(a1, b1);
  v[2] = cadd(a2, b2);
  v[6] = csub(a2, b2);
  v[3] = cadd(a3, b3);
  v[7] = csub(a3, b3);
}

// 16 = 4 x 4: Y[r1][k2] = DFT4_r2 x[r1 + 4 r2]; Y *= W16^(r1 k2);
// X[k2 + 4 k1] = DFT4_r1 Y[r1][k2]
template <int SIGN>
GL_D void dft16(cplx* v) {
  cplx y[16];
#pragma unroll
  for (int r1 = 0; r1 < 4; ++r1) {
    cplx a = v[r1], b = v[r1 + 4], c = v[r1 + 8], d = v[r1 + 12];
    dft4<SIGN>(a, b, c, d);
    y[4 * r1 + 0] = a;
    y[4 * r1 + 1] = b;
    y[4 * r1 + 2] = c;
    y[4 * r1 + 3] = d;
  }
  y[5] = cmul(y[5], wconst<SIGN>(FC8, -FS8));    // W16^1
  y[6] = cmul(y[6], wconst<SIGN>(FH2, -FH2));    // W16^2
  y[7] = cmul(y[7], wconst<SIGN>(FS8, -FC8));    // W16^3
  y[9] = cmul(y[9], wconst<SIGN>(FH2, -FH2));    // W16^2
  y[10] = SIGN < 0 ? cmulmi(y[10]) : cmuli(y[10]);  // W16^4
  y[11] = cmul(y[11], wconst<SIGN>(-FH2, -FH2));  // W16^6
  y[13] = cmul(y[13], wconst<SIGN>(FS8, -FC8));   // W16^3
  y[14] = cmul(y[14], wconst<SIGN>(-FH2, -FH2));  // W16^6
  y[15] = cmul(y[15], wconst<SIGN>(-FC8, FS8));   // W16^9
#pragma unroll
  for (int k2 = 0; k2 < 4; ++k2) {
    cplx a = y[k2], b = y[4 + k2], c = y[8 + k2], d = y[12 + k2];
    dft4<SIGN>(a, b, c, d);
    v[k2] = a;
    v[k2 + 4] = b;
    v[k2 + 8] = c;
    v[k2 + 12] = d;
  }
}

template <int SIGN, int R>
GL_D void dftR(cplx* v) {
  if (R == 2) dft2<SIGN>(v);
  if (R == 4) dft4v<SIGN>(v);
  if (R == 8) dft8<SIGN>(v);
  if (R == 16) dft16<SIGN>(v);
}

// v[r] *= W_{ns R}^(r k) for r = 1..R-1, from table values at m, 2m, 4m, 8m.
template <int SIGN, int R>
GL_D void apply_twiddles(cplx* v, int m, const cplx* __restrict__ tw) {
  const cplx w1 = twiddle<SIGN>(tw, m);
  if (R == 2) {
    v[1] = cmul(v[1], w1);
    return;
  }
  const cplx w2 = twiddle<SIGN>(tw, 2 * m);
  if (R == 4) {
    v[1] = cmul(v[1], w1);
    v[2] = cmul(v[2], w2);
    v[3] = cmul(v[3], twiddle<SIGN>(tw, 3 * m));
    return;
  }
  const cplx w4 = twiddle<SIGN>(tw, 4 * m);
  const cplx w3 = cmul(w1, w2);
  v[1] = cmul(v[1], w1);
  v[2] = cmul(v[2], w2);
  v[3] = cmul(v[3], w3);
  v[4] = cmul(v[4], w4);
  v[5] = cmul(v[5], cmul(w1, w4));
  v[6] = cmul(v[6], cmul(w2, w4));
  v[7] = cmul(v[7], cmul(w3, w4));
  if (R == 8) return;
  const cplx w8 = twiddle<SIGN>(tw, 8 * m);
  v[8] = cmul(v[8], w8);
  v[9] = cmul(v[9], cmul(w1, w8));
  v[10] = cmul(v[10], cmul(w2, w8));
  v[11] = cmul(v[11], cmul(w3, w8));
  const cplx w12 = cmul(w4, w8);
  v[12] = cmul(v[12], w12);
  v[13] = cmul(v[13], cmul(w1, w12));
  v[14] = cmul(v[14], cmul(w2, w12));
  v[15] = cmul(v[15], cmul(w3, w12));
}

// Synchronisation of one group of T threads.
struct GroupSync {
  int T, id;
  GL_D void operator()() const {
    if (T <= 32) {
      __syncwarp();
    } else {
      asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(T) : "memory");
    }
  }
};

struct FftGroup {
  int n, log2n;  // transform length
  int T;         // threads in the group (n / 16)
  int t;         // thread index inside the group
  GroupSync sync;
};

// Group geometry for a block of `threads` threads doing length-n transforms.
GL_D FftGroup fft_group(int n, int log2n, int& g, int& G) {
  FftGroup f;
  f.n = n;
  f.log2n = log2n;
  f.T = n >> 4;
  G = blockDim.x / f.T;
  g = threadIdx.x / f.T;
  f.t = threadIdx.x % f.T;
  f.sync = GroupSync{f.T, 1 + g};  // named barrier id per group (used when T > 32)
  return f;
}

// One Stockham pass of radix R over the padded row `buf`.
//   FIRST: pass inputs come from load(i) (else from buf), LAST: outputs go to
//   store(i, v) (else back to buf).  `active` = false runs the barriers only.
template <int SIGN, int R, bool FIRST, bool LAST, class Load, class Store>
GL_D void fft_pass(cplx* buf, const FftGroup& f, int ns, bool active, const cplx* __restrict__ tw,
                   Load& load, Store& store) {
  constexpr int B = 16 / R;
  const int stride = f.n / R;
  cplx v[16];
#pragma unroll
  for (int b = 0; b < B; ++b) {
    const int j = f.t + f.T * b;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int i = j + r * stride;
      v[b * R + r] = active ? (FIRST ? load(i) : buf[phys(i)]) : czero();
    }
  }
  f.sync();
  if (active) {
    const int twstep = TW_N / (ns * R);
#pragma unroll
    for (int b = 0; b < B; ++b) {
      const int j = f.t + f.T * b;
      const int k = j & (ns - 1);
      if (ns > 1) apply_twiddles<SIGN, R>(v + b * R, k * twstep, tw);
      dftR<SIGN, R>(v + b * R);
      const int o = (j - k) * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int i = o + r * ns;
        if (LAST)
          store(i, v[b * R + r]);
        else
          buf[phys(i)] = v[b * R + r];
      }
    }
  }
  if (!LAST) f.sync();
}

// Full transform of one row.  Requires n >= 16 and all T threads of the
// group to call it with the same arguments (inactive groups pass
// active = false and only meet the barriers).
template <int SIGN, class Load, class Store>
GL_D void fft_row(cplx* buf, const FftGroup& f, bool active, const cplx* __restrict__ tw, Load& load,
                  Store& store) {
  const int full = f.log2n >> 2;  // radix-16 passes
  const int rem = f.log2n & 3;    // last radix 2^rem (0: none)
  const int passes = full + (rem ? 1 : 0);
  int ns = 1;
  for (int p = 0; p < passes; ++p) {
    const bool first = p == 0, last = p == passes - 1;
    const int R = (p < full) ? 16 : (1 << rem);
    if (R == 16) {
      if (first && last) fft_pass<SIGN, 16, true, true>(buf, f, ns, active, tw, load, store);
      else if (first) fft_pass<SIGN, 16, true, false>(buf, f, ns, active, tw, load, store);
      else if (last) fft_pass<SIGN, 16, false, true>(buf, f, ns, active, tw, load, store);
      else fft_pass<SIGN, 16, false, false>(buf, f, ns, active, tw, load, store);
    } else if (R == 8) {
      fft_pass<SIGN, 8, false, true>(buf, f, ns, active, tw, load, store);
    } else if (R == 4) {
      fft_pass<SIGN, 4, false, true>(buf, f, ns, active, tw, load, store);
    } else {
      fft_pass<SIGN, 2, false, true>(buf, f, ns, active, tw, load, store);
    }
    ns *= R;
  }
}

}  // namespace gl
