// Batched complex FFTs of power-of-two length on shared-memory data.
//
// Stockham autosort formulation: every stage reads the current buffer with
// stride n/R, applies the stage twiddles W^(r k), does an R-point DFT in
// registers and writes the "expanded" index, so the result lands in natural
// order without a bit-reversal pass.  Radix 4 throughout, plus one radix-2
// stage when log2(n) is odd.  Forward transforms use e^{-2 pi i/n} (numpy's
// fft), inverse ones e^{+2 pi i/n}, both unnormalised.
//
// Twiddles come from a device table tw[m] = exp(-2 pi i m / TW_N) for
// m < TW_N, computed in FP64 by sincospi at library set-up; a length-n
// transform reads it with stride TW_N/n.
#pragma once
#include "gl_common.cuh"

namespace gl {

constexpr int TW_LOG2 = 12;
constexpr int TW_N = 1 << TW_LOG2;  // largest supported transform length

template <int SIGN>
GL_D cplx twiddle(const cplx* __restrict__ tw, int m) {
  cplx w = __ldg(tw + m);
  return SIGN < 0 ? w : cmk(w.x, -w.y);
}

// One radix-4 butterfly on four values: y_t = sum_s x_s e^{SIGN 2 pi i s t/4}.
template <int SIGN>
GL_D void dft4(cplx& a, cplx& b, cplx& c, cplx& d) {
  cplx s0 = cadd(a, c), d0 = csub(a, c);
  cplx s1 = cadd(b, d), d1 = csub(b, d);
  // SIGN<0: W4 = -i ; SIGN>0: W4 = +i
  cplx rot = SIGN < 0 ? cmulmi(d1) : cmuli(d1);
  a = cadd(s0, s1);
  c = csub(s0, s1);
  b = cadd(d0, rot);
  d = csub(d0, rot);
}

// Transform `cnt` contiguous sequences of length n = 2^log2n held in `buf`
// (sequence c at buf + c*n) using `tmp` (same size) as the ping-pong buffer.
// All threads of the block must call it; returns the buffer holding the
// result.  Caller must __syncthreads() before the call.
template <int SIGN>
__device__ cplx* fft_batch(cplx* buf, cplx* tmp, int n, int log2n, int cnt,
                           const cplx* __restrict__ tw) {
  const int tstride = TW_N >> log2n;
  int ns = 1;
  int rem = log2n;
  cplx* src = buf;
  cplx* dst = tmp;
  if (rem & 1) {  // radix-2 stage first (ns = 1: no twiddles)
    const int half = n >> 1;
    const int total = cnt * half;
    for (int b = threadIdx.x; b < total; b += blockDim.x) {
      const int c = b >> (log2n - 1);
      const int j = b & (half - 1);
      cplx* s = src + c * n;
      cplx* d = dst + c * n;
      cplx x0 = s[j], x1 = s[j + half];
      d[2 * j] = cadd(x0, x1);
      d[2 * j + 1] = csub(x0, x1);
    }
    __syncthreads();
    cplx* t = src; src = dst; dst = t;
    ns = 2;
    rem -= 1;
  }
  while (rem > 0) {
    const int quarter = n >> 2;
    const int total = cnt * quarter;
    const int twscale = tstride * (n / (ns * 4));  // table step per unit angle
    for (int b = threadIdx.x; b < total; b += blockDim.x) {
      const int c = b >> (log2n - 2);
      const int j = b & (quarter - 1);
      const int k = j & (ns - 1);
      cplx* s = src + c * n;
      cplx* d = dst + c * n;
      cplx x0 = s[j];
      cplx x1 = s[j + quarter];
      cplx x2 = s[j + 2 * quarter];
      cplx x3 = s[j + 3 * quarter];
      if (ns > 1) {
        const int m = k * twscale;
        x1 = cmul(x1, twiddle<SIGN>(tw, m));
        x2 = cmul(x2, twiddle<SIGN>(tw, 2 * m));
        x3 = cmul(x3, twiddle<SIGN>(tw, 3 * m));
      }
      dft4<SIGN>(x0, x1, x2, x3);
      const int o = (j - k) * 4 + k;
      d[o] = x0;
      d[o + ns] = x1;
      d[o + 2 * ns] = x2;
      d[o + 3 * ns] = x3;
    }
    __syncthreads();
    cplx* t = src; src = dst; dst = t;
    ns *= 4;
    rem -= 2;
  }
  return src;
}

}  // namespace gl
