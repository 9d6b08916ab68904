// Register-resident FFTs for power-of-two lengths 16..4096 and for the
// mixed lengths 16 m, m in {3, 5, 6, 9, 10, 12, 15} (48 .. 240).
//
// A power-of-two length-n transform is run by a group of T = n/16 threads
// that each hold 16 complex values per pass.  Passes are Stockham autosort
// steps of radix 16 (the last one radix 2, 4 or 8 when log2 n is not a
// multiple of 4), so a 256-point transform is two passes and a 1024-point one
// three, with one shared-memory round trip between passes instead of one per
// radix-4 stage.  A mixed length 16 m is run by T = 16 threads in two passes:
// radix m (one butterfly per thread, no twiddles), then radix 16 over the m
// butterflies (threads t < m) with twiddles from a length-n table.  The first
// pass reads its inputs through a caller functor (global memory, on-the-fly
// multipliers, zero outside a spectral box) and the last pass hands its
// outputs to a caller functor (kept columns only, physical scaling), so
// intermediate rows never exist in global memory.
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

// ---------------------------------------------------------------------------
// small odd-factor DFTs and the two-factor DFTs of the mixed lengths
// ---------------------------------------------------------------------------

constexpr double FR3 = 0.86602540378443864676;  // sin(2 pi/3) = sqrt(3)/2

// y_t = sum_s x_s e^{SIGN 2 pi i s t/3}
template <int SIGN>
GL_D void dft3(cplx* v) {
  const cplx a = v[0], s = cadd(v[1], v[2]), d = csub(v[1], v[2]);
  const cplx m = cmk(a.x - 0.5 * s.x, a.y - 0.5 * s.y);
  const cplx r = cscale(FR3, d);
  const cplx rot = SIGN < 0 ? cmulmi(r) : cmuli(r);
  v[0] = cadd(a, s);
  v[1] = cadd(m, rot);
  v[2] = csub(m, rot);
}

// cos(2 pi k/5), sin(2 pi k/5) for k = 1, 2
constexpr double FC51 = 0.30901699437494742410, FS51 = 0.95105651629515357212;
constexpr double FC52 = -0.80901699437494742410, FS52 = 0.58778525229247312917;

// y_t = sum_s x_s e^{SIGN 2 pi i s t/5}: with s1 = x1 + x4, d1 = x1 - x4,
// s2 = x2 + x3, d2 = x2 - x3 the forward outputs are y1,4 = t1 -/+ i u1 and
// y2,3 = t2 -/+ i u2 (t1 = x0 + c1 s1 + c2 s2, u1 = s1' d1 + s2' d2,
// t2 = x0 + c2 s1 + c1 s2, u2 = s2' d1 - s1' d2); the inverse flips i.
template <int SIGN>
GL_D void dft5(cplx* v) {
  const cplx a = v[0];
  const cplx s1 = cadd(v[1], v[4]), d1 = csub(v[1], v[4]);
  const cplx s2 = cadd(v[2], v[3]), d2 = csub(v[2], v[3]);
  const cplx t1 = cadd(a, cadd(cscale(FC51, s1), cscale(FC52, s2)));
  const cplx t2 = cadd(a, cadd(cscale(FC52, s1), cscale(FC51, s2)));
  const cplx u1 = cadd(cscale(FS51, d1), cscale(FS52, d2));
  const cplx u2 = csub(cscale(FS52, d1), cscale(FS51, d2));
  const cplx r1 = SIGN < 0 ? cmulmi(u1) : cmuli(u1);
  const cplx r2 = SIGN < 0 ? cmulmi(u2) : cmuli(u2);
  v[0] = cadd(a, cadd(s1, s2));
  v[1] = cadd(t1, r1);
  v[4] = csub(t1, r1);
  v[2] = cadd(t2, r2);
  v[3] = csub(t2, r2);
}

template <int SIGN, int R>
GL_D void dft_small(cplx* v) {
  if (R == 2) dft2<SIGN>(v);
  if (R == 3) dft3<SIGN>(v);
  if (R == 4) dft4v<SIGN>(v);
  if (R == 5) dft5<SIGN>(v);
}

// cos and sin of 2 pi e/N for the inner twiddles of the two-factor DFTs
// (N = 6, 9, 10, 12, 15; e = b k_a < N).
GL_HD double tw_cos(int N, int e) {
  switch (N * 16 + e) {
    case 6 * 16 + 1: return 0.5;
    case 6 * 16 + 2: return -0.5;
    case 9 * 16 + 1: return 0.76604444311897803520;
    case 9 * 16 + 2: return 0.17364817766693034885;
    case 9 * 16 + 4: return -0.93969262078590838405;
    case 10 * 16 + 1: return 0.80901699437494742410;
    case 10 * 16 + 2: return 0.30901699437494742410;
    case 10 * 16 + 3: return -0.30901699437494742410;
    case 10 * 16 + 4: return -0.80901699437494742410;
    case 12 * 16 + 1: return 0.86602540378443864676;
    case 12 * 16 + 2: return 0.5;
    case 12 * 16 + 3: return 0.0;
    case 12 * 16 + 4: return -0.5;
    case 12 * 16 + 6: return -1.0;
    case 15 * 16 + 1: return 0.91354545764260089550;
    case 15 * 16 + 2: return 0.66913060635885821383;
    case 15 * 16 + 3: return 0.30901699437494742410;
    case 15 * 16 + 4: return -0.10452846326765347140;
    case 15 * 16 + 6: return -0.80901699437494742410;
    case 15 * 16 + 8: return -0.97814760073380563793;
  }
  return 1.0;
}
GL_HD double tw_sin(int N, int e) {
  switch (N * 16 + e) {
    case 6 * 16 + 1: return 0.86602540378443864676;
    case 6 * 16 + 2: return 0.86602540378443864676;
    case 9 * 16 + 1: return 0.64278760968653932632;
    case 9 * 16 + 2: return 0.98480775301220805937;
    case 9 * 16 + 4: return 0.34202014332566873304;
    case 10 * 16 + 1: return 0.58778525229247312917;
    case 10 * 16 + 2: return 0.95105651629515357212;
    case 10 * 16 + 3: return 0.95105651629515357212;
    case 10 * 16 + 4: return 0.58778525229247312917;
    case 12 * 16 + 1: return 0.5;
    case 12 * 16 + 2: return 0.86602540378443864676;
    case 12 * 16 + 3: return 1.0;
    case 12 * 16 + 4: return 0.86602540378443864676;
    case 12 * 16 + 6: return 0.0;
    case 15 * 16 + 1: return 0.40673664307580020775;
    case 15 * 16 + 2: return 0.74314482547739423501;
    case 15 * 16 + 3: return 0.95105651629515357212;
    case 15 * 16 + 4: return 0.99452189536827333692;
    case 15 * 16 + 6: return 0.58778525229247312917;
    case 15 * 16 + 8: return -0.20791169081775933710;
  }
  return 0.0;
}

// N = A B point DFT in place: x index n = B a + b, output X[k_a + A k_b] =
// DFT_B over b of (W_N^(b k_a) DFT_A over a of x[B a + b]).
template <int SIGN, int A, int B>
GL_D void dft_ab(cplx* v) {
  constexpr int N = A * B;
  cplx y[N];
#pragma unroll
  for (int b = 0; b < B; ++b) {
    cplx t[A];
#pragma unroll
    for (int a = 0; a < A; ++a) t[a] = v[B * a + b];
    dft_small<SIGN, A>(t);
#pragma unroll
    for (int ka = 0; ka < A; ++ka)
      y[b * A + ka] = (b * ka == 0) ? t[ka]
                                    : cmul(t[ka], wconst<SIGN>(tw_cos(N, b * ka), -tw_sin(N, b * ka)));
  }
#pragma unroll
  for (int ka = 0; ka < A; ++ka) {
    cplx t[B];
#pragma unroll
    for (int b = 0; b < B; ++b) t[b] = y[b * A + ka];
    dft_small<SIGN, B>(t);
#pragma unroll
    for (int kb = 0; kb < B; ++kb) v[ka + A * kb] = t[kb];
  }
}

// The radix-m DFT of the first pass of a mixed length 16 m.
template <int SIGN, int M>
GL_D void dft_mixed(cplx* v) {
  if (M == 3) dft3<SIGN>(v);
  if (M == 5) dft5<SIGN>(v);
  if (M == 6) dft_ab<SIGN, 2, 3>(v);
  if (M == 9) dft_ab<SIGN, 3, 3>(v);
  if (M == 10) dft_ab<SIGN, 5, 2>(v);
  if (M == 12) dft_ab<SIGN, 4, 3>(v);
  if (M == 15) dft_ab<SIGN, 3, 5>(v);
}

// Mixed lengths and their twiddle tables W_n^e, e < n, stored after the
// power-of-two table: [TW_N][48][80][96][144][160][192][240].
GL_HD bool mixed_len(int n) {
  return n == 48 || n == 80 || n == 96 || n == 144 || n == 160 || n == 192 || n == 240;
}
GL_HD int mixed_tw_offset(int n) {
  switch (n) {
    case 48: return 0;
    case 80: return 48;
    case 96: return 128;
    case 144: return 224;
    case 160: return 368;
    case 192: return 528;
    case 240: return 720;
  }
  return 0;
}
constexpr int MIXED_TW_TOTAL = 960;
constexpr int TW_ALLOC = TW_N + MIXED_TW_TOTAL;  // entries of a twiddle buffer

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
  int n, log2n;  // transform length (log2n unused for mixed lengths)
  int m;         // mixed length n = 16 m, else 0
  int T;         // threads in the group (n / 16, 16 for mixed lengths)
  int t;         // thread index inside the group
  GroupSync sync;
};

// Group geometry of thread tl of a team of `team` threads (a block, or one
// row's share of a block that carries several rows) doing length-n
// transforms; named barriers of the team's groups start at id_base.
GL_D FftGroup fft_group_team(int n, int log2n, int tl, int team, int id_base, int& g, int& G) {
  FftGroup f;
  f.n = n;
  f.log2n = log2n;
  f.m = mixed_len(n) ? n >> 4 : 0;
  f.T = f.m ? 16 : n >> 4;
  G = team / f.T;
  g = tl / f.T;
  f.t = tl % f.T;
  f.sync = GroupSync{f.T, id_base + g};
  return f;
}

// Group geometry for a block of `threads` threads doing length-n transforms.
GL_D FftGroup fft_group(int n, int log2n, int& g, int& G) {
  FftGroup f;
  f.n = n;
  f.log2n = log2n;
  f.m = mixed_len(n) ? n >> 4 : 0;
  f.T = f.m ? 16 : n >> 4;
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

// Second pass of a mixed length n = 16 m: radix 16 over the m butterflies
// j = t < m, inputs buf[t + m r], twiddles W_n^(r t) from the length-n table.
template <int SIGN, class Store>
GL_D void fft_mixed_last(cplx* buf, const FftGroup& f, bool active, const cplx* __restrict__ twn,
                         Store& store) {
  const int M = f.m, t = f.t;
  const bool act = active && t < M;
  cplx v[16];
  if (act) {
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = buf[phys(t + M * r)];
  }
  f.sync();
  if (act) {
    if (t > 0) apply_twiddles<SIGN, 16>(v, t, twn);
    dft16<SIGN>(v);
#pragma unroll
    for (int r = 0; r < 16; ++r) store(t + M * r, v[r]);
  }
}

// Whole transform of a mixed length n = 16 m: pass 1 radix m over inputs
// load(t + 16 r) (butterfly j = t), outputs at t m + r; then the radix-16 pass.
template <int SIGN, int M, class Load, class Store>
GL_D void fft_row_mixed(cplx* buf, const FftGroup& f, bool active, const cplx* __restrict__ tw, Load& load,
                        Store& store) {
  const int t = f.t;
  cplx v[M];
#pragma unroll
  for (int r = 0; r < M; ++r) v[r] = active ? load(t + 16 * r) : czero();
  f.sync();
  if (active) {
    dft_mixed<SIGN, M>(v);
#pragma unroll
    for (int r = 0; r < M; ++r) buf[phys(t * M + r)] = v[r];
  }
  f.sync();
  fft_mixed_last<SIGN>(buf, f, active, tw + TW_N + mixed_tw_offset(f.n), store);
}

// Full transform of one row.  Requires n >= 16 and all T threads of the
// group to call it with the same arguments (inactive groups pass
// active = false and only meet the barriers).  MIX = 0: power-of-two
// lengths; MIX = m: the mixed length n = 16 m (the twiddle buffer then holds
// TW_ALLOC entries).  Kernels are instantiated per MIX: one kernel carrying
// every radix behind a runtime switch spills heavily.
template <int SIGN, int MIX = 0, class Load, class Store>
GL_D void fft_row(cplx* buf, const FftGroup& f, bool active, const cplx* __restrict__ tw, Load& load,
                  Store& store) {
  if constexpr (MIX > 0) {
    fft_row_mixed<SIGN, MIX>(buf, f, active, tw, load, store);
    return;
  }
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
