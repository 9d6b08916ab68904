// Per-unit support analysis on the device: parent support, Minkowski-sum
// (pair / triple / radial-channel) supports, the reductions behind the GL
// scales and balance shifts, and the per-node scalar tables.
//
// Reference semantics restated here:
//   support        |s| > 1e-13 max(1, max|s|)          spatial.py:163-164
//   pair/triple    ifft2(fft2(1_S)^n) > 0.5            _order3.py:38-40
//                  (computed exactly as a Minkowski sum of bitsets)
//   peak           first argmax of |s|^2 over S        spatial.py:176-178
//   shifts, scales                                     _order3.py:42-52,
//                                                      spatial.py:179-189,
//                                                      spatial.py:260-268
//   radial channels                                    spatial.py:322-346
#pragma once
#include "gl_common.cuh"

namespace gl {

// Reduction slots per unit (bit patterns of non-negative doubles).
struct UnitSlots {
  unsigned long long smax;       // max |s| over the box
  unsigned long long nu_min;     // min nu over S
  unsigned long long nu_max;     // max nu over S
  unsigned long long amp2_max;   // max |s|^2 over S
  unsigned long long peak_flat;  // min reference flat index among argmax bins
  unsigned long long sqa_max2;   // max sqrt(A) over the pair support
  unsigned long long sqa_max3;   // max sqrt(A) over the triple support
  unsigned long long chan_min[2];
  unsigned long long chan_max[2];
  unsigned long long count;      // support size
  unsigned long long nonfinite;  // set when a non-finite value is met
  unsigned long long pad[3];   // [0] min q over S, [1] max |s| outside the box, [2] max sqrt(A) over the quartic support
  unsigned long long dup;      // 1: the unit's support equals unit 0's (its Minkowski sums are copied)
};

constexpr int MAX_RANK = 16;

// Scalars derived per unit (written by unit_scalars_kernel).
struct UnitScalars {
  double peak_q;
  double nu_min, nu_max;
  double shift2, shift3;    // inner (== eta22) and outer balance shifts
  double lam22;             // eta22 determinant-root scale
  double lam2, lam3;        // order-3 inner/outer scales
  double lam_minus, lam_plus;
  double edge_mid;          // psi22 middle radial edge
  double chan_shift[2];     // psi22 channel shifts (compacted)
  int chan_id[2];           // physical channel index of each compacted channel
  int chan_count;
  int status;               // 0 ok, else GL_ERR_* code
  double lam4, shift4;      // order-4 (eta44) outer scale and balance shift
};

constexpr unsigned long long BITS_POS_INF = 0x7ff0000000000000ull;

struct BitRows {
  unsigned long long* fwd;  // [rows][words]
  unsigned long long* rev;  // reversed rows
  int rows, bits, words;
};

GL_D unsigned long long window64(const unsigned long long* row, int words, int nbits, int p) {
  if (p <= -64 || p >= nbits) return 0ull;
  const int wi = p >> 6;  // floor division
  const int sh = p & 63;
  const unsigned long long lo = (wi >= 0 && wi < words) ? row[wi] : 0ull;
  if (sh == 0) return lo;
  const unsigned long long hi = (wi + 1 >= 0 && wi + 1 < words) ? row[wi + 1] : 0ull;
  return (lo >> sh) | (hi << (64 - sh));
}

// First and last set bit of a row of `words` words (32767, -32768 when empty).
GL_D void row_extent(const unsigned long long* row, int words, int& first, int& last) {
  first = 32767;
  last = -32768;
  for (int w = 0; w < words; ++w) {
    const unsigned long long v = row[w];
    if (v == 0ull) continue;
    if (first == 32767) first = 64 * w + __ffsll((long long)v) - 1;
    last = 64 * w + 63 - __clzll((long long)v);
  }
}

// out(oy, ox) = exists py,bx: A[py][bx] and B[oy-py][ox-bx]; A, B are
// bitset rows with box origins a, b; the output box has origin a+b.
// aext/bext: [row][2] first and last set column of each row of A and B (an
// empty row holds (32767, -32768)); a row pair whose column ranges cannot
// reach ox is skipped before its words are compared.
GL_D bool minkowski_bin(const unsigned long long* A, int ha, int wa, int wwa,
                        const unsigned long long* Brev, int hb, int wb, int wwb,
                        int ox, int oy, const short* aext, const short* bext) {
  int py_lo = oy - (hb - 1);
  if (py_lo < 0) py_lo = 0;
  int py_hi = oy < ha - 1 ? oy : ha - 1;
  const int c = wb - 1 - ox;
  for (int py = py_lo; py <= py_hi; ++py) {
    const int q = oy - py;
    if (ox < (int)aext[2 * py] + (int)bext[2 * q] || ox > (int)aext[2 * py + 1] + (int)bext[2 * q + 1])
      continue;
    const unsigned long long* arow = A + (size_t)py * wwa;
    const unsigned long long* brow = Brev + (size_t)(oy - py) * wwb;
    for (int i = 0; i < wwa; ++i) {
      const unsigned long long aw = arow[i];
      if (aw == 0ull) continue;
      if (aw & window64(brow, wwb, wb, c + 64 * i)) return true;
    }
  }
  return false;
}

}  // namespace gl
