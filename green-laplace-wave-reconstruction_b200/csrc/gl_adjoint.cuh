// Device kernels of the adjoint (reverse-mode) pass of the GL graph.
//
// With the supports, balance shifts, scales, peak and roundoff-floor
// decisions held at their forward values, every GL output spectrum is a
// polynomial in the parent spectrum s with no conjugates (eta22: quadratic,
// eta33: cubic).  For a real loss L(eta) of the physical field
// eta = h Re(ifft2(E)) the gradient is therefore one transposed pass:
//
//   dL = Re( sum_k g_k ds_k ),   g = J(s)^T Ebar,   Ebar_k = h/(Nx Ny) sum_n r_n e^{+i k.x_n}
//
// with r = dL/deta.  The transpose of each forward building block is:
//   multiplier m_b(k)          -> the same multiplier at the same bin;
//   inverse transform G        -> a + sign transform with the same scale;
//   forward transform F        -> a - sign transform with the same scale;
//   product P(f_1..f_m)        -> sum_P (dP/df_b) w_P, pointwise;
//   mask / floor (fixed)       -> the same bins kept.
// So the adjoint stages reuse the forward column/row kernels, with the
// transform sign flipped through conj(F(conj x)) on adjoint data, the
// transposed products of row_products_adj, and the kernels below: the
// residual seed, the per-node adjoint spectra, the multiplier-combining
// column transform and the deterministic reduction into g.
#pragma once
#include "gl_kernels.cuh"

namespace gl {

// ---------------------------------------------------------------------------
// seed: Ebar on an output box from the real residual field
// ---------------------------------------------------------------------------

struct SeedArgs {
  const double* r;   // [unit][ny][nx] dL/deta
  int nx, log2nx, ny;
  int x0, w;         // kept columns (modes)
  cplx* out;         // [unit][ny][w]
};

// + sign transform along x of each residual row; only the box columns are
// kept.  The column pass is col_fft_kernel with conj_io = 1.
#ifdef GL_TRANSFORM_TU  // launched by gl_launch_cols.cu
__global__ void __launch_bounds__(256, 2) seed_row_kernel(SeedArgs a, const cplx* __restrict__ tw) {
  extern __shared__ cplx smem[];
  const int n = a.nx;
  const int L = padded_len(n);
  int g, G;
  const FftGroup f = fft_group(n, a.log2nx, g, G);
  const int y = blockIdx.x * G + g;
  const int unit = blockIdx.y;
  const bool active = y < a.ny;
  const int yy = active ? y : 0;
  cplx* buf = smem + (size_t)g * L;
  const double* row = a.r + ((size_t)unit * a.ny + yy) * n;
  cplx* orow = a.out + ((size_t)unit * a.ny + yy) * a.w;
  auto load = [&](int xb) -> cplx { return cmk(row[xb], 0.0); };
  auto store = [&](int xb, cplx v) {
    const int xo = wrap(xb - a.x0, n);
    if (xo < a.w) orow[xo] = v;
  };
  fft_row<+1>(buf, f, active, tw, load, store);
}
#endif  // GL_TRANSFORM_TU

// ---------------------------------------------------------------------------
// column + transform of adjoint bank fields, multipliers, damping, combine
// ---------------------------------------------------------------------------

enum CmbKind : int {
  CMB_ETA22 = 0,  // eta22 banks of node n: damping e^{-tau_n (nu - shift2)}
  CMB_FIRST3,     // order-3 first-order banks of outer node j: e^{-tau3 (nu - shift3)}
  CMB_INNER,      // order-3 inner banks of (j, i): both dampings
  CMB_PAIR,       // order-3 pair banks: no damping, pair-support mask
};

struct CmbArgs {
  int kind;
  int nbanks;
  int mult[MAX_BANKS];     // forward multiplier of each bank
  int dst_of[MAX_BANKS];   // output spectrum each bank adds into
  int nout;
  Box box;
  const double* geo;
  const cplx* in;          // [job][bank][n][box.w] (row-transformed adjoint fields)
  cplx* out;               // [job][nout][box.h][box.w]
  int n, log2n;            // compact grid along y
  double scale;            // the forward inverse transform's 1/(Nx Ny)
  const UnitScalars* us;
  const double* nodes;     // eta22 nodes (ETA22) or outer nodes (FIRST3, INNER)
  const double* nodes2;    // inner nodes (INNER)
  int n_inner;
  int jobs_per_unit;
  const unsigned char* mask;  // [unit][h][w] (PAIR) or null
};

GL_D double cmb_damping(const CmbArgs& a, int job, double nu) {
  const int unit = job / a.jobs_per_unit;
  const int sub = job % a.jobs_per_unit;
  const UnitScalars& u = a.us[unit];
  switch (a.kind) {
    case CMB_ETA22: return exp(-(a.nodes[sub] / u.lam22) * (nu - u.shift2));
    case CMB_FIRST3: return exp(-(a.nodes[sub] / u.lam3) * (nu - u.shift3));
    case CMB_INNER: {
      const double e3 = exp(-(a.nodes[sub / a.n_inner] / u.lam3) * (nu - u.shift3));
      const double e2 = exp(-(a.nodes2[sub % a.n_inner] / u.lam2) * (nu - u.shift2));
      return e3 * e2;
    }
  }
  return 1.0;
}

// One block: `cw` box columns of one job, all banks at once.  The cw x nbanks
// columns are staged (one shared row each), transformed along y with the +
// sign by groups of n/16 threads in parallel, and each box bin then sums its
// banks' multiplied values in bank order (deterministic) into the bank's
// output spectrum, with the job's damping, the scale and the mask applied.
// MIX = m > 0: columns of the mixed length 16 m.
template <int MIX>
__global__ void __launch_bounds__(256, 2) col_combine_kernel(CmbArgs a, const cplx* __restrict__ tw,
                                                            int cw) {
  extern __shared__ cplx smem[];
  const int job = blockIdx.y;
  const int unit = job / a.jobs_per_unit;
  const int x_first = blockIdx.x * cw;
  const int ncol = min(cw, a.box.w - x_first);
  const int nb = a.nbanks;
  const int n = a.n;
  const int L = padded_len(n);
  const int h = a.box.h;
  const int plane = a.box.w * h;
  // stage: shared row (k * cw + c) holds bank k, column c
  const cplx* src = a.in + (size_t)job * nb * n * a.box.w + x_first;
  for (int t = threadIdx.x; t < nb * n * ncol; t += blockDim.x) {
    const int k = t / (n * ncol), r = t % (n * ncol);
    const int y = r / ncol, c = r % ncol;
    smem[(size_t)(k * cw + c) * L + phys(y)] = src[((size_t)k * n + y) * a.box.w + c];
  }
  __syncthreads();
  int g, G;
  const FftGroup f = fft_group(n, a.log2n, g, G);
  const int nrow = nb * ncol;
  for (int it = 0; it < (nrow + G - 1) / G; ++it) {
    const int r = it * G + g;
    const bool active = r < nrow;
    const int rr = active ? r : 0;
    cplx* buf = smem + (size_t)((rr / ncol) * cw + rr % ncol) * L;
    auto load = [&](int yb) -> cplx { return buf[phys(yb)]; };
    auto store = [&](int yb, cplx v) { buf[phys(yb)] = v; };
    fft_row<+1, MIX>(buf, f, active, tw, load, store);
  }
  __syncthreads();
  const unsigned char* mask = a.mask ? a.mask + (size_t)unit * plane : nullptr;
  cplx* dst = a.out + (size_t)job * a.nout * plane;
  for (int t = threadIdx.x; t < ncol * h; t += blockDim.x) {
    const int c = t % ncol, by = t / ncol;
    const int i = by * a.box.w + x_first + c;
    const int yb = phys(wrap_any(a.box.y0 + by, n));
    const GeoRef geo{a.geo, plane, i};
    cplx acc0 = czero(), acc1 = czero(), acc2 = czero(), acc3 = czero();
    for (int k = 0; k < nb; ++k) {
      const cplx v = apply_mult(a.mult[k], geo, smem[(size_t)(k * cw + c) * L + yb]);
      switch (a.dst_of[k]) {
        case 0: acc0 = cadd(acc0, v); break;
        case 1: acc1 = cadd(acc1, v); break;
        case 2: acc2 = cadd(acc2, v); break;
        default: acc3 = cadd(acc3, v); break;
      }
    }
    const bool keep = !mask || mask[i];
    const double fac = keep ? a.scale * cmb_damping(a, job, geo.nu()) : 0.0;
    const cplx accs[4] = {acc0, acc1, acc2, acc3};
#pragma unroll
    for (int o = 0; o < 4; ++o)
      if (o < a.nout) dst[(size_t)o * plane + i] = keep ? cscale(fac, accs[o]) : czero();
  }
}

// ---------------------------------------------------------------------------
// adjoint spectra of the accumulated node products (elementwise)
// ---------------------------------------------------------------------------

#ifndef GL_TRANSFORM_TU  // elementwise kernels: compiled by gl_engine.cu only
// A bin's forward value survived the stage's mask and roundoff floor
// (the forward's floored(): |v| < rel * max zeroes it).
GL_D bool kept(cplx v, double rel, unsigned long long peak_bits, unsigned char in_mask) {
  return in_mask && !abs_below(v, rel * as_double(peak_bits));
}

struct AdjArgs {
  const UnitScalars* us;
  const double* geo;        // geometry planes of the box
  Box box;
  const cplx* seed;         // adjoint of the accumulated spectra
  const cplx* fwd;          // forward node spectra (for the floors)
  const unsigned long long* fwdmax;
  const unsigned char* mask;   // [unit][h][w]
  cplx* out;                // adjoint node spectra
  const double* nodes;
  const double* weights;
  int jobs_per_unit;
  int n_inner;
  double floor_rel;
};

// eta22 node n: acc += coef (-A sh sd + ch sk)  (spatial.py:206-221)
__global__ void adj_eta22_kernel(AdjArgs a) {
  const int job = blockIdx.y;
  const int unit = job / a.jobs_per_unit, nn = job % a.jobs_per_unit;
  const int plane = a.box.w * a.box.h;
  const UnitScalars& u = a.us[unit];
  const double x = a.nodes[nn], w = a.weights[nn];
  const double tau = x / u.lam22;
  const double coef = w * exp(x) / u.lam22 / 4.0 * exp(-2.0 * u.shift2 * tau);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < plane; i += gridDim.x * blockDim.x) {
    const GeoRef G{a.geo, plane, i};
    const double sqa = __ldg(a.geo + 5 * plane + i);
    const double sh = sinh_over_root(sqa, tau), ch = cosh(sqa * tau);
    const cplx e = a.seed[(size_t)unit * plane + i];
    const unsigned char m = a.mask[(size_t)unit * plane + i];
    const cplx* f = a.fwd + (size_t)job * 2 * plane;
    cplx* o = a.out + (size_t)job * 2 * plane;
    o[i] = kept(f[i], a.floor_rel, a.fwdmax[job * 2 + 0], m) ? cscale(coef * (-G.a() * sh), e) : czero();
    o[plane + i] = kept(f[plane + i], a.floor_rel, a.fwdmax[job * 2 + 1], m) ? cscale(coef * ch, e) : czero();
  }
}

// order-3 outer node j: eta += coef (A sh fd - i ch fk)  (_order3.py:124-138)
// adjoint spectra [uj][2] = (fk, fd), the order of the forward forcing rows.
__global__ void adj_outer_kernel(AdjArgs a) {
  const int uj = blockIdx.y;
  const int unit = uj / a.jobs_per_unit, j = uj % a.jobs_per_unit;
  const int plane = a.box.w * a.box.h;
  const UnitScalars& u = a.us[unit];
  const double x = a.nodes[j], w = a.weights[j];
  const double tau = x / u.lam3;
  const double coef = w * exp(x) / u.lam3 * exp(-3.0 * u.shift3 * tau);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < plane; i += gridDim.x * blockDim.x) {
    const GeoRef G{a.geo, plane, i};
    const double sqa = __ldg(a.geo + 5 * plane + i);
    const double sh = sinh_over_root(sqa, tau), ch = cosh(sqa * tau);
    const cplx e = a.seed[(size_t)unit * plane + i];
    const unsigned char m = a.mask[(size_t)unit * plane + i];
    const cplx* f = a.fwd + (size_t)uj * 2 * plane;
    cplx* o = a.out + (size_t)uj * 2 * plane;
    o[i] = kept(f[i], a.floor_rel, a.fwdmax[uj * 2 + 0], m) ? cmul(cmk(0.0, -coef * ch), e) : czero();
    o[plane + i] = kept(f[plane + i], a.floor_rel, a.fwdmax[uj * 2 + 1], m) ? cscale(coef * G.a() * sh, e)
                                                                            : czero();
  }
}

// order-3 inner node i of outer node j (_order3.py:240-259):
//   e  += c (-A sh sd + ch sk),   p  += i c (ch sd - sh sk),
//   pt += c (ch sdt - sh skt)     (eta_t feeds only psi33's contact)
// seed: the pair-spectra adjoints [uj][4] = (e, eta_t, p, pt).
__global__ void adj_inner_kernel(AdjArgs a) {
  const int job = blockIdx.y;
  const int uj = job / a.n_inner, ii = job % a.n_inner;
  const int unit = job / a.jobs_per_unit;
  const int plane = a.box.w * a.box.h;
  const UnitScalars& u = a.us[unit];
  const double x = a.nodes[ii], w = a.weights[ii];
  const double tau = x / u.lam2;
  const double coef = w * exp(x) / u.lam2 * exp(-2.0 * u.shift2 * tau) / 4.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < plane; i += gridDim.x * blockDim.x) {
    const GeoRef G{a.geo, plane, i};
    const double sqa = __ldg(a.geo + 5 * plane + i);
    const double sh = sinh_over_root(sqa, tau), ch = cosh(sqa * tau);
    const cplx* sd = a.seed + (size_t)uj * 4 * plane;
    const cplx ee = sd[i], ep = sd[2 * plane + i], ept = sd[3 * plane + i];
    const unsigned char m = a.mask[(size_t)unit * plane + i];
    const cplx* f = a.fwd + (size_t)job * 4 * plane;
    const unsigned long long* mx = a.fwdmax + (size_t)job * 4;
    cplx* o = a.out + (size_t)job * 4 * plane;
    const cplx v0 = cadd(cscale(-G.a() * sh, ee), cmul(cmk(0.0, ch), ep));
    const cplx v1 = csub(cscale(ch, ee), cmul(cmk(0.0, sh), ep));
    o[i] = kept(f[i], a.floor_rel, mx[0], m) ? cscale(coef, v0) : czero();
    o[plane + i] = kept(f[plane + i], a.floor_rel, mx[1], m) ? cscale(coef, v1) : czero();
    o[2 * plane + i] = kept(f[2 * plane + i], a.floor_rel, mx[2], m) ? cscale(coef * ch, ept) : czero();
    o[3 * plane + i] = kept(f[3 * plane + i], a.floor_rel, mx[3], m) ? cscale(-coef * sh, ept) : czero();
  }
}

// ---------------------------------------------------------------------------
// gradient reduction and the mode deposit's transpose
// ---------------------------------------------------------------------------

struct RedArgs {
  const cplx* e1;     // eta11 seed [unit][plane] or null
  const cplx* da22;   // eta22 node partials [unit][n22][plane]
  int n22;
  const cplx* da1;    // order-3 first-order partials [unit][n1][plane]
  int n1;
  const cplx* dai;    // order-3 inner partials [unit][ni][plane]
  int ni;
  cplx* grad;         // [unit][plane]
  int plane;
};

// g = e1 + sum of every node's partial, in a fixed order.
__global__ void adj_reduce_kernel(RedArgs a) {
  const int unit = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.plane; i += gridDim.x * blockDim.x) {
    cplx g = a.e1 ? a.e1[(size_t)unit * a.plane + i] : czero();
    for (int k = 0; k < a.n22; ++k) g = cadd(g, a.da22[((size_t)unit * a.n22 + k) * a.plane + i]);
    for (int k = 0; k < a.n1; ++k) g = cadd(g, a.da1[((size_t)unit * a.n1 + k) * a.plane + i]);
    for (int k = 0; k < a.ni; ++k) g = cadd(g, a.dai[((size_t)unit * a.ni + k) * a.plane + i]);
    a.grad[(size_t)unit * a.plane + i] = g;
  }
}

// Transpose of deposit_kernel: with s_bin += (Nx Ny / h)(a + i b) e^{-i w t}
// and dL = Re(sum g ds), dL/da = Re(g c) and dL/db = -Im(g c) for
// c = (Nx Ny / h) e^{-i w t}, summed over the units (snapshots) that share
// the modes.  Output [mode][2] in the deposit's (segment) order.
__global__ void deposit_adjoint_kernel(int n_units, int n_seg, const int* seg_off, const int* seg_bin,
                                       const double* omega, const double* times, double scale,
                                       double depth, const cplx* grad, int plane, double* gab) {
  for (int sgi = blockIdx.x * blockDim.x + threadIdx.x; sgi < n_seg; sgi += gridDim.x * blockDim.x) {
    const int bin = seg_bin[sgi];
    for (int k = seg_off[sgi]; k < seg_off[sgi + 1]; ++k) {
      double ga = 0.0, gb = 0.0;
      for (int u = 0; u < n_units; ++u) {
        double s, c;
        sincos(omega[k] * times[u], &s, &c);
        const cplx z = cmul(grad[(size_t)u * plane + bin], cmk(scale / depth * c, -scale / depth * s));
        ga += z.x;
        gb -= z.y;
      }
      gab[2 * k] = ga;
      gab[2 * k + 1] = gb;
    }
  }
}
#endif  // GL_TRANSFORM_TU

}  // namespace gl
