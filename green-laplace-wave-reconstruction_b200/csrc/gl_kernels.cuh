// Device kernels of the Green--Laplace engine.
//
// Every GL stage of the reference (eta22, psi22, the nested order-3 graph)
// is the same three-step pattern: Fourier multiplier banks -> inverse FFTs ->
// pointwise products -> forward FFTs -> support mask / roundoff floor ->
// per-node weighted accumulation.  The engine runs it on a "compact grid"
// (Ncx x Ncy, the smallest power-of-two grid on which every product of the
// stage is alias-free; Ncx = Nx, Ncy = Ny reproduces the reference's own grid)
// with the spectra held in small boxes around their supports:
//
//   col_ifft_kernel  spectral box columns -> multiplier banks -> inverse FFT
//                    along y (only the box's columns carry data);
//   row_kernel       one physical row: inverse FFT along x of every bank,
//                    the stage's pointwise products, forward FFT along x, and
//                    only the output box's columns are kept;
//   col_fft_kernel   forward FFT along y of the kept columns, output-box rows
//                    kept, support mask applied, per-spectrum max |.| taken;
//   *_acc kernels    roundoff floor + per-node accumulation, elementwise;
//   out_row_kernel   final inverse FFT along x on the reference grid.
#pragma once
#include "gl_analysis.cuh"
#include "gl_async.cuh"
#include "gl_fft.cuh"
#include "gl_fftreg.cuh"

namespace gl {

// ---------------------------------------------------------------------------
// FFT helpers over grouped shared-memory rows
// ---------------------------------------------------------------------------

// In-place transform of `cnt` rows of length n held in `data`, in groups of
// at most `gmax` rows through the ping-pong buffer `tmp` (gmax*n values).
template <int SIGN>
__device__ void fft_rows(cplx* data, cplx* tmp, int n, int log2n, int cnt, int gmax,
                         const cplx* __restrict__ tw) {
  for (int g0 = 0; g0 < cnt; g0 += gmax) {
    const int g = cnt - g0 < gmax ? cnt - g0 : gmax;
    cplx* base = data + (size_t)g0 * n;
    cplx* res = fft_batch<SIGN>(base, tmp, n, log2n, g, tw);
    if (res != base) {
      for (int i = threadIdx.x; i < g * n; i += blockDim.x) base[i] = res[i];
      __syncthreads();
    }
  }
}

// ---------------------------------------------------------------------------
// multiplier banks
// ---------------------------------------------------------------------------

enum Mult : int {
  M_ONE = 0, M_NU, M_NU2, M_NU3, M_QX_SNU, M_QY_SNU, M_Q2_SNU, M_QX, M_QY, M_Q2,
  M_NUQX, M_NUQY, M_IQX, M_IQY, M_MI_NU, M_MI_Q2_SNU, M_MI_Q2NU, M_MINUS_A, M_MINUS_Q2,
  M_A, M_PSI11,
  // order-2 banks divide after the multiply: (s * qx) / safe_nu (spatial.py:199-201)
  M_QX_DIVNU, M_QY_DIVNU, M_Q2_DIVNU,
  // order-4 banks (paper/order4/cpp/gl_eta44_fftw.cpp:188-290, 299-529)
  M_MI_NU2QX, M_MI_NU2QY, M_MINUS_Q2A, M_I_ANU, M_PHI_IQXQ2, M_PHI_IQYQ2, M_PHI_Q4, M_NU4,
  M_Q2NU, M_NU2QX, M_NU2QY, M_IQXA, M_IQYA, M_Q2A
};

struct BinGeo {
  double qx, qy, q, nu, a, sqa;
};

GL_D BinGeo load_geo(const double* geo, int plane, int i) {
  BinGeo g;
  g.qx = geo[i];
  g.qy = geo[plane + i];
  g.q = geo[2 * plane + i];
  g.nu = geo[3 * plane + i];
  g.a = geo[4 * plane + i];
  g.sqa = geo[5 * plane + i];
  return g;
}

// Geometry planes of a box: qx, qy, q, nu, A, sqrt(A) at i, plane, 2 plane, ...
struct GeoRef {
  const double* g;
  int plane, i;
  GL_D double qx() const { return __ldg(g + i); }
  GL_D double qy() const { return __ldg(g + plane + i); }
  GL_D double q() const { return __ldg(g + 2 * plane + i); }
  GL_D double nu() const { return __ldg(g + 3 * plane + i); }
  GL_D double a() const { return __ldg(g + 4 * plane + i); }
};

// value = multiplier(bin) * s, in the evaluation order of the reference's
// NumPy expressions (_order3.py:151-193, spatial.py:196-203); only the
// geometry planes a multiplier needs are read.
GL_D cplx apply_mult(int m, const GeoRef& g, cplx s) {
  switch (m) {
    case M_ONE: return s;
    case M_NU: return cscale(g.nu(), s);
    case M_NU2: { const double nu = g.nu(); return cscale(nu * nu, s); }
    case M_NU3: { const double nu = g.nu(); return cscale(nu * nu * nu, s); }
    case M_QX_SNU: return cscale(g.qx() / safe_nu(g.nu()), s);
    case M_QY_SNU: return cscale(g.qy() / safe_nu(g.nu()), s);
    case M_Q2_SNU: { const double q = g.q(); return cscale((q * q) / safe_nu(g.nu()), s); }
    case M_QX: return cscale(g.qx(), s);
    case M_QY: return cscale(g.qy(), s);
    case M_Q2: { const double q = g.q(); return cscale(q * q, s); }
    case M_NUQX: return cscale(g.nu() * g.qx(), s);
    case M_NUQY: return cscale(g.nu() * g.qy(), s);
    case M_IQX: return cmuli(cscale(g.qx(), s));
    case M_IQY: return cmuli(cscale(g.qy(), s));
    case M_MI_NU: return cmulmi(cscale(g.nu(), s));
    case M_MI_Q2_SNU: { const double q = g.q(); return cmulmi(cscale((q * q) / safe_nu(g.nu()), s)); }
    case M_MI_Q2NU: { const double q = g.q(); return cmulmi(cscale((q * q) * g.nu(), s)); }
    case M_MINUS_A: return cscale(-g.a(), s);
    case M_MINUS_Q2: { const double q = g.q(); return cscale(-(q * q), s); }
    case M_A: return cscale(g.a(), s);
    case M_PSI11: { const double nu = g.nu(); return nu > 0.0 ? cmk(s.y / nu, -s.x / nu) : czero(); }
    case M_QX_DIVNU: { const cplx t = cscale(g.qx(), s); const double sn = safe_nu(g.nu()); return cmk(t.x / sn, t.y / sn); }
    case M_QY_DIVNU: { const cplx t = cscale(g.qy(), s); const double sn = safe_nu(g.nu()); return cmk(t.x / sn, t.y / sn); }
    case M_Q2_DIVNU: { const double q = g.q(); const cplx t = cscale(q * q, s); const double sn = safe_nu(g.nu()); return cmk(t.x / sn, t.y / sn); }
    case M_MI_NU2QX: { const double nu = g.nu(); return cmulmi(cscale(nu * nu * g.qx(), s)); }
    case M_MI_NU2QY: { const double nu = g.nu(); return cmulmi(cscale(nu * nu * g.qy(), s)); }
    case M_MINUS_Q2A: { const double q = g.q(); return cscale(-(q * q * g.a()), s); }
    case M_I_ANU: return cmuli(cscale(g.a() * g.nu(), s));
    case M_PHI_IQXQ2: case M_PHI_IQYQ2: case M_PHI_Q4: {
      // phi = (-i s)/nu where nu > 0, then the vertical-derivative multiplier
      const double nu = g.nu();
      if (!(nu > 0.0)) return czero();
      const cplx phi = cmk(s.y / nu, -s.x / nu);
      const double q = g.q();
      if (m == M_PHI_Q4) return cscale(q * q * q * q, phi);
      return cmuli(cscale((m == M_PHI_IQXQ2 ? g.qx() : g.qy()) * q * q, phi));
    }
    case M_NU4: { const double nu = g.nu(); return cscale(nu * nu * nu * nu, s); }
    case M_Q2NU: { const double q = g.q(); return cscale(q * q * g.nu(), s); }
    case M_NU2QX: { const double nu = g.nu(); return cscale(nu * nu * g.qx(), s); }
    case M_NU2QY: { const double nu = g.nu(); return cscale(nu * nu * g.qy(), s); }
    case M_IQXA: return cmuli(cscale(g.qx() * g.a(), s));
    case M_IQYA: return cmuli(cscale(g.qy() * g.a(), s));
    case M_Q2A: { const double q = g.q(); return cscale(q * q * g.a(), s); }
  }
  return czero();
}

// ---------------------------------------------------------------------------
// column inverse FFT (spectral box -> banks along y)
// ---------------------------------------------------------------------------

enum ColKind : int {
  COL_PLAIN = 0,   // bank k reads spectrum k of the job (no damping)
  COL_ETA22,       // s e^{-tau_n (nu - shift)}
  COL_PSI22,       // (s mask_c) e^{-tau (nu - shift_c)}
  COL_INNER,       // (s e^{-tau3 (nu - shift3)}) e^{-tau2 (nu - shift2)}
  COL_OUTER1,      // s e^{-tau3 (nu - shift3)}
  COL_OUTER2,      // pair spectra E (eta, eta_t floored, phi, phi_t)
  COL_E44_PAIR,    // order 4: ((s e4) e3) e2 for third-level pairs, (s e4) e2 for order-4 pairs
  COL_E44_FIRST3,  // order 4: (s e4) e3
  COL_E44_FIRST4,  // order 4: s e4
  COL_FLOORED,     // bank k reads spectrum src_of[k] of the job with its own roundoff floor
};

constexpr int MAX_BANKS = 24;

struct ColArgs {
  int kind;
  int nbanks;
  int mult[MAX_BANKS];     // multiplier per bank
  int src_of[MAX_BANKS];   // spectrum index per bank (COL_PLAIN / COL_OUTER2)
  Box box;                 // input box (modes)
  const double* geo;       // geometry planes of the input box
  const cplx* spec;        // input spectra
  long long spec_job_stride;  // elements between jobs' spectra
  long long spec_sub_stride;  // elements between spectra within a job
  int jobs_per_unit;       // jobs sharing one unit's scalars / masks
  // damping parameters
  const UnitScalars* us;
  const double* nodes;     // GL nodes (outer for OUTER*, eta22 for ETA22)
  const double* nodes2;    // inner nodes
  int n_inner;             // inner rank (COL_INNER) / nodes per branch (PSI22)
  int n_outer;             // outer rank; eta44: outer nodes handled by this call
  int outer0;              // eta44: first outer node handled by this call
  const unsigned char* chan_mask;  // [unit][2][h][w] (COL_PSI22)
  const unsigned long long* floor_max;  // per-job max for floored spectra
  int floor_nsrc;          // COL_FLOORED: maxima per job (indexed job * floor_nsrc + src)
  double floor_rel;
  // output
  cplx* out;               // [job][bank][w][n]
  int n, log2n;            // transform length along y
  double scale;            // applied to the inverse transform (1/(Nx Ny))
  // 1: run the transform with the opposite exponent sign, through
  // conj(F(conj x)) -- the transpose of a forward transform, used by the
  // adjoint to carry adjoint spectra to the grid
  int conj_io;
  // Twin outputs (twins = 1): a bank whose multiplier is a column-constant
  // factor times another bank's (qx, i qx along a box column) is written from
  // that bank's transformed column instead of being transformed itself.  The
  // output then holds nout banks; transformed bank k goes to bank out_of[k]
  // and, when twin[k] >= 0, times twin_fac[k] (1: qx, 2: i qx of the column,
  // from the geometry's qx plane) to bank twin[k].
  int twins;
  int nout;
  int out_of[MAX_BANKS], twin[MAX_BANKS], twin_fac[MAX_BANKS];
  int cw_max;              // > 0: at most this many columns per block (a power of two; tuning)
};

// Damping base value of the job at box bin i (COL_ETA22/PSI22/INNER/OUTER1).
GL_D cplx col_base(const ColArgs& a, int job, int i, double nu) {
  const int unit = job / a.jobs_per_unit;
  const int sub = job % a.jobs_per_unit;
  const UnitScalars& u = a.us[unit];
  const cplx* s = a.spec + (long long)unit * a.spec_job_stride;
  cplx v = s[i];
  switch (a.kind) {
    case COL_ETA22: {
      const double tau = a.nodes[sub] / u.lam22;
      return cscale(exp(-tau * (nu - u.shift2)), v);
    }
    case COL_PSI22: {
      // sub = (branch * n_inner + node) * chan_count + channel
      const int chan = sub % 2;
      const int bn = sub / 2;
      const int branch = bn / a.n_inner;
      const int node = bn % a.n_inner;
      if (chan >= u.chan_count) return czero();
      const double lam = branch == 0 ? u.lam_minus : u.lam_plus;
      const double tau = a.nodes[node] / lam;
      const int cid = u.chan_id[chan];
      const unsigned char m =
          a.chan_mask[((size_t)unit * 2 + cid) * a.box.w * a.box.h + i];
      cplx sm = m ? v : cscale(0.0, v);
      return cscale(exp(-tau * (nu - u.chan_shift[chan])), sm);
    }
    case COL_INNER: {
      const int jo = sub / a.n_inner;
      const int ii = sub % a.n_inner;
      const double tau3 = a.nodes[jo] / u.lam3;
      const double tau2 = a.nodes2[ii] / u.lam2;
      cplx d3 = cscale(exp(-tau3 * (nu - u.shift3)), v);
      return cscale(exp(-tau2 * (nu - u.shift2)), d3);
    }
    case COL_OUTER1: {
      const double tau3 = a.nodes[sub] / u.lam3;
      return cscale(exp(-tau3 * (nu - u.shift3)), v);
    }
    case COL_E44_PAIR: {
      // local outer nodes ol = 0..n_outer-1 map to global o = outer0 + ol
      const int R = a.n_inner, Ro = a.n_outer;
      const int r3 = Ro * R * R;
      int o, t = -1, pn;
      if (sub < r3) {
        o = a.outer0 + sub / (R * R);
        t = (sub / R) % R;
        pn = sub % R;
      } else {
        o = a.outer0 + (sub - r3) / R;
        pn = (sub - r3) % R;
      }
      cplx d = cscale(exp(-(a.nodes[o] / u.lam4) * (nu - u.shift4)), v);
      if (t >= 0) d = cscale(exp(-(a.nodes[t] / u.lam3) * (nu - u.shift3)), d);
      return cscale(exp(-(a.nodes[pn] / u.lam2) * (nu - u.shift2)), d);
    }
    case COL_E44_FIRST3: {
      const int R = a.n_inner;
      const int o = a.outer0 + sub / R, t = sub % R;
      const cplx d = cscale(exp(-(a.nodes[o] / u.lam4) * (nu - u.shift4)), v);
      return cscale(exp(-(a.nodes[t] / u.lam3) * (nu - u.shift3)), d);
    }
    case COL_E44_FIRST4:
      return cscale(exp(-(a.nodes[a.outer0 + sub] / u.lam4) * (nu - u.shift4)), v);
  }
  return v;
}

// One block: `cw` box columns of one job.  Each column is one length-n
// inverse transform along y run by a group of n/16 threads; the damped base
// spectrum of the columns is computed once and every bank applies its
// multiplier while the first FFT pass reads it.  Output layout
// [job][bank][y][column] (rows contiguous for the row kernel).
template <int MIX>
__global__ void __launch_bounds__(256, 2) col_ifft_kernel(ColArgs a, const cplx* __restrict__ tw,
                                                         int cw, int banks_per_block) {
  extern __shared__ cplx smem[];
  const int job = blockIdx.y;
  const int x_first = blockIdx.x * cw;
  const int ncol = min(cw, a.box.w - x_first);
  const int k_first = blockIdx.z * banks_per_block;
  const int k_last = min(a.nbanks, k_first + banks_per_block);
  const int n = a.n;
  const int L = padded_len(n);
  const int h = a.box.h;
  const int plane = a.box.w * a.box.h;
  cplx* bufs = smem;                   // cw * L
  cplx* base = smem + (size_t)cw * L;  // cw * h
  const bool shared_base = a.kind != COL_PLAIN && a.kind != COL_OUTER2 && a.kind != COL_FLOORED;
  const int lcw = 31 - __clz(cw);  // cw is a power of two
  if (shared_base) {
    for (int t = threadIdx.x; t < (h << lcw); t += blockDim.x) {
      const int c = t & (cw - 1), by = t >> lcw;
      if (c >= ncol) continue;
      const int i = by * a.box.w + x_first + c;
      base[c * h + by] = col_base(a, job, i, __ldg(a.geo + 3 * plane + i));
    }
  }
  __syncthreads();
  int g, G;
  const FftGroup f = fft_group(n, a.log2n, g, G);
  const int iters = (ncol + G - 1) / G;
  // with at least two columns per warp the last pass writes the columns
  // straight to global memory (two adjacent columns fill each 32-byte
  // sector) and the banks need no block-wide barrier; longer columns (one
  // column per warp or more) are written back row-major through shared memory
  const bool direct = f.T <= 16;
  for (int k = k_first; k < k_last; ++k) {
    const int mult = a.mult[k];
    const cplx* sk = a.spec + (long long)job * a.spec_job_stride + (long long)a.src_of[k] * a.spec_sub_stride;
    const bool floor_it = a.floor_max && ((a.kind == COL_OUTER2 && a.src_of[k] == 1) || a.kind == COL_FLOORED);
    const double floor_abs =
        !floor_it ? 0.0
                  : a.floor_rel * as_double(a.kind == COL_FLOORED ? a.floor_max[(size_t)job * a.floor_nsrc + a.src_of[k]]
                                                                  : a.floor_max[job]);
    const int nout = a.twins ? a.nout : a.nbanks;
    const int tb = a.twins ? a.twin[k] : -1;
    const int tfac = tb >= 0 ? a.twin_fac[k] : 0;
    cplx* dst = a.out + ((size_t)job * nout + (a.twins ? a.out_of[k] : k)) * n * a.box.w + x_first;
    cplx* dst2 = tb >= 0 ? a.out + ((size_t)job * nout + tb) * n * a.box.w + x_first : nullptr;
    for (int it = 0; it < iters; ++it) {
      const int c = it * G + g;
      const bool active = c < ncol;
      cplx* buf = bufs + (size_t)(active ? c : 0) * L;
      cplx* dcol = dst + (active ? c : 0);
      cplx* dcol2 = dst2 ? dst2 + (active ? c : 0) : nullptr;
      const double qxc = (dst2 && active) ? __ldg(a.geo + x_first + c) : 0.0;  // qx plane, row 0
      // The group first writes its column's multiplied box rows to the front
      // of the column's buffer (one copy of the multiplier code in a short
      // loop, all loads independent); the first transform pass reads them
      // back before it writes the padded column over them.
      if (active) {
        for (int by = f.t; by < h; by += f.T) {
          const int i = by * a.box.w + x_first + c;
          cplx v;
          if (shared_base) {
            v = base[c * h + by];
          } else {
            v = sk[i];
            if (floor_it && abs_below(v, floor_abs)) v = czero();
          }
          const cplx mv = apply_mult(mult, GeoRef{a.geo, plane, i}, v);
          buf[by] = a.conj_io ? cconj(mv) : mv;
        }
      }
      f.sync();
      auto load = [&](int yb) -> cplx {
        const int by = wrap_any(yb - a.box.y0, n);
        return by < h ? buf[by] : czero();
      };
      auto store = [&](int yb, cplx v) {
        if (direct) {
          const cplx w = cscale(a.scale, a.conj_io ? cconj(v) : v);
          dcol[(size_t)yb * a.box.w] = w;
          if (dcol2) {
            const cplx u = cscale(qxc, w);
            dcol2[(size_t)yb * a.box.w] = tfac == 2 ? cmuli(u) : u;
          }
        } else {
          buf[phys(yb)] = v;
        }
      };
      fft_row<+1, MIX>(buf, f, active, tw, load, store);
    }
    if (!direct) {
      __syncthreads();
      for (int t = threadIdx.x; t < (n << lcw); t += blockDim.x) {
        const int y = t >> lcw, c = t & (cw - 1);
        if (c >= ncol) continue;
        const cplx v = bufs[(size_t)c * L + phys(y)];
        const cplx w = cscale(a.scale, a.conj_io ? cconj(v) : v);
        dst[(size_t)y * a.box.w + c] = w;
        if (dst2) {
          const cplx u = cscale(__ldg(a.geo + x_first + c), w);
          dst2[(size_t)y * a.box.w + c] = tfac == 2 ? cmuli(u) : u;
        }
      }
      __syncthreads();
    }
  }
}

// ---------------------------------------------------------------------------
// row kernel: inverse FFT along x, products, forward FFT along x
// ---------------------------------------------------------------------------

enum RowKind : int { ROW_ETA22 = 0, ROW_PSI22, ROW_CONTACT22, ROW_INNER, ROW_OUTER,
                     ROW_E44_PAIR, ROW_E44_THIRD, ROW_E44_ORDER4, ROW_E44_ORDER4_PSI,
                     // adjoint (transposed) products (row kernel family 1)
                     ROW_ADJ_ETA22, ROW_ADJ_INNER, ROW_ADJ_OUTER };

struct BankGroup {
  const cplx* data;  // [job][nb][w][n_y]
  int nb;            // banks in the group
  int x0, w;         // box columns (modes)
  int conj;          // 1: adjoint rows, transformed with the opposite sign
};

struct RowArgs {
  int kind;
  BankGroup grp[3];
  int ngrp;
  int nout;
  int out_x0, out_w;       // kept output columns (modes)
  cplx* out;               // [job][nout][out_w][n_y]
  int nx, log2nx;          // compact grid along x
  int ny;                  // compact grid along y (column length of inputs)
  UnitScalars* us;         // per-unit scalars; status word flagged on a timed-out copy
  int jobs_per_unit;
  int gmax;                // FFT group size (rows through tmp)
  // adjoint extensions (zero in the forward stages):
  int out_conj;            // 1: outputs transformed with the + sign
  int nout_a;              // > 0: outputs [nout_a, nout) go to out2 instead
  int out2_x0, out2_w;
  cplx* out2;              // [job][nout - nout_a][out2_w][n_y]
  int rpb;                 // rows per block (> 1 for short rows; 0 or 1: one)
  // failure-path test hook (gl_plan_set_wait_test; zero in normal runs):
  // bytes added to the staged rows' expected transaction count, so that the
  // bounded wait runs out, and that wait's clock budget (0: BULK_WAIT_CYCLES)
  unsigned int wait_surplus;
  long long wait_cycles;
  int groups;              // > 0: transform groups per row block (tuning); 0: built-in choice
  // order-4 rows of one part of the reference's split mode: 0 every
  // partition, 1 the base partitions 22, 211, 1111 only, 2 partition 31 only
  int e44_part;
};

// Pointwise products of each stage; `b` points at the bank rows (bank k at
// b + k*n), outputs overwrite the first rows at the same point.
GL_D void row_products(int kind, cplx* b, int L, int p, int chan_count) {
#define BK(k) b[(k) * L + p]
  switch (kind) {
    case ROW_ETA22: {  // spatial.py:204-205
      cplx v = BK(0), v1 = BK(1), v2 = BK(2), hx = BK(3), hy = BK(4), rad = BK(5), jx = BK(6),
           jy = BK(7);
      cplx sd = csub(csub(cadd(cmul(cscale(2.0, v), v2), csq(v1)), csq(hx)), csq(hy));
      cplx sk = cadd(cmul(cscale(2.0, v), rad), cscale(2.0, cadd(cmul(hx, jx), cmul(hy, jy))));
      BK(0) = sd;
      BK(1) = sk;
      break;
    }
    case ROW_PSI22: {  // spatial.py:370-380; banks: channel c at 8c..8c+7
      cplx r[8];
      for (int i = 0; i < 2; ++i) {
        for (int j = 0; j < 2; ++j) {
          const int o = 2 * (2 * i + j);
          if (i >= chan_count || j >= chan_count) { r[o] = czero(); r[o + 1] = czero(); continue; }
          const int li = 8 * i, ri = 8 * j;
          cplx sd = csub(csub(cadd(cmul(cscale(2.0, BK(li + 0)), BK(ri + 2)), cmul(BK(li + 1), BK(ri + 1))),
                              cmul(BK(li + 3), BK(ri + 3))),
                         cmul(BK(li + 4), BK(ri + 4)));
          cplx sk = cadd(cmul(cscale(2.0, BK(li + 0)), BK(ri + 5)),
                         cscale(2.0, cadd(cmul(BK(li + 3), BK(ri + 6)), cmul(BK(li + 4), BK(ri + 7)))));
          r[o] = sd;
          r[o + 1] = sk;
        }
      }
      for (int o = 0; o < 8; ++o) BK(o) = r[o];
      break;
    }
    case ROW_CONTACT22: {  // spatial.py:303-306: 0.5 * eta11 * (-i ifft2(s nu))
      cplx e = BK(0);
      cplx pz = cmulmi(BK(1));
      BK(0) = cmul(cscale(0.5, e), pz);
      break;
    }
    case ROW_INNER: {  // _order3.py:228-233
      cplx v = BK(0), v1 = BK(1), v2 = BK(2), v3 = BK(3), hx = BK(4), hy = BK(5), jx = BK(6),
           jy = BK(7), rad = BK(8), qq = BK(9), njx = BK(10), njy = BK(11);
      cplx v2x = cscale(2.0, v);
      cplx sd = csub(csub(cadd(cmul(v2x, v2), csq(v1)), csq(hx)), csq(hy));
      cplx sk = cadd(cmul(v2x, rad), cscale(2.0, cadd(cmul(hx, jx), cmul(hy, jy))));
      cplx sdt = csub(csub(cadd(cmul(v2x, v3), cmul(cscale(4.0, v1), v2)), cmul(cscale(2.0, hx), jx)),
                      cmul(cscale(2.0, hy), jy));
      cplx skt = cadd(cscale(2.0, cadd(cmul(v1, rad), cmul(v, qq))),
                      cscale(2.0, cadd(cadd(cadd(csq(jx), cmul(hx, njx)), csq(jy)), cmul(hy, njy))));
      BK(0) = sd;
      BK(1) = sk;
      BK(2) = sdt;
      BK(3) = skt;
      break;
    }
    case ROW_OUTER: {  // _order3.py:76-102, 275-287
      // first-order banks 0..11: eta etax etay phix phiy phiz phixz phiyz phizz phizzz phitz phitzz
      // pair banks 12..20: eta etax etay phix phiy phiz phizz phitz eta_t
      cplx fe = BK(0), fex = BK(1), fey = BK(2), fpx = BK(3), fpy = BK(4), fpz = BK(5),
           fpxz = BK(6), fpyz = BK(7), fpzz = BK(8), fpzzz = BK(9), fptz = BK(10), fptzz = BK(11);
      cplx pe = BK(12), pex = BK(13), pey = BK(14), ppx = BK(15), ppy = BK(16), ppz = BK(17),
           ppzz = BK(18), pptz = BK(19), pet = BK(20);
      // first-state aliases: eta_t = phiz, phiz_t = phitz, phizz_t = phitzz; pair phiz_t = phitz
      cplx fe2 = csq(fe);
      cplx k_pair = csub(csub(cadd(cadd(cadd(cmul(fpx, pex), cmul(fpy, pey)), cmul(ppx, fex)), cmul(ppy, fey)),
                              cmul(fe, ppzz)),
                         cmul(pe, fpzz));
      cplx k_direct = csub(cmul(fe, cadd(cmul(fpxz, fex), cmul(fpyz, fey))), cmul(cscale(0.5, fe2), fpzzz));
      cplx d_pair = cadd(cadd(cadd(cadd(cmul(fe, pptz), cmul(pe, fptz)), cmul(fpx, ppx)), cmul(fpy, ppy)),
                         cmul(fpz, ppz));
      cplx d_direct = cadd(cmul(cscale(0.5, fe2), fptzz),
                           cmul(fe, cadd(cadd(cmul(fpx, fpxz), cmul(fpy, fpyz)), cmul(fpz, fpzz))));
      cplx fk = cadd(cscale(0.25, k_direct), cscale(0.5, k_pair));
      cplx fd = cadd(cscale(0.25, d_direct), cscale(0.5, d_pair));
      cplx contact = cadd(cadd(cmul(cscale(0.5, fe), ppz), cmul(cscale(0.5, pe), fpz)),
                          cmul(cscale(0.125, fe2), fpzz));
      cplx contact_t =
          cadd(cadd(cadd(cscale(0.5, cadd(cmul(fpz, ppz), cmul(fe, pptz))),
                         cscale(0.5, cadd(cmul(pet, fpz), cmul(pe, fptz)))),
                    cmul(cmul(cscale(0.25, fe), fpz), fpzz)),
               cmul(cscale(0.125, fe2), fptzz));
      BK(0) = fk;
      BK(1) = fd;
      BK(2) = contact;
      BK(3) = contact_t;
      break;
    }
  }
#undef BK
}

// Pointwise products of the order-4 stages (gl_eta44_fftw.cpp), compiled into
// their own row kernel so that the wide order-4 rows do not weigh on the
// register allocation of the order-2/3 stages.
GL_D void row_products_e44(int kind, cplx* b, int L, int p, int part) {
#define BK(k) b[(k) * L + p]
  switch (kind) {
    case ROW_E44_PAIR: {  // gl_eta44_fftw.cpp:375-381: six pair sources from 16 banks
      const cplx v = BK(0), vn = BK(1), vn2 = BK(2), vn3 = BK(3), vn4 = BK(4), hx = BK(5),
                 hy = BK(6), jx = BK(7), jy = BK(8), ro = BK(9), qq = BK(10), q2n = BK(11),
                 njx = BK(12), njy = BK(13), n2jx = BK(14), n2jy = BK(15);
      const cplx v2 = cscale(2.0, v);
      const cplx sd = csub(csub(cadd(cmul(v2, vn2), cmul(vn, vn)), cmul(hx, hx)), cmul(hy, hy));
      const cplx sk = cadd(cmul(v2, ro), cscale(2.0, cadd(cmul(hx, jx), cmul(hy, jy))));
      const cplx sds = csub(csub(cadd(cmul(v2, vn3), cmul(cscale(4.0, vn), vn2)), cmul(cscale(2.0, hx), jx)),
                            cmul(cscale(2.0, hy), jy));
      const cplx jj = cadd(cadd(cadd(cmul(jx, jx), cmul(hx, njx)), cmul(jy, jy)), cmul(hy, njy));
      const cplx sks = cadd(cscale(2.0, cadd(cmul(vn, ro), cmul(v, qq))), cscale(2.0, jj));
      const cplx sdss = csub(cadd(cadd(cmul(v2, vn4), cmul(cscale(6.0, vn), vn3)), cmul(cscale(4.0, vn2), vn2)),
                             cscale(2.0, jj));
      const cplx skss = cadd(cadd(cscale(2.0, cadd(cadd(cmul(vn2, ro), cmul(cscale(2.0, vn), qq)), cmul(v, q2n))),
                                  cscale(6.0, cadd(cmul(jx, njx), cmul(jy, njy)))),
                             cscale(2.0, cadd(cmul(hx, n2jx), cmul(hy, n2jy))));
      BK(0) = sd;
      BK(1) = sk;
      BK(2) = sds;
      BK(3) = sks;
      BK(4) = sdss;
      BK(5) = skss;
      break;
    }
    case ROW_E44_THIRD: {  // gl_eta44_fftw.cpp:548-566: cubic forcing and its time derivative
      // first banks 0..15: eta ex ey px py pz pxz pyz pzz pzzz ptz ptzz pxz_t pyz_t pzzz_t ptz_t
      // pair banks 16..30: eta ex ey eta_t ex_t ey_t px py pz pzz ptz px_t py_t pzz_t ptz_t
      const cplx fe = BK(0), fex = BK(1), fey = BK(2), fpx = BK(3), fpy = BK(4), fpz = BK(5), fpxz = BK(6),
                 fpyz = BK(7), fpzz = BK(8), fpzzz = BK(9), fptz = BK(10), fptzz = BK(11), fpxzt = BK(12),
                 fpyzt = BK(13), fpzzzt = BK(14), fptzt = BK(15);
      const cplx pe = BK(16), pex = BK(17), pey = BK(18), pet = BK(19), pext = BK(20), peyt = BK(21),
                 ppx = BK(22), ppy = BK(23), ppz = BK(24), ppzz = BK(25), pptz = BK(26), ppxt = BK(27),
                 ppyt = BK(28), ppzzt = BK(29), pptzt = BK(30);
      const cplx hfe = cscale(0.5, fe);
      const cplx kp = csub(csub(cadd(cadd(cadd(cmul(fpx, pex), cmul(fpy, pey)), cmul(ppx, fex)), cmul(ppy, fey)),
                                cmul(fe, ppzz)), cmul(pe, fpzz));
      const cplx kd = csub(cmul(fe, cadd(cmul(fpxz, fex), cmul(fpyz, fey))), cmul(cmul(hfe, fe), fpzzz));
      const cplx dp = cadd(cadd(cadd(cadd(cmul(fe, pptz), cmul(pe, fptz)), cmul(fpx, ppx)), cmul(fpy, ppy)),
                           cmul(fpz, ppz));
      const cplx dd = cadd(cmul(cmul(hfe, fe), fptzz),
                           cmul(fe, cadd(cadd(cmul(fpx, fpxz), cmul(fpy, fpyz)), cmul(fpz, fpzz))));
      cplx kpt = cmul(cmk(-fex.x, -fex.y), pex);
      kpt = cadd(kpt, cmul(fpx, pext));
      kpt = csub(kpt, cmul(fey, pey));
      kpt = cadd(kpt, cmul(fpy, peyt));
      kpt = cadd(kpt, cmul(ppxt, fex));
      kpt = cadd(kpt, cmul(ppx, fpxz));
      kpt = cadd(kpt, cmul(ppyt, fey));
      kpt = cadd(kpt, cmul(ppy, fpyz));
      kpt = csub(kpt, cmul(fpz, ppzz));
      kpt = csub(kpt, cmul(fe, ppzzt));
      kpt = csub(kpt, cmul(pet, fpzz));
      kpt = csub(kpt, cmul(pe, fptzz));
      const cplx kdt = csub(csub(cadd(cmul(fpz, cadd(cmul(fpxz, fex), cmul(fpyz, fey))),
                                      cmul(fe, cadd(cadd(cadd(cmul(fpxzt, fex), cmul(fpxz, fpxz)), cmul(fpyzt, fey)),
                                                    cmul(fpyz, fpyz)))),
                                 cmul(cmul(fe, fpz), fpzzz)),
                            cmul(cmul(hfe, fe), fpzzzt));
      cplx dpt = cmul(fpz, pptz);
      dpt = cadd(dpt, cmul(fe, pptzt));
      dpt = cadd(dpt, cmul(pet, fptz));
      dpt = cadd(dpt, cmul(pe, fptzt));
      dpt = csub(dpt, cmul(fex, ppx));
      dpt = cadd(dpt, cmul(fpx, ppxt));
      dpt = csub(dpt, cmul(fey, ppy));
      dpt = cadd(dpt, cmul(fpy, ppyt));
      dpt = cadd(dpt, cmul(fptz, ppz));
      dpt = cadd(dpt, cmul(fpz, pptz));
      cplx inner = cmul(cmk(-fex.x, -fex.y), fpxz);
      inner = cadd(inner, cmul(fpx, fpxzt));
      inner = csub(inner, cmul(fey, fpyz));
      inner = cadd(inner, cmul(fpy, fpyzt));
      inner = cadd(inner, cmul(fptz, fpzz));
      inner = cadd(inner, cmul(fpz, fptzz));
      const cplx ddt = cadd(cadd(csub(cmul(cmul(fe, fpz), fptzz), cmul(cmul(hfe, fe), fpzzz)),
                                 cmul(fpz, cadd(cadd(cmul(fpx, fpxz), cmul(fpy, fpyz)), cmul(fpz, fpzz)))),
                            cmul(fe, inner));
      BK(0) = cadd(cscale(0.25, kd), cscale(0.5, kp));
      BK(1) = cadd(cscale(0.25, dd), cscale(0.5, dp));
      BK(2) = cadd(cscale(0.25, kdt), cscale(0.5, kpt));
      BK(3) = cadd(cscale(0.25, ddt), cscale(0.5, dpt));
      break;
    }
    case ROW_E44_ORDER4:
    case ROW_E44_ORDER4_PSI: {  // gl_eta44_fftw.cpp:712-735: partitions 31, 22, 211, 1111
      // first4 banks 0..18: eta ex ey px py pz pxz pyz pzz pzzz ptz ptzz pxz_t pyz_t pzzz_t ptz_t pxzz pyzz pzzzz
      // pair4 banks 19..36: eta ex ey eta_t ex_t ey_t px py pz pzz ptz px_t py_t pzz_t ptz_t pxz pyz pzzz
      // third banks 37..44: eta ex ey px py pz pzz pzt
      const cplx fe = BK(0), fex = BK(1), fey = BK(2), fpx = BK(3), fpy = BK(4), fpz = BK(5), fpxz = BK(6),
                 fpyz = BK(7), fpzz = BK(8), fpzzz = BK(9), fptz = BK(10), fptzz = BK(11),
                 fpzzzt = BK(14), fpxzz = BK(16), fpyzz = BK(17), fpzzzz = BK(18);
      const cplx pe = BK(19), pex = BK(20), pey = BK(21), ppx = BK(25), ppy = BK(26), ppz = BK(27),
                 ppzz = BK(28), pptz = BK(29), ppzzt = BK(32), ppxz = BK(34), ppyz = BK(35), ppzzz = BK(36);
      const cplx te = BK(37), tex = BK(38), tey = BK(39), tpx = BK(40), tpy = BK(41), tpz = BK(42),
                 tpzz = BK(43), tpzt = BK(44);
      const cplx hfe = cscale(0.5, fe);
      const cplx k31 = csub(csub(cadd(cadd(cadd(cmul(fpx, tex), cmul(fpy, tey)), cmul(tpx, fex)), cmul(tpy, fey)),
                                 cmul(fe, tpzz)), cmul(te, fpzz));
      const cplx d31 = cadd(cadd(cadd(cadd(cmul(fe, tpzt), cmul(te, fptz)), cmul(fpx, tpx)), cmul(fpy, tpy)),
                            cmul(fpz, tpz));
      const cplx k22 = csub(cadd(cmul(ppx, pex), cmul(ppy, pey)), cmul(pe, ppzz));
      const cplx d22 = cadd(cmul(pe, pptz), cscale(0.5, cadd(cadd(cmul(ppx, ppx), cmul(ppy, ppy)), cmul(ppz, ppz))));
      const cplx mx_ = cadd(cmul(fe, ppxz), cmul(pe, fpxz));
      const cplx my_ = cadd(cmul(fe, ppyz), cmul(pe, fpyz));
      const cplx mz_ = cadd(cmul(fe, ppzz), cmul(pe, fpzz));
      const cplx k211 = csub(csub(cadd(cadd(cmul(fe, cadd(cmul(fpxz, pex), cmul(fpyz, pey))), cmul(mx_, fex)),
                                       cmul(my_, fey)),
                                  cmul(cmul(hfe, fe), ppzzz)),
                             cmul(cmul(fe, pe), fpzzz));
      cplx d211 = cmul(cmul(hfe, fe), ppzzt);
      d211 = cadd(d211, cmul(cmul(fe, pe), fptzz));
      d211 = cadd(d211, cmul(fpx, mx_));
      d211 = cadd(d211, cmul(fpy, my_));
      d211 = cadd(d211, cmul(fpz, mz_));
      d211 = cadd(d211, cmul(ppx, cmul(fe, fpxz)));
      d211 = cadd(d211, cmul(ppy, cmul(fe, fpyz)));
      d211 = cadd(d211, cmul(ppz, cmul(fe, fpzz)));
      const cplx hfe2 = cmul(hfe, fe);
      const cplx fe3 = cmul(cmul(fe, fe), fe);
      const cplx k3v = cmul(fe3, fpzzzz);
      const cplx k1111 = csub(cmul(hfe2, cadd(cmul(fpxzz, fex), cmul(fpyzz, fey))), cmk(k3v.x / 6.0, k3v.y / 6.0));
      const cplx d3v = cmul(fe3, fpzzzt);
      const cplx d1111 = cadd(cadd(cmk(d3v.x / 6.0, d3v.y / 6.0),
                                   cmul(hfe2, cadd(cadd(cmul(fpx, fpxzz), cmul(fpy, fpyzz)), cmul(fpz, fpzzz)))),
                              cmul(hfe2, cadd(cadd(cmul(fpxz, fpxz), cmul(fpyz, fpyz)), cmul(fpzz, fpzz))));
      const cplx kb = cadd(cadd(cscale(0.125, k1111), cscale(0.25, k211)), cscale(0.5, k22));
      const cplx db = cadd(cadd(cscale(0.125, d1111), cscale(0.25, d211)), cscale(0.5, d22));
      if (kind == ROW_E44_ORDER4_PSI) {
        // psi44 surface contact and its time derivative
        // (...eta44_three_kernels.m:221-241); bank 45 = third-order eta_t,
        // first-order eta_t = phiz, phiz_t = phitz, phizz_t = phitzz
        const cplx pet = BK(22), tet = BK(45);
        const cplx fefe = cmul(fe, fe);
        const cplx fepe = cmul(fe, pe);
        const cplx c = cadd(cadd(cadd(cscale(0.5, cmul(fe, tpz)), cscale(0.5, cmul(pe, ppz))),
                                 cadd(cscale(0.5, cmul(te, fpz)), cscale(0.125, cmul(fefe, ppzz)))),
                            cadd(cscale(0.25, cmul(fepe, fpzz)),
                                 cscale(1.0 / 48.0, cmul(cmul(fefe, fe), fpzzz))));
        cplx ct = cscale(0.5, cadd(cmul(fpz, tpz), cmul(fe, tpzt)));
        ct = cadd(ct, cscale(0.5, cadd(cmul(pet, ppz), cmul(pe, pptz))));
        ct = cadd(ct, cscale(0.5, cadd(cmul(tet, fpz), cmul(te, fptz))));
        ct = cadd(ct, cscale(0.125, cadd(cscale(2.0, cmul(cmul(fe, fpz), ppzz)), cmul(fefe, ppzzt))));
        ct = cadd(ct, cscale(0.25, cadd(cadd(cmul(cmul(fpz, pe), fpzz), cmul(cmul(fe, pet), fpzz)),
                                        cmul(fepe, fptzz))));
        ct = cadd(ct, cscale(1.0 / 48.0, cadd(cscale(3.0, cmul(cmul(fefe, fpz), fpzzz)),
                                              cmul(cmul(fefe, fe), fpzzzt))));
        BK(2) = c;
        BK(3) = ct;
      }
      // split-mode parts (gl_eta44_fftw.cpp:706-735): base partitions or 31 alone
      BK(0) = part == 1 ? kb : part == 2 ? cscale(0.5, k31) : cadd(cscale(0.5, k31), kb);
      BK(1) = part == 1 ? db : part == 2 ? cscale(0.5, d31) : cadd(cscale(0.5, d31), db);
      break;
    }
  }
#undef BK
}

// Transposed products of the adjoint stages.  Every forward product is a
// polynomial P(f_1..f_m) of the bank fields; given the adjoint field w of
// each product (the transposed forward FFT of its adjoint spectrum) the
// adjoint of bank f_b is sum_P (dP/df_b) w_P, evaluated pointwise with the
// forward bank values recomputed in the same row.  No conjugates appear:
// the GL graph is holomorphic in the parent spectrum.
GL_D void row_products_adj(int kind, cplx* b, int L, int p) {
#define BK(k) b[(k) * L + p]
  switch (kind) {
    case ROW_ADJ_ETA22: {  // transpose of ROW_ETA22; banks 0..7 forward, 8 w(sd), 9 w(sk)
      const cplx v = BK(0), v1 = BK(1), v2 = BK(2), hx = BK(3), hy = BK(4), rad = BK(5), jx = BK(6),
                 jy = BK(7), wd = BK(8), wk = BK(9);
      const cplx d2 = cscale(2.0, wd), k2 = cscale(2.0, wk);
      BK(0) = cadd(cmul(v2, d2), cmul(rad, k2));
      BK(1) = cmul(v1, d2);
      BK(2) = cmul(v, d2);
      BK(3) = csub(cmul(jx, k2), cmul(hx, d2));
      BK(4) = csub(cmul(jy, k2), cmul(hy, d2));
      BK(5) = cmul(v, k2);
      BK(6) = cmul(hx, k2);
      BK(7) = cmul(hy, k2);
      break;
    }
    case ROW_ADJ_INNER: {  // transpose of ROW_INNER; banks 0..11 forward, 12..15 w(sd, sk, sdt, skt)
      const cplx v = BK(0), v1 = BK(1), v2 = BK(2), v3 = BK(3), hx = BK(4), hy = BK(5), jx = BK(6),
                 jy = BK(7), rad = BK(8), qq = BK(9), njx = BK(10), njy = BK(11);
      const cplx w0 = cscale(2.0, BK(12)), w1 = cscale(2.0, BK(13)), w2 = cscale(2.0, BK(14)),
                 w3 = cscale(2.0, BK(15));
      BK(0) = cadd(cadd(cmul(v2, w0), cmul(rad, w1)), cadd(cmul(v3, w2), cmul(qq, w3)));
      BK(1) = cadd(cadd(cmul(v1, w0), cscale(2.0, cmul(v2, w2))), cmul(rad, w3));
      BK(2) = cadd(cmul(v, w0), cscale(2.0, cmul(v1, w2)));
      BK(3) = cmul(v, w2);
      BK(4) = cadd(csub(cmul(jx, w1), cmul(hx, w0)), csub(cmul(njx, w3), cmul(jx, w2)));
      BK(5) = cadd(csub(cmul(jy, w1), cmul(hy, w0)), csub(cmul(njy, w3), cmul(jy, w2)));
      BK(6) = cadd(cmul(hx, csub(w1, w2)), cscale(2.0, cmul(jx, w3)));
      BK(7) = cadd(cmul(hy, csub(w1, w2)), cscale(2.0, cmul(jy, w3)));
      BK(8) = cadd(cmul(v, w1), cmul(v1, w3));
      BK(9) = cmul(v, w3);
      BK(10) = cmul(hx, w3);
      BK(11) = cmul(hy, w3);
      break;
    }
    case ROW_ADJ_OUTER: {
      // transpose of the fk, fd rows of ROW_OUTER; banks 0..11 first-order,
      // 12..20 pair (eta_t at 20 is not used by fk, fd), 21 w(fk), 22 w(fd).
      // Outputs: 0..11 first-order adjoints, 12..19 pair adjoints (banks 12..19).
      const cplx fe = BK(0), fex = BK(1), fey = BK(2), fpx = BK(3), fpy = BK(4), fpz = BK(5),
                 fpxz = BK(6), fpyz = BK(7), fpzz = BK(8), fpzzz = BK(9), fptz = BK(10), fptzz = BK(11);
      const cplx pe = BK(12), pex = BK(13), pey = BK(14), ppx = BK(15), ppy = BK(16), ppz = BK(17),
                 ppzz = BK(18), pptz = BK(19);
      const cplx wk = BK(21), wd = BK(22);
      // fk = k_direct/4 + k_pair/2, fd = d_direct/4 + d_pair/2
      const cplx K = cscale(0.5, wk), Kd = cscale(0.25, wk), D = cscale(0.5, wd), Dd = cscale(0.25, wd);
      const cplx kin = csub(cadd(cmul(fpxz, fex), cmul(fpyz, fey)), cmul(fe, fpzzz));
      const cplx din = cadd(cmul(fe, fptzz),
                            cadd(cadd(cmul(fpx, fpxz), cmul(fpy, fpyz)), cmul(fpz, fpzz)));
      const cplx hfe2 = cmul(cscale(0.5, fe), fe);
      const cplx feKd = cmul(fe, Kd), feDd = cmul(fe, Dd);
      BK(0) = cadd(cadd(cmul(Kd, kin), cmul(Dd, din)), csub(cmul(D, pptz), cmul(K, ppzz)));
      BK(1) = cadd(cmul(feKd, fpxz), cmul(K, ppx));
      BK(2) = cadd(cmul(feKd, fpyz), cmul(K, ppy));
      BK(3) = cadd(cadd(cmul(K, pex), cmul(D, ppx)), cmul(feDd, fpxz));
      BK(4) = cadd(cadd(cmul(K, pey), cmul(D, ppy)), cmul(feDd, fpyz));
      BK(5) = cadd(cmul(D, ppz), cmul(feDd, fpzz));
      BK(6) = cadd(cmul(feKd, fex), cmul(feDd, fpx));
      BK(7) = cadd(cmul(feKd, fey), cmul(feDd, fpy));
      BK(8) = csub(cmul(feDd, fpz), cmul(K, pe));
      BK(9) = cscale(-1.0, cmul(Kd, hfe2));
      BK(10) = cmul(D, pe);
      BK(11) = cmul(Dd, hfe2);
      BK(12) = csub(cmul(D, fptz), cmul(K, fpzz));
      BK(13) = cmul(K, fpx);
      BK(14) = cmul(K, fpy);
      BK(15) = cadd(cmul(K, fex), cmul(D, fpx));
      BK(16) = cadd(cmul(K, fey), cmul(D, fpy));
      BK(17) = cmul(D, fpz);
      BK(18) = cscale(-1.0, cmul(K, fe));
      BK(19) = cmul(D, fe);
      break;
    }
  }
#undef BK
}

// One block per (row y, job): inverse transforms along x of every bank (the
// first pass reads the column-transformed rows straight from global memory,
// zero outside the bank's box columns, 16 loads in flight per thread), the
// stage's products, forward transforms of the outputs, and only the output
// box's columns are written: [job][out][y][col].
// One instantiation per row kind, so that each stage's products are compiled
// (and get registers) on their own.  FAMILY 0: order-2/3 stages, 1: adjoint
// stages, 2: order-4 stages (their rows are wider than 24 banks and are
// staged in shared memory first).
// MIX = m > 0: the row length is the mixed length 16 m (pair stages on a
// product grid narrower than a power of two); 0: a power of two.  MULTI:
// several short rows per block (RowArgs::rpb).
// B192: launched with at most 192 threads (the order-3 outer row of 256
// points: 12 groups of 16, 92 KB of shared memory, 2 blocks per SM), so 2
// blocks per SM leave it 168 registers instead of the 128 of 2 x 256.
template <int KIND, int MIX = 0, bool MULTI = false, bool B192 = false>
__global__ void __launch_bounds__(B192 ? 192 : 256, 2) row_kernel_t(RowArgs a, const cplx* __restrict__ tw) {
  constexpr int FAMILY = KIND >= ROW_ADJ_ETA22 ? 1 : (KIND >= ROW_E44_PAIR && KIND <= ROW_E44_ORDER4_PSI ? 2 : 0);
  extern __shared__ __align__(128) cplx smem[];
  __shared__ __align__(8) unsigned long long stage_bar;
  // MULTI: a.rpb rows per block, each row with its own team of
  // blockDim.x / rpb threads and its own nb bank rows of shared memory
  const int rpb = MULTI && a.rpb > 1 ? a.rpb : 1;
  const int team = blockDim.x / rpb;
  const int rr = MULTI ? threadIdx.x / team : 0;
  const int tl = MULTI ? threadIdx.x % team : threadIdx.x;
  const int y0 = blockIdx.x * rpb;
  const int y = y0 + rr;
  const bool row_ok = !MULTI || y < a.ny;
  const int job = blockIdx.y;
  const int n = a.nx;
  const int L = padded_len(n);
  int nb = 0;
  for (int q = 0; q < a.ngrp; ++q) nb += a.grp[q].nb;
  cplx* banks = smem + (size_t)rr * nb * L;  // this row's nb * L
  // Stage every bank's box row (w contiguous values) into the front of the
  // bank's own row buffer with bulk async copies, all issued at block start,
  // so the later transform rounds find their inputs in shared memory.  The
  // first pass of a bank's transform reads its staged values into registers
  // before the group writes the padded row over them.
  const uint32_t bar = smem_u32(&stage_bar);
  if (threadIdx.x == 0) mbar_init(bar, 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nrows = MULTI ? min(rpb, a.ny - y0) : 1;
    uint32_t bytes = 0;
    for (int q = 0; q < a.ngrp; ++q) bytes += (uint32_t)(a.grp[q].nb * a.grp[q].w * sizeof(cplx));
    mbar_arrive_expect_tx(bar, bytes * (uint32_t)nrows + a.wait_surplus);
    for (int r = 0; r < nrows; ++r) {
      cplx* rb = smem + (size_t)r * nb * L;
      int k0 = 0;
      for (int q = 0; q < a.ngrp; ++q) {
        const BankGroup& B = a.grp[q];
        for (int kk = 0; kk < B.nb; ++kk)
          bulk_g2s(smem_u32(rb + (size_t)(k0 + kk) * L),
                   B.data + (((size_t)job * B.nb + kk) * a.ny + y0 + r) * B.w, (uint32_t)(B.w * sizeof(cplx)),
                   bar);
        k0 += B.nb;
      }
    }
  }
  {
    const long long budget = a.wait_cycles > 0 ? a.wait_cycles : BULK_WAIT_CYCLES;
    bool late = !mbar_wait_bounded(bar, 0, budget);
    if (__syncthreads_or(late)) {
      // a copy never landed: flag the unit, give the copies one more bounded
      // wait so none is left writing this block's shared memory, and leave
      // (a test's planted surplus is completed first, so that wait ends as
      // soon as the real copies have landed)
      if (threadIdx.x == 0) {
        if (a.us && a.jobs_per_unit > 0) atomicCAS(&a.us[job / a.jobs_per_unit].status, 0, (int)GL_ERR_TIMEOUT);
        if (a.wait_surplus) mbar_complete_tx(bar, a.wait_surplus);
      }
      mbar_wait_bounded(bar, 0, budget);
      return;
    }
  }
  int g, G;
  const FftGroup f = fft_group_team(n, a.log2nx, tl, team, 1 + rr * (team / (MIX ? 16 : (n >> 4))), g, G);
  for (int it = 0; it < (nb + G - 1) / G; ++it) {
    const int k = it * G + g;
    const bool active = k < nb && row_ok;
    cplx* buf = banks + (size_t)(active ? k : 0) * L;
    bool cj = false;
    int bx0 = 0, bw = 0;
    {
      const int kk0 = active ? k : 0;
      int k0 = 0;
      for (int q = 0; q < a.ngrp; ++q) {
        if (kk0 >= k0 && kk0 < k0 + a.grp[q].nb) {
          const BankGroup& B = a.grp[q];
          cj = FAMILY == 1 && B.conj != 0;
          bx0 = B.x0;
          bw = B.w;
        }
        k0 += a.grp[q].nb;
      }
    }
    auto load = [&](int xb) -> cplx {
      const int xi = MIX ? wrap_any(xb - bx0, n) : wrap(xb - bx0, n);
      const cplx v = xi < bw ? buf[xi] : czero();  // staged box row
      return cj ? cconj(v) : v;
    };
    auto store = [&](int xb, cplx v) { buf[phys(xb)] = cj ? cconj(v) : v; };
    fft_row<+1, MIX>(buf, f, active, tw, load, store);
  }
  __syncthreads();
  if (row_ok) {
    if constexpr (FAMILY == 0) {
      const int chan_count = KIND == ROW_PSI22 ? a.us[job / a.jobs_per_unit].chan_count : 0;
      for (int p = tl; p < n; p += team) row_products(KIND, banks, L, phys(p), chan_count);
    } else if constexpr (FAMILY == 2) {
      for (int p = tl; p < n; p += team) row_products_e44(KIND, banks, L, phys(p), a.e44_part);
    } else {
      for (int p = tl; p < n; p += team) row_products_adj(KIND, banks, L, phys(p));
    }
  }
  __syncthreads();
  const int na = a.nout_a > 0 ? a.nout_a : a.nout;
  const bool oc = FAMILY == 1 && a.out_conj != 0;
  for (int it = 0; it < (a.nout + G - 1) / G; ++it) {
    const int o = it * G + g;
    const bool active = o < a.nout && row_ok;
    const int oo = active ? o : 0;
    cplx* buf = banks + (size_t)oo * L;
    const bool second = oo >= na;
    const int ox0 = second ? a.out2_x0 : a.out_x0;
    const int ow = second ? a.out2_w : a.out_w;
    const int yr = row_ok ? y : 0;
    cplx* orow = second ? a.out2 + (((size_t)job * (a.nout - na) + (oo - na)) * a.ny + yr) * ow
                        : a.out + (((size_t)job * na + oo) * a.ny + yr) * ow;
    auto load = [&](int xb) -> cplx {
      const cplx v = buf[phys(xb)];
      return oc ? cconj(v) : v;
    };
    auto store = [&](int xb, cplx v) {
      const int xo = MIX ? wrap_any(xb - ox0, n) : wrap(xb - ox0, n);
      if (xo < ow) orow[xo] = oc ? cconj(v) : v;
    };
    fft_row<-1, MIX>(buf, f, active, tw, load, store);
  }
}

// ---------------------------------------------------------------------------
// column forward FFT + support mask + per-spectrum max
// ---------------------------------------------------------------------------

struct ColFftArgs {
  const cplx* in;          // [js][out_w][n]
  cplx* out;               // [js][box h][box w]
  Box box;                 // output box (modes)
  int n, log2n;            // compact grid along y
  int nsrc;                // spectra per job
  int jobs_per_unit;
  const unsigned char* mask;   // [unit][h][w] or null
  unsigned long long* maxslot; // [js] or null
  double scale;            // (Nx Ny)/(Ncx Ncy)
  int conj_io = 0;         // 1: + sign transform, conj(F(conj x)) (adjoint seeds)
  int cw_max = 0;          // > 0: at most this many columns per block (a power of two; tuning)
};

// One block: `cw` kept columns of one (job, source) spectrum.  Rows of the
// input ([js][y][col]) are staged with coalesced loads, each column is one
// forward transform along y, and only the output box's rows are written
// (support-masked), with the spectrum's max |.| folded into maxslot.
template <int MIX>
__global__ void __launch_bounds__(256, 2) col_fft_kernel(ColFftArgs a, const cplx* __restrict__ tw, int cw) {
  extern __shared__ cplx smem[];
  const int js = blockIdx.y;
  const int job = js / a.nsrc;
  const int unit = job / a.jobs_per_unit;
  const int x_first = blockIdx.x * cw;
  const int ncol = min(cw, a.box.w - x_first);
  const int n = a.n;
  const int L = padded_len(n);
  cplx* bufs = smem;  // cw * L
  const cplx* src = a.in + (size_t)js * n * a.box.w + x_first;
  // stage the kept columns ([y][col] rows in global memory) with eight
  // independent loads in flight per thread
  const int lcw = 31 - __clz(cw);  // cw is a power of two: (y, c) = (t >> lcw, t & (cw - 1))
  const int total = n << lcw;
  for (int t0 = threadIdx.x; t0 < total; t0 += 8 * blockDim.x) {
    cplx v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int t = t0 + u * blockDim.x;
      if (t < total && (t & (cw - 1)) < ncol) v[u] = src[(size_t)(t >> lcw) * a.box.w + (t & (cw - 1))];
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int t = t0 + u * blockDim.x;
      if (t < total && (t & (cw - 1)) < ncol)
        bufs[(size_t)(t & (cw - 1)) * L + phys(t >> lcw)] = a.conj_io ? cconj(v[u]) : v[u];
    }
  }
  __syncthreads();
  int g, G;
  const FftGroup f = fft_group(n, a.log2n, g, G);
  for (int it = 0; it < (ncol + G - 1) / G; ++it) {
    const int c = it * G + g;
    const bool active = c < ncol;
    cplx* buf = bufs + (size_t)(active ? c : 0) * L;
    auto load = [&](int yb) -> cplx { return buf[phys(yb)]; };
    auto store = [&](int yb, cplx v) { buf[phys(yb)] = v; };
    fft_row<-1, MIX>(buf, f, active, tw, load, store);
  }
  __syncthreads();
  const unsigned char* mask = a.mask ? a.mask + (size_t)unit * a.box.w * a.box.h : nullptr;
  cplx* dst = a.out + (size_t)js * a.box.w * a.box.h;
  double local = 0.0;
  for (int t = threadIdx.x; t < (a.box.h << lcw); t += blockDim.x) {
    const int c = t & (cw - 1), by = t >> lcw;
    if (c >= ncol) continue;
    const int i = by * a.box.w + x_first + c;
    const cplx raw = bufs[(size_t)c * L + phys(wrap_any(a.box.y0 + by, n))];
    cplx v = cscale(a.scale, a.conj_io ? cconj(raw) : raw);
    if (mask && !mask[i]) v = czero();
    dst[i] = v;
    local = keep_max_abs(local, v);
  }
  if (a.maxslot) {
    for (int o = 16; o > 0; o >>= 1) {
      const double other = __shfl_xor_sync(0xffffffffu, local, o);
      local = (other > local || other != other) ? other : local;
    }
    if ((threadIdx.x & 31) == 0) atomic_max_nonneg(a.maxslot + js, local);
  }
}

// ---------------------------------------------------------------------------
// accumulation kernels (elementwise over output boxes)
// ---------------------------------------------------------------------------

GL_D cplx floored(cplx v, double rel, unsigned long long peak_bits) {
  return abs_below(v, rel * as_double(peak_bits)) ? czero() : v;
}

struct AccArgs {
  const UnitScalars* us;
  const double* geo;        // geometry planes of the output box
  Box box;
  const cplx* in;           // stage spectra
  const unsigned long long* maxin;
  cplx* out;
  unsigned long long* maxout;
  const unsigned char* mask;    // [unit][h][w]
  const unsigned char* pmask;   // psi22 channel-pair masks [unit][3][h][w]
  const cplx* extra;        // psi22 contact spectrum [unit][h][w]
  const double* nodes;
  const double* weights;
  int nnodes;               // rank of the accumulated loop
  int nsub;                 // outer loop count (order-3 inner acc: jobs per unit)
  double floor_rel;
};

constexpr int ACC_TILE = 64;  // a multiple of 32: each warp's items share one outer node

#ifndef GL_TRANSFORM_TU  // elementwise kernels: compiled by gl_engine.cu only
// eta22: sum_n coef_n (-A sh_n sd_n + ch_n sk_n)   (spatial.py:206-221)
__global__ void acc_eta22_kernel(AccArgs a) {
  const int unit = blockIdx.y;
  const int plane = a.box.w * a.box.h;
  const UnitScalars& u = a.us[unit];
  // per-node times and coefficients, once per block
  __shared__ double s_tau[MAX_RANK], s_coef[MAX_RANK];
  if (threadIdx.x < a.nnodes) {
    const double x = a.nodes[threadIdx.x], w = a.weights[threadIdx.x];
    const double tau = x / u.lam22;
    s_tau[threadIdx.x] = tau;
    s_coef[threadIdx.x] = w * exp(x) / u.lam22 / 4.0 * exp(-2.0 * u.shift2 * tau);
  }
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < plane; i += gridDim.x * blockDim.x) {
    BinGeo g = load_geo(a.geo, plane, i);
    cplx acc = czero();
    for (int nn = 0; nn < a.nnodes; ++nn) {
      const int js = unit * a.nnodes + nn;
      const double tau = s_tau[nn];
      const double coef = s_coef[nn];
      const double sh = sinh_over_root(g.sqa, tau);
      const double ch = cosh(g.sqa * tau);
      cplx sd = floored(a.in[((size_t)js * 2 + 0) * plane + i], a.floor_rel, a.maxin[js * 2 + 0]);
      cplx sk = floored(a.in[((size_t)js * 2 + 1) * plane + i], a.floor_rel, a.maxin[js * 2 + 1]);
      cplx term = cadd(cscale(-g.a * sh, sd), cscale(ch, sk));
      acc = cadd(acc, cscale(coef, term));
    }
    a.out[(size_t)unit * plane + i] = acc;
  }
}

// psi22 dual-branch resolvent + Taylor contact, masked to the pair support
// (spatial.py:276-308, 384-393).
__global__ void acc_psi22_kernel(AccArgs a) {
  const int unit = blockIdx.y;
  const int plane = a.box.w * a.box.h;
  const UnitScalars& u = a.us[unit];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < plane; i += gridDim.x * blockDim.x) {
    BinGeo g = load_geo(a.geo, plane, i);
    cplx res = czero();
    for (int branch = 0; branch < 2; ++branch) {
      const double lam = branch == 0 ? u.lam_minus : u.lam_plus;
      const double ksign = branch == 0 ? -1.0 : 1.0;
      for (int nn = 0; nn < a.nnodes; ++nn) {
        const double x = a.nodes[nn], w = a.weights[nn];
        const double tau = x / lam;
        const double coef = w * exp(x) / lam / 8.0;
        const int js = (unit * 2 + branch) * a.nnodes + nn;
        cplx resp = czero();
        for (int ci = 0; ci < u.chan_count; ++ci) {
          for (int cj = 0; cj < u.chan_count; ++cj) {
            const int o = 2 * (2 * ci + cj);
            const cplx sd = a.in[((size_t)js * 8 + o) * plane + i];
            const cplx sk = a.in[((size_t)js * 8 + o + 1) * plane + i];
            const double ssum = u.chan_shift[ci] + u.chan_shift[cj];
            const double factor =
                branch == 0 ? exp((g.sqa - ssum) * tau) : exp(-(g.sqa + ssum) * tau);
            const cplx ks = cscale(ksign, sk);
            const double sa = safe_nu(g.sqa);
            cplx part = cscale(factor, cadd(sd, cmk(ks.x / sa, ks.y / sa)));
            // pair support of the physical channel pair
            const int pi = u.chan_id[ci] + u.chan_id[cj];  // 0: (0,0) 1: (0,1)/(1,0) 2: (1,1)
            const int pidx = (u.chan_count == 1) ? (u.chan_id[0] == 0 ? 0 : 2) : pi;
            if (!a.pmask[((size_t)unit * 3 + pidx) * plane + i]) part = czero();
            resp = cadd(resp, part);
          }
        }
        res = cadd(res, cmul(cmk(0.0, coef), resp));
      }
    }
    cplx total = cadd(res, a.extra[(size_t)unit * plane + i]);
    if (!a.mask[(size_t)unit * plane + i]) total = czero();
    a.out[(size_t)unit * plane + i] = total;
  }
}

// order-3 inner accumulation into the four pair spectra of each outer node
// (_order3.py:240-259); the eta_t max feeds its floor in the outer stage.
// One block takes ACC_TILE bins of one unit for all of its outer nodes
// (AccArgs::nsub of them).  The node responses sinh(sqrt(A) tau)/sqrt(A) and
// cosh(sqrt(A) tau) depend on the unit, the inner node and the bin only, so
// each is evaluated once per block into shared memory; the block's threads
// then accumulate the (outer node, bin) items from there.
__global__ void __launch_bounds__(256, 4) acc_inner_kernel(AccArgs a) {
  const int unit = blockIdx.y;
  const int J = a.nsub, I = a.nnodes;
  const int plane = a.box.w * a.box.h;
  const UnitScalars& u = a.us[unit];
  __shared__ double s_tau[MAX_RANK], s_coef[MAX_RANK];
  __shared__ double s_sh[MAX_RANK][ACC_TILE], s_ch[MAX_RANK][ACC_TILE];
  if (threadIdx.x < I) {
    const double x = a.nodes[threadIdx.x], w = a.weights[threadIdx.x];
    const double tau = x / u.lam2;
    s_tau[threadIdx.x] = tau;
    s_coef[threadIdx.x] = w * exp(x) / u.lam2 * exp(-2.0 * u.shift2 * tau) / 4.0;
  }
  const int ntiles = (plane + ACC_TILE - 1) / ACC_TILE;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int i0 = tile * ACC_TILE;
    __syncthreads();  // s_tau written, the previous tile's responses read
    for (int w = threadIdx.x; w < I * ACC_TILE; w += blockDim.x) {
      const int ii = w / ACC_TILE, b = w % ACC_TILE;
      if (i0 + b < plane) {
        const double sqa = a.geo[5 * plane + i0 + b];
        s_sh[ii][b] = sinh_over_root(sqa, s_tau[ii]);
        s_ch[ii][b] = cosh(sqa * s_tau[ii]);
      }
    }
    __syncthreads();
    for (int w = threadIdx.x; w < J * ACC_TILE; w += blockDim.x) {
      const int j = w / ACC_TILE, b = w % ACC_TILE;
      const int i = i0 + b;
      const int uj = unit * J + j;
      double local = 0.0;
      if (i < plane && !a.mask[(size_t)unit * plane + i]) {
        // off the pair support the four spectra are zero: no loads, no sums
        cplx* dst = a.out + (size_t)uj * 4 * plane;
        dst[i] = czero();
        dst[plane + i] = czero();
        dst[2 * plane + i] = czero();
        dst[3 * plane + i] = czero();
      } else if (i < plane) {
        const double ga = a.geo[4 * plane + i];
        cplx e = czero(), et = czero(), p = czero(), pt = czero();
        for (int ii = 0; ii < I; ++ii) {
          const int js = uj * I + ii;
          const double coef = s_coef[ii];
          const double sh = s_sh[ii][b];
          const double ch = s_ch[ii][b];
          const cplx* src = a.in + (size_t)js * 4 * plane;
          cplx sd = floored(src[i], a.floor_rel, a.maxin[js * 4 + 0]);
          cplx sk = floored(src[plane + i], a.floor_rel, a.maxin[js * 4 + 1]);
          cplx sdt = floored(src[2 * plane + i], a.floor_rel, a.maxin[js * 4 + 2]);
          cplx skt = floored(src[3 * plane + i], a.floor_rel, a.maxin[js * 4 + 3]);
          const double mash = -ga * sh;
          e = cadd(e, cscale(coef, cadd(cscale(mash, sd), cscale(ch, sk))));
          et = csub(et, cmul(cmk(0.0, coef), cadd(cscale(mash, sdt), cscale(ch, skt))));
          p = cadd(p, cmul(cmk(0.0, coef), csub(cscale(ch, sd), cscale(sh, sk))));
          pt = cadd(pt, cscale(coef, csub(cscale(ch, sdt), cscale(sh, skt))));
        }
        cplx* dst = a.out + (size_t)uj * 4 * plane;
        dst[i] = e;
        dst[plane + i] = et;
        dst[2 * plane + i] = p;
        dst[3 * plane + i] = pt;
        local = keep_max_abs(0.0, et);
      }
      // whole warps take this loop's iterations together (blockDim.x and
      // J * ACC_TILE are multiples of 32), and a warp's items share uj
      for (int o = 16; o > 0; o >>= 1) {
        const double other = __shfl_xor_sync(0xffffffffu, local, o);
        local = (other > local || other != other) ? other : local;
      }
      if ((threadIdx.x & 31) == 0) atomic_max_nonneg(a.maxout + uj, local);
    }
  }
}

// The order-3 outer forcings of one (unit, outer node) at bin i: the four
// forcing spectra fk, fd, c, c_t with their roundoff floors, and the psi
// forcings fk + A c and fd - c_t (_order3.py:103-122).  Written with explicit
// fused multiply-adds so that the two kernels that form them (the maxima and
// the accumulation) round them identically.
struct OuterForcing {
  cplx fk, fd, kpsi, dpsi;
};

// From the four spectra's values v[0..3] = fk, fd, c, c_t at the bin.
GL_D OuterForcing outer_forcing_of(const cplx* v, double ga, double floor_rel,
                                   const unsigned long long* mx) {
  OuterForcing o;
  o.fk = floored(v[0], floor_rel, mx[0]);
  o.fd = floored(v[1], floor_rel, mx[1]);
  const cplx c = floored(v[2], floor_rel, mx[2]);
  const cplx ct = floored(v[3], floor_rel, mx[3]);
  o.kpsi = cmk(__fma_rn(ga, c.x, o.fk.x), __fma_rn(ga, c.y, o.fk.y));
  o.dpsi = csub(o.fd, ct);
  return o;
}

GL_D OuterForcing outer_forcing(const cplx* src, int plane, int i, double ga, double floor_rel,
                                const unsigned long long* mx) {
  const cplx v[4] = {src[i], src[plane + i], src[2 * plane + i], src[3 * plane + i]};
  return outer_forcing_of(v, ga, floor_rel, mx);
}

// order-3 outer forcing maxima: the maxima of |fk + A c| and |fd - c_t| over
// the box, which set those forcings' own roundoff floors.  The forcings
// themselves are formed again by acc_outer_kernel from the same spectra, so
// they never travel through memory.  Each thread takes two bins per
// iteration with all ten loads issued first (the kernel is a pure stream of
// four planes); the launch keeps the grid small (48 blocks per unit and
// outer node) so that few blocks share each maximum's atomic slot.
__global__ void acc_outer_max_kernel(AccArgs a) {
  const int uj = blockIdx.y;
  const int plane = a.box.w * a.box.h;
  const cplx* src = a.in + (size_t)uj * 4 * plane;
  const unsigned long long* mx = a.maxin + uj * 4;
  double l0 = 0.0, l1 = 0.0;
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < plane; i += 2 * stride) {
    const bool two = i + stride < plane;
    const int i2 = two ? i + stride : i;
    cplx v[8];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      v[k] = __ldg(src + (size_t)k * plane + i);
      v[4 + k] = __ldg(src + (size_t)k * plane + i2);
    }
    const double ga0 = __ldg(a.geo + 4 * plane + i), ga1 = __ldg(a.geo + 4 * plane + i2);
    // both forcings vanish off the triple support (their inputs were masked)
    const OuterForcing o0 = outer_forcing_of(v, ga0, a.floor_rel, mx);
    l0 = keep_max_abs(l0, o0.kpsi);
    l1 = keep_max_abs(l1, o0.dpsi);
    if (two) {
      const OuterForcing o1 = outer_forcing_of(v + 4, ga1, a.floor_rel, mx);
      l0 = keep_max_abs(l0, o1.kpsi);
      l1 = keep_max_abs(l1, o1.dpsi);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double o0 = __shfl_xor_sync(0xffffffffu, l0, o);
    const double o1 = __shfl_xor_sync(0xffffffffu, l1, o);
    l0 = (o0 > l0 || o0 != o0) ? o0 : l0;
    l1 = (o1 > l1 || o1 != o1) ? o1 : l1;
  }
  if ((threadIdx.x & 31) == 0) {
    atomic_max_nonneg(a.maxout + uj * 2 + 0, l0);
    atomic_max_nonneg(a.maxout + uj * 2 + 1, l1);
  }
}

// order-3 outer accumulation into eta33 / psi33 spectra (_order3.py:124-138):
// `in` holds the four forcing spectra of each outer node, `maxin` their
// maxima and `maxpsi` the psi forcings' maxima (acc_outer_max_kernel).
__global__ void acc_outer_kernel(AccArgs a, const unsigned long long* maxpsi) {
  const int unit = blockIdx.y;
  const int plane = a.box.w * a.box.h;
  const UnitScalars& u = a.us[unit];
  __shared__ double s_tau[MAX_RANK], s_coef[MAX_RANK];
  if (threadIdx.x < a.nnodes) {
    const double x = a.nodes[threadIdx.x], w = a.weights[threadIdx.x];
    const double tau = x / u.lam3;
    s_tau[threadIdx.x] = tau;
    s_coef[threadIdx.x] = w * exp(x) / u.lam3 * exp(-3.0 * u.shift3 * tau);
  }
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < plane; i += gridDim.x * blockDim.x) {
    // off the triple support the output is zero: the bin skips its loads
    // and node responses
    if (!a.mask[(size_t)unit * plane + i]) {
      a.out[((size_t)unit * 2 + 0) * plane + i] = czero();
      a.out[((size_t)unit * 2 + 1) * plane + i] = czero();
      continue;
    }
    BinGeo g = load_geo(a.geo, plane, i);
    cplx eta = czero(), psi = czero();
    for (int j = 0; j < a.nnodes; ++j) {
      const int uj = unit * a.nnodes + j;
      const double tau = s_tau[j];
      const double sh = sinh_over_root(g.sqa, tau);
      const double ch = cosh(g.sqa * tau);
      const double coef = s_coef[j];
      const OuterForcing o = outer_forcing(a.in + (size_t)uj * 4 * plane, plane, i, g.a,
                                           a.floor_rel, a.maxin + uj * 4);
      const cplx kpsi = floored(o.kpsi, a.floor_rel, maxpsi[uj * 2 + 0]);
      const cplx dpsi = floored(o.dpsi, a.floor_rel, maxpsi[uj * 2 + 1]);
      cplx te = csub(cscale(g.a * sh, o.fd), cmul(cmk(0.0, ch), o.fk));
      cplx tp = csub(cmul(cmk(0.0, -ch), dpsi), cscale(sh, kpsi));
      eta = cadd(eta, cscale(coef, te));
      psi = cadd(psi, cscale(coef, tp));
    }
    a.out[((size_t)unit * 2 + 0) * plane + i] = eta;
    a.out[((size_t)unit * 2 + 1) * plane + i] = psi;
  }
}
#endif  // GL_TRANSFORM_TU

// ---------------------------------------------------------------------------
// final inverse FFT along x on the reference grid
// ---------------------------------------------------------------------------

struct OutArgs {
  const cplx* in;       // [uc][w][ny]  (column-transformed box spectra)
  int w, x0;            // box columns
  int nx, log2nx, ny;
  int ncomp;            // components per unit in this launch
  int comp_offset;      // first component slot in the output
  int out_ncomp;        // component slots per unit in the output
  const double* comp_scale;   // physical scale per component of this launch
  double scale_value;   // the scale of every component when comp_scale is null
  void* out;            // [unit][out_ncomp][ny][nx]
  int real_only;        // write float64 real parts instead of complex
  int rows;             // rows per block
  UnitScalars* us;      // non-null: a non-finite output sets the unit's status
};

// Final inverse transform along x on the reference grid: each group of n/16
// threads takes one output row (inputs [uc][y][col], zero outside the box
// columns) and writes scaled complex values or (REAL, OutArgs::real_only)
// real parts; one instantiation per output type keeps one store path per
// kernel.
template <bool REAL, bool B192 = false>
__global__ void __launch_bounds__(B192 ? 192 : 256, 2) out_row_kernel(OutArgs a, const cplx* __restrict__ tw) {
  extern __shared__ __align__(128) cplx smem[];
  __shared__ __align__(8) unsigned long long stage_bar;
  const int n = a.nx;
  const int L = padded_len(n);
  int g, G;
  const FftGroup f = fft_group(n, a.log2nx, g, G);
  const int y0 = blockIdx.x * G;
  const int y = y0 + g;
  const int uc = blockIdx.y;
  const int unit = uc / a.ncomp, comp = uc % a.ncomp;
  const bool active = y < a.ny;
  const int yy = active ? y : 0;
  cplx* buf = smem + (size_t)g * L;
  // Stage the block's input rows (w box columns each) into the front of
  // their groups' row buffers with bulk async copies issued at block start;
  // the first transform pass reads them into registers before the group
  // writes the padded row over them.
  const uint32_t bar = smem_u32(&stage_bar);
  if (threadIdx.x == 0) mbar_init(bar, 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nrows = min(G, a.ny - y0);
    const uint32_t bytes = (uint32_t)(a.w * sizeof(cplx));
    mbar_arrive_expect_tx(bar, bytes * (uint32_t)nrows);
    for (int r = 0; r < nrows; ++r)
      bulk_g2s(smem_u32(smem + (size_t)r * L), a.in + ((size_t)uc * a.ny + y0 + r) * a.w, bytes, bar);
  }
  if (__syncthreads_or(!mbar_wait_bounded(bar, 0, BULK_WAIT_CYCLES))) {
    // a copy never landed: flag the unit, give the copies one more bounded
    // wait so none is left writing this block's shared memory, and leave
    if (threadIdx.x == 0 && a.us) atomicCAS(&a.us[unit].status, 0, (int)GL_ERR_TIMEOUT);
    mbar_wait_bounded(bar, 0, BULK_WAIT_CYCLES);
    return;
  }
  const double s = a.comp_scale ? a.comp_scale[comp] : a.scale_value;
  const size_t base = ((size_t)unit * a.out_ncomp + a.comp_offset + comp) * (size_t)a.ny * n +
                      (size_t)yy * n;
  auto load = [&](int xb) -> cplx {
    const int xi = wrap(xb - a.x0, n);
    return xi < a.w ? buf[xi] : czero();  // staged box row
  };
  bool bad = false;  // the output check of the unit's status, folded into the store
  if constexpr (REAL) {
    double* o = reinterpret_cast<double*>(a.out) + base;
    auto store = [&](int xb, cplx v) {
      const double r = s * v.x;
      bad |= !isfinite(r);
      o[xb] = r;
    };
    fft_row<+1>(buf, f, active, tw, load, store);
  } else {
    cplx* o = reinterpret_cast<cplx*>(a.out) + base;
    auto store = [&](int xb, cplx v) {
      const cplx r = cscale(s, v);
      bad |= !(isfinite(r.x) && isfinite(r.y));
      o[xb] = r;
    };
    fft_row<+1>(buf, f, active, tw, load, store);
  }
  if (a.us) {
    const bool any = __any_sync(0xffffffffu, bad);
    if (any && (threadIdx.x & 31) == 0) atomicCAS(&a.us[unit].status, 0, (int)GL_ERR_NONFINITE);
  }
}

}  // namespace gl
