// Accumulation kernels of the fourth-order GL eta44 graph
// (paper/order4/cpp/gl_eta44_fftw.cpp).  One GL rule of rank R serves the
// three nested levels: outer4 node o, third node t, pair node p.
//
// Job numbering per unit:
//   pair jobs      (o, t, p) -> (o R + t) R + p            for third-level pairs,
//                  (o, p)    -> R^3 + o R + p              for order-4 pairs;
//   pair groups    g = o R + t (third) or R^2 + o (order 4); group g's
//                  jobs are g R + p, p = 0..R-1;
//   third jobs     (o, t) -> o R + t;   outer jobs o.
#pragma once
#include "gl_kernels.cuh"

namespace gl {

struct E44Acc {
  const UnitScalars* us;
  const double* geo;        // geometry planes of the output box
  Box box;
  const cplx* in;
  const unsigned long long* maxin;
  cplx* out;
  unsigned long long* maxout;
  const double* nodes;
  const double* weights;
  int R;
  int groups_per_unit;      // pair stage: Ro R + Ro; third stage: Ro
  int jobs_per_unit;        // pair stage: Ro R^2 + Ro R
  int Ro, outer0;           // outer nodes handled by this call, first one
  double floor_rel;
  int nspec;                // third stage: spectra written (3, or 4 with eta_t);
                            // order 4: forcing rows read (2, or 4 with the contact rows)
  int only_t1;              // third stage: 0 every third-level node, t + 1 node t alone
};

GL_D void e44_max_reduce(double* v, int n, unsigned long long* slots) {
  for (int k = 0; k < n; ++k) {
    double l = v[k];
    for (int o = 16; o > 0; o >>= 1) {
      const double other = __shfl_xor_sync(0xffffffffu, l, o);
      l = (other > l || other != other) ? other : l;
    }
    if ((threadIdx.x & 31) == 0) atomic_max_nonneg(slots + k, l);
  }
}

GL_D double e44_keep_max(double cur, cplx v) { return keep_max_abs(cur, v); }

// Pair level: the five pair spectra of one group (gl_eta44_fftw.cpp:383-402).
__global__ void acc_e44_pair_kernel(E44Acc a) {
  const int grp = blockIdx.y;                 // unit * groups + g
  const int unit = grp / a.groups_per_unit;
  const int g = grp % a.groups_per_unit;
  const int R = a.R;
  const int jobs_per_unit = a.jobs_per_unit;
  const int plane = a.box.w * a.box.h;
  const UnitScalars& u = a.us[unit];
  double lm[5] = {0, 0, 0, 0, 0};
  __shared__ double s_t[MAX_RANK], s_co[MAX_RANK];
  if (threadIdx.x < R) {
    const double x = a.nodes[threadIdx.x], w = a.weights[threadIdx.x];
    const double t = x / u.lam2;
    s_t[threadIdx.x] = t;
    s_co[threadIdx.x] = w * exp(x) / u.lam2 * exp(-2.0 * u.shift2 * t) / 4.0;
  }
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < plane; i += gridDim.x * blockDim.x) {
    const GeoRef G{a.geo, plane, i};
    const double A = G.a(), sqa = __ldg(a.geo + 5 * plane + i);
    cplx es = czero(), ets = czero(), ps = czero(), pts = czero(), ptts = czero();
    for (int p = 0; p < R; ++p) {
      const int job = unit * jobs_per_unit + g * R + p;
      const double t = s_t[p];
      const double co = s_co[p];
      const double sh = sinh_over_root(sqa, t), ch = cosh(sqa * t);
      const cplx* src = a.in + (size_t)job * 6 * plane;
      cplx s[6];
      for (int k = 0; k < 6; ++k) s[k] = floored(src[(size_t)k * plane + i], a.floor_rel, a.maxin[job * 6 + k]);
      const double mash = -A * sh;
      es = cadd(es, cscale(co, cadd(cscale(mash, s[0]), cscale(ch, s[1]))));
      ets = csub(ets, cmul(cmk(0.0, co), cadd(cscale(mash, s[2]), cscale(ch, s[3]))));
      ps = cadd(ps, cmul(cmk(0.0, co), csub(cscale(ch, s[0]), cscale(sh, s[1]))));
      pts = cadd(pts, cscale(co, csub(cscale(ch, s[2]), cscale(sh, s[3]))));
      ptts = csub(ptts, cmul(cmk(0.0, co), csub(cscale(ch, s[4]), cscale(sh, s[5]))));
    }
    cplx* dst = a.out + (size_t)grp * 5 * plane;
    const cplx r[5] = {es, ets, ps, pts, ptts};
    for (int k = 0; k < 5; ++k) {
      dst[(size_t)k * plane + i] = r[k];
      lm[k] = e44_keep_max(lm[k], r[k]);
    }
  }
  e44_max_reduce(lm, 5, a.maxout + (size_t)grp * 5);
}

// Third level: es, ps, pts of one outer node (gl_eta44_fftw.cpp:571-584);
// with nspec = 4 also ets, the third-order eta_t the psi44 contact needs
// (finite_depth_directional_nested_green_laplace_eta33.m:127-131).
__global__ void acc_e44_third_kernel(E44Acc a) {
  const int uo = blockIdx.y;  // unit * Ro + local outer node
  const int unit = uo / a.Ro;
  const int R = a.R;
  const int plane = a.box.w * a.box.h;
  const UnitScalars& u = a.us[unit];
  const int ns = a.nspec;
  double lm[4] = {0, 0, 0, 0};
  __shared__ double s_t[MAX_RANK], s_co[MAX_RANK];
  if (threadIdx.x < R) {
    const double x = a.nodes[threadIdx.x], w = a.weights[threadIdx.x];
    const double tt = x / u.lam3;
    s_t[threadIdx.x] = tt;
    s_co[threadIdx.x] = w * exp(x) / u.lam3 * exp(-3.0 * u.shift3 * tt);
  }
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < plane; i += gridDim.x * blockDim.x) {
    const GeoRef G{a.geo, plane, i};
    const double A = G.a(), sqa = __ldg(a.geo + 5 * plane + i);
    cplx es = czero(), ps = czero(), pts = czero(), ets = czero();
    for (int t = 0; t < R; ++t) {
      if (a.only_t1 && t != a.only_t1 - 1) continue;
      const int job = uo * R + t;
      const double tt = s_t[t];
      const double co = s_co[t];
      const double sh = sinh_over_root(sqa, tt), ch = cosh(sqa * tt);
      const cplx* src = a.in + (size_t)job * 4 * plane;
      cplx s[4];
      for (int k = 0; k < 4; ++k) s[k] = floored(src[(size_t)k * plane + i], a.floor_rel, a.maxin[job * 4 + k]);
      // s = fk, fd, fkt, fdt
      es = cadd(es, cscale(co, csub(cscale(A * sh, s[1]), cmul(cmk(0.0, ch), s[0]))));
      ps = cadd(ps, cscale(co, csub(cmul(cmk(0.0, -ch), s[1]), cscale(sh, s[0]))));
      pts = cadd(pts, cscale(co, csub(cmul(cmk(0.0, -ch), s[3]), cscale(sh, s[2]))));
      if (ns == 4) ets = cadd(ets, cscale(co, csub(cscale(A * sh, s[3]), cmul(cmk(0.0, ch), s[2]))));
    }
    cplx* dst = a.out + (size_t)uo * ns * plane;
    const cplx r[4] = {es, ps, pts, ets};
    for (int k = 0; k < ns; ++k) {
      dst[(size_t)k * plane + i] = r[k];
      lm[k] = e44_keep_max(lm[k], r[k]);
    }
  }
  e44_max_reduce(lm, ns, a.maxout + (size_t)uo * ns);
}

// Order 4: the eta44 spectrum of one unit (gl_eta44_fftw.cpp:736-748); with
// nspec = 4 also psi44 (...eta44_three_kernels.m:93-111): the contact rows
// give the surface forcings fk + A c and fd - c_t and
// psi += coef (-i cosh fd_s - sinh/sqrt(A) fk_s).  Output [unit][1 or 2][plane];
// only eta44 gets a maximum (its final floor), psi44 is masked only.
__global__ void acc_e44_order4_kernel(E44Acc a) {
  const int unit = blockIdx.y;
  const int plane = a.box.w * a.box.h;
  const UnitScalars& u = a.us[unit];
  const int ns = a.nspec;
  const int nout = ns == 4 ? 2 : 1;
  double lm[1] = {0};
  __shared__ double s_t[MAX_RANK], s_co[MAX_RANK];
  if (threadIdx.x < a.Ro) {
    const double x = a.nodes[a.outer0 + threadIdx.x], w = a.weights[a.outer0 + threadIdx.x];
    const double tm = x / u.lam4;
    s_t[threadIdx.x] = tm;
    s_co[threadIdx.x] = w * exp(x) / u.lam4 * exp(-4.0 * u.shift4 * tm);
  }
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < plane; i += gridDim.x * blockDim.x) {
    const GeoRef G{a.geo, plane, i};
    const double A = G.a(), sqa = __ldg(a.geo + 5 * plane + i);
    cplx acc = czero(), psi = czero();
    for (int ol = 0; ol < a.Ro; ++ol) {
      const int job = unit * a.Ro + ol;
      const double tm = s_t[ol];
      const double co = s_co[ol];
      const double sh = sinh_over_root(sqa, tm), ch = cosh(sqa * tm);
      const cplx* src = a.in + (size_t)job * ns * plane;
      const unsigned long long* mx = a.maxin + (size_t)job * ns;
      const cplx fk = floored(src[i], a.floor_rel, mx[0]);
      const cplx fd = floored(src[plane + i], a.floor_rel, mx[1]);
      acc = cadd(acc, cscale(co, csub(cscale(A * sh, fd), cmul(cmk(0.0, ch), fk))));
      if (ns == 4) {
        const cplx c = floored(src[2 * plane + i], a.floor_rel, mx[2]);
        const cplx ct = floored(src[3 * plane + i], a.floor_rel, mx[3]);
        const cplx fks = cadd(fk, cscale(A, c));
        const cplx fds = csub(fd, ct);
        psi = cadd(psi, cscale(co, csub(cmul(cmk(0.0, -ch), fds), cscale(sh, fks))));
      }
    }
    a.out[(size_t)unit * nout * plane + i] = acc;
    if (nout == 2) a.out[((size_t)unit * nout + 1) * plane + i] = psi;
    lm[0] = e44_keep_max(lm[0], acc);
  }
  e44_max_reduce(lm, 1, a.maxout + (size_t)unit * nout);
}

}  // namespace gl
