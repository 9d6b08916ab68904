// Fourth-order Wave-Interaction-Theory (WIT) direct sum over mode quartets.
//
// For every unordered quartet (i <= j <= k <= l) of first-order modes the
// directional fourth-order kernel is evaluated by the degree-ordered
// recursion over the 15 non-empty subsets of the four slots, exactly as the
// reference's FP64 C++ does (paper/order4/cpp/directional_eta4_openmp.cpp,
// DirectionalKernel::evaluate, lines 157-453): first-order states for the
// singletons, then for each subset of degree 2..4 the ordinary kinematic and
// dynamic sources built from the surface Taylor expansion over its set
// partitions, a 2x2 linear solve against the free-surface operator, the
// retained/complement split of near-resonant cubic and quartic outputs, and
// the residual diagnostics.  The result, weighted by 2 a_i a_j a_k a_l over
// the multiset repeat factor, is scattered to the target bin
// (sector 44, lines 690-734).
//
// One thread per quartet (unranked from a linear index through the
// combinatorial number system), FP64 throughout, per-subset state in local
// memory, FP64 atomics into the five output grids.
#pragma once
#include "gl_common.cuh"

namespace gl {

// Set partitions of each subset mask into 1..4 ordered blocks, in the
// reference's enumeration order (assignment codes counted up, slot digits
// least significant first, surjective assignments kept).  Entry = four block
// masks packed one byte each, block 0 holding the potential factor.
__constant__ unsigned int c_wit_parts[160];
__constant__ unsigned char c_wit_off[16][5];
__constant__ unsigned char c_wit_cnt[16][5];

struct WitModel {
  double g, h;
  GL_D double q(double x, double y) const {
    const double m = hypot(x, y);
    return m * tanh(h * m);
  }
  GL_D double omega(double x, double y) const { return sqrt(g * q(x, y)); }
  // vertical derivative factor of order `o` (1, q, |k|^2, |k|^2 q, |k|^4)
  GL_D double zd(double x, double y, int o) const {
    const double m = hypot(x, y);
    const double m2 = m * m;
    switch (o) {
      case 0: return 1.0;
      case 1: return q(x, y);
      case 2: return m2;
      case 3: return m2 * q(x, y);
      default: return m2 * m2;
    }
  }
  // zd from a cached |k| = hypot(x, y) and q(x, y): the same operations
  GL_D double zdc(double m, double qv, int o) const {
    const double m2 = m * m;
    switch (o) {
      case 0: return 1.0;
      case 1: return qv;
      case 2: return m2;
      case 3: return m2 * qv;
      default: return m2 * m2;
    }
  }
  // (eta, psi) response of the free surface to a (kinematic, dynamic) source
  GL_D void solve(cplx s0, cplx s1, double x, double y, double w, cplx& e, cplx& p) const {
    solve_q(s0, s1, q(x, y), w, e, p);
  }
  GL_D void solve_q(cplx s0, cplx s1, double qv, double w, cplx& e, cplx& p) const {
    const double den = w * w - g * qv;
    const cplx a = csub(cmul(cmk(0.0, w), s0), cscale(qv, s1));
    const cplx b = cadd(cscale(g, s0), cmul(cmk(0.0, w), s1));
    e = cmk(a.x / den, a.y / den);
    p = cmk(b.x / den, b.y / den);
  }
  GL_D double g1(double ex, double ey, double px, double py) const {
    return -q(ex + px, ey + py) * q(px, py) + (px * px + py * py) + (ex * px + ey * py);
  }
};

GL_D cplx cdiv_real(cplx a, double d) { return cmk(a.x / d, a.y / d); }

struct WitOut {
  cplx eta, psi, eta_c, psi_c, retained;
  double rho, residual, strict_src;
  int strict_count;
  bool near;
};

struct WitState {
  double kx[16], ky[16], om[16];
  int deg[16], chg[16];
  cplx eta[16], phi[16], psi[16], sh0[16], sh1[16], sv[16], ret[16];
};

GL_D cplx wit_eta_product(const WitState& S, unsigned int part, int count) {
  cplx v = cmk(1.0, 0.0);
  for (int b = 1; b < count; ++b) v = cmul(v, S.eta[(part >> (8 * b)) & 0xFF]);
  return v;
}

__device__ __noinline__ void wit_evaluate(const WitModel& M, const double* pkx, const double* pky,
                                          const int* sign, double thr, WitOut& out) {
  const double fact[5] = {1.0, 1.0, 2.0, 6.0, 24.0};
  WitState S;
  double skx[4], sky[4], som[4];
  for (int s = 0; s < 4; ++s) {
    skx[s] = (double)sign[s] * pkx[s];
    sky[s] = (double)sign[s] * pky[s];
    som[s] = sign[s] * M.omega(pkx[s], pky[s]);
  }
  for (int m = 0; m < 16; ++m) {
    S.kx[m] = 0.0;
    S.ky[m] = 0.0;
    S.om[m] = 0.0;
    S.deg[m] = 0;
    S.chg[m] = 0;
    S.eta[m] = S.phi[m] = S.psi[m] = S.sh0[m] = S.sh1[m] = S.sv[m] = S.ret[m] = czero();
    for (int s = 0; s < 4; ++s) {
      if (m & (1 << s)) {
        S.kx[m] = S.kx[m] + skx[s];
        S.ky[m] = S.ky[m] + sky[s];
        S.om[m] += som[s];
        S.deg[m] += 1;
        S.chg[m] += sign[s];
      }
    }
  }
  // |k| and q of every subset wavenumber, once per quartet (the calls they
  // replace take exactly these arguments, so the values are identical)
  double HK[16], QK[16];
  for (int m = 0; m < 16; ++m) {
    HK[m] = hypot(S.kx[m], S.ky[m]);
    QK[m] = HK[m] * tanh(M.h * HK[m]);
  }
  cplx eff0 = czero(), eff1 = czero(), co0 = czero(), co1 = czero();
  int strict_count = 0;
  double strict_src = 0.0;
  for (int d = 1; d <= 4; ++d) {
    for (int m = 1; m < 16; ++m) {
      if (S.deg[m] != d) continue;
      cplx taylor = czero();
      if (d == 1) {
        S.eta[m] = cmk(0.5, 0.0);
        S.phi[m] = cmk(0.0, -S.om[m] / (2.0 * QK[m]));
        S.psi[m] = S.phi[m];
      } else {
        // ordinary source: horizontal advection and kinetic terms over the
        // two-block partitions, minus the lower vertical / plus lower time terms
        cplx hor = czero(), kin = czero();
        for (int e = 0; e < c_wit_cnt[m][2]; ++e) {
          const unsigned int pt = c_wit_parts[c_wit_off[m][2] + e];
          const int l = pt & 0xFF, r = (pt >> 8) & 0xFF;
          hor = cadd(hor, cmul(cadd(cmul(S.sh0[l], cmk(0.0, S.kx[r])), cmul(S.sh1[l], cmk(0.0, S.ky[r]))),
                               S.eta[r]));
          kin = cadd(kin, cscale(0.5, cadd(cadd(cmul(S.sh0[l], S.sh0[r]), cmul(S.sh1[l], S.sh1[r])),
                                           cmul(S.sv[l], S.sv[r]))));
        }
        cplx lower_v = czero(), lower_t = czero();
        for (int o = 1; o < d; ++o) {
          for (int e = 0; e < c_wit_cnt[m][o + 1]; ++e) {
            const unsigned int pt = c_wit_parts[c_wit_off[m][o + 1] + e];
            const int pm = pt & 0xFF;
            const cplx pe = wit_eta_product(S, pt, o + 1);
            lower_v = cadd(lower_v, cdiv_real(cmul(cscale(M.zdc(HK[pm], QK[pm], o + 1), S.phi[pm]), pe),
                                              fact[o]));
            const double zo = M.zdc(HK[pm], QK[pm], o);
            lower_t = cadd(lower_t, cdiv_real(cmul(cmul(cmk(0.0, -S.om[pm] * zo), S.phi[pm]), pe), fact[o]));
          }
        }
        const cplx ord0 = csub(hor, lower_v);
        const cplx ord1 = cadd(lower_t, kin);
        for (int o = 1; o < d; ++o) {
          for (int e = 0; e < c_wit_cnt[m][o + 1]; ++e) {
            const unsigned int pt = c_wit_parts[c_wit_off[m][o + 1] + e];
            const int pm = pt & 0xFF;
            taylor = cadd(taylor, cdiv_real(cmul(cscale(M.zdc(HK[pm], QK[pm], o), S.phi[pm]),
                                                 wit_eta_product(S, pt, o + 1)), fact[o]));
          }
        }
        const double qm = QK[m];
        const cplx src0 = csub(cmk(-ord0.x, -ord0.y), cscale(qm, taylor));
        const cplx src1 = csub(cmk(-ord1.x, -ord1.y), cmul(cmk(0.0, S.om[m]), taylor));
        const double mag = HK[m];
        const bool strict_zero = mag <= 100.0 * 2.220446049250313e-16 * fmax(mag, 1.0);
        if (strict_zero) {
          S.eta[m] = czero();
          S.psi[m] = czero();
          strict_count += 1;
          strict_src = fmax(strict_src, hypot(cabs_(src0), cabs_(src1)));
        } else if (d == 2 || (d == 3 && abs(S.chg[m]) == 3)) {
          M.solve_q(src0, src1, QK[m], S.om[m], S.eta[m], S.psi[m]);
        } else if (d == 3) {
          const double wo = sqrt(M.g * QK[m]);
          const double ms = sqrt(wo / (2.0 * M.g)), ns = sqrt(M.g / (2.0 * wo));
          const int ts = S.chg[m] > 0 ? 1 : -1;
          const cplx a = cdiv_real(src0, 2.0 * ms);
          const cplx b = cdiv_real(cmul(cmk(0.0, (double)ts), src1), 2.0 * ns);
          S.ret[m] = cadd(a, b);
          const cplx comp = csub(a, b);
          const double den = S.om[m] + ts * wo;
          S.eta[m] = cdiv_real(cmul(cmk(0.0, ms), comp), den);
          S.psi[m] = cdiv_real(cscale(-ts * ns, comp), den);
        } else {
          // quartic: subtract the cubic-retained push, build the coordinate term
          cplx push0 = czero(), push1 = czero();
          for (int sgl = 0; sgl < 4; ++sgl) {
            if (!(m & (1 << sgl))) continue;
            const int cm = m & ~(1 << sgl);
            if (S.ret[cm].x * S.ret[cm].x + S.ret[cm].y * S.ret[cm].y == 0.0) continue;
            // quadratic normal map of (cubic subset, singleton)
            const double ax = S.kx[cm], ay = S.ky[cm], bx = skx[sgl], by = sky[sgl];
            const int sa = S.chg[cm] > 0 ? 1 : -1, sb = sign[sgl];
            const double qa = QK[cm], qb = QK[1 << sgl];  // (ax, ay), (bx, by) of subsets cm, {sgl}
            const double wa = sqrt(M.g * qa), wb = sqrt(M.g * qb);
            const double ma = sqrt(wa / (2.0 * M.g)), na = sqrt(M.g / (2.0 * wa));
            const cplx ea = cmk(ma, 0.0), psa = cmk(0.0, -sa * na);
            const cplx eb = cmk(0.5, 0.0), psb = cmk(0.0, -sb * wb / (2.0 * qb));
            const cplx q0 = cadd(cmul(cscale(M.g1(ax, ay, bx, by), ea), psb), cmul(cscale(M.g1(bx, by, ax, ay), eb), psa));
            const cplx q1 = cmul(cscale((ax * bx + ay * by) + qa * qb, psa), psb);
            cplx pe, pp;
            M.solve(q0, q1, ax + bx, ay + by, sa * wa + sb * wb, pe, pp);
            push0 = cadd(push0, cmul(S.ret[cm], pe));
            push1 = cadd(push1, cmul(S.ret[cm], pp));
          }
          eff0 = csub(src0, push0);
          eff1 = csub(src1, push1);
          co0 = czero();
          co1 = czero();
          for (int sgl = 0; sgl < 4; ++sgl) {
            if (!(m & (1 << sgl))) continue;
            const int cm = m & ~(1 << sgl);
            const int cc = S.chg[cm];
            if (abs(cc) != 1) continue;
            if (cabs_(S.eta[cm]) + cabs_(S.psi[cm]) == 0.0) continue;
            const double cf = sqrt(M.g * QK[cm]);
            const cplx rot = cmul(cmk(0.0, cc * cf / M.g), S.psi[cm]);
            const cplx ae = cscale(0.5, cadd(S.eta[cm], rot));
            const cplx oe = cscale(0.5, csub(S.eta[cm], rot));
            const cplx ap = cmul(cmk(0.0, -M.g * cc / cf), ae);
            const cplx op = cmul(cmk(0.0, M.g * cc / cf), oe);
            const double sq = QK[1 << sgl];
            const cplx se = cmk(0.5, 0.0);
            const cplx sp = cmk(0.0, -sign[sgl] * sqrt(M.g * QK[1 << sgl]) / (2.0 * sq));
            cplx al0 = czero(), al1 = czero();
            for (int pass = 0; pass < 2; ++pass) {
              const double wa = pass == 0 ? cc * cf : -cc * cf;
              const cplx ea = pass == 0 ? ae : oe, pa = pass == 0 ? ap : op;
              const double ax = S.kx[cm], ay = S.ky[cm], bx = skx[sgl], by = sky[sgl];
              const cplx x0 = cadd(cmul(cscale(M.g1(ax, ay, bx, by), ea), sp), cmul(cscale(M.g1(bx, by, ax, ay), se), pa));
              const cplx x1 = cmul(cscale((ax * bx + ay * by) + QK[cm] * sq, pa), sp);
              cplx re = czero(), rp = czero();
              if (hypot(ax + bx, ay + by) != 0.0) M.solve(x0, x1, ax + bx, ay + by, wa + som[sgl], re, rp);
              if (pass == 0) {
                al0 = re;
                al1 = rp;
              } else {
                co0 = cadd(co0, cadd(al0, re));
                co1 = cadd(co1, cadd(al1, rp));
              }
            }
          }
          const double qo = QK[m];
          const double lin = M.g * qo, tem = S.om[m] * S.om[m];
          const double rho = fabs(lin - tem) / fmax(lin + tem, 2.2250738585072014e-308);
          if (rho < thr) {
            const double wo = sqrt(M.g * QK[m]);
            const double ms = sqrt(wo / (2.0 * M.g)), ns = sqrt(M.g / (2.0 * wo));
            const int ts = S.om[m] >= 0.0 ? 1 : -1;
            const cplx a = cdiv_real(eff0, 2.0 * ms);
            const cplx b = cdiv_real(cmul(cmk(0.0, (double)ts), eff1), 2.0 * ns);
            S.ret[m] = cadd(a, b);
            const cplx comp = csub(a, b);
            const double den = S.om[m] + ts * wo;
            S.eta[m] = cdiv_real(cmul(cmk(0.0, ms), comp), den);
            S.psi[m] = cdiv_real(cscale(-ts * ns, comp), den);
          } else {
            M.solve_q(eff0, eff1, QK[m], S.om[m], S.eta[m], S.psi[m]);
          }
        }
        S.phi[m] = csub(S.psi[m], taylor);
      }
      if (d < 4) {
        // surface horizontal gradient and vertical velocity of this subset
        cplx h0 = czero(), h1 = czero(), v = czero();
        for (int o = 0; o < d; ++o) {
          for (int e = 0; e < c_wit_cnt[m][o + 1]; ++e) {
            const unsigned int pt = c_wit_parts[c_wit_off[m][o + 1] + e];
            const int pm = pt & 0xFF;
            const cplx pe = wit_eta_product(S, pt, o + 1);
            const cplx common = cdiv_real(cmul(S.phi[pm], pe), fact[o]);
            const double vert = M.zdc(HK[pm], QK[pm], o);
            h0 = cadd(h0, cmul(cmk(0.0, S.kx[pm] * vert), common));
            h1 = cadd(h1, cmul(cmk(0.0, S.ky[pm] * vert), common));
            v = cadd(v, cdiv_real(cmul(cscale(M.zdc(HK[pm], QK[pm], o + 1), S.phi[pm]), pe), fact[o]));
          }
        }
        S.sh0[m] = h0;
        S.sh1[m] = h1;
        S.sv[m] = v;
      }
    }
  }
  const double qo = QK[15];
  const double lin = M.g * qo, tem = S.om[15] * S.om[15];
  const double rho = fabs(lin - tem) / fmax(lin + tem, 2.2250738585072014e-308);
  cplx er = csub(csub(cmul(cmk(0.0, -S.om[15]), S.eta[15]), cscale(qo, S.psi[15])), eff0);
  cplx pr = csub(cadd(cmul(cmk(0.0, -S.om[15]), S.psi[15]), cscale(M.g, S.eta[15])), eff1);
  if (rho < thr) {
    const double wo = sqrt(M.g * QK[15]);
    const double ms = sqrt(wo / (2.0 * M.g)), ns = sqrt(M.g / (2.0 * wo));
    const int ts = S.om[15] >= 0.0 ? 1 : -1;
    er = cadd(er, cscale(ms, S.ret[15]));
    pr = cadd(pr, cmul(cmk(0.0, -ts * ns), S.ret[15]));
  }
  out.eta = S.eta[15];
  out.psi = S.psi[15];
  out.eta_c = co0;
  out.psi_c = co1;
  out.retained = S.ret[15];
  out.rho = rho;
  out.residual = hypot(cabs_(er), cabs_(pr));
  out.strict_count = strict_count;
  out.strict_src = strict_src;
  out.near = rho < thr;
}

struct WitStats {
  unsigned long long kept, near, strict_zero_output, strict_zero_intermediate;
  unsigned long long max_residual, min_detuning, max_strict_src, pad;
};

struct WitArgs {
  int n_modes;
  const int* modes;         // (mx, my) per mode
  int n_cases;
  const cplx* amp;          // [case][mode]
  int nx, ny;
  double dkx, dky, thr;
  WitModel M;
  cplx* out;                // 5 planes [field][case][ny][nx]
  WitStats* stats;
  unsigned long long q_begin;      // first candidate index of this call
  unsigned long long n_quartets;   // one past the last candidate index of this call
  const unsigned long long* binom;  // binom[r][v] = C(v, r), r = 1..4, v <= n_modes + 3
  int binom_stride;
  int sector;                       // 44, 40 or 42
};

// Largest v with C(v, r) <= q (v in [r-1, hi]).
GL_D int wit_unrank_step(const unsigned long long* row, int hi, unsigned long long q) {
  int lo = 0;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (row[mid] <= q) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Sectors of the fourth-order sum (directional_eta4_openmp.cpp:604-734):
//   44: unordered quartets of + parents, all targets inside the grid;
//   40: unordered + pair x unordered - pair, analytic half-plane targets;
//   42: unordered + triple x one - parent.
__global__ void __launch_bounds__(128) wit44_kernel(WitArgs a) {
  unsigned long long kept = 0, near = 0, szo = 0, szi = 0;
  double max_res = 0.0, min_det = INFINITY, max_src = 0.0;
  const int M = a.n_modes;
  const unsigned long long* b1 = a.binom + 1 * a.binom_stride;
  const unsigned long long* b2 = a.binom + 2 * a.binom_stride;
  const unsigned long long* b3 = a.binom + 3 * a.binom_stride;
  const unsigned long long* b4 = a.binom + 4 * a.binom_stride;
  const unsigned long long pairs = b2[M + 1];  // M (M + 1) / 2
  (void)b1;
  for (unsigned long long qi = a.q_begin + (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
       qi < a.n_quartets; qi += (unsigned long long)gridDim.x * blockDim.x) {
    int idx[4];
    int sign[4] = {1, 1, 1, 1};
    if (a.sector == 44) {
      // combinatorial number system: q = C(d,4) + C(c,3) + C(b,2) + C(a,1),
      // d > c > b > a >= 0; the multiset is (a, b-1, c-2, d-3)
      unsigned long long q = qi;
      const int d4 = wit_unrank_step(b4, M + 2, q);
      q -= b4[d4];
      const int c3 = wit_unrank_step(b3, d4 - 1, q);
      q -= b3[c3];
      const int bb = wit_unrank_step(b2, c3 - 1, q);
      q -= b2[bb];
      idx[0] = (int)q;
      idx[1] = bb - 1;
      idx[2] = c3 - 2;
      idx[3] = d4 - 3;
    } else if (a.sector == 40) {
      unsigned long long qp = qi / pairs, qm = qi % pairs;
      const int pb = wit_unrank_step(b2, M, qp);
      const int mb = wit_unrank_step(b2, M, qm);
      idx[0] = (int)(qp - b2[pb]);
      idx[1] = pb - 1;
      idx[2] = (int)(qm - b2[mb]);
      idx[3] = mb - 1;
      sign[2] = sign[3] = -1;
    } else {
      const unsigned long long qt = qi / M;
      unsigned long long q = qt;
      const int c3 = wit_unrank_step(b3, M + 1, q);
      q -= b3[c3];
      const int bb = wit_unrank_step(b2, c3 - 1, q);
      q -= b2[bb];
      idx[0] = (int)q;
      idx[1] = bb - 1;
      idx[2] = c3 - 2;
      idx[3] = (int)(qi % M);
      sign[3] = -1;
    }
    int tx = 0, ty = 0;
    for (int s = 0; s < 4; ++s) {
      tx += sign[s] * a.modes[2 * idx[s]];
      ty += sign[s] * a.modes[2 * idx[s] + 1];
    }
    if (tx == 0 && ty == 0) {
      ++szo;
      continue;
    }
    if (a.sector == 40 && !(tx > 0 || (tx == 0 && ty > 0))) continue;
    if (abs(tx) >= a.nx / 2 || abs(ty) >= a.ny / 2) continue;
    double pkx[4], pky[4];
    for (int s = 0; s < 4; ++s) {
      pkx[s] = a.modes[2 * idx[s]] * a.dkx;
      pky[s] = a.modes[2 * idx[s] + 1] * a.dky;
    }
    WitOut r;
    wit_evaluate(a.M, pkx, pky, sign, a.thr, r);
    int rep = 1;
    if (a.sector == 44) {
      // multiset repeat factor: product of factorials of run lengths
      int run = 1;
      for (int s = 1; s < 4; ++s) {
        if (idx[s] == idx[s - 1]) {
          ++run;
        } else {
          for (int v = 2; v <= run; ++v) rep *= v;
          run = 1;
        }
      }
      for (int v = 2; v <= run; ++v) rep *= v;
    } else if (a.sector == 40) {
      rep = (1 + (idx[0] == idx[1])) * (1 + (idx[2] == idx[3]));
    } else {
      rep = idx[0] == idx[2] ? 6 : ((idx[0] == idx[1] || idx[1] == idx[2]) ? 2 : 1);
    }
    const int ix = ((tx % a.nx) + a.nx) % a.nx, iy = ((ty % a.ny) + a.ny) % a.ny;  // any even size
    const size_t plane = (size_t)a.nx * a.ny;
    const size_t field = plane * a.n_cases;
    for (int cs = 0; cs < a.n_cases; ++cs) {
      const cplx* amp = a.amp + (size_t)cs * a.n_modes;
      cplx w = cscale(2.0, amp[idx[0]]);
      for (int s = 1; s < 4; ++s) {
        const cplx as = amp[idx[s]];
        w = cmul(w, sign[s] > 0 ? as : cmk(as.x, -as.y));
      }
      w = cdiv_real(w, (double)rep);
      const size_t o = (size_t)cs * plane + (size_t)iy * a.nx + ix;
      const cplx vals[5] = {cmul(w, r.eta), cmul(w, r.psi), cmul(w, r.eta_c), cmul(w, r.psi_c),
                            r.near ? cmul(w, r.retained) : czero()};
      for (int f = 0; f < 5; ++f) {
        double* dst = reinterpret_cast<double*>(a.out + f * field + o);
        atomicAdd(dst, vals[f].x);
        atomicAdd(dst + 1, vals[f].y);
      }
    }
    ++kept;
    near += r.near ? 1 : 0;
    szi += r.strict_count;
    max_res = fmax(max_res, r.residual);
    min_det = fmin(min_det, r.rho);
    max_src = fmax(max_src, r.strict_src);
  }
  for (int o = 16; o > 0; o >>= 1) {
    kept += __shfl_xor_sync(0xffffffffu, kept, o);
    near += __shfl_xor_sync(0xffffffffu, near, o);
    szo += __shfl_xor_sync(0xffffffffu, szo, o);
    szi += __shfl_xor_sync(0xffffffffu, szi, o);
    max_res = fmax(max_res, __shfl_xor_sync(0xffffffffu, max_res, o));
    min_det = fmin(min_det, __shfl_xor_sync(0xffffffffu, min_det, o));
    max_src = fmax(max_src, __shfl_xor_sync(0xffffffffu, max_src, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&a.stats->kept, kept);
    atomicAdd(&a.stats->near, near);
    atomicAdd(&a.stats->strict_zero_output, szo);
    atomicAdd(&a.stats->strict_zero_intermediate, szi);
    atomic_max_nonneg(&a.stats->max_residual, max_res);
    atomicMin(&a.stats->min_detuning, (unsigned long long)__double_as_longlong(min_det));
    atomic_max_nonneg(&a.stats->max_strict_src, max_src);
  }
}

}  // namespace gl
