// Single-direction time path: the modal GL resolvent of a 1-D record
// (python/src/green_laplace/modal_time.py:217-360) and its difference-
// frequency eta20 (_eta20.py:13-151).
//
// A record's retained DFT bins carry the first-order amplitudes; each bin is
// spread onto a q-axis of P modal nodes, giving a joint (q, frequency-bin)
// spectrum [P][M] (M = the work bins padded to a power of two: the products
// of the graph reach at most order x the band, so a longer period leaves every
// kept bin unchanged).  GL products are taken in the joint (x, t) space; each
// output bin then sums its GL node responses over the q-axis.
//
// Transforms: strided_fft_kernel runs batched power-of-two transforms of up to
// 4096 points along any axis of a row-major array (loads and stores staged
// through shared memory, coalesced along whichever index is contiguous).
// q-axes longer than 4096 use two such passes (four-step: P = P1 P2 with a
// twiddle between the passes); their x-space rows then come out in a
// permuted order, which the pointwise products do not see and the inverse
// pass undoes.
#pragma once
#include "gl_kernels.cuh"

namespace gl {

struct SFft {
  cplx* data;
  int n, log2n;          // transform length (16..4096)
  long long stride;      // element step inside one transform
  long long cstride;     // step between consecutive transforms
  int ncount;            // transforms per outer index
  long long ostride;     // step between outer indices
  double scale;          // applied to the outputs
  int tw_mode;           // 0 none; 1: output k of transform c times w^(k (c / tw_div));
                         // 2: output k of outer index o times w^(k o)
  long long tw_div;
  int tw_log2p;          // w = e^{SIGN 2 pi i / 2^tw_log2p}
};

template <int SIGN>
__global__ void __launch_bounds__(256, 2) strided_fft_kernel(SFft a, const cplx* __restrict__ tw, int cw) {
  extern __shared__ cplx smem[];
  const int o = blockIdx.y;
  const int c0 = blockIdx.x * cw;
  const int nc = min(cw, a.ncount - c0);
  const int n = a.n;
  const int L = padded_len(n);
  cplx* base = a.data + (long long)o * a.ostride + (long long)c0 * a.cstride;
  const bool colwise = a.cstride == 1;  // consecutive transforms adjacent in memory
  for (int t = threadIdx.x; t < n * nc; t += blockDim.x) {
    const int i = colwise ? t / nc : t % n;
    const int c = colwise ? t % nc : t / n;
    smem[(size_t)c * L + phys(i)] = base[(long long)c * a.cstride + (long long)i * a.stride];
  }
  __syncthreads();
  int g, G;
  const FftGroup f = fft_group(n, a.log2n, g, G);
  for (int it = 0; it < (nc + G - 1) / G; ++it) {
    const int c = it * G + g;
    const bool active = c < nc;
    cplx* buf = smem + (size_t)(active ? c : 0) * L;
    auto load = [&](int i) -> cplx { return buf[phys(i)]; };
    auto store = [&](int i, cplx v) { buf[phys(i)] = v; };
    fft_row<SIGN>(buf, f, active, tw, load, store);
  }
  __syncthreads();
  const long long pmask = (1LL << a.tw_log2p) - 1;
  const double pinv = a.tw_mode ? 2.0 / (double)(1LL << a.tw_log2p) : 0.0;
  for (int t = threadIdx.x; t < n * nc; t += blockDim.x) {
    const int k = colwise ? t / nc : t % n;
    const int c = colwise ? t % nc : t / n;
    cplx v = cscale(a.scale, smem[(size_t)c * L + phys(k)]);
    if (a.tw_mode) {
      const long long m = a.tw_mode == 1 ? (long long)(c0 + c) / a.tw_div : (long long)o;
      const long long e = ((long long)k * m) & pmask;
      double sn, cs;
      sincospi((double)SIGN * pinv * (double)e, &sn, &cs);
      v = cmul(v, cmk(cs, sn));
    }
    base[(long long)c * a.cstride + (long long)k * a.stride] = v;
  }
}

// ---------------------------------------------------------------------------
// joint arrays: deposit, bank multipliers, products
// ---------------------------------------------------------------------------

#ifndef GL_TRANSFORM_TU  // elementwise kernels: compiled by gl_engine.cu only
// joint[row][col] = val for idx = row * W + col (distinct indices; the joint
// [rows][M] is zeroed first by the caller).
__global__ void modal_scatter_kernel(const long long* idx, const double* val, int nnz, cplx* joint,
                                     int W, int M) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nnz; t += gridDim.x * blockDim.x) {
    const long long row = idx[t] / W, col = idx[t] % W;
    joint[row * M + col] = cmk(val[2 * t], val[2 * t + 1]);
  }
}

enum ModalMult : int {
  MM_ONE = 0, MM_NU, MM_NU2, MM_Q_SNU, MM_Q, MM_Q2_SNU,           // order-2 banks
  MM_IQ, MM_MI_NU, MM_NU_Q, MM_MI_Q2_SNU, MM_MI_Q2_NU, MM_MINUS_NU2, MM_MINUS_Q2,  // first order
  MM_PAIR_E, MM_PAIR_EX, MM_PAIR_PX, MM_PAIR_PZ, MM_PAIR_PZZ, MM_PAIR_PTZ,        // pair fields
};

struct ModalGeo {
  int P, M, W;           // q nodes, padded bins, work bins
  double q_step;         // q-axis spacing
  double fstep;          // dimensionless frequency of one bin
  int b0;                // first retained bin
};

// signed q of row j in numpy's ifftshift order
GL_D double modal_q(const ModalGeo& g, int j) {
  const int s = (j + g.P / 2) & (g.P - 1);
  return (double)(s - g.P / 2) * g.q_step;
}

// out = src * multiplier(row, column) (evaluation order of modal_time.py:240-246, 302-317)
__global__ void modal_bank_kernel(ModalGeo g, const cplx* src, cplx* out, int mult) {
  const long long total = (long long)g.P * g.M;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(t / g.M), w = (int)(t % g.M);
    const cplx s = src[t];
    const double q = modal_q(g, j);
    const double nu = (g.b0 + w) * g.fstep;
    const double snu = nu > 2.2250738585072014e-308 ? nu : 2.2250738585072014e-308;
    const double qa = fabs(q);
    cplx v;
    switch (mult) {
      case MM_ONE: v = s; break;
      case MM_NU: v = cscale(nu, s); break;
      case MM_NU2: v = cscale(nu * nu, s); break;
      case MM_Q_SNU: v = cscale(q / snu, s); break;
      case MM_Q: v = cscale(q, s); break;
      case MM_Q2_SNU: v = cscale((q * q) / snu, s); break;
      case MM_IQ: v = cmul(s, cmk(0.0, q)); break;
      case MM_MI_NU: v = cmul(s, cmk(0.0, -nu)); break;
      case MM_NU_Q: v = cscale(nu * q, s); break;
      case MM_MI_Q2_SNU: v = cmul(s, cmk(0.0, -(q * q) / snu)); break;
      case MM_MI_Q2_NU: v = cmul(s, cmk(0.0, -(q * q) * nu)); break;
      case MM_MINUS_NU2: v = cscale(-(nu * nu), s); break;
      case MM_MINUS_Q2: v = cscale(-(q * q), s); break;
      // pair spectra: columns are the inner (2 b0 + w) bins, A = |q| tanh |q|
      case MM_PAIR_E: v = s; break;
      case MM_PAIR_EX: v = cmul(s, cmk(0.0, q)); break;
      case MM_PAIR_PX: v = cmul(s, cmk(0.0, q)); break;
      case MM_PAIR_PZ: v = cscale(qa * tanh(qa), s); break;
      case MM_PAIR_PZZ: v = cscale(q * q, s); break;
      case MM_PAIR_PTZ: {
        const double inner = (2 * g.b0 + w) * g.fstep;
        v = cscale(qa * tanh(qa), cmul(s, cmk(0.0, -inner)));
        break;
      }
      default: v = czero();
    }
    out[t] = v;
  }
}

// Order-2 sources in place: a = v, b = vn, c = vn2, d = hx, e = jx, f = radial
// -> c = 2 v vn2 + vn^2 - hx^2, f = 2 v radial + 2 hx jx   (modal_time.py:246-247)
__global__ void modal_sources_kernel(long long total, const cplx* v, const cplx* vn, cplx* vn2,
                                     const cplx* hx, const cplx* jx, cplx* rad) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const cplx a = v[t], b = vn[t], c = vn2[t], d = hx[t], e = jx[t], f = rad[t];
    const cplx a2 = cscale(2.0, a);
    vn2[t] = csub(cadd(cmul(a2, c), cmul(b, b)), cmul(d, d));
    rad[t] = cadd(cmul(a2, f), cmul(cscale(2.0, d), e));
  }
}

struct ModalForcing {
  const cplx *fe, *fex, *fpx, *fpz, *fpxz, *fpzz, *fpzzz, *fptz, *fptzz;  // first order
  const cplx *pe, *pex, *ppx, *ppz, *ppzz, *pptz;                          // pair
  cplx *fk, *fd;
  long long total;
};

// Cubic forcing (modal_time.py:318-336)
__global__ void modal_forcing_kernel(ModalForcing a) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < a.total;
       t += (long long)gridDim.x * blockDim.x) {
    const cplx fe = a.fe[t], fex = a.fex[t], fpx = a.fpx[t], fpz = a.fpz[t], fpxz = a.fpxz[t],
               fpzz = a.fpzz[t], fpzzz = a.fpzzz[t], fptz = a.fptz[t], fptzz = a.fptzz[t];
    const cplx pe = a.pe[t], pex = a.pex[t], ppx = a.ppx[t], ppz = a.ppz[t], ppzz = a.ppzz[t],
               pptz = a.pptz[t];
    const cplx fe2 = cmul(fe, fe);
    const cplx kp = csub(csub(cadd(cmul(fpx, pex), cmul(ppx, fex)), cmul(fe, ppzz)), cmul(pe, fpzz));
    const cplx kd = csub(cmul(cmul(fe, fpxz), fex), cmul(cscale(0.5, fe2), fpzzz));
    const cplx dp = cadd(cadd(cadd(cmul(fe, pptz), cmul(pe, fptz)), cmul(fpx, ppx)), cmul(fpz, ppz));
    const cplx dd = cadd(cmul(cscale(0.5, fe2), fptzz), cmul(fe, cadd(cmul(fpx, fpxz), cmul(fpz, fpzz))));
    a.fk[t] = cadd(cscale(0.25, kd), cscale(0.5, kp));
    a.fd[t] = cadd(cscale(0.25, dd), cscale(0.5, dp));
  }
}

// ---------------------------------------------------------------------------
// GL node responses
// ---------------------------------------------------------------------------

struct ModalResp {
  ModalGeo g;
  const cplx* sd;        // spectra [P][M] (order 2: SD, SK; order 3: FD, FK)
  const cplx* sk;
  cplx* out;             // coefficient per output work bin
  int nbins;             // output work bins
  int mult_b0;           // output bin = mult_b0 * b0 + w
  int kind;              // 2: eta22, 3: eta33
  double scale;          // GL scale of the level
  double depth;
  const double* nodes;
  const double* weights;
  int rank;
};

// S, C of a response at output frequency s for |q| response a (modal_time.py:401-416).
GL_D void modal_node_sums(double s, double ra, double scale, const double* nodes, const double* weights,
                          int rank, double& S, double& C) {
  S = 0.0;
  C = 0.0;
  for (int k = 0; k < rank; ++k) {
    const double x = nodes[k], w = weights[k];
    const double tau = x / scale;
    if (ra > 0.0) {
      const double plus = w / scale * exp(x - (s - ra) * tau);
      const double minus = w / scale * exp(x - (s + ra) * tau);
      S += (plus - minus) / (2.0 * ra);
      C += (plus + minus) / 2.0;
    } else {
      const double b = w / scale * exp(x - s * tau);
      S += b * tau;
      C += b;
    }
  }
}

// One block per output work bin: the q-axis sum of the node responses,
// reduced in a fixed order (modal_time.py:268-279, 339-351).
__global__ void modal_response_kernel(ModalResp a) {
  __shared__ double2 part[256];
  const int w = blockIdx.x;
  const double s = (double)(a.mult_b0 * a.g.b0 + w) * a.g.fstep;
  cplx acc = czero();
  for (int j = threadIdx.x; j < a.g.P; j += blockDim.x) {
    const double qa = fabs(modal_q(a.g, j));
    const double ra = sqrt(qa * tanh(qa));
    if (!(s > ra)) continue;
    const double aq = qa * tanh(qa);
    double S, C;
    modal_node_sums(s, ra, a.scale, a.nodes, a.weights, a.rank, S, C);
    const cplx d = a.sd[(long long)j * a.g.M + w], k = a.sk[(long long)j * a.g.M + w];
    cplx r;
    if (a.kind == 2) {
      r = cadd(cscale(-aq * S, d), cscale(C, k));
      r = cmk(r.x / (4.0 * a.depth), r.y / (4.0 * a.depth));
    } else {
      r = csub(cscale(aq * S, d), cmul(cmk(0.0, C), k));
      const double d2 = a.depth * a.depth;
      r = cmk(r.x / d2, r.y / d2);
    }
    acc = cadd(acc, r);
  }
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) part[threadIdx.x] = cadd(part[threadIdx.x], part[threadIdx.x + h]);
    __syncthreads();
  }
  if (threadIdx.x == 0) a.out[w] = part[0];
}

// Inner pair spectra e2, p2 at every (q, inner bin) (modal_time.py:290-299):
// e2 = (-A S sd + C sk)/4, p2 = i (C sd - S sk)/4 with the lambda2 scale.
__global__ void modal_pair_kernel(ModalResp a, cplx* e2, cplx* p2) {
  const long long total = (long long)a.g.P * a.g.M;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(t / a.g.M), w = (int)(t % a.g.M);
    cplx ev = czero(), pv = czero();
    if (w < a.nbins) {
      const double s = (double)(2 * a.g.b0 + w) * a.g.fstep;
      const double qa = fabs(modal_q(a.g, j));
      const double ra = sqrt(qa * tanh(qa));
      if (s > ra) {
        const double aq = qa * tanh(qa);
        double S, C;
        modal_node_sums(s, ra, a.scale, a.nodes, a.weights, a.rank, S, C);
        const cplx d = a.sd[t], k = a.sk[t];
        ev = cadd(cscale(-aq * S, d), cscale(C, k));
        ev = cmk(ev.x / 4.0, ev.y / 4.0);
        pv = cmuli(csub(cscale(C, d), cscale(S, k)));
        pv = cmk(pv.x / 4.0, pv.y / 4.0);
      }
    }
    e2[t] = ev;
    p2[t] = pv;
  }
}

// ---------------------------------------------------------------------------
// eta20 (difference frequency) on a 2-D modal grid
// ---------------------------------------------------------------------------

struct E20Geo {
  int ny, nx, M;         // grid and padded bins
  double qx_step, qy_step;
  double fstep;
  int b0;
};

GL_D void e20_q(const E20Geo& g, int iy, int ix, double& qx, double& qy) {
  qx = (double)(((ix + g.nx / 2) & (g.nx - 1)) - g.nx / 2) * g.qx_step;
  qy = (double)(((iy + g.ny / 2) & (g.ny - 1)) - g.ny / 2) * g.qy_step;
}

enum E20Mult : int { E20_ONE = 0, E20_NU2, E20_NU, E20_BX, E20_BY, E20_QX, E20_QY, E20_RAD };

__global__ void e20_bank_kernel(E20Geo g, const cplx* src, cplx* out, int mult) {
  const long long total = (long long)g.ny * g.nx * g.M;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int w = (int)(t % g.M);
    const long long r = t / g.M;
    const int ix = (int)(r % g.nx), iy = (int)(r / g.nx);
    double qx, qy;
    e20_q(g, iy, ix, qx, qy);
    const double nu = (g.b0 + w) * g.fstep;
    const double snu = nu > 2.2250738585072014e-308 ? nu : 2.2250738585072014e-308;
    double m = 1.0;
    switch (mult) {
      case E20_ONE: m = 1.0; break;
      case E20_NU2: m = nu * nu; break;
      case E20_NU: m = nu; break;
      case E20_BX: m = qx / snu; break;
      case E20_BY: m = qy / snu; break;
      case E20_QX: m = qx; break;
      case E20_QY: m = qy; break;
      case E20_RAD: m = (qx * qx + qy * qy) / snu; break;
    }
    out[t] = cscale(m, src[t]);
  }
}

struct E20Forcing {
  const cplx *one, *dno, *nuf, *bx, *by, *qxf, *qyf, *rad;
  cplx *fd, *fk;
  long long total;
};

// Difference-frequency forcing with conjugates (_eta20.py:77-92)
__global__ void e20_forcing_kernel(E20Forcing a) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < a.total;
       t += (long long)gridDim.x * blockDim.x) {
    const cplx one = a.one[t], dno = a.dno[t], nuf = a.nuf[t], bx = a.bx[t], by = a.by[t],
               qxf = a.qxf[t], qyf = a.qyf[t], rad = a.rad[t];
    // -dno conj(one) - one conj(dno) + nuf conj(nuf) + bx conj(bx) + by conj(by)
    cplx d = cmul(cmk(-dno.x, -dno.y), cconj(one));
    d = csub(d, cmul(one, cconj(dno)));
    d = cadd(d, cmul(nuf, cconj(nuf)));
    d = cadd(d, cmul(bx, cconj(bx)));
    d = cadd(d, cmul(by, cconj(by)));
    // i rad conj(one) - i bx conj(qx) - i by conj(qy) + i qx conj(bx) + i qy conj(by) - i one conj(rad)
    cplx k = cmul(cmuli(rad), cconj(one));
    k = csub(k, cmul(cmuli(bx), cconj(qxf)));
    k = csub(k, cmul(cmuli(by), cconj(qyf)));
    k = cadd(k, cmul(cmuli(qxf), cconj(bx)));
    k = cadd(k, cmul(cmuli(qyf), cconj(by)));
    k = csub(k, cmul(cmuli(one), cconj(rad)));
    a.fd[t] = d;
    a.fk[t] = k;
  }
}

struct E20Resp {
  E20Geo g;
  const cplx* fd;        // spectra [ny][nx][M]
  const cplx* fk;
  cplx* out;             // coefficient per signed bin (index k: bins 0..span, -span..-1)
  int span;
  double dq, depth;
  const double* nodes;
  const double* weights;
  int rank;
};

// One block per signed bin: the grid sum of the eta20 node responses
// (_eta20.py:120-143), reduced in a fixed order.
__global__ void e20_response_kernel(E20Resp a) {
  __shared__ double2 part[256];
  const int k = blockIdx.x;
  const int sb = k <= a.span ? k : k - (2 * a.span + 1);
  const int col = sb >= 0 ? sb : sb + a.g.M;  // padded-period index of the signed bin
  const double sig = sb * a.g.fstep;
  cplx acc = czero();
  const int cells = a.g.ny * a.g.nx;
  for (int c = threadIdx.x; c < cells; c += blockDim.x) {
    const int iy = c / a.g.nx, ix = c % a.g.nx;
    double qx, qy;
    e20_q(a.g, iy, ix, qx, qy);
    const double q = hypot(qx, qy);
    const double ra = sqrt(q * tanh(q));
    if (!(q > 0.0 && ra > fabs(sig))) continue;
    double md = 0.0, mk = 0.0;
    for (int n = 0; n < a.rank; ++n) {
      const double x = a.nodes[n], w = a.weights[n];
      const double tau = x / a.dq;
      const double plus = w / a.dq * exp(x - (ra - sig) * tau);
      const double minus = w / a.dq * exp(x - (ra + sig) * tau);
      md -= ra * (plus + minus) / 4.0;
      mk += (plus - minus) / 4.0;
    }
    const long long idx = (long long)c * a.g.M + col;
    const cplx r = cadd(cscale(md, a.fd[idx]), cmul(cmk(0.0, mk), a.fk[idx]));
    acc = cadd(acc, cmk(r.x / (2.0 * a.depth), r.y / (2.0 * a.depth)));
  }
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) part[threadIdx.x] = cadd(part[threadIdx.x], part[threadIdx.x + h]);
    __syncthreads();
  }
  if (threadIdx.x == 0) a.out[k] = part[0];
}

// ---------------------------------------------------------------------------
// time-series synthesis: out[n] = sum_b c_b e^{-2 pi i bin_b n / count}
// ---------------------------------------------------------------------------

__global__ void series_synth_kernel(const int* bins, const cplx* coef, int nb, int count, void* out,
                                    int real_only) {
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < count; n += gridDim.x * blockDim.x) {
    cplx acc = czero();
    for (int b = 0; b < nb; ++b) {
      const long long e = ((long long)bins[b] * n) % count;  // exact argument reduction
      double sn, cs;
      sincospi(-2.0 * (double)e / (double)count, &sn, &cs);
      acc = cadd(acc, cmul(coef[b], cmk(cs, sn)));
    }
    if (real_only)
      reinterpret_cast<double*>(out)[n] = acc.x;
    else
      reinterpret_cast<cplx*>(out)[n] = acc;
  }
}
#endif  // GL_TRANSFORM_TU

}  // namespace gl
