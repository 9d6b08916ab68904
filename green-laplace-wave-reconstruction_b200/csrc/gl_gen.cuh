// Final transforms on reference grids whose sizes are not powers of two.
//
// The reference takes any even Nx, Ny (python/src/green_laplace/_spectral.py:
// 9-16, src/gl_spectral_surface.m:115-121).  Every product stage of the
// engine runs on its own compact grid (a power of two or 16 m covering the
// stage's box, which may be longer than the reference grid: an alias-free
// product has the same coefficients on any period that covers its box), so
// only the last two transforms -- the inverse transform along y of the kept
// box columns and along x of every row -- run at the reference's Nx and Ny.
// For lengths n = 2^a 3^b 5^c (up to 4096) these kernels run a block-wide
// shared-memory Stockham transform with radix-4, 2, 3 and 5 passes, twiddles
// from a per-length FP64 table W_n^e = exp(-2 pi i e / n) (sincospi at plan
// creation).  Lengths with another prime factor are rejected at plan time.
#pragma once
#include "gl_kernels.cuh"

namespace gl {

constexpr int GEN_MAX_PASSES = 16;

// Radix sequence of a length n = 2^a 3^b 5^c (4s first, then 2, 3, 5).
struct GenPlan {
  int n;
  int np;
  int radix[GEN_MAX_PASSES];
};

inline bool gen_plan(int n, GenPlan& g) {
  g.n = n;
  g.np = 0;
  int r = n;
  const int order[4] = {4, 2, 3, 5};
  for (int q = 0; q < 4; ++q) {
    while (r % order[q] == 0) {
      if (g.np == GEN_MAX_PASSES) return false;
      g.radix[g.np++] = order[q];
      r /= order[q];
    }
  }
  return r == 1 && n >= 2;
}

// One block transforms `cnt` rows of length n held contiguously in `a`
// (ping-pong with `b`), all threads cooperating, __syncthreads between
// passes.  SIGN = +1: inverse (e^{+i}), -1: forward.  `twn` holds W_n^e.
// Returns the buffer that holds the result.
template <int SIGN>
GL_D cplx* gen_fft_block(cplx* a, cplx* b, int cnt, const GenPlan& gp, const cplx* __restrict__ twn) {
  const int n = gp.n;
  int ns = 1;
  for (int p = 0; p < gp.np; ++p) {
    const int R = gp.radix[p];
    const int nb = n / R;
    const int step = n / (ns * R);
    for (int idx = threadIdx.x; idx < cnt * nb; idx += blockDim.x) {
      const int row = idx / nb, j = idx - row * nb;
      const int k = j % ns;
      const cplx* src = a + (size_t)row * n;
      cplx* dst = b + (size_t)row * n;
      cplx v[5];
#pragma unroll
      for (int r = 0; r < 5; ++r) v[r] = r < R ? src[j + r * nb] : czero();
      if (k > 0) {
#pragma unroll
        for (int r = 1; r < 5; ++r)
          if (r < R) v[r] = cmul(v[r], twiddle<SIGN>(twn, (r * k * step) % n));
      }
      switch (R) {
        case 2: dft2<SIGN>(v); break;
        case 3: dft3<SIGN>(v); break;
        case 4: dft4v<SIGN>(v); break;
        default: dft5<SIGN>(v); break;
      }
      const int o = (j - k) * R + k;
#pragma unroll
      for (int r = 0; r < 5; ++r)
        if (r < R) dst[o + r * ns] = v[r];
    }
    __syncthreads();
    cplx* t = a;
    a = b;
    b = t;
    ns *= R;
  }
  return a;
}

// Inverse transform along y of `cw` box columns of one (unit, bank): the box
// rows embedded at their modes (multiplier applied), scaled by `scale`,
// written [job][bank][y][column] like col_ifft_kernel's COL_PLAIN output.
struct GenColArgs {
  int nbanks;
  int mult[4];
  int src_of[4];
  Box box;
  const double* geo;
  const cplx* spec;
  long long spec_job_stride, spec_sub_stride;
  cplx* out;
  GenPlan gp;            // length ny
  const cplx* twn;       // W_ny^e
  double scale;
  int cw;                // columns per block
};

#ifdef GL_TRANSFORM_TU  // launched by gl_launch_cols.cu
__global__ void __launch_bounds__(256) gen_col_kernel(GenColArgs a) {
  extern __shared__ cplx smem[];
  const int n = a.gp.n;
  const int job = blockIdx.y, k = blockIdx.z;
  const int x_first = blockIdx.x * a.cw;
  const int ncol = min(a.cw, a.box.w - x_first);
  const int plane = a.box.w * a.box.h;
  cplx* A = smem;
  cplx* B = smem + (size_t)a.cw * n;
  const cplx* sk = a.spec + (long long)job * a.spec_job_stride + (long long)a.src_of[k] * a.spec_sub_stride;
  for (int t = threadIdx.x; t < a.cw * n; t += blockDim.x) A[t] = czero();
  __syncthreads();
  for (int t = threadIdx.x; t < ncol * a.box.h; t += blockDim.x) {
    const int c = t % ncol, by = t / ncol;
    const int i = by * a.box.w + x_first + c;
    A[(size_t)c * n + wrap_any(a.box.y0 + by, n)] = apply_mult(a.mult[k], GeoRef{a.geo, plane, i}, sk[i]);
  }
  __syncthreads();
  const cplx* res = gen_fft_block<+1>(A, B, a.cw, a.gp, a.twn);
  cplx* dst = a.out + ((size_t)job * a.nbanks + k) * n * a.box.w + x_first;
  for (int t = threadIdx.x; t < ncol * n; t += blockDim.x) {
    const int c = t % ncol, y = t / ncol;
    dst[(size_t)y * a.box.w + c] = cscale(a.scale, res[(size_t)c * n + y]);
  }
}
#endif  // GL_TRANSFORM_TU

// Inverse transform along x of `rows` rows of one (unit, component): the
// column-transformed box columns embedded at their modes, times the
// component's physical scale, written as complex values or real parts, with
// the same non-finite output check as out_row_kernel.
struct GenRowArgs {
  const cplx* in;        // [uc][ny][w]
  int w, x0, ny;
  int ncomp, comp_offset, out_ncomp;
  const double* comp_scale;
  void* out;             // [unit][out_ncomp][ny][nx]
  int real_only;
  int rows;              // rows per block
  UnitScalars* us;
  GenPlan gp;            // length nx
  const cplx* twn;       // W_nx^e
};

#ifdef GL_TRANSFORM_TU  // launched by gl_launch_cols.cu
__global__ void __launch_bounds__(256) gen_row_kernel(GenRowArgs a) {
  extern __shared__ cplx smem[];
  const int n = a.gp.n;
  const int uc = blockIdx.y;
  const int unit = uc / a.ncomp, comp = uc % a.ncomp;
  const int y0 = blockIdx.x * a.rows;
  const int nr = min(a.rows, a.ny - y0);
  cplx* A = smem;
  cplx* B = smem + (size_t)a.rows * n;
  for (int t = threadIdx.x; t < a.rows * n; t += blockDim.x) A[t] = czero();
  __syncthreads();
  for (int t = threadIdx.x; t < nr * a.w; t += blockDim.x) {
    const int r = t / a.w, xi = t % a.w;
    A[(size_t)r * n + wrap_any(a.x0 + xi, n)] = a.in[((size_t)uc * a.ny + y0 + r) * a.w + xi];
  }
  __syncthreads();
  const cplx* res = gen_fft_block<+1>(A, B, a.rows, a.gp, a.twn);
  const double s = a.comp_scale[comp];
  const size_t base = ((size_t)unit * a.out_ncomp + a.comp_offset + comp) * (size_t)a.ny * n + (size_t)y0 * n;
  bool bad = false;
  for (int t = threadIdx.x; t < nr * n; t += blockDim.x) {
    const cplx v = cscale(s, res[t]);
    if (a.real_only) {
      bad |= !isfinite(v.x);
      reinterpret_cast<double*>(a.out)[base + t] = v.x;
    } else {
      bad |= !(isfinite(v.x) && isfinite(v.y));
      reinterpret_cast<cplx*>(a.out)[base + t] = v;
    }
  }
  if (a.us) {
    const bool any = __syncthreads_or(bad);
    if (any && threadIdx.x == 0) atomicCAS(&a.us[unit].status, 0, (int)GL_ERR_NONFINITE);
  }
}
#endif  // GL_TRANSFORM_TU

}  // namespace gl
