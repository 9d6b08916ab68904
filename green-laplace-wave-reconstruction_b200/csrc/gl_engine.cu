// Host side of the Green--Laplace engine: plan creation, workspace layout,
// the per-group launch sequence and the C ABI declared in include/gl_engine.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <atomic>
#include <mutex>
#include <initializer_list>

#include "../../include/gl_engine.h"
#include "gl_kernels.cuh"
#include "gl_wit.cuh"
#include "gl_eta44.cuh"
#include "gl_adjoint.cuh"
#include "gl_modal.cuh"
#include "gl_gen.cuh"
#include "gl_host.h"

using namespace gl;

// ---------------------------------------------------------------------------
// error plumbing and launch accounting (declared in gl_host.h)
// ---------------------------------------------------------------------------

static thread_local std::string g_last_error;

namespace gl {

gl_status fail(gl_status s, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return s;
}

std::atomic<unsigned long long> g_launches{0};
std::mutex g_prof_mu;
bool g_prof_on = false;
std::vector<ProfRecord> g_prof;

cudaError_t ensure_smem_attr(const void* kernel, int bytes) {
  static std::mutex mu;
  static std::vector<std::pair<std::pair<int, const void*>, int>> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  for (const auto& d : done)
    if (d.first.first == dev && d.first.second == kernel && d.second >= bytes) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) done.push_back({{dev, kernel}, bytes});
  return e;
}

}  // namespace gl

extern "C" unsigned long long gl_launch_count(void) { return g_launches.load(); }

extern "C" gl_status gl_profile_begin(void) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  for (auto& r : g_prof) {
    cudaEventDestroy(r.start);
    cudaEventDestroy(r.stop);
  }
  g_prof.clear();
  g_prof_on = true;
  return GL_OK;
}

extern "C" gl_status gl_profile_end(gl_kernel_stat* stats, int max_stats, int* n_stats) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  g_prof_on = false;
  std::vector<gl_kernel_stat> agg;
  for (auto& r : g_prof) {
    float ms = 0.f;
    cudaEventSynchronize(r.stop);
    cudaEventElapsedTime(&ms, r.start, r.stop);
    cudaEventDestroy(r.start);
    cudaEventDestroy(r.stop);
    gl_kernel_stat* hit = nullptr;
    for (auto& a : agg)
      if (std::strncmp(a.name, r.name, sizeof a.name) == 0) hit = &a;
    if (!hit) {
      gl_kernel_stat z;
      std::memset(&z, 0, sizeof z);
      std::strncpy(z.name, r.name, sizeof z.name - 1);
      agg.push_back(z);
      hit = &agg.back();
    }
    hit->launches += 1;
    hit->ms_total += ms;
    hit->bytes_total += r.bytes;
  }
  g_prof.clear();
  const int n = std::min<int>((int)agg.size(), std::max(0, max_stats));
  for (int i = 0; i < n && stats; ++i) stats[i] = agg[i];
  if (n_stats) *n_stats = (int)agg.size();
  return GL_OK;
}

// ---------------------------------------------------------------------------
// analysis kernels
// ---------------------------------------------------------------------------

// Geometry planes of a box on the reference grid.  kx follows numpy's
// 2*pi*fftfreq(nx, d=lx/nx) evaluation order (_spectral.py:9-16).
// dk > 0 selects the order-4 convention qx = (depth dk) mx of
// gl_eta44_fftw.cpp:91-93 instead of numpy's fftfreq evaluation.
__global__ void geo_kernel(double* geo, Box box, int nx, int ny, double lx, double ly,
                           double depth, double dk) {
  const int plane = box.w * box.h;
  const double valx = 1.0 / ((double)nx * (lx / (double)nx));
  const double valy = 1.0 / ((double)ny * (ly / (double)ny));
  const double two_pi = 6.283185307179586;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < plane; i += gridDim.x * blockDim.x) {
    const int mx = box.x0 + i % box.w;
    const int my = box.y0 + i / box.w;
    double qx, qy;
    if (dk > 0.0) {
      qx = depth * dk * (double)mx;
      qy = depth * dk * (double)my;
    } else {
      qx = depth * (two_pi * ((double)mx * valx));
      qy = depth * (two_pi * ((double)my * valy));
    }
    const double q = hypot(qx, qy);
    const double a = q * tanh(q);
    geo[i] = qx;
    geo[plane + i] = qy;
    geo[2 * plane + i] = q;
    geo[3 * plane + i] = sqrt(a);
    geo[4 * plane + i] = a;
    geo[5 * plane + i] = sqrt(a);
  }
}

// tw[m] = exp(-2 pi i m/TW_N) for m < TW_N; with count = TW_ALLOC also the
// tables of the mixed lengths n = 16 m after it (W_n^e, e < n).
__global__ void twiddle_kernel(cplx* tw, int count) {
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < count; m += gridDim.x * blockDim.x) {
    int n = TW_N, e = m;
    if (m >= TW_N) {
      const int lens[7] = {48, 80, 96, 144, 160, 192, 240};
      for (int k = 0; k < 7; ++k) {
        const int off = TW_N + mixed_tw_offset(lens[k]);
        if (m >= off && m < off + lens[k]) {
          n = lens[k];
          e = m - off;
        }
      }
    }
    double s, c;
    sincospi(2.0 * (double)e / (double)n, &s, &c);
    tw[m] = cmk(c, -s);
  }
}

// W_n^e = exp(-2 pi i e / n), e < n, for the final transforms of reference
// grids that are not powers of two.
__global__ void gen_twiddle_kernel(cplx* tw, int n) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    double s, c;
    sincospi(2.0 * (double)e / (double)n, &s, &c);
    tw[e] = cmk(c, -s);
  }
}

__global__ void slots_init_kernel(UnitSlots* slots, int n) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n) return;
  UnitSlots s;
  memset(&s, 0, sizeof s);
  s.nu_min = BITS_POS_INF;
  s.peak_flat = ~0ull;
  s.chan_min[0] = s.chan_min[1] = BITS_POS_INF;
  s.pad[0] = BITS_POS_INF;  // q_min
  slots[u] = s;
}

// Full-grid spectra -> box; max |s| over the whole grid; largest |s| outside
// the box (pad[1]) so a support outside the plan is reported.
__global__ void extract_kernel(const cplx* full, cplx* boxv, Box box, int nx, int ny,
                               UnitSlots* slots) {
  const int u = blockIdx.y;
  const size_t plane = (size_t)nx * ny;
  const cplx* s = full + (size_t)u * plane;
  double lmax = 0.0, lout = 0.0;
  for (size_t f = (size_t)blockIdx.x * blockDim.x + threadIdx.x; f < plane;
       f += (size_t)gridDim.x * blockDim.x) {
    const int iy = (int)(f / nx), ix = (int)(f % nx);
    const int mx = ix < nx / 2 ? ix : ix - nx;
    const int my = iy < ny / 2 ? iy : iy - ny;
    const cplx v = s[f];
    const double m = cabs_(v);
    lmax = (m > lmax || m != m) ? m : lmax;
    const int bx = mx - box.x0, by = my - box.y0;
    if (bx >= 0 && bx < box.w && by >= 0 && by < box.h) {
      boxv[(size_t)u * box.w * box.h + by * box.w + bx] = v;
    } else {
      lout = (m > lout || m != m) ? m : lout;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double a = __shfl_xor_sync(0xffffffffu, lmax, o);
    const double b = __shfl_xor_sync(0xffffffffu, lout, o);
    lmax = (a > lmax || a != a) ? a : lmax;
    lout = (b > lout || b != b) ? b : lout;
  }
  if ((threadIdx.x & 31) == 0) {
    atomic_max_nonneg(&slots[u].smax, lmax);
    atomic_max_nonneg(&slots[u].pad[1], lout);
  }
}

__global__ void box_max_kernel(const cplx* boxv, int plane, UnitSlots* slots) {
  const int u = blockIdx.y;
  double lmax = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < plane; i += gridDim.x * blockDim.x) {
    const double m = cabs_(boxv[(size_t)u * plane + i]);
    lmax = (m > lmax || m != m) ? m : lmax;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double a = __shfl_xor_sync(0xffffffffu, lmax, o);
    lmax = (a > lmax || a != a) ? a : lmax;
  }
  if ((threadIdx.x & 31) == 0) atomic_max_nonneg(&slots[u].smax, lmax);
}

// Parent support and its reductions (spatial.py:163-178, _order3.py:33-47).
__global__ void support_kernel(const cplx* boxv, const double* geo, Box box, UnitSlots* slots,
                               unsigned char* s1) {
  const int u = blockIdx.y;
  const int plane = box.w * box.h;
  const double smax = as_double(slots[u].smax);
  const double thr = 1.0e-13 * (smax > 1.0 ? smax : 1.0);
  double numin = INFINITY, numax = 0.0, amax = 0.0, qmin = INFINITY;
  unsigned long long cnt = 0, bad = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < plane; i += gridDim.x * blockDim.x) {
    const cplx v = boxv[(size_t)u * plane + i];
    const double m = cabs_(v);
    if (!(m == m) || m == INFINITY) bad = 1;
    const bool in = m > thr;
    s1[(size_t)u * plane + i] = in ? 1 : 0;
    if (in) {
      const double nu = geo[3 * plane + i];
      const double q = geo[2 * plane + i];
      numin = fmin(numin, nu);
      numax = fmax(numax, nu);
      qmin = fmin(qmin, q);
      const double a2 = m * m;
      amax = fmax(amax, a2);
      ++cnt;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    numin = fmin(numin, __shfl_xor_sync(0xffffffffu, numin, o));
    numax = fmax(numax, __shfl_xor_sync(0xffffffffu, numax, o));
    qmin = fmin(qmin, __shfl_xor_sync(0xffffffffu, qmin, o));
    amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
    cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    bad |= __shfl_xor_sync(0xffffffffu, bad, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (cnt) {
      atomicMin(&slots[u].nu_min, (unsigned long long)__double_as_longlong(numin));
      atomicMin(&slots[u].pad[0], (unsigned long long)__double_as_longlong(qmin));
      atomic_max_nonneg(&slots[u].nu_max, numax);
      atomic_max_nonneg(&slots[u].amp2_max, amax);
      atomicAdd(&slots[u].count, cnt);
    }
    if (bad) atomicOr(&slots[u].nonfinite, 1ull);
  }
}

// First argmax of |s|^2 in reference flat order; radial channel masks and
// their nu ranges (spatial.py:322-337).
__global__ void peak_kernel(const cplx* boxv, const double* geo, Box box, int nx, int ny,
                            UnitSlots* slots, const unsigned char* s1, unsigned char* chan,
                            int want_channels) {
  const int u = blockIdx.y;
  const int plane = box.w * box.h;
  const double amax = as_double(slots[u].amp2_max);
  const double lo = as_double(slots[u].nu_min), hi = as_double(slots[u].nu_max);
  const double step = (hi - lo) / 2.0;
  const double mid = step == 0.0 ? lo : step + lo;
  unsigned long long best = ~0ull;
  double cmin0 = INFINITY, cmax0 = 0.0, cmin1 = INFINITY, cmax1 = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < plane; i += gridDim.x * blockDim.x) {
    const bool in = s1[(size_t)u * plane + i];
    unsigned char c0 = 0, c1 = 0;
    if (in) {
      const double m = cabs_(boxv[(size_t)u * plane + i]);
      if (m * m == amax) {
        const int mx = box.x0 + i % box.w, my = box.y0 + i / box.w;
        const unsigned long long flat =
            (unsigned long long)wrap_any(my, ny) * (unsigned long long)nx + (unsigned long long)wrap_any(mx, nx);
        best = flat < best ? flat : best;
      }
      if (want_channels) {
        const double nu = geo[3 * plane + i];
        if (nu >= lo && nu < mid) {
          c0 = 1;
          cmin0 = fmin(cmin0, nu);
          cmax0 = fmax(cmax0, nu);
        }
        if (nu >= mid && nu <= hi) {
          c1 = 1;
          cmin1 = fmin(cmin1, nu);
          cmax1 = fmax(cmax1, nu);
        }
      }
    }
    if (want_channels) {
      chan[((size_t)u * 2 + 0) * plane + i] = c0;
      chan[((size_t)u * 2 + 1) * plane + i] = c1;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long ob = __shfl_xor_sync(0xffffffffu, best, o);
    best = ob < best ? ob : best;
    cmin0 = fmin(cmin0, __shfl_xor_sync(0xffffffffu, cmin0, o));
    cmax0 = fmax(cmax0, __shfl_xor_sync(0xffffffffu, cmax0, o));
    cmin1 = fmin(cmin1, __shfl_xor_sync(0xffffffffu, cmin1, o));
    cmax1 = fmax(cmax1, __shfl_xor_sync(0xffffffffu, cmax1, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&slots[u].peak_flat, best);
    if (want_channels) {
      if (cmin0 != INFINITY) {
        atomicMin(&slots[u].chan_min[0], (unsigned long long)__double_as_longlong(cmin0));
        atomic_max_nonneg(&slots[u].chan_max[0], cmax0);
      }
      if (cmin1 != INFINITY) {
        atomicMin(&slots[u].chan_min[1], (unsigned long long)__double_as_longlong(cmin1));
        atomic_max_nonneg(&slots[u].chan_max[1], cmax1);
      }
    }
  }
}

// Byte masks [job][h][w] -> forward / reversed bitset rows [job][h][words].
__global__ void bitrows_kernel(const unsigned char* bytes, int h, int w, int words,
                               unsigned long long* fwd, unsigned long long* rev) {
  const int job = blockIdx.y;
  const int total = h * words;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const int row = t / words, wi = t % words;
    const unsigned char* r = bytes + ((size_t)job * h + row) * w;
    unsigned long long f = 0ull, b = 0ull;
    for (int bit = 0; bit < 64; ++bit) {
      const int x = wi * 64 + bit;
      if (x < w) {
        if (r[x]) f |= 1ull << bit;
        if (r[w - 1 - x]) b |= 1ull << bit;
      }
    }
    fwd[((size_t)job * h + row) * words + wi] = f;
    rev[((size_t)job * h + row) * words + wi] = b;
  }
}

// C = A (+) B as byte masks; optional max sqrt(A) over C (geoC planes).
struct MinkArgs {
  const unsigned long long* a;  // fwd rows of A
  int ha, wa, wwa;
  long long a_job_stride;       // words between jobs
  const unsigned long long* brev;
  int hb, wb, wwb;
  long long b_job_stride;
  unsigned char* c;             // [job][hc][wc]
  int hc, wc;
  long long c_job_stride;       // bytes between jobs
  const double* geoc;
  UnitSlots* slots;
  int which;                    // 2: sqa_max2, 3: sqa_max3, 0: none
  int skip_dup;                 // 1: units flagged dup are filled by mink_copy_kernel instead
};

// Dynamic shared memory: 2 (ha + hb) shorts, the column extents of A's and
// B's rows (each block derives them from the bit rows).
__global__ void minkowski_kernel(MinkArgs m) {
  extern __shared__ short ext[];
  const int job = blockIdx.y;
  if (m.skip_dup && m.slots[job].dup) return;
  const unsigned long long* A = m.a + job * m.a_job_stride;
  const unsigned long long* B = m.brev + job * m.b_job_stride;
  unsigned char* C = m.c + job * m.c_job_stride;
  short* aext = ext;
  short* bext = ext + 2 * m.ha;
  for (int r = threadIdx.x; r < m.ha + m.hb; r += blockDim.x) {
    int first, last;
    if (r < m.ha) {
      row_extent(A + (size_t)r * m.wwa, m.wwa, first, last);
      aext[2 * r] = (short)first;
      aext[2 * r + 1] = (short)last;
    } else {
      // reversed rows: bit j is column wb - 1 - j
      const int q = r - m.ha;
      row_extent(B + (size_t)q * m.wwb, m.wwb, first, last);
      const bool empty = last < first;
      bext[2 * q] = empty ? (short)32767 : (short)(m.wb - 1 - last);
      bext[2 * q + 1] = empty ? (short)-32768 : (short)(m.wb - 1 - first);
    }
  }
  __syncthreads();
  const int plane = m.hc * m.wc;
  double lmax = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < plane; i += gridDim.x * blockDim.x) {
    const int ox = i % m.wc, oy = i / m.wc;
    const bool in = minkowski_bin(A, m.ha, m.wa, m.wwa, B, m.hb, m.wb, m.wwb, ox, oy, aext, bext);
    C[i] = in ? 1 : 0;
    if (in && m.geoc) lmax = fmax(lmax, m.geoc[5 * plane + i]);
  }
  if (m.which) {
    for (int o = 16; o > 0; o >>= 1) lmax = fmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
    if ((threadIdx.x & 31) == 0)
      atomic_max_nonneg(m.which == 2 ? &m.slots[job].sqa_max2
                        : m.which == 3 ? &m.slots[job].sqa_max3 : &m.slots[job].pad[2], lmax);
  }
}

// dup = 1 for a unit u >= 1 whose support rows equal unit 0's: then S2 = S+S
// and S3 = S2+S equal unit 0's too (snapshots of one sea state share their
// support), and the Minkowski sums are copied instead of recomputed.
__global__ void support_dup_kernel(const unsigned long long* s1f, long long words, UnitSlots* slots) {
  const int u = blockIdx.x + 1;
  const unsigned long long* a = s1f + (size_t)u * words;
  bool diff = false;
  for (long long t = threadIdx.x; t < words; t += blockDim.x) diff |= a[t] != s1f[t];
  diff = __syncthreads_or(diff);
  if (threadIdx.x == 0) slots[u].dup = diff ? 0ull : 1ull;
}

// The Minkowski sum of unit 0 (mask plane and its sqrt(A) maximum) copied to
// the units flagged dup.
__global__ void mink_copy_kernel(unsigned char* c, long long plane, int which, UnitSlots* slots) {
  const int u = blockIdx.y + 1;
  if (!slots[u].dup) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < plane; i += (long long)gridDim.x * blockDim.x)
    c[(size_t)u * plane + i] = c[i];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (which == 2) slots[u].sqa_max2 = slots[0].sqa_max2;
    if (which == 3) slots[u].sqa_max3 = slots[0].sqa_max3;
  }
}

struct ScalarArgs {
  const UnitSlots* slots;
  UnitScalars* us;
  const double* geo1;
  Box box;
  int nx, ny;
  int order;
  int want_eta22, want_psi22, want_o3;
  int allow_below;
  int full_input;
  int want_e44;
  double fixed_peak;  // > 0: peak depth supplied by the caller (order 4)
};

// Scales, shifts and status per unit (spatial.py:179-189, 246-268;
// _order3.py:35-52).
__global__ void scalars_kernel(ScalarArgs a, int n) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n) return;
  const UnitSlots& s = a.slots[u];
  UnitScalars r;
  memset(&r, 0, sizeof r);
  int status = 0;
  if (s.nonfinite) status = GL_ERR_COMPONENTS;
  if (!status && s.count == 0) status = GL_ERR_EMPTY_SUPPORT;
  const double smax = as_double(s.smax);
  if (!status && a.full_input) {
    const double thr = 1.0e-13 * (smax > 1.0 ? smax : 1.0);
    if (as_double(s.pad[1]) > thr) status = GL_ERR_OUTSIDE_PLAN;
  }
  const double qmin = as_double(s.pad[0]);
  if (!status && a.want_o3 && !(qmin > 0.5)) status = GL_ERR_ORDER3_DOMAIN;
  if (!status && a.want_psi22 && qmin < 0.3 && !a.allow_below) status = GL_ERR_ORDER2_DOMAIN;
  r.nu_min = as_double(s.nu_min);
  r.nu_max = as_double(s.nu_max);
  if (!status) {
    const unsigned long long flat = s.peak_flat;
    const int ix = (int)(flat % (unsigned long long)a.nx), iy = (int)(flat / (unsigned long long)a.nx);
    const int mx = ix < a.nx / 2 ? ix : ix - a.nx;
    const int my = iy < a.ny / 2 ? iy : iy - a.ny;
    const int i = (my - a.box.y0) * a.box.w + (mx - a.box.x0);
    const double qp = a.fixed_peak > 0.0 ? a.fixed_peak : a.geo1[2 * a.box.w * a.box.h + i];
    r.peak_q = qp;
    const double pnu = sqrt(qp * tanh(qp));
    const double sqa2 = as_double(s.sqa_max2);
    r.shift2 = 0.5 * (r.nu_min + sqa2 / 2.0);
    if (a.want_eta22) {
      const double t1 = 2.0 * sqrt(qp * tanh(qp));
      r.lam22 = sqrt(t1 * t1 - 2.0 * qp * tanh(2.0 * qp));
      if (!(r.lam22 > 0.0) || !isfinite(r.lam22)) status = GL_ERR_SCALE;
    }
    if (a.want_psi22) {
      const double pout = sqrt(2.0 * qp * tanh(2.0 * qp));
      r.lam_minus = 2.0 * pnu - pout;
      r.lam_plus = 2.0 * pnu + pout;
      if (!(r.lam_minus > 0.0) || !isfinite(r.lam_minus) || !(r.lam_plus > 0.0) ||
          !isfinite(r.lam_plus))
        status = GL_ERR_SCALE;
      int cc = 0;
      for (int c = 0; c < 2; ++c) {
        if (s.chan_min[c] != BITS_POS_INF) {
          r.chan_id[cc] = c;
          r.chan_shift[cc] = 0.5 * (as_double(s.chan_min[c]) + as_double(s.chan_max[c]));
          ++cc;
        }
      }
      r.chan_count = cc;
      const double step = (r.nu_max - r.nu_min) / 2.0;
      r.edge_mid = step == 0.0 ? r.nu_min : step + r.nu_min;
    }
    if (a.want_o3) {
      const double sqa3 = as_double(s.sqa_max3);
      r.shift3 = 0.5 * (r.nu_min + sqa3 / 3.0);
      r.lam2 = 2.0 * pnu - sqrt(2.0 * qp * tanh(2.0 * qp));
      r.lam3 = 3.0 * pnu - sqrt(3.0 * qp * tanh(3.0 * qp));
      if (!(r.lam2 > 0.0) || !(r.lam3 > 0.0)) status = GL_ERR_SCALE;
    }
    if (a.want_e44) {  // gl_eta44_fftw.cpp:121-128
      const double sqa3 = as_double(s.sqa_max3), sqa4 = as_double(s.pad[2]);
      r.shift3 = 0.5 * (r.nu_min + sqa3 / 3.0);
      r.shift4 = 0.5 * (r.nu_min + sqa4 / 4.0);
      r.lam2 = 2.0 * pnu - sqrt(2.0 * qp * tanh(2.0 * qp));
      r.lam3 = 3.0 * pnu - sqrt(3.0 * qp * tanh(3.0 * qp));
      r.lam4 = 4.0 * pnu - sqrt(4.0 * qp * tanh(4.0 * qp));
      if (!(r.lam2 > 0.0) || !(r.lam3 > 0.0) || !(r.lam4 > 0.0)) status = GL_ERR_SCALE;
    }
  }
  r.status = status;
  a.us[u] = r;
}

// Deposit N^2 (a+ib)/h e^{-i omega t} per bin segment (gl_spectral_surface.m:123-149).
__global__ void deposit_kernel(int n_seg, const int* seg_off, const int* seg_bin,
                               const double* ab, const double* omega, const double* times,
                               double scale, double depth, cplx* out, int plane) {
  const int u = blockIdx.y;
  const double t = times[u];
  for (int sgi = blockIdx.x * blockDim.x + threadIdx.x; sgi < n_seg; sgi += gridDim.x * blockDim.x) {
    cplx acc = czero();
    for (int k = seg_off[sgi]; k < seg_off[sgi + 1]; ++k) {
      const cplx amp = cmk(ab[2 * k] / depth, ab[2 * k + 1] / depth);
      double s, c;
      sincos(omega[k] * t, &s, &c);
      acc = cadd(acc, cmul(cscale(scale, amp), cmk(c, -s)));
    }
    out[(size_t)u * plane + seg_bin[sgi]] = acc;
  }
}

__global__ void status_kernel(const UnitScalars* us, int n, int* out) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u < n && out) out[u] = us[u].status;
}

__global__ void nonfinite_kernel(const void* outp, size_t per_unit, int real_only,
                                 UnitScalars* us) {
  const int u = blockIdx.y;
  unsigned int bad = 0;
  if (real_only) {
    const double* o = reinterpret_cast<const double*>(outp) + (size_t)u * per_unit;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < per_unit;
         i += (size_t)gridDim.x * blockDim.x)
      if (!isfinite(o[i])) bad = 1;
  } else {
    const cplx* o = reinterpret_cast<const cplx*>(outp) + (size_t)u * per_unit;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < per_unit;
         i += (size_t)gridDim.x * blockDim.x)
      if (!isfinite(o[i].x) || !isfinite(o[i].y)) bad = 1;
  }
  bad = __any_sync(0xffffffffu, bad);
  if (bad && (threadIdx.x & 31) == 0) atomicCAS(&us[u].status, 0, (int)GL_ERR_NONFINITE);
}

// ---------------------------------------------------------------------------
// host helpers: Gauss--Laguerre (Golub--Welsch) and dispersion
// ---------------------------------------------------------------------------

// Eigenvalues of the symmetric tridiagonal Jacobi matrix by implicit-shift QL
// iterations, tracking the first row of the eigenvector matrix so that the
// Gauss weights are its squares (Golub & Welsch 1969).
static bool jacobi_eigen(int n, std::vector<double>& d, std::vector<double> e,
                         std::vector<double>& z) {
  z.assign(n, 0.0);
  z[0] = 1.0;
  e.resize(n, 0.0);
  for (int l = 0; l < n; ++l) {
    int iter = 0;
    while (true) {
      int m = l;
      for (; m < n - 1; ++m) {
        const double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
        if (std::fabs(e[m]) <= 1e-300 + 2.220446049250313e-16 * dd) break;
      }
      if (m == l) break;
      if (++iter > 100) return false;
      double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
      double r = std::hypot(g, 1.0);
      g = d[m] - d[l] + e[l] / (g + (g >= 0 ? r : -r));
      double s = 1.0, c = 1.0, p = 0.0;
      int i = m - 1;
      bool underflow = false;
      for (; i >= l; --i) {
        double f = s * e[i], b = c * e[i];
        r = std::hypot(f, g);
        e[i + 1] = r;
        if (r == 0.0) {
          d[i + 1] -= p;
          e[m] = 0.0;
          underflow = true;
          break;
        }
        s = f / r;
        c = g / r;
        g = d[i + 1] - p;
        r = (d[i] - g) * s + 2.0 * c * b;
        p = s * r;
        d[i + 1] = g + p;
        g = c * r - b;
        const double zf = z[i + 1];
        z[i + 1] = s * z[i] + c * zf;
        z[i] = c * z[i] - s * zf;
      }
      if (underflow) continue;
      d[l] -= p;
      e[l] = g;
      e[m] = 0.0;
    }
  }
  return true;
}

static gl_status gauss_laguerre(int rank, double* nodes, double* weights) {
  if (rank < 1 || rank > MAX_RANK) return fail(GL_ERR_RANK, "rank must be an integer from 1 to %d", MAX_RANK);
  std::vector<double> d(rank), e(rank, 0.0), z;
  for (int i = 0; i < rank; ++i) d[i] = 2.0 * (i + 1) - 1.0;
  for (int i = 0; i + 1 < rank; ++i) e[i] = (double)(i + 1);
  if (!jacobi_eigen(rank, d, e, z)) return fail(GL_ERR_RANK, "Golub-Welsch iteration did not converge");
  std::vector<int> idx(rank);
  for (int i = 0; i < rank; ++i) idx[i] = i;
  std::sort(idx.begin(), idx.end(), [&](int a, int b) { return d[a] < d[b]; });
  for (int i = 0; i < rank; ++i) {
    nodes[i] = d[idx[i]];
    weights[i] = z[idx[i]] * z[idx[i]];
  }
  // moment gate: sum w x^k = k! for k < 2 rank (quadrature.py:23-30)
  double fact = 1.0;
  for (int deg = 0; deg < 2 * rank; ++deg) {
    if (deg > 0) fact *= deg;
    long double sum = 0.0L;
    for (int i = 0; i < rank; ++i) sum += (long double)weights[i] * powl((long double)nodes[i], deg);
    const double rel = std::fabs((double)sum - fact) / std::max(1.0, fact);
    if (rel > 3.0e-11)
      return fail(GL_ERR_RANK, "Gauss--Laguerre moment check failed at rank=%d, degree=%d", rank, deg);
  }
  return GL_OK;
}

// ---------------------------------------------------------------------------
// plan
// ---------------------------------------------------------------------------

struct gl_plan {
  gl_plan_desc d;
  int comps;                    // GL_COMP_* actually produced
  int ncomp;
  int comp_ids[6];
  int ncx, ncy, lncx, lncy, lnx, lny;
  // forward column grids of the pair (eta22, psi22, inner order-3) and triple
  // (outer order-3) stages: the smallest column lengths >= the box heights,
  // mixed lengths 16 m allowed (log2 0 for those); ncy (a power of two) is
  // the adjoint's grid and bounds both
  int ncy2, lncy2, ncy3, lncy3;
  // forward row length of the pair stages (power of two or 144/160/192/240,
  // <= ncx: their products need a period covering only the pair box)
  int ncx2, lncx2;
  int ncx3 = 0;  // eta44 third-level row length (power of two covering B3)
  Box b1, b2, b3;
  int ww1, ww2;                 // bitset words per row (S1, S2)
  bool want_eta22, want_psi22, want_o3, want_first;
  double* geo1 = nullptr;
  double* geo2 = nullptr;
  double* geo3 = nullptr;
  cplx* tw = nullptr;
  double* nodes = nullptr;      // device: [eta22 | psi22 | inner | outer] nodes then weights
  double h_nodes[4][MAX_RANK], h_weights[4][MAX_RANK];
  int ranks[4];
  double* comp_scale = nullptr; // device: physical scale per output component
  double h_comp_scale[6];
  double floor_rel;
  int group;
  // workspace layout (byte offsets), for `group` units
  size_t ws_total;
  size_t o_slots, o_us, o_box, o_s1, o_s1f, o_s1r, o_s2, o_s2f, o_s2r, o_s3, o_ch, o_chf, o_chr,
      o_pm, o_out22, o_outp22, o_out33, o_scratch;
  size_t scratch_bytes;
  // fourth-order eta44 plans (gl_eta44_plan_create)
  bool e44 = false;
  bool e44_psi = false;         // psi44 requested with eta44
  int R44 = 0;
  double dk44 = 0.0, peak44 = 0.0;
  Box b4;
  int ww3 = 0;
  double* geo4 = nullptr;
  size_t o_s3f = 0, o_s3r = 0, o_s4 = 0, o_e44 = 0;
  // reference grids that are not powers of two: the final transforms run the
  // generic-length kernels of gl_gen.cuh with these radix plans and tables
  bool gen = false;
  GenPlan genx, geny;
  cplx* twx = nullptr;
  cplx* twy = nullptr;
  // launch shapes picked by a tuner (gl_plan_set_tuning); zeros: built-in choices
  gl_tuning tune = {0, 0, 0};
  // failure-path test hook of the order-2/3 row stages (gl_plan_set_wait_test)
  unsigned int wait_surplus = 0;
  long long wait_cycles = 0;
  // concurrent lanes (gl_plan_set_lanes): `lanes` workspace regions of
  // lane_bytes each, one per stream; lane 0 is the caller's stream, the others
  // are the plan's own streams, forked from and joined back to the caller's
  // stream by events; the mutex keeps one call's fork/join records together
  int device = 0;
  int lanes = 1;
  size_t lane_bytes = 0;
  cudaStream_t lane_st[GL_MAX_LANES] = {};
  cudaEvent_t lane_ev[GL_MAX_LANES] = {};
  std::mutex lane_mu;
};

// Smallest column-transform length >= v: a power of two (>= 16) or one of the
// mixed lengths 16 m the column kernels run.
static int col_len(int v) {
  int best = std::max(16, next_pow2(v));
  const int mixed[7] = {48, 80, 96, 144, 160, 192, 240};
  for (int k = 0; k < 7; ++k)
    if (mixed[k] >= v && mixed[k] < best) best = mixed[k];
  return best;
}
static int col_log2(int n) { return is_pow2(n) ? ilog2(n) : 0; }

// Smallest row-transform length >= v: a power of two (>= 16) or one of the
// mixed lengths the pair-stage row kernels are instantiated for.
static int row_len(int v) {
  int best = std::max(16, next_pow2(v));
  const int mixed[4] = {144, 160, 192, 240};
  for (int k = 0; k < 4; ++k)
    if (mixed[k] >= v && mixed[k] < best) best = mixed[k];
  return best;
}

struct Bump {
  size_t off = 0;
  size_t take(size_t bytes) {
    const size_t o = off;
    off = align_up(off + bytes);
    return o;
  }
};

// Scratch bytes of each stage, for `g` units.
static size_t stage_scratch(const gl_plan* p, int g) {
  const size_t c = sizeof(cplx);
  const size_t b1 = (size_t)p->b1.w * p->b1.h, b2 = (size_t)p->b2.w * p->b2.h,
               b3 = (size_t)p->b3.w * p->b3.h;
  const size_t ncy = p->ncy;
  size_t need = 0;
  auto upd = [&](size_t v) { need = std::max(need, v); };
  if (p->want_eta22) {
    const size_t J = p->ranks[0];
    Bump b;
    b.take(g * J * 8 * p->b1.w * ncy * c);
    b.take(g * J * 2 * p->b2.w * ncy * c);
    b.take(g * J * 2 * b2 * c);
    b.take(g * J * 2 * 8);
    upd(b.off);
  }
  if (p->want_psi22) {
    Bump b;
    b.take((size_t)g * 8 * 8 * p->b1.w * ncy * c);   // P: jobs (g,2,2,2), 8 banks
    b.take((size_t)g * 4 * 8 * p->b2.w * ncy * c);   // Q
    b.take((size_t)g * 4 * 8 * b2 * c);              // R
    b.take((size_t)g * 2 * p->b1.w * ncy * c);       // contact P
    b.take((size_t)g * 1 * p->b2.w * ncy * c);       // contact Q
    b.take((size_t)g * b2 * c);                      // contact R
    upd(b.off);
  }
  if (p->want_o3) {
    const size_t J = p->ranks[3], I = p->ranks[2];
    Bump b;
    b.take(g * J * 4 * b2 * c);  // E
    b.take(g * J * 8 * 16);      // maxima (E, R_O, F)
    const size_t base = b.off;
    Bump in = b;
    in.take(g * J * I * 12 * p->b1.w * ncy * c);
    in.take(g * J * I * 4 * p->b2.w * ncy * c);
    in.take(g * J * I * 4 * b2 * c);
    in.take(g * J * I * 4 * 8);
    upd(in.off);
    Bump out = b;
    out.take(g * J * 12 * p->b1.w * ncy * c);
    out.take(g * J * 9 * p->b2.w * ncy * c);
    out.take(g * J * 4 * p->b3.w * ncy * c);
    out.take(g * J * 4 * b3 * c);
    upd(out.off);
    (void)base;
  }
  // final column transforms at the reference ny
  {
    const size_t wmax = std::max({(size_t)p->b1.w, (size_t)p->b2.w, (size_t)p->b3.w});
    upd((size_t)g * 2 * wmax * p->d.ny * c);
  }
  (void)b1;
  return need;
}

// The inner accumulation: blocks of 256 threads over (ACC_TILE-bin tiles,
// units); each block covers every outer node of its unit.
static void launch_acc_inner(const AccArgs& c, size_t plane, int units, cudaStream_t st) {
  const int ntiles = (int)((plane + ACC_TILE - 1) / ACC_TILE);
  // at least one block (an empty box runs no tile)
  acc_inner_kernel<<<dim3(std::max(1, std::min(ntiles, 4096)), units), 256, 0, st>>>(c);
}

static void plan_free(gl_plan* p) {
  if (!p) return;
  cudaFree(p->geo4);
  cudaFree(p->geo1);
  cudaFree(p->geo2);
  cudaFree(p->geo3);
  cudaFree(p->tw);
  cudaFree(p->nodes);
  cudaFree(p->comp_scale);
  cudaFree(p->twx);
  cudaFree(p->twy);
  for (int l = 0; l < GL_MAX_LANES; ++l) {
    if (p->lane_st[l]) cudaStreamDestroy(p->lane_st[l]);
    if (p->lane_ev[l]) cudaEventDestroy(p->lane_ev[l]);
  }
  delete p;
}

// Workspace layout of an order-1..3 plan for groups of g units (byte offsets
// into one lane's region); returns the lane's size, a multiple of 256 bytes.
static size_t layout_units(gl_plan* p, int g) {
  p->group = g;
  const size_t c = sizeof(cplx);
  const size_t b1 = (size_t)p->b1.w * p->b1.h, b2 = (size_t)p->b2.w * p->b2.h,
               b3 = (size_t)p->b3.w * p->b3.h;
  Bump b;
  p->o_slots = b.take(g * sizeof(UnitSlots));
  p->o_us = b.take(g * sizeof(UnitScalars));
  p->o_box = b.take(g * b1 * c);
  p->o_s1 = b.take(g * b1);
  p->o_s1f = b.take((size_t)g * p->b1.h * p->ww1 * 8);
  p->o_s1r = b.take((size_t)g * p->b1.h * p->ww1 * 8);
  p->o_s2 = b.take(g * b2);
  p->o_s2f = b.take((size_t)g * p->b2.h * p->ww2 * 8);
  p->o_s2r = b.take((size_t)g * p->b2.h * p->ww2 * 8);
  p->o_s3 = b.take(g * b3);
  p->o_ch = b.take(g * 2 * b1);
  p->o_chf = b.take((size_t)g * 2 * p->b1.h * p->ww1 * 8);
  p->o_chr = b.take((size_t)g * 2 * p->b1.h * p->ww1 * 8);
  p->o_pm = b.take(g * 3 * b2);
  p->o_out22 = b.take(g * b2 * c);
  p->o_outp22 = b.take(g * b2 * c);
  p->o_out33 = b.take(g * 2 * b3 * c);
  p->scratch_bytes = stage_scratch(p, g);
  p->o_scratch = b.take(p->scratch_bytes);
  return b.off;
}

extern "C" gl_status gl_plan_create(gl_plan** out, const gl_plan_desc* desc) {
  if (!out || !desc) return fail(GL_ERR_INVALID_ARGUMENT, "null plan or descriptor");
  *out = nullptr;
  const gl_plan_desc& d = *desc;
  if (d.order < 1 || d.order > 3) return fail(GL_ERR_INVALID_ARGUMENT, "order must be 1, 2, or 3");
  if (!(d.lx > 0) || !(d.ly > 0) || !std::isfinite(d.lx) || !std::isfinite(d.ly))
    return fail(GL_ERR_INVALID_ARGUMENT, "positive domain lengths and positive even grid sizes are required");
  if (d.nx < 2 || d.ny < 2 || (d.nx % 2) || (d.ny % 2))
    return fail(GL_ERR_INVALID_ARGUMENT, "positive domain lengths and positive even grid sizes are required");
  GenPlan gx, gy;
  if (d.nx < 16 || d.ny < 16 || d.nx > TW_N || d.ny > TW_N || !gen_plan(d.nx, gx) || !gen_plan(d.ny, gy))
    return fail(GL_ERR_UNSUPPORTED,
                "the GPU engine runs even grids from 16 to %d whose sizes have no prime factor above 5 "
                "(got %d x %d)", TW_N, d.ny, d.nx);
  const bool gen = !is_pow2(d.nx) || !is_pow2(d.ny);
  if (gen && d.grid == GL_GRID_REFERENCE)
    return fail(GL_ERR_UNSUPPORTED,
                "product stages on a reference grid that is not a power of two are not run (use the compact grid)");
  if (!(d.depth > 0) || !(d.gravity > 0) || !std::isfinite(d.depth) || !std::isfinite(d.gravity))
    return fail(GL_ERR_INVALID_ARGUMENT, "depth and gravity must be positive");
  if (d.max_units < 1) return fail(GL_ERR_INVALID_ARGUMENT, "max_units must be >= 1");
  if (d.output != GL_OUT_COMPLEX && d.output != GL_OUT_REAL)
    return fail(GL_ERR_INVALID_ARGUMENT, "unknown output mode");
  if (d.grid != GL_GRID_COMPACT && d.grid != GL_GRID_REFERENCE)
    return fail(GL_ERR_INVALID_ARGUMENT, "unknown grid mode");
  int all = GL_COMP_ETA11 | GL_COMP_PSI11;
  if (d.order >= 2) all |= GL_COMP_ETA22 | GL_COMP_PSI22;
  if (d.order >= 3) all |= GL_COMP_ETA33 | GL_COMP_PSI33;
  int comps = d.components ? d.components : all;
  if (comps & ~all) return fail(GL_ERR_INVALID_ARGUMENT, "component mask asks for a component above the order");
  if (d.order >= 2 && (d.eta22_rank < 1 || d.eta22_rank > 16))
    return fail(GL_ERR_RANK, "eta22_rank must be an integer from 1 to 16");
  const int inner = d.inner_rank ? d.inner_rank : 4, outer = d.outer_rank ? d.outer_rank : 4;
  if ((comps & (GL_COMP_ETA33 | GL_COMP_PSI33)) &&
      !((inner == 4 || inner == 6 || inner == 8 || inner == 10 || inner == 12) &&
        (outer == 3 || outer == 4 || outer == 6 || outer == 8 || outer == 10)))
    return fail(GL_ERR_RANK, "unsupported inner or outer third-order GL rank");
  if (d.box_w < 1 || d.box_h < 1) return fail(GL_ERR_INVALID_ARGUMENT, "empty parent box");
  if (d.box_x0 < 1)
    return fail(GL_ERR_SUPPORT, "strict-forward nonzero analytic eta1 support is required");
  const int xmax = d.box_x0 + d.box_w - 1;
  const int ymax = std::max(std::abs(d.box_y0), std::abs(d.box_y0 + d.box_h - 1));
  if (xmax >= d.nx / 2 || ymax >= d.ny / 2)
    return fail(GL_ERR_NYQUIST, "An input component reaches or exceeds a Nyquist boundary.");
  const bool o3 = comps & (GL_COMP_ETA33 | GL_COMP_PSI33);
  const bool o2 = comps & (GL_COMP_ETA22 | GL_COMP_PSI22);
  if (o3 && (3 * xmax >= d.nx / 2 || 3 * ymax >= d.ny / 2))
    return fail(GL_ERR_ALIAS, "cubic output support reaches a Nyquist boundary");
  if (o2 && (2 * xmax >= d.nx / 2 || 2 * ymax >= d.ny / 2))
    return fail(GL_ERR_ALIAS, "quadratic output support reaches a Nyquist boundary");

  gl_plan* p = new gl_plan();
  p->d = d;
  p->d.inner_rank = inner;
  p->d.outer_rank = outer;
  p->comps = comps;
  p->ncomp = 0;
  for (int b = 0; b < 6; ++b)
    if (comps & (1 << b)) p->comp_ids[p->ncomp++] = 1 << b;
  p->want_first = comps & (GL_COMP_ETA11 | GL_COMP_PSI11);
  p->want_eta22 = comps & GL_COMP_ETA22;
  p->want_psi22 = comps & GL_COMP_PSI22;
  p->want_o3 = o3;
  p->b1 = Box{d.box_x0, d.box_y0, d.box_w, d.box_h};
  p->b2 = Box{2 * d.box_x0, 2 * d.box_y0, 2 * (d.box_w - 1) + 1, 2 * (d.box_h - 1) + 1};
  p->b3 = Box{3 * d.box_x0, 3 * d.box_y0, 3 * (d.box_w - 1) + 1, 3 * (d.box_h - 1) + 1};
  p->ww1 = (p->b1.w + 63) / 64;
  p->ww2 = (p->b2.w + 63) / 64;
  const int deg = o3 ? 3 : (o2 ? 2 : 1);
  p->gen = gen;
  p->genx = gx;
  p->geny = gy;
  if (d.grid == GL_GRID_REFERENCE || deg == 1) {
    // (order 1 runs no product stage; its final transforms use nx, ny)
    p->ncx = gen ? 16 : d.nx;
    p->ncy = gen ? 16 : d.ny;
  } else {
    // the smallest power of two covering the stage's box; on a power-of-two
    // reference grid never longer than it, on another grid possibly longer
    // (an alias-free product has the same coefficients on any covering period)
    const Box& bd = deg == 3 ? p->b3 : p->b2;
    p->ncx = std::max(16, next_pow2(bd.w));
    p->ncy = std::max(16, next_pow2(bd.h));
    if (is_pow2(d.nx)) p->ncx = std::min(d.nx, p->ncx);
    if (is_pow2(d.ny)) p->ncy = std::min(d.ny, p->ncy);
  }
  p->lncx = ilog2(p->ncx);
  p->lncy = ilog2(p->ncy);
  p->ncy2 = p->ncy3 = p->ncy;
  p->ncx2 = p->ncx;
  if (d.grid != GL_GRID_REFERENCE && deg > 1) {
    p->ncy2 = std::min(p->ncy, col_len(p->b2.h));
    if (deg == 3) p->ncy3 = std::min(p->ncy, col_len(p->b3.h));
    p->ncx2 = std::min(p->ncx, row_len(p->b2.w));
  }
  p->lncx2 = col_log2(p->ncx2);
  p->lncy2 = col_log2(p->ncy2);
  p->lncy3 = col_log2(p->ncy3);
  p->lnx = ilog2(d.nx);
  p->lny = ilog2(d.ny);
  const int max_banks = o3 ? 21 : (p->want_psi22 ? 16 : 8);
  if (deg > 1 && row_smem(max_banks, p->ncx) > ROW_SMEM_LIMIT) {
    plan_free(p);
    return fail(GL_ERR_UNSUPPORTED,
                "product grid %d x %d exceeds the shared-memory row budget (use the compact grid)",
                d.ny, d.nx);
  }
  p->floor_rel = 16.0 * 2.220446049250313e-16 * std::max(1.0, std::log2((double)d.nx * (double)d.ny));
  p->ranks[0] = d.order >= 2 ? d.eta22_rank : 1;
  p->ranks[1] = 2;
  p->ranks[2] = inner;
  p->ranks[3] = outer;
  for (int k = 0; k < 4; ++k) {
    if (k == 1) continue;
    gl_status st = gauss_laguerre(p->ranks[k], p->h_nodes[k], p->h_weights[k]);
    if (st != GL_OK) {
      plan_free(p);
      return st;
    }
  }
  {  // fixed dual-branch GL2 rule (spatial.py:269-275)
    const double r2 = std::sqrt(2.0);
    p->h_nodes[1][0] = 2.0 - r2;
    p->h_nodes[1][1] = 2.0 + r2;
    p->h_weights[1][0] = p->h_nodes[1][0] / (4.0 * (r2 - 1.0) * (r2 - 1.0));
    p->h_weights[1][1] = p->h_nodes[1][1] / (4.0 * (r2 + 1.0) * (r2 + 1.0));
  }
  const double pscale = d.depth * std::sqrt(d.gravity * d.depth);
  for (int c = 0; c < p->ncomp; ++c) {
    const int id = p->comp_ids[c];
    p->h_comp_scale[c] = (id == GL_COMP_ETA11 || id == GL_COMP_ETA22 || id == GL_COMP_ETA33) ? d.depth : pscale;
  }
  // device tables
  cudaError_t e = cudaSuccess;
  auto geo_alloc = [&](double** g, const Box& b) {
    if (e == cudaSuccess) e = cudaMalloc(g, sizeof(double) * 6 * b.w * b.h);
    if (e == cudaSuccess) {
      const int plane = b.w * b.h;
      geo_kernel<<<std::min(1024, (plane + 255) / 256), 256>>>(*g, b, d.nx, d.ny, d.lx, d.ly, d.depth, 0.0);
      e = cudaGetLastError();
    }
  };
  geo_alloc(&p->geo1, p->b1);
  geo_alloc(&p->geo2, p->b2);
  geo_alloc(&p->geo3, p->b3);
  if (e == cudaSuccess) e = cudaMalloc(&p->tw, sizeof(cplx) * TW_ALLOC);
  if (e == cudaSuccess) {
    twiddle_kernel<<<TW_ALLOC / 256 + 1, 256>>>(p->tw, TW_ALLOC);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMalloc(&p->nodes, sizeof(double) * 8 * MAX_RANK);
  if (e == cudaSuccess) {
    double host[8 * MAX_RANK];
    for (int k = 0; k < 4; ++k) {
      std::memcpy(host + k * MAX_RANK, p->h_nodes[k], sizeof(double) * MAX_RANK);
      std::memcpy(host + (4 + k) * MAX_RANK, p->h_weights[k], sizeof(double) * MAX_RANK);
    }
    e = cudaMemcpy(p->nodes, host, sizeof host, cudaMemcpyHostToDevice);
  }
  if (gen) {
    if (e == cudaSuccess) e = cudaMalloc(&p->twx, sizeof(cplx) * d.nx);
    if (e == cudaSuccess) e = cudaMalloc(&p->twy, sizeof(cplx) * d.ny);
    if (e == cudaSuccess) {
      gen_twiddle_kernel<<<(d.nx + 255) / 256, 256>>>(p->twx, d.nx);
      gen_twiddle_kernel<<<(d.ny + 255) / 256, 256>>>(p->twy, d.ny);
      e = cudaGetLastError();
    }
  }
  if (e == cudaSuccess) e = cudaMalloc(&p->comp_scale, sizeof(double) * 6);
  if (e == cudaSuccess)
    e = cudaMemcpy(p->comp_scale, p->h_comp_scale, sizeof(double) * 6, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    plan_free(p);
    return fail(GL_ERR_CUDA, "plan set-up failed: %s", cudaGetErrorString(e));
  }
  // workspace layout (one lane of max_units units until gl_plan_set_lanes)
  p->lane_bytes = layout_units(p, d.max_units);
  p->ws_total = p->lane_bytes;
  if (cudaGetDevice(&p->device) != cudaSuccess) p->device = 0;
  *out = p;
  return GL_OK;
}

extern "C" void gl_plan_destroy(gl_plan* plan) { plan_free(plan); }

extern "C" gl_status gl_plan_get_info(const gl_plan* p, gl_plan_info* info) {
  if (!p || !info) return fail(GL_ERR_INVALID_ARGUMENT, "null plan or info");
  std::memset(info, 0, sizeof *info);
  info->ncx = p->ncx;
  info->ncy = p->ncy;
  info->ncy_pair = p->ncy2;
  info->ncy_triple = p->ncy3;
  info->ncx_pair = p->ncx2;
  const Box* bs[3] = {&p->b1, &p->b2, &p->b3};
  int* dst[3] = {info->box1, info->box2, info->box3};
  for (int k = 0; k < 3; ++k) {
    dst[k][0] = bs[k]->x0;
    dst[k][1] = bs[k]->y0;
    dst[k][2] = bs[k]->w;
    dst[k][3] = bs[k]->h;
  }
  info->n_components = p->ncomp;
  for (int k = 0; k < p->ncomp; ++k) info->component_ids[k] = p->comp_ids[k];
  double t = 0;
  if (p->comps & GL_COMP_ETA11) t += 1;
  if (p->comps & GL_COMP_PSI11) t += 1;
  if (p->want_eta22) t += 10.0 * p->ranks[0] + 3;
  if (p->want_psi22) t += 108;
  if (p->want_o3) t += p->ranks[3] * (25.0 + 16.0 * p->ranks[2]) + 5;
  if (p->e44) {  // gl_eta44_fftw.cpp: third level, first/pair at order 4, forcing, final
    const double R = p->R44;
    const double pair = R * (16 + 6) + 18;
    t = R * (R * (16 + (R * (16 + 6) + 15) + 4) + 8 + 19 + pair + 2) + 1;
    // psi44: the third-level eta_t (its accumulation and bank), the two contact
    // rows of every outer node and the final psi44 transform
    if (p->e44_psi) t += R * (1 + 2) + 1;
  }
  info->transforms_per_unit = t;
  return GL_OK;
}

extern "C" gl_status gl_plan_set_wait_test(gl_plan* p, unsigned int surplus_bytes, long long wait_cycles) {
  if (!p) return fail(GL_ERR_INVALID_ARGUMENT, "null plan");
  if (wait_cycles < 0 || (surplus_bytes && wait_cycles == 0) || surplus_bytes > (1u << 20))
    return fail(GL_ERR_INVALID_ARGUMENT, "a wait test needs a positive clock budget and at most 1 MiB of surplus");
  p->wait_surplus = surplus_bytes;
  p->wait_cycles = wait_cycles;
  return GL_OK;
}

extern "C" gl_status gl_plan_set_tuning(gl_plan* p, const gl_tuning* t) {
  if (!p || !t) return fail(GL_ERR_INVALID_ARGUMENT, "null plan or tuning");
  auto one_of = [](int v, std::initializer_list<int> ok) {
    for (int o : ok)
      if (v == o) return true;
    return false;
  };
  if (!one_of(t->pair_row_groups, {0, 2, 4, 8, 16}) || !one_of(t->triple_row_groups, {0, 4, 6, 8, 12, 16}) ||
      !one_of(t->col_block_columns, {0, 1, 2, 4, 8, 16}))
    return fail(GL_ERR_INVALID_ARGUMENT,
                "tuning: pair row groups 0/2/4/8/16, triple row groups 0/4/6/8/12/16, column block 0/1/2/4/8/16");
  p->tune = *t;
  return GL_OK;
}

extern "C" gl_status gl_plan_set_lanes(gl_plan* p, int lanes) {
  if (!p) return fail(GL_ERR_INVALID_ARGUMENT, "null plan");
  if (p->e44) return fail(GL_ERR_UNSUPPORTED, "concurrent lanes run the order-1..3 plans only");
  if (lanes < 1 || lanes > GL_MAX_LANES)
    return fail(GL_ERR_INVALID_ARGUMENT, "lanes must be 1..%d (got %d)", GL_MAX_LANES, lanes);
  lanes = std::min(lanes, p->d.max_units);  // at least one unit per lane
  std::lock_guard<std::mutex> lk(p->lane_mu);
  int cur = 0;
  CUDA_TRY(cudaGetDevice(&cur));
  CUDA_TRY(cudaSetDevice(p->device));
  cudaError_t e = cudaSuccess;
  for (int l = 0; l < lanes && e == cudaSuccess; ++l) {
    if (l > 0 && !p->lane_st[l]) e = cudaStreamCreateWithFlags(&p->lane_st[l], cudaStreamNonBlocking);
    if (e == cudaSuccess && !p->lane_ev[l]) e = cudaEventCreateWithFlags(&p->lane_ev[l], cudaEventDisableTiming);
  }
  cudaSetDevice(cur);
  if (e != cudaSuccess) return fail(GL_ERR_CUDA, "lane streams: %s", cudaGetErrorString(e));
  // lanes x groups of ceil(max_units / lanes) units: the workspace stays about
  // the size of one group of max_units
  const int g = (p->d.max_units + lanes - 1) / lanes;
  p->lane_bytes = layout_units(p, g);
  p->ws_total = (size_t)lanes * p->lane_bytes;
  p->lanes = lanes;
  return GL_OK;
}

extern "C" gl_status gl_workspace_size(const gl_plan* p, size_t* bytes) {
  if (!p || !bytes) return fail(GL_ERR_INVALID_ARGUMENT, "null plan or size pointer");
  *bytes = p->ws_total;
  return GL_OK;
}

// ---------------------------------------------------------------------------
// launch helpers
// ---------------------------------------------------------------------------

// Twin banks: a bank whose multiplier is a column-constant factor times
// another bank's on the same source (qx, i qx: constant along a column of a
// box) is written by the column stage from that bank's transformed column
// (see ColArgs::twins), so only the other banks are transformed.
// set_banks() fills the column stage's bank lists from the stage's logical
// list (mult[k], src[k]); the output keeps the logical layout.
struct TwinRule {
  int m, parent, fac;  // m = factor(fac) * parent
};
static const TwinRule kTwinRules[] = {
    {M_QX, M_ONE, 1},   {M_NUQX, M_NU, 1}, {M_IQX, M_ONE, 2}, {M_NUQX, M_MI_NU, 2},
    {M_NU2QX, M_NU2, 1}, {M_IQXA, M_A, 2}};

static void set_banks(ColArgs& a, int nb, const int* mult, const int* src) {
  int parent_of[MAX_BANKS], fac_of[MAX_BANKS];
  for (int k = 0; k < nb; ++k) {
    parent_of[k] = -1;
    fac_of[k] = 0;
    for (const TwinRule& r : kTwinRules) {
      if (mult[k] != r.m || parent_of[k] >= 0) continue;
      for (int j = 0; j < nb; ++j) {
        bool taken = false;  // one twin per transformed bank
        for (int q = 0; q < k; ++q) taken = taken || parent_of[q] == j;
        if (j != k && !taken && mult[j] == r.parent && src[j] == src[k]) {
          parent_of[k] = j;
          fac_of[k] = r.fac;
          break;
        }
      }
    }
  }
  a.twins = 1;
  a.nout = nb;
  int ns = 0;
  for (int k = 0; k < nb; ++k) {
    if (parent_of[k] >= 0) continue;
    a.mult[ns] = mult[k];
    a.src_of[ns] = src[k];
    a.out_of[ns] = k;
    a.twin[ns] = -1;
    a.twin_fac[ns] = 0;
    for (int q = 0; q < nb; ++q)
      if (parent_of[q] == k) {
        a.twin[ns] = q;
        a.twin_fac[ns] = fac_of[q];
      }
    ++ns;
  }
  a.nbanks = ns;
}

template <class T>
static T* at(void* ws, size_t off) {
  return reinterpret_cast<T*>(reinterpret_cast<char*>(ws) + off);
}

static size_t mink_smem(const MinkArgs& m) { return (size_t)2 * (m.ha + m.hb) * sizeof(short); }

static void mink_args(MinkArgs& m, const unsigned long long* a, int ha, int wa, int wwa,
                      const unsigned long long* brev, int hb, int wb, int wwb, unsigned char* c,
                      const double* geoc, UnitSlots* slots, int which) {
  m.a = a;
  m.ha = ha;
  m.wa = wa;
  m.wwa = wwa;
  m.a_job_stride = (long long)ha * wwa;
  m.brev = brev;
  m.hb = hb;
  m.wb = wb;
  m.wwb = wwb;
  m.b_job_stride = (long long)hb * wwb;
  m.c = c;
  m.hc = ha + hb - 1;
  m.wc = wa + wb - 1;
  m.c_job_stride = (long long)m.hc * m.wc;
  m.geoc = geoc;
  m.slots = slots;
  m.which = which;
  m.skip_dup = 0;
}

// The plan's tuned launch shapes applied to one stage's arguments.
static RowArgs tuned(const gl_plan* p, RowArgs r) {
  r.groups = r.kind == ROW_OUTER ? p->tune.triple_row_groups : p->tune.pair_row_groups;
  return r;
}
static ColArgs tuned(const gl_plan* p, ColArgs a) {
  a.cw_max = p->tune.col_block_columns;
  return a;
}
static ColFftArgs tuned(const gl_plan* p, ColFftArgs f) {
  f.cw_max = p->tune.col_block_columns;
  return f;
}

// Final transform of box spectra `spec` ([unit][nb][box]) to the reference
// grid, writing output planes comp_offset.. of each unit.
static gl_status final_output(gl_plan* p, int gu, const Box& box, const double* geo,
                              const cplx* spec, long long spec_stride, int nb, const int* mults,
                              const int* srcs, int comp_offset, void* outputs, void* scratch,
                              cudaStream_t st, const double* comp_scale_dev, UnitScalars* us) {
  if (p->gen) {
    if (nb > 4) return fail(GL_ERR_INVALID_ARGUMENT, "at most 4 final components per launch");
    GenColArgs a;
    std::memset(&a, 0, sizeof a);
    a.nbanks = nb;
    for (int k = 0; k < nb; ++k) {
      a.mult[k] = mults[k];
      a.src_of[k] = srcs[k];
    }
    a.box = box;
    a.geo = geo;
    a.spec = spec;
    a.spec_job_stride = spec_stride;
    a.spec_sub_stride = (long long)box.w * box.h;
    a.out = reinterpret_cast<cplx*>(scratch);
    a.gp = p->geny;
    a.twn = p->twy;
    a.scale = 1.0 / ((double)p->d.nx * (double)p->d.ny);
    gl_status s = launch_gen_cols(a, gu, st);
    if (s != GL_OK) return s;
    GenRowArgs o;
    std::memset(&o, 0, sizeof o);
    o.in = reinterpret_cast<cplx*>(scratch);
    o.w = box.w;
    o.x0 = box.x0;
    o.ny = p->d.ny;
    o.ncomp = nb;
    o.comp_offset = comp_offset;
    o.out_ncomp = p->ncomp;
    o.comp_scale = comp_scale_dev + comp_offset;
    o.out = outputs;
    o.real_only = p->d.output == GL_OUT_REAL;
    o.us = us;
    o.gp = p->genx;
    o.twn = p->twx;
    return launch_gen_rows(o, gu * nb, st);
  }
  ColArgs a;
  std::memset(&a, 0, sizeof a);
  a.kind = COL_PLAIN;
  a.nbanks = nb;
  for (int k = 0; k < nb; ++k) {
    a.mult[k] = mults[k];
    a.src_of[k] = srcs[k];
  }
  a.box = box;
  a.geo = geo;
  a.spec = spec;
  a.spec_job_stride = spec_stride;
  a.spec_sub_stride = (long long)box.w * box.h;
  a.jobs_per_unit = 1;
  a.out = reinterpret_cast<cplx*>(scratch);
  a.n = p->d.ny;
  a.log2n = p->lny;
  a.scale = 1.0 / ((double)p->d.nx * (double)p->d.ny);
  gl_status s = launch_col_ifft(tuned(p, a), gu, st, p->tw);
  if (s != GL_OK) return s;
  OutArgs o;
  std::memset(&o, 0, sizeof o);
  o.in = reinterpret_cast<cplx*>(scratch);
  o.w = box.w;
  o.x0 = box.x0;
  o.nx = p->d.nx;
  o.log2nx = p->lnx;
  o.ny = p->d.ny;
  o.ncomp = nb;
  o.comp_offset = comp_offset;
  o.out_ncomp = p->ncomp;
  o.comp_scale = comp_scale_dev + comp_offset;
  o.out = outputs;
  o.real_only = p->d.output == GL_OUT_REAL;
  o.us = us;
  return launch_out_rows(o, gu * nb, st, p->tw);
}

static int comp_slot(const gl_plan* p, int id) {
  for (int k = 0; k < p->ncomp; ++k)
    if (p->comp_ids[k] == id) return k;
  return -1;
}

// ---------------------------------------------------------------------------
// one group of units
// ---------------------------------------------------------------------------

static gl_status run_group_eta44(gl_plan* p, int gu, const void* spectra, int layout,
                                 void* outputs, void* ws, int* status, cudaStream_t st);

// Support analysis of a group of units (spatial.py:160-189, _order3.py:33-52):
// the parent box spectra (extracted from full spectra when needed), the
// supports S, S2 = S+S, S3 = S2+S, the psi22 radial channels and the per-unit
// scalars.  The box spectra pointer is returned in *spec_out.
static gl_status analyse_group(gl_plan* p, int gu, const void* spectra, int layout, void* ws,
                               cudaStream_t st, const cplx** spec_out) {
  const int T = 256;
  const Box B1 = p->b1, B2 = p->b2, B3 = p->b3;
  const int pl1 = B1.w * B1.h, pl2 = B2.w * B2.h, pl3 = B3.w * B3.h;
  UnitSlots* slots = at<UnitSlots>(ws, p->o_slots);
  UnitScalars* us = at<UnitScalars>(ws, p->o_us);
  cplx* boxv = at<cplx>(ws, p->o_box);
  unsigned char* s1 = at<unsigned char>(ws, p->o_s1);
  unsigned long long* s1f = at<unsigned long long>(ws, p->o_s1f);
  unsigned long long* s1r = at<unsigned long long>(ws, p->o_s1r);
  unsigned char* s2 = at<unsigned char>(ws, p->o_s2);
  unsigned long long* s2f = at<unsigned long long>(ws, p->o_s2f);
  unsigned long long* s2r = at<unsigned long long>(ws, p->o_s2r);
  unsigned char* s3 = at<unsigned char>(ws, p->o_s3);
  unsigned char* ch = at<unsigned char>(ws, p->o_ch);
  unsigned long long* chf = at<unsigned long long>(ws, p->o_chf);
  unsigned long long* chr = at<unsigned long long>(ws, p->o_chr);
  unsigned char* pm = at<unsigned char>(ws, p->o_pm);
  {
    LaunchScope ls_("slots_init_kernel", st, 0.0);
    slots_init_kernel<<<(gu + 63) / 64, 64, 0, st>>>(slots, gu);
  }
  LAUNCH_CHECK("slots_init_kernel");
  const cplx* spec = boxv;
  if (layout == GL_SPECTRA_FULL) {
    CUDA_TRY(cudaMemsetAsync(boxv, 0, sizeof(cplx) * (size_t)gu * pl1, st));
    dim3 g(grid_for((size_t)p->d.nx * p->d.ny, T, 1024), gu);
    {
      LaunchScope ls_("extract_kernel", st, 0.0);
      extract_kernel<<<g, T, 0, st>>>(reinterpret_cast<const cplx*>(spectra), boxv, B1, p->d.nx,
                                    p->d.ny, slots);
    }
    LAUNCH_CHECK("extract_kernel");
  } else {
    spec = reinterpret_cast<const cplx*>(spectra);
    dim3 g(grid_for(pl1, T, 64), gu);
    {
      LaunchScope ls_("box_max_kernel", st, 0.0);
      box_max_kernel<<<g, T, 0, st>>>(spec, pl1, slots);
    }
    LAUNCH_CHECK("box_max_kernel");
  }
  {
    dim3 g(grid_for(pl1, T, 64), gu);
    {
      LaunchScope ls_("support_kernel", st, 0.0);
      support_kernel<<<g, T, 0, st>>>(spec, p->geo1, B1, slots, s1);
    }
    LAUNCH_CHECK("support_kernel");
    {
      LaunchScope ls_("peak_kernel", st, 0.0);
      peak_kernel<<<g, T, 0, st>>>(spec, p->geo1, B1, p->d.nx, p->d.ny, slots, s1, ch,
                                 p->want_psi22 ? 1 : 0);
    }
    LAUNCH_CHECK("peak_kernel");
  }
  const bool need_s2 = p->want_eta22 || p->want_psi22 || p->want_o3;
  if (need_s2) {
    dim3 g(grid_for(B1.h * p->ww1, T, 64), gu);
    {
      LaunchScope ls_("bitrows_kernel", st, 0.0);
      bitrows_kernel<<<g, T, 0, st>>>(s1, B1.h, B1.w, p->ww1, s1f, s1r);
    }
    LAUNCH_CHECK("bitrows_kernel");
    if (gu > 1) {
      LaunchScope ls_("support_dup_kernel", st, 0.0);
      support_dup_kernel<<<gu - 1, T, 0, st>>>(s1f, (long long)B1.h * p->ww1, slots);
    }
    LAUNCH_CHECK("support_dup_kernel");
    MinkArgs m;
    mink_args(m, s1f, B1.h, B1.w, p->ww1, s1r, B1.h, B1.w, p->ww1, s2, p->geo2, slots, 2);
    m.skip_dup = 1;
    dim3 g2(grid_for(pl2, T, 256), gu);
    {
      LaunchScope ls_("minkowski_kernel", st, 0.0);
      minkowski_kernel<<<g2, T, mink_smem(m), st>>>(m);
    }
    LAUNCH_CHECK("minkowski_kernel");
    if (gu > 1) {
      LaunchScope ls_("mink_copy_kernel", st, 0.0);
      mink_copy_kernel<<<dim3(grid_for(pl2, T, 64), gu - 1), T, 0, st>>>(s2, pl2, 2, slots);
    }
    LAUNCH_CHECK("mink_copy_kernel");
  }
  if (p->want_o3) {
    dim3 g(grid_for(B2.h * p->ww2, T, 64), gu);
    {
      LaunchScope ls_("bitrows_kernel", st, 0.0);
      bitrows_kernel<<<g, T, 0, st>>>(s2, B2.h, B2.w, p->ww2, s2f, s2r);
    }
    LAUNCH_CHECK("bitrows_kernel");
    MinkArgs m;
    mink_args(m, s2f, B2.h, B2.w, p->ww2, s1r, B1.h, B1.w, p->ww1, s3, p->geo3, slots, 3);
    m.skip_dup = 1;
    dim3 g3(grid_for(pl3, T, 512), gu);
    {
      LaunchScope ls_("minkowski_kernel", st, 0.0);
      minkowski_kernel<<<g3, T, mink_smem(m), st>>>(m);
    }
    LAUNCH_CHECK("minkowski_kernel");
    if (gu > 1) {
      LaunchScope ls_("mink_copy_kernel", st, 0.0);
      mink_copy_kernel<<<dim3(grid_for(pl3, T, 64), gu - 1), T, 0, st>>>(s3, pl3, 3, slots);
    }
    LAUNCH_CHECK("mink_copy_kernel");
  }
  if (p->want_psi22) {
    dim3 g(grid_for(B1.h * p->ww1, T, 64), gu * 2);
    {
      LaunchScope ls_("bitrows_kernel", st, 0.0);
      bitrows_kernel<<<g, T, 0, st>>>(ch, B1.h, B1.w, p->ww1, chf, chr);
    }
    LAUNCH_CHECK("bitrows_kernel");
    const long long cstride = (long long)B1.h * p->ww1;
    const int pairs[3][2] = {{0, 0}, {0, 1}, {1, 1}};
    for (int k = 0; k < 3; ++k) {
      MinkArgs m;
      mink_args(m, chf + pairs[k][0] * cstride, B1.h, B1.w, p->ww1, chr + pairs[k][1] * cstride,
                B1.h, B1.w, p->ww1, pm + (size_t)k * pl2, nullptr, slots, 0);
      m.a_job_stride = 2 * cstride;
      m.b_job_stride = 2 * cstride;
      m.c_job_stride = 3LL * pl2;
      dim3 g2(grid_for(pl2, T, 256), gu);
      {
        LaunchScope ls_("minkowski_kernel", st, 0.0);
        minkowski_kernel<<<g2, T, mink_smem(m), st>>>(m);
      }
      LAUNCH_CHECK("minkowski_kernel");
    }
  }
  {
    ScalarArgs a;
    a.slots = slots;
    a.us = us;
    a.geo1 = p->geo1;
    a.box = B1;
    a.nx = p->d.nx;
    a.ny = p->d.ny;
    a.order = p->d.order;
    a.want_eta22 = p->want_eta22;
    a.want_psi22 = p->want_psi22;
    a.want_o3 = p->want_o3;
    a.allow_below = p->d.allow_below_model_parent_domain;
    a.full_input = layout == GL_SPECTRA_FULL;
    a.want_e44 = 0;
    a.fixed_peak = 0.0;
    {
      LaunchScope ls_("scalars_kernel", st, 0.0);
      scalars_kernel<<<(gu + 63) / 64, 64, 0, st>>>(a, gu);
    }
    LAUNCH_CHECK("scalars_kernel");
  }
  *spec_out = spec;
  return GL_OK;
}

static gl_status run_group(gl_plan* p, int gu, const void* spectra, int layout, void* outputs,
                           void* ws, int* status, cudaStream_t st) {
  if (p->e44) return run_group_eta44(p, gu, spectra, layout, outputs, ws, status, st);
  const int T = 256;
  const Box B1 = p->b1, B2 = p->b2, B3 = p->b3;
  const int pl1 = B1.w * B1.h, pl2 = B2.w * B2.h, pl3 = B3.w * B3.h;
  UnitScalars* us = at<UnitScalars>(ws, p->o_us);
  unsigned char* s2 = at<unsigned char>(ws, p->o_s2);
  unsigned char* s3 = at<unsigned char>(ws, p->o_s3);
  unsigned char* ch = at<unsigned char>(ws, p->o_ch);
  unsigned char* pm = at<unsigned char>(ws, p->o_pm);
  cplx* out22 = at<cplx>(ws, p->o_out22);
  cplx* outp22 = at<cplx>(ws, p->o_outp22);
  cplx* out33 = at<cplx>(ws, p->o_out33);
  char* scratch = at<char>(ws, p->o_scratch);
  const double* dn = p->nodes;  // [k*MAX_RANK] nodes, [(4+k)*MAX_RANK] weights
  gl_status s;
  const cplx* spec = nullptr;
  if ((s = analyse_group(p, gu, spectra, layout, ws, st, &spec)) != GL_OK) return s;
  const double inv_scale = 1.0 / ((double)p->d.nx * (double)p->d.ny);
  const double nn = (double)p->d.nx * (double)p->d.ny;
  const int ncy2 = p->ncy2, ncy3 = p->ncy3;
  const double fwd_scale2 = nn / ((double)p->ncx2 * (double)ncy2);
  const double fwd_scale3 = nn / ((double)p->ncx * (double)ncy3);

  // ---------------- eta22 (spatial.py:156-231) ----------------
  if (p->want_eta22) {
    const int J = p->ranks[0];
    const int njobs = gu * J;
    Bump b;
    cplx* P = reinterpret_cast<cplx*>(scratch + b.take((size_t)njobs * 8 * B1.w * ncy2 * sizeof(cplx)));
    cplx* Q = reinterpret_cast<cplx*>(scratch + b.take((size_t)njobs * 2 * B2.w * ncy2 * sizeof(cplx)));
    cplx* R = reinterpret_cast<cplx*>(scratch + b.take((size_t)njobs * 2 * pl2 * sizeof(cplx)));
    unsigned long long* mx = reinterpret_cast<unsigned long long*>(scratch + b.take((size_t)njobs * 2 * 8));
    CUDA_TRY(cudaMemsetAsync(mx, 0, (size_t)njobs * 2 * 8, st));
    ColArgs a;
    std::memset(&a, 0, sizeof a);
    a.kind = COL_ETA22;
    const int m8[8] = {M_ONE, M_NU, M_NU2, M_QX_DIVNU, M_QY_DIVNU, M_Q2_DIVNU, M_QX, M_QY};
    const int z8[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    set_banks(a, 8, m8, z8);
    a.box = B1;
    a.geo = p->geo1;
    a.spec = spec;
    a.spec_job_stride = pl1;
    a.jobs_per_unit = J;
    a.us = us;
    a.nodes = dn + 0 * MAX_RANK;
    a.out = P;
    a.n = ncy2;
    a.log2n = p->lncy2;
    a.scale = inv_scale;
    if ((s = launch_col_ifft(tuned(p, a), njobs, st, p->tw)) != GL_OK) return s;
    RowArgs r;
    std::memset(&r, 0, sizeof r);
    r.kind = ROW_ETA22;
    r.grp[0] = BankGroup{P, 8, B1.x0, B1.w};
    r.ngrp = 1;
    r.nout = 2;
    r.out_x0 = B2.x0;
    r.out_w = B2.w;
    r.out = Q;
    r.nx = p->ncx2;
    r.log2nx = p->lncx2;
    r.ny = ncy2;
    r.us = us;
    r.jobs_per_unit = J;
    r.gmax = ROW_GMAX;
    r.wait_surplus = p->wait_surplus;
    r.wait_cycles = p->wait_cycles;
    if ((s = launch_row(tuned(p, r), njobs, st, p->tw)) != GL_OK) return s;
    ColFftArgs f;
    f.in = Q;
    f.out = R;
    f.box = B2;
    f.n = ncy2;
    f.log2n = p->lncy2;
    f.nsrc = 2;
    f.jobs_per_unit = J;
    f.mask = s2;
    f.maxslot = mx;
    f.scale = fwd_scale2;
    if ((s = launch_col_fft(tuned(p, f), njobs * 2, st, p->tw)) != GL_OK) return s;
    AccArgs c;
    std::memset(&c, 0, sizeof c);
    c.us = us;
    c.geo = p->geo2;
    c.box = B2;
    c.in = R;
    c.maxin = mx;
    c.out = out22;
    c.nodes = dn + 0 * MAX_RANK;
    c.weights = dn + 4 * MAX_RANK;
    c.nnodes = J;
    c.floor_rel = p->floor_rel;
    dim3 g(grid_for(pl2, T, 256), gu);
    {
      LaunchScope ls_("acc_eta22_kernel", st, 0.0);
      acc_eta22_kernel<<<g, T, 0, st>>>(c);
    }
    LAUNCH_CHECK("acc_eta22_kernel");
  }

  // ---------------- psi22 (spatial.py:234-414) ----------------
  if (p->want_psi22) {
    const int njobs_c = gu * 2 * 2 * 2;  // (unit, branch, node, channel)
    const int njobs_r = gu * 2 * 2;      // (unit, branch, node)
    Bump b;
    cplx* P = reinterpret_cast<cplx*>(scratch + b.take((size_t)njobs_c * 8 * B1.w * ncy2 * sizeof(cplx)));
    cplx* Q = reinterpret_cast<cplx*>(scratch + b.take((size_t)njobs_r * 8 * B2.w * ncy2 * sizeof(cplx)));
    cplx* R = reinterpret_cast<cplx*>(scratch + b.take((size_t)njobs_r * 8 * pl2 * sizeof(cplx)));
    cplx* Pc = reinterpret_cast<cplx*>(scratch + b.take((size_t)gu * 2 * B1.w * ncy2 * sizeof(cplx)));
    cplx* Qc = reinterpret_cast<cplx*>(scratch + b.take((size_t)gu * 1 * B2.w * ncy2 * sizeof(cplx)));
    cplx* Rc = reinterpret_cast<cplx*>(scratch + b.take((size_t)gu * pl2 * sizeof(cplx)));
    ColArgs a;
    std::memset(&a, 0, sizeof a);
    a.kind = COL_PSI22;
    a.nbanks = 8;
    const int m8[8] = {M_ONE, M_NU, M_NU2, M_QX_DIVNU, M_QY_DIVNU, M_Q2_DIVNU, M_QX, M_QY};
    for (int k = 0; k < 8; ++k) a.mult[k] = m8[k];
    a.box = B1;
    a.geo = p->geo1;
    a.spec = spec;
    a.spec_job_stride = pl1;
    a.jobs_per_unit = 8;
    a.us = us;
    a.nodes = dn + 1 * MAX_RANK;
    a.n_inner = 2;
    a.chan_mask = ch;
    a.out = P;
    a.n = ncy2;
    a.log2n = p->lncy2;
    a.scale = inv_scale;
    if ((s = launch_col_ifft(tuned(p, a), njobs_c, st, p->tw)) != GL_OK) return s;
    RowArgs r;
    std::memset(&r, 0, sizeof r);
    r.kind = ROW_PSI22;
    // job (unit, branch, node): its two channels are consecutive col jobs,
    // so a row job sees 16 consecutive banks.
    r.grp[0] = BankGroup{P, 16, B1.x0, B1.w};
    r.ngrp = 1;
    r.nout = 8;
    r.out_x0 = B2.x0;
    r.out_w = B2.w;
    r.out = Q;
    r.nx = p->ncx2;
    r.log2nx = p->lncx2;
    r.ny = ncy2;
    r.us = us;
    r.jobs_per_unit = 4;
    r.gmax = ROW_GMAX;
    r.wait_surplus = p->wait_surplus;
    r.wait_cycles = p->wait_cycles;
    if ((s = launch_row(tuned(p, r), njobs_r, st, p->tw)) != GL_OK) return s;
    ColFftArgs f;
    f.in = Q;
    f.out = R;
    f.box = B2;
    f.n = ncy2;
    f.log2n = p->lncy2;
    f.nsrc = 8;
    f.jobs_per_unit = 4;
    f.mask = nullptr;
    f.maxslot = nullptr;
    f.scale = fwd_scale2;
    if ((s = launch_col_fft(tuned(p, f), njobs_r * 8, st, p->tw)) != GL_OK) return s;
    // Taylor contact 0.5 eta11 phi1z
    ColArgs cc;
    std::memset(&cc, 0, sizeof cc);
    cc.kind = COL_PLAIN;
    cc.nbanks = 2;
    cc.mult[0] = M_ONE;
    cc.mult[1] = M_NU;
    cc.src_of[0] = 0;
    cc.src_of[1] = 0;
    cc.box = B1;
    cc.geo = p->geo1;
    cc.spec = spec;
    cc.spec_job_stride = pl1;
    cc.jobs_per_unit = 1;
    cc.out = Pc;
    cc.n = ncy2;
    cc.log2n = p->lncy2;
    cc.scale = inv_scale;
    if ((s = launch_col_ifft(tuned(p, cc), gu, st, p->tw)) != GL_OK) return s;
    RowArgs rc;
    std::memset(&rc, 0, sizeof rc);
    rc.kind = ROW_CONTACT22;
    rc.grp[0] = BankGroup{Pc, 2, B1.x0, B1.w};
    rc.ngrp = 1;
    rc.nout = 1;
    rc.out_x0 = B2.x0;
    rc.out_w = B2.w;
    rc.out = Qc;
    rc.nx = p->ncx2;
    rc.log2nx = p->lncx2;
    rc.ny = ncy2;
    rc.us = us;
    rc.jobs_per_unit = 1;
    rc.gmax = ROW_GMAX;
    rc.wait_surplus = p->wait_surplus;
    rc.wait_cycles = p->wait_cycles;
    if ((s = launch_row(tuned(p, rc), gu, st, p->tw)) != GL_OK) return s;
    ColFftArgs fc = f;
    fc.in = Qc;
    fc.out = Rc;
    fc.nsrc = 1;
    fc.jobs_per_unit = 1;
    if ((s = launch_col_fft(tuned(p, fc), gu, st, p->tw)) != GL_OK) return s;
    AccArgs c;
    std::memset(&c, 0, sizeof c);
    c.us = us;
    c.geo = p->geo2;
    c.box = B2;
    c.in = R;
    c.out = outp22;
    c.mask = s2;
    c.pmask = pm;
    c.extra = Rc;
    c.nodes = dn + 1 * MAX_RANK;
    c.weights = dn + 5 * MAX_RANK;
    c.nnodes = 2;
    dim3 g(grid_for(pl2, T, 256), gu);
    {
      LaunchScope ls_("acc_psi22_kernel", st, 0.0);
      acc_psi22_kernel<<<g, T, 0, st>>>(c);
    }
    LAUNCH_CHECK("acc_psi22_kernel");
  }

  // ---------------- order 3 (_order3.py:18-148) ----------------
  if (p->want_o3) {
    const int J = p->ranks[3], I = p->ranks[2];
    const int nuj = gu * J;
    const int njobs = nuj * I;
    Bump b;
    cplx* E = reinterpret_cast<cplx*>(scratch + b.take((size_t)nuj * 4 * pl2 * sizeof(cplx)));
    unsigned long long* mxs = reinterpret_cast<unsigned long long*>(scratch + b.take((size_t)nuj * 8 * 16));
    unsigned long long* maxEt = mxs;                 // [nuj]
    unsigned long long* maxRO = mxs + nuj;           // [nuj][4]
    unsigned long long* maxF = mxs + 5 * nuj;        // [nuj][2]
    CUDA_TRY(cudaMemsetAsync(mxs, 0, (size_t)nuj * 8 * 8, st));
    // inner stage buffers
    Bump bi = b;
    cplx* PI = reinterpret_cast<cplx*>(scratch + bi.take((size_t)njobs * 12 * B1.w * ncy2 * sizeof(cplx)));
    cplx* QI = reinterpret_cast<cplx*>(scratch + bi.take((size_t)njobs * 4 * B2.w * ncy2 * sizeof(cplx)));
    cplx* RI = reinterpret_cast<cplx*>(scratch + bi.take((size_t)njobs * 4 * pl2 * sizeof(cplx)));
    unsigned long long* maxRI = reinterpret_cast<unsigned long long*>(scratch + bi.take((size_t)njobs * 4 * 8));
    CUDA_TRY(cudaMemsetAsync(maxRI, 0, (size_t)njobs * 4 * 8, st));
    {
      ColArgs a;
      std::memset(&a, 0, sizeof a);
      a.kind = COL_INNER;
      const int m12[12] = {M_ONE, M_NU, M_NU2, M_NU3, M_QX_SNU, M_QY_SNU,
                           M_QX, M_QY, M_Q2_SNU, M_Q2, M_NUQX, M_NUQY};
      const int z12[12] = {0};
      set_banks(a, 12, m12, z12);
      a.box = B1;
      a.geo = p->geo1;
      a.spec = spec;
      a.spec_job_stride = pl1;
      a.jobs_per_unit = J * I;
      a.us = us;
      a.nodes = dn + 3 * MAX_RANK;
      a.nodes2 = dn + 2 * MAX_RANK;
      a.n_inner = I;
      a.n_outer = J;
      a.out = PI;
      a.n = ncy2;
      a.log2n = p->lncy2;
      a.scale = inv_scale;
      if ((s = launch_col_ifft(tuned(p, a), njobs, st, p->tw)) != GL_OK) return s;
      RowArgs r;
      std::memset(&r, 0, sizeof r);
      r.kind = ROW_INNER;
      r.grp[0] = BankGroup{PI, 12, B1.x0, B1.w};
      r.ngrp = 1;
      r.nout = 4;
      r.out_x0 = B2.x0;
      r.out_w = B2.w;
      r.out = QI;
      r.nx = p->ncx2;
      r.log2nx = p->lncx2;
      r.ny = ncy2;
      r.us = us;
      r.jobs_per_unit = J * I;
      r.gmax = ROW_GMAX;
      r.wait_surplus = p->wait_surplus;
      r.wait_cycles = p->wait_cycles;
      if ((s = launch_row(tuned(p, r), njobs, st, p->tw)) != GL_OK) return s;
      ColFftArgs f;
      f.in = QI;
      f.out = RI;
      f.box = B2;
      f.n = ncy2;
      f.log2n = p->lncy2;
      f.nsrc = 4;
      f.jobs_per_unit = J * I;
      f.mask = s2;
      f.maxslot = maxRI;
      f.scale = fwd_scale2;
      if ((s = launch_col_fft(tuned(p, f), njobs * 4, st, p->tw, "col_fft_kernel[inner]")) != GL_OK) return s;
      AccArgs c;
      std::memset(&c, 0, sizeof c);
      c.us = us;
      c.geo = p->geo2;
      c.box = B2;
      c.in = RI;
      c.maxin = maxRI;
      c.out = E;
      c.maxout = maxEt;
      c.mask = s2;
      c.nodes = dn + 2 * MAX_RANK;
      c.weights = dn + 6 * MAX_RANK;
      c.nnodes = I;
      c.nsub = J;
      c.floor_rel = p->floor_rel;
      {
        LaunchScope ls_("acc_inner_kernel", st, 0.0);
        launch_acc_inner(c, pl2, nuj / c.nsub, st);
      }
      LAUNCH_CHECK("acc_inner_kernel");
    }
    // outer stage buffers (reuse the inner region)
    Bump bo = b;
    cplx* P1 = reinterpret_cast<cplx*>(scratch + bo.take((size_t)nuj * 12 * B1.w * ncy3 * sizeof(cplx)));
    cplx* P2 = reinterpret_cast<cplx*>(scratch + bo.take((size_t)nuj * 9 * B2.w * ncy3 * sizeof(cplx)));
    cplx* QO = reinterpret_cast<cplx*>(scratch + bo.take((size_t)nuj * 4 * B3.w * ncy3 * sizeof(cplx)));
    cplx* RO = reinterpret_cast<cplx*>(scratch + bo.take((size_t)nuj * 4 * pl3 * sizeof(cplx)));
    {
      ColArgs a;
      std::memset(&a, 0, sizeof a);
      a.kind = COL_OUTER1;
      const int m12[12] = {M_ONE, M_IQX, M_IQY, M_QX_SNU, M_QY_SNU, M_MI_NU,
                           M_NUQX, M_NUQY, M_MI_Q2_SNU, M_MI_Q2NU, M_MINUS_A, M_MINUS_Q2};
      const int z12[12] = {0};
      set_banks(a, 12, m12, z12);
      a.box = B1;
      a.geo = p->geo1;
      a.spec = spec;
      a.spec_job_stride = pl1;
      a.jobs_per_unit = J;
      a.us = us;
      a.nodes = dn + 3 * MAX_RANK;
      a.out = P1;
      a.n = ncy3;
      a.log2n = p->lncy3;
      a.scale = inv_scale;
      if ((s = launch_col_ifft(tuned(p, a), nuj, st, p->tw)) != GL_OK) return s;
      ColArgs a2;
      std::memset(&a2, 0, sizeof a2);
      a2.kind = COL_OUTER2;
      const int m9[9] = {M_ONE, M_IQX, M_IQY, M_IQX, M_IQY, M_A, M_Q2, M_A, M_ONE};
      const int src9[9] = {0, 0, 0, 2, 2, 2, 2, 3, 1};
      set_banks(a2, 9, m9, src9);
      a2.box = B2;
      a2.geo = p->geo2;
      a2.spec = E;
      a2.spec_job_stride = 4LL * pl2;
      a2.spec_sub_stride = pl2;
      a2.jobs_per_unit = J;
      a2.us = us;
      a2.floor_max = maxEt;
      a2.floor_rel = p->floor_rel;
      a2.out = P2;
      a2.n = ncy3;
      a2.log2n = p->lncy3;
      a2.scale = inv_scale;
      if ((s = launch_col_ifft(tuned(p, a2), nuj, st, p->tw)) != GL_OK) return s;
      RowArgs r;
      std::memset(&r, 0, sizeof r);
      r.kind = ROW_OUTER;
      r.grp[0] = BankGroup{P1, 12, B1.x0, B1.w};
      r.grp[1] = BankGroup{P2, 9, B2.x0, B2.w};
      r.ngrp = 2;
      r.nout = 4;
      r.out_x0 = B3.x0;
      r.out_w = B3.w;
      r.out = QO;
      r.nx = p->ncx;
      r.log2nx = p->lncx;
      r.ny = ncy3;
      r.us = us;
      r.jobs_per_unit = J;
      r.gmax = ROW_GMAX;
      r.wait_surplus = p->wait_surplus;
      r.wait_cycles = p->wait_cycles;
      if ((s = launch_row(tuned(p, r), nuj, st, p->tw)) != GL_OK) return s;
      ColFftArgs f;
      f.in = QO;
      f.out = RO;
      f.box = B3;
      f.n = ncy3;
      f.log2n = p->lncy3;
      f.nsrc = 4;
      f.jobs_per_unit = J;
      f.mask = s3;
      f.maxslot = maxRO;
      f.scale = fwd_scale3;
      if ((s = launch_col_fft(tuned(p, f), nuj * 4, st, p->tw, "col_fft_kernel[outer]")) != GL_OK) return s;
      AccArgs c;
      std::memset(&c, 0, sizeof c);
      c.us = us;
      c.geo = p->geo3;
      c.box = B3;
      c.in = RO;
      c.maxin = maxRO;
      c.maxout = maxF;
      c.mask = s3;
      c.floor_rel = p->floor_rel;
      c.nsub = J;
      dim3 g(grid_for(pl3, T, 48), nuj);
      {
        LaunchScope ls_("acc_outer_max_kernel", st, 0.0);
        acc_outer_max_kernel<<<g, T, 0, st>>>(c);
      }
      LAUNCH_CHECK("acc_outer_max_kernel");
      c.out = out33;
      c.nodes = dn + 3 * MAX_RANK;
      c.weights = dn + 7 * MAX_RANK;
      c.nnodes = J;
      dim3 g2(grid_for(pl3, T, 256), gu);
      {
        LaunchScope ls_("acc_outer_kernel", st, 0.0);
        acc_outer_kernel<<<g2, T, 0, st>>>(c, maxF);
      }
      LAUNCH_CHECK("acc_outer_kernel");
    }
  }

  // ---------------- outputs on the reference grid ----------------
  if (p->want_first) {
    int mults[2], n = 0, off = -1;
    if (p->comps & GL_COMP_ETA11) {
      mults[n++] = M_ONE;
      off = comp_slot(p, GL_COMP_ETA11);
    }
    if (p->comps & GL_COMP_PSI11) {
      mults[n++] = M_PSI11;
      if (off < 0) off = comp_slot(p, GL_COMP_PSI11);
    }
    const int srcs[2] = {0, 0};  // both read the parent spectrum
    if ((s = final_output(p, gu, B1, p->geo1, spec, pl1, n, mults, srcs, off, outputs, scratch, st,
                          p->comp_scale, us)) != GL_OK)
      return s;
  }
  if (p->want_eta22) {
    const int m1[1] = {M_ONE}, z1[1] = {0};
    if ((s = final_output(p, gu, B2, p->geo2, out22, pl2, 1, m1, z1, comp_slot(p, GL_COMP_ETA22),
                          outputs, scratch, st, p->comp_scale, us)) != GL_OK)
      return s;
  }
  if (p->want_psi22) {
    const int m1[1] = {M_ONE}, z1[1] = {0};
    if ((s = final_output(p, gu, B2, p->geo2, outp22, pl2, 1, m1, z1, comp_slot(p, GL_COMP_PSI22),
                          outputs, scratch, st, p->comp_scale, us)) != GL_OK)
      return s;
  }
  if (p->want_o3) {
    const int m2[2] = {M_ONE, M_ONE}, s01[2] = {0, 1};
    const int ce = comp_slot(p, GL_COMP_ETA33), cp = comp_slot(p, GL_COMP_PSI33);
    if (ce >= 0 && cp >= 0) {
      if ((s = final_output(p, gu, B3, p->geo3, out33, 2LL * pl3, 2, m2, s01, ce, outputs, scratch, st,
                            p->comp_scale, us)) != GL_OK)
        return s;
    } else {
      const int which = ce >= 0 ? 0 : 1;
      if ((s = final_output(p, gu, B3, p->geo3, out33 + (size_t)which * pl3, 2LL * pl3, 1, m2,
                            s01, ce >= 0 ? ce : cp, outputs, scratch, st, p->comp_scale, us)) != GL_OK)
        return s;
    }
  }
  // non-finite outputs were flagged by the final transform (out_row_kernel)
  if (status) {
    {
      LaunchScope ls_("status_kernel", st, 0.0);
      status_kernel<<<(gu + 63) / 64, 64, 0, st>>>(us, gu, status);
    }
    LAUNCH_CHECK("status_kernel");
  }
  return GL_OK;
}

// ---------------------------------------------------------------------------
// fourth-order eta44 (paper/order4/cpp/gl_eta44_fftw.cpp)
// ---------------------------------------------------------------------------

// Bank tables of the eta44 graph (multiplier, source spectrum).
static const int E44_FIRST_MULT[19] = {
    M_ONE, M_IQX, M_IQY, M_QX_SNU, M_QY_SNU, M_MI_NU, M_NUQX, M_NUQY, M_MI_Q2_SNU, M_MI_Q2NU,
    M_MINUS_A, M_MINUS_Q2, M_MI_NU2QX, M_MI_NU2QY, M_MINUS_Q2A, M_I_ANU,
    M_PHI_IQXQ2, M_PHI_IQYQ2, M_PHI_Q4};
static const int E44_PAIR_MULT[16] = {M_ONE, M_NU, M_NU2, M_NU3, M_NU4, M_QX_SNU, M_QY_SNU, M_QX,
                                      M_QY, M_Q2_SNU, M_Q2, M_Q2NU, M_NUQX, M_NUQY, M_NU2QX, M_NU2QY};
// pair outputs from (es, ets, ps, pts, ptts) = sources 0..4
static const int E44_POUT_MULT[18] = {M_ONE, M_IQX, M_IQY, M_ONE, M_IQX, M_IQY, M_IQX, M_IQY, M_A,
                                      M_Q2, M_A, M_IQX, M_IQY, M_Q2, M_A, M_IQXA, M_IQYA, M_Q2A};
static const int E44_POUT_SRC[18] = {0, 0, 0, 1, 1, 1, 2, 2, 2, 2, 3, 3, 3, 3, 4, 2, 2, 2};
// third outputs from (es, ps, pts) = sources 0..2
// third-state banks: eta ex ey px py pz pzz pzt [eta_t] from (es, ps, pts [, ets])
static const int E44_TOUT_MULT[9] = {M_ONE, M_IQX, M_IQY, M_IQX, M_IQY, M_A, M_Q2, M_A, M_ONE};
static const int E44_TOUT_SRC[9] = {0, 0, 0, 1, 1, 1, 1, 2, 3};

struct E44Layout {
  size_t E, maxE, T, maxT, OUT, maxOUT, transient;
  size_t total;
};

static E44Layout e44_layout(const gl_plan* p, int g) {
  const size_t c = sizeof(cplx), R = p->R44, ncy = p->ncy;
  const size_t b2 = (size_t)p->b2.w * p->b2.h, b3 = (size_t)p->b3.w * p->b3.h,
               b4 = (size_t)p->b4.w * p->b4.h;
  const size_t JP = R * R * R + R * R, GP = R * R + R;
  const size_t nts = p->e44_psi ? 4 : 3, nout = p->e44_psi ? 2 : 1;
  E44Layout L;
  Bump b;
  L.E = b.take(g * GP * 5 * b2 * c);
  L.maxE = b.take(g * GP * 5 * 8);
  L.T = b.take(g * R * nts * b3 * c);
  L.maxT = b.take(g * R * nts * 8);
  L.OUT = b.take(g * nout * b4 * c);
  L.maxOUT = b.take(g * nout * 8);
  L.transient = b.off;
  size_t need = 0;
  {  // pair stage
    Bump t;
    t.take(g * JP * 16 * p->b1.w * ncy * c);
    t.take(g * JP * 6 * p->b2.w * ncy * c);
    t.take(g * JP * 6 * b2 * c);
    t.take(g * JP * 6 * 8);
    need = std::max(need, t.off);
  }
  {  // third stage
    Bump t;
    t.take(g * R * R * 16 * p->b1.w * ncy * c);
    t.take(g * R * R * 15 * p->b2.w * ncy * c);
    t.take(g * R * R * 4 * p->b3.w * ncy * c);
    t.take(g * R * R * 4 * b3 * c);
    t.take(g * R * R * 4 * 8);
    need = std::max(need, t.off);
  }
  {  // order-4 stage
    const size_t nf = p->e44_psi ? 4 : 2;
    Bump t;
    t.take(g * R * 19 * p->b1.w * ncy * c);
    t.take(g * R * 18 * p->b2.w * ncy * c);
    t.take(g * R * (nts + 5) * p->b3.w * ncy * c);
    t.take(g * R * nf * p->b4.w * ncy * c);
    t.take(g * R * nf * b4 * c);
    t.take(g * R * nf * 8);
    need = std::max(need, t.off);
  }
  need = std::max(need, (size_t)g * nout * p->b4.w * p->d.ny * c);  // final column transforms
  L.total = L.transient + need;
  return L;
}

extern "C" gl_status gl_eta44_plan_create(gl_plan** out, const gl_eta44_desc* desc) {
  if (!out || !desc) return fail(GL_ERR_INVALID_ARGUMENT, "null plan or descriptor");
  *out = nullptr;
  const gl_eta44_desc& e = *desc;
  if (!is_pow2(e.n) || e.n < 16 || e.n > TW_N)
    return fail(GL_ERR_UNSUPPORTED, "the GPU engine runs power-of-two grids from 16 to %d (got %d)", TW_N, e.n);
  if (!(e.dk > 0) || !(e.depth > 0) || !(e.peak_depth > 0))
    return fail(GL_ERR_INVALID_ARGUMENT, "dk, depth and peak_depth must be positive");
  if (e.rank < 1 || e.rank > MAX_RANK) return fail(GL_ERR_RANK, "rank must be an integer from 1 to %d", MAX_RANK);
  if (e.max_units < 1) return fail(GL_ERR_INVALID_ARGUMENT, "max_units must be >= 1");
  if (e.output != GL_OUT_COMPLEX && e.output != GL_OUT_REAL)
    return fail(GL_ERR_INVALID_ARGUMENT, "unknown output mode");
  if (e.box_w < 1 || e.box_h < 1) return fail(GL_ERR_INVALID_ARGUMENT, "empty parent box");
  if (e.box_x0 < 1) return fail(GL_ERR_SUPPORT, "strict-forward nonzero analytic eta1 support is required");
  const int comps44 = e.components ? e.components : GL_COMP_ETA44;
  if (!(comps44 & GL_COMP_ETA44) || (comps44 & ~(GL_COMP_ETA44 | GL_COMP_PSI44)))
    return fail(GL_ERR_INVALID_ARGUMENT, "fourth-order components: eta44 with optional psi44");
  const bool want_psi = comps44 & GL_COMP_PSI44;
  if (want_psi && !(e.gravity > 0))
    return fail(GL_ERR_INVALID_ARGUMENT, "psi44 needs a positive gravity");
  const int xmax = e.box_x0 + e.box_w - 1;
  const int ymax = std::max(std::abs(e.box_y0), std::abs(e.box_y0 + e.box_h - 1));
  if (4 * xmax >= e.n / 2 || 4 * ymax >= e.n / 2)
    return fail(GL_ERR_ALIAS, "quartic output support reaches a Nyquist boundary");
  gl_plan* p = new gl_plan();
  std::memset(&p->d, 0, sizeof p->d);
  p->d.nx = p->d.ny = e.n;
  p->d.lx = p->d.ly = 6.283185307179586 / e.dk;
  p->d.depth = e.depth;
  p->d.gravity = 1.0;
  p->d.order = 4;
  p->d.max_units = e.max_units;
  p->d.output = e.output;
  p->d.box_x0 = e.box_x0;
  p->d.box_y0 = e.box_y0;
  p->d.box_w = e.box_w;
  p->d.box_h = e.box_h;
  p->e44 = true;
  p->R44 = e.rank;
  p->dk44 = e.dk;
  p->peak44 = e.peak_depth;
  p->comps = 0;
  p->e44_psi = want_psi;
  p->ncomp = want_psi ? 2 : 1;
  p->comp_ids[0] = GL_COMP_ETA44;
  p->comp_ids[1] = GL_COMP_PSI44;
  p->b1 = Box{e.box_x0, e.box_y0, e.box_w, e.box_h};
  p->b2 = Box{2 * e.box_x0, 2 * e.box_y0, 2 * (e.box_w - 1) + 1, 2 * (e.box_h - 1) + 1};
  p->b3 = Box{3 * e.box_x0, 3 * e.box_y0, 3 * (e.box_w - 1) + 1, 3 * (e.box_h - 1) + 1};
  p->b4 = Box{4 * e.box_x0, 4 * e.box_y0, 4 * (e.box_w - 1) + 1, 4 * (e.box_h - 1) + 1};
  p->ww1 = (p->b1.w + 63) / 64;
  p->ww2 = (p->b2.w + 63) / 64;
  p->ww3 = (p->b3.w + 63) / 64;
  p->ncx = std::min(e.n, std::max(16, next_pow2(p->b4.w)));
  p->ncy = std::min(e.n, std::max(16, next_pow2(p->b4.h)));
  p->lncx = ilog2(p->ncx);
  p->lncy = ilog2(p->ncy);
  p->lnx = p->lny = ilog2(e.n);
  // pair and third stages: rows a power of two covering B2 / B3 (the order-4
  // row kernels run powers of two), columns the shortest length covering
  // B2 / B3 that the column kernels run
  p->ncx2 = std::min(p->ncx, std::max(16, next_pow2(p->b2.w)));
  p->ncy2 = std::min(p->ncy, col_len(p->b2.h));
  p->ncx3 = std::min(p->ncx, std::max(16, next_pow2(p->b3.w)));
  p->ncy3 = std::min(p->ncy, col_len(p->b3.h));
  p->lncx2 = col_log2(p->ncx2);
  p->lncy2 = col_log2(p->ncy2);
  p->lncy3 = col_log2(p->ncy3);
  const int row_banks = want_psi ? 46 : 45;
  if (row_smem(row_banks, p->ncx) > ROW_SMEM_LIMIT) {
    plan_free(p);
    return fail(GL_ERR_UNSUPPORTED,
                "eta44 product grid width %d exceeds the shared-memory row budget (%d banks)", p->ncx,
                row_banks);
  }
  p->floor_rel = 16.0 * 2.220446049250313e-16 * std::max(1.0, std::log2((double)e.n * (double)e.n));
  if (e.nodes && e.weights) {
    for (int k = 0; k < e.rank; ++k) {
      p->h_nodes[0][k] = e.nodes[k];
      p->h_weights[0][k] = e.weights[k];
    }
  } else {
    gl_status st = gauss_laguerre(e.rank, p->h_nodes[0], p->h_weights[0]);
    if (st != GL_OK) {
      plan_free(p);
      return st;
    }
  }
  p->h_comp_scale[0] = e.depth;
  p->h_comp_scale[1] = want_psi ? e.depth * std::sqrt(e.gravity * e.depth) : 0.0;
  if (want_psi) p->d.gravity = e.gravity;
  cudaError_t err = cudaSuccess;
  auto geo_alloc = [&](double** g, const Box& b) {
    if (err == cudaSuccess) err = cudaMalloc(g, sizeof(double) * 6 * b.w * b.h);
    if (err == cudaSuccess) {
      const int plane = b.w * b.h;
      geo_kernel<<<std::min(1024, (plane + 255) / 256), 256>>>(*g, b, e.n, e.n, p->d.lx, p->d.ly, e.depth, e.dk);
      err = cudaGetLastError();
    }
  };
  geo_alloc(&p->geo1, p->b1);
  geo_alloc(&p->geo2, p->b2);
  geo_alloc(&p->geo3, p->b3);
  geo_alloc(&p->geo4, p->b4);
  if (err == cudaSuccess) err = cudaMalloc(&p->tw, sizeof(cplx) * TW_ALLOC);
  if (err == cudaSuccess) {
    twiddle_kernel<<<TW_ALLOC / 256 + 1, 256>>>(p->tw, TW_ALLOC);
    err = cudaGetLastError();
  }
  if (err == cudaSuccess) err = cudaMalloc(&p->nodes, sizeof(double) * 2 * MAX_RANK);
  if (err == cudaSuccess) {
    double host[2 * MAX_RANK] = {0};
    std::memcpy(host, p->h_nodes[0], sizeof(double) * MAX_RANK);
    std::memcpy(host + MAX_RANK, p->h_weights[0], sizeof(double) * MAX_RANK);
    err = cudaMemcpy(p->nodes, host, sizeof host, cudaMemcpyHostToDevice);
  }
  if (err == cudaSuccess) err = cudaMalloc(&p->comp_scale, sizeof(double) * 6);
  if (err == cudaSuccess) err = cudaMemcpy(p->comp_scale, p->h_comp_scale, sizeof(double) * 6, cudaMemcpyHostToDevice);
  if (err == cudaSuccess) err = cudaDeviceSynchronize();
  if (err != cudaSuccess) {
    plan_free(p);
    return fail(GL_ERR_CUDA, "eta44 plan set-up failed: %s", cudaGetErrorString(err));
  }
  const int g = e.max_units;
  p->group = g;
  const size_t c = sizeof(cplx);
  const size_t b1 = (size_t)p->b1.w * p->b1.h, b2 = (size_t)p->b2.w * p->b2.h,
               b3 = (size_t)p->b3.w * p->b3.h, b4 = (size_t)p->b4.w * p->b4.h;
  Bump b;
  p->o_slots = b.take(g * sizeof(UnitSlots));
  p->o_us = b.take(g * sizeof(UnitScalars));
  p->o_box = b.take(g * b1 * c);
  p->o_s1 = b.take(g * b1);
  p->o_s1f = b.take((size_t)g * p->b1.h * p->ww1 * 8);
  p->o_s1r = b.take((size_t)g * p->b1.h * p->ww1 * 8);
  p->o_s2 = b.take(g * b2);
  p->o_s2f = b.take((size_t)g * p->b2.h * p->ww2 * 8);
  p->o_s2r = b.take((size_t)g * p->b2.h * p->ww2 * 8);
  p->o_s3 = b.take(g * b3);
  p->o_s3f = b.take((size_t)g * p->b3.h * p->ww3 * 8);
  p->o_s3r = b.take((size_t)g * p->b3.h * p->ww3 * 8);
  p->o_s4 = b.take(g * b4);
  const E44Layout L = e44_layout(p, g);
  p->o_e44 = b.take(L.total);
  p->ws_total = b.off;
  *out = p;
  return GL_OK;
}

// max |x| of the first plane of each unit (units `stride` planes apart) into
// out[u * stride]
__global__ void plane_max_kernel(const cplx* x, int plane, int stride, unsigned long long* out) {
  const int u = blockIdx.y;
  double l = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < plane; i += gridDim.x * blockDim.x) {
    const double m = cabs_(x[(size_t)u * stride * plane + i]);
    l = (m > l || m != m) ? m : l;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double other = __shfl_xor_sync(0xffffffffu, l, o);
    l = (other > l || other != other) ? other : l;
  }
  if ((threadIdx.x & 31) == 0) atomic_max_nonneg(out + (size_t)u * stride, l);
}

// Final roundoff floor of the summed order-4 spectra and transform to the
// reference grid (gl_eta44_fftw.cpp:750-751).
static gl_status e44_finalize(gl_plan* p, int gu, const cplx* OUT, unsigned long long* maxOUT,
                              bool max_ready, void* outputs, char* tr, UnitScalars* us,
                              int* status, cudaStream_t st) {
  const int T = 256;
  const Box B4 = p->b4;
  const int pl4 = B4.w * B4.h;
  const int nout = p->e44_psi ? 2 : 1;  // eta44 [, psi44]: only eta44 is floored
  gl_status s;
  if (!max_ready) {
    CUDA_TRY(cudaMemsetAsync(maxOUT, 0, (size_t)gu * nout * 8, st));
    dim3 g(grid_for(pl4, T, 64), gu);
    {
      LaunchScope ls_("plane_max_kernel", st, 0.0);
      plane_max_kernel<<<g, T, 0, st>>>(OUT, pl4, nout, maxOUT);
    }
    LAUNCH_CHECK("plane_max_kernel");
  }
  ColArgs a;
  std::memset(&a, 0, sizeof a);
  a.kind = COL_FLOORED;
  a.nbanks = nout;
  for (int k = 0; k < nout; ++k) {
    a.mult[k] = M_ONE;
    a.src_of[k] = k;
  }
  a.box = B4;
  a.geo = p->geo4;
  a.spec = OUT;
  a.spec_job_stride = (long long)nout * pl4;
  a.spec_sub_stride = pl4;
  a.jobs_per_unit = 1;
  a.floor_max = maxOUT;  // the psi44 slot stays 0: no floor
  a.floor_nsrc = nout;
  a.floor_rel = p->floor_rel;
  a.out = reinterpret_cast<cplx*>(tr);
  a.n = p->d.ny;
  a.log2n = p->lny;
  a.scale = 1.0 / ((double)p->d.nx * (double)p->d.ny);
  if ((s = launch_col_ifft(a, gu, st, p->tw)) != GL_OK) return s;
  OutArgs o;
  std::memset(&o, 0, sizeof o);
  o.in = reinterpret_cast<cplx*>(tr);
  o.w = B4.w;
  o.x0 = B4.x0;
  o.nx = p->d.nx;
  o.log2nx = p->lnx;
  o.ny = p->d.ny;
  o.ncomp = nout;
  o.comp_offset = 0;
  o.out_ncomp = nout;
  o.comp_scale = p->comp_scale;
  o.out = outputs;
  o.real_only = p->d.output == GL_OUT_REAL;
  o.us = us;  // non-finite outputs set the unit status inside the transform
  if ((s = launch_out_rows(o, gu * nout, st, p->tw)) != GL_OK) return s;
  if (us) {
    if (status) {
      {
        LaunchScope ls_("status_kernel", st, 0.0);
        status_kernel<<<(gu + 63) / 64, 64, 0, st>>>(us, gu, status);
      }
      LAUNCH_CHECK("status_kernel");
    }
  }
  return GL_OK;
}

// One group of units over outer nodes [o0, o0 + Ro).  With `partial` set,
// the accumulated order-4 spectra (before the final floor) are written there
// and nothing else is produced; otherwise the fields are finished.
static gl_status e44_run(gl_plan* p, int gu, const void* spectra, int layout, int o0, int Ro,
                         cplx* partial, void* outputs, void* ws, int* status, cudaStream_t st,
                         int part = -2) {
  const int T = 256, R = p->R44;
  const Box B1 = p->b1, B2 = p->b2, B3 = p->b3, B4 = p->b4;
  const int pl1 = B1.w * B1.h, pl2 = B2.w * B2.h, pl3 = B3.w * B3.h, pl4 = B4.w * B4.h;
  UnitSlots* slots = at<UnitSlots>(ws, p->o_slots);
  UnitScalars* us = at<UnitScalars>(ws, p->o_us);
  cplx* boxv = at<cplx>(ws, p->o_box);
  unsigned char* s1 = at<unsigned char>(ws, p->o_s1);
  unsigned long long* s1f = at<unsigned long long>(ws, p->o_s1f);
  unsigned long long* s1r = at<unsigned long long>(ws, p->o_s1r);
  unsigned char* s2 = at<unsigned char>(ws, p->o_s2);
  unsigned long long* s2f = at<unsigned long long>(ws, p->o_s2f);
  unsigned long long* s2r = at<unsigned long long>(ws, p->o_s2r);
  unsigned char* s3 = at<unsigned char>(ws, p->o_s3);
  unsigned long long* s3f = at<unsigned long long>(ws, p->o_s3f);
  unsigned long long* s3r = at<unsigned long long>(ws, p->o_s3r);
  unsigned char* s4 = at<unsigned char>(ws, p->o_s4);
  char* e44 = at<char>(ws, p->o_e44);
  const E44Layout L = e44_layout(p, p->group);
  cplx* E = reinterpret_cast<cplx*>(e44 + L.E);
  unsigned long long* maxE = reinterpret_cast<unsigned long long*>(e44 + L.maxE);
  cplx* TS = reinterpret_cast<cplx*>(e44 + L.T);
  unsigned long long* maxT = reinterpret_cast<unsigned long long*>(e44 + L.maxT);
  cplx* OUT = partial ? partial : reinterpret_cast<cplx*>(e44 + L.OUT);
  unsigned long long* maxOUT = reinterpret_cast<unsigned long long*>(e44 + L.maxOUT);
  char* tr = e44 + L.transient;
  const double* dn = p->nodes;  // nodes, then weights at +MAX_RANK
  gl_status s;

  // ---- analysis: support, S2..S4, shifts, scales
  {
    LaunchScope ls_("slots_init_kernel", st, 0.0);
    slots_init_kernel<<<(gu + 63) / 64, 64, 0, st>>>(slots, gu);
  }
  LAUNCH_CHECK("slots_init_kernel");
  const cplx* spec = boxv;
  if (layout == GL_SPECTRA_FULL) {
    CUDA_TRY(cudaMemsetAsync(boxv, 0, sizeof(cplx) * (size_t)gu * pl1, st));
    dim3 g(grid_for((size_t)p->d.nx * p->d.ny, T, 1024), gu);
    {
      LaunchScope ls_("extract_kernel", st, 0.0);
      extract_kernel<<<g, T, 0, st>>>(reinterpret_cast<const cplx*>(spectra), boxv, B1, p->d.nx, p->d.ny, slots);
    }
    LAUNCH_CHECK("extract_kernel");
  } else {
    spec = reinterpret_cast<const cplx*>(spectra);
    dim3 g(grid_for(pl1, T, 64), gu);
    {
      LaunchScope ls_("box_max_kernel", st, 0.0);
      box_max_kernel<<<g, T, 0, st>>>(spec, pl1, slots);
    }
    LAUNCH_CHECK("box_max_kernel");
  }
  {
    dim3 g(grid_for(pl1, T, 64), gu);
    {
      LaunchScope ls_("support_kernel", st, 0.0);
      support_kernel<<<g, T, 0, st>>>(spec, p->geo1, B1, slots, s1);
    }
    LAUNCH_CHECK("support_kernel");
    {
      LaunchScope ls_("peak_kernel", st, 0.0);
      peak_kernel<<<g, T, 0, st>>>(spec, p->geo1, B1, p->d.nx, p->d.ny, slots, s1, nullptr, 0);
    }
    LAUNCH_CHECK("peak_kernel");
    dim3 gb(grid_for(B1.h * p->ww1, T, 64), gu);
    {
      LaunchScope ls_("bitrows_kernel", st, 0.0);
      bitrows_kernel<<<gb, T, 0, st>>>(s1, B1.h, B1.w, p->ww1, s1f, s1r);
    }
    LAUNCH_CHECK("bitrows_kernel");
  }
  {
    MinkArgs m;
    mink_args(m, s1f, B1.h, B1.w, p->ww1, s1r, B1.h, B1.w, p->ww1, s2, p->geo2, slots, 2);
    dim3 g2(grid_for(pl2, T, 256), gu);
    {
      LaunchScope ls_("minkowski_kernel", st, 0.0);
      minkowski_kernel<<<g2, T, mink_smem(m), st>>>(m);
    }
    LAUNCH_CHECK("minkowski_kernel");
    dim3 gb(grid_for(B2.h * p->ww2, T, 64), gu);
    {
      LaunchScope ls_("bitrows_kernel", st, 0.0);
      bitrows_kernel<<<gb, T, 0, st>>>(s2, B2.h, B2.w, p->ww2, s2f, s2r);
    }
    LAUNCH_CHECK("bitrows_kernel");
    mink_args(m, s2f, B2.h, B2.w, p->ww2, s1r, B1.h, B1.w, p->ww1, s3, p->geo3, slots, 3);
    dim3 g3(grid_for(pl3, T, 512), gu);
    {
      LaunchScope ls_("minkowski_kernel", st, 0.0);
      minkowski_kernel<<<g3, T, mink_smem(m), st>>>(m);
    }
    LAUNCH_CHECK("minkowski_kernel");
    dim3 gb3(grid_for(B3.h * p->ww3, T, 64), gu);
    {
      LaunchScope ls_("bitrows_kernel", st, 0.0);
      bitrows_kernel<<<gb3, T, 0, st>>>(s3, B3.h, B3.w, p->ww3, s3f, s3r);
    }
    LAUNCH_CHECK("bitrows_kernel");
    mink_args(m, s3f, B3.h, B3.w, p->ww3, s1r, B1.h, B1.w, p->ww1, s4, p->geo4, slots, 4);
    dim3 g4(grid_for(pl4, T, 512), gu);
    {
      LaunchScope ls_("minkowski_kernel", st, 0.0);
      minkowski_kernel<<<g4, T, mink_smem(m), st>>>(m);
    }
    LAUNCH_CHECK("minkowski_kernel");
  }
  {
    ScalarArgs a;
    std::memset(&a, 0, sizeof a);
    a.slots = slots;
    a.us = us;
    a.geo1 = p->geo1;
    a.box = B1;
    a.nx = p->d.nx;
    a.ny = p->d.ny;
    a.order = 4;
    a.full_input = layout == GL_SPECTRA_FULL;
    a.want_e44 = 1;
    a.fixed_peak = p->peak44;
    {
      LaunchScope ls_("scalars_kernel", st, 0.0);
      scalars_kernel<<<(gu + 63) / 64, 64, 0, st>>>(a, gu);
    }
    LAUNCH_CHECK("scalars_kernel");
  }
  const double inv_scale = 1.0 / ((double)p->d.nx * (double)p->d.ny);
  // Product grid of each stage: the pair stage only forms products of two
  // first-order fields and the third stage of three, so they run on grids
  // covering B2 and B3 (rows a power of two, columns a power of two or a
  // mixed length 16 m); the order-4 stage on the plan's grid covering B4.
  struct StageGrid {
    int nx, lnx, ny, lny;
    double fwd;  // (Nx Ny)/(nx ny): forward-transform scale
  };
  auto stage_grid = [&](int nx, int ny) {
    return StageGrid{nx, col_log2(nx), ny, col_log2(ny),
                     ((double)p->d.nx * (double)p->d.ny) / ((double)nx * (double)ny)};
  };
  StageGrid cur = stage_grid(p->ncx, p->ncy);
  const int JP = Ro * R * R + Ro * R, GP = Ro * R + Ro;
  const bool psi = p->e44_psi;
  const int nts = psi ? 4 : 3;   // third-state spectra: es, ps, pts [, ets]
  const int nf4 = psi ? 4 : 2;   // order-4 rows: fk, fd [, contact, contact_t]
  const int nout = psi ? 2 : 1;  // accumulated spectra: eta44 [, psi44]
  CUDA_TRY(cudaMemsetAsync(maxE, 0, (size_t)gu * GP * 5 * 8, st));
  CUDA_TRY(cudaMemsetAsync(maxT, 0, (size_t)gu * R * nts * 8, st));
  CUDA_TRY(cudaMemsetAsync(maxOUT, 0, (size_t)gu * nout * 8, st));

  auto colargs = [&](int kind, int nb, const int* mults, const int* srcs, const Box& box,
                     const double* geo, const cplx* sp, long long job_stride, long long sub_stride,
                     int jobs_per_unit, cplx* outp) {
    ColArgs a;
    std::memset(&a, 0, sizeof a);
    a.kind = kind;
    int src[MAX_BANKS];
    for (int k = 0; k < nb; ++k) src[k] = srcs ? srcs[k] : 0;
    set_banks(a, nb, mults, src);  // qx-multiple banks become twins
    a.box = box;
    a.geo = geo;
    a.spec = sp;
    a.spec_job_stride = job_stride;
    a.spec_sub_stride = sub_stride;
    a.jobs_per_unit = jobs_per_unit;
    a.us = us;
    a.nodes = dn;
    a.n_inner = R;
    a.n_outer = Ro;
    a.outer0 = o0;
    a.floor_rel = p->floor_rel;
    a.out = outp;
    a.n = cur.ny;
    a.log2n = cur.lny;
    a.scale = inv_scale;
    return a;
  };
  auto rowargs = [&](int kind, int nout, const Box& outbox, cplx* outp) {
    RowArgs r;
    std::memset(&r, 0, sizeof r);
    r.kind = kind;
    r.nout = nout;
    r.out_x0 = outbox.x0;
    r.out_w = outbox.w;
    r.out = outp;
    r.nx = cur.nx;
    r.log2nx = cur.lnx;
    r.ny = cur.ny;
    r.us = us;
    r.jobs_per_unit = 1;
    r.gmax = ROW_GMAX;
    return r;
  };
  auto colfft = [&](const cplx* in, cplx* outp, const Box& box, int nsrc, const unsigned char* mask,
                    unsigned long long* mx, int jobs_per_unit, int njs) {
    ColFftArgs f;
    f.in = in;
    f.out = outp;
    f.box = box;
    f.n = cur.ny;
    f.log2n = cur.lny;
    f.nsrc = nsrc;
    f.jobs_per_unit = jobs_per_unit;
    f.mask = mask;
    f.maxslot = mx;
    f.scale = cur.fwd;
    return launch_col_fft(f, njs, st, p->tw);
  };

  // ---- stage 1: every pair level (Ro R^2 third-level + Ro R order-4 pair jobs)
  cur = stage_grid(p->ncx2, p->ncy2);
  {
    const int nj = gu * JP;
    Bump b;
    cplx* P = reinterpret_cast<cplx*>(tr + b.take((size_t)nj * 16 * B1.w * cur.ny * sizeof(cplx)));
    cplx* Q = reinterpret_cast<cplx*>(tr + b.take((size_t)nj * 6 * B2.w * cur.ny * sizeof(cplx)));
    cplx* RP = reinterpret_cast<cplx*>(tr + b.take((size_t)nj * 6 * pl2 * sizeof(cplx)));
    unsigned long long* mRP = reinterpret_cast<unsigned long long*>(tr + b.take((size_t)nj * 6 * 8));
    CUDA_TRY(cudaMemsetAsync(mRP, 0, (size_t)nj * 6 * 8, st));
    ColArgs a = colargs(COL_E44_PAIR, 16, E44_PAIR_MULT, nullptr, B1, p->geo1, spec, pl1, 0, JP, P);
    if ((s = launch_col_ifft(a, nj, st, p->tw)) != GL_OK) return s;
    RowArgs r = rowargs(ROW_E44_PAIR, 6, B2, Q);
    r.grp[0] = BankGroup{P, 16, B1.x0, B1.w};
    r.ngrp = 1;
    if ((s = launch_row(r, nj, st, p->tw)) != GL_OK) return s;
    if ((s = colfft(Q, RP, B2, 6, s2, mRP, JP, nj * 6)) != GL_OK) return s;
    E44Acc c;
    std::memset(&c, 0, sizeof c);
    c.us = us;
    c.geo = p->geo2;
    c.box = B2;
    c.in = RP;
    c.maxin = mRP;
    c.out = E;
    c.maxout = maxE;
    c.nodes = dn;
    c.weights = dn + MAX_RANK;
    c.R = R;
    c.groups_per_unit = GP;
    c.jobs_per_unit = JP;
    c.Ro = Ro;
    c.outer0 = o0;
    c.floor_rel = p->floor_rel;
    dim3 g(grid_for(pl2, T, 64), gu * GP);
    {
      LaunchScope ls_("acc_e44_pair_kernel", st, 0.0);
      acc_e44_pair_kernel<<<g, T, 0, st>>>(c);
    }
    LAUNCH_CHECK("acc_e44_pair_kernel");
  }
  // ---- stage 2: third level (Ro R jobs per unit); the split mode's base part
  // (part -1) has no third state, and part t >= 0 sums third-level node t alone
  cur = stage_grid(p->ncx3, p->ncy3);
  if (part == -1) {
    CUDA_TRY(cudaMemsetAsync(TS, 0, sizeof(cplx) * (size_t)gu * Ro * nts * pl3, st));
    CUDA_TRY(cudaMemsetAsync(maxT, 0, (size_t)gu * Ro * nts * 8, st));
  } else {
    const int nj = gu * Ro * R;
    Bump b;
    cplx* PF = reinterpret_cast<cplx*>(tr + b.take((size_t)nj * 16 * B1.w * cur.ny * sizeof(cplx)));
    cplx* PP = reinterpret_cast<cplx*>(tr + b.take((size_t)nj * 15 * B2.w * cur.ny * sizeof(cplx)));
    cplx* Q = reinterpret_cast<cplx*>(tr + b.take((size_t)nj * 4 * B3.w * cur.ny * sizeof(cplx)));
    cplx* R3 = reinterpret_cast<cplx*>(tr + b.take((size_t)nj * 4 * pl3 * sizeof(cplx)));
    unsigned long long* mR3 = reinterpret_cast<unsigned long long*>(tr + b.take((size_t)nj * 4 * 8));
    CUDA_TRY(cudaMemsetAsync(mR3, 0, (size_t)nj * 4 * 8, st));
    ColArgs a = colargs(COL_E44_FIRST3, 16, E44_FIRST_MULT, nullptr, B1, p->geo1, spec, pl1, 0, Ro * R, PF);
    if ((s = launch_col_ifft(a, nj, st, p->tw)) != GL_OK) return s;
    // pair outputs of third-level groups: group g = ol R + t of unit u sits at
    // E[u GP + g] and job (u, ol, t) = u Ro R + ol R + t.
    for (int u = 0; u < gu; ++u) {
      ColArgs a2 = colargs(COL_FLOORED, 15, E44_POUT_MULT, E44_POUT_SRC, B2, p->geo2,
                           E + (size_t)u * GP * 5 * pl2, 5LL * pl2, pl2, Ro * R,
                           PP + (size_t)u * Ro * R * 15 * B2.w * cur.ny);
      a2.floor_max = maxE + (size_t)u * GP * 5;
      a2.floor_nsrc = 5;
      if ((s = launch_col_ifft(a2, Ro * R, st, p->tw)) != GL_OK) return s;
    }
    RowArgs r = rowargs(ROW_E44_THIRD, 4, B3, Q);
    r.grp[0] = BankGroup{PF, 16, B1.x0, B1.w};
    r.grp[1] = BankGroup{PP, 15, B2.x0, B2.w};
    r.ngrp = 2;
    if ((s = launch_row(r, nj, st, p->tw)) != GL_OK) return s;
    if ((s = colfft(Q, R3, B3, 4, s3, mR3, Ro * R, nj * 4)) != GL_OK) return s;
    E44Acc c;
    std::memset(&c, 0, sizeof c);
    c.us = us;
    c.geo = p->geo3;
    c.box = B3;
    c.in = R3;
    c.maxin = mR3;
    c.out = TS;
    c.maxout = maxT;
    c.nodes = dn;
    c.weights = dn + MAX_RANK;
    c.R = R;
    c.groups_per_unit = Ro;
    c.Ro = Ro;
    c.outer0 = o0;
    c.floor_rel = p->floor_rel;
    c.nspec = nts;
    c.only_t1 = part >= 0 ? part + 1 : 0;
    dim3 g(grid_for(pl3, T, 64), gu * Ro);
    {
      LaunchScope ls_("acc_e44_third_kernel", st, 0.0);
      acc_e44_third_kernel<<<g, T, 0, st>>>(c);
    }
    LAUNCH_CHECK("acc_e44_third_kernel");
  }
  // ---- stage 3: order-4 forcing (Ro jobs per unit)
  cur = stage_grid(p->ncx, p->ncy);
  {
    const int nj = gu * Ro;
    Bump b;
    cplx* PF = reinterpret_cast<cplx*>(tr + b.take((size_t)nj * 19 * B1.w * cur.ny * sizeof(cplx)));
    cplx* PP = reinterpret_cast<cplx*>(tr + b.take((size_t)nj * 18 * B2.w * cur.ny * sizeof(cplx)));
    const int ntb = nts + 5;  // third-state banks (8, or 9 with eta_t)
    cplx* PT = reinterpret_cast<cplx*>(tr + b.take((size_t)nj * ntb * B3.w * cur.ny * sizeof(cplx)));
    cplx* Q = reinterpret_cast<cplx*>(tr + b.take((size_t)nj * nf4 * B4.w * cur.ny * sizeof(cplx)));
    cplx* R4 = reinterpret_cast<cplx*>(tr + b.take((size_t)nj * nf4 * pl4 * sizeof(cplx)));
    unsigned long long* mR4 = reinterpret_cast<unsigned long long*>(tr + b.take((size_t)nj * nf4 * 8));
    CUDA_TRY(cudaMemsetAsync(mR4, 0, (size_t)nj * nf4 * 8, st));
    ColArgs a = colargs(COL_E44_FIRST4, 19, E44_FIRST_MULT, nullptr, B1, p->geo1, spec, pl1, 0, Ro, PF);
    if ((s = launch_col_ifft(a, nj, st, p->tw)) != GL_OK) return s;
    for (int u = 0; u < gu; ++u) {
      ColArgs a2 = colargs(COL_FLOORED, 18, E44_POUT_MULT, E44_POUT_SRC, B2, p->geo2,
                           E + ((size_t)u * GP + Ro * R) * 5 * pl2, 5LL * pl2, pl2, Ro,
                           PP + (size_t)u * Ro * 18 * B2.w * cur.ny);
      a2.floor_max = maxE + ((size_t)u * GP + Ro * R) * 5;
      a2.floor_nsrc = 5;
      if ((s = launch_col_ifft(a2, Ro, st, p->tw)) != GL_OK) return s;
    }
    ColArgs a3 = colargs(COL_FLOORED, ntb, E44_TOUT_MULT, E44_TOUT_SRC, B3, p->geo3, TS,
                         (long long)nts * pl3, pl3, Ro, PT);
    a3.floor_max = maxT;
    a3.floor_nsrc = nts;
    if ((s = launch_col_ifft(a3, nj, st, p->tw)) != GL_OK) return s;
    RowArgs r = rowargs(psi ? ROW_E44_ORDER4_PSI : ROW_E44_ORDER4, nf4, B4, Q);
    r.e44_part = part == -1 ? 1 : part >= 0 ? 2 : 0;
    r.grp[0] = BankGroup{PF, 19, B1.x0, B1.w};
    r.grp[1] = BankGroup{PP, 18, B2.x0, B2.w};
    r.grp[2] = BankGroup{PT, ntb, B3.x0, B3.w};
    r.ngrp = 3;
    if ((s = launch_row(r, nj, st, p->tw)) != GL_OK) return s;
    if ((s = colfft(Q, R4, B4, nf4, s4, mR4, Ro, nj * nf4)) != GL_OK) return s;
    E44Acc c;
    std::memset(&c, 0, sizeof c);
    c.us = us;
    c.geo = p->geo4;
    c.box = B4;
    c.in = R4;
    c.maxin = mR4;
    c.out = OUT;
    c.maxout = maxOUT;
    c.nodes = dn;
    c.weights = dn + MAX_RANK;
    c.R = R;
    c.groups_per_unit = 1;
    c.Ro = Ro;
    c.outer0 = o0;
    c.floor_rel = p->floor_rel;
    c.nspec = nf4;
    dim3 g(grid_for(pl4, T, 64), gu);
    {
      LaunchScope ls_("acc_e44_order4_kernel", st, 0.0);
      acc_e44_order4_kernel<<<g, T, 0, st>>>(c);
    }
    LAUNCH_CHECK("acc_e44_order4_kernel");
  }
  if (partial) return GL_OK;
  return e44_finalize(p, gu, OUT, maxOUT, true, outputs, tr, us, status, st);
}

static gl_status run_group_eta44(gl_plan* p, int gu, const void* spectra, int layout,
                                 void* outputs, void* ws, int* status, cudaStream_t st) {
  return e44_run(p, gu, spectra, layout, 0, p->R44, nullptr, outputs, ws, status, st);
  return GL_OK;
}

extern "C" gl_status gl_eta44_execute_partial(gl_plan* p, int n_units, const void* d_spectra,
                                              int layout, int outer_begin, int outer_end,
                                              void* d_partial, void* d_ws, size_t ws_bytes,
                                              int* d_status, void* stream) {
  if (!p || !p->e44) return fail(GL_ERR_INVALID_ARGUMENT, "not an eta44 plan");
  if (n_units < 0 || !d_spectra || !d_partial) return fail(GL_ERR_INVALID_ARGUMENT, "bad arguments");
  if (outer_begin < 0 || outer_end > p->R44 || outer_begin >= outer_end)
    return fail(GL_ERR_INVALID_ARGUMENT, "outer node range must lie in [0, rank)");
  if (layout != GL_SPECTRA_FULL && layout != GL_SPECTRA_BOX)
    return fail(GL_ERR_INVALID_ARGUMENT, "unknown spectra layout");
  if (!d_ws || ws_bytes < p->ws_total || (reinterpret_cast<uintptr_t>(d_ws) & 255))
    return fail(GL_ERR_WORKSPACE, "workspace must be 256-byte aligned and at least %zu bytes", p->ws_total);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const size_t in_unit = layout == GL_SPECTRA_FULL ? (size_t)p->d.nx * p->d.ny : (size_t)p->b1.w * p->b1.h;
  const size_t part_unit = (size_t)p->ncomp * p->b4.w * p->b4.h;
  for (int u0 = 0; u0 < n_units; u0 += p->group) {
    const int gu = std::min(p->group, n_units - u0);
    gl_status s = e44_run(p, gu, reinterpret_cast<const cplx*>(d_spectra) + (size_t)u0 * in_unit, layout,
                          outer_begin, outer_end - outer_begin,
                          reinterpret_cast<cplx*>(d_partial) + (size_t)u0 * part_unit, nullptr, d_ws,
                          d_status ? d_status + u0 : nullptr, st);
    if (s != GL_OK) return s;
    if (d_status) {
      UnitScalars* us = at<UnitScalars>(d_ws, p->o_us);
      {
        LaunchScope ls_("status_kernel", st, 0.0);
        status_kernel<<<(gu + 63) / 64, 64, 0, st>>>(us, gu, d_status + u0);
      }
      LAUNCH_CHECK("status_kernel");
    }
  }
  return GL_OK;
}

extern "C" gl_status gl_eta44_execute_part(gl_plan* p, int n_units, const void* d_spectra, int layout,
                                           int outer_index, int part_index, void* d_partial, void* d_ws,
                                           size_t ws_bytes, int* d_status, void* stream) {
  if (!p || !p->e44) return fail(GL_ERR_INVALID_ARGUMENT, "not an eta44 plan");
  if (p->e44_psi) return fail(GL_ERR_UNSUPPORTED, "the split mode computes eta44 only");
  if (outer_index < 0 || outer_index >= p->R44) return fail(GL_ERR_INVALID_ARGUMENT, "outer index");
  if (part_index >= p->R44 || part_index < -2) return fail(GL_ERR_INVALID_ARGUMENT, "part index");
  if (n_units < 0 || !d_spectra || !d_partial) return fail(GL_ERR_INVALID_ARGUMENT, "bad arguments");
  if (layout != GL_SPECTRA_FULL && layout != GL_SPECTRA_BOX)
    return fail(GL_ERR_INVALID_ARGUMENT, "unknown spectra layout");
  if (!d_ws || ws_bytes < p->ws_total || (reinterpret_cast<uintptr_t>(d_ws) & 255))
    return fail(GL_ERR_WORKSPACE, "workspace must be 256-byte aligned and at least %zu bytes", p->ws_total);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const size_t in_unit = layout == GL_SPECTRA_FULL ? (size_t)p->d.nx * p->d.ny : (size_t)p->b1.w * p->b1.h;
  const size_t part_unit = (size_t)p->ncomp * p->b4.w * p->b4.h;
  for (int u0 = 0; u0 < n_units; u0 += p->group) {
    const int gu = std::min(p->group, n_units - u0);
    gl_status s = e44_run(p, gu, reinterpret_cast<const cplx*>(d_spectra) + (size_t)u0 * in_unit, layout,
                          outer_index, 1, reinterpret_cast<cplx*>(d_partial) + (size_t)u0 * part_unit,
                          nullptr, d_ws, d_status ? d_status + u0 : nullptr, st, part_index);
    if (s != GL_OK) return s;
    if (d_status) {
      UnitScalars* us = at<UnitScalars>(d_ws, p->o_us);
      {
        LaunchScope ls_("status_kernel", st, 0.0);
        status_kernel<<<(gu + 63) / 64, 64, 0, st>>>(us, gu, d_status + u0);
      }
      LAUNCH_CHECK("status_kernel");
    }
  }
  return GL_OK;
}

extern "C" gl_status gl_eta44_finalize(gl_plan* p, int n_units, const void* d_partial_sum,
                                       void* d_outputs, void* d_ws, size_t ws_bytes, void* stream) {
  if (!p || !p->e44) return fail(GL_ERR_INVALID_ARGUMENT, "not an eta44 plan");
  if (n_units < 0 || !d_partial_sum || !d_outputs) return fail(GL_ERR_INVALID_ARGUMENT, "bad arguments");
  if (!d_ws || ws_bytes < p->ws_total || (reinterpret_cast<uintptr_t>(d_ws) & 255))
    return fail(GL_ERR_WORKSPACE, "workspace must be 256-byte aligned and at least %zu bytes", p->ws_total);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  char* e44 = at<char>(d_ws, p->o_e44);
  const E44Layout L = e44_layout(p, p->group);
  unsigned long long* maxOUT = reinterpret_cast<unsigned long long*>(e44 + L.maxOUT);
  const size_t part_unit = (size_t)p->ncomp * p->b4.w * p->b4.h;
  const size_t out_unit = (size_t)p->ncomp * p->d.nx * p->d.ny *
                          (p->d.output == GL_OUT_REAL ? sizeof(double) : sizeof(cplx));
  for (int u0 = 0; u0 < n_units; u0 += p->group) {
    const int gu = std::min(p->group, n_units - u0);
    gl_status s = e44_finalize(p, gu, reinterpret_cast<const cplx*>(d_partial_sum) + (size_t)u0 * part_unit,
                               maxOUT, false, reinterpret_cast<char*>(d_outputs) + u0 * out_unit,
                               e44 + L.transient, nullptr, nullptr, st);
    if (s != GL_OK) return s;
  }
  return GL_OK;
}

extern "C" gl_status gl_execute(gl_plan* p, int n_units, const void* d_spectra, int layout,
                                void* d_outputs, void* d_ws, size_t ws_bytes, int* d_status,
                                void* stream) {
  if (!p) return fail(GL_ERR_INVALID_ARGUMENT, "null plan");
  if (n_units < 0) return fail(GL_ERR_INVALID_ARGUMENT, "negative unit count");
  if (n_units == 0) return GL_OK;
  if (!d_spectra || !d_outputs) return fail(GL_ERR_INVALID_ARGUMENT, "null spectra or outputs");
  if (layout != GL_SPECTRA_FULL && layout != GL_SPECTRA_BOX)
    return fail(GL_ERR_INVALID_ARGUMENT, "unknown spectra layout");
  if (!d_ws || ws_bytes < p->ws_total || (reinterpret_cast<uintptr_t>(d_ws) & 255))
    return fail(GL_ERR_WORKSPACE, "workspace must be 256-byte aligned and at least %zu bytes", p->ws_total);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const size_t in_unit = layout == GL_SPECTRA_FULL ? (size_t)p->d.nx * p->d.ny
                                                   : (size_t)p->b1.w * p->b1.h;
  const size_t out_unit = (size_t)p->ncomp * p->d.nx * p->d.ny *
                          (p->d.output == GL_OUT_REAL ? sizeof(double) : sizeof(cplx));
  const int ngroups = (n_units + p->group - 1) / p->group;
  const int L = std::min(p->lanes, ngroups);
  if (L <= 1) {
    for (int u0 = 0; u0 < n_units; u0 += p->group) {
      const int gu = std::min(p->group, n_units - u0);
      const void* in = reinterpret_cast<const cplx*>(d_spectra) + (size_t)u0 * in_unit;
      void* outp = reinterpret_cast<char*>(d_outputs) + (size_t)u0 * out_unit;
      gl_status s = run_group(p, gu, in, layout, outp, d_ws, d_status ? d_status + u0 : nullptr, st);
      if (s != GL_OK) return s;
    }
    return GL_OK;
  }
  // concurrent lanes: group i runs on lane i mod L in that lane's workspace
  // region; the lanes start after the work already on the caller's stream and
  // the caller's stream continues after all of them (also inside a stream
  // capture, where this is a fork/join of graph branches)
  std::lock_guard<std::mutex> lk(p->lane_mu);
  CUDA_TRY(cudaEventRecord(p->lane_ev[0], st));
  for (int l = 1; l < L; ++l) CUDA_TRY(cudaStreamWaitEvent(p->lane_st[l], p->lane_ev[0], 0));
  gl_status s = GL_OK;
  for (int gi = 0; gi < ngroups && s == GL_OK; ++gi) {
    const int l = gi % L;
    const int u0 = gi * p->group;
    const int gu = std::min(p->group, n_units - u0);
    const void* in = reinterpret_cast<const cplx*>(d_spectra) + (size_t)u0 * in_unit;
    void* outp = reinterpret_cast<char*>(d_outputs) + (size_t)u0 * out_unit;
    void* ws = reinterpret_cast<char*>(d_ws) + (size_t)l * p->lane_bytes;
    s = run_group(p, gu, in, layout, outp, ws, d_status ? d_status + u0 : nullptr,
                  l == 0 ? st : p->lane_st[l]);
  }
  // joined even after a failed launch, so that the caller's stream never runs
  // ahead of lane work already queued
  for (int l = 1; l < L; ++l) {
    const cudaError_t e1 = cudaEventRecord(p->lane_ev[l], p->lane_st[l]);
    const cudaError_t e2 = e1 == cudaSuccess ? cudaStreamWaitEvent(st, p->lane_ev[l], 0) : e1;
    if (e2 != cudaSuccess && s == GL_OK) s = fail(GL_ERR_CUDA, "lane join: %s", cudaGetErrorString(e2));
  }
  return s;
}

// ---------------------------------------------------------------------------
// adjoint (reverse-mode) pass: gradient of a real loss of the eta components
// ---------------------------------------------------------------------------
//
// The backward pass keeps no tape from the forward call: it re-runs the
// analysis and the forward node stages it needs (to recover the node fields
// and the roundoff-floor decisions) and then runs every stage transposed.
// Stage buffers live only inside one call.

struct AdjLayout {
  size_t e1, e2, e3, da22, da1, dai, stage, total;  // offsets from the scratch base
};

static bool adj_eta22(const gl_plan* p) { return (p->comps & GL_COMP_ETA22) != 0; }
static bool adj_eta33(const gl_plan* p) { return (p->comps & GL_COMP_ETA33) != 0; }

struct AdjStage22 {
  size_t P, Q, R, mx, RA, QA, end;
};
struct AdjStage33 {
  size_t E, mxs, PI, QI, RI, maxRI, P1, P2, QO, RO, RAo, QA1, QA2, EA, RAi, QAi, end;
};

static AdjStage22 adj_stage22(const gl_plan* p, size_t base, int g) {
  const size_t c = sizeof(cplx), ncy = p->ncy, pl2 = (size_t)p->b2.w * p->b2.h;
  const size_t nj = (size_t)g * p->ranks[0];
  Bump b;
  b.off = base;
  AdjStage22 s;
  s.P = b.take(nj * 8 * p->b1.w * ncy * c);
  s.Q = b.take(nj * 2 * p->b2.w * ncy * c);  // also the adjoint columns
  s.R = b.take(nj * 2 * pl2 * c);
  s.mx = b.take(nj * 2 * 8);
  s.RA = b.take(nj * 2 * pl2 * c);
  s.QA = b.take(nj * 8 * p->b1.w * ncy * c);
  s.end = b.off;
  return s;
}

static AdjStage33 adj_stage33(const gl_plan* p, size_t base, int g) {
  const size_t c = sizeof(cplx), ncy = p->ncy;
  const size_t pl2 = (size_t)p->b2.w * p->b2.h, pl3 = (size_t)p->b3.w * p->b3.h;
  const size_t nuj = (size_t)g * p->ranks[3], nj = nuj * p->ranks[2];
  Bump b;
  b.off = base;
  AdjStage33 s;
  s.E = b.take(nuj * 4 * pl2 * c);
  s.mxs = b.take(nuj * 3 * 8);                       // eta_t max [nuj], forcing maxima [nuj][2]
  s.PI = b.take(nj * 12 * p->b1.w * ncy * c);
  s.QI = b.take(nj * 4 * p->b2.w * ncy * c);         // also the inner adjoint columns
  s.RI = b.take(nj * 4 * pl2 * c);
  s.maxRI = b.take(nj * 4 * 8);
  s.P1 = b.take(nuj * 12 * p->b1.w * ncy * c);
  s.P2 = b.take(nuj * 9 * p->b2.w * ncy * c);
  s.QO = b.take(nuj * 2 * p->b3.w * ncy * c);        // also the outer adjoint columns
  s.RO = b.take(nuj * 2 * pl3 * c);
  s.RAo = b.take(nuj * 2 * pl3 * c);
  s.QA1 = b.take(nuj * 12 * p->b1.w * ncy * c);
  s.QA2 = b.take(nuj * 8 * p->b2.w * ncy * c);
  s.EA = b.take(nuj * 4 * pl2 * c);
  s.RAi = b.take(nj * 4 * pl2 * c);
  s.QAi = b.take(nj * 12 * p->b1.w * ncy * c);
  s.end = b.off;
  return s;
}

static AdjLayout adj_layout(const gl_plan* p, int g) {
  const size_t c = sizeof(cplx);
  const size_t pl1 = (size_t)p->b1.w * p->b1.h, pl2 = (size_t)p->b2.w * p->b2.h,
               pl3 = (size_t)p->b3.w * p->b3.h;
  const bool e22 = adj_eta22(p), e33 = adj_eta33(p);
  AdjLayout L;
  Bump b;
  L.e1 = b.take((size_t)g * pl1 * c);
  L.e2 = b.take(e22 ? (size_t)g * pl2 * c : 0);
  L.e3 = b.take(e33 ? (size_t)g * pl3 * c : 0);
  L.da22 = b.take(e22 ? (size_t)g * p->ranks[0] * pl1 * c : 0);
  L.da1 = b.take(e33 ? (size_t)g * p->ranks[3] * pl1 * c : 0);
  L.dai = b.take(e33 ? (size_t)g * p->ranks[3] * p->ranks[2] * pl1 * c : 0);
  L.stage = b.off;
  const size_t wmax = std::max({(size_t)p->b1.w, (size_t)p->b2.w, (size_t)p->b3.w});
  size_t end = L.stage + align_up((size_t)g * p->d.ny * wmax * c);  // seed rows
  if (e22) end = std::max(end, adj_stage22(p, L.stage, g).end);
  if (e33) end = std::max(end, adj_stage33(p, L.stage, g).end);
  L.total = end;
  return L;
}

static gl_status adj_check_plan(const gl_plan* p) {
  if (!p) return fail(GL_ERR_INVALID_ARGUMENT, "null plan");
  if (p->e44) return fail(GL_ERR_UNSUPPORTED, "the adjoint covers the eta11/eta22/eta33 graph only");
  if (p->gen) return fail(GL_ERR_UNSUPPORTED, "the adjoint runs power-of-two reference grids only");
  if (!(p->comps & (GL_COMP_ETA11 | GL_COMP_ETA22 | GL_COMP_ETA33)))
    return fail(GL_ERR_INVALID_ARGUMENT, "the plan has no eta component to differentiate");
  if (adj_eta33(p) && row_smem(23, p->ncx) > ROW_SMEM_LIMIT)
    return fail(GL_ERR_UNSUPPORTED, "the order-3 adjoint row exceeds the shared-memory budget at %d columns",
                p->ncx);
  return GL_OK;
}

extern "C" gl_status gl_adjoint_workspace_size(const gl_plan* p, size_t* bytes) {
  gl_status s = adj_check_plan(p);
  if (s != GL_OK) return s;
  if (!bytes) return fail(GL_ERR_INVALID_ARGUMENT, "null size pointer");
  *bytes = p->o_scratch + adj_layout(p, p->group).total;
  return GL_OK;
}

// Ebar of one output box from the residual: + sign transforms, h/(Nx Ny).
static gl_status adj_seed(gl_plan* p, int gu, const double* resid, const Box& box, cplx* rows,
                          cplx* out, cudaStream_t st) {
  SeedArgs sa;
  sa.r = resid;
  sa.nx = p->d.nx;
  sa.log2nx = p->lnx;
  sa.ny = p->d.ny;
  sa.x0 = box.x0;
  sa.w = box.w;
  sa.out = rows;
  gl_status s = launch_seed_rows(sa, gu, st, p->tw);
  if (s != GL_OK) return s;
  ColFftArgs f;
  f.in = rows;
  f.out = out;
  f.box = box;
  f.n = p->d.ny;
  f.log2n = p->lny;
  f.nsrc = 1;
  f.jobs_per_unit = 1;
  f.mask = nullptr;
  f.maxslot = nullptr;
  f.scale = p->d.depth / ((double)p->d.nx * (double)p->d.ny);
  f.conj_io = 1;
  return launch_col_fft(f, gu, st, p->tw);
}

// Adjoint column stage: + or - sign column transforms of `nb` adjoint
// spectra per job (COL_PLAIN, the transposed forward transform).
// Product grid of one adjoint segment (column transform -> rows -> column
// combine): the pair stages run on (ncx2, ncy2), the triple stage on
// (ncx, ncy3), like the forward stages they transpose.
struct AdjGrid {
  int nx, lnx, ny, lny;
};

static gl_status adj_cols(gl_plan* p, const AdjGrid& gr, const Box& box, const double* geo,
                          const cplx* spec, int nb, int njobs, cplx* out, cudaStream_t st) {
  ColArgs a;
  std::memset(&a, 0, sizeof a);
  a.kind = COL_PLAIN;
  a.nbanks = nb;
  for (int k = 0; k < nb; ++k) {
    a.mult[k] = M_ONE;
    a.src_of[k] = k;
  }
  a.box = box;
  a.geo = geo;
  a.spec = spec;
  a.spec_job_stride = (long long)nb * box.w * box.h;
  a.spec_sub_stride = (long long)box.w * box.h;
  a.jobs_per_unit = 1;
  a.out = out;
  a.n = gr.ny;
  a.log2n = gr.lny;
  a.scale = ((double)p->d.nx * (double)p->d.ny) / ((double)gr.nx * (double)gr.ny);
  a.conj_io = 1;
  return launch_col_ifft(a, njobs, st, p->tw);
}

static CmbArgs cmb_args(gl_plan* p, const AdjGrid& gr, int kind, int nb, const int* mults,
                        const int* dsts, int nout, const Box& box, const double* geo, const cplx* in,
                        cplx* out, const UnitScalars* us, int jobs_per_unit) {
  CmbArgs a;
  std::memset(&a, 0, sizeof a);
  a.kind = kind;
  a.nbanks = nb;
  for (int k = 0; k < nb; ++k) {
    a.mult[k] = mults[k];
    a.dst_of[k] = dsts ? dsts[k] : 0;
  }
  a.nout = nout;
  a.box = box;
  a.geo = geo;
  a.in = in;
  a.out = out;
  a.n = gr.ny;
  a.log2n = gr.lny;
  a.scale = 1.0 / ((double)p->d.nx * (double)p->d.ny);
  a.us = us;
  a.jobs_per_unit = jobs_per_unit;
  return a;
}

static gl_status run_adjoint_group(gl_plan* p, int gu, const void* spectra, int layout,
                                   const double* resid, cplx* grad, void* ws, int* status,
                                   cudaStream_t st) {
  const int T = 256;
  const Box B1 = p->b1, B2 = p->b2, B3 = p->b3;
  const int pl1 = B1.w * B1.h, pl2 = B2.w * B2.h, pl3 = B3.w * B3.h;
  UnitScalars* us = at<UnitScalars>(ws, p->o_us);
  unsigned char* s2 = at<unsigned char>(ws, p->o_s2);
  unsigned char* s3 = at<unsigned char>(ws, p->o_s3);
  char* base = at<char>(ws, p->o_scratch);
  const double* dn = p->nodes;
  const double inv_scale = 1.0 / ((double)p->d.nx * (double)p->d.ny);
  // pair segments on (ncx2, ncy2), the triple segment on (ncx, ncy3)
  const AdjGrid G2{p->ncx2, p->lncx2, p->ncy2, p->lncy2};
  const AdjGrid G3{p->ncx, p->lncx, p->ncy3, p->lncy3};
  const double fwd2 = ((double)p->d.nx * (double)p->d.ny) / ((double)G2.nx * (double)G2.ny);
  const double fwd3 = ((double)p->d.nx * (double)p->d.ny) / ((double)G3.nx * (double)G3.ny);
  const AdjLayout L = adj_layout(p, p->group);
  cplx* E1 = reinterpret_cast<cplx*>(base + L.e1);
  cplx* E2 = reinterpret_cast<cplx*>(base + L.e2);
  cplx* E3 = reinterpret_cast<cplx*>(base + L.e3);
  cplx* DA22 = reinterpret_cast<cplx*>(base + L.da22);
  cplx* DA1 = reinterpret_cast<cplx*>(base + L.da1);
  cplx* DAI = reinterpret_cast<cplx*>(base + L.dai);
  gl_status s;
  const cplx* spec = nullptr;
  if ((s = analyse_group(p, gu, spectra, layout, ws, st, &spec)) != GL_OK) return s;

  // seeds: Ebar on each differentiated component's box
  cplx* rows = reinterpret_cast<cplx*>(base + L.stage);
  const bool e11 = p->comps & GL_COMP_ETA11, e22 = adj_eta22(p), e33 = adj_eta33(p);
  if (e11 && (s = adj_seed(p, gu, resid, B1, rows, E1, st)) != GL_OK) return s;
  if (e22 && (s = adj_seed(p, gu, resid, B2, rows, E2, st)) != GL_OK) return s;
  if (e33 && (s = adj_seed(p, gu, resid, B3, rows, E3, st)) != GL_OK) return s;

  // ---------------- eta22 (spatial.py:156-231), transposed ----------------
  if (e22) {
    const int J = p->ranks[0];
    const int nj = gu * J;
    const AdjStage22 S = adj_stage22(p, L.stage, p->group);
    cplx* P = reinterpret_cast<cplx*>(base + S.P);
    cplx* Q = reinterpret_cast<cplx*>(base + S.Q);
    cplx* R = reinterpret_cast<cplx*>(base + S.R);
    unsigned long long* mx = reinterpret_cast<unsigned long long*>(base + S.mx);
    cplx* RA = reinterpret_cast<cplx*>(base + S.RA);
    cplx* QA = reinterpret_cast<cplx*>(base + S.QA);
    CUDA_TRY(cudaMemsetAsync(mx, 0, (size_t)nj * 2 * 8, st));
    const int m8[8] = {M_ONE, M_NU, M_NU2, M_QX_DIVNU, M_QY_DIVNU, M_Q2_DIVNU, M_QX, M_QY};
    // forward node fields and products (recomputed)
    ColArgs a;
    std::memset(&a, 0, sizeof a);
    a.kind = COL_ETA22;
    const int z8[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    set_banks(a, 8, m8, z8);  // qx-multiple banks become twins
    a.box = B1;
    a.geo = p->geo1;
    a.spec = spec;
    a.spec_job_stride = pl1;
    a.jobs_per_unit = J;
    a.us = us;
    a.nodes = dn + 0 * MAX_RANK;
    a.out = P;
    a.n = G2.ny;
    a.log2n = G2.lny;
    a.scale = inv_scale;
    if ((s = launch_col_ifft(a, nj, st, p->tw)) != GL_OK) return s;
    RowArgs r;
    std::memset(&r, 0, sizeof r);
    r.kind = ROW_ETA22;
    r.grp[0] = BankGroup{P, 8, B1.x0, B1.w};
    r.ngrp = 1;
    r.nout = 2;
    r.out_x0 = B2.x0;
    r.out_w = B2.w;
    r.out = Q;
    r.nx = G2.nx;
    r.log2nx = G2.lnx;
    r.ny = G2.ny;
    r.us = us;
    r.jobs_per_unit = J;
    r.gmax = ROW_GMAX;
    if ((s = launch_row(r, nj, st, p->tw)) != GL_OK) return s;
    ColFftArgs f;
    f.in = Q;
    f.out = R;
    f.box = B2;
    f.n = G2.ny;
    f.log2n = G2.lny;
    f.nsrc = 2;
    f.jobs_per_unit = J;
    f.mask = s2;
    f.maxslot = mx;
    f.scale = fwd2;
    if ((s = launch_col_fft(f, nj * 2, st, p->tw)) != GL_OK) return s;
    // adjoint node spectra -> adjoint fields -> transposed products
    AdjArgs aa;
    std::memset(&aa, 0, sizeof aa);
    aa.us = us;
    aa.geo = p->geo2;
    aa.box = B2;
    aa.seed = E2;
    aa.fwd = R;
    aa.fwdmax = mx;
    aa.mask = s2;
    aa.out = RA;
    aa.nodes = dn + 0 * MAX_RANK;
    aa.weights = dn + 4 * MAX_RANK;
    aa.jobs_per_unit = J;
    aa.floor_rel = p->floor_rel;
    {
      dim3 g(grid_for(pl2, T, 64), nj);
      LaunchScope ls_("adj_eta22_kernel", st, 0.0);
      adj_eta22_kernel<<<g, T, 0, st>>>(aa);
    }
    LAUNCH_CHECK("adj_eta22_kernel");
    if ((s = adj_cols(p, G2, B2, p->geo2, RA, 2, nj, Q, st)) != GL_OK) return s;
    RowArgs ra;
    std::memset(&ra, 0, sizeof ra);
    ra.kind = ROW_ADJ_ETA22;
    ra.grp[0] = BankGroup{P, 8, B1.x0, B1.w, 0};
    ra.grp[1] = BankGroup{Q, 2, B2.x0, B2.w, 1};
    ra.ngrp = 2;
    ra.nout = 8;
    ra.out_x0 = B1.x0;
    ra.out_w = B1.w;
    ra.out = QA;
    ra.out_conj = 1;
    ra.nx = G2.nx;
    ra.log2nx = G2.lnx;
    ra.ny = G2.ny;
    ra.us = us;
    ra.jobs_per_unit = J;
    ra.gmax = ROW_GMAX;
    if ((s = launch_row(ra, nj, st, p->tw)) != GL_OK) return s;
    CmbArgs c = cmb_args(p, G2, CMB_ETA22, 8, m8, nullptr, 1, B1, p->geo1, QA, DA22, us, J);
    c.nodes = dn + 0 * MAX_RANK;
    if ((s = launch_combine(c, nj, st, p->tw)) != GL_OK) return s;
  }

  // ---------------- order 3 (_order3.py:18-148), eta33 transposed ----------------
  if (e33) {
    const int Jo = p->ranks[3], I = p->ranks[2];
    const int nuj = gu * Jo, nj = nuj * I;
    const AdjStage33 S = adj_stage33(p, L.stage, p->group);
    cplx* E = reinterpret_cast<cplx*>(base + S.E);
    unsigned long long* maxEt = reinterpret_cast<unsigned long long*>(base + S.mxs);
    unsigned long long* maxRO = maxEt + nuj;
    cplx* PI = reinterpret_cast<cplx*>(base + S.PI);
    cplx* QI = reinterpret_cast<cplx*>(base + S.QI);
    cplx* RI = reinterpret_cast<cplx*>(base + S.RI);
    unsigned long long* maxRI = reinterpret_cast<unsigned long long*>(base + S.maxRI);
    cplx* P1 = reinterpret_cast<cplx*>(base + S.P1);
    cplx* P2 = reinterpret_cast<cplx*>(base + S.P2);
    cplx* QO = reinterpret_cast<cplx*>(base + S.QO);
    cplx* RO = reinterpret_cast<cplx*>(base + S.RO);
    cplx* RAo = reinterpret_cast<cplx*>(base + S.RAo);
    cplx* QA1 = reinterpret_cast<cplx*>(base + S.QA1);
    cplx* QA2 = reinterpret_cast<cplx*>(base + S.QA2);
    cplx* EA = reinterpret_cast<cplx*>(base + S.EA);
    cplx* RAi = reinterpret_cast<cplx*>(base + S.RAi);
    cplx* QAi = reinterpret_cast<cplx*>(base + S.QAi);
    CUDA_TRY(cudaMemsetAsync(maxEt, 0, (size_t)nuj * 3 * 8, st));
    CUDA_TRY(cudaMemsetAsync(maxRI, 0, (size_t)nj * 4 * 8, st));
    const int mi[12] = {M_ONE, M_NU, M_NU2, M_NU3, M_QX_SNU, M_QY_SNU,
                        M_QX, M_QY, M_Q2_SNU, M_Q2, M_NUQX, M_NUQY};
    const int m1[12] = {M_ONE, M_IQX, M_IQY, M_QX_SNU, M_QY_SNU, M_MI_NU,
                        M_NUQX, M_NUQY, M_MI_Q2_SNU, M_MI_Q2NU, M_MINUS_A, M_MINUS_Q2};
    const int m9[9] = {M_ONE, M_IQX, M_IQY, M_IQX, M_IQY, M_A, M_Q2, M_A, M_ONE};
    const int src9[9] = {0, 0, 0, 2, 2, 2, 2, 3, 1};
    // forward inner stage (recomputed): inner fields PI, sources RI, pair spectra E
    {
      ColArgs a;
      std::memset(&a, 0, sizeof a);
      a.kind = COL_INNER;
      const int z12[12] = {0};
      set_banks(a, 12, mi, z12);
      a.box = B1;
      a.geo = p->geo1;
      a.spec = spec;
      a.spec_job_stride = pl1;
      a.jobs_per_unit = Jo * I;
      a.us = us;
      a.nodes = dn + 3 * MAX_RANK;
      a.nodes2 = dn + 2 * MAX_RANK;
      a.n_inner = I;
      a.n_outer = Jo;
      a.out = PI;
      a.n = G2.ny;
      a.log2n = G2.lny;
      a.scale = inv_scale;
      if ((s = launch_col_ifft(a, nj, st, p->tw)) != GL_OK) return s;
      RowArgs r;
      std::memset(&r, 0, sizeof r);
      r.kind = ROW_INNER;
      r.grp[0] = BankGroup{PI, 12, B1.x0, B1.w};
      r.ngrp = 1;
      r.nout = 4;
      r.out_x0 = B2.x0;
      r.out_w = B2.w;
      r.out = QI;
      r.nx = G2.nx;
      r.log2nx = G2.lnx;
      r.ny = G2.ny;
      r.us = us;
      r.jobs_per_unit = Jo * I;
      r.gmax = ROW_GMAX;
      if ((s = launch_row(r, nj, st, p->tw)) != GL_OK) return s;
      ColFftArgs f;
      f.in = QI;
      f.out = RI;
      f.box = B2;
      f.n = G2.ny;
      f.log2n = G2.lny;
      f.nsrc = 4;
      f.jobs_per_unit = Jo * I;
      f.mask = s2;
      f.maxslot = maxRI;
      f.scale = fwd2;
      if ((s = launch_col_fft(f, nj * 4, st, p->tw)) != GL_OK) return s;
      AccArgs c;
      std::memset(&c, 0, sizeof c);
      c.us = us;
      c.geo = p->geo2;
      c.box = B2;
      c.in = RI;
      c.maxin = maxRI;
      c.out = E;
      c.maxout = maxEt;
      c.mask = s2;
      c.nodes = dn + 2 * MAX_RANK;
      c.weights = dn + 6 * MAX_RANK;
      c.nnodes = I;
      c.nsub = Jo;
      c.floor_rel = p->floor_rel;
      {
        LaunchScope ls_("acc_inner_kernel", st, 0.0);
        launch_acc_inner(c, pl2, nuj / c.nsub, st);
      }
      LAUNCH_CHECK("acc_inner_kernel");
    }
    // forward outer stage (recomputed): first-order fields P1, pair fields P2,
    // the fk, fd forcing spectra RO and their maxima
    {
      ColArgs a;
      std::memset(&a, 0, sizeof a);
      a.kind = COL_OUTER1;
      const int z12[12] = {0};
      set_banks(a, 12, m1, z12);
      a.box = B1;
      a.geo = p->geo1;
      a.spec = spec;
      a.spec_job_stride = pl1;
      a.jobs_per_unit = Jo;
      a.us = us;
      a.nodes = dn + 3 * MAX_RANK;
      a.out = P1;
      a.n = G3.ny;
      a.log2n = G3.lny;
      a.scale = inv_scale;
      if ((s = launch_col_ifft(a, nuj, st, p->tw)) != GL_OK) return s;
      ColArgs a2;
      std::memset(&a2, 0, sizeof a2);
      a2.kind = COL_OUTER2;
      set_banks(a2, 9, m9, src9);
      a2.box = B2;
      a2.geo = p->geo2;
      a2.spec = E;
      a2.spec_job_stride = 4LL * pl2;
      a2.spec_sub_stride = pl2;
      a2.jobs_per_unit = Jo;
      a2.us = us;
      a2.floor_max = maxEt;
      a2.floor_rel = p->floor_rel;
      a2.out = P2;
      a2.n = G3.ny;
      a2.log2n = G3.lny;
      a2.scale = inv_scale;
      if ((s = launch_col_ifft(a2, nuj, st, p->tw)) != GL_OK) return s;
      RowArgs r;
      std::memset(&r, 0, sizeof r);
      r.kind = ROW_OUTER;
      r.grp[0] = BankGroup{P1, 12, B1.x0, B1.w};
      r.grp[1] = BankGroup{P2, 9, B2.x0, B2.w};
      r.ngrp = 2;
      r.nout = 2;  // fk, fd (the contact rows feed psi33 only)
      r.out_x0 = B3.x0;
      r.out_w = B3.w;
      r.out = QO;
      r.nx = G3.nx;
      r.log2nx = G3.lnx;
      r.ny = G3.ny;
      r.us = us;
      r.jobs_per_unit = Jo;
      r.gmax = ROW_GMAX;
      if ((s = launch_row(r, nuj, st, p->tw)) != GL_OK) return s;
      ColFftArgs f;
      f.in = QO;
      f.out = RO;
      f.box = B3;
      f.n = G3.ny;
      f.log2n = G3.lny;
      f.nsrc = 2;
      f.jobs_per_unit = Jo;
      f.mask = s3;
      f.maxslot = maxRO;
      f.scale = fwd3;
      if ((s = launch_col_fft(f, nuj * 2, st, p->tw)) != GL_OK) return s;
    }
    // adjoint outer stage: forcing adjoints -> first-order and pair adjoints
    {
      AdjArgs aa;
      std::memset(&aa, 0, sizeof aa);
      aa.us = us;
      aa.geo = p->geo3;
      aa.box = B3;
      aa.seed = E3;
      aa.fwd = RO;
      aa.fwdmax = maxRO;
      aa.mask = s3;
      aa.out = RAo;
      aa.nodes = dn + 3 * MAX_RANK;
      aa.weights = dn + 7 * MAX_RANK;
      aa.jobs_per_unit = Jo;
      aa.floor_rel = p->floor_rel;
      {
        dim3 g(grid_for(pl3, T, 48), nuj);
        LaunchScope ls_("adj_outer_kernel", st, 0.0);
        adj_outer_kernel<<<g, T, 0, st>>>(aa);
      }
      LAUNCH_CHECK("adj_outer_kernel");
      if ((s = adj_cols(p, G3, B3, p->geo3, RAo, 2, nuj, QO, st)) != GL_OK) return s;
      RowArgs ra;
      std::memset(&ra, 0, sizeof ra);
      ra.kind = ROW_ADJ_OUTER;
      ra.grp[0] = BankGroup{P1, 12, B1.x0, B1.w, 0};
      ra.grp[1] = BankGroup{P2, 9, B2.x0, B2.w, 0};
      ra.grp[2] = BankGroup{QO, 2, B3.x0, B3.w, 1};
      ra.ngrp = 3;
      ra.nout = 20;
      ra.nout_a = 12;
      ra.out_x0 = B1.x0;
      ra.out_w = B1.w;
      ra.out = QA1;
      ra.out2_x0 = B2.x0;
      ra.out2_w = B2.w;
      ra.out2 = QA2;
      ra.out_conj = 1;
      ra.nx = G3.nx;
      ra.log2nx = G3.lnx;
      ra.ny = G3.ny;
      ra.us = us;
      ra.jobs_per_unit = Jo;
      ra.gmax = ROW_GMAX;
      if ((s = launch_row(ra, nuj, st, p->tw)) != GL_OK) return s;
      CmbArgs c1 = cmb_args(p, G3, CMB_FIRST3, 12, m1, nullptr, 1, B1, p->geo1, QA1, DA1, us, Jo);
      c1.nodes = dn + 3 * MAX_RANK;
      if ((s = launch_combine(c1, nuj, st, p->tw)) != GL_OK) return s;
      CmbArgs c2 = cmb_args(p, G3, CMB_PAIR, 8, m9, src9, 4, B2, p->geo2, QA2, EA, us, Jo);
      c2.mask = s2;
      if ((s = launch_combine(c2, nuj, st, p->tw)) != GL_OK) return s;
    }
    // adjoint inner stage: pair-spectra adjoints -> source adjoints -> inner fields
    {
      AdjArgs aa;
      std::memset(&aa, 0, sizeof aa);
      aa.us = us;
      aa.geo = p->geo2;
      aa.box = B2;
      aa.seed = EA;
      aa.fwd = RI;
      aa.fwdmax = maxRI;
      aa.mask = s2;
      aa.out = RAi;
      aa.nodes = dn + 2 * MAX_RANK;
      aa.weights = dn + 6 * MAX_RANK;
      aa.jobs_per_unit = Jo * I;
      aa.n_inner = I;
      aa.floor_rel = p->floor_rel;
      {
        dim3 g(grid_for(pl2, T, 64), nj);
        LaunchScope ls_("adj_inner_kernel", st, 0.0);
        adj_inner_kernel<<<g, T, 0, st>>>(aa);
      }
      LAUNCH_CHECK("adj_inner_kernel");
      if ((s = adj_cols(p, G2, B2, p->geo2, RAi, 4, nj, QI, st)) != GL_OK) return s;
      RowArgs ra;
      std::memset(&ra, 0, sizeof ra);
      ra.kind = ROW_ADJ_INNER;
      ra.grp[0] = BankGroup{PI, 12, B1.x0, B1.w, 0};
      ra.grp[1] = BankGroup{QI, 4, B2.x0, B2.w, 1};
      ra.ngrp = 2;
      ra.nout = 12;
      ra.out_x0 = B1.x0;
      ra.out_w = B1.w;
      ra.out = QAi;
      ra.out_conj = 1;
      ra.nx = G2.nx;
      ra.log2nx = G2.lnx;
      ra.ny = G2.ny;
      ra.us = us;
      ra.jobs_per_unit = Jo * I;
      ra.gmax = ROW_GMAX;
      if ((s = launch_row(ra, nj, st, p->tw)) != GL_OK) return s;
      CmbArgs c = cmb_args(p, G2, CMB_INNER, 12, mi, nullptr, 1, B1, p->geo1, QAi, DAI, us, Jo * I);
      c.nodes = dn + 3 * MAX_RANK;
      c.nodes2 = dn + 2 * MAX_RANK;
      c.n_inner = I;
      if ((s = launch_combine(c, nj, st, p->tw)) != GL_OK) return s;
    }
  }

  // ---------------- gradient on the parent box ----------------
  {
    RedArgs ra;
    ra.e1 = e11 ? E1 : nullptr;
    ra.da22 = DA22;
    ra.n22 = e22 ? p->ranks[0] : 0;
    ra.da1 = DA1;
    ra.n1 = e33 ? p->ranks[3] : 0;
    ra.dai = DAI;
    ra.ni = e33 ? p->ranks[3] * p->ranks[2] : 0;
    ra.grad = grad;
    ra.plane = pl1;
    dim3 g(grid_for(pl1, T, 64), gu);
    {
      LaunchScope ls_("adj_reduce_kernel", st, 0.0);
      adj_reduce_kernel<<<g, T, 0, st>>>(ra);
    }
    LAUNCH_CHECK("adj_reduce_kernel");
  }
  {
    dim3 g(grid_for(pl1, T, 64), gu);
    {
      LaunchScope ls_("nonfinite_kernel", st, 0.0);
      nonfinite_kernel<<<g, T, 0, st>>>(grad, (size_t)pl1, 0, us);
    }
    LAUNCH_CHECK("nonfinite_kernel");
  }
  if (status) {
    {
      LaunchScope ls_("status_kernel", st, 0.0);
      status_kernel<<<(gu + 63) / 64, 64, 0, st>>>(us, gu, status);
    }
    LAUNCH_CHECK("status_kernel");
  }
  return GL_OK;
}

extern "C" gl_status gl_adjoint_execute(gl_plan* p, int n_units, const void* d_spectra, int layout,
                                        const double* d_residual, void* d_grad, void* d_ws,
                                        size_t ws_bytes, int* d_status, void* stream) {
  gl_status s = adj_check_plan(p);
  if (s != GL_OK) return s;
  if (n_units < 0) return fail(GL_ERR_INVALID_ARGUMENT, "negative unit count");
  if (n_units == 0) return GL_OK;
  if (!d_spectra || !d_residual || !d_grad)
    return fail(GL_ERR_INVALID_ARGUMENT, "null spectra, residual or gradient");
  if (layout != GL_SPECTRA_FULL && layout != GL_SPECTRA_BOX)
    return fail(GL_ERR_INVALID_ARGUMENT, "unknown spectra layout");
  const size_t need = p->o_scratch + adj_layout(p, p->group).total;
  if (!d_ws || ws_bytes < need || (reinterpret_cast<uintptr_t>(d_ws) & 255))
    return fail(GL_ERR_WORKSPACE, "workspace must be 256-byte aligned and at least %zu bytes", need);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const size_t in_unit = layout == GL_SPECTRA_FULL ? (size_t)p->d.nx * p->d.ny
                                                   : (size_t)p->b1.w * p->b1.h;
  const size_t r_unit = (size_t)p->d.nx * p->d.ny;
  const size_t g_unit = (size_t)p->b1.w * p->b1.h;
  for (int u0 = 0; u0 < n_units; u0 += p->group) {
    const int gu = std::min(p->group, n_units - u0);
    const void* in = reinterpret_cast<const cplx*>(d_spectra) + (size_t)u0 * in_unit;
    s = run_adjoint_group(p, gu, in, layout, d_residual + (size_t)u0 * r_unit,
                          reinterpret_cast<cplx*>(d_grad) + (size_t)u0 * g_unit, d_ws,
                          d_status ? d_status + u0 : nullptr, st);
    if (s != GL_OK) return s;
  }
  return GL_OK;
}

extern "C" gl_status gl_deposit_modes_adjoint(const gl_plan* p, int n_units, int n_seg,
                                              const int* seg_off, const int* seg_bin, int n_modes,
                                              const double* omega, const double* times,
                                              const void* d_grad, double* d_gab, void* stream) {
  if (!p) return fail(GL_ERR_INVALID_ARGUMENT, "null plan");
  if (n_units < 0 || n_seg < 0 || n_modes < 0) return fail(GL_ERR_INVALID_ARGUMENT, "negative size");
  if (n_modes == 0) return GL_OK;
  if (!d_gab || !d_grad || !times || !seg_off || !seg_bin || !omega)
    return fail(GL_ERR_INVALID_ARGUMENT, "null deposit-adjoint buffer");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  CUDA_TRY(cudaMemsetAsync(d_gab, 0, sizeof(double) * 2 * (size_t)n_modes, st));
  if (n_seg == 0 || n_units == 0) return GL_OK;
  {
    LaunchScope ls_("deposit_adjoint_kernel", st, 0.0);
    deposit_adjoint_kernel<<<grid_for(n_seg, 128, 256), 128, 0, st>>>(
        n_units, n_seg, seg_off, seg_bin, omega, times, (double)p->d.nx * (double)p->d.ny,
        p->d.depth, reinterpret_cast<const cplx*>(d_grad), p->b1.w * p->b1.h, d_gab);
  }
  LAUNCH_CHECK("deposit_adjoint_kernel");
  return GL_OK;
}

extern "C" gl_status gl_deposit_modes(const gl_plan* p, int n_units, int n_seg, const int* seg_off,
                                      const int* seg_bin, int n_modes, const double* ab,
                                      const double* omega, const double* times, void* out,
                                      void* stream) {
  if (!p) return fail(GL_ERR_INVALID_ARGUMENT, "null plan");
  if (n_units < 0 || n_seg < 0 || n_modes < 0) return fail(GL_ERR_INVALID_ARGUMENT, "negative size");
  if (n_units == 0) return GL_OK;
  if (!out || (n_seg && (!seg_off || !seg_bin || !ab || !omega)) || !times)
    return fail(GL_ERR_INVALID_ARGUMENT, "null deposit buffer");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const int plane = p->b1.w * p->b1.h;
  CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(cplx) * (size_t)n_units * plane, st));
  if (n_seg == 0) return GL_OK;
  dim3 g(grid_for(n_seg, 128, 256), n_units);
  {
    LaunchScope ls_("deposit_kernel", st, 0.0);
    deposit_kernel<<<g, 128, 0, st>>>(n_seg, seg_off, seg_bin, ab, omega, times,
                                    (double)p->d.nx * (double)p->d.ny, p->d.depth,
                                    reinterpret_cast<cplx*>(out), plane);
  }
  LAUNCH_CHECK("deposit_kernel");
  return GL_OK;
}

// ---------------------------------------------------------------------------
// plain batched 2-D FFT on the reference grid (numpy fft2 / ifft2 conventions)
// ---------------------------------------------------------------------------

template <int SIGN>
__global__ void fft2_rows_kernel(const cplx* in, cplx* out, int nx, int log2nx, int ny, int rows,
                                 double scale, const cplx* __restrict__ tw) {
  extern __shared__ cplx smem[];
  const int b = blockIdx.y;
  const int y0 = blockIdx.x * rows;
  const int r = min(rows, ny - y0);
  cplx* buf = smem;
  cplx* tmp = smem + (size_t)rows * nx;
  const size_t base = ((size_t)b * ny + y0) * nx;
  for (int t = threadIdx.x; t < r * nx; t += blockDim.x) buf[t] = in[base + t];
  __syncthreads();
  fft_rows<SIGN>(buf, tmp, nx, log2nx, r, rows, tw);
  for (int t = threadIdx.x; t < r * nx; t += blockDim.x) out[base + t] = cscale(scale, buf[t]);
}

template <int SIGN>
__global__ void fft2_cols_kernel(cplx* data, int nx, int ny, int log2ny, int cw,
                                 const cplx* __restrict__ tw) {
  extern __shared__ cplx smem[];
  const int b = blockIdx.y;
  const int x0 = blockIdx.x * cw;
  const int c = min(cw, nx - x0);
  cplx* buf = smem;
  cplx* tmp = smem + (size_t)cw * ny;
  cplx* d = data + (size_t)b * nx * ny;
  for (int t = threadIdx.x; t < c * ny; t += blockDim.x) {
    const int y = t / c, k = t % c;
    buf[k * ny + y] = d[(size_t)y * nx + x0 + k];
  }
  __syncthreads();
  fft_rows<SIGN>(buf, tmp, ny, log2ny, c, cw, tw);
  for (int t = threadIdx.x; t < c * ny; t += blockDim.x) {
    const int y = t / c, k = t % c;
    d[(size_t)y * nx + x0 + k] = buf[k * ny + y];
  }
}

static cplx* g_tw_global[64] = {nullptr};

static gl_status device_twiddles(cplx** out) {
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(GL_ERR_CUDA, "device index out of range");
  if (!g_tw_global[dev]) {
    cplx* tw = nullptr;
    CUDA_TRY(cudaMalloc(&tw, sizeof(cplx) * TW_N));
    twiddle_kernel<<<TW_N / 256, 256>>>(tw, TW_N);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaDeviceSynchronize());
    g_tw_global[dev] = tw;
  }
  *out = g_tw_global[dev];
  return GL_OK;
}

extern "C" gl_status gl_fft2(int batch, int nx, int ny, const void* d_in, void* d_out, int inverse,
                             void* stream) {
  if (batch < 0 || !d_in || !d_out) return fail(GL_ERR_INVALID_ARGUMENT, "bad fft2 arguments");
  if (!is_pow2(nx) || !is_pow2(ny) || nx < 2 || ny < 2 || nx > TW_N || ny > TW_N)
    return fail(GL_ERR_UNSUPPORTED, "gl_fft2 runs power-of-two sizes from 2 to %d", TW_N);
  if (batch == 0) return GL_OK;
  cplx* tw = nullptr;
  gl_status s = device_twiddles(&tw);
  if (s != GL_OK) return s;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const int rows = std::max(1, 2048 / nx);
  const int cw = std::max(1, 2048 / ny);
  const size_t smr = (size_t)2 * rows * nx * sizeof(cplx), smc = (size_t)2 * cw * ny * sizeof(cplx);
  const double scale = inverse ? 1.0 / ((double)nx * (double)ny) : 1.0;
  dim3 gr((ny + rows - 1) / rows, batch), gc((nx + cw - 1) / cw, batch);
  const cplx* in = reinterpret_cast<const cplx*>(d_in);
  cplx* out = reinterpret_cast<cplx*>(d_out);
  if (inverse) {
    ensure_smem_attr((const void*)fft2_rows_kernel<+1>, (int)SMEM_LIMIT);
    ensure_smem_attr((const void*)fft2_cols_kernel<+1>, (int)SMEM_LIMIT);
    fft2_rows_kernel<+1><<<gr, 256, smr, st>>>(in, out, nx, ilog2(nx), ny, rows, scale, tw);
    LAUNCH_CHECK("fft2_rows_kernel");
    fft2_cols_kernel<+1><<<gc, 256, smc, st>>>(out, nx, ny, ilog2(ny), cw, tw);
    LAUNCH_CHECK("fft2_cols_kernel");
  } else {
    ensure_smem_attr((const void*)fft2_rows_kernel<-1>, (int)SMEM_LIMIT);
    ensure_smem_attr((const void*)fft2_cols_kernel<-1>, (int)SMEM_LIMIT);
    fft2_rows_kernel<-1><<<gr, 256, smr, st>>>(in, out, nx, ilog2(nx), ny, rows, scale, tw);
    LAUNCH_CHECK("fft2_rows_kernel");
    fft2_cols_kernel<-1><<<gc, 256, smc, st>>>(out, nx, ny, ilog2(ny), cw, tw);
    LAUNCH_CHECK("fft2_cols_kernel");
  }
  return GL_OK;
}

// ---------------------------------------------------------------------------
// single-direction time path (modal GL resolvent and eta20)
// ---------------------------------------------------------------------------

static SFft sfft(cplx* d, int n, long long stride, long long cstride, int ncount, long long ostride,
                 double scale) {
  SFft a;
  std::memset(&a, 0, sizeof a);
  a.data = d;
  a.n = n;
  a.log2n = ilog2(n);
  a.stride = stride;
  a.cstride = cstride;
  a.ncount = ncount;
  a.ostride = ostride;
  a.scale = scale;
  return a;
}

// Transform along axis 0 of a [P][M] array (length P, power of two).  sign > 0:
// natural input, output rows permuted when P > 4096; sign < 0: the inverse
// ordering (permuted input, natural output).  Four-step split P = P1 P2.
static gl_status axis0_transform(cplx* d, int P, int M, int sign, double scale, cudaStream_t st,
                                 const cplx* tw) {
  if (P <= TW_N) return launch_sfft(sfft(d, P, M, 1, M, 0, scale), 1, sign, st, tw);
  const int p = ilog2(P);
  const int P1 = 1 << (p - p / 2), P2 = 1 << (p / 2);
  gl_status s;
  if (sign > 0) {
    SFft a = sfft(d, P2, (long long)P1 * M, 1, P1 * M, 0, 1.0);
    a.tw_mode = 1;
    a.tw_div = M;
    a.tw_log2p = p;
    if ((s = launch_sfft(a, 1, +1, st, tw)) != GL_OK) return s;
    return launch_sfft(sfft(d, P1, M, 1, M, (long long)P1 * M, scale), P2, +1, st, tw);
  }
  SFft a = sfft(d, P1, M, 1, M, (long long)P1 * M, 1.0);
  a.tw_mode = 2;
  a.tw_log2p = p;
  if ((s = launch_sfft(a, P2, -1, st, tw)) != GL_OK) return s;
  return launch_sfft(sfft(d, P2, (long long)P1 * M, 1, P1 * M, 0, scale), 1, -1, st, tw);
}

// Transform along the contiguous last axis of [rows][M].
static gl_status axis_last_transform(cplx* d, long long rows, int M, int sign, double scale,
                                     cudaStream_t st, const cplx* tw) {
  return launch_sfft(sfft(d, M, 1, M, (int)rows, 0, scale), 1, sign, st, tw);
}

static int modal_pad(int w) { return std::max(16, next_pow2(w)); }

static size_t modal_buffers(int order) { return order >= 3 ? 22 : 7; }

static gl_status modal_check(const gl_modal_desc* d) {
  if (!d) return fail(GL_ERR_INVALID_ARGUMENT, "null modal descriptor");
  if (d->order != 2 && d->order != 3) return fail(GL_ERR_INVALID_ARGUMENT, "modal order must be 2 or 3");
  if (!is_pow2(d->points) || d->points < 16 || d->points > (1 << 24))
    return fail(GL_ERR_UNSUPPORTED, "modal_points must be a power of two from 16 to 2^24 (got %d)", d->points);
  if (d->width < 1 || modal_pad(d->width) > TW_N)
    return fail(GL_ERR_UNSUPPORTED, "the work band (%d bins) exceeds %d", d->width, TW_N);
  if (d->base_bin < 1 || d->count < 1 || d->width > d->count)
    return fail(GL_ERR_INVALID_ARGUMENT, "the nonlinear output band does not fit in the time record");
  if (!(d->q_step > 0) || !(d->freq_step > 0) || !(d->depth > 0))
    return fail(GL_ERR_INVALID_ARGUMENT, "modal spacings and depth must be positive");
  if (d->rank < 1 || d->rank > MAX_RANK || !d->nodes || !d->weights)
    return fail(GL_ERR_RANK, "modal GL rule must have 1..%d nodes", MAX_RANK);
  return GL_OK;
}

extern "C" gl_status gl_modal_workspace_size(const gl_modal_desc* d, size_t* bytes) {
  gl_status s = modal_check(d);
  if (s != GL_OK) return s;
  if (!bytes) return fail(GL_ERR_INVALID_ARGUMENT, "null size pointer");
  const size_t plane = (size_t)d->points * modal_pad(d->width) * sizeof(cplx);
  *bytes = align_up(4096) + modal_buffers(d->order) * align_up(plane) +
           2 * align_up((size_t)(3 * d->width + 3) * (sizeof(cplx) + sizeof(int)));
  return GL_OK;
}

extern "C" gl_status gl_modal_level(const gl_modal_desc* d, int nnz, const long long* d_idx,
                                    const double* d_val, void* d_eta22, void* d_eta33, void* d_ws,
                                    size_t ws_bytes, void* stream) {
  gl_status s = modal_check(d);
  if (s != GL_OK) return s;
  size_t need = 0;
  gl_modal_workspace_size(d, &need);
  if (!d_ws || ws_bytes < need || (reinterpret_cast<uintptr_t>(d_ws) & 255))
    return fail(GL_ERR_WORKSPACE, "workspace must be 256-byte aligned and at least %zu bytes", need);
  if (nnz < 0 || (nnz && (!d_idx || !d_val)) || !d_eta22 || (d->order >= 3 && !d_eta33))
    return fail(GL_ERR_INVALID_ARGUMENT, "null modal buffers");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  cplx* tw = nullptr;
  if ((s = device_twiddles(&tw)) != GL_OK) return s;
  const int P = d->points, W = d->width, M = modal_pad(W);
  const int wmax = (W - 1) / d->order;
  const long long total = (long long)P * M;
  const size_t plane = align_up((size_t)total * sizeof(cplx));
  char* base = reinterpret_cast<char*>(d_ws);
  double* dn = reinterpret_cast<double*>(base);  // nodes then weights
  char* bufs = base + align_up(4096);
  auto buf = [&](int k) { return reinterpret_cast<cplx*>(bufs + (size_t)k * plane); };
  char* small = bufs + modal_buffers(d->order) * plane;
  cplx* coef = reinterpret_cast<cplx*>(small);
  int* bins = reinterpret_cast<int*>(small + align_up((size_t)(3 * W + 3) * sizeof(cplx)));
  {
    double host[2 * MAX_RANK] = {0};
    std::memcpy(host, d->nodes, sizeof(double) * d->rank);
    std::memcpy(host + MAX_RANK, d->weights, sizeof(double) * d->rank);
    CUDA_TRY(cudaMemcpyAsync(dn, host, sizeof host, cudaMemcpyHostToDevice, st));
    std::vector<int> hb(3 * W + 3);
    for (int w = 0; w < 3 * wmax + 1; ++w) hb[w] = 3 * d->base_bin + w;
    for (int w = 0; w < 2 * wmax + 1; ++w) hb[3 * wmax + 1 + w] = 2 * d->base_bin + w;
    CUDA_TRY(cudaMemcpyAsync(bins, hb.data(), sizeof(int) * hb.size(), cudaMemcpyHostToDevice, st));
    // the host vectors must outlive the copies
    CUDA_TRY(cudaStreamSynchronize(st));
  }
  ModalGeo g;
  g.P = P;
  g.M = M;
  g.W = W;
  g.q_step = d->q_step;
  g.fstep = d->freq_step;
  g.b0 = d->base_bin;
  const int T = 256;
  const int eb = grid_for((size_t)total, T, 8192);
  cplx* joint = buf(0);
  CUDA_TRY(cudaMemsetAsync(joint, 0, (size_t)total * sizeof(cplx), st));
  if (nnz) {
    // indices arrive in [P][W]; the joint is [P][M]
    LaunchScope ls_("modal_scatter_kernel", st, 0.0);
    modal_scatter_kernel<<<grid_for(nnz, T, 1024), T, 0, st>>>(d_idx, d_val, nnz, joint, W, M);
  }
  LAUNCH_CHECK("modal_scatter_kernel");
  auto to_field = [&](cplx* b) -> gl_status {
    gl_status r = axis0_transform(b, P, M, +1, 1.0, st, tw);
    if (r != GL_OK) return r;
    return axis_last_transform(b, P, M, -1, 1.0, st, tw);
  };
  auto to_spectrum = [&](cplx* b) -> gl_status {
    gl_status r = axis_last_transform(b, P, M, +1, 1.0 / M, st, tw);
    if (r != GL_OK) return r;
    return axis0_transform(b, P, M, -1, 1.0 / P, st, tw);
  };
  auto bank = [&](const cplx* src, int k, int mult) -> gl_status {
    {
      LaunchScope ls_("modal_bank_kernel", st, 0.0);
      modal_bank_kernel<<<eb, T, 0, st>>>(g, src, buf(k), mult);
    }
    LAUNCH_CHECK("modal_bank_kernel");
    return to_field(buf(k));
  };
  // order-2 banks: 1 v, 2 vn, 3 vn2, 4 hx, 5 jx, 6 radial
  const int m6[6] = {MM_ONE, MM_NU, MM_NU2, MM_Q_SNU, MM_Q, MM_Q2_SNU};
  for (int k = 0; k < 6; ++k)
    if ((s = bank(joint, 1 + k, m6[k])) != GL_OK) return s;
  {
    LaunchScope ls_("modal_sources_kernel", st, 0.0);
    modal_sources_kernel<<<eb, T, 0, st>>>(total, buf(1), buf(2), buf(3), buf(4), buf(5), buf(6));
  }
  LAUNCH_CHECK("modal_sources_kernel");
  cplx* SD = buf(3);
  cplx* SK = buf(6);
  if ((s = to_spectrum(SD)) != GL_OK) return s;
  if ((s = to_spectrum(SK)) != GL_OK) return s;
  ModalResp r;
  std::memset(&r, 0, sizeof r);
  r.g = g;
  r.depth = d->depth;
  r.nodes = dn;
  r.weights = dn + MAX_RANK;
  r.rank = d->rank;
  r.sd = SD;
  r.sk = SK;
  r.out = coef + 3 * wmax + 1;
  r.nbins = 2 * wmax + 1;
  r.mult_b0 = 2;
  r.kind = 2;
  r.scale = d->scale22;
  {
    LaunchScope ls_("modal_response_kernel", st, 0.0);
    modal_response_kernel<<<r.nbins, 256, 0, st>>>(r);
  }
  LAUNCH_CHECK("modal_response_kernel");
  {
    LaunchScope ls_("series_synth_kernel", st, 0.0);
    series_synth_kernel<<<grid_for(d->count, T, 1024), T, 0, st>>>(bins + 3 * wmax + 1, r.out, r.nbins,
                                                                  d->count, d_eta22, 0);
  }
  LAUNCH_CHECK("series_synth_kernel");
  if (d->order < 3) return GL_OK;

  // order 3: inner pair spectra, first-order and pair fields, cubic forcing
  cplx* E2 = buf(7);
  cplx* P2 = buf(8);
  ModalResp ri = r;
  ri.scale = d->lambda2;
  ri.nbins = 2 * wmax + 1;
  {
    LaunchScope ls_("modal_pair_kernel", st, 0.0);
    modal_pair_kernel<<<eb, T, 0, st>>>(ri, E2, P2);
  }
  LAUNCH_CHECK("modal_pair_kernel");
  // first-order fields: v (1) and hx (4) are eta and phix; the others in 9..15
  const int m7[7] = {MM_IQ, MM_MI_NU, MM_NU_Q, MM_MI_Q2_SNU, MM_MI_Q2_NU, MM_MINUS_NU2, MM_MINUS_Q2};
  for (int k = 0; k < 7; ++k)
    if ((s = bank(joint, 9 + k, m7[k])) != GL_OK) return s;
  // pair fields 16..21: eta, etax (from e2); phix, phiz, phizz, phitz (from p2)
  const int mp[6] = {MM_PAIR_E, MM_PAIR_EX, MM_PAIR_PX, MM_PAIR_PZ, MM_PAIR_PZZ, MM_PAIR_PTZ};
  for (int k = 0; k < 6; ++k)
    if ((s = bank(k < 2 ? E2 : P2, 16 + k, mp[k])) != GL_OK) return s;
  ModalForcing fo;
  fo.fe = buf(1);
  fo.fex = buf(9);
  fo.fpx = buf(4);
  fo.fpz = buf(10);
  fo.fpxz = buf(11);
  fo.fpzz = buf(12);
  fo.fpzzz = buf(13);
  fo.fptz = buf(14);
  fo.fptzz = buf(15);
  fo.pe = buf(16);
  fo.pex = buf(17);
  fo.ppx = buf(18);
  fo.ppz = buf(19);
  fo.ppzz = buf(20);
  fo.pptz = buf(21);
  fo.fk = buf(2);  // vn and jx are free after the order-2 sources
  fo.fd = buf(5);
  fo.total = total;
  {
    LaunchScope ls_("modal_forcing_kernel", st, 0.0);
    modal_forcing_kernel<<<eb, T, 0, st>>>(fo);
  }
  LAUNCH_CHECK("modal_forcing_kernel");
  if ((s = to_spectrum(fo.fk)) != GL_OK) return s;
  if ((s = to_spectrum(fo.fd)) != GL_OK) return s;
  ModalResp r3 = r;
  r3.sd = fo.fd;
  r3.sk = fo.fk;
  r3.out = coef;
  r3.nbins = 3 * wmax + 1;
  r3.mult_b0 = 3;
  r3.kind = 3;
  r3.scale = d->lambda3;
  {
    LaunchScope ls_("modal_response_kernel", st, 0.0);
    modal_response_kernel<<<r3.nbins, 256, 0, st>>>(r3);
  }
  LAUNCH_CHECK("modal_response_kernel");
  {
    LaunchScope ls_("series_synth_kernel", st, 0.0);
    series_synth_kernel<<<grid_for(d->count, T, 1024), T, 0, st>>>(bins, coef, r3.nbins, d->count,
                                                                  d_eta33, 0);
  }
  LAUNCH_CHECK("series_synth_kernel");
  return GL_OK;
}

static gl_status e20_check(const gl_eta20_desc* d) {
  if (!d) return fail(GL_ERR_INVALID_ARGUMENT, "null eta20 descriptor");
  if (!is_pow2(d->nx) || !is_pow2(d->ny) || d->nx < 16 || d->ny < 16 || d->nx > TW_N || d->ny > TW_N)
    return fail(GL_ERR_UNSUPPORTED, "eta20 modal grids must be powers of two from 16 to %d", TW_N);
  if (d->span < 0 || modal_pad(2 * d->span + 1) > TW_N)
    return fail(GL_ERR_UNSUPPORTED, "the eta20 band exceeds %d bins", TW_N);
  if (d->base_bin < 1 || d->count < 1 || !(d->qx_step > 0) || !(d->qy_step > 0) || !(d->freq_step > 0) ||
      !(d->depth > 0) || !(d->dq > 0))
    return fail(GL_ERR_INVALID_ARGUMENT, "bad eta20 descriptor");
  if (d->rank < 1 || d->rank > MAX_RANK || !d->nodes || !d->weights)
    return fail(GL_ERR_RANK, "eta20 GL rule must have 1..%d nodes", MAX_RANK);
  return GL_OK;
}

extern "C" gl_status gl_eta20_workspace_size(const gl_eta20_desc* d, size_t* bytes) {
  gl_status s = e20_check(d);
  if (s != GL_OK) return s;
  if (!bytes) return fail(GL_ERR_INVALID_ARGUMENT, "null size pointer");
  const size_t plane = (size_t)d->ny * d->nx * modal_pad(2 * d->span + 1) * sizeof(cplx);
  *bytes = align_up(4096) + 11 * align_up(plane);
  return GL_OK;
}

extern "C" gl_status gl_eta20_level(const gl_eta20_desc* d, int nnz, const long long* d_idx,
                                    const double* d_val, void* d_coef, void* d_ws, size_t ws_bytes,
                                    void* stream) {
  gl_status s = e20_check(d);
  if (s != GL_OK) return s;
  size_t need = 0;
  gl_eta20_workspace_size(d, &need);
  if (!d_ws || ws_bytes < need || (reinterpret_cast<uintptr_t>(d_ws) & 255))
    return fail(GL_ERR_WORKSPACE, "workspace must be 256-byte aligned and at least %zu bytes", need);
  if (nnz < 0 || (nnz && (!d_idx || !d_val)) || !d_coef)
    return fail(GL_ERR_INVALID_ARGUMENT, "null eta20 buffers");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  cplx* tw = nullptr;
  if ((s = device_twiddles(&tw)) != GL_OK) return s;
  const int W = 2 * d->span + 1, M = modal_pad(W), nx = d->nx, ny = d->ny;
  const long long total = (long long)ny * nx * M;
  const size_t plane = align_up((size_t)total * sizeof(cplx));
  char* base = reinterpret_cast<char*>(d_ws);
  double* dn = reinterpret_cast<double*>(base);
  {
    double host[2 * MAX_RANK] = {0};
    std::memcpy(host, d->nodes, sizeof(double) * d->rank);
    std::memcpy(host + MAX_RANK, d->weights, sizeof(double) * d->rank);
    CUDA_TRY(cudaMemcpyAsync(dn, host, sizeof host, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaStreamSynchronize(st));
  }
  auto buf = [&](int k) { return reinterpret_cast<cplx*>(base + align_up(4096) + (size_t)k * plane); };
  E20Geo g;
  g.ny = ny;
  g.nx = nx;
  g.M = M;
  g.qx_step = d->qx_step;
  g.qy_step = d->qy_step;
  g.fstep = d->freq_step;
  g.b0 = d->base_bin;
  const int T = 256;
  const int eb = grid_for((size_t)total, T, 8192);
  cplx* joint = buf(0);
  CUDA_TRY(cudaMemsetAsync(joint, 0, (size_t)total * sizeof(cplx), st));
  if (nnz) {
    LaunchScope ls_("modal_scatter_kernel", st, 0.0);
    modal_scatter_kernel<<<grid_for(nnz, T, 1024), T, 0, st>>>(d_idx, d_val, nnz, joint, W, M);
  }
  LAUNCH_CHECK("modal_scatter_kernel");
  // joint fields: inverse along y and x (unnormalised), forward along the bins
  auto to_field = [&](cplx* b) -> gl_status {
    gl_status r = launch_sfft(sfft(b, ny, (long long)nx * M, 1, nx * M, 0, 1.0), 1, +1, st, tw);
    if (r != GL_OK) return r;
    r = launch_sfft(sfft(b, nx, M, 1, M, (long long)nx * M, 1.0), ny, +1, st, tw);
    if (r != GL_OK) return r;
    return axis_last_transform(b, (long long)ny * nx, M, -1, 1.0, st, tw);
  };
  auto to_spectrum = [&](cplx* b) -> gl_status {
    gl_status r = axis_last_transform(b, (long long)ny * nx, M, +1, 1.0 / M, st, tw);
    if (r != GL_OK) return r;
    r = launch_sfft(sfft(b, ny, (long long)nx * M, 1, nx * M, 0, 1.0), 1, -1, st, tw);
    if (r != GL_OK) return r;
    return launch_sfft(sfft(b, nx, M, 1, M, (long long)nx * M, 1.0 / ((double)nx * ny)), ny, -1, st, tw);
  };
  const int mults[8] = {E20_ONE, E20_NU2, E20_NU, E20_BX, E20_BY, E20_QX, E20_QY, E20_RAD};
  for (int k = 0; k < 8; ++k) {
    {
      LaunchScope ls_("e20_bank_kernel", st, 0.0);
      e20_bank_kernel<<<eb, T, 0, st>>>(g, joint, buf(1 + k), mults[k]);
    }
    LAUNCH_CHECK("e20_bank_kernel");
    if ((s = to_field(buf(1 + k))) != GL_OK) return s;
  }
  E20Forcing fo;
  fo.one = buf(1);
  fo.dno = buf(2);
  fo.nuf = buf(3);
  fo.bx = buf(4);
  fo.by = buf(5);
  fo.qxf = buf(6);
  fo.qyf = buf(7);
  fo.rad = buf(8);
  fo.fd = buf(9);
  fo.fk = buf(10);
  fo.total = total;
  {
    LaunchScope ls_("e20_forcing_kernel", st, 0.0);
    e20_forcing_kernel<<<eb, T, 0, st>>>(fo);
  }
  LAUNCH_CHECK("e20_forcing_kernel");
  if ((s = to_spectrum(fo.fd)) != GL_OK) return s;
  if ((s = to_spectrum(fo.fk)) != GL_OK) return s;
  E20Resp r;
  r.g = g;
  r.fd = fo.fd;
  r.fk = fo.fk;
  r.out = reinterpret_cast<cplx*>(d_coef);
  r.span = d->span;
  r.dq = d->dq;
  r.depth = d->depth;
  r.nodes = dn;
  r.weights = dn + MAX_RANK;
  r.rank = d->rank;
  {
    LaunchScope ls_("e20_response_kernel", st, 0.0);
    e20_response_kernel<<<W, 256, 0, st>>>(r);
  }
  LAUNCH_CHECK("e20_response_kernel");
  return GL_OK;
}

extern "C" gl_status gl_series_synthesize(int count, int n_bins, const int* d_bins, const void* d_coef,
                                          void* d_out, int real_only, void* stream) {
  if (count < 1 || n_bins < 0 || (n_bins && (!d_bins || !d_coef)) || !d_out)
    return fail(GL_ERR_INVALID_ARGUMENT, "bad series synthesis arguments");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  {
    LaunchScope ls_("series_synth_kernel", st, 0.0);
    series_synth_kernel<<<grid_for(count, 256, 1024), 256, 0, st>>>(
        d_bins, reinterpret_cast<const cplx*>(d_coef), n_bins, count, d_out, real_only);
  }
  LAUNCH_CHECK("series_synth_kernel");
  return GL_OK;
}

// ---------------------------------------------------------------------------
// box spectra -> physical grid with no device allocation
// ---------------------------------------------------------------------------
//
// Some callers cannot allocate device memory when they evaluate a field:
// code running inside a captured CUDA graph or a fixed-budget real-time
// loop, and host runtimes whose GPU bindings only hand over buffers they
// already own.  gl_box_synthesize_noalloc serves them.  Its scratch (the
// twiddle table, an unused geometry plane for the multiplier-free bank and
// the column-transformed intermediate) lives in the file-scope array below,
// which every GPU that loads this library holds until the process exits.

#define GL_NOALLOC_SCRATCH_BYTES (16u << 20)
static __device__ __align__(256) unsigned char g_noalloc_scratch[GL_NOALLOC_SCRATCH_BYTES];

static std::mutex g_noalloc_mu;
static unsigned char* g_noalloc_base[64] = {nullptr};

// Device address of the scratch array on the current device.  The first call
// on a device looks the symbol up (a host-side name is not a device address),
// fills the twiddle table and waits for it on `st`; that first call must
// therefore come before any stream capture.
static gl_status noalloc_scratch(cudaStream_t st, unsigned char** out) {
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(GL_ERR_CUDA, "device index out of range");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_base[dev]) {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr)
      return fail(GL_ERR_CUDA, "cudaGetSymbolAddress of the no-alloc scratch failed: %s",
                  cudaGetErrorString(e));
    twiddle_kernel<<<TW_N / 256, 256, 0, st>>>(reinterpret_cast<cplx*>(ptr), TW_N);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(st));
    g_noalloc_base[dev] = reinterpret_cast<unsigned char*>(ptr);
  }
  *out = g_noalloc_base[dev];
  return GL_OK;
}

extern "C" gl_status gl_box_synthesize_noalloc(int n_units, int nx, int ny, int box_x0,
                                               int box_y0, int box_w, int box_h,
                                               const void* d_box_spectra, double scale,
                                               void* d_out, int real_only, void* stream) {
  if (n_units < 0 || box_w < 1 || box_h < 1 || !d_box_spectra || !d_out)
    return fail(GL_ERR_INVALID_ARGUMENT, "bad no-alloc synthesis arguments");
  if (!is_pow2(nx) || !is_pow2(ny) || nx < 16 || ny < 16 || nx > TW_N || ny > TW_N)
    return fail(GL_ERR_UNSUPPORTED, "power-of-two grids from 16 to %d are required", TW_N);
  if (box_w > nx || box_h > ny || std::abs(box_x0) >= nx || std::abs(box_y0) >= ny ||
      std::abs(box_x0 + box_w - 1) >= nx || std::abs(box_y0 + box_h - 1) >= ny)
    return fail(GL_ERR_INVALID_ARGUMENT, "box does not fit the grid");
  const size_t tw_bytes = align_up(sizeof(cplx) * TW_N);
  const size_t geo_bytes = align_up(sizeof(double) * 6 * (size_t)box_w * box_h);
  const size_t mid_bytes = align_up(sizeof(cplx) * (size_t)n_units * box_w * ny);
  if (tw_bytes + geo_bytes + mid_bytes > GL_NOALLOC_SCRATCH_BYTES)
    return fail(GL_ERR_WORKSPACE,
                "no-alloc synthesis needs %zu bytes of scratch but its static array holds %u: "
                "use fewer units per call (n_units * box_w * ny * 16 bytes must stay below "
                "about %u bytes)",
                tw_bytes + geo_bytes + mid_bytes, GL_NOALLOC_SCRATCH_BYTES,
                (unsigned)(GL_NOALLOC_SCRATCH_BYTES - tw_bytes - geo_bytes));
  if (n_units == 0) return GL_OK;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  unsigned char* base = nullptr;
  gl_status s = noalloc_scratch(st, &base);
  if (s != GL_OK) return s;
  const cplx* tw = reinterpret_cast<const cplx*>(base);
  double* geo = reinterpret_cast<double*>(base + tw_bytes);
  cplx* mid = reinterpret_cast<cplx*>(base + tw_bytes + geo_bytes);
  // the multiplier-free bank never reads the geometry plane; clear it so the
  // kernel's loads see defined values whatever an earlier call left there
  CUDA_TRY(cudaMemsetAsync(geo, 0, geo_bytes, st));
  const Box box{box_x0, box_y0, box_w, box_h};
  ColArgs a;
  std::memset(&a, 0, sizeof a);
  a.kind = COL_PLAIN;
  a.nbanks = 1;
  a.mult[0] = M_ONE;
  a.src_of[0] = 0;
  a.box = box;
  a.geo = geo;
  a.spec = reinterpret_cast<const cplx*>(d_box_spectra);
  a.spec_job_stride = (long long)box_w * box_h;
  a.spec_sub_stride = 0;
  a.jobs_per_unit = 1;
  a.out = mid;
  a.n = ny;
  a.log2n = ilog2(ny);
  a.scale = 1.0 / ((double)nx * (double)ny);
  if ((s = launch_col_ifft(a, n_units, st, tw)) != GL_OK) return s;
  OutArgs o;
  std::memset(&o, 0, sizeof o);
  o.in = mid;
  o.w = box_w;
  o.x0 = box_x0;
  o.nx = nx;
  o.log2nx = ilog2(nx);
  o.ny = ny;
  o.ncomp = 1;
  o.comp_offset = 0;
  o.out_ncomp = 1;
  // the scale travels by value in the launch arguments
  o.comp_scale = nullptr;
  o.scale_value = scale;
  o.out = d_out;
  o.real_only = real_only ? 1 : 0;
  return launch_out_rows(o, n_units, st, tw);
}

// ---------------------------------------------------------------------------
// WIT fourth-order quartet sum (sector 44)
// ---------------------------------------------------------------------------

static std::mutex g_wit_mu;
static bool g_wit_tables[64] = {false};

// Set partitions of every subset mask, enumerated like
// directional_eta4_openmp.cpp:60-89 (assignment codes counted up with the
// mask's slots as base-b digits, least significant first; surjective only).
static gl_status wit_upload_tables() {
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_wit_mu);
  if (dev >= 0 && dev < 64 && g_wit_tables[dev]) return GL_OK;
  unsigned int parts[160];
  unsigned char off[16][5], cnt[16][5];
  std::memset(off, 0, sizeof off);
  std::memset(cnt, 0, sizeof cnt);
  int n = 0;
  for (int mask = 1; mask < 16; ++mask) {
    int slots[4], k = 0;
    for (int sl = 0; sl < 4; ++sl)
      if (mask & (1 << sl)) slots[k++] = sl;
    for (int b = 1; b <= 4; ++b) {
      off[mask][b] = (unsigned char)n;
      int total = 1;
      for (int i = 0; i < k; ++i) total *= b;
      for (int code = 0; code < total; ++code) {
        int cur = code, seen = 0;
        unsigned int blocks[4] = {0, 0, 0, 0};
        for (int i = 0; i < k; ++i) {
          const int as = cur % b;
          cur /= b;
          seen |= 1 << as;
          blocks[as] |= 1u << slots[i];
        }
        if (seen == (1 << b) - 1) {
          if (n >= 160) return fail(GL_ERR_CUDA, "partition table overflow");
          parts[n++] = blocks[0] | (blocks[1] << 8) | (blocks[2] << 16) | (blocks[3] << 24);
          cnt[mask][b] += 1;
        }
      }
    }
  }
  CUDA_TRY(cudaMemcpyToSymbol(c_wit_parts, parts, sizeof parts));
  CUDA_TRY(cudaMemcpyToSymbol(c_wit_off, off, sizeof off));
  CUDA_TRY(cudaMemcpyToSymbol(c_wit_cnt, cnt, sizeof cnt));
  if (dev >= 0 && dev < 64) g_wit_tables[dev] = true;
  return GL_OK;
}

static size_t wit_binom_stride(int n_modes) { return (size_t)n_modes + 4; }

extern "C" size_t gl_wit_workspace_size(int n_modes) {
  if (n_modes < 1) return 0;
  return align_up(sizeof(WitStats)) + 5 * wit_binom_stride(n_modes) * sizeof(unsigned long long);
}

extern "C" gl_status gl_wit_read_sector_stats(int sector, const void* d_work, int n_modes,
                                              gl_wit_stats* out);

static unsigned long long wit_candidates(int sector, unsigned long long n) {
  if (sector == 40) {
    const unsigned long long p = n * (n + 1) / 2;
    return p * p;
  }
  if (sector == 42) return n * (n + 1) * (n + 2) / 6 * n;
  return n * (n + 1) * (n + 2) * (n + 3) / 24;
}

extern "C" unsigned long long gl_wit_candidates(int sector, int n_modes) {
  if ((sector != 40 && sector != 42 && sector != 44) || n_modes < 1) return 0;
  return wit_candidates(sector, (unsigned long long)n_modes);
}

extern "C" gl_status gl_wit_sector_range(int sector, int n_modes, const int* d_modes, int n_cases,
                                         const void* d_amp, int nx, int ny, double gravity,
                                         double depth, double dkx, double dky, double threshold,
                                         unsigned long long q_begin, unsigned long long q_end,
                                         void* d_out, void* d_work, size_t work_bytes, void* stream);

extern "C" gl_status gl_wit_sector(int sector, int n_modes, const int* d_modes, int n_cases,
                                   const void* d_amp, int nx, int ny, double gravity, double depth,
                                   double dkx, double dky, double threshold, void* d_out,
                                   void* d_work, size_t work_bytes, void* stream) {
  const unsigned long long all = n_modes > 0 ? wit_candidates(sector, (unsigned long long)n_modes) : 0;
  return gl_wit_sector_range(sector, n_modes, d_modes, n_cases, d_amp, nx, ny, gravity, depth, dkx,
                             dky, threshold, 0, all, d_out, d_work, work_bytes, stream);
}

extern "C" gl_status gl_wit_eta44(int n_modes, const int* d_modes, int n_cases, const void* d_amp,
                                  int nx, int ny, double gravity, double depth, double dkx,
                                  double dky, double threshold, void* d_out, void* d_work,
                                  size_t work_bytes, void* stream) {
  return gl_wit_sector(44, n_modes, d_modes, n_cases, d_amp, nx, ny, gravity, depth, dkx, dky,
                       threshold, d_out, d_work, work_bytes, stream);
}

extern "C" gl_status gl_wit_sector_range(int sector, int n_modes, const int* d_modes, int n_cases,
                                         const void* d_amp, int nx, int ny, double gravity,
                                         double depth, double dkx, double dky, double threshold,
                                         unsigned long long q_begin, unsigned long long q_end,
                                         void* d_out, void* d_work, size_t work_bytes, void* stream) {
  if (sector != 40 && sector != 42 && sector != 44)
    return fail(GL_ERR_SECTOR, "sector must be 40, 42, or 44");
  if (n_modes < 1 || n_modes > 65535 || n_cases < 1 || !d_modes || !d_amp || !d_out || !d_work)
    return fail(GL_ERR_INVALID_ARGUMENT, "bad WIT arguments (modes 1..65535, cases >= 1, non-null buffers)");
  if (nx < 2 || ny < 2 || (nx % 2) || (ny % 2))
    return fail(GL_ERR_INVALID_ARGUMENT, "WIT grid sizes must be positive and even");
  if (!(gravity > 0) || !(depth > 0) || !(dkx > 0) || !(dky > 0) || !(threshold > 0))
    return fail(GL_ERR_INVALID_ARGUMENT, "gravity, depth, dk and the resonance threshold must be positive");
  if (work_bytes < gl_wit_workspace_size(n_modes))
    return fail(GL_ERR_WORKSPACE, "WIT workspace needs %zu bytes", gl_wit_workspace_size(n_modes));
  if (q_begin > q_end || q_end > wit_candidates(sector, (unsigned long long)n_modes))
    return fail(GL_ERR_INVALID_ARGUMENT, "quartet range [%llu, %llu) outside the sector's %llu candidates",
                q_begin, q_end, wit_candidates(sector, (unsigned long long)n_modes));
  gl_status s = wit_upload_tables();
  if (s != GL_OK) return s;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const size_t stride = wit_binom_stride(n_modes);
  std::vector<unsigned long long> binom(5 * stride, 0ull);
  for (size_t v = 0; v < stride; ++v) {
    binom[v] = 1;
    for (int r = 1; r <= 4; ++r)
      binom[r * stride + v] = v == 0 ? 0ull : binom[r * stride + v - 1] + binom[(r - 1) * stride + v - 1];
  }
  WitStats init;
  std::memset(&init, 0, sizeof init);
  init.min_detuning = BITS_POS_INF;
  char* work = reinterpret_cast<char*>(d_work);
  unsigned long long* d_binom = reinterpret_cast<unsigned long long*>(work + align_up(sizeof(WitStats)));
  CUDA_TRY(cudaMemcpyAsync(work, &init, sizeof init, cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(d_binom, binom.data(), binom.size() * sizeof(unsigned long long),
                           cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaMemsetAsync(d_out, 0, sizeof(cplx) * 5 * (size_t)n_cases * nx * ny, st));
  CUDA_TRY(cudaStreamSynchronize(st));  // host staging buffers above go out of scope
  WitArgs a;
  a.n_modes = n_modes;
  a.modes = d_modes;
  a.n_cases = n_cases;
  a.amp = reinterpret_cast<const cplx*>(d_amp);
  a.nx = nx;
  a.ny = ny;
  a.dkx = dkx;
  a.dky = dky;
  a.thr = threshold;
  a.M = WitModel{gravity, depth};
  a.out = reinterpret_cast<cplx*>(d_out);
  a.stats = reinterpret_cast<WitStats*>(work);
  a.q_begin = q_begin;
  a.n_quartets = q_end;
  a.binom = d_binom;
  a.binom_stride = (int)stride;
  a.sector = sector;
  if (q_end == q_begin) return GL_OK;  // an empty share: zero fields, zero counts
  const int blocks = (int)std::min<unsigned long long>((q_end - q_begin + 127) / 128, 148ull * 32);
  {
    LaunchScope ls("wit44_kernel", st, 0.0);
    wit44_kernel<<<blocks, 128, 0, st>>>(a);
  }
  LAUNCH_CHECK("wit44_kernel");
  return GL_OK;
}

extern "C" gl_status gl_wit_read_stats(const void* d_work, int n_modes, gl_wit_stats* out) {
  return gl_wit_read_sector_stats(44, d_work, n_modes, out);
}

extern "C" gl_status gl_wit_read_sector_stats(int sector, const void* d_work, int n_modes,
                                              gl_wit_stats* out) {
  if (!d_work || !out || n_modes < 1) return fail(GL_ERR_INVALID_ARGUMENT, "bad WIT stats arguments");
  WitStats w;
  CUDA_TRY(cudaMemcpy(&w, d_work, sizeof w, cudaMemcpyDeviceToHost));
  out->candidates = wit_candidates(sector, (unsigned long long)n_modes);
  out->kept = w.kept;
  out->near = w.near;
  out->strict_zero_output = w.strict_zero_output;
  out->strict_zero_intermediate = w.strict_zero_intermediate;
  double t;
  std::memcpy(&t, &w.max_residual, sizeof t);
  out->max_residual = t;
  std::memcpy(&t, &w.min_detuning, sizeof t);
  out->min_detuning = t;
  std::memcpy(&t, &w.max_strict_src, sizeof t);
  out->max_strict_zero_source = t;
  return GL_OK;
}

extern "C" gl_status gl_gauss_laguerre(int rank, double* nodes, double* weights) {
  if (!nodes || !weights) return fail(GL_ERR_INVALID_ARGUMENT, "null output");
  return gauss_laguerre(rank, nodes, weights);
}

// Newton iteration of dispersion.py:19-42 (40 steps, damped to q/2, rtol gate).
extern "C" gl_status gl_dispersion_solve(int n, const double* omega, double depth, double gravity,
                                         double* q_out) {
  if (n < 0 || (n && (!omega || !q_out))) return fail(GL_ERR_INVALID_ARGUMENT, "bad arguments");
  if (!(depth > 0) || !(gravity > 0))
    return fail(GL_ERR_INVALID_ARGUMENT, "depth and gravity must be positive and omega nonnegative");
  const double tiny = 2.2250738585072014e-308;
  std::vector<double> target(n), q(n);
  for (int i = 0; i < n; ++i) {
    if (!(omega[i] >= 0))
      return fail(GL_ERR_INVALID_ARGUMENT, "depth and gravity must be positive and omega nonnegative");
    target[i] = omega[i] * omega[i] * depth / gravity;
    q[i] = std::max(target[i] < 1.0 ? std::sqrt(target[i]) : target[i], tiny);
  }
  for (int it = 0; it < 40; ++it) {
    double worst = 0.0;
    for (int i = 0; i < n; ++i) {
      const double t = std::tanh(q[i]);
      const double res = q[i] * t - target[i];
      const double der = t + q[i] * (1.0 - t * t);
      const double upd = res / std::max(der, tiny);
      const double cand = std::max(q[i] - upd, 0.5 * q[i]);
      worst = std::max(worst, std::fabs(cand - q[i]) / std::max(1.0, q[i]));
      q[i] = cand;
    }
    if (worst < 5.0e-15) break;
  }
  for (int i = 0; i < n; ++i) {
    const double lhs = q[i] * std::tanh(q[i]);
    if (!(std::fabs(lhs - target[i]) <= 2.0e-15 + 2.0e-13 * std::fabs(target[i])))
      return fail(GL_ERR_INVALID_ARGUMENT, "finite-depth dispersion solve did not converge");
    q_out[i] = q[i];
  }
  return GL_OK;
}

extern "C" size_t gl_get_last_error(char* buffer, size_t length) {
  if (buffer && length) {
    const size_t n = std::min(length - 1, g_last_error.size());
    std::memcpy(buffer, g_last_error.data(), n);
    buffer[n] = 0;
  }
  return g_last_error.size();
}

extern "C" const char* gl_version(void) { return "gl-b200 0.1.0 (sm_100a)"; }
