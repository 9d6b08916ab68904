// Host-side internals shared by the engine's translation units: error
// plumbing, launch accounting, grid helpers, per-device kernel attributes and
// the transform launchers (defined in gl_launch_cols.cu and gl_rows_*.cu, so
// the heavy kernel instantiations compile in parallel).
//
// Translation units that compile transform kernels (rows, columns, final
// rows, adjoint column combines, strided transforms) define GL_TRANSFORM_TU
// before their includes: the kernel headers then leave out their elementwise
// kernels, which gl_engine.cu alone compiles and launches.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstddef>
#include <mutex>
#include <vector>

#include "../../include/gl_engine.h"
#include "gl_kernels.cuh"

namespace gl {

struct SeedArgs;
struct CmbArgs;
struct SFft;

// ---------------------------------------------------------------------------
// errors: a thread-local message plus the returned status
// ---------------------------------------------------------------------------

gl_status fail(gl_status s, const char* fmt, ...);

#define CUDA_TRY(expr)                                                               \
  do {                                                                               \
    cudaError_t e_ = (expr);                                                         \
    if (e_ != cudaSuccess)                                                           \
      return ::gl::fail(GL_ERR_CUDA, "%s failed: %s", #expr, cudaGetErrorString(e_)); \
  } while (0)

#define LAUNCH_CHECK(what)                                                           \
  do {                                                                               \
    cudaError_t e_ = cudaGetLastError();                                             \
    if (e_ != cudaSuccess)                                                           \
      return ::gl::fail(GL_ERR_CUDA, "launch of %s failed: %s", what, cudaGetErrorString(e_)); \
  } while (0)

// ---------------------------------------------------------------------------
// launch accounting: a launch counter and optional per-kernel event timing
// ---------------------------------------------------------------------------

struct ProfRecord {
  const char* name;
  cudaEvent_t start, stop;
  double bytes;
};
extern std::atomic<unsigned long long> g_launches;
extern std::mutex g_prof_mu;
extern bool g_prof_on;
extern std::vector<ProfRecord> g_prof;

// Wraps one kernel launch: counts it and, while profiling, brackets it with
// events on its own stream.  `bytes` is the launch's algorithmic traffic.
struct LaunchScope {
  const char* name;
  cudaStream_t st;
  double bytes;
  cudaEvent_t a = nullptr, b = nullptr;
  LaunchScope(const char* n, cudaStream_t s, double by) : name(n), st(s), bytes(by) {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (g_prof_on) {
      cudaEventCreate(&a);
      cudaEventCreate(&b);
      cudaEventRecord(a, st);
    }
  }
  ~LaunchScope() {
    if (a) {
      cudaEventRecord(b, st);
      std::lock_guard<std::mutex> lk(g_prof_mu);
      g_prof.push_back(ProfRecord{name, a, b, bytes});
    }
  }
};

// Raises a kernel's dynamic shared-memory ceiling to `bytes` on the current
// device, once per (device, kernel, size).  The attribute belongs to the
// device's context, so a second device in the same process needs its own
// call; the record is guarded by a mutex so plans on different threads may
// launch concurrently.  Returns the attribute call's error, if any.
cudaError_t ensure_smem_attr(const void* kernel, int bytes);

// ---------------------------------------------------------------------------
// sizes and grids
// ---------------------------------------------------------------------------

inline int ilog2(int v) {
  int l = 0;
  while ((1 << l) < v) ++l;
  return l;
}
inline bool is_pow2(int v) { return v > 0 && (v & (v - 1)) == 0; }
inline int next_pow2(int v) {
  int p = 1;
  while (p < v) p <<= 1;
  return p;
}
inline size_t align_up(size_t v) { return (v + 255) & ~(size_t)255; }

constexpr int ROW_GMAX = 4;
constexpr size_t SMEM_LIMIT = 227 * 1024;
// row kernels also hold a static mbarrier: their dynamic budget leaves 1 KB
constexpr size_t ROW_SMEM_LIMIT = SMEM_LIMIT - 1024;

inline size_t row_smem(int nbanks, int ncx) { return (size_t)nbanks * padded_len(ncx) * sizeof(cplx); }

inline int grid_for(size_t n, int threads, int cap = 4096) {
  size_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > (size_t)cap) b = cap;
  return (int)b;
}

inline int fft_cols_per_block(int n, int w) {
  const int T = is_pow2(n) ? n / 16 : 16;  // threads per column transform
  // a power of two (the kernels split thread indices with shifts)
  return std::max(1, std::min(256 / T, next_pow2(w)));
}

// Kernels instantiated per mixed radix (MIX = n/16 for the mixed lengths, 0
// for powers of two).
#define GL_MIX_DISPATCH(n, launcher, ...)                                   \
  switch (mixed_len(n) ? (n) / 16 : 0) {                                   \
    case 3: launcher<3>(__VA_ARGS__); break;                               \
    case 5: launcher<5>(__VA_ARGS__); break;                               \
    case 6: launcher<6>(__VA_ARGS__); break;                               \
    case 9: launcher<9>(__VA_ARGS__); break;                               \
    case 10: launcher<10>(__VA_ARGS__); break;                             \
    case 12: launcher<12>(__VA_ARGS__); break;                             \
    case 15: launcher<15>(__VA_ARGS__); break;                             \
    default: launcher<0>(__VA_ARGS__); break;                              \
  }

// ---------------------------------------------------------------------------
// transform launchers
// ---------------------------------------------------------------------------

gl_status launch_col_ifft(const ColArgs& a, int njobs, cudaStream_t st, const cplx* tw);
gl_status launch_col_fft(const ColFftArgs& a, int njs, cudaStream_t st, const cplx* tw,
                         const char* name = "col_fft_kernel");
gl_status launch_row(const RowArgs& a, int njobs, cudaStream_t st, const cplx* tw);
gl_status launch_out_rows(const OutArgs& a0, int nuc, cudaStream_t st, const cplx* tw);
gl_status launch_seed_rows(const SeedArgs& a, int nunits, cudaStream_t st, const cplx* tw);
gl_status launch_combine(const CmbArgs& a, int njobs, cudaStream_t st, const cplx* tw);
gl_status launch_sfft(const SFft& a, int outer, int sign, cudaStream_t st, const cplx* tw);
// Final transforms of reference grids that are not powers of two (gl_gen.cuh).
struct GenColArgs;
struct GenRowArgs;
gl_status launch_gen_cols(const GenColArgs& a, int njobs, cudaStream_t st);
gl_status launch_gen_rows(const GenRowArgs& a, int nuc, cudaStream_t st);

// Row launches by kind family, one translation unit each.  Each returns
// false when `a.kind` is not in its family or its row length has no
// instantiation; `smem` is the per-row dynamic shared memory.
bool row_dispatch_pair(const RowArgs& a, dim3 grid, int T, size_t smem, cudaStream_t st, const cplx* tw);
bool row_dispatch_wide(const RowArgs& a, dim3 grid, int T, size_t smem, cudaStream_t st, const cplx* tw);
bool row_dispatch_adj(const RowArgs& a, dim3 grid, int T, size_t smem, cudaStream_t st, const cplx* tw);

}  // namespace gl
