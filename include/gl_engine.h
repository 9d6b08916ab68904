/*
 * gl_engine.h -- C ABI of the B200 Green--Laplace (GL) bound-wave engine.
 *
 * The engine evaluates the reference's spatial GL graphs on the GPU:
 * first order (eta11, psi11), the prescribed-rank eta22, the dual-branch
 * psi22 and the nested no-Stokes eta33 + psi33.  Every entry point takes
 * plain pointers and sizes; device buffers are owned by the caller and
 * complex values are interleaved float64 pairs.
 *
 * Reference interfaces replaced (Xinyu01091002/green-laplace-wave-reconstruction):
 *   gl_plan_create/gl_execute   src/gl_spectral_surface.m:1-103 (stage 2 of the
 *                               two-stage API) and its executors
 *                               src/internal/green_laplace_eta22.m:1-79,
 *                               ...dual_branch_green_laplace_psi22.m:1-265,
 *                               src/internal/gl_no_stokes_eta33.m:1-274;
 *                               Python python/src/green_laplace/spatial.py:33-414
 *                               and _order3.py:18-297
 *   gl_deposit_modes            src/gl_spectral_surface.m:123-149 (deposit_analytic_input)
 *   gl_gauss_laguerre           python/src/green_laplace/quadrature.py:11-31
 *   gl_dispersion_solve         python/src/green_laplace/dispersion.py:19-42
 *   gl_status codes             the MATLAB 'green_laplace:<Id>' identifiers of
 *                               src/gl_spectral_coefficients.m:9-70 and
 *                               src/gl_spectral_surface.m:135-141
 */
#ifndef GL_ENGINE_H
#define GL_ENGINE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum gl_status {
  GL_OK = 0,
  GL_ERR_INVALID_ARGUMENT = 1,  /* null pointer, bad size or enum value          */
  GL_ERR_UNSUPPORTED = 2,       /* grid size / layout this engine does not run    */
  GL_ERR_OPTIONS = 3,           /* green_laplace:Options, UnknownOption           */
  GL_ERR_UNIFORM_CURRENT = 4,   /* green_laplace:UniformCurrent                   */
  GL_ERR_COMPONENT_SIZE = 5,    /* green_laplace:ComponentSize                    */
  GL_ERR_COMPONENTS = 6,        /* green_laplace:Components                       */
  GL_ERR_SUPPORT = 7,           /* green_laplace:Support (strict-forward kx>0)    */
  GL_ERR_SECTOR = 8,            /* green_laplace:Sector                           */
  GL_ERR_ZERO_INPUT = 9,        /* green_laplace:ZeroInput                        */
  GL_ERR_ORDER2_DOMAIN = 10,    /* green_laplace:Order2Domain (kh >= 0.3)         */
  GL_ERR_ORDER3_DOMAIN = 11,    /* green_laplace:Order3Domain (kh > 0.5)          */
  GL_ERR_OFF_GRID = 12,         /* green_laplace:OffGridComponent                 */
  GL_ERR_NYQUIST = 13,          /* green_laplace:Nyquist                          */
  GL_ERR_ALIAS = 14,            /* quadratic/cubic output support reaches Nyquist */
  GL_ERR_SCALE = 15,            /* invalid GL tail scale                          */
  GL_ERR_RANK = 16,             /* unsupported quadrature rank                    */
  GL_ERR_EMPTY_SUPPORT = 17,    /* empty analytic support                         */
  GL_ERR_OUTSIDE_PLAN = 18,     /* spectrum support outside the plan's box        */
  GL_ERR_NONFINITE = 19,        /* non-finite value in an output field            */
  GL_ERR_WORKSPACE = 20,        /* workspace too small or misaligned              */
  GL_ERR_CUDA = 21,             /* CUDA runtime error                             */
  GL_ERR_TIMEOUT = 22,          /* a bounded device wait ran out                  */
  GL_ERR_COEFFICIENTS = 23      /* green_laplace:Coefficients                     */
} gl_status;

/* component bits (output order follows the bit order) */
#define GL_COMP_ETA11 0x01
#define GL_COMP_PSI11 0x02
#define GL_COMP_ETA22 0x04
#define GL_COMP_PSI22 0x08
#define GL_COMP_ETA33 0x10
#define GL_COMP_PSI33 0x20
#define GL_COMP_ETA44 0x40  /* fourth-order plans (gl_eta44_plan_create) */
#define GL_COMP_PSI44 0x80  /* fourth-order surface potential (same plans)  */

#define GL_GRID_COMPACT 0   /* smallest alias-free power-of-two product grid */
#define GL_GRID_REFERENCE 1 /* products on the reference's own Nx x Ny grid   */

#define GL_OUT_COMPLEX 0    /* analytic "plus" fields, complex128            */
#define GL_OUT_REAL 1       /* real parts only, float64                      */

#define GL_SPECTRA_FULL 0   /* [unit][ny][nx] complex128, numpy fft2 layout  */
#define GL_SPECTRA_BOX 1    /* [unit][box_h][box_w] complex128               */

typedef struct gl_plan gl_plan;

typedef struct gl_plan_desc {
  int nx, ny;                 /* reference grid: even, 16..4096, prime
                                 factors 2, 3, 5 only                        */
  double lx, ly;              /* periodic domain lengths                    */
  double depth, gravity;      /* h, g                                       */
  int order;                  /* 1, 2 or 3                                  */
  int components;             /* GL_COMP_* mask (0 = all for the order)     */
  int eta22_rank;             /* 1..16 (reference default 6)                */
  int inner_rank;             /* order 3: 4,6,8,10,12 (default 4)           */
  int outer_rank;             /* order 3: 3,4,6,8,10 (default 4)            */
  int allow_below_model_parent_domain;
  int box_x0, box_y0;         /* parent support box: signed mode numbers    */
  int box_w, box_h;
  int grid;                   /* GL_GRID_*                                   */
  int max_units;              /* units processed per internal group (>=1)   */
  int output;                 /* GL_OUT_*                                    */
} gl_plan_desc;

typedef struct gl_plan_info {
  int ncx, ncy;               /* product grid actually used                 */
  int box1[4], box2[4], box3[4];  /* x0, y0, w, h of parent/pair/triple boxes */
  int n_components;           /* output planes per unit                     */
  int component_ids[6];       /* GL_COMP_* of each plane, in order          */
  double transforms_per_unit; /* 2-D transforms of the reference graph      */
  int ncy_pair, ncy_triple;   /* column lengths of the pair and triple stages
                                 (ncy or a mixed length 16 m <= ncy)         */
  int ncx_pair;               /* row length of the pair stages (<= ncx)     */
} gl_plan_info;

/* Create a plan: validates the descriptor, picks the product grid, builds
 * geometry tables, twiddles and GL node tables on the current device. */
gl_status gl_plan_create(gl_plan** plan, const gl_plan_desc* desc);
void gl_plan_destroy(gl_plan* plan);
gl_status gl_plan_get_info(const gl_plan* plan, gl_plan_info* info);

/* Fourth-order pure-sum eta44 (no Stokes corrections) at GL rank R for all
 * three nested levels.  Replaces paper/order4/cpp/gl_eta44_fftw.cpp (the
 * GLRTI001 -> GLE44O01 executor, lines 76-749) and its MATLAB authority
 * src/internal/finite_depth_directional_green_laplace_eta44_three_kernels.m.
 * Conventions follow the C++: qx = (depth dk) mx, the peak depth is supplied,
 * the square grid is n x n.  The plan runs through gl_execute: inputs are the
 * N^2-scaled analytic spectra (full [ny][nx] or box), the output is the
 * analytic eta44 field times depth, [unit][component][ny][nx].
 * With components = GL_COMP_ETA44 | GL_COMP_PSI44 the plan also evaluates the
 * surface potential psi44 of src/gl_pure_sum_order4.m:1-15 (contact terms of
 * ...eta44_three_kernels.m:93-111, 221-241; the C++ has no psi44), as a second
 * plane scaled by depth * sqrt(gravity * depth). */
typedef struct gl_eta44_desc {
  int n;                      /* square grid (power of two)                   */
  double dk, depth, peak_depth;
  int rank;                   /* GL rank of every level (paper: 6, 8, 10)     */
  const double* nodes;        /* optional host rule of length rank (NULL:     */
  const double* weights;      /* the engine's Golub--Welsch rule)             */
  int box_x0, box_y0, box_w, box_h;
  int max_units;
  int output;                 /* GL_OUT_*                                      */
  int components;             /* 0 or GL_COMP_ETA44 [| GL_COMP_PSI44]          */
  double gravity;             /* psi44 scale (> 0 when psi44 is requested)     */
} gl_eta44_desc;

gl_status gl_eta44_plan_create(gl_plan** plan, const gl_eta44_desc* desc);

/* Outer-node sharding of an eta44 plan (the device analogue of the reference's
 * process split, paper/order4/run_gl_split.sh:31-38 + merge_eta44_outer.cpp:12).
 * gl_eta44_execute_partial accumulates the order-4 spectra of outer nodes
 * [outer_begin, outer_end) into d_partial ([unit][component][box4_h][box4_w]
 * complex128, box4 = 4 x the parent box), before the final roundoff floor; summing the
 * partials of a partition of [0, rank) (one NCCL all-reduce across GPUs) and
 * calling gl_eta44_finalize gives the monolithic result. */
gl_status gl_eta44_execute_partial(gl_plan* plan, int n_units, const void* d_spectra,
                                   int spectra_layout, int outer_begin, int outer_end,
                                   void* d_partial, void* d_workspace, size_t workspace_bytes,
                                   int* d_unit_status, void* stream);
/* One part of the reference's split mode (gl_eta44_fftw.cpp:639-647, the
 * OUTER4_INDEX [PART_INDEX] arguments driven by paper/order4/run_gl_split.sh:
 * 31-38): outer node `outer_index` alone, and of its quartic forcing every
 * partition (part_index -2), the base partitions 22, 211 and 1111 (-1), or
 * partition 31 with the third-level node part_index alone (0 .. rank-1, its
 * third state floored on its own).  Writes that part's order-4 spectra to
 * d_partial like gl_eta44_execute_partial; gl_eta44_finalize on it gives the
 * part's field, which is what the reference writes per part and
 * merge_eta44_outer.cpp sums.  eta44 plans only (no psi44). */
gl_status gl_eta44_execute_part(gl_plan* plan, int n_units, const void* d_spectra,
                                int spectra_layout, int outer_index, int part_index,
                                void* d_partial, void* d_workspace, size_t workspace_bytes,
                                int* d_unit_status, void* stream);
gl_status gl_eta44_finalize(gl_plan* plan, int n_units, const void* d_partial_sum,
                            void* d_outputs, void* d_workspace, size_t workspace_bytes,
                            void* stream);

/* Device workspace bytes needed by gl_execute (independent of n_units). */
gl_status gl_workspace_size(const gl_plan* plan, size_t* bytes);

/* Launch shapes of a plan's transform kernels, picked by a tuner (no
 * counterpart in the reference; the batch autotuner of gl_engine/batch.py
 * times them per plan shape).  Zero keeps the built-in choice.  Results do
 * not depend on these: only how the rows and columns are spread over
 * blocks. */
typedef struct gl_tuning {
  int pair_row_groups;    /* transform groups per row block of the pair stages
                             (eta22, psi22, order-3 inner): 0, 2, 4, 8, 16   */
  int triple_row_groups;  /* the same for the order-3 outer rows: 0, 4, 6, 8,
                             12, 16                                         */
  int col_block_columns;  /* at most this many columns per column-transform
                             block: 0, 1, 2, 4, 8, 16                        */
} gl_tuning;
gl_status gl_plan_set_tuning(gl_plan* plan, const gl_tuning* tuning);

/* Concurrent lanes of an order-1..3 plan (no counterpart in the reference,
 * whose Python evaluates one snapshot at a time).  With lanes = L > 1,
 * gl_execute splits its units into groups of ceil(max_units / L) and runs
 * group i on lane i mod L: lane 0 on the caller's stream, the others on
 * streams the plan owns, forked from the caller's stream by an event and
 * joined back to it before gl_execute returns (inside a stream capture these
 * are parallel branches of the graph).  One stage's kernels then overlap
 * another group's, e.g. the memory-bound floor/accumulation kernels with the
 * transforms.  Outputs are bitwise those of lanes = 1.  The workspace becomes
 * L regions of one group each (about the size of one max_units group):
 * query gl_workspace_size again after this call.  1 <= lanes <= GL_MAX_LANES
 * (more lanes than max_units run as max_units lanes of one unit); eta44
 * plans return GL_ERR_UNSUPPORTED.  Not to be called while a
 * gl_execute on the same plan is being enqueued. */
#define GL_MAX_LANES 8
gl_status gl_plan_set_lanes(gl_plan* plan, int lanes);

/* Failure-path test hook of the row stages' bounded waits (no counterpart in
 * the reference; its C++ has no device waits).  With surplus_bytes > 0 every
 * order-2/3 row launch of this plan expects that many bytes more than its
 * staged copies deliver, so its wait on them runs out after wait_cycles SM
 * clocks; the block then marks its unit GL_ERR_TIMEOUT in d_unit_status and
 * returns with the context intact.  (0, 0) restores normal runs (the wait's
 * budget is then about 2 s).  Nothing faults and nothing waits without a
 * bound; the outputs of a timed-out unit are meaningless. */
gl_status gl_plan_set_wait_test(gl_plan* plan, unsigned int surplus_bytes, long long wait_cycles);

/* Deposit N^2 (a+ib)/h e^{-i omega t} for n_units time snapshots into box
 * spectra [unit][box_h][box_w].  Modes are grouped by destination bin:
 * segment s covers modes seg_offsets[s] .. seg_offsets[s+1]-1 (summed in
 * that order) and lands on box bin seg_bins[s] (row-major box index).
 * d_ab holds (a, b) pairs per mode, d_omega the frequencies, d_times the
 * unit times.  The output is fully overwritten. */
gl_status gl_deposit_modes(const gl_plan* plan, int n_units, int n_segments,
                           const int* d_seg_offsets, const int* d_seg_bins, int n_modes,
                           const double* d_ab, const double* d_omega, const double* d_times,
                           void* d_box_spectra, void* stream);

/* Evaluate the plan's components for n_units analytic spectra.  d_outputs
 * receives [unit][n_components][ny][nx] (complex128 or float64 per the plan's
 * output mode) in physical units (eta in metres, psi = phi(x, z=eta, t)).
 * d_unit_status (n_units ints, may be null) receives a gl_status per unit;
 * the call itself is asynchronous on `stream` (a cudaStream_t). */
gl_status gl_execute(gl_plan* plan, int n_units, const void* d_spectra, int spectra_layout,
                     void* d_outputs, void* d_workspace, size_t workspace_bytes,
                     int* d_unit_status, void* stream);

/* Reverse mode of gl_execute for the eta components.  The reference has no
 * gradient path; this is the adjoint of the spatial graph it evaluates
 * (src/gl_spectral_surface.m:26-82: eta11 + the eta22 executor
 * src/internal/green_laplace_eta22.m:1-79 + the eta33 executor
 * src/internal/gl_no_stokes_eta33.m:1-274; Python spatial.py:156-231,
 * _order3.py:18-297).  For a real loss L of the physical field
 * eta = sum of the plan's eta components (psi components are ignored),
 * d_residual = dL/deta ([unit][ny][nx] float64) gives
 * d_grad = g ([unit][box_h][box_w] complex128 on the parent box) with
 * dL = Re(sum_k g_k ds_k) for perturbations ds of the box spectra, the
 * supports, balance shifts, scales, peak and roundoff-floor decisions held at
 * their values for the given spectra.  The call re-evaluates the forward
 * node stages it needs (no state is kept from gl_execute).  Workspace:
 * gl_adjoint_workspace_size bytes, 256-byte aligned. */
gl_status gl_adjoint_workspace_size(const gl_plan* plan, size_t* bytes);
gl_status gl_adjoint_execute(gl_plan* plan, int n_units, const void* d_spectra, int spectra_layout,
                             const double* d_residual, void* d_grad, void* d_workspace,
                             size_t workspace_bytes, int* d_unit_status, void* stream);

/* Transpose of gl_deposit_modes: d_gab ([mode][2] float64, the deposit's
 * mode order) = (dL/da, dL/db) summed over the n_units snapshots, from the
 * box-spectrum gradient d_grad of gl_adjoint_execute. */
gl_status gl_deposit_modes_adjoint(const gl_plan* plan, int n_units, int n_segments,
                                   const int* d_seg_offsets, const int* d_seg_bins, int n_modes,
                                   const double* d_omega, const double* d_times,
                                   const void* d_grad, double* d_gab, void* stream);

/* Single-direction time path: one level of the modal GL resolvent of
 * python/src/green_laplace/modal_time.py:217-360 (_modal_sum_components).
 * The caller selects the record's DFT band and deposits its amplitudes onto
 * the modal q-axis (d_idx = row * width + work bin, rows in numpy's
 * ifftshift order, d_val = complex pairs, indices distinct); the call
 * evaluates the order-2 (and order-3) graph on the joint (q, bin) grid and
 * writes the analytic eta22 (eta33) time series, count complex128 samples
 * each, i.e. numpy.fft.fft of the output-bin coefficients. */
typedef struct gl_modal_desc {
  int points;                 /* modal q nodes P (power of two, 16 .. 2^24)  */
  int width;                  /* work bins W = order * max work bin + 1      */
  int order;                  /* 2 or 3                                      */
  int base_bin;               /* first retained DFT bin                      */
  int count;                  /* samples of the record                      */
  double q_step;              /* q-axis spacing                              */
  double freq_step;           /* 2 pi / (count dt) sqrt(depth / gravity)     */
  double depth;
  double scale22, lambda2, lambda3;  /* GL scales (standalone eta22, inner, outer) */
  int rank;                   /* GL rank                                     */
  const double* nodes;        /* host GL rule of length rank                 */
  const double* weights;
} gl_modal_desc;
gl_status gl_modal_workspace_size(const gl_modal_desc* desc, size_t* bytes);
gl_status gl_modal_level(const gl_modal_desc* desc, int nnz, const long long* d_idx,
                         const double* d_val, void* d_eta22, void* d_eta33, void* d_workspace,
                         size_t workspace_bytes, void* stream);

/* Difference-frequency eta20 on a 2-D modal grid (python/src/green_laplace/
 * _eta20.py:13-143, unidirectional_eta20): deposit indices
 * (iy * nx + ix) * (2 span + 1) + work bin; d_coef receives the 2 span + 1
 * output coefficients at signed bins 0..span, -span..-1 (before the
 * Hermitian projection of _eta20.py:170-180). */
typedef struct gl_eta20_desc {
  int nx, ny;                 /* modal grid (powers of two, 16 .. 4096)      */
  int span;                   /* max work bin                                */
  int base_bin, count;
  double qx_step, qy_step, freq_step, depth;
  double dq;                  /* rms pair wavenumber spread (the GL scale)   */
  int rank;
  const double* nodes;        /* host GL rule                                */
  const double* weights;
} gl_eta20_desc;
gl_status gl_eta20_workspace_size(const gl_eta20_desc* desc, size_t* bytes);
gl_status gl_eta20_level(const gl_eta20_desc* desc, int nnz, const long long* d_idx,
                         const double* d_val, void* d_coef, void* d_workspace,
                         size_t workspace_bytes, void* stream);

/* out[n] = sum_b coef_b exp(-2 pi i bins_b n / count), n < count (a sparse
 * numpy.fft.fft; real parts only when real_only != 0). */
gl_status gl_series_synthesize(int count, int n_bins, const int* d_bins, const void* d_coef,
                               void* d_out, int real_only, void* stream);

/* Batched 2-D complex FFT on [batch][ny][nx] complex128 with numpy's
 * conventions: forward = fft2 (unnormalised), inverse = ifft2 (1/(nx ny)).
 * In-place (d_in == d_out) is allowed.  Replaces the numpy.fft.fft2/ifft2
 * calls of python/src/green_laplace/_spectral.py:29-37. */
gl_status gl_fft2(int batch, int nx, int ny, const void* d_in, void* d_out, int inverse,
                  void* stream);

/* Physical fields from box spectra without allocating device memory.
 * No counterpart in the reference.  It serves callers that cannot call
 * cudaMalloc while they run: a real-time loop with a fixed memory budget,
 * where an allocation may synchronise the device and miss a deadline, or a
 * host runtime whose GPU binding only passes buffers it already owns and
 * allows no allocation behind its own allocator.  out[u] = scale * ifft2(S_u)
 * on the nx x ny grid, S_u being box spectrum u ([n_units][box_h][box_w]
 * complex128, signed-mode origin box_x0, box_y0) embedded at its modes; out is
 * [n_units][ny][nx] complex128, or float64 real parts when real_only != 0.
 * The same transform gl_execute applies to its final spectra.
 * Scratch: one static device array of 16 MiB per GPU (held until the process
 * exits); n_units * box_w * ny * 16 bytes plus ~66 KB of tables must fit, and
 * larger requests return GL_ERR_WORKSPACE.  The first call on a device looks
 * the array's device address up and fills its tables (synchronising
 * `stream`), so make that first call before any stream capture.  `scale` is
 * passed to the kernels by value.  All calls share the array and each one
 * overwrites what it uses: calls that overlap on the GPU race. */
gl_status gl_box_synthesize_noalloc(int n_units, int nx, int ny, int box_x0, int box_y0,
                                    int box_w, int box_h, const void* d_box_spectra,
                                    double scale, void* d_out, int real_only, void* stream);

/* Fourth-order WIT direct sum, sector 44 (all four parents on the + branch).
 * Replaces the sector-44 path of paper/order4/cpp/directional_eta4_openmp.cpp
 * (DirectionalKernel::evaluate :157-453, quartet loop :690-734, output
 * :747-773).  d_modes: (mx, my) int32 pairs; d_amp: [case][mode] complex128;
 * d_out: 5 planes [field][case][ny][nx] complex128 (eta, psi, etaCoordinate,
 * psiCoordinate, retained), zeroed and accumulated by the call; d_work:
 * gl_wit_workspace_size(n_modes) device bytes (statistics + binomial table). */
typedef struct gl_wit_stats {
  unsigned long long candidates, kept, near, strict_zero_output, strict_zero_intermediate;
  double max_residual, min_detuning, max_strict_zero_source;
} gl_wit_stats;

size_t gl_wit_workspace_size(int n_modes);
gl_status gl_wit_eta44(int n_modes, const int* d_modes, int n_cases, const void* d_amp, int nx,
                       int ny, double gravity, double depth, double dkx, double dky,
                       double threshold, void* d_out, void* d_work, size_t work_bytes,
                       void* stream);
gl_status gl_wit_read_stats(const void* d_work, int n_modes, gl_wit_stats* out);

/* Any sector of the same sum: 44 as above; 40 (unordered + pair x unordered
 * - pair, analytic half-plane targets, weight 2 a a conj(a) conj(a)) and 42
 * (unordered + triple x one - parent, weight 2 a a a conj(a)); lines 604-689
 * of directional_eta4_openmp.cpp.  Statistics as gl_wit_read_stats. */
gl_status gl_wit_sector(int sector, int n_modes, const int* d_modes, int n_cases,
                        const void* d_amp, int nx, int ny, double gravity, double depth,
                        double dkx, double dky, double threshold, void* d_out, void* d_work,
                        size_t work_bytes, void* stream);
gl_status gl_wit_read_sector_stats(int sector, const void* d_work, int n_modes, gl_wit_stats* out);

/* Candidate count of a sector (its quartet index space): C(M+3, 4) for 44,
 * (M(M+1)/2)^2 for 40, C(M+2, 3) M for 42; 0 for bad arguments. */
unsigned long long gl_wit_candidates(int sector, int n_modes);

/* gl_wit_sector over the candidate indices [q_begin, q_end) only: the device
 * form of the reference's per-thread quartet shares and their serial merge
 * (directional_eta4_openmp.cpp:734-745).  Ranks that split [0, candidates)
 * into contiguous shares and sum their d_out planes (one all-reduce) get
 * gl_wit_sector's fields; the statistics of the shares add up (counts) or
 * combine by max / min.  d_out is zeroed by the call, as there. */
gl_status gl_wit_sector_range(int sector, int n_modes, const int* d_modes, int n_cases,
                              const void* d_amp, int nx, int ny, double gravity, double depth,
                              double dkx, double dky, double threshold, unsigned long long q_begin,
                              unsigned long long q_end, void* d_out, void* d_work,
                              size_t work_bytes, void* stream);

/* Host FP64 Gauss--Laguerre rule (Golub--Welsch with the moment gate). */
gl_status gl_gauss_laguerre(int rank, double* nodes, double* weights);

/* Host FP64 Newton solve of q tanh q = omega^2 h / g for n frequencies. */
gl_status gl_dispersion_solve(int n, const double* omega, double depth, double gravity,
                              double* q_out);

/* Launch accounting (no reference counterpart: measurement support).
 * gl_launch_count: kernels launched by this library since load.
 * gl_profile_begin / gl_profile_end: while enabled, every launch is bracketed
 * by CUDA events on its own stream; gl_profile_end synchronises them and
 * returns per-kernel launches, total milliseconds and algorithmic bytes. */
typedef struct gl_kernel_stat {
  char name[40];
  int launches;
  double ms_total;
  double bytes_total;
} gl_kernel_stat;

unsigned long long gl_launch_count(void);
gl_status gl_profile_begin(void);
gl_status gl_profile_end(gl_kernel_stat* stats, int max_stats, int* n_stats);

/* Message of the last error raised on the calling thread. */
size_t gl_get_last_error(char* buffer, size_t length);

/* Library version string. */
const char* gl_version(void);

#ifdef __cplusplus
}
#endif

#endif /* GL_ENGINE_H */
