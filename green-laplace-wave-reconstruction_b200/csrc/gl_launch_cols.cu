// Column-transform launchers (and the other transforms that are not rows of a
// product stage): inverse columns with their multiplier banks, forward
// columns with mask and maxima, the final rows on the reference grid, the
// adjoint's seed rows and column combines, and the strided transforms of the
// single-direction time path.  launch_row() picks the row family's unit.
#define GL_TRANSFORM_TU
#include "gl_host.h"
#include "gl_adjoint.cuh"
#include "gl_modal.cuh"
#include "gl_gen.cuh"

namespace gl {

namespace {

template <int MIX>
void col_ifft_launch(dim3 grid, size_t smem, cudaStream_t st, const ColArgs& a, const cplx* tw, int cw,
                     int bpb) {
  ensure_smem_attr((const void*)col_ifft_kernel<MIX>, (int)SMEM_LIMIT);
  col_ifft_kernel<MIX><<<grid, 256, smem, st>>>(a, tw, cw, bpb);
}

template <int MIX>
void col_fft_launch(dim3 grid, size_t smem, cudaStream_t st, const ColFftArgs& a, const cplx* tw, int cw) {
  ensure_smem_attr((const void*)col_fft_kernel<MIX>, (int)SMEM_LIMIT);
  col_fft_kernel<MIX><<<grid, 256, smem, st>>>(a, tw, cw);
}

template <int MIX>
void combine_launch(dim3 grid, size_t smem, cudaStream_t st, const CmbArgs& a, const cplx* tw, int cw) {
  ensure_smem_attr((const void*)col_combine_kernel<MIX>, (int)SMEM_LIMIT);
  col_combine_kernel<MIX><<<grid, 256, smem, st>>>(a, tw, cw);
}

// Per-stage names of the column launches in the launch accounting.
const char* col_ifft_name(int kind) {
  switch (kind) {
    case COL_ETA22: case COL_PSI22: return "col_ifft_kernel[order2]";
    case COL_INNER: return "col_ifft_kernel[inner]";
    case COL_OUTER1: return "col_ifft_kernel[outer1]";
    case COL_OUTER2: return "col_ifft_kernel[outer2]";
    case COL_E44_PAIR: case COL_E44_FIRST3: case COL_E44_FIRST4: return "col_ifft_kernel[order4]";
  }
  return "col_ifft_kernel";
}

}  // namespace

gl_status launch_col_ifft(const ColArgs& a, int njobs, cudaStream_t st, const cplx* tw) {
  if (!is_pow2(a.n) && !mixed_len(a.n)) return fail(GL_ERR_UNSUPPORTED, "column length %d has no transform", a.n);
  const int cw = a.cw_max > 0 ? std::min(a.cw_max, fft_cols_per_block(a.n, a.box.w)) : fft_cols_per_block(a.n, a.box.w);
  // the damped base spectrum of the block's columns is staged only for the
  // kinds that share one base across their banks (col_ifft_kernel)
  const bool shared_base = a.kind != COL_PLAIN && a.kind != COL_OUTER2 && a.kind != COL_FLOORED;
  const size_t smem = ((size_t)cw * padded_len(a.n) + (shared_base ? (size_t)cw * a.box.h : 0)) * sizeof(cplx);
  // banks per block, spread evenly over grid.z: at most 4 (12 banks: 3 x 4,
  // 9 banks: 3 x 3), or all of them for the inner stage when one slice
  // still gives at least two blocks per SM slot pair (each block then
  // computes its columns' damped base once instead of once per slice).
  // Same-box A/Bs on the 1024^2 order-3 workload (16 units in two lanes of
  // 8: 640 blocks per slice): inner in one slice +1.0 %, in 2 slices of 6
  // +0.5 %; the outer first-order banks in slices of 6, or any stage in
  // slices of 2 or 3, slower or no faster.  A single 512^2 unit (64 blocks
  // per slice) keeps the three slices: one slice left most SMs idle.
  const int col_blocks = (a.box.w + cw - 1) / cw;
  const bool one_slice = a.kind == COL_INNER && (long long)col_blocks * njobs >= 4LL * 148;
  const int per = one_slice ? a.nbanks : 4;
  const int nz = (a.nbanks + per - 1) / per;
  const int bpb = (a.nbanks + nz - 1) / nz;
  dim3 grid((a.box.w + cw - 1) / cw, njobs, (a.nbanks + bpb - 1) / bpb);
  const double bytes = (double)njobs * (a.twins ? a.nout : a.nbanks) * a.box.w * a.n * sizeof(cplx) +
                       (double)njobs * a.box.w * a.box.h * sizeof(cplx);
  LaunchScope ls(col_ifft_name(a.kind), st, bytes);
  GL_MIX_DISPATCH(a.n, col_ifft_launch, grid, smem, st, a, tw, cw, bpb);
  LAUNCH_CHECK("col_ifft_kernel");
  return GL_OK;
}

gl_status launch_col_fft(const ColFftArgs& a, int njs, cudaStream_t st, const cplx* tw, const char* name) {
  if (!is_pow2(a.n) && !mixed_len(a.n)) return fail(GL_ERR_UNSUPPORTED, "column length %d has no transform", a.n);
  const int cw = a.cw_max > 0 ? std::min(a.cw_max, fft_cols_per_block(a.n, a.box.w)) : fft_cols_per_block(a.n, a.box.w);
  const size_t smem = (size_t)cw * padded_len(a.n) * sizeof(cplx);
  dim3 grid((a.box.w + cw - 1) / cw, njs);
  const double bytes = (double)njs * a.box.w * (a.n + a.box.h) * sizeof(cplx);
  LaunchScope ls(name, st, bytes);
  GL_MIX_DISPATCH(a.n, col_fft_launch, grid, smem, st, a, tw, cw);
  LAUNCH_CHECK("col_fft_kernel");
  return GL_OK;
}

gl_status launch_row(const RowArgs& a, int njobs, cudaStream_t st, const cplx* tw) {
  int nb = 0;
  for (int g = 0; g < a.ngrp; ++g) nb += a.grp[g].nb;
  const size_t smem = row_smem(nb, a.nx);
  if (smem > ROW_SMEM_LIMIT)
    return fail(GL_ERR_UNSUPPORTED, "row stage of %d banks x %d exceeds the shared-memory budget", nb, a.nx);
  dim3 grid(a.ny, njobs);
  // threads per row transform; row_launch() sets the groups per block
  const int T = is_pow2(a.nx) ? a.nx / 16 : 16;
  const bool pair_kind = a.kind == ROW_ETA22 || a.kind == ROW_PSI22 || a.kind == ROW_CONTACT22 ||
                         a.kind == ROW_INNER || a.kind == ROW_ADJ_ETA22 || a.kind == ROW_ADJ_INNER;
  if (!is_pow2(a.nx) && !pair_kind)
    return fail(GL_ERR_UNSUPPORTED, "row kind %d runs power-of-two rows only (got %d)", a.kind, a.nx);
  double bytes = (double)njobs * a.nout * a.out_w * a.ny * sizeof(cplx);
  for (int g = 0; g < a.ngrp; ++g) bytes += (double)njobs * a.grp[g].nb * a.grp[g].w * a.ny * sizeof(cplx);
  const char* name = a.kind == ROW_INNER         ? "row_kernel[inner]"
                     : a.kind == ROW_OUTER       ? "row_kernel[outer]"
                     : a.kind == ROW_ADJ_INNER   ? "row_kernel[adj_inner]"
                     : a.kind == ROW_ADJ_OUTER   ? "row_kernel[adj_outer]"
                     : a.kind == ROW_ADJ_ETA22   ? "row_kernel[adj_eta22]"
                     : a.kind >= ROW_E44_PAIR    ? "row_kernel[order4]"
                                                 : "row_kernel[order2]";
  if (a.kind < ROW_ETA22 || a.kind > ROW_ADJ_OUTER) return fail(GL_ERR_INVALID_ARGUMENT, "unknown row kind %d", a.kind);
  LaunchScope ls(name, st, bytes);
  const bool ok = row_dispatch_pair(a, grid, T, smem, st, tw) || row_dispatch_wide(a, grid, T, smem, st, tw) ||
                  row_dispatch_adj(a, grid, T, smem, st, tw);
  if (!ok) return fail(GL_ERR_UNSUPPORTED, "row length %d has no transform", a.nx);
  LAUNCH_CHECK("row_kernel");
  return GL_OK;
}

gl_status launch_out_rows(const OutArgs& a0, int nuc, cudaStream_t st, const cplx* tw) {
  OutArgs a = a0;
  // rows of up to 1024 points run in 192-thread blocks: two such blocks per
  // SM leave each thread 168 registers (the 256-thread form is held to 128
  // and spills ~180 bytes), for 12 instead of 16 resident warps (same-box
  // A/B at 1024^2: the kernel 7 % faster)
  const int T = a.nx / 16;
  const bool b192 = T <= 64;
  const int threads = b192 ? 192 : 256;
  const int G = threads / T;
  a.rows = G;
  const size_t smem = (size_t)G * padded_len(a.nx) * sizeof(cplx);
  dim3 grid((a.ny + G - 1) / G, nuc);
  const double bytes = (double)nuc * a.w * a.ny * sizeof(cplx) +
                       (double)nuc * a.nx * a.ny * (a.real_only ? sizeof(double) : sizeof(cplx));
  LaunchScope ls("out_row_kernel", st, bytes);
  const void* k = a.real_only ? (b192 ? (const void*)out_row_kernel<true, true> : (const void*)out_row_kernel<true>)
                              : (b192 ? (const void*)out_row_kernel<false, true> : (const void*)out_row_kernel<false>);
  const cudaError_t e = ensure_smem_attr(k, (int)ROW_SMEM_LIMIT);
  if (e != cudaSuccess) return fail(GL_ERR_CUDA, "out_row_kernel shared-memory limit: %s", cudaGetErrorString(e));
  if (a.real_only) {
    if (b192) out_row_kernel<true, true><<<grid, 192, smem, st>>>(a, tw);
    else out_row_kernel<true><<<grid, 256, smem, st>>>(a, tw);
  } else {
    if (b192) out_row_kernel<false, true><<<grid, 192, smem, st>>>(a, tw);
    else out_row_kernel<false><<<grid, 256, smem, st>>>(a, tw);
  }
  LAUNCH_CHECK("out_row_kernel");
  return GL_OK;
}

gl_status launch_seed_rows(const SeedArgs& a, int nunits, cudaStream_t st, const cplx* tw) {
  const int G = 256 / (a.nx / 16);
  const size_t smem = (size_t)G * padded_len(a.nx) * sizeof(cplx);
  ensure_smem_attr((const void*)seed_row_kernel, (int)SMEM_LIMIT);
  dim3 grid((a.ny + G - 1) / G, nunits);
  const double bytes = (double)nunits * a.ny * ((double)a.nx * sizeof(double) + (double)a.w * sizeof(cplx));
  LaunchScope ls("seed_row_kernel", st, bytes);
  seed_row_kernel<<<grid, 256, smem, st>>>(a, tw);
  LAUNCH_CHECK("seed_row_kernel");
  return GL_OK;
}

gl_status launch_combine(const CmbArgs& a, int njobs, cudaStream_t st, const cplx* tw) {
  // columns per block: all banks of `cw` columns staged at once, within
  // ~110 KB of shared memory (two blocks per SM)
  const size_t col_bytes = (size_t)a.nbanks * padded_len(a.n) * sizeof(cplx);
  const int cw = (int)std::max<size_t>(1, std::min<size_t>((size_t)a.box.w, (110 * 1024) / col_bytes));
  const size_t smem = (size_t)cw * col_bytes;
  if (smem > SMEM_LIMIT) return fail(GL_ERR_UNSUPPORTED, "adjoint column stage exceeds shared memory");
  if (a.nout < 1 || a.nout > 4) return fail(GL_ERR_INVALID_ARGUMENT, "adjoint column stage: 1..4 outputs");
  if (!is_pow2(a.n) && !mixed_len(a.n)) return fail(GL_ERR_UNSUPPORTED, "column length %d has no transform", a.n);
  dim3 grid((a.box.w + cw - 1) / cw, njobs);
  const double bytes = (double)njobs * a.nbanks * a.box.w * a.n * sizeof(cplx) +
                       (double)njobs * a.nout * a.box.w * a.box.h * sizeof(cplx);
  LaunchScope ls("col_combine_kernel", st, bytes);
  GL_MIX_DISPATCH(a.n, combine_launch, grid, smem, st, a, tw, cw);
  LAUNCH_CHECK("col_combine_kernel");
  return GL_OK;
}

gl_status launch_sfft(const SFft& a, int outer, int sign, cudaStream_t st, const cplx* tw) {
  const int T = a.n / 16;
  const int cw = std::max(1, 256 / T);
  const size_t smem = (size_t)cw * padded_len(a.n) * sizeof(cplx);
  dim3 grid((unsigned)((a.ncount + cw - 1) / cw), (unsigned)outer);
  LaunchScope ls("strided_fft_kernel", st, 2.0 * a.n * (double)a.ncount * outer * sizeof(cplx));
  if (sign > 0) {
    ensure_smem_attr((const void*)strided_fft_kernel<+1>, (int)SMEM_LIMIT);
    strided_fft_kernel<+1><<<grid, 256, smem, st>>>(a, tw, cw);
  } else {
    ensure_smem_attr((const void*)strided_fft_kernel<-1>, (int)SMEM_LIMIT);
    strided_fft_kernel<-1><<<grid, 256, smem, st>>>(a, tw, cw);
  }
  LAUNCH_CHECK("strided_fft_kernel");
  return GL_OK;
}

gl_status launch_gen_cols(const GenColArgs& a0, int njobs, cudaStream_t st) {
  GenColArgs a = a0;
  const size_t col_bytes = 2 * (size_t)a.gp.n * sizeof(cplx);
  a.cw = (int)std::max<size_t>(1, std::min<size_t>((size_t)a.box.w, (96 * 1024) / col_bytes));
  const size_t smem = (size_t)a.cw * col_bytes;
  if (smem > SMEM_LIMIT) return fail(GL_ERR_UNSUPPORTED, "column length %d exceeds shared memory", a.gp.n);
  ensure_smem_attr((const void*)gen_col_kernel, (int)SMEM_LIMIT);
  dim3 grid((a.box.w + a.cw - 1) / a.cw, njobs, a.nbanks);
  const double bytes = (double)njobs * a.nbanks * a.box.w * ((double)a.gp.n + a.box.h) * sizeof(cplx);
  LaunchScope ls("gen_col_kernel", st, bytes);
  gen_col_kernel<<<grid, 256, smem, st>>>(a);
  LAUNCH_CHECK("gen_col_kernel");
  return GL_OK;
}

gl_status launch_gen_rows(const GenRowArgs& a0, int nuc, cudaStream_t st) {
  GenRowArgs a = a0;
  const size_t row_bytes = 2 * (size_t)a.gp.n * sizeof(cplx);
  a.rows = (int)std::max<size_t>(1, std::min<size_t>((size_t)a.ny, (96 * 1024) / row_bytes));
  const size_t smem = (size_t)a.rows * row_bytes;
  if (smem > SMEM_LIMIT) return fail(GL_ERR_UNSUPPORTED, "row length %d exceeds shared memory", a.gp.n);
  ensure_smem_attr((const void*)gen_row_kernel, (int)SMEM_LIMIT);
  dim3 grid((a.ny + a.rows - 1) / a.rows, nuc);
  const double bytes = (double)nuc * a.w * a.ny * sizeof(cplx) +
                       (double)nuc * a.gp.n * a.ny * (a.real_only ? sizeof(double) : sizeof(cplx));
  LaunchScope ls("gen_row_kernel", st, bytes);
  gen_row_kernel<<<grid, 256, smem, st>>>(a);
  LAUNCH_CHECK("gen_row_kernel");
  return GL_OK;
}

}  // namespace gl
