// Row launches of the adjoint: the transposed eta22, inner and outer rows.
#define GL_TRANSFORM_TU
#include "gl_rows_launch.cuh"

namespace gl {

bool row_dispatch_adj(const RowArgs& a, dim3 grid, int T, size_t smem, cudaStream_t st, const cplx* tw) {
  switch (a.kind) {
    case ROW_ADJ_ETA22: return row_launch_mixed<ROW_ADJ_ETA22>(grid, T, smem, st, a, tw);
    case ROW_ADJ_INNER: return row_launch_mixed<ROW_ADJ_INNER>(grid, T, smem, st, a, tw);
    case ROW_ADJ_OUTER: row_launch<ROW_ADJ_OUTER>(grid, T, smem, st, a, tw); return true;
  }
  return false;
}

}  // namespace gl
