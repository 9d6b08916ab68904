// Row launches of the pair stages: eta22, psi22 (and its Taylor contact) and
// the order-3 inner loop, on power-of-two and mixed row lengths.
#define GL_TRANSFORM_TU
#include "gl_rows_launch.cuh"

namespace gl {

bool row_dispatch_pair(const RowArgs& a, dim3 grid, int T, size_t smem, cudaStream_t st, const cplx* tw) {
  switch (a.kind) {
    case ROW_ETA22: return row_launch_mixed<ROW_ETA22>(grid, T, smem, st, a, tw);
    case ROW_PSI22: return row_launch_mixed<ROW_PSI22>(grid, T, smem, st, a, tw);
    case ROW_CONTACT22: return row_launch_mixed<ROW_CONTACT22>(grid, T, smem, st, a, tw);
    case ROW_INNER: return row_launch_mixed<ROW_INNER>(grid, T, smem, st, a, tw);
  }
  return false;
}

}  // namespace gl
