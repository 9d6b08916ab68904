// Row launches of the power-of-two product rows: the order-3 outer stage and
// the four order-4 row kinds.
#define GL_TRANSFORM_TU
#include "gl_rows_launch.cuh"

namespace gl {

bool row_dispatch_wide(const RowArgs& a, dim3 grid, int T, size_t smem, cudaStream_t st, const cplx* tw) {
  switch (a.kind) {
    case ROW_OUTER: row_launch<ROW_OUTER>(grid, T, smem, st, a, tw); return true;
    case ROW_E44_PAIR: row_launch<ROW_E44_PAIR>(grid, T, smem, st, a, tw); return true;
    case ROW_E44_THIRD: row_launch<ROW_E44_THIRD>(grid, T, smem, st, a, tw); return true;
    case ROW_E44_ORDER4: row_launch<ROW_E44_ORDER4>(grid, T, smem, st, a, tw); return true;
    case ROW_E44_ORDER4_PSI: row_launch<ROW_E44_ORDER4_PSI>(grid, T, smem, st, a, tw); return true;
  }
  return false;
}

}  // namespace gl
