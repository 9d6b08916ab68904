// The row-stage launch shape shared by the three row translation units
// (gl_rows_pair.cu, gl_rows_wide.cu, gl_rows_adj.cu): groups per block,
// several short rows per block, and the 192-thread outer-row variant.
#pragma once
#include "gl_host.h"

namespace gl {

template <int K, int MIX = 0>
void row_launch(dim3 grid, int T, size_t smem, cudaStream_t st, const RowArgs& a, const cplx* tw) {
  int nb = 0;
  for (int g = 0; g < a.ngrp; ++g) nb += a.grp[g].nb;
  // 8 transform groups per block when the row has at most 12 banks (4
  // blocks fit per SM), 16 for wider rows (2 per SM by shared memory); a
  // forward row with more than 16 banks (the order-3 outer row: 21) gets the
  // fewest whole-warp groups that keep its rounds (12: the same rounds with
  // fewer idle groups measured 6 % faster; more resident blocks for the
  // 12-bank rows measured slower)
  int G = nb <= 12 ? 8 : 16;
  if (K == ROW_OUTER && nb > 16) {
    const int rounds = (nb + 15) / 16;
    G = (nb + rounds - 1) / rounds;
    while ((G * T) % 32 != 0) ++G;
  }
  if (a.groups > 0) G = std::max(1, std::min(a.groups, 256 / std::max(1, T)));  // a plan's tuning
  // Short rows (fewer than 16 threads per transform) carry little work per
  // block, so a block takes several rows (one team of G groups each) while it
  // stays within 256 threads and ~76 KB of shared memory (3 blocks per SM).
  const int team = G * T;
  int rpb = 1;
  if (MIX == 0 && T < 16) {
    int r = std::min(256 / std::max(1, team), (int)((76 * 1024) / std::max<size_t>(1, smem)));
    while (r > 1 && (team * r) % 32 != 0) --r;
    rpb = std::max(1, r);
  }
  const int threads = rpb > 1 ? team * rpb : std::max(32, std::min(256, team));
  RowArgs b = a;
  b.rpb = rpb;
  dim3 g2((a.ny + rpb - 1) / rpb, grid.y);
  if constexpr (MIX == 0) {
    if (rpb > 1) {
      ensure_smem_attr((const void*)row_kernel_t<K, 0, true>, (int)ROW_SMEM_LIMIT);
      row_kernel_t<K, 0, true><<<g2, threads, smem * rpb, st>>>(b, tw);
      return;
    }
  }
  if constexpr (K == ROW_OUTER && MIX == 0) {
    if (threads <= 192) {
      ensure_smem_attr((const void*)row_kernel_t<K, 0, false, true>, (int)ROW_SMEM_LIMIT);
      row_kernel_t<K, 0, false, true><<<g2, threads, smem, st>>>(b, tw);
      return;
    }
  }
  // a failed attribute call surfaces as the launch's own error
  ensure_smem_attr((const void*)row_kernel_t<K, MIX>, (int)ROW_SMEM_LIMIT);
  row_kernel_t<K, MIX><<<g2, threads, smem, st>>>(b, tw);
}

// Pair-stage rows also run on the mixed row lengths 144, 160, 192, 240
// (row_len); each is its own instantiation.
template <int K>
bool row_launch_mixed(dim3 grid, int T, size_t smem, cudaStream_t st, const RowArgs& a, const cplx* tw) {
  switch (mixed_len(a.nx) ? a.nx / 16 : 0) {
    case 0: row_launch<K, 0>(grid, T, smem, st, a, tw); return true;
    case 9: row_launch<K, 9>(grid, T, smem, st, a, tw); return true;
    case 10: row_launch<K, 10>(grid, T, smem, st, a, tw); return true;
    case 12: row_launch<K, 12>(grid, T, smem, st, a, tw); return true;
    case 15: row_launch<K, 15>(grid, T, smem, st, a, tw); return true;
  }
  return false;
}

}  // namespace gl
