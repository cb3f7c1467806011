// Shared-memory layout of padded tiles, shared by the spreading and interpolation kernels.
//
// A tile of T0 x T1 x T2 fine-grid cells plus its (w-1)-cell halo is stored with row stride RS
// (>= T0 + w - 1) and plane stride PS (>= RS (T1 + w - 1)). A warp that processes one point
// gives lane r footprint row r (3D: r = dy + w dz at offset dz PS + dy RS; 2D: r = dx + w dy at
// offset dy RS + dx; 1D: r = dx). The strides are chosen by a small host-side search: among
// the smallest paddings, the pair that puts the 32 lanes of every pass on the fewest
// shared-memory bank groups (16 groups of 8-byte cells, 8 of 16-byte cells), so that each
// access takes the minimum number of wavefronts.
#pragma once

#include "common.cuh"

namespace nnb {

struct TileLayout {
  int P0, P1, P2;  // padded extents (cells)
  int RS, PS;      // strides (cells)
  int cells;       // storage size (cells)
};

// Worst-case number of lanes of one pass that fall into the same bank group.
inline int layout_conflict(int dim, int w, int RS, int PS, int groups) {
  const int nr = dim == 1 ? w : w * w;
  int worst = 0;
  for (int pass = 0; pass * 32 < nr; ++pass) {
    int count[16] = {0};
    for (int lane = 0; lane < 32; ++lane) {
      const int r = pass * 32 + lane;
      if (r >= nr) break;
      int off;
      if (dim == 3) off = (r / w) * PS + (r % w) * RS;
      else if (dim == 2) off = (r / w) * RS + (r % w);
      else off = r;
      const int g = off % groups;
      if (++count[g] > worst) worst = count[g];
    }
  }
  return worst;
}

// T0..T2: interior extents (1 for unused dims); w: kernel width; dim: 1..3.
inline TileLayout make_tile_layout(int dim, int w, int T0, int T1, int T2, int cell_bytes = 8) {
  TileLayout L;
  L.P0 = T0 + w - 1;
  L.P1 = dim > 1 ? T1 + w - 1 : 1;
  L.P2 = dim > 2 ? T2 + w - 1 : 1;
  const int groups = cell_bytes >= 16 ? 8 : 16;
  if (dim == 1) {
    L.RS = L.P0;
    L.PS = L.P0;
    L.cells = L.P0 + L.P0 % 2;
    return L;
  }
  const int lanes_per_pass = (dim == 3 ? w * w : w * w) < 32 ? (w * w) : 32;
  const int ideal = (lanes_per_pass + groups - 1) / groups;
  int best_rs = L.P0, best_ps = L.P0 * L.P1, best_c = 1 << 30;
  long best_cells = -1;
  for (int rs = L.P0; rs < L.P0 + 16; ++rs) {
    const int ps_min = rs * L.P1;
    const int ps_max = dim == 3 ? ps_min + 16 : ps_min + 1;
    for (int ps = ps_min; ps < ps_max; ++ps) {
      const int c = layout_conflict(dim, w, rs, ps, groups);
      const long cells = dim == 3 ? long(ps) * L.P2 : long(rs) * L.P1;
      // prefer the ideal conflict level, then the smallest storage
      const int cc = c <= ideal ? ideal : c;
      if (cc < best_c || (cc == best_c && cells < best_cells)) {
        best_c = cc;
        best_cells = cells;
        best_rs = rs;
        best_ps = ps;
      }
    }
  }
  L.RS = best_rs;
  L.PS = dim == 3 ? best_ps : best_rs * L.P1;
  L.cells = dim == 3 ? L.PS * L.P2 : L.PS;
  L.cells += L.cells % 2;  // keeps consecutive slabs 16-byte aligned
  return L;
}

// Wraps a possibly out-of-range fine-grid index (at most one period beyond) into [0, n).
__device__ __forceinline__ i64 wrap_index(i64 i, i64 n) {
  while (i >= n) i -= n;
  return i;
}

}  // namespace nnb
