// Work lists: launch units split into items of at most `cap` points.
//
// The spreading and interpolation kernels give each launch unit (a z-window column chunk, a
// group of slab tiles, or one tile) to one CTA. With clustered points a few units hold most of
// the points and would serialise on a few CTAs; here every unit with n points becomes
// ceil(n / cap) items (the largest of its tiles' counts for a group of tiles), each taken by its
// own CTA. Item i belongs to unit owner[i] and is that unit's (i - start[owner[i]])-th slice of
// cap points. Splitting is safe because every kernel adds its partial grid with atomics
// (spreading) or writes disjoint outputs (interpolation).
#include "kernels.cuh"

namespace nnb {

namespace {

constexpr int kWlThreads = 256;

__device__ __forceinline__ u32 tile_count(const u32* bs, i64 bin) { return bs[bin + 1] - bs[bin]; }

__global__ void __launch_bounds__(kWlThreads)
    unit_items_kernel(UnitMap m, BinGeom g, const u32* bs, u32 cap, u32* cnt) {
  const i64 u = blockIdx.x * i64(kWlThreads) + threadIdx.x;
  if (u >= m.units) return;
  u32 n = 0;
  if (m.kind == UnitMap::kZwin) {
    const i64 chunk = u / m.ncols;
    const i64 col = u - chunk * m.ncols;
    const i64 z0 = chunk * m.zlen;
    const i64 z1 = min(z0 + m.zlen, i64(m.nz));
    n = bs[col * m.nz + z1] - bs[col * m.nz + z0];
  } else if (m.kind == UnitMap::kSlab) {
    const int LD = g.dim - 1;
    const i64 rest = u / m.groups;
    const i64 grp = u - rest * m.groups;
    const i64 plane = g.total_tiles / g.ntiles[LD];
    for (int w = 0; w < m.nw; ++w) {
      const i64 t = grp * m.nw + w;
      if (t < g.ntiles[LD]) n = max(n, tile_count(bs, rest + plane * t));
    }
  } else {
    n = tile_count(bs, u);
  }
  cnt[u] = (n + cap - 1) / cap;
}

__global__ void __launch_bounds__(kWlThreads)
    owner_kernel(i64 units, const u32* start, u32* owner) {
  const i64 u = blockIdx.x * i64(kWlThreads) + threadIdx.x;
  if (u >= units) return;
  for (u32 i = start[u]; i < start[u + 1]; ++i) owner[i] = u32(u);
}

}  // namespace

WorkList describe_work_list(const UnitMap& m, i64 M, const WorkScratch& s) {
  if (m.units < 1 || m.units > s.max_units) throw_internal("work list larger than its scratch");
  WorkList wl;
  wl.units = m.units;
  wl.cap = kWorkItemPoints;
  wl.grid = m.units + (M + kWorkItemPoints - 1) / kWorkItemPoints + 1;
  if (wl.grid > s.max_items) throw_internal("work list larger than its scratch");
  wl.owner = s.owner;
  wl.start = s.start;
  return wl;
}

WorkList build_work_list(const UnitMap& m, const BinGeom& g, const u32* bin_start, i64 M,
                         const WorkScratch& s, cudaStream_t stream) {
  const WorkList wl = describe_work_list(m, M, s);
  const unsigned blocks = unsigned((m.units + kWlThreads - 1) / kWlThreads);
  unit_items_kernel<<<blocks, kWlThreads, 0, stream>>>(m, g, bin_start, wl.cap, s.cnt);
  NNB_LAUNCH_CHECK();
  launch_exclusive_scan(s.cnt, s.start, m.units, s.tmp, stream);
  owner_kernel<<<blocks, kWlThreads, 0, stream>>>(m.units, s.start, s.owner);
  NNB_LAUNCH_CHECK();
  return wl;
}

}  // namespace nnb
