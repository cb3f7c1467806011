// Shared definitions of the B200 NUFFT engine: complex helpers, error handling, grid geometry.
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>

#include <cstdint>
#include <cstdio>
#include <string>

#include "neonufft/enums.h"
#include "neonufft/exceptions.hpp"

namespace nnb {

using i64 = std::int64_t;
using u32 = std::uint32_t;
using u64 = std::uint64_t;

constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr double kTwoPiInv = 1.0 / (2.0 * kPi);

// ---------------------------------------------------------------------------------------------
// Complex storage types (interleaved re/im, identical layout to cuComplex / cuDoubleComplex).
// ---------------------------------------------------------------------------------------------
template <typename T>
struct Cplx;
template <>
struct Cplx<float> {
  using type = float2;
};
template <>
struct Cplx<double> {
  using type = double2;
};
template <typename T>
using cplx_t = typename Cplx<T>::type;

template <typename C>
__host__ __device__ __forceinline__ C cmul(C a, C b) {
  return C{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}

// ---------------------------------------------------------------------------------------------
// Error handling: host code throws the reference exception types; the C ABI translates them.
// Messages are copied into a per-thread buffer so that the exception may keep a const char*.
// ---------------------------------------------------------------------------------------------
const char* store_message(const std::string& msg);

[[noreturn]] void throw_gpu(cudaError_t err, const char* what, const char* file, int line);
[[noreturn]] void throw_fft(cufftResult err, const char* what, const char* file, int line);
[[noreturn]] void throw_input(const std::string& msg);
[[noreturn]] void throw_internal(const std::string& msg);

#define NNB_CUDA(expr)                                                        \
  do {                                                                        \
    cudaError_t nnb_err_ = (expr);                                            \
    if (nnb_err_ != cudaSuccess) ::nnb::throw_gpu(nnb_err_, #expr, __FILE__, __LINE__); \
  } while (0)

#define NNB_CUFFT(expr)                                                       \
  do {                                                                        \
    cufftResult nnb_err_ = (expr);                                            \
    if (nnb_err_ != CUFFT_SUCCESS) ::nnb::throw_fft(nnb_err_, #expr, __FILE__, __LINE__); \
  } while (0)

// Counts one engine kernel launch and checks the launch status of the last kernel.
void count_launch();
#define NNB_LAUNCH_CHECK()        \
  do {                            \
    ::nnb::count_launch();        \
    NNB_CUDA(cudaGetLastError()); \
  } while (0)

// ---------------------------------------------------------------------------------------------
// Checked build (-DNNB_CHECKED): device bounds checks on every grid, record and output index of
// the spreading, interpolation, deconvolution and binning kernels. A failed check skips the
// access and records (first failure only) the source line, the index and its bound in this
// translation unit's device record; it never traps, so the context stays usable. After every
// C ABI call the checked build synchronises the device and reports a recorded failure as
// InternalError (check_device_records, runtime.cu), the counterpart of the reference's debug
// sync-and-check after each launch (src/neonufft/gpu/util/runtime.hpp:27-30). In the normal
// build NNB_CHECK_INDEX is the constant true and the checks compile away.
// ---------------------------------------------------------------------------------------------
struct CheckRecord {
  int flag;
  int line;
  long long index;
  long long bound;
};
using CheckReadFn = CheckRecord (*)();
// Registers a translation unit's reader and clearer of its device record (host, at load).
bool register_check_record(CheckReadFn read, void (*clear)(), const char* unit);
// Synchronises the device and throws InternalError if any unit recorded a failed check
// (checked build; a no-op otherwise).
void check_device_records();

#ifdef NNB_CHECKED
namespace {
__device__ CheckRecord g_unit_check;
CheckRecord read_unit_check() {
  CheckRecord r{};
  if (cudaMemcpyFromSymbol(&r, g_unit_check, sizeof(r)) != cudaSuccess) r.flag = 0;
  return r;
}
void clear_unit_check() {
  const CheckRecord z{};
  (void)cudaMemcpyToSymbol(g_unit_check, &z, sizeof(z));
}
[[maybe_unused]] const bool g_unit_check_registered =
    register_check_record(&read_unit_check, &clear_unit_check, __BASE_FILE__);
__device__ __noinline__ void record_failed_check(long long i, long long n, int line) {
  if (atomicCAS(&g_unit_check.flag, 0, 1) == 0) {
    g_unit_check.line = line;
    g_unit_check.index = i;
    g_unit_check.bound = n;
  }
}
}  // namespace
__device__ __forceinline__ bool checked_index(long long i, long long n, int line) {
  if (i >= 0 && i < n) return true;
  record_failed_check(i, n, line);
  return false;
}
#define NNB_CHECK_INDEX(i, n) (::nnb::checked_index((long long)(i), (long long)(n), __LINE__))
#else
#define NNB_CHECK_INDEX(i, n) true
#endif

// ---------------------------------------------------------------------------------------------
// Geometry of a binned point set on a fine grid.
//
// Points are rescaled to p = frac(((x - offset) * scale + pi) / 2pi) in [0, 1), placed at
// loc = p * nf on the fine grid, and assigned to the subproblem tile containing their first
// kernel cell i0 = ceil(loc - w/2) (wrapped periodically). This is the rescaling of the
// reference (src/neonufft/gpu/kernels/rescale_loc_kernel.cu:107-121 and :167-179, affine part
// for type 3), computed here in double precision for every plan precision.
// ---------------------------------------------------------------------------------------------
struct BinGeom {
  int dim;
  int w;              // kernel width (n_spread)
  i64 nf[3];          // fine grid dims (1 for unused dims)
  int tile[3];        // tile dims (1 for unused dims)
  int ntiles[3];      // number of tiles per dim
  i64 total_tiles;
  double offset[3];   // affine pre-transform (type 3); 0 / 1 otherwise
  double scale[3];
  int zmajor;         // 3D: bins ordered plane-fastest, tz + ntz (tx + ntx ty); else x-fastest
};

// Linear bin index of tile coordinates t[0..dim).
__host__ __device__ __forceinline__ i64 tile_linear(const BinGeom& g, const i64* t) {
  if (g.dim == 3 && g.zmajor) return t[2] + i64(g.ntiles[2]) * (t[0] + i64(g.ntiles[0]) * t[1]);
  i64 lin = 0, mul = 1;
  for (int d = 0; d < g.dim; ++d) {
    lin += t[d] * mul;
    mul *= g.ntiles[d];
  }
  return lin;
}

// Packed tile-local start cell of a point: 1D 32 bits; 2D 16+16; 3D 11+11+10 (x, y, z).
__host__ __device__ __forceinline__ u32 pack_local(int dim, int lx, int ly, int lz) {
  if (dim == 1) return u32(lx);
  if (dim == 2) return u32(lx) | (u32(ly) << 16);
  return u32(lx) | (u32(ly) << 11) | (u32(lz) << 22);
}
__host__ __device__ __forceinline__ void unpack_local(int dim, u32 v, int& lx, int& ly, int& lz) {
  if (dim == 1) {
    lx = int(v); ly = 0; lz = 0;
  } else if (dim == 2) {
    lx = int(v & 0xFFFFu); ly = int(v >> 16); lz = 0;
  } else {
    lx = int(v & 0x7FFu); ly = int((v >> 11) & 0x7FFu); lz = int(v >> 22);
  }
}
constexpr int kMaxTileBits3[3] = {11, 11, 10};

// Plane-major 3D point sets (BinGeom::zmajor; tiles of at most 16 x 16 x 1 cells) store the
// absolute first kernel plane instead of the tile-local z: x 4 bits, y 4 bits, plane 24 bits.
__host__ __device__ __forceinline__ u32 pack_local_zmajor(int lx, int ly, i64 plane) {
  return u32(lx) | (u32(ly) << 4) | (u32(plane) << 8);
}

// One bin-sorted point: 32 bytes (a full 32-byte sector) for float and double plans, so that
// the binning scatter writes each point with one sector and the kernels read it with two
// 16-byte loads.
template <typename T>
struct alignas(16) PointRec {
  u32 perm;   // original point index
  u32 local;  // packed tile-local start cell
  T frac[3];  // kernel argument of the first cell, i0 - loc, in [-w/2, -w/2 + 1]
};
static_assert(sizeof(PointRec<float>) == 32 && sizeof(PointRec<double>) == 32,
              "point records are one 32-byte sector");

// The whole sector of a record, as two 16-byte vectors (copies keep the sector whole).
template <typename T>
struct RecSector {
  uint4 a, b;
};
// The 32 bytes of a record as two 16-byte vectors, the single-precision padding as zeros: a
// store of the fields alone would leave part of the sector unwritten, and the L2 would read the
// sector from memory to merge it when it writes it back (for records placed at random, a second
// 32 bytes of traffic per point).
__device__ __forceinline__ RecSector<float> rec_sector(const PointRec<float>& r) {
  return RecSector<float>{make_uint4(r.perm, r.local, __float_as_uint(r.frac[0]),
                                     __float_as_uint(r.frac[1])),
                          make_uint4(__float_as_uint(r.frac[2]), 0u, 0u, 0u)};
}
__device__ __forceinline__ RecSector<double> rec_sector(const PointRec<double>& r) {
  return RecSector<double>{
      make_uint4(r.perm, r.local, u32(__double2loint(r.frac[0])), u32(__double2hiint(r.frac[0]))),
      make_uint4(u32(__double2loint(r.frac[1])), u32(__double2hiint(r.frac[1])),
                 u32(__double2loint(r.frac[2])), u32(__double2hiint(r.frac[2])))};
}

// L2 eviction policies (createpolicy, sm_80 and later) for data that should stay in the L2
// (evict_last) or leave it first (evict_first).
__device__ __forceinline__ unsigned long long l2_evict_last_policy() {
  unsigned long long p;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ unsigned long long l2_evict_first_policy() {
  unsigned long long p;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
// A 32-bit global load with an L2 eviction policy.
__device__ __forceinline__ u32 load_u32_policy(const u32* p, unsigned long long policy) {
  u32 v;
  asm("ld.global.L2::cache_hint.u32 %0, [%1], %2;"
      : "=r"(v)
      : "l"(__cvta_generic_to_global(p)), "l"(policy));
  return v;
}
// Stores a record's sector s at dst. Where the record array is 32-byte aligned (`wide`, the same
// for every thread of a launch; a user allocator may return less) it is one 256-bit store
// (st.global.v8.b32, sm_100) with the L2 eviction policy `policy`, else two 16-byte stores. The
// binning scatter, which writes each of 1e8 records to a random slot, takes 4.45 ms with single
// 256-bit stores and 4.10 ms with single evict-first stores, against 5.71 ms with two 16-byte
// stores per record.
template <typename T>
__device__ __forceinline__ void store_sector_policy(PointRec<T>* dst, const RecSector<T>& s,
                                                    bool wide, unsigned long long policy) {
  if (wide) {
    asm volatile(
        "st.global.L2::cache_hint.v8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8}, %9;"
        :
        : "l"(__cvta_generic_to_global(dst)), "r"(s.a.x), "r"(s.a.y), "r"(s.a.z), "r"(s.a.w),
          "r"(s.b.x), "r"(s.b.y), "r"(s.b.z), "r"(s.b.w), "l"(policy)
        : "memory");
  } else {
    store_sector(dst, s);
  }
}
template <typename T>
__device__ __forceinline__ RecSector<T> load_sector(const PointRec<T>* src) {
  const uint4* s = reinterpret_cast<const uint4*>(src);
  return RecSector<T>{s[0], s[1]};
}
template <typename T>
__device__ __forceinline__ void store_sector(PointRec<T>* dst, const RecSector<T>& v) {
  uint4* d = reinterpret_cast<uint4*>(dst);
  d[0] = v.a;
  d[1] = v.b;
}

// Device scratch of a point set for the kernels' work lists (worklist.cu).
struct WorkScratch {
  u32* cnt;       // items per unit (max_units)
  u32* start;     // exclusive scan of cnt (max_units + 1)
  u32* tmp;       // scan partials
  u32* owner;     // unit of each item (max_items)
  i64 max_units;
  i64 max_items;
};

// Device-side view of a bin-sorted point set (records in tile order, length M).
template <typename T>
struct SortedPoints {
  const PointRec<T>* rec;
  const u32* bin_start;  // total_tiles + 1 offsets into the records
  i64 M;
  WorkScratch work;
};

// ES kernel (exponential of semicircle): phi(x) = exp(beta * (sqrt(1 - c x^2) - 1)) for
// |x| < w/2, else 0, c = 4 / w^2 (reference src/neonufft/gpu/kernels/es_kernel_eval.cuh:18-44).
template <typename T>
__device__ __forceinline__ T es_eval(T x, T beta, T c);

template <>
__device__ __forceinline__ float es_eval<float>(float x, float beta, float c) {
  const float arg = 1.f - c * x * x;
  return arg > 0.f ? expf(beta * (sqrtf(arg) - 1.f)) : 0.f;
}
template <>
__device__ __forceinline__ double es_eval<double>(double x, double beta, double c) {
  const double arg = 1.0 - c * x * x;
  return arg > 0.0 ? exp(beta * (sqrt(arg) - 1.0)) : 0.0;
}

// Fast ES kernel for the hot loops: single precision uses the hardware exponential
// (__expf); double precision is the same as es_eval.
template <typename T>
__device__ __forceinline__ T es_eval_fast(T x, T beta, T c);

template <>
__device__ __forceinline__ float es_eval_fast<float>(float x, float beta, float c) {
  const float arg = 1.f - c * x * x;
  return arg > 0.f ? __expf(beta * (sqrtf(arg) - 1.f)) : 0.f;
}
template <>
__device__ __forceinline__ double es_eval_fast<double>(double x, double beta, double c) {
  return es_eval<double>(x, beta, c);
}

}  // namespace nnb
