// User code written against the reference's GPU plan API (include/neonufft/gpu/plan.hpp,
// include/neonufft/gpu/device_allocator.hpp, include/neonufft/exceptions.hpp), compiled with g++
// against this engine's headers and linked to libneonufft_b200.so: the drop-in check for C++
// callers. The flow follows the reference's own GPU tests (tests/test_type_1_2.cpp:130-161,
// tests/test_type_3.cpp:137-200): device buffers, a plan on a stream, copy back, compare with
// FP64 direct sums computed here on the host.
//
//   plan_api cpu   argument errors that need no device map to the reference's exceptions
//   plan_api gpu   every plan class against direct sums; allocator accounting and failures
//
// Prints one line per check and exits non-zero on the first failure.
#include <neonufft/exceptions.hpp>
#include <neonufft/gpu/device_allocator.hpp>
#include <neonufft/gpu/plan.hpp>

#include <cuda_runtime_api.h>

#include <array>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <memory>
#include <random>
#include <string>
#include <vector>

namespace {

using neonufft::IntType;
using neonufft::Options;
using cd = std::complex<double>;

int g_checks = 0;

void fail(const std::string& what) {
  std::printf("FAIL %s\n", what.c_str());
  std::exit(1);
}

void pass(const std::string& what) {
  ++g_checks;
  std::printf("ok   %s\n", what.c_str());
}

void cuda_ok(cudaError_t e, const char* what) {
  if (e != cudaSuccess) fail(std::string(what) + ": " + cudaGetErrorString(e));
}

// Runs f and checks that it throws exactly the exception type E (a subclass of GenericError).
template <typename E>
void expect_throw(const std::string& what, const std::function<void()>& f) {
  try {
    f();
  } catch (const E& e) {
    if (!e.what() || !*e.what()) fail(what + ": empty message");
    pass(what + " -> " + e.what());
    return;
  } catch (const neonufft::GenericError& e) {
    fail(what + ": wrong exception type (" + e.what() + ")");
  }
  fail(what + ": no exception");
}

// Mode index offset of the reference's CMCL order: modes run from -floor(n/2).
IntType k_offset(IntType n) { return n / 2; }

double rel_l2(const std::vector<cd>& got, const std::vector<cd>& ref) {
  double num = 0, den = 0;
  for (std::size_t i = 0; i < ref.size(); ++i) {
    num += std::norm(got[i] - ref[i]);
    den += std::norm(ref[i]);
  }
  return std::sqrt(num / den);
}

// f[k] = sum_j c_j exp(i sign k . x_j) on the CMCL mode box, x-fastest.
template <std::size_t DIM>
std::vector<cd> direct_type1(int sign, const std::array<std::vector<double>, DIM>& x,
                             const std::vector<cd>& c, std::array<IntType, DIM> modes) {
  IntType total = 1;
  for (auto n : modes) total *= n;
  std::vector<cd> f(std::size_t(total), cd(0, 0));
  for (IntType idx = 0; idx < total; ++idx) {
    IntType rem = idx;
    std::array<double, DIM> k;
    for (std::size_t d = 0; d < DIM; ++d) {
      k[d] = double(rem % modes[d] - k_offset(modes[d]));
      rem /= modes[d];
    }
    cd s(0, 0);
    for (std::size_t j = 0; j < c.size(); ++j) {
      double ph = 0;
      for (std::size_t d = 0; d < DIM; ++d) ph += k[d] * x[d][j];
      s += c[j] * std::polar(1.0, sign * ph);
    }
    f[std::size_t(idx)] = s;
  }
  return f;
}

// c_j = sum_k f[k] exp(i sign k . x_j), f on the CMCL mode box, x-fastest.
template <std::size_t DIM>
std::vector<cd> direct_type2(int sign, const std::array<std::vector<double>, DIM>& x,
                             const std::vector<cd>& f, std::array<IntType, DIM> modes) {
  const std::size_t M = x[0].size();
  std::vector<cd> c(M, cd(0, 0));
  for (std::size_t j = 0; j < M; ++j) {
    cd s(0, 0);
    for (std::size_t idx = 0; idx < f.size(); ++idx) {
      IntType rem = IntType(idx);
      double ph = 0;
      for (std::size_t d = 0; d < DIM; ++d) {
        ph += double(rem % modes[d] - k_offset(modes[d])) * x[d][j];
        rem /= modes[d];
      }
      s += f[idx] * std::polar(1.0, sign * ph);
    }
    c[j] = s;
  }
  return c;
}

// f_k = sum_j c_j exp(i sign s_k . x_j)
template <std::size_t DIM>
std::vector<cd> direct_type3(int sign, const std::array<std::vector<double>, DIM>& x,
                             const std::vector<cd>& c, const std::array<std::vector<double>, DIM>& s) {
  const std::size_t K = s[0].size();
  std::vector<cd> f(K, cd(0, 0));
  for (std::size_t k = 0; k < K; ++k) {
    cd acc(0, 0);
    for (std::size_t j = 0; j < c.size(); ++j) {
      double ph = 0;
      for (std::size_t d = 0; d < DIM; ++d) ph += s[d][k] * x[d][j];
      acc += c[j] * std::polar(1.0, sign * ph);
    }
    f[k] = acc;
  }
  return f;
}

// ---------------------------------------------------------------------------------------------
// Device buffers of T (real) or complex<T>, filled from / read back to FP64 host vectors.
// ---------------------------------------------------------------------------------------------
template <typename X>
struct DeviceBuffer {
  X* ptr = nullptr;
  std::size_t n = 0;
  explicit DeviceBuffer(std::size_t count) : n(count) {
    if (n) cuda_ok(cudaMalloc(reinterpret_cast<void**>(&ptr), n * sizeof(X)), "cudaMalloc");
  }
  ~DeviceBuffer() {
    if (ptr) cudaFree(ptr);
  }
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
};

template <typename T>
std::unique_ptr<DeviceBuffer<T>> upload_real(const std::vector<double>& h, cudaStream_t s) {
  std::vector<T> tmp(h.begin(), h.end());
  auto d = std::make_unique<DeviceBuffer<T>>(h.size());
  cuda_ok(cudaMemcpyAsync(d->ptr, tmp.data(), tmp.size() * sizeof(T), cudaMemcpyHostToDevice, s),
          "upload");
  cuda_ok(cudaStreamSynchronize(s), "sync");
  return d;
}

template <typename T>
using DevC = DeviceBuffer<neonufft::gpu::ComplexType<T>>;

template <typename T>
std::unique_ptr<DevC<T>> upload_cplx(const std::vector<cd>& h, cudaStream_t s) {
  std::vector<std::complex<T>> tmp(h.size());
  for (std::size_t i = 0; i < h.size(); ++i) tmp[i] = std::complex<T>(T(h[i].real()), T(h[i].imag()));
  auto d = std::make_unique<DevC<T>>(h.size());
  cuda_ok(cudaMemcpyAsync(d->ptr, tmp.data(), tmp.size() * sizeof(tmp[0]), cudaMemcpyHostToDevice,
                          s),
          "upload");
  cuda_ok(cudaStreamSynchronize(s), "sync");
  return d;
}

template <typename T>
std::vector<cd> download_cplx(const DevC<T>& d, cudaStream_t s) {
  std::vector<std::complex<T>> tmp(d.n);
  cuda_ok(cudaMemcpyAsync(tmp.data(), d.ptr, tmp.size() * sizeof(tmp[0]), cudaMemcpyDeviceToHost,
                          s),
          "download");
  cuda_ok(cudaStreamSynchronize(s), "sync");
  return std::vector<cd>(tmp.begin(), tmp.end());
}

std::vector<double> uniform(std::mt19937_64& rng, std::size_t n, double lo, double hi) {
  std::uniform_real_distribution<double> u(lo, hi);
  std::vector<double> v(n);
  for (auto& a : v) a = u(rng);
  return v;
}

std::vector<cd> strengths(std::mt19937_64& rng, std::size_t n) {
  std::uniform_real_distribution<double> u(-1.0, 1.0);
  std::vector<cd> v(n);
  for (auto& a : v) a = cd(u(rng), u(rng));
  return v;
}

void check_err(const std::string& what, double err, double bound) {
  char buf[160];
  std::snprintf(buf, sizeof(buf), "%s rel-l2 %.3e (bound %.1e)", what.c_str(), err, bound);
  if (!(err <= bound)) fail(buf);
  pass(buf);
}

// Allocator that counts live allocations, optionally failing once `budget` allocations were
// made (allocate returns nullptr, as the reference's Allocator interface allows for failure).
class CountingAllocator : public neonufft::Allocator {
public:
  explicit CountingAllocator(long budget = -1) : budget_(budget) {}
  void* allocate(std::size_t size) override {
    if (budget_ >= 0 && made_ >= budget_) return nullptr;
    void* p = inner_.allocate(size);
    if (p) {
      ++made_;
      ++live_;
    }
    return p;
  }
  void deallocate(void* ptr) noexcept override {
    if (!ptr) return;
    --live_;
    inner_.deallocate(ptr);
  }
  long made() const { return made_; }
  long live() const { return live_; }

private:
  neonufft::gpu::DeviceAllocator inner_;
  long budget_;
  long made_ = 0;
  long live_ = 0;
};

// ---------------------------------------------------------------------------------------------
// Checks without a device.
// ---------------------------------------------------------------------------------------------
void run_cpu() {
  using neonufft::InputError;
  using neonufft::gpu::Plan;
  using neonufft::gpu::PlanT3;
  const cudaStream_t s = nullptr;
  expect_throw<InputError>("Plan tol < 0", [&] {
    Options o;
    o.tol = -1.0;
    Plan<float, 1> p(o, -1, 0, {nullptr}, {8}, s);
  });
  expect_throw<InputError>("Plan upsampfac 1", [&] {
    Options o;
    o.upsampfac = 1.0;
    Plan<double, 2> p(o, -1, 0, {nullptr, nullptr}, {8, 8}, s);
  });
  expect_throw<InputError>("Plan zero modes", [&] {
    Plan<float, 3> p(Options(), 1, 0, {nullptr, nullptr, nullptr}, {8, 0, 8}, s);
  });
  expect_throw<InputError>("Plan bad mode order", [&] {
    Options o;
    o.order = static_cast<NeonufftModeOrder>(7);
    Plan<double, 1> p(o, 1, 0, {nullptr}, {8}, s);
  });
  expect_throw<InputError>("PlanT3 inverted input bounds", [&] {
    PlanT3<double, 2> p(Options(), -1, {1.0, 0.0}, {0.0, 1.0}, {-1.0, -1.0}, {1.0, 1.0}, s);
  });
  expect_throw<InputError>("PlanT3 batch size 0", [&] {
    PlanT3<float, 1> p(Options(), -1, {0.f}, {1.f}, {0.f}, {1.f}, s, 0);
  });
  Options o;
  o.tol = 1e-6;
  const auto small = PlanT3<double, 2>::grid_memory_size(o, {-1, -1}, {1, 1}, {-10, -10}, {10, 10});
  const auto large =
      PlanT3<double, 2>::grid_memory_size(o, {-1, -1}, {1, 1}, {-100, -100}, {100, 100});
  if (!(small > 0 && large > small)) fail("grid_memory_size grows with the output extent");
  pass("grid_memory_size " + std::to_string(small) + " < " + std::to_string(large));
}

// ---------------------------------------------------------------------------------------------
// Transforms on the device.
// ---------------------------------------------------------------------------------------------
template <typename T, std::size_t DIM>
void type12(const std::string& name, std::array<IntType, DIM> modes, std::size_t M, double tol,
            double bound, cudaStream_t stream, std::mt19937_64& rng) {
  using neonufft::gpu::Plan;
  std::array<std::vector<double>, DIM> x;
  for (auto& v : x) v = uniform(rng, M, -M_PI, M_PI);
  // points snapped to the precision of the plan, so that the direct sums see the same points
  for (auto& v : x)
    for (auto& a : v) a = double(T(a));
  IntType total = 1;
  for (auto n : modes) total *= n;
  std::array<IntType, DIM> strides;
  IntType st = 1;
  for (std::size_t d = 0; d < DIM; ++d) {
    strides[d] = st;
    st *= modes[d];
  }
  std::array<std::unique_ptr<DeviceBuffer<T>>, DIM> xd;
  std::array<const T*, DIM> loc;
  for (std::size_t d = 0; d < DIM; ++d) {
    xd[d] = upload_real<T>(x[d], stream);
    loc[d] = xd[d]->ptr;
  }
  Options opt;
  opt.tol = tol;
  Plan<T, DIM> plan(opt, -1, IntType(M), loc, modes, stream);

  const auto c = strengths(rng, M);
  auto cd1 = upload_cplx<T>(c, stream);
  DevC<T> f{std::size_t(total)};
  plan.transform_type_1(cd1->ptr, f.ptr, strides);
  check_err(name + " type 1", rel_l2(download_cplx<T>(f, stream), direct_type1<DIM>(-1, x, c, modes)),
            bound);

  const auto fh = strengths(rng, std::size_t(total));
  auto fd = upload_cplx<T>(fh, stream);
  DevC<T> out(M);
  plan.transform_type_2(fd->ptr, strides, out.ptr);
  check_err(name + " type 2", rel_l2(download_cplx<T>(out, stream), direct_type2<DIM>(-1, x, fh, modes)),
            bound);

  // a new point set of another size on the same plan (reference Plan::set_points)
  const std::size_t M2 = M / 2 + 7;
  std::array<std::vector<double>, DIM> y;
  for (auto& v : y) {
    v = uniform(rng, M2, -M_PI, M_PI);
    for (auto& a : v) a = double(T(a));
  }
  std::array<std::unique_ptr<DeviceBuffer<T>>, DIM> yd;
  for (std::size_t d = 0; d < DIM; ++d) {
    yd[d] = upload_real<T>(y[d], stream);
    loc[d] = yd[d]->ptr;
  }
  plan.set_points(IntType(M2), loc);
  DevC<T> out2(M2);
  plan.transform_type_2(fd->ptr, strides, out2.ptr);
  check_err(name + " set_points + type 2",
            rel_l2(download_cplx<T>(out2, stream), direct_type2<DIM>(-1, y, fh, modes)), bound);
}

template <typename T, std::size_t DIM>
void type3(const std::string& name, std::size_t M, std::size_t K, double in_ext, double out_ext,
           double tol, double bound, cudaStream_t stream, std::mt19937_64& rng) {
  using neonufft::gpu::PlanT3;
  std::array<std::vector<double>, DIM> x, s;
  for (auto& v : x) {
    v = uniform(rng, M, -in_ext, in_ext);
    for (auto& a : v) a = double(T(a));
  }
  for (auto& v : s) {
    v = uniform(rng, K, -out_ext, out_ext);
    for (auto& a : v) a = double(T(a));
  }
  std::array<std::unique_ptr<DeviceBuffer<T>>, DIM> xd, sd;
  std::array<const T*, DIM> xp, sp;
  for (std::size_t d = 0; d < DIM; ++d) {
    xd[d] = upload_real<T>(x[d], stream);
    sd[d] = upload_real<T>(s[d], stream);
    xp[d] = xd[d]->ptr;
    sp[d] = sd[d]->ptr;
  }
  Options opt;
  opt.tol = tol;
  const auto c1 = strengths(rng, M);
  const auto c2 = strengths(rng, M);
  std::vector<cd> c12(M);
  for (std::size_t j = 0; j < M; ++j) c12[j] = c1[j] + c2[j];
  auto d1 = upload_cplx<T>(c1, stream);
  auto d2 = upload_cplx<T>(c2, stream);
  DevC<T> out(K);

  // points constructor; two inputs accumulate until transform (reference PlanT3::add_input)
  {
    PlanT3<T, DIM> plan(opt, 1, IntType(M), xp, IntType(K), sp, stream);
    plan.add_input(d1->ptr);
    plan.add_input(d2->ptr);
    plan.transform(out.ptr);
    check_err(name + " add_input x2", rel_l2(download_cplx<T>(out, stream), direct_type3<DIM>(1, x, c12, s)),
              bound);
    plan.reset();
    plan.add_input(d1->ptr);
    plan.transform(out.ptr);
    check_err(name + " reset + add_input",
              rel_l2(download_cplx<T>(out, stream), direct_type3<DIM>(1, x, c1, s)), bound);
  }
  // bounds constructor, batch of 2 with explicit batch distances
  {
    std::array<T, DIM> in_min, in_max, out_min, out_max;
    for (std::size_t d = 0; d < DIM; ++d) {
      in_min[d] = T(-in_ext);
      in_max[d] = T(in_ext);
      out_min[d] = T(-out_ext);
      out_max[d] = T(out_ext);
    }
    PlanT3<T, DIM> plan(opt, 1, in_min, in_max, out_min, out_max, stream, 2);
    plan.set_input_points(IntType(M), xp);
    plan.set_output_points(IntType(K), sp);
    std::vector<cd> both(c1);
    both.insert(both.end(), c2.begin(), c2.end());
    auto db = upload_cplx<T>(both, stream);
    DevC<T> outb(2 * K);
    plan.add_input(db->ptr, IntType(M));
    plan.transform(outb.ptr, IntType(K));
    const auto got = download_cplx<T>(outb, stream);
    const std::vector<cd> g1(got.begin(), got.begin() + long(K)), g2(got.begin() + long(K), got.end());
    check_err(name + " batch 2 [0]", rel_l2(g1, direct_type3<DIM>(1, x, c1, s)), bound);
    check_err(name + " batch 2 [1]", rel_l2(g2, direct_type3<DIM>(1, x, c2, s)), bound);
  }
}

void allocators(cudaStream_t stream, std::mt19937_64& rng) {
  using neonufft::gpu::Plan;
  const std::size_t M = 500;
  std::array<std::vector<double>, 2> x;
  for (auto& v : x) v = uniform(rng, M, -M_PI, M_PI);
  auto x0 = upload_real<float>(x[0], stream);
  auto x1 = upload_real<float>(x[1], stream);
  const std::array<const float*, 2> loc{x0->ptr, x1->ptr};
  Options opt;
  opt.tol = 1e-4;

  // every device allocation of the plan goes through the caller's allocator, and is returned
  auto counting = std::make_shared<CountingAllocator>();
  {
    Plan<float, 2> plan(opt, -1, IntType(M), loc, {24, 20}, stream, counting);
    const auto c = strengths(rng, M);
    auto cdv = upload_cplx<float>(c, stream);
    DevC<float> f{24 * 20};
    plan.transform_type_1(cdv->ptr, f.ptr, {1, 24});
    cuda_ok(cudaStreamSynchronize(stream), "sync");
    if (counting->made() < 1 || counting->live() < 1) fail("plan allocated through the allocator");
  }
  if (counting->live() != 0) fail("plan returned every allocation");
  pass("plan allocations through the caller's allocator: " + std::to_string(counting->made()) +
       " made, all returned");

  // an allocator that fails at every point of plan construction: MemoryAllocError, no leak
  const long needed = counting->made();
  for (long budget = 0; budget < needed; ++budget) {
    auto failing = std::make_shared<CountingAllocator>(budget);
    try {
      Plan<float, 2> plan(opt, -1, IntType(M), loc, {24, 20}, stream, failing);
      const auto c = strengths(rng, M);
      auto cdv = upload_cplx<float>(c, stream);
      DevC<float> f{24 * 20};
      plan.transform_type_1(cdv->ptr, f.ptr, {1, 24});
      cuda_ok(cudaStreamSynchronize(stream), "sync");
      fail("allocation budget " + std::to_string(budget) + " did not fail");
    } catch (const neonufft::MemoryAllocError&) {
    }
    if (failing->live() != 0) fail("leak after allocation failure at " + std::to_string(budget));
  }
  pass("MemoryAllocError at each of " + std::to_string(needed) +
       " allocation points, nothing leaked");
  // the context is still usable afterwards
  {
    Plan<float, 2> plan(opt, -1, IntType(M), loc, {24, 20}, stream);
    const auto c = strengths(rng, M);
    auto cdv = upload_cplx<float>(c, stream);
    DevC<float> f{24 * 20};
    plan.transform_type_1(cdv->ptr, f.ptr, {1, 24});
    std::array<std::vector<double>, 2> xs{std::vector<double>(x[0].begin(), x[0].end()),
                                          std::vector<double>(x[1].begin(), x[1].end())};
    for (auto& v : xs)
      for (auto& a : v) a = double(float(a));
    check_err("plan after allocation failures",
              rel_l2(download_cplx<float>(f, stream), direct_type1<2>(-1, xs, c, {24, 20})), 1e-3);
  }
}

void run_gpu() {
  std::mt19937_64 rng(42);
  cudaStream_t stream;
  cuda_ok(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
  type12<float, 1>("Plan<float,1>", {37}, 300, 1e-5, 1e-4, stream, rng);
  type12<double, 1>("Plan<double,1>", {64}, 300, 1e-10, 1e-9, stream, rng);
  type12<float, 2>("Plan<float,2>", {20, 17}, 400, 1e-5, 1e-4, stream, rng);
  type12<double, 2>("Plan<double,2>", {16, 24}, 400, 1e-9, 1e-8, stream, rng);
  type12<float, 3>("Plan<float,3>", {12, 10, 9}, 600, 1e-6, 1e-5, stream, rng);
  type12<double, 3>("Plan<double,3>", {8, 12, 10}, 600, 1e-8, 1e-7, stream, rng);
  type3<double, 1>("PlanT3<double,1>", 300, 200, 3.0, 40.0, 1e-9, 1e-8, stream, rng);
  type3<float, 2>("PlanT3<float,2>", 300, 200, 2.0, 20.0, 1e-4, 1e-3, stream, rng);
  type3<double, 3>("PlanT3<double,3>", 200, 150, 1.5, 8.0, 1e-7, 1e-6, stream, rng);
  allocators(stream, rng);
  cuda_ok(cudaStreamDestroy(stream), "cudaStreamDestroy");
}

}  // namespace

int main(int argc, char** argv) {
  const std::string mode = argc > 1 ? argv[1] : "cpu";
  if (mode == "cpu") {
    run_cpu();
  } else if (mode == "gpu") {
    run_gpu();
  } else {
    std::fprintf(stderr, "usage: %s cpu|gpu\n", argv[0]);
    return 2;
  }
  std::printf("%d checks passed\n", g_checks);
  return 0;
}
