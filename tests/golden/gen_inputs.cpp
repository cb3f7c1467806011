// Test-input generator: reproduces the inputs of the reference's tests exactly by drawing them
// with the same standard-library engine and distribution (std::minstd_rand seeded with 42 and
// std::uniform_real_distribution<T>, reference tests/test_type_1_2.cpp:63-81, :120-124,
// :208-226 and tests/test_type_3.cpp:56-87, :243-265). Built by tests/golden/build_gen.py.
//
// gen_segments_{f32,f64}: one generator stream, nseg consecutive segments of n[i] values drawn
// from U(a[i], b[i]); complex segments (cplx[i] != 0) draw 2*n[i] values (re, im per element).
#include <cstdint>
#include <random>

template <typename T>
static void gen(int nseg, const int64_t* n, const double* a, const double* b, const int* cplx,
                T* out) {
  std::minstd_rand rand_gen(42);
  for (int s = 0; s < nseg; ++s) {
    std::uniform_real_distribution<T> dist(T(a[s]), T(b[s]));
    const int64_t m = cplx[s] ? 2 * n[s] : n[s];
    for (int64_t i = 0; i < m; ++i) *out++ = dist(rand_gen);
  }
}

extern "C" {
void gen_segments_f32(int nseg, const int64_t* n, const double* a, const double* b,
                      const int* cplx, float* out) {
  gen<float>(nseg, n, a, b, cplx, out);
}
void gen_segments_f64(int nseg, const int64_t* n, const double* a, const double* b,
                      const int* cplx, double* out) {
  gen<double>(nseg, n, a, b, cplx, out);
}
}
