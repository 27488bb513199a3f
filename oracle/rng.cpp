// Oracle helper (test infrastructure only; never linked into the product library).
//
// Draws the Gaussian sketch exactly as the reference CPU backend does:
// std::mt19937(seed) feeding std::normal_distribution<double>(0, 1), filling a
// column-major matrix in element order.  Reference: src/svd_cpu_rsvd.cpp:10-22
// (gaussian_matrix) and src/fastPLS.cpp:99-115 (gaussian_matrix_local).
// Compiled with g++ so the distribution is libstdc++'s, as in the R build.
#include <cstddef>
#include <cstdint>
#include <random>

extern "C" {

void oracle_gaussian_matrix(double* out, std::size_t n_elem, unsigned int seed) {
  std::mt19937 rng(seed);
  std::normal_distribution<double> norm(0.0, 1.0);
  for (std::size_t i = 0; i < n_elem; ++i) out[i] = norm(rng);
}

// Raw engine output, used to pin the engine against the C++ standard's
// known answer (the 10000th draw of a default-seeded mt19937 is 4123659995).
void oracle_mt19937_raw(std::uint32_t* out, std::size_t n, unsigned int seed) {
  std::mt19937 rng(seed);
  for (std::size_t i = 0; i < n; ++i) out[i] = static_cast<std::uint32_t>(rng());
}

}  // extern "C"
