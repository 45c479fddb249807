// ref_gen.cpp -- the reference's seeded test-matrix generator on the host.
//
// TEST INFRASTRUCTURE ONLY.  Includes the unmodified utils/matrix_gen.hpp of
// the reference tree, so the bench's reference arm draws its inputs with the
// reference's own code.  Compiled without floating-point contraction (unlike
// ref_shim.cpp): the generator's normal distribution computes x*x + y*y, which
// an FMA would round differently from the plain build the fixtures and this
// library's generator follow.  Linked into oracle/_ref/libozaref_cpu.so.
#include <cstring>
#include <vector>

#include "matrix_gen.hpp"

extern "C" {

// Seeded (U - 0.5) * exp(phi * N(0,1)) matrix, row-major, drawn by the
// reference's generate_ozaki_matrix (utils/matrix_gen.hpp:15-34).
void ref_generate_matrix(int rows, int cols, double phi, int seed, double* out) {
    const std::vector<double> m = matrix_utils::generation::generate_ozaki_matrix<double>(rows, cols, phi, seed);
    std::memcpy(out, m.data(), sizeof(double) * m.size());
}

}  // extern "C"
