/*
 * Host-side harness around the reference's thrust-based operations, built
 * with thrust's OpenMP device system so they run on the CPU.
 *
 * TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile from the reference
 * sources where they lie (REF_SRC), into oracle/_ref/.  Nothing of the
 * reference is copied: its headers are #included and instantiated.
 *   cooSort            src/cooSort.hpp:75-99
 *   mlemOperations     src/mlemOperations.hpp:44-169
 *   convertCsr2Ecsr    src/convertCsr2Ecsr.hpp:51-64
 */
#include <cstdint>

/* __host__/__device__ qualifiers used by the reference headers. */
#include <cuda_runtime.h>

#include "cooSort.hpp"
#include "convertCsr2Ecsr.hpp"
#include "mlemOperations.hpp"

extern "C" {

void ref_coo_sort(float* val, int32_t* row, int32_t* col, int32_t n) { cooSort<float>(val, row, col, n); }

void ref_divides(float* res, float* a, float* b, int32_t n) { divides<float>(res, a, b, n); }

void ref_divides_multiplies(float* res, float* a, float* b, float* c, int32_t n) {
  dividesMultiplies<float>(res, a, b, c, n);
}

void ref_scales(float* x, float alpha, int32_t n) { scales<float>(x, alpha, n); }

float ref_sum(float* x, int32_t n) { return sum<float>(x, n); }

void ref_csr2ecsr(int32_t* ecsr, int32_t* yrow, int32_t nnzr, int32_t* csr, int32_t m) {
  convertCsr2Ecsr(ecsr, yrow, nnzr, csr, m);
}

}  // extern "C"
