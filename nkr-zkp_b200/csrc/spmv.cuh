// R1CS sparse matrix-vector products az = A z, bz = B z, cz = C z over Fr.
//
// Reference: CPU multiply (backends/cpu/src/backend.cpp:25-35), CUDA thread-per-
// row kernel (backends/cuda/include/spmvm/spmvm.cuh:12-30) on three streams.
//
// Device layout (built once at prepare): per matrix row_ptr u32[rows + 1],
// col u32[nnz] whose top two bits tag the coefficient (bit 31: the value is
// Montgomery one, so the product is z itself; bit 30: the value is zero, the
// term is skipped; the R1CS builder emits such zero terms, r1cs.hpp:116), and
// values Fr[nnz] read only for untagged terms.  A sub-warp of L lanes serves
// one row with 128-bit loads of the values and the gathered z entries, then
// reduces its partial sums with shuffles.  All three matrices run in one launch.
#pragma once

#include <cstdint>

#include "common.cuh"
#include "field.cuh"

namespace nkr {

constexpr uint32_t kColOne = 0x80000000u;
constexpr uint32_t kColZero = 0x40000000u;
constexpr uint32_t kColMask = 0x3fffffffu;

struct CsrDevice {
    uint64_t rows = 0, cols = 0, nnz = 0;
    DevBuf row_ptr, col, values;
    int lanes = 1; // sub-warp width serving one row
};

// Upload one matrix, tagging unit and zero coefficients.
int csr_upload(CsrDevice &m, uint64_t rows, uint64_t cols, const uint32_t *row_ptr,
               const uint32_t *col_idx, const void *values, cudaStream_t st);

// y_k = M_k z for k < count (count <= 3), all in one launch
int spmv_multi(const CsrDevice *const *mats, int count, const Fr *z, Fr *const *y,
               cudaStream_t st);

} // namespace nkr
