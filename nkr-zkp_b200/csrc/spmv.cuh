// R1CS sparse matrix-vector products az = A z, bz = B z, cz = C z over Fr.
//
// Reference: CPU multiply (backends/cpu/src/backend.cpp:25-35), CUDA thread-per-
// row kernel (backends/cuda/include/spmvm/spmvm.cuh:12-30) on three streams.
//
// Device layout (built once at prepare): per matrix row_ptr u32[rows + 1] and
// col u32[nnz] whose top two bits tag the coefficient: bit 31 = the value is
// Montgomery one and the low bits are the column (the term is z itself); bit 30 =
// the value is zero, the term is skipped (the R1CS builder emits such terms,
// r1cs.hpp:116); untagged = any other value, and the low bits index a compact list
// (nu_col, nu_val) of those terms.  A prove runs two launches:
//   1. products: prod[k] = nu_val[k] z[nu_col[k]] for every non-unit term, one
//      thread per term, so every lane of a warp does a Montgomery product (the
//      matmul and Poseidon matrices mix unit and non-unit terms within a row, and
//      one product in a warp used to stall the lanes that only add);
//   2. sums: a sub-warp of L lanes per row adds z[col] or prod[k] per term and
//      reduces with shuffles.
// Each launch serves all three matrices (blockIdx.y); prod is per-proof scratch.
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
    uint64_t nu = 0;          // terms whose coefficient is neither one nor zero
    DevBuf row_ptr, col;      // col: tagged column or compact index (above)
    DevBuf nu_col, nu_val;    // u32[nu] columns, Fr[nu] coefficients
    int lanes = 1;            // sub-warp width serving one row
};

// Upload one matrix, tagging unit and zero coefficients.
int csr_upload(CsrDevice &m, uint64_t rows, uint64_t cols, const uint32_t *row_ptr,
               const uint32_t *col_idx, const void *values, cudaStream_t st);

// y_k = M_k z for k < count (count <= 3); prod[k] is scratch of Fr[mats[k]->nu]
int spmv_multi(const CsrDevice *const *mats, int count, const Fr *z, Fr *const *y,
               Fr *const *prod, cudaStream_t st);

} // namespace nkr
