// R1CS SpMV kernels (design notes in spmv.cuh).
#include <cstring>
#include <vector>

#include "spmv.cuh"

namespace nkr {

namespace {

struct SpmvArgs {
    const uint32_t *row_ptr[3];
    const uint32_t *col[3];
    const uint32_t *nu_col[3];
    const Fr *nu_val[3];
    Fr *prod[3];
    Fr *y[3];
    uint64_t rows[3];
    uint64_t nu[3];
    int lanes[3];
};

__device__ __forceinline__ Fr shfl_down_fr(const Fr &a, int off, int width)
{
    Fr r;
#pragma unroll
    for (int i = 0; i < 8; ++i) r.v[i] = __shfl_down_sync(0xffffffffu, a.v[i], off, width);
    return r;
}

// phase 1: prod[k] = nu_val[k] * z[nu_col[k]], one thread per non-unit term
__global__ void __launch_bounds__(256) k_spmv_products(SpmvArgs a, const Fr *__restrict__ z)
{
    const int m = blockIdx.y;
    const uint64_t k = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= a.nu[m]) return;
    a.prod[m][k] = a.nu_val[m][k] * z[a.nu_col[m][k]];
}

// phase 2: row sums of z[col] (unit terms) and prod[k] (the others)
__global__ void __launch_bounds__(256) k_spmv(SpmvArgs a, const Fr *__restrict__ z)
{
    const int m = blockIdx.y;
    const int L = a.lanes[m];
    const uint64_t tid = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint64_t row = tid / L;
    const int lane = int(tid % L);
    const uint64_t rows = a.rows[m];
    Fr acc = Fr::zero();
    if (row < rows) {
        const uint32_t *__restrict__ col = a.col[m];
        const Fr *__restrict__ prod = a.prod[m];
        const uint32_t beg = a.row_ptr[m][row], end = a.row_ptr[m][row + 1];
        for (uint32_t j = beg + lane; j < end; j += L) {
            const uint32_t c = col[j];
            if (c & kColZero) continue;
            acc = acc + ((c & kColOne) ? z[c & kColMask] : prod[c]);
        }
    }
    for (int off = L >> 1; off > 0; off >>= 1) acc = acc + shfl_down_fr(acc, off, L);
    if (lane == 0 && row < rows) a.y[m][row] = acc;
}

} // namespace

int csr_upload(CsrDevice &m, uint64_t rows, uint64_t cols, const uint32_t *row_ptr,
               const uint32_t *col_idx, const void *values, cudaStream_t st)
{
    NKR_REQUIRE(rows > 0 && row_ptr != nullptr, "empty CSR matrix");
    NKR_REQUIRE(cols <= kColMask, "column count %llu exceeds 2^30", (unsigned long long)cols);
    const uint64_t nnz = row_ptr[rows];
    NKR_REQUIRE(row_ptr[0] == 0, "CSR row_ptr[0] must be 0");
    for (uint64_t r = 0; r < rows; ++r)
        NKR_REQUIRE(row_ptr[r + 1] >= row_ptr[r], "non-monotonic CSR offsets at row %llu",
                    (unsigned long long)r);
    m.rows = rows;
    m.cols = cols;
    m.nnz = nnz;
    // Montgomery one of Fr, little-endian bytes (R mod r)
    static const uint32_t kOne[8] = {0x4ffffffbu, 0xac96341cu, 0x9f60cd29u, 0x36fc7695u,
                                     0x7879462eu, 0x666ea36fu, 0x9a07df2fu, 0x0e0a77c1u};
    static const uint32_t kZero[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    std::vector<uint32_t> tagged(nnz), nu_col;
    std::vector<uint8_t> nu_val;
    const uint8_t *vb = static_cast<const uint8_t *>(values);
    for (uint64_t j = 0; j < nnz; ++j) {
        NKR_REQUIRE(col_idx[j] < cols, "CSR column %u out of range", col_idx[j]);
        if (std::memcmp(vb + 32 * j, kOne, 32) == 0) {
            tagged[j] = col_idx[j] | kColOne;
        } else if (std::memcmp(vb + 32 * j, kZero, 32) == 0) {
            tagged[j] = kColZero;
        } else {
            NKR_REQUIRE(nu_col.size() < kColZero, "more than 2^30 non-unit terms");
            tagged[j] = uint32_t(nu_col.size());
            nu_col.push_back(col_idx[j]);
            nu_val.insert(nu_val.end(), vb + 32 * j, vb + 32 * j + 32);
        }
    }
    m.nu = nu_col.size();
    NKR_TRY(m.row_ptr.alloc((rows + 1) * 4, "CSR row_ptr"));
    NKR_TRY(m.col.alloc(std::max<uint64_t>(nnz, 1) * 4, "CSR columns"));
    NKR_TRY(m.nu_col.alloc(std::max<uint64_t>(m.nu, 1) * 4, "CSR non-unit columns"));
    NKR_TRY(m.nu_val.alloc(std::max<uint64_t>(m.nu, 1) * 32, "CSR non-unit values"));
    NKR_CUDA(cudaMemcpyAsync(m.row_ptr.p, row_ptr, (rows + 1) * 4, cudaMemcpyHostToDevice, st));
    if (nnz) NKR_CUDA(cudaMemcpyAsync(m.col.p, tagged.data(), nnz * 4, cudaMemcpyHostToDevice, st));
    if (m.nu) {
        NKR_CUDA(cudaMemcpyAsync(m.nu_col.p, nu_col.data(), m.nu * 4, cudaMemcpyHostToDevice, st));
        NKR_CUDA(cudaMemcpyAsync(m.nu_val.p, nu_val.data(), m.nu * 32, cudaMemcpyHostToDevice, st));
    }
    // sub-warp width: power of two near the mean row length, at most 32
    const double avg = double(nnz) / double(rows);
    int L = 1;
    while (L < 32 && L < avg) L <<= 1;
    m.lanes = L;
    NKR_CUDA(cudaStreamSynchronize(st)); // the staging vectors are pageable host memory
    return NKR_B200_OK;
}

int spmv_multi(const CsrDevice *const *mats, int count, const Fr *z, Fr *const *y,
               Fr *const *prod, cudaStream_t st)
{
    NKR_REQUIRE(count >= 1 && count <= 3, "spmv_multi takes 1..3 matrices");
    SpmvArgs a{};
    uint64_t work = 0, nu_max = 0;
    for (int k = 0; k < count; ++k) {
        a.row_ptr[k] = mats[k]->row_ptr.as<uint32_t>();
        a.col[k] = mats[k]->col.as<uint32_t>();
        a.nu_col[k] = mats[k]->nu_col.as<uint32_t>();
        a.nu_val[k] = mats[k]->nu_val.as<Fr>();
        a.prod[k] = prod[k];
        a.y[k] = y[k];
        a.rows[k] = mats[k]->rows;
        a.nu[k] = mats[k]->nu;
        a.lanes[k] = mats[k]->lanes;
        work = std::max<uint64_t>(work, mats[k]->rows * uint64_t(mats[k]->lanes));
        nu_max = std::max<uint64_t>(nu_max, mats[k]->nu);
    }
    if (nu_max) {
        k_spmv_products<<<dim3(blocks_for(nu_max, 256), count), 256, 0, st>>>(a, z);
        NKR_CHECK_LAUNCH();
    }
    k_spmv<<<dim3(blocks_for(work, 256), count), 256, 0, st>>>(a, z);
    NKR_CHECK_LAUNCH();
    return NKR_B200_OK;
}

} // namespace nkr
