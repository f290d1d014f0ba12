// R1CS SpMV kernels (design notes in spmv.cuh).
#include <cstring>
#include <vector>

#include "spmv.cuh"

namespace nkr {

namespace {

struct SpmvArgs {
    const uint32_t *row_ptr[3];
    const uint32_t *col[3];
    const Fr *val[3];
    Fr *y[3];
    uint64_t rows[3];
    int lanes[3];
};

__device__ __forceinline__ Fr shfl_down_fr(const Fr &a, int off, int width)
{
    Fr r;
#pragma unroll
    for (int i = 0; i < 8; ++i) r.v[i] = __shfl_down_sync(0xffffffffu, a.v[i], off, width);
    return r;
}

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
        const Fr *__restrict__ val = a.val[m];
        const uint32_t beg = a.row_ptr[m][row], end = a.row_ptr[m][row + 1];
        for (uint32_t j = beg + lane; j < end; j += L) {
            const uint32_t c = col[j];
            if (c & kColZero) continue;
            const Fr zv = z[c & kColMask];
            acc = acc + ((c & kColOne) ? zv : val[j] * zv);
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
    std::vector<uint32_t> tagged(nnz);
    const uint8_t *vb = static_cast<const uint8_t *>(values);
    for (uint64_t j = 0; j < nnz; ++j) {
        NKR_REQUIRE(col_idx[j] < cols, "CSR column %u out of range", col_idx[j]);
        uint32_t c = col_idx[j];
        if (std::memcmp(vb + 32 * j, kOne, 32) == 0)
            c |= kColOne;
        else if (std::memcmp(vb + 32 * j, kZero, 32) == 0)
            c |= kColZero;
        tagged[j] = c;
    }
    NKR_TRY(m.row_ptr.alloc((rows + 1) * 4, "CSR row_ptr"));
    NKR_TRY(m.col.alloc(std::max<uint64_t>(nnz, 1) * 4, "CSR columns"));
    NKR_TRY(m.values.alloc(std::max<uint64_t>(nnz, 1) * 32, "CSR values"));
    NKR_CUDA(cudaMemcpyAsync(m.row_ptr.p, row_ptr, (rows + 1) * 4, cudaMemcpyHostToDevice, st));
    if (nnz) {
        NKR_CUDA(cudaMemcpyAsync(m.col.p, tagged.data(), nnz * 4, cudaMemcpyHostToDevice, st));
        NKR_CUDA(cudaMemcpyAsync(m.values.p, values, nnz * 32, cudaMemcpyHostToDevice, st));
    }
    // sub-warp width: power of two near the mean row length, at most 32
    const double avg = double(nnz) / double(rows);
    int L = 1;
    while (L < 32 && L < avg) L <<= 1;
    m.lanes = L;
    NKR_CUDA(cudaStreamSynchronize(st)); // `tagged` is pageable host memory
    return NKR_B200_OK;
}

int spmv_multi(const CsrDevice *const *mats, int count, const Fr *z, Fr *const *y,
               cudaStream_t st)
{
    NKR_REQUIRE(count >= 1 && count <= 3, "spmv_multi takes 1..3 matrices");
    SpmvArgs a{};
    uint64_t work = 0;
    for (int k = 0; k < count; ++k) {
        a.row_ptr[k] = mats[k]->row_ptr.as<uint32_t>();
        a.col[k] = mats[k]->col.as<uint32_t>();
        a.val[k] = mats[k]->values.as<Fr>();
        a.y[k] = y[k];
        a.rows[k] = mats[k]->rows;
        a.lanes[k] = mats[k]->lanes;
        work = std::max<uint64_t>(work, mats[k]->rows * uint64_t(mats[k]->lanes));
    }
    dim3 grid(blocks_for(work, 256), count);
    k_spmv<<<grid, 256, 0, st>>>(a, z);
    NKR_CHECK_LAUNCH();
    return NKR_B200_OK;
}

} // namespace nkr
