// Thin C entry points over the reference's own CUDA Groth16 backend
// (protocols/groth16/backends/cuda/src/groth16_backend.cu: CudaBackend::prepare
// :214-240 and ::prove :242-279), compiled in place from the reference sources
// for sm_100a by oracle/Makefile (target refcuda) into oracle/_ref/.
//
// Test infrastructure only: a GPU test times the reference's GPU prove beside
// this repository's on the same circuit and keys.  Every computation is the
// reference's code; this file only converts raw byte buffers into the
// reference's Circuit / ProvingKey types and back.  The reference's prepare
// copies only (X, Y) of each proving-key point (operators/cuda/include/msm/
// msm.cuh:51-57), so the keys handed in must be affine-normalised (Z = 1).
#include <chrono>
#include <cuda_runtime.h>
#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <vector>

#include "groth16/backend.hpp"
#include "groth16/types.hpp"
#include "libff/common/profiling.hpp"

namespace nkr::groth16 {
std::unique_ptr<Backend> make_cuda_backend(); // groth16_backend.cu:284
}

using namespace nkr::groth16;

// A reference-layout circuit handed over as one struct of raw pointers (at
// namespace scope: a type with internal linkage would hide refcuda_open).
struct RawCircuit {
    uint64_t rows, cols, public_inputs;
    const uint32_t *row_ptr[3];
    const uint32_t *col_idx[3];
    const void *values[3];
};

namespace {

thread_local std::string g_error;
thread_local double g_prepare_ms = 0;

template <typename T>
std::vector<T> from_raw(const void *p, std::size_t n)
{
    std::vector<T> v(n);
    if (n) std::memcpy(static_cast<void *>(v.data()), p, n * sizeof(T));
    return v;
}

CsrMatrix<Scalar> csr_from_raw(std::size_t rows, std::size_t cols, const uint32_t *row_ptr,
                               const uint32_t *col_idx, const void *values)
{
    CsrMatrix<Scalar> m;
    m.num_rows = rows;
    m.num_cols = cols;
    m.row_ptr.assign(row_ptr, row_ptr + rows + 1);
    const std::size_t nnz = row_ptr[rows];
    m.col_idx.assign(col_idx, col_idx + nnz);
    m.values = from_raw<Scalar>(values, nnz);
    return m;
}

struct RefCudaProver {
    Circuit circuit;
    ProvingKey pk;
    std::unique_ptr<Backend> backend;
};

bool g_inited = false;

} // namespace

extern "C" {

const char *refcuda_last_error(void) { return g_error.c_str(); }

// Host wall time of the last refcuda_open's CudaBackend::prepare (device
// layout, key upload), followed by a device synchronisation.
double refcuda_last_prepare_ms(void) { return g_prepare_ms; }

// Builds the circuit and proving key from raw buffers and runs the reference's
// CudaBackend::prepare (device layout, key upload).  Queries: a, b_g1, l (G1[cols]),
// b_g2 (G2[cols]), h (G1[rows]) in libff Jacobian layout with Z = 1.
void *refcuda_open(const RawCircuit *rc, const void *a_query, const void *b_g1_query,
                   const void *b_g2_query, const void *l_query, const void *h_query)
{
    try {
        if (!g_inited) {
            libff::inhibit_profiling_info = true;
            libff::inhibit_profiling_counters = true;
            Curve::init_public_params();
            g_inited = true;
        }
        auto p = std::make_unique<RefCudaProver>();
        p->circuit.public_inputs = rc->public_inputs;
        p->circuit.a = csr_from_raw(rc->rows, rc->cols, rc->row_ptr[0], rc->col_idx[0], rc->values[0]);
        p->circuit.b = csr_from_raw(rc->rows, rc->cols, rc->row_ptr[1], rc->col_idx[1], rc->values[1]);
        p->circuit.c = csr_from_raw(rc->rows, rc->cols, rc->row_ptr[2], rc->col_idx[2], rc->values[2]);
        p->pk.a_query = from_raw<G1>(a_query, rc->cols);
        p->pk.b_g1_query = from_raw<G1>(b_g1_query, rc->cols);
        p->pk.b_g2_query = from_raw<G2>(b_g2_query, rc->cols);
        p->pk.l_query = from_raw<G1>(l_query, rc->cols);
        p->pk.h_query = from_raw<G1>(h_query, rc->rows);
        p->pk.alpha_g1 = p->pk.beta_g1 = p->pk.delta_g1 = G1::one();
        p->pk.beta_g2 = p->pk.delta_g2 = G2::one();
        p->backend = make_cuda_backend();
        const auto t0 = std::chrono::steady_clock::now();
        p->backend->prepare(p->circuit, p->pk);
        cudaDeviceSynchronize();
        const auto t1 = std::chrono::steady_clock::now();
        g_prepare_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
        return p.release();
    } catch (const std::exception &e) {
        g_error = e.what();
        return nullptr;
    }
}

// One CudaBackend::prove; ms = host wall time of the call (the reference's
// groth16.cuda.prove.total scope: it returns with the raw proof on the host).
// Outputs: {ar, bs1, zk, qz} G1 affine (64 B each) and bs2 G2 affine (128 B).
int refcuda_prove(void *h, const void *witness, void *g1_out4, void *g2_out, double *ms)
{
    try {
        auto *p = static_cast<RefCudaProver *>(h);
        auto w = from_raw<Scalar>(witness, p->circuit.a.num_cols);
        RawProof raw;
        const auto t0 = std::chrono::steady_clock::now();
        p->backend->prove(p->circuit, p->pk, w, raw);
        const auto t1 = std::chrono::steady_clock::now();
        if (ms) *ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
        char *o = static_cast<char *>(g1_out4);
        G1 pts[4] = {raw.ar, raw.bs1, raw.zk, raw.qz};
        for (int i = 0; i < 4; ++i) {
            pts[i].to_affine_coordinates();
            std::memcpy(o + 64 * i, &pts[i], 64);
        }
        G2 b = raw.bs2;
        b.to_affine_coordinates();
        std::memcpy(g2_out, &b, 128);
        return 0;
    } catch (const std::exception &e) {
        g_error = e.what();
        return 1;
    }
}

void refcuda_close(void *h) { delete static_cast<RefCudaProver *>(h); }

} // extern "C"
