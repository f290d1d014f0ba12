// Drop-in check (test infrastructure): the reference's own Groth16 code driving
// the B200 backend through nkr::groth16::Backend, exactly as groth16-prove does
// (protocols/groth16/app/prove.cpp:70-88): make the backend, prepare, prove,
// the reference's blind_proof and verify.  Built by `make -C oracle dropin`
// into oracle/_ref/libnkr_ref_b200.so from the reference objects, this file and
// nkr-zkp_b200/integration/b200_backend.cpp, linked against libnkr_b200.so.
#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "groth16/backend.hpp"
#include "groth16/io.hpp"
#include "groth16/protocol.hpp"
#include "groth16/types.hpp"
#include "libff/common/profiling.hpp"

namespace nkr::groth16 {
std::unique_ptr<Backend> make_b200_backend();
}

using namespace nkr::groth16;

namespace {

thread_local std::string g_err;

struct RawCircuit {
    uint64_t rows, cols, public_inputs;
    const uint32_t *row_ptr[3];
    const uint32_t *col_idx[3];
    const void *values[3];
};

CsrMatrix<Scalar> csr(std::size_t rows, std::size_t cols, const uint32_t *rp, const uint32_t *ci,
                      const void *vals)
{
    CsrMatrix<Scalar> m;
    m.num_rows = rows;
    m.num_cols = cols;
    m.row_ptr.assign(rp, rp + rows + 1);
    m.col_idx.assign(ci, ci + rp[rows]);
    m.values.resize(rp[rows]);
    if (rp[rows]) std::memcpy(static_cast<void *>(m.values.data()), vals, rp[rows] * 32);
    return m;
}

Circuit circuit(const RawCircuit &r)
{
    Circuit c;
    c.public_inputs = r.public_inputs;
    c.a = csr(r.rows, r.cols, r.row_ptr[0], r.col_idx[0], r.values[0]);
    c.b = csr(r.rows, r.cols, r.row_ptr[1], r.col_idx[1], r.values[1]);
    c.c = csr(r.rows, r.cols, r.row_ptr[2], r.col_idx[2], r.values[2]);
    return c;
}

bool init_done = false;

} // namespace

extern "C" {

const char *dropin_last_error(void) { return g_err.c_str(); }

// Prove with the B200 backend on the reference's types, blind with the
// reference's blind_proof, verify with the reference's verifier, and compare the
// raw proof with the reference CPU backend's (libff projective equality).
// pk_path / vk_path: reference artifacts (e.g. from the CPU setup); when
// gpu_setup != 0 the B200 backend's own setup makes fresh keys instead.
int dropin_prove_verify(const RawCircuit *rc, const char *pk_path, const char *vk_path,
                        const void *witness, int gpu_setup, int *verified, int *raw_equal,
                        char *name_out)
{
    try {
        if (!init_done) {
            libff::inhibit_profiling_info = true;
            libff::inhibit_profiling_counters = true;
            Curve::init_public_params();
            init_done = true;
        }
        const Circuit c = circuit(*rc);
        std::vector<Scalar> w(c.a.num_cols);
        std::memcpy(static_cast<void *>(w.data()), witness, w.size() * 32);
        auto backend = make_backend("cpu"); // registry still serves the CPU backend
        auto b200 = make_b200_backend();
        std::strncpy(name_out, b200->name(), 15);
        ProvingKey pk;
        VerificationKey vk;
        if (gpu_setup) {
            b200->setup(c, pk, vk);
        } else {
            pk = read_proving_key(pk_path);
            vk = read_verification_key(vk_path);
        }
        std::string err;
        if (!validate_circuit(c, err) || !validate_proving_key(c, pk, err))
            throw std::runtime_error("invalid inputs: " + err);
        b200->prepare(c, pk);
        RawProof raw;
        b200->prove(c, pk, w, raw);
        const Proof proof = blind_proof(pk, raw);
        const std::vector<Scalar> pub(w.begin() + 1, w.begin() + 1 + c.public_inputs);
        *verified = verify(vk, pub, proof) ? 1 : 0;
        RawProof cpu;
        backend->prove(c, pk, w, cpu);
        *raw_equal = (raw.ar == cpu.ar && raw.bs1 == cpu.bs1 && raw.zk == cpu.zk &&
                      raw.qz == cpu.qz && raw.bs2 == cpu.bs2)
                         ? 1
                         : 0;
        return 0;
    } catch (const std::exception &e) {
        g_err = e.what();
        return 1;
    }
}

} // extern "C"
