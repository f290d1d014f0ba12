// Reference-side adapter: registers the B200 prover as an NKR-ZKP Groth16
// backend.  A maintainer adds this file to the reference as
// protocols/groth16/backends/b200/src/backend.cpp, with a registry entry and a
// link target for the accelerator value B200; it
// implements nkr::groth16::Backend (common/include/groth16/backend.hpp:11-28) on
// top of the C ABI in include/nkr_b200.h.  It compiles against the reference's
// own headers (libff types) and is exercised that way by the tests.
//
// The reference's types share the C ABI's byte layouts, so the adapter only
// points the ABI structs at the reference's std::vector data: CsrMatrix
// (r1cs/spmat.hpp:206-215), libff Fr / G1 / G2 (types.hpp:11-15), RawProof
// (types.hpp:47-53).
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>

#include "groth16/backend.hpp"
#include "groth16/protocol.hpp"
#include "nkr_b200.h"

namespace nkr::groth16 {

namespace {

static_assert(sizeof(Scalar) == 32 && sizeof(G1) == 96 && sizeof(G2) == 192,
              "libff layout differs from the C ABI's");

void check(int status, const char *what)
{
    if (status != NKR_B200_OK)
        throw std::runtime_error(std::string("b200 ") + what + ": " + nkr_b200_last_error());
}

nkr_b200_circuit circuit_view(const Circuit &c)
{
    nkr_b200_circuit v{};
    v.rows = c.a.num_rows;
    v.cols = c.a.num_cols;
    v.public_inputs = c.public_inputs;
    const CsrMatrix<Scalar> *m[3] = {&c.a, &c.b, &c.c};
    for (int k = 0; k < 3; ++k) {
        v.row_ptr[k] = m[k]->row_ptr.data();
        v.col_idx[k] = m[k]->col_idx.data();
        v.values[k] = m[k]->values.data();
    }
    return v;
}

nkr_b200_proving_key key_view(const ProvingKey &pk)
{
    nkr_b200_proving_key v{};
    v.a_query = pk.a_query.data();
    v.b_g1_query = pk.b_g1_query.data();
    v.b_g2_query = pk.b_g2_query.data();
    v.l_query = pk.l_query.data();
    v.h_query = pk.h_query.data();
    v.alpha_g1 = &pk.alpha_g1;
    v.beta_g1 = &pk.beta_g1;
    v.delta_g1 = &pk.delta_g1;
    v.beta_g2 = &pk.beta_g2;
    v.delta_g2 = &pk.delta_g2;
    return v;
}

class B200Backend final : public Backend {
public:
    // NKR_B200_TUNE_CACHE names a file of measured MSM window widths, kept across
    // the CLI's one-proof processes (a missing or foreign file is measured afresh)
    B200Backend()
    {
        check(nkr_b200_open(0, &ctx_), "open");
        if (const char *p = std::getenv("NKR_B200_TUNE_CACHE")) {
            tune_cache_ = p;
            int n = 0;
            (void)nkr_b200_tune_load(ctx_, p, &n);
        }
    }
    ~B200Backend() override
    {
        nkr_b200_key_free(key_);
        nkr_b200_close(ctx_);
    }

    const char *name() const override { return nkr_b200_backend_name(); }

    // Setup on the GPU with libff's random toxic waste; the verification key's
    // pairing e(alpha, beta) is formed here with libff (backend.cpp:147-153).
    void setup(const Circuit &circuit, ProvingKey &pk, VerificationKey &vk) override
    {
        const Scalar toxic[5] = {Scalar::random_element(), Scalar::random_element(),
                                 Scalar::random_element(), Scalar::random_element(),
                                 Scalar::random_element()};
        const std::size_t cols = circuit.a.num_cols, rows = circuit.constraints();
        pk.a_query.resize(cols);
        pk.b_g1_query.resize(cols);
        pk.b_g2_query.resize(cols);
        pk.l_query.resize(cols);
        pk.h_query.resize(rows);
        vk.ic.resize(circuit.public_inputs + 1);
        G2 gamma_g2;
        nkr_b200_setup_out out{};
        out.a_query = pk.a_query.data();
        out.b_g1_query = pk.b_g1_query.data();
        out.b_g2_query = pk.b_g2_query.data();
        out.l_query = pk.l_query.data();
        out.h_query = pk.h_query.data();
        out.ic = vk.ic.data();
        out.alpha_g1 = &pk.alpha_g1;
        out.beta_g1 = &pk.beta_g1;
        out.delta_g1 = &pk.delta_g1;
        out.beta_g2 = &pk.beta_g2;
        out.delta_g2 = &pk.delta_g2;
        out.gamma_g2 = &gamma_g2;
        const nkr_b200_circuit cv = circuit_view(circuit);
        check(nkr_b200_setup(ctx_, &cv, toxic, &out), "setup");
        vk.alpha_g1_beta_g2 = Curve::reduced_pairing(pk.alpha_g1, pk.beta_g2);
        vk.gamma_g2 = gamma_g2;
        vk.delta_g2 = pk.delta_g2;
    }

    // Backend::prepare: circuit and proving key become resident in HBM.
    void prepare(const Circuit &circuit, const ProvingKey &pk) override
    {
        nkr_b200_key_free(key_);
        key_ = nullptr;
        const nkr_b200_circuit cv = circuit_view(circuit);
        const nkr_b200_proving_key kv = key_view(pk);
        check(nkr_b200_prepare(ctx_, &cv, &kv, &key_), "prepare");
        prepared_for_ = &circuit;
        if (!tune_cache_.empty()) (void)nkr_b200_tune_save(ctx_, tune_cache_.c_str());
    }

    // Backend::prove: raw proof points, affine-normalised libff Jacobian layout.
    void prove(const Circuit &circuit, const ProvingKey &pk, const std::vector<Scalar> &witness,
               RawProof &proof) override
    {
        if (!key_ || prepared_for_ != &circuit) prepare(circuit, pk);
        nkr_b200_raw_proof raw;
        check(nkr_b200_prove(key_, witness.data(), witness.size(), &raw), "prove");
        std::memcpy(static_cast<void *>(&proof.ar), raw.ar, 96);
        std::memcpy(static_cast<void *>(&proof.bs1), raw.bs1, 96);
        std::memcpy(static_cast<void *>(&proof.zk), raw.zk, 96);
        std::memcpy(static_cast<void *>(&proof.qz), raw.qz, 96);
        std::memcpy(static_cast<void *>(&proof.bs2), raw.bs2, 192);
    }

private:
    nkr_b200_ctx *ctx_ = nullptr;
    nkr_b200_key *key_ = nullptr;
    const Circuit *prepared_for_ = nullptr;
    std::string tune_cache_;
};

} // namespace

std::unique_ptr<Backend> make_b200_backend() { return std::make_unique<B200Backend>(); }

} // namespace nkr::groth16
