// extern "C" entry points of the host-side generators (see include/nkr_b200.h).
#include <cstring>
#include <exception>

#include "../../include/nkr_b200.h"
#include "host_api.hpp"

namespace nkr {
void set_error(const char *fmt, ...);
}

struct nkr_b200_r1cs {
    std::unique_ptr<nkr::host::R1cs> r;
};

extern "C" {

int nkr_b200_r1cs_generate(const char *kind, uint64_t param, int density, uint64_t seed,
                           nkr_b200_r1cs **out)
{
    if (!kind || !out) {
        nkr::set_error("null argument");
        return NKR_B200_EINVAL;
    }
    try {
        auto *h = new nkr_b200_r1cs;
        h->r = nkr::host::generate(kind, param, density, seed);
        *out = h;
        return NKR_B200_OK;
    } catch (const std::exception &e) {
        nkr::set_error("generate %s(%llu): %s", kind, (unsigned long long)param, e.what());
        return NKR_B200_EINVAL;
    }
}

int nkr_b200_r1cs_info(const nkr_b200_r1cs *h, uint64_t *sizes)
{
    if (!h || !sizes) {
        nkr::set_error("null argument");
        return NKR_B200_EINVAL;
    }
    const auto &r = *h->r;
    const uint64_t v[8] = {r.rows, r.cols, r.public_inputs, r.constraints, r.variables,
                           r.col_idx[0].size(), r.col_idx[1].size(), r.col_idx[2].size()};
    std::memcpy(sizes, v, sizeof(v));
    return NKR_B200_OK;
}

int nkr_b200_r1cs_view(const nkr_b200_r1cs *h, nkr_b200_circuit *c, const void **witness)
{
    if (!h || !c) {
        nkr::set_error("null argument");
        return NKR_B200_EINVAL;
    }
    const auto &r = *h->r;
    c->rows = r.rows;
    c->cols = r.cols;
    c->public_inputs = r.public_inputs;
    for (int k = 0; k < 3; ++k) {
        c->row_ptr[k] = r.row_ptr[k].data();
        c->col_idx[k] = r.col_idx[k].data();
        c->values[k] = r.values[k].data();
    }
    if (witness) *witness = r.witness.data();
    return NKR_B200_OK;
}

void nkr_b200_r1cs_free(nkr_b200_r1cs *h) { delete h; }

int nkr_b200_poseidon_hash2(const void *left, const void *right, void *out)
{
    if (!left || !right || !out) {
        nkr::set_error("null argument");
        return NKR_B200_EINVAL;
    }
    nkr::host::Fr l, r;
    std::memcpy(l.v, left, 32);
    std::memcpy(r.v, right, 32);
    const nkr::host::Fr d = nkr::host::poseidon(l, r);
    std::memcpy(out, d.v, 32);
    return NKR_B200_OK;
}

int nkr_b200_poseidon_parameters(void *round_constants, void *mds)
{
    if (!round_constants || !mds) {
        nkr::set_error("null argument");
        return NKR_B200_EINVAL;
    }
    nkr::host::Fr rc[195], m[9];
    nkr::host::poseidon_parameters(rc, m);
    std::memcpy(round_constants, rc, sizeof(rc));
    std::memcpy(mds, m, sizeof(m));
    return NKR_B200_OK;
}

} // extern "C"
