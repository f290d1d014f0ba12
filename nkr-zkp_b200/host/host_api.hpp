// Host-side objects behind the generator entry points of the C ABI.
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "fr_host.hpp"

namespace nkr::host {

// A generated R1CS (reference CSR layout, padded) with its satisfying witness.
struct R1cs {
    uint64_t rows = 0, cols = 0, public_inputs = 0;
    uint64_t constraints = 0, variables = 0; // before padding
    std::vector<uint32_t> row_ptr[3], col_idx[3];
    std::vector<Fr> values[3];
    std::vector<Fr> witness;
};

std::unique_ptr<R1cs> generate(const std::string &kind, uint64_t param, int density, uint64_t seed);
Fr poseidon(const Fr &l, const Fr &r);
void poseidon_parameters(Fr rc[195], Fr mds[9]);

} // namespace nkr::host
