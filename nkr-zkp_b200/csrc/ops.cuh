// Elementwise field / group operations and the Montgomery-product
// microbenchmark (device side of nkr_b200_field_op / _group_op / _bench_mul).
#pragma once

#include <cstdint>
#include <vector>

#include "common.cuh"

namespace nkr {

int field_op_device(int field, int op, const void *a, const void *b, void *out, uint64_t n,
                    cudaStream_t st);
int group_op_device(int group, int op, const void *a, const void *b, void *out, uint64_t n,
                    cudaStream_t st);
int bench_mul_device(int field, int sm_count, double *muls_per_s, double *ms, cudaStream_t st);

} // namespace nkr
