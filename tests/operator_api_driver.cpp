// Drives include/nkr_b200_operators.hpp the way the reference's CUDA backend
// drives its operator contexts in a prove (backends/cuda/src/groth16_backend.cu:
// 242-279): the quotient chain through NTTContext on device polynomials, then
// MSMContext over BucketContext scalars (witness scalars from host memory, the
// quotient's scalars straight from the device polynomial).  Built and run by
// tests/test_gpu_operator_api.py, which compares the outputs with the oracle.
//
//   operator_api_driver <dir>
// reads <dir>/{shape,omega,coset,a,b,c,z,g1,g2,hb}.bin and writes
// <dir>/{h,msm_g1,msm_g2,msm_h}.bin.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iterator>
#include <stdexcept>
#include <string>
#include <vector>

#include "nkr_b200_operators.hpp"

namespace {

struct fr_t {
    uint64_t v[4];
};
struct g1_affine_t {
    uint64_t v[8];
};
struct g2_affine_t {
    uint64_t v[16];
};
struct g1_t {
    uint64_t v[12];
};
struct g2_t {
    uint64_t v[24];
};
struct g1_bucket_t {
    uint64_t v[16];
};
struct g2_bucket_t {
    uint64_t v[32];
};
using Scalar = fr_t; // host and device Fr share the layout, as libff's and fr_t do
using G1 = g1_t;
using G2 = g2_t;

template <typename T>
std::vector<T> load(const std::string &path)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot open " + path);
    std::vector<char> raw((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    std::vector<T> out(raw.size() / sizeof(T));
    std::memcpy(out.data(), raw.data(), out.size() * sizeof(T));
    return out;
}

template <typename T>
void store(const std::string &path, const T *data, size_t n)
{
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char *>(data), n * sizeof(T));
}

using namespace nkr_b200::operators;

} // namespace

int main(int argc, char **argv)
{
    if (argc != 2) {
        std::fprintf(stderr, "usage: %s <dir>\n", argv[0]);
        return 2;
    }
    const std::string d = argv[1];
    try {
        const auto shape = load<uint64_t>(d + "/shape.bin"); // rows (domain), witness length
        const size_t rows = shape.at(0), cols = shape.at(1);
        const Scalar omega = load<Scalar>(d + "/omega.bin").at(0);
        const Scalar coset = load<Scalar>(d + "/coset.bin").at(0);

        // the CudaProveLayout members (groth16_backend.cu:69-96)
        BucketContext<fr_t, Scalar> witness_buckets(cols, 13), quotient_buckets(rows, 13);
        NTTContext<fr_t, Scalar> ntt(rows, omega, coset);
        MSMContext<fr_t, g1_affine_t, g1_t, g1_bucket_t, Scalar, G1> a_msm(cols, 13), h_msm(rows, 13);
        MSMContext<fr_t, g2_affine_t, g2_t, g2_bucket_t, Scalar, G2> b_g2_msm(cols, 13);
        fr_t *polynomials[3];
        for (auto &p : polynomials)
            check_cuda(cudaMalloc(reinterpret_cast<void **>(&p), rows * sizeof(fr_t)), "cudaMalloc");

        // prepare: the key's bases
        a_msm.load_bases(load<G1>(d + "/g1.bin").data());
        b_g2_msm.load_bases(load<G2>(d + "/g2.bin").data());
        h_msm.load_bases(load<G1>(d + "/hb.bin").data());

        // SpMV outputs stand in as the three polynomials (evaluations)
        const char *names[3] = {"/a.bin", "/b.bin", "/c.bin"};
        for (int k = 0; k < 3; ++k) {
            const auto v = load<fr_t>(d + names[k]);
            check_cuda(cudaMemcpy(polynomials[k], v.data(), rows * sizeof(fr_t), cudaMemcpyHostToDevice),
                       "cudaMemcpy");
        }
        // the quotient chain (groth16_backend.cu:257-264)
        ntt.intt(polynomials[0]);
        ntt.intt(polynomials[1]);
        ntt.intt(polynomials[2]);
        ntt.coset_ntt(polynomials[0]);
        ntt.coset_ntt(polynomials[1]);
        ntt.coset_ntt(polynomials[2]);
        ntt.A_times_B_minus_C_divided_by_Z(polynomials[0], polynomials[1], polynomials[2]);
        ntt.coset_intt(polynomials[0]);
        quotient_buckets.load_scalars(polynomials[0]);
        std::vector<fr_t> h(rows);
        check_cuda(cudaMemcpy(h.data(), polynomials[0], rows * sizeof(fr_t), cudaMemcpyDeviceToHost),
                   "cudaMemcpy");
        store(d + "/h.bin", h.data(), rows);

        // witness MSMs, then the quotient MSM (groth16_backend.cu:266-278)
        const auto z = load<Scalar>(d + "/z.bin");
        witness_buckets.load_scalars(z.data());
        witness_buckets.process();
        G1 ar;
        G2 bs2;
        a_msm.msm(witness_buckets, &ar);
        b_g2_msm.msm(witness_buckets, &bs2);
        quotient_buckets.process();
        G1 qz;
        h_msm.msm(quotient_buckets, &qz);
        store(d + "/msm_g1.bin", &ar, 1);
        store(d + "/msm_g2.bin", &bs2, 1);
        store(d + "/msm_h.bin", &qz, 1);

        // a coset that is not the generator is refused
        bool refused = false;
        try {
            NTTContext<fr_t, Scalar> bad(rows, omega, omega);
        } catch (const std::invalid_argument &) {
            refused = true;
        }
        if (!refused) throw std::runtime_error("NTTContext accepted a wrong coset");
        for (auto p : polynomials) cudaFree(p);
    } catch (const std::exception &e) {
        std::fprintf(stderr, "operator_api_driver: %s\n", e.what());
        return 1;
    }
    std::printf("ok\n");
    return 0;
}
