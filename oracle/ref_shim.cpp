// Thin C entry points over the reference's own CPU Groth16 path, compiled in
// place from the reference sources by oracle/Makefile into oracle/_ref/.
//
// Test infrastructure only: the parity tests and the CPU-baseline leg of the
// benchmark use it as the checker / the timed reference implementation.  Every
// computation below is done by the reference's code (libff, libfqfft, the
// groth16 CPU backend, protocol.cpp, io.cpp, the Poseidon gadget); this file
// only converts raw byte buffers to and from the reference's types.
//
// Byte layouts are the reference's in-memory layouts (what its BinaryArchive
// writes): Fr/Fq = 4 x u64 little-endian Montgomery limbs; G1 = {X,Y,Z} Fq
// Jacobian (96 B); G2 = {X,Y,Z} Fq2 with Fq2 = {c0,c1} (192 B).

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <exception>
#include <map>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "groth16/backend.hpp"
#include "groth16/io.hpp"
#include "groth16/protocol.hpp"
#include "groth16/types.hpp"
#include "libff/algebra/scalar_multiplication/multiexp.hpp"
#include "libfqfft/evaluation_domain/get_evaluation_domain.hpp"
#include "r1cs/poseidon.hpp"
#include "r1cs/r1cs.hpp"
#include "r1cs/sql_aggregate.hpp"

using namespace nkr::groth16;

static_assert(sizeof(Scalar) == 32, "Fr layout");
static_assert(sizeof(G1) == 96, "G1 layout");
static_assert(sizeof(G2) == 192, "G2 layout");

namespace {

thread_local std::string g_error;

bool g_inited = false;
void init()
{
    if (!g_inited) {
        libff::inhibit_profiling_info = true;
        libff::inhibit_profiling_counters = true;
        Curve::init_public_params();
        g_inited = true;
    }
}

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

// A reference-layout circuit handed over as one struct of raw pointers.
struct RawCircuit {
    uint64_t rows, cols, public_inputs;
    const uint32_t *row_ptr[3];
    const uint32_t *col_idx[3];
    const void *values[3];
};

Circuit circuit_from_raw(const RawCircuit &rc)
{
    Circuit c;
    c.public_inputs = rc.public_inputs;
    c.a = csr_from_raw(rc.rows, rc.cols, rc.row_ptr[0], rc.col_idx[0], rc.values[0]);
    c.b = csr_from_raw(rc.rows, rc.cols, rc.row_ptr[1], rc.col_idx[1], rc.values[1]);
    c.c = csr_from_raw(rc.rows, rc.cols, rc.row_ptr[2], rc.col_idx[2], rc.values[2]);
    return c;
}

template <typename Grp>
void write_affine(Grp p, void *out)
{
    p.to_affine_coordinates();
    std::memcpy(out, &p, sizeof(Grp));
}

} // namespace

// Runs one entry point's body; exceptions become status 1 plus a message.
#define REF_TRY(...)                      \
    try {                                 \
        init();                           \
        __VA_ARGS__;                      \
        return 0;                         \
    } catch (const std::exception &e) {   \
        g_error = e.what();               \
        return 1;                         \
    } catch (...) {                       \
        g_error = "unknown exception";    \
        return 1;                         \
    }

extern "C" {

const char *ref_last_error(void) { return g_error.c_str(); }

int ref_init(void) { REF_TRY((void)0) }

// Poseidon hash2 over Fr (Montgomery limbs in/out): crypto/poseidon.hpp.
int ref_poseidon_hash2(const void *left, const void *right, void *out)
{
    REF_TRY({
        Scalar l, r;
        std::memcpy((void *)&l, left, 32);
        std::memcpy((void *)&r, right, 32);
        const Scalar d = nkr::poseidon::hash2<Scalar>(l, r);
        std::memcpy(out, &d, 32);
    })
}

// Scalar field constants as the reference's libff defines them (Montgomery limbs):
// which = 0 -> Fr::one, 1 -> multiplicative_generator, 2 -> root_of_unity (2^s-th)
int ref_fr_constant(int which, void *out)
{
    REF_TRY({
        Scalar v = which == 0 ? Scalar::one()
                 : which == 1 ? Scalar::multiplicative_generator
                              : Scalar::root_of_unity;
        std::memcpy(out, &v, 32);
    })
}

// libfqfft radix-2 domain transforms, in place over n Fr values.
// op: 0 FFT, 1 iFFT, 2 cosetFFT(g), 3 icosetFFT(g), 4 divide_by_Z_on_coset
int ref_domain_op(int op, void *data, uint64_t n)
{
    REF_TRY({
        auto v = from_raw<Scalar>(data, n);
        auto domain = libfqfft::get_evaluation_domain<Scalar>(n);
        if (!domain || domain->m != n) throw std::invalid_argument("unsupported domain size");
        const Scalar g = Scalar::multiplicative_generator;
        switch (op) {
        case 0: domain->FFT(v); break;
        case 1: domain->iFFT(v); break;
        case 2: domain->cosetFFT(v, g); break;
        case 3: domain->icosetFFT(v, g); break;
        case 4: domain->divide_by_Z_on_coset(v); break;
        default: throw std::invalid_argument("bad op");
        }
        std::memcpy(data, v.data(), n * 32);
    })
}

// libff BDLO12 multi-exponentiation (the CPU backend's multiexp), result affine.
int ref_multiexp_g1(const void *bases_jac, const void *scalars, uint64_t n, void *out_affine)
{
    REF_TRY({
        auto b = from_raw<G1>(bases_jac, n);
        auto s = from_raw<Scalar>(scalars, n);
        G1 r = n ? libff::multi_exp<G1, Scalar, libff::multi_exp_method::multi_exp_method_BDLO12>(
                       b.begin(), b.end(), s.begin(), s.end(), 1)
                 : G1::zero();
        write_affine(r, out_affine);
    })
}

int ref_multiexp_g2(const void *bases_jac, const void *scalars, uint64_t n, void *out_affine)
{
    REF_TRY({
        auto b = from_raw<G2>(bases_jac, n);
        auto s = from_raw<Scalar>(scalars, n);
        G2 r = n ? libff::multi_exp<G2, Scalar, libff::multi_exp_method::multi_exp_method_BDLO12>(
                       b.begin(), b.end(), s.begin(), s.end(), 1)
                 : G2::zero();
        write_affine(r, out_affine);
    })
}

// Generators and scalar multiples, for fixtures: out = k * G (affine)
int ref_g1_mul_gen(const void *k, void *out_affine)
{
    REF_TRY({
        Scalar s;
        std::memcpy((void *)&s, k, 32);
        write_affine(s * G1::one(), out_affine);
    })
}

int ref_g2_mul_gen(const void *k, void *out_affine)
{
    REF_TRY({
        Scalar s;
        std::memcpy((void *)&s, k, 32);
        write_affine(s * G2::one(), out_affine);
    })
}

// libff's reduced pairing e(P, Q) (Curve::reduced_pairing, as protocol.cpp:105-107
// uses it): P, Q libff Jacobian (96 / 192 B), out the GT element (alt_bn128_Fq12,
// 384 B, Montgomery limbs).
int ref_reduced_pairing(const void *p_jac, const void *q_jac, void *out)
{
    REF_TRY({
        G1 a;
        G2 b;
        std::memcpy((void *)&a, p_jac, 96);
        std::memcpy((void *)&b, q_jac, 192);
        const GT e = Curve::reduced_pairing(a, b);
        std::memcpy(out, (const void *)&e, 384);
    })
}

int ref_check_witness(const RawCircuit *rc, const void *witness, uint64_t n, int *ok)
{
    REF_TRY({
        Circuit c = circuit_from_raw(*rc);
        auto w = from_raw<Scalar>(witness, n);
        *ok = check_witness(c, w) ? 1 : 0;
    })
}

int ref_validate_circuit(const RawCircuit *rc, int *ok)
{
    REF_TRY({
        Circuit c = circuit_from_raw(*rc);
        std::string err;
        *ok = validate_circuit(c, err) ? 1 : 0;
        if (!*ok) g_error = err;
    })
}

// The reference CPU backend's prove (backends/cpu/src/backend.cpp:156-201):
// raw proof points {ar, bs1, zk, qz} (G1 affine, 64 B each) and bs2 (G2 affine, 128 B).
// The proving key is read from a reference artifact file.
int ref_cpu_prove(const RawCircuit *rc, const char *pk_path, const void *witness,
                  void *g1_out4, void *g2_out)
{
    REF_TRY({
        Circuit c = circuit_from_raw(*rc);
        ProvingKey pk = read_proving_key(pk_path);
        auto w = from_raw<Scalar>(witness, rc->cols);
        auto backend = make_cpu_backend();
        RawProof raw;
        backend->prove(c, pk, w, raw);
        char *o = static_cast<char *>(g1_out4);
        G1 pts[4] = {raw.ar, raw.bs1, raw.zk, raw.qz};
        for (int i = 0; i < 4; ++i) {
            pts[i].to_affine_coordinates();
            std::memcpy(o + 64 * i, &pts[i], 64);
        }
        G2 b = raw.bs2;
        b.to_affine_coordinates();
        std::memcpy(g2_out, &b, 128);
    })
}

// Same, but the proving key stays loaded across calls (benchmark use).
struct RefProver {
    Circuit circuit;
    ProvingKey pk;
};

void *ref_prover_open(const RawCircuit *rc, const char *pk_path)
{
    try {
        init();
        auto *p = new RefProver;
        p->circuit = circuit_from_raw(*rc);
        p->pk = read_proving_key(pk_path);
        return p;
    } catch (const std::exception &e) {
        g_error = e.what();
        return nullptr;
    }
}

int ref_prover_prove(void *h, const void *witness, void *g1_out4, void *g2_out)
{
    REF_TRY({
        auto *p = static_cast<RefProver *>(h);
        auto w = from_raw<Scalar>(witness, p->circuit.a.num_cols);
        auto backend = make_cpu_backend();
        RawProof raw;
        backend->prove(p->circuit, p->pk, w, raw);
        char *o = static_cast<char *>(g1_out4);
        G1 pts[4] = {raw.ar, raw.bs1, raw.zk, raw.qz};
        for (int i = 0; i < 4; ++i) {
            pts[i].to_affine_coordinates();
            std::memcpy(o + 64 * i, &pts[i], 64);
        }
        G2 b = raw.bs2;
        b.to_affine_coordinates();
        std::memcpy(g2_out, &b, 128);
    })
}

void ref_prover_close(void *h) { delete static_cast<RefProver *>(h); }

// What groth16-prove times as groth16.prove.total (app/prove.cpp:70-88): the CPU
// backend's prove, then the reference's blind_proof (protocol.cpp:85-94) with
// its own unseeded r, s.  Writes the proof affine-normalised in libff's Jacobian
// layout (Z = 1): a (96 B), b (192 B), c (96 B).
int ref_prover_prove_blind(void *h, const void *witness, void *a_out, void *b_out, void *c_out)
{
    REF_TRY({
        auto *p = static_cast<RefProver *>(h);
        auto w = from_raw<Scalar>(witness, p->circuit.a.num_cols);
        auto backend = make_cpu_backend();
        RawProof raw;
        backend->prove(p->circuit, p->pk, w, raw);
        const Proof proof = blind_proof(p->pk, raw);
        write_affine(proof.a, a_out);
        write_affine(proof.b, b_out);
        write_affine(proof.c, c_out);
    })
}

// The SpMV vectors and the quotient H of the CPU backend's prove
// (backends/cpu/src/backend.cpp:163-179) on the reference's own libff / libfqfft
// types.  backend.cpp keeps its `multiply` (lines 25-35) file-local, so the row
// loop below repeats it: per row, value += values[j] * z[col_idx[j]] in CSR order.
int ref_quotient_vectors(const RawCircuit *rc, const void *witness, void *az_out, void *bz_out,
                         void *cz_out, void *h_out)
{
    REF_TRY({
        Circuit c = circuit_from_raw(*rc);
        auto z = from_raw<Scalar>(witness, rc->cols);
        auto multiply = [&](const CsrMatrix<Scalar> &m) {
            std::vector<Scalar> out(m.num_rows, Scalar::zero());
            for (std::size_t row = 0; row < m.num_rows; ++row) {
                Scalar value = Scalar::zero();
                for (std::size_t j = m.row_ptr[row]; j < m.row_ptr[row + 1]; ++j)
                    value += m.values[j] * z[m.col_idx[j]];
                out[row] = value;
            }
            return out;
        };
        const std::size_t rows = c.constraints();
        auto domain = libfqfft::get_evaluation_domain<Scalar>(rows);
        if (!domain || domain->m != rows) throw std::invalid_argument("unsupported R1CS domain size");
        std::vector<Scalar> az = multiply(c.a), bz = multiply(c.b), cz = multiply(c.c);
        std::memcpy(az_out, az.data(), rows * 32);
        std::memcpy(bz_out, bz.data(), rows * 32);
        std::memcpy(cz_out, cz.data(), rows * 32);
        domain->iFFT(az);
        domain->iFFT(bz);
        domain->iFFT(cz);
        const Scalar coset = Scalar::multiplicative_generator;
        domain->cosetFFT(az, coset);
        domain->cosetFFT(bz, coset);
        domain->cosetFFT(cz, coset);
        for (std::size_t i = 0; i < rows; ++i) az[i] = az[i] * bz[i] - cz[i];
        domain->divide_by_Z_on_coset(az);
        domain->icosetFFT(az, coset);
        std::memcpy(h_out, az.data(), rows * 32);
    })
}

// The Poseidon preimages (left, right per hash; 2 * count Fr, Montgomery limbs)
// that this repository's seeded circuit generator draws for
// generate("poseidon", count, density, seed), so that the reference's own
// builders (ref_poseidon_circuit_n) can build the same circuit without it.  The
// reference's generator draws the same distribution from unseeded engines
// (common/include/density.hpp:62,80-98): ceil(N/10) nonzero at sparse density,
// N - N/2 at hybrid, all at full.  One std::mt19937_64(seed) drives every draw:
// a mask with the zeros at its end, shuffled by Fisher-Yates (j = rng() % i for
// i = N down to 2), then, slot by slot, a nonzero uniform Fr for each set bit
// (four 64-bit words, the top one cut to 62 bits, values >= r and zero redrawn).
int ref_seeded_pairs(uint64_t count, int density, uint64_t seed, void *lr_out)
{
    REF_TRY({
        const uint64_t n = 2 * count;
        uint64_t nonzero;
        switch (density) {
        case 0: nonzero = n; break;
        case 1: nonzero = n - n / 2; break;
        case 2: nonzero = n / 10 + (n % 10 != 0); break;
        default: throw std::invalid_argument("density must be 0, 1 or 2");
        }
        std::mt19937_64 rng(seed);
        std::vector<uint8_t> mask(n, 1);
        std::fill(mask.end() - (n - nonzero), mask.end(), 0);
        for (uint64_t i = n; i > 1; --i) std::swap(mask[i - 1], mask[rng() % i]);
        static const uint64_t kR[4] = {0x43e1f593f0000001ull, 0x2833e84879b97091ull,
                                       0xb85045b68181585dull, 0x30644e72e131a029ull};
        auto below_r = [](const uint64_t v[4]) {
            for (int i = 3; i >= 0; --i)
                if (v[i] != kR[i]) return v[i] < kR[i];
            return false;
        };
        uint64_t *out = static_cast<uint64_t *>(lr_out);
        for (uint64_t i = 0; i < n; ++i) {
            uint64_t *v = out + 4 * i;
            if (!mask[i]) {
                v[0] = v[1] = v[2] = v[3] = 0;
                continue;
            }
            do {
                do {
                    for (int k = 0; k < 4; ++k) v[k] = rng();
                    v[3] &= (uint64_t(1) << 62) - 1;
                } while (!below_r(v));
            } while (!(v[0] | v[1] | v[2] | v[3]));
        }
    })
}

// The reference CPU setup (backend.cpp:41-154); unseeded toxic waste as in the
// reference.  Writes the reference's .pk.bin / .vk.bin artifacts.
int ref_cpu_setup(const RawCircuit *rc, const char *pk_path, const char *vk_path)
{
    REF_TRY({
        Circuit c = circuit_from_raw(*rc);
        ProvingKey pk;
        VerificationKey vk;
        make_cpu_backend()->setup(c, pk, vk);
        write_proving_key(pk_path, pk);
        write_verification_key(vk_path, vk);
    })
}

// The reference verifier (protocol.cpp:96-108) on a proof artifact file.
int ref_verify(const char *vk_path, const void *public_inputs, uint64_t n_public,
               const char *proof_path, int *ok)
{
    REF_TRY({
        VerificationKey vk = read_verification_key(vk_path);
        Proof proof = read_proof(proof_path);
        auto x = from_raw<Scalar>(public_inputs, n_public);
        *ok = verify(vk, x, proof) ? 1 : 0;
    })
}

// Reads reference artifacts back through the reference's io.cpp, to check files
// written by other code.  Returns sizes through the out-params.
int ref_read_circuit_shape(const char *path, uint64_t *rows, uint64_t *cols, uint64_t *pub,
                           uint64_t nnz[3])
{
    REF_TRY({
        Circuit c = read_circuit(path);
        *rows = c.a.num_rows;
        *cols = c.a.num_cols;
        *pub = c.public_inputs;
        nnz[0] = c.a.nnz();
        nnz[1] = c.b.nnz();
        nnz[2] = c.c.nnz();
    })
}

// Builds the reference's Poseidon gadget for one hash of (left, right) with the
// reference's R1CSManager and returns the padded CSR sizes and witness, to pin
// the circuit generator.  Buffers are sized by the caller from a first call with
// null outputs (sizes only).
int ref_poseidon_circuit(const void *left, const void *right, uint64_t *rows, uint64_t *cols,
                         uint64_t nnz[3], uint32_t *row_ptr3, uint32_t *col_idx3,
                         void *values3, void *witness)
{
    REF_TRY({
        using namespace LightZK;
        Scalar l, r;
        std::memcpy((void *)&l, left, 32);
        std::memcpy((void *)&r, right, 32);
        R1CSManager<Scalar> mgr;
        std::map<std::size_t, Scalar> assignment;
        Variable<Scalar> digest(VariableType::Public, mgr);
        Variable<Scalar> lv(VariableType::Private, mgr);
        Variable<Scalar> rv(VariableType::Private, mgr);
        assignment[digest.get_id()] = Poseidon::hash2(l, r);
        assignment[lv.get_id()] = l;
        assignment[rv.get_id()] = r;
        Poseidon::add_hash2_constraints(mgr, assignment, lv, l, rv, r, digest);
        Circuit c;
        mgr.gen_spmat(c.a, c.b, c.c, true);
        *rows = c.a.num_rows;
        *cols = c.a.num_cols;
        nnz[0] = c.a.nnz();
        nnz[1] = c.b.nnz();
        nnz[2] = c.c.nnz();
        if (row_ptr3) {
            const CsrMatrix<Scalar> *m[3] = {&c.a, &c.b, &c.c};
            uint32_t *rp = row_ptr3;
            uint32_t *ci = col_idx3;
            char *vv = static_cast<char *>(values3);
            for (int k = 0; k < 3; ++k) {
                std::memcpy(rp, m[k]->row_ptr.data(), (c.a.num_rows + 1) * 4);
                rp += c.a.num_rows + 1;
                std::memcpy(ci, m[k]->col_idx.data(), m[k]->nnz() * 4);
                ci += m[k]->nnz();
                std::memcpy(vv, m[k]->values.data(), m[k]->nnz() * 32);
                vv += m[k]->nnz() * 32;
            }
            std::vector<Scalar> z(c.a.num_cols, Scalar::zero());
            z[0] = Scalar::one();
            for (const auto &[id, val] : assignment) z[mgr.dense_index(id)] = val;
            std::memcpy(witness, z.data(), z.size() * 32);
        }
    })
}

} // extern "C"

// Shared tail of the circuit builders below: padded CSR + witness out of a
// reference R1CSManager, exactly as groth16-gen's finalize_circuit (gen.cpp:30-40).
static void emit_circuit(LightZK::R1CSManager<Scalar> &mgr, std::map<std::size_t, Scalar> &assignment,
                         uint64_t *rows, uint64_t *cols, uint64_t *pub, uint64_t nnz[3],
                         uint32_t *row_ptr3, uint32_t *col_idx3, void *values3, void *witness)
{
    Circuit c;
    mgr.gen_spmat(c.a, c.b, c.c, true);
    *rows = c.a.num_rows;
    *cols = c.a.num_cols;
    *pub = mgr.num_public();
    nnz[0] = c.a.nnz();
    nnz[1] = c.b.nnz();
    nnz[2] = c.c.nnz();
    if (!row_ptr3) return;
    const CsrMatrix<Scalar> *m[3] = {&c.a, &c.b, &c.c};
    uint32_t *rp = row_ptr3;
    uint32_t *ci = col_idx3;
    char *vv = static_cast<char *>(values3);
    for (int k = 0; k < 3; ++k) {
        std::memcpy(rp, m[k]->row_ptr.data(), (c.a.num_rows + 1) * 4);
        rp += c.a.num_rows + 1;
        std::memcpy(ci, m[k]->col_idx.data(), m[k]->nnz() * 4);
        ci += m[k]->nnz();
        std::memcpy(vv, m[k]->values.data(), m[k]->nnz() * 32);
        vv += m[k]->nnz() * 32;
    }
    std::vector<Scalar> z(c.a.num_cols, Scalar::zero());
    z[0] = Scalar::one();
    for (const auto &[id, val] : assignment) z[mgr.dense_index(id)] = val;
    std::memcpy(witness, z.data(), z.size() * 32);
}

extern "C" {

// The matmul circuit of gen.cpp:42-86 built with the reference's R1CSManager for
// given A, B entries (s*s Fr each); call with null outputs first for the sizes.
int ref_matmul_circuit(uint64_t s, const void *av_raw, const void *bv_raw, uint64_t *rows,
                       uint64_t *cols, uint64_t *pub, uint64_t nnz[3], uint32_t *row_ptr3,
                       uint32_t *col_idx3, void *values3, void *witness)
{
    REF_TRY({
        using namespace LightZK;
        R1CSManager<Scalar> mgr;
        std::map<std::size_t, Scalar> assignment;
        std::vector<Variable<Scalar>> A, B, C, P;
        for (uint64_t i = 0; i < s * s; i++) A.push_back(Variable<Scalar>(VariableType::Public, mgr));
        for (uint64_t i = 0; i < s * s; i++) B.push_back(Variable<Scalar>(VariableType::Public, mgr));
        for (uint64_t i = 0; i < s * s; i++) C.push_back(Variable<Scalar>(VariableType::Public, mgr));
        for (uint64_t i = 0; i < s * s * s; i++) P.push_back(Variable<Scalar>(VariableType::Private, mgr));
        for (uint64_t i = 0; i < s; i++)
            for (uint64_t j = 0; j < s; j++)
                for (uint64_t l = 0; l < s; l++)
                    mgr.add_constraint(P[i * s * s + j * s + l], A[i * s + l], B[l * s + j]);
        for (uint64_t i = 0; i < s; i++)
            for (uint64_t j = 0; j < s; j++) {
                LinearCombination<Scalar> sum;
                for (uint64_t l = 0; l < s; l++) sum += P[i * s * s + j * s + l];
                mgr.add_constraint(C[i * s + j], sum);
            }
        auto av = from_raw<Scalar>(av_raw, s * s), bv = from_raw<Scalar>(bv_raw, s * s);
        for (uint64_t i = 0; i < s; i++)
            for (uint64_t j = 0; j < s; j++) {
                Scalar sum = Scalar::zero();
                for (uint64_t l = 0; l < s; l++) {
                    const Scalar p = av[i * s + l] * bv[l * s + j];
                    assignment[P[i * s * s + j * s + l].get_id()] = p;
                    sum += p;
                }
                assignment[C[i * s + j].get_id()] = sum;
            }
        for (uint64_t i = 0; i < s * s; i++) {
            assignment[A[i].get_id()] = av[i];
            assignment[B[i].get_id()] = bv[i];
        }
        emit_circuit(mgr, assignment, rows, cols, pub, nnz, row_ptr3, col_idx3, values3, witness);
    })
}

// count Poseidon hashes of given (left, right) pairs as gen.cpp:139-162 builds them.
int ref_poseidon_circuit_n(uint64_t count, const void *lr_raw, uint64_t *rows, uint64_t *cols,
                           uint64_t *pub, uint64_t nnz[3], uint32_t *row_ptr3, uint32_t *col_idx3,
                           void *values3, void *witness)
{
    REF_TRY({
        using namespace LightZK;
        R1CSManager<Scalar> mgr;
        std::map<std::size_t, Scalar> assignment;
        auto lr = from_raw<Scalar>(lr_raw, 2 * count);
        for (uint64_t i = 0; i < count; ++i) {
            const Scalar lv = lr[2 * i], rv = lr[2 * i + 1];
            Variable<Scalar> digest(VariableType::Public, mgr);
            Variable<Scalar> left(VariableType::Private, mgr);
            Variable<Scalar> right(VariableType::Private, mgr);
            assignment[digest.get_id()] = Poseidon::hash2(lv, rv);
            assignment[left.get_id()] = lv;
            assignment[right.get_id()] = rv;
            Poseidon::add_hash2_constraints(mgr, assignment, left, lv, right, rv, digest);
        }
        emit_circuit(mgr, assignment, rows, cols, pub, nnz, row_ptr3, col_idx3, values3, witness);
    })
}

// SQL aggregate over given rows (categories and amounts as Fr) as gen.cpp:164-197.
int ref_sql_circuit(uint64_t n, const void *cat_raw, const void *amt_raw, uint64_t *rows,
                    uint64_t *cols, uint64_t *pub, uint64_t nnz[3], uint32_t *row_ptr3,
                    uint32_t *col_idx3, void *values3, void *witness)
{
    REF_TRY({
        using namespace LightZK;
        R1CSManager<Scalar> mgr;
        std::map<std::size_t, Scalar> assignment;
        auto cats = from_raw<Scalar>(cat_raw, n), amts = from_raw<Scalar>(amt_raw, n);
        std::vector<SqlAggregate::Row<Scalar>> rws;
        for (uint64_t i = 0; i < n; ++i) rws.push_back({cats[i], amts[i]});
        const Scalar target_value = rws.front().category;
        const auto result = SqlAggregate::evaluate(rws, target_value);
        Variable<Scalar> table_root(VariableType::Public, mgr);
        Variable<Scalar> target_category(VariableType::Public, mgr);
        Variable<Scalar> expected_count(VariableType::Public, mgr);
        Variable<Scalar> expected_sum(VariableType::Public, mgr);
        assignment[table_root.get_id()] = result.table_root;
        assignment[target_category.get_id()] = target_value;
        assignment[expected_count.get_id()] = result.count;
        assignment[expected_sum.get_id()] = result.sum;
        SqlAggregate::add_query_constraints(mgr, assignment, rws, table_root, target_category,
                                            target_value, expected_count, expected_sum);
        emit_circuit(mgr, assignment, rows, cols, pub, nnz, row_ptr3, col_idx3, values3, witness);
    })
}

} // extern "C"

extern "C" {

// Writes a reference verification key artifact (io.cpp:79-84) for keys made
// elsewhere: the reference computes e(alpha_g1, beta_g2) with its own pairing.
// Inputs in libff layout; ic holds n_ic G1 points.
int ref_write_vk(const void *alpha_g1, const void *beta_g2, const void *gamma_g2,
                 const void *delta_g2, const void *ic, uint64_t n_ic, const char *path)
{
    REF_TRY({
        G1 a;
        G2 b, g, d;
        std::memcpy((void *)&a, alpha_g1, 96);
        std::memcpy((void *)&b, beta_g2, 192);
        std::memcpy((void *)&g, gamma_g2, 192);
        std::memcpy((void *)&d, delta_g2, 192);
        VerificationKey vk;
        vk.alpha_g1_beta_g2 = Curve::reduced_pairing(a, b);
        vk.gamma_g2 = g;
        vk.delta_g2 = d;
        vk.ic = from_raw<G1>(ic, n_ic);
        write_verification_key(path, vk);
    })
}

} // extern "C"
