// Seeded R1CS + witness generators for the reference's benchmark circuits.
//
// Restates protocols/groth16/app/gen.cpp (build_matmul :42-86, build_fibonacci
// :88-121, build_poseidon :139-162, build_sql_aggregate :164-197), the R1CS
// manager and linear combinations (common/include/r1cs/r1cs.hpp:25-142), the
// Poseidon gadget (r1cs/poseidon.hpp:33-105), the SQL gadget
// (r1cs/sql_aggregate.hpp:33-165), the SQL evaluation (common/include/
// sql_query.hpp:210-248) and the density sampler (common/include/density.hpp).
// The matrices come out entry for entry as the reference builds them: terms
// ordered by variable id, zero coefficients kept (a default linear combination
// starts with a zero constant term, r1cs.hpp:116), rows and columns padded to
// powers of two (r1cs.hpp:64-98).  The reference draws its randomness from
// unseeded engines (random_device); here one seeded mt19937_64 drives every
// draw so a (circuit, seed) pair is reproducible.
//
// Poseidon parameters (width 3, x^5, 8 full + 57 partial rounds over Fr) are
// produced by the Grain LFSR procedure published with Poseidon (the reference
// ships the resulting constants, common/include/crypto/poseidon_constants.inc).
#include <algorithm>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/nkr_b200.h"
#include "fr_host.hpp"
#include "host_api.hpp"

namespace nkr::host {

namespace {

constexpr uint64_t kHalf = (uint64_t(-1) >> 1) + 1; // first private id (r1cs.hpp:23)

struct Term {
    uint64_t id;
    Fr c;
};

// std::map<size_t, S> semantics on a sorted vector
class LC {
public:
    std::vector<Term> t;
    static LC dflt() { return LC{{Term{0, zero()}}}; }        // LinearCombination()
    static LC constant(const Fr &c) { return LC{{Term{0, c}}}; } // LinearCombination(S)
    static LC var(uint64_t id) { return LC{{Term{id, one()}}}; } // LinearCombination(Variable)
    LC &operator+=(const LC &o)
    {
        std::vector<Term> m;
        m.reserve(t.size() + o.t.size());
        size_t i = 0, j = 0;
        while (i < t.size() || j < o.t.size()) {
            if (j == o.t.size() || (i < t.size() && t[i].id < o.t[j].id))
                m.push_back(t[i++]);
            else if (i == t.size() || o.t[j].id < t[i].id)
                m.push_back(o.t[j++]); // terms[id] += c on a fresh key: 0 + c
            else {
                m.push_back(Term{t[i].id, t[i].c + o.t[j].c});
                ++i;
                ++j;
            }
        }
        t.swap(m);
        return *this;
    }
    LC operator*(const Fr &s) const
    {
        LC r;
        r.t = t;
        for (auto &x : r.t) x.c = x.c * s;
        return r;
    }
};

struct Constraint {
    LC a, b, c;
};

class Builder {
public:
    uint64_t public_count = 1;
    uint64_t private_count = kHalf;
    std::vector<Constraint> cons;
    std::vector<Fr> pub_vals{one()}; // index = id
    std::vector<Fr> priv_vals;       // index = id - kHalf

    uint64_t new_public()
    {
        pub_vals.push_back(zero());
        return public_count++;
    }
    uint64_t new_private()
    {
        priv_vals.push_back(zero());
        return private_count++;
    }
    void assign(uint64_t id, const Fr &v)
    {
        if (id < kHalf)
            pub_vals[id] = v;
        else
            priv_vals[id - kHalf] = v;
    }
    // add_constraint(out, in): in * 1 = out (r1cs.hpp:56-58)
    void add(const LC &out, const LC &in) { cons.push_back({in, LC::constant(one()), out}); }
    // add_constraint(out, in1, in2): in1 * in2 = out (r1cs.hpp:60-62)
    void add(const LC &out, const LC &in1, const LC &in2) { cons.push_back({in1, in2, out}); }

    uint64_t dense(uint64_t id) const { return id < kHalf ? id : id - kHalf + public_count; }
};

// --------------------------------------------------------------------------
// Poseidon parameters: Grain LFSR (80-bit state, taps 0, 13, 23, 38, 51, 62),
// initialised with field = 1 (2 bits), s-box = 0 (4), n = 254 (12), t = 3 (12),
// R_F = 8 (10), R_P = 57 (10) and 30 ones; 160 warm-up clocks; output bits are
// self-shrunk (a 1 keeps the next bit, a 0 drops it).  Round constants take
// n-bit big-endian draws rejected when >= r; the MDS matrix is the Cauchy
// matrix 1 / (x_i + y_j) of 2t further draws reduced mod r.
// --------------------------------------------------------------------------
class Grain {
    uint8_t s[80];
    int pos = 0;
    int clock()
    {
        const int nb = s[pos % 80] ^ s[(pos + 13) % 80] ^ s[(pos + 23) % 80] ^
                       s[(pos + 38) % 80] ^ s[(pos + 51) % 80] ^ s[(pos + 62) % 80];
        s[pos % 80] = uint8_t(nb);
        ++pos;
        return nb;
    }

public:
    Grain()
    {
        int k = 0;
        auto put = [&](uint64_t v, int bits) {
            for (int i = bits - 1; i >= 0; --i) s[k++] = uint8_t((v >> i) & 1);
        };
        put(1, 2);
        put(0, 4);
        put(254, 12);
        put(3, 12);
        put(8, 10);
        put(57, 10);
        for (int i = 0; i < 30; ++i) s[k++] = 1;
        for (int i = 0; i < 160; ++i) clock();
    }
    int bit()
    {
        for (;;) {
            const int keep = clock();
            const int b = clock();
            if (keep) return b;
        }
    }
    void bits254(uint64_t out[4])
    {
        out[0] = out[1] = out[2] = out[3] = 0;
        for (int i = 253; i >= 0; --i)
            if (bit()) out[i / 64] |= uint64_t(1) << (i % 64);
    }
};

struct PoseidonParams {
    Fr rc[195];
    Fr mds[3][3];
};

const PoseidonParams &poseidon_params()
{
    static const PoseidonParams P = [] {
        PoseidonParams p;
        Grain g;
        for (int i = 0; i < 195; ++i) {
            uint64_t c[4];
            do {
                g.bits254(c);
            } while (geq_r(c));
            p.rc[i] = from_canonical(c);
        }
        for (;;) {
            Fr xy[6];
            for (int i = 0; i < 6; ++i) {
                uint64_t c[4];
                g.bits254(c);
                while (geq_r(c)) sub_r(c);
                xy[i] = from_canonical(c);
            }
            bool distinct = true;
            for (int i = 0; i < 6; ++i)
                for (int j = i + 1; j < 6; ++j)
                    if (xy[i] == xy[j]) distinct = false;
            if (!distinct) continue;
            bool ok = true;
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    const Fr d = xy[i] + xy[3 + j];
                    if (d.is_zero()) ok = false;
                    else p.mds[i][j] = inverse(d);
                }
            if (ok) break;
        }
        return p;
    }();
    return P;
}

Fr sbox(const Fr &x)
{
    const Fr sq = x * x;
    return sq * sq * x;
}

// crypto/poseidon.hpp:86-119
Fr poseidon_hash2(const Fr &l, const Fr &r)
{
    const PoseidonParams &P = poseidon_params();
    Fr st[3] = {zero(), l, r};
    int k = 0;
    for (int round = 0; round < 65; ++round) {
        for (auto &w : st) w += P.rc[k++];
        if (round < 4 || round >= 61)
            for (auto &w : st) w = sbox(w);
        else
            st[0] = sbox(st[0]);
        Fr m[3] = {zero(), zero(), zero()};
        for (int row = 0; row < 3; ++row)
            for (int col = 0; col < 3; ++col) m[row] += P.mds[row][col] * st[col];
        std::copy(m, m + 3, st);
    }
    return st[0];
}

// r1cs/poseidon.hpp:33-105: digest = Poseidon([0, left, right])[0]
void poseidon_gadget(Builder &B, uint64_t left, const Fr &lv, uint64_t right, const Fr &rv,
                     uint64_t digest)
{
    const PoseidonParams &P = poseidon_params();
    LC state[3] = {LC::constant(zero()), LC::var(left), LC::var(right)};
    Fr vals[3] = {zero(), lv, rv};
    int k = 0;
    for (int round = 0; round < 65; ++round) {
        LC sboxed[3] = {state[0], state[1], state[2]};
        Fr sv[3] = {vals[0], vals[1], vals[2]};
        for (int i = 0; i < 3; ++i) {
            state[i] += LC::constant(P.rc[k]);
            vals[i] += P.rc[k++];
        }
        const bool full = round < 4 || round >= 61;
        const int sboxes = full ? 3 : 1;
        for (int i = 0; i < sboxes; ++i) {
            const uint64_t sq = B.new_private(), fo = B.new_private(), fi = B.new_private();
            const Fr sqv = vals[i] * vals[i];
            const Fr fov = sqv * sqv;
            const Fr fiv = fov * vals[i];
            B.add(LC::var(sq), state[i], state[i]);
            B.add(LC::var(fo), LC::var(sq), LC::var(sq));
            B.add(LC::var(fi), LC::var(fo), state[i]);
            B.assign(sq, sqv);
            B.assign(fo, fov);
            B.assign(fi, fiv);
            sboxed[i] = LC::var(fi);
            sv[i] = fiv;
        }
        for (int i = sboxes; i < 3; ++i) {
            sboxed[i] = state[i];
            sv[i] = vals[i];
        }
        LC next[3];
        Fr nv[3] = {zero(), zero(), zero()};
        for (int row = 0; row < 3; ++row) {
            LC mixed = LC::dflt();
            for (int col = 0; col < 3; ++col) {
                mixed += sboxed[col] * P.mds[row][col];
                nv[row] += P.mds[row][col] * sv[col];
            }
            const uint64_t o = B.new_private();
            B.add(LC::var(o), mixed);
            B.assign(o, nv[row]);
            next[row] = LC::var(o);
        }
        for (int i = 0; i < 3; ++i) {
            state[i] = next[i];
            vals[i] = nv[i];
        }
    }
    B.add(LC::var(digest), state[0]);
}

// density.hpp:155-163 and the sampler's mask (zeros shuffled into place)
uint64_t density_nonzero(uint64_t count, int density)
{
    switch (density) {
    case 0: return count;
    case 1: return count - count / 2;
    case 2: return count / 10 + (count % 10 != 0);
    }
    throw std::invalid_argument("density must be 0 (full), 1 (hybrid) or 2 (sparse)");
}

struct Sampler {
    std::vector<uint8_t> mask;
    Sampler(uint64_t count, int density, std::mt19937_64 &rng) : mask(count, 1)
    {
        const uint64_t zeros = count - density_nonzero(count, density);
        std::fill(mask.end() - zeros, mask.end(), 0);
        for (uint64_t i = count; i > 1; --i) { // Fisher-Yates
            const uint64_t j = rng() % i;
            std::swap(mask[i - 1], mask[j]);
        }
    }
    template <class Gen>
    Fr sample(uint64_t i, Gen gen) const
    {
        if (!mask.at(i)) return zero();
        Fr v;
        do {
            v = gen();
        } while (v.is_zero());
        return v;
    }
};

void build_matmul(Builder &B, uint64_t s, int density, std::mt19937_64 &rng)
{
    std::vector<uint64_t> A(s * s), Bv(s * s), C(s * s), P(s * s * s);
    for (auto &x : A) x = B.new_public();
    for (auto &x : Bv) x = B.new_public();
    for (auto &x : C) x = B.new_public();
    for (auto &x : P) x = B.new_private();
    for (uint64_t i = 0; i < s; ++i)
        for (uint64_t j = 0; j < s; ++j)
            for (uint64_t l = 0; l < s; ++l)
                B.add(LC::var(P[i * s * s + j * s + l]), LC::var(A[i * s + l]),
                      LC::var(Bv[l * s + j]));
    for (uint64_t i = 0; i < s; ++i)
        for (uint64_t j = 0; j < s; ++j) {
            LC sum = LC::dflt();
            for (uint64_t l = 0; l < s; ++l) sum += LC::var(P[i * s * s + j * s + l]);
            B.add(LC::var(C[i * s + j]), sum);
        }
    const Sampler sa(s * s, density, rng), sb(s * s, density, rng);
    std::vector<Fr> av(s * s), bv(s * s);
    for (uint64_t i = 0; i < s * s; ++i) {
        av[i] = sa.sample(i, [&] { return random_element(rng); });
        bv[i] = sb.sample(i, [&] { return random_element(rng); });
    }
    for (uint64_t i = 0; i < s; ++i)
        for (uint64_t j = 0; j < s; ++j) {
            Fr sum = zero();
            for (uint64_t l = 0; l < s; ++l) {
                const Fr p = av[i * s + l] * bv[l * s + j];
                B.assign(P[i * s * s + j * s + l], p);
                sum += p;
            }
            B.assign(C[i * s + j], sum);
        }
    for (uint64_t i = 0; i < s * s; ++i) {
        B.assign(A[i], av[i]);
        B.assign(Bv[i], bv[i]);
    }
}

void build_fibonacci(Builder &B, uint64_t steps, std::mt19937_64 &rng)
{
    if (steps < 2) throw std::invalid_argument("fibonacci steps must be at least 2");
    const Fr f0 = random_element(rng), f1 = random_element(rng);
    uint64_t prev = B.new_public(), cur = B.new_public();
    const uint64_t expected = B.new_public();
    B.assign(prev, f0);
    B.assign(cur, f1);
    Fr pv = f0, cv = f1;
    for (uint64_t step = 2; step <= steps; ++step) {
        const Fr nv = pv + cv;
        const uint64_t nx = B.new_private();
        LC sum = LC::var(prev);
        sum += LC::var(cur);
        B.add(LC::var(nx), sum);
        B.assign(nx, nv);
        pv = cv;
        cv = nv;
        prev = cur;
        cur = nx;
    }
    B.assign(expected, cv);
    B.add(LC::var(expected), LC::var(cur));
}

void build_poseidon(Builder &B, uint64_t count, int density, std::mt19937_64 &rng)
{
    const Sampler sampler(2 * count, density, rng);
    for (uint64_t i = 0; i < count; ++i) {
        const Fr lv = sampler.sample(2 * i, [&] { return random_element(rng); });
        const Fr rv = sampler.sample(2 * i + 1, [&] { return random_element(rng); });
        const Fr dv = poseidon_hash2(lv, rv);
        const uint64_t d = B.new_public(), l = B.new_private(), r = B.new_private();
        B.assign(d, dv);
        B.assign(l, lv);
        B.assign(r, rv);
        poseidon_gadget(B, l, lv, r, rv, d);
    }
}

uint32_t low_u32(const Fr &v)
{
    uint64_t c[4];
    to_canonical(v, c);
    return uint32_t(c[0]);
}

// sql_aggregate.hpp:33-51
void uint32_gadget(Builder &B, uint64_t var, uint32_t raw)
{
    LC recomposed = LC::dflt();
    Fr coeff = one();
    for (int bit = 0; bit < 32; ++bit) {
        const uint64_t b = B.new_private();
        B.assign(b, (raw >> bit) & 1 ? one() : zero());
        B.add(LC::var(b), LC::var(b), LC::var(b));
        recomposed += LC::var(b) * coeff;
        coeff += coeff;
    }
    B.add(LC::var(var), recomposed);
}

void build_sql(Builder &B, uint64_t rows_n, int density, std::mt19937_64 &rng)
{
    if (rows_n < 2 || (rows_n & (rows_n - 1)))
        throw std::invalid_argument("SQL row count must be a power of two and at least 2");
    struct Row {
        Fr category, amount;
        uint32_t cat_raw, amt_raw;
    };
    std::vector<Row> rows;
    const Sampler sampler(rows_n, density, rng);
    for (uint64_t i = 0; i < rows_n; ++i) {
        uint64_t c[4];
        to_canonical(random_element(rng), c);
        const uint32_t cat = uint32_t(c[0] % 16);
        const Fr amount = sampler.sample(i, [&] {
            uint64_t a[4];
            to_canonical(random_element(rng), a);
            return from_u64(uint32_t(a[0]));
        });
        rows.push_back({from_u64(cat), amount, cat, low_u32(amount)});
    }
    const Fr target = rows.front().category;
    // sql_query.hpp:210-248
    Fr count = zero(), sum = zero();
    std::vector<Fr> level;
    for (const Row &r : rows) {
        level.push_back(poseidon_hash2(r.category, r.amount));
        if (r.category == target) {
            count += one();
            sum += r.amount;
        }
    }
    {
        std::vector<Fr> lv = level;
        while (lv.size() > 1) {
            std::vector<Fr> nx;
            for (size_t i = 0; i < lv.size(); i += 2) nx.push_back(poseidon_hash2(lv[i], lv[i + 1]));
            lv.swap(nx);
        }
        const uint64_t table_root = B.new_public(), target_cat = B.new_public(),
                       expected_count = B.new_public(), expected_sum = B.new_public();
        B.assign(table_root, lv.front());
        B.assign(target_cat, target);
        B.assign(expected_count, count);
        B.assign(expected_sum, sum);
        // sql_aggregate.hpp:58-165
        uint32_gadget(B, target_cat, rows.front().cat_raw);
        std::vector<uint64_t> cats, amts, lvl;
        std::vector<Fr> lvl_vals;
        for (const Row &r : rows) {
            const uint64_t cv = B.new_private(), av = B.new_private();
            B.assign(cv, r.category);
            B.assign(av, r.amount);
            cats.push_back(cv);
            amts.push_back(av);
            uint32_gadget(B, cv, r.cat_raw);
            uint32_gadget(B, av, r.amt_raw);
            const uint64_t leaf = B.new_private();
            const Fr leaf_v = poseidon_hash2(r.category, r.amount);
            B.assign(leaf, leaf_v);
            poseidon_gadget(B, cv, r.category, av, r.amount, leaf);
            lvl.push_back(leaf);
            lvl_vals.push_back(leaf_v);
        }
        while (lvl.size() > 1) {
            std::vector<uint64_t> nl;
            std::vector<Fr> nv;
            const bool final_level = lvl.size() == 2;
            for (size_t i = 0; i < lvl.size(); i += 2) {
                const Fr dv = poseidon_hash2(lvl_vals[i], lvl_vals[i + 1]);
                if (final_level) {
                    B.assign(table_root, dv);
                    poseidon_gadget(B, lvl[i], lvl_vals[i], lvl[i + 1], lvl_vals[i + 1], table_root);
                    nl.push_back(table_root);
                } else {
                    const uint64_t d = B.new_private();
                    B.assign(d, dv);
                    poseidon_gadget(B, lvl[i], lvl_vals[i], lvl[i + 1], lvl_vals[i + 1], d);
                    nl.push_back(d);
                }
                nv.push_back(dv);
            }
            lvl.swap(nl);
            lvl_vals.swap(nv);
        }
        LC count_sum = LC::dflt(), amount_sum = LC::dflt();
        const Fr minus_one = -one();
        for (size_t i = 0; i < rows.size(); ++i) {
            LC delta = LC::var(cats[i]);
            delta += LC::var(target_cat) * minus_one;
            const uint64_t match = B.new_private(), inv = B.new_private(), sel = B.new_private();
            const bool equal = rows[i].category == target;
            const Fr match_v = equal ? one() : zero();
            const Fr delta_v = rows[i].category - target;
            const Fr inv_v = equal ? zero() : inverse(delta_v);
            const Fr sel_v = match_v * rows[i].amount;
            B.assign(match, match_v);
            B.assign(inv, inv_v);
            B.assign(sel, sel_v);
            LC one_minus_match = LC::constant(one());
            one_minus_match += LC::var(match) * minus_one;
            B.add(one_minus_match, delta, LC::var(inv));
            B.add(LC::constant(zero()), delta, LC::var(match));
            B.add(LC::var(sel), LC::var(match), LC::var(amts[i]));
            count_sum += LC::var(match);
            amount_sum += LC::var(sel);
        }
        B.add(LC::var(expected_count), count_sum);
        B.add(LC::var(expected_sum), amount_sum);
    }
}

} // namespace

Fr poseidon(const Fr &l, const Fr &r) { return poseidon_hash2(l, r); }

void poseidon_parameters(Fr rc[195], Fr mds[9])
{
    const PoseidonParams &P = poseidon_params();
    std::copy(P.rc, P.rc + 195, rc);
    for (int i = 0; i < 9; ++i) mds[i] = P.mds[i / 3][i % 3];
}

// gen.cpp finalize_circuit (:30-40) + R1CSManager::gen_spmat with padding
std::unique_ptr<R1cs> generate(const std::string &kind, uint64_t param, int density, uint64_t seed)
{
    std::mt19937_64 rng(seed);
    Builder B;
    if (kind == "matmul") {
        if (param == 0) throw std::invalid_argument("matmul size must be positive");
        build_matmul(B, param, density, rng);
    } else if (kind == "fibonacci") {
        if (density != 0) throw std::invalid_argument("--density applies to matmul, poseidon, sql-aggregate");
        build_fibonacci(B, param, rng);
    } else if (kind == "poseidon") {
        if (param == 0) throw std::invalid_argument("poseidon count must be positive");
        build_poseidon(B, param, density, rng);
    } else if (kind == "sql-aggregate") {
        build_sql(B, param, density, rng);
    } else {
        throw std::invalid_argument("unknown circuit kind: " + kind);
    }
    auto out = std::make_unique<R1cs>();
    uint64_t rows = 1, cols = 1;
    const uint64_t n_cons = B.cons.size();
    const uint64_t n_vars = B.public_count + (B.private_count - kHalf);
    while (rows < n_cons) rows <<= 1;
    while (cols < n_vars) cols <<= 1;
    out->rows = rows;
    out->cols = cols;
    out->public_inputs = B.public_count - 1;
    out->constraints = n_cons;
    out->variables = n_vars;
    for (int k = 0; k < 3; ++k) {
        out->row_ptr[k].assign(rows + 1, 0);
        size_t total = 0;
        for (const auto &c : B.cons) total += (k == 0 ? c.a : k == 1 ? c.b : c.c).t.size();
        out->col_idx[k].reserve(total);
        out->values[k].reserve(total);
    }
    for (uint64_t r = 0; r < n_cons; ++r) {
        const Constraint &c = B.cons[r];
        const LC *lcs[3] = {&c.a, &c.b, &c.c};
        for (int k = 0; k < 3; ++k) {
            for (const Term &t : lcs[k]->t) {
                out->col_idx[k].push_back(uint32_t(B.dense(t.id)));
                out->values[k].push_back(t.c);
            }
            out->row_ptr[k][r + 1] = uint32_t(out->col_idx[k].size());
        }
    }
    for (uint64_t r = n_cons; r < rows; ++r)
        for (int k = 0; k < 3; ++k) out->row_ptr[k][r + 1] = uint32_t(out->col_idx[k].size());
    out->witness.assign(cols, zero());
    out->witness[0] = one();
    for (uint64_t id = 1; id < B.public_count; ++id) out->witness[id] = B.pub_vals[id];
    for (uint64_t k = 0; k < B.priv_vals.size(); ++k) out->witness[B.public_count + k] = B.priv_vals[k];
    return out;
}

} // namespace nkr::host
