// Proving-key artifacts in the reference's BinaryArchive format, read and written
// without the reference reader's 1 GiB per-vector limit.
//
// Format (protocols/groth16/common/src/io.cpp:54-61 over
// common/include/binary_archive.hpp:17-98): the magic "LKZ1", a u32 version (1),
// then a_query, b_g1_query, b_g2_query, l_query, h_query, each as a u64 byte
// length followed by the raw libff points (G1 96 B, G2 192 B, Jacobian), then the
// raw points alpha_g1, beta_g1 (G1), beta_g2 (G2), delta_g1 (G1), delta_g2 (G2).
// The reference refuses vectors above 1 GiB (binary_archive.hpp:19, 76-77,
// 89-90), so it can neither write nor read the keys of circuits from 2^24
// constraints up (a_query alone is 1.5 GiB there); this file has no such limit.
//
// The reader memory-maps the file and hands the mapped queries to
// nkr_b200_prepare, so a key goes from disk to HBM without a second host copy.
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include "../../include/nkr_b200.h"

namespace nkr {
void set_error(const char *fmt, ...);
}

namespace {

constexpr char kMagic[4] = {'L', 'K', 'Z', '1'};
constexpr uint32_t kVersion = 1;
constexpr uint64_t kG1 = 96, kG2 = 192;
constexpr uint64_t kConstBytes = kG1 + kG1 + kG2 + kG1 + kG2; // alpha, beta (G1, G2), delta (G1, G2)

// Offsets of the parts of a mapped proving-key file, checked against its size.
struct PkLayout {
    uint64_t off[5] = {}, bytes[5] = {}; // a, b_g1, b_g2, l, h
    uint64_t consts = 0;                 // offset of alpha_g1
};

int parse(const uint8_t *p, uint64_t size, const char *path, PkLayout &L)
{
    if (size < 8 || std::memcmp(p, kMagic, 4) != 0) {
        nkr::set_error("%s: not a BinaryArchive file (magic LKZ1 missing)", path);
        return NKR_B200_EINVAL;
    }
    uint32_t version = 0;
    std::memcpy(&version, p + 4, 4);
    if (version != kVersion) {
        nkr::set_error("%s: BinaryArchive version %u, expected %u", path, version, kVersion);
        return NKR_B200_EINVAL;
    }
    static const char *names[5] = {"a_query", "b_g1_query", "b_g2_query", "l_query", "h_query"};
    static const uint64_t elem[5] = {kG1, kG1, kG2, kG1, kG1};
    uint64_t pos = 8;
    for (int k = 0; k < 5; ++k) {
        if (size - pos < 8) {
            nkr::set_error("%s: truncated before the length of %s", path, names[k]);
            return NKR_B200_EINVAL;
        }
        uint64_t n = 0;
        std::memcpy(&n, p + pos, 8);
        pos += 8;
        if (n % elem[k] != 0) {
            nkr::set_error("%s: %s has %llu bytes, not a whole number of %llu-byte points", path,
                           names[k], (unsigned long long)n, (unsigned long long)elem[k]);
            return NKR_B200_EINVAL;
        }
        if (n > size - pos) {
            nkr::set_error("%s: truncated inside %s (%llu bytes announced, %llu left)", path, names[k],
                           (unsigned long long)n, (unsigned long long)(size - pos));
            return NKR_B200_EINVAL;
        }
        L.off[k] = pos;
        L.bytes[k] = n;
        pos += n;
    }
    if (size - pos < kConstBytes) {
        nkr::set_error("%s: truncated in the alpha / beta / delta points", path);
        return NKR_B200_EINVAL;
    }
    L.consts = pos;
    return NKR_B200_OK;
}

struct Mapping {
    void *p = MAP_FAILED;
    uint64_t size = 0;
    int fd = -1;
    ~Mapping()
    {
        if (p != MAP_FAILED) munmap(p, size);
        if (fd >= 0) close(fd);
    }
};

int map_file(const char *path, Mapping &m)
{
    m.fd = open(path, O_RDONLY);
    if (m.fd < 0) {
        nkr::set_error("%s: cannot open: %s", path, std::strerror(errno));
        return NKR_B200_EINVAL;
    }
    struct stat st {};
    if (fstat(m.fd, &st) != 0) {
        nkr::set_error("%s: cannot stat: %s", path, std::strerror(errno));
        return NKR_B200_EINVAL;
    }
    m.size = uint64_t(st.st_size);
    if (m.size == 0) {
        nkr::set_error("%s: empty file", path);
        return NKR_B200_EINVAL;
    }
    m.p = mmap(nullptr, m.size, PROT_READ, MAP_PRIVATE, m.fd, 0);
    if (m.p == MAP_FAILED) {
        nkr::set_error("%s: mmap failed: %s", path, std::strerror(errno));
        return NKR_B200_EINVAL;
    }
    madvise(m.p, m.size, MADV_SEQUENTIAL);
    return NKR_B200_OK;
}

bool write_all(FILE *f, const void *p, uint64_t n)
{
    return n == 0 || std::fwrite(p, 1, n, f) == n;
}

} // namespace

extern "C" {

int nkr_b200_pk_file_info(const char *path, uint64_t *rows, uint64_t *cols)
{
    if (!path || !rows || !cols) {
        nkr::set_error("null argument");
        return NKR_B200_EINVAL;
    }
    Mapping m;
    if (int s = map_file(path, m)) return s;
    PkLayout L;
    if (int s = parse(static_cast<const uint8_t *>(m.p), m.size, path, L)) return s;
    const uint64_t c = L.bytes[0] / kG1;
    if (L.bytes[1] / kG1 != c || L.bytes[2] / kG2 != c || L.bytes[3] / kG1 != c) {
        nkr::set_error("%s: the a, b_g1, b_g2 and l queries have different point counts", path);
        return NKR_B200_EINVAL;
    }
    *cols = c;
    *rows = L.bytes[4] / kG1;
    return NKR_B200_OK;
}

int nkr_b200_prepare_file(nkr_b200_ctx *ctx, const nkr_b200_circuit *circuit, const char *pk_path,
                          nkr_b200_key **out)
{
    if (!circuit || !pk_path || !out) {
        nkr::set_error("null argument");
        return NKR_B200_EINVAL;
    }
    Mapping m;
    if (int s = map_file(pk_path, m)) return s;
    PkLayout L;
    const uint8_t *base = static_cast<const uint8_t *>(m.p);
    if (int s = parse(base, m.size, pk_path, L)) return s;
    static const char *names[5] = {"a_query", "b_g1_query", "b_g2_query", "l_query", "h_query"};
    const uint64_t want[5] = {circuit->cols * kG1, circuit->cols * kG1, circuit->cols * kG2,
                              circuit->cols * kG1, circuit->rows * kG1};
    for (int k = 0; k < 5; ++k)
        if (L.bytes[k] != want[k]) {
            nkr::set_error("%s: %s has %llu bytes, the circuit (%llu rows, %llu columns) needs %llu",
                           pk_path, names[k], (unsigned long long)L.bytes[k],
                           (unsigned long long)circuit->rows, (unsigned long long)circuit->cols,
                           (unsigned long long)want[k]);
            return NKR_B200_EINVAL;
        }
    nkr_b200_proving_key pk{};
    pk.a_query = base + L.off[0];
    pk.b_g1_query = base + L.off[1];
    pk.b_g2_query = base + L.off[2];
    pk.l_query = base + L.off[3];
    pk.h_query = base + L.off[4];
    const uint8_t *c = base + L.consts;
    pk.alpha_g1 = c;
    pk.beta_g1 = c + kG1;
    pk.beta_g2 = c + 2 * kG1;
    pk.delta_g1 = c + 2 * kG1 + kG2;
    pk.delta_g2 = c + 3 * kG1 + kG2;
    // prepare copies everything it keeps (to HBM) before it returns; the mapping
    // is released afterwards
    return nkr_b200_prepare(ctx, circuit, &pk, out);
}

int nkr_b200_write_proving_key(const char *path, const nkr_b200_proving_key *pk, uint64_t rows,
                               uint64_t cols)
{
    if (!path || !pk || !pk->a_query || !pk->b_g1_query || !pk->b_g2_query || !pk->l_query ||
        !pk->h_query || !pk->alpha_g1 || !pk->beta_g1 || !pk->beta_g2 || !pk->delta_g1 ||
        !pk->delta_g2) {
        nkr::set_error("null argument");
        return NKR_B200_EINVAL;
    }
    FILE *f = std::fopen(path, "wb");
    if (!f) {
        nkr::set_error("%s: cannot open for writing: %s", path, std::strerror(errno));
        return NKR_B200_EINVAL;
    }
    const void *vec[5] = {pk->a_query, pk->b_g1_query, pk->b_g2_query, pk->l_query, pk->h_query};
    const uint64_t bytes[5] = {cols * kG1, cols * kG1, cols * kG2, cols * kG1, rows * kG1};
    bool ok = write_all(f, kMagic, 4) && write_all(f, &kVersion, 4);
    for (int k = 0; k < 5 && ok; ++k) ok = write_all(f, &bytes[k], 8) && write_all(f, vec[k], bytes[k]);
    ok = ok && write_all(f, pk->alpha_g1, kG1) && write_all(f, pk->beta_g1, kG1) &&
         write_all(f, pk->beta_g2, kG2) && write_all(f, pk->delta_g1, kG1) &&
         write_all(f, pk->delta_g2, kG2);
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) {
        nkr::set_error("%s: write failed", path);
        return NKR_B200_EINVAL;
    }
    return NKR_B200_OK;
}

} // extern "C"
