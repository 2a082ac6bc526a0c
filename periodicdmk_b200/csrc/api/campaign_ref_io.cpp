// Campaign reference files ('PDMC' format, include/pdmk/campaign_ref_io.hpp;
// the reference's cpp/include/pdmk/campaign_ref_io.hpp:13-186) and the SHA-256
// digest that guards their body.
//
// SHA-256 follows FIPS 180-4 (sections 4.1.2, 4.2.2, 5.1.1, 6.2).  Its round
// constants are the first 32 bits of the fractional parts of the cube roots of
// the first 64 primes and its initial state those of the square roots of the
// first 8 primes (sections 4.2.2, 5.3.3); both are computed here, exactly, as
// integer roots: floor(cbrt(p) 2^32) = icbrt(p 2^96), floor(sqrt(p) 2^32) =
// isqrt(p 2^64), keeping the low 32 bits.
#include "pdmk/campaign_ref_io.hpp"

#include <array>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>

namespace pdmk::campaign {

namespace {

using u128 = unsigned __int128;

// largest r with r^k <= x (k = 2 or 3), by bisection on [0, 2^40)
uint64_t iroot(u128 x, int k) {
    uint64_t lo = 0, hi = (uint64_t)1 << 40;
    while (hi - lo > 1) {
        const uint64_t mid = lo + (hi - lo) / 2;
        u128 v = mid;
        for (int i = 1; i < k; ++i) v *= mid;
        if (v <= x) lo = mid;
        else hi = mid;
    }
    return lo;
}

struct Constants {
    std::array<uint32_t, 64> k{};
    std::array<uint32_t, 8> h0{};
    Constants() {
        int primes[64], np = 0;
        for (int c = 2; np < 64; ++c) {
            bool prime = true;
            for (int d = 2; d * d <= c; ++d)
                if (c % d == 0) {
                    prime = false;
                    break;
                }
            if (prime) primes[np++] = c;
        }
        for (int i = 0; i < 64; ++i) k[i] = (uint32_t)iroot((u128)primes[i] << 96, 3);
        for (int i = 0; i < 8; ++i) h0[i] = (uint32_t)iroot((u128)primes[i] << 64, 2);
    }
};

const Constants& constants() {
    static const Constants c;
    return c;
}

inline uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }

// One 64-byte block into the state (FIPS 180-4 6.2.2).
void compress(uint32_t st[8], const uint8_t* blk, const uint32_t* K) {
    uint32_t w[64];
    for (int t = 0; t < 16; ++t)
        w[t] = (uint32_t)blk[4 * t] << 24 | (uint32_t)blk[4 * t + 1] << 16 | (uint32_t)blk[4 * t + 2] << 8 |
               (uint32_t)blk[4 * t + 3];
    for (int t = 16; t < 64; ++t) {
        const uint32_t s0 = rotr(w[t - 15], 7) ^ rotr(w[t - 15], 18) ^ (w[t - 15] >> 3);
        const uint32_t s1 = rotr(w[t - 2], 17) ^ rotr(w[t - 2], 19) ^ (w[t - 2] >> 10);
        w[t] = s1 + w[t - 7] + s0 + w[t - 16];
    }
    uint32_t v[8];
    std::memcpy(v, st, sizeof(v));  // a b c d e f g h
    for (int t = 0; t < 64; ++t) {
        const uint32_t e = v[4], a = v[0];
        const uint32_t t1 = v[7] + (rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25)) + ((e & v[5]) ^ (~e & v[6])) + K[t] + w[t];
        const uint32_t t2 = (rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22)) + ((a & v[1]) ^ (a & v[2]) ^ (v[1] & v[2]));
        std::memmove(v + 1, v, 7 * sizeof(uint32_t));
        v[4] += t1;
        v[0] = t1 + t2;
    }
    for (int i = 0; i < 8; ++i) st[i] += v[i];
}

constexpr size_t body_bytes(uint64_t n, uint64_t m) { return 9 * 8 + m * 4 + m * 8 + n * 24 + n * 8; }

struct File {
    FILE* f = nullptr;
    File(const std::string& path, const char* mode) : f(std::fopen(path.c_str(), mode)) {}
    ~File() {
        if (f) std::fclose(f);
    }
};

}  // namespace

void sha256(const uint8_t* data, size_t len, uint8_t out[32]) {
    const Constants& c = constants();
    uint32_t st[8];
    for (int i = 0; i < 8; ++i) st[i] = c.h0[i];
    size_t off = 0;
    for (; off + 64 <= len; off += 64) compress(st, data + off, c.k.data());
    // padding (5.1.1): 0x80, zeros, the bit length as a big-endian 64-bit word
    uint8_t last[128] = {};
    const size_t rem = len - off;
    if (rem) std::memcpy(last, data + off, rem);
    last[rem] = 0x80;
    const size_t nb = rem < 56 ? 64 : 128;
    const uint64_t bits = (uint64_t)len * 8;
    for (int i = 0; i < 8; ++i) last[nb - 1 - i] = (uint8_t)(bits >> (8 * i));
    for (size_t b = 0; b < nb; b += 64) compress(st, last + b, c.k.data());
    for (int i = 0; i < 8; ++i)
        for (int j = 0; j < 4; ++j) out[4 * i + j] = (uint8_t)(st[i] >> (24 - 8 * j));
}

std::vector<uint8_t> pack_body(const RefData& d) {
    const size_t m = d.ref_idx.size();
    if (d.ref_u.size() != m) throw std::invalid_argument("ref_u and ref_idx differ in length");
    if (d.pos.size() != 3 * (size_t)d.header.N || d.chg.size() != (size_t)d.header.N)
        throw std::invalid_argument("pos / chg do not match header.N");
    std::vector<uint8_t> body(body_bytes(d.header.N, m));
    uint8_t* p = body.data();
    auto put = [&](const void* src, size_t n) {
        if (n) std::memcpy(p, src, n);
        p += n;
    };
    put(d.cell, sizeof(d.cell));
    put(d.ref_idx.data(), m * sizeof(uint32_t));
    put(d.ref_u.data(), m * sizeof(double));
    put(d.pos.data(), d.pos.size() * sizeof(double));
    put(d.chg.data(), d.chg.size() * sizeof(double));
    return body;
}

void write_ref(const std::string& path, const RefData& d) {
    RefHeader h = d.header;
    h.magic = MAGIC;
    h.version = VERSION;
    h.endian_tag = ENDIAN_TAG;
    h.header_len = HEADER_LEN;
    h.M = (uint32_t)d.ref_idx.size();
    const std::vector<uint8_t> body = pack_body(d);
    h.body_len = body.size();
    sha256(body.data(), body.size(), h.body_sha256);
    File f(path, "wb");
    if (!f.f) throw std::runtime_error("cannot open for write: " + path);
    if (std::fwrite(&h, sizeof(h), 1, f.f) != 1 ||
        (body.size() && std::fwrite(body.data(), 1, body.size(), f.f) != body.size()))
        throw std::runtime_error("write failed: " + path);
    if (std::fflush(f.f) != 0) throw std::runtime_error("write failed: " + path);
}

RefData read_ref(const std::string& path) {
    File f(path, "rb");
    if (!f.f) throw std::runtime_error("cannot open for read: " + path);
    RefData d{};
    if (std::fread(&d.header, sizeof(RefHeader), 1, f.f) != 1) throw std::runtime_error("header short read: " + path);
    const RefHeader& h = d.header;
    if (h.magic != MAGIC) throw std::runtime_error("bad magic: " + path);
    if (h.version != VERSION) throw std::runtime_error("bad version: " + path);
    if (h.endian_tag != ENDIAN_TAG) throw std::runtime_error("bad endian tag: " + path);
    if (h.header_len != HEADER_LEN) throw std::runtime_error("bad header_len: " + path);
    if (h.body_len != body_bytes(h.N, h.M)) throw std::runtime_error("body length does not match N and M: " + path);
    std::vector<uint8_t> body(h.body_len);
    if (!body.empty() && std::fread(body.data(), 1, body.size(), f.f) != body.size())
        throw std::runtime_error("body short read: " + path);
    uint8_t digest[32];
    sha256(body.data(), body.size(), digest);
    if (std::memcmp(digest, h.body_sha256, 32) != 0) throw std::runtime_error("sha256 mismatch: " + path);
    const uint8_t* p = body.data();
    auto get = [&](void* dst, size_t n) {
        if (n) std::memcpy(dst, p, n);
        p += n;
    };
    get(d.cell, sizeof(d.cell));
    d.ref_idx.resize(h.M);
    get(d.ref_idx.data(), h.M * sizeof(uint32_t));
    d.ref_u.resize(h.M);
    get(d.ref_u.data(), h.M * sizeof(double));
    d.pos.resize(3 * (size_t)h.N);
    get(d.pos.data(), d.pos.size() * sizeof(double));
    d.chg.resize(h.N);
    get(d.chg.data(), d.chg.size() * sizeof(double));
    return d;
}

}  // namespace pdmk::campaign
