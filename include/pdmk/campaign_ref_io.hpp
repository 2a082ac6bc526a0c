// Campaign reference files: oracle potentials at M sampled points of an
// N-point periodic system, stored with the system itself in the 'PDMC' binary
// format of the reference's cpp/include/pdmk/campaign_ref_io.hpp:13-45 (same
// header fields, byte layout, body order and SHA-256 check, so files written by
// either library read in the other).
//
// File = 80-byte little-endian header, then the body
//   cell[9] (column-major, cell[j*3+i] = component i of lattice vector j),
//   ref_idx[M] (uint32), ref_u[M] (double), pos[3N] (double), chg[N] (double);
// header.body_sha256 is the SHA-256 (FIPS 180-4) of the body.
// The functions are defined in libpdmk_b200.so (csrc/api/campaign_ref_io.cpp).
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace pdmk::campaign {

constexpr uint32_t MAGIC = 0x50444D43u;  // bytes 43 4D 44 50 on disk
constexpr uint32_t VERSION = 1u;
constexpr uint32_t ENDIAN_TAG = 0x01020304u;
constexpr uint32_t HEADER_LEN = 80u;
constexpr uint32_t DEFAULT_M = 1000u;  // sampled points per file

#pragma pack(push, 1)
struct RefHeader {
    uint32_t magic;
    uint32_t version;
    uint32_t endian_tag;
    uint32_t header_len;
    uint32_t config_id;  // caller's label of the configuration
    uint32_t N;          // points
    uint8_t digits;      // accuracy the reference potentials were computed at
    uint8_t prec;        // caller's precision tag
    uint8_t _pad[2];
    uint32_t M;          // sampled points (set from ref_idx by write_ref)
    uint64_t seed;       // caller's generator seed
    uint64_t body_len;   // bytes after the header (set by write_ref)
    uint8_t body_sha256[32];
};
#pragma pack(pop)
static_assert(sizeof(RefHeader) == 80, "RefHeader must be 80 bytes");

struct RefData {
    RefHeader header;
    double cell[9];
    std::vector<uint32_t> ref_idx;  // M sampled point indices
    std::vector<double> ref_u;      // M reference potentials
    std::vector<double> pos;        // 3N, pos[3 i + d]
    std::vector<double> chg;        // N
};

// SHA-256 digest of len bytes.
void sha256(const uint8_t* data, size_t len, uint8_t out[32]);
// The body bytes of d (cell, ref_idx, ref_u, pos, chg).
std::vector<uint8_t> pack_body(const RefData& d);
// Writes d; magic, version, endian tag, header length, M, body length and
// digest are filled in.  Throws std::runtime_error on I/O failure and
// std::invalid_argument if ref_u, pos or chg do not match M and header.N.
void write_ref(const std::string& path, const RefData& d);
// Reads and checks a file; throws std::runtime_error on a short read, a wrong
// magic / version / endian tag / header length, a body length that does not
// match N and M, or a digest mismatch.
RefData read_ref(const std::string& path);

}  // namespace pdmk::campaign
