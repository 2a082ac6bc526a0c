// The C++ form of the campaign reference files (include/pdmk/campaign_ref_io.hpp)
// compiled against libpdmk_b200.so: the cases of the reference's
// cpp/tests/test_campaign_ref_io.cpp (empty-string digest, round trip with
// M = DEFAULT_M and N = 50, tampered body rejected).  Needs no GPU.
#include <pdmk/campaign_ref_io.hpp>

#include <cstdio>
#include <cstring>
#include <random>
#include <stdexcept>
#include <string>

using namespace pdmk::campaign;

static int failures = 0;
static void check(bool ok, const char* what) {
    std::printf("%s %s\n", ok ? "ok  " : "FAIL", what);
    if (!ok) ++failures;
}

int main(int argc, char** argv) {
    const std::string dir = argc > 1 ? argv[1] : ".";
    {
        uint8_t out[32];
        sha256(reinterpret_cast<const uint8_t*>(""), 0, out);
        const uint8_t want[32] = {0xe3, 0xb0, 0xc4, 0x42, 0x98, 0xfc, 0x1c, 0x14, 0x9a, 0xfb, 0xf4,
                                  0xc8, 0x99, 0x6f, 0xb9, 0x24, 0x27, 0xae, 0x41, 0xe4, 0x64, 0x9b,
                                  0x93, 0x4c, 0xa4, 0x95, 0x99, 0x1b, 0x78, 0x52, 0xb8, 0x55};
        check(std::memcmp(out, want, 32) == 0, "sha256_empty");
    }
    {
        RefData in{};
        in.header.config_id = 7;
        in.header.N = 50;
        in.header.digits = 6;
        in.header.prec = 1;
        in.header.seed = 0xDEADBEEFCAFEBABEull;
        for (int i = 0; i < 9; ++i) in.cell[i] = (i % 4 == 0) ? 1.0 : 0.0;
        in.ref_idx.resize(DEFAULT_M);
        in.ref_u.resize(DEFAULT_M);
        for (uint32_t i = 0; i < DEFAULT_M; ++i) {
            in.ref_idx[i] = i % in.header.N;
            in.ref_u[i] = double(i) * 1e-3;
        }
        std::mt19937_64 rng(1);
        std::uniform_real_distribution<double> U(0.0, 1.0);
        in.pos.resize(3 * in.header.N);
        in.chg.resize(in.header.N);
        for (auto& x : in.pos) x = U(rng);
        for (auto& x : in.chg) x = U(rng);
        const std::string path = dir + "/pdmk_ref_roundtrip.bin";
        write_ref(path, in);
        const RefData out = read_ref(path);
        check(out.header.magic == MAGIC && out.header.version == VERSION && out.header.endian_tag == ENDIAN_TAG,
              "roundtrip_tags");
        check(out.header.config_id == 7 && out.header.N == 50 && out.header.M == DEFAULT_M &&
                  out.header.seed == 0xDEADBEEFCAFEBABEull,
              "roundtrip_header");
        check(out.pos == in.pos && out.chg == in.chg && out.ref_idx == in.ref_idx && out.ref_u == in.ref_u,
              "roundtrip_body");
        std::remove(path.c_str());
    }
    {
        RefData in{};
        in.header.N = 10;
        in.header.digits = 6;
        in.header.prec = 1;
        in.pos.assign(30, 0.0);
        in.chg.assign(10, 0.0);
        in.ref_idx.assign(DEFAULT_M, 0);
        in.ref_u.assign(DEFAULT_M, 0.0);
        const std::string path = dir + "/pdmk_ref_tamper.bin";
        write_ref(path, in);
        FILE* fp = std::fopen(path.c_str(), "rb+");
        std::fseek(fp, 80, SEEK_SET);
        const uint8_t tamper = 0xFF;
        std::fwrite(&tamper, 1, 1, fp);
        std::fclose(fp);
        bool threw = false;
        try {
            read_ref(path);
        } catch (const std::runtime_error&) {
            threw = true;
        }
        check(threw, "tampered_body_throws");
        std::remove(path.c_str());
    }
    std::printf("%d failures\n", failures);
    return failures ? 1 : 0;
}
