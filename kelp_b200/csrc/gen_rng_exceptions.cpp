// Generator of kc_rng_exceptions.bin: the Box-Muller inputs at which the host
// C library's log / sin / cos (what the reference's Numba kernels call) do not
// round correctly, scanned over the whole domain of the counter RNG.
//
// The reference draws (diffusion.py:222-249) u1 = (j1 + 1/2) 2^-32 and
// u2 = (j2 + 1/2) 2^-32 from the two 32-bit halves j1, j2 of its key hash,
// then r = sqrt(-2 log u1), g1 = r cos(2 pi u2), g2 = r sin(2 pi u2).  r
// depends on j1 alone and cos / sin on j2 alone, so the 2^32 values of each
// fix every draw.  This program evaluates, for every j, the C library's r,
// cos and sin and the correctly rounded ones (kc_crmath.cuh), and records
// each j where they differ as (j, bit delta) -- the library value's bit
// pattern minus the correctly rounded one's, +-1 (anything else aborts).
// It also checks that the fast paths of log_cr / sincos_cr return the
// double-double paths' results (fast_path_differs must be 0) and prints
// order-independent digests of the library's and the
// correctly rounded values over the whole domain, which the GPU test
// compares against the device (tests/golden/rng_domain.json).
//
// The build (kelp_b200/build.py) compiles and runs it when its output is
// missing or older than its sources (~6 minutes on 8 cores):
//   g++ -O2 -mfma -ffp-contract=off -std=c++17 -pthread -Ikelp_b200/csrc \
//       kelp_b200/csrc/gen_rng_exceptions.cpp -o _build/gen_rng_exceptions
//   _build/gen_rng_exceptions _build/kc_rng_exceptions.bin > _build/rng_domain.json
// tests/golden/rng_domain.json holds the digests of the C library this
// repository's fixtures were made with (glibc 2.39).
//
// File format (little-endian), the device layout (kc::DRngX): "KCRX",
// u32 version (2), u32 nA, u32 nB, u32 bucket bits (20); then for table a
// (r) and table b (cos / sin): 2^20 + 1 u32 bucket offsets (bucket = j >> 12)
// and n u16 entries (j & 0xfff) << 4 | code, ascending within a bucket.
// Codes: table a 1 = +1, 2 = -1 (the library's r bits minus the correctly
// rounded ones); table b bits 0-1 the cos delta, bits 2-3 the sin delta.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>
#include <gnu/libc-version.h>

#include "kc_crmath.cuh"

using kc::cr::bits_of;

static inline uint64_t mix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// digest term of value v at domain index j (the sum over j is order-free)
static inline uint64_t term(uint64_t j, double v) { return mix64(mix64(j) ^ bits_of(v)); }

static int delta_code(double lib, double cr, uint64_t j, const char* what) {
    if (bits_of(lib) == bits_of(cr)) return 0;
    const int64_t d = (int64_t)bits_of(lib) - (int64_t)bits_of(cr);
    if (d == 1) return 1;
    if (d == -1) return 2;
    std::fprintf(stderr, "%s at j=%llu: library %a, correctly rounded %a (not one bit apart)\n", what,
                 (unsigned long long)j, lib, cr);
    std::exit(1);
}

struct Part {
    uint64_t dr_lib = 0, dr_cr = 0, dc_lib = 0, dc_cr = 0, ds_lib = 0, ds_cr = 0;
    uint64_t ambiguous = 0, fast_differs = 0;
    std::vector<std::pair<uint32_t, uint8_t>> a;
    std::vector<std::pair<uint32_t, uint8_t>> b;
};

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s OUT.bin [n]\n", argv[0]);
        return 2;
    }
    const uint64_t n = argc > 2 ? std::strtoull(argv[2], nullptr, 0) : (1ull << 32);
    const unsigned T = std::max(1u, std::thread::hardware_concurrency());
    const double INV = 1.0 / 4294967296.0, HALF = 0.5 * INV, TWO_PI = 2.0 * 3.141592653589793;
    std::vector<Part> parts(T);
    std::vector<std::thread> th;
    for (unsigned t = 0; t < T; ++t) {
        th.emplace_back([&, t] {
            Part& p = parts[t];
            const uint64_t lo = n * t / T, hi = n * (t + 1) / T;
            for (uint64_t j = lo; j < hi; ++j) {
                const double u = (double)j * INV + HALF;
                bool amb = false;
                const double r_lib = std::sqrt(-2.0 * std::log(u));
                const double l_cr = kc::cr::log_cr_checked(u, &amb);
                p.ambiguous += amb;
                p.fast_differs += bits_of(kc::cr::log_cr(u)) != bits_of(l_cr);
                const double r_cr = std::sqrt(-2.0 * l_cr);
                const int rc = delta_code(r_lib, r_cr, j, "r");
                if (rc) p.a.push_back({(uint32_t)j, (uint8_t)rc});
                p.dr_lib += term(j, r_lib);
                p.dr_cr += term(j, r_cr);
                const double th2 = TWO_PI * u;
                double s_cr, c_cr;
                kc::cr::sincos_cr_checked(th2, &s_cr, &c_cr, &amb);
                p.ambiguous += amb;
                double s_f, c_f;
                kc::cr::sincos_cr(th2, &s_f, &c_f);
                p.fast_differs += (bits_of(s_f) != bits_of(s_cr)) + (bits_of(c_f) != bits_of(c_cr));
                const double s_lib = std::sin(th2), c_lib = std::cos(th2);
                const int cc = delta_code(c_lib, c_cr, j, "cos"), sc = delta_code(s_lib, s_cr, j, "sin");
                if (cc || sc) p.b.push_back({(uint32_t)j, (uint8_t)(cc | (sc << 2))});
                p.dc_lib += term(j, c_lib);
                p.dc_cr += term(j, c_cr);
                p.ds_lib += term(j, s_lib);
                p.ds_cr += term(j, s_cr);
            }
        });
    }
    for (auto& x : th) x.join();
    Part all;
    for (auto& p : parts) {   // parts cover ascending ranges: concatenation keeps keys sorted
        all.dr_lib += p.dr_lib; all.dr_cr += p.dr_cr; all.dc_lib += p.dc_lib; all.dc_cr += p.dc_cr;
        all.ds_lib += p.ds_lib; all.ds_cr += p.ds_cr; all.ambiguous += p.ambiguous;
        all.fast_differs += p.fast_differs;
        all.a.insert(all.a.end(), p.a.begin(), p.a.end());
        all.b.insert(all.b.end(), p.b.begin(), p.b.end());
    }
    FILE* f = std::fopen(argv[1], "wb");
    if (!f) return 1;
    const uint32_t BITS = 20, NB = 1u << BITS;
    const uint32_t hdr[5] = {0x5852434bu /* "KCRX" */, 2u, (uint32_t)all.a.size(), (uint32_t)all.b.size(), BITS};
    std::fwrite(hdr, 4, 5, f);
    auto put = [&](const auto& list) {
        std::vector<uint32_t> off(NB + 1, 0);
        std::vector<uint16_t> ent(list.size());
        for (size_t k = 0; k < list.size(); ++k) {
            const uint32_t j = list[k].first;
            const unsigned code = (unsigned)list[k].second;
            ent[k] = (uint16_t)(((j & 0xFFFu) << 4) | (code & 15u));
            off[(j >> 12) + 1]++;
        }
        for (uint32_t b = 0; b < NB; ++b) off[b + 1] += off[b];
        std::fwrite(off.data(), 4, off.size(), f);
        std::fwrite(ent.data(), 2, ent.size(), f);
    };
    put(all.a);
    put(all.b);
    std::fclose(f);
    std::printf("{\n  \"libc\": \"glibc %s\",\n  \"domain\": %llu,\n  \"ambiguous\": %llu,\n"
                "  \"fast_path_differs\": %llu,\n  \"exceptions_r\": %zu,\n  \"exceptions_trig\": %zu,\n"
                "  \"digest_r_lib\": \"%016llx\",\n  \"digest_r_cr\": \"%016llx\",\n"
                "  \"digest_cos_lib\": \"%016llx\",\n  \"digest_cos_cr\": \"%016llx\",\n"
                "  \"digest_sin_lib\": \"%016llx\",\n  \"digest_sin_cr\": \"%016llx\"\n}\n",
                gnu_get_libc_version(), (unsigned long long)n, (unsigned long long)all.ambiguous,
                (unsigned long long)all.fast_differs, all.a.size(),
                all.b.size(), (unsigned long long)all.dr_lib, (unsigned long long)all.dr_cr,
                (unsigned long long)all.dc_lib, (unsigned long long)all.dc_cr, (unsigned long long)all.ds_lib,
                (unsigned long long)all.ds_cr);
    return 0;
}
