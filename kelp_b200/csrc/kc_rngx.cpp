// The Box-Muller exception tables (written by gen_rng_exceptions.cpp at build
// time, already in the device layout kc::DRngX) linked into the library as
// read-only data.
#include <cstdint>
#include <cstring>

#include "kc_host.h"

#ifndef KC_RNGX_PATH
#error "KC_RNGX_PATH must name the scanner's table file (set by kelp_b200/build.py)"
#endif

__asm__(".section .rodata\n"
        ".balign 64\n"
        ".hidden kc_rngx_blob_begin\n"
        ".hidden kc_rngx_blob_end\n"
        "kc_rngx_blob_begin:\n"
        ".incbin \"" KC_RNGX_PATH "\"\n"
        "kc_rngx_blob_end:\n"
        ".previous\n");

extern "C" const unsigned char kc_rngx_blob_begin[];
extern "C" const unsigned char kc_rngx_blob_end[];

namespace kc_host {

bool rng_exception_tables(RngTables& t) {
    const unsigned char* p = kc_rngx_blob_begin;
    const size_t len = (size_t)(kc_rngx_blob_end - kc_rngx_blob_begin);
    uint32_t h[5];
    if (len < sizeof(h)) return false;
    std::memcpy(h, p, sizeof(h));
    if (h[0] != 0x5852434bu || h[1] != 2u || h[4] != 20u) return false;
    const size_t noff = (1u << 20) + 1;
    const size_t need = sizeof(h) + 2 * noff * 4 + 2ull * h[2] + 2ull * h[3];
    if (len != need) return false;
    const unsigned char* q = p + sizeof(h);   // 20 bytes in: 4-byte alignment holds
    t.a_off = (const unsigned*)q;
    q += noff * 4;
    t.a = (const unsigned short*)q;
    q += 2ull * h[2];
    t.b_off = (const unsigned*)q;   // 2-byte aligned only when na is odd: the host copies through memcpy
    q += noff * 4;
    t.b = (const unsigned short*)q;
    t.n_off = noff;
    t.na = h[2];
    t.nb = h[3];
    return true;
}

}  // namespace kc_host
