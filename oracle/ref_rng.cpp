// ref_rng.cpp - extern "C" access to gdt::LCG<16> of the reference renderer
// (common/gdt/gdt/random/random.h:54-87).  TEST INFRASTRUCTURE ONLY.
#include <cstdint>
#include "gdt/random/random.h"

extern "C" void ref_lcg(uint32_t v0, uint32_t v1, int32_t n, float* out) {
    gdt::LCG<16> r;
    r.init(v0, v1);
    for (int i = 0; i < n; i++) out[i] = r();
}
