// ref_philox.cpp — exposes the reference's Philox-2x32-10 and Box-Muller
// (shaders/philox.h:19-50, compiled as C++ through oracle/ref_shim) to the
// tests.  TEST INFRASTRUCTURE ONLY; built into oracle/_ref by oracle/Makefile.
#include <metal_stdlib>

#include <cstdint>

#include "philox.h"

extern "C" {

void ref_philox_words(uint64_t n, const uint32_t* c0, const uint32_t* c1, const uint32_t* key,
                      uint32_t* out) {
  for (uint64_t i = 0; i < n; ++i) {
    const uint2 w = philox2x32_10(uint2(c0[i], c1[i]), key[i]);
    out[2 * i] = w.x;
    out[2 * i + 1] = w.y;
  }
}

void ref_box_muller(uint64_t n, const uint32_t* words, float* out) {
  for (uint64_t i = 0; i < n; ++i) {
    const float2 g = box_muller(uint2(words[2 * i], words[2 * i + 1]));
    out[2 * i] = g.x;
    out[2 * i + 1] = g.y;
  }
}

}  // extern "C"
