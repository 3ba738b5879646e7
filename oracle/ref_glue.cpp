// Test infrastructure: exposes the reference ParaPFor.cpp codec (compiled from
// the reference sources by oracle/Makefile) under C names for the checkers.
#include <stdint.h>

#include "ParaPFor.h"

extern float FRAC;  // ParaPFor.cpp:19

extern "C" {
void ref_set_frac(float f) { FRAC = f; }
uint32_t ref_encode(const uint32_t *in, uint32_t *out, uint32_t n) { return encodeArray(in, out, n); }
uint32_t ref_decode(const uint32_t *in, uint32_t *out, uint32_t n) { return decodeArray(in, out, n); }
}
