// Test infrastructure: exposes the reference NewPFor.cpp codec (compiled from
// the reference sources by oracle/Makefile) under C names for the checkers.
#include <stdint.h>

#include "NewPFor.h"

extern float FRAC;  // NewPFor.cpp:17

extern "C" {
void ref_newpfd_set_frac(float f) { FRAC = f; }
uint32_t ref_newpfd_encode(const uint32_t *in, uint32_t *out, uint32_t n) { return encodeArray(in, out, n); }
uint32_t ref_newpfd_decode(const uint32_t *in, uint32_t *out, uint32_t n) { return decodeArray(in, out, n); }
}
