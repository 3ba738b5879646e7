// Test infrastructure: compiles the reference's getRegressionInfo() bodies
// (cut from SegLRC_Generator.cu:264-331 and LRC_Generator.cu:221-287 by
// oracle/Makefile) with the record layouts those files declare
// (SegLRC_Generator_kernel.cu:37-48, LRC_Generator_kernel.cu:37-47), and
// exposes them under C names so the oracle's and the library's fits can be
// compared with the reference's own arithmetic.
#include <stdint.h>
#include <string.h>

namespace seglrc {
typedef struct {
    float fSlope;
    float fIntercept;
    uint32_t nRangeLeft;
    uint32_t nRangeRight;
} regression_info_t;
typedef struct {
    double dRSquare;
    double dContractionRatio;
    uint32_t nBitsNeeded;
} stat_info_t;
#include "seglrc_fit.inc"
}  // namespace seglrc

namespace lrc {
typedef struct {
    float fSlope;
    int iIntercept;
    float fSearchRange;
} regression_info_t;
typedef struct {
    double dRSquare;
    double dContractionRatio;
    uint32_t nBitsNeeded;
} stat_info_t;
#include "lrc_fit.inc"
}  // namespace lrc

extern "C" {
// out: {fSlope, fIntercept, nRangeLeft, nRangeRight} as raw 32-bit words
void ref_fit_seglrc(const uint32_t *y, uint32_t n, uint32_t *out) {
    seglrc::regression_info_t r;
    seglrc::stat_info_t s;
    memset(&r, 0, sizeof r);
    memset(&s, 0, sizeof s);
    seglrc::getRegressionInfo(y, n, r, s);
    memcpy(out, &r, 16);
}
// out: {fSlope, iIntercept, fSearchRange} as raw 32-bit words
void ref_fit_lrc(const uint32_t *y, uint32_t n, uint32_t *out) {
    lrc::regression_info_t r;
    lrc::stat_info_t s;
    memset(&r, 0, sizeof r);
    memset(&s, 0, sizeof s);
    lrc::getRegressionInfo(y, n, r, s);
    memcpy(out, &r, 12);
}
}
