// Band codes of CAMBI's scale words (value | mask << 15), shared by the c-value and tile-proposal kernels.
#pragma once
#include "es_kernels.h"

namespace es {

// the distances d + 1 at which a code's c-value looks (src/kernels.cu:195-197): bit d
__host__ __device__ inline unsigned cvalue_dists(int code, const Band &bd)
{
    const int value = code + bd.band_base + kDiffs;
    unsigned m = 0;
    for (int d = 0; d < kDiffs; d++) m |= (unsigned)(value <= bd.tvi[d] && value + d + 1 > bd.vlt) << d;
    return m;
}
__device__ __forceinline__ bool needs_cvalue(int code, const Band &bd) { return cvalue_dists(code, bd) != 0; }

// The band code of a word: value - band_base for a masked value in the band, kNone otherwise.
__device__ __forceinline__ uint16_t code_of(unsigned word, const Band &bd)
{
    const unsigned u = (word & 0x7FFFu) - (unsigned)bd.band_base;
    return ((word & kMaskBit) && u < (unsigned)bd.band_size) ? (uint16_t)u : kNone;
}

}  // namespace es
