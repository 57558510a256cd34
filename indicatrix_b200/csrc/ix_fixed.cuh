// ix_fixed.cuh -- adding a path's XYZ into exact fixed-point per-pixel sums (the
// path-pool loop, ix_pool.cu, and the wavefront pipeline, ix_wavefront.cu).  A pixel
// component's sum is three 64-bit words (t, a, b) worth t 2^24 + a 2^-16 + b 2^-56
// (ix_launch.h, FIXED_WORDS); ix_fixed.cu rounds them to f64 once.
#pragma once

#include "ix_launch.h"
#include "ix_transport.cuh"

namespace ix {

// Exact binary expansion of a sample component v (0 <= v < 2^62) in the fixed-point
// digits: v 2^56 = t 2^80 + a 2^40 + b with a, b < 2^40 (bits below 2^-56 truncated).
struct Digits {
    unsigned long long t, a, b;
};
IX_DEV Digits fixed_digits(float v) {
    const uint32_t bits = __float_as_uint(v) & 0x7FFFFFFFu;
    const int e = (int)(bits >> 23);
    Digits d{0ull, 0ull, 0ull};
    if (e == 0) return d;  // zero or subnormal: below the 2^-56 resolution
    const unsigned long long m = (bits & 0x7FFFFFu) | 0x800000u;  // v = m 2^(e - 150)
    const int s = e - 150 + 56;                                    // v 2^56 = m 2^s
    unsigned __int128 x;
    if (s >= 0)
        x = (unsigned __int128)m << s;
    else
        x = (s > -32) ? (unsigned __int128)(m >> (-s)) : (unsigned __int128)0;
    const unsigned long long M40 = (1ull << 40) - 1ull;
    d.b = (unsigned long long)x & M40;
    d.a = (unsigned long long)(x >> 40) & M40;
    d.t = (unsigned long long)(x >> 80);
    return d;
}

// add_finite_sample (optics/raytracer/sampling.rs:237) into fixed-point sums: a sample
// with a non-finite component (or one of 2^62 or more, beyond the sums' range) is dropped
// and counted; otherwise lanes 0-5 of the group each add one digit of X, Y or Z.
// Returns the drop this lane counts (lane 0 of the group).
IX_DEV uint32_t add_sample_fixed(const Group& g, unsigned long long* acc, V3 xyz) {
    const bool ok = isfinite(xyz.x) && isfinite(xyz.y) && isfinite(xyz.z) && xyz.x < FIXED_MAX_VALUE &&
                    xyz.y < FIXED_MAX_VALUE && xyz.z < FIXED_MAX_VALUE;
    if (!ok) return g.c == 0 ? 1u : 0u;
    if (g.c < 6) {
        const int comp = g.c >> 1;
        const float v = comp == 0 ? xyz.x : (comp == 1 ? xyz.y : xyz.z);
        const Digits d = fixed_digits(v);
        unsigned long long* w = acc + comp * 3;
        if (g.c & 1) {
            if (d.b) atomicAdd(w + 2, d.b);
        } else {
            if (d.a) atomicAdd(w + 1, d.a);
            if (d.t) atomicAdd(w, d.t);
        }
    }
    return 0u;
}

}  // namespace ix
