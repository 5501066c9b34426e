// fastdiv.cuh -- division of 32-bit unsigned integers by a runtime constant
// with one multiply-high and two shifts (Granlund & Montgomery, "Division by
// invariant integers using multiplication", PLDI 1994, round-up variant).
#pragma once

#include <cuda_runtime.h>

namespace psum_b200 {

struct FastDiv {
    unsigned d, m;
    int l;
};

inline FastDiv make_fastdiv(unsigned d) {
    FastDiv f{d, 0u, 0};
    int l = 0;
    while ((1ull << l) < d) ++l;
    f.l = l;
    f.m = d <= 1 ? 0u : (unsigned)((((1ull << l) - d) << 32) / d + 1);
    return f;
}

__device__ __forceinline__ unsigned fastdiv(unsigned n, const FastDiv& f) {
    if (f.d == 1) return n;
    const unsigned t = __umulhi(f.m, n);
    return (t + ((n - t) >> 1)) >> (f.l - 1);
}

}  // namespace psum_b200
