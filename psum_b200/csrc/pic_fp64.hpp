// pic_fp64.hpp -- launchers of the FP64 particle kernels (pic_fp64.cu).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>

#include "pic_common.cuh"

namespace psum_b200 {

struct Push64Args {
    GridView g;
    double hi[3];
    double* pos[3];
    double* vel[3];
    int* key;
    const long long* count;
    const double* phi;
    double q_m, dt;
    int pusher;
    double B[3];
    unsigned long long* acc;   // null: no deposit
    double scale;
    unsigned long long* losses;
    unsigned* err;
    double* kin_part;   // per-block kinetic energy of the surviving particles (null: not summed)
    double kin_hmw;     // m * w / 2
    const double* grad; // non-null: the field's gradient at each particle, grad[d*n_upper + i] (the B-spline
                        // gather of a step with interp_order > 1), used instead of the CIC gather of phi
    long long grad_stride;
};

struct Deposit64Args {
    GridView g;
    const double* pos[3];
    const long long* count;
    unsigned long long* acc;
    double scale;
};

// Launchers of the two builds of pic_fp64_kernels.cuh: fp64_exact (no
// contraction, bit-exact with the oracle) and fp64_fma (contracted).
#define PSUM_FP64_LAUNCHERS                                                                                      \
    void launch_push64(const Push64Args& a, long long n_upper, cudaStream_t s);                                   \
    long long push64_blocks(long long n_upper); /* grid size of launch_push64 */                                  \
    void launch_deposit64(const Deposit64Args& a, long long n_upper, cudaStream_t s);                             \
    void launch_keys64(const GridView& g, double* const pos[3], int* key, const long long* count, long long n_upper, \
                       cudaStream_t s);
namespace fp64_exact {
PSUM_FP64_LAUNCHERS
}
namespace fp64_fma {
PSUM_FP64_LAUNCHERS
}
#undef PSUM_FP64_LAUNCHERS

}  // namespace psum_b200
