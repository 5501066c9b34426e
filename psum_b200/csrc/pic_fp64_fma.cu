// pic_fp64_fma.cu -- the contracted build of the FP64 particle kernels
// (pic_fp64_kernels.cuh), fused multiply-adds allowed: the FP64 comparison run.
#define PSUM_FP64_NS fp64_fma
#include "pic_fp64_kernels.cuh"
