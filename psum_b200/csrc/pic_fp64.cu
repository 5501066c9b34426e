// pic_fp64.cu -- the bit-exact build of the FP64 particle kernels
// (pic_fp64_kernels.cuh), compiled with --fmad=false.
#define PSUM_FP64_NS fp64_exact
#include "pic_fp64_kernels.cuh"
