// pic_common.cuh -- device-side pieces shared by the particle kernels.
//
// Grid conventions follow PSuM's simple_grid<D> (src/field/simple_grid.hpp):
// node index last-dimension-fastest over (cells+1) nodes per axis.  The
// particle kernels additionally use an INTERNAL cell lattice per axis:
//   periodic axis : cells+1 cells (the node lattice wraps at cells+1 nodes,
//                   PSuM's wrapping-node idiom, application/benchmark/TSI/main.cpp:94);
//   absorbing axis: cells cells.
// A mixed-precision particle is (int32 internal cell key, FP32 in-cell
// offset per axis in [0,1), FP32 velocity); its CIC base node on each axis is
// the cell index itself (PSuM's cN, simple_grid.hpp:89-95).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fastdiv.cuh"

namespace psum_b200 {

void count_launch();   // registry.cpp: process-wide kernel launch counter

constexpr int kPicThreads = 256;

// device error word bits (one per psum_status code)
constexpr unsigned kErrNonFinite = 1u << 7;   // PSUM_ERR_NONFINITE
constexpr unsigned kErrOverflow = 1u << 6;    // PSUM_ERR_OVERFLOW
constexpr unsigned kErrKeyRange = 1u << 8;    // internal key out of range

// Unsigned division by a run-time invariant divisor d >= 1 with one
// multiply-high (Granlund & Montgomery, "Division by invariant integers
// using multiplication", PLDI 1994, Fig. 4.1): for l = ceil(log2 d) and
// m = floor(2^32 (2^l - d) / d) + 1, q = (t + ((n - t) >> 1)) >> (l - 1)
// with t = mulhi(m, n), exact for every 32-bit n.
struct GridView {
    int dim;
    int cells[3];     // PSuM cell counts (axis >= dim: 1)
    int M[3];         // internal cells per axis (axis >= dim: 1)
    int N[3];         // nodes per axis (axis >= dim: 1)
    int periodic[3];
    double lo[3], dx[3], dr[3];
    long long n_nodes;
    long long n_cells;   // internal cells
    FastDiv div_m12;     // by M[1]*M[2]
    FastDiv div_m2;      // by M[2]
};

__device__ __forceinline__ long long node_index(const GridView& g, int i, int j, int k) {
    return ((long long)i * g.N[1] + j) * g.N[2] + k;
}

__device__ __forceinline__ int next_node(const GridView& g, int a, int c) {
    const int n = c + 1;
    return n == g.N[a] ? 0 : n;   // only reachable on periodic axes
}

// Decompose an internal cell key (>= 0) into per-axis cell indices.
__device__ __forceinline__ void key_to_cell(const GridView& g, int key, int& c0, int& c1, int& c2) {
    c0 = (int)fastdiv((unsigned)key, g.div_m12);
    const int rem = key - c0 * (int)g.div_m12.d;
    c1 = (int)fastdiv((unsigned)rem, g.div_m2);
    c2 = rem - c1 * g.M[2];
}

__device__ __forceinline__ int cell_to_key(const GridView& g, int c0, int c1, int c2) {
    return (c0 * g.M[1] + c1) * g.M[2] + c2;
}

// Warp-level exact deposit of one CIC corner per lane: lanes holding the same
// node in consecutive lanes are summed with a segmented inclusive scan over
// int64 fixed-point values, and the last lane of each run issues one global
// integer atomic.  Integer addition is associative, so the accumulated value
// is independent of lane order, run boundaries and thread timing.
__device__ __forceinline__ void warp_deposit(unsigned long long* __restrict__ acc, long long node, long long val) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const long long prev = __shfl_up_sync(full, node, 1);
    const bool head = (lane == 0) || (prev != node);
    const unsigned heads = __ballot_sync(full, head);
    const unsigned le = (lane == 31) ? full : ((1u << (lane + 1)) - 1u);
    // index of this lane's segment head
    const int my_head = 31 - __clz(heads & le);
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const long long up = __shfl_up_sync(full, val, d);
        if (lane - d >= my_head) val += up;
    }
    const long long next = __shfl_down_sync(full, node, 1);
    const bool tail = (lane == 31) || (next != node);
    if (tail && node >= 0 && val != 0) atomicAdd(acc + node, (unsigned long long)val);
}

// Block sum of one FP64 value per thread in a fixed order (warp butterflies,
// then the warp totals in warp order), written by thread 0 to out[blockIdx.x].
// Every thread of the block calls it; blockDim.x is a multiple of 32, at most 1024.
__device__ __forceinline__ void block_sum_to(double v, double* __restrict__ out) {
    __shared__ double warp_tot[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();   // warp_tot may still be read by an earlier call
    if ((threadIdx.x & 31) == 0) warp_tot[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += warp_tot[w];
        out[blockIdx.x] = s;
    }
}

// Count per (axis, side) losses of a warp with one atomic per nonzero counter.
__device__ __forceinline__ void warp_count_losses(unsigned long long* losses, int dim, int lost_code) {
    // lost_code: -1 none, else axis*2+side
    const unsigned full = 0xffffffffu;
    for (int c = 0; c < 2 * dim; ++c) {
        const unsigned m = __ballot_sync(full, lost_code == c);
        if (m && (threadIdx.x & 31) == 0) atomicAdd(losses + c, (unsigned long long)__popc(m));
    }
}

}  // namespace psum_b200
