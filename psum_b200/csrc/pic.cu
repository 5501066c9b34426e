// pic.cu -- particle-kernel set of the B200 electrostatic PIC step and its C ABI
// (include/psum_pic.h).
//
// Mixed-precision step per species, one kernel: for every particle read the
// SoA state with 128-bit loads (4 particles per thread), gather E = -grad phi
// from FP32 edge differences of the FP64 potential, push (leapfrog or Boris),
// apply the particle boundary, and deposit the new position as exact
// fixed-point CIC weights.  Particles are kept sorted by cell with a stable
// LSD radix sort of the int32 cell key every `sort_interval` steps.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/psum_interp.h"
#include "../../include/psum_pic.h"
#include "common.hpp"
#include "mg_backend.hpp"
#include "pic.hpp"
#include "pic_fp64.hpp"

using psum_b200::DevBuf;
using psum_b200::Error;
using psum_b200::GridView;
using psum_b200::Species;
using psum_b200::cuda_check;

namespace psum_b200 {

namespace {

inline unsigned blocks_for(long long n, int threads) {
    return (unsigned)std::max<long long>(1, (n + threads - 1) / threads);
}
inline unsigned capped_blocks(long long n_items_per_block_unit, long long n) {
    const long long b = (n + n_items_per_block_unit - 1) / n_items_per_block_unit;
    return (unsigned)std::max<long long>(1, std::min<long long>(b, 148LL * 32));
}

// ------------------------------------------------------------ edge field --
// edges[node*S + a] = phi(node + e_a) - phi(node) in FP64, stored as FP32
// (S = 2 in 2-D, 4 in 3-D).  The CIC gradient of PSuM's interp_diff
// (simple_interpolation.hpp:58-98) is a bilinear/trilinear blend of exactly
// these differences, so the FP32 gather loses no precision to cancellation.
// With fe_part set, each block also writes the sum over its nodes of
// sum_a ((phi(n + e_a) - phi(n)) * dr_a)^2 in FP64 (the field-energy terms of
// TSI/main.cpp:141-143, periodic edges included) to fe_part[blockIdx.x].
template <int D>
__global__ void k_edges(GridView g, const double* __restrict__ phi, float* __restrict__ edges,
                        double* __restrict__ fe_part) {
    const long long node = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double fe = 0.0;
    if (node < g.n_nodes) {
        const int n12 = g.N[1] * g.N[2];
        const int i = (int)(node / n12);
        const int rem = (int)(node - (long long)i * n12);
        const int j = rem / g.N[2];
        const int k = rem - j * g.N[2];
        const double p0 = phi[node];
        float e[4] = {0.f, 0.f, 0.f, 0.f};
        const int idx[3] = {i, j, k};
        for (int a = 0; a < D; ++a) {
            int q[3] = {idx[0], idx[1], idx[2]};
            q[a] += 1;
            if (q[a] >= g.N[a]) {
                if (!g.periodic[a]) continue;
                q[a] = 0;
            }
            const double dphi = phi[node_index(g, q[0], q[1], q[2])] - p0;
            e[a] = (float)dphi;
            const double gr = dphi * g.dr[a];
            fe += gr * gr;
        }
        if (edges) {
            if (D <= 2) reinterpret_cast<float2*>(edges)[node] = make_float2(e[0], e[1]);
            else reinterpret_cast<float4*>(edges)[node] = make_float4(e[0], e[1], e[2], 0.f);
        }
    }
    if (fe_part) block_sum_to(fe, fe_part);
}

// ------------------------------------------------------------ mixed push --
struct PushArgs {
    GridView g;
    int* key;
    float* off[3];
    float* vel[3];
    const long long* count;
    const float* edges;
    float kE[3];        // q/m * dt * dr_a  (velocity kick per unit edge difference)
    float dtdr[3];      // dt * dr_a        (offset change per unit velocity)
    float qmdt_half;    // q/m * dt / 2 (Boris)
    float Bt[3];        // B * q/m * dt / 2 (Boris t vector)
    float dr[3];
    unsigned long long* acc;
    int dep_lsh;        // accumulator units per 2^-26 weight unit: 2^dep_lsh
    unsigned long long* losses;
    unsigned* err;
    double* kin_part;   // per-block kinetic energy of the pushed particles (null: not summed)
    double kin_hmw;     // m * w / 2
};

// Field data of one cell for the CIC gather of the edge differences: the
// components that interpolate G_a over the cell (G_a lives on the edges along
// axis a, so it varies with the other axes' offsets only).
template <int D>
struct CellField {
    float e[D == 1 ? 1 : (D == 2 ? 4 : 12)];
};

template <int D>
__device__ __forceinline__ void load_cell_field(const PushArgs& a, int c0, int c1, int c2, CellField<D>& F) {
    const GridView& g = a.g;
    if constexpr (D == 1) {
        // 1-D: the CIC gradient is the cell's one edge difference (constant in the cell)
        F.e[0] = __ldg(reinterpret_cast<const float2*>(a.edges) + c0).x;
        (void)c1;
        (void)c2;
    } else if constexpr (D == 2) {
        const float2* E = reinterpret_cast<const float2*>(a.edges);
        const int n0p = next_node(g, 0, c0), n1p = next_node(g, 1, c1);
        const float2 e00 = __ldg(E + node_index(g, c0, c1, 0));
        const float2 e01 = __ldg(E + node_index(g, c0, n1p, 0));
        const float2 e10 = __ldg(E + node_index(g, n0p, c1, 0));
        F.e[0] = e00.x;
        F.e[1] = e01.x;
        F.e[2] = e00.y;
        F.e[3] = e10.y;
    } else {
        const float4* E = reinterpret_cast<const float4*>(a.edges);
        const int n0p = next_node(g, 0, c0), n1p = next_node(g, 1, c1), n2p = next_node(g, 2, c2);
        const float4 e000 = __ldg(E + node_index(g, c0, c1, c2));
        const float4 e001 = __ldg(E + node_index(g, c0, c1, n2p));
        const float4 e010 = __ldg(E + node_index(g, c0, n1p, c2));
        const float4 e011 = __ldg(E + node_index(g, c0, n1p, n2p));
        const float4 e100 = __ldg(E + node_index(g, n0p, c1, c2));
        const float4 e101 = __ldg(E + node_index(g, n0p, c1, n2p));
        const float4 e110 = __ldg(E + node_index(g, n0p, n1p, c2));
        F.e[0] = e000.x; F.e[1] = e001.x; F.e[2] = e010.x; F.e[3] = e011.x;
        F.e[4] = e000.y; F.e[5] = e001.y; F.e[6] = e100.y; F.e[7] = e101.y;
        F.e[8] = e000.z; F.e[9] = e010.z; F.e[10] = e100.z; F.e[11] = e110.z;
    }
}

template <int D>
__device__ __forceinline__ void interp_grad(const CellField<D>& F, const float f[3], float G[3]) {
#define PSUM_LERP(a_, wa_, b_, wb_) __fmaf_rn((b_), (wb_), __fmul_rn((a_), (wa_)))
    if constexpr (D == 1) {
        G[0] = F.e[0];
        G[1] = G[2] = 0.f;
        (void)f;
    } else if constexpr (D == 2) {
        G[0] = PSUM_LERP(F.e[0], __fsub_rn(1.f, f[1]), F.e[1], f[1]);
        G[1] = PSUM_LERP(F.e[2], __fsub_rn(1.f, f[0]), F.e[3], f[0]);
        G[2] = 0.f;
    } else {
        const float g0 = __fsub_rn(1.f, f[0]), g1 = __fsub_rn(1.f, f[1]), g2 = __fsub_rn(1.f, f[2]);
        G[0] = PSUM_LERP(PSUM_LERP(F.e[0], g2, F.e[1], f[2]), g1, PSUM_LERP(F.e[2], g2, F.e[3], f[2]), f[1]);
        G[1] = PSUM_LERP(PSUM_LERP(F.e[4], g2, F.e[5], f[2]), g0, PSUM_LERP(F.e[6], g2, F.e[7], f[2]), f[0]);
        G[2] = PSUM_LERP(PSUM_LERP(F.e[8], g1, F.e[9], f[1]), g0, PSUM_LERP(F.e[10], g1, F.e[11], f[1]), f[0]);
    }
#undef PSUM_LERP
}

// Velocity update from the gathered edge differences G, then the move in
// cell units.  f holds the new in-cell offsets and dc the cell steps per axis
// on exit (offset carry rule: an offset that rounds to 1.0f moves to the next
// cell with offset 0).  Every operation is an explicit round-to-nearest
// intrinsic (fused multiply-adds where written), so every kernel that calls
// this function moves the same particle bit-identically.  False when the
// state became non-finite (kick_move flags the error word; kick_move_core
// leaves that to its caller).
template <int D, int PUSHER>
__device__ __forceinline__ bool kick_move_core(const PushArgs& a, const float G[3], float f[3], float v[3], int dc[3]) {
    if (PUSHER == PSUM_PIC_LEAPFROG) {
#pragma unroll
        for (int d = 0; d < D; ++d) v[d] = __fmaf_rn(-a.kE[d], G[d], v[d]);   // v += (q/m) E dt, E = -dr G
    } else {
        float E[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for (int d = 0; d < D; ++d) E[d] = -__fmul_rn(a.dr[d], G[d]);
        float vm[3], vp[3], vq[3], s[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) vm[q] = __fadd_rn(v[q], __fmul_rn(E[q], a.qmdt_half));
        const float t2 = __fadd_rn(__fadd_rn(__fmul_rn(a.Bt[0], a.Bt[0]), __fmul_rn(a.Bt[1], a.Bt[1])),
                                   __fmul_rn(a.Bt[2], a.Bt[2]));
#pragma unroll
        for (int q = 0; q < 3; ++q) s[q] = __fdiv_rn(__fmul_rn(2.f, a.Bt[q]), __fadd_rn(1.f, t2));
#define PSUM_CROSS(x1, y1, x2, y2) __fsub_rn(__fmul_rn((x1), (y1)), __fmul_rn((x2), (y2)))
        vq[0] = __fadd_rn(vm[0], PSUM_CROSS(vm[1], a.Bt[2], vm[2], a.Bt[1]));
        vq[1] = __fadd_rn(vm[1], PSUM_CROSS(vm[2], a.Bt[0], vm[0], a.Bt[2]));
        vq[2] = __fadd_rn(vm[2], PSUM_CROSS(vm[0], a.Bt[1], vm[1], a.Bt[0]));
        vp[0] = __fadd_rn(vm[0], PSUM_CROSS(vq[1], s[2], vq[2], s[1]));
        vp[1] = __fadd_rn(vm[1], PSUM_CROSS(vq[2], s[0], vq[0], s[2]));
        vp[2] = __fadd_rn(vm[2], PSUM_CROSS(vq[0], s[1], vq[1], s[0]));
#undef PSUM_CROSS
#pragma unroll
        for (int q = 0; q < 3; ++q) v[q] = __fadd_rn(vp[q], __fmul_rn(E[q], a.qmdt_half));
    }
    bool ok = true;
#pragma unroll
    for (int d = 0; d < D; ++d) {
        const float sd = __fmaf_rn(v[d], a.dtdr[d], f[d]);
        ok = ok && fabsf(sd) < 1.0e9f;   // false for NaN and infinities too
        const float fl = floorf(sd);
        float nf = __fsub_rn(sd, fl);
        int step = (int)fl;
        if (nf >= 1.0f) {
            nf = 0.0f;
            step += 1;
        }
        f[d] = nf;
        dc[d] = step;
    }
    return ok;
}

template <int D, int PUSHER>
__device__ __forceinline__ bool kick_move(const PushArgs& a, const float G[3], float f[3], float v[3], int dc[3]) {
    const bool ok = kick_move_core<D, PUSHER>(a, G, f, v, dc);
    if (!ok) atomicOr(a.err, kErrNonFinite);
    return ok;
}

// Wrap periodic axes and test absorbing ones after c += dc.  Returns the loss
// code (axis*2+side) of the first absorbing axis left, or -1.
template <int D>
__device__ __forceinline__ int apply_step(const GridView& g, int c[3], const int dc[3]) {
    int lost = -1;
#pragma unroll
    for (int d = 0; d < D; ++d) {
        c[d] += dc[d];
        if (g.periodic[d]) {
            if (c[d] < 0 || c[d] >= g.M[d]) {
                c[d] %= g.M[d];
                if (c[d] < 0) c[d] += g.M[d];
            }
        } else if (lost < 0) {
            if (c[d] < 0) lost = 2 * d;
            else if (c[d] >= g.cells[d]) lost = 2 * d + 1;
        }
    }
    return lost;
}

// One particle: gather, push, boundary.  c[] holds the cell on entry and the
// new cell on exit.  Returns the loss code (axis*2+side), -1 when the
// particle stays, or -2 when its state became non-finite.
template <int D, int PUSHER>
__device__ __forceinline__ int push_one(const PushArgs& a, int c[3], float f[3], float v[3]) {
    CellField<D> F;
    load_cell_field<D>(a, c[0], c[1], c[2], F);
    float G[3];
    interp_grad<D>(F, f, G);
    int dc[3] = {0, 0, 0};
    if (!kick_move<D, PUSHER>(a, G, f, v, dc)) return -2;
    return apply_step<D>(a.g, c, dc);
}

// |v|^2 of FP32 velocities, summed in FP64 (the terms of TSI/main.cpp:133-136)
__device__ __forceinline__ double kinetic_v2(const float v[3]) {
    const double x = v[0], y = v[1], z = v[2];
    return x * x + y * y + z * z;
}

// ------------------------------------------------ quantised CIC weights --
// Every mixed-precision deposit uses integer CIC weights on a 2^-26 grid,
// built from quantised moments of the in-cell offsets, indexed by axis set m
// (bit a = axis a):
//   Q_0 = 2^26,  Q_m = rint(2^26 * prod_{a in m} f_a)  (FP32 products, left to right).
// The corner whose upper axes form the set B gets the inclusion-exclusion sum
//   w_B = sum_{T superset of B} (-1)^{|T|-|B|} Q_T,
// the exact expansion of prod_{a in B} f_a * prod_{a not in B} (1 - f_a) with
// every product replaced by its quantised moment.  A particle's weights sum
// to exactly 2^26 and each lies within 2^(D-2) * 2^-26 of the CIC weight of
// its FP32 offsets.  The map from moments to weights is linear, so a group of
// particles sums its moments (exact integers) and forms the corner sums
// once: the deposit is exact and independent of grouping and order.
constexpr int kCicBits = 26;
constexpr float kCicScale = 67108864.0f;   // 2^26

template <int D>
__device__ __forceinline__ void cic_moments(const float f[3], unsigned q[8]) {
    q[0] = 1u << kCicBits;
    q[1] = __float2uint_rn(__fmul_rn(f[0], kCicScale));
    if (D == 1) return;
    q[2] = __float2uint_rn(__fmul_rn(f[1], kCicScale));
    const float f01 = __fmul_rn(f[0], f[1]);
    q[3] = __float2uint_rn(__fmul_rn(f01, kCicScale));
    if (D == 3) {
        q[4] = __float2uint_rn(__fmul_rn(f[2], kCicScale));
        q[5] = __float2uint_rn(__fmul_rn(__fmul_rn(f[0], f[2]), kCicScale));
        q[6] = __float2uint_rn(__fmul_rn(__fmul_rn(f[1], f[2]), kCicScale));
        q[7] = __float2uint_rn(__fmul_rn(__fmul_rn(f01, f[2]), kCicScale));
    }
}

// Corner weight of upper-axis set B from (group sums of) the moments S[m].
template <int D>
__device__ __forceinline__ long long cic_corner(const long long S[8], int B) {
    long long w = 0;
#pragma unroll
    for (int T = 0; T < (1 << D); ++T)
        if ((T & B) == B) w += (__popc(T ^ B) & 1) ? -S[T] : S[T];
    return w;
}

// Node of corner B of cell c (wrapping on periodic axes).
template <int D>
__device__ __forceinline__ void corner_node(const GridView& g, int B, const int c[3], int n[3]) {
    n[0] = (B & 1) ? next_node(g, 0, c[0]) : c[0];
    n[1] = (B & 2) ? next_node(g, 1, c[1]) : c[1];
    n[2] = (D == 3) ? ((B & 4) ? next_node(g, 2, c[2]) : c[2]) : 0;
}

// 4 particles per thread, 128-bit loads/stores of every SoA array.  The
// deposit first sums, per CIC corner, the lane's particles that share the
// lane's first node (consecutive particles are usually in one cell because
// the arrays are sorted by cell), then runs one warp segmented scan per
// corner; the rare other nodes take a direct integer atomic.
template <int D, int PUSHER, bool DEPOSIT_ONLY>
__global__ void __launch_bounds__(kPicThreads) k_push_mixed(PushArgs a) {
    const long long count = *a.count;
    const int lane = threadIdx.x & 31;
    const long long stride = (long long)gridDim.x * blockDim.x * 4;
    unsigned lost_cnt[2 * D];
#pragma unroll
    for (int q = 0; q < 2 * D; ++q) lost_cnt[q] = 0u;
    double kin = 0.0;
    for (long long base = ((long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31)) * 4; base < count;
         base += stride) {
        const long long i0 = base + 4 * lane;
        int key[4];
        float f[4][3], v[4][3];
        int cell[4][3];
        const bool full = i0 + 3 < count;
        if (full) {
            const int4 k4 = *reinterpret_cast<const int4*>(a.key + i0);
            key[0] = k4.x; key[1] = k4.y; key[2] = k4.z; key[3] = k4.w;
#pragma unroll
            for (int d = 0; d < D; ++d) {
                const float4 t = *reinterpret_cast<const float4*>(a.off[d] + i0);
                f[0][d] = t.x; f[1][d] = t.y; f[2][d] = t.z; f[3][d] = t.w;
            }
            if (!DEPOSIT_ONLY) {
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    const float4 t = *reinterpret_cast<const float4*>(a.vel[q] + i0);
                    v[0][q] = t.x; v[1][q] = t.y; v[2][q] = t.z; v[3][q] = t.w;
                }
            }
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const long long i = i0 + j;
                key[j] = i < count ? a.key[i] : -1;
#pragma unroll
                for (int d = 0; d < D; ++d) f[j][d] = i < count ? a.off[d][i] : 0.f;
                if (!DEPOSIT_ONLY)
#pragma unroll
                    for (int q = 0; q < 3; ++q) v[j][q] = i < count ? a.vel[q][i] : 0.f;
            }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
#pragma unroll
            for (int d = D; d < 3; ++d) f[j][d] = 0.f;
            cell[j][0] = cell[j][1] = cell[j][2] = 0;
            if (key[j] < 0) continue;
            key_to_cell(a.g, key[j], cell[j][0], cell[j][1], cell[j][2]);
            if (!DEPOSIT_ONLY) {
                const int lost = push_one<D, PUSHER>(a, cell[j], f[j], v[j]);
                if (lost >= 0) {
#pragma unroll
                    for (int q = 0; q < 2 * D; ++q) lost_cnt[q] += (lost == q);
                }
                key[j] = lost == -1 ? cell_to_key(a.g, cell[j][0], cell[j][1], cell[j][2]) : -1;
                if (a.kin_part && key[j] >= 0) kin += a.kin_hmw * kinetic_v2(v[j]);
            }
        }
        if (a.acc) {
            unsigned q[4][8];
#pragma unroll
            for (int j = 0; j < 4; ++j) cic_moments<D>(f[j], q[j]);
#pragma unroll
            for (int k = 0; k < (1 << D); ++k) {
                long long node0 = -1, sum = 0;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    if (key[j] < 0) continue;
                    long long S[8];
#pragma unroll
                    for (int m = 0; m < (1 << D); ++m) S[m] = q[j][m];
                    const long long val = (long long)((unsigned long long)cic_corner<D>(S, k) << a.dep_lsh);
                    int nd[3];
                    corner_node<D>(a.g, k, cell[j], nd);
                    const long long node = node_index(a.g, nd[0], nd[1], nd[2]);
                    if (node0 < 0) {
                        node0 = node;
                        sum = val;
                    } else if (node == node0) {
                        sum += val;
                    } else if (val != 0) {
                        atomicAdd(a.acc + node, (unsigned long long)val);
                    }
                }
                warp_deposit(a.acc, node0, sum);
            }
        }
        if (DEPOSIT_ONLY) continue;
        if (full) {
            *reinterpret_cast<int4*>(a.key + i0) = make_int4(key[0], key[1], key[2], key[3]);
#pragma unroll
            for (int d = 0; d < D; ++d)
                *reinterpret_cast<float4*>(a.off[d] + i0) = make_float4(f[0][d], f[1][d], f[2][d], f[3][d]);
#pragma unroll
            for (int q = 0; q < 3; ++q)
                *reinterpret_cast<float4*>(a.vel[q] + i0) = make_float4(v[0][q], v[1][q], v[2][q], v[3][q]);
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const long long i = i0 + j;
                if (i >= count) break;
                a.key[i] = key[j];
#pragma unroll
                for (int d = 0; d < D; ++d) a.off[d][i] = f[j][d];
#pragma unroll
                for (int q = 0; q < 3; ++q) a.vel[q][i] = v[j][q];
            }
        }
    }
    if (!DEPOSIT_ONLY) {
        // per-thread loss counters -> one integer atomic per warp and counter
#pragma unroll
        for (int q = 0; q < 2 * D; ++q) {
            unsigned t = lost_cnt[q];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
            if (lane == 0 && t) atomicAdd(a.losses + q, (unsigned long long)t);
        }
        if (a.kin_part) block_sum_to(kin, a.kin_part);
    }
}

// ------------------------------------------------ fused sorted step ------
//
// With the state sorted by cell, a particle can only move to one of the 3^D
// neighbour cells (or further, or out).  Pass 1 pushes every particle without
// writing it, counts particles per (old cell, move class) and deposits the
// new positions.  The offsets kernel turns the class counts into, per new
// cell, its particle count and the offset of every (source cell, class)
// group inside it; groups are ordered by source cell index, which is the
// order of the old positions.  After the exclusive scan of the new counts,
// pass 2 pushes again (bit-identical: every operation is an explicit rounding
// intrinsic) and writes particle i of a group to
//   new_start[new cell] + group offset + (rank of i within its group)
// in the other state buffer.  The result is exactly the stable sort by new
// cell of the pushed state, with absorbed particles removed: what the general
// path (push in place, stable radix sort) produces.
//
// A block owns the cells whose weighted start (first particle index + the
// cell index times T / 2048) lies in [b*T, (b+1)*T) (table from
// k_cls_blocks): at most T particles plus one cell and at most about 2048
// cells, so long runs of empty cells are spread over many blocks.  Each
// cell goes to one warp,
// so ranks and counts need no cross-warp synchronisation.  The pass-1
// deposit sums the quantised CIC moments of the particles of one (cell,
// class) group with warp reductions, forms the 2^D corner sums once per group
// and cell, and adds them to a block node tile in shared memory that is
// flushed with one integer atomic per touched node.
constexpr int kClsWarps = kPicThreads / 32;
constexpr int kClsTileMax = 3072;   // int64 node accumulators in shared memory (24 KB)
// Rounds of 32 particles per warp iteration (all loads issued first): 4, or
// 1 for species with few particles per cell (empty rounds cost a cell's
// whole iteration there).
constexpr int kClsRoundsMax = 4;
constexpr int cls_rounds(double particles_per_cell) { return particles_per_cell < 64.0 ? 1 : kClsRoundsMax; }

// Particles per block: 2D blocks cover a few tens of cells of one row; 3D
// blocks stay short enough that their node box usually fits the tile, and
// their tiles small enough for six blocks per SM.
__host__ __device__ constexpr int cls_block_lg(int dim) { return dim == 2 ? 13 : 10; }
// Second-pass blocks are short (no node tile to amortise), so that a pending
// second pass frees SM slots often for the higher-priority work beside it.
__host__ __device__ constexpr int cls_block_lg2(int) { return 11; }
// weight of a cell in the block table, in particles (at most 2048 cells per
// block; blocks of fewer than 2048 particles weigh every cell 1)
__host__ __device__ constexpr long long cls_cell_weight(int lgT) { return lgT >= 11 ? 1LL << (lgT - 11) : 1LL; }

template <int D>
struct MoveClasses {
    static constexpr int N = D == 2 ? 9 : 27;
    static constexpr int STAY = (N - 1) / 2;   // class of the particles that keep their cell
};

struct ClsArgs {
    PushArgs p;                   // current state, fields, deposit, losses, error word
    const unsigned* starts;       // n_cells + 1 cell offsets of the current state
    const unsigned* block_first;  // first cell of each block (k_cls_blocks)
    unsigned* cls;                // [class][cell]: counts (pass 1), then group offsets (pass 2);
                                  // class-major so that k_cls_offsets reads every class coalesced
    const unsigned* new_starts;   // n_cells + 1 offsets of the new state (pass 2)
    int* far;                     // pass 1: 1 when a particle moved more than one cell on an axis
    float* off_out[3];            // new state (its keys follow from new_starts)
    float* vel_out[3];
    long long n_cells;
};

// Per-axis step of move class d: digits (step_a + 1) in base 3, axis 0 most
// significant.
template <int D>
__device__ __forceinline__ int class_delta(int d, int a) {
    if (D == 2) return a == 0 ? d / 3 - 1 : d % 3 - 1;
    return a == 0 ? d / 9 - 1 : (a == 1 ? (d / 3) % 3 - 1 : d % 3 - 1);
}

// Cell reached from cell c by class d; false when it leaves an absorbing axis.
template <int D>
__device__ __forceinline__ bool class_target(const GridView& g, const int c[3], int d, int out[3]) {
    out[0] = c[0];
    out[1] = c[1];
    out[2] = c[2];
#pragma unroll
    for (int a = 0; a < D; ++a) {
        int x = c[a] + class_delta<D>(d, a);
        if (x < 0 || x >= g.M[a]) {
            if (!g.periodic[a]) return false;
            x = x < 0 ? x + g.M[a] : x - g.M[a];
        }
        out[a] = x;
    }
    return true;
}

// Block -> first owned cell: first[b] = lower bound of b*T in the weighted
// starts w(c) = starts[c] + c * cls_cell_weight(lgT), clamped to n_cells;
// entries 0..nb.  (T = 2^lgT.)
__global__ void k_cls_blocks(const unsigned* __restrict__ starts, long long n_cells, long long nb, int lgT,
                             unsigned* __restrict__ first) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long wc = cls_cell_weight(lgT);
    if (t <= n_cells) {
        const long long hi = ((long long)starts[t] + t * wc) >> lgT;
        for (long long b = t == 0 ? 0 : (((long long)starts[t - 1] + (t - 1) * wc) >> lgT) + 1; b <= hi && b <= nb; ++b)
            first[b] = (unsigned)t;
    }
    if (t <= nb && (t << lgT) > (long long)starts[n_cells] + n_cells * wc) first[t] = (unsigned)n_cells;
}

struct NodeTile {
    int lo[3], ext[3];
    int on;
    int vol;
};

// Cells a block's deposit may reach (its cells +-1 on every axis, the reach
// of a one-cell move; for a block spanning several rows the full rows),
// clamped to the cell lattice, and the nodes of those cells.  Targets across
// a periodic seam and boxes above the tile capacities take the direct
// global path.
template <int D>
__device__ void deposit_boxes(const GridView& g, long long ca, long long cb, int cell_cap, int node_cap, NodeTile& ct,
                              NodeTile& nt) {
    ct.on = nt.on = 0;
    ct.vol = nt.vol = 0;
    if (ca >= cb) return;
    int a[3], b[3];
    key_to_cell(g, (int)ca, a[0], a[1], a[2]);
    key_to_cell(g, (int)(cb - 1), b[0], b[1], b[2]);
    int lo[3], hi[3];
    for (int q = 0; q < 3; ++q) {
        lo[q] = 0;
        hi[q] = g.M[q] - 1;
    }
    lo[0] = a[0];
    hi[0] = b[0];
    if (a[0] == b[0]) {
        lo[1] = a[1];
        hi[1] = b[1];
        if (D == 3 && a[1] == b[1]) {
            lo[2] = a[2];
            hi[2] = b[2];
        }
    }
    long long cvol = 1, nvol = 1;
    for (int q = 0; q < 3; ++q) {
        if (q < D) {
            ct.lo[q] = nt.lo[q] = max(lo[q] - 1, 0);
            ct.ext[q] = min(hi[q] + 1, g.M[q] - 1) - ct.lo[q] + 1;
            nt.ext[q] = min(ct.lo[q] + ct.ext[q], g.N[q] - 1) - nt.lo[q] + 1;
        } else {
            ct.lo[q] = nt.lo[q] = 0;
            ct.ext[q] = nt.ext[q] = 1;
        }
        cvol *= ct.ext[q];
        nvol *= nt.ext[q];
    }
    ct.on = cvol <= cell_cap;
    ct.vol = ct.on ? (int)cvol : 0;
    nt.on = ct.on && nvol <= node_cap;
    nt.vol = nt.on ? (int)nvol : 0;
}

// Slot of cell c in a box, or -1 outside it.
__device__ __forceinline__ int box_slot(const NodeTile& t, const int c[3]) {
    const int i = c[0] - t.lo[0], j = c[1] - t.lo[1], k = c[2] - t.lo[2];
    if (!t.on || (unsigned)i >= (unsigned)t.ext[0] || (unsigned)j >= (unsigned)t.ext[1] || (unsigned)k >= (unsigned)t.ext[2])
        return -1;
    return (i * t.ext[1] + j) * t.ext[2] + k;
}

// Corners of moment sums W (W[0] = count * 2^26) of cell c straight into the
// node accumulators.
template <int D>
__device__ __forceinline__ void deposit_direct(const PushArgs& a, const int c[3], const long long W[8]) {
#pragma unroll
    for (int B = 0; B < (1 << D); ++B) {
        const long long w = cic_corner<D>(W, B);
        if (w == 0) continue;
        int nd[3];
        corner_node<D>(a.g, B, c, nd);
        atomicAdd(a.acc + node_index(a.g, nd[0], nd[1], nd[2]), (unsigned long long)w << a.dep_lsh);
    }
}

// Push of one particle of cell co with the warp's cell field: move class
// (>= 0), -1 far (more than one cell on some axis), -3 absorbed or
// non-finite (loss counted).  cn is the new cell for far particles.
template <int D, int PUSHER>
__device__ __forceinline__ int push_classify(const PushArgs& a, const CellField<D>& F, const int co[3], float f[3],
                                             float v[3], int cn[3], unsigned lost_cnt[2 * D]) {
    float G[3];
    interp_grad<D>(F, f, G);
    int dc[3] = {0, 0, 0};
    const bool ok = kick_move_core<D, PUSHER>(a, G, f, v, dc);
    // common path: the new cell lies inside the lattice on every axis (one
    // unsigned test per axis); wrapping, losses and non-finite states take
    // the rare path, which follows kick_move and apply_step exactly
    const GridView& g = a.g;
    bool out = false;
    cn[2] = co[2];
#pragma unroll
    for (int d = 0; d < D; ++d) {
        cn[d] = co[d] + dc[d];
        out |= (unsigned)cn[d] >= (unsigned)(g.periodic[d] ? g.M[d] : g.cells[d]);
    }
    if (!ok || out) {
        if (!ok) {
            atomicOr(a.err, kErrNonFinite);
            return -3;
        }
        cn[0] = co[0];
        cn[1] = co[1];
        cn[2] = co[2];
        const int lost = apply_step<D>(g, cn, dc);
        if (lost >= 0) {
#pragma unroll
            for (int q = 0; q < 2 * D; ++q) lost_cnt[q] += (lost == q);
            return -3;
        }
    }
    int cls = 0;
    bool far = false;
#pragma unroll
    for (int d = 0; d < D; ++d) {
        far |= (unsigned)(dc[d] + 1) > 2u;
        cls = cls * 3 + dc[d] + 1;
    }
    return far ? -1 : cls;
}

// Exact warp sum of per-lane values below 2^32 (two reductions of 26-bit
// and 6-bit parts).
__device__ __forceinline__ unsigned long long warp_sum_u32(unsigned v) {
    const unsigned lo = __reduce_add_sync(0xffffffffu, v & ((1u << kCicBits) - 1u));
    const unsigned hi = __reduce_add_sync(0xffffffffu, v >> kCicBits);
    return (unsigned long long)lo + ((unsigned long long)hi << kCicBits);
}

// 64-bit shared-memory accumulators kept as 32-bit low/high words: native
// 32-bit atomics, the carry out of the low word goes to the high word, so the
// pair holds the exact sum modulo 2^64 once all adds are done.
__device__ __forceinline__ void smem_add64(unsigned* lo, unsigned* hi, unsigned long long v) {
    const unsigned vl = (unsigned)v, vh = (unsigned)(v >> 32);
    const unsigned old = atomicAdd(lo, vl);
    const unsigned up = vh + (old + vl < old ? 1u : 0u);
    if (up) atomicAdd(hi, up);
}

__device__ __forceinline__ unsigned long long pair64(unsigned lo, unsigned hi) {
    return (unsigned long long)lo | ((unsigned long long)hi << 32);
}

// Cells of the pass-1 moment tile and nodes of its node tile: the boxes of a
// 2D block (one row segment +-1: up to 3 x 170 cells) and of a 3D block (a z-run +-1 in x and y;
// 1024 particles at 32 per cell span 32 cells: 3 x 3 x 34 cells, 4 x 4 x 35
// nodes).  The tiles live in dynamic shared memory.
template <int D>
struct CellTileCap {
    static constexpr int N = D == 2 ? 512 : 320;
    static constexpr int NODES = D == 2 ? kClsTileMax : 576;
    // dynamic shared memory of pass 1: cell counts, moment low/high words, node tile
    static constexpr size_t BYTES = sizeof(unsigned) * ((size_t)N * (1 + 2 * ((1 << D) - 1)) + 2 * (size_t)NODES);
};


template <int D, int PUSHER, int kClsRounds>
__global__ void __launch_bounds__(kPicThreads) k_cls_pass1(ClsArgs a) {
    constexpr int NC = MoveClasses<D>::N;
    constexpr int STAY = MoveClasses<D>::STAY;
    constexpr int NM = 1 << D;
    constexpr int CT = CellTileCap<D>::N;
    constexpr int NT = CellTileCap<D>::NODES;
    // per (warp, moment, class): count (moment 0, low word only) and moment
    // sums of the warp's current cell; per cell of the block's box the count
    // and moment sums (units of 2^-26) of the particles that end there; the
    // box's node tile
    __shared__ unsigned mom_lo[kClsWarps][NM][NC], mom_hi[kClsWarps][NM][NC];
    __shared__ NodeTile cbox, nbox;
    extern __shared__ __align__(16) unsigned dsm[];
    unsigned* const ct_n = dsm;                             // [CT]
    unsigned(*const ct_lo)[CT] = reinterpret_cast<unsigned(*)[CT]>(dsm + CT);   // [NM - 1][CT]
    unsigned(*const ct_hi)[CT] = reinterpret_cast<unsigned(*)[CT]>(dsm + CT + (NM - 1) * CT);
    unsigned* const tile_lo = dsm + CT + 2 * (NM - 1) * CT;  // [NT]
    unsigned* const tile_hi = tile_lo + NT;
    const long long ca = a.block_first[blockIdx.x], cb = a.block_first[blockIdx.x + 1];
    if (ca >= cb) return;
    const GridView& g = a.p.g;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned full = 0xffffffffu;
    if (threadIdx.x == 0) deposit_boxes<D>(g, ca, cb, CT, NT, cbox, nbox);
    for (int q = threadIdx.x; q < kClsWarps * NM * NC; q += blockDim.x) {
        (&mom_lo[0][0][0])[q] = 0u;
        (&mom_hi[0][0][0])[q] = 0u;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < cbox.vol; q += blockDim.x) {
        ct_n[q] = 0u;
#pragma unroll
        for (int m = 0; m < NM - 1; ++m) ct_lo[m][q] = ct_hi[m][q] = 0u;
    }
    for (int q = threadIdx.x; q < nbox.vol; q += blockDim.x) tile_lo[q] = tile_hi[q] = 0u;
    __syncthreads();
    unsigned lost_cnt[2 * D];
#pragma unroll
    for (int q = 0; q < 2 * D; ++q) lost_cnt[q] = 0u;
    bool far_seen = false;
    for (long long c = ca + warp; c < cb; c += kClsWarps) {
        const long long p0 = a.starts[c], p1 = a.starts[c + 1];
        int co[3];
        key_to_cell(g, (int)c, co[0], co[1], co[2]);
        if (p1 > p0) {
            CellField<D> F;
            load_cell_field<D>(a.p, co[0], co[1], co[2], F);
            // particles that keep their cell: per-lane count and moment sums
            // (at most 2^31 over 32 rounds), reduced over the warp every 32 rounds
            unsigned sacc[NM];
#pragma unroll
            for (int m = 0; m < NM; ++m) sacc[m] = 0u;
            int pending = 0;
            for (long long base = p0; base < p1; base += 32 * kClsRounds) {
                // all rounds' loads in flight before the first push
                float f[kClsRounds][3], v[kClsRounds][3];
                bool live[kClsRounds];
#pragma unroll
                for (int r = 0; r < kClsRounds; ++r) {
                    const long long i = base + 32 * r + lane;
                    live[r] = i < p1;
                    f[r][0] = f[r][1] = f[r][2] = 0.f;
                    v[r][0] = v[r][1] = v[r][2] = 0.f;
                    if (live[r]) {
#pragma unroll
                        for (int d = 0; d < D; ++d) f[r][d] = a.p.off[d][i];
#pragma unroll
                        for (int q = 0; q < 3; ++q) v[r][q] = a.p.vel[q][i];
                    }
                }
#pragma unroll
                for (int r = 0; r < kClsRounds; ++r) {
                    int cn[3];
                    const int cls = live[r] ? push_classify<D, PUSHER>(a.p, F, co, f[r], v[r], cn, lost_cnt) : -2;
                    unsigned q[8];
                    cic_moments<D>(f[r], q);
                    if (cls == STAY) {
                        sacc[0] += 1u;
#pragma unroll
                        for (int m = 1; m < NM; ++m) sacc[m] += q[m];
                    } else if (cls >= 0) {
                        // mover: a few per round, distinct classes mostly
                        atomicAdd(&mom_lo[warp][0][cls], 1u);
#pragma unroll
                        for (int m = 1; m < NM; ++m) smem_add64(&mom_lo[warp][m][cls], &mom_hi[warp][m][cls], q[m]);
                    } else if (cls == -1) {
                        // far mover: the species is flagged at the end (one atomic per
                        // warp); the caller redoes its move and its whole deposit
                        far_seen = true;
                    }
                }
                if (++pending == 32 / kClsRounds || base + 32 * kClsRounds >= p1) {
                    pending = 0;
#pragma unroll
                    for (int m = 0; m < NM; ++m) {
                        const unsigned long long t = warp_sum_u32(sacc[m]);
                        sacc[m] = 0u;
                        if (lane == 0) {
                            const unsigned long long v64 = pair64(mom_lo[warp][m][STAY], mom_hi[warp][m][STAY]) + t;
                            mom_lo[warp][m][STAY] = (unsigned)v64;
                            mom_hi[warp][m][STAY] = (unsigned)(v64 >> 32);
                        }
                    }
                }
            }
        }
        __syncwarp();
        // class lanes: count out, the class's moment sums into its target cell
        if (lane < NC) {
            const unsigned n = mom_lo[warp][0][lane];
            a.cls[lane * a.n_cells + c] = n;
            if (n) {
                mom_lo[warp][0][lane] = 0u;
                int cn[3];
                class_target<D>(g, co, lane, cn);   // inside: the class holds no absorbed particle
                const int sl = box_slot(cbox, cn);
                if (sl >= 0) {
                    atomicAdd(&ct_n[sl], n);
#pragma unroll
                    for (int m = 1; m < NM; ++m) {
                        smem_add64(&ct_lo[m - 1][sl], &ct_hi[m - 1][sl], pair64(mom_lo[warp][m][lane], mom_hi[warp][m][lane]));
                        mom_lo[warp][m][lane] = mom_hi[warp][m][lane] = 0u;
                    }
                } else {
                    long long W[8];
                    W[0] = (long long)n << kCicBits;
#pragma unroll
                    for (int m = 1; m < NM; ++m) {
                        W[m] = (long long)pair64(mom_lo[warp][m][lane], mom_hi[warp][m][lane]);
                        mom_lo[warp][m][lane] = mom_hi[warp][m][lane] = 0u;
                    }
                    deposit_direct<D>(a.p, cn, W);
                }
            }
        }
        __syncwarp();
    }
#pragma unroll
    for (int q = 0; q < 2 * D; ++q) {
        unsigned t = lost_cnt[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(full, t, o);
        if (lane == 0 && t) atomicAdd(a.p.losses + q, (unsigned long long)t);
    }
    if (__any_sync(full, far_seen) && lane == 0) atomicOr(a.far, 1);
    __syncthreads();
    // corners of every box cell once, into the node tile
    {
        const int e2 = cbox.ext[2], e12 = cbox.ext[1] * cbox.ext[2];
        for (int q = threadIdx.x; q < cbox.vol; q += blockDim.x) {
            const unsigned n = ct_n[q];
            if (n == 0u) continue;
            long long W[8];
            W[0] = (long long)n << kCicBits;
#pragma unroll
            for (int m = 1; m < NM; ++m) W[m] = (long long)pair64(ct_lo[m - 1][q], ct_hi[m - 1][q]);
            const int ti = q / e12, r = q - ti * e12;
            const int tj = r / e2;
            const int cc[3] = {ti + cbox.lo[0], tj + cbox.lo[1], r - tj * e2 + cbox.lo[2]};
#pragma unroll
            for (int B = 0; B < NM; ++B) {
                const long long w = cic_corner<D>(W, B);
                if (w == 0) continue;
                int nd[3];
                corner_node<D>(g, B, cc, nd);
                const int sl = box_slot(nbox, nd);
                if (sl >= 0) smem_add64(&tile_lo[sl], &tile_hi[sl], (unsigned long long)w);
                else atomicAdd(a.p.acc + node_index(g, nd[0], nd[1], nd[2]), (unsigned long long)w << a.p.dep_lsh);
            }
        }
    }
    __syncthreads();
    const int e2 = nbox.ext[2], e12 = nbox.ext[1] * nbox.ext[2];
    for (int q = threadIdx.x; q < nbox.vol; q += blockDim.x) {
        const unsigned long long val = pair64(tile_lo[q], tile_hi[q]);
        if (val == 0ull) continue;
        const int ti = q / e12, r = q - ti * e12;
        const int tj = r / e2, tk = r - tj * e2;
        atomicAdd(a.p.acc + node_index(g, ti + nbox.lo[0], tj + nbox.lo[1], tk + nbox.lo[2]), val << a.p.dep_lsh);
    }
}

// Per new cell: its particle count, and the offset inside it of every
// (source cell, class) group landing there, written over that group's count.
// Groups are visited by increasing source cell index (per axis: the source
// below, the cell itself, the source above, rotated at periodic seams), so
// the new cell keeps the particles in their old order.  Periodic axes need
// at least 3 cells for the sources to be distinct.
template <int D>
__global__ void k_cls_offsets(GridView g, unsigned* __restrict__ cls, unsigned* __restrict__ newcount,
                              long long n_cells) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c > n_cells) return;
    if (c == n_cells) {
        newcount[c] = 0u;
        return;
    }
    int cc[3];
    key_to_cell(g, (int)c, cc[0], cc[1], cc[2]);
    // steps of the arriving moves in order of increasing source coordinate
    int ord[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const bool seam_lo = g.periodic[a] && cc[a] == 0;
        const bool seam_hi = g.periodic[a] && cc[a] == g.M[a] - 1;
        ord[a][0] = seam_lo ? 0 : (seam_hi ? -1 : 1);
        ord[a][1] = seam_lo ? -1 : (seam_hi ? 1 : 0);
        ord[a][2] = seam_lo ? 1 : (seam_hi ? 0 : -1);
    }
    // all group counts are loaded before the first offset is stored (the
    // loads and stores address one array, so they would otherwise serialise);
    // the store loop recomputes each group's index
    constexpr int n1 = D == 3 ? 3 : 1;
    constexpr int NG = 9 * n1;
    auto group = [&](int j) -> long long {   // index of the j-th arriving group, -1 when none
        const int o0 = j / (3 * n1), o1 = (j / n1) % 3, o2 = j % n1;
        const int st[3] = {ord[0][o0], ord[1][o1], D == 3 ? ord[2][o2] : 0};
        int src[3] = {cc[0], cc[1], cc[2]};
        int d = 0;
#pragma unroll
        for (int a = 0; a < D; ++a) {
            int x = cc[a] - st[a];
            if (x < 0 || x >= g.M[a]) {
                if (!g.periodic[a]) return -1;
                x = x < 0 ? x + g.M[a] : x - g.M[a];
            }
            src[a] = x;
            d = d * 3 + st[a] + 1;
        }
        return (long long)d * n_cells + cell_to_key(g, src[0], src[1], src[2]);
    };
    unsigned cnt[NG];
#pragma unroll
    for (int j = 0; j < NG; ++j) {
        const long long i = group(j);
        cnt[j] = i >= 0 ? __ldg(cls + i) : 0u;
    }
    unsigned total = 0;
#pragma unroll
    for (int j = 0; j < NG; ++j) {
        const long long i = group(j);
        if (i >= 0) cls[i] = total;
        total += cnt[j];
    }
    newcount[c] = total;
}

// Movers a warp stages before writing them out (one list per warp): room for
// one iteration's 32 * rounds particles above the flush threshold.
constexpr int kMoverCap = 192;

// Pass 2: push again and write the re-sorted state.  A cell's particles that
// keep their cell are written at once, coalesced (ballot ranks).  Movers are
// appended to the warp's list in memory order (one ballot per round) and
// written out 32 at a time when the list is past kMoverFlushAt at the start
// of an iteration and at the end of the cell: each gets its rank inside its class from match_any, and every
// class keeps a running next slot (lane k holds the one of class k), so each
// class's run is written in the old particle order.
// (2D: 48 registers, 5 blocks per SM, for more loads in flight.)
template <int D, int PUSHER, int kClsRounds>
__global__ void __launch_bounds__(kPicThreads, D == 2 ? 5 : 4) k_cls_pass2(ClsArgs a) {
    constexpr int kMoverFlushAt = kMoverCap - 32 * kClsRounds;
    constexpr int NC = MoveClasses<D>::N;
    constexpr int STAY = MoveClasses<D>::STAY;
    constexpr int NF = D + 3;   // offsets, then velocities
    __shared__ float mstage[kClsWarps][NF][kMoverCap];
    __shared__ int mcls[kClsWarps][kMoverCap];
    __shared__ unsigned ccount[kClsWarps][32];
    if (*a.far) {   // some particle moved too far: the caller takes the general path (and sums its energy)
        if (a.p.kin_part && threadIdx.x < kClsWarps) a.p.kin_part[(long long)blockIdx.x * kClsWarps + threadIdx.x] = 0.0;
        return;
    }
    double kin = 0.0;   // kinetic energy of the particles this block writes (option "diagnostics 1")
    const long long ca = a.block_first[blockIdx.x], cb = a.block_first[blockIdx.x + 1];
    const GridView& g = a.p.g;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned full = 0xffffffffu;
    const unsigned lt = (1u << lane) - 1u;
    unsigned lost_dummy[2 * D] = {};   // losses were counted by pass 1
    auto out_field = [&](int fld) -> float* { return fld < D ? a.off_out[fld] : a.vel_out[fld - D]; };
    unsigned mpos = 0;   // lane k < NC: next slot of move class k in the new state
    // write the nm staged movers and advance the running slots
    auto flush = [&](int nm) {
        __syncwarp();
        for (int s0 = 0; s0 < nm; s0 += 32) {
            const int s = s0 + lane;
            const bool has = s < nm;
            const int k = has ? mcls[warp][s] : -1;
            const unsigned peers = __match_any_sync(full, k);
            const unsigned p = __shfl_sync(full, mpos, k & 31);
            ccount[warp][lane] = 0u;
            __syncwarp();
            if (has) {
                const unsigned dest = p + (unsigned)__popc(peers & lt);
#pragma unroll
                for (int fld = 0; fld < NF; ++fld) out_field(fld)[dest] = mstage[warp][fld][s];
                if (lane == __ffs(peers) - 1) ccount[warp][k] = (unsigned)__popc(peers);
            }
            __syncwarp();
            mpos += ccount[warp][lane];
            __syncwarp();
        }
    };
    for (long long c = ca + warp; c < cb; c += kClsWarps) {
        const long long p0 = a.starts[c], p1 = a.starts[c + 1];
        if (p1 == p0) continue;
        int co[3];
        key_to_cell(g, (int)c, co[0], co[1], co[2]);
        mpos = 0;
        if (lane < NC) {
            int cn[3];
            if (class_target<D>(g, co, lane, cn))
                mpos = __ldg(a.new_starts + cell_to_key(g, cn[0], cn[1], cn[2])) + __ldg(a.cls + lane * a.n_cells + c);
        }
        CellField<D> F;
        load_cell_field<D>(a.p, co[0], co[1], co[2], F);
        unsigned stay_next = __shfl_sync(full, mpos, STAY);   // next slot of the class that keeps its cell
        int nm = 0;
        for (long long base = p0; base < p1; base += 32 * kClsRounds) {
            if (nm > kMoverFlushAt) {
                flush(nm);
                nm = 0;
            }
            float f[kClsRounds][3], v[kClsRounds][3];
            bool live[kClsRounds];
#pragma unroll
            for (int r = 0; r < kClsRounds; ++r) {
                const long long i = base + 32 * r + lane;
                live[r] = i < p1;
                f[r][0] = f[r][1] = f[r][2] = 0.f;
                v[r][0] = v[r][1] = v[r][2] = 0.f;
                if (live[r]) {
#pragma unroll
                    for (int d = 0; d < D; ++d) f[r][d] = a.p.off[d][i];
#pragma unroll
                    for (int q = 0; q < 3; ++q) v[r][q] = a.p.vel[q][i];
                }
            }
#pragma unroll
            for (int r = 0; r < kClsRounds; ++r) {
                int cn[3];
                const int cls = live[r] ? push_classify<D, PUSHER>(a.p, F, co, f[r], v[r], cn, lost_dummy) : -2;
                if (a.p.kin_part && cls >= 0) kin += a.p.kin_hmw * kinetic_v2(v[r]);
                const unsigned stay = __ballot_sync(full, cls == STAY);
                if (cls == STAY) {
                    const unsigned dest = stay_next + (unsigned)__popc(stay & lt);
#pragma unroll
                    for (int d = 0; d < D; ++d) a.off_out[d][dest] = f[r][d];
#pragma unroll
                    for (int q = 0; q < 3; ++q) a.vel_out[q][dest] = v[r][q];
                }
                stay_next += (unsigned)__popc(stay);
                const bool mover = cls >= 0 && cls != STAY;
                const unsigned mb = __ballot_sync(full, mover);
                if (mb) {
                    const int cnt = __popc(mb);
                    if (mover) {
                        const int slot = nm + __popc(mb & lt);
#pragma unroll
                        for (int d = 0; d < D; ++d) mstage[warp][d][slot] = f[r][d];
#pragma unroll
                        for (int q = 0; q < 3; ++q) mstage[warp][D + q][slot] = v[r][q];
                        mcls[warp][slot] = cls;
                    }
                    nm += cnt;
                }
            }
        }
        if (nm) flush(nm);
    }
    // one partial per warp (fixed butterfly order), so no block barrier at the end
    if (a.p.kin_part) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) kin += __shfl_xor_sync(full, kin, o);
        if (lane == 0) a.p.kin_part[(long long)blockIdx.x * kClsWarps + warp] = kin;
    }
}

// Cell offsets of a sorted key array in O(particles + cells): the first and
// the last particle of every run record its bounds (first[k], last[k] =
// one past the end; both zero for empty cells), k_run_counts turns them into
// per-cell counts and an exclusive scan gives starts[c] = first index with
// key >= c.  (A particle after a long run of empty cells would otherwise
// fill their offsets alone.)
__global__ void k_run_bounds(const int* __restrict__ key, const long long* __restrict__ count, long long n_upper,
                             unsigned* __restrict__ first, unsigned* __restrict__ last) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long cnt = *count;
    if (i >= cnt || i >= n_upper) return;
    const int k = key[i];
    if (i == 0 || key[i - 1] != k) first[k] = (unsigned)i;
    if (i == cnt - 1 || key[i + 1] != k) last[k] = (unsigned)(i + 1);
}

__global__ void k_run_counts(const unsigned* __restrict__ first, unsigned* __restrict__ last, long long n_cells) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < n_cells) last[c] -= first[c];
    else if (c == n_cells) last[c] = 0u;
}

__global__ void k_count_from(long long* __restrict__ count, const unsigned* __restrict__ src) { *count = *src; }

// keys of a sorted state from its cell offsets: one warp per cell
__global__ void k_fill_keys(const unsigned* __restrict__ starts, long long n_cells, int* __restrict__ key) {
    const long long c = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (c >= n_cells) return;
    const unsigned e = starts[c + 1];
    for (unsigned i = starts[c] + (threadIdx.x & 31); i < e; i += 32) key[i] = (int)c;
}

// ------------------------------------------ B-spline step (interp_order) --
// FP64 positions pos[d*n_upper + i] of the stored particles (NaN x for
// invalid entries and for i >= the device count), from the mixed state
// (cell + offset) or the FP64 state: the input of the B-spline deposit and
// gather of a step with interp_order 2-4.
__global__ void k_state_positions(GridView g, int mixed, const int* __restrict__ key, const float* __restrict__ o0,
                                  const float* __restrict__ o1, const float* __restrict__ o2,
                                  const double* __restrict__ q0, const double* __restrict__ q1,
                                  const double* __restrict__ q2, const long long* __restrict__ count,
                                  long long n_upper, double* __restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_upper) return;
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    double p[3] = {nan, 0.0, 0.0};
    if (i < *count) {
        if (mixed) {
            const int k = key[i];
            if (k >= 0) {
                int c[3];
                key_to_cell(g, k, c[0], c[1], c[2]);
                const float* off[3] = {o0, o1, o2};
                for (int a = 0; a < g.dim; ++a) p[a] = g.lo[a] + ((double)c[a] + (double)off[a][i]) * g.dx[a];
            }
        } else {
            const double* q[3] = {q0, q1, q2};
            for (int a = 0; a < g.dim; ++a) p[a] = q[a][i];
        }
    }
    for (int a = 0; a < g.dim; ++a) out[(long long)a * n_upper + i] = p[a];
}

// Mixed push with the field's gradient gathered by the caller (grad[d*n_upper + i],
// per unit length): grad_a * dx_a takes the place of the CIC edge difference,
// then the same kick, move and boundary as every mixed push; no deposit (the
// next step's charge density is the B-spline deposit of the new positions).
template <int D, int PUSHER>
__global__ void __launch_bounds__(kPicThreads) k_push_grad_mixed(PushArgs a, const double* __restrict__ grad,
                                                                 long long n_upper) {
    const long long count = *a.count;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int lost = -1;
    double kin = 0.0;
    if (i < count && i < n_upper) {
        const int k = a.key[i];
        if (k >= 0) {
            int c[3];
            key_to_cell(a.g, k, c[0], c[1], c[2]);
            float f[3] = {0.f, 0.f, 0.f}, v[3];
            for (int d = 0; d < D; ++d) f[d] = a.off[d][i];
            for (int q = 0; q < 3; ++q) v[q] = a.vel[q][i];
            // the gathered gradient times dx is the edge difference the CIC push blends
            float G[3] = {0.f, 0.f, 0.f};
            for (int d = 0; d < D; ++d) G[d] = (float)(grad[(long long)d * n_upper + i] * a.g.dx[d]);
            int dc[3] = {0, 0, 0};
            int nk = -1;
            if (!kick_move<D, PUSHER>(a, G, f, v, dc)) {
                // non-finite: flagged in the error word by kick_move
            } else {
                lost = apply_step<D>(a.g, c, dc);
                if (lost < 0) nk = cell_to_key(a.g, c[0], c[1], c[2]);
            }
            a.key[i] = nk;
            for (int d = 0; d < D; ++d) a.off[d][i] = nk >= 0 ? f[d] : 0.f;
            for (int q = 0; q < 3; ++q) a.vel[q][i] = v[q];
            if (a.kin_part && nk >= 0) kin += a.kin_hmw * kinetic_v2(v);
        }
    }
    warp_count_losses(a.losses, D, lost);
    if (a.kin_part) block_sum_to(kin, a.kin_part);
}

// rho = background before the B-spline deposits add to it
__global__ void k_fill(double* __restrict__ v, long long n, double value) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = value;
}

// per-block sums of rho - background (the charge of a B-spline step's density)
__global__ void __launch_bounds__(256) k_rho_charge(const double* __restrict__ rho, long long n, double background,
                                                   double* __restrict__ part) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    block_sum_to(i < n ? rho[i] - background : 0.0, part);
}

// ------------------------------------------------------- load / export --
__global__ void k_load_mixed(GridView g, long long n, const double* __restrict__ pos, const double* __restrict__ vel,
                             int* __restrict__ key, float* __restrict__ o0, float* __restrict__ o1,
                             float* __restrict__ o2, float* __restrict__ v0, float* __restrict__ v1,
                             float* __restrict__ v2) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float* off[3] = {o0, o1, o2};
    int c[3] = {0, 0, 0};
    bool valid = isfinite(pos[i]);
    for (int a = 0; a < g.dim && valid; ++a) {
        double u = (pos[(long long)a * n + i] - g.lo[a]) * g.dr[a];
        if (!isfinite(u)) {
            valid = false;
            break;
        }
        if (g.periodic[a]) {
            u = u - floor(u / g.M[a]) * g.M[a];
        } else if (u < 0.0 || u >= (double)g.cells[a]) {
            valid = false;
            break;
        }
        double fl = floor(u);
        int ci = (int)fl;
        float f = (float)(u - fl);
        if (f >= 1.0f) {   // carry rule
            f = 0.0f;
            ci += 1;
        }
        if (g.periodic[a]) ci = ci >= g.M[a] ? ci - g.M[a] : ci;
        else if (ci >= g.cells[a]) {
            valid = false;
            break;
        }
        c[a] = ci;
        off[a][i] = f;
    }
    if (!valid)
        for (int a = 0; a < g.dim; ++a) off[a][i] = 0.f;
    key[i] = valid ? cell_to_key(g, c[0], c[1], c[2]) : -1;
    v0[i] = (float)vel[i];
    v1[i] = (float)vel[n + i];
    v2[i] = (float)vel[2 * n + i];
}

__global__ void k_export_mixed(GridView g, long long n, const int* __restrict__ key, const float* __restrict__ o0,
                               const float* __restrict__ o1, const float* __restrict__ o2,
                               const float* __restrict__ v0, const float* __restrict__ v1,
                               const float* __restrict__ v2, double* __restrict__ pos, double* __restrict__ vel) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* off[3] = {o0, o1, o2};
    const int k = key[i];
    if (k < 0) {
        for (int a = 0; a < g.dim; ++a) pos[(long long)a * n + i] = 0.0;
        pos[i] = __longlong_as_double(0x7ff8000000000000LL);
    } else {
        int c[3];
        key_to_cell(g, k, c[0], c[1], c[2]);
        for (int a = 0; a < g.dim; ++a)
            pos[(long long)a * n + i] = g.lo[a] + ((double)c[a] + (double)off[a][i]) * g.dx[a];
    }
    vel[i] = v0[i];
    vel[n + i] = v1[i];
    vel[2 * n + i] = v2[i];
}

__global__ void k_load64(GridView g, long long n, const double* __restrict__ pos, const double* __restrict__ vel,
                         double* p0, double* p1, double* p2, double* v0, double* v1, double* v2) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double* P[3] = {p0, p1, p2};
    bool valid = isfinite(pos[i]);
    for (int a = 0; a < g.dim; ++a) {
        double x = pos[(long long)a * n + i];
        if (valid && !isfinite(x)) valid = false;
        if (valid && g.periodic[a]) {
            const double L = (g.cells[a] + 1) * g.dx[a];
            const double top = g.lo[a] + L;
            int guard = 0;
            while (x < g.lo[a] && guard++ < 64) x += L;
            while (x >= top && guard++ < 128) x -= L;
        } else if (valid && (x < g.lo[a] || x >= g.lo[a] + g.cells[a] * g.dx[a])) {
            valid = false;
        }
        P[a][i] = x;
    }
    if (!valid) p0[i] = __longlong_as_double(0x7ff8000000000000LL);
    v0[i] = vel[i];
    v1[i] = vel[n + i];
    v2[i] = vel[2 * n + i];
}

// ---------------------------------------------------- scans and sorting --
constexpr int kScanBlock = 1024;

// exclusive scan of `n` uint32 values in blocks of kScanBlock; block totals out
__global__ void k_scan_blocks(const unsigned* __restrict__ in, unsigned* __restrict__ out, long long n,
                              unsigned* __restrict__ totals) {
    __shared__ unsigned sh[kScanBlock];
    const long long base = (long long)blockIdx.x * kScanBlock;
    const int t = threadIdx.x;   // blockDim = 256, 4 items per thread
    unsigned v[4], s = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const long long i = base + t * 4 + q;
        v[q] = i < n ? in[i] : 0u;
        s += v[q];
    }
    sh[t] = s;
    __syncthreads();
    for (int d = 1; d < 256; d <<= 1) {
        const unsigned add = t >= d ? sh[t - d] : 0u;
        __syncthreads();
        sh[t] += add;
        __syncthreads();
    }
    unsigned run = sh[t] - s;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const long long i = base + t * 4 + q;
        if (i < n) out[i] = run;
        run += v[q];
    }
    if (t == 255) totals[blockIdx.x] = sh[255];
}

// The same scan in place: every thread reads its 4 values before the
// block's first write, and writes only those.
__global__ void k_scan_blocks_inplace(unsigned* v_io, long long n, unsigned* __restrict__ totals) {
    __shared__ unsigned sh[kScanBlock];
    const long long base = (long long)blockIdx.x * kScanBlock;
    const int t = threadIdx.x;
    unsigned v[4], s = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const long long i = base + t * 4 + q;
        v[q] = i < n ? v_io[i] : 0u;
        s += v[q];
    }
    sh[t] = s;
    __syncthreads();
    for (int d = 1; d < 256; d <<= 1) {
        const unsigned add = t >= d ? sh[t - d] : 0u;
        __syncthreads();
        sh[t] += add;
        __syncthreads();
    }
    unsigned run = sh[t] - s;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const long long i = base + t * 4 + q;
        if (i < n) v_io[i] = run;
        run += v[q];
    }
    if (t == 255) totals[blockIdx.x] = sh[255];
}

__global__ void k_scan_add(unsigned* __restrict__ out, long long n, const unsigned* __restrict__ offsets) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += offsets[i / kScanBlock];
}

// Single-block sequential-by-chunk scan of up to a few million totals.
__global__ void k_scan_single(unsigned* __restrict__ v, long long n) {
    __shared__ unsigned sh[1024];
    __shared__ unsigned carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (long long base = 0; base < n; base += 1024) {
        const long long i = base + threadIdx.x;
        const unsigned x = i < n ? v[i] : 0u;
        sh[threadIdx.x] = x;
        __syncthreads();
        for (int d = 1; d < 1024; d <<= 1) {
            const unsigned add = threadIdx.x >= d ? sh[threadIdx.x - d] : 0u;
            __syncthreads();
            sh[threadIdx.x] += add;
            __syncthreads();
        }
        if (i < n) v[i] = carry + sh[threadIdx.x] - x;
        __syncthreads();
        if (threadIdx.x == 1023) carry += sh[1023];
        __syncthreads();
    }
}

}  // namespace

// exclusive scan (uint32), `tmp1`/`tmp2` scratch of ceil(n/1024) and
// ceil(n/1024^2) entries
void exclusive_scan_u32(const unsigned* in, unsigned* out, long long n, unsigned* tmp1, unsigned* tmp2,
                        cudaStream_t s, long long tmp2_cap = 0) {
    if (n <= 0) return;
    const long long nb = (n + kScanBlock - 1) / kScanBlock;
    { k_scan_blocks<<<(unsigned)nb, 256, 0, s>>>(in, out, n, tmp1); count_launch(); }
    if (nb > 1) {
        const long long nb2 = (nb + kScanBlock - 1) / kScanBlock;
        if (nb > 4 * kScanBlock && tmp2 && nb2 <= tmp2_cap) {
            // many block totals: scan them by blocks too (in place), then their totals
            { k_scan_blocks_inplace<<<(unsigned)nb2, 256, 0, s>>>(tmp1, nb, tmp2); count_launch(); }
            { k_scan_single<<<1, 1024, 0, s>>>(tmp2, nb2); count_launch(); }
            { k_scan_add<<<blocks_for(nb, 256), 256, 0, s>>>(tmp1, nb, tmp2); count_launch(); }
        } else if (nb <= 4 * 1024 * 1024) {
            { k_scan_single<<<1, 1024, 0, s>>>(tmp1, nb); count_launch(); }
        } else {
            throw Error(PSUM_ERR_INVALID_ARGUMENT, "scan: input too large");
        }
        { k_scan_add<<<blocks_for(n, 256), 256, 0, s>>>(out, n, tmp1); count_launch(); }
    }
}

namespace {

constexpr int kRsThreads = 256;
constexpr int kRsItems = 16;
constexpr int kRsTile = kRsThreads * kRsItems;   // 4096
constexpr int kRsBits = 8;
constexpr int kRsBuckets = 1 << kRsBits;

__global__ void __launch_bounds__(kRsThreads) k_rs_hist(const unsigned* __restrict__ keys, long long n, int shift,
                                                        unsigned* __restrict__ hist, int nblocks) {
    __shared__ unsigned h[kRsBuckets];
    h[threadIdx.x] = 0;
    __syncthreads();
    const long long base = (long long)blockIdx.x * kRsTile;
#pragma unroll 4
    for (int r = 0; r < kRsItems; ++r) {
        const long long i = base + r * kRsThreads + threadIdx.x;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & (kRsBuckets - 1)], 1u);
    }
    __syncthreads();
    hist[(long long)threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter: items are ranked in (round, thread) order, i.e. ascending
// input index within a tile; tiles are ordered by the digit-major scan.
__global__ void __launch_bounds__(kRsThreads) k_rs_scatter(const unsigned* __restrict__ kin,
                                                           const int* __restrict__ vin, unsigned* __restrict__ kout,
                                                           int* __restrict__ vout, long long n, int shift,
                                                           const unsigned* __restrict__ offs, int nblocks) {
    __shared__ unsigned wcnt[kRsThreads / 32][kRsBuckets];
    __shared__ unsigned running[kRsBuckets];
    __shared__ unsigned base_off[kRsBuckets];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    running[t] = 0;
    base_off[t] = offs[(long long)t * nblocks + blockIdx.x];
    const long long tile = (long long)blockIdx.x * kRsTile;
    for (int r = 0; r < kRsItems; ++r) {
#pragma unroll
        for (int w = 0; w < kRsThreads / 32; ++w) wcnt[w][t] = 0;
        __syncthreads();
        const long long i = tile + r * kRsThreads + t;
        const bool valid = i < n;
        const unsigned key = valid ? kin[i] : 0u;
        const int dig = valid ? (int)((key >> shift) & (kRsBuckets - 1)) : kRsBuckets;   // kRsBuckets = none
        const unsigned peers = __match_any_sync(0xffffffffu, dig);
        const unsigned lt = (1u << lane) - 1u;
        const int rank_w = __popc(peers & lt);
        if (valid && rank_w == 0) wcnt[warp][dig] = __popc(peers);
        __syncthreads();
        // exclusive prefix over warps for digit t, plus the round total
        {
            unsigned acc = 0;
#pragma unroll
            for (int w = 0; w < kRsThreads / 32; ++w) {
                const unsigned c = wcnt[w][t];
                wcnt[w][t] = acc;
                acc += c;
            }
            __syncthreads();
            if (valid) {
                const unsigned pos = base_off[dig] + running[dig] + wcnt[warp][dig] + (unsigned)rank_w;
                kout[pos] = key;
                vout[pos] = vin[i];
            }
            __syncthreads();
            running[t] += acc;
        }
        __syncthreads();
    }
}

__global__ void k_make_sort_keys(const int* __restrict__ key, long long n, unsigned sentinel,
                                 unsigned* __restrict__ skey, int* __restrict__ sidx) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int k = key[i];
    skey[i] = k < 0 ? sentinel : (unsigned)k;
    sidx[i] = (int)i;
}

template <class T>
__global__ void k_gather(const T* __restrict__ in, T* __restrict__ out, const int* __restrict__ perm, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = in[perm[i]];
}

// Every array of a species' state permuted at once: out[a][i] = in[a][perm[i]]
// for up to 8 arrays of 4-byte and 6 of 8-byte elements.  perm is read once
// and each thread has kGatherPer elements of every array in flight.
struct GatherSet {
    const uint32_t* in4[8];
    uint32_t* out4[8];
    int n4;
    const unsigned long long* in8[6];
    unsigned long long* out8[6];
    int n8;
};
constexpr int kGatherPer = 4;

__global__ void __launch_bounds__(256) k_gather_all(GatherSet g, const int* __restrict__ perm, long long n) {
    const long long i0 = (long long)blockIdx.x * (blockDim.x * kGatherPer) + threadIdx.x;
    int p[kGatherPer];
#pragma unroll
    for (int u = 0; u < kGatherPer; ++u) {
        const long long i = i0 + (long long)u * blockDim.x;
        p[u] = i < n ? __ldg(perm + i) : -1;
    }
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        if (a >= g.n4) break;
        uint32_t v[kGatherPer];
#pragma unroll
        for (int u = 0; u < kGatherPer; ++u) v[u] = p[u] >= 0 ? __ldg(g.in4[a] + p[u]) : 0u;
#pragma unroll
        for (int u = 0; u < kGatherPer; ++u)
            if (p[u] >= 0) g.out4[a][i0 + (long long)u * blockDim.x] = v[u];
    }
#pragma unroll
    for (int a = 0; a < 6; ++a) {
        if (a >= g.n8) break;
        unsigned long long v[kGatherPer];
#pragma unroll
        for (int u = 0; u < kGatherPer; ++u) v[u] = p[u] >= 0 ? __ldg(g.in8[a] + p[u]) : 0ull;
#pragma unroll
        for (int u = 0; u < kGatherPer; ++u)
            if (p[u] >= 0) g.out8[a][i0 + (long long)u * blockDim.x] = v[u];
    }
}

__global__ void k_count_valid(const unsigned* __restrict__ sorted_keys, long long n, unsigned sentinel,
                              long long* __restrict__ count) {
    // first index holding the sentinel (keys are sorted ascending)
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool here = sorted_keys[i] == sentinel && (i == 0 || sorted_keys[i - 1] != sentinel);
    if (here) *count = i;
    if (i == n - 1 && sorted_keys[i] != sentinel) *count = n;
}

__global__ void k_set_count(long long* count, long long v) { *count = v; }

// ------------------------------------------------------- charge density --
struct RhoArgs {
    const unsigned long long* acc[8];
    double coef[8];
    int ns;
    double background;
    unsigned long long* qsum;   // per species: sum of the accumulators (exact integers; null: not summed)
};

__global__ void k_rho(RhoArgs a, double* __restrict__ rho, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = i < n;
    double r = a.background;
    for (int s = 0; s < a.ns; ++s) {
        const long long v = in ? (long long)a.acc[s][i] : 0;
        r += a.coef[s] * (double)v;
        if (a.qsum) {   // the total charge of the density: integer sums, so any order gives the same bits
            long long t = v;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
            if ((threadIdx.x & 31) == 0 && t) atomicAdd(a.qsum + s, (unsigned long long)t);
        }
    }
    if (in) rho[i] = r;
}

// ------------------------------------------------------------ binning ---
__global__ void k_bin_keys_mixed(GridView g, const int* __restrict__ key, const float* __restrict__ o0,
                                 long long n, long long* __restrict__ keys_out, unsigned* __restrict__ skey,
                                 int* __restrict__ sidx, unsigned sentinel) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int k = key[i];
    long long ref = -1;
    if (k >= 0) {
        int c[3];
        key_to_cell(g, k, c[0], c[1], c[2]);
        bool in = true;
        for (int a = 0; a < g.dim; ++a) in = in && c[a] < g.cells[a];   // the wrap cell is outside [lo, hi)
        if (in) ref = ((long long)c[0] * g.cells[1] + c[1]) * g.cells[2] + c[2];
    }
    (void)o0;
    keys_out[i] = ref;
    skey[i] = ref < 0 ? sentinel : (unsigned)ref;
    sidx[i] = (int)i;
}

__global__ void k_bin_keys64(GridView g, const double* __restrict__ x, const double* __restrict__ y,
                             const double* __restrict__ z, long long n, long long* __restrict__ keys_out,
                             unsigned* __restrict__ skey, int* __restrict__ sidx, unsigned sentinel, const double* hi) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double p[3] = {x[i], g.dim > 1 ? y[i] : 0.0, g.dim > 2 ? z[i] : 0.0};
    long long ref = -1;
    bool in = isfinite(p[0]);
    for (int a = 0; a < g.dim && in; ++a) in = p[a] >= g.lo[a] && p[a] < hi[a];   // inGrid, simple_grid.hpp:168-174
    if (in) {
        int c[3] = {0, 0, 0};
        // nC: truncation (simple_grid.hpp:99-104), clamped to the last cell: with dr = 1/dx rounded up, a
        // position just below hi can truncate to `cells`, which has no cell (undefined in the reference)
        for (int a = 0; a < g.dim; ++a) c[a] = min((int)((p[a] - g.lo[a]) * g.dr[a]), g.cells[a] - 1);
        ref = ((long long)c[0] * g.cells[1] + c[1]) * g.cells[2] + c[2];
    }
    keys_out[i] = ref;
    skey[i] = ref < 0 ? sentinel : (unsigned)ref;
    sidx[i] = (int)i;
}

__global__ void k_hist_u32(const long long* __restrict__ keys, long long n, unsigned* __restrict__ counts) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && keys[i] >= 0) atomicAdd(counts + keys[i], 1u);
}

__global__ void k_u32_to_u64(const unsigned* __restrict__ in, unsigned long long* __restrict__ out, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = in[i];
}

__global__ void k_i32_to_u64(const int* __restrict__ in, unsigned long long* __restrict__ out, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (unsigned long long)in[i];
}

// ------------------------------------------------------- diagnostics ----
__global__ void __launch_bounds__(256) k_kinetic_mixed(const int* __restrict__ key, const float* __restrict__ v0,
                                                       const float* __restrict__ v1, const float* __restrict__ v2,
                                                       const long long* __restrict__ count, double mw,
                                                       double* __restrict__ partials) {
    __shared__ double sh[8];
    double acc = 0.0;
    const long long n = *count;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        if (key[i] >= 0) {
            const double a = v0[i], b = v1[i], c = v2[i];
            acc += 0.5 * mw * (a * a + b * b + c * c);
        }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0;
        for (int w = 0; w < 8; ++w) s += sh[w];
        partials[blockIdx.x] = s;
    }
}

__global__ void __launch_bounds__(256) k_kinetic64(const double* __restrict__ x, const double* __restrict__ v0,
                                                   const double* __restrict__ v1, const double* __restrict__ v2,
                                                   const long long* __restrict__ count, double mw,
                                                   double* __restrict__ partials) {
    __shared__ double sh[8];
    double acc = 0.0;
    const long long n = *count;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        if (isfinite(x[i])) acc += 0.5 * mw * (v0[i] * v0[i] + v1[i] * v1[i] + v2[i] * v2[i]);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0;
        for (int w = 0; w < 8; ++w) s += sh[w];
        partials[blockIdx.x] = s;
    }
}

__global__ void __launch_bounds__(256) k_field_energy(GridView g, const double* __restrict__ phi,
                                                      double* __restrict__ partials) {
    __shared__ double sh[8];
    double acc = 0.0;
    for (long long node = (long long)blockIdx.x * blockDim.x + threadIdx.x; node < g.n_nodes;
         node += (long long)gridDim.x * blockDim.x) {
        const int n12 = g.N[1] * g.N[2];
        const int i = (int)(node / n12);
        const int rem = (int)(node - (long long)i * n12);
        const int idx[3] = {i, rem / g.N[2], rem % g.N[2]};
        for (int a = 0; a < g.dim; ++a) {
            int q[3] = {idx[0], idx[1], idx[2]};
            q[a] += 1;
            if (q[a] >= g.N[a]) {
                if (!g.periodic[a]) continue;
                q[a] = 0;
            }
            const double gr = (phi[node_index(g, q[0], q[1], q[2])] - phi[node]) * g.dr[a];
            acc += gr * gr;
        }
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0;
        for (int w = 0; w < 8; ++w) s += sh[w];
        partials[blockIdx.x] = s;
    }
}

__global__ void k_acc_sum(const unsigned long long* __restrict__ acc, long long n, long long* __restrict__ out) {
    long long s = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        s += (long long)acc[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(reinterpret_cast<unsigned long long*>(out), (unsigned long long)s);
}

constexpr int kDiagBlocks = 296;

// Per-step diagnostics from the partial sums the step's kernels wrote:
// out[s] = kinetic energy of species s, out[ns] = (1/2) sum |grad phi|^2 * cell
// volume (the field energy without epsilon), out[ns + 1] = particle charge.
// One block; every sum runs in a fixed order, so repeats give the same bits.
struct DiagFinishArgs {
    const double* fe_part;
    long long fe_n;
    double fe_coef;                 // cell volume / 2
    const double* kin_part[8];
    long long kin_n[8];
    const unsigned long long* qsum;
    double q_coef[8];               // q * w * 2^-dep_shift per species
    const double* rho_part;         // B-spline steps: per-block sums of rho - background (else null)
    long long rho_n;
    double rho_coef;                // cell volume
    int ns;
    double* out;
};

constexpr int kDiagFinishThreads = 256;   // small, so it finds a slot beside a running second pass

__device__ double block_fixed_sum(const double* __restrict__ v, long long n) {
    __shared__ double red[kDiagFinishThreads];
    double t0 = 0.0, t1 = 0.0, t2 = 0.0, t3 = 0.0;
    const long long st = blockDim.x;
    long long i = threadIdx.x;
    for (; i + 3 * st < n; i += 4 * st) {
        t0 += v[i];
        t1 += v[i + st];
        t2 += v[i + 2 * st];
        t3 += v[i + 3 * st];
    }
    for (; i < n; i += st) t0 += v[i];
    const double t = (t0 + t1) + (t2 + t3);
    __syncthreads();
    red[threadIdx.x] = t;
    __syncthreads();
    for (int h = blockDim.x >> 1; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
        __syncthreads();
    }
    return red[0];
}

// First level of the diagnostics reduction: block (x, y) sums slice x of
// array y (y < ns: species y's kinetic partials; ns: the field-energy
// partials; ns + 1: the density partials) in fixed order into
// stage[y * kDiagStageBlocks + x], so the one-block finisher reads only
// kDiagStageBlocks values per array.
constexpr int kDiagStageBlocks = 128;

__global__ void __launch_bounds__(kDiagFinishThreads) k_diag_stage(DiagFinishArgs a, double* __restrict__ stage) {
    const int y = blockIdx.y;
    const double* v = y < a.ns ? a.kin_part[y] : (y == a.ns ? a.fe_part : a.rho_part);
    const long long n = y < a.ns ? a.kin_n[y] : (y == a.ns ? a.fe_n : a.rho_n);
    if (!v) return;
    const long long len = (n + kDiagStageBlocks - 1) / kDiagStageBlocks;
    const long long lo = min((long long)blockIdx.x * len, n), hi = min(lo + len, n);
    const double t = block_fixed_sum(v + lo, hi - lo);
    if (threadIdx.x == 0) stage[(long long)y * kDiagStageBlocks + blockIdx.x] = t;
}

__global__ void __launch_bounds__(kDiagFinishThreads) k_diag_finish(DiagFinishArgs a) {
    for (int s = 0; s < a.ns; ++s) {
        const double k = a.kin_part[s] ? block_fixed_sum(a.kin_part[s], a.kin_n[s]) : 0.0;
        if (threadIdx.x == 0) a.out[s] = k;
    }
    const double fe = a.fe_part ? block_fixed_sum(a.fe_part, a.fe_n) : 0.0;
    if (threadIdx.x == 0) {
        a.out[a.ns] = fe * a.fe_coef;
        double q = 0.0;
        for (int s = 0; s < a.ns; ++s) q += a.q_coef[s] * (double)(long long)a.qsum[s];
        a.out[a.ns + 1] = q;
    }
    if (a.rho_part) {
        const double q = block_fixed_sum(a.rho_part, a.rho_n);
        if (threadIdx.x == 0) a.out[a.ns + 1] = q * a.rho_coef;
    }
}

}  // namespace

// ============================================================ host side ===

static void finish_cls_step(psum_pic_ctx* c);
static void finish_diagnostics(psum_pic_ctx* c, int par);
constexpr int kPhaseContinued = 0x100;   // timing pair that adds time to a phase execution already counted

psum_pic_ctx* ctx_check_nojoin(psum_pic_ctx* c) {
    if (!c || c->magic != kPicMagic) throw Error(PSUM_ERR_INVALID_ARGUMENT, "not a particle context of this library");
    return c;
}

psum_pic_ctx* ctx_check(psum_pic_ctx* c) {
    ctx_check_nojoin(c);
    finish_cls_step(c);
    return c;
}

Species& species_at(psum_pic_ctx* c, int s) {
    if (s < 0 || s >= (int)c->sp.size()) throw Error(PSUM_ERR_INVALID_ARGUMENT, "species index out of range");
    return *c->sp[s];
}

static int bits_for(unsigned long long v) {
    int b = 0;
    while (b < 64 && (1ULL << b) <= v) ++b;
    return b;
}

static void ensure_sort_scratch(psum_pic_ctx* c, long long n) {
    SortScratch& S = c->sort;
    if (S.cap >= n) return;
    S.keyA.alloc(n);
    S.keyB.alloc(n);
    S.idxA.alloc(n);
    S.idxB.alloc(n);
    const long long nb = (n + kRsTile - 1) / kRsTile;
    S.hist.alloc((size_t)kRsBuckets * nb);
    S.hist_scan.alloc((size_t)kRsBuckets * nb);
    S.block_sums.alloc((size_t)((kRsBuckets * nb + kScanBlock - 1) / kScanBlock) + 1);
    S.block_sums2.alloc(16);
    S.cap = n;
}

// Stable LSD radix sort of (skey, sidx) pairs in S.keyA/S.idxA; result in
// the returned pair of buffers.
static void radix_sort(psum_pic_ctx* c, long long n, unsigned max_key, unsigned** keys_out, int** idx_out) {
    SortScratch& S = c->sort;
    cudaStream_t s = c->stream;
    unsigned* kin = S.keyA.p;
    unsigned* kout = S.keyB.p;
    int* vin = S.idxA.p;
    int* vout = S.idxB.p;
    const int nbits = std::max(1, bits_for(max_key));
    const int nb = (int)((n + kRsTile - 1) / kRsTile);
    for (int shift = 0; shift < nbits; shift += kRsBits) {
        { k_rs_hist<<<nb, kRsThreads, 0, s>>>(kin, n, shift, S.hist.p, nb); count_launch(); }
        exclusive_scan_u32(S.hist.p, S.hist_scan.p, (long long)kRsBuckets * nb, S.block_sums.p, S.block_sums2.p, s);
        { k_rs_scatter<<<nb, kRsThreads, 0, s>>>(kin, vin, kout, vout, n, shift, S.hist_scan.p, nb); count_launch(); }
        std::swap(kin, kout);
        std::swap(vin, vout);
    }
    cuda_check(cudaGetLastError(), "radix sort launch");
    *keys_out = kin;
    *idx_out = vin;
}

// The fused sorted step leaves the keys implied by the cell offsets; every
// reader of the keys calls this first.
void ensure_keys(psum_pic_ctx* c, Species& sp) {
    if (!sp.keys_stale) return;
    const long long nc = c->g.n_cells;
    { k_fill_keys<<<blocks_for(nc * 32, 256), 256, 0, c->stream>>>(sp.starts[sp.starts_cur].p, nc, sp.key[sp.cur].p); count_launch(); }
    sp.keys_stale = false;
}

static void sort_species(psum_pic_ctx* c, Species& sp, int sidx) {
    ensure_keys(c, sp);
    const long long n = sp.n;
    if (n <= 0) return;
    cudaStream_t s = c->stream;
    ensure_sort_scratch(c, n);
    const int cur = sp.cur, nxt = 1 - sp.cur;
    const unsigned sentinel = (unsigned)c->g.n_cells;
    { k_make_sort_keys<<<blocks_for(n, 256), 256, 0, s>>>(sp.key[cur].p, n, sentinel, c->sort.keyA.p, c->sort.idxA.p); count_launch(); }
    unsigned* skeys;
    int* perm;
    radix_sort(c, n, sentinel, &skeys, &perm);
    const unsigned gb = blocks_for(n, 256);
    {
        GatherSet gs{};
        auto add4 = [&](const void* in, void* out) {
            gs.in4[gs.n4] = static_cast<const uint32_t*>(in);
            gs.out4[gs.n4++] = static_cast<uint32_t*>(out);
        };
        auto add8 = [&](const void* in, void* out) {
            gs.in8[gs.n8] = static_cast<const unsigned long long*>(in);
            gs.out8[gs.n8++] = static_cast<unsigned long long*>(out);
        };
        add4(sp.key[cur].p, sp.key[nxt].p);
        if (c->precision == PSUM_PIC_MIXED) {
            for (int a = 0; a < c->g.dim; ++a) add4(sp.off[a][cur].p, sp.off[a][nxt].p);
            for (int q = 0; q < 3; ++q) add4(sp.vel[q][cur].p, sp.vel[q][nxt].p);
        } else {
            for (int a = 0; a < c->g.dim; ++a) add8(sp.pos64[a][cur].p, sp.pos64[a][nxt].p);
            for (int q = 0; q < 3; ++q) add8(sp.vel64[q][cur].p, sp.vel64[q][nxt].p);
        }
        { k_gather_all<<<blocks_for((n + kGatherPer - 1) / kGatherPer, 256), 256, 0, s>>>(gs, perm, n); count_launch(); }
    }
    { k_count_valid<<<gb, 256, 0, s>>>(skeys, n, sentinel, c->count.p + sidx); count_launch(); }
    sp.cur = nxt;
    if (c->precision == PSUM_PIC_MIXED) {
        // cell offsets of the sorted state, for the fused sorted step; the
        // other offsets buffer and the new-count buffer are free scratch here
        const long long nc = c->g.n_cells;
        const size_t nscan1 = (size_t)(nc + 1 + kScanBlock - 1) / kScanBlock + 1;
        const size_t nscan2 = (nscan1 + kScanBlock - 1) / kScanBlock + 16;
        if (sp.newcount.n < (size_t)nc + 1) sp.newcount.alloc((size_t)nc + 1);
        if (sp.scan_tmp1.n < nscan1) sp.scan_tmp1.alloc(nscan1);
        if (sp.scan_tmp2.n < nscan2) sp.scan_tmp2.alloc(nscan2);
        unsigned* first = sp.starts[1 - sp.starts_cur].p;
        unsigned* last = sp.newcount.p;
        cuda_check(cudaMemsetAsync(first, 0, sizeof(unsigned) * (nc + 1), s), "memset");
        cuda_check(cudaMemsetAsync(last, 0, sizeof(unsigned) * (nc + 1), s), "memset");
        { k_run_bounds<<<blocks_for(n, 256), 256, 0, s>>>(sp.key[nxt].p, c->count.p + sidx, n, first, last); count_launch(); }
        { k_run_counts<<<blocks_for(nc + 1, 256), 256, 0, s>>>(first, last, nc); count_launch(); }
        exclusive_scan_u32(last, sp.starts[sp.starts_cur].p, nc + 1, sp.scan_tmp1.p, sp.scan_tmp2.p, s,
                           (long long)sp.scan_tmp2.n);
        sp.sorted = true;
    }
    cuda_check(cudaGetLastError(), "sort launch");
}

static void alloc_species_state(psum_pic_ctx* c, Species& sp) {
    for (int b = 0; b < 2; ++b) {
        sp.key[b].alloc(sp.cap);
        if (c->precision == PSUM_PIC_MIXED) {
            for (int a = 0; a < c->g.dim; ++a) sp.off[a][b].alloc(sp.cap);
            for (int q = 0; q < 3; ++q) sp.vel[q][b].alloc(sp.cap);
        } else {
            for (int a = 0; a < c->g.dim; ++a) sp.pos64[a][b].alloc(sp.cap);
            for (int q = 0; q < 3; ++q) sp.vel64[q][b].alloc(sp.cap);
        }
    }
    sp.acc.alloc(c->g.n_nodes);
    cuda_check(cudaMemsetAsync(sp.acc.p, 0, sizeof(unsigned long long) * c->g.n_nodes, c->stream), "memset acc");
    if (c->precision == PSUM_PIC_MIXED)
        for (int b = 0; b < 2; ++b) sp.starts[b].alloc((size_t)c->g.n_cells + 1);
}

static PushArgs make_push_args(psum_pic_ctx* c, Species& sp, int sidx, double dt, int pusher, const double* B) {
    PushArgs a{};
    a.g = c->g;
    a.key = sp.key[sp.cur].p;
    for (int d = 0; d < 3; ++d) {
        a.off[d] = d < c->g.dim ? sp.off[d][sp.cur].p : nullptr;
        a.vel[d] = sp.vel[d][sp.cur].p;
    }
    a.count = c->count.p + sidx;
    a.edges = c->edges.p;
    const double qm = sp.q / sp.m;
    for (int d = 0; d < 3; ++d) {
        a.kE[d] = (float)(qm * dt * c->g.dr[d]);
        a.dtdr[d] = (float)(dt * c->g.dr[d]);
        a.dr[d] = (float)c->g.dr[d];
        a.Bt[d] = (float)((B ? B[d] : 0.0) * qm * dt * 0.5);
    }
    a.qmdt_half = (float)(qm * dt * 0.5);
    (void)pusher;
    a.acc = sp.acc.p;
    a.dep_lsh = sp.dep_shift - kCicBits;
    a.losses = c->losses.p + (size_t)sidx * 6;
    a.err = c->err.p;
    a.kin_part = nullptr;
    a.kin_hmw = 0.5 * sp.m * sp.w;
    return a;
}

static void launch_mixed(const PushArgs& a, int dim, int pusher, bool deposit_only, long long n, cudaStream_t s) {
    const unsigned blocks = capped_blocks(4LL * kPicThreads, n);
    if (deposit_only) {
        if (dim == 1) { k_push_mixed<1, 0, true><<<blocks, kPicThreads, 0, s>>>(a); count_launch(); }
        else if (dim == 2) { k_push_mixed<2, 0, true><<<blocks, kPicThreads, 0, s>>>(a); count_launch(); }
        else { k_push_mixed<3, 0, true><<<blocks, kPicThreads, 0, s>>>(a); count_launch(); }
        return;
    }
    if (dim == 1) {
        if (pusher == PSUM_PIC_BORIS) { k_push_mixed<1, PSUM_PIC_BORIS, false><<<blocks, kPicThreads, 0, s>>>(a); count_launch(); }
        else { k_push_mixed<1, PSUM_PIC_LEAPFROG, false><<<blocks, kPicThreads, 0, s>>>(a); count_launch(); }
    } else if (dim == 2) {
        if (pusher == PSUM_PIC_BORIS) { k_push_mixed<2, PSUM_PIC_BORIS, false><<<blocks, kPicThreads, 0, s>>>(a); count_launch(); }
        else { k_push_mixed<2, PSUM_PIC_LEAPFROG, false><<<blocks, kPicThreads, 0, s>>>(a); count_launch(); }
    } else {
        if (pusher == PSUM_PIC_BORIS) { k_push_mixed<3, PSUM_PIC_BORIS, false><<<blocks, kPicThreads, 0, s>>>(a); count_launch(); }
        else { k_push_mixed<3, PSUM_PIC_LEAPFROG, false><<<blocks, kPicThreads, 0, s>>>(a); count_launch(); }
    }
}

static void zero_accumulators(psum_pic_ctx* c) {
    for (auto& sp : c->sp)
        cuda_check(cudaMemsetAsync(sp->acc.p, 0, sizeof(unsigned long long) * c->g.n_nodes, c->stream), "memset acc");
}

// The FP64 kernels of the context's build: bit-exact with the oracle
// (default) or contracted (option "fp64_fma 1", the FP64 comparison run).
static void push64(const psum_pic_ctx* c, const Push64Args& a, long long n, cudaStream_t s) {
    if (c->fp64_fma) fp64_fma::launch_push64(a, n, s);
    else fp64_exact::launch_push64(a, n, s);
}
static void deposit64(const psum_pic_ctx* c, const Deposit64Args& a, long long n, cudaStream_t s) {
    if (c->fp64_fma) fp64_fma::launch_deposit64(a, n, s);
    else fp64_exact::launch_deposit64(a, n, s);
}
static void keys64(const psum_pic_ctx* c, double* const pos[3], int* key, const long long* count, long long n,
                   cudaStream_t s) {
    if (c->fp64_fma) fp64_fma::launch_keys64(c->g, pos, key, count, n, s);
    else fp64_exact::launch_keys64(c->g, pos, key, count, n, s);
}

// Edge differences of phi for the mixed push, and in a step with
// diagnostics the field-energy partial sums (FP64 mode: the sums only).
static void launch_edges(psum_pic_ctx* c, const double* phi, cudaStream_t s) {
    const bool fe = c->diag_in_step;
    if (c->precision != PSUM_PIC_MIXED && !fe) return;
    const unsigned blocks = blocks_for(c->g.n_nodes, 256);
    float* edges = c->precision == PSUM_PIC_MIXED ? c->edges.p : nullptr;
    double* part = fe ? c->dbuf[c->diag_par].fe.p : nullptr;
    if (fe) c->dbuf[c->diag_par].fe_n = blocks;
    if (c->g.dim == 1) { k_edges<1><<<blocks, 256, 0, s>>>(c->g, phi, edges, part); count_launch(); }
    else if (c->g.dim == 2) { k_edges<2><<<blocks, 256, 0, s>>>(c->g, phi, edges, part); count_launch(); }
    else { k_edges<3><<<blocks, 256, 0, s>>>(c->g, phi, edges, part); count_launch(); }
}

// Kinetic-energy partials of species si for a push launched with `blocks`
// blocks (in a step with diagnostics; null otherwise).
static double* kin_slot(psum_pic_ctx* c, int si, long long blocks) {
    if (!c->diag_in_step || si >= 8) return nullptr;
    auto& d = c->dbuf[c->diag_par];
    d.kin_n[si] = blocks;
    return d.kin.p + d.kin_off[si];
}

static void deposit_all(psum_pic_ctx* c) {
    zero_accumulators(c);
    for (int s = 0; s < (int)c->sp.size(); ++s) {
        Species& sp = *c->sp[s];
        if (sp.n <= 0) continue;
        if (c->precision == PSUM_PIC_MIXED) {
            ensure_keys(c, sp);
            PushArgs a = make_push_args(c, sp, s, 0.0, 0, nullptr);
            launch_mixed(a, c->g.dim, 0, true, sp.n, c->stream);
        } else {
            Deposit64Args a{};
            a.g = c->g;
            for (int d = 0; d < 3; ++d) a.pos[d] = d < c->g.dim ? sp.pos64[d][sp.cur].p : nullptr;
            a.count = c->count.p + s;
            a.acc = sp.acc.p;
            a.scale = std::ldexp(1.0, sp.dep_shift);
            deposit64(c, a, sp.n, c->stream);
        }
    }
    cuda_check(cudaGetLastError(), "deposit launch");
}

static void push_all(psum_pic_ctx* c, const double* phi, double dt, int pusher, const double* B) {
    if (!phi) throw std::invalid_argument("push: null phi");
    if (pusher != PSUM_PIC_LEAPFROG && pusher != PSUM_PIC_BORIS) throw std::invalid_argument("push: unknown pusher");
    if (!(std::isfinite(dt))) throw Error(PSUM_ERR_NONFINITE, "push: non-finite dt");
    cudaStream_t s = c->stream;
    zero_accumulators(c);
    launch_edges(c, phi, s);
    for (int si = 0; si < (int)c->sp.size(); ++si) {
        Species& sp = *c->sp[si];
        if (sp.n <= 0) continue;
        sp.sorted = false;   // moved in place
        if (c->precision == PSUM_PIC_MIXED) {
            ensure_keys(c, sp);
            PushArgs a = make_push_args(c, sp, si, dt, pusher, B);
            a.kin_part = kin_slot(c, si, capped_blocks(4LL * kPicThreads, sp.n));
            launch_mixed(a, c->g.dim, pusher, false, sp.n, s);
        } else {
            Push64Args a{};
            a.g = c->g;
            for (int d = 0; d < 3; ++d) {
                a.hi[d] = c->g.lo[d] + c->g.cells[d] * c->g.dx[d];
                a.pos[d] = d < c->g.dim ? sp.pos64[d][sp.cur].p : nullptr;
                a.vel[d] = sp.vel64[d][sp.cur].p;
                a.B[d] = B ? B[d] : 0.0;
            }
            a.key = sp.key[sp.cur].p;
            a.count = c->count.p + si;
            a.phi = phi;
            a.q_m = sp.q / sp.m;
            a.dt = dt;
            a.pusher = pusher;
            a.acc = sp.acc.p;
            a.scale = std::ldexp(1.0, sp.dep_shift);
            a.losses = c->losses.p + (size_t)si * 6;
            a.err = c->err.p;
            a.kin_part = kin_slot(c, si, fp64_exact::push64_blocks(sp.n));
            a.kin_hmw = 0.5 * sp.m * sp.w;
            push64(c, a, sp.n, s);
        }
    }
    cuda_check(cudaGetLastError(), "push launch");
}

static void sort_all(psum_pic_ctx* c) {
    for (int s = 0; s < (int)c->sp.size(); ++s) sort_species(c, *c->sp[s], s);
}

namespace {
struct PhaseTimer {
    psum_pic_ctx* c;
    int phase;
    cudaEvent_t a = nullptr, b = nullptr;
    PhaseTimer(psum_pic_ctx* ctx, int ph) : c(ctx), phase(ph) {
        if (!c->timing) return;
        cuda_check(cudaEventCreate(&a), "cudaEventCreate");
        cuda_check(cudaEventCreate(&b), "cudaEventCreate");
        cuda_check(cudaEventRecord(a, c->stream), "cudaEventRecord");
    }
    void stop() {
        if (!c->timing) return;
        cuda_check(cudaEventRecord(b, c->stream), "cudaEventRecord");
        c->events.push_back({phase, {a, b}});
    }
};
}  // namespace

// One fused sorted step (push + deposit + re-sort) of every species; see
// k_cls_pass1 / k_cls_pass2.  Species in which some particle moved more
// than one cell along an axis take the general path (in-place push, radix
// sort) for this step; their deposit from pass 1 stands.
// blocks of the two tables for up to n particles over nc cells
// Pass-1 block size (log2 of the particles per block): cls_block_lg, and
// for dense 2-D species (mean p particles per cell) the largest power of
// two up to 128 p, at most 2^15, so that a block's three-row cell box
// (3 x (2^lg / p + 2) cells) stays inside the tile: fewer blocks, less
// per-block work.
static int cls_lg1(long long n, long long nc, int dim) {
    if (dim != 2) return cls_block_lg(dim);
    const double ppc = nc > 0 ? (double)n / (double)nc : 0.0;
    int lg = cls_block_lg(dim);
    while (lg < 15 && (double)(1LL << (lg + 1)) <= 128.0 * ppc) ++lg;
    return lg;
}
static long long cls_blocks(long long n, long long nc, int dim) {
    const int lg = cls_lg1(n, nc, dim);
    return ((n + nc * cls_cell_weight(lg)) >> lg) + 1;
}
static long long cls_blocks2(long long n, long long nc, int dim) {
    return ((n + nc * cls_cell_weight(cls_block_lg2(dim))) >> cls_block_lg2(dim)) + 1;
}

template <int D, int P, int R>
static void launch_pass_t(const ClsArgs& a, int pass, unsigned blocks, cudaStream_t s) {
    if (pass == 1) {
        constexpr size_t bytes = CellTileCap<D>::BYTES;
        static bool attr = false;
        if (!attr) {
            cuda_check(cudaFuncSetAttribute(k_cls_pass1<D, P, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes),
                       "cudaFuncSetAttribute");
            attr = true;
        }
        { k_cls_pass1<D, P, R><<<blocks, kPicThreads, bytes, s>>>(a); count_launch(); }
    } else {
        { k_cls_pass2<D, P, R><<<blocks, kPicThreads, 0, s>>>(a); count_launch(); }
    }
}

template <int D, int P>
static void launch_pass_r(const ClsArgs& a, int pass, unsigned blocks, int rounds, cudaStream_t s) {
    if (rounds == 1) launch_pass_t<D, P, 1>(a, pass, blocks, s);
    else launch_pass_t<D, P, kClsRoundsMax>(a, pass, blocks, s);
}

static void launch_pass(const ClsArgs& a, int dim, int pusher, int pass, long long n, cudaStream_t s) {
    const unsigned blocks = (unsigned)(pass == 1 ? cls_blocks(n, a.n_cells, dim) : cls_blocks2(n, a.n_cells, dim));
    const int rounds = cls_rounds((double)n / (double)a.n_cells);
    if (dim == 2) {
        if (pusher == PSUM_PIC_BORIS) launch_pass_r<2, PSUM_PIC_BORIS>(a, pass, blocks, rounds, s);
        else launch_pass_r<2, PSUM_PIC_LEAPFROG>(a, pass, blocks, rounds, s);
    } else {
        if (pusher == PSUM_PIC_BORIS) launch_pass_r<3, PSUM_PIC_BORIS>(a, pass, blocks, rounds, s);
        else launch_pass_r<3, PSUM_PIC_LEAPFROG>(a, pass, blocks, rounds, s);
    }
}

template <class T>
static void grow(DevBuf<T>& b, size_t count) {
    if (b.n < count) b.alloc(count);
}

static void ensure_cls_buffers(psum_pic_ctx* c) {
    const long long nc = c->g.n_cells;
    const int ncls = c->g.dim == 2 ? 9 : 27;
    for (auto& spp : c->sp) {
        Species& sp = *spp;
        if (sp.n <= 0) continue;
        grow(sp.cls_count, (size_t)nc * ncls);
        grow(sp.cls_first, (size_t)cls_blocks(sp.n, nc, c->g.dim) + 1);
        grow(sp.cls_first2, (size_t)cls_blocks2(sp.n, nc, c->g.dim) + 1);
        grow(sp.newcount, (size_t)nc + 1);
        grow(sp.scan_tmp1, (size_t)(nc + 1 + kScanBlock - 1) / kScanBlock + 1);
        grow(sp.scan_tmp2, (size_t)((nc + 1 + kScanBlock - 1) / kScanBlock + kScanBlock - 1) / kScanBlock + 16);
    }
    grow(c->far_flag, 8);
    if (!c->side) {
        int least = 0, greatest = 0;
        cuda_check(cudaDeviceGetStreamPriorityRange(&least, &greatest), "cudaDeviceGetStreamPriorityRange");
        cuda_check(cudaStreamCreateWithPriority(&c->side, cudaStreamNonBlocking, least), "cudaStreamCreate");
    }
    if (!c->ev_pass1) cuda_check(cudaEventCreateWithFlags(&c->ev_pass1, cudaEventDisableTiming), "cudaEventCreate");
    if (!c->ev_pass2) cuda_check(cudaEventCreateWithFlags(&c->ev_pass2, cudaEventDisableTiming), "cudaEventCreate");
    if (!c->far_host) cuda_check(cudaHostAlloc(&c->far_host, sizeof(int) * 8, cudaHostAllocDefault), "cudaHostAlloc");
}

// The fused step needs distinct source cells for the classes arriving in a
// cell: at least 3 internal cells on every periodic axis.
static bool cls_step_applies(const psum_pic_ctx* c) {
    if (c->g.dim < 2) return false;   // 1-D runs the general path (in-place push, stable sort)
    for (int a = 0; a < c->g.dim; ++a)
        if (c->g.periodic[a] && c->g.M[a] < 3) return false;
    return true;
}

// First passes of every species (push, deposit, per-group counts), the
// group offsets and the new cell offsets on the context stream; then the
// second passes (push again, write the re-sorted state) on the side stream.
// The step stays pending until finish_cls_step joins it: the caller can
// meanwhile enqueue work that needs only the deposit and the loss counts
// (the next step's charge density and Poisson solve).
static void cls_step(psum_pic_ctx* c, const double* phi, double dt, int pusher, const double* B) {
    cudaStream_t s = c->stream;
    ensure_cls_buffers(c);
    // timed in two parts: the context stream's first passes, then the side stream's second passes
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    if (c->timing) {
        cuda_check(cudaEventCreate(&t0), "cudaEventCreate");
        cuda_check(cudaEventCreate(&t1), "cudaEventCreate");
        cuda_check(cudaEventRecord(t0, s), "cudaEventRecord");
    }
    zero_accumulators(c);
    launch_edges(c, phi, s);
    cuda_check(cudaMemsetAsync(c->far_flag.p, 0, sizeof(int) * 8, s), "memset");
    const int ns = (int)c->sp.size();
    const long long nc = c->g.n_cells;
    std::vector<ClsArgs> args(ns);
    for (int si = 0; si < ns; ++si) {
        Species& sp = *c->sp[si];
        if (sp.n <= 0) continue;
        ClsArgs& a = args[si];
        a.p = make_push_args(c, sp, si, dt, pusher, B);
        a.starts = sp.starts[sp.starts_cur].p;
        a.block_first = sp.cls_first.p;
        a.cls = sp.cls_count.p;
        a.new_starts = sp.starts[1 - sp.starts_cur].p;
        a.far = c->far_flag.p + si;
        const int nxt = 1 - sp.cur;
        for (int d = 0; d < 3; ++d) {
            a.off_out[d] = d < c->g.dim ? sp.off[d][nxt].p : nullptr;
            a.vel_out[d] = sp.vel[d][nxt].p;
        }
        a.n_cells = nc;
        const long long nb = cls_blocks(sp.n, nc, c->g.dim);
        { k_cls_blocks<<<blocks_for(std::max(nc, nb) + 1, 256), 256, 0, s>>>(a.starts, nc, nb,
                                                                             cls_lg1(sp.n, nc, c->g.dim),
                                                                             sp.cls_first.p); count_launch(); }
        launch_pass(a, c->g.dim, pusher, 1, sp.n, s);
        const long long nb2 = cls_blocks2(sp.n, nc, c->g.dim);
        { k_cls_blocks<<<blocks_for(std::max(nc, nb2) + 1, 256), 256, 0, s>>>(a.starts, nc, nb2, cls_block_lg2(c->g.dim),
                                                                              sp.cls_first2.p); count_launch(); }
        if (c->g.dim == 2) { k_cls_offsets<2><<<blocks_for(nc + 1, 256), 256, 0, s>>>(c->g, sp.cls_count.p, sp.newcount.p, nc); count_launch(); }
        else { k_cls_offsets<3><<<blocks_for(nc + 1, 256), 256, 0, s>>>(c->g, sp.cls_count.p, sp.newcount.p, nc); count_launch(); }
        exclusive_scan_u32(sp.newcount.p, sp.starts[1 - sp.starts_cur].p, nc + 1, sp.scan_tmp1.p, sp.scan_tmp2.p, s,
                           (long long)sp.scan_tmp2.n);
    }
    cuda_check(cudaMemcpyAsync(c->far_host, c->far_flag.p, sizeof(int) * 8, cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaEventRecord(c->ev_pass1, s), "cudaEventRecord");
    if (c->timing) {
        cuda_check(cudaEventRecord(t1, s), "cudaEventRecord");
        c->events.push_back({2, {t0, t1}});   // push phase: the first passes, offsets and scans
    }
    cuda_check(cudaStreamWaitEvent(c->side, c->ev_pass1, 0), "cudaStreamWaitEvent");
    cudaEvent_t u0 = nullptr, u1 = nullptr;
    if (c->timing) {
        cuda_check(cudaEventCreate(&u0), "cudaEventCreate");
        cuda_check(cudaEventCreate(&u1), "cudaEventCreate");
        cuda_check(cudaEventRecord(u0, c->side), "cudaEventRecord");
    }
    for (int si = 0; si < ns; ++si) {
        if (c->sp[si]->n <= 0) continue;
        args[si].block_first = c->sp[si]->cls_first2.p;
        // the second pass sums the kinetic energy of the particles it writes
        args[si].p.kin_part = kin_slot(c, si, cls_blocks2(c->sp[si]->n, nc, c->g.dim) * kClsWarps);
        launch_pass(args[si], c->g.dim, pusher, 2, c->sp[si]->n, c->side);
    }
    if (c->timing) {
        cuda_check(cudaEventRecord(u1, c->side), "cudaEventRecord");
        c->events.push_back({2 | kPhaseContinued, {u0, u1}});   // push phase: the second passes
    }
    c->pend_diag = c->diag_in_step;
    c->pend_par = c->diag_par;
    if (c->diag_in_step) {
        // the step's diagnostics are reduced beside the next step's solve (the side stream runs
        // it after the second passes); a far-mover fallback at the join redoes it
        cudaStream_t keep = c->stream;
        c->stream = c->side;
        PhaseTimer t(c, 4);
        finish_diagnostics(c, c->diag_par);
        t.stop();
        c->stream = keep;
    }
    cuda_check(cudaEventRecord(c->ev_pass2, c->side), "cudaEventRecord");
    cuda_check(cudaGetLastError(), "fused step launch");
    c->pending = true;
    c->pend_dt = dt;
    c->pend_pusher = pusher;
    c->pend_has_B = B != nullptr;
    for (int d = 0; d < 3; ++d) c->pend_B[d] = B ? B[d] : 0.0;
}

// Joins a pending fused step: the context stream waits for the second
// passes, and each species either takes its re-sorted state or, when one of
// its particles moved more than one cell along an axis (its second pass then
// wrote nothing and its first pass left far movers out of the deposit),
// moves in place, is radix sorted and deposited again from the sorted state.
static void finish_cls_step(psum_pic_ctx* c) {
    if (!c->pending) return;
    c->pending = false;
    cudaStream_t s = c->stream;
    cuda_check(cudaStreamWaitEvent(s, c->ev_pass2, 0), "join second passes");
    cuda_check(cudaEventSynchronize(c->ev_pass1), "far flag wait");
    const int ns = (int)c->sp.size();
    bool redo_diag = false;   // a fallback rewrote a species' energy sums: the side stream's reduction is stale
    bool any_far = false;
    for (int si = 0; si < ns && si < 8; ++si) any_far |= c->sp[si]->n > 0 && c->far_host[si] != 0;
    if (any_far) {
        c->fused_skip = c->fused_backoff;
        c->fused_backoff = std::min(64, 2 * c->fused_backoff);
    } else {
        c->fused_backoff = 1;
    }
    for (int si = 0; si < ns; ++si) {
        Species& sp = *c->sp[si];
        if (sp.n <= 0) continue;
        if (!c->far_host[si]) {
            { k_count_from<<<1, 1, 0, s>>>(c->count.p + si, sp.starts[1 - sp.starts_cur].p + c->g.n_cells); count_launch(); }
            sp.cur = 1 - sp.cur;
            sp.starts_cur = 1 - sp.starts_cur;
            sp.keys_stale = true;
            continue;
        }
        // timed as the sort phase: the cost of a step in which a particle moved too far
        PhaseTimer t(c, 3);
        ensure_keys(c, sp);
        PushArgs pa = make_push_args(c, sp, si, c->pend_dt, c->pend_pusher, c->pend_has_B ? c->pend_B : nullptr);
        pa.acc = nullptr;
        pa.losses = c->losses.p + 6 * 8;   // discard slot: pass 1 already counted this step's losses
        if (c->pend_diag && si < 8) {      // the second pass wrote nothing: the move in place sums the energy
            auto& d = c->dbuf[c->pend_par];
            d.kin_n[si] = capped_blocks(4LL * kPicThreads, sp.n);
            pa.kin_part = d.kin.p + d.kin_off[si];
            redo_diag = true;
        }
        launch_mixed(pa, c->g.dim, c->pend_pusher, false, sp.n, s);
        sort_species(c, sp, si);
        cuda_check(cudaMemsetAsync(sp.acc.p, 0, sizeof(unsigned long long) * c->g.n_nodes, s), "memset acc");
        ensure_keys(c, sp);
        PushArgs da = make_push_args(c, sp, si, 0.0, 0, nullptr);
        launch_mixed(da, c->g.dim, 0, true, sp.n, s);
        t.stop();
    }
    if (c->pend_diag && redo_diag) {
        PhaseTimer t(c, 4);
        finish_diagnostics(c, c->pend_par);
        t.stop();
    }
    c->pend_diag = false;
    cuda_check(cudaGetLastError(), "fused step finish");
}

static void rho_into(psum_pic_ctx* c, double background, double* rho, int only_species, bool with_charge) {
    if (!rho) throw std::invalid_argument("rho: null output");
    RhoArgs a{};
    a.background = background;
    double vol = 1.0;
    for (int d = 0; d < c->g.dim; ++d) vol *= c->g.dx[d];
    for (int s = 0; s < (int)c->sp.size(); ++s) {
        if (only_species >= 0 && s != only_species) continue;
        if (a.ns >= 8) throw Error(PSUM_ERR_INVALID_ARGUMENT, "rho: more than 8 species");
        Species& sp = *c->sp[s];
        a.acc[a.ns] = sp.acc.p;
        a.coef[a.ns] = (with_charge ? sp.q : 1.0) * sp.w / vol * std::ldexp(1.0, -sp.dep_shift);
        a.ns++;
    }
    // in a step with diagnostics the density also sums the charge it holds
    if (c->diag_in_step && only_species < 0 && with_charge) {
        a.qsum = c->dbuf[c->diag_par].qsum.p;
        cuda_check(cudaMemsetAsync(a.qsum, 0, sizeof(unsigned long long) * 8, c->stream), "memset qsum");
    }
    { k_rho<<<blocks_for(c->g.n_nodes, 256), 256, 0, c->stream>>>(a, rho, c->g.n_nodes); count_launch(); }
    cuda_check(cudaGetLastError(), "rho launch");
}

// Buffers of the per-step diagnostics, sized for the largest push grid of
// every species (fused first pass, general mixed push, FP64 push).
static void ensure_diag_buffers(psum_pic_ctx* c) {
    auto& d = c->dbuf[c->diag_par];
    grow(d.fe, (size_t)blocks_for(c->g.n_nodes, 256));
    long long off = 0;
    for (int s = 0; s < (int)c->sp.size() && s < 8; ++s) {
        const long long n = std::max<long long>(c->sp[s]->n, 1);
        d.kin_off[s] = off;
        d.kin_n[s] = 0;
        off += std::max({cls_blocks2(n, c->g.n_cells, c->g.dim) * kClsWarps, (long long)capped_blocks(4LL * kPicThreads, n),
                         fp64_exact::push64_blocks(n), (long long)blocks_for(n, kPicThreads)});
    }
    grow(d.kin, (size_t)std::max<long long>(off, 1));
    grow(d.qsum, 8);
    grow(d.stage, (size_t)kDiagStageBlocks * 10);
    grow(c->diag_out, 16);
    d.fe_n = 0;
    d.rho_n = 0;
    cuda_check(cudaMemsetAsync(d.qsum.p, 0, sizeof(unsigned long long) * 8, c->stream), "memset qsum");
}

// Reduces the step's partial sums into diag_out (context stream, after the push).
static void finish_diagnostics(psum_pic_ctx* c, int par) {
    const auto& d = c->dbuf[par];
    DiagFinishArgs a{};
    a.fe_part = d.fe_n ? d.fe.p : nullptr;
    a.fe_n = d.fe_n;
    double vol = 1.0;
    for (int d = 0; d < c->g.dim; ++d) vol *= c->g.dx[d];
    a.fe_coef = 0.5 * vol;
    a.ns = std::min<int>((int)c->sp.size(), 8);
    for (int s = 0; s < a.ns; ++s) {
        Species& sp = *c->sp[s];
        a.kin_part[s] = d.kin_n[s] ? d.kin.p + d.kin_off[s] : nullptr;
        a.kin_n[s] = d.kin_n[s];
        a.q_coef[s] = sp.q * sp.w * std::ldexp(1.0, -sp.dep_shift);
    }
    a.qsum = d.qsum.p;
    a.rho_part = d.rho_n ? d.rho_part.p : nullptr;
    a.rho_n = d.rho_n;
    a.rho_coef = vol;
    a.out = c->diag_out.p;
    // two levels: slices of every partial array, then the slices' sums
    double* stage = c->dbuf[par].stage.p;
    { k_diag_stage<<<dim3(kDiagStageBlocks, a.ns + 2), kDiagFinishThreads, 0, c->stream>>>(a, stage); count_launch(); }
    DiagFinishArgs b = a;
    for (int s = 0; s < a.ns; ++s) {
        b.kin_part[s] = a.kin_part[s] ? stage + (long long)s * kDiagStageBlocks : nullptr;
        b.kin_n[s] = a.kin_part[s] ? kDiagStageBlocks : 0;
    }
    b.fe_part = a.fe_part ? stage + (long long)a.ns * kDiagStageBlocks : nullptr;
    b.fe_n = a.fe_part ? kDiagStageBlocks : 0;
    b.rho_part = a.rho_part ? stage + (long long)(a.ns + 1) * kDiagStageBlocks : nullptr;
    b.rho_n = a.rho_part ? kDiagStageBlocks : 0;
    { k_diag_finish<<<1, kDiagFinishThreads, 0, c->stream>>>(b); count_launch(); }
    cuda_check(cudaGetLastError(), "diagnostics launch");
}

// Charge density of a step with interp_order > 1: rho = background plus the
// B-spline deposit (add_back_B_spline, higher_order_interp.hpp:196-247) of
// every species' current positions, exported to bs_pos (kept for the push).
static void rho_bspline(psum_pic_ctx* c, double background, double* rho) {
    cudaStream_t s = c->stream;
    const long long nn = c->g.n_nodes;
    { k_fill<<<blocks_for(nn, 256), 256, 0, s>>>(rho, nn, background); count_launch(); }
    grow(c->bs_acc, (size_t)nn);
    double vol = 1.0;
    for (int d = 0; d < c->g.dim; ++d) vol *= c->g.dx[d];
    for (int si = 0; si < (int)c->sp.size(); ++si) {
        Species& sp = *c->sp[si];
        if (sp.n <= 0) continue;
        if (si >= 8) throw Error(PSUM_ERR_INVALID_ARGUMENT, "interp_order: more than 8 species");
        if (c->precision == PSUM_PIC_MIXED) ensure_keys(c, sp);
        grow(c->bs_pos[si], (size_t)sp.n * c->g.dim);
        const int cur = sp.cur;
        const bool mixed = c->precision == PSUM_PIC_MIXED;
        { k_state_positions<<<blocks_for(sp.n, 256), 256, 0, s>>>(
              c->g, mixed ? 1 : 0, mixed ? sp.key[cur].p : nullptr, mixed ? sp.off[0][cur].p : nullptr,
              mixed && c->g.dim > 1 ? sp.off[1][cur].p : nullptr, mixed && c->g.dim > 2 ? sp.off[2][cur].p : nullptr,
              mixed ? nullptr : sp.pos64[0][cur].p, !mixed && c->g.dim > 1 ? sp.pos64[1][cur].p : nullptr,
              !mixed && c->g.dim > 2 ? sp.pos64[2][cur].p : nullptr, c->count.p + si, sp.n, c->bs_pos[si].p); count_launch(); }
        const int st = psum_add_back_bspline(&c->desc, c->interp_order, (unsigned long long)sp.n, c->bs_pos[si].p,
                                             sp.q * sp.w / vol, rho, c->bs_acc.p, nullptr, s);
        if (st != PSUM_OK) throw Error(st, "interp_order: B-spline deposit failed");
    }
    if (c->diag_in_step) {   // the charge of this density, for the step's diagnostics
        auto& d = c->dbuf[c->diag_par];
        const long long nb = blocks_for(nn, 256);
        grow(d.rho_part, (size_t)nb);
        d.rho_n = nb;
        { k_rho_charge<<<(unsigned)nb, 256, 0, s>>>(rho, nn, background, d.rho_part.p); count_launch(); }
    }
    cuda_check(cudaGetLastError(), "rho_bspline launch");
}

// Push of a step with interp_order > 1: the B-spline gradient gather
// (interp_diff_B_spline) of phi at the positions rho_bspline exported, then
// the push with that field (no CIC gather, no deposit) in place.
static void push_bspline(psum_pic_ctx* c, const double* phi, double dt, int pusher, const double* B) {
    if (!(std::isfinite(dt))) throw Error(PSUM_ERR_NONFINITE, "push: non-finite dt");
    cudaStream_t s = c->stream;
    launch_edges(c, phi, s);   // field-energy sums of a step with diagnostics
    for (int si = 0; si < (int)c->sp.size(); ++si) {
        Species& sp = *c->sp[si];
        if (sp.n <= 0) continue;
        sp.sorted = false;
        grow(c->bs_grad, (size_t)sp.n * c->g.dim);
        const int st = psum_interp_diff_bspline(&c->desc, c->interp_order, (unsigned long long)sp.n,
                                                c->bs_pos[si].p, phi, c->bs_grad.p, nullptr, s);
        if (st != PSUM_OK) throw Error(st, "interp_order: B-spline gather failed");
        if (c->precision == PSUM_PIC_MIXED) {
            PushArgs a = make_push_args(c, sp, si, dt, pusher, B);
            a.acc = nullptr;
            const unsigned nb = blocks_for(sp.n, kPicThreads);
            a.kin_part = kin_slot(c, si, nb);
            const int D = c->g.dim;
            const bool boris = pusher == PSUM_PIC_BORIS;
#define PSUM_PG(DD, PP) k_push_grad_mixed<DD, PP><<<nb, kPicThreads, 0, s>>>(a, c->bs_grad.p, sp.n)
            if (D == 1) { if (boris) PSUM_PG(1, PSUM_PIC_BORIS); else PSUM_PG(1, PSUM_PIC_LEAPFROG); }
            else if (D == 2) { if (boris) PSUM_PG(2, PSUM_PIC_BORIS); else PSUM_PG(2, PSUM_PIC_LEAPFROG); }
            else { if (boris) PSUM_PG(3, PSUM_PIC_BORIS); else PSUM_PG(3, PSUM_PIC_LEAPFROG); }
#undef PSUM_PG
            count_launch();
        } else {
            Push64Args a{};
            a.g = c->g;
            for (int d = 0; d < 3; ++d) {
                a.hi[d] = c->g.lo[d] + c->g.cells[d] * c->g.dx[d];
                a.pos[d] = d < c->g.dim ? sp.pos64[d][sp.cur].p : nullptr;
                a.vel[d] = sp.vel64[d][sp.cur].p;
                a.B[d] = B ? B[d] : 0.0;
            }
            a.key = sp.key[sp.cur].p;
            a.count = c->count.p + si;
            a.phi = phi;
            a.q_m = sp.q / sp.m;
            a.dt = dt;
            a.pusher = pusher;
            a.acc = nullptr;
            a.scale = 0.0;
            a.losses = c->losses.p + (size_t)si * 6;
            a.err = c->err.p;
            a.kin_part = kin_slot(c, si, fp64_exact::push64_blocks(sp.n));
            a.kin_hmw = 0.5 * sp.m * sp.w;
            a.grad = c->bs_grad.p;
            a.grad_stride = sp.n;
            push64(c, a, sp.n, s);
        }
    }
    cuda_check(cudaGetLastError(), "push_bspline launch");
}

}  // namespace psum_b200

// =================================================================== ABI ==
using namespace psum_b200;

extern "C" {

EXPORT int psum_pic_create(const psum_pic_grid_desc* gd, int precision, psum_pic_ctx** out) {
    return guarded([&] {
        if (!gd || !out) throw std::invalid_argument("psum_pic_create: null argument");
        *out = nullptr;
        if (gd->dim < 1 || gd->dim > 3) throw std::invalid_argument("psum_pic_create: dim must be 1, 2 or 3");
        if (precision != PSUM_PIC_MIXED && precision != PSUM_PIC_FP64)
            throw std::invalid_argument("psum_pic_create: unknown precision");
        auto c = std::make_unique<psum_pic_ctx>();
        c->desc = *gd;
        GridView& g = c->g;
        g.dim = gd->dim;
        long long nn = 1, nc = 1;
        for (int a = 0; a < 3; ++a) {
            if (a < gd->dim) {
                if (gd->cells[a] < 1) throw std::invalid_argument("psum_pic_create: cells must be positive");
                if (!(gd->lower[a] < gd->upper[a])) throw std::invalid_argument("psum_pic_create: lower >= upper");
                g.cells[a] = gd->cells[a];
                g.periodic[a] = gd->periodic[a] ? 1 : 0;
                g.M[a] = g.periodic[a] ? g.cells[a] + 1 : g.cells[a];
                g.N[a] = g.cells[a] + 1;
                g.lo[a] = gd->lower[a];
                g.dx[a] = (gd->upper[a] - gd->lower[a]) / gd->cells[a];   // simple_grid.hpp:47
                g.dr[a] = 1.0 / g.dx[a];
            } else {
                g.cells[a] = g.M[a] = g.N[a] = 1;
                g.periodic[a] = 0;
                g.lo[a] = 0.0;
                g.dx[a] = g.dr[a] = 1.0;
            }
            nn *= g.N[a];
            nc *= g.M[a];
        }
        if (nc >= 0x7fffffffLL) throw std::invalid_argument("psum_pic_create: more than 2^31-1 cells");
        g.n_nodes = nn;
        g.n_cells = nc;
        g.div_m12 = make_fastdiv((unsigned)(g.M[1] * g.M[2]));
        g.div_m2 = make_fastdiv((unsigned)g.M[2]);
        c->precision = precision;
        cuda_check(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking), "cudaStreamCreate");
        c->stream = c->own_stream;
        if (precision == PSUM_PIC_MIXED) c->edges.alloc((size_t)nn * (g.dim <= 2 ? 2 : 4));
        c->losses.alloc(9 * 6);   // 8 species + one discard slot
        c->err.alloc(1);
        c->count.alloc(8);
        c->partials.alloc(kDiagBlocks);
        c->ipartials.alloc(1);
        cuda_check(cudaMemsetAsync(c->losses.p, 0, sizeof(unsigned long long) * 48, c->stream), "memset");
        cuda_check(cudaMemsetAsync(c->err.p, 0, sizeof(unsigned), c->stream), "memset");
        cuda_check(cudaMemsetAsync(c->count.p, 0, sizeof(long long) * 8, c->stream), "memset");
        cuda_check(cudaStreamSynchronize(c->stream), "create sync");
        *out = c.release();
    });
}

EXPORT int psum_pic_destroy(psum_pic_ctx* ctx) {
    return guarded([&] {
        if (!ctx) return;
        ctx_check(ctx);
        cudaStreamSynchronize(ctx->stream);
        ctx->magic = 0;
        delete ctx;
    });
}

EXPORT int psum_pic_set_stream(psum_pic_ctx* ctx, void* stream) {
    return guarded([&] {
        ctx_check(ctx);
        // work already enqueued on the old stream completes before the new one is used
        cuda_check(cudaStreamSynchronize(ctx->stream), "set_stream sync");
        ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
    });
}

EXPORT int psum_pic_join(psum_pic_ctx* ctx) {
    return guarded([&] { ctx_check(ctx); });
}

EXPORT int psum_pic_set_options(psum_pic_ctx* ctx, const char* options) {
    return guarded([&] {
        ctx_check(ctx);
        if (!options) throw std::invalid_argument("set_options: null option string");
        std::istringstream iss(options);
        std::string key;
        while (iss >> key) {
            int v;
            if (!(iss >> v)) throw std::invalid_argument("set_options: option '" + key + "' needs an integer value");
            if (key == "sort_interval") {
                if (v < 0) throw std::invalid_argument("sort_interval must be >= 0");
                ctx->sort_interval = v;
            } else if (key == "interp_order") {
                if (v < 1 || v > 4) throw std::invalid_argument("interp_order must be 1, 2, 3 or 4");
                ctx->interp_order = v;
            } else if (key == "fp64_fma") {
                if (v != 0 && v != 1) throw std::invalid_argument("fp64_fma must be 0 or 1");
                ctx->fp64_fma = v != 0;
            } else if (key == "diagnostics") {
                if (v != 0 && v != 1) throw std::invalid_argument("diagnostics must be 0 or 1");
                ctx->diag = v != 0;
            } else {
                throw std::invalid_argument("set_options: unknown particle option '" + key + "'");
            }
        }
    });
}

EXPORT int psum_pic_add_species(psum_pic_ctx* ctx, const psum_pic_species_desc* d, unsigned long long capacity,
                                int* id) {
    return guarded([&] {
        ctx_check(ctx);
        if (!d || !id) throw std::invalid_argument("add_species: null argument");
        if (ctx->sp.size() >= 8) throw std::invalid_argument("add_species: at most 8 species");
        if (!(d->mass > 0) || !std::isfinite(d->charge) || !std::isfinite(d->weight))
            throw std::invalid_argument("add_species: mass must be positive, charge and weight finite");
        if (capacity == 0 || capacity >= 0x7fffffffULL) throw std::invalid_argument("add_species: capacity out of range");
        auto sp = std::make_unique<Species>();
        sp->q = d->charge;
        sp->m = d->mass;
        sp->w = d->weight;
        sp->cap = (long long)((capacity + 3) & ~3ULL);
        // fixed point: every node sum stays below 2^62 even if all particles share one node
        sp->dep_shift = 62 - bits_for((unsigned long long)sp->cap);
        if (ctx->precision == PSUM_PIC_MIXED && sp->dep_shift < kCicBits)
            throw Error(PSUM_ERR_INVALID_ARGUMENT, "add_species: capacity above 2^36 particles");
        alloc_species_state(ctx, *sp);
        ctx->sp.push_back(std::move(sp));
        *id = (int)ctx->sp.size() - 1;
        cuda_check(cudaStreamSynchronize(ctx->stream), "add_species sync");
    });
}

static void load_common(psum_pic_ctx* ctx, int species, unsigned long long n, const double* pos_dev,
                        const double* vel_dev) {
    Species& sp = species_at(ctx, species);
    if ((long long)n > sp.cap) throw Error(PSUM_ERR_OVERFLOW, "load: more particles than the species capacity");
    cudaStream_t s = ctx->stream;
    sp.cur = 0;
    if (n > 0) {
        const unsigned gb = blocks_for((long long)n, 256);
        if (ctx->precision == PSUM_PIC_MIXED) {
            { k_load_mixed<<<gb, 256, 0, s>>>(ctx->g, (long long)n, pos_dev, vel_dev, sp.key[0].p, sp.off[0][0].p,
                                            ctx->g.dim > 1 ? sp.off[1][0].p : nullptr,
                                            ctx->g.dim > 2 ? sp.off[2][0].p : sp.off[0][1].p, sp.vel[0][0].p,
                                            sp.vel[1][0].p, sp.vel[2][0].p); count_launch(); }
        } else {
            { k_load64<<<gb, 256, 0, s>>>(ctx->g, (long long)n, pos_dev, vel_dev, sp.pos64[0][0].p,
                                        ctx->g.dim > 1 ? sp.pos64[1][0].p : nullptr,
                                        ctx->g.dim > 2 ? sp.pos64[2][0].p : sp.pos64[0][1].p, sp.vel64[0][0].p,
                                        sp.vel64[1][0].p, sp.vel64[2][0].p); count_launch(); }
        }
    }
    { k_set_count<<<1, 1, 0, s>>>(ctx->count.p + species, (long long)n); count_launch(); }
    sp.n = (long long)n;
    sp.sorted = false;
    sp.keys_stale = false;
    if (ctx->precision == PSUM_PIC_FP64 && n > 0) {
        double* p3[3] = {sp.pos64[0][0].p, ctx->g.dim > 1 ? sp.pos64[1][0].p : nullptr,
                         ctx->g.dim > 2 ? sp.pos64[2][0].p : nullptr};
        keys64(ctx, p3, sp.key[0].p, ctx->count.p + species, (long long)n, s);
    }
    cuda_check(cudaGetLastError(), "load launch");
}

// Appends n particles after the stored ones, in the current buffers (the
// insert of particle_group.hpp:103-167; this library's groups have no holes,
// so the new particles go to the end).  The species is unsorted afterwards:
// the next sort, or the next step, re-sorts it.
static void append_common(psum_pic_ctx* ctx, int species, unsigned long long n, const double* pos_dev,
                          const double* vel_dev) {
    Species& sp = species_at(ctx, species);
    cudaStream_t s = ctx->stream;
    if (ctx->precision == PSUM_PIC_MIXED) ensure_keys(ctx, sp);
    long long cnt = 0;
    cuda_check(cudaMemcpyAsync(&cnt, ctx->count.p + species, sizeof(long long), cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaStreamSynchronize(s), "append sync");
    if (cnt + (long long)n > sp.cap) throw Error(PSUM_ERR_OVERFLOW, "append: more particles than the species capacity");
    const int c = sp.cur;
    if (n > 0) {
        const unsigned gb = blocks_for((long long)n, 256);
        if (ctx->precision == PSUM_PIC_MIXED) {
            { k_load_mixed<<<gb, 256, 0, s>>>(ctx->g, (long long)n, pos_dev, vel_dev, sp.key[c].p + cnt,
                                            sp.off[0][c].p + cnt, ctx->g.dim > 1 ? sp.off[1][c].p + cnt : nullptr,
                                            ctx->g.dim > 2 ? sp.off[2][c].p + cnt : sp.off[0][1 - c].p,
                                            sp.vel[0][c].p + cnt, sp.vel[1][c].p + cnt, sp.vel[2][c].p + cnt); count_launch(); }
        } else {
            { k_load64<<<gb, 256, 0, s>>>(ctx->g, (long long)n, pos_dev, vel_dev, sp.pos64[0][c].p + cnt,
                                        ctx->g.dim > 1 ? sp.pos64[1][c].p + cnt : nullptr,
                                        ctx->g.dim > 2 ? sp.pos64[2][c].p + cnt : sp.pos64[0][1 - c].p,
                                        sp.vel64[0][c].p + cnt, sp.vel64[1][c].p + cnt, sp.vel64[2][c].p + cnt); count_launch(); }
        }
    }
    const long long total = cnt + (long long)n;
    { k_set_count<<<1, 1, 0, s>>>(ctx->count.p + species, total); count_launch(); }
    sp.n = total;
    sp.sorted = false;
    sp.keys_stale = false;
    if (ctx->precision == PSUM_PIC_FP64 && total > 0) {
        double* p3[3] = {sp.pos64[0][c].p, ctx->g.dim > 1 ? sp.pos64[1][c].p : nullptr,
                         ctx->g.dim > 2 ? sp.pos64[2][c].p : nullptr};
        keys64(ctx, p3, sp.key[c].p, ctx->count.p + species, total, s);
    }
    cuda_check(cudaGetLastError(), "append launch");
}

EXPORT int psum_pic_append(psum_pic_ctx* ctx, int species, unsigned long long n, const double* pos_host,
                           const double* vel_host) {
    return guarded([&] {
        ctx_check(ctx);
        if (n > 0 && (!pos_host || !vel_host)) throw std::invalid_argument("append: null host array");
        DevBuf<double> dp, dv;
        dp.upload(pos_host, (size_t)n * ctx->g.dim, ctx->stream);
        dv.upload(vel_host, (size_t)n * 3, ctx->stream);
        append_common(ctx, species, n, dp.p, dv.p);
        cuda_check(cudaStreamSynchronize(ctx->stream), "append sync");
    });
}

EXPORT int psum_pic_append_device(psum_pic_ctx* ctx, int species, unsigned long long n, const double* pos_dev,
                                  const double* vel_dev) {
    return guarded([&] {
        ctx_check(ctx);
        if (n > 0 && (!pos_dev || !vel_dev)) throw std::invalid_argument("append: null device array");
        cuda_check(cudaStreamSynchronize(ctx->stream), "append sync");
        append_common(ctx, species, n, pos_dev, vel_dev);
        cuda_check(cudaStreamSynchronize(ctx->stream), "append sync");
    });
}

EXPORT int psum_pic_load(psum_pic_ctx* ctx, int species, unsigned long long n, const double* pos_host,
                         const double* vel_host) {
    return guarded([&] {
        ctx_check(ctx);
        if (n > 0 && (!pos_host || !vel_host)) throw std::invalid_argument("load: null host array");
        const int D = ctx->g.dim;
        DevBuf<double> dp, dv;
        dp.upload(pos_host, (size_t)n * D, ctx->stream);
        dv.upload(vel_host, (size_t)n * 3, ctx->stream);
        load_common(ctx, species, n, dp.p, dv.p);
        cuda_check(cudaStreamSynchronize(ctx->stream), "load sync");
    });
}

EXPORT int psum_pic_load_device(psum_pic_ctx* ctx, int species, unsigned long long n, const double* pos_dev,
                                const double* vel_dev) {
    return guarded([&] {
        ctx_check(ctx);
        if (n > 0 && (!pos_dev || !vel_dev)) throw std::invalid_argument("load: null device array");
        // The caller may free or reuse pos_dev/vel_dev as soon as this returns
        // (PSuM's particle_group::insert is synchronous as well).
        cuda_check(cudaStreamSynchronize(ctx->stream), "load sync");   // prior work that may write them
        load_common(ctx, species, n, pos_dev, vel_dev);
        cuda_check(cudaStreamSynchronize(ctx->stream), "load sync");
    });
}

EXPORT int psum_pic_count(psum_pic_ctx* ctx, int species, unsigned long long* n_stored, unsigned long long* n_valid) {
    return guarded([&] {
        ctx_check(ctx);
        Species& sp = species_at(ctx, species);
        long long dc = 0;
        cuda_check(cudaMemcpyAsync(&dc, ctx->count.p + species, sizeof(long long), cudaMemcpyDeviceToHost, ctx->stream),
                   "count copy");
        cuda_check(cudaStreamSynchronize(ctx->stream), "count sync");
        sp.n = dc;
        if (n_stored) *n_stored = (unsigned long long)dc;
        if (n_valid) {
            ensure_keys(ctx, sp);
            std::vector<int> keys(dc);
            if (dc > 0)
                cuda_check(cudaMemcpy(keys.data(), sp.key[sp.cur].p, sizeof(int) * dc, cudaMemcpyDeviceToHost),
                           "keys copy");
            unsigned long long v = 0;
            for (long long i = 0; i < dc; ++i) v += keys[i] >= 0;
            *n_valid = v;
        }
    });
}

// The species state (n stored particles, storage order) as FP64 SoA device
// arrays pos[d*n + i], vel[c*n + i]; invalid particles get x = NaN.
static void export_state(psum_pic_ctx* ctx, Species& sp, long long n, double* pos, double* vel) {
    const int D = ctx->g.dim;
    const int cur = sp.cur;
    if (ctx->precision == PSUM_PIC_MIXED) {
        ensure_keys(ctx, sp);
        { k_export_mixed<<<blocks_for(n, 256), 256, 0, ctx->stream>>>(
            ctx->g, n, sp.key[cur].p, sp.off[0][cur].p, D > 1 ? sp.off[1][cur].p : nullptr,
            D > 2 ? sp.off[2][cur].p : nullptr, sp.vel[0][cur].p, sp.vel[1][cur].p, sp.vel[2][cur].p, pos, vel); count_launch(); }
    } else {
        for (int a = 0; a < D; ++a)
            cuda_check(cudaMemcpyAsync(pos + (size_t)a * n, sp.pos64[a][cur].p, sizeof(double) * n,
                                       cudaMemcpyDeviceToDevice, ctx->stream),
                       "copy");
        for (int q = 0; q < 3; ++q)
            cuda_check(cudaMemcpyAsync(vel + (size_t)q * n, sp.vel64[q][cur].p, sizeof(double) * n,
                                       cudaMemcpyDeviceToDevice, ctx->stream),
                       "copy");
    }
}

static long long stored_count(psum_pic_ctx* ctx, Species& sp, int species) {
    long long n = 0;
    cuda_check(cudaMemcpyAsync(&n, ctx->count.p + species, sizeof(long long), cudaMemcpyDeviceToHost, ctx->stream),
               "count copy");
    cuda_check(cudaStreamSynchronize(ctx->stream), "count sync");
    sp.n = n;
    return n;
}

EXPORT int psum_pic_get_state(psum_pic_ctx* ctx, int species, double* pos_host, double* vel_host) {
    return guarded([&] {
        ctx_check(ctx);
        Species& sp = species_at(ctx, species);
        const long long n = stored_count(ctx, sp, species);
        if (n == 0) return;
        if (!pos_host || !vel_host) throw std::invalid_argument("get_state: null host array");
        const int D = ctx->g.dim;
        DevBuf<double> dp, dv;
        dp.alloc((size_t)n * D);
        dv.alloc((size_t)n * 3);
        export_state(ctx, sp, n, dp.p, dv.p);
        cuda_check(cudaMemcpyAsync(pos_host, dp.p, sizeof(double) * n * D, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
        cuda_check(cudaMemcpyAsync(vel_host, dv.p, sizeof(double) * n * 3, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
        cuda_check(cudaStreamSynchronize(ctx->stream), "get_state sync");
    });
}

EXPORT int psum_pic_get_state_device(psum_pic_ctx* ctx, int species, double* pos_dev, double* vel_dev) {
    return guarded([&] {
        ctx_check(ctx);
        Species& sp = species_at(ctx, species);
        const long long n = stored_count(ctx, sp, species);
        if (n == 0) return;
        if (!pos_dev || !vel_dev) throw std::invalid_argument("get_state_device: null device array");
        export_state(ctx, sp, n, pos_dev, vel_dev);
        cuda_check(cudaGetLastError(), "export launch");
        cuda_check(cudaStreamSynchronize(ctx->stream), "get_state sync");
    });
}

// Device snapshot of a species' state (checkpoints of differentiable runs):
// stored count, then the arrays of the current buffer over the capacity.
static size_t state_bytes(const psum_pic_ctx* c, const Species& sp) {
    const size_t n = (size_t)sp.cap, D = (size_t)c->g.dim;
    if (c->precision == PSUM_PIC_MIXED) return 8 + n * (4 + 4 * D + 4 * 3);
    return 8 + n * (8 * D + 8 * 3 + 4);
}

static void state_copy(psum_pic_ctx* c, int species, char* base, bool save) {
    Species& sp = species_at(c, species);
    cudaStream_t s = c->stream;
    const size_t n = (size_t)sp.cap;
    const int D = c->g.dim, cur = sp.cur;
    size_t off = 0;
    auto move = [&](void* dev, size_t bytes) {
        if (save) cuda_check(cudaMemcpyAsync(base + off, dev, bytes, cudaMemcpyDeviceToDevice, s), "save state");
        else cuda_check(cudaMemcpyAsync(dev, base + off, bytes, cudaMemcpyDeviceToDevice, s), "restore state");
        off += bytes;
    };
    move(c->count.p + species, 8);
    if (c->precision == PSUM_PIC_MIXED) {
        move(sp.key[cur].p, 4 * n);
        for (int a = 0; a < D; ++a) move(sp.off[a][cur].p, 4 * n);
        for (int q = 0; q < 3; ++q) move(sp.vel[q][cur].p, 4 * n);
    } else {
        for (int a = 0; a < D; ++a) move(sp.pos64[a][cur].p, 8 * n);
        for (int q = 0; q < 3; ++q) move(sp.vel64[q][cur].p, 8 * n);
        move(sp.key[cur].p, 4 * n);
    }
}

EXPORT int psum_pic_state_bytes(psum_pic_ctx* ctx, int species, unsigned long long* bytes) {
    return guarded([&] {
        ctx_check(ctx);
        if (!bytes) throw std::invalid_argument("state_bytes: null output");
        *bytes = state_bytes(ctx, species_at(ctx, species));
    });
}

EXPORT int psum_pic_save_state(psum_pic_ctx* ctx, int species, void* dst_dev) {
    return guarded([&] {
        ctx_check(ctx);
        Species& sp = species_at(ctx, species);
        if (!dst_dev) throw std::invalid_argument("save_state: null destination");
        if (ctx->precision == PSUM_PIC_MIXED) ensure_keys(ctx, sp);
        state_copy(ctx, species, static_cast<char*>(dst_dev), true);
        cuda_check(cudaGetLastError(), "save state");
    });
}

EXPORT int psum_pic_restore_state(psum_pic_ctx* ctx, int species, const void* src_dev) {
    return guarded([&] {
        ctx_check(ctx);
        Species& sp = species_at(ctx, species);
        if (!src_dev) throw std::invalid_argument("restore_state: null source");
        state_copy(ctx, species, static_cast<char*>(const_cast<void*>(src_dev)), false);
        sp.sorted = false;      // cell offsets are not part of the snapshot
        sp.keys_stale = false;
        cuda_check(cudaGetLastError(), "restore state");
    });
}

EXPORT int psum_pic_get_keys(psum_pic_ctx* ctx, int species, int* keys_dev) {
    return guarded([&] {
        ctx_check(ctx);
        Species& sp = species_at(ctx, species);
        if (!keys_dev) throw std::invalid_argument("get_keys: null output");
        ensure_keys(ctx, sp);
        if (sp.n > 0)
            cuda_check(cudaMemcpyAsync(keys_dev, sp.key[sp.cur].p, sizeof(int) * sp.n, cudaMemcpyDeviceToDevice,
                                       ctx->stream),
                       "keys copy");
        cuda_check(cudaStreamSynchronize(ctx->stream), "keys sync");
    });
}

EXPORT int psum_pic_sort(psum_pic_ctx* ctx) {
    return guarded([&] {
        ctx_check(ctx);
        sort_all(ctx);
    });
}

EXPORT int psum_pic_bin(psum_pic_ctx* ctx, int species, long long* keys_dev, unsigned long long* counts_dev,
                        unsigned long long* offsets_dev, unsigned long long* perm_dev, unsigned long long* n_in_grid) {
    return guarded([&] {
        ctx_check(ctx);
        Species& sp = species_at(ctx, species);
        if (!keys_dev || !counts_dev || !offsets_dev || !perm_dev || !n_in_grid)
            throw std::invalid_argument("bin: null argument");
        cudaStream_t s = ctx->stream;
        const GridView& g = ctx->g;
        long long n = 0;
        cuda_check(cudaMemcpyAsync(&n, ctx->count.p + species, sizeof(long long), cudaMemcpyDeviceToHost, s), "count");
        cuda_check(cudaStreamSynchronize(s), "bin sync");
        long long ncell = 1;
        for (int a = 0; a < g.dim; ++a) ncell *= g.cells[a];
        const unsigned sentinel = (unsigned)ncell;
        ensure_sort_scratch(ctx, std::max<long long>(n, ncell));
        const int cur = sp.cur;
        if (n > 0) {
            if (ctx->precision == PSUM_PIC_MIXED) {
                ensure_keys(ctx, sp);
                { k_bin_keys_mixed<<<blocks_for(n, 256), 256, 0, s>>>(g, sp.key[cur].p, sp.off[0][cur].p, n, keys_dev,
                                                                     ctx->sort.keyA.p, ctx->sort.idxA.p, sentinel); count_launch(); }
            } else {
                DevBuf<double> hi;
                double h[3];
                for (int a = 0; a < 3; ++a) h[a] = g.lo[a] + g.cells[a] * g.dx[a];
                hi.upload(h, 3, s);
                { k_bin_keys64<<<blocks_for(n, 256), 256, 0, s>>>(g, sp.pos64[0][cur].p,
                                                                 g.dim > 1 ? sp.pos64[1][cur].p : nullptr,
                                                                 g.dim > 2 ? sp.pos64[2][cur].p : nullptr, n, keys_dev,
                                                                 ctx->sort.keyA.p, ctx->sort.idxA.p, sentinel, hi.p); count_launch(); }
                cuda_check(cudaStreamSynchronize(s), "bin keys");
            }
        }
        // counts per reference cell and their exclusive prefix
        DevBuf<unsigned> cnt, off;
        cnt.alloc(ncell);
        off.alloc(ncell);
        cuda_check(cudaMemsetAsync(cnt.p, 0, sizeof(unsigned) * ncell, s), "memset");
        if (n > 0) { k_hist_u32<<<blocks_for(n, 256), 256, 0, s>>>(keys_dev, n, cnt.p); count_launch(); }
        DevBuf<unsigned> t1, t2;
        t1.alloc((ncell + kScanBlock - 1) / kScanBlock + 1);
        t2.alloc(16);
        exclusive_scan_u32(cnt.p, off.p, ncell, t1.p, t2.p, s);
        { k_u32_to_u64<<<blocks_for(ncell, 256), 256, 0, s>>>(cnt.p, counts_dev, ncell); count_launch(); }
        { k_u32_to_u64<<<blocks_for(ncell, 256), 256, 0, s>>>(off.p, offsets_dev, ncell); count_launch(); }
        unsigned long long total = 0;
        if (n > 0) {
            unsigned* skeys;
            int* perm;
            radix_sort(ctx, n, sentinel, &skeys, &perm);
            // number of in-grid particles = sum of counts
            unsigned last_off = 0, last_cnt = 0;
            cuda_check(cudaMemcpyAsync(&last_off, off.p + ncell - 1, sizeof(unsigned), cudaMemcpyDeviceToHost, s), "D2H");
            cuda_check(cudaMemcpyAsync(&last_cnt, cnt.p + ncell - 1, sizeof(unsigned), cudaMemcpyDeviceToHost, s), "D2H");
            cuda_check(cudaStreamSynchronize(s), "bin sync");
            total = (unsigned long long)last_off + last_cnt;
            if (total > 0) { k_i32_to_u64<<<blocks_for((long long)total, 256), 256, 0, s>>>(perm, perm_dev, (long long)total); count_launch(); }
        }
        cuda_check(cudaStreamSynchronize(s), "bin sync");
        *n_in_grid = total;
    });
}

EXPORT int psum_pic_deposit(psum_pic_ctx* ctx) {
    return guarded([&] {
        ctx_check(ctx);
        deposit_all(ctx);
    });
}

EXPORT int psum_pic_rho(psum_pic_ctx* ctx, double background, double* rho_dev) {
    return guarded([&] {
        ctx_check(ctx);
        rho_into(ctx, background, rho_dev, -1, true);
    });
}

EXPORT int psum_pic_density(psum_pic_ctx* ctx, int species, double* n_dev) {
    return guarded([&] {
        ctx_check(ctx);
        species_at(ctx, species);
        rho_into(ctx, 0.0, n_dev, species, false);
    });
}

EXPORT int psum_pic_push(psum_pic_ctx* ctx, const double* phi_dev, double dt, int pusher, const double* B) {
    return guarded([&] {
        ctx_check(ctx);
        push_all(ctx, phi_dev, dt, pusher, B);
    });
}

EXPORT int psum_pic_get_losses(psum_pic_ctx* ctx, unsigned long long* losses_host, int reset) {
    return guarded([&] {
        ctx_check_nojoin(ctx);   // a fused step's counts are final after its first passes
        if (!losses_host) throw std::invalid_argument("get_losses: null output");
        std::vector<unsigned long long> all(48);
        cuda_check(cudaMemcpyAsync(all.data(), ctx->losses.p, sizeof(unsigned long long) * 48, cudaMemcpyDeviceToHost,
                                   ctx->stream),
                   "losses D2H");
        cuda_check(cudaStreamSynchronize(ctx->stream), "losses sync");
        const int D = ctx->g.dim;
        for (int s = 0; s < (int)ctx->sp.size(); ++s)
            for (int k = 0; k < 2 * D; ++k) losses_host[s * 2 * D + k] = all[s * 6 + k];
        if (reset)
            cuda_check(cudaMemsetAsync(ctx->losses.p, 0, sizeof(unsigned long long) * 48, ctx->stream), "memset");
    });
}


EXPORT int psum_pic_step(psum_pic_ctx* ctx, psum_field_solver_handle solver, double background, double* rho_dev,
                         double* phi_dev, double dt, int pusher, const double* B) {
    return guarded([&] {
        // the charge density and the solve need only the previous step's
        // first passes: its second passes may still run on the side stream
        ctx_check_nojoin(ctx);
        SolverBase* sv = solver_from_handle(solver);
        if (!rho_dev || !phi_dev) throw std::invalid_argument("step: null field");
        if (!ctx->prio) {
            int least = 0, greatest = 0;
            cuda_check(cudaDeviceGetStreamPriorityRange(&least, &greatest), "cudaDeviceGetStreamPriorityRange");
            cuda_check(cudaStreamCreateWithPriority(&ctx->prio, cudaStreamNonBlocking, greatest), "cudaStreamCreate");
            cuda_check(cudaEventCreateWithFlags(&ctx->ev_in, cudaEventDisableTiming), "cudaEventCreate");
            cuda_check(cudaEventCreateWithFlags(&ctx->ev_out, cudaEventDisableTiming), "cudaEventCreate");
        }
        // a pending step with a far mover finishes first: its deposit is redone
        if (ctx->pending) {
            cuda_check(cudaEventSynchronize(ctx->ev_pass1), "far flag wait");
            bool far = false;
            for (int si = 0; si < (int)ctx->sp.size() && si < 8; ++si) far |= ctx->far_host[si] != 0;
            if (far) finish_cls_step(ctx);
        }
        cudaStream_t user = ctx->stream;
        if (ctx->diag) {
            if (ctx->sp.size() > 8) throw std::invalid_argument("step diagnostics: more than 8 species");
            ctx->diag_par ^= 1;   // the pending step (if any) keeps the other buffers until it is joined
            ensure_diag_buffers(ctx);
        }
        ctx->diag_in_step = ctx->diag;
        struct DiagOff {
            psum_pic_ctx* c;
            ~DiagOff() { c->diag_in_step = false; }
        } diag_off{ctx};
        cuda_check(cudaEventRecord(ctx->ev_in, user), "cudaEventRecord");
        cuda_check(cudaStreamWaitEvent(ctx->prio, ctx->ev_in, 0), "cudaStreamWaitEvent");
        ctx->stream = ctx->prio;
        try {
            {
                PhaseTimer t(ctx, 0);
                if (ctx->interp_order > 1) rho_bspline(ctx, background, rho_dev);
                else rho_into(ctx, background, rho_dev, -1, true);
                t.stop();
            }
            {
                PhaseTimer t(ctx, 1);
                solver_solve_async(sv, rho_dev, phi_dev, ctx->prio);
                t.stop();
            }
        } catch (...) {
            ctx->stream = user;
            throw;
        }
        ctx->stream = user;
        cuda_check(cudaEventRecord(ctx->ev_out, ctx->prio), "cudaEventRecord");
        cuda_check(cudaStreamWaitEvent(user, ctx->ev_out, 0), "cudaStreamWaitEvent");
        finish_cls_step(ctx);
        bool fused = ctx->precision == PSUM_PIC_MIXED && ctx->sort_interval == 1 && cls_step_applies(ctx) &&
                     ctx->interp_order == 1;
        for (auto& sp : ctx->sp) fused = fused && (sp->sorted || sp->n == 0);
        if (fused && ctx->fused_skip > 0) {   // far movers in a recent fused step: the general path for now
            ctx->fused_skip--;
            fused = false;
        }
        if (pusher != PSUM_PIC_LEAPFROG && pusher != PSUM_PIC_BORIS) throw std::invalid_argument("step: unknown pusher");
        if (fused) {
            // push, deposit and re-sort in the two passes of the fused step (timed by cls_step)
            cls_step(ctx, phi_dev, dt, pusher, B);
            ctx->steps++;
        } else {
            {
                PhaseTimer t(ctx, 2);
                if (ctx->interp_order > 1) push_bspline(ctx, phi_dev, dt, pusher, B);
                else push_all(ctx, phi_dev, dt, pusher, B);
                t.stop();
            }
            ctx->steps++;
            if (ctx->sort_interval > 0 && ctx->steps % ctx->sort_interval == 0) {
                PhaseTimer t(ctx, 3);
                sort_all(ctx);
                t.stop();
            }
        }
        // a fused step reduces its sums when it is joined; the general path has none pending
        if (ctx->diag && !ctx->pending) {
            PhaseTimer t(ctx, 4);
            finish_diagnostics(ctx, ctx->diag_par);
            t.stop();
        }
        ctx->diag_valid = ctx->diag;
    });
}

EXPORT int psum_pic_set_timing(psum_pic_ctx* ctx, int enable) {
    return guarded([&] {
        ctx_check(ctx);
        ctx->timing = enable != 0;
    });
}

EXPORT int psum_pic_get_timing(psum_pic_ctx* ctx, double* ms_host, int* count_host, int reset) {
    return guarded([&] {
        ctx_check(ctx);
        if (!ms_host) throw std::invalid_argument("get_timing: null output");
        cuda_check(cudaStreamSynchronize(ctx->stream), "timing sync");
        for (int p = 0; p < 4; ++p) {
            ms_host[p] = 0.0;
            if (count_host) count_host[p] = 0;
        }
        for (auto& e : ctx->events) {
            const int p = e.first & 0xff;
            if (p >= 4) continue;   // the diagnostics phase is reported by psum_pic_get_phase_times
            float ms = 0.f;
            cuda_check(cudaEventElapsedTime(&ms, e.second.first, e.second.second), "cudaEventElapsedTime");
            ms_host[p] += ms;
            if (count_host && !(e.first & kPhaseContinued)) count_host[p] += 1;
        }
        if (reset) ctx->drop_events();
    });
}

EXPORT int psum_pic_get_phase_times(psum_pic_ctx* ctx, double* ms_host, int* count_host, int n_phases, int reset) {
    return guarded([&] {
        ctx_check(ctx);
        if (!ms_host || n_phases < 1) throw std::invalid_argument("get_phase_times: null output or no phases");
        cuda_check(cudaStreamSynchronize(ctx->stream), "timing sync");
        for (int p = 0; p < n_phases; ++p) {
            ms_host[p] = 0.0;
            if (count_host) count_host[p] = 0;
        }
        for (auto& e : ctx->events) {
            const int p = e.first & 0xff;
            if (p >= n_phases) continue;
            float ms = 0.f;
            cuda_check(cudaEventElapsedTime(&ms, e.second.first, e.second.second), "cudaEventElapsedTime");
            ms_host[p] += ms;
            if (count_host && !(e.first & kPhaseContinued)) count_host[p] += 1;
        }
        if (reset) ctx->drop_events();
    });
}

EXPORT int psum_pic_get_step_diagnostics(psum_pic_ctx* ctx, double epsilon, double* out_host) {
    return guarded([&] {
        ctx_check(ctx);
        if (!out_host) throw std::invalid_argument("get_step_diagnostics: null output");
        if (!ctx->diag_valid)
            throw std::invalid_argument("get_step_diagnostics: no step with option 'diagnostics 1' has run");
        const int ns = (int)ctx->sp.size();
        double v[16];
        cuda_check(cudaMemcpyAsync(v, ctx->diag_out.p, sizeof(double) * (ns + 2), cudaMemcpyDeviceToHost, ctx->stream),
                   "D2H");
        cuda_check(cudaStreamSynchronize(ctx->stream), "diag sync");
        for (int s = 0; s < ns; ++s) out_host[s] = v[s];
        out_host[ns] = epsilon * v[ns];
        out_host[ns + 1] = v[ns + 1];
    });
}

EXPORT int psum_pic_diagnostics(psum_pic_ctx* ctx, const double* phi_dev, double epsilon, double* out_host) {
    return guarded([&] {
        ctx_check(ctx);
        if (!out_host) throw std::invalid_argument("diagnostics: null output");
        cudaStream_t s = ctx->stream;
        const int ns = (int)ctx->sp.size();
        std::vector<double> part(kDiagBlocks);
        for (int si = 0; si < ns; ++si) {
            Species& sp = *ctx->sp[si];
            const int cur = sp.cur;
            if (ctx->precision == PSUM_PIC_MIXED) ensure_keys(ctx, *ctx->sp[si]);
            if (ctx->precision == PSUM_PIC_MIXED)
                { k_kinetic_mixed<<<kDiagBlocks, 256, 0, s>>>(sp.key[cur].p, sp.vel[0][cur].p, sp.vel[1][cur].p,
                                                          sp.vel[2][cur].p, ctx->count.p + si, sp.m * sp.w,
                                                          ctx->partials.p); count_launch(); }
            else
                { k_kinetic64<<<kDiagBlocks, 256, 0, s>>>(sp.pos64[0][cur].p, sp.vel64[0][cur].p, sp.vel64[1][cur].p,
                                                      sp.vel64[2][cur].p, ctx->count.p + si, sp.m * sp.w,
                                                      ctx->partials.p); count_launch(); }
            cuda_check(cudaMemcpyAsync(part.data(), ctx->partials.p, sizeof(double) * kDiagBlocks,
                                       cudaMemcpyDeviceToHost, s),
                       "D2H");
            cuda_check(cudaStreamSynchronize(s), "diag sync");
            double t = 0;
            for (double v : part) t += v;
            out_host[si] = t;
        }
        double fe = 0;
        if (phi_dev) {
            { k_field_energy<<<kDiagBlocks, 256, 0, s>>>(ctx->g, phi_dev, ctx->partials.p); count_launch(); }
            cuda_check(cudaMemcpyAsync(part.data(), ctx->partials.p, sizeof(double) * kDiagBlocks,
                                       cudaMemcpyDeviceToHost, s),
                       "D2H");
            cuda_check(cudaStreamSynchronize(s), "diag sync");
            for (double v : part) fe += v;
            double vol = 1;
            for (int a = 0; a < ctx->g.dim; ++a) vol *= ctx->g.dx[a];
            fe = 0.5 * epsilon * fe * vol;
        }
        out_host[ns] = fe;
        double charge = 0;
        for (int si = 0; si < ns; ++si) {
            Species& sp = *ctx->sp[si];
            cuda_check(cudaMemsetAsync(ctx->ipartials.p, 0, sizeof(long long), s), "memset");
            { k_acc_sum<<<kDiagBlocks, 256, 0, s>>>(sp.acc.p, ctx->g.n_nodes, ctx->ipartials.p); count_launch(); }
            long long tot = 0;
            cuda_check(cudaMemcpyAsync(&tot, ctx->ipartials.p, sizeof(long long), cudaMemcpyDeviceToHost, s), "D2H");
            cuda_check(cudaStreamSynchronize(s), "diag sync");
            charge += sp.q * sp.w * std::ldexp((double)tot, -sp.dep_shift);
        }
        out_host[ns + 1] = charge;
    });
}

EXPORT int psum_pic_device_errors(psum_pic_ctx* ctx, unsigned int* flags) {
    return guarded([&] {
        ctx_check(ctx);
        if (!flags) throw std::invalid_argument("device_errors: null output");
        unsigned v = 0;
        cuda_check(cudaMemcpyAsync(&v, ctx->err.p, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream), "D2H");
        cuda_check(cudaMemsetAsync(ctx->err.p, 0, sizeof(unsigned), ctx->stream), "memset");
        cuda_check(cudaStreamSynchronize(ctx->stream), "errors sync");
        *flags = v;
    });
}

}  // extern "C"

// ===================================================== allocation-free bin ==
//
// psum_bin_positions_noalloc: PSuM's cell binning of caller-owned FP64
// positions with no device allocation at all.  Some callers cannot call
// cudaMalloc: a PSuM build whose device memory is owned by another runtime
// (AdaptiveCpp/SYCL USM pools, a framework's caching allocator) or a loop that
// runs under a fixed memory budget, where an extra cudaMalloc either fails or
// fragments the pool.  Those callers pass their own inputs and outputs, and
// the sort/scan scratch lives in the file-scope array below, which every GPU
// that loads this library holds until the process exits.
namespace psum_b200 {
namespace {

constexpr long long kNoAllocMaxParticles = 1LL << 18;   // 262,144 particles
constexpr long long kNoAllocMaxCells = 1LL << 20;       // 1,048,576 cells
constexpr long long kNoAllocTiles = kNoAllocMaxParticles / kRsTile;
// scratch layout (bytes): sort keys A/B, sort payload A/B, per-tile radix
// histogram and its scan, per-cell counts and offsets, scan block totals
constexpr size_t kNaKeyBytes = sizeof(unsigned) * kNoAllocMaxParticles;
constexpr size_t kNaHistBytes = sizeof(unsigned) * kRsBuckets * kNoAllocTiles;
constexpr size_t kNaCellBytes = sizeof(unsigned) * kNoAllocMaxCells;
constexpr size_t kNaTotBytes = sizeof(unsigned) * (kNoAllocMaxCells / kScanBlock + 64);
constexpr size_t kNoAllocScratchBytes = 4 * kNaKeyBytes + 2 * kNaHistBytes + 2 * kNaCellBytes + 2 * kNaTotBytes;

static __device__ __align__(256) unsigned char g_noalloc_bin_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mutex;
void* g_noalloc_addr[64] = {nullptr};   // device address of the scratch, per device ordinal

// Device address of the scratch array for the current device; looked up
// once per device (cudaGetSymbolAddress), with that device current.
unsigned char* noalloc_scratch() {
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= 64) throw Error(PSUM_ERR_INTERNAL, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_noalloc_mutex);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        cuda_check(cudaGetSymbolAddress(&p, g_noalloc_bin_scratch), "cudaGetSymbolAddress");
        g_noalloc_addr[dev] = p;
    }
    return static_cast<unsigned char*>(g_noalloc_addr[dev]);
}

struct BinKeyArgs {
    GridView g;
    double hi[3];
    const double* pos;   // SoA [d*n + i]
    long long n;
};

// keys c2i(nC(p)) for in-grid particles, -1 otherwise (grid_mapped_device_vector.hpp:58-67)
__global__ void k_noalloc_keys(BinKeyArgs a, long long* __restrict__ keys_out, unsigned* __restrict__ skey,
                               int* __restrict__ sidx, unsigned sentinel) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    double p[3] = {0.0, 0.0, 0.0};
    for (int d = 0; d < a.g.dim; ++d) p[d] = a.pos[(long long)d * a.n + i];
    bool in = isfinite(p[0]);
    for (int d = 0; d < a.g.dim && in; ++d) in = p[d] >= a.g.lo[d] && p[d] < a.hi[d];
    long long ref = -1;
    if (in) {
        int c[3] = {0, 0, 0};
        // nC clamped to the last cell, as in k_bin_keys64
        for (int d = 0; d < a.g.dim; ++d) c[d] = min((int)((p[d] - a.g.lo[d]) * a.g.dr[d]), a.g.cells[d] - 1);
        ref = ((long long)c[0] * a.g.cells[1] + c[1]) * a.g.cells[2] + c[2];
    }
    keys_out[i] = ref;
    skey[i] = ref < 0 ? sentinel : (unsigned)ref;
    sidx[i] = (int)i;
}

}  // namespace
}  // namespace psum_b200

extern "C" EXPORT int psum_bin_positions_noalloc(const psum_pic_grid_desc* grid, unsigned long long n,
                                                 const double* pos_dev, long long* keys_dev,
                                                 unsigned long long* counts_dev, unsigned long long* offsets_dev,
                                                 unsigned long long* perm_dev, unsigned long long* n_in_grid,
                                                 void* stream) {
    return guarded([&] {
        if (!grid || !n_in_grid || !counts_dev || !offsets_dev) throw std::invalid_argument("bin_noalloc: null argument");
        if (n > 0 && (!pos_dev || !keys_dev || !perm_dev)) throw std::invalid_argument("bin_noalloc: null device array");
        if (grid->dim != 2 && grid->dim != 3) throw std::invalid_argument("bin_noalloc: dim must be 2 or 3");
        if (n > (unsigned long long)kNoAllocMaxParticles)
            throw std::invalid_argument("bin_noalloc: n = " + std::to_string(n) + " exceeds the fixed scratch limit of " +
                                        std::to_string(kNoAllocMaxParticles) + " particles");
        BinKeyArgs a{};
        long long ncell = 1;
        for (int d = 0; d < 3; ++d) {
            if (d < grid->dim) {
                if (grid->cells[d] < 1 || !(grid->lower[d] < grid->upper[d]))
                    throw std::invalid_argument("bin_noalloc: bad grid");
                // each factor is checked before the product, so the product cannot overflow
                if (grid->cells[d] > kNoAllocMaxCells || ncell * grid->cells[d] > kNoAllocMaxCells)
                    throw std::invalid_argument("bin_noalloc: the grid's cells exceed the fixed scratch limit of " +
                                                std::to_string(kNoAllocMaxCells) + " cells");
                a.g.cells[d] = grid->cells[d];
                a.g.lo[d] = grid->lower[d];
                a.g.dx[d] = (grid->upper[d] - grid->lower[d]) / grid->cells[d];   // simple_grid.hpp:47
                a.g.dr[d] = 1.0 / a.g.dx[d];
                a.hi[d] = grid->upper[d];
            } else {
                a.g.cells[d] = 1;
                a.g.dx[d] = a.g.dr[d] = 1.0;
            }
            ncell *= a.g.cells[d];
        }
        a.g.dim = grid->dim;
        if (ncell > kNoAllocMaxCells)
            throw std::invalid_argument("bin_noalloc: " + std::to_string(ncell) + " cells exceed the fixed scratch limit of " +
                                        std::to_string(kNoAllocMaxCells) + " cells");
        a.pos = pos_dev;
        a.n = (long long)n;
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        unsigned char* base = noalloc_scratch();
        unsigned* keyA = reinterpret_cast<unsigned*>(base);
        unsigned* keyB = reinterpret_cast<unsigned*>(base + kNaKeyBytes);
        int* idxA = reinterpret_cast<int*>(base + 2 * kNaKeyBytes);
        int* idxB = reinterpret_cast<int*>(base + 3 * kNaKeyBytes);
        unsigned* hist = reinterpret_cast<unsigned*>(base + 4 * kNaKeyBytes);
        unsigned* hist_scan = reinterpret_cast<unsigned*>(base + 4 * kNaKeyBytes + kNaHistBytes);
        unsigned* cnt = reinterpret_cast<unsigned*>(base + 4 * kNaKeyBytes + 2 * kNaHistBytes);
        unsigned* off = reinterpret_cast<unsigned*>(base + 4 * kNaKeyBytes + 2 * kNaHistBytes + kNaCellBytes);
        unsigned* tot1 = reinterpret_cast<unsigned*>(base + 4 * kNaKeyBytes + 2 * kNaHistBytes + 2 * kNaCellBytes);
        unsigned* tot2 = tot1 + kNaTotBytes / sizeof(unsigned);
        const unsigned sentinel = (unsigned)ncell;
        // per-cell counts must start at zero: the scratch keeps the previous call's contents
        cuda_check(cudaMemsetAsync(cnt, 0, sizeof(unsigned) * ncell, s), "cudaMemsetAsync");
        if (n > 0) {
            { k_noalloc_keys<<<blocks_for((long long)n, 256), 256, 0, s>>>(a, keys_dev, keyA, idxA, sentinel); count_launch(); }
            { k_hist_u32<<<blocks_for((long long)n, 256), 256, 0, s>>>(keys_dev, (long long)n, cnt); count_launch(); }
        }
        exclusive_scan_u32(cnt, off, ncell, tot1, tot2, s);
        { k_u32_to_u64<<<blocks_for(ncell, 256), 256, 0, s>>>(cnt, counts_dev, ncell); count_launch(); }
        { k_u32_to_u64<<<blocks_for(ncell, 256), 256, 0, s>>>(off, offsets_dev, ncell); count_launch(); }
        unsigned long long total = 0;
        if (n > 0) {
            // stable LSD radix sort of (key, index) in the scratch buffers
            unsigned* kin = keyA;
            unsigned* kout = keyB;
            int* vin = idxA;
            int* vout = idxB;
            const int nbits = std::max(1, bits_for(sentinel));
            const int nb = (int)(((long long)n + kRsTile - 1) / kRsTile);
            for (int shift = 0; shift < nbits; shift += kRsBits) {
                { k_rs_hist<<<nb, kRsThreads, 0, s>>>(kin, (long long)n, shift, hist, nb); count_launch(); }
                exclusive_scan_u32(hist, hist_scan, (long long)kRsBuckets * nb, tot1, tot2, s);
                { k_rs_scatter<<<nb, kRsThreads, 0, s>>>(kin, vin, kout, vout, (long long)n, shift, hist_scan, nb); count_launch(); }
                std::swap(kin, kout);
                std::swap(vin, vout);
            }
            unsigned last_off = 0, last_cnt = 0;
            cuda_check(cudaMemcpyAsync(&last_off, off + ncell - 1, sizeof(unsigned), cudaMemcpyDeviceToHost, s), "D2H");
            cuda_check(cudaMemcpyAsync(&last_cnt, cnt + ncell - 1, sizeof(unsigned), cudaMemcpyDeviceToHost, s), "D2H");
            cuda_check(cudaStreamSynchronize(s), "bin_noalloc sync");
            total = (unsigned long long)last_off + last_cnt;
            if (total > 0) { k_i32_to_u64<<<blocks_for((long long)total, 256), 256, 0, s>>>(vin, perm_dev, (long long)total); count_launch(); }
        }
        cuda_check(cudaGetLastError(), "bin_noalloc launch");
        cuda_check(cudaStreamSynchronize(s), "bin_noalloc sync");
        *n_in_grid = total;
    });
}
