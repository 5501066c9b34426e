// bspline.cu -- node-field interpolation at B-spline orders 1-4: the value
// gather (interp_B_spline), the gradient gather (interp_diff_B_spline) and
// the deposit (add_back_B_spline) of PSuM's src/field/higher_order_interp.hpp:196-247,
// over FP64 SoA positions on the device.
//
// Geometry (src/field/simple_grid.hpp:316-397): with S = order + 1 support
// nodes per axis, odd S (orders 2, 4) centres the support on the nearest node
// round((p - lo) * dr), even S (orders 1, 3) starts it at the corner node
// floor((p - lo) * dr); the offsets run from -(S/2) (odd) or -(S/2 - 1) (even);
// the normalised coordinate is (p - (lo + base * delta)) * dr; node indices
// wrap once by +-(cells + 1) on every axis (the reference's stencil wrap).
//
// 1-D weights (src/field/simple_interpolation.hpp:92-184) are evaluated in
// closed polynomial form, with x the normalised coordinate and a = 0.5 - x,
// b = 0.5 + x, v = 1 - x:
//   order 1: 1 - x, x
//   order 2: a^2/2, 3/4 - x^2, b^2/2
//   order 3: v^3/6, 2/3 - x^2 + x^3/2, 2/3 - v^2 + v^3/2, x^3/6
//   order 4: a^4/24, (19 - 44x + 24x^2 + 16x^3 - 16x^4)/96,
//            115/192 - 5x^2/8 + x^4/4, (19 + 44x + 24x^2 - 16x^3 - 16x^4)/96, b^4/24
// (the reference's piecewise kernels at the support offsets, expanded), and
// their x-derivatives times dr for the gradient.
//
// Gathers sum the tensor product factor by factor (innermost axis first), so
// an order-4 3-D gradient costs about two FMAs per support node instead of
// D products per node and direction.  They do not apply the reference's
// 1e-10 skip of small weights (field_interp.hpp:78-113): the difference is at
// most 1e-10 times the summed |field| over the skipped nodes.
//
// The deposit applies the skip and accumulates each weight as a 64-bit
// fixed-point integer (2^-F units, F = min(40, 62 - ceil(log2(n + 1)))), so
// the result does not depend on particle order or thread timing; the field
// then receives w * sum * 2^-F.  The reference adds w * weight with FP64
// atomics (atomic_add.hpp:34-48), whose result depends on the order.
#include <cuda_runtime.h>
#include <math_constants.h>

#include <cmath>
#include <stdexcept>

#include "../../include/psum_interp.h"
#include "common.hpp"

namespace psum_b200 {
namespace {

constexpr int kBsThreads = 256;

struct BsGrid {
    int N[3];            // nodes per axis (cells + 1); 1 beyond dim
    int stride[3];       // node index stride per axis (last axis fastest)
    double lo[3], delta[3], dr[3];
    long long n_nodes;
};

BsGrid make_grid(const psum_pic_grid_desc* gd) {
    if (!gd) throw std::invalid_argument("bspline: null grid");
    if (gd->dim < 1 || gd->dim > 3) throw std::invalid_argument("bspline: dim must be 1, 2 or 3");
    BsGrid g{};
    for (int a = 0; a < 3; ++a) {
        if (a < gd->dim) {
            if (gd->cells[a] <= 0) throw std::invalid_argument("bspline: cells must be positive");
            if (!(gd->upper[a] > gd->lower[a])) throw std::invalid_argument("bspline: upper must exceed lower");
            g.N[a] = gd->cells[a] + 1;
            g.lo[a] = gd->lower[a];
            g.delta[a] = (gd->upper[a] - gd->lower[a]) / gd->cells[a];   // simple_grid.hpp:46-47
            g.dr[a] = 1.0 / g.delta[a];
        } else {
            g.N[a] = 1;
            g.lo[a] = 0.0;
            g.delta[a] = g.dr[a] = 1.0;
        }
    }
    // last dimension fastest over the first `dim` axes (simple_grid::n2i, :107-112)
    for (int a = 2; a >= 0; --a) g.stride[a] = a >= gd->dim - 1 ? 1 : g.stride[a + 1] * g.N[a + 1];
    g.n_nodes = 1;
    for (int a = 0; a < gd->dim; ++a) g.n_nodes *= g.N[a];
    if (g.n_nodes >= (1LL << 31)) throw std::invalid_argument("bspline: more than 2^31 - 1 nodes");
    return g;
}

template <int ORDER>
__device__ __forceinline__ void weights(double x, double* w) {
    if constexpr (ORDER == 1) {
        w[0] = 1.0 - x;
        w[1] = x;
    } else if constexpr (ORDER == 2) {
        const double a = 0.5 - x, b = 0.5 + x;
        w[0] = 0.5 * a * a;
        w[1] = 0.75 - x * x;
        w[2] = 0.5 * b * b;
    } else if constexpr (ORDER == 3) {
        const double v = 1.0 - x;
        w[0] = v * v * v * (1.0 / 6.0);
        w[1] = 2.0 / 3.0 - x * x + 0.5 * x * x * x;
        w[2] = 2.0 / 3.0 - v * v + 0.5 * v * v * v;
        w[3] = x * x * x * (1.0 / 6.0);
    } else {
        const double a = 0.5 - x, b = 0.5 + x, x2 = x * x;
        w[0] = (a * a) * (a * a) * (1.0 / 24.0);
        w[1] = (19.0 + x * (-44.0 + x * (24.0 + x * (16.0 - 16.0 * x)))) * (1.0 / 96.0);
        w[2] = 115.0 / 192.0 + x2 * (-0.625 + 0.25 * x2);
        w[3] = (19.0 + x * (44.0 + x * (24.0 + x * (-16.0 - 16.0 * x)))) * (1.0 / 96.0);
        w[4] = (b * b) * (b * b) * (1.0 / 24.0);
    }
}

template <int ORDER>
__device__ __forceinline__ void dweights(double x, double* d) {
    if constexpr (ORDER == 1) {
        d[0] = -1.0;
        d[1] = 1.0;
    } else if constexpr (ORDER == 2) {
        d[0] = x - 0.5;
        d[1] = -2.0 * x;
        d[2] = x + 0.5;
    } else if constexpr (ORDER == 3) {
        const double v = 1.0 - x;
        d[0] = -0.5 * v * v;
        d[1] = x * (-2.0 + 1.5 * x);
        d[2] = v * (2.0 - 1.5 * v);
        d[3] = 0.5 * x * x;
    } else {
        const double a = 0.5 - x, b = 0.5 + x;
        d[0] = -(a * a * a) * (1.0 / 6.0);
        d[1] = (-44.0 + x * (48.0 + x * (48.0 - 64.0 * x))) * (1.0 / 96.0);
        d[2] = x * (-1.25 + x * x);
        d[3] = (44.0 + x * (48.0 + x * (-48.0 - 64.0 * x))) * (1.0 / 96.0);
        d[4] = (b * b * b) * (1.0 / 6.0);
    }
}

// Per-axis support of one position: S node offsets (index * stride) and the
// normalised coordinate.  False when the position is not finite or a node
// is still outside the axis after one wrap.
template <int ORDER>
__device__ __forceinline__ bool axis_support(const BsGrid& g, int a, double p, int* off, double& x) {
    constexpr int S = ORDER + 1;
    constexpr bool kNearest = (S % 2) == 1;
    constexpr int kShift = kNearest ? -(S / 2) : -(S / 2 - 1);
    const double u = (p - g.lo[a]) * g.dr[a];
    if (!(u > -(double)(S + 1) && u < (double)(g.N[a] + S + 1))) return false;   // also rejects NaN
    const int base = kNearest ? (int)round(u) : (int)floor(u);
    x = (p - (g.lo[a] + base * g.delta[a])) * g.dr[a];
    const int w = g.N[a];
    bool ok = true;
#pragma unroll
    for (int k = 0; k < S; ++k) {
        int n = base + k + kShift;
        if (n < 0) n += w;
        else if (n >= w) n -= w;
        ok = ok && n >= 0 && n < w;
        off[k] = n * g.stride[a];
    }
    return ok;
}

template <int D, int ORDER, bool GRAD>
__global__ void __launch_bounds__(kBsThreads, 2) k_bs_gather(BsGrid g, long long n, const double* __restrict__ pos,
                                                          const double* __restrict__ field, double* __restrict__ out,
                                                          unsigned long long* __restrict__ skipped) {
    constexpr int S = ORDER + 1;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int off[D][S];
    double w[D][S], dw[D][S];
    bool ok = true;
#pragma unroll
    for (int a = 0; a < D; ++a) {
        double x = 0.0;
        ok = axis_support<ORDER>(g, a, pos[(long long)a * n + i], off[a], x) && ok;
        weights<ORDER>(x, w[a]);
        if constexpr (GRAD) {
            dweights<ORDER>(x, dw[a]);
#pragma unroll
            for (int k = 0; k < S; ++k) dw[a][k] *= g.dr[a];
        }
    }
    if (!ok) {
        if constexpr (GRAD) {
#pragma unroll
            for (int a = 0; a < D; ++a) out[(long long)a * n + i] = CUDART_NAN;
        } else {
            out[i] = CUDART_NAN;
        }
        if (skipped) atomicAdd(skipped, 1ULL);
        return;
    }
    if constexpr (D == 1) {
        double v = 0.0, d0 = 0.0;
#pragma unroll
        for (int k = 0; k < S; ++k) {
            const double f = __ldg(field + off[0][k]);
            if constexpr (GRAD) d0 = fma(dw[0][k], f, d0);
            else v = fma(w[0][k], f, v);
        }
        out[i] = GRAD ? d0 : v;
    } else if constexpr (D == 2) {
        double v = 0.0, g0 = 0.0, g1 = 0.0;
#pragma unroll
        for (int k0 = 0; k0 < S; ++k0) {
            double lw = 0.0, ld = 0.0;   // sums along the last axis
#pragma unroll
            for (int k1 = 0; k1 < S; ++k1) {
                const double f = __ldg(field + off[0][k0] + off[1][k1]);
                lw = fma(w[1][k1], f, lw);
                if constexpr (GRAD) ld = fma(dw[1][k1], f, ld);
            }
            if constexpr (GRAD) {
                g0 = fma(dw[0][k0], lw, g0);
                g1 = fma(w[0][k0], ld, g1);
            } else {
                v = fma(w[0][k0], lw, v);
            }
        }
        if constexpr (GRAD) {
            out[i] = g0;
            out[n + i] = g1;
        } else {
            out[i] = v;
        }
    } else {
        double v = 0.0, g0 = 0.0, g1 = 0.0, g2 = 0.0;
#pragma unroll
        for (int k0 = 0; k0 < S; ++k0) {
            double pw = 0.0, pd1 = 0.0, pd2 = 0.0;   // sums over the two inner axes
#pragma unroll
            for (int k1 = 0; k1 < S; ++k1) {
                double lw = 0.0, ld = 0.0;
                const double* row = field + off[0][k0] + off[1][k1];
#pragma unroll
                for (int k2 = 0; k2 < S; ++k2) {
                    const double f = __ldg(row + off[2][k2]);
                    lw = fma(w[2][k2], f, lw);
                    if constexpr (GRAD) ld = fma(dw[2][k2], f, ld);
                }
                pw = fma(w[1][k1], lw, pw);
                if constexpr (GRAD) {
                    pd1 = fma(dw[1][k1], lw, pd1);
                    pd2 = fma(w[1][k1], ld, pd2);
                }
            }
            if constexpr (GRAD) {
                g0 = fma(dw[0][k0], pw, g0);
                g1 = fma(w[0][k0], pd1, g1);
                g2 = fma(w[0][k0], pd2, g2);
            } else {
                v = fma(w[0][k0], pw, v);
            }
        }
        if constexpr (GRAD) {
            out[i] = g0;
            out[n + i] = g1;
            out[2 * n + i] = g2;
        } else {
            out[i] = v;
        }
    }
}

// Deposit with warp aggregation.  Lanes whose stencils start at the same
// node share all S^D support nodes (the stencil is fixed by its first node
// once the one wrap has succeeded); when a warp holds at most kAggGroups such
// groups (the usual case for particles stored cell by cell), every group's
// per-node weights are summed across the warp with two 32-bit reductions of
// the fixed-point value split at bit 27 (values are at most 2^40, so 32 lanes
// cannot overflow either part) and its first lane issues one atomic per
// node; otherwise every lane adds its own weights.  Integer sums make both
// paths give the same bits.  B-spline weights are non-negative (up to
// rounding of the zero edge weights), so the reference's |w| > 1e-10 test is
// the same set as w > 1e-10.
constexpr int kAggGroups = 4;

// One stencil for the whole warp (the usual case for particles stored cell
// by cell): the support weights are transposed through shared memory, 16
// nodes at a time, and lane j (with lane j + 16 over the other half of the
// warp) sums node j over the 32 lanes -- no warp reductions.  The sums are
// the same integers as the reductions' (32 parts below 2^27 and 2^13), so
// the bits are too.  off holds the lane's per-axis node offsets; the
// leader's are the group's.
constexpr int kTrChunk = 16;
struct TrScratch {
    unsigned lo[kTrChunk][33];
    unsigned hi[kTrChunk][33];
    int off[3][8];
};

template <int N0, int N1, int N2, int NA, class Q>
__device__ __forceinline__ void deposit_one_group(const Q& q_at, bool ok, int leader, const int (&off)[3][NA],
                                                  unsigned long long* __restrict__ acc, TrScratch& t, int lane) {
    constexpr int NN = N0 * N1 * N2;
    if (lane == leader) {
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int j = 0; j < NA; ++j) t.off[a][j] = off[a][j];
    }
#pragma unroll
    for (int base = 0; base < NN; base += kTrChunk) {
#pragma unroll
        for (int j = 0; j < kTrChunk; ++j) {
            const int node = base + j;
            if (node < NN) {
                const unsigned long long q = ok ? q_at(node / (N1 * N2), (node / N2) % N1, node % N2) : 0ULL;
                t.lo[j][lane] = (unsigned)(q & 0x7ffffffULL);
                t.hi[j][lane] = (unsigned)(q >> 27);
            }
        }
        __syncwarp();
        const int j = lane & (kTrChunk - 1), h = lane >> 4, node = base + j;
        unsigned slo = 0, shi = 0;
        if (node < NN) {
#pragma unroll
            for (int l = 0; l < 16; ++l) {
                slo += t.lo[j][h * 16 + l];
                shi += t.hi[j][h * 16 + l];
            }
        }
        slo += __shfl_xor_sync(0xffffffffu, slo, 16);
        shi += __shfl_xor_sync(0xffffffffu, shi, 16);
        const unsigned long long sum = ((unsigned long long)shi << 27) + slo;
        if (h == 0 && node < NN && sum)
            atomicAdd(acc + (t.off[0][node / (N1 * N2)] + t.off[1][(node / N2) % N1] + t.off[2][node % N2]), sum);
        __syncwarp();
    }
}

template <int D, int ORDER>
__global__ void __launch_bounds__(kBsThreads) k_bs_deposit(BsGrid g, long long n, const double* __restrict__ pos,
                                                           double scale, unsigned long long* __restrict__ acc,
                                                           unsigned long long* __restrict__ skipped) {
    constexpr int S = ORDER + 1;
    constexpr int S1 = D > 1 ? S : 1;
    constexpr int S2 = D > 2 ? S : 1;
    constexpr unsigned kFull = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < n;
    int off[3][S];
    double w[3][S];
    bool ok = active;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (a < D) {
            double x = 0.0;
            ok = axis_support<ORDER>(g, a, active ? pos[(long long)a * n + i] : 0.0, off[a], x) && ok;
            weights<ORDER>(x, w[a]);
        } else {
#pragma unroll
            for (int k = 0; k < S; ++k) {
                off[a][k] = 0;
                w[a][k] = k == 0 ? 1.0 : 0.0;
            }
        }
    }
    if (active && !ok && skipped) atomicAdd(skipped, 1ULL);
    // weight of support point (k0, k1, k2) in 2^-F units: the product taken
    // from the last axis to the first as interp_tensor does
    auto q_at = [&](int k0, int k1, int k2) -> unsigned long long {
        double c = 1.0;
        if (D > 2) c *= w[2][k2];
        if (D > 1) c *= w[1][k1];
        c *= w[0][k0];
        return c > 1e-10 ? (unsigned long long)__double2ll_rn(c * scale) : 0ULL;
    };
    const int key = ok ? off[0][0] + off[1][0] + off[2][0] : -1;
    const unsigned grp = __match_any_sync(kFull, key);
    const unsigned leaders = __ballot_sync(kFull, ok && __ffs(grp) - 1 == lane);
    __shared__ TrScratch tr[kBsThreads / 32];
    if (__popc(leaders) == 1) {
        deposit_one_group<S, S1, S2, S>(q_at, ok, __ffs(leaders) - 1, off, acc, tr[threadIdx.x >> 5], lane);
    } else if (__popc(leaders) <= kAggGroups) {
#pragma unroll
        for (int k0 = 0; k0 < S; ++k0)
#pragma unroll
            for (int k1 = 0; k1 < S1; ++k1)
#pragma unroll
                for (int k2 = 0; k2 < S2; ++k2) {
                    const unsigned long long q = ok ? q_at(k0, k1, k2) : 0ULL;
                    for (unsigned rem = leaders; rem; rem &= rem - 1) {
                        const int l = __ffs(rem) - 1;
                        const unsigned long long qm = (grp >> l) & 1u ? q : 0ULL;
                        const unsigned lo = __reduce_add_sync(kFull, (unsigned)(qm & 0x7ffffffULL));
                        const unsigned hi = __reduce_add_sync(kFull, (unsigned)(qm >> 27));
                        const unsigned long long t = ((unsigned long long)hi << 27) + lo;
                        if (lane == l && t) atomicAdd(acc + (off[0][k0] + off[1][k1] + off[2][k2]), t);
                    }
                }
    } else if (ok) {
#pragma unroll
        for (int k0 = 0; k0 < S; ++k0)
#pragma unroll
            for (int k1 = 0; k1 < S1; ++k1)
#pragma unroll
                for (int k2 = 0; k2 < S2; ++k2) {
                    const unsigned long long q = q_at(k0, k1, k2);
                    if (q) atomicAdd(acc + (off[0][k0] + off[1][k1] + off[2][k2]), q);
                }
    }
}

// Deposit of the nearest-node orders (2 and 4).  Particles of one cell have
// up to 2^D different nearest nodes, hence up to 2^D stencils; grouping lanes
// by their floor cell instead, each lane writes its S weights into the
// cell's union stencil of S + 1 nodes per axis (starting at floor - S/2, its
// own stencil at offset 0 or 1), so one cell is one group.  The summed values
// and their bits are those of k_bs_deposit: the same per-node weights, the
// same products, integer sums.  A node of the union stencil that fails the
// single wrap carries zero weight for every supported lane of the group (each
// lane's own nodes all passed it), so it is never written; its offset is
// clamped to 0 all the same.
template <int D, int ORDER>
__global__ void __launch_bounds__(kBsThreads) k_bs_deposit_near(BsGrid g, long long n, const double* __restrict__ pos,
                                                                double scale, unsigned long long* __restrict__ acc,
                                                                unsigned long long* __restrict__ skipped) {
    constexpr int S = ORDER + 1;
    static_assert(S % 2 == 1, "nearest-node orders only");
    constexpr int E = S + 1;
    constexpr int kShift = -(S / 2);
    constexpr int E1 = D > 1 ? E : 1;
    constexpr int E2 = D > 2 ? E : 1;
    constexpr unsigned kFull = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < n;
    int off[3][E];
    double we[3][E];
    long long key = 0;
    bool ok = active;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (a < D) {
            const double p = active ? pos[(long long)a * n + i] : 0.0;
            const double u = (p - g.lo[a]) * g.dr[a];
            bool oka = u > -(double)(S + 1) && u < (double)(g.N[a] + S + 1);   // also rejects NaN
            const double uc = oka ? u : 0.0;
            const int fl = (int)floor(uc);
            const int nr = (int)round(uc);
            const bool up = nr != fl;   // own stencil at offset 1 of the union stencil
            double w[S];
            weights<ORDER>(oka ? (p - (g.lo[a] + nr * g.delta[a])) * g.dr[a] : 0.0, w);
            const int Na = g.N[a];
#pragma unroll
            for (int j = 0; j < E; ++j) {
                int nd = fl + kShift + j;
                if (nd < 0) nd += Na;
                else if (nd >= Na) nd -= Na;
                const bool valid = nd >= 0 && nd < Na;
                const bool mine = up ? j >= 1 : j < S;
                oka = oka && (!mine || valid);
                off[a][j] = valid ? nd * g.stride[a] : 0;
                const double wl = j < S ? w[j] : 0.0;
                const double wu = j >= 1 ? w[j >= 1 ? j - 1 : 0] : 0.0;
                we[a][j] = up ? wu : wl;
            }
            ok = ok && oka;
            key = key * (long long)(Na + 2 * S + 4) + (fl + S + 2);
        } else {
#pragma unroll
            for (int j = 0; j < E; ++j) {
                off[a][j] = 0;
                we[a][j] = j == 0 ? 1.0 : 0.0;
            }
        }
    }
    if (active && !ok && skipped) atomicAdd(skipped, 1ULL);
    auto q_at = [&](int k0, int k1, int k2) -> unsigned long long {
        double c = 1.0;
        if (D > 2) c *= we[2][k2];
        if (D > 1) c *= we[1][k1];
        c *= we[0][k0];
        return c > 1e-10 ? (unsigned long long)__double2ll_rn(c * scale) : 0ULL;
    };
    const long long gkey = ok ? key : -1LL;
    const unsigned grp = __match_any_sync(kFull, gkey);
    const unsigned leaders = __ballot_sync(kFull, ok && __ffs(grp) - 1 == lane);
    __shared__ TrScratch tr[kBsThreads / 32];
    if (__popc(leaders) == 1) {
        deposit_one_group<E, E1, E2, E>(q_at, ok, __ffs(leaders) - 1, off, acc, tr[threadIdx.x >> 5], lane);
    } else if (__popc(leaders) <= kAggGroups) {
#pragma unroll
        for (int k0 = 0; k0 < E; ++k0)
#pragma unroll
            for (int k1 = 0; k1 < E1; ++k1)
#pragma unroll
                for (int k2 = 0; k2 < E2; ++k2) {
                    const unsigned long long q = ok ? q_at(k0, k1, k2) : 0ULL;
                    for (unsigned rem = leaders; rem; rem &= rem - 1) {
                        const int l = __ffs(rem) - 1;
                        const unsigned long long qm = (grp >> l) & 1u ? q : 0ULL;
                        const unsigned lo = __reduce_add_sync(kFull, (unsigned)(qm & 0x7ffffffULL));
                        const unsigned hi = __reduce_add_sync(kFull, (unsigned)(qm >> 27));
                        const unsigned long long t = ((unsigned long long)hi << 27) + lo;
                        if (lane == l && t) atomicAdd(acc + (off[0][k0] + off[1][k1] + off[2][k2]), t);
                    }
                }
    } else if (ok) {
#pragma unroll
        for (int k0 = 0; k0 < E; ++k0)
#pragma unroll
            for (int k1 = 0; k1 < E1; ++k1)
#pragma unroll
                for (int k2 = 0; k2 < E2; ++k2) {
                    const unsigned long long q = q_at(k0, k1, k2);
                    if (q) atomicAdd(acc + (off[0][k0] + off[1][k1] + off[2][k2]), q);
                }
    }
}

__global__ void k_bs_finish(long long n_nodes, const unsigned long long* __restrict__ acc, double w_unit,
                            double* __restrict__ field) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_nodes) return;
    const long long q = (long long)acc[i];
    if (q != 0) field[i] += w_unit * (double)q;
}

unsigned blocks(long long n) { return (unsigned)((n + kBsThreads - 1) / kBsThreads); }

template <int D, int ORDER>
void launch_gather_t(const BsGrid& g, long long n, const double* pos, const double* field, double* out,
                     unsigned long long* skipped, bool grad, cudaStream_t s) {
    if (grad) k_bs_gather<D, ORDER, true><<<blocks(n), kBsThreads, 0, s>>>(g, n, pos, field, out, skipped);
    else k_bs_gather<D, ORDER, false><<<blocks(n), kBsThreads, 0, s>>>(g, n, pos, field, out, skipped);
    count_launch();
}

template <int D>
void launch_gather_d(int order, const BsGrid& g, long long n, const double* pos, const double* field, double* out,
                     unsigned long long* skipped, bool grad, cudaStream_t s) {
    switch (order) {
        case 1: launch_gather_t<D, 1>(g, n, pos, field, out, skipped, grad, s); break;
        case 2: launch_gather_t<D, 2>(g, n, pos, field, out, skipped, grad, s); break;
        case 3: launch_gather_t<D, 3>(g, n, pos, field, out, skipped, grad, s); break;
        default: launch_gather_t<D, 4>(g, n, pos, field, out, skipped, grad, s); break;
    }
}

template <int D>
void launch_deposit_d(int order, const BsGrid& g, long long n, const double* pos, double scale,
                      unsigned long long* acc, unsigned long long* skipped, cudaStream_t s) {
    switch (order) {
        case 1: k_bs_deposit<D, 1><<<blocks(n), kBsThreads, 0, s>>>(g, n, pos, scale, acc, skipped); break;
        case 2: k_bs_deposit_near<D, 2><<<blocks(n), kBsThreads, 0, s>>>(g, n, pos, scale, acc, skipped); break;
        case 3: k_bs_deposit<D, 3><<<blocks(n), kBsThreads, 0, s>>>(g, n, pos, scale, acc, skipped); break;
        default: k_bs_deposit_near<D, 4><<<blocks(n), kBsThreads, 0, s>>>(g, n, pos, scale, acc, skipped); break;
    }
    count_launch();
}

void check_order(int order) {
    if (order < 1 || order > 4) throw std::invalid_argument("bspline: order must be 1, 2, 3 or 4");
}

int gather(const psum_pic_grid_desc* grid, int order, unsigned long long n, const double* pos_dev,
           const double* field_dev, double* out_dev, unsigned long long* skipped_dev, void* stream, bool grad) {
    return guarded([&] {
        const BsGrid g = make_grid(grid);
        check_order(order);
        if (n == 0) return;
        if (!pos_dev || !field_dev || !out_dev) throw std::invalid_argument("bspline: null device array");
        const cudaStream_t s = (cudaStream_t)stream;
        const long long nn = (long long)n;
        switch (grid->dim) {
            case 1: launch_gather_d<1>(order, g, nn, pos_dev, field_dev, out_dev, skipped_dev, grad, s); break;
            case 2: launch_gather_d<2>(order, g, nn, pos_dev, field_dev, out_dev, skipped_dev, grad, s); break;
            default: launch_gather_d<3>(order, g, nn, pos_dev, field_dev, out_dev, skipped_dev, grad, s); break;
        }
        cuda_check(cudaGetLastError(), "bspline gather launch");
    });
}

}  // namespace

int deposit_fraction_bits(unsigned long long n) {
    int lg = 0;
    while (lg < 63 && (1ULL << lg) < n + 1) ++lg;   // ceil(log2(n + 1))
    const int f = 62 - lg;
    return f < 40 ? f : 40;
}

}  // namespace psum_b200

using namespace psum_b200;

EXPORT int psum_interp_bspline(const psum_pic_grid_desc* grid, int order, unsigned long long n, const double* pos_dev,
                               const double* field_dev, double* out_dev, unsigned long long* skipped_dev,
                               void* stream) {
    return gather(grid, order, n, pos_dev, field_dev, out_dev, skipped_dev, stream, false);
}

EXPORT int psum_interp_diff_bspline(const psum_pic_grid_desc* grid, int order, unsigned long long n,
                                    const double* pos_dev, const double* field_dev, double* grad_dev,
                                    unsigned long long* skipped_dev, void* stream) {
    return gather(grid, order, n, pos_dev, field_dev, grad_dev, skipped_dev, stream, true);
}

EXPORT int psum_add_back_bspline(const psum_pic_grid_desc* grid, int order, unsigned long long n,
                                 const double* pos_dev, double weight, double* field_dev, void* scratch_dev,
                                 unsigned long long* skipped_dev, void* stream) {
    return guarded([&] {
        const BsGrid g = make_grid(grid);
        check_order(order);
        if (n == 0) return;
        if (!pos_dev || !field_dev) throw std::invalid_argument("bspline: null device array");
        if (!std::isfinite(weight)) throw Error(PSUM_ERR_NONFINITE, "add_back: non-finite weight");
        if (n >= (1ULL << 40)) throw std::invalid_argument("add_back: more than 2^40 positions");
        const cudaStream_t s = (cudaStream_t)stream;
        const long long nn = (long long)n;
        unsigned long long* acc = (unsigned long long*)scratch_dev;
        if (!acc)
            cuda_check(cudaMallocAsync((void**)&acc, sizeof(unsigned long long) * g.n_nodes, s), "cudaMallocAsync");
        const int F = deposit_fraction_bits(n);
        try {
            cuda_check(cudaMemsetAsync(acc, 0, sizeof(unsigned long long) * g.n_nodes, s), "cudaMemsetAsync");
            switch (grid->dim) {
                case 1: launch_deposit_d<1>(order, g, nn, pos_dev, std::ldexp(1.0, F), acc, skipped_dev, s); break;
                case 2: launch_deposit_d<2>(order, g, nn, pos_dev, std::ldexp(1.0, F), acc, skipped_dev, s); break;
                default: launch_deposit_d<3>(order, g, nn, pos_dev, std::ldexp(1.0, F), acc, skipped_dev, s); break;
            }
            k_bs_finish<<<blocks(g.n_nodes), kBsThreads, 0, s>>>(g.n_nodes, acc, weight * std::ldexp(1.0, -F),
                                                                 field_dev);
            count_launch();
            cuda_check(cudaGetLastError(), "add_back launch");
        } catch (...) {
            if (!scratch_dev) cudaFreeAsync(acc, s);
            throw;
        }
        if (!scratch_dev) cuda_check(cudaFreeAsync(acc, s), "cudaFreeAsync");
    });
}

EXPORT int psum_bspline_deposit_bits(unsigned long long n, int* bits) {
    return guarded([&] {
        if (!bits) throw std::invalid_argument("null output");
        *bits = deposit_fraction_bits(n);
    });
}
