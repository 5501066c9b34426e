// pic_fp64_kernels.cuh -- FP64 particle kernels (the "FP64 GPU step"),
// compiled twice: pic_fp64.cu builds them with --fmad=false so that every
// operation rounds exactly like the host restatement of PSuM's push (no fused
// multiply-add contraction): with the same phi and the same input state the
// new positions, velocities, cell keys and loss counts are bit-identical to
// the CPU oracle's.  pic_fp64_fma.cu builds the same source with contraction
// (option "fp64_fma 1" of a context): the FP64 comparison run, not bit-exact.
// PSUM_FP64_NS names the namespace of each build's launchers.
//
// Arithmetic follows, in order:
//   CIC gradient gather   simple_grid.hpp:352-397 (gen_interp_diff),
//                         simple_interpolation.hpp:58-98 (interp_tensor_diff),
//                         field_interp.hpp:96-113 (1e-10 coefficient skip);
//   leapfrog push         application/benchmark/TSI/main.cpp:59-75;
//   Boris rotation        application/benchmark/EDI/EDI.cpp:216-266 (B along z),
//                         collision-less-flow/particle_ops.hpp:17-51 (3-D);
//   periodic wrap         TSI/main.cpp:70-72 (while loops, period (cells+1)*dx);
//   absorbing walls       EDI.cpp:253-258 + validator.hpp:19-26 (x = NaN).
#include <cuda_runtime.h>

#include "pic_common.cuh"
#include "pic_fp64.hpp"

namespace psum_b200 {
namespace PSUM_FP64_NS {

namespace {

struct Support64 {
    long long idx[8];
    double coef[8];
};

// D = g.dim as a template argument: the loops unroll and the support stays
// in registers; the operations and their order are those of the generic
// restatement, so the bits are too.
template <int D>
__device__ __forceinline__ void cic64(const GridView& g, const double* p, long long* idx, double* coef,
                                      double (*dcoef)[8]) {
    int base[3];
    double xn[3];
    for (int a = 0; a < D; ++a) {
        base[a] = (int)floor((p[a] - g.lo[a]) * g.dr[a]);
        const double base_pos = g.lo[a] + (double)base[a] * g.dx[a];
        xn[a] = (p[a] - base_pos) * g.dr[a];
    }
    constexpr int cnt = 1 << D;
#pragma unroll
    for (int i = 0; i < cnt; ++i) {
        int node[3] = {base[0], base[1], base[2]};
        int t = i;
        for (int j = 0; j < D; ++j) {
            const int a = D - 1 - j;
            node[a] += t % 2;
            const int w = g.cells[a] + 1;
            if (node[a] < 0) node[a] += w;
            else if (node[a] >= w) node[a] -= w;
            t /= 2;
        }
        long long lin = node[0];
        for (int a = 1; a < D; ++a) lin = lin * (g.cells[a] + 1) + node[a];
        idx[i] = lin;
        if (coef) {
            double c = 1;
            t = i;
            for (int j = 0; j < D; ++j) {
                const int a = D - 1 - j;
                c *= (t % 2 == 0) ? (1 - xn[a]) : xn[a];
                t /= 2;
            }
            coef[i] = c;
        }
        if (dcoef) {
            for (int d = 0; d < D; ++d) {
                double cd = 1;
                t = i;
                for (int j = 0; j < D; ++j) {
                    const int a = D - 1 - j;
                    const int b = t % 2;
                    if (a == d) cd *= (b == 0 ? -1.0 : 1.0) * g.dr[a];
                    else cd *= (b == 0) ? (1 - xn[a]) : xn[a];
                    t /= 2;
                }
                dcoef[d][i] = cd;
            }
        }
    }
}

template <int D>
__device__ __forceinline__ int key64_d(const GridView& g, const double* p) {
    int c[3] = {0, 0, 0};
#pragma unroll
    for (int a = 0; a < D; ++a) {
        int v = (int)floor((p[a] - g.lo[a]) * g.dr[a]);
        v = v < 0 ? 0 : (v >= g.M[a] ? g.M[a] - 1 : v);
        c[a] = v;
    }
    return (c[0] * g.M[1] + c[1]) * g.M[2] + c[2];
}

__device__ __forceinline__ int key64(const GridView& g, const double* p) {
    int c[3] = {0, 0, 0};
    for (int a = 0; a < g.dim; ++a) {
        int v = (int)floor((p[a] - g.lo[a]) * g.dr[a]);
        v = v < 0 ? 0 : (v >= g.M[a] ? g.M[a] - 1 : v);
        c[a] = v;
    }
    return (c[0] * g.M[1] + c[1]) * g.M[2] + c[2];
}

template <int D>
__device__ __forceinline__ void deposit64(const GridView& g, const double* p, bool alive,
                                          unsigned long long* acc, double scale) {
    long long idx[8];
    double coef[8];
    constexpr int cnt = 1 << D;
    if (alive) cic64<D>(g, p, idx, coef, nullptr);
#pragma unroll
    for (int k = 0; k < cnt; ++k) {
        long long node = -1, val = 0;
        if (alive && fabs(coef[k]) > 1e-10) {   // field_interp.hpp:73
            node = idx[k];
            val = __double2ll_rn(coef[k] * scale);
        }
        warp_deposit(acc, node, val);
    }
}

template <int D>
__global__ void __launch_bounds__(kPicThreads) k_push64(Push64Args a) {
    const GridView& g = a.g;
    const long long count = *a.count;
    const int lane = threadIdx.x & 31;
    double kin = 0.0;
    for (long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < count;
         base += (long long)gridDim.x * blockDim.x) {
        const long long i = base + lane;
        double p[3] = {0, 0, 0};
        bool alive = i < count;
        if (alive) {
            p[0] = a.pos[0][i];
            alive = isfinite(p[0]);
        }
        int lost = -1;
        if (alive) {
            for (int d = 1; d < D; ++d) p[d] = a.pos[d][i];
            double E[3] = {0, 0, 0};
            if (a.grad) {   // gathered by the caller (B-spline orders 2-4)
                for (int d = 0; d < D; ++d) E[d] = -a.grad[d * a.grad_stride + i];
            } else {
                long long idx[8];
                double dcoef[3][8];
                cic64<D>(g, p, idx, nullptr, dcoef);
                constexpr int cnt = 1 << D;
#pragma unroll
                for (int d = 0; d < D; ++d) {
                    double res = 0;
#pragma unroll
                    for (int k = 0; k < cnt; ++k)
                        if (fabs(dcoef[d][k]) > 1e-10) res += a.phi[idx[k]] * dcoef[d][k];
                    E[d] = -res;
                }
            }
            double v[3] = {a.vel[0][i], a.vel[1][i], a.vel[2][i]};
            if (a.pusher == 0) {
                for (int d = 0; d < D; ++d) v[d] += E[d] * a.q_m * a.dt;
            } else {
                const double kk = a.q_m * a.dt / 2;
                double vm[3], t[3], sv[3], vp[3], vprime[3];
                for (int c = 0; c < 3; ++c) vm[c] = v[c] + E[c] * kk;
                double t2 = 0;
                for (int c = 0; c < 3; ++c) {
                    t[c] = a.B[c] * kk;
                    t2 += t[c] * t[c];
                }
                for (int c = 0; c < 3; ++c) sv[c] = 2 * t[c] / (1 + t2);
                vprime[0] = vm[0] + (vm[1] * t[2] - vm[2] * t[1]);
                vprime[1] = vm[1] + (vm[2] * t[0] - vm[0] * t[2]);
                vprime[2] = vm[2] + (vm[0] * t[1] - vm[1] * t[0]);
                vp[0] = vm[0] + (vprime[1] * sv[2] - vprime[2] * sv[1]);
                vp[1] = vm[1] + (vprime[2] * sv[0] - vprime[0] * sv[2]);
                vp[2] = vm[2] + (vprime[0] * sv[1] - vprime[1] * sv[0]);
                for (int c = 0; c < 3; ++c) v[c] = vp[c] + E[c] * kk;
            }
            for (int c = 0; c < 3; ++c) a.vel[c][i] = v[c];
            for (int d = 0; d < D; ++d) p[d] += v[d] * a.dt;
            bool finite = true;
            for (int d = 0; d < D; ++d) finite = finite && isfinite(p[d]) && fabs(p[d]) < 1e300;
            if (!finite) {
                atomicOr(a.err, kErrNonFinite);
                alive = false;
            }
            for (int d = 0; d < D && alive; ++d) {
                if (g.periodic[d]) {
                    const double L = (g.cells[d] + 1) * g.dx[d];
                    const double top = g.lo[d] + L;
                    int guard = 0;
                    while (p[d] < g.lo[d] && guard++ < 64) p[d] += L;
                    while (p[d] >= top && guard++ < 128) p[d] -= L;
                    if (p[d] < g.lo[d] || p[d] >= top) {   // a particle crossed more than 64 periods
                        atomicOr(a.err, kErrNonFinite);
                        alive = false;
                    }
                } else if (p[d] < g.lo[d]) {
                    lost = 2 * d;
                    alive = false;
                } else if (p[d] >= a.hi[d]) {
                    lost = 2 * d + 1;
                    alive = false;
                }
            }
            for (int d = 0; d < D; ++d) a.pos[d][i] = p[d];
            if (!alive) a.pos[0][i] = __longlong_as_double(0x7ff8000000000000LL);   // NaN x: invalid
            a.key[i] = alive ? key64_d<D>(g, p) : -1;
            if (a.kin_part && alive) kin += a.kin_hmw * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        } else if (i < count) {
            a.key[i] = -1;
        }
        warp_count_losses(a.losses, D, lost);
        if (a.acc) deposit64<D>(g, p, alive, a.acc, a.scale);
    }
    if (a.kin_part) block_sum_to(kin, a.kin_part);
}

template <int D>
__global__ void __launch_bounds__(kPicThreads) k_deposit64(Deposit64Args a) {
    const GridView& g = a.g;
    const long long count = *a.count;
    const int lane = threadIdx.x & 31;
    for (long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < count;
         base += (long long)gridDim.x * blockDim.x) {
        const long long i = base + lane;
        double p[3] = {0, 0, 0};
        bool alive = i < count;
        if (alive) {
            p[0] = a.pos[0][i];
            alive = isfinite(p[0]);
            for (int d = 1; d < D && alive; ++d) p[d] = a.pos[d][i];
        }
        deposit64<D>(g, p, alive, a.acc, a.scale);
    }
}

__global__ void k_keys64(GridView g, const double* __restrict__ x, const double* __restrict__ y,
                         const double* __restrict__ z, int* __restrict__ key, const long long* __restrict__ count) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *count) return;
    double p[3] = {x[i], g.dim > 1 ? y[i] : 0.0, g.dim > 2 ? z[i] : 0.0};
    key[i] = isfinite(p[0]) ? key64(g, p) : -1;
}

}  // namespace

long long push64_blocks(long long n_upper) {
    const long long warps = (std::max<long long>(n_upper, 1) + 31) / 32;
    return std::min<long long>((warps + 7) / 8, 148LL * 16);
}

void launch_push64(const Push64Args& a, long long n_upper, cudaStream_t s) {
    if (n_upper <= 0) return;
    const unsigned blocks = (unsigned)push64_blocks(n_upper);
    if (a.g.dim == 1) k_push64<1><<<blocks, kPicThreads, 0, s>>>(a);
    else if (a.g.dim == 2) k_push64<2><<<blocks, kPicThreads, 0, s>>>(a);
    else k_push64<3><<<blocks, kPicThreads, 0, s>>>(a);
    count_launch();
}

void launch_deposit64(const Deposit64Args& a, long long n_upper, cudaStream_t s) {
    if (n_upper <= 0) return;
    const long long warps = (n_upper + 31) / 32;
    const unsigned blocks = (unsigned)std::min<long long>((warps + 7) / 8, 148LL * 16);
    if (a.g.dim == 1) k_deposit64<1><<<blocks, kPicThreads, 0, s>>>(a);
    else if (a.g.dim == 2) k_deposit64<2><<<blocks, kPicThreads, 0, s>>>(a);
    else k_deposit64<3><<<blocks, kPicThreads, 0, s>>>(a);
    count_launch();
}

void launch_keys64(const GridView& g, double* const pos[3], int* key, const long long* count, long long n_upper,
                   cudaStream_t s) {
    if (n_upper <= 0) return;
    { k_keys64<<<(unsigned)((n_upper + 255) / 256), 256, 0, s>>>(g, pos[0], pos[1], pos[2], key, count); count_launch(); }
}

}  // namespace PSUM_FP64_NS
}  // namespace psum_b200
