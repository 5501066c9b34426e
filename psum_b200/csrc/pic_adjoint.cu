// pic_adjoint.cu -- discrete adjoint of the electrostatic leapfrog step.
//
// Forward step n (cell units s = cell + offset per axis, velocity v):
//   rho^n = D(s^n)                  CIC deposit, rho_node = sum_p q w W_node(s_p) / vol
//   phi^n = S rho^n (+ external)    the Poisson solve (source fix-ups included in S)
//   G_e   = sum_k phi_k dW_k/ds_e   gradient of the bilinear/trilinear interpolant
//   v'    = v - kE G,  kE_e = (q/m) dt dr_e          (E = -dr G)
//   s'    = s + dtdr v',  dtdr_e = dt dr_e
// Backward, given the adjoints lx' = dL/ds', lv' = dL/dv' of the new state:
//   lv  = lv' + dtdr lx'                              (velocity adjoint)
//   lG  = -kE lv
//   lx  = lx' + sum_e lG_e dG_e/ds                    (k_adj_push, direct term)
//   mu  = sum_p sum_e lG_e dG_e/dphi                  (k_adj_push: the adjoint of the gather is a scatter)
//   nu  = S^T mu                                      (caller: a solve with the transposed operator)
//   lx += (q w / vol) sum_k nu_k dW_k/ds              (k_adj_deposit: the adjoint of the deposit is a gather)
// The scatter of mu is done in int64 fixed point with a scale chosen on the
// device from the largest contribution, so it is exact and independent of
// the order of the particles, like the forward deposit.  Arithmetic in FP64;
// the adjoint arrays are FP32 for mixed-precision contexts, FP64 otherwise.
// PSuM has no adjoint; this is new code for differentiable runs.
#include <cuda_runtime.h>

#include <cmath>

#include "../../include/psum_pic.h"
#include "pic.hpp"

namespace psum_b200 {

namespace {

struct AdjState {
    GridView g;
    int mixed;
    const int* key;          // mixed: internal cell keys
    const float* off[3];     // mixed: offsets in the cell
    const double* pos[3];    // FP64: absolute positions
    long long n;             // length of the adjoint arrays
    const long long* count;  // stored particles (device)
};

// Cell and offsets of particle i in FP64; false for an invalid particle.
template <int D>
__device__ __forceinline__ bool adj_cell(const AdjState& s, long long i, int c[3], double f[3]) {
    c[0] = c[1] = c[2] = 0;
    f[0] = f[1] = f[2] = 0.0;
    if (s.mixed) {
        const int k = s.key[i];
        if (k < 0 || k >= s.g.n_cells) return false;
        key_to_cell(s.g, k, c[0], c[1], c[2]);
#pragma unroll
        for (int a = 0; a < D; ++a) f[a] = (double)s.off[a][i];
        return true;
    }
    if (!isfinite(s.pos[0][i])) return false;
#pragma unroll
    for (int a = 0; a < D; ++a) {
        const double p = s.pos[a][i];
        const int base = (int)floor((p - s.g.lo[a]) * s.g.dr[a]);
        if (base < 0 || base >= s.g.M[a]) return false;   // outside the lattice: not a valid state
        f[a] = (p - (s.g.lo[a] + (double)base * s.g.dx[a])) * s.g.dr[a];
        c[a] = base;
    }
    return true;
}

// Node of corner B (bit a = upper on axis a) of cell c.
template <int D>
__device__ __forceinline__ long long adj_node(const GridView& g, int B, const int c[3]) {
    const int i = (B & 1) ? next_node(g, 0, c[0]) : c[0];
    const int j = (B & 2) ? next_node(g, 1, c[1]) : c[1];
    const int k = (D == 3) ? ((B & 4) ? next_node(g, 2, c[2]) : c[2]) : 0;
    return node_index(g, i, j, k);
}

// dW_B/ds_e and d2W_B/(ds_e ds_d), d != e, of the CIC weight of corner B.
template <int D>
__device__ __forceinline__ double dW(int B, int e, const double f[3]) {
    double w = ((B >> e) & 1) ? 1.0 : -1.0;
#pragma unroll
    for (int a = 0; a < D; ++a)
        if (a != e) w *= ((B >> a) & 1) ? f[a] : 1.0 - f[a];
    return w;
}

template <int D>
__device__ __forceinline__ double d2W(int B, int e, int d, const double f[3]) {
    double w = (((B >> e) & 1) ? 1.0 : -1.0) * (((B >> d) & 1) ? 1.0 : -1.0);
#pragma unroll
    for (int a = 0; a < D; ++a)
        if (a != e && a != d) w *= ((B >> a) & 1) ? f[a] : 1.0 - f[a];
    return w;
}

struct AdjPushArgs {
    AdjState s;
    const double* phi;
    double kE[3], dtdr[3];
    void* lx[3];
    void* lv[3];
    unsigned long long* acc;   // int64 fixed-point scatter of mu
    unsigned* maxbits;         // pass 1: max over particles of sum_e |lG_e| (float bits)
    const double* scale;       // pass 2: fixed-point scale
};

template <class T>
__device__ __forceinline__ double ldT(void* p, long long i) {
    return (double)static_cast<T*>(p)[i];
}
template <class T>
__device__ __forceinline__ void stT(void* p, long long i, double v) {
    static_cast<T*>(p)[i] = (T)v;
}

// Pass 1 (SCATTER = false): the largest per-particle scatter magnitude.
// Pass 2 (SCATTER = true): adjoint updates in place and the mu scatter.
template <int D, class T, bool SCATTER>
__global__ void __launch_bounds__(256) k_adj_push(AdjPushArgs a) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    float mymax = 0.f;
    if (i < a.s.n && i < *a.s.count) {
        int c[3];
        double f[3];
        if (adj_cell<D>(a.s, i, c, f)) {
            double lvp[3], lG[3] = {0.0, 0.0, 0.0};
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                lvp[q] = ldT<T>(a.lv[q], i);
                if (q < D) lvp[q] += a.dtdr[q] * ldT<T>(a.lx[q], i);
            }
#pragma unroll
            for (int e = 0; e < D; ++e) lG[e] = -a.kE[e] * lvp[e];
            if (!SCATTER) {
                double m = 0.0;
#pragma unroll
                for (int e = 0; e < D; ++e) m += fabs(lG[e]);
                mymax = (float)m * 1.0001f;
            } else {
                double phic[8];
#pragma unroll
                for (int B = 0; B < (1 << D); ++B) phic[B] = __ldg(a.phi + adj_node<D>(a.s.g, B, c));
                const double sc = *a.scale;
#pragma unroll
                for (int q = 0; q < 3; ++q) stT<T>(a.lv[q], i, lvp[q]);
#pragma unroll
                for (int d = 0; d < D; ++d) {
                    double dx = 0.0;
#pragma unroll
                    for (int e = 0; e < D; ++e) {
                        if (e == d) continue;
                        double h = 0.0;
#pragma unroll
                        for (int B = 0; B < (1 << D); ++B) h += phic[B] * d2W<D>(B, e, d, f);
                        dx += lG[e] * h;
                    }
                    stT<T>(a.lx[d], i, ldT<T>(a.lx[d], i) + dx);
                }
#pragma unroll
                for (int B = 0; B < (1 << D); ++B) {
                    double m = 0.0;
#pragma unroll
                    for (int e = 0; e < D; ++e) m += lG[e] * dW<D>(B, e, f);
                    const long long val = __double2ll_rn(m * sc);
                    if (val != 0) atomicAdd(a.acc + adj_node<D>(a.s.g, B, c), (unsigned long long)val);
                }
            }
        }
    }
    if (!SCATTER) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mymax = fmaxf(mymax, __shfl_xor_sync(0xffffffffu, mymax, o));
        if ((threadIdx.x & 31) == 0 && mymax > 0.f) atomicMax(a.maxbits, __float_as_uint(mymax));
    }
}

// Fixed-point scale 2^e such that n * max * 2^e < 2^60 (power of two: exact).
__global__ void k_adj_scale(const unsigned* maxbits, long long n, double* scale) {
    const double m = (double)__uint_as_float(*maxbits) * (double)(n > 0 ? n : 1);
    int e = 60;
    if (m > 0.0) e = 60 - (int)ceil(log2(m));
    if (e > 400) e = 400;
    scale[0] = ldexp(1.0, e);
    scale[1] = ldexp(1.0, -e);
}

// mu_out += acc * 2^-e; acc = 0
__global__ void k_adj_mu_out(unsigned long long* acc, const double* scale, double* mu, long long n_nodes) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_nodes) return;
    mu[k] += (double)(long long)acc[k] * scale[1];
    acc[k] = 0ull;
}

struct AdjDepArgs {
    AdjState s;
    const double* nu;
    double cq;   // q w / vol
    void* lx[3];
};

template <int D, class T>
__global__ void __launch_bounds__(256) k_adj_deposit(AdjDepArgs a) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.s.n || i >= *a.s.count) return;
    int c[3];
    double f[3];
    if (!adj_cell<D>(a.s, i, c, f)) return;
    double nuc[8];
#pragma unroll
    for (int B = 0; B < (1 << D); ++B) nuc[B] = __ldg(a.nu + adj_node<D>(a.s.g, B, c));
#pragma unroll
    for (int d = 0; d < D; ++d) {
        double g = 0.0;
#pragma unroll
        for (int B = 0; B < (1 << D); ++B) g += nuc[B] * dW<D>(B, d, f);
        stT<T>(a.lx[d], i, ldT<T>(a.lx[d], i) + a.cq * g);
    }
}

unsigned blocks256(long long n) { return (unsigned)((n + 255) / 256 > 0 ? (n + 255) / 256 : 1); }

AdjState make_state(psum_pic_ctx* c, int species) {
    Species& sp = species_at(c, species);
    AdjState s{};
    s.g = c->g;
    s.mixed = c->precision == PSUM_PIC_MIXED;
    s.n = sp.n;
    s.count = c->count.p + species;
    if (s.mixed) {
        ensure_keys(c, sp);
        s.key = sp.key[sp.cur].p;
        for (int a = 0; a < c->g.dim; ++a) s.off[a] = sp.off[a][sp.cur].p;
    } else {
        for (int a = 0; a < c->g.dim; ++a) s.pos[a] = sp.pos64[a][sp.cur].p;
    }
    return s;
}

void split_arrays(psum_pic_ctx* c, Species& sp, void* base, int count, void* out[3]) {
    const size_t elem = c->precision == PSUM_PIC_MIXED ? sizeof(float) : sizeof(double);
    for (int q = 0; q < 3; ++q)
        out[q] = q < count ? static_cast<char*>(base) + (size_t)q * (size_t)sp.n * elem : nullptr;
}

}  // namespace
}  // namespace psum_b200

using namespace psum_b200;

extern "C" {

EXPORT int psum_pic_adjoint_push(psum_pic_ctx* ctx, int species, const double* phi_dev, double dt, void* lam_x_dev,
                                 void* lam_v_dev, double* mu_dev) {
    return guarded([&] {
        ctx_check(ctx);
        Species& sp = species_at(ctx, species);
        if (!phi_dev || !lam_x_dev || !lam_v_dev || !mu_dev) throw std::invalid_argument("adjoint_push: null pointer");
        if (!std::isfinite(dt)) throw Error(PSUM_ERR_NONFINITE, "adjoint_push: non-finite dt");
        if (sp.n <= 0) return;
        cudaStream_t s = ctx->stream;
        const long long nn = ctx->g.n_nodes;
        ctx->adj_acc.alloc((size_t)nn);
        ctx->adj_scale.alloc(2);
        ctx->adj_max.alloc(1);
        cuda_check(cudaMemsetAsync(ctx->adj_acc.p, 0, sizeof(unsigned long long) * nn, s), "memset");
        cuda_check(cudaMemsetAsync(ctx->adj_max.p, 0, sizeof(unsigned), s), "memset");
        AdjPushArgs a{};
        a.s = make_state(ctx, species);
        a.phi = phi_dev;
        const double qm = sp.q / sp.m;
        for (int d = 0; d < 3; ++d) {
            a.kE[d] = qm * dt * ctx->g.dr[d];
            a.dtdr[d] = dt * ctx->g.dr[d];
        }
        split_arrays(ctx, sp, lam_x_dev, ctx->g.dim, a.lx);
        split_arrays(ctx, sp, lam_v_dev, 3, a.lv);
        a.acc = ctx->adj_acc.p;
        a.maxbits = ctx->adj_max.p;
        a.scale = ctx->adj_scale.p;
        const unsigned gb = blocks256(sp.n);
        const bool mixed = ctx->precision == PSUM_PIC_MIXED;
#define PSUM_ADJ(D_, T_)                                                              \
    do {                                                                             \
        { k_adj_push<D_, T_, false><<<gb, 256, 0, s>>>(a); count_launch(); }         \
        { k_adj_scale<<<1, 1, 0, s>>>(ctx->adj_max.p, sp.n, ctx->adj_scale.p); count_launch(); } \
        { k_adj_push<D_, T_, true><<<gb, 256, 0, s>>>(a); count_launch(); }          \
    } while (0)
        if (ctx->g.dim == 2) {
            if (mixed) PSUM_ADJ(2, float);
            else PSUM_ADJ(2, double);
        } else {
            if (mixed) PSUM_ADJ(3, float);
            else PSUM_ADJ(3, double);
        }
#undef PSUM_ADJ
        { k_adj_mu_out<<<blocks256(nn), 256, 0, s>>>(ctx->adj_acc.p, ctx->adj_scale.p, mu_dev, nn); count_launch(); }
        cuda_check(cudaGetLastError(), "adjoint_push launch");
    });
}

EXPORT int psum_pic_adjoint_deposit(psum_pic_ctx* ctx, int species, const double* nu_dev, void* lam_x_dev) {
    return guarded([&] {
        ctx_check(ctx);
        Species& sp = species_at(ctx, species);
        if (!nu_dev || !lam_x_dev) throw std::invalid_argument("adjoint_deposit: null pointer");
        if (sp.n <= 0) return;
        cudaStream_t s = ctx->stream;
        AdjDepArgs a{};
        a.s = make_state(ctx, species);
        a.nu = nu_dev;
        double vol = 1.0;
        for (int d = 0; d < ctx->g.dim; ++d) vol *= ctx->g.dx[d];
        a.cq = sp.q * sp.w / vol;
        split_arrays(ctx, sp, lam_x_dev, ctx->g.dim, a.lx);
        const unsigned gb = blocks256(sp.n);
        const bool mixed = ctx->precision == PSUM_PIC_MIXED;
        if (ctx->g.dim == 2) {
            if (mixed) k_adj_deposit<2, float><<<gb, 256, 0, s>>>(a);
            else k_adj_deposit<2, double><<<gb, 256, 0, s>>>(a);
        } else {
            if (mixed) k_adj_deposit<3, float><<<gb, 256, 0, s>>>(a);
            else k_adj_deposit<3, double><<<gb, 256, 0, s>>>(a);
        }
        count_launch();
        cuda_check(cudaGetLastError(), "adjoint_deposit launch");
    });
}

}  // extern "C"
