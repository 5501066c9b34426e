// mg_kernels.cuh -- sm_100a multigrid kernels of the B200 solver backend.
//
// Every level operator is a constant stencil (<= 27 taps with periodic wrap
// on the level's node box) plus an exception CSR for the rows that differ
// (mg_host.hpp).  All kernels are streaming kernels: one row per thread,
// coalesced along the last (fastest) dimension; neighbour rows are re-read
// through L1/L2.  The tap loop is unrolled for the common tap counts (5, 7,
// 9, 27) so every load of a row is in flight at once, interior rows use
// precomputed linear offsets, and the exception-row test runs beside the
// stencil loads instead of before them.  Kernels in the V-cycle return
// immediately once the solve's device-side `done` flag is set, so a fixed
// launch schedule can stop early without a host round trip; kernels in the
// body of the device-side refinement loop get no flag and skip that load.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/psum_field_solver.h"
#include "fastdiv.cuh"

namespace psum_b200 {

constexpr int kMaxTaps = 27;
constexpr int kThreads = 256;

struct MGState {
    double bnorm2;          // ||b||^2 after the source fix-ups
    double rnorm2_first;    // ||b - A x||^2 at the first check
    double rnorm2_last;     // ||b - A x||^2 at the last check
    int done;               // 1: converged (or diverged) -> gated kernels skip
    int cycles;             // V-cycles run before `done` was raised / in total
    int refinements;        // refinement steps run
    int status;             // psum_status of the solve
    int cycles_run;         // device-side counts of a solve looping in a graph
    int refinements_run;
    int stall;              // a TMA-staged sweep gave up waiting for a copy (never expected)
};

template <class T>
struct StencilDev {
    int n0, n1, n2;
    long long n;            // rows (below 2^31)
    int ns;
    int any_exc;            // some row is an exception row (mask has a bit set)
    signed char di[kMaxTaps], dj[kMaxTaps], dk[kMaxTaps];
    int off[kMaxTaps];      // linear offset of each tap on interior rows
    T c[kMaxTaps];
    FastDiv div12, div2;    // by n1 * n2 and by n2
    const uint32_t* mask;
    const uint32_t* mask_prefix;
    const int* exc_ptr;
    const int* exc_col;
    const T* exc_val;
};

template <class T>
struct AxisDev {
    int nf, nc;
    const int* p_c0;
    const int* p_c1;
    const T* p_w0;
    const T* p_w1;
    const int* r_f;   // stride 3
    const T* r_w;     // stride 3
};

template <class T>
struct XferDev {
    AxisDev<T> ax[3];
    FastDiv divc12, divc2;   // coarse box: by nc1 * nc2 and by nc2
    FastDiv divf12, divf2;   // fine box: by nf1 * nf2 and by nf2
};

__device__ __forceinline__ int wrap_idx(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// (A x)_r for one row of a stencil operator; Acc is the accumulation type.
// NS > 0: the operator has exactly NS taps; NS == 0: any count up to 27.
// Taps are summed in order, so every NS gives the same rounding.
// Load of data that is read-only while the kernel runs (RO = true, through
// the read-only path) or that the running kernel may have written (RO = false).
template <bool RO, class T>
__device__ __forceinline__ T ldv(const T* p) {
    if constexpr (RO) return __ldg(p);
    else return *p;
}

template <class T, class Acc, int NS, bool RO = true>
__device__ __forceinline__ Acc stencil_row(const StencilDev<T>& A, const T* __restrict__ x, int r) {
    const uint32_t word = A.any_exc ? __ldg(A.mask + (r >> 5)) : 0u;
    const int i = (int)fastdiv((unsigned)r, A.div12);
    const int rem = r - i * (int)A.div12.d;
    const int j = (int)fastdiv((unsigned)rem, A.div2);
    const int k = rem - j * A.n2;
    const bool interior = (A.n0 == 1 || (i > 0 && i < A.n0 - 1)) && (A.n1 == 1 || (j > 0 && j < A.n1 - 1)) &&
                          (A.n2 == 1 || (k > 0 && k < A.n2 - 1));
    constexpr int NT = NS > 0 ? NS : kMaxTaps;
    Acc s = Acc(0);
    if (interior) {
#pragma unroll
        for (int t = 0; t < NT; ++t)
            if (NS > 0 || t < A.ns) s += Acc(A.c[t]) * Acc(ldv<RO>(x + r + A.off[t]));
    } else {
#pragma unroll
        for (int t = 0; t < NT; ++t) {
            if (NS > 0 || t < A.ns) {
                const int ii = wrap_idx(i + A.di[t], A.n0);
                const int jj = wrap_idx(j + A.dj[t], A.n1);
                const int kk = wrap_idx(k + A.dk[t], A.n2);
                s += Acc(A.c[t]) * Acc(ldv<RO>(x + (ii * A.n1 + jj) * A.n2 + kk));
            }
        }
    }
    const uint32_t bit = 1u << (r & 31);
    if (word & bit) {
        const int q = (int)__ldg(A.mask_prefix + (r >> 5)) + __popc(word & (bit - 1u));
        const int b = __ldg(A.exc_ptr + q), e = __ldg(A.exc_ptr + q + 1);
        s = Acc(0);
        for (int t = b; t < e; ++t) s += Acc(__ldg(A.exc_val + t)) * Acc(ldv<RO>(x + __ldg(A.exc_col + t)));
    }
    return s;
}

enum SmoothMode { kSmooth = 0, kSmoothFromZero = 1, kResidual = 2 };

// kSmooth:          out = x + w (b - A x)      (damped Jacobi on the scaled system)
// kSmoothFromZero:  out = w b                  (first sweep from x = 0)
// kResidual:        out = b - A x
template <class T, int Mode, int NS, bool RO>
__device__ __forceinline__ void level_row(const StencilDev<T>& A, const T* __restrict__ x, const T* __restrict__ b,
                                          T* __restrict__ out, T omega, int r) {
    if (Mode == kSmoothFromZero) {
        out[r] = omega * ldv<RO>(b + r);
        return;
    }
    const T ax = stencil_row<T, T, NS, RO>(A, x, r);
    if (Mode == kSmooth) out[r] = ldv<RO>(x + r) + omega * (ldv<RO>(b + r) - ax);
    else out[r] = ldv<RO>(b + r) - ax;
}

template <class T, int Mode, int NS>
__global__ void __launch_bounds__(kThreads) k_level_op(StencilDev<T> A, const T* __restrict__ x,
                                                       const T* __restrict__ b, T* __restrict__ out, T omega,
                                                       const MGState* __restrict__ st) {
    if (st && st->done) return;   // st == nullptr: ungated (inside the device-side loop)
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= A.n) return;
    level_row<T, Mode, NS, true>(A, x, b, out, omega, r);
}

// ------------------------------------------------------ TMA-staged sweeps --
// k_level_op_tma: the same smooth / residual sweep as k_level_op for large
// 3-D levels whose rows are a multiple of 16 bytes long, with x staged in
// shared memory by the TMA engine.  The level's node box is viewed as planes
// (i) x rows (j) x columns (k), described by a tensor map.  A block owns a
// tile of TR rows x TC columns over a chunk of planes and marches along the
// planes: each plane's tile plus a halo (one row each side; the columns from
// 16 bytes before the tile to 16 bytes after it, so the box starts on a
// 16-byte boundary) arrives with one cp.async.bulk.tensor.3d into a ring of
// five plane slots, completing on the slot's mbarrier.  The plane index is
// wrapped in the copy's coordinate; halo rows and columns beyond the box
// (zero-filled by the copy) are patched from global memory with the
// stencil's own wrap (PSuM's cyclic neighbour rule), corners included.
// Planes p-1, p, p+1 are resident while p is computed and p+2, p+3 are in
// flight; thread 0 waits on the mbarriers and one block barrier per plane
// (two on edge tiles, around the halo patch) passes the planes on and orders
// the refill of the slot of p-2.
// Taps are summed in the same order as stencil_row, and exception rows take
// the same CSR path, so the results are bit-identical to k_level_op.  b is
// read one plane ahead into registers and out written directly (each once,
// coalesced).  Every mbarrier wait
// is bounded: after 2^16 suspended polls the block records a stall in
// *stall, and once a stall is recorded later waits return at once, so a
// wrong byte count cannot hang the GPU.  The tensor map covers only the
// solver's own level vector on this GPU; no multicast.
struct TmaTile {
    int P, R, C;          // planes, rows, columns of the view (n0, n1, n2)
    int tiles_c, tiles_r;
    int chunk, chunks;    // planes per block, blocks along the planes
};

// The two 3-D stencil shapes the TMA-staged sweep takes, with their taps in
// the order the host's stencil extraction sorts them (by (di, dj, dk)) and
// stencil_row sums them: the 7-point fine operator and the 27-point
// Galerkin coarse operator.  The launcher checks the level's taps against
// these; any other shape keeps the per-row kernel.
__host__ __device__ constexpr int tma_tap_d(int ns, int t, int axis) {
    return ns == 27 ? (axis == 0 ? t / 9 : (axis == 1 ? (t / 3) % 3 : t % 3)) - 1
                    : (axis == 0 ? (t == 0 ? -1 : (t == 6 ? 1 : 0))
                                 : (axis == 1 ? (t == 1 ? -1 : (t == 5 ? 1 : 0)) : (t == 2 ? -1 : (t == 4 ? 1 : 0))));
}

constexpr int kTmaThreads = 256;
constexpr int kTmaSlots = 5;

template <class T, int NS>
struct TmaShape {
    static constexpr int TC = sizeof(T) == 4 ? 128 : 64;   // columns per tile (512 bytes)
    static constexpr int TR = NS == 7 ? 16 : 8;             // rows per tile (27 taps: more tiles, fewer registers)
    static constexpr int KA = 16 / (int)sizeof(T);          // elements per 16 bytes: the column halo of the box
    static constexpr int W = TC + 2 * KA;                   // box columns (multiple of 16 bytes)
    static constexpr int H = TR + 2;                        // box rows
    static constexpr size_t box_bytes() { return sizeof(T) * (size_t)W * H; }
    static constexpr size_t slot_bytes() { return (box_bytes() + 127) / 128 * 128; }   // 128-byte aligned slots
    static constexpr int SLOTS = kTmaSlots;
    static constexpr size_t smem() { return slot_bytes() * SLOTS + 8 * SLOTS; }   // slots, then mbarriers
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Suspended test of phase `parity` of bar (returns after the phase completes
// or a hardware time limit).
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for phase `parity` of bar: at most 2^16 suspended polls; on
// expiry it records a stall in *stall and returns; once a stall is recorded
// (by this block or another) later waits return at once.
__device__ __forceinline__ void mbar_wait_bounded(unsigned long long* bar, unsigned parity, int* stall) {
    if (mbar_try_wait(bar, parity)) return;
    if (*(volatile int*)stall) return;
    for (int it = 0; it < (1 << 16); ++it)
        if (mbar_try_wait(bar, parity)) return;
    atomicExch(stall, 1);
}

// One tiled TMA load of the box at (x, y, z) of the tensor map into shared
// memory, completing its bytes on bar.  x is a multiple of 16 bytes.
__device__ __forceinline__ void tma_load_3d(void* dst, const void* tmap, int x, int y, int z, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(dst)),
        "l"(tmap), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

template <class T, int Mode, int NS>
__global__ void __launch_bounds__(kTmaThreads, 4) k_level_op_tma(const __grid_constant__ CUtensorMap xmap, StencilDev<T> A,
                                                              TmaTile V, const T* __restrict__ x,
                                                              const T* __restrict__ b, T* __restrict__ out, T omega,
                                                              const MGState* __restrict__ st, int* stall) {
    using S = TmaShape<T, NS>;
    constexpr int TC = S::TC, TR = S::TR, KA = S::KA, W = S::W, H = S::H;
    constexpr int NSL = S::SLOTS;
    constexpr int SLOT = (int)(S::slot_bytes() / sizeof(T));   // slot stride in elements
    if (st && st->done) return;   // st == nullptr: ungated (inside the device-side loop)
    extern __shared__ __align__(128) unsigned char tma_smem[];
    T* const ring = reinterpret_cast<T*>(tma_smem);   // [slot][H][W]; column c at index c - (c0 - KA)
    unsigned long long* const bar = reinterpret_cast<unsigned long long*>(tma_smem + S::slot_bytes() * NSL);
    int bid = blockIdx.x;
    const int tc = bid % V.tiles_c;
    bid /= V.tiles_c;
    const int tr = bid % V.tiles_r;
    const int ch = bid / V.tiles_r;
    const int c0 = tc * TC, r0 = tr * TR;
    const int pa = ch * V.chunk, pb = min(pa + V.chunk, V.P);
    const int nlocal = pb - pa + 2;   // local planes pa - 1 .. pb (wrapped)
    const bool edge = r0 == 0 || r0 + TR >= V.R || c0 == 0 || c0 + TC >= V.C;
    if (threadIdx.x == 0) {
        for (int q = 0; q < NSL; ++q) mbar_init(&bar[q], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    auto plane_of = [&](int L) {
        int p = pa - 1 + L;
        return p < 0 ? p + V.P : (p >= V.P ? p - V.P : p);
    };
    auto issue = [&](int L) {   // thread 0: local plane L into slot L % NSL
        const int slot = L % NSL;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(&bar[slot], (unsigned)S::box_bytes());
        tma_load_3d(ring + (size_t)slot * SLOT, &xmap, c0 - KA, r0 - 1, plane_of(L), &bar[slot]);
    };
    auto wrapi = [](int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); };
    // halo cells the box could not read, wrapped: row -1 (first row tile),
    // row R (last row tile), column -1 (first column tile), column C (last
    // column tile); corners belong to both a row and a column and are written
    // twice with the same value
    const bool top = r0 == 0, bottom = r0 + TR >= V.R, left = c0 == 0, right = c0 + TC >= V.C;
    const int lr_bottom = V.R - r0 + 1, k_right = V.C - c0 + 1;   // box row of row R, box column of column C (+1)
    auto patch = [&](int L) {
        if (!edge) return;
        T* slot = ring + (size_t)(L % NSL) * SLOT;
        const long long pbase = (long long)plane_of(L) * V.R;
        auto put = [&](int lr, int k) {   // box row lr (row r0 - 1 + lr), column c0 - 1 + k
            const int r = r0 - 1 + lr, c = c0 - 1 + k;
            slot[lr * W + k - 1 + KA] = x[(pbase + wrapi(r, V.R)) * V.C + wrapi(c, V.C)];
        };
        const int t = threadIdx.x;
        const int kmax = min(TC + 2, k_right + 1);   // columns up to column C
        const int lmax = min(H, lr_bottom + 1);      // rows up to row R
        if (top)
            for (int k = t; k < kmax; k += kTmaThreads) put(0, k);
        if (bottom)
            for (int k = t; k < kmax; k += kTmaThreads) put(lr_bottom, k);
        if (left)
            for (int lr = t; lr < lmax; lr += kTmaThreads) put(lr, 0);
        if (right)
            for (int lr = t; lr < lmax; lr += kTmaThreads) put(lr, k_right);
    };
    if (threadIdx.x == 0)
        for (int L = 0; L < min(NSL - 1, nlocal); ++L) issue(L);
    // each thread owns PER points of the tile (rows lr0 + 2u, column cc): their
    // b values and exception-mask words are loaded one plane ahead, so the
    // loads are in flight while the previous plane is computed
    constexpr int PER = TR * TC / kTmaThreads;
    static_assert(PER * kTmaThreads == TR * TC && kTmaThreads % TC == 0, "tile / block shape");
    constexpr int RSTEP = kTmaThreads / TC;
    const int lr0 = threadIdx.x / TC + 1, cc = threadIdx.x % TC;
    const int c = c0 + cc;
    const bool any_exc = A.any_exc != 0;
    // points u < nu of this thread lie inside the level (rows r0 + lr0 - 1 + u * RSTEP, column c)
    const int rfirst = r0 + lr0 - 1;
    const int nu = c < V.C && rfirst < V.R ? min(PER, (V.R - rfirst + RSTEP - 1) / RSTEP) : 0;
    const long long ustride = (long long)RSTEP * V.C;
    const int at0 = lr0 * W + cc + KA;   // this thread's first point in a slot; point u is RSTEP * W further
    static_assert(NS == 7 || NS == 27, "TMA-staged sweeps take the 7- and 27-point shapes");
    // 7 taps: b one plane ahead in registers; 27 taps (coarse levels, in L2):
    // b read at the point, so the 27 taps' loads have the registers
    constexpr bool BPRE = NS == 7;
    T bnext[PER];
    auto prefetch = [&](int p) {
        const T* bp = b + ((long long)p * V.R + rfirst) * V.C + c;
#pragma unroll
        for (int u = 0; u < PER; ++u) bnext[u] = u < nu ? __ldg(bp + u * ustride) : T(0);
    };
    const int planes = pb - pa;
    if (BPRE) prefetch(pa);
    for (int j = 0; j < planes; ++j) {
        const int p = pa + j;
        T bcur[PER];
        if (BPRE) {
#pragma unroll
            for (int u = 0; u < PER; ++u) bcur[u] = bnext[u];
            if (j + 1 < planes) prefetch(p + 1);
        }
        // local planes j, j + 1, j + 2 (planes p - 1, p, p + 1) must have
        // landed: thread 0 waits (one poller instead of a block of them), the
        // block barrier passes the completed copies on to every thread
        const int Lfirst = j == 0 ? 0 : j + 2;
        if (threadIdx.x == 0)
            for (int L = Lfirst; L <= j + 2; ++L) mbar_wait_bounded(&bar[L % NSL], (unsigned)((L / NSL) & 1), stall);
        __syncthreads();   // planes landed; every thread is done with plane j - 1's slot
        if (edge) {
            for (int L = Lfirst; L <= j + 2; ++L) patch(L);
            __syncthreads();
        }
        if (threadIdx.x == 0 && j + NSL - 1 < nlocal) issue(j + NSL - 1);   // refills the slot of local j - 1
        // ring index of this thread's first point in the slots of planes p - 1, p, p + 1
        const int bm = (j % NSL) * SLOT + at0, b0 = ((j + 1) % NSL) * SLOT + at0, bp = ((j + 2) % NSL) * SLOT + at0;
        const long long row0 = ((long long)p * V.R + rfirst) * V.C + c;   // global row index of point 0
        auto point = [&](int u, T bval) {
            const int du = u * (RSTEP * W);
            const long long row = row0 + u * ustride;
            T s = T(0);
#pragma unroll
            for (int t = 0; t < NS; ++t) {
                const int di = tma_tap_d(NS, t, 0);
                const int base = di < 0 ? bm : (di > 0 ? bp : b0);
                s += A.c[t] * ring[base + tma_tap_d(NS, t, 1) * W + tma_tap_d(NS, t, 2) + du];
            }
            if (any_exc) {
                const int r32 = (int)row;
                const uint32_t word = __ldg(A.mask + (r32 >> 5));
                const uint32_t bit = 1u << (r32 & 31);
                if (word & bit) {
                    const int q = (int)__ldg(A.mask_prefix + (r32 >> 5)) + __popc(word & (bit - 1u));
                    const int e_lo = __ldg(A.exc_ptr + q), e_hi = __ldg(A.exc_ptr + q + 1);
                    s = T(0);
                    for (int t = e_lo; t < e_hi; ++t) s += __ldg(A.exc_val + t) * __ldg(x + __ldg(A.exc_col + t));
                }
            }
            if (Mode == kSmooth) out[row] = ring[b0 + du] + omega * (bval - s);
            else out[row] = bval - s;
        };
        if constexpr (BPRE) {
#pragma unroll
            for (int u = 0; u < PER; ++u)
                if (u < nu) point(u, bcur[u]);
        } else {
#pragma unroll 1
            for (int u = 0; u < nu; ++u) point(u, __ldg(b + row0 + u * ustride));
        }
    }
    // every issued plane was waited on: nothing is in flight at exit
}

// b_c = dinv_c * (R r_f), x_c = 0 at coarse row c
template <class T, bool RO>
__device__ __forceinline__ void restrict_row(const XferDev<T>& X, const T* __restrict__ rf, T* __restrict__ bc,
                                             T* __restrict__ xc, const T* __restrict__ dinv_c, int c) {
    const int nc1 = X.ax[1].nc, nc2 = X.ax[2].nc;
    const int nf1 = X.ax[1].nf, nf2 = X.ax[2].nf;
    const int ci = (int)fastdiv((unsigned)c, X.divc12);
    const int rem = c - ci * nc1 * nc2;
    const int cj = (int)fastdiv((unsigned)rem, X.divc2);
    const int ck = rem - cj * nc2;
    T s = T(0);
#pragma unroll
    for (int qa = 0; qa < 3; ++qa) {
        const int fi = __ldg(X.ax[0].r_f + 3 * ci + qa);
        if (fi < 0) continue;
        const T wi = __ldg(X.ax[0].r_w + 3 * ci + qa);
#pragma unroll
        for (int qb = 0; qb < 3; ++qb) {
            const int fj = __ldg(X.ax[1].r_f + 3 * cj + qb);
            if (fj < 0) continue;
            const T wij = wi * __ldg(X.ax[1].r_w + 3 * cj + qb);
            const T* row = rf + (fi * nf1 + fj) * nf2;
#pragma unroll
            for (int qc = 0; qc < 3; ++qc) {
                const int fk = __ldg(X.ax[2].r_f + 3 * ck + qc);
                if (fk < 0) continue;
                s += (wij * __ldg(X.ax[2].r_w + 3 * ck + qc)) * ldv<RO>(row + fk);
            }
        }
    }
    bc[c] = s * __ldg(dinv_c + c);
    xc[c] = T(0);
}

template <class T>
__global__ void __launch_bounds__(kThreads) k_restrict(XferDev<T> X, const T* __restrict__ rf, T* __restrict__ bc,
                                                       T* __restrict__ xc, const T* __restrict__ dinv_c,
                                                       const MGState* __restrict__ st) {
    if (st && st->done) return;   // st == nullptr: ungated (inside the device-side loop)
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= X.ax[0].nc * X.ax[1].nc * X.ax[2].nc) return;
    restrict_row<T, true>(X, rf, bc, xc, dinv_c, c);
}

// (P x_c) at fine row f
template <class T, bool RO>
__device__ __forceinline__ T prolong_value(const XferDev<T>& X, const T* __restrict__ xc, int f) {
    const int nf1 = X.ax[1].nf, nf2 = X.ax[2].nf;
    const int nc1 = X.ax[1].nc, nc2 = X.ax[2].nc;
    const int fi = (int)fastdiv((unsigned)f, X.divf12);
    const int rem = f - fi * nf1 * nf2;
    const int fj = (int)fastdiv((unsigned)rem, X.divf2);
    const int fk = rem - fj * nf2;
    const int ci[2] = {__ldg(X.ax[0].p_c0 + fi), __ldg(X.ax[0].p_c1 + fi)};
    const int cj[2] = {__ldg(X.ax[1].p_c0 + fj), __ldg(X.ax[1].p_c1 + fj)};
    const int ck[2] = {__ldg(X.ax[2].p_c0 + fk), __ldg(X.ax[2].p_c1 + fk)};
    const T wi[2] = {__ldg(X.ax[0].p_w0 + fi), __ldg(X.ax[0].p_w1 + fi)};
    const T wj[2] = {__ldg(X.ax[1].p_w0 + fj), __ldg(X.ax[1].p_w1 + fj)};
    const T wk[2] = {__ldg(X.ax[2].p_w0 + fk), __ldg(X.ax[2].p_w1 + fk)};
    T s = T(0);
#pragma unroll
    for (int a = 0; a < 2; ++a) {
        if (ci[a] < 0) continue;
#pragma unroll
        for (int b2 = 0; b2 < 2; ++b2) {
            if (cj[b2] < 0) continue;
#pragma unroll
            for (int c2 = 0; c2 < 2; ++c2) {
                if (ck[c2] < 0) continue;
                s += (wi[a] * wj[b2] * wk[c2]) * ldv<RO>(xc + (ci[a] * nc1 + cj[b2]) * nc2 + ck[c2]);
            }
        }
    }
    return s;
}

// x_f += P x_c at fine row f
template <class T, bool RO>
__device__ __forceinline__ void prolong_row(const XferDev<T>& X, const T* __restrict__ xc, T* __restrict__ xf, int f) {
    const T s = prolong_value<T, RO>(X, xc, f);
    xf[f] = s + xf[f];
}

// Four consecutive fine nodes along the last axis per thread (levels whose
// rows are a multiple of 4 nodes long): the first two axes' transfer
// factors and their products are loaded and formed once for the four, and
// x_f moves as one 4-wide access.  Each node's terms are summed in
// prolong_value's order, so the bits are prolong_row's.
template <class T>
__global__ void __launch_bounds__(kThreads) k_prolong_add_row4(XferDev<T> X, const T* __restrict__ xc,
                                                               T* __restrict__ xf, const MGState* __restrict__ st) {
    if (st && st->done) return;
    const int nf1 = X.ax[1].nf, nf2 = X.ax[2].nf;
    const int nc1 = X.ax[1].nc, nc2 = X.ax[2].nc;
    const long long quads = (long long)X.ax[0].nf * nf1 * nf2 / 4;
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= quads) return;
    const int f = (int)(q * 4);
    const int fi = (int)fastdiv((unsigned)f, X.divf12);
    const int rem = f - fi * nf1 * nf2;
    const int fj = (int)fastdiv((unsigned)rem, X.divf2);
    const int fk0 = rem - fj * nf2;
    const int ci[2] = {__ldg(X.ax[0].p_c0 + fi), __ldg(X.ax[0].p_c1 + fi)};
    const int cj[2] = {__ldg(X.ax[1].p_c0 + fj), __ldg(X.ax[1].p_c1 + fj)};
    const T wi[2] = {__ldg(X.ax[0].p_w0 + fi), __ldg(X.ax[0].p_w1 + fi)};
    const T wj[2] = {__ldg(X.ax[1].p_w0 + fj), __ldg(X.ax[1].p_w1 + fj)};
    int ck[4][2];
    T wk[4][2];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        ck[u][0] = __ldg(X.ax[2].p_c0 + fk0 + u);
        ck[u][1] = __ldg(X.ax[2].p_c1 + fk0 + u);
        wk[u][0] = __ldg(X.ax[2].p_w0 + fk0 + u);
        wk[u][1] = __ldg(X.ax[2].p_w1 + fk0 + u);
    }
    T s[4] = {T(0), T(0), T(0), T(0)};
#pragma unroll
    for (int a = 0; a < 2; ++a) {
        if (ci[a] < 0) continue;
#pragma unroll
        for (int b2 = 0; b2 < 2; ++b2) {
            if (cj[b2] < 0) continue;
            const T wij = wi[a] * wj[b2];
            const T* row = xc + (ci[a] * nc1 + cj[b2]) * nc2;
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int c2 = 0; c2 < 2; ++c2) {
                    if (ck[u][c2] < 0) continue;
                    s[u] += (wij * wk[u][c2]) * __ldg(row + ck[u][c2]);
                }
        }
    }
    if constexpr (sizeof(T) == 4) {
        float4* p = reinterpret_cast<float4*>(xf + f);
        float4 o = *p;
        o.x = s[0] + o.x;
        o.y = s[1] + o.y;
        o.z = s[2] + o.z;
        o.w = s[3] + o.w;
        *p = o;
    } else {
#pragma unroll
        for (int u = 0; u < 4; ++u) xf[f + u] = s[u] + xf[f + u];
    }
}

// kProlongPer fine points per thread (a block's points are kProlongPer
// consecutive runs of kThreads), their loads issued together.
constexpr int kProlongPer = 4;

template <class T>
__global__ void __launch_bounds__(kThreads) k_prolong_add(XferDev<T> X, const T* __restrict__ xc, T* __restrict__ xf,
                                                          const MGState* __restrict__ st) {
    if (st && st->done) return;   // st == nullptr: ungated (inside the device-side loop)
    const int nf = X.ax[0].nf * X.ax[1].nf * X.ax[2].nf;
    const int f0 = blockIdx.x * (blockDim.x * kProlongPer) + threadIdx.x;
    T e[kProlongPer], old[kProlongPer];
#pragma unroll
    for (int u = 0; u < kProlongPer; ++u) {
        const int f = f0 + u * (int)blockDim.x;
        e[u] = f < nf ? prolong_value<T, true>(X, xc, f) : T(0);
        old[u] = f < nf ? xf[f] : T(0);
    }
#pragma unroll
    for (int u = 0; u < kProlongPer; ++u) {
        const int f = f0 + u * (int)blockDim.x;
        if (f < nf) xf[f] = e[u] + old[u];
    }
}

// x = Ainv b (dense, row-major), one warp per row, fixed shuffle tree.  The
// inverse and the sums are FP64 in both backends: the coarsest operator of a
// periodic problem pinned at one node is nearly singular (its near-constant
// mode), so its inverse has entries far larger than FP32 can cancel.
template <class T, bool RO>
__device__ __forceinline__ double dense_row(const double* __restrict__ Ainv, const T* __restrict__ b, int n, int row,
                                            int lane) {
    const double* a = Ainv + (long long)row * n;
    double s = 0.0;
    for (int c = lane; c < n; c += 32) s += __ldg(a + c) * (double)ldv<RO>(b + c);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    return s;
}

template <class T>
__global__ void __launch_bounds__(kThreads) k_dense_mv(const double* __restrict__ Ainv, const T* __restrict__ b,
                                                       T* __restrict__ x, int n, const MGState* __restrict__ st) {
    if (st && st->done) return;   // st == nullptr: ungated (inside the device-side loop)
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= n) return;
    const double s = dense_row<T, true>(Ainv, b, n, warp, lane);
    if (lane == 0) x[warp] = (T)s;
}

// Block-level FP64 sum in a fixed order (deterministic for a fixed launch).
__device__ __forceinline__ double block_sum(double v) {
    __shared__ double sh[kThreads / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += sh[q];
    return t;   // valid in thread 0
}

// FP64 residual of the unscaled fine operator: r = b - A x; optional output
// bhat = TOut(dinv * r) (the FP32 defect of the refinement); per-block
// partial sums of r^2 (grid-stride, fixed grid -> deterministic).
template <class TOut, int NS>
__global__ void __launch_bounds__(kThreads, NS == 27 || NS == 0 ? 2 : 3) k_residual64(StencilDev<double> A, const double* __restrict__ x,
                                                         const double* __restrict__ b, const double* __restrict__ dinv,
                                                         TOut* __restrict__ bhat, double* __restrict__ partials,
                                                         const MGState* __restrict__ st, int gated) {
    if (gated && st && st->done) return;
    double acc = 0.0;
    const int S = gridDim.x * blockDim.x;
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    // four grid strides per iteration, all loads first (the sums keep the order of the plain loop)
    constexpr int U = 4;
    for (; r + (U - 1) * S < A.n; r += U * S) {
        double ax[U], bb[U], dd[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            ax[u] = stencil_row<double, double, NS>(A, x, r + u * S);
            bb[u] = b[r + u * S];
            dd[u] = bhat ? dinv[r + u * S] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const double res = bb[u] - ax[u];
            acc += res * res;
            if (bhat) bhat[r + u * S] = TOut(dd[u] * res);
        }
    }
    for (; r < A.n; r += S) {
        const double ax = stencil_row<double, double, NS>(A, x, r);
        const double res = b[r] - ax;
        acc += res * res;
        if (bhat) bhat[r] = TOut(dinv[r] * res);
    }
    const double t = block_sum(acc);
    if (threadIdx.x == 0) partials[blockIdx.x] = t;
}

__global__ void __launch_bounds__(kThreads) k_norm2(const double* __restrict__ v, long long n,
                                                    double* __restrict__ partials) {
    double acc = 0.0;
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x)
        acc += v[r] * v[r];
    const double t = block_sum(acc);
    if (threadIdx.x == 0) partials[blockIdx.x] = t;
}

// Per-block sums of v (the mean of a null-space solve's vectors), in the
// fixed order of k_norm2.
__global__ void __launch_bounds__(kThreads) k_sum(const double* __restrict__ v, long long n,
                                                  double* __restrict__ partials) {
    double acc = 0.0;
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x)
        acc += v[r];
    const double t = block_sum(acc);
    if (threadIdx.x == 0) partials[blockIdx.x] = t;
}

// v -= sum(partials) / n: projection onto the mean-zero vectors.  Every block
// adds the partials in the same order, so all see the same mean.
__global__ void __launch_bounds__(kThreads) k_sub_mean(double* __restrict__ v, long long n,
                                                       const double* __restrict__ partials, int nparts) {
    __shared__ double mean;
    if (threadIdx.x < 32) {
        double a = 0.0;
        for (int i = threadIdx.x; i < nparts; i += 32) a += partials[i];
        for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if (threadIdx.x == 0) mean = a / (double)n;
    }
    __syncthreads();
    const double m = mean;
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x)
        v[r] -= m;
}

// bhat = T(dinv * b) (start of an FP64 solve: hadamard_to, multigrid_core.hpp:208)
template <class T>
__global__ void __launch_bounds__(kThreads) k_scale(const double* __restrict__ b, const double* __restrict__ dinv,
                                                    T* __restrict__ out, long long n) {
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n) out[r] = T(dinv[r] * b[r]);
}

// x += double(e)  (sycl_multigrid32f_gpu.cpp:153-155)
template <class T>
__global__ void __launch_bounds__(kThreads) k_correct(double* __restrict__ x, const T* __restrict__ e, long long n,
                                                      const MGState* __restrict__ st) {
    if (st && st->done) return;   // st == nullptr: ungated (inside the device-side loop)
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n) x[r] += (double)e[r];
}

__global__ void k_addback(double* __restrict__ b, const unsigned long long* __restrict__ idx,
                          const double* __restrict__ v, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) atomicAdd(b + idx[i], v[i]);   // several add-back terms may hit one node, as in cuda_multigrid_gpu.cu:36-44
}

__global__ void k_replace(double* __restrict__ b, const unsigned long long* __restrict__ idx,
                          const double* __restrict__ v, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[idx[i]] = v[i];
}

// Convergence test on ||r||^2 = s between refinements.
__device__ __forceinline__ void check_update(MGState* st, double s, double tol, int cycles, int refinements) {
    if (st && st->done) return;   // st == nullptr: ungated (inside the device-side loop)
    if (st->rnorm2_first < 0) st->rnorm2_first = s;
    st->rnorm2_last = s;
    st->cycles = cycles;
    st->refinements = refinements;
    const double bn = st->bnorm2 > 0 ? st->bnorm2 : 1.0;
    if (!(s == s) || s > 1e300 || (st->rnorm2_first > 0 && s > 1e12 * st->rnorm2_first)) {
        st->status = PSUM_ERR_DIVERGED;
        st->done = 1;
    } else if (tol > 0 && s <= tol * tol * bn) {
        st->done = 1;
    }
}

// Fixed-order two-level sum of the per-block partials (valid in thread 0).
__device__ __forceinline__ double sum_partials(const double* __restrict__ partials, int nparts) {
    __shared__ double sh[32];
    double v = 0.0;
    if (threadIdx.x < 32) {
        for (int q = threadIdx.x; q < nparts; q += 32) v += partials[q];
        sh[threadIdx.x] = v;
    }
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int q = 0; q < 32; ++q) s += sh[q];
    return s;
}

// Check of a solve that loops in a CUDA graph: counts the `batch` cycles just
// run, applies the convergence test, and sets the loop condition (continue
// while not done and below max_cycles).  Each continuation adds the loop
// body's kernel count to the mapped launch counter.
__global__ void k_check_loop(const double* __restrict__ partials, int nparts, MGState* st, int batch,
                             int max_cycles, double tol, cudaGraphConditionalHandle loop,
                             unsigned long long body_kernels, unsigned long long* launch_counter) {
    const double s = sum_partials(partials, nparts);
    if (threadIdx.x != 0) return;
    if (batch > 0) {
        st->cycles_run += batch;
        st->refinements_run += 1;
    }
    check_update(st, s, tol, st->cycles_run, st->refinements_run);
    const bool more = !st->done && st->cycles_run < max_cycles;
    if (more) atomicAdd_system(launch_counter, body_kernels);
    cudaGraphSetConditional(loop, more ? 1u : 0u);
}

// Single-block state update. phase 0: start of solve (partials hold ||b||^2);
// phase 1: convergence check (partials hold ||r||^2); phase 2: final residual.
__global__ void k_check(const double* __restrict__ partials, int nparts, MGState* st, int phase, double tol,
                        int cycles, int refinements) {
    __shared__ double sh[32];
    double v = 0.0;
    // fixed-order two-level sum: thread t sums partials t, t+32, ...
    if (threadIdx.x < 32) {
        for (int q = threadIdx.x; q < nparts; q += 32) v += partials[q];
        sh[threadIdx.x] = v;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    double s = 0.0;
    for (int q = 0; q < 32; ++q) s += sh[q];
    if (phase == 0) {
        st->bnorm2 = s;
        st->rnorm2_first = -1.0;
        st->rnorm2_last = -1.0;
        st->done = 0;
        st->cycles = 0;
        st->refinements = 0;
        st->status = 0;
        st->cycles_run = 0;
        st->refinements_run = 0;
        st->stall = 0;
        return;
    }
    if (phase == 1) {
        check_update(st, s, tol, cycles, refinements);
        return;
    }
    // phase 2: final
    if (st->rnorm2_first < 0) st->rnorm2_first = s;
    st->rnorm2_last = s;
    if (!st->done) {
        st->cycles = cycles;
        st->refinements = refinements;
    }
    const double bn = st->bnorm2 > 0 ? st->bnorm2 : 1.0;
    if (!(s == s) || s > 1e300) st->status = PSUM_ERR_DIVERGED;
    else if (st->status == 0 && tol > 0 && s > tol * tol * bn) st->status = PSUM_ERR_NOT_CONVERGED;
}

}  // namespace psum_b200
