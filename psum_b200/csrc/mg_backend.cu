// mg_backend.cu -- the B200 multigrid solver backends behind PSuM's func_table.
//
//   cuda_multigrid32f_gpu : FP32 V-cycles inside FP64 iterative refinement,
//                           restating sycl_multigrid32f_gpu::solve
//                           (src/field_solver/implements/sycl_multigrid32f_gpu.cpp:106-160)
//   cuda_multigrid64_gpu  : FP64 V-cycles with the caller's x as initial guess,
//                           restating cuda_multigrid_gpu::solve
//                           (src/field_solver/implements/cuda_multigrid_gpu.cu:140-180)
//
// Both accept PSuM's option grammar (sycl_multigrid32f_gpu.cpp:162-196) and
// add `tol` (stop once ||b - A x||_2 <= tol ||b||_2, checked on the device
// every correction_interval cycles; 0 = run exactly max_cycles like PSuM),
// `max_coarse`, and `periodic_I/J/K 1` (wrap-around transfers on that axis
// for operators whose node lattice wraps, where PSuM's open-interval
// transfers make the V-cycle diverge), and `null_space 1` (a periodic
// operator assembled without a pinned node, singular with the constants as
// its null space: the coarse solve inverts Ahat_L + 1 1^T / n and the solve
// returns the mean-zero solution of b minus its mean).  The whole solve is enqueued on one stream without host
// synchronisation; func_table.solve synchronises at the end, like PSuM.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include <cudaTypedefs.h>

#include "common.hpp"
#include "mg_backend.hpp"
#include "mg_host.hpp"
#include "mg_kernels.cuh"

namespace psum_b200 {

namespace mgdetail {

inline unsigned grid_for(long long n, int threads = kThreads) {
    return (unsigned)std::max<long long>(1, (n + threads - 1) / threads);
}

constexpr int kNormBlocks = 444;   // 3 x 148 SMs: fixed grid -> fixed reduction order

template <class T>
struct DevStencil {
    StencilDev<T> view{};
    DevBuf<uint32_t> mask, mask_prefix;
    DevBuf<int> exc_ptr, exc_col;
    DevBuf<T> exc_val;
    long long exceptions = 0;

    void upload(const StencilOp& op, cudaStream_t s) {
        mask.upload(op.mask.data(), op.mask.size(), s);
        mask_prefix.upload(op.mask_prefix.data(), op.mask_prefix.size(), s);
        exc_ptr.upload(op.exc_ptr.data(), op.exc_ptr.size(), s);
        exc_col.upload(op.exc_col.data(), op.exc_col.size(), s);
        std::vector<T> v(op.exc_val.begin(), op.exc_val.end());
        exc_val.upload(v.data(), v.size(), s);
        cuda_check(cudaStreamSynchronize(s), "upload stencil");
        exceptions = (long long)op.exc_rows.size();
        if (op.n >= (1LL << 31)) throw std::invalid_argument("multigrid: more than 2^31 - 1 rows per level");
        view.n0 = op.dims[0];
        view.n1 = op.dims[1];
        view.n2 = op.dims[2];
        view.n = op.n;
        view.ns = op.ns;
        view.any_exc = exceptions > 0;
        view.div12 = make_fastdiv((unsigned)(op.dims[1] * op.dims[2]));
        view.div2 = make_fastdiv((unsigned)op.dims[2]);
        for (int t = 0; t < op.ns && t < kMaxTaps; ++t) {
            view.di[t] = (signed char)op.delta[t][0];
            view.dj[t] = (signed char)op.delta[t][1];
            view.dk[t] = (signed char)op.delta[t][2];
            view.off[t] = (op.delta[t][0] * op.dims[1] + op.delta[t][1]) * op.dims[2] + op.delta[t][2];
            view.c[t] = T(op.coef[t]);
        }
        view.mask = mask.p;
        view.mask_prefix = mask_prefix.p;
        view.exc_ptr = exc_ptr.p;
        view.exc_col = exc_col.p;
        view.exc_val = exc_val.p;
    }
};

template <class T>
struct DevAxis {
    DevBuf<int> p_c0, p_c1, r_f;
    DevBuf<T> p_w0, p_w1, r_w;
    void upload(const Axis1D& a, cudaStream_t s, AxisDev<T>& view) {
        std::vector<T> w0(a.p_w0.begin(), a.p_w0.end()), w1(a.p_w1.begin(), a.p_w1.end()),
            rw(a.r_w.begin(), a.r_w.end());
        p_c0.upload(a.p_c0.data(), a.p_c0.size(), s);
        p_c1.upload(a.p_c1.data(), a.p_c1.size(), s);
        r_f.upload(a.r_f.data(), a.r_f.size(), s);
        p_w0.upload(w0.data(), w0.size(), s);
        p_w1.upload(w1.data(), w1.size(), s);
        r_w.upload(rw.data(), rw.size(), s);
        cuda_check(cudaStreamSynchronize(s), "upload transfer");
        view.nf = a.nf;
        view.nc = a.nc;
        view.p_c0 = p_c0.p;
        view.p_c1 = p_c1.p;
        view.p_w0 = p_w0.p;
        view.p_w1 = p_w1.p;
        view.r_f = r_f.p;
        view.r_w = r_w.p;
    }
};

// Launches of the stencil kernels with the operator's tap count as a
// compile-time constant where it is one of the common ones.
// 3-D levels of at least this many rows whose rows are a multiple of 16
// bytes long take the TMA-staged sweep (when the solver's option `tma` is on;
// option `tma_min_rows` overrides it).  Smaller levels stay in L2, where the
// per-row kernel's cached reads need no staging.
constexpr long long kTmaMinRows = 1LL << 20;

// Blocks of a TMA-staged sweep that fit on the GPU at once (SMs x resident
// blocks of the kernel), cached per kernel.
template <class T, int Mode, int NS>
int tma_resident_blocks() {
    static int blocks = 0;
    if (!blocks) {
        int dev = 0, sms = 0, per_sm = 0;
        cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
        cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
        cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_level_op_tma<T, Mode, NS>, kTmaThreads,
                                                                 TmaShape<T, NS>::smem()),
                   "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        blocks = std::max(1, sms * std::max(1, per_sm));
    }
    return blocks;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library).
inline PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        cuda_check(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q),
                   "cudaGetDriverEntryPoint");
        if (q != cudaDriverEntryPointSuccess || !p) throw Error(PSUM_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// The tensor map of a level vector viewed as (planes, rows, columns) with the
// sweep's box; the vector is one of the solver's own buffers on this GPU.
template <class T, int NS>
CUtensorMap make_level_map(const T* x, int P, int R, int C) {
    using S = TmaShape<T, NS>;
    CUtensorMap m;
    const cuuint64_t dims[3] = {(cuuint64_t)C, (cuuint64_t)R, (cuuint64_t)P};
    const cuuint64_t strides[2] = {(cuuint64_t)C * sizeof(T), (cuuint64_t)R * C * sizeof(T)};
    const cuuint32_t box[3] = {(cuuint32_t)S::W, (cuuint32_t)S::H, 1u};
    const cuuint32_t estr[3] = {1u, 1u, 1u};
    const CUresult r = tmap_encoder()(&m, sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                                      3, const_cast<T*>(x), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                      CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw Error(PSUM_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    return m;
}

// Tensor maps of the level vectors the sweeps read, by pointer, view and
// stencil shape (the shape sets the box).
struct TmapCache {
    struct Entry {
        const void* p;
        int P, R, C, ns;
        CUtensorMap m;
    };
    std::vector<Entry> e;
    template <class T, int NS>
    CUtensorMap get(const T* x, int P, int R, int C) {   // by value: a later insertion may move the entries
        for (auto& q : e)
            if (q.p == x && q.P == P && q.R == R && q.C == C && q.ns == NS) return q.m;
        e.push_back({x, P, R, C, NS, make_level_map<T, NS>(x, P, R, C)});
        return e.back().m;
    }
};

// Launch over V's tiles; the planes are cut into as many chunks as keep one
// wave of resident blocks busy (each chunk re-reads two halo planes).
template <class T, int Mode, int NS>
void launch_tma_ns(TmapCache& cache, const StencilDev<T>& A, const T* x, const T* b, T* out, T omega,
                   const MGState* st, int* stall, cudaStream_t s) {
    using S = TmaShape<T, NS>;
    static bool attr = false;
    if (!attr) {
        cuda_check(cudaFuncSetAttribute(k_level_op_tma<T, Mode, NS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)S::smem()),
                   "cudaFuncSetAttribute");
        attr = true;
    }
    TmaTile V{};
    V.P = A.n0;
    V.R = A.n1;
    V.C = A.n2;
    V.tiles_c = (V.C + S::TC - 1) / S::TC;
    V.tiles_r = (V.R + S::TR - 1) / S::TR;
    const CUtensorMap map = cache.get<T, NS>(x, V.P, V.R, V.C);
    const long long tiles = (long long)V.tiles_c * V.tiles_r;
    const long long want = std::max(1LL, (long long)tma_resident_blocks<T, Mode, NS>() / tiles);
    V.chunk = (int)std::max(1LL, (V.P + want - 1) / want);
    V.chunks = (V.P + V.chunk - 1) / V.chunk;
    const unsigned blocks = (unsigned)(tiles * V.chunks);
    k_level_op_tma<T, Mode, NS><<<blocks, kTmaThreads, S::smem(), s>>>(map, A, V, x, b, out, omega, st, stall);
}

// TMA-staged sweep of a level (k_level_op_tma); false when the level does
// not qualify (small, not 3-D, or rows not a multiple of 16 bytes).
template <class T, int Mode>
bool launch_level_op_tma(TmapCache& cache, long long min_rows, const StencilDev<T>& A, const T* x, const T* b, T* out,
                         T omega, const MGState* st, int* stall, cudaStream_t s) {
    if (Mode == kSmoothFromZero || A.n < min_rows) return false;
    if (!(A.n0 > 2 && A.n1 > 1 && A.n2 > 1)) return false;          // 3-D boxes only (2-D levels stay in L2)
    if ((A.n2 * (int)sizeof(T)) % 16 != 0) return false;             // tensor-map row pitch: 16-byte multiple
    if ((reinterpret_cast<uintptr_t>(x) & 15) != 0) return false;
    if (A.ns != 7 && A.ns != 27) return false;                         // the kernel's two stencil shapes
    for (int t = 0; t < A.ns; ++t)
        if (A.di[t] != tma_tap_d(A.ns, t, 0) || A.dj[t] != tma_tap_d(A.ns, t, 1) || A.dk[t] != tma_tap_d(A.ns, t, 2))
            return false;
    if (A.ns == 7) launch_tma_ns<T, Mode, 7>(cache, A, x, b, out, omega, st, stall, s);
    else launch_tma_ns<T, Mode, 27>(cache, A, x, b, out, omega, st, stall, s);
    count_launch();
    return true;
}

template <class T, int Mode>
void launch_level_op(const StencilDev<T>& A, const T* x, const T* b, T* out, T omega, const MGState* st,
                     cudaStream_t s, int* stall = nullptr, TmapCache* cache = nullptr,
                     long long tma_min_rows = kTmaMinRows) {
    if (stall && cache && launch_level_op_tma<T, Mode>(*cache, tma_min_rows, A, x, b, out, omega, st, stall, s)) return;
    const unsigned g = grid_for(A.n);
    if (Mode == kSmoothFromZero) k_level_op<T, Mode, 0><<<g, kThreads, 0, s>>>(A, x, b, out, omega, st);
    else if (A.ns == 5) k_level_op<T, Mode, 5><<<g, kThreads, 0, s>>>(A, x, b, out, omega, st);
    else if (A.ns == 7) k_level_op<T, Mode, 7><<<g, kThreads, 0, s>>>(A, x, b, out, omega, st);
    else if (A.ns == 9) k_level_op<T, Mode, 9><<<g, kThreads, 0, s>>>(A, x, b, out, omega, st);
    else if (A.ns == 27) k_level_op<T, Mode, 27><<<g, kThreads, 0, s>>>(A, x, b, out, omega, st);
    else k_level_op<T, Mode, 0><<<g, kThreads, 0, s>>>(A, x, b, out, omega, st);
    count_launch();
}

template <class TOut>
void launch_residual64(const StencilDev<double>& A, const double* x, const double* b, const double* dinv, TOut* bhat,
                       double* partials, const MGState* st, int gated, cudaStream_t s) {
    if (A.ns == 5) k_residual64<TOut, 5><<<kNormBlocks, kThreads, 0, s>>>(A, x, b, dinv, bhat, partials, st, gated);
    else if (A.ns == 7) k_residual64<TOut, 7><<<kNormBlocks, kThreads, 0, s>>>(A, x, b, dinv, bhat, partials, st, gated);
    else if (A.ns == 9) k_residual64<TOut, 9><<<kNormBlocks, kThreads, 0, s>>>(A, x, b, dinv, bhat, partials, st, gated);
    else if (A.ns == 27) k_residual64<TOut, 27><<<kNormBlocks, kThreads, 0, s>>>(A, x, b, dinv, bhat, partials, st, gated);
    else k_residual64<TOut, 0><<<kNormBlocks, kThreads, 0, s>>>(A, x, b, dinv, bhat, partials, st, gated);
    count_launch();
}

template <class T>
struct Level {
    long long n = 0;
    DevStencil<T> op;
    DevBuf<T> dinv;
    DevBuf<T> bufA, bufB, b;   // x ping-pong pair and right-hand side
    XferDev<T> xfer{};         // to the next coarser level
    DevAxis<T> axes[3];
};

}  // namespace mgdetail

using namespace mgdetail;

// ------------------------------------------------------------------------
struct SolverBase {
    uint32_t magic = kSolverMagic;
    int precision = 32;   // 32: mixed refinement, 64: FP64 V-cycles
    // options (defaults of sycl_multigrid32f_gpu.cpp:28-38)
    int I = 0, J = 0, K = 0;
    int depth = 3, pre_relax = 2, post_relax = 1, max_cycles = 10, correction_interval = 4;
    int max_coarse = 8192;
    std::array<int, 3> periodic{0, 0, 0};   // wrap-around transfers per axis (option periodic_I/J/K)
    double tol = 0.0;
    int null_space = 0;                     // option `null_space 0|1` (read by set_matrix)
    bool ns_built = false;                  // the hierarchy was built for a singular operator
    int use_graph = 1;                      // option `graph 0|1`: replay the solve as one CUDA graph
    int use_tma = 1;                        // option `tma 0|1`: TMA-staged sweeps on large levels
    long long tma_min_rows = kTmaMinRows;   // option `tma_min_rows`: smallest level (rows) swept that way
    unsigned long long n_row = 0;
    bool ready = false;
    cudaStream_t own_stream = nullptr;
    // The solve's launch sequence depends only on the options, the operator,
    // the sources and the (b, x) pointers: it is captured once into a CUDA
    // graph and replayed while none of them changes (`version` counts the
    // changes of the first three).
    unsigned long long version = 0;
    struct {
        cudaGraphExec_t exec = nullptr;
        const double* b = nullptr;
        const double* x = nullptr;
        unsigned long long version = 0;
        unsigned long long kernels = 0;
    } graph;
    // sources (host copies kept, device copies uploaded at set time)
    std::vector<unsigned long long> rep_idx, add_idx;
    std::vector<double> rep_val, add_val;
    DevBuf<unsigned long long> d_rep_idx, d_add_idx;
    DevBuf<double> d_rep_val, d_add_val;
    // FP64 fine operator for the residual
    DevStencil<double> a0;
    DevBuf<double> dinv0;
    DevBuf<double> partials;
    DevBuf<MGState> state;
    Hierarchy host;   // kept for introspection
    int levels = 0;
    unsigned long long coarse_rows = 0;

    virtual int tma_level_vectors() const { return 0; }   // level vectors swept by the TMA-staged kernel so far
    virtual ~SolverBase() {
        drop_graph();
        if (aux_stream) cudaStreamDestroy(aux_stream);
        if (own_stream) cudaStreamDestroy(own_stream);
    }
    void drop_graph() {
        if (graph.exec) cudaGraphExecDestroy(graph.exec);
        graph.exec = nullptr;
    }
    cudaStream_t aux_stream = nullptr;      // captures the body of a conditional loop
    unsigned long long loop_kernels = 0;    // kernels captured into loop bodies (counted on the device)
    virtual void build_device(cudaStream_t s) = 0;
    virtual void enqueue_solve(double* b, double* x, cudaStream_t s) = 0;
};

namespace {

template <class T>
struct Solver : SolverBase {
    std::vector<std::unique_ptr<Level<T>>> lv;
    DevBuf<double> coarse_inv;   // FP64 in both backends (see k_dense_mv)
    DevBuf<double> x64;   // FP64 level-0 iterate for the FP64 backend
    void build_device(cudaStream_t s) override {
        tmaps.e.clear();
        a0.upload(host.a0, s);
        dinv0.upload(host.dinv[0].data(), host.dinv[0].size(), s);
        partials.alloc(kNormBlocks);
        state.alloc(1);
        lv.clear();
        for (int l = 0; l <= host.L; ++l) {
            auto L = std::make_unique<Level<T>>();
            L->n = (long long)host.dims[l][0] * host.dims[l][1] * host.dims[l][2];
            if (l < host.L) L->op.upload(host.ahat[l], s);
            std::vector<T> d(host.dinv[l].begin(), host.dinv[l].end());
            L->dinv.upload(d.data(), d.size(), s);
            // +16 elements: the TMA-staged sweep's 16-byte-aligned copies may read past a vector's last element
            L->bufA.alloc(L->n + 16);
            L->bufB.alloc(L->n + 16);
            L->b.alloc(L->n + 16);
            if (l < host.L) {
                for (int a = 0; a < 3; ++a) L->axes[a].upload(host.xfer[l][a], s, L->xfer.ax[a]);
                const AxisDev<T>* ax = L->xfer.ax;
                L->xfer.divc12 = make_fastdiv((unsigned)(ax[1].nc * ax[2].nc));
                L->xfer.divc2 = make_fastdiv((unsigned)ax[2].nc);
                L->xfer.divf12 = make_fastdiv((unsigned)(ax[1].nf * ax[2].nf));
                L->xfer.divf2 = make_fastdiv((unsigned)ax[2].nf);
            }
            lv.push_back(std::move(L));
        }
        coarse_inv.upload(host.coarse_inv.data(), host.coarse_inv.size(), s);
        if (precision == 64) x64.alloc(n_row + 16);
        cuda_check(cudaStreamSynchronize(s), "build_device");
        levels = host.L + 1;
        coarse_rows = (unsigned long long)lv.back()->n;
    }

    // the stall word of the TMA-staged sweeps, or null when option `tma` is off
    int* tma_stall() { return use_tma ? &state.p->stall : nullptr; }
    TmapCache tmaps;   // tensor maps of the level vectors (rebuilt with the hierarchy)
    int tma_level_vectors() const override { return (int)tmaps.e.size(); }

    // Enqueue `cycles` V(pre,post) cycles on level-0 (x0 in/out, b0 = scaled rhs).
    // `x_is_zero`: the level-0 iterate starts at zero (first sweep simplified).
    // Returns the buffer holding the final level-0 iterate.
    T* enqueue_vcycles(T* x0, T* other0, T* b0, int cycles, bool x_is_zero, cudaStream_t s, bool gated = true) {
        const MGState* st = gated ? state.p : nullptr;
        const T omega = T(2.0 / 3);
        const int L = host.L;
        std::vector<T*> xcur(L + 1), xoth(L + 1), bl(L + 1);
        xcur[0] = x0;
        xoth[0] = other0;
        bl[0] = b0;
        for (int l = 1; l <= L; ++l) {
            xcur[l] = lv[l]->bufA.p;
            xoth[l] = lv[l]->bufB.p;
            bl[l] = lv[l]->b.p;
        }
        std::vector<bool> zero(L + 1, false);
        zero[0] = x_is_zero;
        auto smooth = [&](int l) {
            Level<T>& V = *lv[l];
            if (zero[l]) {
                launch_level_op<T, kSmoothFromZero>(V.op.view, xcur[l], bl[l], xoth[l], omega, st, s);
                zero[l] = false;
            } else {
                launch_level_op<T, kSmooth>(V.op.view, xcur[l], bl[l], xoth[l], omega, st, s, tma_stall(), &tmaps, tma_min_rows);
            }
            std::swap(xcur[l], xoth[l]);
        };
        for (int c = 0; c < cycles; ++c) {
            for (int l = 0; l < L; ++l) {
                for (int k = 0; k < pre_relax; ++k) smooth(l);
                Level<T>& V = *lv[l];
                if (zero[l]) {
                    // x is zero: residual = b; restrict b directly
                    { k_restrict<T><<<grid_for(lv[l + 1]->n), kThreads, 0, s>>>(V.xfer, bl[l], bl[l + 1], xcur[l + 1],
                                                                             lv[l + 1]->dinv.p, st); count_launch(); }
                } else {
                    launch_level_op<T, kResidual>(V.op.view, xcur[l], bl[l], xoth[l], omega, st, s, tma_stall(), &tmaps, tma_min_rows);
                    { k_restrict<T><<<grid_for(lv[l + 1]->n), kThreads, 0, s>>>(V.xfer, xoth[l], bl[l + 1],
                                                                             xcur[l + 1], lv[l + 1]->dinv.p, st); count_launch(); }
                }
                zero[l + 1] = true;
            }
            {
                const int n = (int)lv[L]->n;
                { k_dense_mv<T><<<grid_for((long long)n * 32), kThreads, 0, s>>>(coarse_inv.p, bl[L], xcur[L], n, st); count_launch(); }
                zero[L] = false;
            }
            for (int l = L - 1; l >= 0; --l) {
                if (zero[l]) {
                    // only possible with pre_relax == 0 on a level that started at zero:
                    // x_l was never written; the restriction kernel did not zero it.
                    cuda_check(cudaMemsetAsync(xcur[l], 0, sizeof(T) * lv[l]->n, s), "memset");
                    zero[l] = false;
                }
                if (lv[l]->xfer.ax[2].nf % 4 == 0) {
                    k_prolong_add_row4<T><<<grid_for(lv[l]->n / 4), kThreads, 0, s>>>(lv[l]->xfer, xcur[l + 1],
                                                                                       xcur[l], st);
                } else {
                    k_prolong_add<T><<<grid_for((lv[l]->n + kProlongPer - 1) / kProlongPer), kThreads, 0, s>>>(
                        lv[l]->xfer, xcur[l + 1], xcur[l], st);
                }
                count_launch();
                for (int k = 0; k < post_relax; ++k) smooth(l);
            }
        }
        cuda_check(cudaGetLastError(), "multigrid kernel launch");
        return xcur[0];
    }

    // [residual, check] then WHILE(check says continue) { V-cycles, correct,
    // residual, check } (sycl_multigrid32f_gpu.cpp:137-157 with the loop kept
    // on the device).  The body's check adds the body's kernel count to the
    // mapped launch counter each time the body runs.
    void enqueue_refinement_loop(double* b, double* x, cudaStream_t s) {
        MGState* st = state.p;
        Level<T>& F = *lv[0];
        const long long n = (long long)n_row;
        const int ci = correction_interval;
        if (!aux_stream) throw Error(PSUM_ERR_INTERNAL, "multigrid: loop stream missing");
        unsigned long long* counter = device_launch_counter();   // created by set_matrix
        cudaStreamCaptureStatus cs;
        cudaGraph_t g = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t nd = 0;
        cuda_check(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd), "cudaStreamGetCaptureInfo");
        cudaGraphConditionalHandle h;
        cuda_check(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault), "conditional handle");
        launch_residual64<T>(a0.view, x, b, dinv0.p, F.b.p, partials.p, st, 1, s);
        { k_check_loop<<<1, 32, 0, s>>>(partials.p, kNormBlocks, st, 0, max_cycles, tol, h, 0ull, counter); count_launch(); }
        cuda_check(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd), "cudaStreamGetCaptureInfo");
        cudaGraphNodeParams np{};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = h;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t loop;
        cuda_check(cudaGraphAddNode(&loop, g, deps, nd, &np), "add conditional node");
        cudaGraph_t body = np.conditional.phGraph_out[0];
        cuda_check(cudaStreamUpdateCaptureDependencies(s, &loop, 1, cudaStreamSetCaptureDependencies),
                   "update capture dependencies");
        cuda_check(cudaStreamBeginCaptureToGraph(aux_stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal),
                   "capture loop body");
        const unsigned long long k0 = thread_launches();
        unsigned long long body_kernels = 0;
        try {
            // inside the loop the solve is never done: the kernels skip the flag
            T* e = enqueue_vcycles(F.bufA.p, F.bufB.p, F.b.p, ci, /*x_is_zero=*/true, aux_stream, /*gated=*/false);
            { k_correct<T><<<grid_for(n), kThreads, 0, aux_stream>>>(x, e, n, nullptr); count_launch(); }
            launch_residual64<T>(a0.view, x, b, dinv0.p, F.b.p, partials.p, nullptr, 0, aux_stream);
            body_kernels = thread_launches() - k0 + 1;
            { k_check_loop<<<1, 32, 0, aux_stream>>>(partials.p, kNormBlocks, st, ci, max_cycles, tol, h,
                                                     body_kernels, counter); count_launch(); }
            cuda_check(cudaGetLastError(), "loop body launch");
        } catch (...) {
            cudaGraph_t tmp = nullptr;
            cudaStreamEndCapture(aux_stream, &tmp);
            uncount_launches(thread_launches() - k0);
            throw;
        }
        cuda_check(cudaStreamEndCapture(aux_stream, &body), "end loop body capture");
        uncount_launches(body_kernels);   // counted by the body's check, once per iteration run
        loop_kernels += body_kernels;
    }

    void enqueue_sources(double* b, cudaStream_t s) {
        const long long na = (long long)add_idx.size(), nr = (long long)rep_idx.size();
        if (na > 0) { k_addback<<<grid_for(na), kThreads, 0, s>>>(b, d_add_idx.p, d_add_val.p, na); count_launch(); }
        if (nr > 0) { k_replace<<<grid_for(nr), kThreads, 0, s>>>(b, d_rep_idx.p, d_rep_val.p, nr); count_launch(); }
    }

    // v -= mean(v) (two launches; fixed reduction order)
    void enqueue_project(double* v, cudaStream_t s) {
        const long long n = (long long)n_row;
        { k_sum<<<kNormBlocks, kThreads, 0, s>>>(v, n, partials.p); count_launch(); }
        { k_sub_mean<<<kNormBlocks, kThreads, 0, s>>>(v, n, partials.p, kNormBlocks); count_launch(); }
    }

    void enqueue_solve(double* b, double* x, cudaStream_t s) override {
        const long long n = (long long)n_row;
        MGState* st = state.p;
        if (ns_built && !rep_idx.empty())
            throw std::invalid_argument("multigrid: null_space 1 with fixed (replaced) nodes");
        enqueue_sources(b, s);
        // singular operator: solve for the consistent part of b (the mean-zero
        // projection; b is the solve's scratch like PSuM's source vector)
        if (ns_built) enqueue_project(b, s);
        { k_norm2<<<kNormBlocks, kThreads, 0, s>>>(b, n, partials.p); count_launch(); }
        { k_check<<<1, 32, 0, s>>>(partials.p, kNormBlocks, st, 0, tol, 0, 0); count_launch(); }
        Level<T>& F = *lv[0];
        int cycles_done = 0, refinements = 0;
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        cuda_check(cudaStreamIsCapturing(s, &cs), "cudaStreamIsCapturing");
        if (precision == 32 && cs == cudaStreamCaptureStatusActive && tol > 0 && max_cycles > 0 &&
            max_cycles % correction_interval == 0) {
            // captured into a graph: the refinements run as a conditional loop
            // that ends on the device once the residual test passes, so no
            // kernel of the cycles after convergence is launched
            enqueue_refinement_loop(b, x, s);
            cycles_done = max_cycles;
            refinements = max_cycles / correction_interval;
        } else if (precision == 32) {
            // FP64 refinement around FP32 V-cycles (sycl_multigrid32f_gpu.cpp:137-157)
            while (cycles_done < max_cycles) {
                const int batch = std::min(correction_interval, max_cycles - cycles_done);
                launch_residual64<T>(a0.view, x, b, dinv0.p, F.b.p, partials.p, st, 1, s);
                { k_check<<<1, 32, 0, s>>>(partials.p, kNormBlocks, st, 1, tol, cycles_done, refinements); count_launch(); }
                T* e = enqueue_vcycles(F.bufA.p, F.bufB.p, F.b.p, batch, /*x_is_zero=*/true, s);
                { k_correct<T><<<grid_for(n), kThreads, 0, s>>>(x, e, n, st); count_launch(); }
                cycles_done += batch;
                ++refinements;
            }
        } else {
            cuda_check(cudaMemcpyAsync(x64.p, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, s), "copy x");
            { k_scale<T><<<grid_for(n), kThreads, 0, s>>>(b, dinv0.p, F.b.p, n); count_launch(); }
            double* xc = x64.p;
            double* xo = reinterpret_cast<double*>(F.bufB.p);
            while (cycles_done < max_cycles) {
                const int batch = tol > 0 ? std::min(correction_interval, max_cycles - cycles_done) : max_cycles;
                if (tol > 0) {
                    launch_residual64<double>(a0.view, xc, b, nullptr, (double*)nullptr, partials.p, st, 1, s);
                    { k_check<<<1, 32, 0, s>>>(partials.p, kNormBlocks, st, 1, tol, cycles_done, refinements); count_launch(); }
                }
                T* r = enqueue_vcycles(reinterpret_cast<T*>(xc), reinterpret_cast<T*>(xo), F.b.p, batch, false, s);
                if ((double*)r != xc) std::swap(xc, xo);
                cycles_done += batch;
            }
            cuda_check(cudaMemcpyAsync(x, xc, sizeof(double) * n, cudaMemcpyDeviceToDevice, s), "copy x");
        }
        if (ns_built) enqueue_project(x, s);   // the mean-zero representative
        launch_residual64<double>(a0.view, x, b, nullptr, (double*)nullptr, partials.p, st, 0, s);
        { k_check<<<1, 32, 0, s>>>(partials.p, kNormBlocks, st, 2, tol, cycles_done, refinements); count_launch(); }
        cuda_check(cudaGetLastError(), "solve launch");
    }
};

int parse_int(std::istringstream& iss, const std::string& key) {
    int v;
    if (!(iss >> v)) throw std::invalid_argument("set_options: option '" + key + "' needs an integer value");
    return v;
}

}  // namespace

SolverBase* solver_from_handle(void* h) {
    SolverBase* s = static_cast<SolverBase*>(h);
    if (!s || s->magic != kSolverMagic) throw Error(PSUM_ERR_INVALID_ARGUMENT, "not a handle of this library");
    return s;
}

cudaStream_t solver_stream(SolverBase* s) { return s->own_stream; }

SolverBase* create_solver(int precision) {
    SolverBase* s = precision == 64 ? static_cast<SolverBase*>(new Solver<double>())
                                    : static_cast<SolverBase*>(new Solver<float>());
    s->precision = precision;
    return s;   // the CUDA stream is created on first device use (set_matrix)
}

static void ensure_stream(SolverBase* s) {
    if (!s->own_stream)
        cuda_check(cudaStreamCreateWithFlags(&s->own_stream, cudaStreamNonBlocking), "cudaStreamCreate");
}

void solver_set_options(SolverBase* s, const char* options) {
    if (!options) throw std::invalid_argument("set_options: null option string");
    std::istringstream iss(options);
    std::string key;
    bool k_provided = false;
    while (iss >> key) {
        if (key == "I") s->I = parse_int(iss, key);
        else if (key == "J") s->J = parse_int(iss, key);
        else if (key == "K") {
            s->K = parse_int(iss, key);
            k_provided = true;
        } else if (key == "depth") s->depth = parse_int(iss, key);
        else if (key == "pre_relax") s->pre_relax = parse_int(iss, key);
        else if (key == "post_relax") s->post_relax = parse_int(iss, key);
        else if (key == "max_cycles") s->max_cycles = parse_int(iss, key);
        else if (key == "max_coarse") s->max_coarse = parse_int(iss, key);
        else if (key == "periodic_I") s->periodic[0] = parse_int(iss, key) != 0;
        else if (key == "periodic_J") s->periodic[1] = parse_int(iss, key) != 0;
        else if (key == "periodic_K") s->periodic[2] = parse_int(iss, key) != 0;
        else if (key == "graph") s->use_graph = parse_int(iss, key) != 0;
        else if (key == "tma") s->use_tma = parse_int(iss, key) != 0;
        else if (key == "tma_min_rows") {
            long long v = 0;
            if (!(iss >> v) || v < 1) throw std::invalid_argument("tma_min_rows must be positive");
            s->tma_min_rows = v;
        }
        else if (key == "null_space") s->null_space = parse_int(iss, key) != 0;
        else if (key == "correction_interval") {
            int v = 0;
            if (!(iss >> v) || v < 1) throw std::invalid_argument("correction_interval must be positive");
            s->correction_interval = v;
        } else if (key == "tol") {
            double v;
            if (!(iss >> v) || !(v >= 0)) throw std::invalid_argument("tol must be a non-negative number");
            s->tol = v;
        } else if (key.rfind("num_conv", 0) == 0 || key == "num_threads") {
            parse_int(iss, key);   // PSuM tuning keys: accepted and ignored
        }
        // other unknown keys are skipped like PSuM's parser does
    }
    if (!k_provided) s->K = 1;
    if (s->pre_relax < 0 || s->post_relax < 0 || s->max_cycles < 0 || s->depth < 1)
        throw std::invalid_argument("set_options: negative relax/cycle counts or depth < 1");
    s->version++;
}

void solver_set_matrix(SolverBase* s, unsigned long long n_row, unsigned long long n_col, unsigned long long nnz,
                       const unsigned long long* rows, const unsigned long long* cols, const double* vals) {
    if (n_row != n_col) throw std::invalid_argument("set_matrix: matrix must be square");
    HostCSR A = csr_from_coo((long long)n_row, (long long)n_col, (long long)nnz, rows, cols, vals);
    s->host = build_hierarchy(A, s->I, s->J, s->K, s->depth, s->max_coarse, s->periodic, s->null_space != 0);
    s->ns_built = s->null_space != 0;
    s->n_row = n_row;
    ensure_stream(s);
    // created here, outside any stream capture: the stream that captures the
    // body of the conditional refinement loop, and the mapped launch counter
    if (!s->aux_stream) cuda_check(cudaStreamCreateWithFlags(&s->aux_stream, cudaStreamNonBlocking), "cudaStreamCreate");
    device_launch_counter();
    s->version++;
    s->drop_graph();
    s->build_device(s->own_stream);
    s->ready = true;
}

static void upload_sources(SolverBase* s) {
    ensure_stream(s);
    s->d_rep_idx.upload(s->rep_idx.data(), s->rep_idx.size(), s->own_stream);
    s->d_rep_val.upload(s->rep_val.data(), s->rep_val.size(), s->own_stream);
    s->d_add_idx.upload(s->add_idx.data(), s->add_idx.size(), s->own_stream);
    s->d_add_val.upload(s->add_val.data(), s->add_val.size(), s->own_stream);
    cuda_check(cudaStreamSynchronize(s->own_stream), "upload sources");
    s->version++;
}

// Graph capture needs a stream that is not the legacy/per-thread default
// stream and is not already being captured by the caller (then the caller's
// capture records the launches directly).
static bool capturable(cudaStream_t st) {
    if (st == nullptr || st == cudaStreamLegacy || st == cudaStreamPerThread) return false;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cuda_check(cudaStreamIsCapturing(st, &cs), "cudaStreamIsCapturing");
    return cs == cudaStreamCaptureStatusNone;
}

static void capture_solve(SolverBase* s, double* b, double* x, cudaStream_t st) {
    s->drop_graph();
    const unsigned long long k0 = thread_launches();
    s->loop_kernels = 0;
    cuda_check(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    cudaGraph_t g = nullptr;
    try {
        s->enqueue_solve(b, x, st);
    } catch (...) {
        cudaStreamEndCapture(st, &g);
        if (g) cudaGraphDestroy(g);
        uncount_launches(thread_launches() - k0 - s->loop_kernels);
        throw;
    }
    cuda_check(cudaStreamEndCapture(st, &g), "cudaStreamEndCapture");
    const unsigned long long kernels = thread_launches() - k0 - s->loop_kernels;   // outside loop bodies
    uncount_launches(kernels);   // counted again at every replay
    const cudaError_t e = cudaGraphInstantiate(&s->graph.exec, g, 0);
    cudaGraphDestroy(g);
    cuda_check(e, "cudaGraphInstantiate");
    s->graph.b = b;
    s->graph.x = x;
    s->graph.version = s->version;
    s->graph.kernels = kernels;
}

void solver_set_source(SolverBase* s, bool replace, unsigned long long n, const unsigned long long* idx,
                       const double* v) {
    if (n > 0 && (!idx || !v)) throw std::invalid_argument("set_source: null array");
    if (s->ready)
        for (unsigned long long i = 0; i < n; ++i)
            if (idx[i] >= s->n_row) throw std::invalid_argument("set_source: index out of range");
    if (replace) {
        s->rep_idx.assign(idx, idx + n);
        s->rep_val.assign(v, v + n);
    } else {
        s->add_idx.assign(idx, idx + n);
        s->add_val.assign(v, v + n);
    }
    upload_sources(s);
}

void solver_solve_async(SolverBase* s, double* b, double* x, cudaStream_t stream) {
    if (!s->ready) throw Error(PSUM_ERR_NOT_READY, "solve called before set_matrix");
    if (!b || !x) throw std::invalid_argument("solve: null device pointer");
    for (auto i : s->rep_idx)
        if (i >= s->n_row) throw std::invalid_argument("set_source_replace: index out of range");
    for (auto i : s->add_idx)
        if (i >= s->n_row) throw std::invalid_argument("set_source_addback: index out of range");
    cudaStream_t st = stream ? stream : s->own_stream;
    if (s->use_graph && capturable(st)) {
        if (!(s->graph.exec && s->graph.b == b && s->graph.x == x && s->graph.version == s->version))
            capture_solve(s, b, x, st);
        cuda_check(cudaGraphLaunch(s->graph.exec, st), "cudaGraphLaunch");
        add_launches(s->graph.kernels);
        return;
    }
    s->enqueue_solve(b, x, st);
}

MGState solver_read_state(SolverBase* s, cudaStream_t stream) {
    MGState st{};
    cuda_check(cudaMemcpyAsync(&st, s->state.p, sizeof(MGState), cudaMemcpyDeviceToHost,
                               stream ? stream : s->own_stream),
               "read state");
    cuda_check(cudaStreamSynchronize(stream ? stream : s->own_stream), "read state sync");
    return st;
}

void solver_destroy(SolverBase* s) {
    if (s->own_stream) cudaStreamSynchronize(s->own_stream);
    s->magic = 0;
    delete s;
}

}  // namespace psum_b200

// ===================================================================== ABI ==
using namespace psum_b200;

namespace {

template <int P>
psum_field_solver_handle ft_init() {
    return create_solver(P);
}

void ft_set_matrix(psum_field_solver_handle h, unsigned long long n_row, unsigned long long n_col,
                   unsigned long long nnz, unsigned long long* rows, unsigned long long* cols, double* vals) {
    solver_set_matrix(solver_from_handle(h), n_row, n_col, nnz, rows, cols, vals);
}

void ft_solve(psum_field_solver_handle h, double* b, double* x) {
    SolverBase* s = solver_from_handle(h);
    solver_solve_async(s, b, x, s->own_stream);
    cuda_check(cudaStreamSynchronize(s->own_stream), "solve sync");
    MGState st = solver_read_state(s, s->own_stream);
    if (st.status == PSUM_ERR_DIVERGED) throw Error(PSUM_ERR_DIVERGED, "multigrid: residual diverged");
    if (st.stall) throw Error(PSUM_ERR_INTERNAL, "multigrid: a TMA-staged sweep stopped waiting for its copies");
}

void ft_set_options(psum_field_solver_handle h, const char* o) { solver_set_options(solver_from_handle(h), o); }

void ft_set_source_replace(psum_field_solver_handle h, unsigned long long n, unsigned long long* idx, double* v) {
    solver_set_source(solver_from_handle(h), true, n, idx, v);
}

void ft_set_source_addback(psum_field_solver_handle h, unsigned long long n, unsigned long long* idx, double* v) {
    solver_set_source(solver_from_handle(h), false, n, idx, v);
}

void ft_free(psum_field_solver_handle h) {
    if (h) solver_destroy(solver_from_handle(h));
}

// Static registration, as the reference backends do (sycl_multigrid32f_gpu.cpp:255-266).
int register_backends() {
    func_table t32{ft_init<32>, ft_set_matrix, ft_solve, ft_set_options, ft_set_source_replace, ft_set_source_addback,
                   ft_free};
    func_table t64{ft_init<64>, ft_set_matrix, ft_solve, ft_set_options, ft_set_source_replace, ft_set_source_addback,
                   ft_free};
    register_solver("cuda_multigrid32f_gpu", t32);
    register_solver("cuda_multigrid64_gpu", t64);
    return 0;
}
const int g_registered = register_backends();

}  // namespace

extern "C" {

EXPORT int psum_mg_create(const char* kind, psum_field_solver_handle* out) {
    return guarded([&] {
        if (!out) throw std::invalid_argument("psum_mg_create: null output");
        *out = nullptr;
        func_table t = get_solver_funcs(kind ? kind : "");
        if (!t.init) throw std::invalid_argument(std::string("unknown solver backend: ") + (kind ? kind : "(null)"));
        *out = t.init();
        if (!*out) throw Error(PSUM_ERR_INTERNAL, "failed to create solver.");
    });
}

EXPORT int psum_mg_set_options(psum_field_solver_handle h, const char* options) {
    return guarded([&] { solver_set_options(solver_from_handle(h), options); });
}

EXPORT int psum_mg_set_matrix(psum_field_solver_handle h, unsigned long long n_row, unsigned long long n_col,
                              unsigned long long nnz, const unsigned long long* rows, const unsigned long long* cols,
                              const double* vals) {
    return guarded([&] { solver_set_matrix(solver_from_handle(h), n_row, n_col, nnz, rows, cols, vals); });
}

EXPORT int psum_mg_set_source_replace(psum_field_solver_handle h, unsigned long long n, const unsigned long long* idx,
                                      const double* values) {
    return guarded([&] { solver_set_source(solver_from_handle(h), true, n, idx, values); });
}

EXPORT int psum_mg_set_source_addback(psum_field_solver_handle h, unsigned long long n, const unsigned long long* idx,
                                      const double* values) {
    return guarded([&] { solver_set_source(solver_from_handle(h), false, n, idx, values); });
}

EXPORT int psum_mg_solve(psum_field_solver_handle h, double* b_dev, double* x_dev) {
    int status = PSUM_OK;
    int rc = guarded([&] {
        SolverBase* s = solver_from_handle(h);
        solver_solve_async(s, b_dev, x_dev, s->own_stream);
        MGState st = solver_read_state(s, s->own_stream);
        status = st.stall ? PSUM_ERR_INTERNAL : st.status;
    });
    if (rc != PSUM_OK) return rc;
    if (status == PSUM_ERR_NOT_CONVERGED) set_last_error("multigrid: tol not reached within max_cycles");
    if (status == PSUM_ERR_DIVERGED) set_last_error("multigrid: residual diverged");
    if (status == PSUM_ERR_INTERNAL) set_last_error("multigrid: a TMA-staged sweep stopped waiting for its copies");
    return status;
}

EXPORT int psum_mg_solve_async(psum_field_solver_handle h, double* b_dev, double* x_dev, void* stream) {
    return guarded([&] {
        SolverBase* s = solver_from_handle(h);
        solver_solve_async(s, b_dev, x_dev, static_cast<cudaStream_t>(stream));
    });
}

EXPORT int psum_mg_last_stats(psum_field_solver_handle h, int* cycles, int* refinements, double* rel_residual,
                              double* initial_rel_residual) {
    return guarded([&] {
        SolverBase* s = solver_from_handle(h);
        if (!s->ready) throw Error(PSUM_ERR_NOT_READY, "no solve has run");
        cuda_check(cudaDeviceSynchronize(), "stats sync");
        MGState st = solver_read_state(s, s->own_stream);
        const double bn = st.bnorm2 > 0 ? std::sqrt(st.bnorm2) : 1.0;
        if (cycles) *cycles = st.cycles;
        if (refinements) *refinements = st.refinements;
        if (rel_residual) *rel_residual = std::sqrt(std::max(0.0, st.rnorm2_last)) / bn;
        if (initial_rel_residual) *initial_rel_residual = std::sqrt(std::max(0.0, st.rnorm2_first)) / bn;
    });
}

EXPORT int psum_mg_hierarchy_info(psum_field_solver_handle h, int* levels, unsigned long long* coarse_rows,
                                  unsigned long long* exception_rows_level0) {
    return guarded([&] {
        SolverBase* s = solver_from_handle(h);
        if (!s->ready) throw Error(PSUM_ERR_NOT_READY, "set_matrix has not been called");
        if (levels) *levels = s->levels;
        if (coarse_rows) *coarse_rows = s->coarse_rows;
        if (exception_rows_level0) *exception_rows_level0 = s->host.ahat[0].exc_rows.size();
    });
}

EXPORT int psum_mg_tma_sweeps(psum_field_solver_handle h, int* level_vectors) {
    return guarded([&] {
        SolverBase* s = solver_from_handle(h);
        if (level_vectors) *level_vectors = s->tma_level_vectors();
    });
}

EXPORT int psum_mg_destroy(psum_field_solver_handle h) {
    return guarded([&] {
        if (h) solver_destroy(solver_from_handle(h));
    });
}

}  // extern "C"
