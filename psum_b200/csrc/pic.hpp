// pic.hpp -- host-side particle context of the B200 PIC step (internal).
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <vector>

#include "common.hpp"
#include "pic_common.cuh"

namespace psum_b200 {

constexpr uint32_t kPicMagic = 0x50494332u;   // "PIC2"

struct Species {
    double q = 0, m = 1, w = 1;
    long long cap = 0;
    long long n = 0;        // host upper bound of stored particles (exact after load / count)
    int dep_shift = 32;     // fixed-point exponent of the charge accumulator
    int cur = 0;            // current buffer of the double-buffered state
    // mixed precision state
    DevBuf<int> key[2];
    DevBuf<float> off[3][2];
    DevBuf<float> vel[3][2];
    // FP64 state
    DevBuf<double> pos64[3][2];
    DevBuf<double> vel64[3][2];
    DevBuf<unsigned long long> acc;   // deposit accumulator, one int64 per node
    // cell offsets of the sorted state (n_cells + 1 entries, double buffered)
    DevBuf<unsigned> starts[2];
    int starts_cur = 0;
    bool sorted = false;              // state sorted by cell and starts valid
    bool keys_stale = false;          // sorted mixed state whose keys follow from starts but are not written
    // fused sorted step: per (class, cell) counts then group offsets, block
    // table, new per-cell counts and scan scratch (per species, so that the
    // second passes of all species run after all first passes)
    DevBuf<unsigned> cls_count, cls_first, cls_first2, newcount, scan_tmp1, scan_tmp2;
};

struct SortScratch {
    DevBuf<unsigned> keyA, keyB;
    DevBuf<int> idxA, idxB;
    DevBuf<unsigned> hist, hist_scan, block_sums, block_sums2;
    long long cap = 0;
};

}  // namespace psum_b200

struct psum_pic_ctx {
    uint32_t magic = psum_b200::kPicMagic;
    psum_b200::GridView g{};
    psum_pic_grid_desc desc{};           // the grid as created (for the B-spline entry points)
    int precision = 0;
    cudaStream_t stream = nullptr;       // active stream
    cudaStream_t own_stream = nullptr;
    std::vector<std::unique_ptr<psum_b200::Species>> sp;
    psum_b200::DevBuf<float> edges;      // mixed: per node (dim components, stride 2 or 4)
    psum_b200::DevBuf<unsigned long long> losses;    // [species][3][2]
    psum_b200::DevBuf<unsigned> err;
    psum_b200::DevBuf<long long> count;  // device stored count per species
    psum_b200::DevBuf<double> partials;
    psum_b200::DevBuf<long long> ipartials;
    psum_b200::SortScratch sort;
    psum_b200::DevBuf<int> far_flag;          // per species: a particle moved more than one cell on an axis
    // The second passes of a fused step run on `side` after the first passes
    // (event ev_pass1) and overlap what the caller enqueues next on the
    // context stream (the next step's charge density and Poisson solve,
    // which need only the first passes' deposit).  `pending` until joined:
    // the context stream then waits for ev_pass2 and the host finishes the
    // step (buffer swap, or the general path of a species whose particle
    // moved more than one cell, with the step's dt, pusher and B kept here).
    cudaStream_t side = nullptr;              // least priority
    cudaEvent_t ev_pass1 = nullptr, ev_pass2 = nullptr;
    cudaEvent_t ev_sp[8] = {};                // per species: its first pass, offsets and scan are done
    // A step's charge density and solve run on `prio` (greatest priority),
    // ordered after the context stream (ev_in) and before it (ev_out), so
    // that their blocks are scheduled ahead of a pending second pass.
    cudaStream_t prio = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    int* far_host = nullptr;                  // pinned copy of far_flag
    bool pending = false;
    double pend_dt = 0;
    int pend_pusher = 0;
    bool pend_has_B = false;
    double pend_B[3] = {0, 0, 0};
    // After a fused step in which a particle moved more than one cell (its
    // species then took the in-place push and full re-sort), the next
    // fused_skip steps go straight to the general path instead of paying a
    // first pass that would be thrown away again; the skip doubles while the
    // far movers persist (up to 64 steps) and resets after a clean step.
    int fused_skip = 0;
    int fused_backoff = 1;
    int sort_interval = 1;
    bool fp64_fma = false;                    // FP64 mode: the contracted kernel build (not bit-exact)
    // option "interp_order k" (2-4): the step deposits and gathers with PSuM's B-spline weights of order k
    // (positions exported to bs_pos per species, the gathered gradient in bs_grad, deposit scratch bs_acc)
    int interp_order = 1;
    psum_b200::DevBuf<double> bs_pos[8];
    psum_b200::DevBuf<double> bs_grad;
    psum_b200::DevBuf<unsigned long long> bs_acc;
    // per-step diagnostics (option "diagnostics 1"): partial sums written by the
    // step's own kernels (field energy by k_edges, kinetic energy by the push,
    // charge by k_rho), reduced by k_diag_finish into diag_out
    // The partial sums are double buffered by step parity: a fused step's sums
    // are reduced when it is joined, after the next step's density has begun.
    struct DiagBufs {
        psum_b200::DevBuf<double> fe, kin;
        psum_b200::DevBuf<unsigned long long> qsum;
        psum_b200::DevBuf<double> rho_part;   // B-spline steps: per-block sums of rho - background
        psum_b200::DevBuf<double> stage;      // first-level sums of the partial arrays (k_diag_stage)
        long long rho_n = 0;
        long long fe_n = 0;
        long long kin_n[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        long long kin_off[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    };
    bool diag = false;
    bool diag_in_step = false;                // set while psum_pic_step launches its kernels
    DiagBufs dbuf[2];
    int diag_par = 0;                         // parity of the current step's buffers
    bool pend_diag = false;                   // the pending fused step's sums await their reduction
    int pend_par = 0;
    psum_b200::DevBuf<double> diag_out;
    bool diag_valid = false;
    long long steps = 0;
    bool timing = false;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> events;   // (phase, start/stop)
    void drop_events() {
        for (auto& e : events) {
            cudaEventDestroy(e.second.first);
            cudaEventDestroy(e.second.second);
        }
        events.clear();
    }
    // adjoint scratch: int64 node accumulator, its fixed-point scale, the max
    psum_b200::DevBuf<unsigned long long> adj_acc;
    psum_b200::DevBuf<double> adj_scale;
    psum_b200::DevBuf<unsigned> adj_max;
    ~psum_pic_ctx() {
        if (side) cudaStreamSynchronize(side);
        drop_events();
        if (ev_pass1) cudaEventDestroy(ev_pass1);
        if (ev_pass2) cudaEventDestroy(ev_pass2);
        for (auto e : ev_sp)
            if (e) cudaEventDestroy(e);
        if (ev_in) cudaEventDestroy(ev_in);
        if (ev_out) cudaEventDestroy(ev_out);
        if (prio) {
            cudaStreamSynchronize(prio);
            cudaStreamDestroy(prio);
        }
        if (far_host) cudaFreeHost(far_host);
        if (side) cudaStreamDestroy(side);
        if (own_stream) cudaStreamDestroy(own_stream);
    }
};

namespace psum_b200 {
// pic.cu: handle and index checks (ctx_check also joins a pending fused
// step; ctx_check_nojoin leaves it running), and the key fill of a sorted
// mixed state
psum_pic_ctx* ctx_check(psum_pic_ctx* c);
psum_pic_ctx* ctx_check_nojoin(psum_pic_ctx* c);
Species& species_at(psum_pic_ctx* c, int s);
void ensure_keys(psum_pic_ctx* c, Species& sp);
}  // namespace psum_b200
