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
    psum_b200::DevBuf<unsigned> cls_count;    // per (cell, move class) counts, then group offsets, of the fused sorted step
    psum_b200::DevBuf<unsigned> cls_first;    // first cell owned by each block of the fused sorted step
    psum_b200::DevBuf<unsigned> newcount;     // per new cell counts (n_cells + 1)
    psum_b200::DevBuf<unsigned> scan_tmp1, scan_tmp2;
    psum_b200::DevBuf<int> far_flag;          // per species: a particle moved more than one cell on an axis
    int sort_interval = 1;
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
        drop_events();
        if (own_stream) cudaStreamDestroy(own_stream);
    }
};

namespace psum_b200 {
// pic.cu: handle and index checks, and the key fill of a sorted mixed state
psum_pic_ctx* ctx_check(psum_pic_ctx* c);
Species& species_at(psum_pic_ctx* c, int s);
void ensure_keys(psum_pic_ctx* c, Species& sp);
}  // namespace psum_b200
