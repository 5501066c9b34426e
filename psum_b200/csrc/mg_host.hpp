// mg_host.hpp -- host-side multigrid setup of the B200 backend.
//
// Builds, from the fine operator A given as COO through the solver ABI, the
// hierarchy multigrid_core::setup builds in PSuM
// (src/field_solver/implements/multigrid/multigrid_core.hpp:49-150):
//   Ahat_0 = D_0^-1 A,  A_{l+1} = R_l Ahat_l P_l,  Ahat_{l+1} = D_{l+1}^-1 A_{l+1},
// with PSuM's structured transfers (multigrid_utilities.hpp:55-104) and the
// dense inverse of the coarsest Ahat (sycl_inner_solver.hpp:51-71).
//
// The device layout differs from PSuM's: every level operator is stored as
//   * one constant stencil (<= 27 entries, 3-D neighbour deltas in {-1,0,1}
//     taken with periodic wrap on the level's node box), applied to every row
//     whose entries equal it exactly, plus
//   * an exception list (CSR) for the remaining rows, flagged by a bitmask,
// and the transfers are stored as their exact 1-D tensor factors
// (P = Px (x) Py (x) Pz and R = Rx (x) Ry (x) Rz), so no per-row index or
// coefficient arrays are read for the bulk of the grid.
#pragma once

#include <array>
#include <cstdint>
#include <string>
#include <vector>

namespace psum_b200 {

struct HostCSR {
    long long n_row = 0, n_col = 0;
    std::vector<long long> ptr;
    std::vector<int> col;
    std::vector<double> val;
};

// setFromTriplets semantics: duplicates summed, columns ascending per row.
HostCSR csr_from_coo(long long n_row, long long n_col, long long nnz, const unsigned long long* rows,
                     const unsigned long long* cols, const double* vals);

struct StencilOp {
    std::array<int, 3> dims{1, 1, 1};   // node box (n0, n1, n2), last fastest
    long long n = 0;
    int ns = 0;                          // number of stencil entries
    std::array<std::array<int, 3>, 27> delta{};
    std::array<double, 27> coef{};
    std::vector<int> exc_rows;           // ascending
    std::vector<int> exc_ptr;            // size exc_rows+1
    std::vector<int> exc_col;
    std::vector<double> exc_val;
    std::vector<uint32_t> mask;          // bit r%32 of word r/32 set for exception rows
    std::vector<uint32_t> mask_prefix;   // exceptions before word w
};

// 1-D factor of the structured transfer of one axis at one level.
struct Axis1D {
    int nf = 1, nc = 1;
    // prolongation: fine index -> up to 2 coarse indices
    std::vector<int> p_c0, p_c1;         // p_c1 = -1 when absent
    std::vector<double> p_w0, p_w1;
    // restriction: coarse index -> up to 3 fine indices (stride 3)
    std::vector<int> r_f;                // -1 when absent
    std::vector<double> r_w;
};

struct Hierarchy {
    int L = 0;                                   // number of transfers
    std::vector<std::array<int, 3>> dims;        // L+1 node boxes
    std::vector<StencilOp> ahat;                 // L+1 scaled operators
    std::vector<std::vector<double>> dinv;       // L+1 inverse diagonals
    std::vector<std::array<Axis1D, 3>> xfer;     // L transfer factors
    StencilOp a0;                                // unscaled fine operator (FP64 residual)
    std::vector<double> coarse_inv;              // dense row-major inverse of ahat[L]
};

// Throws std::invalid_argument / std::runtime_error with PSuM's messages.
// periodic[d] != 0 selects wrap-around transfers on axis d (an extension:
// PSuM's open-interval transfers diverge on wrapping lattices).
// null_space: A is singular with the constants as its null space (a
// periodic operator without a pinned node); the coarse inverse then solves
// the consistent coarse systems.
Hierarchy build_hierarchy(const HostCSR& A, int I, int J, int K, int depth, int max_coarse = 8192,
                          const std::array<int, 3>& periodic = {0, 0, 0}, bool null_space = false);

// Stencil + exception decomposition of one operator on a node box.
StencilOp decompose(const HostCSR& A, const std::array<int, 3>& dims);

}  // namespace psum_b200
