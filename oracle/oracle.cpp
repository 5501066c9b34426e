// oracle.cpp -- FP64 CPU restatement of PSuM's electrostatic PIC path.
//
// TEST INFRASTRUCTURE ONLY.  This library is the checker: the parity tests,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg call it to produce
// the expected results.  No product code path links, loads or calls it.
//
// Parity status: parity unpinned at the source.  The reference path cannot
// be compiled here (it needs AdaptiveCpp `acpp` for every SYCL kernel and
// Eigen 3.4 for every solver frontend and multigrid setup; neither is
// present) and the reference ships no golden vectors for it, so no output of
// PSuM itself checks this restatement.  What constrains it: (1) the
// known-answer properties the reference's own tests assert for this path
// (CIC partition of unity / one-hot / linear reproduction at 1e-12,
// derivative vs central differences, multigrid residual reduction,
// multigrid vs direct solve within 1e-4 in <= 5 cycles, five-point residual
// < 1e-8) and (2) closed-form fixtures committed under tests/golden.
//
// Every function names the reference file:line it restates.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {
struct og_grid {            // same layout as psum_pic_grid_desc
    int dim;
    int cells[3];
    double lower[3];
    double upper[3];
    int periodic[3];
};
}

namespace {

// ---------------------------------------------------------------- grid ----
// simple_grid<D> (src/field/simple_grid.hpp:16-307)
struct Grid {
    int dim;
    int cells[3];
    double lo[3], hi[3], delta[3], dr[3];
    int periodic[3];
    explicit Grid(const og_grid* g) {
        dim = g->dim;
        for (int a = 0; a < 3; ++a) {
            cells[a] = a < dim ? g->cells[a] : 1;
            lo[a] = g->lower[a];
            hi[a] = g->upper[a];
            periodic[a] = g->periodic[a];
            if (a < dim) {
                delta[a] = (hi[a] - lo[a]) / cells[a];   // simple_grid.hpp:47
                dr[a] = 1.0 / delta[a];                  // :48
            } else {
                delta[a] = dr[a] = 1.0;
            }
        }
    }
    int nodes(int a) const { return cells[a] + 1; }
    long long n_nodes() const {
        long long n = 1;
        for (int a = 0; a < dim; ++a) n *= nodes(a);
        return n;
    }
    long long n_cells() const {
        long long n = 1;
        for (int a = 0; a < dim; ++a) n *= cells[a];
        return n;
    }
    // n2i: row-major, last dimension fastest (simple_grid.hpp:107-112)
    long long n2i(const int* n) const {
        long long ans = n[0];
        for (int a = 1; a < dim; ++a) ans = ans * (cells[a] + 1) + n[a];
        return ans;
    }
    // c2i (simple_grid.hpp:122-127)
    long long c2i(const int* c) const {
        long long ans = c[0];
        for (int a = 1; a < dim; ++a) ans = ans * cells[a] + c[a];
        return ans;
    }
    // inGrid: lo <= p < hi on every axis (simple_grid.hpp:168-174)
    bool in_grid(const double* p) const {
        for (int a = 0; a < dim; ++a)
            if (p[a] < lo[a] || p[a] >= hi[a]) return false;
        return true;
    }
};

// gen_interp / gen_interp_diff with linear_interp_1D (simple_grid.hpp:316-397,
// simple_interpolation.hpp:34-103): base node cN = floor((p-lo)*dr), support
// index i has bit 0 on the last dimension, support nodes wrap by +-(cells+1).
struct Support {
    long long idx[8];
    double coef[8];
    double dcoef[3][8];
    int count;
};

Support cic_support(const Grid& g, const double* p, bool diff) {
    Support s{};
    const int D = g.dim;
    s.count = 1 << D;
    int base[3];
    double xn[3];
    for (int a = 0; a < D; ++a) {
        base[a] = int(std::floor((p[a] - g.lo[a]) * g.dr[a]));          // cN, :89-95
        double base_pos = g.lo[a] + base[a] * g.delta[a];                // nodePosition, :209-214
        xn[a] = (p[a] - base_pos) * g.dr[a];                             // normalizedPos, :325-327
    }
    for (int i = 0; i < s.count; ++i) {
        int node[3] = {base[0], base[1], base[2]};
        int idx = i;
        for (int j = 0; j < D; ++j) {
            const int a = D - 1 - j;
            node[a] += idx % 2;
            const int w = g.cells[a] + 1;                                 // :338-343
            if (node[a] < 0) node[a] += w;
            else if (node[a] >= w) node[a] -= w;
            idx /= 2;
        }
        s.idx[i] = g.n2i(node);
        // interp_tensor (simple_interpolation.hpp:34-54): product over j of dim D-1-j
        double c = 1;
        idx = i;
        for (int j = 0; j < D; ++j) {
            const int a = D - 1 - j;
            const int b = idx % 2;
            c *= (b == 0) ? (1 - xn[a]) : xn[a];
            idx /= 2;
        }
        s.coef[i] = c;
        if (diff) {
            // interp_tensor_diff (simple_interpolation.hpp:58-90)
            for (int d = 0; d < D; ++d) {
                double cd = 1;
                idx = i;
                for (int j = 0; j < D; ++j) {
                    const int a = D - 1 - j;
                    const int b = idx % 2;
                    if (a == d) cd *= (b == 0 ? -1.0 : 1.0) * g.dr[a];
                    else cd *= (b == 0) ? (1 - xn[a]) : xn[a];
                    idx /= 2;
                }
                s.dcoef[d][i] = cd;
            }
        }
    }
    return s;
}

// ---------------------------------------------------------------- sparse ---
struct CSR {
    long long n_row = 0, n_col = 0;
    std::vector<long long> ptr;
    std::vector<long long> col;
    std::vector<double> val;
    double coeff(long long r, long long c) const {
        for (long long k = ptr[r]; k < ptr[r + 1]; ++k)
            if (col[k] == c) return val[k];
        return 0.0;
    }
};

// setFromTriplets: duplicates summed, columns sorted within a row.
CSR csr_from_coo(long long n_row, long long n_col, long long nnz, const unsigned long long* rows,
                 const unsigned long long* cols, const double* vals) {
    std::vector<std::map<long long, double>> acc(n_row);
    for (long long k = 0; k < nnz; ++k) {
        if ((long long)rows[k] >= n_row || (long long)cols[k] >= n_col)
            throw std::invalid_argument("coo index out of range");
        acc[rows[k]][cols[k]] += vals[k];
    }
    CSR m;
    m.n_row = n_row;
    m.n_col = n_col;
    m.ptr.assign(n_row + 1, 0);
    for (long long r = 0; r < n_row; ++r) m.ptr[r + 1] = m.ptr[r] + (long long)acc[r].size();
    m.col.resize(m.ptr[n_row]);
    m.val.resize(m.ptr[n_row]);
    for (long long r = 0; r < n_row; ++r) {
        long long k = m.ptr[r];
        for (auto& [c, v] : acc[r]) {
            m.col[k] = c;
            m.val[k] = v;
            ++k;
        }
    }
    return m;
}

CSR transpose(const CSR& a) {
    CSR t;
    t.n_row = a.n_col;
    t.n_col = a.n_row;
    t.ptr.assign(t.n_row + 1, 0);
    for (long long k = 0; k < (long long)a.col.size(); ++k) t.ptr[a.col[k] + 1]++;
    for (long long r = 0; r < t.n_row; ++r) t.ptr[r + 1] += t.ptr[r];
    t.col.resize(a.col.size());
    t.val.resize(a.val.size());
    std::vector<long long> pos(t.ptr.begin(), t.ptr.end() - 1);
    for (long long r = 0; r < a.n_row; ++r)
        for (long long k = a.ptr[r]; k < a.ptr[r + 1]; ++k) {
            long long p = pos[a.col[k]]++;
            t.col[p] = r;
            t.val[p] = a.val[k];
        }
    return t;
}

// C = A * B (row-wise with a dense accumulator); exact zeros are dropped,
// which is what Eigen's pruned() does (multigrid_core.hpp:98-99).
CSR spgemm(const CSR& a, const CSR& b, bool prune) {
    CSR c;
    c.n_row = a.n_row;
    c.n_col = b.n_col;
    std::vector<std::vector<long long>> rc(a.n_row);
    std::vector<std::vector<double>> rv(a.n_row);
#pragma omp parallel
    {
        std::vector<double> acc(b.n_col, 0.0);
        std::vector<char> used(b.n_col, 0);
        std::vector<long long> touched;
#pragma omp for schedule(dynamic, 256)
        for (long long r = 0; r < a.n_row; ++r) {
            touched.clear();
            for (long long ka = a.ptr[r]; ka < a.ptr[r + 1]; ++ka) {
                const long long m = a.col[ka];
                const double av = a.val[ka];
                for (long long kb = b.ptr[m]; kb < b.ptr[m + 1]; ++kb) {
                    const long long cc = b.col[kb];
                    if (!used[cc]) {
                        used[cc] = 1;
                        touched.push_back(cc);
                    }
                    acc[cc] += av * b.val[kb];
                }
            }
            std::sort(touched.begin(), touched.end());
            for (long long cc : touched) {
                if (!prune || acc[cc] != 0.0) {
                    rc[r].push_back(cc);
                    rv[r].push_back(acc[cc]);
                }
                acc[cc] = 0.0;
                used[cc] = 0;
            }
        }
    }
    c.ptr.assign(c.n_row + 1, 0);
    for (long long r = 0; r < c.n_row; ++r) c.ptr[r + 1] = c.ptr[r] + (long long)rc[r].size();
    c.col.resize(c.ptr[c.n_row]);
    c.val.resize(c.ptr[c.n_row]);
    for (long long r = 0; r < c.n_row; ++r) {
        std::copy(rc[r].begin(), rc[r].end(), c.col.begin() + c.ptr[r]);
        std::copy(rv[r].begin(), rv[r].end(), c.val.begin() + c.ptr[r]);
    }
    return c;
}

template <class T>
void spmv(const CSR& a, const std::vector<T>& x, std::vector<T>& y, const std::vector<T>* mat_cast = nullptr) {
    y.resize(a.n_row);
#pragma omp parallel for schedule(static)
    for (long long r = 0; r < a.n_row; ++r) {
        T s = T(0);
        for (long long k = a.ptr[r]; k < a.ptr[r + 1]; ++k)
            s += (mat_cast ? (*mat_cast)[k] : T(a.val[k])) * x[a.col[k]];
        y[r] = s;
    }
}

// ------------------------------------------------- structured transfers ---
// get_structured_transfers (src/field_solver/implements/multigrid/multigrid_utilities.hpp:26-104)
using Axis = std::vector<double>;
Axis coarsen(const Axis& fine) {                                   // :28-33
    Axis coarse;
    for (size_t i = 0; i < fine.size(); i += 2) coarse.push_back(fine[i]);
    if (coarse.back() != fine.back()) coarse.push_back(fine.back());
    return coarse;
}
std::vector<double> volumes(const Axis& x) {                       // :34-42
    std::vector<double> w(x.size(), 1.0);
    if (x.size() == 1) return w;
    for (size_t i = 0; i < x.size(); ++i)
        w[i] = ((i ? x[i] - x[i - 1] : 0.0) + (i + 1 < x.size() ? x[i + 1] - x[i] : 0.0)) * 0.5;
    return w;
}
std::vector<std::pair<int, double>> interpolate(double x, const Axis& coarse) {   // :44-52
    auto it = std::lower_bound(coarse.begin(), coarse.end(), x);
    if (it == coarse.end()) throw std::runtime_error("multigrid: point outside coarse grid");
    const int hi = int(it - coarse.begin());
    if (*it == x) return {{hi, 1.0}};
    if (hi == 0) throw std::runtime_error("multigrid: point outside coarse grid");
    const double t = (x - coarse[hi - 1]) / (coarse[hi] - coarse[hi - 1]);
    return {{hi - 1, 1.0 - t}, {hi, t}};
}

struct Transfers {
    std::vector<CSR> R, P;
    std::vector<std::array<int, 3>> dims;  // node dims per level (level 0 = fine)
};

// Periodic-axis transfers (an extension, not in PSuM): on an axis whose node
// lattice wraps, the coarse axis keeps every second node (n even -> n/2),
// P interpolates linearly with wrap-around and R = Pt/2.  PSuM's open-interval
// transfers (above) make V-cycles diverge on wrapping lattices pinned at one
// node once more than one or two coarse levels are used.
Transfers structured_transfers(int I, int J, int K, int depth, const int* periodic = nullptr) {   // :55-104
    if (I < 1 || J < 1 || K < 1 || depth < 1)
        throw std::invalid_argument("multigrid: positive grid dimensions and depth required");
    std::array<Axis, 3> axes;
    const int sizes[3] = {I, J, K};
    for (int d = 0; d < 3; ++d) {
        axes[d].resize(sizes[d]);
        for (int i = 0; i < sizes[d]; ++i) axes[d][i] = i;
    }
    Transfers t;
    t.dims.push_back({I, J, K});
    std::array<bool, 3> per{periodic && periodic[0], periodic && periodic[1], periodic && periodic[2]};
    for (int level = 0; level < depth; ++level) {
        std::array<Axis, 3> coarse;
        std::array<std::vector<double>, 3> vol;
        std::array<std::vector<std::vector<std::pair<int, double>>>, 3> wts;
        std::array<bool, 3> halve{false, false, false};
        for (int d = 0; d < 3; ++d) {
            const int nf = (int)axes[d].size();
            halve[d] = per[d] && nf >= 4 && nf % 2 == 0;
            if (per[d]) {
                // periodic axis: keep it unchanged when it cannot be halved
                coarse[d].clear();
                const int nc = halve[d] ? nf / 2 : nf;
                for (int i = 0; i < nc; ++i) coarse[d].push_back(i);
                vol[d].assign(nf, 1.0);
                for (int i = 0; i < nf; ++i) {
                    if (!halve[d]) wts[d].push_back({{i, 1.0}});
                    else if (i % 2 == 0) wts[d].push_back({{i / 2, 1.0}});
                    else wts[d].push_back({{i / 2, 0.5}, {(i / 2 + 1) % nc, 0.5}});
                }
                continue;
            }
            coarse[d] = coarsen(axes[d]);
            vol[d] = volumes(axes[d]);
            for (double x : axes[d]) wts[d].push_back(interpolate(x, coarse[d]));
        }
        const int ni = axes[0].size(), nj = axes[1].size(), nk = axes[2].size();
        const int ci = coarse[0].size(), cj = coarse[1].size(), ck = coarse[2].size();
        if (ni == ci && nj == cj && nk == ck) break;
        const long long nf = (long long)ni * nj * nk, nc = (long long)ci * cj * ck;
        std::vector<unsigned long long> rr, cc;
        std::vector<double> vv;
        std::vector<double> fine_volume(nf);
        for (int i = 0; i < ni; ++i)
            for (int j = 0; j < nj; ++j)
                for (int k = 0; k < nk; ++k) {
                    const long long row = ((long long)i * nj + j) * nk + k;
                    fine_volume[row] = vol[0][i] * vol[1][j] * vol[2][k];
                    for (auto [a, wa] : wts[0][i])
                        for (auto [b, wb] : wts[1][j])
                            for (auto [c, wc] : wts[2][k]) {
                                rr.push_back(row);
                                cc.push_back(((long long)a * cj + b) * ck + c);
                                vv.push_back(wa * wb * wc);
                            }
                }
        CSR P = csr_from_coo(nf, nc, (long long)rr.size(), rr.data(), cc.data(), vv.data());
        CSR R = transpose(P);
        std::vector<double> coarse_volume(nc, 0.0);
        for (long long r = 0; r < nc; ++r) {
            double s = 0;
            for (long long k = R.ptr[r]; k < R.ptr[r + 1]; ++k) s += R.val[k] * fine_volume[R.col[k]];
            coarse_volume[r] = s;
        }
        for (long long r = 0; r < nc; ++r)
            for (long long k = R.ptr[r]; k < R.ptr[r + 1]; ++k) R.val[k] *= fine_volume[R.col[k]] / coarse_volume[r];
        t.P.push_back(std::move(P));
        t.R.push_back(std::move(R));
        t.dims.push_back({ci, cj, ck});
        axes = coarse;
    }
    if (t.R.empty()) throw std::invalid_argument("multigrid: grid cannot be coarsened while retaining endpoints");
    return t;
}

// ------------------------------------------------------------ multigrid ---
// multigrid_core::setup / v_cycle_multi / solve_sequence / smooth
// (src/field_solver/implements/multigrid/multigrid_core.hpp:49-272), with the
// dense coarse inverse of sycl_inner_solver::compute (sycl_inner_solver.hpp:51-71).
struct MG {
    CSR A;                               // unscaled fine operator (residual_matrix)
    std::vector<CSR> Ahat, R, P;         // D^-1-scaled operators; transfers
    std::vector<CSR> relax;              // I - (2/3) Ahat per smoothed level (multigrid_core.hpp:129-134)
    std::vector<std::vector<double>> dinv;
    std::vector<double> coarse_inv;      // dense row-major inverse of Ahat[L]
    long long nc = 0;
    std::vector<std::array<int, 3>> dims;
};

std::vector<double> dense_inverse(const CSR& a) {
    const long long n = a.n_row;
    if (n > 8192) throw std::runtime_error("coarse matrix too large (> 8192)");  // sycl_inner_solver.hpp:54-57
    std::vector<double> m(n * n, 0.0), inv(n * n, 0.0);
    for (long long r = 0; r < n; ++r) {
        for (long long k = a.ptr[r]; k < a.ptr[r + 1]; ++k) m[r * n + a.col[k]] = a.val[k];
        inv[r * n + r] = 1.0;
    }
    // Gauss-Jordan elimination with partial pivoting.
    for (long long c = 0; c < n; ++c) {
        long long piv = c;
        for (long long r = c + 1; r < n; ++r)
            if (std::fabs(m[r * n + c]) > std::fabs(m[piv * n + c])) piv = r;
        if (m[piv * n + c] == 0.0) throw std::runtime_error("singular coarse matrix");
        if (piv != c)
            for (long long k = 0; k < n; ++k) {
                std::swap(m[c * n + k], m[piv * n + k]);
                std::swap(inv[c * n + k], inv[piv * n + k]);
            }
        const double d = 1.0 / m[c * n + c];
        for (long long k = 0; k < n; ++k) {
            m[c * n + k] *= d;
            inv[c * n + k] *= d;
        }
#pragma omp parallel for schedule(static)
        for (long long r = 0; r < n; ++r) {
            if (r == c) continue;
            const double f = m[r * n + c];
            if (f == 0.0) continue;
            for (long long k = 0; k < n; ++k) {
                m[r * n + k] -= f * m[c * n + k];
                inv[r * n + k] -= f * inv[c * n + k];
            }
        }
    }
    return inv;
}

void scale_rows(CSR& a, const std::vector<double>& d) {
    for (long long r = 0; r < a.n_row; ++r)
        for (long long k = a.ptr[r]; k < a.ptr[r + 1]; ++k) a.val[k] *= d[r];
}

MG* mg_setup(const CSR& A, int I, int J, int K, int depth, const int* periodic) {
    if ((long long)I * J * K != A.n_row) throw std::invalid_argument("grid dimensions do not match matrix");
    Transfers t = structured_transfers(I, J, K, depth, periodic);
    MG* mg = new MG();
    mg->A = A;
    mg->R = t.R;
    mg->P = t.P;
    mg->dims = t.dims;
    const size_t L = t.R.size();
    mg->Ahat.resize(L + 1);
    mg->dinv.resize(L + 1);
    mg->Ahat[0] = A;
    mg->dinv[0].resize(A.n_row);
    for (long long i = 0; i < A.n_row; ++i) mg->dinv[0][i] = 1 / A.coeff(i, i);    // :76-80
    scale_rows(mg->Ahat[0], mg->dinv[0]);                                            // :95-101
    for (size_t l = 1; l <= L; ++l) {                                                // :108-124
        CSR tmp = spgemm(spgemm(t.R[l - 1], mg->Ahat[l - 1], false), t.P[l - 1], true);
        mg->dinv[l].resize(tmp.n_row);
        for (long long i = 0; i < tmp.n_row; ++i) mg->dinv[l][i] = 1 / tmp.coeff(i, i);
        scale_rows(tmp, mg->dinv[l]);
        mg->Ahat[l] = std::move(tmp);
    }
    mg->coarse_inv = dense_inverse(mg->Ahat[L]);
    mg->nc = mg->Ahat[L].n_row;
    mg->relax.resize(L);
    for (size_t l = 0; l < L; ++l) {                    // Eye - a_mats_tmp[i] * 2.0 / 3
        const CSR& a = mg->Ahat[l];
        CSR& m = mg->relax[l];
        m.n_row = a.n_row;
        m.n_col = a.n_col;
        m.ptr.assign(a.n_row + 1, 0);
        for (long long r = 0; r < a.n_row; ++r) {
            bool has_diag = false;
            for (long long k = a.ptr[r]; k < a.ptr[r + 1]; ++k) {
                const double v = a.val[k] * 2.0 / 3;
                if (a.col[k] == r) has_diag = true;
                if (!has_diag && a.col[k] > r) {
                    m.col.push_back(r);
                    m.val.push_back(1.0);
                    has_diag = true;
                }
                m.col.push_back(a.col[k]);
                m.val.push_back(a.col[k] == r ? 1.0 - v : 0.0 - v);
            }
            if (!has_diag) {
                m.col.push_back(r);
                m.val.push_back(1.0);
            }
            m.ptr[r + 1] = (long long)m.col.size();
        }
    }
    return mg;
}

// solve_sequence for `cycles` V(pre,post) cycles in scalar type T; matrices
// are cast to T as the FP32 backend does at upload
// (conv_sycl_sparse_matrix.hpp:542-549) and accumulate in T (:490-498).
template <class T>
void mg_vcycles(const MG& mg, const std::vector<T>& in, std::vector<T>& out, int cycles, int pre, int post) {
    const size_t L = mg.R.size();
    auto cast_vals = [](const CSR& m) {
        std::vector<T> v(m.val.size());
        for (size_t k = 0; k < v.size(); ++k) v[k] = T(m.val[k]);
        return v;
    };
    std::vector<std::vector<T>> Av(L + 1), Rv(L), Pv(L), dv(L + 1), Xv(L);
    for (size_t l = 0; l <= L; ++l) {
        Av[l] = cast_vals(mg.Ahat[l]);
        dv[l].resize(mg.dinv[l].size());
        for (size_t i = 0; i < dv[l].size(); ++i) dv[l][i] = T(mg.dinv[l][i]);
    }
    for (size_t l = 0; l < L; ++l) {
        Rv[l] = cast_vals(mg.R[l]);
        Pv[l] = cast_vals(mg.P[l]);
        Xv[l] = cast_vals(mg.relax[l]);
    }
    std::vector<T> cinv(mg.coarse_inv.size());
    for (size_t k = 0; k < cinv.size(); ++k) cinv[k] = T(mg.coarse_inv[k]);

    std::vector<std::vector<T>> b(L + 1), x(L + 1), buf(L + 1);
    for (size_t l = 0; l <= L; ++l) {
        b[l].assign(mg.Ahat[l].n_row, T(0));
        x[l].assign(mg.Ahat[l].n_row, T(0));
        buf[l].assign(mg.Ahat[l].n_row, T(0));
    }
    for (size_t i = 0; i < in.size(); ++i) b[0][i] = in[i] * dv[0][i];               // hadamard_to, :208
    x[0] = out;                                                                       // copy_data, :215
    const T omega = T(2.0 / 3);
    auto smooth = [&](size_t l) {                                                     // :266-272
        // multiply_add(relax, x, b, buf, 2/3, 1): buf = relax*x + b*(2/3)
        std::vector<T> rx;
        spmv(mg.relax[l], x[l], rx, &Xv[l]);
        for (size_t i = 0; i < x[l].size(); ++i) buf[l][i] = rx[i] + b[l][i] * omega;
        std::swap(x[l], buf[l]);
    };
    std::vector<T> tmp;
    for (int cyc = 0; cyc < cycles; ++cyc) {
        for (size_t l = 0; l < L; ++l) {                                              // go_coarser
            for (int s = 0; s < pre; ++s) smooth(l);
            spmv(mg.Ahat[l], x[l], tmp, &Av[l]);
            for (size_t i = 0; i < tmp.size(); ++i) buf[l][i] = b[l][i] - tmp[i];     // multiply_add(-1,-1), :229
            spmv(mg.R[l], buf[l], b[l + 1], &Rv[l]);                                 // :230
            for (size_t i = 0; i < b[l + 1].size(); ++i) b[l + 1][i] *= dv[l + 1][i];   // :231
            std::fill(x[l + 1].begin(), x[l + 1].end(), T(0));                        // :232
        }
        // coarsest: dense inverse times vector (sycl_inner_solver.hpp:81-99)
        const long long n = mg.nc;
#pragma omp parallel for schedule(static)
        for (long long r = 0; r < n; ++r) {
            T s = T(0);
            for (long long c = 0; c < n; ++c) s += cinv[r * n + c] * b[L][c];
            x[L][r] = s;
        }
        for (size_t l = L; l-- > 0;) {                                                // go_finer
            spmv(mg.P[l], x[l + 1], tmp, &Pv[l]);
            for (size_t i = 0; i < tmp.size(); ++i) x[l][i] += tmp[i];                // :237, :259
            for (int s = 0; s < post; ++s) smooth(l);
        }
    }
    out = x[0];
}

// FP64 residual r = b - A x (residual_to<float> with T = double computes in FP64).
std::vector<double> residual(const CSR& A, const std::vector<double>& b, const std::vector<double>& x) {
    std::vector<double> ax;
    spmv(A, x, ax);
    std::vector<double> r(b.size());
    for (size_t i = 0; i < b.size(); ++i) r[i] = b[i] - ax[i];
    return r;
}

double norm2(const std::vector<double>& v) {
    double s = 0;
    for (double e : v) s += e * e;
    return std::sqrt(s);
}

thread_local std::string g_err;

// ------------------------------------------------------ B-spline support --
// The 1-D B-spline weights of orders 2-4 exactly as PSuM writes them
// (src/field/simple_interpolation.hpp:105-184): quadratic and quartic on the
// nearest node with s in [-0.5, 0.5], cubic on the corner node with u in
// [0, 1), each as its piecewise kernel evaluated at the support offsets.
double bs3(double t) {                                            // :124-130
    const double a = std::fabs(t);
    if (a <= 1.0) return 2.0 / 3.0 - a * a + a * a * a / 2.0;
    if (a <= 2.0) {
        const double r = 2.0 - a;
        return r * r * r / 6.0;
    }
    return 0.0;
}
double bs3d(double t) {                                           // :134-140
    const double a = std::fabs(t);
    if (a <= 1.0) return -2.0 * t + 1.5 * t * a;
    if (a <= 2.0) {
        const double r = 2.0 - a;
        return -r * r / 2.0 * (t < 0 ? -1.0 : 1.0);
    }
    return 0.0;
}
double pow4(double x) { return (x * x) * (x * x); }
double bs4(double t) {                                            // :153-163
    const double a = std::fabs(t);
    if (a <= 0.5) return 115.0 / 192.0 - a * a * (5.0 / 8.0) + a * a * a * a / 4.0;
    if (a <= 1.5) {
        const double v = a - 0.5;
        return 0.5 - (2.0 * v / 3.0 - v * v * v / 3.0 + v * v * v * v / 8.0) - pow4(1.5 - a) / 24.0;
    }
    if (a <= 2.5) return pow4(2.5 - a) / 24.0;
    return 0.0;
}
double bs4d(double t) {                                           // :167-177
    const double a = std::fabs(t);
    const double sign = t < 0 ? -1.0 : 1.0;
    if (a <= 0.5) return sign * (-a * 1.25 + a * a * a);
    if (a <= 1.5) {
        const double v = a - 0.5;
        const double r = 1.5 - a;
        return sign * (-(2.0 / 3.0 - v * v + v * v * v / 2.0) + r * r * r / 6.0);
    }
    if (a <= 2.5) {
        const double r = 2.5 - a;
        return sign * (-r * r * r / 6.0);
    }
    return 0.0;
}

// 1-D weights and their derivatives in the normalised coordinate.
void bs_weights(int order, double x, double* w, double* dw) {
    switch (order) {
        case 1:                                                    // linear_interp_1D, :92-98
            w[0] = 1 - x; w[1] = x; dw[0] = -1; dw[1] = 1;
            break;
        case 2:                                                    // :106-115
            w[0] = (0.5 - x) * (0.5 - x) * 0.5; w[1] = 0.75 - x * x; w[2] = (0.5 + x) * (0.5 + x) * 0.5;
            dw[0] = x - 0.5; dw[1] = -2.0 * x; dw[2] = x + 0.5;
            break;
        case 3:
            for (int k = 0; k < 4; ++k) {
                w[k] = bs3(x + 1.0 - k);
                dw[k] = bs3d(x + 1.0 - k);
            }
            break;
        default:
            for (int k = 0; k < 5; ++k) {
                w[k] = bs4(x + 2.0 - k);
                dw[k] = bs4d(x + 2.0 - k);
            }
    }
}

// gen_interp / gen_interp_diff for SupportSize1D = order + 1
// (simple_grid.hpp:316-397): odd support sizes use the nearest node nN
// (round, :79-86), even ones the corner node cN (floor, :88-95); the support
// runs from Shift = -(S/2) (odd) or -(S/2 - 1) (even); support index i has
// its base-S digit 0 on the last dimension; nodes wrap once by +-(cells+1);
// interp_tensor(_diff) products as in simple_interpolation.hpp:34-90.
// Returns false (no support) when a wrapped node is still outside the node
// range (a position more than a period away, which the reference does not
// handle) or the position is not finite.
struct BsSupport {
    std::vector<long long> idx;
    std::vector<double> coef;
    std::vector<double> dcoef[3];
};

bool bs_support(const Grid& g, int order, const double* p, bool diff, BsSupport& out) {
    const int D = g.dim, S = order + 1;
    const bool nearest = S % 2 == 1;
    const int shift = nearest ? -(S / 2) : -(S / 2 - 1);
    int base[3];
    double w1[3][5], dw1[3][5];
    for (int a = 0; a < D; ++a) {
        const double u = (p[a] - g.lo[a]) * g.dr[a];
        if (!std::isfinite(u) || u < -1e9 || u > 1e9) return false;
        base[a] = nearest ? (int)std::round(u) : (int)std::floor(u);
        const double base_pos = g.lo[a] + base[a] * g.delta[a];        // nodePosition, :209-214
        bs_weights(order, (p[a] - base_pos) * g.dr[a], w1[a], dw1[a]);
        for (int k = 0; k < S; ++k) dw1[a][k] *= g.dr[a];
    }
    int count = 1;
    for (int a = 0; a < D; ++a) count *= S;
    out.idx.assign(count, 0);
    out.coef.assign(count, 0.0);
    for (int d = 0; d < 3; ++d) out.dcoef[d].assign(diff ? count : 0, 0.0);
    for (int i = 0; i < count; ++i) {
        int node[3] = {base[0], base[1], base[2]};
        int digit[3] = {0, 0, 0};
        int r = i;
        for (int j = 0; j < D; ++j) {
            const int a = D - 1 - j;
            digit[a] = r % S;
            node[a] += digit[a] + shift;
            const int w = g.cells[a] + 1;
            if (node[a] < 0) node[a] += w;
            else if (node[a] >= w) node[a] -= w;
            if (node[a] < 0 || node[a] >= w) return false;
            r /= S;
        }
        out.idx[i] = g.n2i(node);
        double c = 1;
        for (int j = 0; j < D; ++j) c *= w1[D - 1 - j][digit[D - 1 - j]];
        out.coef[i] = c;
        if (diff)
            for (int d = 0; d < D; ++d) {
                double cd = 1;
                for (int j = 0; j < D; ++j) {
                    const int a = D - 1 - j;
                    cd *= a == d ? dw1[a][digit[a]] : w1[a][digit[a]];
                }
                out.dcoef[d][i] = cd;
            }
    }
    return true;
}

}  // namespace

extern "C" {

const char* oracle_last_error() { return g_err.c_str(); }

// ------------------------------------------------------- B-spline API ----
// Support of one point (order 1-4): writes S^D node indices, weights and
// (dim x S^D) derivative weights; returns S^D, or 0 without support.
int oracle_bspline_support(const og_grid* gd, int order, const double* p, long long* idx, double* coef,
                           double* dcoef) {
    Grid g(gd);
    BsSupport s;
    if (!bs_support(g, order, p, true, s)) return 0;
    const int count = (int)s.idx.size();
    for (int i = 0; i < count; ++i) {
        idx[i] = s.idx[i];
        coef[i] = s.coef[i];
        for (int d = 0; d < g.dim; ++d) dcoef[d * count + i] = s.dcoef[d][i];
    }
    return count;
}

// interp_B_spline<order> / interp_diff_B_spline<order>
// (src/field/higher_order_interp.hpp:200-228; generate_interp(_diff),
// field_interp.hpp:78-113, which skips weights of magnitude <= tol, 1e-10 in
// the reference) at n SoA positions; points without support give NaN.
// grad != nullptr selects the gradient (dim x n), else the value (n) goes to out.
void oracle_bspline_gather(const og_grid* gd, int order, long long n, const double* pos, const double* field,
                           double* out, double* grad, double tol) {
    Grid g(gd);
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < n; ++i) {
        double p[3] = {0, 0, 0};
        for (int a = 0; a < g.dim; ++a) p[a] = pos[a * n + i];
        BsSupport s;
        const bool ok = bs_support(g, order, p, grad != nullptr, s);
        if (grad) {
            for (int d = 0; d < g.dim; ++d) {
                double res = 0;
                if (ok)
                    for (size_t k = 0; k < s.idx.size(); ++k)
                        if (std::fabs(s.dcoef[d][k]) > tol) res += field[s.idx[k]] * s.dcoef[d][k];
                grad[d * n + i] = ok ? res : NAN;
            }
        } else {
            double res = 0;
            if (ok)
                for (size_t k = 0; k < s.idx.size(); ++k)
                    if (std::fabs(s.coef[k]) > tol) res += field[s.idx[k]] * s.coef[k];
            out[i] = ok ? res : NAN;
        }
    }
}

// add_back_B_spline<order> (higher_order_interp.hpp:230-245;
// generate_add_back_mutable for host fields, field_interp.hpp:66-75 with the
// weight skip at tol, 1e-10 in the reference) of n SoA positions with
// weight w, in particle order; returns the number of points skipped for lack
// of support.
long long oracle_bspline_deposit(const og_grid* gd, int order, long long n, const double* pos, double w,
                                 double* field, double tol) {
    Grid g(gd);
    long long skipped = 0;
    for (long long i = 0; i < n; ++i) {
        double p[3] = {0, 0, 0};
        for (int a = 0; a < g.dim; ++a) p[a] = pos[a * n + i];
        BsSupport s;
        if (!bs_support(g, order, p, false, s)) {
            ++skipped;
            continue;
        }
        for (size_t k = 0; k < s.idx.size(); ++k)
            if (std::fabs(s.coef[k]) > tol) field[s.idx[k]] += w * s.coef[k];
    }
    return skipped;
}

// ------------------------------------------------------------- CIC API ----
int oracle_interp(const og_grid* gd, const double* p, long long* idx, double* coef) {
    Grid g(gd);
    Support s = cic_support(g, p, false);
    for (int i = 0; i < s.count; ++i) {
        idx[i] = s.idx[i];
        coef[i] = s.coef[i];
    }
    return s.count;
}

int oracle_interp_diff(const og_grid* gd, const double* p, long long* idx, double* dcoef) {
    Grid g(gd);
    Support s = cic_support(g, p, true);
    for (int i = 0; i < s.count; ++i) {
        idx[i] = s.idx[i];
        for (int d = 0; d < g.dim; ++d) dcoef[d * s.count + i] = s.dcoef[d][i];
    }
    return s.count;
}

// generate_interp_diff (field_interp.hpp:96-113) with the 1e-10 skip; returns
// grad(phi) at p (E = -grad).
void oracle_gather_grad(const og_grid* gd, long long n, const double* pos, const double* phi, double* grad) {
    Grid g(gd);
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < n; ++i) {
        double p[3];
        for (int a = 0; a < g.dim; ++a) p[a] = pos[a * n + i];
        Support s = cic_support(g, p, true);
        for (int d = 0; d < g.dim; ++d) {
            double res = 0;
            for (int k = 0; k < s.count; ++k)
                if (std::fabs(s.dcoef[d][k]) > 1e-10) res += phi[s.idx[k]] * s.dcoef[d][k];
            grad[d * n + i] = res;
        }
    }
}

// ------------------------------------------------------------ push API ----
// One push of n particles (SoA FP64, pos[d*n+i], vel[c*n+i]), restating the
// app push idioms: leapfrog `v += E*q_m*dt; x += v*dt`
// (application/benchmark/TSI/main.cpp:59-75) and the Boris rotation
// (EDI/EDI.cpp:216-266 for B along z; collision-less-flow/particle_ops.hpp:17-51
// in 3D).  Boundary: periodic axes wrap by the period (cells+1)*dx into
// [lo, lo + period) with the TSI while-loops (:70-72); absorbing axes
// invalidate (x = NaN, validator.hpp:19-26) particles outside [lo, hi) and
// count them per (axis, side), first offending axis first.
// Invalid particles (non-finite x[0]) are skipped (particle_group.hpp:193-221).
void oracle_push(const og_grid* gd, long long n, double* pos, double* vel, const double* phi, double q_m,
                 double dt, int pusher, const double* B, unsigned long long* losses) {
    Grid g(gd);
    const int D = g.dim;
    std::vector<unsigned long long> loss(2 * D, 0);
#pragma omp parallel
    {
        std::vector<unsigned long long> my(2 * D, 0);
#pragma omp for schedule(static)
        for (long long i = 0; i < n; ++i) {
            if (!std::isfinite(pos[i])) continue;
            double p[3] = {0, 0, 0};
            for (int a = 0; a < D; ++a) p[a] = pos[a * n + i];
            Support s = cic_support(g, p, true);
            double E[3] = {0, 0, 0};
            for (int d = 0; d < D; ++d) {
                double res = 0;
                for (int k = 0; k < s.count; ++k)
                    if (std::fabs(s.dcoef[d][k]) > 1e-10) res += phi[s.idx[k]] * s.dcoef[d][k];
                E[d] = -res;
            }
            double v[3] = {vel[i], vel[n + i], vel[2 * n + i]};
            if (pusher == 0) {
                for (int d = 0; d < D; ++d) v[d] += E[d] * q_m * dt;
            } else {
                const double kk = q_m * dt / 2;
                double vm[3], t[3], sv[3], vp[3], vprime[3];
                for (int c = 0; c < 3; ++c) vm[c] = v[c] + E[c] * kk;
                double t2 = 0;
                for (int c = 0; c < 3; ++c) {
                    t[c] = B[c] * kk;
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
            for (int c = 0; c < 3; ++c) vel[c * n + i] = v[c];
            for (int d = 0; d < D; ++d) p[d] += v[d] * dt;
            bool dead = false;
            for (int d = 0; d < D && !dead; ++d) {
                if (g.periodic[d]) {
                    const double L = (g.cells[d] + 1) * g.delta[d];
                    const double top = g.lo[d] + L;
                    while (p[d] < g.lo[d]) p[d] += L;
                    while (p[d] >= top) p[d] -= L;
                } else if (p[d] < g.lo[d]) {
                    my[2 * d + 0]++;
                    dead = true;
                } else if (p[d] >= g.hi[d]) {
                    my[2 * d + 1]++;
                    dead = true;
                }
            }
            for (int d = 0; d < D; ++d) pos[d * n + i] = p[d];
            if (dead) pos[i] = std::numeric_limits<double>::quiet_NaN();
        }
#pragma omp critical
        for (int k = 0; k < 2 * D; ++k) loss[k] += my[k];
    }
    if (losses)
        for (int k = 0; k < 2 * D; ++k) losses[k] = loss[k];
}

// --------------------------------------------------------- deposit API ----
// Serial host add_back in particle order (host_field.hpp:260-296 with
// generate_add_back, field_interp.hpp:66-75): rho[node] += w * coef, skipping
// |coef| <= 1e-10.
void oracle_deposit(const og_grid* gd, long long n, const double* pos, double w, double* rho) {
    Grid g(gd);
    for (long long i = 0; i < n; ++i) {
        if (!std::isfinite(pos[i])) continue;
        double p[3] = {0, 0, 0};
        for (int a = 0; a < g.dim; ++a) p[a] = pos[a * n + i];
        Support s = cic_support(g, p, false);
        for (int k = 0; k < s.count; ++k)
            if (std::fabs(s.coef[k]) > 1e-10) rho[s.idx[k]] += w * s.coef[k];
    }
}

// ------------------------------------------------------------- binning ----
// grid_mapped_device_vector::update (grid_mapped_device_vector.hpp:47-87) in
// its canonical serial order: key = c2i(nC(p)) for in-grid particles,
// counts per cell, exclusive prefix, and the stable permutation.
long long oracle_bin(const og_grid* gd, long long n, const double* pos, long long* keys,
                     unsigned long long* counts, unsigned long long* offsets, unsigned long long* perm) {
    Grid g(gd);
    const long long nc = g.n_cells();
    std::fill(counts, counts + nc, 0ULL);
    for (long long i = 0; i < n; ++i) {
        double p[3] = {0, 0, 0};
        for (int a = 0; a < g.dim; ++a) p[a] = pos[a * n + i];
        if (!std::isfinite(p[0]) || !g.in_grid(p)) {
            keys[i] = -1;
            continue;
        }
        int c[3];
        // nC (simple_grid.hpp:99-104), clamped to the last cell: a position just below hi can
        // truncate to `cells` when dr = 1/dx rounds up; the reference indexes past its counts there
        for (int a = 0; a < g.dim; ++a) c[a] = std::min(int((p[a] - g.lo[a]) * g.dr[a]), g.cells[a] - 1);
        keys[i] = g.c2i(c);
        counts[keys[i]]++;
    }
    unsigned long long s = 0;
    for (long long c = 0; c < nc; ++c) {
        offsets[c] = s;
        s += counts[c];
    }
    std::vector<unsigned long long> cursor(offsets, offsets + nc);
    for (long long i = 0; i < n; ++i)
        if (keys[i] >= 0) perm[cursor[keys[i]]++] = (unsigned long long)i;
    return (long long)s;
}

// ------------------------------------------------------------ assembly ----
// Poisson_solver_{2,3}d::_init_impl for Cartesian grids, uniform epsilon, no
// mixed boundaries (Poisson_solver_2d.hpp:182-335, Poisson_solver_3d.hpp:221-349):
// fixed node -> identity row; other nodes -> -(1/V) sum_faces eps*S*grad with
// neighbours wrapped cyclically at (cells+1) nodes; terms merged per index as
// local_equation does (local_equation.hpp:28-58).  COO in column-major order.
long long oracle_poisson_assemble(int dim, const int* cells, const double* lo, const double* hi, double eps,
                                  long long n_fixed, const unsigned long long* fixed, unsigned long long* rows,
                                  unsigned long long* cols, double* vals) {
    int nd[3] = {1, 1, 1};
    double del[3] = {1, 1, 1}, dri[3] = {1, 1, 1};
    for (int a = 0; a < dim; ++a) {
        nd[a] = cells[a] + 1;
        del[a] = (hi[a] - lo[a]) / cells[a];
        dri[a] = 1.0 / del[a];
    }
    const long long n = (long long)nd[0] * nd[1] * nd[2];
    std::vector<char> is_fixed(n, 0);
    for (long long k = 0; k < n_fixed; ++k) is_fixed[fixed[k]] = 1;
    typedef std::map<unsigned long long, double> Eq;
    auto add = [](Eq& lhs, const Eq& rhs, double sign) {
        for (auto& [idx, c] : rhs) {
            const double cv = sign > 0 ? c : -c;
            auto it = lhs.find(idx);
            if (it == lhs.end()) lhs[idx] = cv;
            else {
                const double old_scale = std::fabs(c) + std::fabs(it->second);
                if (sign > 0) it->second += c;
                else it->second -= c;
                if (std::fabs(it->second) < old_scale * 1e-14) lhs.erase(it);
            }
        }
    };
    auto scaled = [](Eq e, double s) {
        for (auto& kv : e) kv.second *= s;
        if (std::fabs(s) == 0) e.clear();
        return e;
    };
    auto node = [&](int i, int j, int k) -> unsigned long long {
        i = ((i % nd[0]) + nd[0]) % nd[0];
        j = ((j % nd[1]) + nd[1]) % nd[1];
        k = ((k % nd[2]) + nd[2]) % nd[2];
        return ((unsigned long long)i * nd[1] + j) * nd[2] + k;
    };
    std::vector<std::vector<std::pair<unsigned long long, double>>> by_col(n);
    for (int i = 0; i < nd[0]; ++i)
        for (int j = 0; j < nd[1]; ++j)
            for (int k = 0; k < nd[2]; ++k) {
                const unsigned long long idx = node(i, j, k);
                Eq fin;
                if (is_fixed[idx]) {
                    fin[idx] = 1.0;
                } else if (dim == 2) {
                    const unsigned long long iN = node(i, j + 1, 0), iS = node(i, j - 1, 0), iE = node(i + 1, j, 0),
                                             iW = node(i - 1, j, 0);
                    Eq gN{{idx, dri[1] * -1}}, gS{{iS, dri[1] * -1}}, gE{{idx, dri[0] * -1}}, gW{{iW, dri[0] * -1}};
                    add(gN, Eq{{iN, dri[1]}}, 1);
                    add(gS, Eq{{idx, dri[1]}}, 1);
                    add(gE, Eq{{iE, dri[0]}}, 1);
                    add(gW, Eq{{idx, dri[0]}}, 1);
                    const double sNS = del[0], sEW = del[1], vol = del[0] * del[1];
                    Eq acc = scaled(scaled(gE, sEW), eps);
                    add(acc, scaled(scaled(gW, sEW), eps), -1);
                    add(acc, scaled(scaled(gN, sNS), eps), 1);
                    add(acc, scaled(scaled(gS, sNS), eps), -1);
                    fin = scaled(acc, -1.0 / vol);
                } else {
                    const unsigned long long iN = node(i, j + 1, k), iS = node(i, j - 1, k), iE = node(i + 1, j, k),
                                             iW = node(i - 1, j, k), iU = node(i, j, k + 1), iD = node(i, j, k - 1);
                    Eq gN{{idx, dri[1] * -1}}, gS{{iS, dri[1] * -1}}, gE{{idx, dri[0] * -1}}, gW{{iW, dri[0] * -1}},
                        gU{{idx, dri[2] * -1}}, gD{{iD, dri[2] * -1}};
                    add(gN, Eq{{iN, dri[1]}}, 1);
                    add(gS, Eq{{idx, dri[1]}}, 1);
                    add(gE, Eq{{iE, dri[0]}}, 1);
                    add(gW, Eq{{idx, dri[0]}}, 1);
                    add(gU, Eq{{iU, dri[2]}}, 1);
                    add(gD, Eq{{idx, dri[2]}}, 1);
                    const double sNS = del[0] * del[2], sEW = del[1] * del[2], sUD = del[0] * del[1];
                    const double vol = del[0] * del[1] * del[2];
                    Eq acc = scaled(scaled(gE, sEW), eps);
                    add(acc, scaled(scaled(gW, sEW), eps), -1);
                    add(acc, scaled(scaled(gN, sNS), eps), 1);
                    add(acc, scaled(scaled(gS, sNS), eps), -1);
                    add(acc, scaled(scaled(gU, sUD), eps), 1);
                    add(acc, scaled(scaled(gD, sUD), eps), -1);
                    fin = scaled(acc, -1.0 / vol);
                }
                for (auto& [c, v] : fin) by_col[c].push_back({idx, v});
            }
    long long nnz = 0;
    for (long long c = 0; c < n; ++c) {
        std::sort(by_col[c].begin(), by_col[c].end());
        for (auto& [r, v] : by_col[c]) {
            if (rows) {
                rows[nnz] = r;
                cols[nnz] = (unsigned long long)c;
                vals[nnz] = v;
            }
            ++nnz;
        }
    }
    return nnz;
}

// ---------------------------------------------------------- multigrid API --
void* oracle_mg_create(long long n, long long nnz, const unsigned long long* rows, const unsigned long long* cols,
                       const double* vals, int I, int J, int K, int depth, const int* periodic) {
    try {
        CSR A = csr_from_coo(n, n, nnz, rows, cols, vals);
        return mg_setup(A, I, J, K, depth, periodic);
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

void oracle_mg_destroy(void* h) { delete static_cast<MG*>(h); }

int oracle_mg_levels(void* h) { return (int)static_cast<MG*>(h)->Ahat.size(); }

long long oracle_mg_level_rows(void* h, int l) { return static_cast<MG*>(h)->Ahat[l].n_row; }

// Level operator as COO (for stencil-decomposition checks).
long long oracle_mg_level_coo(void* h, int l, unsigned long long* rows, unsigned long long* cols, double* vals,
                              double* dinv) {
    MG* mg = static_cast<MG*>(h);
    const CSR& a = mg->Ahat[l];
    long long k = 0;
    for (long long r = 0; r < a.n_row; ++r)
        for (long long q = a.ptr[r]; q < a.ptr[r + 1]; ++q, ++k)
            if (rows) {
                rows[k] = r;
                cols[k] = a.col[q];
                vals[k] = a.val[q];
            }
    if (dinv)
        for (long long r = 0; r < a.n_row; ++r) dinv[r] = mg->dinv[l][r];
    return k;
}

// FP64 V-cycles: cuda_multigrid_gpu / sycl_multigrid_gpu solve
// (cuda_multigrid_gpu.cu:140-180): x is the initial guess and the result.
void oracle_mg_vcycles(void* h, const double* b, double* x, int cycles, int pre, int post) {
    MG* mg = static_cast<MG*>(h);
    std::vector<double> in(b, b + mg->A.n_row), out(x, x + mg->A.n_row);
    mg_vcycles<double>(*mg, in, out, cycles, pre, post);
    std::copy(out.begin(), out.end(), x);
}

// The reference's mixed path, sycl_multigrid32f_gpu::solve
// (sycl_multigrid32f_gpu.cpp:106-160): FP64 residual cast to FP32, FP32
// V-cycles in batches of `correction_interval`, FP64 accumulation of the
// correction.  Returns the relative residual history per batch in `hist`
// (capacity max_cycles) and the batch count.
int oracle_mg_solve_mixed(void* h, const double* b, double* x, int max_cycles, int correction_interval, int pre,
                          int post, double* hist) {
    MG* mg = static_cast<MG*>(h);
    const long long n = mg->A.n_row;
    std::vector<double> bv(b, b + n), xv(x, x + n);
    const double bn = norm2(bv);
    int batches = 0;
    for (int cycle = 0; cycle < max_cycles;) {
        const int batch = std::min(correction_interval, max_cycles - cycle);
        std::vector<double> r = residual(mg->A, bv, xv);
        std::vector<float> r32(n), e32(n, 0.0f);
        for (long long i = 0; i < n; ++i) r32[i] = (float)r[i];
        mg_vcycles<float>(*mg, r32, e32, batch, pre, post);
        for (long long i = 0; i < n; ++i) xv[i] += (double)e32[i];
        if (hist) hist[batches] = norm2(residual(mg->A, bv, xv)) / (bn > 0 ? bn : 1.0);
        ++batches;
        cycle += batch;
    }
    std::copy(xv.begin(), xv.end(), x);
    return batches;
}

// The same refinement loop with the GPU backends' stopping rule: stop after
// the first batch whose relative residual ||b - A x|| / ||b|| is at most tol
// (tol 0: run max_cycles).  Returns the batches run; hist[k] = relative
// residual after batch k.
int oracle_mg_solve_mixed_tol(void* h, const double* b, double* x, int max_cycles, int correction_interval, int pre,
                              int post, double tol, double* hist) {
    MG* mg = static_cast<MG*>(h);
    const long long n = mg->A.n_row;
    std::vector<double> bv(b, b + n), xv(x, x + n);
    const double bn = norm2(bv);
    int batches = 0;
    for (int cycle = 0; cycle < max_cycles;) {
        const int batch = std::min(correction_interval, max_cycles - cycle);
        std::vector<double> r = residual(mg->A, bv, xv);
        std::vector<float> r32(n), e32(n, 0.0f);
        for (long long i = 0; i < n; ++i) r32[i] = (float)r[i];
        mg_vcycles<float>(*mg, r32, e32, batch, pre, post);
        for (long long i = 0; i < n; ++i) xv[i] += (double)e32[i];
        const double rel = norm2(residual(mg->A, bv, xv)) / (bn > 0 ? bn : 1.0);
        if (hist) hist[batches] = rel;
        ++batches;
        cycle += batch;
        if (tol > 0 && rel <= tol) break;
    }
    std::copy(xv.begin(), xv.end(), x);
    return batches;
}

double oracle_rel_residual(void* h, const double* b, const double* x) {
    MG* mg = static_cast<MG*>(h);
    const long long n = mg->A.n_row;
    std::vector<double> bv(b, b + n), xv(x, x + n);
    const double bn = norm2(bv);
    return norm2(residual(mg->A, bv, xv)) / (bn > 0 ? bn : 1.0);
}

// -------------------------------------------------------- diagnostics -----
// Energy diagnostics of the TSI app (TSI/main.cpp:132-146) generalised to
// D dimensions: kinetic 0.5*m*w*|v|^2 per particle, field
// 0.5*eps*sum over node edges ((phi_b - phi_a)/dx)^2 * cell volume.
double oracle_kinetic_energy(long long n, const double* pos, const double* vel, double mw) {
    double s = 0;
    for (long long i = 0; i < n; ++i) {
        if (!std::isfinite(pos[i])) continue;
        const double v2 = vel[i] * vel[i] + vel[n + i] * vel[n + i] + vel[2 * n + i] * vel[2 * n + i];
        s += 0.5 * mw * v2;
    }
    return s;
}

double oracle_field_energy(const og_grid* gd, const double* phi, double eps) {
    Grid g(gd);
    const int D = g.dim;
    int nd[3] = {1, 1, 1};
    for (int a = 0; a < D; ++a) nd[a] = g.cells[a] + 1;
    double vol = 1;
    for (int a = 0; a < D; ++a) vol *= g.delta[a];
    double s = 0;
    for (int i = 0; i < nd[0]; ++i)
        for (int j = 0; j < nd[1]; ++j)
            for (int k = 0; k < nd[2]; ++k) {
                int c[3] = {i, j, k};
                const long long a0 = ((long long)i * nd[1] + j) * nd[2] + k;
                for (int d = 0; d < D; ++d) {
                    int e[3] = {c[0], c[1], c[2]};
                    e[d] += 1;
                    if (e[d] >= nd[d]) {
                        if (!g.periodic[d]) continue;
                        e[d] = 0;
                    }
                    const long long b0 = ((long long)e[0] * nd[1] + e[1]) * nd[2] + e[2];
                    const double gr = (phi[b0] - phi[a0]) * g.dr[d];
                    s += gr * gr;
                }
            }
    return 0.5 * eps * s * vol;
}

}  // extern "C"
