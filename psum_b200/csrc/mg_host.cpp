// mg_host.cpp -- host-side multigrid setup (see mg_host.hpp).
#include "mg_host.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <stdexcept>
#include <unordered_map>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace psum_b200 {

HostCSR csr_from_coo(long long n_row, long long n_col, long long nnz, const unsigned long long* rows,
                     const unsigned long long* cols, const double* vals) {
    if (n_row <= 0 || n_col <= 0) throw std::invalid_argument("set_matrix: empty matrix");
    if (n_row > 0x7fffffffLL || n_col > 0x7fffffffLL)
        throw std::invalid_argument("set_matrix: more than 2^31-1 rows is not supported");
    if (nnz > 0 && (!rows || !cols || !vals)) throw std::invalid_argument("set_matrix: null COO array");
    HostCSR m;
    m.n_row = n_row;
    m.n_col = n_col;
    std::vector<long long> cnt(n_row + 1, 0);
    for (long long k = 0; k < nnz; ++k) {
        if (rows[k] >= (unsigned long long)n_row || cols[k] >= (unsigned long long)n_col)
            throw std::invalid_argument("set_matrix: COO index out of range");
        cnt[rows[k] + 1]++;
    }
    for (long long r = 0; r < n_row; ++r) cnt[r + 1] += cnt[r];
    std::vector<int> c(nnz);
    std::vector<double> v(nnz);
    {
        std::vector<long long> pos(cnt.begin(), cnt.end() - 1);
        for (long long k = 0; k < nnz; ++k) {
            const long long p = pos[rows[k]]++;
            c[p] = (int)cols[k];
            v[p] = vals[k];
        }
    }
    // sort each row by column and merge duplicates (summed, like setFromTriplets)
    std::vector<long long> merged(n_row, 0);
#pragma omp parallel for schedule(dynamic, 4096)
    for (long long r = 0; r < n_row; ++r) {
        const long long b = cnt[r], e = cnt[r + 1];
        std::vector<std::pair<int, double>> tmp;
        tmp.reserve(e - b);
        for (long long k = b; k < e; ++k) tmp.push_back({c[k], v[k]});
        std::stable_sort(tmp.begin(), tmp.end(), [](auto& x, auto& y) { return x.first < y.first; });
        long long w = b;
        for (size_t q = 0; q < tmp.size(); ++q) {
            if (w > b && c[w - 1] == tmp[q].first) {
                v[w - 1] += tmp[q].second;
            } else {
                c[w] = tmp[q].first;
                v[w] = tmp[q].second;
                ++w;
            }
        }
        merged[r] = w - b;
    }
    m.ptr.assign(n_row + 1, 0);
    for (long long r = 0; r < n_row; ++r) m.ptr[r + 1] = m.ptr[r] + merged[r];
    m.col.resize(m.ptr[n_row]);
    m.val.resize(m.ptr[n_row]);
#pragma omp parallel for schedule(static)
    for (long long r = 0; r < n_row; ++r) {
        std::copy(c.begin() + cnt[r], c.begin() + cnt[r] + merged[r], m.col.begin() + m.ptr[r]);
        std::copy(v.begin() + cnt[r], v.begin() + cnt[r] + merged[r], m.val.begin() + m.ptr[r]);
    }
    return m;
}

namespace {

// ---- structured transfer factors (multigrid_utilities.hpp:26-104) ----
using Pos = std::vector<double>;

Pos coarsen_axis(const Pos& f) {
    Pos c;
    for (size_t i = 0; i < f.size(); i += 2) c.push_back(f[i]);
    if (c.back() != f.back()) c.push_back(f.back());
    return c;
}

std::vector<double> axis_volumes(const Pos& x) {
    std::vector<double> w(x.size(), 1.0);
    if (x.size() == 1) return w;
    for (size_t i = 0; i < x.size(); ++i)
        w[i] = ((i ? x[i] - x[i - 1] : 0.0) + (i + 1 < x.size() ? x[i + 1] - x[i] : 0.0)) * 0.5;
    return w;
}

Axis1D make_axis(const Pos& fine, const Pos& coarse) {
    Axis1D ax;
    ax.nf = (int)fine.size();
    ax.nc = (int)coarse.size();
    ax.p_c0.resize(ax.nf);
    ax.p_c1.assign(ax.nf, -1);
    ax.p_w0.resize(ax.nf);
    ax.p_w1.assign(ax.nf, 0.0);
    for (int i = 0; i < ax.nf; ++i) {
        const double x = fine[i];
        auto it = std::lower_bound(coarse.begin(), coarse.end(), x);
        if (it == coarse.end()) throw std::runtime_error("multigrid: point outside coarse grid");
        const int hi = int(it - coarse.begin());
        if (*it == x) {
            ax.p_c0[i] = hi;
            ax.p_w0[i] = 1.0;
        } else {
            if (hi == 0) throw std::runtime_error("multigrid: point outside coarse grid");
            const double t = (x - coarse[hi - 1]) / (coarse[hi] - coarse[hi - 1]);
            ax.p_c0[i] = hi - 1;
            ax.p_w0[i] = 1.0 - t;
            ax.p_c1[i] = hi;
            ax.p_w1[i] = t;
        }
    }
    // R_a(c, f) = P_a(f, c) * v(f) / sum_f' P_a(f', c) v(f')
    const std::vector<double> vol = axis_volumes(fine);
    std::vector<double> cvol(ax.nc, 0.0);
    std::vector<std::vector<std::pair<int, double>>> inv(ax.nc);
    for (int i = 0; i < ax.nf; ++i) {
        inv[ax.p_c0[i]].push_back({i, ax.p_w0[i]});
        if (ax.p_c1[i] >= 0) inv[ax.p_c1[i]].push_back({i, ax.p_w1[i]});
    }
    for (int c = 0; c < ax.nc; ++c) {
        for (auto& [f, w] : inv[c]) cvol[c] += w * vol[f];
        if (inv[c].size() > 3) throw std::runtime_error("multigrid: restriction support above 3 per axis");
    }
    ax.r_f.assign(3 * ax.nc, -1);
    ax.r_w.assign(3 * ax.nc, 0.0);
    for (int c = 0; c < ax.nc; ++c)
        for (size_t q = 0; q < inv[c].size(); ++q) {
            ax.r_f[3 * c + q] = inv[c][q].first;
            ax.r_w[3 * c + q] = inv[c][q].second * vol[inv[c][q].first] / cvol[c];
        }
    return ax;
}

// Periodic-axis factor (an extension of PSuM's transfers): coarse node c is
// fine node 2c, odd fine nodes interpolate their two even neighbours with
// wrap-around, and R = P^T / 2 (equal node volumes on a wrapping lattice).
Axis1D make_periodic_axis(int nf) {
    Axis1D ax;
    ax.nf = nf;
    ax.nc = nf / 2;
    ax.p_c0.resize(nf);
    ax.p_c1.assign(nf, -1);
    ax.p_w0.resize(nf);
    ax.p_w1.assign(nf, 0.0);
    for (int i = 0; i < nf; ++i) {
        if (i % 2 == 0) {
            ax.p_c0[i] = i / 2;
            ax.p_w0[i] = 1.0;
        } else {
            ax.p_c0[i] = i / 2;
            ax.p_w0[i] = 0.5;
            ax.p_c1[i] = (i / 2 + 1) % ax.nc;
            ax.p_w1[i] = 0.5;
        }
    }
    ax.r_f.assign(3 * ax.nc, -1);
    ax.r_w.assign(3 * ax.nc, 0.0);
    for (int c = 0; c < ax.nc; ++c) {
        ax.r_f[3 * c + 0] = (2 * c - 1 + nf) % nf;
        ax.r_w[3 * c + 0] = 0.25;
        ax.r_f[3 * c + 1] = 2 * c;
        ax.r_w[3 * c + 1] = 0.5;
        ax.r_f[3 * c + 2] = 2 * c + 1;
        ax.r_w[3 * c + 2] = 0.25;
    }
    return ax;
}

Axis1D identity_axis(int n) {
    Axis1D ax;
    ax.nf = ax.nc = n;
    ax.p_c0.resize(n);
    ax.p_c1.assign(n, -1);
    ax.p_w0.assign(n, 1.0);
    ax.p_w1.assign(n, 0.0);
    ax.r_f.assign(3 * n, -1);
    ax.r_w.assign(3 * n, 0.0);
    for (int i = 0; i < n; ++i) {
        ax.p_c0[i] = i;
        ax.r_f[3 * i] = i;
        ax.r_w[3 * i] = 1.0;
    }
    return ax;
}

inline int wrap_delta(int d, int n) {
    // minimal periodic image of an index difference on an axis of n nodes
    if (n <= 1) return d;
    if (d > 1 && d == n - 1) return -1;
    if (d < -1 && d == -(n - 1)) return 1;
    return d;
}

// ---- Galerkin product R * Ahat * P with the tensor-product transfers ----
// Each fine row's entries are taken in the order of their (wrapped) offsets,
// not of their column indices, so that rows equal up to a translation --
// the rows beside a periodic seam included -- sum in the same order and
// give bit-identical coarse rows (the stencil decomposition then finds no
// exception rows on uniform periodic lattices).
HostCSR galerkin(const HostCSR& ahat, const std::array<int, 3>& fd, const std::array<Axis1D, 3>& ax) {
    const std::array<int, 3> cd{ax[0].nc, ax[1].nc, ax[2].nc};
    const long long nc = (long long)cd[0] * cd[1] * cd[2];
    HostCSR out;
    out.n_row = out.n_col = nc;
    std::vector<std::vector<int>> rc(nc);
    std::vector<std::vector<double>> rv(nc);
#pragma omp parallel
    {
        std::unordered_map<long long, double> acc;
        acc.reserve(256);
        std::vector<std::pair<long long, double>> tmp;
        std::vector<std::pair<long long, long long>> ent;   // (offset order, CSR position) of a fine row's entries
#pragma omp for schedule(dynamic, 1024)
        for (long long c = 0; c < nc; ++c) {
            acc.clear();
            const int ci = int(c / ((long long)cd[1] * cd[2]));
            const int cj = int((c / cd[2]) % cd[1]);
            const int ck = int(c % cd[2]);
            for (int qa = 0; qa < 3; ++qa) {
                const int fi = ax[0].r_f[3 * ci + qa];
                if (fi < 0) continue;
                for (int qb = 0; qb < 3; ++qb) {
                    const int fj = ax[1].r_f[3 * cj + qb];
                    if (fj < 0) continue;
                    for (int qc = 0; qc < 3; ++qc) {
                        const int fk = ax[2].r_f[3 * ck + qc];
                        if (fk < 0) continue;
                        const double wr = ax[0].r_w[3 * ci + qa] * ax[1].r_w[3 * cj + qb] * ax[2].r_w[3 * ck + qc];
                        const long long f = ((long long)fi * fd[1] + fj) * fd[2] + fk;
                        ent.clear();
                        for (long long k = ahat.ptr[f]; k < ahat.ptr[f + 1]; ++k) {
                            const long long g = ahat.col[k];
                            const int di = wrap_delta(int(g / ((long long)fd[1] * fd[2])) - fi, fd[0]);
                            const int dj = wrap_delta(int((g / fd[2]) % fd[1]) - fj, fd[1]);
                            const int dk = wrap_delta(int(g % fd[2]) - fk, fd[2]);
                            const bool near = di >= -1 && di <= 1 && dj >= -1 && dj <= 1 && dk >= -1 && dk <= 1;
                            // offsets within one node first (by offset code), any others after, by column
                            ent.push_back({near ? (di + 1) * 9 + (dj + 1) * 3 + (dk + 1) : 27 + (k - ahat.ptr[f]), k});
                        }
                        std::sort(ent.begin(), ent.end());
                        for (const auto& [order, k] : ent) {
                            (void)order;
                            const long long g = ahat.col[k];
                            const double a = wr * ahat.val[k];
                            const int gi = int(g / ((long long)fd[1] * fd[2]));
                            const int gj = int((g / fd[2]) % fd[1]);
                            const int gk = int(g % fd[2]);
                            const int pi[2] = {ax[0].p_c0[gi], ax[0].p_c1[gi]};
                            const int pj[2] = {ax[1].p_c0[gj], ax[1].p_c1[gj]};
                            const int pk[2] = {ax[2].p_c0[gk], ax[2].p_c1[gk]};
                            const double wi[2] = {ax[0].p_w0[gi], ax[0].p_w1[gi]};
                            const double wj[2] = {ax[1].p_w0[gj], ax[1].p_w1[gj]};
                            const double wk[2] = {ax[2].p_w0[gk], ax[2].p_w1[gk]};
                            for (int a0 = 0; a0 < 2; ++a0) {
                                if (pi[a0] < 0) continue;
                                for (int a1 = 0; a1 < 2; ++a1) {
                                    if (pj[a1] < 0) continue;
                                    for (int a2 = 0; a2 < 2; ++a2) {
                                        if (pk[a2] < 0) continue;
                                        const long long cc = ((long long)pi[a0] * cd[1] + pj[a1]) * cd[2] + pk[a2];
                                        acc[cc] += a * (wi[a0] * wj[a1] * wk[a2]);
                                    }
                                }
                            }
                        }
                    }
                }
            }
            tmp.assign(acc.begin(), acc.end());
            std::sort(tmp.begin(), tmp.end());
            for (auto& [cc, v] : tmp) {
                if (v == 0.0) continue;   // pruned() drops exact zeros (multigrid_core.hpp:112)
                rc[c].push_back((int)cc);
                rv[c].push_back(v);
            }
        }
    }
    out.ptr.assign(nc + 1, 0);
    for (long long r = 0; r < nc; ++r) out.ptr[r + 1] = out.ptr[r] + (long long)rc[r].size();
    out.col.resize(out.ptr[nc]);
    out.val.resize(out.ptr[nc]);
#pragma omp parallel for schedule(static)
    for (long long r = 0; r < nc; ++r) {
        std::copy(rc[r].begin(), rc[r].end(), out.col.begin() + out.ptr[r]);
        std::copy(rv[r].begin(), rv[r].end(), out.val.begin() + out.ptr[r]);
    }
    return out;
}

std::vector<double> inverse_diagonal(const HostCSR& a) {
    std::vector<double> d(a.n_row);
#pragma omp parallel for schedule(static)
    for (long long r = 0; r < a.n_row; ++r) {
        double diag = 0.0;
        for (long long k = a.ptr[r]; k < a.ptr[r + 1]; ++k)
            if (a.col[k] == r) diag = a.val[k];
        d[r] = 1 / diag;   // A.coeff(i,i) may be 0 -> inf, as in PSuM
    }
    return d;
}

void scale_rows(HostCSR& a, const std::vector<double>& d) {
#pragma omp parallel for schedule(static)
    for (long long r = 0; r < a.n_row; ++r)
        for (long long k = a.ptr[r]; k < a.ptr[r + 1]; ++k) a.val[k] *= d[r];
}

// Gauss-Jordan inverse with partial pivoting (textbook method) of a + shift
// (shift added to every entry: the rank-one term of a singular operator
// whose null space is the constants).
std::vector<double> dense_inverse(const HostCSR& a, double shift = 0.0) {
    const long long n = a.n_row;
    std::vector<double> m(n * n, shift), inv(n * n, 0.0);
    for (long long r = 0; r < n; ++r) {
        for (long long k = a.ptr[r]; k < a.ptr[r + 1]; ++k) m[r * n + a.col[k]] += a.val[k];
        inv[r * n + r] = 1.0;
    }
    for (long long c = 0; c < n; ++c) {
        long long piv = c;
        for (long long r = c + 1; r < n; ++r)
            if (std::fabs(m[r * n + c]) > std::fabs(m[piv * n + c])) piv = r;
        if (!(std::fabs(m[piv * n + c]) > 0.0)) throw std::runtime_error("multigrid: singular coarse operator");
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
            double* mr = &m[r * n];
            double* ir = &inv[r * n];
            const double* mc = &m[c * n];
            const double* ic = &inv[c * n];
            for (long long k = 0; k < n; ++k) {
                mr[k] -= f * mc[k];
                ir[k] -= f * ic[k];
            }
        }
    }
    return inv;
}


struct RowPattern {
    std::vector<std::pair<int, double>> e;  // (delta code, value) sorted by code
    bool ok = true;                         // all deltas within {-1,0,1}^3
};

RowPattern row_pattern(const HostCSR& a, long long r, const std::array<int, 3>& dims) {
    RowPattern p;
    const long long n12 = (long long)dims[1] * dims[2];
    const int ri = int(r / n12), rj = int((r / dims[2]) % dims[1]), rk = int(r % dims[2]);
    for (long long k = a.ptr[r]; k < a.ptr[r + 1]; ++k) {
        const long long c = a.col[k];
        const int ci = int(c / n12), cj = int((c / dims[2]) % dims[1]), ck = int(c % dims[2]);
        const int di = wrap_delta(ci - ri, dims[0]);
        const int dj = wrap_delta(cj - rj, dims[1]);
        const int dk = wrap_delta(ck - rk, dims[2]);
        if (di < -1 || di > 1 || dj < -1 || dj > 1 || dk < -1 || dk > 1) {
            p.ok = false;
            return p;
        }
        p.e.push_back({(di + 1) * 9 + (dj + 1) * 3 + (dk + 1), a.val[k]});
    }
    std::sort(p.e.begin(), p.e.end(), [](auto& x, auto& y) { return x.first < y.first; });
    for (size_t q = 1; q < p.e.size(); ++q)
        if (p.e[q].first == p.e[q - 1].first) p.ok = false;   // two columns alias one delta (tiny axes)
    return p;
}

bool same_pattern(const RowPattern& x, const RowPattern& y) {
    if (!x.ok || !y.ok || x.e.size() != y.e.size()) return false;
    for (size_t q = 0; q < x.e.size(); ++q)
        if (x.e[q].first != y.e[q].first || std::memcmp(&x.e[q].second, &y.e[q].second, sizeof(double)) != 0)
            return false;
    return true;
}

}  // namespace

StencilOp decompose(const HostCSR& A, const std::array<int, 3>& dims) {
    StencilOp op;
    op.dims = dims;
    op.n = A.n_row;
    // Choose the stencil: most frequent exact row pattern among evenly spaced
    // sample rows (deterministic; ties go to the earliest sample).
    const long long samples = std::min<long long>(A.n_row, 4096);
    std::vector<RowPattern> cand;
    std::vector<int> votes;
    for (long long s = 0; s < samples; ++s) {
        const long long r = (A.n_row <= samples) ? s : (long long)((double)s * (A.n_row - 1) / (samples - 1));
        RowPattern p = row_pattern(A, r, dims);
        if (!p.ok || p.e.empty()) continue;
        bool found = false;
        for (size_t q = 0; q < cand.size(); ++q)
            if (same_pattern(cand[q], p)) {
                votes[q]++;
                found = true;
                break;
            }
        if (!found && cand.size() < 64) {
            cand.push_back(p);
            votes.push_back(1);
        }
    }
    RowPattern stencil;
    stencil.ok = false;
    if (!cand.empty()) {
        size_t best = 0;
        for (size_t q = 1; q < cand.size(); ++q)
            if (votes[q] > votes[best]) best = q;
        stencil = cand[best];
    }
    if (stencil.ok) {
        op.ns = (int)stencil.e.size();
        for (int s = 0; s < op.ns; ++s) {
            const int code = stencil.e[s].first;
            op.delta[s] = {code / 9 - 1, (code / 3) % 3 - 1, code % 3 - 1};
            op.coef[s] = stencil.e[s].second;
        }
    }
    // Classify every row.
    const long long nw = (A.n_row + 31) / 32;
    op.mask.assign(nw, 0u);
    std::vector<char> is_exc(A.n_row, 0);
#pragma omp parallel for schedule(dynamic, 8192)
    for (long long r = 0; r < A.n_row; ++r) {
        bool regular = false;
        if (stencil.ok) {
            RowPattern p = row_pattern(A, r, dims);
            regular = same_pattern(p, stencil);
        }
        is_exc[r] = regular ? 0 : 1;
    }
    for (long long r = 0; r < A.n_row; ++r)
        if (is_exc[r]) {
            op.mask[r / 32] |= (1u << (r % 32));
            op.exc_rows.push_back((int)r);
        }
    op.mask_prefix.assign(nw, 0u);
    uint32_t run = 0;
    for (long long w = 0; w < nw; ++w) {
        op.mask_prefix[w] = run;
        run += (uint32_t)__builtin_popcount(op.mask[w]);
    }
    op.exc_ptr.assign(op.exc_rows.size() + 1, 0);
    for (size_t q = 0; q < op.exc_rows.size(); ++q) {
        const long long r = op.exc_rows[q];
        const long long cnt = A.ptr[r + 1] - A.ptr[r];
        if ((long long)op.exc_ptr[q] + cnt > 0x7fffffffLL) throw std::runtime_error("multigrid: exception list too large");
        op.exc_ptr[q + 1] = op.exc_ptr[q] + (int)cnt;
    }
    op.exc_col.resize(op.exc_ptr.back());
    op.exc_val.resize(op.exc_ptr.back());
    for (size_t q = 0; q < op.exc_rows.size(); ++q) {
        const long long r = op.exc_rows[q];
        long long w = op.exc_ptr[q];
        for (long long k = A.ptr[r]; k < A.ptr[r + 1]; ++k, ++w) {
            op.exc_col[w] = A.col[k];
            op.exc_val[w] = A.val[k];
        }
    }
    return op;
}

Hierarchy build_hierarchy(const HostCSR& A, int I, int J, int K, int depth, int max_coarse,
                          const std::array<int, 3>& periodic, bool null_space) {
    if (A.n_row != A.n_col) throw std::runtime_error("invalid setup parameter");
    if (I < 1 || J < 1 || K < 1 || depth < 1)
        throw std::invalid_argument("multigrid: positive grid dimensions and depth required");
    if ((long long)I * J * K != A.n_row) throw std::invalid_argument("multigrid: grid dimensions do not match matrix");
    Hierarchy h;
    std::array<Pos, 3> axes;
    const int sizes[3] = {I, J, K};
    for (int d = 0; d < 3; ++d) {
        axes[d].resize(sizes[d]);
        for (int i = 0; i < sizes[d]; ++i) axes[d][i] = i;
    }
    h.dims.push_back({I, J, K});
    for (int level = 0; level < depth; ++level) {
        std::array<Pos, 3> coarse;
        std::array<bool, 3> halve{false, false, false};
        for (int d = 0; d < 3; ++d) {
            const int nf = (int)axes[d].size();
            if (periodic[d]) {
                halve[d] = nf >= 4 && nf % 2 == 0;
                coarse[d].resize(halve[d] ? nf / 2 : nf);
                for (size_t i = 0; i < coarse[d].size(); ++i) coarse[d][i] = (double)i;
            } else {
                coarse[d] = coarsen_axis(axes[d]);
            }
        }
        if (coarse[0].size() == axes[0].size() && coarse[1].size() == axes[1].size() &&
            coarse[2].size() == axes[2].size())
            break;
        std::array<Axis1D, 3> x;
        for (int d = 0; d < 3; ++d) {
            if (periodic[d]) x[d] = halve[d] ? make_periodic_axis((int)axes[d].size()) : identity_axis((int)axes[d].size());
            else x[d] = make_axis(axes[d], coarse[d]);
        }
        h.xfer.push_back(x);
        h.dims.push_back({(int)coarse[0].size(), (int)coarse[1].size(), (int)coarse[2].size()});
        axes = coarse;
    }
    if (h.xfer.empty()) throw std::invalid_argument("multigrid: grid cannot be coarsened while retaining endpoints");
    h.L = (int)h.xfer.size();

    h.a0 = decompose(A, h.dims[0]);
    HostCSR cur = A;
    h.dinv.resize(h.L + 1);
    h.ahat.resize(h.L + 1);
    h.dinv[0] = inverse_diagonal(cur);
    scale_rows(cur, h.dinv[0]);
    h.ahat[0] = decompose(cur, h.dims[0]);
    for (int l = 1; l <= h.L; ++l) {
        HostCSR next = galerkin(cur, h.dims[l - 1], h.xfer[l - 1]);
        h.dinv[l] = inverse_diagonal(next);
        scale_rows(next, h.dinv[l]);
        if (l < h.L) h.ahat[l] = decompose(next, h.dims[l]);
        else {
            if (next.n_row > max_coarse)
                throw std::runtime_error("sycl_inner_solver: coarse matrix too large (" + std::to_string(next.n_row) +
                                         " > " + std::to_string(max_coarse) + ")");
            h.ahat[l] = decompose(next, h.dims[l]);
            // null space = constants at every level (P reproduces constants):
            // (Ahat_L + 1 1^T / n)^-1 solves every consistent coarse system
            h.coarse_inv = dense_inverse(next, null_space ? 1.0 / (double)next.n_row : 0.0);
        }
        cur = std::move(next);
    }
    return h;
}

}  // namespace psum_b200
