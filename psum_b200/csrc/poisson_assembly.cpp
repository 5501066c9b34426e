// poisson_assembly.cpp -- host-side finite-difference Poisson operator, the
// frontend half of PSuM's field solver.
//
// Restates Poisson_solver_2d::_init_impl (src/field_solver/Poisson_solver_2d.hpp:182-410)
// and Poisson_solver_3d::_init_impl (Poisson_solver_3d.hpp:178-349) for
// Cartesian grids with uniform epsilon and Dirichlet nodes:
//   fixed node      -> identity row
//   any other node  -> -(1/V) * sum_faces eps * S * grad, with neighbour
//                      indices wrapped cyclically at (cells+1) nodes per axis.
// Coefficients are formed with the same operation order as PSuM's
// local_equation algebra (local_equation.hpp:28-58, including its 1e-14
// cancellation rule), so the assembled values are bit-identical to what the
// PSuM frontend hands to set_matrix.  The COO is emitted in the column-major
// order of Poisson_solver_2d.hpp:392-402.
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.hpp"

namespace {

// Small ordered map (index -> coefficient) with local_equation's merge rules.
struct Eq {
    int n = 0;
    unsigned long long idx[8];
    double c[8];
    int find(unsigned long long i) const {
        for (int q = 0; q < n; ++q)
            if (idx[q] == i) return q;
        return -1;
    }
    void insert_sorted(unsigned long long i, double v) {
        int q = n;
        while (q > 0 && idx[q - 1] > i) {
            idx[q] = idx[q - 1];
            c[q] = c[q - 1];
            --q;
        }
        idx[q] = i;
        c[q] = v;
        ++n;
    }
    void erase(int q) {
        for (int k = q; k + 1 < n; ++k) {
            idx[k] = idx[k + 1];
            c[k] = c[k + 1];
        }
        --n;
    }
    // operator+= / operator-= (local_equation.hpp:32-58)
    void merge(const Eq& o, bool subtract) {
        for (int q = 0; q < o.n; ++q) {
            const int p = find(o.idx[q]);
            if (p < 0) insert_sorted(o.idx[q], subtract ? -o.c[q] : o.c[q]);
            else {
                const double old_scale = std::fabs(o.c[q]) + std::fabs(c[p]);
                if (subtract) c[p] -= o.c[q];
                else c[p] += o.c[q];
                if (std::fabs(c[p]) < old_scale * 1e-14) erase(p);
            }
        }
    }
    // operator*= (local_equation.hpp:22-30)
    Eq scaled(double s) const {
        Eq e = *this;
        for (int q = 0; q < e.n; ++q) e.c[q] *= s;
        if (std::fabs(s) == 0) e.n = 0;
        return e;
    }
    static Eq pair(unsigned long long a, double va, unsigned long long b, double vb) {
        Eq e;
        e.insert_sorted(a, va);
        if (e.find(b) < 0) e.insert_sorted(b, vb);   // map initializer_list keeps the first duplicate
        return e;
    }
};

}  // namespace

extern "C" EXPORT int psum_poisson_assemble(int dim, const int* cells, const double* lower, const double* upper,
                                            double epsilon, unsigned long long n_fixed,
                                            const unsigned long long* fixed_nodes, unsigned long long* nnz_out,
                                            unsigned long long* rows, unsigned long long* cols, double* vals) {
    return psum_b200::guarded([&] {
        if (dim != 2 && dim != 3) throw std::invalid_argument("psum_poisson_assemble: dim must be 2 or 3");
        if (!cells || !lower || !upper || !nnz_out) throw std::invalid_argument("psum_poisson_assemble: null argument");
        if (n_fixed > 0 && !fixed_nodes) throw std::invalid_argument("psum_poisson_assemble: null fixed node list");
        int nd[3] = {1, 1, 1};
        double del[3] = {1, 1, 1}, dri[3] = {1, 1, 1};
        for (int a = 0; a < dim; ++a) {
            if (cells[a] < 1) throw std::invalid_argument("psum_poisson_assemble: cells must be positive");
            if (!(lower[a] < upper[a])) throw std::invalid_argument("psum_poisson_assemble: lower must be < upper");
            nd[a] = cells[a] + 1;
            del[a] = (upper[a] - lower[a]) / cells[a];   // simple_grid.hpp:47-48
            dri[a] = 1.0 / del[a];
        }
        const long long n = (long long)nd[0] * nd[1] * nd[2];
        std::vector<char> is_fixed(n, 0);
        for (unsigned long long k = 0; k < n_fixed; ++k) {
            if (fixed_nodes[k] >= (unsigned long long)n)
                throw std::invalid_argument("psum_poisson_assemble: fixed node index out of range");
            is_fixed[fixed_nodes[k]] = 1;
        }
        auto node = [&](int i, int j, int k) -> unsigned long long {
            i = ((i % nd[0]) + nd[0]) % nd[0];
            j = ((j % nd[1]) + nd[1]) % nd[1];
            k = ((k % nd[2]) + nd[2]) % nd[2];
            return ((unsigned long long)i * nd[1] + j) * nd[2] + k;
        };
        // row-wise assembly
        std::vector<Eq> eqs(n);
#pragma omp parallel for schedule(static)
        for (long long r = 0; r < n; ++r) {
            const int i = (int)(r / ((long long)nd[1] * nd[2]));
            const int j = (int)((r / nd[2]) % nd[1]);
            const int k = (int)(r % nd[2]);
            const unsigned long long idx = (unsigned long long)r;
            Eq fin;
            if (is_fixed[r]) {
                fin.insert_sorted(idx, 1.0);
            } else if (dim == 2) {
                const unsigned long long iN = node(i, j + 1, 0), iS = node(i, j - 1, 0), iE = node(i + 1, j, 0),
                                         iW = node(i - 1, j, 0);
                const Eq gN = Eq::pair(idx, dri[1] * -1, iN, dri[1]);
                const Eq gS = Eq::pair(iS, dri[1] * -1, idx, dri[1]);
                const Eq gE = Eq::pair(idx, dri[0] * -1, iE, dri[0]);
                const Eq gW = Eq::pair(iW, dri[0] * -1, idx, dri[0]);
                const double sN = del[0], sS = del[0], sE = del[1], sW = del[1];
                const double volume = del[0] * del[1];
                Eq acc = gE.scaled(sE).scaled(epsilon);
                acc.merge(gW.scaled(sW).scaled(epsilon), true);
                acc.merge(gN.scaled(sN).scaled(epsilon), false);
                acc.merge(gS.scaled(sS).scaled(epsilon), true);
                fin = acc.scaled(-1.0 / volume);
            } else {
                const unsigned long long iN = node(i, j + 1, k), iS = node(i, j - 1, k), iE = node(i + 1, j, k),
                                         iW = node(i - 1, j, k), iU = node(i, j, k + 1), iD = node(i, j, k - 1);
                const Eq gN = Eq::pair(idx, dri[1] * -1, iN, dri[1]);
                const Eq gS = Eq::pair(iS, dri[1] * -1, idx, dri[1]);
                const Eq gE = Eq::pair(idx, dri[0] * -1, iE, dri[0]);
                const Eq gW = Eq::pair(iW, dri[0] * -1, idx, dri[0]);
                const Eq gU = Eq::pair(idx, dri[2] * -1, iU, dri[2]);
                const Eq gD = Eq::pair(iD, dri[2] * -1, idx, dri[2]);
                const double sNS = del[0] * del[2], sEW = del[1] * del[2], sUD = del[0] * del[1];
                const double volume = del[0] * del[1] * del[2];
                Eq acc = gE.scaled(sEW).scaled(epsilon);
                acc.merge(gW.scaled(sEW).scaled(epsilon), true);
                acc.merge(gN.scaled(sNS).scaled(epsilon), false);
                acc.merge(gS.scaled(sNS).scaled(epsilon), true);
                acc.merge(gU.scaled(sUD).scaled(epsilon), false);
                acc.merge(gD.scaled(sUD).scaled(epsilon), true);
                fin = acc.scaled(-1.0 / volume);
            }
            eqs[r] = fin;
        }
        // column-major order (CSC of the assembled matrix)
        std::vector<long long> colcount(n + 1, 0);
        for (long long r = 0; r < n; ++r)
            for (int q = 0; q < eqs[r].n; ++q) colcount[eqs[r].idx[q] + 1]++;
        for (long long c = 0; c < n; ++c) colcount[c + 1] += colcount[c];
        const unsigned long long nnz = (unsigned long long)colcount[n];
        *nnz_out = nnz;
        if (!rows) return;
        if (!cols || !vals) throw std::invalid_argument("psum_poisson_assemble: null output array");
        std::vector<long long> pos(colcount.begin(), colcount.end() - 1);
        for (long long r = 0; r < n; ++r)
            for (int q = 0; q < eqs[r].n; ++q) {
                const long long p = pos[eqs[r].idx[q]]++;
                rows[p] = (unsigned long long)r;
                cols[p] = eqs[r].idx[q];
                vals[p] = eqs[r].c[q];
            }
    });
}
