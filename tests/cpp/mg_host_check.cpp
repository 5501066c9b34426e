// Runs the multigrid host setup of the library (psum_b200/csrc/mg_host.cpp,
// compiled into this program from its source) on an operator read from a
// file and writes every level's scaled operator Ahat_l, expanded from its
// stencil + exception form back to COO, with the level's inverse diagonal.
// A Python test compares them with the oracle's restatement of PSuM's
// multigrid_core::setup (multigrid_core.hpp:49-150).
//
// usage: mg_host_check in.bin out.bin
//   in.bin : int64 n, nnz, I, J, K, depth; uint64 rows[nnz]; uint64 cols[nnz]; double vals[nnz]
//   out.bin: int64 levels; per level: int64 n, m; uint64 rows[m]; uint64 cols[m]; double vals[m];
//            double dinv[n]; then int64 c and the c x c dense coarse inverse (row-major)
#include <cstdint>
#include <cstdio>
#include <exception>
#include <map>
#include <vector>

#include "../../psum_b200/csrc/mg_host.hpp"

using namespace psum_b200;

static bool read_all(FILE* f, void* p, size_t bytes) { return std::fread(p, 1, bytes, f) == bytes; }

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: mg_host_check in.bin out.bin\n");
        return 2;
    }
    FILE* in = std::fopen(argv[1], "rb");
    if (!in) return 2;
    int64_t hdr[6];
    if (!read_all(in, hdr, sizeof(hdr))) return 2;
    const int64_t n = hdr[0], nnz = hdr[1];
    std::vector<unsigned long long> rows(nnz), cols(nnz);
    std::vector<double> vals(nnz);
    if (!read_all(in, rows.data(), 8 * nnz) || !read_all(in, cols.data(), 8 * nnz) || !read_all(in, vals.data(), 8 * nnz))
        return 2;
    std::fclose(in);
    Hierarchy h;
    try {
        HostCSR A = csr_from_coo(n, n, nnz, rows.data(), cols.data(), vals.data());
        h = build_hierarchy(A, (int)hdr[2], (int)hdr[3], (int)hdr[4], (int)hdr[5]);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "build_hierarchy: %s\n", e.what());
        return 1;
    }
    FILE* out = std::fopen(argv[2], "wb");
    if (!out) return 2;
    const int64_t levels = (int64_t)h.ahat.size();
    std::fwrite(&levels, 8, 1, out);
    for (const StencilOp& op : h.ahat) {
        const int n0 = op.dims[0], n1 = op.dims[1], n2 = op.dims[2];
        std::map<std::pair<long long, long long>, double> coo;
        size_t t = 0;   // position in the exception list
        for (long long r = 0; r < op.n; ++r) {
            const bool exc = (op.mask[r / 32] >> (r % 32)) & 1u;
            if (exc) {
                for (int q = op.exc_ptr[t]; q < op.exc_ptr[t + 1]; ++q) coo[{r, op.exc_col[q]}] += op.exc_val[q];
                ++t;
                continue;
            }
            const int i = (int)(r / ((long long)n1 * n2)), j = (int)((r / n2) % n1), k = (int)(r % n2);
            for (int s = 0; s < op.ns; ++s) {
                const int a = ((i + op.delta[s][0]) % n0 + n0) % n0;
                const int b = ((j + op.delta[s][1]) % n1 + n1) % n1;
                const int c = ((k + op.delta[s][2]) % n2 + n2) % n2;
                coo[{r, ((long long)a * n1 + b) * n2 + c}] += op.coef[s];
            }
        }
        const int64_t nl = op.n, m = (int64_t)coo.size();
        std::fwrite(&nl, 8, 1, out);
        std::fwrite(&m, 8, 1, out);
        std::vector<unsigned long long> rr, cc;
        std::vector<double> vv;
        for (const auto& e : coo) {
            rr.push_back((unsigned long long)e.first.first);
            cc.push_back((unsigned long long)e.first.second);
            vv.push_back(e.second);
        }
        std::fwrite(rr.data(), 8, m, out);
        std::fwrite(cc.data(), 8, m, out);
        std::fwrite(vv.data(), 8, m, out);
        const std::vector<double>& d = h.dinv[&op - h.ahat.data()];
        std::fwrite(d.data(), 8, d.size(), out);
    }
    const int64_t cn = (int64_t)h.coarse_inv.size();
    std::fwrite(&cn, 8, 1, out);
    std::fwrite(h.coarse_inv.data(), 8, h.coarse_inv.size(), out);
    std::fclose(out);
    return 0;
}
