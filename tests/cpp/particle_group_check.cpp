// Exercises include/psum_particle_group.hpp the way PSuM code uses a
// particle_group (src/particle_container/particle_group.hpp): insert with
// and without validation, size, content with NaN-invalid export, compress,
// clear and the capacity error.  Prints "ok" and exits 0 when every check
// holds; otherwise prints the failed check and exits 1.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "psum_particle_group.hpp"

using psum_b200::particle;
using psum_b200::particle_group;

static int failures = 0;
#define CHECK(cond)                                                       \
    do {                                                                  \
        if (!(cond)) {                                                    \
            std::printf("FAILED line %d: %s\n", __LINE__, #cond);         \
            ++failures;                                                   \
        }                                                                 \
    } while (0)

static double lcg(unsigned long long& s) {
    s = s * 6364136223846793005ULL + 1442695040888963407ULL;
    return (double)(s >> 11) * (1.0 / 9007199254740992.0);
}

static int run(int precision) {
    psum_pic_grid_desc g{};
    g.dim = 2;
    g.cells[0] = 16; g.cells[1] = 8; g.cells[2] = 1;
    g.lower[0] = 0.0; g.lower[1] = -1.0;
    g.upper[0] = 2.0; g.upper[1] = 1.0;
    g.periodic[0] = 0; g.periodic[1] = 0;
    psum_pic_ctx* ctx = nullptr;
    psum_b200::check(psum_pic_create(&g, precision, &ctx));
    psum_pic_species_desc desc{-1.0, 1.0, 1.0};
    const std::size_t cap = 400;
    particle_group<2> grp(ctx, desc, cap);
    CHECK(grp.capacity() == cap);
    CHECK(grp.size() == 0);

    // validating insert: every 10th particle has a NaN position and is dropped
    unsigned long long seed = 12345;
    std::vector<particle<2>> a(100), kept;
    for (std::size_t i = 0; i < a.size(); ++i) {
        a[i].position[0] = 0.05 + 1.9 * lcg(seed);
        a[i].position[1] = -0.95 + 1.9 * lcg(seed);
        for (int c = 0; c < 3; ++c) a[i].velocity[c] = lcg(seed) - 0.5;
        if (i % 10 == 3) a[i].position[0] = std::nan("");
        else kept.push_back(a[i]);
    }
    grp.insert(a);
    CHECK(grp.size() == kept.size());
    CHECK(grp.stored() == kept.size());

    // insert without validation: one particle outside the absorbing y wall is stored invalid
    const std::size_t m = 20;
    std::vector<double> pos(2 * m), vel(3 * m);
    for (std::size_t i = 0; i < m; ++i) {
        pos[i] = 0.05 + 1.9 * lcg(seed);
        pos[m + i] = i == 7 ? 1.5 : -0.95 + 1.9 * lcg(seed);
        for (int c = 0; c < 3; ++c) vel[c * m + i] = lcg(seed) - 0.5;
    }
    grp.insert_soa(m, pos.data(), vel.data());
    CHECK(grp.stored() == kept.size() + m);
    CHECK(grp.size() == kept.size() + m - 1);

    // content: insertion order, positions within the storage precision, the invalid one NaN
    const double tol = precision == PSUM_PIC_FP64 ? 0.0 : 1e-6;
    const double vtol = precision == PSUM_PIC_FP64 ? 0.0 : 1e-7;
    std::vector<particle<2>> all = grp.content();
    CHECK(all.size() == kept.size() + m);
    for (std::size_t i = 0; i < kept.size() && i < all.size(); ++i) {
        for (int d = 0; d < 2; ++d) CHECK(std::fabs(all[i].position[d] - kept[i].position[d]) <= tol);
        for (int c = 0; c < 3; ++c) CHECK(std::fabs(all[i].velocity[c] - kept[i].velocity[c]) <= vtol);
    }
    for (std::size_t i = 0; i < m && kept.size() + i < all.size(); ++i) {
        const auto& p = all[kept.size() + i];
        if (i == 7) {
            CHECK(!particle_group<2>::is_valid(p));
            continue;
        }
        CHECK(std::fabs(p.position[0] - pos[i]) <= tol);
        CHECK(std::fabs(p.position[1] - pos[m + i]) <= tol);
        CHECK(std::fabs(p.velocity[2] - vel[2 * m + i]) <= vtol);
    }

    // compress: only valid particles remain, ordered by cell
    grp.compress();
    CHECK(grp.stored() == grp.size());
    CHECK(grp.size() == kept.size() + m - 1);
    all = grp.content();
    int last_cell = -1;
    bool ordered = true;
    for (const auto& p : all) {
        CHECK(particle_group<2>::is_valid(p));
        const int cx = (int)std::floor((p.position[0] - g.lower[0]) / (2.0 / 16));
        const int cy = (int)std::floor((p.position[1] - g.lower[1]) / (2.0 / 8));
        const int cell = cx * 8 + cy;
        ordered = ordered && cell >= last_cell;
        last_cell = cell;
    }
    CHECK(ordered);

    // capacity: an insert beyond it fails with PSUM_ERR_OVERFLOW and changes nothing
    std::vector<particle<2>> big(cap, kept[0]);
    bool threw = false;
    try {
        grp.insert(big);
    } catch (const psum_b200::error& e) {
        threw = e.status() == PSUM_ERR_OVERFLOW;
    }
    CHECK(threw);
    CHECK(grp.size() == kept.size() + m - 1);

    // clear, then insert again
    grp.clear();
    CHECK(grp.size() == 0);
    CHECK(grp.stored() == 0);
    grp.insert(kept);
    CHECK(grp.size() == kept.size());

    psum_b200::check(psum_pic_destroy(ctx));
    return failures;
}

int main() {
    try {
        run(PSUM_PIC_MIXED);
        run(PSUM_PIC_FP64);
    } catch (const psum_b200::error& e) {
        std::printf("FAILED: library error %d: %s\n", e.status(), e.what());
        return 1;
    }
    if (failures) return 1;
    std::printf("ok\n");
    return 0;
}
