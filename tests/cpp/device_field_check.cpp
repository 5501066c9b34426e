// Exercises include/psum_device_field.hpp the way PSuM's TSI benchmark uses
// its B-spline free functions inside particle_group::for_each
// (application/benchmark/TSI/main.cpp:48-66): deposit a group with
// add_back_B_spline<Order> and gather the gradient with
// interp_diff_B_spline<Order>, at orders 1-4.  Checks: charge kept, a linear
// potential interpolated exactly with its constant gradient (support away from
// the wrap), and invalid particles skipped.  Prints "ok" and exits 0 when
// every check holds.
#include <cmath>
#include <cstdio>
#include <vector>

#include "psum_device_field.hpp"

using namespace psum_b200;

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

template <int Order>
static void check_order(const particle_group<2>& grp, const psum_pic_grid_desc& g) {
    const double w = 0.25;
    const std::vector<particle<2>> parts = grp.content();
    std::size_t valid = 0;
    for (const auto& p : parts) valid += particle_group<2>::is_valid(p);

    device_field<2> rho(g);
    add_back_B_spline<Order>(grp, w, rho);
    double q = 0;
    for (double v : rho.to_host()) q += v;
    CHECK(std::fabs(q - w * valid) < 1e-9 * valid);

    // phi = a.x + b on the nodes
    const double a0 = 0.7, a1 = -1.3, b = 0.4;
    const double dx0 = (g.upper[0] - g.lower[0]) / g.cells[0], dx1 = (g.upper[1] - g.lower[1]) / g.cells[1];
    std::vector<double> phi_h((std::size_t)(g.cells[0] + 1) * (g.cells[1] + 1));
    for (int i = 0; i <= g.cells[0]; ++i)
        for (int j = 0; j <= g.cells[1]; ++j)
            phi_h[(std::size_t)i * (g.cells[1] + 1) + j] = a0 * (g.lower[0] + i * dx0) + a1 * (g.lower[1] + j * dx1) + b;
    device_field<2> phi(g);
    phi.from_host(phi_h);
    const std::vector<double> val = interp_B_spline<Order>(grp, phi).to_host();
    const std::vector<double> grad = interp_diff_B_spline<Order>(grp, phi).to_host();
    const std::size_t n = parts.size();
    CHECK(val.size() == n && grad.size() == 2 * n);
    const double margin = 3.0;   // cells from the edges: no wrapped support
    for (std::size_t i = 0; i < n && val.size() == n && grad.size() == 2 * n; ++i) {
        const auto& p = parts[i];
        if (!particle_group<2>::is_valid(p)) {
            CHECK(std::isnan(val[i]) && std::isnan(grad[i]) && std::isnan(grad[n + i]));
            continue;
        }
        const double u0 = (p.position[0] - g.lower[0]) / dx0, u1 = (p.position[1] - g.lower[1]) / dx1;
        if (u0 < margin || u0 > g.cells[0] - margin || u1 < margin || u1 > g.cells[1] - margin) continue;
        CHECK(std::fabs(val[i] - (a0 * p.position[0] + a1 * p.position[1] + b)) < 1e-10);
        CHECK(std::fabs(grad[i] - a0) < 1e-9);
        CHECK(std::fabs(grad[n + i] - a1) < 1e-9);
    }
}

static void run(int precision) {
    psum_pic_grid_desc g{};
    g.dim = 2;
    g.cells[0] = 40; g.cells[1] = 24; g.cells[2] = 1;
    g.lower[0] = 0.0; g.lower[1] = -1.0;
    g.upper[0] = 4.0; g.upper[1] = 1.4;
    psum_pic_ctx* ctx = nullptr;
    check(psum_pic_create(&g, precision, &ctx));
    {
        particle_group<2> grp(ctx, psum_pic_species_desc{-1.0, 1.0, 1.0}, 30000);
        unsigned long long seed = 777;
        const std::size_t n = 20000;
        std::vector<double> pos(2 * n), vel(3 * n, 0.0);
        for (std::size_t i = 0; i < n; ++i) {
            pos[i] = g.lower[0] + (g.upper[0] - g.lower[0]) * lcg(seed);
            pos[n + i] = g.lower[1] + (g.upper[1] - g.lower[1]) * lcg(seed);
        }
        pos[5] = g.upper[0] + 1.0;   // outside the absorbing x wall: stored invalid
        grp.insert_soa(n, pos.data(), vel.data());
        CHECK(grp.stored() == n && grp.size() == n - 1);
        check_order<1>(grp, g);
        check_order<2>(grp, g);
        check_order<3>(grp, g);
        check_order<4>(grp, g);
    }
    check(psum_pic_destroy(ctx));
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
