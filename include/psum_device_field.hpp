/*
 * psum_device_field.hpp -- header-only C++ adapter for PSuM's node-centred
 * device_field (src/field/device_field.hpp) and its B-spline free functions
 * (src/field/higher_order_interp.hpp:196-247), over include/psum_interp.h.
 *
 * PSuM applies interp_diff_B_spline<Order> / add_back_B_spline<Order> per
 * particle inside particle_group::for_each lambdas (application/benchmark/TSI/main.cpp:48-66);
 * here each is one call over all particles of a psum_b200::particle_group,
 * whose positions are exported to the device first (psum_pic_get_state_device).
 *
 *   device_field<D> f(grid);              // zero-initialised node field, prod(cells + 1) doubles
 *   add_back_B_spline<3>(electrons, w, f); // f += w * W3(x_p) over valid particles
 *   device_array<double> g = interp_diff_B_spline<3>(electrons, phi);   // (D, n) gradient
 *
 * Invalid particles (NaN x) have no support: the gradient is NaN for them and
 * the deposit skips them.  Link against libpsum_b200.so and the CUDA runtime.
 */
#ifndef PSUM_B200_DEVICE_FIELD_HPP
#define PSUM_B200_DEVICE_FIELD_HPP

#include <cuda_runtime.h>

#include <cstddef>
#include <string>
#include <utility>
#include <vector>

#include "psum_interp.h"
#include "psum_particle_group.hpp"

namespace psum_b200 {

inline void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw error(PSUM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

/* Device memory of `n` elements (plays the role of PSuM's device_vector for
 * the arrays these calls exchange). */
template <class T>
class device_array {
public:
    device_array() = default;
    explicit device_array(std::size_t n) : n_(n) {
        if (n_) check_cuda(cudaMalloc(reinterpret_cast<void**>(&p_), n_ * sizeof(T)), "cudaMalloc");
    }
    ~device_array() {
        if (p_) cudaFree(p_);
    }
    device_array(const device_array&) = delete;
    device_array& operator=(const device_array&) = delete;
    device_array(device_array&& o) noexcept : p_(o.p_), n_(o.n_) {
        o.p_ = nullptr;
        o.n_ = 0;
    }
    device_array& operator=(device_array&& o) noexcept {
        std::swap(p_, o.p_);
        std::swap(n_, o.n_);
        return *this;
    }
    T* data() { return p_; }
    const T* data() const { return p_; }
    std::size_t size() const { return n_; }
    std::vector<T> to_host() const {
        std::vector<T> h(n_);
        if (n_) check_cuda(cudaMemcpy(h.data(), p_, n_ * sizeof(T), cudaMemcpyDeviceToHost), "cudaMemcpy D2H");
        return h;
    }
    void from_host(const std::vector<T>& h) {
        if (h.size() != n_) throw error(PSUM_ERR_INVALID_ARGUMENT, "device_array: size mismatch");
        if (n_) check_cuda(cudaMemcpy(p_, h.data(), n_ * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy H2D");
    }

private:
    T* p_ = nullptr;
    std::size_t n_ = 0;
};

/* device_field<D, var_loc::nodeCentered, double, 1>: an FP64 node field on
 * the grid, last dimension fastest (simple_grid::n2i). */
template <int D>
class device_field {
public:
    explicit device_field(const psum_pic_grid_desc& grid) : grid_(grid), data_(node_count(grid)) {
        if (grid.dim != D) throw error(PSUM_ERR_INVALID_ARGUMENT, "device_field: grid dimension mismatch");
        if (data_.size()) check_cuda(cudaMemset(data_.data(), 0, data_.size() * sizeof(double)), "cudaMemset");
    }
    const psum_pic_grid_desc& grid() const { return grid_; }
    std::size_t size() const { return data_.size(); }
    double* data() { return data_.data(); }
    const double* data() const { return data_.data(); }
    void set_zero() { check_cuda(cudaMemset(data_.data(), 0, data_.size() * sizeof(double)), "cudaMemset"); }
    std::vector<double> to_host() const { return data_.to_host(); }
    void from_host(const std::vector<double>& h) { data_.from_host(h); }

private:
    static std::size_t node_count(const psum_pic_grid_desc& g) {
        std::size_t n = 1;
        for (int a = 0; a < g.dim; ++a) n *= (std::size_t)g.cells[a] + 1;
        return n;
    }
    psum_pic_grid_desc grid_;
    device_array<double> data_;
};

/* The stored particles' positions as a (D, n) FP64 SoA device array. */
template <int D>
device_array<double> positions(const particle_group<D>& grp) {
    const std::size_t n = grp.stored();
    device_array<double> pos((std::size_t)D * n), vel(3 * n);
    if (n) check(psum_pic_get_state_device(grp.context(), grp.species(), pos.data(), vel.data()));
    return pos;
}

/* interp_B_spline<Order> of `f` at every stored particle: n values. */
template <int Order, int D>
device_array<double> interp_B_spline(const particle_group<D>& grp, const device_field<D>& f) {
    static_assert(Order >= 1 && Order <= 4, "B-spline order 1-4");
    device_array<double> pos = positions(grp);
    const std::size_t n = pos.size() / D;
    device_array<double> out(n);
    check(psum_interp_bspline(&f.grid(), Order, n, pos.data(), f.data(), out.data(), nullptr, nullptr));
    check_cuda(cudaDeviceSynchronize(), "interp_B_spline");
    return out;
}

/* interp_diff_B_spline<Order>: the (D, n) gradient at every stored particle. */
template <int Order, int D>
device_array<double> interp_diff_B_spline(const particle_group<D>& grp, const device_field<D>& f) {
    static_assert(Order >= 1 && Order <= 4, "B-spline order 1-4");
    device_array<double> pos = positions(grp);
    const std::size_t n = pos.size() / D;
    device_array<double> out((std::size_t)D * n);
    check(psum_interp_diff_bspline(&f.grid(), Order, n, pos.data(), f.data(), out.data(), nullptr, nullptr));
    check_cuda(cudaDeviceSynchronize(), "interp_diff_B_spline");
    return out;
}

/* add_back_B_spline<Order>: f += w * W(x_p) summed over the valid particles. */
template <int Order, int D>
void add_back_B_spline(const particle_group<D>& grp, double w, device_field<D>& f) {
    static_assert(Order >= 1 && Order <= 4, "B-spline order 1-4");
    device_array<double> pos = positions(grp);
    const std::size_t n = pos.size() / D;
    check(psum_add_back_bspline(&f.grid(), Order, n, pos.data(), w, f.data(), nullptr, nullptr, nullptr));
    check_cuda(cudaDeviceSynchronize(), "add_back_B_spline");
}

}  // namespace psum_b200

#endif
