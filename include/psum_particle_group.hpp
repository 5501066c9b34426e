/*
 * psum_particle_group.hpp -- header-only C++ adapter with the member
 * functions of PSuM's particle_group (src/particle_container/particle_group.hpp:11-271)
 * over one species of a psum_pic context (include/psum_pic.h).
 *
 * PSuM keeps a group as an AoS device vector of tagged_struct{position,
 * velocity} particles plus a list of invalid slots; an absorbed particle
 * stays in place with a NaN position until compress() (validator.hpp:19-26).
 * This adapter keeps PSuM's observable behaviour over the library's SoA,
 * cell-sorted storage:
 *
 *   size()       valid particles                  (particle_group.hpp:32-34)
 *   stored()     valid + not yet compacted invalid (data_.size())
 *   capacity()   the species capacity              (particle_group.hpp:36-38)
 *   clear()      no particles                      (particle_group.hpp:40-43)
 *   insert(...)  add particles; invalid input particles are dropped, as the
 *                validating insert does             (particle_group.hpp:103-167)
 *   compress()   drop invalid slots; the library's compaction is its cell
 *                sort, so the order afterwards is by cell (stable within a
 *                cell) where PSuM keeps the storage order (particle_group.hpp:223-238)
 *   content()    the stored particles, invalid ones with a NaN position,
 *                in storage order (get_content, particle_group.hpp:254-256)
 *
 * shuffle() and shrink() are not provided: the storage order is the cell
 * order maintained by the step, and the capacity is fixed when the species
 * is added.  Errors throw psum_b200::error with the library's status and
 * message.  Link against libpsum_b200.so.
 */
#ifndef PSUM_B200_PARTICLE_GROUP_HPP
#define PSUM_B200_PARTICLE_GROUP_HPP

#include <cmath>
#include <cstddef>
#include <stdexcept>
#include <string>
#include <vector>

#include "psum_pic.h"

namespace psum_b200 {

class error : public std::runtime_error {
public:
    error(int status, const std::string& what) : std::runtime_error(what), status_(status) {}
    int status() const { return status_; }

private:
    int status_;
};

inline void check(int status) {
    if (status != PSUM_OK) {
        const char* m = psum_last_error();
        throw error(status, m ? m : "psum_b200 error");
    }
}

/* One particle: tagged_struct<position<D>, velocity> of the reference's
 * examples (position: D doubles, velocity: 3 doubles). */
template <int D>
struct particle {
    double position[D];
    double velocity[3];
};

/* A species of `ctx` seen as a PSuM particle_group of `particle<D>`.  The
 * group does not own the context; the context must outlive it. */
template <int D>
class particle_group {
public:
    using value_type = particle<D>;

    /* Adds a new species to `ctx` with room for `capacity` particles. */
    particle_group(psum_pic_ctx* ctx, const psum_pic_species_desc& desc, std::size_t capacity)
        : ctx_(ctx), capacity_(capacity) {
        check(psum_pic_add_species(ctx_, &desc, capacity, &species_));
    }

    /* Wraps species `species` of `ctx` (added with `capacity`). */
    particle_group(psum_pic_ctx* ctx, int species, std::size_t capacity)
        : ctx_(ctx), species_(species), capacity_(capacity) {}

    particle_group(const particle_group&) = delete;
    particle_group& operator=(const particle_group&) = delete;

    int species() const { return species_; }
    psum_pic_ctx* context() const { return ctx_; }
    std::size_t capacity() const { return capacity_; }

    std::size_t size() const {
        unsigned long long stored = 0, valid = 0;
        check(psum_pic_count(ctx_, species_, &stored, &valid));
        return (std::size_t)valid;
    }

    std::size_t stored() const {
        unsigned long long stored = 0;
        check(psum_pic_count(ctx_, species_, &stored, nullptr));
        return (std::size_t)stored;
    }

    void clear() { check(psum_pic_load(ctx_, species_, 0, nullptr, nullptr)); }

    /* Validating insert of host particles: those with a non-finite position
     * are dropped first (particle_group.hpp:147-159). */
    void insert(const std::vector<value_type>& particles) {
        std::vector<double> pos, vel;
        const std::size_t n = to_soa(particles, pos, vel);
        if (n == 0) return;
        check(psum_pic_append(ctx_, species_, n, pos.data(), vel.data()));
    }

    /* Insert of FP64 SoA host arrays pos[d*n+i], vel[c*n+i] without the
     * validation pass (particle_group.hpp:103-145 with NeedValidation ==
     * false); a particle whose position is outside an absorbing axis is
     * stored as invalid. */
    void insert_soa(std::size_t n, const double* pos, const double* vel) {
        if (n == 0) return;
        check(psum_pic_append(ctx_, species_, n, pos, vel));
    }

    /* The same from FP64 SoA device arrays. */
    void insert_soa_device(std::size_t n, const double* pos_dev, const double* vel_dev) {
        if (n == 0) return;
        check(psum_pic_append_device(ctx_, species_, n, pos_dev, vel_dev));
    }

    /* Drops the invalid slots (with the cell sort of every species of the
     * context, which is how the library compacts). */
    void compress() { check(psum_pic_sort(ctx_)); }

    /* All stored particles in storage order; invalid ones have a NaN
     * position[0], as the reference's validator marks them. */
    std::vector<value_type> content() const {
        const std::size_t n = stored();
        std::vector<double> pos((std::size_t)D * n), vel(3 * n);
        std::vector<value_type> out(n);
        if (n == 0) return out;
        check(psum_pic_get_state(ctx_, species_, pos.data(), vel.data()));
        for (std::size_t i = 0; i < n; ++i) {
            for (int d = 0; d < D; ++d) out[i].position[d] = pos[(std::size_t)d * n + i];
            for (int c = 0; c < 3; ++c) out[i].velocity[c] = vel[(std::size_t)c * n + i];
        }
        return out;
    }

    static bool is_valid(const value_type& p) { return std::isfinite(p.position[0]); }

private:
    static std::size_t to_soa(const std::vector<value_type>& in, std::vector<double>& pos, std::vector<double>& vel) {
        std::size_t n = 0;
        for (const auto& p : in) n += is_valid(p);
        pos.assign((std::size_t)D * n, 0.0);
        vel.assign(3 * n, 0.0);
        std::size_t j = 0;
        for (const auto& p : in) {
            if (!is_valid(p)) continue;
            for (int d = 0; d < D; ++d) pos[(std::size_t)d * n + j] = p.position[d];
            for (int c = 0; c < 3; ++c) vel[(std::size_t)c * n + j] = p.velocity[c];
            ++j;
        }
        return n;
    }

    psum_pic_ctx* ctx_;
    int species_ = -1;
    std::size_t capacity_;
};

}  // namespace psum_b200

#endif
