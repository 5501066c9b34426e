/*
 * psum_pic.h -- C-ABI particle-kernel set of the B200 electrostatic PIC step.
 *
 * PSuM has no C ABI on the particle side: its step is header code,
 * `particle_group<P,Validator>::for_each` plus user lambdas
 * (src/particle_container/particle_group.hpp:169-221) over AoS
 * `tagged_struct{position, velocity}` particles, with CIC gather
 * (`interp_diff`, src/field/device_field.hpp:275-284), CIC deposit
 * (`add_back`, device_field.hpp:300-310) and cell binning
 * (src/particle_collision/grid_mapped_device_vector.hpp:47-87).  The
 * functions below are the plain-pointer entry points a PSuM `particle_group`
 * / `device_field` adapter binds to run the same step on one B200.
 *
 * Semantics kept from the reference:
 *   - grid: `simple_grid<D>` (src/field/simple_grid.hpp:16-307): node index
 *     last-dimension-fastest, node count cells+1 per axis, CIC base node
 *     `cN = floor((p-lo)*dr)`, reference cell key `c2i(nC(p))` with
 *     `nC = int((p-lo)*dr)` (truncation) for in-grid points only;
 *   - a periodic axis is PSuM's wrapping-node idiom (application/benchmark/TSI/main.cpp:94):
 *     `cells` cells between lower and upper, the node lattice wraps at
 *     cells+1 nodes, so the period is (cells+1)*dx;
 *   - an invalid (absorbed) particle exports with x = NaN
 *     (src/particle_container/validator.hpp:19-26);
 *   - E = -grad of the multilinear interpolant of phi (simple_interpolation.hpp:58-98).
 *
 * Layout choices of this implementation (not visible through the ABI):
 *   - SoA storage, sorted by cell with an int32 key;
 *   - PSUM_PIC_MIXED: int32 cell index + FP32 in-cell offset per axis,
 *     FP32 velocity (24 B per 2D3V particle, 28 B per 3D3V particle);
 *   - PSUM_PIC_FP64: FP64 absolute position and velocity (40 / 48 B);
 *   - deposition is exact integer (fixed-point) accumulation of per-particle
 *     CIC weights, so rho does not depend on particle order or thread timing.
 *
 * Bulk arguments named *_dev are device pointers; *_host are host pointers.
 * Every function returns a psum_status (include/psum_field_solver.h).
 * Work is enqueued on the context's stream (psum_pic_set_stream); every
 * *_dev input must be complete with respect to that stream when the call is
 * made (the library does not wait for other streams), and a *_dev argument
 * of an asynchronous call (push, step, rho, density) must stay valid and
 * unmodified until the stream reaches the call.  Calls that return host
 * data, and the loads, synchronise the context's stream before returning.
 */
#ifndef PSUM_B200_PIC_H
#define PSUM_B200_PIC_H

#include "psum_field_solver.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct psum_pic_grid_desc {
    int dim;            /* 1, 2 or 3 (1-D runs take the step's general path) */
    int cells[3];       /* simple_grid<D>::cell_num */
    double lower[3];    /* simple_grid<D>::lower_bounds */
    double upper[3];    /* simple_grid<D>::upper_bounds */
    int periodic[3];    /* 1: periodic axis (wrapping node lattice); 0: absorbing walls at lower/upper */
} psum_pic_grid_desc;

typedef struct psum_pic_species_desc {
    double charge;      /* q */
    double mass;        /* m */
    double weight;      /* macro-particle weight; deposit adds weight/cell_volume per particle */
} psum_pic_species_desc;

enum { PSUM_PIC_MIXED = 0, PSUM_PIC_FP64 = 1 };
enum { PSUM_PIC_LEAPFROG = 0, PSUM_PIC_BORIS = 1 };

typedef struct psum_pic_ctx psum_pic_ctx;

EXPORT int psum_pic_create(const psum_pic_grid_desc* grid, int precision, psum_pic_ctx** out);
EXPORT int psum_pic_destroy(psum_pic_ctx* ctx);
/* Run all later work of this context on `stream` (a cudaStream_t such as
 * cudaStreamLegacy or a user stream; NULL = the context's own stream). */
EXPORT int psum_pic_set_stream(psum_pic_ctx* ctx, void* stream);
/* Options as whitespace `key value` pairs (the solver option grammar):
 *   sort_interval N   re-sort by cell every N steps (default 1; 0 = never)
 *   diagnostics 0|1   sum the energy and charge diagnostics inside every step
 *                     (psum_pic_get_step_diagnostics; default 0)
 *   interp_order K    B-spline order of the step's deposit and gather (1 = CIC,
 *                     the default; 2-4 run the general path, TSI/main.cpp:28-29)
 *   fp64_fma 0|1      FP64 contexts: the kernel build with fused multiply-adds
 *                     (faster, not bit-exact with the oracle; default 0) */
EXPORT int psum_pic_set_options(psum_pic_ctx* ctx, const char* options);

/* Adds a species able to hold `capacity` particles; *id receives its index. */
EXPORT int psum_pic_add_species(psum_pic_ctx* ctx, const psum_pic_species_desc* sp,
                                unsigned long long capacity, int* id);
/* Replaces the species' particles by `n` particles given as FP64 SoA host
 * arrays pos_host[d*n+i] (d < dim) and vel_host[c*n+i] (c < 3), in the given
 * order (no sort).  Particles with non-finite x[0] are loaded as invalid.
 * Periodic coordinates are wrapped into the period; particles outside an
 * absorbing axis are loaded as invalid. */
EXPORT int psum_pic_load(psum_pic_ctx* ctx, int species, unsigned long long n,
                         const double* pos_host, const double* vel_host);
/* Same, from FP64 SoA device arrays (no host staging); returns after the
 * arrays have been consumed, so the caller may free them right away. */
EXPORT int psum_pic_load_device(psum_pic_ctx* ctx, int species, unsigned long long n,
                                const double* pos_dev, const double* vel_dev);
/* Adds `n` particles (FP64 SoA, as psum_pic_load) after the stored ones:
 * particle_group::insert (src/particle_container/particle_group.hpp:103-167),
 * which fills the group's invalid slots first; groups here are compacted,
 * so the new particles go to the end.  The species is unsorted afterwards
 * (the next psum_pic_sort or step re-sorts it).  As after psum_pic_load,
 * the charge accumulators still hold the last deposit: call
 * psum_pic_deposit before the next step.  PSUM_ERR_OVERFLOW beyond the
 * capacity, with nothing stored. */
EXPORT int psum_pic_append(psum_pic_ctx* ctx, int species, unsigned long long n,
                           const double* pos_host, const double* vel_host);
EXPORT int psum_pic_append_device(psum_pic_ctx* ctx, int species, unsigned long long n,
                                  const double* pos_dev, const double* vel_dev);
/* Current array length (valid + not yet compacted invalid) and valid count. */
EXPORT int psum_pic_count(psum_pic_ctx* ctx, int species, unsigned long long* n_stored,
                          unsigned long long* n_valid);
/* Copies the species state, in storage order, into FP64 SoA host arrays of
 * n_stored entries; invalid particles have pos[0] = NaN. */
EXPORT int psum_pic_get_state(psum_pic_ctx* ctx, int species, double* pos_host, double* vel_host);
/* Same, into FP64 SoA device arrays of n_stored entries (pos_dev[d*n + i],
 * vel_dev[c*n + i]); returns after the copy is complete.  These are the
 * positions the B-spline calls of psum_interp.h take. */
EXPORT int psum_pic_get_state_device(psum_pic_ctx* ctx, int species, double* pos_dev, double* vel_dev);
/* Internal cell key per stored particle (row-major over the internal cell
 * lattice; invalid = -1) into an int32 device array of n_stored entries. */
EXPORT int psum_pic_get_keys(psum_pic_ctx* ctx, int species, int* keys_dev);

/* Stable counting sort of every species by internal cell key (invalid
 * particles are dropped: this is also `compress`). */
EXPORT int psum_pic_sort(psum_pic_ctx* ctx);

/* Reference binning (grid_mapped_device_vector::update, :47-87) of one species:
 * keys_dev[i] = c2i(nC(p_i)) for in-grid particles, -1 otherwise (int64, n_stored);
 * counts_dev[c] (uint64, prod(cells)) particles per reference cell;
 * offsets_dev[c] (uint64, prod(cells)) exclusive prefix of counts;
 * perm_dev[s] (uint64, n_in_grid) = stored index of the particle in output slot s,
 * stable: ascending stored index within a cell.  *n_in_grid is returned. */
EXPORT int psum_pic_bin(psum_pic_ctx* ctx, int species, long long* keys_dev, unsigned long long* counts_dev,
                        unsigned long long* offsets_dev, unsigned long long* perm_dev,
                        unsigned long long* n_in_grid);

/* Recomputes the charge accumulators from the current positions (CIC). */
EXPORT int psum_pic_deposit(psum_pic_ctx* ctx);
/* rho_dev (FP64 node field) = background + sum_s charge_s*weight_s/cell_volume * n_s. */
EXPORT int psum_pic_rho(psum_pic_ctx* ctx, double background, double* rho_dev);
/* Per-species deposited particle count density n_s (no charge/background). */
EXPORT int psum_pic_density(psum_pic_ctx* ctx, int species, double* n_dev);

/* Gather E = -grad(phi) at every particle, push (leapfrog, or Boris with the
 * uniform field B[3]), apply the particle boundary, then deposit the new
 * positions into the charge accumulators.  phi_dev is an FP64 node field.
 * Absorbed particles become invalid and are counted per species, axis and
 * side into the context's loss counters (read with psum_pic_get_losses). */
EXPORT int psum_pic_push(psum_pic_ctx* ctx, const double* phi_dev, double dt, int pusher, const double* B);
/* losses_host[(s*dim + axis)*2 + side] since the last reset (side 0 = lower wall). */
EXPORT int psum_pic_get_losses(psum_pic_ctx* ctx, unsigned long long* losses_host, int reset);

/* One full electrostatic step through a solver handle obtained from this
 * library's func_table (cuda_multigrid32f_gpu / cuda_multigrid64_gpu):
 *   rho = background + deposited charge  ->  solve A phi = rho  ->  push + deposit
 *   -> re-sort when due.  phi_dev is the initial guess and the output field;
 * rho_dev is scratch that receives the right-hand side.  Asynchronous. */
EXPORT int psum_pic_step(psum_pic_ctx* ctx, psum_field_solver_handle solver, double background,
                         double* rho_dev, double* phi_dev, double dt, int pusher, const double* B);

/* With the fused sorted step (mixed precision, sort_interval 1), a step's
 * second pass (the re-sorted particle writes) runs on a stream of the
 * context after the step returns, so that the next step's charge density and
 * Poisson solve overlap it; every other function of this header that reads
 * or writes particle state orders the context's stream after it first
 * (psum_pic_get_losses does not need to: loss counts are final earlier).
 * psum_pic_join does only that: after it, work enqueued on the context's
 * stream sees the complete step, e.g. an event that closes a timed region.
 * No counterpart in the reference, whose push is synchronous. */
EXPORT int psum_pic_join(psum_pic_ctx* ctx);

/* Per-phase CUDA-event timing of psum_pic_step on the context's stream.
 * Phases: 0 rho, 1 Poisson solve, 2 gather+push+deposit, 3 sort.
 * get_timing returns accumulated milliseconds and phase executions since the
 * last reset (synchronises the stream). */
EXPORT int psum_pic_set_timing(psum_pic_ctx* ctx, int enable);
EXPORT int psum_pic_get_timing(psum_pic_ctx* ctx, double* ms_host, int* count_host, int reset);
/* The same for the first n_phases phases, including phase 4, the reduction of
 * the per-step diagnostics (option "diagnostics 1").  No counterpart in the
 * reference. */
EXPORT int psum_pic_get_phase_times(psum_pic_ctx* ctx, double* ms_host, int* count_host, int n_phases, int reset);

/* FP64 diagnostics (fixed-order reductions): out_host[s] = kinetic energy of
 * species s (sum 0.5*m*w*|v|^2); out_host[ns] = field energy
 * 0.5*eps*sum over edges (dphi/dx)^2 * cell_volume; out_host[ns+1] = total
 * deposited charge sum_s q_s w_s N_s (exact from the integer accumulators). */
EXPORT int psum_pic_diagnostics(psum_pic_ctx* ctx, const double* phi_dev, double epsilon, double* out_host);

/* The diagnostics of TSI's step loop (application/benchmark/TSI/main.cpp:132-146)
 * computed inside every psum_pic_step when the context has option
 * "diagnostics 1": the push sums the kinetic energy of the pushed particles
 * (FP64, before absorbed ones leave), the edge kernel sums the field energy of
 * the step's phi, and the charge density sums the particle charge it holds
 * (the deposit of the previous step); fixed-order reductions, no extra pass
 * over the particles.  Returns the last step's values in the layout of
 * psum_pic_diagnostics: out_host[s] kinetic energy of species s, out_host[ns]
 * field energy (times epsilon), out_host[ns+1] particle charge.  Errors with
 * PSUM_ERR_INVALID_ARGUMENT before such a step.  No counterpart in the
 * reference (its diagnostics are host loops over copies). */
EXPORT int psum_pic_get_step_diagnostics(psum_pic_ctx* ctx, double epsilon, double* out_host);

/* Error word of the device-side checks since the last call (bit set per
 * psum_status code: non-finite state, overflow, key out of range); resets it. */
EXPORT int psum_pic_device_errors(psum_pic_ctx* ctx, unsigned int* flags);

/* ---- Differentiable runs (no counterpart in the reference: PSuM has no
 * adjoint).  Device snapshots of a species' state for checkpoints, and the
 * discrete adjoint of one leapfrog step on the current state.  Positions are
 * in cell units (cell index + offset per axis), so lam_x is dL/ds. */

/* Size of a snapshot of `species` (stored count + state arrays at capacity). */
EXPORT int psum_pic_state_bytes(psum_pic_ctx* ctx, int species, unsigned long long* bytes);
/* Copy the species' current state into / out of a device buffer of
 * psum_pic_state_bytes bytes (stream-ordered device copies). */
EXPORT int psum_pic_save_state(psum_pic_ctx* ctx, int species, void* dst_dev);
EXPORT int psum_pic_restore_state(psum_pic_ctx* ctx, int species, const void* src_dev);

/* Adjoint of the leapfrog kick and move of `species` at its current state
 * (the state before the step), with the potential phi_dev the step gathered
 * from.  lam_x_dev ([dim][n]) and lam_v_dev ([3][n]) hold the adjoints of the
 * new positions and velocities on entry and of the old ones on exit (FP32
 * for PSUM_PIC_MIXED contexts, FP64 otherwise; n = the loaded count); the
 * deposit term is added by psum_pic_adjoint_deposit.  The adjoint of phi
 * (the scatter of the force adjoint to the nodes) is added to mu_dev
 * (FP64, one value per node) in exact fixed point. */
EXPORT int psum_pic_adjoint_push(psum_pic_ctx* ctx, int species, const double* phi_dev, double dt, void* lam_x_dev,
                                 void* lam_v_dev, double* mu_dev);
/* lam_x += (dL/drho)^T d rho/ds for `species` at its current state, given
 * nu_dev = dL/drho (FP64 per node): the gather of nu's CIC gradient. */
EXPORT int psum_pic_adjoint_deposit(psum_pic_ctx* ctx, int species, const double* nu_dev, void* lam_x_dev);

/* Allocation-free binning of caller-owned FP64 SoA device positions
 * (pos_dev[d*n+i]) on a grid: the same keys, per-cell counts, offsets,
 * stable permutation and in-grid count as psum_pic_bin, without a context
 * and without allocating device memory.  It has no counterpart in the
 * reference.  It exists for callers that cannot call cudaMalloc, e.g. a
 * PSuM build whose device memory belongs to another runtime's pool, or a
 * loop held to a fixed memory budget.  Its sort and scan scratch is one
 * file-scope device array (about 12.6 MB) that every GPU loading this
 * library keeps until the process exits; limits: n <= 262,144 particles and
 * at most 1,048,576 grid cells (larger sizes return
 * PSUM_ERR_INVALID_ARGUMENT).  The array belongs to the library's device
 * module: under CUDA's lazy module loading the driver reserves it when that
 * module is first used on a device, which is this call's first run there
 * unless another call of this library came first.  A caller with a fixed
 * device-memory budget should make one warm-up call (any size, e.g. n = 0)
 * outside the budgeted region.  The first call on a device also looks the
 * array's address up (cudaGetSymbolAddress); make that first call before any
 * stream capture.  All calls share the one array, so calls that overlap on the GPU
 * (other host threads, other streams) race; serialise them.  Work runs on
 * `stream` (a cudaStream_t, NULL = legacy default stream) and the call
 * returns after it has finished. */
EXPORT int psum_bin_positions_noalloc(const psum_pic_grid_desc* grid, unsigned long long n, const double* pos_dev,
                                      long long* keys_dev, unsigned long long* counts_dev,
                                      unsigned long long* offsets_dev, unsigned long long* perm_dev,
                                      unsigned long long* n_in_grid, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PSUM_B200_PIC_H */
