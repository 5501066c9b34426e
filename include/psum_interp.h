/*
 * psum_interp.h -- node-field interpolation at B-spline orders 1-4 on the
 * device: the value gather, the gradient gather and the deposit of
 * src/field/higher_order_interp.hpp:196-247 (interp_B_spline,
 * interp_diff_B_spline, add_back_B_spline; order 1 is the linear
 * interp / interp_diff / add_back of src/field/device_field.hpp:250-310).
 *
 * PSuM calls these per particle inside a particle_group::for_each lambda on
 * a device_field accessor; here one call handles n positions given as an
 * FP64 SoA device array pos_dev[d*n + i] (d < dim) over an FP64 node field of
 * prod(cells + 1) nodes (last dimension fastest, simple_grid::n2i).  The grid
 * is a psum_pic_grid_desc (dim 1, 2 or 3; the periodic flags are not used:
 * like the reference, every support stencil wraps once by +-(cells + 1)
 * nodes on every axis).
 *
 * Support: order + 1 nodes per axis, centred on the nearest node for orders
 * 2 and 4 and starting at the corner node for orders 1 and 3
 * (simple_grid.hpp:316-397).  A position that is not finite, or whose
 * stencil stays outside the node range after the one wrap (more than about a
 * period away; undefined in the reference), is skipped: the gathers write
 * NaN for it, the deposit adds nothing, and *skipped_dev (optional, device
 * counter) is incremented.
 *
 * Numerics: the gathers sum the full tensor product in FP64 (no 1e-10 skip of
 * small weights, which changes a result by at most 1e-10 * sum|field| over
 * the skipped nodes); the deposit keeps the skip and accumulates weights in
 * 64-bit fixed point with psum_bspline_deposit_bits(n) fraction bits, so its
 * result does not depend on the order of the positions.
 *
 * All calls are asynchronous on `stream` (a cudaStream_t; NULL = the legacy
 * default stream) and return a psum_status.
 */
#ifndef PSUM_B200_INTERP_H
#define PSUM_B200_INTERP_H

#include "psum_pic.h"

#ifdef __cplusplus
extern "C" {
#endif

/* out_dev[i] = sum_k field[node_k] * W_k(pos_i)   (interp_B_spline<order>) */
EXPORT int psum_interp_bspline(const psum_pic_grid_desc* grid, int order, unsigned long long n,
                               const double* pos_dev, const double* field_dev, double* out_dev,
                               unsigned long long* skipped_dev, void* stream);
/* grad_dev[d*n + i] = d/dx_d of the interpolant at pos_i   (interp_diff_B_spline<order>;
 * E = -grad for a potential) */
EXPORT int psum_interp_diff_bspline(const psum_pic_grid_desc* grid, int order, unsigned long long n,
                                    const double* pos_dev, const double* field_dev, double* grad_dev,
                                    unsigned long long* skipped_dev, void* stream);
/* field_dev[node_k] += weight * W_k(pos_i) for every position   (add_back_B_spline<order>).
 * scratch_dev: prod(cells + 1) 64-bit words of device memory, or NULL to
 * let the call allocate them from the stream-ordered pool. */
EXPORT int psum_add_back_bspline(const psum_pic_grid_desc* grid, int order, unsigned long long n,
                                 const double* pos_dev, double weight, double* field_dev, void* scratch_dev,
                                 unsigned long long* skipped_dev, void* stream);
/* Fraction bits F of the deposit's fixed point for n positions:
 * min(40, 62 - ceil(log2(n + 1))); each weight is rounded to a multiple of 2^-F. */
EXPORT int psum_bspline_deposit_bits(unsigned long long n, int* bits);

#ifdef __cplusplus
}
#endif

#endif
