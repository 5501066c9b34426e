/*
 * psum_field_solver.h -- linear-solver plugin ABI of the B200 backend.
 *
 * The first block is layout- and signature-compatible with PSuM's solver
 * plugin interface (src/field_solver/register/interface.h:4-28): the same
 * seven-entry `func_table`, the same typedefs, and the same two registry
 * entry points `register_solver` / `get_solver_funcs`
 * (src/field_solver/register/registry.cpp:12-21).  A PSuM build can link this
 * library in place of its own registry and obtain the B200 backends by name:
 *
 *   "cuda_multigrid32f_gpu"  FP32 V-cycles inside FP64 iterative refinement
 *                            (replaces sycl_multigrid32f_gpu,
 *                             src/field_solver/implements/sycl_multigrid32f_gpu.cpp:106-160)
 *   "cuda_multigrid64_gpu"   all-FP64 V-cycles (replaces cuda_multigrid_gpu /
 *                             sycl_multigrid_gpu, cuda_multigrid_gpu.cu:140-180)
 *
 * As in the reference, `solve(b, x)` receives DEVICE pointers, modifies `b`
 * in place (add-back, then replace), and treats `x` as the initial guess on
 * entry and the solution on exit.  The func_table entries report errors by
 * throwing std::runtime_error / std::invalid_argument, exactly like the
 * reference backends; C callers that cannot catch C++ exceptions use the
 * status-returning `psum_mg_*` entry points in the second block instead.
 */
#ifndef PSUM_B200_FIELD_SOLVER_H
#define PSUM_B200_FIELD_SOLVER_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- block 1: PSuM-compatible plugin ABI (interface.h:4-28) ---- */
typedef void* psum_field_solver_handle;
typedef psum_field_solver_handle (*solver_init_func)(void);
typedef void (*solver_set_matrix_func)(psum_field_solver_handle, unsigned long long, unsigned long long,
                                       unsigned long long, unsigned long long*, unsigned long long*, double*);
typedef void (*solver_solve_func)(psum_field_solver_handle, double*, double*);
typedef void (*solver_set_options_func)(psum_field_solver_handle, const char*);
typedef void (*solver_set_source_replace_func)(psum_field_solver_handle, unsigned long long, unsigned long long*, double*);
typedef void (*solver_set_source_addback_func)(psum_field_solver_handle, unsigned long long, unsigned long long*, double*);
typedef void (*solver_free_func)(psum_field_solver_handle);

struct func_table {
    solver_init_func init;
    solver_set_matrix_func set_matrix;
    solver_solve_func solve;
    solver_set_options_func set_options;
    solver_set_source_replace_func set_source_replace;
    solver_set_source_addback_func set_source_addback;
    solver_free_func free;
};

#ifndef EXPORT
#define EXPORT __attribute__((visibility("default")))
#endif

/* registry.cpp:12-15 -- register (or replace) a backend under `name`. */
EXPORT void register_solver(const char* name, struct func_table table);
/* registry.cpp:17-21 -- unknown names return a table whose `init` is NULL. */
EXPORT struct func_table get_solver_funcs(const char* name);

/* ---- block 2: status-returning entry points (no C++ exceptions cross) ---- */

/* Status codes shared by every psum_* entry point of this library. */
typedef enum psum_status {
    PSUM_OK = 0,
    PSUM_ERR_INVALID_ARGUMENT = 1, /* bad option string, size mismatch, null pointer */
    PSUM_ERR_NOT_READY = 2,        /* call order violated (e.g. solve before set_matrix) */
    PSUM_ERR_CUDA = 3,             /* a CUDA runtime call failed */
    PSUM_ERR_NOT_CONVERGED = 4,    /* max_cycles reached above `tol` */
    PSUM_ERR_DIVERGED = 5,         /* residual became non-finite or grew past the divergence guard */
    PSUM_ERR_OVERFLOW = 6,         /* a device buffer or counter exceeded its capacity */
    PSUM_ERR_NONFINITE = 7,        /* non-finite value found in an input */
    PSUM_ERR_INTERNAL = 8
} psum_status;

/* Message of the last failing psum_* call on this thread ("" if none). */
EXPORT const char* psum_last_error(void);
/* Number of CUDA kernels this library has launched in this process. */
EXPORT unsigned long long psum_kernel_launches(void);

/* Mirrors of the func_table entries that return a status instead of throwing.
 * `kind` is a registered backend name; *out receives the handle. */
EXPORT int psum_mg_create(const char* kind, psum_field_solver_handle* out);
EXPORT int psum_mg_set_options(psum_field_solver_handle h, const char* options);
EXPORT int psum_mg_set_matrix(psum_field_solver_handle h, unsigned long long n_row, unsigned long long n_col,
                              unsigned long long nnz, const unsigned long long* rows,
                              const unsigned long long* cols, const double* vals);
EXPORT int psum_mg_set_source_replace(psum_field_solver_handle h, unsigned long long n,
                                      const unsigned long long* idx, const double* values);
EXPORT int psum_mg_set_source_addback(psum_field_solver_handle h, unsigned long long n,
                                      const unsigned long long* idx, const double* values);
/* Synchronous solve; device pointers; same semantics as func_table.solve.
 * Returns PSUM_ERR_NOT_CONVERGED when a `tol` option is set and was not met
 * within `max_cycles` (x still holds the last iterate). */
EXPORT int psum_mg_solve(psum_field_solver_handle h, double* b_dev, double* x_dev);
/* Asynchronous solve on `stream` (a cudaStream_t, NULL = the handle's own
 * stream).  No host synchronisation; convergence is decided on the device.
 * Read the outcome later with psum_mg_last_stats. */
EXPORT int psum_mg_solve_async(psum_field_solver_handle h, double* b_dev, double* x_dev, void* stream);
/* Outcome of the last solve: V-cycles run, refinement steps run, final and
 * initial relative residual ||b - A x||_2 / ||b||_2 (FP64). Synchronises. */
EXPORT int psum_mg_last_stats(psum_field_solver_handle h, int* cycles, int* refinements,
                              double* rel_residual, double* initial_rel_residual);
/* Number of levels actually built and the coarsest level's size. */
EXPORT int psum_mg_hierarchy_info(psum_field_solver_handle h, int* levels, unsigned long long* coarse_rows,
                                  unsigned long long* exception_rows_level0);
/* Level vectors the TMA-staged sweep kernel has read so far (one tensor map
 * each): 0 with option `tma 0`, before the first solve, or when no level
 * qualifies (3-D, at least 2^16 rows, rows a multiple of 16 bytes long). */
EXPORT int psum_mg_tma_sweeps(psum_field_solver_handle h, int* level_vectors);
EXPORT int psum_mg_destroy(psum_field_solver_handle h);

/* ---- block 3: host-side FD operator assembly (the Poisson frontends) ----
 * Restates Poisson_solver_{2,3}d::_init_impl (Poisson_solver_2d.hpp:182-410,
 * Poisson_solver_3d.hpp:178-349) for Cartesian grids with uniform epsilon,
 * Dirichlet nodes given by index, and cyclic wrap of every other node at
 * (cells+1) nodes per axis.  Output is COO in the column-major order the
 * frontend hands to set_matrix (Poisson_solver_2d.hpp:387-404).
 * Call once with rows == NULL to get *nnz, then again with buffers. */
EXPORT int psum_poisson_assemble(int dim, const int* cells, const double* lower, const double* upper,
                                 double epsilon, unsigned long long n_fixed, const unsigned long long* fixed_nodes,
                                 unsigned long long* nnz, unsigned long long* rows, unsigned long long* cols,
                                 double* vals);

#ifdef __cplusplus
}
#endif

#endif /* PSUM_B200_FIELD_SOLVER_H */
