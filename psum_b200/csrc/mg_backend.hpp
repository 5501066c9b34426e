// mg_backend.hpp -- internal interface of the multigrid backends, used by the
// particle step (psum_pic_step) to solve through a func_table handle without
// going back through the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace psum_b200 {

constexpr uint32_t kSolverMagic = 0x4d473230u;   // "MG20"

struct SolverBase;
struct MGState;

SolverBase* create_solver(int precision);
SolverBase* solver_from_handle(void* h);     // throws for foreign handles
void solver_set_options(SolverBase* s, const char* options);
void solver_set_matrix(SolverBase* s, unsigned long long n_row, unsigned long long n_col, unsigned long long nnz,
                       const unsigned long long* rows, const unsigned long long* cols, const double* vals);
void solver_set_source(SolverBase* s, bool replace, unsigned long long n, const unsigned long long* idx,
                       const double* v);
void solver_solve_async(SolverBase* s, double* b, double* x, cudaStream_t stream);
void solver_destroy(SolverBase* s);
cudaStream_t solver_stream(SolverBase* s);

}  // namespace psum_b200
