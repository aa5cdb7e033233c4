// Dense coarsest level (see dense.cu).
#pragma once
#include "common.cuh"
#include <algorithm>

namespace feb {

void launch_dense_from_stencil(const double* A, int nx, int ny, int nz, const int* cmap, double* M, int nd,
                               cudaStream_t s);
void launch_dense_add_terms(int nterms, const int* t_ptr, const int* t_dof, const double* t_val, const double* t_lam,
                            const int* cmap, double* M, int nd, cudaStream_t s);
void launch_dense_add_entries(int nent, const int* rdof, const int* cdof, const double* val, const int* cmap,
                              double* M, int nd, cudaStream_t s);
// In-place M <- M^-1 (symmetrised first); scratch: dense_scratch_doubles(nd); *status = FEB_ERR_COARSE on a
// non-positive pivot.
void launch_dense_invert(double* M, int nd, double* scratch, int* status, cudaStream_t s);
size_t dense_scratch_doubles(int nd);
// x = Minv b on the kept nodes (klist: node of compact index, cmap: compact index of node or -1; x is zeroed on
// the other nodes), one launch
template <typename T>
void launch_dense_solve(const double* Minv, int nd, const int* klist, const int* cmap, int64_t n, const T* b, T* x,
                        const int* skip, cudaStream_t s);

}  // namespace feb
