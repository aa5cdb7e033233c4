// Level-0 (fine) operator: matrix-free hex8 K.u on the voxel grid plus its sparse parts.
#pragma once
#include "common.cuh"
#include "element.cuh"

namespace feb {

// Device view of the level-0 operator in precision T.
//   nodes: full layout, grid nodes (x fastest) then split copies; vectors hold 3 T per node.
//   mat  : structured material per cell, x-fastest cell order, MatWidth values per cell; inactive
//          cells and cells touching split copies ("irregular") are zero here.
template <typename T>
struct FineView {
  int nx, ny, nz;          // cells
  int nxn, nyn, nzn;       // grid nodes per axis
  int64_t nnode;           // grid nodes
  int64_t ntotal;          // grid nodes + copies
  const T* dx; const T* dy; const T* dz;      // cell widths per axis
  const T* idx; const T* idy; const T* idz;   // inverses
  const T* mat;
  // irregular cells (touch split copies): x-fastest cell index, 8 node ids, material
  int nirr; const int* irr_cell; const int* irr_nodes; const T* irr_mat;
  // diagonal penalties: node, k[3]
  int npen; const int* pen_node; const T* pen_k;
  // sparse extra matrix, CSR over the dofs that have entries
  int nrow; const int* row_dof; const int* row_ptr; const int* col; const T* val;
};

// launch shape of the structured K.u kernel: warps per CTA (8, 12 or 16) and node planes per CTA
struct KuConfig {
  int ty = 16;
  int zchunk = 16;
};

template <typename T, int MODE>
void launch_fine_apply(const FineView<T>& F, const T* u, T* y, const int* skip, KuConfig cfg, cudaStream_t s);

// 3x3 diagonal blocks of the level-0 operator at every node (full layout), row-major [n][9].
template <int MODE>
void launch_fine_diag(const FineView<double>& F, double* D, cudaStream_t s);

// Dense matrix of the level-0 operator over the used dofs (cmap: node -> compact node index or -1), for
// problems whose level 0 is already the coarsest multigrid level.
template <int MODE>
void launch_dense_from_fine(const FineView<double>& F, const int* cmap, double* M, int nd, cudaStream_t s);

}  // namespace feb
