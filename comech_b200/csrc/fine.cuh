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
  // tensor-core path (FP32, equal cubic cells): B operand table, h/72 and the lambda factor (h/16 one-point,
  // h/72 integrated), word set to 1 when a bounded wait gave up
  const void* tc_b = nullptr;
  float tc_hmu = 0.f, tc_hlam = 0.f;
  int* tc_status = nullptr;
};

// launch shape of the structured K.u kernel: warps per CTA (8, 12 or 16) and node planes per CTA
struct KuConfig {
  int ty = 16;
  int zchunk = 16;
  int tc = 0;              // 1: tensor-core kernel (zchunk planes per CTA; ty unused)
};

template <typename T, int MODE>
void launch_fine_apply(const FineView<T>& F, const T* u, T* y, const int* skip, KuConfig cfg, cudaStream_t s);

// Tensor-core K.u of the regular cells (MODE ISO_SRI or ISO_FULL, equal cubic cells, FP32): operand columns
// N of the B table (2 faces x 2 node rows x N rows x 8 BF16), kernel attributes (once per process), launch.
template <int MODE> int tc_columns();
template <int MODE> cudaError_t prepare_fine_tc();
template <int MODE>
void launch_fine_struct_tc(const FineView<float>& F, const float* u, float* y, const int* skip, int zchunk,
                           cudaStream_t s);
// K_lambda and K_mu of the unit cube, out[2][24][24] (dof 3 l + c), with the model's integration rule
template <int MODE> void launch_unit_element(double* out, cudaStream_t s);

// 3x3 diagonal blocks of the level-0 operator at every node (full layout), row-major [n][9].
template <int MODE>
void launch_fine_diag(const FineView<double>& F, double* D, cudaStream_t s);

// Dense matrix of the level-0 operator over the used dofs (cmap: node -> compact node index or -1), for
// problems whose level 0 is already the coarsest multigrid level.
template <int MODE>
void launch_dense_from_fine(const FineView<double>& F, const int* cmap, double* M, int nd, cudaStream_t s);

}  // namespace feb
