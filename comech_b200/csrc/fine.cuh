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

// Sparse part of the level-0 operator only (irregular cells, penalties, extra entries), added with atomics
// into acc (3 per node).
template <typename T, int MODE>
void launch_fine_sparse_into(const FineView<T>& F, const T* u, T* acc, const int* skip, cudaStream_t s);

// ------------------------------------------------------------------------------------------------ paired K.u
// Operator of the paired-row kernel (fine_pair.cu): regular cells by 7-bit material ids, the sparse part
// through the accumulator tsp (zero between products), the smoother update fused in the epilogue.
constexpr int kMaxMatIds = 128;   // ids 1..127; 0 = no regular cell

template <typename T>
struct PairView {
  int nx, ny, nz;            // cells
  int nxn, nyn, nzn;         // grid nodes per axis
  int mp;                    // row pairs per (x, z) column: nyn / 2 + 1 (rows 2m-1, 2m)
  int64_t nnode, ntotal;     // grid nodes; grid nodes + split copies
  const uint16_t* cellpair;  // [nzn][mp][nxn]: per row byte bits 0-6 material id, bit 7 node is special
  const double* mtab;        // [kMaxMatIds][W] material values of the ids (FP64)
  int nmat;                  // ids in use are < nmat
  bool cube;                 // equal cubic cells of edge h, SRI model: reduced modal core
  double h;
  const T* dx; const T* dy; const T* dz;      // cell widths per axis (general core)
  const T* idx; const T* idy; const T* idz;
  T* tsp;                    // sparse-part accumulator, 3 per node (ntotal), zero between products
  const T* dinv6;            // symmetric block-Jacobi inverse [6][ntotal]: 00 11 22 01 02 12
};

struct LevelParams;
// Smoother epilogue of one product t = K u (u the direction d of the step):
//   r = r_in - t            -> r_out (if given)
//   d' = a1 u + a2 Dinv r   -> d_out (if given);  x_out = x_in + d' (x_in may be null: zero)
// with (a1, a2) = (0, c_init) for k < 0 and (a1[k], a2[k]) of the level's Chebyshev parameters otherwise.
// With neither d_out nor x_out the step is the residual update r_out = r_in - K u (lp may then be null).
template <typename T>
struct SmoothArgs {
  const T* r_in = nullptr;
  T* r_out = nullptr;
  const T* x_in = nullptr;
  T* x_out = nullptr;
  T* d_out = nullptr;
  double* x_out64 = nullptr;   // the new iterate in FP64 (instead of, or besides, x_out): the V-cycle's result
  const LevelParams* lp = nullptr;
  int k = -1;
  __host__ __device__ bool updates() const { return d_out || x_out || x_out64; }
};

struct PairConfig {
  int wy = 16;            // warps per CTA of products (2 node rows each); 16 only on the cubic SRI path in FP32
  int zchunk = 16;        // node planes per CTA of products
  int zchunk_smooth = 16; // node planes per CTA of the smoothing steps (always 8 warps per CTA)
};

// y = K u (S null) or the smoother step S; returns a status
template <typename T, int MODE>
int launch_fine_pair(const PairView<T>& F, const FineView<T>& G, const T* u, T* y, const SmoothArgs<T>* S,
                     const int* skip, PairConfig cfg, cudaStream_t s);
// sets the shared-memory limits of every paired-kernel variant of this model on the current device (call
// before any stream capture)
int prepare_fine_pair(int mode, bool cube);
// resident CTAs per SM of the paired kernel (smoothing variant) and its x-y tiles per node plane
template <typename T>
int fine_pair_blocks_per_sm(int mode, bool cube, int wy, bool smooth);
int fine_pair_tiles_xy(int nxn, int nyn, int wy);
template <int W>
void launch_mat_ids(const double* mat_s, int64_t ncell, unsigned long long* keys, double* vals, uint8_t* ids,
                    int* status, cudaStream_t s);
void launch_flag_nodes(const int* pen_node, int npen, const int* irr_nodes, int nirr, const int* row_dof, int nrow,
                       int64_t nnode, uint8_t* flag, cudaStream_t s);
template <int W>
void launch_pack_pairs(int nx, int ny, int nz, int mp, const uint8_t* ids, const uint8_t* flag, const double* mat_s,
                       const double* vals, uint16_t* cellpair, int* status, cudaStream_t s);
template <typename T>
void launch_dinv6(const double* D9, int64_t n, T* out, cudaStream_t s);
template <typename T>
void launch_cheb_first6(const T* b, const T* D6, const LevelParams* lp, T* d, T* x, int64_t n, const int* skip,
                        cudaStream_t s);

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
