// Coarse multigrid levels: 27-point 3x3-block stencils on structured node grids, structured transfers,
// and the Galerkin products P^T A P built on the device.
#pragma once
#include <cuda_fp16.h>

#include "common.cuh"
#include "fine.cuh"
#include "vec.cuh"

namespace feb {

// 1-D linear prolongation of one axis from every other node plus the last one (fe/gmg.py:7-26).
struct AxisDev {
  int nf, nc;                      // fine / coarse node counts
  const int* ca; const int* cb;    // per fine node: coarse neighbours a <= b (a == b for coincident nodes)
  const double* wa; const double* wb;
  const int* cidx;                 // per coarse node: fine node index
  const int* iv_first;             // per coarse interval [J, J+1]: first fine cell
  const int* iv_count;             //   and number of fine cells (1 or 2)
};

struct TransferDev {
  AxisDev ax[3];
  int even = 0;   // 1: every axis coarsens 2 n - 1 -> n nodes with weights 1 and 1/2 (uniform spacing, even cell
                  // counts); the transfers then index directly instead of reading the axis tables
  // even coarsening of a level with split copies: per coarse node J the copies that restrict into it,
  // entries cp_ptr[J] .. cp_ptr[J+1] of (copy index, weight), so that the restriction gathers them (no atomics)
  const int* cp_ptr = nullptr;
  const int* cp_copy = nullptr;
  const double* cp_w = nullptr;
};

// Structured level (>= 1): nodes nx*ny*nz (x fastest), stencil A[o*9 + 3r + c][n], o = (dx+1) + 3(dy+1) + 9(dz+1)
template <typename T>
struct StencilView {
  int nx, ny, nz;
  int64_t n;
  const T* A;
  // sparse remainder (entries the stencil cannot hold), CSR over dofs with entries
  int nrow; const int* row_dof; const int* row_ptr; const int* col; const T* val;
};

template <typename T>
void launch_stencil_apply(const StencilView<T>& L, const T* u, T* y, const int* skip, cudaStream_t s);

// Symmetric half storage of a stencil level: blocks of the offsets o = 13..26 (self and the 13 "forward"
// neighbours) as S[(o-13)*9 + 3r + c][p]; the block of a backward offset o' < 13 is the transpose of the
// forward block stored at the neighbour.  The node axis p is row-padded: p = i + nxp (j + ny k) with
// nxp = nx rounded up to a multiple of 4 (padding zero), so that every row of every plane starts 16-byte
// aligned.  Entries the stencil cannot hold are a per-node CSR (natural node ids):
// entries node_ptr[n] .. node_ptr[n+1] with row component ent_r, column dof ent_col, value ent_v.
__host__ __device__ inline int sym_nxp(int nx) { return (nx + 3) & ~3; }
__host__ __device__ inline int64_t sym_np(int nx, int ny, int nz) { return (int64_t)sym_nxp(nx) * ny * nz; }

template <typename T>
struct SymView {
  int nx, ny, nz;
  int64_t n;
  int nxp = 0;             // padded row length of S
  int64_t np = 0;          // padded node count: the stride of S's planes
  int slots = 0;           // the product's slot index: 0 compile-time in FP32, run-time in FP64; 1 run-time;
                           // 2 compile-time
  const T* S;
  const int* node_ptr;     // nullptr when there are no such entries
  const int8_t* ent_r;
  const int* ent_col;
  const T* ent_v;
  const T* Dinv;           // block-Jacobi inverse, SoA [9][n]
  // rank-1 terms lam_t v_t v_t^T (non-local springs projected to this level): entries t_ptr[t] .. t_ptr[t+1]
  // of v_t as (dof, value); per node, the (term, 3 components of v_t at the node) pairs of the terms that
  // touch it: tn_ptr[n] .. tn_ptr[n+1]
  const int* tn_ptr;       // nullptr when the level has no terms
  const int* tn_term;
  const T* tn_coef;
  const int* t_ptr;
  const int* t_dof;
  const T* t_val;
  const T* t_lam;
  int nterms = 0;
  T* tdot = nullptr;        // per term lam_t v_t.u of the current product (formed by k_term_dots before k_sym)
  // compressed stencil: tag[n] > 0 marks a node whose stored half stencil is lam pat[0] + mu pat[1] with
  // (lam, mu) = tmat[2 tag], tmat[2 tag + 1] (all cells around it of one material); such blocks are formed
  // on the fly instead of read.  tag == nullptr: every block is read.
  const uint8_t* tag = nullptr;
  const T* tmat = nullptr;  // [128][2]
  const T* pat = nullptr;   // [2][126]
  // 16-bit storage (FP32 products only): Sh[i] = S[i] / hscale[0] as FP16, hscale a power of two chosen so that
  // the level's largest entry lands below 2^15; the product accumulates in FP32 and is scaled once.  Sh ==
  // nullptr: S is read.
  const __half* Sh = nullptr;
  const float* hscale = nullptr;
};

// Fused level kernels: EPI_APPLY y = A u; EPI_RESID r = b - A u; EPI_CHEB Chebyshev step with ping-pong
// directions: t = A d_in, r -= t, d_out = a1 d_in + a2 Dinv r, x += d_out.
enum SymEpi : int { EPI_APPLY = 0, EPI_RESID = 1, EPI_CHEB = 2 };
struct LevelParams;
// tdot_in: the rank-1 term dots of u, formed by u's producer (TermAcc); null: a k_term_dots pass forms them
// first.  acc (EPI_CHEB): the dots of the new direction d_out are accumulated for the next product.
template <typename T>
void launch_sym(const SymView<T>& L, int epi, const T* u, T* y, const T* b, T* r, T* d_out, T* x,
                const LevelParams* lp, int k, const int* skip, cudaStream_t s, const T* tdot_in = nullptr,
                const TermAcc<T>& acc = TermAcc<T>());
// full [243][n] FP64 stencil of an nx x ny x nz level -> row-padded half storage in T ([126][sym_np])
template <typename T>
void launch_stencil_to_sym(const double* A, int nx, int ny, int nz, T* S, cudaStream_t s);
// FP64 half storage S64 ([126][sym_np]) -> FP16 scaled by a power of two: amax[0] (a scratch word) gets the
// largest |entry|, hscale[0] the scale 2^e with amax < 2^(e + 15), Sh the entries divided by it
void launch_sym_to_half(const double* S64, int nx, int ny, int nz, unsigned* amax, float* hscale, __half* Sh,
                        cudaStream_t s);

template <typename T>
void launch_csr_add(int nrow, const int* row_dof, const int* row_ptr, const int* col, const T* val, const T* u, T* y,
                    const int* skip, cudaStream_t s);

// r_c = P^T r_f.  Fine level given by its grid dims; copies (ids >= nnode) are folded through `orig`.
// zero[0 .. nzero): cleared by the same launch (the coarse level's term-dot buffers of this V-cycle).
template <typename T>
void launch_restrict(const TransferDev& P, int fnx, int fny, int fnz, int64_t fnnode, int64_t fntotal,
                     const int* orig_copy, const T* rf, T* rc, const int* skip, cudaStream_t s, T* zero = nullptr,
                     int nzero = 0);

// x_f += P x_c on used fine nodes (copies take their grid node's value).
// acc: the term dots of the added P x_c (the fine level's iterate changes by it) are accumulated
template <typename T>
void launch_prolong_add(const TransferDev& P, int fnx, int fny, int fnz, int64_t fnnode, int64_t fntotal,
                        const int* orig_copy, const uint8_t* used, const T* xc, T* xf, const int* skip,
                        cudaStream_t s, const TermAcc<T>& acc = TermAcc<T>());

// One axis pass of the separable Galerkin product P^T A P of a [243][n] stencil: axis d of the input grid
// (inx, iny, inz) coarsened by ax to the output grid (onx, ony, onz).
void launch_galerkin_axis(const AxisDev& ax, int d, const double* Ain, int inx, int iny, int inz, double* Aout,
                          int onx, int ony, int onz, cudaStream_t s);

// kept[J] = some used fine node interpolates from coarse node J (fe/gmg.py:95)
void launch_kept_mask(const TransferDev& P, const uint8_t* used_f, uint8_t* kept_c, cudaStream_t s);

// Level-1 stencil from the fine cells (P^T K_cells P), KeC scratch: ncoarse_cells x 576 doubles.
template <int MODE>
void launch_galerkin_cells(const FineView<double>& F, const double* mat_all, const TransferDev& P, double* KeC,
                           double* A1, int cnx, int cny, int cnz, cudaStream_t s);

// Level-1 stencil of a uniform fine grid (cell widths a, b, c) with even cell counts, isotropic models: summed
// directly from the fine cells' (lam, mu) and 16 constant sub-cell matrices (basis: 16 x 576 doubles of scratch).
template <int MODE>
int launch_galerkin_direct(const double* mat_all, int fnx, int fny, double a, double b, double c, double* basis,
                           double* A1, int cnx, int cny, int cnz, cudaStream_t s);

// Interior half-stencil patterns of the uniform level-1 node from the Galerkin basis of
// launch_galerkin_direct: pat[m][126] (m = 0 lam, 1 mu), same layout as the half storage.
void launch_sym_pattern(const double* basis, double* pat, cudaStream_t s);
// Tags of the compressed level-1 stencil: node J gets the material id of fine cell (2 jx, 2 jy, 2 jz) (read
// from the paired kernel's cell-pair words) when its stored FP64 half stencil S64 (row-padded) equals
// lam pat[0] + mu pat[1] to 1e-12 (relative), else 0.
void launch_sym_tags(const double* S64, int cnx, int cny, int cnz, const uint16_t* cellpair, int fnxn, int mp,
                     const double* mtab, const double* pat, uint8_t* tag, cudaStream_t s);

// Fold diagonal penalties / local extra entries of level 0 into the level-1 stencil.
void launch_galerkin_penalty(const TransferDev& P, int fnx, int fny, int64_t fnnode, const int* orig_copy, int npen,
                             const int* pen_node, const double* pen_k, double* A1, int cnx, int cny, int cnz,
                             int64_t cn, cudaStream_t s);
void launch_galerkin_local(const TransferDev& P, int fnx, int fny, int64_t fnnode, const int* orig_copy, int nent,
                           const int* rdof, const int* cdof, const double* val, double* A1, int cnx, int cny, int cnz,
                           int64_t cn, cudaStream_t s);

// Diagonal 3x3 blocks of a stencil into D[n][9].
void launch_stencil_diag(const double* A, int64_t n, double* D, cudaStream_t s);
// D[node][3r+c] += v for a list of (dof row, dof col, v) with equal nodes.
void launch_add_diag_entries(int nent, const int* rdof, const int* cdof, const double* val, double* D, cudaStream_t s);
// Inverse of every diagonal block, |det| < 1e-30 -> identity (fe/gmg.py:29-44); output SoA [9][n].
void launch_block_inverse(const double* D, int64_t n, double* Dinv64, float* Dinv32, cudaStream_t s);

}  // namespace feb
