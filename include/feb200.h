/* feb200 -- C ABI of the B200-native voxel linear-elastic FE solver.
 *
 * Drop-in engine for the solve call of CoMech's data engine.  The reference is pure Python; the entry
 * points below are the C boundary under the Python host layer (comech_b200/), which keeps the
 * reference signatures.  Each function names the reference interface it serves.
 *
 * Conventions
 *   - grid: node id = i + (nx+1) (j + (ny+1) k); cell id = (i ny + j) nz + k (fe/solver.py:93-128);
 *     split copies have ids >= (nx+1)(ny+1)(nz+1) (rb/splitfe.py:261-305).
 *   - "full layout" vectors hold 3 doubles per node id (all grid nodes, then all copies); the reference's
 *     compact dof numbering (dof = 3 nmap[node] + comp over used nodes, rb/splitfe.py:72-76) is the
 *     restriction of it to the used nodes.
 *   - pointers marked [dev] are CUDA device pointers, [host] are host pointers.
 *   - every function returns FEB_OK (0) or a negative status; feb_last_error() describes the failure.
 *     No function aborts, and none falls back to a CPU implementation.
 */
#ifndef FEB200_H
#define FEB200_H
#include <stdint.h>

#if defined(__GNUC__)
#define FEB_API __attribute__((visibility("default")))
#else
#define FEB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define FEB_OK 0
#define FEB_ERR_ARG (-1)
#define FEB_ERR_CUDA (-2)
#define FEB_ERR_BREAKDOWN (-3)   /* p^T A p <= 0 in CG */
#define FEB_ERR_NAN (-4)         /* non-finite residual */
#define FEB_ERR_COARSE (-5)      /* coarsest-level matrix not positive definite */
#define FEB_ERR_TIMEOUT (-6)     /* a bounded device-side wait gave up */
#define FEB_ERR_INJECTED (-7)    /* failure injected on the host for tests (FEB_TEST_FAIL) */
#define FEB_ERR_NOMEM (-8)

#define FEB_MAT_ISO_SRI 0        /* lambda at the cell centre, mu 2x2x2 (rb/splitfe.py:58-69)      */
#define FEB_MAT_ISO_FULL 1       /* lambda and mu 2x2x2 (fe/solver.py:77-90)                       */
#define FEB_MAT_ORTHO 2          /* six orthotropic pattern coefficients (fe/solver.py:43-74)      */

#define FEB_PREC_FP64 0          /* FP64 PCG, FP64 V-cycle                                         */
#define FEB_PREC_MIXED 1         /* FP64 PCG, FP32 V-cycle (rb/gpusolve.py:206-262 mg_dtype=float32) */
#define FEB_PREC_REFINE 2        /* FP64 iterative refinement around an all-FP32 GMG-PCG           */

typedef struct FebHandle FebHandle;

typedef struct FebGrid {
  int32_t nx, ny, nz;            /* cells per axis */
  const double* xe;              /* [host] nx+1 edges */
  const double* ye;              /* [host] ny+1 edges */
  const double* ze;              /* [host] nz+1 edges */
} FebGrid;

/* Level-0 operator K = sum_cells K_e + diag(kd) + E, E a sparse symmetric extra matrix
 * (rb/splitfe.py:123-150, fe/solver.py:202-232). */
typedef struct FebOperator {
  int32_t mat_mode;              /* FEB_MAT_* */
  const double* mat;             /* [dev] ISO: lam[ncell] followed by mu[ncell]; ORTHO: coeffs[ncell][6]; cell-id order */
  const uint8_t* active;         /* [dev] ncell flags */
  const int64_t* cn;             /* [dev] ncell x 8 node ids (split connectivity), NULL = grid connectivity */
  int64_t nnode_total;           /* grid nodes + split copies */
  const int64_t* orig;           /* [dev] grid node of every node id (nnode_total), NULL when there are no copies */
  int64_t npen;                  /* diagonal penalties: kd[3 node + c] += k[3 i + c] */
  const int64_t* pen_node;       /* [host] npen node ids */
  const double* pen_k;           /* [host] npen x 3 */
  int64_t nextra;                /* extra matrix entries (COO, duplicates summed), full-layout dofs */
  const int64_t* extra_row;      /* [host] */
  const int64_t* extra_col;      /* [host] */
  const double* extra_val;       /* [host] */
  int64_t nmark;                 /* nodes used although no active cell references them (an operator given only */
  const int64_t* mark_used;      /* [host] as a matrix, fe/gmg.py:120 pcg_gmg); may be 0 / NULL              */
} FebOperator;

typedef struct FebOptions {
  int32_t precision;             /* FEB_PREC_* */
  int32_t maxiter;               /* CG iterations (all refinement sweeps together) */
  double tol;                    /* stop when ||f - K x|| < tol ||f|| */
  int32_t min_dofs;              /* coarsening stops at <= min_dofs dofs (fe/gmg.py:80: 6000) */
  int32_t max_levels;            /* (fe/gmg.py:80: 6); 0 = operator only (feb_apply, no feb_solve) */
  int32_t cheb_degree;           /* Chebyshev degree (fe/gmg.py:61: 3) */
  int32_t check_every;           /* host polls convergence every k iterations (>= 1) */
  double inner_tol;              /* REFINE: relative residual reduction of each FP32 sweep */
  int32_t inner_maxiter;         /* REFINE: CG iterations per sweep */
  int32_t use_graphs;            /* 0 direct launches; 1 one graph per CG iteration, host polls convergence;
                                    2 the CG loop is a device-side while loop (conditional graph node) */
  uint64_t seed;                 /* power-iteration start vectors */
  int32_t x0_mode;               /* start value x0: 0 as given; 1 its energy-optimal multiple; 2 (default) x0 + M (f -
                                    K x0) (one preconditioner application), then its energy-optimal multiple */
  int32_t level_kernel;          /* coarse-level stencil products (one node per thread, the 14 block slots over 4
                                    warps), bits 0-1: 0 (default) slot index a compile-time constant in FP32
                                    products and a run-time value in FP64 products (the faster form of each); 1
                                    run-time in both; 2 compile-time in both.  Bit 2 (+4): the V-cycle's rank-1 term
                                    dots by a dot pass before every product, instead of accumulated by the kernels
                                    that write the vectors.  FP32 products with compile-time slots read a 16-bit
                                    copy of the stencil (FP16 scaled by a power of two, FP32 sums) on levels
                                    without compressed blocks; bit 3 (+8) gives them an FP32 copy instead */
} FebOptions;

typedef struct FebInfo {
  int32_t iters;                 /* CG iterations (sum over refinement sweeps) */
  int32_t flag;                  /* 0 converged, else maxiter (SciPy cg convention) */
  int32_t levels;                /* multigrid levels incl. the coarsest */
  int32_t sweeps;                /* refinement sweeps (1 for FP64 / MIXED) */
  double relres;                 /* FP64 ||f - K x|| / ||f|| of the returned x */
  double t_setup_ms;             /* device time of feb_create's multigrid set-up, from its start to the end of
                                    the last set-up chain (some finish after feb_create returns) */
  double t_solve_ms;             /* device time of feb_solve */
  int64_t ndof;                  /* 3 x used nodes */
  int64_t level_dofs[8];
  double lmax[8];
  int32_t coarse_n;              /* dofs of the dense coarsest level */
  int32_t kernel_launches;       /* kernels launched by feb_solve */
  int32_t ku_shape[4];           /* autotuned fine K.u launch shape: FP32 (warps per CTA, 0 = tensor cores;
                                    node planes per CTA), FP64 (warps, planes) */
  double t_stage_ms[8];          /* feb_create stages (device time): cells, penalties/extra, diagonal blocks,
                                    K.u tuning, Galerkin hierarchy, work vectors and power-iteration launch, then
                                    the deferred tail (dense coarse level beside the power iterations, measured
                                    from the launch's end to the slowest chain's end); [7] host time of feb_create
                                    before the device-timed set-up (pool reservation, handle) */
  int32_t x0_used;               /* 1: the solve started from the caller's x0 (as FebOptions.x0_mode prepares it); 0:
                                    from zero (no x0, or a start s with s.f <= 0: the fallback of a warm start) */
  float x0_scale;                /* the energy-optimal multiple a = s.f / s.K s applied to the start (1 in mode 0) */
  int32_t ku_kind;               /* level-0 K.u kernel of FP32 products: 0 per-cell kernel, 1 paired-row kernel
                                    (ku_shape then holds warps per CTA and node planes of that kernel), 2 tensor
                                    cores; FP64 products use the paired-row kernel whenever it is set up */
} FebInfo;

/* Default options (tol 1e-6, maxiter 800 as rb/splitfe.py:123; GMG parameters of fe/gmg.py:80). */
FEB_API void feb_default_options(FebOptions* opt);

/* Builds the operator and the multigrid hierarchy on the device (replaces the CPU/SciPy assembly,
 * fe/solver.py:137-162, rb/splitfe.py:72-91, rb/gpusolve.py:306-346, and the hierarchy set-up,
 * fe/gmg.py:79-102, rb/gpusolve.py:39-171).  `stream` is a cudaStream_t (NULL = default).
 * The last set-up steps (the dense coarsest level's inverse, the smoothers' eigenvalue estimates) are still
 * running on the handle's side streams when feb_create returns, so that the caller's next steps
 * (feb_set_rigid_groups, loads, a start value) overlap them; feb_solve, feb_solve_batch, feb_precondition and the
 * benchmark calls wait for them, and a coarsest-level matrix that is not positive definite is reported there
 * (FEB_ERR_COARSE, on that call and every later one). */
FEB_API int feb_create(const FebGrid* grid, const FebOperator* op, const FebOptions* opt, void* stream, FebHandle** out);

/* Per-group rigid-body modes for the additive coarse correction Z pinv(Z^T K Z) Z^T
 * (fe/solver.py:177-199, rb/splitfe.py:105-120, fe/gmg.py:127-135).  Group g is
 * nodes[offsets[g] .. offsets[g+1]) (node ids, [dev] int64); unused nodes are dropped and groups with
 * fewer than 4 used nodes are skipped, as in the reference. */
FEB_API int feb_set_rigid_groups(FebHandle* h, int32_t ngroups, const int64_t* offsets, const int64_t* nodes);

/* Solve K x = f by GMG-preconditioned CG (fe/gmg.py:120-137, rb/gpusolve.py:206-292).
 * f, x: [dev] full layout (3 nnode_total doubles); x0: [dev] start or NULL (zero start).
 * Unused nodes of x are left 0. */
FEB_API int feb_solve(FebHandle* h, const double* f, const double* x0, double* x, FebInfo* info);

/* Solves n independent systems K_i x_i = f_i, one per handle, as ONE CUDA graph launch: per instance a
 * device-side start (stop threshold tol ||f_i|| formed on the device), a device-side while loop of CG iterations
 * whose condition is the instance's own convergence flag (instances stop independently), and a finish (x_i, true
 * residual).  The instances run concurrently on the device; small grids that leave most SMs idle alone share
 * the GPU.  Replaces the per-process engine pool of exp/rb_run_engine_v4.py:113-147, where every process solved
 * one (foot, action) instance with rb/splitfe.py:123-158.
 * hs: n distinct handles (FP64 or mixed precision; the refined precision's host-driven sweeps need feb_solve);
 * f[i], x[i]: [dev] full layout of handle i; x0: NULL (zero starts) or n starts (NULL entries allowed), used as
 * given; info: NULL or n entries (t_solve_ms is the batch's time).  The graph runs on hs[0]'s stream after all
 * callers' streams; each caller's stream continues after the batch. */
FEB_API int feb_solve_batch(FebHandle* const* hs, int32_t n, const double* const* f, const double* const* x0,
                            double* const* x, FebInfo* info);

/* y = K u on the level-0 operator (full layout), prec = 0 FP64 / 1 FP32 (test and benchmark hook). */
FEB_API int feb_apply(FebHandle* h, int32_t prec, const void* u, void* y);

/* z = M r: one application of the solve's preconditioner (V-cycle in the handle's precision plus the rigid-mode
 * correction), FP64 full-layout r and z on the device.  Replaces the M LinearOperator of fe/gmg.py:125-135 for a
 * Krylov loop run by the caller (pcg_gmg with a separate A_op, fe/gmg.py:136). */
FEB_API int feb_precondition(FebHandle* h, const double* r, double* z);

/* U[node][c] = x for used nodes, NaN for unused ones (the reference's U, rb/splitfe.py:154). */
FEB_API int feb_export_solution(FebHandle* h, const double* x, double* U);

/* Number of used nodes and the used-node mask ([dev] uint8 nnode_total). */
FEB_API int feb_used_nodes(FebHandle* h, int64_t* nused, uint8_t* mask);

/* Releases every device buffer of the handle. */
FEB_API int feb_destroy(FebHandle* h);

/* dst[3 node[i] + c] += vals[3 i + c]; nodes/vals [dev], dst [dev] (nodal loads, rb/splitfe.py:144-147). */
FEB_API int feb_accumulate_nodal(int64_t n, const int64_t* nodes, const double* vals, double* dst, void* stream);

/* Centre-point strain, stress and von Mises of listed cells (fe/solver.py:257-272,
 * rb/splitfe.py:161-175).  mat as in FebOperator (ISO uses lam/mu; ORTHO uses D = sum c_k P_k);
 * U [dev] nnode_total x 3 (NaN treated as 0 when nan_to_zero); cells [dev] int64 cell ids;
 * cn [dev] connectivity or NULL; outputs [dev] sig ncells x 6, vm ncells, eps ncells x 6 (eps may be NULL). */
FEB_API int feb_cell_stress(const FebGrid* grid, int32_t mat_mode, const double* mat, const double* U, int64_t ncells,
                    const int64_t* cells, const int64_t* cn, int32_t nan_to_zero, double* sig, double* vm,
                    double* eps, void* stream);

/* feb_cell_stress without any device allocation, for callers that cannot allocate device memory at the
 * point of the call (a fixed memory arena owned by a host framework, a plugin's enqueue callback, a
 * latency-critical loop that must not synchronise on cudaMalloc).  Same arguments and results as
 * feb_cell_stress.  Its scratch (grid edges and cell widths) is one fixed file-scope device array:
 * at most 4096 cells per axis (larger grids: FEB_ERR_ARG), 192 KB held on every GPU that loads the
 * library until exit.  The first call on a device looks up that array's address with the device
 * current.  Every call copies the grid edges from the caller's (pageable) host arrays into that array, so
 * no call may be made under stream capture: a captured copy would read the host arrays when the graph
 * replays.  All calls share the array: calls that overlap on the GPU race, so order them on one stream.  No counterpart in the reference (its stress recovery is NumPy). */
FEB_API int feb_cell_stress_noalloc(const FebGrid* grid, int32_t mat_mode, const double* mat, const double* U,
                                    int64_t ncells, const int64_t* cells, const int64_t* cn, int32_t nan_to_zero,
                                    double* sig, double* vm, double* eps, void* stream);

/* Internal nodal forces K_e u_e of listed cells with the SRI lambda term (rb/splitfe.py:178-193);
 * out [dev] ncells x 8 x 3. */
FEB_API int feb_element_forces(const FebGrid* grid, const double* mat, const double* U, int64_t ncells,
                       const int64_t* cells, const int64_t* cn, double* out, void* stream);

/* Forces on a bone from its neighbourhood (rb/rbfe.py:194-213): the nodes of the active cells of part
 * `target` are marked; every other active cell touching them contributes minus its nodal forces K_e u_e (SRI,
 * as feb_element_forces) at the marked corners, summed per cell label.  part, lab: [dev] int32 per cell
 * (cell-id order); lab in 0..nlab-1 (1 <= nlab <= 64, other values ignored); cn [dev] or NULL; out [dev]
 * nlab x 3; present [dev] nlab flags (1 = some contributing cell has the label). */
FEB_API int feb_region_forces(const FebGrid* grid, const double* mat, const double* U, const int64_t* cn,
                              const uint8_t* active, const int32_t* part, const int32_t* lab, int32_t nlab,
                              int32_t target, int64_t nnode_total, double* out, int32_t* present, void* stream);

/* Rigid-body least-squares fit (rb/rbsim.py:99-107): U ~ t + w x (X - c), c the centroid of X.  X, U [dev] n x 3
 * (U as given: the reference's callers pass nan_to_num(U)); fit [host] 9: t, w, c (minimum-norm solution,
 * numpy.linalg.lstsq convention). */
FEB_API int feb_rigid_fit(const double* X, const double* U, int64_t n, double* fit, void* stream);

/* Displacement relative to a rigid fit (rb/rbsim.py:184): out = nan_to_num(U) - (t + w x (X - c)) at every node;
 * fit [host] 9 as from feb_rigid_fit; U, out [dev] nnode_total x 3. */
FEB_API int feb_relative_displacement(const FebGrid* grid, const int64_t* orig, int64_t nnode_total, const double* U,
                                      const double* fit, double* out, void* stream);

/* Fields on an analysis grid of mx x my x mz cells (cell id z fastest), sub^3 points per cell (rb/rbsim.py:110-138):
 * per axis and point p the FE cell index i[p], the local coordinate t[p] in [0, 1] and the inside flag in[p]
 * ([dev], m*sub entries); relative displacement (trilinear in the FE cell), von Mises VM [dev] float ncell and
 * stress SIG [dev] float ncell x 6 averaged over the points in active FE cells.  Outputs [dev] float:
 * vm mx*my*mz, u x3, frac (fraction of points in active cells), sig x6. */
FEB_API int feb_sample_cells(const FebGrid* grid, int32_t mx, int32_t my, int32_t mz, int32_t sub, const int32_t* ix,
                             const double* tx, const uint8_t* inx, const int32_t* iy, const double* ty,
                             const uint8_t* iny, const int32_t* iz, const double* tz, const uint8_t* inz,
                             const int64_t* cn, const uint8_t* active, const double* Urel, const float* VM,
                             const float* SIG, float* vm_out, float* u_out, float* frac_out, float* sig_out,
                             void* stream);

/* Nearest active cell of every cell (exact Euclidean feature transform over cell indices; ties resolved as
 * scipy.ndimage.distance_transform_edt resolves them: separable passes x, y, z, the lower index first).
 * active [dev] ncell flags (cell id z fastest); ft [dev] int32 ncell: cell id of the nearest active cell, -1 when
 * no cell is active. */
FEB_API int feb_nearest_active(const FebGrid* grid, const uint8_t* active, int32_t* ft, void* stream);

/* Relative displacement at the nodes of an analysis grid (rb/rbsim.py:141-161): node (a, b, c), x fastest, at
 * (px[a], py[b], pz[c]) lies in FE cell (ix[a], iy[b], iz[c]); that cell is replaced by its nearest active cell
 * ft[...] and Urel is interpolated trilinearly there with clamped local coordinates.  Per-axis arrays [dev]
 * (mx1, my1, mz1 entries); out [dev] float mx1*my1*mz1 x 3. */
FEB_API int feb_sample_nodes(const FebGrid* grid, int32_t mx1, int32_t my1, int32_t mz1, const int32_t* ix,
                             const double* px, const int32_t* iy, const double* py, const int32_t* iz, const double* pz,
                             const int32_t* ft, const int64_t* cn, const double* Urel, float* out, void* stream);

/* Split-node connectivity between bones (rb/splitfe.py:261-305 == :17-55), bit for bit.  active [dev] ncell
 * flags, part [dev] int32 ncell (0 joint / soft, 1..nb-1 bone), share [dev] float64 ncell x nb (bone shares of
 * the cells).  Call once with cn = orig = NULL for the sizes: *nnode_total (grid nodes + copies) and *nsplit
 * (split grid nodes); then with cn [dev] ncell x 8 and orig [dev] of orig_cap >= *nnode_total entries. */
FEB_API int feb_split_connectivity(const FebGrid* grid, const uint8_t* active, const int32_t* part, const double* share,
                                   int32_t nb, int64_t* cn, int64_t* orig, int64_t orig_cap, int64_t* nnode_total,
                                   int64_t* nsplit, void* stream);

/* Material mixing of the engine's cells (rb/rbfe.py:75-134), bit for bit: L [dev] int32 ncell x ns3 sub-voxel body
 * labels (cell id z fastest); body_class / body_group [dev] int8 per body id (nbody entries): class 0..9 (void
 * cortical cancellous cartilage fascia soft plate fibrous fat gap) and bone group (0 none, 1..64); class_lam,
 * class_mu, class_M [host] 10 per-class lambda, mu, lambda + 2 mu.  Outputs [dev]: F ncell x 10 class fractions,
 * E, nu (float64), active and joint-cell flags (uint8). */
FEB_API int feb_mix_materials(int32_t nx, int32_t ny, int32_t nz, int32_t ns3, const int32_t* L, int32_t nbody,
                              const int8_t* body_class, const int8_t* body_group, const double* class_lam,
                              const double* class_mu, const double* class_M, double* F, double* E, double* nu,
                              uint8_t* active, uint8_t* ser, void* stream);

/* ---- voxel labelling of a foot lattice (rb/rbgeom.py:493-524 label_lattice, :358-464 label_points) ---------- */
/* One facet of the template (rb/rbgeom.py:152-171): centre c, normal n, in-plane axes e1 (anterior) and e2
 * (medial), footprint raster F0 [dev] uint8 nu x nv (row-major, origin (ua, va), pixel res), semi-axes a0 b0,
 * centre (uc, vc) in the plane, cartilage half-thickness wmax, median joint gap, bounding box. */
typedef struct FebLabelFacet {
  double c[3], n[3], e1[3], e2[3];
  double ua, va, res, a0, b0, uc, vc, wmax, gap;
  double xyz_lo[3], xyz_hi[3];
  const uint8_t* F0;
  int32_t nu, nv;
} FebLabelFacet;

/* A front grown over a facet from its edge (rb/rbgeom.py:332-342): inside when (u - uc) d0 + (v - vc) d1 <= thr;
 * on = 0 when the covered fraction is 0.  The host forms d (unit) and thr (the fraction's quantile over the scaled
 * footprint's pixel centres). */
typedef struct FebLabelGrown {
  int32_t on, pad;
  double d[2];
  double thr;
} FebLabelGrown;

/* Template, foot and action of one labelling call.  Template (rb/rbgeom.py:183-218): lab [dev] int8 lnx x lny x lnz
 * (x slowest; origin o, spacing h), dt / dc [dev] float32 snx x sny x snz distances to talus / calcaneus (origin so,
 * spacing h), facets post, mid, ant, scale centre c0, shear (z_ref, x_w0, x_w1), osteotomy plane (x_cut0, z_cut0,
 * cut_slope, z_frag_top), static_mask bit b = body b never moves with the fragment.  Foot (rb/rbgeom.py:55-73):
 * scale, facet factors fa / fb (post, mid, ant: size / nominal), ant_mode, ctype (0 none, 1 I, 2 II, 3 III, 4 IV),
 * rtype (0 none, 1-4 R1-R4), sust_y, post_dome, tan_align = tan(align in rad) with align_on = (align != 0),
 * cov_mid, fib_frac and the grown fronts of the coalitions (g_cov_mid, g_cov_post).  Action (rb/rbgeom.py:86-93):
 * resect, interp, fusion, osteo, defect fronts (g_d_mid, g_d_post); void_fill = (defect_fill == "void"). */
typedef struct FebLabelParams {
  const int8_t* lab;
  int32_t lnx, lny, lnz, pad0;
  double o[3], h;
  const float* dt;
  const float* dc;
  int32_t snx, sny, snz, pad1;
  double so[3];
  FebLabelFacet facet[3];
  double c0[3], z_ref, x_w0, x_w1, x_cut0, z_cut0, cut_slope, z_frag_top;
  uint32_t static_mask[4];
  double scale, fa[3], fb[3];
  int32_t ant_mode, ctype;
  double sust_y, post_dome, tan_align;
  int32_t align_on, rtype;
  double cov_mid, fib_frac;
  FebLabelGrown g_cov_mid, g_cov_post, g_d_mid, g_d_post;
  int32_t resect, interp, fusion, void_fill;
  double osteo;
} FebLabelParams;

/* Labels of the lattice sx x sy x sz (world frame; [dev] float64 nx, ny, nz) into L [dev] int16 nx x ny x nz
 * (z fastest): equal to rb/rbgeom.py:358 label_points at every lattice point.  One thread per point: the inverse
 * map into the template (scale, fragment shift, alignment shear, local warps by 3 fixed-point steps), the raster
 * lookup, the fragment relabelling and the subtalar edits, in FP64 in the reference's operation order. */
FEB_API int feb_label_lattice(const FebLabelParams* p, const double* sx, int32_t nx, const double* sy, int32_t ny,
                              const double* sz, int32_t nz, int16_t* L, void* stream);

/* ---------------------------------------------------------------------------------------------------------
 * Learned warm start: a 3D convolutional encoder-decoder whose prediction is the PCG initial guess.  The
 * reference has no counterpart (its PCG starts from x0 = 0 or a caller's x0, fe/gmg.py:120-137); these entry
 * points are the network's layers, training steps and its coupling to the solve's inputs and outputs.
 *
 * Activations live on a padded voxel grid: a grid of nx x ny x nz cells has (nx+2)(ny+2)(nz+2) rows, row
 * ((x+1)(ny+2) + (y+1))(nz+2) + (z+1) for cell (x, y, z) (z fastest, like the FE cell id), with a shell of
 * zero rows around the cells.  A row holds `ld` BF16 channels (ld a multiple of 8); a tensor may be a channel
 * range [c0, c0 + C) of a wider buffer (skip connections share one buffer).
 * --------------------------------------------------------------------------------------------------------- */
#define FEB_GATHER_SHIFT 0       /* 3x3x3 taps, stride 1: tap t = 9(dx+1) + 3(dy+1) + (dz+1)                  */
#define FEB_GATHER_DOWN 1        /* 2x2x2 taps, stride 2: coarse row V reads fine cells 2V + (tx, ty, tz),
                                    tap t = 4 tx + 2 ty + tz                                                  */
#define FEB_GATHER_ONE 2         /* one tap: row r reads row r                                                */
#define FEB_GATHER_UP 3          /* (weight gradient only) P rows at fine cells 2V + t, Q rows at coarse V   */

typedef struct FebNetGrid {
  int32_t nx, ny, nz;            /* cells per axis (rows: (nx+2)(ny+2)(nz+2)) */
} FebNetGrid;

/* One implicit-GEMM pass on the tensor cores: out[row][n] = sum over taps t and channels k of
 * in[src(row, t)][in_c0 + k] * wt[t][n][k], then  + bias[n], ReLU, + existing out (accumulate), * (mask > 0).
 * Rows run over `grid` (gather SHIFT / ONE: the input's own grid; DOWN: the coarse output grid reading the
 * fine grid `fine`).  scatter = 1: the GEMM columns are 8 groups of scatter_c channels and the row of coarse
 * cell V in group t is written to fine cell 2V + t of `fine` (a transposed 2x2x2 stride-2 convolution).
 * Shell rows of the output are written as zeros (scatter: never written; callers zero them once).  kc (channels
 * per tap) is a multiple of 32; n a multiple of 32; ld / c0 multiples of 8.  status [dev] is set to 1 if a
 * bounded tensor-core wait ran out (the result is then invalid). */
typedef struct FebConv {
  int32_t gather, scatter;
  FebNetGrid grid, fine;
  const void* in;                /* [dev] bf16 */
  int32_t in_ld, in_c0, kc, n;
  const void* wt;                /* [dev] bf16 [taps][n][kc] */
  void* out;                     /* [dev] bf16 */
  int32_t out_ld, out_c0, scatter_c, relu;
  const float* bias;             /* [dev] n (scatter: scatter_c) or NULL */
  const void* mask;              /* [dev] bf16 or NULL */
  int32_t mask_ld, mask_c0, accumulate, pad_;
  int32_t* status;               /* [dev] or NULL */
} FebConv;

FEB_API int feb_net_conv(const FebConv* c, void* stream);

/* Weight gradient: dw[t][a][b] += sum over rows r of P[rowP(r, t)][p_c0 + a] * Q[rowQ(r, t)][q_c0 + b], rows r over
 * `grid`; mode SHIFT: rowP = r, rowQ = r + tap offset; DOWN: rowP = r (coarse), rowQ = fine cell 2V + t; UP:
 * rowP = fine cell 2V + t, rowQ = r (coarse).  na, nb multiples of 32.  dw [dev] fp32, accumulated. */
typedef struct FebWgrad {
  int32_t mode, pad_;
  FebNetGrid grid, fine;
  const void* p;                 /* [dev] bf16 */
  int32_t p_ld, p_c0, na;
  int32_t q_ld, q_c0, nb;
  const void* q;                 /* [dev] bf16 */
  float* dw;                     /* [dev] [taps][na][nb] */
} FebWgrad;

FEB_API int feb_net_wgrad(const FebWgrad* w, void* stream);

/* out[c] += sum over rows of g[r][c0 + c], c < nc (bias gradients; shell rows of g are zero). */
FEB_API int feb_net_colsum(const void* g, int64_t rows, int32_t ld, int32_t c0, int32_t nc, float* out, void* stream);

/* BF16 weight tables from FP32 master weights W [taps][co][ci]: fwd [taps][co][ci]; bwd (if not NULL)
 * [taps][ci][co], tap order reversed when flip = 1 (the data gradient of a 3x3x3 convolution). */
FEB_API int feb_net_weights(const float* W, int32_t taps, int32_t co, int32_t ci, void* fwd, void* bwd, int32_t flip,
                            void* stream);

/* Output head (1x1 convolution of 32 channels to 3) and, when target is not NULL, the weighted mean squared error
 * with its gradients: pred[r][c] = b[c] + sum_k X[r][k] W[c][k] (pred may be NULL); loss += sum_r wgt[r] |pred -
 * target|^2 * inv_n; dX[r][k] = (X[r][k] > 0) sum_c 2 inv_n wgt[r] (pred - target)[c] W[c][k]; dW, db
 * accumulated.  All [dev]; X, dX bf16 with row stride x_ld / dx_ld. */
FEB_API int feb_net_head(const void* X, int32_t x_ld, int64_t rows, const float* W, const float* b, float* pred,
                         const float* target, const float* wgt, float inv_n, double* loss, void* dX, int32_t dx_ld,
                         float* dW, float* db, void* stream);

/* Backward pass of the head for a given gradient dpred [dev] (fp32, 3 per row) of its output: dX[r][k] = (X[r][k] >
 * 0) sum_c dpred[r][c] W[c][k]; dW, db accumulated. */
FEB_API int feb_net_head_grad(const void* X, int32_t x_ld, int64_t rows, const float* W, const float* dpred, void* dX,
                              int32_t dx_ld, float* dW, float* db, void* stream);

/* Training loss of a prediction pred [dev] (fp32, 3 per row; NULL: zero) against target / wgt on the network grid:
 * mse_scale sum_r wgt |e|^2 plus h1_scale sum over grid edges (node r to its +1 neighbour along x, y, z, both with
 * wgt > 0) of (E / e_ref) |e(r2) - e(r)|^2, e = pred - target, E the Young's modulus of the cell at r read from the
 * network input xin (channel 0 = log10 E / 4, channel 2 = active; 0 for inactive cells).  The second term weighs the
 * error's differences by stiffness, as the strain energy of the error does.  loss [dev] += the sum; dpred [dev] (if
 * not NULL) += its gradient. */
FEB_API int feb_net_loss(FebNetGrid net, const void* xin, const float* pred, const float* target, const float* wgt,
                         float e_ref_inv, float mse_scale, float h1_scale, double* loss, float* dpred, void* stream);

/* Training loss: strain energy of a prediction's error on a network grid equal to the FE grid (spacing h [host 3]):
 * scale * sum over active cells whose 8 corners have targets of e^T K_e e, e = pred - target at the corners, K_e the
 * hex8 element of the solve (lambda at the centre, mu 2x2x2) with the Lame constants of the cell read from the network
 * input xin (channel 0 = log10 E / 4, channel 1 = (nu - 0.3) * 4, channel 2 = active).  pred [dev] NULL: the target's
 * energy.  loss [dev] += the sum; dpred [dev] (if not NULL) += its gradient 2 scale K_e e. */
FEB_API int feb_net_energy_loss(FebNetGrid net, const double* h, const void* xin, const float* pred, const float* target,
                                const float* wgt, float scale, double* loss, float* dpred, void* stream);

/* Adam step on n FP32 parameters (bias-corrected, step >= 1); the gradient is scaled by gscale first and
 * zeroed afterwards.  sumsq (if not NULL) receives += sum of squared gradients before the step is taken. */
FEB_API int feb_net_adam(float* w, float* g, float* m, float* v, int64_t n, float lr, float beta1, float beta2,
                         float eps, int32_t step, float gscale, void* stream);
FEB_API int feb_net_sumsq(const float* g, int64_t n, double* out, void* stream);

/* Network input (32 BF16 channels per row, channels 0-5 used) on the network grid `net` of spacing hn [host 3],
 * from the solve's inputs on the FE grid of uniform spacing h [host 3] covering the same box from the origin:
 * 0 log10(E)/4 and 1 (nu - 0.3) * 4 of the FE cell at the network cell's centre (active cells), 2 active; 3
 * split-node, 4 contact (ground spring) and 5 load marks of the FE grid nodes that fall in the cell (load: the z
 * load of the nodes, times load_scale).  split / contact / load node lists hold grid node ids [dev]; mat =
 * (lambda | mu) [dev] per FE cell; active [dev] uint8 per FE cell.  scratch [dev] 3 floats per network cell. */
FEB_API int feb_net_inputs(FebNetGrid net, const double* hn, const FebGrid* fe, const double* h, const double* mat,
                           const uint8_t* active, int64_t nsplit, const int64_t* split_nodes, int64_t ncontact,
                           const int64_t* contact_nodes, int64_t nload, const int64_t* load_nodes,
                           const double* load_z, double load_scale, float* scratch, void* out, void* stream);

/* Training target on a network grid equal to the FE grid: target[row of cell (i,j,k)] = U[node (i,j,k)] / scale
 * (fp32, 3 per row) and wgt = 1 where that node's displacement is finite, else 0 (shell rows 0).  U [dev] full
 * layout fp64 (NaN on unused nodes), at least (nx+1)(ny+1)(nz+1) nodes. */
FEB_API int feb_net_targets(FebNetGrid net, const double* U, double scale, float* target, float* wgt, void* stream);

/* Initial guess from a prediction: x0[3n + c] = scale * trilinear interpolation of pred (values at the lower
 * corner nodes of the network cells, spacing hn) at the position of FE node n (grid node orig[n], spacing h), for
 * every node id n < nnode_total.  orig may be NULL (no copies). */
FEB_API int feb_net_to_nodes(FebNetGrid net, const double* hn, const float* pred, double scale, const FebGrid* fe,
                             const double* h, const int64_t* orig, int64_t nnode_total, double* x0, void* stream);

/* Benchmark hook: average device time (CUDA events on the handle's stream) of nrep level-0 products. */
FEB_API int feb_benchmark_apply(FebHandle* h, int32_t prec, const void* u, void* y, int32_t nrep, float* ms);
/* Benchmark hook: the same over nbuf (u, y) pairs used in turn, so that a set of buffers larger than the L2
   cache makes every product read its operands from HBM. */
FEB_API int feb_benchmark_apply_set(FebHandle* h, int32_t prec, int32_t nbuf, const void* const* u, void* const* y,
                                    int32_t nrep, float* ms);

/* Benchmark hook: the level-0 smoother step as the V-cycle runs it (the paired K.u with the fused Chebyshev
   update r -= K d, d' = a1 d + a2 D^-1 r, x += d', FP32), over nbuf sets of (d, r, x, d') buffers used in turn,
   each 3 nnode_total floats on the device; the handle needs its hierarchy (the level's Chebyshev
   coefficients).  ms: the average step. */
FEB_API int feb_benchmark_smooth_set(FebHandle* h, int32_t nbuf, void* const* d, void* const* r, void* const* x,
                                     void* const* e, int32_t nrep, float* ms);

/* Kernels launched by this library since it was loaded (graph launches count their kernel nodes). */
FEB_API int64_t feb_launch_count(void);

/* The current device's default memory pool, which serves every handle: bytes reserved, the used-memory peak
   since the last reservation, and how many times feb_create has grown the reservation in this process. */
FEB_API int feb_pool_stats(int64_t* reserved, int64_t* used_peak, int32_t* grow_events);

FEB_API const char* feb_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
