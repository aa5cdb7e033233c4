// Rigid-body-mode coarse correction (see rigid.cu).
#pragma once
#include "common.cuh"

namespace feb {

struct RigidView {
  int ngroups;
  const int* off;            // [ngroups + 1] into nodes
  const int64_t* nodes;      // used node ids of every group
  const double* cen;         // [3 ngroups] centroids
  int nxn, nyn;              // grid nodes per axis (x, y)
  int64_t nnode;             // grid nodes
  const int* orig_copy;      // grid node of every copy
  const double* xe; const double* ye; const double* ze;   // node coordinates per axis
  const double* rho;         // [3 * nodes] (X - centroid) / 20 of every group node, set by launch_rigid_rho
};

// rho of every group node from the centroids (after launch_centroids)
void launch_rigid_rho(const RigidView& Z, double* rho, cudaStream_t s);

int rigid_blocks(const RigidView& Z);
// part: rigid_blocks * ngroups * 6 doubles (scratch)
void launch_centroids(const RigidView& Z, double* cen, double* part, cudaStream_t s);
// z += Z Einv Z^T r   (part: rigid_blocks * ngroups * 6 doubles; zr, coef: 6 ngroups).  ctr (optional): a
// zeroed counter; the reduction is then finished by its last block instead of a second launch.
template <typename T>
void launch_rigid_apply(const RigidView& Z, const T* r, T* z, double* part, double* zr, double* coef,
                        const double* Einv, const int* skip, cudaStream_t s, unsigned int* ctr = nullptr);
// the two halves of launch_rigid_apply (with ctr): coef = Einv Z^T r (reads r only, so it may run beside
// whatever forms z), then z += Z coef
template <typename T>
void launch_rigid_coef(const RigidView& Z, const T* r, double* part, double* zr, double* coef, const double* Einv,
                       const int* skip, cudaStream_t s, unsigned int* ctr);
template <typename T>
void launch_rigid_scatter(const RigidView& Z, const double* coef, T* z, const int* skip, cudaStream_t s);
// zr = Z^T r
void launch_ztr(const RigidView& Z, const double* r, double* part, double* zr, cudaStream_t s);
// v += column col of Z
void launch_z_column(const RigidView& Z, int col, double* v, cudaStream_t s);

}  // namespace feb
