// Material mixing of the engine's cells on the device (rb/rbfe.py:75-134), bit for bit with the NumPy code:
// class fractions of every cell from its sub-voxel body labels, the constrained-modulus mixing of hard
// (cortical, cancellous, fascia), joint-layer (cartilage, fibrous), soft (soft tissue, fat) and gap material,
// joint cells (two or more bone groups within the cell's 3x3x3 neighbourhood, or any layer material), and
// the resulting Young's modulus, Poisson ratio and active flag.  Sums run left to right from zero in the
// reference's column order and every product / sum / quotient is rounded on its own (no fused multiply-add),
// as NumPy evaluates them.
#include <cfloat>

#include "common.cuh"

namespace feb {

namespace {

constexpr int kClasses = 10;   // void cortical cancellous cartilage fascia soft plate fibrous fat gap

struct MixTable {
  double lam[kClasses], mu[kClasses], Mi[kClasses];   // per class: lambda, mu, lambda + 2 mu
};

__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dvd(double a, double b) { return __ddiv_rn(a, b); }

// fractions F[cell][class] = count / ns3, and the bone groups present (bit g-1 for group g)
__global__ void k_mat_fractions(int64_t ncell, int ns3, const int32_t* __restrict__ L, int nbody,
                                const int8_t* __restrict__ body_class, const int8_t* __restrict__ body_group,
                                double* __restrict__ F, unsigned long long* __restrict__ gmask) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  int cnt[kClasses] = {0};
  unsigned long long m = 0ull;
  for (int q = 0; q < ns3; ++q) {
    const int b = L[c * ns3 + q];
    int cl = (b >= 0 && b < nbody) ? body_class[b] : 0;
    cl = (cl >= 0 && cl < kClasses) ? cl : 0;
    cnt[cl] += 1;
    const int g = (b >= 0 && b < nbody) ? body_group[b] : 0;
    if (g > 0 && g <= 64) m |= 1ull << (g - 1);
  }
  for (int k = 0; k < kClasses; ++k) F[c * kClasses + k] = dvd((double)cnt[k], (double)ns3);
  gmask[c] = m;
}

__device__ __forceinline__ double nan_to_num(double v, double nan_value) {
  if (isnan(v)) return nan_value;
  if (isinf(v)) return v > 0 ? DBL_MAX : -DBL_MAX;
  return v;
}

__global__ void k_mat_mix(int nx, int ny, int nz, MixTable T, const double* __restrict__ Fall,
                          const unsigned long long* __restrict__ gmask, double* __restrict__ E_out,
                          double* __restrict__ nu_out, uint8_t* __restrict__ active_out, uint8_t* __restrict__ ser_out) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= (int64_t)nx * ny * nz) return;
  const double* F = Fall + c * kClasses;
  const int PH[7] = {1, 2, 4, 3, 7, 5, 8}, H[3] = {1, 2, 4}, LAY[2] = {3, 7}, SOFTC[2] = {5, 8};
  double occ = 0.0, lamV = 0.0, muV = 0.0;
  for (int q = 0; q < 7; ++q) occ = add(occ, F[PH[q]]);
  for (int q = 0; q < 7; ++q) lamV = add(lamV, mul(F[PH[q]], T.lam[PH[q]]));
  for (int q = 0; q < 7; ++q) muV = add(muV, mul(F[PH[q]], T.mu[PH[q]]));
  lamV = dvd(lamV, occ);
  muV = dvd(muV, occ);
  double hard = 0.0, lam_h = 0.0, mu_h = 0.0;
  for (int q = 0; q < 3; ++q) hard = add(hard, F[H[q]]);
  for (int q = 0; q < 3; ++q) lam_h = add(lam_h, mul(F[H[q]], T.lam[H[q]]));
  for (int q = 0; q < 3; ++q) mu_h = add(mu_h, mul(F[H[q]], T.mu[H[q]]));
  lam_h = dvd(lam_h, hard);
  mu_h = dvd(mu_h, hard);
  const double lay = add(add(0.0, F[3]), F[7]);
  const double fgap = add(0.0, F[9]);
  const double M_h = add(lam_h, mul(2.0, mu_h)), G_h = mu_h;
  const double hM = hard > 0.0 ? dvd(hard, M_h) : 0.0, hG = hard > 0.0 ? dvd(hard, G_h) : 0.0;
  const double gapM = add(0.0, dvd(F[9], T.Mi[9])), gapG = add(0.0, dvd(F[9], T.mu[9]));
  double layM = 0.0, layG = 0.0;
  for (int q = 0; q < 2; ++q) layM = add(layM, dvd(F[LAY[q]], T.Mi[LAY[q]]));
  for (int q = 0; q < 2; ++q) layG = add(layG, dvd(F[LAY[q]], T.mu[LAY[q]]));
  layM = add(layM, gapM);
  layG = add(layG, gapG);
  const double fch = add(add(lay, hard), fgap), occ_g = add(occ, fgap);
  const double M_ch = dvd(fch, add(layM, hM)), G_ch = dvd(fch, add(layG, hG));
  double lam_soft = 0.0, mu_soft = 0.0, softM = 0.0, softG = 0.0;
  for (int q = 0; q < 2; ++q) lam_soft = add(lam_soft, mul(F[SOFTC[q]], T.lam[SOFTC[q]]));
  for (int q = 0; q < 2; ++q) mu_soft = add(mu_soft, mul(F[SOFTC[q]], T.mu[SOFTC[q]]));
  for (int q = 0; q < 2; ++q) softM = add(softM, dvd(F[SOFTC[q]], T.Mi[SOFTC[q]]));
  for (int q = 0; q < 2; ++q) softG = add(softG, dvd(F[SOFTC[q]], T.mu[SOFTC[q]]));
  const double lam_c = dvd(add(mul(fch, sub(M_ch, mul(2.0, G_ch))), lam_soft), occ_g);
  const double mu_c = dvd(add(mul(fch, G_ch), mu_soft), occ_g);
  const double M_s = dvd(occ_g, add(add(softM, hM), gapM)), G_s = dvd(occ_g, add(add(softG, hG), gapG));
  const double lam_s = sub(M_s, mul(2.0, G_s)), mu_s = G_s;
  // bone groups within the 3x3x3 neighbourhood (binary dilation of each group's presence, summed)
  const int k = int(c % nz), j = int((c / nz) % ny), i = int(c / ((int64_t)nz * ny));
  unsigned long long m = 0ull;
  for (int di = -1; di <= 1; ++di)
    for (int dj = -1; dj <= 1; ++dj)
      for (int dk = -1; dk <= 1; ++dk) {
        const int a = i + di, b = j + dj, d = k + dk;
        if (a < 0 || a >= nx || b < 0 || b >= ny || d < 0 || d >= nz) continue;
        m |= gmask[((int64_t)a * ny + b) * nz + d];
      }
  const bool cart = lay > 0.0;
  const bool ser = cart || __popcll(m) >= 2;
  const double lamX = cart ? lam_c : (ser ? lam_s : lamV), muX = cart ? mu_c : (ser ? mu_s : muV);
  double E = dvd(mul(muX, add(mul(3.0, lamX), mul(2.0, muX))), add(lamX, muX));
  double nu = dvd(lamX, mul(2.0, add(lamX, muX)));
  const bool active = ser ? occ > 0.15 : occ >= 0.5;
  if (active) {
    if (!isnan(nu)) nu = nu < 0.0 ? 0.0 : (nu > 0.4995 ? 0.4995 : nu);
  } else {
    E = 1.0;
    nu = 0.3;
  }
  E_out[c] = nan_to_num(E, 1.0);
  nu_out[c] = nan_to_num(nu, 0.3);
  active_out[c] = active ? 1 : 0;
  ser_out[c] = ser ? 1 : 0;
}

}  // namespace
}  // namespace feb

using namespace feb;

extern "C" int feb_mix_materials(int32_t nx, int32_t ny, int32_t nz, int32_t ns3, const int32_t* L, int32_t nbody,
                                 const int8_t* body_class, const int8_t* body_group, const double* class_lam,
                                 const double* class_mu, const double* class_M, double* F, double* E, double* nu,
                                 uint8_t* active, uint8_t* ser, void* stream) {
  if (nx < 1 || ny < 1 || nz < 1 || ns3 < 1 || !L || nbody < 1 || !body_class || !body_group || !class_lam ||
      !class_mu || !class_M || !F || !E || !nu || !active || !ser) {
    set_last_error("feb_mix_materials: bad argument");
    return FEB_ERR_ARG;
  }
  MixTable T;
  for (int k = 0; k < kClasses; ++k) {
    T.lam[k] = class_lam[k];
    T.mu[k] = class_mu[k];
    T.Mi[k] = class_M[k];
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t ncell = (int64_t)nx * ny * nz;
  unsigned long long* gm = nullptr;
  FEB_CUDA(cudaMallocAsync((void**)&gm, ncell * sizeof(unsigned long long), s));
  k_mat_fractions<<<div_up(ncell, kThreads), kThreads, 0, s>>>(ncell, ns3, L, nbody, body_class, body_group, F, gm);
  note_launch();
  k_mat_mix<<<div_up(ncell, kThreads), kThreads, 0, s>>>(nx, ny, nz, T, F, gm, E, nu, active, ser); note_launch();
  FEB_CUDA(cudaGetLastError());
  FEB_CUDA(cudaFreeAsync(gm, s));
  return FEB_OK;
}
