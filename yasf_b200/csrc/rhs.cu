// Right-hand-side block of R plane-wave incidences on the device.
//
// The reference builds one incidence per Simulation on the host
// (yasfpy/initial_field_coefficients.py:79-142: a[s, n] = 4 E0 e^{-i m alpha} B^dagger_{tau l m}(beta)
// e^{i k . (r_s - r_focal)}) and the right-hand side b = T (.) a (yasfpy/simulation.py:189-205).
// Here the per-incidence mode factors coef[r][n] = 4 E0 e^{-i m alpha_r} B^dagger_{tau l m}(beta_r)
// (nmax x R numbers) come from the host and the kernel forms every (incidence, sphere, mode)
// entry: a = coef e^{i k_r . (r_s - r_focal)}, b = T a, written as R columns of length N nmax.
#include <cmath>

#include "capi_internal.h"

namespace yasf {

__global__ void __launch_bounds__(256) plane_wave_kernel(int n_particles, int nmax, int nrhs, long long ld,
                                                         const double* pos, const double* kvec,
                                                         const double2* coef, const double2* tmat,
                                                         double fx, double fy, double fz, double2* a,
                                                         double2* b) {
  const long long n = (long long)n_particles * nmax;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n * nrhs;
       e += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(e / n);
    const long long q = e - (long long)r * n;
    const int s = (int)(q / nmax), m = (int)(q - (long long)s * nmax);
    const double ph = kvec[3 * r] * (pos[3 * s] - fx) + kvec[3 * r + 1] * (pos[3 * s + 1] - fy) +
                      kvec[3 * r + 2] * (pos[3 * s + 2] - fz);
    double sn, cs;
    sincos(ph, &sn, &cs);
    const double2 c = coef[(size_t)r * nmax + m];
    const double2 v = make_double2(c.x * cs - c.y * sn, c.x * sn + c.y * cs);
    if (a) a[(size_t)r * ld + q] = v;
    if (b) {
      const double2 t = tmat[q];
      b[(size_t)r * ld + q] = make_double2(t.x * v.x - t.y * v.y, t.x * v.y + t.y * v.x);
    }
  }
}

}  // namespace yasf

using namespace yasf;

extern "C" int yasf_plane_wave_rhs(int lmax, int n_particles, const double* positions, int nrhs,
                                   const double* kvec, const double* coef, const double* focal_point,
                                   const double* tmat, double* a, double* b, long long ld, void* stream) {
  if (lmax < 1 || lmax > YASF_LMAX_MAX) return YASF_ERR_UNSUPPORTED;
  if (n_particles <= 0 || nrhs <= 0 || !positions || !kvec || !coef || (!a && !b)) return YASF_ERR_INVALID_ARGUMENT;
  if (b && !tmat) return YASF_ERR_INVALID_ARGUMENT;
  const int nmax = nmax_of(lmax);
  const long long n = (long long)n_particles * nmax;
  if (nrhs > 1 && ld < n) return YASF_ERR_INVALID_ARGUMENT;
  if (nrhs == 1) ld = n;
  if (!aligned16(coef) || (a && !aligned16(a)) || (b && !aligned16(b)) || (tmat && !aligned16(tmat)))
    return YASF_ERR_ALIGNMENT;
  const double f[3] = {focal_point ? focal_point[0] : 0.0, focal_point ? focal_point[1] : 0.0,
                       focal_point ? focal_point[2] : 0.0};
  for (double v : f)
    if (!std::isfinite(v)) return YASF_ERR_NOT_FINITE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int blocks = (int)std::min<long long>((n * nrhs + 255) / 256, 8192);
  YASF_COUNTED(plane_wave_kernel<<<blocks, 256, 0, s>>>(n_particles, nmax, nrhs, ld, positions, kvec,
                                                        reinterpret_cast<const double2*>(coef),
                                                        reinterpret_cast<const double2*>(tmat), f[0], f[1],
                                                        f[2], reinterpret_cast<double2*>(a),
                                                        reinterpret_cast<double2*>(b)));
  YASF_CUDA_TRY(cudaGetLastError());
  return YASF_OK;
}
