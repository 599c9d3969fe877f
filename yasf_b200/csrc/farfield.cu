// Far field of the scattered wave on a set of sampling directions, on the device.
//
// The reference evaluates, for every direction a (polar theta_a, azimuth phi_a, unit vector e_r(a))
// and wavelength, E_theta(a) and E_phi(a) as a sum over every particle s and mode
// n = (tau, l, m) of
//   t = i^{tau - l - 2} b[s, n] / sqrt(2 l (l + 1)) e^{i (m phi_a - k r_s . e_r(a))}
// times (i m pi_l|m|(theta_a), -tau_l|m|(theta_a)) for tau = 1 and (tau_l|m|, i m pi_l|m|) for
// tau = 2 (yasfpy/functions/cpu_numba.py:536-601; Numba-CUDA yasfpy/functions/cuda_numba.py:824-894;
// driver yasfpy/optics.py:178-267), then the Stokes parameters I, Q, U, V of (E_theta, E_phi)
// (cpu_numba.py:604-660). The reference's CPU loop adds into shared array elements from a
// parallel loop (a race); its serial evaluation is what the tests compare against.
//
// Here the sum is re-associated per direction: E(a) = sum_n C_n(a) F_n(a) with the far-field
// multipole sums F_n(a) = sum_s b[s, n] e^{-i k r_s . e_r(a)} and the angular factors C_n(a) (all
// but the particle phase). One warp owns kFfDirs directions: lane j holds F_n for the modes
// n = j, j + 32, ... of those directions; per 32 particles every lane forms the phases of one
// particle for the warp's directions, which are then broadcast by shuffles, and the coefficient
// rows b[s, :] are read coalesced (one particle's modes across the lanes). The angular factors
// are applied in the epilogue, the warp reduces, lane 0 writes E_theta, E_phi and (I, Q, U, V).
// The rows of 32 particles at a time are staged in shared memory by asynchronous copies (two
// buffers: the next chunk arrives while the current one is summed), so the block's 8 warps read
// each row from shared memory instead of each waiting on its own L2 load.
// Float64 throughout; every output is written by one warp in a fixed order (deterministic).
#include <cmath>

#include "capi_internal.h"

namespace yasf {

constexpr int kFfDirs = 4;   // directions per warp
constexpr int kFfModes = 5;  // modes per lane: nmax <= 160 = 5 x 32 (lmax 8)

__device__ __forceinline__ void ff_copy16(void* smem_dst, const void* gsrc) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void ff_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void ff_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Dynamic shared memory: two buffers of kFfChunk coefficient rows (kFfChunk x nmax complex128).
constexpr int kFfChunk = 32;
__global__ void __launch_bounds__(256) far_field_kernel(int L, int nmax, int n_particles, int n_dirs,
                                                        const double* pos, double k, const double2* coef,
                                                        const double* polar, const double* azimuthal,
                                                        const double* pilm, const double* taulm,
                                                        double2* e_theta, double2* e_phi, double* stokes) {
  extern __shared__ __align__(16) double2 ff_rows[];  // [2][kFfChunk * nmax]
  const int lane = threadIdx.x & 31;
  const int warp = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
  const int a0 = warp * kFfDirs;  // warps past the last direction still stage rows, write nothing
  double ex[kFfDirs], ey[kFfDirs], ez[kFfDirs];
#pragma unroll
  for (int d = 0; d < kFfDirs; ++d) {
    const int a = min(a0 + d, n_dirs - 1);
    double st, ct, sp, cp;
    sincos(polar[a], &st, &ct);
    sincos(azimuthal[a], &sp, &cp);
    ex[d] = st * cp;
    ey[d] = st * sp;
    ez[d] = ct;
  }
  const int modes = (nmax + 31) >> 5;
  double2 F[kFfDirs][kFfModes];
#pragma unroll
  for (int d = 0; d < kFfDirs; ++d)
#pragma unroll
    for (int j = 0; j < kFfModes; ++j) F[d][j] = make_double2(0.0, 0.0);
  // the block's warps share every coefficient row: a chunk of rows is copied into shared memory
  // once per block (asynchronously, the next chunk while the current one is summed)
  const int chunks = (n_particles + kFfChunk - 1) / kFfChunk;
  const int chunk_elems = kFfChunk * nmax;
  auto stage = [&](int c) {
    double2* dst = ff_rows + (size_t)(c & 1) * chunk_elems;
    const int rows = min(kFfChunk, n_particles - c * kFfChunk);
    const double2* src = coef + (size_t)c * chunk_elems;
    for (int e = threadIdx.x; e < rows * nmax; e += blockDim.x) ff_copy16(dst + e, src + e);
    ff_commit();
  };
  stage(0);
#pragma unroll 1
  for (int c = 0; c < chunks; ++c) {
    if (c + 1 < chunks) {
      stage(c + 1);
      ff_wait<1>();
    } else {
      ff_wait<0>();
    }
    __syncthreads();  // chunk c is in shared memory for every thread
    const int s0 = c * kFfChunk;
    const double2* rows = ff_rows + (size_t)(c & 1) * chunk_elems;
    // phases e^{-i k r_s . e_r} of particle s0 + lane for the warp's directions
    double pr[kFfDirs], pi[kFfDirs];
    const int sl = s0 + lane;
    const double x = sl < n_particles ? pos[3 * sl] : 0.0;
    const double y = sl < n_particles ? pos[3 * sl + 1] : 0.0;
    const double z = sl < n_particles ? pos[3 * sl + 2] : 0.0;
#pragma unroll
    for (int d = 0; d < kFfDirs; ++d) {
      double sn, cs;
      sincos(-k * (x * ex[d] + y * ey[d] + z * ez[d]), &sn, &cs);
      pr[d] = cs;
      pi[d] = sn;
    }
    const int cnt = min(kFfChunk, n_particles - s0);
#pragma unroll 1
    for (int p = 0; p < cnt; ++p) {
      const double2* row = rows + (size_t)p * nmax;
      double qr[kFfDirs], qi[kFfDirs];
#pragma unroll
      for (int d = 0; d < kFfDirs; ++d) {
        qr[d] = __shfl_sync(0xffffffffu, pr[d], p);
        qi[d] = __shfl_sync(0xffffffffu, pi[d], p);
      }
#pragma unroll
      for (int j = 0; j < kFfModes; ++j) {
        const int n = lane + 32 * j;
        if (j < modes && n < nmax) {
          const double2 b = row[n];
#pragma unroll
          for (int d = 0; d < kFfDirs; ++d) {
            F[d][j].x = fma(b.x, qr[d], fma(-b.y, qi[d], F[d][j].x));
            F[d][j].y = fma(b.x, qi[d], fma(b.y, qr[d], F[d][j].y));
          }
        }
      }
    }
    __syncthreads();  // every warp is done with buffer c & 1 before chunk c + 2 is copied into it
  }
  if (a0 >= n_dirs) return;  // whole warps only (after the block's last barrier)
  // angular factors of the lane's modes and the reduction over modes
  const int half = nmax / 2;
#pragma unroll
  for (int d = 0; d < kFfDirs; ++d) {
    const int a = a0 + d;
    const int ac = min(a, n_dirs - 1);
    double thr = 0.0, thi = 0.0, phr = 0.0, phi_ = 0.0;
#pragma unroll
    for (int j = 0; j < kFfModes; ++j) {
      const int n = lane + 32 * j;
      if (j >= modes || n >= nmax) continue;
      const int tau = n < half ? 1 : 2;
      const int rem = n - (tau - 1) * half;        // (l - 1)(l + 1) + l + m
      int l = (int)sqrt((double)(rem + 1));
      while (l * l > rem + 1) --l;
      while ((l + 1) * (l + 1) <= rem + 1) ++l;
      const int m = rem + 1 - l * l - l;
      const int am = m < 0 ? -m : m;
      const double pil = pilm[((size_t)l * (L + 1) + am) * n_dirs + ac];
      const double tal = taulm[((size_t)l * (L + 1) + am) * n_dirs + ac];
      // base = i^{tau - l - 2} / sqrt(2 l (l + 1)) e^{i m phi}
      double sm, cm;
      sincos(m * azimuthal[ac], &sm, &cm);
      const double nrm = 1.0 / sqrt(2.0 * l * (l + 1));
      const int e = ((tau - l - 2) % 4 + 4) % 4;  // i^e
      double br = e == 0 ? 1.0 : (e == 2 ? -1.0 : 0.0);
      double bi = e == 1 ? 1.0 : (e == 3 ? -1.0 : 0.0);
      const double t0r = (br * cm - bi * sm) * nrm, t0i = (br * sm + bi * cm) * nrm;
      // C_theta, C_phi: tau = 1 -> (i m pi, -tau); tau = 2 -> (tau, i m pi)
      double ctr, cti, cpr, cpi;
      if (tau == 1) {
        ctr = -t0i * m * pil; cti = t0r * m * pil;
        cpr = -t0r * tal;     cpi = -t0i * tal;
      } else {
        ctr = t0r * tal;      cti = t0i * tal;
        cpr = -t0i * m * pil; cpi = t0r * m * pil;
      }
      const double2 f = F[d][j];
      thr += ctr * f.x - cti * f.y;
      thi += ctr * f.y + cti * f.x;
      phr += cpr * f.x - cpi * f.y;
      phi_ += cpr * f.y + cpi * f.x;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      thr += __shfl_xor_sync(0xffffffffu, thr, off);
      thi += __shfl_xor_sync(0xffffffffu, thi, off);
      phr += __shfl_xor_sync(0xffffffffu, phr, off);
      phi_ += __shfl_xor_sync(0xffffffffu, phi_, off);
    }
    if (lane == 0 && a < n_dirs) {
      e_theta[a] = make_double2(thr, thi);
      e_phi[a] = make_double2(phr, phi_);
      if (stokes) {
        const double at = thr * thr + thi * thi, ap = phr * phr + phi_ * phi_;
        const double xr = thr * phr + thi * phi_;  // Re(E_theta conj(E_phi))
        const double xi = thi * phr - thr * phi_;  // Im(E_theta conj(E_phi))
        stokes[4 * (size_t)a + 0] = at + ap;
        stokes[4 * (size_t)a + 1] = at - ap;
        stokes[4 * (size_t)a + 2] = -2.0 * xr;
        stokes[4 * (size_t)a + 3] = 2.0 * xi;
      }
    }
  }
}

}  // namespace yasf

using namespace yasf;

extern "C" int yasf_far_field(int lmax, int n_particles, const double* positions, double k_medium,
                              const double* coef, int n_dirs, const double* polar, const double* azimuthal,
                              const double* pilm, const double* taulm, double* e_theta, double* e_phi,
                              double* stokes, void* stream) {
  if (lmax < 1 || lmax > YASF_LMAX_MAX) return YASF_ERR_UNSUPPORTED;
  if (n_particles <= 0 || n_dirs <= 0 || !positions || !coef || !polar || !azimuthal || !pilm || !taulm ||
      !e_theta || !e_phi)
    return YASF_ERR_INVALID_ARGUMENT;
  if (!std::isfinite(k_medium) || k_medium <= 0.0) return YASF_ERR_UNSUPPORTED;
  if (!aligned16(coef) || !aligned16(e_theta) || !aligned16(e_phi)) return YASF_ERR_ALIGNMENT;
  const int nmax = nmax_of(lmax);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const long long warps = ((long long)n_dirs + kFfDirs - 1) / kFfDirs;
  const int blocks = (int)((warps * 32 + 255) / 256);
  const size_t smem = 2 * (size_t)kFfChunk * nmax * sizeof(double2);
  YASF_CUDA_TRY(cudaFuncSetAttribute(far_field_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  YASF_COUNTED(far_field_kernel<<<blocks, 256, smem, s>>>(
      lmax, nmax, n_particles, n_dirs, positions, k_medium, reinterpret_cast<const double2*>(coef), polar,
      azimuthal, pilm, taulm, reinterpret_cast<double2*>(e_theta), reinterpret_cast<double2*>(e_phi), stokes));
  YASF_CUDA_TRY(cudaGetLastError());
  return YASF_OK;
}
