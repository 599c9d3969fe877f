// C-ABI entry points of the multi-right-hand-side tensor-core coupling (see panel.cuh).
#include "capi_internal.h"
#include "panel.cuh"

namespace yasf {

template <int L>
static int launch_panel(const PanelArgs& pa, int groups, cudaStream_t s) {
  using G = PanelGeom<L>;
  {
    const dim3 grid(pa.n_particles, groups);
    YASF_COUNTED(xpanel_kernel<L><<<grid, 256, 0, s>>>(pa.n_particles, pa.nmax, pa.nrhs, pa.ld, pa.x,
                                                     const_cast<float*>(pa.xp)));
    YASF_CUDA_TRY(cudaGetLastError());
  }
  YASF_CUDA_TRY(cudaFuncSetAttribute(panel_kernel<L>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     G::SMEM));
  const dim3 grid(pa.n_particles, groups);
  YASF_COUNTED(panel_kernel<L><<<grid, 160, G::SMEM, s>>>(pa));
  YASF_CUDA_TRY(cudaGetLastError());
  return YASF_OK;
}

static size_t panel_xstage(int L) {
  switch (L) {
    case 1: return PanelGeom<1>::X_STAGE;
    case 2: return PanelGeom<2>::X_STAGE;
    case 3: return PanelGeom<3>::X_STAGE;
    case 4: return PanelGeom<4>::X_STAGE;
    case 5: return PanelGeom<5>::X_STAGE;
    case 6: return PanelGeom<6>::X_STAGE;
    default: return 0;
  }
}

}  // namespace yasf

using namespace yasf;

extern "C" int yasf_panel_workspace_size(const yasf_plan* plan, int n_particles, int nrhs,
                                         size_t* bytes) {
  if (!plan || !bytes || n_particles <= 0 || nrhs <= 0) return YASF_ERR_INVALID_ARGUMENT;
  const size_t xs = panel_xstage(plan->lmax);
  if (!xs) return YASF_ERR_UNSUPPORTED;
  const size_t groups = (size_t)(nrhs + 63) / 64;
  *bytes = ((groups * n_particles * xs + 255) & ~size_t(255)) + 256;
  return YASF_OK;
}

extern "C" int yasf_panel_matvec(const yasf_plan* plan, int n_particles, const double* positions,
                                 double k_medium, const double* tmat, const double* x, double* y,
                                 int nrhs, long long ldx, long long ldy, void* workspace,
                                 size_t workspace_bytes, void* stream) {
  int st = validate_coupling(plan, n_particles, positions, k_medium, YASF_C64);
  if (st != YASF_OK) return st;
  if (!x || !y || x == y || nrhs <= 0) return YASF_ERR_INVALID_ARGUMENT;
  const long long n = (long long)n_particles * plan->nmax;
  if (nrhs == 1) ldx = ldy = n;
  if (ldx < n || ldy < n) return YASF_ERR_INVALID_ARGUMENT;
  if (!aligned16(x) || !aligned16(y) || (tmat && !aligned16(tmat)) || !aligned16(workspace))
    return YASF_ERR_ALIGNMENT;
  size_t need = 0;
  if ((st = yasf_panel_workspace_size(plan, n_particles, nrhs, &need)) != YASF_OK) return st;
  if (!workspace || workspace_bytes < need) return YASF_ERR_WORKSPACE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  char* ws = static_cast<char*>(workspace);
  int* err = reinterpret_cast<int*>(ws + need - 256);
  YASF_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), s));
  PanelArgs pa{};
  pa.n_particles = n_particles;
  pa.nmax = plan->nmax;
  pa.nrhs = nrhs;
  pa.ld = ldx;
  pa.ldy = ldy;
  pa.k = k_medium;
  pa.pos = positions;
  pa.leg = plan->d_leg;
  pa.xp = reinterpret_cast<const float*>(ws);
  pa.w_ptr = plan->d_w_ptr;
  pa.w_p = plan->d_w_p;
  pa.w_coef = plan->d_w_coef;
  pa.x = reinterpret_cast<const double2*>(x);
  pa.tmat = reinterpret_cast<const double2*>(tmat);
  pa.y = reinterpret_cast<double2*>(y);
  pa.err = err;
  const int groups = (nrhs + 63) / 64;
  switch (plan->lmax) {
    case 1: return launch_panel<1>(pa, groups, s);
    case 2: return launch_panel<2>(pa, groups, s);
    case 3: return launch_panel<3>(pa, groups, s);
    case 4: return launch_panel<4>(pa, groups, s);
    case 5: return launch_panel<5>(pa, groups, s);
    case 6: return launch_panel<6>(pa, groups, s);
    default: return YASF_ERR_UNSUPPORTED;
  }
}
