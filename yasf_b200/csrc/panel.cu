// C-ABI entry points of the multi-right-hand-side tensor-core coupling (see panel.cuh).
#include <algorithm>
#include <cmath>

#include "capi_internal.h"
#include "panel.cuh"

namespace yasf {

// Generation terms of the W blocks for the panel kernel, balanced over the 256 generator threads
// (longest-processing-time assignment of whole entries) and laid out [term][thread].
int panel_build_terms(int L, const double* ab5, std::vector<float>& c1, std::vector<unsigned>& meta) {
  c1.clear();
  meta.clear();
  if (L < 1 || L > 6) return YASF_OK;  // no tensor-core panel beyond lmax 6
  const int nmax = 2 * L * (L + 2), P = 2 * L + 1, DW = 4 * L + 1;
  const int H = L * (L + 2), HP = pad8(H);
  const int W_PLANE_F = (HP / 4) * (HP / 8) * 128 / 4;
  const int TM = gen_terms_max(L);
  auto m_of = [](int q) {
    int l = 1;
    while ((l + 1) * (l + 1) - 1 <= q) ++l;
    return q + 1 - l * l - l;
  };
  struct Term { float c; unsigned meta; };
  std::vector<std::vector<Term>> entries;
  double cmax = 0.0;  // terms below 1e-12 of the largest coefficient cannot change a TF32 entry
  for (size_t q = 0; q < (size_t)nmax * nmax * P * 2; ++q) cmax = std::max(cmax, std::fabs(ab5[q]));
  const double cut = 1e-12 * cmax;
  for (int which = 0; which < 2; ++which)
    for (int q1 = 0; q1 < H; ++q1)
      for (int q2 = 0; q2 < H; ++q2) {
        std::vector<Term> ts;
        const int delta = m_of(q2) - m_of(q1) + 2 * L;
        const unsigned dst = (unsigned)(which * 2 * W_PLANE_F + kmajor_offset(q1, q2, HP) / 4);
        for (int p = 0; p < P; ++p) {
          // coefficient A[(tau1=1,q1), (tau2=which+1,q2), p] = translation_ab5[n2][n1][p]
          const size_t idx = ((size_t)(which * H + q2) * nmax + q1) * P + p;
          double cr = ab5[2 * idx], ci = ab5[2 * idx + 1];
          if (std::fabs(cr) <= cut) cr = 0.0;
          if (std::fabs(ci) <= cut) ci = 0.0;
          if (cr == 0.0 && ci == 0.0) continue;
          if (cr != 0.0 && ci != 0.0) return YASF_ERR_INVALID_ARGUMENT;  // not real x i^k
          const bool odd = cr == 0.0;
          Term t;
          t.c = (float)(odd ? -ci : cr);
          t.meta = (unsigned)(p * DW + delta) | (odd ? kMetaOdd : 0u);
          ts.push_back(t);
        }
        if (ts.empty()) continue;
        ts.front().meta |= kMetaFirst;
        ts.back().meta |= kMetaLast | (dst << 13);
        entries.push_back(ts);
      }
  std::vector<int> order(entries.size());
  for (size_t e = 0; e < entries.size(); ++e) order[e] = (int)e;
  std::stable_sort(order.begin(), order.end(),
                   [&](int x, int y) { return entries[x].size() > entries[y].size(); });
  std::vector<std::vector<Term>> per(kGenThreads);
  for (int e : order) {
    int best = 0;
    for (int th = 1; th < kGenThreads; ++th)
      if (per[th].size() < per[best].size()) best = th;
    per[best].insert(per[best].end(), entries[e].begin(), entries[e].end());
    if ((int)per[best].size() > TM) return YASF_ERR_UNSUPPORTED;
  }
  c1.assign((size_t)TM * kGenThreads, 0.f);
  meta.assign((size_t)TM * kGenThreads, 0u);
  for (int th = 0; th < kGenThreads; ++th)
    for (size_t t = 0; t < per[th].size(); ++t) {
      c1[t * kGenThreads + th] = per[th][t].c;
      meta[t * kGenThreads + th] = per[th][t].meta;
    }
  return YASF_OK;
}

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
  YASF_COUNTED(panel_kernel<L><<<grid, kPanelThreads, G::SMEM, s>>>(pa));
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
  if (!plan->d_gen_c1) return YASF_ERR_UNSUPPORTED;
  pa.gen_c1 = plan->d_gen_c1;
  pa.gen_meta = plan->d_gen_meta;
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
