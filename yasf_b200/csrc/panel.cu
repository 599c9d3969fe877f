// C-ABI entry points of the multi-right-hand-side tensor-core coupling (see panel.cuh).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "capi_internal.h"
#include "panel.cuh"

namespace yasf {

// IEEE half-precision bits of a float (round to nearest even; normal range, tiny values flush to 0).
static unsigned short half_bits(float f) {
  unsigned u;
  std::memcpy(&u, &f, sizeof(u));
  const unsigned sign = (u >> 16) & 0x8000u;
  int exp = (int)((u >> 23) & 0xFFu) - 127 + 15;
  unsigned m = (u & 0x7FFFFFu) >> 13;
  const unsigned rem = u & 0x1FFFu;
  if (exp <= 0) return (unsigned short)sign;
  if (exp >= 31) return (unsigned short)(sign | 0x7BFFu);
  if (rem > 0x1000u || (rem == 0x1000u && (m & 1u))) {
    if (++m == 0x400u) {
      m = 0;
      if (++exp >= 31) return (unsigned short)(sign | 0x7BFFu);
    }
  }
  return (unsigned short)(sign | ((unsigned)exp << 10) | m);
}

// Generation data of the panel kernel from the build-time schedule (panel_sched.h). For every
// generator thread and slot: the real coefficient and the byte offset of A[p][|d|] of one term of
// the thread's item; for every step: the W-stage byte offsets of the P_r rows of the item's entry
// and of its mirror, and the byte offset of the entry's phase e^{i d phi}. Up to lmax 6 the slot
// of each term, and the entry a slot without a term reads (zero coefficient), come from the
// schedule's slot table (kPanelSlot: a half-warp's loads of one slot hit different banks). Packed variant
// (lmax 7-8): goff holds the FP16 coefficients two per word and the third dst row the step's
// pair-table bases (Wa | Wb << 10 | phase << 20, entry units); slot q of a step's Wa (Wb) terms is
// the term at p = p0 + 2q, with the window starts p0 from the schedule (kPanelWindow; they keep
// every window inside table rows 0 .. 2L + 1 and are checked here against the item's terms). Wa
// coefficients are real and Wb coefficients purely imaginary (a5 / b5 of the plan); the Wb value
// stored is b / i.
// The mirror entry's coefficients are not stored: they equal the entry's (Wa) or their negatives
// (Wb), which the kernel applies. Terms below 1e-12 of the largest coefficient cannot change a
// TF32 entry and are dropped.
template <int L>
static int build_terms_for(const double* ab5, const unsigned short* entry, const unsigned short* slots,
                           const unsigned short* window,
                           const unsigned char* wa, const unsigned char* wb, std::vector<float>& coef,
                           std::vector<unsigned>& goff, std::vector<unsigned>& dst) {
  using Sched = PanelSched<L>;
  constexpr int S = Sched::kSlots, NS = Sched::kSteps;
  const int nmax = 2 * L * (L + 2), P = 2 * L + 1;
  const int H = L * (L + 2), HP = pad8(H);
  auto lm = [](int q, int& l, int& m) {
    l = 1;
    while ((l + 1) * (l + 1) - 1 <= q) ++l;
    m = q + 1 - l * l - l;
  };
  auto mirror = [&](int q) {
    int l, m;
    lm(q, l, m);
    return l * l + l - 1 - m;
  };
  double cmax = 0.0;
  for (size_t q = 0; q < (size_t)nmax * nmax * P * 2; ++q) cmax = std::max(cmax, std::fabs(ab5[q]));
  const double cut = 1e-12 * cmax;
  auto coefficient = [&](int which, int q1, int q2, int p, double& cr, double& ci) {
    // A[(tau1=1,q1), (tau2=which+1,q2), p] = translation_ab5[n2][n1][p]
    const size_t idx = ((size_t)(which * H + q2) * nmax + q1) * P + p;
    cr = ab5[2 * idx];
    ci = ab5[2 * idx + 1];
    if (std::fabs(cr) <= cut) cr = 0.0;
    if (std::fabs(ci) <= cut) ci = 0.0;
  };
  // the schedule relies on: coefficients only inside the selection rules, Wa real, Wb imaginary,
  // and the mirror entry carrying the same Wa and the negated Wb coefficients
  for (int which = 0; which < 2; ++which)
    for (int q1 = 0; q1 < H; ++q1)
      for (int q2 = 0; q2 < H; ++q2) {
        int l1, m1, l2, m2;
        lm(q1, l1, m1);
        lm(q2, l2, m2);
        const int pmin = std::max(std::abs(l1 - l2), std::abs(m2 - m1));
        for (int p = 0; p < P; ++p) {
          double cr, ci, mr, mi;
          coefficient(which, q1, q2, p, cr, ci);
          coefficient(which, mirror(q1), mirror(q2), p, mr, mi);
          const bool in_rule = p >= pmin && p <= l1 + l2 && ((l1 + l2 + p) % 2 == 0) == (which == 0);
          if (!in_rule && (cr != 0.0 || ci != 0.0)) return YASF_ERR_INVALID_ARGUMENT;
          if ((which == 0 && ci != 0.0) || (which == 1 && cr != 0.0)) return YASF_ERR_INVALID_ARGUMENT;
          const double sgn = which == 0 ? 1.0 : -1.0;
          const double tol = 1e-12 * std::max(1.0, std::fabs(cr) + std::fabs(ci));
          if (std::fabs(mr - sgn * cr) > tol || std::fabs(mi - sgn * ci) > tol)
            return YASF_ERR_INVALID_ARGUMENT;
        }
      }
  constexpr bool PK = PanelGeom<L>::PACKED;
  coef.assign((size_t)S * kGenThreads, 0.f);
  goff.assign((size_t)(PK ? (S + 1) / 2 : S) * kGenThreads, 0u);
  dst.assign((size_t)3 * NS * kGenThreads, 0u);
  for (int th = 0; th < kGenThreads; ++th) {
    const int w = th >> 5, lane = th & 31;
    if constexpr (!PK)  // every slot reads its schedule entry; slots without a term keep coefficient 0
      for (int q = 0; q < S; ++q) goff[(size_t)q * kGenThreads + th] = (slots[(size_t)th * S + q] & 0xFFu) * 8u;
    int base = 0;
    for (int k = 0; k < NS; ++k) {
      const unsigned e = entry[((size_t)w * NS + k) * 32 + lane];
      const int q1 = (int)(e >> 8), q2 = (int)(e & 255);
      const bool real = q1 < H && q2 < H;
      const int mq1 = real ? mirror(q1) : q1, mq2 = real ? mirror(q2) : q2;
      int l1 = 0, m1 = 0, l2 = 0, m2 = 0;
      if (real) {
        lm(q1, l1, m1);
        lm(q2, l2, m2);
      }
      dst[(size_t)k * kGenThreads + th] = (unsigned)kmajor_offset(q1, q2, 2 * HP);
      dst[(size_t)(NS + k) * kGenThreads + th] = (unsigned)kmajor_offset(mq1, mq2, 2 * HP);
      const int ad = std::abs(m2 - m1);
      const int pmin = std::max(std::abs(l1 - l2), ad);
      // packed variant: window starts p0 of the Wa and Wb terms (inside rows 0 .. 2L + 1)
      const unsigned wv = window[((size_t)w * NS + k) * 32 + lane];
      const int p0[2] = {(int)(wv & 255u), (int)(wv >> 8)};
      if (PK && (p0[0] + 2 * (wa[k] - 1) > 2 * L + 1 || p0[1] + 2 * (wb[k] - 1) > 2 * L + 1))
        return YASF_ERR_INVALID_ARGUMENT;
      dst[(size_t)(2 * NS + k) * kGenThreads + th] =
          PK ? (unsigned)(p0[0] * P + ad) | ((unsigned)(p0[1] * P + ad) << 10) |
                   ((unsigned)(P * P + 2 * L + (m2 - m1)) << 20)
             : (unsigned)((P * P + 2 * L + (m2 - m1)) * 8);
      if (real) {
        int na = 0, nb = 0;
        for (int p = pmin; p <= l1 + l2; ++p) {
          const int which = ((l1 + l2 + p) % 2 == 0) ? 0 : 1;
          double cr, ci;
          coefficient(which, q1, q2, p, cr, ci);
          const int T = which == 0 ? wa[k] : wb[k], off = which == 0 ? base : base + wa[k];
          int j = -1;
          if constexpr (PK) {
            j = (p - p0[which]) % 2 == 0 ? (p - p0[which]) / 2 : -1;
          } else {
            // the schedule's slot of this term (entries flagged 0x100 carry no term)
            for (int q = 0; q < T; ++q)
              if (slots[(size_t)th * S + off + q] == (unsigned)(p * P + ad)) j = q;
          }
          which == 0 ? ++na : ++nb;
          if (na > wa[k] || nb > wb[k] || j < 0 || j >= T) return YASF_ERR_INVALID_ARGUMENT;
          const int slot = which == 0 ? base + j : base + wa[k] + j;
          const float cf = (float)(which == 0 ? cr : ci);
          coef[(size_t)slot * kGenThreads + th] = cf;
          if constexpr (PK) goff[(size_t)(slot >> 1) * kGenThreads + th] |= (unsigned)half_bits(cf) << (16 * (slot & 1));
        }
      }
      base += wa[k] + wb[k];
    }
    if (base != S) return YASF_ERR_INVALID_ARGUMENT;
  }
  return YASF_OK;
}

int panel_build_terms(int L, const double* ab5, std::vector<float>& coef, std::vector<unsigned>& goff,
                      std::vector<unsigned>& dst) {
  coef.clear();
  goff.clear();
  dst.clear();
#define YASF_TERMS(n)                                                                             \
  case n:                                                                                         \
    return build_terms_for<n>(ab5, kPanelEntry##n, kPanelSlot##n, kPanelWindow##n, kPanelStepWa##n,   \
                              kPanelStepWb##n, coef, goff, dst);
  switch (L) {
    YASF_TERMS(1)
    YASF_TERMS(2)
    YASF_TERMS(3)
    YASF_TERMS(4)
    YASF_TERMS(5)
    YASF_TERMS(6)
    YASF_TERMS(7)
    YASF_TERMS(8)
    default: return YASF_OK;
  }
#undef YASF_TERMS
}

// Right-hand-side groups of 64 per panel block: two as soon as there are two (each W_ij is then
// generated once for 128 columns), padded to an even count whose extra columns are zero.
// lmax 8 keeps one group per block: two groups' accumulators would exceed tensor memory.
static int panel_groups_per_block(int groups, int lmax) {
  if (tile_config().panel_groups == 1) return 1;
  return groups >= 2 && lmax <= 7 ? 2 : 1;
}
static int panel_padded_groups(int groups, int lmax) {
  const int ng = panel_groups_per_block(groups, lmax);
  return (groups + ng - 1) / ng * ng;
}

template <int L, int NG>
static int launch_panel_ng(const PanelArgs& pa, int padded, cudaStream_t s) {
  using G = PanelGeom<L>;
  YASF_CUDA_TRY(cudaFuncSetAttribute(panel_kernel<L, NG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     G::SMEM));
  const dim3 grid(pa.n_particles, padded / NG);
  YASF_COUNTED(panel_kernel<L, NG><<<grid, kPanelThreads, G::SMEM, s>>>(pa));
  YASF_CUDA_TRY(cudaGetLastError());
  return YASF_OK;
}

template <int L>
static int launch_panel(const PanelArgs& pa, int groups, cudaStream_t s) {
  const int padded = panel_padded_groups(groups, L);
  {
    const dim3 grid(pa.n_particles, padded);
    YASF_COUNTED(xpanel_kernel<L><<<grid, 256, 0, s>>>(pa.n_particles, pa.nmax, pa.nrhs, pa.ld, pa.x,
                                                     const_cast<float*>(pa.xp)));
    YASF_CUDA_TRY(cudaGetLastError());
  }
  if constexpr (4 * PanelGeom<L>::HP * 2 <= 512) {
    if (panel_groups_per_block(groups, L) == 2) return launch_panel_ng<L, 2>(pa, padded, s);
  }
  return launch_panel_ng<L, 1>(pa, padded, s);
}

static size_t panel_xstage(int L) {
  switch (L) {
    case 1: return PanelGeom<1>::X_STAGE;
    case 2: return PanelGeom<2>::X_STAGE;
    case 3: return PanelGeom<3>::X_STAGE;
    case 4: return PanelGeom<4>::X_STAGE;
    case 5: return PanelGeom<5>::X_STAGE;
    case 6: return PanelGeom<6>::X_STAGE;
    case 7: return PanelGeom<7>::X_STAGE;
    case 8: return PanelGeom<8>::X_STAGE;
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
  const size_t groups = (size_t)panel_padded_groups((nrhs + 63) / 64, plan->lmax);
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
  if (!plan->d_gen_c1 || !plan->d_gen_dst) return YASF_ERR_UNSUPPORTED;
  pa.gen_coef = plan->d_gen_c1;
  pa.gen_goff = plan->d_gen_meta;
  pa.gen_dst = plan->d_gen_dst;
  pa.x = reinterpret_cast<const double2*>(x);
  pa.tmat = reinterpret_cast<const double2*>(tmat);
  pa.y = reinterpret_cast<double2*>(y);
  pa.err = err;
  pa.wait_ns = stall_hook().panel_wait_ns;
  pa.stall = stall_hook().role == YASF_STALL_PANEL ? 1 : 0;
  const int groups = (nrhs + 63) / 64;
  switch (plan->lmax) {
    case 1: return launch_panel<1>(pa, groups, s);
    case 2: return launch_panel<2>(pa, groups, s);
    case 3: return launch_panel<3>(pa, groups, s);
    case 4: return launch_panel<4>(pa, groups, s);
    case 5: return launch_panel<5>(pa, groups, s);
    case 6: return launch_panel<6>(pa, groups, s);
    case 7: return launch_panel<7>(pa, groups, s);
    case 8: return launch_panel<8>(pa, groups, s);
    default: return YASF_ERR_UNSUPPORTED;
  }
}
