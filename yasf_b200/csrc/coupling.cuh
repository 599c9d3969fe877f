// Coupling matvec kernels: y = W x with every translation block W_ij generated on the fly.
//
// The reference evaluates, for receiver row j1 = (s1, n1=(tau1,l1,m1))
// (yasfpy/functions/cpu_numba.py:22-95):
//   (W x)[s1,n1] = sum_{s2 != s1} sum_{n2} e^{i(m2-m1)phi} x[s2,n2]
//                  sum_p A[n2,n1,p] Pn_p^{|m1-m2|}(cos theta) h_p(k r)
// with (r, theta, phi) the spherical coordinates of pos[s1] - pos[s2]
// (yasfpy/functions/misc.py:149-166), Pn the CELES-normalised Legendre functions
// (yasfpy/functions/legendre_normalized_trigon.py:61-91) and A the a5/b5 table
// (yasfpy/numerics.py:187-281).
//
// The same bilinear sum is evaluated here in factored form. With delta = m2 - m1,
//   G_ij[p, delta] = Pn_p^{|delta|}(cos theta_ij) h_p(k r_ij) e^{i delta phi_ij}   (pair side)
//   V_j[n1; p, m2] = sum_{tau2,l2} A[(tau2,l2,m2),(tau1,l1,m1),p] x[s_j,(tau2,l2,m2)] (source side)
//   (W x)[s_i, n1] = sum_{j != i} sum_{(p,m2)} G_ij[p, m2-m1] V_j[n1; p, m2].
// V depends on the source particle only, so it is formed once per matvec (vbuild_kernel); the
// pair loop (contract_kernel) keeps the Hankel/Legendre/phase recurrences in registers and
// performs one complex multiply-add per stream entry. Lanes are receiving particles: all lanes
// of a block walk the same source sequence, so every V load is a warp-uniform broadcast.
#pragma once

#include <cuda_runtime.h>

#include "yasf_common.cuh"

namespace yasf {

// Process-wide count of kernels launched by this library (instrumentation for benchmarks).
void count_launch();
#define YASF_COUNTED(...) (::yasf::count_launch(), (__VA_ARGS__))

// Legendre recurrence constants (CELES form, yasfpy/functions/legendre_normalized_trigon.py:61-91)
// live in plan-owned device memory, row stride YASF_PMAX_MAX + 1:
//   Pn_{l+1}^m = alpha[l][m] ct Pn_l^m - beta[l][m] Pn_{l-1}^m,   Pn_m^m = start[m] st^m.
constexpr int kLegStride = YASF_PMAX_MAX + 1;
struct LegendreTables {
  double alpha[kLegStride * kLegStride];
  double beta[kLegStride * kLegStride];
  double start[kLegStride];
};

template <typename Real> struct Cplx;
template <> struct Cplx<double> { using T = double2; };
template <> struct Cplx<float> { using T = float2; };

// One entry of the V stream. Float64: (re, im). Complex64: (re, im, -im, re), 16 bytes, so that
// one broadcast shared load feeds a complex multiply-add as two packed FP32 FMAs (FFMA2):
//   (y_re, y_im) += (g_re, g_re) * (re, im) + (g_im, g_im) * (-im, re).
template <typename Real> struct VEntry;
template <> struct VEntry<double> { using T = double2; };
template <> struct VEntry<float> { using T = float4; };

// ---------------------------------------------------------------------------------------------
// Source side: V[bundle][s][entry] = sum_terms coef * x[s][n2].
// Entries of all bundles are numbered globally; entry_ptr (CSR into term arrays) has one extra
// element; entry_dst gives (bundle offset, in-bundle index) packed as the per-source stride.
struct VBuildArgs {
  int n_particles;
  int nmax;
  int total_entries;             // sum over bundles of padded stream lengths
  int n_bundles;
  int bundle_begin[8];           // global entry index where each bundle starts
  int bundle_len[8];             // padded stream length of each bundle
  const int* entry_ptr;          // [total_entries + 1]
  const int* term_n2;            // source mode index of each term
  const double2* term_coef;      // complex coefficient of each term
  const double2* x;              // source coefficients (complex128), column base
  void* v;                       // output stream buffer (VEntry<Real>)
};

template <typename Real>
__global__ void __launch_bounds__(256) vbuild_kernel(VBuildArgs a) {
  using C = typename VEntry<Real>::T;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= a.total_entries) return;
  int b = 0;
#pragma unroll 1
  while (b + 1 < a.n_bundles && g >= a.bundle_begin[b + 1]) ++b;
  const int t0 = __ldg(a.entry_ptr + g), t1 = __ldg(a.entry_ptr + g + 1);
#pragma unroll 1
  for (int s = blockIdx.y; s < a.n_particles; s += gridDim.y) {
    const double2* xs = a.x + (size_t)s * a.nmax;
    double re = 0.0, im = 0.0;
    for (int t = t0; t < t1; ++t) {
      const double2 c = __ldg(a.term_coef + t);
      const double2 xv = __ldg(xs + __ldg(a.term_n2 + t));
      re = fma(c.x, xv.x, re);
      re = fma(-c.y, xv.y, re);
      im = fma(c.x, xv.y, im);
      im = fma(c.y, xv.x, im);
    }
    C* out = reinterpret_cast<C*>(a.v) + (size_t)a.bundle_begin[b] * a.n_particles +
             (size_t)s * a.bundle_len[b] + (g - a.bundle_begin[b]);
    if constexpr (sizeof(Real) == 8) {
      *out = make_double2(re, im);
    } else {
      *out = make_float4((float)re, (float)im, -(float)im, (float)re);
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Spherical Bessel j_p(x), p = 0..pmax, by Miller's downward recurrence (stable for all x >= 0),
// normalised with whichever of j_0, j_1 is larger in magnitude. j_p(0) = delta_{p0}.
__device__ __forceinline__ void regular_bessel(double x, int pmax, double* jp) {
  if (x == 0.0) {
    jp[0] = 1.0;
    for (int p = 1; p <= pmax; ++p) jp[p] = 0.0;
    return;
  }
  const int nstart = pmax + 20 + (int)x;
  const double inv_x = 1.0 / x;
  double f_next = 0.0, f = 1e-200;
#pragma unroll 1
  for (int q = nstart; q > pmax; --q) {
    const double f_prev = (2.0 * q + 1.0) * inv_x * f - f_next;
    f_next = f;
    f = f_prev;
    if (fabs(f) > 1e200) { f *= 1e-200; f_next *= 1e-200; }
  }
  // f = f_pmax, f_next = f_{pmax+1}
  jp[pmax] = f;
  double fn = f_next;
#pragma unroll 1
  for (int q = pmax; q > 0; --q) {
    const double fp = (2.0 * q + 1.0) * inv_x * jp[q] - fn;
    fn = jp[q];
    jp[q - 1] = fp;
    if (fabs(fp) > 1e200) {
      for (int t = q - 1; t <= pmax; ++t) jp[t] *= 1e-200;
      fn *= 1e-200;
    }
  }
  double s, c;
  sincos(x, &s, &c);
  const double j0 = s * inv_x;
  const double j1 = (s * inv_x - c) * inv_x;
  double scale;
  if (fabs(j0) >= fabs(j1)) scale = j0 / jp[0];
  else scale = j1 / (pmax >= 1 ? jp[1] : ((3.0 * inv_x) * jp[0]));
  for (int p = 0; p <= pmax; ++p) jp[p] *= scale;
}

// ---------------------------------------------------------------------------------------------
// Pair side + contraction. One thread per receiving particle; blockIdx.x = receiver tile,
// blockIdx.y = source chunk, blockIdx.z = bundle of receiving orders m1.
struct ContractArgs {
  int n_particles;
  int nmax;
  int sources_per_chunk;
  double k;
  const double* pos;             // (N,3)
  const void* v;                 // stream buffer (VEntry<Real>), bundle-major
  const LegendreTables* leg;     // device Legendre recurrence constants
  int bundle_begin[8];           // stream offset of each bundle (entries, per-source layout)
  int bundle_len[8];             // padded stream length per source
  void* partial;                 // (chunks, N, nmax) Real2 partial sums
  int* err;                      // set to 1 if a shared-memory stage wait timed out
  double cutoff2;                // >= 0: only pairs with |pos[s1] - pos[s2]|^2 <= cutoff2 (near field)
  int poll_limit;                // polls of one stage wait before it gives up (2^22 normally)
  int stall;                     // test hook: 1 = the first stage copy of every block is never
                                 // issued, so its wait runs out (0 normally)
};

// ---- bulk async copy (TMA, non-tensor) into shared memory with an mbarrier --------------------
__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// One elected thread: expect `bytes` on `bar` and start the copy global -> shared.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes,
                                          unsigned long long* bar) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
// Bounded wait for phase `parity` of `bar`; returns false after `limit` polls.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity,
                                          int limit = 1 << 22) {
  const unsigned a = smem_addr(bar);
#pragma unroll 1
  for (int spin = 0; spin < limit; ++spin) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// One (receiver tile, source chunk) of bundle BID. The two stage barriers are initialised by the
// caller; `uses` (every thread, uniform) counts the phases of each stage consumed so far and
// `issued` (thread 0) the copies issued into each, both carried across calls, so a persistent
// block can process many work items with the same barriers. Returns false when a stage wait ran
// out (the error word is set, the copies in flight are drained, the block must stop).
template <int L, int NB, int BID, typename Real, bool REGULAR>
__device__ __forceinline__ bool contract_body(const ContractArgs& a, int tile, int chunk, char* smem,
                                              unsigned long long* bars, unsigned (&uses)[2],
                                              unsigned (&issued)[2]) {
  using C = typename Cplx<Real>::T;
  using VE = typename VEntry<Real>::T;
  constexpr bool F64 = sizeof(Real) == 8;
  constexpr BundleInfo bi = make_bundle(L, BID, NB);
  constexpr int NR = bi.rows;
  constexpr int PMAX = 2 * L;

  const int s1 = tile * blockDim.x + threadIdx.x;
  const bool active = s1 < a.n_particles;
  const int s1c = active ? s1 : 0;
  const double x1 = __ldg(a.pos + 3 * s1c + 0);
  const double y1 = __ldg(a.pos + 3 * s1c + 1);
  const double z1 = __ldg(a.pos + 3 * s1c + 2);

  // accumulators: float64 as separate real / imaginary arrays, complex64 as packed float2 pairs
  Real yr[F64 ? NR : 1], yi[F64 ? NR : 1];
  float2 yc[F64 ? 1 : NR];
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    if constexpr (F64) { yr[r] = (Real)0; yi[r] = (Real)0; }
    else yc[r] = make_float2(0.f, 0.f);
  }

  const int c = chunk;
  const int sb = c * a.sources_per_chunk;
  const int se = min(a.n_particles, sb + a.sources_per_chunk);
  const VE* vbase = reinterpret_cast<const VE*>(a.v) + (size_t)a.bundle_begin[BID] * a.n_particles;
  const int vstride = a.bundle_len[BID];
  const unsigned stage_bytes = (unsigned)(vstride * sizeof(VE));
  VE* const stage0 = reinterpret_cast<VE*>(smem);
  VE* const stage1 = stage0 + vstride;
  // Thread 0 issues every stage copy and counts them per stage, so that a block that gives up
  // drains exactly the copies still in flight (issued[b] > uses[b]).
  if (threadIdx.x == 0 && sb < se && !a.stall) {
    bulk_load(stage0, vbase + (size_t)sb * vstride, stage_bytes, &bars[0]);
    ++issued[0];
  }
  bool timed_out = false;

#pragma unroll 1
  for (int s2 = sb; s2 < se; ++s2) {
    const int it = s2 - sb;
    const int cur = it & 1;
    // prefetch the next source's stream into the other stage (read last in iteration it-1,
    // released by the barrier at the end of that iteration)
    if (threadIdx.x == 0 && s2 + 1 < se) {
      bulk_load(cur ? stage0 : stage1, vbase + (size_t)(s2 + 1) * vstride, stage_bytes,
                &bars[cur ^ 1]);
      ++issued[cur ^ 1];
    }
    // ---- pair geometry: d = pos[s1] - pos[s2] (yasfpy/functions/misc.py:149-166) ----
    const double dx = x1 - __ldg(a.pos + 3 * s2 + 0);
    const double dy = y1 - __ldg(a.pos + 3 * s2 + 1);
    const double dz = z1 - __ldg(a.pos + 3 * s2 + 2);
    const double r2 = dx * dx + dy * dy + dz * dz;
    const bool self = (s2 == s1c);
    // Regular form keeps self pairs (r = 0: cos theta = 0, phi = 0, j_p(0) = delta_p0). With a
    // near-field cutoff only the pairs within it contribute (the others are masked like self pairs).
    const bool use = active && (REGULAR ? true : !self) && (a.cutoff2 < 0.0 || r2 <= a.cutoff2);
    double r = sqrt(r2);
    double ct = (r > 0.0) ? dz / r : 0.0;
    ct = fmin(1.0, fmax(-1.0, ct));
    const double st = sqrt(1.0 - ct * ct);
    const double rho = sqrt(dx * dx + dy * dy);
    const double ephr = (rho > 0.0) ? dx / rho : 1.0;
    const double ephi = (rho > 0.0) ? dy / rho : 0.0;
    const double kr = a.k * r;
    const double mask = use ? 1.0 : 0.0;

    // Hankel h_0, h_1 of the first kind (h_p = j_p + i y_p), or regular j_p table.
    Real h0r = 0, h0i = 0, h1r = 0, h1i = 0, inv_x = 0;
    double jp[REGULAR ? PMAX + 1 : 1];
    if constexpr (!REGULAR) {
      const double xx = (use && kr > 0.0) ? kr : 1.0;
      double sx, cx;
      sincos(xx, &sx, &cx);
      const double ix = 1.0 / xx;
      // h_0 = -i e^{ix}/x ; h_1 = -e^{ix}(x + i)/x^2
      h0r = (Real)(mask * sx * ix);
      h0i = (Real)(-mask * cx * ix);
      h1r = (Real)(mask * (sx - xx * cx) * ix * ix);
      h1i = (Real)(-mask * (cx + xx * sx) * ix * ix);
      inv_x = (Real)ix;
    } else {
      regular_bessel(use ? kr : 0.0, PMAX, jp);
      for (int p = 0; p <= PMAX; ++p) jp[p] *= mask;
    }

    // block-uniform decision: every thread polls (bounded), then all agree before using the stage
    const bool ok = mbar_wait(&bars[cur], uses[cur] & 1u, a.poll_limit);
    if (__syncthreads_or(!ok)) {
      timed_out = true;
      if (threadIdx.x == 0) atomicExch(a.err, 1);
      break;
    }
    ++uses[cur];
    // with a cutoff, a source that no receiver of the block is near is skipped as a whole
    // (a.cutoff2 is uniform, so is the extra barrier)
    if (a.cutoff2 >= 0.0 && !__syncthreads_or(use)) {
      __syncthreads();
      continue;
    }
    const VE* vp = cur ? stage1 : stage0;
    const Real ctR = (Real)ct, stR = (Real)st;
    const Real eR = (Real)ephr, eI = (Real)ephi;
    Real st_d = (Real)1, ph_r = (Real)1, ph_i = (Real)0;

#pragma unroll 1
    for (int d = 0; d <= PMAX; ++d) {
      if (d > 0) {
        st_d *= stR;
        const Real t = ph_r * eR - ph_i * eI;
        ph_i = ph_r * eI + ph_i * eR;
        ph_r = t;
      }
      Real P_prev = (Real)0;
      Real P_cur = (Real)__ldg(a.leg->start + d) * st_d;
      // Restart the Hankel recurrence and advance it to order d.
      Real ha_r = h0r, ha_i = h0i, hb_r = h1r, hb_i = h1i;
      if constexpr (!REGULAR) {
#pragma unroll 1
        for (int q = 0; q < d; ++q) {
          const Real f = (Real)(2 * q + 3) * inv_x;
          const Real nr = f * hb_r - ha_r;
          const Real ni = f * hb_i - ha_i;
          ha_r = hb_r; ha_i = hb_i; hb_r = nr; hb_i = ni;
        }
      }
      // The orders p of the contraction for this source. With float64 the p loop is unrolled (d is
      // a warp-uniform runtime value): the valid row counts of every (m1, p) become compile-time
      // and the row loops carry no predicates. With float32 the rolled loop from p = d is faster.
      constexpr int kPUnroll = sizeof(Real) == 8 ? PMAX + 1 : 1;
#pragma unroll kPUnroll
      for (int p = (sizeof(Real) == 8 ? 0 : d); p <= PMAX; ++p) {
        if (p < d) continue;
        Real g0r, g0i;
        if constexpr (!REGULAR) {
          g0r = P_cur * ha_r;
          g0i = P_cur * ha_i;
        } else {
          g0r = P_cur * (Real)jp[p];
          g0i = (Real)0;
        }
        // G(+d) = g0 e^{i d phi}, G(-d) = g0 e^{-i d phi}
        const Real gpr = g0r * ph_r - g0i * ph_i;
        const Real gpi = g0r * ph_i + g0i * ph_r;
        const Real gmr = g0r * ph_r + g0i * ph_i;
        const Real gmi = g0i * ph_r - g0r * ph_i;
#pragma unroll kSgnUnroll
        for (int sgn = 0; sgn < 2; ++sgn) {
          if (sgn == 1 && d == 0) break;
          const Real gr = sgn == 0 ? gpr : gmr;
          const Real gi = sgn == 0 ? gpi : gmi;
          float2 grr, gii;  // (g_re, g_re), (g_im, g_im): packed FMA operands (complex64 only)
          if constexpr (!F64) {
            grr = make_float2((float)gr, (float)gr);
            gii = make_float2((float)gi, (float)gi);
          }
#pragma unroll
          for (int i = 0; i < bi.count; ++i) {
            const int m1 = bi.m1[i];
            const int m2 = sgn == 0 ? m1 + d : m1 - d;
            if (m2 < -L || m2 > L) continue;
            const int nv = valid_rows(L, m1, p);
            const int off = bi.row_off[i];
#pragma unroll
            for (int rr = 0; rr < 2 * L; ++rr) {
              if (rr < rows_of_m(L, m1) && rr < nv) {
                const VE v = vp[rr];  // shared-memory stage (plain load; __ldg is global-only)
                if constexpr (F64) {
                  yr[off + rr] = fma(gr, v.x, yr[off + rr]);
                  yr[off + rr] = fma(-gi, v.y, yr[off + rr]);
                  yi[off + rr] = fma(gr, v.y, yi[off + rr]);
                  yi[off + rr] = fma(gi, v.x, yi[off + rr]);
                } else {
                  yc[off + rr] = __ffma2_rn(grr, make_float2(v.x, v.y), yc[off + rr]);
                  yc[off + rr] = __ffma2_rn(gii, make_float2(v.z, v.w), yc[off + rr]);
                }
              }
            }
            vp += nv;
          }
        }
        // advance Legendre (order d fixed) and Hankel recurrences to p + 1
        if (p < PMAX) {
          const Real P_next = (Real)__ldg(a.leg->alpha + p * kLegStride + d) * ctR * P_cur - (Real)__ldg(a.leg->beta + p * kLegStride + d) * P_prev;
          P_prev = P_cur;
          P_cur = P_next;
          if constexpr (!REGULAR) {
            const Real f = (Real)(2 * p + 3) * inv_x;
            const Real nr = f * hb_r - ha_r;
            const Real ni = f * hb_i - ha_i;
            ha_r = hb_r; ha_i = hb_i; hb_r = nr; hb_i = ni;
          }
        }
      }
    }
    __syncthreads();  // every warp is done with this stage before it is refilled
  }
  if (timed_out) {
    // No copy may still be landing in shared memory when the block exits: a stage holds one
    // exactly when thread 0 issued more copies into it than the block consumed, and that copy
    // completes the stage's next phase; wait (bounded) for each. Should a drain itself run out,
    // the block exits with that copy's state undefined; the error word is already set and the
    // result is poisoned.
    if (threadIdx.x == 0) {
#pragma unroll
      for (int b = 0; b < 2; ++b)
        if (issued[b] > uses[b]) (void)mbar_wait(&bars[b], uses[b] & 1u);
    }
    return false;
  }

  if (active) {
    C* out = reinterpret_cast<C*>(a.partial) + ((size_t)c * a.n_particles + s1) * a.nmax;
#pragma unroll
    for (int i = 0; i < bi.count; ++i) {
      const int m1 = bi.m1[i];
#pragma unroll
      for (int rr = 0; rr < 2 * L; ++rr) {
        if (rr < rows_of_m(L, m1)) {
          const int n1 = mode_index(L, row_tau(rr), row_l(L, rr), m1);
          C val;
          if constexpr (F64) {
            val.x = yr[bi.row_off[i] + rr];
            val.y = yi[bi.row_off[i] + rr];
          } else {
            val = yc[bi.row_off[i] + rr];
          }
          out[n1] = val;
        }
      }
    }
  }
  return true;
}

#include "coupling_c64.cuh"

// Receivers per thread of the contraction: kC64Receivers for the complex64 (Hankel) kernel, else one.
template <typename Real, bool REGULAR>
__host__ __device__ constexpr int receivers_per_thread() {
  return (sizeof(Real) == 4 && !REGULAR) ? kC64Receivers : 1;
}

// Bundles of the stream layout a kernel reads: the complex64 (Hankel) kernel has its own.
template <typename Real, bool REGULAR>
__host__ __device__ constexpr bool c64_layout() {
  return sizeof(Real) == 4 && !REGULAR;
}

// Bundle b of NB (B counts down from NB to 0 through the recursion).
template <int L, typename Real, bool REGULAR, int NB, int B>
struct BundleDispatch {
  __device__ static __forceinline__ bool run(const ContractArgs& a, int b, int tile, int chunk,
                                             char* smem, unsigned long long* bars,
                                             unsigned (&uses)[2], unsigned (&issued)[2]) {
    if (b == B - 1) {
      if constexpr (sizeof(Real) == 4 && !REGULAR)
        return contract_body_c64<L, NB, B - 1>(a, tile, chunk, smem, bars, uses, issued);
      else
        return contract_body<L, NB, B - 1, Real, REGULAR>(a, tile, chunk, smem, bars, uses, issued);
    }
    return BundleDispatch<L, Real, REGULAR, NB, B - 1>::run(a, b, tile, chunk, smem, bars, uses, issued);
  }
};
template <int L, typename Real, bool REGULAR, int NB>
struct BundleDispatch<L, Real, REGULAR, NB, 0> {
  __device__ static __forceinline__ bool run(const ContractArgs&, int, int, int, char*,
                                             unsigned long long*, unsigned (&)[2], unsigned (&)[2]) {
    return true;
  }
};

__device__ __forceinline__ void stage_barriers_init(unsigned long long* bars) {
  if (threadIdx.x == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    mbar_fence_init();
  }
  __syncthreads();
}

// Dynamic shared memory: two stages of the largest bundle stream (16-byte aligned).
// blockIdx.x = receiver tile, blockIdx.y = source chunk, blockIdx.z = bundle.
template <int L, typename Real, bool REGULAR>
__global__ void __launch_bounds__(128) contract_kernel(ContractArgs a) {
  extern __shared__ __align__(128) char smem[];
  __shared__ __align__(8) unsigned long long bars[2];
  stage_barriers_init(bars);
  unsigned uses[2] = {0u, 0u}, issued[2] = {0u, 0u};
  constexpr int NB = num_bundles(L, c64_layout<Real, REGULAR>());
  (void)BundleDispatch<L, Real, REGULAR, NB, NB>::run(a, blockIdx.z, blockIdx.x, blockIdx.y, smem, bars, uses,
                                                      issued);
}

// ---------------------------------------------------------------------------------------------
// Persistent work-queue contraction over many right-hand sides of different aggregates.
// Every column (one right-hand side of one aggregate; all of one lmax) contributes
// tiles x chunks x bundles work items, numbered by item_pre. Resident blocks take items from a
// device counter until none is left, so aggregates of very different sizes share one launch and
// one set of resident blocks; a column whose live flag is 0 is skipped. The stage barriers are
// initialised once per block and their phases carried from item to item.
struct GroupColumn {
  const double* pos;      // positions of the column's aggregate (N, 3)
  const double2* tmat;    // T of the column's aggregate (master epilogue; unused by the contraction)
  const void* v;          // the column's V stream (VEntry), bundle-major
  void* partial;          // the column's partial sums (chunks, N, nmax)
  double k;
  int n_particles;
  int tiles;
  int chunks;
  int sources_per_chunk;
};

struct GroupedContractArgs {
  const GroupColumn* cols;
  const int* live;
  const long long* item_pre;     // [n_cols + 1]
  int n_cols;
  long long total_items;
  unsigned long long* counter;   // work-queue head, zero at launch
  const LegendreTables* leg;
  int nmax;
  int n_bundles;
  int bundle_begin[8];
  int bundle_len[8];
  int* err;
  int poll_limit;
  int stall;
};

template <int L, typename Real>
__global__ void __launch_bounds__(128) grouped_contract_kernel(GroupedContractArgs g) {
  extern __shared__ __align__(128) char smem[];
  __shared__ __align__(8) unsigned long long bars[2];
  __shared__ long long item_s;
  stage_barriers_init(bars);
  unsigned uses[2] = {0u, 0u}, issued[2] = {0u, 0u};
  ContractArgs a{};
  a.nmax = g.nmax;
  a.leg = g.leg;
  for (int b = 0; b < 8; ++b) {
    a.bundle_begin[b] = g.bundle_begin[b];
    a.bundle_len[b] = g.bundle_len[b];
  }
  a.err = g.err;
  a.cutoff2 = -1.0;
  a.poll_limit = g.poll_limit;
  a.stall = g.stall;
#pragma unroll 1
  for (;;) {
    if (threadIdx.x == 0) item_s = (long long)atomicAdd(g.counter, 1ull);
    __syncthreads();
    const long long item = item_s;
    __syncthreads();  // every thread has the item before thread 0 takes the next one
    if (item >= g.total_items) break;
    int lo = 0, hi = g.n_cols;  // item_pre[lo] <= item < item_pre[hi]
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (g.item_pre[mid] <= item) lo = mid; else hi = mid;
    }
    if (!g.live[lo]) continue;
    const GroupColumn col = g.cols[lo];
    long long r = item - g.item_pre[lo];
    const int bundle = (int)(r % g.n_bundles);
    r /= g.n_bundles;
    const int chunk = (int)(r % col.chunks);
    const int tile = (int)(r / col.chunks);
    a.n_particles = col.n_particles;
    a.sources_per_chunk = col.sources_per_chunk;
    a.k = col.k;
    a.pos = col.pos;
    a.v = col.v;
    a.partial = col.partial;
    constexpr int NB = num_bundles(L, c64_layout<Real, false>());
    if (!BundleDispatch<L, Real, false, NB, NB>::run(a, bundle, tile, chunk, smem, bars, uses, issued))
      break;  // a stage wait ran out: this block stops (the error word is set)
  }
}

template <int L>
cudaError_t launch_grouped_contract(int precision, const GroupedContractArgs& g, int blocks,
                                    cudaStream_t stream);

// Longest padded bundle stream (entries per source) of the layout with NB bundles.
template <int L, int NB>
constexpr int max_bundle_stream(int b = 0) {
  return b >= NB ? 0
                 : (padded_stream_length(L, b, NB) > max_bundle_stream<L, NB>(b + 1)
                        ? padded_stream_length(L, b, NB)
                        : max_bundle_stream<L, NB>(b + 1));
}

// ---------------------------------------------------------------------------------------------
// Chunk reduction + epilogue. mode 0: y = W x ; mode 1: y = x - T (.) (W x).
template <typename Real>
__global__ void __launch_bounds__(256) reduce_kernel(long long n_elems, int chunks,
                                                     const void* partial, const double2* x,
                                                     const double2* tmat, double2* y, int mode,
                                                     const int* err) {
  using C = typename Cplx<Real>::T;
  const C* pp = reinterpret_cast<const C*>(partial);
  if (*err) {  // a stage wait timed out in the contraction: the result is poisoned, not partial
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n_elems;
         i += (long long)gridDim.x * blockDim.x)
      y[i] = make_double2(nan(""), nan(""));
    return;
  }
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n_elems;
       i += (long long)gridDim.x * blockDim.x) {
    double re = 0.0, im = 0.0;
    for (int c = 0; c < chunks; ++c) {
      const C v = pp[(size_t)c * n_elems + i];
      re += (double)v.x;
      im += (double)v.y;
    }
    double2 out;
    if (mode == 1) {
      const double2 t = tmat[i];
      const double2 xv = x[i];
      out.x = xv.x - (t.x * re - t.y * im);
      out.y = xv.y - (t.x * im + t.y * re);
    } else {
      out.x = re;
      out.y = im;
    }
    y[i] = out;
  }
}

// Block partial sums of conj(b) * (sum over chunks of partial): used for the scattering
// cross-section bilinear form.
template <typename Real>
__global__ void __launch_bounds__(256) reduce_dot_kernel(long long n_elems, int chunks,
                                                         const void* partial, const double2* b,
                                                         double2* block_sums, const int* err) {
  using C = typename Cplx<Real>::T;
  const C* pp = reinterpret_cast<const C*>(partial);
  if (*err) {
    if (threadIdx.x == 0) block_sums[blockIdx.x] = make_double2(nan(""), nan(""));
    return;
  }
  double re = 0.0, im = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n_elems;
       i += (long long)gridDim.x * blockDim.x) {
    double wr = 0.0, wi = 0.0;
    for (int c = 0; c < chunks; ++c) {
      const C v = pp[(size_t)c * n_elems + i];
      wr += (double)v.x;
      wi += (double)v.y;
    }
    const double2 bv = b[i];
    // conj(b) * w
    re += bv.x * wr + bv.y * wi;
    im += bv.x * wi - bv.y * wr;
  }
  __shared__ double sr[256], si[256];
  sr[threadIdx.x] = re;
  si[threadIdx.x] = im;
  __syncthreads();
  for (int off = blockDim.x / 2; off > 0; off >>= 1) {
    if (threadIdx.x < off) {
      sr[threadIdx.x] += sr[threadIdx.x + off];
      si[threadIdx.x] += si[threadIdx.x + off];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) block_sums[blockIdx.x] = make_double2(sr[0], si[0]);
}

// Launch helpers implemented per lmax in coupling_l<L>.cu.
template <int L>
cudaError_t launch_contract(int precision, bool regular, const ContractArgs& a, int tiles,
                            int chunks, int threads, cudaStream_t stream);
// Blocks of the (non-regular) contraction kernel resident per SM at `threads` threads.
template <int L>
int contract_resident_blocks(int precision, int threads);

}  // namespace yasf
