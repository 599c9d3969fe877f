// Multi-right-hand-side coupling on the 5th-generation tensor cores (tcgen05, kind::tf32).
//
// For a panel of R right-hand sides the direct form of the translation is used: every pair block
// W_ij is generated once (complex64, from the pair table G[p][delta] = Pn_p^{|delta|} h_p
// e^{i delta phi} and the a5/b5 coefficients, yasfpy/functions/cpu_numba.py:50-93) and applied to
// the whole nmax x R panel of the source's coefficients. With the a5 (tau1 == tau2) and b5
// (tau1 != tau2) blocks Wa, Wb of W_ij = [[Wa, Wb], [Wb, Wa]], the receiver's panel obeys
//   Y1 += Wa X1 + Wb X2,   Y2 += Wb X1 + Wa X2        (X1, X2: the tau = 1, 2 halves).
// The MMA computes the transposed products Y^T[r][n1] += X^T[r][n2] W[n1][n2]: the right-hand
// sides are the M dimension (64 per block), the receiving modes the N dimension, the source modes
// K. Complex products are four real products; the imaginary-part subtraction uses the MMA's
// A-negate bit. Accumulators stay in tensor memory for the whole source loop.
//
// Roles (160 threads): warps 0-3 generate the pair table and W_ij into shared memory (canonical
// K-major no-swizzle layout, values rounded to TF32) and finally read the accumulators; warp 4
// owns tensor memory and its elected thread issues the MMAs. Source panels X_j arrive by
// cp.async.bulk; two stages of (X_j, W_ij) are in flight. Every wait is bounded: a timeout sets
// the error word, every role stops, the result is written as NaN and tensor memory is freed.
#pragma once

#include <cuda_runtime.h>

#include "coupling.cuh"

namespace yasf {

__host__ __device__ constexpr int half_modes(int L) { return L * (L + 2); }
__host__ __device__ constexpr int pad8(int v) { return (v + 7) & ~7; }

// Panel geometry for lmax L (all sizes in bytes unless noted).
template <int L>
struct PanelGeom {
  static constexpr int H = half_modes(L);       // modes per tau half
  static constexpr int HP = pad8(H);            // padded to the MMA granularity
  static constexpr int M = 64;                  // right-hand sides per block
  static constexpr int P = 2 * L + 1;           // orders p
  static constexpr int DW = 4 * L + 1;          // deltas
  static constexpr int X_LBO = (M / 8) * 128;   // K-chunk stride of an X plane
  static constexpr int X_PLANE = (HP / 4) * X_LBO;
  static constexpr int X_STAGE = 4 * X_PLANE;   // X1r, X1i, X2r, X2i
  static constexpr int W_LBO = (HP / 8) * 128;  // K-chunk stride of a W plane
  static constexpr int W_PLANE = (HP / 4) * W_LBO;
  static constexpr int W_STAGE = 4 * W_PLANE;   // War, Wai, Wbr, Wbi
  static constexpr int G_STAGE = P * DW * 8;    // pair table (float2)
  static constexpr int TMEM_COLS = 4 * HP <= 32 ? 32 : (4 * HP <= 64 ? 64 : (4 * HP <= 128 ? 128 : 256));
  static constexpr int SMEM = 2 * X_STAGE + 2 * W_STAGE + 2 * G_STAGE + 256;
  static constexpr int W_PLANE_F = W_PLANE / 4;
};

// Byte offset of element (row, k) in a canonical K-major no-swizzle operand with `rows` rows.
__host__ __device__ __forceinline__ int kmajor_offset(int row, int k, int rows) {
  return (k >> 2) * ((rows >> 3) * 128) + (row >> 3) * 128 + (row & 7) * 16 + (k & 3) * 4;
}

// Round to TF32 (round to nearest, ties away) keeping the float container.
__device__ __forceinline__ float to_tf32(float v) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
  return __uint_as_float(r);
}

struct PanelArgs {
  int n_particles;
  int nmax;
  int nrhs;
  long long ld;                  // column stride of x (elements)
  long long ldy;                 // column stride of y (elements)
  double k;
  const double* pos;
  const LegendreTables* leg;
  const float* xp;               // source panels, [group][source][X_STAGE bytes]
  const float* gen_c1;           // [TM][256] generation coefficients, thread-minor
  const unsigned* gen_meta;      // [TM][256] generation meta words
  const double2* x;              // input columns (for the master epilogue)
  const double2* tmat;           // T (N*nmax), master epilogue when non-null
  double2* y;                    // output columns
  int* err;
};

// ---- tcgen05 helpers -------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long umma_desc(unsigned saddr, int lbo, int sbo) {
  unsigned long long d = 0;
  d |= (unsigned long long)((saddr >> 4) & 0x3FFF);
  d |= (unsigned long long)((lbo >> 4) & 0x3FFF) << 16;
  d |= (unsigned long long)((sbo >> 4) & 0x3FFF) << 32;
  d |= 1ull << 46;  // descriptor version for sm_100
  // base offset 0, legacy LBO mode, layout type 0 = no swizzle
  return d;
}

// kind::tf32, D = F32, A/B TF32 K-major, M x N.
__host__ __device__ constexpr unsigned umma_idesc_tf32(int M, int N, bool neg_a) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((neg_a ? 1u : 0u) << 13) | ((unsigned)(N >> 3) << 17) |
         ((unsigned)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_tf32(unsigned tmem_d, unsigned long long da,
                                          unsigned long long db, unsigned idesc, unsigned accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accum)
      : "memory");
}

__device__ __forceinline__ void umma_commit(unsigned long long* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void named_sync(int id, int threads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}

template <int N>
__device__ __forceinline__ void tmem_ld32(unsigned addr, float* v);
template <>
__device__ __forceinline__ void tmem_ld32<8>(unsigned addr, float* v) {
  unsigned r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                 "=r"(r[6]), "=r"(r[7])
               : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

// Bounded wait that also gives up when another role has already aborted.
__device__ __forceinline__ bool wait_or_abort(unsigned long long* bar, unsigned parity,
                                              volatile int* abort_flag) {
  if (*abort_flag) return false;
  if (mbar_wait(bar, parity)) return true;
  *abort_flag = 1;
  return false;
}

// ---- the kernel ---------------------------------------------------------------------------
// Threads: warps 0-7 generate W (256 threads, each with a fixed, register-resident list of
// generation terms: coefficient, pair-table offset, rotation, first/last flags, destination);
// warps 0-3 also read the accumulators at the end. Warp 8 owns tensor memory and issues the
// MMAs. Warp 9 issues the source-panel copies and computes the pair table one pair ahead.
constexpr int kGenThreads = 256;
constexpr int kPanelThreads = 320;
__host__ __device__ constexpr int gen_terms_max(int L) {
  return L <= 1 ? 2 : (L == 2 ? 4 : (L == 3 ? 8 : (L == 4 ? 12 : (L == 5 ? 28 : 56))));
}
// meta word: [0,10) pair-table offset, 10 rotate (multiply by i), 11 first term of an entry,
// 12 last term of an entry, [13,32) destination float index in the W stage (real part; the
// imaginary part is one plane further).
constexpr unsigned kMetaOdd = 1u << 10, kMetaFirst = 1u << 11, kMetaLast = 1u << 12;

template <int L>
__global__ void __launch_bounds__(kPanelThreads, 1) panel_kernel(PanelArgs a) {
  using G = PanelGeom<L>;
  constexpr int H = G::H, HP = G::HP, M = G::M, P = G::P, DW = G::DW;
  constexpr int TM = gen_terms_max(L);
  constexpr int PW = G::W_PLANE / 4;  // floats per W plane
  extern __shared__ __align__(1024) unsigned char panel_smem[];
  unsigned char* xs = panel_smem;                               // [2][X_STAGE]
  unsigned char* ws = xs + 2 * G::X_STAGE;                      // [2][W_STAGE]
  float2* gt = reinterpret_cast<float2*>(ws + 2 * G::W_STAGE);  // [2][P*DW]
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(
      reinterpret_cast<unsigned char*>(gt) + 2 * G::G_STAGE);
  unsigned long long* xfull = bars;       // [2] source panel landed
  unsigned long long* wfull = bars + 2;   // [2] W generated
  unsigned long long* empty = bars + 4;   // [2] MMAs of the stage done (X and W reusable)
  unsigned long long* gfull = bars + 6;   // [2] pair table ready
  unsigned long long* gempty = bars + 8;  // [2] pair table consumed
  unsigned long long* accum = bars + 10;  // accumulators final
  unsigned* tmem_slot = reinterpret_cast<unsigned*>(bars + 12);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(bars + 13);
  volatile int* gen_stop = reinterpret_cast<volatile int*>(bars + 14);
  volatile int* last_issued = reinterpret_cast<volatile int*>(bars + 15);

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int i = blockIdx.x;    // receiving sphere
  const int grp = blockIdx.y;  // right-hand-side group of 64
  const int N = a.n_particles;
  const int n_iter = N - 1;    // every source but the receiver itself

  // generation terms of this thread (registers)
  float gc[TM];
  unsigned gm[TM];
  if (tid < kGenThreads) {
#pragma unroll
    for (int t = 0; t < TM; ++t) {
      gc[t] = __ldg(a.gen_c1 + t * kGenThreads + tid);
      gm[t] = __ldg(a.gen_meta + t * kGenThreads + tid);
    }
  }
  for (int o = tid; o < (2 * G::W_STAGE) / 16; o += blockDim.x)
    reinterpret_cast<float4*>(ws)[o] = make_float4(0.f, 0.f, 0.f, 0.f);
  if (tid == 0) {
    for (int b = 0; b < 11; ++b) mbar_init(&bars[b], 1);
    *abort_flag = 0;
    *gen_stop = 0;
    *last_issued = -1;
    mbar_fence_init();
  }
  if (warp == 8) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(tmem_slot)),
                 "r"(G::TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = *tmem_slot;

  if (warp < 8) {
    // ===================== W generation =====================
    for (int t = 0; t < n_iter; ++t) {
      const int s = t & 1;
      const unsigned k = (unsigned)(t >> 1);
      if (tid == 0) {
        bool ok = t < 2 || wait_or_abort(&empty[s], (k - 1) & 1, abort_flag);
        ok = ok && wait_or_abort(&gfull[s], k & 1, abort_flag);
        if (!ok) *gen_stop = 1;
      }
      named_sync(1, kGenThreads);
      if (*gen_stop) break;
      const float2* g = gt + s * (P * DW);
      float* wst = reinterpret_cast<float*>(ws + s * G::W_STAGE);
      float ar = 0.f, ai = 0.f;
#pragma unroll
      for (int q = 0; q < TM; ++q) {
        const unsigned mt = gm[q];
        const float2 gv = g[mt & 1023u];
        const bool odd = (mt & kMetaOdd) != 0;
        const float av = odd ? gv.y : gv.x;
        const float bv = odd ? -gv.x : gv.y;
        if (mt & kMetaFirst) { ar = 0.f; ai = 0.f; }
        ar = fmaf(gc[q], av, ar);
        ai = fmaf(gc[q], bv, ai);
        if (mt & kMetaLast) {
          const unsigned dst = mt >> 13;
          wst[dst] = to_tf32(ar);
          wst[dst + PW] = to_tf32(ai);
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      named_sync(1, kGenThreads);
      if (tid == 0) {
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&wfull[s])) : "memory");
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&gempty[s])) : "memory");
      }
    }
  } else if (warp == 8) {
    // ===================== MMA issuer =====================
    if (lane == 0) {
      constexpr int KS = HP / 8;
      constexpr unsigned idesc = umma_idesc_tf32(M, HP, false);
      constexpr unsigned idesc_neg = umma_idesc_tf32(M, HP, true);
      unsigned long long dx0[4], dw0[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        dx0[q] = umma_desc(smem_addr(xs) + q * G::X_PLANE, G::X_LBO, 128);
        dw0[q] = umma_desc(smem_addr(ws) + q * G::W_PLANE, G::W_LBO, 128);
      }
      constexpr unsigned long long xs_step = (unsigned long long)(G::X_STAGE >> 4);
      constexpr unsigned long long ws_step = (unsigned long long)(G::W_STAGE >> 4);
      constexpr unsigned long long xk = (unsigned long long)((2 * G::X_LBO) >> 4);
      constexpr unsigned long long wk = (unsigned long long)((2 * G::W_LBO) >> 4);
      for (int t = 0; t < n_iter; ++t) {
        const int s = t & 1;
        const unsigned ph = (unsigned)((t >> 1) & 1);
        if (!wait_or_abort(&xfull[s], ph, abort_flag)) break;
        if (!wait_or_abort(&wfull[s], ph, abort_flag)) break;
        tc_fence_after();
        // (x plane, w plane, accumulator region, negate A): Y1 = Wa X1 + Wb X2, Y2 = Wb X1 + Wa X2
        constexpr int XP[16] = {0, 1, 2, 3, 0, 1, 2, 3, 0, 1, 2, 3, 0, 1, 2, 3};
        constexpr int WP[16] = {0, 1, 2, 3, 1, 0, 3, 2, 2, 3, 0, 1, 3, 2, 1, 0};
        constexpr int NG[16] = {0, 1, 0, 1, 0, 0, 0, 0, 0, 1, 0, 1, 0, 0, 0, 0};
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          const unsigned dcol = tmem + (unsigned)((q >> 2) * HP);
          const unsigned long long da0 = dx0[XP[q]] + (unsigned long long)s * xs_step;
          const unsigned long long db0 = dw0[WP[q]] + (unsigned long long)s * ws_step;
#pragma unroll
          for (int kk = 0; kk < KS; ++kk) {
            const unsigned acc = (t == 0 && (q & 3) == 0 && kk == 0) ? 0u : 1u;
            umma_tf32(dcol, da0 + kk * xk, db0 + kk * wk, NG[q] ? idesc_neg : idesc, acc);
          }
        }
        umma_commit(&empty[s]);
      }
      umma_commit(accum);
    }
    __syncwarp();
  } else {
    // ===================== source panels + pair table =====================
    const double xi = a.pos[3 * i], yi = a.pos[3 * i + 1], zi = a.pos[3 * i + 2];
    for (int t = 0; t < n_iter; ++t) {
      const int s = t & 1;
      const unsigned k = (unsigned)(t >> 1);
      const int j = t < i ? t : t + 1;
      int ok = 1;
      if (lane == 0) {
        ok = t < 2 || wait_or_abort(&empty[s], (k - 1) & 1, abort_flag);
        if (ok) {
          const unsigned char* src =
              reinterpret_cast<const unsigned char*>(a.xp) + ((size_t)grp * N + j) * G::X_STAGE;
          bulk_load(xs + s * G::X_STAGE, src, G::X_STAGE, &xfull[s]);
          *last_issued = t;
          ok = t < 2 || wait_or_abort(&gempty[s], (k - 1) & 1, abort_flag);
        }
      }
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) break;
      float2* g = gt + s * (P * DW);
      if (lane < P) {
        const int d = lane;
        const double dx = xi - a.pos[3 * j], dy = yi - a.pos[3 * j + 1], dz = zi - a.pos[3 * j + 2];
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        double ctd = dz / r;
        ctd = fmin(1.0, fmax(-1.0, ctd));
        const float ct = (float)ctd;
        const float st = (float)sqrt(1.0 - ctd * ctd);
        const double rho = sqrt(dx * dx + dy * dy);
        const double phi = (rho > 0.0) ? atan2(dy, dx) : 0.0;
        float sdp, cdp;
        sincosf((float)(d * phi), &sdp, &cdp);
        const double xd = a.k * r;
        double sxd, cxd;
        sincos(xd, &sxd, &cxd);
        const float x = (float)xd, sx = (float)sxd, cx = (float)cxd;
        const float ix = 1.0f / x;
        float hr0 = sx * ix, hi0 = -cx * ix;
        float hr1 = (sx - x * cx) * ix * ix, hi1 = -(cx + x * sx) * ix * ix;
        for (int q = 0; q < d; ++q) {
          const float f = (float)(2 * q + 3) * ix;
          const float nr = f * hr1 - hr0, ni = f * hi1 - hi0;
          hr0 = hr1; hi0 = hi1; hr1 = nr; hi1 = ni;
        }
        float stp = 1.f;
        for (int q = 0; q < d; ++q) stp *= st;
        float Pp = 0.f, Pc = (float)a.leg->start[d] * stp;
        for (int p = d; p < P; ++p) {
          const float gr = Pc * hr0, gi = Pc * hi0;
          g[p * DW + (2 * L + d)] = make_float2(gr * cdp - gi * sdp, gr * sdp + gi * cdp);
          g[p * DW + (2 * L - d)] = make_float2(gr * cdp + gi * sdp, gi * cdp - gr * sdp);
          if (p + 1 < P) {
            const float Pn = (float)a.leg->alpha[p * kLegStride + d] * ct * Pc -
                             (float)a.leg->beta[p * kLegStride + d] * Pp;
            Pp = Pc;
            Pc = Pn;
            const float f = (float)(2 * p + 3) * ix;
            const float nr = f * hr1 - hr0, ni = f * hi1 - hi0;
            hr0 = hr1; hi0 = hi1; hr1 = nr; hi1 = ni;
          }
        }
      }
      __syncwarp();
      if (lane == 0)
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&gfull[s])) : "memory");
    }
  }

  // ===================== epilogue =====================
  if (warp < 4) {
    // wait (bounded) for the MMAs and source copies in flight before reading or freeing TMEM
    const bool ok = n_iter == 0 || mbar_wait(accum, 0);
    if (tid == 0 && *last_issued >= 0) {
      const int tl = *last_issued;
      (void)mbar_wait(&xfull[tl & 1], (unsigned)((tl >> 1) & 1));
      if (tl >= 1) (void)mbar_wait(&xfull[(tl - 1) & 1], (unsigned)(((tl - 1) >> 1) & 1));
    }
    tc_fence_after();
    const bool aborted = *abort_flag != 0;
    if (aborted && tid == 0) atomicExch(a.err, 1);
    const int row = (lane & 15) + 16 * warp;  // M = 64: row l + 16q sits in lane l + 32q
    const int col = grp * M + row;
    const bool live = lane < 16 && col < a.nrhs;
    const unsigned lane_base = tmem + ((unsigned)(32 * warp) << 16);
    for (int n = 0; n < H; n += 8) {
      float v[4][8];
#pragma unroll
      for (int reg = 0; reg < 4; ++reg) tmem_ld32<8>(lane_base + reg * HP + n, v[reg]);
      if (!live) continue;
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int q = n + u;
        if (q >= H) break;
#pragma unroll
        for (int half = 0; half < 2; ++half) {
          const int nn = half * H + q;
          double yr = 0.0, yi = 0.0;
          if (n_iter > 0) {
            yr = (double)v[2 * half][u];
            yi = (double)v[2 * half + 1][u];
          }
          if (aborted || !ok) { yr = nan(""); yi = nan(""); }
          const size_t gi = (size_t)col * a.ldy + (size_t)i * a.nmax + nn;
          double2 out;
          if (a.tmat) {
            const double2 tv = a.tmat[(size_t)i * a.nmax + nn];
            const double2 xv = a.x[(size_t)col * a.ld + (size_t)i * a.nmax + nn];
            out = make_double2(xv.x - (tv.x * yr - tv.y * yi), xv.y - (tv.x * yi + tv.y * yr));
          } else {
            out = make_double2(yr, yi);
          }
          a.y[gi] = out;
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 8) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(G::TMEM_COLS)
                 : "memory");
  }
}

// Source panels: columns [grp*64, grp*64+64) of x rounded to TF32 in the X-operand layout.
template <int L>
__global__ void xpanel_kernel(int n_particles, int nmax, int nrhs, long long ld, const double2* x,
                              float* xp) {
  using G = PanelGeom<L>;
  constexpr int H = G::H, HP = G::HP, M = G::M;
  const int j = blockIdx.x, grp = blockIdx.y;
  unsigned char* dst = reinterpret_cast<unsigned char*>(xp) + ((size_t)grp * n_particles + j) * G::X_STAGE;
  for (int e = threadIdx.x; e < M * HP * 2; e += blockDim.x) {
    const int half = e / (M * HP);
    const int rem = e - half * M * HP;
    const int r = rem / HP, q = rem - (rem / HP) * HP;
    const int col = grp * M + r;
    float re = 0.f, im = 0.f;
    if (q < H && col < nrhs) {
      const double2 v = x[(size_t)col * ld + (size_t)j * nmax + half * H + q];
      re = to_tf32((float)v.x);
      im = to_tf32((float)v.y);
    }
    const int off = kmajor_offset(r, q, M);
    *reinterpret_cast<float*>(dst + (2 * half) * G::X_PLANE + off) = re;
    *reinterpret_cast<float*>(dst + (2 * half + 1) * G::X_PLANE + off) = im;
  }
}

}  // namespace yasf
