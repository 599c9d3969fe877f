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
  const int* w_ptr;              // [2*H*H + 1] term lists of the a (first H*H) and b entries
  const unsigned char* w_p;      // order p of each term
  const float2* w_coef;          // complex coefficient of each term
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
template <int L>
__global__ void __launch_bounds__(160, 1) panel_kernel(PanelArgs a) {
  using G = PanelGeom<L>;
  constexpr int H = G::H, HP = G::HP, M = G::M, P = G::P, DW = G::DW;
  extern __shared__ __align__(1024) unsigned char panel_smem[];
  unsigned char* xs = panel_smem;                             // [2][X_STAGE]
  unsigned char* ws = xs + 2 * G::X_STAGE;                    // [2][W_STAGE]
  float2* gt = reinterpret_cast<float2*>(ws + 2 * G::W_STAGE);  // [2][P*DW]
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(
      reinterpret_cast<unsigned char*>(gt) + 2 * G::G_STAGE);
  unsigned long long* full_x = bars;      // [2]
  unsigned long long* full_w = bars + 2;  // [2]
  unsigned long long* empty = bars + 4;   // [2]
  unsigned long long* accum = bars + 6;   // [1]
  unsigned* tmem_slot = reinterpret_cast<unsigned*>(bars + 8);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(bars + 9);
  volatile int* gen_stop = reinterpret_cast<volatile int*>(bars + 10);  // written by thread 0 only
  volatile int* last_issued = reinterpret_cast<volatile int*>(bars + 11);
  __shared__ signed char m_of[96];

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int i = blockIdx.x;      // receiving sphere
  const int grp = blockIdx.y;    // right-hand-side group of 64
  const int N = a.n_particles;

  // zero both W stages once (padding rows/columns stay zero), mode table, barriers
  for (int o = tid; o < (2 * G::W_STAGE) / 16; o += blockDim.x)
    reinterpret_cast<float4*>(ws)[o] = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int q = tid; q < H; q += blockDim.x) {
    const int l = (int)floorf(sqrtf((float)q + 1.0f) + 1e-4f);
    m_of[q] = (signed char)(q + 1 - l * l - l);
  }
  if (tid == 0) {
    for (int b = 0; b < 7; ++b) mbar_init(&bars[b], 1);
    *abort_flag = 0;
    *gen_stop = 0;
    *last_issued = -1;
    mbar_fence_init();
  }
  if (warp == 4) {  // tensor memory for the four accumulators (Y1r, Y1i, Y2r, Y2i)
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
  const int n_iter = N - 1;  // every source but the receiver itself

  if (warp < 4) {
    // ===================== generators =====================
    const double xi = a.pos[3 * i], yi = a.pos[3 * i + 1], zi = a.pos[3 * i + 2];
    for (int t = 0; t < n_iter; ++t) {
      const int s = t & 1;
      const int j = t < i ? t : t + 1;
      // Only thread 0 waits for the stage to drain; the decision reaches the other generators
      // through gen_stop after the named barrier, so all 128 leave the loop together.
      if (tid == 0) {
        if (t >= 2 && !wait_or_abort(&empty[s], (unsigned)(((t >> 1) - 1) & 1), abort_flag)) {
          *gen_stop = 1;
        } else {
          const unsigned char* src =
              reinterpret_cast<const unsigned char*>(a.xp) + ((size_t)grp * N + j) * G::X_STAGE;
          bulk_load(xs + s * G::X_STAGE, src, G::X_STAGE, &full_x[s]);
          *last_issued = t;
        }
      }
      named_sync(1, 128);
      if (*gen_stop) break;
      // pair table: lane d of warp 0 handles |delta| = d
      float2* g = gt + s * (P * DW);
      if (warp == 0 && lane < P) {
        const int d = lane;
        const double dx = xi - a.pos[3 * j], dy = yi - a.pos[3 * j + 1], dz = zi - a.pos[3 * j + 2];
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        double ct = dz / r;
        ct = fmin(1.0, fmax(-1.0, ct));
        const double st = sqrt(1.0 - ct * ct);
        const double rho = sqrt(dx * dx + dy * dy);
        const double phi = (rho > 0.0) ? atan2(dy, dx) : 0.0;
        double sdp, cdp;
        sincos(d * phi, &sdp, &cdp);
        const double x = a.k * r;
        double sx, cx;
        sincos(x, &sx, &cx);
        const double ix = 1.0 / x;
        double hr0 = sx * ix, hi0 = -cx * ix;
        double hr1 = (sx - x * cx) * ix * ix, hi1 = -(cx + x * sx) * ix * ix;
        // advance the Hankel recurrence to order d
        for (int q = 0; q < d; ++q) {
          const double f = (2 * q + 3) * ix;
          const double nr = f * hr1 - hr0, ni = f * hi1 - hi0;
          hr0 = hr1; hi0 = hi1; hr1 = nr; hi1 = ni;
        }
        double stp = 1.0;
        for (int q = 0; q < d; ++q) stp *= st;
        double Pp = 0.0, Pc = a.leg->start[d] * stp;
        for (int p = d; p < P; ++p) {
          const double gr = Pc * hr0, gi = Pc * hi0;
          g[p * DW + (2 * L + d)] = make_float2((float)(gr * cdp - gi * sdp), (float)(gr * sdp + gi * cdp));
          g[p * DW + (2 * L - d)] = make_float2((float)(gr * cdp + gi * sdp), (float)(gi * cdp - gr * sdp));
          if (p + 1 < P) {
            const double Pn = a.leg->alpha[p * kLegStride + d] * ct * Pc - a.leg->beta[p * kLegStride + d] * Pp;
            Pp = Pc;
            Pc = Pn;
            const double f = (2 * p + 3) * ix;
            const double nr = f * hr1 - hr0, ni = f * hi1 - hi0;
            hr0 = hr1; hi0 = hi1; hr1 = nr; hi1 = ni;
          }
        }
      }
      named_sync(1, 128);
      // W entries: a block (e < H*H) and b block, row n1' (receiver), column n2' (source)
      unsigned char* wst = ws + s * G::W_STAGE;
      for (int e = tid; e < 2 * H * H; e += 128) {
        const int which = e >= H * H;
        const int ee = e - which * H * H;
        const int n1 = ee / H, n2 = ee - (ee / H) * H;
        const int col = m_of[n2] - m_of[n1] + 2 * L;
        float wr = 0.f, wi = 0.f;
        const int t0 = __ldg(a.w_ptr + e), t1 = __ldg(a.w_ptr + e + 1);
        for (int q = t0; q < t1; ++q) {
          const float2 c = __ldg(a.w_coef + q);
          const float2 gv = g[__ldg(a.w_p + q) * DW + col];
          wr = fmaf(c.x, gv.x, wr);
          wr = fmaf(-c.y, gv.y, wr);
          wi = fmaf(c.x, gv.y, wi);
          wi = fmaf(c.y, gv.x, wi);
        }
        const int off = kmajor_offset(n1, n2, HP);
        *reinterpret_cast<float*>(wst + (2 * which) * G::W_PLANE + off) = to_tf32(wr);
        *reinterpret_cast<float*>(wst + (2 * which + 1) * G::W_PLANE + off) = to_tf32(wi);
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      named_sync(1, 128);
      if (tid == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&full_w[s])) : "memory");
    }
  } else {
    // ===================== MMA issuer (one thread of warp 4) =====================
    if (lane == 0) {
      constexpr int KS = HP / 8;  // K steps of 8 (tf32)
      const unsigned idesc = umma_idesc_tf32(M, HP, false);
      const unsigned idesc_neg = umma_idesc_tf32(M, HP, true);
      const unsigned xbase = smem_addr(xs), wbase = smem_addr(ws);
      for (int t = 0; t < n_iter; ++t) {
        const int s = t & 1;
        const unsigned ph = (unsigned)((t >> 1) & 1);
        if (!wait_or_abort(&full_x[s], ph, abort_flag)) break;
        if (!wait_or_abort(&full_w[s], ph, abort_flag)) break;
        tc_fence_after();
        const unsigned xb = xbase + s * G::X_STAGE, wb = wbase + s * G::W_STAGE;
        // planes: X: 0 X1r, 1 X1i, 2 X2r, 3 X2i ; W: 0 War, 1 Wai, 2 Wbr, 3 Wbi
        // out regions (TMEM columns): 0 Y1r, 1 Y1i, 2 Y2r, 3 Y2i
        // Y1 = Wa X1 + Wb X2 ; Y2 = Wb X1 + Wa X2 ; (Xr + i Xi)(Wr + i Wi)
        struct Term { int xpl, wpl, out, neg; };
        const Term terms[16] = {
            {0, 0, 0, 0}, {1, 1, 0, 1}, {2, 2, 0, 0}, {3, 3, 0, 1},   // Y1r
            {0, 1, 1, 0}, {1, 0, 1, 0}, {2, 3, 1, 0}, {3, 2, 1, 0},   // Y1i
            {0, 2, 2, 0}, {1, 3, 2, 1}, {2, 0, 2, 0}, {3, 1, 2, 1},   // Y2r
            {0, 3, 3, 0}, {1, 2, 3, 0}, {2, 1, 3, 0}, {3, 0, 3, 0}};  // Y2i
#pragma unroll 1
        for (int q = 0; q < 16; ++q) {
          const Term tm = terms[q];
          const unsigned dcol = tmem + (unsigned)(tm.out * HP);
          const unsigned id = tm.neg ? idesc_neg : idesc;
#pragma unroll 1
          for (int kk = 0; kk < KS; ++kk) {
            const unsigned long long da =
                umma_desc(xb + tm.xpl * G::X_PLANE + kk * 2 * G::X_LBO, G::X_LBO, 128);
            const unsigned long long db =
                umma_desc(wb + tm.wpl * G::W_PLANE + kk * 2 * G::W_LBO, G::W_LBO, 128);
            // the first product into each region on the first source overwrites it
            const unsigned acc = (t == 0 && (q & 3) == 0 && kk == 0) ? 0u : 1u;
            umma_tf32(dcol, da, db, id, acc);
          }
        }
        umma_commit(&empty[s]);
      }
      umma_commit(accum);
    }
    __syncwarp();
  }

  // ===================== epilogue =====================
  if (warp < 4) {
    // Always wait (bounded) for the MMAs in flight, aborted or not, before reading or freeing TMEM.
    bool ok = n_iter == 0 || mbar_wait(accum, 0);
    if (tid == 0 && *last_issued >= 0) {  // and for the last source copies issued
      const int tl = *last_issued;
      (void)mbar_wait(&full_x[tl & 1], (unsigned)((tl >> 1) & 1));
      if (tl >= 1) (void)mbar_wait(&full_x[(tl - 1) & 1], (unsigned)(((tl - 1) >> 1) & 1));
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
  if (warp == 4) {
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
