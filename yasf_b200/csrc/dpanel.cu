// Float64 coupling for many right-hand sides at once (the float64 residual of batched solves).
//
// The single-column kernel (coupling.cuh) contracts source-side streams against the pair table
// for every column: about 67k float64 FMAs per pair and column at lmax 6. With many columns it
// pays to form W_ij once per pair, in float64, and apply it densely:
//   Y1 = Wa X1 + Wb X2, Y2 = Wb X1 + Wa X2   =>   U = P S, V = Q D,  Y1 = (U + V)/2, Y2 = (U - V)/2
// with P = Wa + Wb, Q = Wa - Wb, S = X1 + X2, D = X1 - X2 (the tau symmetry of W_ij,
// yasfpy/functions/cpu_numba.py:50-93): 4 H^2 complex FMAs, i.e. 18.4k float64 FMAs per pair and
// column at lmax 6, plus the generation of P and Q (about 27k FMAs per pair, shared by the block's
// 32 columns). Entries of P and Q are generated in pairs: an entry (l1 m1, l2 m2) and its mirror
// (l1 -m1, l2 -m2) have equal Wa and negated Wb coefficients on A[p][|m2 - m1|] and conjugate
// phases e^{+-i (m2 - m1) phi}, so both come from one set of loads.
//
// Block = (receiving sphere i, tile of 32 or 64 columns). Worker warps generate P and Q of W_ij
// into shared memory, then apply them: half the warps form U = P S and half V = Q D, each warp
// RPW receiving rows times the tile's columns (one column per lane and 32 columns, W entries
// broadcast: 4 row groups of H/4 rows at 32 columns, 8 row groups of H/8 rows at 64). A
// helper warp runs ahead: it computes the float64 pair table (A[p][d] = Pn_p^d(cos theta)
// h_p(k r), e^{i delta phi}; two stages) and copies the source tile [S; D] (cp.async.bulk; two
// stages at 32 columns, one at 64). All waits
// are bounded in time; on a timeout every role stops, the error word is set and the result is NaN.
#include <algorithm>
#include <cmath>

#include "capi_internal.h"
#include "panel.cuh"

namespace yasf {

// Column tile of a block: 32 columns with 8 worker warps and two source-tile stages, or 64 columns
// with 16 worker warps and one stage (each W_ij then serves 64 columns; the copy of the next tile
// overlaps the generation of the next W).
template <int L, int CT>
struct DpGeom {
  static constexpr int H = L * (L + 2);
  static constexpr int P = 2 * L + 1;
  static constexpr int CPT = CT / 32;                // columns per thread
  static constexpr int RG = 4 * CPT;                 // row groups per block (U or V)
  static constexpr int RPW = (H + RG - 1) / RG;      // receiving rows per worker warp
  static constexpr int HR = RG * RPW;                // padded row count
  static constexpr int WORKERS = 2 * RG;             // worker warps: (block, row group)
  static constexpr int THREADS = 32 * (WORKERS + 1); // + helper warp
  static constexpr int XS = CT == 32 ? 2 : 1;        // source-tile stages
  static constexpr int W_BYTES = 2 * H * HR * 16;    // P, Q as [blk][q2][q1] complex float64
  static constexpr int X_STAGE = 2 * H * CT * 16;    // [S; D] as [blk][q2][c]
  static constexpr int T_ENTRIES = P * P + 4 * L + 1;
  static constexpr int T_STAGE = T_ENTRIES * 16;
  static constexpr int W_OFF = 0;
  static constexpr int X_OFF = W_BYTES;
  static constexpr int T_OFF = X_OFF + XS * X_STAGE;
  static constexpr int BAR_OFF = T_OFF + 2 * T_STAGE;
  static constexpr int SMEM = BAR_OFF + 128;
  static_assert(SMEM <= 232448, "dpanel shared memory exceeds the per-block limit");
  static_assert(W_BYTES % 16 == 0 && X_STAGE % 16 == 0 && T_STAGE % 16 == 0, "alignment");
  static_assert(H * CT * 16 <= XS * X_STAGE, "exchange buffer does not fit");
};

struct DpArgs {
  int n_particles;
  int nmax;
  int nrhs;
  long long ld;     // column stride of x
  long long ldy;    // column stride of y
  double k;
  const double* pos;
  const LegendreTables* leg;
  const double2* xp;         // source tiles [tile][source][X_STAGE bytes]
  int n_chunks;              // chunks of 32 items
  const int4* chunks;        // Wa slots, Wb slots, first term slot, 0
  const int2* items;         // [32 * n_chunks]: entry | mirror packed (-1: none),
                             // delta + 2L | Wa table base << 8 | Wb table base << 18
  const double* term_coef;   // [slot][lane] Wa: real coefficient; Wb: coefficient / i; 0 padding
  const double2* x;          // input columns (master epilogue)
  const double2* tmat;       // T, master epilogue when non-null
  double2* y;
  int* err;
  unsigned long long wait_ns;  // bound of one wait (1 s normally)
  int stall;                   // test hook: 1 = the helper warp never delivers a pair table, so the
                               // workers' waits run out (0 normally)
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {  // conj(a) * b
  return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

// Pair table of one pair in float64, lane d < P: A[p][d] at p*P + d (p >= d), phases at
// P*P + 2L +- d. Same recurrences as the single-column kernel.
template <int L>
__device__ __forceinline__ void dp_pair_table(double2* T, const LegendreTables* leg, int d, double dx,
                                              double dy, double dz, double k) {
  constexpr int P = 2 * L + 1;
  const double r = sqrt(dx * dx + dy * dy + dz * dz);
  const double ct = fmin(1.0, fmax(-1.0, dz / r));
  const double rho = sqrt(dx * dx + dy * dy);
  const double st = rho / r;
  const double c1 = rho > 0.0 ? dx / rho : 1.0, s1 = rho > 0.0 ? dy / rho : 0.0;
  double cdp = 1.0, sdp = 0.0;
  for (int q = 0; q < d; ++q) {
    const double cn = cdp * c1 - sdp * s1;
    sdp = cdp * s1 + sdp * c1;
    cdp = cn;
  }
  T[P * P + 2 * L + d] = make_double2(cdp, sdp);
  if (d) T[P * P + 2 * L - d] = make_double2(cdp, -sdp);
  const double x = k * r;
  double sx, cx;
  sincos(x, &sx, &cx);
  const double ix = 1.0 / x;
  double hr0 = sx * ix, hi0 = -cx * ix;
  double hr1 = (sx - x * cx) * ix * ix, hi1 = -(cx + x * sx) * ix * ix;
  double Pp = 0.0, Pc = 0.0, stp = 1.0;
#pragma unroll
  for (int p = 0; p < P; ++p) {
    if (p == d) Pc = leg->start[d] * stp;
    if (p < d) stp *= st;
    if (p >= d) {
      T[p * P + d] = make_double2(Pc * hr0, Pc * hi0);
      if (p + 1 < P) {
        const double Pn = leg->alpha[p * kLegStride + d] * ct * Pc - leg->beta[p * kLegStride + d] * Pp;
        Pp = Pc;
        Pc = Pn;
      }
    }
    if (p + 1 < P) {
      const double f = (double)(2 * p + 3) * ix;
      const double nr = f * hr1 - hr0, ni = f * hi1 - hi0;
      hr0 = hr1; hi0 = hi1; hr1 = nr; hi1 = ni;
    }
  }
}

template <int L, int CT>
__global__ void __launch_bounds__(DpGeom<L, CT>::THREADS, 1) dpanel_kernel(DpArgs a) {
  using G = DpGeom<L, CT>;
  constexpr int H = G::H, P = G::P, RPW = G::RPW, HR = G::HR, NW = G::WORKERS, XS = G::XS;
  constexpr int CPT = G::CPT, NA = RPW * CPT;  // accumulators (row r, column lane + 32 k) at r CPT + k
  constexpr int NWT = 32 * NW;  // worker threads
  extern __shared__ __align__(128) unsigned char dp_smem[];
  double2* W = reinterpret_cast<double2*>(dp_smem + G::W_OFF);    // [2][H][HR]
  unsigned char* xs = dp_smem + G::X_OFF;                         // [XS][X_STAGE]
  unsigned char* ts = dp_smem + G::T_OFF;                         // [2][T_STAGE]
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(dp_smem + G::BAR_OFF);
  unsigned long long* xfull = bars;      // [XS] source tile landed
  unsigned long long* xfree = bars + 2;  // [XS] source tile consumed (apply done)
  unsigned long long* tfull = bars + 4;  // [2] pair table ready
  unsigned long long* tfree = bars + 6;  // [2] pair table consumed (generation done)
  volatile int* abort_flag = reinterpret_cast<volatile int*>(bars + 8);
  volatile int* issued = reinterpret_cast<volatile int*>(bars + 9);  // [2] newest pair per stage
  volatile int* go = reinterpret_cast<volatile int*>(bars + 10);     // [2] workers' uniform decisions

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int i = blockIdx.x, tile = blockIdx.y;
  const int N = a.n_particles;
  const int n_iter = N - 1;

  for (int o = tid; o < G::W_BYTES / 16; o += blockDim.x) W[o] = make_double2(0.0, 0.0);
  // pair-table entries p < d are never written: zero, as the term windows may read them
  for (int o = tid; o < 2 * G::T_ENTRIES; o += blockDim.x)
    reinterpret_cast<double2*>(ts)[o] = make_double2(0.0, 0.0);
  if (tid == 0) {
    for (int b = 0; b < 2; ++b) {
      mbar_init(&xfull[b], 1);
      mbar_init(&xfree[b], 1);
      mbar_init(&tfull[b], 1);
      mbar_init(&tfree[b], 1);
    }
    *abort_flag = 0;
    issued[0] = issued[1] = -1;
    mbar_fence_init();
  }
  __syncthreads();

  if (warp < NW) {
    // ===================== generation + dense application =====================
    const int blk = warp / G::RG;              // 0: U = P S, 1: V = Q D
    const int r0 = (warp % G::RG) * RPW;
    // 32-column tiles: complex accumulators as two independent partial sums each (re: w.x x.x |
    // -w.y x.y, im: w.x x.y | w.y x.x), so consecutive FMAs of a row do not wait on each other
    double2 acc[NA], acc2[CT == 32 ? NA : 1];
#pragma unroll
    for (int r = 0; r < NA; ++r) acc[r] = make_double2(0.0, 0.0);
#pragma unroll
    for (int r = 0; r < (CT == 32 ? NA : 1); ++r) acc2[r] = make_double2(0.0, 0.0);
    // One thread waits (bounded) and publishes the outcome across a workers' barrier, so every
    // worker warp takes the same branch and no warp is left waiting at a barrier.
    for (int t = 0; t < n_iter; ++t) {
      const int st = t & 1, sx = t % XS;
      if (tid == 0)
        go[0] = wait_or_abort(&tfull[st], (unsigned)((t >> 1) & 1), abort_flag, a.wait_ns) ? 1 : 0;
      named_sync(1, NWT);
      if (!go[0]) break;
      const double2* T = reinterpret_cast<const double2*>(ts + st * G::T_STAGE);
      for (int cc = warp; cc < a.n_chunks; cc += NW) {
        const int4 cm = __ldg(a.chunks + cc);
        const int2 m = __ldg(a.items + 32 * cc + lane);
        const double* tc = a.term_coef + (size_t)cm.z * 32 + lane;
        // slot q of the Wa (Wb) terms is A[p0 + 2q][|delta|]: table entry base + 2 P q
        const double2* Ta = T + ((m.y >> 8) & 1023);
        const double2* Tb = T + ((m.y >> 18) & 1023);
        double2 sa = make_double2(0.0, 0.0), sb = make_double2(0.0, 0.0);
        // at most lmax + 1 Wa and lmax Wb terms per entry: fully unrolled, predicated, so that all
        // coefficient loads of the chunk are in flight together
#pragma unroll
        for (int q = 0; q < L + 1; ++q) {
          if (q < cm.x) {
            const double cf = __ldg(tc + q * 32);
            const double2 g = Ta[2 * P * q];
            sa.x = fma(cf, g.x, sa.x);
            sa.y = fma(cf, g.y, sa.y);
          }
        }
#pragma unroll
        for (int q = 0; q < L; ++q) {
          if (q < cm.y) {
            const double cf = __ldg(tc + (cm.x + q) * 32);
            const double2 g = Tb[2 * P * q];
            sb.x = fma(cf, g.x, sb.x);
            sb.y = fma(cf, g.y, sb.y);
          }
        }
        if (m.x == -1) continue;
        const int q1 = m.x & 255, q2 = (m.x >> 8) & 255, mq1 = (m.x >> 16) & 255, mq2 = (m.x >> 24) & 255;
        const double2 e = T[P * P + (m.y & 255)];
        // entry: Wa = E Sa, Wb = i E Sb ; mirror: Wa' = conj(E) Sa, Wb' = -i conj(E) Sb
        const double2 ua = cmul(e, sa), vb = cmul(e, sb);
        W[q2 * HR + q1] = make_double2(ua.x - vb.y, ua.y + vb.x);            // P = Wa + Wb
        W[(H + q2) * HR + q1] = make_double2(ua.x + vb.y, ua.y - vb.x);      // Q = Wa - Wb
        const double2 ma = cmulc(e, sa), mb = cmulc(e, sb);
        W[mq2 * HR + mq1] = make_double2(ma.x + mb.y, ma.y - mb.x);
        W[(H + mq2) * HR + mq1] = make_double2(ma.x - mb.y, ma.y + mb.x);
      }
      if (tid == 0)
        go[1] = wait_or_abort(&xfull[sx], (unsigned)((t / XS) & 1), abort_flag, a.wait_ns) ? 1 : 0;
      named_sync(1, NWT);  // W complete, source tile decision published
      if (tid == 0) mbar_arrive(&tfree[st]);
      if (!go[1]) break;
      const double2* X = reinterpret_cast<const double2*>(xs + sx * G::X_STAGE) + blk * H * CT + lane;
      const double2* Wb = W + blk * H * HR + r0;
      if constexpr (CT == 32) {
#pragma unroll 2
        for (int q2 = 0; q2 < H; ++q2) {
          const double2 xv = X[q2 * CT];
#pragma unroll
          for (int r = 0; r < RPW; ++r) {
            const double2 w = Wb[q2 * HR + r];
            acc[r].x = fma(w.x, xv.x, acc[r].x);
            acc2[r].x = fma(-w.y, xv.y, acc2[r].x);
            acc[r].y = fma(w.x, xv.y, acc[r].y);
            acc2[r].y = fma(w.y, xv.x, acc2[r].y);
          }
        }
      } else {
        // 64 columns, 96 registers per thread: each W entry serves two columns (8 shared loads
        // per 48 FMAs); one accumulator per row and column, the two FMAs of each component issued
        // in separate passes (2 RPW instructions apart)
#pragma unroll 1
        for (int q2 = 0; q2 < H; ++q2) {
          double2 xv[CPT];
#pragma unroll
          for (int k = 0; k < CPT; ++k) xv[k] = X[q2 * CT + 32 * k];
#pragma unroll
          for (int r = 0; r < RPW; ++r) {
            const double wx = Wb[q2 * HR + r].x;
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
              acc[r * CPT + k].x = fma(wx, xv[k].x, acc[r * CPT + k].x);
              acc[r * CPT + k].y = fma(wx, xv[k].y, acc[r * CPT + k].y);
            }
          }
#pragma unroll
          for (int r = 0; r < RPW; ++r) {
            const double wy = Wb[q2 * HR + r].y;
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
              acc[r * CPT + k].x = fma(-wy, xv[k].y, acc[r * CPT + k].x);
              acc[r * CPT + k].y = fma(wy, xv[k].x, acc[r * CPT + k].y);
            }
          }
        }
      }
      named_sync(1, NWT);  // W and the source tile are consumed
      if (tid == 0) mbar_arrive(&xfree[sx]);
    }
    if constexpr (CT == 32) {
#pragma unroll
      for (int r = 0; r < NA; ++r) acc[r] = make_double2(acc[r].x + acc2[r].x, acc[r].y + acc2[r].y);
    }
    // park V in shared memory after every role has finished (below), then combine
    __syncthreads();
    if (tid == 0)
      for (int b = 0; b < XS; ++b)
        if (issued[b] >= 0) (void)panel_wait(&xfull[b], (unsigned)((issued[b] / XS) & 1));
    named_sync(1, NWT);
    double2* xch = reinterpret_cast<double2*>(xs);  // [H][CT] V
    if (blk == 1) {
#pragma unroll
      for (int r = 0; r < RPW; ++r)
#pragma unroll
        for (int k = 0; k < CPT; ++k)
          if (r0 + r < H) xch[(r0 + r) * CT + 32 * k + lane] = acc[r * CPT + k];
    }
    named_sync(1, NWT);
    const bool aborted = *abort_flag != 0;
    if (aborted && tid == 0) atomicExch(a.err, 1);
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
      const int c = 32 * k + lane, col = tile * CT + c;
      if (blk == 0 && col < a.nrhs) {
#pragma unroll
        for (int r = 0; r < RPW; ++r) {
          const int q = r0 + r;
          if (q >= H) break;
          const double2 v = xch[q * CT + c];
          const double2 u = acc[r * CPT + k];
          double y1r = 0.5 * (u.x + v.x), y1i = 0.5 * (u.y + v.y);
          double y2r = 0.5 * (u.x - v.x), y2i = 0.5 * (u.y - v.y);
          if (aborted) y1r = y1i = y2r = y2i = __longlong_as_double(0x7ff8000000000000LL);
#pragma unroll
          for (int half = 0; half < 2; ++half) {
            const int nn = half * H + q;
            const double yr = half ? y2r : y1r, yi = half ? y2i : y1i;
            double2 out;
            if (a.tmat) {
              const double2 tv = a.tmat[(size_t)i * a.nmax + nn];
              const double2 xv = a.x[(size_t)col * a.ld + (size_t)i * a.nmax + nn];
              out = make_double2(xv.x - (tv.x * yr - tv.y * yi), xv.y - (tv.x * yi + tv.y * yr));
            } else {
              out = make_double2(yr, yi);
            }
            a.y[(size_t)col * a.ldy + (size_t)i * a.nmax + nn] = out;
          }
        }
      }
    }
  } else {
    // ===================== helper: pair tables (two stages) and source tiles (XS stages) =====
    // Pair t's table is written once generation of pair t - 2 has released its stage; pair t's
    // tile is copied once the apply of pair t - XS has released its stage. With one tile stage the
    // table of pair t + 1 is computed while the workers generate and apply pair t.
    const double xi = a.pos[3 * i], yi = a.pos[3 * i + 1], zi = a.pos[3 * i + 2];
    for (int t = 0; t < n_iter && !a.stall; ++t) {
      const int st = t & 1, sx = t % XS;
      const int j = t < i ? t : t + 1;
      int ok = 1;
      if (lane == 0)
        ok = t < 2 ? !*abort_flag
                   : wait_or_abort(&tfree[st], (unsigned)(((t >> 1) - 1) & 1), abort_flag, a.wait_ns);
      __syncwarp();
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) break;
      if (lane < P)
        dp_pair_table<L>(reinterpret_cast<double2*>(ts + st * G::T_STAGE), a.leg, lane, xi - a.pos[3 * j],
                         yi - a.pos[3 * j + 1], zi - a.pos[3 * j + 2], a.k);
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(&tfull[st]);
        ok = t < XS ? !*abort_flag
                    : wait_or_abort(&xfree[sx], (unsigned)(((t / XS) - 1) & 1), abort_flag,
                                    a.wait_ns);
        if (ok) {
          issued[sx] = t;
          bulk_load(xs + sx * G::X_STAGE,
                    reinterpret_cast<const unsigned char*>(a.xp) + ((size_t)tile * N + j) * G::X_STAGE,
                    G::X_STAGE, &xfull[sx]);
        }
      }
      __syncwarp();
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) break;
    }
    __syncthreads();  // pairs with the workers' barrier before the drain
  }
}

// Source tiles: for columns [tile*CT, tile*CT + CT), [S; D] = [X1 + X2; X1 - X2] as [blk][q2][c]
// (zero beyond nrhs); blockIdx.z selects S or D. Read column-contiguous, written row-contiguous
// through shared memory, 32 columns at a time.
template <int L, int CT>
__global__ void __launch_bounds__(256) dpanel_tiles_kernel(int n_particles, int nmax, int nrhs, long long ld,
                                                           const double2* x, double2* xp) {
  using G = DpGeom<L, CT>;
  constexpr int H = G::H;
  __shared__ double2 buf[H][33];
  const int j = blockIdx.x, tile = blockIdx.y, blk = blockIdx.z;
  const double sg = blk ? -1.0 : 1.0;
  double2* dst = xp + ((size_t)tile * n_particles + j) * (G::X_STAGE / 16) + (size_t)blk * H * CT;
  for (int c0 = 0; c0 < CT; c0 += 32) {
    for (int e = threadIdx.x; e < 32 * H; e += blockDim.x) {
      const int c = e / H, q = e - (e / H) * H;
      const int col = tile * CT + c0 + c;
      double2 v = make_double2(0.0, 0.0);
      if (col < nrhs) {
        const double2 v1 = x[(size_t)col * ld + (size_t)j * nmax + q];
        const double2 v2 = x[(size_t)col * ld + (size_t)j * nmax + H + q];
        v = make_double2(v1.x + sg * v2.x, v1.y + sg * v2.y);
      }
      buf[q][c] = v;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < H * 32; e += blockDim.x) {
      const int row = e / 32, c = e - (e / 32) * 32;
      dst[row * CT + c0 + c] = buf[row][c];
    }
    __syncthreads();
  }
}

// Items (an entry and its mirror) of the float64 dense panel and their terms, from the plan's
// a5/b5 table. Items run over q2 then q1, so the 32 items of a chunk (one warp) store to
// consecutive entries of a row (no bank conflicts); the chunk's coefficients are laid out
// slot-major ([slot][lane], coalesced loads). The Wa (Wb) terms of an item sit at orders
// p = p0, p0 + 2, ... of one table column |delta|, so slot q holds the coefficient of
// p = p0 + 2q (zero where the item has no term) and the kernel reads table entry
// p0 P + |delta| + 2 P q: no index loads. The chunk's slot counts are its items' largest spans;
// each item's p0 is its first term, moved down by 2 until the window ends at row 2L + 1 at most
// (row 2L + 1 is the phase row; rows p < |delta| hold zeros).
int dpanel_build_items(int L, const double* ab5, std::vector<int4>& chunks, std::vector<int2>& items,
                       std::vector<double>& term_coef) {
  chunks.clear();
  items.clear();
  term_coef.clear();
  if (L < 1 || L > 6) return YASF_OK;
  const int nmax = 2 * L * (L + 2), P = 2 * L + 1, H = L * (L + 2);
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
  struct Item { int packed, delta, ad; std::vector<int> pa, pb; std::vector<double> ca, cb; };
  std::vector<Item> list;
  std::vector<char> seen((size_t)H * H, 0);
  for (int q2 = 0; q2 < H; ++q2)
    for (int q1 = 0; q1 < H; ++q1) {
      if (seen[(size_t)q1 * H + q2]) continue;
      const int mq1 = mirror(q1), mq2 = mirror(q2);
      seen[(size_t)q1 * H + q2] = seen[(size_t)mq1 * H + mq2] = 1;
      int l1, m1, l2, m2;
      lm(q1, l1, m1);
      lm(q2, l2, m2);
      const int delta = m2 - m1, ad = std::abs(delta);
      Item it;
      it.packed = q1 | (q2 << 8) | (mq1 << 16) | (mq2 << 24);
      it.delta = delta + 2 * L;
      it.ad = ad;
      for (int which = 0; which < 2; ++which)
        for (int p = 0; p < P; ++p) {
          const size_t idx = ((size_t)(which * H + q2) * nmax + q1) * P + p;
          const double cr = ab5[2 * idx], ci = ab5[2 * idx + 1];
          const size_t midx = ((size_t)(which * H + mq2) * nmax + mq1) * P + p;
          const double mr = ab5[2 * midx], mi = ab5[2 * midx + 1];
          const double sgn = which == 0 ? 1.0 : -1.0;
          const double tol = 1e-13 * std::max(1.0, std::fabs(cr) + std::fabs(ci));
          if (std::fabs(mr - sgn * cr) > tol || std::fabs(mi - sgn * ci) > tol) return YASF_ERR_INVALID_ARGUMENT;
          if (cr == 0.0 && ci == 0.0) continue;
          if ((which == 0 && ci != 0.0) || (which == 1 && cr != 0.0) || p < ad) return YASF_ERR_INVALID_ARGUMENT;
          (which == 0 ? it.pa : it.pb).push_back(p);
          (which == 0 ? it.ca : it.cb).push_back(which == 0 ? cr : ci);
        }
      list.push_back(std::move(it));
    }
  auto span = [](const std::vector<int>& ps) { return ps.empty() ? 0 : (ps.back() - ps.front()) / 2 + 1; };
  const int n_chunks = ((int)list.size() + 31) / 32;
  int slot = 0;
  for (int c = 0; c < n_chunks; ++c) {
    int na = 0, nb = 0;
    for (int l = 0; l < 32; ++l) {
      const size_t k = (size_t)c * 32 + l;
      if (k < list.size()) {
        na = std::max(na, span(list[k].pa));
        nb = std::max(nb, span(list[k].pb));
      }
    }
    if (na > L + 1 || nb > L) return YASF_ERR_INVALID_ARGUMENT;
    chunks.push_back(make_int4(na, nb, slot, 0));
    term_coef.resize((size_t)(slot + na + nb) * 32, 0.0);
    for (int l = 0; l < 32; ++l) {
      const size_t k = (size_t)c * 32 + l;
      if (k >= list.size()) {
        items.push_back(make_int2(-1, 2 * L));
        continue;
      }
      const Item& it = list[k];
      int base[2];
      for (int which = 0; which < 2; ++which) {
        const std::vector<int>& ps = which == 0 ? it.pa : it.pb;
        const std::vector<double>& cs = which == 0 ? it.ca : it.cb;
        const int n = which == 0 ? na : nb, s0 = which == 0 ? slot : slot + na;
        int p0 = ps.empty() ? 0 : ps.front();
        while (p0 > 1 && p0 + 2 * (n - 1) > 2 * L + 1) p0 -= 2;
        if (p0 + 2 * (n - 1) > 2 * L + 1) return YASF_ERR_INVALID_ARGUMENT;
        for (size_t q = 0; q < ps.size(); ++q) {
          const int j = (ps[q] - p0) / 2;
          if ((ps[q] - p0) % 2 != 0 || j < 0 || j >= n) return YASF_ERR_INVALID_ARGUMENT;
          term_coef[(size_t)(s0 + j) * 32 + l] = cs[q];
        }
        base[which] = p0 * P + it.ad;
      }
      items.push_back(make_int2(it.packed, it.delta | (base[0] << 8) | (base[1] << 18)));
    }
    slot += na + nb;
  }
  return YASF_OK;
}

// Column tile width for nrhs columns: 64 once there are 64 or more.
static int dpanel_cols(int nrhs) {
  if (tile_config().dpanel_cols) return tile_config().dpanel_cols;
  return nrhs >= 64 ? 64 : 32;
}

template <int L, int CT>
static int launch_dpanel_ct(const DpArgs& da, cudaStream_t s) {
  using G = DpGeom<L, CT>;
  const int tiles = (da.nrhs + CT - 1) / CT;
  YASF_COUNTED(dpanel_tiles_kernel<L, CT><<<dim3(da.n_particles, tiles, 2), 256, 0, s>>>(
      da.n_particles, da.nmax, da.nrhs, da.ld, da.x, const_cast<double2*>(da.xp)));
  YASF_CUDA_TRY(cudaGetLastError());
  YASF_CUDA_TRY(cudaFuncSetAttribute(dpanel_kernel<L, CT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     G::SMEM));
  YASF_COUNTED(dpanel_kernel<L, CT><<<dim3(da.n_particles, tiles), G::THREADS, G::SMEM, s>>>(da));
  YASF_CUDA_TRY(cudaGetLastError());
  return YASF_OK;
}

template <int L>
static int launch_dpanel(const DpArgs& da, cudaStream_t s) {
  return dpanel_cols(da.nrhs) == 64 ? launch_dpanel_ct<L, 64>(da, s) : launch_dpanel_ct<L, 32>(da, s);
}

// Bytes of one source's [S; D] for 32 columns.
static size_t dpanel_tile_bytes(int L) {
  switch (L) {
    case 1: return DpGeom<1, 32>::X_STAGE;
    case 2: return DpGeom<2, 32>::X_STAGE;
    case 3: return DpGeom<3, 32>::X_STAGE;
    case 4: return DpGeom<4, 32>::X_STAGE;
    case 5: return DpGeom<5, 32>::X_STAGE;
    case 6: return DpGeom<6, 32>::X_STAGE;
    default: return 0;
  }
}

}  // namespace yasf

using namespace yasf;

extern "C" int yasf_dpanel_workspace_size(const yasf_plan* plan, int n_particles, int nrhs, size_t* bytes) {
  if (!plan || !bytes || n_particles <= 0 || nrhs <= 0) return YASF_ERR_INVALID_ARGUMENT;
  const size_t tb = dpanel_tile_bytes(plan->lmax);
  if (!tb) return YASF_ERR_UNSUPPORTED;
  const int ct = dpanel_cols(nrhs);
  const size_t tiles = (size_t)(nrhs + ct - 1) / ct;
  *bytes = ((tiles * (ct / 32) * n_particles * tb + 255) & ~size_t(255)) + 256;
  return YASF_OK;
}

extern "C" int yasf_dpanel_matvec(const yasf_plan* plan, int n_particles, const double* positions,
                                  double k_medium, const double* tmat, const double* x, double* y,
                                  int nrhs, long long ldx, long long ldy, void* workspace,
                                  size_t workspace_bytes, void* stream) {
  int st = validate_coupling(plan, n_particles, positions, k_medium, YASF_C128);
  if (st != YASF_OK) return st;
  if (!x || !y || x == y || nrhs <= 0) return YASF_ERR_INVALID_ARGUMENT;
  const long long n = (long long)n_particles * plan->nmax;
  if (nrhs == 1) ldx = ldy = n;
  if (ldx < n || ldy < n) return YASF_ERR_INVALID_ARGUMENT;
  if (!aligned16(x) || !aligned16(y) || (tmat && !aligned16(tmat)) || !aligned16(workspace))
    return YASF_ERR_ALIGNMENT;
  if (!plan->d_dgen_items || !plan->d_dgen_chunks) return YASF_ERR_UNSUPPORTED;
  size_t need = 0;
  if ((st = yasf_dpanel_workspace_size(plan, n_particles, nrhs, &need)) != YASF_OK) return st;
  if (!workspace || workspace_bytes < need) return YASF_ERR_WORKSPACE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  char* ws = static_cast<char*>(workspace);
  int* err = reinterpret_cast<int*>(ws + need - 256);
  YASF_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), s));
  DpArgs da{};
  da.n_particles = n_particles;
  da.nmax = plan->nmax;
  da.nrhs = nrhs;
  da.n_chunks = plan->dgen_chunks;
  da.chunks = plan->d_dgen_chunks;
  da.ld = ldx;
  da.ldy = ldy;
  da.k = k_medium;
  da.pos = positions;
  da.leg = plan->d_leg;
  da.xp = reinterpret_cast<const double2*>(ws);
  da.items = plan->d_dgen_items;
  da.term_coef = plan->d_dgen_coef;
  da.x = reinterpret_cast<const double2*>(x);
  da.tmat = reinterpret_cast<const double2*>(tmat);
  da.y = reinterpret_cast<double2*>(y);
  da.err = err;
  da.wait_ns = stall_hook().panel_wait_ns;
  da.stall = stall_hook().role == YASF_STALL_DPANEL ? 1 : 0;
  switch (plan->lmax) {
    case 1: return launch_dpanel<1>(da, s);
    case 2: return launch_dpanel<2>(da, s);
    case 3: return launch_dpanel<3>(da, s);
    case 4: return launch_dpanel<4>(da, s);
    case 5: return launch_dpanel<5>(da, s);
    case 6: return launch_dpanel<6>(da, s);
    default: return YASF_ERR_UNSUPPORTED;
  }
}
