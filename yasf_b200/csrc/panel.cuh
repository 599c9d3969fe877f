// Multi-right-hand-side coupling on the 5th-generation tensor cores (tcgen05, kind::tf32).
//
// For a panel of R right-hand sides the direct form of the translation is used: every pair block
// W_ij is generated once (FP32, from A[p][d] = Pn_p^d(cos theta) h_p(k r), the phases
// e^{i delta phi} and the a5/b5 coefficients, yasfpy/functions/cpu_numba.py:50-93) and applied to
// the whole nmax x 64 panel of the source's coefficients. With the a5 (tau1 == tau2) and b5
// (tau1 != tau2) blocks Wa, Wb of W_ij = [[Wa, Wb], [Wb, Wa]],
//   Y1 = Wa X1 + Wb X2,  Y2 = Wb X1 + Wa X2   (X1, X2: the tau = 1, 2 halves)
// is computed from two products instead of four:
//   U = P S, V = Q D  with  P = Wa + Wb, Q = Wa - Wb, S = X1 + X2, D = X1 - X2,
//   Y1 = (U + V) / 2, Y2 = (U - V) / 2.
// The MMAs compute transposed products D^T[m][n] += A[m][k] B[n][k] with M = 128 rows
// A = [S_r; S_i] (64 right-hand sides, real parts then imaginary parts), N = 2 HP rows
// B = [P_r; P_i] and K = HP source modes, so one MMA yields all four real products of the complex
// product; the epilogue combines them (U_r = S_r P_r - S_i P_i, U_i = S_r P_i + S_i P_r).
// Accumulators stay in tensor memory for the whole source loop.
//
// Roles (640 threads): warps 0-15 generate P and Q of W_ij into shared memory (canonical K-major
// no-swizzle layout, values rounded to TF32) following the build-time schedule of panel_sched.h:
// every thread keeps its coefficients and pair-table offsets in registers (lmax 7-8: FP16
// coefficient pairs, offsets implicit), computes an entry and its mirror (l, -m) from one set of
// loads, and a warp's 32 stores of a step hit 32 different banks (up to lmax 6 its pair-table
// loads are bank-conflict-free as well); warps 0-3 also read the accumulators at the end. Warp 16
// owns tensor memory and its elected thread issues the MMAs. Warps 17 and 18 compute the pair
// tables of alternate pairs; warp 19 issues the cp.async.bulk copies of the source panels. Two
// source-panel stages, three W stages and four pair-table stages are in flight (lmax 7: two and
// one; lmax 8: one and one). Every wait is bounded in time: a timeout sets the error word, every
// role stops, the result is written as NaN and tensor memory is freed.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "coupling.cuh"
#include "panel_sched.h"

namespace yasf {

__host__ __device__ constexpr int half_modes(int L) { return L * (L + 2); }
__host__ __device__ constexpr int pad8(int v) { return (v + 7) & ~7; }
__host__ __device__ constexpr int tmem_cols(int c) {
  return c <= 32 ? 32 : (c <= 64 ? 64 : (c <= 128 ? 128 : (c <= 256 ? 256 : 512)));
}

// Panel geometry for lmax L (sizes in bytes unless noted).
template <int L>
struct PanelGeom {
  static constexpr int H = half_modes(L);        // modes per tau half
  static constexpr int HP = pad8(H);             // padded to the MMA granularity
  static constexpr int M = 64;                   // right-hand sides per group (1 or 2 per block)
  static constexpr int P = 2 * L + 1;            // orders p
  static constexpr int KS = HP / 8;              // K steps of 8 TF32 columns
  // A operands [S_r; S_i], [D_r; D_i]: 128 rows x HP columns
  static constexpr int A_ROWS = 128;
  static constexpr int A_LBO = (A_ROWS / 8) * 128;   // bytes between 4-column K chunks
  static constexpr int A_BYTES = A_ROWS * HP * 4;
  static constexpr int X_STAGE = 2 * A_BYTES;        // one source panel (S and D operands)
  // source-panel stages: two up to lmax 7, one at lmax 8 (what shared memory allows)
  static constexpr int X_STAGES = L <= 7 ? 2 : 1;
  // B operands [P_r; P_i], [Q_r; Q_i]: 2 HP rows x HP columns
  static constexpr int B_ROWS = 2 * HP;
  static constexpr int B_LBO = (B_ROWS / 8) * 128;
  static constexpr int B_BYTES = B_ROWS * HP * 4;
  static constexpr int W_STAGE = 2 * B_BYTES;
  // W stages: up to lmax 6 generation runs two pairs ahead of the MMAs (the per-pair hand-off
  // latency, not a throughput, bounds the kernel: three stages measured 11 % faster than two with
  // three source-panel stages); lmax 7-8: one, generation waits for the MMAs
  static constexpr int W_STAGES = L <= 6 ? 3 : 1;
  // lmax 7-8 (40 / 62 generation slots per thread): coefficients are held as FP16 pairs and the
  // pair-table addresses of a step's terms are implicit (see gen_step_packed), so the generation
  // state fits the register budget; up to lmax 6 every slot holds an FP32 coefficient and a byte
  // offset
  static constexpr bool PACKED = L >= 7;
  static_assert(!PACKED || W_STAGE / 4 <= 65536, "packed store offsets (4-byte units) exceed 16 bits");
  static constexpr int IM_OFF = (HP / 8) * 128;      // row HP + q of a B operand vs row q
  // pair table: A[p][d] at p*P + d, e^{i delta phi} at P*P + 2L + delta (float2)
  static constexpr int G_STAGE = (P * P + 4 * L + 1) * 8;
  static constexpr int G_STAGES = 4;
  static constexpr int LEG_BYTES = ((2 * P * P + P) * 4 + 15) & ~15;
  static constexpr int X_OFF = 0;
  static constexpr int W_OFF = X_OFF + X_STAGES * X_STAGE;
  static constexpr int G_OFF = W_OFF + W_STAGES * W_STAGE;
  static constexpr int LEG_OFF = G_OFF + G_STAGES * G_STAGE;
  static constexpr int BAR_OFF = (LEG_OFF + LEG_BYTES + 15) & ~15;
  static constexpr int SMEM = BAR_OFF + 256;
  static_assert(SMEM <= 232448, "panel shared memory exceeds the per-block limit");
  static_assert(X_STAGE % 1024 == 0 && W_STAGE % 1024 == 0, "operand stages must stay aligned");
  // epilogue exchange of the imaginary-row accumulators (reuses the source-panel stages)
  static constexpr int XCH_STRIDE = 4 * HP + 1;  // floats per row (odd: conflict-free)
  // (the source-panel and W stages are contiguous and both idle when the exchange runs)
  static_assert(64 * XCH_STRIDE * 4 <= X_STAGES * X_STAGE + W_STAGES * W_STAGE,
                "exchange buffer does not fit");
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

constexpr int kGenWarps = 16;
constexpr int kGenThreads = 32 * kGenWarps;
constexpr int kMmaWarp = 16;
constexpr int kGeomWarp0 = 17;  // warps 17, 18: pair tables of alternate pairs
constexpr int kLoadWarp = 19;   // source-panel copies
constexpr int kPanelThreads = 640;

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
  const float* gen_coef;         // [slot][gen thread] generation coefficients (Wa real, Wb / i)
  const unsigned* gen_goff;      // [slot][gen thread] pair-table byte offsets
  const unsigned* gen_dst;       // [3][step][gen thread] W-stage byte offsets of the item's entry
                                 // and mirror P_r rows, pair-table byte offset of its phase
  const double2* x;              // input columns (for the master epilogue)
  const double2* tmat;           // T (N*nmax), master epilogue when non-null
  double2* y;                    // output columns
  int* err;
  unsigned long long wait_ns;    // bound of one wait (1 s normally)
  int stall;                     // test hook: 1 = the pair-table warps never deliver a table, so
                                 // the generation warps' waits run out (0 normally)
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

__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
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

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Wait for phase `parity` of `bar`, bounded in time (`bound_ns`, one second unless a launch asks
// for less) rather than in polls. Each try_wait may suspend the thread for up to 2 us (it resumes
// when the phase completes), so waiting warps take few issue slots.
__device__ __forceinline__ bool panel_wait(unsigned long long* bar, unsigned parity,
                                           unsigned long long bound_ns = 1000000000ull) {
  const unsigned a = smem_addr(bar);
  unsigned long long t0 = 0;
#pragma unroll 1
  for (unsigned spin = 0;; ++spin) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity), "r"(2000u)
        : "memory");
    if (done) return true;
    if (spin == 0) {
      t0 = global_ns();
    } else if ((spin & 7) == 0 && global_ns() - t0 > bound_ns) {
      return false;
    }
  }
}

// Bounded wait that also gives up when another role has already aborted.
__device__ __forceinline__ bool wait_or_abort(unsigned long long* bar, unsigned parity,
                                              volatile int* abort_flag,
                                              unsigned long long bound_ns = 1000000000ull) {
  if (*abort_flag) return false;
  if (panel_wait(bar, parity, bound_ns)) return true;
  *abort_flag = 1;
  return false;
}

// Pair-table load. Not volatile: the address operand carries the ordering (it is derived from a
// value produced after the stage's mbarrier wait), so the compiler may batch these loads ahead of
// the previous step's stores.
__device__ __forceinline__ float2 lds_f2(unsigned addr) {
  float2 v;
  asm("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(addr));
  return v;
}
__device__ __forceinline__ void sts_f32(unsigned addr, float v) {
  asm volatile("st.shared.f32 [%0], %1;" ::"r"(addr), "f"(v) : "memory");
}
// Opaque copy: values derived from it cannot be computed before this point in program order.
__device__ __forceinline__ unsigned after_wait(unsigned v) {
  unsigned r;
  asm volatile("mov.b32 %0, %1;" : "=r"(r) : "r"(v));
  return r;
}

// P = Wa + Wb and Q = Wa - Wb of an item to their four operand rows each, from the term sums
// Sa = (ar, ai), Sb = (br, bi) and E = e^{i d phi}:
//   entry:  Wa = E Sa,       Wb = i E Sb
//   mirror: Wa' = conj(E) Sa, Wb' = -i conj(E) Sb
template <int IM_OFF, int B_BYTES>
__device__ __forceinline__ void store_item(float2 e, float ar, float ai, float br, float bi, unsigned dst,
                                           unsigned dstm) {
  {
    const float ur = e.x * ar - e.y * ai, ui = e.x * ai + e.y * ar;
    const float vr = e.x * br - e.y * bi, vi = e.x * bi + e.y * br;
    sts_f32(dst, to_tf32(ur - vi));
    sts_f32(dst + IM_OFF, to_tf32(ui + vr));
    sts_f32(dst + B_BYTES, to_tf32(ur + vi));
    sts_f32(dst + B_BYTES + IM_OFF, to_tf32(ui - vr));
  }
  {
    const float ur = e.x * ar + e.y * ai, ui = e.x * ai - e.y * ar;
    const float vr = e.x * br + e.y * bi, vi = e.x * bi - e.y * br;
    sts_f32(dstm, to_tf32(ur + vi));
    sts_f32(dstm + IM_OFF, to_tf32(ui - vr));
    sts_f32(dstm + B_BYTES, to_tf32(ur - vi));
    sts_f32(dstm + B_BYTES + IM_OFF, to_tf32(ui + vr));
  }
}

// One schedule step of W generation for this thread (lmax <= 6): the item's TA Wa terms and TB Wb
// terms, each an FP32 coefficient gc[q] on the pair-table entry at byte offset go[q].
template <int BASE, int TA, int TB, int S, int IM_OFF, int B_BYTES>
__device__ __forceinline__ void gen_step(const float (&gc)[S], const unsigned (&go)[S], unsigned gbase,
                                         unsigned eoff, unsigned dst, unsigned dstm) {
  float ar = 0.f, ai = 0.f, br = 0.f, bi = 0.f;
#pragma unroll
  for (int q = 0; q < TA; ++q) {
    const float2 g = lds_f2(gbase + go[BASE + q]);
    ar = fmaf(gc[BASE + q], g.x, ar);
    ai = fmaf(gc[BASE + q], g.y, ai);
  }
#pragma unroll
  for (int q = 0; q < TB; ++q) {
    const float2 g = lds_f2(gbase + go[BASE + TA + q]);
    br = fmaf(gc[BASE + TA + q], g.x, br);
    bi = fmaf(gc[BASE + TA + q], g.y, bi);
  }
  store_item<IM_OFF, B_BYTES>(lds_f2(gbase + eoff), ar, ai, br, bi, dst, dstm);
}

// FP16 coefficient of slot q from the packed pairs (slot 2w in the low half of word w).
template <int NW>
__device__ __forceinline__ float packed_coef(const unsigned (&gh)[NW], int q) {
  const unsigned w = gh[q >> 1];
  return __half2float(__ushort_as_half((unsigned short)((q & 1) ? (w >> 16) : (w & 0xFFFFu))));
}

// One schedule step of W generation for this thread (lmax 7-8). The Wa terms of an item run over
// p = p0, p0 + 2, ... at one |d|, so slot q of the step reads A[p0a + 2q][|d|]: table entry
// ia + 2 P q, with the step's bases ia, ib (Wb) and the phase entry ie packed in `bases` (10 bits
// each, entry units). The plan places each lane's window [p0, p0 + 2 (T - 1)] inside rows
// 0 .. 2L + 1 of the table (row 2L + 1 is the phase row) with zero coefficients on the slots
// outside the item's own terms; rows p < d are never written and stay zero.
template <int BASE, int TA, int TB, int P, int NW, int IM_OFF, int B_BYTES>
__device__ __forceinline__ void gen_step_packed(const unsigned (&gh)[NW], unsigned gbase, unsigned bases,
                                                unsigned dst, unsigned dstm) {
  const unsigned ga = gbase + ((bases & 1023u) << 3);
  const unsigned gb = gbase + (((bases >> 10) & 1023u) << 3);
  float ar = 0.f, ai = 0.f, br = 0.f, bi = 0.f;
#pragma unroll
  for (int q = 0; q < TA; ++q) {
    const float c = packed_coef(gh, BASE + q);
    const float2 g = lds_f2(ga + (unsigned)(q * 16 * P));
    ar = fmaf(c, g.x, ar);
    ai = fmaf(c, g.y, ai);
  }
#pragma unroll
  for (int q = 0; q < TB; ++q) {
    const float c = packed_coef(gh, BASE + TA + q);
    const float2 g = lds_f2(gb + (unsigned)(q * 16 * P));
    br = fmaf(c, g.x, br);
    bi = fmaf(c, g.y, bi);
  }
  store_item<IM_OFF, B_BYTES>(lds_f2(gbase + ((bases >> 20) << 3)), ar, ai, br, bi, dst, dstm);
}

// The pair table of one pair, lane d (< P): A[p][d] = Pn_p^d(cos theta) h_p(x) for p >= d at
// p*P + d, and the phases e^{+-i d phi} at P*P + 2L +- d.
template <int L>
__device__ __forceinline__ void pair_table(float2* g, int d, float ct, float st, float cdp, float sdp,
                                           float x, float sx, float cx, const float* legA,
                                           const float* legB, const float* legS) {
  constexpr int P = 2 * L + 1;
  g[P * P + 2 * L + d] = make_float2(cdp, sdp);
  if (d) g[P * P + 2 * L - d] = make_float2(cdp, -sdp);
  const float ix = __fdividef(1.0f, x);
  float hr0 = sx * ix, hi0 = -cx * ix;                                         // h_0
  float hr1 = (sx - x * cx) * ix * ix, hi1 = -(cx + x * sx) * ix * ix;         // h_1
  float Pp = 0.f, Pc = 0.f, stp = 1.f;
#pragma unroll
  for (int p = 0; p < P; ++p) {
    if (p == d) Pc = legS[d] * stp;
    if (p < d) stp *= st;
    if (p >= d) {
      g[p * P + d] = make_float2(Pc * hr0, Pc * hi0);
      if (p + 1 < P) {
        const float Pn = legA[p * P + d] * ct * Pc - legB[p * P + d] * Pp;
        Pp = Pc;
        Pc = Pn;
      }
    }
    if (p + 1 < P) {
      const float f = (float)(2 * p + 3) * ix;
      const float nr = f * hr1 - hr0, ni = f * hi1 - hi0;
      hr0 = hr1; hi0 = hi1; hr1 = nr; hi1 = ni;
    }
  }
}

// ---- the kernel ---------------------------------------------------------------------------
// NG right-hand-side groups of 64 per block (1 or 2): with two, every W_ij is generated once for
// 128 columns; the source panels of the two groups pass through the stage ring one after the
// other and the accumulators of group g sit at tensor-memory column g * 4 HP.
template <int L, int NG>
__global__ void __launch_bounds__(kPanelThreads, 1) panel_kernel(PanelArgs a) {
  using G = PanelGeom<L>;
  constexpr int TMEM_COLS = tmem_cols(4 * G::HP * NG);
  static_assert(4 * G::HP * NG <= 512, "accumulators exceed tensor memory");
  using Sched = PanelSched<L>;
  static_assert(Sched::kWarps == kGenWarps, "schedule built for another warp count");
  constexpr int H = G::H, HP = G::HP, P = G::P, KS = G::KS;
  constexpr int S = Sched::kSlots, NS = Sched::kSteps;
  constexpr int XS = G::X_STAGES, WS = G::W_STAGES;
  constexpr bool PK = G::PACKED;
  constexpr int NW = (S + 1) / 2;  // packed coefficient words
  extern __shared__ __align__(1024) unsigned char panel_smem[];
  unsigned char* xs = panel_smem + G::X_OFF;                                  // [XS][X_STAGE]
  unsigned char* ws = panel_smem + G::W_OFF;                                  // [WS][W_STAGE]
  unsigned char* gt = panel_smem + G::G_OFF;                                  // [4][G_STAGE]
  float* legA = reinterpret_cast<float*>(panel_smem + G::LEG_OFF);            // [P][P]
  float* legB = legA + P * P;
  float* legS = legB + P * P;
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(panel_smem + G::BAR_OFF);
  unsigned long long* xfull = bars;        // [XS] source panel landed
  unsigned long long* xempty = bars + 3;   // [XS] MMAs of the panel done
  unsigned long long* wfull = bars + 6;    // [WS] W generated (one arrival per generator warp)
  unsigned long long* wempty = bars + 9;   // [WS] MMAs of the W stage done
  unsigned long long* gfull = bars + 12;   // [4] pair table ready
  unsigned long long* gempty = bars + 16;  // [4] pair table consumed (one arrival per generator warp)
  unsigned long long* accum = bars + 20;   // accumulators final
  unsigned* tmem_slot = reinterpret_cast<unsigned*>(bars + 21);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(bars + 22);
  volatile int* issued = reinterpret_cast<volatile int*>(bars + 23);  // [XS] newest unit loaded per stage

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int i = blockIdx.x;    // receiving sphere
  const int grp0 = blockIdx.y * NG;  // first right-hand-side group of 64 of this block
  const int N = a.n_particles;
  const int n_iter = N - 1;    // every source but the receiver itself

  // generation data of this thread (registers): per slot an FP32 coefficient and a pair-table
  // offset, or (packed variant) two FP16 coefficients per word
  float gc[PK ? 1 : S];
  unsigned go[PK ? 1 : S], gh[PK ? NW : 1];
  // store offsets of the entry and mirror rows: absolute shared addresses, or (packed variant)
  // both W-stage offsets in 4-byte units in one register, entry in the low half; ge: the phase
  // offset, or (packed variant) the step's table bases
  unsigned gd[NS], gm[PK ? 1 : NS], ge[NS];
  if (tid < kGenThreads) {
    if constexpr (PK) {
#pragma unroll
      for (int w = 0; w < NW; ++w) gh[w] = __ldg(a.gen_goff + w * kGenThreads + tid);
    } else {
#pragma unroll
      for (int q = 0; q < S; ++q) {
        gc[q] = __ldg(a.gen_coef + q * kGenThreads + tid);
        go[q] = __ldg(a.gen_goff + q * kGenThreads + tid);
      }
    }
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      const unsigned od = __ldg(a.gen_dst + k * kGenThreads + tid);
      const unsigned om = __ldg(a.gen_dst + (NS + k) * kGenThreads + tid);
      if constexpr (PK) {
        gd[k] = (od >> 2) | ((om >> 2) << 16);  // 4-byte units
      } else {
        gd[k] = smem_addr(ws) + od;
        gm[k] = smem_addr(ws) + om;
      }
      ge[k] = __ldg(a.gen_dst + (2 * NS + k) * kGenThreads + tid);
    }
  }
  // zero the W stages (padding rows and columns stay zero) and the pair-table stages (entries
  // p < d are never written), Legendre tables to shared memory
  static_assert(G::G_STAGE % 16 == 0 && G::G_OFF == G::W_OFF + G::W_STAGES * G::W_STAGE, "layout");
  for (int o = tid; o < (G::W_STAGES * G::W_STAGE + G::G_STAGES * G::G_STAGE) / 16; o += blockDim.x)
    reinterpret_cast<float4*>(ws)[o] = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int o = tid; o < P * P; o += blockDim.x) {
    const int p = o / P, d = o - (o / P) * P;
    legA[o] = (float)a.leg->alpha[p * kLegStride + d];
    legB[o] = (float)a.leg->beta[p * kLegStride + d];
  }
  for (int o = tid; o < P; o += blockDim.x) legS[o] = (float)a.leg->start[o];
  if (tid == 0) {
    for (int b = 0; b < 3; ++b) mbar_init(&xfull[b], 1);
    for (int b = 0; b < 3; ++b) mbar_init(&xempty[b], 1);
    for (int b = 0; b < 3; ++b) mbar_init(&wfull[b], kGenWarps);
    for (int b = 0; b < 3; ++b) mbar_init(&wempty[b], 1);
    for (int b = 0; b < 4; ++b) mbar_init(&gfull[b], 1);
    for (int b = 0; b < 4; ++b) mbar_init(&gempty[b], kGenWarps);
    mbar_init(accum, 1);
    *abort_flag = 0;
    for (int b = 0; b < 3; ++b) issued[b] = -1;  // stages beyond XS stay unused
    mbar_fence_init();
  }
  if (warp == kMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = *tmem_slot;

  if (warp < kGenWarps) {
    // ===================== W generation =====================
    const unsigned gt0 = smem_addr(gt);
    for (int t = 0; t < n_iter; ++t) {
      const int sw = t % WS, sg = t & 3;
      int ok = 1;
      if (lane == 0) {
        ok = (t < WS || wait_or_abort(&wempty[sw], (unsigned)(((t / WS) - 1) & 1), abort_flag,
                                      a.wait_ns)) &&
             wait_or_abort(&gfull[sg], (unsigned)((t >> 2) & 1), abort_flag, a.wait_ns);
      }
      __syncwarp();  // orders the other lanes' reads after lane 0's acquire
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) break;
      const unsigned gbase = after_wait(gt0 + (unsigned)(sg * G::G_STAGE));
      const unsigned woff = (unsigned)(sw * G::W_STAGE);
      const unsigned wsb = smem_addr(ws) + woff;
#define YASF_GEN_STEP(k, base, ta, tb)                                                         \
  if constexpr (PK) {                                                                           \
    gen_step_packed<base, ta, tb, P, NW, G::IM_OFF, G::B_BYTES>(                                \
        gh, gbase, ge[k], wsb + ((gd[k] & 0xFFFFu) << 2), wsb + ((gd[k] >> 16) << 2));           \
  } else {                                                                                      \
    gen_step<base, ta, tb, (PK ? 1 : S), G::IM_OFF, G::B_BYTES>(gc, go, gbase, ge[k],           \
                                                                 gd[k] + woff, gm[PK ? 0 : k] + woff); \
  }
      if constexpr (L == 1) { YASF_PANEL_STEPS_1(YASF_GEN_STEP) }
      if constexpr (L == 2) { YASF_PANEL_STEPS_2(YASF_GEN_STEP) }
      if constexpr (L == 3) { YASF_PANEL_STEPS_3(YASF_GEN_STEP) }
      if constexpr (L == 4) { YASF_PANEL_STEPS_4(YASF_GEN_STEP) }
      if constexpr (L == 5) { YASF_PANEL_STEPS_5(YASF_GEN_STEP) }
      if constexpr (L == 6) { YASF_PANEL_STEPS_6(YASF_GEN_STEP) }
      if constexpr (L == 7) { YASF_PANEL_STEPS_7(YASF_GEN_STEP) }
      if constexpr (L == 8) { YASF_PANEL_STEPS_8(YASF_GEN_STEP) }
#undef YASF_GEN_STEP
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(&wfull[sw]);
        mbar_arrive(&gempty[sg]);
      }
    }
  } else if (warp == kMmaWarp) {
    // ===================== MMA issuer =====================
    if (lane == 0) {
      constexpr unsigned idesc = umma_idesc_tf32(128, 2 * HP, false);
      const unsigned long long da0 = umma_desc(smem_addr(xs), G::A_LBO, 128);
      const unsigned long long db0 = umma_desc(smem_addr(ws), G::B_LBO, 128);
      constexpr unsigned long long a_op = (unsigned long long)(G::A_BYTES >> 4);
      constexpr unsigned long long b_op = (unsigned long long)(G::B_BYTES >> 4);
      constexpr unsigned long long ak = (unsigned long long)((2 * G::A_LBO) >> 4);
      constexpr unsigned long long bk = (unsigned long long)((2 * G::B_LBO) >> 4);
      bool stop = false;
      for (int t = 0; t < n_iter && !stop; ++t) {
        const int sw = t % WS;
        if (!wait_or_abort(&wfull[sw], (unsigned)((t / WS) & 1), abort_flag, a.wait_ns)) break;
        const unsigned long long dw = db0 + (unsigned long long)sw * (unsigned long long)(G::W_STAGE >> 4);
#pragma unroll
        for (int g = 0; g < NG; ++g) {
          const int u = t * NG + g;  // source-panel unit: pair t, group g
          const int sx = u % XS;
          if (!wait_or_abort(&xfull[sx], (unsigned)((u / XS) & 1), abort_flag, a.wait_ns)) {
            stop = true;
            break;
          }
          tc_fence_after();
          const unsigned long long dx = da0 + (unsigned long long)sx * (unsigned long long)(G::X_STAGE >> 4);
          const unsigned td = tmem + (unsigned)(g * 4 * HP);
#pragma unroll
          for (int kk = 0; kk < KS; ++kk) {
            const unsigned acc = (t == 0 && kk == 0) ? 0u : 1u;
            umma_tf32(td, dx + kk * ak, dw + kk * bk, idesc, acc);                         // [S;Si] [P;Pi]
            umma_tf32(td + 2 * HP, dx + a_op + kk * ak, dw + b_op + kk * bk, idesc, acc);  // [D;Di] [Q;Qi]
          }
          umma_commit(&xempty[sx]);
        }
        if (stop) break;
        umma_commit(&wempty[sw]);
      }
      umma_commit(accum);
    }
    __syncwarp();
  } else if (warp == kLoadWarp) {
    // ===================== source panels =====================
    if (lane == 0) {
      for (int u = 0; u < n_iter * NG; ++u) {
        const int t = u / NG, g = u - (u / NG) * NG;
        const int sx = u % XS;
        const int j = t < i ? t : t + 1;
        if (*abort_flag) break;
        if (u >= XS &&
            !wait_or_abort(&xempty[sx], (unsigned)(((u / XS) - 1) & 1), abort_flag, a.wait_ns))
          break;
        const unsigned char* src =
            reinterpret_cast<const unsigned char*>(a.xp) + ((size_t)(grp0 + g) * N + j) * G::X_STAGE;
        issued[sx] = u;  // written before the copy: the next load into this stage waits for its MMAs
        bulk_load(xs + sx * G::X_STAGE, src, G::X_STAGE, &xfull[sx]);
      }
    }
    __syncwarp();
  } else {
    // ===================== pair tables (two warps take alternate pairs) =====================
    const int par = warp - kGeomWarp0;
    const double xi = a.pos[3 * i], yi = a.pos[3 * i + 1], zi = a.pos[3 * i + 2];
    const float kf = (float)a.k;
    for (int t = par; t < n_iter && !a.stall; t += 2) {
      const int sg = t & 3;
      const int j = t < i ? t : t + 1;
      int ok = 1;
      if (lane == 0)
        ok = t < 4 ? !*abort_flag
                   : wait_or_abort(&gempty[sg], (unsigned)(((t >> 2) - 1) & 1), abort_flag,
                                   a.wait_ns);
      __syncwarp();
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) break;
      if (lane < P) {
        const float dx = (float)(xi - a.pos[3 * j]);
        const float dy = (float)(yi - a.pos[3 * j + 1]);
        const float dz = (float)(zi - a.pos[3 * j + 2]);
        const float rho2 = dx * dx + dy * dy;
        const float r2 = rho2 + dz * dz;
        const float rinv = rsqrtf(r2);
        const float r = r2 * rinv;
        const float ct = fminf(1.f, fmaxf(-1.f, dz * rinv));
        float c1 = 1.f, s1 = 0.f, st = 0.f;  // e^{i phi}, sin theta
        if (rho2 > 0.f) {
          const float rhoinv = rsqrtf(rho2);
          c1 = dx * rhoinv;
          s1 = dy * rhoinv;
          st = rho2 * rhoinv * rinv;
        }
        float cdp = 1.f, sdp = 0.f;  // e^{i d phi} by powers of e^{i phi}
#pragma unroll
        for (int q = 0; q < P - 1; ++q) {
          if (q < lane) {
            const float cn = cdp * c1 - sdp * s1;
            sdp = cdp * s1 + sdp * c1;
            cdp = cn;
          }
        }
        const float x = kf * r;
        float sx, cx;
        sincosf(x, &sx, &cx);
        pair_table<L>(reinterpret_cast<float2*>(gt + sg * G::G_STAGE), lane, ct, st, cdp, sdp, x, sx,
                      cx, legA, legB, legS);
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&gfull[sg]);
    }
  }
  __syncthreads();  // every role has left its loop: no further source copy will be issued

  // ===================== epilogue =====================
  if (warp < 4) {
    // No copy may still be landing when the stages are reused or the block exits. A load into a
    // stage is issued only after the MMAs consumed the previous one, so only the newest load of
    // each stage can be in flight (bounded waits).
    if (tid == 0)
      for (int b = 0; b < XS; ++b)
        if (issued[b] >= 0) (void)panel_wait(&xfull[b], (unsigned)((issued[b] / XS) & 1));
    // wait (bounded) for the MMAs before reading tensor memory
    const bool ok = n_iter == 0 || panel_wait(accum, 0, a.wait_ns);
    tc_fence_after();
    named_sync(1, 128);  // the drain above precedes every write to the exchange buffer
    const bool aborted = *abort_flag != 0;
    if (aborted && tid == 0) atomicExch(a.err, 1);
    float* xch = reinterpret_cast<float*>(xs);  // [64][XCH_STRIDE]: imaginary-row accumulators
#pragma unroll 1
    for (int g = 0; g < NG; ++g) {
      const unsigned lane_base = tmem + ((unsigned)(32 * warp) << 16) + (unsigned)(g * 4 * HP);
      if (g > 0) named_sync(1, 128);  // the previous group's exchange rows are consumed
      if (warp >= 2) {
        const int r = 32 * (warp - 2) + lane;
#pragma unroll 1
        for (int n = 0; n < 4 * HP; n += 8) {
          float v[8];
          tmem_ld32<8>(lane_base + n, v);
#pragma unroll
          for (int u = 0; u < 8; ++u) xch[r * G::XCH_STRIDE + n + u] = v[u];
        }
      }
      named_sync(1, 128);
      if (warp < 2) {
        const int c = 32 * warp + lane;  // column within the group
        const int col = (grp0 + g) * G::M + c;
        const bool live = col < a.nrhs;
        const float* im = xch + c * G::XCH_STRIDE;
#pragma unroll 1
        for (int n = 0; n < H; n += 8) {
          float pr[8], pi[8], qr[8], qi[8];
          tmem_ld32<8>(lane_base + n, pr);                // S_r P_r^T
          tmem_ld32<8>(lane_base + HP + n, pi);           // S_r P_i^T
          tmem_ld32<8>(lane_base + 2 * HP + n, qr);       // D_r Q_r^T
          tmem_ld32<8>(lane_base + 3 * HP + n, qi);       // D_r Q_i^T
          if (!live) continue;
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            const int q = n + u;
            if (q >= H) break;
            const float ur = pr[u] - im[HP + q], ui = pi[u] + im[q];
            const float vr = qr[u] - im[3 * HP + q], vi = qi[u] + im[2 * HP + q];
            double y1r = 0.5 * ((double)ur + (double)vr), y1i = 0.5 * ((double)ui + (double)vi);
            double y2r = 0.5 * ((double)ur - (double)vr), y2i = 0.5 * ((double)ui - (double)vi);
            if (n_iter == 0) { y1r = y1i = y2r = y2i = 0.0; }
            if (aborted || !ok) { y1r = y1i = y2r = y2i = __longlong_as_double(0x7ff8000000000000LL); }
#pragma unroll
            for (int half = 0; half < 2; ++half) {
              const int nn = half * H + q;
              const double yr = half ? y2r : y1r, yi = half ? y2i : y1i;
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
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kMmaWarp) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(TMEM_COLS)
                 : "memory");
  }
}

// Source panels: columns [grp*64, grp*64+64) of x as the A operands [S_r; S_i] and [D_r; D_i]
// (S = X1 + X2, D = X1 - X2 of every column, rounded to TF32).
template <int L>
__global__ void xpanel_kernel(int n_particles, int nmax, int nrhs, long long ld, const double2* x,
                              float* xp) {
  using G = PanelGeom<L>;
  constexpr int H = G::H, HP = G::HP, M = G::M;
  const int j = blockIdx.x, grp = blockIdx.y;
  unsigned char* dst = reinterpret_cast<unsigned char*>(xp) + ((size_t)grp * n_particles + j) * G::X_STAGE;
  for (int e = threadIdx.x; e < M * HP; e += blockDim.x) {
    const int r = e / HP, q = e - (e / HP) * HP;
    const int col = grp * M + r;
    float sr = 0.f, si = 0.f, dr = 0.f, di = 0.f;
    if (q < H && col < nrhs) {
      const double2 v1 = x[(size_t)col * ld + (size_t)j * nmax + q];
      const double2 v2 = x[(size_t)col * ld + (size_t)j * nmax + H + q];
      sr = to_tf32((float)(v1.x + v2.x));
      si = to_tf32((float)(v1.y + v2.y));
      dr = to_tf32((float)(v1.x - v2.x));
      di = to_tf32((float)(v1.y - v2.y));
    }
    *reinterpret_cast<float*>(dst + kmajor_offset(r, q, 128)) = sr;
    *reinterpret_cast<float*>(dst + kmajor_offset(64 + r, q, 128)) = si;
    *reinterpret_cast<float*>(dst + G::A_BYTES + kmajor_offset(r, q, 128)) = dr;
    *reinterpret_cast<float*>(dst + G::A_BYTES + kmajor_offset(64 + r, q, 128)) = di;
  }
}

}  // namespace yasf
