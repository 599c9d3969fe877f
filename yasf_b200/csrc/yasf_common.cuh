// Shared definitions for the yasf_b200 CUDA sources: status codes, mode indexing,
// the canonical order of the per-source "V stream" that couples the source-side and
// pair-side halves of the factored translation, and the bundle partition of the
// receiving azimuthal orders m1.
//
// Index conventions follow the reference exactly:
//   per-particle mode index n(tau,l,m) = (tau-1)*L*(L+2) + (l-1)*(l+1) + l + m
//   (yasfpy/functions/cpu_numba.py:371-407), global index s*nmax + n (particle-major).
#pragma once

#include <cstddef>
#include <cstdint>

#include "../../include/yasf_b200.h"

#define YASF_LMAX_MAX 8
#define YASF_PMAX_MAX (2 * YASF_LMAX_MAX)

namespace yasf {

__host__ __device__ constexpr int nmax_of(int L) { return 2 * L * (L + 2); }

__host__ __device__ constexpr int mode_index(int L, int tau, int l, int m) {
  return (tau - 1) * L * (L + 2) + (l - 1) * (l + 1) + l + m;
}

__host__ __device__ constexpr int iabs_c(int v) { return v < 0 ? -v : v; }
__host__ __device__ constexpr int imax_c(int a, int b) { return a > b ? a : b; }
__host__ __device__ constexpr int imin_c(int a, int b) { return a < b ? a : b; }

// Number of receiving rows (tau1, l1) for a given m1: l1 in [max(1,|m1|), L], tau1 in {1,2}.
__host__ __device__ constexpr int rows_of_m(int L, int m1) {
  return 2 * (L - imax_c(1, iabs_c(m1)) + 1);
}

// Row r of the m1 group: l1 descending from L, tau1 = 1,2 innermost. With this order the
// rows that can couple to order p (those with l1 + L >= p) form a prefix of the group.
__host__ __device__ constexpr int row_l(int L, int r) { return L - r / 2; }
__host__ __device__ constexpr int row_tau(int r) { return 1 + (r & 1); }

// Length of the valid prefix of the m1 group for translation order p.
__host__ __device__ constexpr int valid_rows(int L, int m1, int p) {
  return (imax_c(imax_c(1, iabs_c(m1)), p - L) > L)
             ? 0
             : 2 * (L - imax_c(imax_c(1, iabs_c(m1)), p - L) + 1);
}

// Receiving orders m1 are split into bundles so that one thread keeps the accumulators of a
// whole bundle in registers while the pair-side factors (Hankel, Legendre, azimuthal phase)
// are generated once per bundle. Bundles are a snake deal of m1 sorted by |m1|, which
// balances both the row count and the stream length. The float64 and complex64 kernels may use
// different counts (each its own stream layout): at lmax 6 on B200 the float64 contraction runs
// fastest with 3 bundles of 32 rows (22.3 ms per C2 matvec against 25.7 ms with 4), the complex64
// one with 4 of 24 rows (15.3 ms against 18.9 ms with 3, whose accumulators cost occupancy).
// Unroll factor of the contraction's (+d, -d) loop: 2 (unrolled) or 1 (rolled, half the code).
#ifndef YASF_SGN_UNROLL
#define YASF_SGN_UNROLL 2
#endif
constexpr int kSgnUnroll = YASF_SGN_UNROLL;  // (pragma arguments are not macro-expanded)
#ifndef YASF_BUNDLES_L6_F64
#define YASF_BUNDLES_L6_F64 3
#endif
#ifndef YASF_BUNDLES_L6_C64
#define YASF_BUNDLES_L6_C64 4
#endif
__host__ __device__ constexpr int num_bundles(int L, bool c64) {
  return L <= 3 ? 1
                : (L == 4 ? 2
                          : (L == 5 ? 3
                                    : (L == 6 ? (c64 ? YASF_BUNDLES_L6_C64 : YASF_BUNDLES_L6_F64)
                                              : (L == 7 ? 6 : 8))));
}

// The i-th m1 in the order 0, 1, -1, 2, -2, ...
__host__ __device__ constexpr int m_in_abs_order(int i) {
  return i == 0 ? 0 : ((i & 1) ? (i + 1) / 2 : -(i / 2));
}

// Bundle that the i-th m1 (abs order) belongs to.
__host__ __device__ constexpr int bundle_of_index(int i, int B) {
  return ((i / B) & 1) ? (B - 1 - (i % B)) : (i % B);
}

struct BundleInfo {
  int count;                          // number of m1 values
  int m1[2 * YASF_LMAX_MAX + 1];      // m1 values in kernel order
  int row_off[2 * YASF_LMAX_MAX + 1]; // accumulator offset of each m1 group
  int rows;                           // total rows (accumulators) of the bundle
};

// Bundle b of B at lmax L.
__host__ __device__ constexpr BundleInfo make_bundle(int L, int b, int B) {
  BundleInfo info{};
  info.count = 0;
  info.rows = 0;
  for (int i = 0; i < 2 * L + 1; ++i) {
    if (bundle_of_index(i, B) == b) {
      const int m1 = m_in_abs_order(i);
      info.m1[info.count] = m1;
      info.row_off[info.count] = info.rows;
      info.rows += rows_of_m(L, m1);
      info.count += 1;
    }
  }
  return info;
}

// Stream length (entries) of one bundle for one source particle. The stream order is
//   for d in 0..2L, for p in d..2L, for sign in (+,-) (only + when d == 0),
//     for m1 in bundle order with |m1 + sign*d| <= L, for r < valid_rows(m1, p).
// Each entry (tau1,l1,m1; p; m2=m1+sign*d) holds
//   V = sum_{tau2,l2} A[(tau1,l1,m1),(tau2,l2,m2),p] * x_source[(tau2,l2,m2)].
__host__ __device__ constexpr int bundle_stream_length(int L, int b, int B) {
  const BundleInfo bi = make_bundle(L, b, B);
  int len = 0;
  for (int d = 0; d <= 2 * L; ++d)
    for (int p = d; p <= 2 * L; ++p)
      for (int s = 0; s < (d == 0 ? 1 : 2); ++s) {
        const int sg = s == 0 ? 1 : -1;
        for (int i = 0; i < bi.count; ++i) {
          const int m2 = bi.m1[i] + sg * d;
          if (m2 < -L || m2 > L) continue;
          len += valid_rows(L, bi.m1[i], p);
        }
      }
  return len;
}

// Streams of consecutive sources start on 32-byte boundaries (even entry counts).
__host__ __device__ constexpr int padded_stream_length(int L, int b, int B) {
  return (bundle_stream_length(L, b, B) + 1) & ~1;
}

}  // namespace yasf
