// Complex64 contraction body: Q receivers per thread (build-time, one by default).
//
// Same factored sum, stream order, stage pipeline, cutoff and timeout behaviour as contract_body
// (coupling.cuh), with the pair side and the accumulators in float. Thread q-slot j owns receiver
// (Q tile + j) blockDim.x + threadIdx.x; each V entry read from the stage (one broadcast 16-byte
// shared load of (re, im, -im, re)) feeds two packed FP32 FMAs (FFMA2) per receiver:
//   (y_re, y_im) += (g_re, g_re) * (re, im) + (g_im, g_im) * (-im, re).
// The order-p loop is unrolled so every (m1, p) has a compile-time row count. Measured on B200
// (2000 spheres, lmax 6): one receiver per thread 15.4 ms, two 22.3 ms (the second receiver's
// pair-side registers push the kernel to fewer resident blocks), against 24.5 ms for float64.
// Pair geometry and h_0, h_1 are evaluated in float64 (positions stay exact), then rounded; every
// recurrence runs in float.
//
// Included by coupling.cuh inside namespace yasf, after contract_body (it uses the stage helpers).
#pragma once

// Receivers per thread and whether the order-p loop is unrolled: build-time choices (defaults 1, 1),
// the host layout follows kC64Receivers.
#ifndef YASF_C64_RECEIVERS
#define YASF_C64_RECEIVERS 1
#endif
#ifndef YASF_C64_UNROLL_P
#define YASF_C64_UNROLL_P 1
#endif
constexpr int kC64Receivers = YASF_C64_RECEIVERS;  // receivers per thread of the complex64 contraction

template <int L, int NB, int BID>
__device__ __forceinline__ bool contract_body_c64(const ContractArgs& a, int tile, int chunk, char* smem,
                                                  unsigned long long* bars, unsigned (&uses)[2],
                                                  unsigned (&issued)[2]) {
  using VE = float4;
  constexpr int Q = kC64Receivers;
  constexpr BundleInfo bi = make_bundle(L, BID, NB);
  constexpr int NR = bi.rows;
  constexpr int PMAX = 2 * L;

  int s1[Q];
  bool active[Q];
  double px[Q], py[Q], pz[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    s1[q] = (tile * Q + q) * blockDim.x + threadIdx.x;
    active[q] = s1[q] < a.n_particles;
    const int sc = active[q] ? s1[q] : 0;
    px[q] = __ldg(a.pos + 3 * sc + 0);
    py[q] = __ldg(a.pos + 3 * sc + 1);
    pz[q] = __ldg(a.pos + 3 * sc + 2);
  }
  float2 yc[Q][NR];
#pragma unroll
  for (int q = 0; q < Q; ++q)
#pragma unroll
    for (int r = 0; r < NR; ++r) yc[q][r] = make_float2(0.f, 0.f);

  const int sb = chunk * a.sources_per_chunk;
  const int se = min(a.n_particles, sb + a.sources_per_chunk);
  const VE* vbase = reinterpret_cast<const VE*>(a.v) + (size_t)a.bundle_begin[BID] * a.n_particles;
  const int vstride = a.bundle_len[BID];
  const unsigned stage_bytes = (unsigned)(vstride * sizeof(VE));
  VE* const stage0 = reinterpret_cast<VE*>(smem);
  VE* const stage1 = stage0 + vstride;
  if (threadIdx.x == 0 && sb < se && !a.stall) {
    bulk_load(stage0, vbase + (size_t)sb * vstride, stage_bytes, &bars[0]);
    ++issued[0];
  }
  bool timed_out = false;

#pragma unroll 1
  for (int s2 = sb; s2 < se; ++s2) {
    const int it = s2 - sb;
    const int cur = it & 1;
    if (threadIdx.x == 0 && s2 + 1 < se) {
      bulk_load(cur ? stage0 : stage1, vbase + (size_t)(s2 + 1) * vstride, stage_bytes, &bars[cur ^ 1]);
      ++issued[cur ^ 1];
    }
    const double sx2 = __ldg(a.pos + 3 * s2 + 0);
    const double sy2 = __ldg(a.pos + 3 * s2 + 1);
    const double sz2 = __ldg(a.pos + 3 * s2 + 2);
    // pair geometry d = pos[s1] - pos[s2] (yasfpy/functions/misc.py:149-166) and h_0, h_1
    float ctf[Q], stf[Q], eR[Q], eI[Q], h0r[Q], h0i[Q], h1r[Q], h1i[Q], inv_x[Q];
    bool use_any = false;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const double dx = px[q] - sx2, dy = py[q] - sy2, dz = pz[q] - sz2;
      const double r2 = dx * dx + dy * dy + dz * dz;
      const bool use = active[q] && s2 != s1[q] && (a.cutoff2 < 0.0 || r2 <= a.cutoff2);
      use_any |= use;
      const double r = sqrt(r2);
      double ct = (r > 0.0) ? dz / r : 0.0;
      ct = fmin(1.0, fmax(-1.0, ct));
      const double rho = sqrt(dx * dx + dy * dy);
      ctf[q] = (float)ct;
      stf[q] = (float)sqrt(1.0 - ct * ct);
      eR[q] = (float)((rho > 0.0) ? dx / rho : 1.0);
      eI[q] = (float)((rho > 0.0) ? dy / rho : 0.0);
      const double xx = (use && r > 0.0) ? a.k * r : 1.0;
      const double mask = use ? 1.0 : 0.0;
      double sx, cx;
      sincos(xx, &sx, &cx);
      const double ix = 1.0 / xx;
      // h_0 = -i e^{ix}/x ; h_1 = -e^{ix}(x + i)/x^2
      h0r[q] = (float)(mask * sx * ix);
      h0i[q] = (float)(-mask * cx * ix);
      h1r[q] = (float)(mask * (sx - xx * cx) * ix * ix);
      h1i[q] = (float)(-mask * (cx + xx * sx) * ix * ix);
      inv_x[q] = (float)ix;
    }
    const bool ok = mbar_wait(&bars[cur], uses[cur] & 1u, a.poll_limit);
    if (__syncthreads_or(!ok)) {
      timed_out = true;
      if (threadIdx.x == 0) atomicExch(a.err, 1);
      break;
    }
    ++uses[cur];
    if (a.cutoff2 >= 0.0 && !__syncthreads_or(use_any)) {
      __syncthreads();
      continue;
    }
    const VE* vp = cur ? stage1 : stage0;
    float st_d[Q], ph_r[Q], ph_i[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) { st_d[q] = 1.f; ph_r[q] = 1.f; ph_i[q] = 0.f; }

#pragma unroll 1
    for (int d = 0; d <= PMAX; ++d) {
      float P_prev[Q], P_cur[Q], ha_r[Q], ha_i[Q], hb_r[Q], hb_i[Q];
      const float start = __ldg(a.leg->start + d);
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        if (d > 0) {
          st_d[q] *= stf[q];
          const float t = ph_r[q] * eR[q] - ph_i[q] * eI[q];
          ph_i[q] = ph_r[q] * eI[q] + ph_i[q] * eR[q];
          ph_r[q] = t;
        }
        P_prev[q] = 0.f;
        P_cur[q] = start * st_d[q];
        ha_r[q] = h0r[q]; ha_i[q] = h0i[q]; hb_r[q] = h1r[q]; hb_i[q] = h1i[q];
      }
      // restart the Hankel recurrences and advance them to order d
#pragma unroll 1
      for (int o = 0; o < d; ++o) {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
          const float f = (float)(2 * o + 3) * inv_x[q];
          const float nr = f * hb_r[q] - ha_r[q];
          const float ni = f * hb_i[q] - ha_i[q];
          ha_r[q] = hb_r[q]; ha_i[q] = hb_i[q]; hb_r[q] = nr; hb_i[q] = ni;
        }
      }
      // The order-p loop is unrolled (d is a warp-uniform runtime value, p < d is skipped): the
      // valid row count of every (m1, p) is a compile-time constant, so the row loops below are
      // straight-line code without predicated-off row slots taking issue slots.
      constexpr int kPU = YASF_C64_UNROLL_P ? PMAX + 1 : 1;
#pragma unroll kPU
      for (int p = YASF_C64_UNROLL_P ? 0 : d; p <= PMAX; ++p) {
        if (p < d) continue;
        float2 gpr2[Q], gpi2[Q], gmr2[Q], gmi2[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
          const float g0r = P_cur[q] * ha_r[q], g0i = P_cur[q] * ha_i[q];
          // G(+d) = g0 e^{i d phi}, G(-d) = g0 e^{-i d phi}, as packed (g, g) operands
          const float gpr = g0r * ph_r[q] - g0i * ph_i[q];
          const float gpi = g0r * ph_i[q] + g0i * ph_r[q];
          const float gmr = g0r * ph_r[q] + g0i * ph_i[q];
          const float gmi = g0i * ph_r[q] - g0r * ph_i[q];
          gpr2[q] = make_float2(gpr, gpr);
          gpi2[q] = make_float2(gpi, gpi);
          gmr2[q] = make_float2(gmr, gmr);
          gmi2[q] = make_float2(gmi, gmi);
        }
#pragma unroll kSgnUnroll
        for (int sgn = 0; sgn < 2; ++sgn) {
          if (sgn == 1 && d == 0) break;
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
                const float2 v01 = make_float2(v.x, v.y), v23 = make_float2(v.z, v.w);
#pragma unroll
                for (int q = 0; q < Q; ++q) {
                  const float2 gr = sgn == 0 ? gpr2[q] : gmr2[q];
                  const float2 gi = sgn == 0 ? gpi2[q] : gmi2[q];
                  yc[q][off + rr] = __ffma2_rn(gr, v01, yc[q][off + rr]);
                  yc[q][off + rr] = __ffma2_rn(gi, v23, yc[q][off + rr]);
                }
              }
            }
            vp += nv;
          }
        }
        // advance Legendre (order d fixed) and Hankel recurrences to p + 1
        if (p < PMAX) {
          const float al = __ldg(a.leg->alpha + p * kLegStride + d);
          const float be = __ldg(a.leg->beta + p * kLegStride + d);
          const float f0 = (float)(2 * p + 3);
#pragma unroll
          for (int q = 0; q < Q; ++q) {
            const float P_next = al * ctf[q] * P_cur[q] - be * P_prev[q];
            P_prev[q] = P_cur[q];
            P_cur[q] = P_next;
            const float f = f0 * inv_x[q];
            const float nr = f * hb_r[q] - ha_r[q];
            const float ni = f * hb_i[q] - ha_i[q];
            ha_r[q] = hb_r[q]; ha_i[q] = hb_i[q]; hb_r[q] = nr; hb_i[q] = ni;
          }
        }
      }
    }
    __syncthreads();  // every warp is done with this stage before it is refilled
  }
  if (timed_out) {
    if (threadIdx.x == 0) {
#pragma unroll
      for (int b = 0; b < 2; ++b)
        if (issued[b] > uses[b]) (void)mbar_wait(&bars[b], uses[b] & 1u);
    }
    return false;
  }
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    if (!active[q]) continue;
    float2* out = reinterpret_cast<float2*>(a.partial) + ((size_t)chunk * a.n_particles + s1[q]) * a.nmax;
#pragma unroll
    for (int i = 0; i < bi.count; ++i) {
      const int m1 = bi.m1[i];
#pragma unroll
      for (int rr = 0; rr < 2 * L; ++rr)
        if (rr < rows_of_m(L, m1)) out[mode_index(L, row_tau(rr), row_l(L, rr), m1)] = yc[q][bi.row_off[i] + rr];
    }
  }
  return true;
}
