// Batched solve of (I - T W) X = B for R right-hand sides (incidence directions x polarisations).
//
// Float64 iterative refinement around lockstep GMRES cycles. Each column keeps its own Krylov
// basis (float64, classical Gram-Schmidt with one re-orthogonalisation pass), Givens rotations
// and Hessenberg solve (float64, on the device); one operator application serves all live columns
// at once, so every W_ij is generated once per step for the whole panel:
//   refine:  R_c = B_c - A X_c            (float64 master operator: the dense multi-column kernel
//                                          for 12 or more live columns up to lmax 6, else column
//                                          by column)
//            solve A~ D_c = R_c to inner_rtol (A~: tensor-core TF32 panel, or the complex64 /
//                                            complex128 coupling kernels), X_c += D_c
// until ||B_c - A X_c|| <= rtol ||B_c|| for every column. The block-Jacobi preconditioner, when
// given, is applied on the left in the inner solves (complex64 factors for the reduced-precision
// operators). Columns that reach their inner tolerance, or break down, leave the cycle; columns
// that meet the outer tolerance leave the refinement.
#include <cmath>
#include <vector>

#include "capi_internal.h"

extern "C" int yasf_panel_workspace_size(const yasf_plan* plan, int n_particles, int nrhs,
                                         size_t* bytes);
extern "C" int yasf_panel_matvec(const yasf_plan* plan, int n_particles, const double* positions,
                                 double k_medium, const double* tmat, const double* x, double* y,
                                 int nrhs, long long ldx, long long ldy, void* workspace,
                                 size_t workspace_bytes, void* stream);
extern "C" int yasf_precond_apply(const yasf_precond* pc, const double* x, double* y, int nrhs,
                                  long long ld, int precision, void* stream);

namespace yasf {

constexpr int kBDot = 64;  // dot-product blocks per column

// partial[c][blk][k] = sum conj(Q_c[k]) w_c over the block's slice, live columns only.
__global__ void __launch_bounds__(256) bmdot_kernel(long long n, const double2* Q, long long q_col,
                                                    int nvec, const double2* w, long long w_col,
                                                    const int* live, double2* partial) {
  const int c = blockIdx.y;
  if (!live[c]) return;
  __shared__ double sr[8], si[8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const double2* wc = w + (size_t)c * w_col;
  for (int k = 0; k < nvec; ++k) {
    const double2* q = Q + (size_t)c * q_col + (size_t)k * n;
    double re = 0.0, im = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
      const double2 a = q[i], b = wc[i];
      re += a.x * b.x + a.y * b.y;
      im += a.x * b.y - a.y * b.x;
    }
    for (int off = 16; off > 0; off >>= 1) {
      re += __shfl_down_sync(0xffffffffu, re, off);
      im += __shfl_down_sync(0xffffffffu, im, off);
    }
    if (lane == 0) { sr[wid] = re; si[wid] = im; }
    __syncthreads();
    if (threadIdx.x == 0) {
      double tr = 0.0, ti = 0.0;
      for (int t = 0; t < (int)(blockDim.x >> 5); ++t) { tr += sr[t]; ti += si[t]; }
      partial[((size_t)c * gridDim.x + blockIdx.x) * nvec + k] = make_double2(tr, ti);
    }
    __syncthreads();
  }
}

// out[c][k] (+)= sum over blocks; norm mode: norm[c] = sqrt(re of vector 0).
__global__ void bfinal_kernel(int nvec, int nblk, const double2* partial, double2* out,
                              long long out_col, int accumulate, double* norm, const int* live) {
  const int k = blockIdx.x, c = blockIdx.y;
  if (!live[c]) return;
  __shared__ double sr[64], si[64];
  double re = 0.0, im = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
    const double2 v = partial[((size_t)c * nblk + b) * nvec + k];
    re += v.x;
    im += v.y;
  }
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
  if (threadIdx.x == 0) {
    if (norm) {
      // a NaN sum stays NaN (fmax alone would turn it into 0, a converged-looking norm)
      norm[c] = (isnan(sr[0]) ? sr[0] : sqrt(fmax(sr[0], 0.0)));
    } else if (accumulate) {
      double2* o = out + (size_t)c * out_col + k;
      o->x += sr[0];
      o->y += si[0];
    } else {
      out[(size_t)c * out_col + k] = make_double2(sr[0], si[0]);
    }
  }
}

// w_c += sign * sum_k h_c[k] Q_c[k] for live columns (h_c at h + c*h_col).
__global__ void __launch_bounds__(256) bupdate_kernel(long long n, const double2* Q, long long q_col,
                                                      int nvec, const double2* h, long long h_col,
                                                      double sign, double2* w, long long w_col,
                                                      const int* live) {
  const int c = blockIdx.y;
  if (!live[c]) return;
  __shared__ double2 sh[512];
  for (int k = threadIdx.x; k < nvec && k < 512; k += blockDim.x) sh[k] = h[(size_t)c * h_col + k];
  __syncthreads();
  double2* wc = w + (size_t)c * w_col;
  const double2* qc = Q + (size_t)c * q_col;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    double re = 0.0, im = 0.0;
    for (int k = 0; k < nvec; ++k) {
      const double2 q = qc[(size_t)k * n + i];
      const double2 cc = sh[k];
      re += cc.x * q.x - cc.y * q.y;
      im += cc.x * q.y + cc.y * q.x;
    }
    double2 v = wc[i];
    v.x += sign * re;
    v.y += sign * im;
    wc[i] = v;
  }
}

// out_c = in_c / norm[c] for live columns; zero for the others.
__global__ void bscale_kernel(long long n, const double2* in, long long in_col, const double* norm,
                              double2* out, long long out_col, const int* live) {
  const int c = blockIdx.y;
  const double nv = norm[c];
  const bool on = live[c] && nv > 0.0;
  const double f = on ? 1.0 / nv : 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double2 v = on ? in[(size_t)c * in_col + i] : make_double2(0.0, 0.0);
    out[(size_t)c * out_col + i] = make_double2(v.x * f, v.y * f);
  }
}

// Elementwise over the panel: mode 0: out = a - b ; 1: out += a ; 2: out = a.  (cols with mask)
__global__ void bax_kernel(long long n, int mode, const double2* a, const double2* b, double2* out,
                           const int* mask) {
  const int c = blockIdx.y;
  if (mask && !mask[c]) return;
  const size_t base = (size_t)c * n;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double2 av = a[base + i];
    if (mode == 0) {
      const double2 bv = b[base + i];
      out[base + i] = make_double2(av.x - bv.x, av.y - bv.y);
    } else if (mode == 1) {
      double2 o = out[base + i];
      o.x += av.x;
      o.y += av.y;
      out[base + i] = o;
    } else {
      out[base + i] = av;
    }
  }
}

__device__ inline double cabs_b(double2 z) { return hypot(z.x, z.y); }

// One thread per column: S_c = (beta_c, 0, ...).
__global__ void bstart_kernel(int R, int m, const double* beta, double2* S, const int* live) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= R || !live[c]) return;
  double2* s = S + (size_t)c * (m + 1);
  for (int i = 0; i <= m; ++i) s[i] = make_double2(0.0, 0.0);
  s[0] = make_double2(beta[c], 0.0);
}

// One thread per live column: finish column j of H_c (h1, rotations, S, presid, breakdown).
__global__ void bgivens_kernel(int R, int j, int m, double2* H, double* gc, double2* gs, double2* S,
                               const double* h0, const double* h1, double* presid, int* brk,
                               const int* live, double eps) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= R || !live[c]) return;
  double2* h = H + ((size_t)c * m + j) * (m + 1);
  double* g_c = gc + (size_t)c * m;
  double2* g_s = gs + (size_t)c * m;
  double2* s = S + (size_t)c * (m + 1);
  int b = 0;
  if (h1[c] <= eps * h0[c]) {
    h[j + 1] = make_double2(0.0, 0.0);
    b = 1;
  } else {
    h[j + 1] = make_double2(h1[c], 0.0);
  }
  for (int k = 0; k < j; ++k) {
    const double cc = g_c[k];
    const double2 sn = g_s[k];
    const double2 n0 = h[k], n1 = h[k + 1];
    h[k] = make_double2(cc * n0.x + sn.x * n1.x - sn.y * n1.y, cc * n0.y + sn.x * n1.y + sn.y * n1.x);
    h[k + 1] = make_double2(-(sn.x * n0.x + sn.y * n0.y) + cc * n1.x, -(sn.x * n0.y - sn.y * n0.x) + cc * n1.y);
  }
  const double2 f = h[j], g = h[j + 1];
  const double af = cabs_b(f), ag = cabs_b(g);
  double cc;
  double2 sn, r;
  if (ag == 0.0) {
    cc = 1.0; sn = make_double2(0.0, 0.0); r = f;
  } else if (af == 0.0) {
    cc = 0.0; sn = make_double2(g.x / ag, -g.y / ag); r = make_double2(ag, 0.0);
  } else {
    const double t = hypot(af, ag);
    cc = af / t;
    const double2 fu = make_double2(f.x / af, f.y / af);
    sn = make_double2((fu.x * g.x + fu.y * g.y) / t, (fu.y * g.x - fu.x * g.y) / t);
    r = make_double2(fu.x * t, fu.y * t);
  }
  g_c[j] = cc;
  g_s[j] = sn;
  h[j] = r;
  h[j + 1] = make_double2(0.0, 0.0);
  const double2 Sc = s[j];
  const double2 tmp = make_double2(-(sn.x * Sc.x + sn.y * Sc.y), -(sn.x * Sc.y - sn.y * Sc.x));
  s[j] = make_double2(cc * Sc.x, cc * Sc.y);
  s[j + 1] = tmp;
  presid[c] = cabs_b(tmp);
  brk[c] = b || !isfinite(presid[c]);
}

// One thread per column with stop[c] >= 0: y_c = H_c(0:stop,0:stop)^{-1} S_c.
__global__ void bbacksolve_kernel(int R, int m, const int* stop, const double2* H, double2* S,
                                  double2* y) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= R) return;
  const int col = stop[c];
  double2* yc = y + (size_t)c * (m + 1);
  for (int i = 0; i <= m; ++i) yc[i] = make_double2(0.0, 0.0);
  if (col < 0) return;
  const double2* Hc = H + (size_t)c * m * (m + 1);
  double2* s = S + (size_t)c * (m + 1);
  auto Hk = [&](int row, int cc) { return Hc[(size_t)cc * (m + 1) + row]; };
  if (Hk(col, col).x == 0.0 && Hk(col, col).y == 0.0) s[col] = make_double2(0.0, 0.0);
  for (int i = 0; i <= col; ++i) yc[i] = s[i];
  for (int k = col; k >= 0; --k) {
    if (yc[k].x != 0.0 || yc[k].y != 0.0) {
      const double2 d = Hk(k, k);
      const double den = d.x * d.x + d.y * d.y;
      const double2 q = make_double2((yc[k].x * d.x + yc[k].y * d.y) / den, (yc[k].y * d.x - yc[k].x * d.y) / den);
      yc[k] = q;
      for (int i = 0; i < k; ++i) {
        const double2 hk = Hk(i, k);
        yc[i].x -= q.x * hk.x - q.y * hk.y;
        yc[i].y -= q.x * hk.y + q.y * hk.x;
      }
    }
  }
}

constexpr int kDenseMin = 12;  // columns from which the float64 dense kernel replaces column matvecs

struct BatchWs {
  size_t o_cpl = 0, cpl = 0, o_pnl = 0, pnl = 0, o_dpn = 0, dpn = 0, o_Q = 0, o_W = 0, o_Z = 0, o_R = 0, o_D = 0,
         o_H = 0, o_gc = 0, o_gs = 0, o_S = 0, o_y = 0, o_part = 0, o_vec = 0, o_int = 0, total = 0;
};

static BatchWs batch_layout(const yasf_plan* plan, int N, int R, int m, int inner_kind) {
  BatchWs L;
  auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
  const size_t n = (size_t)N * plan->nmax;
  L.cpl = std::max(coupling_layout(plan, N, YASF_C128).total, coupling_layout(plan, N, YASF_C64).total);
  if (inner_kind == 0) {
    size_t b = 0;
    if (yasf_panel_workspace_size(plan, N, R, &b) == YASF_OK) L.pnl = b;
  }
  // float64 dense multi-column coupling for the float64 applications (lmax <= 6): one pass costs
  // about as much as 10 single-column matvecs at 32 columns, so it is used from kDenseMin columns
  if (R >= kDenseMin && plan->d_dgen_chunks) {
    size_t b = 0;
    if (yasf_dpanel_workspace_size(plan, N, R, &b) == YASF_OK) L.dpn = b;
  }
  size_t o = 0;
  L.o_cpl = o; o += up(L.cpl);
  L.o_pnl = o; o += up(L.pnl);
  L.o_dpn = o; o += up(L.dpn);
  L.o_Q = o; o += up((size_t)R * (m + 1) * n * sizeof(double2));
  L.o_W = o; o += up((size_t)R * n * sizeof(double2));
  L.o_Z = o; o += up((size_t)R * n * sizeof(double2));
  L.o_R = o; o += up((size_t)R * n * sizeof(double2));
  L.o_D = o; o += up((size_t)R * n * sizeof(double2));
  L.o_H = o; o += up((size_t)R * m * (m + 1) * sizeof(double2));
  L.o_gc = o; o += up((size_t)R * m * sizeof(double));
  L.o_gs = o; o += up((size_t)R * m * sizeof(double2));
  L.o_S = o; o += up((size_t)R * (m + 1) * sizeof(double2));
  L.o_y = o; o += up((size_t)R * (m + 1) * sizeof(double2));
  L.o_part = o; o += up((size_t)R * kBDot * (m + 1) * sizeof(double2));
  L.o_vec = o; o += up((size_t)R * 8 * sizeof(double));   // bnorm, beta, h0, h1, presid, rnorm
  L.o_int = o; o += up((size_t)R * 4 * sizeof(int));       // live, brk, stop, active
  L.total = o;
  return L;
}

}  // namespace yasf

using namespace yasf;

extern "C" int yasf_batched_workspace_size(const yasf_plan* plan, int n_particles, int nrhs,
                                           int restart, int inner_kind, size_t* bytes) {
  if (!plan || !bytes || n_particles <= 0 || nrhs <= 0 || restart <= 0 || restart > 512)
    return YASF_ERR_INVALID_ARGUMENT;
  if (inner_kind < 0 || inner_kind > 2) return YASF_ERR_INVALID_ARGUMENT;
  if (inner_kind == 0 && plan->lmax > 8) return YASF_ERR_UNSUPPORTED;
  *bytes = batch_layout(plan, n_particles, nrhs, restart, inner_kind).total;
  return YASF_OK;
}

extern "C" int yasf_batched_solve(const yasf_plan* plan, int n_particles, const double* positions,
                                  double k_medium, const double* tmat, const yasf_precond* pc,
                                  const double* b, double* x, int nrhs, double rtol, int restart,
                                  int max_refine, double inner_rtol, int inner_kind,
                                  void* workspace, size_t workspace_bytes, double* stats,
                                  double* column_residuals, void* stream) {
  int st = validate_coupling(plan, n_particles, positions, k_medium, YASF_C128);
  if (st != YASF_OK) return st;
  if (!tmat || !b || !x || nrhs <= 0 || restart <= 0 || restart > 512 || max_refine < 1 ||
      !(rtol >= 0.0) || !(inner_rtol > 0.0) || inner_kind < 0 || inner_kind > 2)
    return YASF_ERR_INVALID_ARGUMENT;
  if (inner_kind == 0 && plan->lmax > 8) return YASF_ERR_UNSUPPORTED;
  if (!aligned16(tmat) || !aligned16(b) || !aligned16(x) || !aligned16(workspace))
    return YASF_ERR_ALIGNMENT;
  const int R = nrhs;
  const long long n = (long long)n_particles * plan->nmax;
  const int m = (int)std::min<long long>(restart, n);
  const BatchWs L = batch_layout(plan, n_particles, R, m, inner_kind);
  if (!workspace || workspace_bytes < L.total) return YASF_ERR_WORKSPACE;
  char* ws = static_cast<char*>(workspace);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double2* Q = reinterpret_cast<double2*>(ws + L.o_Q);
  double2* W = reinterpret_cast<double2*>(ws + L.o_W);
  double2* Z = reinterpret_cast<double2*>(ws + L.o_Z);
  double2* Rr = reinterpret_cast<double2*>(ws + L.o_R);
  double2* D = reinterpret_cast<double2*>(ws + L.o_D);
  double2* H = reinterpret_cast<double2*>(ws + L.o_H);
  double* gc = reinterpret_cast<double*>(ws + L.o_gc);
  double2* gs = reinterpret_cast<double2*>(ws + L.o_gs);
  double2* S = reinterpret_cast<double2*>(ws + L.o_S);
  double2* yv = reinterpret_cast<double2*>(ws + L.o_y);
  double2* part = reinterpret_cast<double2*>(ws + L.o_part);
  double* vec = reinterpret_cast<double*>(ws + L.o_vec);
  double *d_bnorm = vec, *d_beta = vec + R, *d_h0 = vec + 2 * R, *d_h1 = vec + 3 * R,
         *d_presid = vec + 4 * R, *d_rnorm = vec + 5 * R;
  int* ints = reinterpret_cast<int*>(ws + L.o_int);
  int *d_live = ints, *d_brk = ints + R, *d_stop = ints + 2 * R, *d_active = ints + 3 * R;
  const double2* B = reinterpret_cast<const double2*>(b);
  double2* X = reinterpret_cast<double2*>(x);
  void* cws = ws + L.o_cpl;
  void* pws = ws + L.o_pnl;
  void* dws = ws + L.o_dpn;
  const double eps = 2.220446049250313e-16;
  const dim3 pgrid(256, R);

  std::vector<int> h_live(R), h_active(R), h_stop(R), h_brk(R);
  auto to_host_d = [&](const double* src, double* dst, int count) -> int {
    YASF_CUDA_TRY(cudaMemcpyAsync(dst, src, count * sizeof(double), cudaMemcpyDeviceToHost, s));
    YASF_CUDA_TRY(cudaStreamSynchronize(s));
    return YASF_OK;
  };
  auto to_dev_i = [&](int* dst, const int* src) -> int {
    YASF_CUDA_TRY(cudaMemcpyAsync(dst, src, R * sizeof(int), cudaMemcpyHostToDevice, s));
    return YASF_OK;
  };
  // column norms of a panel (ld = stride) into dst for columns in mask
  auto panel_norm = [&](const double2* V, long long col_stride, double* dst, const int* mask) -> int {
    YASF_COUNTED(bmdot_kernel<<<dim3(kBDot, R), 256, 0, s>>>(n, V, col_stride, 1, V, col_stride, mask, part));
    YASF_COUNTED(bfinal_kernel<<<dim3(1, R), 64, 0, s>>>(1, kBDot, part, nullptr, 0, 0, dst, mask));
    YASF_CUDA_TRY(cudaGetLastError());
    return YASF_OK;
  };
  // A at `prec` on the live columns of V (stride col_stride) into out (ld n)
  long long mv_panel = 0, mv_col = 0, mv64 = 0;
  auto op_inner = [&](const double2* V, long long col_stride, double2* out) -> int {
    if (inner_kind == 0) {
      mv_panel++;
      return yasf_panel_matvec(plan, n_particles, positions, k_medium, tmat,
                               reinterpret_cast<const double*>(V), reinterpret_cast<double*>(out),
                               R, col_stride, n, pws, L.pnl, s);
    }
    const int prec = inner_kind == 1 ? YASF_C64 : YASF_C128;
    if (prec == YASF_C128 && L.dpn) {  // all columns in one float64 dense pass (R >= kDenseMin)
      mv_col += R;
      return yasf_dpanel_matvec(plan, n_particles, positions, k_medium, tmat,
                                reinterpret_cast<const double*>(V), reinterpret_cast<double*>(out), R,
                                col_stride, n, dws, L.dpn, s);
    }
    for (int c = 0; c < R; ++c) {
      if (!h_live[c]) continue;
      mv_col++;
      const int st2 = coupling_column(plan, n_particles, positions, k_medium, tmat,
                                      reinterpret_cast<const double*>(V + (size_t)c * col_stride),
                                      reinterpret_cast<double*>(out + (size_t)c * n), prec, 1, cws,
                                      L.cpl, s);
      if (st2 != YASF_OK) return st2;
    }
    return YASF_OK;
  };
  const int inner_prec = inner_kind == 2 ? YASF_C128 : YASF_C64;
  auto psolve = [&](const double2* V, long long col_stride, double2* out) -> int {
    if (pc) {
      if (col_stride == n)
        return yasf_precond_apply(pc, reinterpret_cast<const double*>(V), reinterpret_cast<double*>(out),
                                  R, n, inner_prec, s);
      // strided input: gather into W first
      YASF_COUNTED(bax_kernel<<<pgrid, 256, 0, s>>>(n, 2, V, nullptr, W, nullptr));
      return yasf_precond_apply(pc, reinterpret_cast<const double*>(W), reinterpret_cast<double*>(out),
                                R, n, inner_prec, s);
    }
    for (int c = 0; c < R; ++c)
      YASF_CUDA_TRY(cudaMemcpyAsync(out + (size_t)c * n, V + (size_t)c * col_stride, n * sizeof(double2),
                                    cudaMemcpyDeviceToDevice, s));
    return YASF_OK;
  };

  // ---- b norms, X = 0, R = B --------------------------------------------------------------
  for (int c = 0; c < R; ++c) h_active[c] = 1;
  if ((st = to_dev_i(d_active, h_active.data())) != YASF_OK) return st;
  if ((st = panel_norm(B, n, d_bnorm, d_active)) != YASF_OK) return st;
  std::vector<double> bnorm(R);
  if ((st = to_host_d(d_bnorm, bnorm.data(), R)) != YASF_OK) return st;
  for (int c = 0; c < R; ++c)
    if (!std::isfinite(bnorm[c])) return YASF_ERR_NOT_FINITE;
  YASF_CUDA_TRY(cudaMemsetAsync(X, 0, (size_t)R * n * sizeof(double2), s));
  YASF_COUNTED(bax_kernel<<<pgrid, 256, 0, s>>>(n, 2, B, nullptr, Rr, nullptr));
  std::vector<double> rnorm(bnorm);
  int refine = 0;
  long long inner_steps = 0;
  for (int c = 0; c < R; ++c) h_active[c] = rnorm[c] > rtol * bnorm[c];
  for (refine = 0; refine < max_refine; ++refine) {
    bool any = false;
    for (int c = 0; c < R; ++c) any |= h_active[c] != 0;
    if (!any) break;
    // ---- inner lockstep GMRES cycle on A~ D = Rr for active columns, D0 = 0 ----------------
    h_live = h_active;
    if ((st = to_dev_i(d_live, h_live.data())) != YASF_OK) return st;
    if ((st = psolve(Rr, n, Z)) != YASF_OK) return st;
    if ((st = panel_norm(Z, n, d_beta, d_live)) != YASF_OK) return st;
    YASF_COUNTED(bscale_kernel<<<pgrid, 256, 0, s>>>(n, Z, n, d_beta, Q, (long long)(m + 1) * n, d_live));
    YASF_COUNTED(bstart_kernel<<<(R + 63) / 64, 64, 0, s>>>(R, m, d_beta, S, d_live));
    YASF_CUDA_TRY(cudaGetLastError());
    std::vector<double> beta(R);
    if ((st = to_host_d(d_beta, beta.data(), R)) != YASF_OK) return st;
    for (int c = 0; c < R; ++c) h_stop[c] = -1;
    int j = 0;
    for (j = 0; j < m; ++j) {
      const long long qs = (long long)(m + 1) * n;
      if ((st = op_inner(Q + (size_t)j * n, qs, W)) != YASF_OK) return st;
      if ((st = psolve(W, n, Z)) != YASF_OK) return st;
      if ((st = panel_norm(Z, n, d_h0, d_live)) != YASF_OK) return st;
      for (int pass = 0; pass < 2; ++pass) {
        YASF_COUNTED(bmdot_kernel<<<dim3(kBDot, R), 256, 0, s>>>(n, Q, qs, j + 1, Z, n, d_live, part));
        double2* hcol = H + (size_t)j * (m + 1);  // column j of each H_c (c stride m*(m+1))
        if (pass == 0) {
          YASF_COUNTED(bfinal_kernel<<<dim3(j + 1, R), 64, 0, s>>>(j + 1, kBDot, part, hcol,
                                                                 (long long)m * (m + 1), 0, nullptr, d_live));
          YASF_COUNTED(bupdate_kernel<<<pgrid, 256, 0, s>>>(n, Q, qs, j + 1, hcol, (long long)m * (m + 1),
                                                          -1.0, Z, n, d_live));
        } else {
          YASF_COUNTED(bfinal_kernel<<<dim3(j + 1, R), 64, 0, s>>>(j + 1, kBDot, part, yv, m + 1, 0,
                                                                 nullptr, d_live));
          YASF_COUNTED(bupdate_kernel<<<pgrid, 256, 0, s>>>(n, Q, qs, j + 1, yv, m + 1, -1.0, Z, n, d_live));
          YASF_COUNTED(bfinal_kernel<<<dim3(j + 1, R), 64, 0, s>>>(j + 1, kBDot, part, hcol,
                                                                 (long long)m * (m + 1), 1, nullptr, d_live));
        }
        YASF_CUDA_TRY(cudaGetLastError());
      }
      if ((st = panel_norm(Z, n, d_h1, d_live)) != YASF_OK) return st;
      YASF_COUNTED(bscale_kernel<<<pgrid, 256, 0, s>>>(n, Z, n, d_h1, Q + (size_t)(j + 1) * n, qs, d_live));
      YASF_COUNTED(bgivens_kernel<<<(R + 63) / 64, 64, 0, s>>>(R, j, m, H, gc, gs, S, d_h0, d_h1,
                                                             d_presid, d_brk, d_live, eps));
      YASF_CUDA_TRY(cudaGetLastError());
      std::vector<double> presid(R);
      if ((st = to_host_d(d_presid, presid.data(), R)) != YASF_OK) return st;
      YASF_CUDA_TRY(cudaMemcpyAsync(h_brk.data(), d_brk, R * sizeof(int), cudaMemcpyDeviceToHost, s));
      YASF_CUDA_TRY(cudaStreamSynchronize(s));
      inner_steps++;
      bool any_live = false;
      for (int c = 0; c < R; ++c) {
        if (!h_live[c]) continue;
        if (!std::isfinite(presid[c])) return YASF_ERR_NOT_FINITE;
        if (presid[c] <= inner_rtol * beta[c] || h_brk[c] || j == m - 1) {
          h_stop[c] = j;
          h_live[c] = 0;
        } else {
          any_live = true;
        }
      }
      if ((st = to_dev_i(d_live, h_live.data())) != YASF_OK) return st;
      if (!any_live) break;
    }
    // ---- D_c = Q_c y_c ; X += D ---------------------------------------------------------------
    if ((st = to_dev_i(d_stop, h_stop.data())) != YASF_OK) return st;
    YASF_COUNTED(bbacksolve_kernel<<<(R + 63) / 64, 64, 0, s>>>(R, m, d_stop, H, S, yv));
    YASF_CUDA_TRY(cudaMemsetAsync(D, 0, (size_t)R * n * sizeof(double2), s));
    std::vector<int> has(R);
    for (int c = 0; c < R; ++c) has[c] = h_stop[c] >= 0;
    if ((st = to_dev_i(d_live, has.data())) != YASF_OK) return st;
    int maxstop = -1;
    for (int c = 0; c < R; ++c) maxstop = std::max(maxstop, h_stop[c]);
    if (maxstop >= 0) {
      // y_c is zero beyond stop[c], so one update with maxstop+1 terms is exact for all columns
      YASF_COUNTED(bupdate_kernel<<<pgrid, 256, 0, s>>>(n, Q, (long long)(m + 1) * n, maxstop + 1, yv,
                                                      m + 1, 1.0, D, n, d_live));
    }
    YASF_COUNTED(bax_kernel<<<pgrid, 256, 0, s>>>(n, 1, D, nullptr, X, d_live));
    YASF_CUDA_TRY(cudaGetLastError());
    // ---- float64 residual of the active columns -------------------------------------------------
    int n_active = 0;
    for (int c = 0; c < R; ++c) n_active += h_active[c] != 0;
    if (L.dpn && n_active >= kDenseMin) {  // every column in one float64 dense pass
      mv64 += R;
      st = yasf_dpanel_matvec(plan, n_particles, positions, k_medium, tmat, reinterpret_cast<const double*>(X),
                              reinterpret_cast<double*>(W), R, n, n, dws, L.dpn, s);
      if (st != YASF_OK) return st;
    } else {
      for (int c = 0; c < R; ++c) {
        if (!h_active[c]) continue;
        mv64++;
        st = coupling_column(plan, n_particles, positions, k_medium, tmat,
                             reinterpret_cast<const double*>(X + (size_t)c * n),
                             reinterpret_cast<double*>(W + (size_t)c * n), YASF_C128, 1, cws, L.cpl, s);
        if (st != YASF_OK) return st;
      }
    }
    if ((st = to_dev_i(d_active, h_active.data())) != YASF_OK) return st;
    YASF_COUNTED(bax_kernel<<<pgrid, 256, 0, s>>>(n, 0, B, W, Rr, d_active));
    if ((st = panel_norm(Rr, n, d_rnorm, d_active)) != YASF_OK) return st;
    std::vector<double> rn(R);
    if ((st = to_host_d(d_rnorm, rn.data(), R)) != YASF_OK) return st;
    for (int c = 0; c < R; ++c) {
      if (!h_active[c]) continue;
      if (!std::isfinite(rn[c])) return YASF_ERR_NOT_FINITE;
      rnorm[c] = rn[c];
      if (rnorm[c] <= rtol * bnorm[c]) h_active[c] = 0;
    }
  }
  double worst = 0.0;
  int unconverged = 0;
  for (int c = 0; c < R; ++c) {
    const double rel = bnorm[c] > 0.0 ? rnorm[c] / bnorm[c] : 0.0;
    worst = std::max(worst, rel);
    unconverged += rnorm[c] > rtol * bnorm[c];
    if (column_residuals) column_residuals[c] = rel;
  }
  if (stats) {
    stats[0] = (double)inner_steps;
    stats[1] = (double)mv_panel;
    stats[2] = (double)mv_col;
    stats[3] = (double)mv64;
    stats[4] = worst;
    stats[5] = (double)unconverged;
    stats[6] = (double)refine;
  }
  YASF_CUDA_TRY(cudaStreamSynchronize(s));
  return YASF_OK;
}

// =============================================================================================
// Grouped solve: the right-hand sides of several aggregates of one lmax (different sphere counts,
// positions, wavenumbers, T) in one lockstep refined GMRES. Column c (one right-hand side of one
// aggregate) has n[c] = N_p nmax unknowns; the solver's vectors are ragged panels (column c at
// offset voff[c], its Krylov basis at qoff[c]). Each operator application is three launches for
// all live columns together: the source-side streams (grouped_vbuild_kernel), the persistent
// work-queue contraction (grouped_contract_kernel) and the reduction with the master epilogue
// (grouped_reduce_kernel). Float64 refinement as in yasf_batched_solve; no preconditioner.
namespace yasf {

namespace {

constexpr int kGroupThreads = 128;   // threads per contraction block
constexpr int kGroupSpc = 64;        // sources per chunk of a grouped column

__device__ __forceinline__ int ragged_find(const long long* pre, int n, long long v) {
  int lo = 0, hi = n;  // pre[lo] <= v < pre[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (pre[mid] <= v) lo = mid; else hi = mid;
  }
  return lo;
}

// partial[c][blk][k] = sum conj(Q_c[k]) w_c over the block's slice (live columns).
__global__ void __launch_bounds__(256) gmdot_kernel(const long long* n, const long long* qoff, int nvec,
                                                    const double2* Q, const double2* w, const long long* woff,
                                                    const int* live, double2* partial) {
  const int c = blockIdx.y;
  if (!live[c]) return;
  __shared__ double sr[8], si[8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const long long nc = n[c];
  const double2* wc = w + woff[c];
  for (int k = 0; k < nvec; ++k) {
    const double2* q = Q + qoff[c] + (size_t)k * nc;
    double re = 0.0, im = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nc; i += (long long)gridDim.x * blockDim.x) {
      const double2 a = q[i], b = wc[i];
      re += a.x * b.x + a.y * b.y;
      im += a.x * b.y - a.y * b.x;
    }
    for (int off = 16; off > 0; off >>= 1) {
      re += __shfl_down_sync(0xffffffffu, re, off);
      im += __shfl_down_sync(0xffffffffu, im, off);
    }
    if (lane == 0) { sr[wid] = re; si[wid] = im; }
    __syncthreads();
    if (threadIdx.x == 0) {
      double tr = 0.0, ti = 0.0;
      for (int t = 0; t < (int)(blockDim.x >> 5); ++t) { tr += sr[t]; ti += si[t]; }
      partial[((size_t)c * gridDim.x + blockIdx.x) * nvec + k] = make_double2(tr, ti);
    }
    __syncthreads();
  }
}

// w_c += sign * sum_k h_c[k] Q_c[k] (live columns; h_c at h + c * h_col).
__global__ void __launch_bounds__(256) gupdate_kernel(const long long* n, const long long* qoff, int nvec,
                                                      const double2* Q, const double2* h, long long h_col,
                                                      double sign, double2* w, const long long* woff,
                                                      const int* live) {
  const int c = blockIdx.y;
  if (!live[c]) return;
  __shared__ double2 sh[512];
  for (int k = threadIdx.x; k < nvec && k < 512; k += blockDim.x) sh[k] = h[(size_t)c * h_col + k];
  __syncthreads();
  const long long nc = n[c];
  double2* wc = w + woff[c];
  const double2* qc = Q + qoff[c];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nc; i += (long long)gridDim.x * blockDim.x) {
    double re = 0.0, im = 0.0;
    for (int k = 0; k < nvec; ++k) {
      const double2 q = qc[(size_t)k * nc + i];
      const double2 cc = sh[k];
      re += cc.x * q.x - cc.y * q.y;
      im += cc.x * q.y + cc.y * q.x;
    }
    double2 v = wc[i];
    v.x += sign * re;
    v.y += sign * im;
    wc[i] = v;
  }
}

// out_c (at out_off[c] + out_j n[c]) = in_c (at in_off[c]) / norm[c] for live columns, else zero.
__global__ void gscale_kernel(const long long* n, const double2* in, const long long* in_off, const double* norm,
                              double2* out, const long long* out_off, long long out_j, const int* live) {
  const int c = blockIdx.y;
  const double nv = norm[c];
  const bool on = live[c] && nv > 0.0;
  const double f = on ? 1.0 / nv : 0.0;
  const long long nc = n[c];
  const double2* ic = in + in_off[c];
  double2* oc = out + out_off[c] + out_j * nc;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nc; i += (long long)gridDim.x * blockDim.x) {
    const double2 v = on ? ic[i] : make_double2(0.0, 0.0);
    oc[i] = make_double2(v.x * f, v.y * f);
  }
}

// Ragged elementwise (columns with mask): mode 0: out = a - b ; 1: out += a ; 2: out = a.
// Column c of a / b / out sits at ptr + off[c] (the same offsets for all three).
__global__ void gax_kernel(const long long* n, const long long* off, int mode, const double2* a, const double2* b,
                           double2* out, const int* mask) {
  const int c = blockIdx.y;
  if (mask && !mask[c]) return;
  const long long nc = n[c];
  const size_t base = off[c];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nc; i += (long long)gridDim.x * blockDim.x) {
    const double2 av = a[base + i];
    if (mode == 0) {
      const double2 bv = b[base + i];
      out[base + i] = make_double2(av.x - bv.x, av.y - bv.y);
    } else if (mode == 1) {
      double2 o = out[base + i];
      o.x += av.x;
      o.y += av.y;
      out[base + i] = o;
    } else {
      out[base + i] = av;
    }
  }
}

// Source-side streams of every live column: V_c[bundle][s][entry] from the column's input x_c at
// in + in_off[c] + in_j n[c] (the stream layout of vbuild_kernel).
struct GroupedVBuildArgs {
  const GroupColumn* cols;
  const int* live;
  const long long* src_pre;   // [n_cols + 1] prefix of the columns' sphere counts
  const long long* in_off;
  const long long* n;
  const double2* in;
  long long in_j;
  int n_cols;
  long long total_src;
  int nmax, total_entries, n_bundles;
  int bundle_begin[8], bundle_len[8];
  const int* entry_ptr;
  const int* term_n2;
  const double2* term_coef;
};

template <typename Real>
__global__ void __launch_bounds__(256) grouped_vbuild_kernel(GroupedVBuildArgs a) {
  using C = typename VEntry<Real>::T;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= a.total_entries) return;
  int b = 0;
  while (b + 1 < a.n_bundles && g >= a.bundle_begin[b + 1]) ++b;
  const int t0 = __ldg(a.entry_ptr + g), t1 = __ldg(a.entry_ptr + g + 1);
  for (long long gs = blockIdx.y; gs < a.total_src; gs += gridDim.y) {
    const int c = ragged_find(a.src_pre, a.n_cols, gs);
    if (!a.live[c]) continue;
    const int s = (int)(gs - a.src_pre[c]);
    const GroupColumn& col = a.cols[c];
    const double2* xs = a.in + a.in_off[c] + a.in_j * a.n[c] + (size_t)s * a.nmax;
    double re = 0.0, im = 0.0;
    for (int t = t0; t < t1; ++t) {
      const double2 cf = __ldg(a.term_coef + t);
      const double2 xv = xs[__ldg(a.term_n2 + t)];
      re = fma(cf.x, xv.x, re);
      re = fma(-cf.y, xv.y, re);
      im = fma(cf.x, xv.y, im);
      im = fma(cf.y, xv.x, im);
    }
    C* out = reinterpret_cast<C*>(const_cast<void*>(col.v)) + (size_t)a.bundle_begin[b] * col.n_particles +
             (size_t)s * a.bundle_len[b] + (g - a.bundle_begin[b]);
    if constexpr (sizeof(Real) == 8) *out = make_double2(re, im);
    else *out = make_float4((float)re, (float)im, -(float)im, (float)re);
  }
}

// out_c = x_c - T_c (.) sum over chunks of the partials (live columns), NaN if a wait ran out.
template <typename Real>
__global__ void __launch_bounds__(256) grouped_reduce_kernel(const GroupColumn* cols, const int* live,
                                                             const long long* elem_pre, int n_cols,
                                                             long long total, int nmax, const double2* in,
                                                             const long long* in_off, const long long* n,
                                                             long long in_j, double2* out,
                                                             const long long* out_off, const int* err) {
  using Cx = typename Cplx<Real>::T;
  const bool bad = *err != 0;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const int c = ragged_find(elem_pre, n_cols, e);
    if (!live[c]) continue;
    const long long i = e - elem_pre[c];
    const GroupColumn& col = cols[c];
    const long long nc = n[c];
    double2 o;
    if (bad) {
      o = make_double2(nan(""), nan(""));
    } else {
      const Cx* pp = reinterpret_cast<const Cx*>(col.partial);
      double re = 0.0, im = 0.0;
      for (int ch = 0; ch < col.chunks; ++ch) {
        const Cx v = pp[(size_t)ch * nc + i];
        re += (double)v.x;
        im += (double)v.y;
      }
      const double2 t = col.tmat[i];
      const double2 xv = in[in_off[c] + in_j * nc + i];
      o = make_double2(xv.x - (t.x * re - t.y * im), xv.y - (t.x * im + t.y * re));
    }
    out[out_off[c] + i] = o;
  }
}

struct GroupWs {
  int C = 0;
  long long sum_n = 0, sum_q = 0, total_src = 0, items[2] = {0, 0};
  size_t o_col64 = 0, o_col32 = 0, o_ipre64 = 0, o_ipre32 = 0, o_spre = 0, o_epre = 0, o_n = 0, o_voff = 0,
         o_qoff = 0;
  size_t o_V = 0, o_P = 0, o_X = 0, o_B = 0, o_W = 0, o_Z = 0, o_R = 0, o_D = 0, o_Q = 0, o_H = 0, o_gc = 0,
         o_gs = 0, o_S = 0, o_y = 0, o_part = 0, o_vec = 0, o_int = 0, o_cnt = 0, total = 0;
  std::vector<long long> n, voff, qoff, src_pre, elem_pre, ipre64, ipre32, vsoff, psoff;
  std::vector<int> prob, chunks, tiles64, tiles32;
};

GroupWs group_layout(const yasf_plan* plan, int P, const yasf_problem* pr, int m) {
  GroupWs L;
  auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
  const int nmax = plan->nmax;
  for (int p = 0; p < P; ++p)
    for (int j = 0; j < pr[p].nrhs; ++j) L.prob.push_back(p);
  const int C = L.C = (int)L.prob.size();
  long long vs = 0, ps = 0;
  L.src_pre.push_back(0);
  L.elem_pre.push_back(0);
  L.ipre64.push_back(0);
  L.ipre32.push_back(0);
  for (int c = 0; c < C; ++c) {
    const int N = pr[L.prob[c]].n_particles;
    const long long nc = (long long)N * nmax;
    L.n.push_back(nc);
    L.voff.push_back(L.sum_n);
    L.qoff.push_back(L.sum_q);
    L.sum_n += nc;
    L.sum_q += (long long)(m + 1) * nc;
    const int spc = std::min(N, kGroupSpc);
    const int ch = (N + spc - 1) / spc;
    L.chunks.push_back(ch);
    L.tiles64.push_back((N + kGroupThreads - 1) / kGroupThreads);
    L.tiles32.push_back((N + kC64Receivers * kGroupThreads - 1) / (kC64Receivers * kGroupThreads));
    L.src_pre.push_back(L.src_pre.back() + N);
    L.elem_pre.push_back(L.elem_pre.back() + nc);
    L.ipre64.push_back(L.ipre64.back() + (long long)L.tiles64.back() * ch * plan->stream[0].n_bundles);
    L.ipre32.push_back(L.ipre32.back() + (long long)L.tiles32.back() * ch * plan->stream[1].n_bundles);
    L.vsoff.push_back(vs);
    L.psoff.push_back(ps);
    vs += up((size_t)N * std::max(plan->stream[0].total_entries, plan->stream[1].total_entries) * 16);
    ps += up((size_t)ch * nc * 16);
  }
  L.total_src = L.src_pre.back();
  L.items[0] = L.ipre64.back();
  L.items[1] = L.ipre32.back();
  size_t o = 0;
  const size_t cz = std::max(C, 1);
  L.o_col64 = o; o += up(cz * sizeof(GroupColumn));
  L.o_col32 = o; o += up(cz * sizeof(GroupColumn));
  L.o_ipre64 = o; o += up((cz + 1) * 8);
  L.o_ipre32 = o; o += up((cz + 1) * 8);
  L.o_spre = o; o += up((cz + 1) * 8);
  L.o_epre = o; o += up((cz + 1) * 8);
  L.o_n = o; o += up(cz * 8);
  L.o_voff = o; o += up(cz * 8);
  L.o_qoff = o; o += up(cz * 8);
  L.o_V = o; o += (size_t)vs;
  L.o_P = o; o += (size_t)ps;
  const size_t vb = up((size_t)L.sum_n * 16);
  L.o_X = o; o += vb;
  L.o_B = o; o += vb;
  L.o_W = o; o += vb;
  L.o_Z = o; o += vb;
  L.o_R = o; o += vb;
  L.o_D = o; o += vb;
  L.o_Q = o; o += up((size_t)L.sum_q * 16);
  L.o_H = o; o += up(cz * m * (m + 1) * 16);
  L.o_gc = o; o += up(cz * m * 8);
  L.o_gs = o; o += up(cz * m * 16);
  L.o_S = o; o += up(cz * (m + 1) * 16);
  L.o_y = o; o += up(cz * (m + 1) * 16);
  L.o_part = o; o += up(cz * kBDot * (m + 1) * 16);
  L.o_vec = o; o += up(cz * 8 * 8);
  L.o_int = o; o += up(cz * 4 * 4);
  L.o_cnt = o; o += 256;  // work-queue counter and error word
  L.total = o;
  return L;
}

int group_check(const yasf_plan* plan, int P, const yasf_problem* pr) {
  if (!plan || P <= 0 || !pr) return YASF_ERR_INVALID_ARGUMENT;
  for (int p = 0; p < P; ++p) {
    const yasf_problem& q = pr[p];
    int st = validate_coupling(plan, q.n_particles, q.positions, q.k_medium, YASF_C128);
    if (st != YASF_OK) return st;
    if (q.nrhs <= 0 || !q.tmat || !q.b || !q.x) return YASF_ERR_INVALID_ARGUMENT;
    if (!aligned16(q.tmat) || !aligned16(q.b) || !aligned16(q.x)) return YASF_ERR_ALIGNMENT;
  }
  return YASF_OK;
}

}  // namespace

int dispatch_grouped_contract(int lmax, int precision, const GroupedContractArgs& g, int blocks, cudaStream_t s) {
  cudaError_t e = cudaErrorInvalidValue;
  switch (lmax) {
    case 1: e = launch_grouped_contract<1>(precision, g, blocks, s); break;
    case 2: e = launch_grouped_contract<2>(precision, g, blocks, s); break;
    case 3: e = launch_grouped_contract<3>(precision, g, blocks, s); break;
    case 4: e = launch_grouped_contract<4>(precision, g, blocks, s); break;
    case 5: e = launch_grouped_contract<5>(precision, g, blocks, s); break;
    case 6: e = launch_grouped_contract<6>(precision, g, blocks, s); break;
    case 7: e = launch_grouped_contract<7>(precision, g, blocks, s); break;
    case 8: e = launch_grouped_contract<8>(precision, g, blocks, s); break;
    default: return YASF_ERR_UNSUPPORTED;
  }
  YASF_CUDA_TRY(e);
  return YASF_OK;
}

}  // namespace yasf

extern "C" int yasf_grouped_workspace_size(const yasf_plan* plan, int n_problems, const yasf_problem* problems,
                                           int restart, size_t* bytes) {
  if (!bytes || restart <= 0 || restart > 512) return YASF_ERR_INVALID_ARGUMENT;
  // the size depends only on the counts: a caller may size a group before its buffers exist
  if (!plan || n_problems <= 0 || !problems) return YASF_ERR_INVALID_ARGUMENT;
  for (int p = 0; p < n_problems; ++p)
    if (problems[p].n_particles <= 0 || problems[p].nrhs <= 0) return YASF_ERR_INVALID_ARGUMENT;
  *bytes = group_layout(plan, n_problems, problems, restart).total;
  return YASF_OK;
}

extern "C" int yasf_grouped_solve(const yasf_plan* plan, int n_problems, const yasf_problem* problems,
                                  double rtol, int restart, int max_refine, double inner_rtol, int inner_precision,
                                  void* workspace, size_t workspace_bytes, double* stats, double* column_residuals,
                                  void* stream) {
  if (int st = group_check(plan, n_problems, problems)) return st;
  if (restart <= 0 || restart > 512 || max_refine < 1 || !(rtol >= 0.0) || !(inner_rtol > 0.0) ||
      (inner_precision != YASF_C64 && inner_precision != YASF_C128))
    return YASF_ERR_INVALID_ARGUMENT;
  const int m = restart;
  const GroupWs L = group_layout(plan, n_problems, problems, m);
  if (!workspace || workspace_bytes < L.total) return YASF_ERR_WORKSPACE;
  if (!aligned16(workspace)) return YASF_ERR_ALIGNMENT;
  const int C = L.C;
  const int nmax = plan->nmax;
  char* ws = static_cast<char*>(workspace);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  auto dv = [&](size_t o) { return reinterpret_cast<double2*>(ws + o); };
  const long long* d_n = reinterpret_cast<const long long*>(ws + L.o_n);
  const long long* d_voff = reinterpret_cast<const long long*>(ws + L.o_voff);
  const long long* d_qoff = reinterpret_cast<const long long*>(ws + L.o_qoff);
  double2 *X = dv(L.o_X), *Bp = dv(L.o_B), *W = dv(L.o_W), *Z = dv(L.o_Z), *Rr = dv(L.o_R), *D = dv(L.o_D),
          *Q = dv(L.o_Q), *H = dv(L.o_H), *gs = dv(L.o_gs), *S = dv(L.o_S), *yv = dv(L.o_y), *part = dv(L.o_part);
  double* gc = reinterpret_cast<double*>(ws + L.o_gc);
  double* vec = reinterpret_cast<double*>(ws + L.o_vec);
  double *d_bnorm = vec, *d_beta = vec + C, *d_h0 = vec + 2 * C, *d_h1 = vec + 3 * C, *d_presid = vec + 4 * C,
         *d_rnorm = vec + 5 * C;
  int* ints = reinterpret_cast<int*>(ws + L.o_int);
  int *d_live = ints, *d_brk = ints + C, *d_stop = ints + 2 * C, *d_active = ints + 3 * C;
  unsigned long long* d_counter = reinterpret_cast<unsigned long long*>(ws + L.o_cnt);
  int* d_err = reinterpret_cast<int*>(ws + L.o_cnt + 8);

  // ---- tables: columns (per precision: tiles differ), prefixes, lengths, offsets ---------------
  {
    std::vector<GroupColumn> c64(C), c32(C);
    for (int c = 0; c < C; ++c) {
      const yasf_problem& q = problems[L.prob[c]];
      GroupColumn g{};
      g.pos = q.positions;
      g.tmat = reinterpret_cast<const double2*>(q.tmat);
      g.v = ws + L.o_V + L.vsoff[c];
      g.partial = ws + L.o_P + L.psoff[c];
      g.k = q.k_medium;
      g.n_particles = q.n_particles;
      g.chunks = L.chunks[c];
      g.sources_per_chunk = std::min(q.n_particles, kGroupSpc);
      g.tiles = L.tiles64[c];
      c64[c] = g;
      g.tiles = L.tiles32[c];
      c32[c] = g;
    }
    auto put = [&](size_t off, const void* src, size_t bytes) -> int {
      YASF_CUDA_TRY(cudaMemcpyAsync(ws + off, src, bytes, cudaMemcpyHostToDevice, s));
      return YASF_OK;
    };
    int st = YASF_OK;
    if ((st = put(L.o_col64, c64.data(), C * sizeof(GroupColumn))) ||
        (st = put(L.o_col32, c32.data(), C * sizeof(GroupColumn))) ||
        (st = put(L.o_ipre64, L.ipre64.data(), (C + 1) * 8)) || (st = put(L.o_ipre32, L.ipre32.data(), (C + 1) * 8)) ||
        (st = put(L.o_spre, L.src_pre.data(), (C + 1) * 8)) || (st = put(L.o_epre, L.elem_pre.data(), (C + 1) * 8)) ||
        (st = put(L.o_n, L.n.data(), C * 8)) || (st = put(L.o_voff, L.voff.data(), C * 8)) ||
        (st = put(L.o_qoff, L.qoff.data(), C * 8)))
      return st;
    // the caller's right-hand sides into the packed panel
    for (int c = 0, first = 0; c < C; ++c) {
      const yasf_problem& q = problems[L.prob[c]];
      if (c > 0 && L.prob[c] != L.prob[c - 1]) first = c;
      const double* src = q.b + 2 * (size_t)(c - first) * L.n[c];
      YASF_CUDA_TRY(cudaMemcpyAsync(Bp + L.voff[c], src, L.n[c] * 16, cudaMemcpyDeviceToDevice, s));
    }
  }
  YASF_CUDA_TRY(cudaMemsetAsync(d_err, 0, sizeof(int), s));
  int sms = 148;
  {
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  }
  // operator application A at `prec` on the live columns: in_c at in + in_off[c] + in_j n[c],
  // out_c at out + voff[c]
  long long mv_inner = 0, mv64 = 0;
  auto apply = [&](int prec, const double2* in, const long long* in_off, long long in_j, double2* out,
                   const int* live) -> int {
    GroupedVBuildArgs va{};
    va.cols = reinterpret_cast<const GroupColumn*>(ws + (prec == YASF_C64 ? L.o_col32 : L.o_col64));
    va.live = live;
    va.src_pre = reinterpret_cast<const long long*>(ws + L.o_spre);
    va.in_off = in_off;
    va.n = d_n;
    va.in = in;
    va.in_j = in_j;
    va.n_cols = C;
    va.total_src = L.total_src;
    va.nmax = nmax;
    const yasf_stream_layout& sl = plan->layout(prec);
    va.total_entries = sl.total_entries;
    va.n_bundles = sl.n_bundles;
    for (int b = 0; b < 8; ++b) {
      va.bundle_begin[b] = sl.bundle_begin[b];
      va.bundle_len[b] = sl.bundle_len[b];
    }
    va.entry_ptr = sl.d_entry_ptr;
    va.term_n2 = sl.d_term_n2;
    va.term_coef = sl.d_term_coef;
    const dim3 vgrid((sl.total_entries + 255) / 256, (unsigned)std::min<long long>(L.total_src, 65535));
    if (prec == YASF_C64) YASF_COUNTED(grouped_vbuild_kernel<float><<<vgrid, 256, 0, s>>>(va));
    else YASF_COUNTED(grouped_vbuild_kernel<double><<<vgrid, 256, 0, s>>>(va));
    YASF_CUDA_TRY(cudaGetLastError());
    GroupedContractArgs ga{};
    ga.cols = va.cols;
    ga.live = live;
    ga.item_pre = reinterpret_cast<const long long*>(ws + (prec == YASF_C64 ? L.o_ipre32 : L.o_ipre64));
    ga.n_cols = C;
    ga.total_items = L.items[prec == YASF_C64 ? 1 : 0];
    ga.counter = d_counter;
    ga.leg = plan->d_leg;
    ga.nmax = nmax;
    ga.n_bundles = sl.n_bundles;
    for (int b = 0; b < 8; ++b) {
      ga.bundle_begin[b] = sl.bundle_begin[b];
      ga.bundle_len[b] = sl.bundle_len[b];
    }
    ga.err = d_err;
    ga.poll_limit = stall_hook().contract_polls;
    ga.stall = stall_hook().role == YASF_STALL_CONTRACT ? 1 : 0;
    YASF_CUDA_TRY(cudaMemsetAsync(d_counter, 0, sizeof(unsigned long long), s));
    const int resident = std::max(1, resident_blocks(plan->lmax, prec, kGroupThreads));
    const int blocks = (int)std::min<long long>(ga.total_items, (long long)resident * sms);
    if (int st = dispatch_grouped_contract(plan->lmax, prec, ga, std::max(1, blocks), s)) return st;
    const int rblocks = (int)std::min<long long>((L.sum_n + 255) / 256, 8192);
    if (prec == YASF_C64)
      YASF_COUNTED(grouped_reduce_kernel<float><<<rblocks, 256, 0, s>>>(
          va.cols, live, reinterpret_cast<const long long*>(ws + L.o_epre), C, L.sum_n, nmax, in, in_off, d_n,
          in_j, out, d_voff, d_err));
    else
      YASF_COUNTED(grouped_reduce_kernel<double><<<rblocks, 256, 0, s>>>(
          va.cols, live, reinterpret_cast<const long long*>(ws + L.o_epre), C, L.sum_n, nmax, in, in_off, d_n,
          in_j, out, d_voff, d_err));
    YASF_CUDA_TRY(cudaGetLastError());
    return YASF_OK;
  };
  const dim3 pgrid(256, C);
  std::vector<int> h_live(C), h_active(C), h_stop(C), h_brk(C);
  auto to_host_d = [&](const double* src, double* dst, int count) -> int {
    YASF_CUDA_TRY(cudaMemcpyAsync(dst, src, count * sizeof(double), cudaMemcpyDeviceToHost, s));
    YASF_CUDA_TRY(cudaStreamSynchronize(s));
    return YASF_OK;
  };
  auto to_dev_i = [&](int* dst, const int* src) -> int {
    YASF_CUDA_TRY(cudaMemcpyAsync(dst, src, C * sizeof(int), cudaMemcpyHostToDevice, s));
    return YASF_OK;
  };
  auto norms = [&](const double2* V, const long long* off, double* dst, const int* mask) -> int {
    YASF_COUNTED(gmdot_kernel<<<dim3(kBDot, C), 256, 0, s>>>(d_n, off, 1, V, V, off, mask, part));
    YASF_COUNTED(bfinal_kernel<<<dim3(1, C), 64, 0, s>>>(1, kBDot, part, nullptr, 0, 0, dst, mask));
    YASF_CUDA_TRY(cudaGetLastError());
    return YASF_OK;
  };
  const double eps = 2.220446049250313e-16;
  int st = YASF_OK;
  for (int c = 0; c < C; ++c) h_active[c] = 1;
  if ((st = to_dev_i(d_active, h_active.data()))) return st;
  if ((st = norms(Bp, d_voff, d_bnorm, d_active))) return st;
  std::vector<double> bnorm(C);
  if ((st = to_host_d(d_bnorm, bnorm.data(), C))) return st;
  for (int c = 0; c < C; ++c)
    if (!std::isfinite(bnorm[c])) return YASF_ERR_NOT_FINITE;
  YASF_CUDA_TRY(cudaMemsetAsync(X, 0, (size_t)L.sum_n * 16, s));
  YASF_COUNTED(gax_kernel<<<pgrid, 256, 0, s>>>(d_n, d_voff, 2, Bp, nullptr, Rr, nullptr));
  std::vector<double> rnorm(bnorm);
  int refine = 0;
  long long inner_steps = 0;
  for (int c = 0; c < C; ++c) h_active[c] = rnorm[c] > rtol * bnorm[c];
  for (refine = 0; refine < max_refine; ++refine) {
    bool any = false;
    for (int c = 0; c < C; ++c) any |= h_active[c] != 0;
    if (!any) break;
    h_live = h_active;
    if ((st = to_dev_i(d_live, h_live.data()))) return st;
    if ((st = norms(Rr, d_voff, d_beta, d_live))) return st;
    YASF_COUNTED(gscale_kernel<<<pgrid, 256, 0, s>>>(d_n, Rr, d_voff, d_beta, Q, d_qoff, 0, d_live));
    YASF_COUNTED(bstart_kernel<<<(C + 63) / 64, 64, 0, s>>>(C, m, d_beta, S, d_live));
    YASF_CUDA_TRY(cudaGetLastError());
    std::vector<double> beta(C);
    if ((st = to_host_d(d_beta, beta.data(), C))) return st;
    for (int c = 0; c < C; ++c) h_stop[c] = -1;
    for (int j = 0; j < m; ++j) {
      if ((st = apply(inner_precision, Q, d_qoff, j, W, d_live))) return st;
      ++mv_inner;
      if ((st = norms(W, d_voff, d_h0, d_live))) return st;
      double2* hcol = H + (size_t)j * (m + 1);
      for (int pass = 0; pass < 2; ++pass) {
        YASF_COUNTED(gmdot_kernel<<<dim3(kBDot, C), 256, 0, s>>>(d_n, d_qoff, j + 1, Q, W, d_voff, d_live, part));
        if (pass == 0) {
          YASF_COUNTED(bfinal_kernel<<<dim3(j + 1, C), 64, 0, s>>>(j + 1, kBDot, part, hcol, (long long)m * (m + 1), 0,
                                                                 nullptr, d_live));
          YASF_COUNTED(gupdate_kernel<<<pgrid, 256, 0, s>>>(d_n, d_qoff, j + 1, Q, hcol, (long long)m * (m + 1), -1.0,
                                                          W, d_voff, d_live));
        } else {
          YASF_COUNTED(bfinal_kernel<<<dim3(j + 1, C), 64, 0, s>>>(j + 1, kBDot, part, yv, m + 1, 0, nullptr, d_live));
          YASF_COUNTED(gupdate_kernel<<<pgrid, 256, 0, s>>>(d_n, d_qoff, j + 1, Q, yv, m + 1, -1.0, W, d_voff, d_live));
          YASF_COUNTED(bfinal_kernel<<<dim3(j + 1, C), 64, 0, s>>>(j + 1, kBDot, part, hcol, (long long)m * (m + 1), 1,
                                                                 nullptr, d_live));
        }
        YASF_CUDA_TRY(cudaGetLastError());
      }
      if ((st = norms(W, d_voff, d_h1, d_live))) return st;
      YASF_COUNTED(gscale_kernel<<<pgrid, 256, 0, s>>>(d_n, W, d_voff, d_h1, Q, d_qoff, j + 1, d_live));
      YASF_COUNTED(bgivens_kernel<<<(C + 63) / 64, 64, 0, s>>>(C, j, m, H, gc, gs, S, d_h0, d_h1, d_presid, d_brk,
                                                             d_live, eps));
      YASF_CUDA_TRY(cudaGetLastError());
      std::vector<double> presid(C);
      if ((st = to_host_d(d_presid, presid.data(), C))) return st;
      YASF_CUDA_TRY(cudaMemcpyAsync(h_brk.data(), d_brk, C * sizeof(int), cudaMemcpyDeviceToHost, s));
      YASF_CUDA_TRY(cudaStreamSynchronize(s));
      inner_steps++;
      bool any_live = false;
      for (int c = 0; c < C; ++c) {
        if (!h_live[c]) continue;
        if (!std::isfinite(presid[c])) return YASF_ERR_NOT_FINITE;
        if (presid[c] <= inner_rtol * beta[c] || h_brk[c] || j == m - 1) {
          h_stop[c] = j;
          h_live[c] = 0;
        } else {
          any_live = true;
        }
      }
      if ((st = to_dev_i(d_live, h_live.data()))) return st;
      if (!any_live) break;
    }
    // ---- D_c = Q_c y_c ; X += D ------------------------------------------------------------------
    if ((st = to_dev_i(d_stop, h_stop.data()))) return st;
    YASF_COUNTED(bbacksolve_kernel<<<(C + 63) / 64, 64, 0, s>>>(C, m, d_stop, H, S, yv));
    YASF_CUDA_TRY(cudaMemsetAsync(D, 0, (size_t)L.sum_n * 16, s));
    std::vector<int> has(C);
    int maxstop = -1;
    for (int c = 0; c < C; ++c) {
      has[c] = h_stop[c] >= 0;
      maxstop = std::max(maxstop, h_stop[c]);
    }
    if ((st = to_dev_i(d_live, has.data()))) return st;
    if (maxstop >= 0)
      YASF_COUNTED(gupdate_kernel<<<pgrid, 256, 0, s>>>(d_n, d_qoff, maxstop + 1, Q, yv, m + 1, 1.0, D, d_voff, d_live));
    YASF_COUNTED(gax_kernel<<<pgrid, 256, 0, s>>>(d_n, d_voff, 1, D, nullptr, X, d_live));
    YASF_CUDA_TRY(cudaGetLastError());
    // ---- float64 residual of the active columns ----------------------------------------------
    if ((st = to_dev_i(d_active, h_active.data()))) return st;
    if ((st = apply(YASF_C128, X, d_voff, 0, W, d_active))) return st;
    ++mv64;
    YASF_COUNTED(gax_kernel<<<pgrid, 256, 0, s>>>(d_n, d_voff, 0, Bp, W, Rr, d_active));
    if ((st = norms(Rr, d_voff, d_rnorm, d_active))) return st;
    std::vector<double> rn(C);
    if ((st = to_host_d(d_rnorm, rn.data(), C))) return st;
    for (int c = 0; c < C; ++c) {
      if (!h_active[c]) continue;
      if (!std::isfinite(rn[c])) return YASF_ERR_NOT_FINITE;
      rnorm[c] = rn[c];
      if (rnorm[c] <= rtol * bnorm[c]) h_active[c] = 0;
    }
  }
  // solutions back into the caller's columns
  for (int c = 0, first = 0; c < C; ++c) {
    const yasf_problem& q = problems[L.prob[c]];
    if (c > 0 && L.prob[c] != L.prob[c - 1]) first = c;
    YASF_CUDA_TRY(cudaMemcpyAsync(q.x + 2 * (size_t)(c - first) * L.n[c], X + L.voff[c], L.n[c] * 16,
                                  cudaMemcpyDeviceToDevice, s));
  }
  double worst = 0.0;
  int unconverged = 0;
  for (int c = 0; c < C; ++c) {
    const double rel = bnorm[c] > 0.0 ? rnorm[c] / bnorm[c] : 0.0;
    worst = std::max(worst, rel);
    unconverged += rnorm[c] > rtol * bnorm[c];
    if (column_residuals) column_residuals[c] = rel;
  }
  if (stats) {
    stats[0] = (double)inner_steps;
    stats[1] = (double)mv_inner;
    stats[2] = (double)mv64;
    stats[3] = worst;
    stats[4] = (double)unconverged;
    stats[5] = (double)refine;
    stats[6] = (double)C;
    stats[7] = (double)L.items[inner_precision == YASF_C64 ? 1 : 0];
  }
  YASF_CUDA_TRY(cudaStreamSynchronize(s));
  return YASF_OK;
}
