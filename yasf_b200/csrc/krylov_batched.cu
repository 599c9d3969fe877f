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
