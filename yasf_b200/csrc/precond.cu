// Block-Jacobi preconditioner for M = I - T W (yasfpy/preconditioner.py:58-219, re-designed).
//
// The reference assembles each spatial block with Python loops that fail for blocks holding two
// or more spheres (yasfpy/preconditioner.py:408-423), gathers with a coefficient-major map
// (yasfpy/preconditioner.py:138) while the unknown vector is particle-major, and applies LU
// factors with per-block Python triangular solves (yasfpy/preconditioner.py:177-219, 470-519).
// Here every block M_B = (I - T W)[B, B] is assembled on the device in particle-major order from
// the same pair generator as the matvec (receiver Mie factor, pair vector pos[s1] - pos[s2]),
// inverted once (the caller factorises it in place between assemble and finalize), and applied
// as a gather / dense GEMV / scatter that streams the inverse once per application.
#include <atomic>
#include <cmath>
#include <new>

#include "blocklu.cuh"
#include "capi_internal.h"

struct yasf_precond {
  const yasf_plan* plan = nullptr;
  int n_particles = 0;
  int n_blocks = 0;
  int total_rows = 0;
  std::vector<int> block_ptr;
  std::vector<long long> mat_off;
  int* d_block_ptr = nullptr;
  int* d_particles = nullptr;
  int* d_particle_block = nullptr;  // block of each particle
  int* d_particle_local = nullptr;  // position of each particle inside its block
  long long* d_mat_off = nullptr;
  int* d_row_block = nullptr;       // block of each flattened row
  int* d_row_local = nullptr;       // local row index
  double2* d_mat = nullptr;
  float2* d_mat32 = nullptr;
  size_t mat_elems = 0;
  bool assembled = false;
  bool prepared = false;
  // batched LU (yasf_precond_factor): per-block geometry, per-step work prefix sums, pivots, the
  // complex64 factors' diagonal-tile inverses (and complex128 ones when the float64 factors are
  // kept), the sweep buffer of the apply
  bool factored = false;   // blocks hold LU factors (else: the caller's inverses)
  bool keep_f64 = false;   // factor in complex128 and keep those factors (yasf_precond_keep_float64)
  bool factored_c64 = false;  // the factorisation ran in complex64 (d_mat32, complex128 released)
  int lu_steps = 0;        // tiles of the largest block
  int n_tiles = 0;         // diagonal tiles of all blocks
  std::vector<int> pre_diag, pre_panel, pre_update, pre_sweep;  // [step][n_blocks + 1]
  int* d_dim = nullptr;
  int* d_row0 = nullptr;
  int* d_tile0 = nullptr;
  int* d_pre = nullptr;    // the four prefix tables, one after the other
  int* d_piv = nullptr;
  int* d_err = nullptr;
  float2* d_dinv = nullptr;
  double2* d_dinv64 = nullptr;
  double2* d_z = nullptr;
  int z_cols = 0;
  // one-column applies: ticket order of the tile rows (forward sweep, then backward) and the
  // ticket / abort / finished-row words of the single-launch solve
  int2* d_order = nullptr;
  int* d_sync = nullptr;
  // the sweep launches of an apply, captured once per (columns, factor precision) as a CUDA graph
  // on a private stream and replayed on the caller's stream
  struct SweepGraph {
    int nrhs;
    bool f64;
    int launches;
    cudaGraphExec_t exec;
  };
  std::vector<SweepGraph> graphs;
  cudaStream_t capture_stream = nullptr;
};

namespace yasf {

constexpr int kAsmChunk = 8;  // source particles whose pair tables sit in shared memory at once

// Pair table Gt[p][delta + 2L] = Pn_p^{|delta|}(cos theta) h_p(kr) e^{i delta phi}, p <= 2L.
__device__ void pair_table(double dx, double dy, double dz, double k, int L,
                           const LegendreTables* leg, double2* Gt) {
  const int PM = 2 * L;
  const int W = 4 * L + 1;
  const double r = sqrt(dx * dx + dy * dy + dz * dz);
  double ct = dz / r;
  ct = fmin(1.0, fmax(-1.0, ct));
  const double st = sqrt(1.0 - ct * ct);
  const double rho = sqrt(dx * dx + dy * dy);
  const double er = (rho > 0.0) ? dx / rho : 1.0;
  const double ei = (rho > 0.0) ? dy / rho : 0.0;
  const double x = k * r;
  double h_r[YASF_PMAX_MAX + 2], h_i[YASF_PMAX_MAX + 2];
  double sx, cx;
  sincos(x, &sx, &cx);
  const double ix = 1.0 / x;
  h_r[0] = sx * ix;
  h_i[0] = -cx * ix;
  h_r[1] = (sx - x * cx) * ix * ix;
  h_i[1] = -(cx + x * sx) * ix * ix;
  for (int p = 1; p < PM; ++p) {
    const double f = (2 * p + 1) * ix;
    h_r[p + 1] = f * h_r[p] - h_r[p - 1];
    h_i[p + 1] = f * h_i[p] - h_i[p - 1];
  }
  double st_d = 1.0, ph_r = 1.0, ph_i = 0.0;
  for (int d = 0; d <= PM; ++d) {
    if (d > 0) {
      st_d *= st;
      const double t = ph_r * er - ph_i * ei;
      ph_i = ph_r * ei + ph_i * er;
      ph_r = t;
    }
    double Pp = 0.0, Pc = leg->start[d] * st_d;
    for (int p = d; p <= PM; ++p) {
      const double gr = Pc * h_r[p], gi = Pc * h_i[p];
      Gt[p * W + (d + 2 * L)] = make_double2(gr * ph_r - gi * ph_i, gr * ph_i + gi * ph_r);
      Gt[p * W + (-d + 2 * L)] = make_double2(gr * ph_r + gi * ph_i, gi * ph_r - gr * ph_i);
      if (p < PM) {
        const double Pn = leg->alpha[p * kLegStride + d] * ct * Pc - leg->beta[p * kLegStride + d] * Pp;
        Pp = Pc;
        Pc = Pn;
      }
    }
  }
}

struct AsmArgs {
  int L, nmax;
  double k;
  const double* pos;
  const double2* tmat;
  const int* block_ptr;
  const int* particles;
  const int* particle_block;
  const int* particle_local;
  const long long* mat_off;
  const int* pair_ptr;
  const int* pair_p;
  const double2* pair_coef;
  const LegendreTables* leg;
  double2* mat;
};

// One block per receiving particle: writes its nmax rows of its block matrix.
__global__ void __launch_bounds__(256) assemble_kernel(AsmArgs a) {
  extern __shared__ double2 sGt[];  // kAsmChunk * (2L+1) * (4L+1)
  const int s1 = blockIdx.x;
  const int blk = a.particle_block[s1];
  const int li = a.particle_local[s1];
  const int p0 = a.block_ptr[blk], p1 = a.block_ptr[blk + 1];
  const int nb = p1 - p0;
  const int dim = nb * a.nmax;
  double2* M = a.mat + a.mat_off[blk];
  const int W = 4 * a.L + 1, TS = (2 * a.L + 1) * W;
  const int nn = a.nmax * a.nmax;
  for (int j0 = 0; j0 < nb; j0 += kAsmChunk) {
    const int jc = min(kAsmChunk, nb - j0);
    __syncthreads();
    if (threadIdx.x < jc) {
      const int s2 = a.particles[p0 + j0 + threadIdx.x];
      if (s2 != s1) {
        pair_table(a.pos[3 * s1] - a.pos[3 * s2], a.pos[3 * s1 + 1] - a.pos[3 * s2 + 1],
                   a.pos[3 * s1 + 2] - a.pos[3 * s2 + 2], a.k, a.L, a.leg,
                   sGt + threadIdx.x * TS);
      }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nn; e += blockDim.x) {
      const int n1 = e / a.nmax, n2 = e % a.nmax;
      // m of a mode index: n = (tau-1)L(L+2) + l^2 + l + m - 1
      int q1 = n1 % (a.L * (a.L + 2)), q2 = n2 % (a.L * (a.L + 2));
      int l1 = (int)floor(sqrt((double)q1 + 1.0)), l2 = (int)floor(sqrt((double)q2 + 1.0));
      const int m1 = q1 + 1 - l1 * l1 - l1, m2 = q2 + 1 - l2 * l2 - l2;
      const int col_d = m2 - m1 + 2 * a.L;
      double accr[kAsmChunk], acci[kAsmChunk];
#pragma unroll
      for (int j = 0; j < kAsmChunk; ++j) { accr[j] = 0.0; acci[j] = 0.0; }
      const int t0 = a.pair_ptr[n1 * a.nmax + n2], t1 = a.pair_ptr[n1 * a.nmax + n2 + 1];
      for (int t = t0; t < t1; ++t) {
        const double2 c = a.pair_coef[t];
        const int off = a.pair_p[t] * W + col_d;
#pragma unroll
        for (int j = 0; j < kAsmChunk; ++j) {
          if (j < jc) {
            const double2 g = sGt[j * TS + off];
            accr[j] += c.x * g.x - c.y * g.y;
            acci[j] += c.x * g.y + c.y * g.x;
          }
        }
      }
      const double2 t = a.tmat[(size_t)s1 * a.nmax + n1];
      for (int j = 0; j < jc; ++j) {
        const int jj = j0 + j;
        const int s2 = a.particles[p0 + jj];
        double2 val;
        if (s2 == s1) {
          val = make_double2(n1 == n2 ? 1.0 : 0.0, 0.0);
        } else {
          val = make_double2(-(t.x * accr[j] - t.y * acci[j]), -(t.x * acci[j] + t.y * accr[j]));
        }
        M[(size_t)(li * a.nmax + n1) * dim + (size_t)jj * a.nmax + n2] = val;
      }
    }
  }
}

__global__ void to_c64_kernel(size_t n, const double2* in, float2* out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = make_float2((float)in[i].x, (float)in[i].y);
}

// y[rows of block] = Minv_B x[rows of block]; one warp per flattened row. The row of the inverse
// is streamed once per group of CPP columns (CPP = 16 when several right-hand sides are applied).
template <typename MT, int CPP>
__global__ void __launch_bounds__(256) apply_kernel(int total_rows, int nmax, int nrhs, long long ld,
                                                    const int* row_block, const int* row_local,
                                                    const int* block_ptr, const int* particles,
                                                    const long long* mat_off, const MT* mat,
                                                    const double2* x, double2* y) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= total_rows) return;
  const int b = row_block[warp];
  const int i = row_local[warp];
  const int p0 = block_ptr[b];
  const int dim = (block_ptr[b + 1] - p0) * nmax;
  const MT* row = mat + mat_off[b] + (size_t)i * dim;
  const int gi = particles[p0 + i / nmax] * nmax + i % nmax;
  for (int c0 = 0; c0 < nrhs; c0 += CPP) {
    const int nc = min(CPP, nrhs - c0);
    double ar[CPP], ai[CPP];
#pragma unroll
    for (int q = 0; q < CPP; ++q) { ar[q] = 0.0; ai[q] = 0.0; }
    for (int c = lane; c < dim; c += 32) {
      const MT m = row[c];
      const double mr = (double)m.x, mi = (double)m.y;
      const int gc = particles[p0 + c / nmax] * nmax + c % nmax;
#pragma unroll
      for (int q = 0; q < CPP; ++q) {
        if (q < nc) {
          const double2 xv = x[(size_t)(c0 + q) * ld + gc];
          ar[q] += mr * xv.x - mi * xv.y;
          ai[q] += mr * xv.y + mi * xv.x;
        }
      }
    }
#pragma unroll
    for (int q = 0; q < CPP; ++q) {
      for (int off = 16; off > 0; off >>= 1) {
        ar[q] += __shfl_down_sync(0xffffffffu, ar[q], off);
        ai[q] += __shfl_down_sync(0xffffffffu, ai[q], off);
      }
    }
    if (lane == 0) {
      for (int q = 0; q < nc; ++q) y[(size_t)(c0 + q) * ld + gi] = make_double2(ar[q], ai[q]);
    }
  }
}

}  // namespace yasf

using namespace yasf;

extern "C" int yasf_precond_create(const yasf_plan* plan, int n_particles, int n_blocks,
                                   const int* block_ptr, const int* particles, yasf_precond** out) {
  if (!out || !plan || !block_ptr || !particles || n_particles <= 0 || n_blocks <= 0)
    return YASF_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (block_ptr[0] != 0 || block_ptr[n_blocks] != n_particles) return YASF_ERR_INVALID_ARGUMENT;
  std::vector<int> pblock(n_particles, -1), plocal(n_particles, -1);
  for (int b = 0; b < n_blocks; ++b) {
    if (block_ptr[b + 1] <= block_ptr[b]) return YASF_ERR_INVALID_ARGUMENT;
    for (int q = block_ptr[b]; q < block_ptr[b + 1]; ++q) {
      const int s = particles[q];
      if (s < 0 || s >= n_particles || pblock[s] != -1) return YASF_ERR_INVALID_ARGUMENT;
      pblock[s] = b;
      plocal[s] = q - block_ptr[b];
    }
  }
  yasf_precond* pc = new (std::nothrow) yasf_precond();
  if (!pc) return YASF_ERR_OUT_OF_MEMORY;
  pc->plan = plan;
  pc->n_particles = n_particles;
  pc->n_blocks = n_blocks;
  pc->block_ptr.assign(block_ptr, block_ptr + n_blocks + 1);
  const int nmax = plan->nmax;
  std::vector<int> row_block, row_local;
  long long off = 0;
  for (int b = 0; b < n_blocks; ++b) {
    const int dim = (block_ptr[b + 1] - block_ptr[b]) * nmax;
    pc->mat_off.push_back(off);
    off += (long long)dim * dim;
    for (int i = 0; i < dim; ++i) {
      row_block.push_back(b);
      row_local.push_back(i);
    }
  }
  pc->mat_elems = (size_t)off;
  pc->total_rows = (int)row_block.size();
  cudaError_t e = cudaSuccess;
  auto up = [&](auto** dst, const auto* src, size_t count) {
    if (e != cudaSuccess) return;
    e = cudaMalloc(reinterpret_cast<void**>(dst), std::max<size_t>(1, count) * sizeof(**dst));
    if (e == cudaSuccess) e = cudaMemcpy(*dst, src, count * sizeof(**dst), cudaMemcpyHostToDevice);
  };
  up(&pc->d_block_ptr, block_ptr, n_blocks + 1);
  up(&pc->d_particles, particles, n_particles);
  up(&pc->d_particle_block, pblock.data(), n_particles);
  up(&pc->d_particle_local, plocal.data(), n_particles);
  up(&pc->d_mat_off, pc->mat_off.data(), pc->mat_off.size());
  up(&pc->d_row_block, row_block.data(), row_block.size());
  up(&pc->d_row_local, row_local.data(), row_local.size());
  // LU geometry: block orders, first rows, first diagonal tiles; per step k the prefix sums over
  // blocks of the CTAs of the diagonal / panel / update launches and of sweep step k
  {
    std::vector<int> dims(n_blocks), row0(n_blocks), tile0(n_blocks);
    int rows = 0, tiles = 0, steps = 0;
    for (int b = 0; b < n_blocks; ++b) {
      dims[b] = (block_ptr[b + 1] - block_ptr[b]) * nmax;
      row0[b] = rows;
      tile0[b] = tiles;
      rows += dims[b];
      const int nt = (dims[b] + kLuT - 1) / kLuT;
      tiles += nt;
      steps = std::max(steps, nt);
    }
    pc->lu_steps = steps;
    pc->n_tiles = tiles;
    const int W = n_blocks + 1;
    for (auto* v : {&pc->pre_diag, &pc->pre_panel, &pc->pre_update, &pc->pre_sweep}) v->assign((size_t)steps * W, 0);
    for (int k = 0; k < steps; ++k)
      for (int b = 0; b < n_blocks; ++b) {
        const int nt = (dims[b] + kLuT - 1) / kLuT;
        const int live = k < nt;
        const int rest = live ? nt - k - 1 : 0;
        pc->pre_diag[(size_t)k * W + b + 1] = pc->pre_diag[(size_t)k * W + b] + live;
        pc->pre_panel[(size_t)k * W + b + 1] = pc->pre_panel[(size_t)k * W + b] + (live ? nt - 1 + rest : 0);
        pc->pre_update[(size_t)k * W + b + 1] = pc->pre_update[(size_t)k * W + b] + rest * rest;
        pc->pre_sweep[(size_t)k * W + b + 1] = pc->pre_sweep[(size_t)k * W + b] + (live ? nt - k : 0);
      }
    std::vector<int> pre;
    for (auto* v : {&pc->pre_diag, &pc->pre_panel, &pc->pre_update, &pc->pre_sweep})
      pre.insert(pre.end(), v->begin(), v->end());
    up(&pc->d_dim, dims.data(), dims.size());
    up(&pc->d_row0, row0.data(), row0.size());
    up(&pc->d_tile0, tile0.data(), tile0.size());
    up(&pc->d_pre, pre.data(), pre.size());
    std::vector<int2> order;
    order.reserve(2 * (size_t)tiles);
    for (int upper = 0; upper < 2; ++upper)
      for (int c = 0; c < steps; ++c)
        for (int b = 0; b < n_blocks; ++b) {
          const int nt = (dims[b] + kLuT - 1) / kLuT;
          if (c < nt) order.push_back(make_int2(b, upper ? nt - 1 - c : c));
        }
    up(&pc->d_order, order.data(), order.size());
    if (e == cudaSuccess)
      e = cudaMalloc(reinterpret_cast<void**>(&pc->d_sync), (2 + 2 * (size_t)n_blocks) * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&pc->d_piv), std::max(1, rows) * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&pc->d_err), sizeof(int));
  }
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&pc->d_mat), pc->mat_elems * sizeof(double2));
  if (e != cudaSuccess) {
    set_cuda_error(e);
    yasf_precond_destroy(pc);
    return e == cudaErrorMemoryAllocation ? YASF_ERR_OUT_OF_MEMORY : YASF_ERR_CUDA;
  }
  *out = pc;
  return YASF_OK;
}

extern "C" int yasf_precond_destroy(yasf_precond* pc) {
  if (!pc) return YASF_OK;
  cudaFree(pc->d_block_ptr);
  cudaFree(pc->d_particles);
  cudaFree(pc->d_particle_block);
  cudaFree(pc->d_particle_local);
  cudaFree(pc->d_mat_off);
  cudaFree(pc->d_row_block);
  cudaFree(pc->d_row_local);
  cudaFree(pc->d_mat);
  cudaFree(pc->d_mat32);
  cudaFree(pc->d_dim);
  cudaFree(pc->d_row0);
  cudaFree(pc->d_tile0);
  cudaFree(pc->d_pre);
  cudaFree(pc->d_piv);
  cudaFree(pc->d_err);
  cudaFree(pc->d_dinv);
  cudaFree(pc->d_dinv64);
  cudaFree(pc->d_z);
  cudaFree(pc->d_order);
  cudaFree(pc->d_sync);
  for (auto& g : pc->graphs) cudaGraphExecDestroy(g.exec);
  if (pc->capture_stream) cudaStreamDestroy(pc->capture_stream);
  delete pc;
  return YASF_OK;
}

namespace {
yasf::LuGeom lu_geom(const yasf_precond* pc) {
  yasf::LuGeom g;
  g.mat_off = pc->d_mat_off;
  g.dim = pc->d_dim;
  g.row0 = pc->d_row0;
  g.tile0 = pc->d_tile0;
  g.n_blocks = pc->n_blocks;
  return g;
}
// prefix table `which` (0 diag, 1 panel, 2 update, 3 sweep) of step k on the device, and its CTA count
const int* lu_pre(const yasf_precond* pc, int which, int k, int* ctas) {
  const size_t W = (size_t)pc->n_blocks + 1;
  const std::vector<int>* v[4] = {&pc->pre_diag, &pc->pre_panel, &pc->pre_update, &pc->pre_sweep};
  *ctas = (*v[which])[(size_t)k * W + pc->n_blocks];
  return pc->d_pre + (size_t)which * pc->lu_steps * W + (size_t)k * W;
}
// The kernels' dynamic shared-memory limits are function attributes of the current device: set
// once per device (a process may drive several GPUs, from several host threads).
int lu_smem_attributes() {
  static std::atomic<unsigned long long> done{0};
  int dev = 0;
  YASF_CUDA_TRY(cudaGetDevice(&dev));
  const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
  if (bit && (done.load(std::memory_order_acquire) & bit)) return YASF_OK;
  const int one = (int)(yasf::kLuT * yasf::kLuS * sizeof(double2));
  YASF_CUDA_TRY(cudaFuncSetAttribute(yasf::lu_diag_kernel<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, one));
  YASF_CUDA_TRY(cudaFuncSetAttribute(yasf::lu_diag_kernel<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, one));
  YASF_CUDA_TRY(cudaFuncSetAttribute(yasf::lu_panel_inv_kernel<double2>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)yasf::kLuUpdateSmem));
  YASF_CUDA_TRY(cudaFuncSetAttribute(yasf::lu_panel_inv_kernel<float2>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)yasf::kLuUpdateSmem));
  YASF_CUDA_TRY(cudaFuncSetAttribute(yasf::lu_diag_inverse_kernel<double2>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * one));
  YASF_CUDA_TRY(cudaFuncSetAttribute(yasf::lu_diag_inverse_kernel<float2>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * one));
  YASF_CUDA_TRY(cudaFuncSetAttribute(yasf::lu_update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)yasf::kLuUpdateSmem));
  YASF_CUDA_TRY(cudaFuncSetAttribute(yasf::lu_update32_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)yasf::kLuUpdateSmem32));
  YASF_CUDA_TRY(cudaFuncSetAttribute(yasf::lu_solve_kernel<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)yasf::lu_solve_smem<float2>()));
  YASF_CUDA_TRY(cudaFuncSetAttribute(yasf::lu_solve_kernel<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)yasf::lu_solve_smem<double2>()));
  done.fetch_or(bit, std::memory_order_release);
  return YASF_OK;
}
}  // namespace

extern "C" int yasf_precond_factor(yasf_precond* pc, void* stream) {
  if (!pc) return YASF_ERR_INVALID_ARGUMENT;
  if (!pc->assembled || !pc->d_mat) return YASF_ERR_NOT_PREPARED;
  if (int st = check_current_device(pc->plan->device)) return st;
  if (int st = lu_smem_attributes()) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const LuGeom g = lu_geom(pc);
  const int one = (int)(kLuT * kLuS * sizeof(double2));
  const bool c64 = !pc->keep_f64;
  if (c64) {  // the reference's precision: convert the blocks, release the complex128 copy
    if (!pc->d_mat32) {
      cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&pc->d_mat32), pc->mat_elems * sizeof(float2));
      if (e != cudaSuccess) {
        set_cuda_error(e);
        pc->d_mat32 = nullptr;
        return e == cudaErrorMemoryAllocation ? YASF_ERR_OUT_OF_MEMORY : YASF_ERR_CUDA;
      }
    }
    YASF_COUNTED(to_c64_kernel<<<2048, 256, 0, s>>>(pc->mat_elems, pc->d_mat, pc->d_mat32));
    YASF_CUDA_TRY(cudaGetLastError());
    YASF_CUDA_TRY(cudaStreamSynchronize(s));
    YASF_CUDA_TRY(cudaFree(pc->d_mat));
    pc->d_mat = nullptr;
  }
  {  // the diagonal-tile inverses: complex64 for the apply, complex128 for the panel products
    const size_t tile_elems = (size_t)pc->n_tiles * 2 * kLuT * kLuT;
    for (int w = 0; w < 2; ++w) {
      void** p = w ? reinterpret_cast<void**>(&pc->d_dinv64) : reinterpret_cast<void**>(&pc->d_dinv);
      if (*p) continue;
      cudaError_t e = cudaMalloc(p, tile_elems * (w ? sizeof(double2) : sizeof(float2)));
      if (e != cudaSuccess) {
        set_cuda_error(e);
        *p = nullptr;
        return e == cudaErrorMemoryAllocation ? YASF_ERR_OUT_OF_MEMORY : YASF_ERR_CUDA;
      }
    }
  }
  YASF_CUDA_TRY(cudaMemsetAsync(pc->d_err, 0, sizeof(int), s));
  for (int k = 0; k < pc->lu_steps; ++k) {
    int n = 0;
    const int* pre = lu_pre(pc, 0, k, &n);
    if (n && c64) {
      YASF_COUNTED(lu_diag_kernel<float2><<<n, 256, one, s>>>(g, pre, k, pc->d_mat32, pc->d_piv, pc->d_err));
      YASF_COUNTED(lu_diag_inverse_kernel<float2><<<n, 256, 2 * one, s>>>(g, pre, pc->d_mat32, pc->d_dinv,
                                                                          pc->d_dinv64, pc->d_err, k));
    } else if (n) {
      YASF_COUNTED(lu_diag_kernel<double2><<<n, 256, one, s>>>(g, pre, k, pc->d_mat, pc->d_piv, pc->d_err));
      YASF_COUNTED(lu_diag_inverse_kernel<double2><<<n, 256, 2 * one, s>>>(g, pre, pc->d_mat, pc->d_dinv,
                                                                           pc->d_dinv64, pc->d_err, k));
    }
    pre = lu_pre(pc, 1, k, &n);
    if (n && c64)
      YASF_COUNTED(lu_panel_inv_kernel<float2><<<n, 256, kLuUpdateSmem, s>>>(g, pre, k, pc->d_mat32, pc->d_piv,
                                                                             pc->d_dinv64));
    else if (n)
      YASF_COUNTED(lu_panel_inv_kernel<double2><<<n, 256, kLuUpdateSmem, s>>>(g, pre, k, pc->d_mat, pc->d_piv,
                                                                              pc->d_dinv64));
    pre = lu_pre(pc, 2, k, &n);
    if (n && c64)
      YASF_COUNTED(lu_update32_kernel<<<n, kLuUpd32Threads, kLuUpdateSmem32, s>>>(g, pre, k, pc->d_mat32));
    else if (n) YASF_COUNTED(lu_update_kernel<<<n, 256, kLuUpdateSmem, s>>>(g, pre, k, pc->d_mat));
    YASF_CUDA_TRY(cudaGetLastError());
  }
  pc->factored = true;
  pc->factored_c64 = c64;
  pc->prepared = false;
  return YASF_OK;
}

extern "C" int yasf_precond_keep_float64(yasf_precond* pc, int keep) {
  if (!pc) return YASF_ERR_INVALID_ARGUMENT;
  pc->keep_f64 = keep != 0;
  return YASF_OK;
}

extern "C" int yasf_precond_assemble(yasf_precond* pc, const double* positions, double k_medium,
                                     const double* tmat, void* stream) {
  if (!pc || !positions || !tmat) return YASF_ERR_INVALID_ARGUMENT;
  if (!std::isfinite(k_medium) || k_medium <= 0.0) return YASF_ERR_UNSUPPORTED;
  if (!aligned16(tmat)) return YASF_ERR_ALIGNMENT;
  const yasf_plan* plan = pc->plan;
  if (int st = check_current_device(plan->device)) return st;
  if (!pc->d_mat) {  // released by a finalize that kept only the complex64 factors
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&pc->d_mat), pc->mat_elems * sizeof(double2));
    if (e != cudaSuccess) {
      set_cuda_error(e);
      pc->d_mat = nullptr;
      return e == cudaErrorMemoryAllocation ? YASF_ERR_OUT_OF_MEMORY : YASF_ERR_CUDA;
    }
  }
  AsmArgs a{};
  a.L = plan->lmax;
  a.nmax = plan->nmax;
  a.k = k_medium;
  a.pos = positions;
  a.tmat = reinterpret_cast<const double2*>(tmat);
  a.block_ptr = pc->d_block_ptr;
  a.particles = pc->d_particles;
  a.particle_block = pc->d_particle_block;
  a.particle_local = pc->d_particle_local;
  a.mat_off = pc->d_mat_off;
  a.pair_ptr = plan->d_pair_ptr;
  a.pair_p = plan->d_pair_p;
  a.pair_coef = plan->d_pair_coef;
  a.leg = plan->d_leg;
  a.mat = pc->d_mat;
  const size_t smem = (size_t)kAsmChunk * (2 * a.L + 1) * (4 * a.L + 1) * sizeof(double2);
  if (smem > 48 * 1024)
    YASF_CUDA_TRY(cudaFuncSetAttribute(assemble_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  YASF_COUNTED(assemble_kernel<<<pc->n_particles, 256, smem, s>>>(a));
  YASF_CUDA_TRY(cudaGetLastError());
  pc->assembled = true;
  pc->prepared = false;
  pc->factored = false;
  pc->factored_c64 = false;
  return YASF_OK;
}

extern "C" int yasf_precond_block(const yasf_precond* pc, int block, double** matrix, int* dim) {
  if (!pc || !matrix || !dim || block < 0 || block >= pc->n_blocks) return YASF_ERR_INVALID_ARGUMENT;
  if (!pc->d_mat) {
    set_error_text("the complex128 blocks were released (complex64 factorisation or finalize)");
    return YASF_ERR_NOT_PREPARED;
  }
  *matrix = reinterpret_cast<double*>(pc->d_mat + pc->mat_off[block]);
  *dim = (pc->block_ptr[block + 1] - pc->block_ptr[block]) * pc->plan->nmax;
  return YASF_OK;
}

extern "C" int yasf_precond_finalize(yasf_precond* pc, void* stream) {
  if (!pc) return YASF_ERR_INVALID_ARGUMENT;
  if (!pc->assembled || (!pc->d_mat && !pc->factored_c64)) return YASF_ERR_NOT_PREPARED;
  if (pc->factored_c64 && pc->keep_f64) {
    set_error_text("keep_float64 must be set before factor: the blocks were factored in complex64");
    return YASF_ERR_INVALID_ARGUMENT;
  }
  if (int st = check_current_device(pc->plan->device)) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  auto alloc = [&](void** p, size_t bytes) -> int {
    if (*p) return YASF_OK;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
      set_cuda_error(e);
      *p = nullptr;
      return e == cudaErrorMemoryAllocation ? YASF_ERR_OUT_OF_MEMORY : YASF_ERR_CUDA;
    }
    return YASF_OK;
  };
  if (!pc->factored_c64) {  // the complex64 copy of the complex128 factors (or inverses)
    if (int st = alloc(reinterpret_cast<void**>(&pc->d_mat32), pc->mat_elems * sizeof(float2))) return st;
    YASF_COUNTED(to_c64_kernel<<<2048, 256, 0, s>>>(pc->mat_elems, pc->d_mat, pc->d_mat32));
    YASF_CUDA_TRY(cudaGetLastError());
  }
  if (pc->factored) {  // the inverses of the diagonal tiles were made during the factorisation
    int err = 0;
    YASF_CUDA_TRY(cudaMemcpyAsync(&err, pc->d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    YASF_CUDA_TRY(cudaStreamSynchronize(s));
    if (err) {
      set_error_text("a block has a zero pivot (singular diagonal tile)");
      return YASF_ERR_NOT_FINITE;
    }
    if (!pc->keep_f64) {  // the solves stream the complex64 factors and inverses only
      if (pc->d_mat) YASF_CUDA_TRY(cudaFree(pc->d_mat));
      pc->d_mat = nullptr;
      if (pc->d_dinv64) YASF_CUDA_TRY(cudaFree(pc->d_dinv64));
      pc->d_dinv64 = nullptr;
    }
  }
  for (auto& gr : pc->graphs) cudaGraphExecDestroy(gr.exec);  // captured the previous factors
  pc->graphs.clear();
  pc->prepared = true;
  return YASF_OK;
}

extern "C" int yasf_precond_apply(const yasf_precond* pc, const double* x, double* y, int nrhs,
                                  long long ld, int precision, void* stream) {
  if (!pc || !x || !y || nrhs <= 0) return YASF_ERR_INVALID_ARGUMENT;
  if (!pc->prepared) return YASF_ERR_NOT_PREPARED;
  if (x == y) return YASF_ERR_INVALID_ARGUMENT;
  const long long n = (long long)pc->n_particles * pc->plan->nmax;
  if (nrhs > 1 && ld < n) return YASF_ERR_INVALID_ARGUMENT;
  if (nrhs == 1) ld = n;
  if (!aligned16(x) || !aligned16(y)) return YASF_ERR_ALIGNMENT;
  if (int st = check_current_device(pc->plan->device)) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (pc->factored) {
    if (precision != YASF_C64 && precision != YASF_C128) return YASF_ERR_INVALID_ARGUMENT;
    const bool f64 = precision == YASF_C128 && pc->d_mat && pc->d_dinv64;
    if (nrhs > pc->z_cols) {  // the sweep buffer grows to the widest apply seen
      double2* z = nullptr;
      cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&z), (size_t)pc->total_rows * nrhs * sizeof(double2));
      if (e != cudaSuccess) {
        set_cuda_error(e);
        return e == cudaErrorMemoryAllocation ? YASF_ERR_OUT_OF_MEMORY : YASF_ERR_CUDA;
      }
      YASF_CUDA_TRY(cudaStreamSynchronize(s));
      cudaFree(pc->d_z);
      yasf_precond* mpc = const_cast<yasf_precond*>(pc);
      mpc->d_z = z;
      mpc->z_cols = nrhs;
      for (auto& gr : mpc->graphs) cudaGraphExecDestroy(gr.exec);  // they captured the old buffer
      mpc->graphs.clear();
    }
    yasf_precond* mpc = const_cast<yasf_precond*>(pc);
    const int gb = (int)std::min<long long>(((long long)pc->total_rows * nrhs + 255) / 256, 8192);
    YASF_COUNTED(lu_gather_kernel<<<gb, 256, 0, s>>>(pc->total_rows, pc->plan->nmax, nrhs, ld, pc->d_row_block,
                                                     pc->d_row_local, pc->d_block_ptr, pc->d_particles,
                                                     pc->d_row0, pc->d_piv, reinterpret_cast<const double2*>(x),
                                                     pc->d_z));
    const LuGeom g = lu_geom(pc);
    if (nrhs == 1) {  // both sweeps in one launch, rows ordered by tickets
      if (int st = lu_smem_attributes()) return st;
      LuSolveArgs sa;
      sa.g = g;
      sa.order = pc->d_order;
      sa.n_tiles = pc->n_tiles;
      sa.z = pc->d_z;
      sa.sync = pc->d_sync;
      sa.wait_ns = stall_hook().panel_wait_ns;
      sa.stall = stall_hook().role == YASF_STALL_PRECOND ? 1 : 0;
      YASF_CUDA_TRY(cudaMemsetAsync(pc->d_sync, 0, (2 + 2 * (size_t)pc->n_blocks) * sizeof(int), s));
      if (f64)
        YASF_COUNTED(lu_solve_kernel<double2><<<2 * pc->n_tiles, 256, lu_solve_smem<double2>(), s>>>(
            sa, pc->d_mat, pc->d_dinv64));
      else
        YASF_COUNTED(lu_solve_kernel<float2><<<2 * pc->n_tiles, 256, lu_solve_smem<float2>(), s>>>(
            sa, pc->d_mat32, pc->d_dinv));
      YASF_COUNTED(lu_scatter_kernel<<<gb, 256, 0, s>>>(pc->total_rows, pc->plan->nmax, nrhs, ld, pc->d_row_block,
                                                        pc->d_row_local, pc->d_block_ptr, pc->d_particles, pc->d_z,
                                                        reinterpret_cast<double2*>(y)));
      YASF_CUDA_TRY(cudaGetLastError());
      return YASF_OK;
    }
    // several columns: the forward and backward sweeps (one launch per tile row) into stream `ss`
    auto sweeps = [&](cudaStream_t ss) -> int {
      int launched = 0;
      for (int upper = 0; upper < 2; ++upper)
        for (int step = 0; step < pc->lu_steps; ++step) {
          int n = 0;
          const int* pre = lu_pre(pc, 3, step, &n);
          if (!n) continue;
          if (f64 && nrhs == 1)
            lu_sweep_kernel<double2, 1><<<n, 256, 0, ss>>>(g, pre, step, upper, pc->d_mat, pc->d_dinv64, nrhs,
                                                           pc->total_rows, pc->d_z);
          else if (f64)
            lu_sweep_kernel<double2, kLuCols><<<n, 256, 0, ss>>>(g, pre, step, upper, pc->d_mat, pc->d_dinv64,
                                                                 nrhs, pc->total_rows, pc->d_z);
          else if (nrhs == 1)
            lu_sweep_kernel<float2, 1><<<n, 256, 0, ss>>>(g, pre, step, upper, pc->d_mat32, pc->d_dinv, nrhs,
                                                          pc->total_rows, pc->d_z);
          else
            lu_sweep_kernel<float2, kLuCols><<<n, 256, 0, ss>>>(g, pre, step, upper, pc->d_mat32, pc->d_dinv,
                                                                nrhs, pc->total_rows, pc->d_z);
          ++launched;
        }
      return launched;
    };
    const yasf_precond::SweepGraph* graph = nullptr;
    for (const auto& gr : pc->graphs)
      if (gr.nrhs == nrhs && gr.f64 == f64) graph = &gr;
    if (!graph) {  // capture once on the private stream; a failed capture falls back to launches
      if (!mpc->capture_stream) YASF_CUDA_TRY(cudaStreamCreateWithFlags(&mpc->capture_stream, cudaStreamNonBlocking));
      cudaGraph_t gr = nullptr;
      cudaGraphExec_t exec = nullptr;
      int launched = 0;
      if (cudaStreamBeginCapture(mpc->capture_stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        launched = sweeps(mpc->capture_stream);
        if (cudaStreamEndCapture(mpc->capture_stream, &gr) == cudaSuccess && gr &&
            cudaGraphInstantiate(&exec, gr, 0) == cudaSuccess) {
          mpc->graphs.push_back({nrhs, f64, launched, exec});
          graph = &mpc->graphs.back();
        }
        if (gr) cudaGraphDestroy(gr);
      }
      (void)cudaGetLastError();  // a refused capture leaves no sticky error
    }
    if (graph) {
      YASF_CUDA_TRY(cudaGraphLaunch(graph->exec, s));
      for (int i = 0; i < graph->launches; ++i) count_launch();
    } else {
      const int launched = sweeps(s);
      for (int i = 0; i < launched; ++i) count_launch();
      YASF_CUDA_TRY(cudaGetLastError());
    }
    YASF_COUNTED(lu_scatter_kernel<<<gb, 256, 0, s>>>(pc->total_rows, pc->plan->nmax, nrhs, ld, pc->d_row_block,
                                                      pc->d_row_local, pc->d_block_ptr, pc->d_particles, pc->d_z,
                                                      reinterpret_cast<double2*>(y)));
    YASF_CUDA_TRY(cudaGetLastError());
    return YASF_OK;
  }
  const int blocks = (pc->total_rows + 7) / 8;
  const double2* xx = reinterpret_cast<const double2*>(x);
  double2* yy = reinterpret_cast<double2*>(y);
#define YASF_APPLY(MT, CPP, MAT)                                                                    \
  YASF_COUNTED(apply_kernel<MT, CPP><<<blocks, 256, 0, s>>>(                                        \
      pc->total_rows, pc->plan->nmax, nrhs, ld, pc->d_row_block, pc->d_row_local, pc->d_block_ptr, \
      pc->d_particles, pc->d_mat_off, MAT, xx, yy))
  if (precision == YASF_C64) {
    if (nrhs == 1) YASF_APPLY(float2, 1, pc->d_mat32);
    else if (nrhs <= 4) YASF_APPLY(float2, 4, pc->d_mat32);
    else YASF_APPLY(float2, 16, pc->d_mat32);
  } else if (precision == YASF_C128) {
    if (nrhs == 1) YASF_APPLY(double2, 1, pc->d_mat);
    else if (nrhs <= 4) YASF_APPLY(double2, 4, pc->d_mat);
    else YASF_APPLY(double2, 16, pc->d_mat);
  } else {
    return YASF_ERR_INVALID_ARGUMENT;
  }
#undef YASF_APPLY
  YASF_CUDA_TRY(cudaGetLastError());
  return YASF_OK;
}

extern "C" int yasf_precond_bytes(const yasf_precond* pc, size_t* bytes) {
  if (!pc || !bytes) return YASF_ERR_INVALID_ARGUMENT;
  const size_t tiles = (size_t)pc->n_tiles * 2 * kLuT * kLuT;
  *bytes = pc->mat_elems * ((pc->d_mat ? sizeof(double2) : 0) + (pc->d_mat32 ? sizeof(float2) : 0)) +
           (pc->d_dinv ? tiles * sizeof(float2) : 0) + (pc->d_dinv64 ? tiles * sizeof(double2) : 0) +
           (size_t)pc->total_rows * pc->z_cols * sizeof(double2);
  return YASF_OK;
}
