// Batched LU factorisation of the block-Jacobi blocks and the triangular sweeps that apply it.
//
// The reference factors each block with LU and applies it by a unit-lower then an upper
// triangular solve (yasfpy/preconditioner.py:445-519, scipy.linalg.lu on complex64 blocks,
// :391). Here every block of one preconditioner is factored on the device in one sequence of
// launches (variable block orders batched together), in complex128, in place:
//
//   right-looking tile LU, tiles of kLuT = 64 rows / columns. Step k factors the diagonal tile
//   with partial pivoting inside it (its 64 rows; the interchanges are applied to the whole tile
//   row, left and right), solves the tile row for U and the tile column for L, and updates the
//   trailing tiles A_ij -= L_ik U_kj. The result is P A = L U with P block diagonal (a permutation
//   within each tile row). Pivoting inside the diagonal tile rather than over the whole column
//   keeps every step parallel over tiles; on the blocks of I - T W the growth factor stays near 1.
//
// Each step is four launches over all blocks that still have a tile k (diagonal tile, its inverses,
// tile row and column as products with those inverses, trailing update); host-built prefix sums
// (one row per step) map a CTA index to (block, tile). Ragged edges (block order not a multiple of
// 64) are padded with the identity in the diagonal tile and zeros elsewhere; padded entries are
// never stored.
//
// Apply (finalize keeps only a complex64 copy of the factors plus the complex64 inverses of the
// diagonal tiles of L and U, and frees the complex128 matrices): z = P x gathered from the
// particle-major vector, forward sweep with L, backward sweep with U, scattered back. One column
// (every Krylov step): both sweeps in ONE launch whose CTAs take tile rows in ticket order and wait
// on per-block finished-row counters (lu_solve_kernel). Several columns: one launch per sweep
// step; step s of the forward pass: every tile row i >= s subtracts L_{i,s-1} z_{s-1} (finished by
// the previous launch), and tile row s then multiplies by L_ss^{-1}; the backward pass mirrors it.
// Both forms sum every row in a fixed order, so applies are deterministic. Arithmetic is float64
// throughout.
#pragma once

#include "capi_internal.h"

namespace yasf {

constexpr int kLuT = 64;        // tile order
constexpr int kLuS = kLuT + 1;  // shared-memory row stride (complex128), breaks bank conflicts
constexpr int kLuKc = 32;       // inner-dimension chunk of the tile products

struct LuGeom {
  const long long* mat_off;  // element offset of block b's matrix (row-major, order dim[b])
  const int* dim;            // order of block b
  const int* row0;           // first flattened row of block b
  const int* tile0;          // first flattened diagonal tile of block b
  int n_blocks;
};

__device__ __forceinline__ double2 c_mul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 c_sub_mul(double2 c, double2 a, double2 b) {  // c - a b
  return make_double2(c.x - (a.x * b.x - a.y * b.y), c.y - (a.x * b.y + a.y * b.x));
}
__device__ __forceinline__ double2 c_inv(double2 d, bool* zero) {
  const double m = d.x * d.x + d.y * d.y;
  if (m == 0.0) { *zero = true; return make_double2(0.0, 0.0); }
  return make_double2(d.x / m, -d.y / m);
}

// Block of work item `item` given the prefix sums pre[0..n_blocks] of one step.
__device__ __forceinline__ int lu_block_of(const int* pre, int n_blocks, int item) {
  int lo = 0, hi = n_blocks;  // pre[lo] <= item < pre[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (pre[mid] <= item) lo = mid; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ int lu_tiles(int dim) { return (dim + kLuT - 1) / kLuT; }

// Matrix storage of a factorisation: complex128 (double2) or complex64 (float2). The diagonal,
// panel and inverse steps compute in float64 in shared memory whatever the storage.
__device__ __forceinline__ double2 lu_load(const double2& v) { return v; }
__device__ __forceinline__ double2 lu_load(const float2& v) { return make_double2(v.x, v.y); }
template <typename T> __device__ __forceinline__ T lu_cast(double2 v);
template <> __device__ __forceinline__ double2 lu_cast<double2>(double2 v) { return v; }
template <> __device__ __forceinline__ float2 lu_cast<float2>(double2 v) {
  return make_float2((float)v.x, (float)v.y);
}

// ---- step k, part 1: the diagonal tile, partial pivoting inside it -----------------------------
// piv[row0 + k*64 + r] = local source row (0..63) of row r after the interchanges.
template <typename T>
__global__ void __launch_bounds__(256) lu_diag_kernel(LuGeom g, const int* pre, int k, T* mat, int* piv,
                                                      int* err) {
  extern __shared__ double2 lu_smem[];
  double2* t = lu_smem;  // [64][kLuS]
  __shared__ int perm[kLuT];
  __shared__ int pivrow;
  __shared__ int singular;
  const int b = lu_block_of(pre, g.n_blocks, blockIdx.x);
  const int dim = g.dim[b];
  const int k0 = k * kLuT;
  const int v = min(kLuT, dim - k0);
  T* A = mat + g.mat_off[b];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int e = tid; e < kLuT * kLuT; e += blockDim.x) {
    const int r = e >> 6, c = e & 63;
    t[r * kLuS + c] = (r < v && c < v) ? lu_load(A[(size_t)(k0 + r) * dim + k0 + c])
                                       : make_double2(r == c ? 1.0 : 0.0, 0.0);
  }
  if (tid < kLuT) perm[tid] = tid;
  if (tid == 0) singular = 0;
  for (int c = 0; c < kLuT; ++c) {
    __syncthreads();
    if (warp == 0) {
      // argmax |t[r][c]|, r >= c (ties: the smaller row)
      double best = -1.0;
      int br = c;
      for (int r = c + lane; r < kLuT; r += 32) {
        const double2 x = t[r * kLuS + c];
        const double m = x.x * x.x + x.y * x.y;
        if (m > best) { best = m; br = r; }
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double ob = __shfl_down_sync(0xffffffffu, best, off);
        const int orow = __shfl_down_sync(0xffffffffu, br, off);
        if (ob > best || (ob == best && orow < br)) { best = ob; br = orow; }
      }
      if (lane == 0) pivrow = br;
    }
    __syncthreads();
    const int p = pivrow;
    if (p != c) {
      if (tid < kLuT) {
        const double2 a = t[c * kLuS + tid];
        t[c * kLuS + tid] = t[p * kLuS + tid];
        t[p * kLuS + tid] = a;
      }
      if (tid == 0) {
        const int q = perm[c];
        perm[c] = perm[p];
        perm[p] = q;
      }
      __syncthreads();
    }
    bool zero = false;
    const double2 inv = c_inv(t[c * kLuS + c], &zero);
    if (zero && tid == 0) singular = 1;
    const int rem = kLuT - 1 - c;
    if (tid < rem) {
      const int r = c + 1 + tid;
      t[r * kLuS + c] = c_mul(t[r * kLuS + c], inv);
    }
    __syncthreads();
    for (int e = tid; e < rem * rem; e += blockDim.x) {
      const int r = c + 1 + e / rem, j = c + 1 + e % rem;
      t[r * kLuS + j] = c_sub_mul(t[r * kLuS + j], t[r * kLuS + c], t[c * kLuS + j]);
    }
  }
  __syncthreads();
  for (int e = tid; e < kLuT * kLuT; e += blockDim.x) {
    const int r = e >> 6, c = e & 63;
    if (r < v && c < v) A[(size_t)(k0 + r) * dim + k0 + c] = lu_cast<T>(t[r * kLuS + c]);
  }
  if (tid < v) piv[g.row0[b] + k0 + tid] = perm[tid];
  if (tid == 0 && singular) atomicExch(err, 1);
}

// ---- step k, part 2: tile row k and tile column k, as products with the inverses of the diagonal
// tile (lu_diag_inverse_kernel, run right after the tile was factored; the apply uses the same
// inverses): U_kj = L_kk^{-1} (P A_kj) for j > k, P A_kj for j < k (the interchanges applied to
// the left part), and L_ik = A_ik U_kk^{-1} for i > k. Each tile is a 64 x 64 x 64 complex product
// in float64 (256 threads, 4 x 4 outputs each, the inner dimension staged in two chunks of 32)
// instead of 64 dependent elimination steps with a barrier each.
template <typename T>
__global__ void __launch_bounds__(256, 2) lu_panel_inv_kernel(LuGeom g, const int* pre, int k, T* mat,
                                                             const int* piv, const double2* dinv64) {
  extern __shared__ double2 lu_smem[];
  double2(*Ls)[kLuS] = reinterpret_cast<double2(*)[kLuS]>(lu_smem);                 // Ls[kk][row] = Left[row][kc + kk]
  double2(*Us)[kLuS] = reinterpret_cast<double2(*)[kLuS]>(lu_smem + kLuKc * kLuS);  // Us[kk][col] = Right[kc + kk][col]
  const int b = lu_block_of(pre, g.n_blocks, blockIdx.x);
  const int item = blockIdx.x - pre[b];
  const int dim = g.dim[b];
  const int nt = lu_tiles(dim);
  const int k0 = k * kLuT;
  const int vk = min(kLuT, dim - k0);
  T* A = mat + g.mat_off[b];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int nrow = nt - 1;
  const bool row_tile = item < nrow;
  const int j = row_tile ? (item < k ? item : item + 1) : k;  // output tile column
  const int i = row_tile ? k : k + 1 + (item - nrow);         // output tile row
  const int i0 = i * kLuT, j0 = j * kLuT;
  const int vi = min(kLuT, dim - i0), vj = min(kLuT, dim - j0);
  const int* p = piv + g.row0[b] + k0;
  if (row_tile && j < k) {  // left of the diagonal: the interchanges only (rows of one tile row)
    double2* X = lu_smem;   // [64][kLuS]
    for (int e = tid; e < kLuT * kLuT; e += blockDim.x) {
      const int r = e >> 6, c = e & 63;
      X[r * kLuS + c] = (r < vk && c < vj) ? lu_load(A[(size_t)(k0 + p[r]) * dim + j0 + c]) : make_double2(0.0, 0.0);
    }
    __syncthreads();
    for (int e = tid; e < kLuT * kLuT; e += blockDim.x) {
      const int r = e >> 6, c = e & 63;
      if (r < vk && c < vj) A[(size_t)(k0 + r) * dim + j0 + c] = lu_cast<T>(X[r * kLuS + c]);
    }
    return;
  }
  // Left (rows) x Right (columns): row tile L_kk^{-1} x (P A_kj); column tile A_ik x U_kk^{-1}
  const double2* inv = dinv64 + ((size_t)(g.tile0[b] + k) * 2 + (row_tile ? 0 : 1)) * kLuT * kLuT;
  double2 acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[a][q] = make_double2(0.0, 0.0);
  for (int kc = 0; kc < kLuT; kc += kLuKc) {
    __syncthreads();
    for (int e = tid; e < kLuT * kLuKc; e += blockDim.x) {
      const int r = e / kLuKc, kk = e % kLuKc;  // Left[r][kc + kk]
      double2 lv;
      if (row_tile) lv = inv[r * kLuT + kc + kk];  // padded part: identity
      else lv = (r < vi && kc + kk < vk) ? lu_load(A[(size_t)(i0 + r) * dim + k0 + kc + kk]) : make_double2(0.0, 0.0);
      Ls[kk][r] = lv;
      const int kk2 = e / kLuT, c = e % kLuT;  // Right[kc + kk2][c]
      double2 rv;
      if (row_tile)
        rv = (kc + kk2 < vk && c < vj) ? lu_load(A[(size_t)(k0 + p[kc + kk2]) * dim + j0 + c]) : make_double2(0.0, 0.0);
      else
        rv = inv[(kc + kk2) * kLuT + c];
      Us[kk2][c] = rv;
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < kLuKc; ++kk) {
      double2 l[4], u[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) l[a] = Ls[kk][ty + 16 * a];
#pragma unroll
      for (int q = 0; q < 4; ++q) u[q] = Us[kk][tx + 16 * q];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          acc[a][q].x = fma(l[a].x, u[q].x, acc[a][q].x);
          acc[a][q].x = fma(-l[a].y, u[q].y, acc[a][q].x);
          acc[a][q].y = fma(l[a].x, u[q].y, acc[a][q].y);
          acc[a][q].y = fma(l[a].y, u[q].x, acc[a][q].y);
        }
    }
  }
  __syncthreads();  // every read of the tile (row tile: in place) precedes the stores
  const int vr = row_tile ? vk : vi, vc = row_tile ? vj : vk;
  const int c0 = row_tile ? j0 : k0;
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int r = ty + 16 * a;
    if (r >= vr) continue;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int c = tx + 16 * q;
      if (c < vc) A[(size_t)(i0 + r) * dim + c0 + c] = lu_cast<T>(acc[a][q]);
    }
  }
}

// ---- step k, part 3: trailing update A_ij -= L_ik U_kj for i, j > k ----------------------------
// 256 threads, 4 x 4 outputs each (rows ty + 16p, columns tx + 16q); the inner dimension is
// staged in two chunks of 32 (L transposed, U as is).
constexpr size_t kLuUpdateSmem = 2 * (size_t)kLuKc * kLuS * sizeof(double2);
__global__ void __launch_bounds__(256, 2) lu_update_kernel(LuGeom g, const int* pre, int k, double2* mat) {
  extern __shared__ double2 lu_smem[];
  double2(*Ls)[kLuS] = reinterpret_cast<double2(*)[kLuS]>(lu_smem);                 // Ls[kk][row] = L_ik[row][kc + kk]
  double2(*Us)[kLuS] = reinterpret_cast<double2(*)[kLuS]>(lu_smem + kLuKc * kLuS);  // Us[kk][col] = U_kj[kc + kk][col]
  const int b = lu_block_of(pre, g.n_blocks, blockIdx.x);
  const int item = blockIdx.x - pre[b];
  const int dim = g.dim[b];
  const int nt = lu_tiles(dim);
  const int nc = nt - k - 1;
  const int i = k + 1 + item / nc, j = k + 1 + item % nc;
  const int k0 = k * kLuT, i0 = i * kLuT, j0 = j * kLuT;
  const int vk = min(kLuT, dim - k0), vi = min(kLuT, dim - i0), vj = min(kLuT, dim - j0);
  double2* A = mat + g.mat_off[b];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  double2 acc[4][4];
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[p][q] = make_double2(0.0, 0.0);
  for (int kc = 0; kc < vk; kc += kLuKc) {
    __syncthreads();
    for (int e = tid; e < kLuT * kLuKc; e += blockDim.x) {
      const int r = e / kLuKc, kk = e % kLuKc;  // L: consecutive threads along the row
      Ls[kk][r] = (r < vi && kc + kk < vk) ? A[(size_t)(i0 + r) * dim + k0 + kc + kk] : make_double2(0.0, 0.0);
      const int kk2 = e / kLuT, c = e % kLuT;   // U: consecutive threads along the row
      Us[kk2][c] = (kc + kk2 < vk && c < vj) ? A[(size_t)(k0 + kc + kk2) * dim + j0 + c]
                                             : make_double2(0.0, 0.0);
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < kLuKc; ++kk) {
      double2 l[4], u[4];
#pragma unroll
      for (int p = 0; p < 4; ++p) l[p] = Ls[kk][ty + 16 * p];
#pragma unroll
      for (int q = 0; q < 4; ++q) u[q] = Us[kk][tx + 16 * q];
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          acc[p][q].x = fma(l[p].x, u[q].x, acc[p][q].x);
          acc[p][q].x = fma(-l[p].y, u[q].y, acc[p][q].x);
          acc[p][q].y = fma(l[p].x, u[q].y, acc[p][q].y);
          acc[p][q].y = fma(l[p].y, u[q].x, acc[p][q].y);
        }
    }
  }
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    const int r = ty + 16 * p;
    if (r >= vi) continue;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int c = tx + 16 * q;
      if (c >= vj) continue;
      double2* a = A + (size_t)(i0 + r) * dim + j0 + c;
      const double2 o = *a;
      *a = make_double2(o.x - acc[p][q].x, o.y - acc[p][q].y);
    }
  }
}

// Complex64 storage: the same update in FP32, as packed FMAs (FFMA2). The staged operands are laid
// out as the packed instructions consume them, L negated: Ls[kk][row] = (-l_re, -l_re, l_im, -l_im)
// and Us[kk][col] = (u_re, u_im, u_im, u_re), so each complex multiply-subtract is two FFMA2:
//   (acc_re, acc_im) += (-l_re, -l_re) * (u_re, u_im) + (l_im, -l_im) * (u_im, u_re).
// 128 threads, 8 x 4 outputs each (rows ty + 8p, columns tx + 16q): per inner index a warp issues
// 12 shared loads (16 wavefronts) for 64 FFMA2, so the FP32 pipe, not shared memory, is the bound
// (with 4 x 4 outputs it was 12 wavefronts per 32 FFMA2). Three CTAs per SM.
constexpr int kLuUpd32Threads = 128;
constexpr size_t kLuUpdateSmem32 = 2 * (size_t)kLuKc * kLuS * sizeof(float4);
__global__ void __launch_bounds__(kLuUpd32Threads, 3) lu_update32_kernel(LuGeom g, const int* pre, int k,
                                                                        float2* mat) {
  extern __shared__ float4 lu_smem32[];
  float4(*Ls)[kLuS] = reinterpret_cast<float4(*)[kLuS]>(lu_smem32);
  float4(*Us)[kLuS] = reinterpret_cast<float4(*)[kLuS]>(lu_smem32 + kLuKc * kLuS);
  const int b = lu_block_of(pre, g.n_blocks, blockIdx.x);
  const int item = blockIdx.x - pre[b];
  const int dim = g.dim[b];
  const int nt = lu_tiles(dim);
  const int nc = nt - k - 1;
  const int i = k + 1 + item / nc, j = k + 1 + item % nc;
  const int k0 = k * kLuT, i0 = i * kLuT, j0 = j * kLuT;
  const int vk = min(kLuT, dim - k0), vi = min(kLuT, dim - i0), vj = min(kLuT, dim - j0);
  float2* A = mat + g.mat_off[b];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  // the accumulators start from the C tile (its loads overlap the first staging): C - L U is
  // accumulated directly and the epilogue is a plain store
  float2 acc[8][4];
#pragma unroll
  for (int p = 0; p < 8; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int r = ty + 8 * p, c = tx + 16 * q;
      acc[p][q] = (r < vi && c < vj) ? A[(size_t)(i0 + r) * dim + j0 + c] : make_float2(0.f, 0.f);
    }
  for (int kc = 0; kc < vk; kc += kLuKc) {
    __syncthreads();
    for (int e = tid; e < kLuT * kLuKc; e += kLuUpd32Threads) {
      const int r = e / kLuKc, kk = e % kLuKc;
      const float2 l = (r < vi && kc + kk < vk) ? A[(size_t)(i0 + r) * dim + k0 + kc + kk] : make_float2(0.f, 0.f);
      Ls[kk][r] = make_float4(-l.x, -l.x, l.y, -l.y);  // negated: acc = C - L U
      const int kk2 = e / kLuT, c = e % kLuT;
      const float2 u = (kc + kk2 < vk && c < vj) ? A[(size_t)(k0 + kc + kk2) * dim + j0 + c] : make_float2(0.f, 0.f);
      Us[kk2][c] = make_float4(u.x, u.y, u.y, u.x);
    }
    __syncthreads();
#pragma unroll 2
    for (int kk = 0; kk < kLuKc; ++kk) {
      float4 l[8], u[4];
#pragma unroll
      for (int p = 0; p < 8; ++p) l[p] = Ls[kk][ty + 8 * p];
#pragma unroll
      for (int q = 0; q < 4; ++q) u[q] = Us[kk][tx + 16 * q];
#pragma unroll
      for (int p = 0; p < 8; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          acc[p][q] = __ffma2_rn(make_float2(l[p].x, l[p].y), make_float2(u[q].x, u[q].y), acc[p][q]);
          acc[p][q] = __ffma2_rn(make_float2(l[p].z, l[p].w), make_float2(u[q].z, u[q].w), acc[p][q]);
        }
    }
  }
#pragma unroll
  for (int p = 0; p < 8; ++p) {
    const int r = ty + 8 * p;
    if (r >= vi) continue;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int c = tx + 16 * q;
      if (c >= vj) continue;
      A[(size_t)(i0 + r) * dim + j0 + c] = acc[p][q];
    }
  }
}

// ---- step k, part 1b: the inverses of the factored diagonal tile k of every block ----------------
// dinv[(tile0[b] + t) * 2 + 0] = L_tt^{-1} (unit lower), [.. + 1] = U_tt^{-1}, each 64 x 64
// row-major complex64 (identity in the padded part); dinv64 the same in complex128 (the panel
// products read it; finalize keeps it only with the complex128 factors).
template <typename T>
__global__ void __launch_bounds__(256) lu_diag_inverse_kernel(LuGeom g, const int* pre, const T* mat, float2* dinv,
                                                              double2* dinv64, int* err, int step) {
  extern __shared__ double2 lu_smem[];
  double2* D = lu_smem;                // [64][kLuS] factored diagonal tile
  double2* X = lu_smem + kLuT * kLuS;  // [64][kLuS] inverse under construction
  const int b = lu_block_of(pre, g.n_blocks, blockIdx.x);
  const int t = step;  // diagonal tile `step` of every block that has one
  const int dim = g.dim[b];
  const int t0 = t * kLuT, v = min(kLuT, dim - t0);
  const T* A = mat + g.mat_off[b];
  const int tid = threadIdx.x;
  __shared__ int singular;
  if (tid == 0) singular = 0;
  for (int e = tid; e < kLuT * kLuT; e += blockDim.x) {
    const int r = e >> 6, c = e & 63;
    D[r * kLuS + c] =
        (r < v && c < v) ? lu_load(A[(size_t)(t0 + r) * dim + t0 + c]) : make_double2(r == c ? 1.0 : 0.0, 0.0);
    X[r * kLuS + c] = make_double2(r == c ? 1.0 : 0.0, 0.0);
  }
  // L X = I (unit lower): row c of X is final before rows below use it
  for (int c = 0; c < kLuT; ++c) {
    __syncthreads();
    const int rem = kLuT - 1 - c;
    for (int e = tid; e < rem * kLuT; e += blockDim.x) {
      const int r = c + 1 + e / kLuT, col = e % kLuT;
      X[r * kLuS + col] = c_sub_mul(X[r * kLuS + col], D[r * kLuS + c], X[c * kLuS + col]);
    }
  }
  __syncthreads();
  const size_t obase = (size_t)(g.tile0[b] + t) * 2 * kLuT * kLuT;
  float2* out = dinv + obase;
  for (int e = tid; e < kLuT * kLuT; e += blockDim.x) {
    const int r = e >> 6, c = e & 63;
    const double2 x = X[r * kLuS + c];
    out[e] = make_float2((float)x.x, (float)x.y);
    if (dinv64) dinv64[obase + e] = x;
    X[r * kLuS + c] = make_double2(r == c ? 1.0 : 0.0, 0.0);
  }
  // U X = I: rows from the bottom
  for (int c = kLuT - 1; c >= 0; --c) {
    __syncthreads();
    bool zero = false;
    const double2 inv = c_inv(D[c * kLuS + c], &zero);
    if (zero && tid == 0) singular = 1;
    if (tid < kLuT) X[c * kLuS + tid] = c_mul(X[c * kLuS + tid], inv);
    __syncthreads();
    for (int e = tid; e < c * kLuT; e += blockDim.x) {
      const int r = e / kLuT, col = e % kLuT;
      X[r * kLuS + col] = c_sub_mul(X[r * kLuS + col], D[r * kLuS + c], X[c * kLuS + col]);
    }
  }
  __syncthreads();
  out += kLuT * kLuT;
  for (int e = tid; e < kLuT * kLuT; e += blockDim.x) {
    const double2 x = X[(e >> 6) * kLuS + (e & 63)];
    out[e] = make_float2((float)x.x, (float)x.y);
    if (dinv64) dinv64[obase + kLuT * kLuT + e] = x;
  }
  if (tid == 0 && singular) atomicExch(err, 1);
}

// ---- apply ---------------------------------------------------------------------------------------
// z[row0[b] + r][col] = x[col][global index of block-local row (r & ~63) + piv[row0[b] + r]]
__global__ void lu_gather_kernel(int total_rows, int nmax, int nrhs, long long ld, const int* row_block,
                                 const int* row_local, const int* block_ptr, const int* particles,
                                 const int* row0, const int* piv, const double2* x, double2* z) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)total_rows * nrhs;
       e += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(e % total_rows), col = (int)(e / total_rows);
    const int b = row_block[q], r = row_local[q];
    const int src = (r & ~(kLuT - 1)) + piv[q];
    const int gi = particles[block_ptr[b] + src / nmax] * nmax + src % nmax;
    z[(size_t)col * total_rows + q] = x[(size_t)col * ld + gi];
  }
}

__global__ void lu_scatter_kernel(int total_rows, int nmax, int nrhs, long long ld, const int* row_block,
                                  const int* row_local, const int* block_ptr, const int* particles,
                                  const double2* z, double2* y) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)total_rows * nrhs;
       e += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(e % total_rows), col = (int)(e / total_rows);
    const int b = row_block[q], r = row_local[q];
    const int gi = particles[block_ptr[b] + r / nmax] * nmax + r % nmax;
    y[(size_t)col * ld + gi] = z[(size_t)col * total_rows + q];
  }
}

// One step of a sweep. Forward (upper = 0), launch s: tile rows i = s .. nt-1 of every block with
// s < nt: z_i -= L_{i,s-1} z_{s-1} (s > 0), then z_s = L_ss^{-1} z_s. Backward (upper = 1), launch
// t, s = nt - 1 - t: tile rows i = 0 .. s: z_i -= U_{i,s+1} z_{s+1} (t > 0), then z_s = U_ss^{-1} z_s.
// 256 threads: thread (row = tid >> 2, part = tid & 3) owns 16 of the 64 products of its row, all of
// whose factor loads are issued at once (the loop is fully unrolled, predicated only on the ragged
// edge); the four parts are combined by shuffles. Two blocks per SM. Right-hand sides are processed
// NC at a time (NC = 1 for a single column, else kLuCols).
// FT: float2 (the complex64 factors the solves stream) or double2 (complex128 factors, when kept).
constexpr int kLuCols = 8;
template <typename FT, int NC>
__global__ void __launch_bounds__(256, 2) lu_sweep_kernel(LuGeom g, const int* pre, int step, int upper,
                                                          const FT* lu, const FT* dinv, int nrhs,
                                                          int total_rows, double2* z) {
  __shared__ double2 zin[NC][kLuT];   // z of the eliminated tile row
  __shared__ double2 zacc[NC][kLuT];  // the diagonal tile row before its inverse is applied
  const int b = lu_block_of(pre, g.n_blocks, blockIdx.x);
  const int item = blockIdx.x - pre[b];
  const int dim = g.dim[b];
  const int nt = lu_tiles(dim);
  const int s = upper ? nt - 1 - step : step;        // diagonal tile row of this step
  const int i = upper ? item : s + item;              // tile row of this CTA
  const int e_tile = upper ? s + 1 : s - 1;           // tile row eliminated in this step
  const bool has_e = step > 0;
  const int i0 = i * kLuT, vi = min(kLuT, dim - i0);
  const int e0 = e_tile * kLuT, ve = has_e ? min(kLuT, dim - e0) : 0;
  const FT* M = lu + g.mat_off[b];
  const int tid = threadIdx.x, row = tid >> 2, part = tid & 3;
  const size_t zb = g.row0[b];
  const bool diag = i == s;
  // this thread's 16 factor entries of the eliminated tile
  FT m[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const int q = part + 4 * k;
    m[k] = (has_e && row < vi && q < ve) ? M[(size_t)(i0 + row) * dim + e0 + q] : FT{};
  }
  const FT* inv = dinv + ((size_t)(g.tile0[b] + s) * 2 + (upper ? 1 : 0)) * kLuT * kLuT + (size_t)row * kLuT;
  for (int c0 = 0; c0 < nrhs; c0 += NC) {
    const int nc = min(NC, nrhs - c0);
    __syncthreads();
    if (has_e)
      for (int e = tid; e < NC * kLuT; e += blockDim.x) {
        const int cc = e / kLuT, r = e % kLuT;
        zin[cc][r] = (cc < nc && r < ve) ? z[(size_t)(c0 + cc) * total_rows + zb + e0 + r] : make_double2(0.0, 0.0);
      }
    __syncthreads();
    double2 acc[NC];
#pragma unroll
    for (int cc = 0; cc < NC; ++cc) acc[cc] = make_double2(0.0, 0.0);
    if (has_e) {
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const double mx = m[k].x, my = m[k].y;
        const int q = part + 4 * k;
#pragma unroll
        for (int cc = 0; cc < NC; ++cc) {
          const double2 zv = zin[cc][q];
          acc[cc].x = fma(mx, zv.x, fma(-my, zv.y, acc[cc].x));
          acc[cc].y = fma(mx, zv.y, fma(my, zv.x, acc[cc].y));
        }
      }
    }
#pragma unroll
    for (int cc = 0; cc < NC; ++cc) {
      acc[cc].x += __shfl_xor_sync(0xffffffffu, acc[cc].x, 1);
      acc[cc].y += __shfl_xor_sync(0xffffffffu, acc[cc].y, 1);
      acc[cc].x += __shfl_xor_sync(0xffffffffu, acc[cc].x, 2);
      acc[cc].y += __shfl_xor_sync(0xffffffffu, acc[cc].y, 2);
    }
    if (!diag) {
      if (part == 0 && row < vi)
        for (int cc = 0; cc < nc; ++cc) {
          double2* zp = z + (size_t)(c0 + cc) * total_rows + zb + i0 + row;
          const double2 o = *zp;
          *zp = make_double2(o.x - acc[cc].x, o.y - acc[cc].y);
        }
      continue;
    }
    // diagonal tile row: r = z_s - (eliminated part), then z_s = inverse(diagonal tile) r
    if (part == 0)
      for (int cc = 0; cc < NC; ++cc) {
        double2 o = make_double2(0.0, 0.0);
        if (row < vi && cc < nc) o = z[(size_t)(c0 + cc) * total_rows + zb + i0 + row];
        zacc[cc][row] = make_double2(o.x - acc[cc].x, o.y - acc[cc].y);
      }
    __syncthreads();
    double2 out[NC];
#pragma unroll
    for (int cc = 0; cc < NC; ++cc) out[cc] = make_double2(0.0, 0.0);
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const FT wv = inv[part + 4 * k];
      const double mx = wv.x, my = wv.y;
      const int q = part + 4 * k;
#pragma unroll
      for (int cc = 0; cc < NC; ++cc) {
        const double2 zv = zacc[cc][q];
        out[cc].x = fma(mx, zv.x, fma(-my, zv.y, out[cc].x));
        out[cc].y = fma(mx, zv.y, fma(my, zv.x, out[cc].y));
      }
    }
#pragma unroll
    for (int cc = 0; cc < NC; ++cc) {
      out[cc].x += __shfl_xor_sync(0xffffffffu, out[cc].x, 1);
      out[cc].y += __shfl_xor_sync(0xffffffffu, out[cc].y, 1);
      out[cc].x += __shfl_xor_sync(0xffffffffu, out[cc].x, 2);
      out[cc].y += __shfl_xor_sync(0xffffffffu, out[cc].y, 2);
    }
    if (part == 0 && row < vi)
      for (int cc = 0; cc < nc; ++cc) z[(size_t)(c0 + cc) * total_rows + zb + i0 + row] = out[cc];
  }
}

// ---- both sweeps of a one-column apply in ONE launch ------------------------------------------
// Each CTA takes a ticket from a global counter when it starts; ticket t names one tile row: the
// forward sweep's rows first (ordered by tile row, then block), then the backward sweep's rows
// (ordered by distance from the block's last tile row, then block). The CTA computes its whole row,
// z_i = D_i^{-1} (z_i - sum_j F_ij z_j) over the finished rows j (forward: j < i, F = L; backward:
// j > i, F = U; D_i^{-1} the inverse of the diagonal tile), consuming the rows as its block's
// finished-row counter announces them, then publishes row i by raising that counter. Rows of one
// block finish strictly in order (row i needs row i-1), so one counter per block and sweep carries
// every dependency, and a backward row starts once its block's forward counter reaches nt. Every
// row a CTA waits for has a smaller ticket, held by a CTA that is already running, so the launch
// progresses whatever order the hardware schedules CTAs in. The factor streams once, as in the
// step-per-launch sweep, but without one launch (and one tail) per tile row.
// Waits are bounded in time; a wait that runs out raises the abort word, after which every CTA
// writes NaN for its row and publishes at once, so the launch ends quickly and the solve reports a
// non-finite result. Arithmetic is float64 (the factor entries are widened as they are read); the
// sum over j runs in the order of the sweep, not the step-per-launch order, so results differ from
// that kernel's only by rounding.
struct LuSolveArgs {
  LuGeom g;
  const int2* order;  // [2 * n_tiles]: (block, tile row) of each ticket
  int n_tiles;
  double2* z;
  int* sync;  // [0] ticket, [1] abort, [2, 2 + n_blocks) forward rows done, then backward rows done
  unsigned long long wait_ns;
  int stall;  // test hook: the CTA of ticket 0 never delivers its row
};
constexpr int kLuBatch = 32;     // finished tile rows whose z is staged in shared memory at once
constexpr int kLuInvS = kLuT + 4;  // row stride of the staged inverse (conflict-free 8/16 B reads)
template <typename FT>
constexpr size_t lu_solve_smem() {
  return (size_t)kLuT * kLuInvS * sizeof(FT) + (size_t)(kLuBatch + 1) * kLuT * sizeof(double2);
}

__device__ __forceinline__ int lu_ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long lu_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Waits until *done > need and returns the count seen, or returns -1 once the abort word is set or
// `bound_ns` has passed (raising the abort word).
__device__ int lu_wait_rows(const int* done, int need, int* abort_word, unsigned long long bound_ns) {
  unsigned long long t0 = 0;
#pragma unroll 1
  for (unsigned spin = 0;; ++spin) {
    const int v = lu_ld_acquire(done);
    if (v > need) return v;
    if (lu_ld_acquire(abort_word)) return -1;
    if (spin == 0) {
      t0 = lu_ns();
    } else if ((spin & 15) == 0 && lu_ns() - t0 > bound_ns) {
      atomicExch(abort_word, 1);
      return -1;
    }
    if (spin >= 32) __nanosleep(64);  // the first polls spin: a row usually arrives within a few us
  }
}

template <typename FT>
__device__ __forceinline__ void lu_row_products(const FT (&m)[16], const double2* zt, int part, double& ax,
                                                double& ay) {
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const double mx = m[k].x, my = m[k].y;
    const double2 zv = zt[part + 4 * k];
    ax = fma(mx, zv.x, fma(-my, zv.y, ax));
    ay = fma(mx, zv.y, fma(my, zv.x, ay));
  }
}

// entries 2 (part + 4k) and 2 (part + 4k) + 1 of a complex64 tile row, as float4 pairs
__device__ __forceinline__ void lu_pair_products(const float4 (&m)[8], const double2* zt, int part, double& ax,
                                                 double& ay) {
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int q = 2 * (part + 4 * k);
    const double2 z0 = zt[q], z1 = zt[q + 1];
    const double m0x = m[k].x, m0y = m[k].y, m1x = m[k].z, m1y = m[k].w;
    ax = fma(m0x, z0.x, fma(-m0y, z0.y, ax));
    ay = fma(m0x, z0.y, fma(m0y, z0.x, ay));
    ax = fma(m1x, z1.x, fma(-m1y, z1.y, ax));
    ay = fma(m1x, z1.y, fma(m1y, z1.x, ay));
  }
}

template <typename FT>
__global__ void __launch_bounds__(256, 2) lu_solve_kernel(LuSolveArgs a, const FT* lu, const FT* dinv) {
  extern __shared__ __align__(16) unsigned char lu_solve_raw[];
  FT* winv = reinterpret_cast<FT*>(lu_solve_raw);  // [64][kLuInvS] the diagonal tile's inverse
  double2* zs = reinterpret_cast<double2*>(lu_solve_raw + (size_t)kLuT * kLuInvS * sizeof(FT));  // [kLuBatch][64]
  double2* zrow = zs + kLuBatch * kLuT;  // [64] this row's right-hand side
  __shared__ int s_ticket, s_avail;
  const int tid = threadIdx.x, row = tid >> 2, part = tid & 3;
  if (tid == 0) s_ticket = atomicAdd(a.sync, 1);
  __syncthreads();
  const int t = s_ticket;
  if (t >= 2 * a.n_tiles || (a.stall && t == 0)) return;
  const bool upper = t >= a.n_tiles;
  const int2 bi = a.order[t];
  const int b = bi.x, i = bi.y;
  const int dim = a.g.dim[b], nt = lu_tiles(dim);
  const int i0 = i * kLuT, vi = min(kLuT, dim - i0);
  // this thread's factor row (rows past a ragged edge re-read the last row; never stored)
  const FT* M = lu + a.g.mat_off[b] + (size_t)(i0 + min(row, vi - 1)) * dim;
  double2* zb = a.z + a.g.row0[b];
  int* abort_word = a.sync + 1;
  int* done = a.sync + 2 + (upper ? a.g.n_blocks : 0) + b;
  {
    const FT* inv = dinv + ((size_t)(a.g.tile0[b] + i) * 2 + (upper ? 1 : 0)) * kLuT * kLuT;
    for (int e = tid; e < kLuT * kLuT; e += blockDim.x) winv[(e >> 6) * kLuInvS + (e & 63)] = inv[e];
  }
  const int ndep = upper ? nt - 1 - i : i;
  bool ok = true;
  if (upper) {  // the backward sweep reads the block's finished forward sweep
    if (tid == 0) s_avail = lu_wait_rows(a.sync + 2 + b, nt - 1, abort_word, a.wait_ns);
    __syncthreads();
    ok = s_avail >= 0;
    __syncthreads();
  }
  double ax = 0.0, ay = 0.0;
  int c = 0;  // finished rows consumed
  while (ok && c < ndep) {
    // The factor entries of the next dependency do not depend on z: they are loaded before the
    // wait for its row, so a row that arrives late costs the chain no DRAM latency.
    float4 pre[8];
    if constexpr (sizeof(FT) == 8) {
      const float4* M4 = reinterpret_cast<const float4*>(M);
      const int j0 = (upper ? nt - 1 - c : c) * kLuT;
      const int vj = min(kLuT, dim - j0);
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int q = 2 * (part + 4 * k);
        pre[k] = q < vj ? M4[(j0 + q) >> 1] : make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
    if (tid == 0) s_avail = lu_wait_rows(done, c, abort_word, a.wait_ns);
    __syncthreads();
    if (s_avail < 0) {
      ok = false;
      break;
    }
    const int avail = min(ndep, s_avail);
    for (int c0 = c; c0 < avail; c0 += kLuBatch) {
      const int nb = min(kLuBatch, avail - c0);
      for (int e = tid; e < nb * kLuT; e += blockDim.x) {
        const int cc = c0 + (e >> 6);
        const int r = (upper ? nt - 1 - cc : cc) * kLuT + (e & 63);
        zs[e] = r < dim ? __ldcg(zb + r) : make_double2(0.0, 0.0);
      }
      __syncthreads();
      if constexpr (sizeof(FT) == 8) {
        // complex64 factors as pairs (float4): thread part owns entries 2 (part + 4k) and +1; two
        // tiles' loads in flight. Block orders are even, so a pair never straddles the edge.
        const float4* M4 = reinterpret_cast<const float4*>(M);
        int u = 0;
        if (c0 == c) {  // the prefetched tile
          lu_pair_products(pre, zs, part, ax, ay);
          u = 1;
        }
#pragma unroll 1
        for (; u + 1 < nb; u += 2) {
          const int ja = (upper ? nt - 1 - (c0 + u) : c0 + u) * kLuT;
          const int jb = (upper ? nt - 2 - (c0 + u) : c0 + u + 1) * kLuT;
          const int va = min(kLuT, dim - ja), vb = min(kLuT, dim - jb);
          float4 m0[8], m1[8];
#pragma unroll
          for (int k = 0; k < 8; ++k) {
            const int q = 2 * (part + 4 * k);
            m0[k] = q < va ? M4[(ja + q) >> 1] : make_float4(0.f, 0.f, 0.f, 0.f);
            m1[k] = q < vb ? M4[(jb + q) >> 1] : make_float4(0.f, 0.f, 0.f, 0.f);
          }
          lu_pair_products(m0, zs + u * kLuT, part, ax, ay);
          lu_pair_products(m1, zs + (u + 1) * kLuT, part, ax, ay);
        }
        if (u < nb) {
          const int j0 = (upper ? nt - 1 - (c0 + u) : c0 + u) * kLuT;
          const int vj = min(kLuT, dim - j0);
          float4 m0[8];
#pragma unroll
          for (int k = 0; k < 8; ++k) {
            const int q = 2 * (part + 4 * k);
            m0[k] = q < vj ? M4[(j0 + q) >> 1] : make_float4(0.f, 0.f, 0.f, 0.f);
          }
          lu_pair_products(m0, zs + u * kLuT, part, ax, ay);
        }
      } else {
#pragma unroll 1
        for (int u = 0; u < nb; ++u) {
          const int j0 = (upper ? nt - 1 - (c0 + u) : c0 + u) * kLuT;
          const int vj = min(kLuT, dim - j0);
          FT m0[16];
#pragma unroll
          for (int k = 0; k < 16; ++k) {
            const int q = part + 4 * k;
            m0[k] = q < vj ? M[j0 + q] : FT{};
          }
          lu_row_products(m0, zs + u * kLuT, part, ax, ay);
        }
      }
      __syncthreads();
    }
    c = avail;
  }
  ax += __shfl_xor_sync(0xffffffffu, ax, 1);
  ay += __shfl_xor_sync(0xffffffffu, ay, 1);
  ax += __shfl_xor_sync(0xffffffffu, ax, 2);
  ay += __shfl_xor_sync(0xffffffffu, ay, 2);
  if (ok) {
    if (part == 0) {  // rows past a ragged edge stage zero (their clamped products are not theirs)
      const double2 o = row < vi ? __ldcg(zb + i0 + row) : make_double2(0.0, 0.0);
      zrow[row] = row < vi ? make_double2(o.x - ax, o.y - ay) : make_double2(0.0, 0.0);
    }
    __syncthreads();
    double ox = 0.0, oy = 0.0;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const FT w = winv[row * kLuInvS + part + 4 * k];
      const double2 zv = zrow[part + 4 * k];
      const double wx = w.x, wy = w.y;
      ox = fma(wx, zv.x, fma(-wy, zv.y, ox));
      oy = fma(wx, zv.y, fma(wy, zv.x, oy));
    }
    ox += __shfl_xor_sync(0xffffffffu, ox, 1);
    oy += __shfl_xor_sync(0xffffffffu, oy, 1);
    ox += __shfl_xor_sync(0xffffffffu, ox, 2);
    oy += __shfl_xor_sync(0xffffffffu, oy, 2);
    if (part == 0 && row < vi) __stcg(zb + i0 + row, make_double2(ox, oy));
  } else if (part == 0 && row < vi) {
    __stcg(zb + i0 + row, make_double2(__longlong_as_double(0x7ff8000000000000ll),
                                       __longlong_as_double(0x7ff8000000000000ll)));
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) {  // release: the row's stores (ordered before the barrier) precede the count
    __threadfence();
    atomicMax(done, upper ? nt - i : i + 1);
  }
}

}  // namespace yasf
