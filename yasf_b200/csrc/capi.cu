// C-ABI: library status, translation plan, coupling matvec, cross-section reductions.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <atomic>
#include <mutex>
#include <new>

#include "capi_internal.h"

namespace yasf {

static thread_local std::string g_last_error;
static std::atomic<unsigned long long> g_launches{0};
static thread_local StallHook g_stall;
static thread_local TileConfig g_tiles;

const StallHook& stall_hook() { return g_stall; }
const TileConfig& tile_config() { return g_tiles; }

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

void set_cuda_error(cudaError_t e) { g_last_error = cudaGetErrorString(e); }
void set_error_text(const std::string& s) { g_last_error = s; }

template <int L>
cudaError_t launch_contract(int precision, bool regular, const ContractArgs& a, int tiles,
                            int chunks, int threads, cudaStream_t stream);

int dispatch_contract(int lmax, int precision, bool regular, const ContractArgs& a, int tiles,
                      int chunks, int threads, cudaStream_t stream) {
  cudaError_t e = cudaErrorInvalidValue;
  switch (lmax) {
    case 1: e = launch_contract<1>(precision, regular, a, tiles, chunks, threads, stream); break;
    case 2: e = launch_contract<2>(precision, regular, a, tiles, chunks, threads, stream); break;
    case 3: e = launch_contract<3>(precision, regular, a, tiles, chunks, threads, stream); break;
    case 4: e = launch_contract<4>(precision, regular, a, tiles, chunks, threads, stream); break;
    case 5: e = launch_contract<5>(precision, regular, a, tiles, chunks, threads, stream); break;
    case 6: e = launch_contract<6>(precision, regular, a, tiles, chunks, threads, stream); break;
    case 7: e = launch_contract<7>(precision, regular, a, tiles, chunks, threads, stream); break;
    case 8: e = launch_contract<8>(precision, regular, a, tiles, chunks, threads, stream); break;
    default: return YASF_ERR_UNSUPPORTED;
  }
  YASF_CUDA_TRY(e);
  return YASF_OK;
}

static int sm_count_of(int device) {
  static std::mutex mu;
  static int cached[64] = {0};
  std::lock_guard<std::mutex> lock(mu);
  if (device < 0 || device >= 64) return 148;
  if (cached[device] == 0) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || v <= 0)
      v = 148;
    cached[device] = v;
  }
  return cached[device];
}

template <int L>
int contract_resident_blocks(int precision, int threads);

// Resident contraction blocks per SM for (lmax, precision, threads), from the occupancy query
// (cached per device state of this process).
int resident_blocks(int lmax, int precision, int threads) {
  static std::mutex mu;
  static int cache[YASF_LMAX_MAX + 1][2][5] = {};
  const int pi = precision == YASF_C64 ? 1 : 0, wi = std::min(4, std::max(1, threads / 32));
  std::lock_guard<std::mutex> lock(mu);
  int& c = cache[lmax][pi][wi];
  if (c == 0) {
    switch (lmax) {
      case 1: c = contract_resident_blocks<1>(precision, threads); break;
      case 2: c = contract_resident_blocks<2>(precision, threads); break;
      case 3: c = contract_resident_blocks<3>(precision, threads); break;
      case 4: c = contract_resident_blocks<4>(precision, threads); break;
      case 5: c = contract_resident_blocks<5>(precision, threads); break;
      case 6: c = contract_resident_blocks<6>(precision, threads); break;
      case 7: c = contract_resident_blocks<7>(precision, threads); break;
      case 8: c = contract_resident_blocks<8>(precision, threads); break;
      default: c = 2;
    }
  }
  return c;
}

CouplingLayout coupling_layout(const yasf_plan* plan, int n_particles, int precision) {
  CouplingLayout lay;
  // partial sums: complex at the kernel's precision; V stream: 16-byte entries at both precisions
  // (complex64 entries carry (re, im, -im, re) for the packed FMAs)
  const size_t csize = (precision == YASF_C64) ? sizeof(float2) : sizeof(double2);
  const size_t vsize = (precision == YASF_C64) ? sizeof(float4) : sizeof(double2);
  const int N = n_particles;
  // Receivers per block: whole warps, at most 4, one receiver per thread (two in complex64).
  const int rpt = precision == YASF_C64 ? kC64Receivers : 1;
  const int warps = std::min(4, std::max(1, (N + 32 * rpt - 1) / (32 * rpt)));
  lay.threads = 32 * warps;
  lay.tiles = (N + lay.threads * rpt - 1) / (lay.threads * rpt);
  const int sms = sm_count_of(plan->device);
  // Two full waves of resident blocks (or the thread's tile configuration); the source loop is
  // split into chunks to get there.
  const int waves = tile_config().contract_waves > 0 ? tile_config().contract_waves : 2;
  const long long want = (long long)waves * resident_blocks(plan->lmax, precision, lay.threads) * sms;
  const yasf_stream_layout& sl = plan->layout(precision);
  const long long base = (long long)lay.tiles * sl.n_bundles;
  int chunks = (int)std::max<long long>(1, (want + base - 1) / base);
  chunks = std::min(chunks, N);
  // Cap the partial-sum buffer at 1 GiB.
  const size_t per_chunk = (size_t)N * plan->nmax * csize;
  while (chunks > 1 && per_chunk * chunks > (1ull << 30)) --chunks;
  lay.sources_per_chunk = (N + chunks - 1) / chunks;
  lay.chunks = (N + lay.sources_per_chunk - 1) / lay.sources_per_chunk;
  auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
  lay.v_bytes = up((size_t)N * sl.total_entries * vsize);
  lay.partial_bytes = up(per_chunk * lay.chunks);
  lay.dot_bytes = up(1024 * sizeof(double2) + 256);  // block sums + the stage-timeout word
  lay.total = lay.v_bytes + lay.partial_bytes + lay.dot_bytes;
  return lay;
}

int validate_coupling(const yasf_plan* plan, int n_particles, const double* positions, double k,
                      int precision) {
  if (!plan || !positions || n_particles <= 0) return YASF_ERR_INVALID_ARGUMENT;
  if (precision != YASF_C128 && precision != YASF_C64) return YASF_ERR_INVALID_ARGUMENT;
  if (!std::isfinite(k) || k <= 0.0) return YASF_ERR_UNSUPPORTED;
  if (reinterpret_cast<uintptr_t>(positions) & 7u) return YASF_ERR_ALIGNMENT;
  // The plan's tables live on plan->device: launching with another device current would make the
  // kernels read a different GPU's memory.
  return check_current_device(plan->device);
}

int check_current_device(int device) {
  int dev = -1;
  YASF_CUDA_TRY(cudaGetDevice(&dev));
  if (dev != device) {
    set_error_text("the current CUDA device (" + std::to_string(dev) +
                   ") is not the device the plan was created on (" + std::to_string(device) + ")");
    return YASF_ERR_INVALID_ARGUMENT;
  }
  return YASF_OK;
}

int coupling_column(const yasf_plan* plan, int n_particles, const double* positions, double k,
                    const double* tmat, const double* x, double* y, int precision, int mode,
                    void* workspace, size_t workspace_bytes, cudaStream_t stream, double cutoff2) {
  const CouplingLayout lay = coupling_layout(plan, n_particles, precision);
  if (!workspace || workspace_bytes < lay.total) return YASF_ERR_WORKSPACE;
  if (!aligned16(workspace)) return YASF_ERR_ALIGNMENT;
  char* ws = static_cast<char*>(workspace);
  void* vbuf = ws;
  void* partial = ws + lay.v_bytes;
  double2* dots = reinterpret_cast<double2*>(ws + lay.v_bytes + lay.partial_bytes);
  int* err = reinterpret_cast<int*>(dots + 1024);
  YASF_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), stream));
  const bool regular = (mode == 2);
  if (regular && precision != YASF_C128) return YASF_ERR_UNSUPPORTED;

  // 1) source side: V streams
  const yasf_stream_layout& sl = plan->layout(precision);
  VBuildArgs va{};
  va.n_particles = n_particles;
  va.nmax = plan->nmax;
  va.total_entries = sl.total_entries;
  va.n_bundles = sl.n_bundles;
  for (int b = 0; b < 8; ++b) {
    va.bundle_begin[b] = sl.bundle_begin[b];
    va.bundle_len[b] = sl.bundle_len[b];
  }
  va.entry_ptr = sl.d_entry_ptr;
  va.term_n2 = sl.d_term_n2;
  va.term_coef = sl.d_term_coef;
  va.x = reinterpret_cast<const double2*>(x);
  va.v = vbuf;
  {
    const dim3 grid((sl.total_entries + 255) / 256, std::min(n_particles, 65535));
    if (precision == YASF_C64) YASF_COUNTED(vbuild_kernel<float><<<grid, 256, 0, stream>>>(va));
    else YASF_COUNTED(vbuild_kernel<double><<<grid, 256, 0, stream>>>(va));
    YASF_CUDA_TRY(cudaGetLastError());
  }
  // 2) pair side + contraction
  ContractArgs ca{};
  ca.n_particles = n_particles;
  ca.nmax = plan->nmax;
  ca.sources_per_chunk = lay.sources_per_chunk;
  ca.k = k;
  ca.pos = positions;
  ca.v = vbuf;
  ca.leg = plan->d_leg;
  for (int b = 0; b < 8; ++b) {
    ca.bundle_begin[b] = sl.bundle_begin[b];
    ca.bundle_len[b] = sl.bundle_len[b];
  }
  ca.partial = partial;
  ca.err = err;
  ca.cutoff2 = cutoff2;
  ca.poll_limit = stall_hook().contract_polls;
  ca.stall = stall_hook().role == YASF_STALL_CONTRACT ? 1 : 0;
  int st = dispatch_contract(plan->lmax, precision, regular, ca, lay.tiles, lay.chunks,
                             lay.threads, stream);
  if (st != YASF_OK) return st;
  // 3) chunk reduction + epilogue
  const long long n_elems = (long long)n_particles * plan->nmax;
  if (mode == 2) {
    YASF_COUNTED(reduce_dot_kernel<double><<<1024, 256, 0, stream>>>(
        n_elems, lay.chunks, partial, reinterpret_cast<const double2*>(x), dots, err));
    YASF_CUDA_TRY(cudaGetLastError());
  } else {
    const int blocks = (int)std::min<long long>((n_elems + 255) / 256, 4096);
    if (precision == YASF_C64)
      YASF_COUNTED(reduce_kernel<float><<<blocks, 256, 0, stream>>>(
          n_elems, lay.chunks, partial, reinterpret_cast<const double2*>(x),
          reinterpret_cast<const double2*>(tmat), reinterpret_cast<double2*>(y), mode, err));
    else
      YASF_COUNTED(reduce_kernel<double><<<blocks, 256, 0, stream>>>(
          n_elems, lay.chunks, partial, reinterpret_cast<const double2*>(x),
          reinterpret_cast<const double2*>(tmat), reinterpret_cast<double2*>(y), mode, err));
    YASF_CUDA_TRY(cudaGetLastError());
  }
  return YASF_OK;
}

// Sum of n block partials -> out[0..1].
__global__ void final_sum_kernel(int n, const double2* parts, double* out) {
  __shared__ double sr[256], si[256];
  double re = 0.0, im = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    re += parts[i].x;
    im += parts[i].y;
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
    out[0] = sr[0];
    out[1] = si[0];
  }
}

__global__ void dotc_blocks_kernel(long long n, const double2* a, const double2* b,
                                   double2* parts) {
  __shared__ double sr[256], si[256];
  double re = 0.0, im = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double2 av = a[i], bv = b[i];
    re += av.x * bv.x + av.y * bv.y;
    im += av.x * bv.y - av.y * bv.x;
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
  if (threadIdx.x == 0) parts[blockIdx.x] = make_double2(sr[0], si[0]);
}

}  // namespace yasf

using namespace yasf;

// ------------------------------------------------------------------------------------------------
extern "C" int yasf_abi_version(void) { return YASF_ABI_VERSION; }

extern "C" const char* yasf_status_string(int status) {
  switch (status) {
    case YASF_OK: return "ok";
    case YASF_ERR_INVALID_ARGUMENT: return "invalid argument";
    case YASF_ERR_UNSUPPORTED: return "unsupported parameter";
    case YASF_ERR_ALIGNMENT: return "pointer not 16-byte aligned";
    case YASF_ERR_CUDA: return "CUDA runtime error";
    case YASF_ERR_OUT_OF_MEMORY: return "device allocation failed";
    case YASF_ERR_WORKSPACE: return "workspace too small";
    case YASF_ERR_NOT_FINITE: return "non-finite value";
    case YASF_ERR_NOT_PREPARED: return "preconditioner not prepared";
    case YASF_ERR_SCRATCH_LIMIT: return "problem exceeds the static scratch of the no-alloc call";
    default: return "unknown status";
  }
}

extern "C" const char* yasf_last_cuda_error(void) { return g_last_error.c_str(); }

extern "C" int yasf_set_tiles(int contract_waves, int dpanel_cols, int panel_groups) {
  const bool ok_w = contract_waves == 0 || contract_waves == 1 || contract_waves == 2 || contract_waves == 4 ||
                    contract_waves == 8;
  const bool ok_c = dpanel_cols == 0 || dpanel_cols == 32 || dpanel_cols == 64;
  const bool ok_g = panel_groups == 0 || panel_groups == 1 || panel_groups == 2;
  if (!ok_w || !ok_c || !ok_g) return YASF_ERR_INVALID_ARGUMENT;
  g_tiles.contract_waves = contract_waves;
  g_tiles.dpanel_cols = dpanel_cols;
  g_tiles.panel_groups = panel_groups;
  return YASF_OK;
}

extern "C" int yasf_test_stall(int role, int contract_polls, double panel_wait_seconds) {
  if (role < YASF_STALL_NONE || role > YASF_STALL_PRECOND) return YASF_ERR_INVALID_ARGUMENT;
  if (contract_polls < 0 || !(panel_wait_seconds >= 0.0) || panel_wait_seconds > 10.0)
    return YASF_ERR_INVALID_ARGUMENT;
  StallHook h;
  h.role = role;
  if (contract_polls > 0) h.contract_polls = contract_polls;
  if (panel_wait_seconds > 0.0)
    h.panel_wait_ns = std::max(1000ull, (unsigned long long)(panel_wait_seconds * 1e9));
  g_stall = h;
  return YASF_OK;
}

extern "C" unsigned long long yasf_kernel_launches(void) {
  return g_launches.load(std::memory_order_relaxed);
}

static void free_stream_layouts(yasf_plan* plan) {
  for (auto& lay : plan->stream) {
    if (!lay.owns) continue;
    cudaFree(lay.d_entry_ptr);
    cudaFree(lay.d_term_n2);
    cudaFree(lay.d_term_coef);
    lay.d_entry_ptr = nullptr;
    lay.d_term_n2 = nullptr;
    lay.d_term_coef = nullptr;
  }
}

// Build the bundle streams from the dense a5/b5 table. The stream order is the one the
// contraction kernel walks (yasf_common.cuh: bundle_stream_length).
extern "C" int yasf_plan_create(int lmax, const double* ab5, yasf_plan** out) {
  if (!out || !ab5) return YASF_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (lmax < 1 || lmax > YASF_LMAX_MAX) return YASF_ERR_UNSUPPORTED;
  const int L = lmax, nmax = nmax_of(L), P = 2 * L + 1;
  auto A = [&](int n1, int n2, int p, double* re, double* im) {
    // reference layout translation_ab5[n_source][n_receiver][p]
    const size_t idx = ((size_t)n2 * nmax + n1) * P + p;
    *re = ab5[2 * idx];
    *im = ab5[2 * idx + 1];
  };
  for (size_t i = 0; i < (size_t)nmax * nmax * P * 2; ++i)
    if (!std::isfinite(ab5[i])) return YASF_ERR_NOT_FINITE;

  yasf_plan* plan = new (std::nothrow) yasf_plan();
  if (!plan) return YASF_ERR_OUT_OF_MEMORY;
  plan->lmax = L;
  plan->nmax = nmax;
  if (cudaGetDevice(&plan->device) != cudaSuccess) {
    delete plan;
    return YASF_ERR_CUDA;
  }
  // the stream layouts of the float64 and complex64 kernels (shared when their bundle counts agree)
  std::vector<int> entry_ptr_l[2], term_n2_l[2];
  std::vector<double2> term_coef_l[2];
  for (int li = 0; li < 2; ++li) {
    yasf_stream_layout& lay = plan->stream[li];
    lay.n_bundles = num_bundles(L, li == 1);
    if (li == 1 && lay.n_bundles == plan->stream[0].n_bundles) continue;
    std::vector<int>& entry_ptr = entry_ptr_l[li];
    std::vector<int>& term_n2 = term_n2_l[li];
    std::vector<double2>& term_coef = term_coef_l[li];
    entry_ptr.assign(1, 0);
    int begin = 0;
    for (int b = 0; b < lay.n_bundles; ++b) {
      const BundleInfo bi = make_bundle(L, b, lay.n_bundles);
      lay.bundle_begin[b] = begin;
      int len = 0;
      for (int d = 0; d <= 2 * L; ++d)
        for (int p = d; p <= 2 * L; ++p)
          for (int s = 0; s < (d == 0 ? 1 : 2); ++s) {
            const int sg = s == 0 ? 1 : -1;
            for (int i = 0; i < bi.count; ++i) {
              const int m1 = bi.m1[i];
              const int m2 = m1 + sg * d;
              if (m2 < -L || m2 > L) continue;
              const int nv = valid_rows(L, m1, p);
              for (int r = 0; r < nv; ++r) {
                const int n1 = mode_index(L, row_tau(r), row_l(L, r), m1);
                for (int tau2 = 1; tau2 <= 2; ++tau2)
                  for (int l2 = std::max(1, std::abs(m2)); l2 <= L; ++l2) {
                    const int n2 = mode_index(L, tau2, l2, m2);
                    double re, im;
                    A(n1, n2, p, &re, &im);
                    if (re != 0.0 || im != 0.0) {
                      term_n2.push_back(n2);
                      term_coef.push_back(make_double2(re, im));
                    }
                  }
                entry_ptr.push_back((int)term_n2.size());
                ++len;
              }
            }
          }
      if (len != bundle_stream_length(L, b, lay.n_bundles)) {
        delete plan;
        set_error_text("internal: stream length mismatch");
        return YASF_ERR_INVALID_ARGUMENT;
      }
      if (len & 1) {  // pad to an even entry count (32-byte aligned per-source streams)
        entry_ptr.push_back((int)term_n2.size());
        ++len;
      }
      lay.bundle_len[b] = len;
      begin += len;
    }
    lay.total_entries = begin;
    lay.total_terms = (long long)term_n2.size();
  }

  // Explicit (n1, n2) term lists for block assembly.
  std::vector<int> pair_ptr(1, 0), pair_p;
  std::vector<double2> pair_coef;
  for (int n1 = 0; n1 < nmax; ++n1)
    for (int n2 = 0; n2 < nmax; ++n2) {
      for (int p = 0; p < P; ++p) {
        double re, im;
        A(n1, n2, p, &re, &im);
        if (re != 0.0 || im != 0.0) {
          pair_p.push_back(p);
          pair_coef.push_back(make_double2(re, im));
        }
      }
      pair_ptr.push_back((int)pair_p.size());
    }
  plan->pair_terms = (long long)pair_p.size();

  // Generation terms for the tensor-core panel path (lmax <= 6).
  std::vector<float> gen_c1;
  std::vector<unsigned> gen_meta, gen_dst;
  std::vector<int4> dgen_chunks;
  std::vector<int2> dgen_items;
  std::vector<double> dgen_coef;
  {
    int bst = panel_build_terms(L, ab5, gen_c1, gen_meta, gen_dst);
    if (bst == YASF_OK) bst = dpanel_build_items(L, ab5, dgen_chunks, dgen_items, dgen_coef);
    if (bst != YASF_OK) {
      delete plan;
      set_error_text("translation table does not follow the a5/b5 selection rules of the panel schedule");
      return bst;
    }
  }

  // Legendre recurrence constants (CELES normalisation).
  LegendreTables leg;
  std::memset(&leg, 0, sizeof(leg));
  for (int m = 0; m <= YASF_PMAX_MAX; ++m) {
    long double fact2m = 1.0L, dfact = 1.0L;
    for (int t = 2; t <= 2 * m; ++t) fact2m *= t;
    for (int t = 1; t <= 2 * m - 1; t += 2) dfact *= t;
    leg.start[m] = (double)(std::sqrt((2.0L * m + 1.0L) / 2.0L / fact2m) * dfact);
    for (int l = m; l < YASF_PMAX_MAX; ++l) {
      const long double a2 = (long double)(2 * l + 1) * (2 * l + 3) /
                             ((long double)(l + 1 - m) * (l + 1 + m));
      leg.alpha[l * kLegStride + m] = (double)std::sqrt(a2);
      if (l > m) {
        const long double b2 = (long double)(2 * l + 3) * (l - m) * (l + m) /
                               ((long double)(2 * l - 1) * (l + 1 - m) * (l + 1 + m));
        leg.beta[l * kLegStride + m] = (double)std::sqrt(b2);
      }
    }
  }

  auto fail = [&](cudaError_t e) {
    set_cuda_error(e);
    free_stream_layouts(plan);
    cudaFree(plan->d_leg);
    cudaFree(plan->d_pair_ptr);
    cudaFree(plan->d_pair_p);
    cudaFree(plan->d_pair_coef);
    cudaFree(plan->d_gen_c1);
    cudaFree(plan->d_gen_meta);
    cudaFree(plan->d_gen_dst);
    cudaFree(plan->d_dgen_chunks);
    cudaFree(plan->d_dgen_items);
    cudaFree(plan->d_dgen_coef);
    delete plan;
    return e == cudaErrorMemoryAllocation ? YASF_ERR_OUT_OF_MEMORY : YASF_ERR_CUDA;
  };
  cudaError_t e;
#define YASF_UPLOAD(dst, vec)                                                           \
  do {                                                                                  \
    const size_t nb = std::max<size_t>(1, (vec).size()) * sizeof((vec)[0]);           \
    if ((e = cudaMalloc(reinterpret_cast<void**>(&(dst)), nb)) != cudaSuccess) return fail(e); \
    if (!(vec).empty() &&                                                               \
        (e = cudaMemcpy((dst), (vec).data(), (vec).size() * sizeof((vec)[0]),         \
                        cudaMemcpyHostToDevice)) != cudaSuccess)                        \
      return fail(e);                                                                   \
  } while (0)
  for (int li = 0; li < 2; ++li) {
    yasf_stream_layout& lay = plan->stream[li];
    if (li == 1 && lay.n_bundles == plan->stream[0].n_bundles) {
      lay = plan->stream[0];
      lay.owns = false;
      continue;
    }
    YASF_UPLOAD(lay.d_entry_ptr, entry_ptr_l[li]);
    YASF_UPLOAD(lay.d_term_n2, term_n2_l[li]);
    YASF_UPLOAD(lay.d_term_coef, term_coef_l[li]);
  }
  YASF_UPLOAD(plan->d_pair_ptr, pair_ptr);
  YASF_UPLOAD(plan->d_pair_p, pair_p);
  YASF_UPLOAD(plan->d_pair_coef, pair_coef);
  if (!gen_c1.empty()) {
    YASF_UPLOAD(plan->d_gen_c1, gen_c1);
    YASF_UPLOAD(plan->d_gen_meta, gen_meta);
    YASF_UPLOAD(plan->d_gen_dst, gen_dst);
  }
  if (!dgen_chunks.empty()) {
    YASF_UPLOAD(plan->d_dgen_chunks, dgen_chunks);
    YASF_UPLOAD(plan->d_dgen_items, dgen_items);
    YASF_UPLOAD(plan->d_dgen_coef, dgen_coef);
    plan->dgen_chunks = (int)dgen_chunks.size();
  }
#undef YASF_UPLOAD
  if ((e = cudaMalloc(reinterpret_cast<void**>(&plan->d_leg), sizeof(LegendreTables))) != cudaSuccess)
    return fail(e);
  if ((e = cudaMemcpy(plan->d_leg, &leg, sizeof(leg), cudaMemcpyHostToDevice)) != cudaSuccess)
    return fail(e);
  *out = plan;
  return YASF_OK;
}

extern "C" int yasf_plan_destroy(yasf_plan* plan) {
  if (!plan) return YASF_OK;
  free_stream_layouts(plan);
  cudaFree(plan->d_leg);
  cudaFree(plan->d_pair_ptr);
  cudaFree(plan->d_pair_p);
  cudaFree(plan->d_pair_coef);
  cudaFree(plan->d_gen_c1);
  cudaFree(plan->d_gen_meta);
  cudaFree(plan->d_gen_dst);
  cudaFree(plan->d_dgen_chunks);
  cudaFree(plan->d_dgen_items);
  cudaFree(plan->d_dgen_coef);
  delete plan;
  return YASF_OK;
}

extern "C" int yasf_plan_check_table(int lmax, const double* ab5) {
  if (!ab5) return YASF_ERR_INVALID_ARGUMENT;
  if (lmax < 1 || lmax > YASF_LMAX_MAX) return YASF_ERR_UNSUPPORTED;
  const int nmax = nmax_of(lmax), P = 2 * lmax + 1;
  for (size_t i = 0; i < (size_t)nmax * nmax * P * 2; ++i)
    if (!std::isfinite(ab5[i])) return YASF_ERR_NOT_FINITE;
  std::vector<float> gen_c1;
  std::vector<unsigned> gen_meta, gen_dst;
  std::vector<int4> dgen_chunks;
  std::vector<int2> dgen_items;
  std::vector<double> dgen_coef;
  int st = panel_build_terms(lmax, ab5, gen_c1, gen_meta, gen_dst);
  if (st == YASF_OK) st = dpanel_build_items(lmax, ab5, dgen_chunks, dgen_items, dgen_coef);
  if (st != YASF_OK)
    set_error_text("translation table does not follow the a5/b5 selection rules of the panel schedule");
  return st;
}

extern "C" int yasf_plan_info(const yasf_plan* plan, int* nmax, long long* stream_entries,
                              long long* source_terms) {
  if (!plan) return YASF_ERR_INVALID_ARGUMENT;
  if (nmax) *nmax = plan->nmax;
  if (stream_entries) *stream_entries = plan->stream[0].total_entries;
  if (source_terms) *source_terms = plan->stream[0].total_terms;
  return YASF_OK;
}

extern "C" int yasf_coupling_workspace_size(const yasf_plan* plan, int n_particles, int nrhs,
                                            int precision, size_t* bytes) {
  if (!plan || !bytes || n_particles <= 0 || nrhs <= 0) return YASF_ERR_INVALID_ARGUMENT;
  if (precision != YASF_C128 && precision != YASF_C64) return YASF_ERR_INVALID_ARGUMENT;
  *bytes = coupling_layout(plan, n_particles, precision).total;
  return YASF_OK;
}

static int matvec_common(const yasf_plan* plan, int n_particles, const double* positions,
                         double k, const double* tmat, const double* x, double* y, int nrhs,
                         long long ld, int precision, int mode, void* workspace,
                         size_t workspace_bytes, void* stream, double cutoff2 = -1.0) {
  int st = validate_coupling(plan, n_particles, positions, k, precision);
  if (st != YASF_OK) return st;
  if (!x || !y || nrhs <= 0) return YASF_ERR_INVALID_ARGUMENT;
  if (mode == 1 && !tmat) return YASF_ERR_INVALID_ARGUMENT;
  const long long n = (long long)n_particles * plan->nmax;
  if (nrhs > 1 && ld < n) return YASF_ERR_INVALID_ARGUMENT;
  if (!aligned16(x) || !aligned16(y) || (tmat && !aligned16(tmat))) return YASF_ERR_ALIGNMENT;
  if (x == y) return YASF_ERR_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  for (int c = 0; c < nrhs; ++c) {
    st = coupling_column(plan, n_particles, positions, k, tmat, x + 2 * ld * c, y + 2 * ld * c,
                         precision, mode, workspace, workspace_bytes, s, cutoff2);
    if (st != YASF_OK) return st;
  }
  return YASF_OK;
}

extern "C" int yasf_coupling_matvec_nearfield(const yasf_plan* plan, int n_particles,
                                              const double* positions, double k_medium,
                                              double near_field_radius, const double* x, double* y,
                                              int nrhs, long long ld, int precision, void* workspace,
                                              size_t workspace_bytes, void* stream) {
  if (!(near_field_radius >= 0.0) || !std::isfinite(near_field_radius)) return YASF_ERR_INVALID_ARGUMENT;
  return matvec_common(plan, n_particles, positions, k_medium, nullptr, x, y, nrhs, ld, precision, 0,
                       workspace, workspace_bytes, stream, near_field_radius * near_field_radius);
}

extern "C" int yasf_coupling_matvec(const yasf_plan* plan, int n_particles,
                                    const double* positions, double k_medium, const double* x,
                                    double* y, int nrhs, long long ld, int precision,
                                    void* workspace, size_t workspace_bytes, void* stream) {
  return matvec_common(plan, n_particles, positions, k_medium, nullptr, x, y, nrhs, ld,
                       precision, 0, workspace, workspace_bytes, stream);
}

extern "C" int yasf_master_matvec(const yasf_plan* plan, int n_particles, const double* positions,
                                  double k_medium, const double* tmat, const double* x, double* y,
                                  int nrhs, long long ld, int precision, void* workspace,
                                  size_t workspace_bytes, void* stream) {
  return matvec_common(plan, n_particles, positions, k_medium, tmat, x, y, nrhs, ld, precision,
                       1, workspace, workspace_bytes, stream);
}

extern "C" int yasf_scattering_bilinear(const yasf_plan* plan, int n_particles,
                                        const double* positions, double k_medium, const double* b,
                                        double* out, void* workspace, size_t workspace_bytes,
                                        void* stream) {
  int st = validate_coupling(plan, n_particles, positions, k_medium, YASF_C128);
  if (st != YASF_OK) return st;
  if (!b || !out) return YASF_ERR_INVALID_ARGUMENT;
  if (!aligned16(b) || !aligned16(out)) return YASF_ERR_ALIGNMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  st = coupling_column(plan, n_particles, positions, k_medium, nullptr, b, nullptr, YASF_C128, 2,
                       workspace, workspace_bytes, s);
  if (st != YASF_OK) return st;
  const CouplingLayout lay = coupling_layout(plan, n_particles, YASF_C128);
  const double2* dots = reinterpret_cast<const double2*>(static_cast<char*>(workspace) +
                                                         lay.v_bytes + lay.partial_bytes);
  YASF_COUNTED(final_sum_kernel<<<1, 256, 0, s>>>(1024, dots, out));
  YASF_CUDA_TRY(cudaGetLastError());
  return YASF_OK;
}

extern "C" int yasf_dotc(long long n, const double* a, const double* b, double* out,
                         void* workspace, size_t workspace_bytes, void* stream) {
  if (n <= 0 || !a || !b || !out) return YASF_ERR_INVALID_ARGUMENT;
  if (!workspace || workspace_bytes < 1024 * sizeof(double2)) return YASF_ERR_WORKSPACE;
  if (!aligned16(a) || !aligned16(b) || !aligned16(out) || !aligned16(workspace))
    return YASF_ERR_ALIGNMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double2* parts = static_cast<double2*>(workspace);
  YASF_COUNTED(dotc_blocks_kernel<<<1024, 256, 0, s>>>(n, reinterpret_cast<const double2*>(a),
                                           reinterpret_cast<const double2*>(b), parts));
  YASF_CUDA_TRY(cudaGetLastError());
  YASF_COUNTED(final_sum_kernel<<<1, 256, 0, s>>>(1024, parts, out));
  YASF_CUDA_TRY(cudaGetLastError());
  return YASF_OK;
}
