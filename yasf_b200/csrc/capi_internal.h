// Internal host-side declarations shared by the C-ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "coupling.cuh"

// One V-stream layout: how a source's stream is split into bundles, and the source-side term lists
// (CSR over the stream's entries) that vbuild evaluates.
struct yasf_stream_layout {
  int n_bundles = 0;
  int bundle_begin[8] = {0};
  int bundle_len[8] = {0};
  int total_entries = 0;          // per source, all bundles (padded)
  long long total_terms = 0;
  int* d_entry_ptr = nullptr;
  int* d_term_n2 = nullptr;
  double2* d_term_coef = nullptr;
  bool owns = true;               // false: the device arrays belong to the other layout
};

struct yasf_plan {
  int lmax = 0;
  int nmax = 0;
  int device = -1;
  // [0]: the float64 kernels (and the regular-Bessel C_sca kernel), [1]: the complex64 kernel;
  // the same arrays when both use the same bundle count
  yasf_stream_layout stream[2];
  const yasf_stream_layout& layout(int precision) const { return stream[precision == YASF_C64 ? 1 : 0]; }
  // device arrays
  yasf::LegendreTables* d_leg = nullptr;
  // nonzero (n1, n2, p) terms for explicit block assembly, CSR over (n1, n2)
  int* d_pair_ptr = nullptr;      // [nmax*nmax + 1]
  int* d_pair_p = nullptr;        // p of each term
  double2* d_pair_coef = nullptr; // A[n2][n1][p]
  long long pair_terms = 0;
  // direct-form generation terms of the tau blocks Wa (a5) and Wb (b5) for the tensor-core panel,
  // one fixed list per generator thread ([term][thread]); null when lmax > 6
  float* d_gen_c1 = nullptr;       // panel generation coefficients [slot][gen thread]
  unsigned* d_gen_meta = nullptr;  // panel pair-table byte offsets [slot][gen thread]
  unsigned* d_gen_dst = nullptr;   // panel store and phase offsets [3][step][gen thread]
  // float64 dense multi-column path (lmax <= 6): chunks of 32 entry/mirror items and their terms
  int4* d_dgen_chunks = nullptr;
  int2* d_dgen_items = nullptr;
  double* d_dgen_coef = nullptr;
  int dgen_chunks = 0;
};

namespace yasf {

void set_cuda_error(cudaError_t e);

void set_error_text(const std::string& s);

#define YASF_CUDA_TRY(expr)                   \
  do {                                        \
    cudaError_t _e = (expr);                  \
    if (_e != cudaSuccess) {                  \
      ::yasf::set_cuda_error(_e);             \
      return YASF_ERR_CUDA;                   \
    }                                         \
  } while (0)

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Coupling launch geometry and workspace layout for one matvec column.
struct CouplingLayout {
  int threads = 128;
  int tiles = 1;
  int chunks = 1;
  int sources_per_chunk = 1;
  size_t v_bytes = 0;        // stream buffer
  size_t partial_bytes = 0;  // chunk partial sums
  size_t dot_bytes = 0;      // block sums of the bilinear form
  size_t total = 0;
};

CouplingLayout coupling_layout(const yasf_plan* plan, int n_particles, int precision);

// Launch the full coupling pipeline for one column (vbuild, contract, reduce).
// mode: 0 -> y = W x, 1 -> y = x - T (.) W x, 2 -> block sums of conj(x) (.) W_reg x.
// cutoff2 >= 0 keeps only the pairs within sqrt(cutoff2) of each other (near-field variant).
int coupling_column(const yasf_plan* plan, int n_particles, const double* positions, double k,
                    const double* tmat, const double* x, double* y, int precision, int mode,
                    void* workspace, size_t workspace_bytes, cudaStream_t stream,
                    double cutoff2 = -1.0);

int dispatch_contract(int lmax, int precision, bool regular, const ContractArgs& a, int tiles,
                      int chunks, int threads, cudaStream_t stream);

// Resident blocks per SM of the contraction kernel for (lmax, precision, threads per block).
int resident_blocks(int lmax, int precision, int threads);

int validate_coupling(const yasf_plan* plan, int n_particles, const double* positions,
                      double k, int precision);

// YASF_OK when `device` is the current CUDA device, else YASF_ERR_INVALID_ARGUMENT with an error
// text (objects' device memory must not be used with another device current).
int check_current_device(int device);

// Wait bounds and the withheld role of the next launches from this host thread (set by
// yasf_test_stall; defaults: nothing withheld, 2^22 polls, one second).
struct StallHook {
  int role = YASF_STALL_NONE;
  int contract_polls = 1 << 22;
  unsigned long long panel_wait_ns = 1000000000ull;
};
const StallHook& stall_hook();

// Tile shapes of the next launches and workspace queries from this host thread (set by
// yasf_set_tiles; 0 = the built-in rule): waves of resident blocks the contraction's source chunks
// are sized for, columns per tile of the float64 dense panel, column groups per tensor-core panel
// block.
struct TileConfig {
  int contract_waves = 0;
  int dpanel_cols = 0;
  int panel_groups = 0;
};
const TileConfig& tile_config();

int panel_build_terms(int L, const double* ab5, std::vector<float>& coef, std::vector<unsigned>& goff,
                      std::vector<unsigned>& dst);
int dpanel_build_items(int L, const double* ab5, std::vector<int4>& chunks, std::vector<int2>& items,
                       std::vector<double>& term_coef);

}  // namespace yasf
