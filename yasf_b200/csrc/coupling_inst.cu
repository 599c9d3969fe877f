// Explicit instantiation of the coupling kernels for one lmax. The build compiles this file
// once per lmax in [1, 8] with -DYASF_INST_L=<lmax> so the per-lmax kernels compile in parallel.
#include "coupling.cuh"

#ifndef YASF_INST_L
#error "compile with -DYASF_INST_L=<lmax>"
#endif

namespace yasf {

template <>
cudaError_t launch_contract<YASF_INST_L>(int precision, bool regular, const ContractArgs& a,
                                          int tiles, int chunks, int threads,
                                          cudaStream_t stream) {
  constexpr int L = YASF_INST_L;
  constexpr int NB64 = num_bundles(L, false), NB32 = num_bundles(L, true);
  const bool c64 = precision == YASF_C64 && !regular;
  const dim3 grid(tiles, chunks, c64 ? NB32 : NB64);
  const size_t stage64 = 2 * (size_t)max_bundle_stream<L, NB64>() * sizeof(double2);
  const size_t stage32 = 2 * (size_t)max_bundle_stream<L, NB32>() * sizeof(float4);
  cudaError_t e;
  if (regular) {
    e = cudaFuncSetAttribute(contract_kernel<L, double, true>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stage64);
    if (e != cudaSuccess) return e;
    YASF_COUNTED(contract_kernel<L, double, true><<<grid, threads, stage64, stream>>>(a));
  } else if (precision == YASF_C64) {
    e = cudaFuncSetAttribute(contract_kernel<L, float, false>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stage32);
    if (e != cudaSuccess) return e;
    YASF_COUNTED(contract_kernel<L, float, false><<<grid, threads, stage32, stream>>>(a));
  } else {
    e = cudaFuncSetAttribute(contract_kernel<L, double, false>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stage64);
    if (e != cudaSuccess) return e;
    YASF_COUNTED(contract_kernel<L, double, false><<<grid, threads, stage64, stream>>>(a));
  }
  return cudaGetLastError();
}

template <>
cudaError_t launch_grouped_contract<YASF_INST_L>(int precision, const GroupedContractArgs& g, int blocks,
                                                 cudaStream_t stream) {
  constexpr int L = YASF_INST_L;
  const size_t stage = precision == YASF_C64
                           ? 2 * (size_t)max_bundle_stream<L, num_bundles(L, true)>() * sizeof(float4)
                           : 2 * (size_t)max_bundle_stream<L, num_bundles(L, false)>() * sizeof(double2);
  cudaError_t e;
  if (precision == YASF_C64) {
    e = cudaFuncSetAttribute(grouped_contract_kernel<L, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)stage);
    if (e != cudaSuccess) return e;
    YASF_COUNTED(grouped_contract_kernel<L, float><<<blocks, 128, stage, stream>>>(g));
  } else {
    e = cudaFuncSetAttribute(grouped_contract_kernel<L, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)stage);
    if (e != cudaSuccess) return e;
    YASF_COUNTED(grouped_contract_kernel<L, double><<<blocks, 128, stage, stream>>>(g));
  }
  return cudaGetLastError();
}

template <>
int contract_resident_blocks<YASF_INST_L>(int precision, int threads) {
  constexpr int L = YASF_INST_L;
  const size_t stage = precision == YASF_C64
                           ? 2 * (size_t)max_bundle_stream<L, num_bundles(L, true)>() * sizeof(float4)
                           : 2 * (size_t)max_bundle_stream<L, num_bundles(L, false)>() * sizeof(double2);
  int blocks = 0;
  cudaError_t e;
  if (precision == YASF_C64) {
    e = cudaFuncSetAttribute(contract_kernel<L, float, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stage);
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, contract_kernel<L, float, false>, threads, stage);
  } else {
    e = cudaFuncSetAttribute(contract_kernel<L, double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stage);
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, contract_kernel<L, double, false>, threads, stage);
  }
  return (e == cudaSuccess && blocks > 0) ? blocks : 2;
}

}  // namespace yasf
