// Test harness (not part of the product): exposes the large-molecule path's
// tcgen05/TMA BF16 GEMM (sparrow_b200/csrc/tc_gemm.cuh) on raw device
// pointers, so tests/test_gpu_tc_gemm.py can check it against an FP32
// product of the same BF16 terms.
#include <cuda_runtime.h>

#include <string>

#include "../../sparrow_b200/csrc/tc_gemm.cuh"

// T: nterms stacked Np x Np BF16 matrices; C: Np x ldc FP32; err: one
// device word.  Returns 0 on success, else the CUDA error code (a host-side
// argument error is cudaErrorInvalidValue).
extern "C" int tc_gemm_probe(const void* T, int nterms, int Np, const int* a_term, const int* b_term, int nseg,
                             float* C, int ldc, unsigned* err) {
  std::string msg;
  cudaError_t e = sgb::tc::gemm_terms(static_cast<const __nv_bfloat16*>(T), nterms, Np, a_term, b_term, nseg, C, ldc,
                                      err, 0, msg);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  return (int)e;
}

// Tile width the launcher picks for Np on this device.
extern "C" int tc_gemm_tile_n(int Np) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sgb::tc::pick_bn(Np, sms);
}
