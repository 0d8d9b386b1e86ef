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
// C2 (may be null): second output of a launch that splits K (the product is
// then C + C2); *ksplit_out reports the split the launcher chose.
extern "C" int tc_gemm_probe(const void* T, int nterms, int Np, const int* a_term, const int* b_term, int nseg,
                             float* C, float* C2, int ldc, unsigned* err, int* ksplit_out) {
  std::string msg;
  cudaError_t e = sgb::tc::gemm_terms(static_cast<const __nv_bfloat16*>(T), nterms, Np, a_term, b_term, nseg, C, C2,
                                      ldc, err, 0, msg, ksplit_out);
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

namespace {

// One thread waits with the GEMM's bounded barrier wait (sgb::tc::mbar_wait)
// on a fresh barrier.  arrive = 0: nothing ever arrives, so the wait must
// give up after its limit and report it; arrive = 1: the thread arrives
// first, so the wait must succeed at once.  out[0] = 1 when the wait
// succeeded, out[1] = milliseconds spent waiting.
__global__ void k_wait_probe(int arrive, unsigned* out) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    sgb::tc::mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (arrive)
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(sgb::tc::smem_u32(&bar)) : "memory");
    const unsigned long long t0 = sgb::tc::global_ns();
    const bool ok = sgb::tc::mbar_wait(&bar, 0);
    const unsigned long long t1 = sgb::tc::global_ns();
    out[0] = ok ? 1u : 0u;
    out[1] = (unsigned)((t1 - t0) / 1000000ull);
  }
}

}  // namespace

// out: two device words.  Returns 0 or the CUDA error code.
extern "C" int tc_wait_probe(int arrive, unsigned* out) {
  k_wait_probe<<<1, 32>>>(arrive, out);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  return (int)e;
}

// The bounded wait's limit in milliseconds.
extern "C" int tc_wait_limit_ms() { return (int)(sgb::tc::kWaitLimitNs / 1000000ull); }

// The launcher's plan for Np on a device with `sms` SMs (host logic only, no
// device call): tile width and K split, with and without a second output.
extern "C" void tc_gemm_plan(int Np, int sms, int nseg, int have_c2, int* bn, int* ksplit) {
  *ksplit = sgb::tc::pick_ksplit(Np, sms, nseg, have_c2 != 0);
  *bn = *ksplit == 2 ? 256 : sgb::tc::pick_bn(Np, sms);
}
