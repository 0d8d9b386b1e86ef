// Test harness (not part of the product): runs the SCF kernels' CTA
// eigensolver on a batch of symmetric matrices, one thread block each, so
// tests/test_gpu_eigh.py can check it against numpy.linalg.eigh.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../sparrow_b200/csrc/scf_core.cuh"

namespace {

struct ProbeShared {
  double red[32];
  int flag;
  int pad[3];
};

// Matrix m: F + off[m] (N[m] x N[m], row-major); outputs at the same offsets
// (Ct rows = vectors), eps at eoff[m], global tile scratch at gA + aoff[m];
// status[m] = 0 ok, 1 fallback needed.
__global__ void __launch_bounds__(512, 1) k_eigh_probe(const int* N, const long long* off, const long long* eoff,
                                                        const long long* aoff, const int* nvec, const double* F,
                                                        double* Ct, double* eps, double* gA, double* gZl,
                                                        double* gV, int* status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ProbeShared& sh = *reinterpret_cast<ProbeShared*>(smem_raw);
  double* ws = reinterpret_cast<double*>(smem_raw + sizeof(ProbeShared));
  unsigned dyn;
  asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
  const size_t ws_doubles = (dyn - sizeof(ProbeShared)) / sizeof(double);
  const int m = blockIdx.x, n = N[m];
  const long long o = off[m];
  const int st = sgb::eigh_tridiag(n, F + o, n, nvec[m], Ct + o, n, eps + eoff[m], ws, ws_doubles, gA + aoff[m], gZl + o,
                                   Ct + o, gV + o, sh.red, &sh.flag);
  if (threadIdx.x == 0) status[m] = st;
}

}  // namespace

// All pointers are device pointers.  smem_limit: dynamic shared memory per
// block (bytes; 0 = the device's opt-in maximum), so tests can force the
// global-memory path of the tiled matrix.
extern "C" int eigh_probe(int nmat, const int* N, const long long* off, const long long* eoff,
                          const long long* aoff, const int* nvec, const double* F, double* Ct, double* eps,
                          double* gA, double* gZl, double* gV, int* status, int smem_limit) {
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  const int bytes = smem_limit > 0 && smem_limit < optin ? smem_limit : optin;
  cudaFuncSetAttribute(k_eigh_probe, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  k_eigh_probe<<<nmat, 512, bytes>>>(N, off, eoff, aoff, nvec, F, Ct, eps, gA, gZl, gV, status);
  cudaError_t e = cudaDeviceSynchronize();
  return (int)e;
}
