// Large-molecule SCF: one NDDO molecule over the whole GPU.
//
// For molecules past the per-CTA limit (or on request) the SCF runs as a
// host-driven sequence of grid-wide kernels instead of the persistent
// one-CTA-per-molecule kernel:
//   Fock build     launch_fock_grid (pair phases over the grid, then the
//                  one-centre phase), F = H + G(P) and E_el
//   DIIS           Pulay on FP - PF with FP64 GEMMs, coefficients solved on
//                  the host (the same rule as the batched kernel)
//   density        SP2 purification (Niklasson): X0 = (e_max I - F) /
//                  (e_max - e_min) from Gershgorin bounds, then X <- X^2 or
//                  2X - X^2, whichever trace is closer to n_occ, until X is
//                  idempotent; P = 2X.  Only matrix products: no eigensolver.
// Precision: FP64 throughout (X X as a symmetric rank-k update, half the
// flops of a GEMM), or "mixed": the SP2 products run on the tensor cores from
// a three-term BF16 split (X = X1 + X2 + X3, keeping X1X1 + X1X2 + X2X1 +
// X1X3 + X2X2 + X3X1, as one GEMM of K = 4N by symmetry) with FP32
// accumulation.  FP64
// stays for the Fock build, DIIS, energy and gradient, and once the density
// change falls below a switch threshold (1e-5 by default) the remaining
// iterations run SP2 in FP64 (the residual correction), so the converged
// density is the FP64 one.
// The split-BF16 product is this library's own tcgen05/TMA kernel
// (tc_gemm.cuh); the FP64 squares and the DIIS product FP use cuBLAS.
#include <cublas_v2.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "engine.h"
#include "kernels.h"
#include "tc_gemm.cuh"

namespace sgb {

namespace {

constexpr int kLT = 256;

__device__ __forceinline__ double lw_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Gershgorin bounds of the rows of symmetric F: out[0] = max(F_ii + r_i),
// out[1] = max(r_i - F_ii) (so e_min >= -out[1]).  One warp per row.
__global__ void k_gershgorin(const double* __restrict__ F, int N, unsigned long long* out) {
  const int lane = threadIdx.x & 31;
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (row >= N) return;
  double r = 0;
  for (int j = lane; j < N; j += 32)
    if (j != row) r += fabs(F[(size_t)row * N + j]);
  r = lw_sum(r);
  if (lane == 0) {
    const double d = F[(size_t)row * N + row];
    // order-preserving map of doubles to unsigned for atomicMax
    auto key = [](double x) {
      unsigned long long u = __double_as_longlong(x);
      return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
    };
    atomicMax(&out[0], key(d + r));
    atomicMax(&out[1], key(r - d));
  }
}

__device__ __forceinline__ double key_to_double(unsigned long long u) {
  return __longlong_as_double((long long)((u & 0x8000000000000000ull) ? (u & 0x7fffffffffffffffull) : ~u));
}

// Block sums of (a, b) added into out[0], out[1] (1-D or 2-D blocks).
__device__ void block_add2(double a, double b, double* out) {
  __shared__ double r0[kLT / 32], r1[kLT / 32];
  const int t = threadIdx.y * blockDim.x + threadIdx.x, nw = (blockDim.x * blockDim.y) >> 5;
  a = lw_sum(a);
  b = lw_sum(b);
  if ((t & 31) == 0) {
    r0[t >> 5] = a;
    r1[t >> 5] = b;
  }
  __syncthreads();
  if (t == 0) {
    double x = 0, y = 0;
    for (int w = 0; w < nw; ++w) {
      x += r0[w];
      y += r1[w];
    }
    atomicAdd(&out[0], x);
    atomicAdd(&out[1], y);
  }
}

// X0 = (e_max I - F) / (e_max - e_min) with the Gershgorin bounds in keys;
// out[0] += trace(X0), out[1] += sum X0_ij^2 (= trace(X0^2), X0 symmetric).
__global__ void __launch_bounds__(kLT) k_sp2_init(const double* __restrict__ F, int N,
                                                  const unsigned long long* __restrict__ keys, double* X,
                                                  double* out) {
  const double emax = key_to_double(keys[0]), emin = -key_to_double(keys[1]);
  const double s = 1.0 / (emax - emin);
  double t = 0, t2 = 0;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < (size_t)N * N; k += (size_t)gridDim.x * blockDim.x) {
    const bool diag = k % (N + 1) == 0;
    const double x = ((diag ? emax : 0.0) - F[k]) * s;
    X[k] = x;
    t2 += x * x;
    if (diag) t += x;
  }
  block_add2(t, t2, out);
}

// One SP2 step from the product X2 = X X: with n_occ the target trace,
// X <- X2 when |tr(X2) - n_occ| < |2 tr(X) - tr(X2) - n_occ|, else 2X - X2
// (tr(X), tr(X2) in cur[0], cur[1]); the traces of the new X go to next.
// Only the upper triangle (column >= row) of X2 holds the product (a
// symmetric rank-k update); 32 x 32 tiles (block 32 x 8), lower tiles read
// their mirror tile through shared memory.
__global__ void __launch_bounds__(kLT) k_sp2_step_upper(double* X, const double* __restrict__ X2, int N, double nocc,
                                                        const double* __restrict__ cur, double* next) {
  __shared__ double tile[32][33];
  const double tr = cur[0], tr2 = cur[1];
  const int square = fabs(tr2 - nocc) < fabs(2.0 * tr - tr2 - nocc);
  const int i0 = blockIdx.y * 32, j0 = blockIdx.x * 32, tx = threadIdx.x, ty = threadIdx.y;
  const bool mirror = blockIdx.y > blockIdx.x;
  if (mirror) {
    for (int r = ty; r < 32; r += 8) {
      const int i = j0 + r, j = i0 + tx;  // tile (j0.., i0..) of the upper triangle
      tile[r][tx] = (i < N && j < N) ? X2[(size_t)i * N + j] : 0.0;
    }
    __syncthreads();
  }
  double t = 0, t2 = 0;
  for (int r = ty; r < 32; r += 8) {
    const int i = i0 + r, j = j0 + tx;
    if (i >= N || j >= N) continue;
    const size_t k = (size_t)i * N + j;
    // diagonal tiles: the strictly lower entries come from their mirror
    const double x2 = mirror ? tile[tx][r] : (j >= i ? X2[k] : X2[(size_t)j * N + i]);
    const double x = square ? x2 : 2.0 * X[k] - x2;
    X[k] = x;
    t2 += x * x;
    if (i == j) t += x;
  }
  block_add2(t, t2, next);
}

// The same step when the product is X X = A + A^T (A in FP32 from the
// split-BF16 GEMM, leading dimension lda; A = A1 + A2 when the GEMM split its
// K range, A2 null otherwise); 32 x 32 tiles (block 32 x 8), the mirror tile
// of A read through shared memory.
__global__ void __launch_bounds__(kLT) k_sp2_step_sym(double* X, const float* __restrict__ A,
                                                      const float* __restrict__ A2, int lda, int N, double nocc,
                                                      const double* __restrict__ cur, double* next) {
  __shared__ float tile[32][33];
  const double tr = cur[0], tr2 = cur[1];
  const int square = fabs(tr2 - nocc) < fabs(2.0 * tr - tr2 - nocc);
  const int i0 = blockIdx.y * 32, j0 = blockIdx.x * 32, tx = threadIdx.x, ty = threadIdx.y;
  for (int r = ty; r < 32; r += 8) {
    const int i = j0 + r, j = i0 + tx;
    tile[r][tx] = (i < N && j < N) ? A[(size_t)i * lda + j] + (A2 ? A2[(size_t)i * lda + j] : 0.0f) : 0.0f;
  }
  __syncthreads();
  double t = 0, t2 = 0;
  for (int r = ty; r < 32; r += 8) {
    const int i = i0 + r, j = j0 + tx;
    if (i >= N || j >= N) continue;
    const size_t k = (size_t)i * N + j;
    const size_t ka = (size_t)i * lda + j;
    const double x2 = (double)A[ka] + (A2 ? (double)A2[ka] : 0.0) + (double)tile[tx][r];
    const double x = square ? x2 : 2.0 * X[k] - x2;
    X[k] = x;
    t2 += x * x;
    if (i == j) t += x;
  }
  block_add2(t, t2, next);
}

// Three-term BF16 split X = X1 + X2 + X3 (each term the rounding of the
// remainder).  With every term symmetric,
//   X1 X1 + X1 X2 + X2 X1 + X1 X3 + X3 X1 + X2 X2 = A + A^T,
//   A = X1 (X1 / 2) + X1 X2 + X1 X3 + X2 (X2 / 2),
// one tensor-core GEMM with K = 4 Np over the five stacked terms
// T = [X1, X2, X3, X1/2, X2/2] (halving is exact in BF16), each Np x Np and
// zero past N.
constexpr int kTermX1 = 0, kTermX2 = 1, kTermX3 = 2, kTermX1h = 3, kTermX2h = 4, kTerms = 5;
__global__ void __launch_bounds__(kLT) k_split_terms(const double* __restrict__ X, int N, int Np,
                                                     __nv_bfloat16* __restrict__ T) {
  const size_t nn = (size_t)Np * Np;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < nn; k += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(k / Np), j = (int)(k % Np);
    const double x = (i < N && j < N) ? X[(size_t)i * N + j] : 0.0;
    const __nv_bfloat16 a = __double2bfloat16(x);
    const double r1 = x - (double)__bfloat162float(a);
    const __nv_bfloat16 b = __double2bfloat16(r1);
    const double r2 = r1 - (double)__bfloat162float(b);
    const __nv_bfloat16 half = __float2bfloat16(0.5f);
    T[kTermX1 * nn + k] = a;
    T[kTermX2 * nn + k] = b;
    T[kTermX3 * nn + k] = __double2bfloat16(r2);
    T[kTermX1h * nn + k] = __hmul(a, half);
    T[kTermX2h * nn + k] = __hmul(b, half);
  }
}

// DIIS store over 32 x 32 tiles (block 32 x 8): E = W - W^T (W = FP) into
// e_slot, F into f_slot, and out[j] += <E, E_j> for the m stored error
// matrices (slot j of histE; the new one is E itself).
__global__ void __launch_bounds__(kLT) k_diis_store(const double* __restrict__ W, const double* __restrict__ F, int N,
                                                    double* histE, double* histF, int slot, int m, double* out) {
  __shared__ double tw[32][33], tt[32][33];
  __shared__ double red[kDiisMax][kLT / 32];
  const size_t NN = (size_t)N * N;
  const int i0 = blockIdx.y * 32, j0 = blockIdx.x * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int r = ty; r < 32; r += 8) {
    const int i = i0 + r, j = j0 + tx;
    tw[r][tx] = (i < N && j < N) ? W[(size_t)i * N + j] : 0.0;
    const int it = j0 + r, jt = i0 + tx;  // W^T tile: rows j0.., columns i0..
    tt[r][tx] = (it < N && jt < N) ? W[(size_t)it * N + jt] : 0.0;
  }
  __syncthreads();
  double d[kDiisMax];
#pragma unroll
  for (int q = 0; q < kDiisMax; ++q) d[q] = 0.0;
  double* es = histE + (size_t)slot * NN;
  double* fs = histF + (size_t)slot * NN;
  for (int r = ty; r < 32; r += 8) {
    const int i = i0 + r, j = j0 + tx;
    if (i >= N || j >= N) continue;
    const size_t k = (size_t)i * N + j;
    const double e = tw[r][tx] - tt[tx][r];
    es[k] = e;
    fs[k] = F[k];
#pragma unroll
    for (int q = 0; q < kDiisMax; ++q)
      if (q < m) d[q] += e * (q == slot ? e : histE[(size_t)q * NN + k]);
  }
  const int t = ty * 32 + tx, lane = t & 31, w = t >> 5;
#pragma unroll
  for (int q = 0; q < kDiisMax; ++q) {
    const double v = lw_sum(d[q]);
    if (lane == 0) red[q][w] = v;
  }
  __syncthreads();
  if (t < m) {
    double v = 0;
    for (int x = 0; x < kLT / 32; ++x) v += red[t][x];
    atomicAdd(&out[t], v);
  }
}

// dst = sum_i c_i src_i (m terms, stride n between terms)
__global__ void k_combine(const double* __restrict__ src, size_t n, int m, const double* __restrict__ c, double* dst) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    double s = 0;
    for (int i = 0; i < m; ++i) s += c[i] * src[(size_t)i * n + k];
    dst[k] = s;
  }
}

// P_new = 2 X; out[0] += sum (P_new - P)^2; P = P_new
__global__ void k_density_update(const double* __restrict__ X, size_t n, double* P, double* out) {
  __shared__ double red[kLT / 32];
  double s = 0;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    const double p = 2.0 * X[k];
    const double d = p - P[k];
    s += d * d;
    P[k] = p;
  }
  s = lw_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < kLT / 32; ++w) t += red[w];
    atomicAdd(out, t);
  }
}

// Reduction slots of the large path (doubles at the start of the scratch).
constexpr int kSlotKeys = 0;     // 2 Gershgorin keys
constexpr int kSlotEnergy = 8;   // E_el of the last Fock build
constexpr int kSlotDots = 16;    // kDiisMax DIIS dot products
constexpr int kSlotCoef = 24;    // kDiisMax DIIS coefficients
constexpr int kSlotRms = 32;     // sum (dP)^2
constexpr int kSlotTcErr = 40;   // bounded-wait bits of the tensor-core GEMM (as unsigned)
constexpr int kSlotTraces = 64;  // (trace X, trace X^2) per SP2 step
constexpr int kSp2MaxSteps = 200;
constexpr size_t kStateBytes = 8192;
static_assert(kSlotTraces + 2 * (kSp2MaxSteps + 1) <= (int)(kStateBytes / sizeof(double)), "state slots");

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// cuBLAS handle of this host thread (created once, on first use)
cublasHandle_t blas_handle(std::string& err) {
  thread_local cublasHandle_t h = nullptr;
  thread_local int hdev = -1;
  int dev = 0;
  cudaGetDevice(&dev);
  if (h && hdev == dev) return h;
  if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS) {
    h = nullptr;
    err = "cublasCreate failed";
    return nullptr;
  }
  hdev = dev;
  return h;
}

// Pulay DIIS coefficients from the B matrix (row-major kDiisMax stride) of n
// vectors: the same scaled, pivoted elimination as the batched kernel.
// Returns false when the system is singular or the error vectors are rounding
// noise.
bool diis_solve(const double* bm, int n, double* coef) {
  const int ld = n + 2;
  std::vector<double> sys((size_t)(n + 1) * ld);
  double scale = 0;
  for (int i = 0; i < n; ++i) scale = std::max(scale, std::fabs(bm[i * kDiisMax + i]));
  if (!(scale > kDiisNoiseNorm)) return false;
  scale = scale > 0 ? 1.0 / scale : 1.0;
  for (int i = 0; i <= n; ++i) {
    for (int j = 0; j <= n; ++j)
      sys[i * ld + j] = (i < n && j < n) ? bm[i * kDiisMax + j] * scale : (i == n && j == n ? 0.0 : -1.0);
    sys[i * ld + n + 1] = i == n ? -1.0 : 0.0;
  }
  for (int c = 0; c <= n; ++c) {
    int piv = c;
    for (int r = c + 1; r <= n; ++r)
      if (std::fabs(sys[r * ld + c]) > std::fabs(sys[piv * ld + c])) piv = r;
    if (std::fabs(sys[piv * ld + c]) < 1e-300) return false;
    if (piv != c)
      for (int k = 0; k <= n + 1; ++k) std::swap(sys[c * ld + k], sys[piv * ld + k]);
    for (int r = c + 1; r <= n; ++r) {
      const double f = sys[r * ld + c] / sys[c * ld + c];
      for (int k = c; k <= n + 1; ++k) sys[r * ld + k] -= f * sys[c * ld + k];
    }
  }
  std::vector<double> x(n + 1);
  for (int c = n; c >= 0; --c) {
    double s = sys[c * ld + n + 1];
    for (int k = c + 1; k <= n; ++k) s -= sys[c * ld + k] * x[k];
    x[c] = s / sys[c * ld + c];
  }
  for (int i = 0; i < n; ++i) {
    if (!std::isfinite(x[i])) return false;
    coef[i] = x[i];
  }
  return true;
}

}  // namespace

// The split-BF16 products run on Np = nao rounded up to the GEMM tile.
int padded_order(long long nao) { return (int)((nao + tc::kBM - 1) / tc::kBM * tc::kBM); }

size_t large_scf_scratch_bytes(long long nao) {
  const size_t NP = (size_t)padded_order(nao) * padded_order(nao);
  return kStateBytes + align256(kTerms * NP * 2) + 2 * align256(NP * 4);
}

namespace {

// Pinned readback buffer and the two events of the SP2 pipeline, released on
// every return path.
struct LargeHost {
  double* hp = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  ~LargeHost() {
    if (hp) cudaFreeHost(hp);
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
  }
};

// Timing events around the purification products of one SCF iteration
// (two per product), created once per host thread and device and reused by
// every later call.
struct EventSets {
  std::unordered_map<int, std::vector<cudaEvent_t>> per_device;
  ~EventSets() {
    for (auto& kv : per_device)
      for (auto e : kv.second) cudaEventDestroy(e);
  }
};

const std::vector<cudaEvent_t>* product_events(cudaError_t& ce) {
  thread_local EventSets sets;
  auto& per_device = sets.per_device;
  int dev = 0;
  ce = cudaGetDevice(&dev);
  if (ce != cudaSuccess) return nullptr;
  std::vector<cudaEvent_t>& ev = per_device[dev];
  if (!ev.empty()) return &ev;
  for (int k = 0; k < 2 * kSp2MaxSteps; ++k) {
    cudaEvent_t e = nullptr;
    ce = cudaEventCreate(&e);
    if (ce != cudaSuccess) {
      for (auto& x : ev) cudaEventDestroy(x);
      ev.clear();
      return nullptr;
    }
    ev.push_back(e);
  }
  return &ev;
}

const char* blas_message(cublasStatus_t st) {
  switch (st) {
    case CUBLAS_STATUS_NOT_INITIALIZED: return "cuBLAS not initialised";
    case CUBLAS_STATUS_ALLOC_FAILED: return "cuBLAS allocation failed";
    case CUBLAS_STATUS_INVALID_VALUE: return "cuBLAS invalid value";
    case CUBLAS_STATUS_ARCH_MISMATCH: return "cuBLAS architecture mismatch";
    case CUBLAS_STATUS_EXECUTION_FAILED: return "cuBLAS execution failed";
    case CUBLAS_STATUS_NOT_SUPPORTED: return "cuBLAS operation not supported";
    default: return "cuBLAS error";
  }
}

// SP2 stop rule on the idempotency measure e_j = tr(X_j) - tr(X_j^2) =
// sum lambda (1 - lambda) of the j-th iterate (hp holds the trace pairs),
// which bounds every eigenvalue's distance from 0 or 1: e_j below 1e-12 N
// (the step already queued behind X_j squares that distance away), or, once
// every eigenvalue is within about 0.1 of 0 or 1 (e_j < 0.1), no decrease
// against two steps before (the rounding floor of the working precision).
bool sp2_converged(const double* hp, int j, int N) {
  const double e = std::fabs(hp[2 * j] - hp[2 * j + 1]);
  if (!std::isfinite(e)) return true;
  if (e < 1e-12 * N) return true;
  return j >= 2 && e < 0.1 && e >= std::fabs(hp[2 * (j - 2)] - hp[2 * (j - 2) + 1]);
}

}  // namespace

int run_large_scf(const DeviceBatch& b, const MolDev& m, const ScfParams& sp, int precision, cudaStream_t s,
                  int* launches, std::string& err) {
  cublasHandle_t h = blas_handle(err);
  if (!h) return kErrCuda;
  cublasStatus_t bs = cublasSetStream(h, s);
  if (bs == CUBLAS_STATUS_SUCCESS) bs = cublasSetMathMode(h, CUBLAS_DEFAULT_MATH);
  if (bs != CUBLAS_STATUS_SUCCESS) {
    err = blas_message(bs);
    return kErrCuda;
  }
  const int N = m.nao;
  const size_t NN = (size_t)N * N;
  const double nocc = m.nocc;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = sms * 8;
  char* scr = static_cast<char*>(b.large_scratch);
  double* st = reinterpret_cast<double*>(scr);
  const int Np = padded_order(N);
  const size_t NP = (size_t)Np * Np;
  __nv_bfloat16* T = reinterpret_cast<__nv_bfloat16*>(scr + kStateBytes);
  float* C32 = reinterpret_cast<float*>(scr + kStateBytes + align256(kTerms * NP * 2));
  float* C32b = reinterpret_cast<float*>(scr + kStateBytes + align256(kTerms * NP * 2) + align256(NP * 4));
  unsigned* tc_err = reinterpret_cast<unsigned*>(st + kSlotTcErr);
  static const int a_terms[4] = {kTermX1, kTermX1, kTermX1, kTermX2};
  static const int b_terms[4] = {kTermX1h, kTermX2, kTermX3, kTermX2h};
  double* histF = b.diis;
  double* histE = b.diis + (size_t)kDiisMax * NN;
  double* X = b.C;
  double* X2 = b.W1;
  double* W = b.W2;
  LargeHost hb;
  cudaError_t ce = cudaMallocHost(&hb.hp, sizeof(double) * 2 * (kSp2MaxSteps + 2));
  if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&hb.ev[0], cudaEventDisableTiming);
  if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&hb.ev[1], cudaEventDisableTiming);
  const std::vector<cudaEvent_t>* pevp = ce == cudaSuccess ? product_events(ce) : nullptr;
  if (ce != cudaSuccess || !pevp) {
    err = cuda_message(ce);
    return kErrCuda;
  }
  const std::vector<cudaEvent_t>& pev = *pevp;
  const double one = 1.0, zero = 0.0;
  const int msize = sp.diis_size < 1 ? 1 : (sp.diis_size > kDiisMax ? kDiisMax : sp.diis_size);
  double bmat[kDiisMax * kDiisMax] = {};
  int nhist = 0, head = 0, nl = 0;
  double Eold = 0, last_dE = 0, last_rms = 0, prev_rms = 1e300;
  int it = 0, converged = 0, status = kDevOk, sp2_total = 0, mixed_iters = 0;
  // device time and count of the purification products, split-BF16 and FP64
  double prod_ms[2] = {0, 0};
  long long prod_n[2] = {0, 0};
  bool mixed = precision == 1;
  const dim3 tgrid((N + 31) / 32, (N + 31) / 32), tblock(32, 8);
  auto fail_cuda = [&](cudaError_t e) {
    err = cuda_message(e);
    return kErrCuda;
  };
  for (it = 1; it <= sp.max_iter; ++it) {
    // F = H + G(P) and E_el(P)
    launch_fock_grid(b, b.P, b.F, st + kSlotEnergy, s);
    nl += 2;
    // DIIS: W = F P (row-major; the column-major product P F), E = W - W^T
    bs = cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, N, N, N, &one, b.P, N, b.F, N, &zero, W, N);
    if (bs != CUBLAS_STATUS_SUCCESS) {
      err = blas_message(bs);
      return kErrCuda;
    }
    const int slot = head;
    head = (head + 1) % msize;
    if (nhist < msize) ++nhist;
    cudaMemsetAsync(st + kSlotDots, 0, sizeof(double) * kDiisMax, s);
    k_diis_store<<<tgrid, tblock, 0, s>>>(W, b.F, N, histE, histF, slot, nhist, st + kSlotDots);
    ++nl;
    cudaMemcpyAsync(hb.hp, st + kSlotEnergy, sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(hb.hp + 1, st + kSlotDots, sizeof(double) * kDiisMax, cudaMemcpyDeviceToHost, s);
    ce = cudaStreamSynchronize(s);
    if (ce == cudaSuccess) ce = cudaGetLastError();
    if (ce != cudaSuccess) return fail_cuda(ce);
    const double E = hb.hp[0];
    for (int q = 0; q < nhist; ++q) bmat[slot * kDiisMax + q] = bmat[q * kDiisMax + slot] = hb.hp[1 + q];
    if (nhist >= 2) {
      double c[kDiisMax];
      if (diis_solve(bmat, nhist, c)) {
        cudaMemcpyAsync(st + kSlotCoef, c, sizeof(double) * nhist, cudaMemcpyHostToDevice, s);
        k_combine<<<grid, kLT, 0, s>>>(histF, NN, nhist, st + kSlotCoef, b.F);
        ++nl;
      }
    }
    // SP2 purification of the (extrapolated) F into X
    const bool use_mixed = mixed;
    cudaMemsetAsync(st + kSlotKeys, 0, sizeof(double) * 2, s);
    cudaMemsetAsync(st + kSlotTraces, 0, sizeof(double) * 2 * (kSp2MaxSteps + 1), s);
    cudaMemsetAsync(tc_err, 0, sizeof(unsigned), s);
    k_gershgorin<<<(N * 32 + kLT - 1) / kLT, kLT, 0, s>>>(b.F, N, reinterpret_cast<unsigned long long*>(st + kSlotKeys));
    k_sp2_init<<<grid, kLT, 0, s>>>(b.F, N, reinterpret_cast<const unsigned long long*>(st + kSlotKeys), X,
                                    st + kSlotTraces);
    nl += 2;
    cudaMemcpyAsync(hb.hp, st + kSlotTraces, 2 * sizeof(double), cudaMemcpyDeviceToHost, s);
    bool sp2_ok = false;
    int nprod = 0;
    for (int k = 0; k < kSp2MaxSteps; ++k) {
      nprod = k + 1;
      double* cur = st + kSlotTraces + 2 * k;
      if (use_mixed) {
        k_split_terms<<<grid, kLT, 0, s>>>(X, N, Np, T);
        cudaEventRecord(pev[2 * k], s);
        int ksplit = 1;
        ce = tc::gemm_terms(T, kTerms, Np, a_terms, b_terms, 4, C32, C32b, Np, tc_err, s, err, &ksplit);
        cudaEventRecord(pev[2 * k + 1], s);
        if (ce != cudaSuccess) {
          if (err.empty()) err = cuda_message(ce);
          return kErrCuda;
        }
        k_sp2_step_sym<<<tgrid, tblock, 0, s>>>(X, C32, ksplit == 2 ? C32b : nullptr, Np, N, nocc, cur, cur + 2);
        nl += 3;
      } else {
        // X X = X X^T: half the flops of a GEMM; the column-major lower
        // triangle is the row-major upper one
        cudaEventRecord(pev[2 * k], s);
        bs = cublasDsyrk(h, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, N, N, &one, X, N, &zero, X2, N);
        cudaEventRecord(pev[2 * k + 1], s);
        k_sp2_step_upper<<<tgrid, tblock, 0, s>>>(X, X2, N, nocc, cur, cur + 2);
        ++nl;
      }
      if (bs != CUBLAS_STATUS_SUCCESS) {
        err = blas_message(bs);
        return kErrCuda;
      }
      cudaMemcpyAsync(hb.hp + 2 * (k + 1), cur + 2, 2 * sizeof(double), cudaMemcpyDeviceToHost, s);
      cudaEventRecord(hb.ev[k & 1], s);
      ++sp2_total;
      // test the previous iterate while this step runs (one step of look-ahead)
      if (k >= 1) {
        ce = cudaEventSynchronize(hb.ev[(k - 1) & 1]);
        if (ce != cudaSuccess) return fail_cuda(ce);
        if (sp2_converged(hb.hp, k, N)) {
          sp2_ok = std::isfinite(hb.hp[2 * k] - hb.hp[2 * k + 1]);
          break;
        }
      }
    }
    if (use_mixed) ++mixed_iters;
    if (!sp2_ok) status = kDevSp2NotConverged;
    // P = 2 X and rms(dP)
    cudaMemsetAsync(st + kSlotRms, 0, sizeof(double), s);
    k_density_update<<<grid, kLT, 0, s>>>(X, NN, b.P, st + kSlotRms);
    ++nl;
    cudaMemcpyAsync(hb.hp, st + kSlotRms, sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(hb.hp + 1, tc_err, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
    ce = cudaStreamSynchronize(s);
    if (ce == cudaSuccess) ce = cudaGetLastError();
    if (ce != cudaSuccess) return fail_cuda(ce);
    for (int k = 0; k < nprod; ++k) {
      float ms = 0;
      if (cudaEventElapsedTime(&ms, pev[2 * k], pev[2 * k + 1]) == cudaSuccess) {
        prod_ms[use_mixed ? 0 : 1] += ms;
        ++prod_n[use_mixed ? 0 : 1];
      }
    }
    cudaGetLastError();
    unsigned tc_bits = 0;
    std::memcpy(&tc_bits, hb.hp + 1, sizeof(unsigned));
    if (tc_bits != 0) {
      err = "tensor-core GEMM: a bounded barrier wait ran out (bits " + std::to_string(tc_bits) + ")";
      return kErrCuda;
    }
    const double rms = std::sqrt(hb.hp[0] / (double)NN);
    last_rms = rms;
    last_dE = it > 1 ? std::fabs(E - Eold) : 0.0;
    const bool dE_ok = it > 1 && std::fabs(E - Eold) < sp.scc;
    Eold = E;
    if (!std::isfinite(E) || !std::isfinite(rms)) {
      status = kDevNonFinite;
      break;
    }
    if (status != kDevOk) break;
    // the residual correction: once the mixed density is this close, the
    // remaining purifications run in FP64 (convergence is only accepted on
    // an FP64 density)
    // (or when the mixed densities stop improving: the precision floor)
    if (mixed && (rms < sp.mixed_switch_rmsd || (rms < 1e-4 && rms > 0.5 * prev_rms))) mixed = false;
    prev_rms = rms;
    if (dE_ok && rms < sp.rmsd && !use_mixed) {
      converged = 1;
      break;
    }
  }
  if (it > sp.max_iter) it = sp.max_iter;
  // energy of the final density (the Fock matrix is rebuilt from it)
  launch_fock_grid(b, b.P, b.F, st + kSlotEnergy, s);
  nl += 2;
  MolResult r{};
  cudaMemcpyAsync(hb.hp, st + kSlotEnergy, sizeof(double), cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(&r, b.res, sizeof(MolResult), cudaMemcpyDeviceToHost, s);
  ce = cudaStreamSynchronize(s);
  if (ce != cudaSuccess) return fail_cuda(ce);
  r.e_el = hb.hp[0];
  r.energy = r.e_el + r.e_rep;
  r.iterations = it;
  r.converged = converged;
  r.status = status;
  r.last_dE = last_dE;
  r.last_rmsd = last_rms;
  r.full_diag = mixed_iters;
  r.jacobi_sweeps = sp2_total;
  // the cycle slots carry the purification products on this path: device ns
  // and count of the split-BF16 tensor-core GEMMs, then of the FP64 squares
  r.cycles[0] = (long long)(prod_ms[0] * 1e6);
  r.cycles[1] = prod_n[0];
  r.cycles[2] = (long long)(prod_ms[1] * 1e6);
  r.cycles[3] = prod_n[1];
  r.cycles[4] = 0;
  ce = cudaMemcpyAsync(b.res, &r, sizeof(MolResult), cudaMemcpyHostToDevice, s);
  // no orbitals on this path: the orbital energies read as zero
  if (ce == cudaSuccess) ce = cudaMemsetAsync(b.eps, 0, sizeof(double) * N, s);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
  if (ce != cudaSuccess) return fail_cuda(ce);
  if (launches) *launches += nl;
  return kOk;
}

}  // namespace sgb
