// BF16 tensor-core GEMM for sm_100a: tcgen05.mma with the FP32 accumulator in
// tensor memory, operand tiles brought into shared memory by TMA
// (cp.async.bulk.tensor, 128-byte swizzle); persistent, one CTA per SM.
//
//   C[i][j] = sum_s sum_c T[a_term[s]][i][c] * T[b_term[s]][j][c]
//
// T is a stack of nterms BF16 matrices of Np x Np (row-major, Np a multiple
// of 128, zero-padded past the caller's size); segment s of the K dimension
// pairs term a_term[s] (rows of A) with term b_term[s] (rows of B), so both
// operands are K-major and a product such as X1 (X1/2) + X1 X2 + X1 X3 +
// X2 (X2/2) is one launch with K = 4 Np and no repeated copy of X1 in memory.
// C is FP32, row-major with leading dimension ldc.
//
// Warp roles (192 threads): warp 0 issues the TMA loads into a ring of
// STAGES shared-memory stages, warp 1 owns the tensor-memory allocation and
// issues the MMAs (one elected thread; each stage is released back to the
// producer by tcgen05.commit on its "empty" barrier) into one of two
// accumulators, warps 2-5 read the other accumulator back with tcgen05.ld
// (each warp the 32 lanes of its quarter) and store it.  Every barrier wait is bounded (kWaitLimitNs): a wait that
// runs out sets a bit in the caller's error word, the thread stops issuing,
// the producer first waits (bounded) for its own loads in flight, and the
// CTA still frees its tensor memory before it returns.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstdint>
#include <string>

namespace sgb {
namespace tc {

constexpr int kBM = 128;       // tile rows (MMA M, tensor-memory lanes)
constexpr int kBK = 64;        // K per stage: 64 BF16 = one 128-byte swizzle row
constexpr int kUmmaK = 16;     // K of one tcgen05.mma kind::f16
constexpr int kThreads = 192;  // producer warp, MMA warp, four epilogue warps
constexpr int kMaxSeg = 8;
constexpr unsigned long long kWaitLimitNs = 2000000000ull;  // 2 s per wait

// error bits written to the caller's word
constexpr unsigned kErrEmpty = 1u, kErrFull = 2u, kErrAcc = 4u, kErrInflight = 8u;

struct Segments {
  int nseg;        // number of K segments
  int kb_per_seg;  // K blocks (of kBK) per segment = Np / kBK
  int a_row[kMaxSeg];  // first row of segment s's A term in the stacked tensor
  int b_row[kMaxSeg];
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t* bar, unsigned parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Wait for the phase of the given parity to complete; false after about
// kWaitLimitNs.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (;;) {
#pragma unroll 1
    for (int i = 0; i < 32; ++i)
      if (mbar_try(bar, parity)) return true;
    if (global_ns() - t0 > kWaitLimitNs) return false;
  }
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], "
      "[%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

// Shared-memory matrix descriptor of a K-major tile with the 128-byte
// swizzle: rows of 128 bytes, 8-row groups 1024 bytes apart (stride byte
// offset), descriptor version 1, layout type 2 (SWIZZLE_128B).  The leading
// byte offset is unused for this layout.
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr) {
  return (uint64_t)((addr & 0x3FFFFu) >> 4) | (1ull << 16) | ((uint64_t)(1024 >> 4) << 32) | (1ull << 46) |
         (2ull << 61);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, M = 128, N = bn.
__host__ __device__ constexpr uint32_t instr_desc_bf16(int bn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(bn >> 3) << 17) | ((uint32_t)(kBM >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
          tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 consecutive FP32 columns of this warp's 32 tensor-memory lanes.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

template <int BN, int STAGES>
struct Layout {
  static constexpr int kABytes = kBM * kBK * 2;
  static constexpr int kBBytes = BN * kBK * 2;
  static constexpr int kStage = kABytes + kBBytes;
  static constexpr int kBarOff = STAGES * kStage;
  // ring, then full[STAGES], empty[STAGES], acc_full[2], acc_empty[2],
  // tensor-memory address
  static constexpr int kBytes = kBarOff + (2 * STAGES + 4) * 8 + 16;
  static constexpr int kDynamic = kBytes + 1024;  // slack for the 1024-byte alignment of the ring
  static constexpr int kTmemCols = 2 * BN;        // two accumulators
  static_assert(kTmemCols <= 512, "tensor memory columns");
};

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Output tile t of the grouped raster: groups of kGroupM tile rows, column by
// column inside a group, so the CTAs working at the same time share A and B
// panels in L2.
__device__ __forceinline__ void tile_coords(int t, int mtiles, int ntiles, int& mt, int& nt) {
  constexpr int kGroupM = 16;
  const int per_group = kGroupM * ntiles;
  const int g = t / per_group, first_m = g * kGroupM;
  const int gm = min(mtiles - first_m, kGroupM);
  mt = first_m + (t % per_group) % gm;
  nt = (t % per_group) / gm;
}

// Persistent: CTA b takes work units b, b + gridDim.x, ...  A unit is a
// tile, or with ksplit = 2 half of a tile's K blocks (the first half's sum
// goes to C, the second's to C2; the caller adds them).  The load ring runs
// on across units; the accumulator alternates between two tensor-memory
// buffers, so the epilogue of one unit overlaps the main loop of the next
// (acc_full[b]: the MMAs of a unit into buffer b are complete; acc_empty[b]:
// the four epilogue warps have read buffer b out).
template <int BN, int STAGES>
__global__ void __launch_bounds__(kThreads, 1)
    k_tc_gemm_bf16(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, float* __restrict__ C,
                   float* __restrict__ C2, int ksplit, int ldc, int ncols, int mtiles, int ntiles,
                   const __grid_constant__ Segments seg, unsigned* __restrict__ err) {
  using L = Layout<BN, STAGES>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + L::kBarOff);
  uint64_t* empty = full + STAGES;
  uint64_t* accf = empty + STAGES;  // [2]
  uint64_t* acce = accf + 2;        // [2]
  uint32_t* tslot = reinterpret_cast<uint32_t*>(acce + 2);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int total = mtiles * ntiles * ksplit;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&accf[b], 1);
      mbar_init(&acce[b], 4);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(L::kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const int nk = seg.nseg * seg.kb_per_seg / ksplit;  // K blocks per unit

  if (warp == 0) {
    if (lane == 0) {
      long long issued = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < total && ok; t += gridDim.x) {
        int mt, nt;
        tile_coords(t / ksplit, mtiles, ntiles, mt, nt);
        const int m0 = mt * kBM, n0 = nt * BN, kb0 = (t % ksplit) * nk;
        for (int kb = kb0; kb < kb0 + nk; ++kb) {
          const int s = (int)(issued % STAGES);
          const unsigned ph = (unsigned)((issued / STAGES) & 1);
          if (!mbar_wait(&empty[s], ph ^ 1u)) {
            atomicOr(err, kErrEmpty);
            ok = false;
            break;
          }
          uint8_t* sa = smem + s * L::kStage;
          uint8_t* sb = sa + L::kABytes;
          const int sg = kb / seg.kb_per_seg, kx = (kb % seg.kb_per_seg) * kBK;
          mbar_expect_tx(&full[s], L::kStage);
          tma_load_2d(sa, &ta, &full[s], kx, seg.a_row[sg] + m0);
          tma_load_2d(sb, &tb, &full[s], kx, seg.b_row[sg] + n0);
          ++issued;
        }
      }
      if (!ok) {
        // wait (bounded) for this thread's loads still in flight
        for (long long q = issued - STAGES < 0 ? 0 : issued - STAGES; q < issued; ++q)
          if (!mbar_wait(&full[q % STAGES], (unsigned)((q / STAGES) & 1))) atomicOr(err, kErrInflight);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      constexpr uint32_t idesc = instr_desc_bf16(BN);
      long long consumed = 0;
      int i = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < total && ok; t += gridDim.x, ++i) {
        const int b = i & 1;
        // the epilogue has read buffer b out of its previous tile (none on first use)
        if (!mbar_wait(&acce[b], (unsigned)(((i >> 1) & 1) ^ 1))) {
          atomicOr(err, kErrAcc);
          break;
        }
        tc_fence_after();
        const uint32_t acc = tmem + (uint32_t)(b * BN);
        for (int kb = 0; kb < nk; ++kb) {
          const int s = (int)(consumed % STAGES);
          if (!mbar_wait(&full[s], (unsigned)((consumed / STAGES) & 1))) {
            atomicOr(err, kErrFull);
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t a0 = smem_u32(smem + s * L::kStage);
          const uint32_t b0 = a0 + L::kABytes;
#pragma unroll
          for (int k = 0; k < kBK / kUmmaK; ++k)
            umma_bf16(acc, smem_desc_sw128(a0 + k * kUmmaK * 2), smem_desc_sw128(b0 + k * kUmmaK * 2), idesc,
                      (kb | k) != 0);
          umma_commit(&empty[s]);
          ++consumed;
        }
        // buffer b complete (also on an early exit, so the epilogue is released)
        umma_commit(&accf[b]);
      }
    }
  } else {
    const int q = warp & 3;  // tensor-memory lane quarter of this warp
    int i = 0;
    for (int t = blockIdx.x; t < total; t += gridDim.x, ++i) {
      const int b = i & 1;
      const bool ready = __all_sync(0xffffffffu, mbar_wait(&accf[b], (unsigned)((i >> 1) & 1)));
      if (!ready) {
        if (lane == 0) atomicOr(err, kErrAcc);
        break;
      }
      tc_fence_after();
      int mt, nt;
      tile_coords(t / ksplit, mtiles, ntiles, mt, nt);
      const int row = mt * kBM + q * 32 + lane, n0 = nt * BN;
      float* crow = (t % ksplit ? C2 : C) + (size_t)row * ldc + n0;
#pragma unroll 1
      for (int c0 = 0; c0 < BN; c0 += 32) {
        float v[32];
        tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * BN + c0), v);
        if (n0 + c0 < ncols) {
          float4* dst = reinterpret_cast<float4*>(crow + c0);
#pragma unroll
          for (int u = 0; u < 8; ++u) dst[u] = make_float4(v[4 * u], v[4 * u + 1], v[4 * u + 2], v[4 * u + 3]);
        }
      }
      // this warp's reads of buffer b are done: hand it back to the MMA thread
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acce[b]);
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(L::kTmemCols) : "memory");
}

// The driver's tensor-map encoder, looked up once (thread-safe static
// initialisation); null when the driver does not export it.
inline PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    return static_cast<PFN_cuTensorMapEncodeTiled_v12000>(nullptr);
  }();
  return fn;
}

// 2-D map over the stacked terms (rows x Np BF16, row-major), box 64 x box_rows.
inline bool make_term_map(CUtensorMap* m, const void* base, int rows, int Np, int box_rows) {
  auto enc = tensor_map_encoder();
  if (!enc) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)Np, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)Np * 2};
  const cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)box_rows};
  const cuuint32_t es[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tile width for Np: 256 unless 128 fills the SMs' waves clearly better.
inline int pick_bn(int Np, int sms) {
  auto eff = [&](int bn) {
    const long long t = (long long)(Np / kBM) * ((Np + bn - 1) / bn);
    const long long waves = (t + sms - 1) / sms;
    return (double)t / (double)(waves * sms);
  };
  return eff(256) + 0.02 >= eff(128) ? 256 : 128;
}

// K split of the launch: 2 (with 256-wide tiles) when C2 is given and the
// 256-wide tiles of Np number at most half the SMs, else 1.  Sizes that fill
// the SMs only with 128-wide tiles run 256-wide tiles on half the K range each
// instead: twice the arithmetic per byte loaded, the same number of CTAs.
inline int pick_ksplit(int Np, int sms, int nseg, bool have_c2) {
  const long long t256 = (long long)(Np / kBM) * ((Np + 255) / 256);
  return have_c2 && (nseg * (Np / kBK)) % 2 == 0 && 2 * t256 <= sms ? 2 : 1;
}

// C (Np x Np, ldc) = the segment sum above over the stacked terms T
// (nterms x Np x Np BF16); with C2 (same shape, may be null) the launch may
// split K in two, and then C + C2 is the product (*ksplit_out tells which:
// 1 means C alone holds it).  Returns cudaSuccess or the launch error;
// err_msg names a host-side failure.  *d_err (device word) collects the
// kernel's bounded-wait bits; the caller clears and reads it.
inline cudaError_t gemm_terms(const __nv_bfloat16* T, int nterms, int Np, const int* a_term, const int* b_term,
                              int nseg, float* C, float* C2, int ldc, unsigned* d_err, cudaStream_t s,
                              std::string& err_msg, int* ksplit_out = nullptr) {
  if (Np <= 0 || Np % kBM != 0 || nseg < 1 || nseg > kMaxSeg || ldc < Np || (ldc % 4) != 0 ||
      (reinterpret_cast<uintptr_t>(T) & 15) != 0 || (reinterpret_cast<uintptr_t>(C) & 15) != 0 ||
      (reinterpret_cast<uintptr_t>(C2) & 15) != 0) {
    err_msg = "tensor-core GEMM: invalid shape or alignment";
    return cudaErrorInvalidValue;
  }
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int ksplit = pick_ksplit(Np, sms, nseg, C2 != nullptr);
  const int bn = ksplit == 2 ? 256 : pick_bn(Np, sms);
  if (ksplit_out) *ksplit_out = ksplit;
  Segments sg{};
  sg.nseg = nseg;
  sg.kb_per_seg = Np / kBK;
  for (int i = 0; i < nseg; ++i) {
    if (a_term[i] < 0 || a_term[i] >= nterms || b_term[i] < 0 || b_term[i] >= nterms) {
      err_msg = "tensor-core GEMM: term index out of range";
      return cudaErrorInvalidValue;
    }
    sg.a_row[i] = a_term[i] * Np;
    sg.b_row[i] = b_term[i] * Np;
  }
  CUtensorMap ma, mb;
  if (!make_term_map(&ma, T, nterms * Np, Np, kBM) || !make_term_map(&mb, T, nterms * Np, Np, bn)) {
    err_msg = "tensor-core GEMM: cuTensorMapEncodeTiled failed";
    return cudaErrorInvalidValue;
  }
  const int mtiles = Np / kBM, ntiles = (Np + bn - 1) / bn;
  const int units = mtiles * ntiles * ksplit;
  const int blocks = units < sms ? units : sms;  // persistent: at most one CTA per SM
  cudaError_t e;
  if (bn == 256) {
    using Lt = Layout<256, 4>;
    e = cudaFuncSetAttribute(k_tc_gemm_bf16<256, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, Lt::kDynamic);
    if (e != cudaSuccess) return e;
    k_tc_gemm_bf16<256, 4><<<blocks, kThreads, Lt::kDynamic, s>>>(ma, mb, C, C2, ksplit, ldc, Np, mtiles, ntiles, sg,
                                                                   d_err);
  } else {
    using Lt = Layout<128, 6>;
    e = cudaFuncSetAttribute(k_tc_gemm_bf16<128, 6>, cudaFuncAttributeMaxDynamicSharedMemorySize, Lt::kDynamic);
    if (e != cudaSuccess) return e;
    k_tc_gemm_bf16<128, 6><<<blocks, kThreads, Lt::kDynamic, s>>>(ma, mb, C, C2, ksplit, ldc, Np, mtiles, ntiles, sg,
                                                                   d_err);
  }
  return cudaGetLastError();
}

}  // namespace tc
}  // namespace sgb
