// Device building blocks of the persistent per-molecule SCF kernels (NDDO
// and DFTB): CTA reductions, the FP64 tensor-core CTA GEMM, the cyclic
// Jacobi eigensolver with deferred rotation replay, Pulay DIIS and the
// occupied-virtual orbital rotation.  Included by the SCF kernel sources;
// everything lives in an unnamed namespace (one copy per module).
#pragma once
#include <cuda_runtime.h>

#include "kernels.h"

namespace sgb {
namespace {

constexpr int kScfThreads = 512;
constexpr int kGemmGroup = 256;       // threads per GEMM tile group
constexpr int kJacobiMaxPairs = 512;  // supports N <= 1024
// K depth of one pipeline slice of the CTA GEMM (8 or 16)
#ifndef SGB_GEMM_BK
#define SGB_GEMM_BK 8
#endif
constexpr int kGemmBM = 64, kGemmBN = 64, kGemmBK = SGB_GEMM_BK;
static_assert(kGemmBK == 8 || kGemmBK == 16, "CTA GEMM slice depth");
constexpr size_t kRotBudgetBytes = kScfRotationBytesPerCta;
// shared strides of the GEMM input tiles: k-contiguous rows of 8 (+4 pad) or
// m/n-contiguous rows of 64 (+8 pad); one stage holds an A and a B tile
constexpr int kGemmLdK = kGemmBK + 4, kGemmLdMN = kGemmBM + 8;
constexpr int kGemmStage = 2 * (kGemmBM * kGemmLdK > kGemmBK * kGemmLdMN ? kGemmBM * kGemmLdK : kGemmBK * kGemmLdMN);
// cp.async pipeline depth of the GEMM (stages in flight per tile group)
#ifndef SGB_GEMM_STAGES
#define SGB_GEMM_STAGES 3
#endif
constexpr int kGemmStages = SGB_GEMM_STAGES;

// ---------------------------------------------------------------------------
// CTA helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Block-wide sum; every thread gets the result.
__device__ double cta_sum(double v, double* red) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double s = 0;
  for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += red[i];
  return s;
}
__device__ double cta_max(double v, double* red) {
  v = warp_max(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double s = red[0];
  for (int i = 1; i < (int)(blockDim.x >> 5); ++i) s = fmax(s, red[i]);
  return s;
}

__device__ __forceinline__ void group_sync(int grp) {
  asm volatile("bar.sync %0, %1;" ::"r"(grp + 1), "r"(kGemmGroup) : "memory");
}

__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool valid) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  const int n = valid ? 8 : 0;  // zero-fill when out of bounds
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }
template <int kPending>
__device__ __forceinline__ void cp_async_wait_pending() {
  asm volatile("cp.async.wait_group %0;" ::"n"(kPending) : "memory");
}

// C = alpha * op(A) * op(B) + beta * C, row-major, op(X) = X or X^T, on the
// FP64 tensor cores (mma.sync m16n8k8 f64, the sm_90+ shape: one instruction
// for the work of four m8n8k4).  The CTA (512 threads) is split into two
// groups of 256 that work on different 64x64 output tiles; in a group each of
// the 8 warps owns a 16x32 block (4 MMA tiles of 16x8, 16 accumulators per
// thread).  The 64x8 / 8x64 input tiles stream through a kGemmStages-deep
// cp.async ring in shared memory, so the global-load latency of the next
// slices overlaps the MMAs of the current one.  Their layout follows the
// global one so the copies stay coalesced: A row-major [m][k] (stride 12) or,
// when op(A) = A^T, [k][m] (stride 72), and likewise for B; with these
// strides both the copies and the fragment reads touch every bank twice (two
// wavefronts per warp).
// Fragments (g = lane / 4, t = lane % 4): a[v] = A(g + 8 (v % 2), t + 4 (v / 2)),
// b[v] = B(t + 4 v, g), c[v] = C(g + 8 (v / 2), 2 t + v % 2).
__device__ __forceinline__ void dmma_16x8x8(double (&c)[4], const double (&a)[4], const double (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
      "{%0, %1, %2, %3};"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// sym: the result is known to be symmetric (M == Nn): only the tiles on or
// above the diagonal are computed, off-diagonal tiles are mirrored.
// kDiff: the epilogue also adds to *diff2 this thread's share of the squared
// difference sum_ij (C_ij - ref_ij)^2 over the whole result (a mirrored entry
// counts twice, so ref must be symmetric when sym is set), sparing a pass
// over C and ref.
template <bool kDiff = false>
__device__ __forceinline__ void cta_gemm(int M, int Nn, int K, double alpha, const double* __restrict__ A, int lda, bool tA,
                         const double* __restrict__ B, int ldb, bool tB, double beta, double* C, int ldc,
                         double* smem, bool sym = false, const double* __restrict__ ref = nullptr,
                         double* diff2 = nullptr) {
  const int grp = threadIdx.x / kGemmGroup, tid = threadIdx.x % kGemmGroup;
  const int lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  double* base = smem + grp * kGemmStages * kGemmStage;
  const int tilesM = (M + kGemmBM - 1) / kGemmBM, tilesN = (Nn + kGemmBN - 1) / kGemmBN;
  const int ntiles = sym ? tilesM * (tilesM + 1) / 2 : tilesM * tilesN;
  const int nk = (K + kGemmBK - 1) / kGemmBK;
  // shared strides of A(m, k) and B(k, n)
  const int a_sm = tA ? 1 : kGemmLdK, a_sk = tA ? kGemmLdMN : 1;
  const int b_sn = tB ? kGemmLdK : 1, b_sk = tB ? 1 : kGemmLdMN;
  // the source address is only formed when in bounds; out-of-bounds slots copy 0 bytes
  auto load_stage = [&](int stage, int m0, int n0, int k0) {
    double* smA = base + stage * kGemmStage;
    double* smB = smA + kGemmStage / 2;
#pragma unroll
    for (int r = 0; r < (kGemmBM * kGemmBK) / kGemmGroup; ++r) {
      const int e = tid + r * kGemmGroup;
      int mm, kk;
      if (!tA) { mm = e / kGemmBK; kk = e % kGemmBK; }
      else { kk = e >> 6; mm = e & 63; }
      const int gm = m0 + mm, gk = k0 + kk;
      const bool ok = gm < M && gk < K;
      const double* src = ok ? (tA ? A + (size_t)gk * lda + gm : A + (size_t)gm * lda + gk) : A;
      cp_async8(&smA[mm * a_sm + kk * a_sk], src, ok);
    }
#pragma unroll
    for (int r = 0; r < (kGemmBK * kGemmBN) / kGemmGroup; ++r) {
      const int e = tid + r * kGemmGroup;
      int nn, kk;
      if (!tB) { kk = e >> 6; nn = e & 63; }
      else { nn = e / kGemmBK; kk = e % kGemmBK; }
      const int gn = n0 + nn, gk = k0 + kk;
      const bool ok = gn < Nn && gk < K;
      const double* src = ok ? (tB ? B + (size_t)gn * ldb + gk : B + (size_t)gk * ldb + gn) : B;
      cp_async8(&smB[nn * b_sn + kk * b_sk], src, ok);
    }
    cp_async_commit();
  };
  const int fr = lane >> 2, fc = lane & 3;  // fragment row / column-in-group
  for (int tile = grp; tile < ntiles; tile += 2) {
    int tm = tile / tilesN, tn = tile % tilesN;
    if (sym) {  // tile-th upper tile, row-major over (tm, tn >= tm)
      int t = tile;
      tm = 0;
      while (t >= tilesM - tm) {
        t -= tilesM - tm;
        ++tm;
      }
      tn = tm + t;
    }
    const int m0 = tm * kGemmBM, n0 = tn * kGemmBN;
    // 8 x 8 blocks of this warp that lie inside the product: edge tiles skip
    // the MMAs (and fragment loads) of their padding, which frees the FP64
    // tensor pipe for the other warps of the SM (warp-uniform masks)
    const bool rows_in = M > m0 + wm * 16;
    const int cols_left = Nn - (n0 + wn * 32);
    const int nbj = !rows_in ? 0 : (cols_left >= 32 ? 4 : (cols_left > 0 ? (cols_left + 7) >> 3 : 0));
    double acc[4][4];
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0;
#pragma unroll
    for (int st = 0; st < kGemmStages - 1; ++st) {
      if (st < nk) load_stage(st, m0, n0, st * kGemmBK);
      else cp_async_commit();  // empty group: keeps the group count per slice fixed
    }
    for (int kt = 0; kt < nk; ++kt) {
      cp_async_wait_pending<kGemmStages - 2>();
      group_sync(grp);  // slice kt visible; the ring slot of slice kt-1 is no longer read
      const int nxt = kt + kGemmStages - 1;
      if (nxt < nk) load_stage(nxt % kGemmStages, m0, n0, nxt * kGemmBK);
      else cp_async_commit();
      const double* smA = base + (kt % kGemmStages) * kGemmStage;
      const double* smB = smA + kGemmStage / 2;
#pragma unroll
      for (int ks = 0; ks < kGemmBK; ks += 8) {
        double a[4], b[4][2];
#pragma unroll
        for (int v = 0; v < 4; ++v)
          a[v] = smA[(wm * 16 + fr + 8 * (v & 1)) * a_sm + (ks + fc + 4 * (v >> 1)) * a_sk];
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
          for (int v = 0; v < 2; ++v) b[j][v] = smB[(wn * 32 + j * 8 + fr) * b_sn + (ks + fc + 4 * v) * b_sk];
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (j < nbj) dmma_16x8x8(acc[j], a, b[j]);
      }
    }
    group_sync(grp);  // all reads of the last stage done before the next tile overwrites it
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int gm = m0 + wm * 16 + fr + 8 * (q >> 1), gn = n0 + wn * 32 + j * 8 + fc * 2 + (q & 1);
        if (gm < M && gn < Nn) {
          double* c = &C[(size_t)gm * ldc + gn];
          const double v = beta == 0.0 ? alpha * acc[j][q] : alpha * acc[j][q] + beta * (*c);
          *c = v;
          if (sym && tn > tm) C[(size_t)gn * ldc + gm] = v;
          if (kDiff) {
            const double d = v - ref[(size_t)gm * ldc + gn];
            *diff2 += (sym && tn > tm ? 2.0 : 1.0) * d * d;
          }
        }
      }
  }
  __syncthreads();
}

__device__ __forceinline__ long long pair_slot(const MolDev& m, int lo, int hi) {
  return (long long)m.pair0 + (long long)lo * m.nat - (long long)lo * (lo + 1) / 2 + (hi - lo - 1);
}


// Fock-build warp scratch of the NDDO kernel (part of the phase-scratch union)
constexpr int kFockWarpScratch = 100 + 16 + 10 + 10;  // W block, P_AB, pv_A, pv_B

// ---------------------------------------------------------------------------
// Cyclic Jacobi on a packed symmetric matrix (lower triangle, row i holds
// columns 0..i at i(i+1)/2) with deferred eigenvector accumulation.
//
// The sweeps only touch the packed matrix A (shared memory).  Every round's
// rotation parameters are recorded to a per-CTA list in global memory; the
// recorded rounds are then replayed onto the orbital matrix Ct (rows =
// orbitals) one AO-column tile at a time, with the tile held in shared
// memory.  Ct therefore crosses L2 once per flush instead of once per round.
// ---------------------------------------------------------------------------
struct JacobiShared {
  double c[kJacobiMaxPairs], s[kJacobiMaxPairs], t[kJacobiMaxPairs];
  int p[kJacobiMaxPairs], q[kJacobiMaxPairs];
};

__device__ __forceinline__ int packed(int i, int j) { return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i; }

// Round-robin pairing of round r (Ne even, index Ne-1 is padding when N is
// odd): pair 0 is (r, Ne-1), pair k >= 1 is (r+k, r-k) mod (Ne-1); p < q.
__device__ __forceinline__ void rr_pair(int r, int k, int Ne, int& p, int& q) {
  const int m = Ne - 1;
  if (k == 0) {
    p = r;
    q = m;
  } else {
    p = r + k;
    if (p >= m) p -= m;
    q = r - k;
    if (q < 0) q += m;
    if (p > q) { const int t = p; p = q; q = t; }
  }
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// Replay nrec recorded rounds (the first is global round g0) onto the N rows
// of Ct (ncols AO columns, row stride ldc).  Ct is processed in tiles of w AO columns (w a power of two, T laid out
// [row][w]); the rounds' (c, s) are streamed into the staging buffer St in
// chunks of rb rounds, double-buffered with cp.async.  cold: Ct is the
// identity and is not read.  rank: when non-null, row k of the result is
// written to row rank[k] (eigenvalue order).
__device__ void replay_rotations(int N, int Ne, int npair, long long g0, int nrec, const double* __restrict__ rot,
                                 double* Ct, bool cold, const int* rank, double* T, int w, double* St, int rb,
                                 int ncols, int ldc) {
  const int tid = threadIdx.x, bd = blockDim.x;
  const int lw = __ffs(w) - 1;
  const int jj = tid & (w - 1), k_first = tid >> lw, k_step = bd >> lw;
  const int round_doubles = 2 * npair;  // a multiple of 2: 16-byte chunks
  const int nchunk = (nrec + rb - 1) / rb;
  for (int j0 = 0; j0 < ncols; j0 += w) {
    const int wj = min(w, ncols - j0);
    auto stage = [&](int c) {
      const int g = c * rb, n = min(rb, nrec - g);
      const double* src = rot + (size_t)g * round_doubles;
      double* dst = St + (size_t)(c & 1) * rb * round_doubles;
      for (int e = tid; e < n * round_doubles / 2; e += bd) cp_async16(dst + 2 * e, src + 2 * e);
    };
    if (nchunk > 0) stage(0);
    cp_async_commit();
    for (int e = tid; e < N * w; e += bd) {
      const int k = e >> lw, j = e & (w - 1);
      T[e] = (j >= wj) ? 0.0 : cold ? (k == j0 + j ? 1.0 : 0.0) : Ct[(size_t)k * ldc + j0 + j];
    }
    for (int c = 0; c < nchunk; ++c) {
      if (c + 1 < nchunk) stage(c + 1);
      cp_async_commit();
      cp_async_wait_one();
      __syncthreads();
      const double* buf = St + (size_t)(c & 1) * rb * round_doubles;
      const int n = min(rb, nrec - c * rb);
      for (int g = 0; g < n; ++g) {
        const long long gg = g0 + (long long)c * rb + g;
        const int r = (int)(gg % (Ne - 1));
        const double* rc = buf + (size_t)g * round_doubles;
        if (jj < wj) {
          for (int k = k_first; k < npair; k += k_step) {
            const double sn = rc[npair + k];
            if (sn == 0.0) continue;
            int p, q;
            rr_pair(r, k, Ne, p, q);
            const double cs = rc[k];
            const double tp = T[(p << lw) + jj], tq = T[(q << lw) + jj];
            T[(p << lw) + jj] = cs * tp - sn * tq;
            T[(q << lw) + jj] = sn * tp + cs * tq;
          }
        }
        __syncthreads();
      }
    }
    cp_async_wait_all();
    __syncthreads();
    for (int e = tid; e < N * w; e += bd) {
      const int k = e >> lw, j = e & (w - 1);
      if (j < wj) Ct[(size_t)(rank ? rank[k] : k) * ldc + j0 + j] = T[e];
    }
    __syncthreads();
  }
}

// Split a shared region between the replay tile (N x w doubles) and the
// double-buffered staging of recorded rounds.  Region 'tile' may be separate
// (tile_bytes > 0) or carved from 'shared' (tile == nullptr).
struct ReplayPlan {
  double* T;
  int w;
  double* St;
  int rb;
};
__device__ __forceinline__ int pow2_floor(int x) { return x <= 0 ? 0 : 1 << (31 - __clz(x)); }
__device__ ReplayPlan plan_replay(int N, int npair, double* tile, size_t tile_bytes, double* shared,
                                  size_t shared_bytes, int max_w) {
  ReplayPlan pl;
  const size_t round_bytes = sizeof(double) * 2 * (size_t)npair;
  if (tile) {
    pl.T = tile;
    pl.w = min(max_w, pow2_floor((int)(tile_bytes / (sizeof(double) * N))));
    pl.St = shared;
    pl.rb = (int)(shared_bytes / (2 * round_bytes));
  } else {
    const size_t st_min = 2 * round_bytes;
    pl.w = min(max_w, pow2_floor((int)((shared_bytes - st_min) / (sizeof(double) * N))));
    pl.T = shared;
    const size_t tb = ((sizeof(double) * N * pl.w + 15) / 16) * 16;
    pl.St = shared + tb / sizeof(double);
    pl.rb = (int)((shared_bytes - tb) / (2 * round_bytes));
  }
  return pl;
}

// Diagonalise the packed A; Ct <- Ct J (all rotations), sorted by eigenvalue
// into eps / rows of Ct (N rows of ncols entries, row stride ldc; both
// default to N).  Returns the sweep count (-1 if not converged).
// U: the shared phase-scratch region (tiles and staging while A is alive);
// Afree: A's shared storage, reused as the tile of the last replay (or null).
__device__ int jacobi_diagonalise(int N, double* A, double* Ct, bool cold, double* rot, int cap_rounds,
                                  double* U, size_t U_bytes, double* Afree, size_t Afree_bytes, int* rank, double* eps,
                                  JacobiShared& js, double* red, int max_sweeps, double tol, int ncols = -1,
                                  int ldc = -1) {
  if (ncols < 0) ncols = N;
  if (ldc < 0) ldc = N;
  const int Ne = N + (N & 1);
  const int npair = Ne / 2;
  const int tid = threadIdx.x;
  long long g_all = 0, g0 = 0;
  int nrec = 0;
  bool identity = cold;
  int sweeps = -1;
  for (int sweep = 0; sweep < max_sweeps; ++sweep) {
    double offmax = 0;
    for (int r = 0; r < Ne - 1; ++r) {
      double* rc = rot + (size_t)nrec * 2 * npair;
      for (int k = tid; k < npair; k += blockDim.x) {
        int p, q;
        rr_pair(r, k, Ne, p, q);
        double c = 1, s = 0, t = 0;
        if (q < N) {
          const double apq = A[packed(q, p)];
          offmax = fmax(offmax, fabs(apq));
          if (apq != 0.0) {
            const double app = A[packed(p, p)], aqq = A[packed(q, q)];
            const double tau = (aqq - app) / (2.0 * apq);
            t = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
            c = 1.0 / sqrt(1.0 + t * t);
            s = t * c;
          }
        }
        js.p[k] = p;
        js.q[k] = q < N ? q : -1;
        js.c[k] = c;
        js.s[k] = s;
        js.t[k] = t;
        rc[k] = c;
        rc[npair + k] = s;
      }
      __syncthreads();
      // A <- J^T A J on 2x2 blocks (pair k1 rows, pair k2 columns), k2 <= k1:
      // the triangle of blocks is flattened over the CTA so every lane works
      const int nblk = npair * (npair + 1) / 2;
      for (int b = tid; b < nblk; b += blockDim.x) {
        int k1 = (int)((sqrtf(8.0f * (float)b + 1.0f) - 1.0f) * 0.5f);
        while (k1 * (k1 + 1) / 2 > b) --k1;
        while ((k1 + 1) * (k1 + 2) / 2 <= b) ++k1;
        const int k2 = b - k1 * (k1 + 1) / 2;
        const int p1 = js.p[k1], q1 = js.q[k1];
        const double c1 = js.c[k1], s1 = js.s[k1];
        {
          const int p2 = js.p[k2], q2 = js.q[k2];
          if (k1 == k2) {
            if (q1 < 0) continue;
            const double t = js.t[k1];
            const int ipq = packed(q1, p1);
            const double apq = A[ipq];
            A[packed(p1, p1)] -= t * apq;
            A[packed(q1, q1)] += t * apq;
            A[ipq] = 0.0;
            continue;
          }
          const double c2 = js.c[k2], s2 = js.s[k2];
          if (s1 == 0.0 && s2 == 0.0) continue;
          const double m00 = A[packed(p1, p2)];
          const double m01 = q2 >= 0 ? A[packed(p1, q2)] : 0.0;
          const double m10 = q1 >= 0 ? A[packed(q1, p2)] : 0.0;
          const double m11 = (q1 >= 0 && q2 >= 0) ? A[packed(q1, q2)] : 0.0;
          const double x00 = c1 * m00 - s1 * m10, x01 = c1 * m01 - s1 * m11;
          const double x10 = s1 * m00 + c1 * m10, x11 = s1 * m01 + c1 * m11;
          A[packed(p1, p2)] = x00 * c2 - x01 * s2;
          if (q2 >= 0) A[packed(p1, q2)] = x00 * s2 + x01 * c2;
          if (q1 >= 0) A[packed(q1, p2)] = x10 * c2 - x11 * s2;
          if (q1 >= 0 && q2 >= 0) A[packed(q1, q2)] = x10 * s2 + x11 * c2;
        }
      }
      __syncthreads();
      ++nrec;
      ++g_all;
      if (nrec == cap_rounds) {
        const ReplayPlan pl = plan_replay(N, npair, nullptr, 0, U, U_bytes, 32);
        replay_rotations(N, Ne, npair, g0, nrec, rot, Ct, identity, nullptr, pl.T, pl.w, pl.St, pl.rb, ncols, ldc);
        identity = false;
        g0 = g_all;
        nrec = 0;
      }
    }
    offmax = cta_max(offmax, red);
    if (offmax < tol) {
      sweeps = sweep + 1;
      break;
    }
  }
  // eigenvalues and ranks (A still alive), then the final replay with sorting.
  // The order compares eigenvalues on a 1e-9 Hartree grid and breaks ties by
  // the current index: orbitals that are degenerate to rounding keep their
  // order from one diagonalisation to the next (a half-filled degenerate
  // shell then keeps the same occupied member, as a stable eigensolver
  // would), and the ranks still form a permutation.
  for (int k = tid; k < N; k += blockDim.x) {
    const double ek = A[packed(k, k)];
    const long long qk = __double2ll_rd(ek * 1e9);
    int rk = 0;
    for (int j = 0; j < N; ++j) {
      const long long qj = __double2ll_rd(A[packed(j, j)] * 1e9);
      rk += (qj < qk || (qj == qk && j < k)) ? 1 : 0;
    }
    eps[rk] = ek;
    rank[k] = rk;
  }
  __syncthreads();
  const ReplayPlan pl = Afree ? plan_replay(N, npair, Afree, Afree_bytes, U, U_bytes, 64)
                              : plan_replay(N, npair, nullptr, 0, U, U_bytes, 32);
  replay_rotations(N, Ne, npair, g0, nrec, rot, Ct, identity, rank, pl.T, pl.w, pl.St, pl.rb, ncols, ldc);
  return sweeps;
}

// ---------------------------------------------------------------------------
// Persistent SCF kernel
// ---------------------------------------------------------------------------
struct ScfShared {
  double red[32];
  double bmat[kDiisMax * kDiisMax];
  double sys[(kDiisMax + 1) * (kDiisMax + 2)];
  double coef[kDiisMax + 1];
  double scal[4];
  int mol;
  int diis_ok;
  int flag;
  int pad;
  int rank[2 * kJacobiMaxPairs];
  // phase scratch: GEMM stages, Fock-build warp buffers and Jacobi rotations
  // are never live at the same time
  union __align__(16) {
    double gemm[2 * kGemmStages * kGemmStage];
    double fockw[(kScfThreads / 32) * (kFockWarpScratch > 320 ? kFockWarpScratch : 320)];
    JacobiShared js;
  };
};

// q-th tile (a, b), a >= b, of the lower triangle of tiles in row-major order.
__device__ __forceinline__ void tri_decode(int q, int& a, int& b) {
  int r = (int)((sqrtf(8.0f * (float)q + 1.0f) - 1.0f) * 0.5f);
  while (r * (r + 1) / 2 > q) --r;
  while ((r + 1) * (r + 2) / 2 <= q) ++r;
  a = r;
  b = q - r * (r + 1) / 2;
}

// Pulay DIIS: store (F, FP - PF) in the ring, extend the B matrix, solve.
// Returns the extrapolated Fock matrix (F itself or dst).  The ring keeps the
// error vectors E = FP - PF (antisymmetric) as their strict upper triangles
// and the Fock matrices (symmetric) as their upper triangles, row by row:
// half the traffic of full matrices, and the dot products <E_i, E_j> are
// twice the upper-triangle sums (a common factor the extrapolation ignores).
__device__ __forceinline__ int diis_row_e(int N, int i) { return i * (N - 1) - i * (i - 1) / 2; }
__device__ __forceinline__ int diis_row_f(int N, int i) { return i * N - i * (i - 1) / 2; }

// One spin's store pass: F and E = W - W^T (W = FP) into ring slot `slot`,
// with <E, E_j> for every stored error vector j accumulated into d (the new
// one is E itself).  The error vectors only enter the B matrix: they are kept
// in FP32 (half the ring traffic; relative precision 6e-8 at any magnitude),
// the Fock matrices that are combined stay FP64.
__device__ __forceinline__ void diis_store(int N, const double* F, const double* W, double* histF, double* histE,
                                           int slot, int nhist, double (&d)[kDiisMax]) {
  const int TE = N * (N - 1) / 2, TF = N * (N + 1) / 2;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  float* hE = reinterpret_cast<float*>(histE);
  float* eS = hE + (size_t)slot * TE;
  double* fS = histF + (size_t)slot * TF;
  for (int i = warp; i < N; i += nwarps) {
    const int re = diis_row_e(N, i) - i - 1, rf = diis_row_f(N, i) - i;
    for (int c = i + lane; c < N; c += 32) {
      fS[rf + c] = F[i * N + c];
      if (c == i) continue;
      const float ef = (float)(W[i * N + c] - W[c * N + i]);
      eS[re + c] = ef;
      const double e = (double)ef;
#pragma unroll
      for (int j = 0; j < kDiisMax; ++j)
        if (j < nhist) d[j] += e * (j == slot ? e : (double)hE[(size_t)j * TE + re + c]);
    }
  }
}

// CTA reduction of the dot products into row and column `slot` of the B
// matrix, then the solve for the coefficients (sh.coef).  False when there is
// nothing to extrapolate (fewer than two entries, error vectors at rounding
// level, or a singular system).
__device__ __forceinline__ bool diis_solve(int slot, int nhist, double (&d)[kDiisMax], ScfShared& sh) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  double* part = sh.gemm;  // idle GEMM scratch
#pragma unroll
  for (int j = 0; j < kDiisMax; ++j) d[j] = warp_sum(d[j]);
  if (lane == 0)
#pragma unroll
    for (int j = 0; j < kDiisMax; ++j) part[warp * kDiisMax + j] = d[j];
  __syncthreads();
  if (tid < nhist) {
    double b = 0;
    for (int w = 0; w < nwarps; ++w) b += part[w * kDiisMax + tid];
    sh.bmat[slot * kDiisMax + tid] = b;
    sh.bmat[tid * kDiisMax + slot] = b;
  }
  __syncthreads();
  if (nhist < 2) return false;
  if (tid == 0) {
    const int n = nhist, ld = n + 2;
    double scale = 0;
    for (int i = 0; i < n; ++i) scale = fmax(scale, fabs(sh.bmat[i * kDiisMax + i]));
    int ok = scale > kDiisNoiseNorm ? 1 : 0;
    scale = scale > 0 ? 1.0 / scale : 1.0;
    for (int i = 0; i <= n; ++i)
      for (int j = 0; j <= n; ++j) {
        double v;
        if (i < n && j < n) v = sh.bmat[i * kDiisMax + j] * scale;
        else if (i == n && j == n) v = 0;
        else v = -1;
        sh.sys[i * ld + j] = v;
      }
    for (int i = 0; i <= n; ++i) sh.sys[i * ld + n + 1] = (i == n) ? -1.0 : 0.0;
    for (int c = 0; c <= n && ok; ++c) {
      int piv = c;
      for (int r = c + 1; r <= n; ++r)
        if (fabs(sh.sys[r * ld + c]) > fabs(sh.sys[piv * ld + c])) piv = r;
      if (fabs(sh.sys[piv * ld + c]) < 1e-300) { ok = 0; break; }
      if (piv != c)
        for (int k = 0; k <= n + 1; ++k) {
          double t = sh.sys[c * ld + k];
          sh.sys[c * ld + k] = sh.sys[piv * ld + k];
          sh.sys[piv * ld + k] = t;
        }
      for (int r = c + 1; r <= n; ++r) {
        double f = sh.sys[r * ld + c] / sh.sys[c * ld + c];
        for (int k = c; k <= n + 1; ++k) sh.sys[r * ld + k] -= f * sh.sys[c * ld + k];
      }
    }
    if (ok) {
      for (int c = n; c >= 0; --c) {
        double s = sh.sys[c * ld + n + 1];
        for (int k = c + 1; k <= n; ++k) s -= sh.sys[c * ld + k] * sh.coef[k];
        sh.coef[c] = s / sh.sys[c * ld + c];
      }
      for (int i = 0; i < n; ++i)
        if (!isfinite(sh.coef[i])) ok = 0;
    }
    sh.diis_ok = ok;
  }
  __syncthreads();
  return sh.diis_ok != 0;
}

// dst = sum_i c_i F_i from the packed upper triangles, written to both halves.
__device__ __forceinline__ void diis_extrapolate(int N, const double* histF, int nhist, double* dst,
                                                 ScfShared& sh) {
  const int TF = N * (N + 1) / 2;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (int i = warp; i < N; i += nwarps) {
    const int rf = diis_row_f(N, i) - i;
    for (int c = i + lane; c < N; c += 32) {
      // the ring's entries are independent loads: all in flight at once
      double f[kDiisMax];
#pragma unroll
      for (int k = 0; k < kDiisMax; ++k) f[k] = k < nhist ? histF[(size_t)k * TF + rf + c] : 0.0;
      double v = 0;
#pragma unroll
      for (int k = 0; k < kDiisMax; ++k)
        if (k < nhist) v += sh.coef[k] * f[k];
      dst[i * N + c] = v;
      dst[c * N + i] = v;
    }
  }
  __syncthreads();
}

// Profiling builds: thread 0 adds the cycles since *t to prof[k] and moves *t on.
__device__ __forceinline__ void prof_mark(long long* prof, int k, long long& t) {
  if (prof && threadIdx.x == 0) {
    const long long now = clock64();
    prof[k] += now - t;
    t = now;
  }
}

// prof (optional): cycles of the FP product, the store pass, the solve and
// the extrapolation added to prof[0..3].
__device__ const double* diis_step(int N, const double* F, const double* P, double* W, double* dst, double* histF,
                                   double* histE, int msize, int& nhist, int& head, ScfShared& sh,
                                   long long* prof = nullptr) {
  long long t = clock64();
  cta_gemm(N, N, N, 1.0, F, N, false, P, N, false, 0.0, W, N, sh.gemm);  // W = FP
  prof_mark(prof, 0, t);
  const int slot = head;
  head = (head + 1) % msize;
  if (nhist < msize) ++nhist;
  double d[kDiisMax];
#pragma unroll
  for (int j = 0; j < kDiisMax; ++j) d[j] = 0.0;
  diis_store(N, F, W, histF, histE, slot, nhist, d);
  prof_mark(prof, 1, t);
  const bool ok = diis_solve(slot, nhist, d, sh);
  prof_mark(prof, 2, t);
  if (!ok) return F;
  diis_extrapolate(N, histF, nhist, dst, sh);
  prof_mark(prof, 3, t);
  return dst;
}

// Unrestricted DIIS: one B matrix over the stacked error vectors of both
// spins, <E_i, E_j> = <Ea_i, Ea_j> + <Eb_i, Eb_j>, and one set of coefficients
// for both Fock matrices, which are replaced in place by the extrapolations
// (left unchanged when there is nothing to extrapolate).  W scratch.
__device__ void diis_step_uhf(int N, double* Fa, const double* Pa, double* Fb, const double* Pb, double* W,
                              double* histFa, double* histEa, double* histFb, double* histEb, int msize, int& nhist,
                              int& head, ScfShared& sh) {
  const int slot = head;
  head = (head + 1) % msize;
  if (nhist < msize) ++nhist;
  double d[kDiisMax];
#pragma unroll
  for (int j = 0; j < kDiisMax; ++j) d[j] = 0.0;
  cta_gemm(N, N, N, 1.0, Fa, N, false, Pa, N, false, 0.0, W, N, sh.gemm);
  diis_store(N, Fa, W, histFa, histEa, slot, nhist, d);
  __syncthreads();
  cta_gemm(N, N, N, 1.0, Fb, N, false, Pb, N, false, 0.0, W, N, sh.gemm);
  diis_store(N, Fb, W, histFb, histEb, slot, nhist, d);
  if (!diis_solve(slot, nhist, d, sh)) return;
  diis_extrapolate(N, histFa, nhist, Fa, sh);
  diis_extrapolate(N, histFb, nhist, Fb, sh);
}

// Full diagonalisation of Fx (held in F) into orbital-major Ct, sorted by energy.
// Cold: Ct = I and A = F.  Warm: A = C^T F C from the current Ct.  A is the
// packed lower triangle, in shared memory (Abytes > 0 reserved there) or, when
// it does not fit, in F (free once the transform is done).  W1, W2 scratch.
__device__ int full_diagonalise(int N, double* F, double* Ct, double* W1, double* W2, double* eps, double* A,
                                size_t A_smem_bytes, bool warm, double* rot, int cap_rounds, int max_sweeps,
                                double tol, ScfShared& sh) {
  const int tid = threadIdx.x;
  const double* src;
  if (warm) {
    cta_gemm(N, N, N, 1.0, F, N, false, Ct, N, true, 0.0, W1, N, sh.gemm);  // F C
    cta_gemm(N, N, N, 1.0, Ct, N, false, W1, N, false, 0.0, W2, N, sh.gemm, true);  // C^T F C
    src = W2;
  } else {
    src = F;
    if (A == F) {
      const size_t NN = (size_t)N * N;
      for (size_t k = tid; k < NN; k += blockDim.x) W2[k] = F[k];
      __syncthreads();
      src = W2;
    }
  }
  for (int e = tid; e < N * (N + 1) / 2; e += blockDim.x) {
    int i = (int)((sqrt(8.0 * e + 1.0) - 1.0) * 0.5);
    while ((i + 1) * (i + 2) / 2 <= e) ++i;
    while (i * (i + 1) / 2 > e) --i;
    const int j = e - i * (i + 1) / 2;
    A[e] = 0.5 * (src[(size_t)i * N + j] + src[(size_t)j * N + i]);
  }
  __syncthreads();
  // replay tiles: the phase-scratch union while A lives; A's shared storage
  // (when it holds at least 32 columns) for the last replay
  double* Afree = A_smem_bytes >= sizeof(double) * 32 * (size_t)N ? A : nullptr;
  return jacobi_diagonalise(N, A, Ct, !warm, rot, cap_rounds, sh.gemm, sizeof(sh.gemm), Afree, A_smem_bytes, sh.rank,
                            eps, sh.js, sh.red, max_sweeps, tol);
}

// Occupied-virtual rotation of Ct toward the eigenvectors of F (second order).
// Returns 1 when the occupied/virtual ordering is broken or the step is too
// large (a full diagonalisation is needed instead); Ct is unchanged then.
// F holds the (extrapolated) Fock matrix on entry and is used as scratch.
// Scratch: W1 (N x N), W2 (N x N).  eps receives diag(C^T F C).
// prof (optional): cycles of C^T F with the diagonal, the X step and its
// quadratic terms, the rotation product, the re-orthonormalisation added to
// prof[0..3].
// swaps (optional): instead of copying the rotated orbitals back into Ct, the
// function leaves them where the product put them and reports it: bit 0 set
// when they moved to F's buffer (Ct's buffer is then free for F's role), bit 1
// when a re-orthonormalisation then moved them on to W2's buffer (the caller
// exchanges the buffer roles in that order).
__device__ int ov_rotation(int N, int no, double* F, double* Ct, double* W1, double* W2, double* eps, double& drift,
                           ScfShared& sh, long long* prof = nullptr, int* swaps = nullptr) {
  const int nv = N - no;
  const size_t NN = (size_t)N * N;
  const int tid = threadIdx.x;
  if (no == 0 || nv == 0) return 0;
  long long tprof = clock64();
  cta_gemm(N, N, N, 1.0, Ct, N, false, F, N, false, 0.0, W1, N, sh.gemm);  // W1 = C^T F (row k = c_k^T F)
  {
    const int lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    for (int k = warp; k < N; k += nwarps) {
      double s = 0;
#pragma unroll 4
      for (int nu = lane; nu < N; nu += 32) s += W1[(size_t)k * N + nu] * Ct[(size_t)k * N + nu];
      s = warp_sum(s);
      if (lane == 0) eps[k] = s;
    }
  }
  __syncthreads();
  double homo = -1e300, lumo = 1e300;
  for (int k = tid; k < N; k += blockDim.x) {
    if (k < no) homo = fmax(homo, eps[k]);
    else lumo = fmin(lumo, eps[k]);
  }
  homo = cta_max(homo, sh.red);
  lumo = -cta_max(-lumo, sh.red);
  prof_mark(prof, 0, tprof);
  if (!(homo < lumo - 1e-4)) return 1;
  // X (nv x no) = F_vo / (e_i - e_a), F_vo[a][i] = c_a^T F c_i = sum_nu Ct[a][nu] W1[i][nu]
  double* X = W2;
  cta_gemm(nv, no, N, 1.0, Ct + (size_t)no * N, N, false, W1, N, true, 0.0, X, no, sh.gemm);
  double xmax = 0;
#pragma unroll 4
  for (int e = tid; e < nv * no; e += blockDim.x) {
    const int a = e / no, i = e % no;
    double d = eps[i] - eps[no + a];
    if (d > -0.02) d = -0.02;  // level-shift guard for a tiny gap
    const double x = X[e] / d;
    X[e] = x;
    xmax = fmax(xmax, fabs(x));
  }
  xmax = cta_max(xmax, sh.red);
  if (xmax > 0.5) return 1;
  // Ct <- M Ct with M = I + K + K^2/2, K = [[0, X^T], [-X, 0]] (orbital space):
  //   M = [[I - X^T X / 2, X^T], [-X, I - X X^T / 2]], assembled in W1
  cta_gemm(no, no, nv, -0.5, X, no, true, X, no, false, 0.0, W1, N, sh.gemm, true);
  cta_gemm(nv, nv, no, -0.5, X, no, false, X, no, true, 0.0, W1 + (size_t)no * N + no, N, sh.gemm, true);
#pragma unroll 4
  for (int e = tid; e < nv * no; e += blockDim.x) {
    const int a = e / no, i = e % no;
    W1[(size_t)i * N + no + a] = X[e];
    W1[(size_t)(no + a) * N + i] = -X[e];
  }
  for (int k = tid; k < N; k += blockDim.x) W1[(size_t)k * N + k] += 1.0;
  __syncthreads();
  prof_mark(prof, 1, tprof);
  cta_gemm(N, N, N, 1.0, W1, N, false, Ct, N, false, 0.0, F, N, sh.gemm);
  if (swaps) {
    double* t = Ct;
    Ct = F;
    F = t;
    *swaps |= 1;
  } else {
    for (size_t e = tid; e < NN; e += blockDim.x) Ct[e] = F[e];
    __syncthreads();
  }
  prof_mark(prof, 2, tprof);
  // the second-order rotation is orthogonal up to |K|^4 / 4: re-orthonormalise when needed
  drift += 0.25 * xmax * xmax * xmax * xmax;
  if (drift > 1e-12) {
    // S = Ct Ct^T, Ct <- (3/2 I - 1/2 S) Ct  (Newton-Schulz step for S^-1/2)
    for (size_t e = tid; e < NN; e += blockDim.x) W1[e] = 0.0;
    __syncthreads();
    for (int k = tid; k < N; k += blockDim.x) W1[(size_t)k * N + k] = 1.5;
    __syncthreads();
    cta_gemm(N, N, N, -0.5, Ct, N, false, Ct, N, true, 1.0, W1, N, sh.gemm, true);
    cta_gemm(N, N, N, 1.0, W1, N, false, Ct, N, false, 0.0, W2, N, sh.gemm);
    if (swaps) {
      *swaps |= 2;
    } else {
      for (size_t e = tid; e < NN; e += blockDim.x) Ct[e] = W2[e];
      __syncthreads();
    }
    drift = 0;
    prof_mark(prof, 3, tprof);
  }
  return 0;
}

// Dynamic shared memory of the launch (bytes).
__device__ __forceinline__ unsigned dynamic_smem_bytes() {
  unsigned r;
  asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(r));
  return r;
}

}  // namespace
}  // namespace sgb

#include "eigh_tridiag.cuh"

namespace sgb {
namespace {

// Doubles of the eigensolver's shared workspace: the phase-scratch union and
// everything after it in the dynamic shared memory (the packed-matrix region).
__device__ __forceinline__ size_t eig_workspace_doubles(const ScfShared& sh, const unsigned char* smem_raw) {
  const size_t off = (size_t)(reinterpret_cast<const unsigned char*>(sh.gemm) - smem_raw);
  const size_t total = dynamic_smem_bytes();
  return total > off ? (total - off) / sizeof(double) : 0;
}

}  // namespace
// New orbitals of one spin from its (extrapolated) Fock matrix Fs: the
// occupied-virtual rotation of the previous orbitals, or a full
// diagonalisation at the start, when the rotation asks for one, and when
// the spin has no occupied or no virtual orbitals.  Returns the Jacobi
// sweeps of a full diagonalisation (0 when none ran, < 0 when it did not
// converge).
// Unless sp selects the rotation mode for this size, a full diagonalisation
// runs the tridiagonal solver first (ws: its shared workspace of ws_doubles)
// and falls back to a cold Jacobi on clustered spectra.
__device__ int uhf_orbitals(int N, int ns, double* Fs, double* Cs, double* W1, double* W2, double* epss,
                            double* Apk, size_t packed_bytes, bool& have, double& drift, double* rot, int cap_rounds,
                            const ScfParams& sp, int cold_sweeps, int& nfull, ScfShared& sh, double* ws,
                            size_t ws_doubles) {
  int need_full = !have || ns == 0 || ns == N;
  if (!need_full) need_full = ov_rotation(N, ns, Fs, Cs, W1, W2, epss, drift, sh);
  if (!need_full) return 0;
  if (scf_eig_mode(sp, N) != kEigRotation) {
    if (eigh_tridiag(N, Fs, N, N, Cs, N, epss, ws, ws_doubles, W2, W1, Cs, Fs, sh.red, &sh.flag) == 0) {
      ++nfull;
      have = true;
      drift = 0;
      return 0;
    }
    have = false;  // the solver used Cs as scratch: the fallback starts cold
  }
  const int sw = full_diagonalise(N, Fs, Cs, W1, W2, epss, Apk ? Apk : Fs, Apk ? packed_bytes : 0, have, rot,
                                  cap_rounds, have ? sp.jacobi_max_sweeps : cold_sweeps, have ? 1e-10 : 1e-3, sh);
  ++nfull;
  const bool warm = have;
  have = true;
  drift = 0;
  return sw < 0 ? (warm ? -sp.jacobi_max_sweeps : cold_sweeps) : sw;
}

// P_s = C_occ C_occ^T of one spin into Ps; returns sum (P_s,new - P_s,old)^2.
__device__ double uhf_density(int N, int ns, const double* Cs, double* Ps, double* W1, ScfShared& sh) {
  const size_t NN = (size_t)N * N;
  if (ns > 0) {
    cta_gemm(N, N, ns, 1.0, Cs, N, true, Cs, N, false, 0.0, W1, N, sh.gemm, true);
  } else {
    for (size_t k = threadIdx.x; k < NN; k += blockDim.x) W1[k] = 0.0;
    __syncthreads();
  }
  double d2 = 0;
  for (size_t k = threadIdx.x; k < NN; k += blockDim.x) {
    const double d = W1[k] - Ps[k];
    d2 += d * d;
    Ps[k] = W1[k];
  }
  return cta_sum(d2, sh.red);
}

}  // namespace sgb
