// CTA-wide symmetric eigensolver of the per-molecule SCF kernels: one
// molecule's Fock matrix (N <= 1024) diagonalised by one thread block.
//
//   1. Householder tridiagonalisation A = Q T Q^T (lower, one reflector per
//      column, the LAPACK dsytd2 sequence).  A is held as the lower triangle
//      of 32 x 32 tiles (diagonal tiles in full, row stride 33 so that row and
//      column walks are both free of bank conflicts), in shared memory when
//      it fits and in global scratch otherwise.  Per column: the reflector by
//      one warp; the symmetric product p = tau A v by tiles (a warp per tile,
//      a lane per tile row for T v_J and per tile column for T^T v_I, no
//      shuffles), the tile partials summed per row; then the rank-2 update
//      of the trailing tiles.  v and w are zero outside the trailing block,
//      so whole tiles are processed without masks.
//   2. Eigenvalues of T by multisection: S lanes per eigenvalue evaluate S
//      points of its bracket, a warp ballot picks the sub-interval; the
//      Sturm count is division-free (three-term recurrence of the leading
//      principal minors, rescaled by powers of two every four steps).
//   3. Eigenvectors of T for the lowest nvec eigenvalues by one twisted
//      factorisation each (a thread per vector): forward and backward
//      stationary factorisations of T - lambda I, twist index at the
//      smallest |gamma_r|, the vector filled outward from z_r = 1 (Dhillon &
//      Parlett, "Orthogonal eigenvectors and relative gaps", SIAM J. Matrix
//      Anal. Appl. 25, 2003).  Scratch is column-major (coalesced).
//   4. Back-transformation x = Q z with the reflectors grouped in fours,
//      each group applied as I - V T V^T (compact WY, forward columnwise T):
//      a warp per vector, the vector in registers.
//
// Vectors of eigenvalues closer than 1e-5 ||T|| to a neighbour are checked
// for mutual orthogonality; a (near-)degenerate cluster whose twisted vectors
// are not orthogonal, or a degenerate frontier between vector nvec-1 and
// nvec, makes the solver return 1 and the caller diagonalises with its
// Jacobi solver instead.  This replaces the reference's delegation of the
// eigenproblem to its SCF library (the self-adjoint eigensolver used by
// scine_utilities, hooked at Nddo/Pm6/PM6Method.cpp:27-41): the same
// eigenpairs, sorted ascending.
#pragma once
#include <cuda_runtime.h>

#include <cfloat>

namespace sgb {
namespace {

constexpr int kTileLd = 33;                 // row stride of a 32 x 32 tile
constexpr int kTileDoubles = 32 * kTileLd;  // one tile
constexpr int kEigMaxS = 8;                 // lanes per eigenvalue in the multisection

__device__ __forceinline__ int tri_index(int I, int J) { return I * (I + 1) / 2 + J; }
// element (i, j) of the tiled lower triangle, i/32 >= j/32
__device__ __forceinline__ int tile_elem(int i, int j) {
  return tri_index(i >> 5, j >> 5) * kTileDoubles + (i & 31) * kTileLd + (j & 31);
}
__device__ __forceinline__ size_t tiled_doubles(int N) {
  const int nt = (N + 31) >> 5;
  return (size_t)tri_index(nt, 0) * kTileDoubles;
}
// (tri_decode, the q-th lower tile in row-major order, comes with the SCF helpers)

// Number of eigenvalues of T (diagonal d, squared off-diagonal e2) below x:
// sign changes of the leading principal minors of T - x I.  The minors are
// rescaled by 2^-600 / 2^600 every four steps (exact, signs kept); within
// four steps they grow or shrink by far less than 2^400 for |T| < 1e20.
__device__ __forceinline__ int sturm_count(int N, const double* d, const double* e2, double x) {
  double p0 = 1.0, p1 = d[0] - x;
  int neg1 = __double2hiint(p1) < 0 ? 1 : 0;
  int cnt = neg1;
  int i = 1;
  for (; i + 3 < N; i += 4) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const double p2 = fma(d[i + u] - x, p1, -e2[i + u - 1] * p0);
      const int neg2 = __double2hiint(p2) < 0 ? 1 : 0;
      cnt += neg2 ^ neg1;
      neg1 = neg2;
      p0 = p1;
      p1 = p2;
    }
    const int ex = (__double2hiint(p1) >> 20) & 0x7ff;
    const int ex0 = (__double2hiint(p0) >> 20) & 0x7ff;
    if (ex > 1023 + 600 || ex0 > 1023 + 600) {
      p0 *= 0x1p-600;
      p1 *= 0x1p-600;
    } else if (ex < 1023 - 600 && ex0 < 1023 - 600) {
      p0 *= 0x1p600;
      p1 *= 0x1p600;
    }
  }
  for (; i < N; ++i) {
    const double p2 = fma(d[i] - x, p1, -e2[i - 1] * p0);
    const int neg2 = __double2hiint(p2) < 0 ? 1 : 0;
    cnt += neg2 ^ neg1;
    neg1 = neg2;
    p0 = p1;
    p1 = p2;
  }
  return cnt;
}

// Householder reduction of the tiled A to T = (d, e); reflector k
// (tau[k], v = (1, A(k+2..N-1, k))) is left in column k.
// v, w: 32 * nt doubles each (zero outside the trailing block); part: 64
// doubles per tile.
__device__ __forceinline__ void tridiagonalise_tiles(int N, double* A, double* v, double* w, double* part, double* d,
                                                     double* e, double* tau, double* red) {
  const int tid = threadIdx.x, bd = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = bd >> 5;
  const int nt = (N + 31) >> 5, npad = 32 * nt;
  for (int i = tid; i < npad; i += bd) v[i] = w[i] = 0.0;
  __syncthreads();
  for (int k = 0; k + 2 < N; ++k) {
    const int k1 = k + 1;
    if (warp == 0) {
      const double alpha = A[tile_elem(k1, k)];
      double s = 0.0;
      for (int i = k + 2 + lane; i < N; i += 32) {
        const double x = A[tile_elem(i, k)];
        s += x * x;
      }
      s = warp_sum(s);
      double beta = alpha, t = 0.0, sc = 0.0;
      if (s > 0.0) {
        beta = -copysign(sqrt(alpha * alpha + s), alpha);
        t = (beta - alpha) / beta;
        sc = 1.0 / (alpha - beta);
      }
      for (int i = k + 2 + lane; i < N; i += 32) {
        const int ix = tile_elem(i, k);
        const double x = A[ix] * sc;
        A[ix] = x;
        v[i] = x;
      }
      if (lane == 0) {
        v[k] = 0.0;  // the previous step's unit entry leaves the trailing block
        v[k1] = 1.0;
        d[k] = A[tile_elem(k, k)];
        e[k] = beta;
        tau[k] = t;
      }
    }
    __syncthreads();
    const double t = tau[k];
    if (t == 0.0) continue;  // column already reduced: the trailing block is unchanged
    const int K0 = k1 >> 5, na = nt - K0, ntile = na * (na + 1) / 2;
    // tile partials of A v: rows of I (T v_J) and rows of J (T^T v_I, off-diagonal tiles)
    for (int q = warp; q < ntile; q += nw) {
      int a, b;
      tri_decode(q, a, b);
      const int I = K0 + a, J = K0 + b;
      const double* __restrict__ T = A + tri_index(I, J) * kTileDoubles;
      const double* __restrict__ vI = v + 32 * I;
      const double* __restrict__ vJ = v + 32 * J;
      double yr0 = 0.0, yr1 = 0.0, yc0 = 0.0, yc1 = 0.0;
      if (I != J) {
#pragma unroll 8
        for (int c = 0; c < 32; c += 2) {
          yr0 = fma(T[lane * kTileLd + c], vJ[c], yr0);
          yc0 = fma(T[c * kTileLd + lane], vI[c], yc0);
          yr1 = fma(T[lane * kTileLd + c + 1], vJ[c + 1], yr1);
          yc1 = fma(T[(c + 1) * kTileLd + lane], vI[c + 1], yc1);
        }
      } else {
#pragma unroll 8
        for (int c = 0; c < 32; c += 2) {
          yr0 = fma(T[lane * kTileLd + c], vJ[c], yr0);
          yr1 = fma(T[lane * kTileLd + c + 1], vJ[c + 1], yr1);
        }
      }
      double* pt = part + tri_index(I, J) * 64;
      pt[lane] = yr0 + yr1;
      pt[32 + lane] = yc0 + yc1;
    }
    __syncthreads();
    // p = t A v (sum of the partials), w = p - t/2 (p.v) v
    double s = 0.0;
    for (int i = k1 + tid; i < N; i += bd) {
      const int I = i >> 5, r = i & 31;
      double y = 0.0;
      for (int J = K0; J <= I; ++J) y += part[tri_index(I, J) * 64 + r];
      for (int I2 = I + 1; I2 < nt; ++I2) y += part[tri_index(I2, I) * 64 + 32 + r];
      const double p = t * y;
      w[i] = p;
      s += p * v[i];
    }
    s = cta_sum(s, red);
    const double al = -0.5 * t * s;
    for (int i = k1 + tid; i < N; i += bd) w[i] += al * v[i];
    __syncthreads();
    // A_s -= v w^T + w v^T on the trailing tiles (diagonal tiles in full)
    for (int q = warp; q < ntile; q += nw) {
      int a, b;
      tri_decode(q, a, b);
      const int I = K0 + a, J = K0 + b;
      // lane = tile column: v, w of the column in registers, of the row broadcast
      double* __restrict__ T = A + tri_index(I, J) * kTileDoubles + lane;
      const double* __restrict__ vI = v + 32 * I;
      const double* __restrict__ wI = w + 32 * I;
      const double vc = v[32 * J + lane], wc = w[32 * J + lane];
#pragma unroll 8
      for (int r = 0; r < 32; ++r) T[r * kTileLd] -= fma(vI[r], wc, wI[r] * vc);
    }
    __syncthreads();
    // w leaves the trailing block with this step: zero it (the next use is
    // behind the next step's barriers)
    for (int i = k1 + tid; i < N; i += bd) w[i] = 0.0;
  }
  if (tid == 0) {
    if (N >= 2) {
      d[N - 2] = A[tile_elem(N - 2, N - 2)];
      e[N - 2] = A[tile_elem(N - 1, N - 2)];
      d[N - 1] = A[tile_elem(N - 1, N - 1)];
      tau[N - 2] = 0.0;
    } else {
      d[0] = A[0];
    }
  }
  __syncthreads();
}

// Offset (doubles) of reflector group g in the group layout: group g holds
// reflectors 4g .. 4g+3 as rows i = 4g+1 .. N-1 of 4 values v_{4g+a}[i]
// (1 on the unit entry, 0 above it).
__device__ __forceinline__ int group_off(int N, int g) { return 4 * (g * (N - 1) - 2 * g * (g - 1)); }

// Forward columnwise T of each group of four reflectors (4g .. 4g+3):
// H_4g ... H_4g+3 = I - V T V^T, T upper triangular, 16 doubles per group;
// and the reflectors copied from the tiles into the group layout V.
__device__ __forceinline__ void group_factors(int N, const double* A, const double* tau, double* Tg, double* V) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int nref = N - 2, ngroup = nref > 0 ? (nref + 3) >> 2 : 0;
  for (int g = warp; g < ngroup; g += nw) {
    const int k0 = 4 * g;
    double* __restrict__ Vg = V + group_off(N, g);
    // dots v_a^T v_b, a < b within the group
    double dt[6] = {0, 0, 0, 0, 0, 0};
    for (int i = k0 + 1 + lane; i < N; i += 32) {
      double vv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        const int k = k0 + a;
        vv[a] = (k < nref) ? (i == k + 1 ? 1.0 : (i > k + 1 ? A[tile_elem(i, k)] : 0.0)) : 0.0;
        Vg[4 * (i - k0 - 1) + a] = vv[a];
      }
      dt[0] += vv[0] * vv[1];
      dt[1] += vv[0] * vv[2];
      dt[2] += vv[0] * vv[3];
      dt[3] += vv[1] * vv[2];
      dt[4] += vv[1] * vv[3];
      dt[5] += vv[2] * vv[3];
    }
#pragma unroll
    for (int q = 0; q < 6; ++q) dt[q] = warp_sum(dt[q]);
    if (lane == 0) {
      double T[4][4] = {};
      const double g01 = dt[0], g02 = dt[1], g03 = dt[2], g12 = dt[3], g13 = dt[4], g23 = dt[5];
      double ta[4];
      for (int a = 0; a < 4; ++a) ta[a] = (k0 + a < nref) ? tau[k0 + a] : 0.0;
      T[0][0] = ta[0];
      T[1][1] = ta[1];
      T[0][1] = -ta[1] * T[0][0] * g01;
      T[2][2] = ta[2];
      T[0][2] = -ta[2] * (T[0][0] * g02 + T[0][1] * g12);
      T[1][2] = -ta[2] * (T[1][1] * g12);
      T[3][3] = ta[3];
      T[0][3] = -ta[3] * (T[0][0] * g03 + T[0][1] * g13 + T[0][2] * g23);
      T[1][3] = -ta[3] * (T[1][1] * g13 + T[1][2] * g23);
      T[2][3] = -ta[3] * (T[2][2] * g23);
      for (int a = 0; a < 4; ++a)
        for (int b = 0; b < 4; ++b) Tg[16 * g + 4 * a + b] = T[a][b];
    }
  }
}

// x_k = Q z_k for the nvec vectors (column k of Z, column-major with leading
// dimension ldz, scaled by zscale[k]), written as rows of Ct.  A warp per
// pair of vectors, lane l holding elements l, l + 32, ... (N <= 32 * NR);
// the reflectors stream from the group layout V.
template <int NR>
__device__ __forceinline__ void back_transform_groups(int N, int nvec, const double* __restrict__ V,
                                                      const double* __restrict__ Tg, const double* __restrict__ Z,
                                                      int ldz, const double* __restrict__ zscale, double* Ct,
                                                      int ldc) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int nref = N - 2, ngroup = nref > 0 ? (nref + 3) >> 2 : 0;
  for (int kv = 2 * warp; kv < nvec; kv += 2 * nw) {
    const bool two = kv + 1 < nvec;
    double x0[NR], x1[NR];
    const double sc0 = zscale[kv], sc1 = two ? zscale[kv + 1] : 0.0;
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      const int i = lane + 32 * r;
      x0[r] = i < N ? sc0 * Z[(size_t)i * ldz + kv] : 0.0;
      x1[r] = (two && i < N) ? sc1 * Z[(size_t)i * ldz + kv + 1] : 0.0;
    }
    for (int g = ngroup - 1; g >= 0; --g) {
      const int k0 = 4 * g;
      const double* __restrict__ Vg = V + group_off(N, g) - 4 * (k0 + 1);  // Vg[4 i + a] = v_{k0+a}[i]
      double s0[4] = {0, 0, 0, 0}, s1[4] = {0, 0, 0, 0};
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        if (32 * r + 31 <= k0) continue;  // warp-uniform: the chunk lies above the group
        const int i = lane + 32 * r;
        if (i > k0 && i < N) {
#pragma unroll
          for (int a = 0; a < 4; ++a) {
            const double va = Vg[4 * i + a];
            s0[a] = fma(va, x0[r], s0[a]);
            s1[a] = fma(va, x1[r], s1[a]);
          }
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int a = 0; a < 4; ++a) {
          s0[a] += __shfl_xor_sync(0xffffffffu, s0[a], o);
          s1[a] += __shfl_xor_sync(0xffffffffu, s1[a], o);
        }
      }
      const double* T = Tg + 16 * g;
      double u0[4], u1[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        double c0 = 0.0, c1 = 0.0;
#pragma unroll
        for (int b = a; b < 4; ++b) {
          c0 = fma(T[4 * a + b], s0[b], c0);
          c1 = fma(T[4 * a + b], s1[b], c1);
        }
        u0[a] = c0;
        u1[a] = c1;
      }
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        if (32 * r + 31 <= k0) continue;
        const int i = lane + 32 * r;
        if (i > k0 && i < N) {
          double y0 = x0[r], y1 = x1[r];
#pragma unroll
          for (int a = 0; a < 4; ++a) {
            const double va = Vg[4 * i + a];
            y0 = fma(-va, u0[a], y0);
            y1 = fma(-va, u1[a], y1);
          }
          x0[r] = y0;
          x1[r] = y1;
        }
      }
    }
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      const int i = lane + 32 * r;
      if (i < N) {
        Ct[(size_t)kv * ldc + i] = x0[r];
        if (two) Ct[(size_t)(kv + 1) * ldc + i] = x1[r];
      }
    }
  }
}

// The same for any N: the vector in its row of Ct (global memory).
__device__ __forceinline__ void back_transform_groups_mem(int N, int nvec, const double* __restrict__ V,
                                                          const double* __restrict__ Tg,
                                                          const double* __restrict__ Z, int ldz,
                                                          const double* __restrict__ zscale, double* Ct, int ldc) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int nref = N - 2, ngroup = nref > 0 ? (nref + 3) >> 2 : 0;
  for (int kv = warp; kv < nvec; kv += nw) {
    double* x = Ct + (size_t)kv * ldc;
    const double sc = zscale[kv];
    for (int i = lane; i < N; i += 32) x[i] = sc * Z[(size_t)i * ldz + kv];
    __syncwarp();
    for (int g = ngroup - 1; g >= 0; --g) {
      const int k0 = 4 * g;
      const double* __restrict__ Vg = V + group_off(N, g) - 4 * (k0 + 1);
      double s[4] = {0, 0, 0, 0};
      for (int i = k0 + 1 + lane; i < N; i += 32) {
        const double xi = x[i];
#pragma unroll
        for (int a = 0; a < 4; ++a) s[a] = fma(Vg[4 * i + a], xi, s[a]);
      }
#pragma unroll
      for (int a = 0; a < 4; ++a) s[a] = warp_sum(s[a]);
      const double* T = Tg + 16 * g;
      double u[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        double acc = 0.0;
#pragma unroll
        for (int b = a; b < 4; ++b) acc = fma(T[4 * a + b], s[b], acc);
        u[a] = acc;
      }
      for (int i = k0 + 1 + lane; i < N; i += 32) {
        double xv = x[i];
#pragma unroll
        for (int a = 0; a < 4; ++a) xv = fma(-Vg[4 * i + a], u[a], xv);
        x[i] = xv;
      }
      __syncwarp();
    }
  }
}

// Shared-memory doubles the solver needs besides the tiled matrix: v, w,
// the tile partials, d, e, e2, tau, the vector scales and the group factors.
__device__ __forceinline__ size_t eig_small_doubles(int N) {
  const int nt = (N + 31) >> 5, npad = 32 * nt;
  const int ngroup = N > 2 ? (N + 1) / 4 + 1 : 1;
  return 7 * (size_t)npad + (size_t)tri_index(nt, 0) * 64 + 16 * (size_t)ngroup;
}

// Eigenvalues of the symmetric F (N x N, row-major; the upper triangle is
// read) ascending into eps[0..nvals-1], and the eigenvectors of the lowest
// nvec as rows 0..nvec-1 of Ct (row stride ldc).  ws: shared scratch of
// ws_doubles (16-byte aligned); gA: global scratch of at least N * N doubles
// (the tiled matrix when it does not fit ws); gZl, gZu: global scratch of at
// least N * nvec doubles each (gZu may alias Ct: it is dead before Ct is
// written); gV: global scratch of N * N doubles for the reflectors in group
// layout (may alias F: F is dead once the solver has decided not to fall
// back).  Returns 0, or 1 when the caller must use its
// fallback solver (clustered eigenvalues whose vectors came out
// non-orthogonal, a degenerate frontier between vector nvec-1 and nvec, a
// non-finite value, or too little shared scratch).  Every thread of the
// block calls it and gets the same result.  prof (optional, thread 0's):
// cycles of the four stages are added to prof[0..3] (tridiagonalisation,
// bisection, vectors with the cluster check, back-transformation).
__device__ __forceinline__ int eigh_tridiag(int N, const double* __restrict__ F, int nvals, int nvec, double* Ct,
                                            int ldc, double* eps, double* ws, size_t ws_doubles, double* gA,
                                            double* gZl, double* gZu, double* gV, double* red, int* flag,
                                            long long* prof = nullptr) {
  const int tid = threadIdx.x, bd = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = bd >> 5;
  long long tp0 = clock64();
  const int nt = (N + 31) >> 5, npad = 32 * nt;
  const size_t small = eig_small_doubles(N);
  if (small > ws_doubles) return 1;  // uniform
  double* v = ws;
  double* w = v + npad;
  double* part = w + npad;
  double* d = part + (size_t)tri_index(nt, 0) * 64;
  double* e = d + npad;
  double* e2 = e + npad;
  double* tau = e2 + npad;
  double* zscale = tau + npad;
  double* Tg = zscale + npad;
  const size_t tiles = tiled_doubles(N);
  const bool in_smem = small + tiles <= ws_doubles;
  double* A = in_smem ? ws + small : gA;
  // load the tiles from the rows of F (F symmetric): element (i, j) of tile
  // (I, J) is F[j][i]; lanes walk i, so the reads of F are coalesced
  for (int q = warp; q < tri_index(nt, 0); q += nw) {
    int I, J;
    tri_decode(q, I, J);
    double* T = A + (size_t)q * kTileDoubles;
    const int i = 32 * I + lane;
    for (int c = 0; c < 32; ++c) {
      const int j = 32 * J + c;
      T[lane * kTileLd + c] = (i < N && j < N) ? F[(size_t)j * N + i] : 0.0;
    }
  }
  if (tid == 0) *flag = 0;
  __syncthreads();
  tridiagonalise_tiles(N, A, v, w, part, d, e, tau, red);
  for (int i = tid; i + 1 < N; i += bd) e2[i] = e[i] * e[i];
  long long tp1 = clock64();
  if (prof && tid == 0) prof[0] += tp1 - tp0;

  // Gershgorin interval and the scale of T
  double lo = 1e300, hi = -1e300;
  for (int i = tid; i < N; i += bd) {
    const double r = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i + 1 < N ? fabs(e[i]) : 0.0);
    lo = fmin(lo, d[i] - r);
    hi = fmax(hi, d[i] + r);
  }
  lo = -cta_max(-lo, red);  // (its barriers also publish e2)
  hi = cta_max(hi, red);
  const double tnorm = fmax(fmax(fabs(lo), fabs(hi)), 1e-300);
  const double pad = 8.0 * DBL_EPSILON * tnorm * N;
  lo -= pad;
  hi += pad;
  // multisection: S lanes per eigenvalue, S a power of two
  int S = 1;
  while (S < kEigMaxS && 2 * S * nvals <= bd) S *= 2;
  const double width_tol = 4.0 * DBL_EPSILON * tnorm;
  int steps = 0;
  for (double wdt = hi - lo; wdt > width_tol && steps < 200; wdt /= (double)(S + 1)) ++steps;
  const int per_pass = bd / S;
  for (int base = 0; base < nvals; base += per_pass) {
    const int k = base + tid / S, s = tid % S;
    const bool act = k < nvals;
    const unsigned gmask = ((S == 32) ? 0xffffffffu : ((1u << S) - 1u)) << (lane & ~(S - 1));
    double a = lo, b = hi;
    for (int st = 0; st < steps; ++st) {
      const double h = (b - a) / (double)(S + 1);
      const double x = a + (double)(s + 1) * h;
      const int c = act ? sturm_count(N, d, e2, x) : 0;
      const unsigned bal = __ballot_sync(0xffffffffu, c <= k) & gmask;
      const int m = __popc(bal);
      const double na = a + (double)m * h;
      const double nb = (m == S) ? b : a + (double)(m + 1) * h;
      a = na;
      b = nb;
    }
    if (act && s == 0) eps[k] = 0.5 * (a + b);
  }
  __syncthreads();
  long long tp2 = clock64();
  if (prof && tid == 0) prof[1] += tp2 - tp1;

  // twisted-factorisation vectors of T, column-major: L+ and then z in
  // column k of gZl, U- in column k of gZu
  const double tiny = DBL_EPSILON * tnorm;
  const int ldz = nvec;
  double* __restrict__ Zl = gZl;
  double* __restrict__ Zu = gZu;
  for (int k = tid; k < nvec; k += bd) {
    const double lam = eps[k];
    int bad = 0;
    double ss = 1.0;
    if (N == 1) {
      Zl[k] = 1.0;
    } else {
      double Dp = d[0] - lam;
      for (int i = 0; i + 1 < N; ++i) {
        if (fabs(Dp) < tiny) Dp = Dp < 0.0 ? -tiny : tiny;
        const double l = e[i] / Dp;
        Zl[(size_t)i * ldz + k] = l;
        Dp = d[i + 1] - lam - l * e[i];
      }
      double Dm = d[N - 1] - lam;
      int r = N - 1;
      double best = fabs(Dm - Zl[(size_t)(N - 2) * ldz + k] * e[N - 2]);
#pragma unroll 4
      for (int i = N - 2; i >= 0; --i) {
        if (fabs(Dm) < tiny) Dm = Dm < 0.0 ? -tiny : tiny;
        const double u = e[i] / Dm;
        Zu[(size_t)i * ldz + k] = u;
        Dm = d[i] - lam - u * e[i];
        const double g = fabs(Dm - (i > 0 ? Zl[(size_t)(i - 1) * ldz + k] * e[i - 1] : 0.0));
        if (g < best) {
          best = g;
          r = i;
        }
      }
      double zz = 1.0;
#pragma unroll 4
      for (int i = r - 1; i >= 0; --i) {
        zz = -Zl[(size_t)i * ldz + k] * zz;
        Zl[(size_t)i * ldz + k] = zz;
        ss += zz * zz;
      }
      Zl[(size_t)r * ldz + k] = 1.0;
      zz = 1.0;
#pragma unroll 4
      for (int i = r + 1; i < N; ++i) {
        zz = -Zu[(size_t)(i - 1) * ldz + k] * zz;
        Zl[(size_t)i * ldz + k] = zz;
        ss += zz * zz;
      }
      if (!(ss < 1e300)) bad = 1;
    }
    zscale[k] = 1.0 / sqrt(ss);
    if (bad) *flag = 1;
  }
  __syncthreads();
  // clusters: vectors of (nearly) equal eigenvalues must come out orthogonal
  const double clus = 1e-5 * tnorm;
  for (int k = tid; k < nvec; k += bd) {
    for (int j = k + 1; j < nvec && eps[j] - eps[j - 1] < clus; ++j) {
      double s = 0.0;
      for (int i = 0; i < N; ++i) s += Zl[(size_t)i * ldz + k] * Zl[(size_t)i * ldz + j];
      if (!(fabs(s) * zscale[k] * zscale[j] < 1e-9)) *flag = 1;
    }
  }
  if (tid == 0 && nvec > 0 && nvec < nvals && !(eps[nvec] - eps[nvec - 1] >= clus)) *flag = 1;
  __syncthreads();
  const int failed = *flag;
  __syncthreads();  // every thread has read the flag before a later call resets it
  long long tp3 = clock64();
  if (prof && tid == 0) prof[2] += tp3 - tp2;
  if (failed) return 1;
  group_factors(N, A, tau, Tg, gV);
  __syncthreads();
  // the tiles are dead now: stage the reflectors' group layout in their
  // shared-memory place when the tiles lived there
  const int nref = N - 2, ngroup = nref > 0 ? (nref + 3) >> 2 : 0;
  const size_t vsize = (size_t)group_off(N, ngroup);
  const double* V = gV;
  if (in_smem && vsize <= tiles) {
    for (size_t q = tid; q < vsize; q += bd) A[q] = gV[q];
    __syncthreads();
    V = A;
  }
  if (N <= 128) back_transform_groups<4>(N, nvec, V, Tg, Zl, ldz, zscale, Ct, ldc);
  else if (N <= 256) back_transform_groups<8>(N, nvec, V, Tg, Zl, ldz, zscale, Ct, ldc);
  else back_transform_groups_mem(N, nvec, V, Tg, Zl, ldz, zscale, Ct, ldc);
  __syncthreads();
  if (prof && tid == 0) prof[3] += clock64() - tp3;
  return 0;
}

}  // namespace
}  // namespace sgb
