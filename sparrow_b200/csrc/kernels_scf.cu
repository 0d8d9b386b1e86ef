// One-electron assembly and the persistent batched SCF kernel.
//
// The SCF kernel runs one CTA per molecule: CTAs take molecules from a work
// counter (largest first) and iterate each to self-consistency on the device
// with no host round trips.  Per iteration (restricted, orthonormal NDDO
// basis):
//   F = H + G(P), E_el = 1/2 sum P (H + F)        TwoElectronMatrix.cpp:63-166,
//                                                 NDDOElectronicEnergyCalculator.cpp:48-67
//   Pulay DIIS on the commutator FP - PF          (restated; the reference's
//                                                 SCF driver is in scine_utilities)
//   new orbitals:
//     first iteration (and whenever the occupied/virtual ordering changes):
//       full diagonalisation by cyclic Jacobi with the packed matrix held in
//       shared memory, orbitals sorted by energy (aufbau: n_occ lowest)
//     later iterations: occupied-virtual rotation of the previous orbitals
//       (pseudo-diagonalisation): X_ai = F_ai / (e_i - e_a) from
//       F_mo = C^T F C, C <- C exp([[0, -X^T], [X, 0]]) to second order, with
//       a Newton-Schulz re-orthonormalisation when the second-order error can
//       exceed 1e-14.  The fixed point is the same (F_ov = 0 at
//       self-consistency), and every step is a dense GEMM.
//   P = 2 C_occ C_occ^T, convergence on |dE| and rms(dP)
// and, after convergence, G is rebuilt from the final density
// (FockMatrix::finalize, FockMatrix.cpp:147-150).
//
// Orbitals are stored orbital-major: Ct[k][mu] is the coefficient of AO mu in
// orbital k (so rotating two orbitals touches two contiguous rows).
#include <cuda_runtime.h>

#include <cstdio>

#include "kernels.h"
#include "nddo_math.cuh"
#include "scf_core.cuh"

namespace sgb {

// ---------------------------------------------------------------------------
// One-electron matrix, start density and repulsion energy (one CTA per molecule)
// ---------------------------------------------------------------------------
// H (OneElectronMatrix.cpp:43-134, both triangles):
//   same atom:  U on the diagonal + sum over other atoms B of V^B[p(mu,nu)]
//   two atoms:  1/2 (beta_mu + beta_nu) S_mu,nu
// start density (NDDODensityGuess.cpp:31-66): S * n_el / (2N) between atoms,
// zero within an atom off the diagonal, core charge / n_AO on the diagonal.
// Entries idx0, idx0 + step, ... of H (and of the start density when
// write_guess) of molecule m.
__device__ void one_electron_range(const MolDev& m, const AtomDev* __restrict__ atoms,
                                   const ElemDev* __restrict__ elems, const int* __restrict__ ao_atom,
                                   const double* __restrict__ vcore, const double* __restrict__ ovl, double* H,
                                   double* P, int write_guess, long long idx0, long long step) {
  const int N = m.nao;
  for (long long idx = idx0; idx < (long long)N * N; idx += step) {
    const int i = (int)(idx / N), j = (int)(idx % N);
    const int A = ao_atom[m.ao_base + i], B = ao_atom[m.ao_base + j];
    const AtomDev aA = atoms[A], aB = atoms[B];
    const ElemDev& eA = elems[aA.slot];
    const int mu = i - aA.ao0, nu = j - aB.ao0;
    double h, p;
    if (A == B) {
      h = (mu == nu) ? (mu == 0 ? eA.Uss : eA.Upp) : 0.0;
      const int a = A - m.atom0;
      const int pk = pair_index(mu, nu);
      for (int c = 0; c < m.nat; ++c) {
        if (c == a) continue;
        long long s = a < c ? pair_slot(m, a, c) : pair_slot(m, c, a);
        h += vcore[s * 20 + (a < c ? 0 : 10) + pk];
      }
      p = (mu == nu) ? eA.core / eA.nao : 0.0;
    } else {
      const ElemDev& eB = elems[aB.slot];
      const int a = A - m.atom0, b = B - m.atom0;
      double s = a < b ? ovl[pair_slot(m, a, b) * 16 + mu * 4 + nu] : ovl[pair_slot(m, b, a) * 16 + nu * 4 + mu];
      double ba = mu == 0 ? eA.betaS : eA.betaP, bb = nu == 0 ? eB.betaS : eB.betaP;
      h = 0.5 * (ba + bb) * s;
      p = s * m.nel / (2.0 * N);
    }
    H[idx] = h;
    if (write_guess) P[idx] = p;
  }
}

__global__ void __launch_bounds__(kScfThreads) k_one_electron(const MolDev* __restrict__ mols,
                                                              const AtomDev* __restrict__ atoms,
                                                              const ElemDev* __restrict__ elems,
                                                              const int* __restrict__ ao_atom,
                                                              const double* __restrict__ vcore,
                                                              const double* __restrict__ ovl,
                                                              const double* __restrict__ erep, double* Hall,
                                                              double* Pall, MolResult* res, int write_guess) {
  __shared__ double red[32];
  const MolDev m = mols[blockIdx.x];
  one_electron_range(m, atoms, elems, ao_atom, vcore, ovl, Hall + m.mat_off, Pall + m.mat_off, write_guess,
                     threadIdx.x, blockDim.x);
  double e = 0;
  for (int k = threadIdx.x; k < m.npairs; k += blockDim.x) e += erep[m.pair0 + k];
  e = cta_sum(e, red);
  if (threadIdx.x == 0) res[blockIdx.x].e_rep = e;
}

// The same for the single molecule of a batch over the whole grid; e_rep is
// accumulated into res[0].e_rep (zeroed by the launcher).
__global__ void __launch_bounds__(256) k_one_electron_grid(const MolDev* __restrict__ mols,
                                                           const AtomDev* __restrict__ atoms,
                                                           const ElemDev* __restrict__ elems,
                                                           const int* __restrict__ ao_atom,
                                                           const double* __restrict__ vcore,
                                                           const double* __restrict__ ovl,
                                                           const double* __restrict__ erep, double* H, double* P,
                                                           MolResult* res, int write_guess) {
  __shared__ double red[32];
  const MolDev m = mols[0];
  const long long gtid = blockIdx.x * (long long)blockDim.x + threadIdx.x, gthreads = (long long)gridDim.x * blockDim.x;
  one_electron_range(m, atoms, elems, ao_atom, vcore, ovl, H + m.mat_off, P + m.mat_off, write_guess, gtid, gthreads);
  double e = 0;
  for (long long k = gtid; k < m.npairs; k += gthreads) e += erep[m.pair0 + k];
  e = cta_sum(e, red);
  if (threadIdx.x == 0) atomicAdd(&res[0].e_rep, e);
}

void launch_one_electron(const DeviceBatch& b, cudaStream_t s) {
  if (b.nmol == 0) return;
  if (b.large) {
    // one large molecule: spread H over the whole GPU
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaMemsetAsync(&b.res[0].e_rep, 0, sizeof(double), s);
    k_one_electron_grid<<<sms * 4, 256, 0, s>>>(b.mols, b.atoms, b.elems, b.ao_atom, b.vcore, b.ovl, b.erep, b.H,
                                                b.P, b.res, b.use_guess);
    return;
  }
  k_one_electron<<<b.nmol, kScfThreads, 0, s>>>(b.mols, b.atoms, b.elems, b.ao_atom, b.vcore, b.ovl, b.erep, b.H,
                                                b.P, b.res, b.use_guess);
}

// ---------------------------------------------------------------------------
// Fock matrix F = H + G(P) and the electronic energy 1/2 sum P (H + F)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double one_centre_g(const ElemDev& e, int mu, int nu, const double* P, int N, int o) {
  auto Pm = [&](int i, int j) { return P[(o + i) * N + o + j]; };
  if (e.nao == 1) return 0.5 * Pm(0, 0) * e.gss;
  if (mu == nu) {
    if (mu == 0) return 0.5 * Pm(0, 0) * e.gss + (Pm(1, 1) + Pm(2, 2) + Pm(3, 3)) * (e.gsp - 0.5 * e.hsp);
    double g = Pm(0, 0) * (e.gsp - 0.5 * e.hsp) + 0.5 * Pm(mu, mu) * e.gpp;
    for (int q = 1; q < 4; ++q)
      if (q != mu) g += Pm(q, q) * (e.gp2 - 0.5 * e.hpp);
    return g;
  }
  if (mu == 0 || nu == 0) return Pm(mu, nu) * (1.5 * e.hsp - 0.5 * e.gsp);
  return Pm(mu, nu) * (1.5 * e.hpp - 0.5 * e.gp2);
}

// Orbital pair (mu, nu), mu <= nu, of each packed index p = nu(nu+1)/2 + mu.
__constant__ int c_pair_mu[10] = {0, 0, 1, 0, 1, 2, 0, 1, 2, 3};
__constant__ int c_pair_nu[10] = {0, 1, 1, 2, 2, 2, 3, 3, 3, 3};


// F = H + G(P) and the electronic energy 1/2 sum P (H + F), pair-centric.
// Phase 1: per atom pair (A < B) the Coulomb vectors J_A = W pv_B and
// J_B = W^T pv_A (pv = packed diagonal-block density with the factor 2 for
// mu != nu) go to jbuf, and the exchange block F_AB = H_AB - 1/2 K_AB with
// K_AB[mu][lam] = sum P_{nu sig} (mu nu|lam sig) is written directly (each
// pair owns its block).  s/p-s/p pairs are handled by a warp each, pairs with
// an s-only atom by a thread each.
// Phase 2: diagonal blocks F_AA = H_AA + G_1c(P_AA) + sum of the partners' J_A.
// Fock build, phase 1a: pairs with at most one s/p atom, pair k0, k0 + kstep, ...
// (one thread each).  Writes the off-diagonal F blocks and the per-pair
// Coulomb vectors; returns this thread's share of sum P (H + F).
__device__ double fock_light_pairs(const MolDev& m, const AtomDev* __restrict__ atoms, const ElemDev* __restrict__ elems,
                             const PairDev* __restrict__ pairs, const double* __restrict__ ints,
                             const int* __restrict__ hh_pairs, double* __restrict__ jbuf,
                             const double* __restrict__ H, const double* __restrict__ P, double* F, int k0, int kstep) {
  const int N = m.nao;
  double e = 0;
  for (int k = k0; k < m.npairs; k += kstep) {
    const int pi = m.pair0 + k;
    const PairDev pr = pairs[pi];
    const AtomDev aA = atoms[pr.a], aB = atoms[pr.b];
    const int nA = elems[aA.slot].nao, nB = elems[aB.slot].nao;
    if (nA == 4 && nB == 4) continue;
    const int oa = aA.ao0, ob = aB.ao0;
    const double* W = ints + pr.int_off;
    double* jb = jbuf + (size_t)pi * 20;
    if (nA == 1 && nB == 1) {
      const double w = W[0];
      jb[0] = w * P[(size_t)ob * N + ob];
      jb[10] = w * P[(size_t)oa * N + oa];
      const double pab = P[(size_t)oa * N + ob];
      const double h = H[(size_t)oa * N + ob];
      const double f = h - 0.5 * pab * w;
      F[(size_t)oa * N + ob] = f;
      F[(size_t)ob * N + oa] = f;
      e += pab * (h + f);
      continue;
    }
    // one s/p atom (X) and one s-only atom (Hs): W is 10 x 1 or 1 x 10
    const bool xfirst = nA == 4;
    const int ox = xfirst ? oa : ob, oh = xfirst ? ob : oa;
    double pvx[10];
#pragma unroll
    for (int p = 0; p < 10; ++p) {
      const int mu = c_pair_mu[p], nu = c_pair_nu[p];
      pvx[p] = (mu == nu ? 1.0 : 2.0) * P[(size_t)(ox + mu) * N + ox + nu];
    }
    const double pvh = P[(size_t)oh * N + oh];
    double jh = 0;
#pragma unroll
    for (int p = 0; p < 10; ++p) {
      const double w = W[p];  // (p on X | s s on Hs) in either storage order
      jh += w * pvx[p];
      jb[(xfirst ? 0 : 10) + p] = w * pvh;
    }
    jb[xfirst ? 10 : 0] = jh;
    // exchange K[mu on X] = sum_nu P[X_nu][Hs] (mu nu | s s)
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) {
      double kx = 0;
#pragma unroll
      for (int nu = 0; nu < 4; ++nu) kx += P[(size_t)(ox + nu) * N + oh] * W[pair_index(mu, nu)];
      const size_t ixh = (size_t)(ox + mu) * N + oh, ihx = (size_t)oh * N + ox + mu;
      const double h = H[ixh];
      const double f = h - 0.5 * kx;
      F[ixh] = f;
      F[ihx] = f;
      e += P[ixh] * (h + f);
    }
  }
  return e;
}

// Fock build, phase 1b: s/p-s/p pairs h0, h0 + hstep, ... of the molecule's
// heavy-pair list, one warp each (ws: this warp's kFockWarpScratch doubles).
__device__ double fock_heavy_pairs(const MolDev& m, const AtomDev* __restrict__ atoms, const ElemDev* __restrict__ elems,
                             const PairDev* __restrict__ pairs, const double* __restrict__ ints,
                             const int* __restrict__ hh_pairs, double* __restrict__ jbuf,
                             const double* __restrict__ H, const double* __restrict__ P, double* F, double* ws, int h0, int hstep) {
  const int N = m.nao;
  const int lane = threadIdx.x & 31;
  double e = 0;
  double* Wsm = ws;
  double* Pab = ws + 100;
  double* pvA = ws + 116;
  double* pvB = ws + 126;
  for (int h = h0; h < m.nhh; h += hstep) {
    const int pi = hh_pairs[m.hh0 + h];
    const PairDev pr = pairs[pi];
    const int oa = atoms[pr.a].ao0, ob = atoms[pr.b].ao0;
    const double* W = ints + pr.int_off;
    for (int q = lane; q < 100; q += 32) Wsm[q] = W[q];
    if (lane < 16) Pab[lane] = P[(size_t)(oa + (lane >> 2)) * N + ob + (lane & 3)];
    if (lane < 10) {
      const int mu = c_pair_mu[lane], nu = c_pair_nu[lane];
      pvA[lane] = (mu == nu ? 1.0 : 2.0) * P[(size_t)(oa + mu) * N + oa + nu];
      pvB[lane] = (mu == nu ? 1.0 : 2.0) * P[(size_t)(ob + mu) * N + ob + nu];
    }
    __syncwarp();
    double* jb = jbuf + (size_t)pi * 20;
    if (lane < 10) {
      double s = 0;
#pragma unroll
      for (int q = 0; q < 10; ++q) s += Wsm[lane * 10 + q] * pvB[q];
      jb[lane] = s;
    } else if (lane < 20) {
      const int q = lane - 10;
      double s = 0;
#pragma unroll
      for (int p = 0; p < 10; ++p) s += Wsm[p * 10 + q] * pvA[p];
      jb[10 + q] = s;
    }
    if (lane < 16) {
      const int mu = lane >> 2, la = lane & 3;
      double kx = 0;
#pragma unroll
      for (int nu = 0; nu < 4; ++nu)
#pragma unroll
        for (int si = 0; si < 4; ++si) kx += Pab[nu * 4 + si] * Wsm[pair_index(mu, nu) * 10 + pair_index(la, si)];
      const size_t iab = (size_t)(oa + mu) * N + ob + la, iba = (size_t)(ob + la) * N + oa + mu;
      const double hv = H[iab];
      const double f = hv - 0.5 * kx;
      F[iab] = f;
      F[iba] = f;
      e += Pab[lane] * (hv + f);
    }
    __syncwarp();
  }
  return e;
}

// Fock build, phase 2 (after every pair of the molecule is done): one-centre
// blocks for entries i0, i0 + istep, ... of (atom, orbital pair).
__device__ double fock_diagonal(const MolDev& m, const AtomDev* __restrict__ atoms, const ElemDev* __restrict__ elems,
                             const PairDev* __restrict__ pairs, const double* __restrict__ ints,
                             const int* __restrict__ hh_pairs, double* __restrict__ jbuf,
                             const double* __restrict__ H, const double* __restrict__ P, double* F, int i0, int istep) {
  const int N = m.nao;
  double e = 0;
  for (int idx = i0; idx < m.nat * 10; idx += istep) {
    const int a = idx / 10, p = idx % 10;
    const AtomDev aA = atoms[m.atom0 + a];
    const ElemDev& eA = elems[aA.slot];
    if (p >= (eA.nao == 1 ? 1 : 10)) continue;
    const int mu = c_pair_mu[p], nu = c_pair_nu[p];
    double g = one_centre_g(eA, mu, nu, P, N, aA.ao0);
    double j0 = 0, j1 = 0;
    int c = 0;
    for (; c + 1 < m.nat; c += 2) {
      const int c0 = c, c1 = c + 1;
      if (c0 != a) j0 += jbuf[(size_t)(a < c0 ? pair_slot(m, a, c0) : pair_slot(m, c0, a)) * 20 + (a < c0 ? p : 10 + p)];
      if (c1 != a) j1 += jbuf[(size_t)(a < c1 ? pair_slot(m, a, c1) : pair_slot(m, c1, a)) * 20 + (a < c1 ? p : 10 + p)];
    }
    if (c < m.nat && c != a) j0 += jbuf[(size_t)(a < c ? pair_slot(m, a, c) : pair_slot(m, c, a)) * 20 + (a < c ? p : 10 + p)];
    g += j0 + j1;
    const size_t i1 = (size_t)(aA.ao0 + mu) * N + aA.ao0 + nu;
    const double h = H[i1];
    const double f = h + g;
    F[i1] = f;
    if (mu != nu) F[(size_t)(aA.ao0 + nu) * N + aA.ao0 + mu] = f;
    e += (mu == nu ? 0.5 : 1.0) * P[i1] * (h + f);
  }
  return e;
}

// The same with a warp per atom: lanes walk the partner atoms (the Coulomb
// vectors of many pairs in flight at once), a warp-private row of 10
// partials per lane in ws (32 * 10 doubles per warp) is summed by lanes 0-9,
// which then add the one-centre terms.  Warp w of nw handles atoms w, w + nw, ...
__device__ double fock_diagonal_warp(const MolDev& m, const AtomDev* __restrict__ atoms,
                                     const ElemDev* __restrict__ elems, const double* __restrict__ jbuf,
                                     const double* __restrict__ H, const double* __restrict__ P, double* F, double* ws,
                                     int warp, int nw) {
  const int N = m.nao, lane = threadIdx.x & 31;
  double e = 0;
  for (int a = warp; a < m.nat; a += nw) {
    const AtomDev aA = atoms[m.atom0 + a];
    const ElemDev& eA = elems[aA.slot];
    const int np = eA.nao == 1 ? 1 : 10;
    double js[10];
#pragma unroll
    for (int q = 0; q < 10; ++q) js[q] = 0.0;
    for (int c = lane; c < m.nat; c += 32) {
      if (c == a) continue;
      const double* jb = jbuf + (size_t)(a < c ? pair_slot(m, a, c) : pair_slot(m, c, a)) * 20 + (a < c ? 0 : 10);
      if (np == 1) {
        js[0] += jb[0];
      } else {
#pragma unroll
        for (int q = 0; q < 10; ++q) js[q] += jb[q];
      }
    }
#pragma unroll
    for (int q = 0; q < 10; ++q) ws[lane * 10 + q] = js[q];
    __syncwarp();
    if (lane < np) {
      double j = 0;
      for (int l = 0; l < 32; ++l) j += ws[l * 10 + lane];
      const int mu = c_pair_mu[lane], nu = c_pair_nu[lane];
      const double g = one_centre_g(eA, mu, nu, P, N, aA.ao0) + j;
      const size_t i1 = (size_t)(aA.ao0 + mu) * N + aA.ao0 + nu;
      const double h = H[i1];
      const double f = h + g;
      F[i1] = f;
      if (mu != nu) F[(size_t)(aA.ao0 + nu) * N + aA.ao0 + mu] = f;
      e += (mu == nu ? 0.5 : 1.0) * P[i1] * (h + f);
    }
    __syncwarp();
  }
  return e;
}

// prof (optional): cycles of the light pairs, the heavy pairs with the
// barrier, the diagonal blocks with the barrier and the energy sum added to
// prof[0..3].
__device__ double build_fock(const MolDev& m, const AtomDev* __restrict__ atoms, const ElemDev* __restrict__ elems,
                             const PairDev* __restrict__ pairs, const double* __restrict__ ints,
                             const int* __restrict__ hh_pairs, double* __restrict__ jbuf,
                             const double* __restrict__ H, const double* __restrict__ P, double* F, double* red,
                             double* wscratch, long long* prof = nullptr) {
  const int tid = threadIdx.x, warp = tid >> 5, nwarps = blockDim.x >> 5;
  long long t = clock64();
  double e = fock_light_pairs(m, atoms, elems, pairs, ints, hh_pairs, jbuf, H, P, F, tid, blockDim.x);
  prof_mark(prof, 0, t);
  e += fock_heavy_pairs(m, atoms, elems, pairs, ints, hh_pairs, jbuf, H, P, F, wscratch + (size_t)warp * kFockWarpScratch,
                        warp, nwarps);
  __syncthreads();
  prof_mark(prof, 1, t);
  // wscratch holds kFockWarpScratch doubles per warp for the heavy pairs; the
  // diagonal phase needs 320 per warp: the phase-scratch union has room for
  // that (a barrier separates the two uses)
  e += fock_diagonal_warp(m, atoms, elems, jbuf, H, P, F, wscratch + (size_t)warp * 320, warp, nwarps);
  __syncthreads();
  prof_mark(prof, 2, t);
  const double s = cta_sum(e, red);
  prof_mark(prof, 3, t);
  return s;
}

__global__ void __launch_bounds__(kScfThreads, 1) k_scf(const MolDev* __restrict__ mols, int nmol,
                                                     const int* __restrict__ order, int* counter,
                                                     const AtomDev* __restrict__ atoms,
                                                     const ElemDev* __restrict__ elems,
                                                     const PairDev* __restrict__ pairs,
                                                     const double* __restrict__ ints,
                                                     const int* __restrict__ hh_pairs, double* jbuf,
                                                     const double* __restrict__ Hall,
                                                     double* Pall, double* Fall, double* Call, double* W1all,
                                                     double* W2all, double* epsall, double* diisall, double* rotbuf,
                                                     MolResult* res, ScfParams sp, int packed_in_smem) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ScfShared& sh = *reinterpret_cast<ScfShared*>(smem_raw);
  double* smemA = reinterpret_cast<double*>(smem_raw + ((sizeof(ScfShared) + 15) / 16) * 16);
  const int tid = threadIdx.x;
  for (;;) {
    if (tid == 0) {
      int k = atomicAdd(counter, 1);
      sh.mol = k < nmol ? order[k] : -1;
    }
    __syncthreads();
    const int mi = sh.mol;
    __syncthreads();
    if (mi < 0) return;
    const MolDev m = mols[mi];
    const int N = m.nao, no = m.nocc;
    const size_t NN = (size_t)N * N;
    const double* H = Hall + m.mat_off;
    // The five N x N buffers of the molecule trade roles during the SCF
    // instead of being copied into each other: role r (F, C, W1, W2, P) lives
    // in buffer (roles >> 3r) & 7 of Fall, Call, W1all, W2all, Pall.
    int roles = 0 | (1 << 3) | (2 << 6) | (3 << 9) | (4 << 12);
    auto buf = [&](int r) -> double* {
      const int b = (roles >> (3 * r)) & 7;
      double* base = b == 0 ? Fall : b == 1 ? Call : b == 2 ? W1all : b == 3 ? W2all : Pall;
      return base + m.mat_off;
    };
    auto trade = [&](int r1, int r2) {
      const int b1 = (roles >> (3 * r1)) & 7, b2 = (roles >> (3 * r2)) & 7;
      roles &= ~((7 << (3 * r1)) | (7 << (3 * r2)));
      roles |= (b2 << (3 * r1)) | (b1 << (3 * r2));
    };
    constexpr int kRF = 0, kRC = 1, kRW1 = 2, kRW2 = 3, kRP = 4;
    double* P = Pall + m.mat_off;
    double* F = Fall + m.mat_off;
    double* Ct = Call + m.mat_off;
    double* W1 = W1all + m.mat_off;
    double* W2 = W2all + m.mat_off;
    double* eps = epsall + m.ao_base;
    double* histF = diisall + m.diis_off;
    double* histE = histF + (size_t)kDiisMax * NN;
    // packed matrix of the Jacobi solver: shared memory when it fits, else F
    double* Apk = packed_in_smem ? smemA : nullptr;
    const size_t packed_bytes = sizeof(double) * (size_t)N * (N + 1) / 2;
    // recorded Jacobi rotations: this CTA's slice of the rotation buffer
    double* rot = rotbuf + (size_t)blockIdx.x * (kRotBudgetBytes / sizeof(double));
    const int cap_rounds = (int)((kRotBudgetBytes / sizeof(double)) / (2 * ((N + 1) / 2)));
    const int msize = scf_diis_size(sp, N);
    const int cold_sweeps = sp.cold_sweeps > 0 ? sp.cold_sweeps : 3;
    int nhist = 0, head = 0;
    bool have_orbitals = false;
    double drift = 0;
    double Eold = 0;
    const int mode = scf_eig_mode(sp, N);
    int it = 0, converged = 0, status = kDevOk;
    double last_dE = 0, last_rms = 0;

    long long cyc[5] = {0, 0, 0, 0, 0};
#ifdef SGB_PROFILE_GROUP
    // profiling build: the result's cycle counters report four stages of one
    // phase (SGB_PROFILE_GROUP 1: the eigensolver, 2: DIIS, 3: the
    // occupied-virtual rotation, 4: the Fock build) and everything else
    long long gprof[4] = {0, 0, 0, 0};
    long long* eprof = SGB_PROFILE_GROUP == 1 ? gprof : nullptr;
    long long* dprof = SGB_PROFILE_GROUP == 2 ? gprof : nullptr;
    long long* oprof = SGB_PROFILE_GROUP == 3 ? gprof : nullptr;
    long long* fprof = SGB_PROFILE_GROUP == 4 ? gprof : nullptr;
#else
    long long* eprof = nullptr;
    long long* dprof = nullptr;
    long long* oprof = nullptr;
    long long* fprof = nullptr;
#endif
    int nfull = 0, nsweeps = 0;
    for (it = 1; it <= sp.max_iter; ++it) {
      F = buf(kRF);
      Ct = buf(kRC);
      W1 = buf(kRW1);
      W2 = buf(kRW2);
      P = buf(kRP);
      long long t0 = clock64();
      const double E = build_fock(m, atoms, elems, pairs, ints, hh_pairs, jbuf, H, P, F, sh.red, sh.fockw, fprof);
      __syncthreads();
      long long t1 = clock64();
      cyc[0] += t1 - t0;
      const double* Fx = diis_step(N, F, P, W1, W2, histF, histE, msize, nhist, head, sh, dprof);
      // Fx lives in F or W2: when in W2, F and W2 trade buffers
      if (Fx != F) {
        trade(kRF, kRW2);
        F = buf(kRF);
        W2 = buf(kRW2);
      }
      long long t2 = clock64();
      cyc[1] += t2 - t1;
      int need_full = !have_orbitals;
      if (mode != kEigExact && have_orbitals) {
        int sw = 0;
        need_full = ov_rotation(N, no, F, Ct, W1, W2, eps, drift, sh, oprof, &sw);
        if (sw & 1) trade(kRC, kRF);
        if (sw & 2) trade(kRC, kRW2);
        F = buf(kRF);
        Ct = buf(kRC);
        W2 = buf(kRW2);
      }
      if (mode == kEigExact || (need_full && mode == kEigHybrid)) {
        // exact: every iteration the lowest eigenvalues and the occupied
        // eigenvectors of the extrapolated F; hybrid: every eigenpair at the
        // start (or when the occupied/virtual ordering breaks), the rotations
        // take over from there.  Jacobi only for clustered spectra.
        const bool all = mode != kEigExact;
        need_full = eigh_tridiag(N, F, all ? N : (no < N ? no + 1 : N), all ? N : no, Ct, N, eps, sh.gemm,
                                 eig_workspace_doubles(sh, smem_raw), W2, W1, Ct, F, sh.red, &sh.flag, eprof);
        if (!all || need_full) {
          // a fallback diagonalises from scratch (the solver used Ct as scratch)
          have_orbitals = false;
        } else {
          have_orbitals = true;
          drift = 0;
          ++nfull;
        }
      }
      long long t3 = clock64();
      cyc[2] += t3 - t2;
      if (need_full) {
        // the first (cold) diagonalisation of the rotation mode only has to
        // separate occupied from virtual orbitals; a fallback of the
        // tridiagonal mode converges fully
        const bool full_acc = have_orbitals || mode == kEigExact;
        const int sw = full_diagonalise(N, F, Ct, W1, W2, eps, Apk ? Apk : F, Apk ? packed_bytes : 0, have_orbitals,
                                        rot, cap_rounds, full_acc ? sp.jacobi_max_sweeps : cold_sweeps,
                                        full_acc ? 1e-10 : 1e-3, sh);
        if (sw < 0 && full_acc) status = kDevJacobiNotConverged;
        nsweeps += sw < 0 ? (full_acc ? sp.jacobi_max_sweeps : cold_sweeps) : sw;
        ++nfull;
        have_orbitals = true;
        drift = 0;
      }
      long long t4 = clock64();
      cyc[3] += t4 - t3;
      // new density P = 2 C_occ C_occ^T = 2 Ct_o^T Ct_o into W1, rms change
      // against P; then P and W1 trade buffers
      // (the squared change against P is summed in the product's epilogue)
      double d2 = 0;
      cta_gemm<true>(N, N, no, 2.0, Ct, N, true, Ct, N, false, 0.0, W1, N, sh.gemm, true, P, &d2);
      d2 = cta_sum(d2, sh.red);
      trade(kRP, kRW1);
      const double rms = sqrt(d2 / (double)NN);
      last_rms = rms;
      last_dE = it > 1 ? fabs(E - Eold) : 0.0;
      const bool dE_ok = it > 1 && fabs(E - Eold) < sp.scc;
      Eold = E;
      cyc[4] += clock64() - t4;
      if (!isfinite(E) || !isfinite(rms)) { status = kDevNonFinite; break; }
      if (dE_ok && rms < sp.rmsd) { converged = 1; break; }
      __syncthreads();
    }
    if (it > sp.max_iter) it = sp.max_iter;
    __syncthreads();
    // Back to the home buffers: the density to Pall's (the gradient kernels
    // read it), the orbitals to Call's (the canonical-orbital kernel reads
    // them); the final Fock matrix is built in Fall's.  W1's buffer holds
    // nothing live and takes the orbitals when they sit in the density's.
    {
      double* const bP = Pall + m.mat_off;
      double* const bC = Call + m.mat_off;
      P = buf(kRP);
      Ct = buf(kRC);
      if (P != bP) {
        if (Ct == bP) {
          W1 = buf(kRW1);
          for (size_t k = tid; k < NN; k += blockDim.x) W1[k] = Ct[k];
          __syncthreads();
          Ct = W1;
        }
        for (size_t k = tid; k < NN; k += blockDim.x) bP[k] = P[k];
        __syncthreads();
      }
      if (Ct != bC) {
        for (size_t k = tid; k < NN; k += blockDim.x) bC[k] = Ct[k];
        __syncthreads();
      }
      P = bP;
      F = Fall + m.mat_off;
    }
    const double Efin = build_fock(m, atoms, elems, pairs, ints, hh_pairs, jbuf, H, P, F, sh.red, sh.fockw);
    if (tid == 0) {
      MolResult& r = res[mi];
      r.e_el = Efin;
      r.energy = Efin + r.e_rep;
      r.iterations = it;
      r.converged = converged;
      r.status = status;
      r.last_dE = last_dE;
      r.last_rmsd = last_rms;
      r.full_diag = nfull;
      r.jacobi_sweeps = nsweeps;
#ifdef SGB_PROFILE_GROUP
      long long tot = 0;
      for (int k = 0; k < 5; ++k) tot += cyc[k];
      for (int k = 0; k < 4; ++k) {
        r.cycles[k] = gprof[k];
        tot -= gprof[k];
      }
      r.cycles[4] = tot;
#else
      for (int k = 0; k < 5; ++k) r.cycles[k] = cyc[k];
#endif
    }
    __syncthreads();
  }
}

namespace {
// The persistent SCF kernels run one CTA per SM, so they take all the shared
// memory a block may opt in to: the Jacobi solver's packed matrix sits there
// when it fits, and the tridiagonal solver tiles molecules of up to 192 AOs.
size_t scf_smem_bytes(int max_nao, int* packed_in_smem) {
  const size_t base = ((sizeof(ScfShared) + 15) / 16) * 16;
  const size_t pk = sizeof(double) * (size_t)max_nao * (max_nao + 1) / 2;
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  *packed_in_smem = base + pk <= (size_t)optin ? 1 : 0;
  return (size_t)optin > base ? (size_t)optin : base;
}
}  // namespace

size_t scf_rotation_bytes_per_cta() { return kRotBudgetBytes; }

int scf_max_grid(int max_nao) {
  int dev = 0, sms = 0, per_sm = 0, in_smem = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const size_t bytes = scf_smem_bytes(max_nao, &in_smem);
  cudaFuncSetAttribute(k_scf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_scf, kScfThreads, bytes);
  if (per_sm < 1) per_sm = 1;
  return sms * per_sm;
}

void launch_scf(const DeviceBatch& b, const ScfParams& sp, int grid, cudaStream_t s) {
  if (b.nmol == 0) return;
  int in_smem = 0;
  const size_t bytes = scf_smem_bytes(b.max_nao, &in_smem);
  cudaFuncSetAttribute(k_scf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  cudaMemsetAsync(b.counter, 0, sizeof(int), s);
  if (grid > b.nmol) grid = b.nmol;
  k_scf<<<grid, kScfThreads, bytes, s>>>(b.mols, b.nmol, b.order, b.counter, b.atoms, b.elems, b.pairs, b.ints,
                                         b.hh_pairs, b.jbuf, b.H, b.P, b.F, b.C, b.W1, b.W2, b.eps, b.diis,
                                         b.rotbuf, b.res, sp, in_smem);
}

// ---------------------------------------------------------------------------
// Unrestricted (UHF) SCF
// ---------------------------------------------------------------------------
// With P_T = P_a + P_b and the spin density P_s = P_a - P_b, the unrestricted
// Fock matrices (TwoElectronMatrix.cpp:98-103, 142-161: G_s = sum P_T (mn|ls)
// - P_s' (ml|ns) for spin s') are the restricted build on the total density
// plus a spin-exchange term,
//   F_a = F_R(P_T) - 1/2 K(P_s),   F_b = F_R(P_T) + 1/2 K(P_s),
//   K(P)_mn = sum_ls P_ls (ml|ns),
// and the electronic energy 1/2 sum [P_T H + P_a F_a + P_b F_b]
// (NDDOElectronicEnergyCalculator.cpp:68-90) is E_R(P_T) - 1/4 sum P_s K(P_s).
// spin_exchange applies the term: F holds F_R on entry and F_a on return, Fb
// receives F_b.  Two-centre blocks (exchange only couples the atoms of a pair)
// take a thread per pair; one-centre blocks a thread per (atom, orbital pair),
// with K_ss = S_ss g_ss + sum_p S_pp h_sp, K_pp = S_ss h_sp + S_pp g_pp +
// sum_q!=p S_qq h_pp, K_sp = S_sp (g_sp + h_sp), K_pq = S_pq (g_p2 + h_pp).
// Returns sum P_s K(P_s) over the CTA.
__device__ double spin_exchange(const MolDev& m, const AtomDev* __restrict__ atoms, const ElemDev* __restrict__ elems,
                                const PairDev* __restrict__ pairs, const double* __restrict__ ints,
                                const double* __restrict__ Pa, const double* __restrict__ Pb, double* F, double* Fb,
                                double* red) {
  const int N = m.nao, tid = threadIdx.x;
  double e = 0;
  for (int k = tid; k < m.npairs; k += blockDim.x) {
    const PairDev pr = pairs[m.pair0 + k];
    const AtomDev aA = atoms[pr.a], aB = atoms[pr.b];
    const int nA = elems[aA.slot].nao, nB = elems[aB.slot].nao;
    const int oa = aA.ao0, ob = aB.ao0, dB = nB == 4 ? 10 : 1;
    const double* W = ints + pr.int_off;
    double S[4][4];
    for (int i = 0; i < nA; ++i)
      for (int j = 0; j < nB; ++j) {
        const size_t ij = (size_t)(oa + i) * N + ob + j;
        S[i][j] = Pa[ij] - Pb[ij];
      }
    for (int mu = 0; mu < nA; ++mu)
      for (int la = 0; la < nB; ++la) {
        double kx = 0;
        for (int nu = 0; nu < nA; ++nu)
          for (int si = 0; si < nB; ++si)
            kx += S[nu][si] * W[(nA == 4 ? pair_index(mu, nu) : 0) * dB + (nB == 4 ? pair_index(la, si) : 0)];
        const size_t iab = (size_t)(oa + mu) * N + ob + la, iba = (size_t)(ob + la) * N + oa + mu;
        const double fr = F[iab];
        F[iab] = F[iba] = fr - 0.5 * kx;
        Fb[iab] = Fb[iba] = fr + 0.5 * kx;
        e += 2.0 * S[mu][la] * kx;
      }
  }
  for (int idx = tid; idx < m.nat * 10; idx += blockDim.x) {
    const int a = idx / 10, p = idx % 10;
    const AtomDev aA = atoms[m.atom0 + a];
    const ElemDev& eA = elems[aA.slot];
    if (p >= (eA.nao == 1 ? 1 : 10)) continue;
    const int mu = c_pair_mu[p], nu = c_pair_nu[p], o = aA.ao0;
    auto Sm = [&](int i, int j) {
      const size_t ij = (size_t)(o + i) * N + o + j;
      return Pa[ij] - Pb[ij];
    };
    double kx;
    if (eA.nao == 1) {
      kx = Sm(0, 0) * eA.gss;
    } else if (mu == nu) {
      if (mu == 0) {
        kx = Sm(0, 0) * eA.gss + (Sm(1, 1) + Sm(2, 2) + Sm(3, 3)) * eA.hsp;
      } else {
        kx = Sm(0, 0) * eA.hsp + Sm(mu, mu) * eA.gpp;
        for (int q = 1; q < 4; ++q)
          if (q != mu) kx += Sm(q, q) * eA.hpp;
      }
    } else {
      kx = Sm(mu, nu) * (mu == 0 ? eA.gsp + eA.hsp : eA.gp2 + eA.hpp);
    }
    const size_t i1 = (size_t)(o + mu) * N + o + nu, i2 = (size_t)(o + nu) * N + o + mu;
    const double fr = F[i1];
    F[i1] = F[i2] = fr - 0.5 * kx;
    Fb[i1] = Fb[i2] = fr + 0.5 * kx;
    e += (mu == nu ? 1.0 : 2.0) * Sm(mu, nu) * kx;
  }
  __syncthreads();
  return cta_sum(e, red);
}

// The persistent kernel of k_scf for unrestricted molecules (MolDev.nocc
// alpha and MolDev.nocc_b beta electrons): start P_a = P_b = P / 2 from the
// restricted guess or a given total density (or from given spin densities,
// spin_given, with P = P_a + P_b), then per iteration the Fock
// pair, one DIIS over both spins, new orbitals and densities per spin;
// convergence on |dE| and the larger rms change of the two spin densities.
__global__ void __launch_bounds__(kScfThreads, 1) k_uhf_scf(
    const MolDev* __restrict__ mols, int nmol, const int* __restrict__ order, int* counter,
    const AtomDev* __restrict__ atoms, const ElemDev* __restrict__ elems, const PairDev* __restrict__ pairs,
    const double* __restrict__ ints, const int* __restrict__ hh_pairs, double* jbuf, const double* __restrict__ Hall,
    double* Pall, double* Fall, double* Call, double* W1all, double* W2all, double* epsall, double* diisall,
    double* Paall, double* Pball, double* Fball, double* Cball, double* epsball, double* diisball, double* rotbuf,
    MolResult* res, ScfParams sp, int packed_in_smem, int spin_given) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ScfShared& sh = *reinterpret_cast<ScfShared*>(smem_raw);
  double* smemA = reinterpret_cast<double*>(smem_raw + ((sizeof(ScfShared) + 15) / 16) * 16);
  const int tid = threadIdx.x;
  for (;;) {
    if (tid == 0) {
      int k = atomicAdd(counter, 1);
      sh.mol = k < nmol ? order[k] : -1;
    }
    __syncthreads();
    const int mi = sh.mol;
    __syncthreads();
    if (mi < 0) return;
    const MolDev m = mols[mi];
    const int N = m.nao, na = m.nocc, nb = m.nocc_b;
    const size_t NN = (size_t)N * N;
    const double* H = Hall + m.mat_off;
    double* P = Pall + m.mat_off;
    double* Pa = Paall + m.mat_off;
    double* Pb = Pball + m.mat_off;
    double* Fa = Fall + m.mat_off;
    double* Fb = Fball + m.mat_off;
    double* Ca = Call + m.mat_off;
    double* Cb = Cball + m.mat_off;
    double* W1 = W1all + m.mat_off;
    double* W2 = W2all + m.mat_off;
    double* epsa = epsall + m.ao_base;
    double* epsb = epsball + m.ao_base;
    double* histFa = diisall + m.diis_off;
    double* histEa = histFa + (size_t)kDiisMax * NN;
    double* histFb = diisball + m.diis_off;
    double* histEb = histFb + (size_t)kDiisMax * NN;
    double* Apk = packed_in_smem ? smemA : nullptr;
    const size_t packed_bytes = sizeof(double) * (size_t)N * (N + 1) / 2;
    double* rot = rotbuf + (size_t)blockIdx.x * (kRotBudgetBytes / sizeof(double));
    const int cap_rounds = (int)((kRotBudgetBytes / sizeof(double)) / (2 * ((N + 1) / 2)));
    const int msize = scf_diis_size(sp, N);
    const int cold_sweeps = sp.cold_sweeps > 0 ? sp.cold_sweeps : 3;
    if (!spin_given)
      for (size_t k = tid; k < NN; k += blockDim.x) Pa[k] = Pb[k] = 0.5 * P[k];
    __syncthreads();
    int nhist = 0, head = 0;
    bool have_a = false, have_b = false;
    double drift_a = 0, drift_b = 0, Eold = 0, last_dE = 0, last_rms = 0;
    int it = 0, converged = 0, status = kDevOk, nfull = 0, nsweeps = 0;
    for (it = 1; it <= sp.max_iter; ++it) {
      const double ER = build_fock(m, atoms, elems, pairs, ints, hh_pairs, jbuf, H, P, Fa, sh.red, sh.fockw);
      __syncthreads();
      const double E = ER - 0.25 * spin_exchange(m, atoms, elems, pairs, ints, Pa, Pb, Fa, Fb, sh.red);
      diis_step_uhf(N, Fa, Pa, Fb, Pb, W1, histFa, histEa, histFb, histEb, msize, nhist, head, sh);
      const bool warm_a = have_a, warm_b = have_b;
      const size_t wsd = eig_workspace_doubles(sh, smem_raw);
      int sw = uhf_orbitals(N, na, Fa, Ca, W1, W2, epsa, Apk, packed_bytes, have_a, drift_a, rot, cap_rounds, sp,
                            cold_sweeps, nfull, sh, sh.gemm, wsd);
      if (sw < 0 && warm_a) status = kDevJacobiNotConverged;
      nsweeps += sw < 0 ? -sw : sw;
      sw = uhf_orbitals(N, nb, Fb, Cb, W1, W2, epsb, Apk, packed_bytes, have_b, drift_b, rot, cap_rounds, sp,
                        cold_sweeps, nfull, sh, sh.gemm, wsd);
      if (sw < 0 && warm_b) status = kDevJacobiNotConverged;
      nsweeps += sw < 0 ? -sw : sw;
      const double da = uhf_density(N, na, Ca, Pa, W1, sh);
      const double db = uhf_density(N, nb, Cb, Pb, W1, sh);
      for (size_t k = tid; k < NN; k += blockDim.x) P[k] = Pa[k] + Pb[k];
      __syncthreads();
      const double rms = sqrt(fmax(da, db) / (double)NN);
      last_rms = rms;
      last_dE = it > 1 ? fabs(E - Eold) : 0.0;
      const bool dE_ok = it > 1 && fabs(E - Eold) < sp.scc;
      Eold = E;
      if (!isfinite(E) || !isfinite(rms)) { status = kDevNonFinite; break; }
      if (dE_ok && rms < sp.rmsd) { converged = 1; break; }
    }
    if (it > sp.max_iter) it = sp.max_iter;
    __syncthreads();
    const double ER = build_fock(m, atoms, elems, pairs, ints, hh_pairs, jbuf, H, P, Fa, sh.red, sh.fockw);
    __syncthreads();
    const double Efin = ER - 0.25 * spin_exchange(m, atoms, elems, pairs, ints, Pa, Pb, Fa, Fb, sh.red);
    if (tid == 0) {
      MolResult& r = res[mi];
      r.e_el = Efin;
      r.energy = Efin + r.e_rep;
      r.iterations = it;
      r.converged = converged;
      r.status = status;
      r.last_dE = last_dE;
      r.last_rmsd = last_rms;
      r.full_diag = nfull;
      r.jacobi_sweeps = nsweeps;
      for (int k = 0; k < 5; ++k) r.cycles[k] = 0;
    }
    __syncthreads();
  }
}

// Canonical orbitals after convergence (ScfParams::canonical): a warm
// diagonalisation of the final Fock matrix of each spin from the current
// orbitals, so the orbital energies are its eigenvalues.  The SCF kernels
// leave the final Fock matrices in F (and Fb).
__global__ void __launch_bounds__(kScfThreads, 1) k_canonical(const MolDev* __restrict__ mols, int nmol,
                                                            const int* __restrict__ order, int* counter, double* Fall,
                                                            double* Call, double* W1all, double* W2all,
                                                            double* epsall, double* Fball, double* Cball,
                                                            double* epsball, double* rotbuf, ScfParams sp,
                                                            int packed_in_smem) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ScfShared& sh = *reinterpret_cast<ScfShared*>(smem_raw);
  double* smemA = reinterpret_cast<double*>(smem_raw + ((sizeof(ScfShared) + 15) / 16) * 16);
  for (;;) {
    if (threadIdx.x == 0) {
      const int k = atomicAdd(counter, 1);
      sh.mol = k < nmol ? order[k] : -1;
    }
    __syncthreads();
    const int mi = sh.mol;
    __syncthreads();
    if (mi < 0) return;
    const MolDev m = mols[mi];
    const int N = m.nao;
    double* Apk = packed_in_smem ? smemA : nullptr;
    const size_t packed_bytes = sizeof(double) * (size_t)N * (N + 1) / 2;
    double* rot = rotbuf + (size_t)blockIdx.x * (kRotBudgetBytes / sizeof(double));
    const int cap_rounds = (int)((kRotBudgetBytes / sizeof(double)) / (2 * ((N + 1) / 2)));
    for (int spin = 0; spin < (Fball ? 2 : 1); ++spin) {
      double* F = (spin ? Fball : Fall) + m.mat_off;
      double* Ct = (spin ? Cball : Call) + m.mat_off;
      double* eps = (spin ? epsball : epsall) + m.ao_base;
      // all eigenpairs of the final Fock matrix by the tridiagonal solver;
      // clustered spectra by a Jacobi diagonalisation from scratch
      const int st = eigh_tridiag(N, F, N, N, Ct, N, eps, sh.gemm, eig_workspace_doubles(sh, smem_raw),
                                  W2all + m.mat_off, W1all + m.mat_off, Ct, F, sh.red, &sh.flag);
      if (st != 0)
        full_diagonalise(N, F, Ct, W1all + m.mat_off, W2all + m.mat_off, eps, Apk ? Apk : F, Apk ? packed_bytes : 0,
                         false, rot, cap_rounds, sp.jacobi_max_sweeps, 1e-10, sh);
    }
    __syncthreads();
  }
}

void launch_canonical(const DeviceBatch& b, const ScfParams& sp, int grid, cudaStream_t s) {
  if (b.nmol == 0) return;
  int in_smem = 0;
  const size_t bytes = scf_smem_bytes(b.max_nao, &in_smem);
  cudaFuncSetAttribute(k_canonical, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  cudaMemsetAsync(b.counter, 0, sizeof(int), s);
  if (grid > b.nmol) grid = b.nmol;
  k_canonical<<<grid, kScfThreads, bytes, s>>>(b.mols, b.nmol, b.order, b.counter, b.F, b.C, b.W1, b.W2, b.eps,
                                               b.uhf ? b.Fb : nullptr, b.Cb, b.epsb, b.rotbuf, sp, in_smem);
}

void launch_uhf_scf(const DeviceBatch& b, const ScfParams& sp, int grid, cudaStream_t s) {
  if (b.nmol == 0) return;
  int in_smem = 0;
  const size_t bytes = scf_smem_bytes(b.max_nao, &in_smem);
  cudaFuncSetAttribute(k_uhf_scf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  cudaMemsetAsync(b.counter, 0, sizeof(int), s);
  if (grid > b.nmol) grid = b.nmol;
  k_uhf_scf<<<grid, kScfThreads, bytes, s>>>(b.mols, b.nmol, b.order, b.counter, b.atoms, b.elems, b.pairs, b.ints,
                                             b.hh_pairs, b.jbuf, b.H, b.P, b.F, b.C, b.W1, b.W2, b.eps, b.diis, b.Pa,
                                             b.Pb, b.Fb, b.Cb, b.epsb, b.diisb, b.rotbuf, b.res, sp, in_smem,
                                             b.spin_given);
}

}  // namespace sgb

// ---------------------------------------------------------------------------
// Whole-GPU Fock build of one large molecule (the large-molecule SCF path):
// the pair phases over the full grid (threads for pairs with hydrogen, warps
// for s/p pairs), then the one-centre phase in a second launch; sum P (H + F)
// is accumulated into *energy.
// ---------------------------------------------------------------------------
namespace sgb {
namespace {

__device__ void block_add(double v, double* red, double* out) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) red[w] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += red[i];
    atomicAdd(out, s);
  }
}

__global__ void __launch_bounds__(256) k_fock_pairs_grid(const MolDev* __restrict__ mols, const AtomDev* __restrict__ atoms,
                                                         const ElemDev* __restrict__ elems,
                                                         const PairDev* __restrict__ pairs,
                                                         const double* __restrict__ ints, const int* __restrict__ hh,
                                                         double* jbuf, const double* __restrict__ H,
                                                         const double* __restrict__ P, double* F, double* energy) {
  __shared__ double red[32];
  __shared__ double ws[8 * kFockWarpScratch];
  const MolDev m = mols[0];
  const int gtid = blockIdx.x * blockDim.x + threadIdx.x, gthreads = gridDim.x * blockDim.x;
  const int gwarp = gtid >> 5, gwarps = gthreads >> 5;
  double e = fock_light_pairs(m, atoms, elems, pairs, ints, hh, jbuf, H, P, F, gtid, gthreads);
  e += fock_heavy_pairs(m, atoms, elems, pairs, ints, hh, jbuf, H, P, F, ws + (threadIdx.x >> 5) * kFockWarpScratch,
                        gwarp, gwarps);
  block_add(e, red, energy);
}

__global__ void __launch_bounds__(256) k_fock_diag_grid(const MolDev* __restrict__ mols, const AtomDev* __restrict__ atoms,
                                                        const ElemDev* __restrict__ elems,
                                                        const PairDev* __restrict__ pairs,
                                                        const double* __restrict__ ints, const int* __restrict__ hh,
                                                        double* jbuf, const double* __restrict__ H,
                                                        const double* __restrict__ P, double* F, double* energy) {
  __shared__ double red[32];
  const MolDev m = mols[0];
  const int gtid = blockIdx.x * blockDim.x + threadIdx.x, gthreads = gridDim.x * blockDim.x;
  const double e = fock_diagonal(m, atoms, elems, pairs, ints, hh, jbuf, H, P, F, gtid, gthreads);
  block_add(e, red, energy);
}

}  // namespace

void launch_fock_grid(const DeviceBatch& b, const double* P, double* F, double* energy, cudaStream_t s) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaMemsetAsync(energy, 0, sizeof(double), s);
  k_fock_pairs_grid<<<sms * 8, 256, 0, s>>>(b.mols, b.atoms, b.elems, b.pairs, b.ints, b.hh_pairs, b.jbuf, b.H, P, F,
                                            energy);
  k_fock_diag_grid<<<sms * 8, 256, 0, s>>>(b.mols, b.atoms, b.elems, b.pairs, b.ints, b.hh_pairs, b.jbuf, b.H, P, F,
                                           energy);
}

}  // namespace sgb
