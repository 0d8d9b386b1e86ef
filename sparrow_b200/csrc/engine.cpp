#include "engine.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>

#include "nddo_math.cuh"
#include "params.h"
#include "dftb_params.h"

namespace sgb {

void build_local_term_table(LocalTermTable& tab);

std::string cuda_message(cudaError_t e) { return std::string("CUDA error: ") + cudaGetErrorString(e); }

namespace {

// The local term table lives in __constant__ memory of each device; upload it
// once per device.
std::mutex g_terms_mu;
std::map<int, bool> g_terms_uploaded;

int ensure_terms(cudaStream_t s, std::string& err) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    err = cuda_message(e);
    return kErrCuda;
  }
  std::lock_guard<std::mutex> lk(g_terms_mu);
  if (g_terms_uploaded[dev]) return kOk;
  static LocalTermTable tab;
  build_local_term_table(tab);
  upload_local_terms(tab, s);
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    err = cuda_message(e);
    return kErrCuda;
  }
  g_terms_uploaded[dev] = true;
  return kOk;
}

size_t align_up(size_t x, size_t a = 256) { return (x + a - 1) / a * a; }

struct CachedBlock {
  int device;
  void* ptr;
  size_t bytes;
  bool pinned;
};
std::mutex g_pool_mu;
std::vector<CachedBlock> g_pool;

// Take the smallest cached block of the kind that fits, or nullptr.
void* pool_take(bool pinned, size_t bytes, size_t* got) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_pool_mu);
  int best = -1;
  for (size_t i = 0; i < g_pool.size(); ++i) {
    const auto& b = g_pool[i];
    if (b.pinned != pinned || (!pinned && b.device != dev) || b.bytes < bytes) continue;
    if (best < 0 || b.bytes < g_pool[best].bytes) best = (int)i;
  }
  if (best < 0) return nullptr;
  void* p = g_pool[best].ptr;
  *got = g_pool[best].bytes;
  g_pool.erase(g_pool.begin() + best);
  return p;
}

void pool_give(bool pinned, void* ptr, size_t bytes) {
  if (!ptr) return;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_pool_mu);
  g_pool.push_back({dev, ptr, bytes, pinned});
}

}  // namespace

void release_cached_memory() {
  std::lock_guard<std::mutex> lk(g_pool_mu);
  for (auto& b : g_pool) {
    if (b.pinned) cudaFreeHost(b.ptr);
    else cudaFree(b.ptr);
  }
  g_pool.clear();
}

namespace {

// cudaMalloc that, when the device is full, frees the process-wide cache of
// idle arenas and tries once more.
cudaError_t device_alloc(void** p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    release_cached_memory();
    e = cudaMalloc(p, bytes);
  }
  return e;
}

}  // namespace

Batch::Batch(Method m) : method_(m) {}

Batch::~Batch() {
  if (stream_) cudaStreamSynchronize(stream_);
  pool_give(false, arena_, arena_bytes_);
  pool_give(true, pinned_, pinned_bytes_);
  if (large_scratch_) cudaFree(large_scratch_);
  if (td_scratch_) cudaFree(td_scratch_);
  for (auto& e : stage_ev_)
    if (e) cudaEventDestroy(e);
  for (auto& e : user_ev_)
    if (e) cudaEventDestroy(e);
  if (stream_) cudaStreamDestroy(stream_);
}

int Batch::ensure_arena(size_t bytes, std::string& err) {
  if (!stream_) {
    cudaError_t e = cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      err = cuda_message(e);
      return kErrCuda;
    }
  }
  if (bytes <= arena_bytes_) return kOk;
  if (arena_) {
    cudaStreamSynchronize(stream_);
    pool_give(false, arena_, arena_bytes_);
    arena_ = nullptr;
    arena_bytes_ = 0;
  }
  size_t got = 0;
  if (void* p = pool_take(false, bytes, &got)) {
    arena_ = p;
    arena_bytes_ = got;
    return kOk;
  }
  cudaError_t e = device_alloc(&arena_, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    err = "device allocation of " + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? kErrOutOfMemory : kErrCuda;
  }
  arena_bytes_ = bytes;
  return kOk;
}

int Batch::setup(const std::vector<MoleculeInput>& in, std::string& err, bool check_pairs) {
  mols_.clear();
  atoms_.clear();
  npairs_ = 0;
  nhh_ = 0;
  elems_.clear();
  ao_atom_.clear();
  order_.clear();
  density_given_ = false;
  spin_given_ = false;
  stages_recorded_ = false;
  td_roots_ = 0;
  if (in.empty()) {
    err = "empty batch";
    return kErrEmptyStructure;
  }
  nddo_set_.reset();
  if (!is_dftb(method_) && !param_source_.empty()) {
    nddo_set_ = nddo_parameter_set(method_, param_source_, err);
    if (!nddo_set_) return kErrParameters;
  }
  if (is_dftb(method_) && !dftb_parameter_set(param_source_.empty() ? dftb_default_set(method_) : param_source_, err))
    return kErrParameters;
  // element slots
  int slot_of[128];
  for (int& v : slot_of) v = -1;
  for (const auto& m : in) {
    if (m.Z.empty()) {
      err = "molecule without atoms";
      return kErrEmptyStructure;
    }
    if (m.xyz.size() != 3 * m.Z.size()) {
      err = "positions must have 3 entries per atom";
      return kErrInvalidArgument;
    }
    for (int z : m.Z) {
      if (z < 0 || z >= 128) {
        err = "invalid atomic number " + std::to_string(z);
        return kErrUnsupportedElement;
      }
      if (slot_of[z] >= 0) continue;
      ElemDev e;
      std::string why;
      if (is_dftb(method_)) {
        // DFTB: orbitals and core charge from the parameter set (records built below)
        const char* set = param_source_.empty() ? dftb_default_set(method_) : param_source_.c_str();
        e = ElemDev();
        e.Z = z;
        e.nao = dftb_n_aos(set, z);
        e.core = dftb_core_charge(set, z);
        if (e.nao == 0 || e.core < 0) {
          err = std::string("no ") + set + " s/p parameters for element Z=" + std::to_string(z);
          return kErrUnsupportedElement;
        }
      } else if (!make_elem(method_, z, e, why, nddo_set_.get())) {
        err = why;
        return kErrUnsupportedElement;
      }
      if ((int)elems_.size() >= kMaxElementSlots) {
        err = "more than 16 distinct elements in one batch";
        return kErrInvalidArgument;
      }
      slot_of[z] = (int)elems_.size();
      elems_.push_back(e);
    }
  }
  diat_.assign(kMaxElementSlots * kMaxElementSlots, DiatomicDev());
  DftbPrepared dftb;
  if (is_dftb(method_)) {
    std::vector<int> zs;
    for (const auto& e : elems_) zs.push_back(e.Z);
    const std::string set = param_source_.empty() ? dftb_default_set(method_) : param_source_;
    if (!dftb_prepare(set, method_ == kDFTB3 ? 3 : 2, zs, dftb, err)) return kErrUnsupportedElement;
    if (uhf_)
      for (const auto& e : dftb.elems)
        if (!e.has_w) {
          err = "spin-polarised DFTB needs spin constants (spin.dat) for element Z=" + std::to_string(e.Z);
          return kErrUnsupportedElement;
        }
  }
  for (size_t i = 0; i < elems_.size() && !is_dftb(method_); ++i)
    for (size_t j = 0; j < elems_.size(); ++j) {
      DiatomicDev d = make_diatomic(method_, elems_[i].Z, elems_[j].Z, nddo_set_.get());
      if (method_ == kPM6 && !d.present) {
        err = "no PM6 diatomic parameters for the element pair Z=" + std::to_string(elems_[i].Z) + ", Z=" +
              std::to_string(elems_[j].Z);
        return kErrUnsupportedElement;
      }
      diat_[i * kMaxElementSlots + j] = d;
    }
  long long int_off = 0, mat_off = 0, diis_off = 0, gam_off = 0;
  int ao_base = 0, max_nao = 0;
  {
    size_t natoms_total = 0, nao_total = 0;
    for (const auto& m : in) {
      natoms_total += m.Z.size();
      for (int z : m.Z) nao_total += (size_t)elems_[slot_of[z]].nao;
    }
    mols_.reserve(in.size());
    atoms_.reserve(natoms_total);
    ao_atom_.reserve(nao_total);
  }
  for (size_t mi = 0; mi < in.size(); ++mi) {
    const auto& mol = in[mi];
    MolDev md{};
    md.nat = (int)mol.Z.size();
    if (md.nat > kMaxAtomsPerMolecule) {
      err = "molecule larger than the per-molecule atom limit";
      return kErrInvalidArgument;
    }
    md.atom0 = (int)atoms_.size();
    md.pair0 = (int)npairs_;
    md.ao_base = ao_base;
    int nao = 0, heavy = 0;
    double ncore = 0;
    long long s_sum = 0, s_sq = 0;  // integral block sizes per atom: 1 (s) or 10 (sp)
    for (int a = 0; a < md.nat; ++a) {
      const int slot = slot_of[mol.Z[a]];
      const ElemDev& e = elems_[slot];
      AtomDev ad{};
      ad.x = mol.xyz[3 * a];
      ad.y = mol.xyz[3 * a + 1];
      ad.z = mol.xyz[3 * a + 2];
      if (!std::isfinite(ad.x) || !std::isfinite(ad.y) || !std::isfinite(ad.z)) {
        err = "non-finite position in molecule " + std::to_string(mi);
        return kErrInvalidArgument;
      }
      ad.slot = slot;
      ad.ao0 = nao;
      ad.mol = (int)mi;
      atoms_.push_back(ad);
      for (int k = 0; k < e.nao; ++k) ao_atom_.push_back(md.atom0 + a);
      nao += e.nao;
      ncore += e.core;
      const int sz = e.nao == 1 ? 1 : 10;
      s_sum += sz;
      s_sq += sz * sz;
      heavy += e.nao == 4 ? 1 : 0;
    }
    md.nao = nao;
    // electron count in 64 bits: any int charge or multiplicity is range-checked
    // before it can size an orbital block (n_occ <= n_AO for every spin)
    const long long nel = std::llround(ncore) - (long long)mol.charge;
    if (uhf_) {
      // n_alpha - n_beta = multiplicity - 1
      const long long na2 = nel + (long long)mol.multiplicity - 1;
      if (nel < 0 || mol.multiplicity < 1 || (na2 & 1) || nel - ((long long)mol.multiplicity - 1) < 0 ||
          na2 / 2 > nao) {
        err = "molecule " + std::to_string(mi) + ": " + std::to_string(nel) +
              " electrons do not fit spin multiplicity " + std::to_string(mol.multiplicity) + " in " +
              std::to_string(nao) + " orbitals";
        return kErrOddElectrons;
      }
      md.nel = (int)nel;
      md.nocc = (int)(na2 / 2);
      md.nocc_b = md.nel - md.nocc;
    } else {
      if (nel < 0 || (nel & 1) || mol.multiplicity != 1 || nel / 2 > nao) {
        err = "molecule " + std::to_string(mi) + " has " + std::to_string(nel) + " electrons, " +
              std::to_string(nao) + " orbitals and multiplicity " + std::to_string(mol.multiplicity) +
              ": the restricted closed-shell SCF needs an even, non-negative count of at most two per "
              "orbital and a singlet (use the unrestricted SCF)";
        return kErrOddElectrons;
      }
      md.nel = (int)nel;
      md.nocc = md.nel / 2;
      md.nocc_b = md.nocc;
    }
    if (nao > 1024 && (in.size() > 1 || is_dftb(method_))) {
      err = "molecule " + std::to_string(mi) + " has more than 1024 AOs: the batched SCF limit (a single NDDO "
            "molecule of that size runs the large-molecule path)";
      return kErrInvalidArgument;
    }
    // pair p of the molecule is (lo, hi) in row-major order over lo < hi; its
    // integral block follows the blocks of the earlier pairs (sizes 1 x 1,
    // 1 x 10 or 10 x 10); the device builds the per-pair table
    md.int_off = int_off;
    md.npairs = md.nat * (md.nat - 1) / 2;
    int_off += (s_sum * s_sum - s_sq) / 2;
    if (int_off > 2000000000LL) {
      err = "batch too large: more than 2e9 two-centre integrals";
      return kErrInvalidArgument;
    }
    npairs_ += md.npairs;
    md.hh0 = (int)nhh_;
    md.nhh = heavy * (heavy - 1) / 2;
    nhh_ += md.nhh;
    md.mat_off = mat_off;
    md.diis_off = diis_off;
    md.gam_off = gam_off;
    gam_off += (long long)md.nat * md.nat;
    mat_off += (long long)nao * nao;
    diis_off += 2LL * kDiisMax * nao * nao;
    ao_base += nao;
    max_nao = std::max(max_nao, nao);
    mols_.push_back(md);
  }
  order_.resize(mols_.size());
  for (size_t i = 0; i < order_.size(); ++i) order_[i] = (int)i;
  std::stable_sort(order_.begin(), order_.end(), [&](int a, int b) { return mols_[a].nao > mols_[b].nao; });

  // arena layout
  DeviceBatch d;
  d.method = method_;
  d.nmol = (int)mols_.size();
  d.natoms = (int)atoms_.size();
  d.npairs = (int)npairs_;
  d.nhh_total = (int)nhh_;
  d.nao_total = ao_base;
  d.mat_total = mat_off;
  d.diis_total = diis_off;
  d.int_total = int_off;
  d.max_nao = max_nao;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off = align_up(off + bytes);
    return o;
  };
  const size_t o_mols = take(sizeof(MolDev) * mols_.size());
  const size_t o_atoms = take(sizeof(AtomDev) * atoms_.size());
  const size_t o_elems = take(sizeof(ElemDev) * elems_.size());
  const size_t o_diat = take(sizeof(DiatomicDev) * diat_.size());
  const size_t o_ao = take(sizeof(int) * ao_atom_.size());
  const size_t o_order = take(sizeof(int) * order_.size());
  // DFTB records, tables and splines (in the upload region)
  const bool dftb_batch = is_dftb(method_);
  size_t o_delems = 0, o_dpairs = 0, o_dtable = 0, o_dspl = 0;
  if (dftb_batch) {
    o_delems = take(sizeof(DftbElemDev) * kMaxElementSlots);
    o_dpairs = take(sizeof(DftbPairDev) * dftb.pairs.size());
    o_dtable = take(sizeof(double) * std::max<size_t>(dftb.table.size(), 1));
    o_dspl = take(sizeof(DftbSplineDev) * std::max<size_t>(dftb.splines.size(), 1));
  }
  const size_t upload_end = off;
  const size_t o_pairs = take(sizeof(PairDev) * std::max<long long>(npairs_, 1));
  const size_t o_hh = take(sizeof(int) * std::max<long long>(nhh_, 1));
  const size_t o_counter = take(sizeof(int));
  const size_t o_flag = take(sizeof(int));
  const size_t np = (size_t)std::max<long long>(npairs_, 1);
  const size_t npn = dftb_batch ? 1 : np;  // NDDO-only per-pair buffers
  const size_t o_ints = take(sizeof(double) * (dftb_batch ? 1 : std::max<long long>(int_off, 1)));
  const size_t o_vcore = take(sizeof(double) * 20 * npn);
  const size_t o_jbuf = take(sizeof(double) * 20 * npn);
  const size_t o_ovl = take(sizeof(double) * 16 * npn);
  const size_t o_erep = take(sizeof(double) * np);
  const size_t o_gpair = take(sizeof(double) * 3 * np);
  const size_t mat_bytes = sizeof(double) * (size_t)mat_off;
  const size_t o_H = take(mat_bytes), o_P = take(mat_bytes), o_F = take(mat_bytes), o_C = take(mat_bytes);
  const size_t o_W1 = take(mat_bytes), o_W2 = take(mat_bytes);
  const size_t o_eps = take(sizeof(double) * (size_t)ao_base);
  const size_t o_diis = take(sizeof(double) * (size_t)diis_off);
  const size_t o_grad = take(sizeof(double) * 3 * atoms_.size());
  if (scf_grid_ == 0 || max_nao > scf_grid_nao_) {
    scf_grid_ = scf_max_grid(max_nao);
    scf_grid_nao_ = max_nao;
  }
  const int grid_eff = std::min<int>(scf_grid_, (int)mols_.size());
  const size_t o_rot = take(scf_rotation_bytes_per_cta() * (size_t)grid_eff);
  const size_t o_res = take(sizeof(MolResult) * mols_.size());
  const size_t mat_dftb = dftb_batch ? mat_bytes : sizeof(double);
  const size_t o_S = take(mat_dftb), o_X = take(mat_dftb), o_Pp = take(mat_dftb), o_W3 = take(mat_dftb);
  const size_t gam_bytes = sizeof(double) * (dftb_batch ? std::max<long long>(gam_off, 1) : 1);
  const size_t o_gam = take(gam_bytes);
  const size_t o_Gam = take(method_ == kDFTB3 ? gam_bytes : sizeof(double));
  const size_t o_qat = take(sizeof(double) * (dftb_batch ? atoms_.size() : 1));
  const size_t o_shift = take(sizeof(double) * 4 * (dftb_batch ? atoms_.size() : 1));
  // unrestricted: spin densities, beta Fock matrix, orbitals, energies and DIIS ring
  const size_t mat_uhf = uhf_ ? mat_bytes : sizeof(double);
  const size_t o_Pa = take(mat_uhf), o_Pb = take(mat_uhf), o_Fb = take(mat_uhf), o_Cb = take(mat_uhf);
  const size_t o_epsb = take(uhf_ ? sizeof(double) * (size_t)ao_base : sizeof(double));
  const size_t o_diisb = take(uhf_ ? sizeof(double) * (size_t)diis_off : sizeof(double));
  const bool uhf_dftb = uhf_ && dftb_batch;  // spin-polarised DFTB: beta orthogonal-basis density, shell shifts
  const size_t o_Ppb = take(uhf_dftb ? mat_bytes : sizeof(double));
  const size_t o_sshift = take(sizeof(double) * 2 * (uhf_dftb ? atoms_.size() : 1));
  int rc = ensure_arena(off, err);
  if (rc) return rc;
  rc = ensure_terms(stream_, err);
  if (rc) return rc;
  char* base = static_cast<char*>(arena_);
  d.mols = reinterpret_cast<MolDev*>(base + o_mols);
  d.atoms = reinterpret_cast<AtomDev*>(base + o_atoms);
  d.pairs = reinterpret_cast<PairDev*>(base + o_pairs);
  d.elems = reinterpret_cast<ElemDev*>(base + o_elems);
  d.diat = reinterpret_cast<DiatomicDev*>(base + o_diat);
  d.ao_atom = reinterpret_cast<int*>(base + o_ao);
  d.order = reinterpret_cast<int*>(base + o_order);
  d.counter = reinterpret_cast<int*>(base + o_counter);
  d.ints = reinterpret_cast<double*>(base + o_ints);
  d.vcore = reinterpret_cast<double*>(base + o_vcore);
  d.jbuf = reinterpret_cast<double*>(base + o_jbuf);
  d.hh_pairs = reinterpret_cast<int*>(base + o_hh);
  d.ovl = reinterpret_cast<double*>(base + o_ovl);
  d.erep = reinterpret_cast<double*>(base + o_erep);
  d.gpair = reinterpret_cast<double*>(base + o_gpair);
  d.H = reinterpret_cast<double*>(base + o_H);
  d.P = reinterpret_cast<double*>(base + o_P);
  d.F = reinterpret_cast<double*>(base + o_F);
  d.C = reinterpret_cast<double*>(base + o_C);
  d.W1 = reinterpret_cast<double*>(base + o_W1);
  d.W2 = reinterpret_cast<double*>(base + o_W2);
  d.eps = reinterpret_cast<double*>(base + o_eps);
  d.diis = reinterpret_cast<double*>(base + o_diis);
  d.grad = reinterpret_cast<double*>(base + o_grad);
  d.rotbuf = reinterpret_cast<double*>(base + o_rot);
  d.scf_grid = grid_eff;
  d.res = reinterpret_cast<MolResult*>(base + o_res);
  d.S = reinterpret_cast<double*>(base + o_S);
  d.X = reinterpret_cast<double*>(base + o_X);
  d.Pp = reinterpret_cast<double*>(base + o_Pp);
  d.W3 = reinterpret_cast<double*>(base + o_W3);
  d.gam = reinterpret_cast<double*>(base + o_gam);
  d.Gam = reinterpret_cast<double*>(base + o_Gam);
  d.qat = reinterpret_cast<double*>(base + o_qat);
  d.ashift = reinterpret_cast<double*>(base + o_shift);
  d.uhf = uhf_ ? 1 : 0;
  if (uhf_) {
    d.Pa = reinterpret_cast<double*>(base + o_Pa);
    d.Pb = reinterpret_cast<double*>(base + o_Pb);
    d.Fb = reinterpret_cast<double*>(base + o_Fb);
    d.Cb = reinterpret_cast<double*>(base + o_Cb);
    d.epsb = reinterpret_cast<double*>(base + o_epsb);
    d.diisb = reinterpret_cast<double*>(base + o_diisb);
    if (uhf_dftb) {
      d.Ppb = reinterpret_cast<double*>(base + o_Ppb);
      d.sshift = reinterpret_cast<double*>(base + o_sshift);
    }
  }
  if (dftb_batch) {
    d.dftb_order = method_ == kDFTB3 ? 3 : 2;
    d.gam_total = gam_off;
    d.delems = reinterpret_cast<DftbElemDev*>(base + o_delems);
    d.dpairs = reinterpret_cast<DftbPairDev*>(base + o_dpairs);
    d.dtable = reinterpret_cast<double*>(base + o_dtable);
    d.dsplines = reinterpret_cast<DftbSplineDev*>(base + o_dspl);
  }
  dev_ = d;

  // stage the descriptors in pinned memory and upload them with one copy
  if (pinned_bytes_ < upload_end) {
    pool_give(true, pinned_, pinned_bytes_);
    pinned_ = nullptr;
    pinned_bytes_ = 0;
    size_t got = 0;
    if (void* p = pool_take(true, upload_end, &got)) {
      pinned_ = p;
      pinned_bytes_ = got;
    } else {
      cudaError_t e = cudaMallocHost(&pinned_, upload_end);
      if (e != cudaSuccess) {
        err = cuda_message(e);
        return kErrCuda;
      }
      pinned_bytes_ = upload_end;
    }
  }
  cudaStreamSynchronize(stream_);
  char* h = static_cast<char*>(pinned_);
  std::memcpy(h + o_mols, mols_.data(), sizeof(MolDev) * mols_.size());
  std::memcpy(h + o_atoms, atoms_.data(), sizeof(AtomDev) * atoms_.size());
  std::memcpy(h + o_elems, elems_.data(), sizeof(ElemDev) * elems_.size());
  std::memcpy(h + o_diat, diat_.data(), sizeof(DiatomicDev) * diat_.size());
  std::memcpy(h + o_ao, ao_atom_.data(), sizeof(int) * ao_atom_.size());
  std::memcpy(h + o_order, order_.data(), sizeof(int) * order_.size());
  if (dftb_batch) {
    std::memset(h + o_delems, 0, sizeof(DftbElemDev) * kMaxElementSlots);
    std::memcpy(h + o_delems, dftb.elems.data(), sizeof(DftbElemDev) * dftb.elems.size());
    std::memcpy(h + o_dpairs, dftb.pairs.data(), sizeof(DftbPairDev) * dftb.pairs.size());
    if (!dftb.table.empty()) std::memcpy(h + o_dtable, dftb.table.data(), sizeof(double) * dftb.table.size());
    if (!dftb.splines.empty())
      std::memcpy(h + o_dspl, dftb.splines.data(), sizeof(DftbSplineDev) * dftb.splines.size());
  }
  cudaError_t e = cudaMemcpyAsync(arena_, pinned_, upload_end, cudaMemcpyHostToDevice, stream_);
  if (e != cudaSuccess) {
    err = cuda_message(e);
    return kErrCuda;
  }
  h2d_bytes_ = (long long)upload_end;
  d2h_bytes_ = 0;
  e = cudaMemsetAsync(d.res, 0, sizeof(MolResult) * mols_.size(), stream_);
  if (e == cudaSuccess) e = cudaMemsetAsync(base + o_flag, 0, sizeof(int), stream_);
  if (e != cudaSuccess) {
    err = cuda_message(e);
    return kErrCuda;
  }
  // pair and heavy-pair tables, built on the device; coincident atoms are
  // reported through the flag (1 + global index of one offending pair)
  int max_nat = 0;
  for (const auto& m : mols_) max_nat = std::max(max_nat, m.nat);
  launch_build_pairs(d, max_nat, reinterpret_cast<int*>(base + o_flag), stream_);
  e = cudaGetLastError();
  if (!check_pairs) {
    if (e != cudaSuccess) {
      err = cuda_message(e);
      return kErrCuda;
    }
    return kOk;
  }
  int bad = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, base + o_flag, sizeof(int), cudaMemcpyDeviceToHost, stream_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
  if (e != cudaSuccess) {
    err = cuda_message(e);
    return kErrCuda;
  }
  if (bad > 0) {
    const long long pidx = bad - 1;
    size_t mi = 0;
    while (mi + 1 < mols_.size() && mols_[mi + 1].pair0 <= pidx) ++mi;
    const MolDev& m = mols_[mi];
    long long p = pidx - m.pair0;
    int lo = 0;
    while (p >= m.nat - 1 - lo) {
      p -= m.nat - 1 - lo;
      ++lo;
    }
    const int hi = lo + 1 + (int)p;
    err = "atoms " + std::to_string(lo) + " and " + std::to_string(hi) + " of molecule " + std::to_string(mi) +
          " coincide";
    mols_.clear();
    return kErrInvalidArgument;
  }
  return kOk;
}

int Batch::set_scf_path(int path, std::string& err) {
  if (path < 0 || path > 3) {
    err = "SCF path must be 0 (automatic), 1 (batched), 2 (large, FP64) or 3 (large, mixed precision)";
    return kErrInvalidArgument;
  }
  if (path >= 2 && (is_dftb(method_) || mols_.size() > 1)) {
    err = "the large-molecule SCF path takes one NDDO molecule";
    return kErrInvalidArgument;
  }
  scf_path_ = path;
  return kOk;
}

int Batch::set_positions(const double* xyz, std::string& err) {
  if (mols_.empty()) {
    err = "no structure";
    return kErrEmptyStructure;
  }
  for (size_t a = 0; a < atoms_.size(); ++a) {
    atoms_[a].x = xyz[3 * a];
    atoms_[a].y = xyz[3 * a + 1];
    atoms_[a].z = xyz[3 * a + 2];
    if (!std::isfinite(atoms_[a].x) || !std::isfinite(atoms_[a].y) || !std::isfinite(atoms_[a].z)) {
      err = "non-finite position";
      return kErrInvalidArgument;
    }
  }
  cudaStreamSynchronize(stream_);
  cudaError_t e = cudaMemcpyAsync(dev_.atoms, atoms_.data(), sizeof(AtomDev) * atoms_.size(), cudaMemcpyHostToDevice,
                                  stream_);
  h2d_bytes_ += (long long)(sizeof(AtomDev) * atoms_.size());
  if (e != cudaSuccess) {
    err = cuda_message(e);
    return kErrCuda;
  }
  return cudaStreamSynchronize(stream_) == cudaSuccess ? kOk : kErrCuda;
}

int Batch::set_start_density(const double* P, std::string& err) {
  if (mols_.empty()) {
    err = "no structure";
    return kErrEmptyStructure;
  }
  cudaError_t e = cudaMemcpyAsync(dev_.P, P, sizeof(double) * (size_t)dev_.mat_total, cudaMemcpyHostToDevice, stream_);
  if (e != cudaSuccess) {
    err = cuda_message(e);
    return kErrCuda;
  }
  density_given_ = true;
  return cudaStreamSynchronize(stream_) == cudaSuccess ? kOk : kErrCuda;
}

int Batch::set_start_spin_densities(const double* Pa, const double* Pb, std::string& err) {
  if (mols_.empty()) {
    err = "no structure";
    return kErrEmptyStructure;
  }
  if (!uhf_) {
    err = "spin densities apply to unrestricted calculations";
    return kErrInvalidArgument;
  }
  const size_t n = (size_t)dev_.mat_total;
  std::vector<double> P(n);
  for (size_t k = 0; k < n; ++k) P[k] = Pa[k] + Pb[k];
  cudaError_t e = cudaMemcpyAsync(dev_.Pa, Pa, sizeof(double) * n, cudaMemcpyHostToDevice, stream_);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dev_.Pb, Pb, sizeof(double) * n, cudaMemcpyHostToDevice, stream_);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dev_.P, P.data(), sizeof(double) * n, cudaMemcpyHostToDevice, stream_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
  if (e != cudaSuccess) {
    err = cuda_message(e);
    return kErrCuda;
  }
  density_given_ = true;
  spin_given_ = true;
  return kOk;
}

int Batch::fetch_spin_densities(int mol, std::vector<double>& Pa, std::vector<double>& Pb, std::string& err) {
  if (mol < 0 || mol >= (int)mols_.size()) {
    err = "molecule index out of range";
    return kErrInvalidArgument;
  }
  if (!dev_.uhf) {
    err = "spin densities exist for unrestricted calculations only";
    return kErrNoResults;
  }
  const MolDev& m = mols_[mol];
  Pa.resize((size_t)m.nao * m.nao);
  Pb.resize(Pa.size());
  cudaError_t e = cudaMemcpyAsync(Pa.data(), dev_.Pa + m.mat_off, sizeof(double) * Pa.size(), cudaMemcpyDeviceToHost,
                                  stream_);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(Pb.data(), dev_.Pb + m.mat_off, sizeof(double) * Pb.size(), cudaMemcpyDeviceToHost, stream_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
  if (e != cudaSuccess) {
    err = cuda_message(e);
    return kErrCuda;
  }
  return kOk;
}

int Batch::run(const ScfParams& sp_in, bool gradient, std::string& err) {
  if (mols_.empty()) {
    err = "no structure";
    return kErrEmptyStructure;
  }
  // From a given (converged) start density the first diagonalisation is
  // already the answer: give it the sweeps to resolve the orbitals fully.
  ScfParams sp = sp_in;
  if (density_given_) sp.cold_sweeps = std::max(sp.cold_sweeps, 6);
  dev_.use_guess = density_given_ ? 0 : 1;
  dev_.spin_given = spin_given_ ? 1 : 0;
  for (auto& ev : stage_ev_)
    if (!ev) cudaEventCreate(&ev);
  launches_ = 0;
  cudaEventRecord(stage_ev_[0], stream_);
  if (is_dftb(method_)) {
    // pair and on-site terms (+ start density) | SCC loop | gradient
    launch_dftb_setup(dev_, stream_);
    launches_ += dev_.npairs > 0 ? 2 : 1;
    cudaEventRecord(stage_ev_[1], stream_);
    cudaEventRecord(stage_ev_[2], stream_);
    launch_dftb_scf(dev_, sp, dev_.scf_grid, stream_);
    launches_ += 1;
    if (sp.canonical) {
      launch_dftb_canonical(dev_, sp, dev_.scf_grid, stream_);
      launches_ += 1;
    }
    cudaEventRecord(stage_ev_[3], stream_);
    if (gradient) {
      launch_dftb_gradient(dev_, stream_);
      launches_ += dev_.npairs > 0 ? 2 : 1;
    }
  } else {
    const int N = mols_[0].nao;
    const bool large = mols_.size() == 1 && (scf_path_ >= 2 || (scf_path_ == 0 && N > 1024));
    if (scf_path_ >= 2 && mols_.size() > 1) {
      err = "the large-molecule SCF path takes one NDDO molecule";
      return kErrInvalidArgument;
    }
    if (large && uhf_) {
      err = "the unrestricted SCF runs on the batched path (at most 1024 AOs)";
      return kErrInvalidArgument;
    }
    if (!large && mols_[0].nao > 1024) {
      err = "more than 1024 AOs needs the large-molecule SCF path";
      return kErrInvalidArgument;
    }
    if (large) {
      const size_t need = large_scf_scratch_bytes(N);
      if (large_scratch_bytes_ < need) {
        if (large_scratch_) {
          cudaStreamSynchronize(stream_);
          cudaFree(large_scratch_);
          large_scratch_ = nullptr;
          large_scratch_bytes_ = 0;
        }
        cudaError_t e = device_alloc(&large_scratch_, need);
        if (e != cudaSuccess) {
          cudaGetLastError();
          large_scratch_ = nullptr;
          err = "device allocation of " + std::to_string(need) + " bytes failed: " + cudaGetErrorString(e);
          return e == cudaErrorMemoryAllocation ? kErrOutOfMemory : kErrCuda;
        }
        large_scratch_bytes_ = need;
      }
    }
    dev_.large = large ? 1 : 0;
    dev_.large_scratch = large ? large_scratch_ : nullptr;
    launch_pair_values(dev_, stream_);
    launches_ += (dev_.npairs > 0 ? 1 : 0) + (dev_.nhh_total > 0 ? 1 : 0);
    cudaEventRecord(stage_ev_[1], stream_);
    launch_one_electron(dev_, stream_);
    launches_ += 1;
    cudaEventRecord(stage_ev_[2], stream_);
    if (large) {
      // host-driven: returns when the SCF is done
      const int rc = run_large_scf(dev_, mols_[0], sp, scf_path_ == 3 ? 1 : 0, stream_, &launches_, err);
      if (rc != kOk) return rc;
    } else {
      if (uhf_) launch_uhf_scf(dev_, sp, dev_.scf_grid, stream_);
      else launch_scf(dev_, sp, dev_.scf_grid, stream_);
      launches_ += 1;
      if (sp.canonical) {
        launch_canonical(dev_, sp, dev_.scf_grid, stream_);
        launches_ += 1;
      }
    }
    cudaEventRecord(stage_ev_[3], stream_);
    if (gradient) {
      launch_gradient(dev_, stream_);
      launches_ += dev_.npairs > 0 ? 2 : 1;
    }
  }
  cudaEventRecord(stage_ev_[4], stream_);
  stages_recorded_ = true;
  density_given_ = false;
  spin_given_ = false;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    err = cuda_message(e);
    return kErrCuda;
  }
  return kOk;
}

int Batch::fetch(std::vector<MoleculeOutput>& out, bool gradient, std::string& err) {
  std::vector<MolResult> r(mols_.size());
  cudaError_t e = cudaMemcpyAsync(r.data(), dev_.res, sizeof(MolResult) * r.size(), cudaMemcpyDeviceToHost, stream_);
  std::vector<double> g;
  if (e == cudaSuccess && gradient) {
    g.resize(3 * atoms_.size());
    e = cudaMemcpyAsync(g.data(), dev_.grad, sizeof(double) * g.size(), cudaMemcpyDeviceToHost, stream_);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
  if (e != cudaSuccess) {
    err = cuda_message(e);
    return kErrCuda;
  }
  d2h_bytes_ += (long long)(sizeof(MolResult) * r.size() + sizeof(double) * g.size());
  out.resize(mols_.size());
  for (size_t i = 0; i < mols_.size(); ++i) {
    MoleculeOutput& o = out[i];
    o.energy = r[i].energy;
    o.e_el = r[i].e_el;
    o.e_rep = r[i].e_rep;
    o.iterations = r[i].iterations;
    o.converged = r[i].converged;
    o.status = r[i].status;
    o.nao = mols_[i].nao;
    o.nocc = mols_[i].nocc;
    o.nocc_b = mols_[i].nocc_b;
    o.nel = mols_[i].nel;
    if (gradient)
      o.gradient.assign(g.begin() + 3 * mols_[i].atom0, g.begin() + 3 * (mols_[i].atom0 + mols_[i].nat));
    else
      o.gradient.clear();
  }
  return kOk;
}

int Batch::run_tddftb(int nroots, bool triplet, double tol, int max_iter, std::string& err) {
  if (mols_.empty()) {
    err = "no structure";
    return kErrEmptyStructure;
  }
  if (!is_dftb(method_) || uhf_) {
    err = "TD-DFTB needs a restricted DFTB2 or DFTB3 reference";
    return kErrInvalidArgument;
  }
  if (!stages_recorded_) {
    err = "TD-DFTB needs a converged reference: run the batch first";
    return kErrNoResults;
  }
  if (nroots < 1 || nroots > 16 || !(tol > 0) || max_iter < 1) {
    err = "TD-DFTB: 1 <= nroots <= 16, tol > 0, max_iter >= 1";
    return kErrInvalidArgument;
  }
  // per-molecule scratch blocks, then the result arrays
  std::vector<long long> off(mols_.size());
  long long total = 0;
  for (size_t i = 0; i < mols_.size(); ++i) {
    const MolDev& m = mols_[i];
    const int dim = m.nocc * (m.nao - m.nocc);
    const int k = nroots < dim ? nroots : dim;
    off[i] = total;
    total += dim > 0 ? td_block_doubles(dim, m.nat, k) : 0;
    total = (total + 31) & ~31LL;
  }
  const size_t n = mols_.size();
  const size_t need = sizeof(double) * (size_t)total + sizeof(long long) * n + sizeof(double) * n * nroots * 4 +
                      sizeof(int) * 2 * n + sizeof(long long) * 3 * n + 5 * 256;
  if (td_scratch_bytes_ < need) {
    if (td_scratch_) {
      cudaStreamSynchronize(stream_);
      cudaFree(td_scratch_);
      td_scratch_ = nullptr;
      td_scratch_bytes_ = 0;
    }
    cudaError_t e = device_alloc(&td_scratch_, need);
    if (e != cudaSuccess) {
      cudaGetLastError();
      td_scratch_ = nullptr;
      err = "device allocation of " + std::to_string(need) + " bytes failed: " + cudaGetErrorString(e);
      return e == cudaErrorMemoryAllocation ? kErrOutOfMemory : kErrCuda;
    }
    td_scratch_bytes_ = need;
  }
  char* p = static_cast<char*>(td_scratch_);
  double* td = reinterpret_cast<double*>(p);
  size_t o = align_up(sizeof(double) * (size_t)total);
  long long* d_off = reinterpret_cast<long long*>(p + o);
  o = align_up(o + sizeof(long long) * n);
  td_omega_ = reinterpret_cast<double*>(p + o);
  o = align_up(o + sizeof(double) * n * nroots);
  td_dip_ = reinterpret_cast<double*>(p + o);
  o = align_up(o + sizeof(double) * n * nroots * 3);
  td_info_ = reinterpret_cast<int*>(p + o);
  o = align_up(o + sizeof(int) * 2 * n);
  td_cycles_ = reinterpret_cast<long long*>(p + o);
  td_roots_ = nroots;
  cudaError_t e = cudaMemcpyAsync(d_off, off.data(), sizeof(long long) * n, cudaMemcpyHostToDevice, stream_);
  if (e != cudaSuccess) {
    err = cuda_message(e);
    return kErrCuda;
  }
  // the copy reads the host vector: wait before it goes out of scope
  e = cudaStreamSynchronize(stream_);
  if (e != cudaSuccess) {
    err = cuda_message(e);
    return kErrCuda;
  }
  h2d_bytes_ += (long long)(sizeof(long long) * n);
  launch_tddftb(dev_, td, d_off, nroots, triplet ? 1 : 0, tol, max_iter, td_omega_, td_dip_, td_info_, td_cycles_,
                dev_.scf_grid, stream_);
  launches_ += 1;
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    err = cuda_message(e);
    return kErrCuda;
  }
  return kOk;
}

int Batch::fetch_tddftb(std::vector<double>& omega, std::vector<double>& dip, std::vector<int>& info, std::string& err) {
  if (!td_roots_) {
    err = "no TD-DFTB run";
    return kErrNoResults;
  }
  const size_t n = mols_.size();
  omega.resize(n * td_roots_);
  dip.resize(n * td_roots_ * 3);
  info.resize(2 * n);
  cudaError_t e = cudaMemcpyAsync(omega.data(), td_omega_, sizeof(double) * omega.size(), cudaMemcpyDeviceToHost,
                                  stream_);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dip.data(), td_dip_, sizeof(double) * dip.size(), cudaMemcpyDeviceToHost, stream_);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(info.data(), td_info_, sizeof(int) * info.size(), cudaMemcpyDeviceToHost, stream_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
  if (e != cudaSuccess) {
    err = cuda_message(e);
    return kErrCuda;
  }
  d2h_bytes_ += (long long)(sizeof(double) * (omega.size() + dip.size()) + sizeof(int) * info.size());
  return kOk;
}

int Batch::fetch_tddftb_cycles(std::vector<long long>& cycles, std::string& err) {
  if (!td_roots_) {
    err = "no TD-DFTB run";
    return kErrNoResults;
  }
  cycles.resize(3 * mols_.size());
  cudaError_t e = cudaMemcpyAsync(cycles.data(), td_cycles_, sizeof(long long) * cycles.size(), cudaMemcpyDeviceToHost,
                                  stream_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
  if (e != cudaSuccess) {
    err = cuda_message(e);
    return kErrCuda;
  }
  return kOk;
}

int Batch::fetch_raw_results(std::vector<MolResult>& r, std::string& err) {
  r.resize(mols_.size());
  cudaError_t e = cudaMemcpyAsync(r.data(), dev_.res, sizeof(MolResult) * r.size(), cudaMemcpyDeviceToHost, stream_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
  if (e != cudaSuccess) {
    err = cuda_message(e);
    return kErrCuda;
  }
  return kOk;
}

int Batch::fetch_density(int mol, std::vector<double>& P, std::string& err) {
  if (mol < 0 || mol >= (int)mols_.size()) {
    err = "molecule index out of range";
    return kErrInvalidArgument;
  }
  const MolDev& m = mols_[mol];
  P.resize((size_t)m.nao * m.nao);
  cudaError_t e = cudaMemcpyAsync(P.data(), dev_.P + m.mat_off, sizeof(double) * P.size(), cudaMemcpyDeviceToHost,
                                  stream_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
  if (e != cudaSuccess) {
    err = cuda_message(e);
    return kErrCuda;
  }
  return kOk;
}

int Batch::fetch_charges(int mol, std::vector<double>& q, std::string& err) {
  if (mol < 0 || mol >= (int)mols_.size()) {
    err = "molecule index out of range";
    return kErrInvalidArgument;
  }
  const MolDev& m = mols_[mol];
  q.resize(m.nat);
  if (is_dftb(method_)) {
    cudaError_t e = cudaMemcpyAsync(q.data(), dev_.qat + m.atom0, sizeof(double) * m.nat, cudaMemcpyDeviceToHost,
                                    stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    if (e != cudaSuccess) {
      err = cuda_message(e);
      return kErrCuda;
    }
    return kOk;
  }
  std::vector<double> P;
  const int rc = fetch_density(mol, P, err);
  if (rc) return rc;
  for (int a = 0; a < m.nat; ++a) {
    const AtomDev& A = atoms_[m.atom0 + a];
    const ElemDev& E = elems_[A.slot];
    double pop = 0;
    for (int k = 0; k < E.nao; ++k) pop += P[(size_t)(A.ao0 + k) * m.nao + A.ao0 + k];
    q[a] = E.core - pop;
  }
  return kOk;
}

int Batch::dipole(int mol, double out[3], std::string& err) {
  std::vector<double> q;
  int rc = fetch_charges(mol, q, err);
  if (rc) return rc;
  const MolDev& m = mols_[mol];
  out[0] = out[1] = out[2] = 0.0;
  if (is_dftb(method_)) {
    for (int a = 0; a < m.nat; ++a) {
      const AtomDev& A = atoms_[m.atom0 + a];
      out[0] += q[a] * A.x;
      out[1] += q[a] * A.y;
      out[2] += q[a] * A.z;
    }
    return kOk;
  }
  std::vector<double> P;
  rc = fetch_density(mol, P, err);
  if (rc) return rc;
  double com[3] = {0, 0, 0}, mass = 0;
  for (int a = 0; a < m.nat; ++a) {
    const AtomDev& A = atoms_[m.atom0 + a];
    const double w = standard_atomic_mass(elems_[A.slot].Z);
    com[0] += w * A.x;
    com[1] += w * A.y;
    com[2] += w * A.z;
    mass += w;
  }
  for (double& c : com) c = mass > 0 ? c / mass : 0.0;
  for (int a = 0; a < m.nat; ++a) {
    const AtomDev& A = atoms_[m.atom0 + a];
    const ElemDev& E = elems_[A.slot];
    out[0] += q[a] * (A.x - com[0]);
    out[1] += q[a] * (A.y - com[1]);
    out[2] += q[a] * (A.z - com[2]);
    if (E.nao == 4)
      for (int k = 0; k < 3; ++k) out[k] -= 2.0 * E.D[1] * P[(size_t)A.ao0 * m.nao + A.ao0 + 1 + k];
  }
  return kOk;
}

int Batch::fetch_orbital_energies(int mol, std::vector<double>& eps, std::string& err, bool beta) {
  if (mol < 0 || mol >= (int)mols_.size()) {
    err = "molecule index out of range";
    return kErrInvalidArgument;
  }
  if (beta && !dev_.uhf) {
    err = "beta orbital energies exist for unrestricted calculations only";
    return kErrNoResults;
  }
  if (dev_.large) {
    err = "the large-molecule path (density purification) computes no orbitals";
    return kErrNoResults;
  }
  const MolDev& m = mols_[mol];
  eps.resize(m.nao);
  const double* src = (beta ? dev_.epsb : dev_.eps) + m.ao_base;
  cudaError_t e = cudaMemcpyAsync(eps.data(), src, sizeof(double) * m.nao, cudaMemcpyDeviceToHost, stream_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
  if (e != cudaSuccess) {
    err = cuda_message(e);
    return kErrCuda;
  }
  return kOk;
}

int Batch::stage_times(double ms[4], std::string& err) {
  if (!stages_recorded_) {
    err = "no run recorded";
    return kErrNoResults;
  }
  cudaError_t e = cudaEventSynchronize(stage_ev_[4]);
  for (int i = 0; i < 4 && e == cudaSuccess; ++i) {
    float t = 0;
    e = cudaEventElapsedTime(&t, stage_ev_[i], stage_ev_[i + 1]);
    ms[i] = t;
  }
  if (e != cudaSuccess) {
    err = cuda_message(e);
    return kErrCuda;
  }
  return kOk;
}

int Batch::record_event(int slot, std::string& err) {
  if (slot < 0 || slot >= 8 || !stream_) {
    err = "bad event slot or no stream";
    return kErrInvalidArgument;
  }
  if (!user_ev_[slot]) cudaEventCreate(&user_ev_[slot]);
  cudaError_t e = cudaEventRecord(user_ev_[slot], stream_);
  if (e != cudaSuccess) {
    err = cuda_message(e);
    return kErrCuda;
  }
  return kOk;
}

int Batch::event_elapsed(int s0, int s1, double* ms, std::string& err) {
  if (s0 < 0 || s0 >= 8 || s1 < 0 || s1 >= 8 || !user_ev_[s0] || !user_ev_[s1]) {
    err = "event not recorded";
    return kErrInvalidArgument;
  }
  cudaError_t e = cudaEventSynchronize(user_ev_[s1]);
  float t = 0;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, user_ev_[s0], user_ev_[s1]);
  if (e != cudaSuccess) {
    err = cuda_message(e);
    return kErrCuda;
  }
  *ms = t;
  return kOk;
}

}  // namespace sgb
