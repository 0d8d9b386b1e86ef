#include "server.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <map>

#include "params.h"
#include "dftb_params.h"

namespace sgb {

namespace {

// Core charge of (method, Z), or -1 when the engine cannot treat the element.
double core_charge(Method m, int z) {
  static std::mutex mu;
  static std::map<std::pair<int, int>, double> cache;
  std::lock_guard<std::mutex> lk(mu);
  auto key = std::make_pair((int)m, z);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  double c = -1;
  if (is_dftb(m)) {
    if (engine_n_aos(m, z) > 0) c = dftb_core_charge(dftb_default_set(m), z);
  } else if (engine_n_aos(m, z) > 0) {
    ElemDev e;
    std::string why;
    if (make_elem(m, z, e, why)) c = e.core;
  }
  cache[key] = c;
  return c;
}

}  // namespace

double Server::now() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

size_t Server::estimate_bytes(Method m, const MoleculeInput& mol, bool uhf) {
  long long nao = 0, s_sum = 0, s_sq = 0;
  for (int z : mol.Z) {
    const int n = engine_n_aos(m, z);
    nao += n;
    const int s = n == 1 ? 1 : 10;
    s_sum += s;
    s_sq += s * s;
  }
  const long long nat = (long long)mol.Z.size();
  const long long pairs = nat * (nat - 1) / 2;
  const long long nint = (s_sum * s_sum - s_sq) / 2;
  // matrices H P F C W1 W2 + DIIS ring + eps, integrals, per-pair buffers and tables, atoms, AO map
  // (unrestricted: four more matrices, a second DIIS ring and orbital energies)
  const long long spin = uhf ? 8 * (5 * nao * nao + 2LL * kDiisMax * nao * nao + nao + 2 * nat) : 0;
  long long b = spin + 8 * (6 * nao * nao + 2LL * kDiisMax * nao * nao + nao) + 8 * nint +
                pairs * (8 * (20 + 20 + 16 + 1 + 3) + (long long)sizeof(PairDev) + 4) +
                nat * ((long long)sizeof(AtomDev) + 24) + 4 * nao + (long long)sizeof(MolDev) + sizeof(MolResult) + 4096;
  return (size_t)b;
}

Server::Server(size_t budget, int slots, int max_batch, const ScfParams& sp)
    : budget_(budget), max_batch_(max_batch < 1 ? 1 : max_batch), sp_(sp) {
  cudaGetDevice(&device_);
  slots_.resize(slots < 1 ? 1 : slots);
  thread_ = std::thread(&Server::worker, this);
}

Server::~Server() {
  {
    std::lock_guard<std::mutex> lk(mu_);
    stop_ = true;
  }
  cv_work_.notify_all();
  if (thread_.joinable()) thread_.join();
}

long long Server::submit(Method m, MoleculeInput&& mol, bool gradient, std::string& err) {
  const int n = (int)mol.Z.size();
  if (n == 0) {
    err = "empty molecular structure";
    return -kErrEmptyStructure;
  }
  if (mol.xyz.size() != 3 * (size_t)n) {
    err = "positions must have 3 entries per atom";
    return -kErrInvalidArgument;
  }
  if (n > kMaxAtomsPerMolecule) {
    err = "molecule larger than the per-molecule atom limit";
    return -kErrInvalidArgument;
  }
  double ncore = 0;
  long long nao = 0;
  for (int z : mol.Z) {
    const double c = core_charge(m, z);
    if (c < 0) {
      err = std::string("no ") + method_name(m) + " s/p parameters for element Z=" + std::to_string(z);
      return -kErrUnsupportedElement;
    }
    ncore += c;
    nao += engine_n_aos(m, z);
  }
  if (nao > 1024) {
    err = "more than 1024 AOs (batched SCF limit)";
    return -kErrInvalidArgument;
  }
  const long long nel = std::lround(ncore) - mol.charge;
  const bool uhf = mol.multiplicity != 1;
  if (uhf) {
    const long long na2 = nel + mol.multiplicity - 1;
    if (mol.multiplicity < 1 || nel < 0 || (na2 & 1) || nel - (mol.multiplicity - 1) < 0 || na2 / 2 > nao) {
      err = std::to_string(nel) + " electrons do not fit spin multiplicity " + std::to_string(mol.multiplicity);
      return -kErrOddElectrons;
    }
  } else if (nel < 0 || (nel & 1)) {
    err = std::to_string(nel) + " electrons: a singlet needs an even, non-negative count";
    return -kErrOddElectrons;
  }
  for (int a = 0; a < n; ++a) {
    const double* p = &mol.xyz[3 * a];
    if (!std::isfinite(p[0]) || !std::isfinite(p[1]) || !std::isfinite(p[2])) {
      err = "non-finite position of atom " + std::to_string(a);
      return -kErrInvalidArgument;
    }
    for (int b = 0; b < a; ++b) {
      const double* q = &mol.xyz[3 * b];
      const double dx = p[0] - q[0], dy = p[1] - q[1], dz = p[2] - q[2];
      if (dx * dx + dy * dy + dz * dz < 1e-12) {
        err = "atoms " + std::to_string(b) + " and " + std::to_string(a) + " coincide";
        return -kErrInvalidArgument;
      }
    }
  }
  ServerRequest r;
  r.method = m;
  r.gradient = gradient;
  r.uhf = uhf;
  r.bytes = estimate_bytes(m, mol, uhf);
  r.size_class = (int)std::min<long long>((nao - 1) / 64, 7);
  r.mol = std::move(mol);
  r.t_submit = now();
  long long id;
  {
    std::lock_guard<std::mutex> lk(mu_);
    id = next_id_++;
    r.id = id;
    known_[id] = true;
    pending_.push_back(std::move(r));
    ++stats_.submitted;
  }
  cv_work_.notify_one();
  return id;
}

int Server::wait(long long id, ServerResult& out, double timeout_s) {
  std::unique_lock<std::mutex> lk(mu_);
  if (!known_.count(id)) return kErrInvalidArgument;
  auto ready = [&] { return done_.count(id) > 0; };
  if (timeout_s < 0) {
    cv_done_.wait(lk, ready);
  } else if (!cv_done_.wait_for(lk, std::chrono::duration<double>(timeout_s), ready)) {
    return 1;
  }
  out = std::move(done_[id]);
  done_.erase(id);
  known_.erase(id);
  return 0;
}

int Server::poll(long long id, ServerResult& out) {
  std::lock_guard<std::mutex> lk(mu_);
  if (!known_.count(id)) return kErrInvalidArgument;
  auto it = done_.find(id);
  if (it == done_.end()) return 1;
  out = std::move(it->second);
  done_.erase(it);
  known_.erase(id);
  return 0;
}

void Server::drain() {
  std::unique_lock<std::mutex> lk(mu_);
  cv_done_.wait(lk, [&] { return pending_.empty() && inflight_ == 0; });
}

ServerStats Server::stats() {
  std::lock_guard<std::mutex> lk(mu_);
  return stats_;
}

bool Server::launch(Slot& s, std::vector<ServerRequest>&& reqs) {
  const Method m = reqs.front().method;
  const bool uhf = reqs.front().uhf;
  std::vector<MoleculeInput> mols(reqs.size());
  s.gradient = false;
  for (size_t i = 0; i < reqs.size(); ++i) {
    mols[i] = std::move(reqs[i].mol);
    s.gradient = s.gradient || reqs[i].gradient;
  }
  s.reqs = std::move(reqs);
  if (!s.batch || s.batch->method() != m) s.batch.reset(new Batch(m));
  s.batch->set_unrestricted(uhf);
  std::string err;
  int rc = s.batch->setup(mols, err, false);
  if (rc == kOk) rc = s.batch->run(sp_, s.gradient, err);
  cudaError_t e = cudaSuccess;
  if (rc == kOk) {
    if (!s.done) e = cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(s.done, s.batch->stream());
    if (e != cudaSuccess) {
      rc = kErrCuda;
      err = cuda_message(e);
    }
  }
  if (rc != kOk) {
    const double t = now();
    std::lock_guard<std::mutex> lk(mu_);
    for (auto& r : s.reqs) {
      ServerResult& o = done_[r.id];
      o.status = rc;
      o.error = err;
      o.t_submit = r.t_submit;
      o.t_admit = s.t_admit;
      o.t_done = t;
      ++stats_.completed;
    }
    s.reqs.clear();
    s.busy = false;
    inflight_bytes_ -= s.bytes;
    --inflight_;
    cv_done_.notify_all();
    return false;
  }
  return true;
}

void Server::retire(Slot& s) {
  std::vector<MoleculeOutput> outs;
  std::string err;
  const int rc = s.batch->fetch(outs, s.gradient, err);
  const double t = now();
  std::lock_guard<std::mutex> lk(mu_);
  for (size_t i = 0; i < s.reqs.size(); ++i) {
    const ServerRequest& r = s.reqs[i];
    ServerResult& o = done_[r.id];
    o.t_submit = r.t_submit;
    o.t_admit = s.t_admit;
    o.t_done = t;
    o.batch_size = (int)s.reqs.size();
    if (rc != kOk) {
      o.status = rc;
      o.error = err;
    } else {
      const MoleculeOutput& mo = outs[i];
      o.energy = mo.energy;
      o.iterations = mo.iterations;
      o.converged = mo.converged;
      if (r.gradient) o.gradient = mo.gradient;
      if (mo.status != kDevOk) {
        o.status = kErrDevice;
        o.error = "device SCF failure code " + std::to_string(mo.status);
      } else {
        o.status = mo.converged ? kOk : kErrNotConverged;
      }
    }
    ++stats_.completed;
  }
  s.reqs.clear();
  s.busy = false;
  inflight_bytes_ -= s.bytes;
  --inflight_;
  // an arena grown past the slot's share (a request larger than the share)
  // goes back to the pool instead of staying with the idle slot
  if (s.batch && (size_t)s.batch->device_bytes() > budget_ / slots_.size()) s.batch.reset();
  cv_done_.notify_all();
}

void Server::worker() {
  cudaSetDevice(device_);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_);
  std::unique_lock<std::mutex> lk(mu_);
  while (true) {
    bool progress = false;
    // retire finished batches
    for (auto& s : slots_) {
      if (!s.busy) continue;
      if (cudaEventQuery(s.done) != cudaSuccess) continue;
      lk.unlock();
      retire(s);
      lk.lock();
      progress = true;
    }
    // admit pending requests into free slots: the oldest request fixes the
    // method, spin treatment and size class; later matching requests follow in arrival order while
    // the device budget allows (one batch is always admitted when the device
    // is otherwise idle, so progress never depends on the budget)
    // a batch stays within the budget's per-slot share (one request larger
    // than that runs alone): every slot keeps its arena between batches, so
    // the arenas held by all slots, busy or idle, stay within the budget
    const size_t share = budget_ / slots_.size();
    for (auto& s : slots_) {
      if (s.busy || pending_.empty()) continue;
      const Method m = pending_.front().method;
      const int cls = pending_.front().size_class;
      const bool uhf = pending_.front().uhf;
      std::vector<ServerRequest> take;
      size_t bytes = 0;
      for (auto it = pending_.begin(); it != pending_.end() && (int)take.size() < max_batch_;) {
        if (it->method != m || it->size_class != cls || it->uhf != uhf) {
          ++it;
          continue;
        }
        const size_t add = it->bytes + ((int)take.size() < sms ? kScfRotationBytesPerCta : 0);
        if (!take.empty() && bytes + add > share) break;
        if (inflight_bytes_ + bytes + add > budget_ && (!take.empty() || inflight_ > 0)) break;
        bytes += add;
        take.push_back(std::move(*it));
        it = pending_.erase(it);
      }
      if (take.empty()) break;
      s.busy = true;
      s.bytes = bytes;
      s.t_admit = now();
      inflight_bytes_ += bytes;
      ++inflight_;
      ++stats_.batches;
      stats_.max_batch = std::max<long long>(stats_.max_batch, (long long)take.size());
      lk.unlock();
      launch(s, std::move(take));
      lk.lock();
      progress = true;
    }
    if (stop_ && pending_.empty() && inflight_ == 0) break;
    if (!progress) {
      if (inflight_ > 0) {
        lk.unlock();
        std::this_thread::sleep_for(std::chrono::microseconds(20));
        lk.lock();
      } else {
        cv_work_.wait(lk, [&] { return stop_ || !pending_.empty(); });
      }
    }
  }
  lk.unlock();
  for (auto& s : slots_) {
    if (s.done) cudaEventDestroy(s.done);
    s.batch.reset();
  }
}

}  // namespace sgb
