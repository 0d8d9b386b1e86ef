// Request server: continuous batching of single-point requests on one GPU.
//
// Requests (method, structure, charge, properties) are queued by any number
// of client threads.  A worker thread keeps up to `slots` batches in flight,
// each on its own CUDA stream with its own device arena.  Whenever a slot is
// free it admits the oldest pending requests of one method, in arrival order,
// as long as the estimated device memory of all in-flight batches stays
// within the budget and the batch within the budget's per-slot share (each
// slot keeps its arena between batches), and launches them; finished batches are retired by
// event polling, their results handed to the waiting clients, and the slot
// is refilled at once.  A batch holds one method and one size class (AO
// count in steps of 64 up to 448, then larger): a batch finishes with its
// slowest molecule, so small requests are never held behind large ones.  Every request's integrals, density and DIIS history
// stay resident on the device for the whole SCF of its batch.  Each
// molecule is solved by its own CTA with the same code path whatever else is
// in the batch, so a result does not depend on the mix it was admitted with.
#pragma once
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "engine.h"

namespace sgb {

struct ServerRequest {
  long long id = 0;
  Method method = kPM6;
  MoleculeInput mol;
  bool gradient = false;
  double t_submit = 0;  // seconds, steady clock
  size_t bytes = 0;     // estimated device bytes
  int size_class = 0;   // AO-count class: batches never mix classes
  bool uhf = false;     // unrestricted (multiplicity != 1): batches never mix spin treatments
};

struct ServerResult {
  int status = kOk;
  double energy = 0;
  int iterations = 0, converged = 0;
  std::vector<double> gradient;
  double t_submit = 0, t_admit = 0, t_done = 0;  // seconds, steady clock
  int batch_size = 0;
  std::string error;
};

struct ServerStats {
  long long submitted = 0, completed = 0, batches = 0;
  long long max_batch = 0;
  double busy_seconds = 0;
};

class Server {
 public:
  Server(size_t device_budget_bytes, int slots, int max_batch, const ScfParams& sp);
  ~Server();
  Server(const Server&) = delete;
  Server& operator=(const Server&) = delete;

  // Queue a request; returns its id (> 0) or a negative Status on invalid input.
  // mol.multiplicity != 1 runs the unrestricted SCF (the reference's spin mode "any")
  long long submit(Method m, MoleculeInput&& mol, bool gradient, std::string& err);
  // Block until request id is done (timeout_s < 0: forever).  Returns 0 and
  // moves the result out, or 1 on timeout, or kErrInvalidArgument for an
  // unknown id.
  int wait(long long id, ServerResult& out, double timeout_s);
  // Non-blocking: 0 done (result moved out), 1 pending, kErrInvalidArgument unknown.
  int poll(long long id, ServerResult& out);
  // Block until every submitted request is done.
  void drain();
  ServerStats stats();
  static double now();
  // Estimated device bytes a molecule occupies inside a batch.
  static size_t estimate_bytes(Method m, const MoleculeInput& mol, bool uhf = false);

 private:
  struct Slot {
    std::unique_ptr<Batch> batch;
    std::vector<ServerRequest> reqs;
    cudaEvent_t done = nullptr;
    bool busy = false, gradient = false;
    size_t bytes = 0;
    double t_admit = 0;
  };
  void worker();
  bool launch(Slot& slot, std::vector<ServerRequest>&& reqs);
  void retire(Slot& slot);

  size_t budget_;
  int max_batch_;
  ScfParams sp_;
  std::vector<Slot> slots_;
  std::mutex mu_;
  std::condition_variable cv_work_, cv_done_;
  std::deque<ServerRequest> pending_;
  std::unordered_map<long long, ServerResult> done_;
  std::unordered_map<long long, bool> known_;
  long long next_id_ = 1;
  size_t inflight_bytes_ = 0;
  int inflight_ = 0;
  bool stop_ = false;
  int device_ = 0;
  ServerStats stats_;
  std::thread thread_;
};

}  // namespace sgb
