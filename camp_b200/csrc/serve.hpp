// Serving loop (continuous batching of column solves); see serve.cpp.
#pragma once

#include <condition_variable>
#include <cstddef>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "engine.hpp"

namespace campb {

// First-fit allocator over one pre-allocated range (device or pinned host).
class Arena {
 public:
  void reset(char* base, size_t bytes) {
    base_ = base;
    free_.clear();
    if (bytes) free_[0] = bytes;
  }
  char* alloc(size_t bytes) {
    bytes = (bytes + 255) & ~size_t(255);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < bytes) continue;
      size_t off = it->first, len = it->second;
      free_.erase(it);
      if (len > bytes) free_[off + bytes] = len - bytes;
      used_[off] = bytes;
      return base_ + off;
    }
    return nullptr;
  }
  void release(char* p) {
    if (!p) return;
    size_t off = (size_t)(p - base_);
    auto u = used_.find(off);
    if (u == used_.end()) return;
    size_t len = u->second;
    used_.erase(u);
    auto next = free_.lower_bound(off);
    if (next != free_.end() && off + len == next->first) {
      len += next->second;
      next = free_.erase(next);
    }
    if (next != free_.begin()) {
      auto prev = std::prev(next);
      if (prev->first + prev->second == off) {
        prev->second += len;
        return;
      }
    }
    free_[off] = len;
  }

 private:
  char* base_ = nullptr;
  std::map<size_t, size_t> free_, used_;
};

class Server {
 public:
  Server();
  ~Server();
  // n_slots concurrent requests; device and pinned-host budgets in bytes for
  // the requests' buffers (slot scratch comes on top, sized per mechanism)
  bool init(int n_slots, size_t device_bytes, size_t host_bytes, std::string* err);
  // a mechanism = an initialised engine and the settings its solves use
  int add_mechanism(Engine* engine, const SolveSettings& settings, int n_state, int n_photo,
                    std::string* err);
  // Queues a column solve.  The caller's arrays (state [n * n_state], env
  // [n * 2], photo [n * n_photo]) stay valid until wait() returns; state is
  // updated there.  Returns the request id or -1.
  long submit(int mech, double* state, const double* env, const double* photo, int n,
              double t0, double t1, std::string* err);
  // Blocks until the request is done: 0 every cell ok, 1 some cell failed,
  // -1 error.  Latency is submit-to-completion.
  int wait(long id, double* latency_ms, std::vector<CellStats>* stats, std::string* err);
  int pending();

  // Device-resident columns: the column's concentrations are copied to the
  // device once (open_column) and stay there; each submit_column advances
  // them over one host step, taking only the step's env and host-set rates
  // from the host, and the next step of a column starts when its previous
  // one is done.  read_column copies the current concentrations back (after
  // the column's queued steps), close_column returns its memory.  Each step
  // restarts the BDF history, as every solver_run of the reference does
  // (CVodeReInit), so k steps of a column equal k solver_run calls.
  long open_column(int mech, const double* state, int n, std::string* err);
  long submit_column(long column, const double* env, const double* photo, double t0, double t1,
                     std::string* err);
  int read_column(long column, double* state, std::string* err);
  int close_column(long column, std::string* err);

 private:
  struct Req;
  struct Batch;
  struct Slot;
  struct Column {
    int mech = 0, n = 0;
    char* d_state = nullptr;  // n * n_state doubles in the device budget
    int queued = 0;           // submitted steps not yet finished
    bool running = false;     // a step is in a launched batch
  };
  bool column_idle(long column);
  struct Mech {
    Engine* engine;
    SolveSettings settings;
    int n_state, n_photo;
  };
  void loop();
  size_t batch_bytes(const Mech& m, int n) const;
  void start(std::unique_ptr<Batch> b, int slot);
  void finish(Batch& b);

  int device_ = 0;
  void* d_base_ = nullptr;
  void* h_base_ = nullptr;
  size_t device_bytes_ = 0, host_bytes_ = 0;
  Arena dev_, host_;
  std::vector<Mech> mechs_;
  std::vector<Slot> slots_;
  std::map<long, std::unique_ptr<Req>> requests_;
  std::map<long, Column> columns_;
  long next_column_ = 0;
  int max_batch_cells_ = 16384;
  std::deque<long> queue_;
  long next_id_ = 0;
  bool stop_ = false;
  std::mutex mu_;
  std::condition_variable cv_;
  std::thread worker_;
};

}  // namespace campb
