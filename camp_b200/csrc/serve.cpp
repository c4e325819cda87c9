// Serving loop: column solves of different sizes, mechanisms and time steps
// submitted as they arrive and solved with continuous batching.
//
// A request is one column (a set of cells) of one mechanism over one host
// time step.  A dispatcher thread turns the queue into batches: whenever a
// slot (a CUDA stream with its own kernel scratch) is free, the oldest
// request and every later queued request of the same mechanism that fits the
// device and pinned-host budgets are merged into one launch whose cells each
// carry their own (t0, t1).  The persistent kernel's warps take the cells of
// all merged requests from one counter, so a long (stiff) cell of one request
// does not leave the warps of that launch idle while other requests wait;
// batches on different slots run concurrently, the next one filling the SMs
// the previous one's tail leaves free.  Completion is detected per batch with
// an event; results are copied back into the callers' arrays and memory is
// returned to the budgets.  Each cell's integration is independent of which
// request, batch, slot or SM runs it, so a result is the same alone and in
// the mix.
//
// A device-resident column keeps its concentrations in the device budget
// between its host steps: a step copies them into the batch and back with
// device-to-device copies, so only the step's env and host-set rates cross
// PCIe.  A column's steps run in submission order, one at a time; other
// requests pass a column whose previous step is still running.
#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <algorithm>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "engine.hpp"
#include "serve.hpp"

namespace campb {

namespace {
double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}
size_t align256(size_t b) { return (b + 255) & ~size_t(255); }
}  // namespace

struct Server::Req {
  long id = 0;
  int mech = 0;
  long column = -1;         // device-resident column, or -1 (caller's state)
  double* state = nullptr;  // caller's arrays
  const double* env = nullptr;
  const double* photo = nullptr;
  int n = 0;
  double t0 = 0, t1 = 0;
  double t_submit = 0, t_start = 0, t_done = 0;
  bool done = false;
  int rc = 0;  // 0 every cell ok, 1 some cell failed, -1 error
  std::string err;
  std::vector<CellStats> stats;
};

// Requests of one mechanism merged into one launch: their cells are laid out
// back to back (same offsets on the device and in pinned host memory), each
// with its own (t0, t1), so the kernel's warps share the cells of every
// request in the batch.
struct Server::Batch {
  int mech = 0;
  std::vector<long> reqs;
  std::vector<int> first;  // first cell of each request
  int n = 0;
  char *d_buf = nullptr, *h_buf = nullptr;
  size_t off_env = 0, off_photo = 0, off_tspan = 0, off_stats = 0, off_flag = 0, bytes = 0;
};

struct Server::Slot {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  char* scratch = nullptr;
  size_t scratch_bytes = 0;
  std::unique_ptr<Batch> batch;
};

Server::Server() {}

bool Server::init(int n_slots, size_t device_bytes, size_t host_bytes, std::string* err) {
  if (n_slots < 1 || n_slots > 64) {
    *err = "n_slots must be in 1..64";
    return false;
  }
  if (cudaGetDevice(&device_) != cudaSuccess) {
    *err = "no CUDA device";
    return false;
  }
  if (cudaMalloc(&d_base_, device_bytes) != cudaSuccess) {
    *err = "device budget allocation failed";
    return false;
  }
  if (cudaHostAlloc(&h_base_, host_bytes, cudaHostAllocDefault) != cudaSuccess) {
    *err = "pinned host budget allocation failed";
    return false;
  }
  dev_.reset((char*)d_base_, device_bytes);
  host_.reset((char*)h_base_, host_bytes);
  device_bytes_ = device_bytes;
  host_bytes_ = host_bytes;
  slots_.resize(n_slots);
  for (auto& s : slots_) {
    if (cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming) != cudaSuccess) {
      *err = "stream or event creation failed";
      return false;
    }
  }
  worker_ = std::thread([this] { loop(); });
  return true;
}

Server::~Server() {
  {
    std::lock_guard<std::mutex> lk(mu_);
    stop_ = true;
  }
  cv_.notify_all();
  if (worker_.joinable()) worker_.join();
  for (auto& s : slots_) {
    if (s.stream) cudaStreamSynchronize(s.stream);
    if (s.stream) cudaStreamDestroy(s.stream);
    if (s.done) cudaEventDestroy(s.done);
    if (s.scratch) cudaFree(s.scratch);
  }
  if (d_base_) cudaFree(d_base_);
  if (h_base_) cudaFreeHost(h_base_);
}

int Server::add_mechanism(Engine* engine, const SolveSettings& settings, int n_state,
                          int n_photo, std::string* err) {
  std::lock_guard<std::mutex> lk(mu_);
  if (!requests_.empty()) {
    *err = "mechanisms must be added before the first request";
    return -1;
  }
  Mech m{engine, settings, n_state, n_photo};
  mechs_.push_back(m);
  // every slot can run any mechanism: size its scratch for the largest
  const int blocks = engine->sm_count();
  const size_t need = engine->slot_scratch_bytes(settings, blocks);
  for (auto& s : slots_) {
    if (need <= s.scratch_bytes) continue;
    if (s.scratch) cudaFree(s.scratch);
    s.scratch = nullptr;
    if (cudaMalloc(&s.scratch, need) != cudaSuccess) {
      *err = "slot scratch allocation failed";
      return -1;
    }
    s.scratch_bytes = need;
  }
  return (int)mechs_.size() - 1;
}

long Server::submit(int mech, double* state, const double* env, const double* photo, int n,
                    double t0, double t1, std::string* err) {
  std::lock_guard<std::mutex> lk(mu_);
  if (mech < 0 || mech >= (int)mechs_.size() || n <= 0 || !state || !env) {
    *err = "invalid request";
    return -1;
  }
  const Mech& m = mechs_[mech];
  if (m.n_photo > 0 && !photo) {
    *err = "the mechanism has photolysis reactions: photolysis rates are required";
    return -1;
  }
  auto r = std::make_unique<Req>();
  r->id = next_id_++;
  r->mech = mech;
  r->state = state;
  r->env = env;
  r->photo = photo;
  r->n = n;
  r->t0 = t0;
  r->t1 = t1;
  r->t_submit = now_s();
  if (batch_bytes(m, n) > device_bytes_ || batch_bytes(m, n) > host_bytes_) {
    *err = "request larger than the memory budget";
    return -1;
  }
  const long id = r->id;
  queue_.push_back(id);
  requests_[id] = std::move(r);
  cv_.notify_all();
  return id;
}

size_t Server::batch_bytes(const Mech& m, int n) const {
  size_t off = align256(sizeof(double) * (size_t)n * m.n_state);
  off += align256(sizeof(double) * 2 * (size_t)n);                // env
  off += align256(sizeof(double) * (size_t)n * m.n_photo);        // photolysis
  off += align256(sizeof(double) * 2 * (size_t)n);                // (t0, t1)
  off += align256(sizeof(CellStats) * (size_t)n);                 // stats
  return off + 256;                                               // error flag
}

void Server::loop() {
  cudaSetDevice(device_);
  std::unique_lock<std::mutex> lk(mu_);
  while (!stop_) {
    bool progress = false;
    // completions
    for (auto& s : slots_) {
      if (!s.batch) continue;
      if (cudaEventQuery(s.done) != cudaSuccess) continue;
      finish(*s.batch);
      s.batch.reset();
      progress = true;
    }
    // admissions: the oldest admissible request (a column's step waits for
    // its previous one) and every later admissible queued request of its
    // mechanism (up to max_batch_cells_) form the next batch
    while (!queue_.empty()) {
      int free_slot = -1;
      for (size_t k = 0; k < slots_.size(); ++k)
        if (!slots_[k].batch) {
          free_slot = (int)k;
          break;
        }
      if (free_slot < 0) break;
      std::vector<long> take, cols;
      int cells = 0, mech = -1;
      for (long id : queue_) {
        const Req& r = *requests_[id];
        if (mech >= 0 && r.mech != mech) continue;
        if (r.column >= 0 && (columns_[r.column].running ||
                              std::find(cols.begin(), cols.end(), r.column) != cols.end())) {
          // a later step of a column waits behind its earlier one
          if (std::find(cols.begin(), cols.end(), r.column) == cols.end())
            cols.push_back(r.column);
          continue;
        }
        if (!take.empty() && cells + r.n > max_batch_cells_) break;
        mech = r.mech;
        take.push_back(id);
        cells += r.n;
        if (r.column >= 0) cols.push_back(r.column);
      }
      if (take.empty()) break;
      // shrink the batch until its buffers fit what the budgets have free
      char *d = nullptr, *h = nullptr;
      size_t bytes = 0;
      while (!take.empty()) {
        bytes = batch_bytes(mechs_[mech], cells);
        d = dev_.alloc(bytes);
        h = d ? host_.alloc(bytes) : nullptr;
        if (d && h) break;
        dev_.release(d);
        d = nullptr;
        if (take.size() == 1) {
          take.clear();
          break;
        }
        const size_t keep = take.size() / 2;
        for (size_t k = keep; k < take.size(); ++k) cells -= requests_[take[k]]->n;
        take.resize(keep);
      }
      if (take.empty()) break;  // the head waits until memory frees up
      for (long id : take)
        if (requests_[id]->column >= 0) columns_[requests_[id]->column].running = true;
      auto b = std::make_unique<Batch>();
      b->mech = mech;
      b->reqs = take;
      b->n = cells;
      b->d_buf = d;
      b->h_buf = h;
      b->bytes = bytes;
      for (long id : take) queue_.erase(std::find(queue_.begin(), queue_.end(), id));
      start(std::move(b), free_slot);
      progress = true;
    }
    if (progress) cv_.notify_all();
    bool busy = false;
    for (auto& s : slots_) busy |= (bool)s.batch;
    if (busy)
      cv_.wait_for(lk, std::chrono::microseconds(50));
    else
      cv_.wait(lk, [this] { return stop_ || !queue_.empty(); });
  }
}

void Server::start(std::unique_ptr<Batch> bp, int slot) {
  Slot& s = slots_[slot];
  Batch& b = *bp;
  const Mech& m = mechs_[b.mech];
  const int n = b.n;
  const size_t sb = align256(sizeof(double) * (size_t)n * m.n_state);
  b.off_env = sb;
  b.off_photo = b.off_env + align256(sizeof(double) * 2 * (size_t)n);
  b.off_tspan = b.off_photo + align256(sizeof(double) * (size_t)n * m.n_photo);
  b.off_stats = b.off_tspan + align256(sizeof(double) * 2 * (size_t)n);
  b.off_flag = b.off_stats + align256(sizeof(CellStats) * (size_t)n);
  const double now = now_s();
  int c0 = 0;
  for (long id : b.reqs) {
    Req& r = *requests_[id];
    r.t_start = now;
    b.first.push_back(c0);
    if (r.column < 0)
      std::memcpy(b.h_buf + sizeof(double) * (size_t)c0 * m.n_state, r.state,
                  sizeof(double) * (size_t)r.n * m.n_state);
    std::memcpy(b.h_buf + b.off_env + sizeof(double) * 2 * (size_t)c0, r.env,
                sizeof(double) * 2 * (size_t)r.n);
    if (m.n_photo > 0)
      std::memcpy(b.h_buf + b.off_photo + sizeof(double) * (size_t)c0 * m.n_photo, r.photo,
                  sizeof(double) * (size_t)r.n * m.n_photo);
    double* ts = (double*)(b.h_buf + b.off_tspan) + 2 * (size_t)c0;
    for (int c = 0; c < r.n; ++c) {
      ts[2 * c] = r.t0;
      ts[2 * c + 1] = r.t1;
    }
    c0 += r.n;
  }
  std::string err;
  bool ok = cudaMemcpyAsync(b.d_buf, b.h_buf, b.off_stats, cudaMemcpyHostToDevice, s.stream) ==
            cudaSuccess;
  // resident columns: their concentrations from the device, after the host
  // range above (stream order)
  for (size_t k = 0; k < b.reqs.size() && ok; ++k) {
    const Req& r = *requests_[b.reqs[k]];
    if (r.column < 0) continue;
    ok = cudaMemcpyAsync(b.d_buf + sizeof(double) * (size_t)b.first[k] * m.n_state,
                         columns_[r.column].d_state, sizeof(double) * (size_t)r.n * m.n_state,
                         cudaMemcpyDeviceToDevice, s.stream) == cudaSuccess;
  }
  ok = ok && m.engine->launch_solve_slot(
                 (double*)b.d_buf, (const double*)(b.d_buf + b.off_env),
                 (const double*)(b.d_buf + b.off_photo), (CellStats*)(b.d_buf + b.off_stats),
                 (const double*)(b.d_buf + b.off_tspan), n, m.settings, s.scratch,
                 s.scratch_bytes, m.engine->sm_count(), s.stream, &err);
  // results: a caller's column back to the host, a resident column back to
  // its device memory
  for (size_t k = 0; k < b.reqs.size() && ok; ++k) {
    const Req& r = *requests_[b.reqs[k]];
    const size_t off = sizeof(double) * (size_t)b.first[k] * m.n_state;
    const size_t len = sizeof(double) * (size_t)r.n * m.n_state;
    ok = (r.column < 0 ? cudaMemcpyAsync(b.h_buf + off, b.d_buf + off, len,
                                         cudaMemcpyDeviceToHost, s.stream)
                       : cudaMemcpyAsync(columns_[r.column].d_state, b.d_buf + off, len,
                                         cudaMemcpyDeviceToDevice, s.stream)) == cudaSuccess;
  }
  ok = ok && cudaMemcpyAsync(b.h_buf + b.off_stats, b.d_buf + b.off_stats,
                             sizeof(CellStats) * (size_t)n, cudaMemcpyDeviceToHost,
                             s.stream) == cudaSuccess;
  ok = ok && cudaMemcpyAsync(b.h_buf + b.off_flag, s.scratch + sizeof(int), sizeof(int),
                             cudaMemcpyDeviceToHost, s.stream) == cudaSuccess;
  if (!ok && err.empty()) err = "copy failed";
  cudaEventRecord(s.done, s.stream);
  if (!ok)
    for (long id : b.reqs) {
      requests_[id]->rc = -1;
      requests_[id]->err = err;
    }
  s.batch = std::move(bp);
}

void Server::finish(Batch& b) {
  const Mech& m = mechs_[b.mech];
  int flag = 0;
  std::memcpy(&flag, b.h_buf + b.off_flag, sizeof(int));
  const double now = now_s();
  for (size_t k = 0; k < b.reqs.size(); ++k) {
    Req& r = *requests_[b.reqs[k]];
    const int c0 = b.first[k];
    if (r.rc == 0 && flag) {
      r.rc = -1;
      r.err = "solve kernel: the table stage into shared memory did not complete";
    }
    if (r.rc == 0) {
      r.stats.resize(r.n);
      std::memcpy(r.stats.data(), b.h_buf + b.off_stats + sizeof(CellStats) * (size_t)c0,
                  sizeof(CellStats) * (size_t)r.n);
      if (r.column < 0)
        std::memcpy(r.state, b.h_buf + sizeof(double) * (size_t)c0 * m.n_state,
                    sizeof(double) * (size_t)r.n * m.n_state);
      for (const auto& c : r.stats)
        if (c.status != 0) r.rc = 1;
    }
    if (r.column >= 0) {
      Column& col = columns_[r.column];
      col.running = false;
      --col.queued;
    }
    r.t_done = now;
    r.done = true;
  }
  dev_.release(b.d_buf);
  host_.release(b.h_buf);
}

int Server::wait(long id, double* latency_ms, std::vector<CellStats>* stats, std::string* err) {
  std::unique_lock<std::mutex> lk(mu_);
  auto it = requests_.find(id);
  if (it == requests_.end()) {
    *err = "unknown request id";
    return -1;
  }
  cv_.wait(lk, [&] { return it->second->done; });
  Req& r = *it->second;
  if (latency_ms) *latency_ms = 1e3 * (r.t_done - r.t_submit);
  if (stats) *stats = r.stats;
  const int rc = r.rc;
  if (rc < 0) *err = r.err;
  requests_.erase(it);
  return rc;
}

int Server::pending() {
  std::lock_guard<std::mutex> lk(mu_);
  return (int)requests_.size();
}

long Server::open_column(int mech, const double* state, int n, std::string* err) {
  std::lock_guard<std::mutex> lk(mu_);
  if (mech < 0 || mech >= (int)mechs_.size() || n <= 0 || !state) {
    *err = "invalid column";
    return -1;
  }
  const size_t bytes = sizeof(double) * (size_t)n * mechs_[mech].n_state;
  char* d = dev_.alloc(bytes);
  if (!d) {
    *err = "the device budget has no room for the column";
    return -1;
  }
  if (cudaMemcpy(d, state, bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
    dev_.release(d);
    *err = "column copy to the device failed";
    return -1;
  }
  Column c;
  c.mech = mech;
  c.n = n;
  c.d_state = d;
  const long id = next_column_++;
  columns_[id] = c;
  return id;
}

long Server::submit_column(long column, const double* env, const double* photo, double t0,
                           double t1, std::string* err) {
  std::lock_guard<std::mutex> lk(mu_);
  auto it = columns_.find(column);
  if (it == columns_.end() || !env) {
    *err = "unknown column or no env";
    return -1;
  }
  const Mech& m = mechs_[it->second.mech];
  if (m.n_photo > 0 && !photo) {
    *err = "the mechanism has host-set rates: they are required";
    return -1;
  }
  auto r = std::make_unique<Req>();
  r->id = next_id_++;
  r->mech = it->second.mech;
  r->column = column;
  r->env = env;
  r->photo = photo;
  r->n = it->second.n;
  r->t0 = t0;
  r->t1 = t1;
  r->t_submit = now_s();
  ++it->second.queued;
  const long id = r->id;
  queue_.push_back(id);
  requests_[id] = std::move(r);
  cv_.notify_all();
  return id;
}

bool Server::column_idle(long column) {
  auto it = columns_.find(column);
  return it == columns_.end() || it->second.queued == 0;
}

int Server::read_column(long column, double* state, std::string* err) {
  std::unique_lock<std::mutex> lk(mu_);
  if (!columns_.count(column) || !state) {
    *err = "unknown column";
    return -1;
  }
  cv_.wait(lk, [&] { return column_idle(column); });
  const Column& c = columns_[column];
  if (cudaMemcpy(state, c.d_state, sizeof(double) * (size_t)c.n * mechs_[c.mech].n_state,
                 cudaMemcpyDeviceToHost) != cudaSuccess) {
    *err = "column copy from the device failed";
    return -1;
  }
  return 0;
}

int Server::close_column(long column, std::string* err) {
  std::unique_lock<std::mutex> lk(mu_);
  if (!columns_.count(column)) {
    *err = "unknown column";
    return -1;
  }
  cv_.wait(lk, [&] { return column_idle(column); });
  dev_.release(columns_[column].d_state);
  columns_.erase(column);
  return 0;
}

}  // namespace campb
