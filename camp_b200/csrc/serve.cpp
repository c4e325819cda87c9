// Serving loop: column solves of different sizes, mechanisms and time steps
// submitted as they arrive and solved with continuous batching.
//
// A request is one column (a set of cells) of one mechanism over one host
// time step.  A dispatcher thread admits queued requests in arrival order as
// soon as a slot (a CUDA stream with its own kernel scratch) is free and the
// request's buffers fit the device and pinned-host budgets; admitted requests
// run concurrently, each kernel spreading over as many SMs as its cells fill,
// so a request that arrives while others are on the GPU starts on the SMs
// they leave free.  Completion is detected per request with an event; the
// results are copied back into the caller's arrays and the memory returned to
// the budgets.  Each cell's integration is independent of which request,
// slot or SM runs it, so a result is the same alone and in the mix.
#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
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
  double* state = nullptr;  // caller's arrays
  const double* env = nullptr;
  const double* photo = nullptr;
  int n = 0;
  double t0 = 0, t1 = 0;
  double t_submit = 0, t_start = 0, t_done = 0;
  int slot = -1;
  char *d_buf = nullptr, *h_buf = nullptr;
  size_t off_env = 0, off_photo = 0, off_stats = 0, off_flag = 0;
  bool done = false;
  int rc = 0;  // 0 every cell ok, 1 some cell failed, -1 error
  std::string err;
  std::vector<CellStats> stats;
};

struct Server::Slot {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  char* scratch = nullptr;
  size_t scratch_bytes = 0;
  long req = -1;
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
  // buffer layout (same offsets on the device and in pinned host memory)
  size_t off = align256(sizeof(double) * (size_t)n * m.n_state);
  r->off_env = off;
  off += align256(sizeof(double) * 2 * (size_t)n);
  r->off_photo = off;
  off += align256(sizeof(double) * (size_t)n * m.n_photo);
  r->off_stats = off;
  off += align256(sizeof(CellStats) * (size_t)n);
  r->off_flag = off;  // the kernel's error flag, read back into pinned memory
  off += 256;
  if (off > device_bytes_ || off > host_bytes_) {
    *err = "request larger than the memory budget";
    return -1;
  }
  bytes_[r->id] = off;
  const long id = r->id;
  queue_.push_back(id);
  requests_[id] = std::move(r);
  cv_.notify_all();
  return id;
}

void Server::loop() {
  cudaSetDevice(device_);
  std::unique_lock<std::mutex> lk(mu_);
  while (!stop_) {
    bool progress = false;
    // completions
    for (size_t k = 0; k < slots_.size(); ++k) {
      Slot& s = slots_[k];
      if (s.req < 0) continue;
      if (cudaEventQuery(s.done) != cudaSuccess) continue;
      finish(*requests_[s.req]);
      s.req = -1;
      progress = true;
    }
    // admissions in arrival order; the head waits until it fits
    while (!queue_.empty()) {
      int free_slot = -1;
      for (size_t k = 0; k < slots_.size(); ++k)
        if (slots_[k].req < 0) {
          free_slot = (int)k;
          break;
        }
      if (free_slot < 0) break;
      Req& r = *requests_[queue_.front()];
      const size_t bytes = bytes_[r.id];
      char* d = dev_.alloc(bytes);
      char* h = d ? host_.alloc(bytes) : nullptr;
      if (!d || !h) {
        dev_.release(d);
        break;
      }
      queue_.pop_front();
      r.d_buf = d;
      r.h_buf = h;
      start(r, free_slot);
      progress = true;
    }
    if (progress) cv_.notify_all();
    bool busy = false;
    for (auto& s : slots_) busy |= s.req >= 0;
    if (busy)
      cv_.wait_for(lk, std::chrono::microseconds(50));
    else
      cv_.wait(lk, [this] { return stop_ || !queue_.empty(); });
  }
}

void Server::start(Req& r, int slot) {
  Slot& s = slots_[slot];
  const Mech& m = mechs_[r.mech];
  r.slot = slot;
  r.t_start = now_s();
  const size_t sb = sizeof(double) * (size_t)r.n * m.n_state;
  std::memcpy(r.h_buf, r.state, sb);
  std::memcpy(r.h_buf + r.off_env, r.env, sizeof(double) * 2 * (size_t)r.n);
  if (m.n_photo > 0)
    std::memcpy(r.h_buf + r.off_photo, r.photo, sizeof(double) * (size_t)r.n * m.n_photo);
  const size_t in_bytes = r.off_stats;
  std::string err;
  bool ok = cudaMemcpyAsync(r.d_buf, r.h_buf, in_bytes, cudaMemcpyHostToDevice, s.stream) ==
            cudaSuccess;
  ok = ok && m.engine->launch_solve_slot(
                 (double*)r.d_buf, (const double*)(r.d_buf + r.off_env),
                 (const double*)(r.d_buf + r.off_photo), (CellStats*)(r.d_buf + r.off_stats),
                 r.n, r.t0, r.t1, m.settings, s.scratch, s.scratch_bytes,
                 m.engine->sm_count(), s.stream, &err);
  ok = ok && cudaMemcpyAsync(r.h_buf, r.d_buf, sb, cudaMemcpyDeviceToHost, s.stream) ==
                 cudaSuccess;
  ok = ok && cudaMemcpyAsync(r.h_buf + r.off_stats, r.d_buf + r.off_stats,
                             sizeof(CellStats) * (size_t)r.n, cudaMemcpyDeviceToHost,
                             s.stream) == cudaSuccess;
  ok = ok && cudaMemcpyAsync(r.h_buf + r.off_flag, s.scratch + sizeof(int), sizeof(int),
                             cudaMemcpyDeviceToHost, s.stream) == cudaSuccess;
  if (!ok && err.empty()) err = "copy failed";
  cudaEventRecord(s.done, s.stream);
  s.req = r.id;
  if (!ok) {
    r.rc = -1;
    r.err = err;
  }
}

void Server::finish(Req& r) {
  const Mech& m = mechs_[r.mech];
  int flag = 0;
  std::memcpy(&flag, r.h_buf + r.off_flag, sizeof(int));
  if (r.rc == 0 && flag) {
    r.rc = -1;
    r.err = "solve kernel: the table stage into shared memory did not complete";
  }
  if (r.rc == 0) {
    r.stats.resize(r.n);
    std::memcpy(r.stats.data(), r.h_buf + r.off_stats, sizeof(CellStats) * (size_t)r.n);
    std::memcpy(r.state, r.h_buf, sizeof(double) * (size_t)r.n * m.n_state);
    for (const auto& c : r.stats)
      if (c.status != 0) r.rc = 1;
  }
  dev_.release(r.d_buf);
  host_.release(r.h_buf);
  r.d_buf = r.h_buf = nullptr;
  r.t_done = now_s();
  r.done = true;
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
  bytes_.erase(id);
  return rc;
}

int Server::pending() {
  std::lock_guard<std::mutex> lk(mu_);
  return (int)requests_.size();
}

}  // namespace campb
