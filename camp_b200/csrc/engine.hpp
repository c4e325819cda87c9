// Device engine: mechanism tables in device memory and the launches of the
// per-cell solve and evaluation kernels.
#pragma once

#include <atomic>

#include <cstdint>
#include <string>
#include <vector>

#include "model.hpp"

namespace campb {

struct CellStats {
  int status;
  int nst, nfe, nsetups, netf, nni, ncfn, nje;
  double hu, hcur;
};

struct SolveSettings {
  double rtol = 1e-4;
  int max_steps = 10000;
  int max_conv_fails = 1000;
  int precision = 0;       // 0 = FP64, 1 = mixed
  int warps_per_block = 0; // 0 = as many as fit
  int blocks_per_sm = 1;
  int lu_mode = 0;         // 0 = level schedule over the warp, 1 = one lane
  int kernel = 0;          // 0 = warp per cell, 1 = lane per cell, 2 = block per cell
  int lane_place = 7;      // lane kernel: bit0 y, bit1 LU, bit2 z in shared memory
  int use_graph = 0;       // warp kernel: launch the device step as a CUDA graph
  int hist_global = 0;     // warp kernel: Nordsieck history + rate constants in
                           // global memory (1) or shared memory (0)
};

class Engine {
 public:
  Engine();
  ~Engine();
  // Uploads the tables of a built model and the absolute tolerances of the
  // dependent variables; sizes per-cell buffers for `capacity` cells.
  bool init(const Model& model, const std::vector<double>& atol_dep, int capacity,
            std::string* err);
  // Launches the solve of n_cells cells whose state/env live on the device.
  // photo (device, [n_cells * n_photo]) may be null when there is no
  // photolysis.  order (device, n_cells) may be null for identity order.
  bool launch_solve(double* d_state, const double* d_env, const double* d_photo,
                    const int* d_order, int n_cells, double t0, double t1,
                    const SolveSettings& s, void* stream, std::string* err);
  // The same solve without any device allocation: its scratch lives in a
  // fixed static device array (solve.cu), per-cell stats go to the caller's
  // d_stats, the Nordsieck history stays in shared memory.  Waits for the
  // stream; false with a message on a usage error, on a scratch need above
  // the static size, or on a kernel error.
  bool run_solve_static(double* d_state, const double* d_env, const double* d_photo,
                        CellStats* d_stats, int n_cells, double t0, double t1,
                        const SolveSettings& s, void* stream, std::string* err);
  // Copies per-cell stats of the last launch to the host (synchronising).
  bool fetch_stats(std::vector<CellStats>* out, int n_cells, void* stream,
                   std::string* err);
  bool eval_deriv(const double* h_state, const double* h_env, const double* h_photo,
                  int n_cells, double h, double* r_p, double* r_l, double* f,
                  std::string* err);
  bool eval_jac(const double* h_state, const double* h_env, const double* h_photo,
                int n_cells, double h, double* jp, double* jl, std::string* err);
  // Finite-difference audit of the analytic Jacobian (debug tool): per cell,
  // elements that fail at every step size and the worst best-step relative
  // difference (-1: f or J could not be evaluated at this state).
  // Precision audit: per cell, the error-weighted RMS difference between the
  // FP32 and the FP64 solve of M = I - h J for a tolerance-sized right-hand
  // side, relative to the FP64 solution's (-1 where f / J or a factorization
  // fails at the state)
  bool check_precision(const double* h_state, const double* h_env, const double* h_photo,
                       int n_cells, double h, double rtol, double* rel_err, std::string* err);
  bool check_jac(const double* h_state, const double* h_env, const double* h_photo,
                 int n_cells, double h, double rel_tol, double abs_tol, double* worst,
                 int* nfail, std::string* err);

  double* d_state_buf(int n_cells, std::string* err);
  double* d_env_buf(int n_cells, std::string* err);
  double* d_photo_buf(int n_cells, std::string* err);
  int* d_order_buf(int n_cells, std::string* err);
  bool sync(void* stream, std::string* err);
  // cells (warps) per block that fit the shared memory for these settings
  int max_cells_per_block(const SolveSettings& s) const;
  // false (with the reason) when the mechanism exceeds the warp-per-cell
  // tables, so that only the lane-per-cell kernel can run it
  bool warp_tables(std::string* err) const;
  // the lane-per-cell kernel's tables were built (it runs this mechanism)
  bool lane_tables() const;
  // the CTA-per-cell kernel's tables were built (it runs this mechanism)
  bool block_tables() const;
  // the kernel a launch with these settings runs (kernel 0 on a mechanism
  // beyond the warp tables: the CTA form where it has its tables, else the
  // lane form)
  int effective_kernel(const SolveSettings& s) const;
  // Serving slots: a launch on caller-provided buffers and scratch (from
  // slot_scratch_bytes for at most max_blocks blocks), so several launches
  // can be in flight on different streams; d_tspan holds each cell's
  // (t0, t1).  No allocation, no sync.
  size_t slot_scratch_bytes(const SolveSettings& s, int max_blocks) const;
  bool launch_solve_slot(double* d_state, const double* d_env, const double* d_photo,
                         CellStats* d_stats, const double* d_tspan, int n_cells,
                         const SolveSettings& s, char* scratch, size_t scratch_bytes,
                         int max_blocks, void* stream, std::string* err);
  int sm_count() const;
  long launches() const { return launches_; }
  double last_kernel_ms() const { return last_ms_; }
  bool read_last_ms(void* stream);

 private:
  bool ensure(void** p, size_t* cap, size_t bytes, std::string* err);
  bool launch_block(double* d_state, const double* d_env, const double* d_photo,
                    const int* d_order, int n_cells, double t0, double t1,
                    const SolveSettings& s, void* stream, std::string* err);
  bool launch_graph(struct SolveArgs& a, const struct WarpLaunch& w, int precision,
                    void* stream, std::string* err);
  void fill_args(struct SolveArgs* a, const struct WarpLaunch& w, const SolveSettings& s,
                 double* d_state, const double* d_env, const double* d_photo,
                 const int* d_order, int n_cells, double t0, double t1) const;
  struct Impl;
  Impl* impl_;
  std::atomic<long> launches_{0};
  double last_ms_ = 0.0;
};

}  // namespace campb
