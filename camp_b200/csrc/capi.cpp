// C ABI of libcamp_b200: the reference's solver entry points plus the
// camp_b200_* extensions (declared in include/camp_b200.h).
#include "../../include/camp_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "blob.hpp"
#include "engine.hpp"
#include "loader.hpp"
#include "model.hpp"
#include "serve.hpp"

using campb::CellStats;
using campb::Engine;
using campb::Model;
using campb::SolveSettings;

namespace {

thread_local std::string g_last_error;

void set_error(const std::string& msg) {
  g_last_error = msg;
  fprintf(stderr, "camp_b200: %s\n", msg.c_str());
}

constexpr double kTiny = 1.0e-60;

struct Solver {
  int n_state = 0, n_cells = 0;
  std::vector<int> var_type;
  int n_rxn = 0;
  std::unique_ptr<Model> model;
  std::unique_ptr<Engine> engine;
  // aerosol phases, representations and sub-models
  int n_aero_phase = 0, n_aero_rep = 0, n_sub_model = 0;
  int n_aero_phase_added = 0, n_aero_rep_added = 0, n_sub_model_added = 0;
  bool add_error = false;
  std::string add_error_msg;
  // per-cell host-set base rates [n_cells * n_photo]: one column per
  // reaction of a host-rate type (PHOTOLYSIS, FIRST_ORDER_LOSS, EMISSION,
  // WET_DEPOSITION) in mechanism order
  std::vector<double> photo;
  int n_photo = 0;
  // device-resident photolysis rates set by camp_b200_set_photo_rates_device
  // (used instead of the host copy while set)
  const double* d_photo_user = nullptr;
  int d_photo_cells = 0;
  SolveSettings settings;
  std::vector<double> atol_dep;
  bool ready = false;
  bool debug_out = false, eval_jac = false;
  cudaStream_t stream = nullptr;
  std::vector<CellStats> stats;
  int last_n = 0;
  bool cost_order = false;
  double tuned_ms = -1.0;  // sample kernel time of the autotuned settings
  std::vector<int> order;
  // state layout and tolerances of a solver created from CAMP JSON files
  std::vector<std::string> state_names;
  std::vector<double> json_abs_tol;
  double json_rel_tol = 0.0;

  int photo_count() const { return model->n_host_rate(); }
  void ensure_photo() {
    int np = photo_count();
    if (np != n_photo || photo.size() != (size_t)np * n_cells) {
      std::vector<double> nw((size_t)np * n_cells, 0.0);
      n_photo = np;
      photo.swap(nw);
    }
  }
};

Solver* S(void* p) { return static_cast<Solver*>(p); }

bool run_common(Solver* s, double* d_state, const double* d_env, int n_cells,
                double t0, double t1, cudaStream_t st, bool sync) {
  std::string err;
  const double* d_photo = nullptr;
  if (s->n_photo > 0 && s->d_photo_user) {
    if (n_cells > s->d_photo_cells) {
      set_error("device photolysis rates cover fewer cells than the run");
      return false;
    }
    d_photo = s->d_photo_user;
  } else if (s->n_photo > 0) {
    double* dp = s->engine->d_photo_buf(n_cells, &err);
    if (!dp) {
      set_error(err);
      return false;
    }
    if (cudaMemcpyAsync(dp, s->photo.data(), sizeof(double) * (size_t)n_cells * s->n_photo,
                        cudaMemcpyHostToDevice, st) != cudaSuccess) {
      set_error("photolysis rate upload failed");
      return false;
    }
    d_photo = dp;
  }
  const int* d_order = nullptr;
  if (s->cost_order && s->last_n == n_cells && (int)s->stats.size() >= n_cells) {
    s->order.resize(n_cells);
    std::iota(s->order.begin(), s->order.end(), 0);
    std::stable_sort(s->order.begin(), s->order.end(), [&](int a, int b) {
      return s->stats[a].nst > s->stats[b].nst;
    });
    int* dor = s->engine->d_order_buf(n_cells, &err);
    if (!dor) {
      set_error(err);
      return false;
    }
    cudaMemcpyAsync(dor, s->order.data(), sizeof(int) * n_cells, cudaMemcpyHostToDevice, st);
    d_order = dor;
  }
  if (!s->engine->launch_solve(d_state, d_env, d_photo, d_order, n_cells, t0, t1,
                               s->settings, st, &err)) {
    set_error(err);
    return false;
  }
  if (sync) {
    if (!s->engine->fetch_stats(&s->stats, n_cells, st, &err)) {
      set_error(err);
      return false;
    }
    s->last_n = n_cells;
  }
  return true;
}

int status_of(Solver* s, int n_cells) {
  for (int c = 0; c < n_cells; ++c)
    if (s->stats[c].status != 0) return 1;
  return 0;
}

}  // namespace

extern "C" {

void* solver_new(int n_state_var, int n_cells, int* var_type, int n_rxn,
                 int n_rxn_int_param, int n_rxn_float_param, int n_rxn_env_param,
                 int n_aero_phase, int n_aero_phase_int_param,
                 int n_aero_phase_float_param, int n_aero_rep,
                 int n_aero_rep_int_param, int n_aero_rep_float_param,
                 int n_aero_rep_env_param, int n_sub_model,
                 int n_sub_model_int_param, int n_sub_model_float_param,
                 int n_sub_model_env_param) {
  (void)n_aero_phase_int_param;
  (void)n_aero_phase_float_param;
  (void)n_aero_rep_int_param;
  (void)n_aero_rep_float_param;
  (void)n_aero_rep_env_param;
  (void)n_sub_model_int_param;
  (void)n_sub_model_float_param;
  (void)n_sub_model_env_param;
  if (n_state_var <= 0 || n_cells <= 0 || !var_type) {
    set_error("solver_new: invalid sizes");
    return nullptr;
  }
  Solver* s = new Solver;
  s->n_state = n_state_var;
  s->n_cells = n_cells;
  s->var_type.assign(var_type, var_type + n_state_var);
  s->n_rxn = n_rxn;
  s->n_aero_phase = n_aero_phase;
  s->n_aero_rep = n_aero_rep;
  s->n_sub_model = n_sub_model;
  s->model.reset(new Model(n_state_var, n_cells, var_type, n_rxn, n_rxn_int_param,
                           n_rxn_float_param, n_rxn_env_param));
  return s;
}

void rxn_add_condensed_data(int rxn_type, int n_int_param, int n_float_param,
                            int n_env_param, int* int_param, double* float_param,
                            void* solver_data) {
  Solver* s = S(solver_data);
  std::string err;
  if (!s->model->add_rxn(rxn_type, n_int_param, n_float_param, n_env_param, int_param,
                         float_param, &err)) {
    s->add_error = true;
    if (s->add_error_msg.empty()) s->add_error_msg = err;
  }
}

void aero_phase_add_condensed_data(int n_int_param, int n_float_param, int* int_param,
                                   double* float_param, void* solver_data) {
  Solver* s = S(solver_data);
  s->n_aero_phase_added++;
  std::string err;
  if (!s->model->add_aero_phase(n_int_param, n_float_param, int_param, float_param, &err) &&
      !s->add_error) {
    s->add_error = true;
    s->add_error_msg = err;
  }
}
void aero_rep_add_condensed_data(int aero_rep_type, int n_int_param, int n_float_param,
                                 int n_env_param, int* int_param, double* float_param,
                                 void* solver_data) {
  Solver* s = S(solver_data);
  s->n_aero_rep_added++;
  std::string err;
  if (!s->model->add_aero_rep(aero_rep_type, n_int_param, n_float_param, n_env_param, int_param,
                              float_param, &err) &&
      !s->add_error) {
    s->add_error = true;
    s->add_error_msg = err;
  }
}
// sub_model_add_condensed_data (src/sub_model_solver.c:425-470): ZSR
// aerosol water and PD-FiTE activity; other types are refused at
// solver_initialize with the reason
void sub_model_add_condensed_data(int sub_model_type, int n_int_param, int n_float_param,
                                  int n_env_param, int* int_param, double* float_param,
                                  void* solver_data) {
  Solver* s = S(solver_data);
  s->n_sub_model_added++;
  std::string err;
  if (!s->model->add_sub_model(sub_model_type, n_int_param, n_float_param, n_env_param,
                               int_param, float_param, &err) &&
      !s->add_error) {
    s->add_error = true;
    s->add_error_msg = err;
  }
}
// GMD / GSD updates of the modal/binned representation
// (src/aero_rep_solver.c:492-545,
// src/aero_reps/aero_rep_modal_binned_mass.c:602-650): the update data is
// {int rep id, int update type (0 GMD, 1 GSD), int section, double value};
// the value becomes the cell's column of that mode.  The search starts at
// *aero_rep_id and leaves it on the representation that took the update.
void aero_rep_update_data(int cell_id, int* aero_rep_id, int update_aero_rep_type,
                          void* update_data, void* solver_data) {
  Solver* s = S(solver_data);
  if (cell_id < 0 || cell_id >= s->n_cells) return;
  const int n_rep = s->model->n_aero_rep();
  if (update_aero_rep_type != campb::AERO_REP_MODAL_BINNED_MASS) {
    *aero_rep_id = n_rep;
    return;
  }
  s->ensure_photo();
  int head[3];
  double value;
  memcpy(head, update_data, sizeof(head));
  memcpy(&value, (char*)update_data + sizeof(head), sizeof(double));
  for (; *aero_rep_id < n_rep; (*aero_rep_id)++) {
    const int col = s->model->aero_column(head[0], head[2], head[1]);
    if (col < 0) continue;
    s->photo[(size_t)cell_id * s->n_photo + col] = value;
    return;
  }
}

namespace {
void* create_aero_update_data(const char* what) {
  void* p = malloc(3 * sizeof(int) + sizeof(double));
  if (!p) {
    set_error(std::string("out of memory allocating ") + what + " update data");
    exit(1);
  }
  return p;
}
void set_aero_update_data(void* update_data, int rep_id, int type, int section, double v) {
  const int head[3] = {rep_id, type, section};
  memcpy(update_data, head, sizeof(head));
  memcpy((char*)update_data + sizeof(head), &v, sizeof(double));
}
}  // namespace

void* aero_rep_modal_binned_mass_create_gmd_update_data(void) {
  return create_aero_update_data("GMD");
}
void aero_rep_modal_binned_mass_set_gmd_update_data(void* update_data, int aero_rep_id,
                                                    int section_id, double gmd) {
  set_aero_update_data(update_data, aero_rep_id, 0, section_id, gmd);
}
void* aero_rep_modal_binned_mass_create_gsd_update_data(void) {
  return create_aero_update_data("GSD");
}
void aero_rep_modal_binned_mass_set_gsd_update_data(void* update_data, int aero_rep_id,
                                                    int section_id, double gsd) {
  set_aero_update_data(update_data, aero_rep_id, 1, section_id, gsd);
}
void sub_model_update_data(int, int*, int, void*, void*) {}

void solver_initialize(void* solver_data, double* abs_tol, double rel_tol, int max_steps,
                       int max_conv_fails) {
  Solver* s = S(solver_data);
  s->ready = false;
  if (s->add_error) {
    set_error("solver_initialize: " + s->add_error_msg);
    return;
  }
  if (s->n_aero_phase_added != s->n_aero_phase || s->n_aero_rep_added != s->n_aero_rep ||
      s->n_sub_model_added != s->n_sub_model) {
    set_error("solver_initialize: fewer aerosol phases, representations or sub-models were "
              "added than declared in solver_new");
    return;
  }
  std::string err;
  s->model->set_abs_tol(abs_tol);
  if (!s->model->build(&err)) {
    set_error("solver_initialize: " + err);
    return;
  }
  s->atol_dep.clear();
  for (int i = 0; i < s->n_state; ++i)
    if (s->var_type[i] == campb::VAR_VARIABLE) s->atol_dep.push_back(abs_tol[i]);
  s->settings.rtol = rel_tol;
  s->settings.max_steps = max_steps;
  s->settings.max_conv_fails = max_conv_fails;
  s->ensure_photo();
  if (!s->stream) {
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
      set_error("solver_initialize: no CUDA device available");
      return;
    }
  }
  s->engine.reset(new Engine);
  if (!s->engine->init(*s->model, s->atol_dep, s->n_cells, &err)) {
    set_error("solver_initialize: " + err);
    return;
  }
  s->ready = true;
}

int solver_run(void* solver_data, double* state, double* env, double t_initial,
               double t_final) {
  Solver* s = S(solver_data);
  if (!s || !s->ready) {
    set_error("solver_run: solver is not initialized");
    return 1;
  }
  const int nc = s->n_cells, ns = s->n_state;
  if (s->n_rxn == 0) {
    // no reactions: the reference skips CVODE and writes back the clamped
    // values (src/camp_solver.c:554-567, 672-683)
    for (int c = 0; c < nc; ++c)
      for (int i = 0; i < ns; ++i) {
        double& v = state[(size_t)c * ns + i];
        if (s->var_type[i] == campb::VAR_VARIABLE || s->var_type[i] == campb::VAR_CONSTANT)
          v = v > kTiny ? v : kTiny;
      }
    return 0;
  }
  std::string err;
  double* ds = s->engine->d_state_buf(nc, &err);
  double* de = ds ? s->engine->d_env_buf(nc, &err) : nullptr;
  if (!ds || !de) {
    set_error("solver_run: " + err);
    return 1;
  }
  cudaStream_t st = s->stream;
  size_t bytes = sizeof(double) * (size_t)nc * ns;
  if (cudaMemcpyAsync(ds, state, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(de, env, sizeof(double) * 2 * nc, cudaMemcpyHostToDevice, st) !=
          cudaSuccess) {
    set_error("solver_run: host to device copy failed");
    return 1;
  }
  if (!run_common(s, ds, de, nc, t_initial, t_final, st, false)) return 1;
  if (cudaMemcpyAsync(state, ds, bytes, cudaMemcpyDeviceToHost, st) != cudaSuccess) {
    set_error("solver_run: device to host copy failed");
    return 1;
  }
  if (!s->engine->fetch_stats(&s->stats, nc, st, &err)) {
    set_error("solver_run: " + err);
    return 1;
  }
  s->last_n = nc;
  return status_of(s, nc);
}

void solver_get_statistics(void* solver_data, int* solver_flag, int* num_steps,
                           int* RHS_evals, int* LS_setups, int* error_test_fails,
                           int* NLS_iters, int* NLS_convergence_fails, int* DLS_Jac_evals,
                           int* DLS_RHS_evals, double* last_time_step__s,
                           double* next_time_step__s, int* Jac_eval_fails,
                           int* RHS_evals_total, int* Jac_evals_total, double* RHS_time__s,
                           double* Jac_time__s, double* max_loss_precision) {
  Solver* s = S(solver_data);
  int flag = 0, nst = 0, nfe = 0, ns = 0, netf = 0, nni = 0, ncf = 0, nje = 0;
  double hu = 0.0, hc = 0.0;
  for (int c = 0; c < s->last_n; ++c) {
    const CellStats& x = s->stats[c];
    if (x.status != 0 && flag == 0) flag = x.status;
    nst = std::max(nst, x.nst);
    nfe = std::max(nfe, x.nfe);
    ns = std::max(ns, x.nsetups);
    netf = std::max(netf, x.netf);
    nni = std::max(nni, x.nni);
    ncf = std::max(ncf, x.ncfn);
    nje = std::max(nje, x.nje);
    if (c == 0 || x.hu < hu) hu = x.hu;
    if (c == 0 || x.hcur < hc) hc = x.hcur;
  }
  *solver_flag = flag;
  *num_steps = nst;
  *RHS_evals = nfe;
  *LS_setups = ns;
  *error_test_fails = netf;
  *NLS_iters = nni;
  *NLS_convergence_fails = ncf;
  *DLS_Jac_evals = nje;
  *DLS_RHS_evals = 0;  // no difference-quotient Jacobian is used
  *last_time_step__s = hu;
  *next_time_step__s = hc;
  *Jac_eval_fails = 0;
  // the reference reports -1/0 for these outside CAMP_DEBUG builds
  *RHS_evals_total = -1;
  *Jac_evals_total = -1;
  *RHS_time__s = 0.0;
  *Jac_time__s = 0.0;
  *max_loss_precision = 0.0;
}

void solver_reset_timers(void* solver_data) { (void)solver_data; }

int solver_set_debug_out(void* solver_data, int do_output) {
  S(solver_data)->debug_out = do_output != 0;
  return 0;
}
int solver_set_eval_jac(void* solver_data, int eval_jac) {
  S(solver_data)->eval_jac = eval_jac != 0;
  return 0;
}

void solver_free(void* solver_data) {
  Solver* s = S(solver_data);
  if (!s) return;
  s->engine.reset();
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

void solver_free_update_data(void* update_data) { free(update_data); }
void rxn_free_update_data(void* update_data) { free(update_data); }

namespace {
// Update data of the host-rate types: an int reaction id followed, unaligned,
// by the double base rate (src/rxns/rxn_photolysis.c:262-283,
// rxn_emission.c:192-213, rxn_first_order_loss.c:208-229,
// rxn_wet_deposition.c:218-239).
void* create_rate_update_data(const char* what) {
  void* p = malloc(sizeof(int) + sizeof(double));
  if (!p) {
    set_error(std::string("out of memory allocating ") + what + " update data");
    exit(1);
  }
  return p;
}
void set_rate_update_data(void* update_data, int rxn_id, double base_rate) {
  memcpy(update_data, &rxn_id, sizeof(int));
  memcpy((char*)update_data + sizeof(int), &base_rate, sizeof(double));
}
}  // namespace

void* rxn_photolysis_create_rate_update_data(void) {
  return create_rate_update_data("photolysis");
}
void rxn_photolysis_set_rate_update_data(void* update_data, int photo_id, double base_rate) {
  set_rate_update_data(update_data, photo_id, base_rate);
}
void* rxn_emission_create_rate_update_data(void) { return create_rate_update_data("emission"); }
void rxn_emission_set_rate_update_data(void* update_data, int rxn_id, double base_rate) {
  set_rate_update_data(update_data, rxn_id, base_rate);
}
void* rxn_first_order_loss_create_rate_update_data(void) {
  return create_rate_update_data("first-order loss");
}
void rxn_first_order_loss_set_rate_update_data(void* update_data, int rxn_id,
                                               double base_rate) {
  set_rate_update_data(update_data, rxn_id, base_rate);
}
void* rxn_wet_deposition_create_rate_update_data(void) {
  return create_rate_update_data("wet deposition");
}
void rxn_wet_deposition_set_rate_update_data(void* update_data, int rxn_id, double base_rate) {
  set_rate_update_data(update_data, rxn_id, base_rate);
}

// The reference walks the reactions from *rxn_id and stops at the first one
// of update_rxn_type whose RXN_ID_ matches (> 0), leaving *rxn_id on it
// (src/rxn_solver.c:700-760).  Here the match sets that reaction's column of
// the cell's host-set base rates.
void rxn_update_data(int cell_id, int* rxn_id, int update_rxn_type, void* update_data,
                     void* solver_data) {
  Solver* s = S(solver_data);
  if (cell_id < 0 || cell_id >= s->n_cells) return;
  const auto& rx = s->model->rxns();
  const int n_rxn = (int)rx.size();
  if (!campb::host_rate_type(update_rxn_type)) {
    // condensed-phase photolysis updates have no reaction of that type here
    *rxn_id = n_rxn;
    return;
  }
  s->ensure_photo();
  int id;
  double base;
  memcpy(&id, update_data, sizeof(int));
  memcpy(&base, (char*)update_data + sizeof(int), sizeof(double));
  const auto& slot = s->model->photo_slot();
  for (; *rxn_id < n_rxn; (*rxn_id)++) {
    if (rx[*rxn_id].type != update_rxn_type) continue;
    const int rid = s->model->photo_id(*rxn_id);
    if (id == rid && rid > 0) {
      s->photo[(size_t)cell_id * s->n_photo + slot[*rxn_id]] = base;
      return;
    }
  }
}

void rxn_print_data(void* solver_data) {
  Solver* s = S(solver_data);
  printf("\n\nReaction data\n\nnumber of reactions: %d\n\n", s->n_rxn);
  for (const auto& r : s->model->rxns()) {
    const char* name = "Unknown";
    switch (r.type) {
      case campb::RXN_ARRHENIUS: name = "Arrhenius"; break;
      case campb::RXN_TROE: name = "Troe"; break;
      case campb::RXN_CMAQ_H2O2: name = "CMAQ_H2O2"; break;
      case campb::RXN_CMAQ_OH_HNO3: name = "CMAQ_OH_HNO3"; break;
      case campb::RXN_PHOTOLYSIS: name = "Photolysis"; break;
      case campb::RXN_FIRST_ORDER_LOSS: name = "First-Order loss"; break;
      case campb::RXN_EMISSION: name = "Emission"; break;
      case campb::RXN_WET_DEPOSITION: name = "Wet Deposition"; break;
    }
    printf("\n\n%s reaction\n", name);
  }
  fflush(stdout);
}
void aero_phase_print_data(void* solver_data) {
  printf("\n\nAerosol phase data\n\nnumber of aerosol phases: %d\n\n",
         S(solver_data)->n_aero_phase);
}
void aero_rep_print_data(void* solver_data) {
  printf("\n\nAerosol representation data\n\nnumber of aerosol representations: %d\n\n",
         S(solver_data)->n_aero_rep);
}
void sub_model_print_data(void* solver_data) {
  printf("\n\nSub-model data\n\nnumber of sub-models: %d\n\n", S(solver_data)->n_sub_model);
}

// ----------------------------------------------------------------------------
// extension API
// ----------------------------------------------------------------------------
const char* camp_b200_last_error(void) { return g_last_error.c_str(); }

int camp_b200_is_ready(void* solver_data) { return S(solver_data)->ready ? 1 : 0; }

int camp_b200_set_precision(void* solver_data, int mode) {
  if (mode != CAMP_B200_FP64 && mode != CAMP_B200_MIXED) {
    set_error("camp_b200_set_precision: unknown mode");
    return -1;
  }
  S(solver_data)->settings.precision = mode;
  return 0;
}

int camp_b200_set_launch(void* solver_data, int warps_per_block, int blocks_per_sm) {
  S(solver_data)->settings.warps_per_block = std::max(0, warps_per_block);
  S(solver_data)->settings.blocks_per_sm = std::max(1, blocks_per_sm);
  return 0;
}

int camp_b200_set_lu_mode(void* solver_data, int mode) {
  if (mode != 0 && mode != 1) {
    set_error("camp_b200_set_lu_mode: mode must be 0 or 1");
    return -1;
  }
  S(solver_data)->settings.lu_mode = mode;
  return 0;
}

int camp_b200_set_graph(void* solver_data, int enable) {
  S(solver_data)->settings.use_graph = enable ? 1 : 0;
  return 0;
}

int camp_b200_set_layout(void* solver_data, int hist_global) {
  if (hist_global != 0 && hist_global != 1) {
    set_error("camp_b200_set_layout: hist_global must be 0 or 1");
    return -1;
  }
  S(solver_data)->settings.hist_global = hist_global;
  return 0;
}

int camp_b200_autotune(void* solver_data, const double* state, const double* env, int n_cells,
                       double t_initial, double t_final) {
  Solver* s = S(solver_data);
  if (!s->ready || n_cells <= 0 || n_cells > s->n_cells || !state || !env) {
    set_error("camp_b200_autotune: solver not ready, or sample empty or above capacity");
    return -1;
  }
  std::string err;
  double* ds = s->engine->d_state_buf(n_cells, &err);
  double* de = ds ? s->engine->d_env_buf(n_cells, &err) : nullptr;
  if (!ds || !de) {
    set_error("camp_b200_autotune: " + err);
    return -1;
  }
  cudaStream_t st = s->stream;
  const size_t bytes = sizeof(double) * (size_t)n_cells * s->n_state;
  if (cudaMemcpyAsync(de, env, sizeof(double) * 2 * n_cells, cudaMemcpyHostToDevice, st) !=
      cudaSuccess) {
    set_error("camp_b200_autotune: host to device copy failed");
    return -1;
  }
  // candidates: the warp-per-cell kernel with its resident cells per block,
  // where the Nordsieck history lives and the LU strategy, and the
  // block-per-cell kernel where the mechanism has their tables; the
  // lane-per-cell kernel (32 cells per warp, 14-30x slower than the warp
  // kernel on cb05 and 11x slower than the block kernel on a 200-species
  // mechanism) only where neither has; the precision stays as set
  campb::SolveSettings base = s->settings, best = s->settings;
  double best_ms = -1.0;
  const bool cost_order = s->cost_order;
  s->cost_order = false;
  std::vector<campb::SolveSettings> cands;
  for (int lu = 0; lu <= 1; ++lu)
    for (int hg = 0; hg <= 1; ++hg) {
      campb::SolveSettings c = base;
      c.kernel = 0;
      c.lu_mode = lu;
      c.hist_global = hg;
      const int mx = s->engine->max_cells_per_block(c);
      std::vector<int> ws;
      for (int w : {mx, mx - 1, mx - 2, (2 * mx) / 3, mx / 2, 8, 11})
        if (w >= 2 && w <= mx && std::find(ws.begin(), ws.end(), w) == ws.end()) ws.push_back(w);
      for (int w : ws) {
        c.warps_per_block = w;
        c.blocks_per_sm = 1;
        cands.push_back(c);
      }
    }
  if (s->engine->lane_tables() && cands.empty() && !s->engine->block_tables()) {
    campb::SolveSettings c = base;
    c.kernel = 1;
    cands.push_back(c);
  }
  if (s->engine->block_tables()) {
    campb::SolveSettings c = base;
    c.kernel = 2;
    cands.push_back(c);
  }
  for (const campb::SolveSettings& c : cands) {
    s->settings = c;
    if (cudaMemcpyAsync(ds, state, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        !run_common(s, ds, de, n_cells, t_initial, t_final, st, true)) {
      s->settings = base;
      s->cost_order = cost_order;
      set_error("camp_b200_autotune: trial run failed: " + std::string(camp_b200_last_error()));
      return -1;
    }
    const double ms = s->engine->last_kernel_ms();
    if (best_ms < 0.0 || ms < best_ms) {
      best_ms = ms;
      best = c;
    }
  }
  s->settings = best;
  s->tuned_ms = best_ms;
  s->cost_order = cost_order;
  return 0;
}

int camp_b200_get_tuning(void* solver_data, int* warps_per_block, int* hist_global,
                         int* lu_mode, double* sample_ms) {
  Solver* s = S(solver_data);
  if (warps_per_block) *warps_per_block = s->settings.warps_per_block;
  if (hist_global) *hist_global = s->settings.hist_global;
  if (lu_mode) *lu_mode = s->settings.lu_mode;
  if (sample_ms) *sample_ms = s->tuned_ms;
  return 0;
}

int camp_b200_get_kernel(void* solver_data) {
  const Solver* s = S(solver_data);
  return s->ready ? s->engine->effective_kernel(s->settings) : s->settings.kernel;
}

int camp_b200_set_kernel(void* solver_data, int kernel, int place) {
  if (kernel < 0 || kernel > 2) {
    set_error("camp_b200_set_kernel: kernel must be 0, 1 or 2");
    return -1;
  }
  S(solver_data)->settings.kernel = kernel;
  if (place >= 0) S(solver_data)->settings.lane_place = place & 7;
  return 0;
}

int camp_b200_set_cost_ordering(void* solver_data, int enable) {
  S(solver_data)->cost_order = enable != 0;
  return 0;
}

int camp_b200_run_device(void* solver_data, double* d_state, const double* d_env, int n_cells,
                         double t_initial, double t_final, void* stream) {
  Solver* s = S(solver_data);
  if (!s->ready || n_cells <= 0 || n_cells > s->n_cells) {
    set_error("camp_b200_run_device: solver not ready or n_cells out of range");
    return -1;
  }
  cudaStream_t st = stream ? (cudaStream_t)stream : s->stream;
  if (!run_common(s, d_state, d_env, n_cells, t_initial, t_final, st, true)) return -1;
  return status_of(s, n_cells);
}

static_assert(sizeof(camp_b200_cell_stats) == sizeof(campb::CellStats),
              "camp_b200_cell_stats must mirror the device CellStats");

int camp_b200_run_device_noalloc(void* solver_data, double* d_state, const double* d_env,
                                 const double* d_photo, camp_b200_cell_stats* d_stats,
                                 int n_cells, double t_initial, double t_final, void* stream) {
  Solver* s = S(solver_data);
  if (!s->ready || n_cells <= 0) {
    set_error("camp_b200_run_device_noalloc: solver not ready or n_cells <= 0");
    return -1;
  }
  cudaStream_t st = stream ? (cudaStream_t)stream : s->stream;
  std::string err;
  if (!s->engine->run_solve_static(d_state, d_env, d_photo, (campb::CellStats*)d_stats, n_cells,
                                   t_initial, t_final, s->settings, st, &err)) {
    set_error("camp_b200_run_device_noalloc: " + err);
    return -1;
  }
  return 0;
}

int camp_b200_launch_device(void* solver_data, double* d_state, const double* d_env,
                            int n_cells, double t_initial, double t_final, void* stream) {
  Solver* s = S(solver_data);
  if (!s->ready || n_cells <= 0 || n_cells > s->n_cells) {
    set_error("camp_b200_launch_device: solver not ready or n_cells out of range");
    return -1;
  }
  cudaStream_t st = stream ? (cudaStream_t)stream : s->stream;
  if (!run_common(s, d_state, d_env, n_cells, t_initial, t_final, st, false)) return -1;
  s->last_n = -n_cells;  // pending
  return 0;
}

int camp_b200_sync_status(void* solver_data, void* stream) {
  Solver* s = S(solver_data);
  cudaStream_t st = stream ? (cudaStream_t)stream : s->stream;
  int n = s->last_n < 0 ? -s->last_n : s->last_n;
  std::string err;
  if (!s->engine->fetch_stats(&s->stats, n, st, &err)) {
    set_error(err);
    return -1;
  }
  s->last_n = n;
  return status_of(s, n);
}

int camp_b200_n_photo(void* solver_data) {
  Solver* s = S(solver_data);
  s->ensure_photo();
  return s->n_photo;
}

int camp_b200_rate_column(void* solver_data, int column, int* rxn_index, int* rxn_type,
                          int* rxn_id) {
  Solver* s = S(solver_data);
  if (!s || !s->model) return -1;
  const auto& slot = s->model->photo_slot();
  const auto& rx = s->model->rxns();
  for (int i = 0; i < (int)rx.size(); ++i)
    if (slot[i] == column && column >= 0) {
      if (rxn_index) *rxn_index = i;
      if (rxn_type) *rxn_type = rx[i].type;
      if (rxn_id) *rxn_id = s->model->photo_id(i);
      return 0;
    }
  // the GMD / GSD columns of the modes follow the reaction columns
  const auto& modes = s->model->modes();
  const int first = s->model->n_host_rate() - 2 * (int)modes.size();
  if (column >= first && column < s->model->n_host_rate()) {
    const int k = (column - first) / 2, what = (column - first) % 2;
    if (rxn_index) *rxn_index = -1 - modes[k].first;
    if (rxn_type) *rxn_type = what == 0 ? CAMP_B200_COLUMN_GMD : CAMP_B200_COLUMN_GSD;
    if (rxn_id) *rxn_id = modes[k].second;
    return 0;
  }
  set_error("no host-rate column " + std::to_string(column));
  return -1;
}

int camp_b200_set_photo_rates(void* solver_data, const double* rates, int n_cells) {
  Solver* s = S(solver_data);
  s->ensure_photo();
  if (n_cells < 0 || n_cells > s->n_cells) return -1;
  std::copy(rates, rates + (size_t)n_cells * s->n_photo, s->photo.begin());
  return 0;
}

int camp_b200_set_photo_rates_device(void* solver_data, const double* d_rates, int n_cells) {
  Solver* s = S(solver_data);
  s->ensure_photo();
  if (n_cells < 0) return -1;
  s->d_photo_user = n_cells > 0 ? d_rates : nullptr;
  s->d_photo_cells = d_rates ? n_cells : 0;
  return 0;
}

int camp_b200_get_cell_stats(void* solver_data, camp_b200_cell_stats* out, int n_cells) {
  Solver* s = S(solver_data);
  int n = std::min(n_cells, std::abs(s->last_n));
  for (int c = 0; c < n; ++c) {
    const CellStats& x = s->stats[c];
    out[c].status = x.status;
    out[c].nst = x.nst;
    out[c].nfe = x.nfe;
    out[c].nsetups = x.nsetups;
    out[c].netf = x.netf;
    out[c].nni = x.nni;
    out[c].ncfn = x.ncfn;
    out[c].nje = x.nje;
    out[c].hu = x.hu;
    out[c].hcur = x.hcur;
  }
  for (int c = n; c < n_cells; ++c) {
    memset(&out[c], 0, sizeof(out[c]));
    out[c].status = CAMP_B200_NOT_RUN;
  }
  return n;
}

long camp_b200_kernel_launches(void* solver_data) {
  Solver* s = S(solver_data);
  return s->engine ? s->engine->launches() : 0;
}

double camp_b200_last_kernel_ms(void* solver_data) {
  Solver* s = S(solver_data);
  return s->engine ? s->engine->last_kernel_ms() : 0.0;
}

int camp_b200_n_dep_var(void* solver_data) { return S(solver_data)->model->n_dep(); }
int camp_b200_n_jac_elem(void* solver_data) {
  return (int)S(solver_data)->model->solver_rowid().size();
}
int camp_b200_n_lu_elem(void* solver_data) { return S(solver_data)->model->tables().n_lu; }
int camp_b200_rxn_int_data_size(void* solver_data) {
  return (int)S(solver_data)->model->rxn_int().size();
}
int camp_b200_get_solver_jac(void* solver_data, int* col_ptrs, int* row_ids) {
  const Model& m = *S(solver_data)->model;
  if (!m.built()) return -1;
  std::copy(m.solver_colptr().begin(), m.solver_colptr().end(), col_ptrs);
  std::copy(m.solver_rowid().begin(), m.solver_rowid().end(), row_ids);
  return 0;
}
int camp_b200_get_rxn_int_data(void* solver_data, int* out) {
  const Model& m = *S(solver_data)->model;
  std::copy(m.rxn_int().begin(), m.rxn_int().end(), out);
  return 0;
}
int camp_b200_n_mapped_values(void* solver_data) {
  const Model& m = *S(solver_data)->model;
  return m.built() ? (int)m.jac_map().size() / 3 : -1;
}
int camp_b200_get_jac_map(void* solver_data, int* triplets) {
  const Model& m = *S(solver_data)->model;
  if (!m.built()) return -1;
  std::copy(m.jac_map().begin(), m.jac_map().end(), triplets);
  return 0;
}
long camp_b200_get_block_tables(void* solver_data, void* out, long capacity) {
  const Model& m = *S(solver_data)->model;
  if (!m.built()) {
    set_error("camp_b200_get_block_tables: sparsity not built");
    return -1;
  }
  std::vector<uint8_t> blob;
  campb::BlockOff off{};
  std::string err;
  if (!campb::build_block_blob(m.tables(), std::vector<double>(m.tables().n, 0.0), &blob, &off,
                               &err)) {
    set_error("camp_b200_get_block_tables: " + err);
    return -1;
  }
  if (out && capacity >= (long)blob.size()) memcpy(out, blob.data(), blob.size());
  return (long)blob.size();
}

int camp_b200_get_lu_order(void* solver_data, int* perm) {
  const Model& m = *S(solver_data)->model;
  if (!m.built()) return -1;
  std::copy(m.tables().lu_perm.begin(), m.tables().lu_perm.end(), perm);
  return 0;
}

int camp_b200_eval_deriv(void* solver_data, const double* state, const double* env,
                         int n_cells, double h, double* r_p, double* r_l, double* deriv) {
  Solver* s = S(solver_data);
  if (!s->ready || n_cells <= 0 || n_cells > s->n_cells) return -1;
  std::string err;
  if (!s->engine->eval_deriv(state, env, s->n_photo ? s->photo.data() : nullptr, n_cells, h,
                             r_p, r_l, deriv, &err)) {
    set_error(err);
    return -1;
  }
  return 0;
}

int camp_b200_eval_jac(void* solver_data, const double* state, const double* env, int n_cells,
                       double h, double* j_prod, double* j_loss) {
  Solver* s = S(solver_data);
  if (!s->ready || n_cells <= 0 || n_cells > s->n_cells) return -1;
  std::string err;
  // the device evaluates the live entries; the output has every solver
  // Jacobian entry, the others (HL's element partials) being zero
  const campb::Model& m = *s->model;
  const std::vector<int>& map = m.device_to_solver();
  const size_t nd = map.size(), ns = m.solver_rowid().size();
  const bool same = nd == ns;
  std::vector<double> dp, dl;
  if (!same) {
    dp.resize((size_t)n_cells * nd);
    dl.resize((size_t)n_cells * nd);
  }
  if (!s->engine->eval_jac(state, env, s->n_photo ? s->photo.data() : nullptr, n_cells, h,
                           same ? j_prod : dp.data(), same ? j_loss : dl.data(), &err)) {
    set_error(err);
    return -1;
  }
  if (!same) {
    std::fill(j_prod, j_prod + (size_t)n_cells * ns, 0.0);
    std::fill(j_loss, j_loss + (size_t)n_cells * ns, 0.0);
    for (int c = 0; c < n_cells; ++c)
      for (size_t e = 0; e < nd; ++e) {
        j_prod[(size_t)c * ns + map[e]] = dp[(size_t)c * nd + e];
        j_loss[(size_t)c * ns + map[e]] = dl[(size_t)c * nd + e];
      }
  }
  return 0;
}

int camp_b200_check_precision(void* solver_data, const double* state, const double* env,
                              int n_cells, double h, double* rel_err) {
  Solver* s = S(solver_data);
  if (!s->ready || n_cells <= 0 || n_cells > s->n_cells || !state || !env || !rel_err) {
    set_error("camp_b200_check_precision: solver not ready, bad sizes or missing outputs");
    return -1;
  }
  std::string err;
  if (!s->engine->check_precision(state, env, s->n_photo ? s->photo.data() : nullptr, n_cells,
                                  h, s->settings.rtol, rel_err, &err)) {
    set_error("camp_b200_check_precision: " + err);
    return -1;
  }
  return 0;
}

int camp_b200_check_jac(void* solver_data, const double* state, const double* env, int n_cells,
                        double h, double rel_tol, double abs_tol, double* worst_rel,
                        int* n_failed) {
  Solver* s = S(solver_data);
  if (!s->ready || n_cells <= 0 || n_cells > s->n_cells || !worst_rel || !n_failed) {
    set_error("camp_b200_check_jac: solver not ready, bad sizes or missing outputs");
    return -1;
  }
  s->ensure_photo();
  std::string err;
  if (!s->engine->check_jac(state, env, s->n_photo ? s->photo.data() : nullptr, n_cells, h,
                            rel_tol, abs_tol, worst_rel, n_failed, &err)) {
    set_error(err);
    return -1;
  }
  int total = 0;
  for (int c = 0; c < n_cells; ++c) total += n_failed[c] > 0 ? n_failed[c] : 0;
  return total;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Serving loop
// ---------------------------------------------------------------------------
extern "C" {

void* camp_b200_server_new(int n_slots, double device_mb, double host_mb) {
  auto* sv = new campb::Server;
  std::string err;
  if (!sv->init(n_slots, (size_t)(device_mb * 1048576.0), (size_t)(host_mb * 1048576.0), &err)) {
    set_error("camp_b200_server_new: " + err);
    delete sv;
    return nullptr;
  }
  return sv;
}

int camp_b200_server_add_solver(void* server, void* solver_data) {
  Solver* s = S(solver_data);
  if (!server || !s->ready) {
    set_error("camp_b200_server_add_solver: no server, or the solver is not initialised");
    return -1;
  }
  s->ensure_photo();
  std::string err;
  int id = static_cast<campb::Server*>(server)->add_mechanism(s->engine.get(), s->settings,
                                                              s->n_state, s->n_photo, &err);
  if (id < 0) set_error("camp_b200_server_add_solver: " + err);
  return id;
}

long camp_b200_server_submit(void* server, int mech, double* state, const double* env,
                             const double* photo, int n_cells, double t_initial,
                             double t_final) {
  std::string err;
  long id = static_cast<campb::Server*>(server)->submit(mech, state, env, photo, n_cells,
                                                        t_initial, t_final, &err);
  if (id < 0) set_error("camp_b200_server_submit: " + err);
  return id;
}

int camp_b200_server_wait(void* server, long request, double* latency_ms,
                          camp_b200_cell_stats* stats, int n_cells) {
  std::string err;
  std::vector<campb::CellStats> st;
  int rc = static_cast<campb::Server*>(server)->wait(request, latency_ms, &st, &err);
  if (rc < 0) {
    set_error("camp_b200_server_wait: " + err);
    return rc;
  }
  if (stats)
    for (int c = 0; c < n_cells && c < (int)st.size(); ++c)
      std::memcpy(&stats[c], &st[c], sizeof(camp_b200_cell_stats));
  return rc;
}

int camp_b200_server_pending(void* server) {
  return static_cast<campb::Server*>(server)->pending();
}

void camp_b200_server_free(void* server) { delete static_cast<campb::Server*>(server); }

long camp_b200_server_open_column(void* server, int mech, const double* state, int n_cells) {
  std::string err;
  const long id = static_cast<campb::Server*>(server)->open_column(mech, state, n_cells, &err);
  if (id < 0) set_error("camp_b200_server_open_column: " + err);
  return id;
}

long camp_b200_server_submit_column(void* server, long column, const double* env,
                                    const double* photo, double t_initial, double t_final) {
  std::string err;
  const long id = static_cast<campb::Server*>(server)->submit_column(column, env, photo,
                                                                      t_initial, t_final, &err);
  if (id < 0) set_error("camp_b200_server_submit_column: " + err);
  return id;
}

int camp_b200_server_read_column(void* server, long column, double* state) {
  std::string err;
  const int rc = static_cast<campb::Server*>(server)->read_column(column, state, &err);
  if (rc < 0) set_error("camp_b200_server_read_column: " + err);
  return rc;
}

int camp_b200_server_close_column(void* server, long column) {
  std::string err;
  const int rc = static_cast<campb::Server*>(server)->close_column(column, &err);
  if (rc < 0) set_error("camp_b200_server_close_column: " + err);
  return rc;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// CAMP JSON input without the Fortran camp_core
// ---------------------------------------------------------------------------
extern "C" {

void* camp_b200_solver_from_json(const char* const* files, int n_files, int n_cells) {
  if (!files || n_files <= 0 || n_cells <= 0) {
    set_error("camp_b200_solver_from_json: no files or no cells");
    return nullptr;
  }
  std::vector<std::string> paths;
  for (int k = 0; k < n_files; ++k) paths.emplace_back(files[k] ? files[k] : "");
  campb::LoadedMechanism lm;
  std::string err;
  if (!campb::load_mechanism_json(paths, &lm, &err)) {
    set_error("camp_b200_solver_from_json: " + err);
    return nullptr;
  }
  int ph_i = 0, ph_f = 0, rp_i = 0, rp_f = 0, rp_e = 0;
  for (const auto& p : lm.phases) {
    ph_i += (int)p.ints.size();
    ph_f += (int)p.floats.size();
  }
  for (const auto& r : lm.reps) {
    rp_i += (int)r.ints.size();
    rp_f += (int)r.floats.size();
    rp_e += r.n_env;
  }
  int sm_i = 0, sm_f = 0, sm_e = 0;
  for (const auto& m : lm.subs) {
    sm_i += (int)m.ints.size();
    sm_f += (int)m.floats.size();
    sm_e += m.n_env;
  }
  void* sd = solver_new((int)lm.species.size(), n_cells, lm.var_type.data(), (int)lm.rxns.size(),
                        lm.n_int(), lm.n_float(), lm.n_env(), (int)lm.phases.size(), ph_i, ph_f,
                        (int)lm.reps.size(), rp_i, rp_f, rp_e, (int)lm.subs.size(), sm_i, sm_f,
                        sm_e);
  if (!sd) return nullptr;
  // reactions, then phases and representations, the order of
  // camp_solver_data%initialize (src/camp_solver_data.F90:635-700)
  for (auto& r : lm.rxns)
    rxn_add_condensed_data(r.type, (int)r.ints.size(), (int)r.floats.size(), r.n_env,
                           r.ints.data(), r.floats.data(), sd);
  for (auto& p : lm.phases)
    aero_phase_add_condensed_data((int)p.ints.size(), (int)p.floats.size(), p.ints.data(),
                                  p.floats.data(), sd);
  for (auto& r : lm.reps)
    aero_rep_add_condensed_data(r.type, (int)r.ints.size(), (int)r.floats.size(), r.n_env,
                                r.ints.data(), r.floats.data(), sd);
  for (auto& m : lm.subs)
    sub_model_add_condensed_data(m.type, (int)m.ints.size(), (int)m.floats.size(), m.n_env,
                                 m.ints.data(), m.floats.data(), sd);
  Solver* s = S(sd);
  if (s->add_error) {
    set_error("camp_b200_solver_from_json: " + s->add_error_msg);
    solver_free(sd);
    return nullptr;
  }
  s->state_names = lm.species;
  s->json_abs_tol = lm.abs_tol;
  s->json_rel_tol = lm.rel_tol;
  return sd;
}

int camp_b200_n_state_var(void* solver_data) { return S(solver_data)->n_state; }

int camp_b200_state_name(void* solver_data, int i, char* buf, int buf_len) {
  Solver* s = S(solver_data);
  if (i < 0 || i >= (int)s->state_names.size()) return -1;
  const std::string& n = s->state_names[i];
  if (buf && buf_len > 0) {
    const int k = std::min<int>((int)n.size(), buf_len - 1);
    std::memcpy(buf, n.data(), k);
    buf[k] = '\0';
  }
  return (int)n.size();
}

int camp_b200_json_tolerances(void* solver_data, double* abs_tol, double* rel_tol) {
  Solver* s = S(solver_data);
  if (s->json_abs_tol.empty()) return -1;
  if (abs_tol) std::copy(s->json_abs_tol.begin(), s->json_abs_tol.end(), abs_tol);
  if (rel_tol) *rel_tol = s->json_rel_tol;
  return 0;
}

int camp_b200_get_var_type(void* solver_data, int* out) {
  Solver* s = S(solver_data);
  std::copy(s->var_type.begin(), s->var_type.end(), out);
  return 0;
}

int camp_b200_get_aero_data(void* solver_data, int which, int index, int* n_int, int* n_float,
                            int* ints, double* floats) {
  const Model& m = *S(solver_data)->model;
  const int count = which == 0   ? m.n_aero_phase()
                    : which == 1 ? m.n_aero_rep()
                    : which == 2 ? m.n_sub_model()
                                 : -1;
  if (index < 0 || index >= count) return -1;
  const std::vector<int>& I = which == 0   ? m.aero_phase_int(index)
                              : which == 1 ? m.aero_rep_int(index)
                                           : m.sub_model_int(index);
  const std::vector<double>& F = which == 0   ? m.aero_phase_float(index)
                                 : which == 1 ? m.aero_rep_float(index)
                                              : m.sub_model_float(index);
  if (n_int) *n_int = (int)I.size();
  if (n_float) *n_float = (int)F.size();
  if (ints) std::copy(I.begin(), I.end(), ints);
  if (floats) std::copy(F.begin(), F.end(), floats);
  return 0;
}

int camp_b200_rxn_float_data_size(void* solver_data) {
  return (int)S(solver_data)->model->rxn_float().size();
}

int camp_b200_get_rxn_float_data(void* solver_data, double* out) {
  const Model& m = *S(solver_data)->model;
  std::copy(m.rxn_float().begin(), m.rxn_float().end(), out);
  return 0;
}

}  // extern "C"
