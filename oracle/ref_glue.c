/* Test-infrastructure glue around the reference CAMP C sources.
 *
 * This file is ORACLE code: only tests/, the smoke check and the CPU-baseline
 * leg of bench.py load it.  It is linked with the reference's own reaction,
 * derivative, Jacobian, aerosol and sub-model C files (compiled from the
 * reference tree by oracle/Makefile) so that the derivative, Jacobian and
 * sparsity used as the parity target are produced by the reference's code.
 *
 * The reference's driver, src/camp_solver.c, cannot be compiled here (it needs
 * the modified CVODE and KLU), so the few pieces of it that the parity target
 * needs are restated below in the same order of operations:
 *   - the allocations of solver_new            (src/camp_solver.c:83-362)
 *   - the sparsity build of get_jac_init       (src/camp_solver.c:1417-1712)
 *   - the per-cell env update of solver_run    (src/camp_solver.c:587-603)
 *   - the per-cell body of f without the J-estimated blend
 *                                              (src/camp_solver.c:901-954)
 *   - the per-cell body of Jac and the jac_map fold
 *                                              (src/camp_solver.c:1052-1108)
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "camp_common.h"
#include "aero_phase_solver.h"
#include "aero_rep_solver.h"
#include "rxn_solver.h"
#include "sub_model_solver.h"

/* SolverData must be the first member so that the reference's
 * *_add_condensed_data(…, void *solver_data) functions, which cast their
 * argument to SolverData*, work on this object directly. */
typedef struct {
  SolverData sd;
  int n_cells;
  int built;
  /* reaction Jacobian (full state space) is sd.jac */
  Jacobian param_jac;
  Jacobian solver_jac;
  int *deriv_ids;       /* state id -> dependent-variable id, or -1 */
  double *J_params;     /* per-cell sub-model parameter Jacobian values */
  double *J_rxn;        /* per-cell reaction Jacobian values */
  int n_rxn_jac_elem;
  int n_param_jac_elem;
  int n_solver_jac_elem;
  int *solver_col_ptrs; /* n_dep_var+1, one cell */
  int *solver_row_ids;  /* n_solver_jac_elem, dependent-variable rows */
} RefSolver;

static void *xmalloc(size_t n) {
  void *p = calloc(n ? n : 1, 1);
  if (!p) {
    fprintf(stderr, "ref_glue: out of memory\n");
    exit(EXIT_FAILURE);
  }
  return p;
}

void *ref_new(int n_state_var, int n_cells, const int *var_type, int n_rxn,
              int n_rxn_int_param, int n_rxn_float_param, int n_rxn_env_param,
              int n_aero_phase, int n_aero_phase_int_param,
              int n_aero_phase_float_param, int n_aero_rep,
              int n_aero_rep_int_param, int n_aero_rep_float_param,
              int n_aero_rep_env_param, int n_sub_model,
              int n_sub_model_int_param, int n_sub_model_float_param,
              int n_sub_model_env_param) {
  RefSolver *rs = (RefSolver *)xmalloc(sizeof(RefSolver));
  ModelData *md = &rs->sd.model_data;
  rs->n_cells = n_cells;
  md->n_per_cell_state_var = n_state_var;
  md->n_cells = n_cells;
  md->var_type = (int *)xmalloc(sizeof(int) * n_state_var);
  int n_dep = 0;
  for (int i = 0; i < n_state_var; ++i) {
    md->var_type[i] = var_type[i];
    if (var_type[i] == CHEM_SPEC_VARIABLE) ++n_dep;
  }
  md->n_per_cell_dep_var = n_dep;
  /* solver_initialize points the model at the caller's absolute tolerances
   * before the sparsity build (src/camp_solver.c:431); HL phase transfer
   * reads them in its update_ids (src/rxns/rxn_HL_phase_transfer.c:188-193).
   * Zero until ref_set_abs_tol. */
  md->abs_tol = (double *)xmalloc(sizeof(double) * n_state_var);
  if (time_derivative_initialize(&rs->sd.time_deriv, (unsigned)n_dep) != 1) {
    fprintf(stderr, "ref_glue: time derivative init failed\n");
    exit(EXIT_FAILURE);
  }
  /* reaction data (one extra int per reaction holds its type) */
  md->rxn_int_data = (int *)xmalloc(sizeof(int) * (n_rxn_int_param + n_rxn));
  md->rxn_float_data = (double *)xmalloc(sizeof(double) * n_rxn_float_param);
  md->rxn_env_data =
      (double *)xmalloc(sizeof(double) * (size_t)n_cells * n_rxn_env_param);
  md->rxn_int_indices = (int *)xmalloc(sizeof(int) * (n_rxn + 1));
  md->rxn_float_indices = (int *)xmalloc(sizeof(int) * (n_rxn + 1));
  md->rxn_env_idx = (int *)xmalloc(sizeof(int) * (n_rxn + 1));
  md->n_rxn = n_rxn;
  /* aerosol phases */
  md->aero_phase_int_data = (int *)xmalloc(sizeof(int) * n_aero_phase_int_param);
  md->aero_phase_float_data =
      (double *)xmalloc(sizeof(double) * n_aero_phase_float_param);
  md->aero_phase_int_indices = (int *)xmalloc(sizeof(int) * (n_aero_phase + 1));
  md->aero_phase_float_indices =
      (int *)xmalloc(sizeof(int) * (n_aero_phase + 1));
  md->n_aero_phase = n_aero_phase;
  /* aerosol representations */
  md->aero_rep_int_data =
      (int *)xmalloc(sizeof(int) * (n_aero_rep_int_param + n_aero_rep));
  md->aero_rep_float_data =
      (double *)xmalloc(sizeof(double) * n_aero_rep_float_param);
  md->aero_rep_env_data =
      (double *)xmalloc(sizeof(double) * (size_t)n_cells * n_aero_rep_env_param);
  md->aero_rep_int_indices = (int *)xmalloc(sizeof(int) * (n_aero_rep + 1));
  md->aero_rep_float_indices = (int *)xmalloc(sizeof(int) * (n_aero_rep + 1));
  md->aero_rep_env_idx = (int *)xmalloc(sizeof(int) * (n_aero_rep + 1));
  md->n_aero_rep = n_aero_rep;
  /* sub-models */
  md->sub_model_int_data =
      (int *)xmalloc(sizeof(int) * (n_sub_model_int_param + n_sub_model));
  md->sub_model_float_data =
      (double *)xmalloc(sizeof(double) * n_sub_model_float_param);
  md->sub_model_env_data = (double *)xmalloc(
      sizeof(double) * (size_t)n_cells * n_sub_model_env_param);
  md->sub_model_int_indices = (int *)xmalloc(sizeof(int) * (n_sub_model + 1));
  md->sub_model_float_indices =
      (int *)xmalloc(sizeof(int) * (n_sub_model + 1));
  md->sub_model_env_idx = (int *)xmalloc(sizeof(int) * (n_sub_model + 1));
  md->n_sub_model = n_sub_model;
  rs->sd.no_solve = (n_rxn == 0);
  return rs;
}

/* Per-state absolute tolerances (the array solver_initialize receives). */
void ref_set_abs_tol(void *h, const double *abs_tol) {
  ModelData *md = &((RefSolver *)h)->sd.model_data;
  memcpy(md->abs_tol, abs_tol, sizeof(double) * md->n_per_cell_state_var);
}

/* Sparsity, id update and Jacobian map: restates get_jac_init
 * (src/camp_solver.c:1417-1712) without the SUNDIALS matrices. */
int ref_build(void *h) {
  RefSolver *rs = (RefSolver *)h;
  ModelData *md = &rs->sd.model_data;
  int n_state = md->n_per_cell_state_var;
  int n_dep = md->n_per_cell_dep_var;

  if (jacobian_initialize_empty(&rs->sd.jac, (unsigned)n_state) != 1) return 1;
  for (int i = 0; i < n_state; ++i)
    jacobian_register_element(&rs->sd.jac, (unsigned)i, (unsigned)i);
  rxn_get_used_jac_elem(md, &rs->sd.jac);
  if (jacobian_build_matrix(&rs->sd.jac) != 1) return 1;
  rs->n_rxn_jac_elem = (int)jacobian_number_of_elements(rs->sd.jac);
  md->n_per_cell_rxn_jac_elem = rs->n_rxn_jac_elem;

  rs->deriv_ids = (int *)xmalloc(sizeof(int) * n_state);
  for (int i = 0, d = 0; i < n_state; ++i)
    rs->deriv_ids[i] = md->var_type[i] == CHEM_SPEC_VARIABLE ? d++ : -1;
  rxn_update_ids(md, rs->deriv_ids, rs->sd.jac);

  if (jacobian_initialize_empty(&rs->param_jac, (unsigned)n_state) != 1)
    return 1;
  jacobian_register_element(&rs->param_jac, 0, 0);
  sub_model_get_used_jac_elem(md, &rs->param_jac);
  if (jacobian_build_matrix(&rs->param_jac) != 1) return 1;
  rs->n_param_jac_elem = (int)jacobian_number_of_elements(rs->param_jac);
  md->n_per_cell_param_jac_elem = rs->n_param_jac_elem;
  sub_model_update_ids(md, rs->deriv_ids, rs->param_jac);

  if (jacobian_initialize_empty(&rs->solver_jac, (unsigned)n_state) != 1)
    return 1;
  int n_mapped = 0;
  for (int i_ind = 0; i_ind < n_state; ++i_ind) {
    for (int i_dep = 0; i_dep < n_state; ++i_dep) {
      if (md->var_type[i_dep] != CHEM_SPEC_VARIABLE ||
          (int)jacobian_get_element_id(rs->sd.jac, (unsigned)i_dep,
                                       (unsigned)i_ind) == -1)
        continue;
      if (md->var_type[i_ind] == CHEM_SPEC_VARIABLE) {
        jacobian_register_element(&rs->solver_jac, (unsigned)i_dep,
                                  (unsigned)i_ind);
        ++n_mapped;
        continue;
      }
      for (int j_ind = 0; j_ind < n_state; ++j_ind) {
        if ((int)jacobian_get_element_id(rs->param_jac, (unsigned)i_ind,
                                         (unsigned)j_ind) != -1 &&
            md->var_type[j_ind] == CHEM_SPEC_VARIABLE) {
          jacobian_register_element(&rs->solver_jac, (unsigned)i_dep,
                                    (unsigned)j_ind);
          ++n_mapped;
        }
      }
    }
  }
  if (jacobian_build_matrix(&rs->solver_jac) != 1) return 1;
  rs->n_solver_jac_elem = (int)jacobian_number_of_elements(rs->solver_jac);
  md->n_per_cell_solver_jac_elem = rs->n_solver_jac_elem;

  rs->solver_col_ptrs = (int *)xmalloc(sizeof(int) * (n_dep + 1));
  rs->solver_row_ids = (int *)xmalloc(sizeof(int) * (rs->n_solver_jac_elem + 1));
  for (int col = 0; col < n_state; ++col) {
    if (rs->deriv_ids[col] == -1) continue;
    rs->solver_col_ptrs[rs->deriv_ids[col]] =
        (int)jacobian_column_pointer_value(rs->solver_jac, (unsigned)col);
  }
  rs->solver_col_ptrs[n_dep] = rs->n_solver_jac_elem;
  for (int e = 0; e < rs->n_solver_jac_elem; ++e)
    rs->solver_row_ids[e] =
        rs->deriv_ids[jacobian_row_index(rs->solver_jac, (unsigned)e)];

  md->n_mapped_values = n_mapped;
  md->jac_map = (JacMap *)xmalloc(sizeof(JacMap) * (n_mapped + 1));
  int i_map = 0;
  for (int i_ind = 0; i_ind < n_state; ++i_ind) {
    for (unsigned e = jacobian_column_pointer_value(rs->sd.jac, (unsigned)i_ind);
         e < jacobian_column_pointer_value(rs->sd.jac, (unsigned)i_ind + 1);
         ++e) {
      int i_dep = (int)jacobian_row_index(rs->sd.jac, e);
      if (md->var_type[i_dep] != CHEM_SPEC_VARIABLE) continue;
      if (md->var_type[i_ind] == CHEM_SPEC_VARIABLE) {
        md->jac_map[i_map].solver_id = (int)jacobian_get_element_id(
            rs->solver_jac, (unsigned)i_dep, (unsigned)i_ind);
        md->jac_map[i_map].rxn_id = (int)e;
        md->jac_map[i_map].param_id = 0;
        ++i_map;
        continue;
      }
      for (int j_ind = 0; j_ind < n_state; ++j_ind) {
        if ((int)jacobian_get_element_id(rs->param_jac, (unsigned)i_ind,
                                         (unsigned)j_ind) != -1 &&
            md->var_type[j_ind] == CHEM_SPEC_VARIABLE) {
          md->jac_map[i_map].solver_id = (int)jacobian_get_element_id(
              rs->solver_jac, (unsigned)i_dep, (unsigned)j_ind);
          md->jac_map[i_map].rxn_id = (int)e;
          md->jac_map[i_map].param_id = (int)jacobian_get_element_id(
              rs->param_jac, (unsigned)i_ind, (unsigned)j_ind);
          ++i_map;
        }
      }
    }
  }
  if (i_map != n_mapped) return 2;
  rs->J_params = (double *)xmalloc(sizeof(double) * (rs->n_param_jac_elem + 1));
  rs->J_rxn = (double *)xmalloc(sizeof(double) * (rs->n_rxn_jac_elem + 1));
  rs->built = 1;
  return 0;
}

int ref_n_dep_var(void *h) {
  return ((RefSolver *)h)->sd.model_data.n_per_cell_dep_var;
}
int ref_n_rxn_jac_elem(void *h) { return ((RefSolver *)h)->n_rxn_jac_elem; }
int ref_n_solver_jac_elem(void *h) {
  return ((RefSolver *)h)->n_solver_jac_elem;
}
int ref_n_mapped_values(void *h) {
  return ((RefSolver *)h)->sd.model_data.n_mapped_values;
}
int ref_n_rxn_env_data(void *h) {
  return ((RefSolver *)h)->sd.model_data.n_rxn_env_data;
}
int ref_rxn_int_data_size(void *h) {
  ModelData *md = &((RefSolver *)h)->sd.model_data;
  return md->rxn_int_indices[md->n_rxn];
}

/* Copies out the reference sparsity: the reaction Jacobian CSC over all state
 * variables, the one-cell solver Jacobian CSC over dependent variables, the
 * jac_map triplets and the reaction int data after rxn_update_ids wrote its
 * DERIV_ID/JAC_ID entries. */
void ref_get_rxn_jac(void *h, int *col_ptrs, int *row_ids) {
  RefSolver *rs = (RefSolver *)h;
  int n = rs->sd.model_data.n_per_cell_state_var;
  for (int c = 0; c <= n; ++c)
    col_ptrs[c] = (int)jacobian_column_pointer_value(rs->sd.jac, (unsigned)c);
  for (int e = 0; e < rs->n_rxn_jac_elem; ++e)
    row_ids[e] = (int)jacobian_row_index(rs->sd.jac, (unsigned)e);
}
void ref_get_solver_jac(void *h, int *col_ptrs, int *row_ids) {
  RefSolver *rs = (RefSolver *)h;
  int n = rs->sd.model_data.n_per_cell_dep_var;
  memcpy(col_ptrs, rs->solver_col_ptrs, sizeof(int) * (n + 1));
  memcpy(row_ids, rs->solver_row_ids, sizeof(int) * rs->n_solver_jac_elem);
}
void ref_get_jac_map(void *h, int *triplets) {
  ModelData *md = &((RefSolver *)h)->sd.model_data;
  for (int i = 0; i < md->n_mapped_values; ++i) {
    triplets[3 * i] = md->jac_map[i].solver_id;
    triplets[3 * i + 1] = md->jac_map[i].rxn_id;
    triplets[3 * i + 2] = md->jac_map[i].param_id;
  }
}
void ref_get_rxn_int_data(void *h, int *out) {
  ModelData *md = &((RefSolver *)h)->sd.model_data;
  memcpy(out, md->rxn_int_data, sizeof(int) * md->rxn_int_indices[md->n_rxn]);
}
void ref_get_rxn_env_data(void *h, int cell, double *out) {
  ModelData *md = &((RefSolver *)h)->sd.model_data;
  memcpy(out, md->rxn_env_data + (size_t)cell * md->n_rxn_env_data,
         sizeof(double) * md->n_rxn_env_data);
}
void ref_set_rxn_env_data(void *h, int cell, const double *in) {
  ModelData *md = &((RefSolver *)h)->sd.model_data;
  memcpy(md->rxn_env_data + (size_t)cell * md->n_rxn_env_data, in,
         sizeof(double) * md->n_rxn_env_data);
}

static void set_cell(ModelData *md, int cell) {
  md->grid_cell_id = cell;
  md->grid_cell_state = &md->total_state[(size_t)cell * md->n_per_cell_state_var];
  md->grid_cell_env = &md->total_env[(size_t)cell * CAMP_NUM_ENV_PARAM_];
  md->grid_cell_rxn_env_data = &md->rxn_env_data[(size_t)cell * md->n_rxn_env_data];
  md->grid_cell_aero_rep_env_data =
      &md->aero_rep_env_data[(size_t)cell * md->n_aero_rep_env_data];
  md->grid_cell_sub_model_env_data =
      &md->sub_model_env_data[(size_t)cell * md->n_sub_model_env_data];
}

/* Points the model at caller-owned state [n_cells*n_state_var] and env
 * [n_cells*2] arrays, as solver_run does (src/camp_solver.c:570-571). */
void ref_set_state(void *h, double *state, double *env) {
  ModelData *md = &((RefSolver *)h)->sd.model_data;
  md->total_state = state;
  md->total_env = env;
}

/* Environment update for one cell (src/camp_solver.c:587-603). */
void ref_update_env(void *h, int cell) {
  ModelData *md = &((RefSolver *)h)->sd.model_data;
  set_cell(md, cell);
  aero_rep_update_env_state(md);
  sub_model_update_env_state(md);
  rxn_update_env_state(md);
}

/* One cell's derivative through the reference code: production and loss
 * sums (converted from the reference's long double accumulators) and the
 * unblended output r_p - r_l (time_derivative_output with deriv_est NULL). */
void ref_calc_deriv(void *h, int cell, double time_step, double *deriv,
                    double *r_p, double *r_l) {
  RefSolver *rs = (RefSolver *)h;
  ModelData *md = &rs->sd.model_data;
  set_cell(md, cell);
  aero_rep_update_state(md);
  sub_model_calculate(md);
  time_derivative_reset(rs->sd.time_deriv);
  rxn_calc_deriv(md, rs->sd.time_deriv, time_step);
  time_derivative_output(rs->sd.time_deriv, deriv, NULL, 0);
  for (int i = 0; i < md->n_per_cell_dep_var; ++i) {
    if (r_p) r_p[i] = (double)rs->sd.time_deriv.production_rates[i];
    if (r_l) r_l[i] = (double)rs->sd.time_deriv.loss_rates[i];
  }
}

/* One cell's Jacobian through the reference code: the reaction Jacobian over
 * all state variables and the solver Jacobian after the jac_map fold
 * (src/camp_solver.c:1052-1108).  J_solver has n_solver_jac_elem entries. */
void ref_calc_jac(void *h, int cell, double time_step, double *J_rxn_out,
                  double *J_solver) {
  RefSolver *rs = (RefSolver *)h;
  ModelData *md = &rs->sd.model_data;
  set_cell(md, cell);
  for (int i = 0; i < rs->n_param_jac_elem; ++i) rs->J_params[i] = 0.0;
  jacobian_reset(rs->sd.jac);
  aero_rep_update_state(md);
  sub_model_calculate(md);
  sub_model_get_jac_contrib(md, rs->J_params, time_step);
  rxn_calc_jac(md, rs->sd.jac, time_step);
  jacobian_output(rs->sd.jac, rs->J_rxn);
  rs->J_params[0] = 1.0;
  for (int i = 0; i < rs->n_solver_jac_elem; ++i) J_solver[i] = 0.0;
  for (int i = 0; i < md->n_mapped_values; ++i)
    J_solver[md->jac_map[i].solver_id] +=
        rs->J_rxn[md->jac_map[i].rxn_id] * rs->J_params[md->jac_map[i].param_id];
  if (J_rxn_out)
    memcpy(J_rxn_out, rs->J_rxn, sizeof(double) * rs->n_rxn_jac_elem);
}

void ref_free(void *h) {
  RefSolver *rs = (RefSolver *)h;
  if (!rs) return;
  /* The packed data arrays are left to process exit: the reference frees
   * them in model_free, which lives in the uncompilable camp_solver.c. */
  free(rs->deriv_ids);
  free(rs->J_params);
  free(rs->J_rxn);
  free(rs->solver_col_ptrs);
  free(rs->solver_row_ids);
  free(rs->sd.model_data.abs_tol);
  free(rs);
}

/* ------------------------------------------------------------------------ */
/* Callback form for the oracle's restated BDF (oracle/camp_oracle.c): one  */
/* cell's f and Jac through the reference code, over dependent variables.   */
/* ------------------------------------------------------------------------ */
typedef struct {
  RefSolver *rs;
  int cell;
  double h0;
} RefCellCtx;

void *ref_cell_ctx_new(void *h, int cell, double h0) {
  RefCellCtx *c = (RefCellCtx *)xmalloc(sizeof(RefCellCtx));
  c->rs = (RefSolver *)h;
  c->cell = cell;
  c->h0 = h0;
  return c;
}
void ref_cell_ctx_free(void *c) { free(c); }

/* camp_solver_update_model_state (src/camp_solver.c:805-833) for one cell */
static int ref_load_y(RefCellCtx *c, const double *y) {
  ModelData *md = &c->rs->sd.model_data;
  double *st = md->total_state + (size_t)c->cell * md->n_per_cell_state_var;
  for (int i = 0, d = 0; i < md->n_per_cell_state_var; ++i) {
    if (md->var_type[i] != CHEM_SPEC_VARIABLE) continue;
    if (y[d] < -SMALL) return 1;
    st[i] = y[d] > -SMALL ? y[d] : TINY;
    ++d;
  }
  return 0;
}

int ref_cb_rhs(void *ctx, double t, const double *y, double h, double *ydot) {
  (void)t;
  RefCellCtx *c = (RefCellCtx *)ctx;
  if (ref_load_y(c, y)) return 1;
  ref_calc_deriv(c->rs, c->cell, h > 0.0 ? h : c->h0, ydot, NULL, NULL);
  return 0;
}

int ref_cb_jac(void *ctx, double t, const double *y, double h, double *jvals) {
  (void)t;
  RefCellCtx *c = (RefCellCtx *)ctx;
  if (ref_load_y(c, y)) return 1;
  ref_calc_jac(c->rs, c->cell, h > 0.0 ? h : c->h0, NULL, jvals);
  return 0;
}
