/* CPU oracle for the CAMP per-cell chemistry solve (TEST INFRASTRUCTURE).
 *
 * Only tests/, the smoke check and bench.py's CPU-baseline leg use this
 * library, as the checker.  The product (libcamp_b200) never links it.
 *
 * Contents, each restated from the reference and cited at its definition:
 *   - gas-phase reaction rate constants, derivative and Jacobian
 *     contributions for the ARRHENIUS, TROE, CMAQ_H2O2, CMAQ_OH_HNO3 and
 *     PHOTOLYSIS types (src/rxns/rxn_*.c), with long double accumulators
 *     as in src/time_derivative.c and src/Jacobian.c;
 *   - the Jacobian sparsity build and DERIV_ID/JAC_ID update
 *     (src/Jacobian.c, src/camp_solver.c:1417-1712), with the sub-model
 *     parameter Jacobian and the J_rxn x J_params fold;
 *   - the ZSR aerosol-water and PD-FiTE activity sub-models
 *     (src/sub_models/sub_model_ZSR_aerosol_water.c,
 *     src/sub_models/sub_model_PDFiTE.c), run before every f and J;
 *   - a sparse LU of I - gamma*J on a Markowitz diagonal-pivot order (the
 *     reference uses SuiteSparse KLU, which is not in the reference tree);
 *   - the variable-order BDF integrator of CVODE (Hindmarsh et al., ACM TOMS
 *     31(3) 2005 and the CVODE documentation), restated per cell, because the
 *     reference's modified CVODE 3.4-alpha source is not in the tree.
 */
#ifndef CAMP_ORACLE_H
#define CAMP_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OracleMech OracleMech;

/* Solver outcome codes (CVODE flag values) */
#define OR_SUCCESS 0
#define OR_TOO_MUCH_WORK (-1)
#define OR_TOO_MUCH_ACC (-2)
#define OR_ERR_FAILURE (-3)
#define OR_CONV_FAILURE (-4)
#define OR_LSETUP_FAIL (-6)
#define OR_RHSFUNC_FAIL (-8)
#define OR_REPTD_RHSFUNC_ERR (-10)
#define OR_UNREC_RHSFUNC_ERR (-11)
#define OR_ILL_INPUT (-22)
#define OR_TOO_CLOSE (-27)

/* per-cell statistics (CVODE counters) */
typedef struct {
  long nst, nfe, nsetups, netf, nni, ncfn, nje;
  double hu, hcur;
  int flag;
  int qu;
} OracleStats;

/* Callback form of the right-hand side and Jacobian, so the same BDF can
 * run on the oracle's own f/J or on the reference's (through ref_glue.c).
 * f returns 0 on success, >0 for a recoverable failure, <0 unrecoverable.
 * jac fills the solver Jacobian values in the CSC order of the pattern. */
typedef int (*or_rhs_fn)(void *ctx, double t, const double *y, double h,
                         double *ydot);
typedef int (*or_jac_fn)(void *ctx, double t, const double *y, double h,
                         double *jvals);

OracleMech *om_new(int n_state_var, const int *var_type, int n_rxn);
int om_add_rxn(OracleMech *m, int type, int n_int, int n_float, int n_env,
               const int *ints, const double *floats);
/* aero_phase_add_condensed_data / aero_rep_add_condensed_data (the
 * modal/binned mass representation, type 2, only) */
int om_add_aero_phase(OracleMech *m, int n_int, int n_float, const int *ints,
                      const double *floats);
int om_add_aero_rep(OracleMech *m, int type, int n_int, int n_float, int n_env,
                    const int *ints, const double *floats);
/* GMD (what 0) or GSD (what 1) of a mode in one cell's rxn_env buffer, whose
 * representation part follows the reaction env parameters */
int om_set_aero_env(const OracleMech *m, double *rxn_env_cell, int rep, int section,
                    int what, double value);
/* sub_model_add_condensed_data: ZSR aerosol water (2) and PD-FiTE (3);
 * ints without the type slot.  Returns 0, or 2 for another type. */
int om_add_sub_model(OracleMech *m, int type, int n_int, int n_float, int n_env,
                     const int *ints, const double *floats);
int om_build(OracleMech *m);
/* the absolute tolerances (per state variable) that set the aqueous
 * equilibrium's minimum water, as solver_initialize's do; om_solve sets
 * them from its own argument */
void om_set_abs_tol(const OracleMech *m, const double *abs_tol);
void om_free(OracleMech *m);

/* Experiment switches of the integrator (defaults 0, 0):
 *   guard_step  0 = f and J get the integrator's current step as their
 *               time_step, as the reference's f does through
 *               CVodeGetCurrentStep (src/camp_solver.c:872-876), which the
 *               negative-yield product guard multiplies
 *               (src/rxns/rxn_arrhenius.c:153-160); > 0 = that fixed step
 *               instead (not the reference's semantics; it shows what the
 *               step dependence of the guard costs);
 *   positivity  how a predicted or corrected state below zero is handled:
 *               OM_POS_PROJECT (this oracle's rule and the device's),
 *               OM_POS_GUESS_HELPER (the reference's guess_helper restated,
 *               with the constraint check), OM_POS_GUESS_HELPER_ONLY, or
 *               OM_POS_NONE (plain CVODE).
 * Returns nonzero for an invalid setting. */
#define OM_POS_PROJECT 0
#define OM_POS_GUESS_HELPER 1
#define OM_POS_GUESS_HELPER_ONLY 2
#define OM_POS_NONE 3
int om_set_experiment(OracleMech *m, double guard_step, int positivity);

int om_n_dep_var(const OracleMech *m);
int om_n_rxn_env_data(const OracleMech *m);
int om_n_param_jac_elem(const OracleMech *m);
int om_n_mapped_values(const OracleMech *m);
/* the solver-Jacobian fold as (solver id, reaction-Jacobian id, parameter
 * id) triplets, src/camp_solver.c:1649-1681 */
void om_get_jac_map(const OracleMech *m, int *triplets);
int om_n_rxn_jac_elem(const OracleMech *m);
int om_n_solver_jac_elem(const OracleMech *m);
int om_n_lu_elem(const OracleMech *m);
int om_rxn_int_data_size(const OracleMech *m);
void om_get_rxn_jac(const OracleMech *m, int *col_ptrs, int *row_ids);
void om_get_solver_jac(const OracleMech *m, int *col_ptrs, int *row_ids);
void om_get_rxn_int_data(const OracleMech *m, int *out);
void om_get_lu_order(const OracleMech *m, int *perm);

/* Base rate of the first reaction of rxn_type (PHOTOLYSIS, FIRST_ORDER_LOSS,
 * EMISSION, WET_DEPOSITION) whose RXN_ID_ equals rxn_id, in one cell's
 * rxn_env_data, as rxn_update_data does (src/rxn_solver.c:700-760); returns
 * whether one matched.  om_set_photo_rate is the PHOTOLYSIS case. */
int om_set_rate(const OracleMech *m, double *rxn_env_cell, int rxn_type, int rxn_id,
                double base_rate);
int om_set_photo_rate(const OracleMech *m, double *rxn_env_cell, int photo_id,
                      double base_rate);
/* Rate constants for one cell from env = {T [K], P [Pa]}. */
void om_update_env(const OracleMech *m, const double *env, double *rxn_env_cell);
/* One cell's derivative: production, loss and net over dependent vars. */
void om_deriv(const OracleMech *m, const double *state, const double *rxn_env_cell,
              double time_step, double *deriv, double *r_p, double *r_l);
/* One cell's solver Jacobian values (solver CSC order). */
void om_jac(const OracleMech *m, const double *state, const double *rxn_env_cell,
            double time_step, double *jvals);

/* Integrates n_cells independent cells from t0 to t1 (per-cell CVODE
 * semantics), with the oracle's own f/J.  state is [n_cells*n_state_var] and
 * is updated in place like solver_run; env is [n_cells*2]; rxn_env is
 * [n_cells*n_rxn_env_data] and must hold the photolysis base rates.
 * status[c] receives the per-cell flag; stats may be NULL.
 * Returns the number of failed cells. */
int om_solve(const OracleMech *m, int n_cells, double *state, const double *env,
             double *rxn_env, double t0, double t1, double rtol,
             const double *abs_tol, int max_steps, int max_conv_fails,
             int n_threads, int *status, OracleStats *stats);

/* The same integrator driven by external f/J callbacks.  ctxs[i] is the
 * callback context for cell i; the callbacks see only dependent variables.
 * abs_tol_dep has one entry per dependent variable. */
int om_solve_cb(const OracleMech *m, int n_cells, double *y_dep, double t0,
                double t1, double rtol, const double *abs_tol_dep,
                int max_steps, int max_conv_fails, or_rhs_fn f, or_jac_fn jac,
                void **ctxs, int *status, OracleStats *stats);

#ifdef __cplusplus
}
#endif
#endif
