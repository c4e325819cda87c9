/* libcamp_b200 — drop-in C ABI for CAMP's per-cell chemistry solve on B200.
 *
 * The first group of entry points keeps the names, argument meaning and
 * error behaviour of the reference's C solver interface, so the reference's
 * Fortran caller (src/camp_solver_data.F90:43-363, bind(c)) links against
 * this library unchanged.  Each declaration cites the reference interface it
 * replaces.  The second group (camp_b200_*) is this library's own extension
 * API: device-resident runs, precision selection, per-cell status and the
 * evaluation hooks the parity tests use.
 *
 * Per-cell semantics: every grid cell is integrated independently with its
 * own BDF step size and order (the reference couples all cells of a call into
 * one CVODE system, src/camp_solver.c:145).  solver_run returns 1 if any cell
 * failed; failed cells keep their input state.
 */
#ifndef CAMP_B200_H
#define CAMP_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------------- */
/* Reference-compatible entry points                                        */
/* ---------------------------------------------------------------------- */

/* replaces src/camp_solver.c:83 (declared src/camp_solver.h:16-24) */
void *solver_new(int n_state_var, int n_cells, int *var_type, int n_rxn,
                 int n_rxn_int_param, int n_rxn_float_param,
                 int n_rxn_env_param, int n_aero_phase,
                 int n_aero_phase_int_param, int n_aero_phase_float_param,
                 int n_aero_rep, int n_aero_rep_int_param,
                 int n_aero_rep_float_param, int n_aero_rep_env_param,
                 int n_sub_model, int n_sub_model_int_param,
                 int n_sub_model_float_param, int n_sub_model_env_param);

/* replaces src/camp_solver.c:374 (src/camp_solver.h:25-26) */
void solver_initialize(void *solver_data, double *abs_tol, double rel_tol,
                       int max_steps, int max_conv_fails);

/* replaces src/camp_solver.c:544 (src/camp_solver.h:31-32); 0 = success,
 * 1 = at least one cell failed */
int solver_run(void *solver_data, double *state, double *env, double t_initial,
               double t_final);

/* replaces src/camp_solver.c:725 (src/camp_solver.h:33-40).  Counters are the
 * maximum over the cells of the last run (the per-cell analogue of the single
 * coupled CVODE's counters); per-cell values come from
 * camp_b200_get_cell_stats. */
void solver_get_statistics(void *solver_data, int *solver_flag, int *num_steps,
                           int *RHS_evals, int *LS_setups,
                           int *error_test_fails, int *NLS_iters,
                           int *NLS_convergence_fails, int *DLS_Jac_evals,
                           int *DLS_RHS_evals, double *last_time_step__s,
                           double *next_time_step__s, int *Jac_eval_fails,
                           int *RHS_evals_total, int *Jac_evals_total,
                           double *RHS_time__s, double *Jac_time__s,
                           double *max_loss_precision);

/* replaces src/camp_solver.c:1764 */
void solver_reset_timers(void *solver_data);
/* replaces src/camp_solver.c:1832 */
void solver_free(void *solver_data);
/* replaces src/camp_solver.c:1962 */
void solver_free_update_data(void *update_data);

/* replace src/camp_solver.c:502 and :522 (CAMP_DEBUG builds of the
 * reference); accepted and recorded, they change nothing here */
int solver_set_debug_out(void *solver_data, int do_output);
int solver_set_eval_jac(void *solver_data, int eval_Jac);

/* replaces src/rxn_solver.c:658 (src/rxn_solver.h) */
void rxn_add_condensed_data(int rxn_type, int n_int_param, int n_float_param,
                            int n_env_param, int *int_param,
                            double *float_param, void *solver_data);
/* replaces src/rxn_solver.c:708; rxn_id is the in/out cursor of the
 * reference: the search starts at *rxn_id and stops at the first reaction
 * that accepts the update */
void rxn_update_data(int cell_id, int *rxn_id, int update_rxn_type,
                     void *update_data, void *solver_data);
/* replaces src/rxn_solver.c:769 */
void rxn_print_data(void *solver_data);
/* replaces src/rxn_solver.c:851 */
void rxn_free_update_data(void *update_data);
/* replace src/rxns/rxn_photolysis.c:262-283 (bound from
 * src/rxns/rxn_photolysis.F90:135-152) */
void *rxn_photolysis_create_rate_update_data(void);
void rxn_photolysis_set_rate_update_data(void *update_data, int photo_id,
                                         double base_rate);
/* replace src/aero_reps/aero_rep_modal_binned_mass.c:677-739 (bound from
 * src/aero_reps/aero_rep_modal_binned_mass.F90:258-263): GMD [m] and GSD
 * update data of one mode (section) of the representation with that id */
void *aero_rep_modal_binned_mass_create_gmd_update_data(void);
void aero_rep_modal_binned_mass_set_gmd_update_data(void *update_data, int aero_rep_id,
                                                    int section_id, double gmd);
void *aero_rep_modal_binned_mass_create_gsd_update_data(void);
void aero_rep_modal_binned_mass_set_gsd_update_data(void *update_data, int aero_rep_id,
                                                    int section_id, double gsd);
/* replace src/rxns/rxn_emission.c:192-213 (bound from
 * src/rxns/rxn_emission.F90:118-135) */
void *rxn_emission_create_rate_update_data(void);
void rxn_emission_set_rate_update_data(void *update_data, int rxn_id,
                                       double base_rate);
/* replace src/rxns/rxn_first_order_loss.c:208-229 (bound from
 * src/rxns/rxn_first_order_loss.F90:121-138) */
void *rxn_first_order_loss_create_rate_update_data(void);
void rxn_first_order_loss_set_rate_update_data(void *update_data, int rxn_id,
                                               double base_rate);
/* replace src/rxns/rxn_wet_deposition.c:218-239 (bound from
 * src/rxns/rxn_wet_deposition.F90:124-141) */
void *rxn_wet_deposition_create_rate_update_data(void);
void rxn_wet_deposition_set_rate_update_data(void *update_data, int rxn_id,
                                             double base_rate);

/* replace src/aero_phase_solver.c:175,210, src/aero_rep_solver.c:443,492,546
 * and src/sub_model_solver.c:413,468,509.  Aerosol phases and the
 * modal/binned mass representation (type 2) are solved with SIMPOL
 * (reaction type 10) and HL (type 6) partitioning and aqueous equilibrium
 * (type 7), the aerosol-phase water and ion pairs being constant species;
 * other representation types and any sub-model are rejected at
 * solver_initialize. */
void aero_phase_add_condensed_data(int n_int_param, int n_float_param,
                                   int *int_param, double *float_param,
                                   void *solver_data);
void aero_rep_add_condensed_data(int aero_rep_type, int n_int_param,
                                 int n_float_param, int n_env_param,
                                 int *int_param, double *float_param,
                                 void *solver_data);
void aero_rep_update_data(int cell_id, int *aero_rep_id, int update_aero_rep_type,
                          void *update_data, void *solver_data);
void sub_model_add_condensed_data(int sub_model_type, int n_int_param,
                                  int n_float_param, int n_env_param,
                                  int *int_param, double *float_param,
                                  void *solver_data);
void sub_model_update_data(int cell_id, int *sub_model_id,
                           int update_sub_model_type, void *update_data,
                           void *solver_data);
void aero_phase_print_data(void *solver_data);
void aero_rep_print_data(void *solver_data);
void sub_model_print_data(void *solver_data);

/* ---------------------------------------------------------------------- */
/* Extension API                                                            */
/* ---------------------------------------------------------------------- */

/* precision modes */
#define CAMP_B200_FP64 0  /* everything in FP64 */
#define CAMP_B200_MIXED 1 /* FP32 Jacobian and LU, FP64 residual/state/error test */

/* per-cell status codes (CVODE flag values) */
#define CAMP_B200_OK 0
#define CAMP_B200_TOO_MUCH_WORK (-1)
#define CAMP_B200_TOO_MUCH_ACC (-2)
#define CAMP_B200_ERR_FAILURE (-3)
#define CAMP_B200_CONV_FAILURE (-4)
#define CAMP_B200_LSETUP_FAIL (-6)
#define CAMP_B200_RHSFUNC_FAIL (-8)
#define CAMP_B200_REPTD_RHSFUNC_ERR (-10)
#define CAMP_B200_UNREC_RHSFUNC_ERR (-11)
#define CAMP_B200_ILL_INPUT (-22)
#define CAMP_B200_TOO_CLOSE (-27)
#define CAMP_B200_NOT_RUN (-99)

/* per-cell counters of the last run */
typedef struct {
  int status;
  int nst, nfe, nsetups, netf, nni, ncfn, nje;
  double hu, hcur;
} camp_b200_cell_stats;

/* Last error message of this thread ("" if none). */
const char *camp_b200_last_error(void);
/* 1 if the solver finished solver_initialize without error. */
int camp_b200_is_ready(void *solver_data);

int camp_b200_set_precision(void *solver_data, int mode);
/* cells per block (warps per block); 0 = automatic */
int camp_b200_set_launch(void *solver_data, int warps_per_block, int blocks_per_sm);
/* LU strategy of the per-cell linear algebra: 0 = level schedules spread over
 * the 32 lanes of a cell's warp, 1 = one lane factors and solves row by row
 * (fewer warp synchronisations).  The autotuner picks per mechanism. */
int camp_b200_set_lu_mode(void *solver_data, int mode);
/* Kernel organisation: 0 = one warp per cell (lanes share a cell's sparse
 * work), 1 = one lane per cell (32 cells per warp share every instruction),
 * 2 = one thread block per cell (the cell's LU in the block's shared memory,
 * f, J, factorization and solves on all its warps; gas-phase mechanisms, for
 * LUs beyond the warp kernel's tables).  With 0 on a mechanism beyond the
 * warp kernel's tables the solve runs the block form where it has its
 * tables, else the lane form.  place (lane kernel only): bit 0 keeps the state y, bit 1 the LU factors and
 * bit 2 the solve vector in shared memory; the rest of a cell's working set
 * lives in a lane-interleaved global scratch.  -1 keeps the current value. */
int camp_b200_set_kernel(void *solver_data, int kernel, int place);
/* 1: the device step of each run (cell-counter reset + solve kernel) is
 * launched as one instantiated CUDA graph whose kernel node is updated with
 * the run's arguments, instead of as separate launches.  Results are the
 * same either way.  Default 0. */
int camp_b200_set_graph(void *solver_data, int enable);
/* Where the warp-per-cell kernel keeps each cell's Nordsieck history and rate
 * constants: 0 = shared memory (default), 1 = global memory (L1/L2 cached),
 * which leaves shared memory for more resident cells.  The autotuner picks. */
int camp_b200_set_layout(void *solver_data, int hist_global);
/* Autotuner: solves the given sample of cells (host buffers, state is not
 * modified) once per candidate launch configuration -- for the warp-per-cell
 * kernel the cells per block, the history layout of camp_b200_set_layout and
 * the LU mode of camp_b200_set_lu_mode, and the block-per-cell kernel where
 * the mechanism has its tables (the lane-per-cell kernel only where neither
 * has) -- for the current
 * precision, and keeps the fastest by kernel time.  Use a sample
 * representative of the cells to be solved (a few thousand cells, the host
 * step of the run).  0 or -1. */
int camp_b200_autotune(void *solver_data, const double *state, const double *env,
                       int n_cells, double t_initial, double t_final);
/* The launch configuration in use and the autotuner's sample time (ms, -1
 * when not tuned). */
int camp_b200_get_tuning(void *solver_data, int *warps_per_block, int *hist_global,
                         int *lu_mode, double *sample_ms);
/* The kernel solver_run uses: 0 warp per cell, 1 lane per cell, 2 block per
 * cell (camp_b200_set_kernel, the autotuner's choice, or the form a
 * mechanism beyond the warp kernel's tables falls back to). */
int camp_b200_get_kernel(void *solver_data);
/* Orders the cells of the next run by decreasing internal step count of the
 * previous run (longest-first scheduling of the persistent kernel). */
int camp_b200_set_cost_ordering(void *solver_data, int enable);

/* Runs on caller-owned device buffers (state [n_cells*n_state_var], env
 * [n_cells*2]) on the given cudaStream_t (NULL = the solver's own stream, not
 * the legacy default stream) without host copies; n_cells may be below the capacity given to solver_new.  Returns 0
 * or 1 like solver_run after the stream has been synchronised, or -1 on a
 * usage error. */
int camp_b200_run_device(void *solver_data, double *d_state, const double *d_env,
                         int n_cells, double t_initial, double t_final,
                         void *stream);
/* Same, but returns right after the launch (no synchronisation, status not
 * read back).  Use camp_b200_sync_status afterwards. */
int camp_b200_launch_device(void *solver_data, double *d_state,
                            const double *d_env, int n_cells, double t_initial,
                            double t_final, void *stream);
int camp_b200_sync_status(void *solver_data, void *stream);

/* No counterpart in the reference: a device-resident solve that allocates no
 * device memory, for callers that cannot call cudaMalloc while they run (a
 * host model whose pool allocator owns the device heap, or code running where
 * allocation is not allowed).  All buffers are the caller's: state
 * [n_cells*n_state_var] (updated in place), env [n_cells*2], the per-cell
 * rate matrix d_photo [n_cells*camp_b200_n_photo()] laid out as for
 * camp_b200_set_photo_rates (host-set reaction rates, then the GMD and GSD
 * columns of every aerosol mode, see camp_b200_rate_column; NULL only when
 * camp_b200_n_photo() is 0) and the per-cell results d_stats [n_cells], all
 * in device memory.  The solve's scratch lives in one static 8 MiB device
 * array that every GPU loading this library holds until exit; a mechanism
 * needing more than that for one resident cell per SM is rejected with an
 * error, fewer resident cells are used when it needs less.  The first call
 * on a device looks up the array's address and keeps it for the life of the
 * process (do not use this call on a device after cudaDeviceReset); make
 * that first call before any stream capture.  Calls share the array, so two
 * calls that overlap on the GPU race.  This call records no timing and no
 * statistics in the solver: camp_b200_last_kernel_ms and
 * camp_b200_get_cell_stats keep describing its last regular run.  The
 * Nordsieck history stays in shared memory whatever camp_b200_set_layout
 * chose.  Waits for the stream; returns 0 when the solve ran (per-cell
 * status in d_stats) or -1 with camp_b200_last_error() set. */
int camp_b200_run_device_noalloc(void *solver_data, double *d_state,
                                 const double *d_env, const double *d_photo,
                                 camp_b200_cell_stats *d_stats, int n_cells,
                                 double t_initial, double t_final, void *stream);

/* Per-cell host-set base rates: rates[c * n_photo + j] for column j of cell
 * c, as if rxn_update_data had been called for every cell and reaction.
 * There is one column per reaction whose rate the host sets (PHOTOLYSIS,
 * FIRST_ORDER_LOSS, EMISSION, WET_DEPOSITION), in mechanism order; for a
 * mechanism whose only such reactions are photolysis, column j is photolysis
 * reaction j. */
int camp_b200_n_photo(void *solver_data);
int camp_b200_set_photo_rates(void *solver_data, const double *rates, int n_cells);
/* Which reaction column `column` of the base rates belongs to: its index in
 * mechanism order, its type and its RXN_ID_ (the id update data carries).
 * The columns after the reaction columns hold the geometric mean diameter
 * [m] and standard deviation of every mode of the modal/binned aerosol
 * representations (their update data sets them per cell); for those the
 * reaction index is -1 - (representation index), the type
 * CAMP_B200_COLUMN_GMD or _GSD and the id the section (mode) index.
 * Any pointer may be NULL.  0, or -1 when there is no such column. */
#define CAMP_B200_COLUMN_GMD (-1)
#define CAMP_B200_COLUMN_GSD (-2)
int camp_b200_rate_column(void *solver_data, int column, int *rxn_index, int *rxn_type,
                          int *rxn_id);
/* Device-resident form: rates [n_cells * n_photo] in device memory, read by
 * every following run (no per-run upload) until called with NULL, which
 * returns to the host rates.  The buffer must stay valid meanwhile. */
int camp_b200_set_photo_rates_device(void *solver_data, const double *d_rates, int n_cells);

int camp_b200_get_cell_stats(void *solver_data, camp_b200_cell_stats *out, int n_cells);
/* number of GPU kernel launches made by this solver since creation */
long camp_b200_kernel_launches(void *solver_data);
/* duration of the last solve kernel in ms (CUDA events on its stream) */
double camp_b200_last_kernel_ms(void *solver_data);

/* Sparsity and data after solver_initialize (for parity tests). */
int camp_b200_n_dep_var(void *solver_data);
int camp_b200_n_jac_elem(void *solver_data);
int camp_b200_n_lu_elem(void *solver_data);
int camp_b200_rxn_int_data_size(void *solver_data);
int camp_b200_get_solver_jac(void *solver_data, int *col_ptrs, int *row_ids);
int camp_b200_get_rxn_int_data(void *solver_data, int *out);
int camp_b200_get_lu_order(void *solver_data, int *perm);
/* The block-per-cell kernel's tables (the BlockOff header of blob.hpp, then
 * its sections; absolute tolerances zeroed), built on the host from the
 * sparsity: returns their size in bytes and copies them to out when
 * capacity allows; -1 (with camp_b200_last_error) when the mechanism has no
 * such tables. */
long camp_b200_get_block_tables(void *solver_data, void *out, long capacity);
/* The solver-Jacobian fold J_solver[s] += J_rxn[r] * J_params[p] as (s, r,
 * p) triplets in the reference's order (src/camp_solver.c:1649-1681; p = 0
 * is the unit parameter, the others the sub-model parameter Jacobian's
 * elements): camp_b200_n_mapped_values() triplets, or -1 before
 * solver_initialize. */
int camp_b200_n_mapped_values(void *solver_data);
int camp_b200_get_jac_map(void *solver_data, int *triplets);

/* Device evaluation of the derivative and Jacobian for n_cells states (host
 * buffers), through the same device code the solver uses: rate constants
 * from env and the photolysis rates set for those cells, then f (production,
 * loss, net) and the solver Jacobian (CSC order of camp_b200_get_solver_jac,
 * production and loss parts) at time step h.  Entries that no reaction can
 * make non-zero (HL's partials over the mode's mass species, zero for the
 * modal/binned representation) are output as zero; the LU leaves them out. */
int camp_b200_eval_deriv(void *solver_data, const double *state, const double *env,
                         int n_cells, double h, double *r_p, double *r_l,
                         double *deriv);
int camp_b200_eval_jac(void *solver_data, const double *state, const double *env,
                       int n_cells, double h, double *j_prod, double *j_loss);

/* ---------------------------------------------------------------------- */
/* Serving loop (continuous batching of column solves)                      */
/* ---------------------------------------------------------------------- */

/* A request is one column: n_cells cells of one mechanism (an initialised
 * solver registered with the server) over its own host step.  Whenever one of
 * n_slots slots is free, the oldest queued request and the later queued
 * requests of the same mechanism that fit the device and pinned-host budgets
 * (MiB) are merged into one launch whose warps share all their cells;
 * launches on different slots run concurrently.  Each cell's result does not
 * depend on what else runs. */
void *camp_b200_server_new(int n_slots, double device_mb, double host_mb);
/* Registers an initialised solver (its tables and current settings); returns
 * the mechanism index, or -1.  Register every mechanism before submitting. */
int camp_b200_server_add_solver(void *server, void *solver_data);
/* Queues a request; state [n_cells*n_state_var], env [n_cells*2] and photo
 * [n_cells*n_photo] (NULL without photolysis) are host arrays that must stay
 * valid until camp_b200_server_wait returns, which writes the new state.
 * Returns the request id (>= 0) or -1. */
long camp_b200_server_submit(void *server, int mech, double *state,
                             const double *env, const double *photo, int n_cells,
                             double t_initial, double t_final);
/* Blocks until the request is done; 0 = every cell succeeded, 1 = some cell
 * failed (its state is left as submitted), -1 = error.  latency_ms (may be
 * NULL) receives submit-to-completion time; stats (may be NULL) n_cells
 * per-cell counters. */
int camp_b200_server_wait(void *server, long request, double *latency_ms,
                          camp_b200_cell_stats *stats, int n_cells);
/* Requests submitted and not yet waited for. */
int camp_b200_server_pending(void *server);
void camp_b200_server_free(void *server);

/* Device-resident columns.  open_column copies a column's concentrations
 * (state [n_cells*n_state_var], host) into the server's device budget once
 * and returns the column id, or -1.  submit_column queues one host step of
 * it: only env [n_cells*2] and photo [n_cells*n_photo] come from the host
 * (valid until camp_b200_server_wait returns for the request id it
 * returns); the concentrations stay on the device, and a column's steps run
 * one after another in submission order while other requests pass them.
 * Every step restarts the BDF history as solver_run does, so k steps equal k
 * solver_run calls.  read_column copies the concentrations after the
 * column's queued steps into state; close_column waits for them and returns
 * the memory.  0 or -1 with camp_b200_last_error() set. */
long camp_b200_server_open_column(void *server, int mech, const double *state,
                                  int n_cells);
long camp_b200_server_submit_column(void *server, long column, const double *env,
                                    const double *photo, double t_initial,
                                    double t_final);
int camp_b200_server_read_column(void *server, long column, double *state);
int camp_b200_server_close_column(void *server, long column);

/* ---------------------------------------------------------------------- */
/* CAMP JSON input without the Fortran camp_core                            */
/* ---------------------------------------------------------------------- */

/* replaces the Fortran camp_core's input reading and packing
 * (src/camp_core.F90:303-798, src/chem_spec_data.F90, src/rxns/rxn_*.F90
 * initialize, src/aero_phase_data.F90:306-385,
 * src/aero_reps/aero_rep_modal_binned_mass.F90:334-661): reads CAMP JSON
 * files (CHEM_SPEC, MECHANISM, RELATIVE_TOLERANCE, AERO_PHASE and
 * AERO_REP_MODAL_BINNED_MASS objects), orders the state (gas species in order
 * of first appearance, then each representation's species), packs every
 * reaction (SIMPOL, HL, aqueous equilibrium and wet deposition over the
 * phase instances included), phase and representation and calls solver_new,
 * rxn_add_condensed_data, aero_phase_add_condensed_data and
 * aero_rep_add_condensed_data.  Reactions whose rate the host sets
 * (PHOTOLYSIS, FIRST_ORDER_LOSS, EMISSION, WET_DEPOSITION) get the ids
 * 1, 2, ... in mechanism order, representations the ids 1, 2, ... in order.
 * Other representation types and sub-models are rejected.  Then call
 * solver_initialize (tolerances from camp_b200_json_tolerances) and
 * solver_run.  NULL on error. */
void *camp_b200_solver_from_json(const char *const *files, int n_files, int n_cells);
int camp_b200_n_state_var(void *solver_data);
/* name of state variable i into buf (NUL-terminated, truncated to buf_len);
 * returns the full length, or -1 (no JSON layout or i out of range) */
int camp_b200_state_name(void *solver_data, int i, char *buf, int buf_len);
/* per-state-variable absolute tolerances and the relative tolerance read
 * from the JSON files (defaults 1e-14 and 1e-8); -1 without a JSON layout */
int camp_b200_json_tolerances(void *solver_data, double *abs_tol, double *rel_tol);
int camp_b200_get_var_type(void *solver_data, int *out);
int camp_b200_rxn_float_data_size(void *solver_data);
int camp_b200_get_rxn_float_data(void *solver_data, double *out);
/* condensed data of aerosol phase (which 0), representation (which 1) or
 * sub-model (which 2; ints without the type slot) `index` as added
 * (aero_phase_add_condensed_data / aero_rep_add_condensed_data /
 * sub_model_add_condensed_data; a representation's element counts are
 * written at solver_initialize): sizes into n_int / n_float and, where
 * non-NULL, the arrays; -1 for a bad index */
int camp_b200_get_aero_data(void *solver_data, int which, int index, int *n_int,
                            int *n_float, int *ints, double *floats);

/* ---------------------------------------------------------------------- */
/* Debug: finite-difference audit of the analytic Jacobian                  */
/* ---------------------------------------------------------------------- */

/* replaces check_Jac (src/camp_solver.c:1146-1257, CAMP_DEBUG builds): for
 * n_cells states (host buffers) and the photolysis rates set for those cells,
 * compares every solver-Jacobian element at step size h with forward
 * differences of f over steps x_j * 10^-12 .. 10^0 of its column's
 * concentration (columns below 1e-30 skipped); an element passes at the
 * first step where |J - FD| < abs_tol or the relative difference < rel_tol
 * (the reference uses 1e-9 and 1e-4).  Per cell: n_failed = elements that
 * never passed (-1 when f or J fails at the state), worst_rel = their
 * largest best-step relative difference.  Returns the total of failed
 * elements, or -1. */
int camp_b200_check_jac(void *solver_data, const double *state, const double *env,
                        int n_cells, double h, double rel_tol, double abs_tol,
                        double *worst_rel, int *n_failed);

/* No counterpart in the reference (the check the mixed form needs): for
 * n_cells states (host buffers) and the rates set for those cells, solves
 * M = I - h J for a right-hand side of tolerance size (+-(rtol |y| + atol)
 * per species) with M factored in FP32 and in FP64 on the solver's fixed
 * order, and writes per cell the error-weighted RMS difference of the two
 * solutions relative to the FP64 one's (-1 where f, J or a factorization
 * fails at the state).  The mixed form's Newton iteration refines the FP32
 * solves, which needs this well below 1: on cb05cl_ae5 and mod37 without
 * sub-models it stays below 1e-2 at steps of 0.01-1 s (single cells reach
 * 0.4 at a whole 60 s step), on the shipped mod37 configuration it reaches
 * 0.7 at 1 s, where the FP64 form is the one to use.
 * 0 or -1. */
int camp_b200_check_precision(void *solver_data, const double *state, const double *env,
                              int n_cells, double h, double *rel_err);

#ifdef __cplusplus
}
#endif
#endif
