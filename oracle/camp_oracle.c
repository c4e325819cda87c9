/* CPU oracle for the CAMP per-cell chemistry solve (TEST INFRASTRUCTURE).
 * See camp_oracle.h for what is restated from where.  Nothing in the product
 * links this file; it exists to check the CUDA path and to time the CPU
 * baseline. */
#include "camp_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* constants of src/camp_common.h:34-45 */
#define VAR_VARIABLE 1
#define SMALL 1.0e-30
#define TINY 1.0e-60

/* reaction type ids, src/rxn_solver.c:19-35 */
#define T_ARRHENIUS 1
#define T_TROE 2
#define T_CMAQ_H2O2 3
#define T_CMAQ_OH_HNO3 4
#define T_PHOTOLYSIS 5
#define T_FIRST_ORDER_LOSS 12
#define T_EMISSION 13
#define T_WET_DEPOSITION 14
#define T_SIMPOL 10
#define T_HL 6
#define T_AQ 7

/* sub-model type ids, src/sub_model_solver.c:16-18 */
#define SM_ZSR_AEROSOL_WATER 2
#define SM_PDFITE 3

/* types whose packed data is not the NUM_REACT_/NUM_PROD_ layout */
static int species_rate_type(int t) {
  return t == T_FIRST_ORDER_LOSS || t == T_EMISSION || t == T_WET_DEPOSITION;
}

static void *zalloc(size_t n) {
  void *p = calloc(n ? n : 1, 1);
  if (!p) {
    fprintf(stderr, "camp_oracle: out of memory\n");
    exit(EXIT_FAILURE);
  }
  return p;
}

/* ------------------------------------------------------------------------ */
/* Mechanism                                                                 */
/* ------------------------------------------------------------------------ */

typedef struct {
  int type;
  int nr, np;
  int n_int_prop;      /* 2, or 3 for photolysis (RXN_ID) */
  int *ints;           /* points at NUM_REACT_ inside the packed int data */
  const double *fl;    /* packed float data of this reaction */
  int n_float_prop;
  int env_off;
  /* aqueous equilibrium: per phase instance, the water below which the
   * reaction is off (MIN_WATER_ x SMALL_WATER_CONC_, set from the absolute
   * tolerances as update_ids does) */
  double *aq_thr;
} ORxn;

#define R_REACT(r, x) ((r)->ints[(r)->n_int_prop + (x)] - 1)
#define R_PROD(r, x) ((r)->ints[(r)->n_int_prop + (r)->nr + (x)] - 1)
#define R_DERIV_ID(r, x) ((r)->ints[(r)->n_int_prop + (r)->nr + (r)->np + (x)])
#define R_JAC_ID(r, x) \
  ((r)->ints[(r)->n_int_prop + 2 * ((r)->nr + (r)->np) + (x)])
#define R_YIELD(r, x) ((r)->fl[(r)->n_float_prop + (x)])

typedef struct {
  int n;          /* dimension (dependent variables) */
  int nnz;        /* entries of L+U */
  int *perm;      /* pivot k -> original index */
  int *iperm;     /* original index -> pivot position */
  int *rowptr;    /* n+1, rows in pivot order */
  int *colidx;    /* column (pivot order), ascending within a row */
  int *diag;      /* position of the diagonal in each row */
  int *a_to_lu;   /* solver CSC element -> LU position */
} LUSym;

struct OracleMech {
  int n_state, n_dep, n_rxn, n_added;
  int *var_type;
  int *int_data, int_size, int_cap;
  double *float_data;
  int float_size, float_cap;
  int n_env;
  ORxn *rx;
  int built;
  int *deriv_ids;
  int n_rxn_jac;
  int *rj_colptr, *rj_rowid;
  int n_solver_jac;
  int *sj_colptr, *sj_rowid;
  int *rxn_to_solver;
  LUSym lu;
  /* aerosol phases and representations, condensed data as added; a cell's
   * representation env parameters (GMD, GSD per section) follow its
   * reaction env parameters in the rxn_env buffer */
  int n_aphase, n_arep, n_aero_env;
  int *aph_int, *aph_ioff, *aph_foff, aph_ilen, aph_flen;
  double *aph_flt;
  int *arep_int, *arep_ioff, *arep_foff, *arep_eoff, *arep_type, arep_ilen, arep_flen;
  double *arep_flt;
  /* sub-models as sub_model_add_condensed_data receives them (ints after
   * the type slot; the JAC ids in them are written at om_build); a cell's
   * sub-model env parameters follow the representation's in rxn_env */
  int n_sub, n_sub_env;
  int *sub_type, *sub_ioff, *sub_foff, *sub_eoff, sub_ilen, sub_flen;
  int *sub_int;
  double *sub_flt;
  /* sub-model parameter Jacobian (src/camp_solver.c:1520-1550): CSC over
   * state variables with the dummy element (0, 0) first */
  int n_param_jac;
  int *pj_colptr, *pj_rowid;
  /* solver Jacobian fold J_solver[s] += J_rxn[r] * J_params[p]
   * (src/camp_solver.c:1636-1681) */
  int n_map;
  int *map_s, *map_r, *map_p;
  /* experiment switches (om_set_experiment); zero = the reference's semantics
   * and this oracle's positivity rule */
  double guard_step;
  int positivity;
};

OracleMech *om_new(int n_state_var, const int *var_type, int n_rxn) {
  OracleMech *m = (OracleMech *)zalloc(sizeof(OracleMech));
  m->n_state = n_state_var;
  m->n_rxn = n_rxn;
  m->var_type = (int *)zalloc(sizeof(int) * n_state_var);
  for (int i = 0; i < n_state_var; ++i) {
    m->var_type[i] = var_type[i];
    if (var_type[i] == VAR_VARIABLE) m->n_dep++;
  }
  m->rx = (ORxn *)zalloc(sizeof(ORxn) * (n_rxn + 1));
  return m;
}

/* Mirrors rxn_add_condensed_data (src/rxn_solver.c:658-700): the type id is
 * stored ahead of the reaction's ints, and the float and env offsets advance
 * by the reaction's sizes. */
int om_add_rxn(OracleMech *m, int type, int n_int, int n_float, int n_env,
               const int *ints, const double *floats) {
  if (m->n_added >= m->n_rxn) return 1;
  if ((type < T_ARRHENIUS || type > T_PHOTOLYSIS) && !species_rate_type(type) &&
      type != T_SIMPOL && type != T_HL && type != T_AQ)
    return 2;
  if (m->int_size + n_int + 1 > m->int_cap) {
    m->int_cap = 2 * (m->int_size + n_int + 1) + 64;
    m->int_data = (int *)realloc(m->int_data, sizeof(int) * m->int_cap);
  }
  if (m->float_size + n_float > m->float_cap) {
    m->float_cap = 2 * (m->float_size + n_float) + 64;
    m->float_data =
        (double *)realloc(m->float_data, sizeof(double) * m->float_cap);
  }
  ORxn *r = &m->rx[m->n_added];
  r->type = type;
  r->env_off = m->n_env;
  /* offsets only for now: the arrays may still move on realloc */
  r->ints = (int *)(size_t)(m->int_size + 1);
  r->fl = (const double *)(size_t)m->float_size;
  m->int_data[m->int_size] = type;
  memcpy(m->int_data + m->int_size + 1, ints, sizeof(int) * n_int);
  memcpy(m->float_data + m->float_size, floats, sizeof(double) * n_float);
  m->int_size += n_int + 1;
  m->float_size += n_float;
  m->n_env += n_env;
  m->n_added++;
  return 0;
}

/* sub_model_add_condensed_data (src/sub_model_solver.c:425-470): the packed
 * ints (after the type) and floats of one sub-model, in priority order */
int om_add_sub_model(OracleMech *m, int type, int n_int, int n_float, int n_env,
                     const int *ints, const double *floats) {
  if (type != SM_ZSR_AEROSOL_WATER && type != SM_PDFITE) return 2;
  const int k = m->n_sub;
  m->sub_type = (int *)realloc(m->sub_type, sizeof(int) * (k + 1));
  m->sub_ioff = (int *)realloc(m->sub_ioff, sizeof(int) * (k + 1));
  m->sub_foff = (int *)realloc(m->sub_foff, sizeof(int) * (k + 1));
  m->sub_eoff = (int *)realloc(m->sub_eoff, sizeof(int) * (k + 1));
  m->sub_int = (int *)realloc(m->sub_int, sizeof(int) * (m->sub_ilen + n_int + 1));
  m->sub_flt = (double *)realloc(m->sub_flt, sizeof(double) * (m->sub_flen + n_float + 1));
  m->sub_type[k] = type;
  m->sub_ioff[k] = m->sub_ilen;
  m->sub_foff[k] = m->sub_flen;
  m->sub_eoff[k] = m->n_sub_env;
  memcpy(m->sub_int + m->sub_ilen, ints, sizeof(int) * n_int);
  memcpy(m->sub_flt + m->sub_flen, floats, sizeof(double) * n_float);
  m->sub_ilen += n_int;
  m->sub_flen += n_float;
  m->n_sub_env += n_env;
  m->n_sub = k + 1;
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Aerosol phases, the modal/binned mass representation (restating           */
/* src/aero_phase_solver.c and src/aero_reps/aero_rep_modal_binned_mass.c)   */
/* ------------------------------------------------------------------------ */

#define AREP_MODAL_BINNED 2
#define SEC_BINNED 1
#define SEC_MODAL 2
/* src/aero_phase_solver.c:14-19 */
#define PH_MIN_MASS 1.0e-25L
#define PH_MIN_MW 0.1L
#define PH_MIN_DENSITY 1800.0L
#define R_GAS 8.314472 /* src/util.h:15 */

static void grow_i(int **p, int need, int *cap) {
  if (need <= *cap) return;
  *cap = 2 * need + 64;
  *p = (int *)realloc(*p, sizeof(int) * (size_t)*cap);
}
static void grow_d(double **p, int need, int *cap) {
  if (need <= *cap) return;
  *cap = 2 * need + 64;
  *p = (double *)realloc(*p, sizeof(double) * (size_t)*cap);
}

/* aero_phase_add_condensed_data (src/aero_phase_solver.c:162-189) */
int om_add_aero_phase(OracleMech *m, int n_int, int n_float, const int *ints,
                      const double *floats) {
  int ic = m->aph_ilen, fc = m->aph_flen;
  int icap = ic, fcap = fc;
  grow_i(&m->aph_int, ic + n_int, &icap);
  grow_d(&m->aph_flt, fc + n_float, &fcap);
  m->aph_ioff = (int *)realloc(m->aph_ioff, sizeof(int) * (m->n_aphase + 1));
  m->aph_foff = (int *)realloc(m->aph_foff, sizeof(int) * (m->n_aphase + 1));
  memcpy(m->aph_int + ic, ints, sizeof(int) * n_int);
  memcpy(m->aph_flt + fc, floats, sizeof(double) * n_float);
  m->aph_ioff[m->n_aphase] = ic;
  m->aph_foff[m->n_aphase] = fc;
  m->aph_ilen += n_int;
  m->aph_flen += n_float;
  m->n_aphase++;
  return 0;
}

/* aero_rep_add_condensed_data (src/aero_rep_solver.c:443-490); only the
 * modal/binned mass representation is restated */
int om_add_aero_rep(OracleMech *m, int type, int n_int, int n_float, int n_env,
                    const int *ints, const double *floats) {
  if (type != AREP_MODAL_BINNED) return 2;
  int ic = m->arep_ilen, fc = m->arep_flen;
  int icap = ic, fcap = fc;
  grow_i(&m->arep_int, ic + n_int, &icap);
  grow_d(&m->arep_flt, fc + n_float, &fcap);
  const int k = m->n_arep;
  m->arep_ioff = (int *)realloc(m->arep_ioff, sizeof(int) * (k + 1));
  m->arep_foff = (int *)realloc(m->arep_foff, sizeof(int) * (k + 1));
  m->arep_eoff = (int *)realloc(m->arep_eoff, sizeof(int) * (k + 1));
  m->arep_type = (int *)realloc(m->arep_type, sizeof(int) * (k + 1));
  memcpy(m->arep_int + ic, ints, sizeof(int) * n_int);
  memcpy(m->arep_flt + fc, floats, sizeof(double) * n_float);
  m->arep_ioff[k] = ic;
  m->arep_foff[k] = fc;
  m->arep_eoff[k] = m->n_aero_env;
  m->arep_type[k] = type;
  m->arep_ilen += n_int;
  m->arep_flen += n_float;
  m->n_aero_env += n_env;
  m->n_arep++;
  return 0;
}

/* one aerosol phase: species count, types, MW and density */
typedef struct {
  int n;
  const int *type;
  const double *mw, *dens;
} APh;

static APh aphase(const OracleMech *m, int p) {
  const int *I = m->aph_int + m->aph_ioff[p];
  const double *F = m->aph_flt + m->aph_foff[p];
  APh a = {I[0], I + 1, F, F + I[0]};
  return a;
}

static int counts_in_mass(int t) { return t == 1 || t == 2 || t == 3; }

/* aero_phase_get_mass__kg_m3 (src/aero_phase_solver.c:88-117) */
static void aph_mass(APh a, const double *y, double *mass, double *mw, double *dmass,
                     double *dmw) {
  long double lm = PH_MIN_MASS, mol = PH_MIN_MASS / PH_MIN_MW;
  int k = 0;
  for (int i = 0; i < a.n; ++i) {
    if (!counts_in_mass(a.type[i])) continue;
    lm += y[i];
    mol += y[i] / (long double)a.mw[i];
    if (dmass) dmass[k] = 1.0L;
    if (dmw) dmw[k] = 1.0L / a.mw[i];
    ++k;
  }
  *mw = (double)lm / mol;
  if (dmw)
    for (int j = 0; j < k; ++j) dmw[j] = (mol - dmw[j] * lm) / (mol * mol);
  *mass = (double)lm;
}

/* aero_phase_get_volume__m3_m3 (src/aero_phase_solver.c:130-147) */
static void aph_volume(APh a, const double *y, double *vol, double *dvol) {
  *vol = PH_MIN_MASS / PH_MIN_DENSITY;
  int k = 0;
  for (int i = 0; i < a.n; ++i) {
    if (!counts_in_mass(a.type[i])) continue;
    *vol += y[i] / a.dens[i];
    if (dvol) dvol[k++] = 1.0 / a.dens[i];
  }
}

/* one modal/binned representation and a cell's env parameters */
typedef struct {
  int ns;
  int *I; /* mutable: the element counts are written at registration */
  const double *F;
  const double *env; /* GMD[ns], GSD[ns] */
} ARep;

static ARep arep(const OracleMech *m, int r, const double *rxn_env) {
  ARep a;
  a.I = m->arep_int + m->arep_ioff[r];
  a.F = m->arep_flt + m->arep_foff[r];
  a.ns = a.I[0];
  a.env = rxn_env ? rxn_env + m->n_env + m->arep_eoff[r] : NULL;
  return a;
}
/* layout of src/aero_reps/aero_rep_modal_binned_mass.c:29-84 */
static int sec_i(ARep a, int x) { return a.I[4 + x] - 1; }
static int sec_f(ARep a, int x) { return a.I[4 + a.ns + x] - 1; }
static int sec_type(ARep a, int x) { return a.I[sec_i(a, x)]; }
static int sec_nb(ARep a, int x) { return a.I[sec_i(a, x) + 1]; }
static int sec_np(ARep a, int x) { return a.I[sec_i(a, x) + 2]; }
static int ph_state(ARep a, int x, int y, int b) {
  return a.I[sec_i(a, x) + 3 + b * sec_np(a, x) + y] - 1;
}
static int ph_model(ARep a, int x, int y, int b) {
  return a.I[sec_i(a, x) + 3 + sec_nb(a, x) * sec_np(a, x) + b * sec_np(a, x) + y] - 1;
}
static int *ph_njac(ARep a, int x, int y, int b) {
  return &a.I[sec_i(a, x) + 3 + 2 * sec_nb(a, x) * sec_np(a, x) + b * sec_np(a, x) + y];
}

/* The C functions find a phase instance by walking sections, then bins,
 * then the phases of a bin (src/aero_reps/aero_rep_modal_binned_mass.c:
 * 300-330, 462-505): instance idx -> (section, bin, phase). */
static int arep_locate(ARep a, int idx, int *x, int *b, int *y) {
  for (int s = 0; s < a.ns; ++s)
    for (int k = 0; k < sec_nb(a, s); ++k) {
      if (idx < sec_np(a, s)) {
        *x = s;
        *b = k;
        *y = idx;
        return 1;
      }
      idx -= sec_np(a, s);
    }
  return 0;
}

/* effective radius [m]: modes from GMD/GSD (the update-data formula,
 * :640-645), bins the bin radius; no state dependence */
static double arep_radius(ARep a, int x, int b) {
  if (sec_type(a, x) == SEC_MODAL) {
    double ln_gsd = log(a.env[a.ns + x]);
    return a.env[x] / 2.0 * exp(5.0 * ln_gsd * ln_gsd / 2.0);
  }
  return a.F[sec_f(a, x) + 3 * b + 2];
}

/* number concentration [# m-3] of a mode / bin and, if nconc_d, its partial
 * derivatives over the mass species of all phases of the mode / bin
 * (:176-236, :340-380) */
static double arep_number(const OracleMech *m, ARep a, int x, int b, const double *state,
                          double *nconc_d) {
  double volume = 0.0;
  double *d = nconc_d;
  for (int y = 0; y < sec_np(a, x); ++y) {
    APh ph = aphase(m, ph_model(a, x, y, b));
    double pv = 0.0;
    aph_volume(ph, state + ph_state(a, x, y, b), &pv, d);
    volume += pv;
    if (d) {
      int k = 0;
      for (int i = 0; i < ph.n; ++i) k += counts_in_mass(ph.type[i]);
      d += k;
    }
  }
  double n;
  if (sec_type(a, x) == SEC_MODAL) {
    const double gmd = a.env[x], gsd = a.env[a.ns + x];
    n = volume * 6.0 / (M_PI * pow(gmd, 3) * exp(9.0 / 2.0 * pow(log(gsd), 2)));
    if (nconc_d) {
      const double f = 6.0 / (M_PI * pow(gmd, 3) * exp(9.0 / 2.0 * pow(log(gsd), 2)));
      for (double *q = nconc_d; q < d; ++q) *q *= f;
    }
  } else {
    const double dp = a.F[sec_f(a, x) + 3 * b];
    n = volume * 3.0 / (4.0 * M_PI) / pow(dp / 2.0, 3);
    if (nconc_d) {
      const double f = 3.0 / (4.0 * M_PI) / pow(dp / 2.0, 3);
      for (double *q = nconc_d; q < d; ++q) *q *= f;
    }
  }
  return n;
}

/* mass [kg m-3] and average MW [kg mol-1] of phase y of a mode / bin, with
 * their partials over all the mode's / bin's mass species (zero for the
 * other phases, :462-560) */
static void arep_phase_mass(const OracleMech *m, ARep a, int x, int b, int y0,
                            const double *state, double *mass, double *mw, double *dmass,
                            double *dmw) {
  int off = 0;
  for (int y = 0; y < sec_np(a, x); ++y) {
    APh ph = aphase(m, ph_model(a, x, y, b));
    int k = 0;
    for (int i = 0; i < ph.n; ++i) k += counts_in_mass(ph.type[i]);
    if (y == y0) {
      aph_mass(ph, state + ph_state(a, x, y, b), mass, mw, dmass ? dmass + off : NULL,
               dmw ? dmw + off : NULL);
    } else {
      for (int j = 0; j < k; ++j) {
        if (dmass) dmass[off + j] = 0.0;
        if (dmw) dmw[off + j] = 0.0;
      }
    }
    off += k;
  }
}

/* GMD (what 0) or GSD (what 1) of section x of representation r in one
 * cell's env buffer, as the GMD/GSD update data set them
 * (src/aero_reps/aero_rep_modal_binned_mass.c:602-650) */
int om_set_aero_env(const OracleMech *m, double *rxn_env, int rep, int section, int what,
                    double value) {
  if (rep < 0 || rep >= m->n_arep) return 0;
  ARep a = arep(m, rep, rxn_env);
  if (section < 0 || section >= a.ns || sec_type(a, section) != SEC_MODAL) return 0;
  rxn_env[m->n_env + m->arep_eoff[rep] + what * a.ns + section] = value;
  return 1;
}

/* --- SIMPOL phase transfer (src/rxns/rxn_SIMPOL_phase_transfer.c) -------- */
/* packed layout of :37-78 */
typedef struct {
  int n;
  int *I;
  const double *F;
} SIM;
static SIM simpol(const ORxn *r) {
  SIM s = {r->ints[0], r->ints, r->fl};
  return s;
}
static int sim_gas(SIM s) { return s.I[1] - 1; }
static int sim_aero(SIM s, int x) { return s.I[2 + x] - 1; }
static int sim_act(SIM s, int x) { return s.I[2 + s.n + x] - 1; }
static int sim_phase(SIM s, int x) { return s.I[2 + 2 * s.n + x] - 1; }
static int sim_rep(SIM s, int x) { return s.I[2 + 3 * s.n + x] - 1; }
static int *sim_deriv(SIM s, int x) { return &s.I[2 + 4 * s.n + x]; }
static int *sim_gas_act_jac(SIM s, int x) { return &s.I[3 + 5 * s.n + x]; }
static int *sim_aero_act_jac(SIM s, int x) { return &s.I[3 + 6 * s.n + x]; }
static int *sim_jac(SIM s, int x) { return &s.I[3 + 7 * s.n + x]; }
static int sim_iloc(SIM s, int x) { return s.I[4 + 10 * s.n + x] - 1; }
static int sim_nelem(SIM s, int x) { return s.I[sim_iloc(s, x)]; }
static int *sim_phase_jac(SIM s, int x, int set, int e) {
  return &s.I[sim_iloc(s, x) + 1 + set * sim_nelem(s, x) + e];
}

/* transition-regime condensation rate constant and its radius derivative
 * (src/util.h:69-161, Fuchs-Sutugin) */
static double fs_factor(double mfp, double r, double alpha) {
  double kn = mfp / r;
  return (0.75 * alpha * (1.0 + kn)) / (kn * kn + (1.0 + 0.283 * alpha) * kn + 0.75 * alpha);
}
static double fs_factor_dr(double mfp, double r, double alpha) {
  double kn = mfp / r;
  return (0.75 * alpha * mfp * (kn * kn + 2.0 * kn + 1.0 + (0.283 - 0.75) * alpha)) /
         pow(r * (kn * kn + (1.0 + 0.283 * alpha) * kn + 0.75 * alpha), 2);
}
static double cond_k(double D, double mfp, double r, double alpha) {
  return 4.0 * M_PI * r * D * fs_factor(mfp, r, alpha);
}
static double cond_k_dr(double D, double mfp, double r, double alpha) {
  return 4.0 * M_PI * D * (fs_factor(mfp, r, alpha) + r * fs_factor_dr(mfp, r, alpha));
}

/* rate constants of one SIMPOL reaction (:220-262): MFP, alpha, K_eq and
 * the kg m-3 -> ppm factor */
static void simpol_env(const ORxn *r, double T, double P, double *k) {
  const double *f = r->fl;
  k[1] = 0.1;
  if (f[0] != 0.0 || f[1] != 0.0) {
    double del_g = f[0] - T * f[1];
    k[1] = exp(-del_g / (R_GAS * T));
    k[1] = k[1] / (1.0 + k[1]);
  }
  k[0] = 3.0 * f[2] / sqrt(8.0 * R_GAS * T / (M_PI * f[9]));
  double vp = f[4] / T + f[5] + f[6] * T + f[7] * log(T);
  vp = 101325.0 * pow(10, vp);
  k[3] = f[8] * T / P;
  k[2] = vp / P / f[9] * 1.0e6;
}

/* --- HL phase transfer (src/rxns/rxn_HL_phase_transfer.c) --------------- */
/* packed layout of :29-63 */
typedef struct {
  int n;
  int *I;
  const double *F;
} HLV;
static HLV hlv(const ORxn *r) {
  HLV s = {r->ints[0], r->ints, r->fl};
  return s;
}
static int hl_gas(HLV s) { return s.I[1] - 1; }
static int *hl_deriv(HLV s, int x) { return &s.I[2 + x]; }
static int *hl_jac(HLV s, int x) { return &s.I[3 + s.n + x]; }
static int hl_iloc(HLV s, int x) { return s.I[4 + 6 * s.n + x] - 1; }
static int hl_aero(HLV s, int x) { return s.I[hl_iloc(s, x)] - 1; }
static int hl_water(HLV s, int x) { return s.I[hl_iloc(s, x) + 1] - 1; }
static int hl_phase(HLV s, int x) { return s.I[hl_iloc(s, x) + 2] - 1; }
static int hl_rep(HLV s, int x) { return s.I[hl_iloc(s, x) + 3] - 1; }
static int hl_nelem(HLV s, int x) { return s.I[hl_iloc(s, x) + 4]; }
static int *hl_phase_jac(HLV s, int x, int set, int e) {
  return &s.I[hl_iloc(s, x) + 5 + set * hl_nelem(s, x) + e];
}

/* rate constants of one HL reaction (:209-247): MFP, alpha, the Henry's law
 * equilibrium constant in kg_x / kg_H2O / ppm and the kg m-3 -> ppm factor */
static void hl_env(const ORxn *r, double T, double P, double *k) {
  const double *f = r->fl;
  k[1] = 0.1;
  if (f[0] != 0.0 || f[1] != 0.0) {
    double del_g = f[0] - T * f[1];
    k[1] = exp(-del_g / (R_GAS * T));
    k[1] = k[1] / (1.0 + k[1]);
  }
  k[0] = 3.0 * f[2] / sqrt(8.0 * R_GAS * T / (M_PI * f[7]));
  if (f[5] == 0.0)
    k[2] = f[4] * P * 1.0e-6 * f[7];
  else
    k[2] = f[4] * P * 1.0e-6 * exp(f[5] * (1.0 / T - 1.0 / 298.0)) * f[7];
  k[3] = f[6] * T / P;
}

/* --- aqueous equilibrium (src/rxns/rxn_aqueous_equilibrium.c) ---------- */
/* packed layout of :27-56 */
#define AQ_MIN_WATER 1.0e-4 /* :24 */
typedef struct {
  int nr, np, P;
  int *I;
  const double *F;
} AQV;
static AQV aqv(const ORxn *r) {
  AQV q = {r->ints[0], r->ints[1], r->ints[2], r->ints, r->fl};
  return q;
}
static int aq_react(AQV q, int x) { return q.I[3 + x] - 1; }
static int aq_prod(AQV q, int x) { return q.I[3 + q.nr * q.P + x] - 1; }
static int aq_water(AQV q, int x) { return q.I[3 + (q.nr + q.np) * q.P + x] - 1; }
static int aq_act(AQV q, int x) { return q.I[3 + (q.nr + q.np + 1) * q.P + x] - 1; }
static int *aq_deriv(AQV q, int x) { return &q.I[3 + (q.nr + q.np + 2) * q.P + x]; }
static int *aq_jac(AQV q, int x) { return &q.I[3 + (2 * (q.nr + q.np) + 2) * q.P + x]; }
static double aq_m2m(AQV q, int x) { return q.F[5 + x]; }

/* SMALL_WATER_CONC_ = abs_tol[water] / 10 (:222-227), times MIN_WATER_ */
static void aq_thresholds(const OracleMech *m, const double *abs_tol) {
  for (int i = 0; i < m->n_rxn; ++i) {
    const ORxn *r = &m->rx[i];
    if (r->type != T_AQ) continue;
    AQV q = aqv(r);
    for (int p = 0; p < q.P; ++p)
      r->aq_thr[p] = AQ_MIN_WATER * (abs_tol ? abs_tol[aq_water(q, p)] / 10.0 : 0.0);
  }
}

/* --- Jacobian element registry (restates src/Jacobian.c:105-214) -------- */
typedef struct {
  int n;
  int *cnt, *cap;
  int **rows;
  int *colptr, *rowid, nnz;
} JacReg;

static void jr_init(JacReg *j, int n) {
  j->n = n;
  j->cnt = (int *)zalloc(sizeof(int) * n);
  j->cap = (int *)zalloc(sizeof(int) * n);
  j->rows = (int **)zalloc(sizeof(int *) * n);
  j->colptr = NULL;
  j->rowid = NULL;
  j->nnz = 0;
}
/* a (dep, ind) pair is kept once per column */
static void jr_register(JacReg *j, int dep, int ind) {
  for (int i = 0; i < j->cnt[ind]; ++i)
    if (j->rows[ind][i] == dep) return;
  if (j->cnt[ind] == j->cap[ind]) {
    j->cap[ind] = j->cap[ind] ? 2 * j->cap[ind] : 8;
    j->rows[ind] = (int *)realloc(j->rows[ind], sizeof(int) * j->cap[ind]);
  }
  j->rows[ind][j->cnt[ind]++] = dep;
}
static int cmp_int(const void *a, const void *b) {
  int x = *(const int *)a, y = *(const int *)b;
  return (x > y) - (x < y);
}
/* rows sorted ascending within each column, columns in index order */
static void jr_build(JacReg *j) {
  j->nnz = 0;
  for (int c = 0; c < j->n; ++c) {
    qsort(j->rows[c], (size_t)j->cnt[c], sizeof(int), cmp_int);
    j->nnz += j->cnt[c];
  }
  j->colptr = (int *)zalloc(sizeof(int) * (j->n + 1));
  j->rowid = (int *)zalloc(sizeof(int) * (j->nnz + 1));
  int e = 0;
  for (int c = 0; c < j->n; ++c) {
    j->colptr[c] = e;
    for (int i = 0; i < j->cnt[c]; ++i) j->rowid[e++] = j->rows[c][i];
    free(j->rows[c]);
  }
  j->colptr[j->n] = e;
  free(j->rows);
  free(j->cnt);
  free(j->cap);
  j->rows = NULL;
  j->cnt = j->cap = NULL;
}
static int jr_elem_id(const int *colptr, const int *rowid, int dep, int ind) {
  for (int e = colptr[ind]; e < colptr[ind + 1]; ++e)
    if (rowid[e] == dep) return e;
  return -1;
}

/* --- sub-models: ZSR aerosol water and PD-FiTE activity ----------------- */
/* Packed layouts (ints after the type slot) of
 * src/sub_models/sub_model_ZSR_aerosol_water.c:27-71 and
 * src/sub_models/sub_model_PDFiTE.c:21-64; both start with NUM_PHASE,
 * GAS_WATER_ID (1-based), NUM_ION_PAIR, INT_DATA_SIZE, FLOAT_DATA_SIZE, then
 * the phase water / first-species ids (1-based) and the per-ion-pair int and
 * float locations (1-based).  Species ids of an ion pair are relative to the
 * phase's first state id. */
typedef struct {
  int *I;
  const double *F;
  int np, gw, npair;
} SubV;

static SubV subv(const OracleMech *m, int k) {
  SubV s;
  s.I = m->sub_int + m->sub_ioff[k];
  s.F = m->sub_flt + m->sub_foff[k];
  s.np = s.I[0];
  s.gw = s.I[1] - 1;
  s.npair = s.I[2];
  return s;
}
static int sv_phase(SubV s, int p) { return s.I[5 + p] - 1; }
static int sv_il(SubV s, int x) { return s.I[5 + s.np + x] - 1; }
static int sv_fl(SubV s, int x) { return s.I[5 + s.np + s.npair + x] - 1; }
/* ZSR, per ion pair: type 1 = Jacobson et al. (1996), 2 = EQSAM */
#define ZSR_JACOBSON 1
#define ZSR_EQSAM 2
static int zsr_type(SubV s, int x) { return s.I[sv_il(s, x)]; }
static int zj_ncat(SubV s, int x) { return s.I[sv_il(s, x) + 1]; }
static int zj_nan(SubV s, int x) { return s.I[sv_il(s, x) + 2]; }
static int zj_cat(SubV s, int x) { return s.I[sv_il(s, x) + 3]; }
static int zj_an(SubV s, int x) { return s.I[sv_il(s, x) + 4]; }
static int zj_ny(SubV s, int x) { return s.I[sv_il(s, x) + 5]; }
static int *zj_gw_jac(SubV s, int p, int x) { return &s.I[sv_il(s, x) + 6 + p]; }
static int *zj_cat_jac(SubV s, int p, int x) { return &s.I[sv_il(s, x) + 6 + s.np + p]; }
static int *zj_an_jac(SubV s, int p, int x) { return &s.I[sv_il(s, x) + 6 + 2 * s.np + p]; }
static double zj_low_rh(SubV s, int x) { return s.F[sv_fl(s, x)]; }
static double zj_cat_mw(SubV s, int x) { return s.F[sv_fl(s, x) + 1]; }
static double zj_an_mw(SubV s, int x) { return s.F[sv_fl(s, x) + 2]; }
static double zj_y(SubV s, int x, int k) { return s.F[sv_fl(s, x) + 3 + k]; }
static int ze_nion(SubV s, int x) { return s.I[sv_il(s, x) + 1]; }
static int *ze_gw_jac(SubV s, int p, int x) { return &s.I[sv_il(s, x) + 2 + p]; }
static int ze_ion(SubV s, int x, int k) { return s.I[sv_il(s, x) + 2 + s.np + k]; }
static int *ze_ion_jac(SubV s, int p, int x, int k) {
  return &s.I[sv_il(s, x) + 2 + s.np + ze_nion(s, x) + k * s.np + p];
}
static double ze_nw(SubV s, int x) { return s.F[sv_fl(s, x)]; }
static double ze_zw(SubV s, int x) { return s.F[sv_fl(s, x) + 1]; }
static double ze_pair_mw(SubV s, int x) { return s.F[sv_fl(s, x) + 2]; }
static double ze_ion_mw(SubV s, int x, int k) { return s.F[sv_fl(s, x) + 3 + k]; }
/* PD-FiTE, per ion pair */
static int pd_act(SubV s, int x) { return s.I[sv_il(s, x)]; }
static int pd_ncat(SubV s, int x) { return s.I[sv_il(s, x) + 1]; }
static int pd_nan(SubV s, int x) { return s.I[sv_il(s, x) + 2]; }
static int pd_cat(SubV s, int x) { return s.I[sv_il(s, x) + 3]; }
static int pd_an(SubV s, int x) { return s.I[sv_il(s, x) + 4]; }
static int pd_ninter(SubV s, int x) { return s.I[sv_il(s, x) + 5]; }
static int *pd_w_jac(SubV s, int p, int x) { return &s.I[sv_il(s, x) + 6 + p]; }
static int *pd_cat_jac(SubV s, int p, int x, int y) {
  return &s.I[sv_il(s, x) + 6 + s.np + p * s.npair + y];
}
static int *pd_an_jac(SubV s, int p, int x, int y) {
  return &s.I[sv_il(s, x) + 6 + (1 + s.npair) * s.np + p * s.npair + y];
}
static int pd_nb(SubV s, int x, int y) {
  return s.I[sv_il(s, x) + 6 + (1 + 2 * s.npair) * s.np + y];
}
static int pd_inter_pair(SubV s, int x, int y) {
  return s.I[sv_il(s, x) + 6 + (1 + 2 * s.npair) * s.np + pd_ninter(s, x) + y] - 1;
}
static int pd_inter_loc(SubV s, int x, int y) {
  return s.I[sv_il(s, x) + 6 + (1 + 2 * s.npair) * s.np + 2 * pd_ninter(s, x) + y] - 1;
}
static double pd_cat_mw(SubV s, int x) { return s.F[sv_fl(s, x)]; }
static double pd_an_mw(SubV s, int x) { return s.F[sv_fl(s, x) + 1]; }
static double pd_min_rh(SubV s, int x, int y) { return s.F[pd_inter_loc(s, x, y)]; }
static double pd_max_rh(SubV s, int x, int y) { return s.F[pd_inter_loc(s, x, y) + 1]; }
static double pd_b(SubV s, int x, int y, int z) { return s.F[pd_inter_loc(s, x, y) + 2 + z]; }
/* an interaction applies in (min RH, max RH], or [0, max RH] at a_w = 0
 * (src/sub_models/sub_model_PDFiTE.c:218-224) */
static int pd_in_range(SubV s, int x, int y, double a_w) {
  const double lo = pd_min_rh(s, x, y), hi = pd_max_rh(s, x, y);
  return !((a_w <= lo || a_w > hi) && !(a_w <= 0.0 && lo <= 0.0));
}

static const double *sub_env(const OracleMech *m, const double *rxn_env, int k) {
  return rxn_env + m->n_env + m->n_aero_env + m->sub_eoff[k];
}

/* PPM_TO_RH_ from T and P, the MOSAIC water vapour pressure fit
 * (src/sub_models/sub_model_ZSR_aerosol_water.c:198-214; the PD-FiTE
 * sub-model computes the same) */
static double ppm_to_rh(double T, double P) {
  double a = 1.0 - 373.15 / T;
  a = (((-0.1299 * a - 0.6445) * a - 1.976) * a + 13.3185) * a;
  const double water_vp = 101325.0 * exp(a);
  return P / water_vp / 1.0e6;
}

/* Jacobson molality polynomial value (squared in the water sum) and its
 * derivative in a_w */
static void zsr_calc(SubV s, const double *e, double *state) {
  const long double a_w = e[0] * state[s.gw];
  for (int p = 0; p < s.np; ++p) {
    const int w = sv_phase(s, p);
    long double water = 1.0e-30L; /* MINIMUM_WATER_MASS_ */
    for (int x = 0; x < s.npair; ++x) {
      if (zsr_type(s, x) == ZSR_JACOBSON) {
        const long double j_aw = a_w > zj_low_rh(s, x) ? a_w : zj_low_rh(s, x);
        long double molal = 0.0;
        for (int k = 0; k < zj_ny(s, x); ++k) molal += zj_y(s, x, k) * pow((double)j_aw, k);
        molal *= molal;
        const long double cat = state[w + zj_cat(s, x)] / zj_ncat(s, x) / zj_cat_mw(s, x) / 1000.0;
        const long double an = state[w + zj_an(s, x)] / zj_nan(s, x) / zj_an_mw(s, x) / 1000.0;
        /* smooth minimum of the two ion concentrations, alpha = -100 */
        const long double ec = exp((double)(-100.0 * cat)), ea = exp((double)(-100.0 * an));
        const long double conc = (cat * ec + an * ea) / (ec + ea);
        water += conc / molal * 1000.0;
      } else if (zsr_type(s, x) == ZSR_EQSAM) {
        long double e_aw = a_w > 0.99 ? 0.99 : a_w;
        e_aw = e_aw < 0.001 ? 0.001 : e_aw;
        long double molal =
            ze_nw(s, x) * 55.51 * 18.01 / ze_pair_mw(s, x) / 1000.0 * (1.0 / e_aw - 1.0);
        molal = pow((double)molal, ze_zw(s, x));
        for (int k = 0; k < ze_nion(s, x); ++k) {
          long double c = state[w + ze_ion(s, x, k)];
          c = c > 0.0 ? c : 0.0;
          water += c / ze_ion_mw(s, x, k) / molal;
        }
      }
    }
    state[w] = (double)water;
  }
}

/* src/sub_models/sub_model_ZSR_aerosol_water.c:318-437 */
static void zsr_jac(SubV s, const double *e, const double *state, double *JP) {
  const long double a_w = e[0] * state[s.gw];
  const long double daw = e[0];
  for (int p = 0; p < s.np; ++p) {
    const int w = sv_phase(s, p);
    for (int x = 0; x < s.npair; ++x) {
      if (zsr_type(s, x) == ZSR_JACOBSON) {
        const long double j_aw = a_w > zj_low_rh(s, x) ? a_w : zj_low_rh(s, x);
        const long double dj = a_w > zj_low_rh(s, x) ? daw : 0.0;
        long double molal = zj_y(s, x, 0), dmolal = 0.0;
        for (int k = 1; k < zj_ny(s, x); ++k) {
          molal += zj_y(s, x, k) * pow((double)j_aw, k);
          dmolal += zj_y(s, x, k) * k * pow((double)j_aw, k - 1);
        }
        dmolal *= dj;
        const long double cat = state[w + zj_cat(s, x)] / zj_ncat(s, x) / zj_cat_mw(s, x) / 1000.0;
        const long double dcat = 1.0 / zj_ncat(s, x) / zj_cat_mw(s, x) / 1000.0;
        const long double an = state[w + zj_an(s, x)] / zj_nan(s, x) / zj_an_mw(s, x) / 1000.0;
        const long double dan = 1.0 / zj_nan(s, x) / zj_an_mw(s, x) / 1000.0;
        const long double ec = exp((double)(-100.0 * cat)), ea = exp((double)(-100.0 * an));
        const long double conc = (cat * ec + an * ea) / (ec + ea);
        const long double den = (ec + ea) * (ec + ea);
        const long double dc_dcat = (ec * ec + ec * ea * (1.0 + 100.0 * an - 100.0 * cat)) / den;
        const long double dc_dan = (ea * ea + ec * ea * (1.0 + 100.0 * cat - 100.0 * an)) / den;
        JP[*zj_gw_jac(s, p, x)] += -2.0 * conc / pow((double)molal, 3) * 1000.0 * dmolal;
        JP[*zj_an_jac(s, p, x)] += 1.0 / pow((double)molal, 2) * 1000.0 * dc_dan * dan;
        JP[*zj_cat_jac(s, p, x)] += 1.0 / pow((double)molal, 2) * 1000.0 * dc_dcat * dcat;
      } else if (zsr_type(s, x) == ZSR_EQSAM) {
        long double e_aw = a_w > 0.99 ? 0.99 : a_w;
        e_aw = e_aw < 0.001 ? 0.001 : e_aw;
        long double de = a_w > 0.99 ? 0.0 : daw;
        de = a_w < 0.001 ? 0.0 : de;
        const long double pre = ze_nw(s, x) * 55.51 * 18.01 / ze_pair_mw(s, x) / 1000.0;
        long double molal = pre * (1.0 / e_aw - 1.0);
        long double dmolal = -pre / pow((double)e_aw, 2) * de;
        dmolal = ze_zw(s, x) * pow((double)molal, ze_zw(s, x) - 1.0) * dmolal;
        molal = pow((double)molal, ze_zw(s, x));
        for (int k = 0; k < ze_nion(s, x); ++k) {
          long double c = state[w + ze_ion(s, x, k)];
          c = c > 0.0 ? c : 0.0;
          const long double dc = c > 0.0 ? 1.0 : 0.0;
          JP[*ze_gw_jac(s, p, x)] += -1.0 * c / ze_ion_mw(s, x, k) / pow((double)molal, 2) * dmolal;
          JP[*ze_ion_jac(s, p, x, k)] += dc / ze_ion_mw(s, x, k) / molal;
        }
      }
    }
  }
}

/* moles of each ion [mol m-3] of phase instance p
 * (src/sub_models/sub_model_PDFiTE.c:183-194) */
static void pd_moles(SubV s, int p, const double *state, double *cn, double *an) {
  const int base = sv_phase(s, p);
  for (int x = 0; x < s.npair; ++x) {
    cn[x] = state[base + pd_cat(s, x)] / pd_cat_mw(s, x) / 1000000.0;
    an[x] = state[base + pd_an(s, x)] / pd_an_mw(s, x) / 1000000.0;
  }
}
static long double pd_omega(SubV s, int x, const double *cn, const double *an) {
  long double omega = 0.0;
  for (int y = 0; y < s.npair; ++y) {
    if (y == x) continue;
    omega += (long double)2.0 * (pd_ncat(s, y) + pd_nan(s, y)) * cn[y] * an[y];
  }
  return omega;
}

/* src/sub_models/sub_model_PDFiTE.c:167-259 */
static void pd_calc(SubV s, const double *e, double *state, double *cn, double *an) {
  long double a_w = e[0] * state[s.gw];
  if (a_w < 0.0) a_w = 0.0;
  if (a_w > 1.0) a_w = 1.0;
  for (int p = 0; p < s.np; ++p) {
    pd_moles(s, p, state, cn, an);
    for (int x = 0; x < s.npair; ++x) {
      if (pd_ninter(s, x) == 0) break;
      const long double omega = pd_omega(s, x, cn, an);
      long double lng = 0.0;
      for (int y = 0; y < pd_ninter(s, x); ++y) {
        if (!pd_in_range(s, x, y, (double)a_w)) continue;
        const int j = pd_inter_pair(s, x, y);
        long double li = 0.0;
        for (int z = 0; z < pd_nb(s, x, y); ++z) li += pd_b(s, x, y, z) * pow((double)a_w, z);
        if (j == x)
          lng += li;
        else if (omega > 0.0)
          lng += li * cn[j] * an[j] / omega;
      }
      state[sv_phase(s, p) + pd_act(s, x)] = exp((double)lng);
    }
  }
}

/* src/sub_models/sub_model_PDFiTE.c:273-432; a_w is a double here, as in
 * the reference's Jacobian */
static void pd_jac(SubV s, const double *e, const double *state, double *JP, double *cn,
                   double *an) {
  double a_w = e[0] * state[s.gw];
  if (a_w < 0.0) a_w = 0.0;
  if (a_w > 1.0) a_w = 1.0;
  for (int p = 0; p < s.np; ++p) {
    pd_moles(s, p, state, cn, an);
    for (int x = 0; x < s.npair; ++x) {
      if (pd_ninter(s, x) == 0) break;
      const long double omega = pd_omega(s, x, cn, an);
      long double lng = 0.0;
      for (int y = 0; y < pd_ninter(s, x); ++y) {
        if (!pd_in_range(s, x, y, a_w)) continue;
        const int j = pd_inter_pair(s, x, y);
        long double li = 0.0;
        for (int z = 0; z < pd_nb(s, x, y); ++z) li += pd_b(s, x, y, z) * pow(a_w, z);
        if (j == x)
          lng += li;
        else if (omega > 0.0)
          lng += li * cn[j] * an[j] / omega;
      }
      const long double g = exp((double)lng);
      for (int y = 0; y < pd_ninter(s, x); ++y) {
        if (!pd_in_range(s, x, y, a_w)) continue;
        const int j = pd_inter_pair(s, x, y);
        long double li = pd_b(s, x, y, 0), dli = 0.0;
        for (int z = 1; z < pd_nb(s, x, y); ++z) {
          li += pd_b(s, x, y, z) * pow(a_w, z);
          dli += pd_b(s, x, y, z) * z * pow(a_w, z - 1);
        }
        dli *= e[0];
        if (j == x) {
          JP[*pd_w_jac(s, p, x)] += g * dli;
        } else if (omega > 0.0) {
          JP[*pd_cat_jac(s, p, x, j)] += g * li * an[j] / pd_cat_mw(s, j) / omega * 1.0e-6;
          JP[*pd_an_jac(s, p, x, j)] += g * li * cn[j] / pd_an_mw(s, j) / omega * 1.0e-6;
          JP[*pd_w_jac(s, p, x)] += g * cn[j] * an[j] / omega * dli;
          for (int k = 0; k < s.npair; ++k) {
            if (k == x) continue;
            JP[*pd_cat_jac(s, p, x, k)] += -g * li * cn[j] * an[j] / (omega * omega) * 2.0 *
                                           (pd_ncat(s, k) + pd_nan(s, k)) * an[k] /
                                           pd_cat_mw(s, k) * 1.0e-6;
            JP[*pd_an_jac(s, p, x, k)] += -g * li * cn[j] * an[j] / (omega * omega) * 2.0 *
                                          (pd_ncat(s, k) + pd_nan(s, k)) * cn[k] /
                                          pd_an_mw(s, k) * 1.0e-6;
          }
        }
      }
    }
  }
}

/* sub_model_calculate (src/sub_model_solver.c:300-333): in priority order,
 * each writes its computed species into the state */
static void sub_calculate(const OracleMech *m, double *state, const double *rxn_env) {
  double cn[64], an[64];
  for (int k = 0; k < m->n_sub; ++k) {
    SubV s = subv(m, k);
    if (m->sub_type[k] == SM_ZSR_AEROSOL_WATER)
      zsr_calc(s, sub_env(m, rxn_env, k), state);
    else
      pd_calc(s, sub_env(m, rxn_env, k), state, cn, an);
  }
}

/* sub_model_get_jac_contrib (src/sub_model_solver.c:341-381) into J_params
 * (zeroed here); element 0 is the fold's unit parameter */
static void sub_jacobian(const OracleMech *m, const double *state, const double *rxn_env,
                         double *JP) {
  double cn[64], an[64];
  for (int i = 0; i < m->n_param_jac; ++i) JP[i] = 0.0;
  for (int k = 0; k < m->n_sub; ++k) {
    SubV s = subv(m, k);
    if (m->sub_type[k] == SM_ZSR_AEROSOL_WATER)
      zsr_jac(s, sub_env(m, rxn_env, k), state, JP);
    else
      pd_jac(s, sub_env(m, rxn_env, k), state, JP, cn, an);
  }
  JP[0] = 1.0;
}

/* the sub-model's parameter Jacobian elements (dep = computed species, ind =
 * the species it is computed from) through a callback; the same walk
 * registers them (get_used_jac_elem) and looks up their ids (update_ids) */
typedef void (*sub_elem_fn)(void *ctx, int dep, int ind, int *id);
static void sub_elements(const OracleMech *m, int k, sub_elem_fn fn, void *ctx) {
  SubV s = subv(m, k);
  for (int p = 0; p < s.np; ++p) {
    const int w = sv_phase(s, p);
    if (m->sub_type[k] == SM_ZSR_AEROSOL_WATER) {
      /* src/sub_models/sub_model_ZSR_aerosol_water.c:81-129, 140-185 */
      fn(ctx, w, s.gw, NULL);
      for (int x = 0; x < s.npair; ++x) {
        if (zsr_type(s, x) == ZSR_JACOBSON) {
          fn(ctx, w, s.gw, zj_gw_jac(s, p, x));
          fn(ctx, w, w + zj_cat(s, x), zj_cat_jac(s, p, x));
          fn(ctx, w, w + zj_an(s, x), zj_an_jac(s, p, x));
        } else if (zsr_type(s, x) == ZSR_EQSAM) {
          fn(ctx, w, s.gw, ze_gw_jac(s, p, x));
          for (int i = 0; i < ze_nion(s, x); ++i)
            fn(ctx, w, w + ze_ion(s, x, i), ze_ion_jac(s, p, x, i));
        }
      }
    } else {
      /* src/sub_models/sub_model_PDFiTE.c:73-130 */
      for (int x = 0; x < s.npair; ++x) {
        const int g = w + pd_act(s, x);
        fn(ctx, g, s.gw, pd_w_jac(s, p, x));
        for (int y = 0; y < s.npair; ++y) {
          fn(ctx, g, w + pd_cat(s, y), pd_cat_jac(s, p, x, y));
          fn(ctx, g, w + pd_an(s, y), pd_an_jac(s, p, x, y));
        }
      }
    }
  }
}
static void sub_register_cb(void *ctx, int dep, int ind, int *id) {
  (void)id;
  jr_register((JacReg *)ctx, dep, ind);
}
typedef struct {
  const int *colptr, *rowid;
} PJLookup;
static void sub_ids_cb(void *ctx, int dep, int ind, int *id) {
  const PJLookup *l = (const PJLookup *)ctx;
  if (id) *id = jr_elem_id(l->colptr, l->rowid, dep, ind);
}

/* --- LU symbolic: Markowitz order over diagonal pivots ------------------- */
static void lu_symbolic(LUSym *lu, int n, const int *colptr, const int *rowid) {
  unsigned char *P = (unsigned char *)zalloc((size_t)n * n);
  for (int c = 0; c < n; ++c)
    for (int e = colptr[c]; e < colptr[c + 1]; ++e) P[rowid[e] * n + c] = 1;
  for (int i = 0; i < n; ++i) P[i * n + i] = 1;
  unsigned char *done = (unsigned char *)zalloc(n);
  lu->n = n;
  lu->perm = (int *)zalloc(sizeof(int) * n);
  lu->iperm = (int *)zalloc(sizeof(int) * n);
  for (int k = 0; k < n; ++k) {
    long best = -1;
    int bi = -1;
    for (int i = 0; i < n; ++i) {
      if (done[i]) continue;
      long r = 0, c = 0;
      for (int j = 0; j < n; ++j) {
        if (done[j]) continue;
        r += P[i * n + j];
        c += P[j * n + i];
      }
      long score = (r - 1) * (c - 1);
      if (best < 0 || score < best) {
        best = score;
        bi = i;
      }
    }
    done[bi] = 1;
    lu->perm[k] = bi;
    lu->iperm[bi] = k;
    /* eliminate bi: fill rows i with P[i][bi] in columns j with P[bi][j] */
    for (int i = 0; i < n; ++i) {
      if (done[i] || !P[i * n + bi]) continue;
      for (int j = 0; j < n; ++j)
        if (!done[j] && P[bi * n + j]) P[i * n + j] = 1;
    }
  }
  /* P now holds the filled pattern in original indices */
  lu->rowptr = (int *)zalloc(sizeof(int) * (n + 1));
  int nnz = 0;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) nnz += P[i * n + j];
  lu->nnz = nnz;
  lu->colidx = (int *)zalloc(sizeof(int) * nnz);
  lu->diag = (int *)zalloc(sizeof(int) * n);
  int e = 0;
  for (int pi = 0; pi < n; ++pi) {
    lu->rowptr[pi] = e;
    int oi = lu->perm[pi];
    for (int pj = 0; pj < n; ++pj) {
      if (!P[oi * n + lu->perm[pj]]) continue;
      if (pj == pi) lu->diag[pi] = e;
      lu->colidx[e++] = pj;
    }
  }
  lu->rowptr[n] = e;
  int annz = colptr[n];
  lu->a_to_lu = (int *)zalloc(sizeof(int) * (annz + 1));
  for (int c = 0; c < n; ++c)
    for (int a = colptr[c]; a < colptr[c + 1]; ++a) {
      int pr = lu->iperm[rowid[a]], pc = lu->iperm[c];
      for (int q = lu->rowptr[pr]; q < lu->rowptr[pr + 1]; ++q)
        if (lu->colidx[q] == pc) {
          lu->a_to_lu[a] = q;
          break;
        }
    }
  free(P);
  free(done);
}

static void lu_free(LUSym *lu) {
  free(lu->perm);
  free(lu->iperm);
  free(lu->rowptr);
  free(lu->colidx);
  free(lu->diag);
  free(lu->a_to_lu);
}

/* The representation's elements for a phase instance: the mass species of
 * every phase of the instance's mode / bin (aero_rep_modal_binned_mass.c:
 * 86-125), flagged in state order; the representation's PHASE_NUM_JAC_ELEM_
 * is written as its get_used_jac_elem writes it. */
static void instance_elements(const OracleMech *m, int rep, int phase, char *flag) {
  memset(flag, 0, (size_t)m->n_state);
  ARep ar = arep(m, rep, NULL);
  int sx, sb, sy;
  if (!arep_locate(ar, phase, &sx, &sb, &sy)) return;
  for (int y = 0; y < sec_np(ar, sx); ++y) {
    APh ph = aphase(m, ph_model(ar, sx, y, sb));
    int k = 0;
    for (int i = 0; i < ph.n; ++i)
      if (counts_in_mass(ph.type[i])) {
        flag[ph_state(ar, sx, y, sb) + i] = 1;
        ++k;
      }
    *ph_njac(ar, sx, y, sb) = k;
  }
}

/* Builds the sparsity as get_jac_init does for a gas-only model
 * (src/camp_solver.c:1440-1683): diagonal plus the reaction elements of
 * every reaction (src/rxns/rxn_arrhenius.c:44-60 and the same loop in the
 * other gas types), then DERIV_ID/JAC_ID (src/rxns/rxn_arrhenius.c:71-91),
 * then the var x var solver Jacobian with its map. */
int om_build(OracleMech *m) {
  if (m->n_added != m->n_rxn) return 1;
  for (int i = 0; i < m->n_rxn; ++i) {
    ORxn *r = &m->rx[i];
    r->ints = m->int_data + (size_t)r->ints;
    r->fl = m->float_data + (size_t)r->fl;
    if (r->type == T_AQ) {
      AQV q = aqv(r);
      r->aq_thr = (double *)zalloc(sizeof(double) * (size_t)(q.P + 1));
      r->nr = r->np = 0;
      r->n_int_prop = 3;
      r->n_float_prop = 5;
      continue;
    }
    if (species_rate_type(r->type) || r->type == T_SIMPOL || r->type == T_HL) {
      /* RXN_ID_ first (host-rate types); the reactant / product fields stay
       * unused */
      r->nr = r->np = 0;
      r->n_int_prop = 0;
      r->n_float_prop = 1;
      continue;
    }
    r->nr = r->ints[0];
    r->np = r->ints[1];
    r->n_int_prop = r->type == T_PHOTOLYSIS ? 3 : 2;
    switch (r->type) {
      case T_ARRHENIUS: r->n_float_prop = 6; break;
      case T_TROE: r->n_float_prop = 10; break;
      case T_CMAQ_H2O2: r->n_float_prop = 7; break;
      case T_CMAQ_OH_HNO3: r->n_float_prop = 11; break;
      default: r->n_float_prop = 1; break;
    }
  }
  int n = m->n_state;
  JacReg rj;
  jr_init(&rj, n);
  for (int i = 0; i < n; ++i) jr_register(&rj, i, i);
  for (int i = 0; i < m->n_rxn; ++i) {
    ORxn *r = &m->rx[i];
    const int *I = r->ints;
    switch (r->type) {
      case T_FIRST_ORDER_LOSS: /* src/rxns/rxn_first_order_loss.c:37-46 */
        jr_register(&rj, I[1] - 1, I[1] - 1);
        continue;
      case T_EMISSION: /* src/rxns/rxn_emission.c:36-42: none */
        continue;
      case T_WET_DEPOSITION: /* src/rxns/rxn_wet_deposition.c:38-49 */
        for (int s = 0; s < I[1]; ++s) jr_register(&rj, I[2 + s] - 1, I[2 + s] - 1);
        continue;
      case T_SIMPOL: { /* src/rxns/rxn_SIMPOL_phase_transfer.c:86-151 */
        SIM sm = simpol(r);
        const int g = sim_gas(sm);
        jr_register(&rj, g, g);
        char *flag = (char *)zalloc((size_t)n);
        for (int x = 0; x < sm.n; ++x) {
          const int a = sim_aero(sm, x);
          jr_register(&rj, a, g);
          jr_register(&rj, g, a);
          jr_register(&rj, a, a);
          if (sim_act(sm, x) > 0) {
            jr_register(&rj, g, sim_act(sm, x));
            jr_register(&rj, a, sim_act(sm, x));
          }
          instance_elements(m, sim_rep(sm, x), sim_phase(sm, x), flag);
          int used = 0;
          for (int e = 0; e < n; ++e) {
            if (!flag[e]) continue;
            jr_register(&rj, g, e);
            jr_register(&rj, a, e);
            *sim_phase_jac(sm, x, 0, used) = e;
            *sim_phase_jac(sm, x, 1, used) = e;
            ++used;
          }
          for (; used < sim_nelem(sm, x); ++used)
            *sim_phase_jac(sm, x, 0, used) = *sim_phase_jac(sm, x, 1, used) = -1;
        }
        free(flag);
        continue;
      }
      case T_AQ: { /* src/rxns/rxn_aqueous_equilibrium.c:70-127 */
        AQV q = aqv(r);
        for (int p = 0; p < q.P; ++p) {
          for (int i = 0; i < q.nr; ++i) {
            const int ind = aq_react(q, p * q.nr + i);
            for (int d = 0; d < q.nr; ++d) jr_register(&rj, aq_react(q, p * q.nr + d), ind);
            for (int d = 0; d < q.np; ++d) jr_register(&rj, aq_prod(q, p * q.np + d), ind);
          }
          for (int i = 0; i < q.np; ++i) {
            const int ind = aq_prod(q, p * q.np + i);
            for (int d = 0; d < q.nr; ++d) jr_register(&rj, aq_react(q, p * q.nr + d), ind);
            for (int d = 0; d < q.np; ++d) jr_register(&rj, aq_prod(q, p * q.np + d), ind);
          }
          for (int d = 0; d < q.nr; ++d) jr_register(&rj, aq_react(q, p * q.nr + d), aq_water(q, p));
          for (int d = 0; d < q.np; ++d) jr_register(&rj, aq_prod(q, p * q.np + d), aq_water(q, p));
          if (aq_act(q, p) < 0) continue;
          for (int d = 0; d < q.nr; ++d) jr_register(&rj, aq_react(q, p * q.nr + d), aq_act(q, p));
          for (int d = 0; d < q.np; ++d) jr_register(&rj, aq_prod(q, p * q.np + d), aq_act(q, p));
        }
        continue;
      }
      case T_HL: { /* src/rxns/rxn_HL_phase_transfer.c:72-138 */
        HLV hl = hlv(r);
        const int g = hl_gas(hl);
        jr_register(&rj, g, g);
        char *flag = (char *)zalloc((size_t)n);
        for (int x = 0; x < hl.n; ++x) {
          const int a = hl_aero(hl, x), w = hl_water(hl, x);
          jr_register(&rj, a, g);
          jr_register(&rj, g, a);
          jr_register(&rj, a, a);
          jr_register(&rj, g, w);
          jr_register(&rj, a, w);
          instance_elements(m, hl_rep(hl, x), hl_phase(hl, x), flag);
          int used = 0;
          for (int e = 0; e < n; ++e) {
            if (!flag[e]) continue;
            jr_register(&rj, g, e);
            jr_register(&rj, a, e);
            *hl_phase_jac(hl, x, 0, used) = e;
            *hl_phase_jac(hl, x, 1, used) = e;
            ++used;
          }
          for (; used < hl_nelem(hl, x); ++used)
            *hl_phase_jac(hl, x, 0, used) = *hl_phase_jac(hl, x, 1, used) = -1;
        }
        free(flag);
        continue;
      }
    }
    for (int ind = 0; ind < r->nr; ++ind) {
      for (int d = 0; d < r->nr; ++d) jr_register(&rj, R_REACT(r, d), R_REACT(r, ind));
      for (int d = 0; d < r->np; ++d) jr_register(&rj, R_PROD(r, d), R_REACT(r, ind));
    }
  }
  jr_build(&rj);
  m->n_rxn_jac = rj.nnz;
  m->rj_colptr = rj.colptr;
  m->rj_rowid = rj.rowid;

  m->deriv_ids = (int *)zalloc(sizeof(int) * n);
  for (int i = 0, d = 0; i < n; ++i)
    m->deriv_ids[i] = m->var_type[i] == VAR_VARIABLE ? d++ : -1;
  for (int i = 0; i < m->n_rxn; ++i) {
    ORxn *r = &m->rx[i];
    int *I = r->ints;
    switch (r->type) {
      case T_FIRST_ORDER_LOSS: /* src/rxns/rxn_first_order_loss.c:56-69 */
        I[2] = m->deriv_ids[I[1] - 1];
        I[3] = jr_elem_id(m->rj_colptr, m->rj_rowid, I[1] - 1, I[1] - 1);
        continue;
      case T_EMISSION: /* src/rxns/rxn_emission.c:52-62 */
        I[2] = m->deriv_ids[I[1] - 1];
        continue;
      case T_WET_DEPOSITION: { /* src/rxns/rxn_wet_deposition.c:59-75 */
        const int ns = I[1];
        for (int s = 0; s < ns; ++s) {
          I[2 + ns + s] = m->deriv_ids[I[2 + s] - 1];
          I[2 + 2 * ns + s] =
              jr_elem_id(m->rj_colptr, m->rj_rowid, I[2 + s] - 1, I[2 + s] - 1);
        }
        continue;
      }
      case T_SIMPOL: { /* src/rxns/rxn_SIMPOL_phase_transfer.c:160-205 */
        SIM sm = simpol(r);
        const int *cp = m->rj_colptr, *ri = m->rj_rowid;
        const int g = sim_gas(sm);
        *sim_deriv(sm, 0) = m->deriv_ids[g];
        for (int x = 0; x < sm.n; ++x) *sim_deriv(sm, x + 1) = m->deriv_ids[sim_aero(sm, x)];
        int ij = 0;
        *sim_jac(sm, ij++) = jr_elem_id(cp, ri, g, g);
        for (int x = 0; x < sm.n; ++x) {
          const int a = sim_aero(sm, x);
          *sim_jac(sm, ij++) = jr_elem_id(cp, ri, a, g);
          *sim_jac(sm, ij++) = jr_elem_id(cp, ri, g, a);
          *sim_jac(sm, ij++) = jr_elem_id(cp, ri, a, a);
          if (sim_act(sm, x) > 0) {
            *sim_gas_act_jac(sm, x) = jr_elem_id(cp, ri, g, sim_act(sm, x));
            *sim_aero_act_jac(sm, x) = jr_elem_id(cp, ri, a, sim_act(sm, x));
          } else {
            *sim_gas_act_jac(sm, x) = -1;
            *sim_aero_act_jac(sm, x) = -1;
          }
          for (int e = 0; e < sim_nelem(sm, x); ++e) {
            int *pg = sim_phase_jac(sm, x, 0, e), *pa = sim_phase_jac(sm, x, 1, e);
            if (*pg > 0) *pg = jr_elem_id(cp, ri, g, *pg);
            if (*pa > 0) *pa = jr_elem_id(cp, ri, a, *pa);
          }
        }
        continue;
      }
      case T_AQ: { /* src/rxns/rxn_aqueous_equilibrium.c:132-209 */
        AQV q = aqv(r);
        const int *cp = m->rj_colptr, *ri = m->rj_rowid;
        int id = 0;
        for (int p = 0; p < q.P; ++p) {
          for (int i = 0; i < q.nr; ++i) *aq_deriv(q, id++) = m->deriv_ids[aq_react(q, p * q.nr + i)];
          for (int i = 0; i < q.np; ++i) *aq_deriv(q, id++) = m->deriv_ids[aq_prod(q, p * q.np + i)];
        }
        int ij = 0;
        for (int p = 0; p < q.P; ++p) {
          for (int i = 0; i < q.nr; ++i) {
            const int ind = aq_react(q, p * q.nr + i);
            for (int d = 0; d < q.nr; ++d) *aq_jac(q, ij++) = jr_elem_id(cp, ri, aq_react(q, p * q.nr + d), ind);
            for (int d = 0; d < q.np; ++d) *aq_jac(q, ij++) = jr_elem_id(cp, ri, aq_prod(q, p * q.np + d), ind);
          }
          for (int i = 0; i < q.np; ++i) {
            const int ind = aq_prod(q, p * q.np + i);
            for (int d = 0; d < q.nr; ++d) *aq_jac(q, ij++) = jr_elem_id(cp, ri, aq_react(q, p * q.nr + d), ind);
            for (int d = 0; d < q.np; ++d) *aq_jac(q, ij++) = jr_elem_id(cp, ri, aq_prod(q, p * q.np + d), ind);
          }
          for (int d = 0; d < q.nr; ++d) *aq_jac(q, ij++) = jr_elem_id(cp, ri, aq_react(q, p * q.nr + d), aq_water(q, p));
          for (int d = 0; d < q.np; ++d) *aq_jac(q, ij++) = jr_elem_id(cp, ri, aq_prod(q, p * q.np + d), aq_water(q, p));
          const int a = aq_act(q, p);
          for (int d = 0; d < q.nr; ++d) *aq_jac(q, ij++) = a < 0 ? -1 : jr_elem_id(cp, ri, aq_react(q, p * q.nr + d), a);
          for (int d = 0; d < q.np; ++d) *aq_jac(q, ij++) = a < 0 ? -1 : jr_elem_id(cp, ri, aq_prod(q, p * q.np + d), a);
        }
        continue;
      }
      case T_HL: { /* src/rxns/rxn_HL_phase_transfer.c:149-186; the small
                    * water concentration it also sets (:188-193) is unused */
        HLV hl = hlv(r);
        const int *cp = m->rj_colptr, *ri = m->rj_rowid;
        const int g = hl_gas(hl);
        *hl_deriv(hl, 0) = m->deriv_ids[g];
        for (int x = 0; x < hl.n; ++x) *hl_deriv(hl, x + 1) = m->deriv_ids[hl_aero(hl, x)];
        int ij = 0;
        *hl_jac(hl, ij++) = jr_elem_id(cp, ri, g, g);
        for (int x = 0; x < hl.n; ++x) {
          const int a = hl_aero(hl, x), w = hl_water(hl, x);
          *hl_jac(hl, ij++) = jr_elem_id(cp, ri, a, g);
          *hl_jac(hl, ij++) = jr_elem_id(cp, ri, g, a);
          *hl_jac(hl, ij++) = jr_elem_id(cp, ri, a, a);
          *hl_jac(hl, ij++) = jr_elem_id(cp, ri, g, w);
          *hl_jac(hl, ij++) = jr_elem_id(cp, ri, a, w);
          for (int e = 0; e < hl_nelem(hl, x); ++e) {
            int *pg = hl_phase_jac(hl, x, 0, e), *pa = hl_phase_jac(hl, x, 1, e);
            if (*pg > 0) *pg = jr_elem_id(cp, ri, g, *pg);
            if (*pa > 0) *pa = jr_elem_id(cp, ri, a, *pa);
          }
        }
        continue;
      }
    }
    for (int k = 0; k < r->nr; ++k) R_DERIV_ID(r, k) = m->deriv_ids[R_REACT(r, k)];
    for (int k = 0; k < r->np; ++k)
      R_DERIV_ID(r, r->nr + k) = m->deriv_ids[R_PROD(r, k)];
    int ij = 0;
    for (int ind = 0; ind < r->nr; ++ind) {
      for (int d = 0; d < r->nr; ++d)
        R_JAC_ID(r, ij++) =
            jr_elem_id(m->rj_colptr, m->rj_rowid, R_REACT(r, d), R_REACT(r, ind));
      for (int d = 0; d < r->np; ++d)
        R_JAC_ID(r, ij++) =
            jr_elem_id(m->rj_colptr, m->rj_rowid, R_PROD(r, d), R_REACT(r, ind));
    }
  }

  /* sub-model parameter Jacobian (src/camp_solver.c:1520-1550): the dummy
   * element (0, 0), then the sub-models' elements through a local Jacobian
   * (src/sub_model_solver.c:25-104); an element whose independent species is
   * itself computed by a sub-model would need the interdependence map, which
   * no supported configuration has: refused */
  JacReg pj, lj;
  jr_init(&pj, n);
  jr_register(&pj, 0, 0);
  jr_init(&lj, n);
  for (int k = 0; k < m->n_sub; ++k) sub_elements(m, k, sub_register_cb, &lj);
  jr_build(&lj);
  for (int ind = 0; ind < n; ++ind)
    for (int e = lj.colptr[ind]; e < lj.colptr[ind + 1]; ++e) {
      const int dep = lj.rowid[e];
      jr_register(&pj, dep, ind);
      if (dep != ind && m->var_type[ind] != VAR_VARIABLE)
        for (int j = 0; j < n; ++j)
          if (jr_elem_id(lj.colptr, lj.rowid, ind, j) != -1) return 3;
    }
  free(lj.colptr);
  free(lj.rowid);
  jr_build(&pj);
  m->n_param_jac = pj.nnz;
  m->pj_colptr = pj.colptr;
  m->pj_rowid = pj.rowid;
  {
    PJLookup l = {m->pj_colptr, m->pj_rowid};
    for (int k = 0; k < m->n_sub; ++k) sub_elements(m, k, sub_ids_cb, &l);
  }

  /* solver Jacobian (src/camp_solver.c:1559-1633): a variable row keeps its
   * variable columns, and a non-variable column c maps to every variable
   * species the sub-model parameter c depends on */
  JacReg sj;
  jr_init(&sj, n);
  for (int ind = 0; ind < n; ++ind)
    for (int dep = 0; dep < n; ++dep) {
      if (m->var_type[dep] != VAR_VARIABLE ||
          jr_elem_id(m->rj_colptr, m->rj_rowid, dep, ind) == -1)
        continue;
      if (m->var_type[ind] == VAR_VARIABLE) {
        jr_register(&sj, dep, ind);
        continue;
      }
      for (int j = 0; j < n; ++j)
        if (jr_elem_id(m->pj_colptr, m->pj_rowid, ind, j) != -1 &&
            m->var_type[j] == VAR_VARIABLE)
          jr_register(&sj, dep, j);
    }
  jr_build(&sj);
  m->n_solver_jac = sj.nnz;
  m->sj_colptr = (int *)zalloc(sizeof(int) * (m->n_dep + 1));
  m->sj_rowid = (int *)zalloc(sizeof(int) * (sj.nnz + 1));
  for (int c = 0; c < n; ++c)
    if (m->deriv_ids[c] >= 0) m->sj_colptr[m->deriv_ids[c]] = sj.colptr[c];
  m->sj_colptr[m->n_dep] = sj.nnz;
  for (int e = 0; e < sj.nnz; ++e) m->sj_rowid[e] = m->deriv_ids[sj.rowid[e]];
  /* the fold map (src/camp_solver.c:1649-1681), in reaction-Jacobian order;
   * param 0 is the unit parameter */
  int cap = m->n_rxn_jac + 16, nm = 0;
  m->map_s = (int *)zalloc(sizeof(int) * cap);
  m->map_r = (int *)zalloc(sizeof(int) * cap);
  m->map_p = (int *)zalloc(sizeof(int) * cap);
  m->rxn_to_solver = (int *)zalloc(sizeof(int) * (m->n_rxn_jac + 1));
  for (int ind = 0; ind < n; ++ind)
    for (int e = m->rj_colptr[ind]; e < m->rj_colptr[ind + 1]; ++e) {
      const int dep = m->rj_rowid[e];
      m->rxn_to_solver[e] = -1;
      if (m->var_type[dep] != VAR_VARIABLE) continue;
      for (int j = 0; j < n; ++j) {
        int s = -1, pid = 0;
        if (m->var_type[ind] == VAR_VARIABLE) {
          if (j > 0) break;
          s = jr_elem_id(sj.colptr, sj.rowid, dep, ind);
          m->rxn_to_solver[e] = s;
        } else {
          pid = jr_elem_id(m->pj_colptr, m->pj_rowid, ind, j);
          if (pid == -1 || m->var_type[j] != VAR_VARIABLE) continue;
          s = jr_elem_id(sj.colptr, sj.rowid, dep, j);
        }
        if (nm == cap) {
          cap *= 2;
          m->map_s = (int *)realloc(m->map_s, sizeof(int) * cap);
          m->map_r = (int *)realloc(m->map_r, sizeof(int) * cap);
          m->map_p = (int *)realloc(m->map_p, sizeof(int) * cap);
        }
        m->map_s[nm] = s;
        m->map_r[nm] = e;
        m->map_p[nm] = pid;
        ++nm;
      }
    }
  m->n_map = nm;
  free(sj.colptr);
  free(sj.rowid);
  lu_symbolic(&m->lu, m->n_dep, m->sj_colptr, m->sj_rowid);
  m->built = 1;
  return 0;
}

void om_free(OracleMech *m) {
  if (!m) return;
  for (int i = 0; i < m->n_rxn; ++i) free(m->rx[i].aq_thr);
  free(m->sub_type);
  free(m->sub_ioff);
  free(m->sub_foff);
  free(m->sub_eoff);
  free(m->sub_int);
  free(m->sub_flt);
  free(m->pj_colptr);
  free(m->pj_rowid);
  free(m->map_s);
  free(m->map_r);
  free(m->map_p);
  free(m->var_type);
  free(m->int_data);
  free(m->float_data);
  free(m->rx);
  free(m->deriv_ids);
  free(m->rj_colptr);
  free(m->rj_rowid);
  free(m->sj_colptr);
  free(m->sj_rowid);
  free(m->rxn_to_solver);
  free(m->aph_int);
  free(m->aph_ioff);
  free(m->aph_foff);
  free(m->aph_flt);
  free(m->arep_int);
  free(m->arep_ioff);
  free(m->arep_foff);
  free(m->arep_eoff);
  free(m->arep_type);
  free(m->arep_flt);
  if (m->built) lu_free(&m->lu);
  free(m);
}

int om_n_dep_var(const OracleMech *m) { return m->n_dep; }
int om_n_rxn_env_data(const OracleMech *m) { return m->n_env + m->n_aero_env + m->n_sub_env; }
int om_n_param_jac_elem(const OracleMech *m) { return m->n_param_jac; }
int om_n_mapped_values(const OracleMech *m) { return m->n_map; }
void om_get_jac_map(const OracleMech *m, int *triplets) {
  for (int i = 0; i < m->n_map; ++i) {
    triplets[3 * i] = m->map_s[i];
    triplets[3 * i + 1] = m->map_r[i];
    triplets[3 * i + 2] = m->map_p[i];
  }
}
int om_n_rxn_jac_elem(const OracleMech *m) { return m->n_rxn_jac; }
int om_n_solver_jac_elem(const OracleMech *m) { return m->n_solver_jac; }
int om_n_lu_elem(const OracleMech *m) { return m->lu.nnz; }
int om_rxn_int_data_size(const OracleMech *m) { return m->int_size; }
void om_get_rxn_jac(const OracleMech *m, int *colptr, int *rowid) {
  memcpy(colptr, m->rj_colptr, sizeof(int) * (m->n_state + 1));
  memcpy(rowid, m->rj_rowid, sizeof(int) * m->n_rxn_jac);
}
void om_get_solver_jac(const OracleMech *m, int *colptr, int *rowid) {
  memcpy(colptr, m->sj_colptr, sizeof(int) * (m->n_dep + 1));
  memcpy(rowid, m->sj_rowid, sizeof(int) * m->n_solver_jac);
}
void om_get_rxn_int_data(const OracleMech *m, int *out) {
  memcpy(out, m->int_data, sizeof(int) * m->int_size);
}
void om_get_lu_order(const OracleMech *m, int *perm) {
  memcpy(perm, m->lu.perm, sizeof(int) * m->n_dep);
}

/* ------------------------------------------------------------------------ */
/* Rate constants (update_env_state of each gas type)                        */
/* ------------------------------------------------------------------------ */

/* rxn_update_data (src/rxn_solver.c:700-760) with the update_data function
 * of each host-rate type (src/rxns/rxn_photolysis.c:109-125,
 * rxn_emission.c:82-98, rxn_first_order_loss.c:89-106,
 * rxn_wet_deposition.c:95-112): the first reaction of the type whose RXN_ID_
 * (> 0) matches takes BASE_RATE_ and RATE_ = SCALING_ * BASE_RATE_. */
int om_set_rate(const OracleMech *m, double *rxn_env, int type, int rxn_id,
                double base_rate) {
  for (int i = 0; i < m->n_rxn; ++i) {
    const ORxn *r = &m->rx[i];
    if (r->type != type) continue;
    int rid;
    if (type == T_PHOTOLYSIS)
      rid = r->ints[2];
    else if (species_rate_type(type))
      rid = r->ints[0];
    else
      return 0;
    if (rid != rxn_id || rid <= 0) continue;
    rxn_env[r->env_off + 1] = base_rate;
    rxn_env[r->env_off] = r->fl[0] * base_rate;
    return 1;
  }
  return 0;
}

int om_set_photo_rate(const OracleMech *m, double *rxn_env, int photo_id,
                      double base_rate) {
  return om_set_rate(m, rxn_env, T_PHOTOLYSIS, photo_id, base_rate);
}

void om_update_env(const OracleMech *m, const double *env, double *rxn_env) {
  const double T = env[0], P = env[1];
  for (int i = 0; i < m->n_rxn; ++i) {
    const ORxn *r = &m->rx[i];
    const double *f = r->fl;
    double *k = rxn_env + r->env_off;
    switch (r->type) {
      case T_ARRHENIUS: /* src/rxns/rxn_arrhenius.c:103-118 */
        k[0] = f[0] * exp(f[2] / T) * (f[1] == 0.0 ? 1.0 : pow(T / f[3], f[1])) *
               (f[4] == 0.0 ? 1.0 : (1.0 + f[4] * P)) *
               pow(f[5] * P / T, r->nr - 1);
        break;
      case T_TROE: { /* src/rxns/rxn_troe.c:118-140 */
        double conv = f[9] * P / T;
        double k0 = f[0] * (f[2] == 0.0 ? 1.0 : exp(f[2] / T)) *
                    (f[1] == 0.0 ? 1.0 : pow(T / 300.0, f[1])) * conv;
        double kinf = k0 / (f[3] * (f[5] == 0.0 ? 1.0 : exp(f[5] / T)) *
                            (f[4] == 0.0 ? 1.0 : pow(T / 300.0, f[4])));
        k[0] = (k0 / (1.0 + kinf)) *
               pow(f[6], (1.0 / (1.0 + pow(log10(kinf) / f[7], 2)))) *
               pow(conv, r->nr - 1) * f[8];
        break;
      }
      case T_CMAQ_H2O2: { /* src/rxns/rxn_CMAQ_H2O2.c:106-125 */
        double conv = f[6] * P / T;
        k[0] = (f[0] * (f[2] == 0.0 ? 1.0 : exp(f[2] / T)) *
                    (f[1] == 0.0 ? 1.0 : pow(T / 300.0, f[1])) +
                f[3] * (f[5] == 0.0 ? 1.0 : exp(f[5] / T)) *
                    (f[4] == 0.0 ? 1.0 : pow(T / 300.0, f[4])) * conv) *
               pow(conv, r->nr - 1);
        break;
      }
      case T_CMAQ_OH_HNO3: { /* src/rxns/rxn_CMAQ_OH_HNO3.c:110-133 */
        double conv = f[10] * P / T;
        double k2 = f[3] * (f[5] == 0.0 ? 1.0 : exp(f[5] / T)) *
                    (f[4] == 0.0 ? 1.0 : pow(T / 300.0, f[4]));
        double k3 = f[6] * (f[8] == 0.0 ? 1.0 : exp(f[8] / T)) *
                    (f[7] == 0.0 ? 1.0 : pow(T / 300.0, f[7])) * conv;
        k[0] = (f[0] * (f[2] == 0.0 ? 1.0 : exp(f[2] / T)) *
                    (f[1] == 0.0 ? 1.0 : pow(T / 300.0, f[1])) +
                k3 / (1.0 + k3 / k2)) *
               pow(conv, r->nr - 1) * f[9];
        break;
      }
      case T_PHOTOLYSIS:         /* src/rxns/rxn_photolysis.c:137-148 */
      case T_FIRST_ORDER_LOSS:   /* src/rxns/rxn_first_order_loss.c:118-130 */
      case T_EMISSION:           /* src/rxns/rxn_emission.c:109-120 */
      case T_WET_DEPOSITION:     /* src/rxns/rxn_wet_deposition.c:124-136 */
        k[0] = f[0] * k[1];
        break;
      case T_SIMPOL:
        simpol_env(r, T, P, k);
        break;
      case T_HL:
        hl_env(r, T, P, k);
        break;
      case T_AQ: /* src/rxns/rxn_aqueous_equilibrium.c:244-262 */
        k[0] = (f[1] == 0.0 ? f[0] : f[0] * exp(f[1] * (1.0 / T - 1.0 / 298.0))) * f[2];
        break;
    }
  }
  /* sub_model_update_env_state (src/sub_model_solver.c:264-295): both
   * sub-model types keep PPM_TO_RH_ as their one env parameter */
  for (int k = 0; k < m->n_sub; ++k)
    rxn_env[m->n_env + m->n_aero_env + m->sub_eoff[k]] = ppm_to_rh(T, P);
}

/* ------------------------------------------------------------------------ */
/* Derivative and Jacobian (calc_deriv_contrib / calc_jac_contrib)           */
/* ------------------------------------------------------------------------ */

/* time_derivative_add_value (src/time_derivative.c:90-97) */
static void add_value(long double *P, long double *L, int d, long double v) {
  if (v > 0.0)
    P[d] += v;
  else
    L[d] += -v;
}

/* The gas types share one mass-action form: rate = k * prod(y_react), loss of
 * rate on each reactant, rate*yield on each product unless a negative yield
 * would drive the product below zero within one step
 * (src/rxns/rxn_arrhenius.c:131-165).  Contributions are split by sign into
 * production and loss sums (src/time_derivative.c:90-97). */
void om_deriv(const OracleMech *m, const double *state_in, const double *rxn_env,
              double time_step, double *deriv, double *r_p, double *r_l) {
  /* the sub-models first write their computed species into (a copy of) the
   * state, as f does (src/camp_solver.c:907-911) */
  double *tmp = NULL;
  const double *state = state_in;
  if (m->n_sub > 0) {
    tmp = (double *)zalloc(sizeof(double) * m->n_state);
    memcpy(tmp, state_in, sizeof(double) * m->n_state);
    sub_calculate(m, tmp, rxn_env);
    state = tmp;
  }
  long double *P = (long double *)zalloc(sizeof(long double) * m->n_dep * 2);
  long double *L = P + m->n_dep;
  for (int i = 0; i < m->n_rxn; ++i) {
    const ORxn *r = &m->rx[i];
    const int *I = r->ints;
    const double k = rxn_env[r->env_off];
    switch (r->type) {
      case T_FIRST_ORDER_LOSS: /* src/rxns/rxn_first_order_loss.c:143-158 */
        if (I[2] >= 0) add_value(P, L, I[2], -(k * (long double)state[I[1] - 1]));
        continue;
      case T_EMISSION: /* src/rxns/rxn_emission.c:133-147 */
        if (I[2] >= 0) add_value(P, L, I[2], (long double)k);
        continue;
      case T_WET_DEPOSITION: { /* src/rxns/rxn_wet_deposition.c:149-166 */
        const int ns = I[1];
        for (int s = 0; s < ns; ++s)
          if (I[2 + ns + s] >= 0)
            add_value(P, L, I[2 + ns + s], -(k * (long double)state[I[2 + s] - 1]));
        continue;
      }
      case T_SIMPOL: { /* src/rxns/rxn_SIMPOL_phase_transfer.c:337-450 */
        SIM sm = simpol(r);
        const double *kk = rxn_env + r->env_off;
        for (int x = 0; x < sm.n; ++x) {
          ARep ar = arep(m, sim_rep(sm, x), rxn_env);
          int sx, sb, sy;
          if (!arep_locate(ar, sim_phase(sm, x), &sx, &sb, &sy)) continue;
          const double radius = arep_radius(ar, sx, sb);
          const double nconc = arep_number(m, ar, sx, sb, state, NULL);
          double mass, mw;
          arep_phase_mass(m, ar, sx, sb, sy, state, &mass, &mw, NULL, NULL);
          long double cond = cond_k(sm.F[2], kk[0], radius, kk[1]);
          long double evap = cond * (kk[2] * mw / mass);
          long double act = 1.0;
          if (sim_act(sm, x) > -1) act = state[sim_act(sm, x)];
          evap *= act;
          cond *= state[sim_gas(sm)];
          evap *= state[sim_aero(sm, x)];
          /* total-particle mass concentrations (this representation's
           * aero_conc_type) */
          const int dg = *sim_deriv(sm, 0), da = *sim_deriv(sm, 1 + x);
          if (dg >= 0) {
            add_value(P, L, dg, nconc * evap);
            add_value(P, L, dg, -nconc * cond);
          }
          if (da >= 0) {
            add_value(P, L, da, -nconc * evap / kk[3]);
            add_value(P, L, da, nconc * cond / kk[3]);
          }
        }
        continue;
      }
      case T_AQ: { /* src/rxns/rxn_aqueous_equilibrium.c:266-393 */
        AQV q = aqv(r);
        const double kf = rxn_env[r->env_off], kr = q.F[2];
        for (int p = 0, id = 0; p < q.P; ++p) {
          const long double water = state[aq_water(q, p)];
          if (water < r->aq_thr[p]) {
            id += q.nr + q.np;
            continue;
          }
          long double rf = (long double)state[aq_react(q, p * q.nr)] * aq_m2m(q, 0);
          for (int i = 1; i < q.nr; ++i)
            rf *= state[aq_react(q, p * q.nr + i)] * aq_m2m(q, i) / water;
          long double rr = (long double)state[aq_prod(q, p * q.np)] * aq_m2m(q, q.nr);
          rr *= (long double)(aq_act(q, p) >= 0 ? state[aq_act(q, p)] : 1.0);
          for (int i = 1; i < q.np; ++i)
            rr *= state[aq_prod(q, p * q.np + i)] * aq_m2m(q, q.nr + i) / water;
          rf = kf * rf;
          rr = kr * rr;
          if (rf - rr == 0.0) {
            id += q.nr + q.np;
            continue;
          }
          for (int i = 0; i < q.nr; ++i, ++id) {
            const int d = *aq_deriv(q, id);
            if (d < 0) continue;
            add_value(P, L, d, -rf / aq_m2m(q, i));
            add_value(P, L, d, rr / aq_m2m(q, i));
          }
          for (int i = 0; i < q.np; ++i, ++id) {
            const int d = *aq_deriv(q, id);
            if (d < 0) continue;
            add_value(P, L, d, rf / aq_m2m(q, q.nr + i));
            add_value(P, L, d, -rr / aq_m2m(q, q.nr + i));
          }
        }
        continue;
      }
      case T_HL: { /* src/rxns/rxn_HL_phase_transfer.c:262-330 */
        HLV hl = hlv(r);
        const double *kk = rxn_env + r->env_off;
        for (int x = 0; x < hl.n; ++x) {
          ARep ar = arep(m, hl_rep(hl, x), rxn_env);
          int sx, sb, sy;
          if (!arep_locate(ar, hl_phase(hl, x), &sx, &sb, &sy)) continue;
          const double radius = arep_radius(ar, sx, sb);
          /* total-particle mass concentrations: number_conc stays 1 */
          const double nconc = 1.0;
          long double cond = cond_k(hl.F[2], kk[0], radius, kk[1]);
          long double evap = cond / kk[2];
          cond *= state[hl_gas(hl)];
          evap *= state[hl_aero(hl, x)] / state[hl_water(hl, x)];
          const int dg = *hl_deriv(hl, 0), da = *hl_deriv(hl, 1 + x);
          if (dg >= 0) {
            add_value(P, L, dg, nconc * evap);
            add_value(P, L, dg, -nconc * cond);
          }
          if (da >= 0) {
            add_value(P, L, da, -evap / kk[3]);
            add_value(P, L, da, cond / kk[3]);
          }
        }
        continue;
      }
    }
    long double rate = rxn_env[r->env_off];
    for (int s = 0; s < r->nr; ++s) rate *= state[R_REACT(r, s)];
    if (rate == 0.0) continue;
    for (int s = 0; s < r->nr; ++s) {
      int d = R_DERIV_ID(r, s);
      if (d < 0) continue;
      L[d] += rate; /* -rate is negative: a loss */
    }
    for (int s = 0; s < r->np; ++s) {
      int d = R_DERIV_ID(r, r->nr + s);
      if (d < 0) continue;
      if (-rate * R_YIELD(r, s) * time_step <= state[R_PROD(r, s)]) {
        long double c = rate * R_YIELD(r, s);
        if (c > 0.0)
          P[d] += c;
        else
          L[d] += -c;
      }
    }
  }
  for (int d = 0; d < m->n_dep; ++d) {
    /* time_derivative_output without the estimate (src/time_derivative.c:46-88) */
    deriv[d] = (P[d] + L[d] != 0.0) ? (double)(P[d] - L[d]) : 0.0;
    if (r_p) r_p[d] = (double)P[d];
    if (r_l) r_l[d] = (double)L[d];
  }
  free(P);
  free(tmp);
}

/* src/rxns/rxn_arrhenius.c:178-212 and src/Jacobian.c:223-241, then the
 * jac_map fold with the sub-model parameters (src/camp_solver.c:1063-1106):
 * J_solver[s] += J_rxn[r] * J_params[p], J_params[0] = 1. */
void om_jac(const OracleMech *m, const double *state_in, const double *rxn_env,
            double time_step, double *jvals) {
  double *tmp = (double *)zalloc(sizeof(double) * (m->n_state + m->n_param_jac + 1));
  double *JP = tmp + m->n_state;
  const double *state = state_in;
  if (m->n_sub > 0) {
    memcpy(tmp, state_in, sizeof(double) * m->n_state);
    sub_calculate(m, tmp, rxn_env);
    state = tmp;
  }
  sub_jacobian(m, state, rxn_env, JP);
  long double *P = (long double *)zalloc(sizeof(long double) * m->n_rxn_jac * 2);
  long double *L = P + m->n_rxn_jac;
  for (int i = 0; i < m->n_rxn; ++i) {
    const ORxn *r = &m->rx[i];
    const int *I = r->ints;
    switch (r->type) {
      case T_FIRST_ORDER_LOSS: /* src/rxns/rxn_first_order_loss.c:171-187 */
        if (I[3] >= 0) L[I[3]] += rxn_env[r->env_off];
        continue;
      case T_EMISSION: /* src/rxns/rxn_emission.c:160-171: none */
        continue;
      case T_WET_DEPOSITION: { /* src/rxns/rxn_wet_deposition.c:179-197 */
        const int ns = I[1];
        for (int s = 0; s < ns; ++s)
          if (I[2 + 2 * ns + s] >= 0) L[I[2 + 2 * ns + s]] += rxn_env[r->env_off];
        continue;
      }
      case T_SIMPOL: { /* src/rxns/rxn_SIMPOL_phase_transfer.c:463-744 */
        SIM sm = simpol(r);
        const double *kk = rxn_env + r->env_off;
        const double Kp = kk[3];
        for (int x = 0; x < sm.n; ++x) {
          ARep ar = arep(m, sim_rep(sm, x), rxn_env);
          int sx, sb, sy;
          if (!arep_locate(ar, sim_phase(sm, x), &sx, &sb, &sy)) continue;
          const int ne = sim_nelem(sm, x);
          double *nd = (double *)zalloc(sizeof(double) * (3 * (size_t)ne + 1));
          const double radius = arep_radius(ar, sx, sb);
          const double nconc = arep_number(m, ar, sx, sb, state, nd);
          double mass, mw;
          arep_phase_mass(m, ar, sx, sb, sy, state, &mass, &mw, nd + ne, nd + 2 * ne);
          long double cond = cond_k(sm.F[2], kk[0], radius, kk[1]);
          long double evap = cond * (kk[2] * mw / mass);
          long double act = 1.0;
          if (sim_act(sm, x) > -1) act = state[sim_act(sm, x)];
          const double yg = state[sim_gas(sm)], ya = state[sim_aero(sm, x)];
          const int jgg = *sim_jac(sm, 0), jag = *sim_jac(sm, 1 + 3 * x);
          const int jga = *sim_jac(sm, 2 + 3 * x), jaa = *sim_jac(sm, 3 + 3 * x);
          if (jga >= 0) P[jga] += nconc * evap * act;
          if (jgg >= 0) L[jgg] += nconc * cond;
          if (jag >= 0) P[jag] += nconc * cond / Kp;
          if (jaa >= 0) L[jaa] += nconc * evap * act / Kp;
          if (*sim_gas_act_jac(sm, x) > 0) P[*sim_gas_act_jac(sm, x)] += nconc * evap * ya;
          if (*sim_aero_act_jac(sm, x) > 0)
            L[*sim_aero_act_jac(sm, x)] += nconc * evap / Kp * ya;
          evap *= act;
          cond *= yg;
          evap *= ya;
          /* radius partials are zero for this representation (its radii do
           * not depend on the state), added as the reference adds them */
          const double dcdr = cond_k_dr(sm.F[2], kk[0], radius, kk[1]) * yg;
          const double dedr = dcdr / yg * kk[2] * mw / mass * ya;
          const double dedm = -evap / mass;
          const double dedw = evap / mw;
          for (int e = 0; e < ne; ++e) {
            const double eff = 0.0, num = nd[e], ms = nd[ne + e], mwj = nd[2 * ne + e];
            const int jg = *sim_phase_jac(sm, x, 0, e), ja = *sim_phase_jac(sm, x, 1, e);
            if (jg > 0) {
              P[jg] += nconc * dedr * eff;
              L[jg] += nconc * dcdr * eff;
              P[jg] += evap * num;
              L[jg] += cond * num;
              P[jg] += nconc * dedm * ms;
              P[jg] += nconc * dedw * mwj;
            }
            if (ja > 0) {
              L[ja] += nconc * dedr / Kp * eff;
              P[ja] += nconc * dcdr / Kp * eff;
              L[ja] += evap / Kp * num;
              P[ja] += cond / Kp * num;
              L[ja] += nconc * dedm / Kp * ms;
              L[ja] += nconc * dedw / Kp * mwj;
            }
          }
          free(nd);
        }
        continue;
      }
      case T_AQ: { /* src/rxns/rxn_aqueous_equilibrium.c:403-540 */
        AQV q = aqv(r);
        const int ns = q.nr + q.np;
        for (int p = 0, ij = 0; p < q.P; ++p) {
          const long double water = state[aq_water(q, p)];
          if (water < r->aq_thr[p]) {
            ij += ns * (ns + 2);
            continue;
          }
          long double fr = rxn_env[r->env_off];
          for (int i = 0; i < q.nr; ++i) fr *= state[aq_react(q, p * q.nr + i)] * aq_m2m(q, i) / water;
          long double rr = q.F[2];
          for (int i = 0; i < q.np; ++i)
            rr *= state[aq_prod(q, p * q.np + i)] * aq_m2m(q, q.nr + i) / water;
          const int a = aq_act(q, p);
          if (a >= 0) rr *= state[a];
          for (int i = 0; i < q.nr; ++i) {
            const double c = state[aq_react(q, p * q.nr + i)];
            for (int d = 0; d < q.nr; ++d, ++ij)
              if (*aq_jac(q, ij) >= 0 && fr != 0.0) L[*aq_jac(q, ij)] += fr / c / aq_m2m(q, d) * water;
            for (int d = 0; d < q.np; ++d, ++ij)
              if (*aq_jac(q, ij) >= 0 && fr != 0.0)
                P[*aq_jac(q, ij)] += fr / c / aq_m2m(q, q.nr + d) * water;
          }
          for (int i = 0; i < q.np; ++i) {
            const double c = state[aq_prod(q, p * q.np + i)];
            for (int d = 0; d < q.nr; ++d, ++ij)
              if (*aq_jac(q, ij) >= 0 && rr != 0.0) P[*aq_jac(q, ij)] += rr / c / aq_m2m(q, d) * water;
            for (int d = 0; d < q.np; ++d, ++ij)
              if (*aq_jac(q, ij) >= 0 && rr != 0.0)
                L[*aq_jac(q, ij)] += rr / c / aq_m2m(q, q.nr + d) * water;
          }
          for (int d = 0; d < q.nr; ++d, ++ij) {
            if (*aq_jac(q, ij) < 0) continue;
            L[*aq_jac(q, ij)] += -fr / aq_m2m(q, d) * (q.nr - 1);
            P[*aq_jac(q, ij)] += -rr / aq_m2m(q, d) * (q.np - 1);
          }
          for (int d = 0; d < q.np; ++d, ++ij) {
            if (*aq_jac(q, ij) < 0) continue;
            P[*aq_jac(q, ij)] += -fr / aq_m2m(q, q.nr + d) * (q.nr - 1);
            L[*aq_jac(q, ij)] += -rr / aq_m2m(q, q.nr + d) * (q.np - 1);
          }
          if (a < 0) {
            ij += ns;
            continue;
          }
          for (int d = 0; d < q.nr; ++d, ++ij)
            if (*aq_jac(q, ij) >= 0) P[*aq_jac(q, ij)] += rr / state[a] / aq_m2m(q, d) * water;
          for (int d = 0; d < q.np; ++d, ++ij)
            if (*aq_jac(q, ij) >= 0)
              L[*aq_jac(q, ij)] += rr / state[a] / aq_m2m(q, q.nr + d) * water;
        }
        continue;
      }
      case T_HL: { /* src/rxns/rxn_HL_phase_transfer.c:343-494 */
        HLV hl = hlv(r);
        const double *kk = rxn_env + r->env_off;
        const double Kp = kk[3];
        for (int x = 0; x < hl.n; ++x) {
          ARep ar = arep(m, hl_rep(hl, x), rxn_env);
          int sx, sb, sy;
          if (!arep_locate(ar, hl_phase(hl, x), &sx, &sb, &sy)) continue;
          const double radius = arep_radius(ar, sx, sb);
          /* total-particle mass concentrations: number 1, its partials 0;
           * the radius partials of modes and bins are 0 as well */
          const double nconc = 1.0, eff = 0.0, num = 0.0;
          long double cond = cond_k(hl.F[2], kk[0], radius, kk[1]);
          long double evap = cond / kk[2];
          const double yg = state[hl_gas(hl)], ya = state[hl_aero(hl, x)];
          const double yw = state[hl_water(hl, x)];
          const int j0 = *hl_jac(hl, 0), jag = *hl_jac(hl, 1 + 5 * x);
          const int jga = *hl_jac(hl, 2 + 5 * x), jaa = *hl_jac(hl, 3 + 5 * x);
          const int jgw = *hl_jac(hl, 4 + 5 * x), jaw = *hl_jac(hl, 5 + 5 * x);
          if (j0 >= 0) L[j0] += nconc * cond;
          if (jga >= 0) P[jga] += nconc * evap / yw;
          if (jgw >= 0) P[jgw] += -nconc * evap * ya / yw / yw;
          if (jag >= 0) P[jag] += cond / Kp;
          if (jaa >= 0) L[jaa] += evap / yw / Kp;
          if (jaw >= 0) L[jaw] += -evap * ya / Kp / yw / yw;
          cond *= yg;
          evap *= ya / yw;
          const long double dcdr = cond_k_dr(hl.F[2], kk[0], radius, kk[1]) * yg;
          const long double dedr = dcdr / yg / kk[2] * ya / yw;
          for (int e = 0; e < hl_nelem(hl, x); ++e) {
            const int jg = *hl_phase_jac(hl, x, 0, e), ja = *hl_phase_jac(hl, x, 1, e);
            if (jg > 0) {
              P[jg] += nconc * dedr * eff;
              L[jg] += nconc * dcdr * eff;
              P[jg] += evap * num;
              L[jg] += cond * num;
            }
            if (ja > 0) {
              L[ja] += dedr / Kp * eff;
              P[ja] += dcdr / Kp * eff;
            }
          }
        }
        continue;
      }
    }
    int e = 0;
    for (int ind = 0; ind < r->nr; ++ind) {
      double rate = rxn_env[r->env_off];
      for (int s = 0; s < r->nr; ++s)
        if (s != ind) rate *= state[R_REACT(r, s)];
      for (int d = 0; d < r->nr; ++d, ++e) {
        int id = R_JAC_ID(r, e);
        if (id < 0) continue;
        L[id] += rate;
      }
      for (int d = 0; d < r->np; ++d, ++e) {
        int id = R_JAC_ID(r, e);
        if (id < 0) continue;
        if (-rate * state[R_REACT(r, ind)] * R_YIELD(r, d) * time_step <=
            state[R_PROD(r, d)])
          P[id] += R_YIELD(r, d) * rate;
      }
    }
  }
  for (int s = 0; s < m->n_solver_jac; ++s) jvals[s] = 0.0;
  for (int i = 0; i < m->n_map; ++i)
    jvals[m->map_s[i]] += (double)(P[m->map_r[i]] - L[m->map_r[i]]) * JP[m->map_p[i]];
  free(P);
  free(tmp);
}

/* ------------------------------------------------------------------------ */
/* Sparse LU of M = I - gamma*J                                             */
/* ------------------------------------------------------------------------ */

/* Forms M in LU storage, factors it row by row (IKJ order with a dense work
 * row), returns 0, or 1 when a pivot is zero or not finite (the linear solver
 * setup then fails recoverably, as a singular KLU factorization does). */
static int lu_factor(const LUSym *lu, const double *jvals, int annz,
                     double gamma, double *LU, double *w) {
  int n = lu->n;
  for (int q = 0; q < lu->nnz; ++q) LU[q] = 0.0;
  for (int a = 0; a < annz; ++a) LU[lu->a_to_lu[a]] = -gamma * jvals[a];
  for (int i = 0; i < n; ++i) LU[lu->diag[i]] += 1.0;
  for (int i = 0; i < n; ++i) {
    for (int q = lu->rowptr[i]; q < lu->rowptr[i + 1]; ++q) w[lu->colidx[q]] = LU[q];
    for (int q = lu->rowptr[i]; q < lu->diag[i]; ++q) {
      int k = lu->colidx[q];
      double lik = w[k] / LU[lu->diag[k]];
      w[k] = lik;
      for (int p = lu->diag[k] + 1; p < lu->rowptr[k + 1]; ++p)
        w[lu->colidx[p]] -= lik * LU[p];
    }
    for (int q = lu->rowptr[i]; q < lu->rowptr[i + 1]; ++q) LU[q] = w[lu->colidx[q]];
    double piv = LU[lu->diag[i]];
    if (piv == 0.0 || !isfinite(piv)) return 1;
  }
  return 0;
}

/* Solves M x = b in place (b in original variable order). */
static void lu_solve(const LUSym *lu, const double *LU, double *b, double *z) {
  int n = lu->n;
  for (int i = 0; i < n; ++i) z[i] = b[lu->perm[i]];
  for (int i = 0; i < n; ++i) {
    double s = z[i];
    for (int q = lu->rowptr[i]; q < lu->diag[i]; ++q) s -= LU[q] * z[lu->colidx[q]];
    z[i] = s;
  }
  for (int i = n - 1; i >= 0; --i) {
    double s = z[i];
    for (int q = lu->diag[i] + 1; q < lu->rowptr[i + 1]; ++q)
      s -= LU[q] * z[lu->colidx[q]];
    z[i] = s / LU[lu->diag[i]];
  }
  for (int i = 0; i < n; ++i) b[lu->perm[i]] = z[i];
}

/* ------------------------------------------------------------------------ */
/* BDF integrator (restated CVODE algorithm, one cell)                       */
/* ------------------------------------------------------------------------ */

#define QMAX 5
#define LMAX (QMAX + 1)
#define ETAMX1 10000.0
#define ETAMX2 10.0
#define ETAMX3 10.0
#define ETAMXF 0.2
#define ETAMIN 0.1
#define ETACF 0.25
#define ADDON 0.000001
#define BIAS1 6.0
#define BIAS2 6.0
#define BIAS3 10.0
#define ONEPSM 1.000001
#define THRESH 1.5
#define SMALL_NST 10
#define MXNEF1 3
#define SMALL_NEF 2
#define LONG_WAIT 10
#define MAXCOR 3
#define CRDOWN 0.3
#define DGMAX 0.3
#define RDIV 2.0
#define MSBP 20
#define MSBJ 50
#define DGMAX_J 0.2
#define NLSCOEF 0.1
#define UROUND 2.220446049250313e-16

/* nonlinear solver outcomes */
#define NL_OK 0
#define NL_CONV_FAIL 1
#define NL_RHS_RECVR 2
#define NL_TRY_AGAIN 3
#define NL_CONSTR_RECVR 4
/* convfail values passed to the linear solver setup */
#define NO_FAILURES 0
#define FAIL_BAD_J 1
#define FAIL_OTHER 2
/* nflag values */
#define FIRST_CALL 0
#define PREV_CONV_FAIL 1
#define PREV_ERR_FAIL 2

typedef struct {
  const LUSym *lu;
  int n, annz;
  or_rhs_fn f;
  or_jac_fn jac;
  void *ctx;
  double rtol;
  const double *atol;
  int max_steps, maxncf, maxnef;
  /* work */
  double *zn[LMAX];
  double *ewt, *acor, *tempv, *ftemp, *y, *savedJ, *LU, *w, *z;
  /* state of the method */
  int q, qprime, qwait, L, indx_acor;
  double h, hprime, hscale, eta, etamax, hu, next_h;
  double tn, tau[LMAX + 1], tq[6], l[LMAX];
  double rl1, gamma, gammap, gamrat, crate, acnrm, saved_tq5;
  long nst, nfe, nsetups, netf, nni, ncfn, nje, nstlp, nstlj;
  int jcur;
  double etaqm1, etaq, etaqp1;
  /* experiment switches copied from the mechanism (om_set_experiment) */
  double guard_step;
  int positivity;
  double *yprev, *hfprev, *gtmp; /* guess-helper work (y_{n-1}, h f_{n-1}) */
} Bdf;

/* The step that f and J see as their time_step: the integrator's current
 * step (CVodeGetCurrentStep, src/camp_solver.c:872-876), or a fixed step
 * when an experiment sets one. */
static double f_step(const Bdf *b) { return b->guard_step > 0.0 ? b->guard_step : b->h; }

static double wrms(const double *v, const double *w, int n) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) {
    double t = v[i] * w[i];
    s += t * t;
  }
  return sqrt(s / n);
}

static int set_ewt(Bdf *b, const double *y) {
  for (int i = 0; i < b->n; ++i) {
    double t = b->rtol * fabs(y[i]) + b->atol[i];
    if (t <= 0.0) return 1;
    b->ewt[i] = 1.0 / t;
  }
  return 0;
}

static void bdf_rescale(Bdf *b) {
  double factor = b->eta;
  for (int j = 1; j <= b->q; ++j) {
    for (int i = 0; i < b->n; ++i) b->zn[j][i] *= factor;
    factor *= b->eta;
  }
  b->h = b->hscale * b->eta;
  b->next_h = b->h;
  b->hscale = b->h;
}

static void bdf_predict(Bdf *b) {
  b->tn += b->h;
  for (int k = 1; k <= b->q; ++k)
    for (int j = b->q; j >= k; --j)
      for (int i = 0; i < b->n; ++i) b->zn[j - 1][i] += b->zn[j][i];
}

static void bdf_restore(Bdf *b, double saved_t) {
  b->tn = saved_t;
  for (int k = 1; k <= b->q; ++k)
    for (int j = b->q; j >= k; --j)
      for (int i = 0; i < b->n; ++i) b->zn[j - 1][i] -= b->zn[j][i];
}

/* l and tq coefficients of the fixed-leading-coefficient BDF formula */
static void bdf_set(Bdf *b) {
  int q = b->q;
  double *l = b->l, *tau = b->tau;
  double alpha0, alpha0_hat, xi_inv, xistar_inv, hsum;
  l[0] = l[1] = xi_inv = xistar_inv = 1.0;
  for (int i = 2; i <= q; ++i) l[i] = 0.0;
  alpha0 = alpha0_hat = -1.0;
  hsum = b->h;
  if (q > 1) {
    for (int j = 2; j < q; ++j) {
      hsum += tau[j - 1];
      xi_inv = b->h / hsum;
      alpha0 -= 1.0 / j;
      for (int i = j; i >= 1; --i) l[i] += l[i - 1] * xi_inv;
    }
    alpha0 -= 1.0 / q;
    xistar_inv = -l[1] - alpha0;
    hsum += tau[q - 1];
    xi_inv = b->h / hsum;
    alpha0_hat = -l[1] - xi_inv;
    for (int i = q; i >= 1; --i) l[i] += l[i - 1] * xistar_inv;
  }
  /* test quantities */
  double A1 = 1.0 - alpha0_hat + alpha0;
  double A2 = 1.0 + q * A1;
  b->tq[2] = fabs(A1 / (alpha0 * A2));
  b->tq[5] = fabs(A2 * xistar_inv / (l[q] * xi_inv));
  if (b->qwait == 1) {
    if (q > 1) {
      double C = xistar_inv / l[q];
      double A3 = alpha0 + 1.0 / q;
      double A4 = alpha0_hat + xi_inv;
      double Cpinv = (1.0 - A4 + A3) / A3;
      b->tq[1] = fabs(C * Cpinv);
    } else {
      b->tq[1] = 1.0;
    }
    hsum += tau[q];
    xi_inv = b->h / hsum;
    double A5 = alpha0 - 1.0 / (q + 1);
    double A6 = alpha0_hat - xi_inv;
    double Cppinv = (1.0 - A6 + A5) / A2;
    b->tq[3] = fabs(Cppinv / (xi_inv * (q + 2) * A5));
  }
  b->tq[4] = NLSCOEF / b->tq[2];
  b->rl1 = 1.0 / l[1];
  b->gamma = b->h * b->rl1;
  if (b->nst == 0) b->gammap = b->gamma;
  b->gamrat = (b->nst > 0) ? b->gamma / b->gammap : 1.0;
}

static void bdf_increase_order(Bdf *b) {
  double *l = b->l;
  int q = b->q;
  for (int i = 0; i <= QMAX; ++i) l[i] = 0.0;
  l[2] = 1.0;
  double alpha1 = 1.0, prod = 1.0, xiold = 1.0, alpha0 = -1.0,
         hsum = b->hscale;
  if (q > 1) {
    for (int j = 1; j < q; ++j) {
      hsum += b->tau[j + 1];
      double xi = hsum / b->hscale;
      prod *= xi;
      alpha0 -= 1.0 / (j + 1);
      alpha1 += 1.0 / xi;
      for (int i = j + 2; i >= 2; --i) l[i] = l[i] * xiold + l[i - 1];
      xiold = xi;
    }
  }
  double A1 = (-alpha0 - alpha1) / prod;
  int Lnew = q + 2; /* zn[L] with L = q+1 becomes the new top column */
  (void)Lnew;
  for (int i = 0; i < b->n; ++i) b->zn[q + 1][i] = A1 * b->zn[b->indx_acor][i];
  for (int j = 2; j <= q; ++j)
    for (int i = 0; i < b->n; ++i) b->zn[j][i] += l[j] * b->zn[q + 1][i];
}

static void bdf_decrease_order(Bdf *b) {
  double *l = b->l;
  int q = b->q;
  for (int i = 0; i <= QMAX; ++i) l[i] = 0.0;
  l[2] = 1.0;
  double hsum = 0.0;
  for (int j = 1; j <= q - 2; ++j) {
    hsum += b->tau[j];
    double xi = hsum / b->hscale;
    for (int i = j + 2; i >= 2; --i) l[i] = l[i] * xi + l[i - 1];
  }
  for (int j = 2; j < q; ++j)
    for (int i = 0; i < b->n; ++i) b->zn[j][i] -= l[j] * b->zn[q][i];
}

static void bdf_adjust_order(Bdf *b, int deltaq) {
  if (deltaq == 1)
    bdf_increase_order(b);
  else if (deltaq == -1)
    bdf_decrease_order(b);
}

static void bdf_adjust_params(Bdf *b) {
  if (b->qprime != b->q) {
    bdf_adjust_order(b, b->qprime - b->q);
    b->q = b->qprime;
    b->L = b->q + 1;
    b->qwait = b->L;
  }
  bdf_rescale(b);
}

/* Linear solver setup: J reuse rule of the CVODE direct interface, then
 * M = I - gamma J factored. Returns 0, >0 recoverable, <0 fatal. */
static int bdf_lsetup(Bdf *b, int convfail, const double *ypred) {
  double dgamma = fabs(b->gamma / b->gammap - 1.0);
  int jbad = (b->nst == 0) || (b->nst > b->nstlj + MSBJ) ||
             ((convfail == FAIL_BAD_J) && (dgamma < DGMAX_J)) ||
             (convfail == FAIL_OTHER);
  if (!jbad) {
    b->jcur = 0;
  } else {
    b->nje++;
    b->nstlj = b->nst;
    b->jcur = 1;
    int r = b->jac(b->ctx, b->tn, ypred, f_step(b), b->savedJ);
    if (r < 0) return -1;
    if (r > 0) return 1;
  }
  return lu_factor(b->lu, b->savedJ, b->annz, b->gamma, b->LU, b->w);
}

static int bdf_newton_iteration(Bdf *b, int projected) {
  int n = b->n, m = 0;
  double del, delp = 0.0;
  for (;;) {
    for (int i = 0; i < n; ++i)
      b->tempv[i] = b->gamma * b->ftemp[i] - (b->rl1 * b->zn[1][i] + b->acor[i]);
    lu_solve(b->lu, b->LU, b->tempv, b->z);
    if (b->gamrat != 1.0) {
      double s = 2.0 / (1.0 + b->gamrat);
      for (int i = 0; i < n; ++i) b->tempv[i] *= s;
    }
    b->nni++;
    del = wrms(b->tempv, b->ewt, n);
    for (int i = 0; i < n; ++i) {
      b->acor[i] += b->tempv[i];
      b->y[i] = b->zn[0][i] + b->acor[i];
    }
    if (m > 0) b->crate = fmax(CRDOWN * b->crate, del / delp);
    double dcon = del * fmin(1.0, b->crate) / b->tq[4];
    if (dcon <= 1.0) {
      b->acnrm = (m == 0 && !projected) ? del : wrms(b->acor, b->ewt, n);
      b->jcur = 0;
      return NL_OK;
    }
    ++m;
    if ((m == MAXCOR) || ((m >= 2) && (del > RDIV * delp))) {
      if (!b->jcur) return NL_TRY_AGAIN;
      return NL_CONV_FAIL;
    }
    delp = del;
    int r = b->f(b->ctx, b->tn, b->y, f_step(b), b->ftemp);
    b->nfe++;
    if (r < 0) return -1;
    if (r > 0) {
      if (!b->jcur) return NL_TRY_AGAIN;
      return NL_RHS_RECVR;
    }
  }
}

/* Newton solve of one step; returns NL_OK, NL_CONV_FAIL, NL_RHS_RECVR,
 * NL_CONSTR_RECVR or negative for an unrecoverable failure (OR_* codes).
 *
 * Positivity: the reference's f rejects any concentration below -1e-30
 * (src/camp_solver.c:805-833) and its modified CVODE steers around negative
 * predictions with a guess helper (src/camp_solver.c:1321-1408) whose call
 * sites are in the missing CVODE source.  This restatement instead
 *   (a) starts the Newton iteration from the predicted state with negative
 *       components raised to zero (acor starts at that projection), and
 *   (b) applies CVODE's published non-negativity constraint check to the
 *       converged iterate (cvCheckConstraints, SUNDIALS >= 5.0): a violation
 *       whose WRMS norm is within the Newton tolerance tq[4] is projected to
 *       zero, a larger one rejects the step with eta = max(0.1, 0.9 * min over
 *       violated i of zn0_i / (zn0_i - y_i)). */
static int bdf_check_constraints(Bdf *b) {
  int n = b->n, viol = 0;
  for (int i = 0; i < n; ++i)
    if (b->y[i] < 0.0) {
      viol = 1;
      break;
    }
  if (!viol) return NL_OK;
  double s = 0.0;
  for (int i = 0; i < n; ++i)
    if (b->y[i] < 0.0) {
      double t = b->y[i] * b->ewt[i];
      s += t * t;
    }
  double vnorm = sqrt(s / n);
  if (vnorm <= b->tq[4]) {
    for (int i = 0; i < n; ++i)
      if (b->y[i] < 0.0) {
        b->acor[i] -= b->y[i];
        b->y[i] = 0.0;
      }
    b->acnrm = wrms(b->acor, b->ewt, n);
    return NL_OK;
  }
  double eta = 1.0e300;
  for (int i = 0; i < n; ++i)
    if (b->y[i] < 0.0) {
      double d = b->zn[0][i] - b->y[i];
      double qv = b->zn[0][i] / d;
      if (qv < eta) eta = qv;
    }
  eta *= 0.9;
  b->eta = eta > 0.1 ? eta : 0.1;
  return NL_CONSTR_RECVR;
}

/* Restatement of the reference's guess_helper (src/camp_solver.c:1321-1408)
 * in its prediction form (h_n > 0), for the positivity experiments: when the
 * predicted state has a value below -SMALL, advance y_{n-1} over the step by
 * at most GUESS_MAX_ITER explicit Euler sub-steps, each cut just short of the
 * first zero crossing (x 0.95 + 0.1 iter / GUESS_MAX_ITER), re-evaluating f
 * after each, and start Newton from 0.999 of the resulting correction.  The
 * modified CVODE's call site is not in the reference tree; this calls it once
 * per prediction.  Returns 1 when acor holds a correction, 0 when none was
 * needed, -1 when f failed. */
#define GUESS_MAX_ITER 5
static int guess_helper(Bdf *b) {
  int n = b->n;
  double ymin = b->zn[0][0];
  for (int i = 1; i < n; ++i) ymin = b->zn[0][i] < ymin ? b->zn[0][i] : ymin;
  if (ymin > -SMALL) return 0;
  double h_n = b->h, t_n = b->tn;
  double *y = b->gtmp, *f = b->acor;
  memcpy(y, b->yprev, sizeof(double) * n);
  for (int i = 0; i < n; ++i) f[i] = b->hfprev[i] / h_n;
  double t_0 = t_n - h_n, t_j = 0.0;
  for (int iter = 0; iter < GUESS_MAX_ITER && t_0 + t_j < t_n; iter++) {
    double h_j = t_n - (t_0 + t_j);
    int i_fast = -1;
    for (int i = 0; i < n; i++) {
      double t_star = -y[i] / f[i];
      if ((t_star > 0.0 || (t_star == 0.0 && f[i] < 0.0)) && t_star < h_j) {
        h_j = t_star;
        i_fast = i;
      }
    }
    if (i_fast >= 0) h_j *= 0.95 + 0.1 * iter / (double)GUESS_MAX_ITER;
    if (t_n < t_0 + t_j + h_j) h_j = t_n - (t_0 + t_j);
    for (int i = 0; i < n; ++i) y[i] += h_j * f[i];
    t_j += h_j;
    int r = b->f(b->ctx, t_0 + t_j, y, f_step(b), f);
    b->nfe++;
    if (r != 0) return -1;
  }
  for (int i = 0; i < n; ++i) b->acor[i] = 0.999 * (y[i] - b->zn[0][i]);
  return 1;
}

static int bdf_nls(Bdf *b, int nflag) {
  int convfail = ((nflag == FIRST_CALL) || (nflag == PREV_ERR_FAIL))
                     ? NO_FAILURES
                     : FAIL_OTHER;
  int call_setup = (nflag == PREV_CONV_FAIL) || (nflag == PREV_ERR_FAIL) ||
                   (b->nst == 0) || (b->nst >= b->nstlp + MSBP) ||
                   (fabs(b->gamrat - 1.0) > DGMAX);
  int projected = 0;
  if (b->positivity == OM_POS_GUESS_HELPER || b->positivity == OM_POS_GUESS_HELPER_ONLY) {
    projected = guess_helper(b) == 1;
    for (int i = 0; i < b->n; ++i) {
      if (!projected) b->acor[i] = 0.0;
      b->y[i] = b->zn[0][i] + b->acor[i];
    }
  } else {
    int project = b->positivity == OM_POS_PROJECT;
    for (int i = 0; i < b->n; ++i) {
      double a = (project && b->zn[0][i] < 0.0) ? -b->zn[0][i] : 0.0;
      if (a != 0.0) projected = 1;
      b->acor[i] = a;
      b->y[i] = b->zn[0][i] + a;
    }
  }
  for (;;) {
    int r = b->f(b->ctx, b->tn, b->y, f_step(b), b->ftemp);
    b->nfe++;
    if (r < 0) return OR_RHSFUNC_FAIL;
    if (r > 0) return NL_RHS_RECVR;
    if (call_setup) {
      int ier = bdf_lsetup(b, convfail, b->y);
      b->nsetups++;
      call_setup = 0;
      b->gamrat = b->crate = 1.0;
      b->gammap = b->gamma;
      b->nstlp = b->nst;
      if (ier < 0) return OR_LSETUP_FAIL;
      if (ier > 0) return NL_CONV_FAIL;
    }
    int ier = bdf_newton_iteration(b, projected);
    if (ier < 0) return OR_RHSFUNC_FAIL;
    if (ier == NL_OK)
      return (b->positivity == OM_POS_PROJECT || b->positivity == OM_POS_GUESS_HELPER)
                 ? bdf_check_constraints(b)
                 : NL_OK;
    if (ier != NL_TRY_AGAIN) return ier;
    call_setup = 1;
    convfail = FAIL_BAD_J;
    for (int i = 0; i < b->n; ++i) {
      double a = (b->positivity == OM_POS_PROJECT && b->zn[0][i] < 0.0) ? -b->zn[0][i] : 0.0;
      b->acor[i] = a;
      b->y[i] = b->zn[0][i] + a;
    }
  }
}

#define DO_ERROR_TEST 100
#define PREDICT_AGAIN 101
#define TRY_AGAIN 102

static int bdf_handle_nflag(Bdf *b, int *nflag, double saved_t, int *ncf) {
  int nf = *nflag;
  if (nf == NL_OK) return DO_ERROR_TEST;
  b->ncfn++;
  bdf_restore(b, saved_t);
  if (nf < 0) return nf;
  (*ncf)++;
  b->etamax = 1.0;
  if (*ncf == b->maxncf)
    return nf == NL_RHS_RECVR ? OR_REPTD_RHSFUNC_ERR : OR_CONV_FAILURE;
  if (nf != NL_CONSTR_RECVR) b->eta = ETACF;
  *nflag = PREV_CONV_FAIL;
  bdf_rescale(b);
  return PREDICT_AGAIN;
}

static int bdf_error_test(Bdf *b, int *nflag, double saved_t, int *nef,
                          double *dsm) {
  *dsm = b->acnrm * b->tq[2];
  if (*dsm <= 1.0) return OR_SUCCESS;
  (*nef)++;
  b->netf++;
  *nflag = PREV_ERR_FAIL;
  bdf_restore(b, saved_t);
  if (*nef == b->maxnef) return OR_ERR_FAILURE;
  b->etamax = 1.0;
  if (*nef <= MXNEF1) {
    b->eta = 1.0 / (pow(BIAS2 * *dsm, 1.0 / b->L) + ADDON);
    b->eta = fmax(ETAMIN, b->eta);
    if (*nef >= SMALL_NEF) b->eta = fmin(b->eta, ETAMXF);
    bdf_rescale(b);
    return TRY_AGAIN;
  }
  if (b->q > 1) {
    b->eta = ETAMIN;
    bdf_adjust_order(b, -1);
    b->L = b->q;
    b->q--;
    b->qwait = b->L;
    bdf_rescale(b);
    return TRY_AGAIN;
  }
  b->eta = ETAMIN;
  b->h *= b->eta;
  b->next_h = b->h;
  b->hscale = b->h;
  b->qwait = LONG_WAIT;
  int r = b->f(b->ctx, b->tn, b->zn[0], f_step(b), b->tempv);
  b->nfe++;
  if (r < 0) return OR_RHSFUNC_FAIL;
  if (r > 0) return OR_UNREC_RHSFUNC_ERR;
  for (int i = 0; i < b->n; ++i) b->zn[1][i] = b->h * b->tempv[i];
  return TRY_AGAIN;
}

static void bdf_complete_step(Bdf *b) {
  b->nst++;
  b->hu = b->h;
  for (int i = b->q; i >= 2; --i) b->tau[i] = b->tau[i - 1];
  if ((b->q == 1) && (b->nst > 1)) b->tau[2] = b->tau[1];
  b->tau[1] = b->h;
  for (int j = 0; j <= b->q; ++j)
    for (int i = 0; i < b->n; ++i) b->zn[j][i] += b->l[j] * b->acor[i];
  b->qwait--;
  if ((b->qwait == 1) && (b->q != QMAX)) {
    memcpy(b->zn[QMAX], b->acor, sizeof(double) * b->n);
    b->saved_tq5 = b->tq[5];
    b->indx_acor = QMAX;
  }
}

static void bdf_set_eta(Bdf *b) {
  if (b->eta < THRESH) {
    b->eta = 1.0;
    b->hprime = b->h;
  } else {
    b->eta = fmin(b->eta, b->etamax);
    b->hprime = b->h * b->eta;
  }
}

static void bdf_prepare_next_step(Bdf *b, double dsm) {
  if (b->etamax == 1.0) {
    b->qwait = b->qwait > 2 ? b->qwait : 2;
    b->qprime = b->q;
    b->hprime = b->h;
    b->eta = 1.0;
    return;
  }
  b->etaq = 1.0 / (pow(BIAS2 * dsm, 1.0 / b->L) + ADDON);
  if (b->qwait != 0) {
    b->eta = b->etaq;
    b->qprime = b->q;
    bdf_set_eta(b);
    return;
  }
  b->qwait = 2;
  /* eta for order q-1 */
  b->etaqm1 = 0.0;
  if (b->q > 1) {
    double ddn = wrms(b->zn[b->q], b->ewt, b->n) * b->tq[1];
    b->etaqm1 = 1.0 / (pow(BIAS1 * ddn, 1.0 / b->q) + ADDON);
  }
  /* eta for order q+1 */
  b->etaqp1 = 0.0;
  if (b->q != QMAX && b->saved_tq5 != 0.0) {
    double cquot = (b->tq[5] / b->saved_tq5) * pow(b->h / b->tau[2], b->L);
    for (int i = 0; i < b->n; ++i)
      b->tempv[i] = b->acor[i] - cquot * b->zn[QMAX][i];
    double dup = wrms(b->tempv, b->ewt, b->n) * b->tq[3];
    b->etaqp1 = 1.0 / (pow(BIAS3 * dup, 1.0 / (b->L + 1)) + ADDON);
  }
  /* choose */
  double etam = fmax(b->etaqm1, fmax(b->etaq, b->etaqp1));
  if (etam < THRESH) {
    b->eta = 1.0;
    b->qprime = b->q;
  } else if (etam == b->etaq) {
    b->eta = b->etaq;
    b->qprime = b->q;
  } else if (etam == b->etaqm1) {
    b->eta = b->etaqm1;
    b->qprime = b->q - 1;
  } else {
    b->eta = b->etaqp1;
    b->qprime = b->q + 1;
    memcpy(b->zn[QMAX], b->acor, sizeof(double) * b->n);
  }
  bdf_set_eta(b);
}

static int bdf_step(Bdf *b) {
  double saved_t = b->tn, dsm = 0.0;
  int ncf = 0, nef = 0, nflag = FIRST_CALL;
  if ((b->nst > 0) && (b->hprime != b->h)) bdf_adjust_params(b);
  for (;;) {
    if (b->positivity == OM_POS_GUESS_HELPER || b->positivity == OM_POS_GUESS_HELPER_ONLY) {
      memcpy(b->yprev, b->zn[0], sizeof(double) * b->n);
      memcpy(b->hfprev, b->zn[1], sizeof(double) * b->n);
    }
    bdf_predict(b);
    bdf_set(b);
    nflag = bdf_nls(b, nflag);
    int kflag = bdf_handle_nflag(b, &nflag, saved_t, &ncf);
    if (kflag == PREDICT_AGAIN) continue;
    if (kflag != DO_ERROR_TEST) return kflag;
    int eflag = bdf_error_test(b, &nflag, saved_t, &nef, &dsm);
    if (eflag == TRY_AGAIN) continue;
    if (eflag != OR_SUCCESS) return eflag;
    break;
  }
  bdf_complete_step(b);
  bdf_prepare_next_step(b, dsm);
  b->etamax = (b->nst <= SMALL_NST) ? ETAMX2 : ETAMX3;
  for (int i = 0; i < b->n; ++i) b->acor[i] *= b->tq[2];
  return OR_SUCCESS;
}

/* Interpolated solution at t from the Nordsieck array (CVodeGetDky, k=0). */
static void bdf_dky(const Bdf *b, double t, double *out) {
  double s = (t - b->tn) / b->h;
  for (int i = 0; i < b->n; ++i) {
    double v = b->zn[b->q][i];
    for (int j = b->q - 1; j >= 0; --j) v = b->zn[j][i] + s * v;
    out[i] = v;
  }
}

typedef struct {
  double *mem;
} BdfWork;

static void bdf_alloc(Bdf *b, BdfWork *wk, int n, int annz, int lunnz) {
  size_t tot = (size_t)n * (LMAX + 11) + (size_t)annz + (size_t)lunnz;
  wk->mem = (double *)zalloc(sizeof(double) * (tot + 8));
  double *p = wk->mem;
  for (int j = 0; j < LMAX; ++j, p += n) b->zn[j] = p;
  b->ewt = p; p += n;
  b->acor = p; p += n;
  b->tempv = p; p += n;
  b->ftemp = p; p += n;
  b->y = p; p += n;
  b->w = p; p += n;
  b->z = p; p += n;
  b->savedJ = p; p += annz;
  b->LU = p; p += lunnz;
  b->yprev = p; p += n;
  b->hfprev = p; p += n;
  b->gtmp = p;
}

/* One cell from t0 to tout with initial step h0 (CVodeReInit + CVode in
 * CV_NORMAL mode with CVodeSetInitStep(h0), src/camp_solver.c:619-633). */
static int bdf_integrate(Bdf *b, double t0, double tout, double h0, double *y,
                         OracleStats *st) {
  int n = b->n;
  memset(b->tau, 0, sizeof(b->tau));
  memset(b->tq, 0, sizeof(b->tq));
  b->q = 1;
  b->L = 2;
  b->qwait = b->L;
  b->etamax = ETAMX1;
  b->qprime = 1;
  b->nst = b->nfe = b->nsetups = b->netf = b->nni = b->ncfn = b->nje = 0;
  b->nstlp = b->nstlj = 0;
  b->saved_tq5 = 0.0;
  b->indx_acor = QMAX;
  b->crate = 1.0;
  b->jcur = 0;
  b->hu = 0.0;
  b->tn = t0;
  b->gammap = b->gamma = 0.0;
  memcpy(b->zn[0], y, sizeof(double) * n);
  for (int j = 1; j < LMAX; ++j) memset(b->zn[j], 0, sizeof(double) * n);
  int flag = OR_SUCCESS;
  if (set_ewt(b, b->zn[0])) {
    flag = OR_ILL_INPUT;
    goto done;
  }
  b->next_h = 0.0;
  {
    int r = b->f(b->ctx, t0, b->zn[0], b->guard_step > 0.0 ? b->guard_step : h0, b->zn[1]);
    b->nfe++;
    if (r != 0) {
      flag = r < 0 ? OR_RHSFUNC_FAIL : OR_REPTD_RHSFUNC_ERR;
      goto done;
    }
  }
  b->h = h0;
  /* CVODE with a zero initial step estimates one (cvHin), which refuses an
   * output time at the initial time: CV_TOO_CLOSE */
  if (h0 == 0.0) {
    flag = OR_TOO_CLOSE;
    goto done;
  }
  if ((tout - t0) * b->h < 0.0) {
    flag = OR_ILL_INPUT;
    goto done;
  }
  b->hscale = b->h;
  b->hprime = b->h;
  for (int i = 0; i < n; ++i) b->zn[1][i] *= b->h;
  long nstloc = 0;
  for (;;) {
    b->next_h = b->h;
    if (b->nst > 0 && set_ewt(b, b->zn[0])) {
      flag = OR_ILL_INPUT;
      break;
    }
    if (b->max_steps > 0 && nstloc >= b->max_steps) {
      flag = OR_TOO_MUCH_WORK;
      break;
    }
    double tolsf = UROUND * wrms(b->zn[0], b->ewt, n);
    if (tolsf > 1.0) {
      flag = OR_TOO_MUCH_ACC;
      break;
    }
    int kflag = bdf_step(b);
    if (kflag != OR_SUCCESS) {
      flag = kflag;
      break;
    }
    nstloc++;
    if ((b->tn - tout) * b->h >= 0.0) {
      bdf_dky(b, tout, y);
      b->next_h = b->hprime;
      break;
    }
  }
done:
  if (st) {
    st->nst = b->nst;
    st->nfe = b->nfe;
    st->nsetups = b->nsetups;
    st->netf = b->netf;
    st->nni = b->nni;
    st->ncfn = b->ncfn;
    st->nje = b->nje;
    st->hu = b->hu;
    st->hcur = b->next_h;
    st->flag = flag;
    st->qu = b->q;
  }
  return flag;
}

/* ------------------------------------------------------------------------ */
/* Oracle's own f/J as BDF callbacks                                         */
/* ------------------------------------------------------------------------ */

typedef struct {
  const OracleMech *m;
  double *state;         /* one cell's state (constants kept, deps overwritten) */
  const double *rxn_env; /* one cell's rate constants */
  double *scratch_rp;
  double h0;
} CellCtx;

/* src/camp_solver.c:805-833: y < -SMALL is a recoverable failure; other
 * values are copied (exactly -SMALL becomes TINY). */
static int load_state(CellCtx *c, const double *y) {
  const OracleMech *m = c->m;
  for (int i = 0, d = 0; i < m->n_state; ++i) {
    if (m->var_type[i] != VAR_VARIABLE) continue;
    if (y[d] < -SMALL) return 1;
    c->state[i] = y[d] > -SMALL ? y[d] : TINY;
    ++d;
  }
  return 0;
}

static int cell_rhs(void *ctx, double t, const double *y, double h,
                    double *ydot) {
  (void)t;
  CellCtx *c = (CellCtx *)ctx;
  if (load_state(c, y)) return 1;
  double ts = h > 0.0 ? h : c->h0;
  om_deriv(c->m, c->state, c->rxn_env, ts, ydot, NULL, NULL);
  return 0;
}

static int cell_jac(void *ctx, double t, const double *y, double h,
                    double *jvals) {
  (void)t;
  CellCtx *c = (CellCtx *)ctx;
  if (load_state(c, y)) return 1;
  om_jac(c->m, c->state, c->rxn_env, h > 0.0 ? h : c->h0, jvals);
  return 0;
}

typedef struct {
  const OracleMech *m;
  int c0, c1;
  double *state;
  const double *env;
  double *rxn_env;
  double t0, t1, rtol;
  const double *abs_tol;
  int max_steps, max_conv_fails;
  int *status;
  OracleStats *stats;
  int n_fail;
} SolveJob;

static void *solve_job(void *arg) {
  SolveJob *jb = (SolveJob *)arg;
  const OracleMech *m = jb->m;
  int n = m->n_dep, ns = m->n_state;
  Bdf b;
  memset(&b, 0, sizeof(b));
  BdfWork wk;
  bdf_alloc(&b, &wk, n, m->n_solver_jac, m->lu.nnz);
  double *atol = (double *)zalloc(sizeof(double) * (n + 1));
  for (int i = 0, d = 0; i < ns; ++i)
    if (m->var_type[i] == VAR_VARIABLE) atol[d++] = jb->abs_tol[i];
  double *y = (double *)zalloc(sizeof(double) * (n + 1));
  b.lu = &m->lu;
  b.n = n;
  b.annz = m->n_solver_jac;
  b.f = cell_rhs;
  b.jac = cell_jac;
  b.rtol = jb->rtol;
  b.atol = atol;
  b.max_steps = jb->max_steps;
  b.maxncf = jb->max_conv_fails;
  b.maxnef = jb->max_conv_fails;
  b.guard_step = m->guard_step;
  b.positivity = m->positivity;
  CellCtx ctx;
  ctx.m = m;
  b.ctx = &ctx;
  for (int c = jb->c0; c < jb->c1; ++c) {
    double *st = jb->state + (size_t)c * ns;
    double *re = jb->rxn_env + (size_t)c * om_n_rxn_env_data(m);
    /* solver_run: dependent values clamped to >= TINY, constants too
     * (src/camp_solver.c:554-567); rate constants from env (:587-603) */
    for (int i = 0, d = 0; i < ns; ++i) {
      if (m->var_type[i] == VAR_VARIABLE)
        y[d++] = st[i] > TINY ? st[i] : TINY;
      else if (m->var_type[i] == 2)
        st[i] = st[i] > TINY ? st[i] : TINY;
    }
    om_update_env(m, jb->env + 2 * (size_t)c, re);
    ctx.state = st;
    ctx.rxn_env = re;
    ctx.h0 = jb->t1 - jb->t0;
    OracleStats s;
    int flag = bdf_integrate(&b, jb->t0, jb->t1, jb->t1 - jb->t0, y, &s);
    if (jb->status) jb->status[c] = flag;
    if (jb->stats) jb->stats[c] = s;
    if (flag != OR_SUCCESS) {
      jb->n_fail++;
      continue;
    }
    for (int i = 0, d = 0; i < ns; ++i)
      if (m->var_type[i] == VAR_VARIABLE) {
        st[i] = y[d] > 0.0 ? y[d] : 0.0;
        ++d;
      }
    /* the species the sub-models compute, at the final concentrations */
    if (m->n_sub > 0) sub_calculate(m, st, re);
  }
  free(wk.mem);
  free(atol);
  free(y);
  return NULL;
}

/* The absolute tolerances solver_initialize receives (per state variable):
 * they set the aqueous equilibrium's minimum water. */
void om_set_abs_tol(const OracleMech *m, const double *abs_tol) { aq_thresholds(m, abs_tol); }

int om_set_experiment(OracleMech *m, double guard_step, int positivity) {
  if (guard_step < 0.0 || positivity < OM_POS_PROJECT || positivity > OM_POS_NONE) return 1;
  m->guard_step = guard_step;
  m->positivity = positivity;
  return 0;
}

int om_solve(const OracleMech *m, int n_cells, double *state, const double *env,
             double *rxn_env, double t0, double t1, double rtol,
             const double *abs_tol, int max_steps, int max_conv_fails,
             int n_threads, int *status, OracleStats *stats) {
  if (!m->built) return -1;
  aq_thresholds(m, abs_tol);
  if (n_threads < 1) n_threads = 1;
  if (n_threads > n_cells) n_threads = n_cells > 0 ? n_cells : 1;
  SolveJob *jobs = (SolveJob *)zalloc(sizeof(SolveJob) * n_threads);
  pthread_t *th = (pthread_t *)zalloc(sizeof(pthread_t) * n_threads);
  for (int t = 0; t < n_threads; ++t) {
    SolveJob *jb = &jobs[t];
    jb->m = m;
    jb->c0 = (int)((long)n_cells * t / n_threads);
    jb->c1 = (int)((long)n_cells * (t + 1) / n_threads);
    jb->state = state;
    jb->env = env;
    jb->rxn_env = rxn_env;
    jb->t0 = t0;
    jb->t1 = t1;
    jb->rtol = rtol;
    jb->abs_tol = abs_tol;
    jb->max_steps = max_steps;
    jb->max_conv_fails = max_conv_fails;
    jb->status = status;
    jb->stats = stats;
  }
  if (n_threads == 1) {
    solve_job(&jobs[0]);
  } else {
    for (int t = 0; t < n_threads; ++t)
      pthread_create(&th[t], NULL, solve_job, &jobs[t]);
    for (int t = 0; t < n_threads; ++t) pthread_join(th[t], NULL);
  }
  int nf = 0;
  for (int t = 0; t < n_threads; ++t) nf += jobs[t].n_fail;
  free(jobs);
  free(th);
  return nf;
}

int om_solve_cb(const OracleMech *m, int n_cells, double *y_dep, double t0,
                double t1, double rtol, const double *abs_tol_dep,
                int max_steps, int max_conv_fails, or_rhs_fn f, or_jac_fn jac,
                void **ctxs, int *status, OracleStats *stats) {
  if (!m->built) return -1;
  int n = m->n_dep;
  Bdf b;
  memset(&b, 0, sizeof(b));
  BdfWork wk;
  bdf_alloc(&b, &wk, n, m->n_solver_jac, m->lu.nnz);
  b.lu = &m->lu;
  b.n = n;
  b.annz = m->n_solver_jac;
  b.f = f;
  b.jac = jac;
  b.rtol = rtol;
  b.atol = abs_tol_dep;
  b.max_steps = max_steps;
  b.maxncf = max_conv_fails;
  b.maxnef = max_conv_fails;
  b.guard_step = m->guard_step;
  b.positivity = m->positivity;
  int nf = 0;
  for (int c = 0; c < n_cells; ++c) {
    b.ctx = ctxs[c];
    double *y = y_dep + (size_t)c * n;
    OracleStats s;
    int flag = bdf_integrate(&b, t0, t1, t1 - t0, y, &s);
    if (status) status[c] = flag;
    if (stats) stats[c] = s;
    if (flag != OR_SUCCESS) nf++;
  }
  free(wk.mem);
  return nf;
}
