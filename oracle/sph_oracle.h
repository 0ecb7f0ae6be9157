/*
 * ORACLE - test infrastructure only. Not part of the product.
 *
 * CPU restatement (C11 + OpenMP) of the reference's explicit SPH step
 * (leap_frog::step, leap_frog.cu:94-155, and everything it calls). Every function in
 * sph_oracle.c cites the reference file:line it restates. Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load this library, and only
 * as the checker / the reported CPU baseline.
 *
 * Parity pinning: the scene setup, tool geometry, SPH kernel functions and the
 * Johnson-Cook yield/secant functions are checked bit-for-bit against the reference's own
 * sources compiled on the host (oracle/_ref/libref_host.so, see oracle/build_oracle.py).
 * The device-only kernel bodies (pair loop, per-particle actions, contact, sort/reorder)
 * are restated line by line from the reference source and pinned against the reference's
 * own CUDA build: its device sources compiled unchanged for sm_100a with a shim for the
 * texture-reference API that CUDA 12 removed (oracle/ref_gpu, oracle/_ref/libref_gpu.so and
 * the PSE build libref_gpu_pse.so), compared live on a GPU and through golden vectors of its
 * outputs (tests/golden/ref_gpu_steps.npz) on any host.
 *
 * Layout mirrors particle_gpu (particle_gpu.h:33-87): SoA arrays of doubles, vector fields
 * interleaved (pos = x0 y0 x1 y1 ..., S = xx xy yy zz per particle), flags stored as
 * doubles 0/1, idx/hash as int.
 */
#ifndef MF_SPH_ORACLE_H
#define MF_SPH_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* field ids: same numbering as the product's MF_FIELD_* (include/mfree_b200.h) */
enum {
  ORC_POS = 0, ORC_VEL = 1, ORC_H = 2, ORC_RHO = 3, ORC_P = 4, ORC_S = 5, ORC_R = 6,
  ORC_FC = 7, ORC_FT = 8, ORC_N = 9, ORC_FIXED = 10, ORC_BLANKED = 11, ORC_TOOL = 12,
  ORC_EPS_PL = 13, ORC_EPS_PL_DOT = 14, ORC_T = 15, ORC_POS_T = 16, ORC_VEL_T = 17,
  ORC_RHO_T = 18, ORC_S_T = 19, ORC_T_T = 20, ORC_S_DER = 21, ORC_V_DER = 22,
  ORC_IDX = 23, ORC_HASH = 24, ORC_NUM_FIELDS = 25
};

typedef struct { double E, nu, rho0, K, G, mass, mass_tool; } orc_phys;        /* constants_structs.h:25-33 */
typedef struct { double cp, tq, k, alpha, T_init, eta; } orc_trml;             /* constants_structs.h:37-44 */
typedef struct { double wdeltap, stresseps, xspheps, alpha, beta, eta; } orc_corr; /* :48-55 */
typedef struct {
  double A, B, C, n, m, Tmelt, Tref, eps_dot_ref, tanh_a, tanh_b, tanh_c, tanh_d;
} orc_joco;                                                                    /* :59-72 */

/* tool_gpu.cuh:32-52 */
typedef struct {
  double left[2], right[2];
  double a, b;
  int vertical;
  double n[2];
} orc_segment;
typedef struct { double r, t1, t2, p[2]; } orc_fillet;
typedef struct {
  int num_seg;
  orc_segment seg[5];
  int has_fillet;
  orc_fillet fillet;
  double mu, contact_alpha, slave_mass;
  double vel[2];
} orc_tool;

typedef struct orc_state orc_state;

orc_state *orc_create(int N);
void orc_destroy(orc_state *s);
int orc_num(const orc_state *s);
/* current pointer of a field (the Green sort swaps buffers, so re-query after a sort) */
void *orc_field(orc_state *s, int field);
int orc_field_width(int field); /* doubles (or ints) per particle */

void orc_set_threads(int n);
int orc_get_threads(void);

/* constants (actions_setup_* / interactions_setup_*). joco may be NULL (no plasticity). */
void orc_set_constants(orc_state *s, const orc_phys *phys, const orc_corr *corr, const orc_joco *joco,
                       const orc_trml *trml_wp, const orc_trml *trml_tool);
/* thermal_solver: 0 Brookshaw, 1 PSE. jc_model: 0 Johnson-Cook, 1 tanh variant */
void orc_set_options(orc_state *s, int thermal_solver, int jc_model);
/* The reference's own per-particle functions in place of this file's restatements at their call
   sites: kernels.cuh cubic_spline and lapl_pse, plasticity.cuh sigma_yield and solve_secant (the
   Johnson-Cook law; the tanh law keeps the restatement), compiled for the host by
   oracle/build_oracle.py (refh_cubic_spline, refh_lapl_pse, refh_sigma_yield,
   refh_solve_secant_jc). The Johnson-Cook constants are passed as the 12 doubles of orc_joco.
   NULL pointers restore the restatements. */
typedef void (*orc_ref_kernel_fn)(double xi, double yi, double xj, double yj, double hi, double *out3);
typedef double (*orc_ref_pse_fn)(double xi, double yi, double xj, double yj, double hi);
typedef double (*orc_ref_yield_fn)(const double *jc12, double eps_pl, double eps_pl_dot, double T);
typedef double (*orc_ref_secant_fn)(const double *jc12, double init, double tol, double norm_Strial,
                                    double eps_pl_init, double T, double dt, double mu);
void orc_set_reference_functions(orc_state *s, orc_ref_kernel_fn kernel, orc_ref_pse_fn pse,
                                 orc_ref_yield_fn yield, orc_ref_secant_fn secant);
void orc_set_dt(orc_state *s, double dt);
/* grid_kind: 0 Green, 1 Rothlin. Locked bbox (grid.cu:139-158) */
int orc_set_grid_locked(orc_state *s, int grid_kind, double bbmin_x, double bbmin_y, double bbmax_x,
                        double bbmax_y, double h);
/* adaptive grid (grid.cu:97-136) with a cell budget */
int orc_set_grid_adaptive(orc_state *s, int grid_kind, int max_cell);
/* geometry: nx ny num_cell ; bbmin_x bbmin_y bbmax_x bbmax_y dx */
void orc_get_geometry(const orc_state *s, int *iout3, double *dout5);
int *orc_cells(orc_state *s, int which); /* 0 start, 1 end (leap_frog copies) */
int orc_num_cell(const orc_state *s);
/* NULL tool -> no tool (contact and friction heat off) */
void orc_set_tool(orc_state *s, const orc_tool *tool);
void orc_get_tool(const orc_state *s, orc_tool *out);

/* stages of leap_frog::step (leap_frog.cu:94-155) */
int orc_grid_update(orc_state *s);      /* update_geometry + assign_hashes + sort + get_cells */
void orc_stage_predict(orc_state *s);   /* init + predict + eos + artificial stress */
void orc_stage_interact(orc_state *s);  /* interactions_monaghan (+Brookshaw) [+ PSE] */
void orc_stage_rates(orc_state *s);     /* jaumann, continuity, momentum, advection */
void orc_stage_finish(orc_state *s);    /* correct .. invalidate */
int orc_step(orc_state *s);             /* one complete step */
int orc_steps(orc_state *s, int n);
int orc_steps_force_log(orc_state *s, int n, double *out); /* report_force after each step */
void orc_usui(orc_state *s, double K, double alpha, double tool_vx, double tool_vy, double out3[3]); /* tool_wear.cu:20-64 */
void orc_report_force(orc_state *s, double out2[2]); /* output.cu:31-39 */
long long orc_out_of_grid(const orc_state *s);       /* hashes clamped so far */

/* single functions (for unit tests against the host-compiled reference) */
void orc_cubic_spline(double xi, double yi, double xj, double yj, double hi, double *out3);
double orc_lapl_pse(double xi, double yi, double xj, double yj, double hi);
double orc_sigma_yield(const orc_joco *jc, double eps_pl, double eps_pl_dot, double t);
double orc_sigma_yield_tanh(const orc_joco *jc, double eps_pl, double eps_pl_dot, double t);
double orc_solve_secant(const orc_joco *jc, int model, double init, double tol, double norm_Strial,
                        double eps_pl_init, double t, double delta_t, double mu, int *iters);
void orc_line_from_points(double x1, double y1, double x2, double y2, double *a, double *b, int *vertical);

#ifdef __cplusplus
}
#endif
#endif
