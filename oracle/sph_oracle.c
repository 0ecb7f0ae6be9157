/*
 * ORACLE - test infrastructure only. Not part of the product.
 * CPU restatement of the reference step; see sph_oracle.h for the scope and the pinning.
 *
 * Arithmetic follows the reference expressions term by term and in the same evaluation
 * order, including the float-precision calls the reference makes on double arguments
 * (sqrtf, atan2f, cosf, sinf, fmaxf narrow to float: kernels.cuh:50, actions_gpu.cu:38,47,
 * 76-77,145,159,239,252,264-265, interactions_gpu.cu:293-294). Built with
 * -ffp-contract=off: no fused multiply-add anywhere.
 */
#include "sph_oracle.h"

#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PI_FAC 0.454728408833987 /* kernels.cuh:28 */
#define TOOL_MAX_SEG 5           /* tool_gpu.cuh:52 */

typedef struct { double x, y; } d2;
typedef struct { double x, y, z, w; } d4;

struct orc_state {
  int N;
  /* particle_gpu (particle_gpu.h:33-87); *_b are the Green double buffer (grid_gpu_green.h:38-72) */
  d2 *pos, *vel, *fc, *ft, *n, *pos_t, *vel_t;
  double *h, *rho, *p, *fixed, *blanked, *tool_particle, *eps_pl, *eps_pl_dot, *T, *rho_t, *T_t;
  d4 *S, *R, *S_t, *S_der, *v_der;
  int *idx, *hash;
  /* Green buffer (swap mode, grid_gpu_green.h:54) */
  d2 *b_pos, *b_vel, *b_fc, *b_ft, *b_pos_t, *b_vel_t;
  double *b_h, *b_rho, *b_eps_pl, *b_eps_pl_dot, *b_T, *b_fixed, *b_blanked, *b_tool, *b_rho_t, *b_T_t;
  d4 *b_S, *b_S_t;
  /* leap_frog (leap_frog.h:36-50) */
  d2 *pos_init, *vel_init;
  d4 *S_init;
  double *rho_init, *T_init;
  int *cell_start, *cell_end;
  /* grid_base (grid.h:32-73) */
  int grid_kind, locked, max_cell;
  double dx, lx, ly, bbmin_x, bbmin_y, bbmax_x, bbmax_y;
  int nx, ny, num_cell;
  int *g_cell_start, *g_cell_end; /* the grid's own arrays (Green) */
  int *perm;                      /* scratch: sort values */
  /* constants */
  orc_phys phys;
  orc_corr corr;
  orc_joco joco;
  orc_trml trml_wp, trml_tool;
  int plastic, thermal_bc, fric_heat, thermal_wp, thermal_tool_on;
  int thermal_solver, jc_model;
  int has_tool;
  orc_tool tool;
  double dt;
  long long out_of_grid;
  /* the reference's host-compiled functions, when set (orc_set_reference_functions) */
  orc_ref_kernel_fn ref_kernel;
  orc_ref_pse_fn ref_pse;
  orc_ref_yield_fn ref_yield;
  orc_ref_secant_fn ref_secant;
};

static int g_threads = 0;
void orc_set_threads(int n) { g_threads = n; }
int orc_get_threads(void) {
#ifdef _OPENMP
  return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
  return 1;
#endif
}
#ifdef _OPENMP
#define OMP_FOR _Pragma("omp parallel for schedule(static) num_threads(orc_get_threads())")
#define OMP_FOR_DYN _Pragma("omp parallel for schedule(dynamic, 256) num_threads(orc_get_threads())")
#else
#define OMP_FOR
#define OMP_FOR_DYN
#endif

static void *xcalloc(size_t n, size_t sz) {
  void *p = calloc(n ? n : 1, sz);
  return p;
}

orc_state *orc_create(int N) {
  orc_state *s = (orc_state *)xcalloc(1, sizeof(orc_state));
  s->N = N;
#define A2(f) s->f = (d2 *)xcalloc((size_t)N, sizeof(d2))
#define A1(f) s->f = (double *)xcalloc((size_t)N, sizeof(double))
#define A4(f) s->f = (d4 *)xcalloc((size_t)N, sizeof(d4))
  A2(pos); A2(vel); A2(fc); A2(ft); A2(n); A2(pos_t); A2(vel_t);
  A1(h); A1(rho); A1(p); A1(fixed); A1(blanked); A1(tool_particle); A1(eps_pl); A1(eps_pl_dot);
  A1(T); A1(rho_t); A1(T_t);
  A4(S); A4(R); A4(S_t); A4(S_der); A4(v_der);
  A2(b_pos); A2(b_vel); A2(b_fc); A2(b_ft); A2(b_pos_t); A2(b_vel_t);
  A1(b_h); A1(b_rho); A1(b_eps_pl); A1(b_eps_pl_dot); A1(b_T); A1(b_fixed); A1(b_blanked);
  A1(b_tool); A1(b_rho_t); A1(b_T_t);
  A4(b_S); A4(b_S_t);
  A2(pos_init); A2(vel_init); A4(S_init); A1(rho_init); A1(T_init);
#undef A1
#undef A2
#undef A4
  s->idx = (int *)xcalloc((size_t)N, sizeof(int));
  s->hash = (int *)xcalloc((size_t)N, sizeof(int));
  s->perm = (int *)xcalloc((size_t)N, sizeof(int));
  for (int i = 0; i < N; ++i) s->idx[i] = i; /* particle_gpu.cu:53-54 */
  s->corr.wdeltap = 1.;                      /* make_corr_constants, constants_structs.cpp:31-35 */
  return s;
}

void orc_destroy(orc_state *s) {
  if (!s) return;
  void *ptrs[] = {s->pos, s->vel, s->fc, s->ft, s->n, s->pos_t, s->vel_t, s->h, s->rho, s->p, s->fixed,
                  s->blanked, s->tool_particle, s->eps_pl, s->eps_pl_dot, s->T, s->rho_t, s->T_t, s->S,
                  s->R, s->S_t, s->S_der, s->v_der, s->idx, s->hash, s->b_pos, s->b_vel, s->b_fc, s->b_ft,
                  s->b_pos_t, s->b_vel_t, s->b_h, s->b_rho, s->b_eps_pl, s->b_eps_pl_dot, s->b_T,
                  s->b_fixed, s->b_blanked, s->b_tool, s->b_rho_t, s->b_T_t, s->b_S, s->b_S_t,
                  s->pos_init, s->vel_init, s->S_init, s->rho_init, s->T_init, s->cell_start,
                  s->cell_end, s->g_cell_start, s->g_cell_end, s->perm};
  for (size_t k = 0; k < sizeof(ptrs) / sizeof(ptrs[0]); ++k) free(ptrs[k]);
  free(s);
}

int orc_num(const orc_state *s) { return s->N; }

void *orc_field(orc_state *s, int f) {
  switch (f) {
    case ORC_POS: return s->pos;
    case ORC_VEL: return s->vel;
    case ORC_H: return s->h;
    case ORC_RHO: return s->rho;
    case ORC_P: return s->p;
    case ORC_S: return s->S;
    case ORC_R: return s->R;
    case ORC_FC: return s->fc;
    case ORC_FT: return s->ft;
    case ORC_N: return s->n;
    case ORC_FIXED: return s->fixed;
    case ORC_BLANKED: return s->blanked;
    case ORC_TOOL: return s->tool_particle;
    case ORC_EPS_PL: return s->eps_pl;
    case ORC_EPS_PL_DOT: return s->eps_pl_dot;
    case ORC_T: return s->T;
    case ORC_POS_T: return s->pos_t;
    case ORC_VEL_T: return s->vel_t;
    case ORC_RHO_T: return s->rho_t;
    case ORC_S_T: return s->S_t;
    case ORC_T_T: return s->T_t;
    case ORC_S_DER: return s->S_der;
    case ORC_V_DER: return s->v_der;
    case ORC_IDX: return s->idx;
    case ORC_HASH: return s->hash;
    default: return NULL;
  }
}

int orc_field_width(int f) {
  switch (f) {
    case ORC_POS: case ORC_VEL: case ORC_FC: case ORC_FT: case ORC_N: case ORC_POS_T: case ORC_VEL_T:
      return 2;
    case ORC_S: case ORC_R: case ORC_S_T: case ORC_S_DER: case ORC_V_DER:
      return 4;
    default:
      return 1;
  }
}

/* actions_setup_* (actions_gpu.cu:438-469) and interactions_setup_* (interactions_gpu.cu:433-459) */
void orc_set_constants(orc_state *s, const orc_phys *phys, const orc_corr *corr, const orc_joco *joco,
                       const orc_trml *trml_wp, const orc_trml *trml_tool) {
  if (phys) s->phys = *phys;
  if (corr) s->corr = *corr;
  s->plastic = 0;
  if (joco) { s->joco = *joco; s->plastic = 1; }
  memset(&s->trml_wp, 0, sizeof(orc_trml));
  memset(&s->trml_tool, 0, sizeof(orc_trml));
  if (trml_wp) s->trml_wp = *trml_wp;
  if (trml_tool) s->trml_tool = *trml_tool;
  s->fric_heat = s->trml_wp.eta != 0.;        /* actions_gpu.cu:457-460 */
  s->thermal_bc = s->trml_tool.alpha != 0.;   /* actions_gpu.cu:466-468 */
  s->thermal_wp = s->trml_wp.alpha != 0.;     /* interactions_gpu.cu:443 */
  s->thermal_tool_on = s->trml_tool.alpha != 0.; /* interactions_gpu.cu:453 */
}

void orc_set_reference_functions(orc_state *s, orc_ref_kernel_fn kernel, orc_ref_pse_fn pse,
                                 orc_ref_yield_fn yield, orc_ref_secant_fn secant) {
  s->ref_kernel = kernel;
  s->ref_pse = pse;
  s->ref_yield = yield;
  s->ref_secant = secant;
}

void orc_set_options(orc_state *s, int thermal_solver, int jc_model) {
  s->thermal_solver = thermal_solver;
  s->jc_model = jc_model;
}

void orc_set_dt(orc_state *s, double dt) { s->dt = dt; }

static int alloc_cells(orc_state *s, int max_cell) {
  free(s->cell_start); free(s->cell_end); free(s->g_cell_start); free(s->g_cell_end);
  s->cell_start = (int *)xcalloc((size_t)max_cell + 1, sizeof(int));
  s->cell_end = (int *)xcalloc((size_t)max_cell + 1, sizeof(int));
  s->g_cell_start = (int *)xcalloc((size_t)max_cell + 1, sizeof(int));
  s->g_cell_end = (int *)xcalloc((size_t)max_cell + 1, sizeof(int));
  return s->cell_start && s->cell_end && s->g_cell_start && s->g_cell_end ? 0 : -1;
}

/* grid_base::set_geometry (grid.cu:139-158) */
int orc_set_grid_locked(orc_state *s, int grid_kind, double bbmin_x, double bbmin_y, double bbmax_x,
                        double bbmax_y, double h) {
  s->grid_kind = grid_kind;
  s->bbmin_x = bbmin_x - 1e-6;
  s->bbmin_y = bbmin_y - 1e-6;
  s->bbmax_x = bbmax_x + 1e-6;
  s->bbmax_y = bbmax_y + 1e-6;
  double kernel_width = 2.;
  s->dx = h * kernel_width / 2.;
  s->lx = s->bbmax_x - s->bbmin_x;
  s->ly = s->bbmax_y - s->bbmin_y;
  s->nx = (int)(unsigned int)ceil(s->lx / s->dx);
  s->ny = (int)(unsigned int)ceil(s->ly / s->dx);
  s->num_cell = s->nx * s->ny;
  s->max_cell = s->num_cell;
  s->locked = 1;
  return alloc_cells(s, s->max_cell);
}

/* grid_base(int max_cell, int num_part) (grid.cu:160-162) */
int orc_set_grid_adaptive(orc_state *s, int grid_kind, int max_cell) {
  s->grid_kind = grid_kind;
  s->locked = 0;
  s->max_cell = max_cell;
  s->num_cell = max_cell;
  return alloc_cells(s, max_cell);
}

void orc_get_geometry(const orc_state *s, int *iout3, double *dout5) {
  iout3[0] = s->nx; iout3[1] = s->ny; iout3[2] = s->num_cell;
  dout5[0] = s->bbmin_x; dout5[1] = s->bbmin_y; dout5[2] = s->bbmax_x; dout5[3] = s->bbmax_y;
  dout5[4] = s->dx;
}

int *orc_cells(orc_state *s, int which) { return which == 0 ? s->cell_start : s->cell_end; }
int orc_num_cell(const orc_state *s) { return s->num_cell; }
long long orc_out_of_grid(const orc_state *s) { return s->out_of_grid; }

void orc_set_tool(orc_state *s, const orc_tool *t) {
  if (!t || t->num_seg <= 0) { s->has_tool = 0; memset(&s->tool, 0, sizeof(orc_tool)); return; }
  s->has_tool = 1;
  s->tool = *t;
}
void orc_get_tool(const orc_state *s, orc_tool *out) { *out = s->tool; }

/* ------------------------------------------------------------------------------------- */
/* grid */

/* grid_base::update_geometry (grid.cu:97-136). thrust::min_element/max_element return the
   first extremal element; the comparisons below keep the first one as well. */
static int update_geometry(orc_state *s) {
  if (s->locked) return 0;
  int N = s->N;
  if (N <= 0) return 0;
  int iminx = 0, iminy = 0, imaxx = 0, imaxy = 0, imaxh = 0;
  for (int i = 1; i < N; ++i) {
    if (s->pos[i].x < s->pos[iminx].x) iminx = i;
    if (s->pos[i].y < s->pos[iminy].y) iminy = i;
    if (s->pos[imaxx].x < s->pos[i].x) imaxx = i;
    if (s->pos[imaxy].y < s->pos[i].y) imaxy = i;
    if (s->h[imaxh] < s->h[i]) imaxh = i;
  }
  s->bbmin_x = s->pos[iminx].x - 1e-6;
  s->bbmin_y = s->pos[iminy].y - 1e-6;
  s->bbmax_x = s->pos[imaxx].x + 1e-6;
  s->bbmax_y = s->pos[imaxy].y + 1e-6;
  double kernel_width = 2.0;
  s->dx = s->h[imaxh] * kernel_width / 2;
  s->lx = s->bbmax_x - s->bbmin_x;
  s->ly = s->bbmax_y - s->bbmin_y;
  s->nx = (int)(unsigned int)ceil(s->lx / s->dx);
  s->ny = (int)(unsigned int)ceil(s->ly / s->dx);
  s->num_cell = s->nx * s->ny;
  if (!(s->num_cell < s->max_cell)) return -1; /* grid.cu:135 assert */
  return 0;
}

/* CUDA's double->int conversion saturates and maps NaN to 0 (cvt.rzi.s32.f64). */
static int trunc_sat(double v) {
  if (v != v) return 0;
  if (v >= 2147483647.0) return INT_MAX;
  if (v <= -2147483648.0) return INT_MIN;
  return (int)v;
}

/* compute_hashes (grid.cu:34-51). Blanked particles keep their previous hash (:39-41).
   A hash outside [0, num_cell) is undefined behaviour in the reference (the reorder kernel
   writes cell_start[hash]); here it is clamped to the nearest valid cell and counted. */
static void assign_hashes(orc_state *s) {
  long long oog = 0;
  for (int i = 0; i < s->N; ++i) {
    long long hsh;
    if (s->blanked[i] == 1.) {
      hsh = s->hash[i];
    } else {
      int ix = trunc_sat((s->pos[i].x - s->bbmin_x) / s->dx);
      int iy = trunc_sat((s->pos[i].y - s->bbmin_y) / s->dx);
      hsh = (long long)ix * (long long)s->ny + (long long)iy;
    }
    if (hsh < 0) { hsh = 0; ++oog; }
    else if (hsh >= s->num_cell) { hsh = s->num_cell - 1; ++oog; }
    s->hash[i] = (int)hsh;
  }
  s->out_of_grid += oog;
}

/* stable sort by hash, values = 0..N-1 (thrust::sequence + thrust::sort_by_key,
   grid_gpu_green.cu:179-185; grid_gpu_rothlin.cu:141-181). A counting sort is stable. */
static void stable_sort_by_hash(orc_state *s) {
  int N = s->N, nc = s->num_cell;
  int *cnt = (int *)xcalloc((size_t)nc + 1, sizeof(int));
  for (int i = 0; i < N; ++i) cnt[s->hash[i] + 1]++;
  for (int c = 0; c < nc; ++c) cnt[c + 1] += cnt[c];
  int *keys = (int *)xcalloc((size_t)N, sizeof(int));
  for (int i = 0; i < N; ++i) {
    int dst = cnt[s->hash[i]]++;
    s->perm[dst] = i;
    keys[dst] = s->hash[i];
  }
  memcpy(s->hash, keys, sizeof(int) * (size_t)N);
  free(keys);
  free(cnt);
}

#define SWAPP(a, b) do { void *t_ = (void *)(a); *(void **)&(a) = (void *)(b); *(void **)&(b) = t_; } while (0)

/* grid_gpu_green::sort -> do_sort (grid_gpu_green.cu:177-205), swap mode:
   reorder_data_and_find_cell_start (:22-116) then double_buffer (:149-175). */
static void sort_green(orc_state *s) {
  int N = s->N;
  stable_sort_by_hash(s);
  for (int i = 0; i < N; ++i) s->idx[i] = s->perm[i];
  for (int c = 0; c < s->num_cell; ++c) s->g_cell_start[c] = -1; /* cudaMemset 0xff (:187) */
  for (int i = 0; i < N; ++i) {
    int hsh = s->hash[i];
    if (i == 0 || hsh != s->hash[i - 1]) {
      s->g_cell_start[hsh] = i;
      if (i > 0) s->g_cell_end[s->hash[i - 1]] = i;
    }
    if (i == N - 1) s->g_cell_end[hsh] = i + 1;
  }
  OMP_FOR
  for (int i = 0; i < N; ++i) {
    int k = s->idx[i];
    s->b_pos[i] = s->pos[k]; s->b_vel[i] = s->vel[k]; s->b_fc[i] = s->fc[k]; s->b_ft[i] = s->ft[k];
    s->b_h[i] = s->h[k]; s->b_rho[i] = s->rho[k]; s->b_S[i] = s->S[k]; s->b_eps_pl[i] = s->eps_pl[k];
    s->b_eps_pl_dot[i] = s->eps_pl_dot[k]; s->b_T[i] = s->T[k]; s->b_fixed[i] = s->fixed[k];
    s->b_blanked[i] = s->blanked[k]; s->b_tool[i] = s->tool_particle[k];
    s->b_pos_t[i] = s->pos_t[k]; s->b_vel_t[i] = s->vel_t[k]; s->b_rho_t[i] = s->rho_t[k];
    s->b_S_t[i] = s->S_t[k]; s->b_T_t[i] = s->T_t[k];
  }
  SWAPP(s->pos, s->b_pos); SWAPP(s->vel, s->b_vel); SWAPP(s->fc, s->b_fc); SWAPP(s->ft, s->b_ft);
  SWAPP(s->h, s->b_h); SWAPP(s->rho, s->b_rho); SWAPP(s->S, s->b_S); SWAPP(s->eps_pl, s->b_eps_pl);
  SWAPP(s->eps_pl_dot, s->b_eps_pl_dot); SWAPP(s->T, s->b_T); SWAPP(s->fixed, s->b_fixed);
  SWAPP(s->blanked, s->b_blanked); SWAPP(s->tool_particle, s->b_tool);
  SWAPP(s->pos_t, s->b_pos_t); SWAPP(s->vel_t, s->b_vel_t); SWAPP(s->rho_t, s->b_rho_t);
  SWAPP(s->S_t, s->b_S_t); SWAPP(s->T_t, s->b_T_t);
}

/* grid_gpu_rothlin::sort (grid_gpu_rothlin.cu:138-250): gathers of idx and 17 fields;
   ft is not among them (it stays in place). */
static void sort_rothlin(orc_state *s) {
  int N = s->N;
  stable_sort_by_hash(s);
  int *ti = (int *)xcalloc((size_t)N, sizeof(int));
  for (int i = 0; i < N; ++i) ti[i] = s->idx[s->perm[i]];
  memcpy(s->idx, ti, sizeof(int) * (size_t)N);
  free(ti);
  OMP_FOR
  for (int i = 0; i < N; ++i) {
    int k = s->perm[i];
    s->b_pos[i] = s->pos[k]; s->b_vel[i] = s->vel[k]; s->b_fc[i] = s->fc[k];
    s->b_h[i] = s->h[k]; s->b_rho[i] = s->rho[k]; s->b_S[i] = s->S[k]; s->b_eps_pl[i] = s->eps_pl[k];
    s->b_eps_pl_dot[i] = s->eps_pl_dot[k]; s->b_fixed[i] = s->fixed[k]; s->b_blanked[i] = s->blanked[k];
    s->b_tool[i] = s->tool_particle[k]; s->b_T[i] = s->T[k];
    s->b_pos_t[i] = s->pos_t[k]; s->b_vel_t[i] = s->vel_t[k]; s->b_rho_t[i] = s->rho_t[k];
    s->b_S_t[i] = s->S_t[k]; s->b_T_t[i] = s->T_t[k];
  }
  /* gather to temp then copy back: same values as a swap */
  SWAPP(s->pos, s->b_pos); SWAPP(s->vel, s->b_vel); SWAPP(s->fc, s->b_fc);
  SWAPP(s->h, s->b_h); SWAPP(s->rho, s->b_rho); SWAPP(s->S, s->b_S); SWAPP(s->eps_pl, s->b_eps_pl);
  SWAPP(s->eps_pl_dot, s->b_eps_pl_dot); SWAPP(s->T, s->b_T); SWAPP(s->fixed, s->b_fixed);
  SWAPP(s->blanked, s->b_blanked); SWAPP(s->tool_particle, s->b_tool);
  SWAPP(s->pos_t, s->b_pos_t); SWAPP(s->vel_t, s->b_vel_t); SWAPP(s->rho_t, s->b_rho_t);
  SWAPP(s->S_t, s->b_S_t); SWAPP(s->T_t, s->b_T_t);
}

/* grid_gpu_green::get_cells (grid_gpu_green.cu:207-210): copy; empty cells start = -1 and
   their cell_end is left as it was. grid_gpu_rothlin::get_cells (grid_gpu_rothlin.cu:129-136):
   start[c] = number of particles with hash < c, end[c] = start[c+1]. */
static void get_cells(orc_state *s) {
  int nc = s->num_cell;
  if (s->grid_kind == 0) {
    memcpy(s->cell_start, s->g_cell_start, sizeof(int) * (size_t)nc);
    memcpy(s->cell_end, s->g_cell_end, sizeof(int) * (size_t)nc);
  } else {
    int k = 0;
    for (int c = 0; c < nc; ++c) {
      s->cell_start[c] = k;
      while (k < s->N && s->hash[k] <= c) ++k;
      s->cell_end[c] = k;
    }
  }
}

int orc_grid_update(orc_state *s) {
  if (update_geometry(s) != 0) return -1;
  assign_hashes(s);
  if (s->grid_kind == 0) sort_green(s); else sort_rothlin(s);
  get_cells(s);
  return 0;
}

/* ------------------------------------------------------------------------------------- */
/* SPH kernel functions (kernels.cuh:30-89) */

typedef struct { double x, y, z; } d3;

static inline d3 cubic_spline(d2 posi, d2 posj, double hi) {
  d3 w; w.x = 0.; w.y = 0.; w.z = 0.;
  double xij = posi.x - posj.x;
  double yij = posi.y - posj.y;
  double rr2 = xij * xij + yij * yij;
  double h1 = 1 / hi;
  double fourh2 = 4 * hi * hi;
  if (rr2 >= fourh2 || rr2 < 1e-8) return w;
  double der, val;
  double rad = sqrtf((float)rr2);
  double q = rad * h1;
  double fac = PI_FAC * h1 * h1;
  const int radgt = q > 1;
  if (radgt) {
    double _2mq = 2 - q;
    double _2mq2 = _2mq * _2mq;
    val = 0.25 * _2mq2 * _2mq2 * _2mq2;
    der = -0.75 * _2mq2 * h1 / rad;
  } else {
    val = 1 - 1.5 * q * q * (1 - 0.5 * q);
    der = -3.0 * q * (1 - 0.75 * q) * h1 / rad;
  }
  w.x = val * fac;
  w.y = der * xij * fac;
  w.z = der * yij * fac;
  return w;
}

static inline double lapl_pse(d2 posi, d2 posj, double hi) {
  double xij = posi.x - posj.x;
  double yij = posi.y - posj.y;
  double xx = sqrt(xij * xij + yij * yij);
  double h2 = hi * hi;
  double h4 = h2 * h2;
  double w2_pse = +4. / (h4 * M_PI) * exp(-xx * xx / (h2));
  return w2_pse;
}

void orc_cubic_spline(double xi, double yi, double xj, double yj, double hi, double *out3) {
  d2 a = {xi, yi}, b = {xj, yj};
  d3 w = cubic_spline(a, b, hi);
  out3[0] = w.x; out3[1] = w.y; out3[2] = w.z;
}
double orc_lapl_pse(double xi, double yi, double xj, double yj, double hi) {
  d2 a = {xi, yi}, b = {xj, yj};
  return lapl_pse(a, b, hi);
}

/* ------------------------------------------------------------------------------------- */
/* leap frog (leap_frog.cu:30-92) */

static void lf_init(orc_state *s) {
  OMP_FOR
  for (int i = 0; i < s->N; ++i) {
    if (s->blanked[i] == 1.) continue;
    s->pos_init[i] = s->pos[i];
    s->vel_init[i] = s->vel[i];
    s->S_init[i] = s->S[i];
    s->rho_init[i] = s->rho[i];
    s->T_init[i] = s->T[i];
  }
}

static void lf_predict(orc_state *s) {
  double dt = s->dt;
  OMP_FOR
  for (int i = 0; i < s->N; ++i) {
    if (s->blanked[i] == 1.) continue;
    s->pos[i].x = s->pos_init[i].x + 0.5 * dt * s->pos_t[i].x;
    s->pos[i].y = s->pos_init[i].y + 0.5 * dt * s->pos_t[i].y;
    s->vel[i].x = s->vel_init[i].x + 0.5 * dt * s->vel_t[i].x;
    s->vel[i].y = s->vel_init[i].y + 0.5 * dt * s->vel_t[i].y;
    s->S[i].x = s->S_init[i].x + 0.5 * dt * s->S_t[i].x;
    s->S[i].y = s->S_init[i].y + 0.5 * dt * s->S_t[i].y;
    s->S[i].z = s->S_init[i].z + 0.5 * dt * s->S_t[i].z;
    s->S[i].w = s->S_init[i].w + 0.5 * dt * s->S_t[i].w;
    s->rho[i] = s->rho_init[i] + 0.5 * dt * s->rho_t[i];
    s->T[i] = s->T_init[i] + 0.5 * dt * s->T_t[i];
  }
}

static void lf_correct(orc_state *s) {
  double dt = s->dt;
  OMP_FOR
  for (int i = 0; i < s->N; ++i) {
    if (s->blanked[i] == 1.) continue;
    s->pos[i].x = s->pos_init[i].x + dt * s->pos_t[i].x;
    s->pos[i].y = s->pos_init[i].y + dt * s->pos_t[i].y;
    s->vel[i].x = s->vel_init[i].x + dt * s->vel_t[i].x;
    s->vel[i].y = s->vel_init[i].y + dt * s->vel_t[i].y;
    s->S[i].x = s->S_init[i].x + dt * s->S_t[i].x;
    s->S[i].y = s->S_init[i].y + dt * s->S_t[i].y;
    s->S[i].z = s->S_init[i].z + dt * s->S_t[i].z;
    s->S[i].w = s->S_init[i].w + dt * s->S_t[i].w;
    s->rho[i] = s->rho_init[i] + dt * s->rho_t[i];
    s->T[i] = s->T_init[i] + dt * s->T_t[i];
  }
}

/* ------------------------------------------------------------------------------------- */
/* per-particle actions (actions_gpu.cu) */

/* do_material_eos (actions_gpu.cu:41-51) */
static void material_eos(orc_state *s) {
  double rho0 = s->phys.rho0;
  double c0 = sqrtf((float)(s->phys.K / rho0));
  OMP_FOR
  for (int i = 0; i < s->N; ++i) {
    if (s->tool_particle[i] != 0.) continue;
    double rhoi = s->rho[i];
    s->p[i] = c0 * c0 * (rhoi - rho0);
  }
}

/* stress_angle (actions_gpu.cu:35-39) */
static inline double stress_angle(double sxx, double sxy, double syy, double eps) {
  double numer = 2. * sxy;
  double denom = sxx - syy + eps;
  return 0.5 * atan2f((float)numer, (float)denom);
}

/* do_corrector_artificial_stress (actions_gpu.cu:53-97) */
static void corrector_artificial_stress(orc_state *s) {
  double eps = s->corr.stresseps;
  OMP_FOR
  for (int i = 0; i < s->N; ++i) {
    if (s->tool_particle[i] != 0.) continue;
    double rhoi = s->rho[i];
    double pi = s->p[i];
    d4 Si = s->S[i];
    double sxx = Si.x, sxy = Si.y, syy = Si.z;
    sxx -= pi;
    syy -= pi;
    double rhoi21 = 1. / (rhoi * rhoi);
    double theta = stress_angle(sxx, sxy, syy, 0.);
    double cos_theta = cosf((float)theta);
    double sin_theta = sinf((float)theta);
    double cos_theta2 = cos_theta * cos_theta;
    double sin_theta2 = sin_theta * sin_theta;
    double rot_sxx = cos_theta2 * sxx + 2.0 * cos_theta * sin_theta * sxy + sin_theta2 * syy;
    double rot_syy = sin_theta2 * sxx - 2.0 * cos_theta * sin_theta * sxy + cos_theta2 * syy;
    double rot_rxx = 0., rot_ryy = 0.;
    if (rot_sxx > 0) rot_rxx = -eps * rot_sxx * rhoi21;
    if (rot_syy > 0) rot_ryy = -eps * rot_syy * rhoi21;
    d4 Ri;
    Ri.x = cos_theta2 * rot_rxx + sin_theta2 * rot_ryy;
    Ri.y = cos_theta * sin_theta * (rot_rxx - rot_ryy);
    Ri.z = sin_theta2 * rot_rxx + cos_theta2 * rot_ryy;
    Ri.w = 0.;
    s->R[i] = Ri;
  }
}

/* 3x3 column-major helpers with GLM semantics (m[c][r], products summed left to right) */
typedef struct { double m[3][3]; } mat3;
static inline mat3 mat3_make(double x0, double y0, double z0, double x1, double y1, double z1, double x2,
                             double y2, double z2) {
  mat3 r;
  r.m[0][0] = x0; r.m[0][1] = y0; r.m[0][2] = z0;
  r.m[1][0] = x1; r.m[1][1] = y1; r.m[1][2] = z1;
  r.m[2][0] = x2; r.m[2][1] = y2; r.m[2][2] = z2;
  return r;
}
static inline mat3 mat3_mul(mat3 a, mat3 b) {
  mat3 r;
  for (int c = 0; c < 3; ++c)
    for (int w = 0; w < 3; ++w) r.m[c][w] = (a.m[0][w] * b.m[c][0] + a.m[1][w] * b.m[c][1]) + a.m[2][w] * b.m[c][2];
  return r;
}
static inline mat3 mat3_transpose(mat3 a) {
  mat3 r;
  for (int c = 0; c < 3; ++c)
    for (int w = 0; w < 3; ++w) r.m[c][w] = a.m[w][c];
  return r;
}
static inline mat3 mat3_add(mat3 a, mat3 b) {
  mat3 r;
  for (int c = 0; c < 3; ++c)
    for (int w = 0; w < 3; ++w) r.m[c][w] = a.m[c][w] + b.m[c][w];
  return r;
}
static inline mat3 mat3_sub(mat3 a, mat3 b) {
  mat3 r;
  for (int c = 0; c < 3; ++c)
    for (int w = 0; w < 3; ++w) r.m[c][w] = a.m[c][w] - b.m[c][w];
  return r;
}
static inline mat3 mat3_scale(double s, mat3 a) {
  mat3 r;
  for (int c = 0; c < 3; ++c)
    for (int w = 0; w < 3; ++w) r.m[c][w] = s * a.m[c][w];
  return r;
}

/* do_material_stress_rate_jaumann (actions_gpu.cu:99-133) */
static void stress_rate_jaumann(orc_state *s) {
  double G = s->phys.G;
  OMP_FOR
  for (int i = 0; i < s->N; ++i) {
    if (s->tool_particle[i] == 1.) continue;
    d4 vi_der = s->v_der[i];
    d4 Si = s->S[i];
    double vx_x = vi_der.x, vx_y = vi_der.y, vy_x = vi_der.z, vy_y = vi_der.w;
    double Sxx = Si.x, Sxy = Si.y, Syy = Si.z, Szz = Si.w;
    mat3 epsdot = mat3_make(vx_x, 0.5 * (vx_y + vy_x), 0., 0.5 * (vx_y + vy_x), vy_y, 0., 0., 0., 0.);
    mat3 omega = mat3_make(0., 0.5 * (vy_x - vx_y), 0., 0.5 * (vx_y - vy_x), 0., 0., 0., 0., 0.);
    mat3 S = mat3_make(Sxx, Sxy, 0., Sxy, Syy, 0., 0., 0., Szz);
    mat3 I = mat3_make(1., 0., 0., 0., 1., 0., 0., 0., 1.);
    double trace_epsdot = epsdot.m[0][0] + epsdot.m[1][1] + epsdot.m[2][2];
    mat3 dev = mat3_sub(epsdot, mat3_scale((double)(1. / 3.) * trace_epsdot, I));
    mat3 Si_t = mat3_add(mat3_add(mat3_scale((double)(2.) * G, dev), mat3_mul(omega, S)),
                         mat3_mul(S, mat3_transpose(omega)));
    s->S_t[i].x = Si_t.m[0][0];
    s->S_t[i].y = Si_t.m[0][1];
    s->S_t[i].z = Si_t.m[1][1];
    s->S_t[i].w = Si_t.m[2][2];
  }
}

/* do_material_fric_heat_gen (actions_gpu.cu:135-162) */
static void fric_heat_gen(orc_state *s) {
  double eta = s->trml_wp.eta, dt = s->dt;
  d2 vel_tool = {s->tool.vel[0], s->tool.vel[1]};
  OMP_FOR
  for (int i = 0; i < s->N; ++i) {
    if (s->tool_particle[i] != 0.) continue;
    d2 f_T = s->ft[i];
    double f_fric_mag = sqrtf((float)(f_T.x * f_T.x + f_T.y * f_T.y));
    if (f_fric_mag == 0.) continue;
    d2 normal = s->n[i];
    d2 v_particle = s->vel[i];
    d2 v_diff = {v_particle.x - vel_tool.x, v_particle.y - vel_tool.y};
    double v_diff_dot_normal = v_diff.x * normal.x + v_diff.y * normal.y;
    d2 v_relative = {v_diff.x - v_diff_dot_normal, v_diff.y - v_diff_dot_normal};
    double v_rel_mag = sqrtf((float)(v_relative.x * v_relative.x + v_relative.y * v_relative.y));
    s->T[i] += eta * dt * f_fric_mag * v_rel_mag / (s->trml_wp.cp * s->phys.mass);
  }
}

/* do_contmech_continuity / momentum / advection (actions_gpu.cu:164-224) */
static void contmech(orc_state *s) {
  double mass = s->phys.mass;
  OMP_FOR
  for (int i = 0; i < s->N; ++i) {
    if (s->tool_particle[i] != 0.) continue;
    double rhoi = s->rho[i];
    d4 vi_der = s->v_der[i];
    s->rho_t[i] = -rhoi * (vi_der.x + vi_der.w);
  }
  OMP_FOR
  for (int i = 0; i < s->N; ++i) {
    if (s->tool_particle[i] != 0.) continue;
    d4 Si_der = s->S_der[i];
    d2 fci = s->fc[i], fti = s->ft[i];
    d2 veli_t = s->vel_t[i];
    veli_t.x += Si_der.x + Si_der.y + fci.x / mass + fti.x / mass;
    veli_t.y += Si_der.z + Si_der.w + fci.y / mass + fti.y / mass;
    s->vel_t[i] = veli_t;
  }
  OMP_FOR
  for (int i = 0; i < s->N; ++i) {
    if (s->tool_particle[i] != 0.) continue;
    d2 veli = s->vel[i];
    d2 posi_t = s->pos_t[i];
    s->pos_t[i].x = posi_t.x + veli.x;
    s->pos_t[i].y = posi_t.y + veli.y;
  }
}

/* plasticity.cuh:30-46 */
double orc_sigma_yield(const orc_joco *jc, double eps_pl, double eps_pl_dot, double t) {
  double theta = (t - jc->Tref) / (jc->Tmelt - jc->Tref);
  double Term_A = jc->A + jc->B * pow(eps_pl, jc->n);
  double Term_B = 1.0;
  double eps_dot = eps_pl_dot / jc->eps_dot_ref;
  if (eps_dot > 1.0) {
    Term_B = 1.0 + jc->C * log(eps_dot);
  } else {
    Term_B = pow((1.0 + eps_dot), jc->C);
  }
  double Term_C = 1.0 - pow(theta, jc->m);
  return Term_A * Term_B * Term_C;
}

/* plasticity.cuh:48-70 */
double orc_sigma_yield_tanh(const orc_joco *jc, double eps_pl, double eps_dot_pl, double t) {
  double theta = (t - jc->Tref) / (jc->Tmelt - jc->Tref);
  double Term_A = jc->A + jc->B * pow(eps_pl, jc->n) * 1.0 / exp(pow(eps_pl, jc->tanh_a));
  double Term_B = 1.0;
  double eps_dot = eps_dot_pl / jc->eps_dot_ref;
  if (eps_dot > 1.0) {
    Term_B = 1.0 + jc->C * log(eps_dot);
  } else {
    Term_B = pow((1.0 + eps_dot), jc->C);
  }
  double Term_C = 1.0 - pow(theta, jc->m);
  double tanh_D = 1.0 - pow((t / jc->Tmelt), jc->tanh_d);
  double tanh_S = pow(t / jc->Tmelt, jc->tanh_b);
  double Term_D = tanh_D + (1.0 - tanh_D) * tanh(1.0 / (pow(eps_pl + tanh_S, jc->tanh_c)));
  return Term_A * Term_B * Term_C * Term_D;
}

/* opt_fun (plasticity.cuh:74-83); m_s_yield (:72) selected by model */
static inline double opt_fun(const orc_joco *jc, int model, double delta_lambda, double norm_Strial,
                             double eps_pl_init, double t, double delta_t, double mu) {
  double eps_pl_equiv = eps_pl_init + sqrt(2.0 / 3.0) * fmax(delta_lambda, 0.);
  double eps_pl_equiv_dot = sqrt(2.0 / 3.0) * fmax(delta_lambda, 0.) / delta_t;
  double sigmaY = model == 1 ? orc_sigma_yield_tanh(jc, eps_pl_equiv, eps_pl_equiv_dot, t)
                             : orc_sigma_yield(jc, eps_pl_equiv, eps_pl_equiv_dot, t);
  return norm_Strial - 2 * mu * delta_lambda - sqrt(2.0 / 3.0) * sigmaY;
}

/* solve_secant (plasticity.cuh:85-119) */
double orc_solve_secant(const orc_joco *jc, int model, double init, double tol, double norm_Strial,
                        double eps_pl_init, double t, double delta_t, double mu, int *iters) {
  double delta_lambda = init;
  double delta_lambda_old = delta_lambda;
  int iter = 0;
  int max_iter = 100;
  for (;;) {
    double g = opt_fun(jc, model, delta_lambda, norm_Strial, eps_pl_init, t, delta_t, mu);
    double delta_lambda_1 = delta_lambda * 1.01;
    double g_1 = opt_fun(jc, model, delta_lambda_1, norm_Strial, eps_pl_init, t, delta_t, mu);
    double slope = (g - g_1) / (delta_lambda - delta_lambda_1);
    delta_lambda_old = delta_lambda;
    delta_lambda = delta_lambda - g / slope;
    if (delta_lambda < 0.) delta_lambda = -0.1 * delta_lambda;
    if (fabs(delta_lambda - delta_lambda_old) < tol) { if (iters) *iters = iter; return delta_lambda; }
    if (iter > max_iter) { if (iters) *iters = -1; return delta_lambda; }
    iter++;
  }
}

/* do_plasticity_johnson_cook (actions_gpu.cu:226-285) */
static void plasticity_johnson_cook(orc_state *s) {
  double dt = s->dt, mu = s->phys.G;
  const orc_joco *jc = &s->joco;
  OMP_FOR_DYN
  for (int i = 0; i < s->N; ++i) {
    if (s->tool_particle[i] != 0.) continue;
    d4 S = s->S[i];
    double Strialxx = S.x, Strialyy = S.z, Strialzz = S.w, Strialxy = S.y;
    double norm_Strial = sqrtf((float)(Strialxx * Strialxx + Strialyy * Strialyy + Strialzz * Strialzz +
                                       Strialxy * Strialxy));
    double p = s->p[i];
    double cxx = Strialxx - p, cyy = Strialyy - p, czz = Strialzz - p, cxy = Strialxy;
    double eps_pl = s->eps_pl[i], eps_pl_dot = s->eps_pl_dot[i], T = s->T[i];
    double svm = sqrtf((float)((cxx * cxx + cyy * cyy + czz * czz) - cxx * cyy - cxx * czz - cyy * czz +
                               3.0 * cxy * cxy));
    const int ref_jc = s->jc_model == 0;  /* the reference's functions cover its default law */
    double sigma_Y = (s->ref_yield && ref_jc) ? s->ref_yield((const double *)jc, eps_pl, eps_pl_dot, T)
                                               : orc_sigma_yield(jc, eps_pl, eps_pl_dot, T);
    if (svm < sigma_Y) {
      s->eps_pl_dot[i] = 0.;
      continue;
    }
    const double init = fmax(eps_pl_dot * dt * sqrt(2. / 3.), 1e-8);
    double delta_lambda =
        (s->ref_secant && ref_jc)
            ? s->ref_secant((const double *)jc, init, 1e-6, norm_Strial, eps_pl, T, dt, s->phys.G)
            : orc_solve_secant(jc, s->jc_model, init, 1e-6, norm_Strial, eps_pl, T, dt, s->phys.G, NULL);
    double eps_pl_new = eps_pl + (double)(sqrtf((float)(2.0 / 3.0)) * fmaxf((float)delta_lambda, 0.f));
    double eps_pl_dot_new = (double)(sqrtf((float)(2.0 / 3.0)) * fmaxf((float)delta_lambda, 0.f)) / dt;
    s->eps_pl[i] = eps_pl_new;
    s->eps_pl_dot[i] = eps_pl_dot_new;
    d4 S_new;
    S_new.x = Strialxx - Strialxx / norm_Strial * delta_lambda * 2. * mu;
    S_new.z = Strialyy - Strialyy / norm_Strial * delta_lambda * 2. * mu;
    S_new.w = Strialzz - Strialzz / norm_Strial * delta_lambda * 2. * mu;
    S_new.y = Strialxy - Strialxy / norm_Strial * delta_lambda * 2. * mu;
    s->S[i] = S_new;
    if (s->trml_wp.tq != 0.) {
      double delta_eps_pl = eps_pl_new - eps_pl;
      double sY = (s->ref_yield && ref_jc) ? s->ref_yield((const double *)jc, eps_pl_new, eps_pl_dot_new, T)
                                           : orc_sigma_yield(jc, eps_pl_new, eps_pl_dot_new, T);
      double rho = s->rho[i];
      s->T[i] += s->trml_wp.tq / (s->trml_wp.cp * rho) * delta_eps_pl * sY;
    }
  }
}

/* do_boundary_conditions_thermal (actions_gpu.cu:287-294) */
static void boundary_conditions_thermal(orc_state *s) {
  OMP_FOR
  for (int i = 0; i < s->N; ++i)
    if (s->fixed[i] == 1.) s->T[i] = s->trml_wp.T_init;
}

/* do_boundary_conditions (actions_gpu.cu:296-311) */
static void boundary_conditions(orc_state *s) {
  OMP_FOR
  for (int i = 0; i < s->N; ++i) {
    if (s->tool_particle[i] != 0.) continue;
    if (s->fixed[i] != 0.) {
      s->vel[i].x = 0.; s->vel[i].y = 0.;
      s->fc[i].x = 0.; s->fc[i].y = 0.;
      s->pos_t[i].x = 0.; s->pos_t[i].y = 0.;
      s->vel_t[i].x = 0.; s->vel_t[i].y = 0.;
    }
  }
}

static inline int isnaninf(double v) { return isnan(v) || isinf(v); }

/* do_invalidate (actions_gpu.cu:317-349); the device printf is not restated */
static void invalidate(orc_state *s) {
  OMP_FOR
  for (int i = 0; i < s->N; ++i) {
    if (s->blanked[i] == 1.) continue;
    int invalid = 0;
    invalid = invalid || isnaninf(s->pos_t[i].x);
    invalid = invalid || isnaninf(s->pos_t[i].y);
    invalid = invalid || isnaninf(s->vel_t[i].x);
    invalid = invalid || isnaninf(s->vel_t[i].y);
    invalid = invalid || isnaninf(s->S_t[i].x);
    invalid = invalid || isnaninf(s->S_t[i].y);
    invalid = invalid || isnaninf(s->S_t[i].z);
    invalid = invalid || isnaninf(s->S_t[i].w);
    invalid = invalid || isnaninf(s->rho_t[i]);
    invalid = invalid || isnaninf(s->T_t[i]);
    if (invalid) s->blanked[i] = 1.;
  }
}

/* ------------------------------------------------------------------------------------- */
/* pair interactions (interactions_gpu.cu) */

/* do_interactions_monaghan, Brookshaw variant (interactions_gpu.cu:147-345). With the PSE
   solver selected the reference is compiled without Thermal_Conduction_Brookshaw: tool
   particles i return early (:160-162) and no temperature terms are computed. */
static void interactions_monaghan(orc_state *s) {
  const int brookshaw = s->thermal_solver == 0;
  const double mass = s->phys.mass, K = s->phys.K;
  const double wdeltap = s->corr.wdeltap, alpha = s->corr.alpha, beta = s->corr.beta, eta = s->corr.eta;
  const double eps = s->corr.xspheps;
  const int nx = s->nx, ny = s->ny;
  const double trml_alpha = s->trml_wp.alpha;
  const double trml_tool_alpha = s->thermal_tool_on ? s->trml_tool.alpha : 0.;
  OMP_FOR_DYN
  for (int pidx = 0; pidx < s->N; ++pidx) {
    if (s->blanked[pidx] == 1.) continue;
    double is_tool_particle_i = s->tool_particle[pidx];
    if (!brookshaw && is_tool_particle_i == 1.) continue;
    double thermal_alpha = 0.;
    if (brookshaw) thermal_alpha = (is_tool_particle_i == 0.) ? trml_alpha : trml_tool_alpha;
    d2 pi = s->pos[pidx], vi = s->vel[pidx];
    d4 Si = s->S[pidx], Ri = s->R[pidx];
    double hi = s->h[pidx], rhoi = s->rho[pidx], prsi = s->p[pidx];
    double Ti = 0.;
    if (brookshaw && thermal_alpha != 0.) Ti = s->T[pidx];
    double rhoi21 = 1. / (rhoi * rhoi);
    int hashi = s->hash[pidx];
    int gi = hashi / ny;
    int gj = hashi - (gi * ny);
    int low_i = gi - 2 < 0 ? 0 : gi - 2;
    int low_j = gj - 2 < 0 ? 0 : gj - 2;
    int high_i = gi + 3 > nx ? nx : gi + 3;
    int high_j = gj + 3 > ny ? ny : gj + 3;
    d4 vi_der = {0., 0., 0., 0.}, Si_der = {0., 0., 0., 0.};
    d2 vi_t = {0., 0.}, xi_t = {0., 0.};
    double T_lapl = 0.;
    for (int ii = low_i; ii < high_i; ii++) {
      for (int jj = low_j; jj < high_j; jj++) {
        int idx = ii * ny + jj;
        int c_start = s->cell_start[idx];
        int c_end = s->cell_end[idx];
        if (c_start == -1) continue;
        for (int iter = c_start; iter < c_end; iter++) {
          if (s->blanked[iter] == 1.) continue;
          d2 pj = s->pos[iter], vj = s->vel[iter];
          d4 Sj = s->S[iter], Rj = s->R[iter];
          double hj = s->h[iter], rhoj = s->rho[iter], prsj = s->p[iter];
          double Tj = 0.;
          if (brookshaw && thermal_alpha != 0.) Tj = s->T[iter];
          double is_tool_particle_j = s->tool_particle[iter];
          double volj = mass / rhoj;
          double rhoj21 = 1. / (rhoj * rhoj);
          d3 ww;
          if (s->ref_kernel) {
            double o3[3];
            s->ref_kernel(pi.x, pi.y, pj.x, pj.y, hi, o3);
            ww.x = o3[0]; ww.y = o3[1]; ww.z = o3[2];
          } else {
            ww = cubic_spline(pi, pj, hi);
          }
          double w = ww.x, w_x = ww.y, w_y = ww.z;
          if (!(is_tool_particle_i == 1.) && !(is_tool_particle_j == 1.)) {
            vi_der.x += (vj.x - vi.x) * w_x * volj;
            vi_der.y += (vj.x - vi.x) * w_y * volj;
            vi_der.z += (vj.y - vi.y) * w_x * volj;
            vi_der.w += (vj.y - vi.y) * w_y * volj;
            double fab = w / wdeltap;
            fab *= fab;
            fab *= fab;
            d3 R;
            R.x = fab * (Ri.x + Rj.x);
            R.y = fab * (Ri.y + Rj.y);
            R.z = fab * (Ri.z + Rj.z);
            Si_der.x += mass * ((Si.x - prsi) * rhoi21 + (Sj.x - prsj) * rhoj21 + R.x) * w_x;
            Si_der.y += mass * (Si.y * rhoi21 + Sj.y * rhoj21 + R.y) * w_y;
            Si_der.z += mass * (Si.y * rhoi21 + Sj.y * rhoj21 + R.y) * w_x;
            Si_der.w += mass * ((Si.z - prsi) * rhoi21 + (Sj.z - prsj) * rhoj21 + R.z) * w_y;
            double xij = pi.x - pj.x;
            double yij = pi.y - pj.y;
            double vijx = vi.x - vj.x;
            double vijy = vi.y - vj.y;
            double vijposij = vijx * xij + vijy * yij;
            double rhoij = 0.5 * (rhoi + rhoj);
            if (vijposij < 0.) {
              double ci = sqrtf((float)(K / rhoi));
              double cj = sqrtf((float)(K / rhoj));
              double cij = 0.5 * (ci + cj);
              double hij = 0.5 * (hi + hj);
              double r2ij = xij * xij + yij * yij;
              double muij = (hij * vijposij) / (r2ij + eta * eta * hij * hij);
              double piij = (-alpha * cij * muij + beta * muij * muij) / rhoij;
              vi_t.x += -mass * piij * w_x;
              vi_t.y += -mass * piij * w_y;
            }
            xi_t.x += -eps * w * mass / rhoij * vijx;
            xi_t.y += -eps * w * mass / rhoij * vijy;
          }
          if (brookshaw && thermal_alpha != 0.) {
            double xij = pi.x - pj.x;
            double yij = pi.y - pj.y;
            double rij = sqrt(xij * xij + yij * yij);
            if (rij > 1e-8) {
              double eijx = xij / rij;
              double eijy = yij / rij;
              double rij1 = 1. / rij;
              T_lapl += 2.0 * (mass / rhoj) * (Ti - Tj) * rij1 * (eijx * w_x + eijy * w_y);
            }
          }
        }
      }
    }
    s->S_der[pidx] = Si_der;
    s->v_der[pidx] = vi_der;
    s->pos_t[pidx] = xi_t;
    s->vel_t[pidx] = vi_t;
    if (brookshaw && thermal_alpha != 0.) s->T_t[pidx] = thermal_alpha * T_lapl;
  }
}

/* do_interactions_heat_pse (interactions_gpu.cu:88-144), launched by interactions_heat_pse
   (:391-421) only if the workpiece diffusivity is non-zero. tool_particle is read through a
   texture bound with sizeof(int)*N bytes of an 8-byte type (:405): indices >= N/2 read 0. */
static void interactions_heat_pse(orc_state *s) {
  if (!s->thermal_wp) return;
  const double mass = s->phys.mass;
  const int nx = s->nx, ny = s->ny, N = s->N;
  const double alpha_wp = s->trml_wp.alpha, alpha_tool = s->trml_tool.alpha;
  const int tex_elems = (int)(((long long)sizeof(int) * N) / 8);
  OMP_FOR_DYN
  for (int pidx = 0; pidx < N; ++pidx) {
    if (s->blanked[pidx] != 0.) continue;
    d2 pi = s->pos[pidx];
    double hi = s->h[pidx], Ti = s->T[pidx];
    int hashi = s->hash[pidx];
    int gi = hashi / ny;
    int gj = hashi - (gi * ny);
    int low_i = gi - 2 < 0 ? 0 : gi - 2;
    int low_j = gj - 2 < 0 ? 0 : gj - 2;
    int high_i = gi + 3 > nx ? nx : gi + 3;
    int high_j = gj + 3 > ny ? ny : gj + 3;
    double T_ti = 0.;
    double is_tool_particle = pidx < tex_elems ? s->tool_particle[pidx] : 0.;
    double alpha = (is_tool_particle == 1.) ? alpha_tool : alpha_wp;
    for (int ii = low_i; ii < high_i; ii++) {
      for (int jj = low_j; jj < high_j; jj++) {
        int idx = ii * ny + jj;
        int c_start = s->cell_start[idx];
        int c_end = s->cell_end[idx];
        if (c_start == -1) continue;
        for (int iter = c_start; iter < c_end; iter++) {
          d2 pj = s->pos[iter];
          double Tj = s->T[iter], rhoj = s->rho[iter];
          double w2_pse = s->ref_pse ? s->ref_pse(pi.x, pi.y, pj.x, pj.y, hi) : lapl_pse(pi, pj, hi);
          T_ti += (Tj - Ti) * w2_pse * mass / rhoj;
        }
      }
    }
    s->T_t[pidx] = alpha * T_ti;
  }
}

/* ------------------------------------------------------------------------------------- */
/* tool (tool.cpp, geometric_primitives.cpp, tool_gpu.cu) */

/* line::line(vec2_t p1, vec2_t p2) (geometric_primitives.cpp:70-85) */
void orc_line_from_points(double x1, double y1, double x2, double y2, double *a, double *b, int *vertical) {
  double Mxx = x1, Mxy = 1.;
  double Myx = x2, Myy = 1.;
  double detM = Mxx * Myy - Mxy * Myx;
  if (fabs(detM) < 1e-12) {
    *vertical = 1;
    *a = DBL_MAX;
    *b = x1;
    return;
  }
  *vertical = 0;
  *a = (y1 * Myy - Mxy * y2) / detM;
  *b = (y2 * Mxx - Myx * y1) / detM;
}

/* tool::update_tool (tool.cpp:211-221) + update_tool_particles (tool_gpu.cu:210-221) */
static void tool_update(orc_state *s) {
  double dt = s->dt;
  orc_tool *t = &s->tool;
  for (int k = 0; k < t->num_seg; ++k) {
    orc_segment *g = &t->seg[k];
    g->left[0] = g->left[0] + dt * t->vel[0];
    g->left[1] = g->left[1] + dt * t->vel[1];
    g->right[0] = g->right[0] + dt * t->vel[0];
    g->right[1] = g->right[1] + dt * t->vel[1];
    orc_line_from_points(g->left[0], g->left[1], g->right[0], g->right[1], &g->a, &g->b, &g->vertical);
  }
  if (t->has_fillet) {
    t->fillet.p[0] = t->fillet.p[0] + dt * t->vel[0];
    t->fillet.p[1] = t->fillet.p[1] + dt * t->vel[1];
  }
  OMP_FOR
  for (int i = 0; i < s->N; ++i) {
    if (s->tool_particle[i] == 0.) continue;
    s->pos[i].x += dt * t->vel[0];
    s->pos[i].y += dt * t->vel[1];
  }
}

static inline double dot2(d2 a, d2 b) { return a.x * b.x + a.y * b.y; }
static inline double len2(d2 a) { return sqrt(dot2(a, a)); }
static inline d2 normalize2(d2 a) {
  double inv = 1. / sqrt(dot2(a, a));
  d2 r = {a.x * inv, a.y * inv};
  return r;
}

/* myatan2 (tool_gpu.cu:29-36) */
static inline double myatan2(double y, double x) {
  double t = atan2(y, x);
  if (t > 0.) return t;
  return t + 2 * M_PI;
}

/* circle_segment_distance (tool_gpu.cu:38-63) */
static inline double circle_segment_distance(const orc_fillet *f, d2 qp) {
  d2 p = {f->p[0], f->p[1]};
  double r = f->r, t1 = f->t1, t2 = f->t2;
  double Ax = p.x, Ay = p.y, Bx = qp.x, By = qp.y;
  double Cx = Ax + r * (Bx - Ax) / sqrt((Bx - Ax) * (Bx - Ax) + (By - Ay) * (By - Ay));
  double Cy = Ay + r * (By - Ay) / sqrt((Bx - Ax) * (Bx - Ax) + (By - Ay) * (By - Ay));
  d2 cp = {Cx, Cy};
  double t = myatan2(p.y - cp.y, p.x - cp.x);
  int valid = t > fmin(t1, t2) && t < fmax(t1, t2);
  if (valid) {
    d2 d = {cp.x - qp.x, cp.y - qp.y};
    return len2(d);
  }
  return FLT_MAX;
}

/* segment_closest_point (tool_gpu.cu:65-81) */
static inline d2 segment_closest_point(const orc_segment *g, d2 xq) {
  if (g->vertical) { d2 r = {g->b, xq.y}; return r; }
  double b = g->b, a = g->a;
  double bb = -1, cc = b, aa = a;
  double px = (bb * (bb * xq.x - aa * xq.y) - aa * cc) / (aa * aa + bb * bb);
  double py = (aa * (-bb * xq.x + aa * xq.y) - bb * cc) / (aa * aa + bb * bb);
  d2 r = {px, py};
  return r;
}

/* establish_contact (tool_gpu.cu:87-139) */
static int establish_contact(const orc_tool *t, d2 qp, d2 *cp, d2 *n) {
  int has_fillet = t->num_seg == TOOL_MAX_SEG;
  int in = 1;
  for (int i = 0; i < t->num_seg; i++) {
    d2 left = {t->seg[i].left[0], t->seg[i].left[1]};
    d2 nn = {t->seg[i].n[0], t->seg[i].n[1]};
    d2 d = {left.x - qp.x, left.y - qp.y};
    in = in && dot2(d, nn) < 0.;
  }
  if (has_fillet) {
    d2 d = {t->fillet.p[0] - qp.x, t->fillet.p[1] - qp.y};
    in = in || len2(d) < t->fillet.r;
  }
  if (!in) return 0;
  double depth = FLT_MAX;
  for (int i = 0; i < t->num_seg; i++) {
    double d;
    if (t->seg[i].vertical) {
      d = fabs(t->seg[i].left[0] - qp.x);
      if (d < depth) {
        depth = d;
        d2 v = {t->seg[i].left[0] - qp.x, 0.};
        *n = normalize2(v);
        cp->x = t->seg[i].left[0];
        cp->y = qp.y;
      }
    } else if (has_fillet && i == 2) {
      d = circle_segment_distance(&t->fillet, qp);
      if (d < depth) {
        depth = d;
        d2 p = {t->fillet.p[0], t->fillet.p[1]};
        d2 v = {qp.x - p.x, qp.y - p.y};
        *n = normalize2(v);
        cp->x = p.x + n->x * t->fillet.r;
        cp->y = p.y + n->y * t->fillet.r;
      }
    } else {
      d2 p = segment_closest_point(&t->seg[i], qp);
      d2 v = {p.x - qp.x, p.y - qp.y};
      d = len2(v);
      if (d < depth) {
        depth = d;
        n->x = -t->seg[i].n[0];
        n->y = -t->seg[i].n[1];
        *cp = p;
      }
    }
  }
  return 1;
}

/* do_compute_contact_forces (tool_gpu.cu:151-207) */
static void compute_contact_forces(orc_state *s) {
  const orc_tool *t = &s->tool;
  double dt = s->dt;
  double slave_mass = t->slave_mass, contact_alpha = t->contact_alpha, friction_mu = t->mu;
  OMP_FOR
  for (int i = 0; i < s->N; ++i) {
    if (s->tool_particle[i] != 0.) continue;
    d2 xs = s->pos[i], vs = s->vel[i];
    d2 xm = {0., 0.}, n = {0., 0.};
    int inside = establish_contact(t, xs, &xm, &n);
    if (!inside) {
      s->fc[i].x = 0.; s->fc[i].y = 0.;
      s->ft[i].x = 0.; s->ft[i].y = 0.;
      s->n[i].x = 0.; s->n[i].y = 0.;
      continue;
    }
    double dt2 = dt * dt;
    d2 dxm = {xs.x - xm.x, xs.y - xm.y};
    double gN = dot2(dxm, n);
    double sc = -slave_mass * gN;
    d2 fN = {sc * n.x, sc * n.y};
    fN.x = fN.x / dt2; fN.y = fN.y / dt2;
    fN.x = fN.x * contact_alpha; fN.y = fN.y * contact_alpha;
    d2 fT = {0., 0.};
    if (friction_mu != 0.) {
      d2 vm = {t->vel[0], t->vel[1]};
      d2 v = {vs.x - vm.x, vs.y - vm.y};
      d2 vr = {v.x - v.x * n.x, v.y - v.y * n.y};
      d2 fricold = s->ft[i];
      double ks = contact_alpha * slave_mass;
      d2 kdeltae = {ks * vr.x, ks * vr.y};
      kdeltae.x = kdeltae.x / dt; kdeltae.y = kdeltae.y / dt;
      double fy = friction_mu * len2(fN);
      d2 fstar = {fricold.x - kdeltae.x, fricold.y - kdeltae.y};
      if (len2(fstar) > fy) {
        double l = len2(fstar);
        fT.x = fy * fstar.x / l;
        fT.y = fy * fstar.y / l;
      } else {
        fT = fstar;
      }
    }
    s->fc[i] = fN;
    s->ft[i] = fT;
    s->n[i] = n;
  }
}

/* report_force (output.cu:31-39): sum of fc then ft over all particles (sequential order) */
void orc_report_force(orc_state *s, double out2[2]) {
  double x = 0., y = 0.;
  for (int i = 0; i < s->N; ++i) { x = x + s->fc[i].x; y = y + s->fc[i].y; }
  for (int i = 0; i < s->N; ++i) { x = x + s->ft[i].x; y = y + s->ft[i].y; }
  out2[0] = x;
  out2[1] = y;
}

/* ------------------------------------------------------------------------------------- */
/* leap_frog::step stages (leap_frog.cu:94-155) */

void orc_stage_predict(orc_state *s) {
  lf_init(s);
  lf_predict(s);
  material_eos(s);
  corrector_artificial_stress(s);
}

void orc_stage_interact(orc_state *s) {
  interactions_monaghan(s);
  if (s->thermal_solver == 1) interactions_heat_pse(s);
}

void orc_stage_rates(orc_state *s) {
  stress_rate_jaumann(s);
  contmech(s);
}

void orc_stage_finish(orc_state *s) {
  lf_correct(s);
  if (s->has_tool && s->fric_heat) fric_heat_gen(s);
  if (s->plastic) plasticity_johnson_cook(s);
  if (s->has_tool) {
    tool_update(s);
    compute_contact_forces(s);
  }
  boundary_conditions(s);
  if (s->thermal_bc) boundary_conditions_thermal(s);
  invalidate(s);
}

int orc_step(orc_state *s) {
  if (orc_grid_update(s) != 0) return -1;
  orc_stage_predict(s);
  orc_stage_interact(s);
  orc_stage_rates(s);
  orc_stage_finish(s);
  return 0;
}

int orc_steps(orc_state *s, int n) {
  for (int k = 0; k < n; ++k)
    if (orc_step(s) != 0) return -1;
  return 0;
}

/* Usui tool wear rate (tool_wear.cu:20-64) over the particles in contact: out = min, max,
   average of K exp(alpha/T) p |v_r|, p = |fc| / (2 pi h), v_r = v - v*n component-wise with
   v = vel - tool velocity. "In contact" tests fc.x, fc.y, ft.x and fc.y again (ft.y is never
   tested), as the reference does. */
void orc_usui(orc_state *s, double K, double alpha, double tool_vx, double tool_vy, double out3[3]) {
  double mn = 3.402823466e+38, mx = 0., total = 0.;
  long long count = 0;
  for (int i = 0; i < s->N; ++i) {
    const double fcx = s->fc[i].x, fcy = s->fc[i].y, ftx = s->ft[i].x;
    const int in_contact = fabs(fcx) > 0. || fabs(fcy) > 0. || fabs(ftx) > 0. || fabs(fcy) > 0.;
    if (!in_contact) continue;
    count++;
    const double vx = s->vel[i].x - tool_vx, vy = s->vel[i].y - tool_vy;
    const double nx = s->n[i].x, ny = s->n[i].y;
    const double vrx = vx - vx * nx, vry = vy - vy * ny;
    const double vmag = sqrt(vrx * vrx + vry * vry);
    const double fmag = sqrt(fcx * fcx + fcy * fcy);
    const double A = 2 * s->h[i] * M_PI;
    const double p = fmag / A;
    const double w = K * exp(alpha / s->T[i]) * p * vmag;
    total += w;
    mn = fmin(mn, w);
    mx = fmax(mx, w);
  }
  out3[0] = count == 0 ? 0. : mn;
  out3[1] = mx;
  out3[2] = count == 0 ? 0. : total / count;
}

/* n steps, with report_force (output.cu:31-39) after each one into out[2k], out[2k+1] */
int orc_steps_force_log(orc_state *s, int n, double *out) {
  for (int k = 0; k < n; ++k) {
    if (orc_step(s) != 0) return -1;
    orc_report_force(s, out + 2 * k);
  }
  return 0;
}
