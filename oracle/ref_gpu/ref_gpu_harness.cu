// ORACLE recipe - test infrastructure only, never part of the product.
//
// The reference's own FP64 CUDA step on the GPU: a C entry-point harness around its sources,
// compiled unchanged where they lie (actions_gpu.cu, interactions_gpu.cu, leap_frog.cu,
// tool_gpu.cu, grid*.cu, particle_gpu.cu, output.cu, and the host files they need) with the
// texture shim (ref_texture_shim.h, force-included) and the project's GLM subset, into
// oracle/_ref/libref_gpu.so by oracle/build_oracle.py (build_ref_gpu). That is the
// reference's default build: USE_DOUBLE and the Brookshaw heat solver are #defined in its
// types.h. oracle/_ref/libref_gpu_pse.so is the same sources and harness with its PSE heat
// solver: a copy of types.h with the solver switch turned, generated into oracle/_ref at build
// time, is force-included so that its guard makes the sources' own types.h a no-op.
//
// The harness does what the reference's main() (mfree_gpu.cpp:206-308) and setup_ref_cut
// (benchmarks.cpp:255-537) do, from caller-given arrays instead of a built-in scene: a
// particle_gpu from the upload constructor (particle_gpu.cu), the remaining fields written
// into its public device arrays, the constants through actions_setup_* / interactions_setup_*
// in setup_ref_cut's order, a locked grid_gpu_green, the rigid tool (its segments, fillet and
// velocity set from the caller's tool state) through tool_gpu_set_up_tool, a leap_frog, and
// then leap_frog::step as main() calls it.
//
// Safety: the reference writes out of bounds when a particle's cell hash leaves the grid
// (grid_gpu_green.cu:22-116). refg_step copies the positions back before every step and
// refuses to step (returns -3) if an unblanked particle lies outside the locked grid.
//
// The reference keeps process-wide state: __constant__ memory per translation unit, the
// option flags of actions_gpu.cu (set, never cleared) and global_tool / global_dt. So one
// process holds one reference system at a time (refg_create frees the previous one's
// stepper and grid; particle_gpu has no destructor, so its arrays stay allocated until
// exit), and one process should use one set of options (heat, plasticity, tool).
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "types.h"
#include "geometric_primitives.h"
#include "particle_gpu.h"
#include "constants_structs.h"
// the tool's geometry is private to class tool: the harness sets it from the caller's tool
// state (bit for bit the state the product and the oracle hold), which no public member allows
#define private public
#include "tool.h"
#undef private
#include "actions_gpu.h"
#include "grid_gpu_green.h"
#include "interactions_gpu.h"
#include "leap_frog.h"
#include "output.h"
#include "tool_gpu.h"

#include "sph_oracle.h"  // orc_tool layout and the field numbering (ORC_*)

// globals the reference defines in mfree_gpu.cpp (its NVML/getopt driver) and in
// benchmarks.cpp (its built-in scenes), neither of which this build compiles
int global_step = 0;
tool *global_tool = 0;
float_t global_dt = 0.;
float_t global_t_final = 0.;

namespace {

struct ref_system {
  particle_gpu *p = nullptr;
  grid_gpu_green *grid = nullptr;
  leap_frog *stepper = nullptr;
  tool *tl = nullptr;
  int N = 0;
  double bbmin_x = 0., bbmin_y = 0., dx = 0.;
  int nx = 0, ny = 0;
};
ref_system g;

int ck(cudaError_t e) { return e == cudaSuccess ? 0 : -2; }

// the device array of a field and its width in doubles (ints for idx/hash)
void *field_ptr(int field, int *width) {
  particle_gpu *p = g.p;
  *width = 1;
  switch (field) {
    case ORC_POS: *width = 2; return p->pos;
    case ORC_VEL: *width = 2; return p->vel;
    case ORC_H: return p->h;
    case ORC_RHO: return p->rho;
    case ORC_P: return p->p;
    case ORC_S: *width = 4; return p->S;
    case ORC_R: *width = 4; return p->R;
    case ORC_FC: *width = 2; return p->fc;
    case ORC_FT: *width = 2; return p->ft;
    case ORC_N: *width = 2; return p->n;
    case ORC_FIXED: return p->fixed;
    case ORC_BLANKED: return p->blanked;
    case ORC_TOOL: return p->tool_particle;
    case ORC_EPS_PL: return p->eps_pl;
    case ORC_EPS_PL_DOT: return p->eps_pl_dot;
    case ORC_T: return p->T;
    case ORC_POS_T: *width = 2; return p->pos_t;
    case ORC_VEL_T: *width = 2; return p->vel_t;
    case ORC_RHO_T: return p->rho_t;
    case ORC_S_T: *width = 4; return p->S_t;
    case ORC_T_T: return p->T_t;
    case ORC_S_DER: *width = 4; return p->S_der;
    case ORC_V_DER: *width = 4; return p->v_der;
    case ORC_IDX: return p->idx;
    case ORC_HASH: return p->hash;
    default: return nullptr;
  }
}

}  // namespace

extern "C" {

// A reference system of N particles from host arrays (pos, vel: 2N; the rest N; T, fixed,
// tool_p may be NULL: 0) on a locked grid_gpu_green (grid_gpu_green.h:90). 0 on success.
int refg_create(int N, const double *pos, const double *vel, const double *rho, const double *T, const double *h,
                const double *fixed, const double *tool_p, double bbmin_x, double bbmin_y, double bbmax_x,
                double bbmax_y, double grid_h) {
  if (N <= 0 || !pos || !vel || !rho || !h) return -1;
  delete g.stepper;
  delete g.grid;
  g = ref_system{};
  std::vector<float2_t> p2((size_t)N), v2((size_t)N);
  std::vector<float_t> r((size_t)N), t((size_t)N, 0.), hh((size_t)N), f((size_t)N, 0.), tp((size_t)N, 0.);
  for (int i = 0; i < N; ++i) {
    p2[i] = make_float2_t(pos[2 * i], pos[2 * i + 1]);
    v2[i] = make_float2_t(vel[2 * i], vel[2 * i + 1]);
    r[i] = rho[i];
    hh[i] = h[i];
    if (T) t[i] = T[i];
    if (fixed) f[i] = fixed[i];
    if (tool_p) tp[i] = tool_p[i];
  }
  // particle_gpu.cu: the upload constructor with temperature, fixed and tool flags
  g.p = new particle_gpu(p2.data(), v2.data(), r.data(), t.data(), hh.data(), f.data(), tp.data(), (unsigned)N);
  g.grid = new grid_gpu_green(N, make_float2_t(bbmin_x, bbmin_y), make_float2_t(bbmax_x, bbmax_y), grid_h);
  g.N = N;
  g.bbmin_x = g.grid->bbmin_x();
  g.bbmin_y = g.grid->bbmin_y();
  g.dx = g.grid->dx();
  g.nx = g.grid->nx();
  g.ny = g.grid->ny();
  g.stepper = new leap_frog((unsigned)N, (unsigned)g.grid->num_cell());
  return ck(cudaDeviceSynchronize());
}

// grid geometry: nx, ny, num_cell; bbmin_x, bbmin_y, dx
void refg_geometry(int *i3, double *d3) {
  i3[0] = g.nx; i3[1] = g.ny; i3[2] = g.grid ? g.grid->num_cell() : 0;
  d3[0] = g.bbmin_x; d3[1] = g.bbmin_y; d3[2] = g.dx;
}

// Constants in the struct layouts of constants_structs.h (7, 6, 6, 12 doubles); joco NULL:
// no plasticity. The order of setup_ref_cut (benchmarks.cpp:510-521).
int refg_set_constants(const double *phys7, const double *corr6, const double *joco12, const double *trml_wp6,
                       const double *trml_tool6, double dt) {
  if (!g.p || !phys7 || !corr6 || !trml_wp6 || !trml_tool6) return -1;
  phys_constants phys;
  corr_constants corr;
  joco_constants joco;
  trml_constants tw, tt;
  static_assert(sizeof(phys_constants) == 7 * sizeof(double), "phys_constants layout");
  static_assert(sizeof(corr_constants) == 6 * sizeof(double), "corr_constants layout");
  static_assert(sizeof(joco_constants) == 12 * sizeof(double), "joco_constants layout");
  static_assert(sizeof(trml_constants) == 6 * sizeof(double), "trml_constants layout");
  std::memcpy(&phys, phys7, sizeof(phys));
  std::memcpy(&corr, corr6, sizeof(corr));
  std::memcpy(&tw, trml_wp6, sizeof(tw));
  std::memcpy(&tt, trml_tool6, sizeof(tt));
  actions_setup_corrector_constants(corr);
  actions_setup_physical_constants(phys);
  if (joco12) {
    std::memcpy(&joco, joco12, sizeof(joco));
    actions_setup_johnson_cook_constants(joco);
  }
  actions_setup_thermal_constants_wp(tw);
  actions_setup_thermal_constants_tool(tt);
  interactions_setup_geometry_constants(g.grid);
  interactions_setup_corrector_constants(corr);
  interactions_setup_physical_constants(phys);
  if (g.tl) interactions_setup_thermal_constants_tool(tt, g.tl);
  interactions_setup_thermal_constants_workpiece(tw);
  global_dt = dt;
  return ck(cudaDeviceSynchronize());
}

// The rigid tool from a tool state (orc_tool, the layout of the product's mf_tool_state):
// segments, fillet, velocity and friction coefficient set on a reference tool object, then
// tool_gpu_set_up_tool(tool, contact_alpha, phys with mass = slave_mass) (tool_gpu.cu:224-271).
// Call before refg_set_constants (interactions_setup_thermal_constants_tool marks the tool).
int refg_set_tool(const orc_tool *ts, const double *phys7) {
  if (!g.p || !ts || !phys7) return -1;
  if (ts->num_seg < 0 || ts->num_seg > 5) return -1;
  tool *t = new tool();
  t->m_segments.clear();
  for (int i = 0; i < ts->num_seg; ++i) {
    segment s;
    s.left = vec2_t(ts->seg[i].left[0], ts->seg[i].left[1]);
    s.right = vec2_t(ts->seg[i].right[0], ts->seg[i].right[1]);
    s.l.a = ts->seg[i].a;
    s.l.b = ts->seg[i].b;
    s.l.vertical = ts->seg[i].vertical != 0;
    s.n = vec2_t(ts->seg[i].n[0], ts->seg[i].n[1]);
    t->m_segments.push_back(s);
  }
  t->m_fillet = 0;
  if (ts->has_fillet)
    t->m_fillet = new circle_segment(ts->fillet.r, ts->fillet.t1, ts->fillet.t2,
                                     vec2_t(ts->fillet.p[0], ts->fillet.p[1]));
  t->m_velocity = vec2_t(ts->vel[0], ts->vel[1]);
  t->m_mu = ts->mu;
  phys_constants phys;
  std::memcpy(&phys, phys7, sizeof(phys));
  phys.mass = ts->slave_mass;
  tool_gpu_set_up_tool(t, ts->contact_alpha, phys);
  g.tl = t;
  global_tool = t;
  return ck(cudaDeviceSynchronize());
}

// the tool's current segments and fillet (advanced on the host by tool::update_tool)
int refg_get_tool(orc_tool *out) {
  if (!g.tl || !out) return -1;
  std::vector<segment> s = g.tl->get_segments();
  out->num_seg = (int)s.size();
  for (size_t i = 0; i < s.size() && i < 5; ++i) {
    out->seg[i].left[0] = s[i].left.x; out->seg[i].left[1] = s[i].left.y;
    out->seg[i].right[0] = s[i].right.x; out->seg[i].right[1] = s[i].right.y;
    out->seg[i].a = s[i].l.a; out->seg[i].b = s[i].l.b; out->seg[i].vertical = s[i].l.vertical ? 1 : 0;
    out->seg[i].n[0] = s[i].n.x; out->seg[i].n[1] = s[i].n.y;
  }
  circle_segment *f = g.tl->get_fillet();
  out->has_fillet = f ? 1 : 0;
  if (f) {
    out->fillet.r = f->r; out->fillet.t1 = f->t1; out->fillet.t2 = f->t2;
    out->fillet.p[0] = f->p.x; out->fillet.p[1] = f->p.y;
  }
  return 0;
}

// host <-> device copies of one field (the current arrays: the Green grid swaps them)
int refg_set_field(int field, const void *host) {
  if (!g.p || !host) return -1;
  int w = 1;
  void *d = field_ptr(field, &w);
  if (!d) return -1;
  const size_t el = (field == ORC_IDX || field == ORC_HASH) ? sizeof(int) : sizeof(double);
  return ck(cudaMemcpy(d, host, el * (size_t)w * (size_t)g.N, cudaMemcpyHostToDevice));
}

int refg_get_field(int field, void *host) {
  if (!g.p || !host) return -1;
  int w = 1;
  void *d = field_ptr(field, &w);
  if (!d) return -1;
  const size_t el = (field == ORC_IDX || field == ORC_HASH) ? sizeof(int) : sizeof(double);
  return ck(cudaMemcpy(host, d, el * (size_t)w * (size_t)g.N, cudaMemcpyDeviceToHost));
}

// n steps of leap_frog::step (leap_frog.cu:94-155) as main() runs them (mfree_gpu.cpp:306-307),
// each after the in-grid check. Returns 0, -2 on a CUDA error, -3 if a particle left the grid.
int refg_step(int n) {
  if (!g.p || !g.stepper || n < 0) return -1;
  std::vector<double> pos(2 * (size_t)g.N), bl((size_t)g.N);
  const long long num_cell = (long long)g.nx * g.ny;
  for (int k = 0; k < n; ++k) {
    if (cudaMemcpy(pos.data(), g.p->pos, sizeof(double) * pos.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
      return -2;
    if (cudaMemcpy(bl.data(), g.p->blanked, sizeof(double) * bl.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
      return -2;
    for (int i = 0; i < g.N; ++i) {
      if (bl[i] == 1.) continue;  // blanked particles keep their previous, valid hash
      // the reference's cell index truncates toward zero (grid.cu:34-51): a particle up to one
      // cell below or left of the box still lands in the first row or column
      const double fx = (pos[2 * i] - g.bbmin_x) / g.dx, fy = (pos[2 * i + 1] - g.bbmin_y) / g.dx;
      if (!(fx > -1. && fy > -1. && fx < (double)g.nx && fy < (double)g.ny)) return -3;
      const long long hsh = (long long)(int)fx * g.ny + (long long)(int)fy;
      if (hsh < 0 || hsh >= num_cell) return -3;
    }
    g.stepper->step(g.p, g.grid);
    global_step++;
  }
  return ck(cudaDeviceSynchronize());
}

// Timing: n steps of leap_frog::step between two CUDA events on the legacy default stream
// (the reference's stream), the in-grid check made once before them; *ms = elapsed time.
// n is limited to 4096: at the cut's speeds (~1e-4 cm/us, dt ~ 2e-4 us) no particle moves
// more than ~1e-4 cm in that many steps, far inside the locked grid's margins.
int refg_run_timed(int n, float *ms) {
  if (!g.p || !g.stepper || n < 1 || n > 4096 || !ms) return -1;
  int rc = refg_step(0);
  if (rc != 0) return rc;
  std::vector<double> pos(2 * (size_t)g.N), bl((size_t)g.N);
  if (cudaMemcpy(pos.data(), g.p->pos, sizeof(double) * pos.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
    return -2;
  if (cudaMemcpy(bl.data(), g.p->blanked, sizeof(double) * bl.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
    return -2;
  const double margin = 2e-4;  // cm, against at most ~1e-4 cm of travel
  for (int i = 0; i < g.N; ++i) {
    if (bl[i] == 1.) continue;
    const double x = pos[2 * i], y = pos[2 * i + 1];
    if (!(x - margin > g.bbmin_x - g.dx && y - margin > g.bbmin_y - g.dx && x + margin < g.bbmin_x + g.nx * g.dx &&
          y + margin < g.bbmin_y + g.ny * g.dx))
      return -3;
  }
  cudaEvent_t a, b;
  if (cudaEventCreate(&a) != cudaSuccess) return -2;
  if (cudaEventCreate(&b) != cudaSuccess) { cudaEventDestroy(a); return -2; }
  cudaEventRecord(a, 0);
  for (int k = 0; k < n; ++k) {
    g.stepper->step(g.p, g.grid);
    global_step++;
  }
  cudaEventRecord(b, 0);
  rc = ck(cudaEventSynchronize(b));
  if (rc == 0) rc = ck(cudaEventElapsedTime(ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (rc == 0) rc = ck(cudaDeviceSynchronize());
  return rc;
}

// cell_start / cell_end of the last sort (grid_gpu_green::get_cells, grid_gpu_green.cu:207-210)
int refg_get_cells(int *start, int *end) {
  if (!g.grid || !start || !end) return -1;
  const int nc = g.grid->num_cell();
  int *ds = nullptr, *de = nullptr;
  if (cudaMalloc(&ds, sizeof(int) * (size_t)nc) != cudaSuccess) return -2;
  if (cudaMalloc(&de, sizeof(int) * (size_t)nc) != cudaSuccess) { cudaFree(ds); return -2; }
  g.grid->get_cells(g.p, ds, de);
  int rc = ck(cudaMemcpy(start, ds, sizeof(int) * (size_t)nc, cudaMemcpyDeviceToHost));
  if (rc == 0) rc = ck(cudaMemcpy(end, de, sizeof(int) * (size_t)nc, cudaMemcpyDeviceToHost));
  cudaFree(ds);
  cudaFree(de);
  return rc;
}

// report_force (output.cu:31-39): sum of fc + ft over all particles
int refg_report_force(double *out2) {
  if (!g.p || !out2) return -1;
  float2_t f = report_force(g.p);
  out2[0] = f.x;
  out2[1] = f.y;
  return ck(cudaDeviceSynchronize());
}

}  // extern "C"
