// Oracle recipe: host harness around the reference's own sources (test infrastructure only).
//
// Built by oracle/build_oracle.py into oracle/_ref/libref_host.so, together with these
// reference files compiled where they lie (src/ of the reference):
//   benchmarks.cpp, tool.cpp, geometric_primitives.cpp, constants_structs.cpp,
//   grid.cu (grid_base geometry), tool_wear.cu (Usui wear, host side).
// The reference's GPU entry points that setup_ref_cut() calls are replaced by the
// recording stubs below, so that setup_ref_cut() runs on a machine without a GPU and its
// complete output (particle arrays, constants, tool, grid geometry, dt) can be read back.
// kernels.cuh is included directly (its functions are __host__ __device__).
// plasticity.cuh is compiled separately for the host (ref_host_plasticity.cpp).
//
// Nothing in the product links this file. Only tests/ and the golden-fixture script use it.
#include <cmath>
#include <cfloat>
#include <cstdio>
#include <cstring>
#include <vector>

#include "benchmarks.h"
#include "vtk_writer.h"
#include "kernels.cuh"

// ---------------------------------------------------------------------------------------
// globals the reference defines in mfree_gpu.cpp (not compiled: it is the NVML/getopt driver)
int global_step = 0;
extern float_t global_t_final;  // defined in benchmarks.cpp
tool *global_tool = 0;
tool_wear *global_wear = 0;

// ---------------------------------------------------------------------------------------
// recorded outputs of the last setup_* call
namespace {
struct recorded {
  std::vector<double> pos, vel, rho, T, h, fixed, tool_p;
  unsigned int N = 0;
  phys_constants phys_a, phys_i;
  corr_constants corr_a, corr_i;
  joco_constants joco;
  trml_constants trml_wp_a, trml_tool_a, trml_wp_i, trml_tool_i;
  bool has_joco = false;
  geom_constants geom;
  double contact_alpha = 0.;
  phys_constants contact_phys;
  tool *contact_tool = 0;
  grid_base *grid = 0;
  unsigned int grid_max_cell = 0;  // max_cell of an adaptive grid_gpu_green, 0 for a locked one
};
recorded g_rec;

void record_particles(float2_t *pos, float2_t *vel, float_t *rho, float_t *T, float_t *h,
                      float_t *fixed, float_t *tool_p, unsigned int N) {
  g_rec.N = N;
  g_rec.pos.assign(2 * (size_t)N, 0.);
  g_rec.vel.assign(2 * (size_t)N, 0.);
  g_rec.rho.assign(N, 0.);
  g_rec.T.assign(N, 0.);
  g_rec.h.assign(N, 0.);
  g_rec.fixed.assign(N, 0.);
  g_rec.tool_p.assign(N, 0.);
  for (unsigned int i = 0; i < N; ++i) {
    g_rec.pos[2 * i] = pos[i].x;
    g_rec.pos[2 * i + 1] = pos[i].y;
    g_rec.vel[2 * i] = vel[i].x;
    g_rec.vel[2 * i + 1] = vel[i].y;
    g_rec.rho[i] = rho[i];
    g_rec.h[i] = h[i];
    if (T) g_rec.T[i] = T[i];
    if (fixed) g_rec.fixed[i] = fixed[i];
    if (tool_p) g_rec.tool_p[i] = tool_p[i];
  }
}
}  // namespace

// ---------------------------------------------------------------------------------------
// stubs for the reference's device-side setup calls (record instead of cudaMemcpyToSymbol)
bool check_cuda_error() { return true; }
bool check_cuda_error(const char *) { return true; }

void actions_setup_corrector_constants(corr_constants c) { g_rec.corr_a = c; }
void actions_setup_physical_constants(phys_constants p) { g_rec.phys_a = p; }
void actions_setup_johnson_cook_constants(joco_constants j) { g_rec.joco = j; g_rec.has_joco = true; }
void actions_setup_thermal_constants_wp(trml_constants t) { g_rec.trml_wp_a = t; }
void actions_setup_thermal_constants_tool(trml_constants t) { g_rec.trml_tool_a = t; }

void interactions_setup_geometry_constants(grid_base *g) {
  g_rec.grid = g;
  g_rec.geom.nx = g->nx();
  g_rec.geom.ny = g->ny();
  g_rec.geom.bbmin_x = g->bbmin_x();
  g_rec.geom.bbmin_y = g->bbmin_y();
  g_rec.geom.dx = g->dx();
}
void interactions_setup_physical_constants(phys_constants p) { g_rec.phys_i = p; }
void interactions_setup_corrector_constants(corr_constants c) { g_rec.corr_i = c; }
void interactions_setup_thermal_constants_workpiece(trml_constants t) { g_rec.trml_wp_i = t; }
void interactions_setup_thermal_constants_tool(trml_constants t, tool *tl) {
  g_rec.trml_tool_i = t;
  if (t.alpha != 0.) tl->set_thermal(true);
}

void tool_gpu_set_up_tool(tool *t, float_t alpha, phys_constants phys) {
  g_rec.contact_tool = t;
  g_rec.contact_alpha = alpha;
  g_rec.contact_phys = phys;
}

// particle_gpu upload constructors: record the host arrays
particle_gpu::particle_gpu(float2_t *pos, float2_t *vel_init, float_t *rho, float_t *h, unsigned int N) {
  record_particles(pos, vel_init, rho, 0, h, 0, 0, N);
  this->N = N;
}
particle_gpu::particle_gpu(float2_t *pos, float2_t *vel_init, float_t *rho, float_t *T_init, float_t *h,
                           float_t *fixed, unsigned int N) {
  record_particles(pos, vel_init, rho, T_init, h, fixed, 0, N);
  this->N = N;
}
particle_gpu::particle_gpu(float2_t *pos, float2_t *vel_init, float_t *rho, float_t *T_init, float_t *h,
                           float_t *fixed, float_t *tool_p, unsigned int N) {
  record_particles(pos, vel_init, rho, T_init, h, fixed, tool_p, N);
  this->N = N;
}

// grid_gpu_green: geometry only (the buffers are device memory; not needed here)
grid_gpu_green::grid_gpu_green(unsigned int max_cell, unsigned int N) : grid_base(max_cell, N) {
  g_rec.grid_max_cell = max_cell;
}
grid_gpu_green::grid_gpu_green(int num_part, float2_t bbmin, float2_t bbmax, float_t h)
    : grid_base(num_part, bbmin, bbmax, h) {
  g_rec.grid_max_cell = 0;
}
void grid_gpu_green::sort(particle_gpu *, tool *) const {}
void grid_gpu_green::get_cells(particle_gpu *, int *, int *) {}

// ---------------------------------------------------------------------------------------
// C entry points used by the tests (ctypes)
extern "C" {

// kernels.cuh
void refh_cubic_spline(double xi, double yi, double xj, double yj, double hi, double *out3) {
  float2_t pi = make_double2(xi, yi), pj = make_double2(xj, yj);
  float3_t w = cubic_spline(pi, pj, hi);
  out3[0] = w.x; out3[1] = w.y; out3[2] = w.z;
}
double refh_lapl_pse(double xi, double yi, double xj, double yj, double hi) {
  return lapl_pse(make_double2(xi, yi), make_double2(xj, yj), hi);
}

// tool geometry: the (tl, length, height, rake, clearance, r, mu) constructor
// out layout per segment (11 doubles): left.x left.y right.x right.y a b vertical n.x n.y 0 0
// fillet (5 doubles): r t1 t2 p.x p.y ; misc (3 doubles): front low mu
static tool *g_tool = 0;
int refh_tool_create(double tl_x, double tl_y, double length, double height, double rake,
                     double clear, double r, double mu) {
  delete g_tool;
  g_tool = new tool(glm::dvec2(tl_x, tl_y), length, height, rake, clear, r, mu);
  return (int)g_tool->get_segments().size();
}
int refh_tool_create_points(const double *pts8, double r, double mu) {
  delete g_tool;
  glm::dvec2 tl(pts8[0], pts8[1]), tr(pts8[2], pts8[3]), br(pts8[4], pts8[5]), bl(pts8[6], pts8[7]);
  g_tool = new tool(tl, tr, br, bl, r, mu);
  return (int)g_tool->get_segments().size();
}
static int dump_tool(tool *t, double *seg_out, double *fillet_out, double *misc_out) {
  if (!t) return -1;
  std::vector<segment> s = t->get_segments();
  for (size_t i = 0; i < s.size(); ++i) {
    double *o = seg_out + 11 * i;
    o[0] = s[i].left.x; o[1] = s[i].left.y; o[2] = s[i].right.x; o[3] = s[i].right.y;
    o[4] = s[i].l.a; o[5] = s[i].l.b; o[6] = s[i].l.vertical ? 1. : 0.;
    o[7] = s[i].n.x; o[8] = s[i].n.y; o[9] = 0.; o[10] = 0.;
  }
  circle_segment *f = t->get_fillet();
  if (f) {
    fillet_out[0] = f->r; fillet_out[1] = f->t1; fillet_out[2] = f->t2;
    fillet_out[3] = f->p.x; fillet_out[4] = f->p.y;
  } else {
    for (int k = 0; k < 5; ++k) fillet_out[k] = 0.;
  }
  misc_out[0] = t->front();
  misc_out[1] = t->low();
  misc_out[2] = t->mu();
  return (int)s.size();
}
int refh_tool_dump(double *seg_out, double *fillet_out, double *misc_out) {
  return dump_tool(g_tool, seg_out, fillet_out, misc_out);
}
// vtk_writer_write(const tool*, int) (vtk_writer.cpp:185-264) on the current tool: writes
// results/vtk_tool_<step>.vtk under the working directory
int refh_vtk_tool(int step) {
  if (!g_tool) return -1;
  vtk_writer_write(g_tool, step);
  return 0;
}
// vtk_writer_write(const particle_gpu*, int) (vtk_writer.cpp:20-178) on host arrays: writes
// results/vtk_out_<step>.vtk under the working directory. The reference never fills its
// blanked array (Q12), so which particles it skips depends on uninitialised memory; callers
// check the POINTS count.
int refh_vtk_particles(int step, int N, const double *pos, const double *vel, const double *rho, const double *h,
                       const double *p, const double *T, const double *eps, const double *S, const double *fixed,
                       const double *tool_p) {
  std::vector<int> idx((size_t)N);
  for (int i = 0; i < N; ++i) idx[i] = i;
  particle_gpu pg((float2_t *)pos, (float2_t *)vel, (float_t *)rho, (float_t *)h, (unsigned)N);
  pg.idx = idx.data();
  pg.pos = (float2_t *)pos;
  pg.vel = (float2_t *)vel;
  pg.rho = (float_t *)rho;
  pg.h = (float_t *)h;
  pg.p = (float_t *)p;
  pg.T = (float_t *)T;
  pg.eps_pl = (float_t *)eps;
  pg.S = (float4_t *)S;
  pg.fixed = (float_t *)fixed;
  pg.tool_particle = (float_t *)tool_p;
  vtk_writer_write(&pg, step);
  return 0;
}
void refh_tool_set_vel(double vx, double vy) { if (g_tool) g_tool->set_vel(glm::dvec2(vx, vy)); }
void refh_tool_update(double dt) { if (g_tool) g_tool->update_tool(dt); }
int refh_tool_sample(double dx, double *out_xy, int cap) {
  if (!g_tool) return -1;
  std::vector<float2_t> s = g_tool->sample_tool(dx, 300., 1., 1.5);
  int n = (int)s.size();
  for (int i = 0; i < n && i < cap; ++i) { out_xy[2 * i] = s[i].x; out_xy[2 * i + 1] = s[i].y; }
  return n;
}
void refh_tool_safe_bb(double safety, double *out4) {
  bbox b = g_tool->safe_bb(safety);
  out4[0] = b.bbmin_x; out4[1] = b.bbmax_x; out4[2] = b.bbmin_y; out4[3] = b.bbmax_y;
}

// geometric primitives
void refh_line_from_points(double x1, double y1, double x2, double y2, double *out3) {
  line l(glm::dvec2(x1, y1), glm::dvec2(x2, y2));
  out3[0] = l.a; out3[1] = l.b; out3[2] = l.vertical ? 1. : 0.;
}

// setup_ref_cut: run the reference scene setup and keep its outputs for the getters below
int refh_setup_ref_cut(int ny, double rake, double clear, double chamfer, double speed, double feed) {
  grid_base *grid = 0;
  global_tool = 0;
  particle_gpu *p = setup_ref_cut(ny, &grid, rake, clear, chamfer, speed, feed);
  (void)p;
  return (int)g_rec.N;
}
// (each setup starts from an empty record and no tool: the rings and impact scenes set
// neither Johnson-Cook nor thermal constants nor a tool)
int refh_setup_rings(int nbox) {
  grid_base *grid = 0;
  g_rec = recorded();
  global_tool = 0;
  setup_rings(nbox, &grid);
  g_rec.grid = grid;
  return (int)g_rec.N;
}
int refh_setup_impact(int nbox) {
  grid_base *grid = 0;
  g_rec = recorded();
  global_tool = 0;
  setup_impact(nbox, &grid);
  g_rec.grid = grid;
  return (int)g_rec.N;
}
// particle arrays: field 0 pos(2N) 1 vel(2N) 2 rho 3 T 4 h 5 fixed 6 tool_p
int refh_get_array(int field, double *out) {
  const std::vector<double> *v = 0;
  switch (field) {
    case 0: v = &g_rec.pos; break;
    case 1: v = &g_rec.vel; break;
    case 2: v = &g_rec.rho; break;
    case 3: v = &g_rec.T; break;
    case 4: v = &g_rec.h; break;
    case 5: v = &g_rec.fixed; break;
    case 6: v = &g_rec.tool_p; break;
    default: return -1;
  }
  std::memcpy(out, v->data(), sizeof(double) * v->size());
  return (int)v->size();
}
// constants, as flat doubles in struct order:
// phys(7) corr(6) joco(12) trml_wp(6) trml_tool(6) = 37, then dt, t_final, contact_alpha
int refh_get_constants(double *out) {
  int k = 0;
  const phys_constants &p = g_rec.phys_a;
  double ph[7] = {p.E, p.nu, p.rho0, p.K, p.G, p.mass, p.mass_tool};
  for (double v : ph) out[k++] = v;
  const corr_constants &c = g_rec.corr_a;
  double co[6] = {c.wdeltap, c.stresseps, c.xspheps, c.alpha, c.beta, c.eta};
  for (double v : co) out[k++] = v;
  const joco_constants &j = g_rec.joco;
  double jc[12] = {j.A, j.B, j.C, j.n, j.m, j.Tmelt, j.Tref, j.eps_dot_ref, j.tanh_a, j.tanh_b, j.tanh_c, j.tanh_d};
  for (double v : jc) out[k++] = v;
  const trml_constants &w = g_rec.trml_wp_a;
  double tw[6] = {w.cp, w.tq, w.k, w.alpha, w.T_init, w.eta};
  for (double v : tw) out[k++] = v;
  const trml_constants &t = g_rec.trml_tool_a;
  double tt[6] = {t.cp, t.tq, t.k, t.alpha, t.T_init, t.eta};
  for (double v : tt) out[k++] = v;
  out[k++] = global_dt;
  out[k++] = global_t_final;
  out[k++] = g_rec.contact_alpha;
  out[k++] = g_rec.has_joco ? 1. : 0.;
  return k;
}
// grid: nx ny bbmin_x bbmin_y bbmax_x bbmax_y dx num_cell locked
int refh_get_grid(double *out) {
  grid_base *g = g_rec.grid;
  if (!g) return -1;
  out[0] = g->nx(); out[1] = g->ny(); out[2] = g->bbmin_x(); out[3] = g->bbmin_y();
  out[4] = g->bbmax_x(); out[5] = g->bbmax_y(); out[6] = g->dx(); out[7] = g->num_cell();
  out[8] = g->is_locked() ? 1. : 0.;
  return 9;
}
// max_cell of the last scene's grid when it is an adaptive grid_gpu_green, else 0
int refh_get_grid_max_cell() { return (int)g_rec.grid_max_cell; }
// the scene's tool (after positioning) and its velocity
int refh_get_scene_tool(double *seg_out, double *fillet_out, double *misc_out, double *vel_out) {
  if (!global_tool) return -1;
  glm::dvec2 v = global_tool->get_vel();
  vel_out[0] = v.x; vel_out[1] = v.y;
  return dump_tool(global_tool, seg_out, fillet_out, misc_out);
}

}  // extern "C"
