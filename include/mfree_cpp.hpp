// C++ mirror of the reference's host API over the C ABI (mfree_b200.h), header-only.
//
// Keeps the names and argument meaning of the reference's classes and free functions so
// that its driver (mfree_gpu.cpp) and scene code read the same:
//   particle_gpu                   particle_gpu.h:33-87
//   grid_base / grid_gpu_green /   grid.h:32-73, grid_gpu_green.h:38-91,
//   grid_gpu_rothlin               grid_gpu_rothlin.h:55-91
//   leap_frog                      leap_frog.h:36-50
//   tool, tool_gpu_*               tool.h:36-144, tool_gpu.h:29-35
//   actions_setup_* / interactions_setup_*   actions_gpu.h:59-63, interactions_gpu.h:36-51
//   setup_ref_cut, setup_rings,    benchmarks.h:48, benchmarks.cpp:23-253
//   setup_impact
//   report_force                   output.h:26
//   vtk_writer_write               vtk_writer.h:28-29
//   global_dt, global_t_final, global_tool, global_step   benchmarks.cpp:20-21, mfree_gpu.cpp:46-48
//
// One process-wide mf_ctx (the "device state" the reference keeps in globals and
// __constant__ memory) holds particles, grid, constants and tool. Errors throw
// mfree::error carrying the C ABI status (the reference printed or exited instead).
#pragma once

#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "mfree_b200.h"

namespace mfree {

struct error : std::runtime_error {
  int code;
  error(int c, const std::string &where) : std::runtime_error(where + ": " + mf_error_string(c)), code(c) {}
};

inline void check(int rc, const char *where) {
  if (rc != MF_OK) throw error(rc, where);
}

struct double2_ {
  double x, y;
};

// the process-wide context (created on first use, on device 0 unless set before)
inline int &default_device() {
  static int dev = 0;
  return dev;
}
inline mf_ctx *context() {
  static mf_ctx *ctx = nullptr;
  if (!ctx) check(mf_ctx_create(default_device(), &ctx), "mf_ctx_create");
  return ctx;
}

}  // namespace mfree

// ---- globals of the reference (benchmarks.cpp:20-21, mfree_gpu.cpp:46-48) ----
inline double global_dt = 0.;
inline double global_t_final = 0.;
inline int global_step = 0;

typedef mfree::double2_ float2_t;

// ---- particle_gpu (particle_gpu.h:33-87): the particle system of the context ----
struct particle_gpu {
  unsigned int N = 0;
  mf_ctx *ctx = nullptr;
  // particle_gpu(pos, vel, rho, T, h, fixed, tool_p, N) (particle_gpu.cu:97-125)
  particle_gpu(const float2_t *pos, const float2_t *vel, const double *rho, const double *T, const double *h,
               const double *fixed, const double *tool_p, unsigned int n)
      : N(n), ctx(mfree::context()) {
    mfree::check(mf_particles_create(ctx, (int)n, &pos[0].x, &vel[0].x, rho, T, h, fixed, tool_p, nullptr),
                 "particle_gpu");
  }
  particle_gpu(const float2_t *pos, const float2_t *vel, const double *rho, const double *h, unsigned int n)
      : particle_gpu(pos, vel, rho, nullptr, h, nullptr, nullptr, n) {}
  particle_gpu(const float2_t *pos, const float2_t *vel, const double *rho, const double *h, const double *fixed,
               unsigned int n)
      : particle_gpu(pos, vel, rho, nullptr, h, fixed, nullptr, n) {}
  particle_gpu(const float2_t *pos, const float2_t *vel, const double *rho, const double *T, const double *h,
               const double *fixed, unsigned int n)
      : particle_gpu(pos, vel, rho, T, h, fixed, nullptr, n) {}
  // copy one field (MF_FIELD_*) to host memory
  std::vector<double> get(int field, int width) const {
    std::vector<double> v((size_t)N * width);
    mfree::check(mf_get_field(ctx, field, v.data()), "mf_get_field");
    return v;
  }
};

// ---- grid_base and its two implementations (grid.h:32-73) ----
class grid_base {
 protected:
  int kind_ = MF_GRID_GREEN;
  bool locked_ = false;
  double bbmin_[2] = {0, 0}, bbmax_[2] = {0, 0}, h_ = 0.;
  int max_cell_ = 0;
  bool bound_ = false;

 public:
  grid_base(int kind, int max_cell, int) : kind_(kind), locked_(false), max_cell_(max_cell) {}
  grid_base(int kind, int, float2_t bbmin, float2_t bbmax, double h)
      : kind_(kind), locked_(true), bbmin_{bbmin.x, bbmin.y}, bbmax_{bbmax.x, bbmax.y}, h_(h) {}
  virtual ~grid_base() = default;
  // attach the geometry to the particle system (done by the first step or sort)
  void bind(particle_gpu *p) {
    if (bound_) return;
    if (locked_)
      mfree::check(mf_grid_create_locked(p->ctx, kind_, bbmin_[0], bbmin_[1], bbmax_[0], bbmax_[1], h_), "grid");
    else
      mfree::check(mf_grid_create_adaptive(p->ctx, kind_, max_cell_), "grid");
    bound_ = true;
  }
  void geometry(int *nx, int *ny, int *nc, double *b5) const {
    mfree::check(mf_grid_geometry(mfree::context(), nx, ny, nc, b5), "mf_grid_geometry");
  }
  int nx() const { int a, b, c; double d[5]; geometry(&a, &b, &c, d); return a; }
  int ny() const { int a, b, c; double d[5]; geometry(&a, &b, &c, d); return b; }
  int num_cell() const {
    if (!bound_ && locked_) {  // before binding: the locked geometry (grid.cu:139-158)
      double dx = h_ * 2. / 2.;
      double lx = (bbmax_[0] + 1e-6) - (bbmin_[0] - 1e-6), ly = (bbmax_[1] + 1e-6) - (bbmin_[1] - 1e-6);
      return (int)(unsigned)__builtin_ceil(lx / dx) * (int)(unsigned)__builtin_ceil(ly / dx);
    }
    if (!bound_) return max_cell_;
    int a, b, c; double d[5]; geometry(&a, &b, &c, d); return c;
  }
  double dx() const { int a, b, c; double d[5]; geometry(&a, &b, &c, d); return d[4]; }
  double bbmin_x() const { int a, b, c; double d[5]; geometry(&a, &b, &c, d); return d[0]; }
  double bbmin_y() const { int a, b, c; double d[5]; geometry(&a, &b, &c, d); return d[1]; }
  double bbmax_x() const { int a, b, c; double d[5]; geometry(&a, &b, &c, d); return d[2]; }
  double bbmax_y() const { int a, b, c; double d[5]; geometry(&a, &b, &c, d); return d[3]; }
  bool is_locked() const { return locked_; }
  // assign_hashes + sort (grid.cu:89-95, grid_gpu_green.cu:203-205)
  void sort(particle_gpu *p) {
    bind(p);
    mfree::check(mf_grid_build(p->ctx), "mf_grid_build");
  }
  // get_cells into host arrays of num_cell() ints
  void get_cells(particle_gpu *p, int *cell_start, int *cell_end) {
    bind(p);
    mfree::check(mf_grid_get_cells(p->ctx, cell_start, cell_end), "mf_grid_get_cells");
  }
};

class grid_gpu_green : public grid_base {
 public:
  grid_gpu_green(unsigned int max_cell, unsigned int N) : grid_base(MF_GRID_GREEN, (int)max_cell, (int)N) {}
  grid_gpu_green(int num_part, float2_t bbmin, float2_t bbmax, double h)
      : grid_base(MF_GRID_GREEN, num_part, bbmin, bbmax, h) {}
};

class grid_gpu_rothlin : public grid_base {
 public:
  grid_gpu_rothlin(int max_cell, int N) : grid_base(MF_GRID_ROTHLIN, max_cell, N) {}
  grid_gpu_rothlin(int num_part, float2_t bbmin, float2_t bbmax, double h)
      : grid_base(MF_GRID_ROTHLIN, num_part, bbmin, bbmax, h) {}
};

// ---- constants (actions_setup_* / interactions_setup_*: one call sets both halves) ----
struct mfree_constants_state {
  mf_phys_constants phys{};
  mf_corr_constants corr{1., 0, 0, 0, 0, 0};
  mf_joco_constants joco{};
  mf_trml_constants trml_wp{}, trml_tool{};
  bool has_joco = false;
  void apply() {
    mfree::check(mf_set_constants(mfree::context(), &phys, &corr, has_joco ? &joco : nullptr, &trml_wp,
                                  &trml_tool),
                 "mf_set_constants");
  }
};
inline mfree_constants_state &mfree_constants() {
  static mfree_constants_state s;
  return s;
}
inline void actions_setup_physical_constants(mf_phys_constants p) { mfree_constants().phys = p; mfree_constants().apply(); }
inline void actions_setup_corrector_constants(mf_corr_constants c) { mfree_constants().corr = c; mfree_constants().apply(); }
inline void actions_setup_johnson_cook_constants(mf_joco_constants j) {
  mfree_constants().joco = j;
  mfree_constants().has_joco = true;
  mfree_constants().apply();
}
inline void actions_setup_thermal_constants_wp(mf_trml_constants t) { mfree_constants().trml_wp = t; mfree_constants().apply(); }
inline void actions_setup_thermal_constants_tool(mf_trml_constants t) { mfree_constants().trml_tool = t; mfree_constants().apply(); }

// ---- tool (tool.h:36-144) and tool_gpu (tool_gpu.h:29-35) ----
class tool {
 public:
  mf_tool_state s{};
  tool() = default;
  // tool(tl, length, height, rake, clearance, r, mu) (tool.cpp:342-375)
  tool(float2_t tl, double length, double height, double rake, double clear, double r, double mu) {
    mfree::check(mf_tool_construct(tl.x, tl.y, length, height, rake, clear, r, mu, &s), "tool");
  }
  void set_vel(float2_t v) { s.vel[0] = v.x; s.vel[1] = v.y; }
  float2_t get_vel() const { return {s.vel[0], s.vel[1]}; }
  double mu() const { return s.mu; }
  void update_tool(double dt) { mfree::check(mf_tool_translate(&s, dt), "update_tool"); }
  std::vector<float2_t> sample_tool(double dx) const {
    int n = 0;
    mf_tool_sample(&s, dx, nullptr, 0, &n);
    std::vector<float2_t> out((size_t)n);
    mfree::check(mf_tool_sample(&s, dx, &out[0].x, n, &n), "sample_tool");
    return out;
  }
};
inline tool *global_tool = nullptr;

// tool_gpu_set_up_tool (tool_gpu.cu:224-271)
inline void tool_gpu_set_up_tool(tool *t, double alpha, mf_phys_constants phys) {
  t->s.contact_alpha = alpha;
  t->s.slave_mass = phys.mass;
  mfree::check(mf_tool_set(mfree::context(), &t->s), "tool_gpu_set_up_tool");
}

// ---- leap_frog (leap_frog.h:36-50) ----
class leap_frog {
 public:
  leap_frog(unsigned int, unsigned int) {}
  // one explicit step (leap_frog.cu:94-155); the tool moves on the device
  void step(particle_gpu *p, grid_base *g) {
    g->bind(p);
    mfree::check(mf_set_dt(p->ctx, global_dt), "mf_set_dt");
    mfree::check(mf_step(p->ctx, 1), "mf_step");
    if (global_tool) mfree::check(mf_tool_get(p->ctx, &global_tool->s), "mf_tool_get");
  }
};

// ---- report_force (output.cu:31-39): x = cutting force, y = feed force ----
inline float2_t report_force(particle_gpu *p) {
  double f[2];
  mfree::check(mf_report_force(p->ctx, f), "report_force");
  return {f[0], f[1]};
}

// ---- vtk_writer_write (vtk_writer.cpp:20-264): results/vtk_out_%06d.vtk, vtk_tool_%06d.vtk ----
inline void vtk_writer_write(const particle_gpu *p, int step) {
  char buf[256];
  std::snprintf(buf, sizeof(buf), "results/vtk_out_%06d.vtk", step);
  mfree::check(mf_vtk_write_particles(p->ctx, buf), "vtk_writer_write");
}
inline void vtk_writer_write(const tool *t, int step) {
  if (!t) return;  // a scene without a tool (setup_rings, setup_impact) leaves global_tool null
  char buf[256];
  std::snprintf(buf, sizeof(buf), "results/vtk_tool_%06d.vtk", step);
  mfree::check(mf_vtk_write_tool(&t->s, buf), "vtk_writer_write");
}

// the same particle file written while the steps go on; vtk_writer_flush waits for all
inline void vtk_writer_write_async(const particle_gpu *p, int step) {
  char buf[256];
  std::snprintf(buf, sizeof(buf), "results/vtk_out_%06d.vtk", step);
  mfree::check(mf_vtk_write_particles_async(p->ctx, buf), "vtk_writer_write_async");
}
inline void vtk_writer_flush(const particle_gpu *p) { mfree::check(mf_vtk_flush(p->ctx), "vtk_writer_flush"); }

// ---- tool_wear (tool_wear.h, tool_wear.cu:20-64): Usui wear evaluated on the device ----
class tool_wear {
 public:
  tool_wear(double usui_K, double usui_alpha, unsigned int /*N_part*/, mf_phys_constants /*phys*/,
            float2_t /*tool_vel: the tool's own velocity is used*/)
      : m_K(usui_K), m_alpha(usui_alpha) {}
  void eval_usui(const particle_gpu *particles, double dt, double &usui_min, double &usui_max, double &usui_avg) {
    double out[3];
    mfree::check(mf_tool_wear_usui(particles->ctx, m_K, m_alpha, out), "tool_wear::eval_usui");
    usui_min = out[0];
    usui_max = out[1];
    usui_avg = out[2];
    m_accum_wear += dt * usui_avg;
  }
  double get_accum_wear() const { return m_accum_wear; }

 private:
  double m_K = 0., m_alpha = 0., m_accum_wear = 0.;
};
inline tool_wear *global_wear = nullptr;

// ---- the scenes of benchmarks.cpp: a host scene made into particles, a grid and constants ----
// (the grid is the scene's locked box, or adaptive when the scene asks for one; a scene
// with a tool also becomes global_tool)
inline particle_gpu *particles_from_scene(mf_scene *sc, grid_base **grid) {
  std::vector<float2_t> pos((size_t)sc->N), vel((size_t)sc->N);
  for (int i = 0; i < sc->N; ++i) {
    pos[i] = {sc->pos[2 * i], sc->pos[2 * i + 1]};
    vel[i] = {sc->vel[2 * i], sc->vel[2 * i + 1]};
  }
  particle_gpu *p = new particle_gpu(pos.data(), vel.data(), sc->rho, sc->T, sc->h, sc->fixed, sc->tool_p, sc->N);
  if (sc->grid_max_cell > 0)
    *grid = new grid_gpu_green((unsigned)sc->grid_max_cell, (unsigned)sc->N);
  else
    *grid = new grid_gpu_green(sc->N, float2_t{sc->grid_bbmin[0], sc->grid_bbmin[1]},
                               float2_t{sc->grid_bbmax[0], sc->grid_bbmax[1]}, sc->grid_h);
  auto &C = mfree_constants();
  C.phys = sc->phys;
  C.corr = sc->corr;
  C.joco = sc->joco;
  C.has_joco = sc->has_joco != 0;
  C.trml_wp = sc->trml_wp;
  C.trml_tool = sc->trml_tool;
  C.apply();
  if (sc->tool.num_seg > 0) {
    global_tool = new tool();
    global_tool->s = sc->tool;
    mfree::check(mf_tool_set(p->ctx, &global_tool->s), "tool_gpu_set_up_tool");
  }
  global_dt = sc->dt;
  global_t_final = sc->t_final;
  mf_scene_free(sc);
  return p;
}

// setup_ref_cut (benchmarks.cpp:255-537)
inline particle_gpu *setup_ref_cut(int ny, grid_base **grid, double rake = 0., double clear = 0., double chamfer = 0.,
                                   double speed = 0., double feed = 0.01) {
  mf_scene *sc = nullptr;
  mfree::check(mf_scene_setup_ref_cut(ny, rake, clear, chamfer, speed, feed, &sc), "setup_ref_cut");
  return particles_from_scene(sc, grid);
}

// setup_rings (benchmarks.cpp:161-253) and setup_impact (benchmarks.cpp:23-159): no tool
inline particle_gpu *setup_rings(int nbox, grid_base **grid) {
  mf_scene *sc = nullptr;
  mfree::check(mf_scene_setup_rings(nbox, &sc), "setup_rings");
  return particles_from_scene(sc, grid);
}
inline particle_gpu *setup_impact(int nbox, grid_base **grid) {
  mf_scene *sc = nullptr;
  mfree::check(mf_scene_setup_impact(nbox, &sc), "setup_impact");
  return particles_from_scene(sc, grid);
}
