// Host-side scene setup and rigid-tool geometry.
//
// Restates, in this project's own code, the reference's host geometry and the reference
// cut scene:
//   * line / segment / circle segment   geometric_primitives.cpp:20-148
//   * tool construction and sampling    tool.cpp:20-144, 156-221, 342-375
//   * setup_ref_cut                     benchmarks.cpp:255-537
//   * tool VTK output                   vtk_writer.cpp:180-264
// The arithmetic keeps the reference's operation order so that the scene (positions,
// constants, tool polygon, grid box, dt) is bit-identical to what setup_ref_cut produces;
// the tests compare it against the reference's own sources compiled on the host.
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "mfree_b200.h"

namespace {

struct v2 {
  double x, y;
};
inline v2 mk(double x, double y) { return v2{x, y}; }
inline v2 operator+(v2 a, v2 b) { return mk(a.x + b.x, a.y + b.y); }
inline v2 operator-(v2 a, v2 b) { return mk(a.x - b.x, a.y - b.y); }
inline v2 operator*(double s, v2 a) { return mk(s * a.x, s * a.y); }
inline double dot(v2 a, v2 b) { return a.x * b.x + a.y * b.y; }
inline double length(v2 a) { return std::sqrt(dot(a, a)); }
inline v2 normalize(v2 a) {
  double inv = 1. / std::sqrt(dot(a, a));
  return mk(a.x * inv, a.y * inv);
}

// line through two points: y = a x + b, or vertical x = b (geometric_primitives.cpp:70-85)
struct line_t {
  double a = 0., b = 0.;
  bool vertical = false;
};
line_t line_through(v2 p1, v2 p2) {
  line_t l;
  double detM = p1.x * 1. - 1. * p2.x;
  if (std::fabs(detM) < 1e-12) {
    l.vertical = true;
    l.a = DBL_MAX;
    l.b = p1.x;
    return l;
  }
  l.a = (p1.y * 1. - 1. * p2.y) / detM;
  l.b = (p2.y * p1.x - p2.x * p1.y) / detM;
  return l;
}
// geometric_primitives.cpp:20-47
v2 intersect(const line_t &s, const line_t &l) {
  if (s.vertical && l.vertical) return mk(DBL_MAX, DBL_MAX);
  if (std::fabs(s.a - l.a) < 1e-12) return mk(DBL_MAX, DBL_MAX);
  if (s.vertical) return mk(s.b, l.a * s.b + l.b);
  if (l.vertical) return mk(l.b, s.a * l.b + s.b);
  double x = (l.b - s.b) / (s.a - l.a);
  return mk(x, s.a * x + s.b);
}
// foot of the perpendicular from xq (geometric_primitives.cpp:49-64)
v2 closest_point(const line_t &l, v2 xq) {
  if (l.vertical) return mk(l.b, xq.y);
  double bb = -1, cc = l.b, aa = l.a;
  double px = (bb * (bb * xq.x - aa * xq.y) - aa * cc) / (aa * aa + bb * bb);
  double py = (aa * (-bb * xq.x + aa * xq.y) - bb * cc) / (aa * aa + bb * bb);
  return mk(px, py);
}

// atan2 mapped to (0, 2 pi] (tool.cpp:27-34)
double angle_0_2pi(double y, double x) {
  double t = std::atan2(y, x);
  return t > 0. ? t : t + 2 * M_PI;
}

struct tool_geom {
  std::vector<mf_segment> segs;
  bool has_fillet = false;
  mf_fillet fillet{};
  double front = 0.;
  double mu = 0.;
  v2 vel = mk(0., 0.);
};

mf_segment make_segment(v2 left, v2 right) {  // geometric_primitives.cpp:112-122
  mf_segment s;
  std::memset(&s, 0, sizeof(s));
  s.left[0] = left.x; s.left[1] = left.y;
  s.right[0] = right.x; s.right[1] = right.y;
  v2 dist = right - left;
  v2 n = normalize(mk(dist.y, -dist.x));
  s.n[0] = n.x; s.n[1] = n.y;
  line_t l = line_through(left, right);
  s.a = l.a; s.b = l.b; s.vertical = l.vertical ? 1 : 0;
  return s;
}

void build_segments(tool_geom &t, const std::vector<v2> &pts) {  // tool.cpp:64-71
  size_t n = pts.size();
  for (size_t i = 0; i < n; ++i) t.segs.push_back(make_segment(pts[i], pts[i + 1 > n - 1 ? 0 : i + 1]));
}

v2 quad_roots(double a, double b, double c) {  // tool.cpp:20-25
  double x1 = (-b + std::sqrt(b * b - 4 * a * c)) / (2 * a);
  double x2 = (-b - std::sqrt(b * b - 4 * a * c)) / (2 * a);
  return mk(x1, x2);
}

// centre of a fillet of radius r on the bisector lm, tangent to l1 (tool.cpp:36-62)
v2 fillet_centre(double r, const line_t &lm, const line_t &l1) {
  if (l1.vertical) {
    line_t par;
    par.a = DBL_MAX; par.b = l1.b - r; par.vertical = true;
    return intersect(par, lm);
  }
  double A = l1.a - lm.a, B = l1.b - lm.b, C = r * std::sqrt(l1.a * l1.a + 1.);
  v2 sol = quad_roots(A * A, 2 * A * B, B * B - C * C);
  double xm = std::fmin(sol.x, sol.y);
  return mk(xm, lm.a * xm + lm.b);
}

// replace the corner br by a fillet of radius r (tool.cpp:73-102)
std::vector<v2> corner_with_fillet(tool_geom &t, v2 tl, v2 tr, v2 br, v2 bl, double r) {
  v2 nt = normalize(tr - br), nl = normalize(bl - br);
  v2 nm = normalize(0.5 * (nt + nl));
  line_t lm = line_through(br, br + nm);
  line_t l1 = line_through(tr, br), l2 = line_through(bl, br);
  v2 p = fillet_centre(r, lm, l1);
  v2 trc = closest_point(l1, p), blc = closest_point(l2, p);
  t.has_fillet = true;
  t.fillet.r = r;
  t.fillet.t1 = angle_0_2pi(p.y - trc.y, p.x - trc.x);
  t.fillet.t2 = angle_0_2pi(p.y - blc.y, p.x - blc.x);
  t.fillet.p[0] = p.x; t.fillet.p[1] = p.y;
  return {tl, tr, trc, blc, bl};
}

// tool(tl, length, height, rake, clearance, r, mu) (tool.cpp:342-375)
tool_geom construct_tool(v2 tl, double length, double height, double rake, double clear, double r, double mu) {
  tool_geom t;
  t.mu = mu;
  v2 tr = mk(tl.x + length, tl.y), bl = mk(tl.x, tl.y - height);
  double a_rake = rake * M_PI / 180.;
  double a_free = (90. - clear) * M_PI / 180.;
  // row vector (0,-1) times the column-major rotation [[c, -s], [s, c]]
  double cr = std::cos(a_rake), sr = std::sin(a_rake), cf = std::cos(a_free), sf = std::sin(a_free);
  v2 d_rake = mk(0. * cr + -1. * -sr, 0. * sr + -1. * cr);
  v2 d_free = mk(0. * cf + -1. * -sf, 0. * sf + -1. * cf);
  v2 trc = tr + d_rake, blc = bl + d_free;
  v2 br = intersect(line_through(tr, trc), line_through(bl, blc));
  if (r == 0.) build_segments(t, {tl, tr, br, bl});
  else build_segments(t, corner_with_fillet(t, tl, tr, br, bl, r));
  t.front = br.x;
  return t;
}

double tool_low(const tool_geom &t) {  // tool.cpp:187-197
  if (t.has_fillet) return t.fillet.p[1] - t.fillet.r;
  double y = DBL_MAX;
  for (auto &s : t.segs) y = std::fmin(y, s.left[1]);
  return y;
}

void tool_box(const tool_geom &t, double safety, double *bb) {  // tool.cpp:156-185
  double x_min = DBL_MAX, x_max = -DBL_MAX, y_min = DBL_MAX, y_max = -DBL_MAX;
  for (auto &s : t.segs) {
    x_min = std::fmin(s.left[0], x_min);
    x_max = std::fmax(s.left[0], x_max);
    y_min = std::fmin(s.left[1], y_min);
    y_max = std::fmax(s.left[1], y_max);
  }
  if (t.has_fillet) {
    y_min = tool_low(t);
    x_max = t.fillet.p[0] + t.fillet.r;
  }
  bb[0] = x_min - safety; bb[1] = x_max + safety; bb[2] = y_min - safety; bb[3] = y_max + safety;
}

// translate with the tool velocity over dt (tool.cpp:211-221)
void translate(tool_geom &t, double dt) {
  for (auto &s : t.segs) {
    s.left[0] = s.left[0] + dt * t.vel.x; s.left[1] = s.left[1] + dt * t.vel.y;
    s.right[0] = s.right[0] + dt * t.vel.x; s.right[1] = s.right[1] + dt * t.vel.y;
    line_t l = line_through(mk(s.left[0], s.left[1]), mk(s.right[0], s.right[1]));
    s.a = l.a; s.b = l.b; s.vertical = l.vertical ? 1 : 0;
  }
  if (t.has_fillet) {
    t.fillet.p[0] = t.fillet.p[0] + dt * t.vel.x;
    t.fillet.p[1] = t.fillet.p[1] + dt * t.vel.y;
  }
}

bool inside_tool(const tool_geom &t, v2 qp) {  // tool.cpp:104-119
  bool in = true;
  for (auto &s : t.segs) in = in && dot(mk(s.left[0], s.left[1]) - qp, mk(s.n[0], s.n[1])) < 0.;
  if (t.has_fillet) in = in || length(mk(t.fillet.p[0], t.fillet.p[1]) - qp) < t.fillet.r;
  return in;
}

std::vector<v2> sample(const tool_geom &t, double dx) {  // tool.cpp:121-144
  std::vector<v2> out;
  double bb[4];
  tool_box(t, 0.1 * dx, bb);
  int nx = (int)((bb[1] - bb[0]) / dx + 1);
  int ny = (int)((bb[3] - bb[2]) / dx + 1);
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++) {
      v2 p = mk(i * dx + bb[0], j * dx + bb[2]);
      if (inside_tool(t, p)) out.push_back(p);
    }
  return out;
}

void to_state(const tool_geom &t, mf_tool_state *o) {
  std::memset(o, 0, sizeof(*o));
  o->num_seg = (int)t.segs.size();
  for (size_t i = 0; i < t.segs.size() && i < 5; ++i) o->seg[i] = t.segs[i];
  o->has_fillet = t.has_fillet ? 1 : 0;
  o->fillet = t.fillet;
  o->mu = t.mu;
  o->vel[0] = t.vel.x; o->vel[1] = t.vel.y;
}
tool_geom from_state(const mf_tool_state *s) {
  tool_geom t;
  for (int i = 0; i < s->num_seg && i < 5; ++i) t.segs.push_back(s->seg[i]);
  t.has_fillet = s->has_fillet != 0;
  t.fillet = s->fillet;
  t.mu = s->mu;
  t.vel = mk(s->vel[0], s->vel[1]);
  return t;
}

// deterministic uniform doubles in [0,1) for the lattice jitter (splitmix64)
struct splitmix {
  unsigned long long s;
  double next() {
    unsigned long long z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
  }
};

}  // namespace

extern "C" {

int mf_tool_construct(double tl_x, double tl_y, double length, double height, double rake, double clear,
                      double r, double mu, mf_tool_state *out) {
  if (!out) return MF_ERR_INVALID;
  tool_geom t = construct_tool(mk(tl_x, tl_y), length, height, rake, clear, r, mu);
  to_state(t, out);
  return MF_OK;
}

int mf_tool_sample(const mf_tool_state *tool, double dx, double *xy_out, int capacity, int *n_out) {
  if (!tool || !(dx > 0.) || !n_out) return MF_ERR_INVALID;
  std::vector<v2> s = sample(from_state(tool), dx);
  *n_out = (int)s.size();
  if (xy_out)
    for (int i = 0; i < (int)s.size() && i < capacity; ++i) { xy_out[2 * i] = s[i].x; xy_out[2 * i + 1] = s[i].y; }
  return (xy_out && capacity < (int)s.size()) ? MF_ERR_RANGE : MF_OK;
}

int mf_tool_translate(mf_tool_state *tool, double dt) {
  if (!tool) return MF_ERR_INVALID;
  tool_geom t = from_state(tool);
  translate(t, dt);
  double ca = tool->contact_alpha, sm = tool->slave_mass;
  to_state(t, tool);
  tool->contact_alpha = ca;
  tool->slave_mass = sm;
  return MF_OK;
}

int mf_cut_params_reference(mf_cut_params *p, int ny, double rake, double clear, double chamfer, double speed,
                            double feed) {
  if (!p) return MF_ERR_INVALID;
  std::memset(p, 0, sizeof(*p));
  p->ny = ny;
  p->nx_lattice = 0;
  p->hi_x = 0.200; p->hi_y = 0.060;
  p->lo_x = 0.005; p->lo_y = p->hi_y - 3 * feed;
  p->hdx = 1.5;
  p->rake = rake; p->clear = clear; p->chamfer = chamfer; p->speed = speed; p->feed = feed;
  p->mu_fric = 0.35;
  p->contact_alpha = 0.1;
  double nudge = 0.004;
  p->tool_tl_x = -0.05 + nudge;
  p->tool_tl_y = 0.0986074;
  p->tool_length = -0.0086824 - -0.05;
  p->tool_height = 0.0986074 - 0.0555074;
  p->tool_front_x = NAN;
  p->sample_tool = 1;
  p->use_thermals = 1;
  p->E = 1.1; p->nu = 0.35; p->rho0 = 4.429998; p->rho_tool = 15.25;
  p->joco.A = 0.0086200; p->joco.B = 0.0033100; p->joco.C = 0.0100000; p->joco.m = 0.8; p->joco.n = 0.34;
  p->joco.Tref = 300.; p->joco.Tmelt = 1836.0000; p->joco.eps_dot_ref = 1e-6;
  p->joco.tanh_a = 1.1; p->joco.tanh_b = 0.4; p->joco.tanh_c = 12.; p->joco.tanh_d = 1.;
  p->trml_wp.cp = 553 * 1e-8; p->trml_wp.tq = 0.9; p->trml_wp.k = 7.1 * 1e-13; p->trml_wp.eta = 0.9;
  p->trml_tool.cp = 292 * 1e-08; p->trml_tool.tq = .0; p->trml_tool.k = 88 * 1e-13;
  p->corr.alpha = 1.; p->corr.beta = 1.; p->corr.eta = 0.1; p->corr.xspheps = 0.5; p->corr.stresseps = 0.3;
  p->cfl = 0.5;
  p->cutting_distance = 0.1;
  return MF_OK;
}

int mf_scene_free(mf_scene *s) {
  if (!s) return MF_OK;
  std::free(s->pos); std::free(s->vel); std::free(s->rho); std::free(s->T); std::free(s->h);
  std::free(s->fixed); std::free(s->tool_p);
  delete s;
  return MF_OK;
}

// setup_ref_cut (benchmarks.cpp:255-537), generalised: the reference parameters
// (mf_cut_params_reference) reproduce it exactly.
int mf_scene_cut(const mf_cut_params *P, mf_scene **out) {
  if (!P || !out) return MF_ERR_INVALID;
  *out = nullptr;
  const bool ref_lattice = P->nx_lattice <= 0;
  if (ref_lattice && P->ny < 2) return MF_ERR_INVALID;
  if (!ref_lattice && (P->ny < 1 || !(P->dx > 0.))) return MF_ERR_INVALID;
  if (!(P->hdx > 0.)) return MF_ERR_INVALID;

  double hi_x = P->hi_x, hi_y = P->hi_y, lo_x = P->lo_x, lo_y = P->lo_y;
  double dx;
  int nx, ny = P->ny;
  if (ref_lattice) {
    lo_y = hi_y - 3 * P->feed;
    double dy = (hi_y - lo_y) / (ny - 1);
    dx = dy;
    nx = (int)((hi_x - lo_x) / dx);
  } else {
    dx = P->dx;
    nx = P->nx_lattice;
  }
  const double hdx = P->hdx;

  mf_scene *S = new (std::nothrow) mf_scene;
  if (!S) return MF_ERR_NOMEM;
  std::memset(S, 0, sizeof(*S));

  mf_phys_constants &phys = S->phys;
  phys.E = P->E;
  phys.nu = P->nu;
  phys.rho0 = P->rho0;
  phys.G = phys.E / (2. * (1. + phys.nu));
  phys.K = 2.0 * phys.G * (1 + phys.nu) / (3 * (1 - 2 * phys.nu));
  phys.mass = dx * dx * phys.rho0;
  S->joco = P->joco;
  S->has_joco = 1;
  phys.mass_tool = dx * dx * P->rho_tool;
  if (P->use_thermals) {
    S->trml_wp = P->trml_wp;
    S->trml_wp.alpha = S->trml_wp.k / (phys.rho0 * S->trml_wp.cp);
    S->trml_wp.T_init = S->joco.Tref;
    S->trml_tool = P->trml_tool;
    S->trml_tool.alpha = S->trml_tool.k / (P->rho_tool * S->trml_tool.cp);
    S->trml_tool.T_init = S->joco.Tref;
  }
  S->corr = P->corr;
  {
    double h1 = 1. / (hdx * dx);
    double q = dx * h1;
    double fac = 10 * (M_1_PI) / 7.0 * h1 * h1;
    S->corr.wdeltap = fac * (1 - 1.5 * q * q * (1 - 0.5 * q));
  }

  // workpiece lattice (benchmarks.cpp:334-381)
  const int n = nx * ny;
  std::vector<v2> pos((size_t)n);
  double min_x = FLT_MAX, max_x = -FLT_MAX, min_y = FLT_MAX, max_y = -FLT_MAX;
  splitmix rng{P->seed};
  int it = 0;
  for (int i = 0; i < nx; i++) {
    for (int j = 0; j < ny; j++) {
      v2 q = mk(i * dx + lo_x, j * dx + lo_y);
      if (P->jitter != 0.) {
        double ux = rng.next(), uy = rng.next();
        q.x += (2. * ux - 1.) * P->jitter * dx;
        q.y += (2. * uy - 1.) * P->jitter * dx;
      }
      pos[it] = q;
      max_x = std::fmax(max_x, q.x);
      min_x = std::fmin(min_x, q.x);
      max_y = std::fmax(max_y, q.y);
      min_y = std::fmin(min_y, q.y);
      it++;
    }
  }
  if (!ref_lattice) {
    // explicit lattice: the top and right edges are the lattice's own
    hi_y = lo_y + (ny - 1) * dx;
    hi_x = lo_x + nx * dx;
  }
  std::vector<double> fixed((size_t)n), vel2(2 * (size_t)n, 0.), rho((size_t)n), h((size_t)n), T((size_t)n),
      tool_p((size_t)n, 0.);
  for (int i = 0; i < n; i++) {
    rho[i] = phys.rho0;
    h[i] = hdx * dx;
    T[i] = S->joco.Tref;
    bool f = pos[i].y < min_y + 0.5 * dx;
    f = f || (pos[i].x < min_x + dx / 2 && pos[i].y < min_y + 0.5 * (hi_y - lo_y));
    f = f || (pos[i].x > max_x - dx);
    fixed[i] = f ? 1. : 0.;
  }

  // tool (benchmarks.cpp:383-421)
  double vel_tool = (P->speed == 0.f) ? 83.333328 * 1e-5 : P->speed;
  tool_geom t = construct_tool(mk(P->tool_tl_x, P->tool_tl_y), P->tool_length, P->tool_height, P->rake,
                               P->clear, P->chamfer, P->mu_fric);
  if (ref_lattice || std::isnan(P->tool_front_x)) {
    if (t.front > lo_x) {
      double distance = t.front - lo_x;
      double time = distance / vel_tool;
      t.vel = mk(vel_tool, 0.);
      translate(t, -time);
    }
  } else {
    double distance = t.front - P->tool_front_x;
    double time = distance / vel_tool;
    t.vel = mk(vel_tool, 0.);
    translate(t, -time);
  }
  {
    double target_feed = P->feed;
    double current_feed = hi_y - tool_low(t);
    double dist_to_target_feed = std::fabs(current_feed - target_feed);
    double correction_time = dist_to_target_feed / vel_tool;
    double sign = (current_feed > target_feed) ? 1 : -1.;
    t.vel = mk(0., vel_tool);
    translate(t, correction_time * sign);
  }
  t.vel = mk(vel_tool, 0.);
  to_state(t, &S->tool);
  S->tool.contact_alpha = P->contact_alpha;
  S->tool.slave_mass = phys.mass;

  // tool particles (benchmarks.cpp:423-459)
  std::vector<v2> samples;
  if (P->sample_tool) samples = sample(t, dx);
  const int n_tool = (int)samples.size();
  const int N = n + n_tool;
  double bbmin_tool_x = FLT_MAX, bbmax_tool_y = -FLT_MAX;
  for (auto &s : samples) {
    bbmin_tool_x = std::fmin(bbmin_tool_x, s.x);
    bbmax_tool_y = std::fmax(bbmax_tool_y, s.y);
  }
  S->N = N;
  S->n_workpiece = n;
  S->n_tool = n_tool;
  S->pos = (double *)std::malloc(sizeof(double) * 2 * (size_t)N);
  S->vel = (double *)std::calloc(2 * (size_t)N, sizeof(double));
  S->rho = (double *)std::malloc(sizeof(double) * (size_t)N);
  S->T = (double *)std::malloc(sizeof(double) * (size_t)N);
  S->h = (double *)std::malloc(sizeof(double) * (size_t)N);
  S->fixed = (double *)std::malloc(sizeof(double) * (size_t)N);
  S->tool_p = (double *)std::malloc(sizeof(double) * (size_t)N);
  if (!S->pos || !S->vel || !S->rho || !S->T || !S->h || !S->fixed || !S->tool_p) {
    mf_scene_free(S);
    return MF_ERR_NOMEM;
  }
  for (int i = 0; i < n; ++i) {
    S->pos[2 * i] = pos[i].x; S->pos[2 * i + 1] = pos[i].y;
    S->rho[i] = rho[i]; S->T[i] = T[i]; S->h[i] = h[i]; S->fixed[i] = fixed[i]; S->tool_p[i] = 0.;
  }
  for (int k = 0; k < n_tool; ++k) {
    int i = n + k;
    S->pos[2 * i] = samples[k].x; S->pos[2 * i + 1] = samples[k].y;
    S->rho[i] = P->rho_tool;
    S->h[i] = hdx * dx;
    S->fixed[i] = (samples[k].x < bbmin_tool_x + dx / 2 || samples[k].y > bbmax_tool_y - dx / 2) ? 1. : 0.;
    S->T[i] = S->joco.Tref;
    S->tool_p[i] = 1.;
  }

  // grid box (benchmarks.cpp:464-495)
  double bmin_x = FLT_MAX, bmin_y = FLT_MAX, bmax_x = -FLT_MAX, bmax_y = -FLT_MAX;
  for (int i = 0; i < N; i++) {
    bmin_x = std::fmin(S->pos[2 * i], bmin_x);
    bmin_y = std::fmin(S->pos[2 * i + 1], bmin_y);
    bmax_x = std::fmax(S->pos[2 * i], bmax_x);
    bmax_y = std::fmax(S->pos[2 * i + 1], bmax_y);
  }
  bmin_x -= 1e-8; bmin_y -= 1e-8;
  bmax_x += 1e-8; bmax_y += 1e-8;
  double tb[4];
  tool_box(t, 1e-3, tb);
  bmin_x = std::fmin(bmin_x, tb[0]);
  bmin_y = std::fmin(bmin_y, tb[2]);
  bmax_x = std::fmax(bmax_x, tb[1]) + 10 * dx;
  bmax_y = std::fmax(bmax_y, tb[3]);
  double max_height = hi_y + hi_x - lo_x;
  bmax_y = std::fmax(bmax_y, max_height);
  S->grid_bbmin[0] = bmin_x; S->grid_bbmin[1] = bmin_y;
  S->grid_bbmax[0] = bmax_x; S->grid_bbmax[1] = bmax_y;
  S->grid_h = hdx * dx;

  // time step (benchmarks.cpp:529-531)
  S->dt = P->cfl * hdx * dx / (std::sqrt(phys.K / phys.rho0) + std::sqrt(vel_tool));
  S->t_final = P->cutting_distance / vel_tool;
  S->feed = P->feed;
  S->speed = vel_tool;
  *out = S;
  return MF_OK;
}

int mf_scene_setup_ref_cut(int ny, double rake, double clear, double chamfer, double speed, double feed,
                           mf_scene **out) {
  mf_cut_params p;
  int rc = mf_cut_params_reference(&p, ny, rake, clear, chamfer, speed, feed);
  if (rc != MF_OK) return rc;
  return mf_scene_cut(&p, out);
}

namespace {

// a scene of N particles with every array allocated (velocities zero) and no tool
mf_scene *scene_alloc(int N) {
  mf_scene *S = new (std::nothrow) mf_scene;
  if (!S) return nullptr;
  std::memset(S, 0, sizeof(*S));
  S->N = N;
  S->n_workpiece = N;
  S->pos = (double *)std::malloc(sizeof(double) * 2 * (size_t)N);
  S->vel = (double *)std::calloc(2 * (size_t)N, sizeof(double));
  S->rho = (double *)std::calloc((size_t)N, sizeof(double));
  S->T = (double *)std::calloc((size_t)N, sizeof(double));
  S->h = (double *)std::calloc((size_t)N, sizeof(double));
  S->fixed = (double *)std::calloc((size_t)N, sizeof(double));
  S->tool_p = (double *)std::calloc((size_t)N, sizeof(double));
  if (!S->pos || !S->vel || !S->rho || !S->T || !S->h || !S->fixed || !S->tool_p) {
    mf_scene_free(S);
    return nullptr;
  }
  return S;
}

// elastic constants from E, nu and rho0, with the particle mass of a dx x dx cell
void set_elastic(mf_phys_constants &phys, double E, double nu, double rho0, double dx) {
  std::memset(&phys, 0, sizeof(phys));
  phys.E = E;
  phys.nu = nu;
  phys.rho0 = rho0;
  phys.G = phys.E / (2. * (1. + phys.nu));
  phys.K = 2.0 * phys.G * (1 + phys.nu) / (3 * (1 - 2 * phys.nu));
  phys.mass = dx * dx * phys.rho0;
}

// the correction constants both validation scenes use, with W(dx) at h = hdx dx
void set_validation_corr(mf_corr_constants &corr, double dx, double hdx) {
  std::memset(&corr, 0, sizeof(corr));
  corr.alpha = 1.;
  corr.beta = 1.;
  corr.eta = 0.1;
  corr.xspheps = 0.5;
  corr.stresseps = 0.3;
  double h1 = 1. / (hdx * dx);
  double q = dx * h1;
  double fac = 10 * (M_1_PI) / 7.0 * h1 * h1;
  corr.wdeltap = fac * (1 - 1.5 * q * q * (1 - 0.5 * q));
}

}  // namespace

// setup_rings (benchmarks.cpp:161-253): a lattice of nbox x nbox points over the square
// [-ro, ro]^2 keeps the annulus ri <= r < ro, once shifted left and once right by ro + 0.001,
// the two copies interleaved point by point; the left ring moves at +200, the right at -200
// (the 170 of the time-step formula is not the velocity given)
int mf_scene_setup_rings(int nbox, mf_scene **out) {
  if (!out) return MF_ERR_INVALID;
  *out = nullptr;
  if (nbox < 2 || nbox > 46340) return MF_ERR_INVALID;
  const double ri = 0.03, ro = 0.04;
  const double spacing = ro + 0.001;
  const double dx = 2 * ro / (nbox - 1);
  const double hdx = 1.7;

  std::vector<v2> pos;
  for (int i = 0; i < nbox; i++) {
    for (int j = 0; j < nbox; j++) {
      double px = -ro + i * dx, py = -ro + j * dx;
      double dist = std::sqrt(px * px + py * py);
      if (dist < ro && dist >= ri) {
        pos.push_back(mk(px - spacing, py));
        pos.push_back(mk(px + spacing, py));
      }
    }
  }
  // the reference holds the points in an array of nbox^2 and asserts that fewer were made
  if (pos.empty() || pos.size() >= (size_t)nbox * (size_t)nbox) return MF_ERR_INVALID;
  const int n = (int)pos.size();

  mf_scene *S = scene_alloc(n);
  if (!S) return MF_ERR_NOMEM;
  set_elastic(S->phys, 1e7, 0.4, 1., dx);
  set_validation_corr(S->corr, dx, hdx);
  const double vel_ring = 170.;
  S->t_final = 2.5 * ro / vel_ring;
  S->dt = 0.5 * hdx * dx / (std::sqrt(S->phys.K / S->phys.rho0) + std::sqrt(vel_ring));
  for (int i = 0; i < n; i++) {
    S->pos[2 * i] = pos[i].x;
    S->pos[2 * i + 1] = pos[i].y;
    S->rho[i] = S->phys.rho0;
    S->h[i] = hdx * dx;
    S->vel[2 * i] = (pos[i].x < 0) ? 200 : -200;
  }
  S->grid_bbmin[0] = -5 * ro; S->grid_bbmin[1] = -2 * ro;
  S->grid_bbmax[0] = 5 * ro; S->grid_bbmax[1] = 2 * ro;
  S->grid_h = hdx * dx;
  *out = S;
  return MF_OK;
}

// setup_impact (benchmarks.cpp:23-159): the flyer is the disc r < ro of an nbox x nbox lattice
// over [-ro, ro]^2 shifted left by ro + 0.05, at +1000; the wall is nbox/2 columns from x = 0
// and the rows y = j dx - 1 <= 1, its top and bottom rows fixed; T = Tref everywhere
int mf_scene_setup_impact(int nbox, mf_scene **out) {
  if (!out) return MF_ERR_INVALID;
  *out = nullptr;
  if (nbox < 2 || nbox > 4096) return MF_ERR_INVALID;
  const double ro = 0.2;
  const double dx = 2 * ro / (nbox - 1);
  const double hdx = 1.7;
  const double spacing = ro + 0.05;

  std::vector<v2> pos;
  for (int i = 0; i < nbox; i++) {
    for (int j = 0; j < nbox; j++) {
      double px = -ro + i * dx, py = -ro + j * dx;
      double dist = std::sqrt(px * px + py * py);
      if (dist < ro) pos.push_back(mk(px - spacing, py));
    }
  }
  const int n_flyer = (int)pos.size();
  for (int i = 0; i < nbox / 2; i++) {
    for (int j = 0; j < 10 * nbox; j++) {
      if (j * dx - 1. > 1.) continue;
      pos.push_back(mk(i * dx, j * dx - 1.));
    }
  }
  const int n = (int)pos.size();
  if (n == 0) return MF_ERR_INVALID;

  mf_scene *S = scene_alloc(n);
  if (!S) return MF_ERR_NOMEM;
  set_elastic(S->phys, 200e9, 0.29, 7830.0, dx);
  set_validation_corr(S->corr, dx, hdx);
  mf_joco_constants &joco = S->joco;
  std::memset(&joco, 0, sizeof(joco));
  joco.A = 792.0e6;
  joco.B = 510.0e6;
  joco.C = 0.014;
  joco.m = 1.03;
  joco.n = 0.26;
  joco.Tref = 273.0;
  joco.Tmelt = 1793.0;
  joco.eps_dot_ref = 1;
  S->has_joco = 1;
  const double vel_flyer = 1e3;
  S->dt = 0.3 * hdx * dx / (std::sqrt(S->phys.K / S->phys.rho0) + std::sqrt(vel_flyer));
  S->t_final = 2 * ro / vel_flyer;
  for (int i = 0; i < n; i++) {
    S->pos[2 * i] = pos[i].x;
    S->pos[2 * i + 1] = pos[i].y;
    S->rho[i] = S->phys.rho0;
    S->h[i] = hdx * dx;
    if (i < n_flyer) S->vel[2 * i] = 1e3;
    S->fixed[i] = (pos[i].y < -1 + dx / 2 || pos[i].y > 1 - dx / 2) ? 1. : 0.;
    S->T[i] = joco.Tref;
  }
  S->grid_max_cell = 10 * n;
  S->grid_h = hdx * dx;
  *out = S;
  return MF_OK;
}

// tool triangles for VTK (vtk_writer.cpp:185-264)
int mf_vtk_write_tool(const mf_tool_state *ts, const char *path) {
  if (!ts || !path) return MF_ERR_INVALID;
  if (ts->num_seg == 0) return MF_OK;
  if (ts->num_seg != 4 && ts->num_seg != 5) return MF_ERR_INVALID;
  struct tri { v2 a, b, c; };
  std::vector<tri> tris;
  auto L = [&](int i) { return mk(ts->seg[i].left[0], ts->seg[i].left[1]); };
  auto R = [&](int i) { return mk(ts->seg[i].right[0], ts->seg[i].right[1]); };
  if (ts->num_seg == 4) {
    tris.push_back({L(0), R(0), R(1)});
    tris.push_back({L(2), R(2), R(3)});
  } else {
    tris.push_back({L(0), R(0), R(2)});
    tris.push_back({L(1), R(1), R(2)});
    tris.push_back({L(3), R(3), R(4)});
  }
  if (ts->has_fillet) {
    const int num_discr = 20;
    double t1 = std::fmin(ts->fillet.t1, ts->fillet.t2), t2 = std::fmax(ts->fillet.t1, ts->fillet.t2);
    double lo = t1 - 0.1 * t1;
    double d_angle = (t2 - t1) / (num_discr - 1);
    double r = ts->fillet.r;
    for (int i = 0; i < num_discr - 1; i++) {
      double a1 = lo + (i + 0) * d_angle, a2 = lo + (i + 1) * d_angle;
      v2 p1 = mk(ts->fillet.p[0], ts->fillet.p[1]);
      tris.push_back({p1, mk(p1.x + r * std::sin(a1), p1.y + r * std::cos(a1)),
                      mk(p1.x + r * std::sin(a2), p1.y + r * std::cos(a2))});
    }
  }
  FILE *fp = std::fopen(path, "w+");
  if (!fp) return MF_ERR_INVALID;
  int num_tri = (int)tris.size();
  std::fprintf(fp, "# vtk DataFile Version 2.0\nmfree iwf\nASCII\n\nDATASET UNSTRUCTURED_GRID\n");
  std::fprintf(fp, "POINTS %d float\n", 3 * num_tri);
  for (auto &t : tris) {
    std::fprintf(fp, "%f %f %f\n", t.a.x, t.a.y, 0.);
    std::fprintf(fp, "%f %f %f\n", t.b.x, t.b.y, 0.);
    std::fprintf(fp, "%f %f %f\n", t.c.x, t.c.y, 0.);
  }
  std::fprintf(fp, "\nCELLS %d %d\n", num_tri, 3 * num_tri + num_tri);
  for (int i = 0; i < num_tri; i++) std::fprintf(fp, "3 %d %d %d\n", 3 * i + 0, 3 * i + 1, 3 * i + 2);
  std::fprintf(fp, "\nCELL_TYPES %d\n", num_tri);
  for (int i = 0; i < num_tri; i++) std::fprintf(fp, "5\n");
  std::fclose(fp);
  return MF_OK;
}

}  // extern "C"
