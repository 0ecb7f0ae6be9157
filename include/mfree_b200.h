/*
 * mfree_b200: C ABI of the B200-native explicit 2D SPH cutting step.
 *
 * One context (mf_ctx) owns one particle system on one GPU: the particle_gpu state, the
 * cell-list grid (grid_gpu_green / grid_gpu_rothlin semantics), the leap_frog stepper,
 * the constants and the rigid tool. Every entry point returns an int status (MF_OK = 0,
 * negative on error); no entry point exits the process or prints.
 *
 * Units and layouts are the reference's: cm, g, microseconds; vector fields interleaved
 * (pos = x0 y0 x1 y1 ..., S = Sxx Sxy Syy Szz per particle), flags as 0/1 doubles.
 * The comment above each function names the reference interface it replaces
 * (file:line within the reference project iwf-inspire/mfree_iwf-ul_cut_gpu).
 */
#ifndef MFREE_B200_H
#define MFREE_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define MF_ABI_VERSION 2

/* ---- status codes ---- */
#define MF_OK 0
#define MF_ERR_INVALID (-1)     /* bad argument (null pointer, size, enum, flag value) */
#define MF_ERR_CUDA (-2)        /* a CUDA runtime call failed (see mf_last_cuda_error) */
#define MF_ERR_STATE (-3)       /* call out of order (e.g. step before particles/grid) */
#define MF_ERR_RANGE (-4)       /* size beyond a documented maximum / grid budget exceeded */
#define MF_ERR_NOMEM (-5)       /* device or host allocation failed */
#define MF_ERR_NO_DEVICE (-6)   /* no CUDA device (the product has no CPU fallback) */
#define MF_ERR_DEVICE_FAULT (-7) /* a kernel reported an internal error (bounded wait expired) */
#define MF_ERR_IO (-8)          /* a state file could not be written or read */
#define MF_ERR_CORRUPT (-9)     /* a state file failed its checks (format, size, checksum) */

/* ---- particle fields (particle_gpu.h:33-87) ---- */
#define MF_FIELD_POS 0        /* 2 doubles */
#define MF_FIELD_VEL 1        /* 2 */
#define MF_FIELD_H 2          /* 1 */
#define MF_FIELD_RHO 3        /* 1 */
#define MF_FIELD_P 4          /* 1: pressure of the last predictor (0 for tool particles) */
#define MF_FIELD_S 5          /* 4: Sxx Sxy Syy Szz */
#define MF_FIELD_R 6          /* 4: artificial stress Rxx Rxy Ryy 0 (0 for tool particles) */
#define MF_FIELD_FC 7         /* 2 */
#define MF_FIELD_FT 8         /* 2 */
#define MF_FIELD_N 9          /* 2: contact normal, indexed by array position (not permuted) */
#define MF_FIELD_FIXED 10     /* 1: 0/1 */
#define MF_FIELD_BLANKED 11   /* 1: 0/1 */
#define MF_FIELD_TOOL 12      /* 1: 0/1 (tool_particle) */
#define MF_FIELD_EPS_PL 13    /* 1 */
#define MF_FIELD_EPS_PL_DOT 14 /* 1 */
#define MF_FIELD_T 15         /* 1 */
#define MF_FIELD_POS_T 16     /* 2 */
#define MF_FIELD_VEL_T 17     /* 2 */
#define MF_FIELD_RHO_T 18     /* 1 */
#define MF_FIELD_S_T 19       /* 4 */
#define MF_FIELD_T_T 20       /* 1 */
#define MF_FIELD_S_DER 21     /* 4: only with MF_OPT_KEEP_DERIVATIVES */
#define MF_FIELD_V_DER 22     /* 4: only with MF_OPT_KEEP_DERIVATIVES */
#define MF_FIELD_IDX 23       /* 1 int: Green = sort permutation, Rothlin = persistent id */
#define MF_FIELD_HASH 24      /* 1 int: cell hash of the last sort, in array order */
#define MF_FIELD_ID 25        /* 1 int: particle number at creation, carried through every sort
                                 (no counterpart in the reference: its Green grid keeps none) */
#define MF_NUM_FIELDS 26

/* ---- enums ---- */
#define MF_GRID_GREEN 0        /* grid_gpu_green.h:38-91 */
#define MF_GRID_ROTHLIN 1      /* grid_gpu_rothlin.h:55-91 */
#define MF_THERMAL_BROOKSHAW 0 /* types.h:94 */
#define MF_THERMAL_PSE 1       /* types.h:95 */
#define MF_JC_JOHNSON_COOK 0   /* plasticity.cuh:30-46 */
#define MF_JC_TANH 1           /* plasticity.cuh:48-70 (used by the secant solve, as m_s_yield) */
#define MF_PRECISION_FP64 0    /* plain FP64 */
#define MF_PRECISION_MIXED 1   /* FP32 pair sums on cell-relative coordinates, FP64 integration */

/* option bits for mf_set_flags */
#define MF_OPT_KEEP_DERIVATIVES 1 /* also store S_der / v_der (the reference's public arrays) */
#define MF_OPT_NO_GRAPHS 2        /* launch kernels directly instead of replaying CUDA graphs */
#define MF_OPT_SORT_EVERY_STEP 4  /* mixed form: sort the cell list every step, as the FP64 form
                                     does (the default; overrides MF_OPT_NEIGHBOUR_LISTS) */
#define MF_OPT_FUSED_PREDICTOR 8  /* with MF_OPT_NEIGHBOUR_LISTS: run the next step's predictor in
                                     the finish kernel instead of the reorder kernel (measured
                                     ~3 % slower per step on the ~150k-particle cut) */
#define MF_OPT_NEIGHBOUR_LISTS 16 /* mixed form: keep neighbour lists between cell-list sorts,
                                     sorting when a particle's next predicted position is more
                                     than 0.45 skin from where its list was built (the fastest
                                     form; over a 1 mm cut of the ~150k-particle scene no pair
                                     was missing from the lists in 1,053 brute-force checks) */

/* ---- constants (constants_structs.h:25-82), same member order ---- */
typedef struct { double E, nu, rho0, K, G, mass, mass_tool; } mf_phys_constants;
typedef struct { double cp, tq, k, alpha, T_init, eta; } mf_trml_constants;
typedef struct { double wdeltap, stresseps, xspheps, alpha, beta, eta; } mf_corr_constants;
typedef struct {
  double A, B, C, n, m, Tmelt, Tref, eps_dot_ref, tanh_a, tanh_b, tanh_c, tanh_d;
} mf_joco_constants;

/* ---- rigid tool (tool_gpu.cuh:32-52 + the __constant__ block of tool_gpu.cu:21-27) ---- */
typedef struct {
  double left[2], right[2];
  double a, b;  /* line y = a x + b, or x = b if vertical */
  int vertical;
  double n[2];  /* outward normal (not updated when the tool moves, as in the reference) */
} mf_segment;
typedef struct { double r, t1, t2, p[2]; } mf_fillet;
typedef struct {
  int num_seg;        /* 0 (no tool), 4, or 5 (5 means segment 2 is the fillet) */
  mf_segment seg[5];
  int has_fillet;
  mf_fillet fillet;
  double mu;            /* friction coefficient */
  double contact_alpha; /* penalty factor */
  double slave_mass;    /* workpiece particle mass */
  double vel[2];        /* tool velocity */
} mf_tool_state;

/* ---- run-time status (replaces printf / exit diagnostics) ---- */
typedef struct {
  long long steps;            /* steps taken by this context */
  long long blanked;          /* particles currently blanked */
  long long newly_blanked;    /* blanked by invalidate() since the last status read */
  long long out_of_grid;      /* hashes outside [0, num_cell) clamped since creation */
  long long secant_cap_hits;  /* JC secant solves that hit the iteration cap */
  int max_cell_occupancy;     /* largest particles-per-cell seen in the last sort */
  int error_flags;            /* bit 1: the adaptive grid outgrew max_cell; bit 2: a neighbour
                                 list was full (neighbours dropped); bit 3: a persistent batch
                                 launch's barrier wait expired (mf_batch_set_form); bit 0 (a bounded wait in
                                 the cell scan expired) is no longer raised: the scan waits
                                 for nothing */
  long long secant_iterations; /* JC secant iterations since creation (cost diagnostic) */
  long long sorts;            /* cell-list sorts since creation (one per step, except for the
                                 mixed form with neighbour lists) */
} mf_status;

typedef struct mf_ctx mf_ctx;

/* ---- context ---- */
int mf_version(void);
const char *mf_error_string(int code);
int mf_last_cuda_error(const mf_ctx *ctx);            /* cudaError_t of the last failure */
int mf_ctx_create(int device, mf_ctx **out);
int mf_ctx_destroy(mf_ctx *ctx);
int mf_ctx_stream(mf_ctx *ctx, void **cuda_stream);   /* the stream all work is queued on */
int mf_set_flags(mf_ctx *ctx, int flags);
/* Skin of the mixed form's neighbour lists (a length; <= 0 restores the default, a tenth of
   the cell size; larger values are limited to half the cell size): each particle lists its
   candidates within 2 h + skin, and the cell list is sorted again on the steps where some
   particle would otherwise be more than 0.45 skin from where its list was built. No
   counterpart in the reference, which sorts every step. */
int mf_set_neighbour_skin(mf_ctx *ctx, double skin);
/* Diagnostic of the neighbour lists (no counterpart in the reference), O(N^2): after a step on
   lists, counts the pairs of unblanked, finite particles closer than 2 h_i in the current pair
   records (*pairs) and those of them missing from the lists (*missing, 0 when the lists hold
   what they promise). *stale = 1 when the records are already the next step's (fused predictor)
   and that step sorts, so that the lists need not hold for them. MF_ERR_STATE unless the last
   step ran on neighbour lists. */
int mf_list_check(mf_ctx *ctx, long long *pairs, long long *missing, int *stale);
int mf_synchronize(mf_ctx *ctx);

/* ---- particles: particle_gpu(...) constructors (particle_gpu.h:81-86, particle_gpu.cu:97-125).
   pos, vel, rho and h are required; T, fixed, tool_p and S may be NULL (zero). Flag arrays
   must hold exactly 0 or 1. ---- */
int mf_particles_create(mf_ctx *ctx, int N, const double *pos, const double *vel, const double *rho,
                        const double *T, const double *h, const double *fixed, const double *tool_p,
                        const double *S);
int mf_particles_count(const mf_ctx *ctx, int *N);
/* copy a field to / from host memory: N * width doubles (ints for IDX and HASH) */
int mf_get_field(mf_ctx *ctx, int field, void *host);
int mf_set_field(mf_ctx *ctx, int field, const void *host);

/* ---- grid: grid_gpu_green(N, bbmin, bbmax, h) / grid_gpu_rothlin(...) locked geometry
   (grid.cu:139-158), or the adaptive grid(max_cell, N) (grid.cu:97-136,160-162) ---- */
int mf_grid_create_locked(mf_ctx *ctx, int kind, double bbmin_x, double bbmin_y, double bbmax_x,
                          double bbmax_y, double h);
int mf_grid_create_adaptive(mf_ctx *ctx, int kind, int max_cell);
/* grid_base accessors (grid.h:51-72): out5 = bbmin_x bbmin_y bbmax_x bbmax_y dx */
int mf_grid_geometry(mf_ctx *ctx, int *nx, int *ny, int *num_cell, double *out5);
/* update_geometry + assign_hashes + sort (leap_frog.cu:106-108) without stepping */
int mf_grid_build(mf_ctx *ctx);
/* get_cells (grid_gpu_green.cu:207-210 / grid_gpu_rothlin.cu:129-136) into host arrays of
   num_cell ints. Green: empty cells have start = -1 (their end is -1 here; the reference
   leaves it stale). Rothlin: start[c] = #particles with hash < c, end[c] = start[c+1]. */
int mf_grid_get_cells(mf_ctx *ctx, int *start, int *end);

/* ---- constants: actions_setup_* (actions_gpu.cu:438-469) and interactions_setup_*
   (interactions_gpu.cu:433-459) in one call. joco NULL = no plasticity; trml_* NULL = 0. */
int mf_set_constants(mf_ctx *ctx, const mf_phys_constants *phys, const mf_corr_constants *corr,
                     const mf_joco_constants *joco, const mf_trml_constants *trml_wp,
                     const mf_trml_constants *trml_tool);
/* the constants last set (has_joco: 0 when the material is not plastic) */
int mf_get_constants(const mf_ctx *ctx, mf_phys_constants *phys, mf_corr_constants *corr, mf_joco_constants *joco,
                     mf_trml_constants *trml_wp, mf_trml_constants *trml_tool, int *has_joco);
int mf_set_options(mf_ctx *ctx, int thermal_solver, int jc_model, int precision);
int mf_set_dt(mf_ctx *ctx, double dt); /* global_dt (benchmarks.cpp:20) */
/* Tool-workpiece contact conductance, an extension with no counterpart in the reference (whose
   heat crosses the interface only through the sampled tool particles' conduction terms,
   interactions_gpu.cu:314-326): each step, a workpiece particle that the contact treatment finds
   inside the tool gains dt h (T_tool - T) / (cp sqrt(m rho)) in temperature, h in the library's
   units (1e8 W/m^2K = 1e-7 g/(us^3 K)), sqrt(m / rho) being its contact length per unit depth;
   applied after the friction heat, before the return map, where the workpiece's cp > 0.
   h = 0 (the default) switches it off and leaves the reference's step unchanged. Contexts with
   it on step in the child-graph batch form and have no differentiable step (MF_ERR_INVALID). */
int mf_set_contact_conductance(mf_ctx *ctx, double h_contact, double T_tool);

/* ---- tool: tool_gpu_set_up_tool (tool_gpu.cu:224-271); the per-step tool_gpu_update_tool
   (tool_gpu.cu:275-316) happens on the device inside mf_step. NULL or num_seg = 0: no tool. */
int mf_tool_set(mf_ctx *ctx, const mf_tool_state *tool);
int mf_tool_get(mf_ctx *ctx, mf_tool_state *tool);

/* ---- stepping: leap_frog::step (leap_frog.cu:94-155), n times, queued asynchronously ---- */
int mf_step(mf_ctx *ctx, int n_steps);
/* One step, launched kernel by kernel (no graph) with CUDA events between its four parts
   (the cell sort, predictor, interactions + rates, corrector .. plasticity); their durations
   in stage_ms[4], in milliseconds. Synchronizes the context's stream. For timing only: the
   step is the same as one of mf_step. No counterpart in the reference. */
int mf_step_timed(mf_ctx *ctx, float *stage_ms);
/* parts of one step, for parity tests: 0 grid (sort), 1 predictor (init, predict, eos,
   artificial stress), 2 interactions + rates, 3 corrector .. invalidate. */
int mf_step_stage(mf_ctx *ctx, int stage);
/* report_force (output.cu:31-39): sum of fc + ft after the last step, compensated */
int mf_report_force(mf_ctx *ctx, double out[2]);
/* queue a copy of the last step's tool force (2 doubles) to host memory; with pinned host
   memory the copy is asynchronous and complete after the next mf_synchronize */
int mf_force_last_async(mf_ctx *ctx, double *host_out2);
/* per-step force log since the last call (or creation), at most max entries of 2 doubles */
int mf_force_log(mf_ctx *ctx, double *out, int max_entries, int *n_out);
int mf_status_get(mf_ctx *ctx, mf_status *status);

/* ---- cell list without device allocation (no counterpart in the reference) ----
   For callers that cannot allocate device memory (a host that reserves all device memory at
   start-up and allows no driver allocation later, or a foreign-language binding that passes
   device pointers but has no access to the CUDA allocator): the hash, stable permutation and
   grid_gpu_green-format cell bounds that mf_grid_build computes for a locked grid, from
   caller-owned device buffers only (d_pos: 2N doubles; d_hash_sorted, d_idx: N ints;
   d_cell_start, d_cell_end: nx*ny ints, -1 on empty cells), queued on `stream`. The grid is
   given directly (origin bbmin, cell size dx, nx x ny cells, as mf_grid_geometry reports).
   d_pos must be 16-byte aligned, the int buffers 4-byte aligned (MF_ERR_INVALID otherwise,
   before anything is launched). Scratch is one fixed device array of 26 MiB inside the
   library, so N is limited to MF_NOALLOC_MAX_PARTICLES and nx*ny to MF_NOALLOC_MAX_CELLS
   (MF_ERR_RANGE beyond). A particle outside the grid is put into the nearest cell and counted;
   a cell of m particles costs O(m^2) in all. d_status (optional, caller-owned device memory,
   8-byte aligned; NULL: not written) receives, after every other kernel of the call, the
   number of such clamped particles, the error flags (0: the scan has no bounded waits left to
   expire; the field is kept for callers that test it) and the largest cell occupancy; a nonzero out_of_grid or error_flags means
   the cell list is not the reference's. The return code covers the launches only (each
   launch's own error; an earlier error of the caller's work is neither read nor cleared). The
   first call on a device looks up the scratch array's address and caches it; make it before
   any stream capture. After a cudaDeviceReset the cached address is stale: do not call this
   again on a device that was reset. Calls share the array: calls that overlap on the GPU race.
   No cudaMalloc/cudaFree is made. */
#define MF_NOALLOC_MAX_PARTICLES (1 << 19)
#define MF_NOALLOC_MAX_CELLS (1 << 21)
typedef struct {
  unsigned long long out_of_grid;        /* particles clamped into the grid */
  unsigned long long error_flags;        /* 0 (the scan has no bounded waits) */
  unsigned long long max_cell_occupancy; /* largest number of particles in one cell */
} mf_noalloc_status;
int mf_cells_build_noalloc(const double *d_pos, int N, double bbmin_x, double bbmin_y, double dx, int nx, int ny,
                           int *d_hash_sorted, int *d_idx, int *d_cell_start, int *d_cell_end,
                           mf_noalloc_status *d_status, void *stream);

/* ---- host scene setup: setup_ref_cut (benchmarks.cpp:255-537) and its generalisation ---- */
typedef struct {
  int N, n_workpiece, n_tool;
  double *pos, *vel, *rho, *T, *h, *fixed, *tool_p; /* host arrays owned by the scene */
  mf_phys_constants phys;
  mf_corr_constants corr;
  mf_joco_constants joco;
  mf_trml_constants trml_wp, trml_tool;
  int has_joco;
  mf_tool_state tool;
  double grid_bbmin[2], grid_bbmax[2], grid_h;
  double dt, t_final;
  double feed, speed;
  int grid_max_cell; /* > 0: an adaptive grid of at most this many cells, its box taken from the
                        particles at every sort (grid_gpu_green(max_cell, N), grid.cu:139-158);
                        0: the locked box grid_bbmin .. grid_bbmax with cells of grid_h */
} mf_scene;

typedef struct {
  /* lattice: reference mode (nx_lattice == 0): ny rows spanning [hi_y - 3 feed, hi_y]
     (benchmarks.cpp:266-273); explicit mode: nx_lattice x ny rows at spacing dx from lo. */
  int ny;
  int nx_lattice;
  double dx;
  double lo_x, lo_y, hi_x, hi_y;
  double hdx;
  double jitter;            /* uniform jitter amplitude as a fraction of dx (0 = none) */
  unsigned long long seed;
  /* tool (tool.cpp:342-375; positioning benchmarks.cpp:398-414) */
  double rake, clear, chamfer, speed, feed, mu_fric, contact_alpha;
  double tool_tl_x, tool_tl_y, tool_length, tool_height;
  double tool_front_x;      /* explicit mode: translate the tool so front() = this x */
  int sample_tool;          /* add thermal-only tool particles (benchmarks.cpp:425-459) */
  int use_thermals;
  /* material */
  double E, nu, rho0, rho_tool;
  mf_joco_constants joco;
  mf_trml_constants trml_wp, trml_tool;
  mf_corr_constants corr;   /* wdeltap is computed */
  double cfl;               /* dt = cfl*hdx*dx/(sqrt(K/rho0) + sqrt(speed)) (benchmarks.cpp:530) */
  double cutting_distance;
} mf_cut_params;

/* parameters that reproduce setup_ref_cut(ny, grid, rake, clear, chamfer, speed, feed) */
int mf_cut_params_reference(mf_cut_params *p, int ny, double rake, double clear, double chamfer,
                            double speed, double feed);
int mf_scene_cut(const mf_cut_params *p, mf_scene **out);
int mf_scene_setup_ref_cut(int ny, double rake, double clear, double chamfer, double speed, double feed,
                           mf_scene **out);
/* the reference's two validation scenes, SI units, no tool (num_seg 0), no thermal constants:
   setup_rings(nbox) (benchmarks.cpp:161-253): two rubber-like rings (inner radius 0.03, outer
   0.04) moving at +-200 toward each other, locked box (-0.2, -0.08) .. (0.2, 0.08), no
   plasticity; setup_impact(nbox) (benchmarks.cpp:23-159): a steel disc (radius 0.2) at 1000
   against a wall of nbox/2 columns fixed at top and bottom, Johnson-Cook plasticity, an
   adaptive Green grid of at most 10 N cells. nbox >= 2 lattice points across the outer
   diameter; a lattice that puts no particle in the body is refused (MF_ERR_INVALID). */
int mf_scene_setup_rings(int nbox, mf_scene **out);
int mf_scene_setup_impact(int nbox, mf_scene **out);
int mf_scene_free(mf_scene *scene);
/* particles + grid (locked box, or adaptive when grid_max_cell > 0) + constants + tool + dt
   from a scene */
int mf_scene_upload(mf_ctx *ctx, const mf_scene *scene, int grid_kind);

/* ---- host tool geometry (tool.cpp): the (tl, length, height, rake, clear, r, mu) constructor,
   sample_tool (tool.cpp:121-144) and update_tool (tool.cpp:211-221) ---- */
int mf_tool_construct(double tl_x, double tl_y, double length, double height, double rake, double clear,
                      double r, double mu, mf_tool_state *out);
int mf_tool_sample(const mf_tool_state *tool, double dx, double *xy_out, int capacity, int *n_out);
int mf_tool_translate(mf_tool_state *tool, double dt); /* tool::update_tool with tool->vel */

/* ---- checkpoint / resume (no counterpart in the reference, whose state lives only on the
   device): the complete particle state in its current array order (every per-particle field,
   the cell hash of blanked particles included), the rigid tool and the step count, in a binary
   file with a format tag, the particle count and an FNV-1a checksum over everything before it.
   mf_state_load needs a context set up with the same particle count (the scene's constants,
   grid, options and dt are not part of the state) and refuses a file that fails any check
   (MF_ERR_CORRUPT) without changing the context. ---- */
int mf_state_save(mf_ctx *ctx, const char *path);
int mf_state_load(mf_ctx *ctx, const char *path);

/* ---- fields to and from device memory (caller's pointers, no host round trip): the copy is
   queued on `cuda_stream` (the context's stream when null) after the context's pending work,
   and the context's later work waits for it; layout as mf_get_field / mf_set_field ---- */
int mf_get_field_device(mf_ctx *ctx, int field, void *device_dst, void *cuda_stream);
int mf_set_field_device(mf_ctx *ctx, int field, const void *device_src, void *cuda_stream);

/* ---- tool wear: tool_wear::eval_usui (tool_wear.cu:20-64) on the device, from the current
   state and the tool's velocity; out3 = min, max, mean of the Usui wear rate
   K exp(alpha/T) p |v_r| over the particles in contact. The accumulated wear of the reference
   (m_accum_wear += dt * mean) is the caller's sum. ---- */
int mf_tool_wear_usui(mf_ctx *ctx, double K, double alpha, double out3[3]);

/* ---- output: vtk_writer_write (vtk_writer.cpp:20-178, 185-264), legacy ASCII ---- */
int mf_vtk_write_particles(mf_ctx *ctx, const char *path);
/* the same file from host arrays (layouts as mf_get_field; fixed, blanked, tool_p 0/1), e.g.
   for a state read back from a checkpoint; no device needed */
int mf_vtk_write_particle_arrays(const char *path, int n, const double *pos, const double *vel, const double *rho,
                                 const double *p, const double *T, const double *eps_pl, const double *S,
                                 const double *fixed, const double *blanked, const double *tool_p);
/* the same file, written while the steps go on (no counterpart in the reference): the fields
   are snapshotted inside the device, stream-ordered after the last step, copied to pinned host
   memory on a side stream and written by a host thread; mf_vtk_flush waits for every pending
   dump and returns the first error (mf_ctx_destroy flushes too) */
int mf_vtk_write_particles_async(mf_ctx *ctx, const char *path);
int mf_vtk_flush(mf_ctx *ctx);
int mf_vtk_write_tool(const mf_tool_state *tool, const char *path);

/* ---- graphs and the batched form (no counterpart in the reference) ----
   mf_graph_capture: n_steps (even, so that the double buffer returns to its parity) of the
   context captured into a cudaGraph_t (returned as void*; the caller owns and destroys it).
   It may be launched on any stream, also as a child of the caller's own graph; it stays
   valid until the context's buffers, constants, options, dt or flags change, and the steps it
   runs are counted on the device (mf_force_log) but not in mf_status.steps.
   mf_batch_*: many contexts on one device advanced together by one graph launch of
   steps_per_launch steps, so that small instances run side by side instead of each
   underfilling the GPU. Where every context steps a locked grid without neighbour lists and
   all share the precision, heat solver, yield law and plasticity setting, each step of the
   graph is one launch per phase (cell scan, scatter, reorder + predictor, pair sums, finish,
   return map) over all instances: their constants and buffers are entries of a device array
   (the reference keeps them in __constant__ memory, actions_gpu.cu:438-469,
   interactions_gpu.cu:423-459, tool_gpu.cu:20-27, one system per process) and every block
   finds its instance; each instance's results equal its own context's steps bit for bit.
   Otherwise the graph holds one child graph per context, with no edges between them.
   steps_per_launch = 0 lets the batch tune itself over a few launches, which advance the
   instances: the block size of the batched pair kernel (64, 128 or 256 threads) and the steps
   per launch (2, 4, 8 or 16), by the highest measured throughput; mf_batch_config reports the
   choice (fused: 1 for the batched kernels). After a host write to an instance its
   cell counts are re-primed before the next launch; after a change that invalidates its
   graphs (buffers, constants, options, dt, flags) mf_batch_step returns MF_ERR_STATE and the
   batch must be rebuilt. */
typedef struct mf_batch mf_batch;
int mf_graph_capture(mf_ctx *ctx, int n_steps, void **cuda_graph);
int mf_graph_destroy(void *cuda_graph);
int mf_batch_create(mf_ctx **ctxs, int n, int steps_per_launch, mf_batch **out);
int mf_batch_steps_per_launch(const mf_batch *batch, int *steps_per_launch);
int mf_batch_config(const mf_batch *batch, int *fused, int *pair_block, int *steps_per_launch);
int mf_batch_step(mf_batch *batch, int n_launches); /* n_launches x steps_per_launch steps each */
/* Launch form of a batch on the batched kernels. MF_BATCH_PHASES: each step one launch per
   phase, as above. MF_BATCH_PERSISTENT: the K steps of a launch run inside ONE cooperative
   launch (captured in the batch's graph) of blocks_per_sm 256-thread blocks per SM (0: as many
   as are resident); its blocks take each phase's blocks of all instances in turn and meet at a
   grid-wide barrier between phases, every instance's results still equal to its own context's
   bit for bit. Each barrier wait is bounded (mf_batch_set_wait_limit, seconds in [0, 3600],
   default 2 s; 0 makes the first wait give up at once): if one expires, that barrier releases no
   block, the launch ends early with the instances' states part-stepped, and every instance's
   mf_status.error_flags gets bit 3.
   The persistent form steps mixed-precision batches only (an FP64 build of it contracted the
   pair sums' multiply-adds differently, ~1e-16 relative off the single-system step).
   mf_batch_set_form rebuilds the batch's graph (MF_ERR_INVALID for a child-graph or FP64 batch
   in the persistent form, an odd or < 2 steps_per_launch); the tuner of steps_per_launch = 0
   also measures the persistent form of a mixed batch (1 and 2 blocks per SM, 4 and 16 steps
   per launch) and keeps the fastest form. ---- */
#define MF_BATCH_PHASES 0
#define MF_BATCH_PERSISTENT 1
int mf_batch_set_form(mf_batch *batch, int form, int blocks_per_sm, int steps_per_launch);
int mf_batch_form(const mf_batch *batch, int *form, int *blocks_per_sm);
int mf_batch_set_wait_limit(mf_batch *batch, double seconds);
int mf_batch_destroy(mf_batch *batch);

/* ---- differentiable form (no counterpart in the reference): from the context's current
   state, runs skip_steps + window_steps FP64 steps on dual numbers and returns the mean over
   the window of the tool force (report_force, output.cu:31-39: [0] cutting Fc, [1] feed Ff)
   and, for param 0..5 = Johnson-Cook A, B, n, C, m or the friction coefficient mu, its
   derivative with respect to that parameter (forward-mode tangents through every step; param
   -1: the mean only). The context's state is not changed. Locked Green grid, Brookshaw or no
   conduction, Johnson-Cook law only (MF_ERR_INVALID otherwise). ---- */
int mf_tangent_mean_force(mf_ctx *ctx, int skip_steps, int window_steps, int param, double out_mean[2],
                          double out_dmean[2]);
/* the same for all six parameters in one pass (six tangent directions carried together):
   out_dmean[2k], out_dmean[2k + 1] = d(mean Fc), d(mean Ff) with respect to parameter k =
   A, B, n, C, m, mu; each equals what mf_tangent_mean_force returns for param k. */
int mf_tangent_mean_force_all(mf_ctx *ctx, int skip_steps, int window_steps, double out_mean[2],
                              double out_dmean[12]);

#ifdef __cplusplus
}
#endif
#endif
