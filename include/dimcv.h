/*
 * dimcv.h — C ABI of the B200 DIMCV-SPH substep library (libdimcv.so).
 *
 * The reference (Haok-Z/DIMCV-SPH) is Python + Taichi: every operator below
 * replaces one or more `@ti.kernel`s that the reference's Python classes
 * `ParticleSystem` (particle_system.py), `SPHBase` (sph_base.py) and
 * `DIMCVSPHSolver` (dimcv_sph.py) launch.  The reference has no FFI of its
 * own; each declaration cites the reference method whose behaviour it takes
 * over, and the Python operator shim in dimcv_sph_b200/ binds these entry
 * points with ctypes under the reference's method names.
 *
 * Conventions
 *  - Plain pointers and sizes only.  Every `float*`/`int32_t*`/`uint8_t*`
 *    inside dv_fields / dv_solver_fields is a DEVICE pointer allocated by the
 *    caller at `capacity` particles (the reference's `particle_max_num`).
 *  - Vector fields are array-of-vectors with a padded stride: position-like
 *    fields (x, x_0, v, acceleration, v_star, x_temp) use DV_VSTRIDE(dim)
 *    floats per particle (2 in 2D, 4 in 3D; the 4th float is padding), and
 *    3-vector fields (vorticity, d_vort, d_vort_smoothed, vorticity_vis,
 *    v_vort) always use 4 floats.  grad_v uses dim*dim floats, row-major.
 *  - Calls are asynchronous on the context's stream and ordered; none
 *    allocates device memory (workspace is sized once by dv_create).  Calls
 *    that return a host value say so and synchronise the stream.
 *  - Return value: DV_OK (0) or a negative dv_status; dv_last_error() holds
 *    the message.  Warnings raised on the device (iteration cap reached, a
 *    position outside the cell grid, capacity clamp) accumulate in
 *    dv_counters.status as DV_WARN_* bits; they do not fail a call.
 *  - Particle count: the exact count lives on the device (dv_counters.n);
 *    the host passes nothing per call, kernels are sized by the context's
 *    upper bound (capacity-limited) and read the exact count on the device.
 *  - A context is not thread-safe; use one per host thread / stream.
 */
#ifndef DIMCV_H_
#define DIMCV_H_

#include <stdint.h>

#ifdef __cplusplus
#define DV_EXTERN_C extern "C"
#else
#define DV_EXTERN_C
#endif
#define DV_API DV_EXTERN_C __attribute__((visibility("default")))

#define DV_VSTRIDE(dim) ((dim) == 2 ? 2 : 4)

/* material codes (particle_system.py:37-38) */
#define DV_MATERIAL_SOLID 0
#define DV_MATERIAL_FLUID 1

enum dv_status {
  DV_OK = 0,
  DV_EINVAL = -1,      /* bad argument */
  DV_ECAPACITY = -2,   /* a size exceeds the context's capacity */
  DV_ECUDA = -3,       /* a CUDA runtime call failed */
  DV_ENAN = -4,        /* a non-finite value was found where one is fatal */
  DV_EUNSUPPORTED = -5 /* option not built into this library */
};

/* device-raised warning bits in dv_counters.status */
#define DV_WARN_DIV_NOT_CONVERGED (1 << 0) /* divergence solve hit max_iter (dimcv_sph.py:385) */
#define DV_WARN_P_NOT_CONVERGED (1 << 1)   /* pressure solve hit max_iter (dimcv_sph.py:608) */
#define DV_WARN_OUTSIDE_GRID (1 << 2)      /* a cell index fell outside [0, grid_num): clamped */
#define DV_WARN_CAPACITY (1 << 3)          /* emission clamped at capacity (particle_system.py:361) */
#define DV_WARN_NAN (1 << 4)               /* a non-finite error norm was seen in a solve */
#define DV_WARN_BAD_INDEX (1 << 5)         /* an injected sample index was outside [0, n): ignored */

/* Sampling modes of dv_sample (new: the reference only has the Bernoulli
 * birth/death process of dimcv_sph.py:305-335). */
#define DV_SAMPLE_BERNOULLI 0 /* reference KVN birth/death + compaction */
#define DV_SAMPLE_INVERSE_CDF 1 /* M i.i.d. draws from p ∝ kden (FP64 CDF) */
#define DV_SAMPLE_INJECTED 2    /* caller supplies sample_idx / num_samples */
#define DV_SAMPLE_STRATIFIED 3  /* M stratified draws u_s = (s + ξ_s)/M through the same CDF */

/* Velocity kernels for the VVPE / Biot-Savart sums. */
#define DV_KERNEL_REF2D 0 /* reference: 0.1592 V Kε(|r|) (r_xy × ω), dimcv_sph.py:649-719 */
#define DV_KERNEL_BLOB3D 1 /* 3-D regularised blob (1/4π) V (r × ω)/(|r|²+δ²)^{3/2} (segment_solver.py:378-417 form) */

/*
 * Scalar parameters.  Every derived f32 constant is computed by the caller
 * in float64 from the reference's own Python expressions and rounded once
 * (that is how Taichi folds Python-scope constants into f32 kernels), so the
 * CUDA kernels and the CPU oracle consume identical bits.
 */
typedef struct dv_params {
  int32_t dim;                /* 2 or 3 (particle_system.py:26) */
  int32_t grid_num[3];        /* ceil(domain_size / h), float64 (particle_system.py:54) */
  float domain_start[3];      /* particle_system.py:17 */
  float domain_end[3];        /* particle_system.py:20 */
  float grid_size;            /* f32(h): pos_to_index divides by it (particle_system.py:383) */
  float support_radius;       /* f32(h) = 4 r (particle_system.py:44) */
  float inv_support_radius;   /* f32(1/h) (particle_system.py:45) */
  float nbr_r2_limit;         /* smallest f32 t with sqrtf(t) >= h: j is a neighbour iff r2 < t (particle_system.py:584) */
  float far_r2_limit;         /* largest f32 t with sqrtf(t) <= h: sample is far iff r2 > t (dimcv_sph.py:700) */
  float kW;                   /* f32(k_d h^-d) cubic W scale (sph_base.py:28-35) */
  float kW2;                  /* f32(2 k_d h^-d) (sph_base.py:43) */
  float kG;                   /* f32(6 k_d h^-d) ∇W scale (sph_base.py:50-57) */
  float grad_r_min;           /* 1e-5: ∇W is zero for |r| <= this (sph_base.py:61) */
  float density0;             /* sph_base.py:17 */
  float dt;                   /* f32 time step (dimcv_sph.py:13) */
  float inv_dt;               /* f32(1/dt) (dimcv_sph.py:27) */
  float inv_dt2;              /* f32(1/dt²) (dimcv_sph.py:28) */
  float gravity[3];           /* sph_base.py:12 */
  float visc_coef;            /* f32(2(d+2) ν) (dimcv_sph.py:170,177) */
  float visc_h2;              /* f32(0.01 h²) (dimcv_sph.py:178) */
  float m_eps;                /* 1e-5 Jacobi pair threshold (dimcv_sph.py:24) */
  float factor_min;           /* 1e-6 DFSPH factor threshold (dimcv_sph.py:102) */
  double eta_div;             /* inv_dt·max_error_V·0.01·ρ0 (dimcv_sph.py:389) */
  double eta_p;               /* max_error·0.01·ρ0 (dimcv_sph.py:611) */
  int32_t max_iter_div;       /* 100 (dimcv_sph.py:22) */
  int32_t max_iter_p;         /* 100 (dimcv_sph.py:23) */
  int32_t neighbor_min;       /* 20 in 3D, 7 in 2D (dimcv_sph.py:351-356) */
  int32_t has_transit;        /* divergenceTransitArea given (dimcv_sph.py:401-405) */
  float transit_a0;           /* f32(area[0]) */
  float transit_span;         /* f32(area[1] - area[0]) */
  int32_t has_vortex_domain;  /* vortexEnforcingDomainStart given (dimcv_sph.py:77-84) */
  float vd_start[3];
  float vd_end[3];
  float vvpe_coef;            /* f32(0.1592 · vp_volume) (dimcv_sph.py:691) */
  float eps;                  /* 1e-6 (dimcv_sph.py:15) */
  float inv_eps;              /* f32(1/eps) (dimcv_sph.py:16) */
  float gen_a;                /* GenProbPara (dimcv_sph.py:58) */
  float del_b;                /* DelProbPara (dimcv_sph.py:59) */
  float kden_eps;             /* 1e-8 (dimcv_sph.py:709) */
  float kvn_eps;              /* 1e-8 (dimcv_sph.py:316) */
  /* options that have no reference counterpart (defaults = reference) */
  int32_t skip_cell0;         /* 1: flat cell 0 is never visited (particle_system.py:581-583 quirk) */
  int32_t cell_origin_offset; /* 0: cell = int(x/h) (reference); 1: cell = int((x - domain_start)/h) */
  int32_t kernel_mode;        /* DV_KERNEL_* for VVPE and full BS */
  float blob_delta2;          /* δ² of DV_KERNEL_BLOB3D */
  float blob_coef;            /* f32(V / 4π) of DV_KERNEL_BLOB3D */
  int32_t compensated;        /* 1: compensated (Kahan) f32 accumulation in the N-body sums */
  /* periodic box (new): every axis wraps with period box[d] = domain_end - domain_start;
   * needs cell_origin_offset = 1, grid_size = box[d] / grid_num[d] on every axis
   * (cells at least h wide) and grid_num[d] >= 3; distances use the minimum image */
  int32_t periodic;
  float box[3];
  /* scene batch (new): n_scenes > 1 reserves the top bits of the cell key for
   * a scene id (dv_batch_*); grid_num is then the largest scene grid */
  int32_t n_scenes;
  int32_t reserved[3];
} dv_params;

/* Fields that travel with a particle: dv_grid_build permutes them
 * (particle_system.py:429-553).  `color` is 4 int32 per particle (3 used). */
typedef struct dv_fields {
  float *x, *x0, *v, *acceleration;  /* DV_VSTRIDE(dim) floats each */
  float *vorticity;                  /* 4 floats */
  float *m_V, *m, *density, *pressure, *dfsph_factor, *density_adv, *life_time;
  int32_t *material, *object_id, *color, *grid_ids;
  uint8_t *is_dynamic, *is_active, *is_sample;
} dv_fields;

/* Solver fields indexed by slot, NOT permuted by the grid build — the
 * reference keeps them on DIMCVSPHSolver / vis buffers and never reorders
 * them (dimcv_sph.py:30-53, particle_system.py:167), so a slot that is not
 * rewritten in a step keeps the previous occupant's value.  The caller
 * zero-initialises them once. */
typedef struct dv_solver_fields {
  float *v_star;          /* DV_VSTRIDE(dim) */
  float *grad_v;          /* dim*dim, row-major */
  float *d_vort;          /* 4 */
  float *d_vort_smoothed; /* 4 */
  float *kvn;             /* kinematic_vort_num */
  float *kden;            /* kernel_density */
  float *x_temp;          /* DV_VSTRIDE(dim) */
  float *vorticity_vis;   /* 4 */
  float *v_vort;          /* 4, optional (may be NULL): VVPE increment before the gate */
  int32_t *sample_idx;    /* capacity */
} dv_solver_fields;

/* Device-side counters, mirrored to the host by dv_get_counters. */
typedef struct dv_counters {
  int32_t n;            /* particle_num */
  int32_t n_fluid;      /* fluid_particle_num */
  int32_t n_solid;      /* solid_particle_num */
  int32_t num_samples;  /* num_samples */
  int32_t iters_div;    /* last divergence-solve iteration count */
  int32_t iters_p;      /* last pressure-solve iteration count */
  int32_t status;       /* DV_WARN_* bits, sticky until dv_clear_status */
  int32_t n_targets;    /* VVPE targets (fluid in the vortex domain) in the last vort2vel */
  double err_div;       /* last divergence-solve average error */
  double err_p;         /* last pressure-solve average error */
  double kden_sum;      /* FP64 Σ kden (kden_sum field holds its f32 rounding) */
  float kden_sum_f32;
  int32_t pad;
} dv_counters;

typedef struct dv_ctx dv_ctx;

/* ---------------------------------------------------------------- lifetime */
/* Creates a context for `capacity` particles on the current CUDA device and
 * the given stream (cudaStream_t, NULL = legacy default).  Allocates all
 * workspace (sort buffers, cell table, reduction and sampling scratch).
 * Replaces the allocations of ParticleSystem.__init__ (particle_system.py:136-141)
 * and DIMCVSPHSolver.__init__ (dimcv_sph.py:30-53); field memory stays with
 * the caller.  Returns NULL on failure (message via dv_last_error(NULL)). */
DV_API dv_ctx* dv_create(const dv_params* params, int64_t capacity, void* stream);
/* Frees the context's workspace (the caller's fields are not touched). */
DV_API void dv_destroy(dv_ctx* ctx);
/* Message of the last failed call on ctx; with NULL, of the calling thread's
 * last failed dv_create or context-free call. */
DV_API const char* dv_last_error(const dv_ctx* ctx);
/* Later calls on ctx run on `stream` (cudaStream_t, NULL = legacy default). */
DV_API int dv_set_stream(dv_ctx* ctx, void* stream);
/* Replaces the scalar parameters (time step, tolerances, options) of a live
 * context.  The cell grid (dim, grid_num) must stay the same.  Stands in for
 * assignments to the reference's Python-side solver attributes such as
 * `solver.dt[None] = ...` (dimcv_sph.py:13). */
DV_API int dv_set_params(dv_ctx* ctx, const dv_params* params);
/* Library version string and the number of kernels launched so far by this
 * context (used by benchmarks to report launch counts). */
DV_API const char* dv_version(void);
DV_API int64_t dv_launch_count(const dv_ctx* ctx);

/* Host view of the device counters (synchronises the stream). */
DV_API int dv_get_counters(dv_ctx* ctx, dv_counters* out);
/* Sets n / n_fluid / n_solid (after the caller filled fields on its own). */
DV_API int dv_set_counts(dv_ctx* ctx, int32_t n, int32_t n_fluid, int32_t n_solid);
/* Clears the sticky DV_WARN_* bits of dv_counters.status. */
DV_API int dv_clear_status(dv_ctx* ctx);

/* --------------------------------------------------------------- particles */
/* Appends `count` particles at slots [n, n+count) clamped at capacity, as
 * ParticleSystem._add_particles / add_particle (particle_system.py:317-380).
 * pos/vel: device arrays of count*dim floats (dense rows).  Fields not set by
 * the reference's add_particle are zeroed (acceleration, vorticity,
 * dfsph_factor, density_adv, is_sample, life_time).  Asynchronous. */
DV_API int dv_add_particles(dv_ctx* ctx, const dv_fields* f, const float* pos, const float* vel,
                            int32_t count, int32_t object_id, float density, float pressure,
                            int32_t material, int32_t is_dynamic, int32_t color_r,
                            int32_t color_g, int32_t color_b, float m_V0);

/* ParticleSystem.update_activity (particle_system.py:413-427). */
DV_API int dv_update_activity(dv_ctx* ctx, const dv_fields* f);

/* ParticleSystem.particle_partition + update_grid_id + prefix sum +
 * counting_sort (particle_system.py:429-560) in one call: active particles
 * are stably sorted by Morton cell key (an LSD radix sort built from
 * atomic-free counting passes) and every dv_fields array is gathered from
 * `src` into `dst` (which must not alias `src`).  Slots past the new count
 * get the reference's partition fill values.  The cell table used by every
 * neighbour sweep is rebuilt.  Call dv_update_activity first. */
DV_API int dv_grid_build(dv_ctx* ctx, const dv_fields* src, const dv_fields* dst);
/* Reads back the permutation of the last dv_grid_build: perm[p] = the src
 * slot now at p (host pointer, n_cap entries; synchronises). */
DV_API int dv_get_permutation(dv_ctx* ctx, int32_t* host_perm, int64_t n_cap);

/* Neighbour lists in CSR form, for tests and tooling: for each particle p
 * (in the current order) the slots q that ParticleSystem.for_all_neighbors
 * (particle_system.py:562-586) visits, in visit order.  offsets: n+1 int64,
 * nbrs: up to max_pairs int32 (device pointers; either may be NULL — call
 * with nbrs = NULL first to learn the pair count).  Returns the pair count
 * or a negative dv_status (DV_ECAPACITY if max_pairs is too small).
 * Synchronises. */
DV_API int64_t dv_neighbor_lists(dv_ctx* ctx, const dv_fields* f, int64_t* offsets,
                                 int32_t* nbrs, int64_t max_pairs);
/* New (checking): the neighbour lists the sweeps read, as the last grid build
 * (dv_grid_build) stored them: CSR offsets (n+1 uint32) and entries in visit
 * order, copied into device buffers.  Rows of static solids are empty: no
 * sweep of the step walks them (dv_neighbor_lists has every row).  Either
 * buffer may be NULL; call with
 * nbrs = NULL first to learn the entry count).  Returns the entry count, or a
 * negative dv_status: DV_EINVAL when no valid lists are stored (positions
 * or the particle count changed since the build, or they did not fit),
 * DV_ECAPACITY when max_entries is too small.  Synchronises. */
DV_API int64_t dv_stored_lists(dv_ctx* ctx, uint32_t* offsets, int32_t* nbrs, int64_t max_entries);

/* ------------------------------------------------------------ SPH / DFSPH */
/* SPHBase.compute_static_boundary_volume (sph_base.py:91-103). */
DV_API int dv_boundary_volume(dv_ctx* ctx, const dv_fields* f);
/* compute_moving_boundary_volume (sph_base.py:105-112): the same volume for
 * the dynamic solids, once per step. */
DV_API int dv_moving_boundary_volume(dv_ctx* ctx, const dv_fields* f);
/* New (switch): the scene has dynamic rigid particles.  While on, every
 * pressure iteration (dv_pressure_iteration, dv_pressure_solve) also forms
 * the reaction on them (dimcv_sph.py:540-549), gathered per solid in its
 * neighbour order instead of the reference's unordered atomic adds.  Not
 * available in a scene batch. */
DV_API int dv_set_dynamic_rigid(dv_ctx* ctx, int32_t on);
/* DIMCVSPHSolver.compute_densities (dimcv_sph.py:126-148). */
DV_API int dv_densities(dv_ctx* ctx, const dv_fields* f);
/* DIMCVSPHSolver.compute_DFSPH_factor (dimcv_sph.py:86-124). */
DV_API int dv_dfsph_factor(dv_ctx* ctx, const dv_fields* f);
/* compute_densities followed by compute_DFSPH_factor (dimcv_sph.py:86-148)
 * in one neighbour sweep: both fields bit-identical to dv_densities then
 * dv_dfsph_factor. */
DV_API int dv_densities_factor(dv_ctx* ctx, const dv_fields* f);
/* dv_densities_factor and, in the same neighbour sweep, the
 * compute_density_change that opens divergence_solve (dimcv_sph.py:337-374,
 * :377): density_adv bit-identical to dv_density_change's.  It reads v, x
 * and m_V, which the two sweeps do not write; follow it with
 * dv_divergence_solve_prepared while those are unchanged. */
DV_API int dv_densities_factor_change(dv_ctx* ctx, const dv_fields* f);
/* DIMCVSPHSolver.multiply_time_step(dfsph_factor, s) (dimcv_sph.py:395-399). */
DV_API int dv_scale_factor(dv_ctx* ctx, const dv_fields* f, float s);
/* DIMCVSPHSolver.compute_density_change (dimcv_sph.py:337-374). */
DV_API int dv_density_change(dv_ctx* ctx, const dv_fields* f);
/* DIMCVSPHSolver.compute_density_adv (dimcv_sph.py:470-493). */
DV_API int dv_density_adv(dv_ctx* ctx, const dv_fields* f);
/* DIMCVSPHSolver.compute_density_error(offset) (dimcv_sph.py:407-419):
 * returns the FP64 sum through *out (synchronises). */
DV_API int dv_density_error(dv_ctx* ctx, const dv_fields* f, float offset, double* out);
/* One divergence_solver_iteration_kernel (dimcv_sph.py:421-468). */
DV_API int dv_divergence_iteration(dv_ctx* ctx, const dv_fields* f);
/* One pressure_solve_iteration_kernel (dimcv_sph.py:495-549). */
DV_API int dv_pressure_iteration(dv_ctx* ctx, const dv_fields* f);
/* DIMCVSPHSolver.divergence_solve (dimcv_sph.py:376-393): density change,
 * factor·1/dt, Jacobi iterations until avg error <= eta_div or max_iter,
 * factor·dt.  The loop runs on the device (early-exit flag), polled by the
 * host once per chunk of iterations.  *iters (host, may be NULL) receives
 * the iteration count (synchronises only if non-NULL). */
DV_API int dv_divergence_solve(dv_ctx* ctx, const dv_fields* f, int32_t* iters);
/* dv_divergence_solve without its opening density change: density_adv must
 * hold compute_density_change's result for the current v (from
 * dv_densities_factor_change or dv_density_change). */
DV_API int dv_divergence_solve_prepared(dv_ctx* ctx, const dv_fields* f, int32_t* iters);
/* dv_divergence_solve with options (flags, OR-ed):
 *   DV_SOLVE_PREPARED: as dv_divergence_solve_prepared;
 *   DV_SOLVE_NONPRESSURE: the Jacobi loop's residual sweeps also compute
 *     compute_non_pressure_forces (dimcv_sph.py:150-208, which the substep
 *     calls next, karman_vortex.py:236); afterwards acceleration is
 *     bit-identical to dv_nonpressure on the solved velocity. */
#define DV_SOLVE_PREPARED 1
#define DV_SOLVE_NONPRESSURE 2
DV_API int dv_divergence_solve_ex(dv_ctx* ctx, const dv_fields* f, int32_t flags, int32_t* iters);
/* DIMCVSPHSolver.pressure_solve (dimcv_sph.py:597-614), same loop form. */
DV_API int dv_pressure_solve(dv_ctx* ctx, const dv_fields* f, int32_t* iters);
/* dv_pressure_solve with options (flags):
 *   DV_SOLVE_VIS: the solve's opening density_adv sweep also does
 *     copy_x_temp + compute_vorticity_vis (dimcv_sph.py:778-801, which the
 *     substep calls after the solve, karman_vortex.py:240-241) into s's
 *     x_temp and vorticity_vis, bit-identical to dv_vis after the solve (the
 *     iterations write only v, which the vis sweep does not read). */
#define DV_SOLVE_VIS 4
DV_API int dv_pressure_solve_ex(dv_ctx* ctx, const dv_fields* f, const dv_solver_fields* s, int32_t flags,
                                int32_t* iters);
/* DIMCVSPHSolver.compute_non_pressure_forces (dimcv_sph.py:150-208). */
DV_API int dv_nonpressure(dv_ctx* ctx, const dv_fields* f);
/* DIMCVSPHSolver.predict_velocity (dimcv_sph.py:220-226). */
DV_API int dv_predict_velocity(dv_ctx* ctx, const dv_fields* f);
/* DIMCVSPHSolver.advect (dimcv_sph.py:210-218). */
DV_API int dv_advect(dv_ctx* ctx, const dv_fields* f);
/* enforce_boundary_2D / _3D with simulate_collisions (sph_base.py:118-179),
 * the bounceBackBoundary option of karman_vortex.py:226-230: every slot of the
 * capacity with this material that is dynamic is clamped into [lo, hi] per
 * axis (dim floats each; host pointers) and its velocity loses 1.5x its
 * component along the normalised clamp normal. */
DV_API int dv_enforce_boundary(dv_ctx* ctx, const dv_fields* f, int32_t material, const float* lo,
                               const float* hi);

/* --------------------------------------------------------------- DIMCV */
/* compute_v_star + compute_vorticity + compute_grad_v (dimcv_sph.py:228-293,
 * `init` at :803-806) fused into one neighbour sweep. */
DV_API int dv_dimcv_vorticity(dv_ctx* ctx, const dv_fields* f, const dv_solver_fields* s);
/* compute_d_vorticity (dimcv_sph.py:551-583). */
DV_API int dv_d_vorticity(dv_ctx* ctx, const dv_fields* f, const dv_solver_fields* s);
/* dv_dimcv_vorticity followed by dv_d_vorticity (dimcv_sph.py:228-293,
 * 551-583) in one neighbour sweep, v*_j formed per neighbour: v_star,
 * vorticity, grad_v and d_vort bit-identical to the two calls. */
DV_API int dv_vorticity_dvort(dv_ctx* ctx, const dv_fields* f, const dv_solver_fields* s);
/* compute_all_d_vort_smoothed (dimcv_sph.py:660-677). */
DV_API int dv_smooth_d_vort(dv_ctx* ctx, const dv_fields* f, const dv_solver_fields* s);
/* compute_kinematic_vorticity_num_sample (dimcv_sph.py:295-324): KVN and
 * the Bernoulli birth/death of is_sample with a Philox-4x32-10 counter RNG
 * keyed by (seed, step, slot) in place of the time-seeded ti.random.
 * birth_death = 0 computes KVN only (the inverse-CDF sampling mode). */
DV_API int dv_kvn_sample(dv_ctx* ctx, const dv_fields* f, const dv_solver_fields* s,
                         uint64_t seed, uint64_t step, int32_t birth_death);
/* record_vort_part_sample_idx (dimcv_sph.py:326-335): deterministic stable
 * compaction of is_sample into sample_idx (ascending slot). */
DV_API int dv_record_samples(dv_ctx* ctx, const dv_fields* f, const dv_solver_fields* s);
/* compute_kernel_density (dimcv_sph.py:721-751); kden_sum is reduced in FP64. */
DV_API int dv_akde(dv_ctx* ctx, const dv_fields* f, const dv_solver_fields* s);
/* compute_all_d_vort_smoothed and compute_kernel_density (dimcv_sph.py:
 * 660-677, 721-751) in one neighbour sweep: d_vort_smoothed, kden and
 * kden_sum bit-identical to dv_smooth_d_vort then dv_akde.  Needs the KVN of
 * this step (dv_kvn_sample first; the smoothing does not depend on it). */
DV_API int dv_smooth_akde(dv_ctx* ctx, const dv_fields* f, const dv_solver_fields* s);
/* New (no reference counterpart): FP64 CDF of kden over the VVPE targets
 * and M i.i.d. inverse-CDF draws (Philox keyed by seed, step, draw) into
 * sample_idx; or, for DV_SAMPLE_INJECTED, adopt num_samples = M with
 * sample_idx already filled by the caller. */
DV_API int dv_sample(dv_ctx* ctx, const dv_fields* f, const dv_solver_fields* s, int32_t mode,
                     uint64_t seed, uint64_t step, int32_t M);
/* vort2vel (dimcv_sph.py:649-719): near-field neighbour sum, Monte-Carlo
 * far field over sample_idx[0:num_samples], the ‖v_vort‖ < ‖v‖ gate. */
DV_API int dv_vvpe_mc(dv_ctx* ctx, const dv_fields* f, const dv_solver_fields* s);
/* New (tuning): times the far-field main loop of dv_vvpe_mc for 2, 4, 6 and 8
 * targets per thread (6 runs as 8 where the loop is not the paired one) and
 * 1-8 sample chunks on the current targets / samples and keeps the fastest
 * for this context (synchronises; *best_tt / *best_ms may be NULL).
 * dv_set_far_tile sets the tile directly (2, 4, 6 or 8). */
DV_API int dv_autotune(dv_ctx* ctx, const dv_fields* f, const dv_solver_fields* s, int32_t* best_tt,
                       float* best_ms);
DV_API int dv_set_far_tile(dv_ctx* ctx, int32_t tt);
/* update_particle_life_time (dimcv_sph.py:753-760). */
DV_API int dv_life_time(dv_ctx* ctx, const dv_fields* f);
/* copy_x_temp + compute_vorticity_vis (dimcv_sph.py:778-801). */
DV_API int dv_vis(dv_ctx* ctx, const dv_fields* f, const dv_solver_fields* s);

/* New: full O(N²) Biot-Savart velocity with the same kernel as the VVPE.
 * Targets: slots targets[0:nt) (device int32, or NULL for 0..nt-1); sources:
 * every slot in [0, n) with material fluid, weights omega (4-stride, device).
 * out: nt×4 floats (precision 32) or nt×4 doubles (precision 64), device. */
DV_API int dv_bs_full(dv_ctx* ctx, const dv_fields* f, const float* omega, const int32_t* targets,
                      int32_t nt, void* out, int32_t precision);

/* Kernel timing of the Monte-Carlo far-field kernel (the FP32-bound hot
 * loop of dv_vvpe_mc): when enabled, CUDA events bracket every far-field
 * launch on the context stream and a device counter accumulates the pair
 * count n_targets × num_samples.  dv_profile resets; dv_profile_read
 * synchronises and returns the totals since the reset. */
DV_API int dv_profile(dv_ctx* ctx, int32_t enable);
DV_API int dv_profile_read(dv_ctx* ctx, double* far_ms, int64_t* launches, double* pairs);

/* Allocation-free FP64 density error, for callers that cannot allocate
 * device memory: real-time step loops that forbid allocation after
 * start-up, and hosts whose own allocator owns all device memory (a pool
 * that reserved the GPU, or an embedding application that hands this
 * library only device pointers).  No counterpart in the reference; it
 * computes what dv_density_error computes (the reference's
 * compute_density_error sum, in FP64) without a context: no dv_create, no
 * cudaMalloc / cudaFree.  Its scratch is a 512 KB file-scope __device__
 * array that every GPU loading the library keeps until exit.  Limit: n <=
 * 16,777,216 particles (larger n returns DV_ECAPACITY).  Each call looks up
 * the array's device address on the current device (cudaGetSymbolAddress),
 * so the address stays right after a device reset.  The call copies the
 * sum to the host and synchronises `stream`, so it cannot be made on a
 * stream that is being captured into a CUDA graph: it avoids allocation,
 * nothing more.  All calls share the array: calls that overlap on the GPU
 * race.  Fields are device pointers of slots [0, n); *out (host) receives
 * the sum.  Errors: negative dv_status, message via dv_last_error(NULL). */
DV_API int dv_density_error_noalloc(const dv_params* params, const dv_fields* f, int32_t n,
                                    float offset, double* out, void* stream);

/* Measured FP32 FMA throughput of this GPU (FLOP/s, an FMA counts 2): runs a
 * short register-resident FMA chain kernel; used as the roofline peak of the
 * FP32-pipe-bound N-body kernels.  Synchronises. */
DV_API int dv_fp32_peak(dv_ctx* ctx, double* flops_out);

/* Number of sample chunks of the far-field grid (1..8; dv_autotune picks it
 * with the tile): the main loop runs (target tiles x sample chunks) blocks
 * and the correction kernel sums the chunk partials in chunk order. */
DV_API int dv_set_far_chunks(dv_ctx* ctx, int32_t chunks);
DV_API int32_t dv_get_far_chunks(dv_ctx* ctx);

/* ------------------------------------------------------------------------
 * Differentiable vortex-particle step (2-D).  No reference counterpart: the
 * reference has no derivatives.  The step is the SPH vorticity smoothing
 * (dimcv_sph.py:660-677) followed by the Monte-Carlo Biot-Savart velocity
 * (dimcv_sph.py:649-719) without the gate, on caller arrays in the sorted
 * slot order of a plan:
 *   ω̃_i = m_V_i W(0) ω_i + Σ_{j∈N(i)} m_V_j W(r_ij) ω_j
 *   u_i = Σ_{j∈N(i)} [c Kε(r_ij) − f_i a_j / r_ij²] ω̃_j r_ij⊥ + f_i Σ_s a_s ω̃_s r_is⊥ / r_is²
 * (r⊥ = (r_y, −r_x), c = 0.1592 vp_volume, a_s = multiplicity / (kden_s + 1e-8),
 * f_i = c (S − S_i) / (M − near samples of i)).  A plan freezes neighbour
 * lists, sources, weights and (with xbar) the periodic images, so the VJPs
 * are exact derivatives of the frozen step.  Arrays: x [n][2], ω [n],
 * u [n][2], of the call precision (32: float, 64: double).
 * ------------------------------------------------------------------------ */
#define DV_VPM_MC 0   /* sources = the current samples (dv_sample), MC weights */
#define DV_VPM_FULL 1 /* sources = every particle, a = 1, f = c: full Biot-Savart */

typedef struct dv_vpm_plan {
  int32_t n;         /* particles = targets, slots [0, n) */
  int32_t src_cap;   /* capacity of the source arrays (>= M; >= n for DV_VPM_FULL) */
  int64_t nbr_cap;   /* capacity of nbr */
  int32_t* n_src;    /* device scalar: number of sources, -1 if the build failed */
  int32_t* perm;     /* [n] slot -> index of the particle in the caller's order */
  int32_t* inv_perm; /* [n] caller index -> slot */
  int32_t* nbr_off;  /* [n+1] CSR offsets */
  int32_t* nbr;      /* [nbr_cap] neighbour slots, |r| < h */
  int32_t* src;      /* [src_cap] source slots, ascending */
  float* src_a;      /* [src_cap] a_s */
  int32_t* slot_src; /* [n] index in src, or -1 */
  float* slot_a;     /* [n] a_j (0 where j is no source) */
  float* f;          /* [n] far factor f_i */
  float* m_V;        /* [n] volumes */
  const void* xbar;  /* [n][2] nominal positions fixing the periodic image of every pair,
                        of the call precision; NULL: minimum image */
} dv_vpm_plan;

/* Bytes of the caller workspace of dv_vpm_velocity / dv_vpm_velocity_bwd. */
DV_API int64_t dv_vpm_workspace_bytes(dv_ctx* ctx, int32_t n, int32_t src_cap, int32_t precision);
/* Fill a plan from the state after dv_grid_build (neighbour lists, sort
 * permutation) and, for DV_VPM_MC, dv_akde + dv_sample.  Every particle must
 * be fluid (n == n_fluid).  Asynchronous; *n_src = -1 reports a failed
 * build (count mismatch, missing lists, capacity). */
DV_API int dv_vpm_plan_build(dv_ctx* ctx, const dv_fields* f, const dv_solver_fields* s, int32_t mode,
                             dv_vpm_plan* plan);
/* w_s = ω̃ of w (the smoothing above, dimcv_sph.py:660-677) on the plan's
 * neighbours; x [n][2], w and w_s [n], in the plan's slot order. */
DV_API int dv_vpm_smooth(dv_ctx* ctx, const dv_vpm_plan* plan, int32_t precision, const void* x,
                         const void* w, void* w_s);
/* g_w = (∂ω̃/∂ω)^T g_ws, g_x = (∂ω̃/∂x)^T g_ws (written, not accumulated) */
DV_API int dv_vpm_smooth_bwd(dv_ctx* ctx, const dv_vpm_plan* plan, int32_t precision, const void* x,
                             const void* w, const void* g_ws, void* g_w, void* g_x);
/* SPH vorticity of a velocity field (compute_vorticity, dimcv_sph.py:228-248,
 * 2-D): ω_i = Σ_{j∈N(i)} m_V_j ((v_j − v_i) × ∇W(r_ij))_z; v [n][2]. */
DV_API int dv_vpm_curl(dv_ctx* ctx, const dv_vpm_plan* plan, int32_t precision, const void* x, const void* v,
                       void* w);
/* g_v = (∂ω/∂v)^T g_w, g_x = (∂ω/∂x)^T g_w (written, not accumulated) */
DV_API int dv_vpm_curl_bwd(dv_ctx* ctx, const dv_vpm_plan* plan, int32_t precision, const void* x,
                           const void* v, const void* g_w, void* g_v, void* g_x);
/* u = the velocity above (dimcv_sph.py:649-719 without the gate) of w_s on
 * the plan's neighbours and sources; u [n][2]; workspace of
 * dv_vpm_workspace_bytes bytes (device). */
DV_API int dv_vpm_velocity(dv_ctx* ctx, const dv_vpm_plan* plan, int32_t precision, const void* x,
                           const void* w_s, void* u, void* workspace, int64_t workspace_bytes);
/* g_ws = (∂u/∂ω̃)^T g_u, g_x = (∂u/∂x)^T g_u (written, not accumulated) */
DV_API int dv_vpm_velocity_bwd(dv_ctx* ctx, const dv_vpm_plan* plan, int32_t precision, const void* x,
                               const void* w_s, const void* g_u, void* g_ws, void* g_x, void* workspace,
                               int64_t workspace_bytes);

/* ------------------------------------------------------------------------
 * Scene batch (new: the reference steps one scene per process).  One context
 * created with params.n_scenes = S > 1 holds S independent scenes that share
 * every dv_params constant except the box: particle slots carry their scene
 * id in object_id, positions are scene-local, the cell key puts the scene id
 * above the Morton bits (params.grid_num = the largest scene grid), so every
 * neighbour sweep of the single-scene path runs on the whole batch at once
 * and never crosses scenes.  The per-scene parts are: activity box, emitter
 * schedule, DFSPH convergence (each scene iterates until its own average
 * error passes, as a lone scene would), kden_sum, the sampler
 * (M_s = max(1, floor(mc_fraction · fluid_s)) stratified draws from the
 * scene's own CDF with the scene's seed) and the far field (scene targets
 * against scene samples).  dv_batch_step enqueues one whole step
 * (karman_vortex.py:216-242 without the export sweep) with no host
 * synchronisation, so it can be captured in a CUDA graph (dv_batch_graph_*).
 * ------------------------------------------------------------------------ */
typedef struct dv_batch_scene {
  float domain_end[3];    /* the scene's box is [params.domain_start, domain_end] */
  int32_t cap;            /* upper bound of the scene's particle count */
  int32_t emit_offset;    /* the scene's emitter particles: [emit_offset, +emit_count) of emit_pos */
  int32_t emit_count;
  int32_t emit_interval;  /* emit every emit_interval steps (dimcv_sph.py:66-74); 0: no emitter */
  float emit_velocity[3];
  float emit_density;
  int32_t emit_color[3];
  float emit_volume;      /* m_V of emitted particles, 0.8 (2r)^dim as f32 (particle_system.py:46) */
  int32_t pad;
  uint64_t seed;          /* sampler seed of the scene */
} dv_batch_scene;

typedef struct dv_scene_state {  /* per scene, device-resident; read with dv_batch_read */
  int32_t start, end;            /* sorted slot range of the scene's active particles */
  int32_t n_fluid, n_solid;
  int32_t t_start, n_targets;    /* range in the target list */
  int32_t m_off, num_samples;    /* range in sample_idx */
  int32_t tile_off, iters_div;  /* tile_off: first far-field block of the scene (blocks go out most samples first) */
  int32_t iters_p, done;
  int32_t status, emitted;       /* DV_WARN_* bits of the scene; particles emitted so far */
  double err_div, err_p, kden_sum;
  float kden_sum_f32;
  int32_t pad;
} dv_scene_state;

/* Per-scene tables; emit_pos is [n_emit][dim] (host); sample_mode is
 * DV_SAMPLE_INVERSE_CDF or DV_SAMPLE_STRATIFIED.  Sets the device step counter
 * to 0.  Synchronises. */
DV_API int dv_batch_setup(dv_ctx* ctx, const dv_batch_scene* scenes, int32_t n_scenes, const float* emit_pos,
                          int32_t n_emit, float mc_fraction, int32_t sample_mode);
/* One step of every scene: emit (scenes whose interval divides the step
 * counter), update_activity, grid build src -> dst, then the substep on dst
 * (densities, DFSPH factor, divergence solve, non-pressure forces, DIMCV with
 * stratified sampling, predict, pressure solve, advect); step counter += 1. */
DV_API int dv_batch_step(dv_ctx* ctx, const dv_fields* src, const dv_fields* dst, const dv_solver_fields* s);
/* Captures `steps` (even) steps alternating src -> dst, dst -> src into a CUDA
 * graph owned by the context (replaces the previous one). */
DV_API int dv_batch_graph_capture(dv_ctx* ctx, const dv_fields* a, const dv_fields* b,
                                  const dv_solver_fields* s, int32_t steps);
/* Launches the captured graph once, ordered after the work already on the
 * context stream and before the work enqueued after it. */
DV_API int dv_batch_graph_launch(dv_ctx* ctx);
/* Copies the per-scene state to the host and the device step counter to
 * *step (may be NULL).  Synchronises. */
DV_API int dv_batch_read(dv_ctx* ctx, dv_scene_state* out, int32_t n_scenes, int64_t* step);

#endif /* DIMCV_H_ */
