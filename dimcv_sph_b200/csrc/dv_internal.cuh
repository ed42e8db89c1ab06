// Internal declarations of libdimcv: the context object, device helpers
// shared by every translation unit, and the launch helpers.
//
// Numerics contract of the SPH sweeps (dv_grid.cu, dv_sph.cu, dv_dimcv.cu):
// those files are compiled with -fmad=false and IEEE division / square root,
// and every per-pair expression follows the operation order of the
// reference's Taichi functions (cited at each helper), so that the CPU
// oracle, which restates the same order in C++ with -ffp-contract=off,
// produces the same f32 bits for the same inputs and visit order.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

#include "../../include/dimcv.h"

#define DV_THREADS 256
#define DV_MAX_FAR_CHUNKS 8

// ------------------------------------------------------------------ context
struct dv_ctx {
  dv_params p;
  int64_t cap = 0;
  cudaStream_t stream = nullptr;
  int device = 0;
  int num_sms = 148;
  std::string err;
  int64_t launches = 0;
  int64_t n_upper = 0;  // host-side upper bound of the device particle count

  dv_counters* d_cnt = nullptr;  // device counters
  dv_counters* h_cnt = nullptr;  // pinned mirror
  int32_t* d_flag = nullptr;     // [0]: solve done flag, [1]: scratch
  int32_t* h_flag = nullptr;     // pinned mirror

  // grid / sort
  uint32_t* keys[2] = {nullptr, nullptr};
  uint32_t* vals[2] = {nullptr, nullptr};
  uint32_t* hist = nullptr;  // 256 * max_tiles
  int64_t max_tiles = 0;
  int32_t* cell_start = nullptr;
  int32_t* cell_end = nullptr;
  int64_t ncells = 0;  // padded Morton cell count
  int kbits = 0;       // sort key bits (Morton bits + 1 for the inactive key)
  int npasses = 0;
  int perm_buf = 0;    // which vals[] holds the last permutation
  uint32_t* mt[3] = {nullptr, nullptr, nullptr};  // per-axis Morton tables

  // scans and reductions
  uint32_t* scan_part = nullptr;  // uint32 block partials
  double* dscan_part = nullptr;   // double block partials
  int64_t scan_part_cap = 0;
  double* red_part = nullptr;     // FP64 per-block partials of sweeps
  int32_t* ired_part = nullptr;   // int per-block partials
  int64_t red_cap = 0;

  // DIMCV scratch
  uint32_t* flags = nullptr;   // cap+1
  uint32_t* offs = nullptr;    // cap+1
  int32_t* targets = nullptr;  // cap
  double* cdf = nullptr;       // cap
  float4* spos = nullptr;      // cap
  float4* sw = nullptr;        // cap
  float4* near_v = nullptr;    // cap
  float* near_S = nullptr;     // cap
  float4* far_acc = nullptr;   // cap: far-field sums of the main loop, per target
  int32_t* mult = nullptr;     // cap: sample multiplicity per slot
  uint32_t* sflag = nullptr;   // cap + 1: 1 where mult > 0
  uint32_t* srank = nullptr;   // cap + 1: exclusive scan of sflag (sampled slots before a slot)
  int32_t* sslot = nullptr;    // cap: the sampled slots in slot order, srank[j] -> j
  int far_tt = 4;              // targets per thread of the far-field main loop (autotuned)
  int far_chunks = 1;          // sample chunks of the far-field grid (autotuned, <= DV_MAX_FAR_CHUNKS)
  bool dyn_rigid = false;      // dynamic rigid particles present: pressure iterations add their reaction

  // per-step neighbour lists (CSR, visit order) built by dv_grid_build
  uint32_t* nbr_off = nullptr;  // cap + 1
  int32_t* nbr_idx = nullptr;   // nbr_cap
  int64_t nbr_cap = 0;
  int32_t* d_nbr_ok = nullptr;  // [0]: 1 while the lists match the current positions; [1]: build scratch
  int32_t* nbr_rows = nullptr;  // 3-D: cap * nbr_slots, the first pass's fixed row of particle i at i * nbr_slots
  int nbr_slots = 0;

  // scene batch (n_scenes > 1): cell keys carry the scene id above
  // scene_shift bits; scene_ptr is the scene id of each slot of the sorted
  // set (its object_id array); scene_end is [n_scenes][3] per-scene domain ends
  int scene_shift = 0;
  const int32_t* scene_ptr = nullptr;
  float* d_scene_end = nullptr;
  struct dv_batch_state* batch = nullptr;

  // far-field kernel profiling (dv_profile)
  bool prof = false;
  static constexpr int kProfPool = 512;
  cudaEvent_t prof_ev[2 * kProfPool] = {};
  int prof_used = 0;
  double prof_ms = 0.0;
  int64_t prof_launches = 0;
  double* d_prof = nullptr;  // device: [0] pairs
};

int dv_fail(dv_ctx* c, int code, const char* fmt, ...);
int dv_cuda_check(dv_ctx* c, cudaError_t e, const char* what);
#define DV_CK(ctx, call)                                    \
  do {                                                      \
    cudaError_t e_ = (call);                                \
    if (e_ != cudaSuccess) return dv_cuda_check(ctx, e_, #call); \
  } while (0)
#define DV_LAUNCHED(ctx)                                             \
  do {                                                               \
    (ctx)->launches++;                                               \
    cudaError_t e_ = cudaGetLastError();                             \
    if (e_ != cudaSuccess) return dv_cuda_check(ctx, e_, "kernel launch"); \
  } while (0)

static inline int dv_blocks(int64_t n, int threads = DV_THREADS) {
  int64_t b = (n + threads - 1) / threads;
  return (int)(b < 1 ? 1 : b);
}

// Bounds of the particle loops: the device count, capped by capacity.
struct DevGrid {
  const int32_t* start;
  const int32_t* end;
  const uint32_t* mt0;
  const uint32_t* mt1;
  const uint32_t* mt2;
  // neighbour lists of the last grid build (CSR in visit order); used while
  // *nok != 0, i.e. until positions move or particles are added
  const uint32_t* noff;
  const int32_t* nidx;
  const int32_t* nok;
  // scene batch: the cell key of slot i is (scene[i] << scene_shift) | Morton
  const int32_t* scene;
  int scene_shift;
};
static inline DevGrid dv_grid(const dv_ctx* c) {
  return DevGrid{c->cell_start, c->cell_end, c->mt[0], c->mt[1], c->mt[2], c->nbr_off, c->nbr_idx,
                 c->d_nbr_ok, c->scene_ptr, c->scene_shift};
}
// the cell-scan form only (used to build the neighbour lists)
static inline DevGrid dv_grid_cells(const dv_ctx* c) {
  return DevGrid{c->cell_start, c->cell_end, c->mt[0], c->mt[1], c->mt[2], nullptr, nullptr, nullptr,
                 c->scene_ptr, c->scene_shift};
}

// ------------------------------------------------------------- scene batch
// Host-side state of a scene batch (dv_batch_setup); every pointer is device.
struct dv_batch_state {
  int S = 0;
  float mc_fraction = 0.0625f;
  dv_batch_scene* d_scenes = nullptr; // [S]
  dv_scene_state* d_state = nullptr;  // [S]
  int32_t* d_done = nullptr;          // [S + 1]: per-scene solve done; [S]: every scene done
  int32_t* d_wl = nullptr;            // [S + 1]: work list of the scenes still iterating (block offsets)
  int32_t* d_ctr = nullptr;           // iterations of the captured Jacobi loop
  int32_t* d_misc = nullptr;          // [0]: far-field tiles this step
  int32_t* d_order = nullptr;         // [S]: scenes in far-field block order (most samples per tile first)
  double* d_err = nullptr;            // [cap] residual block sums of the solves (one per work-list block)
  int64_t* d_step = nullptr;          // step counter (emission schedule, sampler stream)
  float* d_emit = nullptr;            // [n_emit][dim]
  int32_t n_emit = 0;
  int64_t cap_tiles = 0;              // launch bound of the far-field work list
  int64_t m_cap = 0;                  // launch bound of the total sample count
  bool capturing = false;             // unroll the Jacobi loops (no host polling)
  int stratified = 0;                 // DV_SAMPLE_STRATIFIED draws, else i.i.d.
  cudaGraphExec_t graph = nullptr;
  cudaStream_t gstream = nullptr;
  cudaStream_t bstream = nullptr;     // captures the Jacobi loop bodies
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};
// dv_batch.cu
void dv_batch_free(dv_ctx* c);
int dv_batch_solve_reset(dv_ctx* c, int which);
int dv_batch_solve_finalize(dv_ctx* c, int which);
int dv_batch_loop_condition(dv_ctx* c, cudaGraphConditionalHandle h, int max_iter);
// dv_sph.cu: one DFSPH Jacobi solve with per-scene convergence
// which 0 (divergence) or 1 (pressure); nonpressure: the divergence residual
// sweeps also compute compute_non_pressure_forces (as DV_SOLVE_NONPRESSURE)
int dv_batch_solve(dv_ctx* c, const dv_fields* f, int which, bool nonpressure = false);
// dv_dimcv.cu: per-scene inverse-CDF draws (targets built)
int dv_batch_draw(dv_ctx* c, const dv_solver_fields* s);
// dv_vvpe.cu: near field, far field (scene targets x scene samples), gate
int dv_batch_vvpe(dv_ctx* c, const dv_fields* f, const dv_solver_fields* s);
int dv_far_tile_width(const dv_ctx* c);
int dv_far_min_tile_width();  // the narrowest far-field tile (threads per CTA x 2 targets)
int dv_build_targets(dv_ctx* c, const dv_fields* f);

// ------------------------------------------------------------- scan helpers
// Exclusive scan of uint32 / double arrays on the context stream
// (deterministic three-phase: block reduce, scan of partials, block scan).
int dv_scan_u32(dv_ctx* c, const uint32_t* in, uint32_t* out, int64_t m);
int dv_scan_f64(dv_ctx* c, const double* in, double* out, int64_t m);
// Sum of `nparts` FP64 partials into *dst (device), one block, fixed order.
int dv_finalize_sum(dv_ctx* c, const double* parts, int nparts, double* dst);
// Marks the per-step neighbour lists stale (positions or counts changed).
int dv_invalidate_lists(dv_ctx* c);

// ------------------------------------------------------------ device helpers
struct V3 {
  float x, y, z;
};

template <int D>
__device__ __forceinline__ V3 ldv(const float* a, int i) {
  if (D == 2) {
    float2 t = reinterpret_cast<const float2*>(a)[i];
    return V3{t.x, t.y, 0.0f};
  } else {
    float4 t = reinterpret_cast<const float4*>(a)[i];
    return V3{t.x, t.y, t.z};
  }
}
template <int D>
__device__ __forceinline__ void stv(float* a, int i, V3 v) {
  if (D == 2) {
    reinterpret_cast<float2*>(a)[i] = make_float2(v.x, v.y);
  } else {
    reinterpret_cast<float4*>(a)[i] = make_float4(v.x, v.y, v.z, 0.0f);
  }
}
__device__ __forceinline__ V3 ld4(const float* a, int i) {
  float4 t = reinterpret_cast<const float4*>(a)[i];
  return V3{t.x, t.y, t.z};
}
__device__ __forceinline__ void st4(float* a, int i, V3 v) {
  reinterpret_cast<float4*>(a)[i] = make_float4(v.x, v.y, v.z, 0.0f);
}

// r = x_i - x_j and its squared norm ((rx*rx + ry*ry) + rz*rz), the order of
// Taichi's Matrix.norm_sqr (sum of entries left to right).
template <int D>
__device__ __forceinline__ float sqnorm(V3 r) {
  float s = __fadd_rn(__fmul_rn(r.x, r.x), __fmul_rn(r.y, r.y));
  if (D == 3) s = __fadd_rn(s, __fmul_rn(r.z, r.z));
  return s;
}
template <int D>
__device__ __forceinline__ float dot(V3 a, V3 b) {
  float s = __fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y));
  if (D == 3) s = __fadd_rn(s, __fmul_rn(a.z, b.z));
  return s;
}
__device__ __forceinline__ V3 cross3(V3 a, V3 b) {
  // Taichi cross: (a1 b2 - a2 b1, a2 b0 - a0 b2, a0 b1 - a1 b0)
  return V3{__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)),
            __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
            __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x))};
}

// Cubic spline W (sph_base.py:23-44).  (1-q)^3 is evaluated as ((1-q)(1-q))(1-q).
__device__ __forceinline__ float cubic_W(const dv_params& P, float r_norm) {
  float res = 0.0f;
  float q = r_norm * P.inv_support_radius;
  if (q <= 1.0f) {
    if (q <= 0.5f) {
      float q2 = q * q;
      float q3 = q2 * q;
      res = P.kW * (6.0f * q3 - 6.0f * q2 + 1.0f);
    } else {
      float f = 1.0f - q;
      res = P.kW2 * ((f * f) * f);
    }
  }
  return res;
}

// Cubic spline gradient (sph_base.py:46-68); r2 is sqnorm(r).
template <int D>
__device__ __forceinline__ V3 cubic_gradW(const dv_params& P, V3 r, float r2) {
  V3 res{0.0f, 0.0f, 0.0f};
  float h = P.inv_support_radius;
  float r_norm = sqrtf(r2);
  float q = r_norm * h;
  if (r_norm > P.grad_r_min && q <= 1.0f) {
    // r / r_norm * h with the division as one IEEE reciprocal (the arcp form
    // of the reference's fast-math codegen); the oracle does the same
    const float inv = 1.0f / r_norm;
    V3 gq{(r.x * inv) * h, (r.y * inv) * h, D == 3 ? (r.z * inv) * h : 0.0f};
    float s;
    if (q <= 0.5f) {
      s = (P.kG * q) * (3.0f * q - 2.0f);
    } else {
      float f = 1.0f - q;
      s = P.kG * (-(f * f));
    }
    res.x = s * gq.x;
    res.y = s * gq.y;
    if (D == 3) res.z = s * gq.z;
  }
  return res;
}

// pos_to_index (particle_system.py:382-384): truncation of x / grid_size.
// Optionally offset by domain_start (new option).  Clamped before the int
// conversion so that non-finite or huge positions stay defined.
__device__ __forceinline__ int cell_coord(const dv_params& P, float x, int d) {
  float t = P.cell_origin_offset ? (x - P.domain_start[d]) : x;
  float q = t / P.grid_size;
  if (!(q > -1.0e9f)) q = -1.0e9f;
  if (q > 1.0e9f) q = 1.0e9f;
  int g = (int)q;
  // a periodic box holds every position in [start, start + box): a quotient
  // that rounds up to grid_num belongs to the last cell
  if (P.periodic) g = g < 0 ? 0 : (g >= P.grid_num[d] ? P.grid_num[d] - 1 : g);
  return g;
}

// minimum-image difference on a periodic axis of length L (|d| < L assumed)
__device__ __forceinline__ float min_image(float d, float L) {
  const float hl = 0.5f * L;
  return d > hl ? __fsub_rn(d, L) : (d < -hl ? __fadd_rn(d, L) : d);
}
// r = x_i - x_j, minimum image when the box is periodic
template <int D>
__device__ __forceinline__ V3 rel(const dv_params& P, V3 xi, V3 xj) {
  V3 r{__fsub_rn(xi.x, xj.x), __fsub_rn(xi.y, xj.y), D == 3 ? __fsub_rn(xi.z, xj.z) : 0.0f};
  if (P.periodic) {
    r.x = min_image(r.x, P.box[0]);
    r.y = min_image(r.y, P.box[1]);
    if (D == 3) r.z = min_image(r.z, P.box[2]);
  }
  return r;
}
// cell coordinate c + a on an axis of n cells: wrapped when periodic, -1 if outside
__device__ __forceinline__ int cell_step(const dv_params& P, int c, int a, int n) {
  int g = c + a;
  if (P.periodic) return g < 0 ? g + n : (g >= n ? g - n : g);
  return (g < 0 || g >= n) ? -1 : g;
}

template <int D>
__device__ __forceinline__ bool in_vortex_domain(const dv_params& P, V3 x) {
  if (!P.has_vortex_domain) return true;
  if (x.x < P.vd_start[0] || x.x > P.vd_end[0]) return false;
  if (x.y < P.vd_start[1] || x.y > P.vd_end[1]) return false;
  if (D == 3 && (x.z < P.vd_start[2] || x.z > P.vd_end[2])) return false;
  return true;
}

// compute_divergence_transit_weight (dimcv_sph.py:401-405)
__device__ __forceinline__ float transit_weight(const dv_params& P, float x0) {
  float w = (x0 - P.transit_a0) / P.transit_span;
  return fminf(fmaxf(w, 0.0f), 1.0f);
}

// The neighbour visit of ParticleSystem.for_all_neighbors
// (particle_system.py:562-586): the 3^d cells around the cell of x_i in
// offset order (-1..1 per axis, last axis fastest), skipping cells outside
// [0, grid_num) and, in reference mode, flat cell 0; within a cell the slots
// in ascending order; j is visited iff j != i and |x_i - x_j| < h, which is
// tested exactly as r2 < nbr_r2_limit (sqrtf is monotone, so
// sqrtf(r2) < h  <=>  r2 < the smallest float whose sqrtf reaches h).
// f(j, r, r2) receives r = x_i - x_j; for_each_neighbor_m also passes the
// neighbour's material mj (fluid or solid): on the list path it is the top
// bit of the list entry (DV_NBR_SOLID), so it costs no load; on the
// cell-scan path it is mat[j].
// A stored list entry: the neighbour's slot in the low 31 bits, bit 31 set
// for a solid neighbour.  The list build marks the lists invalid when it
// meets a material other than fluid or solid, so the sweeps then scan cells.
#define DV_NBR_SOLID 0x80000000u
#define DV_NBR_SLOT 0x7fffffffu
__device__ __forceinline__ int nbr_slot(uint32_t e) { return (int)(e & DV_NBR_SLOT); }
__device__ __forceinline__ int nbr_mat(uint32_t e) { return (e & DV_NBR_SOLID) ? DV_MATERIAL_SOLID : DV_MATERIAL_FLUID; }

template <int D, bool MAT, typename F>
__device__ __forceinline__ void for_each_neighbor_impl(const dv_params& P, const DevGrid& G,
                                                       const float* __restrict__ x,
                                                       const int32_t* __restrict__ mat, int i, V3 xi, F&& f) {
  if (G.nok && __ldg(G.nok)) {  // the lists hold exactly these j, in this order
    uint32_t k = __ldg(G.noff + i);
    const uint32_t k1 = __ldg(G.noff + i + 1);
    if (k >= k1) return;
    // one-deep software pipeline: the next neighbour's entry and position
    // are loaded before f runs on the current one (f still runs in list
    // order).  Sweeps -5% at 2.37M particles; a two-deep pipeline was slower.
    const uint32_t* __restrict__ nl = reinterpret_cast<const uint32_t*>(G.nidx);
    uint32_t e = __ldg(nl + k);
    int j = nbr_slot(e);
    V3 xj = ldv<D>(x, j);
    int mj = nbr_mat(e);
#pragma unroll 1
    while (true) {
      const bool more = ++k < k1;
      const uint32_t en = more ? __ldg(nl + k) : e;
      const int jn = nbr_slot(en);
      const V3 xn = ldv<D>(x, jn);
      const int mn = nbr_mat(en);
      V3 r = rel<D>(P, xi, xj);
      if constexpr (MAT)
        f(j, r, sqnorm<D>(r), mj);
      else
        f(j, r, sqnorm<D>(r));
      if (!more) break;
      j = jn;
      xj = xn;
      mj = mn;
    }
    return;
  }
  int c0 = cell_coord(P, xi.x, 0), c1 = cell_coord(P, xi.y, 1);
  int c2 = D == 3 ? cell_coord(P, xi.z, 2) : 0;
  const float lim = P.nbr_r2_limit;
  const uint32_t sk = G.scene ? ((uint32_t)__ldg(G.scene + i) << G.scene_shift) : 0u;
#pragma unroll 1
  for (int a = -1; a <= 1; ++a) {
    int gx = cell_step(P, c0, a, P.grid_num[0]);
    if (gx < 0) continue;
    uint32_t kx = __ldg(G.mt0 + gx);
#pragma unroll 1
    for (int b = -1; b <= 1; ++b) {
      int gy = cell_step(P, c1, b, P.grid_num[1]);
      if (gy < 0) continue;
      uint32_t kxy = kx | __ldg(G.mt1 + gy);
#pragma unroll 1
      for (int c = (D == 3 ? -1 : 0); c <= (D == 3 ? 1 : 0); ++c) {
        uint32_t key = kxy;
        if (D == 3) {
          int gz = cell_step(P, c2, c, P.grid_num[2]);
          if (gz < 0) continue;
          key |= __ldg(G.mt2 + gz);
        }
        if (P.skip_cell0 && key == 0u) continue;  // the scene's own flat cell 0
        key |= sk;
        int s = __ldg(G.start + key), e = __ldg(G.end + key);
#pragma unroll 1
        for (int j = s; j < e; ++j) {
          if (j == i) continue;
          V3 r = rel<D>(P, xi, ldv<D>(x, j));
          float r2 = sqnorm<D>(r);
          if (r2 < lim) {
            if constexpr (MAT)
              f(j, r, r2, __ldg(mat + j));
            else
              f(j, r, r2);
          }
        }
      }
    }
  }
}

template <int D, typename F>
__device__ __forceinline__ void for_each_neighbor(const dv_params& P, const DevGrid& G,
                                                  const float* __restrict__ x, int i, V3 xi, F&& f) {
  for_each_neighbor_impl<D, false>(P, G, x, nullptr, i, xi, f);
}

template <int D, typename F>
__device__ __forceinline__ void for_each_neighbor_m(const dv_params& P, const DevGrid& G,
                                                    const float* __restrict__ x, const int32_t* __restrict__ mat,
                                                    int i, V3 xi, F&& f) {
  for_each_neighbor_impl<D, true>(P, G, x, mat, i, xi, f);
}

// ---------------------------------------------------------------- Philox
// Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC'11): 10 rounds of the published multipliers and Weyl
// key increments.  Counter = (slot, draw, step lo, step hi), key = seed.
struct DvRand4 {
  uint32_t v[4];
};
__host__ __device__ inline DvRand4 dv_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                            uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)M0 * c0;
    uint64_t p1 = (uint64_t)M1 * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n1 = lo1;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    uint32_t n3 = lo0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += W0;
    k1 += W1;
  }
  DvRand4 o;
  o.v[0] = c0; o.v[1] = c1; o.v[2] = c2; o.v[3] = c3;
  return o;
}
// uniform float in [0, 1) with 24 random bits (exact on host and device)
__host__ __device__ inline float dv_u01f(uint32_t u) { return (float)(u >> 8) * (1.0f / 16777216.0f); }
// uniform double in [0, 1) with 53 random bits
__host__ __device__ inline double dv_u01d(uint32_t a, uint32_t b) {
  uint64_t m = ((uint64_t)(a >> 5) << 26) | (uint64_t)(b >> 6);
  return (double)m * (1.0 / 9007199254740992.0);
}

// --------------------------------------------------- deterministic reductions
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
// Block sum in a fixed tree; result valid in thread 0.  blockDim.x <= 1024.
template <typename T>
__device__ __forceinline__ T block_sum(T v) {
  __shared__ T s_ws[32];
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) s_ws[w] = v;
  __syncthreads();
  int nw = (blockDim.x + 31) >> 5;
  T t = (threadIdx.x < nw) ? s_ws[threadIdx.x] : T(0);
  if (w == 0) t = warp_sum(t);
  return t;
}
