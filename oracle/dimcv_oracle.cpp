// CPU oracle of the DIMCV-SPH substep — TEST INFRASTRUCTURE ONLY.
//
// A plain C++17 restatement of the reference's Taichi kernels (Haok-Z/
// DIMCV-SPH: particle_system.py, sph_base.py, dimcv_sph.py), used by tests/,
// by the smoke check and by bench.py's CPU baseline as the checker; it is
// never part of the product path.  Each function cites the reference lines
// it restates.  Arithmetic is f32 in the reference's operation order
// (compiled with -ffp-contract=off, no fast-math); the N-body sums also have
// an FP64 mode.  Reductions that the reference does with f32 atomics
// (kden_sum, the DFSPH error norms) are FP64 here, summed in slot order.
//
// Parity is UNPINNED against the reference itself: Taichi is not installed
// and the reference ships no tests or golden vectors.  The oracle is pinned
// by known-answer tests and by a NumPy restatement (tests/golden/).
//
// Visit order: the reference sorts by the row-major flat cell id
// (particle_system.py:386-393) and, when its counting sort runs serially,
// keeps slot order inside a cell (:500-510).  order_mode 1 reproduces that;
// order_mode 0 sorts by the Morton key layout of the CUDA library instead
// (same bits: per level, axes from last to first, lowest bit first), so that
// the two implementations visit neighbours in the same order.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstddef>
#include <cstring>
#include <vector>

#include "../include/dimcv.h"

#define DVO_API extern "C" __attribute__((visibility("default")))

namespace {

struct Ctx {
  dv_params p;
  int64_t cap;
  int order_mode;
  dv_counters cnt;
  // cell table: start/end per key
  std::vector<int32_t> cstart, cend;
  std::vector<uint32_t> mt[3];
  int64_t nkeys = 0;
  std::vector<int32_t> perm;
  std::vector<int32_t> targets;
  std::vector<float> near_v;  // 4 per target
  std::vector<float> near_S;
  // bounded samples for CPU timing: per-particle loops cover [lo, hi) only
  // (neighbours are still read everywhere); fixed Jacobi iteration counts
  int lo = 0, hi = 0x7fffffff;
  int fixed_div = 0, fixed_p = 0;
  bool dyn_rigid = false;  // pressure iterations add the reaction on dynamic solids
};

inline int range_lo(const Ctx* c) { return std::max(0, c->lo); }
inline int range_hi(const Ctx* c) { return std::min(c->cnt.n, c->hi); }

inline int vs(const Ctx& c) { return c.p.dim == 2 ? 2 : 4; }

struct V {
  float x = 0, y = 0, z = 0;
};
inline V ldv(const Ctx& c, const float* a, int i) {
  int s = vs(c);
  V v;
  v.x = a[(int64_t)i * s];
  v.y = a[(int64_t)i * s + 1];
  if (c.p.dim == 3) v.z = a[(int64_t)i * s + 2];
  return v;
}
inline void stv(const Ctx& c, float* a, int i, V v) {
  int s = vs(c);
  a[(int64_t)i * s] = v.x;
  a[(int64_t)i * s + 1] = v.y;
  if (c.p.dim == 3) a[(int64_t)i * s + 2] = v.z;
}
inline V ld4(const float* a, int i) { return V{a[4 * (int64_t)i], a[4 * (int64_t)i + 1], a[4 * (int64_t)i + 2]}; }
inline void st4(float* a, int i, V v) {
  a[4 * (int64_t)i] = v.x;
  a[4 * (int64_t)i + 1] = v.y;
  a[4 * (int64_t)i + 2] = v.z;
  a[4 * (int64_t)i + 3] = 0.0f;
}

// Matrix.norm_sqr: entries summed left to right
inline float norm_sqr(const Ctx& c, V r) {
  float s = r.x * r.x + r.y * r.y;
  if (c.p.dim == 3) s = s + r.z * r.z;
  return s;
}
inline float dotv(const Ctx& c, V a, V b) {
  float s = a.x * b.x + a.y * b.y;
  if (c.p.dim == 3) s = s + a.z * b.z;
  return s;
}
inline V cross(V a, V b) {
  return V{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// SPHBase.cubic_kernel (sph_base.py:23-44); ti.pow(1-q, 3.0) as (f f) f
inline float cubic_kernel(const dv_params& P, float r_norm) {
  float res = 0.0f;
  float h = P.inv_support_radius;
  float k = P.kW;
  float q = r_norm * h;
  if (q <= 1.0f) {
    if (q <= 0.5f) {
      float q2 = q * q;
      float q3 = q2 * q;
      res = k * (6.0f * q3 - 6.0f * q2 + 1.0f);
    } else {
      float f = 1.0f - q;
      res = P.kW2 * (f * f * f);
    }
  }
  return res;
}

// SPHBase.cubic_kernel_derivative (sph_base.py:46-68)
inline V cubic_kernel_derivative(const Ctx& c, V r) {
  const dv_params& P = c.p;
  float h = P.inv_support_radius;
  float k = P.kG;
  float r_norm = std::sqrt(norm_sqr(c, r));
  float q = r_norm * h;
  V res;
  if (r_norm > P.grad_r_min && q <= 1.0f) {
    // `r / r_norm * h` with the division taken as one reciprocal, the form
    // Taichi's default fast-math (arcp) codegen is allowed to emit
    const float inv = 1.0f / r_norm;
    V gq{r.x * inv * h, r.y * inv * h, c.p.dim == 3 ? r.z * inv * h : 0.0f};
    float s;
    if (q <= 0.5f) {
      s = k * q * (3.0f * q - 2.0f);
    } else {
      float factor = 1.0f - q;
      s = k * (-factor * factor);
    }
    res.x = s * gq.x;
    res.y = s * gq.y;
    if (c.p.dim == 3) res.z = s * gq.z;
  }
  return res;
}

// pos_to_index (particle_system.py:382-384)
inline int pos_to_index(const dv_params& P, float x, int d) {
  float t = P.cell_origin_offset ? x - P.domain_start[d] : x;
  float q = t / P.grid_size;
  if (!(q > -1.0e9f)) q = -1.0e9f;
  if (q > 1.0e9f) q = 1.0e9f;
  int g = (int)q;
  // a periodic box holds every position in [start, start + box): a quotient
  // that rounds up to grid_num belongs to the last cell
  if (P.periodic) g = g < 0 ? 0 : (g >= P.grid_num[d] ? P.grid_num[d] - 1 : g);
  return g;
}

inline int64_t cell_key(const Ctx& c, const int g[3]) {
  const dv_params& P = c.p;
  if (c.order_mode == 1) {  // flatten_grid_index_2d/3d (particle_system.py:386-393)
    if (P.dim == 2) return (int64_t)g[0] * P.grid_num[1] + g[1];
    return (int64_t)g[0] * P.grid_num[1] * P.grid_num[2] + (int64_t)g[1] * P.grid_num[2] + g[2];
  }
  uint32_t k = c.mt[0][g[0]] | c.mt[1][g[1]];
  if (P.dim == 3) k |= c.mt[2][g[2]];
  return k;
}

inline bool in_vortex_domain(const Ctx& c, V x) {  // dimcv_sph.py:77-84
  const dv_params& P = c.p;
  if (!P.has_vortex_domain) return true;
  float xs[3] = {x.x, x.y, x.z};
  for (int i = 0; i < P.dim; ++i)
    if (xs[i] < P.vd_start[i] || xs[i] > P.vd_end[i]) return false;
  return true;
}

inline float transit_weight(const dv_params& P, float x0) {  // dimcv_sph.py:401-405
  float w = (x0 - P.transit_a0) / P.transit_span;
  return std::min(std::max(w, 0.0f), 1.0f);
}

// minimum image on a periodic axis of length L (new option; the reference
// has no periodic boxes)
inline float min_image(float d, float L) {
  const float hl = 0.5f * L;
  return d > hl ? d - L : (d < -hl ? d + L : d);
}
inline V rel(const Ctx& c, V a, V b) {
  V r{a.x - b.x, a.y - b.y, a.z - b.z};
  if (c.p.periodic) {
    r.x = min_image(r.x, c.p.box[0]);
    r.y = min_image(r.y, c.p.box[1]);
    if (c.p.dim == 3) r.z = min_image(r.z, c.p.box[2]);
  }
  return r;
}

// for_all_neighbors (particle_system.py:562-586): literal distance test
template <typename F>
void for_all_neighbors(const Ctx& c, const float* x, int i, F&& task) {
  const dv_params& P = c.p;
  V xi = ldv(c, x, i);
  int ci[3] = {pos_to_index(P, xi.x, 0), pos_to_index(P, xi.y, 1), P.dim == 3 ? pos_to_index(P, xi.z, 2) : 0};
  int lo2 = P.dim == 3 ? -1 : 0, hi2 = P.dim == 3 ? 1 : 0;
  for (int a = -1; a <= 1; ++a)
    for (int b = -1; b <= 1; ++b)
      for (int cc = lo2; cc <= hi2; ++cc) {
        int g[3] = {ci[0] + a, ci[1] + b, ci[2] + cc};
        bool ok = true;
        for (int d = 0; d < P.dim; ++d) {
          if (P.periodic) g[d] = g[d] < 0 ? g[d] + P.grid_num[d] : (g[d] >= P.grid_num[d] ? g[d] - P.grid_num[d] : g[d]);
          if (g[d] < 0 || g[d] >= P.grid_num[d]) ok = false;
        }
        if (!ok) continue;
        int64_t key = cell_key(c, g);
        int s, e;
        if (c.order_mode == 1) {
          // range [P[max(0, c-1)], P[c]) over the inclusive prefix sum: flat
          // cell 0 is never visited (particle_system.py:581-583)
          int64_t f = key;
          s = f > 0 ? c.cend[f - 1] : c.cend[0];
          e = c.cend[f];
          if (!P.skip_cell0 && f == 0) s = 0;
        } else {
          if (P.skip_cell0 && key == 0) continue;
          s = c.cstart[key];
          e = c.cend[key];
        }
        for (int j = s; j < e; ++j) {
          if (j == i) continue;
          V r = rel(c, xi, ldv(c, x, j));
          if (std::sqrt(norm_sqr(c, r)) < P.support_radius) task(j, r);
        }
      }
}

void build_morton_tables(Ctx& c) {
  const dv_params& P = c.p;
  int bits[3] = {0, 0, 0};
  for (int d = 0; d < P.dim; ++d)
    while ((1 << bits[d]) < P.grid_num[d]) ++bits[d];
  int pos[3][21];
  int next = 0, maxb = std::max(bits[0], std::max(bits[1], bits[2]));
  for (int l = 0; l < maxb; ++l)
    for (int d = P.dim - 1; d >= 0; --d)
      if (l < bits[d]) pos[d][l] = next++;
  for (int d = 0; d < 3; ++d) {
    int g = d < P.dim ? P.grid_num[d] : 1;
    c.mt[d].assign(g, 0u);
    if (d < P.dim)
      for (int v = 0; v < g; ++v)
        for (int l = 0; l < bits[d]; ++l)
          if ((v >> l) & 1) c.mt[d][v] |= 1u << pos[d][l];
  }
  c.nkeys = (int64_t)1 << (bits[0] + bits[1] + bits[2]);
}

// Philox-4x32-10 (Salmon et al., SC'11), same counter / key convention as
// the CUDA library: counter (slot, draw, step lo, step hi), key (seed lo, hi)
void philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1, uint32_t out[4]) {
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    uint32_t n1 = (uint32_t)p1;
    uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    uint32_t n3 = (uint32_t)p0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

}  // namespace

// ======================================================================= API
DVO_API void* dvo_create(const dv_params* p, int64_t cap, int order_mode) {
  Ctx* c = new Ctx();
  c->p = *p;
  c->cap = cap;
  c->order_mode = order_mode;
  std::memset(&c->cnt, 0, sizeof(c->cnt));
  build_morton_tables(*c);
  if (order_mode == 1) {
    int64_t nf = 1;
    for (int d = 0; d < p->dim; ++d) nf *= p->grid_num[d];
    c->nkeys = nf;
  }
  c->cstart.assign(c->nkeys, 0);
  c->cend.assign(c->nkeys, 0);
  return c;
}
DVO_API void dvo_destroy(void* h) { delete (Ctx*)h; }
// sizeof / offsetof of the shared structs, compiled from include/dimcv.h
DVO_API void dvo_abi_layout(int64_t* out) {
  out[0] = sizeof(dv_params);
  out[1] = sizeof(dv_fields);
  out[2] = sizeof(dv_solver_fields);
  out[3] = sizeof(dv_counters);
  out[4] = offsetof(dv_params, eta_div);
  out[5] = offsetof(dv_params, compensated);
  out[6] = offsetof(dv_counters, err_div);
  out[7] = offsetof(dv_counters, kden_sum_f32);
  out[8] = sizeof(dv_vpm_plan);
  out[9] = sizeof(dv_batch_scene);
  out[10] = offsetof(dv_batch_scene, seed);
  out[11] = sizeof(dv_scene_state);
  out[12] = offsetof(dv_scene_state, err_div);
  out[13] = offsetof(dv_params, n_scenes);
}
DVO_API void dvo_set_counts(void* h, int n, int nf, int ns) {
  Ctx* c = (Ctx*)h;
  c->cnt.n = n;
  c->cnt.n_fluid = nf;
  c->cnt.n_solid = ns;
}
DVO_API void dvo_get_counters(void* h, dv_counters* out) { *out = ((Ctx*)h)->cnt; }
DVO_API void dvo_set_num_samples(void* h, int m) { ((Ctx*)h)->cnt.num_samples = m; }
DVO_API void dvo_set_counters(void* h, const dv_counters* in) { ((Ctx*)h)->cnt = *in; }
// bounded CPU-timing samples: restrict per-particle loops to slots [lo, hi)
// and run the Jacobi solves for exactly it_div / it_p iterations (0 = converge)
DVO_API void dvo_set_sample(void* h, int lo, int hi, int it_div, int it_p) {
  Ctx* c = (Ctx*)h;
  c->lo = lo;
  c->hi = hi;
  c->fixed_div = it_div;
  c->fixed_p = it_p;
}

// _add_particles / add_particle (particle_system.py:317-380)
DVO_API int dvo_add_particles(void* h, dv_fields* f, const float* pos, const float* vel, int count,
                              int obj, float density, float pressure, int material, int is_dyn,
                              int cr, int cg, int cb, float m_V0) {
  Ctx* c = (Ctx*)h;
  int n = c->cnt.n, added = 0;
  for (int k = 0; k < count; ++k) {
    int p = n + k;
    if (p >= c->cap) break;
    V x{pos[k * c->p.dim], pos[k * c->p.dim + 1], c->p.dim == 3 ? pos[k * c->p.dim + 2] : 0.0f};
    V v{vel[k * c->p.dim], vel[k * c->p.dim + 1], c->p.dim == 3 ? vel[k * c->p.dim + 2] : 0.0f};
    stv(*c, f->x, p, x);
    stv(*c, f->x0, p, x);
    stv(*c, f->v, p, v);
    stv(*c, f->acceleration, p, V{});
    st4(f->vorticity, p, V{});
    f->object_id[p] = obj;
    f->density[p] = density;
    f->m_V[p] = m_V0;
    f->m[p] = m_V0 * density;
    f->pressure[p] = pressure;
    f->material[p] = material;
    f->is_dynamic[p] = is_dyn != 0;
    f->color[4 * p] = cr; f->color[4 * p + 1] = cg; f->color[4 * p + 2] = cb; f->color[4 * p + 3] = 0;
    f->is_active[p] = 1;
    f->dfsph_factor[p] = 0; f->density_adv[p] = 0; f->is_sample[p] = 0; f->life_time[p] = 0;
    f->grid_ids[p] = -1;
    ++added;
  }
  if (added < count) c->cnt.status |= DV_WARN_CAPACITY;
  c->cnt.n += added;
  if (material == DV_MATERIAL_FLUID) c->cnt.n_fluid += added; else c->cnt.n_solid += added;
  return 0;
}

// update_activity (particle_system.py:413-427)
DVO_API int dvo_update_activity(void* h, dv_fields* f) {
  Ctx* c = (Ctx*)h;
  const dv_params& P = c->p;
  for (int i = range_lo(c); i < range_hi(c); ++i) {
    if (f->material[i] == DV_MATERIAL_SOLID) {
      f->is_active[i] = 1;
    } else if (f->material[i] == DV_MATERIAL_FLUID && !P.periodic) {
      V x = ldv(*c, f->x, i);
      float xs[3] = {x.x, x.y, x.z};
      for (int j = 0; j < P.dim; ++j)
        if (xs[j] < P.domain_start[j] || xs[j] > P.domain_end[j]) {
          f->is_active[i] = 0;
          c->cnt.n_fluid -= 1;
          break;
        }
    }
  }
  return 0;
}

// particle_partition + update_grid_id + prefix sum + counting_sort
// (particle_system.py:429-560): stable compaction of active slots, then a
// stable sort by cell key; every field gathered from src into dst.
DVO_API int dvo_grid_build(void* h, dv_fields* S, dv_fields* T) {
  Ctx* c = (Ctx*)h;
  const dv_params& P = c->p;
  const int n = c->cnt.n;
  std::vector<int> act;
  act.reserve(n);
  for (int i = 0; i < n; ++i)
    if (S->is_active[i] == 1) act.push_back(i);
  const int m = (int)act.size();
  std::vector<int64_t> key(m);
  for (int k = 0; k < m; ++k) {
    V x = ldv(*c, S->x, act[k]);
    int g[3] = {pos_to_index(P, x.x, 0), pos_to_index(P, x.y, 1), P.dim == 3 ? pos_to_index(P, x.z, 2) : 0};
    for (int d = 0; d < P.dim; ++d) {
      if (g[d] < 0 || g[d] >= P.grid_num[d]) c->cnt.status |= DV_WARN_OUTSIDE_GRID;
      g[d] = std::min(std::max(g[d], 0), P.grid_num[d] - 1);
    }
    key[k] = cell_key(*c, g);
  }
  // counting sort by key: histogram, inclusive prefix sum, stable placement
  std::vector<int32_t> cnt(c->nkeys, 0);
  for (int k = 0; k < m; ++k) cnt[key[k]]++;
  std::vector<int32_t> incl(c->nkeys);
  int32_t run = 0;
  for (int64_t q = 0; q < c->nkeys; ++q) {
    run += cnt[q];
    incl[q] = run;
  }
  std::vector<int32_t> fill(c->nkeys);
  for (int64_t q = 0; q < c->nkeys; ++q) fill[q] = incl[q] - cnt[q];
  c->perm.assign(m, 0);
  std::vector<int64_t> skey(m);
  for (int k = 0; k < m; ++k) {
    int pos = fill[key[k]]++;
    c->perm[pos] = act[k];
    skey[pos] = key[k];
  }
  for (int64_t q = 0; q < c->nkeys; ++q) {
    c->cend[q] = incl[q];
    c->cstart[q] = incl[q] - cnt[q];
  }
  // gather
  const int s = vs(*c);
  int nf = 0, ns = 0;
  for (int p = 0; p < m; ++p) {
    int j = c->perm[p];
    for (int d = 0; d < s; ++d) {
      T->x[p * s + d] = S->x[j * s + d];
      T->x0[p * s + d] = S->x0[j * s + d];
      T->v[p * s + d] = S->v[j * s + d];
      T->acceleration[p * s + d] = S->acceleration[j * s + d];
    }
    for (int d = 0; d < 4; ++d) {
      T->vorticity[p * 4 + d] = S->vorticity[j * 4 + d];
      T->color[p * 4 + d] = S->color[j * 4 + d];
    }
    T->m_V[p] = S->m_V[j];
    T->m[p] = S->m[j];
    T->density[p] = S->density[j];
    T->pressure[p] = S->pressure[j];
    T->dfsph_factor[p] = S->dfsph_factor[j];
    T->density_adv[p] = S->density_adv[j];
    T->life_time[p] = S->life_time[j];
    T->material[p] = S->material[j];
    T->object_id[p] = S->object_id[j];
    T->grid_ids[p] = (int32_t)skey[p];
    T->is_dynamic[p] = S->is_dynamic[j];
    T->is_active[p] = S->is_active[j];
    T->is_sample[p] = S->is_sample[j];
    nf += S->material[j] == DV_MATERIAL_FLUID;
    ns += S->material[j] == DV_MATERIAL_SOLID;
  }
  for (int p = m; p < n; ++p) {  // partition fill values (particle_system.py:455-465)
    for (int d = 0; d < s; ++d) {
      T->x[p * s + d] = -1.0f;
      T->x0[p * s + d] = -1.0f;
      T->v[p * s + d] = 0.0f;
      T->acceleration[p * s + d] = 0.0f;
    }
    for (int d = 0; d < 4; ++d) {
      T->vorticity[p * 4 + d] = S->vorticity[p * 4 + d];
      T->color[p * 4 + d] = 255;
    }
    T->m_V[p] = S->m_V[p];
    T->m[p] = S->m[p];
    T->density[p] = S->density[p];
    T->pressure[p] = S->pressure[p];
    T->dfsph_factor[p] = S->dfsph_factor[p];
    T->density_adv[p] = S->density_adv[p];
    T->life_time[p] = 0.0f;
    T->material[p] = S->material[p];
    T->object_id[p] = -1;
    T->grid_ids[p] = -1;
    T->is_dynamic[p] = 0;
    T->is_active[p] = 0;
    T->is_sample[p] = 0;
  }
  c->cnt.n = m;
  c->cnt.n_fluid = nf;
  c->cnt.n_solid = ns;
  return 0;
}

DVO_API int dvo_get_permutation(void* h, int32_t* out) {
  Ctx* c = (Ctx*)h;
  std::copy(c->perm.begin(), c->perm.end(), out);
  return (int)c->perm.size();
}

DVO_API int64_t dvo_neighbor_lists(void* h, const dv_fields* f, int64_t* off, int32_t* nbrs, int64_t max_pairs) {
  Ctx* c = (Ctx*)h;
  int64_t k = 0;
  for (int i = range_lo(c); i < range_hi(c); ++i) {
    off[i] = k;
    for_all_neighbors(*c, f->x, i, [&](int j, V) {
      if (nbrs && k < max_pairs) nbrs[k] = j;
      ++k;
    });
  }
  off[c->cnt.n] = k;
  return k;
}

// ------------------------------------------------------------------- SPH
// compute_static_boundary_volume (sph_base.py:91-103)
// compute_static_boundary_volume (sph_base.py:91-98) and, for the dynamic
// solids, compute_moving_boundary_volume (:105-112)
static int boundary_volume(void* h, dv_fields* f, bool dynamic) {
  Ctx* c = (Ctx*)h;
  const dv_params& P = c->p;
#pragma omp parallel for schedule(static)
  for (int i = range_lo(c); i < range_hi(c); ++i) {
    if (!(f->material[i] == DV_MATERIAL_SOLID && (f->is_dynamic[i] != 0) == dynamic)) continue;
    float delta = cubic_kernel(P, 0.0f);
    V xi = ldv(*c, f->x, i);
    for_all_neighbors(*c, f->x, i, [&](int j, V) {
      if (f->material[j] == DV_MATERIAL_SOLID) {
        V xj = ldv(*c, f->x, j);
        V r = rel(*c, xi, xj);
        delta += cubic_kernel(P, std::sqrt(norm_sqr(*c, r)));
      }
    });
    f->m_V[i] = 1.0f / delta * 3.0f;
  }
  return 0;
}

DVO_API int dvo_boundary_volume(void* h, dv_fields* f) { return boundary_volume(h, f, false); }
DVO_API int dvo_moving_boundary_volume(void* h, dv_fields* f) { return boundary_volume(h, f, true); }
DVO_API void dvo_set_dynamic_rigid(void* h, int on) { ((Ctx*)h)->dyn_rigid = on != 0; }

// the reaction of one pressure iteration on the dynamic solids
// (dimcv_sph.py:540-549): -vel_change * inv_dt * rho_fluid / rho_solid from
// every fluid neighbour, gathered per solid in its neighbour visit order
static void rigid_reaction(Ctx* c, dv_fields* f) {
  const dv_params& P = c->p;
  const float dt = P.dt;
#pragma omp parallel for schedule(static)
  for (int i = range_lo(c); i < range_hi(c); ++i) {
    if (!(f->material[i] == DV_MATERIAL_SOLID && f->is_dynamic[i])) continue;
    const float rho_j = f->density[i];
    const float s = f->m_V[i] * P.density0;
    V acc = ldv(*c, f->acceleration, i);
    for_all_neighbors(*c, f->x, i, [&](int q, V r) {  // r = x_i - x_q
      if (f->material[q] != DV_MATERIAL_FLUID) return;
      const float k_q = (f->density_adv[q] - P.density0) * f->dfsph_factor[q];
      if (!(std::fabs(k_q) > P.m_eps)) return;
      V g = cubic_kernel_derivative(*c, V{-r.x, -r.y, -r.z});  // at x_q - x_i, as in q's task
      V gp{s * g.x, s * g.y, s * g.z};
      const float vc0 = -dt * 1.0f * k_q;
      V vc{vc0 * gp.x, vc0 * gp.y, vc0 * gp.z};
      const float rq = f->density[q];
      acc.x += -vc.x * P.inv_dt * rq / rho_j;
      acc.y += -vc.y * P.inv_dt * rq / rho_j;
      acc.z += -vc.z * P.inv_dt * rq / rho_j;
    });
    stv(*c, f->acceleration, i, acc);
  }
}

// compute_densities (dimcv_sph.py:126-148)
DVO_API int dvo_densities(void* h, dv_fields* f) {
  Ctx* c = (Ctx*)h;
  const dv_params& P = c->p;
#pragma omp parallel for schedule(static)
  for (int i = range_lo(c); i < range_hi(c); ++i) {
    if (f->material[i] != DV_MATERIAL_FLUID) continue;
    float d = f->m_V[i] * cubic_kernel(P, 0.0f);
    float den = 0.0f;
    for_all_neighbors(*c, f->x, i, [&](int j, V r) {
      if (f->material[j] == DV_MATERIAL_FLUID || f->material[j] == DV_MATERIAL_SOLID)
        den += f->m_V[j] * cubic_kernel(P, std::sqrt(norm_sqr(*c, r)));
    });
    d += den;
    d *= P.density0;
    f->density[i] = d;
  }
  return 0;
}

// compute_DFSPH_factor (dimcv_sph.py:86-124)
DVO_API int dvo_dfsph_factor(void* h, dv_fields* f) {
  Ctx* c = (Ctx*)h;
  const dv_params& P = c->p;
#pragma omp parallel for schedule(static)
  for (int i = range_lo(c); i < range_hi(c); ++i) {
    if (f->material[i] != DV_MATERIAL_FLUID) continue;
    V gi;
    float sum_grad_p_k = 0.0f;
    for_all_neighbors(*c, f->x, i, [&](int j, V r) {
      if (f->material[j] == DV_MATERIAL_FLUID) {
        V g = cubic_kernel_derivative(*c, r);
        V gp{f->m[j] * g.x, f->m[j] * g.y, f->m[j] * g.z};
        sum_grad_p_k += norm_sqr(*c, gp);
        gi.x += gp.x; gi.y += gp.y; gi.z += gp.z;
      } else if (f->material[j] == DV_MATERIAL_SOLID) {
        V g = cubic_kernel_derivative(*c, r);
        float s = f->m_V[j] * P.density0;
        gi.x += s * g.x; gi.y += s * g.y; gi.z += s * g.z;
      }
    });
    sum_grad_p_k += norm_sqr(*c, gi);
    f->dfsph_factor[i] = sum_grad_p_k > P.factor_min ? 1.0f / sum_grad_p_k : 0.0f;
  }
  return 0;
}

// multiply_time_step (dimcv_sph.py:395-399)
DVO_API int dvo_scale_factor(void* h, dv_fields* f, float s) {
  Ctx* c = (Ctx*)h;
  for (int i = range_lo(c); i < range_hi(c); ++i)
    if (f->material[i] == DV_MATERIAL_FLUID) f->dfsph_factor[i] *= s;
  return 0;
}

// compute_density_change (dimcv_sph.py:337-374)
DVO_API int dvo_density_change(void* h, dv_fields* f) {
  Ctx* c = (Ctx*)h;
  const dv_params& P = c->p;
#pragma omp parallel for schedule(static)
  for (int i = range_lo(c); i < range_hi(c); ++i) {
    if (f->material[i] != DV_MATERIAL_FLUID) continue;
    V vi = ldv(*c, f->v, i);
    float adv = 0.0f;
    int num = 0;
    for_all_neighbors(*c, f->x, i, [&](int j, V r) {
      V vj = ldv(*c, f->v, j);
      V dv{vi.x - vj.x, vi.y - vj.y, vi.z - vj.z};
      if (f->material[j] == DV_MATERIAL_FLUID)
        adv += f->m_V[j] * dotv(*c, dv, cubic_kernel_derivative(*c, r));
      else if (f->material[j] == DV_MATERIAL_SOLID)
        adv += f->m_V[j] * dotv(*c, dv, cubic_kernel_derivative(*c, r));
      num += 1;
    });
    float da = std::max(adv, 0.0f);
    if (num < P.neighbor_min) da = 0.0f;
    f->density_adv[i] = da;
  }
  return 0;
}

// compute_density_adv (dimcv_sph.py:470-493)
DVO_API int dvo_density_adv(void* h, dv_fields* f) {
  Ctx* c = (Ctx*)h;
  const dv_params& P = c->p;
#pragma omp parallel for schedule(static)
  for (int i = range_lo(c); i < range_hi(c); ++i) {
    if (f->material[i] != DV_MATERIAL_FLUID) continue;
    V vi = ldv(*c, f->v, i);
    float delta = 0.0f;
    for_all_neighbors(*c, f->x, i, [&](int j, V r) {
      V vj = ldv(*c, f->v, j);
      V dv{vi.x - vj.x, vi.y - vj.y, vi.z - vj.z};
      if (f->material[j] == DV_MATERIAL_FLUID)
        delta += f->m[j] * dotv(*c, dv, cubic_kernel_derivative(*c, r));
      else if (f->material[j] == DV_MATERIAL_SOLID)
        delta += f->m_V[j] * P.density0 * dotv(*c, dv, cubic_kernel_derivative(*c, r));
    });
    float da = f->density[i] + P.dt * delta;
    f->density_adv[i] = std::max(da, P.density0);
  }
  return 0;
}

// compute_density_error (dimcv_sph.py:407-419), summed in FP64
DVO_API double dvo_density_error(void* h, dv_fields* f, float offset) {
  Ctx* c = (Ctx*)h;
  const dv_params& P = c->p;
  double s = 0.0;
  for (int i = range_lo(c); i < range_hi(c); ++i) {
    if (f->material[i] != DV_MATERIAL_FLUID) continue;
    if (P.has_transit) {
      V x = ldv(*c, f->x, i);
      s += (double)(transit_weight(P, x.x) * (f->density_adv[i] - offset));
    } else {
      s += (double)(f->density_adv[i] - offset);
    }
  }
  return s;
}

// divergence_solver_iteration_kernel (dimcv_sph.py:421-468)
DVO_API int dvo_divergence_iteration(void* h, dv_fields* f) {
  Ctx* c = (Ctx*)h;
  const dv_params& P = c->p;
  const float dt = P.dt;
#pragma omp parallel for schedule(static)
  for (int i = range_lo(c); i < range_hi(c); ++i) {
    if (f->material[i] != DV_MATERIAL_FLUID) continue;
    float b_i = f->density_adv[i];
    float k_i = b_i * f->dfsph_factor[i] * f->density[i];
    V dv;
    for_all_neighbors(*c, f->x, i, [&](int j, V r) {
      if (f->material[j] == DV_MATERIAL_FLUID) {
        float b_j = f->density_adv[j];
        float k_j = b_j * f->dfsph_factor[j] * f->density[j];
        float k_sum = k_i + k_j;
        if (std::fabs(k_sum) > P.m_eps) {
          V g = cubic_kernel_derivative(*c, r);
          V gp{f->m[j] * g.x, f->m[j] * g.y, f->m[j] * g.z};
          dv.x -= dt * k_sum * gp.x;
          dv.y -= dt * k_sum * gp.y;
          dv.z -= dt * k_sum * gp.z;
        }
      } else if (f->material[j] == DV_MATERIAL_SOLID) {
        if (std::fabs(k_i) > P.m_eps) {
          V g = cubic_kernel_derivative(*c, r);
          float s = f->m_V[j] * P.density0;
          V gp{s * g.x, s * g.y, s * g.z};
          float vc = -dt * 1.0f * k_i;
          dv.x += vc * gp.x;
          dv.y += vc * gp.y;
          dv.z += vc * gp.z;
        }
      }
    });
    V vi = ldv(*c, f->v, i);
    if (P.has_transit) {
      float w = transit_weight(P, ldv(*c, f->x, i).x);
      vi.x += w * dv.x; vi.y += w * dv.y; vi.z += w * dv.z;
    } else {
      vi.x += dv.x; vi.y += dv.y; vi.z += dv.z;
    }
    stv(*c, f->v, i, vi);
  }
  return 0;
}

// pressure_solve_iteration_kernel (dimcv_sph.py:495-549)
DVO_API int dvo_pressure_iteration(void* h, dv_fields* f) {
  Ctx* c = (Ctx*)h;
  const dv_params& P = c->p;
  const float dt = P.dt;
#pragma omp parallel for schedule(static)
  for (int i = range_lo(c); i < range_hi(c); ++i) {
    if (f->material[i] != DV_MATERIAL_FLUID) continue;
    float b_i = f->density_adv[i] - P.density0;
    float k_i = b_i * f->dfsph_factor[i];
    V vi = ldv(*c, f->v, i);
    float w = P.has_transit ? transit_weight(P, ldv(*c, f->x, i).x) : 1.0f;
    for_all_neighbors(*c, f->x, i, [&](int j, V r) {
      if (f->material[j] == DV_MATERIAL_FLUID) {
        float b_j = f->density_adv[j] - P.density0;
        float k_j = b_j * f->dfsph_factor[j];
        float k_sum = k_i + k_j;
        if (std::fabs(k_sum) > P.m_eps) {
          V g = cubic_kernel_derivative(*c, r);
          V gp{f->m[j] * g.x, f->m[j] * g.y, f->m[j] * g.z};
          if (!P.has_transit) {
            vi.x -= dt * k_sum * gp.x; vi.y -= dt * k_sum * gp.y; vi.z -= dt * k_sum * gp.z;
          } else {
            vi.x -= w * dt * k_sum * gp.x; vi.y -= w * dt * k_sum * gp.y; vi.z -= w * dt * k_sum * gp.z;
          }
        }
      } else if (f->material[j] == DV_MATERIAL_SOLID) {
        if (std::fabs(k_i) > P.m_eps) {
          V g = cubic_kernel_derivative(*c, r);
          float s = f->m_V[j] * P.density0;
          V gp{s * g.x, s * g.y, s * g.z};
          float vc0 = -dt * 1.0f * k_i;
          V vc{vc0 * gp.x, vc0 * gp.y, vc0 * gp.z};
          if (!P.has_transit) {
            vi.x += vc.x; vi.y += vc.y; vi.z += vc.z;
          } else {
            vi.x += w * vc.x; vi.y += w * vc.y; vi.z += w * vc.z;
          }
        }
      }
    });
    stv(*c, f->v, i, vi);
  }
  if (c->dyn_rigid) rigid_reaction(c, f);
  return 0;
}

// divergence_solve (dimcv_sph.py:376-393) and divergence_solver_iteration (:591-595)
DVO_API int dvo_divergence_solve(void* h, dv_fields* f, int* iters) {
  Ctx* c = (Ctx*)h;
  const dv_params& P = c->p;
  dvo_density_change(h, f);
  dvo_scale_factor(h, f, P.inv_dt);
  int it = 0;
  double avg = 0.0;
  while (it < 1 || it < P.max_iter_div) {
    dvo_divergence_iteration(h, f);
    dvo_density_change(h, f);
    double err = dvo_density_error(h, f, 0.0f);
    int nf = c->cnt.n_fluid;
    avg = nf > 0 ? err / nf : 0.0;
    it += 1;
    if (c->fixed_div > 0) {
      if (it >= c->fixed_div) break;
      continue;
    }
    if (avg <= P.eta_div || nf == 0) break;
  }
  if (!(avg <= P.eta_div) && it >= P.max_iter_div) c->cnt.status |= DV_WARN_DIV_NOT_CONVERGED;
  dvo_scale_factor(h, f, P.dt);
  c->cnt.iters_div = it;
  c->cnt.err_div = avg;
  if (iters) *iters = it;
  return 0;
}

// pressure_solve (dimcv_sph.py:597-614) and pressure_solve_iteration (:585-589)
DVO_API int dvo_pressure_solve(void* h, dv_fields* f, int* iters) {
  Ctx* c = (Ctx*)h;
  const dv_params& P = c->p;
  dvo_density_adv(h, f);
  dvo_scale_factor(h, f, P.inv_dt2);
  int it = 0;
  double avg = 0.0;
  while (it < 1 || it < P.max_iter_p) {
    dvo_pressure_iteration(h, f);
    dvo_density_adv(h, f);
    double err = dvo_density_error(h, f, P.density0);
    int nf = c->cnt.n_fluid;
    avg = nf > 0 ? err / nf : 0.0;
    it += 1;
    if (c->fixed_p > 0) {
      if (it >= c->fixed_p) break;
      continue;
    }
    if (avg <= P.eta_p || nf == 0) break;
  }
  if (!(avg <= P.eta_p) && it >= P.max_iter_p) c->cnt.status |= DV_WARN_P_NOT_CONVERGED;
  c->cnt.iters_p = it;
  c->cnt.err_p = avg;
  if (iters) *iters = it;
  return 0;
}

// compute_non_pressure_forces (dimcv_sph.py:150-208); the surface tension
// (coefficient 0, :12) and boundary viscosity (0, :182) terms add zero
DVO_API int dvo_nonpressure(void* h, dv_fields* f) {
  Ctx* c = (Ctx*)h;
  const dv_params& P = c->p;
#pragma omp parallel for schedule(static)
  for (int i = range_lo(c); i < range_hi(c); ++i) {
    if (f->material[i] == DV_MATERIAL_SOLID && !f->is_dynamic[i]) {
      stv(*c, f->acceleration, i, V{});
      continue;
    }
    V d_v{P.gravity[0], P.gravity[1], c->p.dim == 3 ? P.gravity[2] : 0.0f};
    if (f->material[i] == DV_MATERIAL_FLUID) {
      V vi = ldv(*c, f->v, i);
      for_all_neighbors(*c, f->x, i, [&](int j, V r) {
        if (f->material[j] != DV_MATERIAL_FLUID) return;
        V vj = ldv(*c, f->v, j);
        float v_xy = dotv(*c, V{vi.x - vj.x, vi.y - vj.y, vi.z - vj.z}, r);
        float rn = std::sqrt(norm_sqr(*c, r));
        float s = P.visc_coef * f->m_V[j] * v_xy / (rn * rn + P.visc_h2);
        V g = cubic_kernel_derivative(*c, r);
        d_v.x += s * g.x; d_v.y += s * g.y; d_v.z += s * g.z;
      });
    }
    stv(*c, f->acceleration, i, d_v);
  }
  return 0;
}

DVO_API int dvo_predict_velocity(void* h, dv_fields* f) {  // dimcv_sph.py:220-226
  Ctx* c = (Ctx*)h;
  for (int i = range_lo(c); i < range_hi(c); ++i) {
    if (!(f->is_dynamic[i] && f->material[i] == DV_MATERIAL_FLUID)) continue;
    V v = ldv(*c, f->v, i), a = ldv(*c, f->acceleration, i);
    v.x += c->p.dt * a.x; v.y += c->p.dt * a.y; v.z += c->p.dt * a.z;
    stv(*c, f->v, i, v);
  }
  return 0;
}

// enforce_boundary_2D / _3D + simulate_collisions (sph_base.py:118-179):
// all `cap` slots, as the reference's ti.grouped(x) loop over the field
DVO_API int dvo_enforce_boundary(void* h, dv_fields* f, int material, const float* lo, const float* hi) {
  Ctx* c = (Ctx*)h;
  const int D = c->p.dim;
  for (int64_t i = 0; i < c->cap; ++i) {
    if (!(f->material[i] == material && f->is_dynamic[i])) continue;
    const V pos = ldv(*c, f->x, (int)i);
    V x = pos, n;
    const float p[3] = {pos.x, pos.y, pos.z};
    float* xs[3] = {&x.x, &x.y, &x.z};
    float* ns[3] = {&n.x, &n.y, &n.z};
    for (int d = 0; d < D; ++d) {
      if (p[d] > hi[d]) { *ns[d] += 1.0f; *xs[d] = hi[d]; }
      if (p[d] <= lo[d]) { *ns[d] += -1.0f; *xs[d] = lo[d]; }
    }
    stv(*c, f->x, (int)i, x);
    const float len = std::sqrt(norm_sqr(*c, n));
    if (len > 1.0e-6f) {
      const V e{n.x / len, n.y / len, D == 3 ? n.z / len : 0.0f};
      V v = ldv(*c, f->v, (int)i);
      const float s = (1.0f + 0.5f) * dotv(*c, v, e);  // c_f = 0.5 (sph_base.py:121)
      v.x -= s * e.x;
      v.y -= s * e.y;
      if (D == 3) v.z -= s * e.z;
      stv(*c, f->v, (int)i, v);
    }
  }
  return 0;
}

DVO_API int dvo_advect(void* h, dv_fields* f) {  // dimcv_sph.py:210-218
  Ctx* c = (Ctx*)h;
  const float dt = c->p.dt;
  for (int i = range_lo(c); i < range_hi(c); ++i) {
    if (!f->is_dynamic[i]) continue;
    V v = ldv(*c, f->v, i);
    if (f->material[i] == DV_MATERIAL_SOLID) {
      V a = ldv(*c, f->acceleration, i);
      v.x += dt * a.x; v.y += dt * a.y; v.z += dt * a.z;
      stv(*c, f->v, i, v);
    }
    V x = ldv(*c, f->x, i);
    x.x += dt * v.x; x.y += dt * v.y; x.z += dt * v.z;
    if (c->p.periodic) {
      float* cs[3] = {&x.x, &x.y, &x.z};
      for (int d = 0; d < c->p.dim; ++d) {
        if (*cs[d] >= c->p.domain_start[d] + c->p.box[d]) *cs[d] -= c->p.box[d];
        if (*cs[d] < c->p.domain_start[d]) {
          *cs[d] += c->p.box[d];
          // -tiny + box rounds to box: that point is the start of the axis
          if (*cs[d] >= c->p.domain_start[d] + c->p.box[d]) *cs[d] = c->p.domain_start[d];
        }
      }
    }
    stv(*c, f->x, i, x);
  }
  return 0;
}

// ----------------------------------------------------------------- DIMCV
// compute_v_star, compute_vorticity, compute_grad_v (dimcv_sph.py:228-293)
DVO_API int dvo_dimcv_vorticity(void* h, dv_fields* f, dv_solver_fields* s) {
  Ctx* c = (Ctx*)h;
  const dv_params& P = c->p;
  const int D = P.dim, DD = D * D;
#pragma omp parallel for schedule(static)
  for (int i = range_lo(c); i < range_hi(c); ++i) {
    if (f->material[i] != DV_MATERIAL_FLUID) {
      stv(*c, s->v_star, i, V{});
      st4(f->vorticity, i, V{});
      for (int k = 0; k < DD; ++k) s->grad_v[(int64_t)i * DD + k] = 0.0f;
      continue;
    }
    V vi = ldv(*c, f->v, i), ai = ldv(*c, f->acceleration, i);
    stv(*c, s->v_star, i, V{vi.x + ai.x * P.dt, vi.y + ai.y * P.dt, vi.z + ai.z * P.dt});
    V vort;
    float g[9] = {0};
    for_all_neighbors(*c, f->x, i, [&](int j, V r) {
      if (f->material[j] != DV_MATERIAL_FLUID) return;
      V vj = ldv(*c, f->v, j);
      V kd = cubic_kernel_derivative(*c, r);
      V cr = cross(V{vj.x - vi.x, vj.y - vi.y, vj.z - vi.z}, kd);
      float mv = f->m_V[j];
      vort.x += mv * cr.x; vort.y += mv * cr.y; vort.z += mv * cr.z;
      float vji[3] = {vj.x - vi.x, vj.y - vi.y, vj.z - vi.z};
      float kg[3] = {kd.x, kd.y, kd.z};
      for (int a = 0; a < D; ++a)
        for (int b = 0; b < D; ++b) g[a * D + b] += mv * vji[a] * kg[b];
    });
    st4(f->vorticity, i, vort);
    for (int k = 0; k < DD; ++k) s->grad_v[(int64_t)i * DD + k] = g[k];
  }
  return 0;
}

// compute_d_vorticity (dimcv_sph.py:551-583)
DVO_API int dvo_d_vorticity(void* h, dv_fields* f, dv_solver_fields* s) {
  Ctx* c = (Ctx*)h;
#pragma omp parallel for schedule(static)
  for (int i = range_lo(c); i < range_hi(c); ++i) {
    if (f->material[i] != DV_MATERIAL_FLUID) {
      st4(s->d_vort, i, V{});
      continue;
    }
    V vsi = ldv(*c, s->v_star, i);
    V curl;
    for_all_neighbors(*c, f->x, i, [&](int j, V r) {
      if (f->material[j] != DV_MATERIAL_FLUID) return;
      V vsj = ldv(*c, s->v_star, j);
      V cr = cross(V{vsj.x - vsi.x, vsj.y - vsi.y, vsj.z - vsi.z}, cubic_kernel_derivative(*c, r));
      float mv = f->m_V[j];
      curl.x += mv * cr.x; curl.y += mv * cr.y; curl.z += mv * cr.z;
    });
    V w = ld4(f->vorticity, i);
    st4(s->d_vort, i, V{w.x - curl.x, w.y - curl.y, w.z - curl.z});
  }
  return 0;
}

// compute_all_d_vort_smoothed (dimcv_sph.py:660-677)
DVO_API int dvo_smooth_d_vort(void* h, dv_fields* f, dv_solver_fields* s) {
  Ctx* c = (Ctx*)h;
  const dv_params& P = c->p;
#pragma omp parallel for schedule(static)
  for (int i = range_lo(c); i < range_hi(c); ++i) {
    if (f->material[i] != DV_MATERIAL_FLUID || !in_vortex_domain(*c, ldv(*c, f->x, i))) continue;
    V di = ld4(s->d_vort, i);
    float w0 = cubic_kernel(P, 0.0f);
    V acc{f->m_V[i] * di.x * w0, f->m_V[i] * di.y * w0, f->m_V[i] * di.z * w0};
    for_all_neighbors(*c, f->x, i, [&](int j, V r) {
      if (f->material[j] != DV_MATERIAL_FLUID) return;
      V dj = ld4(s->d_vort, j);
      float wk = cubic_kernel(P, std::sqrt(norm_sqr(*c, r)));
      acc.x += f->m_V[j] * dj.x * wk; acc.y += f->m_V[j] * dj.y * wk; acc.z += f->m_V[j] * dj.z * wk;
    });
    st4(s->d_vort_smoothed, i, acc);
  }
  return 0;
}

// compute_kinematic_vorticity_num_sample (dimcv_sph.py:295-324)
DVO_API int dvo_kvn_sample(void* h, dv_fields* f, dv_solver_fields* s, uint64_t seed, uint64_t step,
                           int birth_death) {
  Ctx* c = (Ctx*)h;
  const dv_params& P = c->p;
  const int D = P.dim;
  for (int i = range_lo(c); i < range_hi(c); ++i) {
    if (f->material[i] != DV_MATERIAL_FLUID || !in_vortex_domain(*c, ldv(*c, f->x, i))) continue;
    const float* g = s->grad_v + (int64_t)i * D * D;
    float wn = 0, sn = 0;
    bool first = true;
    for (int a = 0; a < D; ++a)
      for (int b = 0; b < D; ++b) {
        float wv = g[a * D + b] - g[b * D + a];
        float sv = g[a * D + b] + g[b * D + a];
        if (first) {
          wn = wv * wv;
          sn = sv * sv;
          first = false;
        } else {
          wn = wn + wv * wv;
          sn = sn + sv * sv;
        }
      }
    float kvn = std::sqrt(wn) / (std::sqrt(sn) + P.kvn_eps);
    s->kvn[i] = kvn;
    if (!birth_death) continue;
    float t0 = std::min(std::max(f->life_time[i], 0.0f), 1.0f);
    float r = 0.018f * std::exp(-P.gen_a * t0) + 0.004f;
    float produce = 1.0f - 1.0f / std::pow(kvn + 1.0f, r);
    float del = std::exp(-P.del_b * kvn);
    uint32_t o[4];
    philox((uint32_t)i, 0u, (uint32_t)step, (uint32_t)(step >> 32), (uint32_t)seed, (uint32_t)(seed >> 32), o);
    float u1 = (float)(o[0] >> 8) * (1.0f / 16777216.0f);
    float u2 = (float)(o[1] >> 8) * (1.0f / 16777216.0f);
    if (f->is_sample[i] == 0 && u1 < produce)
      f->is_sample[i] = 1;
    else if (f->is_sample[i] == 1 && kvn < 2.0f && u2 < del)
      f->is_sample[i] = 0;
  }
  return 0;
}

// record_vort_part_sample_idx (dimcv_sph.py:326-335), ascending slot order
DVO_API int dvo_record_samples(void* h, dv_fields* f, dv_solver_fields* s) {
  Ctx* c = (Ctx*)h;
  int m = 0;
  for (int p = 0; p < c->cnt.n; ++p)
    if (f->is_sample[p] == 1) s->sample_idx[m++] = p;
  c->cnt.num_samples = m;
  return 0;
}

// epanechnikov_kernel (dimcv_sph.py:721-730)
static float epanechnikov(const Ctx& c, V r) {
  float ret = 1.0f;
  float rc[3] = {r.x, r.y, r.z};
  for (int i = 0; i < c.p.dim; ++i) {
    float q = std::fabs(rc[i]) * c.p.inv_support_radius;
    if (q < 1.0f)
      ret *= 0.75f * (1.0f - q * q);
    else
      ret *= 0.0f;
  }
  return ret;
}

// compute_kernel_density (dimcv_sph.py:732-751)
DVO_API int dvo_akde(void* h, dv_fields* f, dv_solver_fields* s) {
  Ctx* c = (Ctx*)h;
  const int n = c->cnt.n;
  std::vector<double> term(n, 0.0);
#pragma omp parallel for schedule(static)
  for (int i = range_lo(c); i < range_hi(c); ++i) {
    if (f->material[i] != DV_MATERIAL_FLUID || !in_vortex_domain(*c, ldv(*c, f->x, i))) continue;
    float kden = s->kvn[i] * epanechnikov(*c, V{});
    for_all_neighbors(*c, f->x, i, [&](int j, V r) {
      if (f->material[j] == DV_MATERIAL_FLUID) kden += s->kvn[j] * epanechnikov(*c, r);
    });
    s->kden[i] = kden;
    term[i] = kden;
  }
  double sum = 0.0;
  for (int i = 0; i < n; ++i) sum += term[i];
  c->cnt.kden_sum = sum;
  c->cnt.kden_sum_f32 = (float)sum;
  return 0;
}

static void build_targets(Ctx* c, dv_fields* f) {
  c->targets.clear();
  for (int i = range_lo(c); i < range_hi(c); ++i)
    if (f->material[i] == DV_MATERIAL_FLUID && in_vortex_domain(*c, ldv(*c, f->x, i))) c->targets.push_back(i);
  c->cnt.n_targets = (int)c->targets.size();
}

// New sampler: FP64 CDF over targets, M draws, upper_bound - 1 search
DVO_API int dvo_sample(void* h, dv_fields* f, dv_solver_fields* s, int mode, uint64_t seed, uint64_t step, int M) {
  Ctx* c = (Ctx*)h;
  if (mode == DV_SAMPLE_BERNOULLI) return dvo_record_samples(h, f, s);
  if (mode == DV_SAMPLE_INJECTED) {
    c->cnt.num_samples = M;
    return 0;
  }
  build_targets(c, f);
  const int nt = c->cnt.n_targets;
  std::vector<double> cdf(nt);
  double run = 0.0;
  for (int k = 0; k < nt; ++k) {
    cdf[k] = run;
    run += (double)s->kden[c->targets[k]];
  }
  if (nt == 0 || !(run > 0.0)) {
    c->cnt.num_samples = 0;
    return 0;
  }
  for (int q = 0; q < M; ++q) {
    uint32_t o[4];
    philox((uint32_t)q, 2u, (uint32_t)step, (uint32_t)(step >> 32), (uint32_t)seed, (uint32_t)(seed >> 32), o);
    uint64_t mant = ((uint64_t)(o[0] >> 5) << 26) | (uint64_t)(o[1] >> 6);
    double u = (double)mant * (1.0 / 9007199254740992.0);
    if (mode == DV_SAMPLE_STRATIFIED) u = ((double)q + u) / (double)M;  // stratum q of M
    double y = u * run;
    int k = (int)(std::upper_bound(cdf.begin(), cdf.end(), y) - cdf.begin()) - 1;
    if (k < 0) k = 0;
    while (k > 0 && !(s->kden[c->targets[k]] > 0.0f)) --k;
    s->sample_idx[q] = c->targets[k];
  }
  c->cnt.num_samples = M;
  return 0;
}

// vort2vel (dimcv_sph.py:649-719).  precision 32: every pair literally in
// f32 in the reference order; precision 64: the near and far sums in FP64.
template <typename T>
static void vvpe_target(Ctx* c, dv_fields* f, dv_solver_fields* s, int i, bool blob) {
  const dv_params& P = c->p;
  V xi = ldv(*c, f->x, i);
  T nx = 0, ny = 0, nz = 0;
  T S_i = (T)s->kden[i];
  const T eps = (T)P.eps, inv_eps = (T)P.inv_eps;
  for_all_neighbors(*c, f->x, i, [&](int j, V r) {
    if (f->material[j] != DV_MATERIAL_FLUID) return;
    V w = ld4(s->d_vort_smoothed, j);
    if (!blob) {
      T rx = (T)r.x, ry = (T)r.y;
      T rn = std::sqrt(rx * rx + ry * ry + (T)0 * (T)0);
      T e = std::exp(-rn * inv_eps);
      T K = ((T)1 - e) / (rn * (rn + eps * e));
      // cross((rx, ry, 0), w)
      T cx = ry * (T)w.z - (T)0 * (T)w.y, cy = (T)0 * (T)w.x - rx * (T)w.z, cz = rx * (T)w.y - ry * (T)w.x;
      nx += K * cx; ny += K * cy; nz += K * cz;
    } else {
      T rx = (T)r.x, ry = (T)r.y, rz = (T)r.z;
      T r2 = rx * rx + ry * ry + rz * rz;
      T sv = r2 + (T)P.blob_delta2;
      T K = (T)1 / (sv * std::sqrt(sv));
      nx += K * (ry * (T)w.z - rz * (T)w.y);
      ny += K * (rz * (T)w.x - rx * (T)w.z);
      nz += K * (rx * (T)w.y - ry * (T)w.x);
    }
    S_i += (T)s->kden[j];
  });
  const T coef = blob ? (T)P.blob_coef : (T)P.vvpe_coef;
  nx *= coef; ny *= coef; nz *= coef;
  T fx = 0, fy = 0, fz = 0;
  int added = 0;
  const T ksum = (T)c->cnt.kden_sum_f32;
  for (int q = 0; q < c->cnt.num_samples; ++q) {
    int j = s->sample_idx[q];
    V xj = ldv(*c, f->x, j);
    V r32 = rel(*c, xi, xj);
    float rn32 = std::sqrt(norm_sqr(*c, r32));
    if (!(rn32 > P.support_radius)) continue;  // dimcv_sph.py:700
    V w = ld4(s->d_vort_smoothed, j);
    T rx = (T)r32.x, ry = (T)r32.y, rz = (T)r32.z;
    T fac = (ksum - S_i) / ((T)s->kden[j] + (T)P.kden_eps);
    if (!blob) {
      T rn = (T)rn32;
      if (sizeof(T) == 8) rn = std::sqrt(rx * rx + ry * ry + rz * rz);
      T e = std::exp(-rn * inv_eps);
      T K = ((T)1 - e) / (rn * (rn + eps * e));
      T cx = ry * (T)w.z - (T)0 * (T)w.y, cy = (T)0 * (T)w.x - rx * (T)w.z, cz = rx * (T)w.y - ry * (T)w.x;
      fx += K * cx * (ksum - S_i) / ((T)s->kden[j] + (T)P.kden_eps);
      fy += K * cy * (ksum - S_i) / ((T)s->kden[j] + (T)P.kden_eps);
      fz += K * cz * (ksum - S_i) / ((T)s->kden[j] + (T)P.kden_eps);
    } else {
      T r2 = rx * rx + ry * ry + rz * rz;
      T sv = r2 + (T)P.blob_delta2;
      T K = (T)1 / (sv * std::sqrt(sv));
      fx += K * (ry * (T)w.z - rz * (T)w.y) * fac;
      fy += K * (rz * (T)w.x - rx * (T)w.z) * fac;
      fz += K * (rx * (T)w.y - ry * (T)w.x) * fac;
    }
    added += 1;
  }
  if (added == 0) {
    fx = fy = fz = 0;
  } else {
    T sc = coef / (T)added;
    fx *= sc; fy *= sc; fz *= sc;
  }
  T vx = fx + nx, vy = fy + ny, vz = fz + nz;
  if (s->v_vort) st4(s->v_vort, i, V{(float)vx, (float)vy, (float)vz});
  V vi = ldv(*c, f->v, i);
  T n1 = std::sqrt(vx * vx + vy * vy + vz * vz);
  T n2 = std::sqrt((T)norm_sqr(*c, vi));
  if (n1 < n2) {
    vi.x = (float)((T)vi.x + vx);
    vi.y = (float)((T)vi.y + vy);
    if (P.dim == 3) vi.z = (float)((T)vi.z + vz);
    stv(*c, f->v, i, vi);
  }
}

DVO_API int dvo_vvpe_mc(void* h, dv_fields* f, dv_solver_fields* s, int precision) {
  Ctx* c = (Ctx*)h;
  build_targets(c, f);
  const bool blob = c->p.kernel_mode == DV_KERNEL_BLOB3D;
  const int nt = c->cnt.n_targets;
  // all targets read v only of themselves: safe to run in parallel
#pragma omp parallel for schedule(dynamic, 64)
  for (int k = 0; k < nt; ++k) {
    if (precision == 64)
      vvpe_target<double>(c, f, s, c->targets[k], blob);
    else
      vvpe_target<float>(c, f, s, c->targets[k], blob);
  }
  return 0;
}

// the full Biot-Savart comparator: Σ_{fluid j != i} kernel (r × ω_j)
DVO_API int dvo_bs_full(void* h, dv_fields* f, const float* omega, const int32_t* targets, int nt,
                        double* out) {
  Ctx* c = (Ctx*)h;
  const dv_params& P = c->p;
  const bool blob = P.kernel_mode == DV_KERNEL_BLOB3D;
  std::vector<int> src;
  for (int j = 0; j < c->cnt.n; ++j)
    if (f->material[j] == DV_MATERIAL_FLUID) src.push_back(j);
#pragma omp parallel for schedule(dynamic, 16)
  for (int t = 0; t < nt; ++t) {
    int i = targets ? targets[t] : t;
    V xi = ldv(*c, f->x, i);
    double ax = 0, ay = 0, az = 0;
    for (int j : src) {
      if (j == i) continue;
      V xj = ldv(*c, f->x, j);
      double dx = (double)xi.x - xj.x, dy = (double)xi.y - xj.y, dz = P.dim == 3 ? (double)xi.z - xj.z : 0.0;
      if (P.periodic) {
        const double L0 = P.box[0], L1 = P.box[1], L2 = P.box[2];
        dx = dx > L0 / 2 ? dx - L0 : (dx < -L0 / 2 ? dx + L0 : dx);
        dy = dy > L1 / 2 ? dy - L1 : (dy < -L1 / 2 ? dy + L1 : dy);
        if (P.dim == 3) dz = dz > L2 / 2 ? dz - L2 : (dz < -L2 / 2 ? dz + L2 : dz);
      }
      double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 == 0.0) continue;
      const float* w = omega + 4 * (int64_t)j;
      if (!blob) {
        double rn = std::sqrt(r2);
        double e = std::exp(-rn * (double)P.inv_eps);
        double K = (1.0 - e) / (rn * (rn + (double)P.eps * e));
        ax += K * (dy * w[2]);
        ay -= K * (dx * w[2]);
        az += K * (dx * w[1] - dy * w[0]);
      } else {
        double sv = r2 + (double)P.blob_delta2;
        double K = 1.0 / (sv * std::sqrt(sv));
        ax += K * (dy * w[2] - dz * w[1]);
        ay += K * (dz * w[0] - dx * w[2]);
        az += K * (dx * w[1] - dy * w[0]);
      }
    }
    double coef = blob ? (double)P.blob_coef : (double)P.vvpe_coef;
    out[4 * (int64_t)t] = ax * coef;
    out[4 * (int64_t)t + 1] = ay * coef;
    out[4 * (int64_t)t + 2] = az * coef;
    out[4 * (int64_t)t + 3] = 0.0;
  }
  return 0;
}

// update_particle_life_time (dimcv_sph.py:753-760)
DVO_API int dvo_life_time(void* h, dv_fields* f) {
  Ctx* c = (Ctx*)h;
  for (int p = range_lo(c); p < range_hi(c); ++p)
    if (f->material[p] == DV_MATERIAL_FLUID && in_vortex_domain(*c, ldv(*c, f->x, p))) f->life_time[p] += c->p.dt;
  return 0;
}

// copy_x_temp + compute_vorticity_vis (dimcv_sph.py:778-801)
DVO_API int dvo_vis(void* h, dv_fields* f, dv_solver_fields* s) {
  Ctx* c = (Ctx*)h;
  const dv_params& P = c->p;
#pragma omp parallel for schedule(static)
  for (int i = range_lo(c); i < range_hi(c); ++i) {
    stv(*c, s->x_temp, i, ldv(*c, f->x, i));
    if (f->material[i] != DV_MATERIAL_FLUID) {
      st4(s->vorticity_vis, i, V{});
      continue;
    }
    float w = f->m_V[i] * cubic_kernel(P, 0.0f);
    V wi = ld4(f->vorticity, i);
    V vort{w * wi.x, w * wi.y, w * wi.z};
    float ws = w;
    for_all_neighbors(*c, f->x, i, [&](int j, V r) {
      float wj = f->m_V[j] * cubic_kernel(P, std::sqrt(norm_sqr(*c, r)));
      V oj = ld4(f->vorticity, j);
      vort.x += wj * oj.x; vort.y += wj * oj.y; vort.z += wj * oj.z;
      ws += wj;
    });
    float den = ws + 1e-6f;
    st4(s->vorticity_vis, i, V{vort.x / den, vort.y / den, vort.z / den});
  }
  return 0;
}
