// Neighbour grid of the DIMCV-SPH substep (reference: ParticleSystem,
// particle_system.py:382-586): activity update, compaction + cell sort as a
// stable LSD radix sort on Morton cell keys (every pass is an atomic-free
// counting sort: warp-level __match_any_sync ranks, per-tile digit counts,
// a device-wide exclusive scan, stable scatter), the cell table, the
// permutation of all particle fields, emission and CSR neighbour lists.
#include <algorithm>

#include "dv_internal.cuh"

// ------------------------------------------------------------ activity
// update_activity (particle_system.py:413-427): solids are forced active,
// fluid outside [domain_start, domain_end] (strict) becomes inactive.  The
// fluid count is recomputed from the compaction (dv_grid_build).
// In a scene batch (scene_end != NULL) the box of slot i ends at
// scene_end[3 * object_id[i]].
template <int D>
__global__ void k_update_activity(dv_params P, dv_fields F, const dv_counters* __restrict__ C,
                                  const float* __restrict__ scene_end) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= C->n) return;
  int mat = F.material[i];
  if (mat == DV_MATERIAL_SOLID) {
    F.is_active[i] = 1;
  } else if (mat == DV_MATERIAL_FLUID && !P.periodic) {  // nothing leaves a periodic box
    V3 x = ldv<D>(F.x, i);
    float e0 = P.domain_end[0], e1 = P.domain_end[1], e2 = P.domain_end[2];
    if (scene_end) {
      const int s = F.object_id[i];
      if (s < 0 || s >= P.n_scenes) return;
      e0 = scene_end[3 * s];
      e1 = scene_end[3 * s + 1];
      e2 = scene_end[3 * s + 2];
    }
    bool out = x.x < P.domain_start[0] || x.x > e0 || x.y < P.domain_start[1] || x.y > e1;
    if (D == 3) out = out || x.z < P.domain_start[2] || x.z > e2;
    if (out) F.is_active[i] = 0;
  }
}

DV_API int dv_update_activity(dv_ctx* c, const dv_fields* f) {
  if (!c || !f) return DV_EINVAL;
  int nb = dv_blocks(c->n_upper);
  const float* se = c->p.n_scenes > 1 ? c->d_scene_end : nullptr;
  if (c->p.n_scenes > 1 && !se) return dv_fail(c, DV_EINVAL, "scene batch without scene table");
  if (c->p.dim == 2)
    k_update_activity<2><<<nb, DV_THREADS, 0, c->stream>>>(c->p, *f, c->d_cnt, se);
  else
    k_update_activity<3><<<nb, DV_THREADS, 0, c->stream>>>(c->p, *f, c->d_cnt, se);
  DV_LAUNCHED(c);
  return DV_OK;
}

// ------------------------------------------------------------- cell keys
// Morton key of the particle's cell; inactive particles get the all-ones key
// of kbits bits so that they sort behind every cell (this fuses
// particle_partition, which is order-preserving, into the stable sort).
template <int D>
__global__ void k_cell_keys(dv_params P, dv_fields F, DevGrid G, dv_counters* C, uint32_t* keys,
                            uint32_t invalid, const int32_t* __restrict__ scene, int shift) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int n = C->n;
  if (i >= n) return;
  uint32_t key = invalid;
  if (F.is_active[i]) {
    V3 x = ldv<D>(F.x, i);
    int c0 = cell_coord(P, x.x, 0), c1 = cell_coord(P, x.y, 1), c2 = D == 3 ? cell_coord(P, x.z, 2) : 0;
    bool outside = c0 < 0 || c0 >= P.grid_num[0] || c1 < 0 || c1 >= P.grid_num[1] ||
                   (D == 3 && (c2 < 0 || c2 >= P.grid_num[2]));
    if (outside) {
      // undefined in the reference (out-of-range field index); clamped here
      atomicOr(&C->status, DV_WARN_OUTSIDE_GRID);
      c0 = min(max(c0, 0), P.grid_num[0] - 1);
      c1 = min(max(c1, 0), P.grid_num[1] - 1);
      if (D == 3) c2 = min(max(c2, 0), P.grid_num[2] - 1);
    }
    key = G.mt0[c0] | G.mt1[c1];
    if (D == 3) key |= G.mt2[c2];
    if (scene) key |= (uint32_t)scene[i] << shift;  // scene batch: scene-major cell order
  }
  keys[i] = key;
}

// ------------------------------------------------------------ radix sort
#define RS_T 256
#define RS_W (RS_T / 32)
#define RS_R 8
#define RS_TILE (RS_T * RS_R)

// per-tile digit counts, digit-major: hist[d * ntiles + tile]
__global__ void __launch_bounds__(RS_T) k_rs_hist(const uint32_t* __restrict__ keys,
                                                  const dv_counters* __restrict__ C, int shift,
                                                  int ntiles, uint32_t* __restrict__ hist) {
  __shared__ uint32_t s_cnt[RS_W][256];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int n = C->n;
  for (int k = tid; k < RS_W * 256; k += RS_T) (&s_cnt[0][0])[k] = 0;
  __syncthreads();
  const int base = blockIdx.x * RS_TILE;
  for (int r = 0; r < RS_R; ++r) {
    int e = base + r * RS_T + tid;
    bool valid = e < n;
    uint32_t dig = valid ? ((keys[e] >> shift) & 255u) : 256u;
    unsigned peers = __match_any_sync(0xffffffffu, dig);
    int leader = __ffs(peers) - 1;
    if (valid && lane == leader) s_cnt[warp][dig] += __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  uint32_t tot = 0;
  for (int w = 0; w < RS_W; ++w) tot += s_cnt[w][tid];
  hist[(int64_t)tid * ntiles + blockIdx.x] = tot;
}

// stable scatter: element order inside a tile is (round, warp, lane)
__global__ void __launch_bounds__(RS_T) k_rs_scatter(const uint32_t* __restrict__ kin,
                                                     const uint32_t* __restrict__ vin,
                                                     uint32_t* __restrict__ kout,
                                                     uint32_t* __restrict__ vout,
                                                     const dv_counters* __restrict__ C, int shift,
                                                     int ntiles, const uint32_t* __restrict__ offs) {
  __shared__ uint32_t s_cnt[RS_W][256];
  __shared__ uint32_t s_base[256];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int n = C->n;
  for (int k = tid; k < RS_W * 256; k += RS_T) (&s_cnt[0][0])[k] = 0;
  s_base[tid] = offs[(int64_t)tid * ntiles + blockIdx.x];
  __syncthreads();
  const int base = blockIdx.x * RS_TILE;
  const unsigned lt = (1u << lane) - 1u;
  for (int r = 0; r < RS_R; ++r) {
    int e = base + r * RS_T + tid;
    bool valid = e < n;
    uint32_t key = valid ? kin[e] : 0u;
    uint32_t val = valid ? (vin ? vin[e] : (uint32_t)e) : 0u;
    uint32_t dig = valid ? ((key >> shift) & 255u) : 256u;
    unsigned peers = __match_any_sync(0xffffffffu, dig);
    int rank = __popc(peers & lt);
    int leader = __ffs(peers) - 1;
    if (valid && lane == leader) s_cnt[warp][dig] = __popc(peers);
    __syncthreads();
    {  // thread d turns the per-warp counts of digit d into offsets
      uint32_t run = s_base[tid];
      for (int w = 0; w < RS_W; ++w) {
        uint32_t cnt = s_cnt[w][tid];
        s_cnt[w][tid] = run;
        run += cnt;
      }
      s_base[tid] = run;
    }
    __syncthreads();
    if (valid) {
      uint32_t pos = s_cnt[warp][dig] + (uint32_t)rank;
      kout[pos] = key;
      vout[pos] = val;
    }
    __syncthreads();
    for (int w = 0; w < RS_W; ++w) s_cnt[w][tid] = 0;
    __syncthreads();
  }
}

// cell table from sorted keys; n_new = number of valid keys
__global__ void k_cell_ranges(const uint32_t* __restrict__ keys, const dv_counters* __restrict__ C,
                              uint32_t invalid, int32_t* __restrict__ cstart,
                              int32_t* __restrict__ cend, int32_t* __restrict__ n_new_out) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  const int n_old = C->n;  // the sorted range; keys past it are stale
  if (p >= n_old) return;
  uint32_t k = keys[p];
  if (k == invalid) return;
  uint32_t kp = p > 0 ? keys[p - 1] : 0xffffffffu;
  uint32_t kn = p + 1 < n_old ? keys[p + 1] : invalid;
  if (p == 0 || kp != k) cstart[k] = p;
  if (kn != k) cend[k] = p + 1;
  if (kn == invalid) *n_new_out = p + 1;
}

// Gathers every dv_fields array into the new order; counts fluid / solid
// per block (deterministic partials).  Slots in [n_new, n_old) receive the
// reference's partition fill values (particle_system.py:455-465) for the
// filled fields and keep their own values for the others.
template <int D>
__global__ void k_permute(dv_fields S, dv_fields T, const uint32_t* __restrict__ perm,
                          const uint32_t* __restrict__ keys, const int32_t* __restrict__ n_new_p,
                          int n_old_cap, const dv_counters* __restrict__ C,
                          int32_t* __restrict__ part) {
  const int VS = D == 2 ? 2 : 4;
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  int n_old = C->n, n_new = *n_new_p;
  int fl = 0, so = 0;
  if (p < n_new) {
    int j = (int)perm[p];
    if (D == 2) {
      reinterpret_cast<float2*>(T.x)[p] = reinterpret_cast<const float2*>(S.x)[j];
      reinterpret_cast<float2*>(T.x0)[p] = reinterpret_cast<const float2*>(S.x0)[j];
      reinterpret_cast<float2*>(T.v)[p] = reinterpret_cast<const float2*>(S.v)[j];
      reinterpret_cast<float2*>(T.acceleration)[p] = reinterpret_cast<const float2*>(S.acceleration)[j];
    } else {
      reinterpret_cast<float4*>(T.x)[p] = reinterpret_cast<const float4*>(S.x)[j];
      reinterpret_cast<float4*>(T.x0)[p] = reinterpret_cast<const float4*>(S.x0)[j];
      reinterpret_cast<float4*>(T.v)[p] = reinterpret_cast<const float4*>(S.v)[j];
      reinterpret_cast<float4*>(T.acceleration)[p] = reinterpret_cast<const float4*>(S.acceleration)[j];
    }
    reinterpret_cast<float4*>(T.vorticity)[p] = reinterpret_cast<const float4*>(S.vorticity)[j];
    reinterpret_cast<int4*>(T.color)[p] = reinterpret_cast<const int4*>(S.color)[j];
    T.m_V[p] = S.m_V[j];
    T.m[p] = S.m[j];
    T.density[p] = S.density[j];
    T.pressure[p] = S.pressure[j];
    T.dfsph_factor[p] = S.dfsph_factor[j];
    T.density_adv[p] = S.density_adv[j];
    T.life_time[p] = S.life_time[j];
    int mat = S.material[j];
    T.material[p] = mat;
    T.object_id[p] = S.object_id[j];
    T.grid_ids[p] = (int32_t)keys[p];
    T.is_dynamic[p] = S.is_dynamic[j];
    T.is_active[p] = S.is_active[j];
    T.is_sample[p] = S.is_sample[j];
    fl = mat == DV_MATERIAL_FLUID;
    so = mat == DV_MATERIAL_SOLID;
  } else if (p < n_old && p < n_old_cap) {
    for (int d = 0; d < VS; ++d) {
      T.x[p * VS + d] = -1.0f;
      T.x0[p * VS + d] = -1.0f;
      T.v[p * VS + d] = 0.0f;
      T.acceleration[p * VS + d] = 0.0f;
    }
    reinterpret_cast<float4*>(T.vorticity)[p] = reinterpret_cast<const float4*>(S.vorticity)[p];
    reinterpret_cast<int4*>(T.color)[p] = make_int4(255, 255, 255, 255);
    T.m_V[p] = S.m_V[p];
    T.m[p] = S.m[p];
    T.density[p] = S.density[p];
    T.pressure[p] = S.pressure[p];
    T.dfsph_factor[p] = S.dfsph_factor[p];
    T.density_adv[p] = S.density_adv[p];
    T.life_time[p] = 0.0f;
    T.material[p] = S.material[p];
    T.object_id[p] = -1;
    T.grid_ids[p] = -1;
    T.is_dynamic[p] = 0;
    T.is_active[p] = 0;
    T.is_sample[p] = 0;
  }
  int sfl = block_sum<int>(fl);
  int sso = block_sum<int>(so);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = sfl;
    part[2 * blockIdx.x + 1] = sso;
  }
}

__global__ void k_finalize_counts(const int32_t* __restrict__ part, int nparts,
                                  const int32_t* __restrict__ n_new_p, dv_counters* C) {
  int fl = 0, so = 0;
  for (int k = threadIdx.x; k < nparts; k += blockDim.x) {
    fl += part[2 * k];
    so += part[2 * k + 1];
  }
  fl = block_sum<int>(fl);
  so = block_sum<int>(so);
  if (threadIdx.x == 0) {
    C->n = *n_new_p;
    C->n_fluid = fl;
    C->n_solid = so;
  }
}

// ------------------------------------------------- per-step neighbour lists
// After the sort, every sweep of the step visits the same neighbour sets in
// the same order, so the cell scan (3^d cells) is done once here and the
// sweeps read the lists as CSR (offsets = exclusive scan of the counts).
//
// Each entry carries the neighbour's material in its top bit (DV_NBR_SOLID),
// so the sweeps do not gather it; a material other than fluid or solid sets
// bad[0] and the lists are not used.
//
// Rows of static solids stay empty: every neighbour walk of the step has a
// fluid particle (or, for the rigid coupling, a dynamic solid) at its centre,
// and the static boundary volume (once, at initialisation) scans cells.
//
// 3-D (27 cells, ~8 candidates each): one cell-scan pass stores each
// particle's first `slots` neighbours in its own fixed row and its count; a
// warp-wide copy then moves the rows into CSR (a particle with more
// neighbours than slots scans its cells again there).  This saves a second
// 27-cell scan.  2-D (9 cells): counting is cheap and the fixed rows cost
// more write traffic than they save, so a count pass and a fill pass.
__device__ __forceinline__ bool nbr_row_built(const int32_t* __restrict__ mat, const uint8_t* __restrict__ dyn,
                                              int i) {
  return !(mat[i] == DV_MATERIAL_SOLID && !dyn[i]);
}

__device__ __forceinline__ int32_t nbr_entry(int j, int mj, int32_t* bad) {
  if (mj != DV_MATERIAL_FLUID && mj != DV_MATERIAL_SOLID) *bad = 1;
  return (int32_t)((uint32_t)j | (mj == DV_MATERIAL_SOLID ? DV_NBR_SOLID : 0u));
}

template <int D>
__global__ void k_csr_count(dv_params P, DevGrid G, const float* __restrict__ x, const int32_t* __restrict__ mat,
                            const uint8_t* __restrict__ dyn, const dv_counters* __restrict__ C, int m,
                            uint32_t* __restrict__ cnt) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  uint32_t k = 0;
  if (i < C->n && nbr_row_built(mat, dyn, i))
    for_each_neighbor<D>(P, G, x, i, ldv<D>(x, i), [&](int, V3, float) { ++k; });
  cnt[i] = k;
}

template <int D>
__global__ void k_csr_fill(dv_params P, DevGrid G, const float* __restrict__ x,
                           const int32_t* __restrict__ mat, const dv_counters* __restrict__ C,
                           const uint32_t* __restrict__ off, int32_t* __restrict__ ok,
                           int32_t* __restrict__ out, const uint8_t* __restrict__ dyn) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= C->n || !ok[0] || !nbr_row_built(mat, dyn, i)) return;
  uint32_t k = off[i];
  for_each_neighbor_m<D>(P, G, x, mat, i, ldv<D>(x, i),
                         [&](int j, V3, float, int mj) { out[k++] = nbr_entry(j, mj, ok + 1); });
}

template <int D>
__global__ void k_csr_rows(dv_params P, DevGrid G, const float* __restrict__ x, const int32_t* __restrict__ mat,
                           const uint8_t* __restrict__ dyn, const dv_counters* __restrict__ C, int m, int slots,
                           uint32_t* __restrict__ cnt, int32_t* __restrict__ rows) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  uint32_t k = 0;
  if (i < C->n && nbr_row_built(mat, dyn, i)) {
    int32_t* row = rows + (int64_t)i * slots;
    for_each_neighbor<D>(P, G, x, i, ldv<D>(x, i), [&](int j, V3, float) {
      if (k < (uint32_t)slots) row[k] = j;
      ++k;
    });
  }
  cnt[i] = k;
}

// one warp per group of 32 particles; each row is copied by the whole warp
// (coalesced reads of the row, coalesced writes of the CSR segment), and the
// neighbours' materials are gathered here, 32 independent loads at a time,
// rather than in the row scan's dependent chain
template <int D>
__global__ void k_csr_compact(dv_params P, DevGrid G, const float* __restrict__ x, const int32_t* __restrict__ mat,
                              const dv_counters* __restrict__ C, int slots, const int32_t* __restrict__ rows,
                              const uint32_t* __restrict__ off, int32_t* __restrict__ ok,
                              int32_t* __restrict__ out) {
  if (!ok[0]) return;
  const int n = C->n;
  const int lane = threadIdx.x & 31;
  const int i0 = (blockIdx.x * blockDim.x + threadIdx.x) & ~31;
  const int iend = min(i0 + 32, n);
  for (int i = i0; i < iend; ++i) {
    const uint32_t k0 = off[i], cnt = off[i + 1] - k0;
    if (cnt <= (uint32_t)slots) {
      const int32_t* row = rows + (int64_t)i * slots;
      for (uint32_t k = lane; k < cnt; k += 32) {
        const int j = row[k];
        out[k0 + k] = nbr_entry(j, __ldg(mat + j), ok + 1);
      }
    } else if (lane == (i & 31)) {
      uint32_t k = k0;
      for_each_neighbor_m<D>(P, G, x, mat, i, ldv<D>(x, i),
                             [&](int j, V3, float, int mj) { out[k++] = nbr_entry(j, mj, ok + 1); });
    }
  }
}

__global__ void k_csr_ok(const uint32_t* __restrict__ off, const dv_counters* __restrict__ C, int64_t cap,
                         int32_t* __restrict__ ok) {
  ok[0] = (int64_t)off[C->n] <= cap ? 1 : 0;
}

// after the fill: lists that met a material other than fluid or solid are
// not used (their entries cannot encode it)
__global__ void k_csr_material_check(int32_t* __restrict__ ok) {
  if (ok[1]) ok[0] = 0;
}

static int build_csr(dv_ctx* c, const dv_fields* f) {
  const int m = (int)std::min<int64_t>(c->n_upper, c->cap) + 1;
  const int nb = dv_blocks(m);
  DevGrid G = dv_grid_cells(c);
  const bool rows = c->p.dim == 3;
  DV_CK(c, cudaMemsetAsync(c->d_nbr_ok + 1, 0, sizeof(int32_t), c->stream));
  if (rows)
    k_csr_rows<3><<<nb, DV_THREADS, 0, c->stream>>>(c->p, G, f->x, f->material, f->is_dynamic, c->d_cnt, m,
                                                    c->nbr_slots, c->flags, c->nbr_rows);
  else
    k_csr_count<2><<<nb, DV_THREADS, 0, c->stream>>>(c->p, G, f->x, f->material, f->is_dynamic, c->d_cnt, m,
                                                     c->flags);
  DV_LAUNCHED(c);
  int rc = dv_scan_u32(c, c->flags, c->nbr_off, m);
  if (rc) return rc;
  k_csr_ok<<<1, 1, 0, c->stream>>>(c->nbr_off, c->d_cnt, c->nbr_cap, c->d_nbr_ok);
  DV_LAUNCHED(c);
  if (rows)
    k_csr_compact<3><<<nb, DV_THREADS, 0, c->stream>>>(c->p, G, f->x, f->material, c->d_cnt, c->nbr_slots,
                                                       c->nbr_rows, c->nbr_off, c->d_nbr_ok, c->nbr_idx);
  else
    k_csr_fill<2><<<nb, DV_THREADS, 0, c->stream>>>(c->p, G, f->x, f->material, c->d_cnt, c->nbr_off,
                                                    c->d_nbr_ok, c->nbr_idx, f->is_dynamic);
  DV_LAUNCHED(c);
  k_csr_material_check<<<1, 1, 0, c->stream>>>(c->d_nbr_ok);
  DV_LAUNCHED(c);
  return DV_OK;
}

// positions or the particle count changed: sweeps go back to the cell scan
int dv_invalidate_lists(dv_ctx* c) {
  DV_CK(c, cudaMemsetAsync(c->d_nbr_ok, 0, sizeof(int32_t), c->stream));
  return DV_OK;
}

static int check_fields(dv_ctx* c, const dv_fields* f, const char* who) {
  if (!f->x || !f->x0 || !f->v || !f->acceleration || !f->vorticity || !f->m_V || !f->m ||
      !f->density || !f->pressure || !f->dfsph_factor || !f->density_adv || !f->life_time ||
      !f->material || !f->object_id || !f->color || !f->grid_ids || !f->is_dynamic ||
      !f->is_active || !f->is_sample)
    return dv_fail(c, DV_EINVAL, "%s: a dv_fields pointer is NULL", who);
  return DV_OK;
}

DV_API int dv_grid_build(dv_ctx* c, const dv_fields* src, const dv_fields* dst) {
  if (!c || !src || !dst) return DV_EINVAL;
  int rc = check_fields(c, src, "dv_grid_build(src)");
  if (rc) return rc;
  rc = check_fields(c, dst, "dv_grid_build(dst)");
  if (rc) return rc;
  if (src->x == dst->x || src->v == dst->v || src->m_V == dst->m_V)
    return dv_fail(c, DV_EINVAL, "dv_grid_build: src and dst alias");
  const int64_t nu = std::min<int64_t>(c->n_upper, c->cap);
  const uint32_t invalid = (c->kbits >= 32) ? 0xffffffffu : ((1u << c->kbits) - 1u);
  const int nb = dv_blocks(nu);
  rc = dv_invalidate_lists(c);
  if (rc) return rc;
  DevGrid G = dv_grid_cells(c);
  const bool batch = c->p.n_scenes > 1;
  const int32_t* scn = batch ? src->object_id : nullptr;
  if (c->p.dim == 2)
    k_cell_keys<2><<<nb, DV_THREADS, 0, c->stream>>>(c->p, *src, G, c->d_cnt, c->keys[0], invalid, scn,
                                                     c->scene_shift);
  else
    k_cell_keys<3><<<nb, DV_THREADS, 0, c->stream>>>(c->p, *src, G, c->d_cnt, c->keys[0], invalid, scn,
                                                     c->scene_shift);
  DV_LAUNCHED(c);
  // radix passes
  const int ntiles = (int)std::max<int64_t>(1, (nu + RS_TILE - 1) / RS_TILE);
  if (ntiles > c->max_tiles) return dv_fail(c, DV_ECAPACITY, "sort tiles exceed workspace");
  int cur = 0;
  for (int pass = 0; pass < c->npasses; ++pass) {
    int shift = pass * 8;
    k_rs_hist<<<ntiles, RS_T, 0, c->stream>>>(c->keys[cur], c->d_cnt, shift, ntiles, c->hist);
    DV_LAUNCHED(c);
    rc = dv_scan_u32(c, c->hist, c->hist, (int64_t)256 * ntiles);
    if (rc) return rc;
    k_rs_scatter<<<ntiles, RS_T, 0, c->stream>>>(c->keys[cur], pass == 0 ? nullptr : c->vals[cur],
                                                c->keys[cur ^ 1], c->vals[cur ^ 1], c->d_cnt, shift,
                                                ntiles, c->hist);
    DV_LAUNCHED(c);
    cur ^= 1;
  }
  c->perm_buf = cur;
  // cell table
  DV_CK(c, cudaMemsetAsync(c->cell_start, 0, sizeof(int32_t) * c->ncells, c->stream));
  DV_CK(c, cudaMemsetAsync(c->cell_end, 0, sizeof(int32_t) * c->ncells, c->stream));
  DV_CK(c, cudaMemsetAsync(c->d_flag + 1, 0, sizeof(int32_t), c->stream));
  k_cell_ranges<<<nb, DV_THREADS, 0, c->stream>>>(c->keys[cur], c->d_cnt, invalid, c->cell_start,
                                                  c->cell_end, c->d_flag + 1);
  DV_LAUNCHED(c);
  if (c->p.dim == 2)
    k_permute<2><<<nb, DV_THREADS, 0, c->stream>>>(*src, *dst, c->vals[cur], c->keys[cur],
                                                   c->d_flag + 1, (int)c->cap, c->d_cnt, c->ired_part);
  else
    k_permute<3><<<nb, DV_THREADS, 0, c->stream>>>(*src, *dst, c->vals[cur], c->keys[cur],
                                                   c->d_flag + 1, (int)c->cap, c->d_cnt, c->ired_part);
  DV_LAUNCHED(c);
  k_finalize_counts<<<1, 1024, 0, c->stream>>>(c->ired_part, nb, c->d_flag + 1, c->d_cnt);
  DV_LAUNCHED(c);
  c->scene_ptr = batch ? dst->object_id : nullptr;  // scene of each sorted slot
  return build_csr(c, dst);
}

DV_API int dv_get_permutation(dv_ctx* c, int32_t* host_perm, int64_t n_cap) {
  if (!c || !host_perm) return DV_EINVAL;
  dv_counters cnt;
  int rc = dv_get_counters(c, &cnt);
  if (rc) return rc;
  int64_t n = std::min<int64_t>(cnt.n, n_cap);
  DV_CK(c, cudaMemcpyAsync(host_perm, c->vals[c->perm_buf], sizeof(int32_t) * n,
                           cudaMemcpyDeviceToHost, c->stream));
  DV_CK(c, cudaStreamSynchronize(c->stream));
  return DV_OK;
}

// --------------------------------------------------------------- emission
template <int D>
__global__ void k_add_particles(dv_fields F, const float* __restrict__ pos,
                                const float* __restrict__ vel, int count, int cap, int32_t obj,
                                float density, float pressure, int32_t material, int32_t is_dyn,
                                int4 color, float m_V0, const dv_counters* __restrict__ C) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  int p = C->n + k;
  if (p >= cap) return;
  V3 x{pos[k * D], pos[k * D + 1], D == 3 ? pos[k * D + 2] : 0.0f};
  V3 v{vel[k * D], vel[k * D + 1], D == 3 ? vel[k * D + 2] : 0.0f};
  stv<D>(F.x, p, x);
  stv<D>(F.x0, p, x);
  stv<D>(F.v, p, v);
  stv<D>(F.acceleration, p, V3{0.f, 0.f, 0.f});
  st4(F.vorticity, p, V3{0.f, 0.f, 0.f});
  F.object_id[p] = obj;
  F.density[p] = density;
  F.m_V[p] = m_V0;
  F.m[p] = m_V0 * density;  // particle_system.py:325
  F.pressure[p] = pressure;
  F.material[p] = material;
  F.is_dynamic[p] = (uint8_t)(is_dyn != 0);
  reinterpret_cast<int4*>(F.color)[p] = color;
  F.is_active[p] = 1;
  F.dfsph_factor[p] = 0.0f;
  F.density_adv[p] = 0.0f;
  F.is_sample[p] = 0;
  F.life_time[p] = 0.0f;
  F.grid_ids[p] = -1;
}

__global__ void k_add_counts(dv_counters* C, int count, int cap, int material) {
  int room = cap - C->n;
  int added = count < room ? count : (room > 0 ? room : 0);
  if (added < count) C->status |= DV_WARN_CAPACITY;
  C->n += added;
  if (material == DV_MATERIAL_FLUID)
    C->n_fluid += added;
  else
    C->n_solid += added;
}

DV_API int dv_add_particles(dv_ctx* c, const dv_fields* f, const float* pos, const float* vel,
                            int32_t count, int32_t object_id, float density, float pressure,
                            int32_t material, int32_t is_dynamic, int32_t color_r,
                            int32_t color_g, int32_t color_b, float m_V0) {
  if (!c || !f || (count > 0 && (!pos || !vel))) return DV_EINVAL;
  if (count < 0) return dv_fail(c, DV_EINVAL, "dv_add_particles: negative count");
  if (count == 0) return DV_OK;
  int rc = check_fields(c, f, "dv_add_particles");
  if (rc) return rc;
  int4 col = make_int4(color_r, color_g, color_b, 0);
  int nb = dv_blocks(count);
  if (c->p.dim == 2)
    k_add_particles<2><<<nb, DV_THREADS, 0, c->stream>>>(*f, pos, vel, count, (int)c->cap, object_id,
                                                         density, pressure, material, is_dynamic,
                                                         col, m_V0, c->d_cnt);
  else
    k_add_particles<3><<<nb, DV_THREADS, 0, c->stream>>>(*f, pos, vel, count, (int)c->cap, object_id,
                                                         density, pressure, material, is_dynamic,
                                                         col, m_V0, c->d_cnt);
  DV_LAUNCHED(c);
  k_add_counts<<<1, 1, 0, c->stream>>>(c->d_cnt, count, (int)c->cap, material);
  DV_LAUNCHED(c);
  c->n_upper = std::min<int64_t>(c->n_upper + count, c->cap);
  return dv_invalidate_lists(c);
}

// ----------------------------------------------------------- neighbour CSR
template <int D>
__global__ void k_nbr_count(dv_params P, DevGrid G, const float* __restrict__ x,
                            const dv_counters* __restrict__ C, uint32_t* __restrict__ cnt) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= C->n) return;
  uint32_t k = 0;
  for_each_neighbor<D>(P, G, x, i, ldv<D>(x, i), [&](int, V3, float) { ++k; });
  cnt[i] = k;
}

template <int D>
__global__ void k_nbr_fill(dv_params P, DevGrid G, const float* __restrict__ x,
                           const dv_counters* __restrict__ C, const uint32_t* __restrict__ off,
                           int32_t* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= C->n) return;
  uint32_t k = off[i];
  for_each_neighbor<D>(P, G, x, i, ldv<D>(x, i), [&](int j, V3, float) { out[k++] = j; });
}

__global__ void k_u32_to_i64(const uint32_t* __restrict__ a, int64_t* __restrict__ b, int m) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) b[i] = a[i];
}

__global__ void k_nbr_slots(const int32_t* __restrict__ in, int64_t m, int32_t* __restrict__ out) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < m) out[k] = nbr_slot((uint32_t)in[k]);
}

DV_API int64_t dv_stored_lists(dv_ctx* c, uint32_t* dev_offsets, int32_t* dev_nbrs, int64_t max_entries) {
  if (!c) return DV_EINVAL;
  dv_counters cnt;
  int rc = dv_get_counters(c, &cnt);
  if (rc) return rc;
  int32_t ok = 0;
  uint32_t total32 = 0;
  const int n = cnt.n;
  DV_CK(c, cudaMemcpyAsync(&ok, c->d_nbr_ok, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
  DV_CK(c, cudaMemcpyAsync(&total32, c->nbr_off + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
  DV_CK(c, cudaStreamSynchronize(c->stream));
  if (!ok) return dv_fail(c, DV_EINVAL, "dv_stored_lists: no valid lists (positions changed since the grid build)");
  const int64_t total = total32;
  if (dev_offsets)
    DV_CK(c, cudaMemcpyAsync(dev_offsets, c->nbr_off, sizeof(uint32_t) * ((size_t)n + 1), cudaMemcpyDeviceToDevice,
                             c->stream));
  if (dev_nbrs) {
    if (total > max_entries)
      return dv_fail(c, DV_ECAPACITY, "dv_stored_lists: %lld entries > max_entries %lld", (long long)total,
                     (long long)max_entries);
    if (total > 0) {  // the slots, without the material bit
      k_nbr_slots<<<dv_blocks(total), DV_THREADS, 0, c->stream>>>(c->nbr_idx, total, dev_nbrs);
      DV_LAUNCHED(c);
    }
  }
  DV_CK(c, cudaStreamSynchronize(c->stream));
  return total;
}

DV_API int64_t dv_neighbor_lists(dv_ctx* c, const dv_fields* f, int64_t* dev_offsets,
                                 int32_t* dev_nbrs, int64_t max_pairs) {
  if (!c || !f || !f->x) return DV_EINVAL;
  dv_counters cnt;
  int rc = dv_get_counters(c, &cnt);
  if (rc) return rc;
  const int n = cnt.n;
  // always the cell scan: this entry point checks the lists the sweeps use
  DevGrid G = dv_grid_cells(c);
  int nb = dv_blocks(n);
  if (c->p.dim == 2)
    k_nbr_count<2><<<nb, DV_THREADS, 0, c->stream>>>(c->p, G, f->x, c->d_cnt, c->flags);
  else
    k_nbr_count<3><<<nb, DV_THREADS, 0, c->stream>>>(c->p, G, f->x, c->d_cnt, c->flags);
  DV_LAUNCHED(c);
  DV_CK(c, cudaMemsetAsync(c->flags + n, 0, sizeof(uint32_t), c->stream));
  rc = dv_scan_u32(c, c->flags, c->offs, (int64_t)n + 1);
  if (rc) return rc;
  uint32_t total32 = 0;
  DV_CK(c, cudaMemcpyAsync(&total32, c->offs + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
  DV_CK(c, cudaStreamSynchronize(c->stream));
  const int64_t total = total32;
  if (dev_offsets) {
    k_u32_to_i64<<<dv_blocks(n + 1), DV_THREADS, 0, c->stream>>>(c->offs, dev_offsets, n + 1);
    DV_LAUNCHED(c);
  }
  if (!dev_nbrs) {
    DV_CK(c, cudaStreamSynchronize(c->stream));
    return total;
  }
  if (total > max_pairs)
    return dv_fail(c, DV_ECAPACITY, "dv_neighbor_lists: %lld pairs > max_pairs %lld",
                   (long long)total, (long long)max_pairs);
  if (c->p.dim == 2)
    k_nbr_fill<2><<<nb, DV_THREADS, 0, c->stream>>>(c->p, G, f->x, c->d_cnt, c->offs, dev_nbrs);
  else
    k_nbr_fill<3><<<nb, DV_THREADS, 0, c->stream>>>(c->p, G, f->x, c->d_cnt, c->offs, dev_nbrs);
  DV_LAUNCHED(c);
  DV_CK(c, cudaStreamSynchronize(c->stream));
  return total;
}
