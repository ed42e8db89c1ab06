// DIMCV vorticity pipeline (reference: dimcv_sph.py:228-335, 551-583,
// 649-801): vorticity / ∇v / v*, Δω = ω - ∇×v*, SPH smoothing, kinematic
// vorticity number with the Bernoulli sample birth/death, sample compaction,
// Epanechnikov AKDE with an FP64 kden_sum, the FP64-CDF inverse-CDF sampler,
// the near-field part of vort2vel, life time and the export-only fields.
// Same numerics contract as dv_sph.cu (-fmad=false, IEEE, reference order).
#include <algorithm>

#include "dv_internal.cuh"

#define FOR_I                                    \
  int i = blockIdx.x * blockDim.x + threadIdx.x; \
  if (i >= C->n) return;

// Δ = (a - b) as 3-vectors padded with zeros (dimcv_sph.py:236-248)
__device__ __forceinline__ V3 sub3(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }

// ------------------------------------------- v*, vorticity, ∇v (one sweep)
// compute_v_star (:264-271), compute_vorticity (:228-248, 284-293),
// compute_grad_v (:250-262, 273-282).  Non-fluid slots get zeros (the
// reference fills these fields with 0 first).
template <int D>
__global__ void k_vorticity(dv_params P, DevGrid G, dv_fields F, dv_solver_fields S,
                            const dv_counters* __restrict__ C) {
  FOR_I;
  const int DD = D * D;
  if (F.material[i] != DV_MATERIAL_FLUID) {
    stv<D>(S.v_star, i, V3{0.f, 0.f, 0.f});
    st4(F.vorticity, i, V3{0.f, 0.f, 0.f});
    for (int k = 0; k < DD; ++k) S.grad_v[(int64_t)i * DD + k] = 0.0f;
    return;
  }
  V3 xi = ldv<D>(F.x, i);
  V3 vi = ldv<D>(F.v, i);
  V3 ai = ldv<D>(F.acceleration, i);
  V3 vs{vi.x + ai.x * P.dt, vi.y + ai.y * P.dt, D == 3 ? vi.z + ai.z * P.dt : 0.0f};
  stv<D>(S.v_star, i, vs);
  V3 w{0.f, 0.f, 0.f};
  float g[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  for_each_neighbor_m<D>(P, G, F.x, F.material, i, xi, [&](int j, V3 r, float r2, int mj) {
    if (mj != DV_MATERIAL_FLUID) return;
    V3 vj = ldv<D>(F.v, j);
    V3 gw = cubic_gradW<D>(P, r, r2);
    float mv = F.m_V[j];
    V3 c = cross3(sub3(vj, vi), gw);
    w.x += mv * c.x;
    w.y += mv * c.y;
    w.z += mv * c.z;
    V3 vji = sub3(vj, vi);
    float vc[3] = {vji.x, vji.y, vji.z};
    float gc[3] = {gw.x, gw.y, gw.z};
#pragma unroll
    for (int a = 0; a < D; ++a)
#pragma unroll
      for (int b = 0; b < D; ++b) g[a * D + b] += (mv * vc[a]) * gc[b];
  });
  st4(F.vorticity, i, w);
#pragma unroll
  for (int k = 0; k < DD; ++k) S.grad_v[(int64_t)i * DD + k] = g[k];
}

// compute_d_vorticity (dimcv_sph.py:551-583)
template <int D>
__global__ void k_d_vorticity(dv_params P, DevGrid G, dv_fields F, dv_solver_fields S,
                              const dv_counters* __restrict__ C) {
  FOR_I;
  if (F.material[i] != DV_MATERIAL_FLUID) {
    st4(S.d_vort, i, V3{0.f, 0.f, 0.f});
    return;
  }
  V3 xi = ldv<D>(F.x, i);
  V3 vsi = ldv<D>(S.v_star, i);
  V3 curl{0.f, 0.f, 0.f};
  for_each_neighbor_m<D>(P, G, F.x, F.material, i, xi, [&](int j, V3 r, float r2, int mj) {
    if (mj != DV_MATERIAL_FLUID) return;
    V3 vsj = ldv<D>(S.v_star, j);
    V3 c = cross3(sub3(vsj, vsi), cubic_gradW<D>(P, r, r2));
    float mv = F.m_V[j];
    curl.x += mv * c.x;
    curl.y += mv * c.y;
    curl.z += mv * c.z;
  });
  V3 w = ld4(F.vorticity, i);
  st4(S.d_vort, i, V3{w.x - curl.x, w.y - curl.y, w.z - curl.z});
}

// k_vorticity and k_d_vorticity in one neighbour walk: v*_j = v_j + a_j·dt
// is formed per neighbour by the same multiply and add that k_vorticity
// stores v*_j with, so every sum (ω, ∇v, ∇×v*) and Δω are bit-identical to
// the two separate sweeps, without re-reading the list, positions and
// materials or storing and gathering v*.
template <int D>
__global__ void k_vorticity_dvort(dv_params P, DevGrid G, dv_fields F, dv_solver_fields S,
                                  const dv_counters* __restrict__ C) {
  FOR_I;
  const int DD = D * D;
  if (F.material[i] != DV_MATERIAL_FLUID) {
    stv<D>(S.v_star, i, V3{0.f, 0.f, 0.f});
    st4(F.vorticity, i, V3{0.f, 0.f, 0.f});
    for (int k = 0; k < DD; ++k) S.grad_v[(int64_t)i * DD + k] = 0.0f;
    st4(S.d_vort, i, V3{0.f, 0.f, 0.f});
    return;
  }
  V3 xi = ldv<D>(F.x, i);
  V3 vi = ldv<D>(F.v, i);
  V3 ai = ldv<D>(F.acceleration, i);
  V3 vs{vi.x + ai.x * P.dt, vi.y + ai.y * P.dt, D == 3 ? vi.z + ai.z * P.dt : 0.0f};
  stv<D>(S.v_star, i, vs);
  V3 w{0.f, 0.f, 0.f};
  V3 curl{0.f, 0.f, 0.f};
  float g[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  for_each_neighbor_m<D>(P, G, F.x, F.material, i, xi, [&](int j, V3 r, float r2, int mj) {
    if (mj != DV_MATERIAL_FLUID) return;
    V3 vj = ldv<D>(F.v, j);
    V3 aj = ldv<D>(F.acceleration, j);
    V3 vsj{vj.x + aj.x * P.dt, vj.y + aj.y * P.dt, D == 3 ? vj.z + aj.z * P.dt : 0.0f};
    V3 gw = cubic_gradW<D>(P, r, r2);
    float mv = F.m_V[j];
    V3 c = cross3(sub3(vj, vi), gw);
    w.x += mv * c.x;
    w.y += mv * c.y;
    w.z += mv * c.z;
    V3 vji = sub3(vj, vi);
    float vc[3] = {vji.x, vji.y, vji.z};
    float gc[3] = {gw.x, gw.y, gw.z};
#pragma unroll
    for (int a = 0; a < D; ++a)
#pragma unroll
      for (int b = 0; b < D; ++b) g[a * D + b] += (mv * vc[a]) * gc[b];
    V3 c2 = cross3(sub3(vsj, vs), gw);
    curl.x += mv * c2.x;
    curl.y += mv * c2.y;
    curl.z += mv * c2.z;
  });
  st4(F.vorticity, i, w);
#pragma unroll
  for (int k = 0; k < DD; ++k) S.grad_v[(int64_t)i * DD + k] = g[k];
  st4(S.d_vort, i, V3{w.x - curl.x, w.y - curl.y, w.z - curl.z});
}

// compute_all_d_vort_smoothed (dimcv_sph.py:660-677); slots outside the
// vortex domain keep their previous value (index-stable field)
template <int D>
__global__ void k_smooth(dv_params P, DevGrid G, dv_fields F, dv_solver_fields S,
                         const dv_counters* __restrict__ C) {
  FOR_I;
  if (F.material[i] != DV_MATERIAL_FLUID) return;
  V3 xi = ldv<D>(F.x, i);
  if (!in_vortex_domain<D>(P, xi)) return;
  float mvi = F.m_V[i];
  V3 di = ld4(S.d_vort, i);
  float w0 = cubic_W(P, 0.0f);
  V3 acc{mvi * di.x * w0, mvi * di.y * w0, mvi * di.z * w0};
  for_each_neighbor_m<D>(P, G, F.x, F.material, i, xi, [&](int j, V3, float r2, int mj) {
    if (mj != DV_MATERIAL_FLUID) return;
    float mv = F.m_V[j];
    V3 dj = ld4(S.d_vort, j);
    float wk = cubic_W(P, sqrtf(r2));
    acc.x += mv * dj.x * wk;
    acc.y += mv * dj.y * wk;
    acc.z += mv * dj.z * wk;
  });
  st4(S.d_vort_smoothed, i, acc);
}

// ------------------------------------------------- KVN + birth / death
// compute_kinematic_vorticity_num_sample (dimcv_sph.py:295-324).  The
// uniform draws come from Philox keyed by (slot, draw, step, seed).
template <int D>
__global__ void k_kvn_sample(dv_params P, dv_fields F, dv_solver_fields S,
                             const dv_counters* __restrict__ C, uint32_t s0, uint32_t s1,
                             uint32_t t0, uint32_t t1, int birth_death) {
  FOR_I;
  if (F.material[i] != DV_MATERIAL_FLUID) return;
  V3 xi = ldv<D>(F.x, i);
  if (!in_vortex_domain<D>(P, xi)) return;
  const int DD = D * D;
  float g[9];
#pragma unroll
  for (int k = 0; k < DD; ++k) g[k] = S.grad_v[(int64_t)i * DD + k];
  // Frobenius norms of G - G^T and G + G^T, entries summed row-major
  float wn = 0.0f, sn = 0.0f;
#pragma unroll
  for (int a = 0; a < D; ++a)
#pragma unroll
    for (int b = 0; b < D; ++b) {
      float wv = g[a * D + b] - g[b * D + a];
      float sv = g[a * D + b] + g[b * D + a];
      wn = (a == 0 && b == 0) ? wv * wv : wn + wv * wv;
      sn = (a == 0 && b == 0) ? sv * sv : sn + sv * sv;
    }
  float kvn = sqrtf(wn) / (sqrtf(sn) + P.kvn_eps);
  S.kvn[i] = kvn;
  if (!birth_death) return;
  float t = fminf(fmaxf(F.life_time[i], 0.0f), 1.0f);
  float rr = 0.018f * expf(-P.gen_a * t) + 0.004f;
  float produce = 1.0f - 1.0f / powf(kvn + 1.0f, rr);
  float del = expf(-P.del_b * kvn);
  DvRand4 rnd = dv_philox((uint32_t)i, 0u, t0, t1, s0, s1);
  float u1 = dv_u01f(rnd.v[0]);
  float u2 = dv_u01f(rnd.v[1]);
  uint8_t smp = F.is_sample[i];
  if (smp == 0 && u1 < produce) {
    F.is_sample[i] = 1;
  } else if (smp == 1 && kvn < 2.0f && u2 < del) {
    F.is_sample[i] = 0;
  }
}

// ------------------------------------------------------ compaction helpers
__global__ void k_flag_samples(const dv_fields F, const dv_counters* __restrict__ C, int m,
                               uint32_t* __restrict__ flags) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  flags[i] = (i < C->n && F.is_sample[i] == 1) ? 1u : 0u;
}

template <int D>
__global__ void k_flag_targets(dv_params P, const dv_fields F, const dv_counters* __restrict__ C,
                               int m, uint32_t* __restrict__ flags) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  uint32_t f = 0;
  if (i < C->n && F.material[i] == DV_MATERIAL_FLUID) f = in_vortex_domain<D>(P, ldv<D>(F.x, i)) ? 1u : 0u;
  flags[i] = f;
}

__global__ void k_compact(const uint32_t* __restrict__ flags, const uint32_t* __restrict__ offs,
                          int m, int32_t* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  if (flags[i]) out[offs[i]] = i;
}

// count = offs[n] (the scan covers [0, m) with flags[n..m) = 0)
__global__ void k_store_count(const uint32_t* __restrict__ offs, dv_counters* C, int which) {
  int c = (int)offs[C->n];
  if (which == 0)
    C->num_samples = c;
  else
    C->n_targets = c;
}

// Fills c->targets with the slots of fluid particles inside the vortex
// domain, in ascending slot order; count in C->n_targets.
int dv_build_targets(dv_ctx* c, const dv_fields* f) {
  const int m = (int)std::min<int64_t>(c->n_upper, c->cap) + 1;
  const int nb = dv_blocks(m);
  if (c->p.dim == 2)
    k_flag_targets<2><<<nb, DV_THREADS, 0, c->stream>>>(c->p, *f, c->d_cnt, m, c->flags);
  else
    k_flag_targets<3><<<nb, DV_THREADS, 0, c->stream>>>(c->p, *f, c->d_cnt, m, c->flags);
  DV_LAUNCHED(c);
  int rc = dv_scan_u32(c, c->flags, c->offs, m);
  if (rc) return rc;
  k_compact<<<nb, DV_THREADS, 0, c->stream>>>(c->flags, c->offs, m, c->targets);
  DV_LAUNCHED(c);
  k_store_count<<<1, 1, 0, c->stream>>>(c->offs, c->d_cnt, 1);
  DV_LAUNCHED(c);
  return DV_OK;
}

// ------------------------------------------------------------------ AKDE
// epanechnikov_kernel (dimcv_sph.py:721-730)
template <int D>
__device__ __forceinline__ float epan(const dv_params& P, V3 r) {
  float ret = 1.0f;
  float rc[3] = {r.x, r.y, r.z};
#pragma unroll
  for (int d = 0; d < D; ++d) {
    float q = fabsf(rc[d]) * P.inv_support_radius;
    if (q < 1.0f)
      ret *= 0.75f * (1.0f - q * q);
    else
      ret *= 0.0f;
  }
  return ret;
}

// compute_kernel_density (dimcv_sph.py:732-751) + FP64 block partials of
// kden_sum (the reference accumulates it with an f32 atomic add)
template <int D>
__global__ void k_akde(dv_params P, DevGrid G, dv_fields F, dv_solver_fields S,
                       const dv_counters* __restrict__ C, double* __restrict__ part) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double contrib = 0.0;
  if (i < C->n && F.material[i] == DV_MATERIAL_FLUID) {
    V3 xi = ldv<D>(F.x, i);
    if (in_vortex_domain<D>(P, xi)) {
      float kd = S.kvn[i] * epan<D>(P, V3{0.f, 0.f, 0.f});
      for_each_neighbor_m<D>(P, G, F.x, F.material, i, xi, [&](int j, V3 r, float, int mj) {
        if (mj == DV_MATERIAL_FLUID) kd += S.kvn[j] * epan<D>(P, r);
      });
      S.kden[i] = kd;
      contrib = (double)kd;
    }
  }
  double s = block_sum<double>(contrib);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// k_smooth and k_akde in one neighbour walk (both over the fluid neighbours
// of a vortex-domain fluid slot): the smoothed Δω and kden of slot i and
// the FP64 block partials of kden_sum come out bit-identical to the two
// separate sweeps.  KVN must be current (k_kvn_sample first); the smoothing
// does not read it.
template <int D>
__global__ void k_smooth_akde(dv_params P, DevGrid G, dv_fields F, dv_solver_fields S,
                              const dv_counters* __restrict__ C, double* __restrict__ part) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double contrib = 0.0;
  if (i < C->n && F.material[i] == DV_MATERIAL_FLUID) {
    V3 xi = ldv<D>(F.x, i);
    if (in_vortex_domain<D>(P, xi)) {
      float mvi = F.m_V[i];
      V3 di = ld4(S.d_vort, i);
      float w0 = cubic_W(P, 0.0f);
      V3 acc{mvi * di.x * w0, mvi * di.y * w0, mvi * di.z * w0};
      float kd = S.kvn[i] * epan<D>(P, V3{0.f, 0.f, 0.f});
      for_each_neighbor_m<D>(P, G, F.x, F.material, i, xi, [&](int j, V3 r, float r2, int mj) {
        if (mj != DV_MATERIAL_FLUID) return;
        float mv = F.m_V[j];
        V3 dj = ld4(S.d_vort, j);
        float wk = cubic_W(P, sqrtf(r2));
        acc.x += mv * dj.x * wk;
        acc.y += mv * dj.y * wk;
        acc.z += mv * dj.z * wk;
        kd += S.kvn[j] * epan<D>(P, r);
      });
      st4(S.d_vort_smoothed, i, acc);
      S.kden[i] = kd;
      contrib = (double)kd;
    }
  }
  double s = block_sum<double>(contrib);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void k_akde_finalize(const double* __restrict__ part, int nparts, dv_counters* C) {
  double s = 0.0;
  for (int k = threadIdx.x; k < nparts; k += blockDim.x) s += part[k];
  s = block_sum<double>(s);
  if (threadIdx.x == 0) {
    C->kden_sum = s;
    C->kden_sum_f32 = (float)s;
  }
}

// ------------------------------------------------------- inverse-CDF draws
__global__ void k_cdf_weights(const int32_t* __restrict__ targets, const float* __restrict__ kden,
                              const dv_counters* __restrict__ C, int m, double* __restrict__ w) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  w[k] = k < C->n_targets ? (double)kden[targets[k]] : 0.0;
}

// draw s: u ~ U[0,1) (53 bits, Philox keyed by (s, 2, step, seed)), or in
// stratified mode u = (s + ξ)/M with ξ that draw; the target k with
// cdf_ex[k] <= u·total < cdf_ex[k] + w_k (w_k > 0)
__global__ void k_cdf_draw(const double* __restrict__ cdf_ex, const int32_t* __restrict__ targets,
                           const float* __restrict__ kden, dv_counters* C, int M, uint32_t s0,
                           uint32_t s1, uint32_t t0, uint32_t t1, int stratified,
                           int32_t* __restrict__ out) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int nt = C->n_targets;
  if (nt <= 0) {
    if (s == 0) C->num_samples = 0;
    return;
  }
  const double total = cdf_ex[nt - 1] + (double)kden[targets[nt - 1]];
  if (!(total > 0.0)) {
    if (s == 0) C->num_samples = 0;
    return;
  }
  if (s == 0) C->num_samples = M;
  if (s >= M) return;
  DvRand4 rnd = dv_philox((uint32_t)s, 2u, t0, t1, s0, s1);
  double u = dv_u01d(rnd.v[0], rnd.v[1]);
  if (stratified) u = ((double)s + u) / (double)M;
  double y = u * total;
  // upper_bound(cdf_ex, y) - 1
  int lo = 0, hi = nt;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (cdf_ex[mid] <= y)
      lo = mid + 1;
    else
      hi = mid;
  }
  int k = lo - 1;
  if (k < 0) k = 0;
  // y at or past the last boundary: step back to the last positive weight
  while (k > 0 && !(kden[targets[k]] > 0.0f)) --k;
  out[s] = targets[k];
}

__global__ void k_set_num_samples(dv_counters* C, int M) { C->num_samples = M; }

// Scene batch: draw t belongs to the scene s with m_off_s <= t < m_off_s + M_s;
// with local index k = t - m_off_s it is k_cdf_draw of that scene alone
// (Philox keyed by (k, 2, step, seed_s); stratified: u = (k + ξ)/M_s) through
// the scene's segment [t_start_s, t_start_s + n_targets_s) of the batch CDF.
__global__ void k_batch_draw(const double* __restrict__ cdf_ex, const int32_t* __restrict__ targets,
                             const float* __restrict__ kden, const dv_scene_state* __restrict__ st,
                             const dv_batch_scene* __restrict__ sc, int S, const int64_t* __restrict__ step,
                             const dv_counters* __restrict__ C, int stratified, int32_t* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= C->num_samples) return;
  int lo = 0, hi = S;  // last s with m_off_s <= t
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (st[mid].m_off <= t)
      lo = mid + 1;
    else
      hi = mid;
  }
  const int s = lo - 1;
  const int k = t - st[s].m_off, M = st[s].num_samples;
  const int a = st[s].t_start, nt = st[s].n_targets;
  const uint64_t seed = sc[s].seed, stp = (uint64_t)*step;
  DvRand4 rnd = dv_philox((uint32_t)k, 2u, (uint32_t)stp, (uint32_t)(stp >> 32), (uint32_t)seed,
                          (uint32_t)(seed >> 32));
  double u = dv_u01d(rnd.v[0], rnd.v[1]);
  if (stratified) u = ((double)k + u) / (double)M;
  const double base = cdf_ex[a];
  const double total = cdf_ex[a + nt - 1] + (double)kden[targets[a + nt - 1]] - base;
  const double y = base + u * total;
  int l = a, h = a + nt;  // upper_bound in the scene's segment
  while (l < h) {
    const int mid = (l + h) >> 1;
    if (cdf_ex[mid] <= y)
      l = mid + 1;
    else
      h = mid;
  }
  int q = l - 1;
  if (q < a) q = a;
  while (q > a && !(kden[targets[q]] > 0.0f)) --q;
  out[t] = targets[q];
}

int dv_batch_draw(dv_ctx* c, const dv_solver_fields* s) {
  dv_batch_state* b = c->batch;
  const int m = (int)std::min<int64_t>(c->n_upper, c->cap);
  k_cdf_weights<<<dv_blocks(m), DV_THREADS, 0, c->stream>>>(c->targets, s->kden, c->d_cnt, m,
                                                          reinterpret_cast<double*>(c->near_v));
  DV_LAUNCHED(c);
  int rc = dv_scan_f64(c, reinterpret_cast<double*>(c->near_v), c->cdf, m);
  if (rc) return rc;
  k_batch_draw<<<dv_blocks(b->m_cap), DV_THREADS, 0, c->stream>>>(c->cdf, c->targets, s->kden, b->d_state,
                                                                  b->d_scenes, b->S, b->d_step, c->d_cnt,
                                                                  b->stratified, s->sample_idx);
  DV_LAUNCHED(c);
  return DV_OK;
}

// --------------------------------------------------------- VVPE near field
// vort2vel_neighbors_2d_task (dimcv_sph.py:649-658) for each target:
// near_v = 0.1592 V Σ_fluid Kε(|r_xy|) (r_xy × ω̃_j) and
// S_i = kden_i + Σ_fluid kden_j.  DV_KERNEL_BLOB3D uses the blob kernel.
template <int D>
__global__ void k_vvpe_near(dv_params P, DevGrid G, dv_fields F, dv_solver_fields S,
                            const dv_counters* __restrict__ C, const int32_t* __restrict__ targets,
                            float4* __restrict__ near_v, float* __restrict__ near_S) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= C->n_targets) return;
  int i = targets[t];
  V3 xi = ldv<D>(F.x, i);
  V3 acc{0.f, 0.f, 0.f};
  float Ssum = S.kden[i];
  const bool blob = P.kernel_mode == DV_KERNEL_BLOB3D;
  for_each_neighbor_m<D>(P, G, F.x, F.material, i, xi, [&](int j, V3 r, float r2, int mj) {
    if (mj != DV_MATERIAL_FLUID) return;
    V3 w = ld4(S.d_vort_smoothed, j);
    if (!blob) {
      V3 rp{r.x, r.y, 0.0f};
      float rn = sqrtf(__fadd_rn(__fadd_rn(__fmul_rn(rp.x, rp.x), __fmul_rn(rp.y, rp.y)), 0.0f * 0.0f));
      float e = expf(-rn * P.inv_eps);
      float K = (1.0f - e) / (rn * (rn + P.eps * e));
      V3 c = cross3(rp, w);
      acc.x += K * c.x;
      acc.y += K * c.y;
      acc.z += K * c.z;
    } else {
      float s = r2 + P.blob_delta2;
      float inv = 1.0f / (s * sqrtf(s));
      V3 c = cross3(r, w);
      acc.x += inv * c.x;
      acc.y += inv * c.y;
      acc.z += inv * c.z;
    }
    Ssum += S.kden[j];
  });
  float coef = blob ? P.blob_coef : P.vvpe_coef;
  near_v[t] = make_float4(acc.x * coef, acc.y * coef, acc.z * coef, 0.0f);
  near_S[t] = Ssum;
}

int dv_launch_vvpe_near(dv_ctx* c, const dv_fields* f, const dv_solver_fields* s) {
  const int nb = dv_blocks(std::min<int64_t>(c->n_upper, c->cap));
  if (c->p.dim == 2)
    k_vvpe_near<2><<<nb, DV_THREADS, 0, c->stream>>>(c->p, dv_grid(c), *f, *s, c->d_cnt, c->targets,
                                                     c->near_v, c->near_S);
  else
    k_vvpe_near<3><<<nb, DV_THREADS, 0, c->stream>>>(c->p, dv_grid(c), *f, *s, c->d_cnt, c->targets,
                                                     c->near_v, c->near_S);
  DV_LAUNCHED(c);
  return DV_OK;
}

// ------------------------------------------------------------- life time
template <int D>
__global__ void k_life_time(dv_params P, dv_fields F, const dv_counters* __restrict__ C) {
  FOR_I;
  if (F.material[i] != DV_MATERIAL_FLUID) return;
  if (!in_vortex_domain<D>(P, ldv<D>(F.x, i))) return;
  F.life_time[i] += P.dt;
}

// --------------------------------------------------- export-only fields
// copy_x_temp + compute_vorticity_vis (dimcv_sph.py:778-801)
template <int D>
__global__ void k_vis(dv_params P, DevGrid G, dv_fields F, dv_solver_fields S,
                      const dv_counters* __restrict__ C) {
  FOR_I;
  V3 xi = ldv<D>(F.x, i);
  stv<D>(S.x_temp, i, xi);
  if (F.material[i] != DV_MATERIAL_FLUID) {
    st4(S.vorticity_vis, i, V3{0.f, 0.f, 0.f});
    return;
  }
  float w = F.m_V[i] * cubic_W(P, 0.0f);
  V3 wi = ld4(F.vorticity, i);
  V3 vort{w * wi.x, w * wi.y, w * wi.z};
  float ws = w;
  for_each_neighbor<D>(P, G, F.x, i, xi, [&](int j, V3, float r2) {
    float wj = F.m_V[j] * cubic_W(P, sqrtf(r2));
    V3 oj = ld4(F.vorticity, j);
    vort.x += wj * oj.x;
    vort.y += wj * oj.y;
    vort.z += wj * oj.z;
    ws += wj;
  });
  float den = ws + 1e-6f;
  st4(S.vorticity_vis, i, V3{vort.x / den, vort.y / den, vort.z / den});
}

// ------------------------------------------------------------- host side
#define LAUNCH_D(kern, nb, ...)                                 \
  do {                                                          \
    if (c->p.dim == 2)                                          \
      kern<2><<<(nb), DV_THREADS, 0, c->stream>>>(__VA_ARGS__); \
    else                                                        \
      kern<3><<<(nb), DV_THREADS, 0, c->stream>>>(__VA_ARGS__); \
    DV_LAUNCHED(c);                                             \
  } while (0)

static inline int nblk(const dv_ctx* c) { return dv_blocks(std::min<int64_t>(c->n_upper, c->cap)); }

static int check_solver(dv_ctx* c, const dv_solver_fields* s) {
  if (!s || !s->v_star || !s->grad_v || !s->d_vort || !s->d_vort_smoothed || !s->kvn || !s->kden ||
      !s->x_temp || !s->vorticity_vis || !s->sample_idx)
    return dv_fail(c, DV_EINVAL, "a dv_solver_fields pointer is NULL");
  return DV_OK;
}

DV_API int dv_dimcv_vorticity(dv_ctx* c, const dv_fields* f, const dv_solver_fields* s) {
  if (!c || !f) return DV_EINVAL;
  if (int rc = check_solver(c, s)) return rc;
  LAUNCH_D(k_vorticity, nblk(c), c->p, dv_grid(c), *f, *s, c->d_cnt);
  return DV_OK;
}

DV_API int dv_vorticity_dvort(dv_ctx* c, const dv_fields* f, const dv_solver_fields* s) {
  if (!c || !f) return DV_EINVAL;
  if (int rc = check_solver(c, s)) return rc;
  LAUNCH_D(k_vorticity_dvort, nblk(c), c->p, dv_grid(c), *f, *s, c->d_cnt);
  return DV_OK;
}

DV_API int dv_d_vorticity(dv_ctx* c, const dv_fields* f, const dv_solver_fields* s) {
  if (!c || !f) return DV_EINVAL;
  if (int rc = check_solver(c, s)) return rc;
  LAUNCH_D(k_d_vorticity, nblk(c), c->p, dv_grid(c), *f, *s, c->d_cnt);
  return DV_OK;
}

DV_API int dv_smooth_d_vort(dv_ctx* c, const dv_fields* f, const dv_solver_fields* s) {
  if (!c || !f) return DV_EINVAL;
  if (int rc = check_solver(c, s)) return rc;
  LAUNCH_D(k_smooth, nblk(c), c->p, dv_grid(c), *f, *s, c->d_cnt);
  return DV_OK;
}

DV_API int dv_kvn_sample(dv_ctx* c, const dv_fields* f, const dv_solver_fields* s, uint64_t seed,
                         uint64_t step, int32_t birth_death) {
  if (!c || !f) return DV_EINVAL;
  if (int rc = check_solver(c, s)) return rc;
  LAUNCH_D(k_kvn_sample, nblk(c), c->p, *f, *s, c->d_cnt, (uint32_t)seed, (uint32_t)(seed >> 32),
           (uint32_t)step, (uint32_t)(step >> 32), (int)birth_death);
  return DV_OK;
}

DV_API int dv_record_samples(dv_ctx* c, const dv_fields* f, const dv_solver_fields* s) {
  if (!c || !f) return DV_EINVAL;
  if (int rc = check_solver(c, s)) return rc;
  const int m = (int)std::min<int64_t>(c->n_upper, c->cap) + 1;
  const int nb = dv_blocks(m);
  k_flag_samples<<<nb, DV_THREADS, 0, c->stream>>>(*f, c->d_cnt, m, c->flags);
  DV_LAUNCHED(c);
  int rc = dv_scan_u32(c, c->flags, c->offs, m);
  if (rc) return rc;
  k_compact<<<nb, DV_THREADS, 0, c->stream>>>(c->flags, c->offs, m, s->sample_idx);
  DV_LAUNCHED(c);
  k_store_count<<<1, 1, 0, c->stream>>>(c->offs, c->d_cnt, 0);
  DV_LAUNCHED(c);
  return DV_OK;
}

DV_API int dv_akde(dv_ctx* c, const dv_fields* f, const dv_solver_fields* s) {
  if (!c || !f) return DV_EINVAL;
  if (int rc = check_solver(c, s)) return rc;
  const int nb = nblk(c);
  LAUNCH_D(k_akde, nb, c->p, dv_grid(c), *f, *s, c->d_cnt, c->red_part);
  k_akde_finalize<<<1, 1024, 0, c->stream>>>(c->red_part, nb, c->d_cnt);
  DV_LAUNCHED(c);
  return DV_OK;
}

DV_API int dv_smooth_akde(dv_ctx* c, const dv_fields* f, const dv_solver_fields* s) {
  if (!c || !f) return DV_EINVAL;
  if (int rc = check_solver(c, s)) return rc;
  const int nb = nblk(c);
  LAUNCH_D(k_smooth_akde, nb, c->p, dv_grid(c), *f, *s, c->d_cnt, c->red_part);
  k_akde_finalize<<<1, 1024, 0, c->stream>>>(c->red_part, nb, c->d_cnt);
  DV_LAUNCHED(c);
  return DV_OK;
}

DV_API int dv_sample(dv_ctx* c, const dv_fields* f, const dv_solver_fields* s, int32_t mode,
                     uint64_t seed, uint64_t step, int32_t M) {
  if (!c || !f) return DV_EINVAL;
  if (int rc = check_solver(c, s)) return rc;
  if (M < 0 || M > c->cap) return dv_fail(c, DV_EINVAL, "dv_sample: M=%d outside [0, capacity]", M);
  if (mode == DV_SAMPLE_BERNOULLI) {
    return dv_record_samples(c, f, s);
  } else if (mode == DV_SAMPLE_INJECTED) {
    k_set_num_samples<<<1, 1, 0, c->stream>>>(c->d_cnt, M);
    DV_LAUNCHED(c);
    return DV_OK;
  } else if (mode != DV_SAMPLE_INVERSE_CDF && mode != DV_SAMPLE_STRATIFIED) {
    return dv_fail(c, DV_EINVAL, "dv_sample: unknown mode %d", mode);
  }
  int rc = dv_build_targets(c, f);
  if (rc) return rc;
  const int m = (int)std::min<int64_t>(c->n_upper, c->cap);
  k_cdf_weights<<<dv_blocks(m), DV_THREADS, 0, c->stream>>>(c->targets, s->kden, c->d_cnt, m,
                                                          reinterpret_cast<double*>(c->near_v));
  DV_LAUNCHED(c);
  // near_v (16 B per slot) is free scratch here: it holds the FP64 weights
  rc = dv_scan_f64(c, reinterpret_cast<double*>(c->near_v), c->cdf, m);
  if (rc) return rc;
  k_cdf_draw<<<dv_blocks(std::max(M, 1)), DV_THREADS, 0, c->stream>>>(
      c->cdf, c->targets, s->kden, c->d_cnt, M, (uint32_t)seed, (uint32_t)(seed >> 32),
      (uint32_t)step, (uint32_t)(step >> 32), mode == DV_SAMPLE_STRATIFIED ? 1 : 0, s->sample_idx);
  DV_LAUNCHED(c);
  return DV_OK;
}

DV_API int dv_life_time(dv_ctx* c, const dv_fields* f) {
  if (!c || !f) return DV_EINVAL;
  LAUNCH_D(k_life_time, nblk(c), c->p, *f, c->d_cnt);
  return DV_OK;
}

DV_API int dv_vis(dv_ctx* c, const dv_fields* f, const dv_solver_fields* s) {
  if (!c || !f) return DV_EINVAL;
  if (int rc = check_solver(c, s)) return rc;
  LAUNCH_D(k_vis, nblk(c), c->p, dv_grid(c), *f, *s, c->d_cnt);
  return DV_OK;
}
