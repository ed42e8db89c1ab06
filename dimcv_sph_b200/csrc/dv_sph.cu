// DFSPH sweeps of the DIMCV-SPH substep (reference: DIMCVSPHSolver /
// SPHBase, dimcv_sph.py:86-226, 337-614; sph_base.py:91-112).  One thread
// per particle slot in the cell-sorted order; each per-pair expression keeps
// the reference's operation order (compiled with -fmad=false, IEEE div/sqrt).
// The Jacobi loops run on the device: every iteration kernel returns at once
// when the solve's done flag is set, so the host launches iterations in
// chunks and polls the flag once per chunk instead of once per iteration.
#include <algorithm>

#include "dv_internal.cuh"

#define FOR_I                                      \
  int i = blockIdx.x * blockDim.x + threadIdx.x;   \
  if (i >= C->n) return;

// --------------------------------------------------------- boundary volume
// compute_static_boundary_volume (sph_base.py:91-103) for the static solids,
// compute_moving_boundary_volume (:105-112) for the dynamic ones
template <int D>
__global__ void k_boundary_volume(dv_params P, DevGrid G, dv_fields F, const dv_counters* __restrict__ C,
                                  int dynamic) {
  FOR_I;
  if (!(F.material[i] == DV_MATERIAL_SOLID && (F.is_dynamic[i] != 0) == (dynamic != 0))) return;
  V3 xi = ldv<D>(F.x, i);
  float delta = cubic_W(P, 0.0f);
  for_each_neighbor_m<D>(P, G, F.x, F.material, i, xi, [&](int j, V3, float r2, int mj) {
    if (mj == DV_MATERIAL_SOLID) delta += cubic_W(P, sqrtf(r2));
  });
  F.m_V[i] = 1.0f / delta * 3.0f;
}

// ---------------------------------------------------------------- density
// compute_densities (dimcv_sph.py:126-148)
template <int D>
__global__ void k_densities(dv_params P, DevGrid G, dv_fields F, const dv_counters* __restrict__ C) {
  FOR_I;
  if (F.material[i] != DV_MATERIAL_FLUID) return;
  V3 xi = ldv<D>(F.x, i);
  float dens = F.m_V[i] * cubic_W(P, 0.0f);
  float den = 0.0f;
  for_each_neighbor_m<D>(P, G, F.x, F.material, i, xi, [&](int j, V3, float r2, int mj) {
    if (mj == DV_MATERIAL_FLUID || mj == DV_MATERIAL_SOLID) den += F.m_V[j] * cubic_W(P, sqrtf(r2));
  });
  dens += den;
  dens *= P.density0;
  F.density[i] = dens;
}

// ---------------------------------------------------------- DFSPH factor
// compute_DFSPH_factor (dimcv_sph.py:86-124)
template <int D>
__global__ void k_dfsph_factor(dv_params P, DevGrid G, dv_fields F, const dv_counters* __restrict__ C) {
  FOR_I;
  if (F.material[i] != DV_MATERIAL_FLUID) return;
  V3 xi = ldv<D>(F.x, i);
  V3 gi{0.f, 0.f, 0.f};
  float sum_k = 0.0f;
  for_each_neighbor_m<D>(P, G, F.x, F.material, i, xi, [&](int j, V3 r, float r2, int mj) {
    if (mj == DV_MATERIAL_FLUID) {
      V3 gw = cubic_gradW<D>(P, r, r2);
      float mm = F.m[j];
      V3 g{mm * gw.x, mm * gw.y, mm * gw.z};
      sum_k += sqnorm<D>(g);
      gi.x += g.x;
      gi.y += g.y;
      if (D == 3) gi.z += g.z;
    } else if (mj == DV_MATERIAL_SOLID) {
      V3 gw = cubic_gradW<D>(P, r, r2);
      float s = F.m_V[j] * P.density0;
      gi.x += s * gw.x;
      gi.y += s * gw.y;
      if (D == 3) gi.z += s * gw.z;
    }
  });
  sum_k += sqnorm<D>(gi);
  F.dfsph_factor[i] = sum_k > P.factor_min ? 1.0f / sum_k : 0.0f;
}

// compute_densities + compute_DFSPH_factor in one neighbour walk: the two
// reference sweeps visit the same neighbours in the same order, and each sum
// here is built by the same operations in that order, so density and factor
// are bit-identical to k_densities and k_dfsph_factor; the list, position and
// material of each neighbour are read once instead of twice.  With DC the
// same walk also does the compute_density_change that opens the divergence
// solve (dimcv_sph.py:337-374): it reads only v, x and m_V, which neither of
// the two sweeps changes, and shares their ∇W; density_adv is bit-identical
// to k_density_change's.
template <int D, bool DC>
__device__ __forceinline__ void densities_factor_body(const dv_params& P, const DevGrid& G, const dv_fields& F,
                                                      const dv_counters* __restrict__ C) {
  FOR_I;
  if (F.material[i] != DV_MATERIAL_FLUID) return;
  V3 xi = ldv<D>(F.x, i);
  V3 vi = DC ? ldv<D>(F.v, i) : V3{0.f, 0.f, 0.f};
  float dens = F.m_V[i] * cubic_W(P, 0.0f);
  float den = 0.0f;
  V3 gi{0.f, 0.f, 0.f};
  float sum_k = 0.0f;
  float adv = 0.0f;
  int nn = 0;
  for_each_neighbor_m<D>(P, G, F.x, F.material, i, xi, [&](int j, V3 r, float r2, int mj) {
    if (mj == DV_MATERIAL_FLUID || mj == DV_MATERIAL_SOLID) {
      const float mvj = F.m_V[j];
      den += mvj * cubic_W(P, sqrtf(r2));
      V3 gw = cubic_gradW<D>(P, r, r2);
      if (mj == DV_MATERIAL_FLUID) {
        float mm = F.m[j];
        V3 g{mm * gw.x, mm * gw.y, mm * gw.z};
        sum_k += sqnorm<D>(g);
        gi.x += g.x;
        gi.y += g.y;
        if (D == 3) gi.z += g.z;
      } else {
        float s = mvj * P.density0;
        gi.x += s * gw.x;
        gi.y += s * gw.y;
        if (D == 3) gi.z += s * gw.z;
      }
      if (DC) {
        V3 vj = ldv<D>(F.v, j);
        V3 dv{vi.x - vj.x, vi.y - vj.y, vi.z - vj.z};
        adv += mvj * dot<D>(dv, gw);
      }
    }
    nn += 1;
  });
  dens += den;
  dens *= P.density0;
  F.density[i] = dens;
  sum_k += sqnorm<D>(gi);
  F.dfsph_factor[i] = sum_k > P.factor_min ? 1.0f / sum_k : 0.0f;
  if (DC) {
    float da = fmaxf(adv, 0.0f);
    if (nn < P.neighbor_min) da = 0.0f;
    F.density_adv[i] = da;
  }
}

// multiply_time_step (dimcv_sph.py:395-399)
__global__ void k_scale_factor(dv_fields F, float s, const dv_counters* __restrict__ C) {
  FOR_I;
  if (F.material[i] == DV_MATERIAL_FLUID) F.dfsph_factor[i] *= s;
}

// ------------------------------------------------------- density change
// compute_density_change (dimcv_sph.py:337-374) of slot i; returns the
// compute_density_error(0) term (dimcv_sph.py:407-419), 0 for non-fluid.
template <int D>
__device__ __forceinline__ double density_change_one(const dv_params& P, const DevGrid& G, const dv_fields& F,
                                                     int i) {
  if (F.material[i] != DV_MATERIAL_FLUID) return 0.0;
  V3 xi = ldv<D>(F.x, i);
  V3 vi = ldv<D>(F.v, i);
  float adv = 0.0f;
  int nn = 0;
  for_each_neighbor_m<D>(P, G, F.x, F.material, i, xi, [&](int j, V3 r, float r2, int mj) {
    if (mj == DV_MATERIAL_FLUID || mj == DV_MATERIAL_SOLID) {
      V3 vj = ldv<D>(F.v, j);
      V3 dv{vi.x - vj.x, vi.y - vj.y, vi.z - vj.z};
      adv += F.m_V[j] * dot<D>(dv, cubic_gradW<D>(P, r, r2));
    }
    nn += 1;
  });
  float da = fmaxf(adv, 0.0f);
  if (nn < P.neighbor_min) da = 0.0f;
  F.density_adv[i] = da;
  float term = P.has_transit ? transit_weight(P, xi.x) * (da - 0.0f) : (da - 0.0f);
  return (double)term;
}

// density_change_one and, in the same walk, compute_non_pressure_forces
// (dimcv_sph.py:150-208) of slot i: the fluid neighbours' viscosity term
// takes v_i - v_j, ∇W and m_V_j from the density change and adds up in the
// visit order with the operations of k_nonpressure, so the acceleration is
// bit-identical to k_nonpressure's for the same v.  Every slot gets its
// acceleration as k_nonpressure writes it (static solids 0, other non-fluid
// slots gravity).
template <int D>
__device__ __forceinline__ double density_change_np_one(const dv_params& P, const DevGrid& G, const dv_fields& F,
                                                        int i) {
  const int mi = F.material[i];
  const V3 g{P.gravity[0], P.gravity[1], D == 3 ? P.gravity[2] : 0.0f};
  if (mi != DV_MATERIAL_FLUID) {
    stv<D>(F.acceleration, i, (mi == DV_MATERIAL_SOLID && !F.is_dynamic[i]) ? V3{0.f, 0.f, 0.f} : g);
    return 0.0;
  }
  V3 xi = ldv<D>(F.x, i);
  V3 vi = ldv<D>(F.v, i);
  float adv = 0.0f;
  int nn = 0;
  V3 acc = g;
  for_each_neighbor_m<D>(P, G, F.x, F.material, i, xi, [&](int j, V3 r, float r2, int mj) {
    if (mj == DV_MATERIAL_FLUID || mj == DV_MATERIAL_SOLID) {
      V3 vj = ldv<D>(F.v, j);
      V3 dv{vi.x - vj.x, vi.y - vj.y, vi.z - vj.z};
      const float mvj = F.m_V[j];
      V3 gw = cubic_gradW<D>(P, r, r2);
      adv += mvj * dot<D>(dv, gw);
      if (mj == DV_MATERIAL_FLUID) {
        float v_xy = dot<D>(dv, r);
        float rn = sqrtf(r2);
        float s = P.visc_coef * mvj * v_xy / (rn * rn + P.visc_h2);
        acc.x += s * gw.x;
        acc.y += s * gw.y;
        if (D == 3) acc.z += s * gw.z;
      }
    }
    nn += 1;
  });
  stv<D>(F.acceleration, i, acc);
  float da = fmaxf(adv, 0.0f);
  if (nn < P.neighbor_min) da = 0.0f;
  F.density_adv[i] = da;
  float term = P.has_transit ? transit_weight(P, xi.x) * (da - 0.0f) : (da - 0.0f);
  return (double)term;
}

// optionally the FP64 block partial of the error terms
template <int D>
__global__ void k_density_change(dv_params P, DevGrid G, dv_fields F, const dv_counters* __restrict__ C,
                                 const int32_t* __restrict__ done, double* __restrict__ part) {
  if (done && *done) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double err = 0.0;
  if (i < C->n) err = density_change_one<D>(P, G, F, i);
  if (part) {
    double s = block_sum<double>(err);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
  }
}

// the divergence Jacobi loop's residual sweep with the non-pressure forces
template <int D>
__global__ void k_density_change_np(dv_params P, DevGrid G, dv_fields F, const dv_counters* __restrict__ C,
                                    const int32_t* __restrict__ done, double* __restrict__ part) {
  if (*done) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double err = 0.0;
  if (i < C->n) err = density_change_np_one<D>(P, G, F, i);
  double s = block_sum<double>(err);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// ------------------------------------------------------------ density adv
// compute_density_adv (dimcv_sph.py:470-493) of slot i; returns the
// compute_density_error(density0) term, 0 for non-fluid.
template <int D>
__device__ __forceinline__ double density_adv_one(const dv_params& P, const DevGrid& G, const dv_fields& F,
                                                  int i) {
  if (F.material[i] != DV_MATERIAL_FLUID) return 0.0;
  V3 xi = ldv<D>(F.x, i);
  V3 vi = ldv<D>(F.v, i);
  float delta = 0.0f;
  for_each_neighbor_m<D>(P, G, F.x, F.material, i, xi, [&](int j, V3 r, float r2, int mj) {
    if (mj == DV_MATERIAL_FLUID) {
      V3 vj = ldv<D>(F.v, j);
      V3 dv{vi.x - vj.x, vi.y - vj.y, vi.z - vj.z};
      delta += F.m[j] * dot<D>(dv, cubic_gradW<D>(P, r, r2));
    } else if (mj == DV_MATERIAL_SOLID) {
      V3 vj = ldv<D>(F.v, j);
      V3 dv{vi.x - vj.x, vi.y - vj.y, vi.z - vj.z};
      delta += F.m_V[j] * P.density0 * dot<D>(dv, cubic_gradW<D>(P, r, r2));
    }
  });
  float da = F.density[i] + P.dt * delta;
  da = fmaxf(da, P.density0);
  F.density_adv[i] = da;
  float term = P.has_transit ? transit_weight(P, xi.x) * (da - P.density0) : (da - P.density0);
  return (double)term;
}

template <int D>
__global__ void k_density_adv(dv_params P, DevGrid G, dv_fields F, const dv_counters* __restrict__ C,
                              const int32_t* __restrict__ done, double* __restrict__ part) {
  if (done && *done) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double err = 0.0;
  if (i < C->n) err = density_adv_one<D>(P, G, F, i);
  if (part) {
    double s = block_sum<double>(err);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
  }
}

// The pressure solve's opening density_adv sweep and, in the same walk,
// copy_x_temp + compute_vorticity_vis (dimcv_sph.py:778-801), with the
// operations and order of k_vis: the vis sweep reads x, m_V, material and
// vorticity, which the pressure iterations (they write v) leave unchanged, so
// the solve's first sweep gives what the vis sweep after the solve would.
template <int D>
__global__ void k_density_adv_vis(dv_params P, DevGrid G, dv_fields F, dv_solver_fields S,
                                  const dv_counters* __restrict__ C) {
  FOR_I;
  const V3 xi = ldv<D>(F.x, i);
  stv<D>(S.x_temp, i, xi);
  if (F.material[i] != DV_MATERIAL_FLUID) {
    st4(S.vorticity_vis, i, V3{0.f, 0.f, 0.f});
    return;
  }
  const V3 vi = ldv<D>(F.v, i);
  float delta = 0.0f;
  const float w = F.m_V[i] * cubic_W(P, 0.0f);
  const V3 wi = ld4(F.vorticity, i);
  V3 vort{w * wi.x, w * wi.y, w * wi.z};
  float ws = w;
  for_each_neighbor_m<D>(P, G, F.x, F.material, i, xi, [&](int j, V3 r, float r2, int mj) {
    const float mvj = F.m_V[j];
    if (mj == DV_MATERIAL_FLUID) {
      V3 vj = ldv<D>(F.v, j);
      V3 dv{vi.x - vj.x, vi.y - vj.y, vi.z - vj.z};
      delta += F.m[j] * dot<D>(dv, cubic_gradW<D>(P, r, r2));
    } else if (mj == DV_MATERIAL_SOLID) {
      V3 vj = ldv<D>(F.v, j);
      V3 dv{vi.x - vj.x, vi.y - vj.y, vi.z - vj.z};
      delta += mvj * P.density0 * dot<D>(dv, cubic_gradW<D>(P, r, r2));
    }
    const float wj = mvj * cubic_W(P, sqrtf(r2));
    const V3 oj = ld4(F.vorticity, j);
    vort.x += wj * oj.x;
    vort.y += wj * oj.y;
    vort.z += wj * oj.z;
    ws += wj;
  });
  float da = F.density[i] + P.dt * delta;
  da = fmaxf(da, P.density0);
  F.density_adv[i] = da;
  const float den = ws + 1e-6f;
  st4(S.vorticity_vis, i, V3{vort.x / den, vort.y / den, vort.z / den});
}

// compute_density_error without a preceding sweep (operator surface)
template <int D>
__global__ void k_density_error(dv_params P, dv_fields F, const dv_counters* __restrict__ C,
                                float offset, double* __restrict__ part) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double err = 0.0;
  if (i < C->n && F.material[i] == DV_MATERIAL_FLUID) {
    float da = F.density_adv[i];
    float term;
    if (P.has_transit) {
      V3 xi = ldv<D>(F.x, i);
      term = transit_weight(P, xi.x) * (da - offset);
    } else {
      term = da - offset;
    }
    err = (double)term;
  }
  double s = block_sum<double>(err);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// ---------------------------------------------------- Jacobi iterations
// divergence_solver_iteration_kernel (dimcv_sph.py:421-468)
template <int D>
__device__ __forceinline__ void divergence_iter_one(const dv_params& P, const DevGrid& G, const dv_fields& F,
                                                    int i) {
  if (F.material[i] != DV_MATERIAL_FLUID) return;
  V3 xi = ldv<D>(F.x, i);
  float b_i = F.density_adv[i];
  float k_i = b_i * F.dfsph_factor[i] * F.density[i];
  V3 dv{0.f, 0.f, 0.f};
  const float dt = P.dt;
  for_each_neighbor_m<D>(P, G, F.x, F.material, i, xi, [&](int j, V3 r, float r2, int mj) {
    if (mj == DV_MATERIAL_FLUID) {
      float b_j = F.density_adv[j];
      float k_j = b_j * F.dfsph_factor[j] * F.density[j];
      float k_sum = k_i + k_j;
      if (fabsf(k_sum) > P.m_eps) {
        V3 gw = cubic_gradW<D>(P, r, r2);
        float mm = F.m[j];
        float s = dt * k_sum;
        dv.x -= s * (mm * gw.x);
        dv.y -= s * (mm * gw.y);
        if (D == 3) dv.z -= s * (mm * gw.z);
      }
    } else if (mj == DV_MATERIAL_SOLID) {
      if (fabsf(k_i) > P.m_eps) {
        V3 gw = cubic_gradW<D>(P, r, r2);
        float sm = F.m_V[j] * P.density0;
        float s = -dt * 1.0f * k_i;
        dv.x += s * (sm * gw.x);
        dv.y += s * (sm * gw.y);
        if (D == 3) dv.z += s * (sm * gw.z);
      }
    }
  });
  V3 vi = ldv<D>(F.v, i);
  if (P.has_transit) {
    float w = transit_weight(P, xi.x);
    vi.x += w * dv.x;
    vi.y += w * dv.y;
    if (D == 3) vi.z += w * dv.z;
  } else {
    vi.x += dv.x;
    vi.y += dv.y;
    if (D == 3) vi.z += dv.z;
  }
  stv<D>(F.v, i, vi);
}

// pressure_solve_iteration_kernel (dimcv_sph.py:495-549): the velocity is
// updated pair by pair (the reference writes v[p_i] inside the task).
template <int D>
__device__ __forceinline__ void pressure_iter_one(const dv_params& P, const DevGrid& G, const dv_fields& F,
                                                  int i) {
  if (F.material[i] != DV_MATERIAL_FLUID) return;
  V3 xi = ldv<D>(F.x, i);
  V3 vi = ldv<D>(F.v, i);
  float b_i = F.density_adv[i] - P.density0;
  float k_i = b_i * F.dfsph_factor[i];
  const float dt = P.dt;
  const float w = P.has_transit ? transit_weight(P, xi.x) : 1.0f;
  for_each_neighbor_m<D>(P, G, F.x, F.material, i, xi, [&](int j, V3 r, float r2, int mj) {
    if (mj == DV_MATERIAL_FLUID) {
      float b_j = F.density_adv[j] - P.density0;
      float k_j = b_j * F.dfsph_factor[j];
      float k_sum = k_i + k_j;
      if (fabsf(k_sum) > P.m_eps) {
        V3 gw = cubic_gradW<D>(P, r, r2);
        float mm = F.m[j];
        float s = P.has_transit ? (w * dt) * k_sum : dt * k_sum;
        vi.x -= s * (mm * gw.x);
        vi.y -= s * (mm * gw.y);
        if (D == 3) vi.z -= s * (mm * gw.z);
      }
    } else if (mj == DV_MATERIAL_SOLID) {
      if (fabsf(k_i) > P.m_eps) {
        V3 gw = cubic_gradW<D>(P, r, r2);
        float sm = F.m_V[j] * P.density0;
        float s = -dt * 1.0f * k_i;
        V3 vc{s * (sm * gw.x), s * (sm * gw.y), D == 3 ? s * (sm * gw.z) : 0.0f};
        if (P.has_transit) {
          vi.x += w * vc.x;
          vi.y += w * vc.y;
          if (D == 3) vi.z += w * vc.z;
        } else {
          vi.x += vc.x;
          vi.y += vc.y;
          if (D == 3) vi.z += vc.z;
        }
      }
    }
  });
  stv<D>(F.v, i, vi);
}

// The reaction on dynamic rigid particles of one pressure iteration
// (dimcv_sph.py:540-549): the reference adds, inside the fluid particle's
// task, -vel_change * inv_dt * rho_fluid / rho_solid to the acceleration of
// each dynamic solid neighbour, with atomic adds in no fixed order.  Here each
// dynamic solid gathers the same terms over its fluid neighbours, in its
// neighbour visit order, after the iteration (which leaves every input of the
// terms unchanged): the same sum up to the order of its additions, and
// deterministic.  The divergence solve's reactions (:465-468) are not formed:
// compute_non_pressure_forces overwrites them with gravity before anything
// reads them.
template <int D>
__global__ void k_rigid_reaction(dv_params P, DevGrid G, dv_fields F, const dv_counters* __restrict__ C,
                                 const int32_t* __restrict__ done) {
  if (done && *done) return;
  FOR_I;
  if (!(F.material[i] == DV_MATERIAL_SOLID && F.is_dynamic[i])) return;
  const V3 xi = ldv<D>(F.x, i);
  const float rho_j = F.density[i];
  const float sm = F.m_V[i] * P.density0;
  const float dt = P.dt;
  V3 acc = ldv<D>(F.acceleration, i);
  for_each_neighbor_m<D>(P, G, F.x, F.material, i, xi, [&](int q, V3 r, float r2, int mq) {
    if (mq != DV_MATERIAL_FLUID) return;
    const float k_q = (F.density_adv[q] - P.density0) * F.dfsph_factor[q];
    if (!(fabsf(k_q) > P.m_eps)) return;
    const V3 gw = cubic_gradW<D>(P, V3{-r.x, -r.y, -r.z}, r2);  // at x_q - x_i, as in q's task
    const float s = -dt * 1.0f * k_q;
    const V3 vc{s * (sm * gw.x), s * (sm * gw.y), D == 3 ? s * (sm * gw.z) : 0.0f};
    const float rq = F.density[q];
    acc.x += -vc.x * P.inv_dt * rq / rho_j;
    acc.y += -vc.y * P.inv_dt * rq / rho_j;
    if (D == 3) acc.z += -vc.z * P.inv_dt * rq / rho_j;
  });
  stv<D>(F.acceleration, i, acc);
}

template <int D>
__global__ void k_divergence_iter(dv_params P, DevGrid G, dv_fields F, const dv_counters* __restrict__ C,
                                  const int32_t* __restrict__ done) {
  if (done && *done) return;
  FOR_I;
  divergence_iter_one<D>(P, G, F, i);
}

template <int D>
__global__ void k_pressure_iter(dv_params P, DevGrid G, dv_fields F, const dv_counters* __restrict__ C,
                                const int32_t* __restrict__ done) {
  if (done && *done) return;
  FOR_I;
  pressure_iter_one<D>(P, G, F, i);
}

// Scene batch forms: a grid of a few blocks per SM walks the work list of
// the scenes still iterating (wl[s] = first block of scene s, wl[S] = total,
// blocks of DV_THREADS slots from the scene's start).
__device__ __forceinline__ int wl_scene(const int32_t* __restrict__ wl, int S, int b) {
  int lo = 0, hi = S;  // last s with wl[s] <= b
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (wl[mid] <= b)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo - 1;
}

template <int D, int WHICH>
__global__ void k_batch_iter(dv_params P, DevGrid G, dv_fields F, const dv_scene_state* __restrict__ st,
                             const int32_t* __restrict__ wl, int S) {
  const int tot = wl[S];
  for (int b = blockIdx.x; b < tot; b += gridDim.x) {
    const int s = wl_scene(wl, S, b);
    const int i = st[s].start + (b - wl[s]) * DV_THREADS + threadIdx.x;
    if (i >= st[s].end) continue;
    if (WHICH == 0)
      divergence_iter_one<D>(P, G, F, i);
    else
      pressure_iter_one<D>(P, G, F, i);
  }
}

// residual sweep: FP64 block sum of the error terms of work-list block b
// (a block never spans two scenes) into part[b]; WHICH 2 is the divergence
// residual with the non-pressure forces (density_change_np_one)
template <int D, int WHICH>
__global__ void k_batch_residual(dv_params P, DevGrid G, dv_fields F, const dv_scene_state* __restrict__ st,
                                 const int32_t* __restrict__ wl, int S, double* __restrict__ part) {
  const int tot = wl[S];
  for (int b = blockIdx.x; b < tot; b += gridDim.x) {  // block-uniform bounds
    const int s = wl_scene(wl, S, b);
    const int i = st[s].start + (b - wl[s]) * DV_THREADS + threadIdx.x;
    double e = 0.0;
    if (i < st[s].end)
      e = WHICH == 0   ? density_change_one<D>(P, G, F, i)
          : WHICH == 1 ? density_adv_one<D>(P, G, F, i)
                       : density_change_np_one<D>(P, G, F, i);
    e = block_sum<double>(e);
    if (threadIdx.x == 0) part[b] = e;
  }
}

// convergence test of one Jacobi iteration: average error over the fluid
// count against eta; sets the done flag at convergence or at max_iter
__global__ void k_solve_finalize(const double* __restrict__ part, int nparts, dv_counters* C,
                                 int32_t* done, double eta, int max_iter, int which) {
  if (*done) return;
  double s = 0.0;
  for (int k = threadIdx.x; k < nparts; k += blockDim.x) s += part[k];
  s = block_sum<double>(s);
  if (threadIdx.x == 0) {
    int nf = C->n_fluid;
    double avg = nf > 0 ? s / (double)nf : 0.0;
    int it = (which == 0 ? ++C->iters_div : ++C->iters_p);
    if (which == 0)
      C->err_div = avg;
    else
      C->err_p = avg;
    if (!isfinite(avg)) C->status |= DV_WARN_NAN;
    if (avg <= eta || nf == 0) {
      *done = 1;
    } else if (it >= max_iter) {
      *done = 1;
      C->status |= (which == 0 ? DV_WARN_DIV_NOT_CONVERGED : DV_WARN_P_NOT_CONVERGED);
    }
  }
}

__global__ void k_solve_reset(dv_counters* C, int32_t* done, int which) {
  *done = 0;
  if (which == 0)
    C->iters_div = 0;
  else
    C->iters_p = 0;
}

// ------------------------------------------------------- non-pressure forces
// compute_non_pressure_forces (dimcv_sph.py:150-208).  The surface tension
// coefficient is 0 in the reference (dimcv_sph.py:12) and boundary viscosity
// is 0 (:182), so those terms add exactly zero and are not evaluated.
template <int D>
__global__ void k_nonpressure(dv_params P, DevGrid G, dv_fields F, const dv_counters* __restrict__ C) {
  FOR_I;
  int mi = F.material[i];
  if (mi == DV_MATERIAL_SOLID && !F.is_dynamic[i]) {
    stv<D>(F.acceleration, i, V3{0.f, 0.f, 0.f});
    return;
  }
  V3 dv{P.gravity[0], P.gravity[1], D == 3 ? P.gravity[2] : 0.0f};
  if (mi == DV_MATERIAL_FLUID) {
    V3 xi = ldv<D>(F.x, i);
    V3 vi = ldv<D>(F.v, i);
    for_each_neighbor_m<D>(P, G, F.x, F.material, i, xi, [&](int j, V3 r, float r2, int mj) {
      if (mj == DV_MATERIAL_FLUID) {
        V3 vj = ldv<D>(F.v, j);
        V3 dvij{vi.x - vj.x, vi.y - vj.y, vi.z - vj.z};
        float v_xy = dot<D>(dvij, r);
        float rn = sqrtf(r2);
        float s = P.visc_coef * F.m_V[j] * v_xy / (rn * rn + P.visc_h2);
        V3 gw = cubic_gradW<D>(P, r, r2);
        dv.x += s * gw.x;
        dv.y += s * gw.y;
        if (D == 3) dv.z += s * gw.z;
      }
    });
  }
  stv<D>(F.acceleration, i, dv);
}

// predict_velocity (dimcv_sph.py:220-226)
template <int D>
__global__ void k_predict_velocity(dv_params P, dv_fields F, const dv_counters* __restrict__ C) {
  FOR_I;
  if (!(F.is_dynamic[i] && F.material[i] == DV_MATERIAL_FLUID)) return;
  V3 v = ldv<D>(F.v, i), a = ldv<D>(F.acceleration, i);
  v.x += P.dt * a.x;
  v.y += P.dt * a.y;
  if (D == 3) v.z += P.dt * a.z;
  stv<D>(F.v, i, v);
}

// advect (dimcv_sph.py:210-218)
template <int D>
__global__ void k_advect(dv_params P, dv_fields F, const dv_counters* __restrict__ C) {
  FOR_I;
  if (!F.is_dynamic[i]) return;
  V3 v = ldv<D>(F.v, i);
  if (F.material[i] == DV_MATERIAL_SOLID) {
    V3 a = ldv<D>(F.acceleration, i);
    v.x += P.dt * a.x;
    v.y += P.dt * a.y;
    if (D == 3) v.z += P.dt * a.z;
    stv<D>(F.v, i, v);
  }
  V3 x = ldv<D>(F.x, i);
  x.x += P.dt * v.x;
  x.y += P.dt * v.y;
  if (D == 3) x.z += P.dt * v.z;
  if (P.periodic) {  // wrap into [domain_start, domain_start + box)
    float* c[3] = {&x.x, &x.y, &x.z};
    for (int d = 0; d < D; ++d) {
      if (*c[d] >= P.domain_start[d] + P.box[d]) *c[d] -= P.box[d];
      if (*c[d] < P.domain_start[d]) {
        *c[d] += P.box[d];
        // -tiny + box rounds to box: that point is the start of the axis
        if (*c[d] >= P.domain_start[d] + P.box[d]) *c[d] = P.domain_start[d];
      }
    }
  }
  stv<D>(F.x, i, x);
}

// ------------------------------------------------------------- host side
#define LAUNCH_D(kern, nb, ...)                                                          \
  do {                                                                                   \
    if (c->p.dim == 2)                                                                   \
      kern<2><<<(nb), DV_THREADS, 0, c->stream>>>(__VA_ARGS__);                          \
    else                                                                                 \
      kern<3><<<(nb), DV_THREADS, 0, c->stream>>>(__VA_ARGS__);                          \
    DV_LAUNCHED(c);                                                                      \
  } while (0)

static inline int nblk(const dv_ctx* c) { return dv_blocks(std::min<int64_t>(c->n_upper, c->cap)); }

DV_API int dv_boundary_volume(dv_ctx* c, const dv_fields* f) {
  if (!c || !f) return DV_EINVAL;
  // the stored lists leave static solids' rows empty: scan cells
  LAUNCH_D(k_boundary_volume, nblk(c), c->p, dv_grid_cells(c), *f, c->d_cnt, 0);
  return DV_OK;
}

DV_API int dv_moving_boundary_volume(dv_ctx* c, const dv_fields* f) {
  if (!c || !f) return DV_EINVAL;
  LAUNCH_D(k_boundary_volume, nblk(c), c->p, dv_grid(c), *f, c->d_cnt, 1);
  return DV_OK;
}

DV_API int dv_set_dynamic_rigid(dv_ctx* c, int32_t on) {
  if (!c) return DV_EINVAL;
  if (on && c->batch) return dv_fail(c, DV_EUNSUPPORTED, "dynamic rigid particles in a scene batch are not built");
  c->dyn_rigid = on != 0;
  return DV_OK;
}

DV_API int dv_densities(dv_ctx* c, const dv_fields* f) {
  if (!c || !f) return DV_EINVAL;
  LAUNCH_D(k_densities, nblk(c), c->p, dv_grid(c), *f, c->d_cnt);
  return DV_OK;
}

DV_API int dv_dfsph_factor(dv_ctx* c, const dv_fields* f) {
  if (!c || !f) return DV_EINVAL;
  LAUNCH_D(k_dfsph_factor, nblk(c), c->p, dv_grid(c), *f, c->d_cnt);
  return DV_OK;
}

template <int D>
__global__ void k_densities_factor_only(dv_params P, DevGrid G, dv_fields F, const dv_counters* __restrict__ C) {
  densities_factor_body<D, false>(P, G, F, C);
}
template <int D>
__global__ void k_densities_factor_change(dv_params P, DevGrid G, dv_fields F, const dv_counters* __restrict__ C) {
  densities_factor_body<D, true>(P, G, F, C);
}

DV_API int dv_densities_factor(dv_ctx* c, const dv_fields* f) {
  if (!c || !f) return DV_EINVAL;
  LAUNCH_D(k_densities_factor_only, nblk(c), c->p, dv_grid(c), *f, c->d_cnt);
  return DV_OK;
}

DV_API int dv_densities_factor_change(dv_ctx* c, const dv_fields* f) {
  if (!c || !f) return DV_EINVAL;
  LAUNCH_D(k_densities_factor_change, nblk(c), c->p, dv_grid(c), *f, c->d_cnt);
  return DV_OK;
}

DV_API int dv_scale_factor(dv_ctx* c, const dv_fields* f, float s) {
  if (!c || !f) return DV_EINVAL;
  k_scale_factor<<<nblk(c), DV_THREADS, 0, c->stream>>>(*f, s, c->d_cnt);
  DV_LAUNCHED(c);
  return DV_OK;
}

DV_API int dv_density_change(dv_ctx* c, const dv_fields* f) {
  if (!c || !f) return DV_EINVAL;
  LAUNCH_D(k_density_change, nblk(c), c->p, dv_grid(c), *f, c->d_cnt, (const int32_t*)nullptr,
           (double*)nullptr);
  return DV_OK;
}

DV_API int dv_density_adv(dv_ctx* c, const dv_fields* f) {
  if (!c || !f) return DV_EINVAL;
  LAUNCH_D(k_density_adv, nblk(c), c->p, dv_grid(c), *f, c->d_cnt, (const int32_t*)nullptr,
           (double*)nullptr);
  return DV_OK;
}

DV_API int dv_density_error(dv_ctx* c, const dv_fields* f, float offset, double* out) {
  if (!c || !f || !out) return DV_EINVAL;
  int nb = nblk(c);
  LAUNCH_D(k_density_error, nb, c->p, *f, c->d_cnt, offset, c->red_part);
  double* dst = reinterpret_cast<double*>(c->dscan_part);  // scratch word
  int rc = dv_finalize_sum(c, c->red_part, nb, dst);
  if (rc) return rc;
  DV_CK(c, cudaMemcpyAsync(out, dst, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  DV_CK(c, cudaStreamSynchronize(c->stream));
  return DV_OK;
}

DV_API int dv_divergence_iteration(dv_ctx* c, const dv_fields* f) {
  if (!c || !f) return DV_EINVAL;
  LAUNCH_D(k_divergence_iter, nblk(c), c->p, dv_grid(c), *f, c->d_cnt, (const int32_t*)nullptr);
  return DV_OK;
}

DV_API int dv_pressure_iteration(dv_ctx* c, const dv_fields* f) {
  if (!c || !f) return DV_EINVAL;
  LAUNCH_D(k_pressure_iter, nblk(c), c->p, dv_grid(c), *f, c->d_cnt, (const int32_t*)nullptr);
  if (c->dyn_rigid) LAUNCH_D(k_rigid_reaction, nblk(c), c->p, dv_grid(c), *f, c->d_cnt, (const int32_t*)nullptr);
  return DV_OK;
}

// Runs Jacobi iterations in chunks of 2, 4, 8, ... launches; every iteration
// is (update sweep, residual sweep + FP64 block partials, finalize) and all
// three return at once once the done flag is set.
static int jacobi_loop(dv_ctx* c, const dv_fields* f, int which, bool nonpressure = false) {
  const int nb = nblk(c);
  const int max_iter = which == 0 ? c->p.max_iter_div : c->p.max_iter_p;
  const double eta = which == 0 ? c->p.eta_div : c->p.eta_p;
  int32_t* done = c->d_flag;
  k_solve_reset<<<1, 1, 0, c->stream>>>(c->d_cnt, done, which);
  DV_LAUNCHED(c);
  int launched = 0, chunk = 2;
  while (launched < max_iter) {
    int m = std::min(chunk, max_iter - launched);
    for (int k = 0; k < m; ++k) {
      if (which == 0) {
        LAUNCH_D(k_divergence_iter, nb, c->p, dv_grid(c), *f, c->d_cnt, (const int32_t*)done);
        if (nonpressure)
          LAUNCH_D(k_density_change_np, nb, c->p, dv_grid(c), *f, c->d_cnt, (const int32_t*)done,
                   c->red_part);
        else
          LAUNCH_D(k_density_change, nb, c->p, dv_grid(c), *f, c->d_cnt, (const int32_t*)done,
                   c->red_part);
      } else {
        LAUNCH_D(k_pressure_iter, nb, c->p, dv_grid(c), *f, c->d_cnt, (const int32_t*)done);
        if (c->dyn_rigid) LAUNCH_D(k_rigid_reaction, nb, c->p, dv_grid(c), *f, c->d_cnt, (const int32_t*)done);
        LAUNCH_D(k_density_adv, nb, c->p, dv_grid(c), *f, c->d_cnt, (const int32_t*)done,
                 c->red_part);
      }
      k_solve_finalize<<<1, 1024, 0, c->stream>>>(c->red_part, nb, c->d_cnt, done, eta, max_iter,
                                                  which);
      DV_LAUNCHED(c);
    }
    launched += m;
    if (launched >= max_iter) break;
    DV_CK(c, cudaMemcpyAsync(c->h_flag, done, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    DV_CK(c, cudaStreamSynchronize(c->stream));
    if (*c->h_flag) break;
    chunk *= 2;
  }
  return DV_OK;
}

// Scene batch: the same Jacobi iteration with per-scene convergence.  One
// iteration is (update sweep, residual sweep, per-scene finalize, work list
// of the scenes still iterating).  Eagerly the host polls after chunks of
// 2, 4, 8, ... iterations; under graph capture the iteration is the body of
// a conditional WHILE node whose condition kernel counts its own iterations
// and stops at max_iter whatever the data, or earlier when every scene has
// converged.
static int batch_iteration(dv_ctx* c, const dv_fields* f, int which, bool nonpressure) {
  dv_batch_state* b = c->batch;
  const int grid = c->num_sms * 8;
  const DevGrid G = dv_grid(c);
#define LB(K, ...)                                                                           \
  do {                                                                                       \
    if (c->p.dim == 2)                                                                       \
      which == 0 ? K<2, 0><<<grid, DV_THREADS, 0, c->stream>>>(__VA_ARGS__)                 \
                 : K<2, 1><<<grid, DV_THREADS, 0, c->stream>>>(__VA_ARGS__);                \
    else                                                                                     \
      which == 0 ? K<3, 0><<<grid, DV_THREADS, 0, c->stream>>>(__VA_ARGS__)                 \
                 : K<3, 1><<<grid, DV_THREADS, 0, c->stream>>>(__VA_ARGS__);                \
    DV_LAUNCHED(c);                                                                          \
  } while (0)
  LB(k_batch_iter, c->p, G, *f, b->d_state, b->d_wl, b->S);
  if (which == 0 && nonpressure) {
    if (c->p.dim == 2)
      k_batch_residual<2, 2><<<grid, DV_THREADS, 0, c->stream>>>(c->p, G, *f, b->d_state, b->d_wl, b->S, b->d_err);
    else
      k_batch_residual<3, 2><<<grid, DV_THREADS, 0, c->stream>>>(c->p, G, *f, b->d_state, b->d_wl, b->S, b->d_err);
    DV_LAUNCHED(c);
  } else {
    LB(k_batch_residual, c->p, G, *f, b->d_state, b->d_wl, b->S, b->d_err);
  }
#undef LB
  return dv_batch_solve_finalize(c, which);
}

int dv_batch_solve(dv_ctx* c, const dv_fields* f, int which, bool nonpressure) {
  dv_batch_state* b = c->batch;
  const int max_iter = which == 0 ? c->p.max_iter_div : c->p.max_iter_p;
  int rc = dv_batch_solve_reset(c, which);
  if (rc) return rc;
  if (b->capturing) {
    cudaStream_t st = c->stream;
    cudaStreamCaptureStatus cs;
    unsigned long long id = 0;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    DV_CK(c, cudaStreamGetCaptureInfo(st, &cs, &id, &g, &deps, &nd));
    if (cs != cudaStreamCaptureStatusActive) return dv_fail(c, DV_EINVAL, "dv_batch_solve: stream not capturing");
    cudaGraphConditionalHandle h;
    DV_CK(c, cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    DV_CK(c, cudaGraphAddNode(&node, g, deps, nd, &np));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    DV_CK(c, cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
    DV_CK(c, cudaStreamBeginCaptureToGraph(b->bstream, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    c->stream = b->bstream;
    rc = batch_iteration(c, f, which, nonpressure);
    if (rc == DV_OK) rc = dv_batch_loop_condition(c, h, max_iter);
    c->stream = st;
    cudaGraph_t out = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->bstream, &out);
    if (rc) return rc;
    if (e != cudaSuccess) return dv_cuda_check(c, e, "capture of the Jacobi loop body");
    return DV_OK;
  }
  int launched = 0, chunk = 2;
  while (launched < max_iter) {
    const int m = std::min(chunk, max_iter - launched);
    for (int k = 0; k < m; ++k) {
      rc = batch_iteration(c, f, which, nonpressure);
      if (rc) return rc;
    }
    launched += m;
    if (launched >= max_iter) break;
    DV_CK(c, cudaMemcpyAsync(c->h_flag, b->d_done + b->S, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    DV_CK(c, cudaStreamSynchronize(c->stream));
    if (*c->h_flag) break;
    chunk *= 2;
  }
  return DV_OK;
}

static int read_iters(dv_ctx* c, int which, int32_t* iters) {
  if (!iters) return DV_OK;
  dv_counters cnt;
  int rc = dv_get_counters(c, &cnt);
  if (rc) return rc;
  *iters = which == 0 ? cnt.iters_div : cnt.iters_p;
  return DV_OK;
}

// the residual sweep after the last iteration sees the solved velocity, and
// nothing writes v after it: with DV_SOLVE_NONPRESSURE that sweep's
// accelerations are compute_non_pressure_forces of the result (a loop of no
// iterations runs the sweep itself)
static int divergence_solve(dv_ctx* c, const dv_fields* f, int32_t* iters, int32_t flags) {
  const bool nonpressure = (flags & DV_SOLVE_NONPRESSURE) != 0;
  int rc = (flags & DV_SOLVE_PREPARED) ? DV_OK : dv_density_change(c, f);
  if (rc) return rc;
  rc = dv_scale_factor(c, f, c->p.inv_dt);
  if (rc) return rc;
  rc = jacobi_loop(c, f, 0, nonpressure);
  if (rc) return rc;
  if (nonpressure && c->p.max_iter_div < 1) {
    rc = dv_nonpressure(c, f);
    if (rc) return rc;
  }
  rc = dv_scale_factor(c, f, c->p.dt);
  if (rc) return rc;
  return read_iters(c, 0, iters);
}

DV_API int dv_divergence_solve(dv_ctx* c, const dv_fields* f, int32_t* iters) {
  if (!c || !f) return DV_EINVAL;
  return divergence_solve(c, f, iters, 0);
}

DV_API int dv_divergence_solve_prepared(dv_ctx* c, const dv_fields* f, int32_t* iters) {
  if (!c || !f) return DV_EINVAL;
  return divergence_solve(c, f, iters, DV_SOLVE_PREPARED);
}

DV_API int dv_divergence_solve_ex(dv_ctx* c, const dv_fields* f, int32_t flags, int32_t* iters) {
  if (!c || !f) return DV_EINVAL;
  if (flags & ~(DV_SOLVE_PREPARED | DV_SOLVE_NONPRESSURE))
    return dv_fail(c, DV_EINVAL, "dv_divergence_solve_ex: unknown flags 0x%x", (unsigned)flags);
  return divergence_solve(c, f, iters, flags);
}

DV_API int dv_pressure_solve_ex(dv_ctx* c, const dv_fields* f, const dv_solver_fields* s, int32_t flags,
                                int32_t* iters) {
  if (!c || !f) return DV_EINVAL;
  if (flags & ~DV_SOLVE_VIS)
    return dv_fail(c, DV_EINVAL, "dv_pressure_solve_ex: unknown flags 0x%x", (unsigned)flags);
  int rc;
  if (flags & DV_SOLVE_VIS) {
    if (!s || !s->x_temp || !s->vorticity_vis)
      return dv_fail(c, DV_EINVAL, "dv_pressure_solve_ex: DV_SOLVE_VIS needs x_temp and vorticity_vis");
    LAUNCH_D(k_density_adv_vis, nblk(c), c->p, dv_grid(c), *f, *s, c->d_cnt);
    rc = DV_OK;
  } else {
    rc = dv_density_adv(c, f);
  }
  if (rc) return rc;
  rc = dv_scale_factor(c, f, c->p.inv_dt2);
  if (rc) return rc;
  rc = jacobi_loop(c, f, 1);
  if (rc) return rc;
  return read_iters(c, 1, iters);
}

DV_API int dv_pressure_solve(dv_ctx* c, const dv_fields* f, int32_t* iters) {
  if (!c || !f) return DV_EINVAL;
  int rc = dv_density_adv(c, f);
  if (rc) return rc;
  rc = dv_scale_factor(c, f, c->p.inv_dt2);
  if (rc) return rc;
  rc = jacobi_loop(c, f, 1);
  if (rc) return rc;
  return read_iters(c, 1, iters);
}

DV_API int dv_nonpressure(dv_ctx* c, const dv_fields* f) {
  if (!c || !f) return DV_EINVAL;
  LAUNCH_D(k_nonpressure, nblk(c), c->p, dv_grid(c), *f, c->d_cnt);
  return DV_OK;
}

DV_API int dv_predict_velocity(dv_ctx* c, const dv_fields* f) {
  if (!c || !f) return DV_EINVAL;
  LAUNCH_D(k_predict_velocity, nblk(c), c->p, *f, c->d_cnt);
  return DV_OK;
}

// enforce_boundary_2D / _3D with simulate_collisions (sph_base.py:118-179,
// called at karman_vortex.py:226-230): every slot of the capacity whose
// material is `material` and that is dynamic is clamped into [lo, hi] per
// axis (a coordinate above hi goes to hi, one at or below lo to lo), and if
// any axis was clamped its velocity loses (1 + c_f) of its component along
// the normalised sum of the face normals, c_f = 0.5.
template <int D>
__global__ void k_enforce_boundary(dv_fields F, int64_t cap, int material, float lo0, float lo1, float lo2,
                                   float hi0, float hi1, float hi2) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= cap) return;
  if (!(F.material[i] == material && F.is_dynamic[i])) return;
  const V3 pos = ldv<D>(F.x, (int)i);
  V3 x = pos, n{0.f, 0.f, 0.f};
  const float lo[3] = {lo0, lo1, lo2}, hi[3] = {hi0, hi1, hi2};
  const float p[3] = {pos.x, pos.y, pos.z};
  float* xs[3] = {&x.x, &x.y, &x.z};
  float* ns[3] = {&n.x, &n.y, &n.z};
#pragma unroll
  for (int d = 0; d < D; ++d) {
    if (p[d] > hi[d]) {
      *ns[d] += 1.0f;
      *xs[d] = hi[d];
    }
    if (p[d] <= lo[d]) {
      *ns[d] += -1.0f;
      *xs[d] = lo[d];
    }
  }
  stv<D>(F.x, (int)i, x);
  const float len = sqrtf(sqnorm<D>(n));
  if (len > 1.0e-6f) {
    const V3 e{n.x / len, n.y / len, D == 3 ? n.z / len : 0.0f};
    V3 v = ldv<D>(F.v, (int)i);
    const float s = (1.0f + 0.5f) * dot<D>(v, e);
    v.x -= s * e.x;
    v.y -= s * e.y;
    if (D == 3) v.z -= s * e.z;
    stv<D>(F.v, (int)i, v);
  }
}

DV_API int dv_enforce_boundary(dv_ctx* c, const dv_fields* f, int32_t material, const float* lo, const float* hi) {
  if (!c || !f || !lo || !hi) return DV_EINVAL;
  const int nb = dv_blocks(c->cap);
  if (c->p.dim == 2)
    k_enforce_boundary<2><<<nb, DV_THREADS, 0, c->stream>>>(*f, c->cap, material, lo[0], lo[1], 0.f, hi[0], hi[1],
                                                            0.f);
  else
    k_enforce_boundary<3><<<nb, DV_THREADS, 0, c->stream>>>(*f, c->cap, material, lo[0], lo[1], lo[2], hi[0], hi[1],
                                                            hi[2]);
  DV_LAUNCHED(c);
  return dv_invalidate_lists(c);  // positions moved
}

DV_API int dv_advect(dv_ctx* c, const dv_fields* f) {
  if (!c || !f) return DV_EINVAL;
  LAUNCH_D(k_advect, nblk(c), c->p, *f, c->d_cnt);
  return dv_invalidate_lists(c);  // positions moved
}
