// Scene batch: S independent scenes stepped together (new: the reference
// steps one scene per process).  One context holds every scene; a slot's
// scene id is its object_id, positions are scene-local, and the cell key
// carries the scene id above the Morton bits, so the sort keeps each scene
// contiguous and the neighbour sweeps of the single-scene path run on the
// whole batch without ever crossing scenes.  This unit holds the per-scene
// pieces: emission on the device, scene ranges and counts after the sort,
// the per-scene DFSPH convergence test, kden_sum, the sample / target / tile
// offsets, the step orchestration and its CUDA-graph capture.  Every
// per-scene reduction is one block per scene summing its slots in a fixed
// order, so a batch step is deterministic.
#include <algorithm>
#include <vector>

#include "dv_internal.cuh"

namespace {

// exclusive scan of v over the threads of one block (blockDim.x <= 1024);
// returns the thread's offset, *total gets the sum
__device__ __forceinline__ int block_excl_scan(int v, int* total) {
  __shared__ int part[1024];
  const int tid = threadIdx.x, nt = blockDim.x;
  __syncthreads();
  part[tid] = v;
  __syncthreads();
  for (int o = 1; o < nt; o <<= 1) {  // inclusive Hillis-Steele scan
    const int u = tid >= o ? part[tid - o] : 0;
    __syncthreads();
    part[tid] += u;
    __syncthreads();
  }
  *total = part[nt - 1];
  return part[tid] - v;
}

// ---------------------------------------------------------------- emission
// emit_particle (dimcv_sph.py:616-637) for every scene whose interval
// divides the step counter: its emitter lattice is appended after the
// current particles with the fields dv_add_particles writes.
template <int D>
__global__ void k_batch_emit(dv_fields F, const dv_batch_scene* __restrict__ sc, int S,
                             const float* __restrict__ pos, const int64_t* __restrict__ step, dv_counters* C,
                             int cap, dv_scene_state* st) {
  extern __shared__ int off[];  // [S + 1]
  const int64_t t = *step;
  {
    const int per = (S + blockDim.x - 1) / blockDim.x;
    const int s0 = min(S, (int)threadIdx.x * per), s1 = min(S, s0 + per);
    int mine = 0;
    for (int s = s0; s < s1; ++s) {
      const int iv = sc[s].emit_interval;
      if (iv > 0 && sc[s].emit_count > 0 && t % iv == 0) mine += sc[s].emit_count;
    }
    int total;
    int o = block_excl_scan(mine, &total);
    for (int s = s0; s < s1; ++s) {
      off[s] = o;
      const int iv = sc[s].emit_interval;
      if (iv > 0 && sc[s].emit_count > 0 && t % iv == 0) o += sc[s].emit_count;
    }
    if (threadIdx.x == 0) off[S] = total;
  }
  __syncthreads();
  const int n0 = C->n, total = off[S];
  const int room = cap - n0 > 0 ? cap - n0 : 0;
  const int added = total < room ? total : room;
  for (int k = threadIdx.x; k < added; k += blockDim.x) {
    int lo = 0, hi = S;  // scene: last s with off[s] <= k
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (off[mid] <= k)
        lo = mid + 1;
      else
        hi = mid;
    }
    const int s = lo - 1;
    const int e = sc[s].emit_offset + (k - off[s]);
    const int p = n0 + k;
    const V3 x{pos[e * D], pos[e * D + 1], D == 3 ? pos[e * D + 2] : 0.0f};
    const V3 v{sc[s].emit_velocity[0], sc[s].emit_velocity[1], D == 3 ? sc[s].emit_velocity[2] : 0.0f};
    const float rho = sc[s].emit_density, m_V0 = sc[s].emit_volume;
    stv<D>(F.x, p, x);
    stv<D>(F.x0, p, x);
    stv<D>(F.v, p, v);
    stv<D>(F.acceleration, p, V3{0.f, 0.f, 0.f});
    st4(F.vorticity, p, V3{0.f, 0.f, 0.f});
    F.object_id[p] = s;
    F.density[p] = rho;
    F.m_V[p] = m_V0;
    F.m[p] = m_V0 * rho;  // particle_system.py:325
    F.pressure[p] = 0.0f;
    F.material[p] = DV_MATERIAL_FLUID;
    F.is_dynamic[p] = 1;
    reinterpret_cast<int4*>(F.color)[p] =
        make_int4(sc[s].emit_color[0], sc[s].emit_color[1], sc[s].emit_color[2], 0);
    F.is_active[p] = 1;
    F.dfsph_factor[p] = 0.0f;
    F.density_adv[p] = 0.0f;
    F.is_sample[p] = 0;
    F.life_time[p] = 0.0f;
    F.grid_ids[p] = -1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    C->n = n0 + added;
    C->n_fluid += added;
    if (added < total) C->status |= DV_WARN_CAPACITY;
  }
  for (int s = threadIdx.x; s < S; s += blockDim.x) {
    const int a = min(off[s], added), b = min(off[s + 1], added);
    st[s].emitted += b - a;
    if (b - a < off[s + 1] - off[s]) st[s].status |= DV_WARN_CAPACITY;
  }
}

// ----------------------------------------------------- ranges and counts
__global__ void k_batch_clear_ranges(dv_scene_state* st, int S) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < S) {
    st[s].start = 0;
    st[s].end = 0;
  }
}

// scene ranges from the sorted keys (scene id above `shift` bits)
__global__ void k_batch_ranges(const uint32_t* __restrict__ keys, const dv_counters* __restrict__ C, int shift,
                               int S, dv_scene_state* st) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = C->n;
  if (p >= n) return;
  // a batch of one scene has no scene bits in its keys: every active slot is scene 0
  auto scene = [&](uint32_t k) { return S == 1 ? 0 : (int)(k >> shift); };
  const int s = scene(keys[p]);
  if (s < 0 || s >= S) return;
  if (p == 0 || scene(keys[p - 1]) != s) st[s].start = p;
  if (p == n - 1 || scene(keys[p + 1]) != s) st[s].end = p + 1;
}

// fluid / solid / target counts per scene (one block per scene)
template <int D>
__global__ void k_batch_counts(dv_params P, dv_fields F, dv_scene_state* st) {
  const int s = blockIdx.x;
  const int a = st[s].start, b = st[s].end;
  int fl = 0, so = 0, tg = 0;
  for (int i = a + threadIdx.x; i < b; i += blockDim.x) {
    const int m = F.material[i];
    fl += m == DV_MATERIAL_FLUID;
    so += m == DV_MATERIAL_SOLID;
    tg += m == DV_MATERIAL_FLUID && in_vortex_domain<D>(P, ldv<D>(F.x, i));
  }
  fl = block_sum<int>(fl);
  so = block_sum<int>(so);
  tg = block_sum<int>(tg);
  if (threadIdx.x == 0) {
    st[s].n_fluid = fl;
    st[s].n_solid = so;
    st[s].n_targets = tg;
  }
}

// kden_sum of every scene (compute_kernel_density, dimcv_sph.py:738-751):
// FP64 over the scene's targets, in slot order
template <int D>
__global__ void k_batch_kden(dv_params P, dv_fields F, const float* __restrict__ kden, dv_scene_state* st) {
  const int s = blockIdx.x;
  const int a = st[s].start, b = st[s].end;
  double acc = 0.0;
  for (int i = a + threadIdx.x; i < b; i += blockDim.x)
    if (F.material[i] == DV_MATERIAL_FLUID && in_vortex_domain<D>(P, ldv<D>(F.x, i))) acc += (double)kden[i];
  acc = block_sum<double>(acc);
  if (threadIdx.x == 0) {
    st[s].kden_sum = acc;
    st[s].kden_sum_f32 = (float)acc;
  }
}

// target, sample and far-field tile offsets; M_s = max(1, floor(frac · fluid_s))
// where the scene has targets with a positive kden_sum, else 0 (dv_sample).
// One block; each thread owns a contiguous run of scenes.
// Far-field blocks go out longest first: every block of scene s runs its
// tile of targets over the scene's num_samples samples, so the scenes are
// ranked by num_samples (descending, ties by scene index; scenes without
// targets last), tile_off is assigned in rank order and order[r] is the scene
// of rank r.  A block's sums depend only on its scene and tile, so the order
// changes which blocks form the tail of the launch, not the results.  With
// more than kOrderMax scenes the order is the scene order.
constexpr int kOrderMax = 1024;
__global__ void k_batch_offsets(dv_scene_state* st, int S, float frac, int tile_w, dv_counters* C,
                                int32_t* misc, int32_t* __restrict__ order) {
  __shared__ int s_key[kOrderMax];
  __shared__ int s_ord[kOrderMax];
  const bool ranked = S <= kOrderMax;
  const int per = (S + blockDim.x - 1) / blockDim.x;
  const int s0 = min(S, (int)threadIdx.x * per), s1 = min(S, s0 + per);
  int t = 0, m = 0;
  for (int s = s0; s < s1; ++s) {
    const int nt = st[s].n_targets;
    int M = 0;
    if (nt > 0 && st[s].kden_sum > 0.0) {
      M = (int)((double)frac * (double)st[s].n_fluid);
      if (M < 1) M = 1;
    }
    st[s].num_samples = M;
    if (ranked) s_key[s] = nt > 0 ? M : -1;
    t += nt;
    m += M;
  }
  int tt, mt, ct;
  int ot = block_excl_scan(t, &tt);  // its barriers publish s_key
  int om = block_excl_scan(m, &mt);
  for (int s = s0; s < s1; ++s) {
    st[s].t_start = ot;
    st[s].m_off = om;
    ot += st[s].n_targets;
    om += st[s].num_samples;
  }
  if (ranked) {
    for (int s = s0; s < s1; ++s) {
      const int k = s_key[s];
      int r = 0;
      for (int q = 0; q < S; ++q) {
        const int kq = s_key[q];
        r += (kq > k || (kq == k && q < s)) ? 1 : 0;
      }
      s_ord[r] = s;
    }
    __syncthreads();
  }
  int tiles = 0;
  for (int r = s0; r < s1; ++r) tiles += (st[ranked ? s_ord[r] : r].n_targets + tile_w - 1) / tile_w;
  int oc = block_excl_scan(tiles, &ct);
  for (int r = s0; r < s1; ++r) {
    const int s = ranked ? s_ord[r] : r;
    st[s].tile_off = oc;
    order[r] = s;
    oc += (st[s].n_targets + tile_w - 1) / tile_w;
  }
  if (threadIdx.x == 0) {
    C->num_samples = mt;
    misc[0] = ct;
  }
}

// ----------------------------------------------------------- DFSPH solves
__global__ void k_batch_solve_reset(dv_scene_state* st, int32_t* done, int S, int which, int32_t* ctr) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < S) {
    done[s] = 0;
    if (which == 0)
      st[s].iters_div = 0;
    else
      st[s].iters_p = 0;
  }
  if (s == 0) {
    done[S] = 0;
    *ctr = 0;
  }
}

// k_solve_finalize per scene: FP64 sum of the scene's residual block sums
// (part[wl[s] .. wl[s+1]) of the iteration's work list), average over its
// fluid count, convergence test against eta or the iteration cap
__global__ void k_batch_solve_finalize(const double* __restrict__ part, const int32_t* __restrict__ wl,
                                       dv_scene_state* st, int32_t* done, double eta, int max_iter, int which) {
  const int s = blockIdx.x;
  if (done[s]) return;
  double acc = 0.0;
  for (int k = wl[s] + threadIdx.x; k < wl[s + 1]; k += blockDim.x) acc += part[k];
  acc = block_sum<double>(acc);
  if (threadIdx.x == 0) {
    const int nf = st[s].n_fluid;
    const double avg = nf > 0 ? acc / (double)nf : 0.0;
    const int it = which == 0 ? ++st[s].iters_div : ++st[s].iters_p;
    if (which == 0)
      st[s].err_div = avg;
    else
      st[s].err_p = avg;
    if (!isfinite(avg)) st[s].status |= DV_WARN_NAN;
    if (avg <= eta || nf == 0) {
      done[s] = 1;
    } else if (it >= max_iter) {
      done[s] = 1;
      st[s].status |= which == 0 ? DV_WARN_DIV_NOT_CONVERGED : DV_WARN_P_NOT_CONVERGED;
    }
  }
}

// work list of the scenes still iterating: wl[s] = first block of scene s
// (blocks of DV_THREADS slots), wl[S] = total; done[S] = nothing left.
// One block; each thread owns a contiguous run of scenes.
__global__ void k_batch_worklist(const dv_scene_state* __restrict__ st, int32_t* done, int S,
                                 int32_t* __restrict__ wl) {
  __shared__ int part[1024];
  const int tid = threadIdx.x, nt = blockDim.x;
  const int per = (S + nt - 1) / nt;
  const int s0 = min(S, tid * per), s1 = min(S, s0 + per);
  int sum = 0;
  for (int s = s0; s < s1; ++s) {
    const int n = st[s].end - st[s].start;
    if (!done[s] && n > 0) sum += (n + DV_THREADS - 1) / DV_THREADS;
  }
  part[tid] = sum;
  __syncthreads();
  for (int o = 1; o < nt; o <<= 1) {  // inclusive Hillis-Steele scan
    const int v = tid >= o ? part[tid - o] : 0;
    __syncthreads();
    part[tid] += v;
    __syncthreads();
  }
  int off = part[tid] - sum;
  for (int s = s0; s < s1; ++s) {
    wl[s] = off;
    const int n = st[s].end - st[s].start;
    if (!done[s] && n > 0) off += (n + DV_THREADS - 1) / DV_THREADS;
  }
  if (tid == nt - 1) {
    wl[S] = part[nt - 1];
    done[S] = part[nt - 1] == 0 ? 1 : 0;
  }
}

// condition of the captured Jacobi loop: continue while a scene iterates,
// at most max_iter times (own counter, independent of the data)
__global__ void k_batch_cond(cudaGraphConditionalHandle h, const int32_t* __restrict__ wl, int S, int32_t* ctr,
                             int max_iter) {
  const int it = ++*ctr;
  cudaGraphSetConditional(h, (wl[S] > 0 && it < max_iter) ? 1u : 0u);
}

__global__ void k_batch_step_inc(int64_t* step) { *step += 1; }

int check_batch(dv_ctx* c) {
  if (!c) return DV_EINVAL;
  if (!c->batch) return dv_fail(c, DV_EINVAL, "the context has no scene batch (dv_batch_setup)");
  return DV_OK;
}

}  // namespace

int dv_batch_solve_reset(dv_ctx* c, int which) {
  dv_batch_state* b = c->batch;
  k_batch_solve_reset<<<dv_blocks(b->S), DV_THREADS, 0, c->stream>>>(b->d_state, b->d_done, b->S, which,
                                                                      b->d_ctr);
  DV_LAUNCHED(c);
  k_batch_worklist<<<1, 1024, 0, c->stream>>>(b->d_state, b->d_done, b->S, b->d_wl);
  DV_LAUNCHED(c);
  return DV_OK;
}

int dv_batch_loop_condition(dv_ctx* c, cudaGraphConditionalHandle h, int max_iter) {
  dv_batch_state* b = c->batch;
  k_batch_cond<<<1, 1, 0, c->stream>>>(h, b->d_wl, b->S, b->d_ctr, max_iter);
  DV_LAUNCHED(c);
  return DV_OK;
}

int dv_batch_solve_finalize(dv_ctx* c, int which) {
  dv_batch_state* b = c->batch;
  const int max_iter = which == 0 ? c->p.max_iter_div : c->p.max_iter_p;
  const double eta = which == 0 ? c->p.eta_div : c->p.eta_p;
  k_batch_solve_finalize<<<b->S, DV_THREADS, 0, c->stream>>>(b->d_err, b->d_wl, b->d_state, b->d_done, eta,
                                                              max_iter, which);
  DV_LAUNCHED(c);
  k_batch_worklist<<<1, 1024, 0, c->stream>>>(b->d_state, b->d_done, b->S, b->d_wl);
  DV_LAUNCHED(c);
  return DV_OK;
}

DV_API int dv_batch_setup(dv_ctx* c, const dv_batch_scene* scenes, int32_t n_scenes, const float* emit_pos,
                          int32_t n_emit, float mc_fraction, int32_t sample_mode) {
  if (!c || !scenes || n_scenes < 1) return DV_EINVAL;
  if (sample_mode != DV_SAMPLE_INVERSE_CDF && sample_mode != DV_SAMPLE_STRATIFIED)
    return dv_fail(c, DV_EINVAL, "dv_batch_setup: sample_mode must be inverse-CDF or stratified");
  if (c->p.n_scenes != n_scenes)
    return dv_fail(c, DV_EINVAL, "dv_batch_setup: %d scenes, the context was created for %d", n_scenes,
                   c->p.n_scenes);
  if (c->p.periodic) return dv_fail(c, DV_EUNSUPPORTED, "scene batches of periodic boxes are not built");
  if (c->dyn_rigid) return dv_fail(c, DV_EUNSUPPORTED, "dynamic rigid particles in a scene batch are not built");
  if (n_emit < 0 || (n_emit > 0 && !emit_pos)) return dv_fail(c, DV_EINVAL, "dv_batch_setup: emitter arrays");
  if (n_scenes > 4096) return dv_fail(c, DV_EINVAL, "dv_batch_setup: at most 4096 scenes");
  int64_t cap_sum = 0;
  for (int s = 0; s < n_scenes; ++s) {
    const dv_batch_scene& q = scenes[s];
    if (q.cap < 0 || q.emit_count < 0 || q.emit_offset < 0 || q.emit_offset + q.emit_count > n_emit ||
        q.emit_interval < 0)
      return dv_fail(c, DV_EINVAL, "dv_batch_setup: scene %d has an invalid emitter or capacity", s);
    cap_sum += q.cap;
  }
  (void)cap_sum;
  if (c->batch) return dv_fail(c, DV_EINVAL, "dv_batch_setup: already set up");
  dv_batch_state* b = new dv_batch_state();
  b->S = n_scenes;
  b->mc_fraction = mc_fraction;
  b->stratified = sample_mode == DV_SAMPLE_STRATIFIED;
  b->n_emit = n_emit;
  // far-field tiles are at least w = dv_far_min_tile_width() targets wide:
  // sum_s ceil(n_s / w) <= cap / w + S
  const int w = dv_far_min_tile_width();
  b->cap_tiles = c->cap / w + n_scenes + 2;
  b->m_cap = c->cap;
  cudaError_t e = cudaSuccess;
  auto al = [&](void** p, size_t bytes) {
    if (e == cudaSuccess) e = cudaMalloc(p, bytes < 1 ? 1 : bytes);
  };
  al((void**)&b->d_scenes, sizeof(dv_batch_scene) * n_scenes);
  al((void**)&b->d_state, sizeof(dv_scene_state) * n_scenes);
  al((void**)&b->d_done, sizeof(int32_t) * (n_scenes + 1));
  al((void**)&b->d_wl, sizeof(int32_t) * (n_scenes + 1));
  al((void**)&b->d_ctr, sizeof(int32_t));
  al((void**)&b->d_misc, sizeof(int32_t) * 4);
  al((void**)&b->d_order, sizeof(int32_t) * n_scenes);
  al((void**)&b->d_err, sizeof(double) * c->cap);
  al((void**)&b->d_step, sizeof(int64_t));
  al((void**)&b->d_emit, sizeof(float) * c->p.dim * std::max(n_emit, 1));
  al((void**)&c->d_scene_end, sizeof(float) * 3 * n_scenes);
  std::vector<float> ends(3 * n_scenes);
  for (int s = 0; s < n_scenes; ++s)
    for (int d = 0; d < 3; ++d) ends[3 * s + d] = scenes[s].domain_end[d];
  if (e == cudaSuccess) e = cudaMemcpy(b->d_scenes, scenes, sizeof(dv_batch_scene) * n_scenes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(b->d_state, 0, sizeof(dv_scene_state) * n_scenes);
  if (e == cudaSuccess) e = cudaMemset(b->d_done, 0, sizeof(int32_t) * (n_scenes + 1));
  if (e == cudaSuccess) e = cudaMemset(b->d_misc, 0, sizeof(int32_t) * 4);
  if (e == cudaSuccess) e = cudaMemset(b->d_order, 0, sizeof(int32_t) * n_scenes);
  if (e == cudaSuccess) e = cudaMemset(b->d_err, 0, sizeof(double) * c->cap);
  if (e == cudaSuccess) e = cudaMemset(b->d_step, 0, sizeof(int64_t));
  if (e == cudaSuccess && n_emit > 0)
    e = cudaMemcpy(b->d_emit, emit_pos, sizeof(float) * c->p.dim * n_emit, cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(c->d_scene_end, ends.data(), sizeof(float) * 3 * n_scenes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(b->d_wl, 0, sizeof(int32_t) * (n_scenes + 1));
  if (e == cudaSuccess) e = cudaMemset(b->d_ctr, 0, sizeof(int32_t));
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->gstream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->bstream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev0, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev1, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  c->batch = b;  // freed by dv_destroy even on failure
  if (e != cudaSuccess) return dv_cuda_check(c, e, "dv_batch_setup");
  c->n_upper = c->cap;  // static launch shapes
  return DV_OK;
}

void dv_batch_free(dv_ctx* c) {
  dv_batch_state* b = c->batch;
  if (!b) return;
  if (b->graph) cudaGraphExecDestroy(b->graph);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->gstream) cudaStreamDestroy(b->gstream);
  if (b->bstream) cudaStreamDestroy(b->bstream);
  cudaFree(b->d_scenes);
  cudaFree(b->d_state);
  cudaFree(b->d_done);
  cudaFree(b->d_wl);
  cudaFree(b->d_ctr);
  cudaFree(b->d_misc);
  cudaFree(b->d_order);
  cudaFree(b->d_err);
  cudaFree(b->d_step);
  cudaFree(b->d_emit);
  cudaFree(c->d_scene_end);
  c->d_scene_end = nullptr;
  delete b;
  c->batch = nullptr;
}

#define DV_TRY(call)         \
  do {                       \
    int rc_ = (call);        \
    if (rc_) return rc_;     \
  } while (0)

DV_API int dv_batch_step(dv_ctx* c, const dv_fields* src, const dv_fields* dst, const dv_solver_fields* s) {
  DV_TRY(check_batch(c));
  if (!src || !dst || !s) return DV_EINVAL;
  dv_batch_state* b = c->batch;
  const int S = b->S;
  // emission + activity on the current set, grid build into the other
  if (c->p.dim == 2)
    k_batch_emit<2><<<1, 1024, sizeof(int) * (S + 1), c->stream>>>(*src, b->d_scenes, S, b->d_emit, b->d_step,
                                                                   c->d_cnt, (int)c->cap, b->d_state);
  else
    k_batch_emit<3><<<1, 1024, sizeof(int) * (S + 1), c->stream>>>(*src, b->d_scenes, S, b->d_emit, b->d_step,
                                                                   c->d_cnt, (int)c->cap, b->d_state);
  DV_LAUNCHED(c);
  DV_TRY(dv_invalidate_lists(c));
  DV_TRY(dv_update_activity(c, src));
  DV_TRY(dv_grid_build(c, src, dst));
  k_batch_clear_ranges<<<dv_blocks(S), DV_THREADS, 0, c->stream>>>(b->d_state, S);
  DV_LAUNCHED(c);
  k_batch_ranges<<<dv_blocks(c->cap), DV_THREADS, 0, c->stream>>>(c->keys[c->perm_buf], c->d_cnt, c->scene_shift,
                                                                  S, b->d_state);
  DV_LAUNCHED(c);
  if (c->p.dim == 2)
    k_batch_counts<2><<<S, 1024, 0, c->stream>>>(c->p, *dst, b->d_state);
  else
    k_batch_counts<3><<<S, 1024, 0, c->stream>>>(c->p, *dst, b->d_state);
  DV_LAUNCHED(c);
  // substep (karman_vortex.py:232-242)
  // compute_densities + compute_DFSPH_factor + the divergence solve's first
  // compute_density_change, one sweep
  DV_TRY(dv_densities_factor_change(c, dst));
  DV_TRY(dv_scale_factor(c, dst, c->p.inv_dt));
  // the divergence loop's last residual sweep also gives the non-pressure
  // forces of the solved velocity; a loop of no iterations runs that sweep
  DV_TRY(dv_batch_solve(c, dst, 0, true));
  if (c->p.max_iter_div < 1) DV_TRY(dv_nonpressure(c, dst));
  DV_TRY(dv_scale_factor(c, dst, c->p.dt));
  // v*, ω, ∇v and Δω in one sweep; KVN (independent of the smoothing) before
  // the sweep that smooths Δω and sums the AKDE
  DV_TRY(dv_vorticity_dvort(c, dst, s));
  DV_TRY(dv_kvn_sample(c, dst, s, 0, 0, 0));
  DV_TRY(dv_smooth_akde(c, dst, s));
  if (c->p.dim == 2)
    k_batch_kden<2><<<S, 1024, 0, c->stream>>>(c->p, *dst, s->kden, b->d_state);
  else
    k_batch_kden<3><<<S, 1024, 0, c->stream>>>(c->p, *dst, s->kden, b->d_state);
  DV_LAUNCHED(c);
  k_batch_offsets<<<1, 1024, 0, c->stream>>>(b->d_state, S, b->mc_fraction, dv_far_tile_width(c), c->d_cnt,
                                             b->d_misc, b->d_order);
  DV_LAUNCHED(c);
  DV_TRY(dv_build_targets(c, dst));
  DV_TRY(dv_batch_draw(c, s));
  DV_TRY(dv_batch_vvpe(c, dst, s));
  DV_TRY(dv_life_time(c, dst));
  DV_TRY(dv_predict_velocity(c, dst));
  DV_TRY(dv_density_adv(c, dst));
  DV_TRY(dv_scale_factor(c, dst, c->p.inv_dt2));
  DV_TRY(dv_batch_solve(c, dst, 1));
  DV_TRY(dv_advect(c, dst));
  k_batch_step_inc<<<1, 1, 0, c->stream>>>(b->d_step);
  DV_LAUNCHED(c);
  return DV_OK;
}

DV_API int dv_batch_graph_capture(dv_ctx* c, const dv_fields* a, const dv_fields* bf, const dv_solver_fields* s,
                                  int32_t steps) {
  DV_TRY(check_batch(c));
  if (!a || !bf || !s || steps < 2 || steps % 2) return dv_fail(c, DV_EINVAL, "dv_batch_graph_capture: need an even step count >= 2");
  dv_batch_state* b = c->batch;
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  // capture on the context's own non-blocking stream (a legacy default stream cannot be captured)
  cudaStream_t saved = c->stream;
  DV_CK(c, cudaEventRecord(b->ev0, saved));
  DV_CK(c, cudaStreamWaitEvent(b->gstream, b->ev0, 0));
  c->stream = b->gstream;
  b->capturing = true;
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamBeginCapture(b->gstream, cudaStreamCaptureModeThreadLocal);
  int rc = DV_OK;
  if (e == cudaSuccess) {
    for (int k = 0; k < steps && rc == DV_OK; ++k) rc = dv_batch_step(c, k % 2 ? bf : a, k % 2 ? a : bf, s);
    e = cudaStreamEndCapture(b->gstream, &g);
  }
  b->capturing = false;
  c->stream = saved;
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return dv_cuda_check(c, e, "dv_batch_graph_capture");
  e = cudaGraphInstantiate(&b->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return dv_cuda_check(c, e, "cudaGraphInstantiate");
  return DV_OK;
}

DV_API int dv_batch_graph_launch(dv_ctx* c) {
  DV_TRY(check_batch(c));
  dv_batch_state* b = c->batch;
  if (!b->graph) return dv_fail(c, DV_EINVAL, "dv_batch_graph_launch: no captured graph");
  DV_CK(c, cudaEventRecord(b->ev0, c->stream));
  DV_CK(c, cudaStreamWaitEvent(b->gstream, b->ev0, 0));
  DV_CK(c, cudaGraphLaunch(b->graph, b->gstream));
  DV_CK(c, cudaEventRecord(b->ev1, b->gstream));
  DV_CK(c, cudaStreamWaitEvent(c->stream, b->ev1, 0));
  c->launches++;
  return DV_OK;
}

DV_API int dv_batch_read(dv_ctx* c, dv_scene_state* out, int32_t n_scenes, int64_t* step) {
  DV_TRY(check_batch(c));
  dv_batch_state* b = c->batch;
  if (out && n_scenes > 0) {
    DV_CK(c, cudaMemcpyAsync(out, b->d_state, sizeof(dv_scene_state) * std::min(n_scenes, b->S),
                             cudaMemcpyDeviceToHost, c->stream));
  }
  int64_t st = 0;
  DV_CK(c, cudaMemcpyAsync(&st, b->d_step, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
  DV_CK(c, cudaStreamSynchronize(c->stream));
  if (step) *step = st;
  return DV_OK;
}
