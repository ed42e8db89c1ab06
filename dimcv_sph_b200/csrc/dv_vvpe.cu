// N-body parts of the VVPE (reference: DIMCVSPHSolver.vort2vel,
// dimcv_sph.py:679-719) and the full Biot-Savart comparator.  These are
// FP32-pipe bound: each CTA stages tiles of sources (position, weighted
// vorticity) in shared memory and every thread accumulates TT targets in
// registers, so one broadcast shared load feeds TT pair evaluations.
//
// Far-field pair (reference kernel): the sample counts iff
// sqrtf(|r|²) > h, tested exactly as r2 > far_r2_limit with r2 summed in the
// reference order without FMA; Kε(|r|) = 1/(|r|·|r|) there because
// exp(-|r|/ε) underflows to 0 for |r| > h >= 1.05e-4 (checked on the host,
// otherwise the exact regularised form is used).  The sample's 1/(kden+1e-8)
// and the target's (kden_sum - S_i) are folded out of the pair loop.
// This file is compiled with FMA contraction on.
#include <algorithm>

#include "dv_internal.cuh"

int dv_build_targets(dv_ctx* c, const dv_fields* f);
int dv_launch_vvpe_near(dv_ctx* c, const dv_fields* f, const dv_solver_fields* s);

#define FT 256  // threads per CTA
#define FTILE 256

// ------------------------------------------------------------ sample pack
// spos = (x, y, z|0, 0), sw = ω̃ / (kden + 1e-8)  (dimcv_sph.py:706-709)
template <int D>
__global__ void k_pack_samples(const dv_fields F, const dv_solver_fields S,
                               const dv_counters* __restrict__ C, float4* __restrict__ spos,
                               float4* __restrict__ sw, float kden_eps) {
  const int M = C->num_samples;
  const int n = C->n;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < M; s += gridDim.x * blockDim.x) {
    int j = S.sample_idx[s];
    if (j < 0 || j >= n) {  // a caller-injected index outside [0, n): no contribution
      atomicOr(const_cast<int32_t*>(&C->status), DV_WARN_BAD_INDEX);
      spos[s] = make_float4(0.f, 0.f, 0.f, 0.f);
      sw[s] = make_float4(0.f, 0.f, 0.f, 0.f);
      continue;
    }
    V3 x = ldv<D>(F.x, j);
    V3 w = ld4(S.d_vort_smoothed, j);
    float inv = 1.0f / (S.kden[j] + kden_eps);
    spos[s] = make_float4(x.x, x.y, x.z, 0.0f);
    sw[s] = make_float4(w.x * inv, w.y * inv, w.z * inv, 0.0f);
  }
}

template <bool COMP>
struct Acc {
  float s = 0.0f, c = 0.0f;
  __device__ __forceinline__ void add(float t) {
    if (COMP) {  // Kahan: y = t - c; u = s + y; c = (u - s) - y; s = u
      float y = __fsub_rn(t, c);
      float u = __fadd_rn(s, y);
      c = __fsub_rn(__fsub_rn(u, s), y);
      s = u;
    } else {
      s += t;
    }
  }
  __device__ __forceinline__ float val() const { return COMP ? __fsub_rn(s, c) : s; }
};

// Regularised reference kernel Kε(r) for r2 below the underflow bound.
__device__ __forceinline__ float k_eps_exact(const dv_params& P, float r2) {
  float rn = sqrtf(r2);
  float e = expf(-rn * P.inv_eps);
  return (1.0f - e) / (rn * (rn + P.eps * e));
}

template <int D, int TT, bool BLOB, bool COMP, bool FASTK>
__global__ void __launch_bounds__(FT) k_vvpe_far(dv_params P, dv_fields F, dv_solver_fields S,
                                                 const dv_counters* __restrict__ C,
                                                 const int32_t* __restrict__ targets,
                                                 const float4* __restrict__ spos,
                                                 const float4* __restrict__ sw,
                                                 const float4* __restrict__ near_v,
                                                 const float* __restrict__ near_S) {
  __shared__ float4 s_p[FTILE];
  __shared__ float4 s_w[FTILE];
  const int nt = C->n_targets;
  const int M = C->num_samples;
  const int tbase = blockIdx.x * FT * TT;
  if (tbase >= nt) return;  // uniform per CTA
  float px[TT], py[TT], pz[TT];
  Acc<COMP> ax[TT], ay[TT], az[TT];
  int cnt[TT];
#pragma unroll
  for (int k = 0; k < TT; ++k) {
    int t = tbase + k * FT + threadIdx.x;
    int i = targets[t < nt ? t : nt - 1];
    V3 x = ldv<D>(F.x, i);
    px[k] = x.x;
    py[k] = x.y;
    pz[k] = x.z;
    cnt[k] = 0;
  }
  const float lim = P.far_r2_limit;
  const float d2 = P.blob_delta2;
  for (int base = 0; base < M; base += FTILE) {
    const int m = min(FTILE, M - base);
    __syncthreads();
    for (int q = threadIdx.x; q < m; q += FT) {
      s_p[q] = spos[base + q];
      s_w[q] = sw[base + q];
    }
    __syncthreads();
#pragma unroll 2
    for (int q = 0; q < m; ++q) {
      const float4 sp = s_p[q];
      const float4 w = s_w[q];
#pragma unroll
      for (int k = 0; k < TT; ++k) {
        float dx = __fsub_rn(px[k], sp.x);
        float dy = __fsub_rn(py[k], sp.y);
        float dz = D == 3 ? __fsub_rn(pz[k], sp.z) : 0.0f;
        float r2 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
        if (D == 3) r2 = __fadd_rn(r2, __fmul_rn(dz, dz));
        const bool far = r2 > lim;
        cnt[k] += far ? 1 : 0;
        if (!BLOB) {
          float kk;
          if (FASTK)
            kk = far ? __fdividef(1.0f, r2) : 0.0f;
          else
            kk = far ? k_eps_exact(P, r2) : 0.0f;
          // K (r_xy × w) with r_xy = (dx, dy, 0)
          float t = kk * w.z;
          ax[k].add(t * dy);
          ay[k].add(-t * dx);
          az[k].add(kk * (dx * w.y - dy * w.x));
        } else {
          float s = r2 + d2;
          float inv = rsqrtf(s);
          float kk = far ? inv * inv * inv : 0.0f;
          ax[k].add(kk * (dy * w.z - dz * w.y));
          ay[k].add(kk * (dz * w.x - dx * w.z));
          az[k].add(kk * (dx * w.y - dy * w.x));
        }
      }
    }
  }
  const float coef = BLOB ? P.blob_coef : P.vvpe_coef;
  const float kden_sum = C->kden_sum_f32;
#pragma unroll
  for (int k = 0; k < TT; ++k) {
    int t = tbase + k * FT + threadIdx.x;
    if (t >= nt) continue;
    int i = targets[t];
    float4 nv = near_v[t];
    float fac = kden_sum - near_S[t];
    V3 fv{0.f, 0.f, 0.f};
    if (cnt[k] > 0) {
      float sc = coef / (float)cnt[k];
      fv.x = (ax[k].val() * fac) * sc;
      fv.y = (ay[k].val() * fac) * sc;
      fv.z = (az[k].val() * fac) * sc;
    }
    V3 vv{fv.x + nv.x, fv.y + nv.y, fv.z + nv.z};
    if (S.v_vort) st4(S.v_vort, i, vv);
    // gate ‖v_vort‖ < ‖v_i‖ (dimcv_sph.py:717-719)
    float n1 = sqrtf(__fadd_rn(__fadd_rn(__fmul_rn(vv.x, vv.x), __fmul_rn(vv.y, vv.y)),
                               __fmul_rn(vv.z, vv.z)));
    V3 vi = ldv<D>(F.v, i);
    float n2 = sqrtf(sqnorm<D>(vi));
    if (n1 < n2) {
      vi.x = __fadd_rn(vi.x, vv.x);
      vi.y = __fadd_rn(vi.y, vv.y);
      if (D == 3) vi.z = __fadd_rn(vi.z, vv.z);
      stv<D>(F.v, i, vi);
    }
  }
}

template <int D, int TT, bool BLOB, bool COMP, bool FASTK>
static void launch_far(dv_ctx* c, const dv_fields* f, const dv_solver_fields* s, int nb) {
  k_vvpe_far<D, TT, BLOB, COMP, FASTK><<<nb, FT, 0, c->stream>>>(
      c->p, *f, *s, c->d_cnt, c->targets, c->spos, c->sw, c->near_v, c->near_S);
}

template <int D>
static void dispatch_far(dv_ctx* c, const dv_fields* f, const dv_solver_fields* s, int nb, bool fastk) {
  constexpr int TT = 2;
  const bool blob = c->p.kernel_mode == DV_KERNEL_BLOB3D;
  const bool comp = c->p.compensated != 0;
  if (blob) {
    if (comp)
      launch_far<D, TT, true, true, true>(c, f, s, nb);
    else
      launch_far<D, TT, true, false, true>(c, f, s, nb);
  } else if (fastk) {
    if (comp)
      launch_far<D, TT, false, true, true>(c, f, s, nb);
    else
      launch_far<D, TT, false, false, true>(c, f, s, nb);
  } else {
    if (comp)
      launch_far<D, TT, false, true, false>(c, f, s, nb);
    else
      launch_far<D, TT, false, false, false>(c, f, s, nb);
  }
}

// exp(-h/ε) underflows to zero in f32 once h/ε > 103.97
static bool fast_kernel_ok(const dv_params& P) {
  return (double)P.support_radius * (double)P.inv_eps > 104.5;
}

// ------------------------------------------------- far field, split form
// The main loop evaluates every (target, sample) pair WITHOUT the far test:
// for the reference kernel the weight is 1/max(|r|², T) with T =
// far_r2_limit, so a near sample (|r| <= h, including the target itself)
// adds a bounded term (|r_xy|/T·|ω̂| <= |ω̂|/h, the size of the largest far
// terms).  A second kernel then finds, per target, the few samples with
// |r| <= h — exactly, with the reference's non-FMA |r|² test — among the
// particles of the target's cell window, subtracts their terms (recomputed
// bit for bit as the main loop computed them) and removes them from the far
// count.  Per pair this leaves ~14 issue slots instead of ~28.

__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// 1/sqrt(x) in one MUFU operation.  The blob kernel's argument |r|² + δ² is
// at least δ² > 0 and never subnormal, so flushing subnormals changes no
// result; without .ftz the approximate rsqrt also carries the code that
// rescales subnormal inputs, which every pair would pay for.
__device__ __forceinline__ float rsqrt_approx(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// The blob kernel's (|r|² + δ²)^(-3/2): s = δ² + dx² + dy² + dz² by three
// fma (δ² enters first, saving an add), then 1/s · 1/sqrt(s) from two MUFU
// operations and one multiply instead of the cube of 1/sqrt(s) (two
// multiplies): 16 FP32-pipe operations per pair instead of 18 in a loop the
// FP32 pipe bounds, one more on the otherwise idle MUFU.  The scalar loop,
// the paired loop and the near-sample correction all use this one form.
__device__ __forceinline__ float blob_k(float dx, float dy, float dz, float d2) {
  float s = __fmaf_rn(dx, dx, d2);
  s = __fmaf_rn(dy, dy, s);
  s = __fmaf_rn(dz, dz, s);
  return __fmul_rn(rcp_approx(s), rsqrt_approx(s));
}

// coordinate difference, minimum image on a periodic box
template <bool PER>
__device__ __forceinline__ float wrapd(float d, float L) {
  return PER ? min_image(d, L) : d;
}

// one pair of the main loop: returns the three increments (r × ω̂ weighted)
template <int D, bool BLOB, bool PER = false>
__device__ __forceinline__ void far_terms(float px, float py, float pz, float4 sp, float4 w, float lim,
                                          float d2, float& cx, float& cy, float& cz,
                                          float3 bx = float3{0.f, 0.f, 0.f}) {
  const float dx = wrapd<PER>(__fsub_rn(px, sp.x), bx.x);
  const float dy = wrapd<PER>(__fsub_rn(py, sp.y), bx.y);
  const float dz = D == 3 ? wrapd<PER>(__fsub_rn(pz, sp.z), bx.z) : 0.0f;
  if (!BLOB) {
    float r2 = __fmul_rn(dx, dx);
    r2 = __fmaf_rn(dy, dy, r2);
    if (D == 3) r2 = __fmaf_rn(dz, dz, r2);
    // Kε = 1/|r|² (exp term underflows for |r| > h); cross with r_xy = (dx, dy, 0)
    const float kk = rcp_approx(fmaxf(r2, lim));
    const float a = __fmul_rn(kk, dx), b = __fmul_rn(kk, dy);
    cx = __fmul_rn(b, w.z);
    cy = -__fmul_rn(a, w.z);
    cz = __fmaf_rn(a, w.y, -__fmul_rn(b, w.x));
  } else {
    const float kk = blob_k(dx, dy, dz, d2);
    const float a = __fmul_rn(kk, dx), b = __fmul_rn(kk, dy), e = __fmul_rn(kk, dz);
    cx = __fmaf_rn(b, w.z, -__fmul_rn(e, w.y));
    cy = __fmaf_rn(e, w.x, -__fmul_rn(a, w.z));
    cz = __fmaf_rn(a, w.y, -__fmul_rn(b, w.x));
  }
}

// main loop accumulation form of far_terms (lets the increments fuse into FMAs)
template <int D, bool BLOB, bool COMP, bool PER = false>
__device__ __forceinline__ void far_accum(float px, float py, float pz, float4 sp, float4 w, float lim, float d2,
                                          Acc<COMP>& ax, Acc<COMP>& ay, Acc<COMP>& az,
                                          float3 bx = float3{0.f, 0.f, 0.f}) {
  const float dx = wrapd<PER>(__fsub_rn(px, sp.x), bx.x);
  const float dy = wrapd<PER>(__fsub_rn(py, sp.y), bx.y);
  const float dz = D == 3 ? wrapd<PER>(__fsub_rn(pz, sp.z), bx.z) : 0.0f;
  if (COMP) {
    float cx, cy, cz;
    far_terms<D, BLOB, PER>(px, py, pz, sp, w, lim, d2, cx, cy, cz, bx);
    ax.add(cx);
    ay.add(cy);
    az.add(cz);
  } else if (!BLOB) {
    float r2 = __fmul_rn(dx, dx);
    r2 = __fmaf_rn(dy, dy, r2);
    if (D == 3) r2 = __fmaf_rn(dz, dz, r2);
    const float kk = rcp_approx(fmaxf(r2, lim));
    const float a = __fmul_rn(kk, dx), b = __fmul_rn(kk, dy);
    ax.s = __fmaf_rn(b, w.z, ax.s);
    ay.s = __fmaf_rn(-a, w.z, ay.s);
    if (D == 3) {  // in 2-D ω̃ = (0, 0, ω_z) by construction: the z row is exactly 0
      az.s = __fmaf_rn(a, w.y, az.s);
      az.s = __fmaf_rn(-b, w.x, az.s);
    }
  } else {
    const float kk = blob_k(dx, dy, dz, d2);
    const float a = __fmul_rn(kk, dx), b = __fmul_rn(kk, dy), e = __fmul_rn(kk, dz);
    ax.s = __fmaf_rn(b, w.z, ax.s);
    ax.s = __fmaf_rn(-e, w.y, ax.s);
    ay.s = __fmaf_rn(e, w.x, ay.s);
    ay.s = __fmaf_rn(-a, w.z, ay.s);
    az.s = __fmaf_rn(a, w.y, az.s);
    az.s = __fmaf_rn(-b, w.x, az.s);
  }
}

#ifndef FT2
#define FT2 256  // threads per CTA of the far-field main loops
#endif
#ifndef FTILE2
#define FTILE2 512  // samples staged in shared memory per tile
#endif
// resident CTAs per SM asked of the register allocator for the paired loop
// (for 256-thread CTAs; scaled for other sizes): 3 for 2 and 4 targets per thread (80 registers, 24 warps per SM, which hides
// more of the rcp -> mul -> fma latency than 16: sphere3d far field 57.5 ->
// 54.6 ms per step), 2 for 6 and 8 (their wider register tiles spill at 80)
#define DV_FAR_MINB(TT) (((TT) <= 4 ? 3 : 2) * (256 / FT2))
#ifndef DV_FAR_QUNROLL
#define DV_FAR_QUNROLL 2  // samples per unrolled step of the paired loop
#endif
constexpr int kFarQUnroll = DV_FAR_QUNROLL;

// sample chunk blockIdx.y of nchunk: [m0, m0 + M) of the M_total samples;
// the chunk's partial sums go to far_acc[chunk * stride + t]
__device__ __forceinline__ void sample_chunk(int M_total, int nchunk, int& m0, int& M) {
  const int clen = (M_total + nchunk - 1) / nchunk;
  m0 = (int)blockIdx.y * clen;
  M = max(0, min(clen, M_total - m0));
}

template <int D, int TT, bool BLOB, bool COMP, bool PER>
__global__ void __launch_bounds__(FT2) k_far_main(dv_params P, const float* __restrict__ x,
                                                  const dv_counters* __restrict__ C,
                                                  const int32_t* __restrict__ targets,
                                                  const float4* __restrict__ spos,
                                                  const float4* __restrict__ sw,
                                                  float4* __restrict__ far_acc, int nchunk, int64_t stride) {
  __shared__ float4 s_p[FTILE2];
  __shared__ float4 s_w[FTILE2];
  const int nt = C->n_targets;
  int m0, M;
  sample_chunk(C->num_samples, nchunk, m0, M);
  spos += m0;
  sw += m0;
  far_acc += blockIdx.y * stride;
  const int tbase = blockIdx.x * FT2 * TT;
  if (tbase >= nt) return;  // uniform per CTA
  float px[TT], py[TT], pz[TT];
  Acc<COMP> ax[TT], ay[TT], az[TT];
#pragma unroll
  for (int k = 0; k < TT; ++k) {
    int t = tbase + k * FT2 + threadIdx.x;
    V3 xi = ldv<D>(x, targets[t < nt ? t : nt - 1]);
    px[k] = xi.x;
    py[k] = xi.y;
    pz[k] = xi.z;
  }
  const float lim = P.far_r2_limit;
  const float d2 = P.blob_delta2;
  const float3 bx = make_float3(P.box[0], P.box[1], P.box[2]);
  for (int base = 0; base < M; base += FTILE2) {
    const int m = min(FTILE2, M - base);
    __syncthreads();
    for (int q = threadIdx.x; q < m; q += FT2) {
      s_p[q] = spos[base + q];
      s_w[q] = sw[base + q];
    }
    __syncthreads();
#pragma unroll 4
    for (int q = 0; q < m; ++q) {
      const float4 sp = s_p[q];
      const float4 w = s_w[q];
#pragma unroll
      for (int k = 0; k < TT; ++k)
        far_accum<D, BLOB, COMP, PER>(px[k], py[k], pz[k], sp, w, lim, d2, ax[k], ay[k], az[k], bx);
    }
  }
#pragma unroll
  for (int k = 0; k < TT; ++k) {
    int t = tbase + k * FT2 + threadIdx.x;
    if (t < nt) far_acc[t] = make_float4(ax[k].val(), ay[k].val(), az[k].val(), 0.0f);
  }
}

// sample multiplicities per slot (a slot may be drawn several times)
__global__ void k_mult(const int32_t* __restrict__ sample_idx, const dv_counters* __restrict__ C,
                       int32_t* __restrict__ mult) {
  const int M = C->num_samples, n = C->n;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < M; s += gridDim.x * blockDim.x) {
    int j = sample_idx[s];
    if (j >= 0 && j < n) atomicAdd(mult + j, 1);
  }
}

// The sampled slots in slot order (sslot) and, per slot, the number of
// sampled slots before it (srank): the samples among the particles
// [s, e) of a cell are sslot[srank[s] .. srank[e]), in slot order, so the
// correction kernel reads a cell's few samples instead of testing every
// particle's multiplicity.
__global__ void k_sample_flags(const int32_t* __restrict__ mult, int nu, uint32_t* __restrict__ flag) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j <= nu; j += gridDim.x * blockDim.x)
    flag[j] = (j < nu && mult[j] > 0) ? 1u : 0u;
}

__global__ void k_sample_slots(const int32_t* __restrict__ mult, int nu, const uint32_t* __restrict__ rank,
                               int32_t* __restrict__ slot) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nu; j += gridDim.x * blockDim.x)
    if (mult[j] > 0) slot[rank[j]] = j;
}

static int sample_slots(dv_ctx* c) {
  const int nu = (int)std::min<int64_t>(c->n_upper, c->cap);
  k_sample_flags<<<c->num_sms * 4, DV_THREADS, 0, c->stream>>>(c->mult, nu, c->sflag);
  DV_LAUNCHED(c);
  int rc = dv_scan_u32(c, c->sflag, c->srank, (int64_t)nu + 1);
  if (rc) return rc;
  k_sample_slots<<<c->num_sms * 4, DV_THREADS, 0, c->stream>>>(c->mult, nu, c->srank, c->sslot);
  DV_LAUNCHED(c);
  return DV_OK;
}

// cell window of a target that contains every particle within h: the 3^d
// cells around its cell, widened by one cell on a side where the target's
// cell coordinate is within rounding of a cell face (a particle exactly h
// away can then sit two cells over).  On a periodic axis the window wraps
// (lo/hi are then offsets to be wrapped by cell_step, see k_far_fix).
__device__ __forceinline__ void far_window(const dv_params& P, float xv, int d, int& lo, int& hi) {
  float t = P.cell_origin_offset ? (xv - P.domain_start[d]) : xv;
  float q = t / P.grid_size;
  int c = cell_coord(P, xv, d);
  float tol = 4.8e-7f * fmaxf(1.0f, fabsf(q));
  float frac = q - (float)c;
  lo = c - 1 - (frac <= tol ? 1 : 0);
  hi = c + 1 + (frac >= 1.0f - tol ? 1 : 0);
  if (!P.periodic) {
    lo = max(lo, 0);
    hi = min(hi, P.grid_num[d] - 1);
  }
}

__device__ __forceinline__ int wrap_cell(const dv_params& P, int g, int d) {
  if (!P.periodic) return g;
  const int n = P.grid_num[d];
  return g < 0 ? g + n : (g >= n ? g - n : g);
}

// Near-sample correction and finalize of target t (slot i): removes from the
// main loop's sum the samples within h (cell window, classification
// r2 <= far_r2_limit), counts the rest, scales by (S - S_i)/count and
// applies the gate.  M, kden_sum: the scene's sample count and kden_sum;
// sk: the scene prefix of the cell keys (0 for a single scene).
template <int D, bool BLOB, bool PER>
__device__ __forceinline__ void far_fix_one(const dv_params& P, const DevGrid& G, const dv_fields& F,
                                            const dv_solver_fields& S, int t, int i, int M, float kden_sum,
                                            uint32_t sk, const int32_t* __restrict__ mult,
                                            const uint32_t* __restrict__ srank, const int32_t* __restrict__ sslot,
                                            const float4* __restrict__ far_acc, const float4* __restrict__ near_v,
                                            const float* __restrict__ near_S, int nchunk, int64_t stride) {
  const V3 xi = ldv<D>(F.x, i);
  const float lim = P.far_r2_limit, d2 = P.blob_delta2;
  const float3 bx = make_float3(P.box[0], P.box[1], P.box[2]);
  float4 acc = far_acc[t];
  for (int k = 1; k < nchunk; ++k) {  // sample-chunk partials, in chunk order
    const float4 q = far_acc[k * stride + t];
    acc.x = __fadd_rn(acc.x, q.x);
    acc.y = __fadd_rn(acc.y, q.y);
    acc.z = __fadd_rn(acc.z, q.z);
  }
  int near_cnt = 0;
  int lo0, hi0, lo1, hi1, lo2 = 0, hi2 = 0;
  far_window(P, xi.x, 0, lo0, hi0);
  far_window(P, xi.y, 1, lo1, hi1);
  if (D == 3) far_window(P, xi.z, 2, lo2, hi2);
  for (int a = lo0; a <= hi0; ++a) {
    const uint32_t ka = __ldg(G.mt0 + wrap_cell(P, a, 0));
    for (int b = lo1; b <= hi1; ++b) {
      const uint32_t kab = ka | __ldg(G.mt1 + wrap_cell(P, b, 1));
      for (int cc = lo2; cc <= hi2; ++cc) {
        const uint32_t key = (D == 3 ? (kab | __ldg(G.mt2 + wrap_cell(P, cc, 2))) : kab) | sk;
        const int s0 = __ldg(G.start + key), e0 = __ldg(G.end + key);
        if (s0 >= e0) continue;
        const uint32_t p1 = __ldg(srank + e0);
        for (uint32_t p = __ldg(srank + s0); p < p1; ++p) {  // the cell's samples, in slot order
          const int j = __ldg(sslot + p);
          const int m = mult[j];
          const V3 xj = ldv<D>(F.x, j);
          if (sqnorm<D>(rel<D>(P, xi, xj)) > lim) continue;  // far: the main loop's term stays
          near_cnt += m;
          const V3 w3 = ld4(S.d_vort_smoothed, j);
          const float inv = 1.0f / (S.kden[j] + P.kden_eps);
          const float4 w = make_float4(w3.x * inv, w3.y * inv, w3.z * inv, 0.0f);
          float cx, cy, cz;
          far_terms<D, BLOB, PER>(xi.x, xi.y, xi.z, make_float4(xj.x, xj.y, xj.z, 0.0f), w, lim, d2, cx, cy,
                                  cz, bx);
          const float fm = (float)m;
          acc.x = __fmaf_rn(-fm, cx, acc.x);
          acc.y = __fmaf_rn(-fm, cy, acc.y);
          acc.z = __fmaf_rn(-fm, cz, acc.z);
        }
      }
    }
  }
  const int cnt = M - near_cnt;
  const float coef = BLOB ? P.blob_coef : P.vvpe_coef;
  const float fac = kden_sum - near_S[t];
  V3 fv{0.f, 0.f, 0.f};
  if (cnt > 0) {
    const float sc = coef / (float)cnt;
    fv.x = (acc.x * fac) * sc;
    fv.y = (acc.y * fac) * sc;
    fv.z = (acc.z * fac) * sc;
  }
  const float4 nv = near_v[t];
  V3 vv{__fadd_rn(fv.x, nv.x), __fadd_rn(fv.y, nv.y), __fadd_rn(fv.z, nv.z)};
  if (S.v_vort) st4(S.v_vort, i, vv);
  // gate ‖v_vort‖ < ‖v_i‖ (dimcv_sph.py:717-719)
  const float n1 = sqrtf(__fadd_rn(__fadd_rn(__fmul_rn(vv.x, vv.x), __fmul_rn(vv.y, vv.y)), __fmul_rn(vv.z, vv.z)));
  V3 v = ldv<D>(F.v, i);
  const float n2 = sqrtf(sqnorm<D>(v));
  if (n1 < n2) {
    v.x = __fadd_rn(v.x, vv.x);
    v.y = __fadd_rn(v.y, vv.y);
    if (D == 3) v.z = __fadd_rn(v.z, vv.z);
    stv<D>(F.v, i, v);
  }
}

template <int D, bool BLOB, bool PER>
__global__ void k_far_fix(dv_params P, DevGrid G, dv_fields F, dv_solver_fields S,
                          const dv_counters* __restrict__ C, const int32_t* __restrict__ targets,
                          const int32_t* __restrict__ mult, const uint32_t* __restrict__ srank,
                          const int32_t* __restrict__ sslot, const float4* __restrict__ far_acc,
                          const float4* __restrict__ near_v, const float* __restrict__ near_S, int nchunk,
                          int64_t stride) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= C->n_targets) return;
  far_fix_one<D, BLOB, PER>(P, G, F, S, t, targets[t], C->num_samples, C->kden_sum_f32, 0u, mult, srank, sslot,
                            far_acc, near_v, near_S, nchunk, stride);
}

// scene batch: the target's scene gives M, kden_sum and the key prefix
template <int D, bool BLOB>
__global__ void k_far_fix_b(dv_params P, DevGrid G, dv_fields F, dv_solver_fields S,
                            const dv_counters* __restrict__ C, const int32_t* __restrict__ targets,
                            const int32_t* __restrict__ mult, const uint32_t* __restrict__ srank,
                            const int32_t* __restrict__ sslot, const float4* __restrict__ far_acc,
                            const float4* __restrict__ near_v, const float* __restrict__ near_S,
                            const dv_scene_state* __restrict__ st) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= C->n_targets) return;
  const int i = targets[t];
  const int sc = F.object_id[i];
  far_fix_one<D, BLOB, false>(P, G, F, S, t, i, st[sc].num_samples, st[sc].kden_sum_f32,
                              (uint32_t)sc << G.scene_shift, mult, srank, sslot, far_acc, near_v, near_S, 1, 0);
}

// scene of far-field block blk: the last scene in block order whose first
// block is at or before blk (tile_off increases along order[], one or more
// blocks per scene with targets)
__device__ __forceinline__ int batch_block_scene(const dv_scene_state* __restrict__ st,
                                                 const int32_t* __restrict__ order, int S, int blk) {
  int lo = 0, hi = S;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (st[order[mid]].tile_off <= blk)
      lo = mid + 1;
    else
      hi = mid;
  }
  return order[lo - 1];
}

// scene batch main loop: block b is tile b - tile_off_s of its scene s
// (batch_block_scene); its targets [t_start_s + tile·FT2·TT, ...) of the
// scene run over the scene's samples [m_off_s, m_off_s + M_s) in the order
// and tiling of k_far_main
template <int D, int TT, bool BLOB, bool COMP>
__global__ void __launch_bounds__(FT2) k_far_main_b(dv_params P, const float* __restrict__ x,
                                                    const int32_t* __restrict__ targets,
                                                    const float4* __restrict__ spos,
                                                    const float4* __restrict__ sw,
                                                    const dv_scene_state* __restrict__ st,
                                                    const int32_t* __restrict__ order, int S,
                                                    const int32_t* __restrict__ ntiles,
                                                    float4* __restrict__ far_acc) {
  __shared__ float4 s_p[FTILE2];
  __shared__ float4 s_w[FTILE2];
  const int blk = blockIdx.x;
  if (blk >= *ntiles) return;  // uniform per CTA
  const int sc = batch_block_scene(st, order, S, blk);
  const int t0 = st[sc].t_start, nt = st[sc].n_targets;
  const int m0 = st[sc].m_off, M = st[sc].num_samples;
  const int tbase = (blk - st[sc].tile_off) * FT2 * TT;
  float px[TT], py[TT], pz[TT];
  Acc<COMP> ax[TT], ay[TT], az[TT];
#pragma unroll
  for (int k = 0; k < TT; ++k) {
    const int t = tbase + k * FT2 + threadIdx.x;
    V3 xi = ldv<D>(x, targets[t0 + (t < nt ? t : nt - 1)]);
    px[k] = xi.x;
    py[k] = xi.y;
    pz[k] = xi.z;
  }
  const float lim = P.far_r2_limit;
  const float d2 = P.blob_delta2;
  for (int base = 0; base < M; base += FTILE2) {
    const int m = min(FTILE2, M - base);
    __syncthreads();
    for (int q = threadIdx.x; q < m; q += FT2) {
      s_p[q] = spos[m0 + base + q];
      s_w[q] = sw[m0 + base + q];
    }
    __syncthreads();
#pragma unroll 4
    for (int q = 0; q < m; ++q) {
      const float4 sp = s_p[q];
      const float4 w = s_w[q];
#pragma unroll
      for (int k = 0; k < TT; ++k) far_accum<D, BLOB, COMP, false>(px[k], py[k], pz[k], sp, w, lim, d2, ax[k], ay[k], az[k]);
    }
  }
#pragma unroll
  for (int k = 0; k < TT; ++k) {
    const int t = tbase + k * FT2 + threadIdx.x;
    if (t < nt) far_acc[t0 + t] = make_float4(ax[k].val(), ay[k].val(), az[k].val(), 0.0f);
  }
}

// ------------------------------------------------ paired-FP32 main loop
// The reference-kernel main loop with two targets per instruction
// (Blackwell's sub/mul/fma.rn.f32x2): every lane operation is the scalar
// loop's own IEEE operation in the same order, so far_acc is bit-identical;
// the pairs halve the issue slots of a loop that is issue-bound, not
// FP32-pipe-bound.  Samples are staged in shared memory pre-duplicated
// ({s, s} pairs, ω̃/kden components negated where the loop subtracts).
typedef unsigned long long f2_t;
__device__ __forceinline__ f2_t f2_pack(float a, float b) {
  f2_t r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ void f2_unpack(f2_t v, float& a, float& b) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ f2_t f2_sub(f2_t a, f2_t b) {
  f2_t d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f2_t f2_mul(f2_t a, f2_t b) {
  f2_t d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f2_t f2_fma(f2_t a, f2_t b, f2_t c) {
  f2_t d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

// float4 words per staged sample of the paired loops: the reference kernel
// needs {x, y, (z,) ω̂z, -ω̂z, (ω̂y, -ω̂x)}, the blob kernel {x, y, z, ω̂, -ω̂}
template <int D, bool BLOB>
constexpr int far_x2_words() {
  return BLOB ? 5 : (D == 3 ? 4 : 2);
}

// targets [tbase + k·FT2 + tid] (k < TT) of targets[0, nt) against samples
// [m0, m0 + M); writes far_acc[t] for t < nt.  Block-uniform bounds.
// BLOB (3-D only): the regularised blob kernel, lane for lane the scalar
// loop's far_accum<3, true, false>: blob_k's three fma and its two MUFU
// operations per lane (scalar) and one multiply, then six fma into the
// accumulators; fma(-e, ω̂y, acc) is taken as fma(e, -ω̂y, acc), the same
// IEEE result.  targets may be null (target t is slot t); n_valid >= 0 zeroes
// the output of target slots outside [0, n_valid) (the full Biot-Savart's
// caller-given targets).
template <int D, int TT, bool BLOB = false>
__device__ __forceinline__ void far_x2_run(const dv_params& P, const float* __restrict__ x,
                                           const int32_t* __restrict__ targets, int nt, int tbase,
                                           const float4* __restrict__ spos, const float4* __restrict__ sw, int m0,
                                           int M, float4* __restrict__ far_acc, float4* s4, int n_valid = -1) {
  static_assert(!BLOB || D == 3, "the paired blob loop is 3-D");
  constexpr int NP = TT / 2;
  constexpr int NQ = far_x2_words<D, BLOB>();  // duplicated float4 per sample
  f2_t PX[NP], PY[NP], PZ[NP], AX[NP], AY[NP], AZ[NP];
  bool OK[2 * NP];
#pragma unroll
  for (int p = 0; p < NP; ++p) {
    const int t0 = tbase + (2 * p) * FT2 + threadIdx.x, t1 = tbase + (2 * p + 1) * FT2 + threadIdx.x;
    int i0 = t0 < nt ? t0 : nt - 1, i1 = t1 < nt ? t1 : nt - 1;
    if (targets) {
      i0 = targets[i0];
      i1 = targets[i1];
    }
    OK[2 * p] = n_valid < 0 || (i0 >= 0 && i0 < n_valid);
    OK[2 * p + 1] = n_valid < 0 || (i1 >= 0 && i1 < n_valid);
    const V3 a = ldv<D>(x, OK[2 * p] ? i0 : 0);
    const V3 b = ldv<D>(x, OK[2 * p + 1] ? i1 : 0);
    PX[p] = f2_pack(a.x, b.x);
    PY[p] = f2_pack(a.y, b.y);
    PZ[p] = f2_pack(a.z, b.z);
    AX[p] = AY[p] = AZ[p] = 0ull;
  }
  const float lim = P.far_r2_limit;
  const ulonglong2* s2 = reinterpret_cast<const ulonglong2*>(s4);
  for (int base = 0; base < M; base += FTILE2) {
    const int m = min(FTILE2, M - base);
    __syncthreads();
    for (int q = threadIdx.x; q < m; q += FT2) {
      const float4 sp = spos[m0 + base + q];
      const float4 w = sw[m0 + base + q];
      if (BLOB) {
        s4[5 * q] = make_float4(sp.x, sp.x, sp.y, sp.y);
        s4[5 * q + 1] = make_float4(sp.z, sp.z, w.z, w.z);
        s4[5 * q + 2] = make_float4(-w.y, -w.y, w.x, w.x);
        s4[5 * q + 3] = make_float4(-w.z, -w.z, w.y, w.y);
        s4[5 * q + 4] = make_float4(-w.x, -w.x, 0.0f, 0.0f);
      } else if (D == 3) {
        s4[4 * q] = make_float4(sp.x, sp.x, sp.y, sp.y);
        s4[4 * q + 1] = make_float4(sp.z, sp.z, w.z, w.z);
        s4[4 * q + 2] = make_float4(-w.z, -w.z, w.y, w.y);
        s4[4 * q + 3] = make_float4(-w.x, -w.x, 0.0f, 0.0f);
      } else {
        s4[2 * q] = make_float4(sp.x, sp.x, sp.y, sp.y);
        s4[2 * q + 1] = make_float4(w.z, w.z, -w.z, -w.z);
      }
    }
    __syncthreads();
    if (BLOB) {
      const float d2v = P.blob_delta2;
      const f2_t D2 = f2_pack(d2v, d2v);
#pragma unroll kFarQUnroll
      for (int q = 0; q < m; ++q) {
        const ulonglong2 v0 = s2[NQ * q], v1 = s2[NQ * q + 1], v2 = s2[NQ * q + 2], v3 = s2[NQ * q + 3];
        const ulonglong2 v4 = s2[NQ * q + 4];
        const f2_t SZ = v1.x, WZ = v1.y, NWY = v2.x, WX = v2.y, NWZ = v3.x, WY = v3.y, NWX = v4.x;
#pragma unroll
        for (int p = 0; p < NP; ++p) {
          const f2_t DX = f2_sub(PX[p], v0.x), DY = f2_sub(PY[p], v0.y), DZ = f2_sub(PZ[p], SZ);
          f2_t S2 = f2_fma(DX, DX, D2);
          S2 = f2_fma(DY, DY, S2);
          S2 = f2_fma(DZ, DZ, S2);
          float sa, sb;
          f2_unpack(S2, sa, sb);
          const f2_t KK = f2_mul(f2_pack(rcp_approx(sa), rcp_approx(sb)), f2_pack(rsqrt_approx(sa), rsqrt_approx(sb)));
          const f2_t A = f2_mul(KK, DX), B = f2_mul(KK, DY), E = f2_mul(KK, DZ);
          AX[p] = f2_fma(B, WZ, AX[p]);
          AX[p] = f2_fma(E, NWY, AX[p]);
          AY[p] = f2_fma(E, WX, AY[p]);
          AY[p] = f2_fma(A, NWZ, AY[p]);
          AZ[p] = f2_fma(A, WY, AZ[p]);
          AZ[p] = f2_fma(B, NWX, AZ[p]);
        }
      }
      continue;
    }
#pragma unroll kFarQUnroll
    for (int q = 0; q < m; ++q) {
      const ulonglong2 v0 = s2[NQ * q], v1 = s2[NQ * q + 1];
      f2_t SZ = 0ull, WZ, NWZ, WY = 0ull, NWX = 0ull;
      if (D == 3) {
        const ulonglong2 v2 = s2[NQ * q + 2], v3 = s2[NQ * q + 3];
        SZ = v1.x;
        WZ = v1.y;
        NWZ = v2.x;
        WY = v2.y;
        NWX = v3.x;
      } else {
        WZ = v1.x;
        NWZ = v1.y;
      }
#pragma unroll
      for (int p = 0; p < NP; ++p) {
        const f2_t DX = f2_sub(PX[p], v0.x), DY = f2_sub(PY[p], v0.y);
        f2_t R2 = f2_mul(DX, DX);
        R2 = f2_fma(DY, DY, R2);
        if (D == 3) {
          const f2_t DZ = f2_sub(PZ[p], SZ);
          R2 = f2_fma(DZ, DZ, R2);
        }
        float ra, rb;
        f2_unpack(R2, ra, rb);
        const f2_t KK = f2_pack(rcp_approx(fmaxf(ra, lim)), rcp_approx(fmaxf(rb, lim)));
        const f2_t A = f2_mul(KK, DX), B = f2_mul(KK, DY);
        AX[p] = f2_fma(B, WZ, AX[p]);
        AY[p] = f2_fma(A, NWZ, AY[p]);
        if (D == 3) {
          AZ[p] = f2_fma(A, WY, AZ[p]);
          AZ[p] = f2_fma(B, NWX, AZ[p]);
        }
      }
    }
  }
#pragma unroll
  for (int p = 0; p < NP; ++p) {
    float x0, x1, y0, y1, z0, z1;
    f2_unpack(AX[p], x0, x1);
    f2_unpack(AY[p], y0, y1);
    f2_unpack(AZ[p], z0, z1);
    const int t0 = tbase + (2 * p) * FT2 + threadIdx.x, t1 = tbase + (2 * p + 1) * FT2 + threadIdx.x;
    if (t0 < nt) far_acc[t0] = OK[2 * p] ? make_float4(x0, y0, z0, 0.0f) : make_float4(0.f, 0.f, 0.f, 0.f);
    if (t1 < nt) far_acc[t1] = OK[2 * p + 1] ? make_float4(x1, y1, z1, 0.0f) : make_float4(0.f, 0.f, 0.f, 0.f);
  }
}

template <int D, int TT, bool BLOB>
__global__ void __launch_bounds__(FT2, DV_FAR_MINB(TT)) k_far_main_x2(dv_params P, const float* __restrict__ x,
                                                     const dv_counters* __restrict__ C,
                                                     const int32_t* __restrict__ targets,
                                                     const float4* __restrict__ spos,
                                                     const float4* __restrict__ sw, float4* __restrict__ far_acc,
                                                     int nchunk, int64_t stride) {
  __shared__ float4 s4[far_x2_words<D, BLOB>() * FTILE2];
  const int nt = C->n_targets;
  const int tbase = blockIdx.x * FT2 * TT;
  if (tbase >= nt) return;  // uniform per CTA
  int m0, M;
  sample_chunk(C->num_samples, nchunk, m0, M);
  far_x2_run<D, TT, BLOB>(P, x, targets, nt, tbase, spos, sw, m0, M, far_acc + blockIdx.y * stride, s4);
}

template <int D, int TT>
__global__ void __launch_bounds__(FT2, DV_FAR_MINB(TT)) k_far_main_x2_b(dv_params P, const float* __restrict__ x,
                                                       const int32_t* __restrict__ targets,
                                                       const float4* __restrict__ spos,
                                                       const float4* __restrict__ sw,
                                                       const dv_scene_state* __restrict__ st,
                                                       const int32_t* __restrict__ order, int S,
                                                       const int32_t* __restrict__ ntiles,
                                                       float4* __restrict__ far_acc) {
  __shared__ float4 s4[(D == 3 ? 4 : 2) * FTILE2];
  const int blk = blockIdx.x;
  if (blk >= *ntiles) return;  // uniform per CTA
  const int sc = batch_block_scene(st, order, S, blk);
  const int t0 = st[sc].t_start;
  far_x2_run<D, TT>(P, x, targets + t0, st[sc].n_targets, (blk - st[sc].tile_off) * FT2 * TT, spos, sw,
                    st[sc].m_off, st[sc].num_samples, far_acc + t0, s4);
}

// targets per thread actually run for a requested tile: 2, 4 or 8, and 6
// for the paired loop (the scalar kernels have no 6)
static inline int far_tile_run(int tt, bool paired) {
  return tt <= 2 ? 2 : tt <= 4 ? 4 : (tt <= 6 && paired) ? 6 : 8;
}

template <int D, bool BLOB, bool COMP, bool PER>
static void launch_main_tt(dv_ctx* c, const dv_fields* f, int tt_req) {
  // the plain (uncompensated, non-periodic) loops: the reference kernel, and
  // the blob kernel in 3-D
  constexpr bool paired = !COMP && !PER && (!BLOB || D == 3);
  const int tt = far_tile_run(tt_req, paired);
  const int64_t nu = std::min<int64_t>(c->n_upper, c->cap);
  const int nb = (int)std::max<int64_t>(1, (nu + (int64_t)FT2 * tt - 1) / ((int64_t)FT2 * tt));
  const dim3 grid(nb, c->far_chunks);
#define L(TTV)                                                                                                 \
  k_far_main<D, TTV, BLOB, COMP, PER><<<grid, FT2, 0, c->stream>>>(c->p, f->x, c->d_cnt, c->targets, c->spos, \
                                                                   c->sw, c->far_acc, c->far_chunks, c->cap)
#define L2(TTV)                                                                                              \
  k_far_main_x2<D, TTV, BLOB && D == 3><<<grid, FT2, 0, c->stream>>>(c->p, f->x, c->d_cnt, c->targets, c->spos, \
                                                                     c->sw, c->far_acc, c->far_chunks, c->cap)
  if (tt == 2)
    L(2);
  else if (tt == 4) {
    if (paired)
      L2(4);
    else
      L(4);
  } else if (tt == 6) {
    L2(6);
  } else {
    if (paired)
      L2(8);
    else
      L(8);
  }
#undef L
#undef L2
}

template <int D, bool PER>
static void launch_main_p(dv_ctx* c, const dv_fields* f, int tt) {
  const bool blob = c->p.kernel_mode == DV_KERNEL_BLOB3D;
  const bool comp = c->p.compensated != 0;
  if (blob)
    comp ? launch_main_tt<D, true, true, PER>(c, f, tt) : launch_main_tt<D, true, false, PER>(c, f, tt);
  else
    comp ? launch_main_tt<D, false, true, PER>(c, f, tt) : launch_main_tt<D, false, false, PER>(c, f, tt);
}

template <int D>
static void launch_main(dv_ctx* c, const dv_fields* f, int tt) {
  if (c->p.periodic)
    launch_main_p<D, true>(c, f, tt);
  else
    launch_main_p<D, false>(c, f, tt);
}

template <int D>
static void launch_fix(dv_ctx* c, const dv_fields* f, const dv_solver_fields* s) {
  const int nb = dv_blocks(std::min<int64_t>(c->n_upper, c->cap), 128);
#define LF(B, PR)                                                                                      \
  k_far_fix<D, B, PR><<<nb, 128, 0, c->stream>>>(c->p, dv_grid(c), *f, *s, c->d_cnt, c->targets, c->mult, \
                                                 c->srank, c->sslot, c->far_acc, c->near_v, c->near_S,    \
                                                 c->far_chunks, c->cap)
  const bool blob = c->p.kernel_mode == DV_KERNEL_BLOB3D;
  if (c->p.periodic)
    blob ? LF(true, true) : LF(false, true);
  else
    blob ? LF(true, false) : LF(false, false);
#undef LF
}

__global__ void k_prof_pairs(const dv_counters* __restrict__ C, double* acc) {
  acc[0] += (double)C->n_targets * (double)C->num_samples;
}

static int prof_fold(dv_ctx* c) {
  for (int k = 0; k < c->prof_used; ++k) {
    float ms = 0.f;
    DV_CK(c, cudaEventSynchronize(c->prof_ev[2 * k + 1]));
    DV_CK(c, cudaEventElapsedTime(&ms, c->prof_ev[2 * k], c->prof_ev[2 * k + 1]));
    c->prof_ms += ms;
  }
  c->prof_used = 0;
  return DV_OK;
}

DV_API int dv_profile(dv_ctx* c, int32_t enable) {
  if (!c) return DV_EINVAL;
  int rc = prof_fold(c);
  if (rc) return rc;
  if (enable && !c->prof_ev[0])
    for (int k = 0; k < 2 * dv_ctx::kProfPool; ++k) DV_CK(c, cudaEventCreate(&c->prof_ev[k]));
  c->prof = enable != 0;
  c->prof_ms = 0.0;
  c->prof_launches = 0;
  DV_CK(c, cudaMemsetAsync(c->d_prof, 0, sizeof(double) * 4, c->stream));
  return DV_OK;
}

DV_API int dv_profile_read(dv_ctx* c, double* far_ms, int64_t* launches, double* pairs) {
  if (!c) return DV_EINVAL;
  int rc = prof_fold(c);
  if (rc) return rc;
  double h[4];
  DV_CK(c, cudaMemcpyAsync(h, c->d_prof, sizeof(double) * 4, cudaMemcpyDeviceToHost, c->stream));
  DV_CK(c, cudaStreamSynchronize(c->stream));
  if (far_ms) *far_ms = c->prof_ms;
  if (launches) *launches = c->prof_launches;
  if (pairs) *pairs = h[0];
  return DV_OK;
}

// Times the far-field main loop for 2, 4, 6 and 8 targets per thread on the
// current targets and samples (CUDA events, best of two launches after one
// warm-up) and keeps the fastest for this context.
DV_API int dv_autotune(dv_ctx* c, const dv_fields* f, const dv_solver_fields* s, int32_t* best_tt,
                       float* best_ms) {
  if (!c || !f || !s || !s->sample_idx) return DV_EINVAL;
  if (!fast_kernel_ok(c->p) && c->p.kernel_mode != DV_KERNEL_BLOB3D) return DV_OK;
  int rc = dv_build_targets(c, f);
  if (rc) return rc;
  const int packb = c->num_sms * 4;
  if (c->p.dim == 2)
    k_pack_samples<2><<<packb, DV_THREADS, 0, c->stream>>>(*f, *s, c->d_cnt, c->spos, c->sw, c->p.kden_eps);
  else
    k_pack_samples<3><<<packb, DV_THREADS, 0, c->stream>>>(*f, *s, c->d_cnt, c->spos, c->sw, c->p.kden_eps);
  DV_LAUNCHED(c);
  cudaEvent_t e0, e1;
  DV_CK(c, cudaEventCreate(&e0));
  DV_CK(c, cudaEventCreate(&e1));
  const int cand[4] = {2, 4, 6, 8};
  float best = 1e30f;
  int best_t = c->far_tt, best_c = c->far_chunks;
  for (int nc = 1; nc <= DV_MAX_FAR_CHUNKS; nc += nc < 4 ? 1 : 2) {  // 1, 2, 3, 4, 6, 8
    c->far_chunks = nc;
    for (int tt : cand) {
      for (int rep = 0; rep < 3; ++rep) {
        DV_CK(c, cudaEventRecord(e0, c->stream));
        if (c->p.dim == 2)
          launch_main<2>(c, f, tt);
        else
          launch_main<3>(c, f, tt);
        DV_LAUNCHED(c);
        DV_CK(c, cudaEventRecord(e1, c->stream));
        DV_CK(c, cudaEventSynchronize(e1));
        float ms = 0.f;
        DV_CK(c, cudaEventElapsedTime(&ms, e0, e1));
        if (rep > 0 && ms < best) {
          best = ms;
          best_t = tt;
          best_c = nc;
        }
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->far_tt = best_t;
  c->far_chunks = best_c;
  if (best_tt) *best_tt = best_t;
  if (best_ms) *best_ms = best;
  return DV_OK;
}

DV_API int dv_set_far_tile(dv_ctx* c, int32_t tt) {
  if (!c || (tt != 2 && tt != 4 && tt != 6 && tt != 8)) return DV_EINVAL;
  c->far_tt = tt;
  return DV_OK;
}

DV_API int dv_set_far_chunks(dv_ctx* c, int32_t chunks) {
  if (!c || chunks < 1 || chunks > DV_MAX_FAR_CHUNKS) return DV_EINVAL;
  c->far_chunks = chunks;
  return DV_OK;
}

DV_API int32_t dv_get_far_chunks(dv_ctx* c) { return c ? c->far_chunks : DV_EINVAL; }

DV_API int dv_vvpe_mc(dv_ctx* c, const dv_fields* f, const dv_solver_fields* s) {
  if (!c || !f || !s || !s->sample_idx || !s->kden || !s->d_vort_smoothed)
    return c ? dv_fail(c, DV_EINVAL, "dv_vvpe_mc: NULL field") : DV_EINVAL;
  int rc = dv_build_targets(c, f);
  if (rc) return rc;
  rc = dv_launch_vvpe_near(c, f, s);
  if (rc) return rc;
  const int packb = c->num_sms * 4;
  if (c->p.dim == 2)
    k_pack_samples<2><<<packb, DV_THREADS, 0, c->stream>>>(*f, *s, c->d_cnt, c->spos, c->sw,
                                                          c->p.kden_eps);
  else
    k_pack_samples<3><<<packb, DV_THREADS, 0, c->stream>>>(*f, *s, c->d_cnt, c->spos, c->sw,
                                                          c->p.kden_eps);
  DV_LAUNCHED(c);
  const int64_t nu = std::min<int64_t>(c->n_upper, c->cap);
  const bool fastk = fast_kernel_ok(c->p) || c->p.kernel_mode == DV_KERNEL_BLOB3D;
  if (!fastk && c->p.periodic)
    return dv_fail(c, DV_EUNSUPPORTED, "dv_vvpe_mc: periodic boxes need h > 1.05e-4 (reference kernel)");
  if (fastk) {  // split form: sample multiplicities for the correction kernel
    DV_CK(c, cudaMemsetAsync(c->mult, 0, sizeof(int32_t) * nu, c->stream));
    k_mult<<<c->num_sms * 4, DV_THREADS, 0, c->stream>>>(s->sample_idx, c->d_cnt, c->mult);
    DV_LAUNCHED(c);
    rc = sample_slots(c);
    if (rc) return rc;
  }
  if (c->prof) {
    if (c->prof_used == dv_ctx::kProfPool) {
      int rc2 = prof_fold(c);
      if (rc2) return rc2;
    }
    DV_CK(c, cudaEventRecord(c->prof_ev[2 * c->prof_used], c->stream));
  }
  if (fastk) {
    if (c->p.dim == 2)
      launch_main<2>(c, f, c->far_tt);
    else
      launch_main<3>(c, f, c->far_tt);
  } else {  // |r| > h may not underflow exp(-|r|/ε): per-pair exact kernel
    const int nb = (int)std::max<int64_t>(1, (nu + FT * 2 - 1) / (FT * 2));
    if (c->p.dim == 2)
      dispatch_far<2>(c, f, s, nb, false);
    else
      dispatch_far<3>(c, f, s, nb, false);
  }
  DV_LAUNCHED(c);
  if (c->prof) {
    DV_CK(c, cudaEventRecord(c->prof_ev[2 * c->prof_used + 1], c->stream));
  }
  if (fastk) {
    if (c->p.dim == 2)
      launch_fix<2>(c, f, s);
    else
      launch_fix<3>(c, f, s);
    DV_LAUNCHED(c);
  }
  if (c->prof) {
    c->prof_used++;
    c->prof_launches++;
    k_prof_pairs<<<1, 1, 0, c->stream>>>(c->d_cnt, c->d_prof);
    DV_LAUNCHED(c);
  }
  return DV_OK;
}

static inline bool batch_paired(const dv_ctx* c) {
  return c->p.kernel_mode != DV_KERNEL_BLOB3D && c->p.compensated == 0;
}

int dv_far_tile_width(const dv_ctx* c) { return FT2 * far_tile_run(c->far_tt, batch_paired(c)); }
int dv_far_min_tile_width() { return FT2 * 2; }

template <int D, bool BLOB, bool COMP>
static void launch_main_b(dv_ctx* c, const dv_fields* f) {
  dv_batch_state* b = c->batch;
  const int nb = (int)b->cap_tiles;
#define L(TTV)                                                                                             \
  k_far_main_b<D, TTV, BLOB, COMP><<<nb, FT2, 0, c->stream>>>(c->p, f->x, c->targets, c->spos, c->sw,      \
                                                              b->d_state, b->d_order, b->S, b->d_misc, c->far_acc)
#define L2(TTV)                                                                                            \
  k_far_main_x2_b<D, TTV><<<nb, FT2, 0, c->stream>>>(c->p, f->x, c->targets, c->spos, c->sw, b->d_state,    \
                                                     b->d_order, b->S, b->d_misc, c->far_acc)
  constexpr bool paired = !BLOB && !COMP;
  const int tt = far_tile_run(c->far_tt, paired);  // as dv_far_tile_width, which sized the tiles
  if (tt == 2) {
    if (paired)
      L2(2);
    else
      L(2);
  } else if (tt == 4) {
    if (paired)
      L2(4);
    else
      L(4);
  } else if (tt == 6) {
    L2(6);
  } else {
    if (paired)
      L2(8);
    else
      L(8);
  }
#undef L
#undef L2
}

// Scene batch VVPE: the targets are built (dv_build_targets) and the samples
// drawn (dv_batch_draw); near field and packing are the single-scene kernels
int dv_batch_vvpe(dv_ctx* c, const dv_fields* f, const dv_solver_fields* s) {
  dv_batch_state* b = c->batch;
  if (!fast_kernel_ok(c->p) && c->p.kernel_mode != DV_KERNEL_BLOB3D)
    return dv_fail(c, DV_EUNSUPPORTED, "scene batches need h > 1.05e-4 (reference kernel)");
  int rc = dv_launch_vvpe_near(c, f, s);
  if (rc) return rc;
  const int packb = c->num_sms * 4;
  if (c->p.dim == 2)
    k_pack_samples<2><<<packb, DV_THREADS, 0, c->stream>>>(*f, *s, c->d_cnt, c->spos, c->sw, c->p.kden_eps);
  else
    k_pack_samples<3><<<packb, DV_THREADS, 0, c->stream>>>(*f, *s, c->d_cnt, c->spos, c->sw, c->p.kden_eps);
  DV_LAUNCHED(c);
  DV_CK(c, cudaMemsetAsync(c->mult, 0, sizeof(int32_t) * c->cap, c->stream));
  k_mult<<<c->num_sms * 4, DV_THREADS, 0, c->stream>>>(s->sample_idx, c->d_cnt, c->mult);
  DV_LAUNCHED(c);
  rc = sample_slots(c);
  if (rc) return rc;
  const bool blob = c->p.kernel_mode == DV_KERNEL_BLOB3D, comp = c->p.compensated != 0;
#define LB(DD)                                                                             \
  if (blob)                                                                                \
    comp ? launch_main_b<DD, true, true>(c, f) : launch_main_b<DD, true, false>(c, f);     \
  else                                                                                     \
    comp ? launch_main_b<DD, false, true>(c, f) : launch_main_b<DD, false, false>(c, f);
  if (c->p.dim == 2) {
    LB(2);
  } else {
    LB(3);
  }
#undef LB
  DV_LAUNCHED(c);
  const int nb = dv_blocks(c->cap, 128);
#define LF(DD, B)                                                                                         \
  k_far_fix_b<DD, B><<<nb, 128, 0, c->stream>>>(c->p, dv_grid(c), *f, *s, c->d_cnt, c->targets, c->mult,   \
                                                c->srank, c->sslot, c->far_acc, c->near_v, c->near_S,     \
                                                b->d_state)
  if (c->p.dim == 2)
    blob ? LF(2, true) : LF(2, false);
  else
    blob ? LF(3, true) : LF(3, false);
#undef LF
  DV_LAUNCHED(c);
  return DV_OK;
}

// ------------------------------------------------------------ full BS
// sources: fluid slots in ascending order, (x, y, z, slot bits) and ω
template <int D>
__global__ void k_flag_fluid(const dv_fields F, const dv_counters* __restrict__ C, int m,
                             uint32_t* __restrict__ flags) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  flags[i] = (i < C->n && F.material[i] == DV_MATERIAL_FLUID) ? 1u : 0u;
}

template <int D>
__global__ void k_pack_sources(const dv_fields F, const float* __restrict__ omega,
                               const uint32_t* __restrict__ flags, const uint32_t* __restrict__ offs,
                               const dv_counters* __restrict__ C, float4* __restrict__ spos,
                               float4* __restrict__ sw, int32_t* __restrict__ ns_out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = C->n;
  if (i == 0) *ns_out = (int32_t)offs[n];
  if (i >= n || !flags[i]) return;
  uint32_t q = offs[i];
  V3 x = ldv<D>(F.x, i);
  float4 w = reinterpret_cast<const float4*>(omega)[i];
  spos[q] = make_float4(x.x, x.y, x.z, __int_as_float(i));
  sw[q] = make_float4(w.x, w.y, w.z, 0.0f);
}

// Σ_{j fluid, j != i} kernel(r_ij) (r × ω_j) for target slots; T = float or
// double (the FP64 comparator).  Reference kernel: Kε(|r|) (r_xy × ω), with
// the exact regularised form where exp(-|r|/ε) does not underflow and a zero
// contribution from coincident pairs (the limit of Kε(r) r as r -> 0).
template <int D, typename T, bool BLOB>
__global__ void __launch_bounds__(FT) k_bs_full(dv_params P, const float* __restrict__ x,
                                                const int32_t* __restrict__ tlist, int nt,
                                                const float4* __restrict__ spos,
                                                const float4* __restrict__ sw,
                                                const int32_t* __restrict__ ns_p, const dv_counters* __restrict__ C,
                                                T* __restrict__ out) {
  __shared__ float4 s_p[FTILE];
  __shared__ float4 s_w[FTILE];
  const int ns = *ns_p;
  const int t = blockIdx.x * FT + threadIdx.x;
  int i = t < nt ? (tlist ? tlist[t] : t) : -1;
  if (t < nt && (i < 0 || i >= C->n)) {  // caller target outside [0, n): zero output
    out[(int64_t)t * 4 + 0] = 0;
    out[(int64_t)t * 4 + 1] = 0;
    out[(int64_t)t * 4 + 2] = 0;
    out[(int64_t)t * 4 + 3] = 0;
    i = -1;
  }
  T px = 0, py = 0, pz = 0;
  if (i >= 0) {
    V3 xi = ldv<D>(x, i);
    px = (T)xi.x;
    py = (T)xi.y;
    pz = (T)xi.z;
  }
  T ax = 0, ay = 0, az = 0;
  const T eps = (T)P.eps, inv_eps = (T)P.inv_eps, d2 = (T)P.blob_delta2;
  // exp(-|r|/ε) underflows below these |r|² bounds (f32: 104 ε, f64: 746 ε)
  const T under = sizeof(T) == 4 ? (T)(104.5 * 104.5) * eps * eps : (T)(746.0 * 746.0) * eps * eps;
  for (int base = 0; base < ns; base += FTILE) {
    const int m = min(FTILE, ns - base);
    __syncthreads();
    for (int q = threadIdx.x; q < m; q += FT) {
      s_p[q] = spos[base + q];
      s_w[q] = sw[base + q];
    }
    __syncthreads();
    if (i < 0) continue;
    for (int q = 0; q < m; ++q) {
      const float4 sp = s_p[q];
      if (__float_as_int(sp.w) == i) continue;
      const float4 w = s_w[q];
      T dx = px - (T)sp.x, dy = py - (T)sp.y, dz = D == 3 ? pz - (T)sp.z : (T)0;
      if (P.periodic) {  // minimum image
        const T L0 = (T)P.box[0], L1 = (T)P.box[1], L2 = (T)P.box[2];
        dx = dx > L0 / 2 ? dx - L0 : (dx < -L0 / 2 ? dx + L0 : dx);
        dy = dy > L1 / 2 ? dy - L1 : (dy < -L1 / 2 ? dy + L1 : dy);
        if (D == 3) dz = dz > L2 / 2 ? dz - L2 : (dz < -L2 / 2 ? dz + L2 : dz);
      }
      T r2 = dx * dx + dy * dy + dz * dz;
      if (r2 == (T)0) continue;
      if (!BLOB) {
        T kk;
        if (r2 > under) {
          kk = (T)1 / r2;
        } else {
          T rn = sqrt(r2);
          T e = exp(-rn * inv_eps);
          kk = ((T)1 - e) / (rn * (rn + eps * e));
        }
        T tz = kk * (T)w.z;
        ax += tz * dy;
        ay -= tz * dx;
        az += kk * (dx * (T)w.y - dy * (T)w.x);
      } else {
        T s = r2 + d2;
        T kk = (T)1 / (s * sqrt(s));
        ax += kk * (dy * (T)w.z - dz * (T)w.y);
        ay += kk * (dz * (T)w.x - dx * (T)w.z);
        az += kk * (dx * (T)w.y - dy * (T)w.x);
      }
    }
  }
  if (i < 0) return;
  const T coef = BLOB ? (T)P.blob_coef : (T)P.vvpe_coef;
  out[(int64_t)t * 4 + 0] = ax * coef;
  out[(int64_t)t * 4 + 1] = ay * coef;
  out[(int64_t)t * 4 + 2] = az * coef;
  out[(int64_t)t * 4 + 3] = 0;
}

// FP32 full Biot-Savart with the blob kernel, in the register-tiled form of
// the far-field main loop: the blob kernel is regular at r = 0 and the self
// pair contributes r × ω = 0 exactly, so every (target, source) pair is
// summed without a test.
template <int D, int TT, bool COMP>
__global__ void __launch_bounds__(FT2) k_bs_fast(dv_params P, const float* __restrict__ x,
                                                 const int32_t* __restrict__ tlist, int nt,
                                                 const float4* __restrict__ spos, const float4* __restrict__ sw,
                                                 const int32_t* __restrict__ ns_p,
                                                 const dv_counters* __restrict__ C, float* __restrict__ out) {
  __shared__ float4 s_p[FTILE2];
  __shared__ float4 s_w[FTILE2];
  const int ns = *ns_p;
  const int n = C->n;
  const int tbase = blockIdx.x * FT2 * TT;
  if (tbase >= nt) return;
  float px[TT], py[TT], pz[TT];
  Acc<COMP> ax[TT], ay[TT], az[TT];
  bool ok[TT];
#pragma unroll
  for (int k = 0; k < TT; ++k) {
    int t = tbase + k * FT2 + threadIdx.x;
    int i = t < nt ? (tlist ? tlist[t] : t) : 0;
    ok[k] = t < nt && i >= 0 && i < n;
    V3 xi = ldv<D>(x, ok[k] ? i : 0);
    px[k] = xi.x;
    py[k] = xi.y;
    pz[k] = xi.z;
  }
  const float d2 = P.blob_delta2;
  for (int base = 0; base < ns; base += FTILE2) {
    const int m = min(FTILE2, ns - base);
    __syncthreads();
    for (int q = threadIdx.x; q < m; q += FT2) {
      s_p[q] = spos[base + q];
      s_w[q] = sw[base + q];
    }
    __syncthreads();
#pragma unroll 4
    for (int q = 0; q < m; ++q) {
      const float4 sp = s_p[q];
      const float4 w = s_w[q];
#pragma unroll
      for (int k = 0; k < TT; ++k) far_accum<D, true, COMP>(px[k], py[k], pz[k], sp, w, 0.0f, d2, ax[k], ay[k], az[k]);
    }
  }
  const float coef = P.blob_coef;
#pragma unroll
  for (int k = 0; k < TT; ++k) {
    int t = tbase + k * FT2 + threadIdx.x;
    if (t >= nt) continue;
    float4 o = ok[k] ? make_float4(ax[k].val() * coef, ay[k].val() * coef, az[k].val() * coef, 0.0f)
                     : make_float4(0.f, 0.f, 0.f, 0.f);
    reinterpret_cast<float4*>(out)[t] = o;
  }
}

// The same sum with two targets per f32x2 instruction (3-D): the grid is
// (target tiles) x (source chunks), each CTA writes its chunk's partial sums
// to acc[chunk * stride + t] and k_bs_chunk_sum adds the chunks in order, so
// the result does not depend on the schedule.  The chunks give a grid of many
// waves on a 1M x 1M sum, where whole-range CTAs would leave most of the
// last wave idle.
template <int TT>
__global__ void __launch_bounds__(FT2, DV_FAR_MINB(TT)) k_bs_x2(dv_params P, const float* __restrict__ x,
                                                               const int32_t* __restrict__ tlist, int nt,
                                                               const float4* __restrict__ spos,
                                                               const float4* __restrict__ sw,
                                                               const int32_t* __restrict__ ns_p,
                                                               const dv_counters* __restrict__ C, int nchunk,
                                                               int64_t stride, float4* __restrict__ acc) {
  __shared__ float4 s4[far_x2_words<3, true>() * FTILE2];
  const int tbase = blockIdx.x * FT2 * TT;
  if (tbase >= nt) return;  // uniform per CTA
  const int ns = *ns_p;
  const int clen = (ns + nchunk - 1) / nchunk;
  const int m0 = (int)blockIdx.y * clen;
  const int M = max(0, min(clen, ns - m0));
  far_x2_run<3, TT, true>(P, x, tlist, nt, tbase, spos, sw, m0, M, acc + blockIdx.y * stride, s4, C->n);
}

__global__ void k_bs_chunk_sum(const float4* __restrict__ acc, int nt, int nchunk, int64_t stride, float coef,
                               float* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  float4 a = acc[t];
  for (int k = 1; k < nchunk; ++k) {
    const float4 b = acc[k * stride + t];
    a.x += b.x;
    a.y += b.y;
    a.z += b.z;
  }
  reinterpret_cast<float4*>(out)[t] = make_float4(a.x * coef, a.y * coef, a.z * coef, 0.0f);
}

template <int TTV>
static int launch_bs_x2(dv_ctx* c, const dv_fields* f, const int32_t* targets, int nt, const int32_t* ns,
                        float* out) {
  const int64_t tiles = ((int64_t)nt + (int64_t)FT2 * TTV - 1) / ((int64_t)FT2 * TTV);
  const int64_t resident = (int64_t)c->num_sms * DV_FAR_MINB(TTV) * 256 / FT2;
  // enough chunks for about eight waves, within the partial-sum buffer
  const int nchunk =
      (int)std::max<int64_t>(1, std::min<int64_t>(DV_MAX_FAR_CHUNKS, (8 * resident + tiles - 1) / tiles));
  const dim3 grid((unsigned)tiles, nchunk);
  k_bs_x2<TTV><<<grid, FT2, 0, c->stream>>>(c->p, f->x, targets, nt, c->spos, c->sw, ns, c->d_cnt, nchunk, c->cap,
                                            c->far_acc);
  DV_LAUNCHED(c);
  k_bs_chunk_sum<<<dv_blocks(nt), DV_THREADS, 0, c->stream>>>(c->far_acc, nt, nchunk, c->cap, c->p.blob_coef, out);
  DV_LAUNCHED(c);
  return DV_OK;
}

template <int D>
static int bs_dispatch(dv_ctx* c, const dv_fields* f, const int32_t* targets, int nt, void* out,
                       int precision) {
  const int nb = dv_blocks(nt, FT);
  const bool blob = c->p.kernel_mode == DV_KERNEL_BLOB3D;
  const int32_t* ns = c->d_flag + 2;
  if (precision == 32 && blob && !c->p.periodic && !c->p.compensated && D == 3 && c->far_tt > 2) {
    // the paired loop (a tile of 2 keeps the scalar loop below)
    if (c->far_tt <= 4) return launch_bs_x2<4>(c, f, targets, nt, ns, (float*)out);
    if (c->far_tt <= 6) return launch_bs_x2<6>(c, f, targets, nt, ns, (float*)out);
    return launch_bs_x2<8>(c, f, targets, nt, ns, (float*)out);
  }
  if (precision == 32 && blob && !c->p.periodic) {
    const int tt = c->far_tt <= 2 ? 2 : (c->far_tt <= 4 ? 4 : 8);
    const int nbf = (int)std::max<int64_t>(1, ((int64_t)nt + (int64_t)FT2 * tt - 1) / ((int64_t)FT2 * tt));
#define LBS(TTV, CV)                                                                                          \
  k_bs_fast<D, TTV, CV><<<nbf, FT2, 0, c->stream>>>(c->p, f->x, targets, nt, c->spos, c->sw, ns, c->d_cnt, \
                                                    (float*)out)
    const bool comp = c->p.compensated != 0;
    if (tt == 2)
      comp ? LBS(2, true) : LBS(2, false);
    else if (tt == 4)
      comp ? LBS(4, true) : LBS(4, false);
    else
      comp ? LBS(8, true) : LBS(8, false);
#undef LBS
    DV_LAUNCHED(c);
    return DV_OK;
  }
  if (precision == 64) {
    if (blob)
      k_bs_full<D, double, true><<<nb, FT, 0, c->stream>>>(c->p, f->x, targets, nt, c->spos, c->sw, ns, c->d_cnt,
                                                           (double*)out);
    else
      k_bs_full<D, double, false><<<nb, FT, 0, c->stream>>>(c->p, f->x, targets, nt, c->spos, c->sw, ns, c->d_cnt,
                                                            (double*)out);
  } else {
    if (blob)
      k_bs_full<D, float, true><<<nb, FT, 0, c->stream>>>(c->p, f->x, targets, nt, c->spos, c->sw, ns, c->d_cnt,
                                                          (float*)out);
    else
      k_bs_full<D, float, false><<<nb, FT, 0, c->stream>>>(c->p, f->x, targets, nt, c->spos, c->sw, ns, c->d_cnt,
                                                           (float*)out);
  }
  DV_LAUNCHED(c);
  return DV_OK;
}

DV_API int dv_bs_full(dv_ctx* c, const dv_fields* f, const float* omega, const int32_t* targets,
                      int32_t nt, void* out, int32_t precision) {
  if (!c || !f || !f->x || !f->material || !omega || !out) return DV_EINVAL;
  if (precision != 32 && precision != 64)
    return dv_fail(c, DV_EINVAL, "dv_bs_full: precision must be 32 or 64");
  if (nt < 0 || nt > c->cap) return dv_fail(c, DV_EINVAL, "dv_bs_full: nt=%d out of range", nt);
  if (nt == 0) return DV_OK;
  const int m = (int)std::min<int64_t>(c->n_upper, c->cap) + 1;
  const int nb = dv_blocks(m);
  if (c->p.dim == 2)
    k_flag_fluid<2><<<nb, DV_THREADS, 0, c->stream>>>(*f, c->d_cnt, m, c->flags);
  else
    k_flag_fluid<3><<<nb, DV_THREADS, 0, c->stream>>>(*f, c->d_cnt, m, c->flags);
  DV_LAUNCHED(c);
  int rc = dv_scan_u32(c, c->flags, c->offs, m);
  if (rc) return rc;
  if (c->p.dim == 2)
    k_pack_sources<2><<<nb, DV_THREADS, 0, c->stream>>>(*f, omega, c->flags, c->offs, c->d_cnt, c->spos,
                                                        c->sw, c->d_flag + 2);
  else
    k_pack_sources<3><<<nb, DV_THREADS, 0, c->stream>>>(*f, omega, c->flags, c->offs, c->d_cnt, c->spos,
                                                        c->sw, c->d_flag + 2);
  DV_LAUNCHED(c);
  return c->p.dim == 2 ? bs_dispatch<2>(c, f, targets, nt, out, precision)
                       : bs_dispatch<3>(c, f, targets, nt, out, precision);
}
