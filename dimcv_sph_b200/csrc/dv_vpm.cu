// Differentiable vortex-particle step (2-D, scalar vorticity ω = ω_z) with
// hand-written vector-Jacobian products.  New form: the reference has no
// derivatives.  The step is the reference's SPH vorticity smoothing followed
// by its Monte-Carlo Biot-Savart velocity, on arrays in sorted-slot order:
//
//   ω̃_i = m_V_i W(0) ω_i + Σ_{j∈N(i)} m_V_j W(r_ij) ω_j
//         (compute_all_d_vort_smoothed, dimcv_sph.py:660-677)
//   u_i = Σ_{j∈N(i)} [c Kε(r_ij) − f_i a_j / r_ij²] ω̃_j r_ij⊥
//         + f_i Σ_s a_s ω̃_s r_is⊥ / r_is²              (vort2vel, dimcv_sph.py:649-719)
//
// with r⊥ = (r_y, −r_x) (the z-cross of the 2-D-projected kernel), c the
// 0.1592·vp_volume factor, Kε the regularised kernel (1 − e)/(r(r + εe)),
// e = exp(−r/ε), a_s = multiplicity_s / (kden_s + 1e-8), and
// f_i = c (S − S_i) / (M − near samples of i).  The second sum runs over the
// distinct sampled particles; the −f_i a_j / r² term removes the samples
// inside the support of i from it, as the reference's `r > h` test does.
//
// A plan freezes everything that is piecewise constant in the positions:
// neighbour lists, samples and their weights, the far factors f_i and, when
// `xbar` is given, the periodic image of every pair.  The VJPs are the exact
// derivatives of the step with that structure held fixed, which is the
// derivative of the Monte-Carlo step wherever it exists (everywhere except on
// the measure-zero sets where a pair crosses the support radius or half a
// periodic box).
//
// Kernels are templates on the precision T (float, double).  The far field
// runs as a 2-D grid (target blocks × source chunks) with per-chunk partials
// summed in fixed order, so every result is deterministic.  Its VJP computes
// the target-side and the source-side gradient in one pass over the pairs:
// the target side in registers, the source side by a butterfly warp
// reduction per source and a fixed-order sum over warps and target blocks.
#include <algorithm>

#include "dv_internal.cuh"

namespace {

constexpr int VT = 256;  // threads per block of the pair kernels
constexpr int VTT = 2;   // targets per thread
constexpr int VTS = 128; // sources per shared-memory tile

template <typename T>
struct Geo {
  T Lx, Ly, iLx, iLy;  // periodic box and its inverse
  T invh, kW, c, eps, inv_eps, tiny, rmin;
};

template <typename T>
Geo<T> make_geo(const dv_params& P) {
  Geo<T> g;
  g.Lx = (T)P.box[0];
  g.Ly = (T)P.box[1];
  g.iLx = P.periodic ? (T)(1.0 / (double)P.box[0]) : T(0);
  g.iLy = P.periodic ? (T)(1.0 / (double)P.box[1]) : T(0);
  g.invh = (T)P.inv_support_radius;
  g.kW = (T)P.kW;
  g.c = (T)P.vvpe_coef;
  g.eps = (T)P.eps;
  g.inv_eps = (T)P.inv_eps;
  g.tiny = sizeof(T) == 4 ? (T)1e-30 : (T)1e-280;
  g.rmin = (T)P.grad_r_min;
  return g;
}

template <typename T>
__device__ __forceinline__ T rnd(T v);
template <>
__device__ __forceinline__ float rnd(float v) { return rintf(v); }
template <>
__device__ __forceinline__ double rnd(double v) { return rint(v); }

template <typename T>
__device__ __forceinline__ T ex(T v);
template <>
__device__ __forceinline__ float ex(float v) { return expf(v); }
template <>
__device__ __forceinline__ double ex(double v) { return exp(v); }

// 1/r² of the far-field kernel; 0 for coincident points (whose r⊥ is 0)
template <typename T>
__device__ __forceinline__ T inv_r2(T r2, T tiny);
template <>
__device__ __forceinline__ float inv_r2(float r2, float tiny) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(r2));
  return r2 > tiny ? r : 0.0f;
}
template <>
__device__ __forceinline__ double inv_r2(double r2, double tiny) {
  return r2 > tiny ? 1.0 / r2 : 0.0;
}

template <typename T>
struct P2 {
  T x, y;
};
template <typename T>
__device__ __forceinline__ P2<T> ld2(const T* a, int i) {
  return P2<T>{a[2 * i], a[2 * i + 1]};
}

// pair difference a − b on one axis: IMG 0 plain, 1 minimum image,
// 2 the image that the nominal positions abar, bbar select
template <typename T, int IMG>
__device__ __forceinline__ T pd(T a, T b, T abar, T bbar, T L, T iL) {
  T d = a - b;
  if (IMG == 1) d -= L * rnd<T>(d * iL);
  if (IMG == 2) d -= L * rnd<T>((abar - bbar) * iL);
  return d;
}

// cubic spline W(r) and dW/dr (sph_base.py:23-68 with kW = k h^-d)
template <typename T>
__device__ __forceinline__ void w_dw(const Geo<T>& g, T r, T& W, T& dW) {
  const T q = r * g.invh;
  if (q > T(1)) {
    W = T(0);
    dW = T(0);
  } else if (q <= T(0.5)) {
    W = g.kW * (T(6) * q * q * (q - T(1)) + T(1));
    dW = g.kW * g.invh * (T(6) * q * (T(3) * q - T(2)));
  } else {
    const T f = T(1) - q;
    W = T(2) * g.kW * f * f * f;
    dW = T(-6) * g.kW * g.invh * f * f;
  }
}

// dW/dr and d²W/dr² of the cubic spline (C² at q = 1/2 and q = 1)
template <typename T>
__device__ __forceinline__ void w_d12(const Geo<T>& g, T r, T& d1, T& d2) {
  const T q = r * g.invh;
  if (q > T(1)) {
    d1 = T(0);
    d2 = T(0);
  } else if (q <= T(0.5)) {
    d1 = g.kW * g.invh * (T(6) * q * (T(3) * q - T(2)));
    d2 = g.kW * g.invh * g.invh * (T(36) * q - T(12));
  } else {
    const T f = T(1) - q;
    d1 = T(-6) * g.kW * g.invh * f * f;
    d2 = T(12) * g.kW * g.invh * g.invh * f;
  }
}

// regularised kernel Kε(r) = (1 − e)/(r (r + ε e)), e = exp(−r/ε), and dKε/dr
template <typename T>
__device__ __forceinline__ void keps(const Geo<T>& g, T rn, T& K, T& dK) {
  if (!(rn > T(0))) {
    K = T(0);
    dK = T(0);
    return;
  }
  const T e = ex<T>(-rn * g.inv_eps);
  const T D = rn * (rn + g.eps * e);
  const T N = T(1) - e;
  const T iD = T(1) / D;
  K = N * iD;
  dK = ((e * g.inv_eps) * D - N * (T(2) * rn + g.eps * e - rn * e)) * iD * iD;
}

template <typename T, int IMG>
__device__ __forceinline__ P2<T> rel(const Geo<T>& g, const T* x, const T* xb, int i, int j) {
  const P2<T> a = ld2(x, i), b = ld2(x, j);
  P2<T> ab{T(0), T(0)}, bb{T(0), T(0)};
  if (IMG == 2) {
    ab = ld2(xb, i);
    bb = ld2(xb, j);
  }
  return P2<T>{pd<T, IMG>(a.x, b.x, ab.x, bb.x, g.Lx, g.iLx), pd<T, IMG>(a.y, b.y, ab.y, bb.y, g.Ly, g.iLy)};
}

// ------------------------------------------------------------ smoothing
template <typename T, int IMG>
__global__ void k_smooth(Geo<T> g, dv_vpm_plan p, const T* __restrict__ x, const T* __restrict__ xb,
                         const T* __restrict__ w, T* __restrict__ ws) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.n) return;
  T acc = (T)p.m_V[i] * g.kW * w[i];  // W(0) = kW
  const int k1 = p.nbr_off[i + 1];
  for (int k = p.nbr_off[i]; k < k1; ++k) {
    const int j = p.nbr[k];
    const P2<T> r = rel<T, IMG>(g, x, xb, i, j);
    T W, dW;
    w_dw<T>(g, sqrt(r.x * r.x + r.y * r.y), W, dW);
    acc += (T)p.m_V[j] * W * w[j];
  }
  ws[i] = acc;
}

template <typename T, int IMG>
__global__ void k_smooth_bwd(Geo<T> g, dv_vpm_plan p, const T* __restrict__ x, const T* __restrict__ xb,
                             const T* __restrict__ w, const T* __restrict__ gs, T* __restrict__ gw,
                             T* __restrict__ gx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.n) return;
  const T mi = (T)p.m_V[i], gsi = gs[i], wi = w[i];
  T a = mi * g.kW * gsi;
  T ax = T(0), ay = T(0);
  const int k1 = p.nbr_off[i + 1];
  for (int k = p.nbr_off[i]; k < k1; ++k) {
    const int j = p.nbr[k];
    const P2<T> r = rel<T, IMG>(g, x, xb, i, j);
    const T rn = sqrt(r.x * r.x + r.y * r.y);
    T W, dW;
    w_dw<T>(g, rn, W, dW);
    const T gsj = gs[j];
    a += mi * W * gsj;  // ∂ω̃_j/∂ω_i = m_V_i W(r_ij)
    if (rn > T(0)) {
      const T cf = dW / rn * (gsi * (T)p.m_V[j] * w[j] + gsj * mi * wi);
      ax += cf * r.x;
      ay += cf * r.y;
    }
  }
  gw[i] = a;
  gx[2 * i] = ax;
  gx[2 * i + 1] = ay;
}

// ------------------------------------------------------------ SPH curl
// compute_vorticity (dimcv_sph.py:228-248) in 2-D: ω_i = Σ_{j∈N(i)} m_V_j
// ((v_j − v_i) × ∇W(r_ij))_z with ∇W = W'(|r|) r/|r|, zero for |r| <= 1e-5.
template <typename T, int IMG>
__global__ void k_curl(Geo<T> g, dv_vpm_plan p, const T* __restrict__ x, const T* __restrict__ xb,
                       const T* __restrict__ v, T* __restrict__ w) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.n) return;
  const P2<T> vi = ld2(v, i);
  T acc = T(0);
  const int k1 = p.nbr_off[i + 1];
  for (int k = p.nbr_off[i]; k < k1; ++k) {
    const int j = p.nbr[k];
    const P2<T> r = rel<T, IMG>(g, x, xb, i, j);
    const T rn = sqrt(r.x * r.x + r.y * r.y);
    if (!(rn > g.rmin)) continue;
    T d1, d2;
    w_d12<T>(g, rn, d1, d2);
    const T s = d1 / rn;
    const P2<T> vj = ld2(v, j);
    const T ax = vj.x - vi.x, ay = vj.y - vi.y;
    acc += (T)p.m_V[j] * (ax * (s * r.y) - ay * (s * r.x));
  }
  w[i] = acc;
}

// VJP of k_curl.  With G = ∇W(r_kj), a = v_j − v_k, H = ∂G/∂r:
//   g_v_k = −Σ_j (g_j m_k + g_k m_j) (G_y, −G_x)
//   g_x_k =  Σ_j (g_j m_k + g_k m_j) H (−a_y, a_x)
// H = (W'' − W'/|r|) r̂ r̂ᵀ + (W'/|r|) I (the Hessian of W(|r|), even in r).
template <typename T, int IMG>
__global__ void k_curl_bwd(Geo<T> g, dv_vpm_plan p, const T* __restrict__ x, const T* __restrict__ xb,
                           const T* __restrict__ v, const T* __restrict__ gw, T* __restrict__ gv,
                           T* __restrict__ gx) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= p.n) return;
  const P2<T> vk = ld2(v, k);
  const T gk = gw[k], mk = (T)p.m_V[k];
  T vx = T(0), vy = T(0), xx = T(0), xy = T(0);
  const int k1 = p.nbr_off[k + 1];
  for (int e = p.nbr_off[k]; e < k1; ++e) {
    const int j = p.nbr[e];
    const P2<T> r = rel<T, IMG>(g, x, xb, k, j);
    const T rn = sqrt(r.x * r.x + r.y * r.y);
    if (!(rn > g.rmin)) continue;
    T d1, d2;
    w_d12<T>(g, rn, d1, d2);
    const T sw = gw[j] * mk + gk * (T)p.m_V[j];
    const T s = d1 / rn;
    vx -= sw * (s * r.y);
    vy += sw * (s * r.x);
    const P2<T> vj = ld2(v, j);
    const T bx = -(vj.y - vk.y), by = vj.x - vk.x;  // Rᵀ a
    const T hx = r.x / rn, hy = r.y / rn;
    const T proj = (d2 - s) * (hx * bx + hy * by);
    xx += sw * (proj * hx + s * bx);
    xy += sw * (proj * hy + s * by);
  }
  gv[2 * k] = vx;
  gv[2 * k + 1] = vy;
  gx[2 * k] = xx;
  gx[2 * k + 1] = xy;
}

// ------------------------------------------------------------ velocity
struct Layout {
  int ntb, nch, chunk;
  int64_t sp, spb, part, tpart, spart, sg, total;  // byte offsets / total
};

template <typename T>
Layout layout(int n, int src_cap, int num_sms) {
  Layout L;
  L.ntb = std::max(1, (n + VT * VTT - 1) / (VT * VTT));
  const int want = (2 * num_sms + L.ntb - 1) / L.ntb;
  const int maxch = std::max(1, (src_cap + VTS - 1) / VTS);
  L.nch = std::max(1, std::min(want, maxch));
  L.chunk = std::max(1, (src_cap + L.nch - 1) / L.nch);
  auto al = [](int64_t b) { return (b + 255) & ~int64_t(255); };
  const int64_t t = sizeof(T);
  int64_t o = 0;
  L.sp = o;
  o += al(t * 3 * (int64_t)std::max(src_cap, 1));
  L.spb = o;
  o += al(t * 2 * (int64_t)std::max(src_cap, 1));
  L.part = o;
  o += al(t * 2 * (int64_t)L.nch * n);
  L.tpart = o;
  o += al(t * 3 * (int64_t)L.nch * n);
  L.spart = o;
  o += al(t * 5 * (int64_t)L.ntb * std::max(src_cap, 1));
  L.sg = o;
  o += al(t * 3 * (int64_t)std::max(src_cap, 1));
  L.total = o;
  return L;
}

template <typename T>
__global__ void k_pack(dv_vpm_plan p, const T* __restrict__ x, const T* __restrict__ xb,
                       const T* __restrict__ wt, T* __restrict__ sp, T* __restrict__ spb) {
  const int ns = *p.n_src;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < ns; s += gridDim.x * blockDim.x) {
    const int j = p.src[s];
    sp[3 * s] = x[2 * j];
    sp[3 * s + 1] = x[2 * j + 1];
    sp[3 * s + 2] = (T)p.src_a[s] * wt[j];
    if (xb) {
      spb[2 * s] = xb[2 * j];
      spb[2 * s + 1] = xb[2 * j + 1];
    }
  }
}

template <typename T, int IMG>
__global__ void __launch_bounds__(VT) k_far(Geo<T> g, dv_vpm_plan p, const T* __restrict__ x,
                                            const T* __restrict__ xb, const T* __restrict__ sp,
                                            const T* __restrict__ spb, int chunk, T* __restrict__ part) {
  __shared__ T s_p[VTS * 3];
  __shared__ T s_b[IMG == 2 ? VTS * 2 : 2];
  const int n = p.n, ns = *p.n_src;
  const int tid = threadIdx.x, ch = blockIdx.y;
  const int s0 = ch * chunk, s1 = min(ns, s0 + chunk);
  T px[VTT], py[VTT], bx[VTT], by[VTT], ax[VTT], ay[VTT];
#pragma unroll
  for (int k = 0; k < VTT; ++k) {
    const int t = blockIdx.x * VT * VTT + k * VT + tid;
    const bool ok = t < n;
    px[k] = ok ? x[2 * t] : T(0);
    py[k] = ok ? x[2 * t + 1] : T(0);
    bx[k] = (IMG == 2 && ok) ? xb[2 * t] : T(0);
    by[k] = (IMG == 2 && ok) ? xb[2 * t + 1] : T(0);
    ax[k] = T(0);
    ay[k] = T(0);
  }
  for (int base = s0; base < s1; base += VTS) {
    const int cnt = min(VTS, s1 - base);
    __syncthreads();
    if (tid < cnt) {
      s_p[3 * tid] = sp[3 * (base + tid)];
      s_p[3 * tid + 1] = sp[3 * (base + tid) + 1];
      s_p[3 * tid + 2] = sp[3 * (base + tid) + 2];
      if (IMG == 2) {
        s_b[2 * tid] = spb[2 * (base + tid)];
        s_b[2 * tid + 1] = spb[2 * (base + tid) + 1];
      }
    }
    __syncthreads();
#pragma unroll 4
    for (int q = 0; q < cnt; ++q) {
      const T sx = s_p[3 * q], sy = s_p[3 * q + 1], b = s_p[3 * q + 2];
      const T sbx = IMG == 2 ? s_b[2 * q] : T(0), sby = IMG == 2 ? s_b[2 * q + 1] : T(0);
#pragma unroll
      for (int k = 0; k < VTT; ++k) {
        const T dx = pd<T, IMG>(px[k], sx, bx[k], sbx, g.Lx, g.iLx);
        const T dy = pd<T, IMG>(py[k], sy, by[k], sby, g.Ly, g.iLy);
        const T s = inv_r2<T>(dx * dx + dy * dy, g.tiny);
        const T bs = b * s;
        ax[k] += bs * dy;
        ay[k] -= bs * dx;
      }
    }
  }
#pragma unroll
  for (int k = 0; k < VTT; ++k) {
    const int t = blockIdx.x * VT * VTT + k * VT + tid;
    if (t < n) {
      part[2 * ((int64_t)ch * n + t)] = ax[k];
      part[2 * ((int64_t)ch * n + t) + 1] = ay[k];
    }
  }
}

// near term Φ_ij = c Kε(r) − f_i a_j / r² and dΦ/dr
template <typename T>
__device__ __forceinline__ void phi(const Geo<T>& g, T r2, T fa, T& F, T& dF) {
  const T rn = sqrt(r2);
  T K, dK;
  keps<T>(g, rn, K, dK);
  const T s = inv_r2<T>(r2, g.tiny);
  F = g.c * K - fa * s;
  dF = rn > T(0) ? g.c * dK + T(2) * fa * s / rn : T(0);
}

template <typename T, int IMG>
__global__ void k_vel_fin(Geo<T> g, dv_vpm_plan p, const T* __restrict__ x, const T* __restrict__ xb,
                          const T* __restrict__ wt, const T* __restrict__ part, int nch, T* __restrict__ u) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.n) return;
  T fx = T(0), fy = T(0);
  for (int c = 0; c < nch; ++c) {
    fx += part[2 * ((int64_t)c * p.n + i)];
    fy += part[2 * ((int64_t)c * p.n + i) + 1];
  }
  const T fi = (T)p.f[i];
  T ux = fi * fx, uy = fi * fy;
  const int k1 = p.nbr_off[i + 1];
  for (int k = p.nbr_off[i]; k < k1; ++k) {
    const int j = p.nbr[k];
    const P2<T> r = rel<T, IMG>(g, x, xb, i, j);
    T F, dF;
    phi<T>(g, r.x * r.x + r.y * r.y, fi * (T)p.slot_a[j], F, dF);
    const T fw = F * wt[j];
    ux += fw * r.y;
    uy -= fw * r.x;
  }
  u[2 * i] = ux;
  u[2 * i + 1] = uy;
}

template <typename T>
__device__ __forceinline__ T warp_allsum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// far-field VJP.  For ĝ_i = f_i ∂L/∂u_i, s = 1/r², c = ĝ·r⊥:
//   ∂L/∂x_i (target) = Σ_s b_s [s (−ĝ_y, ĝ_x) − 2 s² c r]
//   ∂L/∂b_s          = Σ_i s c
//   ∂L/∂x_s (source) = −b_s Σ_i [s (−ĝ_y, ĝ_x) − 2 s² c r]
template <typename T, int IMG>
__global__ void __launch_bounds__(VT) k_far_bwd(Geo<T> g, dv_vpm_plan p, const T* __restrict__ x,
                                                const T* __restrict__ xb, const T* __restrict__ sp,
                                                const T* __restrict__ spb, const T* __restrict__ gu, int chunk,
                                                T* __restrict__ tpart, T* __restrict__ spart) {
  __shared__ T s_p[VTS * 3];
  __shared__ T s_b[IMG == 2 ? VTS * 2 : 2];
  __shared__ T s_r[(VT / 32) * VTS * 5];
  const int n = p.n, ns = *p.n_src;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, ch = blockIdx.y;
  const int s0 = ch * chunk, s1 = min(ns, s0 + chunk);
  T px[VTT], py[VTT], bx[VTT], by[VTT], gx[VTT], gy[VTT], aP[VTT], aQx[VTT], aQy[VTT];
#pragma unroll
  for (int k = 0; k < VTT; ++k) {
    const int t = blockIdx.x * VT * VTT + k * VT + tid;
    const bool ok = t < n;
    px[k] = ok ? x[2 * t] : T(0);
    py[k] = ok ? x[2 * t + 1] : T(0);
    bx[k] = (IMG == 2 && ok) ? xb[2 * t] : T(0);
    by[k] = (IMG == 2 && ok) ? xb[2 * t + 1] : T(0);
    const T f = ok ? (T)p.f[t] : T(0);
    gx[k] = ok ? f * gu[2 * t] : T(0);
    gy[k] = ok ? f * gu[2 * t + 1] : T(0);
    aP[k] = aQx[k] = aQy[k] = T(0);
  }
  for (int base = s0; base < s1; base += VTS) {
    const int cnt = min(VTS, s1 - base);
    __syncthreads();
    if (tid < cnt) {
      s_p[3 * tid] = sp[3 * (base + tid)];
      s_p[3 * tid + 1] = sp[3 * (base + tid) + 1];
      s_p[3 * tid + 2] = sp[3 * (base + tid) + 2];
      if (IMG == 2) {
        s_b[2 * tid] = spb[2 * (base + tid)];
        s_b[2 * tid + 1] = spb[2 * (base + tid) + 1];
      }
    }
    __syncthreads();
#pragma unroll 2
    for (int q = 0; q < cnt; ++q) {
      const T sx = s_p[3 * q], sy = s_p[3 * q + 1], b = s_p[3 * q + 2];
      const T sbx = IMG == 2 ? s_b[2 * q] : T(0), sby = IMG == 2 ? s_b[2 * q + 1] : T(0);
      T bw = T(0), bgx = T(0), bgy = T(0), cx = T(0), cy = T(0);
#pragma unroll
      for (int k = 0; k < VTT; ++k) {
        const T dx = pd<T, IMG>(px[k], sx, bx[k], sbx, g.Lx, g.iLx);
        const T dy = pd<T, IMG>(py[k], sy, by[k], sby, g.Ly, g.iLy);
        const T s = inv_r2<T>(dx * dx + dy * dy, g.tiny);
        const T c = gx[k] * dy - gy[k] * dx;
        const T sc = s * c;
        const T u = s * sc;
        aP[k] += b * s;
        const T bu = b * u;
        aQx[k] += bu * dx;
        aQy[k] += bu * dy;
        bw += sc;
        bgx += s * gx[k];
        bgy += s * gy[k];
        cx += u * dx;
        cy += u * dy;
      }
      bw = warp_allsum(bw);
      bgx = warp_allsum(bgx);
      bgy = warp_allsum(bgy);
      cx = warp_allsum(cx);
      cy = warp_allsum(cy);
      if (lane == 0) {
        T* r = s_r + ((int64_t)warp * VTS + q) * 5;
        r[0] = bw;
        r[1] = bgx;
        r[2] = bgy;
        r[3] = cx;
        r[4] = cy;
      }
    }
    __syncthreads();
    for (int q = tid; q < cnt; q += VT) {
      T acc[5] = {T(0), T(0), T(0), T(0), T(0)};
      for (int w = 0; w < VT / 32; ++w)
#pragma unroll
        for (int e = 0; e < 5; ++e) acc[e] += s_r[((int64_t)w * VTS + q) * 5 + e];
      T* o = spart + ((int64_t)blockIdx.x * p.src_cap + base + q) * 5;
#pragma unroll
      for (int e = 0; e < 5; ++e) o[e] = acc[e];
    }
  }
#pragma unroll
  for (int k = 0; k < VTT; ++k) {
    const int t = blockIdx.x * VT * VTT + k * VT + tid;
    if (t < n) {
      T* o = tpart + 3 * ((int64_t)ch * n + t);
      o[0] = aP[k];
      o[1] = aQx[k];
      o[2] = aQy[k];
    }
  }
}

template <typename T>
__global__ void k_src_fin(dv_vpm_plan p, const T* __restrict__ sp, const T* __restrict__ spart, int ntb,
                          T* __restrict__ sg) {
  const int ns = *p.n_src;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  T a[5] = {T(0), T(0), T(0), T(0), T(0)};
  for (int b = 0; b < ntb; ++b)
#pragma unroll
    for (int e = 0; e < 5; ++e) a[e] += spart[((int64_t)b * p.src_cap + s) * 5 + e];
  const T bs = sp[3 * s + 2];
  // −b_s [(−Σ s ĝ_y, Σ s ĝ_x) − 2 Σ s² c r]
  sg[3 * s] = bs * (a[2] + T(2) * a[3]);
  sg[3 * s + 1] = bs * (T(2) * a[4] - a[1]);
  sg[3 * s + 2] = (T)p.src_a[s] * a[0];
}

template <typename T, int IMG>
__global__ void k_vel_bwd_fin(Geo<T> g, dv_vpm_plan p, const T* __restrict__ x, const T* __restrict__ xb,
                              const T* __restrict__ wt, const T* __restrict__ gu, const T* __restrict__ tpart,
                              int nch, const T* __restrict__ sg, T* __restrict__ gwt, T* __restrict__ gxo) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= p.n) return;
  const T fk = (T)p.f[k];
  const P2<T> gk{gu[2 * k], gu[2 * k + 1]};
  T P = T(0), Qx = T(0), Qy = T(0);
  for (int c = 0; c < nch; ++c) {
    const T* t = tpart + 3 * ((int64_t)c * p.n + k);
    P += t[0];
    Qx += t[1];
    Qy += t[2];
  }
  const T hx = fk * gk.x, hy = fk * gk.y;
  T ox = -hy * P - T(2) * Qx, oy = hx * P - T(2) * Qy;
  T ow = T(0);
  const int ss = p.slot_src[k];
  if (ss >= 0) {
    ox += sg[3 * ss];
    oy += sg[3 * ss + 1];
    ow += sg[3 * ss + 2];
  }
  const T ak = (T)p.slot_a[k], wk = wt[k];
  const int k1 = p.nbr_off[k + 1];
  for (int e = p.nbr_off[k]; e < k1; ++e) {
    const int j = p.nbr[e];
    const P2<T> r = rel<T, IMG>(g, x, xb, k, j);  // r = x_k − x_j
    const T r2 = r.x * r.x + r.y * r.y;
    const T rn = sqrt(r2);
    if (!(rn > T(0))) continue;
    const T irn = T(1) / rn;
    const T hxr = r.x * irn, hyr = r.y * irn;
    T Fkj, dFkj, Fjk, dFjk;
    phi<T>(g, r2, fk * (T)p.slot_a[j], Fkj, dFkj);
    phi<T>(g, r2, (T)p.f[j] * ak, Fjk, dFjk);
    const T wj = wt[j];
    const P2<T> gj{gu[2 * j], gu[2 * j + 1]};
    // k as target, j as source: + ω̃_j J(r_kj)^T g_k
    const T ck = gk.x * r.y - gk.y * r.x;
    ox += wj * (dFkj * ck * hxr - Fkj * gk.y);
    oy += wj * (dFkj * ck * hyr + Fkj * gk.x);
    // j as target, k as source: − ω̃_k J(r_jk)^T g_j, r_jk = −r
    const T cj = gj.x * r.y - gj.y * r.x;
    ox -= wk * (dFjk * cj * hxr - Fjk * gj.y);
    oy -= wk * (dFjk * cj * hyr + Fjk * gj.x);
    ow -= Fjk * cj;
  }
  gwt[k] = ow;
  gxo[2 * k] = ox;
  gxo[2 * k + 1] = oy;
}

// ------------------------------------------------------------ plan build
__global__ void k_plan_mult(const dv_solver_fields S, const dv_counters* __restrict__ C, int n,
                            int32_t* __restrict__ mult) {
  const int M = C->num_samples;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < M; s += gridDim.x * blockDim.x) {
    const int j = S.sample_idx[s];
    if (j >= 0 && j < n) atomicAdd(mult + j, 1);
  }
}

__global__ void k_plan_slots(dv_params P, DevGrid G, dv_fields F, dv_solver_fields S,
                             const dv_counters* __restrict__ C, const uint32_t* __restrict__ perm_src,
                             const int32_t* __restrict__ mult, int mode, dv_vpm_plan p,
                             uint32_t* __restrict__ flags, int32_t* __restrict__ err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = p.n;
  if (i == 0) {
    int bad = 0;
    if (C->n != n || C->n_fluid != n) bad |= 1;
    if (!G.nok || !*G.nok) bad |= 2;
    if (bad == 0 && (int64_t)G.noff[n] > p.nbr_cap) bad |= 4;
    *err = bad;
    flags[n] = 0;
    p.nbr_off[n] = bad ? 0 : (int32_t)G.noff[n];
  }
  if (i >= n) return;
  const int32_t o = (int32_t)perm_src[i];
  p.perm[i] = o;
  if (o >= 0 && o < n) p.inv_perm[o] = i;
  p.m_V[i] = F.m_V[i];
  const bool listed = G.nok && *G.nok && (int64_t)G.noff[n] <= p.nbr_cap;
  const uint32_t k0 = listed ? G.noff[i] : 0, k1 = listed ? G.noff[i + 1] : 0;
  p.nbr_off[i] = (int32_t)k0;
  float Si = S.kden[i];
  int near = mult[i];
  for (uint32_t k = k0; k < k1; ++k) {
    const int j = nbr_slot((uint32_t)G.nidx[k]);
    p.nbr[k] = j;
    if (F.material[j] == DV_MATERIAL_FLUID) Si += S.kden[j];
    near += mult[j];
  }
  if (mode == DV_VPM_FULL) {
    p.slot_a[i] = 1.0f;
    p.f[i] = P.vvpe_coef;
    flags[i] = 1;
  } else {
    const int m = mult[i];
    p.slot_a[i] = m > 0 ? (float)m / (S.kden[i] + P.kden_eps) : 0.0f;
    const int cnt = C->num_samples - near;
    const float fac = C->kden_sum_f32 - Si;
    p.f[i] = cnt > 0 ? fac * (P.vvpe_coef / (float)cnt) : 0.0f;
    flags[i] = m > 0 ? 1u : 0u;
  }
}

__global__ void k_plan_src(dv_vpm_plan p, const uint32_t* __restrict__ flags, const uint32_t* __restrict__ offs,
                           const int32_t* __restrict__ err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = p.n;
  if (i == 0) *p.n_src = (*err || (int64_t)offs[n] > p.src_cap) ? -1 : (int32_t)offs[n];
  if (i >= n) return;
  if (flags[i] && (int64_t)offs[i] < p.src_cap) {
    const int s = (int)offs[i];
    p.src[s] = i;
    p.src_a[s] = p.slot_a[i];
    p.slot_src[i] = s;
  } else {
    p.slot_src[i] = -1;
  }
}

// ------------------------------------------------------------ dispatch
int check_plan(dv_ctx* c, const dv_vpm_plan* p, int prec) {
  if (!c || !p) return DV_EINVAL;
  if (c->p.dim != 2) return dv_fail(c, DV_EUNSUPPORTED, "the differentiable step is 2-D only");
  if (prec != 32 && prec != 64) return dv_fail(c, DV_EINVAL, "precision must be 32 or 64");
  if (p->n < 0 || p->n > c->cap || p->src_cap < 0)
    return dv_fail(c, DV_EINVAL, "plan size out of range (n %d, capacity %lld)", p->n, (long long)c->cap);
  if (!p->n_src || !p->nbr_off || !p->nbr || !p->src || !p->src_a || !p->slot_src || !p->slot_a || !p->f ||
      !p->m_V)
    return dv_fail(c, DV_EINVAL, "a plan pointer is NULL");
  return DV_OK;
}

inline int img_mode(const dv_ctx* c, const dv_vpm_plan* p) {
  return c->p.periodic ? (p->xbar ? 2 : 1) : 0;
}

#define DV_IMG_DISPATCH(img, KERNEL_CALL) \
  do {                                    \
    if ((img) == 0) {                     \
      constexpr int IMG = 0;              \
      KERNEL_CALL;                        \
    } else if ((img) == 1) {              \
      constexpr int IMG = 1;              \
      KERNEL_CALL;                        \
    } else {                              \
      constexpr int IMG = 2;              \
      KERNEL_CALL;                        \
    }                                     \
  } while (0)

template <typename T>
int smooth_t(dv_ctx* c, const dv_vpm_plan* p, const void* x, const void* w, void* ws) {
  const Geo<T> g = make_geo<T>(c->p);
  const T* xb = (const T*)p->xbar;
  const int nb = dv_blocks(p->n);
  DV_IMG_DISPATCH(img_mode(c, p), (k_smooth<T, IMG><<<nb, DV_THREADS, 0, c->stream>>>(
                                       g, *p, (const T*)x, xb, (const T*)w, (T*)ws)));
  DV_LAUNCHED(c);
  return DV_OK;
}

template <typename T>
int smooth_bwd_t(dv_ctx* c, const dv_vpm_plan* p, const void* x, const void* w, const void* gs, void* gw,
                 void* gx) {
  const Geo<T> g = make_geo<T>(c->p);
  const T* xb = (const T*)p->xbar;
  const int nb = dv_blocks(p->n);
  DV_IMG_DISPATCH(img_mode(c, p), (k_smooth_bwd<T, IMG><<<nb, DV_THREADS, 0, c->stream>>>(
                                       g, *p, (const T*)x, xb, (const T*)w, (const T*)gs, (T*)gw, (T*)gx)));
  DV_LAUNCHED(c);
  return DV_OK;
}

template <typename T>
int curl_t(dv_ctx* c, const dv_vpm_plan* p, const void* x, const void* v, void* w) {
  const Geo<T> g = make_geo<T>(c->p);
  const T* xb = (const T*)p->xbar;
  DV_IMG_DISPATCH(img_mode(c, p), (k_curl<T, IMG><<<dv_blocks(p->n), DV_THREADS, 0, c->stream>>>(
                                       g, *p, (const T*)x, xb, (const T*)v, (T*)w)));
  DV_LAUNCHED(c);
  return DV_OK;
}

template <typename T>
int curl_bwd_t(dv_ctx* c, const dv_vpm_plan* p, const void* x, const void* v, const void* gw, void* gv, void* gx) {
  const Geo<T> g = make_geo<T>(c->p);
  const T* xb = (const T*)p->xbar;
  DV_IMG_DISPATCH(img_mode(c, p), (k_curl_bwd<T, IMG><<<dv_blocks(p->n), DV_THREADS, 0, c->stream>>>(
                                       g, *p, (const T*)x, xb, (const T*)v, (const T*)gw, (T*)gv, (T*)gx)));
  DV_LAUNCHED(c);
  return DV_OK;
}

template <typename T>
int velocity_t(dv_ctx* c, const dv_vpm_plan* p, const void* x, const void* wt, void* u, void* ws,
               int64_t ws_bytes) {
  const Layout L = layout<T>(p->n, p->src_cap, c->num_sms);
  if (!ws || ws_bytes < L.total)
    return dv_fail(c, DV_EINVAL, "workspace of %lld bytes, need %lld", (long long)ws_bytes, (long long)L.total);
  char* base = (char*)ws;
  T* sp = (T*)(base + L.sp);
  T* spb = (T*)(base + L.spb);
  T* part = (T*)(base + L.part);
  const Geo<T> g = make_geo<T>(c->p);
  const T* xb = (const T*)p->xbar;
  const int img = img_mode(c, p);
  if (p->src_cap > 0) {
    k_pack<T><<<dv_blocks(p->src_cap), DV_THREADS, 0, c->stream>>>(*p, (const T*)x, xb, (const T*)wt, sp, spb);
    DV_LAUNCHED(c);
  }
  if (p->n > 0) {
    const dim3 grid(L.ntb, L.nch);
    DV_IMG_DISPATCH(img, (k_far<T, IMG><<<grid, VT, 0, c->stream>>>(g, *p, (const T*)x, xb, sp, spb, L.chunk,
                                                                     part)));
    DV_LAUNCHED(c);
    DV_IMG_DISPATCH(img, (k_vel_fin<T, IMG><<<dv_blocks(p->n), DV_THREADS, 0, c->stream>>>(
                             g, *p, (const T*)x, xb, (const T*)wt, part, L.nch, (T*)u)));
    DV_LAUNCHED(c);
  }
  return DV_OK;
}

template <typename T>
int velocity_bwd_t(dv_ctx* c, const dv_vpm_plan* p, const void* x, const void* wt, const void* gu, void* gwt,
                   void* gx, void* ws, int64_t ws_bytes) {
  const Layout L = layout<T>(p->n, p->src_cap, c->num_sms);
  if (!ws || ws_bytes < L.total)
    return dv_fail(c, DV_EINVAL, "workspace of %lld bytes, need %lld", (long long)ws_bytes, (long long)L.total);
  char* base = (char*)ws;
  T* sp = (T*)(base + L.sp);
  T* spb = (T*)(base + L.spb);
  T* tpart = (T*)(base + L.tpart);
  T* spart = (T*)(base + L.spart);
  T* sg = (T*)(base + L.sg);
  const Geo<T> g = make_geo<T>(c->p);
  const T* xb = (const T*)p->xbar;
  const int img = img_mode(c, p);
  if (p->n == 0) return DV_OK;
  if (p->src_cap > 0) {
    k_pack<T><<<dv_blocks(p->src_cap), DV_THREADS, 0, c->stream>>>(*p, (const T*)x, xb, (const T*)wt, sp, spb);
    DV_LAUNCHED(c);
  }
  const dim3 grid(L.ntb, L.nch);
  DV_IMG_DISPATCH(img, (k_far_bwd<T, IMG><<<grid, VT, 0, c->stream>>>(g, *p, (const T*)x, xb, sp, spb,
                                                                       (const T*)gu, L.chunk, tpart, spart)));
  DV_LAUNCHED(c);
  if (p->src_cap > 0) {
    k_src_fin<T><<<dv_blocks(p->src_cap), DV_THREADS, 0, c->stream>>>(*p, sp, spart, L.ntb, sg);
    DV_LAUNCHED(c);
  }
  DV_IMG_DISPATCH(img, (k_vel_bwd_fin<T, IMG><<<dv_blocks(p->n), DV_THREADS, 0, c->stream>>>(
                           g, *p, (const T*)x, xb, (const T*)wt, (const T*)gu, tpart, L.nch, sg, (T*)gwt,
                           (T*)gx)));
  DV_LAUNCHED(c);
  return DV_OK;
}

}  // namespace

DV_API int64_t dv_vpm_workspace_bytes(dv_ctx* c, int32_t n, int32_t src_cap, int32_t precision) {
  if (!c || n < 0 || src_cap < 0 || (precision != 32 && precision != 64)) return DV_EINVAL;
  return precision == 64 ? layout<double>(n, src_cap, c->num_sms).total
                         : layout<float>(n, src_cap, c->num_sms).total;
}

DV_API int dv_vpm_plan_build(dv_ctx* c, const dv_fields* f, const dv_solver_fields* s, int32_t mode,
                             dv_vpm_plan* p) {
  if (!c || !f || !s || !p) return DV_EINVAL;
  if (mode != DV_VPM_MC && mode != DV_VPM_FULL) return dv_fail(c, DV_EINVAL, "unknown plan mode %d", mode);
  if (!p->perm || !p->inv_perm) return dv_fail(c, DV_EINVAL, "a plan pointer is NULL");
  if (int rc = check_plan(c, p, 32)) return rc;
  if (mode == DV_VPM_FULL && p->src_cap < p->n)
    return dv_fail(c, DV_EINVAL, "a full plan needs src_cap >= n (%d < %d)", p->src_cap, p->n);
  const int n = p->n;
  DV_CK(c, cudaMemsetAsync(c->mult, 0, sizeof(int32_t) * std::max(n, 1), c->stream));
  if (mode == DV_VPM_MC) {
    k_plan_mult<<<2 * c->num_sms, DV_THREADS, 0, c->stream>>>(*s, c->d_cnt, n, c->mult);
    DV_LAUNCHED(c);
  }
  k_plan_slots<<<dv_blocks(n + 1), DV_THREADS, 0, c->stream>>>(c->p, dv_grid(c), *f, *s, c->d_cnt,
                                                                c->vals[c->perm_buf], c->mult, mode, *p,
                                                                c->flags, c->d_flag + 1);
  DV_LAUNCHED(c);
  if (int rc = dv_scan_u32(c, c->flags, c->offs, (int64_t)n + 1)) return rc;
  k_plan_src<<<dv_blocks(n + 1), DV_THREADS, 0, c->stream>>>(*p, c->flags, c->offs, c->d_flag + 1);
  DV_LAUNCHED(c);
  return DV_OK;
}

DV_API int dv_vpm_smooth(dv_ctx* c, const dv_vpm_plan* p, int32_t precision, const void* x, const void* w,
                         void* w_s) {
  if (int rc = check_plan(c, p, precision)) return rc;
  if (!x || !w || !w_s) return dv_fail(c, DV_EINVAL, "a tensor pointer is NULL");
  return precision == 64 ? smooth_t<double>(c, p, x, w, w_s) : smooth_t<float>(c, p, x, w, w_s);
}

DV_API int dv_vpm_smooth_bwd(dv_ctx* c, const dv_vpm_plan* p, int32_t precision, const void* x, const void* w,
                             const void* g_ws, void* g_w, void* g_x) {
  if (int rc = check_plan(c, p, precision)) return rc;
  if (!x || !w || !g_ws || !g_w || !g_x) return dv_fail(c, DV_EINVAL, "a tensor pointer is NULL");
  return precision == 64 ? smooth_bwd_t<double>(c, p, x, w, g_ws, g_w, g_x)
                         : smooth_bwd_t<float>(c, p, x, w, g_ws, g_w, g_x);
}

DV_API int dv_vpm_velocity(dv_ctx* c, const dv_vpm_plan* p, int32_t precision, const void* x, const void* w_s,
                           void* u, void* ws, int64_t ws_bytes) {
  if (int rc = check_plan(c, p, precision)) return rc;
  if (!x || !w_s || !u) return dv_fail(c, DV_EINVAL, "a tensor pointer is NULL");
  return precision == 64 ? velocity_t<double>(c, p, x, w_s, u, ws, ws_bytes)
                         : velocity_t<float>(c, p, x, w_s, u, ws, ws_bytes);
}

DV_API int dv_vpm_velocity_bwd(dv_ctx* c, const dv_vpm_plan* p, int32_t precision, const void* x,
                               const void* w_s, const void* g_u, void* g_ws, void* g_x, void* ws,
                               int64_t ws_bytes) {
  if (int rc = check_plan(c, p, precision)) return rc;
  if (!x || !w_s || !g_u || !g_ws || !g_x) return dv_fail(c, DV_EINVAL, "a tensor pointer is NULL");
  return precision == 64 ? velocity_bwd_t<double>(c, p, x, w_s, g_u, g_ws, g_x, ws, ws_bytes)
                         : velocity_bwd_t<float>(c, p, x, w_s, g_u, g_ws, g_x, ws, ws_bytes);
}

DV_API int dv_vpm_curl(dv_ctx* c, const dv_vpm_plan* p, int32_t precision, const void* x, const void* v, void* w) {
  if (int rc = check_plan(c, p, precision)) return rc;
  if (!x || !v || !w) return dv_fail(c, DV_EINVAL, "a tensor pointer is NULL");
  return precision == 64 ? curl_t<double>(c, p, x, v, w) : curl_t<float>(c, p, x, v, w);
}

DV_API int dv_vpm_curl_bwd(dv_ctx* c, const dv_vpm_plan* p, int32_t precision, const void* x, const void* v,
                           const void* g_w, void* g_v, void* g_x) {
  if (int rc = check_plan(c, p, precision)) return rc;
  if (!x || !v || !g_w || !g_v || !g_x) return dv_fail(c, DV_EINVAL, "a tensor pointer is NULL");
  return precision == 64 ? curl_bwd_t<double>(c, p, x, v, g_w, g_v, g_x)
                         : curl_bwd_t<float>(c, p, x, v, g_w, g_v, g_x);
}
