// Context lifetime, error reporting, counters and the generic scan /
// reduction helpers of libdimcv.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <algorithm>

#include "dv_internal.cuh"

static thread_local std::string g_create_error;

int dv_fail(dv_ctx* c, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (c)
    c->err = buf;
  else
    g_create_error = buf;
  return code;
}

int dv_cuda_check(dv_ctx* c, cudaError_t e, const char* what) {
  return dv_fail(c, DV_ECUDA, "%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
}

DV_API const char* dv_version(void) { return "dimcv-b200 0.1 (sm_100a)"; }

DV_API const char* dv_last_error(const dv_ctx* ctx) {
  return ctx ? ctx->err.c_str() : g_create_error.c_str();
}

DV_API int64_t dv_launch_count(const dv_ctx* ctx) { return ctx ? ctx->launches : 0; }

DV_API int dv_set_stream(dv_ctx* ctx, void* stream) {
  if (!ctx) return DV_EINVAL;
  ctx->stream = (cudaStream_t)stream;
  return DV_OK;
}

DV_API int dv_set_params(dv_ctx* ctx, const dv_params* params) {
  if (!ctx || !params) return DV_EINVAL;
  if (params->dim != ctx->p.dim || params->grid_num[0] != ctx->p.grid_num[0] ||
      params->grid_num[1] != ctx->p.grid_num[1] || params->grid_num[2] != ctx->p.grid_num[2])
    return dv_fail(ctx, DV_EINVAL, "dv_set_params: dim and grid_num must not change");
  ctx->p = *params;
  return DV_OK;
}

// Builds the per-axis Morton tables: T_d[c] is the key contribution of cell
// coordinate c on axis d; key = T_0[cx] | T_1[cy] | T_2[cz].  Bits are
// interleaved level by level (z lowest), axes with fewer bits drop out, so the
// key space is the product of the per-axis power-of-two paddings.
static int build_morton(dv_ctx* c) {
  const dv_params& P = c->p;
  int bits[3] = {0, 0, 0};
  for (int d = 0; d < P.dim; ++d) {
    int g = P.grid_num[d];
    if (g < 1 || g > (1 << 20)) return dv_fail(c, DV_EINVAL, "grid_num[%d]=%d out of range", d, g);
    while ((1 << bits[d]) < g) ++bits[d];
  }
  int total = bits[0] + bits[1] + bits[2];
  if (total > 26)
    return dv_fail(c, DV_EUNSUPPORTED, "cell grid needs %d Morton bits (max 26): domain/h too large",
                   total);
  int pos[3][21];
  int next = 0;
  int maxb = bits[0] > bits[1] ? bits[0] : bits[1];
  if (bits[2] > maxb) maxb = bits[2];
  for (int l = 0; l < maxb; ++l)
    for (int d = P.dim - 1; d >= 0; --d)
      if (l < bits[d]) pos[d][l] = next++;
  c->ncells = (int64_t)1 << total;
  c->kbits = total + 1;
  if (P.n_scenes > 1) {  // scene id above the Morton bits
    int sbits = 0;
    while ((1 << sbits) < P.n_scenes) ++sbits;
    if (total + sbits > 30)
      return dv_fail(c, DV_EUNSUPPORTED, "scene batch needs %d key bits (max 30)", total + sbits);
    c->scene_shift = total;
    c->ncells = (int64_t)1 << (total + sbits);
    c->kbits = total + sbits + 1;
  }
  c->npasses = (c->kbits + 7) / 8;
  for (int d = 0; d < 3; ++d) {
    int g = d < P.dim ? P.grid_num[d] : 1;
    uint32_t* h = (uint32_t*)malloc(sizeof(uint32_t) * g);
    for (int v = 0; v < g; ++v) {
      uint32_t k = 0;
      if (d < P.dim)
        for (int l = 0; l < bits[d]; ++l)
          if ((v >> l) & 1) k |= 1u << pos[d][l];
      h[v] = k;
    }
    cudaError_t e = cudaMalloc(&c->mt[d], sizeof(uint32_t) * g);
    if (e == cudaSuccess) e = cudaMemcpy(c->mt[d], h, sizeof(uint32_t) * g, cudaMemcpyHostToDevice);
    free(h);
    if (e != cudaSuccess) return dv_cuda_check(c, e, "morton table");
  }
  return DV_OK;
}

template <typename T>
static cudaError_t alloc(T** p, int64_t count) {
  return cudaMalloc((void**)p, sizeof(T) * (size_t)(count < 1 ? 1 : count));
}

DV_API void dv_destroy(dv_ctx* c) {
  if (!c) return;
  dv_batch_free(c);
  void* ptrs[] = {c->d_cnt,   c->d_flag,    c->keys[0],   c->keys[1],   c->vals[0], c->vals[1],
                  c->hist,    c->cell_start, c->cell_end, c->mt[0],     c->mt[1],   c->mt[2],
                  c->scan_part, c->dscan_part, c->red_part, c->ired_part, c->flags, c->offs,
                  c->targets, c->cdf,       c->spos,      c->sw,        c->near_v,  c->near_S,
                  c->far_acc, c->mult,      c->nbr_off,   c->nbr_idx,   c->d_nbr_ok,
                  c->nbr_rows, c->sflag,   c->srank,     c->sslot};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (int k = 0; k < 2 * dv_ctx::kProfPool; ++k)
    if (c->prof_ev[k]) cudaEventDestroy(c->prof_ev[k]);
  if (c->d_prof) cudaFree(c->d_prof);
  if (c->h_cnt) cudaFreeHost(c->h_cnt);
  if (c->h_flag) cudaFreeHost(c->h_flag);
  delete c;
}

DV_API dv_ctx* dv_create(const dv_params* params, int64_t capacity, void* stream) {
  if (!params) {
    dv_fail(nullptr, DV_EINVAL, "params is NULL");
    return nullptr;
  }
  if (params->dim != 2 && params->dim != 3) {
    dv_fail(nullptr, DV_EINVAL, "dim must be 2 or 3 (got %d)", params->dim);
    return nullptr;
  }
  if (capacity < 1 || capacity > (int64_t)1 << 30) {
    dv_fail(nullptr, DV_EINVAL, "capacity %lld out of range [1, 2^30]", (long long)capacity);
    return nullptr;
  }
  if (params->periodic) {
    if (!params->cell_origin_offset) {
      dv_fail(nullptr, DV_EINVAL, "periodic boxes need cell_origin_offset = 1");
      return nullptr;
    }
    for (int d = 0; d < params->dim; ++d) {
      const double cells = (double)params->box[d] / (double)params->grid_size;
      if (params->grid_num[d] < 5 || fabs(cells - params->grid_num[d]) > 1e-4 * params->grid_num[d] ||
          params->grid_size < params->support_radius) {
        dv_fail(nullptr, DV_EINVAL,
                "periodic axis %d: need >= 5 cells of size box/grid_num >= h (box %g, grid_size %g, %d cells)", d,
                (double)params->box[d], (double)params->grid_size, params->grid_num[d]);
        return nullptr;
      }
    }
  }
  dv_ctx* c = new dv_ctx();
  c->p = *params;
  c->cap = capacity;
  c->stream = (cudaStream_t)stream;
  cudaGetDevice(&c->device);
  cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device);
  int rc = build_morton(c);
  if (rc != DV_OK) {
    g_create_error = c->err;
    dv_destroy(c);
    return nullptr;
  }
  const int64_t cap = capacity;
  c->max_tiles = (cap + 2047) / 2048 + 1;
  c->red_cap = (cap + 127) / 128 + 1024;
  c->scan_part_cap = (std::max<int64_t>(cap + 1, 256 * c->max_tiles) + 4095) / 4096 + 1024;
  cudaError_t e = cudaSuccess;
#define A(ptr, cnt) \
  if (e == cudaSuccess) e = alloc(&(ptr), (cnt));
  A(c->d_cnt, 1);
  A(c->d_flag, 4);
  A(c->keys[0], cap);
  A(c->keys[1], cap);
  A(c->vals[0], cap);
  A(c->vals[1], cap);
  A(c->hist, 256 * c->max_tiles);
  A(c->cell_start, c->ncells);
  A(c->cell_end, c->ncells);
  A(c->scan_part, c->scan_part_cap);
  A(c->dscan_part, c->scan_part_cap);
  A(c->red_part, c->red_cap);
  A(c->ired_part, c->red_cap);
  A(c->flags, cap + 1);
  A(c->offs, cap + 1);
  A(c->targets, cap);
  A(c->cdf, cap);
  A(c->spos, cap);
  A(c->sw, cap);
  A(c->near_v, cap);
  A(c->near_S, cap);
  A(c->far_acc, cap * DV_MAX_FAR_CHUNKS);
  A(c->mult, cap);
  A(c->sflag, cap + 1);
  A(c->srank, cap + 1);
  A(c->sslot, cap);
  // neighbour lists: 48 (3-D) / 24 (2-D) entries per particle on average,
  // beyond which the sweeps keep scanning cells
  c->nbr_cap = cap * (params->dim == 3 ? 48 : 24);
  A(c->nbr_off, cap + 1);
  A(c->nbr_idx, c->nbr_cap);
  A(c->d_nbr_ok, 2);  // [0]: lists valid, [1]: a material other than fluid / solid seen by the build
  // the 3-D build's first pass stores up to 64 neighbours per particle in
  // fixed rows (a settled lattice has at most 36); 2-D builds have none
  c->nbr_slots = params->dim == 3 ? 64 : 0;
  if (c->nbr_slots) A(c->nbr_rows, cap * c->nbr_slots);
  A(c->d_prof, 4);
#undef A
  if (e == cudaSuccess) e = cudaMallocHost((void**)&c->h_cnt, sizeof(dv_counters));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&c->h_flag, sizeof(int32_t) * 4);
  if (e == cudaSuccess) e = cudaMemset(c->d_cnt, 0, sizeof(dv_counters));
  if (e == cudaSuccess) e = cudaMemset(c->d_flag, 0, sizeof(int32_t) * 4);
  if (e == cudaSuccess) e = cudaMemset(c->d_prof, 0, sizeof(double) * 4);
  if (e == cudaSuccess) e = cudaMemset(c->d_nbr_ok, 0, 2 * sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMemset(c->cell_start, 0, sizeof(int32_t) * c->ncells);
  if (e == cudaSuccess) e = cudaMemset(c->cell_end, 0, sizeof(int32_t) * c->ncells);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    dv_cuda_check(c, e, "dv_create allocation");
    g_create_error = c->err;
    dv_destroy(c);
    return nullptr;
  }
  return c;
}

DV_API int dv_get_counters(dv_ctx* c, dv_counters* out) {
  if (!c || !out) return DV_EINVAL;
  DV_CK(c, cudaMemcpyAsync(c->h_cnt, c->d_cnt, sizeof(dv_counters), cudaMemcpyDeviceToHost, c->stream));
  DV_CK(c, cudaStreamSynchronize(c->stream));
  *out = *c->h_cnt;
  c->n_upper = c->batch ? c->cap : out->n;  // a scene batch keeps capacity-sized launch shapes
  return DV_OK;
}

__global__ void k_set_counts(dv_counters* C, int n, int nf, int ns) {
  C->n = n;
  C->n_fluid = nf;
  C->n_solid = ns;
}

DV_API int dv_set_counts(dv_ctx* c, int32_t n, int32_t n_fluid, int32_t n_solid) {
  if (!c) return DV_EINVAL;
  if (n < 0 || n > c->cap || n_fluid < 0 || n_solid < 0 || n_fluid + n_solid != n)
    return dv_fail(c, DV_EINVAL, "dv_set_counts: inconsistent counts n=%d fluid=%d solid=%d cap=%lld",
                   n, n_fluid, n_solid, (long long)c->cap);
  k_set_counts<<<1, 1, 0, c->stream>>>(c->d_cnt, n, n_fluid, n_solid);
  DV_LAUNCHED(c);
  c->n_upper = c->batch ? c->cap : n;
  return dv_invalidate_lists(c);
}

__global__ void k_clear_status(dv_counters* C) { C->status = 0; }

DV_API int dv_clear_status(dv_ctx* c) {
  if (!c) return DV_EINVAL;
  k_clear_status<<<1, 1, 0, c->stream>>>(c->d_cnt);
  DV_LAUNCHED(c);
  return DV_OK;
}

// ------------------------------------------------------------------- scans
// Block of 512 threads scans 4096 elements (8 per thread, blocked layout).
#define SCAN_T 512
#define SCAN_I 8
#define SCAN_TILE (SCAN_T * SCAN_I)

template <typename T>
__device__ __forceinline__ T block_excl_scan(T v, T* total) {
  // exclusive scan of one value per thread in thread order
  __shared__ T s_w[SCAN_T / 32];
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  T inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) s_w[w] = inc;
  __syncthreads();
  if (w == 0) {
    T x = lane < SCAN_T / 32 ? s_w[lane] : T(0);
    T xi = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      T t = __shfl_up_sync(0xffffffffu, xi, o);
      if (lane >= o) xi += t;
    }
    if (lane < SCAN_T / 32) s_w[lane] = xi - x;  // exclusive warp offsets
    if (lane == SCAN_T / 32 - 1) s_w[SCAN_T / 32 - 1] = xi - x, *total = xi;
  }
  __syncthreads();
  T r = s_w[w] + inc - v;
  __syncthreads();
  return r;
}

template <typename T>
__global__ void k_scan_reduce(const T* __restrict__ in, int64_t m, T* __restrict__ part) {
  int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
  T s = T(0);
  for (int k = 0; k < SCAN_I; ++k) {
    int64_t e = base + (int64_t)threadIdx.x * SCAN_I + k;
    if (e < m) s += in[e];
  }
  // fixed-order block sum
  __shared__ T s_w[SCAN_T / 32];
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) s_w[w] = s;
  __syncthreads();
  if (w == 0) {
    T x = lane < SCAN_T / 32 ? s_w[lane] : T(0);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) part[blockIdx.x] = x;
  }
}

// one block: exclusive scan of the partials in place (chunks of SCAN_T)
template <typename T>
__global__ void k_scan_top(T* part, int nb) {
  __shared__ T s_total;
  T carry = T(0);
  for (int base = 0; base < nb; base += SCAN_T) {
    int e = base + threadIdx.x;
    T v = e < nb ? part[e] : T(0);
    T ex = block_excl_scan<T>(v, &s_total);
    if (e < nb) part[e] = carry + ex;
    __syncthreads();
    carry += s_total;
    __syncthreads();
  }
}

template <typename T>
__global__ void k_scan_down(const T* __restrict__ in, T* __restrict__ out, int64_t m,
                            const T* __restrict__ part) {
  __shared__ T s_total;
  int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_I;
  T loc[SCAN_I];
  T s = T(0);
#pragma unroll
  for (int k = 0; k < SCAN_I; ++k) {
    int64_t e = base + k;
    loc[k] = e < m ? in[e] : T(0);
    s += loc[k];
  }
  T ex = block_excl_scan<T>(s, &s_total) + part[blockIdx.x];
#pragma unroll
  for (int k = 0; k < SCAN_I; ++k) {
    int64_t e = base + k;
    if (e < m) out[e] = ex;
    ex += loc[k];
  }
}

template <typename T>
static int scan_impl(dv_ctx* c, const T* in, T* out, int64_t m, T* part) {
  if (m <= 0) return DV_OK;
  int64_t nb = (m + SCAN_TILE - 1) / SCAN_TILE;
  if (nb > c->scan_part_cap) return dv_fail(c, DV_ECAPACITY, "scan of %lld elements too large", (long long)m);
  k_scan_reduce<T><<<(unsigned)nb, SCAN_T, 0, c->stream>>>(in, m, part);
  DV_LAUNCHED(c);
  k_scan_top<T><<<1, SCAN_T, 0, c->stream>>>(part, (int)nb);
  DV_LAUNCHED(c);
  k_scan_down<T><<<(unsigned)nb, SCAN_T, 0, c->stream>>>(in, out, m, part);
  DV_LAUNCHED(c);
  return DV_OK;
}

int dv_scan_u32(dv_ctx* c, const uint32_t* in, uint32_t* out, int64_t m) {
  return scan_impl<uint32_t>(c, in, out, m, c->scan_part);
}
int dv_scan_f64(dv_ctx* c, const double* in, double* out, int64_t m) {
  return scan_impl<double>(c, in, out, m, c->dscan_part);
}

__global__ void k_finalize_sum(const double* __restrict__ parts, int nparts, double* dst) {
  double s = 0.0;
  // each thread sums a strided subset in index order, then a fixed tree
  for (int k = threadIdx.x; k < nparts; k += blockDim.x) s += parts[k];
  s = block_sum<double>(s);
  if (threadIdx.x == 0) *dst = s;
}

int dv_finalize_sum(dv_ctx* c, const double* parts, int nparts, double* dst) {
  k_finalize_sum<<<1, 1024, 0, c->stream>>>(parts, nparts, dst);
  DV_LAUNCHED(c);
  return DV_OK;
}

// ------------------------------------------------------------- FP32 peak
__global__ void k_fma_chain(float* out, int iters, float a, float b) {
  float x0 = threadIdx.x * 1e-7f, x1 = x0 + 1e-7f, x2 = x0 + 2e-7f, x3 = x0 + 3e-7f;
  float x4 = x0 + 4e-7f, x5 = x0 + 5e-7f, x6 = x0 + 6e-7f, x7 = x0 + 7e-7f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      x0 = fmaf(x0, a, b); x1 = fmaf(x1, a, b); x2 = fmaf(x2, a, b); x3 = fmaf(x3, a, b);
      x4 = fmaf(x4, a, b); x5 = fmaf(x5, a, b); x6 = fmaf(x6, a, b); x7 = fmaf(x7, a, b);
    }
  }
  float s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
  if (s == 12345.678f) out[0] = s;  // keeps the chain live
}

DV_API int dv_fp32_peak(dv_ctx* c, double* flops_out) {
  if (!c || !flops_out) return DV_EINVAL;
  float* d = nullptr;
  // scratch: one float in the flag buffer's spare word
  d = reinterpret_cast<float*>(c->d_flag + 3);
  const int threads = 256, blocks = c->num_sms * 8, iters = 4096;
  cudaEvent_t e0, e1;
  DV_CK(c, cudaEventCreate(&e0));
  DV_CK(c, cudaEventCreate(&e1));
  k_fma_chain<<<blocks, threads, 0, c->stream>>>(d, 64, 0.999999f, 1e-7f);  // warm-up
  DV_LAUNCHED(c);
  DV_CK(c, cudaEventRecord(e0, c->stream));
  k_fma_chain<<<blocks, threads, 0, c->stream>>>(d, iters, 0.999999f, 1e-7f);
  DV_LAUNCHED(c);
  DV_CK(c, cudaEventRecord(e1, c->stream));
  DV_CK(c, cudaEventSynchronize(e1));
  float ms = 0.f;
  DV_CK(c, cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  double fmas = (double)blocks * threads * iters * 16.0 * 8.0;
  *flops_out = 2.0 * fmas / (ms * 1e-3);
  return DV_OK;
}
