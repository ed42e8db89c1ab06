// Allocation-free variant of the FP64 density-error reduction
// (dv_density_error), for callers that must not allocate device memory:
// real-time step loops that forbid allocation after start-up, and host
// frameworks whose own allocator owns all device memory.  It avoids
// allocation only: it copies its result to the host and synchronises the
// stream, so it is not made on a stream that is being captured.
//
// The scratch (one FP64 partial per 256-particle block plus the result) lives
// in a file-scope __device__ array, so every GPU that loads this library holds
// its 512 KB until the process exits.  In host code the array's name is only
// a host-side stand-in, so its device address is fetched with
// cudaGetSymbolAddress on every call, with the caller's device current (a
// lookup in the loaded module, not an allocation); a cached address could
// point at freed memory after a device reset.  Every call shares the array:
// calls that overlap on the GPU (different streams, or different host
// threads on one device) race on it.  Each call writes every partial it
// reads, so nothing has to start at zero.
#include "dv_internal.cuh"

#define DV_NOALLOC_BLOCK 256
#define DV_NOALLOC_MAX_BLOCKS 65536  // 16,777,216 particles
#define DV_NOALLOC_MAX_N ((int64_t)DV_NOALLOC_BLOCK * DV_NOALLOC_MAX_BLOCKS)

static __device__ __align__(256) double g_dv_noalloc_scratch[DV_NOALLOC_MAX_BLOCKS + 32];

namespace {
// block partials of compute_density_error (dimcv_sph.py:407-419) over slots
// [0, n); the same per-block layout and term as k_density_error in dv_sph.cu
template <int D>
__global__ void k_density_error_noalloc(dv_params P, dv_fields F, int n, float offset,
                                        double* __restrict__ part) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double err = 0.0;
  if (i < n && F.material[i] == DV_MATERIAL_FLUID) {
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

// the fixed summation order of dv_finalize_sum (1024 strided partial sums,
// then a block tree)
__global__ void k_noalloc_finalize(const double* __restrict__ part, int nparts, double* dst) {
  double s = 0.0;
  for (int k = threadIdx.x; k < nparts; k += blockDim.x) s += part[k];
  s = block_sum<double>(s);
  if (threadIdx.x == 0) *dst = s;
}
}  // namespace

DV_API int dv_density_error_noalloc(const dv_params* params, const dv_fields* f, int32_t n, float offset,
                                    double* out, void* stream) {
  if (!params || !f || !out) return dv_fail(nullptr, DV_EINVAL, "dv_density_error_noalloc: NULL argument");
  if (params->dim != 2 && params->dim != 3)
    return dv_fail(nullptr, DV_EINVAL, "dv_density_error_noalloc: dim must be 2 or 3");
  if (n < 0) return dv_fail(nullptr, DV_EINVAL, "dv_density_error_noalloc: negative n");
  if ((int64_t)n > DV_NOALLOC_MAX_N)
    return dv_fail(nullptr, DV_ECAPACITY,
                   "dv_density_error_noalloc: n=%d exceeds the allocation-free limit of %lld particles", n,
                   (long long)DV_NOALLOC_MAX_N);
  if (n > 0 && (!f->material || !f->density_adv || (params->has_transit && !f->x)))
    return dv_fail(nullptr, DV_EINVAL, "dv_density_error_noalloc: a needed field pointer is NULL");
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_dv_noalloc_scratch);
  if (e != cudaSuccess) return dv_cuda_check(nullptr, e, "cudaGetSymbolAddress(noalloc scratch)");
  double* scratch = static_cast<double*>(p);
  cudaStream_t s = (cudaStream_t)stream;
  const int nb = n > 0 ? (int)((n + DV_NOALLOC_BLOCK - 1) / DV_NOALLOC_BLOCK) : 1;
  double* result = scratch + DV_NOALLOC_MAX_BLOCKS;
  if (params->dim == 2)
    k_density_error_noalloc<2><<<nb, DV_NOALLOC_BLOCK, 0, s>>>(*params, *f, n, offset, scratch);
  else
    k_density_error_noalloc<3><<<nb, DV_NOALLOC_BLOCK, 0, s>>>(*params, *f, n, offset, scratch);
  e = cudaGetLastError();
  if (e != cudaSuccess) return dv_cuda_check(nullptr, e, "dv_density_error_noalloc launch");
  k_noalloc_finalize<<<1, 1024, 0, s>>>(scratch, nb, result);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, result, sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return dv_cuda_check(nullptr, e, "dv_density_error_noalloc");
  return DV_OK;
}
