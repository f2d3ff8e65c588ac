// FP64 energy norm sqrt(sum_f sum_k |J_k| u_fk^T M u_fk) of DG volume vectors
// (the reference's Discretization.norm, hedge/discretization/__init__.py:
// 1126-1139, which compiles sqrt(integral(u * MassOperator u))).
//
// Pass 1: block b owns a fixed range of elements; thread (element, node i)
// forms u_i (M u)_i |J| in FP64 and the block reduces them in a fixed tree
// order into partials[b].  Pass 2: one block reduces the partials in a fixed
// order and writes sqrt(sum).  The result is bitwise reproducible.
#include <cstdio>
#include <mutex>

#include "common.cuh"

namespace hb {

int norm_elems_per_block(int np) {
  const int e = NORM_THREADS / np;
  return e < 1 ? 1 : e;
}

template <typename T>
__global__ void __launch_bounds__(NORM_THREADS) norm_partial_kernel(
    int64_t K, int np, int nfields, int epb, const double* __restrict__ mass,
    const double* __restrict__ absjac, const T* __restrict__ u,
    double* __restrict__ partials) {
  __shared__ double red[NORM_THREADS];
  const int tid = threadIdx.x;
  const int el = tid / np, i = tid - el * np;
  const int64_t e = (int64_t)blockIdx.x * epb + el;
  double acc = 0.0;
  if (el < epb && e < K) {
    const double jac = absjac[e];
    for (int f = 0; f < nfields; ++f) {
      const T* ue = u + (int64_t)f * K * np + e * np;
      double mu = 0.0;
      for (int j = 0; j < np; ++j) mu += mass[i * np + j] * (double)ue[j];
      acc += (double)ue[i] * mu * jac;
    }
  }
  red[tid] = acc;
  __syncthreads();
  for (int w = NORM_THREADS / 2; w > 0; w >>= 1) {
    if (tid < w) red[tid] += red[tid + w];
    __syncthreads();
  }
  if (tid == 0) partials[blockIdx.x] = red[0];
}

__global__ void __launch_bounds__(NORM_THREADS) norm_final_kernel(
    const double* __restrict__ partials, int n, double* __restrict__ out) {
  __shared__ double red[NORM_THREADS];
  const int tid = threadIdx.x;
  double acc = 0.0;
  for (int b = tid; b < n; b += NORM_THREADS) acc += partials[b];
  red[tid] = acc;
  __syncthreads();
  for (int w = NORM_THREADS / 2; w > 0; w >>= 1) {
    if (tid < w) red[tid] += red[tid + w];
    __syncthreads();
  }
  if (tid == 0) out[0] = sqrt(red[0] > 0.0 ? red[0] : 0.0);
}

hb_status launch_norm(int64_t K, int np, int nfields, int dtype, const double* mass,
                      const double* absjac, const void* u, double* partials, int nblocks,
                      double* out, cudaStream_t s) {
  if (np < 1 || np > NORM_THREADS)
    return fail(HB_ERR_UNSUPPORTED, "norm: element node count beyond one block");
  const int epb = norm_elems_per_block(np);
  if ((int64_t)nblocks * epb < K)
    return fail(HB_ERR_INVALID_ARGUMENT, "norm: partial-sum buffer too small for K");
  const int grid = (int)((K + epb - 1) / epb);
  if (dtype == 0)
    norm_partial_kernel<double><<<grid, NORM_THREADS, 0, s>>>(
        K, np, nfields, epb, mass, absjac, static_cast<const double*>(u), partials);
  else
    norm_partial_kernel<float><<<grid, NORM_THREADS, 0, s>>>(
        K, np, nfields, epb, mass, absjac, static_cast<const float*>(u), partials);
  HB_CUDA(cudaGetLastError());
  norm_final_kernel<<<1, NORM_THREADS, 0, s>>>(partials, grid, out);
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

}  // namespace hb

// ---------------------------------------------------------------------------
// Allocation-free energy norm (hb_norm_noalloc).  Same two kernels as hb_norm;
// the per-block partial sums live in a fixed device array of this file instead
// of a buffer owned by an hb_discr.  Some callers cannot allocate device
// memory while they run: code that holds no hb_discr (it brings its own mass
// matrix and Jacobians) and must not grow the footprint of a time loop that
// has reserved the device's memory for its fields, or that must not let an
// allocation synchronise the device between two time steps.  They call this
// entry point instead.
//
// The array keeps whatever the last call on the device left in it.  Nothing
// in it has to start at zero: the partial pass of a call writes every slot
// [0, blocks) that the final pass of the same call reads.  Two calls whose
// kernels overlap on one device (other streams, other host threads) share the
// array and race; callers serialise them.
// ---------------------------------------------------------------------------
namespace hb {

static __device__ __align__(256) double norm_noalloc_partials[HB_NORM_NOALLOC_MAX_BLOCKS];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
double* g_noalloc_ptr[kMaxDevices] = {};

// Address of the array on the current device, looked up once per device.
// The lookup may load this library's device code on that device, which is why
// the first call on a device belongs before any stream capture.
hb_status noalloc_scratch(double** ptr) {
  int dev = -1;
  HB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices)
    return fail(HB_ERR_UNSUPPORTED, "norm_noalloc: device index beyond 63");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, norm_noalloc_partials);
    if (e != cudaSuccess || !p)
      return cuda_fail(e != cudaSuccess ? e : cudaErrorInvalidSymbol,
                       "norm_noalloc: cudaGetSymbolAddress of the scratch array");
    g_noalloc_ptr[dev] = static_cast<double*>(p);
  }
  *ptr = g_noalloc_ptr[dev];
  return HB_OK;
}
}  // namespace

}  // namespace hb

extern "C" hb_status hb_norm_noalloc(int64_t num_elements, int32_t np, int32_t nfields,
                                     int32_t dtype, const double* mass,
                                     const double* abs_jacobian, const void* u, double* out,
                                     void* stream) {
  using namespace hb;
  if (!mass || !abs_jacobian || !u || !out)
    return fail(HB_ERR_INVALID_ARGUMENT, "norm_noalloc: null argument");
  if (num_elements < 1 || nfields < 1 || (dtype != 0 && dtype != 1))
    return fail(HB_ERR_INVALID_ARGUMENT,
                "norm_noalloc: need num_elements >= 1, nfields >= 1, dtype 0 or 1");
  if (np < 1 || np > NORM_THREADS)
    return fail(HB_ERR_UNSUPPORTED, "norm_noalloc: element node count must be 1..256");
  const int epb = norm_elems_per_block(np);
  const int64_t max_elements = (int64_t)HB_NORM_NOALLOC_MAX_BLOCKS * epb;
  if (num_elements > max_elements) {
    char msg[160];
    snprintf(msg, sizeof msg,
             "norm_noalloc: %lld elements exceed the scratch limit of %lld for %d nodes "
             "per element (8192 blocks of %d elements); use hb_norm",
             (long long)num_elements, (long long)max_elements, (int)np, epb);
    return fail(HB_ERR_INVALID_ARGUMENT, msg);
  }
  double* partials = nullptr;
  const hb_status st = noalloc_scratch(&partials);
  if (st != HB_OK) return st;
  // the scratch address is the current device's: every operand must be
  // device (or managed) memory of that same device
  {
    int dev = -1;
    HB_CUDA(cudaGetDevice(&dev));
    const void* ptrs[4] = {mass, abs_jacobian, u, out};
    const char* names[4] = {"mass", "abs_jacobian", "u", "out"};
    for (int i = 0; i < 4; ++i) {
      cudaPointerAttributes attr;
      const cudaError_t e = cudaPointerGetAttributes(&attr, ptrs[i]);
      if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(HB_ERR_INVALID_ARGUMENT,
                    std::string("norm_noalloc: cannot query the pointer ") + names[i]);
      }
      const bool on_device = attr.type == cudaMemoryTypeDevice ||
                             attr.type == cudaMemoryTypeManaged;
      if (!on_device || attr.device != dev)
        return fail(HB_ERR_INVALID_ARGUMENT,
                    std::string("norm_noalloc: ") + names[i] +
                        " is not device memory of the current device");
    }
  }
  return launch_norm(num_elements, np, nfields, dtype, mass, abs_jacobian, u, partials,
                     HB_NORM_NOALLOC_MAX_BLOCKS, out, reinterpret_cast<cudaStream_t>(stream));
}
