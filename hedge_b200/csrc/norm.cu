// FP64 energy norm sqrt(sum_f sum_k |J_k| u_fk^T M u_fk) of DG volume vectors
// (the reference's Discretization.norm, hedge/discretization/__init__.py:
// 1126-1139, which compiles sqrt(integral(u * MassOperator u))).
//
// Pass 1: block b owns a fixed range of elements; thread (element, node i)
// forms u_i (M u)_i |J| in FP64 and the block reduces them in a fixed tree
// order into partials[b].  Pass 2: one block reduces the partials in a fixed
// order and writes sqrt(sum).  The result is bitwise reproducible.
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
