// Shared declarations of the hedge_b200 CUDA library.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/hedge_b200.h"

namespace hb {

// Per-thread last-error text (hb_last_error_string).
void set_error(const std::string& msg);
hb_status fail(hb_status st, const std::string& msg);
hb_status cuda_fail(cudaError_t err, const char* what);

#define HB_CUDA(call)                                              \
  do {                                                             \
    cudaError_t err__ = (call);                                    \
    if (err__ != cudaSuccess) return ::hb::cuda_fail(err__, #call); \
  } while (0)

// Model parameters passed by value to every kernel.
struct ModelParams {
  double v[3];
  double c, eps, mu, alpha, bdry_alpha, time_sign;
  double Z, Y;   // Maxwell impedance sqrt(mu/eps) and admittance 1/Z
  int flux_type, bdry_flux_type;
};

// Device error-flag codes (first error wins).
enum : int {
  DEV_OK = 0,
  DEV_BAD_NEIGHBOUR = 1,
  DEV_BAD_CODE = 2,
  DEV_BAD_BDRY_INDEX = 3,
  DEV_MISSING_INPUT = 4,
  DEV_MMA_TIMEOUT = 5
};

// Makes `dev` current for the guard's lifetime, restoring the caller's device.
struct DeviceGuard {
  int prev = -1;
  bool ok = false;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) return;
    ok = prev == dev || cudaSetDevice(dev) == cudaSuccess;
  }
  ~DeviceGuard() {
    int cur;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

// Operator data uploaded once per discretization.
struct Discr {
  int device;
  int dim, order, np, nfp, nfaces, nperm, G;
  int64_t K;
  // FP64 copies (device)
  double* dmats_t = nullptr;   // [dim][np(j)][np(i)] transposed
  double* lift_t = nullptr;    // [nfaces*nfp(k)][np(i)] transposed
  double* geo = nullptr;       // [K][G]
  // FP32 copies (device), made on first FP32 operator
  float* dmats_t32 = nullptr;
  float* lift_t32 = nullptr;
  float* geo32 = nullptr;
  double* mass = nullptr;      // [np][np] reference mass matrix
  double* absjac = nullptr;    // [K]
  double* norm_partials = nullptr;  // one FP64 partial sum per norm block
  int norm_blocks = 0;
  int* fmask = nullptr;        // [nfaces][nfp]
  int* shuffle = nullptr;      // [nperm][nfp]
  // host copies kept for split-operator construction
  std::string host_blob;
  std::vector<double> unit_nodes;   // [np][dim]
};

struct Op {
  Discr* d;
  int model, F, precision;   // precision: HB_PREC_FP64 .. HB_PREC_FP16X3 (FP32_SIMT is stored as FP32)
  int split = 0;             // 1: the tensor-core kernels (launch_split), else CUDA cores
  ModelParams mp;
  int2* conn = nullptr;        // [K][nfaces] (nbr, code)
  int64_t n_given;
  int64_t n_halo = 0;          // halo faces (neighbours K .. K + n_halo - 1)
  const void* halo = nullptr;  // [n_halo * nfp][F] ext values, state dtype (caller's)
  const double* halo_c = nullptr;  // [n_halo * nfp] ext c values (var-c wave)
  int* err_flag = nullptr;     // device int
  // launch configuration chosen at create time
  int elems_per_block = 0;
  int threads = 0;
  size_t smem = 0;
  int grid = 0;
  int ops_in_smem = 1;
  int blocks_per_sm = 0;
  // split-precision operator planes (BF16X3)
  void* split_ops = nullptr;
  // quadrature operator (variable-coefficient advection): point counts, the
  // four matrices (FP64 and, for FP32 operators, FP32 copies) and the
  // element maxima of |v|^2 the LF flux reads
  int nq = 0, nqf = 0;
  double* quad64 = nullptr;
  double* elmax = nullptr;
};

hb_status check_device_flag(Op* op, cudaStream_t s);

// energy norm (norm.cu)
constexpr int NORM_THREADS = 256;
int norm_elems_per_block(int np);
hb_status launch_norm(int64_t K, int np, int nfields, int dtype, const double* mass,
                      const double* absjac, const void* u, double* partials, int nblocks,
                      double* out, cudaStream_t s);

// adjoint of the RHS (adjoint.cu)
int64_t adjoint_work_bytes(const Op* op);
hb_status launch_adjoint(Op* op, const double* q, const double* lam, double* q_bar,
                         double* c_bar, const double* coeff, double* work, cudaStream_t s);

// gather for halo exchange (rhs_simt.cu): dst[j][f] = src[f][idx[j]]
hb_status launch_pack(int64_t n, int dtype, int nfields, int64_t field_stride,
                      const int64_t* idx, const void* src, void* dst, cudaStream_t s);

// kernel launchers (rhs_simt.cu)
// e0, e1: the elements [e0, e1) the launch updates
hb_status launch_simt(Op* op, int mode, double a, double b, double dt,
                      const void* q_in, void* q_out, void* res,
                      const double* coeff, const double* bdry,
                      const double* source, int64_t e0, int64_t e1, cudaStream_t s);
hb_status prepare_simt(Op* op);

// quadrature kernel (rhs_quad.cu); vel = the velocity field [dim][K*Np]
hb_status prepare_quad(Op* op);
hb_status launch_quad(Op* op, int mode, double ra, double rb, double dt, const void* q_in,
                      void* q_out, void* res, const double* vel, const double* bdry,
                      cudaStream_t s);

}  // namespace hb
