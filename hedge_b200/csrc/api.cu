// C-ABI entry points of libhedge_b200 (declared in include/hedge_b200.h).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "common.cuh"

namespace hb {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

hb_status fail(hb_status st, const std::string& msg) {
  set_error(msg);
  return st;
}

hb_status cuda_fail(cudaError_t err, const char* what) {
  set_error(std::string(what) + ": " + cudaGetErrorString(err));
  return HB_ERR_CUDA;
}

// Makes `dev` current for the scope of one C-ABI call and restores the
// caller's device afterwards.

template <typename T>
static hb_status upload(T** dst, const T* src, size_t n) {
  HB_CUDA(cudaMalloc(reinterpret_cast<void**>(dst), sizeof(T) * (n ? n : 1)));
  if (n) HB_CUDA(cudaMemcpy(*dst, src, sizeof(T) * n, cudaMemcpyHostToDevice));
  return HB_OK;
}

static void free_discr(Discr* d) {
  if (!d) return;
  cudaFree(d->dmats_t); cudaFree(d->lift_t); cudaFree(d->geo);
  cudaFree(d->dmats_t32); cudaFree(d->lift_t32); cudaFree(d->geo32);
  cudaFree(d->fmask); cudaFree(d->shuffle);
  cudaFree(d->mass); cudaFree(d->absjac); cudaFree(d->norm_partials);
  delete d;
}

hb_status ensure_fp32(Discr* d) {
  if (d->geo32) return HB_OK;
  const double* host = reinterpret_cast<const double*>(d->host_blob.data());
  const size_t nd = (size_t)d->dim * d->np * d->np;
  const size_t nl = (size_t)d->nfaces * d->nfp * d->np;
  const size_t ng = (size_t)d->K * d->G;
  std::vector<float> tmp(nd + nl + ng);
  for (size_t x = 0; x < nd + nl + ng; ++x) tmp[x] = (float)host[x];
  hb_status st;
  if ((st = upload(&d->dmats_t32, tmp.data(), nd))) return st;
  if ((st = upload(&d->lift_t32, tmp.data() + nd, nl))) return st;
  if ((st = upload(&d->geo32, tmp.data() + nd + nl, ng))) return st;
  return HB_OK;
}

hb_status check_device_flag(Op* op, cudaStream_t s) {
  int flag = 0;
  HB_CUDA(cudaMemcpyAsync(&flag, op->err_flag, sizeof(int), cudaMemcpyDeviceToHost, s));
  HB_CUDA(cudaStreamSynchronize(s));
  if (flag != DEV_OK) {
    static const char* what[] = {"ok", "face neighbour out of range",
                                 "invalid neighbour face / permutation code",
                                 "boundary index out of range", "missing input vector",
                                 "a tensor-core kernel's bounded wait ran out "
                                 "(MMA completion or a data hand-off)"};
    // reported once: the flag is cleared so that the operator can be used
    // again once the caller has dealt with the error
    HB_CUDA(cudaMemsetAsync(op->err_flag, 0, sizeof(int), s));
    HB_CUDA(cudaStreamSynchronize(s));
    return fail(HB_ERR_DEVICE_FLAG,
                std::string("device check failed: ") + (flag < 6 ? what[flag] : "unknown"));
  }
  return HB_OK;
}

hb_status launch_gather_map(Op* op, int64_t* int_idx, int64_t* ext_idx, cudaStream_t s);
hb_status launch_lincomb(int64_t n, int dtype, double a, const void* x, double b,
                         const void* y, void* out, cudaStream_t s);
hb_status prepare_split(Op* op);
hb_status launch_split(Op* op, int mode, double ra, double rb, double dt,
                       const void* q_in, void* q_out, void* res, const double* coeff,
                       const double* bdry, const double* source, int64_t e0, int64_t e1,
                       cudaStream_t s);
void free_split(Op* op);
hb_status launch_wait_selftest(int* err, uint64_t limit_ns, cudaStream_t s);

// The quadrature matrices in the kernel's layouts (each transposed so that
// consecutive threads read consecutive entries): It [np][nq],
// Bt [dim][nq][np], Ft [nf][nfp][nqf], Lt [nf*nqf][np], back to back; FP32
// copies for FP32 operators; the element-maximum buffer for the LF flux.
static hb_status upload_quadrature(Op* op, const hb_quad_desc* qd) {
  const Discr* d = op->d;
  const int np = d->np, nfp = d->nfp, nf = d->nfaces, dim = d->dim;
  const int nq = qd->nq, nqf = qd->nqf;
  const size_t nI = (size_t)np * nq, nB = (size_t)dim * nq * np, nF = (size_t)nf * nfp * nqf;
  const size_t nL = (size_t)nf * nqf * np;
  std::vector<double> h(nI + nB + nF + nL);
  for (int q = 0; q < nq; ++q)
    for (int j = 0; j < np; ++j) h[(size_t)j * nq + q] = qd->vol_interp[(size_t)q * np + j];
  for (int r = 0; r < dim; ++r)
    for (int i = 0; i < np; ++i)
      for (int q = 0; q < nq; ++q)
        h[nI + ((size_t)r * nq + q) * np + i] = qd->vol_project[((size_t)r * np + i) * nq + q];
  for (int f = 0; f < nf; ++f)
    for (int q = 0; q < nqf; ++q)
      for (int k = 0; k < nfp; ++k)
        h[nI + nB + ((size_t)f * nfp + k) * nqf + q] =
            qd->face_interp[((size_t)f * nqf + q) * nfp + k];
  for (int i = 0; i < np; ++i)
    for (int p = 0; p < nf * nqf; ++p)
      h[nI + nB + nF + (size_t)p * np + i] = qd->face_lift[(size_t)i * nf * nqf + p];
  for (double x : h)
    if (!std::isfinite(x)) return fail(HB_ERR_INVALID_ARGUMENT, "non-finite quadrature matrix");
  op->nq = nq;
  op->nqf = nqf;
  hb_status st;
  // FP64 matrices for both precisions (the FP32 path computes in FP64)
  if ((st = upload(&op->quad64, h.data(), h.size()))) return st;
  if (cudaMalloc(&op->elmax, sizeof(double) * d->K) != cudaSuccess)
    return fail(HB_ERR_CUDA, "cannot allocate the element maxima");
  return HB_OK;
}

}  // namespace hb

using namespace hb;

extern "C" {

const char* hb_last_error_string(void) { return g_last_error.c_str(); }

hb_status hb_discr_create(const hb_discr_desc* desc, hb_discr** out) {
  if (!desc || !out) return fail(HB_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  if (desc->dim != 2 && desc->dim != 3)
    return fail(HB_ERR_UNSUPPORTED, "dim must be 2 or 3");
  if (desc->nfaces != desc->dim + 1 || desc->np < 1 || desc->nfp < 1 ||
      desc->num_elements < 1 || desc->nperm < 1 || desc->nperm > 6)
    return fail(HB_ERR_INVALID_ARGUMENT, "inconsistent element sizes");
  if (!desc->dmats || !desc->lift || !desc->geometry || !desc->fmask || !desc->shuffle ||
      !desc->unit_nodes || !desc->mass || !desc->abs_jacobian)
    return fail(HB_ERR_INVALID_ARGUMENT, "null operator or geometry pointer");
  const int np = desc->np, nfp = desc->nfp, nf = desc->nfaces, dim = desc->dim;
  for (int x = 0; x < nf * nfp; ++x)
    if (desc->fmask[x] < 0 || desc->fmask[x] >= np)
      return fail(HB_ERR_INVALID_ARGUMENT, "fmask entry out of range");
  for (int x = 0; x < desc->nperm * nfp; ++x)
    if (desc->shuffle[x] < 0 || desc->shuffle[x] >= nfp)
      return fail(HB_ERR_INVALID_ARGUMENT, "shuffle entry out of range");
  DeviceGuard g(desc->device);
  if (!g.ok) return fail(HB_ERR_CUDA, "cannot select the CUDA device");
  Discr* d = new (std::nothrow) Discr();
  if (!d) return fail(HB_ERR_INVALID_ARGUMENT, "out of host memory");
  d->device = desc->device;
  d->dim = dim; d->order = desc->order; d->np = np; d->nfp = nfp; d->nfaces = nf;
  d->nperm = desc->nperm; d->K = desc->num_elements;
  d->G = dim * dim + nf * (dim + 1);
  const size_t nd = (size_t)dim * np * np, nl = (size_t)nf * nfp * np;
  const size_t ng = (size_t)d->K * d->G;
  // transposed operators + geometry, kept on the host for other precisions
  d->host_blob.resize(sizeof(double) * (nd + nl + ng));
  double* h = reinterpret_cast<double*>(&d->host_blob[0]);
  for (int r = 0; r < dim; ++r)
    for (int i = 0; i < np; ++i)
      for (int j = 0; j < np; ++j)
        h[((size_t)r * np + j) * np + i] = desc->dmats[((size_t)r * np + i) * np + j];
  for (int i = 0; i < np; ++i)
    for (int k = 0; k < nf * nfp; ++k)
      h[nd + (size_t)k * np + i] = desc->lift[(size_t)i * nf * nfp + k];
  std::memcpy(h + nd + nl, desc->geometry, sizeof(double) * ng);
  d->unit_nodes.assign(desc->unit_nodes, desc->unit_nodes + (size_t)np * dim);
  hb_status st;
  if ((st = upload(&d->dmats_t, h, nd)) || (st = upload(&d->lift_t, h + nd, nl)) ||
      (st = upload(&d->geo, h + nd + nl, ng)) ||
      (st = upload(&d->fmask, desc->fmask, (size_t)nf * nfp)) ||
      (st = upload(&d->shuffle, desc->shuffle, (size_t)desc->nperm * nfp)) ||
      (st = upload(&d->mass, desc->mass, (size_t)np * np)) ||
      (st = upload(&d->absjac, desc->abs_jacobian, (size_t)d->K))) {
    free_discr(d);
    return st;
  }
  {
    const int epb = norm_elems_per_block(np);
    d->norm_blocks = (int)((d->K + epb - 1) / epb);
    if (cudaMalloc(&d->norm_partials, sizeof(double) * d->norm_blocks) != cudaSuccess) {
      free_discr(d);
      return fail(HB_ERR_CUDA, "cannot allocate the norm partial sums");
    }
  }
  *out = reinterpret_cast<hb_discr*>(d);
  return HB_OK;
}

hb_status hb_discr_destroy(hb_discr* discr) {
  if (!discr) return HB_OK;
  Discr* d = reinterpret_cast<Discr*>(discr);
  DeviceGuard g(d->device);
  free_discr(d);
  return HB_OK;
}

hb_status hb_op_create(hb_discr* discr, const hb_op_desc* desc, hb_op** out) {
  if (!discr || !desc || !out) return fail(HB_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  Discr* d = reinterpret_cast<Discr*>(discr);
  const int model = desc->model;
  int F;
  switch (model) {
    case HB_MODEL_ADVECTION: F = 1; break;
    case HB_MODEL_WAVE: case HB_MODEL_VARWAVE: F = d->dim + 1; break;
    case HB_MODEL_MAXWELL:
      if (d->dim != 3) return fail(HB_ERR_UNSUPPORTED, "Maxwell needs a 3D mesh");
      F = 6; break;
    case HB_MODEL_MAXWELL_TM: case HB_MODEL_MAXWELL_TE:
      if (d->dim != 2) return fail(HB_ERR_UNSUPPORTED, "TM / TE Maxwell needs a 2D mesh");
      F = 3; break;
    case HB_MODEL_VARADV: F = 1; break;
    default: return fail(HB_ERR_INVALID_ARGUMENT, "unknown model id");
  }
  const hb_quad_desc* qd = desc->quadrature;
  if (model == HB_MODEL_VARADV) {
    if (!qd) return fail(HB_ERR_INVALID_ARGUMENT, "variable-coefficient advection needs the "
                                                  "quadrature grid (hb_op_desc.quadrature)");
    if (qd->nq < 1 || qd->nqf < 1 || qd->nq > 4096 || qd->nqf > 1024 || !qd->vol_interp ||
        !qd->vol_project || !qd->face_interp || !qd->face_lift)
      return fail(HB_ERR_INVALID_ARGUMENT, "bad quadrature descriptor");
    if (desc->flux_type < 0 || desc->flux_type > 2)
      return fail(HB_ERR_INVALID_ARGUMENT, "flux type: 0 central, 1 upwind, 2 LF");
    if (desc->num_halo_faces != 0)
      return fail(HB_ERR_UNSUPPORTED, "quadrature operator: no halo faces");
    if (desc->precision != HB_PREC_FP64 && desc->precision != HB_PREC_FP32 &&
        desc->precision != HB_PREC_FP32_SIMT)
      return fail(HB_ERR_UNSUPPORTED, "quadrature operator: FP64 or FP32 only");
  } else if (qd) {
    return fail(HB_ERR_INVALID_ARGUMENT, "quadrature grid given for a model without one");
  }
  if (desc->num_fields != F)
    return fail(HB_ERR_INVALID_ARGUMENT, "num_fields does not match the model");
  if (desc->precision < HB_PREC_FP64 || desc->precision > HB_PREC_FP32_SIMT)
    return fail(HB_ERR_INVALID_ARGUMENT, "unknown precision");
  if (!desc->conn) return fail(HB_ERR_INVALID_ARGUMENT, "null connectivity");
  if ((model == HB_MODEL_MAXWELL || model == HB_MODEL_MAXWELL_TM ||
       model == HB_MODEL_MAXWELL_TE) && !(desc->eps > 0 && desc->mu > 0))
    return fail(HB_ERR_INVALID_ARGUMENT, "Maxwell material must be positive");
  // host validation of the face table (the kernels also flag bad entries)
  const int64_t nfc = d->K * d->nfaces;
  if (desc->num_halo_faces < 0) return fail(HB_ERR_INVALID_ARGUMENT, "negative halo face count");
  const int64_t nb_end = d->K + desc->num_halo_faces;   // neighbours K.. are halo slots
  int64_t max_given = 0;
  for (int64_t x = 0; x < nfc; ++x) {
    const int nbr = desc->conn[2 * x], code = desc->conn[2 * x + 1];
    if (nbr >= 0) {
      if (nbr >= nb_end || (code & 3) >= d->nfaces || (code >> 2) >= d->nperm || code < 0)
        return fail(HB_ERR_INVALID_ARGUMENT, "connectivity entry out of range");
    } else {
      if (code < HB_BC_NONE || code > HB_BC_INCIDENT)
        return fail(HB_ERR_INVALID_ARGUMENT, "unknown boundary-condition kind");
      if (code == HB_BC_INCIDENT && model != HB_MODEL_MAXWELL &&
          model != HB_MODEL_MAXWELL_TM && model != HB_MODEL_MAXWELL_TE)
        return fail(HB_ERR_INVALID_ARGUMENT, "incident boundary on a model other than Maxwell");
      if (code == HB_BC_GIVEN || (code == HB_BC_INCIDENT && desc->num_given_bdry_nodes > 0))
        max_given = std::max<int64_t>(max_given, ((int64_t)(-1 - nbr) + 1) * d->nfp);
    }
  }
  if (max_given > desc->num_given_bdry_nodes)
    return fail(HB_ERR_INVALID_ARGUMENT, "given-BC face beyond num_given_bdry_nodes");
  DeviceGuard g(d->device);
  if (!g.ok) return fail(HB_ERR_CUDA, "cannot select the CUDA device");
  Op* op = new (std::nothrow) Op();
  if (!op) return fail(HB_ERR_INVALID_ARGUMENT, "out of host memory");
  op->d = d;
  op->model = model;
  op->F = F;
  // FP32_SIMT is the FP32 path kept on the CUDA cores
  op->precision = desc->precision == HB_PREC_FP32_SIMT ? HB_PREC_FP32 : desc->precision;
  op->n_given = desc->num_given_bdry_nodes;
  op->n_halo = desc->num_halo_faces;
  ModelParams& mp = op->mp;
  for (int k = 0; k < 3; ++k) mp.v[k] = desc->v[k];
  mp.c = desc->c; mp.eps = desc->eps; mp.mu = desc->mu;
  mp.Z = (desc->eps > 0 && desc->mu > 0) ? std::sqrt(desc->mu / desc->eps) : 1.0;
  mp.Y = 1.0 / mp.Z;
  mp.alpha = desc->alpha; mp.bdry_alpha = desc->bdry_alpha;
  mp.time_sign = desc->time_sign;
  mp.flux_type = desc->flux_type; mp.bdry_flux_type = desc->bdry_flux_type;
  hb_status st;
  auto bail = [&](hb_status s) {
    cudaFree(op->conn); cudaFree(op->err_flag);
    cudaFree(op->quad64); cudaFree(op->elmax);
    free_split(op);
    delete op;
    return s;
  };
  if ((st = upload(&op->conn, reinterpret_cast<const int2*>(desc->conn), (size_t)nfc)))
    return bail(st);
  if (cudaMalloc(&op->err_flag, sizeof(int)) != cudaSuccess ||
      cudaMemset(op->err_flag, 0, sizeof(int)) != cudaSuccess)
    return bail(fail(HB_ERR_CUDA, "cannot allocate the device error flag"));
  if (op->precision == HB_PREC_FP32 && (st = ensure_fp32(d))) return bail(st);
  if (model == HB_MODEL_VARADV) {
    st = upload_quadrature(op, qd);
    if (!st) st = prepare_quad(op);
  } else if (op->precision == HB_PREC_BF16X3 || op->precision == HB_PREC_FP16X3) {
    st = prepare_split(op);
    op->split = 1;
  } else if (op->precision == HB_PREC_FP32 && desc->precision != HB_PREC_FP32_SIMT) {
    // FP32 state on the tensor cores where a resident kernel is built for
    // this (model, dimension, order), else on the CUDA cores
    st = prepare_split(op);
    op->split = st == HB_OK;
    if (st == HB_ERR_UNSUPPORTED) {
      free_split(op);
      st = prepare_simt(op);
    }
  } else {
    st = prepare_simt(op);
  }
  if (st) return bail(st);
  *out = reinterpret_cast<hb_op*>(op);
  return HB_OK;
}

hb_status hb_op_destroy(hb_op* handle) {
  if (!handle) return HB_OK;
  Op* op = reinterpret_cast<Op*>(handle);
  DeviceGuard g(op->d->device);
  cudaFree(op->conn);
  cudaFree(op->err_flag);
  cudaFree(op->quad64); cudaFree(op->elmax);
  free_split(op);
  delete op;
  return HB_OK;
}

static hb_status check_inputs(Op* op, const void* q_in, const void* q_out,
                              const double* coeff, const double* bdry) {
  if (!q_in || !q_out) return fail(HB_ERR_INVALID_ARGUMENT, "null state pointer");
  if (q_in == q_out) return fail(HB_ERR_INVALID_ARGUMENT, "output aliases the input state");
  if (op->n_halo > 0 && !op->halo)
    return fail(HB_ERR_INVALID_ARGUMENT, "halo faces but no halo buffer (hb_op_set_halo)");
  if (op->model == HB_MODEL_VARWAVE && !coeff)
    return fail(HB_ERR_INVALID_ARGUMENT, "variable-velocity wave needs the c field");
  if (op->model == HB_MODEL_VARADV && !coeff)
    return fail(HB_ERR_INVALID_ARGUMENT, "variable-coefficient advection needs the velocity");
  const bool maxwell = op->model == HB_MODEL_MAXWELL || op->model == HB_MODEL_MAXWELL_TM ||
                       op->model == HB_MODEL_MAXWELL_TE;
  if (maxwell && coeff && op->split)
    return fail(HB_ERR_UNSUPPORTED, "Maxwell with variable material: CUDA-core kernels only "
                                    "(HB_PREC_FP64, HB_PREC_FP32_SIMT)");
  if (maxwell && bdry && op->split)
    return fail(HB_ERR_UNSUPPORTED, "Maxwell incident data: CUDA-core kernels only "
                                    "(HB_PREC_FP64, HB_PREC_FP32_SIMT)");
  return HB_OK;
}

static hb_status run(Op* op, int mode, double a, double b, double dt, const void* q_in,
                     void* q_out, void* res, const double* coeff, const double* bdry,
                     const double* source, void* stream, int64_t e0 = 0, int64_t e1 = -1) {
  DeviceGuard g(op->d->device);
  if (!g.ok) return fail(HB_ERR_CUDA, "cannot select the CUDA device");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const bool whole = e0 == 0 && (e1 < 0 || e1 == op->d->K);
  if (e1 < 0) e1 = op->d->K;
  if (e0 == e1) return HB_OK;
  if (op->model == HB_MODEL_VARADV) {
    if (!whole) return fail(HB_ERR_UNSUPPORTED, "element ranges: not on the quadrature kernel");
    return launch_quad(op, mode, a, b, dt, q_in, q_out, res, coeff, bdry, s);
  }
  if (op->split)
    return launch_split(op, mode, a, b, dt, q_in, q_out, res, coeff, bdry, source, e0, e1, s);
  return launch_simt(op, mode, a, b, dt, q_in, q_out, res, coeff, bdry, source, e0, e1, s);
}

static hb_status check_range(Op* op, int64_t e0, int64_t e1) {
  if (e0 < 0 || e1 < e0 || e1 > op->d->K)
    return fail(HB_ERR_INVALID_ARGUMENT, "element range outside [0, K]");
  return HB_OK;
}

hb_status hb_rhs(hb_op* handle, const void* q, void* rhs, const double* coeff,
                 const double* bdry, const double* source, void* stream) {
  if (!handle) return fail(HB_ERR_INVALID_ARGUMENT, "null operator");
  Op* op = reinterpret_cast<Op*>(handle);
  hb_status st = check_inputs(op, q, rhs, coeff, bdry);
  if (st) return st;
  return run(op, 0, 0, 0, 0, q, rhs, nullptr, coeff, bdry, source, stream);
}

hb_status hb_lsrk_stage(hb_op* handle, double a, double b, double dt, const void* q_in,
                        void* q_out, void* res, const double* coeff, const double* bdry,
                        const double* source, void* stream) {
  if (!handle) return fail(HB_ERR_INVALID_ARGUMENT, "null operator");
  Op* op = reinterpret_cast<Op*>(handle);
  hb_status st = check_inputs(op, q_in, q_out, coeff, bdry);
  if (st) return st;
  if (!res) return fail(HB_ERR_INVALID_ARGUMENT, "null residual pointer");
  return run(op, 1, a, b, dt, q_in, q_out, res, coeff, bdry, source, stream);
}

hb_status hb_rhs_elements(hb_op* handle, int64_t el_begin, int64_t el_end, const void* q,
                          void* rhs, const double* coeff, const double* bdry,
                          const double* source, void* stream) {
  if (!handle) return fail(HB_ERR_INVALID_ARGUMENT, "null operator");
  Op* op = reinterpret_cast<Op*>(handle);
  hb_status st = check_inputs(op, q, rhs, coeff, bdry);
  if (st) return st;
  if ((st = check_range(op, el_begin, el_end))) return st;
  return run(op, 0, 0, 0, 0, q, rhs, nullptr, coeff, bdry, source, stream, el_begin, el_end);
}

hb_status hb_lsrk_stage_elements(hb_op* handle, int64_t el_begin, int64_t el_end, double a,
                                 double b, double dt, const void* q_in, void* q_out,
                                 void* res, const double* coeff, const double* bdry,
                                 const double* source, void* stream) {
  if (!handle) return fail(HB_ERR_INVALID_ARGUMENT, "null operator");
  Op* op = reinterpret_cast<Op*>(handle);
  hb_status st = check_inputs(op, q_in, q_out, coeff, bdry);
  if (st) return st;
  if (!res) return fail(HB_ERR_INVALID_ARGUMENT, "null residual pointer");
  if ((st = check_range(op, el_begin, el_end))) return st;
  return run(op, 1, a, b, dt, q_in, q_out, res, coeff, bdry, source, stream, el_begin, el_end);
}

hb_status hb_lincomb(int64_t n, int32_t dtype, double a, const void* x, double b,
                     const void* y, void* out, void* stream) {
  if (n < 0 || (dtype != 0 && dtype != 1))
    return fail(HB_ERR_INVALID_ARGUMENT, "bad size or dtype");
  if (n > 0 && (!x || !y || !out)) return fail(HB_ERR_INVALID_ARGUMENT, "null vector");
  return launch_lincomb(n, dtype, a, x, b, y, out, reinterpret_cast<cudaStream_t>(stream));
}

hb_status hb_gather_map(hb_op* handle, int64_t* int_idx, int64_t* ext_idx, void* stream) {
  if (!handle || !int_idx || !ext_idx) return fail(HB_ERR_INVALID_ARGUMENT, "null argument");
  Op* op = reinterpret_cast<Op*>(handle);
  DeviceGuard g(op->d->device);
  return launch_gather_map(op, int_idx, ext_idx, reinterpret_cast<cudaStream_t>(stream));
}

hb_status hb_op_launch_info(hb_op* handle, int64_t* info, int32_t n) {
  if (!handle || !info || n < 1) return fail(HB_ERR_INVALID_ARGUMENT, "null argument");
  Op* op = reinterpret_cast<Op*>(handle);
  const int64_t v[6] = {op->grid, op->threads, (int64_t)op->smem, op->elems_per_block,
                        op->ops_in_smem, op->blocks_per_sm};
  for (int k = 0; k < n && k < 6; ++k) info[k] = v[k];
  return HB_OK;
}

hb_status hb_norm(hb_discr* discr, int32_t nfields, int32_t dtype, const void* u,
                  double* out, void* stream) {
  if (!discr || !u || !out) return fail(HB_ERR_INVALID_ARGUMENT, "null argument");
  if (nfields < 1 || (dtype != 0 && dtype != 1))
    return fail(HB_ERR_INVALID_ARGUMENT, "bad field count or dtype");
  Discr* d = reinterpret_cast<Discr*>(discr);
  DeviceGuard g(d->device);
  if (!g.ok) return fail(HB_ERR_CUDA, "cannot select the CUDA device");
  return launch_norm(d->K, d->np, nfields, dtype, d->mass, d->absjac, u, d->norm_partials,
                     d->norm_blocks, out, reinterpret_cast<cudaStream_t>(stream));
}

hb_status hb_rhs_adjoint_work_size(hb_op* handle, int64_t* bytes) {
  if (!handle || !bytes) return fail(HB_ERR_INVALID_ARGUMENT, "null argument");
  *bytes = adjoint_work_bytes(reinterpret_cast<Op*>(handle));
  return HB_OK;
}

hb_status hb_rhs_adjoint(hb_op* handle, const double* q, const double* lam, double* q_bar,
                         double* c_bar, const double* coeff, void* work, void* stream) {
  if (!handle) return fail(HB_ERR_INVALID_ARGUMENT, "null operator");
  Op* op = reinterpret_cast<Op*>(handle);
  if (!lam || !q_bar || !work) return fail(HB_ERR_INVALID_ARGUMENT, "null argument");
  if (lam == q_bar) return fail(HB_ERR_INVALID_ARGUMENT, "q_bar aliases lam");
  if (op->model == HB_MODEL_VARWAVE && !coeff)
    return fail(HB_ERR_INVALID_ARGUMENT, "variable-velocity wave needs the c field");
  if (c_bar && op->model != HB_MODEL_VARWAVE)
    return fail(HB_ERR_INVALID_ARGUMENT, "c_bar: only the variable-velocity wave has a c field");
  if (coeff && (op->model == HB_MODEL_MAXWELL || op->model == HB_MODEL_MAXWELL_TM ||
                op->model == HB_MODEL_MAXWELL_TE))
    return fail(HB_ERR_UNSUPPORTED, "adjoint: Maxwell with variable material is not built");
  if (c_bar && !q) return fail(HB_ERR_INVALID_ARGUMENT, "c_bar needs the state q");
  DeviceGuard g(op->d->device);
  if (!g.ok) return fail(HB_ERR_CUDA, "cannot select the CUDA device");
  return launch_adjoint(op, q, lam, q_bar, c_bar, coeff, static_cast<double*>(work),
                        reinterpret_cast<cudaStream_t>(stream));
}

hb_status hb_op_set_halo(hb_op* handle, const void* halo, const double* halo_coeff) {
  if (!handle) return fail(HB_ERR_INVALID_ARGUMENT, "null operator");
  Op* op = reinterpret_cast<Op*>(handle);
  if (op->n_halo == 0) return fail(HB_ERR_INVALID_ARGUMENT, "operator has no halo faces");
  if (!halo) return fail(HB_ERR_INVALID_ARGUMENT, "null halo buffer");
  if (op->model == HB_MODEL_VARWAVE && !halo_coeff)
    return fail(HB_ERR_INVALID_ARGUMENT, "variable-velocity wave needs the halo c values");
  op->halo = halo;
  op->halo_c = halo_coeff;
  return HB_OK;
}

hb_status hb_pack(int64_t n, int32_t dtype, int32_t nfields, int64_t field_stride,
                  const int64_t* idx, const void* src, void* dst, void* stream) {
  if (n < 0 || nfields < 1 || (dtype != 0 && dtype != 1))
    return fail(HB_ERR_INVALID_ARGUMENT, "bad pack size, field count or dtype");
  if (n == 0) return HB_OK;
  if (!idx || !src || !dst) return fail(HB_ERR_INVALID_ARGUMENT, "null argument");
  return launch_pack(n, dtype, nfields, field_stride, idx, src, dst,
                     reinterpret_cast<cudaStream_t>(stream));
}

hb_status hb_op_check(hb_op* handle, void* stream) {
  if (!handle) return fail(HB_ERR_INVALID_ARGUMENT, "null operator");
  Op* op = reinterpret_cast<Op*>(handle);
  DeviceGuard g(op->d->device);
  return check_device_flag(op, reinterpret_cast<cudaStream_t>(stream));
}

hb_status hb_op_wait_selftest(hb_op* handle, int64_t limit_ns, void* stream) {
  if (!handle) return fail(HB_ERR_INVALID_ARGUMENT, "null operator");
  if (limit_ns < 1000 || limit_ns > 2000000000)
    return fail(HB_ERR_INVALID_ARGUMENT, "wait self-test: limit must be 1 us .. 2 s");
  Op* op = reinterpret_cast<Op*>(handle);
  DeviceGuard g(op->d->device);
  if (!g.ok) return fail(HB_ERR_CUDA, "cannot select the operator's device");
  return launch_wait_selftest(op->err_flag, (uint64_t)limit_ns,
                              reinterpret_cast<cudaStream_t>(stream));
}

}  // extern "C"
