// Adjoint (transpose) of the DG right-hand side, FP64.
//
// For R(q; c) as computed by hb_rhs (volume terms from the chain rule of the
// reference derivatives, face fluxes lifted with LIFT and the inverse-Jacobian
// face scale, the model's output scaling), this evaluates for a cotangent
// lam of R:
//
//   q_bar = (dR/dq)^T lam          (every model: R is linear in the state)
//   c_bar = (dR/dc)^T lam at q     (variable-velocity wave, per node of c)
//
// Two kernels.  adj_face: for every element face point p,
//   w[e][p][f] = s_f * Fscale(e, face(p)) * sum_i LIFT[i][p] * lam_f[e][i]
// (s_f the model's output scale) into caller-provided scratch.  adj_element:
// one block per element forms
//   * the transposed chain rule and transposed differentiation,
//     q_bar_g[j] += sum_r sum_i D_r[i][j] y_rg[i],
//     y_rg[i] = sum_x rx_e[r][x] sum_f lam'_f[i] dvol_f / d(d_x q_g)(c_i);
//   * the transposed own-side flux at each face point, (d flux / d q-)^T w_e,
//     added to the face point's volume node;
//   * the transposed neighbour-side flux: the neighbour's face point matched
//     to this one (through the same face-pair map the forward gather uses)
//     applied (d flux_nb / d q+)^T to its w, added to this element's node --
//     the scatter-add of the reference's ext_native_write_map written as a
//     gather, so no atomics.
// The flux and volume Jacobians come from evaluating the model's own flux and
// volume functions (models.cuh) on unit vectors: each is linear in the state
// for fixed coefficients and normals, and the variable-velocity flux is
// linear in c- and c+ separately.  Boundary conditions enter through
// model_bc with the given data set to zero (their linear part); given data
// and sources do not depend on q or c.  Restated reference: the forward loops
// of jit/diff.py:137-175, jit/flux.py:239-480 and jit/lift.py:110-141, with
// the models of hedge/models/{advection,wave,em}.py.
#include <algorithm>

#include "common.cuh"
#include "models.cuh"

namespace hb {

namespace {

template <int MODEL, int DIM>
__global__ void adj_face_kernel(int64_t K, int np, int nfp, const double* __restrict__ lift_t,
                                const double* __restrict__ geo, int G, ModelParams mp,
                                const double* __restrict__ lam, double* __restrict__ work) {
  constexpr int F = Traits<MODEL, DIM>::F;
  constexpr int NF = DIM + 1;
  const int nfpt = NF * nfp;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= K * nfpt) return;
  const int64_t e = t / nfpt;
  const int p = (int)(t - e * nfpt);
  const int face = p / nfp;
  const double fscale = geo[e * G + DIM * DIM + face * (DIM + 1) + DIM];
  const double* lrow = lift_t + (int64_t)p * np;
  const int64_t Knp = K * np;
#pragma unroll
  for (int f = 0; f < F; ++f) {
    const double* l = lam + f * Knp + e * np;
    double s = 0.0;
    for (int i = 0; i < np; ++i) s += lrow[i] * l[i];
    const double sf = model_finish<MODEL, DIM, double>(mp, f, 1.0, 0.0, 0.0);
    work[t * F + f] = sf * fscale * s;
  }
}

// flux at one face point with the given argument vectors (zero when the
// boundary carries no flux)
template <int MODEL, int DIM>
__device__ __forceinline__ void flux_at(const ModelParams& mp, bool bdry, int kind,
                                        const double (&uM)[Args<MODEL, DIM>::N],
                                        const double (&uPin)[Args<MODEL, DIM>::N],
                                        const double (&n)[DIM],
                                        double (&fl)[Traits<MODEL, DIM>::F]) {
  constexpr int NA = Args<MODEL, DIM>::N;
  constexpr int F = Traits<MODEL, DIM>::F;
  double uP[NA];
#pragma unroll
  for (int q = 0; q < NA; ++q) uP[q] = uPin[q];
  if (bdry && !model_bc<MODEL, DIM, double>(mp, kind, uM, n, 0.0, uP)) {
#pragma unroll
    for (int f = 0; f < F; ++f) fl[f] = 0.0;
    return;
  }
  model_flux<MODEL, DIM, double>(mp, bdry, uM, uP, n, fl);
}

template <int MODEL, int DIM>
__global__ void adj_element_kernel(int64_t K, int np, int nfp, int nperm, int G,
                                   const double* __restrict__ dmats_t,
                                   const double* __restrict__ geo,
                                   const int* __restrict__ fmask,
                                   const int* __restrict__ shuffle,
                                   const int2* __restrict__ conn, ModelParams mp,
                                   const double* __restrict__ q,
                                   const double* __restrict__ lam,
                                   const double* __restrict__ coeff,
                                   const double* __restrict__ work,
                                   double* __restrict__ q_bar, double* __restrict__ c_bar,
                                   int* err) {
  constexpr int F = Traits<MODEL, DIM>::F;
  constexpr int C = Traits<MODEL, DIM>::COEFF;
  constexpr int NA = F + C;
  constexpr int NF = DIM + 1;
  const int nfpt = NF * nfp;
  const int64_t e = blockIdx.x;
  const int tid = threadIdx.x;
  const int64_t Knp = K * np;
  const bool want_c = C != 0 && c_bar != nullptr;

  extern __shared__ double sh[];
  double* lamp = sh;                       // [F][np]  s_f * lam_f
  double* qv = lamp + F * np;              // [F][np]  state (c gradient only)
  double* cv = qv + F * np;                // [np]     coefficient
  double* y = cv + np;                     // [DIM][F][np]
  double* acon = y + DIM * F * np;         // [nfpt][F] flux contributions
  double* gcon = acon + nfpt * F;          // [nfpt]    c-gradient contributions
  const double* ge = geo + e * G;

  for (int x = tid; x < F * np; x += blockDim.x) {
    const int f = x / np, i = x - f * np;
    const double sf = model_finish<MODEL, DIM, double>(mp, f, 1.0, 0.0, 0.0);
    lamp[x] = sf * lam[f * Knp + e * np + i];
    qv[x] = want_c ? q[f * Knp + e * np + i] : 0.0;
  }
  for (int i = tid; i < np; i += blockDim.x) cv[i] = C ? coeff[e * np + i] : 0.0;
  __syncthreads();

  // ---- volume: y_rg[i] from the model's volume map on unit gradients ----
  for (int i = tid; i < np; i += blockDim.x) {
    double m[DIM][F];
#pragma unroll
    for (int x = 0; x < DIM; ++x)
#pragma unroll
      for (int g = 0; g < F; ++g) {
        double gr[DIM][F];
#pragma unroll
        for (int xx = 0; xx < DIM; ++xx)
#pragma unroll
          for (int gg = 0; gg < F; ++gg) gr[xx][gg] = (xx == x && gg == g) ? 1.0 : 0.0;
        double vol[F];
        model_volume<MODEL, DIM, double>(mp, gr, cv[i], vol);
        double s = 0.0;
#pragma unroll
        for (int f = 0; f < F; ++f) s += lamp[f * np + i] * vol[f];
        m[x][g] = s;
      }
#pragma unroll
    for (int r = 0; r < DIM; ++r)
#pragma unroll
      for (int g = 0; g < F; ++g) {
        double s = 0.0;
#pragma unroll
        for (int x = 0; x < DIM; ++x) s += ge[r * DIM + x] * m[x][g];
        y[(r * F + g) * np + i] = s;
      }
  }

  // ---- faces: transposed own-side and neighbour-side fluxes ----
  for (int p = tid; p < nfpt; p += blockDim.x) {
    const int face = p / nfp, k = p - face * nfp;
    const int lnode = fmask[p];
    double n[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) n[d] = ge[DIM * DIM + face * (DIM + 1) + d];
    const int2 cn = conn[e * NF + face];
    const bool bdry = cn.x < 0;
    const int kind = bdry ? cn.y : 0;
    double we[F];
#pragma unroll
    for (int f = 0; f < F; ++f) we[f] = work[(e * nfpt + p) * F + f];
    // neighbour face point matched to this one
    int64_t nb = -1;
    int pn = 0, nn = 0;
    if (!bdry) {
      const int nface = cn.y & 3, perm = cn.y >> 2;
      if (cn.x < K && nface < NF && perm < nperm) {
        nb = cn.x;
        const int kk = shuffle[perm * nfp + k];
        pn = nface * nfp + kk;
        nn = fmask[pn];
      } else {
        atomicCAS(err, 0, DEV_BAD_CODE);
      }
    }
    double wn[F], nnb[DIM];
    if (nb >= 0) {
#pragma unroll
      for (int f = 0; f < F; ++f) wn[f] = work[(nb * nfpt + pn) * F + f];
      const int nface = cn.y & 3;
#pragma unroll
      for (int d = 0; d < DIM; ++d) nnb[d] = geo[nb * G + DIM * DIM + nface * (DIM + 1) + d];
    } else {
#pragma unroll
      for (int f = 0; f < F; ++f) wn[f] = 0.0;
#pragma unroll
      for (int d = 0; d < DIM; ++d) nnb[d] = 0.0;
    }
    const double cm = C ? cv[lnode] : 0.0;
    const double cp = (C && nb >= 0) ? coeff[nb * np + nn] : cm;
#pragma unroll
    for (int g = 0; g < F; ++g) {
      double uM[NA], uP[NA], fl[F];
      // own side: d flux / d q-_g
#pragma unroll
      for (int a = 0; a < NA; ++a) { uM[a] = 0.0; uP[a] = 0.0; }
      if (C) { uM[0] = cm; uP[0] = cp; }
      uM[C + g] = 1.0;
      flux_at<MODEL, DIM>(mp, bdry, kind, uM, uP, n, fl);
      double s = 0.0;
#pragma unroll
      for (int f = 0; f < F; ++f) s += we[f] * fl[f];
      // neighbour side: the neighbour's flux at its matched point, d / d q+_g
      if (nb >= 0) {
#pragma unroll
        for (int a = 0; a < NA; ++a) { uM[a] = 0.0; uP[a] = 0.0; }
        if (C) { uM[0] = cp; uP[0] = cm; }
        uP[C + g] = 1.0;
        flux_at<MODEL, DIM>(mp, false, 0, uM, uP, nnb, fl);
#pragma unroll
        for (int f = 0; f < F; ++f) s += wn[f] * fl[f];
      }
      acon[p * F + g] = s;
    }
    double gc = 0.0;
    if (want_c) {
      double uM[NA], uP[NA], fl[F];
      // own side: d flux / d c- (on a boundary c+ = c-, model_bc copies it)
      uM[0] = 1.0;
      uP[0] = 0.0;
#pragma unroll
      for (int f = 0; f < F; ++f) {
        uM[C + f] = qv[f * np + lnode];
        uP[C + f] = nb >= 0 ? q[f * Knp + nb * np + nn] : 0.0;
      }
      flux_at<MODEL, DIM>(mp, bdry, kind, uM, uP, n, fl);
#pragma unroll
      for (int f = 0; f < F; ++f) gc += we[f] * fl[f];
      if (nb >= 0) {
        // neighbour side: d flux_nb / d c+ (its c+ is this node's c)
        uM[0] = 0.0;
        uP[0] = 1.0;
#pragma unroll
        for (int f = 0; f < F; ++f) {
          uM[C + f] = q[f * Knp + nb * np + nn];
          uP[C + f] = qv[f * np + lnode];
        }
        flux_at<MODEL, DIM>(mp, false, 0, uM, uP, nnb, fl);
#pragma unroll
        for (int f = 0; f < F; ++f) gc += wn[f] * fl[f];
      }
    }
    gcon[p] = gc;
  }
  __syncthreads();

  // ---- per node: transposed differentiation + face contributions ----
  for (int j = tid; j < np; j += blockDim.x) {
    double out[F];
#pragma unroll
    for (int g = 0; g < F; ++g) out[g] = 0.0;
    for (int r = 0; r < DIM; ++r) {
      const double* drow = dmats_t + ((int64_t)r * np + j) * np;   // D_r[i][j], i = 0..np
#pragma unroll
      for (int g = 0; g < F; ++g) {
        const double* yy = y + (r * F + g) * np;
        double s = 0.0;
        for (int i = 0; i < np; ++i) s += drow[i] * yy[i];
        out[g] += s;
      }
    }
    double gc = 0.0;
    for (int p = 0; p < nfpt; ++p) {
      if (fmask[p] != j) continue;
#pragma unroll
      for (int g = 0; g < F; ++g) out[g] += acon[p * F + g];
      gc += gcon[p];
    }
#pragma unroll
    for (int g = 0; g < F; ++g) q_bar[g * Knp + e * np + j] = out[g];
    if (want_c) {
      // volume part: d vol / d c at this node = vol(grad q, c = 1)
      double gr[DIM][F];
#pragma unroll
      for (int x = 0; x < DIM; ++x)
#pragma unroll
        for (int g = 0; g < F; ++g) gr[x][g] = 0.0;
      for (int r = 0; r < DIM; ++r) {
#pragma unroll
        for (int g = 0; g < F; ++g) {
          double s = 0.0;
          for (int i = 0; i < np; ++i) s += dmats_t[((int64_t)r * np + i) * np + j] * qv[g * np + i];
#pragma unroll
          for (int x = 0; x < DIM; ++x) gr[x][g] += ge[r * DIM + x] * s;
        }
      }
      double vol[F];
      model_volume<MODEL, DIM, double>(mp, gr, 1.0, vol);
#pragma unroll
      for (int f = 0; f < F; ++f) gc += lamp[f * np + j] * vol[f];
      c_bar[e * np + j] = gc;
    }
  }
}

template <int MODEL, int DIM>
hb_status launch_adjoint_t(Op* op, const double* q, const double* lam, double* q_bar,
                           double* c_bar, const double* coeff, double* work, cudaStream_t s) {
  constexpr int F = Traits<MODEL, DIM>::F;
  Discr* d = op->d;
  const int np = d->np, nfp = d->nfp, nfpt = (DIM + 1) * nfp;
  const int64_t nface_pts = d->K * nfpt;
  const int tpb = 256;
  adj_face_kernel<MODEL, DIM><<<(unsigned)((nface_pts + tpb - 1) / tpb), tpb, 0, s>>>(
      d->K, np, nfp, d->lift_t, d->geo, d->G, op->mp, lam, work);
  HB_CUDA(cudaGetLastError());
  int threads = std::max(np, nfpt);
  threads = std::min(1024, (threads + 31) / 32 * 32);
  const size_t smem = sizeof(double) * ((size_t)F * np * 2 + np + (size_t)DIM * F * np +
                                        (size_t)nfpt * F + nfpt);
  if (smem > 48 * 1024) {
    HB_CUDA(cudaFuncSetAttribute(adj_element_kernel<MODEL, DIM>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  }
  adj_element_kernel<MODEL, DIM><<<(unsigned)d->K, threads, smem, s>>>(
      d->K, np, nfp, d->nperm, d->G, d->dmats_t, d->geo, d->fmask, d->shuffle, op->conn,
      op->mp, q, lam, coeff, work, q_bar, c_bar, op->err_flag);
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

}  // namespace

int64_t adjoint_work_bytes(const Op* op) {
  const Discr* d = op->d;
  return (int64_t)d->K * d->nfaces * d->nfp * op->F * (int64_t)sizeof(double);
}

hb_status launch_adjoint(Op* op, const double* q, const double* lam, double* q_bar,
                         double* c_bar, const double* coeff, double* work, cudaStream_t s) {
  const int dim = op->d->dim;
  switch (op->model) {
    case HB_MODEL_ADVECTION:
      return dim == 2 ? launch_adjoint_t<HB_MODEL_ADVECTION, 2>(op, q, lam, q_bar, c_bar, coeff, work, s)
                      : launch_adjoint_t<HB_MODEL_ADVECTION, 3>(op, q, lam, q_bar, c_bar, coeff, work, s);
    case HB_MODEL_WAVE:
      return dim == 2 ? launch_adjoint_t<HB_MODEL_WAVE, 2>(op, q, lam, q_bar, c_bar, coeff, work, s)
                      : launch_adjoint_t<HB_MODEL_WAVE, 3>(op, q, lam, q_bar, c_bar, coeff, work, s);
    case HB_MODEL_VARWAVE:
      return dim == 2 ? launch_adjoint_t<HB_MODEL_VARWAVE, 2>(op, q, lam, q_bar, c_bar, coeff, work, s)
                      : launch_adjoint_t<HB_MODEL_VARWAVE, 3>(op, q, lam, q_bar, c_bar, coeff, work, s);
    case HB_MODEL_MAXWELL:
      if (dim != 3) return fail(HB_ERR_UNSUPPORTED, "Maxwell adjoint: 3D only");
      return launch_adjoint_t<HB_MODEL_MAXWELL, 3>(op, q, lam, q_bar, c_bar, coeff, work, s);
    case HB_MODEL_MAXWELL_TM:
      return launch_adjoint_t<HB_MODEL_MAXWELL_TM, 2>(op, q, lam, q_bar, c_bar, coeff, work, s);
    case HB_MODEL_MAXWELL_TE:
      return launch_adjoint_t<HB_MODEL_MAXWELL_TE, 2>(op, q, lam, q_bar, c_bar, coeff, work, s);
    default:
      return fail(HB_ERR_INVALID_ARGUMENT, "unknown model id");
  }
}

}  // namespace hb
