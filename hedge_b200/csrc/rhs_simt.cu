// CUDA-core (FP64 / FP32) fused DG right-hand side and LSRK stage.
//
// One persistent CTA loops over batches of E elements.  Per batch:
//   1. stage the batch's state (all F fields), geometry and face table in
//      shared memory (coalesced: each field's batch slice is contiguous);
//   2. thread (e, i) computes d_r q_f at node i for all r, f from the
//      shared-memory operators D_r (transposed, so node i's column reads are
//      bank-conflict free), applies the chain rule with the element's
//      d r / d x, and forms the model's volume term (hedge jit diff loop,
//      jit/diff.py:137-175, plus the chain-rule vector expression);
//   3. the same threads evaluate the numerical flux at the element's
//      Nf*Nfp face points: int value from shared memory, ext value gathered
//      from the neighbour's volume node (global, L2-resident) or built from
//      the boundary condition, times Fscale = Fjac / J (jit/flux.py:311-353,
//      429-472);
//   4. after a barrier, thread (e, i) applies LIFT = M^-1 E to the staged
//      face fluxes (jit/lift.py:110-141 with the inverse mass folded in,
//      jit/__init__.py:501-519) and writes either the RHS or the LSRK stage
//      update res = a res + dt rhs, q_out = q_in + b res
//      (hedge/timestep/runge_kutta.py:123-128).
// Operators stay resident in shared memory for the CTA's lifetime.
#include "common.cuh"
#include "models.cuh"

#include <algorithm>

namespace hb {

template <typename T, typename S>
struct SimtArgs {
  int64_t K, nbatch, n_given;
  int64_t e_begin, e_end;   // the elements this launch updates (of K)
  int np, nfp, nf, nperm, G, E;
  const T* dmats_t;
  const T* lift_t;
  const T* geo;
  const int2* conn;
  const int* fmask;
  const int* shuffle;
  const S* q_in;
  S* q_out;
  S* res;
  S* rhs_out;
  const double* coeff;
  const double* bdry;
  const double* source;
  const S* halo;            // [n_halo * nfp][F] ext values of halo faces
  const double* halo_c;     // [n_halo * nfp] ext c (var-c wave)
  int64_t n_halo;
  double ra, rb, dt;
  int mode;  // 0: write rhs, 1: LSRK stage
  int ops_in_smem;  // operators staged in shared memory (else read via L1)
  ModelParams mp;
  int* err;
};

__device__ __forceinline__ void flag(int* err, int code) {
  atomicCAS(err, 0, code);
}

// The ext-side volume node of face point (nbr code, face node k), as the
// reference's ext index list gives it: fmask[nbr_face][shuffle[perm][k]].
__device__ __forceinline__ int ext_node(int code, int k, int nfp, int nf,
                                        int nperm, const int* fmask,
                                        const int* shuffle, bool& ok) {
  const int nface = code & 3;
  const int perm = code >> 2;
  ok = (nface < nf) && (perm >= 0) && (perm < nperm);
  if (!ok) return 0;
  return fmask[nface * nfp + shuffle[perm * nfp + k]];
}

template <typename T>
__device__ __forceinline__ T ldg_as(const double* p) { return T(__ldg(p)); }
template <typename T>
__device__ __forceinline__ T ldg_as(const float* p) { return T(__ldg(p)); }

// Shared-memory carve-up of the SIMT kernel (16-byte aligned sections).
struct SimtLayout {
  size_t oD, oL, oq, ofl, ogeo, oc, oconn, ofm, osh, total;
};

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

__host__ __device__ inline SimtLayout simt_layout(int tsize, int dim, int np, int nfp,
                                                  int nf, int nperm, int G, int E,
                                                  int F, int C, int ops) {
  SimtLayout L;
  const int nfpt = nf * nfp;
  size_t o = 0;
  L.oD = o;    o = align16(o + (size_t)tsize * dim * np * np * ops);
  L.oL = o;    o = align16(o + (size_t)tsize * nfpt * np * ops);
  L.oq = o;    o = align16(o + (size_t)tsize * F * E * np);
  L.ofl = o;   o = align16(o + (size_t)tsize * F * E * nfpt);
  L.ogeo = o;  o = align16(o + (size_t)tsize * E * G);
  L.oc = o;    o = align16(o + (size_t)tsize * C * E * np);
  L.oconn = o; o = align16(o + sizeof(int2) * E * nf);
  L.ofm = o;   o = align16(o + sizeof(int) * nfpt);
  L.osh = o;   o = align16(o + sizeof(int) * nperm * nfp);
  L.total = o;
  return L;
}

template <int MODEL, int DIM, typename T, typename S>
__global__ void __launch_bounds__(256) rhs_simt_kernel(SimtArgs<T, S> a) {
  constexpr int F = Traits<MODEL, DIM>::F;
  constexpr int C = Traits<MODEL, DIM>::COEFF;
  constexpr int NA = F + C;
  extern __shared__ __align__(16) unsigned char smem_raw[];

  const int np = a.np, nfp = a.nfp, nf = a.nf, E = a.E, G = a.G;
  const int nfpt = nf * nfp;
  const SimtLayout L = simt_layout((int)sizeof(T), DIM, np, nfp, nf, a.nperm, G, E, F, C,
                                   a.ops_in_smem);
  const T* sD = a.ops_in_smem ? reinterpret_cast<T*>(smem_raw + L.oD) : a.dmats_t;
  const T* sL = a.ops_in_smem ? reinterpret_cast<T*>(smem_raw + L.oL) : a.lift_t;
  T* sq = reinterpret_cast<T*>(smem_raw + L.oq);
  T* sfl = reinterpret_cast<T*>(smem_raw + L.ofl);
  T* sgeo = reinterpret_cast<T*>(smem_raw + L.ogeo);
  T* sc = reinterpret_cast<T*>(smem_raw + L.oc);
  int2* sconn = reinterpret_cast<int2*>(smem_raw + L.oconn);
  int* sfm = reinterpret_cast<int*>(smem_raw + L.ofm);
  int* ssh = reinterpret_cast<int*>(smem_raw + L.osh);

  const int tid = threadIdx.x;
  const int nthr = blockDim.x;
  if (a.ops_in_smem) {
    T* wD = reinterpret_cast<T*>(smem_raw + L.oD);
    T* wL = reinterpret_cast<T*>(smem_raw + L.oL);
    for (int x = tid; x < DIM * np * np; x += nthr) wD[x] = a.dmats_t[x];
    for (int x = tid; x < nfpt * np; x += nthr) wL[x] = a.lift_t[x];
  }
  for (int x = tid; x < nfpt; x += nthr) sfm[x] = a.fmask[x];
  for (int x = tid; x < a.nperm * nfp; x += nthr) ssh[x] = a.shuffle[x];

  const int e = tid / np;
  const int i = tid - e * np;
  const int64_t Knp = a.K * np;
  // Maxwell with variable material: coeff = [eps | mu], [2][K*Np] FP64
  // (em.py:38-100, 309-371): per-node divisors, both sides' impedances in
  // the flux, the local impedance in the absorbing condition
  constexpr bool MAXW = IsMaxwell<MODEL>::value;
  const bool varmat = MAXW && a.coeff != nullptr;

  for (int64_t batch = blockIdx.x; batch < a.nbatch; batch += gridDim.x) {
    const int64_t el0 = a.e_begin + batch * E;
    const int ne = (int)((a.e_end - el0) < E ? (a.e_end - el0) : E);
    __syncthreads();  // previous batch done with shared buffers
    for (int f = 0; f < F; ++f) {
      const S* src = a.q_in + f * Knp + el0 * np;
      T* dst = sq + f * E * np;
      for (int x = tid; x < ne * np; x += nthr) dst[x] = T(src[x]);
    }
    for (int x = tid; x < ne * G; x += nthr) sgeo[x] = a.geo[el0 * G + x];
    for (int x = tid; x < ne * nf; x += nthr) sconn[x] = a.conn[el0 * nf + x];
    if constexpr (C != 0) {
      for (int x = tid; x < ne * np; x += nthr) sc[x] = T(a.coeff[el0 * np + x]);
    }
    __syncthreads();

    const bool active = e < ne;
    T vol[F];
    if (active) {
      // ---- volume: reference derivatives, chain rule, model terms ----
      T dr[DIM][F];
#pragma unroll
      for (int r = 0; r < DIM; ++r)
#pragma unroll
        for (int f = 0; f < F; ++f) dr[r][f] = T(0);
      const T* qe = sq + e * np;
#pragma unroll 4
      for (int j = 0; j < np; ++j) {
        T d[DIM];
#pragma unroll
        for (int r = 0; r < DIM; ++r) d[r] = sD[(r * np + j) * np + i];
#pragma unroll
        for (int f = 0; f < F; ++f) {
          const T u = qe[f * E * np + j];
#pragma unroll
          for (int r = 0; r < DIM; ++r) dr[r][f] += d[r] * u;
        }
      }
      const T* ge = sgeo + e * G;
      T g[DIM][F];
#pragma unroll
      for (int x = 0; x < DIM; ++x)
#pragma unroll
        for (int f = 0; f < F; ++f) {
          T s = T(0);
#pragma unroll
          for (int r = 0; r < DIM; ++r) s += ge[r * DIM + x] * dr[r][f];
          g[x][f] = s;
        }
      const T cnode = C ? sc[e * np + i] : T(0);
      model_volume<MODEL, DIM, T>(a.mp, g, cnode, vol);
      const int64_t el_base = (el0 + e) * np;

      // ---- surface: flux at this thread's face points ----
      for (int p = i; p < nfpt; p += np) {
        const int face = p / nfp;
        const int k = p - face * nfp;
        const int lnode = sfm[p];
        T uM[NA], uP[NA], n[DIM], fl[F];
        if constexpr (C != 0) uM[0] = sc[e * np + lnode];
#pragma unroll
        for (int f = 0; f < F; ++f) uM[C + f] = qe[f * E * np + lnode];
        const T* gf = ge + DIM * DIM + face * (DIM + 1);
#pragma unroll
        for (int x = 0; x < DIM; ++x) n[x] = gf[x];
        const T fscale = gf[DIM];
        const int2 cn = sconn[e * nf + face];
        bool have = true;
        bool bdry = false;
        // variable material: interior and exterior impedances (the exterior
        // side's at the matched neighbour node; the interior one on
        // boundary faces)
        T Zi = T(1), Ze = T(1);
        if (varmat) {
          const int64_t gm = el_base + lnode;
          Zi = sqrt(T(a.coeff[Knp + gm]) / T(a.coeff[gm]));
          Ze = Zi;
        }
        if (cn.x >= a.K) {
          if (varmat) {
            // the halo carries no material values
            flag(a.err, DEV_MISSING_INPUT);
            have = false;
          }
          // neighbour on another partition: ext values from the halo buffer
          const int64_t h = (int64_t)cn.x - a.K;
          if (h >= a.n_halo || a.halo == nullptr) {
            flag(a.err, DEV_BAD_NEIGHBOUR);
            have = false;
          } else {
            const int64_t hi = h * nfp + k;
            if constexpr (C != 0) uP[0] = T(a.halo_c[hi]);
#pragma unroll
            for (int f = 0; f < F; ++f) uP[C + f] = T(a.halo[hi * F + f]);
          }
        } else if (cn.x >= 0) {
          bool ok;
          const int nn = ext_node(cn.y, k, nfp, nf, a.nperm, sfm, ssh, ok);
          if (!ok) {
            flag(a.err, DEV_BAD_CODE);
            have = false;
          } else {
            const int64_t gi = (int64_t)cn.x * np + nn;
            if constexpr (C != 0) uP[0] = T(__ldg(a.coeff + gi));
#pragma unroll
            for (int f = 0; f < F; ++f) uP[C + f] = ldg_as<T>(a.q_in + f * Knp + gi);
            if (varmat) Ze = sqrt(T(__ldg(a.coeff + Knp + gi)) / T(__ldg(a.coeff + gi)));
          }
        } else {
          bdry = true;
          T given = T(0);
          if (cn.y == HB_BC_GIVEN) {
            const int64_t bi = (int64_t)(-1 - cn.x) * nfp + k;
            if (a.bdry == nullptr || bi >= a.n_given) {
              flag(a.err, a.bdry == nullptr ? DEV_MISSING_INPUT : DEV_BAD_BDRY_INDEX);
              have = false;
            } else {
              given = T(__ldg(a.bdry + bi));
            }
          }
          if (have) {
            ModelParams mpl = a.mp;
            if (varmat) {
              mpl.Z = (double)Zi;
              mpl.Y = 1.0 / (double)Zi;
            }
            have = model_bc<MODEL, DIM, T>(mpl, cn.y, uM, n, given, uP);
          }
          if constexpr (MAXW) {
            // incident data d (em.py:289-307): exterior state -d, field f's
            // values at bdry[f * n_given + node]; no data: zero exterior
            if (have && cn.y == HB_BC_INCIDENT && a.bdry != nullptr) {
              const int64_t bi = (int64_t)(-1 - cn.x) * nfp + k;
              if (bi >= a.n_given) {
                flag(a.err, DEV_BAD_BDRY_INDEX);
                have = false;
              } else {
#pragma unroll
                for (int f = 0; f < F; ++f) uP[f] = -T(__ldg(a.bdry + f * a.n_given + bi));
              }
            }
          }
        }
        T* dst = sfl + e * nfpt + p;
        if (have) {
          if (varmat) {
            if constexpr (MAXW) maxwell_flux_var<MODEL, DIM, T>(a.mp, bdry, uM, uP, n, Zi, Ze, fl);
          } else {
            model_flux<MODEL, DIM, T>(a.mp, bdry, uM, uP, n, fl);
          }
#pragma unroll
          for (int f = 0; f < F; ++f) dst[f * E * nfpt] = fscale * fl[f];
        } else {
#pragma unroll
          for (int f = 0; f < F; ++f) dst[f * E * nfpt] = T(0);
        }
      }
    }
    __syncthreads();

    if (active) {
      // ---- lift and output ----
      T acc[F];
#pragma unroll
      for (int f = 0; f < F; ++f) acc[f] = T(0);
      const T* fe = sfl + e * nfpt;
#pragma unroll 4
      for (int p = 0; p < nfpt; ++p) {
        const T l = sL[p * np + i];
#pragma unroll
        for (int f = 0; f < F; ++f) acc[f] += l * fe[f * E * nfpt + p];
      }
      const int64_t node = (el0 + e) * np + i;
      ModelParams mpn = a.mp;
      if (varmat) {
        // the material divisor at this node
        mpn.eps = a.coeff[node];
        mpn.mu = a.coeff[Knp + node];
      }
#pragma unroll
      for (int f = 0; f < F; ++f) {
        const int64_t si = model_src_index<MODEL>(f, node, Knp);
        const T src = (a.source && si >= 0) ? T(a.source[si]) : T(0);
        const T r = model_finish<MODEL, DIM, T>(mpn, f, vol[f], acc[f], src);
        const int64_t idx = f * Knp + node;
        if (a.mode == 0) {
          a.rhs_out[idx] = S(r);
        } else {
          const T rv = T(a.ra) * T(a.res[idx]) + T(a.dt) * r;
          a.res[idx] = S(rv);
          a.q_out[idx] = S(sq[f * E * np + e * np + i] + T(a.rb) * rv);
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
template <typename T>
static size_t simt_smem(const Op* op, int E, int ops) {
  const Discr* d = op->d;
  const int C = op->model == HB_MODEL_VARWAVE ? 1 : 0;
  return simt_layout((int)sizeof(T), d->dim, d->np, d->nfp, d->nfaces, d->nperm,
                     d->G, E, op->F, C, ops).total;
}

template <int MODEL, int DIM, typename T, typename S>
static hb_status launch_one(Op* op, int mode, double ra, double rb, double dt,
                            const void* q_in, void* q_out, void* res,
                            const double* coeff, const double* bdry,
                            const double* source, int64_t e0, int64_t e1, cudaStream_t s,
                            bool configure) {
  auto kern = rhs_simt_kernel<MODEL, DIM, T, S>;
  Discr* d = op->d;
  if (configure) {
    int E = 256 / d->np;
    if (E < 1) E = 1;
    int dev;
    HB_CUDA(cudaGetDevice(&dev));
    int max_optin = 0;
    HB_CUDA(cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    // operators in shared memory when they leave room for two CTAs per SM
    int ops = simt_smem<T>(op, E, 1) * 2 <= (size_t)max_optin ? 1 : 0;
    size_t smem = simt_smem<T>(op, E, ops);
    while (E > 1 && smem > (size_t)max_optin) {
      --E;
      smem = simt_smem<T>(op, E, ops);
    }
    op->ops_in_smem = ops;
    if (smem > (size_t)max_optin)
      return fail(HB_ERR_UNSUPPORTED, "element too large for the shared-memory kernel");
    HB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int threads = ((E * d->np + 31) / 32) * 32;
    int per_sm = 0;
    HB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem));
    if (per_sm < 1)
      return fail(HB_ERR_UNSUPPORTED, "kernel does not fit on an SM");
    int sms = 0;
    HB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int64_t nbatch = (d->K + E - 1) / E;
    op->elems_per_block = E;
    op->blocks_per_sm = per_sm;
    op->threads = threads;
    op->smem = smem;
    op->grid = (int)std::min<int64_t>(nbatch, (int64_t)sms * per_sm);
    return HB_OK;
  }
  SimtArgs<T, S> a;
  a.K = d->K;
  a.e_begin = e0;
  a.e_end = e1;
  a.E = op->elems_per_block;
  a.nbatch = (e1 - e0 + a.E - 1) / a.E;
  a.n_given = op->n_given;
  a.np = d->np; a.nfp = d->nfp; a.nf = d->nfaces; a.nperm = d->nperm; a.G = d->G;
  if constexpr (sizeof(T) == 8) {
    a.dmats_t = d->dmats_t; a.lift_t = d->lift_t; a.geo = d->geo;
  } else {
    a.dmats_t = d->dmats_t32; a.lift_t = d->lift_t32; a.geo = d->geo32;
  }
  a.conn = op->conn; a.fmask = d->fmask; a.shuffle = d->shuffle;
  a.q_in = static_cast<const S*>(q_in);
  a.q_out = static_cast<S*>(q_out);
  a.res = static_cast<S*>(res);
  a.rhs_out = static_cast<S*>(q_out);
  a.coeff = coeff; a.bdry = bdry; a.source = source;
  a.halo = static_cast<const S*>(op->halo);
  a.halo_c = op->halo_c;
  a.n_halo = op->n_halo;
  a.ra = ra; a.rb = rb; a.dt = dt; a.mode = mode;
  a.ops_in_smem = op->ops_in_smem;
  a.mp = op->mp;
  a.err = op->err_flag;
  kern<<<(unsigned)std::min<int64_t>(op->grid, a.nbatch), op->threads, op->smem, s>>>(a);
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

template <typename T, typename S>
static hb_status dispatch(Op* op, int mode, double ra, double rb, double dt,
                          const void* q_in, void* q_out, void* res,
                          const double* coeff, const double* bdry,
                          const double* source, int64_t e0, int64_t e1, cudaStream_t s,
                          bool configure) {
  const int dim = op->d->dim;
#define HB_CASE(M, D)                                                          \
  if (op->model == M && dim == D)                                              \
    return launch_one<M, D, T, S>(op, mode, ra, rb, dt, q_in, q_out, res,      \
                                  coeff, bdry, source, e0, e1, s, configure);
  HB_CASE(HB_MODEL_ADVECTION, 2)
  HB_CASE(HB_MODEL_ADVECTION, 3)
  HB_CASE(HB_MODEL_WAVE, 2)
  HB_CASE(HB_MODEL_WAVE, 3)
  HB_CASE(HB_MODEL_VARWAVE, 2)
  HB_CASE(HB_MODEL_VARWAVE, 3)
  HB_CASE(HB_MODEL_MAXWELL, 3)
  HB_CASE(HB_MODEL_MAXWELL_TM, 2)
  HB_CASE(HB_MODEL_MAXWELL_TE, 2)
#undef HB_CASE
  return fail(HB_ERR_UNSUPPORTED, "model/dimension combination not built");
}

hb_status prepare_simt(Op* op) {
  if (op->precision == HB_PREC_FP32)
    return dispatch<float, float>(op, 0, 0, 0, 0, nullptr, nullptr, nullptr,
                                  nullptr, nullptr, nullptr, 0, op->d->K, 0, true);
  return dispatch<double, double>(op, 0, 0, 0, 0, nullptr, nullptr, nullptr,
                                  nullptr, nullptr, nullptr, 0, op->d->K, 0, true);
}

hb_status launch_simt(Op* op, int mode, double ra, double rb, double dt,
                      const void* q_in, void* q_out, void* res,
                      const double* coeff, const double* bdry,
                      const double* source, int64_t e0, int64_t e1, cudaStream_t s) {
  if (op->precision == HB_PREC_FP32)
    return dispatch<float, float>(op, mode, ra, rb, dt, q_in, q_out, res, coeff,
                                  bdry, source, e0, e1, s, false);
  return dispatch<double, double>(op, mode, ra, rb, dt, q_in, q_out, res, coeff,
                                  bdry, source, e0, e1, s, false);
}

// ---------------------------------------------------------------------------
// gather-map expansion (hb_gather_map) and linear combination (hb_lincomb)

__global__ void gather_map_kernel(int64_t K, int np, int nfp, int nf, int nperm,
                                  const int2* conn, const int* fmask,
                                  const int* shuffle, int64_t* int_idx,
                                  int64_t* ext_idx, int* err) {
  const int64_t total = K * nf * nfp;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t ef = t / nfp;
    const int k = (int)(t - ef * nfp);
    const int64_t e = ef / nf;
    const int face = (int)(ef - e * nf);
    int_idx[t] = e * np + fmask[face * nfp + k];
    const int2 cn = conn[ef];
    if (cn.x >= 0) {
      bool ok;
      const int nn = ext_node(cn.y, k, nfp, nf, nperm, fmask, shuffle, ok);
      if (!ok || cn.x >= K) flag(err, DEV_BAD_CODE);
      ext_idx[t] = ok ? (int64_t)cn.x * np + nn : INT64_MIN;
    } else {
      ext_idx[t] = -1 - ((int64_t)(-1 - cn.x) * nfp + k);
    }
  }
}

template <typename S>
__global__ void lincomb_kernel(int64_t n, S a, const S* __restrict__ x, S b,
                               const S* __restrict__ y, S* __restrict__ out) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x)
    out[t] = a * x[t] + b * y[t];
}

hb_status launch_gather_map(Op* op, int64_t* int_idx, int64_t* ext_idx,
                            cudaStream_t s) {
  Discr* d = op->d;
  const int64_t total = d->K * d->nfaces * d->nfp;
  const int grid = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
  gather_map_kernel<<<grid, 256, 0, s>>>(d->K, d->np, d->nfp, d->nfaces, d->nperm,
                                         op->conn, d->fmask, d->shuffle, int_idx,
                                         ext_idx, op->err_flag);
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

hb_status launch_lincomb(int64_t n, int dtype, double a, const void* x, double b,
                         const void* y, void* out, cudaStream_t s) {
  const int grid = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
  if (n == 0) return HB_OK;
  if (dtype == 0)
    lincomb_kernel<double><<<grid, 256, 0, s>>>(n, a, (const double*)x, b,
                                                (const double*)y, (double*)out);
  else
    lincomb_kernel<float><<<grid, 256, 0, s>>>(n, (float)a, (const float*)x, (float)b,
                                               (const float*)y, (float*)out);
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

// ---------------------------------------------------------------------------
// halo exchange pack: dst[j][f] = src[f][idx[j]] (thread per (j, f) pair)
template <typename T>
__global__ void pack_kernel(int64_t n, int nfields, int64_t field_stride,
                            const int64_t* __restrict__ idx, const T* __restrict__ src,
                            T* __restrict__ dst) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * nfields) return;
  const int64_t j = t / nfields;
  const int f = (int)(t - j * nfields);
  dst[t] = src[f * field_stride + idx[j]];
}

hb_status launch_pack(int64_t n, int dtype, int nfields, int64_t field_stride,
                      const int64_t* idx, const void* src, void* dst, cudaStream_t s) {
  const int64_t total = n * nfields;
  const unsigned grid = (unsigned)((total + 255) / 256);
  if (dtype == 0)
    pack_kernel<double><<<grid, 256, 0, s>>>(n, nfields, field_stride, idx,
                                             static_cast<const double*>(src),
                                             static_cast<double*>(dst));
  else
    pack_kernel<float><<<grid, 256, 0, s>>>(n, nfields, field_stride, idx,
                                            static_cast<const float*>(src),
                                            static_cast<float*>(dst));
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

}  // namespace hb
