// Over-integrated (quadrature) right-hand side of the variable-coefficient
// advection operator (hedge/models/advection.py:190-368), weak form:
//
//   rhs = M^-1 [ sum_x S^T_x,quad (v_x u) - int_faces F(w-, w+, n) phi ]
//
// with w = (u, v, c), c the element maximum of |v|^2 (ElementwiseMaxOperator
// of ptwise_dot(v, v)), and F the central, Lax-Friedrichs or upwind flux of
// advection.py:239-266.  The integrals are taken on the quadrature grid of
// the operator's degree (hedge/discretization/local.py:545-690): the volume
// integrand v_x u d(phi)/dx at the volume points
// (QuadratureStiffnessTOperator, operators.py:149-168 with the chain rule of
// mappers/__init__.py:1266-1410), the flux at the face points of every face
// (QuadratureInteriorFacesGridUpsampler + the quadrature face mass,
// operators.py:278-314, 593-631).  The inverse mass is folded into the
// projection matrices; |J| cancels against the element Jacobian of the
// integrals, and the face integrals carry Fscale = face Jacobian / |J|.
//
// One persistent CTA of 256 threads loops over batches of E elements:
//   A. stage u and v (all components) of the batch in shared memory
//      (coalesced), the geometry and the face table;
//   B. gather the other side's u and v at every face node (the matched
//      neighbour node, or the boundary data: u = given values or 0, v = this
//      side's trace); the element maxima c come from a pre-pass (LF only);
//   C. volume points: u_q, v_q by the interpolation matrix, then
//      g_r(q) = u_q sum_x (d r / d x) v_x,q; face points: both traces by the
//      face interpolation matrix, flux times Fscale;
//   D. node i: sum_r sum_q B_r[i, q] g_r(q) - sum_p L[i, p] flux_p, written
//      as the RHS or as the LSRK stage update
//      (hedge/timestep/runge_kutta.py:123-128).
// The element work is FP64 FMA on the CUDA cores, also for FP32 state
// vectors; the matrices sit in shared memory when they leave room for a
// batch, else they are read through L1.  The kernel is bound by its
// shared-memory loads, so each thread computes two volume points in C and
// one node of two elements in D (every matrix entry loaded once serves two
// products), and the rows of g_r have an odd stride so that the two
// elements a warp reads in D sit in different banks.
#include "common.cuh"

#include <algorithm>

namespace hb {

// T: the type the kernel computes and stages in; IO: the type of the state,
// residual and output vectors (the FP32 path: FP64 arithmetic on FP32
// vectors, since the weak form's volume and face integrals nearly cancel for
// smooth fields and FP32 sums of them miss the FP32 path's 1e-5 bound)
template <typename T, typename IO = T>
struct QuadArgs {
  int64_t K, nbatch, n_given;
  int np, nfp, nf, nperm, G, E, nq, nqf;
  const T* It;    // [np][nq]       nodal -> volume points, transposed
  const T* Bt;    // [dim][nq][np]  M^-1 (d phi / d r)^T W, transposed
  const T* Ft;    // [nf][nfp][nqf] face nodes -> face points, transposed
  const T* Lt;    // [nf*nqf][np]   M^-1 phi(face points)^T W_face, transposed
  const T* geo;
  const int2* conn;
  const int* fmask;
  const int* shuffle;
  const IO* q_in;
  IO* q_out;
  IO* res;
  IO* rhs_out;
  const double* vel;     // [dim][K*np]
  const double* bdry;    // given boundary values (BC_GIVEN faces)
  const double* elmax;   // [K] element maxima of |v|^2 (LF flux), else null
  double ra, rb, dt;
  int mode;              // 0: write rhs, 1: LSRK stage
  int flux_type;         // 0 central, 1 upwind, 2 LF
  int ops_in_smem;
  int* err;
};

struct QuadLayout {
  size_t oI, oB, oF, oL, ow, og, ox, ofl, ogeo, oc, oconn, ofm, osh, total;
};

__host__ __device__ inline size_t qalign16(size_t x) { return (x + 15) & ~size_t(15); }

__host__ __device__ inline QuadLayout quad_layout(int ts, int dim, int np, int nfp, int nf,
                                                  int nperm, int G, int E, int nq, int nqf,
                                                  int ops) {
  QuadLayout L;
  const int nv = 1 + dim;
  size_t o = 0;
  L.oI = o;    o = qalign16(o + (size_t)ts * np * nq * ops);
  L.oB = o;    o = qalign16(o + (size_t)ts * dim * nq * np * ops);
  L.oF = o;    o = qalign16(o + (size_t)ts * nf * nfp * nqf * ops);
  L.oL = o;    o = qalign16(o + (size_t)ts * nf * nqf * np * ops);
  L.ow = o;    o = qalign16(o + (size_t)ts * nv * E * np);
  L.og = o;    o = qalign16(o + (size_t)ts * dim * E * (nq | 1));
  L.ox = o;    o = qalign16(o + (size_t)ts * E * nf * nv * nfp);
  L.ofl = o;   o = qalign16(o + (size_t)ts * E * nf * nqf);
  L.ogeo = o;  o = qalign16(o + (size_t)ts * E * G);
  L.oc = o;    o = qalign16(o + (size_t)ts * E * (nf + 1));
  L.oconn = o; o = qalign16(o + sizeof(int2) * E * nf);
  L.ofm = o;   o = qalign16(o + sizeof(int) * nf * nfp);
  L.osh = o;   o = qalign16(o + sizeof(int) * nperm * nfp);
  L.total = o;
  return L;
}

__device__ __forceinline__ void qflag(int* err, int code) { atomicCAS(err, 0, code); }

// Element maxima of |v|^2 over the element's nodes (perform_elwise_max of
// ptwise_dot(v, v), volume_operators.hpp:356-369), FP64.
__global__ void elmax_kernel(int64_t K, int np, int dim, const double* __restrict__ vel,
                             double* __restrict__ out) {
  const int64_t Knp = K * np;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < K;
       e += (int64_t)gridDim.x * blockDim.x) {
    double m = 0.0;
    for (int i = 0; i < np; ++i) {
      double s = 0.0;
      for (int x = 0; x < dim; ++x) {
        const double v = vel[x * Knp + e * np + i];
        s += v * v;
      }
      m = i == 0 ? s : (s > m ? s : m);
    }
    out[e] = m;
  }
}

template <int DIM, typename T, typename IO>
__global__ void __launch_bounds__(256) rhs_quad_kernel(QuadArgs<T, IO> a) {
  constexpr int NV = 1 + DIM;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int np = a.np, nfp = a.nfp, nf = a.nf, E = a.E, G = a.G;
  const int nq = a.nq, nqf = a.nqf, nfq = nf * nqf;
  // an odd row stride of the volume-point integrands: the rows of two
  // elements that one warp reads in the projection start in different banks
  const int nqs = nq | 1;
  const QuadLayout L = quad_layout((int)sizeof(T), DIM, np, nfp, nf, a.nperm, G, E, nq, nqf,
                                   a.ops_in_smem);
  const T* sI = a.ops_in_smem ? reinterpret_cast<const T*>(smem_raw + L.oI) : a.It;
  const T* sB = a.ops_in_smem ? reinterpret_cast<const T*>(smem_raw + L.oB) : a.Bt;
  const T* sF = a.ops_in_smem ? reinterpret_cast<const T*>(smem_raw + L.oF) : a.Ft;
  const T* sL = a.ops_in_smem ? reinterpret_cast<const T*>(smem_raw + L.oL) : a.Lt;
  T* sw = reinterpret_cast<T*>(smem_raw + L.ow);      // [NV][E][np]: u, v_0 ..
  T* sg = reinterpret_cast<T*>(smem_raw + L.og);      // [DIM][E][nqs]
  T* sx = reinterpret_cast<T*>(smem_raw + L.ox);      // [E][nf][NV][nfp] other side
  T* sfl = reinterpret_cast<T*>(smem_raw + L.ofl);    // [E][nf*nqf]
  T* sgeo = reinterpret_cast<T*>(smem_raw + L.ogeo);  // [E][G]
  T* sc = reinterpret_cast<T*>(smem_raw + L.oc);      // [E][nf+1]: own c, other side's c
  int2* sconn = reinterpret_cast<int2*>(smem_raw + L.oconn);
  int* sfm = reinterpret_cast<int*>(smem_raw + L.ofm);
  int* ssh = reinterpret_cast<int*>(smem_raw + L.osh);

  const int tid = threadIdx.x, nthr = blockDim.x;
  if (a.ops_in_smem) {
    T* w;
    w = reinterpret_cast<T*>(smem_raw + L.oI);
    for (int x = tid; x < np * nq; x += nthr) w[x] = a.It[x];
    w = reinterpret_cast<T*>(smem_raw + L.oB);
    for (int x = tid; x < DIM * nq * np; x += nthr) w[x] = a.Bt[x];
    w = reinterpret_cast<T*>(smem_raw + L.oF);
    for (int x = tid; x < nf * nfp * nqf; x += nthr) w[x] = a.Ft[x];
    w = reinterpret_cast<T*>(smem_raw + L.oL);
    for (int x = tid; x < nfq * np; x += nthr) w[x] = a.Lt[x];
  }
  for (int x = tid; x < nf * nfp; x += nthr) sfm[x] = a.fmask[x];
  for (int x = tid; x < a.nperm * nfp; x += nthr) ssh[x] = a.shuffle[x];
  const int64_t Knp = a.K * np;
  const bool lf = a.flux_type == 2;

  for (int64_t batch = blockIdx.x; batch < a.nbatch; batch += gridDim.x) {
    const int64_t el0 = batch * E;
    const int ne = (int)((a.K - el0) < E ? (a.K - el0) : E);
    __syncthreads();  // previous batch done with the shared buffers
    // ---- A: stage u, v, geometry, face table ----
    for (int x = tid; x < ne * np; x += nthr) {
      sw[x] = (T)a.q_in[el0 * np + x];
#pragma unroll
      for (int c = 0; c < DIM; ++c)
        sw[((1 + c) * E) * np + x] = T(a.vel[c * Knp + el0 * np + x]);
    }
    for (int x = tid; x < ne * G; x += nthr) sgeo[x] = a.geo[el0 * G + x];
    for (int x = tid; x < ne * nf; x += nthr) sconn[x] = a.conn[el0 * nf + x];
    __syncthreads();

    // ---- B: the other side's u, v at every face node; element maxima ----
    for (int it = tid; it < ne * nf * nfp; it += nthr) {
      const int e = it / (nf * nfp);
      const int rem = it - e * nf * nfp;
      const int f = rem / nfp;
      const int k = rem - f * nfp;
      const int2 cn = sconn[e * nf + f];
      T* dst = sx + ((e * nf + f) * NV) * nfp + k;
      T w[NV];
#pragma unroll
      for (int c = 0; c < NV; ++c) w[c] = T(0);
      if (cn.x >= 0) {
        const int nface = cn.y & 3, perm = cn.y >> 2;
        if (cn.x >= a.K || nface >= nf || perm < 0 || perm >= a.nperm) {
          qflag(a.err, cn.x >= a.K ? DEV_BAD_NEIGHBOUR : DEV_BAD_CODE);
        } else {
          const int64_t gi = (int64_t)cn.x * np + sfm[nface * nfp + ssh[perm * nfp + k]];
          w[0] = (T)a.q_in[gi];
#pragma unroll
          for (int c = 0; c < DIM; ++c) w[1 + c] = T(__ldg(a.vel + c * Knp + gi));
        }
      } else {
        const int lnode = sfm[f * nfp + k];
#pragma unroll
        for (int c = 0; c < DIM; ++c) w[1 + c] = sw[((1 + c) * E + e) * np + lnode];
        if (cn.y == HB_BC_GIVEN) {
          const int64_t bi = (int64_t)(-1 - cn.x) * nfp + k;
          if (a.bdry == nullptr || bi >= a.n_given)
            qflag(a.err, a.bdry == nullptr ? DEV_MISSING_INPUT : DEV_BAD_BDRY_INDEX);
          else
            w[0] = T(__ldg(a.bdry + bi));
        } else if (cn.y != HB_BC_DIRICHLET && cn.y != HB_BC_NONE) {
          qflag(a.err, DEV_BAD_CODE);
        }
      }
#pragma unroll
      for (int c = 0; c < NV; ++c) dst[c * nfp] = w[c];
    }
    if (lf) {
      for (int it = tid; it < ne * (nf + 1); it += nthr) {
        const int e = it / (nf + 1);
        const int j = it - e * (nf + 1);
        int64_t src = el0 + e;
        if (j > 0) {
          const int2 cn = sconn[e * nf + j - 1];
          if (cn.x >= 0 && cn.x < a.K) src = cn.x;
        }
        sc[it] = T(a.elmax[src]);
      }
    }
    __syncthreads();

    // ---- C: volume points ----
    // two volume points per thread (q and q + nqh): each staged nodal value
    // serves both
    const int nqh = (nq + 1) >> 1;
    for (int it = tid; it < ne * nqh; it += nthr) {
      const int e = it / nqh;
      const int q = it - e * nqh;
      const int q2 = q + nqh;
      const bool two = q2 < nq;
      const int q2c = two ? q2 : q;
      T acc[NV], acc2[NV];
#pragma unroll
      for (int c = 0; c < NV; ++c) acc[c] = acc2[c] = T(0);
#pragma unroll 4
      for (int j = 0; j < np; ++j) {
        const T I = sI[j * nq + q];
        const T I2 = sI[j * nq + q2c];
#pragma unroll
        for (int c = 0; c < NV; ++c) {
          const T w = sw[(c * E + e) * np + j];
          acc[c] += I * w;
          acc2[c] += I2 * w;
        }
      }
      const T* ge = sgeo + e * G;
#pragma unroll
      for (int r = 0; r < DIM; ++r) {
        T g = T(0), g2 = T(0);
#pragma unroll
        for (int x = 0; x < DIM; ++x) {
          g += ge[r * DIM + x] * acc[1 + x];
          g2 += ge[r * DIM + x] * acc2[1 + x];
        }
        sg[(r * E + e) * nqs + q] = acc[0] * g;
        if (two) sg[(r * E + e) * nqs + q2] = acc2[0] * g2;
      }
    }
    // ---- C: face points ----
    for (int it = tid; it < ne * nfq; it += nthr) {
      const int e = it / nfq;
      const int p = it - e * nfq;
      const int f = p / nqf;
      const int qq = p - f * nqf;
      const int2 cn = sconn[e * nf + f];
      T out = T(0);
      if (cn.x >= 0 || cn.y != HB_BC_NONE) {
        T wm[NV], wp[NV];
#pragma unroll
        for (int c = 0; c < NV; ++c) wm[c] = wp[c] = T(0);
        const T* xs = sx + ((e * nf + f) * NV) * nfp;
        for (int k = 0; k < nfp; ++k) {
          const T I = sF[(f * nfp + k) * nqf + qq];
          const int lnode = sfm[f * nfp + k];
#pragma unroll
          for (int c = 0; c < NV; ++c) {
            wm[c] += I * sw[(c * E + e) * np + lnode];
            wp[c] += I * xs[c * nfp + k];
          }
        }
        const T* gf = sgeo + e * G + DIM * DIM + f * (DIM + 1);
        T nvm = T(0), nvp = T(0);
#pragma unroll
        for (int x = 0; x < DIM; ++x) {
          nvm += gf[x] * wm[1 + x];
          nvp += gf[x] * wp[1 + x];
        }
        T fl;
        if (a.flux_type == 0) {
          fl = (wm[0] * nvm + wp[0] * nvp) * T(0.5);
        } else if (a.flux_type == 2) {
          const T cm = sc[e * (nf + 1)];
          const T cp = cn.x >= 0 ? sc[e * (nf + 1) + 1 + f] : cm;
          fl = T(0.5) * (nvm * wm[0] + nvp * wp[0]) -
               T(0.5) * (wp[0] - wm[0]) * (cm > cp ? cm : cp);
        } else {
          T navg = T(0);
#pragma unroll
          for (int x = 0; x < DIM; ++x) navg += gf[x] * (T(0.5) * (wm[1 + x] + wp[1 + x]));
          fl = navg > T(0) ? nvm * wm[0] : nvp * wp[0];
        }
        out = gf[DIM] * fl;
      }
      sfl[e * nfq + p] = out;
    }
    __syncthreads();

    // ---- D: projection, lift, output ----
    // two elements per thread (e and e + eh): each operator entry serves both
    const int eh = (ne + 1) >> 1;
    for (int it = tid; it < eh * np; it += nthr) {
      const int e = it / np;
      const int i = it - e * np;
      const int e2 = e + eh;
      const bool two = e2 < ne;
      const int e2c = two ? e2 : e;
      T acc = T(0), acc2 = T(0);
#pragma unroll
      for (int r = 0; r < DIM; ++r) {
        const T* gr = sg + (r * E + e) * nqs;
        const T* gr2 = sg + (r * E + e2c) * nqs;
        const T* br = sB + (size_t)r * nq * np + i;
#pragma unroll 4
        for (int q = 0; q < nq; ++q) {
          const T b = br[q * np];
          acc += b * gr[q];
          acc2 += b * gr2[q];
        }
      }
      const T* fe = sfl + e * nfq;
      const T* fe2 = sfl + e2c * nfq;
#pragma unroll 4
      for (int p = 0; p < nfq; ++p) {
        const T l = sL[p * np + i];
        acc -= l * fe[p];
        acc2 -= l * fe2[p];
      }
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        if (h == 1 && !two) break;
        const int ee = h ? e2 : e;
        const T v = h ? acc2 : acc;
        const int64_t node = (el0 + ee) * np + i;
        if (a.mode == 0) {
          a.rhs_out[node] = (IO)v;
        } else {
          const T rv = T(a.ra) * (T)a.res[node] + T(a.dt) * v;
          a.res[node] = (IO)rv;
          a.q_out[node] = (IO)(sw[ee * np + i] + T(a.rb) * rv);
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
template <typename T>
static size_t quad_smem(const Op* op, int E, int ops) {
  const Discr* d = op->d;
  return quad_layout((int)sizeof(T), d->dim, d->np, d->nfp, d->nfaces, d->nperm, d->G, E,
                     op->nq, op->nqf, ops).total;
}

template <int DIM, typename T, typename IO>
static hb_status quad_launch(Op* op, int mode, double ra, double rb, double dt,
                             const void* q_in, void* q_out, void* res, const double* vel,
                             const double* bdry, cudaStream_t s, bool configure) {
  auto kern = rhs_quad_kernel<DIM, T, IO>;
  Discr* d = op->d;
  if (configure) {
    int dev;
    HB_CUDA(cudaGetDevice(&dev));
    int max_optin = 0, sms = 0;
    HB_CUDA(cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    HB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    // a batch of about 256 / np elements (two elements' node per thread in
    // the output phase; twice that batch costs the third CTA per SM and ran
    // slower); the matrices in shared memory when a batch of at least a
    // quarter of that still fits beside them
    int E = std::max(1, 256 / d->np);
    int ops = 1;
    const int Emin = std::max(1, E / 4);
    if (quad_smem<T>(op, Emin, 1) > (size_t)max_optin) ops = 0;
    while (E > 1 && quad_smem<T>(op, E, ops) > (size_t)max_optin) --E;
    const size_t smem = quad_smem<T>(op, E, ops);
    if (smem > (size_t)max_optin)
      return fail(HB_ERR_UNSUPPORTED, "quadrature batch does not fit in shared memory");
    HB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    HB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, smem));
    if (per_sm < 1) return fail(HB_ERR_UNSUPPORTED, "quadrature kernel does not fit on an SM");
    const int64_t nbatch = (d->K + E - 1) / E;
    op->elems_per_block = E;
    op->ops_in_smem = ops;
    op->blocks_per_sm = per_sm;
    op->threads = 256;
    op->smem = smem;
    op->grid = (int)std::min<int64_t>(nbatch, (int64_t)sms * per_sm);
    return HB_OK;
  }
  if (op->mp.flux_type == 2) {
    const int grid = (int)std::min<int64_t>((d->K + 255) / 256, 148 * 8);
    elmax_kernel<<<grid, 256, 0, s>>>(d->K, d->np, d->dim, vel, op->elmax);
    HB_CUDA(cudaGetLastError());
  }
  QuadArgs<T, IO> a;
  a.K = d->K;
  a.E = op->elems_per_block;
  a.nbatch = (d->K + a.E - 1) / a.E;
  a.n_given = op->n_given;
  a.np = d->np; a.nfp = d->nfp; a.nf = d->nfaces; a.nperm = d->nperm; a.G = d->G;
  a.nq = op->nq; a.nqf = op->nqf;
  static_assert(sizeof(T) == 8, "the quadrature kernel computes in FP64");
  const T* ops = op->quad64;
  const size_t nI = (size_t)d->np * op->nq, nB = (size_t)d->dim * op->nq * d->np;
  const size_t nF = (size_t)d->nfaces * d->nfp * op->nqf;
  a.It = ops;
  a.Bt = ops + nI;
  a.Ft = ops + nI + nB;
  a.Lt = ops + nI + nB + nF;
  a.geo = d->geo;
  a.conn = op->conn; a.fmask = d->fmask; a.shuffle = d->shuffle;
  a.q_in = static_cast<const IO*>(q_in);
  a.q_out = static_cast<IO*>(q_out);
  a.res = static_cast<IO*>(res);
  a.rhs_out = static_cast<IO*>(q_out);
  a.vel = vel; a.bdry = bdry;
  a.elmax = op->mp.flux_type == 2 ? op->elmax : nullptr;
  a.ra = ra; a.rb = rb; a.dt = dt; a.mode = mode;
  a.flux_type = op->mp.flux_type;
  a.ops_in_smem = op->ops_in_smem;
  a.err = op->err_flag;
  kern<<<op->grid, op->threads, op->smem, s>>>(a);
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

template <typename T, typename IO>
static hb_status quad_dispatch(Op* op, int mode, double ra, double rb, double dt,
                               const void* q_in, void* q_out, void* res, const double* vel,
                               const double* bdry, cudaStream_t s, bool configure) {
  if (op->d->dim == 2)
    return quad_launch<2, T, IO>(op, mode, ra, rb, dt, q_in, q_out, res, vel, bdry, s,
                                 configure);
  return quad_launch<3, T, IO>(op, mode, ra, rb, dt, q_in, q_out, res, vel, bdry, s,
                               configure);
}

hb_status prepare_quad(Op* op) {
  if (op->precision == HB_PREC_FP32)
    return quad_dispatch<double, float>(op, 0, 0, 0, 0, nullptr, nullptr, nullptr, nullptr,
                                        nullptr, 0, true);
  return quad_dispatch<double, double>(op, 0, 0, 0, 0, nullptr, nullptr, nullptr, nullptr,
                                       nullptr, 0, true);
}

hb_status launch_quad(Op* op, int mode, double ra, double rb, double dt, const void* q_in,
                      void* q_out, void* res, const double* vel, const double* bdry,
                      cudaStream_t s) {
  if (op->precision == HB_PREC_FP32)
    return quad_dispatch<double, float>(op, mode, ra, rb, dt, q_in, q_out, res, vel, bdry, s,
                                        false);
  return quad_dispatch<double, double>(op, mode, ra, rb, dt, q_in, q_out, res, vel, bdry, s,
                                       false);
}

}  // namespace hb
