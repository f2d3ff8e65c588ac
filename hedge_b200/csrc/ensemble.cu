// Batched ensemble: one persistent launch advances an LSRK stage of many
// independent discretizations (meshes of uneven size and order, advection
// or wave), each with its own operator, geometry, face table, model
// parameters and time step.
//
// The host flattens the members into a tile list (member, first element,
// element count, tile capacity E); tiles are sorted by (order, model) so
// that a CTA's consecutive tiles mostly share operators, which then stay in
// shared memory.  A tile runs the same element-local algorithm as the
// single-mesh CUDA-core kernel -- reference derivatives, chain rule and
// model volume terms (jit/diff.py:137-175), numerical fluxes at the face
// points with the neighbour trace gathered from global memory
// (jit/flux.py:311-353, 429-472), LIFT with the inverse mass folded in
// (jit/lift.py:110-141) -- in FP32, then the LSRK stage in FP64:
//   res = a res + dt R(q_src)   (FP64 residual)
//   q_dst = q_src + b res       (FP64 arithmetic, stored FP32)
// (hedge/timestep/runge_kutta.py:123-128).  q_src / q_dst alternate between
// each member's two state buffers by the stage's parity.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "models.cuh"

namespace hb {

hb_status ensure_fp32(Discr* d);

namespace {

constexpr int ENS_THREADS = 256;
constexpr int ENS_MAX_F = 4;   // wave in 3D

struct EnsInst {
  int model, F, dim, np, nfp, nperm, G;
  int64_t K;
  const float* dmats_t;   // [dim][np(j)][np(i)]
  const float* lift_t;    // [nfpt][np]
  const float* geo;       // [K][G]
  const int2* conn;       // [K][nf]
  const int* fmask;
  const int* shuffle;
  float* q[2];
  double* res;
  double dt;
  ModelParams mp;
};

struct EnsTile {
  int inst, E;
  int64_t el0;
  int ne, pad;
};

struct EnsLayout {
  size_t oD, oL, oq, ov, ofl, ogeo, oconn, ofm, osh, total;
};

__host__ __device__ inline size_t a16(size_t x) { return (x + 15) & ~size_t(15); }

// shared-memory carve-up: the largest operator (np, nfpt), tile state
// (E*np, E*nfpt) and tile element count E over the batch's members
struct EnsSizes {
  int dim = 0, np = 0, nfpt = 0, enp = 0, enfpt = 0, e = 0, permnfp = 0;
};

__host__ __device__ inline EnsLayout ens_layout(const EnsSizes& z) {
  EnsLayout L;
  const int nf = z.dim + 1, G = z.dim * z.dim + nf * (z.dim + 1);
  size_t o = 0;
  L.oD = o;    o = a16(o + 4 * (size_t)z.dim * z.np * z.np);
  L.oL = o;    o = a16(o + 4 * (size_t)z.nfpt * z.np);
  L.oq = o;    o = a16(o + 4 * (size_t)ENS_MAX_F * z.enp);
  L.ov = o;    o = a16(o + 4 * (size_t)ENS_MAX_F * z.enp);
  L.ofl = o;   o = a16(o + 4 * (size_t)ENS_MAX_F * z.enfpt);
  L.ogeo = o;  o = a16(o + 4 * (size_t)z.e * G);
  L.oconn = o; o = a16(o + 8 * (size_t)z.e * nf);
  L.ofm = o;   o = a16(o + 4 * (size_t)z.nfpt);
  L.osh = o;   o = a16(o + 4 * (size_t)z.permnfp);
  L.total = o;
  return L;
}

template <int MODEL, int DIM>
__device__ void ens_tile(const EnsInst& I, const EnsTile& T, const EnsLayout& L,
                         unsigned char* smem, double ra, double rb, int src, int* err) {
  constexpr int F = Traits<MODEL, DIM>::F;
  constexpr int NA = F;   // no coefficient field in the batch models
  constexpr int NF = DIM + 1;
  const int np = I.np, nfp = I.nfp, G = I.G, E = T.E, ne = T.ne;
  const int nfpt = NF * nfp;
  const float* sD = reinterpret_cast<const float*>(smem + L.oD);
  const float* sL = reinterpret_cast<const float*>(smem + L.oL);
  float* sq = reinterpret_cast<float*>(smem + L.oq);
  float* sv = reinterpret_cast<float*>(smem + L.ov);
  float* sfl = reinterpret_cast<float*>(smem + L.ofl);
  float* sgeo = reinterpret_cast<float*>(smem + L.ogeo);
  int2* sconn = reinterpret_cast<int2*>(smem + L.oconn);
  const int* sfm = reinterpret_cast<const int*>(smem + L.ofm);
  const int* ssh = reinterpret_cast<const int*>(smem + L.osh);
  const int tid = threadIdx.x;
  const int64_t Knp = I.K * np, el0 = T.el0;
  const float* q_in = I.q[src];
  float* q_out = I.q[src ^ 1];

  // ---- stage the tile's state, geometry and face table ----
  for (int f = 0; f < F; ++f)
    for (int x = tid; x < ne * np; x += ENS_THREADS)
      sq[f * E * np + x] = q_in[f * Knp + el0 * np + x];
  for (int x = tid; x < ne * G; x += ENS_THREADS) sgeo[x] = I.geo[el0 * G + x];
  for (int x = tid; x < ne * NF; x += ENS_THREADS) sconn[x] = I.conn[el0 * NF + x];
  __syncthreads();

  // ---- volume terms at every node of the tile ----
  for (int s = tid; s < ne * np; s += ENS_THREADS) {
    const int e = s / np, i = s - e * np;
    float dr[DIM][F];
#pragma unroll
    for (int r = 0; r < DIM; ++r)
#pragma unroll
      for (int f = 0; f < F; ++f) dr[r][f] = 0.f;
    const float* qe = sq + e * np;
    for (int j = 0; j < np; ++j) {
      float d[DIM];
#pragma unroll
      for (int r = 0; r < DIM; ++r) d[r] = sD[(r * np + j) * np + i];
#pragma unroll
      for (int f = 0; f < F; ++f) {
        const float u = qe[f * E * np + j];
#pragma unroll
        for (int r = 0; r < DIM; ++r) dr[r][f] += d[r] * u;
      }
    }
    const float* ge = sgeo + e * G;
    float g[DIM][F], vol[F];
#pragma unroll
    for (int x = 0; x < DIM; ++x)
#pragma unroll
      for (int f = 0; f < F; ++f) {
        float t = 0.f;
#pragma unroll
        for (int r = 0; r < DIM; ++r) t += ge[r * DIM + x] * dr[r][f];
        g[x][f] = t;
      }
    model_volume<MODEL, DIM, float>(I.mp, g, 0.f, vol);
#pragma unroll
    for (int f = 0; f < F; ++f) sv[f * E * np + s] = vol[f];
  }

  // ---- numerical fluxes at every face point of the tile ----
  for (int s = tid; s < ne * nfpt; s += ENS_THREADS) {
    const int e = s / nfpt, p = s - e * nfpt;
    const int face = p / nfp, k = p - face * nfp;
    const int lnode = sfm[p];
    const float* qe = sq + e * np;
    const float* gf = sgeo + e * G + DIM * DIM + face * (DIM + 1);
    float uM[NA], uP[NA], n[DIM], fl[F];
#pragma unroll
    for (int f = 0; f < F; ++f) uM[f] = qe[f * E * np + lnode];
#pragma unroll
    for (int x = 0; x < DIM; ++x) n[x] = gf[x];
    const float fscale = gf[DIM];
    const int2 cn = sconn[e * NF + face];
    bool have = true, bdry = false;
    if (cn.x >= 0) {
      const int nface = cn.y & 3, perm = cn.y >> 2;
      if (nface < NF && perm < I.nperm && cn.x < I.K) {
        const int nn = sfm[nface * nfp + ssh[perm * nfp + k]];
        const int64_t gi = (int64_t)cn.x * np + nn;
#pragma unroll
        for (int f = 0; f < F; ++f) uP[f] = __ldg(q_in + f * Knp + gi);
      } else {
        atomicCAS(err, 0, DEV_BAD_CODE);
        have = false;
      }
    } else {
      bdry = true;
      have = model_bc<MODEL, DIM, float>(I.mp, cn.y, uM, n, 0.f, uP);
    }
    if (have) model_flux<MODEL, DIM, float>(I.mp, bdry, uM, uP, n, fl);
#pragma unroll
    for (int f = 0; f < F; ++f) sfl[f * E * nfpt + s] = have ? fscale * fl[f] : 0.f;
  }
  __syncthreads();

  // ---- lift, FP64 residual and state update ----
  for (int s = tid; s < ne * np; s += ENS_THREADS) {
    const int e = s / np, i = s - e * np;
    float acc[F];
#pragma unroll
    for (int f = 0; f < F; ++f) acc[f] = 0.f;
    for (int p = 0; p < nfpt; ++p) {
      const float l = sL[p * np + i];
#pragma unroll
      for (int f = 0; f < F; ++f) acc[f] += l * sfl[f * E * nfpt + e * nfpt + p];
    }
#pragma unroll
    for (int f = 0; f < F; ++f) {
      const double r = (double)model_finish<MODEL, DIM, float>(I.mp, f, sv[f * E * np + s],
                                                                acc[f], 0.f);
      const int64_t idx = f * Knp + el0 * np + s;
      const double nr = ra * I.res[idx] + I.dt * r;
      I.res[idx] = nr;
      q_out[idx] = (float)((double)sq[f * E * np + s] + rb * nr);
    }
  }
}

// 6 CTAs per SM (40 registers): the stage is latency-bound on its
// global loads, and the extra resident warps hide more of that latency
// than the few spilled registers cost (64 registers, 4 CTAs: 6.43 ms per
// C5 step; 6 CTAs: 5.86 ms)
__global__ void __launch_bounds__(ENS_THREADS, 6) ens_kernel(const EnsInst* __restrict__ insts,
                                                           const EnsTile* __restrict__ tiles,
                                                           int ntiles, EnsLayout L, double ra,
                                                           double rb, int src, int* err) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int tid = threadIdx.x;
  const float* cached = nullptr;   // operators resident in shared memory
  for (int ti = blockIdx.x; ti < ntiles; ti += gridDim.x) {
    const EnsTile T = tiles[ti];
    const EnsInst& I = insts[T.inst];
    __syncthreads();   // the previous tile is done with shared memory
    if (I.dmats_t != cached) {
      const int nfpt = (I.dim + 1) * I.nfp;
      float* wD = reinterpret_cast<float*>(smem + L.oD);
      float* wL = reinterpret_cast<float*>(smem + L.oL);
      int* wfm = reinterpret_cast<int*>(smem + L.ofm);
      int* wsh = reinterpret_cast<int*>(smem + L.osh);
      for (int x = tid; x < I.dim * I.np * I.np; x += ENS_THREADS) wD[x] = I.dmats_t[x];
      for (int x = tid; x < nfpt * I.np; x += ENS_THREADS) wL[x] = I.lift_t[x];
      for (int x = tid; x < nfpt; x += ENS_THREADS) wfm[x] = I.fmask[x];
      for (int x = tid; x < I.nperm * I.nfp; x += ENS_THREADS) wsh[x] = I.shuffle[x];
      cached = I.dmats_t;
    }
    if (I.dim == 2) {
      if (I.model == HB_MODEL_ADVECTION)
        ens_tile<HB_MODEL_ADVECTION, 2>(I, T, L, smem, ra, rb, src, err);
      else
        ens_tile<HB_MODEL_WAVE, 2>(I, T, L, smem, ra, rb, src, err);
    } else {
      if (I.model == HB_MODEL_ADVECTION)
        ens_tile<HB_MODEL_ADVECTION, 3>(I, T, L, smem, ra, rb, src, err);
      else
        ens_tile<HB_MODEL_WAVE, 3>(I, T, L, smem, ra, rb, src, err);
    }
  }
}

}  // namespace

struct Batch {
  int device = 0;
  EnsInst* d_insts = nullptr;
  EnsTile* d_tiles = nullptr;
  int* err = nullptr;
  int ntiles = 0, grid = 0;
  EnsLayout L{};
  int64_t dofs = 0;
};

hb_status batch_create(const hb_batch_member* m, int32_t n, Batch** out) {
  if (!m || n < 1 || !out) return fail(HB_ERR_INVALID_ARGUMENT, "batch: no members");
  std::vector<EnsInst> insts(n);
  std::vector<EnsTile> tiles;
  int dim = -1;
  EnsSizes z;
  int64_t dofs = 0;
  int device = -1;
  for (int k = 0; k < n; ++k) {
    Op* op = reinterpret_cast<Op*>(m[k].op);
    if (!op || !m[k].q0 || !m[k].q1 || !m[k].res)
      return fail(HB_ERR_INVALID_ARGUMENT, "batch: null member field");
    if (op->model != HB_MODEL_ADVECTION && op->model != HB_MODEL_WAVE)
      return fail(HB_ERR_UNSUPPORTED, "batch: advection and constant-c wave members only");
    if (op->n_given != 0)
      return fail(HB_ERR_UNSUPPORTED, "batch: members with given boundary data");
    Discr* d = op->d;
    if (device >= 0 && d->device != device)
      return fail(HB_ERR_INVALID_ARGUMENT, "batch: members on different devices");
    device = d->device;
    if (dim >= 0 && d->dim != dim) return fail(HB_ERR_INVALID_ARGUMENT, "batch: mixed dimensions");
    dim = d->dim;
    DeviceGuard g(device);
    hb_status st = ensure_fp32(d);
    if (st) return st;
    EnsInst& I = insts[k];
    I.model = op->model;
    I.F = op->F;
    I.dim = d->dim;
    I.np = d->np;
    I.nfp = d->nfp;
    I.nperm = d->nperm;
    I.G = d->G;
    I.K = d->K;
    I.dmats_t = d->dmats_t32;
    I.lift_t = d->lift_t32;
    I.geo = d->geo32;
    I.conn = op->conn;
    I.fmask = d->fmask;
    I.shuffle = d->shuffle;
    I.q[0] = m[k].q0;
    I.q[1] = m[k].q1;
    I.res = m[k].res;
    I.dt = m[k].dt;
    I.mp = op->mp;
    int E = m[k].tile_elems > 0 ? m[k].tile_elems : std::max(1, ENS_THREADS / d->np);
    E = std::min<int64_t>(E, d->K);
    if ((int64_t)E * d->np > 4 * ENS_THREADS)
      return fail(HB_ERR_INVALID_ARGUMENT, "batch: tile larger than 4 nodes per thread");
    const int nfpt = d->nfaces * d->nfp;
    z.np = std::max(z.np, d->np);
    z.nfpt = std::max(z.nfpt, nfpt);
    z.enp = std::max(z.enp, E * d->np);
    z.enfpt = std::max(z.enfpt, E * nfpt);
    z.e = std::max(z.e, E);
    z.permnfp = std::max(z.permnfp, d->nperm * d->nfp);
    for (int64_t el0 = 0; el0 < d->K; el0 += E)
      tiles.push_back({k, E, el0, (int)std::min<int64_t>(E, d->K - el0), 0});
    dofs += d->K * d->np * op->F;
  }
  // group tiles by (order, model) so a CTA's tiles mostly reuse its operators
  std::stable_sort(tiles.begin(), tiles.end(), [&](const EnsTile& x, const EnsTile& y) {
    const EnsInst &a = insts[x.inst], &b = insts[y.inst];
    return a.np != b.np ? a.np < b.np : a.model < b.model;
  });
  DeviceGuard g(device);
  if (!g.ok) return fail(HB_ERR_CUDA, "cannot select the CUDA device");
  Batch* B = new (std::nothrow) Batch();
  if (!B) return fail(HB_ERR_INVALID_ARGUMENT, "out of host memory");
  B->device = device;
  z.dim = dim;
  B->L = ens_layout(z);
  B->ntiles = (int)tiles.size();
  B->dofs = dofs;
  auto bail = [&](hb_status s) {
    cudaFree(B->d_insts); cudaFree(B->d_tiles); cudaFree(B->err);
    delete B;
    return s;
  };
  int dev = 0, sms = 0, max_optin = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) !=
          cudaSuccess)
    return bail(fail(HB_ERR_CUDA, "batch: device query"));
  if (B->L.total > (size_t)max_optin) return bail(fail(HB_ERR_UNSUPPORTED, "batch: tiles too large"));
  if (cudaFuncSetAttribute(ens_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)B->L.total) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ens_kernel, ENS_THREADS,
                                                    B->L.total) != cudaSuccess)
    return bail(fail(HB_ERR_CUDA, "batch: occupancy query"));
  B->grid = std::max(1, std::min(B->ntiles, sms * std::max(per_sm, 1)));
  if (cudaMalloc(&B->d_insts, sizeof(EnsInst) * n) != cudaSuccess ||
      cudaMalloc(&B->d_tiles, sizeof(EnsTile) * tiles.size()) != cudaSuccess ||
      cudaMalloc(&B->err, sizeof(int)) != cudaSuccess ||
      cudaMemcpy(B->d_insts, insts.data(), sizeof(EnsInst) * n, cudaMemcpyHostToDevice) !=
          cudaSuccess ||
      cudaMemcpy(B->d_tiles, tiles.data(), sizeof(EnsTile) * tiles.size(),
                 cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(B->err, 0, sizeof(int)) != cudaSuccess)
    return bail(fail(HB_ERR_CUDA, "batch: upload"));
  *out = B;
  return HB_OK;
}

void batch_destroy(Batch* B) {
  if (!B) return;
  DeviceGuard g(B->device);
  cudaFree(B->d_insts);
  cudaFree(B->d_tiles);
  cudaFree(B->err);
  delete B;
}

hb_status batch_stage(Batch* B, double a, double b, int parity, cudaStream_t s) {
  DeviceGuard g(B->device);
  if (!g.ok) return fail(HB_ERR_CUDA, "cannot select the CUDA device");
  ens_kernel<<<B->grid, ENS_THREADS, B->L.total, s>>>(B->d_insts, B->d_tiles, B->ntiles, B->L,
                                                      a, b, parity & 1, B->err);
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

hb_status batch_info(Batch* B, int64_t* info, int n) {
  const int64_t v[5] = {B->ntiles, B->grid, ENS_THREADS, (int64_t)B->L.total, B->dofs};
  for (int k = 0; k < n && k < 5; ++k) info[k] = v[k];
  return HB_OK;
}

hb_status batch_check(Batch* B, cudaStream_t s) {
  DeviceGuard g(B->device);
  int flag = 0;
  HB_CUDA(cudaMemcpyAsync(&flag, B->err, sizeof(int), cudaMemcpyDeviceToHost, s));
  HB_CUDA(cudaStreamSynchronize(s));
  if (flag != 0) return fail(HB_ERR_DEVICE_FLAG, "batch: a kernel flagged bad face data");
  return HB_OK;
}

}  // namespace hb

extern "C" {

hb_status hb_batch_create(const hb_batch_member* members, int32_t n, hb_batch** out) {
  if (!out) return hb::fail(HB_ERR_INVALID_ARGUMENT, "null output");
  hb::Batch* B = nullptr;
  const hb_status st = hb::batch_create(members, n, &B);
  if (st) return st;
  *out = reinterpret_cast<hb_batch*>(B);
  return HB_OK;
}

hb_status hb_batch_destroy(hb_batch* b) {
  hb::batch_destroy(reinterpret_cast<hb::Batch*>(b));
  return HB_OK;
}

hb_status hb_batch_stage(hb_batch* b, double a, double bcoef, int32_t parity, void* stream) {
  if (!b) return hb::fail(HB_ERR_INVALID_ARGUMENT, "null batch");
  return hb::batch_stage(reinterpret_cast<hb::Batch*>(b), a, bcoef, parity,
                         reinterpret_cast<cudaStream_t>(stream));
}

hb_status hb_batch_info(hb_batch* b, int64_t* info, int32_t n) {
  if (!b || !info) return hb::fail(HB_ERR_INVALID_ARGUMENT, "null argument");
  return hb::batch_info(reinterpret_cast<hb::Batch*>(b), info, n);
}

hb_status hb_batch_check(hb_batch* b, void* stream) {
  if (!b) return hb::fail(HB_ERR_INVALID_ARGUMENT, "null batch");
  return hb::batch_check(reinterpret_cast<hb::Batch*>(b), reinterpret_cast<cudaStream_t>(stream));
}

}  // extern "C"
