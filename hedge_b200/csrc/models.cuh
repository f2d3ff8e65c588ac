// Device-side model physics: volume terms, numerical fluxes, boundary states.
//
// Each function restates one model template of the reference:
//   advection  hedge/models/advection.py:62-81 (weak flux), 125-149 (strong)
//   wave       hedge/models/wave.py:80-108 (flux), 110-180 (op template, BCs)
//   var-c wave hedge/models/wave.py:246-273 (flux), 287-395 (op template)
//   Maxwell    hedge/models/em.py:145-187 (flux), 192-214 (curls),
//              226-287 (PEC/PMC/absorbing BCs), 309-371 (op template)
// g[x][f] is the physical derivative d/dx_x of field f.
#pragma once

#include "common.cuh"

namespace hb {

template <int MODEL, int DIM>
struct Traits;
template <int DIM>
struct Traits<HB_MODEL_ADVECTION, DIM> { static constexpr int F = 1, COEFF = 0; };
template <int DIM>
struct Traits<HB_MODEL_WAVE, DIM> { static constexpr int F = DIM + 1, COEFF = 0; };
template <int DIM>
struct Traits<HB_MODEL_VARWAVE, DIM> { static constexpr int F = DIM + 1, COEFF = 1; };
template <int DIM>
struct Traits<HB_MODEL_MAXWELL, DIM> { static constexpr int F = 6, COEFF = 0; };

// Flux argument vector: [coeff (var-c wave)] + fields.
template <int MODEL, int DIM>
struct Args {
  static constexpr int F = Traits<MODEL, DIM>::F;
  static constexpr int C = Traits<MODEL, DIM>::COEFF;
  static constexpr int N = F + C;
};

template <typename T>
__device__ __forceinline__ void cross3(const T* a, const T* b, T* r) {
  r[0] = a[1] * b[2] - a[2] * b[1];
  r[1] = a[2] * b[0] - a[0] * b[2];
  r[2] = a[0] * b[1] - a[1] * b[0];
}

// ---- volume terms ---------------------------------------------------------
template <int MODEL, int DIM, typename T>
__device__ __forceinline__ void model_volume(const ModelParams& mp,
                                             const T (&g)[DIM][Traits<MODEL, DIM>::F],
                                             T cnode,
                                             T (&vol)[Traits<MODEL, DIM>::F]) {
  if constexpr (MODEL == HB_MODEL_ADVECTION) {
    T s = 0;
#pragma unroll
    for (int x = 0; x < DIM; ++x) s += T(mp.v[x]) * g[x][0];
    vol[0] = -s;
  } else if constexpr (MODEL == HB_MODEL_WAVE || MODEL == HB_MODEL_VARWAVE) {
    const T c = (MODEL == HB_MODEL_WAVE) ? T(mp.c) : T(mp.time_sign) * cnode;
    T div = 0;
#pragma unroll
    for (int x = 0; x < DIM; ++x) div += g[x][1 + x];
    vol[0] = c * div;
#pragma unroll
    for (int x = 0; x < DIM; ++x) vol[1 + x] = c * g[x][0];
  } else {  // Maxwell: (curl H, -curl E)
    vol[0] = g[1][5] - g[2][4];
    vol[1] = g[2][3] - g[0][5];
    vol[2] = g[0][4] - g[1][3];
    vol[3] = -(g[1][2] - g[2][1]);
    vol[4] = -(g[2][0] - g[0][2]);
    vol[5] = -(g[0][1] - g[1][0]);
  }
}

// rhs component f from its volume term, lifted flux and optional source
template <int MODEL, int DIM, typename T>
__device__ __forceinline__ T model_finish(const ModelParams& mp, int f, T vol,
                                          T lift, T src) {
  if constexpr (MODEL == HB_MODEL_MAXWELL) {
    return (vol + lift) / (f < 3 ? T(mp.eps) : T(mp.mu));
  } else if constexpr (MODEL == HB_MODEL_WAVE) {
    return f == 0 ? vol + lift + src : vol + lift;
  } else if constexpr (MODEL == HB_MODEL_VARWAVE) {
    return f == 0 ? vol - src + lift : vol + lift;
  } else {
    return vol + lift;
  }
}

// ---- boundary exterior states ---------------------------------------------
// Returns false when the face carries no boundary flux (BC_NONE).
template <int MODEL, int DIM, typename T>
__device__ __forceinline__ bool model_bc(const ModelParams& mp, int kind,
                                         const T (&uM)[Args<MODEL, DIM>::N],
                                         const T (&n)[DIM], T given,
                                         T (&uP)[Args<MODEL, DIM>::N]) {
  constexpr int NA = Args<MODEL, DIM>::N;
  constexpr int C = Args<MODEL, DIM>::C;
  if (kind == HB_BC_NONE) return false;
  if constexpr (MODEL == HB_MODEL_ADVECTION) {
    if (kind != HB_BC_GIVEN) return false;
    uP[0] = given;
    return true;
  } else if constexpr (MODEL == HB_MODEL_WAVE || MODEL == HB_MODEL_VARWAVE) {
    const T sgn = (MODEL == HB_MODEL_WAVE) ? (mp.c > 0 ? T(1) : T(-1)) : T(mp.time_sign);
    if (C) uP[0] = uM[0];  // boundarized c
    const T u = uM[C];
    if (kind == HB_BC_DIRICHLET) {
      uP[C] = -u;
#pragma unroll
      for (int x = 0; x < DIM; ++x) uP[C + 1 + x] = uM[C + 1 + x];
    } else if (kind == HB_BC_NEUMANN) {
      uP[C] = u;
#pragma unroll
      for (int x = 0; x < DIM; ++x) uP[C + 1 + x] = -uM[C + 1 + x];
    } else if (kind == HB_BC_RADIATION) {
      T nv = 0;
#pragma unroll
      for (int x = 0; x < DIM; ++x) nv += n[x] * uM[C + 1 + x];
      uP[C] = T(0.5) * (u - sgn * nv);
#pragma unroll
      for (int x = 0; x < DIM; ++x) uP[C + 1 + x] = T(0.5) * n[x] * (nv - sgn * u);
    } else {
      return false;
    }
    return true;
  } else {  // Maxwell
    const T* e = uM;
    const T* h = uM + 3;
    if (kind == HB_BC_PEC) {
#pragma unroll
      for (int k = 0; k < 3; ++k) { uP[k] = -e[k]; uP[3 + k] = h[k]; }
    } else if (kind == HB_BC_PMC) {
#pragma unroll
      for (int k = 0; k < 3; ++k) { uP[k] = e[k]; uP[3 + k] = -h[k]; }
    } else if (kind == HB_BC_ABSORB) {
      const T Z = T(mp.Z), Y = T(mp.Y);
      T ne[3], nh[3], nne[3], nnh[3];
      cross3(&n[0], e, ne);
      cross3(&n[0], h, nh);
      cross3(&n[0], ne, nne);
      cross3(&n[0], nh, nnh);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        uP[k] = e[k] + T(0.5) * (nne[k] - Z * nh[k]);
        uP[3 + k] = h[k] + T(0.5) * (nnh[k] + Y * ne[k]);
      }
    } else {
      return false;
    }
    (void)NA;
    return true;
  }
}

// ---- numerical fluxes (strong form, before the face-Jacobian scale) --------
template <int MODEL, int DIM, typename T>
__device__ __forceinline__ void model_flux(const ModelParams& mp, bool bdry,
                                           const T (&uM)[Args<MODEL, DIM>::N],
                                           const T (&uP)[Args<MODEL, DIM>::N],
                                           const T (&n)[DIM],
                                           T (&f)[Traits<MODEL, DIM>::F]) {
  if constexpr (MODEL == HB_MODEL_ADVECTION) {
    T nv = 0;
#pragma unroll
    for (int x = 0; x < DIM; ++x) nv += n[x] * T(mp.v[x]);
    T weak;
    if (mp.flux_type == 0) {
      weak = T(0.5) * (uM[0] + uP[0]) * nv;
    } else if (mp.flux_type == 1) {
      weak = nv * (nv > T(0) ? uM[0] : uP[0]);
    } else {
      T vv = 0;
#pragma unroll
      for (int x = 0; x < DIM; ++x) vv += T(mp.v[x] * mp.v[x]);
      weak = T(0.5) * (uM[0] + uP[0]) * nv + T(0.5) * sqrt(vv) * (uM[0] - uP[0]);
    }
    f[0] = uM[0] * nv - weak;
  } else if constexpr (MODEL == HB_MODEL_WAVE) {
    const T c = T(mp.c);
    const T sign = mp.c > 0 ? T(1) : T(-1);
    T vavg_n = 0, vint_n = 0, ndv = 0;
#pragma unroll
    for (int x = 0; x < DIM; ++x) {
      vavg_n += T(0.5) * (uM[1 + x] + uP[1 + x]) * n[x];
      vint_n += uM[1 + x] * n[x];
      ndv += n[x] * (uM[1 + x] - uP[1 + x]);
    }
    const T uavg = T(0.5) * (uM[0] + uP[0]);
    T w0 = vavg_n;
    T wk[DIM];
#pragma unroll
    for (int x = 0; x < DIM; ++x) wk[x] = uavg * n[x];
    if (mp.flux_type == 1) {
      w0 -= sign * T(0.5) * (uM[0] - uP[0]);
#pragma unroll
      for (int x = 0; x < DIM; ++x) wk[x] -= sign * T(0.5) * (n[x] * ndv);
    }
    f[0] = -c * (vint_n - w0);
#pragma unroll
    for (int x = 0; x < DIM; ++x) f[1 + x] = -c * (uM[0] * n[x] - wk[x]);
  } else if constexpr (MODEL == HB_MODEL_VARWAVE) {
    const T ci = uM[0], ce = uP[0];
    T vi_n = 0, ve_n = 0;
#pragma unroll
    for (int x = 0; x < DIM; ++x) { vi_n += uM[2 + x] * n[x]; ve_n += uP[2 + x] * n[x]; }
    const T h = T(mp.time_sign) * T(0.5);
    f[0] = h * (ce * ve_n - ci * vi_n);
#pragma unroll
    for (int x = 0; x < DIM; ++x) f[1 + x] = h * (n[x] * (ce * uP[1] - ci * uM[1]));
    if (mp.flux_type == 1) {
      f[0] += ce * uP[1] - ci * uM[1];
#pragma unroll
      for (int x = 0; x < DIM; ++x) f[1 + x] += ce * n[x] * ve_n - ci * n[x] * vi_n;
    }
  } else {  // Maxwell
    const int ft = bdry ? mp.bdry_flux_type : mp.flux_type;
    const T alpha = T(bdry ? mp.bdry_alpha : mp.alpha);
    T de[3], dh[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) { de[k] = uM[k] - uP[k]; dh[k] = uM[3 + k] - uP[3 + k]; }
    T t[3];
    if (ft == 1) {
      cross3(&n[0], dh, t);
#pragma unroll
      for (int k = 0; k < 3; ++k) f[k] = T(0.5) * (-t[k]);
      cross3(&n[0], de, t);
#pragma unroll
      for (int k = 0; k < 3; ++k) f[3 + k] = T(0.5) * t[k];
    } else {
      const T Z = T(mp.Z), Y = T(mp.Y);
      T nde[3], ndh[3], a[3];
      cross3(&n[0], de, nde);
      cross3(&n[0], dh, ndh);
#pragma unroll
      for (int k = 0; k < 3; ++k) a[k] = Z * dh[k] - alpha * nde[k];
      cross3(&n[0], a, t);
      const T fe = T(-0.5) * Y, fh = T(0.5) * Z;   // -1/(2Z), 1/(2Y)
#pragma unroll
      for (int k = 0; k < 3; ++k) f[k] = fe * t[k];
#pragma unroll
      for (int k = 0; k < 3; ++k) a[k] = Y * de[k] + alpha * ndh[k];
      cross3(&n[0], a, t);
#pragma unroll
      for (int k = 0; k < 3; ++k) f[3 + k] = fh * t[k];
    }
  }
}

}  // namespace hb
