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
// the 2D TM and TE systems: three of the six components, no z dependence
template <int DIM>
struct Traits<HB_MODEL_MAXWELL_TM, DIM> { static constexpr int F = 3, COEFF = 0; };
template <int DIM>
struct Traits<HB_MODEL_MAXWELL_TE, DIM> { static constexpr int F = 3, COEFF = 0; };

// Position of field f of a 2D Maxwell system in (Ex Ey Ez Hx Hy Hz): TM
// carries (Ez, Hx, Hy), TE (Ex, Ey, Hz) (em.py get_eh_subset); and how many
// of its fields are E components (they come first).
template <int MODEL>
__host__ __device__ constexpr int maxwell_slot(int f) {
  return MODEL == HB_MODEL_MAXWELL_TM ? (f == 0 ? 2 : 2 + f) : (f < 2 ? f : 5);
}
template <int MODEL>
__host__ __device__ constexpr int maxwell_ne() {
  return MODEL == HB_MODEL_MAXWELL ? 3 : (MODEL == HB_MODEL_MAXWELL_TM ? 1 : 2);
}
template <int MODEL>
struct IsMaxwell {
  static constexpr bool value = MODEL == HB_MODEL_MAXWELL || MODEL == HB_MODEL_MAXWELL_TM ||
                                MODEL == HB_MODEL_MAXWELL_TE;
};

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
  } else if constexpr (MODEL == HB_MODEL_MAXWELL_TM) {
    // (Ez, Hx, Hy): (curl H)_z = dx Hy - dy Hx; -curl E = (-dy Ez, dx Ez)
    vol[0] = g[0][2] - g[1][1];
    vol[1] = -g[1][0];
    vol[2] = g[0][0];
  } else if constexpr (MODEL == HB_MODEL_MAXWELL_TE) {
    // (Ex, Ey, Hz): curl H = (dy Hz, -dx Hz); -(curl E)_z = -(dx Ey - dy Ex)
    vol[0] = g[1][2];
    vol[1] = -g[0][2];
    vol[2] = -(g[0][1] - g[1][0]);
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
// (wave, var-c wave: the source of u; Maxwell: the value added to E_f's rhs,
// -J_f / eps for a current J, zero for the H components)
template <int MODEL, int DIM, typename T>
__device__ __forceinline__ T model_finish(const ModelParams& mp, int f, T vol,
                                          T lift, T src) {
  if constexpr (IsMaxwell<MODEL>::value) {
    constexpr int NE = maxwell_ne<MODEL>();
    return (vol + lift) / (f < NE ? T(mp.eps) : T(mp.mu)) + (f < NE ? src : T(0));
  } else if constexpr (MODEL == HB_MODEL_WAVE) {
    return f == 0 ? vol + lift + src : vol + lift;
  } else if constexpr (MODEL == HB_MODEL_VARWAVE) {
    return f == 0 ? vol - src + lift : vol + lift;
  } else {
    return vol + lift;
  }
}

// Index of field f's source value at volume node `node` in the caller's
// source vector: one [K*Np] vector for the wave models (field 0), [3][K*Np]
// for Maxwell (the E components); -1 where the field has none.
template <int MODEL>
__device__ __forceinline__ int64_t model_src_index(int f, int64_t node, int64_t knp) {
  if constexpr (IsMaxwell<MODEL>::value) return f < maxwell_ne<MODEL>() ? f * knp + node : -1;
  else return f == 0 ? node : -1;
}

// Maxwell boundary states of (E, H) = u[0..3), u[3..6) (em.py:226-307):
// PEC (-E, H), PMC (E, -H), first-order absorbing, incident (zero data).
// False: no boundary flux.
template <typename T>
__device__ __forceinline__ bool maxwell_bc3(const ModelParams& mp, int kind, const T* u,
                                            const T* n, T* uP) {
  const T* e = u;
  const T* h = u + 3;
  if (kind == HB_BC_PEC) {
#pragma unroll
    for (int k = 0; k < 3; ++k) { uP[k] = -e[k]; uP[3 + k] = h[k]; }
  } else if (kind == HB_BC_PMC) {
#pragma unroll
    for (int k = 0; k < 3; ++k) { uP[k] = e[k]; uP[3 + k] = -h[k]; }
  } else if (kind == HB_BC_ABSORB) {
    const T Z = T(mp.Z), Y = T(mp.Y);
    T ne[3], nh[3], nne[3], nnh[3];
    cross3(n, e, ne);
    cross3(n, h, nh);
    cross3(n, ne, nne);
    cross3(n, nh, nnh);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      uP[k] = e[k] + T(0.5) * (nne[k] - Z * nh[k]);
      uP[3 + k] = h[k] + T(0.5) * (nnh[k] + Y * ne[k]);
    }
  } else if (kind == HB_BC_INCIDENT) {
    // the reference's default incident data is zero (em.py:289-307)
#pragma unroll
    for (int k = 0; k < 6; ++k) uP[k] = T(0);
  } else {
    return false;
  }
  return true;
}

// ---- boundary exterior states ---------------------------------------------
// Returns false when the face carries no boundary flux (BC_NONE).  `given`
// is the caller's boundary datum at the node (HB_BC_GIVEN): the advection
// inflow value, or the wave's Dirichlet value.
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
    } else if (kind == HB_BC_GIVEN && MODEL == HB_MODEL_WAVE) {
      // inhomogeneous Dirichlet data g (wave.py:133-142): (2 g - u, v)
      uP[C] = T(2) * given - u;
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
  } else if constexpr (MODEL == HB_MODEL_MAXWELL) {
    (void)NA;
    return maxwell_bc3<T>(mp, kind, uM, n, uP);
  } else {
    // 2D TM / TE: the 3D conditions on the embedded fields, n_z = 0
    T u6[6] = {T(0), T(0), T(0), T(0), T(0), T(0)}, p6[6];
    const T n3[3] = {n[0], n[1], T(0)};
#pragma unroll
    for (int f = 0; f < 3; ++f) u6[maxwell_slot<MODEL>(f)] = uM[f];
    if (!maxwell_bc3<T>(mp, kind, u6, n3, p6)) return false;
#pragma unroll
    for (int f = 0; f < 3; ++f) uP[f] = p6[maxwell_slot<MODEL>(f)];
    (void)NA;
    return true;
  }
}

// Maxwell numerical flux of the jumps [E] = de, [H] = dh (em.py:145-187,
// fixed material): "lf" (flux type 1 here) or the numeric flux type alpha.
template <typename T>
__device__ __forceinline__ void maxwell_flux3(const ModelParams& mp, bool bdry, const T* de,
                                              const T* dh, const T* n, T* f) {
  {
    const int ft = bdry ? mp.bdry_flux_type : mp.flux_type;
    const T alpha = T(bdry ? mp.bdry_alpha : mp.alpha);
    T t[3];
    if (ft == 1) {
      cross3(n, dh, t);
#pragma unroll
      for (int k = 0; k < 3; ++k) f[k] = T(0.5) * (-t[k]);
      cross3(n, de, t);
#pragma unroll
      for (int k = 0; k < 3; ++k) f[3 + k] = T(0.5) * t[k];
    } else {
      const T Z = T(mp.Z), Y = T(mp.Y);
      T nde[3], ndh[3], a[3];
      cross3(n, de, nde);
      cross3(n, dh, ndh);
#pragma unroll
      for (int k = 0; k < 3; ++k) a[k] = Z * dh[k] - alpha * nde[k];
      cross3(n, a, t);
      const T fe = T(-0.5) * Y, fh = T(0.5) * Z;   // -1/(2Z), 1/(2Y)
#pragma unroll
      for (int k = 0; k < 3; ++k) f[k] = fe * t[k];
#pragma unroll
      for (int k = 0; k < 3; ++k) a[k] = Y * de[k] + alpha * ndh[k];
      cross3(n, a, t);
#pragma unroll
      for (int k = 0; k < 3; ++k) f[3 + k] = fh * t[k];
    }
  }
}

// The same flux for variable material (em.py:118-190 with epsilon, mu volume
// fields): the impedances Z = sqrt(mu / eps) of the interior and exterior
// sides enter the numeric flux type; "lf" does not depend on the material.
template <typename T>
__device__ __forceinline__ void maxwell_flux3_var(const ModelParams& mp, bool bdry, const T* de,
                                                  const T* dh, const T* n, T Zi, T Ze, T* f) {
  const int ft = bdry ? mp.bdry_flux_type : mp.flux_type;
  const T alpha = T(bdry ? mp.bdry_alpha : mp.alpha);
  T t[3];
  if (ft == 1) {
    cross3(n, dh, t);
#pragma unroll
    for (int k = 0; k < 3; ++k) f[k] = T(0.5) * (-t[k]);
    cross3(n, de, t);
#pragma unroll
    for (int k = 0; k < 3; ++k) f[3 + k] = T(0.5) * t[k];
  } else {
    const T Yi = T(1) / Zi, Ye = T(1) / Ze;
    T nde[3], ndh[3], a[3];
    cross3(n, de, nde);
    cross3(n, dh, ndh);
#pragma unroll
    for (int k = 0; k < 3; ++k) a[k] = Ze * dh[k] - alpha * nde[k];
    cross3(n, a, t);
    const T fe = T(-1) / (Zi + Ze), fh = T(1) / (Yi + Ye);
#pragma unroll
    for (int k = 0; k < 3; ++k) f[k] = fe * t[k];
#pragma unroll
    for (int k = 0; k < 3; ++k) a[k] = Ye * de[k] + alpha * ndh[k];
    cross3(n, a, t);
#pragma unroll
    for (int k = 0; k < 3; ++k) f[3 + k] = fh * t[k];
  }
}

// Maxwell systems (3D, TM, TE) with variable material: the flux of the jumps
// with the interior and exterior impedances Zi, Ze.
template <int MODEL, int DIM, typename T>
__device__ __forceinline__ void maxwell_flux_var(const ModelParams& mp, bool bdry,
                                                 const T (&uM)[Args<MODEL, DIM>::N],
                                                 const T (&uP)[Args<MODEL, DIM>::N],
                                                 const T (&n)[DIM], T Zi, T Ze,
                                                 T (&f)[Traits<MODEL, DIM>::F]) {
  if constexpr (MODEL == HB_MODEL_MAXWELL) {
    T de[3], dh[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) { de[k] = uM[k] - uP[k]; dh[k] = uM[3 + k] - uP[3 + k]; }
    maxwell_flux3_var<T>(mp, bdry, de, dh, &n[0], Zi, Ze, f);
  } else if constexpr (IsMaxwell<MODEL>::value) {
    T d6[6] = {T(0), T(0), T(0), T(0), T(0), T(0)}, f6[6];
    const T n3[3] = {n[0], n[1], T(0)};
#pragma unroll
    for (int q = 0; q < 3; ++q) d6[maxwell_slot<MODEL>(q)] = uM[q] - uP[q];
    maxwell_flux3_var<T>(mp, bdry, d6, d6 + 3, n3, Zi, Ze, f6);
#pragma unroll
    for (int q = 0; q < 3; ++q) f[q] = f6[maxwell_slot<MODEL>(q)];
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
  } else if constexpr (MODEL == HB_MODEL_MAXWELL) {
    T de[3], dh[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) { de[k] = uM[k] - uP[k]; dh[k] = uM[3 + k] - uP[3 + k]; }
    maxwell_flux3<T>(mp, bdry, de, dh, &n[0], f);
  } else {
    // 2D TM / TE: the 3D flux of the embedded jumps, n_z = 0
    T d6[6] = {T(0), T(0), T(0), T(0), T(0), T(0)}, f6[6];
    const T n3[3] = {n[0], n[1], T(0)};
#pragma unroll
    for (int q = 0; q < 3; ++q) d6[maxwell_slot<MODEL>(q)] = uM[q] - uP[q];
    maxwell_flux3<T>(mp, bdry, d6, d6 + 3, n3, f6);
#pragma unroll
    for (int q = 0; q < 3; ++q) f[q] = f6[maxwell_slot<MODEL>(q)];
  }
}

}  // namespace hb
