// CPU ORACLE -- test infrastructure only.
//
// A plain C++ restatement of the loops that hedge's jit CPU backend generates
// for the DG right-hand side.  Only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline leg load this library, as the checker; the product
// path never does.
//
// Parity pinning: the reference cannot be imported or built here (Python 2
// source, missing pymbolic/codepy/PyUblas/Boost), so this restatement is
// pinned against the reference's own known-answer tests (monomial
// mass/differentiation, Gauss theorem, interior flux integrals, symmetry
// preservation, convergence orders), restated in tests/.
//
// Restated loops (file:line in the reference project):
//   or_diff            hedge/backends/jit/diff.py:137-175
//   or_gather_interior hedge/backends/jit/flux.py:239-360 (generated loop
//                      311-353: int slot i, ext slot ext_native_write_map[i],
//                      both scaled by the int-side face Jacobian)
//   or_gather_boundary hedge/backends/jit/flux.py:365-480
//   or_lift            hedge/backends/jit/lift.py:110-141 (result = tmp [*s])
//   or_elwise          hedge/include/hedge/volume_operators.hpp:213-272
//                      (perform_elwise_[scaled_]operator)
// The numerical fluxes are the model templates' formulas:
//   advection  hedge/models/advection.py:62-81, 125-131
//   wave       hedge/models/wave.py:80-108
//   var-c wave hedge/models/wave.py:246-273
//   Maxwell    hedge/models/em.py:145-187
// The flipped flux (ext side) swaps int/ext values and negates the normal,
// as hedge/flux FluxFlipper does.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {

enum { OR_ADVECTION = 1, OR_WAVE = 2, OR_VARWAVE = 3, OR_MAXWELL = 4,
       OR_MAXWELL_TM = 5, OR_MAXWELL_TE = 6,  // 2D (Ez, Hx, Hy) and (Ex, Ey, Hz)
       OR_NORMAL_DOT = 9 };  // test flux sum_k n_k (u_int,k - alpha u_ext,k)

struct or_flux_params {
  int model;
  int dim;
  int flux_type;      // advection: 0 central 1 upwind 2 lf; wave: 0 central 1 upwind;
                      // maxwell: 0 numeric alpha (params[4]) 1 lf
  int n_args;         // flux argument fields
  double v[3];        // advection velocity
  double c;           // wave speed (constant-c wave)
  double eps, mu;     // maxwell
  double alpha;       // maxwell numeric flux type
  double time_sign;   // var-c wave
};

struct or_face_group {
  int64_t n_pairs;
  int face_length;     // Nfp
  int face_count;      // Nf
  int64_t n_local_els;
  int double_sided;
  const int64_t* int_el_base;
  const int32_t* int_ilist;
  const int64_t* int_fof_base;
  const int64_t* ext_el_base;
  const int32_t* ext_ilist;
  const int64_t* ext_fof_base;
  const int32_t* ext_write_map;
  const double* normal;          // [n_pairs, dim] (int side)
  const double* face_jacobian;   // [n_pairs] (int side)
  const uint32_t* index_lists;   // [n_lists, face_length]
  const int64_t* local_el_write_base;
  const double* local_el_inverse_jacobians;
};

static inline int set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

int or_max_threads(int n) { return set_threads(n); }

// d_r u[el, i] = sum_j D_r(i, j) u[el, j]   (jit/diff.py:137-175)
void or_diff(int64_t K, int np_, int dim, const double* dmats,
             const double* field, double* out) {
#pragma omp parallel for schedule(static)
  for (int64_t el = 0; el < K; ++el) {
    const int64_t base = el * np_;
    for (int i = 0; i < np_; ++i) {
      double acc[3] = {0, 0, 0};
      for (int j = 0; j < np_; ++j) {
        const double u = field[base + j];
        for (int r = 0; r < dim; ++r)
          acc[r] += dmats[(size_t)r * np_ * np_ + (size_t)i * np_ + j] * u;
      }
      for (int r = 0; r < dim; ++r) out[(size_t)r * K * np_ + base + i] = acc[r];
    }
  }
}

// out[el] = (s[el] *) M in[el]   (volume_operators.hpp:213-272)
void or_elwise(int64_t K, int rows, int cols, const double* mat,
               const double* coeffs, const double* in, double* out) {
#pragma omp parallel for schedule(static)
  for (int64_t el = 0; el < K; ++el) {
    for (int i = 0; i < rows; ++i) {
      double acc = 0;
      for (int j = 0; j < cols; ++j) acc += mat[(size_t)i * cols + j] * in[el * cols + j];
      out[el * rows + i] = coeffs ? coeffs[el] * acc : acc;
    }
  }
}

// The model flux: in[a] int/ext values of the flux arguments, n the normal.
static void model_flux(const or_flux_params& p, const double* ui,
                       const double* ue, const double* n, double* f) {
  const int d = p.dim;
  switch (p.model) {
    case OR_ADVECTION: {
      double nv = 0;
      for (int k = 0; k < d; ++k) nv += n[k] * p.v[k];
      double weak;
      if (p.flux_type == 0) {
        weak = 0.5 * (ui[0] + ue[0]) * nv;
      } else if (p.flux_type == 1) {
        weak = nv * (nv > 0 ? ui[0] : ue[0]);
      } else {
        double vn = 0;
        for (int k = 0; k < d; ++k) vn += p.v[k] * p.v[k];
        weak = 0.5 * (ui[0] + ue[0]) * nv + 0.5 * std::sqrt(vn) * (ui[0] - ue[0]);
      }
      f[0] = ui[0] * nv - weak;
      break;
    }
    case OR_WAVE: {
      // w = (u, v_1..v_d); flux = -c * ((v.int.n, u.int n) - flux_weak)
      const double sign = p.c > 0 ? 1.0 : -1.0;
      double vavg_n = 0, vint_n = 0, ndv = 0;
      for (int k = 0; k < d; ++k) {
        vavg_n += 0.5 * (ui[1 + k] + ue[1 + k]) * n[k];
        vint_n += ui[1 + k] * n[k];
        ndv += n[k] * (ui[1 + k] - ue[1 + k]);
      }
      const double uavg = 0.5 * (ui[0] + ue[0]);
      double w0 = vavg_n;
      double wk[3];
      for (int k = 0; k < d; ++k) wk[k] = uavg * n[k];
      if (p.flux_type == 1) {
        w0 -= sign * 0.5 * (ui[0] - ue[0]);
        for (int k = 0; k < d; ++k) wk[k] -= sign * 0.5 * (n[k] * ndv);
      }
      f[0] = -p.c * (vint_n - w0);
      for (int k = 0; k < d; ++k) f[1 + k] = -p.c * (ui[0] * n[k] - wk[k]);
      break;
    }
    case OR_VARWAVE: {
      // args (c, u, v_1..v_d)
      const double ci = ui[0], ce = ue[0];
      double vi_n = 0, ve_n = 0;
      for (int k = 0; k < d; ++k) { vi_n += ui[2 + k] * n[k]; ve_n += ue[2 + k] * n[k]; }
      const double h = p.time_sign * 0.5;
      f[0] = h * (ce * ve_n - ci * vi_n);
      for (int k = 0; k < d; ++k) f[1 + k] = h * (n[k] * (ce * ue[1] - ci * ui[1]));
      if (p.flux_type == 1) {
        f[0] += ce * ue[1] - ci * ui[1];
        for (int k = 0; k < d; ++k) f[1 + k] += ce * n[k] * ve_n - ci * n[k] * vi_n;
      }
      break;
    }
    case OR_NORMAL_DOT: {
      // the known-answer tests' fluxes, e.g. f.int * n_x (one-sided) or
      // (u.int - u.ext) * n_y (test/test_jit_discretization.py:164-236, 528-618)
      double s = 0;
      for (int k = 0; k < d; ++k) s += n[k] * (ui[k] - p.alpha * ue[k]);
      f[0] = s;
      break;
    }
    case OR_MAXWELL_TM: case OR_MAXWELL_TE: {
      // em.py:485-515: the 3D flux of the embedded fields (the others zero),
      // normal with a zero z component; variable material (5 arguments):
      // epsilon and mu lead the argument vector
      const int slot_tm[3] = {2, 3, 4}, slot_te[3] = {0, 1, 5};
      const int* slot = p.model == OR_MAXWELL_TM ? slot_tm : slot_te;
      const int off = p.n_args == 5 ? 2 : 0;
      double ui8[8] = {0, 0, 0, 0, 0, 0, 0, 0}, ue8[8] = {0, 0, 0, 0, 0, 0, 0, 0}, f6[6];
      for (int k = 0; k < off; ++k) { ui8[k] = ui[k]; ue8[k] = ue[k]; }
      for (int k = 0; k < 3; ++k) {
        ui8[off + slot[k]] = ui[off + k];
        ue8[off + slot[k]] = ue[off + k];
      }
      const double n3[3] = {n[0], n[1], 0.0};
      or_flux_params p3 = p;
      p3.model = OR_MAXWELL;
      p3.dim = 3;
      p3.n_args = 6 + off;
      model_flux(p3, ui8, ue8, n3, f6);
      for (int k = 0; k < 3; ++k) f[k] = f6[slot[k]];
      break;
    }
    case OR_MAXWELL: {
      // variable material (em.py:118-190 with flux_w = (epsilon, mu, w)):
      // 8 arguments, the impedances from each side's epsilon and mu
      const int off = p.n_args == 8 ? 2 : 0;
      const double* ei = ui + off; const double* hi = ui + off + 3;
      const double* ee = ue + off; const double* he = ue + off + 3;
      double de[3], dh[3];
      for (int k = 0; k < 3; ++k) { de[k] = ei[k] - ee[k]; dh[k] = hi[k] - he[k]; }
      auto cross = [](const double* a, const double* b, double* r) {
        r[0] = a[1] * b[2] - a[2] * b[1];
        r[1] = a[2] * b[0] - a[0] * b[2];
        r[2] = a[0] * b[1] - a[1] * b[0];
      };
      if (p.flux_type == 1) {   // "lf"
        double t[3];
        cross(n, dh, t);
        for (int k = 0; k < 3; ++k) f[k] = 0.5 * (-t[k]);
        cross(n, de, t);
        for (int k = 0; k < 3; ++k) f[3 + k] = 0.5 * t[k];
      } else {
        const double Zi = off ? std::sqrt(ui[1] / ui[0]) : std::sqrt(p.mu / p.eps);
        const double Ze = off ? std::sqrt(ue[1] / ue[0]) : Zi;
        const double Yi = 1.0 / Zi, Ye = 1.0 / Ze;
        double nde[3], ndh[3], a[3], t[3];
        cross(n, de, nde);
        cross(n, dh, ndh);
        for (int k = 0; k < 3; ++k) a[k] = Ze * dh[k] - p.alpha * nde[k];
        cross(n, a, t);
        for (int k = 0; k < 3; ++k) f[k] = -1.0 / (Zi + Ze) * t[k];
        for (int k = 0; k < 3; ++k) a[k] = Ye * de[k] + p.alpha * ndh[k];
        cross(n, a, t);
        for (int k = 0; k < 3; ++k) f[3 + k] = 1.0 / (Yi + Ye) * t[k];
      }
      break;
    }
  }
}

static int n_flux_components(const or_flux_params& p) {
  switch (p.model) {
    case OR_ADVECTION: return 1;
    case OR_WAVE: return p.dim + 1;
    case OR_VARWAVE: return p.dim + 1;
    case OR_MAXWELL: return 6;
    case OR_MAXWELL_TM: case OR_MAXWELL_TE: return 3;
    case OR_NORMAL_DOT: return 1;
  }
  return 0;
}

// Interior gather (jit/flux.py:311-353).  args: [n_args][n_vol];
// fof: [n_comp][n_local_els * Nf * Nfp], zero-initialised by the caller.
void or_gather_interior(const or_face_group* fg, const or_flux_params* p,
                        int64_t n_vol, const double* args, double* fof) {
  const int nfp = fg->face_length;
  const int nc = n_flux_components(*p);
  const int64_t fof_len = fg->n_local_els * fg->face_count * nfp;
  const int d = p->dim;
#pragma omp parallel for schedule(static)
  for (int64_t fp = 0; fp < fg->n_pairs; ++fp) {
    const uint32_t* il_int = fg->index_lists + (size_t)fg->int_ilist[fp] * nfp;
    const uint32_t* il_ext = fg->index_lists + (size_t)fg->ext_ilist[fp] * nfp;
    const uint32_t* wmap = fg->index_lists + (size_t)fg->ext_write_map[fp] * nfp;
    const double fj = fg->face_jacobian[fp];
    double n[3], nflip[3];
    for (int k = 0; k < d; ++k) { n[k] = fg->normal[fp * d + k]; nflip[k] = -n[k]; }
    for (int i = 0; i < nfp; ++i) {
      const int64_t int_idx = fg->int_el_base[fp] + il_int[i];
      const int64_t ext_idx = fg->ext_el_base[fp] + il_ext[i];
      double ui[8], ue[8], f[8], ff[8];
      for (int a = 0; a < p->n_args; ++a) {
        ui[a] = args[a * n_vol + int_idx];
        ue[a] = args[a * n_vol + ext_idx];
      }
      model_flux(*p, ui, ue, n, f);
      model_flux(*p, ue, ui, nflip, ff);
      for (int c = 0; c < nc; ++c) {
        fof[c * fof_len + fg->int_fof_base[fp] + i] = fj * f[c];
        fof[c * fof_len + fg->ext_fof_base[fp] + wmap[i]] = fj * ff[c];
      }
    }
  }
}

// Boundary gather (jit/flux.py:429-472): ext values come from the
// boundary vectors bargs [n_args][n_bdry].
void or_gather_boundary(const or_face_group* fg, const or_flux_params* p,
                        int64_t n_vol, const double* args, int64_t n_bdry,
                        const double* bargs, double* fof) {
  const int nfp = fg->face_length;
  const int nc = n_flux_components(*p);
  const int64_t fof_len = fg->n_local_els * fg->face_count * nfp;
  const int d = p->dim;
#pragma omp parallel for schedule(static)
  for (int64_t fp = 0; fp < fg->n_pairs; ++fp) {
    const uint32_t* il_int = fg->index_lists + (size_t)fg->int_ilist[fp] * nfp;
    const uint32_t* il_ext = fg->index_lists + (size_t)fg->ext_ilist[fp] * nfp;
    const double fj = fg->face_jacobian[fp];
    double n[3];
    for (int k = 0; k < d; ++k) n[k] = fg->normal[fp * d + k];
    for (int i = 0; i < nfp; ++i) {
      const int64_t int_idx = fg->int_el_base[fp] + il_int[i];
      const int64_t ext_idx = fg->ext_el_base[fp] + il_ext[i];
      double ui[8], ue[8], f[8];
      for (int a = 0; a < p->n_args; ++a) {
        ui[a] = args[a * n_vol + int_idx];
        ue[a] = bargs[a * n_bdry + ext_idx];
      }
      model_flux(*p, ui, ue, n, f);
      for (int c = 0; c < nc; ++c)
        fof[c * fof_len + fg->int_fof_base[fp] + i] = fj * f[c];
    }
  }
}

// result[dest_el_base + i] = (sum_j L(i, j) fof[src + j]) (* s[el])
// (jit/lift.py:110-141).  out is zero-initialised by the caller.
void or_lift(const or_face_group* fg, int np_, const double* mat,
             const double* scaling, const double* fof, double* out) {
  const int ncols = fg->face_count * fg->face_length;
#pragma omp parallel for schedule(static)
  for (int64_t el = 0; el < fg->n_local_els; ++el) {
    const int64_t dest = fg->local_el_write_base[el];
    const int64_t src = (int64_t)ncols * el;
    for (int i = 0; i < np_; ++i) {
      double tmp = 0;
      for (int j = 0; j < ncols; ++j) tmp += mat[(size_t)i * ncols + j] * fof[src + j];
      out[dest + i] = scaling ? tmp * scaling[el] : tmp;
    }
  }
}

// y = a*x + b*y elementwise, the LSRK combination (vector_primitives.py:58-77)
void or_lincomb(int64_t n, double a, const double* x, double b, const double* y,
                double* out) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) out[i] = a * x[i] + b * y[i];
}

}  // extern "C"
