/* hedge_b200 -- B200 (sm_100a) DG right-hand-side backend, C ABI.
 *
 * Plain pointers and sizes only.  All state/field buffers are device memory
 * owned by the caller (the reference writes into caller-allocated
 * volume_zeros() arrays the same way, hedge/backends/jit/__init__.py:167-168);
 * the library owns only the descriptor objects it creates (create/destroy
 * pairs).  Every call returns an hb_status; no call aborts or traps.  Device
 * kernels report bad input through a device error flag that the host turns
 * into HB_ERR_DEVICE_FLAG.  Calls on distinct descriptors are re-entrant;
 * each call is enqueued on the stream it is given (a cudaStream_t passed as
 * void*; NULL = legacy default stream).
 *
 * Layouts.  A volume vector is [K * Np], element-major, node order of the
 * reference element (hedge/discretization/__init__.py:405-417).  A state of
 * F fields is F such vectors back to back: [F][K * Np].
 */
#ifndef HEDGE_B200_H
#define HEDGE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  HB_OK = 0,
  HB_ERR_INVALID_ARGUMENT = 1,
  HB_ERR_UNSUPPORTED = 2,
  HB_ERR_CUDA = 3,
  HB_ERR_DEVICE_FLAG = 4
} hb_status;

enum {
  HB_MODEL_ADVECTION = 1, /* hedge/models/advection.py:124-149 */
  HB_MODEL_WAVE = 2,      /* hedge/models/wave.py:37-197 */
  HB_MODEL_VARWAVE = 3,   /* hedge/models/wave.py:204-418 */
  HB_MODEL_MAXWELL = 4,   /* hedge/models/em.py:38-387 */
  HB_MODEL_MAXWELL_TM = 5, /* hedge/models/em.py:485-498, 2D, fields (Ez, Hx, Hy) */
  HB_MODEL_MAXWELL_TE = 6, /* hedge/models/em.py:501-515, 2D, fields (Ex, Ey, Hz) */
  HB_MODEL_VARADV = 7      /* hedge/models/advection.py:190-368: variable-coefficient
                              advection, weak form, integrals by quadrature (one
                              field u; the velocity field is the coeff argument,
                              [dim][K*Np] FP64; hb_op_desc.quadrature required).
                              Boundary kinds: HB_BC_GIVEN (u outside = the given
                              values, bc_u_f), HB_BC_DIRICHLET (u outside = 0,
                              bc_u_f "None"), HB_BC_NONE (no flux); v outside =
                              v inside.  FP64 and FP32 precisions. */
};

enum {
  HB_PREC_FP64 = 0,   /* FP64 state, FP64 arithmetic */
  HB_PREC_FP32 = 1,   /* FP32 state and residual, FP32 arithmetic; where a resident
                         tensor-core kernel is built for the (model, dimension,
                         order), the two contractions run as split-FP16 products
                         (as HB_PREC_FP16X3, FP32 accumulation), else on CUDA cores
                         (hedge/discretization/__init__.py:217-219,
                         default_scalar_type float32) */
  HB_PREC_BF16X3 = 2, /* FP64 state, split-BF16 tensor-core products, FP32 accumulation */
  HB_PREC_FP16X3 = 3, /* FP64 state, split-FP16 products of power-of-two-scaled rows,
                         FP32 accumulation (same cost as BF16X3, ~8x more accurate) */
  HB_PREC_FP32_SIMT = 4 /* FP32 state, FP32 arithmetic, always on CUDA cores */
};

enum {
  HB_BC_NONE = 0, HB_BC_GIVEN = 1, HB_BC_DIRICHLET = 2, HB_BC_NEUMANN = 3,
  HB_BC_RADIATION = 4, HB_BC_PEC = 5, HB_BC_PMC = 6, HB_BC_ABSORB = 7,
  HB_BC_INCIDENT = 8  /* Maxwell models only: incident-field boundary
                         (em.py:289-307), exterior state -(incident data):
                         the bdry argument's [F][n] values, or zero (the
                         reference's default incident_bc) when it is NULL */
};

typedef struct hb_discr hb_discr;
typedef struct hb_op hb_op;

/* Reference element + mesh geometry of one discretization, host FP64.
 * geometry: [K][G], G = dim*dim + nfaces*(dim+1); per element first
 *   d(r_a)/d(x_b) at [a*dim + b], then per face f its outward unit normal
 *   (dim values) and Fscale = face Jacobian / |element Jacobian|. */
typedef struct {
  int32_t dim, order, np, nfp, nfaces, nperm;
  int64_t num_elements;
  const double* dmats;     /* [dim][np][np] row-major: D_r = V_r V^-1 */
  const double* lift;      /* [np][nfaces*nfp]: LIFT = M^-1 E */
  const double* geometry;  /* [K][G] */
  const int32_t* fmask;    /* [nfaces][nfp] local node of each face node */
  const int32_t* shuffle;  /* [nperm][nfp] face-node shuffle per vertex perm */
  int32_t device;          /* CUDA device ordinal */
  const double* unit_nodes;/* [np][dim] reference-element nodes (r, s, t) */
  const double* mass;      /* [np][np] reference mass matrix (V V^T)^-1 */
  const double* abs_jacobian; /* [K] |det A| of each element's map */
} hb_discr_desc;

/* Replaces the device-side part of Discretization.__init__ /
 * _calculate_local_matrices (hedge/discretization/__init__.py:217-262,
 * 440-453): uploads operators and geometry once. */
hb_status hb_discr_create(const hb_discr_desc* desc, hb_discr** out);
hb_status hb_discr_destroy(hb_discr* discr);

/* One compiled model operator.  conn: host [K][nfaces][2] int32,
 * interior face: (neighbour element, nbr_face | perm_id << 2);
 * boundary face: (-1 - b, bc kind), b = the face's number in the
 * BC_GIVEN (or Maxwell HB_BC_INCIDENT) boundary vector (nodes
 * b*nfp .. b*nfp+nfp-1); num_given_bdry_nodes = that vector's length. */
/* Quadrature matrices of one reference element for one degree
 * (hedge/discretization/local.py:545-690, QuadratureInfo), host FP64,
 * row-major.  Weights are the reference element's: d r / d x and
 * Fscale = face Jacobian / |J| are applied per element. */
typedef struct {
  int32_t nq;                /* volume quadrature points */
  int32_t nqf;               /* quadrature points per face */
  const double* vol_interp;  /* [nq][np]: nodal values -> volume points */
  const double* vol_project; /* [dim][np][nq]: M^-1 (d phi_i / d r_r at q)^T w_q */
  const double* face_interp; /* [nfaces][nqf][nfp]: face f's nodes (fmask order)
                                -> its quadrature points */
  const double* face_lift;   /* [np][nfaces*nqf]: M^-1 phi_i(face point) w_face */
} hb_quad_desc;

typedef struct {
  int32_t model, num_fields, precision;
  int32_t flux_type, bdry_flux_type;
  double v[3];             /* advection velocity */
  double c;                /* constant wave speed */
  double eps, mu;          /* Maxwell material */
  double alpha, bdry_alpha;/* Maxwell numeric flux weight (1 = upwind) */
  double time_sign;        /* variable-velocity wave */
  const int32_t* conn;
  int64_t num_given_bdry_nodes;
  int64_t num_halo_faces;  /* faces whose neighbour lives on another partition
                              (conn neighbour K + h, h < num_halo_faces); their
                              ext values come from hb_op_set_halo; 0 = none */
  const hb_quad_desc* quadrature; /* HB_MODEL_VARADV: the quadrature grid (copied
                              at create); NULL for every other model.  Replaces
                              Discretization.get_quadrature_info
                              (hedge/discretization/__init__.py:779-889). */
} hb_op_desc;

/* Replaces Discretization.compile -> jit Executor construction
 * (hedge/discretization/__init__.py:1288-1302,
 *  hedge/backends/jit/__init__.py:366-438). */
hb_status hb_op_create(hb_discr* discr, const hb_op_desc* desc, hb_op** out);
hb_status hb_op_destroy(hb_op* op);

/* rhs = RHS(q).  Replaces Executor.__call__ (hedge/backends/jit/__init__.py:
 * 521-523): diff batch (jit/diff.py:137-175), chain rule vector expressions,
 * flux gather interior + boundary (jit/flux.py:239-480), lift
 * (jit/lift.py:110-141) and inverse mass (jit/__init__.py:501-519).
 * q, rhs: [F][K*Np] in the operator's state dtype.  coeff: var-c wave
 * speed [K*Np] FP64, or the variable-coefficient advection velocity
 * [dim][K*Np] FP64, or for the Maxwell models the material [eps | mu]
 * [2][K*Np] FP64 (variable material, em.py:38-100, 309-371; NULL: the
 * descriptor's eps, mu; CUDA-core precisions only, no halo faces) (else
 * NULL); bdry: BC_GIVEN values [n] FP64, or for the Maxwell models the
 * incident data [F][n] FP64 (exterior state -data on HB_BC_INCIDENT faces;
 * NULL: zero data; CUDA-core precisions only), n = num_given_bdry_nodes
 * (else NULL);
 * source: var-c / constant-c wave source on u, [K*Np] FP64 (else NULL). */
hb_status hb_rhs(hb_op* op, const void* q, void* rhs, const double* coeff,
                 const double* bdry, const double* source, void* stream);

/* Fused LSRK stage: res = a*res + dt*RHS(q_in); q_out = q_in + b*res.
 * Replaces one pass of the LSRK4TimeStepper loop body
 * (hedge/timestep/runge_kutta.py:123-128).  q_out must not alias q_in. */
hb_status hb_lsrk_stage(hb_op* op, double a, double b, double dt,
                        const void* q_in, void* q_out, void* res,
                        const double* coeff, const double* bdry,
                        const double* source, void* stream);

/* hb_rhs / hb_lsrk_stage for the elements [el_begin, el_end) of the
 * operator's K only (the other elements' outputs are left as they are; the
 * inputs are the whole [F][K*Np] vectors).  They split one stage of an
 * element partition into the elements without halo faces, launched while
 * the face traces of the cut faces are exchanged, and the elements with
 * halo faces, launched once the halo buffer is filled: the reference posts
 * its trace exchange as futures and evaluates the local terms in between
 * (hedge/backends/mpi/__init__.py:184-216, hedge/compiler.py:414-467).
 * HB_ERR_INVALID_ARGUMENT for a range outside [0, K]; HB_ERR_UNSUPPORTED
 * for a partial range of the quadrature operator. */
hb_status hb_rhs_elements(hb_op* op, int64_t el_begin, int64_t el_end, const void* q,
                          void* rhs, const double* coeff, const double* bdry,
                          const double* source, void* stream);
hb_status hb_lsrk_stage_elements(hb_op* op, int64_t el_begin, int64_t el_end, double a,
                                 double b, double dt, const void* q_in, void* q_out,
                                 void* res, const double* coeff, const double* bdry,
                                 const double* source, void* stream);

/* out = a*x + b*y, n elements of dtype (0 = FP64, 1 = FP32).  Replaces
 * NumpyLinearCombiner (hedge/vector_primitives.py:58-77). */
hb_status hb_lincomb(int64_t n, int32_t dtype, double a, const void* x,
                     double b, const void* y, void* out, void* stream);

/* The face gather maps the kernels use, expanded on the device: for every
 * element face node (e, f, i) in [K][nfaces][nfp] order, the int volume
 * index and the ext volume index (interior) or -1 - boundary node
 * (boundary).  Device int64 buffers of K*nfaces*nfp entries.  Replaces the
 * face-pair index lists of hedge/discretization/data.py:199-248. */
hb_status hb_gather_map(hb_op* op, int64_t* int_idx, int64_t* ext_idx,
                        void* stream);

/* out[0] = sqrt(sum_f sum_k |J_k| u_fk^T M u_fk): the L2 (energy) norm of
 * nfields volume vectors u [nfields][K*Np] of dtype (0 = FP64, 1 = FP32),
 * accumulated in FP64 with a fixed-order (deterministic) reduction.  out is
 * one device double.  Replaces Discretization.norm
 * (hedge/discretization/__init__.py:1126-1139). */
hb_status hb_norm(hb_discr* discr, int32_t nfields, int32_t dtype, const void* u,
                  double* out, void* stream);

/* Allocation-free variant of hb_norm.  This entry point has no counterpart in
 * the reference.  It is for callers that may not allocate device memory while
 * they run: code that holds no hb_discr and brings its own device copies of
 * the element mass matrix `mass` [np][np] (FP64) and |J_k| `abs_jacobian`
 * [num_elements] (FP64), inside a time loop that has reserved the device's
 * memory for its fields or must not let an allocation synchronise the device
 * between steps.  Same result and reduction order as hb_norm on the current
 * CUDA device; u and out as for hb_norm, all pointers on the current device
 * (a pointer that is not device or managed memory of the current device is
 * rejected with HB_ERR_INVALID_ARGUMENT before any launch).
 *
 * The partial sums go to a fixed device array inside the library of
 * HB_NORM_NOALLOC_MAX_BLOCKS doubles (64 KiB), so the call allocates nothing.
 * Limit: num_elements <= HB_NORM_NOALLOC_MAX_BLOCKS * max(1, 256 / np)
 * (e.g. 57344 tetrahedra at order 4, np = 35); larger meshes are rejected
 * with HB_ERR_INVALID_ARGUMENT and must use hb_norm.
 * The first call on a device looks up the array's device address (which may
 * load the library's device code) and should come before any stream capture.
 * The array keeps the last call's contents; nothing in it has to start at
 * zero, since each call writes every partial it reads.  Calls whose kernels
 * overlap on one device (several streams or host threads) share the array and
 * race: serialise them. */
#define HB_NORM_NOALLOC_MAX_BLOCKS 8192
hb_status hb_norm_noalloc(int64_t num_elements, int32_t np, int32_t nfields,
                          int32_t dtype, const double* mass, const double* abs_jacobian,
                          const void* u, double* out, void* stream);

/* Adjoint of the right-hand side, FP64.  For R(q; c) as evaluated by hb_rhs
 * with this operator, and a cotangent lam [F][K*Np] of R:
 *   q_bar = (dR/dq)^T lam                        [F][K*Np], overwritten
 *   c_bar = (dR/dc)^T lam at the state q         [K*Np] per node of the c field,
 *           overwritten; variable-velocity wave only, else pass NULL.
 * R is linear in q (given boundary data and sources are constants), so q_bar
 * does not depend on q, which may be NULL when c_bar is NULL.  coeff is the c
 * field the forward used (variable-velocity wave).  work: device scratch of
 * hb_rhs_adjoint_work_size() bytes, owned by the caller.  The transposed
 * lift, differentiation and the scatter-add back through the face-pair map
 * (written as a gather over the matched neighbour face points) adjoin
 * jit/diff.py:137-175, jit/flux.py:239-480 (ext_native_write_map) and
 * jit/lift.py:110-141; the reference has no adjoint of its own. */
hb_status hb_rhs_adjoint_work_size(hb_op* op, int64_t* bytes);
hb_status hb_rhs_adjoint(hb_op* op, const double* q, const double* lam, double* q_bar,
                         double* c_bar, const double* coeff, void* work, void* stream);

/* Batched ensemble: one launch per LSRK stage advances many independent
 * discretizations of uneven size and order.  Each member is a compiled
 * operator (advection or constant-c wave, HB_PREC_FP32, no given boundary
 * data) with two FP32 state buffers q0, q1 [F][K*Np], an FP64 residual res
 * [F][K*Np] (zero before the first stage), its own time step dt and tile
 * size (elements per tile; 0 = 256 / Np).  A stage with parity p computes,
 * for every member, res = a*res + dt*RHS(q_p) (RHS in FP32, residual FP64)
 * and q_(1-p) = q_p + b*res (FP64 arithmetic, stored FP32).  The batch
 * descriptor owns its instance and tile tables; members' buffers stay the
 * caller's.  No reference counterpart: the reference advances one
 * discretization at a time (hedge/timestep/runge_kutta.py:104-131). */
typedef struct hb_batch hb_batch;
typedef struct {
  hb_op* op;
  float* q0;
  float* q1;
  double* res;
  double dt;
  int32_t tile_elems;
} hb_batch_member;
hb_status hb_batch_create(const hb_batch_member* members, int32_t n, hb_batch** out);
hb_status hb_batch_destroy(hb_batch* batch);
hb_status hb_batch_stage(hb_batch* batch, double a, double b, int32_t parity, void* stream);
/* up to n of {tiles, grid, threads per CTA, dynamic shared bytes, DOFs} */
hb_status hb_batch_info(hb_batch* batch, int64_t* info, int32_t n);
/* synchronises `stream`; HB_ERR_DEVICE_FLAG if a stage met bad face data */
hb_status hb_batch_check(hb_batch* batch, void* stream);

/* Element-partitioned operators (several devices or processes, one
 * partition each): a face whose neighbour lives on another partition is
 * coded (K + h, nbr_face | perm << 2) with h < num_halo_faces, and its ext
 * values are read from a halo buffer [num_halo_faces * nfp][F] (state dtype;
 * row h*nfp + k = the neighbour's values at this face's node k, already in
 * this face's node order) and, for the variable-velocity wave, halo_coeff
 * [num_halo_faces * nfp].  Both are device buffers of the caller, refreshed
 * between stages (typically by hb_pack on the owner + a point-to-point
 * exchange).  Every kernel path reads it (CUDA cores, the resident and the
 * streamed split kernels).  Replaces the reference's MPI face-trace
 * exchange (hedge/backends/mpi/__init__.py:184-216, 284-340). */
hb_status hb_op_set_halo(hb_op* op, const void* halo, const double* halo_coeff);

/* dst[j * nfields + f] = src[f * field_stride + idx[j]], j < n: packs the
 * volume values a peer needs (idx device int64) for the halo exchange;
 * dtype 0 = FP64, 1 = FP32. */
hb_status hb_pack(int64_t n, int32_t dtype, int32_t nfields, int64_t field_stride,
                  const int64_t* idx, const void* src, void* dst, void* stream);

/* Synchronises `stream` and returns HB_ERR_DEVICE_FLAG if a kernel of this
 * operator flagged bad input (out-of-range neighbour or code, missing
 * boundary vector) or a bounded wait of a tensor-core kernel ran out.  The
 * first flag raised since the last check is reported, once: the check clears
 * it, so the operator can be launched again afterwards.  The reference
 * raises a Python exception per call instead (e.g. the generated size checks
 * of hedge/backends/jit/diff.py:111-126). */
hb_status hb_op_check(hb_op* op, void* stream);

/* Failure-detection self-test, no reference counterpart: launches one CTA
 * that allocates tensor memory as the split-precision kernels do, waits on an
 * mbarrier that nothing arrives on with their bounded wait (limit_ns, 1 us to
 * 2 s), raises this operator's device error flag when the wait runs out,
 * releases the tensor memory and returns.  Nothing else is in flight.  A
 * following hb_op_check returns HB_ERR_DEVICE_FLAG, and the operator (and the
 * CUDA context) stays usable. */
hb_status hb_op_wait_selftest(hb_op* op, int64_t limit_ns, void* stream);

/* Launch configuration chosen at hb_op_create, for diagnostics: up to n of
 * {grid, threads per CTA, dynamic shared bytes, elements per batch,
 *  operators in shared memory (0/1), CTAs per SM}. */
hb_status hb_op_launch_info(hb_op* op, int64_t* info, int32_t n);

/* Thread-local text of the last error. */
const char* hb_last_error_string(void);

#ifdef __cplusplus
}
#endif

#endif /* HEDGE_B200_H */
