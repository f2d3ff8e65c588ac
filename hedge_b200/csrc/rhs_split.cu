// Split-precision (BF16x3 / FP16x3) fused DG right-hand side + LSRK stage on
// the sm_100a tensor cores (tcgen05.mma kind::f16, FP32 accumulation in TMEM).
//
// The two contractions of the DG operator run as GEMMs whose M dimension is
// the batch's (element, field) pairs -- one TMEM lane per pair, EPW = 32/F
// elements per 32-lane quadrant, EB = 4*EPW elements per batch:
//
//   diff:  C[(e,f)][(r,i)] = sum_j q[(e,f)][j] * D_r[i][j]
//          A = state (K-major, j contiguous), B = [D_r]^T stacked over r,
//          M = 128, N = dim*Np (padded to 16), K = Np (padded to 16)
//   lift:  L[(e,f)][i] = sum_p flux[(e,f)][p] * LIFT[i][p]
//          A = face fluxes, B = LIFT^T, M = 128, N = Np, K = Nf*Nfp
//
// Each operand x is split into 16-bit planes hi = h(x), lo = h(x - hi); a
// product is hi*hi + hi*lo + lo*hi, accumulated in FP32.  The operator planes
// are built once on the host in the tensor core's canonical K-major layout
// and stay resident in shared memory; the state and flux planes are written
// per batch.  The state is split after subtracting its element-wise linear
// interpolant through the vertex nodes (D_r maps it to constants that the
// epilogue adds back exactly), so only the within-element variation goes
// through 16 bits; face jumps are formed in FP64.
//
// One CTA per SM runs a persistent loop over batches with warp roles:
//   * an I/O warp streams each batch's FP64 state, geometry and face table
//     into one of two stage buffers (bulk copies, completion counted on an
//     mbarrier) while the previous batch is computed, the batch's residual
//     into a residual buffer where one fits, and prefetches the upcoming
//     states and residuals into L2;
//   * an MMA warp issues the diff and lift MMAs once the consumers have
//     written the state and flux planes;
//   * 20 consumer warps split the state, evaluate the face fluxes into the
//     lift planes, read the accumulators back (chain rule and volume terms
//     first, parked in spare TMEM columns, then + lift: one lane holds every
//     derivative of its (e, f); the model's curl/div/grad gather the
//     element's other fields with warp shuffles) into FP32 rhs rows in
//     shared memory, and then apply the FP64 stage update in a coalesced
//     pass that writes q_out and the residual straight to global memory.
//     Where the buffers allow, each warp splits batch i + 1 between the
//     volume terms and the lift epilogue of batch i (software pipeline), so
//     the lift MMA's latency overlaps that work.
// All waits are bounded (2 s); a timeout sets the device error flag and the
// CTA leaves after releasing its TMEM.  Element shapes are compile-time
// (template on the order).  Restated reference loops: jit/diff.py:137-175,
// jit/flux.py:311-353 and 429-472, jit/lift.py:110-141,
// jit/__init__.py:501-519, timestep/runge_kutta.py:123-128.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <type_traits>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "models.cuh"
#include "tc.cuh"

namespace hb {

hb_status ensure_fp32(Discr* d);

// Consumer warps (the phases of a batch; a multiple of 4: warp w reads TMEM
// lane quadrant w % 4), one I/O warp that streams the next batches' state
// (and residual) into shared memory, and one warp that issues the
// tensor-core MMAs.  Registers are split over the SM's 4 sub-partitions
// (16K each) by warp: 22 warps put at most 6 warps on one, which leaves 80
// registers per thread.  20 consumer warps give one element (face phase) and
// one state-split item per warp in a 20-element Maxwell batch; across the
// built instances (K ~ 48000-51000) they run 2-19 % faster than 12.
#ifndef HB_SPLIT_NCW
#define HB_SPLIT_NCW 20
#endif
constexpr int NCW = HB_SPLIT_NCW;
// coalesced update: 16-byte accesses where the alignment allows
#ifndef HB_SPLIT_VUPD
#define HB_SPLIT_VUPD 1
#endif
// face-flux phase: elements a consumer warp takes per round (0: the default
// per dimension)
#ifndef HB_SPLIT_ER
#define HB_SPLIT_ER 0
#endif
static_assert(NCW % 4 == 0, "consumer warps must cover the TMEM quadrants evenly");
constexpr int CONSUMERS = NCW * 32;
constexpr int SPLIT_THREADS = CONSUMERS + 64;
// programmatic dependent launch (the next kernel's set-up overlaps the end
// of this one)
#ifndef HB_SPLIT_PDL
#define HB_SPLIT_PDL 1
#endif
// bounded waits (tensor core, producer/consumer hand-offs): 2 s, far above any
// batch's time
constexpr uint64_t MBAR_MAX_NS = 2000000000ull;
// dynamic shared memory one CTA may use on sm_100
constexpr uint32_t SMEM_LIMIT = 232448;

__host__ __device__ constexpr int ru16(int x) { return (x + 15) / 16 * 16; }
__host__ __device__ constexpr int ru32(int x) { return (x + 31) / 32 * 32; }
__host__ __device__ constexpr uint32_t al128(uint32_t x) { return (x + 127u) & ~127u; }
__host__ __device__ constexpr uint32_t al16(uint32_t x) { return (x + 15u) & ~15u; }
__host__ __device__ constexpr uint32_t al1024(uint32_t x) { return (x + 1023u) & ~1023u; }

// Compile-time shape of one (model, dim, order) instance with a state of SB
// bytes per value (8: FP64, 4: FP32).
template <int MODEL, int DIM, int ORDER, int SB = 8>
struct Shape {
  static constexpr int F = Traits<MODEL, DIM>::F;
  static constexpr int C = Traits<MODEL, DIM>::COEFF;
  static constexpr int NA = F + C;
  static constexpr int NP = DIM == 2 ? (ORDER + 1) * (ORDER + 2) / 2
                                     : (ORDER + 1) * (ORDER + 2) * (ORDER + 3) / 6;
  static constexpr int NFP = DIM == 2 ? ORDER + 1 : (ORDER + 1) * (ORDER + 2) / 2;
  static constexpr int NF = DIM + 1;
  static constexpr int NFPT = NF * NFP;
  static constexpr int G = DIM * DIM + NF * (DIM + 1);
  static constexpr int EPW = 32 / F;
  static constexpr int EB = 4 * EPW;
  static constexpr int KD = ru16(NP), KL = ru16(NFPT);
  static constexpr int ND = ru16(DIM * NP), NL = ru16(NP);
  static constexpr int LIFT_COL = ru32(ND);
  // Field stride (in values) of the staged state and residual: the EB * NP
  // values of a field, padded so that the consumer lanes' rows (lane =
  // element * F + field) at one node hit distinct shared-memory banks as far
  // as the layout allows (worst lanes per bank: 8-byte bank pairs in a
  // half-warp for FP64, 4-byte banks in a warp for FP32), and to 16-byte rows.
  static constexpr int LPW = SB == 8 ? 16 : 32;   // lanes per wavefront
  static constexpr int VPR = 16 / SB;             // values per 16 bytes
  static constexpr int bank_collisions(int stride) {
    int worst = 0;
    for (int g = 0; g < 32 / LPW; ++g) {
      int count[32] = {};
      for (int l = LPW * g; l < LPW * g + LPW; ++l) {
        if (l / F >= EPW) continue;
        const int b = ((l % F) * stride + (l / F) * NP) % LPW;
        if (++count[b] > worst) worst = count[b];
      }
    }
    return worst;
  }
  static constexpr int padded_fnp() {
    const int base = SB == 8 ? EB * NP : (EB * NP + VPR - 1) / VPR * VPR;
    int best = base, bw = bank_collisions(base);
    for (int p = VPR; p < 32; p += VPR) {
      const int c = bank_collisions(base + p);
      if (c < bw) { bw = c; best = base + p; }
    }
    return best;
  }
  static constexpr int FNP = padded_fnp();        // >= EB * NP, even (16-byte rows)
  static constexpr int NVAL = F * FNP;
  static constexpr int NFACE = EB * NFPT;
  static constexpr int NFV = (NFACE + CONSUMERS - 1) / CONSUMERS;
  // epilogue: the NCW/4 warps of a TMEM quadrant split the nodes, NPQ each
  // (a multiple of 4: TMEM is read 4 columns at a time)
  static constexpr int NPQ = (((NP + NCW / 4 - 1) / (NCW / 4)) + 3) & ~3;
  // split pass: (quadrant, 8-column chunk) items, IPW per consumer warp
  static constexpr int NITEM = 4 * (KD / 8);
  static constexpr int IPW = (NITEM + NCW - 1) / NCW;

  // rhs staging rows (FP32, aliasing the state planes once the diff MMA has
  // read them): NPR floats per (element, field) row, 16-byte aligned
  static constexpr int NPR = (NP + 3) & ~3;
  // flux planes in the 128-byte swizzled K-major layout when a row is exactly
  // one swizzle atom wide (64 K entries): the face phase's stores of one row's
  // consecutive face points then fall in distinct banks
  static constexpr bool FSW = KL == 64;

  static constexpr uint32_t bD = ND * KD * 2, bL = NL * KL * 2;
  static constexpr uint32_t bAq = 128 * KD * 2, bAf = 128 * KL * 2;
  static constexpr uint32_t bState = NVAL * SB;
  // one stage buffer: state [F][EB][NP] FP64, geometry [EB][G] FP32,
  // face table [EB][NF] int2, coefficient [EB][NP] FP64
  static constexpr uint32_t sGeo = bState;
  static constexpr uint32_t sConn = al16(sGeo + EB * G * 4);
  static constexpr uint32_t sCoef = al16(sConn + EB * NF * 8);
  static constexpr uint32_t bStage = al128(sCoef + (C ? FNP * 8 : 0));

  static constexpr uint32_t oDh = 0;
  static constexpr uint32_t oDl = al128(oDh + bD);
  static constexpr uint32_t oLh = al128(oDl + bD);
  static constexpr uint32_t oLl = al128(oLh + bL);
  static constexpr uint32_t oAqh = al128(oLl + bL);
  static constexpr uint32_t oAql = al128(oAqh + bAq);
  static constexpr uint32_t oAfh = FSW ? al1024(oAql + bAq) : al128(oAql + bAq);
  static constexpr uint32_t oAfl = FSW ? al1024(oAfh + bAf) : al128(oAfh + bAf);
  static constexpr uint32_t ostg = al128(oAfl + bAf);
  static constexpr uint32_t SMALL = 1024 + NFPT + 6 * NF * NFP + 4 + 768 * 4 + 96;
  // FP32 rhs rows [128][NPR]: a buffer of their own when it fits next to the
  // stage buffers, else aliasing the state planes (free once the diff MMA
  // has read them; the state split rewrites every plane column each batch)
  static constexpr uint32_t bRhs = al128(128u * NPR * 4u);
  static_assert(128u * NPR * 4u <= 2u * bAq, "rhs staging must fit in the state planes");
  // double-buffered stages when they fit, else one; then the rhs rows' own
  // buffer; then a residual buffer (the I/O warp loads the batch's residual
  // one batch ahead; without it the update reads the residual from global
  // memory)
  static constexpr bool fits(int nstg, bool own_rhs, bool res) {
    return ostg + nstg * bStage + (own_rhs ? bRhs : 0) + (res ? bState : 0) + SMALL <=
           SMEM_LIMIT;
  }
  static constexpr int NSTG = fits(2, false, false) ? 2 : 1;
  static constexpr bool RHS_OWN = fits(NSTG, true, false);
  static constexpr bool RES = fits(NSTG, RHS_OWN, true);
  static constexpr uint32_t orhs = RHS_OWN ? ostg + NSTG * bStage : oAqh;
  static constexpr uint32_t ores = ostg + NSTG * bStage + (RHS_OWN ? bRhs : 0);
  static constexpr uint32_t ofm = al16(ores + (RES ? bState : 0));     // uint8 fmask
  // uint8 neighbour node of face node k seen through (perm, neighbour face):
  // fmask[nface][shuffle[perm][k]] at [(perm * NF + nface) * NFP + k]
  static constexpr uint32_t osh = al16(ofm + NFPT);
  static constexpr uint32_t overt = al16(osh + 6 * NF * NFP);          // uint8 vertex nodes
  // row maxima (FP16 planes): state rows [2][128] then flux rows [2][128]
  static constexpr uint32_t ors = al16(overt + 4);
  static constexpr uint32_t obar = al16(ors + 768 * 4);                // mbarriers + TMEM slot
  static constexpr uint32_t total = al16(obar + 96);
  static constexpr uint32_t LIN_BYTES = 8 + NP * DIM * 8;  // vertex nodes + weights (image)
  // epilogue: the volume terms are formed before the lift MMA completes and
  // parked in TMEM columns [VCOL, ...), NPQ per consumer part of a lane
  // quadrant, wherever those columns fit in TMEM
  static constexpr int VCOL = LIFT_COL + NL + 4;
  static constexpr bool PARK = VCOL + (NCW / 4) * NPQ <= 512;
  static constexpr int TMEM_NEED = VCOL + (PARK ? (NCW / 4) * NPQ : 0);
  static constexpr uint32_t TMEM_COLS = TMEM_NEED <= 32 ? 32 : TMEM_NEED <= 64 ? 64
                                        : TMEM_NEED <= 128 ? 128 : TMEM_NEED <= 256 ? 256 : 512;
  static constexpr bool FITS = ND <= 256 && NL <= 256 && TMEM_NEED <= 512 &&
                               total <= SMEM_LIMIT;
};

template <typename ST>
struct SplitArgsT {
  int64_t K, nbatch, n_given;
  // the elements [e_begin, e_end) this launch updates (of K); batch b starts
  // at element e_begin + bunit (b bq + min(b, brem)), the last one ends at
  // e_end
  int64_t e_begin, e_end;
  int64_t bq, brem;
  int bunit;
  int nperm;
  const uint8_t* ops;   // [D_hi | D_lo | L_hi | L_lo] canonical images
  const float* geo32;
  const int2* conn;
  const int* fmask;
  const int* shuffle;
  const ST* q_in;
  ST* q_out;
  ST* res;
  const double* coeff;
  const double* bdry;
  const double* source;
  const ST* halo;         // [n_halo * nfp][F] ext values of faces on other partitions
  const double* halo_c;   // [n_halo * nfp] ext c (var-c wave)
  int64_t n_halo;
  double ra, rb, dt;
  float op_scale_d, op_scale_l;   // operator plane scales (powers of two)
  int mode;
  ModelParams mp;
  int* err;
};
using SplitArgs = SplitArgsT<double>;

// the elements of batch b: [batch_first(b), batch_first(b + 1)), the last
// batch ending at K
template <typename A>
__device__ __forceinline__ int64_t batch_first(const A& a, int64_t b) {
  return a.e_begin + (int64_t)a.bunit * (b * a.bq + (b < a.brem ? b : a.brem));
}
template <typename A>
__device__ __forceinline__ int batch_size(const A& a, int64_t b) {
  return (int)((b + 1 >= a.nbatch ? a.e_end : batch_first(a, b + 1)) - batch_first(a, b));
}

// byte offset of element (row, k) in a K-major no-swizzle operand image with
// K padded to kp: 8x8 core matrices (8 rows x 16 bytes), K chunks 128 B
// apart, 8-row groups kp*16 B apart
__host__ __device__ constexpr uint32_t kmajor_off(int row, int k, int kp) {
  return (uint32_t)((row >> 3) * (kp * 16) + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// Plane types: BF16 split (PT_BF16, unscaled) or FP16 split of a row scaled
// by a power of two that maps the row's largest magnitude into [2^13, 2^14)
// (PT_FP16: 11 significant bits per plane, so hi*hi + hi*lo + lo*hi is ~8x
// more accurate than the BF16 split at the same tensor-core cost).
enum { PT_BF16 = 0, PT_FP16 = 1 };

template <int PT>
__device__ __forceinline__ void store_split(uint8_t* hi, uint8_t* lo, uint32_t off, float v) {
  if constexpr (PT == PT_BF16) {
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    const __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));
    *reinterpret_cast<__nv_bfloat16*>(hi + off) = h;
    *reinterpret_cast<__nv_bfloat16*>(lo + off) = l;
  } else {
    const __half h = __float2half_rn(v);
    const __half l = __float2half_rn(v - __half2float(h));
    *reinterpret_cast<__half*>(hi + off) = h;
    *reinterpret_cast<__half*>(lo + off) = l;
  }
}

// A plane pair (hi, lo) holds 32 bits per entry: before the FP16 row scale
// is known, an entry's raw FP32 bits are parked there (upper half in hi, lower
// half in lo) and split in place once the row maximum is known.
__device__ __forceinline__ void park_f32(uint8_t* hi, uint8_t* lo, uint32_t off, float v) {
  const uint32_t b = __float_as_uint(v);
  *reinterpret_cast<uint16_t*>(hi + off) = (uint16_t)(b >> 16);
  *reinterpret_cast<uint16_t*>(lo + off) = (uint16_t)(b & 0xffffu);
}
__device__ __forceinline__ float unpark_f32(const uint8_t* hi, const uint8_t* lo, uint32_t off) {
  return __uint_as_float(((uint32_t)*reinterpret_cast<const uint16_t*>(hi + off) << 16) |
                         *reinterpret_cast<const uint16_t*>(lo + off));
}
// the same for 8 consecutive K entries (one 16-byte chunk per plane)
__device__ __forceinline__ void park8(uint8_t* hi, uint8_t* lo, uint32_t off, const float (&v)[8]) {
  uint32_t hw[4], lw[4];
#pragma unroll
  for (int c = 0; c < 8; c += 2) {
    const uint32_t b0 = __float_as_uint(v[c]), b1 = __float_as_uint(v[c + 1]);
    hw[c / 2] = (b1 & 0xffff0000u) | (b0 >> 16);
    lw[c / 2] = (b1 << 16) | (b0 & 0xffffu);
  }
  *reinterpret_cast<uint4*>(hi + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
  *reinterpret_cast<uint4*>(lo + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
}
__device__ __forceinline__ void unpark8(const uint8_t* hi, const uint8_t* lo, uint32_t off,
                                        float (&v)[8]) {
  const uint4 h = *reinterpret_cast<const uint4*>(hi + off);
  const uint4 l = *reinterpret_cast<const uint4*>(lo + off);
  const uint32_t hw[4] = {h.x, h.y, h.z, h.w}, lw[4] = {l.x, l.y, l.z, l.w};
#pragma unroll
  for (int c = 0; c < 8; c += 2) {
    v[c] = __uint_as_float((hw[c / 2] << 16) | (lw[c / 2] & 0xffffu));
    v[c + 1] = __uint_as_float((hw[c / 2] & 0xffff0000u) | (lw[c / 2] >> 16));
  }
}

// power-of-two row scale from the bit pattern of the row's largest |value|
__device__ __forceinline__ float row_scale(uint32_t maxbits) {
  int e = (int)((maxbits >> 23) & 0xffu) - 13;   // max / 2^(e-127) in [2^13, 2^14)
  e = e < 1 ? 1 : (e > 253 ? 253 : e);
  return maxbits == 0 ? 1.0f : __uint_as_float((uint32_t)e << 23);
}
// its exact reciprocal (also a power of two)
__device__ __forceinline__ float row_scale_inv(uint32_t maxbits) {
  int e = (int)((maxbits >> 23) & 0xffu) - 13;
  e = e < 1 ? 1 : (e > 253 ? 253 : e);
  return maxbits == 0 ? 1.0f : __uint_as_float((uint32_t)(254 - e) << 23);
}

// Ampere-style asynchronous 8-byte global -> shared copy (no registers held)
__device__ __forceinline__ void cp_async8(void* sdst, const void* gsrc) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(tc::smem_u32(sdst)), "l"(gsrc)
               : "memory");
}

// models whose numerical flux depends on the state only through the jump
// q- - q+ (so f(q-, q+) == f(q- - q+, 0))
template <int MODEL>
struct JumpLinear { static constexpr bool value = MODEL != HB_MODEL_VARWAVE; };

// The volume term of this lane's own field at one node, from the physical
// gradients g[x] that every lane of the element's F lanes (base..base+F-1)
// holds for its own field; the other fields' gradients come over warp
// shuffles, only the ones the model needs (warp-collective: every lane of
// the warp calls this).
template <int MODEL, int DIM>
__device__ __forceinline__ float volume_own(const ModelParams& mp, const float (&g)[DIM],
                                            int base, int fown, float cnode) {
  constexpr unsigned FULL = 0xffffffffu;
  if constexpr (MODEL == HB_MODEL_ADVECTION) {
    float s = 0.f;
#pragma unroll
    for (int x = 0; x < DIM; ++x) s += (float)mp.v[x] * g[x];
    return -s;
  } else if constexpr (MODEL == HB_MODEL_WAVE || MODEL == HB_MODEL_VARWAVE) {
    // u lane: c div v = c sum_x d_x v_x; v_x lane: c d_x u
    const float c = (MODEL == HB_MODEL_WAVE) ? (float)mp.c : (float)mp.time_sign * cnode;
    float offer = g[0];
#pragma unroll
    for (int x = 1; x < DIM; ++x) offer = (fown == 1 + x) ? g[x] : offer;
    float div = 0.f;
#pragma unroll
    for (int x = 0; x < DIM; ++x) div += __shfl_sync(FULL, offer, base + 1 + x);
    float gu = 0.f;
#pragma unroll
    for (int x = 0; x < DIM; ++x) {
      const float v = __shfl_sync(FULL, g[x], base);
      gu = (fown == 1 + x) ? v : gu;
    }
    return c * (fown == 0 ? div : gu);
  } else {
    // Maxwell: E_c lane: (curl H)_c; H_c lane: -(curl E)_c, with
    // curl(A)_c = d_{c+1} A_{c+2} - d_{c+2} A_{c+1}
    const int c = fown % 3;
    const int other = fown < 3 ? 3 : 0;
    const int c1 = (c + 1) % 3, c2 = (c + 2) % 3;
    float a0[3], a1[3];
#pragma unroll
    for (int x = 0; x < 3; ++x) {
      a0[x] = __shfl_sync(FULL, g[x], base + other + c2);
      a1[x] = __shfl_sync(FULL, g[x], base + other + c1);
    }
    float t0 = a0[0], t1 = a1[0];
#pragma unroll
    for (int x = 1; x < 3; ++x) {
      t0 = (x == c1) ? a0[x] : t0;
      t1 = (x == c2) ? a1[x] : t1;
    }
    const float curl = t0 - t1;
    return fown < 3 ? curl : -curl;
  }
}

// consumer-only barriers (named barrier 1; the I/O and MMA warps never join)
__device__ __forceinline__ void cbar() {
  asm volatile("bar.sync 1, %0;" ::"n"(CONSUMERS) : "memory");
}
__device__ __forceinline__ int cbar_or(int v) {
  int r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.s32 p, %1, 0;\n\t"
      "bar.red.or.pred q, 1, %2, p;\n\t"
      "selp.s32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"(v), "n"(CONSUMERS)
      : "memory");
  return r;
}
__device__ __forceinline__ void cp_async4(void* sdst, const void* gsrc) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(tc::smem_u32(sdst)), "l"(gsrc)
               : "memory");
}
// the mbarrier counts one arrival once all earlier cp.async of this thread landed
__device__ __forceinline__ void cp_async_arrive(uint64_t* mbar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(tc::smem_u32(mbar))
               : "memory");
}
__device__ __forceinline__ void cp_async_drain() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}
// bulk (untiled, no multicast) copies: 16-byte aligned addresses and sizes
__device__ __forceinline__ void mbar_expect_tx(uint64_t* mbar, uint32_t bytes) {
  asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;"
               ::"r"(tc::smem_u32(mbar)), "r"(bytes)
               : "memory");
}
// pull a 16-byte-aligned range into L2 in the background (no destination)
__device__ __forceinline__ void prefetch_l2(const void* gsrc, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(gsrc), "r"(bytes) : "memory");
}
// one arrival on `mbar` that also announces `bytes` of transactions
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
               ::"r"(tc::smem_u32(mbar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_load(void* sdst, const void* gsrc, uint32_t bytes,
                                          uint64_t* mbar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(tc::smem_u32(sdst)), "l"(gsrc), "r"(bytes), "r"(tc::smem_u32(mbar))
      : "memory");
}
__device__ __forceinline__ void bulk_store(void* gdst, const void* ssrc, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;"
               ::"l"(gdst), "r"(tc::smem_u32(ssrc)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_all() {
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}
// Programmatic dependent launch: wait until the preceding kernel of the
// stream has completed and its memory is visible (a no-op without the launch
// attribute); then allow the next kernel to be scheduled.
__device__ __forceinline__ void grid_dep_wait() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}
__device__ __forceinline__ void grid_dep_launch() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ bool aligned16(const void* p, uint32_t bytes) {
  return ((reinterpret_cast<uintptr_t>(p) | bytes) & 15u) == 0;
}

// One contiguous range global -> shared: a bulk copy (counted as transaction
// bytes on `mbar`, announced beforehand) when aligned, else 8- or 4-byte
// cp.async by the warp's lanes (counted by their arrivals).
template <typename T>
__device__ __forceinline__ void stage_in(T* sdst, const T* gsrc, int n, int lane,
                                         uint64_t* mbar) {
  const uint32_t bytes = (uint32_t)n * sizeof(T);
  if (n <= 0) return;
  if (aligned16(gsrc, bytes)) {
    if (lane == 0) bulk_load(sdst, gsrc, bytes, mbar);
    return;
  }
  for (int x = lane; x < n; x += 32) {
    if constexpr (sizeof(T) == 8) cp_async8(sdst + x, gsrc + x);
    else cp_async4(sdst + x, gsrc + x);
  }
}
template <typename T>
__device__ __forceinline__ uint32_t bulk_bytes(const T* gsrc, int n) {
  const uint32_t bytes = (uint32_t)n * sizeof(T);
  return (n > 0 && aligned16(gsrc, bytes)) ? bytes : 0u;
}
// One contiguous range shared -> global (bulk store when aligned, else lanes).
__device__ __forceinline__ void stage_out(double* gdst, const double* ssrc, int n, int lane) {
  const uint32_t bytes = (uint32_t)n * 8u;
  if (n <= 0) return;
  if (aligned16(gdst, bytes)) {
    if (lane == 0) bulk_store(gdst, ssrc, bytes);
  } else {
    for (int x = lane; x < n; x += 32) gdst[x] = ssrc[x];
  }
}

// mbarriers
enum {
  MB_DIFF = 0,      // diff MMAs done (tcgen05.commit)
  MB_LIFT = 1,      // lift MMAs done
  MB_FULL = 2,      // 2..3: stage buffer loaded
  MB_AREADY = 4,    // every consumer warp wrote its state-plane rows
  MB_FREADY = 5,    // every consumer warp wrote its flux-plane entries
  MB_DONE = 6,      // 6..7: every consumer warp is done with that stage buffer
  MB_RES_FULL = 8,  // residual buffer loaded
  MB_COUNT = 9
};

// FP64 weights (1 + r_d)/2 of every node of the reference element, per
// (dimension, order) of the resident kernel: the element's linear interpolant
// through its vertex nodes is v0 + sum_d lam[j][d] (v_d - v0).  Read by the
// whole warp at one address (constant cache, not the shared-memory pipe).
constexpr int LAM_MAX = 56 * 3;   // up to 3D N = 5 (Np = 56)
constexpr int LAM_ORDERS = 7;     // orders 0..6
__constant__ double c_lam[2][LAM_ORDERS][LAM_MAX];
__constant__ float c_lamf[2][LAM_ORDERS][LAM_MAX];   // the same, FP32 (FP32 state)

// byte offset of (row, k) in a flux plane: the 128-byte swizzled K-major
// layout (8-row atoms of 128-byte rows, 16-byte chunk index XOR row & 7) when
// SW, else the plain K-major core-matrix layout
template <bool SW>
__device__ __forceinline__ uint32_t fplane_off(int row, int k, int kp) {
  if constexpr (SW)
    return (uint32_t)((row >> 3) * 1024 + (row & 7) * 128 + (((k >> 3) ^ (row & 7)) << 4) +
                      (k & 7) * 2);
  else
    return kmajor_off(row, k, kp);
}

// barrier of the NCW / 4 consumer warps that read one TMEM lane quadrant
// (named barriers 2..5)
__device__ __forceinline__ void qbar(int quad) {
  asm volatile("bar.sync %0, %1;" ::"r"(2 + quad), "n"(32 * (NCW / 4)) : "memory");
}

template <int MODEL, int DIM, int ORDER, int PT, typename ST>
__global__ void __launch_bounds__(SPLIT_THREADS, 1) rhs_split_kernel(SplitArgsT<ST> a) {
  using S = Shape<MODEL, DIM, ORDER, (int)sizeof(ST)>;
  constexpr int F = S::F, C = S::C, NA = S::NA, NP = S::NP, NFP = S::NFP, NF = S::NF;
  constexpr int NFPT = S::NFPT, G = S::G, EPW = S::EPW, EB = S::EB, FNP = S::FNP;
  constexpr int KD = S::KD, KL = S::KL, NSTG = S::NSTG, NPR = S::NPR;
  constexpr bool FSW = S::FSW;
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* Aqh = smem + S::oAqh;
  uint8_t* Aql = smem + S::oAql;
  uint8_t* Afh = smem + S::oAfh;
  uint8_t* Afl = smem + S::oAfl;
  float* rhs_s = reinterpret_cast<float*>(smem + S::orhs);  // [128][NPR] FP32 rhs rows
  const ST* lamc;                                            // [NP][DIM] interpolant weights
  if constexpr (sizeof(ST) == 8) lamc = reinterpret_cast<const ST*>(&c_lam[DIM - 2][ORDER][0]);
  else lamc = reinterpret_cast<const ST*>(&c_lamf[DIM - 2][ORDER][0]);
  ST* rbuf = reinterpret_cast<ST*>(smem + S::ores);          // residual [F][EB][NP]
  uint8_t* sfm = smem + S::ofm;
  uint8_t* ssh = smem + S::osh;
  const uint8_t* svert = smem + S::overt;                  // vertex nodes B, C(, D)
  uint32_t* rsq = reinterpret_cast<uint32_t*>(smem + S::ors);        // [2][128] state rows
  uint32_t* rsf = reinterpret_cast<uint32_t*>(smem + S::ors) + 256;  // [2][128] flux rows
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + S::obar);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + S::obar + 8 * MB_COUNT);

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;

  // ---- one-time set-up: resident operators, zeroed operand planes ----
  {
    constexpr uint32_t dD = S::bD, dL = S::bL;
    constexpr uint32_t nchunk = (2 * dD + 2 * dL) / 16;
    const uint4* src = reinterpret_cast<const uint4*>(a.ops);
    for (uint32_t x = tid; x < nchunk; x += SPLIT_THREADS) {
      const uint32_t b = x * 16;
      uint32_t o;
      if (b < dD) o = S::oDh + b;
      else if (b < 2 * dD) o = S::oDl + (b - dD);
      else if (b < 2 * dD + dL) o = S::oLh + (b - 2 * dD);
      else o = S::oLl + (b - 2 * dD - dL);
      *reinterpret_cast<uint4*>(smem + o) = src[x];
    }
    // the planes' K padding and unused rows: zero (the flux planes' are never
    // written again; the state planes' padding chunks are rewritten per batch
    // only where the rhs rows alias them)
    const uint4 z = make_uint4(0, 0, 0, 0);
    for (uint32_t o = S::oAqh + tid * 16; o < S::ostg; o += SPLIT_THREADS * 16)
      *reinterpret_cast<uint4*>(smem + o) = z;
    {
      // image tail: 4 vertex-node bytes (the FP64 weights are in c_lam)
      const uint8_t* lsrc = a.ops + 2 * dD + 2 * dL;
      if (tid < 4) smem[S::overt + tid] = lsrc[tid];
    }
    for (int x = tid; x < NFPT; x += SPLIT_THREADS) sfm[x] = (uint8_t)a.fmask[x];
    for (int x = tid; x < a.nperm * NF * NFP; x += SPLIT_THREADS) {
      const int perm = x / (NF * NFP), r = x - perm * (NF * NFP);
      const int nface = r / NFP, k = r - nface * NFP;
      ssh[x] = (uint8_t)a.fmask[nface * NFP + a.shuffle[perm * NFP + k]];
    }
    for (int x = tid; x < 768; x += SPLIT_THREADS) rsq[x] = 0u;
    if (tid == 0) {
      tc::mbar_init(&mbar[MB_DIFF], 1);
      tc::mbar_init(&mbar[MB_LIFT], 1);
      tc::mbar_init(&mbar[MB_FULL], 32);
      tc::mbar_init(&mbar[MB_FULL + 1], 32);
      tc::mbar_init(&mbar[MB_AREADY], NCW);
      tc::mbar_init(&mbar[MB_FREADY], NCW);
      tc::mbar_init(&mbar[MB_DONE], NCW);
      tc::mbar_init(&mbar[MB_DONE + 1], NCW);
      tc::mbar_init(&mbar[MB_RES_FULL], 32);
      // the swizzled flux planes need 1024-byte aligned atoms
      if (FSW && (tc::smem_u32(smem) & 1023u) != 0u) atomicCAS(a.err, 0, DEV_MMA_TIMEOUT);
    }
    if (warp == 0) tc::tmem_alloc(tmem_slot, S::TMEM_COLS);
    tc::fence_proxy_async();
    // launched as a programmatic dependent of the previous kernel in the
    // stream: everything above (constant operators and tables) overlapped
    // its last CTAs; the state, residual and data it wrote are read only
    // after this wait; the next launch may then start its own set-up
    grid_dep_wait();
    grid_dep_launch();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
  }
  const uint32_t tmem = *tmem_slot;
  const uint32_t tmem_diff = tmem;
  const uint32_t tmem_lift = tmem + S::LIFT_COL;
  const int64_t Knp = a.K * NP;
  const bool stage_res = S::RES && a.mode != 0;
  const int64_t nb_cta = a.nbatch > (int64_t)blockIdx.x
                             ? (a.nbatch - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  // bounded wait by lane 0, result shared with (and ordered for) the warp
  auto warp_wait = [&](uint64_t* mb, uint32_t parity) -> bool {
    int ok = 0;
    if (lane == 0) ok = tc::mbar_wait(mb, parity, MBAR_MAX_NS);
    ok = __shfl_sync(FULL, ok, 0);
    __syncwarp();
    return ok != 0;
  };

  if (warp == NCW + 1) {
    // ================= MMA-issue warp =================
    constexpr uint32_t ID_DIFF = tc::idesc_16bit(128, S::ND, PT == PT_BF16);
    constexpr uint32_t ID_LIFT = tc::idesc_16bit(128, S::NL, PT == PT_BF16);
    (void)rbuf;
    int64_t diff_issued = -1, lift_issued = -1;
    for (int64_t i = 0; i < nb_cta; ++i) {
      const uint32_t par = (uint32_t)(i & 1);
      // diff MMAs once every consumer warp wrote its state-plane rows
      if (!warp_wait(&mbar[MB_AREADY], par)) break;
      if (lane == 0) {
        tc::fence_after_sync();
        const uint32_t aq_h = tc::smem_u32(Aqh), aq_l = tc::smem_u32(Aql);
        const uint32_t d_h = tc::smem_u32(smem + S::oDh), d_l = tc::smem_u32(smem + S::oDl);
#pragma unroll
        for (int kk = 0; kk < KD / 16; ++kk) {
          const uint32_t off = kk * 256;
          const uint64_t ah = tc::smem_desc(aq_h + off, 128, KD * 16);
          const uint64_t al = tc::smem_desc(aq_l + off, 128, KD * 16);
          const uint64_t bh = tc::smem_desc(d_h + off, 128, KD * 16);
          const uint64_t bl = tc::smem_desc(d_l + off, 128, KD * 16);
          tc::mma_bf16(tmem_diff, ah, bh, ID_DIFF, kk > 0 ? 1u : 0u);
          tc::mma_bf16(tmem_diff, ah, bl, ID_DIFF, 1u);
          tc::mma_bf16(tmem_diff, al, bh, ID_DIFF, 1u);
        }
        tc::mma_commit(&mbar[MB_DIFF]);
      }
      diff_issued = i;
      // lift MMAs once every consumer warp wrote its flux-plane entries
      if (!warp_wait(&mbar[MB_FREADY], par)) break;
      if (lane == 0) {
        tc::fence_after_sync();
        const uint32_t af_h = tc::smem_u32(Afh), af_l = tc::smem_u32(Afl);
        const uint32_t l_h = tc::smem_u32(smem + S::oLh), l_l = tc::smem_u32(smem + S::oLl);
#pragma unroll
        for (int kk = 0; kk < KL / 16; ++kk) {
          uint64_t ah, al;
          if constexpr (FSW) {
            // K step kk: 32 bytes further into the swizzle atom's rows
            ah = tc::smem_desc_sw128(af_h + kk * 32, 1024);
            al = tc::smem_desc_sw128(af_l + kk * 32, 1024);
          } else {
            ah = tc::smem_desc(af_h + kk * 256, 128, KL * 16);
            al = tc::smem_desc(af_l + kk * 256, 128, KL * 16);
          }
          const uint64_t bh = tc::smem_desc(l_h + kk * 256, 128, KL * 16);
          const uint64_t bl = tc::smem_desc(l_l + kk * 256, 128, KL * 16);
          tc::mma_bf16(tmem_lift, ah, bh, ID_LIFT, kk > 0 ? 1u : 0u);
          tc::mma_bf16(tmem_lift, ah, bl, ID_LIFT, 1u);
          tc::mma_bf16(tmem_lift, al, bh, ID_LIFT, 1u);
        }
        tc::mma_commit(&mbar[MB_LIFT]);
      }
      lift_issued = i;
    }
    if (lane == 0 && lift_issued + 1 < nb_cta) {
      // left early: let the MMAs already issued finish before TMEM is released
      atomicCAS(a.err, 0, DEV_MMA_TIMEOUT);
      if (diff_issued >= 0)
        tc::mbar_wait(&mbar[MB_DIFF], (uint32_t)(diff_issued & 1), MBAR_MAX_NS);
      if (lift_issued >= 0)
        tc::mbar_wait(&mbar[MB_LIFT], (uint32_t)(lift_issued & 1), MBAR_MAX_NS);
    }
    __syncwarp();
  } else if (warp == NCW) {
    // ====== I/O warp: stage buffers in (bulk copies), L2 prefetches ======
    auto batch_el0 = [&](int64_t i) { return batch_first(a, (int64_t)blockIdx.x + i * gridDim.x); };
    auto batch_ne = [&](int64_t i) { return batch_size(a, (int64_t)blockIdx.x + i * gridDim.x); };
    auto load_stage = [&](int64_t i) {
      const int b = NSTG == 2 ? (int)(i & 1) : 0;
      const int64_t el0 = batch_el0(i);
      const int ne = batch_ne(i);
      uint8_t* stg = smem + S::ostg + b * S::bStage;
      uint64_t* mb = &mbar[MB_FULL + b];
      if (lane == 0) {
        uint32_t want = 0;
        for (int f = 0; f < F; ++f) want += bulk_bytes(a.q_in + f * Knp + el0 * NP, ne * NP);
        want += bulk_bytes(a.geo32 + el0 * G, ne * G);
        want += bulk_bytes(a.conn + el0 * NF, ne * NF);
        if constexpr (C != 0) want += bulk_bytes(a.coeff + el0 * NP, ne * NP);
        if (want) mbar_expect_tx(mb, want);
      }
      __syncwarp();
      ST* st = reinterpret_cast<ST*>(stg);
      for (int f = 0; f < F; ++f)
        stage_in(st + f * FNP, a.q_in + f * Knp + el0 * NP, ne * NP, lane, mb);
      stage_in(reinterpret_cast<float*>(stg + S::sGeo), a.geo32 + el0 * G, ne * G, lane, mb);
      stage_in(reinterpret_cast<int2*>(stg + S::sConn), a.conn + el0 * NF, ne * NF, lane, mb);
      if constexpr (C != 0)
        stage_in(reinterpret_cast<double*>(stg + S::sCoef), a.coeff + el0 * NP, ne * NP, lane, mb);
      cp_async_arrive(mb);
    };
    auto load_res = [&](int64_t i) {
      const int64_t el0 = batch_el0(i);
      const int ne = batch_ne(i);
      uint64_t* mb = &mbar[MB_RES_FULL];
      if (lane == 0) {
        uint32_t want = 0;
        for (int f = 0; f < F; ++f) want += bulk_bytes(a.res + f * Knp + el0 * NP, ne * NP);
        if (want) mbar_expect_tx(mb, want);
      }
      __syncwarp();
      for (int f = 0; f < F; ++f)
        stage_in(rbuf + f * FNP, a.res + f * Knp + el0 * NP, ne * NP, lane, mb);
      cp_async_arrive(mb);
    };
    // pull batch j's state (and residual) into L2 ahead of their reads
    auto prefetch = [&](int64_t j, bool state, bool res) {
      if (lane != 0 || j >= nb_cta) return;
      const int64_t e0 = batch_el0(j);
      const uint32_t bytes = (uint32_t)batch_ne(j) * NP * (uint32_t)sizeof(ST);
      for (int f = 0; f < F; ++f) {
        const ST* q = a.q_in + f * Knp + e0 * NP;
        if (state && aligned16(q, bytes)) prefetch_l2(q, bytes);
        const ST* r = a.res + f * Knp + e0 * NP;
        if (res && a.mode != 0 && aligned16(r, bytes)) prefetch_l2(r, bytes);
      }
    };
    bool ok = true;
    if (nb_cta > 0) {
      load_stage(0);
      if (NSTG == 2 && nb_cta > 1) load_stage(1);
      if (stage_res) load_res(0);
      else prefetch(0, false, true);
      prefetch(NSTG, true, false);
    }
    for (int64_t i = 0; i < nb_cta; ++i) {
      const int b = NSTG == 2 ? (int)(i & 1) : 0;
      // the state loaded once this batch is done, and the next batch's
      // residual (read by the consumers' coalesced update)
      prefetch(i + NSTG + 1, true, false);
      prefetch(i + 1, false, true);
      if (!warp_wait(&mbar[MB_DONE + b], (uint32_t)((i / NSTG) & 1))) {
        ok = false;
        break;
      }
      // the consumers are done with this stage buffer (and the residual
      // buffer): refill them
      if (i + NSTG < nb_cta) load_stage(i + NSTG);
      if (stage_res && i + 1 < nb_cta) load_res(i + 1);
    }
    if (lane == 0 && !ok) atomicCAS(a.err, 0, DEV_MMA_TIMEOUT);
    cp_async_drain();
    __syncwarp();
  } else {
    // ================= consumer warps =================
    // TMEM lane of this thread (epilogue) = state-plane row (split pass)
    const int quad = warp & 3, part = warp >> 2;
    const int lf = lane / F;                 // element within the quadrant
    const int fown = lane - lf * F;          // own field
    const bool lane_used = lf < EPW;
    const int e_lane = quad * EPW + lf;
    const uint32_t lane_addr = (uint32_t)(quad * 32) << 16;
    const int row = quad * 32 + lane;
    auto warp_arrive = [&](uint64_t* mb) {
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(mb);
    };
    // A warp whose bounded wait gave up sets `bad` and does no more work, but
    // still takes every barrier of the batch; at the next batch's consumer
    // barrier every warp learns of it and all leave together, so no warp is
    // left waiting at a barrier.
    int bad = 0;
    // Phase A of the batch with local index `its`: wait for its stage buffer,
    // split its state into the planes, signal the MMA warp.  Returns true
    // when the consumers must leave (a warp's bounded wait gave up).
    auto split = [&](uint32_t its, float (&lin_out)[DIM]) -> bool {
      const int b = NSTG == 2 ? (int)(its & 1u) : 0;
      const uint32_t par = its & 1u;
      const int64_t el0 = batch_first(a, (int64_t)blockIdx.x + (int64_t)its * gridDim.x);
      const int ne = batch_size(a, (int64_t)blockIdx.x + (int64_t)its * gridDim.x);
      ST* st = reinterpret_cast<ST*>(smem + S::ostg + b * S::bStage);
      const bool valid = lane_used && e_lane < ne;
      const int e_own = valid ? e_lane : 0;
      uint32_t* rmx = rsq + par * 128;
      if (!bad && !warp_wait(&mbar[MB_FULL + b], (its / NSTG) & 1u)) {
        if (lane == 0) atomicCAS(a.err, 0, DEV_MMA_TIMEOUT);
        bad = 1;
      }
        // ---- A: remainders after the element's FP64 linear interpolant, split
        // into the state planes (one row per lane, 8 columns per item) ----
        {
          ST v0 = 0, dv[DIM];
#pragma unroll
          for (int d = 0; d < DIM; ++d) dv[d] = 0.0;
          if (valid && !bad) {
            const ST* q = st + fown * FNP + e_own * NP;
            v0 = q[0];
#pragma unroll
            for (int d = 0; d < DIM; ++d) dv[d] = q[svert[d]] - v0;
          }
#pragma unroll
          for (int d = 0; d < DIM; ++d) lin_out[d] = (float)(ST(0.5) * dv[d]);
          // chunks wholly in the K padding stay zero from the set-up unless the
          // rhs rows alias the planes
          constexpr int NCHUNK = S::RHS_OWN ? (NP + 7) / 8 : KD / 8;
          constexpr int NITEM = 4 * NCHUNK;
          constexpr int IPW = (NITEM + NCW - 1) / NCW;
          float rem[IPW][8];
          uint32_t rmax = 0u;
#pragma unroll
          for (int k = 0; k < IPW; ++k) {
            const int item = warp + k * NCW;
            const int chunk = item >> 2;
#pragma unroll
            for (int c = 0; c < 8; ++c) {
              const int j = chunk * 8 + c;
              float v = 0.f;
              if (item < NITEM && valid && !bad && j < NP) {
                ST l = v0;
#pragma unroll
                for (int d = 0; d < DIM; ++d) l += lamc[j * DIM + d] * dv[d];
                v = (float)(st[fown * FNP + e_own * NP + j] - l);
              }
              rem[k][c] = v;
              rmax = max(rmax, __float_as_uint(fabsf(v)));
            }
          }
          float inv = 1.0f;
          if constexpr (PT == PT_FP16) atomicMax(&rmx[row], rmax);
          // every consumer is past the previous batch's epilogue (the rhs rows
          // may alias these planes); FP16: the row maxima are complete
          if (cbar_or(bad)) return true;
          if constexpr (PT == PT_FP16) {
            // clear the next batch's maxima
            if (tid < 128) rsq[(par ^ 1u) * 128 + tid] = 0u;
            inv = row_scale_inv(rmx[row]);
          }
#pragma unroll
          for (int k = 0; k < IPW; ++k) {
            const int item = warp + k * NCW;
            if (item < NITEM) {
              const int chunk = item >> 2;
              uint32_t hw[4], lw[4];
#pragma unroll
              for (int c = 0; c < 8; c += 2) {
                const float x0 = rem[k][c] * inv, x1 = rem[k][c + 1] * inv;
                if constexpr (PT == PT_BF16) {
                  const __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
                  const float2 hf = __bfloat1622float2(h);
                  const __nv_bfloat162 l = __floats2bfloat162_rn(x0 - hf.x, x1 - hf.y);
                  hw[c / 2] = *reinterpret_cast<const uint32_t*>(&h);
                  lw[c / 2] = *reinterpret_cast<const uint32_t*>(&l);
                } else {
                  const __half2 h = __floats2half2_rn(x0, x1);
                  const float2 hf = __half22float2(h);
                  const __half2 l = __floats2half2_rn(x0 - hf.x, x1 - hf.y);
                  hw[c / 2] = *reinterpret_cast<const uint32_t*>(&h);
                  lw[c / 2] = *reinterpret_cast<const uint32_t*>(&l);
                }
              }
              const uint32_t off = kmajor_off(row, chunk * 8, KD);
              *reinterpret_cast<uint4*>(Aqh + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
              *reinterpret_cast<uint4*>(Aql + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
            }
          }
        }
        // the diff MMA (issued by the MMA warp) reads the planes
        tc::fence_proxy_async();
        tc::fence_before_sync();
        warp_arrive(&mbar[MB_AREADY]);
      return false;
    };
    // Phase E2 of the batch with local index `its`, once the quadrant's rhs
    // rows are complete: the coalesced FP64 update, then the stage buffer
    // (and the residual buffer) go back to the I/O warp.
    auto update = [&](uint32_t its) {
      const int b = NSTG == 2 ? (int)(its & 1u) : 0;
      const int64_t el0 = batch_first(a, (int64_t)blockIdx.x + (int64_t)its * gridDim.x);
      const int ne = batch_size(a, (int64_t)blockIdx.x + (int64_t)its * gridDim.x);
      ST* st = reinterpret_cast<ST*>(smem + S::ostg + b * S::bStage);
      if (!bad && stage_res && !warp_wait(&mbar[MB_RES_FULL], its & 1u)) {
        if (lane == 0) atomicCAS(a.err, 0, DEV_MMA_TIMEOUT);
        bad = 1;
      }
        // ---- E2: FP64 stage update of the quadrant's elements, coalesced: a
        // field's values of consecutive elements are contiguous in the state
        // vectors (q_in from the stage buffer; res and q_out in global memory,
        // res in place).  Thread t takes positions x = t + QT k of every field,
        // so its index arithmetic is done once per batch ----
        if (!bad) {
          const int e_first = quad * EPW;
          const int nq = ne - e_first < EPW ? ne - e_first : EPW;
          if (nq > 0) {
            constexpr int QT = 32 * (NCW / 4);
            constexpr int KX = (EPW * NP + QT - 1) / QT;   // positions per thread
            const int cnt = nq * NP;                       // values per field
            const int t = part * 32 + lane;
            const ST* qs = st + e_first * NP;
            const float* rq = rhs_s + quad * 32 * NPR;
            const int64_t g0 = (el0 + e_first) * NP;
            // position k of this thread: x = t + QT k; rhs row (el, f) at node
            // x - el Np is at rhs offset x + el (F NPR - Np) + f NPR
            if (a.mode == 0) {
#pragma unroll
              for (int k = 0; k < KX; ++k) {
                const int x = t + QT * k;
                if (x < cnt) {
                  const int ro = x + (x / NP) * (F * NPR - NP);
#pragma unroll
                  for (int f = 0; f < F; ++f)
                    a.q_out[(int64_t)f * Knp + g0 + x] = (ST)rq[ro + f * NPR];
                }
              }
            } else {
              // the stage update in the state's precision (FP64 or FP32)
              const ST ra = (ST)a.ra, rb = (ST)a.rb, dtt = (ST)a.dt;
              ST* res0 = a.res + g0;
              ST* qo0 = a.q_out + g0;
              // 16-byte accesses where every field's vectors share the
              // alignment of position 0 (K Np a multiple of the vector
              // width) and the output vectors are 16-byte aligned
              constexpr int V = 16 / (int)sizeof(ST);
              // (the stage and residual buffers hold the batch from their
              // first byte: their alignment equals the global one only when
              // the batch's first value el0 Np is a multiple of V)
              const bool vec = HB_SPLIT_VUPD && S::RES && Knp % V == 0 &&
                               ((el0 * NP) & (V - 1)) == 0 &&
                               ((reinterpret_cast<uintptr_t>(a.res) |
                                 reinterpret_cast<uintptr_t>(a.q_out)) & 15u) == 0;
              if (vec) {
                // positions [0, h) and [h + V nv, cnt) one at a time, the
                // V-groups between as 16-byte loads and stores (the stage
                // and residual buffers share the global offsets' alignment:
                // their field strides and el0 Np are multiples of V)
                using VT = typename std::conditional<sizeof(ST) == 8, double2, float4>::type;
                const ST* rs = rbuf + e_first * NP;
                const int h = (int)((V - (g0 & (V - 1))) & (V - 1));
                const int nv = (cnt - h) / V;
                const int nsc = h + (cnt - h - nv * V);      // scalar positions
                auto one = [&](int x) {
                  const int ro = x + (x / NP) * (F * NPR - NP);
#pragma unroll
                  for (int f = 0; f < F; ++f) {
                    const ST nr = ra * rs[f * FNP + x] + dtt * (ST)rq[ro + f * NPR];
                    res0[(int64_t)f * Knp + x] = nr;
                    qo0[(int64_t)f * Knp + x] = qs[f * FNP + x] + rb * nr;
                  }
                };
#pragma unroll 1
                for (int m = t; m < nv; m += QT) {
                  const int x = h + m * V;
                  int ro[V];
#pragma unroll
                  for (int j = 0; j < V; ++j) ro[j] = x + j + ((x + j) / NP) * (F * NPR - NP);
#pragma unroll
                  for (int f = 0; f < F; ++f) {
                    const VT qv = *reinterpret_cast<const VT*>(qs + f * FNP + x);
                    const VT rv = *reinterpret_cast<const VT*>(rs + f * FNP + x);
                    const ST* qa = reinterpret_cast<const ST*>(&qv);
                    const ST* ra0 = reinterpret_cast<const ST*>(&rv);
                    VT nrv, qov;
                    ST* nr = reinterpret_cast<ST*>(&nrv);
                    ST* qo = reinterpret_cast<ST*>(&qov);
#pragma unroll
                    for (int j = 0; j < V; ++j) {
                      nr[j] = ra * ra0[j] + dtt * (ST)rq[ro[j] + f * NPR];
                      qo[j] = qa[j] + rb * nr[j];
                    }
                    *reinterpret_cast<VT*>(res0 + (int64_t)f * Knp + x) = nrv;
                    *reinterpret_cast<VT*>(qo0 + (int64_t)f * Knp + x) = qov;
                  }
                }
                if (t >= QT - nsc) {
                  const int j = t - (QT - nsc);
                  one(j < h ? j : h + nv * V + (j - h));
                }
              } else if constexpr (S::RES) {
                // residual from the residual buffer (short latency): one
                // value at a time, few registers live
                const ST* rs = rbuf + e_first * NP;
#pragma unroll 1
                for (int k = 0; k < KX; ++k) {
                  const int x = t + QT * k;
                  if (x < cnt) {
                    const int ro = x + (x / NP) * (F * NPR - NP);
#pragma unroll
                    for (int f = 0; f < F; ++f) {
                      const ST nr = ra * rs[f * FNP + x] + dtt * (ST)rq[ro + f * NPR];
                      res0[(int64_t)f * Knp + x] = nr;
                      qo0[(int64_t)f * Knp + x] = qs[f * FNP + x] + rb * nr;
                    }
                  }
                }
              } else {
                // residual from global memory: every load first (they are
                // independent of the stores)
                ST r0[KX][F];
#pragma unroll
                for (int k = 0; k < KX; ++k) {
                  const int x = t + QT * k;
#pragma unroll
                  for (int f = 0; f < F; ++f)
                    r0[k][f] = x < cnt ? res0[(int64_t)f * Knp + x] : ST(0);
                }
#pragma unroll
                for (int k = 0; k < KX; ++k) {
                  const int x = t + QT * k;
                  if (x < cnt) {
                    const int ro = x + (x / NP) * (F * NPR - NP);
#pragma unroll
                    for (int f = 0; f < F; ++f) {
                      const ST nr = ra * r0[k][f] + dtt * (ST)rq[ro + f * NPR];
                      res0[(int64_t)f * Knp + x] = nr;
                      qo0[(int64_t)f * Knp + x] = qs[f * FNP + x] + rb * nr;
                    }
                  }
                }
              }
            }
          }
        }
        // generic reads of the stage buffer before the I/O warp refills it
        tc::fence_proxy_async();
        warp_arrive(&mbar[MB_DONE + b]);
    };
    // Software pipeline (when two stage buffers, an rhs buffer of its own and
    // parked volume terms allow it): each warp splits batch i + 1 between
    // the volume terms and the lift epilogue of batch i, so the wait for
    // batch i's lift MMA overlaps that work.  Otherwise batch i's split
    // opens its own iteration.
    constexpr bool PIPE = S::PARK && NSTG == 2 && S::RHS_OWN;
    float lin[DIM], lin_next[DIM];   // reference derivatives of the removed interpolants
    bool leave = false;
    if constexpr (PIPE) {
      if (nb_cta > 0) leave = split(0u, lin_next);
    }
    uint32_t it = 0;
    for (int64_t batch = blockIdx.x; !leave && batch < a.nbatch; batch += gridDim.x, ++it) {
      const int b = NSTG == 2 ? (int)(it & 1u) : 0;
      const uint32_t par = it & 1u;
      const int64_t el0 = batch_first(a, batch);
      const int ne = batch_size(a, batch);
      ST* st = reinterpret_cast<ST*>(smem + S::ostg + b * S::bStage);  // [F][EB][NP]
      const uint8_t* stg = smem + S::ostg + b * S::bStage;
      const float* sgeo = reinterpret_cast<const float*>(stg + S::sGeo);
      const int2* sconn = reinterpret_cast<const int2*>(stg + S::sConn);
      const double* scoef = reinterpret_cast<const double*>(stg + S::sCoef);
      const bool valid = lane_used && e_lane < ne;
      const int e_own = valid ? e_lane : 0;
      uint32_t* rmx = rsq + par * 128;     // this batch's state row maxima
      uint32_t* fmx = rsf + par * 128;     // this batch's flux row maxima

      if constexpr (!PIPE) {
        if (split(it, lin_next)) { leave = true; break; }
      }
#pragma unroll
      for (int d = 0; d < DIM; ++d) lin[d] = lin_next[d];
      // ---- C: face fluxes (FP32 on jumps formed in FP64) -> lift planes.
      // Warp w takes the elements w, w + NCW, ... of the batch and lane l
      // their face points l, l + 32, ..., so each flux row (e, f) lies in one
      // warp (its FP16 scale is a warp reduction) ----
      constexpr int SPE = (NFPT + 31) / 32;                  // point slots per element
      constexpr int NEPW = (EB + NCW - 1) / NCW;             // elements per warp
      static_assert(SPE * NA <= 32, "face points in flight exceed the register budget");
      constexpr int ER0 = 32 / (SPE * NA);
      // 3D: one element per round -- the smaller unrolled body of the
      // three passes runs 3-6 % faster than two elements' worth of points
      // in flight; 2D: as many as the point registers allow (5 % faster)
      constexpr int ERX = HB_SPLIT_ER > 0 ? HB_SPLIT_ER : (DIM == 3 ? 1 : ER0);
      constexpr int ER = ERX < NEPW ? ERX : NEPW;            // elements per round
      constexpr int FR = ER * SPE;
#pragma unroll 1
      for (int j0 = 0; j0 < NEPW; j0 += ER) {
        float uPs[FR][NA];
        bool okp[FR];
        // pass 1: ext-side values (global gathers for neighbours outside the batch)
#pragma unroll
        for (int u = 0; u < FR; ++u) {
          const int j = j0 + u / SPE;
          const int e = warp + j * NCW, p = lane + (u % SPE) * 32;
          const int face = p / NFP, k = p % NFP;
          okp[u] = false;
          if (j < NEPW && e < ne && p < NFPT) {
            const int2 cn = sconn[e * NF + face];
            const int nb = cn.x;
            if (nb >= a.K) {
              // neighbour on another partition: ext values from the halo buffer
              const int64_t hk = ((int64_t)nb - a.K) * NFP + k;
              if (nb - a.K < a.n_halo && a.halo != nullptr) {
                const int lnode = sfm[p];
                if constexpr (JumpLinear<MODEL>::value) {
#pragma unroll
                  for (int f = 0; f < F; ++f)
                    uPs[u][f] = (float)(st[f * FNP + e * NP + lnode] - a.halo[hk * F + f]);
                } else {
                  if constexpr (C != 0) uPs[u][0] = (float)a.halo_c[hk];
#pragma unroll
                  for (int f = 0; f < F; ++f) uPs[u][C + f] = (float)a.halo[hk * F + f];
                }
                okp[u] = true;
              } else {
                atomicCAS(a.err, 0, DEV_BAD_NEIGHBOUR);
              }
            } else if (nb >= 0) {
              const int code = cn.y;
              const int nface = code & 3, perm = code >> 2;
              if (nface < NF && perm < a.nperm && nb < a.K) {
                const int nn = ssh[(perm * NF + nface) * NFP + k];
                const int64_t gi = (int64_t)nb * NP + nn;
                const int lnode = sfm[p];
                const int lb = (int)(nb - el0);   // neighbour inside this batch?
                const bool inb = lb >= 0 && lb < ne;
                if constexpr (JumpLinear<MODEL>::value) {
#pragma unroll
                  for (int f = 0; f < F; ++f) {
                    const ST qm = st[f * FNP + e * NP + lnode];
                    const ST qp = inb ? st[f * FNP + lb * NP + nn]
                                      : __ldg(a.q_in + f * Knp + gi);
                    uPs[u][f] = (float)(qm - qp);
                  }
                } else {
                  if constexpr (C != 0)
                    uPs[u][0] = inb ? (float)scoef[lb * NP + nn] : (float)__ldg(a.coeff + gi);
#pragma unroll
                  for (int f = 0; f < F; ++f)
                    uPs[u][C + f] = inb ? (float)st[f * FNP + lb * NP + nn]
                                        : (float)__ldg(a.q_in + f * Knp + gi);
                }
                okp[u] = true;
              } else {
                atomicCAS(a.err, 0, DEV_BAD_CODE);
              }
            }
          }
        }
        // pass 2: fluxes times Fscale -> uPs[u][0..F)
#pragma unroll
        for (int u = 0; u < FR; ++u) {
          const int j = j0 + u / SPE;
          const int e = warp + j * NCW, p = lane + (u % SPE) * 32;
          const int face = p / NFP, k = p % NFP;
          float fl[F];
#pragma unroll
          for (int f = 0; f < F; ++f) fl[f] = 0.f;
          if (j < NEPW && e < ne && p < NFPT) {
            const int lnode = sfm[p];
            float uM[NA], uP[NA], n[DIM];
            const float* gf = sgeo + e * G + DIM * DIM + face * (DIM + 1);
#pragma unroll
            for (int d = 0; d < DIM; ++d) n[d] = gf[d];
            const float fscale = gf[DIM];
            const int2 cn = sconn[e * NF + face];
            const int nb = cn.x;
            bool have = true, bdry = false;
            if (nb >= 0 && JumpLinear<MODEL>::value) {
              have = okp[u];
#pragma unroll
              for (int q = 0; q < NA; ++q) { uM[q] = uPs[u][q]; uP[q] = 0.f; }
            } else {
              if constexpr (C != 0) uM[0] = (float)scoef[e * NP + lnode];
#pragma unroll
              for (int f = 0; f < F; ++f) uM[C + f] = (float)st[f * FNP + e * NP + lnode];
              if (nb >= 0) {
                have = okp[u];
#pragma unroll
                for (int q = 0; q < NA; ++q) uP[q] = uPs[u][q];
              } else {
                bdry = true;
                const int kind = cn.y;
                float given = 0.f;
                if (kind == HB_BC_GIVEN) {
                  const int64_t bi = (int64_t)(-1 - nb) * NFP + k;
                  if (a.bdry == nullptr || bi >= a.n_given) {
                    atomicCAS(a.err, 0, a.bdry == nullptr ? DEV_MISSING_INPUT : DEV_BAD_BDRY_INDEX);
                    have = false;
                  } else {
                    given = (float)__ldg(a.bdry + bi);
                  }
                }
                if (have) have = model_bc<MODEL, DIM, float>(a.mp, kind, uM, n, given, uP);
              }
            }
            if (have) {
              model_flux<MODEL, DIM, float>(a.mp, bdry, uM, uP, n, fl);
#pragma unroll
              for (int f = 0; f < F; ++f) fl[f] *= fscale;
            }
          }
#pragma unroll
          for (int f = 0; f < F; ++f) uPs[u][f] = fl[f];
        }
        // pass 3: split into the lift planes; FP16 rows are scaled by a power
        // of two from the row's largest |flux| (a warp reduction), which the
        // epilogue undoes
#pragma unroll
        for (int jj = 0; jj < ER; ++jj) {
          const int j = j0 + jj;
          const int e = warp + j * NCW;
          if (j < NEPW && e < ne) {      // warp-uniform
            const int rowb = (e / EPW) * 32 + (e % EPW) * F;
#pragma unroll
            for (int f = 0; f < F; ++f) {
              float inv = 1.0f;
              if constexpr (PT == PT_FP16) {
                uint32_t m = 0u;
#pragma unroll
                for (int sl = 0; sl < SPE; ++sl)
                  m = max(m, __float_as_uint(fabsf(uPs[jj * SPE + sl][f])));
                m = __reduce_max_sync(FULL, m);
                if (lane == 0) fmx[rowb + f] = m;
                inv = row_scale_inv(m);
              }
              const int frow = rowb + f;
              // slots in pairs: one packed conversion splits both values
#pragma unroll
              for (int sl = 0; sl + 1 < SPE; sl += 2) {
                const int p0 = lane + sl * 32, p1 = p0 + 32;
                const float x0 = uPs[jj * SPE + sl][f] * inv, x1 = uPs[jj * SPE + sl + 1][f] * inv;
                uint32_t hh, ll;
                if constexpr (PT == PT_BF16) {
                  const __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
                  const float2 hf = __bfloat1622float2(h);
                  const __nv_bfloat162 l = __floats2bfloat162_rn(x0 - hf.x, x1 - hf.y);
                  hh = *reinterpret_cast<const uint32_t*>(&h);
                  ll = *reinterpret_cast<const uint32_t*>(&l);
                } else {
                  const __half2 h = __floats2half2_rn(x0, x1);
                  const float2 hf = __half22float2(h);
                  const __half2 l = __floats2half2_rn(x0 - hf.x, x1 - hf.y);
                  hh = *reinterpret_cast<const uint32_t*>(&h);
                  ll = *reinterpret_cast<const uint32_t*>(&l);
                }
                if (p0 < NFPT) {
                  const uint32_t o0 = fplane_off<FSW>(frow, p0, KL);
                  *reinterpret_cast<uint16_t*>(Afh + o0) = (uint16_t)hh;
                  *reinterpret_cast<uint16_t*>(Afl + o0) = (uint16_t)ll;
                }
                if (p1 < NFPT) {
                  const uint32_t o1 = fplane_off<FSW>(frow, p1, KL);
                  *reinterpret_cast<uint16_t*>(Afh + o1) = (uint16_t)(hh >> 16);
                  *reinterpret_cast<uint16_t*>(Afl + o1) = (uint16_t)(ll >> 16);
                }
              }
              if constexpr (SPE % 2 == 1) {
                const int p = lane + (SPE - 1) * 32;
                if (p < NFPT)
                  store_split<PT>(Afh, Afl, fplane_off<FSW>(frow, p, KL),
                                  uPs[jj * SPE + SPE - 1][f] * inv);
              }
            }
          }
        }
      }
      tc::fence_proxy_async();
      warp_arrive(&mbar[MB_FREADY]);

      // ---- E1: TMEM -> chain rule, volume terms, + lift -> FP32 rhs rows in
      // shared memory, 4 nodes per pass.  With few nodes per warp (S::PARK)
      // the volume terms (diff accumulators only) are formed first and parked
      // in this warp's own TMEM columns, so the wait for the lift MMA
      // overlaps them and both loops stay rolled up (a small instruction
      // footprint) ----
      constexpr int CHK = S::NPQ < 8 ? S::NPQ : 8;   // TMEM columns per wait
      constexpr int NCH = (S::NPQ + CHK - 1) / CHK;
      constexpr bool VOL_FIRST = S::PARK;
      const int i_lo = part * S::NPQ;
      const int i_hi = (part + 1) * S::NPQ < NP ? (part + 1) * S::NPQ : NP;
      const int base = lf * F;
      // parked volume terms: columns [VCOL + i_lo, VCOL + i_lo + NPQ), this
      // warp's lanes only
      const uint32_t tmem_vol = tmem + S::VCOL + lane_addr;
      float* rrow = rhs_s + row * NPR;
      float gm[DIM][DIM];
      float sdiff = a.op_scale_d;
      // Maxwell divides by eps (E) or mu (H): one reciprocal per lane
      const float inv_m = MODEL == HB_MODEL_MAXWELL
                              ? 1.0f / (float)(fown < 3 ? a.mp.eps : a.mp.mu) : 1.0f;
      auto rhs_of = [&](int i, float vol, float lift) -> float {
        const int64_t si = model_src_index<MODEL>(fown, (el0 + e_own) * NP + i, Knp);
        const float src = (a.source && si >= 0) ? (float)a.source[si] : 0.f;
        if constexpr (MODEL == HB_MODEL_MAXWELL) {
          return (vol + lift) * inv_m + src;
        } else {
          return model_finish<MODEL, DIM, float>(a.mp, fown, vol, lift, src);
        }
      };
      if constexpr (VOL_FIRST) {
        if (!bad && !warp_wait(&mbar[MB_DIFF], par)) {
          if (lane == 0) atomicCAS(a.err, 0, DEV_MMA_TIMEOUT);
          bad = 1;
        }
        if (!bad) {
          tc::fence_after_sync();
          const float* ge = sgeo + e_own * G;
          if constexpr (PT == PT_FP16) sdiff *= row_scale(rmx[row]);
          // gradient component x of the lane's field at a node:
          //   g_x = off_x + sum_r gs[r][x] acc_r, with gs = (dr/dx) * scale
          //   and off_x = sum_r (dr/dx) lin_r (the removed interpolant)
          float gs[DIM][DIM], off[DIM];
#pragma unroll
          for (int x = 0; x < DIM; ++x) {
            off[x] = 0.f;
#pragma unroll
            for (int r = 0; r < DIM; ++r) {
              const float gmv = ge[r * DIM + x];
              gs[r][x] = gmv * sdiff;
              off[x] += gmv * lin[r];
            }
          }
          if constexpr (MODEL == HB_MODEL_MAXWELL) {
            // The curls read of each field's gradient only two components,
            // on other lanes: the lane of field j (E_j or H_j) offers
            // oA = d/dx_(j+1) and oB = d/dx_(j+2) (indices mod 3), and
            //   (curl H)_c = oB(H_(c+2)) - oA(H_(c+1)),
            //   (curl E)_c = oB(E_(c+2)) - oA(E_(c+1));
            // E_c takes +curl H, H_c takes -curl E.
            const int cc = fown % 3;
            const int xa = cc == 2 ? 0 : cc + 1, xb = cc == 0 ? 2 : cc - 1;
            float cA[3], cB[3];
#pragma unroll
            for (int r = 0; r < 3; ++r) {
              cA[r] = xa == 0 ? gs[r][0] : (xa == 1 ? gs[r][1] : gs[r][2]);
              cB[r] = xb == 0 ? gs[r][0] : (xb == 1 ? gs[r][1] : gs[r][2]);
            }
            const float offA = xa == 0 ? off[0] : (xa == 1 ? off[1] : off[2]);
            const float offB = xb == 0 ? off[0] : (xb == 1 ? off[1] : off[2]);
            const int other = fown < 3 ? 3 : 0;
            const int srcB = base + other + (cc == 0 ? 2 : cc - 1);   // field (c + 2) mod 3
            const int srcA = base + other + (cc == 2 ? 0 : cc + 1);   // field (c + 1) mod 3
            const float sgn = fown < 3 ? 1.f : -1.f;
#pragma unroll 1
            for (int c0 = i_lo; c0 < i_hi; c0 += 4) {
              float dv[DIM][4], v4[4];
#pragma unroll
              for (int r = 0; r < DIM; ++r) tc::tmem_ld4(tmem_diff + lane_addr + r * NP + c0, dv[r]);
              tc::tmem_wait_ld();
#pragma unroll
              for (int c = 0; c < 4; ++c) {
                float oA = offA, oB = offB;
#pragma unroll
                for (int r = 0; r < 3; ++r) {
                  oA += cA[r] * dv[r][c];
                  oB += cB[r] * dv[r][c];
                }
                const float t0 = __shfl_sync(FULL, oB, srcB);
                const float t1 = __shfl_sync(FULL, oA, srcA);
                v4[c] = sgn * (t0 - t1);
              }
              tc::tmem_st4(tmem_vol + c0, v4);
            }
          } else {
#pragma unroll 1
            for (int c0 = i_lo; c0 < i_hi; c0 += 4) {
              float dv[DIM][4], v4[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
              for (int r = 0; r < DIM; ++r) tc::tmem_ld4(tmem_diff + lane_addr + r * NP + c0, dv[r]);
              tc::tmem_wait_ld();
#pragma unroll
              for (int c = 0; c < 4; ++c) {
                const int i = c0 + c;
                if (i >= i_hi) break;        // warp-uniform
                float g[DIM];
#pragma unroll
                for (int x = 0; x < DIM; ++x) {
                  float t = off[x];
#pragma unroll
                  for (int r = 0; r < DIM; ++r) t += gs[r][x] * dv[r][c];
                  g[x] = t;
                }
                const float cnode = C ? (float)scoef[e_own * NP + i] : 0.f;
                v4[c] = volume_own<MODEL, DIM>(a.mp, g, base, fown, cnode);
              }
              tc::tmem_st4(tmem_vol + c0, v4);
            }
          }
          tc::tmem_wait_st();
        }
      }
      if constexpr (PIPE) {
        // the next batch's split, while this batch's lift MMA runs
        if ((int64_t)it + 1 < nb_cta && split(it + 1u, lin_next)) { leave = true; break; }
      }
      // (FREADY also orders the flux row maxima the other warps wrote)
      {
        bool ok = !bad;
        if (ok && PT == PT_FP16) ok = warp_wait(&mbar[MB_FREADY], par);
        if (ok && !VOL_FIRST) ok = warp_wait(&mbar[MB_DIFF], par);
        if (ok) ok = warp_wait(&mbar[MB_LIFT], par);
        if (!bad && !ok) {
          if (lane == 0) atomicCAS(a.err, 0, DEV_MMA_TIMEOUT);
          bad = 1;
        }
      }
      if (!bad) {
        tc::fence_after_sync();
        if constexpr (!VOL_FIRST) {
          const float* ge = sgeo + e_own * G;
#pragma unroll
          for (int r = 0; r < DIM; ++r)
#pragma unroll
            for (int x = 0; x < DIM; ++x) gm[r][x] = ge[r * DIM + x];
          if constexpr (PT == PT_FP16) sdiff *= row_scale(rmx[row]);
        }
        float slift = a.op_scale_l;
        if constexpr (PT == PT_FP16)
          slift *= row_scale(fmx[row]);   // written in C by the row's owner warp
        if constexpr (VOL_FIRST) {
#pragma unroll 1
          for (int c0 = i_lo; c0 < i_hi; c0 += 4) {
            float lv[4], v4[4], o[4];
            tc::tmem_ld4(tmem_lift + lane_addr + c0, lv);
            tc::tmem_ld4(tmem_vol + c0, v4);
            tc::tmem_wait_ld();
#pragma unroll
            for (int c = 0; c < 4; ++c) o[c] = rhs_of(c0 + c, v4[c], lv[c] * slift);
            // parts own 4-aligned node ranges; the last part's nodes past
            // Np land in the row's padding (NPR)
            if (valid) *reinterpret_cast<float4*>(rrow + c0) = make_float4(o[0], o[1], o[2], o[3]);
          }
        } else {
#pragma unroll
          for (int kc = 0; kc < NCH; ++kc) {
            const int c0 = i_lo + kc * CHK;
            if (c0 >= i_hi) break;         // warp-uniform
            float dv[DIM][CHK], lv[CHK], o[CHK];
#pragma unroll
            for (int g = 0; g < CHK / 4; ++g) {
              if (c0 + 4 * g < i_hi) {     // warp-uniform
#pragma unroll
                for (int r = 0; r < DIM; ++r)
                  tc::tmem_ld4(tmem_diff + lane_addr + r * NP + c0 + 4 * g,
                               *reinterpret_cast<float(*)[4]>(&dv[r][4 * g]));
                tc::tmem_ld4(tmem_lift + lane_addr + c0 + 4 * g,
                             *reinterpret_cast<float(*)[4]>(&lv[4 * g]));
              }
            }
            tc::tmem_wait_ld();
#pragma unroll
            for (int c = 0; c < CHK; ++c) {
              const int i = c0 + c;
              o[c] = 0.f;
              if (i >= i_hi) continue;     // warp-uniform
              float g[DIM];
#pragma unroll
              for (int x = 0; x < DIM; ++x) {
                float t = 0.f;
#pragma unroll
                for (int r = 0; r < DIM; ++r) t += gm[r][x] * (dv[r][c] * sdiff + lin[r]);
                g[x] = t;
              }
              const float cnode = C ? (float)scoef[e_own * NP + i] : 0.f;
              o[c] = rhs_of(i, volume_own<MODEL, DIM>(a.mp, g, base, fown, cnode),
                            lv[c] * slift);
            }
#pragma unroll
            for (int g = 0; g < CHK / 4; ++g)
              if (valid && c0 + 4 * g < i_hi)
                *reinterpret_cast<float4*>(rrow + c0 + 4 * g) =
                    make_float4(o[4 * g], o[4 * g + 1], o[4 * g + 2], o[4 * g + 3]);
          }
        }
      }
      // this warp's TMEM reads are done before the next MMAs may be issued
      tc::fence_before_sync();
      // the quadrant's rhs rows are complete
      qbar(quad);

      update(it);
    }
  }

  // ---- tear-down ----
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, S::TMEM_COLS);
}

// ---------------------------------------------------------------------------
// Streamed-operator variant for high orders, whose operator planes do not fit
// in shared memory next to the data planes (3D, N >= 6), or leave room for a
// single state stage only (3D, N = 5, operators without halo faces).  Same contraction
// layout, split, epilogue and stage update as rhs_split_kernel; differences:
//   * the operator planes stream from global memory (L2-resident) through a
//     two-buffer ring, one 16-column K chunk at a time; each chunk's MMAs are
//     committed to that buffer's mbarrier, which is waited on before the
//     buffer is refilled;
//   * d*Np may exceed one MMA's N (256): the diff accumulator is then filled
//     by two MMAs per product (N = ND1 + ND2 columns);
//   * the state is read from global memory (FP64) in the split and face
//     phases, the rhs is staged (FP32) in the state-plane area after the diff
//     MMAs completed, and the FP64 stage update is a coalesced pass;
//   * all 8 warps run every phase; thread 0 issues the MMAs.
template <int MODEL, int DIM, int ORDER>
struct ShapeS {
  static constexpr int F = Traits<MODEL, DIM>::F;
  static constexpr int C = Traits<MODEL, DIM>::COEFF;
  static constexpr int NA = F + C;
  static constexpr int NP = DIM == 2 ? (ORDER + 1) * (ORDER + 2) / 2
                                     : (ORDER + 1) * (ORDER + 2) * (ORDER + 3) / 6;
  static constexpr int NFP = DIM == 2 ? ORDER + 1 : (ORDER + 1) * (ORDER + 2) / 2;
  static constexpr int NF = DIM + 1;
  static constexpr int NFPT = NF * NFP;
  static constexpr int G = DIM * DIM + NF * (DIM + 1);
  static constexpr int EPW = 32 / F;
  static constexpr int EB = 4 * EPW;
  static constexpr int FNP = EB * NP;
  static constexpr int NVAL = F * FNP;
  static constexpr int KD = ru16(NP), KL = ru16(NFPT);
  static constexpr int ND = ru16(DIM * NP), NL = ru16(NP);
  static constexpr int ND1 = ND <= 256 ? ND : ru16(ND / 2);
  static constexpr int ND2 = ND - ND1;
  static constexpr int LIFT_COL = ru32(ND);
  static constexpr int NKD = KD / 16, NKL = KL / 16;
  static constexpr int THREADS = 256;
  static constexpr int NW = THREADS / 32;
  static constexpr int NPQ = (((NP + 1) / 2) + 3) & ~3;       // nodes per epilogue warp
  static constexpr int NFACE = EB * NFPT;
  static constexpr int NFV = (NFACE + THREADS - 1) / THREADS;
  static constexpr int NITEM = 4 * (KD / 8);
  static constexpr uint32_t bDc = ND * 16 * 2, bLc = NL * 16 * 2;   // one plane, one chunk
  static constexpr uint32_t RING = al128(2 * (bDc > bLc ? bDc : bLc));
  static constexpr uint32_t bAq = 128 * KD * 2, bAf = 128 * KL * 2;
  static constexpr uint32_t oAqh = 0;
  static constexpr uint32_t oAql = al128(oAqh + bAq);
  static constexpr uint32_t oAfh = al128(oAql + bAq);
  static constexpr uint32_t oAfl = al128(oAfh + bAf);
  static constexpr uint32_t oR0 = al128(oAfl + bAf);
  static constexpr uint32_t oR1 = al128(oR0 + RING);
  static constexpr uint32_t osv = al128(oR1 + RING);                 // FP64 [F][EB][DIM+1]
  static constexpr uint32_t olam = al16(osv + F * EB * (DIM + 1) * 8);
  static constexpr uint32_t ogeo = al16(olam + NP * DIM * 8);
  static constexpr uint32_t oconn = al16(ogeo + EB * G * 4);
  static constexpr uint32_t ocoef = al16(oconn + EB * NF * 8);       // FP32 c [EB][NP]
  static constexpr uint32_t ofm = al16(ocoef + (C ? EB * NP * 4 : 0));
  static constexpr uint32_t osh = al16(ofm + NFPT);
  static constexpr uint32_t overt = al16(osh + 6 * NFP);
  static constexpr uint32_t ors = al16(overt + 4);                   // [2][128] row maxima
  // mbarriers: [0..1] ring MMAs done, [2] batch MMAs done, [5..6] ring copy
  // landed; the TMEM address word sits at byte 32
  static constexpr uint32_t obar = al16(ors + 256 * 4);
  static constexpr uint32_t total = al16(obar + 64);
  static constexpr uint32_t LIN_BYTES = 8 + NP * DIM * 8;
  static constexpr int TMEM_NEED = LIFT_COL + NL;
  static constexpr uint32_t TMEM_COLS = TMEM_NEED <= 128 ? 128 : TMEM_NEED <= 256 ? 256 : 512;
  static constexpr bool FITS = ND1 <= 256 && ND2 <= 256 && NL <= 256 && TMEM_NEED <= 512 &&
                               LIFT_COL + NP + 3 < 512 && total <= SMEM_LIMIT &&
                               F * FNP * 4 <= (int)(2 * bAq);
};

template <int MODEL, int DIM, int ORDER, int PT>
__global__ void __launch_bounds__(256, 1) rhs_split_stream_kernel(SplitArgs a) {
  using S = ShapeS<MODEL, DIM, ORDER>;
  constexpr int F = S::F, C = S::C, NA = S::NA, NP = S::NP, NFP = S::NFP, NF = S::NF;
  constexpr int NFPT = S::NFPT, G = S::G, EPW = S::EPW, EB = S::EB, FNP = S::FNP;
  constexpr int KD = S::KD, KL = S::KL, NV1 = DIM + 1;
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* Aqh = smem + S::oAqh;
  uint8_t* Aql = smem + S::oAql;
  uint8_t* Afh = smem + S::oAfh;
  uint8_t* Afl = smem + S::oAfl;
  float* sq = reinterpret_cast<float*>(smem + S::oAqh);            // staged rhs (after diff)
  double* sv = reinterpret_cast<double*>(smem + S::osv);
  const double* slam = reinterpret_cast<const double*>(smem + S::olam);
  float* sgeo = reinterpret_cast<float*>(smem + S::ogeo);
  int2* sconn = reinterpret_cast<int2*>(smem + S::oconn);
  float* scoef = reinterpret_cast<float*>(smem + S::ocoef);
  uint8_t* sfm = smem + S::ofm;
  uint8_t* ssh = smem + S::osh;
  const uint8_t* svert = smem + S::overt;
  uint32_t* rsq = reinterpret_cast<uint32_t*>(smem + S::ors);        // state rows
  uint32_t* rsf = rsq + 128;                                         // flux rows
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + S::obar);      // see ShapeS::obar
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + S::obar + 32);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint8_t* dimg = a.ops;                                       // D chunks
  const uint8_t* limg = a.ops + (size_t)S::NKD * 2 * S::bDc;          // L chunks
  const uint8_t* tail = limg + (size_t)S::NKL * 2 * S::bLc;

  {
    if (tid < 4) smem[S::overt + tid] = tail[tid];
    double* lam = reinterpret_cast<double*>(smem + S::olam);
    const double* lsrcd = reinterpret_cast<const double*>(tail + 8);
    for (int x = tid; x < NP * DIM; x += S::THREADS) lam[x] = lsrcd[x];
    for (int x = tid; x < NFPT; x += S::THREADS) sfm[x] = (uint8_t)a.fmask[x];
    for (int x = tid; x < a.nperm * NFP; x += S::THREADS) ssh[x] = (uint8_t)a.shuffle[x];
    // the lift planes' K padding and unused rows are never written again
    const uint4 z = make_uint4(0, 0, 0, 0);
    for (uint32_t o = S::oAfh + tid * 16; o < S::oR0; o += S::THREADS * 16)
      *reinterpret_cast<uint4*>(smem + o) = z;
    if (tid == 0) {
      tc::mbar_init(&mbar[0], 1);
      tc::mbar_init(&mbar[1], 1);
      tc::mbar_init(&mbar[2], 1);
      tc::mbar_init(&mbar[5], 1);
      tc::mbar_init(&mbar[6], 1);
    }
    if (warp == 0) tc::tmem_alloc(tmem_slot, S::TMEM_COLS);
    tc::fence_proxy_async();
    // programmatic dependent launch, as in the resident kernel
    grid_dep_wait();
    grid_dep_launch();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
  }
  const uint32_t tmem = *tmem_slot;
  const uint32_t tmem_diff = tmem, tmem_lift = tmem + S::LIFT_COL;
  constexpr uint32_t ID_D1 = tc::idesc_16bit(128, S::ND1, PT == PT_BF16);
  constexpr uint32_t ID_D2 = tc::idesc_16bit(128, S::ND2 > 0 ? S::ND2 : 16, PT == PT_BF16);
  constexpr uint32_t ID_L = tc::idesc_16bit(128, S::NL, PT == PT_BF16);
  const int64_t Knp = a.K * NP;
  const int quad = warp & 3, part = warp >> 2;
  const int lf = lane / F, fown = lane - lf * F;
  const bool lane_used = lf < EPW;
  const int e_lane = quad * EPW + lf;
  const uint32_t lane_addr = (uint32_t)(quad * 32) << 16;
  const int row = quad * 32 + lane;
  uint32_t ring_uses[2] = {0u, 0u};   // MMA commits so far on each ring buffer
  uint32_t ring_fills[2] = {0u, 0u};  // bulk copies started into each ring buffer
  uint32_t ring_waits[2] = {0u, 0u};  // copies waited for on each ring buffer
  uint32_t chunk = 0;                 // running chunk counter (ring buffer = chunk & 1)
  int bad = 0;

  // Thread 0 only: streams n operator chunks of `bytes` (at src + k * bytes)
  // through the two ring buffers with bulk copies, the copy of chunk k + 1
  // in flight while chunk k's MMAs (issue(k, buffer)) run.  A buffer is
  // refilled once the MMAs that read it completed.  False on a timeout.
  auto stream_chunks = [&](const uint8_t* src, int n, uint32_t bytes, auto issue) -> bool {
    const uint32_t c0 = chunk;          // running number of this stream's chunk 0
    auto fill = [&](int k) -> bool {
      const int b = (int)((c0 + (uint32_t)k) & 1u);
      if (ring_uses[b] > 0 && !tc::mbar_wait(&mbar[b], (ring_uses[b] - 1) & 1u, MBAR_MAX_NS))
        return false;
      mbar_arrive_expect_tx(&mbar[5 + b], bytes);
      bulk_load(smem + (b ? S::oR1 : S::oR0), src + (size_t)k * bytes, bytes, &mbar[5 + b]);
      ++ring_fills[b];
      return true;
    };
    if (n > 0 && !fill(0)) return false;
    for (int k = 0; k < n; ++k) {
      const int b = (int)(chunk & 1u);
      if (k + 1 < n && !fill(k + 1)) return false;
      if (!tc::mbar_wait(&mbar[5 + b], ring_waits[b] & 1u, MBAR_MAX_NS)) return false;
      ++ring_waits[b];
      issue(k, tc::smem_u32(smem + (b ? S::oR1 : S::oR0)));
      tc::mma_commit(&mbar[b]);
      ++ring_uses[b];
      ++chunk;
    }
    return true;
  };

  uint32_t it = 0;
  for (int64_t batch = blockIdx.x; batch < a.nbatch; batch += gridDim.x, ++it) {
    const int64_t el0 = batch_first(a, batch);
    const int ne = batch_size(a, batch);
    const bool valid = lane_used && e_lane < ne;
    const int e_own = valid ? e_lane : 0;
    uint32_t* rmx = rsq;
    uint32_t* fmx = rsf;

    // ---- A: element data, vertex values, split state planes ----
    for (int x = tid; x < ne * G; x += S::THREADS) sgeo[x] = a.geo32[el0 * G + x];
    for (int x = tid; x < ne * NF; x += S::THREADS) sconn[x] = a.conn[el0 * NF + x];
    if constexpr (C != 0)
      for (int x = tid; x < ne * NP; x += S::THREADS) scoef[x] = (float)a.coeff[el0 * NP + x];
    for (int x = tid; x < F * EB * NV1; x += S::THREADS) {
      const int fe = x / NV1, vv = x % NV1, f = fe / EB, e = fe % EB;
      const int node = vv == 0 ? 0 : svert[vv - 1];
      sv[x] = e < ne ? a.q_in[f * Knp + (el0 + e) * NP + node] : 0.0;
    }
    if (tid < 256) rsq[tid] = 0u;   // both row-maxima arrays
    __syncthreads();
    float lin[DIM];
    {
      const double* v = sv + (fown * EB + e_own) * NV1;
#pragma unroll
      for (int d = 0; d < DIM; ++d) lin[d] = valid ? (float)(0.5 * (v[1 + d] - v[0])) : 0.f;
    }
    // remainders of 8 consecutive nodes of this thread's row (item chunk8):
    // the 8 state loads are issued before any is used
    auto rem8 = [&](int chunk8, float (&v)[8]) {
      const double* v3 = sv + (fown * EB + e_own) * NV1;
      const double* src = a.q_in + fown * Knp + (el0 + e_own) * NP;
      double q[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const int j = chunk8 * 8 + c;
        q[c] = (valid && j < NP) ? __ldg(src + j) : 0.0;
      }
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const int j = chunk8 * 8 + c;
        const int jj = j < NP ? j : 0;
        double l = v3[0];
#pragma unroll
        for (int d = 0; d < DIM; ++d) l += slam[jj * DIM + d] * (v3[1 + d] - v3[0]);
        v[c] = (valid && j < NP) ? (float)(q[c] - l) : 0.f;
      }
    };
    // this warp's items are warp + k * NW (all in its TMEM quadrant), NI
    // at a time so that 8 NI state loads are in flight
    constexpr int IPWS = S::NITEM / S::NW;
    constexpr int NI = IPWS % 4 == 0 ? 4 : 2;
    static_assert(IPWS % 2 == 0, "items per warp must be even");
    float inv = 1.0f;
    if constexpr (PT == PT_FP16) {
      // remainders once: row maxima, raw values parked in the planes
      uint32_t m = 0u;
#pragma unroll 1
      for (int k = 0; k < IPWS; k += NI) {
        float v[NI][8];
#pragma unroll
        for (int t = 0; t < NI; ++t) rem8((warp + (k + t) * S::NW) >> 2, v[t]);
#pragma unroll
        for (int t = 0; t < NI; ++t) {
#pragma unroll
          for (int c = 0; c < 8; ++c) m = max(m, __float_as_uint(fabsf(v[t][c])));
          park8(Aqh, Aql, kmajor_off(row, ((warp + (k + t) * S::NW) >> 2) * 8, KD), v[t]);
        }
      }
      atomicMax(&rmx[row], m);
      __syncthreads();
      inv = row_scale_inv(rmx[row]);
    }
#pragma unroll 1
    for (int k = 0; k < S::NITEM / S::NW; ++k) {
      const int chunk8 = (warp + k * S::NW) >> 2;
      const uint32_t off = kmajor_off(row, chunk8 * 8, KD);
      float v[8];
      if constexpr (PT == PT_FP16) {
        unpark8(Aqh, Aql, off, v);
#pragma unroll
        for (int c = 0; c < 8; ++c) v[c] *= inv;
      } else {
        rem8(chunk8, v);
      }
      uint32_t hw[4], lw[4];
#pragma unroll
      for (int c = 0; c < 8; c += 2) {
        const float x0 = v[c], x1 = v[c + 1];
        if constexpr (PT == PT_BF16) {
          const __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
          const float2 hf = __bfloat1622float2(h);
          const __nv_bfloat162 l = __floats2bfloat162_rn(x0 - hf.x, x1 - hf.y);
          hw[c / 2] = *reinterpret_cast<const uint32_t*>(&h);
          lw[c / 2] = *reinterpret_cast<const uint32_t*>(&l);
        } else {
          const __half2 h = __floats2half2_rn(x0, x1);
          const float2 hf = __half22float2(h);
          const __half2 l = __floats2half2_rn(x0 - hf.x, x1 - hf.y);
          hw[c / 2] = *reinterpret_cast<const uint32_t*>(&h);
          lw[c / 2] = *reinterpret_cast<const uint32_t*>(&l);
        }
      }
      *reinterpret_cast<uint4*>(Aqh + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
      *reinterpret_cast<uint4*>(Aql + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
    }
    tc::fence_proxy_async();
    __syncthreads();

    // ---- B: diff MMAs, operator chunks streamed by warp 0 (lane 0) while
    // the other warps start on the face fluxes, which do not need them ----
    if (warp == 0) {
      int ok = 1;
      if (lane == 0) {
        // L2 prefetch of the next batch's state (its remainders) and of this
        // batch's residual (the stage update), overlapping this batch's work
        const int64_t nxt = batch + gridDim.x;
        if (nxt < a.nbatch) {
          const int64_t n0 = batch_first(a, nxt);
          const int nn = batch_size(a, nxt);
          for (int f = 0; f < F; ++f) {
            const double* src = a.q_in + f * Knp + n0 * NP;
            if (aligned16(src, (uint32_t)(nn * NP * 8))) prefetch_l2(src, (uint32_t)(nn * NP * 8));
          }
        }
        if (a.mode != 0)
          for (int f = 0; f < F; ++f) {
            const double* src = a.res + f * Knp + el0 * NP;
            if (aligned16(src, (uint32_t)(ne * NP * 8))) prefetch_l2(src, (uint32_t)(ne * NP * 8));
          }
        const uint32_t aq_h = tc::smem_u32(Aqh), aq_l = tc::smem_u32(Aql);
        ok = stream_chunks(dimg, S::NKD, 2 * S::bDc, [&](int kk, uint32_t buf) {
          const uint32_t bh = buf, bl = buf + S::bDc;
          const uint64_t ah = tc::smem_desc(aq_h + kk * 256, 128, KD * 16);
          const uint64_t al = tc::smem_desc(aq_l + kk * 256, 128, KD * 16);
          const uint32_t acc0 = kk > 0 ? 1u : 0u;
          tc::mma_bf16(tmem_diff, ah, tc::smem_desc(bh, 128, 256), ID_D1, acc0);
          tc::mma_bf16(tmem_diff, ah, tc::smem_desc(bl, 128, 256), ID_D1, 1u);
          tc::mma_bf16(tmem_diff, al, tc::smem_desc(bh, 128, 256), ID_D1, 1u);
          if constexpr (S::ND2 > 0) {
            const uint32_t o2 = (S::ND1 / 8) * 256;
            tc::mma_bf16(tmem_diff + S::ND1, ah, tc::smem_desc(bh + o2, 128, 256), ID_D2, acc0);
            tc::mma_bf16(tmem_diff + S::ND1, ah, tc::smem_desc(bl + o2, 128, 256), ID_D2, 1u);
            tc::mma_bf16(tmem_diff + S::ND1, al, tc::smem_desc(bh + o2, 128, 256), ID_D2, 1u);
          }
        }) ? 1 : 0;
      }
      __syncwarp();
      if (!__shfl_sync(FULL, ok, 0)) bad = 1;
    }

    // ---- C: face fluxes (FP32 on jumps formed in FP64) -> lift planes ----
    auto face_flux = [&](int x, float (&fl)[F]) -> bool {
      const int e = x / NFPT, p = x % NFPT, face = p / NFP, k = p % NFP;
#pragma unroll
      for (int f = 0; f < F; ++f) fl[f] = 0.f;
      if (x >= S::NFACE || e >= ne) return false;
      const int lnode = sfm[p];
      float uM[NA], uP[NA], n[DIM];
      const float* gf = sgeo + e * G + DIM * DIM + face * (DIM + 1);
#pragma unroll
      for (int d = 0; d < DIM; ++d) n[d] = gf[d];
      const float fscale = gf[DIM];
      const int2 cn = sconn[e * NF + face];
      const int nb = cn.x;
      const int64_t gm = (el0 + e) * NP + lnode;
      bool have = true, bdry = false;
      if (nb >= a.K) {
        // neighbour on another partition: ext values from the halo buffer
        if (nb - a.K >= a.n_halo || a.halo == nullptr) {
          atomicCAS(a.err, 0, DEV_BAD_NEIGHBOUR);
          return false;
        }
        const int64_t hk = ((int64_t)nb - a.K) * NFP + k;
        if constexpr (JumpLinear<MODEL>::value) {
#pragma unroll
          for (int f = 0; f < F; ++f) {
            uM[f] = (float)(__ldg(a.q_in + f * Knp + gm) - a.halo[hk * F + f]);
            uP[f] = 0.f;
          }
        } else {
          if constexpr (C != 0) {
            uM[0] = scoef[e * NP + lnode];
            uP[0] = (float)a.halo_c[hk];
          }
#pragma unroll
          for (int f = 0; f < F; ++f) {
            uM[C + f] = (float)__ldg(a.q_in + f * Knp + gm);
            uP[C + f] = (float)a.halo[hk * F + f];
          }
        }
      } else if (nb >= 0) {
        const int nface = cn.y & 3, perm = cn.y >> 2;
        if (!(nface < NF && perm < a.nperm && nb < a.K)) {
          atomicCAS(a.err, 0, DEV_BAD_CODE);
          return false;
        }
        const int nn = sfm[nface * NFP + ssh[perm * NFP + k]];
        const int64_t gp = (int64_t)nb * NP + nn;
        if constexpr (JumpLinear<MODEL>::value) {
#pragma unroll
          for (int f = 0; f < F; ++f) {
            uM[f] = (float)(__ldg(a.q_in + f * Knp + gm) - __ldg(a.q_in + f * Knp + gp));
            uP[f] = 0.f;
          }
        } else {
          if constexpr (C != 0) {
            uM[0] = scoef[e * NP + lnode];
            uP[0] = (float)__ldg(a.coeff + gp);
          }
#pragma unroll
          for (int f = 0; f < F; ++f) {
            uM[C + f] = (float)__ldg(a.q_in + f * Knp + gm);
            uP[C + f] = (float)__ldg(a.q_in + f * Knp + gp);
          }
        }
      } else {
        bdry = true;
        if constexpr (C != 0) uM[0] = scoef[e * NP + lnode];
#pragma unroll
        for (int f = 0; f < F; ++f) uM[C + f] = (float)__ldg(a.q_in + f * Knp + gm);
        float given = 0.f;
        if (cn.y == HB_BC_GIVEN) {
          const int64_t bi = (int64_t)(-1 - nb) * NFP + k;
          if (a.bdry == nullptr || bi >= a.n_given) {
            atomicCAS(a.err, 0, a.bdry == nullptr ? DEV_MISSING_INPUT : DEV_BAD_BDRY_INDEX);
            have = false;
          } else {
            given = (float)__ldg(a.bdry + bi);
          }
        }
        if (have) have = model_bc<MODEL, DIM, float>(a.mp, cn.y, uM, n, given, uP);
      }
      if (!have) return false;
      model_flux<MODEL, DIM, float>(a.mp, bdry, uM, uP, n, fl);
#pragma unroll
      for (int f = 0; f < F; ++f) fl[f] *= fscale;
      return true;
    };
    // warps 1.. compute the fluxes (warp 0 drives the diff stream meanwhile);
    // face point x of thread ct is ct + u * CT
    constexpr int CT = S::THREADS - 32;
    constexpr int NFVC = (S::NFACE + CT - 1) / CT;
    const int ct = tid - 32;
    if constexpr (PT == PT_FP16) {
      // fluxes once: row maxima, raw values parked in the planes; then
      // every thread splits its own entries with the row scale
      for (int u = 0; u < NFVC && warp != 0; ++u) {
        const int x = ct + u * CT;
        float fl[F];
        face_flux(x, fl);
        const int e = x < S::NFACE ? x / NFPT : -1;
        const unsigned grp = __match_any_sync(FULL, e);
        const bool leader = (__ffs(grp) - 1) == lane;
#pragma unroll
        for (int f = 0; f < F; ++f) {
          const unsigned m = __reduce_max_sync(grp, __float_as_uint(fabsf(fl[f])));
          if (leader && e >= 0 && e < ne) atomicMax(&fmx[(e / EPW) * 32 + (e % EPW) * F + f], m);
        }
        if (e >= 0 && e < ne) {
          const int p = x % NFPT, rowb = (e / EPW) * 32 + (e % EPW) * F;
#pragma unroll
          for (int f = 0; f < F; ++f) park_f32(Afh, Afl, kmajor_off(rowb + f, p, KL), fl[f]);
        }
      }
      __syncthreads();
      for (int u = 0; u < NFVC && warp != 0; ++u) {
        const int x = ct + u * CT;
        const int e = x / NFPT, p = x % NFPT;
        if (x < S::NFACE && e < ne) {
          const int rowb = (e / EPW) * 32 + (e % EPW) * F;
#pragma unroll
          for (int f = 0; f < F; ++f) {
            const uint32_t off = kmajor_off(rowb + f, p, KL);
            store_split<PT>(Afh, Afl, off,
                            unpark_f32(Afh, Afl, off) * row_scale_inv(fmx[rowb + f]));
          }
        }
      }
    } else {
      for (int u = 0; u < NFVC && warp != 0; ++u) {
        const int x = ct + u * CT;
        float fl[F];
        face_flux(x, fl);
        const int e = x / NFPT, p = x % NFPT;
        if (x < S::NFACE && e < ne) {
          const int rowb = (e / EPW) * 32 + (e % EPW) * F;
#pragma unroll
          for (int f = 0; f < F; ++f)
            store_split<PT>(Afh, Afl, kmajor_off(rowb + f, p, KL), fl[f]);
        }
      }
    }
    tc::fence_proxy_async();
    // (every thread learns whether the diff stream gave up)
    if (__syncthreads_or(bad)) {
      if (tid == 0) atomicCAS(a.err, 0, DEV_MMA_TIMEOUT);
      break;
    }

    // ---- D: lift MMAs, operator chunks streamed by thread 0 ----
    {
      int ok = 1;
      if (tid == 0) {
        tc::fence_after_sync();
        const uint32_t af_h = tc::smem_u32(Afh), af_l = tc::smem_u32(Afl);
        ok = stream_chunks(limg, S::NKL, 2 * S::bLc, [&](int kk, uint32_t buf) {
          const uint32_t bh = buf, bl = buf + S::bLc;
          const uint64_t ah = tc::smem_desc(af_h + kk * 256, 128, KL * 16);
          const uint64_t al = tc::smem_desc(af_l + kk * 256, 128, KL * 16);
          tc::mma_bf16(tmem_lift, ah, tc::smem_desc(bh, 128, 256), ID_L, kk > 0 ? 1u : 0u);
          tc::mma_bf16(tmem_lift, ah, tc::smem_desc(bl, 128, 256), ID_L, 1u);
          tc::mma_bf16(tmem_lift, al, tc::smem_desc(bh, 128, 256), ID_L, 1u);
        }) ? 1 : 0;
        if (ok) tc::mma_commit(&mbar[2]);   // all of this batch's MMAs
      }
      if (__syncthreads_or(!ok)) {
        if (tid == 0) atomicCAS(a.err, 0, DEV_MMA_TIMEOUT);
        break;
      }
    }

    // ---- E: TMEM -> chain rule, volume terms, + lift -> staged rhs ----
    {
      int late = 0;
      if (tid == 0) late = !tc::mbar_wait(&mbar[2], it & 1u, MBAR_MAX_NS);
      if (__syncthreads_or(late)) {
        if (tid == 0) {
          atomicCAS(a.err, 0, DEV_MMA_TIMEOUT);
          tc::mbar_wait(&mbar[2], it & 1u, MBAR_MAX_NS);
        }
        __syncthreads();
        break;
      }
    }
    tc::fence_after_sync();
    {
      const float* ge = sgeo + e_own * G;
      float gm[DIM][DIM];
#pragma unroll
      for (int r = 0; r < DIM; ++r)
#pragma unroll
        for (int x = 0; x < DIM; ++x) gm[r][x] = ge[r * DIM + x];
      const int base = lf * F;
      float sdiff = a.op_scale_d, slift = a.op_scale_l;
      if constexpr (PT == PT_FP16) {
        sdiff *= row_scale(rmx[row]);
        slift *= row_scale(fmx[row]);
      }
      const int i_lo = part * S::NPQ;
      const int i_hi = (part + 1) * S::NPQ < NP ? (part + 1) * S::NPQ : NP;
      constexpr int CHK = 8;
#pragma unroll 1
      for (int c0 = i_lo; c0 < i_hi; c0 += CHK) {
        float dv[DIM][CHK], lv[CHK];
#pragma unroll
        for (int g = 0; g < CHK / 4; ++g) {
          if (c0 + 4 * g < i_hi) {
#pragma unroll
            for (int r = 0; r < DIM; ++r)
              tc::tmem_ld4(tmem_diff + lane_addr + r * NP + c0 + 4 * g,
                           *reinterpret_cast<float(*)[4]>(&dv[r][4 * g]));
            tc::tmem_ld4(tmem_lift + lane_addr + c0 + 4 * g,
                         *reinterpret_cast<float(*)[4]>(&lv[4 * g]));
          }
        }
        tc::tmem_wait_ld();
#pragma unroll
        for (int c = 0; c < CHK; ++c) {
          const int i = c0 + c;
          if (i >= i_hi) break;
          float g[DIM];
#pragma unroll
          for (int x = 0; x < DIM; ++x) {
            float s = 0.f;
#pragma unroll
            for (int r = 0; r < DIM; ++r) s += gm[r][x] * (dv[r][c] * sdiff + lin[r]);
            g[x] = s;
          }
          const float cnode = C ? scoef[e_own * NP + i] : 0.f;
          const float mine = volume_own<MODEL, DIM>(a.mp, g, base, fown, cnode);
          if (valid) {
            const int64_t si = model_src_index<MODEL>(fown, (el0 + e_own) * NP + i, Knp);
            const float src = (a.source && si >= 0) ? (float)a.source[si] : 0.f;
            sq[fown * FNP + e_own * NP + i] =
                model_finish<MODEL, DIM, float>(a.mp, fown, mine, lv[c] * slift, src);
          }
        }
      }
    }
    tc::fence_before_sync();
    __syncthreads();

    // ---- F: FP64 stage update (coalesced; UF values per thread in flight) ----
    {
      constexpr int UF = 10;
      for (int x0 = tid; x0 < S::NVAL; x0 += UF * S::THREADS) {
        double r0[UF], q0[UF];
        int64_t idx[UF];
        bool ok[UF];
#pragma unroll
        for (int u = 0; u < UF; ++u) {
          const int x = x0 + u * S::THREADS;
          const int f = x / FNP, r = x - f * FNP;
          ok[u] = x < S::NVAL && r < ne * NP;
          idx[u] = f * Knp + el0 * NP + r;
          r0[u] = q0[u] = 0.0;
          if (ok[u] && a.mode != 0) {
            r0[u] = a.res[idx[u]];
            q0[u] = __ldg(a.q_in + idx[u]);
          }
        }
#pragma unroll
        for (int u = 0; u < UF; ++u) {
          if (!ok[u]) continue;
          const double rr = (double)sq[x0 + u * S::THREADS];
          if (a.mode == 0) {
            a.q_out[idx[u]] = rr;
          } else {
            const double nr = a.ra * r0[u] + a.dt * rr;
            a.res[idx[u]] = nr;
            a.q_out[idx[u]] = q0[u] + a.rb * nr;
          }
        }
      }
    }
    __syncthreads();
  }

  // ---- tear-down: wait for copies and MMAs still using the ring, release TMEM ----
  if (tid == 0) {
    for (int b = 0; b < 2; ++b) {
      for (uint32_t w = ring_waits[b]; w < ring_fills[b]; ++w)
        tc::mbar_wait(&mbar[5 + b], w & 1u, MBAR_MAX_NS);
      if (ring_uses[b] > 0) tc::mbar_wait(&mbar[b], (ring_uses[b] - 1) & 1u, MBAR_MAX_NS);
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, S::TMEM_COLS);
}

// ---------------------------------------------------------------------------
// host side

struct SplitOps {
  uint8_t* dev = nullptr;
  int order = 0;
  int stream = 0;   // 1: streamed-operator variant
  float scale_d = 1.f, scale_l = 1.f;
};

static uint16_t host_bf16(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7fffffffu) > 0x7f800000u) return 0x7fc0;  // NaN
  const uint32_t lsb = (u >> 16) & 1u;
  u += 0x7fffu + lsb;
  return (uint16_t)(u >> 16);
}
static float host_bf16_to_float(uint16_t h) {
  uint32_t u = (uint32_t)h << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

static uint16_t host_fp16(float f) {
  // round-to-nearest-even FP32 -> FP16 for normal-range values (the operator
  // planes are scaled into [2^-14, 2^14))
  uint32_t u;
  std::memcpy(&u, &f, 4);
  const uint32_t sign = (u >> 16) & 0x8000u;
  const int exp = (int)((u >> 23) & 0xff) - 127 + 15;
  uint32_t mant = u & 0x7fffffu;
  if (exp <= 0) {  // subnormal / zero in FP16
    if (exp < -10) return (uint16_t)sign;
    mant |= 0x800000u;
    const int shift = 14 - exp;
    uint32_t half = mant >> shift;
    const uint32_t rem = mant & ((1u << shift) - 1), mid = 1u << (shift - 1);
    if (rem > mid || (rem == mid && (half & 1u))) ++half;
    return (uint16_t)(sign | half);
  }
  uint32_t half = ((uint32_t)exp << 10) | (mant >> 13);
  const uint32_t rem = mant & 0x1fffu;
  if (rem > 0x1000u || (rem == 0x1000u && (half & 1u))) ++half;
  return (uint16_t)(sign | half);
}
static float host_fp16_to_float(uint16_t h) {
  const uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
  const int exp = (h >> 10) & 0x1f;
  const uint32_t mant = h & 0x3ffu;
  float f;
  if (exp == 0) {
    f = std::ldexp((float)mant, -24);
  } else {
    f = std::ldexp((float)(mant | 0x400u), exp - 25);
  }
  uint32_t u;
  std::memcpy(&u, &f, 4);
  u |= sign;
  std::memcpy(&f, &u, 4);
  return f;
}

// hi/lo planes of a (rows x cols) FP64 matrix (scaled by 1/scale) in the
// canonical K-major image, BF16 or FP16
static void build_planes(const std::vector<double>& m, int rows, int cols, int rp, int kp,
                         int pt, double scale, uint8_t* hi, uint8_t* lo) {
  std::memset(hi, 0, (size_t)rp * kp * 2);
  std::memset(lo, 0, (size_t)rp * kp * 2);
  for (int r = 0; r < rows; ++r)
    for (int k = 0; k < cols; ++k) {
      const double v = m[(size_t)r * cols + k] / scale;
      uint16_t h, l;
      if (pt == PT_BF16) {
        h = host_bf16((float)v);
        l = host_bf16((float)(v - (double)host_bf16_to_float(h)));
      } else {
        h = host_fp16((float)v);
        l = host_fp16((float)(v - (double)host_fp16_to_float(h)));
      }
      const uint32_t off = kmajor_off(r, k, kp);
      std::memcpy(hi + off, &h, 2);
      std::memcpy(lo + off, &l, 2);
    }
}

// power of two that maps max|m| into [2^13, 2^14) (FP16 planes), else 1
static double plane_scale(const std::vector<double>& m, int pt) {
  if (pt == PT_BF16) return 1.0;
  double mx = 0;
  for (double v : m) mx = std::max(mx, std::fabs(v));
  if (mx == 0) return 1.0;
  int e;
  std::frexp(mx, &e);          // mx in [2^(e-1), 2^e)
  return std::ldexp(1.0, e - 14);
}

// Batches of a persistent grid of `grid` CTAs.  ceil(K / EB) batches of EB
// elements leave the last round partly empty (2400 batches on 148 CTAs: 16
// rounds and 32 batches of 20 elements, so 32 CTAs run one batch more than
// the rest).  Rounding the count up to whole rounds and spreading the
// elements evenly over them, in units of `unit` elements (at most EB per
// batch; the last batch also takes the K % unit elements left over), makes
// the batches of every CTA add up to about the same work.  `unit` keeps every
// batch's state, geometry and face-table slices 16-byte aligned (bulk copies,
// 16-byte update accesses).  Fills nbatch, bq, brem, bunit.
template <typename A>
static void balance_batches(A& a, int64_t K, int EB, int unit, int grid) {
  const int64_t nb0 = (K + EB - 1) / EB;
  a.nbatch = nb0; a.bq = 1; a.brem = 0; a.bunit = EB;   // plain batches of EB
  if (grid <= 0 || nb0 <= grid || unit < 1 || EB % unit != 0) return;
  const int64_t nb = (nb0 + grid - 1) / grid * grid;
  const int64_t units = K / unit, left = K % unit;
  const int64_t bq = units / nb, brem = units % nb;
  const int64_t largest = std::max<int64_t>(unit * (bq + (brem > 0 ? 1 : 0)), unit * bq + left);
  if (bq < 1 || largest > EB) return;
  a.nbatch = nb; a.bq = bq; a.brem = brem; a.bunit = unit;
}
// smallest element count whose slices of `bytes_per_element` bytes end on a
// 16-byte boundary
static constexpr int align_unit(int bytes_per_element) {
  int u = 1;
  while ((u * bytes_per_element) % 16 != 0) ++u;
  return u;
}
static constexpr int lcm_small(int x, int y) {
  int m = x;
  while (m % y != 0) m += x;
  return m;
}

template <int MODEL, int DIM, int ORDER, int PT, typename ST = double>
static hb_status configure_split(Op* op) {
  using S = Shape<MODEL, DIM, ORDER, (int)sizeof(ST)>;
  Discr* d = op->d;
  if constexpr (!S::FITS) {
    return fail(HB_ERR_UNSUPPORTED, "BF16x3 kernel: element beyond one MMA (N <= 256)");
  } else {
    if (d->np != S::NP || d->nfp != S::NFP)
      return fail(HB_ERR_INVALID_ARGUMENT, "element sizes do not match the order");
    auto kern = rhs_split_kernel<MODEL, DIM, ORDER, PT, ST>;
    int dev;
    HB_CUDA(cudaGetDevice(&dev));
    int max_optin = 0, sms = 0, smem_sm = 0;
    HB_CUDA(cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    HB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    HB_CUDA(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    if (S::total > (uint32_t)max_optin)
      return fail(HB_ERR_UNSUPPORTED, "BF16x3 kernel: element too large for shared memory");
    // TMEM: at most 512 columns per SM are shared by the resident CTAs; pad
    // the shared-memory request so that no more CTAs fit than TMEM allows.
    const int max_ctas = 512 / (int)S::TMEM_COLS;
    size_t smem = S::total;
    if ((size_t)smem_sm / (smem + 1024) > (size_t)max_ctas)
      smem = (size_t)smem_sm / max_ctas - 1024 + 16;
    if (smem > (size_t)max_optin) smem = max_optin;
    HB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    HB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    // resident CTAs per SM from the kernel's own resource use (the runtime's
    // occupancy query under-reports this kernel)
    cudaFuncAttributes fa;
    HB_CUDA(cudaFuncGetAttributes(&fa, kern));
    int regs_sm = 0, thr_sm = 0;
    HB_CUDA(cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev));
    HB_CUDA(cudaDeviceGetAttribute(&thr_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev));
    const int by_smem = (int)(smem_sm / (smem + 1024));
    // registers: each of the 4 sub-partitions holds a quarter of the file and
    // receives every 4th warp
    const int regs_warp = (fa.numRegs * 32 + 255) / 256 * 256;
    const int warps_part = (SPLIT_THREADS / 32 + 3) / 4;
    const int by_regs = (regs_sm / 4) / std::max(regs_warp * warps_part, 1);
    const int per_sm = std::min(std::min(by_smem, by_regs), thr_sm / SPLIT_THREADS);
    if (per_sm < 1) return fail(HB_ERR_UNSUPPORTED, "BF16x3 kernel does not fit on an SM");
    if (per_sm > max_ctas) return fail(HB_ERR_UNSUPPORTED, "TMEM oversubscribed");
    const int64_t nbatch = (d->K + S::EB - 1) / S::EB;
    op->threads = SPLIT_THREADS;
    op->blocks_per_sm = per_sm;
    op->smem = smem;
    op->grid = (int)std::min<int64_t>(nbatch, (int64_t)sms * per_sm);
    op->elems_per_block = S::EB;
    // operator images from the FP64 operators (host copies, transposed blob)
    const int np = S::NP, nfpt = S::NFPT;
    const double* h = reinterpret_cast<const double*>(d->host_blob.data());
    const size_t ndm = (size_t)DIM * np * np;
    std::vector<double> Dt((size_t)DIM * np * np);   // rows (r, i), cols j
    for (int r = 0; r < DIM; ++r)
      for (int j = 0; j < np; ++j)
        for (int i = 0; i < np; ++i)
          Dt[((size_t)r * np + i) * np + j] = h[((size_t)r * np + j) * np + i];
    std::vector<double> Lt((size_t)np * nfpt);        // rows i, cols p
    for (int k = 0; k < nfpt; ++k)
      for (int i = 0; i < np; ++i) Lt[(size_t)i * nfpt + k] = h[ndm + (size_t)k * np + i];
    const size_t bD = (size_t)S::ND * S::KD * 2, bL = (size_t)S::NL * S::KL * 2;
    std::vector<uint8_t> img(2 * bD + 2 * bL + S::LIN_BYTES);
    {
      // vertex nodes B, C(, D) of the reference element and the FP64 linear
      // barycentric weights (1 + r_d)/2 of every node
      uint8_t vert[4] = {0, 0, 0, 0};
      for (int dd = 0; dd < DIM; ++dd) {
        int best = -1;
        for (int j = 0; j < np; ++j) {
          bool hit = true;
          for (int c = 0; c < DIM; ++c) {
            const double want = (c == dd) ? 1.0 : -1.0;
            if (std::fabs(d->unit_nodes[(size_t)j * DIM + c] - want) > 1e-12) hit = false;
          }
          if (hit) best = j;
        }
        if (best < 0) return fail(HB_ERR_INVALID_ARGUMENT, "reference element lacks vertex nodes");
        vert[dd] = (uint8_t)best;
      }
      for (int c = 0; c < DIM; ++c)
        if (std::fabs(d->unit_nodes[c] + 1.0) > 1e-12)
          return fail(HB_ERR_INVALID_ARGUMENT, "node 0 is not the first vertex");
      std::memcpy(img.data() + 2 * bD + 2 * bL, vert, 4);
      double* lam = reinterpret_cast<double*>(img.data() + 2 * bD + 2 * bL + 8);
      for (int j = 0; j < np; ++j)
        for (int dd = 0; dd < DIM; ++dd)
          lam[j * DIM + dd] = 0.5 * (1.0 + d->unit_nodes[(size_t)j * DIM + dd]);
      // the kernel reads the weights from constant memory (per dimension and
      // order; every discretization of that order writes the same values)
      static_assert(S::NP * DIM <= LAM_MAX && ORDER < LAM_ORDERS, "weight table too small");
      const size_t slot = ((size_t)(DIM - 2) * LAM_ORDERS + ORDER) * LAM_MAX;
      if constexpr (sizeof(ST) == 8) {
        HB_CUDA(cudaMemcpyToSymbol(c_lam, lam, sizeof(double) * np * DIM,
                                   sizeof(double) * slot));
      } else {
        std::vector<float> lamf((size_t)np * DIM);
        for (size_t x = 0; x < lamf.size(); ++x) lamf[x] = (float)lam[x];
        HB_CUDA(cudaMemcpyToSymbol(c_lamf, lamf.data(), sizeof(float) * lamf.size(),
                                   sizeof(float) * slot));
      }
    }
    const double sd = plane_scale(Dt, PT), sl = plane_scale(Lt, PT);
    build_planes(Dt, DIM * np, np, S::ND, S::KD, PT, sd, img.data(), img.data() + bD);
    build_planes(Lt, np, nfpt, S::NL, S::KL, PT, sl, img.data() + 2 * bD,
                 img.data() + 2 * bD + bL);
    SplitOps* so = static_cast<SplitOps*>(op->split_ops);
    so->scale_d = (float)sd;
    so->scale_l = (float)sl;
    if (cudaMalloc(&so->dev, img.size()) != cudaSuccess ||
        cudaMemcpy(so->dev, img.data(), img.size(), cudaMemcpyHostToDevice) != cudaSuccess)
      return fail(HB_ERR_CUDA, "cannot upload the split operator planes");
    return HB_OK;
  }
}

template <int MODEL, int DIM, int ORDER, int PT, typename ST = double>
static hb_status launch_split_t(Op* op, int mode, double ra, double rb, double dt,
                                const void* q_in, void* q_out, void* res,
                                const double* coeff, const double* bdry,
                                const double* source, int64_t e0, int64_t e1,
                                cudaStream_t s) {
  using S = Shape<MODEL, DIM, ORDER, (int)sizeof(ST)>;
  if constexpr (!S::FITS) {
    return fail(HB_ERR_UNSUPPORTED, "BF16x3 kernel: element beyond one MMA");
  } else {
    Discr* d = op->d;
    SplitOps* so = static_cast<SplitOps*>(op->split_ops);
    SplitArgsT<ST> a;
    a.K = d->K;
    a.e_begin = e0;
    a.e_end = e1;
    {
      constexpr int unit = lcm_small(
          lcm_small(align_unit(S::NP * (int)sizeof(ST)), align_unit(S::G * 4)),
          lcm_small(align_unit(S::NF * 8), S::C ? align_unit(S::NP * 8) : 1));
      balance_batches(a, e1 - e0, S::EB, unit, op->grid);
    }
    a.n_given = op->n_given;
    a.nperm = d->nperm;
    a.ops = so->dev;
    a.geo32 = d->geo32;
    a.conn = op->conn; a.fmask = d->fmask; a.shuffle = d->shuffle;
    a.q_in = static_cast<const ST*>(q_in);
    a.q_out = static_cast<ST*>(q_out);
    a.res = static_cast<ST*>(res);
    a.coeff = coeff; a.bdry = bdry; a.source = source;
    a.halo = static_cast<const ST*>(op->halo);
    a.halo_c = op->halo_c;
    a.n_halo = op->n_halo;
    a.ra = ra; a.rb = rb; a.dt = dt; a.mode = mode;
    a.op_scale_d = so->scale_d;
    a.op_scale_l = so->scale_l;
    a.mp = op->mp;
    a.err = op->err_flag;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)std::min<int64_t>(op->grid, a.nbatch));
    cfg.blockDim = dim3((unsigned)op->threads);
    cfg.dynamicSmemBytes = op->smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = HB_SPLIT_PDL ? 1 : 0;
    HB_CUDA(cudaLaunchKernelEx(&cfg, rhs_split_kernel<MODEL, DIM, ORDER, PT, ST>, a));
    return HB_OK;
  }
}


// ---- streamed-operator variant (high orders) ----

// one 16-column K chunk [k0, k0 + 16) of a (rows x cols) FP64 matrix (scaled
// by 1/scale) as hi/lo planes of rp rows in the canonical K-major layout
static void build_chunk(const std::vector<double>& m, int rows, int cols, int rp, int k0,
                        int pt, double scale, uint8_t* hi, uint8_t* lo) {
  std::memset(hi, 0, (size_t)rp * 16 * 2);
  std::memset(lo, 0, (size_t)rp * 16 * 2);
  for (int r = 0; r < rows; ++r)
    for (int k = k0; k < cols && k < k0 + 16; ++k) {
      const double v = m[(size_t)r * cols + k] / scale;
      uint16_t h, l;
      if (pt == PT_BF16) {
        h = host_bf16((float)v);
        l = host_bf16((float)(v - (double)host_bf16_to_float(h)));
      } else {
        h = host_fp16((float)v);
        l = host_fp16((float)(v - (double)host_fp16_to_float(h)));
      }
      const uint32_t off = kmajor_off(r, k - k0, 16);
      std::memcpy(hi + off, &h, 2);
      std::memcpy(lo + off, &l, 2);
    }
}

template <int MODEL, int DIM, int ORDER, int PT>
static hb_status configure_stream(Op* op) {
  using S = ShapeS<MODEL, DIM, ORDER>;
  Discr* d = op->d;
  if constexpr (!S::FITS) {
    return fail(HB_ERR_UNSUPPORTED, "split kernel: element too large for the streamed variant");
  } else {
    if (d->np != S::NP || d->nfp != S::NFP)
      return fail(HB_ERR_INVALID_ARGUMENT, "element sizes do not match the order");
    auto kern = rhs_split_stream_kernel<MODEL, DIM, ORDER, PT>;
    int dev, max_optin = 0, sms = 0;
    HB_CUDA(cudaGetDevice(&dev));
    HB_CUDA(cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    HB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (S::total > (uint32_t)max_optin)
      return fail(HB_ERR_UNSUPPORTED, "split kernel: streamed variant exceeds shared memory");
    // one CTA per SM: pad the request so that TMEM is never oversubscribed
    int smem_sm = 0;
    HB_CUDA(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    size_t smem = S::total;
    const int max_ctas = 512 / (int)S::TMEM_COLS;
    if ((size_t)smem_sm / (smem + 1024) > (size_t)max_ctas)
      smem = std::min<size_t>((size_t)smem_sm / max_ctas - 1024 + 16, (size_t)max_optin);
    HB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int64_t nbatch = (d->K + S::EB - 1) / S::EB;
    op->threads = S::THREADS;
    op->blocks_per_sm = 1;
    op->smem = smem;
    op->grid = (int)std::min<int64_t>(nbatch, (int64_t)sms);
    op->elems_per_block = S::EB;
    const int np = S::NP, nfpt = S::NFPT;
    const double* h = reinterpret_cast<const double*>(d->host_blob.data());
    const size_t ndm = (size_t)DIM * np * np;
    std::vector<double> Dt((size_t)DIM * np * np);
    for (int r = 0; r < DIM; ++r)
      for (int j = 0; j < np; ++j)
        for (int i = 0; i < np; ++i)
          Dt[((size_t)r * np + i) * np + j] = h[((size_t)r * np + j) * np + i];
    std::vector<double> Lt((size_t)np * nfpt);
    for (int k = 0; k < nfpt; ++k)
      for (int i = 0; i < np; ++i) Lt[(size_t)i * nfpt + k] = h[ndm + (size_t)k * np + i];
    const size_t dbytes = (size_t)S::NKD * 2 * S::bDc, lbytes = (size_t)S::NKL * 2 * S::bLc;
    std::vector<uint8_t> img(dbytes + lbytes + S::LIN_BYTES);
    const double sd = plane_scale(Dt, PT), sl = plane_scale(Lt, PT);
    for (int kk = 0; kk < S::NKD; ++kk) {
      uint8_t* c = img.data() + (size_t)kk * 2 * S::bDc;
      build_chunk(Dt, DIM * np, np, S::ND, 16 * kk, PT, sd, c, c + S::bDc);
    }
    for (int kk = 0; kk < S::NKL; ++kk) {
      uint8_t* c = img.data() + dbytes + (size_t)kk * 2 * S::bLc;
      build_chunk(Lt, np, nfpt, S::NL, 16 * kk, PT, sl, c, c + S::bLc);
    }
    {
      uint8_t vert[4] = {0, 0, 0, 0};
      for (int dd = 0; dd < DIM; ++dd) {
        int best = -1;
        for (int j = 0; j < np; ++j) {
          bool hit = true;
          for (int c = 0; c < DIM; ++c) {
            const double want = (c == dd) ? 1.0 : -1.0;
            if (std::fabs(d->unit_nodes[(size_t)j * DIM + c] - want) > 1e-12) hit = false;
          }
          if (hit) best = j;
        }
        if (best < 0) return fail(HB_ERR_INVALID_ARGUMENT, "reference element lacks vertex nodes");
        vert[dd] = (uint8_t)best;
      }
      uint8_t* t = img.data() + dbytes + lbytes;
      std::memcpy(t, vert, 4);
      double* lam = reinterpret_cast<double*>(t + 8);
      for (int j = 0; j < np; ++j)
        for (int dd = 0; dd < DIM; ++dd)
          lam[j * DIM + dd] = 0.5 * (1.0 + d->unit_nodes[(size_t)j * DIM + dd]);
    }
    SplitOps* so = static_cast<SplitOps*>(op->split_ops);
    so->scale_d = (float)sd;
    so->scale_l = (float)sl;
    so->stream = 1;
    if (cudaMalloc(&so->dev, img.size()) != cudaSuccess ||
        cudaMemcpy(so->dev, img.data(), img.size(), cudaMemcpyHostToDevice) != cudaSuccess)
      return fail(HB_ERR_CUDA, "cannot upload the split operator planes");
    return HB_OK;
  }
}

template <int MODEL, int DIM, int ORDER, int PT>
static hb_status launch_stream_t(Op* op, int mode, double ra, double rb, double dt,
                                 const void* q_in, void* q_out, void* res,
                                 const double* coeff, const double* bdry,
                                 const double* source, int64_t e0, int64_t e1,
                                 cudaStream_t s) {
  using S = ShapeS<MODEL, DIM, ORDER>;
  if constexpr (!S::FITS) {
    return fail(HB_ERR_UNSUPPORTED, "split kernel: element too large for the streamed variant");
  } else {
    Discr* d = op->d;
    SplitOps* so = static_cast<SplitOps*>(op->split_ops);
    SplitArgs a;
    a.K = d->K;
    a.e_begin = e0;
    a.e_end = e1;
    {
      constexpr int unit = lcm_small(lcm_small(align_unit(S::NP * 8), align_unit(S::G * 4)),
                                     align_unit(S::NF * 8));
      balance_batches(a, e1 - e0, S::EB, unit, op->grid);
    }
    a.n_given = op->n_given;
    a.nperm = d->nperm;
    a.ops = so->dev;
    a.geo32 = d->geo32;
    a.conn = op->conn; a.fmask = d->fmask; a.shuffle = d->shuffle;
    a.q_in = static_cast<const double*>(q_in);
    a.q_out = static_cast<double*>(q_out);
    a.res = static_cast<double*>(res);
    a.coeff = coeff; a.bdry = bdry; a.source = source;
    a.halo = static_cast<const double*>(op->halo);
    a.halo_c = op->halo_c;
    a.n_halo = op->n_halo;
    a.ra = ra; a.rb = rb; a.dt = dt; a.mode = mode;
    a.op_scale_d = so->scale_d;
    a.op_scale_l = so->scale_l;
    a.mp = op->mp;
    a.err = op->err_flag;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)std::min<int64_t>(op->grid, a.nbatch));
    cfg.blockDim = dim3((unsigned)op->threads);
    cfg.dynamicSmemBytes = op->smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = HB_SPLIT_PDL ? 1 : 0;
    HB_CUDA(cudaLaunchKernelEx(&cfg, rhs_split_stream_kernel<MODEL, DIM, ORDER, PT>, a));
    return HB_OK;
  }
}

// high-order instances of the streamed variant
#define HB_SPLIT_STREAM_INSTANCES(X) \
  X(HB_MODEL_WAVE, 3, 5) X(HB_MODEL_MAXWELL, 3, 5) \
  X(HB_MODEL_WAVE, 3, 6) X(HB_MODEL_WAVE, 3, 7) X(HB_MODEL_MAXWELL, 3, 6)

// (model, dim, order) instances built into the library
#define HB_SPLIT_INSTANCES(X)                                                          \
  X(HB_MODEL_ADVECTION, 2, 3) X(HB_MODEL_ADVECTION, 2, 4) X(HB_MODEL_ADVECTION, 2, 5)  \
  X(HB_MODEL_ADVECTION, 2, 6) X(HB_MODEL_ADVECTION, 3, 3) X(HB_MODEL_ADVECTION, 3, 4)  \
  X(HB_MODEL_WAVE, 2, 3) X(HB_MODEL_WAVE, 2, 4) X(HB_MODEL_WAVE, 2, 5)                 \
  X(HB_MODEL_WAVE, 2, 6) X(HB_MODEL_WAVE, 3, 3) X(HB_MODEL_WAVE, 3, 4)                 \
  X(HB_MODEL_WAVE, 3, 5)                                                               \
  X(HB_MODEL_VARWAVE, 2, 3) X(HB_MODEL_VARWAVE, 2, 4) X(HB_MODEL_VARWAVE, 2, 5)        \
  X(HB_MODEL_VARWAVE, 2, 6) X(HB_MODEL_VARWAVE, 3, 3) X(HB_MODEL_VARWAVE, 3, 4)        \
  X(HB_MODEL_MAXWELL, 3, 3) X(HB_MODEL_MAXWELL, 3, 4) X(HB_MODEL_MAXWELL, 3, 5)

// The streamed-operator kernel serves the instances it is built for (with or
// without halo faces): at 3D N = 5 the resident kernel's operator planes
// leave room for one state stage and no residual buffer, and the streamed
// kernel is 13-14 % faster there; at N >= 6 it is the only one.
hb_status prepare_split(Op* op) {
  Discr* d = op->d;
  hb_status st = ensure_fp32(d);
  if (st) return st;
  op->split_ops = new SplitOps();
  static_cast<SplitOps*>(op->split_ops)->order = d->order;
  const int dim = d->dim, order = d->order;
  if (op->precision == HB_PREC_FP32) {
    // FP32 state: resident kernels with FP16 planes
#define HB_CASE(M, D, O)                                                       \
  if (op->model == M && dim == D && order == O)                                \
    return configure_split<M, D, O, PT_FP16, float>(op);
    HB_SPLIT_INSTANCES(HB_CASE)
#undef HB_CASE
    return fail(HB_ERR_UNSUPPORTED, "no FP32-state tensor-core kernel for this instance");
  }
  const int pt = op->precision == HB_PREC_FP16X3 ? PT_FP16 : PT_BF16;
  {
    // a streamed variant that this device refuses (e.g. its shared memory)
    // falls back to the resident kernel where one is built
    bool tried = false;
    hb_status sst = HB_ERR_UNSUPPORTED;
#define HB_CASE(M, D, O)                                                       \
  if (!tried && op->model == M && dim == D && order == O) {                    \
    tried = true;                                                              \
    sst = pt == PT_FP16 ? configure_stream<M, D, O, PT_FP16>(op)               \
                        : configure_stream<M, D, O, PT_BF16>(op);              \
  }
    HB_SPLIT_STREAM_INSTANCES(HB_CASE)
#undef HB_CASE
    if (tried && sst == HB_OK) return HB_OK;
    if (tried) {
      SplitOps* so = static_cast<SplitOps*>(op->split_ops);
      if (so->dev) cudaFree(so->dev);
      so->dev = nullptr;
      so->stream = 0;
      so->scale_d = so->scale_l = 1.f;
    }
  }
#define HB_CASE(M, D, O)                                                       \
  if (op->model == M && dim == D && order == O)                                \
    return pt == PT_FP16 ? configure_split<M, D, O, PT_FP16>(op)               \
                         : configure_split<M, D, O, PT_BF16>(op);
  HB_SPLIT_INSTANCES(HB_CASE)
#undef HB_CASE
  return fail(HB_ERR_UNSUPPORTED,
              "split path: this (model, dimension, order) is not built (see "
              "HB_SPLIT_INSTANCES, HB_SPLIT_STREAM_INSTANCES)");
}

hb_status launch_split(Op* op, int mode, double ra, double rb, double dt,
                       const void* q_in, void* q_out, void* res, const double* coeff,
                       const double* bdry, const double* source, int64_t e0, int64_t e1,
                       cudaStream_t s) {
  const int dim = op->d->dim, order = op->d->order;
  const int pt = op->precision == HB_PREC_FP16X3 ? PT_FP16 : PT_BF16;
  const SplitOps* so = static_cast<const SplitOps*>(op->split_ops);
  if (so == nullptr) return fail(HB_ERR_INVALID_ARGUMENT, "split operator not prepared");
  if (op->precision == HB_PREC_FP32) {
#define HB_CASE(M, D, O)                                                              \
  if (op->model == M && dim == D && order == O)                                       \
    return launch_split_t<M, D, O, PT_FP16, float>(op, mode, ra, rb, dt, q_in, q_out,  \
                                                   res, coeff, bdry, source, e0, e1, s);
    HB_SPLIT_INSTANCES(HB_CASE)
#undef HB_CASE
    return fail(HB_ERR_UNSUPPORTED, "model/dimension/order combination not built");
  }
  if (so->stream) {
#define HB_CASE(M, D, O)                                                              \
  if (op->model == M && dim == D && order == O)                                       \
    return pt == PT_FP16                                                              \
               ? launch_stream_t<M, D, O, PT_FP16>(op, mode, ra, rb, dt, q_in, q_out, \
                                                   res, coeff, bdry, source, e0, e1, s) \
               : launch_stream_t<M, D, O, PT_BF16>(op, mode, ra, rb, dt, q_in, q_out, \
                                                   res, coeff, bdry, source, e0, e1, s);
    HB_SPLIT_STREAM_INSTANCES(HB_CASE)
#undef HB_CASE
  } else {
#define HB_CASE(M, D, O)                                                              \
  if (op->model == M && dim == D && order == O)                                       \
    return pt == PT_FP16                                                              \
               ? launch_split_t<M, D, O, PT_FP16>(op, mode, ra, rb, dt, q_in, q_out,  \
                                                  res, coeff, bdry, source, e0, e1, s) \
               : launch_split_t<M, D, O, PT_BF16>(op, mode, ra, rb, dt, q_in, q_out,  \
                                                  res, coeff, bdry, source, e0, e1, s);
    HB_SPLIT_INSTANCES(HB_CASE)
#undef HB_CASE
  }
  return fail(HB_ERR_UNSUPPORTED, "model/dimension/order combination not built");
}

void free_split(Op* op) {
  SplitOps* so = static_cast<SplitOps*>(op->split_ops);
  if (!so) return;
  cudaFree(so->dev);
  delete so;
  op->split_ops = nullptr;
}

}  // namespace hb
