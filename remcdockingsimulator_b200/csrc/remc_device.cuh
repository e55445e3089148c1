// Device building blocks of the B200 REMC engine: Philox stream, pair energy,
// bead packing, exact-rounding move arithmetic.
//
// Pair energy: the Kim-Hummer-style contact term + Debye-Hueckel term of
// Replica::E (simulation engine/src/Replica.cpp:603-745), with the crowder
// branch of Replica.cpp:637-690 (mode 0) or an eps_c ((rho_i+rho_j)/r)^12 wall
// (mode 1). Pair terms are FP32 with MUFU rsqrt/ex2; all per-type constants
// (4 eps, sigma^2, the repulsive-branch threshold, q_i q_j and the unit
// conversion factors) are folded into one float4 table entry per type pair.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/remc_b200.h"

namespace remc {

constexpr int kNT = REMC_MAX_TYPES;  // type-table edge
constexpr int kNumAmino = REMC_NUM_AMINO;

// ---------------------------------------------------------------- packing
// A bead is one float4 in HBM and shared memory: x, y, z and, in .w, the bits
// of (molecule index << 8 | type).
__host__ __device__ __forceinline__ int pack_meta(int mol, int type) { return (mol << 8) | type; }
__device__ __forceinline__ int bead_type(float w) { return __float_as_int(w) & 0xff; }
__device__ __forceinline__ int bead_mol(float w) { return __float_as_int(w) >> 8; }

// ---------------------------------------------------------------- Philox
// Philox4x32-10 (Salmon et al., SC'11): multipliers 0xD2511F53 / 0xCD9E8D57,
// key increments 0x9E3779B9 / 0xBB67AE85, ten rounds.
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r > 0) {
      k.x += 0x9E3779B9u;
      k.y += 0xBB67AE85u;
    }
    uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
    uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
  }
  return c;
}
__device__ __forceinline__ double u32_unit(uint32_t x) {
  return __dmul_rn((double)x, 2.3283064365386963e-10);  // 2^-32, exact
}

// ---------------------------------------------------------------- MUFU
__device__ __forceinline__ float fast_rsqrt(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float fast_rcp(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float fast_ex2(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// ---------------------------------------------------------------- bulk copies
// One-dimensional TMA bulk copy global -> shared memory completed on an
// mbarrier (no tensor map: the source is contiguous and 16-byte aligned, the
// size a multiple of 16 bytes), without cluster multicast.
__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes,
                                          unsigned long long* bar) {
  // order this CTA's earlier generic-proxy reads of dst before the async write
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
// Wait for the mbarrier phase with the given parity to complete, at most
// `limit` polls; returns false if it did not.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, int limit) {
  for (int i = 0; i < limit; ++i) {
    unsigned done;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; "
        "selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// ---------------------------------------------------------------- energy
struct EnergyConsts {
  float c_xi;        // -log2(e) / Xi: exp(-r/Xi) = ex2(r * c_xi)
  int crowder_mode;  // 0: A r^-6; 1: A r^-12
  int crowder_cut;   // 1: crowder pairs beyond the cutoff contribute nothing
};

// Minimum image d - L*rint(d/L) per axis (CudaFunctions.cu:430-442 uses
// rintf), on the FMA pipe: the FMA adds 1.5 * 2^23 to the exact product
// d * (1/L) and rounds once, which leaves rint of that product (ties to even)
// as the integer part of the sum for any |d/L| < 2^22; subtracting the
// constant is exact. Rounding the product first and then adding would round
// twice, and differ only where the product lies within half an ulp of a
// half-integer, where both images are half a box away.
__device__ __forceinline__ float min_image(float d, float L, float invL) {
  const float kMagic = 12582912.0f;  // 1.5 * 2^23
  const float n = __fsub_rn(__fmaf_rn(d, invL, kMagic), kMagic);
  return fmaf(-L, n, d);
}

// Energy (kcal/mol) of one pair of beads of different molecules at squared
// distance r2. T = table entry {4 eps', sigma^2, select threshold r^2, q q'}
// for residue pairs, {A, 0, cutoff^2, 0} for crowder pairs.
__device__ __forceinline__ float pair_energy_r2(float r2, float4 T, bool crowd,
                                                const EnergyConsts& K) {
  float rinv = fast_rsqrt(r2);
  float rinv2 = rinv * rinv;
  if (crowd) {
    float i6 = rinv2 * rinv2 * rinv2;
    float e = T.x * i6;
    if (K.crowder_mode) e *= i6;
    return (r2 < T.z) ? e : 0.0f;
  }
  float s2 = T.y * rinv2;
  float s6 = s2 * s2 * s2;
  float lj = T.x * fmaf(-s6, s6, s6);  // 4 eps' s6 (1 - s6) = -4 eps' s6 (s6 - 1)
  lj = (r2 < T.z) ? fmaf(0.5f, T.x, -lj) : lj;  // repulsive branch: 2 eps' - LJ
  float r = r2 * rinv;
  float dh = T.w * fast_ex2(r * K.c_xi) * rinv;
  return lj + dh;
}

// The crowder branch of pair_energy_r2 with the model fixed at compile time
// (R12: A r^-12, else A r^-6; CUT: zero at r^2 >= cut2). Same operations in
// the same order, so the same value.
template <bool R12, bool CUT>
__device__ __forceinline__ float crowd_energy(float r2, float A, float cut2) {
  float rinv2 = fast_rcp(r2);  // 1/r^2 in one MUFU operation
  float i6 = rinv2 * rinv2 * rinv2;
  float e = A * i6;
  if (R12) e *= i6;
  if (CUT) e = (r2 < cut2) ? e : 0.0f;
  return e;
}

__device__ __forceinline__ float pair_r2(float4 a, float4 b, float L, float invL) {
  float dx = min_image(a.x - b.x, L, invL);
  float dy = min_image(a.y - b.y, L, invL);
  float dz = min_image(a.z - b.z, L, invL);
  return fmaf(dx, dx, fmaf(dy, dy, dz * dz));
}

// The minimum image folded, scalar (fold_image2 below, one element): the
// image distance min(|d|, L - |d|) in magnitude, for |d| < 1.5 L.
__device__ __forceinline__ float fold_image(float d, float L) {
  const float a = fabsf(d);
  return fminf(a, __fsub_rn(L, a));
}
__device__ __forceinline__ float pair_r2_fold(float4 a, float4 b, float L) {
  float dx = fold_image(a.x - b.x, L);
  float dy = fold_image(a.y - b.y, L);
  float dz = fold_image(a.z - b.z, L);
  return fmaf(dx, dx, fmaf(dy, dy, dz * dz));
}
// pair_r2, folded where the caller knows every |d| < 1.5 L (FOLD)
template <bool FOLD>
__device__ __forceinline__ float pair_r2_f(float4 a, float4 b, float L, float invL) {
  if constexpr (FOLD)
    return pair_r2_fold(a, b, L);
  else
    return pair_r2(a, b, L, invL);
}

// ---------------------------------------------------------------- packed pairs
// Two pairs per lane in packed FP32 (f32x2: one instruction for both pairs,
// each element rounded as the scalar operation is). The displacement is taken
// as p_j - p_i, the exact negation of pair_r2's p_i - p_j; the minimum image
// is odd in d (rint rounds ties to even, which is symmetric), so the squared
// distance and the crowder energy equal pair_r2's and crowd_energy's.
struct PackedBox {
  float2 iL, nL, M, nM, L;  // 1/L, -L, +-1.5 * 2^23, L
};
__device__ __forceinline__ PackedBox packed_box(float L, float invL) {
  const float kMagic = 12582912.0f;  // 1.5 * 2^23, as in min_image
  return PackedBox{make_float2(invL, invL), make_float2(-L, -L), make_float2(kMagic, kMagic),
                   make_float2(-kMagic, -kMagic), make_float2(L, L)};
}
__device__ __forceinline__ float2 min_image2(float2 d, const PackedBox& B) {
  return __ffma2_rn(B.nL, __fadd2_rn(__ffma2_rn(d, B.iL, B.M), B.nM), d);
}
// The minimum image folded: for |d| < 1.5 L the nearer image is at distance
// min(|d|, L - |d|) in magnitude (negative past L, where the square is still
// right), one add on the FMA pipe and a min instead of three FMA-pipe
// operations. L - |d| is rounded once, as d -+ L is in min_image, so the
// result equals min_image's in magnitude except where d/L lies within a
// rounding of +-1/2, where both images are half a box away. Only for systems
// whose every bead pair is known to satisfy |d| < 1.5 L.
__device__ __forceinline__ float2 fold_image2(float2 d, const PackedBox& B) {
  const float2 a = make_float2(fabsf(d.x), fabsf(d.y));
  const float2 t = __fadd2_rn(B.L, make_float2(-a.x, -a.y));
  return make_float2(fminf(a.x, t.x), fminf(a.y, t.y));
}
// squared minimum-image distance from p_i (given negated, npx = (-x_i, -x_i)
// and so on) to two j beads; FOLD: fold_image2 (the caller knows |d| < 1.5 L)
template <bool FOLD = false>
__device__ __forceinline__ float2 pair_r2_2(float2 xj, float2 yj, float2 zj, float2 npx,
                                            float2 npy, float2 npz, const PackedBox& B) {
  float2 ex = __fadd2_rn(xj, npx), ey = __fadd2_rn(yj, npy), ez = __fadd2_rn(zj, npz);
  if constexpr (FOLD) {
    ex = fold_image2(ex, B);
    ey = fold_image2(ey, B);
    ez = fold_image2(ez, B);
  } else {
    ex = min_image2(ex, B);
    ey = min_image2(ey, B);
    ez = min_image2(ez, B);
  }
  return __ffma2_rn(ex, ex, __ffma2_rn(ey, ey, __fmul2_rn(ez, ez)));
}
template <bool R12, bool CUT>
__device__ __forceinline__ float2 crowd_energy2(float2 r2, float2 A, float2 cut2) {
  const float2 rinv2 = make_float2(fast_rcp(r2.x), fast_rcp(r2.y));
  const float2 i6 = __fmul2_rn(__fmul2_rn(rinv2, rinv2), rinv2);
  float2 e = __fmul2_rn(A, i6);
  if (R12) e = __fmul2_rn(e, i6);
  if (CUT) {
    e.x = (r2.x < cut2.x) ? e.x : 0.0f;
    e.y = (r2.y < cut2.y) ? e.y : 0.0f;
  }
  return e;
}

// Kim-Hummer + Debye-Hueckel energy of two residue pairs that share the table
// entry T (the moved bead's new and old position against one bead j), in
// packed FP32: pair_energy_r2's operations for a residue pair, each product
// and sum rounded on its own.
__device__ __forceinline__ float2 kh_energy2(float2 r2, float4 T, float c_xi) {
  const float2 rinv = make_float2(fast_rsqrt(r2.x), fast_rsqrt(r2.y));
  const float2 rinv2 = __fmul2_rn(rinv, rinv);
  const float2 s2 = __fmul2_rn(make_float2(T.y, T.y), rinv2);
  const float2 s6 = __fmul2_rn(__fmul2_rn(s2, s2), s2);
  const float2 g = __ffma2_rn(make_float2(-s6.x, -s6.y), s6, s6);  // s6 (1 - s6)
  float2 lj = __fmul2_rn(make_float2(T.x, T.x), g);
  const float2 ljr =
      __ffma2_rn(make_float2(0.5f, 0.5f), make_float2(T.x, T.x), make_float2(-lj.x, -lj.y));
  lj.x = (r2.x < T.z) ? ljr.x : lj.x;  // repulsive branch: 2 eps' - LJ
  lj.y = (r2.y < T.z) ? ljr.y : lj.y;
  const float2 r = __fmul2_rn(r2, rinv);
  const float2 arg = __fmul2_rn(r, make_float2(c_xi, c_xi));
  const float2 ex = make_float2(fast_ex2(arg.x), fast_ex2(arg.y));
  const float2 dh = __fmul2_rn(__fmul2_rn(make_float2(T.w, T.w), ex), rinv);
  return __fadd2_rn(lj, dh);
}

// ---------------------------------------------------------------- moves
// Exact-rounding (no FMA contraction) restatement of the reference's rigid-move
// arithmetic so device trajectories round exactly like the host engine's:
// Replica::createNormalisedRandomVector{,d} (Replica.cpp:303-318),
// Replica::translate (:333-364), Molecule::rotateQ (Molecule.cpp:288-333),
// Quaternion::rotateVector (Quaternion.cpp:84-101), Quaternion::multiply
// (Quaternion.cpp:36-48).
struct QuatProducts {
  double a, b, c;  // row-0 terms: (w2+x2-y2-z2), (xy-wz), (wy+xz)
  double d, e, f;  // row-1 terms: (wz+xy), (yz-wx), (w2-x2+y2-z2)
  double g, h, i;  // row-2 terms: (xz-wy), (yz+wx), (w2-x2-y2+z2)
};

__device__ __forceinline__ QuatProducts quat_products(double w, double x, double y, double z) {
  double w2 = __dmul_rn(w, w), x2 = __dmul_rn(x, x), y2 = __dmul_rn(y, y), z2 = __dmul_rn(z, z);
  double wx = __dmul_rn(w, x), wy = __dmul_rn(w, y), wz = __dmul_rn(w, z);
  double xy = __dmul_rn(x, y), xz = __dmul_rn(x, z), yz = __dmul_rn(y, z);
  QuatProducts p;
  p.a = __dsub_rn(__dsub_rn(__dadd_rn(w2, x2), y2), z2);
  p.b = __dsub_rn(xy, wz);
  p.c = __dadd_rn(wy, xz);
  p.d = __dadd_rn(wz, xy);
  p.e = __dsub_rn(yz, wx);
  p.f = __dsub_rn(__dadd_rn(__dsub_rn(w2, x2), y2), z2);
  p.g = __dsub_rn(xz, wy);
  p.h = __dadd_rn(yz, wx);
  p.i = __dadd_rn(__dsub_rn(__dsub_rn(w2, x2), y2), z2);
  return p;
}

// rel' = q.rotateVector(rel), rounded to float as the reference's Vector3f
// constructor does.
__device__ __forceinline__ float3 rotate_rel(const QuatProducts& p, float rx, float ry, float rz) {
  double vx = rx, vy = ry, vz = rz;
  double X = __dadd_rn(__dmul_rn(vx, p.a),
                       __dmul_rn(__dadd_rn(__dmul_rn(vy, p.b), __dmul_rn(vz, p.c)), 2.0));
  double Y = __dadd_rn(__dmul_rn(__dadd_rn(__dmul_rn(vx, p.d), __dmul_rn(vz, p.e)), 2.0),
                       __dmul_rn(vy, p.f));
  double Z = __dadd_rn(__dmul_rn(__dadd_rn(__dmul_rn(vx, p.g), __dmul_rn(vy, p.h)), 2.0),
                       __dmul_rn(vz, p.i));
  return make_float3(__double2float_rn(X), __double2float_rn(Y), __double2float_rn(Z));
}

// q * r (Quaternion::multiply), exact rounding, left-to-right sums.
__device__ __forceinline__ void quat_mul(double qw, double qx, double qy, double qz, double rw,
                                         double rx, double ry, double rz, double out[4]) {
  out[0] = __dsub_rn(__dsub_rn(__dsub_rn(__dmul_rn(qw, rw), __dmul_rn(qx, rx)), __dmul_rn(qy, ry)),
                     __dmul_rn(qz, rz));
  out[1] = __dsub_rn(__dadd_rn(__dadd_rn(__dmul_rn(qw, rx), __dmul_rn(qx, rw)), __dmul_rn(qy, rz)),
                     __dmul_rn(qz, ry));
  out[2] = __dadd_rn(__dadd_rn(__dsub_rn(__dmul_rn(qw, ry), __dmul_rn(qx, rz)), __dmul_rn(qy, rw)),
                     __dmul_rn(qz, rx));
  out[3] = __dadd_rn(__dsub_rn(__dadd_rn(__dmul_rn(qw, rz), __dmul_rn(qx, ry)), __dmul_rn(qy, rx)),
                     __dmul_rn(qz, rw));
}

// fmod(x, L) for the wrapped centre of Replica::translate (Replica.cpp:359-361).
// For x in [0, 3L) the result is x, x - L or x - 2L, and each subtraction is
// exact (Sterbenz: y/2 <= x <= 2y), so this equals fmodf bit for bit; other
// inputs (centres placed outside the box) take fmodf itself.
__device__ __forceinline__ float wrap_box(float x, float L) {
  if (x >= 0.0f) {
    if (x < L) return x;
    const float L2 = 2.0f * L;  // exact
    if (x < L2) return __fsub_rn(x, L);
    if (x <= 2.0f * L2) {
      const float d = __fsub_rn(x, L2);  // exact for L2/2 <= x <= 2 L2
      if (d < L) return d;
    }
  }
  return fmodf(x, L);
}

// Translation vector: translate_step * normalise(u2-.5, .5-u3, u4-.5) in FP32.
__device__ __forceinline__ float3 translate_vector(double u2, double u3, double u4, float step) {
  float vx = __double2float_rn(__dsub_rn(u2, 0.5));
  float vy = __double2float_rn(__dsub_rn(0.5, u3));
  float vz = __double2float_rn(__dsub_rn(u4, 0.5));
  float mag = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(vx, vx), __fmul_rn(vy, vy)),
                                   __fmul_rn(vz, vz)));
  if (mag != 0.0f) {
    vx = __fdiv_rn(vx, mag);
    vy = __fdiv_rn(vy, mag);
    vz = __fdiv_rn(vz, mag);
  }
  return make_float3(__fmul_rn(vx, step), __fmul_rn(vy, step), __fmul_rn(vz, step));
}

// Step quaternion for a rotation by a fixed angle about the random axis
// normalise(u2-.5, .5-u3, u4-.5); cos/sin of the half angle come from the
// host (they are per-replica constants).
__device__ __forceinline__ void step_quaternion(double u2, double u3, double u4, double cosa,
                                                double sina, double q[4]) {
  double ax = __dsub_rn(u2, 0.5), ay = __dsub_rn(0.5, u3), az = __dsub_rn(u4, 0.5);
  double am = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(ax, ax), __dmul_rn(ay, ay)),
                                   __dmul_rn(az, az)));
  ax = __ddiv_rn(ax, am);
  ay = __ddiv_rn(ay, am);
  az = __ddiv_rn(az, am);
  double qw = cosa, qx = __dmul_rn(sina, ax), qy = __dmul_rn(sina, ay), qz = __dmul_rn(sina, az);
  double qm = __dsqrt_rn(__dadd_rn(
      __dadd_rn(__dadd_rn(__dmul_rn(qw, qw), __dmul_rn(qx, qx)), __dmul_rn(qy, qy)),
      __dmul_rn(qz, qz)));
  q[0] = __ddiv_rn(qw, qm);
  q[1] = __ddiv_rn(qx, qm);
  q[2] = __ddiv_rn(qy, qm);
  q[3] = __ddiv_rn(qz, qm);
}

// ---------------------------------------------------------------- reductions
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  return v;
}

}  // namespace remc
