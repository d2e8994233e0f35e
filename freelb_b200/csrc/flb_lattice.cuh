// flb_lattice.cuh -- D3Q19 constants, population storage forms and the
// per-cell collision operators of the stream-and-collide path.
//
// Everything here is device code compiled for sm_100a.  The arithmetic of each
// operator follows the reference policy it replaces (cited per function) so the
// FP32 results stay within rounding of the reference's CPU path.
#pragma once

#include <cstdint>
#include <cuda_fp16.h>
#include <type_traits>

namespace flb {

constexpr int Q = 19;

// D3Q19 velocities in the reference ordering (src/lbm/lattice_set.h:263-266):
// rest, 6 axis directions, 12 diagonals; opposite of odd i is i+1.
__host__ __device__ constexpr int cx(int i) {
  constexpr int v[Q] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0};
  return v[i];
}
__host__ __device__ constexpr int cy(int i) {
  constexpr int v[Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1};
  return v[i];
}
__host__ __device__ constexpr int cz(int i) {
  constexpr int v[Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1};
  return v[i];
}
__host__ __device__ constexpr int opp(int i) { return i == 0 ? 0 : ((i & 1) ? i + 1 : i - 1); }

// Weights as the reference evaluates its Fraction<> table: T(num)/T(den).
template <typename R>
__host__ __device__ constexpr R weight(int i) {
  return i == 0 ? R(1) / R(3) : (i < 7 ? R(1) / R(18) : R(1) / R(36));
}

// ---------------------------------------------------------------------------
// D3Q19 Gram-Schmidt moment basis (d'Humieres, Ginzburg, Krafczyk, Lallemand,
// Luo, Phil. Trans. R. Soc. A 360 (2002)), rows in the paper's order
// (rho, e, eps, jx, qx, jy, qy, jz, qz, 3pxx, 3pixx, pww, piww, pxy, pyz, pxz,
// mx, my, mz), evaluated on the reference velocity ordering.  The reference
// provides the generic algorithm (src/lbm/collisionMRT.h:132-190) but no D3Q19
// matrix.
__host__ __device__ constexpr int mrt_m(int k, int i) {
  const int x = cx(i), y = cy(i), z = cz(i);
  const int c2 = x * x + y * y + z * z;
  return k == 0    ? 1
         : k == 1  ? 19 * c2 - 30
         : k == 2  ? (21 * c2 * c2 - 53 * c2 + 24) / 2
         : k == 3  ? x
         : k == 4  ? (5 * c2 - 9) * x
         : k == 5  ? y
         : k == 6  ? (5 * c2 - 9) * y
         : k == 7  ? z
         : k == 8  ? (5 * c2 - 9) * z
         : k == 9  ? 3 * x * x - c2
         : k == 10 ? (3 * c2 - 5) * (3 * x * x - c2)
         : k == 11 ? y * y - z * z
         : k == 12 ? (3 * c2 - 5) * (y * y - z * z)
         : k == 13 ? x * y
         : k == 14 ? y * z
         : k == 15 ? x * z
         : k == 16 ? x * (y * y - z * z)
         : k == 17 ? y * (z * z - x * x)
                   : z * (x * x - y * y);
}
__host__ __device__ constexpr int mrt_norm(int k) {
  int s = 0;
  for (int i = 0; i < Q; ++i) s += mrt_m(k, i) * mrt_m(k, i);
  return s;
}
// |M_k|^2 as literals: device code with a run-time k reads no table (a loop
// over the velocity tables would put them on the stack).
__host__ __device__ constexpr int mrt_norm_lit(int k) {
  return k == 0 ? 19 : k == 1 ? 2394 : k == 2 ? 252 : k == 4 || k == 6 || k == 8 ? 40
       : k == 9 ? 36 : k == 10 ? 72 : k == 11 ? 12 : k == 12 ? 24
       : k >= 13 && k <= 15 ? 4 : k >= 16 ? 8 : 10;
}
static_assert(mrt_norm_lit(0) == mrt_norm(0) && mrt_norm_lit(1) == mrt_norm(1) &&
                  mrt_norm_lit(2) == mrt_norm(2) && mrt_norm_lit(3) == mrt_norm(3) &&
                  mrt_norm_lit(4) == mrt_norm(4) && mrt_norm_lit(5) == mrt_norm(5) &&
                  mrt_norm_lit(6) == mrt_norm(6) && mrt_norm_lit(7) == mrt_norm(7) &&
                  mrt_norm_lit(8) == mrt_norm(8) && mrt_norm_lit(9) == mrt_norm(9) &&
                  mrt_norm_lit(10) == mrt_norm(10) && mrt_norm_lit(11) == mrt_norm(11) &&
                  mrt_norm_lit(12) == mrt_norm(12) && mrt_norm_lit(13) == mrt_norm(13) &&
                  mrt_norm_lit(14) == mrt_norm(14) && mrt_norm_lit(15) == mrt_norm(15) &&
                  mrt_norm_lit(16) == mrt_norm(16) && mrt_norm_lit(17) == mrt_norm(17) &&
                  mrt_norm_lit(18) == mrt_norm(18),
              "MRT row norms");
// Moments that are even under c -> -c (depend on f_i + f_opp(i) only).
__host__ __device__ constexpr bool mrt_even(int k) {
  return k == 0 || k == 1 || k == 2 || (k >= 9 && k <= 15);
}
__host__ __device__ constexpr bool mrt_conserved(int k) {
  return k == 0 || k == 3 || k == 5 || k == 7;
}
__host__ __device__ constexpr bool mrt_shear(int k) {
  return k == 9 || k == 11 || k == 13 || k == 14 || k == 15;
}

// ---------------------------------------------------------------------------
// Storage forms.  Load converts a stored population to the arithmetic type R,
// store converts back.  FP16S keeps (f_i - rho0*w_i) * scale in binary16
// (round to nearest even); scale is a power of two so the shift/scale are exact.
template <typename S, typename R>
struct Storage;

template <>
struct Storage<float, float> {
  __device__ static __forceinline__ float load(const float* p, float, float) { return *p; }
  __device__ static __forceinline__ void store(float* p, float v, float, float) { *p = v; }
};

template <>
struct Storage<double, double> {
  __device__ static __forceinline__ double load(const double* p, double, double) { return *p; }
  __device__ static __forceinline__ void store(double* p, double v, double, double) { *p = v; }
};

template <>
struct Storage<__half, float> {
  __device__ static __forceinline__ float load(const __half* p, float shift, float inv_scale) {
    return fmaf(__half2float(*p), inv_scale, shift);
  }
  // scale is a power of two, so (v - shift) * scale == v * scale - shift * scale
  // exactly before the single rounding of the fused multiply-add.
  __device__ static __forceinline__ void store(__half* p, float v, float shift, float scale) {
    *p = __float2half_rn(fmaf(v, scale, -shift * scale));
  }
};

// FP32S storage element: d_i = f_i - rho0 w_i held as a float.  A type of its
// own, so that every kernel templated on the storage knows the stored values
// are deviations: the step and adjoint kernels work on them directly (a
// deviation of size ~1e-3 keeps ~5e-11 of absolute resolution, where f_i ~ 0.1
// in a float keeps ~7e-9), while these load / store forms convert to and from
// f_i for the readers and writers of populations.
struct dev32 {
  float v;
};
static_assert(sizeof(dev32) == 4, "FP32S element is one float");

template <>
struct Storage<dev32, float> {
  __device__ static __forceinline__ float load(const dev32* p, float shift, float) {
    return p->v + shift;
  }
  __device__ static __forceinline__ void store(dev32* p, float v, float shift, float) {
    p->v = v - shift;
  }
};

// ---------------------------------------------------------------------------
// Per-cell operators.  f[] holds the 19 populations of one cell in registers.

// moment::rhoUImpl<D3Q19> (src/lbm/moment.ur.h:505-517)
template <typename R>
__device__ __forceinline__ void rho_u(const R* f, R& rho, R& ux, R& uy, R& uz) {
  rho = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8] + f[9] + f[10] + f[11] +
        f[12] + f[13] + f[14] + f[15] + f[16] + f[17] + f[18];
  ux = (f[1] - f[2] + f[7] - f[8] + f[9] - f[10] + f[13] - f[14] + f[15] - f[16]) / rho;
  uy = (f[3] - f[4] + f[7] - f[8] + f[11] - f[12] - f[13] + f[14] + f[17] - f[18]) / rho;
  uz = (f[5] - f[6] + f[9] - f[10] + f[11] - f[12] - f[15] + f[16] - f[17] + f[18]) / rho;
}

// rho_u with u = m * (1 / rho) through the hardware reciprocal (FP32 only).
__device__ __forceinline__ void rho_u_fast(const float* f, float& rho, float& ux, float& uy,
                                           float& uz) {
  rho = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8] + f[9] + f[10] + f[11] +
        f[12] + f[13] + f[14] + f[15] + f[16] + f[17] + f[18];
  const float ir = __fdividef(1.0f, rho);
  ux = (f[1] - f[2] + f[7] - f[8] + f[9] - f[10] + f[13] - f[14] + f[15] - f[16]) * ir;
  uy = (f[3] - f[4] + f[7] - f[8] + f[11] - f[12] - f[13] + f[14] + f[17] - f[18]) * ir;
  uz = (f[5] - f[6] + f[9] - f[10] + f[11] - f[12] - f[15] + f[16] - f[17] + f[18]) * ir;
}

// equilibrium::SecondOrderImpl<D3Q19> (src/lbm/equilibrium.ur.h:166-215)
template <typename R>
__device__ __forceinline__ void feq2(R* feq, R rho, R ux, R uy, R uz) {
  const R InvCs2 = R(3);
  const R var0 = R(1) - (ux * ux + uy * uy + uz * uz) * (R(0.5) * InvCs2);
  const R rw0 = weight<R>(0) * rho;
  const R rw1 = weight<R>(1) * rho;
  const R rw7 = weight<R>(7) * rho;
  const R k1 = InvCs2 * ux, v1 = var0 + k1 * k1 * R(0.5);
  const R k3 = InvCs2 * uy, v3 = var0 + k3 * k3 * R(0.5);
  const R k5 = InvCs2 * uz, v5 = var0 + k5 * k5 * R(0.5);
  const R k7 = InvCs2 * (ux + uy), v7 = var0 + k7 * k7 * R(0.5);
  const R k9 = InvCs2 * (ux + uz), v9 = var0 + k9 * k9 * R(0.5);
  const R k11 = InvCs2 * (uy + uz), v11 = var0 + k11 * k11 * R(0.5);
  const R k13 = InvCs2 * (ux - uy), v13 = var0 + k13 * k13 * R(0.5);
  const R k15 = InvCs2 * (ux - uz), v15 = var0 + k15 * k15 * R(0.5);
  const R k17 = InvCs2 * (uy - uz), v17 = var0 + k17 * k17 * R(0.5);
  feq[0] = rw0 * var0;
  feq[1] = rw1 * (v1 + k1);
  feq[2] = rw1 * (v1 - k1);
  feq[3] = rw1 * (v3 + k3);
  feq[4] = rw1 * (v3 - k3);
  feq[5] = rw1 * (v5 + k5);
  feq[6] = rw1 * (v5 - k5);
  feq[7] = rw7 * (v7 + k7);
  feq[8] = rw7 * (v7 - k7);
  feq[9] = rw7 * (v9 + k9);
  feq[10] = rw7 * (v9 - k9);
  feq[11] = rw7 * (v11 + k11);
  feq[12] = rw7 * (v11 - k11);
  feq[13] = rw7 * (v13 + k13);
  feq[14] = rw7 * (v13 - k13);
  feq[15] = rw7 * (v15 + k15);
  feq[16] = rw7 * (v15 - k15);
  feq[17] = rw7 * (v17 + k17);
  feq[18] = rw7 * (v17 - k17);
}

// collision::BGK (src/lbm/collision.h:40-57): f <- omega*feq + (1-omega)*f
template <typename R>
__device__ __forceinline__ void bgk(R* f, R omega, R omega_c) {
  R rho, ux, uy, uz, feq[Q];
  rho_u(f, rho, ux, uy, uz);
  feq2(feq, rho, ux, uy, uz);
#pragma unroll
  for (int i = 0; i < Q; ++i) f[i] = omega * feq[i] + omega_c * f[i];
}

// Brinkman drag F = -alpha u through the reference's Guo forcing:
// moment::forcerhoU (src/lbm/moment.h:402-422) gives u = (sum c f + F/2)/rho,
// which with F = -alpha u is u = sum c f / (rho + alpha/2); force::ForcePopImpl
// (src/lbm/force.h:29-36) gives F_i = w_i F.(3 (c_i - u) + 9 (c_i.u) c_i);
// collision::BGKForce (src/lbm/collision.h:61-90) relaxes
// f <- omega feq + (1-omega) f + (1 - omega/2) F_i.
template <typename R>
__device__ __forceinline__ void bgk_brinkman(R* f, R omega, R alpha) {
  const R rho = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8] + f[9] + f[10] +
                f[11] + f[12] + f[13] + f[14] + f[15] + f[16] + f[17] + f[18];
  const R mx = f[1] - f[2] + f[7] - f[8] + f[9] - f[10] + f[13] - f[14] + f[15] - f[16];
  const R my = f[3] - f[4] + f[7] - f[8] + f[11] - f[12] - f[13] + f[14] + f[17] - f[18];
  const R mz = f[5] - f[6] + f[9] - f[10] + f[11] - f[12] - f[15] + f[16] - f[17] + f[18];
  const R den = rho + R(0.5) * alpha;
  const R ux = mx / den, uy = my / den, uz = mz / den;
  const R Fx = -alpha * ux, Fy = -alpha * uy, Fz = -alpha * uz;
  R feq[Q];
  feq2(feq, rho, ux, uy, uz);
  const R fomega = R(1) - R(0.5) * omega;
  const R omega_c = R(1) - omega;
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const R cu = R(cx(i)) * ux + R(cy(i)) * uy + R(cz(i)) * uz;
    const R vx = (R(cx(i)) - ux) * R(3) + cu * R(9) * R(cx(i));
    const R vy = (R(cy(i)) - uy) * R(3) + cu * R(9) * R(cy(i));
    const R vz = (R(cz(i)) - uz) * R(3) + cu * R(9) * R(cz(i));
    const R Fi = weight<R>(i) * (Fx * vx + Fy * vy + Fz * vz);
    f[i] = omega * feq[i] + omega_c * f[i] + fomega * Fi;
  }
}

// Forced moments of a Brinkman cell: rho = sum f, u = sum c f / (rho + alpha/2)
// (moment::forcerhoU with F = -alpha u, src/lbm/moment.h:402-422).
template <typename R>
__device__ __forceinline__ void forced_moments(const R* f, R alpha, R& rho, R& den, R& ux, R& uy,
                                               R& uz) {
  rho = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8] + f[9] + f[10] + f[11] +
        f[12] + f[13] + f[14] + f[15] + f[16] + f[17] + f[18];
  const R mx = f[1] - f[2] + f[7] - f[8] + f[9] - f[10] + f[13] - f[14] + f[15] - f[16];
  const R my = f[3] - f[4] + f[7] - f[8] + f[11] - f[12] - f[13] + f[14] + f[17] - f[18];
  const R mz = f[5] - f[6] + f[9] - f[10] + f[11] - f[12] - f[15] + f[16] - f[17] + f[18];
  den = rho + R(0.5) * alpha;
  ux = mx / den;
  uy = my / den;
  uz = mz / den;
}

// collision::BGK<moment::useFieldrhoU, ...>: rho, u from the fields.
template <typename R>
__device__ __forceinline__ void bgk_field(R* f, R omega, R omega_c, R rho, R ux, R uy, R uz) {
  R feq[Q];
  feq2(feq, rho, ux, uy, uz);
#pragma unroll
  for (int i = 0; i < Q; ++i) f[i] = omega * feq[i] + omega_c * f[i];
}

// collision::BounceBack<D3Q19> (src/lbm/collision.ur.h:62-93): swap i, i+1.
template <typename R>
__device__ __forceinline__ void bounce_back(R* f) {
#pragma unroll
  for (int i = 1; i < Q; i += 2) {
    const R t = f[i];
    f[i] = f[i + 1];
    f[i + 1] = t;
  }
}

// collision::BounceBackMovingWall<D3Q19> (src/lbm/collision.ur.h:130-187):
// f_i <- f_opp + 6 w_i rho_w (u_w.c_i), f_opp <- f_i - same, i odd.
template <typename R>
__device__ __forceinline__ void moving_wall(R* f, R rho_w, R ux, R uy, R uz) {
  const R rhox = R(6) * rho_w;
#pragma unroll
  for (int i = 1; i < Q; i += 2) {
    R uc;
    const int a = cx(i), b = cy(i), c = cz(i);
    // u.c_i evaluated in the reference's term order (u0 +/- u1 etc.)
    if (b == 0 && c == 0) uc = ux;
    else if (a == 0 && c == 0) uc = uy;
    else if (a == 0 && b == 0) uc = uz;
    else if (c == 0) uc = (b > 0) ? ux + uy : ux - uy;
    else if (b == 0) uc = (c > 0) ? ux + uz : ux - uz;
    else uc = (c > 0) ? uy + uz : uy - uz;
    uc = uc * weight<R>(i) * rhox;
    const R t = f[i];
    f[i] = f[i + 1] + uc;
    f[i + 1] = t - uc;
  }
}

// collision::SmagorinskyBGK (src/lbm/collisionLES.h:36-62) with
// moment::Pi_ab_neq<D3Q19> (src/lbm/moment.ur.h:751-762).  The momenta scheme
// writes RHO, so the density in the eddy-viscosity coefficient is this cell's
// current rho.  cs_coeff = Cs^2 * 9 * 2 * sqrt(2) is precomputed on the host in
// double, as the reference evaluates that product in double.
template <typename R>
__device__ __forceinline__ void smagorinsky_bgk(R* f, R rt_mol, R cs_coeff) {
  R rho, ux, uy, uz, feq[Q];
  rho_u(f, rho, ux, uy, uz);
  const R cs2 = R(1) / R(3);
  const R p0 = f[1] + f[2] + f[7] + f[8] + f[9] + f[10] + f[13] + f[14] + f[15] + f[16] -
               rho * (ux * ux + cs2);
  const R p1 = f[7] + f[8] - f[13] - f[14] - rho * (ux * uy);
  const R p2 = f[9] + f[10] - f[15] - f[16] - rho * (ux * uz);
  const R p3 = f[3] + f[4] + f[7] + f[8] + f[11] + f[12] + f[13] + f[14] + f[17] + f[18] -
               rho * (uy * uy + cs2);
  const R p4 = f[11] + f[12] - f[17] - f[18] - rho * (uy * uz);
  const R p5 = f[5] + f[6] + f[9] + f[10] + f[11] + f[12] + f[15] + f[16] + f[17] + f[18] -
               rho * (uz * uz + cs2);
  const R nsq = p0 * p0 + p1 * p1 * R(2) + p2 * p2 * R(2) + p3 * p3 + p4 * p4 * R(2) + p5 * p5;
  R eomega;
  if constexpr (std::is_same<R, float>::value) {
    // FP32: the hardware square-root and reciprocal approximations (about one
    // ulp, far inside the 1e-5 parity with the reference's FP32 run) instead
    // of the IEEE sequences with their slow paths; FP64 keeps IEEE (the
    // oracle is matched to 1e-12 there)
    const float norm = nsq > 0.0f ? nsq * rsqrtf(nsq) : 0.0f;
    const float coeff = cs_coeff * __fdividef(1.0f, rho);
    const float t = rt_mol * rt_mol + coeff * norm;
    const float rt_tur = 0.5f * (t * rsqrtf(t) - rt_mol);
    eomega = __fdividef(1.0f, rt_mol + rt_tur);
  } else {
    const R norm = sqrt(nsq);
    const R coeff = cs_coeff / rho;
    const R rt_tur = R(0.5) * (sqrt(rt_mol * rt_mol + coeff * norm) - rt_mol);
    eomega = R(1) / (rt_mol + rt_tur);
  }
  const R eomega_c = R(1) - eomega;
  feq2(feq, rho, ux, uy, uz);
#pragma unroll
  for (int i = 0; i < Q; ++i) f[i] = eomega * feq[i] + eomega_c * f[i];
}

// collision::MRT_Feq_RhoU (src/lbm/collisionMRT.h:142-188):
//   f <- f - M^-1 S (M f - M feq),  M^-1[i][k] = M[k][i] / |M_k|^2.
// Evaluated on f - feq with the basis split into moments even and odd under
// c -> -c, so even moments see only f_i + f_opp and odd ones only f_i - f_opp;
// all basis entries are compile-time constants (zeros and unit factors fold).
// s[k] already holds the per-moment rate divided by |M_k|^2.
// Moment k of x given as r0 = x_0, a_p = x_{2p+1} + x_{2p+2}, b_p = x_{2p+1} -
// x_{2p+2}: even moments see only a, odd ones only b.
template <typename R>
__device__ __forceinline__ R mrt_moment(int k, R r0, const R (&a)[9], const R (&b)[9]) {
  R m = R(0);
  if (mrt_even(k)) {
    if (mrt_m(k, 0) != 0) m = R(mrt_m(k, 0)) * r0;
#pragma unroll
    for (int p = 0; p < 9; ++p) {
      const int c = mrt_m(k, 2 * p + 1);
      if (c == 1) m += a[p];
      else if (c == -1) m -= a[p];
      else if (c != 0) m += R(c) * a[p];
    }
  } else {
#pragma unroll
    for (int p = 0; p < 9; ++p) {
      const int c = mrt_m(k, 2 * p + 1);
      if (c == 1) m += b[p];
      else if (c == -1) m -= b[p];
      else if (c != 0) m += R(c) * b[p];
    }
  }
  return m;
}

// The moment-space relaxation of the non-equilibrium part: r0 = n_0,
// a_p = n_{2p+1} + n_{2p+2}, b_p = n_{2p+1} - n_{2p+2}; x_i -= sum_k M[k][i] mu_k.
template <typename R>
__device__ __forceinline__ void mrt_relax(R* f, R r0, const R (&a)[9], const R (&b)[9],
                                          const R* s_over_norm) {
  R mu[Q];
#pragma unroll
  for (int k = 0; k < Q; ++k) {
    if (mrt_conserved(k)) {
      mu[k] = R(0);
      continue;
    }
    R m = R(0);
    if (mrt_even(k)) {
      if (mrt_m(k, 0) != 0) m = R(mrt_m(k, 0)) * r0;
#pragma unroll
      for (int p = 0; p < 9; ++p) {
        const int c = mrt_m(k, 2 * p + 1);
        if (c == 1) m += a[p];
        else if (c == -1) m -= a[p];
        else if (c != 0) m += R(c) * a[p];
      }
    } else {
#pragma unroll
      for (int p = 0; p < 9; ++p) {
        const int c = mrt_m(k, 2 * p + 1);
        if (c == 1) m += b[p];
        else if (c == -1) m -= b[p];
        else if (c != 0) m += R(c) * b[p];
      }
    }
    mu[k] = m * s_over_norm[k];
  }
  // back-transform: delta f_i = sum_k M[k][i] mu_k
  R d0 = R(0);
#pragma unroll
  for (int k = 0; k < Q; ++k)
    if (mrt_even(k) && !mrt_conserved(k) && mrt_m(k, 0) != 0) d0 += R(mrt_m(k, 0)) * mu[k];
  f[0] -= d0;
#pragma unroll
  for (int p = 0; p < 9; ++p) {
    R e = R(0), o = R(0);
#pragma unroll
    for (int k = 0; k < Q; ++k) {
      if (mrt_conserved(k)) continue;
      const int c = mrt_m(k, 2 * p + 1);
      if (c == 0) continue;
      if (mrt_even(k)) e += R(c) * mu[k];
      else o += R(c) * mu[k];
    }
    f[2 * p + 1] -= e + o;
    f[2 * p + 2] -= e - o;
  }
}

// Two-rate MRT: every non-conserved moment outside the five (even) shear
// moments relaxes at sg, so M^-1 S M n = sg (n - C n) + (omega - sg) P n with
// n = f - feq, C the projection on the conserved moments (rho, j) and P the
// projection on the shear moments, which the pair sums of n give (both members
// of a pair get the same correction).  C n is zero in exact arithmetic, but in
// floating point it carries the rounding of f - feq, which is relative to f,
// not to n: relaxing it too (as plain BGK does) leaks mass and momentum and
// took the 512^3 FP32 cavity from 2.6e-5 to 1.7e-4 against FP64, so it is
// taken out, as the general form (which never touches conserved moments)
// does.  The same operator as mrt() for such rate sets, with 9 moment sums
// instead of 15.
template <typename R>
__device__ __forceinline__ void mrt_two_rate(R* f, R omega, R sg) {
  constexpr int SH[5] = {9, 11, 13, 14, 15};
  R rho, ux, uy, uz, feq[Q];
  if constexpr (std::is_same<R, float>::value) {
    // one hardware reciprocal instead of three IEEE divisions: a velocity off
    // by an ulp only moves feq, whose conserved moments the projection below
    // removes anyway
    rho_u_fast(f, rho, ux, uy, uz);
  } else {
    rho_u(f, rho, ux, uy, uz);
  }
  feq2(feq, rho, ux, uy, uz);
  R m[5];
#pragma unroll
  for (int j = 0; j < 5; ++j) m[j] = R(0);
  const R n0 = f[0] - feq[0];
  R mr = n0, jx = R(0), jy = R(0), jz = R(0);  // conserved moments of n
#pragma unroll
  for (int i = 1; i < Q; i += 2) {
    const R n1 = f[i] - feq[i], n2 = f[i + 1] - feq[i + 1];
    const R a = n1 + n2, b = n1 - n2;
    mr += a;
    if (cx(i) == 1) jx += b; else if (cx(i) == -1) jx -= b;
    if (cy(i) == 1) jy += b; else if (cy(i) == -1) jy -= b;
    if (cz(i) == 1) jz += b; else if (cz(i) == -1) jz -= b;
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      const int c = mrt_m(SH[j], i);
      if (c == 1) m[j] += a;
      else if (c == -1) m[j] -= a;
      else if (c != 0) m[j] += R(c) * a;
    }
  }
#pragma unroll
  for (int j = 0; j < 5; ++j) m[j] *= (omega - sg) * (R(1) / R(mrt_norm_lit(SH[j])));
  // C n_i = mr / 19 + c_i . j / 10  (|M_rho|^2 = 19, |M_j|^2 = 10)
  const R r = mr * (R(1) / R(19));
  jx *= R(1) / R(10);
  jy *= R(1) / R(10);
  jz *= R(1) / R(10);
  f[0] -= sg * (n0 - r);
#pragma unroll
  for (int i = 1; i < Q; i += 2) {
    R corr = R(0);
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      const int c = mrt_m(SH[j], i);
      if (c == 1) corr += m[j];
      else if (c == -1) corr -= m[j];
      else if (c != 0) corr += R(c) * m[j];
    }
    R kj = R(0);
    if (cx(i) == 1) kj += jx; else if (cx(i) == -1) kj -= jx;
    if (cy(i) == 1) kj += jy; else if (cy(i) == -1) kj -= jy;
    if (cz(i) == 1) kj += jz; else if (cz(i) == -1) kj -= jz;
    f[i] -= sg * ((f[i] - feq[i]) - r - kj) + corr;
    f[i + 1] -= sg * ((f[i + 1] - feq[i + 1]) - r + kj) + corr;
  }
}

template <typename R>
__device__ __forceinline__ void mrt(R* f, const R* s_over_norm) {
  R rho, ux, uy, uz, feq[Q];
  rho_u(f, rho, ux, uy, uz);
  feq2(feq, rho, ux, uy, uz);
  R a[9], b[9];  // symmetric / antisymmetric non-equilibrium parts per pair
  const R r0 = f[0] - feq[0];
#pragma unroll
  for (int p = 0; p < 9; ++p) {
    const R n1 = f[2 * p + 1] - feq[2 * p + 1];
    const R n2 = f[2 * p + 2] - feq[2 * p + 2];
    a[p] = n1 + n2;
    b[p] = n1 - n2;
  }
  mrt_relax<R>(f, r0, a, b, s_over_norm);
}

}  // namespace flb
