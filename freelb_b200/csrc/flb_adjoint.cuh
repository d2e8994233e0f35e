// flb_adjoint.cuh -- hand-written discrete adjoint of the stream-and-collide step.
//
// Forward step (flb_pull.cuh):  R_{t+1} = S(C(R_t)),  S = streaming (a
// permutation), C = per-cell collision chosen by the flag.  Objective
// J = sum over bulk cells of |u|^2 at step T, with u the forced moment
// u = sum c f / (rho + alpha/2).  The adjoint lambda_t = dJ/dR_t obeys
//     mu_t = S^T lambda_{t+1}            (mu_t(x,i) = lambda_{t+1}(x + c_i, i))
//     lambda_t = J_C(R_t)^T mu_t          (local 19 x 19, applied analytically)
// and parameter gradients accumulate mu_t . dC/dtheta(R_t) in FP64.
//
// Per-cell transposed Jacobians:
//   none:            lambda = mu
//   BounceBack:      lambda_j = mu_opp(j)       (collision.ur.h:62-93 is a swap)
//   MovingWall:      lambda_j = mu_opp(j); d/du_lid adds
//                    sum_{i odd} (mu_i - mu_{i+1}) 6 w_i rho_w c_ix
//   bulk (BGK with Brinkman drag, alpha = 0 for plain BGK):
//     C_i = (1-w) f_i + w feq_i(rho, u) + (1 - w/2) G_i(u),  rho = sum f,
//     u = m / (rho + alpha/2),  G_i = -alpha w_i (3 c.u - 3|u|^2 + 9 (c.u)^2)
//     lambda_j = (1-w) mu_j + w sum_i mu_i feq_i / rho
//                + b . (c_j - u) / (rho + alpha/2),
//     b = sum_i mu_i (w dfeq_i/du + (1 - w/2) dG_i/du)
//     dJ/dtau   += -w^2 sum_i mu_i (feq_i - f_i - G_i/2)
//     dJ/dalpha += b . (-u / (2 (rho + alpha/2))) + (1 - w/2) sum_i mu_i dG_i/dalpha|_u
//   bulk MRT: C = f - A (f - feq), A = M^-1 S M, which is symmetric for the
//   orthogonal basis (M^-1 = M^T diag(1/|M_k|^2)), so with nu = A mu
//     lambda_j = mu_j - nu_j + sum nu feq / rho + (c_j - u) . b / rho,
//     b = sum_i nu_i dfeq_i/du,
//     dJ/dtau += w^2 sum over shear moments k of (M_k.mu)(M_k.(f - feq)) / |M_k|^2
//   (the shear rates are w = 1/tau).
// with the state R_t recomputed from checkpoints (flb_api.cu drives it).
#pragma once

#include "flb_pull.cuh"

namespace flb {

struct AdjParams {
  const void* lam_in;   // lambda_{t+1}, own-cell layout, arithmetic type
  void* lam_out;        // lambda_t
  const void* q;        // Q_t: stored forward state with R_t = stream(Q_t)
  double* galpha;       // per-cell dJ/dalpha (FP64), own-cell layout
  double* gpart;        // per thread block: [2b] dJ/dtau, [2b+1] dJ/du_lid partial sums
};

// Transposed Jacobian of a bulk MRT cell (see above).  s: per-moment rate over
// |M_k|^2 as the forward step uses it.  The state enters as rho, u and the
// non-equilibrium part n = f - feq.
template <typename R>
__device__ __forceinline__ void mrt_vjp(R rho, R ux, R uy, R uz, const R* n, const R* mu, R* lam,
                                        R omega, const R* s, double& gtau) {
  R am[9], bm[9], an[9], bn[9];
#pragma unroll
  for (int p = 0; p < 9; ++p) {
    am[p] = mu[2 * p + 1] + mu[2 * p + 2];
    bm[p] = mu[2 * p + 1] - mu[2 * p + 2];
    const R n1 = n[2 * p + 1], n2 = n[2 * p + 2];
    an[p] = n1 + n2;
    bn[p] = n1 - n2;
  }
  // dJ/dtau over the shear moments
  double gt = 0;
#pragma unroll
  for (int k = 0; k < Q; ++k)
    if (mrt_shear(k))
      gt += double(mrt_moment<R>(k, mu[0], am, bm)) * double(mrt_moment<R>(k, n[0], an, bn)) /
            double(mrt_norm_lit(k));
  gtau += double(omega) * double(omega) * gt;
  // nu = A mu, from the forward relaxation applied to zero
  R nu[Q];
#pragma unroll
  for (int i = 0; i < Q; ++i) nu[i] = R(0);
  mrt_relax<R>(nu, mu[0], am, bm, s);
#pragma unroll
  for (int i = 0; i < Q; ++i) nu[i] = -nu[i];
  // weighted moments of nu (as in the BGK transpose)
  R sp[Q], dp[Q];
#pragma unroll
  for (int i = 1; i < Q; i += 2) {
    sp[i] = nu[i] + nu[i + 1];
    dp[i] = nu[i] - nu[i + 1];
  }
  const R w0 = R(1) / R(3), wa = R(1) / R(18), wd = R(1) / R(36);
  const R M0 = w0 * nu[0] + wa * ((sp[1] + sp[3]) + sp[5]) +
               wd * (((sp[7] + sp[9]) + (sp[11] + sp[13])) + (sp[15] + sp[17]));
  const R M1x = wa * dp[1] + wd * ((dp[7] + dp[9]) + (dp[13] + dp[15]));
  const R M1y = wa * dp[3] + wd * ((dp[7] + dp[11]) + (dp[17] - dp[13]));
  const R M1z = wa * dp[5] + wd * ((dp[9] + dp[11]) - (dp[15] + dp[17]));
  const R Pxx = wa * sp[1] + wd * ((sp[7] + sp[9]) + (sp[13] + sp[15]));
  const R Pyy = wa * sp[3] + wd * ((sp[7] + sp[11]) + (sp[13] + sp[17]));
  const R Pzz = wa * sp[5] + wd * ((sp[9] + sp[11]) + (sp[15] + sp[17]));
  const R Pxy = wd * (sp[7] - sp[13]);
  const R Pxz = wd * (sp[9] - sp[15]);
  const R Pyz = wd * (sp[11] - sp[17]);
  const R Pux = Pxx * ux + Pxy * uy + Pxz * uz;
  const R Puy = Pxy * ux + Pyy * uy + Pyz * uz;
  const R Puz = Pxz * ux + Pyz * uy + Pzz * uz;
  const R u2 = ux * ux + uy * uy + uz * uz;
  const R feq_sum = M0 * (R(1) - R(1.5) * u2) + R(3) * (M1x * ux + M1y * uy + M1z * uz) +
                    R(4.5) * (ux * Pux + uy * Puy + uz * Puz);
  // b / rho = 3 M1 + 9 P u - 3 M0 u
  const R qx = R(3) * M1x + R(9) * Pux - R(3) * M0 * ux;
  const R qy = R(3) * M1y + R(9) * Puy - R(3) * M0 * uy;
  const R qz = R(3) * M1z + R(9) * Puz - R(3) * M0 * uz;
  const R base = feq_sum - (qx * ux + qy * uy + qz * uz);
#pragma unroll
  for (int j = 0; j < Q; ++j) {
    R cb = base;
    if (cx(j) > 0) cb += qx; else if (cx(j) < 0) cb -= qx;
    if (cy(j) > 0) cb += qy; else if (cy(j) < 0) cb -= qy;
    if (cz(j) > 0) cb += qz; else if (cz(j) < 0) cb -= qz;
    lam[j] = mu[j] - nu[j] + cb;
  }
}

// Transposed Jacobian of one cell.  f: R_t of the cell as stored (DEV: the
// FP32S deviations f - rho0 w), mu in, lam out.
template <typename R, int MODEL, bool DEV>
__device__ __forceinline__ void cell_vjp(const StepParams& p, int op, const R* f, const R* mu,
                                         R* lam, R omega, R alpha, R rho_w, double& gtau,
                                         double& gulid, double& galpha) {
  if (op == OP_BB || op == OP_MBB) {
    lam[0] = mu[0];
#pragma unroll
    for (int i = 1; i < Q; i += 2) {
      lam[i] = mu[i + 1];
      lam[i + 1] = mu[i];
    }
    if (op == OP_MBB) {
      double s = 0;
#pragma unroll
      for (int i = 1; i < Q; i += 2)
        if (cx(i) != 0) s += double(mu[i] - mu[i + 1]) * double(cx(i)) * double(weight<R>(i));
      gulid += 6.0 * double(rho_w) * s;
    }
    return;
  }
  if (op != OP_BULK) {
#pragma unroll
    for (int i = 0; i < Q; ++i) lam[i] = mu[i];
    return;
  }
  if constexpr (MODEL == MODEL_MRT) {
    R s[Q];
#pragma unroll
    for (int k = 0; k < Q; ++k)
      s[k] = mrt_shear(k) ? omega * (R(1) / R(mrt_norm_lit(k))) : R(p.s_over_norm[k]);
    R rho, ux, uy, uz, n[Q];
    if constexpr (DEV) {
      R delta, den;
      dev_moments(reinterpret_cast<const float(&)[Q]>(*f), p.rho0, 0.0f, delta, rho, den, ux, uy,
                  uz);
      dev_neq(reinterpret_cast<const float(&)[Q]>(*f), delta, rho, ux, uy, uz, n);
    } else {
      R feq[Q];
      rho_u(f, rho, ux, uy, uz);
      feq2(feq, rho, ux, uy, uz);
#pragma unroll
      for (int i = 0; i < Q; ++i) n[i] = f[i] - feq[i];
    }
    mrt_vjp<R>(rho, ux, uy, uz, n, mu, lam, omega, s, gtau);
    return;
  }
  R rho, den, ux, uy, uz, delta = R(0);
  if constexpr (DEV)
    dev_moments(reinterpret_cast<const float(&)[Q]>(*f), p.rho0, alpha, delta, rho, den, ux, uy,
                uz);
  else
    forced_moments(f, alpha, rho, den, ux, uy, uz);
  const R u2 = ux * ux + uy * uy + uz * uz;
  const R fo = R(1) - R(0.5) * omega;
  // The sums over i above need only the weighted moments of mu:
  //   M0 = sum w_i mu_i, M1 = sum w_i mu_i c_i, P = sum w_i mu_i c_i c_i^T,
  // since feq_i, G_i and their u-derivatives are polynomials in c_i:
  //   sum mu_i feq_i = rho (M0 (1 - 3|u|^2/2) + 3 M1.u + 9/2 u.P.u)
  //   sum mu_i w_i poly_i = 3 M1.u - 3 |u|^2 M0 + 9 u.P.u
  //   b = 3 (w rho - fo alpha) M1 + (9 w rho - 18 fo alpha) P u - (3 w rho - 6 fo alpha) M0 u
  // (w = omega, fo = 1 - omega/2).  Pair sums s and differences d of opposite
  // directions carry all of it.
  R sp[Q], dp[Q];
#pragma unroll
  for (int i = 1; i < Q; i += 2) {
    sp[i] = mu[i] + mu[i + 1];
    dp[i] = mu[i] - mu[i + 1];
  }
  const R w0 = R(1) / R(3), wa = R(1) / R(18), wd = R(1) / R(36);
  const R M0 = w0 * mu[0] + wa * ((sp[1] + sp[3]) + sp[5]) +
               wd * (((sp[7] + sp[9]) + (sp[11] + sp[13])) + (sp[15] + sp[17]));
  const R M1x = wa * dp[1] + wd * ((dp[7] + dp[9]) + (dp[13] + dp[15]));
  const R M1y = wa * dp[3] + wd * ((dp[7] + dp[11]) + (dp[17] - dp[13]));
  const R M1z = wa * dp[5] + wd * ((dp[9] + dp[11]) - (dp[15] + dp[17]));
  const R Pxx = wa * sp[1] + wd * ((sp[7] + sp[9]) + (sp[13] + sp[15]));
  const R Pyy = wa * sp[3] + wd * ((sp[7] + sp[11]) + (sp[13] + sp[17]));
  const R Pzz = wa * sp[5] + wd * ((sp[9] + sp[11]) + (sp[15] + sp[17]));
  const R Pxy = wd * (sp[7] - sp[13]);
  const R Pxz = wd * (sp[9] - sp[15]);
  const R Pyz = wd * (sp[11] - sp[17]);
  const R Pux = Pxx * ux + Pxy * uy + Pxz * uz;
  const R Puy = Pxy * ux + Pyy * uy + Pyz * uz;
  const R Puz = Pxz * ux + Pyz * uy + Pzz * uz;
  const R uPu = ux * Pux + uy * Puy + uz * Puz;
  const R M1u = M1x * ux + M1y * uy + M1z * uz;
  const R feq_sum = M0 * (R(1) - R(1.5) * u2) + R(3) * M1u + R(4.5) * uPu;  // sum mu feq / rho
  const R poly_sum = R(3) * M1u - R(3) * u2 * M0 + R(9) * uPu;
  const R sF = rho * feq_sum;
  const R sGa = -poly_sum;
  const R sG = alpha * sGa;
  const R wr = omega * rho, fa = fo * alpha;
  const R A = R(3) * (wr - fa), B = R(9) * wr - R(18) * fa, Cc = R(3) * wr - R(6) * fa;
  const R bx = A * M1x + B * Pux - Cc * M0 * ux;
  const R by = A * M1y + B * Puy - Cc * M0 * uy;
  const R bz = A * M1z + B * Puz - Cc * M0 * uz;
  R sR = 0;  // sum mu f (DEV: sum mu d)
#pragma unroll
  for (int i = 0; i < Q; ++i) sR += mu[i] * f[i];
  // sum mu (feq - f); DEV, with f = d + rho0 w and sum mu rho0 w = rho0 M0:
  // delta M0 + rho (feq_sum - M0) - sum mu d, all of deviation size
  double s_neq;
  if constexpr (DEV)
    s_neq = double(delta * M0 + rho * (R(3) * M1u + R(4.5) * uPu - R(1.5) * u2 * M0)) - double(sR);
  else
    s_neq = double(sF) - double(sR);
  const R inv_den = R(1) / den;
  const R ub = bx * ux + by * uy + bz * uz;
  // lambda_j = (1-w) mu_j + w sum mu feq / rho + (c_j - u).b / den
  const R base = omega * feq_sum - ub * inv_den;
  const R qx = bx * inv_den, qy = by * inv_den, qz = bz * inv_den;
  const R c1 = R(1) - omega;
#pragma unroll
  for (int j = 0; j < Q; ++j) {
    R cb = base;
    if (cx(j) > 0) cb += qx; else if (cx(j) < 0) cb -= qx;
    if (cy(j) > 0) cb += qy; else if (cy(j) < 0) cb -= qy;
    if (cz(j) > 0) cb += qz; else if (cz(j) < 0) cb -= qz;
    lam[j] = c1 * mu[j] + cb;
  }
  gtau += -double(omega) * double(omega) * (s_neq - 0.5 * double(sG));
  galpha += double(-ub * R(0.5) * inv_den) + double(fo) * double(sGa);
}

// One backward step over a single block: lam_out = J_C^T S^T lam_in.  DEV: the
// forward states are FP32S deviations (read as stored).
template <typename R, int V, int MODEL, bool DEV>
__global__ void __launch_bounds__(256) k_adjoint_step(const StepParams p, const AdjParams a) {
  const Geom g{p.nx, p.ny, p.nz, p.pitch, p.plane, 0};
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int x0, y, z;
  const bool valid = chunk_coords<V>(g, q, x0, y, z);
  double gtau = 0, gulid = 0;
  if (valid) {
  R mu[Q][V], fr[Q][V];
  gather_chunk<R, R, V, -1>(static_cast<const R*>(a.lam_in), p.dstride, g, p.shift, 1.f, x0, y,
                            z, mu);
  gather_chunk<R, R, V, 1>(static_cast<const R*>(a.q), p.dstride, g, p.shift, 1.f, x0, y, z, fr);
  {
    const long long cell0 = (long long)y * g.pitch + (long long)z * g.plane + x0;
    const int nvalid = min(V, g.nx - x0);
    uint8_t fl[V];
    load_flags<V>(p.flags + cell0, fl);
    const R* alpha = static_cast<const R*>(p.alpha);
    const R* rho = static_cast<const R*>(p.rho);
    const R omega = R(p.omega);
    R lam[Q][V];
#pragma unroll
    for (int k = 0; k < V; ++k) {
      R f[Q], m[Q], l[Q];
#pragma unroll
      for (int i = 0; i < Q; ++i) {
        f[i] = fr[i][k];
        m[i] = mu[i][k];
      }
      double ga = 0;
      if (k < nvalid) {
        const int op = select_op(p, fl[k]);
        const R al = alpha ? alpha[cell0 + k] : R(0);
        const R rw = op == OP_MBB ? rho[cell0 + k] : R(1);
        cell_vjp<R, MODEL, DEV>(p, op, f, m, l, omega, al, rw, gtau, gulid, ga);
        if (op == OP_BULK && alpha) a.galpha[cell0 + k] += ga;
      } else {
#pragma unroll
        for (int i = 0; i < Q; ++i) l[i] = R(0);
      }
#pragma unroll
      for (int i = 0; i < Q; ++i) lam[i][k] = l[i];
    }
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      R v[V];
#pragma unroll
      for (int k = 0; k < V; ++k) v[k] = lam[i][k];
      vstore<R, R, V>(static_cast<R*>(a.lam_out) + i * p.dstride + cell0, v, 0.f, 1.f);
    }
  }
  }
  // Thread block b adds its sums to its own slots (same grid every step, one
  // stream): no atomics, and the final sum over blocks has a fixed order.
  gtau = warp_sum(gtau);
  gulid = warp_sum(gulid);
  __shared__ double red[2][8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    red[0][wid] = gtau;
    red[1][wid] = gulid;
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    double v = 0;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) v += red[threadIdx.x][w];
    a.gpart[2 * blockIdx.x + threadIdx.x] += v;
  }
}

// Objective J = sum_{bulk cells} |u|^2 at the current state, its seed
// lambda_T = dJ/dR_T and the direct term dJ/dalpha = -|u|^2 / (rho + alpha/2).
// With seed == false only J is accumulated (finite-difference evaluations).
// Compensated (double-double) sums: CTA b writes its share of J as the pair
// partials[2b], partials[2b + 1]; k_sum_partials_dd adds them in a fixed order,
// so J is the same bits on every evaluation of the same state and carries no
// summation error that a central difference of J would divide by 2h.
template <typename S, typename R>
__global__ void __launch_bounds__(256) k_objective(LayoutParams L, Geom g, const S* pops,
                                                   StepParams sp, R* lam, double* galpha,
                                                   double* partials, bool seed) {
  dd jsum;
  const long long total = L.plane * L.nz;
  const R* alpha = static_cast<const R*>(sp.alpha);
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total;
       c += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    if (!decode_cell(L, c, x, y, z)) continue;
    const int op = select_op(sp, sp.flags[c]);
    if (op != OP_BULK) {
      if (seed)
#pragma unroll
        for (int i = 0; i < Q; ++i) lam[i * L.dstride + c] = R(0);
      continue;
    }
    R f[Q];
    const R al = alpha ? alpha[c] : R(0);
    R rho, den, ux, uy, uz;
    if constexpr (std::is_same<S, dev32>::value) {
      R delta;
      gather_stored<S, R>(pops, L.dstride, g, x, y, z, sp, f);
      dev_moments(f, sp.rho0, al, delta, rho, den, ux, uy, uz);
    } else {
      gather_R<S, R>(pops, L.dstride, g, x, y, z, sp, f);
      forced_moments(f, al, rho, den, ux, uy, uz);
    }
    const R u2 = ux * ux + uy * uy + uz * uz;
    jsum.add(double(u2));
    if (seed) {
#pragma unroll
      for (int j = 0; j < Q; ++j)
        lam[j * L.dstride + c] =
            R(2) * ((R(cx(j)) - ux) * ux + (R(cy(j)) - uy) * uy + (R(cz(j)) - uz) * uz) / den;
      if (galpha) galpha[c] = -double(u2) / double(den);
    }
  }
  jsum = warp_sum_dd(jsum);
  __shared__ double red[2][8];
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = jsum.hi;
    red[1][threadIdx.x >> 5] = jsum.lo;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    dd v;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) {
      dd x;
      x.hi = red[0][w];
      x.lo = red[1][w];
      v.add(x);
    }
    partials[2 * blockIdx.x] = v.hi;
    partials[2 * blockIdx.x + 1] = v.lo;
  }
}

}  // namespace flb
