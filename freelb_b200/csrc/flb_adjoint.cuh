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
// with the state R_t recomputed from checkpoints (flb_api.cu drives it).
#pragma once

#include "flb_pull.cuh"

namespace flb {

struct AdjParams {
  const void* lam_in;   // lambda_{t+1}, own-cell layout, arithmetic type
  void* lam_out;        // lambda_t
  const void* q;        // Q_t: stored forward state with R_t = stream(Q_t)
  double* galpha;       // per-cell dJ/dalpha (FP64), own-cell layout
  double* gscal;        // [0] dJ/dtau, [1] dJ/du_lid
};

// Transposed Jacobian of one cell.  f: R_t of the cell, mu in, lam out.
template <typename R>
__device__ __forceinline__ void cell_vjp(int op, const R* f, const R* mu, R* lam, R omega,
                                         R alpha, R rho_w, double& gtau, double& gulid,
                                         double& galpha) {
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
  R rho, den, ux, uy, uz;
  forced_moments(f, alpha, rho, den, ux, uy, uz);
  const R u2 = ux * ux + uy * uy + uz * uz;
  const R fo = R(1) - R(0.5) * omega;
  R sF = 0, sR = 0, sG = 0, sGa = 0, bx = 0, by = 0, bz = 0;
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const R c0 = R(cx(i)), c1 = R(cy(i)), c2 = R(cz(i));
    const R w = weight<R>(i);
    const R cu = c0 * ux + c1 * uy + c2 * uz;
    const R feq = w * rho * (R(1) + R(3) * cu + R(4.5) * cu * cu - R(1.5) * u2);
    const R poly = R(3) * cu - R(3) * u2 + R(9) * cu * cu;
    const R G = -alpha * w * poly;
    // w dfeq/du + (1 - w/2) dG/du
    const R kf = omega * w * rho, kg = -fo * alpha * w;
    const R t9 = R(9) * cu, t18 = R(18) * cu;
    const R dx = kf * (R(3) * c0 + t9 * c0 - R(3) * ux) + kg * (R(3) * c0 - R(6) * ux + t18 * c0);
    const R dy = kf * (R(3) * c1 + t9 * c1 - R(3) * uy) + kg * (R(3) * c1 - R(6) * uy + t18 * c1);
    const R dz = kf * (R(3) * c2 + t9 * c2 - R(3) * uz) + kg * (R(3) * c2 - R(6) * uz + t18 * c2);
    const R m = mu[i];
    sF += m * feq;
    sR += m * f[i];
    sG += m * G;
    sGa += m * (-w * poly);
    bx += m * dx;
    by += m * dy;
    bz += m * dz;
  }
  const R a = omega * sF / rho;
  const R inv_den = R(1) / den;
#pragma unroll
  for (int j = 0; j < Q; ++j) {
    const R cj = (R(cx(j)) - ux) * bx + (R(cy(j)) - uy) * by + (R(cz(j)) - uz) * bz;
    lam[j] = (R(1) - omega) * mu[j] + a + cj * inv_den;
  }
  gtau += -double(omega) * double(omega) * (double(sF) - double(sR) - 0.5 * double(sG));
  galpha += double(-(bx * ux + by * uy + bz * uz) * R(0.5) * inv_den) + double(fo) * double(sGa);
}

// One backward step over a single block: lam_out = J_C^T S^T lam_in.
template <typename R, int V>
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
        cell_vjp<R>(op, f, m, l, omega, al, rw, gtau, gulid, ga);
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
  gtau = warp_sum(gtau);
  gulid = warp_sum(gulid);
  if ((threadIdx.x & 31) == 0) {
    if (gtau != 0.0) atomicAdd(a.gscal + 0, gtau);
    if (gulid != 0.0) atomicAdd(a.gscal + 1, gulid);
  }
}

// Objective J = sum_{bulk cells} |u|^2 at the current state, its seed
// lambda_T = dJ/dR_T and the direct term dJ/dalpha = -|u|^2 / (rho + alpha/2).
// With seed == false only J is accumulated (finite-difference evaluations).
template <typename S, typename R>
__global__ void __launch_bounds__(256) k_objective(LayoutParams L, Geom g, const S* pops,
                                                   StepParams sp, R* lam, double* galpha,
                                                   double* jacc, bool seed) {
  double jsum = 0;
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
    gather_R<S, R>(pops, L.dstride, g, x, y, z, sp, f);
    const R al = alpha ? alpha[c] : R(0);
    R rho, den, ux, uy, uz;
    forced_moments(f, al, rho, den, ux, uy, uz);
    const R u2 = ux * ux + uy * uy + uz * uz;
    jsum += double(u2);
    if (seed) {
#pragma unroll
      for (int j = 0; j < Q; ++j)
        lam[j * L.dstride + c] =
            R(2) * ((R(cx(j)) - ux) * ux + (R(cy(j)) - uy) * uy + (R(cz(j)) - uz) * uz) / den;
      if (galpha) galpha[c] = -double(u2) / double(den);
    }
  }
  jsum = warp_sum(jsum);
  if ((threadIdx.x & 31) == 0 && jsum != 0.0) atomicAdd(jacc, jsum);
}

}  // namespace flb
