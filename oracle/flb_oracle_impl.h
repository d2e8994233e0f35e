/* Oracle restatement body, included twice by flb_oracle.c with
 *   OT  = float | double   (the reference's T)
 *   OS  = f32   | f64      (symbol suffix)
 *
 * TEST INFRASTRUCTURE ONLY -- a CPU restatement of the reference FreeLB D3Q19
 * stream-and-collide path, used by tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py as the checker.  Never linked into the product.
 *
 * Every function follows the reference arithmetic order:
 *   moments      src/lbm/moment.ur.h:505-517 (rhoUImpl<D3Q19>)
 *   Pi_neq       src/lbm/moment.ur.h:751-762 (Pi_ab_neq<D3Q19>)
 *   equilibrium  src/lbm/equilibrium.ur.h:166-215 (SecondOrderImpl<D3Q19>)
 *   BGK          src/lbm/collision.h:40-57
 *   BounceBack   src/lbm/collision.ur.h:62-93
 *   moving wall  src/lbm/collision.ur.h:130-187
 *   LES          src/lbm/collisionLES.h:36-62
 *   MRT          src/lbm/collisionMRT.h:142-188 (generic algorithm; D3Q19 basis of
 *                d'Humieres et al. 2002, see gen_mrt_d3q19.py)
 *   streaming    src/data_struct/field.h:626-697 (CyclicArray periodic shift: after
 *                rotate(), a[x] = old a[(x - Delta_i) mod N] over the whole linear index)
 */

#define CAT2(a, b) a##_##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, OS)

static void FN(rhou)(const OT* f, OT* rho, OT u[3]) {
  OT r = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8] + f[9] + f[10] + f[11] +
         f[12] + f[13] + f[14] + f[15] + f[16] + f[17] + f[18];
  u[0] = (f[1] - f[2] + f[7] - f[8] + f[9] - f[10] + f[13] - f[14] + f[15] - f[16]) / r;
  u[1] = (f[3] - f[4] + f[7] - f[8] + f[11] - f[12] - f[13] + f[14] + f[17] - f[18]) / r;
  u[2] = (f[5] - f[6] + f[9] - f[10] + f[11] - f[12] - f[15] + f[16] - f[17] + f[18]) / r;
  *rho = r;
}

static void FN(feq)(OT* feq, OT rho, const OT u[3]) {
  const OT InvCs2 = (OT)3;
  const OT InvCs2x = (OT)0.5 * InvCs2;
  const OT var0 = (OT)1 - (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]) * InvCs2x;
  const OT rhowk0 = ((OT)1 / (OT)3) * rho;
  const OT rhowk1 = ((OT)1 / (OT)18) * rho;
  const OT rhowk7 = ((OT)1 / (OT)36) * rho;
  const OT k1 = InvCs2 * (u[0]);
  const OT v1 = var0 + k1 * k1 * (OT)0.5;
  const OT k3 = InvCs2 * (u[1]);
  const OT v3 = var0 + k3 * k3 * (OT)0.5;
  const OT k5 = InvCs2 * (u[2]);
  const OT v5 = var0 + k5 * k5 * (OT)0.5;
  const OT k7 = InvCs2 * (u[0] + u[1]);
  const OT v7 = var0 + k7 * k7 * (OT)0.5;
  const OT k9 = InvCs2 * (u[0] + u[2]);
  const OT v9 = var0 + k9 * k9 * (OT)0.5;
  const OT k11 = InvCs2 * (u[1] + u[2]);
  const OT v11 = var0 + k11 * k11 * (OT)0.5;
  const OT k13 = InvCs2 * (u[0] - u[1]);
  const OT v13 = var0 + k13 * k13 * (OT)0.5;
  const OT k15 = InvCs2 * (u[0] - u[2]);
  const OT v15 = var0 + k15 * k15 * (OT)0.5;
  const OT k17 = InvCs2 * (u[1] - u[2]);
  const OT v17 = var0 + k17 * k17 * (OT)0.5;
  feq[0] = rhowk0 * var0;
  feq[1] = rhowk1 * (v1 + k1);
  feq[2] = rhowk1 * (v1 - k1);
  feq[3] = rhowk1 * (v3 + k3);
  feq[4] = rhowk1 * (v3 - k3);
  feq[5] = rhowk1 * (v5 + k5);
  feq[6] = rhowk1 * (v5 - k5);
  feq[7] = rhowk7 * (v7 + k7);
  feq[8] = rhowk7 * (v7 - k7);
  feq[9] = rhowk7 * (v9 + k9);
  feq[10] = rhowk7 * (v9 - k9);
  feq[11] = rhowk7 * (v11 + k11);
  feq[12] = rhowk7 * (v11 - k11);
  feq[13] = rhowk7 * (v13 + k13);
  feq[14] = rhowk7 * (v13 - k13);
  feq[15] = rhowk7 * (v15 + k15);
  feq[16] = rhowk7 * (v15 - k15);
  feq[17] = rhowk7 * (v17 + k17);
  feq[18] = rhowk7 * (v17 - k17);
}

static void FN(bgk_relax)(OT* f, const OT* feq, OT omega) {
  const OT _omega = (OT)1 - omega;
  for (int i = 0; i < 19; ++i) f[i] = omega * feq[i] + _omega * f[i];
}

static void FN(bounceback)(OT* f) {
  for (int i = 1; i < 19; i += 2) {
    const OT t = f[i];
    f[i] = f[i + 1];
    f[i + 1] = t;
  }
}

static void FN(movingwall)(OT* f, OT rho_w, const OT uw[3]) {
  const OT InvCs2_2 = (OT)2 * (OT)3;
  const OT rhox = InvCs2_2 * rho_w;
  const OT w1 = (OT)1 / (OT)18, w7 = (OT)1 / (OT)36;
  const OT uc[19] = {0,
                     uw[0] * w1 * rhox, 0,
                     uw[1] * w1 * rhox, 0,
                     uw[2] * w1 * rhox, 0,
                     (uw[0] + uw[1]) * w7 * rhox, 0,
                     (uw[0] + uw[2]) * w7 * rhox, 0,
                     (uw[1] + uw[2]) * w7 * rhox, 0,
                     (uw[0] - uw[1]) * w7 * rhox, 0,
                     (uw[0] - uw[2]) * w7 * rhox, 0,
                     (uw[1] - uw[2]) * w7 * rhox, 0};
  for (int i = 1; i < 19; i += 2) {
    const OT t = f[i];
    f[i] = f[i + 1] + uc[i];
    f[i + 1] = t - uc[i];
  }
}

static void FN(les)(OT* f, OT omega, OT cs, OT rho_field_unused) {
  (void)rho_field_unused;
  OT rho, u[3], feq[19], pi[6];
  FN(rhou)(f, &rho, u);
  const OT cs2 = (OT)1 / (OT)3;
  pi[0] = f[1] + f[2] + f[7] + f[8] + f[9] + f[10] + f[13] + f[14] + f[15] + f[16] -
          rho * (u[0] * u[0] + cs2);
  pi[1] = f[7] + f[8] - f[13] - f[14] - rho * (u[0] * u[1]);
  pi[2] = f[9] + f[10] - f[15] - f[16] - rho * (u[0] * u[2]);
  pi[3] = f[3] + f[4] + f[7] + f[8] + f[11] + f[12] + f[13] + f[14] + f[17] + f[18] -
          rho * (u[1] * u[1] + cs2);
  pi[4] = f[11] + f[12] - f[17] - f[18] - rho * (u[1] * u[2]);
  pi[5] = f[5] + f[6] + f[9] + f[10] + f[11] + f[12] + f[15] + f[16] + f[17] + f[18] -
          rho * (u[2] * u[2] + cs2);
  const OT nsq = pi[0] * pi[0] + pi[1] * pi[1] * 2 + pi[2] * pi[2] * 2 + pi[3] * pi[3] +
                 pi[4] * pi[4] * 2 + pi[5] * pi[5];
  const OT norm = (OT)sqrt((double)nsq);
  /* collisionLES.h:47: the RHO field holds this step's density because the
   * momenta scheme writes to the field; sqrt(2) is evaluated in double there. */
  const OT coeff = (OT)((double)(cs * cs * (OT)3 * (OT)3 * 2) * sqrt(2.0) / (double)rho);
  const OT rt_mol = (OT)1 / omega;
  const OT rt_tur = (OT)0.5 * ((OT)sqrt((double)(rt_mol * rt_mol + coeff * norm)) - rt_mol);
  const OT eomega = (OT)1 / (rt_mol + rt_tur);
  FN(feq)(feq, rho, u);
  FN(bgk_relax)(f, feq, eomega);
}

/* BGK with Brinkman drag F = -alpha u: the forced moment of
 * moment::forcerhoUImpl (src/lbm/moment.h:408-422) solved for F = -alpha u,
 * u = sum c f / (rho + alpha/2); force::ForcePop (src/lbm/force.h:29-36)
 * F_i = (w_i F).(3 (c_i - u) + 9 (c_i.u) c_i); collision::BGKForce
 * (src/lbm/collision.h:61-90) f <- omega feq + (1-omega) f + (1-omega/2) F_i. */
static void FN(brinkman)(OT* f, OT omega, OT alpha) {
  OT rho = 0, m[3] = {0, 0, 0}, u[3], F[3], feq[19];
  for (int i = 0; i < 19; ++i) {
    rho += f[i];
    for (int d = 0; d < 3; ++d) m[d] += (OT)ORC_C[i][d] * f[i];
  }
  const OT den = rho + (OT)0.5 * alpha;
  for (int d = 0; d < 3; ++d) {
    u[d] = m[d] / den;
    F[d] = u[d] * (-alpha);
  }
  FN(feq)(feq, rho, u);
  const OT _omega = (OT)1 - omega;
  const OT fomega = (OT)1 - (OT)0.5 * omega;
  for (int i = 0; i < 19; ++i) {
    const OT w = (i == 0) ? (OT)1 / (OT)3 : (i < 7 ? (OT)1 / (OT)18 : (OT)1 / (OT)36);
    const OT cu = (OT)ORC_C[i][0] * u[0] + (OT)ORC_C[i][1] * u[1] + (OT)ORC_C[i][2] * u[2];
    OT fi = 0;
    for (int d = 0; d < 3; ++d) {
      const OT v = ((OT)ORC_C[i][d] - u[d]) * (OT)3 + (cu * (OT)9) * (OT)ORC_C[i][d];
      fi += (w * F[d]) * v;
    }
    f[i] = omega * feq[i] + _omega * f[i] + fomega * fi;
  }
}

static void FN(mrt)(OT* f, OT omega, const double* M, const int* inv_num, const int* inv_den,
                    const double* s) {
  OT rho, u[3], feq[19], m[19], meq[19], rt[19];
  for (int i = 0; i < 19; ++i) rt[i] = (OT)s[i];
  rt[9] = rt[11] = rt[13] = rt[14] = rt[15] = omega;
  FN(rhou)(f, &rho, u);
  for (int i = 0; i < 19; ++i) {
    m[i] = 0;
    for (int j = 0; j < 19; ++j) m[i] += (OT)M[i * 19 + j] * f[j];
  }
  FN(feq)(feq, rho, u);
  for (int i = 0; i < 19; ++i) {
    meq[i] = 0;
    for (int j = 0; j < 19; ++j) meq[i] += (OT)M[i * 19 + j] * feq[j];
  }
  for (int i = 0; i < 19; ++i) {
    OT acc = 0;
    for (int j = 0; j < 19; ++j) {
      const OT invm = (OT)inv_num[i * 19 + j] / (OT)inv_den[i * 19 + j];
      acc += (invm * rt[j]) * (m[j] - meq[j]);
    }
    f[i] -= acc;
  }
}

/* One time step over a single block: collide every cell in place by its flag
 * (first matching key, src/utils/tmp.h:283-309), then PS-stream every
 * direction (src/data_struct/block_lattice.hh:64-70).  `pops` is 19*N in the
 * reference's logical order; `tmp` is scratch of the same size. */
int FN(oracle_step)(const oracle_desc* d, const uint8_t* flags, OT* pops, OT* tmp,
                    const OT* rho_field, const OT* u_field, int nsteps) {
  const long nx = d->nx, ny = d->ny, nz = d->nz;
  const long N = nx * ny * nz;
  const OT omega = (OT)d->omega;
  const OT cs = (OT)d->cs_smag;
  long delta[19];
  orc_init_basis();
  for (int i = 0; i < 19; ++i) delta[i] = ORC_C[i][0] + ORC_C[i][1] * nx + ORC_C[i][2] * nx * ny;
  for (int step = 0; step < nsteps; ++step) {
#pragma omp parallel for schedule(static)
    for (long id = 0; id < N; ++id) {
      const int op = d->op_lut[flags[id]];
      if (op == ORC_OP_NONE) continue;
      OT f[19];
      for (int i = 0; i < 19; ++i) f[i] = pops[i * N + id];
      if (op == ORC_OP_BULK) {
        if (d->model == ORC_MODEL_BGK) {
          OT rho, u[3], feq[19];
          FN(rhou)(f, &rho, u);
          FN(feq)(feq, rho, u);
          FN(bgk_relax)(f, feq, omega);
        } else if (d->model == ORC_MODEL_LES) {
          FN(les)(f, omega, cs, 0);
        } else if (d->model == ORC_MODEL_BRINKMAN) {
          FN(brinkman)(f, omega, d->alpha ? ((const OT*)d->alpha)[id] : (OT)0);
        } else {
          FN(mrt)(f, omega, ORC_M, ORC_INV_NUM, ORC_INV_DEN, d->mrt_s);
        }
      } else if (op == ORC_OP_FIELD_BGK) {
        OT feq[19], u[3] = {u_field[3 * id], u_field[3 * id + 1], u_field[3 * id + 2]};
        FN(feq)(feq, rho_field[id], u);
        FN(bgk_relax)(f, feq, omega);
      } else if (op == ORC_OP_BB) {
        FN(bounceback)(f);
      } else if (op == ORC_OP_MBB) {
        const OT uw[3] = {u_field[3 * id], u_field[3 * id + 1], u_field[3 * id + 2]};
        FN(movingwall)(f, rho_field[id], uw);
      }
      for (int i = 0; i < 19; ++i) pops[i * N + id] = f[i];
    }
    /* streaming: new[x] = old[(x - delta) mod N] over the linear index */
#pragma omp parallel for schedule(static)
    for (long id = 0; id < N; ++id) {
      for (int i = 0; i < 19; ++i) {
        long src = id - delta[i];
        if (src < 0) src += N;
        else if (src >= N) src -= N;
        tmp[i * N + id] = pops[i * N + src];
      }
    }
    memcpy(pops, tmp, sizeof(OT) * 19 * (size_t)N);
  }
  return 0;
}

/* rho/u of every cell whose flag matches `key` (moment::rhoU<CELL,true> as a
 * task, src/lbm/moment.h:382-398), written into the RHO and VELOCITY fields. */
void FN(oracle_rhou_fields)(long N, const uint8_t* flags, uint8_t key, const OT* pops,
                            OT* rho_field, OT* u_field) {
#pragma omp parallel for schedule(static)
  for (long id = 0; id < N; ++id) {
    if (!(flags[id] & key)) continue;
    OT f[19], rho, u[3];
    for (int i = 0; i < 19; ++i) f[i] = pops[i * N + id];
    FN(rhou)(f, &rho, u);
    rho_field[id] = rho;
    u_field[3 * id] = u[0];
    u_field[3 * id + 1] = u[1];
    u_field[3 * id + 2] = u[2];
  }
}

/* Population initialisation f_i = rho0 * w_i (src/data_struct/block_lattice.hh:673-680). */
void FN(oracle_init_pops)(long N, double rho0_d, OT* pops) {
  const OT rho0 = (OT)rho0_d;
  for (int i = 0; i < 19; ++i) {
    const OT w = (i == 0) ? (OT)1 / (OT)3 : (i < 7 ? (OT)1 / (OT)18 : (OT)1 / (OT)36);
    const OT v = rho0 * w;
    for (long id = 0; id < N; ++id) pops[i * N + id] = v;
  }
}

#undef FN
#undef CAT
#undef CAT2
