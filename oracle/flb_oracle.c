/* flb_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference FreeLB (zdxying/FreeLB) D3Q19
 * stream-and-collide path and of its lid-driven cavity set-up.  It is the
 * checker for the CUDA path: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py load it.  The product library never links it.
 *
 * Parity of this restatement with the reference itself is pinned by
 * tests/test_oracle_golden.py against fixtures generated by running the
 * reference's own CPU code (oracle/ref_cavity.cpp compiled from the reference
 * headers; generator: tests/golden/make_golden.py).
 *
 * Build: see oracle/Makefile (gcc -O2 -ffp-contract=off -fopenmp -shared).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* D3Q19 velocities, reference ordering (src/lbm/lattice_set.h:263-266). */
static const int ORC_C[19][3] = {
    {0, 0, 0},  {1, 0, 0},   {-1, 0, 0}, {0, 1, 0},   {0, -1, 0}, {0, 0, 1},   {0, 0, -1},
    {1, 1, 0},  {-1, -1, 0}, {1, 0, 1},  {-1, 0, -1}, {0, 1, 1},  {0, -1, -1}, {1, -1, 0},
    {-1, 1, 0}, {1, 0, -1},  {-1, 0, 1}, {0, 1, -1},  {0, -1, 1}};

enum { ORC_OP_NONE = 0, ORC_OP_BULK = 1, ORC_OP_BB = 2, ORC_OP_MBB = 3, ORC_OP_FIELD_BGK = 4 };
enum { ORC_MODEL_BGK = 0, ORC_MODEL_MRT = 1, ORC_MODEL_LES = 2, ORC_MODEL_BRINKMAN = 3 };

typedef struct {
  int nx, ny, nz;       /* stored mesh, x fastest */
  int model;            /* ORC_MODEL_* used by ORC_OP_BULK cells */
  double omega;         /* 1/tau */
  double cs_smag;       /* Smagorinsky constant (LES) */
  double mrt_s[19];     /* MRT rates; shear entries are replaced by omega */
  uint8_t op_lut[256];  /* op for each flag value (first matching task key) */
  const void* alpha;    /* Brinkman porosity per cell (ORC_MODEL_BRINKMAN), OT[N] */
} oracle_desc;

/* D3Q19 d'Humieres 2002 basis on the reference ordering and its inverse
 * (InvM[i][j] = M[j][i] / |M_j|^2), filled once by orc_init_basis(). */
static double ORC_M[19 * 19];
static double ORC_INVM[19 * 19];
static int ORC_INV_NUM[19 * 19];
static int ORC_INV_DEN[19 * 19];
static int orc_basis_ready = 0;

static int orc_basis_row(int k, const int* c) {
  const int x = c[0], y = c[1], z = c[2];
  const int c2 = x * x + y * y + z * z;
  switch (k) {
    case 0: return 1;
    case 1: return 19 * c2 - 30;
    case 2: return (21 * c2 * c2 - 53 * c2 + 24) / 2;
    case 3: return x;
    case 4: return (5 * c2 - 9) * x;
    case 5: return y;
    case 6: return (5 * c2 - 9) * y;
    case 7: return z;
    case 8: return (5 * c2 - 9) * z;
    case 9: return 3 * x * x - c2;
    case 10: return (3 * c2 - 5) * (3 * x * x - c2);
    case 11: return y * y - z * z;
    case 12: return (3 * c2 - 5) * (y * y - z * z);
    case 13: return x * y;
    case 14: return y * z;
    case 15: return x * z;
    case 16: return x * (y * y - z * z);
    case 17: return y * (z * z - x * x);
    default: return z * (x * x - y * y);
  }
}

static void orc_init_basis(void) {
  if (orc_basis_ready) return;
  int norm[19];
  for (int k = 0; k < 19; ++k) {
    norm[k] = 0;
    for (int i = 0; i < 19; ++i) {
      const int v = orc_basis_row(k, ORC_C[i]);
      ORC_M[k * 19 + i] = v;
      norm[k] += v * v;
    }
  }
  /* InvM entries are evaluated like the reference's Fraction<>: T(num)/T(den);
   * the float path recomputes them from these integers (see _impl). */
  for (int i = 0; i < 19; ++i)
    for (int j = 0; j < 19; ++j) {
      ORC_INV_NUM[i * 19 + j] = (int)ORC_M[j * 19 + i];
      ORC_INV_DEN[i * 19 + j] = norm[j];
      ORC_INVM[i * 19 + j] = ORC_M[j * 19 + i] / (double)norm[j];
    }
  orc_basis_ready = 1;
}

void oracle_mrt_basis(double* M, double* invM) {
  orc_init_basis();
  memcpy(M, ORC_M, sizeof(ORC_M));
  memcpy(invM, ORC_INVM, sizeof(ORC_INVM));
}

/* Lid-driven cavity flags for Ni^3 interior cells on the stored (Ni+2)^3 mesh.
 * Restates benchmarks/cavity3d/cavity3d.cpp:136-142 with
 * BasicBlock::forEach(AABB) (src/geometry/basic_geometry.hh:484-505),
 * Block3D::SetupBoundary (src/geometry/block_geometry3d.hh:78-104) and
 * AABB::isInside (src/geometry/basic_geometry.hh:39-48) for Cell_Len = 1:
 * cell centres are idx - 0.5, so cells 1..Ni are inside the cavity AABB (2),
 * the outer layer of those gets bounce-back (4) and the top layer z = Ni with
 * 2 <= x,y <= Ni-1 becomes the moving wall (8); the rest stays void (1). */
void oracle_cavity_flags(int ni, uint8_t* flags) {
  const long n = ni + 2;
  for (long z = 0; z < n; ++z)
    for (long y = 0; y < n; ++y)
      for (long x = 0; x < n; ++x) {
        uint8_t f = 1;
        const int in = x >= 1 && x <= ni && y >= 1 && y <= ni && z >= 1 && z <= ni;
        if (in) {
          const int wall = x == 1 || x == ni || y == 1 || y == ni || z == 1 || z == ni;
          f = wall ? 4 : 2;
          if (wall && z == ni && x >= 2 && x <= ni - 1 && y >= 2 && y <= ni - 1) f = 8;
        }
        flags[(z * n + y) * n + x] = f;
      }
}

#define OT float
#define OS f32
#include "flb_oracle_impl.h"
#undef OT
#undef OS

#define OT double
#define OS f64
#include "flb_oracle_impl.h"
#undef OT
#undef OS

/* Build the op lookup table from an ordered (key, op) task list: a flag value
 * takes the op of the first task whose key shares a bit with it
 * (src/utils/tmp.h:283-309 util::isFlag). */
void oracle_build_lut(int ntasks, const uint8_t* keys, const uint8_t* ops, uint8_t* lut) {
  for (int v = 0; v < 256; ++v) {
    lut[v] = ORC_OP_NONE;
    for (int t = 0; t < ntasks; ++t)
      if (v & keys[t]) {
        lut[v] = ops[t];
        break;
      }
  }
}

int oracle_prepare(oracle_desc* d) {
  orc_init_basis();
  (void)d;
  return 0;
}
