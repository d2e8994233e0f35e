/* flb_boundary.h -- post-stream halfway bounce-back managers and the fixed
 * periodic boundary manager (libflb_b200.so).
 *
 * Replaces BBLikeFixedBlockBdManager<bounceback::POLICY<CELL>, ...>
 * (src/boundary/boundary.h:86-140) with BlockBoundaryManager::Apply(): after a
 * step, every inner cell whose flag shares a bit with `cell_flag` sets, for
 * each direction k pointing at a neighbour whose flag shares a bit with
 * `void_flag`, the returning population j = opp(k) from prev = f_k before
 * streaming and the cell's RHO (rho) and VELOCITY (u) fields
 * (bounce_back_boundary.h:167-256):
 *   FLB_BB_NORMAL         f_j = prev                                  (normal)
 *   FLB_BB_MOVINGWALL     f_j = prev + 2 InvCs2 w_j rho (u . c_j)      (movingwall)
 *   FLB_BB_ANTI_SIMPLE    f_j = 2 rho w_j - prev                       (anti_simple)
 *   FLB_BB_ANTI_O1        f_j = 2 feq1_j(rho, u) - prev                (anti_O1)
 *   FLB_BB_ANTI_O2        f_j = 2 feq2_j(rho, u) - prev                (anti_O2)
 *   FLB_BB_ANTI_PRESSURE  f_j = 2 rho w_j (1 + (uw.c_j)^2 InvCs4/2 - |uw|^2 InvCs2/2) - prev,
 *                         uw = u + (u - u(x + c_k))/2                  (anti_pressure)
 * Links are found once from the lattice's flags when the manager is created.
 * Single-block lattices.  Conventions as in flb.h.
 */
#ifndef FLB_BOUNDARY_H_
#define FLB_BOUNDARY_H_

#include "flb.h"

#ifdef __cplusplus
extern "C" {
#endif

#define FLB_BB_NORMAL 0
#define FLB_BB_MOVINGWALL 1
#define FLB_BB_ANTI_SIMPLE 2
#define FLB_BB_ANTI_O1 3
#define FLB_BB_ANTI_O2 4
#define FLB_BB_ANTI_PRESSURE 5

typedef struct flb_bb flb_bb;

/* Build a manager from the lattice's current flags (BlockFixedBoundary::Setup,
 * basic_boundary.h:213-262).  rho0 is the FP16S / FP32S shift density of the lattice. */
FLB_API int flb_bb_create(flb_lattice* lat, uint8_t cell_flag, uint8_t void_flag, int kind,
                          double rho0, flb_bb** out);
/* Boundary cells and (cell, direction) links of the manager. */
FLB_API int flb_bb_count(const flb_bb* bb, long long* ncells, long long* nlinks);
/* Apply after flb_step (BBLikeFixedBlockBdManager::Apply). */
FLB_API int flb_bb_apply(flb_bb* bb, flb_lattice* lat, void* stream);
FLB_API int flb_bb_destroy(flb_bb* bb);

/* FixedPeriodicBoundaryManager (src/boundary/periodic_boundary.h:136-321):
 * Setup(box0, dir0, box1, dir1) pairs the cells of box0 with those of box1
 * (each box's cells in z, y, x order, BasicBlock::getCellIdx,
 * geometry/basic_geometry.hh:593-619) and Apply(), called between
 * ApplyCellDynamics and Stream, copies the post-collision populations
 *   box0 cell[k] = box1 cell[k]  for k in getCommPopDir(dir0)
 *   box1 cell[k] = box0 cell[k]  for k in getCommPopDir(dir1)
 * (getCommPopDir, parallel/communicator.h:74-150: XN selects c_x > 0, XP
 * c_x < 0, ... unioned over the set bits).  This is the exchange the
 * reference performs when the two boxes lie in different blocks; its
 * same-block pairing takes the first send of the block for both receives and
 * keeps references into vectors that grow (the file's own "known bugs" note),
 * so the two-way exchange above is the defined behaviour implemented here.
 *
 * Boxes are inclusive stored-cell index ranges {x0, x1, y0, y1, z0, z1} of the
 * (single-block) lattice, clamped to the mesh like BasicBlock::getLocIdxRange;
 * a box that misses the interior [1, n-2] in some axis (the base block)
 * makes the manager empty, as does a lattice without a cell whose flag
 * shares a bit with cell_flag.  The boxes must hold the same number of cells.
 * Apply copies all sources first and then writes, so the result does not
 * depend on the order of the copies. */
#define FLB_NBR_XN 1
#define FLB_NBR_XP 2
#define FLB_NBR_YN 4
#define FLB_NBR_YP 8
#define FLB_NBR_ZN 16
#define FLB_NBR_ZP 32

typedef struct flb_periodic flb_periodic;

FLB_API int flb_periodic_create(flb_lattice* lat, const int box0[6], int dir0, const int box1[6],
                                int dir1, uint8_t cell_flag, flb_periodic** out);
/* Cell pairs and population copies of the manager. */
FLB_API int flb_periodic_count(const flb_periodic* per, long long* pairs, long long* copies);
/* Apply to the lattice's current populations: after the flb_step whose
 * collision the reference's Apply() follows, before the next flb_step. */
FLB_API int flb_periodic_apply(flb_periodic* per, flb_lattice* lat, void* stream);
FLB_API int flb_periodic_destroy(flb_periodic* per);

#ifdef __cplusplus
}
#endif

#endif /* FLB_BOUNDARY_H_ */
