/* flb_boundary.h -- post-stream halfway bounce-back managers (libflb_b200.so).
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
 * basic_boundary.h:213-262).  rho0 is the FP16S shift density of the lattice. */
FLB_API int flb_bb_create(flb_lattice* lat, uint8_t cell_flag, uint8_t void_flag, int kind,
                          double rho0, flb_bb** out);
/* Boundary cells and (cell, direction) links of the manager. */
FLB_API int flb_bb_count(const flb_bb* bb, long long* ncells, long long* nlinks);
/* Apply after flb_step (BBLikeFixedBlockBdManager::Apply). */
FLB_API int flb_bb_apply(flb_bb* bb, flb_lattice* lat, void* stream);
FLB_API int flb_bb_destroy(flb_bb* bb);

#ifdef __cplusplus
}
#endif

#endif /* FLB_BOUNDARY_H_ */
