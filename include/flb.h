/* flb.h -- C ABI of the B200 D3Q19 stream-and-collide library (libflb_b200.so).
 *
 * This is the drop-in boundary for FreeLB's lattice-Boltzmann hot path.  The
 * reference exposes that path only as C++ templates (no ABI); each entry point
 * below names the reference member it replaces.  Host-side C++17 classes with
 * the reference's names (freelb_b200/cpp/freelb.h) and the Python module
 * freelb_b200 call through this header.
 *
 * Conventions (all entry points):
 *   - return FLB_OK (0) or a negative FLB_ERR_* code; nothing calls exit();
 *     flb_last_error() gives a message for the calling host thread.
 *   - plain pointers and sizes only; `stream` is a cudaStream_t passed as
 *     void* (NULL = legacy default stream).  Every device operation is
 *     ordered on that stream.  Host buffers are owned by the caller; device
 *     memory is owned by the handle.  Calls that read or write host memory
 *     synchronise `stream` before returning.
 *   - a handle is used from one host thread at a time.
 *   - cell indexing is the reference's: id = x + nx*(y + ny*z) over the stored
 *     mesh (interior + overlap layer), x fastest (BasicBlock::getIndex,
 *     src/geometry/basic_geometry.h:310-330); populations are 19 arrays of N
 *     cells in D3Q19 order (src/lbm/lattice_set.h:263-266), each array in the
 *     logical (post-rotation) order of CyclicArray::operator[]
 *     (src/data_struct/field.h:626-629).
 */
#ifndef FLB_H_
#define FLB_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FLB_ABI_VERSION 1

#if defined(__GNUC__)
#define FLB_API __attribute__((visibility("default")))
#else
#define FLB_API
#endif

/* status codes */
#define FLB_OK 0
#define FLB_ERR_INVALID (-1)     /* bad argument or descriptor */
#define FLB_ERR_CUDA (-2)        /* a CUDA runtime call failed */
#define FLB_ERR_OOM (-3)         /* device allocation failed */
#define FLB_ERR_TIMEOUT (-4)     /* a bounded device wait gave up (flb_device_status) */
#define FLB_ERR_NUMERIC (-5)     /* non-finite population detected (flb_check_finite) */
#define FLB_ERR_UNSUPPORTED (-6) /* combination not built */
#define FLB_ERR_STATE (-7)       /* call not valid in the handle's state */

/* population storage in HBM */
#define FLB_STORAGE_FP32 0  /* f_i as float */
#define FLB_STORAGE_FP16S 1 /* f_i - rho0*w_i as half, float arithmetic */
#define FLB_STORAGE_FP64 2  /* f_i as double, double arithmetic */
#define FLB_STORAGE_FP32S 3 /* f_i - rho0*w_i as float, float arithmetic on the deviations */

/* bulk collision model (the policy bound to FLB_OP_BULK) */
#define FLB_MODEL_BGK 0 /* collision::BGK<moment::rhoU, equilibrium::SecondOrder> */
#define FLB_MODEL_MRT 1 /* collision::MRT_Feq_RhoU, D3Q19 Gram-Schmidt basis */
#define FLB_MODEL_LES 2 /* collision::SmagorinskyBGK<moment::rhoU<CELL,true>, ...> */
#define FLB_MODEL_BRINKMAN 3 /* collision::BGKForce with Guo drag F = -alpha u (ALPHA field) */

/* per-flag operations (the policy of a tmp::Key_TypePair) */
#define FLB_OP_NONE 0       /* no collision (void cells) */
#define FLB_OP_BULK 1       /* the bulk model above */
#define FLB_OP_BOUNCEBACK 2 /* collision::BounceBack (full-way swap) */
#define FLB_OP_MOVINGWALL 3 /* collision::BounceBackMovingWall (RHO, VELOCITY fields) */
#define FLB_OP_FIELD_BGK 4  /* collision::BGK<moment::useFieldrhoU, SecondOrder> */

/* host buffer element types */
#define FLB_DTYPE_F32 0
#define FLB_DTYPE_F64 1

/* fields */
#define FLB_FIELD_RHO 0      /* RHO<T>: N values */
#define FLB_FIELD_VELOCITY 1 /* VELOCITY<T,3>: N x 3 values, AoS like Vector<T,3> */
#define FLB_FIELD_ALPHA 2    /* Brinkman porosity alpha (FLB_MODEL_BRINKMAN): N values */

#define FLB_MAX_TASKS 8

/* One block lattice.  Replaces the template arguments and constructor inputs
 * of BlockLatticeManager<T, D3Q19<T>, TypePack<RHO, VELOCITY, POP>>
 * (src/data_struct/block_lattice.h:234-433) plus the NSTask selector
 * (src/utils/tmp.h:283-309): tasks are tried in order and a cell takes the op
 * of the first task whose key shares a bit with its flag. */
typedef struct flb_lattice_desc {
  int nx, ny, nz;         /* stored cells per axis (interior + overlap) */
  int storage;            /* FLB_STORAGE_* */
  int model;              /* FLB_MODEL_* for FLB_OP_BULK cells */
  double omega;           /* 1/tau: BlockLattice::Omega (block_lattice.hh:27-35) */
  double smagorinsky;     /* Cs: SMAGORINSKY<T> (collisionLES.h:45) */
  double mrt_rates[19];   /* s_k in moment order; entries 9,11,13,14,15 use omega */
  double rho0;            /* reference density (init value, FP16S shift) */
  int ntasks;             /* number of (key, op) pairs, <= FLB_MAX_TASKS */
  uint8_t task_keys[FLB_MAX_TASKS];
  uint8_t task_ops[FLB_MAX_TASKS];
} flb_lattice_desc;

typedef struct flb_lattice flb_lattice;

/* One block of a multi-block lattice (a BlockLattice of BlockLatticeManager,
 * src/data_struct/block_lattice.h:234-433; geometry of Block3D,
 * src/geometry/block_geometry3d.h).  Sizes include the one-cell overlap. */
typedef struct flb_block_desc {
  int nx, ny, nz; /* stored cells per axis (interior + 2*overlap) */
  int ox, oy, oz; /* global stored index of the block's local cell (0,0,0) */
  double omega;   /* 1/tau of this block; 0 = the lattice descriptor's omega */
} flb_block_desc;

/* multi-block modes */
#define FLB_BLOCKS_INDEPENDENT 0 /* separate lattices stepped together (ensemble) */
#define FLB_BLOCKS_HALO 1        /* blocks of one domain: device halo after each step */

/* Library identification: ABI version and the sm arch the kernels target. */
FLB_API int flb_version(int* abi_version, int* sm_arch);

/* Message for the last failed call on this host thread (never NULL). */
FLB_API const char* flb_last_error(void);

/* Fill `d` with the lid-driven cavity defaults: D3Q19 BGK, FP32, tasks
 * {2: bulk, 4: bounce-back, 8: moving wall} as in
 * benchmarks/cavity3d/cavity3d.cpp:173-182, rho0 = 1, MRT rates 1.2. */
FLB_API int flb_desc_default(flb_lattice_desc* d, int nx, int ny, int nz, double tau);

/* Allocate a block lattice on the current device.  Replaces the
 * BlockLatticeManager constructor (block_lattice.hh:651-681); populations are
 * initialised to rho0*w_i, RHO to rho0, VELOCITY to 0, flags to 1 (void). */
FLB_API int flb_create(const flb_lattice_desc* desc, flb_lattice** out);
FLB_API int flb_destroy(flb_lattice* lat);

/* Allocate `nblocks` blocks in one handle (desc->nx/ny/nz are ignored).
 * Every block keeps the reference's own streaming (periodic over the block's
 * linear index).  FLB_BLOCKS_HALO: after each step, overlap cells receive the
 * populations that cross into the block from the neighbour owning that cell,
 * as BlockLatticeManager::NormalCommunicate (block_lattice.hh:1419-1430,
 * 1668-1685; directions of getCommPopDir, communicator.h:76-150), on the
 * device.  FLB_BLOCKS_INDEPENDENT: blocks are unrelated lattices (the batched
 * ensemble), each with its own omega.  All blocks advance in one launch per
 * step through a tile work table. */
FLB_API int flb_create_blocks(const flb_lattice_desc* desc, int nblocks,
                              const flb_block_desc* blocks, int mode, flb_lattice** out);
FLB_API int flb_block_count(const flb_lattice* lat, int* nblocks);
/* number of halo copy records (overlap cells fed by a neighbour) */
FLB_API int flb_halo_count(const flb_lattice* lat, long long* nrecords);

/* Halo exchange of an FLB_BLOCKS_HALO handle.  FLB_HALO_NORMAL (default):
 * NormalCommunicate, the directions crossing into the block.  FLB_HALO_FULL:
 * NormalFullCommunicate / NormalAllCommunicate (block_lattice.hh:1448-1503,
 * 1687-1720): all 19 populations of every overlap cell from its owner (with
 * one overlap layer the first layer is all of them, so the two coincide). */
#define FLB_HALO_NORMAL 0
#define FLB_HALO_FULL 1
FLB_API int flb_set_halo_mode(flb_lattice* lat, int mode);

/* Blocks on several GPUs (one process per GPU).  The domain is a global list
 * of blocks, each owned by a rank; a rank's handle is an FLB_BLOCKS_HALO handle
 * holding the blocks it owns, in global order.  The handle's own halo copies
 * between its local blocks after each step; the records whose source block
 * lives on another rank (the same NormalCommunicate / NormalFullCommunicate
 * copies, block_lattice.hh:1419-1503) become per-peer exchanges: after
 * flb_step, flb_exchange_pack gathers the populations a peer needs into a
 * device buffer, the caller moves the buffers (NCCL send / recv), and
 * flb_exchange_unpack scatters a peer's buffer into the overlap slots, before
 * the next flb_step.  Every rank enumerates the global records in the same
 * order (block, overlap cell z-y-x, direction), so a sender's buffer matches
 * its receiver's slots element for element.  Buffers hold storage elements
 * (2 / 4 / 8 bytes for FP16S / FP32 / FP64).
 *
 * The plan follows the handle's halo mode at creation (flb_set_halo_mode
 * first); pack / unpack refuse a handle whose mode changed since.
 *
 * flb_exchange_plan is host-only (no device or handle): the peers of my_rank
 * and the element counts it sends to and receives from each, sorted by peer
 * rank; max_peers bounds the output arrays. */
typedef struct flb_exchange flb_exchange;
FLB_API int flb_exchange_plan(int nglobal, const flb_block_desc* blocks, const int* owner_rank,
                              int my_rank, int halo_mode, int max_peers, int* npeers,
                              int* peer_ranks, long long* send_counts, long long* recv_counts);
FLB_API int flb_exchange_create(flb_lattice* lat, int nglobal, const flb_block_desc* blocks,
                                const int* owner_rank, int my_rank, flb_exchange** out);
FLB_API int flb_exchange_peers(const flb_exchange* ex, int max_peers, int* npeers,
                               int* peer_ranks, long long* send_counts, long long* recv_counts);
FLB_API int flb_exchange_pack(flb_exchange* ex, flb_lattice* lat, int peer_rank, void* device_buf,
                              void* stream);
FLB_API int flb_exchange_unpack(flb_exchange* ex, flb_lattice* lat, int peer_rank,
                                const void* device_buf, void* stream);
FLB_API int flb_exchange_destroy(flb_exchange* ex);

/* Rebind the per-flag task list and the bulk model (the NSTask type of
 * ApplyCellDynamics<NSTask>, src/utils/tmp.h:283-309): tasks are tried in order,
 * a cell takes the op of the first task whose key shares a bit with its flag. */
FLB_API int flb_set_tasks(flb_lattice* lat, int ntasks, const uint8_t* keys, const uint8_t* ops,
                          int model);

/* Device bytes held by the handle. */
FLB_API int flb_memory_bytes(const flb_lattice* lat, size_t* bytes);

/* Flag field (uint8 per cell).  Replaces BlockFieldManager<FLAG>::copyToDevice
 * (src/data_struct/field_struct.h:176-177). */
FLB_API int flb_upload_flags(flb_lattice* lat, const uint8_t* host_flags, void* stream);
FLB_API int flb_download_flags(flb_lattice* lat, uint8_t* host_flags, void* stream);

/* Populations, 19 x N in logical order, host dtype FLB_DTYPE_*.  Replaces
 * getField<POP<T,19>>() access and copyToDevice/copyToHost of POP. */
FLB_API int flb_upload_pops(flb_lattice* lat, const void* host, int host_dtype, void* stream);
FLB_API int flb_download_pops(flb_lattice* lat, void* host, int host_dtype, void* stream);

/* RHO (N) or VELOCITY (3N, AoS) field.  Replaces getField<RHO>/getField<VELOCITY>
 * with copyToDevice/copyToHost. */
FLB_API int flb_upload_field(flb_lattice* lat, int field, const void* host, int host_dtype,
                     void* stream);
FLB_API int flb_download_field(flb_lattice* lat, int field, void* host, int host_dtype, void* stream);

/* f_i = rho0*w_i on every cell (block_lattice.hh:673-680). */
FLB_API int flb_init_equilibrium(flb_lattice* lat, double rho0, void* stream);

/* n time steps, each the fused equivalent of
 *   ApplyCellDynamics<NSTask>(FlagFM); Stream();
 * (block_lattice.hh:72-92 + 64-70; CUDA twins block_lattice.hh:210-231).
 * Streaming keeps the reference's periodic wrap over the linear cell index. */
FLB_API int flb_step(flb_lattice* lat, int nsteps, void* stream);

/* Write RHO and VELOCITY from the current populations on cells whose flag
 * shares a bit with `key`: ApplyCellDynamics<TaskSelector<Key_TypePair<key,
 * moment::rhoU<CELL,true>>>> (src/lbm/moment.h:382-398). */
FLB_API int flb_compute_rhou(flb_lattice* lat, uint8_t key, void* stream);

/* FP64 sums over cells whose flag shares a bit with `key`:
 * out[0] = sum rho, out[1..3] = sum rho*u (mass and momentum).  Summed in a
 * fixed order: the same state gives the same bits on every call. */
FLB_API int flb_reduce_conservation(flb_lattice* lat, uint8_t key, double out[4], void* stream);

/* Steady-state check: max |u - u_prev| over cells matching `key` since the
 * previous call (first call: against u = 0), FP64 reduction.  Replaces
 * BlockLattice::getToleranceU (block_lattice.hh:266-288). */
FLB_API int flb_tolerance_u(flb_lattice* lat, uint8_t key, double* max_du, void* stream);

/* Non-finite check of the populations of every cell whose flag selects an
 * op (void cells, which only carry the reference's wrapped values, are left
 * out: over long FP16S runs such values can leave the binary16 range without
 * touching any cell that is updated): *bad = number of non-finite values;
 * returns FLB_ERR_NUMERIC when that number is not zero. */
FLB_API int flb_check_finite(flb_lattice* lat, uint64_t* bad, void* stream);

/* Device pointers for zero-copy consumers: populations (current buffer),
 * flags, RHO, VELOCITY (SoA planes), with the padded layout
 * (pitch_x elements per row, rows per plane = ny, plane stride, direction
 * stride, all in elements). */
typedef struct flb_layout {
  int nx, ny, nz;
  int pitch_x;
  size_t plane;      /* pitch_x * ny */
  size_t dir_stride; /* elements between consecutive directions */
  int elem_bytes;    /* population element size */
} flb_layout;
FLB_API int flb_get_layout(const flb_lattice* lat, flb_layout* layout);
FLB_API int flb_device_pointers(flb_lattice* lat, void** pops, void** flags, void** rho, void** vel);

/* The same mass and momentum sums as flb_reduce_conservation, for callers that
 * may not allocate GPU memory.  This entry point has no counterpart in the
 * reference (FreeLB has no GPU reduction of this kind).
 *
 * Who needs it: a program whose GPU memory is handed out only by its own
 * caching pool (so that memory accounting stays exact and no component
 * triggers the implicit synchronisation a cudaMalloc/cudaFree can cause), or a
 * latency-bound loop that must not wait on an allocation, cannot let this
 * library call cudaMalloc behind its back.  Here the caller passes its own
 * device pointers -- populations `pops` and `flags` of ONE block laid out as
 * `layout` describes (flb_get_layout / flb_device_pointers give both for a
 * single-block handle; on a multi-block handle they describe block 0 only),
 * `storage` (FLB_STORAGE_*) and `rho0` (the FP16S / FP32S shift density) --
 * and a host array `out` for the four sums; the function allocates nothing.
 * `pops`, `flags` and `stream` must belong to the current device
 * (FLB_ERR_INVALID otherwise).
 *
 * Its scratch is a fixed device array inside the library: 128 KiB, held on
 * every GPU that loads the library until the process exits.  That bounds the
 * lattice to 268,435,456 padded cells (layout->plane * layout->nz); larger
 * layouts are rejected with FLB_ERR_INVALID.  The first call on a device looks
 * up the array's device address for that device and keeps it for the process,
 * so do not call it on a device after a cudaDeviceReset of that device.  Every
 * call on a device uses the same scratch and it keeps the previous call's
 * contents; nothing in it needs to start at zero (each call writes every slot
 * it reads), but calls whose work overlaps on the GPU (different streams,
 * different host threads) race on it and must be serialised by the caller.
 * `stream` orders the work; the call copies the sums to `out` and
 * synchronises `stream` before returning, so it cannot be called while
 * `stream` is being captured into a CUDA graph. */
FLB_API int flb_reduce_conservation_noalloc(const void* pops, const uint8_t* flags,
                                            const flb_layout* layout, int storage, double rho0,
                                            uint8_t key, double out[4], void* stream);

/* Per-block transfers of a multi-block handle (the functions above act on
 * block 0).  Replace BlockFieldManager::getBlockField(i) and
 * BlockLatticeManager::getBlockLat(i).getField<...>() access. */
FLB_API int flb_upload_flags_block(flb_lattice* lat, int block, const uint8_t* host,
                                   void* stream);
FLB_API int flb_download_flags_block(flb_lattice* lat, int block, uint8_t* host, void* stream);
FLB_API int flb_upload_pops_block(flb_lattice* lat, int block, const void* host, int host_dtype,
                                  void* stream);
FLB_API int flb_download_pops_block(flb_lattice* lat, int block, void* host, int host_dtype,
                                    void* stream);
FLB_API int flb_upload_field_block(flb_lattice* lat, int block, int field, const void* host,
                                   int host_dtype, void* stream);
FLB_API int flb_download_field_block(flb_lattice* lat, int block, int field, void* host,
                                     int host_dtype, void* stream);

/* Launch shape of the stream-collide kernel: tile_y warps (rows) per CTA
 * (1, 2, 4 or 8), ctas_per_sm CTAs per SM for a persistent grid over the tile
 * work table (0 = one CTA per tile), and cells_per_thread (2 or 4 for FP32
 * and FP16S, 1 or 2 for FP64; 0 = default 2 / 4 / 2).  ctas_per_sm = -1
 * selects, for single-block FP16S handles, the async-copy pipeline: a
 * persistent grid (as many 4-warp CTAs as fit per SM) whose warps copy the next
 * tile's sources into shared memory while the current tile collides; it runs 4
 * cells per thread and ignores tile_y (FLB_ERR_UNSUPPORTED elsewhere).
 * ctas_per_sm = -2 / -3 selects, for single-block FP16S handles whose rows
 * start on 16-byte boundaries, the bulk-copy kernel: one CTA per SM in which
 * one thread stages each tile's 19 source ranges and flags in shared memory
 * with bulk asynchronous copies (3 / 5 stages) while 15 warps collide the
 * staged tiles; 4 cells per thread (cells_per_thread 4 or 0; the staged
 * warps run 2-cell chunks).  Its waits are bounded (flb_set_wait_limit;
 * flb_device_status reports one that gave up).
 * Defaults: tile_y 4, no persistent grid. */
FLB_API int flb_set_launch(flb_lattice* lat, int tile_y, int ctas_per_sm, int cells_per_thread);
FLB_API int flb_get_launch(const flb_lattice* lat, int* tile_y, int* ctas_per_sm,
                           int* cells_per_thread);

/* Device-side failure detection (no reference counterpart: the reference's
 * CUDA path exit()s on errors, src/utils/cuda_device.h:37-44).  Kernels whose
 * threads wait on one another (the bulk-copy kernel) bound every wait; a wait
 * that runs past the limit records FLB_ERR_TIMEOUT in the handle's status word
 * and the kernel ends early, leaving that step incomplete.
 * flb_set_wait_limit sets the bound of one wait (seconds, default 2, at most
 * 60).  flb_device_status synchronises `stream` and returns FLB_OK, or the
 * recorded code (which it clears). */
FLB_API int flb_set_wait_limit(flb_lattice* lat, double seconds);
FLB_API int flb_device_status(flb_lattice* lat, void* stream);
/* Population snapshots (checkpoint / resume; no reference counterpart: FreeLB
 * only writes VTK output and never reads populations back).  A snapshot is a
 * 64-byte header followed by the populations of every block in the device
 * layout, exactly as stored, so a restored handle continues bit for bit.
 * flb_snapshot_bytes gives its size.  flb_snapshot_save copies the current
 * state into `dst` (device memory, or host memory: pinned for an asynchronous
 * copy), ordered on `stream`; `dst` must stay valid until the stream reaches
 * it.  flb_snapshot_restore checks the header (synchronising `stream` for
 * it) and copies the populations back: FLB_ERR_INVALID for a buffer that is
 * not a snapshot, too short, or taken from a handle of another storage or
 * block geometry.  Flags and fields are inputs and are not part of it. */
FLB_API int flb_snapshot_bytes(const flb_lattice* lat, size_t* bytes);
FLB_API int flb_snapshot_save(flb_lattice* lat, void* dst, size_t cap, void* stream);
FLB_API int flb_snapshot_restore(flb_lattice* lat, const void* src, size_t bytes, void* stream);

/* Rounding of FP16S stores (no reference counterpart: the reference stores
 * populations in T).  FLB_ROUND_NEAREST rounds every stored deviation to the
 * nearest binary16 value; FLB_ROUND_STOCHASTIC rounds it up or down with the
 * probabilities that make the stored value exact on average (the sm_100a
 * cvt.rs conversion; the random bits come from a hash of binary16 values the
 * cell pulled, so runs are reproducible and every kernel gives the same
 * bits).  Round to nearest can make the same error step after step where the
 * flow changes slowly, and in MRT that error accumulates (the 512^3 cavity
 * ends 1.17e-3 from FP64 after 2000 steps, 2.2e-4 with stochastic rounding).
 * FLB_ROUND_DEFAULT (the default) is stochastic for MRT and round to nearest
 * otherwise; other storages ignore the mode.  flb_get_rounding returns the
 * mode in effect (NEAREST or STOCHASTIC). */
#define FLB_ROUND_DEFAULT (-1)
#define FLB_ROUND_NEAREST 0
#define FLB_ROUND_STOCHASTIC 1
FLB_API int flb_set_rounding(flb_lattice* lat, int mode);
FLB_API int flb_get_rounding(const flb_lattice* lat, int* mode);

/* Failure-detection test hook: while `tile` >= 0, the bulk-copy kernel never
 * signals that tile's stage, so every wait on it runs out after the wait limit
 * (and the waits behind it after theirs): the path flb_device_status reports,
 * exercised without a device fault.  -1 (the default) turns it off. */
FLB_API int flb_test_withhold_tile(flb_lattice* lat, long long tile);

/* Autotuner: times every candidate launch shape for `trial_steps` steps on
 * `stream` (CUDA events) and keeps the fastest.  The trial steps are real
 * time steps: the lattice advances by *steps_taken.  best_ms = time per step
 * of the winner. */
FLB_API int flb_autotune(flb_lattice* lat, int trial_steps, void* stream, int* tile_y,
                         int* ctas_per_sm, int* cells_per_thread, double* best_ms,
                         int* steps_taken);

/* CUDA-graph stepping: the two-step ping-pong cycle (stream-collide, halo) is
 * captured once per handle and replayed; equivalent to flb_step. */
FLB_API int flb_step_graph(flb_lattice* lat, int nsteps, void* stream);

/* Objective J = sum over bulk cells of |u|^2 at the current state, with the
 * forced moment u = sum c f / (rho + alpha/2) (alpha = 0 without a porosity
 * field), reduced in FP64 in a fixed order (the same state gives the same
 * bits, so central differences of J are not swamped by summation order). */
FLB_API int flb_objective_u2(flb_lattice* lat, double* J, void* stream);

/* Discrete adjoint of the step (no reference counterpart: the reference has no
 * differentiation).  Single-block handles, FP32, FP32S or FP64 storage, ops
 * none / bulk (BGK, BRINKMAN or MRT) / bounce-back / moving wall.  FP32S keeps
 * the forward trajectory within ~1e-7 of an FP64 run where FP32 storage of f
 * drifts by ~1e-5, which is what a per-cell gradient needs.
 * flb_adjoint_forward advances nsteps from the current state, keeping a copy of
 * the state every `checkpoint_every` steps, and returns J at the end.
 * flb_adjoint_backward returns dJ/dalpha (per cell, N doubles in reference
 * order; may be NULL), dJ/dtau and dJ/du_lid (x-velocity of the moving-wall
 * cells), accumulated in FP64; the states between checkpoints are recomputed.
 * The lattice keeps the forward end state.  flb_adjoint_forward allocates all
 * device memory of the pair (ceil(nsteps / checkpoint_every) checkpoints and
 * checkpoint_every - 1 recompute slots of the population size, two adjoint
 * arrays, the dJ/dalpha array), so flb_adjoint_backward allocates nothing;
 * a later flb_adjoint_forward with the same nsteps / checkpoint_every reuses
 * them, and flb_adjoint_release frees them. */
FLB_API int flb_adjoint_forward(flb_lattice* lat, int nsteps, int checkpoint_every, double* J,
                                void* stream);
FLB_API int flb_adjoint_backward(flb_lattice* lat, double* dJ_dalpha, double* dJ_dtau,
                                 double* dJ_dulid, void* stream);
FLB_API int flb_adjoint_release(flb_lattice* lat);

#ifdef __cplusplus
}
#endif

#endif /* FLB_H_ */
