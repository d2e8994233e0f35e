// flb_tma.cuh -- FP16S stream-and-collide with the sources staged in shared
// memory by bulk asynchronous copies (TMA, cp.async.bulk) on mbarriers.
//
// Why: the direct FP16S kernel (pull_chunk_half32) keeps its 29 loads per
// thread in registers while they are in flight, so its 128-register pair
// collision runs at 16 warps per SM and the warps alternate between a load
// phase and a long compute phase: latency-bound at ~78 % of the HBM copy rate.
// Here the loads leave the compute warps entirely.
//
// Layout.  A persistent CTA per SM (512 threads) walks tiles of TMA_CELLS
// consecutive cells of the padded linear index (rows may split between tiles:
// the addressing is linear).  Warp 0 is the producer: its lane 0 copies, for
// tile t, the 19 source ranges [t*TMA_CELLS + off_i - TMA_HALO,
// t*TMA_CELLS + off_i + TMA_CELLS + TMA_HALO) (off_i = -c_y pitch - c_z plane,
// the source row of direction i) and the tile's flags into one stage of a ring
// of NS stages, each copy one cp.async.bulk completing on the stage's "full"
// mbarrier.  Warps 1..15 are consumers: thread (w, l) owns chunk
// c = 32 (w - 1) + l of the tile, CV = 2 or 4 cells (one chunk per thread and
// tile: a second one made the compiler keep values live across both and
// spill), reads the chunk's 19 words from the stage exactly as
// the direct kernel reads them from global memory (own word, the adjacent word
// for the x-shifted directions, the row-end fixups, all inside the TMA_HALO
// margins), collides with collide_half and stores to global memory; then the
// warp releases the stage on its "empty" mbarrier.  The result is the direct
// kernel's bit for bit: same words, same collision, same stores.
//
// Tiles that touch the block's first or last ny + 3 rows (where the reference's
// linear wrap needs the general rule) and would read outside the array carry
// no copies: their consumers take the direct kernel's path for their chunks.
//
// Requirements (tma_supported): single-block FP16S handle with 32-bit offsets,
// pitch a multiple of 8 halves (16-byte aligned rows, so every range starts on
// a 16-byte boundary) and pitch - nx <= 16 (row-end sources inside the margins).
//
// Every mbarrier wait is bounded in time (TmaParams::wait_ns on the global
// timer); a wait that gives up writes TMA_TIMEOUT to *status and the thread
// leaves the loop.  The producer thread leaves last: it first waits for the
// copies it issued to land (bounded by drain_ns, never shorter than a second),
// so no copy is in flight into the shared memory of a CTA that has ended.  The
// host reads the status with flb_device_status.  No wait depends on another
// CTA.
#pragma once

#include <cstdint>

#include "flb_pull.cuh"

namespace flb {

constexpr int TMA_THREADS = 512;
constexpr int TMA_CONSUMER_WARPS = TMA_THREADS / 32 - 1;  // 15
constexpr int TMA_CHUNKS = 32 * TMA_CONSUMER_WARPS;      // 480 chunks per tile
constexpr int TMA_HALO = 24;                             // halves before / after a range

// Tile geometry for chunks of CV cells (2 or 4): TMA_CHUNKS chunks per tile.
template <int CV>
struct TmaTile {
  static constexpr int cells = CV * TMA_CHUNKS;        // 960 / 1920 cells per tile
  static constexpr int dirh = cells + 2 * TMA_HALO;    // halves per direction range
  static constexpr int dirb = 2 * dirh;                // bytes per direction range
  static constexpr int stage = Q * dirb + cells;       // + the tile's flags
  static_assert(dirb % 16 == 0 && stage % 16 == 0 && (2 * TMA_HALO) % 16 == 0,
                "bulk copies need 16-byte sizes and destinations");
  static_assert((2 * cells) % 16 == 0, "tile starts stay 16-byte aligned");
};

template <int NS, int CV>
constexpr int tma_smem_bytes() {
  return NS * TmaTile<CV>::stage + 2 * NS * 8;  // stages, then the full / empty mbarriers
}

// Written to the status word by a wait that gave up (FLB_ERR_TIMEOUT).
constexpr int TMA_TIMEOUT = -4;

struct TmaParams {
  long long ntiles;
  int* status;                 // device word, TMA_TIMEOUT after a wait gave up
  unsigned long long wait_ns;  // bound of one mbarrier wait of the pipeline
  unsigned long long drain_ns; // bound of the producer's wait for its last copies
  long long withhold;          // failure-detection test: this tile is never signalled (-1: none)
  long long staged_lo, staged_hi;  // the staged tiles: t in [staged_lo, staged_hi]
};

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return unsigned(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(b)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(b)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t* b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(b)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_addr(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Wait for the phase of the given parity, at most limit_ns; false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, unsigned parity,
                                          unsigned long long limit_ns) {
  if (mbar_try(b, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (;;) {
    for (int k = 0; k < 16; ++k)
      if (mbar_try(b, parity)) return true;
    if (global_ns() - t0 > limit_ns) return false;
  }
}
// One bulk copy global -> this CTA's shared memory, completing on mbarrier b.
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, unsigned bytes,
                                          uint64_t* b) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(b))
      : "memory");
}

// Tiles whose ranges stay inside the block and away from the wrap rows are
// those whose rows lie in [ny + 3, ny nz - ny - 4]: one contiguous range of
// tiles, computed on the host (tma_staged_range) so that no thread divides.
__host__ __device__ __forceinline__ void tma_staged_range(long long cells, long long pitch,
                                                          long long ny, long long nz,
                                                          long long& lo, long long& hi) {
  lo = ((ny + 3) * pitch + cells - 1) / cells;
  const long long num = (ny * nz - ny - 3) * pitch - cells;
  hi = num >= 0 ? num / cells : -1;
}
__device__ __forceinline__ bool tma_tile_staged(const TmaParams& tp, long long t) {
  return t >= tp.staged_lo && t <= tp.staged_hi;
}

// The words of CV-cell chunk c (first cell at x0 of its row) of a staged tile
// in stage `sb`: the same words gather_words_dir reads from global memory.
template <int CV>
__device__ __forceinline__ void gather_words_stage(const StepParams& p, const __half* sb, int c,
                                                   int x0, typename HWord<CV>::type (&h)[Q]) {
  using W = typename HWord<CV>::type;
  constexpr int DIRH = TmaTile<CV>::dirh;
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const W* own = reinterpret_cast<const W*>(sb + i * DIRH + TMA_HALO + CV * c);
    const W v = own[0];
    if (cx(i) == 0) h[i] = v;
    else if (cx(i) > 0) h[i] = hsplice_prev(own[-1], v);
    else h[i] = hsplice_next(v, own[1]);
  }
  const unsigned short* s16 = reinterpret_cast<const unsigned short*>(sb);
  if (x0 == 0) {  // x = nx-1 of the row before the source row
#pragma unroll
    for (int i = 1; i < Q; ++i)
      if (cx(i) > 0) hset(h[i], 0, s16[i * DIRH + TMA_HALO + CV * c - p.pitch + p.nx - 1]);
  }
  const int klast = p.nx - 1 - x0;
  if (klast >= 0 && klast < CV) {  // x = 0 of the row after the source row
#pragma unroll
    for (int i = 1; i < Q; ++i)
      if (cx(i) < 0) {
        const unsigned e = s16[i * DIRH + TMA_HALO + CV * c + p.pitch - x0];
#pragma unroll
        for (int k = 0; k < CV; ++k)
          if (k == klast) hset(h[i], k, e);
      }
  }
}

// Chunks of unstaged tiles: the direct kernel's path, out of line so that its
// registers do not weigh on the staged path.
template <int MODEL, int CV>
__device__ __noinline__ void tma_direct_chunk(const StepParams& p, float omega, int x0,
                                              unsigned row, unsigned cell) {
  pull_chunk_half32<MODEL, CV>(p, Geom{p.nx, p.ny, p.nz, p.pitch, p.plane, 0}, omega, x0, row,
                               cell);
}

template <int MODEL, int NS, int CV>
__global__ void __launch_bounds__(TMA_THREADS, 1)
    k_pull_tma(const __grid_constant__ StepParams p, const TmaParams tp) {
  constexpr int TMA_CELLS = TmaTile<CV>::cells, TMA_DIRB = TmaTile<CV>::dirb,
                TMA_STAGE = TmaTile<CV>::stage;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + NS * TMA_STAGE);
  uint64_t* empty = full + NS;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < NS; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], TMA_CONSUMER_WARPS);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const long long ntiles = tp.ntiles;
  const unsigned cells_total = unsigned(p.plane) * unsigned(p.nz);

  if (warp == 0) {
    if (lane != 0) return;
    // producer: stage k % NS of the k-th tile of this CTA
    const __half* src = static_cast<const __half*>(p.src);
    long long k = 0;
    bool ok = true;
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x, ++k) {
      const int s = int(k % NS);
      const unsigned use = unsigned(k / NS);
      if (use > 0 && !mbar_wait(&empty[s], (use - 1) & 1u, tp.wait_ns)) {
        ok = false;
        break;
      }
      unsigned char* st = smem + s * TMA_STAGE;
      if (t == tp.withhold) {
        // nothing arrives on this stage: its consumers' waits run out
      } else if (tma_tile_staged(tp, t)) {
        mbar_arrive_tx(&full[s], unsigned(TMA_STAGE));
        const long long c0 = t * TMA_CELLS;
#pragma unroll 1
        for (int i = 0; i < Q; ++i)
          bulk_copy(st + i * TMA_DIRB, src + (c0 + p.row_off[i] - TMA_HALO), TMA_DIRB, &full[s]);
        bulk_copy(st + Q * TMA_DIRB, p.flags + c0, TMA_CELLS, &full[s]);
      } else {
        mbar_arrive(&full[s]);  // consumers take the direct path
      }
    }
    if (!ok) atomicExch(tp.status, TMA_TIMEOUT);
    // the last NS stages armed (earlier ones were released by the consumers,
    // so their copies have landed): wait for them before this thread leaves
    const long long issued = k;
    for (long long j = issued > NS ? issued - NS : 0; j < issued; ++j) {
      const int s = int(j % NS);
      if (!mbar_wait(&full[s], unsigned(j / NS) & 1u, tp.drain_ns))
        atomicExch(tp.status, TMA_TIMEOUT);
    }
    return;
  }

  // consumers
  const float omega = float(p.omega);
  const unsigned cpr = unsigned(p.pitch) / CV;
  long long k = 0;
  for (long long t = blockIdx.x; t < ntiles; t += gridDim.x, ++k) {
    const int s = int(k % NS);
    if (!mbar_wait(&full[s], unsigned(k / NS) & 1u, tp.wait_ns)) {
      if (lane == 0) atomicExch(tp.status, TMA_TIMEOUT);
      return;
    }
    const int c = (warp - 1) * 32 + lane;
    const unsigned cell = unsigned(t) * unsigned(TMA_CELLS) + unsigned(CV * c);
    const unsigned q = cell / CV;
    const unsigned row = p.cpr_m ? __umulhi(q, p.cpr_m) >> (p.cpr_s - 1) : q;
    const int x0 = int(q - row * cpr) * CV;
    if (cell < cells_total && x0 < p.nx) {
      if (tma_tile_staged(tp, t)) {
        const unsigned char* st = smem + s * TMA_STAGE;
        typename HWord<CV>::type h[Q];
        gather_words_stage<CV>(p, reinterpret_cast<const __half*>(st), c, x0, h);
        uint8_t fl[CV];
        load_flags<CV>(st + Q * TMA_DIRB + CV * c, fl);
        collide_half<MODEL, CV>(p, omega, (long long)cell, fl, h);
#pragma unroll
        for (int i = 0; i < Q; ++i)
          hstore<CV>(static_cast<__half*>(p.dst_dir[i]) + cell, h[i]);
      } else {
        tma_direct_chunk<MODEL, CV>(p, omega, x0, row, cell);
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
  }
}

}  // namespace flb
