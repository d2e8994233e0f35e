// flb_pipe.cuh -- the FP16S single-block step with the next tile's sources in
// flight while the current tile collides.
//
// The direct kernel (k_pull) issues a chunk's 29 loads and then waits for them
// before it can collide; with the 128 registers the collision needs, 16 warps
// per SM do not cover the DRAM latency.  Here every warp walks its tiles of 32
// chunks (4 cells per lane) in a persistent loop and, before colliding tile t,
// starts asynchronous copies (cp.async, LDGSTS: no registers held while in
// flight) of tile t + 1's source words into a second shared-memory stage.
//
// Stage layout per warp: own[i][2 + lane] is the lane's aligned source word of
// direction i (the same word k_pull loads at cell + row_off32[i]); slots 0-1
// and 34-35 hold the chunks just before and after the tile, so the adjacent
// chunk of every lane is a neighbouring slot; fix[][lane] holds the row-end
// sources of lanes at x = 0 or x = nx-1 (the 4-byte aligned pair that contains
// the half).  Flags travel in a register loaded one tile ahead.  Rows that are
// not interior (the first and last two planes' rows) gather through the wrap
// rule from global memory.
//
// Copies.  On interior rows the 32 sources of a tile in direction i are one
// contiguous 256-byte range (rows are linear), so when rows are 16-byte
// aligned (pitch a multiple of 8: WIDE) the warp moves each direction as
// sixteen 16-byte cp.async.cg copies, which bypass L1; a 16-byte block is
// copied when either of its two chunks lies on an interior row (its neighbour
// row is then in bounds too).  Otherwise every lane copies its own 8-byte word
// (cp.async.ca), which allocates L1 lines while in flight.
//
// Waits: cp.async.wait_group waits for the thread's own copies only (no flag
// or barrier another thread must release), then __syncwarp publishes them to
// the warp.  Every copy is 16, 8 or 4 bytes from an aligned address inside
// the population array.
#pragma once

#include "flb_pull.cuh"

namespace flb {

constexpr int PIPE_WARPS = 4;   // warps per CTA
constexpr int PIPE_SLOTS = 36;  // per direction: 2 chunks before the tile, 32 lanes, 2 after
constexpr int PIPE_V = 4;       // cells per lane

// Fixup slot of direction i: the five directions with c_x = +1 take 0..4, the
// five with c_x = -1 take 5..9.
__host__ __device__ constexpr int pipe_fix_slot(int i) {
  constexpr int s[Q] = {-1, 0, 5, -1, -1, -1, -1, 1, 6, 2, 7, -1, -1, 3, 8, 4, 9, -1, -1};
  return s[i];
}

struct PipeStage {
  uint2 own[Q][PIPE_SLOTS];
  unsigned fix[10][32];
};

constexpr int pipe_smem_bytes() { return int(sizeof(PipeStage)) * 2 * PIPE_WARPS; }

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Chunk column xc (x0 = 4 xc) and row (y, z) of a lane; z >= nz past the end.
struct PipeCursor {
  unsigned xc, y, z;
};

// The directions with c_x = +1 and c_x = -1, five 5-bit fields each.
constexpr unsigned PIPE_XP = 1u | 7u << 5 | 9u << 10 | 13u << 15 | 15u << 20;
constexpr unsigned PIPE_XM = 2u | 8u << 5 | 10u << 10 | 14u << 15 | 16u << 20;

// Start the copies of one tile into stage st and load the lane's flags.  t0
// is the tile's first chunk (warp-uniform), c the lane's chunk t0 + lane.
template <bool WIDE>
__device__ __forceinline__ void pipe_issue(const StepParams& p, const Geom& g, unsigned t0,
                                           const PipeCursor& c, int lane, PipeStage& st,
                                           unsigned& flags) {
  const int x0 = int(c.xc) * PIPE_V;
  const bool inb = c.z < unsigned(g.nz);
  const bool valid = inb && x0 < g.nx;
  const unsigned cell = c.y * unsigned(g.pitch) + c.z * unsigned(g.plane) + unsigned(x0);
  if (valid) flags = __ldg(reinterpret_cast<const unsigned*>(p.flags + cell));
  const bool inter = inb && interior_row(g, int(c.y), int(c.z));
  const __half* arr = static_cast<const __half*>(p.src);
  if constexpr (WIDE) {
    const unsigned mask = __ballot_sync(0xffffffffu, inter);
    const unsigned tcell = t0 * PIPE_V;  // first cell of the tile
    const int j = lane & 15, half = lane >> 4;
    if ((mask >> (2 * j)) & 3u) {
#pragma unroll
      for (int m = 0; m < (Q + 1) / 2; ++m) {
        const int i = 2 * m + half;
        if (i < Q) {
          const unsigned off = half ? p.row_off32[2 * m + 1] : p.row_off32[2 * m];
          cp_async16(&st.own[i][2 + 2 * j], arr + (tcell + off + unsigned(8 * j)));
        }
      }
    }
    if (lane < 5 && (mask & 1u)) {  // chunks -2, -1 of the c_x = +1 directions
      const int i = int(PIPE_XP >> (5 * lane)) & 31;
      cp_async16(&st.own[i][0], arr + (tcell + p.row_off32[i] - 8u));
    } else if (lane >= 5 && lane < 10 && (mask >> 31)) {  // chunks 32, 33 of c_x = -1
      const int i = int(PIPE_XM >> (5 * (lane - 5))) & 31;
      cp_async16(&st.own[i][PIPE_SLOTS - 2], arr + (tcell + p.row_off32[i] + 128u));
    }
  }
  if (!valid || !inter) return;
  if constexpr (!WIDE) {
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      const __half* s = arr + (cell + p.row_off32[i]);
      cp_async8(&st.own[i][2 + lane], s);
      if (cx(i) > 0 && lane == 0) cp_async8(&st.own[i][1], s - PIPE_V);
      if (cx(i) < 0 && lane == 31) cp_async8(&st.own[i][PIPE_SLOTS - 2], s + PIPE_V);
    }
  }
  if (x0 == 0) {  // x = nx-1 of the row before the source row
#pragma unroll
    for (int i = 1; i < Q; ++i)
      if (cx(i) > 0) {
        const unsigned e = cell + p.row_off32[i] - unsigned(g.pitch) + unsigned(g.nx - 1);
        cp_async4(&st.fix[pipe_fix_slot(i)][lane], arr + (e & ~1u));
      }
  }
  if (g.nx - 1 - x0 < PIPE_V) {  // x = 0 of the row after the source row (an even element)
#pragma unroll
    for (int i = 1; i < Q; ++i)
      if (cx(i) < 0) {
        const unsigned e = cell + p.row_off32[i] + unsigned(g.pitch) - unsigned(x0);
        cp_async4(&st.fix[pipe_fix_slot(i)][lane], arr + e);
      }
  }
}

// Collide and store one lane's chunk from stage st.
template <int MODEL>
__device__ __forceinline__ void pipe_compute(const StepParams& p, const Geom& g,
                                             const PipeCursor& c, int lane, const PipeStage& st,
                                             unsigned flags, float omega) {
  const int x0 = int(c.xc) * PIPE_V;
  if (c.z >= unsigned(g.nz) || x0 >= g.nx) return;
  uint2 h[Q];
  if (interior_row(g, int(c.y), int(c.z))) {
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      const uint2 v = st.own[i][2 + lane];
      if (cx(i) == 0) h[i] = v;
      else if (cx(i) > 0) h[i] = hsplice_prev(st.own[i][1 + lane], v);
      else h[i] = hsplice_next(v, st.own[i][3 + lane]);
    }
    if (x0 == 0) {
      const int hi = (g.nx - 1) & 1;  // the element's half in its aligned pair
#pragma unroll
      for (int i = 1; i < Q; ++i)
        if (cx(i) > 0) {
          const unsigned w = st.fix[pipe_fix_slot(i)][lane];
          hset(h[i], 0, hi ? w >> 16 : w);
        }
    }
    const int klast = g.nx - 1 - x0;
    if (klast < PIPE_V) {
#pragma unroll
      for (int i = 1; i < Q; ++i)
        if (cx(i) < 0) {
          const unsigned w = st.fix[pipe_fix_slot(i)][lane];
#pragma unroll
          for (int k = 0; k < PIPE_V; ++k)
            if (k == klast) hset(h[i], k, w);
        }
    }
  } else {
    gather_words_wrap<PIPE_V>(static_cast<const __half*>(p.src), p.dstride, g, x0, int(c.y),
                              int(c.z), h);
  }
  const unsigned cell = c.y * unsigned(g.pitch) + c.z * unsigned(g.plane) + unsigned(x0);
  uint8_t fl[PIPE_V];
#pragma unroll
  for (int k = 0; k < PIPE_V; ++k) fl[k] = uint8_t(flags >> (8 * k));
  collide_half<MODEL, PIPE_V>(p, omega, (long long)cell, fl, h);
  __half* __restrict__ dst = static_cast<__half*>(p.dst);
#pragma unroll
  for (int i = 0; i < Q; ++i) hstore<PIPE_V>(dst + (p.dir_off32[i] + cell), h[i]);
}

#ifndef FLB_PIPE_MIN_CTAS
#define FLB_PIPE_MIN_CTAS 4
#endif

// Persistent grid: warp w of CTA b takes the tiles (b * PIPE_WARPS + w) + k * (all warps)
// of 32 consecutive chunks.  Single block (base 0), 19 * dstride < 2^32, pitch a
// multiple of 4 (of 8 for WIDE), 4 cells per lane.
template <int MODEL, bool WIDE>
__global__ void __launch_bounds__(PIPE_WARPS * 32, FLB_PIPE_MIN_CTAS)
    k_pull_pipe(const StepParams p) {
  extern __shared__ __align__(16) unsigned char pipe_smem[];
  const int lane = int(threadIdx.x) & 31, warp = int(threadIdx.x) >> 5;
  PipeStage* st = reinterpret_cast<PipeStage*>(pipe_smem) + 2 * warp;
  const Geom g{p.nx, p.ny, p.nz, p.pitch, p.plane, 0};
  const unsigned cpr = unsigned(p.pitch) / PIPE_V;
  const unsigned ny = unsigned(p.ny);
  const unsigned total = cpr * ny * unsigned(p.nz);  // < 2^32 (checked at creation)
  const unsigned step = gridDim.x * PIPE_WARPS * 32u;
  unsigned t0 = (blockIdx.x * PIPE_WARPS + unsigned(warp)) * 32u;  // first chunk of the tile
  if (t0 >= total) return;
  // the cursor advances by `step` chunks per tile: precomputed carries
  const unsigned drow = step / cpr, dxc = step - drow * cpr;
  const unsigned dz = drow / ny, dy = drow - dz * ny;
  PipeCursor c;
  {
    const unsigned q = t0 + unsigned(lane);
    const unsigned row = q / cpr;
    c.xc = q - row * cpr;
    c.z = row / ny;
    c.y = row - c.z * ny;
  }
  const float omega = float(p.omega);
  unsigned fl_next = 0;
  pipe_issue<WIDE>(p, g, t0, c, lane, st[0], fl_next);
  cp_async_commit();
  int s = 0;
  for (;;) {
    PipeCursor n = c;
    n.xc += dxc;
    const unsigned c1 = n.xc >= cpr ? 1u : 0u;
    n.xc -= c1 * cpr;
    n.y += dy + c1;
    const unsigned c2 = n.y >= ny ? 1u : 0u;
    n.y -= c2 * ny;
    n.z += dz + c2;
    const bool more = total - t0 > step;  // t0 + step < total without overflow
    const unsigned fl = fl_next;
    if (more) pipe_issue<WIDE>(p, g, t0 + step, n, lane, st[s ^ 1], fl_next);
    cp_async_commit();
    cp_async_wait<1>();
    __syncwarp();
    pipe_compute<MODEL>(p, g, c, lane, st[s], fl, omega);
    __syncwarp();
    if (!more) break;
    t0 += step;
    c = n;
    s ^= 1;
  }
  cp_async_wait<0>();
}

}  // namespace flb
