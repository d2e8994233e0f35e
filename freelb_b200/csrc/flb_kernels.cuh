// flb_kernels.cuh -- fused stream-and-collide and helper kernels (sm_100a).
//
// HBM layout of one block lattice (all arrays padded the same way):
//   cell (x,y,z) -> x + y*pitch + z*plane, pitch = nx rounded up to 32
//   elements (rows start on 128-byte boundaries for FP32), plane = pitch*ny;
//   population i lives at pops + i*dstride + cell (structure of arrays), with
//   dstride = plane*nz rounded up to 64 elements.
// The reference keeps the same SoA split (GenericFieldBase, field.h:1419-1575)
// on an unpadded mesh; padding is invisible at the C ABI, which converts to
// and from the reference's linear order on upload/download.
//
// Streaming is a push from two ping-pong buffers: a thread loads the 19
// populations of its own cell (aligned, coalesced), applies the op selected by
// the cell's flag, and writes population i to the cell Delta_i away in the
// other buffer.  Stored state between launches is therefore exactly the
// reference's post-stream state.  The reference streams by rotating each
// direction array as a whole (CyclicArray::rotate, field.h:676-697), i.e.
// periodically over the linear index; for cells off the outer layer that is a
// plain 3-D neighbour, and for outer-layer (void) cells the kernel reproduces
// the linear wrap exactly.
#pragma once

#include "flb_lattice.cuh"

namespace flb {

struct StepParams {
  const void* src;
  void* dst;
  const uint8_t* flags;
  const void* rho;  // RHO field, arithmetic type
  const void* vel;  // VELOCITY field, 3 SoA planes of dstride elements
  int nx, ny, nz, pitch;
  long long plane;    // pitch * ny
  long long dstride;  // elements between population arrays (and field planes)
  long long ncells;   // nx * ny * nz: the reference's linear cell count
  long long delta[Q]; // reference linear offset c_i . (1, nx, nx*ny)
  long long off[Q];   // padded-layout offset c_i . (1, pitch, plane)
  int ntasks;
  uint8_t keys[8];
  uint8_t ops[8];
  double omega;       // 1/tau, already rounded to the arithmetic type
  double cs_coeff;    // Cs^2 * 9 * 2 * sqrt(2) (LES)
  double s_over_norm[Q];  // MRT: s_k / |M_k|^2
  float shift[Q];     // FP16S: rho0 * w_i
  float scale, inv_scale;
};

// First task whose key shares a bit with the flag (src/utils/tmp.h:283-309).
__device__ __forceinline__ int select_op(const StepParams& p, uint8_t flag) {
  int op = 0;
  bool found = false;
#pragma unroll
  for (int t = 0; t < 8; ++t) {
    if (!found && t < p.ntasks && (flag & p.keys[t])) {
      op = p.ops[t];
      found = true;
    }
  }
  return op;
}

enum : int { OP_NONE = 0, OP_BULK = 1, OP_BB = 2, OP_MBB = 3, OP_FIELD_BGK = 4 };
enum : int { MODEL_BGK = 0, MODEL_MRT = 1, MODEL_LES = 2 };

template <typename R, int MODEL>
__device__ __forceinline__ void apply_op(const StepParams& p, int op, R* f, long long cell,
                                         R omega) {
  if (op == OP_BULK) {
    if constexpr (MODEL == MODEL_BGK) {
      bgk<R>(f, omega, R(1) - omega);
    } else if constexpr (MODEL == MODEL_LES) {
      smagorinsky_bgk<R>(f, R(1) / omega, R(p.cs_coeff));
    } else {
      R s[Q];
#pragma unroll
      for (int k = 0; k < Q; ++k)
        s[k] = mrt_shear(k) ? omega * (R(1) / R(mrt_norm(k))) : R(p.s_over_norm[k]);
      mrt<R>(f, s);
    }
  } else if (op == OP_BB) {
    bounce_back<R>(f);
  } else if (op == OP_MBB || op == OP_FIELD_BGK) {
    const R* rho = static_cast<const R*>(p.rho);
    const R* vel = static_cast<const R*>(p.vel);
    const R rw = rho[cell];
    const R ux = vel[cell], uy = vel[cell + p.dstride], uz = vel[cell + 2 * p.dstride];
    if (op == OP_MBB) moving_wall<R>(f, rw, ux, uy, uz);
    else bgk_field<R>(f, omega, R(1) - omega, rw, ux, uy, uz);
  }
}

// Geometry of one block inside the population / field arrays.
struct Geom {
  int nx, ny, nz, pitch;
  long long plane;  // pitch * ny
  long long base;   // element offset of the block's cell (0,0,0)
};

// Destination of population i pushed from an outer-layer cell.  The reference
// adds Delta_i = cx + nx*cy + nx*ny*cz to the linear index modulo ncells
// (CyclicArray::rotate).  With |c| <= 1 per axis that sum is the mixed-radix
// (nx, ny, nz) addition below: each digit carries at most one unit into the
// next and the last digit wraps modulo nz, which is the modulo-ncells wrap.
__device__ __forceinline__ long long wrap_dest(const Geom& g, int x, int y, int z, int i) {
  int dx = x + cx(i), dy = y + cy(i), dz = z + cz(i);
  if (dx < 0) { dx += g.nx; --dy; } else if (dx >= g.nx) { dx -= g.nx; ++dy; }
  if (dy < 0) { dy += g.ny; --dz; } else if (dy >= g.ny) { dy -= g.ny; ++dz; }
  if (dz < 0) dz += g.nz; else if (dz >= g.nz) dz -= g.nz;
  return g.base + dx + (long long)dy * g.pitch + (long long)dz * g.plane;
}

// One cell of one step: load the 19 populations of (x,y,z), apply the op its
// flag selects, push population i to the cell Delta_i away in dst.
template <typename S, typename R, int MODEL>
__device__ __forceinline__ void update_cell(const StepParams& p, const Geom& g, R omega, int x,
                                            int y, int z) {
  const long long cell = g.base + x + (long long)y * g.pitch + (long long)z * g.plane;
  const S* __restrict__ src = static_cast<const S*>(p.src);
  S* __restrict__ dst = static_cast<S*>(p.dst);

  R f[Q];
#pragma unroll
  for (int i = 0; i < Q; ++i)
    f[i] = Storage<S, R>::load(src + i * p.dstride + cell, p.shift[i], p.inv_scale);

  const int op = select_op(p, p.flags[cell]);
  apply_op<R, MODEL>(p, op, f, cell, omega);

  const bool outer =
      x == 0 || y == 0 || z == 0 || x == g.nx - 1 || y == g.ny - 1 || z == g.nz - 1;
  if (!outer) {
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      const long long off = cx(i) + (long long)cy(i) * g.pitch + (long long)cz(i) * g.plane;
      Storage<S, R>::store(dst + i * p.dstride + cell + off, f[i], p.shift[i], p.scale);
    }
  } else {
#pragma unroll
    for (int i = 0; i < Q; ++i)
      Storage<S, R>::store(dst + i * p.dstride + wrap_dest(g, x, y, z, i), f[i], p.shift[i],
                           p.scale);
  }
}

// Single block: block (32, BY), grid (pitch/32, ceil(ny/BY), nz).
template <typename S, typename R, int MODEL>
__global__ void __launch_bounds__(256) k_stream_collide(const StepParams p) {
  const int x = blockIdx.x * 32 + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= p.nx || y >= p.ny) return;
  const Geom g{p.nx, p.ny, p.nz, p.pitch, p.plane, 0};
  update_cell<S, R, MODEL>(p, g, R(p.omega), x, y, z);
}

// Many blocks in one launch.  Tiles of 32 x blockDim.y cells are numbered
// block by block (x fastest, then y, then z); tile_start is the first tile of
// each block.  CTAs walk the tiles with a grid stride, so the grid can be
// sized to the GPU (persistent) or to the tile count.
struct BlockEntry {
  Geom g;
  double omega;          // per-block 1/tau in the arithmetic type
  long long tile_start;  // first tile of this block
  int tiles_x, tiles_y;  // tiles per row and per plane
};

template <typename S, typename R, int MODEL>
__global__ void __launch_bounds__(256)
    k_stream_collide_blocks(const StepParams p, const BlockEntry* __restrict__ blocks,
                            int nblocks, long long ntiles) {
  for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
    int lo = 0, hi = nblocks - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (blocks[mid].tile_start <= t) lo = mid;
      else hi = mid - 1;
    }
    const BlockEntry& b = blocks[lo];
    long long r = t - b.tile_start;
    const int tx = int(r % b.tiles_x);
    r /= b.tiles_x;
    const int ty = int(r % b.tiles_y);
    const int z = int(r / b.tiles_y);
    const int x = tx * 32 + threadIdx.x;
    const int y = ty * blockDim.y + threadIdx.y;
    if (x < b.g.nx && y < b.g.ny) update_cell<S, R, MODEL>(p, b.g, R(b.omega), x, y, z);
  }
}

// Device halo exchange between blocks (BlockLatticeManager::normalCommunicate,
// block_lattice.hh:1668-1685): after the push, each record copies the listed
// directions of one neighbour inner cell into one overlap cell.
struct HaloRec {
  long long src, dst;  // element offsets within a direction array
  unsigned int mask;   // bit i: population i crosses the shared face/edge/corner
};

template <typename S>
__global__ void k_halo(const HaloRec* __restrict__ recs, int nrecs, S* pops, long long dstride) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nrecs; r += gridDim.x * blockDim.x) {
    const HaloRec h = recs[r];
#pragma unroll
    for (int i = 1; i < Q; ++i)
      if (h.mask & (1u << i)) pops[i * dstride + h.dst] = pops[i * dstride + h.src];
  }
}

// ---------------------------------------------------------------------------
// helpers over the padded layout (1-D grid-stride over padded cells)

struct LayoutParams {
  int nx, ny, nz, pitch;
  long long plane, dstride;
};

__device__ __forceinline__ bool decode_cell(const LayoutParams& L, long long c, int& x, int& y,
                                            int& z) {
  z = int(c / L.plane);
  const long long r = c - (long long)z * L.plane;
  y = int(r / L.pitch);
  x = int(r - (long long)y * L.pitch);
  return z < L.nz && x < L.nx;
}

// f_i = rho0 * w_i on every cell (block_lattice.hh:673-680)
template <typename S, typename R>
__global__ void k_init_equilibrium(LayoutParams L, S* pops, double rho0, StepParams sp) {
  const long long total = L.plane * L.nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total;
       c += (long long)gridDim.x * blockDim.x) {
#pragma unroll
    for (int i = 0; i < Q; ++i)
      Storage<S, R>::store(pops + i * L.dstride + c, R(rho0) * weight<R>(i), sp.shift[i],
                           sp.scale);
  }
}

// staging (host dtype H, padded layout) -> population array i
template <typename S, typename R, typename H>
__global__ void k_pops_in(LayoutParams L, const H* stage, S* pops_i, float shift, float scale) {
  const long long total = L.plane * L.nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total;
       c += (long long)gridDim.x * blockDim.x)
    Storage<S, R>::store(pops_i + c, R(stage[c]), shift, scale);
}

template <typename S, typename R, typename H>
__global__ void k_pops_out(LayoutParams L, H* stage, const S* pops_i, float shift,
                           float inv_scale) {
  const long long total = L.plane * L.nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total;
       c += (long long)gridDim.x * blockDim.x)
    stage[c] = H(Storage<S, R>::load(pops_i + c, shift, inv_scale));
}

template <typename R>
__global__ void k_fill(long long n, R* out, R v) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x)
    out[c] = v;
}

template <typename A, typename B>
__global__ void k_convert(long long n, const A* in, B* out) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x)
    out[c] = B(in[c]);
}

// AoS velocity staging (3*pitch per row) <-> SoA planes
template <typename R, typename H>
__global__ void k_vel_in(LayoutParams L, const H* stage, R* vel) {
  const long long total = L.plane * L.nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total;
       c += (long long)gridDim.x * blockDim.x) {
    const long long row = c / L.pitch, x = c - row * L.pitch;
    const long long s = row * 3 * L.pitch + 3 * x;
#pragma unroll
    for (int d = 0; d < 3; ++d) vel[c + d * L.dstride] = R(stage[s + d]);
  }
}

template <typename R, typename H>
__global__ void k_vel_out(LayoutParams L, H* stage, const R* vel) {
  const long long total = L.plane * L.nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total;
       c += (long long)gridDim.x * blockDim.x) {
    const long long row = c / L.pitch, x = c - row * L.pitch;
    const long long s = row * 3 * L.pitch + 3 * x;
#pragma unroll
    for (int d = 0; d < 3; ++d) stage[s + d] = H(vel[c + d * L.dstride]);
  }
}

// RHO/VELOCITY from populations on cells matching key (moment::rhoU<CELL,true>)
template <typename S, typename R>
__global__ void k_rhou(LayoutParams L, const S* pops, const uint8_t* flags, uint8_t key, R* rho,
                       R* vel, StepParams sp) {
  const long long total = L.plane * L.nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total;
       c += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    if (!decode_cell(L, c, x, y, z)) continue;
    if (!(flags[c] & key)) continue;
    R f[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i)
      f[i] = Storage<S, R>::load(pops + i * L.dstride + c, sp.shift[i], sp.inv_scale);
    R r, ux, uy, uz;
    rho_u<R>(f, r, ux, uy, uz);
    rho[c] = r;
    vel[c] = ux;
    vel[c + L.dstride] = uy;
    vel[c + 2 * L.dstride] = uz;
  }
}

// ---------------------------------------------------------------------------
// FP64 reductions.  acc points to handle-owned device scratch:
//   conservation: acc[0..3] (double sums); tolerance: acc_u64[0] (max as bits);
//   finite: acc_u64[0] (count).

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

template <typename S, typename R>
__global__ void __launch_bounds__(256) k_conservation(LayoutParams L, const S* pops,
                                                      const uint8_t* flags, uint8_t key,
                                                      double* acc, StepParams sp) {
  double s[4] = {0, 0, 0, 0};
  const long long total = L.plane * L.nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total;
       c += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    if (!decode_cell(L, c, x, y, z)) continue;
    if (!(flags[c] & key)) continue;
    double f[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i)
      f[i] = double(Storage<S, R>::load(pops + i * L.dstride + c, sp.shift[i], sp.inv_scale));
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      s[0] += f[i];
      s[1] += cx(i) * f[i];
      s[2] += cy(i) * f[i];
      s[3] += cz(i) * f[i];
    }
  }
  __shared__ double red[8][4];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const double v = warp_sum(s[k]);
    if (lane == 0) red[wid][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double v = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[w][threadIdx.x];
    atomicAdd(acc + threadIdx.x, v);
  }
}

template <typename S, typename R>
__global__ void __launch_bounds__(256) k_tolerance(LayoutParams L, const S* pops,
                                                   const uint8_t* flags, uint8_t key,
                                                   double* uprev, unsigned long long* acc,
                                                   StepParams sp) {
  double m = 0;
  const long long total = L.plane * L.nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total;
       c += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    if (!decode_cell(L, c, x, y, z)) continue;
    if (!(flags[c] & key)) continue;
    R f[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i)
      f[i] = Storage<S, R>::load(pops + i * L.dstride + c, sp.shift[i], sp.inv_scale);
    R r, ux, uy, uz;
    rho_u<R>(f, r, ux, uy, uz);
    const double u[3] = {double(ux), double(uy), double(uz)};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      m = fmax(m, fabs(u[d] - uprev[c + d * L.dstride]));
      uprev[c + d * L.dstride] = u[d];
    }
  }
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0)
    atomicMax(acc, (unsigned long long)__double_as_longlong(m));  // m >= 0: bits order
}

template <typename S, typename R>
__global__ void __launch_bounds__(256) k_finite(LayoutParams L, const S* pops,
                                                unsigned long long* acc, StepParams sp) {
  unsigned long long bad = 0;
  const long long total = L.plane * L.nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total;
       c += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    if (!decode_cell(L, c, x, y, z)) continue;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      const R v = Storage<S, R>::load(pops + i * L.dstride + c, sp.shift[i], sp.inv_scale);
      if (!isfinite(v)) ++bad;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) bad += __shfl_xor_sync(0xffffffffu, bad, o);
  if ((threadIdx.x & 31) == 0 && bad) atomicAdd(acc, bad);
}

}  // namespace flb
