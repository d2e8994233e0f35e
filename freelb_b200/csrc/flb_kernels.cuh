// flb_kernels.cuh -- fused stream-and-collide and helper kernels (sm_100a).
//
// HBM layout of one block lattice (all arrays padded the same way):
//   cell (x,y,z) -> base + x + y*pitch + z*plane, pitch = nx rounded up to 16
//   elements for nx >= 240 (rows start on 64-byte boundaries for FP32) and to
//   4 below (row_pitch in flb_api.cu), plane = pitch*ny; each block starts at
//   `base`, the sum of the blocks before it rounded up to 64 elements each;
//   population i lives at pops + i*dstride + cell (structure of arrays), with
//   dstride = the whole padded lattice.
// The reference keeps the same SoA split (GenericFieldBase, field.h:1419-1575)
// on an unpadded mesh; padding is invisible at the C ABI, which converts to
// and from the reference's linear order on upload/download.
//
// The step kernels themselves (a vectorised pull over ping-pong buffers) are in
// flb_pull.cuh; this file holds the per-cell op dispatch, the block geometry
// and the layout helpers shared by all kernels.
#pragma once

#include "flb_lattice.cuh"

namespace flb {

struct StepParams {
  const void* src;
  void* dst;
  const uint8_t* flags;
  const void* rho;  // RHO field, arithmetic type
  const void* vel;  // VELOCITY field, 3 SoA planes of dstride elements
  const void* alpha;  // Brinkman porosity field (MODEL_BRINKMAN), arithmetic type
  int nx, ny, nz, pitch;
  long long plane;    // pitch * ny
  long long dstride;  // elements between population arrays (and field planes)
  long long row_off[Q];  // block 0: i * dstride - (cy_i + cz_i ny) * pitch
  // 32-bit element offsets for single-block handles with 19 * dstride < 2^32
  unsigned row_off32[Q];  // row_off as an unsigned 32-bit offset
  unsigned dir_off32[Q];  // i * dstride
  int idx32;              // the 32-bit offsets above are valid
  // Per-launch direction bases of the single-block FP16S step (set from
  // src / dst at launch): the source row of direction i relative to a cell,
  // src + row_off[i], and the destination array, dst + i * dstride, so each
  // address is the base plus the cell's 32-bit index.
  const void* src_dir[Q];
  void* dst_dir[Q];
  // chunk -> row: row = umulhi(q, cpr_m) >> (cpr_s - 1) for q < 2^31, the
  // round-up division by an invariant integer (Granlund & Montgomery, PLDI
  // 1994); cpr_m = 0 when there is one chunk per row.
  unsigned cpr_m, cpr_s;
  int ntasks;
  uint8_t keys[8];
  uint8_t ops[8];
  const uint8_t* op_lut;  // op of every flag value (device, 256 entries)
  double omega;       // 1/tau, already rounded to the arithmetic type
  double cs_coeff;    // Cs^2 * 9 * 2 * sqrt(2) (LES)
  double s_over_norm[Q];  // MRT: s_k / |M_k|^2
  float shift[Q];     // FP16S: rho0 * w_i
  float scale, inv_scale;
  float rho0;         // FP16S: density of the shift
  int fp16_round;     // FP16S stores: 0 round to nearest, 1 stochastic (cvt.rs)
  float mrt_sg;       // the one rate of every non-conserved, non-shear MRT
                      // moment, or 0 when the rates differ (MRT then runs
                      // the general form instead of MODEL_MRT2)
};

// First task whose key shares a bit with the flag (src/utils/tmp.h:283-309),
// tabulated on the host for all 256 flag values.
__device__ __forceinline__ int select_op(const StepParams& p, uint8_t flag) {
  return __ldg(p.op_lut + flag);
}

enum : int { OP_NONE = 0, OP_BULK = 1, OP_BB = 2, OP_MBB = 3, OP_FIELD_BGK = 4 };
enum : int { MODEL_BGK = 0, MODEL_MRT = 1, MODEL_LES = 2, MODEL_BRINKMAN = 3, MODEL_MRT2 = 4 };
// MODEL_MRT2: the two-rate MRT form (every non-conserved, non-shear moment at
// one rate), chosen on the host for FP16S and FP32 storage; it is MRT in every
// other respect.
__host__ __device__ constexpr bool is_mrt(int model) {
  return model == MODEL_MRT || model == MODEL_MRT2;
}

// The ops every model shares: bounce-back, moving wall, field-velocity BGK.
template <typename R>
__device__ __forceinline__ void apply_wall_op(const StepParams& p, int op, R* f, long long cell,
                                              R omega) {
  if (op == OP_BB) {
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

template <typename R, int MODEL>
__device__ __forceinline__ void apply_op(const StepParams& p, int op, R* f, long long cell,
                                         R omega) {
  if (op == OP_BULK) {
    if constexpr (MODEL == MODEL_BGK) {
      bgk<R>(f, omega, R(1) - omega);
    } else if constexpr (MODEL == MODEL_LES) {
      smagorinsky_bgk<R>(f, R(1) / omega, R(p.cs_coeff));
    } else if constexpr (MODEL == MODEL_BRINKMAN) {
      bgk_brinkman<R>(f, omega, static_cast<const R*>(p.alpha)[cell]);
    } else if constexpr (MODEL == MODEL_MRT2) {
      mrt_two_rate<R>(f, omega, R(p.mrt_sg));
    } else {
      R s[Q];
#pragma unroll
      for (int k = 0; k < Q; ++k)
        s[k] = mrt_shear(k) ? omega * (R(1) / R(mrt_norm_lit(k))) : R(p.s_over_norm[k]);
      mrt<R>(f, s);
    }
  } else {
    apply_wall_op<R>(p, op, f, cell, omega);
  }
}

// Geometry of one block inside the population / field arrays.
struct Geom {
  int nx, ny, nz, pitch;
  long long plane;  // pitch * ny
  long long base;   // element offset of the block's cell (0,0,0)
};

// Many blocks in one launch.  Tiles of 32 x blockDim.y cells are numbered
// block by block (x fastest, then y, then z); tile_start is the first tile of
// each block.  CTAs walk the tiles with a grid stride, so the grid can be
// sized to the GPU (persistent) or to the tile count.
struct BlockEntry {
  Geom g;
  double omega;          // per-block 1/tau in the arithmetic type
  long long tile_start;  // first tile of this block
};

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

// Host order (x fastest, nx values per row, contiguous) <-> the padded rows of
// a block, with the element conversion A -> B: transfers stage the host
// array contiguously on the device so that each crosses the bus as one copy.
template <typename A, typename B>
__global__ void k_pad(LayoutParams L, const A* in, B* out) {
  const long long total = (long long)L.nx * L.ny * L.nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total;
       c += (long long)gridDim.x * blockDim.x) {
    const long long r = c / L.nx, x = c - r * L.nx;
    out[r * L.pitch + x] = B(in[c]);
  }
}
template <typename A, typename B>
__global__ void k_unpad(LayoutParams L, const A* in, B* out) {
  const long long total = (long long)L.nx * L.ny * L.nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total;
       c += (long long)gridDim.x * blockDim.x) {
    const long long r = c / L.nx, x = c - r * L.nx;
    out[c] = B(in[r * L.pitch + x]);
  }
}

// AoS velocity staging (host order, 3 values per cell) <-> SoA planes
template <typename R, typename H>
__global__ void k_vel_in(LayoutParams L, const H* stage, R* vel) {
  const long long total = (long long)L.nx * L.ny * L.nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total;
       c += (long long)gridDim.x * blockDim.x) {
    const long long r = c / L.nx, p = r * L.pitch + (c - r * L.nx);
#pragma unroll
    for (int d = 0; d < 3; ++d) vel[p + d * L.dstride] = R(stage[3 * c + d]);
  }
}

template <typename R, typename H>
__global__ void k_vel_out(LayoutParams L, H* stage, const R* vel) {
  const long long total = (long long)L.nx * L.ny * L.nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total;
       c += (long long)gridDim.x * blockDim.x) {
    const long long r = c / L.nx, p = r * L.pitch + (c - r * L.nx);
#pragma unroll
    for (int d = 0; d < 3; ++d) stage[3 * c + d] = H(vel[p + d * L.dstride]);
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

// Deterministic FP64 sums: every CTA of a reduction writes its own slot(s) of
// `partials` (ncomp values per slot, in a fixed order within the CTA) and this
// kernel adds slots 0..nslots-1 in a fixed order to acc[0..ncomp).  The result
// does not depend on CTA scheduling, unlike atomics (~1e-14 relative jitter on
// a sum of millions of terms, enough to swamp a finite difference of it).
constexpr int RED_SLOTS = 148 * 32;  // the largest grid_1d grid
// Error-free addition (Knuth's TwoSum): s + e == a + b exactly, s = fl(a + b).
__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  const double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}
// Compensated (double-double) accumulation: hi + lo carries the running sum
// with ~2^-106 relative error, so a sum of millions of FP64 terms keeps every
// digit of the terms (Ogita, Rump & Oishi, SIAM J. Sci. Comput. 26 (2005)).
struct dd {
  double hi = 0, lo = 0;
  __device__ __forceinline__ void add(double v) {
    double s, e;
    two_sum(hi, v, s, e);
    hi = s;
    lo += e;
  }
  __device__ __forceinline__ void add(dd o) {
    double s, e;
    two_sum(hi, o.hi, s, e);
    hi = s;
    lo += e + o.lo;
  }
};
__device__ __forceinline__ dd warp_sum_dd(dd v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    dd w;
    w.hi = __shfl_xor_sync(0xffffffffu, v.hi, o);
    w.lo = __shfl_xor_sync(0xffffffffu, v.lo, o);
    v.add(w);
  }
  return v;
}
// Slots of (hi, lo) pairs, summed in a fixed order with compensation: acc[0]
// += the rounded double-double total (k_objective).
static __global__ void __launch_bounds__(256) k_sum_partials_dd(const double* partials,
                                                                int nslots, double* acc) {
  __shared__ double red[2][256];
  dd s;
  for (int b = threadIdx.x; b < nslots; b += 256) {
    dd v;
    v.hi = partials[2 * b];
    v.lo = partials[2 * b + 1];
    s.add(v);
  }
  red[0][threadIdx.x] = s.hi;
  red[1][threadIdx.x] = s.lo;
  __syncthreads();
  if (threadIdx.x == 0) {
    dd t;
    for (int k = 0; k < 256; ++k) {
      dd v;
      v.hi = red[0][k];
      v.lo = red[1][k];
      t.add(v);
    }
    acc[0] += t.hi + t.lo;
  }
}

static __global__ void __launch_bounds__(256) k_sum_partials(const double* partials,
                                                             int nslots, int ncomp, double* acc) {
  __shared__ double red[256];
  for (int k = 0; k < ncomp; ++k) {
    double s = 0;
    for (int b = threadIdx.x; b < nslots; b += 256) s += partials[b * ncomp + k];
    red[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double v = 0;
      for (int t = 0; t < 256; ++t) v += red[t];
      acc[k] += v;
    }
    __syncthreads();
  }
}

template <typename S, typename R>
__global__ void __launch_bounds__(256) k_finite(LayoutParams L, const S* pops,
                                                const uint8_t* flags, unsigned long long* acc,
                                                StepParams sp) {
  unsigned long long bad = 0;
  const long long total = L.plane * L.nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total;
       c += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    if (!decode_cell(L, c, x, y, z)) continue;
    if (select_op(sp, flags[c]) == OP_NONE) continue;  // void: the reference's wrapped values
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
