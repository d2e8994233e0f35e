// flb_pull.cuh -- the fused stream-and-collide step as a vectorised pull.
//
// State between launches.  A handle stores P, the post-collision populations
// at their own cell; the reference's post-stream populations are R = stream(P),
// R_i(x) = P_i(x - Delta_i) with the reference's periodic wrap over each
// block's linear index (CyclicArray::rotate, src/data_struct/field.h:676-697).
// One launch maps P to P' = collide(stream(P)) = collide(R), so that
// stream(P') is the reference state after ApplyCellDynamics + Stream
// (block_lattice.hh:64-92).  Upload and download apply stream^-1 / stream,
// which are exact permutations, so the C ABI still speaks R.
//
// Thread mapping.  A warp covers 32*V consecutive cells of one row, lane l
// owning the aligned chunk x0 = 32*V*w + V*l; V (cells per thread) is a launch
// parameter: 2 or 4 for FP32 and FP16S, 1 or 2 for FP64.  Every
// population array is read with aligned V-wide loads (the x-shifted directions
// also read the adjacent chunk: reads may be duplicated, writes never are) and
// written with one aligned V-wide store per direction at the thread's own
// chunk.  See gather_chunk for the edge rules.
#pragma once

#include "flb_kernels.cuh"

namespace flb {

// V-wide aligned loads and stores of one chunk of a population array, with
// the storage conversion of Storage<S, R> (FP16S: shift and scale).
template <typename S, typename R, int V>
__device__ __forceinline__ void vload(const S* p, R* out, float shift, float inv_scale) {
  if constexpr (std::is_same<S, float>::value && V == 4) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(p));
    out[0] = v.x;
    out[1] = v.y;
    out[2] = v.z;
    out[3] = v.w;
  } else if constexpr (std::is_same<S, float>::value && V == 2) {
    const float2 v = __ldg(reinterpret_cast<const float2*>(p));
    out[0] = v.x;
    out[1] = v.y;
  } else if constexpr (std::is_same<S, double>::value && V == 2) {
    const double2 v = __ldg(reinterpret_cast<const double2*>(p));
    out[0] = v.x;
    out[1] = v.y;
  } else if constexpr (std::is_same<S, __half>::value && V == 2) {
    const unsigned v = __ldg(reinterpret_cast<const unsigned*>(p));
    const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&v));
    out[0] = fmaf(a.x, inv_scale, shift);
    out[1] = fmaf(a.y, inv_scale, shift);
  } else if constexpr (std::is_same<S, __half>::value && V == 4) {
    const uint2 v = __ldg(reinterpret_cast<const uint2*>(p));
    const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&v.x));
    const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&v.y));
    out[0] = fmaf(a.x, inv_scale, shift);
    out[1] = fmaf(a.y, inv_scale, shift);
    out[2] = fmaf(b.x, inv_scale, shift);
    out[3] = fmaf(b.y, inv_scale, shift);
  } else {
#pragma unroll
    for (int k = 0; k < V; ++k) out[k] = Storage<S, R>::load(p + k, shift, inv_scale);
  }
}

template <typename S, typename R, int V>
__device__ __forceinline__ void vstore(S* p, const R* in, float shift, float scale) {
  if constexpr (std::is_same<S, float>::value && V == 4) {
    *reinterpret_cast<float4*>(p) = make_float4(in[0], in[1], in[2], in[3]);
  } else if constexpr (std::is_same<S, float>::value && V == 2) {
    *reinterpret_cast<float2*>(p) = make_float2(in[0], in[1]);
  } else if constexpr (std::is_same<S, double>::value && V == 2) {
    *reinterpret_cast<double2*>(p) = make_double2(in[0], in[1]);
  } else if constexpr (std::is_same<S, __half>::value && V == 2) {
    const __half2 a = __floats2half2_rn((in[0] - shift) * scale, (in[1] - shift) * scale);
    *reinterpret_cast<unsigned*>(p) = *reinterpret_cast<const unsigned*>(&a);
  } else if constexpr (std::is_same<S, __half>::value && V == 4) {
    const __half2 a = __floats2half2_rn((in[0] - shift) * scale, (in[1] - shift) * scale);
    const __half2 b = __floats2half2_rn((in[2] - shift) * scale, (in[3] - shift) * scale);
    uint2 v;
    v.x = *reinterpret_cast<const unsigned*>(&a);
    v.y = *reinterpret_cast<const unsigned*>(&b);
    *reinterpret_cast<uint2*>(p) = v;
  } else {
#pragma unroll
    for (int k = 0; k < V; ++k) Storage<S, R>::store(p + k, in[k], shift, scale);
  }
}

// Source of population i for cell (x,y,z) under the reference's streaming:
// the cell Delta_i *before* it in the block's linear order, with wrap.
__device__ __forceinline__ long long wrap_src(const Geom& g, int x, int y, int z, int i) {
  int sx = x - cx(i), sy = y - cy(i), sz = z - cz(i);
  if (sx < 0) { sx += g.nx; --sy; } else if (sx >= g.nx) { sx -= g.nx; ++sy; }
  if (sy < 0) { sy += g.ny; --sz; } else if (sy >= g.ny) { sy -= g.ny; ++sz; }
  if (sz < 0) sz += g.nz; else if (sz >= g.nz) sz -= g.nz;
  return g.base + sx + (long long)sy * g.pitch + (long long)sz * g.plane;
}

// Cell (x + dx, y + dy, z + dz) under the reference's linear wrap (|d| <= 1).
__device__ __forceinline__ long long wrap_off(const Geom& g, int x, int y, int z, int dx, int dy,
                                              int dz) {
  int sx = x + dx, sy = y + dy, sz = z + dz;
  if (sx < 0) { sx += g.nx; --sy; } else if (sx >= g.nx) { sx -= g.nx; ++sy; }
  if (sy < 0) { sy += g.ny; --sz; } else if (sy >= g.ny) { sy -= g.ny; ++sz; }
  if (sz < 0) sz += g.nz; else if (sz >= g.nz) sz -= g.nz;
  return g.base + sx + (long long)sy * g.pitch + (long long)sz * g.plane;
}

// Gather, for the V cells x0.. of row (y, z), population i from the cell
// SIGN*c_i away *before* it: SIGN = +1 reads x - c_i (streaming pull),
// SIGN = -1 reads x + c_i (the transpose of streaming).
//
// Inner rows: every direction is one aligned V-wide load of the source row at
// the lane's own chunk; the ten x-shifted directions add one aligned load of
// the adjacent chunk (the neighbour lane's, an L1 hit for all but one lane per
// warp) and splice the element crossing the chunk edge.  The adjacent-chunk
// addresses are clamped into the row, so the 29 loads carry no branches and can
// all be in flight together.  Cells x = 0 / x = nx-1 whose sources cross the
// row end and whole outer rows (y or z on the block surface) then re-load
// through the wrap rule.  Called for chunks with x0 < nx only.
template <typename S, typename R, int V, int SIGN>
__device__ __forceinline__ void gather_chunk(const S* __restrict__ arr, long long dstride,
                                             const Geom& g, const float* shift, float inv_scale,
                                             int x0, int y, int z, R (&vals)[Q][V]) {
  const bool inner_row = y > 0 && z > 0 && y < g.ny - 1 && z < g.nz - 1;
  const bool active = true;
  if (inner_row) {
    const int xl = x0;
    const int xprev = xl >= V ? xl - V : xl;
    const int xnext = xl + V < g.nx ? xl + V : xl;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      const int ex = SIGN * cx(i), ey = SIGN * cy(i), ez = SIGN * cz(i);
      const S* rowp = arr + i * dstride + g.base + (long long)(y - ey) * g.pitch +
                      (long long)(z - ez) * g.plane;
      R v[V];
      vload<S, R, V>(rowp + xl, v, shift[i], inv_scale);
      if (ex == 0) {
#pragma unroll
        for (int k = 0; k < V; ++k) vals[i][k] = v[k];
      } else if (ex > 0) {
        R w[V];  // chunk before: its last element is x0 - 1
        vload<S, R, V>(rowp + xprev, w, shift[i], inv_scale);
        vals[i][0] = w[V - 1];
#pragma unroll
        for (int k = 1; k < V; ++k) vals[i][k] = v[k - 1];
      } else {
        R w[V];  // chunk after: its first element is x0 + V
        vload<S, R, V>(rowp + xnext, w, shift[i], inv_scale);
#pragma unroll
        for (int k = 0; k < V - 1; ++k) vals[i][k] = v[k + 1];
        vals[i][V - 1] = w[0];
      }
    }
    // x = 0 and x = nx-1: sources crossing the row end wrap into the
    // neighbouring row (carry of the linear index).
    if (active && x0 == 0) {
#pragma unroll
      for (int i = 1; i < Q; ++i)
        if (SIGN * cx(i) > 0)
          vals[i][0] = Storage<S, R>::load(
              arr + i * dstride + wrap_off(g, 0, y, z, -SIGN * cx(i), -SIGN * cy(i), -SIGN * cz(i)),
              shift[i], inv_scale);
    }
    const int klast = g.nx - 1 - x0;
    if (active && klast >= 0 && klast < V) {
#pragma unroll
      for (int k = 0; k < V; ++k)
        if (k == klast) {
#pragma unroll
          for (int i = 1; i < Q; ++i)
            if (SIGN * cx(i) < 0)
              vals[i][k] = Storage<S, R>::load(
                  arr + i * dstride +
                      wrap_off(g, g.nx - 1, y, z, -SIGN * cx(i), -SIGN * cy(i), -SIGN * cz(i)),
                  shift[i], inv_scale);
        }
    }
  } else if (active) {
    // outer row: every source through the wrap rule
#pragma unroll
    for (int k = 0; k < V; ++k) {
      const int x = min(x0 + k, g.nx - 1);
#pragma unroll
      for (int i = 0; i < Q; ++i)
        vals[i][k] = Storage<S, R>::load(
            arr + i * dstride + wrap_off(g, x, y, z, -SIGN * cx(i), -SIGN * cy(i), -SIGN * cz(i)),
            shift[i], inv_scale);
    }
  }
}

template <int V>
__device__ __forceinline__ void load_flags(const uint8_t* p, uint8_t (&fl)[V]) {
  if constexpr (V == 4) {
    const uchar4 fv = *reinterpret_cast<const uchar4*>(p);
    fl[0] = fv.x;
    fl[1] = fv.y;
    fl[2] = fv.z;
    fl[3] = fv.w;
  } else if constexpr (V == 2) {
    const uchar2 fv = *reinterpret_cast<const uchar2*>(p);
    fl[0] = fv.x;
    fl[1] = fv.y;
  } else {
#pragma unroll
    for (int k = 0; k < V; ++k) fl[k] = p[k];
  }
}

// Collide the V cells of a chunk in place (vals[i][k]) by their flags.
template <typename R, int MODEL, int V>
__device__ __forceinline__ void collide_chunk(const StepParams& p, const Geom& g, R omega,
                                              R (&vals)[Q][V], const uint8_t* fl,
                                              long long cell0, int nvalid) {
#pragma unroll
  for (int k = 0; k < V; ++k) {
    if (k < nvalid) {
      R f[Q];
#pragma unroll
      for (int i = 0; i < Q; ++i) f[i] = vals[i][k];
      const int op = select_op(p, fl[k]);
      apply_op<R, MODEL>(p, op, f, cell0 + k, omega);
#pragma unroll
      for (int i = 0; i < Q; ++i) vals[i][k] = f[i];
    }
  }
}

// One chunk: the thread owns cells x0 .. x0+V-1 of row (y, z), x0 < nx.
template <typename S, typename R, int MODEL, int V>
__device__ __forceinline__ void pull_chunk(const StepParams& p, const Geom& g, R omega, int lane,
                                           int x0, int y, int z) {
  const S* __restrict__ src = static_cast<const S*>(p.src);
  S* __restrict__ dst = static_cast<S*>(p.dst);
  R vals[Q][V];
  gather_chunk<S, R, V, 1>(src, p.dstride, g, p.shift, p.inv_scale, x0, y, z, vals);
  const int nvalid = min(V, g.nx - x0);
  const long long cell0 = g.base + (long long)y * g.pitch + (long long)z * g.plane + x0;
  uint8_t fl[V];
  load_flags<V>(p.flags + cell0, fl);
  collide_chunk<R, MODEL, V>(p, g, omega, vals, fl, cell0, nvalid);
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    R v[V];
#pragma unroll
    for (int k = 0; k < V; ++k) v[k] = vals[i][k];
    vstore<S, R, V>(dst + i * p.dstride + cell0, v, p.shift[i], p.scale);
  }
}

// Chunk q of a block (V cells, counted over the padded rows: pitch / V chunks
// per row) -> (x0, y, z); false for chunks in the row padding or past the end.
template <int V>
__device__ __forceinline__ bool chunk_coords(const Geom& g, long long q, int& x0, int& y,
                                             int& z) {
  const int cpr = g.pitch / V;
  const long long row = q / cpr;
  x0 = int(q - row * cpr) * V;
  y = int(row % g.ny);
  z = int(row / g.ny);
  return z < g.nz && x0 < g.nx;
}

// Single block: one thread per chunk; consecutive threads take consecutive
// chunks, so a warp may span the end of one row and the start of the next and
// only padding lanes idle.  Grid: ceil(chunks / blockDim.x) CTAs.
template <typename S, typename R, int MODEL, int V>
__global__ void __launch_bounds__(256) k_pull(const StepParams p) {
  const Geom g{p.nx, p.ny, p.nz, p.pitch, p.plane, 0};
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int x0, y, z;
  if (!chunk_coords<V>(g, q, x0, y, z)) return;
  pull_chunk<S, R, MODEL, V>(p, g, R(p.omega), 0, x0, y, z);
}

// Many blocks: tiles of blockDim.x consecutive chunks, numbered block by block
// (tile_start = first tile of the block); CTAs walk the tiles with a grid stride
// (persistent) or take one tile each.
template <typename S, typename R, int MODEL, int V>
__global__ void __launch_bounds__(256)
    k_pull_blocks(const StepParams p, const BlockEntry* __restrict__ blocks, int nblocks,
                  long long ntiles) {
  for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
    int lo = 0, hi = nblocks - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (blocks[mid].tile_start <= t) lo = mid;
      else hi = mid - 1;
    }
    const BlockEntry& b = blocks[lo];
    const long long q = (t - b.tile_start) * blockDim.x + threadIdx.x;
    int x0, y, z;
    if (chunk_coords<V>(b.g, q, x0, y, z))
      pull_chunk<S, R, MODEL, V>(p, b.g, R(b.omega), 0, x0, y, z);
  }
}

// ---------------------------------------------------------------------------
// Transfers and helpers in R = stream(P) space.

// population array i: R (staging, host dtype, padded layout) -> P slots
template <typename S, typename R, typename H>
__global__ void k_unstream_in(LayoutParams L, Geom g, const H* stage, S* pops_i, int i,
                              float shift, float scale) {
  const long long total = L.plane * L.nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total;
       c += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    if (!decode_cell(L, c, x, y, z)) continue;
    Storage<S, R>::store(pops_i + wrap_src(g, x, y, z, i), R(stage[c]), shift, scale);
  }
}

template <typename S, typename R, typename H>
__global__ void k_stream_out(LayoutParams L, Geom g, H* stage, const S* pops_i, int i,
                             float shift, float inv_scale) {
  const long long total = L.plane * L.nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total;
       c += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    if (!decode_cell(L, c, x, y, z)) continue;
    stage[c] = H(Storage<S, R>::load(pops_i + wrap_src(g, x, y, z, i), shift, inv_scale));
  }
}

// the 19 post-stream populations of cell (x,y,z)
template <typename S, typename R>
__device__ __forceinline__ void gather_R(const S* pops, long long dstride, const Geom& g, int x,
                                         int y, int z, const StepParams& sp, R* f) {
#pragma unroll
  for (int i = 0; i < Q; ++i)
    f[i] = Storage<S, R>::load(pops + i * dstride + wrap_src(g, x, y, z, i), sp.shift[i],
                               sp.inv_scale);
}

template <typename S, typename R>
__global__ void k_rhou_pull(LayoutParams L, Geom g, const S* pops, const uint8_t* flags,
                            uint8_t key, R* rho, R* vel, StepParams sp) {
  const long long total = L.plane * L.nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total;
       c += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    if (!decode_cell(L, c, x, y, z)) continue;
    if (!(flags[g.base + c] & key)) continue;
    R f[Q], r, ux, uy, uz;
    gather_R<S, R>(pops, L.dstride, g, x, y, z, sp, f);
    if (sp.alpha) {
      R den;
      forced_moments<R>(f, static_cast<const R*>(sp.alpha)[g.base + c], r, den, ux, uy, uz);
    } else {
      rho_u<R>(f, r, ux, uy, uz);
    }
    rho[g.base + c] = r;
    vel[g.base + c] = ux;
    vel[g.base + c + L.dstride] = uy;
    vel[g.base + c + 2 * L.dstride] = uz;
  }
}

template <typename S, typename R>
__global__ void __launch_bounds__(256) k_conservation_pull(LayoutParams L, Geom g, const S* pops,
                                                           const uint8_t* flags, uint8_t key,
                                                           double* acc, StepParams sp) {
  double s[4] = {0, 0, 0, 0};
  const long long total = L.plane * L.nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total;
       c += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    if (!decode_cell(L, c, x, y, z)) continue;
    if (!(flags[g.base + c] & key)) continue;
    R f[Q];
    gather_R<S, R>(pops, L.dstride, g, x, y, z, sp, f);
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      const double v = double(f[i]);
      s[0] += v;
      s[1] += cx(i) * v;
      s[2] += cy(i) * v;
      s[3] += cz(i) * v;
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
__global__ void __launch_bounds__(256) k_tolerance_pull(LayoutParams L, Geom g, const S* pops,
                                                        const uint8_t* flags, uint8_t key,
                                                        double* uprev, unsigned long long* acc,
                                                        StepParams sp) {
  double m = 0;
  const long long total = L.plane * L.nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total;
       c += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    if (!decode_cell(L, c, x, y, z)) continue;
    if (!(flags[g.base + c] & key)) continue;
    R f[Q], r, ux, uy, uz;
    gather_R<S, R>(pops, L.dstride, g, x, y, z, sp, f);
    rho_u<R>(f, r, ux, uy, uz);
    const double u[3] = {double(ux), double(uy), double(uz)};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      double* up = uprev + g.base + c + d * L.dstride;
      m = fmax(m, fabs(u[d] - *up));
      *up = u[d];
    }
  }
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) atomicMax(acc, (unsigned long long)__double_as_longlong(m));
}

// Halo in pull form: the overlap value R_b(g, i) lives in P_b at
// wrap_b(g - c_i); it is set from the neighbour's P_nb at wrap_nb(g - c_i).
struct HaloCopy {
  long long src, dst;  // offsets in population array `dir`
  int dir;
};

template <typename S>
__global__ void k_halo_pull(const HaloCopy* __restrict__ recs, long long n, S* pops,
                            long long dstride) {
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n;
       r += (long long)gridDim.x * blockDim.x) {
    const HaloCopy h = recs[r];
    pops[h.dir * dstride + h.dst] = pops[h.dir * dstride + h.src];
  }
}

}  // namespace flb
