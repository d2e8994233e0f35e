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
  if constexpr (std::is_same<S, dev32>::value) {
    // FP32S: the step and adjoint kernels work on the stored deviations
    vload<float, R, V>(reinterpret_cast<const float*>(p), out, shift, inv_scale);
  } else if constexpr (std::is_same<S, float>::value && V == 4) {
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
  if constexpr (std::is_same<S, dev32>::value) {
    vstore<float, R, V>(reinterpret_cast<float*>(p), in, shift, scale);
  } else if constexpr (std::is_same<S, float>::value && V == 4) {
    *reinterpret_cast<float4*>(p) = make_float4(in[0], in[1], in[2], in[3]);
  } else if constexpr (std::is_same<S, float>::value && V == 2) {
    *reinterpret_cast<float2*>(p) = make_float2(in[0], in[1]);
  } else if constexpr (std::is_same<S, double>::value && V == 2) {
    *reinterpret_cast<double2*>(p) = make_double2(in[0], in[1]);
  } else if constexpr (std::is_same<S, __half>::value && V == 2) {
    const float ns = -shift * scale;  // exact: scale is a power of two
    const __half2 a = __floats2half2_rn(fmaf(in[0], scale, ns), fmaf(in[1], scale, ns));
    *reinterpret_cast<unsigned*>(p) = *reinterpret_cast<const unsigned*>(&a);
  } else if constexpr (std::is_same<S, __half>::value && V == 4) {
    const float ns = -shift * scale;
    const __half2 a = __floats2half2_rn(fmaf(in[0], scale, ns), fmaf(in[1], scale, ns));
    const __half2 b = __floats2half2_rn(fmaf(in[2], scale, ns), fmaf(in[3], scale, ns));
    uint2 v;
    v.x = *reinterpret_cast<const unsigned*>(&a);
    v.y = *reinterpret_cast<const unsigned*>(&b);
    *reinterpret_cast<uint2*>(p) = v;
  } else {
#pragma unroll
    for (int k = 0; k < V; ++k) Storage<S, R>::store(p + k, in[k], shift, scale);
  }
}

// One stored value as the step kernels see it (vload's form for one element):
// FP32S deviations as stored, every other storage through its load form.
template <typename S, typename R>
__device__ __forceinline__ R gload(const S* p, float shift, float inv_scale) {
  if constexpr (std::is_same<S, dev32>::value) return p->v;
  else return Storage<S, R>::load(p, shift, inv_scale);
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

// Linear rows.  Rows are numbered r = z * ny + y over the block and the padded
// layout stores row r at r * pitch, so the carry of y into z in the reference's
// periodic shift over the linear cell index (CyclicArray::rotate,
// field.h:676-697) is the linear order itself: the source row of direction i
// is r - c_y - c_z ny, and a source x outside [0, nx) is x + nx of the row
// before or x - nx of the row after.  Only the wrap of the whole block needs a
// rule; rows with r in [ny + 2, ny nz - ny - 3] never reach it for any
// direction or row-end source ("interior rows", which include the y = 0 and
// y = ny-1 rows of all planes but the first two and last two).
__device__ __forceinline__ bool interior_row(const Geom& g, int y, int z) {
  const long long r = (long long)z * g.ny + y;
  return r >= g.ny + 2 && r <= (long long)g.ny * g.nz - g.ny - 3;
}

// Gather, for the V cells x0.. of row (y, z), population i from the cell
// SIGN*c_i away *before* it: SIGN = +1 reads x - c_i (streaming pull),
// SIGN = -1 reads x + c_i (the transpose of streaming).
//
// Interior rows: every direction is one aligned V-wide load of the source row at
// the lane's own chunk; the ten x-shifted directions add one aligned load of
// the adjacent chunk (the neighbour lane's, an L1 hit for all but one lane per
// warp) and splice the element crossing the chunk edge.  The adjacent-chunk
// addresses are clamped into the row, so the 29 loads carry no branches and can
// all be in flight together.  Cells x = 0 / x = nx-1 whose sources cross the
// row end then re-load through the wrap rule; the rows near the block's first
// and last planes (not interior) take every source through it.  Called for
// chunks with x0 < nx only.
template <typename S, typename R, int V, int SIGN>
__device__ __forceinline__ void gather_chunk(const S* __restrict__ arr, long long dstride,
                                             const Geom& g, const float* shift, float inv_scale,
                                             int x0, int y, int z, R (&vals)[Q][V]) {
  const bool active = true;
  if (interior_row(g, y, z)) {
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
          vals[i][0] = gload<S, R>(
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
              vals[i][k] = gload<S, R>(
                  arr + i * dstride +
                      wrap_off(g, g.nx - 1, y, z, -SIGN * cx(i), -SIGN * cy(i), -SIGN * cz(i)),
                  shift[i], inv_scale);
        }
    }
  } else if (active) {
    // rows near the first and last planes: every source through the wrap rule
#pragma unroll
    for (int k = 0; k < V; ++k) {
      const int x = min(x0 + k, g.nx - 1);
#pragma unroll
      for (int i = 0; i < Q; ++i)
        vals[i][k] = gload<S, R>(
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

// ---------------------------------------------------------------------------
// FP16S storage: populations stay packed (V halves per direction) from the
// load to the store, and bulk BGK cells collide on the stored deviations.
//
// The stored value is H_i = (f_i - w_i rho0) S, S = 2^10.  With
// delta = rho - rho0 = sum_i H_i / S and u = sum_i c_i H_i / (S rho) (the
// weights w_i carry no momentum), BGK f'_i = omega feq_i + (1 - omega) f_i with
// feq_i = w_i rho (1 + g_i) (equilibrium::SecondOrder, src/lbm/equilibrium.ur.h:
// 166-215) reads, on deviations,
//   H'_i = (1 - omega) H_i + omega S w_i (delta + rho g_i),
//   g_i = k_i + k_i^2 / 2 - 3 |u|^2 / 2,  k_i = 3 c_i . u,
// in FP32 without forming f_i = w_i rho0 + H_i / S: no shift or scale per
// population and no cancellation against w_i rho0.  Other ops convert to f_i,
// apply the generic operator and convert back; cells without an op keep their
// stored bits.

template <int V> struct HWord;
template <> struct HWord<2> { using type = unsigned; };
template <> struct HWord<4> { using type = uint2; };

template <int V>
__device__ __forceinline__ typename HWord<V>::type hload(const __half* p) {
  if constexpr (V == 4) return __ldg(reinterpret_cast<const uint2*>(p));
  else return __ldg(reinterpret_cast<const unsigned*>(p));
}
template <int V>
__device__ __forceinline__ void hstore(__half* p, const typename HWord<V>::type& w) {
  if constexpr (V == 4) *reinterpret_cast<uint2*>(p) = w;
  else *reinterpret_cast<unsigned*>(p) = w;
}
__device__ __forceinline__ unsigned hscalar(const __half* p) {
  return __ldg(reinterpret_cast<const unsigned short*>(p));
}
// 32-bit part holding halves k and k+1 (k even) of a word
__device__ __forceinline__ unsigned& hpart(unsigned& w, int) { return w; }
__device__ __forceinline__ unsigned& hpart(uint2& w, int k) { return k < 2 ? w.x : w.y; }
// half k of the word := bits h (low 16)
template <typename W>
__device__ __forceinline__ void hset(W& w, int k, unsigned h) {
  unsigned& q = hpart(w, k);
  q = (k & 1) ? __byte_perm(q, h, 0x5410) : __byte_perm(q, h, 0x3254);
}
// [a.hi, b.lo]: the halves on both sides of a 32-bit boundary
__device__ __forceinline__ unsigned hcross(unsigned a, unsigned b) {
  return __byte_perm(a, b, 0x5432);
}
// source chunk shifted by one cell: v = own chunk, w = chunk before (prev) or after (next)
__device__ __forceinline__ unsigned hsplice_prev(unsigned w, unsigned v) { return hcross(w, v); }
__device__ __forceinline__ unsigned hsplice_next(unsigned v, unsigned w) { return hcross(v, w); }
__device__ __forceinline__ uint2 hsplice_prev(uint2 w, uint2 v) {
  return make_uint2(hcross(w.y, v.x), hcross(v.x, v.y));
}
__device__ __forceinline__ uint2 hsplice_next(uint2 v, uint2 w) {
  return make_uint2(hcross(v.x, v.y), hcross(v.y, w.x));
}

// The V post-stream words of chunk x0 of row (y, z): the same loads and edge
// rules as gather_chunk (SIGN = +1), without conversion.  row_off, when given,
// holds i * dstride - cy_i * pitch - cz_i * plane for the block (the source
// row of direction i relative to the cell's own row).
//
// Row ends of interior rows: the source of x = 0 in a direction with c_x = +1 is
// x = nx-1 of the row before (y - c_y - 1), and that of x = nx-1 with
// c_x = -1 is x = 0 of the row after (y - c_y + 1); with at most two non-zero
// components per D3Q19 velocity the carry reaches z only when the y row wraps,
// and then c_z = 0.
// Rows near the block's first and last planes: every source through the wrap rule.
template <int V>
__device__ __forceinline__ void gather_words_wrap(const __half* __restrict__ arr,
                                                  long long dstride, const Geom& g, int x0,
                                                  int y, int z, typename HWord<V>::type (&h)[Q]) {
  using W = typename HWord<V>::type;
#pragma unroll
  for (int i = 0; i < Q; ++i) h[i] = W{};
#pragma unroll
  for (int k = 0; k < V; ++k) {
    const int x = min(x0 + k, g.nx - 1);
#pragma unroll
    for (int i = 0; i < Q; ++i)
      hset(h[i], k, hscalar(arr + i * dstride + wrap_off(g, x, y, z, -cx(i), -cy(i), -cz(i))));
  }
}

// Single-block handles (19 * dstride < 2^32), interior rows: the source word
// of direction i is src_dir[i] + cell (one wide multiply-add on a
// kernel-parameter base), the adjacent chunk at a fixed +-V (no clamp: the
// chunk before / after the row lies in the neighbouring row or the padding,
// inside the array, and row-end lanes replace that element anyway).
template <int V>
__device__ __forceinline__ void gather_words_dir(const StepParams& p, const Geom& g, int x0,
                                                 unsigned cell,
                                                 typename HWord<V>::type (&h)[Q]) {
  using W = typename HWord<V>::type;
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const __half* own = static_cast<const __half*>(p.src_dir[i]) + cell;
    const W v = hload<V>(own);
    if (cx(i) == 0) {
      h[i] = v;
    } else if (cx(i) > 0) {
      h[i] = hsplice_prev(hload<V>(own - V), v);
    } else {
      h[i] = hsplice_next(v, hload<V>(own + V));
    }
  }
  if (x0 == 0) {  // x = nx-1 of the row before the source row
    const unsigned e = cell - unsigned(g.pitch) + unsigned(g.nx - 1);
#pragma unroll
    for (int i = 1; i < Q; ++i)
      if (cx(i) > 0) hset(h[i], 0, hscalar(static_cast<const __half*>(p.src_dir[i]) + e));
  }
  const int klast = g.nx - 1 - x0;
  if (klast >= 0 && klast < V) {  // x = 0 of the row after the source row
    const unsigned e = cell + unsigned(g.pitch) - unsigned(x0);
#pragma unroll
    for (int i = 1; i < Q; ++i)
      if (cx(i) < 0) {
        const unsigned w = hscalar(static_cast<const __half*>(p.src_dir[i]) + e);
#pragma unroll
        for (int k = 0; k < V; ++k)
          if (k == klast) hset(h[i], k, w);
      }
  }
}

template <int V>
__device__ __forceinline__ void gather_words(const __half* __restrict__ arr, long long dstride,
                                             const Geom& g, int x0, int y, int z,
                                             const long long* __restrict__ row_off,
                                             typename HWord<V>::type (&h)[Q]) {
  using W = typename HWord<V>::type;
  if (interior_row(g, y, z)) {
    const __half* row = arr + g.base + (long long)y * g.pitch + (long long)z * g.plane;
    const int xprev = x0 >= V ? x0 - V : x0;
    const int xnext = x0 + V < g.nx ? x0 + V : x0;
    const __half* rowp[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      rowp[i] = row + (row_off ? row_off[i]
                               : i * dstride - (long long)cy(i) * g.pitch -
                                     (long long)cz(i) * g.plane);
      const W v = hload<V>(rowp[i] + x0);
      if (cx(i) == 0) {
        h[i] = v;
      } else if (cx(i) > 0) {
        h[i] = hsplice_prev(hload<V>(rowp[i] + xprev), v);
      } else {
        h[i] = hsplice_next(v, hload<V>(rowp[i] + xnext));
      }
    }
    if (x0 == 0) {  // x = nx-1 of the row before the source row
#pragma unroll
      for (int i = 1; i < Q; ++i)
        if (cx(i) > 0) hset(h[i], 0, hscalar(rowp[i] - g.pitch + (g.nx - 1)));
    }
    const int klast = g.nx - 1 - x0;
    if (klast >= 0 && klast < V) {  // x = 0 of the row after the source row
#pragma unroll
      for (int i = 1; i < Q; ++i)
        if (cx(i) < 0) {
          const unsigned e = hscalar(rowp[i] + g.pitch);
#pragma unroll
          for (int k = 0; k < V; ++k)
            if (k == klast) hset(h[i], k, e);
        }
    }
  } else {
    gather_words_wrap<V>(arr, dstride, g, x0, y, z, h);
  }
}

// Packed FP32 pairs: the two cells of a 32-bit half2 part travel as one float2
// through sm_100's two-wide FP32 instructions (one instruction per pair).
__device__ __forceinline__ float2 p2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {  // a - b, one rounding
  return __ffma2_rn(b, p2(-1.0f), a);
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
  return __ffma2_rn(a, b, c);
}

// BGK on deviations (see above) for two cells at once; H[] in and out in units
// of the stored value.  Every operation is an explicit two-wide instruction, so
// each cell's result is the same whichever cell shares its pair.
__device__ __forceinline__ void bgk_deviation2(float2 (&H)[Q], float omega, float rho0,
                                               float scale, float inv_scale) {
  float2 sp[Q], df[Q];  // pair sums / differences, index of the first of the pair
#pragma unroll
  for (int i = 1; i < Q; i += 2) {
    sp[i] = add2(H[i], H[i + 1]);
    df[i] = sub2(H[i], H[i + 1]);
  }
  const float2 sum = add2(add2(add2(add2(H[0], sp[1]), add2(sp[3], sp[5])),
                               add2(add2(sp[7], sp[9]), add2(sp[11], sp[13]))),
                          add2(sp[15], sp[17]));
  const float2 mx = add2(add2(add2(df[1], df[7]), add2(df[9], df[13])), df[15]);
  const float2 my = add2(add2(add2(df[3], df[7]), sub2(df[11], df[13])), df[17]);
  const float2 mz = sub2(add2(add2(df[5], df[9]), sub2(df[11], df[15])), df[17]);
  const float2 delta = mul2(sum, p2(inv_scale));
  const float2 rho = add2(p2(rho0), delta);
  // 1 / (S rho)
  const float2 ir = make_float2(__fdividef(inv_scale, rho.x), __fdividef(inv_scale, rho.y));
  const float2 ux = mul2(mx, ir), uy = mul2(my, ir), uz = mul2(mz, ir);
  const float2 q = mul2(p2(-1.5f), fma2(ux, ux, fma2(uy, uy, mul2(uz, uz))));
  const float2 c1 = p2(1.0f - omega);
  const float2 W0 = p2(omega * scale * (1.0f / 3.0f));
  const float2 W1 = p2(omega * scale * (1.0f / 18.0f));
  const float2 W2 = p2(omega * scale * (1.0f / 36.0f));
  const float2 d0 = mul2(W0, delta), d1 = mul2(W1, delta), d2 = mul2(W2, delta);
  const float2 r0 = mul2(W0, rho), r1 = mul2(W1, rho), r2 = mul2(W2, rho);
  const float2 k1 = mul2(p2(3.0f), ux), k3 = mul2(p2(3.0f), uy), k5 = mul2(p2(3.0f), uz);
  float2 k[Q];
  k[1] = k1;
  k[3] = k3;
  k[5] = k5;
  k[7] = add2(k1, k3);
  k[9] = add2(k1, k5);
  k[11] = add2(k3, k5);
  k[13] = sub2(k1, k3);
  k[15] = sub2(k1, k5);
  k[17] = sub2(k3, k5);
  H[0] = fma2(r0, q, fma2(c1, H[0], d0));
#pragma unroll
  for (int i = 1; i < Q; i += 2) {
    const float2 dw = i < 7 ? d1 : d2;
    const float2 rw = i < 7 ? r1 : r2;
    const float2 e = fma2(mul2(p2(0.5f), k[i]), k[i], q);
    H[i] = fma2(rw, add2(e, k[i]), fma2(c1, H[i], dw));
    H[i + 1] = fma2(rw, sub2(e, k[i]), fma2(c1, H[i + 1], dw));
  }
}


// k_i = 3 c_i . u of direction i (odd i; its pair partner i + 1 has -k_i)
__device__ __forceinline__ float2 kdir2(int i, float2 k1, float2 k3, float2 k5) {
  return i == 1 ? k1 : i == 3 ? k3 : i == 5 ? k5 : i == 7 ? add2(k1, k3) : i == 9 ? add2(k1, k5)
       : i == 11 ? add2(k3, k5) : i == 13 ? sub2(k1, k3) : i == 15 ? sub2(k1, k5) : sub2(k3, k5);
}

// Two-rate MRT on deviations (pair form): every non-conserved moment outside
// the shear set relaxes at s_g = p.mrt_sg, so M^-1 S M N = s_g N +
// (omega - s_g) P N with P the projection on the five shear moments (the
// conserved moments of N vanish up to FP32 rounding, as in the BGK form).  The
// shear moments are even: the pair sums of N give them, and both members of a
// pair get the same correction.  With E_i = S w_i (delta + rho (e_i +- k_i)):
//   H'_i = (1 - s_g) H_i + s_g E_i - sum_shear M_ki mu_k,
//   mu_k = (omega - s_g) / |M_k|^2 * sum_pairs M_ki (N_i + N_opp(i)).
// Only the five moment sums live across the two passes over the pairs (the
// pair terms are recomputed), which keeps it inside the step kernels'
// register budget.  Explicit two-wide operations, as in mrt_deviation2.
__device__ __forceinline__ void mrt_two_rate2(const StepParams& p, float2 (&H)[Q], float omega,
                                              float2 rho, float2 delta, float2 q, float2 k1,
                                              float2 k3, float2 k5) {
  constexpr int SH[5] = {9, 11, 13, 14, 15};
  const float s0 = p.scale * (1.0f / 3.0f), s1 = p.scale * (1.0f / 18.0f),
              s2 = p.scale * (1.0f / 36.0f);
  const float sg = p.mrt_sg;
  float2 m[5];
#pragma unroll
  for (int j = 0; j < 5; ++j) m[j] = p2(0.0f);
#pragma unroll
  for (int i = 1; i < Q; i += 2) {
    const float sw = i < 7 ? s1 : s2;
    const float2 k = kdir2(i, k1, k3, k5);
    const float2 t = fma2(rho, fma2(mul2(p2(0.5f), k), k, q), delta);
    const float2 a = fma2(p2(-2.0f * sw), t, add2(H[i], H[i + 1]));  // N_i + N_opp(i)
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      const int c = mrt_m(SH[j], i);
      if (c == 1) m[j] = add2(m[j], a);
      else if (c == -1) m[j] = sub2(m[j], a);
      else if (c != 0) m[j] = fma2(p2(float(c)), a, m[j]);
    }
  }
#pragma unroll
  for (int j = 0; j < 5; ++j) m[j] = mul2(m[j], p2((omega - sg) * (1.0f / float(mrt_norm_lit(SH[j])))));
  const float2 keep = p2(1.0f - sg);
  static_assert(mrt_m(9, 0) == 0 && mrt_m(11, 0) == 0 && mrt_m(13, 0) == 0 &&
                    mrt_m(14, 0) == 0 && mrt_m(15, 0) == 0,
                "shear moments leave the rest population alone");
  H[0] = fma2(keep, H[0], mul2(p2(sg * s0), fma2(rho, q, delta)));
#pragma unroll
  for (int i = 1; i < Q; i += 2) {
    const float sw = sg * (i < 7 ? s1 : s2);
    const float2 k = kdir2(i, k1, k3, k5);
    const float2 t = fma2(rho, fma2(mul2(p2(0.5f), k), k, q), delta);
    const float2 rk = mul2(rho, k);
    float2 corr = p2(0.0f);
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      const int c = mrt_m(SH[j], i);
      if (c == 1) corr = add2(corr, m[j]);
      else if (c == -1) corr = sub2(corr, m[j]);
      else if (c != 0) corr = fma2(p2(float(c)), m[j], corr);
    }
    H[i] = sub2(fma2(keep, H[i], mul2(p2(sw), add2(t, rk))), corr);
    H[i + 1] = sub2(fma2(keep, H[i + 1], mul2(p2(sw), sub2(t, rk))), corr);
  }
}

// MRT on deviations for two cells at once (the pair form of bgk_deviation2):
// the non-equilibrium part N = H - E in stored units, the 15 non-conserved
// moments of N, their relaxation and the back-transform, every operation one
// two-wide FP32 instruction (explicit fma2 / add2 / mul2, no contraction left
// to the compiler), so each cell's result is the same whichever cell shares
// its pair.  Every FP16S MRT bulk cell goes through it (a lone one on a
// duplicated lane).
template <int MODEL>
__device__ __forceinline__ void mrt_deviation2(const StepParams& p, float2 (&H)[Q], float omega) {
  float2 sp[Q], df[Q];
#pragma unroll
  for (int i = 1; i < Q; i += 2) {
    sp[i] = add2(H[i], H[i + 1]);
    df[i] = sub2(H[i], H[i + 1]);
  }
  const float2 sum = add2(add2(add2(add2(H[0], sp[1]), add2(sp[3], sp[5])),
                               add2(add2(sp[7], sp[9]), add2(sp[11], sp[13]))),
                          add2(sp[15], sp[17]));
  const float2 mx = add2(add2(add2(df[1], df[7]), add2(df[9], df[13])), df[15]);
  const float2 my = add2(add2(add2(df[3], df[7]), sub2(df[11], df[13])), df[17]);
  const float2 mz = sub2(add2(add2(df[5], df[9]), sub2(df[11], df[15])), df[17]);
  const float2 delta = mul2(sum, p2(p.inv_scale));
  const float2 rho = add2(p2(p.rho0), delta);
  const float2 ir = make_float2(__fdividef(p.inv_scale, rho.x), __fdividef(p.inv_scale, rho.y));
  const float2 ux = mul2(mx, ir), uy = mul2(my, ir), uz = mul2(mz, ir);
  const float2 q = mul2(p2(-1.5f), fma2(ux, ux, fma2(uy, uy, mul2(uz, uz))));
  const float2 k1 = mul2(p2(3.0f), ux), k3 = mul2(p2(3.0f), uy), k5 = mul2(p2(3.0f), uz);
  float2 k[Q];
  k[1] = k1;
  k[3] = k3;
  k[5] = k5;
  k[7] = add2(k1, k3);
  k[9] = add2(k1, k5);
  k[11] = add2(k3, k5);
  k[13] = sub2(k1, k3);
  k[15] = sub2(k1, k5);
  k[17] = sub2(k3, k5);
  // N_i = H_i - S w_i (delta + rho g_i); pair sums a and differences b of N
  const float s0 = p.scale * (1.0f / 3.0f), s1 = p.scale * (1.0f / 18.0f),
              s2 = p.scale * (1.0f / 36.0f);
  const float2 n0 = fma2(p2(-s0), fma2(rho, q, delta), H[0]);
  if constexpr (MODEL == MODEL_MRT2) {  // host: p.mrt_sg != 0
    mrt_two_rate2(p, H, omega, rho, delta, q, k1, k3, k5);
    return;
  }
  float2 a[9], b[9];
#pragma unroll
  for (int i = 1; i < Q; i += 2) {
    const float sw = i < 7 ? s1 : s2;
    const float2 e = fma2(mul2(p2(0.5f), k[i]), k[i], q);
    const float2 n1 = fma2(p2(-sw), fma2(rho, add2(e, k[i]), delta), H[i]);
    const float2 n2 = fma2(p2(-sw), fma2(rho, sub2(e, k[i]), delta), H[i + 1]);
    a[i / 2] = add2(n1, n2);
    b[i / 2] = sub2(n1, n2);
  }
  // mu_k = s_k / |M_k|^2 * (M_k . N) over the non-conserved moments
  float2 mu[Q];
#pragma unroll
  for (int kk = 0; kk < Q; ++kk) {
    if (mrt_conserved(kk)) {
      mu[kk] = p2(0.0f);
      continue;
    }
    float2 m = p2(0.0f);
    if (mrt_even(kk)) {
      if (mrt_m(kk, 0) != 0) m = mul2(p2(float(mrt_m(kk, 0))), n0);
#pragma unroll
      for (int pp = 0; pp < 9; ++pp) {
        const int c = mrt_m(kk, 2 * pp + 1);
        if (c == 1) m = add2(m, a[pp]);
        else if (c == -1) m = sub2(m, a[pp]);
        else if (c != 0) m = fma2(p2(float(c)), a[pp], m);
      }
    } else {
#pragma unroll
      for (int pp = 0; pp < 9; ++pp) {
        const int c = mrt_m(kk, 2 * pp + 1);
        if (c == 1) m = add2(m, b[pp]);
        else if (c == -1) m = sub2(m, b[pp]);
        else if (c != 0) m = fma2(p2(float(c)), b[pp], m);
      }
    }
    const float sk = mrt_shear(kk) ? omega * (1.0f / float(mrt_norm_lit(kk)))
                                   : float(p.s_over_norm[kk]);
    mu[kk] = mul2(m, p2(sk));
  }
  // back-transform: H_i -= sum_k M[k][i] mu_k
  float2 d0 = p2(0.0f);
#pragma unroll
  for (int kk = 0; kk < Q; ++kk)
    if (mrt_even(kk) && !mrt_conserved(kk) && mrt_m(kk, 0) != 0)
      d0 = fma2(p2(float(mrt_m(kk, 0))), mu[kk], d0);
  H[0] = sub2(H[0], d0);
#pragma unroll
  for (int pp = 0; pp < 9; ++pp) {
    float2 e = p2(0.0f), o = p2(0.0f);
#pragma unroll
    for (int kk = 0; kk < Q; ++kk) {
      if (mrt_conserved(kk)) continue;
      const int c = mrt_m(kk, 2 * pp + 1);
      if (c == 0) continue;
      if (mrt_even(kk)) e = c == 1 ? add2(e, mu[kk]) : c == -1 ? sub2(e, mu[kk])
                                                               : fma2(p2(float(c)), mu[kk], e);
      else o = c == 1 ? add2(o, mu[kk]) : c == -1 ? sub2(o, mu[kk])
                                                  : fma2(p2(float(c)), mu[kk], o);
    }
    H[2 * pp + 1] = sub2(H[2 * pp + 1], add2(e, o));
    H[2 * pp + 2] = sub2(H[2 * pp + 2], sub2(e, o));
  }
}

// MRT (collision::MRT_Feq_RhoU) on deviations: H <- H - M^-1 S M N, given the
// non-equilibrium part N.
__device__ __forceinline__ void mrt_relax_neq(const StepParams& p, float (&H)[Q], float omega,
                                              const float (&N)[Q]) {
  float a[9], b[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    a[q] = N[2 * q + 1] + N[2 * q + 2];
    b[q] = N[2 * q + 1] - N[2 * q + 2];
  }
  float s[Q];
#pragma unroll
  for (int k = 0; k < Q; ++k)
    s[k] = mrt_shear(k) ? omega * (1.0f / float(mrt_norm_lit(k))) : float(p.s_over_norm[k]);
  mrt_relax<float>(H, N[0], a, b, s);
}

// Smagorinsky BGK (collision::SmagorinskyBGK) on deviations: Pi^neq =
// sum c c N / S, the effective rate from it, H <- H - omega_eff N, given the
// cell's density and non-equilibrium part (the FP32S path).  Products that
// meet additions are explicit, so no contraction is left to the compiler.
__device__ __forceinline__ void les_relax_neq(const StepParams& p, float (&H)[Q], float omega,
                                              float rho, const float (&N)[Q]) {
  const float is = p.inv_scale;  // a power of two: the scaling is exact
  const float p0 = is * ((((N[1] + N[2]) + (N[7] + N[8])) + ((N[9] + N[10]) + (N[13] + N[14]))) +
                         (N[15] + N[16]));
  const float p1 = is * ((N[7] + N[8]) - (N[13] + N[14]));
  const float p2 = is * ((N[9] + N[10]) - (N[15] + N[16]));
  const float p3 = is * ((((N[3] + N[4]) + (N[7] + N[8])) + ((N[11] + N[12]) + (N[13] + N[14]))) +
                         (N[17] + N[18]));
  const float p4 = is * ((N[11] + N[12]) - (N[17] + N[18]));
  const float p5 = is * ((((N[5] + N[6]) + (N[9] + N[10])) + ((N[11] + N[12]) + (N[15] + N[16]))) +
                         (N[17] + N[18]));
  float nsq = __fmul_rn(p0, p0);
  nsq = fmaf(__fmul_rn(p1, p1), 2.0f, nsq);
  nsq = fmaf(__fmul_rn(p2, p2), 2.0f, nsq);
  nsq = fmaf(p3, p3, nsq);
  nsq = fmaf(__fmul_rn(p4, p4), 2.0f, nsq);
  nsq = fmaf(p5, p5, nsq);
  const float rt_mol = 1.0f / omega;
  const float coeff = float(p.cs_coeff) / rho;
  const float rt_tur = __fmul_rn(0.5f, sqrtf(fmaf(rt_mol, rt_mol, coeff * sqrtf(nsq))) - rt_mol);
  const float eomega = 1.0f / (rt_mol + rt_tur);
#pragma unroll
  for (int i = 0; i < Q; ++i) H[i] = fmaf(-eomega, N[i], H[i]);
}


// Smagorinsky BGK on deviations for two cells at once (the pair form of
// bgk_deviation2).  Pi^neq needs no N array: with E the equilibrium part,
// sum_i c_a c_b E_i / S = delta / 3 [a = b] + rho u_a u_b exactly for D3Q19,
// so Pi^neq_ab = sum_i c_a c_b H_i / S - delta / 3 [a = b] - rho u_a u_b, and
// c_a c_b is even, so the pair sums of H give it.  The effective rate
// 1 / (tau + tau_t), tau_t = (sqrt(tau^2 + C |Pi| / rho) - tau) / 2
// (collision::SmagorinskyBGK, src/lbm/collisionLES.h:36-62) is then a per-lane
// scalar, and the update is BGK's H' = (1 - w) H + w E with w per lane.  The
// square roots and reciprocals use the hardware approximations (MUFU, about
// one FP32 ulp), far below the binary16 spacing the result is stored at; every
// other operation is an explicit two-wide instruction, so each cell's result
// is the same whichever cell shares its pair.
__device__ __forceinline__ float les_rate(float nsq, float rho_inv, float rt_mol, float cs_coeff) {
  const float norm = nsq > 0.0f ? __fmul_rn(nsq, rsqrtf(nsq)) : 0.0f;
  const float t = __fmaf_rn(rt_mol, rt_mol, __fmul_rn(__fmul_rn(cs_coeff, rho_inv), norm));
  const float rt_tur = __fmul_rn(0.5f, __fmul_rn(t, rsqrtf(t)) - rt_mol);
  return __fdividef(1.0f, rt_mol + rt_tur);
}

__device__ __forceinline__ void les_deviation2(const StepParams& p, float2 (&H)[Q], float omega) {
  float2 sp[Q], df[Q];
#pragma unroll
  for (int i = 1; i < Q; i += 2) {
    sp[i] = add2(H[i], H[i + 1]);
    df[i] = sub2(H[i], H[i + 1]);
  }
  const float2 sum = add2(add2(add2(add2(H[0], sp[1]), add2(sp[3], sp[5])),
                               add2(add2(sp[7], sp[9]), add2(sp[11], sp[13]))),
                          add2(sp[15], sp[17]));
  const float2 mx = add2(add2(add2(df[1], df[7]), add2(df[9], df[13])), df[15]);
  const float2 my = add2(add2(add2(df[3], df[7]), sub2(df[11], df[13])), df[17]);
  const float2 mz = sub2(add2(add2(df[5], df[9]), sub2(df[11], df[15])), df[17]);
  const float is = p.inv_scale, scale = p.scale;
  const float2 delta = mul2(sum, p2(is));
  const float2 rho = add2(p2(p.rho0), delta);
  const float2 ir = make_float2(__fdividef(is, rho.x), __fdividef(is, rho.y));  // 1 / (S rho)
  const float2 ux = mul2(mx, ir), uy = mul2(my, ir), uz = mul2(mz, ir);
  // Pi^neq in f units
  const float2 d3 = mul2(delta, p2(1.0f / 3.0f));
  const float2 rux = mul2(rho, ux), ruy = mul2(rho, uy);
  const float2 pxx = sub2(fma2(add2(add2(add2(sp[1], sp[7]), add2(sp[9], sp[13])), sp[15]), p2(is),
                              mul2(p2(-1.0f), d3)), mul2(rux, ux));
  const float2 pyy = sub2(fma2(add2(add2(add2(sp[3], sp[7]), add2(sp[11], sp[13])), sp[17]), p2(is),
                              mul2(p2(-1.0f), d3)), mul2(ruy, uy));
  const float2 pzz = sub2(fma2(add2(add2(add2(sp[5], sp[9]), add2(sp[11], sp[15])), sp[17]), p2(is),
                              mul2(p2(-1.0f), d3)), mul2(mul2(rho, uz), uz));
  const float2 pxy = sub2(mul2(sub2(sp[7], sp[13]), p2(is)), mul2(rux, uy));
  const float2 pxz = sub2(mul2(sub2(sp[9], sp[15]), p2(is)), mul2(rux, uz));
  const float2 pyz = sub2(mul2(sub2(sp[11], sp[17]), p2(is)), mul2(ruy, uz));
  float2 nsq = mul2(pxx, pxx);
  nsq = fma2(mul2(pxy, pxy), p2(2.0f), nsq);
  nsq = fma2(mul2(pxz, pxz), p2(2.0f), nsq);
  nsq = fma2(pyy, pyy, nsq);
  nsq = fma2(mul2(pyz, pyz), p2(2.0f), nsq);
  nsq = fma2(pzz, pzz, nsq);
  const float rt_mol = __fdividef(1.0f, omega);
  const float csc = float(p.cs_coeff);
  const float2 w = make_float2(les_rate(nsq.x, __fmul_rn(ir.x, scale), rt_mol, csc),
                               les_rate(nsq.y, __fmul_rn(ir.y, scale), rt_mol, csc));
  // BGK update with the per-lane rate w (bgk_deviation2's form)
  const float2 q = mul2(p2(-1.5f), fma2(ux, ux, fma2(uy, uy, mul2(uz, uz))));
  const float2 c1 = sub2(p2(1.0f), w);
  const float2 W0 = mul2(w, p2(scale * (1.0f / 3.0f)));
  const float2 W1 = mul2(w, p2(scale * (1.0f / 18.0f)));
  const float2 W2 = mul2(w, p2(scale * (1.0f / 36.0f)));
  const float2 d0 = mul2(W0, delta), d1 = mul2(W1, delta), d2 = mul2(W2, delta);
  const float2 r0 = mul2(W0, rho), r1 = mul2(W1, rho), r2 = mul2(W2, rho);
  const float2 k1 = mul2(p2(3.0f), ux), k3 = mul2(p2(3.0f), uy), k5 = mul2(p2(3.0f), uz);
  H[0] = fma2(r0, q, fma2(c1, H[0], d0));
#pragma unroll
  for (int i = 1; i < Q; i += 2) {
    const float2 dw = i < 7 ? d1 : d2;
    const float2 rw = i < 7 ? r1 : r2;
    const float2 k = kdir2(i, k1, k3, k5);
    const float2 e = fma2(mul2(p2(0.5f), k), k, q);
    H[i] = fma2(rw, add2(e, k), fma2(c1, H[i], dw));
    H[i + 1] = fma2(rw, sub2(e, k), fma2(c1, H[i + 1], dw));
  }
}

// ---------------------------------------------------------------------------
// FP32S storage (dev32): d_i = f_i - rho0 w_i in FP32, collided as stored, the
// FP16S deviation form at full FP32 width with IEEE divisions.

// delta = sum d (= rho - rho0), rho, den = rho + alpha/2 and u = sum c d / den
// (the weights carry no momentum, so sum c d = sum c f); alpha = 0 gives
// moment::rhoU, alpha > 0 the forced moments of the Brinkman model.
__device__ __forceinline__ void dev_moments(const float (&d)[Q], float rho0, float alpha,
                                            float& delta, float& rho, float& den, float& ux,
                                            float& uy, float& uz) {
  float sp[Q], df[Q];
#pragma unroll
  for (int i = 1; i < Q; i += 2) {
    sp[i] = d[i] + d[i + 1];
    df[i] = d[i] - d[i + 1];
  }
  delta = ((d[0] + sp[1]) + (sp[3] + sp[5])) + ((sp[7] + sp[9]) + (sp[11] + sp[13])) +
          (sp[15] + sp[17]);
  const float mx = (df[1] + df[7]) + (df[9] + df[13]) + df[15];
  const float my = (df[3] + df[7]) + (df[11] - df[13]) + df[17];
  const float mz = (df[5] + df[9]) + (df[11] - df[15]) - df[17];
  rho = rho0 + delta;
  den = fmaf(0.5f, alpha, rho);
  ux = mx / den;
  uy = my / den;
  uz = mz / den;
}

// k_i = 3 c_i.u for the first direction of each opposite pair (k of i + 1 is -k_i).
__device__ __forceinline__ void dev_k(float ux, float uy, float uz, float (&k)[Q]) {
  const float k1 = __fmul_rn(3.0f, ux), k3 = __fmul_rn(3.0f, uy), k5 = __fmul_rn(3.0f, uz);
  k[1] = k1;
  k[3] = k3;
  k[5] = k5;
  k[7] = k1 + k3;
  k[9] = k1 + k5;
  k[11] = k3 + k5;
  k[13] = k1 - k3;
  k[15] = k1 - k5;
  k[17] = k3 - k5;
}

// Non-equilibrium part N_i = d_i - E_i with E_i = feq_i - rho0 w_i
// = w_i (delta + rho g_i), g_i = k_i + k_i^2/2 - 3|u|^2/2 (SecondOrder).
__device__ __forceinline__ void dev_neq(const float (&d)[Q], float delta, float rho, float ux,
                                        float uy, float uz, float (&N)[Q]) {
  const float q = -1.5f * fmaf(ux, ux, fmaf(uy, uy, __fmul_rn(uz, uz)));
  float k[Q];
  dev_k(ux, uy, uz, k);
  N[0] = fmaf(-(1.0f / 3.0f), fmaf(rho, q, delta), d[0]);
#pragma unroll
  for (int i = 1; i < Q; i += 2) {
    const float w = i < 7 ? 1.0f / 18.0f : 1.0f / 36.0f;
    const float e = fmaf(0.5f * k[i], k[i], q);
    N[i] = fmaf(-w, fmaf(rho, e + k[i], delta), d[i]);
    N[i + 1] = fmaf(-w, fmaf(rho, e - k[i], delta), d[i + 1]);
  }
}

// collision::BGKForce with the Brinkman drag (bgk_brinkman) on deviations:
//   d'_i = (1 - omega) d_i + omega w_i (delta + rho g_i) + (1 - omega/2) F_i,
// F_i = w_i F.(3 (c_i - u) + 9 (c_i.u) c_i) with F = -alpha u, which is
// -alpha w_i (k_i + k_i^2 - 3|u|^2); the part of both terms odd in c_i is
// (omega rho - (1 - omega/2) alpha) k_i.
__device__ __forceinline__ void brinkman_deviation(const StepParams& p, float (&d)[Q],
                                                   float omega, float alpha) {
  float delta, rho, den, ux, uy, uz;
  dev_moments(d, p.rho0, alpha, delta, rho, den, ux, uy, uz);
  const float u2 = fmaf(ux, ux, fmaf(uy, uy, __fmul_rn(uz, uz)));
  const float q = -1.5f * u2, t = -3.0f * u2;
  const float c1 = 1.0f - omega;
  const float fa = __fmul_rn(1.0f - 0.5f * omega, alpha);
  const float odd = fmaf(omega, rho, -fa);
  float k[Q];
  dev_k(ux, uy, uz, k);
  d[0] = fmaf(c1, d[0], (1.0f / 3.0f) * fmaf(omega, fmaf(rho, q, delta), -__fmul_rn(fa, t)));
#pragma unroll
  for (int i = 1; i < Q; i += 2) {
    const float w = i < 7 ? 1.0f / 18.0f : 1.0f / 36.0f;
    const float e = fmaf(0.5f * k[i], k[i], q);
    const float h = fmaf(k[i], k[i], t);
    const float ge = fmaf(omega, fmaf(rho, e, delta), -__fmul_rn(fa, h));
    const float go = __fmul_rn(odd, k[i]);
    d[i] = fmaf(c1, d[i], w * (ge + go));
    d[i + 1] = fmaf(c1, d[i + 1], w * (ge - go));
  }
}

// One FP32S cell by its op.  Bounce-back and the moving wall act on the
// deviations as they act on f (w_i = w_opp(i), and the wall term is additive);
// the field-velocity BGK goes through f.
template <int MODEL>
__device__ __forceinline__ void collide_dev32(const StepParams& p, int op, float (&d)[Q],
                                              long long cell, float omega) {
  if (op == OP_NONE) return;
  if (op == OP_BB || op == OP_MBB) {
    apply_wall_op<float>(p, op, d, cell, omega);
    return;
  }
  if (op == OP_BULK) {
    if constexpr (MODEL == MODEL_BRINKMAN) {
      brinkman_deviation(p, d, omega, static_cast<const float*>(p.alpha)[cell]);
    } else {
      float delta, rho, den, ux, uy, uz, N[Q];
      dev_moments(d, p.rho0, 0.0f, delta, rho, den, ux, uy, uz);
      dev_neq(d, delta, rho, ux, uy, uz, N);
      if constexpr (is_mrt(MODEL)) {
        mrt_relax_neq(p, d, omega, N);
      } else if constexpr (MODEL == MODEL_LES) {
        les_relax_neq(p, d, omega, rho, N);
      } else {
#pragma unroll
        for (int i = 0; i < Q; ++i) d[i] = fmaf(-omega, N[i], d[i]);
      }
    }
    return;
  }
  float f[Q];
#pragma unroll
  for (int i = 0; i < Q; ++i) f[i] = d[i] + p.shift[i];
  apply_wall_op<float>(p, op, f, cell, omega);
#pragma unroll
  for (int i = 0; i < Q; ++i) d[i] = f[i] - p.shift[i];
}

// One cell: bulk BGK through the pair form (both lanes the same cell), bulk
// MRT and LES on deviations, other ops through the generic operator on
// f = w_i rho0 + H / S.
template <int MODEL>
__device__ __forceinline__ void collide_deviation(const StepParams& p, int op, float (&H)[Q],
                                                  long long cell, float omega) {
  if (op == OP_NONE) return;
  if constexpr (is_mrt(MODEL)) {
    if (op == OP_BULK) {
      float2 H2[Q];
#pragma unroll
      for (int i = 0; i < Q; ++i) H2[i] = p2(H[i]);
      mrt_deviation2<MODEL>(p, H2, omega);
#pragma unroll
      for (int i = 0; i < Q; ++i) H[i] = H2[i].x;
      return;
    }
  }
  if constexpr (MODEL == MODEL_LES) {
    if (op == OP_BULK) {
      float2 H2[Q];
#pragma unroll
      for (int i = 0; i < Q; ++i) H2[i] = p2(H[i]);
      les_deviation2(p, H2, omega);
#pragma unroll
      for (int i = 0; i < Q; ++i) H[i] = H2[i].x;
      return;
    }
  }
  if constexpr (MODEL == MODEL_BGK) {
    if (op == OP_BULK) {
      float2 H2[Q];
#pragma unroll
      for (int i = 0; i < Q; ++i) H2[i] = p2(H[i]);
      bgk_deviation2(H2, omega, p.rho0, p.scale, p.inv_scale);
#pragma unroll
      for (int i = 0; i < Q; ++i) H[i] = H2[i].x;
      return;
    }
  }
  float f[Q];
#pragma unroll
  for (int i = 0; i < Q; ++i) f[i] = fmaf(H[i], p.inv_scale, p.shift[i]);
  apply_op<float, MODEL>(p, op, f, cell, omega);
#pragma unroll
  for (int i = 0; i < Q; ++i) H[i] = fmaf(f[i], p.scale, -p.shift[i] * p.scale);
}

// Stochastic rounding of FP16S stores.  cvt.rs.f16x2.f32 (sm_100a) adds a
// random fraction of the last kept bit to each value's magnitude and then
// truncates, so E[stored] = value: bits [12:0] of its random word are the
// fraction of the low half, bits [28:16] that of the high half.  Round to
// nearest can make the same error step after step where the flow changes
// slowly, and that error adds up: MRT FP16S on the 512^3 cavity drifts
// linearly to a velocity error of 1.2e-3 against FP64 after 2000 steps, while
// BGK, and MRT with every rate at 1/tau, stay at 3.2e-4 (so the drift comes
// with MRT's other rates of 1.2); stochastic rounding removes it (2.2e-4).
// The random fraction of a cell comes from a hash of four of the binary16
// values it pulled (directions 0, 1, 9, 18), XORed with a per-direction key
// that has the same 13 bits in both fields.  Those inputs are the same bits in
// every kernel (the FP32 collision results need not be: a one-ulp difference
// of a fused multiply-add would change a hash of them entirely), a cell's bits
// do not depend on the cell it is paired with or on its half, so every FP16S
// kernel still gives the same result.  The inputs change from step to step
// because the neighbours' stores are themselves rounded at random; only a
// state that needs no rounding at all (a fluid at rest) stays put.  A value
// that is already a binary16 number (a cell without an op) is stored unchanged.
__device__ __forceinline__ unsigned sr_hash(unsigned a, unsigned b) {
  unsigned h = a * 0x9e3779b9u ^ b;
  h ^= h >> 15;
  h *= 0x2c1b3c6du;
  h ^= h >> 12;
  return h;
}
__device__ __forceinline__ constexpr unsigned sr_key(int i) {
  return ((0x9e3u * unsigned(i) + 0x3b5u) & 0x1fffu) * 0x00010001u;
}
// lo -> low half, hi -> high half (the order of __floats2half2_rn)
__device__ __forceinline__ unsigned cvt_rs_half2(float lo, float hi, unsigned rbits) {
  unsigned d;
  asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(rbits));
  return d;
}
// Random word of a pair from its pulled words w0, w1, w9, w18 (directions 0,
// 1, 9, 18; low halves = cell a, high halves = cell b): low field from cell
// a's hash, high field from cell b's.
__device__ __forceinline__ unsigned sr_pair(unsigned w0, unsigned w1, unsigned w9,
                                            unsigned w18) {
  const unsigned ha = sr_hash(__byte_perm(w0, w1, 0x5410), __byte_perm(w9, w18, 0x5410));
  const unsigned hb = sr_hash(__byte_perm(w0, w1, 0x7632), __byte_perm(w9, w18, 0x7632));
  return __byte_perm(ha, hb, 0x5410);
}

// Collide one FP16S chunk in place, cells processed in pairs (the two halves
// of a 32-bit part); fl holds the V cells' flags.
template <int MODEL, int V>
__device__ __forceinline__ void collide_half(const StepParams& p, float omega, long long cell0,
                                             const uint8_t (&fl)[V],
                                             typename HWord<V>::type (&h)[Q]) {
#pragma unroll
  for (int k = 0; k < V; k += 2) {
    const int opa = select_op(p, fl[k]), opb = select_op(p, fl[k + 1]);
    if (opa == OP_NONE && opb == OP_NONE) continue;
    // stochastic rounding: every FP16S model (FP16S has no Brinkman kernels)
    constexpr bool kSR = MODEL != MODEL_BRINKMAN;
    const bool sr = kSR && p.fp16_round;
    unsigned c = 0u;
    if (sr) c = sr_pair(hpart(h[0], k), hpart(h[1], k), hpart(h[9], k), hpart(h[18], k));
    if ((MODEL == MODEL_BGK || is_mrt(MODEL) || MODEL == MODEL_LES) && opa == OP_BULK &&
        opb == OP_BULK) {
      float2 H2[Q];
#pragma unroll
      for (int i = 0; i < Q; ++i) {
        const unsigned q = hpart(h[i], k);
        H2[i] = __half22float2(*reinterpret_cast<const __half2*>(&q));
      }
      if constexpr (is_mrt(MODEL)) mrt_deviation2<MODEL>(p, H2, omega);
      else if constexpr (MODEL == MODEL_LES) les_deviation2(p, H2, omega);
      else bgk_deviation2(H2, omega, p.rho0, p.scale, p.inv_scale);
      if (sr) {
#pragma unroll
        for (int i = 0; i < Q; ++i) hpart(h[i], k) = cvt_rs_half2(H2[i].x, H2[i].y, c ^ sr_key(i));
      } else {
#pragma unroll
        for (int i = 0; i < Q; ++i) {
          const __half2 r = __float22half2_rn(H2[i]);
          hpart(h[i], k) = *reinterpret_cast<const unsigned*>(&r);
        }
      }
      continue;
    }
    float a[Q], b[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      const unsigned q = hpart(h[i], k);
      const __half2 h2 = *reinterpret_cast<const __half2*>(&q);
      a[i] = __low2float(h2);
      b[i] = __high2float(h2);
    }
    collide_deviation<MODEL>(p, opa, a, cell0 + k, omega);
    collide_deviation<MODEL>(p, opb, b, cell0 + k + 1, omega);
    // a cell without an op round-trips exactly (half -> float -> half), in
    // either rounding
    if (sr) {
#pragma unroll
      for (int i = 0; i < Q; ++i) hpart(h[i], k) = cvt_rs_half2(a[i], b[i], c ^ sr_key(i));
    } else {
#pragma unroll
      for (int i = 0; i < Q; ++i) {
        const __half2 r = __floats2half2_rn(a[i], b[i]);
        hpart(h[i], k) = *reinterpret_cast<const unsigned*>(&r);
      }
    }
  }
}

// One FP16S chunk: flags, collision, one V-wide store per direction.
template <int MODEL, int V>
__device__ __forceinline__ void collide_store_half(const StepParams& p, float omega,
                                                   long long cell0,
                                                   typename HWord<V>::type (&h)[Q]) {
  __half* __restrict__ dst = static_cast<__half*>(p.dst);
  uint8_t fl[V];
  load_flags<V>(p.flags + cell0, fl);
  collide_half<MODEL, V>(p, omega, cell0, fl, h);
#pragma unroll
  for (int i = 0; i < Q; ++i) hstore<V>(dst + i * p.dstride + cell0, h[i]);
}

template <int MODEL, int V>
__device__ __forceinline__ void pull_chunk_half(const StepParams& p, const Geom& g, float omega,
                                                int x0, int y, int z) {
  typename HWord<V>::type h[Q];
  const __half* src = static_cast<const __half*>(p.src);
  const long long cell0 = g.base + (long long)y * g.pitch + (long long)z * g.plane + x0;
  gather_words<V>(src, p.dstride, g, x0, y, z, nullptr, h);
  collide_store_half<MODEL, V>(p, omega, cell0, h);
}

// Single-block FP16S chunk (19 * dstride < 2^32): linear row `row`, first cell
// `cell` = row * pitch + x0; sources and stores through the direction bases.
template <int MODEL, int V>
__device__ __forceinline__ void pull_chunk_half32(const StepParams& p, const Geom& g, float omega,
                                                  int x0, unsigned row, unsigned cell) {
  typename HWord<V>::type h[Q];
  if (int(row) >= g.ny + 2 && int(row) <= g.ny * g.nz - g.ny - 3) {  // interior_row
    gather_words_dir<V>(p, g, x0, cell, h);
  } else {
    const unsigned z = row / unsigned(g.ny);
    gather_words_wrap<V>(static_cast<const __half*>(p.src), p.dstride, g, x0,
                         int(row - z * unsigned(g.ny)), int(z), h);
  }
  uint8_t fl[V];
  load_flags<V>(p.flags + cell, fl);
  collide_half<MODEL, V>(p, omega, (long long)cell, fl, h);
#pragma unroll
  for (int i = 0; i < Q; ++i) hstore<V>(static_cast<__half*>(p.dst_dir[i]) + cell, h[i]);
}

// One chunk: the thread owns cells x0 .. x0+V-1 of row (y, z), x0 < nx.
// Multi-block FP16S chunk with 32-bit element offsets (19 x dstride < 2^32).
// Blocks differ in pitch and plane, so the direction bases carry no row
// offset here: p.src_dir[i] = src + i * dstride, p.dst_dir[i] = dst + i *
// dstride, and the source of direction i is its base plus the chunk's cell
// index moved by -c_y pitch - c_z plane.  On interior rows every such index
// lies inside the block, so the unsigned offsets never wrap.  The loads, the
// splices and the collision are those of gather_words / collide_store_half,
// so the result is the same bit for bit; only the addressing differs (no
// 64-bit row pointers live across the gather).
template <int V>
__device__ __forceinline__ void gather_words_blk(const StepParams& p, const Geom& g, int x0,
                                                 unsigned cell,
                                                 typename HWord<V>::type (&h)[Q]) {
  using W = typename HWord<V>::type;
  const unsigned pitch = unsigned(g.pitch), plane = unsigned(g.plane);
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const unsigned sc = cell - unsigned(cy(i)) * pitch - unsigned(cz(i)) * plane;
    const __half* own = static_cast<const __half*>(p.src_dir[i]) + sc;
    const W v = hload<V>(own);
    if (cx(i) == 0) {
      h[i] = v;
    } else if (cx(i) > 0) {
      h[i] = hsplice_prev(hload<V>(x0 >= V ? own - V : own), v);
    } else {
      h[i] = hsplice_next(v, hload<V>(x0 + V < g.nx ? own + V : own));
    }
  }
  if (x0 == 0) {  // x = nx-1 of the row before the source row
#pragma unroll
    for (int i = 1; i < Q; ++i)
      if (cx(i) > 0) {
        const unsigned e = cell - unsigned(cy(i)) * pitch - unsigned(cz(i)) * plane - pitch +
                           unsigned(g.nx - 1);
        hset(h[i], 0, hscalar(static_cast<const __half*>(p.src_dir[i]) + e));
      }
  }
  const int klast = g.nx - 1 - x0;
  if (klast >= 0 && klast < V) {  // x = 0 of the row after the source row
#pragma unroll
    for (int i = 1; i < Q; ++i)
      if (cx(i) < 0) {
        const unsigned e = cell - unsigned(cy(i)) * pitch - unsigned(cz(i)) * plane + pitch -
                           unsigned(x0);
        const unsigned w = hscalar(static_cast<const __half*>(p.src_dir[i]) + e);
#pragma unroll
        for (int k = 0; k < V; ++k)
          if (k == klast) hset(h[i], k, w);
      }
  }
}

template <int MODEL, int V>
__device__ __forceinline__ void pull_chunk_half_blk32(const StepParams& p, const Geom& g,
                                                      float omega, int x0, int y, int z) {
  typename HWord<V>::type h[Q];
  const unsigned cell = unsigned(g.base) + unsigned(y) * unsigned(g.pitch) +
                        unsigned(z) * unsigned(g.plane) + unsigned(x0);
  if (interior_row(g, y, z))
    gather_words_blk<V>(p, g, x0, cell, h);
  else
    gather_words_wrap<V>(static_cast<const __half*>(p.src), p.dstride, g, x0, y, z, h);
  uint8_t fl[V];
  load_flags<V>(p.flags + cell, fl);
  collide_half<MODEL, V>(p, omega, (long long)cell, fl, h);
#pragma unroll
  for (int i = 0; i < Q; ++i) hstore<V>(static_cast<__half*>(p.dst_dir[i]) + cell, h[i]);
}

template <typename S, typename R, int MODEL, int V>
__device__ __forceinline__ void pull_chunk(const StepParams& p, const Geom& g, R omega, int lane,
                                           int x0, int y, int z) {
  if constexpr (std::is_same<S, __half>::value && V >= 2) {
    pull_chunk_half<MODEL, V>(p, g, omega, x0, y, z);
    return;
  }
  const S* __restrict__ src = static_cast<const S*>(p.src);
  S* __restrict__ dst = static_cast<S*>(p.dst);
  R vals[Q][V];
  gather_chunk<S, R, V, 1>(src, p.dstride, g, p.shift, p.inv_scale, x0, y, z, vals);
  const int nvalid = min(V, g.nx - x0);
  const long long cell0 = g.base + (long long)y * g.pitch + (long long)z * g.plane + x0;
  uint8_t fl[V];
  load_flags<V>(p.flags + cell0, fl);
  if constexpr (std::is_same<S, dev32>::value) {
#pragma unroll
    for (int k = 0; k < V; ++k) {
      if (k < nvalid) {
        float d[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) d[i] = vals[i][k];
        collide_dev32<MODEL>(p, select_op(p, fl[k]), d, cell0 + k, omega);
#pragma unroll
        for (int i = 0; i < Q; ++i) vals[i][k] = d[i];
      }
    }
  } else {
    collide_chunk<R, MODEL, V>(p, g, omega, vals, fl, cell0, nvalid);
  }
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
// 32-bit arithmetic: a block holds fewer than 2^32 chunks (checked at creation).
template <int V>
__device__ __forceinline__ bool chunk_coords(const Geom& g, long long q, int& x0, int& y,
                                             int& z) {
  const unsigned cpr = unsigned(g.pitch / V);
  const unsigned total = cpr * unsigned(g.ny) * unsigned(g.nz);
  if (q >= (long long)total) return false;
  const unsigned uq = unsigned(q);
  const unsigned row = uq / cpr;
  x0 = int(uq - row * cpr) * V;
  const unsigned zz = row / unsigned(g.ny);
  y = int(row - zz * unsigned(g.ny));
  z = int(zz);
  return x0 < g.nx;
}

// Single block: one thread per chunk; consecutive threads take consecutive
// chunks, so a warp may span the end of one row and the start of the next and
// only padding lanes idle.  Grid: ceil(chunks / blockDim.x) CTAs.
// Minimum resident 256-thread CTAs per SM asked of the compiler, i.e. the
// register cap: 3 (85 registers, 24 warps per SM) for the FP32 kernels at 2
// cells per thread, 2 (128 registers) for the FP16S kernels (their two-wide
// pair code spills badly at 85: LES 1.1 KB at 4 cells per thread) and FP32 at
// 4 cells per thread; FP64 is left free.  Measured at 512^3 against the other
// caps.
template <typename S, int MODEL, int V>
struct PullBounds {
  static constexpr int min_ctas =
      std::is_same<S, double>::value                          ? 1
      : std::is_same<S, __half>::value ? 2
      : (std::is_same<S, float>::value || std::is_same<S, dev32>::value) && V == 4 ? 2
                                                              : 3;
};

template <typename S, typename R, int MODEL, int V>
__global__ void __launch_bounds__(256, PullBounds<S, MODEL, V>::min_ctas) k_pull(const StepParams p) {
  const Geom g{p.nx, p.ny, p.nz, p.pitch, p.plane, 0};
  if constexpr (std::is_same<S, __half>::value && V >= 2) {
    // 32-bit chunk index (fewer than 2^31 chunks: 19 * dstride < 2^32)
    const unsigned q = blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned cpr = unsigned(p.pitch) / V;
    if (q >= cpr * unsigned(p.ny) * unsigned(p.nz)) return;
    const unsigned row = p.cpr_m ? __umulhi(q, p.cpr_m) >> (p.cpr_s - 1) : q;
    const int x0 = int(q - row * cpr) * V;
    if (x0 >= p.nx) return;
    pull_chunk_half32<MODEL, V>(p, g, float(p.omega), x0, row, q * V);
    return;
  }
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int x0, y, z;
  if (!chunk_coords<V>(g, q, x0, y, z)) return;
  pull_chunk<S, R, MODEL, V>(p, g, R(p.omega), 0, x0, y, z);
}

// Many blocks: tiles of blockDim.x consecutive chunks, numbered block by block
// (tile_start = first tile of the block, tile_block = block of every tile);
// CTAs walk the tiles with a grid stride (persistent) or take one tile each.
template <typename S, typename R, int MODEL, int V>
__global__ void __launch_bounds__(256, PullBounds<S, MODEL, V>::min_ctas)
    k_pull_blocks(const StepParams p, const BlockEntry* __restrict__ blocks,
                  const int* __restrict__ tile_block, long long ntiles) {
  for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const BlockEntry& b = blocks[__ldg(tile_block + t)];
    const long long q = (t - b.tile_start) * blockDim.x + threadIdx.x;
    int x0, y, z;
    if (chunk_coords<V>(b.g, q, x0, y, z))
      pull_chunk<S, R, MODEL, V>(p, b.g, R(b.omega), 0, x0, y, z);
  }
}

// k_pull_blocks for FP16S storage with 32-bit offsets (pull_chunk_half_blk32).
template <int MODEL, int V>
__global__ void __launch_bounds__(256, PullBounds<__half, MODEL, V>::min_ctas)
    k_pull_blocks_half32(const StepParams p, const BlockEntry* __restrict__ blocks,
                         const int* __restrict__ tile_block, long long ntiles) {
  for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const BlockEntry& b = blocks[__ldg(tile_block + t)];
    const long long q = (t - b.tile_start) * blockDim.x + threadIdx.x;
    int x0, y, z;
    if (chunk_coords<V>(b.g, q, x0, y, z))
      pull_chunk_half_blk32<MODEL, V>(p, b.g, float(b.omega), x0, y, z);
  }
}

// ---------------------------------------------------------------------------
// Transfers and helpers in R = stream(P) space.

// population array i: R (staging, host dtype, host order) -> P slots
template <typename S, typename R, typename H>
__global__ void k_unstream_in(LayoutParams L, Geom g, const H* stage, S* pops_i, int i,
                              float shift, float scale) {
  const long long total = L.plane * L.nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total;
       c += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    if (!decode_cell(L, c, x, y, z)) continue;
    const H v = stage[((long long)z * L.ny + y) * L.nx + x];
    if constexpr (std::is_same<S, dev32>::value)  // the deviation in the host precision
      pops_i[wrap_src(g, x, y, z, i)].v = float(v - H(shift));
    else
      Storage<S, R>::store(pops_i + wrap_src(g, x, y, z, i), R(v), shift, scale);
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
    H v;
    if constexpr (std::is_same<S, dev32>::value)
      v = H(pops_i[wrap_src(g, x, y, z, i)].v) + H(shift);
    else
      v = H(Storage<S, R>::load(pops_i + wrap_src(g, x, y, z, i), shift, inv_scale));
    stage[((long long)z * L.ny + y) * L.nx + x] = v;
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

// the same as stored values (FP32S: the deviations, unconverted)
template <typename S, typename R>
__device__ __forceinline__ void gather_stored(const S* pops, long long dstride, const Geom& g,
                                              int x, int y, int z, const StepParams& sp, R* v) {
#pragma unroll
  for (int i = 0; i < Q; ++i)
    v[i] = gload<S, R>(pops + i * dstride + wrap_src(g, x, y, z, i), sp.shift[i], sp.inv_scale);
}

// rho and u of cell (x,y,z) (forced moments where a porosity field is given)
template <typename S, typename R>
__device__ __forceinline__ void cell_rho_u(const S* pops, long long dstride, const Geom& g, int x,
                                           int y, int z, const StepParams& sp, R alpha, R& r,
                                           R& ux, R& uy, R& uz) {
  R f[Q];
  if constexpr (std::is_same<S, dev32>::value) {
    gather_stored<S, R>(pops, dstride, g, x, y, z, sp, f);
    R delta, den;
    dev_moments(f, sp.rho0, alpha, delta, r, den, ux, uy, uz);
  } else {
    gather_R<S, R>(pops, dstride, g, x, y, z, sp, f);
    if (sp.alpha) {
      R den;
      forced_moments<R>(f, alpha, r, den, ux, uy, uz);
    } else {
      rho_u<R>(f, r, ux, uy, uz);
    }
  }
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
    R r, ux, uy, uz;
    cell_rho_u<S, R>(pops, L.dstride, g, x, y, z, sp,
                     sp.alpha ? static_cast<const R*>(sp.alpha)[g.base + c] : R(0), r, ux, uy,
                     uz);
    rho[g.base + c] = r;
    vel[g.base + c] = ux;
    vel[g.base + c + L.dstride] = uy;
    vel[g.base + c + 2 * L.dstride] = uz;
  }
}

// Mass and momentum sums of one block: CTA b writes partials[4b .. 4b+3]
// (k_sum_partials adds them in a fixed order).
template <typename S, typename R>
__global__ void __launch_bounds__(256) k_conservation_pull(LayoutParams L, Geom g, const S* pops,
                                                           const uint8_t* flags, uint8_t key,
                                                           double* partials, StepParams sp) {
  double s[4] = {0, 0, 0, 0};
  const long long total = L.plane * L.nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total;
       c += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    if (!decode_cell(L, c, x, y, z)) continue;
    if (!(flags[g.base + c] & key)) continue;
    R f[Q];
    gather_stored<S, R>(pops, L.dstride, g, x, y, z, sp, f);
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      // FP16S values come converted; FP32S deviations get their shift in FP64
      const double v = std::is_same<S, dev32>::value ? double(f[i]) + double(sp.shift[i])
                                                     : double(f[i]);
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
    partials[blockIdx.x * 4 + threadIdx.x] = v;
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
    R r, ux, uy, uz;
    if constexpr (std::is_same<S, dev32>::value) {
      cell_rho_u<S, R>(pops, L.dstride, g, x, y, z, sp, R(0), r, ux, uy, uz);
    } else {
      R f[Q];
      gather_R<S, R>(pops, L.dstride, g, x, y, z, sp, f);
      rho_u<R>(f, r, ux, uy, uz);
    }
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

// The same copies as (source, destination) element indices into the whole
// population buffer, 8 bytes per record instead of 24, when 19 x dstride <
// 2^32; records sorted by destination.  A thread takes HALO_BATCH records a
// grid stride apart and issues all their record loads, then all their
// gathers, then all their stores: the x-face gathers each miss to DRAM, and
// one outstanding gather per thread leaves the memory system idle.  Sources
// are interior cells and destinations overlap cells, so no record reads what
// another writes and the order inside a thread does not matter.
constexpr int HALO_BATCH = 4;

template <typename S>
__global__ void k_halo_pull32(const uint2* __restrict__ recs, long long n, S* pops) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long r0 = blockIdx.x * (long long)blockDim.x + threadIdx.x; r0 < n;
       r0 += stride * HALO_BATCH) {
    uint2 h[HALO_BATCH];
    S v[HALO_BATCH];
#pragma unroll
    for (int k = 0; k < HALO_BATCH; ++k) {
      const long long r = r0 + k * stride;
      h[k] = r < n ? __ldg(recs + r) : make_uint2(0u, 0u);
    }
#pragma unroll
    for (int k = 0; k < HALO_BATCH; ++k)
      if (r0 + k * stride < n) v[k] = pops[h[k].x];
#pragma unroll
    for (int k = 0; k < HALO_BATCH; ++k)
      if (r0 + k * stride < n) pops[h[k].y] = v[k];
  }
}

}  // namespace flb
