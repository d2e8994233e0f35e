// flb_vtk.cuh -- base64 payloads of VTK ImageData arrays from device fields.
//
// The reference's vtmo writers (src/io/vtm_writer.h:288-663 over
// src/io/vti_writer.h:424-986) write each field of a block as one
// <DataArray format="binary" encoding="base64"> whose body is two base64
// streams back to back (src/io/base64.h, Base64Encoder): the data size in
// bytes as a 4-byte unsigned int on its own, then the data -- the cells of
// the block without `overlap` layers on each side, x fastest, components
// interleaved for vectors (util::CopyFromFieldArray, src/utils/util.h:439-540),
// optionally mapped by the Phys writers' unit conversion.  Here one kernel
// gathers, converts and encodes on the device, so only the text crosses to
// the host.
#pragma once

#include <cstdint>

#include "flb_kernels.cuh"

namespace flb {

struct VtkArgs {
  const void* src;       // component 0 of the field at the block's cell (0,0,0)
  long long comp_stride; // elements between component planes
  int pitch;
  long long plane;
  int sx, sy, sz;        // cells written per axis
  int ox, oy, oz;        // first cell written (the overlap)
  int ncomp;
  int map;               // apply v * scale (+ offset) in the field's type
  double scale, offset;
  long long nbytes;      // data bytes after conversion
};

__device__ __forceinline__ char b64_char(unsigned v) {
  // RFC 4648 alphabet: A-Z a-z 0-9 + /
  return v < 26 ? char('A' + v)
                : v < 52 ? char('a' + (v - 26)) : v < 62 ? char('0' + (v - 52)) : (v == 62 ? '+' : '/');
}

// 3 bytes (n valid, 1..3) -> 4 characters with '=' padding
__device__ __forceinline__ unsigned b64_group(unsigned b0, unsigned b1, unsigned b2, int n) {
  const unsigned c0 = b0 >> 2;
  const unsigned c1 = ((b0 & 3u) << 4) | (b1 >> 4);
  const unsigned c2 = ((b1 & 15u) << 2) | (b2 >> 6);
  const unsigned c3 = b2 & 63u;
  const unsigned ch0 = (unsigned char)b64_char(c0), ch1 = (unsigned char)b64_char(c1);
  const unsigned ch2 = n >= 2 ? (unsigned char)b64_char(c2) : (unsigned char)'=';
  const unsigned ch3 = n >= 3 ? (unsigned char)b64_char(c3) : (unsigned char)'=';
  return ch0 | (ch1 << 8) | (ch2 << 16) | (ch3 << 24);
}

template <typename O>
__device__ __forceinline__ unsigned long long bits_of(O v) {
  if constexpr (sizeof(O) == 8) return (unsigned long long)__double_as_longlong(double(v));
  else if constexpr (sizeof(O) == 4) return (unsigned long long)__float_as_uint(float(v));
  else return (unsigned long long)(unsigned char)v;
}

// element e of the written array, converted to O
template <typename R, typename O>
__device__ __forceinline__ O vtk_elem(const VtkArgs& a, long long e) {
  const long long c = e / a.ncomp;
  const int comp = int(e - c * a.ncomp);
  const long long row = c / a.sx;
  const int x = int(c - row * a.sx);
  const long long z = row / a.sy;
  const int y = int(row - z * a.sy);
  const long long off = (long long)(x + a.ox) + (long long)(y + a.oy) * a.pitch +
                        (z + a.oz) * a.plane + comp * a.comp_stride;
  R v = static_cast<const R*>(a.src)[off];
  if constexpr (sizeof(R) >= 4) {
    if (a.map) {
      v = v * R(a.scale);  // the unit conversion in the field's type, unfused
      if (a.offset != 0.0) v = v + R(a.offset);
    }
  }
  return O(v);
}

// out[0, 8): the 4-byte size block; out[8 + 4 g, 12 + 4 g): data group g.
template <typename R, typename O>
__global__ void __launch_bounds__(256) k_vtk_base64(VtkArgs a, unsigned* out) {
  const long long ngroups = (a.nbytes + 2) / 3;
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < ngroups;
       g += (long long)gridDim.x * blockDim.x) {
    const long long b0 = 3 * g;
    long long e = b0 / (long long)sizeof(O);
    int o = int(b0 - e * (long long)sizeof(O));
    unsigned long long v = bits_of<O>(vtk_elem<R, O>(a, e));
    unsigned b[3] = {0u, 0u, 0u};
    int n = 0;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      if (b0 + j >= a.nbytes) break;
      if (o == int(sizeof(O))) {
        ++e;
        o = 0;
        v = bits_of<O>(vtk_elem<R, O>(a, e));
      }
      b[j] = unsigned((v >> (8 * o)) & 0xffu);
      ++o;
      ++n;
    }
    out[2 + g] = b64_group(b[0], b[1], b[2], n);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    // (unsigned int)(bytes): the reference narrows the size_t the same way
    const unsigned len = unsigned((unsigned long long)a.nbytes);
    out[0] = b64_group(len & 0xffu, (len >> 8) & 0xffu, (len >> 16) & 0xffu, 3);
    out[1] = b64_group((len >> 24) & 0xffu, 0u, 0u, 1);
  }
}

}  // namespace flb
