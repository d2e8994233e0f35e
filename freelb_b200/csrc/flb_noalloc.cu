// flb_noalloc.cu -- mass/momentum reduction that allocates no memory.
//
// flb_reduce_conservation (flb_api.cu) accumulates into a result area the
// lattice handle allocated with cudaMalloc.  Some callers cannot let a library
// allocate device memory: runtimes that hand GPU memory out only through their
// own caching pool (so that their accounting stays exact and no component
// triggers the implicit synchronisation a cudaMalloc / cudaFree can cause),
// and plugin hosts that call into this library from threads where a
// driver-level allocation could block on another context's work.  This
// variant takes the populations and flags as plain device pointers and keeps
// its scratch -- one partial sum per thread block and the final four sums --
// in the file-scope device array below, which every GPU that loads the library
// holds until the process exits.  It copies the sums to the caller's host
// array and synchronises the caller's stream before returning, so it is not a
// call to make inside a stream capture.
//
// Two passes, both deterministic: pass 1 has thread block b reduce the padded
// cells [b*kCellsPerBlock, (b+1)*kCellsPerBlock) into partial slot b; pass 2
// sums the slots in order into the result slot, which is copied to the
// caller's host array.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/flb.h"
#include "flb_pull.cuh"

using namespace flb;

namespace flb {
int report_error(int code, const char* msg);  // flb_api.cu: sets flb_last_error()
}

namespace {

constexpr int kMaxPartials = 4096;          // thread blocks of pass 1
constexpr long long kCellsPerBlock = 65536;  // padded cells reduced by one thread block
constexpr long long kMaxCells = kMaxPartials * kCellsPerBlock;  // 268,435,456
constexpr int kThreads = 256;

// 4 sums per partial slot plus the final 4 sums: (4096 + 1) * 4 doubles = 128 KiB.
__device__ __align__(256) double g_noalloc_scratch[(kMaxPartials + 1) * 4];

// Device address of g_noalloc_scratch, looked up on the first call on each
// device (with that device current) and kept for the process.  A
// cudaDeviceReset on that device unloads the library's device code with this
// array, after which the kept address is stale: the entry point is not to be
// called on a device after resetting it.
std::mutex g_mu;
void* g_scratch_ptr[64] = {};

int scratch_for_current_device(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 64) {
    char m[160];
    std::snprintf(m, sizeof m, "flb_reduce_conservation_noalloc: cudaGetDevice: %s",
                  cudaGetErrorString(e));
    return report_error(FLB_ERR_CUDA, m);
  }
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      char m[160];
      std::snprintf(m, sizeof m, "flb_reduce_conservation_noalloc: cudaGetSymbolAddress: %s",
                    cudaGetErrorString(e));
      return report_error(FLB_ERR_CUDA, m);
    }
    g_scratch_ptr[dev] = p;
  }
  *out = static_cast<double*>(g_scratch_ptr[dev]);
  return FLB_OK;
}

// Pass 1: thread block b writes partial slot b (always, also when its cells
// sum to zero), so no slot needs clearing beforehand.
template <typename S, typename R>
__global__ void __launch_bounds__(kThreads)
    k_cons_partials(LayoutParams L, Geom g, const S* pops, const uint8_t* flags, uint8_t key,
                    StepParams sp, double* partials) {
  double s[4] = {0, 0, 0, 0};
  const long long total = L.plane * L.nz;
  const long long begin = (long long)blockIdx.x * kCellsPerBlock;
  const long long end = begin + kCellsPerBlock < total ? begin + kCellsPerBlock : total;
  for (long long c = begin + threadIdx.x; c < end; c += kThreads) {
    int x, y, z;
    if (!decode_cell(L, c, x, y, z)) continue;
    if (!(flags[c] & key)) continue;
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
  __shared__ double red[kThreads / 32][4];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const double v = warp_sum(s[k]);
    if (lane == 0) red[wid][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double v = 0;
    for (int w = 0; w < kThreads / 32; ++w) v += red[w][threadIdx.x];
    partials[blockIdx.x * 4 + threadIdx.x] = v;
  }
}

// Pass 2: one thread block sums slots 0..n-1 in a fixed order into result.
__global__ void __launch_bounds__(kThreads) k_cons_final(const double* partials, int n,
                                                         double* result) {
  __shared__ double red[kThreads][4];
  double s[4] = {0, 0, 0, 0};
  for (int b = threadIdx.x; b < n; b += kThreads)
#pragma unroll
    for (int k = 0; k < 4; ++k) s[k] += partials[b * 4 + k];
#pragma unroll
  for (int k = 0; k < 4; ++k) red[threadIdx.x][k] = s[k];
  __syncthreads();
  if (threadIdx.x < 4) {
    double v = 0;
    for (int t = 0; t < kThreads; ++t) v += red[t][threadIdx.x];
    result[threadIdx.x] = v;
  }
}

template <typename S, typename R>
int run(const void* pops, const uint8_t* flags, const flb_layout* lay, double rho0, uint8_t key,
        double out[4], cudaStream_t st) {
  double* scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc) return rc;
  LayoutParams L{};
  L.nx = lay->nx;
  L.ny = lay->ny;
  L.nz = lay->nz;
  L.pitch = lay->pitch_x;
  L.plane = (long long)lay->plane;
  L.dstride = (long long)lay->dir_stride;
  const Geom g{L.nx, L.ny, L.nz, L.pitch, L.plane, 0};
  StepParams sp{};
  for (int i = 0; i < Q; ++i) {
    const double w = i == 0 ? 1.0 / 3.0 : (i < 7 ? 1.0 / 18.0 : 1.0 / 36.0);
    sp.shift[i] = float(rho0 * w);
  }
  // FP16S storage scale of the library (FP32S deviations are unscaled)
  sp.scale = std::is_same<S, __half>::value ? 1024.0f : 1.0f;
  sp.inv_scale = 1.0f / sp.scale;
  const long long total = L.plane * L.nz;
  const int nblocks = int((total + kCellsPerBlock - 1) / kCellsPerBlock);
  k_cons_partials<S, R><<<nblocks, kThreads, 0, st>>>(L, g, static_cast<const S*>(pops), flags,
                                                      key, sp, scratch);
  double* result = scratch + kMaxPartials * 4;
  k_cons_final<<<1, kThreads, 0, st>>>(scratch, nblocks, result);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, result, 4 * sizeof(double),
                                            cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    char m[160];
    std::snprintf(m, sizeof m, "flb_reduce_conservation_noalloc: %s", cudaGetErrorString(e));
    return report_error(FLB_ERR_CUDA, m);
  }
  return FLB_OK;
}

}  // namespace

extern "C" {

int flb_reduce_conservation_noalloc(const void* pops, const uint8_t* flags,
                                    const flb_layout* layout, int storage, double rho0,
                                    uint8_t key, double out[4], void* stream) {
  if (!pops || !flags || !layout || !out)
    return report_error(FLB_ERR_INVALID, "flb_reduce_conservation_noalloc: null argument");
  const flb_layout& L = *layout;
  const int elem = storage == FLB_STORAGE_FP16S ? 2 : (storage == FLB_STORAGE_FP64 ? 8 : 4);
  if (storage < 0 || storage > 3 || L.elem_bytes != elem) {
    char m[160];
    std::snprintf(m, sizeof m,
                  "flb_reduce_conservation_noalloc: storage %d does not match %d-byte elements",
                  storage, L.elem_bytes);
    return report_error(FLB_ERR_INVALID, m);
  }
  if (L.nx < 3 || L.ny < 3 || L.nz < 3 || L.pitch_x < L.nx ||
      L.plane != size_t(L.pitch_x) * size_t(L.ny) || L.dir_stride < L.plane * size_t(L.nz))
    return report_error(FLB_ERR_INVALID, "flb_reduce_conservation_noalloc: inconsistent layout");
  const long long cells = (long long)L.plane * L.nz;
  if (cells > kMaxCells) {
    char m[200];
    std::snprintf(m, sizeof m,
                  "flb_reduce_conservation_noalloc: %lld padded cells exceed the static scratch "
                  "limit of %lld (%d thread blocks x %lld cells)",
                  cells, kMaxCells, kMaxPartials, kCellsPerBlock);
    return report_error(FLB_ERR_INVALID, m);
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // the scratch is the current device's: the stream and the arrays must be on it
  int dev = 0, sdev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess && st) e = cudaStreamGetDevice(st, &sdev);
  else sdev = dev;  // the legacy default stream belongs to the current device
  if (e != cudaSuccess) {
    char m[160];
    std::snprintf(m, sizeof m, "flb_reduce_conservation_noalloc: stream device: %s",
                  cudaGetErrorString(e));
    return report_error(FLB_ERR_CUDA, m);
  }
  for (const void* ptr : {pops, static_cast<const void*>(flags)}) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess ||
        !(a.type == cudaMemoryTypeManaged || (a.type == cudaMemoryTypeDevice && a.device == dev))) {
      cudaGetLastError();  // clear a failed query
      return report_error(FLB_ERR_INVALID,
                          "flb_reduce_conservation_noalloc: pops and flags must be device memory "
                          "of the current device");
    }
  }
  if (sdev != dev)
    return report_error(FLB_ERR_INVALID,
                        "flb_reduce_conservation_noalloc: stream belongs to another device than "
                        "the current one");
  if (storage == FLB_STORAGE_FP32) return run<float, float>(pops, flags, layout, rho0, key, out, st);
  if (storage == FLB_STORAGE_FP32S) return run<dev32, float>(pops, flags, layout, rho0, key, out, st);
  if (storage == FLB_STORAGE_FP64)
    return run<double, double>(pops, flags, layout, rho0, key, out, st);
  return run<__half, float>(pops, flags, layout, rho0, key, out, st);
}

}  // extern "C"
