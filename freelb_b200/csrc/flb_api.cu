// flb_api.cu -- the extern "C" boundary (include/flb.h) over the sm_100a kernels.
//
// A handle owns the device state of one block lattice: two population buffers
// (ping-pong), the flag field, the RHO and VELOCITY fields, a 64-byte result
// word area for reductions and, on first use, a staging buffer for host
// transfers.  The C++17 classes in freelb_b200/cpp/freelb.h and the Python
// module call only these functions.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>

#include "../../include/flb.h"
#include "flb_kernels.cuh"

using namespace flb;

namespace {

thread_local std::string g_err = "no error";

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define FLB_CUDA(call)                                                                   \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return fail(e_ == cudaErrorMemoryAllocation ? FLB_ERR_OOM : FLB_ERR_CUDA,          \
                  "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__,      \
                  __LINE__);                                                             \
  } while (0)

inline cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

}  // namespace

struct flb_lattice {
  flb_lattice_desc desc;
  int device = 0;
  LayoutParams L{};
  int elem_bytes = 4;   // population element
  int real_bytes = 4;   // field / arithmetic element
  void* pops[2] = {nullptr, nullptr};
  int cur = 0;
  uint8_t* flags = nullptr;
  void* rho = nullptr;
  void* vel = nullptr;
  double* acc = nullptr;   // 64 bytes of reduction results
  void* stage = nullptr;   // host-transfer staging, lazily allocated
  size_t stage_bytes = 0;
  double* uprev = nullptr; // tolerance history (3 planes), lazily allocated
  StepParams sp{};
  int block_y = 8;
};

namespace {

int ensure_stage(flb_lattice* h, size_t bytes) {
  if (h->stage_bytes >= bytes) return FLB_OK;
  if (h->stage) cudaFree(h->stage);
  h->stage = nullptr;
  h->stage_bytes = 0;
  FLB_CUDA(cudaMalloc(&h->stage, bytes));
  h->stage_bytes = bytes;
  return FLB_OK;
}

int grid_1d(long long n) {
  long long b = (n + 255) / 256;
  if (b > 148 * 32) b = 148 * 32;
  return int(b < 1 ? 1 : b);
}

int validate_desc(const flb_lattice_desc* d) {
  if (!d) return fail(FLB_ERR_INVALID, "null descriptor");
  if (d->nx < 3 || d->ny < 3 || d->nz < 3)
    return fail(FLB_ERR_INVALID, "mesh %dx%dx%d: each axis needs >= 3 stored cells", d->nx,
                d->ny, d->nz);
  if (d->nz > 65535) return fail(FLB_ERR_INVALID, "nz %d exceeds 65535", d->nz);
  if ((long long)d->nx * d->ny > (1LL << 30))
    return fail(FLB_ERR_INVALID, "nx*ny too large");
  if (d->storage < 0 || d->storage > 2) return fail(FLB_ERR_INVALID, "bad storage %d", d->storage);
  if (d->model < 0 || d->model > 2) return fail(FLB_ERR_INVALID, "bad model %d", d->model);
  if (!(d->omega > 0.0 && d->omega < 2.0))
    return fail(FLB_ERR_INVALID, "omega %g outside (0, 2)", d->omega);
  if (d->ntasks < 0 || d->ntasks > FLB_MAX_TASKS)
    return fail(FLB_ERR_INVALID, "ntasks %d outside [0, %d]", d->ntasks, FLB_MAX_TASKS);
  for (int t = 0; t < d->ntasks; ++t)
    if (d->task_ops[t] > FLB_OP_FIELD_BGK)
      return fail(FLB_ERR_INVALID, "task %d has unknown op %d", t, d->task_ops[t]);
  if (d->storage == FLB_STORAGE_FP16S && d->model != FLB_MODEL_BGK && d->model != FLB_MODEL_MRT &&
      d->model != FLB_MODEL_LES)
    return fail(FLB_ERR_UNSUPPORTED, "model not built for FP16S");
  return FLB_OK;
}

// Parameters shared by every kernel of the handle.
void build_params(flb_lattice* h) {
  const flb_lattice_desc& d = h->desc;
  StepParams& p = h->sp;
  std::memset(&p, 0, sizeof p);
  p.flags = h->flags;
  p.rho = h->rho;
  p.vel = h->vel;
  p.nx = d.nx;
  p.ny = d.ny;
  p.nz = d.nz;
  p.pitch = h->L.pitch;
  p.plane = h->L.plane;
  p.dstride = h->L.dstride;
  p.ncells = (long long)d.nx * d.ny * d.nz;
  for (int i = 0; i < Q; ++i) {
    p.delta[i] = cx(i) + (long long)cy(i) * d.nx + (long long)cz(i) * d.nx * d.ny;
    p.off[i] = cx(i) + (long long)cy(i) * p.pitch + (long long)cz(i) * p.plane;
  }
  p.ntasks = d.ntasks;
  for (int t = 0; t < d.ntasks; ++t) {
    p.keys[t] = d.task_keys[t];
    p.ops[t] = d.task_ops[t];
  }
  const bool dbl = d.storage == FLB_STORAGE_FP64;
  // omega in the arithmetic type, as BlockLattice stores T(Conv.getOMEGA())
  p.omega = dbl ? d.omega : double(float(d.omega));
  const double cs = dbl ? d.smagorinsky : double(float(d.smagorinsky));
  // collisionLES.h:45: Cs*Cs*InvCs2*InvCs2*2 in T, times std::sqrt(2) in double
  const double prod = dbl ? cs * cs * 3.0 * 3.0 * 2.0
                          : double(float(float(float(float(cs) * float(cs)) * 3.0f) * 3.0f) * 2.0f);
  p.cs_coeff = prod * std::sqrt(2.0);
  for (int k = 0; k < Q; ++k) {
    double s = d.mrt_rates[k];
    if (mrt_shear(k)) s = p.omega;
    if (mrt_conserved(k)) s = 0.0;
    p.s_over_norm[k] = s / double(mrt_norm(k));
  }
  for (int i = 0; i < Q; ++i) {
    const double w = i == 0 ? 1.0 / 3.0 : (i < 7 ? 1.0 / 18.0 : 1.0 / 36.0);
    p.shift[i] = float(d.rho0 * w);
  }
  // 2^10: keeps deviations down to ~6e-8 out of the binary16 subnormal range
  // while leaving headroom to |f - w| = 64.
  p.scale = 1024.0f;
  p.inv_scale = 1.0f / 1024.0f;
}

template <typename S, typename R>
int launch_step_t(flb_lattice* h, int nsteps, cudaStream_t st) {
  const dim3 block(32, h->block_y);
  const dim3 grid(h->L.pitch / 32, (h->desc.ny + h->block_y - 1) / h->block_y, h->desc.nz);
  for (int s = 0; s < nsteps; ++s) {
    h->sp.src = h->pops[h->cur];
    h->sp.dst = h->pops[h->cur ^ 1];
    switch (h->desc.model) {
      case FLB_MODEL_BGK: k_stream_collide<S, R, MODEL_BGK><<<grid, block, 0, st>>>(h->sp); break;
      case FLB_MODEL_MRT: k_stream_collide<S, R, MODEL_MRT><<<grid, block, 0, st>>>(h->sp); break;
      default: k_stream_collide<S, R, MODEL_LES><<<grid, block, 0, st>>>(h->sp); break;
    }
    h->cur ^= 1;
  }
  FLB_CUDA(cudaGetLastError());
  return FLB_OK;
}

template <typename S, typename R, typename H>
int pops_transfer(flb_lattice* h, void* host, bool upload, cudaStream_t st) {
  const LayoutParams& L = h->L;
  const size_t hb = sizeof(H);
  const size_t N = size_t(L.nx) * L.ny * L.nz;
  const bool direct = sizeof(S) == sizeof(H) && std::is_same<S, H>::value;
  if (!direct) {
    int rc = ensure_stage(h, size_t(L.dstride) * sizeof(H));
    if (rc) return rc;
  }
  S* pops = static_cast<S*>(h->pops[h->cur]);
  for (int i = 0; i < Q; ++i) {
    char* hp = static_cast<char*>(host) + i * N * hb;
    void* dev = direct ? static_cast<void*>(pops + i * L.dstride) : h->stage;
    if (upload) {
      FLB_CUDA(cudaMemcpy2DAsync(dev, L.pitch * hb, hp, L.nx * hb, L.nx * hb,
                                 size_t(L.ny) * L.nz, cudaMemcpyHostToDevice, st));
      if (!direct)
        k_pops_in<S, R, H><<<grid_1d(L.plane * L.nz), 256, 0, st>>>(
            L, static_cast<const H*>(h->stage), pops + i * L.dstride, h->sp.shift[i], h->sp.scale);
    } else {
      if (!direct)
        k_pops_out<S, R, H><<<grid_1d(L.plane * L.nz), 256, 0, st>>>(
            L, static_cast<H*>(h->stage), pops + i * L.dstride, h->sp.shift[i],
            h->sp.inv_scale);
      FLB_CUDA(cudaMemcpy2DAsync(hp, L.nx * hb, dev, L.pitch * hb, L.nx * hb,
                                 size_t(L.ny) * L.nz, cudaMemcpyDeviceToHost, st));
    }
    FLB_CUDA(cudaGetLastError());
  }
  FLB_CUDA(cudaStreamSynchronize(st));
  return FLB_OK;
}

template <typename S, typename R>
int pops_transfer_any(flb_lattice* h, void* host, int host_dtype, bool upload, cudaStream_t st) {
  if (host_dtype == FLB_DTYPE_F32) return pops_transfer<S, R, float>(h, host, upload, st);
  if (host_dtype == FLB_DTYPE_F64) return pops_transfer<S, R, double>(h, host, upload, st);
  return fail(FLB_ERR_INVALID, "bad host dtype %d", host_dtype);
}

template <typename R, typename H>
int field_transfer(flb_lattice* h, int field, void* host, bool upload, cudaStream_t st) {
  const LayoutParams& L = h->L;
  const size_t hb = sizeof(H);
  if (field == FLB_FIELD_RHO) {
    const bool direct = std::is_same<R, H>::value;
    if (!direct) {
      int rc = ensure_stage(h, size_t(L.dstride) * sizeof(H));
      if (rc) return rc;
    }
    void* dev = direct ? h->rho : h->stage;
    if (upload) {
      FLB_CUDA(cudaMemcpy2DAsync(dev, L.pitch * hb, host, L.nx * hb, L.nx * hb,
                                 size_t(L.ny) * L.nz, cudaMemcpyHostToDevice, st));
      if (!direct)
        k_convert<H, R><<<grid_1d(L.plane * L.nz), 256, 0, st>>>(
            L.plane * L.nz, static_cast<const H*>(h->stage), static_cast<R*>(h->rho));
    } else {
      if (!direct)
        k_convert<R, H><<<grid_1d(L.plane * L.nz), 256, 0, st>>>(
            L.plane * L.nz, static_cast<const R*>(h->rho), static_cast<H*>(h->stage));
      FLB_CUDA(cudaMemcpy2DAsync(host, L.nx * hb, dev, L.pitch * hb, L.nx * hb,
                                 size_t(L.ny) * L.nz, cudaMemcpyDeviceToHost, st));
    }
  } else if (field == FLB_FIELD_VELOCITY) {
    int rc = ensure_stage(h, 3 * size_t(L.dstride) * sizeof(H));
    if (rc) return rc;
    if (upload) {
      FLB_CUDA(cudaMemcpy2DAsync(h->stage, 3 * L.pitch * hb, host, 3 * L.nx * hb, 3 * L.nx * hb,
                                 size_t(L.ny) * L.nz, cudaMemcpyHostToDevice, st));
      k_vel_in<R, H><<<grid_1d(L.plane * L.nz), 256, 0, st>>>(
          L, static_cast<const H*>(h->stage), static_cast<R*>(h->vel));
    } else {
      k_vel_out<R, H><<<grid_1d(L.plane * L.nz), 256, 0, st>>>(
          L, static_cast<H*>(h->stage), static_cast<const R*>(h->vel));
      FLB_CUDA(cudaMemcpy2DAsync(host, 3 * L.nx * hb, h->stage, 3 * L.pitch * hb, 3 * L.nx * hb,
                                 size_t(L.ny) * L.nz, cudaMemcpyDeviceToHost, st));
    }
  } else {
    return fail(FLB_ERR_INVALID, "unknown field %d", field);
  }
  FLB_CUDA(cudaGetLastError());
  FLB_CUDA(cudaStreamSynchronize(st));
  return FLB_OK;
}

// Dispatch a functor on the handle's (storage, arithmetic) types.
template <typename F>
int with_types(flb_lattice* h, F&& f) {
  switch (h->desc.storage) {
    case FLB_STORAGE_FP32: return f((float*)nullptr, (float*)nullptr);
    case FLB_STORAGE_FP16S: return f((__half*)nullptr, (float*)nullptr);
    default: return f((double*)nullptr, (double*)nullptr);
  }
}

}  // namespace

// ===========================================================================
extern "C" {

int flb_version(int* abi_version, int* sm_arch) {
  if (abi_version) *abi_version = FLB_ABI_VERSION;
  if (sm_arch) *sm_arch = 100;
  return FLB_OK;
}

const char* flb_last_error(void) { return g_err.c_str(); }

int flb_desc_default(flb_lattice_desc* d, int nx, int ny, int nz, double tau) {
  if (!d) return fail(FLB_ERR_INVALID, "null descriptor");
  std::memset(d, 0, sizeof *d);
  d->nx = nx;
  d->ny = ny;
  d->nz = nz;
  d->storage = FLB_STORAGE_FP32;
  d->model = FLB_MODEL_BGK;
  d->omega = 1.0 / tau;
  d->smagorinsky = 0.1;
  for (int k = 0; k < 19; ++k) d->mrt_rates[k] = 1.2;
  d->rho0 = 1.0;
  d->ntasks = 3;
  d->task_keys[0] = 2;
  d->task_ops[0] = FLB_OP_BULK;
  d->task_keys[1] = 4;
  d->task_ops[1] = FLB_OP_BOUNCEBACK;
  d->task_keys[2] = 8;
  d->task_ops[2] = FLB_OP_MOVINGWALL;
  return FLB_OK;
}

int flb_create(const flb_lattice_desc* desc, flb_lattice** out) {
  if (!out) return fail(FLB_ERR_INVALID, "null output handle");
  *out = nullptr;
  int rc = validate_desc(desc);
  if (rc) return rc;
  flb_lattice* h = new (std::nothrow) flb_lattice();
  if (!h) return fail(FLB_ERR_OOM, "host allocation failed");
  h->desc = *desc;
  cudaGetDevice(&h->device);
  const int elem =
      desc->storage == FLB_STORAGE_FP16S ? 2 : (desc->storage == FLB_STORAGE_FP64 ? 8 : 4);
  const int real = desc->storage == FLB_STORAGE_FP64 ? 8 : 4;
  h->elem_bytes = elem;
  h->real_bytes = real;
  LayoutParams& L = h->L;
  L.nx = desc->nx;
  L.ny = desc->ny;
  L.nz = desc->nz;
  L.pitch = (desc->nx + 31) / 32 * 32;
  L.plane = (long long)L.pitch * L.ny;
  L.dstride = (L.plane * L.nz + 63) / 64 * 64;
  const size_t popb = size_t(Q) * L.dstride * elem;
  auto cleanup = [&](int code) {
    flb_destroy(h);
    return code;
  };
  cudaError_t e;
  for (int b = 0; b < 2; ++b) {
    e = cudaMalloc(&h->pops[b], popb);
    if (e != cudaSuccess)
      return cleanup(fail(FLB_ERR_OOM, "cudaMalloc populations (%zu bytes): %s", popb,
                          cudaGetErrorString(e)));
  }
  if ((e = cudaMalloc((void**)&h->flags, size_t(L.dstride))) != cudaSuccess ||
      (e = cudaMalloc(&h->rho, size_t(L.dstride) * real)) != cudaSuccess ||
      (e = cudaMalloc(&h->vel, 3 * size_t(L.dstride) * real)) != cudaSuccess ||
      (e = cudaMalloc((void**)&h->acc, 64)) != cudaSuccess)
    return cleanup(fail(FLB_ERR_OOM, "cudaMalloc fields: %s", cudaGetErrorString(e)));
  build_params(h);
  // defaults: void flags, RHO = rho0, VELOCITY = 0, f = rho0 * w_i
  cudaStream_t st = 0;
  if ((e = cudaMemsetAsync(h->flags, 1, size_t(L.dstride), st)) != cudaSuccess ||
      (e = cudaMemsetAsync(h->vel, 0, 3 * size_t(L.dstride) * real, st)) != cudaSuccess)
    return cleanup(fail(FLB_ERR_CUDA, "init memset: %s", cudaGetErrorString(e)));
  if (real == 8)
    k_fill<double><<<grid_1d(L.dstride), 256, 0, st>>>(L.dstride, static_cast<double*>(h->rho),
                                                        desc->rho0);
  else
    k_fill<float><<<grid_1d(L.dstride), 256, 0, st>>>(L.dstride, static_cast<float*>(h->rho),
                                                       float(desc->rho0));
  rc = flb_init_equilibrium(h, desc->rho0, nullptr);
  if (rc) return cleanup(rc);
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess)
    return cleanup(fail(FLB_ERR_CUDA, "create: %s", cudaGetErrorString(e)));
  *out = h;
  return FLB_OK;
}

int flb_destroy(flb_lattice* h) {
  if (!h) return FLB_OK;
  for (void* p : {h->pops[0], h->pops[1], (void*)h->flags, h->rho, h->vel, (void*)h->acc,
                  h->stage, (void*)h->uprev})
    if (p) cudaFree(p);
  delete h;
  return FLB_OK;
}

int flb_memory_bytes(const flb_lattice* h, size_t* bytes) {
  if (!h || !bytes) return fail(FLB_ERR_INVALID, "null argument");
  const size_t ds = size_t(h->L.dstride);
  *bytes = 2 * size_t(Q) * ds * h->elem_bytes + ds + 4 * ds * h->real_bytes + 64 +
           h->stage_bytes + (h->uprev ? 3 * ds * sizeof(double) : 0);
  return FLB_OK;
}

int flb_upload_flags(flb_lattice* h, const uint8_t* host, void* stream) {
  if (!h || !host) return fail(FLB_ERR_INVALID, "null argument");
  const LayoutParams& L = h->L;
  cudaStream_t st = as_stream(stream);
  FLB_CUDA(cudaMemcpy2DAsync(h->flags, L.pitch, host, L.nx, L.nx, size_t(L.ny) * L.nz,
                             cudaMemcpyHostToDevice, st));
  FLB_CUDA(cudaStreamSynchronize(st));
  return FLB_OK;
}

int flb_download_flags(flb_lattice* h, uint8_t* host, void* stream) {
  if (!h || !host) return fail(FLB_ERR_INVALID, "null argument");
  const LayoutParams& L = h->L;
  cudaStream_t st = as_stream(stream);
  FLB_CUDA(cudaMemcpy2DAsync(host, L.nx, h->flags, L.pitch, L.nx, size_t(L.ny) * L.nz,
                             cudaMemcpyDeviceToHost, st));
  FLB_CUDA(cudaStreamSynchronize(st));
  return FLB_OK;
}

int flb_upload_pops(flb_lattice* h, const void* host, int host_dtype, void* stream) {
  if (!h || !host) return fail(FLB_ERR_INVALID, "null argument");
  return with_types(h, [&](auto* sp, auto* rp) {
    using S = std::remove_pointer_t<decltype(sp)>;
    using R = std::remove_pointer_t<decltype(rp)>;
    return pops_transfer_any<S, R>(h, const_cast<void*>(host), host_dtype, true,
                                   as_stream(stream));
  });
}

int flb_download_pops(flb_lattice* h, void* host, int host_dtype, void* stream) {
  if (!h || !host) return fail(FLB_ERR_INVALID, "null argument");
  return with_types(h, [&](auto* sp, auto* rp) {
    using S = std::remove_pointer_t<decltype(sp)>;
    using R = std::remove_pointer_t<decltype(rp)>;
    return pops_transfer_any<S, R>(h, host, host_dtype, false, as_stream(stream));
  });
}

static int field_any(flb_lattice* h, int field, void* host, int host_dtype, bool upload,
                     void* stream) {
  if (!h || !host) return fail(FLB_ERR_INVALID, "null argument");
  cudaStream_t st = as_stream(stream);
  if (h->real_bytes == 8) {
    if (host_dtype == FLB_DTYPE_F64) return field_transfer<double, double>(h, field, host, upload, st);
    if (host_dtype == FLB_DTYPE_F32) return field_transfer<double, float>(h, field, host, upload, st);
  } else {
    if (host_dtype == FLB_DTYPE_F64) return field_transfer<float, double>(h, field, host, upload, st);
    if (host_dtype == FLB_DTYPE_F32) return field_transfer<float, float>(h, field, host, upload, st);
  }
  return fail(FLB_ERR_INVALID, "bad host dtype %d", host_dtype);
}

int flb_upload_field(flb_lattice* h, int field, const void* host, int host_dtype, void* stream) {
  return field_any(h, field, const_cast<void*>(host), host_dtype, true, stream);
}

int flb_download_field(flb_lattice* h, int field, void* host, int host_dtype, void* stream) {
  return field_any(h, field, host, host_dtype, false, stream);
}

int flb_init_equilibrium(flb_lattice* h, double rho0, void* stream) {
  if (!h) return fail(FLB_ERR_INVALID, "null handle");
  cudaStream_t st = as_stream(stream);
  const LayoutParams& L = h->L;
  int rc = with_types(h, [&](auto* sp, auto* rp) {
    using S = std::remove_pointer_t<decltype(sp)>;
    using R = std::remove_pointer_t<decltype(rp)>;
    k_init_equilibrium<S, R><<<grid_1d(L.plane * L.nz), 256, 0, st>>>(
        L, static_cast<S*>(h->pops[h->cur]), rho0, h->sp);
    return FLB_OK;
  });
  if (rc) return rc;
  FLB_CUDA(cudaGetLastError());
  return FLB_OK;
}

int flb_step(flb_lattice* h, int nsteps, void* stream) {
  if (!h) return fail(FLB_ERR_INVALID, "null handle");
  if (nsteps < 0) return fail(FLB_ERR_INVALID, "nsteps %d < 0", nsteps);
  if (nsteps == 0) return FLB_OK;
  cudaStream_t st = as_stream(stream);
  return with_types(h, [&](auto* sp, auto* rp) {
    using S = std::remove_pointer_t<decltype(sp)>;
    using R = std::remove_pointer_t<decltype(rp)>;
    return launch_step_t<S, R>(h, nsteps, st);
  });
}

int flb_compute_rhou(flb_lattice* h, uint8_t key, void* stream) {
  if (!h) return fail(FLB_ERR_INVALID, "null handle");
  cudaStream_t st = as_stream(stream);
  const LayoutParams& L = h->L;
  int rc = with_types(h, [&](auto* sp, auto* rp) {
    using S = std::remove_pointer_t<decltype(sp)>;
    using R = std::remove_pointer_t<decltype(rp)>;
    k_rhou<S, R><<<grid_1d(L.plane * L.nz), 256, 0, st>>>(
        L, static_cast<const S*>(h->pops[h->cur]), h->flags, key, static_cast<R*>(h->rho),
        static_cast<R*>(h->vel), h->sp);
    return FLB_OK;
  });
  if (rc) return rc;
  FLB_CUDA(cudaGetLastError());
  return FLB_OK;
}

int flb_reduce_conservation(flb_lattice* h, uint8_t key, double out[4], void* stream) {
  if (!h || !out) return fail(FLB_ERR_INVALID, "null argument");
  cudaStream_t st = as_stream(stream);
  const LayoutParams& L = h->L;
  FLB_CUDA(cudaMemsetAsync(h->acc, 0, 4 * sizeof(double), st));
  int rc = with_types(h, [&](auto* sp, auto* rp) {
    using S = std::remove_pointer_t<decltype(sp)>;
    using R = std::remove_pointer_t<decltype(rp)>;
    k_conservation<S, R><<<grid_1d(L.plane * L.nz), 256, 0, st>>>(
        L, static_cast<const S*>(h->pops[h->cur]), h->flags, key, h->acc, h->sp);
    return FLB_OK;
  });
  if (rc) return rc;
  FLB_CUDA(cudaGetLastError());
  FLB_CUDA(cudaMemcpyAsync(out, h->acc, 4 * sizeof(double), cudaMemcpyDeviceToHost, st));
  FLB_CUDA(cudaStreamSynchronize(st));
  return FLB_OK;
}

int flb_tolerance_u(flb_lattice* h, uint8_t key, double* max_du, void* stream) {
  if (!h || !max_du) return fail(FLB_ERR_INVALID, "null argument");
  cudaStream_t st = as_stream(stream);
  const LayoutParams& L = h->L;
  if (!h->uprev) {
    FLB_CUDA(cudaMalloc((void**)&h->uprev, 3 * size_t(L.dstride) * sizeof(double)));
    FLB_CUDA(cudaMemsetAsync(h->uprev, 0, 3 * size_t(L.dstride) * sizeof(double), st));
  }
  unsigned long long* acc = reinterpret_cast<unsigned long long*>(h->acc);
  FLB_CUDA(cudaMemsetAsync(acc, 0, sizeof(unsigned long long), st));
  int rc = with_types(h, [&](auto* sp, auto* rp) {
    using S = std::remove_pointer_t<decltype(sp)>;
    using R = std::remove_pointer_t<decltype(rp)>;
    k_tolerance<S, R><<<grid_1d(L.plane * L.nz), 256, 0, st>>>(
        L, static_cast<const S*>(h->pops[h->cur]), h->flags, key, h->uprev, acc, h->sp);
    return FLB_OK;
  });
  if (rc) return rc;
  FLB_CUDA(cudaGetLastError());
  unsigned long long bits = 0;
  FLB_CUDA(cudaMemcpyAsync(&bits, acc, sizeof bits, cudaMemcpyDeviceToHost, st));
  FLB_CUDA(cudaStreamSynchronize(st));
  std::memcpy(max_du, &bits, sizeof(double));
  return FLB_OK;
}

int flb_check_finite(flb_lattice* h, uint64_t* bad, void* stream) {
  if (!h || !bad) return fail(FLB_ERR_INVALID, "null argument");
  cudaStream_t st = as_stream(stream);
  const LayoutParams& L = h->L;
  unsigned long long* acc = reinterpret_cast<unsigned long long*>(h->acc);
  FLB_CUDA(cudaMemsetAsync(acc, 0, sizeof(unsigned long long), st));
  int rc = with_types(h, [&](auto* sp, auto* rp) {
    using S = std::remove_pointer_t<decltype(sp)>;
    using R = std::remove_pointer_t<decltype(rp)>;
    k_finite<S, R><<<grid_1d(L.plane * L.nz), 256, 0, st>>>(
        L, static_cast<const S*>(h->pops[h->cur]), acc, h->sp);
    return FLB_OK;
  });
  if (rc) return rc;
  FLB_CUDA(cudaGetLastError());
  unsigned long long v = 0;
  FLB_CUDA(cudaMemcpyAsync(&v, acc, sizeof v, cudaMemcpyDeviceToHost, st));
  FLB_CUDA(cudaStreamSynchronize(st));
  *bad = v;
  return FLB_OK;
}

int flb_get_layout(const flb_lattice* h, flb_layout* layout) {
  if (!h || !layout) return fail(FLB_ERR_INVALID, "null argument");
  layout->nx = h->L.nx;
  layout->ny = h->L.ny;
  layout->nz = h->L.nz;
  layout->pitch_x = h->L.pitch;
  layout->plane = size_t(h->L.plane);
  layout->dir_stride = size_t(h->L.dstride);
  layout->elem_bytes = h->elem_bytes;
  return FLB_OK;
}

int flb_device_pointers(flb_lattice* h, void** pops, void** flags, void** rho, void** vel) {
  if (!h) return fail(FLB_ERR_INVALID, "null handle");
  if (pops) *pops = h->pops[h->cur];
  if (flags) *flags = h->flags;
  if (rho) *rho = h->rho;
  if (vel) *vel = h->vel;
  return FLB_OK;
}

}  // extern "C"
