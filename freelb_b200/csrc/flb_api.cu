// flb_api.cu -- the extern "C" boundary (include/flb.h) over the sm_100a kernels.
//
// A handle owns the device state of one lattice made of one or more blocks:
// two population buffers (ping-pong), the flag field, the RHO and VELOCITY
// fields, a 64-byte result area for reductions, the block table and halo
// records, and, on first use, a staging buffer for host transfers and the
// captured CUDA graphs.  Blocks are packed one after another inside every
// direction array (each block padded to a row pitch, see row_pitch, and to a
// multiple of 64 elements).  The C++17 classes in freelb_b200/cpp/freelb.h and
// the Python module call only these functions.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/flb.h"
#include "../../include/flb_vtk.h"
#include "flb_adjoint.cuh"
#include "flb_pipe.cuh"
#include "flb_tma.cuh"
#include "flb_vtk.cuh"

using namespace flb;
static_assert(TMA_TIMEOUT == FLB_ERR_TIMEOUT, "device status code");

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

#define FLB_TRY(expr)      \
  do {                     \
    int rc_ = (expr);      \
    if (rc_) return rc_;   \
  } while (0)

inline cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

}  // namespace

// Error reporting shared with the library's other translation units.
namespace flb {
int report_error(int code, const char* msg) { return fail(code, "%s", msg); }
}  // namespace flb

namespace {

struct HostBlock {
  LayoutParams L;   // this block's layout; L.dstride is the handle's direction stride
  long long base;   // element offset of the block inside every direction array
  int ox, oy, oz;   // global stored index of local (0,0,0)
  double omega;     // 1/tau in the arithmetic type
  long long padded() const { return L.plane * L.nz; }
};

}  // namespace

struct flb_lattice {
  flb_lattice_desc desc;
  int device = 0;
  int sm_count = 148;
  int mode = -1;  // -1: single block (flb_create)
  std::vector<HostBlock> blocks;
  long long dstride = 0;
  int elem_bytes = 4;
  int real_bytes = 4;
  void* pops[2] = {nullptr, nullptr};
  int cur = 0;
  uint8_t* flags = nullptr;
  void* rho = nullptr;
  void* vel = nullptr;
  double* acc = nullptr;
  double* red = nullptr;  // per-CTA partial sums of the FP64 reductions (RED_SLOTS x 4)
  void* stage = nullptr;
  size_t stage_bytes = 0;
  double* uprev = nullptr;
  uint8_t* d_lut = nullptr;  // op of every flag value
  StepParams sp{};
  // multi-block launch data
  BlockEntry* d_blocks = nullptr;
  int* d_tile_block = nullptr;  // block of every tile (tile kernel)
  long long tile_block_cap = 0;
  long long ntiles = 0;
  int table_tile_y = 0;
  int table_vec = 0;
  HaloCopy* d_halo = nullptr;   // records, or uint2 (src, dst) pairs when halo32
  long long nhalo = 0;
  bool halo32 = false;
  int halo_mode = FLB_HALO_NORMAL;
  int tile_y = 4;
  int ctas_per_sm = 0;  // -1: the FP16S async-copy pipeline (k_pull_pipe);
                        // -2 / -3: the FP16S bulk-copy kernel, 2-cell chunks in 5
                        // stages / 4-cell chunks in 3 stages (k_pull_tma)
  int pipe_ctas = 0;    // resident k_pull_pipe CTAs per SM (0 = not yet queried)
  bool tma_ready = false;  // k_pull_tma shared-memory attributes set
  double wait_s = 2.0;     // bound of one device-side wait (k_pull_tma)
  long long withhold = -1; // failure-detection test hook (flb_test_withhold_tile)
  int vec = 0;  // cells per thread of the step kernel; 0 = storage default
  int rounding = FLB_ROUND_DEFAULT;  // FP16S stores (flb_set_rounding)
  alignas(8) char snap_hdr[64] = {};  // source of the snapshot header copies
  // CUDA graphs of the two-step cycle, one per starting buffer parity
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  // Brinkman porosity (FLB_FIELD_ALPHA), arithmetic type
  void* alpha = nullptr;
  // adjoint workspace
  int adj_T = 0, adj_k = 0;
  std::vector<void*> adj_ckpt;  // Q_0, Q_k, Q_2k, ...
  std::vector<void*> adj_seg;   // recomputed Q_{t0+1} .. Q_{t0+k-1}
  void* adj_lam[2] = {nullptr, nullptr};
  double* adj_galpha = nullptr;
  double* adj_gpart = nullptr;  // per-thread-block dJ/dtau, dJ/du_lid sums
  size_t adj_gpart_n = 0;
};

// Storage kind of a handle, for the library's other translation units.
namespace flb {
int lattice_storage(const flb_lattice* h) { return h->desc.storage; }
}  // namespace flb

// Device status word of a handle: the last slot of its 64-byte result area
// (zeroed at creation; the reductions use the first five slots).
inline int* status_word(flb_lattice* h) { return reinterpret_cast<int*>(h->acc + 7); }

namespace {

void drop_graphs(flb_lattice* h) {
  for (auto& g : h->graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
}

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

// k_halo_pull32: enough 256-thread CTAs for one batch of HALO_BATCH records
// per thread, so that no thread starts a second, mostly idle, round.
int halo32_grid(long long n) {
  const long long per_cta = 256LL * HALO_BATCH;
  const long long b = (n + per_cta - 1) / per_cta;
  return int(std::min(std::max(b, 1LL), 1LL << 20));
}

int validate_common(const flb_lattice_desc* d) {
  if (!d) return fail(FLB_ERR_INVALID, "null descriptor");
  if (d->storage < 0 || d->storage > 3) return fail(FLB_ERR_INVALID, "bad storage %d", d->storage);
  if (d->model < 0 || d->model > 3) return fail(FLB_ERR_INVALID, "bad model %d", d->model);
  if (d->model == FLB_MODEL_BRINKMAN && d->storage == FLB_STORAGE_FP16S)
    return fail(FLB_ERR_UNSUPPORTED, "BRINKMAN model is built for FP32 and FP64 storage");
  if (!(d->omega > 0.0 && d->omega < 2.0))
    return fail(FLB_ERR_INVALID, "omega %g outside (0, 2)", d->omega);
  if (d->ntasks < 0 || d->ntasks > FLB_MAX_TASKS)
    return fail(FLB_ERR_INVALID, "ntasks %d outside [0, %d]", d->ntasks, FLB_MAX_TASKS);
  for (int t = 0; t < d->ntasks; ++t)
    if (d->task_ops[t] > FLB_OP_FIELD_BGK)
      return fail(FLB_ERR_INVALID, "task %d has unknown op %d", t, d->task_ops[t]);
  return FLB_OK;
}

int validate_block(int nx, int ny, int nz) {
  if (nx < 3 || ny < 3 || nz < 3)
    return fail(FLB_ERR_INVALID, "mesh %dx%dx%d: each axis needs >= 3 stored cells", nx, ny, nz);
  if (nz > 65535) return fail(FLB_ERR_INVALID, "nz %d exceeds 65535", nz);
  if ((long long)nx * ny > (1LL << 30)) return fail(FLB_ERR_INVALID, "nx*ny too large");
  return FLB_OK;
}

double arith_omega(const flb_lattice_desc& d, double omega) {
  // BlockLattice stores Omega as T (block_lattice.hh:27-35)
  return d.storage == FLB_STORAGE_FP64 ? omega : double(float(omega));
}

// Parameters shared by every kernel of the handle.
void build_params(flb_lattice* h) {
  const flb_lattice_desc& d = h->desc;
  StepParams& p = h->sp;
  std::memset(&p, 0, sizeof p);
  const HostBlock& b0 = h->blocks[0];
  p.flags = h->flags;
  p.rho = h->rho;
  p.vel = h->vel;
  p.alpha = h->alpha;
  p.nx = b0.L.nx;
  p.ny = b0.L.ny;
  p.nz = b0.L.nz;
  p.pitch = b0.L.pitch;
  p.plane = b0.L.plane;
  p.dstride = h->dstride;
  for (int i = 0; i < Q; ++i)
    p.row_off[i] = i * h->dstride - ((long long)cy(i) + (long long)cz(i) * p.ny) * p.pitch;
  p.idx32 = h->blocks.size() == 1 && (long long)Q * h->dstride < (1LL << 32) ? 1 : 0;
  for (int i = 0; i < Q; ++i) {
    p.row_off32[i] = p.idx32 ? unsigned(p.row_off[i]) : 0u;
    p.dir_off32[i] = p.idx32 ? unsigned(i * h->dstride) : 0u;
  }
  // chunks per row of the single-block FP16S step (4 cells per chunk, or 2:
  // the division constants depend on the chunk width, set at launch)
  p.cpr_m = 0;
  p.cpr_s = 0;
  p.ntasks = d.ntasks;
  for (int t = 0; t < d.ntasks; ++t) {
    p.keys[t] = d.task_keys[t];
    p.ops[t] = d.task_ops[t];
  }
  p.op_lut = h->d_lut;
  const bool dbl = d.storage == FLB_STORAGE_FP64;
  p.omega = arith_omega(d, d.omega);
  const double cs = dbl ? d.smagorinsky : double(float(d.smagorinsky));
  // collisionLES.h:45: Cs*Cs*InvCs2*InvCs2*2 in T, times std::sqrt(2) in double
  const double prod = dbl ? cs * cs * 3.0 * 3.0 * 2.0
                          : double(float(float(float(float(cs) * float(cs)) * 3.0f) * 3.0f) * 2.0f);
  p.cs_coeff = prod * std::sqrt(2.0);
  for (int k = 0; k < Q; ++k) {
    double s = d.mrt_rates[k];
    if (mrt_conserved(k)) s = 0.0;
    p.s_over_norm[k] = s / double(mrt_norm(k));
  }
  // one rate for all moments outside the conserved and shear sets: the
  // two-rate form of the FP16S MRT collision
  p.mrt_sg = float(d.mrt_rates[1]);
  for (int k = 0; k < Q; ++k)
    if (!mrt_conserved(k) && !mrt_shear(k) && d.mrt_rates[k] != d.mrt_rates[1]) p.mrt_sg = 0.0f;
  if (!(p.mrt_sg > 0.0f)) p.mrt_sg = 0.0f;
  for (int i = 0; i < Q; ++i) {
    const double w = i == 0 ? 1.0 / 3.0 : (i < 7 ? 1.0 / 18.0 : 1.0 / 36.0);
    p.shift[i] = float(d.rho0 * w);
  }
  // FP16S: 2^10 keeps deviations down to ~6e-8 out of the binary16 subnormal
  // range while leaving headroom to |f - w| = 64.  FP32S stores the deviations
  // unscaled.
  const bool fp32s = d.storage == FLB_STORAGE_FP32S;
  p.scale = fp32s ? 1.0f : 1024.0f;
  p.inv_scale = fp32s ? 1.0f : 1.0f / 1024.0f;
  p.rho0 = float(d.rho0);
  // FP16S rounding: stochastic for MRT unless the caller chose (its round to
  // nearest drifts, see the cvt.rs helpers of the step kernels)
  const int r = h->rounding == FLB_ROUND_DEFAULT
                    ? (d.model == FLB_MODEL_MRT ? FLB_ROUND_STOCHASTIC : FLB_ROUND_NEAREST)
                    : h->rounding;
  p.fp16_round = d.storage == FLB_STORAGE_FP16S && r == FLB_ROUND_STOCHASTIC ? 1 : 0;
}

// Cells per thread of the pull kernel (launch parameter; defaults are the
// measured best per storage).
int default_vec(int storage) { return storage == FLB_STORAGE_FP16S ? 4 : 2; }
int vec_width(const flb_lattice* h) { return h->vec ? h->vec : default_vec(h->desc.storage); }
bool vec_allowed(int storage, int v) {
  return storage == FLB_STORAGE_FP64 ? (v == 1 || v == 2) : (v == 2 || v == 4);
}

Geom geom_of(const HostBlock& b) {
  return Geom{b.L.nx, b.L.ny, b.L.nz, b.L.pitch, b.L.plane, b.base};
}

// Op lookup table: for every flag value, the op of the first task whose key
// shares a bit with it (src/utils/tmp.h:283-309).
int upload_op_lut(flb_lattice* h) {
  uint8_t lut[256];
  for (int v = 0; v < 256; ++v) {
    lut[v] = FLB_OP_NONE;
    for (int t = 0; t < h->desc.ntasks; ++t)
      if (v & h->desc.task_keys[t]) {
        lut[v] = h->desc.task_ops[t];
        break;
      }
  }
  FLB_CUDA(cudaMemcpy(h->d_lut, lut, sizeof lut, cudaMemcpyHostToDevice));
  return FLB_OK;
}

// Elements per stored row: rows of wide blocks start on 64-byte (FP32)
// boundaries (nx rounded up to 16); narrow blocks, where that padding would
// idle a large share of the lanes, round up to 4 only (the vector loads need
// 16-byte alignment at most).
int row_pitch(int nx) { return nx >= 240 ? (nx + 15) / 16 * 16 : (nx + 3) / 4 * 4; }

// Block table for the tile kernel (rebuilt when tile_y changes).
int upload_block_table(flb_lattice* h) {
  if (h->d_blocks && h->table_tile_y == h->tile_y && h->table_vec == vec_width(h)) return FLB_OK;
  std::vector<BlockEntry> t(h->blocks.size());
  long long start = 0;
  for (size_t b = 0; b < h->blocks.size(); ++b) {
    const HostBlock& hb = h->blocks[b];
    BlockEntry& e = t[b];
    e.g = Geom{hb.L.nx, hb.L.ny, hb.L.nz, hb.L.pitch, hb.L.plane, hb.base};
    e.omega = hb.omega;
    const long long chunks = (long long)(hb.L.pitch / vec_width(h)) * hb.L.ny * hb.L.nz;
    const long long per_tile = 32LL * h->tile_y;
    e.tile_start = start;
    start += (chunks + per_tile - 1) / per_tile;
  }
  if (!h->d_blocks) FLB_CUDA(cudaMalloc((void**)&h->d_blocks, t.size() * sizeof(BlockEntry)));
  FLB_CUDA(cudaMemcpy(h->d_blocks, t.data(), t.size() * sizeof(BlockEntry),
                      cudaMemcpyHostToDevice));
  // tile -> block, so that a CTA finds its block with one load
  std::vector<int> tb(static_cast<size_t>(start));
  for (size_t b = 0; b < t.size(); ++b) {
    const long long end = b + 1 < t.size() ? t[b + 1].tile_start : start;
    for (long long k = t[b].tile_start; k < end; ++k) tb[size_t(k)] = int(b);
  }
  if (start > h->tile_block_cap) {
    if (h->d_tile_block) cudaFree(h->d_tile_block);
    h->d_tile_block = nullptr;
    h->tile_block_cap = 0;
    FLB_CUDA(cudaMalloc((void**)&h->d_tile_block, size_t(start) * sizeof(int)));
    h->tile_block_cap = start;
  }
  FLB_CUDA(cudaMemcpy(h->d_tile_block, tb.data(), tb.size() * sizeof(int), cudaMemcpyHostToDevice));
  h->ntiles = start;
  h->table_tile_y = h->tile_y;
  h->table_vec = vec_width(h);
  return FLB_OK;
}

// Host twin of wrap_src (flb_pull.cuh): P slot feeding R_i at (x,y,z).
long long host_wrap_src(const Geom& g, int x, int y, int z, int i) {
  int sx = x - cx(i), sy = y - cy(i), sz = z - cz(i);
  if (sx < 0) { sx += g.nx; --sy; } else if (sx >= g.nx) { sx -= g.nx; ++sy; }
  if (sy < 0) { sy += g.ny; --sz; } else if (sy >= g.ny) { sy -= g.ny; ++sz; }
  if (sz < 0) sz += g.nz; else if (sz >= g.nz) sz -= g.nz;
  return g.base + sx + (long long)sy * g.pitch + (long long)sz * g.plane;
}

// Halo records: every overlap cell of block b owned by a neighbour's interior
// receives, from that neighbour cell, the populations pointing into b across
// each face it lies beyond (union over axes: getCommPopDir, communicator.h:76).
int build_halo(flb_lattice* h) {
  const int nb = int(h->blocks.size());
  int gx = 0, gy = 0, gz = 0;
  for (const HostBlock& b : h->blocks) {
    if (b.ox < 0 || b.oy < 0 || b.oz < 0)
      return fail(FLB_ERR_INVALID, "block origin must be non-negative");
    gx = std::max(gx, b.ox + b.L.nx);
    gy = std::max(gy, b.oy + b.L.ny);
    gz = std::max(gz, b.oz + b.L.nz);
  }
  const long long gn = (long long)gx * gy * gz;
  if (gn > (1LL << 33)) return fail(FLB_ERR_INVALID, "global block extent too large");
  std::vector<int> owner(size_t(gn), -1);
  for (int k = 0; k < nb; ++k) {
    const HostBlock& b = h->blocks[k];
    for (int z = b.oz + 1; z < b.oz + b.L.nz - 1; ++z)
      for (int y = b.oy + 1; y < b.oy + b.L.ny - 1; ++y)
        for (int x = b.ox + 1; x < b.ox + b.L.nx - 1; ++x) {
          int& o = owner[size_t((long long)(z * (long long)gy + y) * gx + x)];
          if (o >= 0) return fail(FLB_ERR_INVALID, "blocks %d and %d overlap in their interiors", o, k);
          o = k;
        }
  }
  std::vector<HaloCopy> recs;
  for (int k = 0; k < nb; ++k) {
    const HostBlock& b = h->blocks[k];
    const Geom gb = geom_of(b);
    for (int lz = 0; lz < b.L.nz; ++lz)
      for (int ly = 0; ly < b.L.ny; ++ly)
        for (int lx = 0; lx < b.L.nx; ++lx) {
          const bool inner = lx > 0 && ly > 0 && lz > 0 && lx < b.L.nx - 1 && ly < b.L.ny - 1 &&
                             lz < b.L.nz - 1;
          if (inner) continue;
          const int x = b.ox + lx, y = b.oy + ly, z = b.oz + lz;
          const int o = owner[size_t((long long)(z * (long long)gy + y) * gx + x)];
          if (o < 0) continue;
          const HostBlock& n = h->blocks[o];
          const Geom gn = geom_of(n);
          const int l[3] = {lx, ly, lz};
          const int m[3] = {b.L.nx, b.L.ny, b.L.nz};
          const bool full = h->halo_mode == FLB_HALO_FULL;
          for (int i = full ? 0 : 1; i < Q; ++i) {
            const int c[3] = {cx(i), cy(i), cz(i)};
            bool cross = false;
            for (int a = 0; a < 3; ++a)
              if ((l[a] == 0 && c[a] > 0) || (l[a] == m[a] - 1 && c[a] < 0)) cross = true;
            if (!cross && !full) continue;
            HaloCopy r;
            r.dir = i;
            r.dst = host_wrap_src(gb, lx, ly, lz, i);
            r.src = host_wrap_src(gn, x - n.ox, y - n.oy, z - n.oz, i);
            recs.push_back(r);
          }
        }
  }
  if (h->d_halo) cudaFree(h->d_halo);
  h->d_halo = nullptr;
  h->nhalo = (long long)recs.size();
  h->halo32 = (long long)Q * h->dstride < (1LL << 32);
  if (recs.empty()) return FLB_OK;
  if (h->halo32) {
    std::vector<uint2> pairs(recs.size());
    for (size_t k = 0; k < recs.size(); ++k)
      pairs[k] = make_uint2(unsigned(recs[k].dir * h->dstride + recs[k].src),
                            unsigned(recs[k].dir * h->dstride + recs[k].dst));
    std::sort(pairs.begin(), pairs.end(),
              [](const uint2& a, const uint2& b) { return a.y < b.y; });
    FLB_CUDA(cudaMalloc((void**)&h->d_halo, pairs.size() * sizeof(uint2)));
    FLB_CUDA(cudaMemcpy(h->d_halo, pairs.data(), pairs.size() * sizeof(uint2),
                        cudaMemcpyHostToDevice));
  } else {
    FLB_CUDA(cudaMalloc((void**)&h->d_halo, recs.size() * sizeof(HaloCopy)));
    FLB_CUDA(cudaMemcpy(h->d_halo, recs.data(), recs.size() * sizeof(HaloCopy),
                        cudaMemcpyHostToDevice));
  }
  return FLB_OK;
}

// Dispatch a functor on the handle's (storage, arithmetic) types.
template <typename F>
int with_types(flb_lattice* h, F&& f) {
  switch (h->desc.storage) {
    case FLB_STORAGE_FP32: return f((float*)nullptr, (float*)nullptr);
    case FLB_STORAGE_FP16S: return f((__half*)nullptr, (float*)nullptr);
    case FLB_STORAGE_FP32S: return f((dev32*)nullptr, (float*)nullptr);
    default: return f((double*)nullptr, (double*)nullptr);
  }
}

// The async-copy pipeline covers single-block FP16S handles with 32-bit
// offsets (BGK, MRT, LES) at 4 cells per thread.
bool pipe_supported(const flb_lattice* h) {
  return h->desc.storage == FLB_STORAGE_FP16S && h->mode < 0 && h->sp.idx32 &&
         h->desc.model != FLB_MODEL_BRINKMAN;
}

// 16-byte copies need 16-byte aligned rows.
bool pipe_wide(const flb_lattice* h) { return h->blocks[0].L.pitch % 8 == 0; }

template <int MODEL, bool WIDE>
int pipe_prepare_w(flb_lattice* h) {
  const int bytes = pipe_smem_bytes();
  FLB_CUDA(cudaFuncSetAttribute(k_pull_pipe<MODEL, WIDE>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  FLB_CUDA(cudaFuncSetAttribute(k_pull_pipe<MODEL, WIDE>,
                                cudaFuncAttributePreferredSharedMemoryCarveout,
                                int(cudaSharedmemCarveoutMaxShared)));
  int n = 0;
  FLB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_pull_pipe<MODEL, WIDE>,
                                                         PIPE_WARPS * 32, size_t(bytes)));
  if (n < 1) return fail(FLB_ERR_CUDA, "k_pull_pipe does not fit on an SM");
  h->pipe_ctas = n;
  return FLB_OK;
}

template <int MODEL>
int pipe_prepare_t(flb_lattice* h) {
  return pipe_wide(h) ? pipe_prepare_w<MODEL, true>(h) : pipe_prepare_w<MODEL, false>(h);
}

// FP16S and FP32 MRT with one rate for every non-conserved, non-shear moment
// run the two-rate kernels (MODEL_MRT2); FP32S and FP64 keep the general form.
bool use_mrt2(const flb_lattice* h) {
  return (h->desc.storage == FLB_STORAGE_FP16S || h->desc.storage == FLB_STORAGE_FP32) &&
         h->desc.model == FLB_MODEL_MRT && h->sp.mrt_sg != 0.0f;
}

int pipe_prepare(flb_lattice* h) {
  if (h->pipe_ctas > 0) return FLB_OK;
  switch (h->desc.model) {
    case FLB_MODEL_MRT:
      return use_mrt2(h) ? pipe_prepare_t<MODEL_MRT2>(h) : pipe_prepare_t<MODEL_MRT>(h);
    case FLB_MODEL_LES: return pipe_prepare_t<MODEL_LES>(h);
    default: return pipe_prepare_t<MODEL_BGK>(h);
  }
}

// The bulk-copy kernel covers single-block FP16S handles with 32-bit offsets
// whose rows start on 16-byte boundaries and end at most 16 halves before the
// next row (BGK, MRT, LES) at 4 cells per thread.
bool tma_supported(const flb_lattice* h) {
  const LayoutParams& L = h->blocks[0].L;
  return h->desc.storage == FLB_STORAGE_FP16S && h->mode < 0 && h->sp.idx32 &&
         h->desc.model != FLB_MODEL_BRINKMAN && L.pitch % 8 == 0 && L.pitch - L.nx <= 16;
}

// Launch modes: ctas_per_sm -2 = 2-cell chunks, 5 stages; -3 = 4-cell chunks, 3 stages.
template <int MODEL, int NS, int CV>
int tma_attr() {
  FLB_CUDA(cudaFuncSetAttribute(k_pull_tma<MODEL, NS, CV>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                tma_smem_bytes<NS, CV>()));
  return FLB_OK;
}

int tma_prepare(flb_lattice* h) {
  if (h->tma_ready) return FLB_OK;
  FLB_TRY((tma_attr<MODEL_BGK, 5, 2>()));
  FLB_TRY((tma_attr<MODEL_BGK, 3, 4>()));
  FLB_TRY((tma_attr<MODEL_MRT, 5, 2>()));
  FLB_TRY((tma_attr<MODEL_MRT, 3, 4>()));
  FLB_TRY((tma_attr<MODEL_MRT2, 5, 2>()));
  FLB_TRY((tma_attr<MODEL_MRT2, 3, 4>()));
  FLB_TRY((tma_attr<MODEL_LES, 5, 2>()));
  FLB_TRY((tma_attr<MODEL_LES, 3, 4>()));
  h->tma_ready = true;
  return FLB_OK;
}

// Round-up division constants for q / d, q < 2^31 (Granlund & Montgomery,
// "Division by invariant integers using multiplication", PLDI 1994, Thm 4.2):
// s = ceil(log2 d), m = ceil(2^(31+s) / d) < 2^32, q / d = (q m >> 32) >> (s - 1).
// d = 1 gives m = 0 (no division).
void division_constants(unsigned d, unsigned& m, unsigned& s) {
  if (d <= 1) {
    m = 0;
    s = 0;
    return;
  }
  unsigned sh = 0;
  while ((1ull << sh) < d) ++sh;
  m = unsigned(((1ull << (31 + sh)) + d - 1) / d);
  s = sh;
}

// Direction bases of the single-block FP16S step for the launch's src / dst.
template <int V>
StepParams half_step_params(const flb_lattice* h) {
  StepParams p = h->sp;
  const __half* src = static_cast<const __half*>(p.src);
  __half* dst = static_cast<__half*>(p.dst);
  for (int i = 0; i < Q; ++i) {
    p.src_dir[i] = src + p.row_off[i];
    p.dst_dir[i] = dst + i * p.dstride;
  }
  division_constants(unsigned(p.pitch / V), p.cpr_m, p.cpr_s);
  return p;
}

// Direction bases of the multi-block FP16S tile kernel: src + i * dstride and
// dst + i * dstride (blocks differ in their row steps, which the kernel adds).
StepParams block_half_params(const flb_lattice* h) {
  StepParams p = h->sp;
  const __half* src = static_cast<const __half*>(p.src);
  __half* dst = static_cast<__half*>(p.dst);
  for (int i = 0; i < Q; ++i) {
    p.src_dir[i] = src + i * p.dstride;
    p.dst_dir[i] = dst + i * p.dstride;
  }
  return p;
}

template <typename S, typename R, int MODEL, int V>
void launch_one_step_v(flb_lattice* h, cudaStream_t st) {
  if constexpr (std::is_same<S, __half>::value && V == 4 && MODEL != MODEL_BRINKMAN) {
    if (h->ctas_per_sm <= -2) {  // flb_set_launch admits it only where tma_supported
      const HostBlock& b = h->blocks[0];
      const int cv = h->ctas_per_sm == -2 ? 2 : 4;
      const long long cells = (long long)cv * TMA_CHUNKS;
      TmaParams tp{};
      tp.ntiles = (b.padded() + cells - 1) / cells;
      tp.status = status_word(h);
      tp.wait_ns = (unsigned long long)(h->wait_s * 1e9);
      tp.drain_ns = std::max(tp.wait_ns, 1000000000ULL);
      tp.withhold = h->withhold;
      tma_staged_range(cells, b.L.pitch, b.L.ny, b.L.nz, tp.staged_lo, tp.staged_hi);
      const unsigned g = unsigned(std::max(1LL, std::min(tp.ntiles, (long long)h->sm_count)));
      if (cv == 2)
        k_pull_tma<MODEL, 5, 2><<<g, TMA_THREADS, tma_smem_bytes<5, 2>(), st>>>(
            half_step_params<2>(h), tp);
      else
        k_pull_tma<MODEL, 3, 4><<<g, TMA_THREADS, tma_smem_bytes<3, 4>(), st>>>(
            half_step_params<4>(h), tp);
      return;
    }
  }
  if constexpr (std::is_same<S, __half>::value && V == PIPE_V && MODEL != MODEL_BRINKMAN) {
    if (h->ctas_per_sm < 0) {  // flb_set_launch admits -1 only where pipe_supported
      const HostBlock& b = h->blocks[0];
      const long long chunks = (long long)(b.L.pitch / V) * b.L.ny * b.L.nz;
      const long long ctas_needed = ((chunks + 31) / 32 + PIPE_WARPS - 1) / PIPE_WARPS;
      const long long g = std::max(1LL, std::min(ctas_needed, (long long)h->pipe_ctas * h->sm_count));
      if (pipe_wide(h))
        k_pull_pipe<MODEL, true><<<unsigned(g), PIPE_WARPS * 32, pipe_smem_bytes(), st>>>(h->sp);
      else
        k_pull_pipe<MODEL, false><<<unsigned(g), PIPE_WARPS * 32, pipe_smem_bytes(), st>>>(h->sp);
      return;
    }
  }
  // the single-block kernel addresses with 32-bit offsets; larger lattices
  // take the tile-table kernel
  const bool single = h->mode < 0 && h->ctas_per_sm == 0 && h->sp.idx32;
  if (single) {
    const HostBlock& b = h->blocks[0];
    const long long chunks = (long long)(b.L.pitch / V) * b.L.ny * b.L.nz;
    const long long per_cta = 32LL * h->tile_y;
    const dim3 grid(unsigned((chunks + per_cta - 1) / per_cta));
    if constexpr (std::is_same<S, __half>::value && V >= 2)
      k_pull<S, R, MODEL, V><<<grid, dim3(32 * h->tile_y), 0, st>>>(half_step_params<V>(h));
    else
      k_pull<S, R, MODEL, V><<<grid, dim3(32 * h->tile_y), 0, st>>>(h->sp);
  } else {
    long long g = h->ctas_per_sm > 0 ? (long long)h->ctas_per_sm * h->sm_count : h->ntiles;
    g = std::max(1LL, std::min(g, h->ntiles));
    if constexpr (std::is_same<S, __half>::value && V >= 2) {
      if ((long long)Q * h->dstride < (1LL << 32)) {
        k_pull_blocks_half32<MODEL, V><<<unsigned(g), dim3(32 * h->tile_y), 0, st>>>(
            block_half_params(h), h->d_blocks, h->d_tile_block, h->ntiles);
        return;
      }
    }
    k_pull_blocks<S, R, MODEL, V><<<unsigned(g), dim3(32 * h->tile_y), 0, st>>>(
        h->sp, h->d_blocks, h->d_tile_block, h->ntiles);
  }
}

template <typename S, typename R, int MODEL>
void launch_one_step(flb_lattice* h, cudaStream_t st) {
  const int v = vec_width(h);
  if constexpr (std::is_same<S, double>::value) {
    if (v == 1) launch_one_step_v<S, R, MODEL, 1>(h, st);
    else launch_one_step_v<S, R, MODEL, 2>(h, st);
  } else {
    if (v == 2) launch_one_step_v<S, R, MODEL, 2>(h, st);
    else launch_one_step_v<S, R, MODEL, 4>(h, st);
  }
  if (h->nhalo > 0) {
    if (h->halo32)
      k_halo_pull32<S><<<halo32_grid(h->nhalo), 256, 0, st>>>(
          reinterpret_cast<const uint2*>(h->d_halo), h->nhalo, static_cast<S*>(h->sp.dst));
    else
      k_halo_pull<S><<<grid_1d(h->nhalo), 256, 0, st>>>(h->d_halo, h->nhalo,
                                                        static_cast<S*>(h->sp.dst), h->dstride);
  }
}

template <typename S, typename R>
int launch_steps(flb_lattice* h, int nsteps, cudaStream_t st) {
  if (h->mode >= 0 || h->ctas_per_sm > 0) FLB_TRY(upload_block_table(h));
  for (int s = 0; s < nsteps; ++s) {
    h->sp.src = h->pops[h->cur];
    h->sp.dst = h->pops[h->cur ^ 1];
    switch (h->desc.model) {
      case FLB_MODEL_BGK: launch_one_step<S, R, MODEL_BGK>(h, st); break;
      case FLB_MODEL_MRT:
        if constexpr (std::is_same<S, __half>::value || std::is_same<S, float>::value) {
          if (use_mrt2(h)) {
            launch_one_step<S, R, MODEL_MRT2>(h, st);
            break;
          }
        }
        launch_one_step<S, R, MODEL_MRT>(h, st);
        break;
      case FLB_MODEL_LES: launch_one_step<S, R, MODEL_LES>(h, st); break;
      default:
        if constexpr (!std::is_same<S, __half>::value)
          launch_one_step<S, R, MODEL_BRINKMAN>(h, st);
        break;
    }
    h->cur ^= 1;
  }
  FLB_CUDA(cudaGetLastError());
  return FLB_OK;
}

// One step from buffer src into buffer dst (adjoint recompute), leaving the
// handle's own ping-pong state untouched.
int step_between(flb_lattice* h, const void* src, void* dst, cudaStream_t st) {
  const void* s0 = h->sp.src;
  void* d0 = h->sp.dst;
  h->sp.src = src;
  h->sp.dst = dst;
  int rc = with_types(h, [&](auto* sp, auto* rp) {
    using S = std::remove_pointer_t<decltype(sp)>;
    using R = std::remove_pointer_t<decltype(rp)>;
    switch (h->desc.model) {
      case FLB_MODEL_BGK: launch_one_step<S, R, MODEL_BGK>(h, st); break;
      case FLB_MODEL_MRT:
        if constexpr (std::is_same<S, __half>::value || std::is_same<S, float>::value) {
          if (use_mrt2(h)) {
            launch_one_step<S, R, MODEL_MRT2>(h, st);
            break;
          }
        }
        launch_one_step<S, R, MODEL_MRT>(h, st);
        break;
      case FLB_MODEL_LES: launch_one_step<S, R, MODEL_LES>(h, st); break;
      default:
        if constexpr (!std::is_same<S, __half>::value)
          launch_one_step<S, R, MODEL_BRINKMAN>(h, st);
        break;
    }
    return FLB_OK;
  });
  h->sp.src = s0;
  h->sp.dst = d0;
  if (rc) return rc;
  FLB_CUDA(cudaGetLastError());
  return FLB_OK;
}

int step_any(flb_lattice* h, int nsteps, cudaStream_t st) {
  return with_types(h, [&](auto* sp, auto* rp) {
    using S = std::remove_pointer_t<decltype(sp)>;
    using R = std::remove_pointer_t<decltype(rp)>;
    return launch_steps<S, R>(h, nsteps, st);
  });
}

int check_block(flb_lattice* h, int b) {
  if (!h) return fail(FLB_ERR_INVALID, "null handle");
  if (b < 0 || b >= int(h->blocks.size()))
    return fail(FLB_ERR_INVALID, "block %d outside [0, %zu)", b, h->blocks.size());
  return FLB_OK;
}

template <typename S, typename R, typename H>
int pops_transfer(flb_lattice* h, const HostBlock& B, void* host, bool upload, cudaStream_t st) {
  const LayoutParams& L = B.L;
  const size_t hb = sizeof(H);
  const size_t N = size_t(L.nx) * L.ny * L.nz;
  FLB_TRY(ensure_stage(h, N * sizeof(H)));
  S* pops = static_cast<S*>(h->pops[h->cur]);
  const Geom g = geom_of(B);
  for (int i = 0; i < Q; ++i) {
    char* hp = static_cast<char*>(host) + i * N * hb;
    if (upload) {
      FLB_CUDA(cudaMemcpyAsync(h->stage, hp, N * hb, cudaMemcpyHostToDevice, st));
      k_unstream_in<S, R, H><<<grid_1d(B.padded()), 256, 0, st>>>(
          L, g, static_cast<const H*>(h->stage), pops + i * h->dstride, i, h->sp.shift[i],
          h->sp.scale);
    } else {
      k_stream_out<S, R, H><<<grid_1d(B.padded()), 256, 0, st>>>(
          L, g, static_cast<H*>(h->stage), pops + i * h->dstride, i, h->sp.shift[i],
          h->sp.inv_scale);
      FLB_CUDA(cudaMemcpyAsync(hp, h->stage, N * hb, cudaMemcpyDeviceToHost, st));
    }
    FLB_CUDA(cudaGetLastError());
  }
  FLB_CUDA(cudaStreamSynchronize(st));
  return FLB_OK;
}

int pops_any(flb_lattice* h, int b, void* host, int host_dtype, bool upload, void* stream) {
  FLB_TRY(check_block(h, b));
  if (!host) return fail(FLB_ERR_INVALID, "null host buffer");
  if (host_dtype != FLB_DTYPE_F32 && host_dtype != FLB_DTYPE_F64)
    return fail(FLB_ERR_INVALID, "bad host dtype %d", host_dtype);
  const HostBlock& B = h->blocks[b];
  cudaStream_t st = as_stream(stream);
  return with_types(h, [&](auto* sp, auto* rp) {
    using S = std::remove_pointer_t<decltype(sp)>;
    using R = std::remove_pointer_t<decltype(rp)>;
    if (host_dtype == FLB_DTYPE_F32) return pops_transfer<S, R, float>(h, B, host, upload, st);
    return pops_transfer<S, R, double>(h, B, host, upload, st);
  });
}

template <typename R, typename H>
int field_transfer(flb_lattice* h, const HostBlock& B, int field, void* host, bool upload,
                   cudaStream_t st) {
  const LayoutParams& L = B.L;
  const size_t hb = sizeof(H);
  R* rho = static_cast<R*>(field == FLB_FIELD_ALPHA ? h->alpha : h->rho) + B.base;
  R* vel = static_cast<R*>(h->vel) + B.base;
  if (field == FLB_FIELD_ALPHA && !h->alpha)
    return fail(FLB_ERR_STATE, "no ALPHA field: the lattice model is not BRINKMAN");
  // host order staged contiguously: one bus copy per transfer, padding on the device
  const size_t N = size_t(L.nx) * L.ny * L.nz;
  const int grid = grid_1d((long long)N);
  if (field == FLB_FIELD_RHO || field == FLB_FIELD_ALPHA) {
    FLB_TRY(ensure_stage(h, N * hb));
    if (upload) {
      FLB_CUDA(cudaMemcpyAsync(h->stage, host, N * hb, cudaMemcpyHostToDevice, st));
      k_pad<H, R><<<grid, 256, 0, st>>>(L, static_cast<const H*>(h->stage), rho);
    } else {
      k_unpad<R, H><<<grid, 256, 0, st>>>(L, rho, static_cast<H*>(h->stage));
      FLB_CUDA(cudaMemcpyAsync(host, h->stage, N * hb, cudaMemcpyDeviceToHost, st));
    }
  } else if (field == FLB_FIELD_VELOCITY) {
    FLB_TRY(ensure_stage(h, 3 * N * hb));
    if (upload) {
      FLB_CUDA(cudaMemcpyAsync(h->stage, host, 3 * N * hb, cudaMemcpyHostToDevice, st));
      k_vel_in<R, H><<<grid, 256, 0, st>>>(L, static_cast<const H*>(h->stage), vel);
    } else {
      k_vel_out<R, H><<<grid, 256, 0, st>>>(L, static_cast<H*>(h->stage), vel);
      FLB_CUDA(cudaMemcpyAsync(host, h->stage, 3 * N * hb, cudaMemcpyDeviceToHost, st));
    }
  } else {
    return fail(FLB_ERR_INVALID, "unknown field %d", field);
  }
  FLB_CUDA(cudaGetLastError());
  FLB_CUDA(cudaStreamSynchronize(st));
  return FLB_OK;
}

int field_any(flb_lattice* h, int b, int field, void* host, int host_dtype, bool upload,
              void* stream) {
  FLB_TRY(check_block(h, b));
  if (!host) return fail(FLB_ERR_INVALID, "null host buffer");
  const HostBlock& B = h->blocks[b];
  cudaStream_t st = as_stream(stream);
  if (h->real_bytes == 8) {
    if (host_dtype == FLB_DTYPE_F64) return field_transfer<double, double>(h, B, field, host, upload, st);
    if (host_dtype == FLB_DTYPE_F32) return field_transfer<double, float>(h, B, field, host, upload, st);
  } else {
    if (host_dtype == FLB_DTYPE_F64) return field_transfer<float, double>(h, B, field, host, upload, st);
    if (host_dtype == FLB_DTYPE_F32) return field_transfer<float, float>(h, B, field, host, upload, st);
  }
  return fail(FLB_ERR_INVALID, "bad host dtype %d", host_dtype);
}

int flags_any(flb_lattice* h, int b, uint8_t* host, bool upload, void* stream) {
  FLB_TRY(check_block(h, b));
  if (!host) return fail(FLB_ERR_INVALID, "null host buffer");
  const HostBlock& B = h->blocks[b];
  const LayoutParams& L = B.L;
  cudaStream_t st = as_stream(stream);
  const size_t N = size_t(L.nx) * L.ny * L.nz;
  FLB_TRY(ensure_stage(h, N));
  uint8_t* stage = static_cast<uint8_t*>(h->stage);
  if (upload) {
    FLB_CUDA(cudaMemcpyAsync(stage, host, N, cudaMemcpyHostToDevice, st));
    k_pad<uint8_t, uint8_t><<<grid_1d((long long)N), 256, 0, st>>>(L, stage, h->flags + B.base);
  } else {
    k_unpad<uint8_t, uint8_t><<<grid_1d((long long)N), 256, 0, st>>>(L, h->flags + B.base, stage);
    FLB_CUDA(cudaMemcpyAsync(host, stage, N, cudaMemcpyDeviceToHost, st));
  }
  FLB_CUDA(cudaGetLastError());
  FLB_CUDA(cudaStreamSynchronize(st));
  return FLB_OK;
}

// Common allocation for flb_create / flb_create_blocks.
int create_common(const flb_lattice_desc* desc, std::vector<HostBlock> blocks, int mode,
                  flb_lattice** out) {
  flb_lattice* h = new (std::nothrow) flb_lattice();
  if (!h) return fail(FLB_ERR_OOM, "host allocation failed");
  auto cleanup = [&](int code) {
    flb_destroy(h);
    return code;
  };
  h->desc = *desc;
  h->mode = mode;
  cudaGetDevice(&h->device);
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device) == cudaSuccess &&
      sms > 0)
    h->sm_count = sms;
  h->elem_bytes =
      desc->storage == FLB_STORAGE_FP16S ? 2 : (desc->storage == FLB_STORAGE_FP64 ? 8 : 4);
  h->real_bytes = desc->storage == FLB_STORAGE_FP64 ? 8 : 4;
  long long off = 0;
  for (HostBlock& b : blocks) {
    b.L.pitch = row_pitch(b.L.nx);
    b.L.plane = (long long)b.L.pitch * b.L.ny;
    b.base = off;
    off += (b.padded() + 63) / 64 * 64;
  }
  h->dstride = off;
  for (HostBlock& b : blocks) b.L.dstride = h->dstride;
  h->blocks = std::move(blocks);
  const size_t ds = size_t(h->dstride);
  const size_t popb = size_t(Q) * ds * h->elem_bytes;
  cudaError_t e;
  for (int k = 0; k < 2; ++k)
    if ((e = cudaMalloc(&h->pops[k], popb)) != cudaSuccess)
      return cleanup(fail(FLB_ERR_OOM, "cudaMalloc populations (%zu bytes): %s", popb,
                          cudaGetErrorString(e)));
  if ((e = cudaMalloc((void**)&h->flags, ds)) != cudaSuccess ||
      (e = cudaMalloc(&h->rho, ds * h->real_bytes)) != cudaSuccess ||
      (e = cudaMalloc(&h->vel, 3 * ds * h->real_bytes)) != cudaSuccess ||
      (e = cudaMalloc((void**)&h->acc, 64)) != cudaSuccess ||
      (e = cudaMemset(h->acc, 0, 64)) != cudaSuccess ||
      (e = cudaMalloc((void**)&h->red, RED_SLOTS * 4 * sizeof(double))) != cudaSuccess ||
      (e = cudaMalloc((void**)&h->d_lut, 256)) != cudaSuccess)
    return cleanup(fail(FLB_ERR_OOM, "cudaMalloc fields: %s", cudaGetErrorString(e)));
  if (desc->model == FLB_MODEL_BRINKMAN) {
    if ((e = cudaMalloc(&h->alpha, ds * h->real_bytes)) != cudaSuccess ||
        (e = cudaMemset(h->alpha, 0, ds * h->real_bytes)) != cudaSuccess)
      return cleanup(fail(FLB_ERR_OOM, "cudaMalloc alpha: %s", cudaGetErrorString(e)));
  }
  build_params(h);
  if (int rc0 = upload_op_lut(h)) return cleanup(rc0);
  for (const HostBlock& b : h->blocks)
    if ((long long)(b.L.pitch) * b.L.ny * b.L.nz >= (1LL << 32))
      return cleanup(fail(FLB_ERR_INVALID, "block of %lld padded cells exceeds 2^32",
                          (long long)(b.L.pitch) * b.L.ny * b.L.nz));
  if (mode == FLB_BLOCKS_HALO) {
    int rc = build_halo(h);
    if (rc) return cleanup(rc);
  }
  cudaStream_t st = 0;
  if ((e = cudaMemsetAsync(h->flags, 1, ds, st)) != cudaSuccess ||
      (e = cudaMemsetAsync(h->vel, 0, 3 * ds * h->real_bytes, st)) != cudaSuccess)
    return cleanup(fail(FLB_ERR_CUDA, "init memset: %s", cudaGetErrorString(e)));
  if (h->real_bytes == 8)
    k_fill<double><<<grid_1d(ds), 256, 0, st>>>(h->dstride, static_cast<double*>(h->rho),
                                                 desc->rho0);
  else
    k_fill<float><<<grid_1d(ds), 256, 0, st>>>(h->dstride, static_cast<float*>(h->rho),
                                                float(desc->rho0));
  int rc = flb_init_equilibrium(h, desc->rho0, nullptr);
  if (rc) return cleanup(rc);
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess)
    return cleanup(fail(FLB_ERR_CUDA, "create: %s", cudaGetErrorString(e)));
  *out = h;
  return FLB_OK;
}

// Run a per-block helper kernel over every block.
template <typename F>
int for_blocks(flb_lattice* h, F&& f) {
  for (const HostBlock& b : h->blocks) {
    int rc = f(b);
    if (rc) return rc;
  }
  return FLB_OK;
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
  FLB_TRY(validate_common(desc));
  FLB_TRY(validate_block(desc->nx, desc->ny, desc->nz));
  HostBlock b{};
  b.L.nx = desc->nx;
  b.L.ny = desc->ny;
  b.L.nz = desc->nz;
  b.omega = arith_omega(*desc, desc->omega);
  return create_common(desc, {b}, -1, out);
}

int flb_create_blocks(const flb_lattice_desc* desc, int nblocks, const flb_block_desc* blocks,
                      int mode, flb_lattice** out) {
  if (!out) return fail(FLB_ERR_INVALID, "null output handle");
  *out = nullptr;
  FLB_TRY(validate_common(desc));
  if (nblocks < 1 || !blocks) return fail(FLB_ERR_INVALID, "need at least one block");
  if (mode != FLB_BLOCKS_INDEPENDENT && mode != FLB_BLOCKS_HALO)
    return fail(FLB_ERR_INVALID, "bad multi-block mode %d", mode);
  std::vector<HostBlock> v(nblocks);
  for (int k = 0; k < nblocks; ++k) {
    const flb_block_desc& d = blocks[k];
    FLB_TRY(validate_block(d.nx, d.ny, d.nz));
    const double om = d.omega > 0.0 ? d.omega : desc->omega;
    if (!(om > 0.0 && om < 2.0)) return fail(FLB_ERR_INVALID, "block %d omega %g", k, om);
    v[k] = HostBlock{};
    v[k].L.nx = d.nx;
    v[k].L.ny = d.ny;
    v[k].L.nz = d.nz;
    v[k].ox = d.ox;
    v[k].oy = d.oy;
    v[k].oz = d.oz;
    v[k].omega = arith_omega(*desc, om);
  }
  return create_common(desc, std::move(v), mode, out);
}

int flb_destroy(flb_lattice* h) {
  if (!h) return FLB_OK;
  drop_graphs(h);
  flb_adjoint_release(h);
  if (h->alpha) cudaFree(h->alpha);
  for (void* p : {h->pops[0], h->pops[1], (void*)h->flags, h->rho, h->vel, (void*)h->acc,
                  (void*)h->red,
                  h->stage, (void*)h->uprev, (void*)h->d_blocks, (void*)h->d_halo,
                  (void*)h->d_lut, (void*)h->d_tile_block})
    if (p) cudaFree(p);
  delete h;
  return FLB_OK;
}

int flb_set_tasks(flb_lattice* h, int ntasks, const uint8_t* keys, const uint8_t* ops, int model) {
  if (!h) return fail(FLB_ERR_INVALID, "null handle");
  if (ntasks < 0 || ntasks > FLB_MAX_TASKS || (ntasks > 0 && (!keys || !ops)))
    return fail(FLB_ERR_INVALID, "ntasks %d outside [0, %d] or null lists", ntasks, FLB_MAX_TASKS);
  flb_lattice_desc d = h->desc;
  d.ntasks = ntasks;
  for (int t = 0; t < ntasks; ++t) {
    d.task_keys[t] = keys[t];
    d.task_ops[t] = ops[t];
  }
  d.model = model;
  FLB_TRY(validate_common(&d));
  if (model == FLB_MODEL_BRINKMAN && !h->alpha)
    return fail(FLB_ERR_STATE, "BRINKMAN needs the ALPHA field: create the lattice with it");
  h->desc = d;
  const StepParams keep = h->sp;
  build_params(h);
  h->sp.src = keep.src;
  h->sp.dst = keep.dst;
  drop_graphs(h);
  return upload_op_lut(h);
}

int flb_block_count(const flb_lattice* h, int* n) {
  if (!h || !n) return fail(FLB_ERR_INVALID, "null argument");
  *n = int(h->blocks.size());
  return FLB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Exchange between ranks: the global halo records whose two blocks have
// different owners.

namespace {

struct ExchPeer {
  int rank = -1;
  std::vector<long long> send, recv;  // element offsets (direction included)
  long long* d_send = nullptr;
  long long* d_recv = nullptr;
};

// Enumerate the global records in canonical order (block k, overlap cell
// z-y-x, direction) and hand every cross-rank one to `fn(k, lx, ly, lz, o, i)`
// (destination block k, local cell of k; source block o owning that cell).
template <typename F>
int for_each_cross_record(int nglobal, const flb_block_desc* blocks, const int* owner_rank,
                          int halo_mode, F&& fn) {
  int gx = 0, gy = 0, gz = 0;
  for (int k = 0; k < nglobal; ++k) {
    const flb_block_desc& b = blocks[k];
    if (b.ox < 0 || b.oy < 0 || b.oz < 0 || b.nx < 3 || b.ny < 3 || b.nz < 3)
      return fail(FLB_ERR_INVALID, "global block %d: bad extent or origin", k);
    gx = std::max(gx, b.ox + b.nx);
    gy = std::max(gy, b.oy + b.ny);
    gz = std::max(gz, b.oz + b.nz);
  }
  const long long gn = (long long)gx * gy * gz;
  if (gn > (1LL << 33)) return fail(FLB_ERR_INVALID, "global block extent too large");
  std::vector<int> owner(size_t(gn), -1);
  for (int k = 0; k < nglobal; ++k) {
    const flb_block_desc& b = blocks[k];
    for (int z = b.oz + 1; z < b.oz + b.nz - 1; ++z)
      for (int y = b.oy + 1; y < b.oy + b.ny - 1; ++y)
        for (int x = b.ox + 1; x < b.ox + b.nx - 1; ++x) {
          int& o = owner[size_t((long long)(z * (long long)gy + y) * gx + x)];
          if (o >= 0) return fail(FLB_ERR_INVALID, "blocks %d and %d overlap in their interiors", o, k);
          o = k;
        }
  }
  const bool full = halo_mode == FLB_HALO_FULL;
  for (int k = 0; k < nglobal; ++k) {
    const flb_block_desc& b = blocks[k];
    for (int lz = 0; lz < b.nz; ++lz)
      for (int ly = 0; ly < b.ny; ++ly)
        for (int lx = 0; lx < b.nx; ++lx) {
          if (lx > 0 && ly > 0 && lz > 0 && lx < b.nx - 1 && ly < b.ny - 1 && lz < b.nz - 1)
            continue;
          const int o = owner[size_t((long long)((b.oz + lz) * (long long)gy + (b.oy + ly)) * gx +
                                     (b.ox + lx))];
          if (o < 0 || owner_rank[o] == owner_rank[k]) continue;
          const int l[3] = {lx, ly, lz};
          const int m[3] = {b.nx, b.ny, b.nz};
          for (int i = full ? 0 : 1; i < Q; ++i) {
            const int c[3] = {cx(i), cy(i), cz(i)};
            bool cross = false;
            for (int a = 0; a < 3; ++a)
              if ((l[a] == 0 && c[a] > 0) || (l[a] == m[a] - 1 && c[a] < 0)) cross = true;
            if (!cross && !full) continue;
            fn(k, lx, ly, lz, o, i);
          }
        }
  }
  return FLB_OK;
}

template <typename E>
__global__ void k_exch_gather(const long long* __restrict__ idx, long long n, const E* pops,
                              E* buf) {
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n;
       r += (long long)gridDim.x * blockDim.x)
    buf[r] = pops[idx[r]];
}
template <typename E>
__global__ void k_exch_scatter(const long long* __restrict__ idx, long long n, const E* buf,
                               E* pops) {
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n;
       r += (long long)gridDim.x * blockDim.x)
    pops[idx[r]] = buf[r];
}

}  // namespace

struct flb_exchange {
  int my_rank = 0;
  int elem_bytes = 4;
  int halo_mode = FLB_HALO_NORMAL;  // the handle's mode the plan was built for
  long long dstride = 0;
  std::vector<ExchPeer> peers;  // sorted by rank
};

namespace {
ExchPeer* find_peer(flb_exchange* ex, int rank) {
  for (ExchPeer& p : ex->peers)
    if (p.rank == rank) return &p;
  return nullptr;
}
template <typename E>
void exch_launch(const long long* idx, long long n, const void* src, void* dst, bool gather,
                 cudaStream_t st) {
  const unsigned grid = unsigned(std::min<long long>(n / 256 + 1, 4096));
  if (gather)
    k_exch_gather<E><<<grid, 256, 0, st>>>(idx, n, static_cast<const E*>(src),
                                           static_cast<E*>(dst));
  else
    k_exch_scatter<E><<<grid, 256, 0, st>>>(idx, n, static_cast<const E*>(src),
                                            static_cast<E*>(dst));
}
int exch_move(flb_exchange* ex, flb_lattice* h, int peer, void* buf, bool pack, void* stream) {
  if (!ex || !h || !buf) return fail(FLB_ERR_INVALID, "null argument");
  if (h->dstride != ex->dstride || h->elem_bytes != ex->elem_bytes)
    return fail(FLB_ERR_INVALID, "lattice differs from the one the exchange was built for");
  if (h->halo_mode != ex->halo_mode)
    return fail(FLB_ERR_STATE, "halo mode changed after flb_exchange_create: rebuild the exchange");
  ExchPeer* p = find_peer(ex, peer);
  if (!p) return fail(FLB_ERR_INVALID, "rank %d is not a peer of rank %d", peer, ex->my_rank);
  const long long n = pack ? (long long)p->send.size() : (long long)p->recv.size();
  if (n == 0) return FLB_OK;
  const long long* idx = pack ? p->d_send : p->d_recv;
  cudaStream_t st = as_stream(stream);
  void* pops = h->pops[h->cur];
  const void* src = pack ? pops : buf;
  void* dst = pack ? buf : pops;
  if (ex->elem_bytes == 2) exch_launch<unsigned short>(idx, n, src, dst, pack, st);
  else if (ex->elem_bytes == 8) exch_launch<unsigned long long>(idx, n, src, dst, pack, st);
  else exch_launch<unsigned>(idx, n, src, dst, pack, st);
  FLB_CUDA(cudaGetLastError());
  return FLB_OK;
}
}  // namespace

extern "C" {

int flb_exchange_plan(int nglobal, const flb_block_desc* blocks, const int* owner_rank,
                      int my_rank, int halo_mode, int max_peers, int* npeers, int* peer_ranks,
                      long long* send_counts, long long* recv_counts) {
  if (nglobal < 1 || !blocks || !owner_rank || !npeers)
    return fail(FLB_ERR_INVALID, "flb_exchange_plan: bad arguments");
  std::map<int, std::pair<long long, long long>> cnt;  // peer -> (send, recv)
  FLB_TRY(for_each_cross_record(nglobal, blocks, owner_rank, halo_mode,
                                [&](int k, int, int, int, int o, int) {
                                  if (owner_rank[k] == my_rank) ++cnt[owner_rank[o]].second;
                                  if (owner_rank[o] == my_rank) ++cnt[owner_rank[k]].first;
                                }));
  *npeers = int(cnt.size());
  if (int(cnt.size()) > max_peers)
    return fail(FLB_ERR_INVALID, "flb_exchange_plan: %d peers > max_peers %d", int(cnt.size()),
                max_peers);
  int j = 0;
  for (const auto& kv : cnt) {
    if (peer_ranks) peer_ranks[j] = kv.first;
    if (send_counts) send_counts[j] = kv.second.first;
    if (recv_counts) recv_counts[j] = kv.second.second;
    ++j;
  }
  return FLB_OK;
}

int flb_exchange_create(flb_lattice* h, int nglobal, const flb_block_desc* blocks,
                        const int* owner_rank, int my_rank, flb_exchange** out) {
  if (!h || !out || nglobal < 1 || !blocks || !owner_rank)
    return fail(FLB_ERR_INVALID, "flb_exchange_create: bad arguments");
  *out = nullptr;
  // the handle's blocks must be the ones my_rank owns, in global order
  std::vector<int> local(size_t(nglobal), -1);
  int nl = 0;
  for (int k = 0; k < nglobal; ++k) {
    if (owner_rank[k] != my_rank) continue;
    if (nl >= int(h->blocks.size()))
      return fail(FLB_ERR_INVALID, "rank %d owns more blocks than the handle holds", my_rank);
    const HostBlock& hb = h->blocks[size_t(nl)];
    const flb_block_desc& b = blocks[k];
    if (hb.L.nx != b.nx || hb.L.ny != b.ny || hb.L.nz != b.nz || hb.ox != b.ox ||
        hb.oy != b.oy || hb.oz != b.oz)
      return fail(FLB_ERR_INVALID, "handle block %d differs from global block %d", nl, k);
    local[size_t(k)] = nl++;
  }
  if (nl != int(h->blocks.size()))
    return fail(FLB_ERR_INVALID, "the handle holds %d blocks, rank %d owns %d",
                int(h->blocks.size()), my_rank, nl);
  std::map<int, ExchPeer> peers;
  FLB_TRY(for_each_cross_record(
      nglobal, blocks, owner_rank, h->halo_mode, [&](int k, int lx, int ly, int lz, int o, int i) {
        if (owner_rank[k] == my_rank) {  // receive into block k's overlap slot
          ExchPeer& p = peers[owner_rank[o]];
          const Geom g = geom_of(h->blocks[size_t(local[size_t(k)])]);
          p.recv.push_back(i * h->dstride + host_wrap_src(g, lx, ly, lz, i));
        }
        if (owner_rank[o] == my_rank) {  // send from block o's interior slot
          ExchPeer& p = peers[owner_rank[k]];
          const HostBlock& hb = h->blocks[size_t(local[size_t(o)])];
          const flb_block_desc& bk = blocks[k];
          p.send.push_back(i * h->dstride + host_wrap_src(geom_of(hb), bk.ox + lx - hb.ox,
                                                          bk.oy + ly - hb.oy,
                                                          bk.oz + lz - hb.oz, i));
        }
      }));
  flb_exchange* ex = new (std::nothrow) flb_exchange();
  if (!ex) return fail(FLB_ERR_OOM, "flb_exchange_create: host allocation");
  ex->my_rank = my_rank;
  ex->elem_bytes = h->elem_bytes;
  ex->halo_mode = h->halo_mode;
  ex->dstride = h->dstride;
  for (auto& kv : peers) {
    kv.second.rank = kv.first;
    ex->peers.push_back(std::move(kv.second));
  }
  for (ExchPeer& p : ex->peers) {
    cudaError_t e = cudaSuccess;
    if (!p.send.empty()) {
      e = cudaMalloc((void**)&p.d_send, p.send.size() * sizeof(long long));
      if (e == cudaSuccess)
        e = cudaMemcpy(p.d_send, p.send.data(), p.send.size() * sizeof(long long),
                       cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess && !p.recv.empty()) {
      e = cudaMalloc((void**)&p.d_recv, p.recv.size() * sizeof(long long));
      if (e == cudaSuccess)
        e = cudaMemcpy(p.d_recv, p.recv.data(), p.recv.size() * sizeof(long long),
                       cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) {
      flb_exchange_destroy(ex);
      return fail(FLB_ERR_OOM, "flb_exchange_create: %s", cudaGetErrorString(e));
    }
  }
  *out = ex;
  return FLB_OK;
}

int flb_exchange_peers(const flb_exchange* ex, int max_peers, int* npeers, int* peer_ranks,
                       long long* send_counts, long long* recv_counts) {
  if (!ex || !npeers) return fail(FLB_ERR_INVALID, "null argument");
  *npeers = int(ex->peers.size());
  if (*npeers > max_peers)
    return fail(FLB_ERR_INVALID, "%d peers > max_peers %d", *npeers, max_peers);
  for (size_t j = 0; j < ex->peers.size(); ++j) {
    if (peer_ranks) peer_ranks[j] = ex->peers[j].rank;
    if (send_counts) send_counts[j] = (long long)ex->peers[j].send.size();
    if (recv_counts) recv_counts[j] = (long long)ex->peers[j].recv.size();
  }
  return FLB_OK;
}

int flb_exchange_pack(flb_exchange* ex, flb_lattice* h, int peer, void* buf, void* stream) {
  return exch_move(ex, h, peer, buf, true, stream);
}

int flb_exchange_unpack(flb_exchange* ex, flb_lattice* h, int peer, const void* buf,
                        void* stream) {
  return exch_move(ex, h, peer, const_cast<void*>(buf), false, stream);
}

int flb_exchange_destroy(flb_exchange* ex) {
  if (!ex) return FLB_OK;
  for (ExchPeer& p : ex->peers) {
    if (p.d_send) cudaFree(p.d_send);
    if (p.d_recv) cudaFree(p.d_recv);
  }
  delete ex;
  return FLB_OK;
}

int flb_halo_count(const flb_lattice* h, long long* n) {
  if (!h || !n) return fail(FLB_ERR_INVALID, "null argument");
  *n = h->nhalo;
  return FLB_OK;
}

int flb_set_halo_mode(flb_lattice* h, int mode) {
  if (!h) return fail(FLB_ERR_INVALID, "null handle");
  if (mode != FLB_HALO_NORMAL && mode != FLB_HALO_FULL)
    return fail(FLB_ERR_INVALID, "unknown halo mode %d", mode);
  if (h->mode != FLB_BLOCKS_HALO)
    return fail(FLB_ERR_STATE, "halo mode applies to FLB_BLOCKS_HALO handles");
  if (mode == h->halo_mode) return FLB_OK;
  FLB_CUDA(cudaDeviceSynchronize());  // the old records may be in use by queued steps
  h->halo_mode = mode;
  drop_graphs(h);
  return build_halo(h);
}

int flb_memory_bytes(const flb_lattice* h, size_t* bytes) {
  if (!h || !bytes) return fail(FLB_ERR_INVALID, "null argument");
  const size_t ds = size_t(h->dstride);
  *bytes = 2 * size_t(Q) * ds * h->elem_bytes + ds + 4 * ds * h->real_bytes + 64 +
           h->stage_bytes + (h->uprev ? 3 * ds * sizeof(double) : 0) +
           h->blocks.size() * sizeof(BlockEntry) + size_t(h->tile_block_cap) * sizeof(int) +
           size_t(h->nhalo) * (h->halo32 ? sizeof(uint2) : sizeof(HaloCopy));
  return FLB_OK;
}

int flb_upload_flags(flb_lattice* h, const uint8_t* host, void* stream) {
  return flags_any(h, 0, const_cast<uint8_t*>(host), true, stream);
}
int flb_download_flags(flb_lattice* h, uint8_t* host, void* stream) {
  return flags_any(h, 0, host, false, stream);
}
int flb_upload_flags_block(flb_lattice* h, int b, const uint8_t* host, void* stream) {
  return flags_any(h, b, const_cast<uint8_t*>(host), true, stream);
}
int flb_download_flags_block(flb_lattice* h, int b, uint8_t* host, void* stream) {
  return flags_any(h, b, host, false, stream);
}

int flb_upload_pops(flb_lattice* h, const void* host, int dt, void* stream) {
  return pops_any(h, 0, const_cast<void*>(host), dt, true, stream);
}
int flb_download_pops(flb_lattice* h, void* host, int dt, void* stream) {
  return pops_any(h, 0, host, dt, false, stream);
}
int flb_upload_pops_block(flb_lattice* h, int b, const void* host, int dt, void* stream) {
  return pops_any(h, b, const_cast<void*>(host), dt, true, stream);
}
int flb_download_pops_block(flb_lattice* h, int b, void* host, int dt, void* stream) {
  return pops_any(h, b, host, dt, false, stream);
}

int flb_upload_field(flb_lattice* h, int field, const void* host, int dt, void* stream) {
  return field_any(h, 0, field, const_cast<void*>(host), dt, true, stream);
}
int flb_download_field(flb_lattice* h, int field, void* host, int dt, void* stream) {
  return field_any(h, 0, field, host, dt, false, stream);
}
int flb_upload_field_block(flb_lattice* h, int b, int field, const void* host, int dt,
                           void* stream) {
  return field_any(h, b, field, const_cast<void*>(host), dt, true, stream);
}
int flb_download_field_block(flb_lattice* h, int b, int field, void* host, int dt,
                             void* stream) {
  return field_any(h, b, field, host, dt, false, stream);
}

int flb_init_equilibrium(flb_lattice* h, double rho0, void* stream) {
  if (!h) return fail(FLB_ERR_INVALID, "null handle");
  cudaStream_t st = as_stream(stream);
  FLB_TRY(with_types(h, [&](auto* sp, auto* rp) {
    using S = std::remove_pointer_t<decltype(sp)>;
    using R = std::remove_pointer_t<decltype(rp)>;
    return for_blocks(h, [&](const HostBlock& b) {
      k_init_equilibrium<S, R><<<grid_1d(b.padded()), 256, 0, st>>>(
          b.L, static_cast<S*>(h->pops[h->cur]) + b.base, rho0, h->sp);
      return FLB_OK;
    });
  }));
  FLB_CUDA(cudaGetLastError());
  return FLB_OK;
}

int flb_step(flb_lattice* h, int nsteps, void* stream) {
  if (!h) return fail(FLB_ERR_INVALID, "null handle");
  if (nsteps < 0) return fail(FLB_ERR_INVALID, "nsteps %d < 0", nsteps);
  if (nsteps == 0) return FLB_OK;
  return step_any(h, nsteps, as_stream(stream));
}

int flb_step_graph(flb_lattice* h, int nsteps, void* stream) {
  if (!h) return fail(FLB_ERR_INVALID, "null handle");
  if (nsteps < 0) return fail(FLB_ERR_INVALID, "nsteps %d < 0", nsteps);
  cudaStream_t st = as_stream(stream);
  const int pairs = nsteps / 2;
  if (pairs > 0) {
    const int parity = h->cur;
    if (!h->graph[parity]) {
      if (h->mode >= 0 || h->ctas_per_sm > 0) FLB_TRY(upload_block_table(h));
      cudaStream_t cap;
      FLB_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
      cudaGraph_t graph = nullptr;
      cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
      int rc = FLB_OK;
      if (e == cudaSuccess) {
        rc = step_any(h, 2, cap);  // advances h->cur by two: parity unchanged
        e = cudaStreamEndCapture(cap, &graph);
      }
      cudaStreamDestroy(cap);
      if (rc) return rc;
      if (e != cudaSuccess) return fail(FLB_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
      e = cudaGraphInstantiate(&h->graph[parity], graph, 0);
      cudaGraphDestroy(graph);
      if (e != cudaSuccess)
        return fail(FLB_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    }
    for (int k = 0; k < pairs; ++k) FLB_CUDA(cudaGraphLaunch(h->graph[parity], st));
  }
  if (nsteps & 1) return step_any(h, 1, st);
  return FLB_OK;
}

int flb_set_launch(flb_lattice* h, int tile_y, int ctas_per_sm, int cells_per_thread) {
  if (!h) return fail(FLB_ERR_INVALID, "null handle");
  if (cells_per_thread != 0 && !vec_allowed(h->desc.storage, cells_per_thread))
    return fail(FLB_ERR_INVALID, "cells_per_thread %d not built for this storage",
                cells_per_thread);
  if (tile_y != 1 && tile_y != 2 && tile_y != 4 && tile_y != 8)
    return fail(FLB_ERR_INVALID, "tile_y %d not in {1,2,4,8}", tile_y);
  if (ctas_per_sm < -3 || ctas_per_sm > 32)
    return fail(FLB_ERR_INVALID, "ctas_per_sm %d outside [-3, 32]", ctas_per_sm);
  const int v = cells_per_thread ? cells_per_thread : default_vec(h->desc.storage);
  if (ctas_per_sm <= -2) {
    if (!tma_supported(h))
      return fail(FLB_ERR_UNSUPPORTED,
                  "ctas_per_sm -2 / -3 (bulk-copy kernel) needs a single-block FP16S handle "
                  "with 16-byte aligned rows");
    if (v != 4) return fail(FLB_ERR_INVALID, "ctas_per_sm -2 / -3 runs 4 cells per thread");
    FLB_TRY(tma_prepare(h));
  } else if (ctas_per_sm < 0) {
    if (!pipe_supported(h))
      return fail(FLB_ERR_UNSUPPORTED,
                  "ctas_per_sm -1 (async-copy pipeline) needs a single-block FP16S handle");
    if (v != PIPE_V)
      return fail(FLB_ERR_INVALID, "ctas_per_sm -1 runs %d cells per thread", PIPE_V);
    FLB_TRY(pipe_prepare(h));
  }
  if (tile_y != h->tile_y || ctas_per_sm != h->ctas_per_sm || v != vec_width(h)) drop_graphs(h);
  h->tile_y = tile_y;
  h->ctas_per_sm = ctas_per_sm;
  h->vec = v;
  return FLB_OK;
}

int flb_set_wait_limit(flb_lattice* h, double seconds) {
  if (!h) return fail(FLB_ERR_INVALID, "null handle");
  if (!(seconds >= 0.0 && seconds <= 60.0))
    return fail(FLB_ERR_INVALID, "wait limit %g s outside [0, 60]", seconds);
  h->wait_s = seconds;
  drop_graphs(h);  // the captured launches carry the old limit
  return FLB_OK;
}

int flb_set_rounding(flb_lattice* h, int mode) {
  if (!h) return fail(FLB_ERR_INVALID, "null handle");
  if (mode != FLB_ROUND_DEFAULT && mode != FLB_ROUND_NEAREST && mode != FLB_ROUND_STOCHASTIC)
    return fail(FLB_ERR_INVALID, "rounding mode %d", mode);
  h->rounding = mode;
  const StepParams keep = h->sp;
  build_params(h);
  h->sp.src = keep.src;
  h->sp.dst = keep.dst;
  drop_graphs(h);  // the captured launches carry the old mode
  return FLB_OK;
}

int flb_get_rounding(const flb_lattice* h, int* mode) {
  if (!h || !mode) return fail(FLB_ERR_INVALID, "null argument");
  *mode = h->sp.fp16_round ? FLB_ROUND_STOCHASTIC : FLB_ROUND_NEAREST;
  return FLB_OK;
}

int flb_test_withhold_tile(flb_lattice* h, long long tile) {
  if (!h) return fail(FLB_ERR_INVALID, "null handle");
  if (tile < -1) return fail(FLB_ERR_INVALID, "tile %lld < -1", tile);
  h->withhold = tile;
  drop_graphs(h);
  return FLB_OK;
}

int flb_device_status(flb_lattice* h, void* stream) {
  if (!h) return fail(FLB_ERR_INVALID, "null handle");
  cudaStream_t st = as_stream(stream);
  int v = 0;
  FLB_CUDA(cudaMemcpyAsync(&v, status_word(h), sizeof v, cudaMemcpyDeviceToHost, st));
  FLB_CUDA(cudaStreamSynchronize(st));
  if (v == 0) return FLB_OK;
  FLB_CUDA(cudaMemsetAsync(status_word(h), 0, sizeof v, st));
  FLB_CUDA(cudaStreamSynchronize(st));
  return fail(v, "a device-side wait gave up (status %d): the steps since the last check "
                 "are incomplete", v);
}

int flb_get_launch(const flb_lattice* h, int* tile_y, int* ctas_per_sm, int* cells_per_thread) {
  if (!h) return fail(FLB_ERR_INVALID, "null handle");
  if (tile_y) *tile_y = h->tile_y;
  if (ctas_per_sm) *ctas_per_sm = h->ctas_per_sm;
  if (cells_per_thread) *cells_per_thread = vec_width(h);
  return FLB_OK;
}

int flb_autotune(flb_lattice* h, int trial_steps, void* stream, int* tile_y, int* ctas_per_sm,
                 int* cells_per_thread, double* best_ms, int* steps_taken) {
  if (!h) return fail(FLB_ERR_INVALID, "null handle");
  if (trial_steps < 1) return fail(FLB_ERR_INVALID, "trial_steps %d < 1", trial_steps);
  cudaStream_t st = as_stream(stream);
  const int tys[] = {1, 2, 4, 8};
  const int ctas_list[] = {0, 8, 16, 32};
  const int nctas = 4;
  const int vecs_d[] = {1, 2}, vecs_f[] = {2, 4};
  const int* vecs = h->desc.storage == FLB_STORAGE_FP64 ? vecs_d : vecs_f;
  const int ty0 = h->tile_y, c0 = h->ctas_per_sm, v0 = vec_width(h);
  int best_ty = ty0, best_c = c0, best_v = v0, taken = 0;
  float best = 1e30f;
  cudaEvent_t e0, e1;
  FLB_CUDA(cudaEventCreate(&e0));
  FLB_CUDA(cudaEventCreate(&e1));
  int rc = FLB_OK;
  for (int vi = 0; vi < 2 && !rc; ++vi) {
    for (int ty : tys) {
      for (int ci = 0; ci < nctas; ++ci) {
        const int c = ctas_list[ci];
        if ((rc = flb_set_launch(h, ty, c, vecs[vi]))) break;
        if ((rc = step_any(h, 1, st))) break;  // warm-up (block table upload, caches)
        cudaEventRecord(e0, st);
        if ((rc = step_any(h, trial_steps, st))) break;
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        taken += trial_steps + 1;
        if (ms < best) {
          best = ms;
          best_ty = ty;
          best_c = c;
          best_v = vecs[vi];
        }
      }
      if (rc) break;
    }
  }
  if (!rc && pipe_supported(h)) {  // the async-copy pipeline (fixed shape)
    rc = flb_set_launch(h, 4, -1, PIPE_V);
    if (!rc) rc = step_any(h, 1, st);
    if (!rc) {
      cudaEventRecord(e0, st);
      rc = step_any(h, trial_steps, st);
      cudaEventRecord(e1, st);
    }
    if (!rc) {
      cudaEventSynchronize(e1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      taken += trial_steps + 1;
      if (ms < best) {
        best = ms;
        best_ty = 4;
        best_c = -1;
        best_v = PIPE_V;
      }
    }
  }
  for (int ns = -2; !rc && ns >= -3 && tma_supported(h); --ns) {  // the bulk-copy kernel
    rc = flb_set_launch(h, 4, ns, 4);
    if (!rc) rc = step_any(h, 1, st);
    if (!rc) {
      cudaEventRecord(e0, st);
      rc = step_any(h, trial_steps, st);
      cudaEventRecord(e1, st);
    }
    if (!rc) {
      cudaEventSynchronize(e1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      taken += trial_steps + 1;
      if (ms < best) {
        best = ms;
        best_ty = 4;
        best_c = ns;
        best_v = 4;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) {
    flb_set_launch(h, ty0, c0, v0);
    return rc;
  }
  FLB_TRY(flb_set_launch(h, best_ty, best_c, best_v));
  if (tile_y) *tile_y = best_ty;
  if (ctas_per_sm) *ctas_per_sm = best_c;
  if (cells_per_thread) *cells_per_thread = best_v;
  if (best_ms) *best_ms = double(best) / trial_steps;
  if (steps_taken) *steps_taken = taken;
  return FLB_OK;
}

int flb_compute_rhou(flb_lattice* h, uint8_t key, void* stream) {
  if (!h) return fail(FLB_ERR_INVALID, "null handle");
  cudaStream_t st = as_stream(stream);
  FLB_TRY(with_types(h, [&](auto* sp, auto* rp) {
    using S = std::remove_pointer_t<decltype(sp)>;
    using R = std::remove_pointer_t<decltype(rp)>;
    return for_blocks(h, [&](const HostBlock& b) {
      k_rhou_pull<S, R><<<grid_1d(b.padded()), 256, 0, st>>>(
          b.L, geom_of(b), static_cast<const S*>(h->pops[h->cur]), h->flags, key,
          static_cast<R*>(h->rho), static_cast<R*>(h->vel), h->sp);
      return FLB_OK;
    });
  }));
  FLB_CUDA(cudaGetLastError());
  return FLB_OK;
}

int flb_reduce_conservation(flb_lattice* h, uint8_t key, double out[4], void* stream) {
  if (!h || !out) return fail(FLB_ERR_INVALID, "null argument");
  cudaStream_t st = as_stream(stream);
  FLB_CUDA(cudaMemsetAsync(h->acc, 0, 4 * sizeof(double), st));
  FLB_TRY(with_types(h, [&](auto* sp, auto* rp) {
    using S = std::remove_pointer_t<decltype(sp)>;
    using R = std::remove_pointer_t<decltype(rp)>;
    return for_blocks(h, [&](const HostBlock& b) {
      const int grid = grid_1d(b.padded());
      k_conservation_pull<S, R><<<grid, 256, 0, st>>>(
          b.L, geom_of(b), static_cast<const S*>(h->pops[h->cur]), h->flags, key, h->red,
          h->sp);
      k_sum_partials<<<1, 256, 0, st>>>(h->red, grid, 4, h->acc);  // blocks in order
      return FLB_OK;
    });
  }));
  FLB_CUDA(cudaGetLastError());
  FLB_CUDA(cudaMemcpyAsync(out, h->acc, 4 * sizeof(double), cudaMemcpyDeviceToHost, st));
  FLB_CUDA(cudaStreamSynchronize(st));
  return FLB_OK;
}

int flb_tolerance_u(flb_lattice* h, uint8_t key, double* max_du, void* stream) {
  if (!h || !max_du) return fail(FLB_ERR_INVALID, "null argument");
  cudaStream_t st = as_stream(stream);
  if (!h->uprev) {
    FLB_CUDA(cudaMalloc((void**)&h->uprev, 3 * size_t(h->dstride) * sizeof(double)));
    FLB_CUDA(cudaMemsetAsync(h->uprev, 0, 3 * size_t(h->dstride) * sizeof(double), st));
  }
  unsigned long long* acc = reinterpret_cast<unsigned long long*>(h->acc);
  FLB_CUDA(cudaMemsetAsync(acc, 0, sizeof(unsigned long long), st));
  FLB_TRY(with_types(h, [&](auto* sp, auto* rp) {
    using S = std::remove_pointer_t<decltype(sp)>;
    using R = std::remove_pointer_t<decltype(rp)>;
    return for_blocks(h, [&](const HostBlock& b) {
      k_tolerance_pull<S, R><<<grid_1d(b.padded()), 256, 0, st>>>(
          b.L, geom_of(b), static_cast<const S*>(h->pops[h->cur]), h->flags, key, h->uprev,
          acc, h->sp);
      return FLB_OK;
    });
  }));
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
  unsigned long long* acc = reinterpret_cast<unsigned long long*>(h->acc);
  FLB_CUDA(cudaMemsetAsync(acc, 0, sizeof(unsigned long long), st));
  FLB_TRY(with_types(h, [&](auto* sp, auto* rp) {
    using S = std::remove_pointer_t<decltype(sp)>;
    using R = std::remove_pointer_t<decltype(rp)>;
    return for_blocks(h, [&](const HostBlock& b) {
      k_finite<S, R><<<grid_1d(b.padded()), 256, 0, st>>>(
          b.L, static_cast<const S*>(h->pops[h->cur]) + b.base, h->flags + b.base, acc, h->sp);
      return FLB_OK;
    });
  }));
  FLB_CUDA(cudaGetLastError());
  unsigned long long v = 0;
  FLB_CUDA(cudaMemcpyAsync(&v, acc, sizeof v, cudaMemcpyDeviceToHost, st));
  FLB_CUDA(cudaStreamSynchronize(st));
  *bad = v;
  if (v) return fail(FLB_ERR_NUMERIC, "%llu non-finite populations", v);
  return FLB_OK;
}

// Snapshots: a 64-byte header, then the populations of every block in the
// device layout (padded rows, the post-collision convention), as stored.
namespace {
struct SnapHeader {
  char magic[8];        // "FLBSNAP1"
  long long nbytes;     // population bytes after the header
  long long dstride;    // elements per population array
  int storage, nblocks;
  unsigned long long geom;  // hash of the block shapes and origins
  long long reserved[3];
};
static_assert(sizeof(SnapHeader) == 64, "snapshot header");

unsigned long long geom_hash(const flb_lattice* h) {
  unsigned long long x = 1469598103934665603ULL;  // FNV-1a over the block table
  auto mix = [&](long long v) {
    for (int b = 0; b < 8; ++b) {
      x ^= (unsigned long long)(v >> (8 * b)) & 0xffULL;
      x *= 1099511628211ULL;
    }
  };
  for (const HostBlock& b : h->blocks) {
    mix(b.L.nx); mix(b.L.ny); mix(b.L.nz); mix(b.ox); mix(b.oy); mix(b.oz); mix(b.base);
  }
  return x;
}

SnapHeader snap_header(const flb_lattice* h) {
  SnapHeader hd{};
  std::memcpy(hd.magic, "FLBSNAP1", 8);
  hd.nbytes = (long long)Q * h->dstride * h->elem_bytes;
  hd.dstride = h->dstride;
  hd.storage = h->desc.storage;
  hd.nblocks = int(h->blocks.size());
  hd.geom = geom_hash(h);
  return hd;
}
}  // namespace

int flb_snapshot_bytes(const flb_lattice* h, size_t* bytes) {
  if (!h || !bytes) return fail(FLB_ERR_INVALID, "null argument");
  *bytes = sizeof(SnapHeader) + size_t(Q) * size_t(h->dstride) * h->elem_bytes;
  return FLB_OK;
}

int flb_snapshot_save(flb_lattice* h, void* dst, size_t cap, void* stream) {
  if (!h || !dst) return fail(FLB_ERR_INVALID, "null argument");
  const SnapHeader hd = snap_header(h);
  if (cap < sizeof hd + size_t(hd.nbytes))
    return fail(FLB_ERR_INVALID, "snapshot buffer of %zu bytes < %zu", cap,
                sizeof hd + size_t(hd.nbytes));
  cudaStream_t st = as_stream(stream);
  char* d = static_cast<char*>(dst);
  // the header is copied from the handle, which outlives the stream's copy
  // (every header of a handle is the same bytes); the populations follow
  static_assert(sizeof hd == sizeof h->snap_hdr, "snapshot header size");
  std::memcpy(h->snap_hdr, &hd, sizeof hd);
  FLB_CUDA(cudaMemcpyAsync(d, h->snap_hdr, sizeof hd, cudaMemcpyDefault, st));
  FLB_CUDA(cudaMemcpyAsync(d + sizeof hd, h->pops[h->cur], size_t(hd.nbytes), cudaMemcpyDefault,
                           st));
  return FLB_OK;
}

int flb_snapshot_restore(flb_lattice* h, const void* src, size_t bytes, void* stream) {
  if (!h || !src) return fail(FLB_ERR_INVALID, "null argument");
  const SnapHeader want = snap_header(h);
  if (bytes < sizeof want + size_t(want.nbytes))
    return fail(FLB_ERR_INVALID, "snapshot of %zu bytes < %zu", bytes,
                sizeof want + size_t(want.nbytes));
  cudaStream_t st = as_stream(stream);
  SnapHeader got{};
  FLB_CUDA(cudaMemcpyAsync(&got, src, sizeof got, cudaMemcpyDefault, st));
  FLB_CUDA(cudaStreamSynchronize(st));
  if (std::memcmp(got.magic, want.magic, 8) != 0) return fail(FLB_ERR_INVALID, "not a snapshot");
  if (got.nbytes != want.nbytes || got.dstride != want.dstride || got.storage != want.storage ||
      got.nblocks != want.nblocks || got.geom != want.geom)
    return fail(FLB_ERR_INVALID, "snapshot of another lattice (storage, blocks or shape)");
  FLB_CUDA(cudaMemcpyAsync(h->pops[h->cur], static_cast<const char*>(src) + sizeof got,
                           size_t(want.nbytes), cudaMemcpyDefault, st));
  return FLB_OK;
}

int flb_get_layout(const flb_lattice* h, flb_layout* layout) {
  if (!h || !layout) return fail(FLB_ERR_INVALID, "null argument");
  const HostBlock& b = h->blocks[0];
  layout->nx = b.L.nx;
  layout->ny = b.L.ny;
  layout->nz = b.L.nz;
  layout->pitch_x = b.L.pitch;
  layout->plane = size_t(b.L.plane);
  layout->dir_stride = size_t(h->dstride);
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

int flb_objective_u2(flb_lattice* h, double* J, void* stream) {
  if (!h || !J) return fail(FLB_ERR_INVALID, "null argument");
  if (h->blocks.size() != 1) return fail(FLB_ERR_UNSUPPORTED, "objective on single-block handles");
  if (h->desc.storage == FLB_STORAGE_FP16S)
    return fail(FLB_ERR_UNSUPPORTED, "objective is built for FP32, FP32S and FP64 storage");
  cudaStream_t st = as_stream(stream);
  double* jacc = h->acc + 4;
  FLB_CUDA(cudaMemsetAsync(jacc, 0, sizeof(double), st));
  const HostBlock& b = h->blocks[0];
  int rc = with_types(h, [&](auto* sp, auto* rp) {
    using S = std::remove_pointer_t<decltype(sp)>;
    using R = std::remove_pointer_t<decltype(rp)>;
    if constexpr (!std::is_same<S, __half>::value) {
      const int grid = grid_1d(b.padded());
      k_objective<S, R><<<grid, 256, 0, st>>>(
          b.L, geom_of(b), static_cast<const S*>(h->pops[h->cur]), h->sp, (R*)nullptr,
          (double*)nullptr, h->red, false);
      k_sum_partials_dd<<<1, 256, 0, st>>>(h->red, grid, jacc);
    }
    return FLB_OK;
  });
  if (rc) return rc;
  FLB_CUDA(cudaGetLastError());
  FLB_CUDA(cudaMemcpyAsync(J, jacc, sizeof(double), cudaMemcpyDeviceToHost, st));
  FLB_CUDA(cudaStreamSynchronize(st));
  return FLB_OK;
}

int flb_adjoint_release(flb_lattice* h) {
  if (!h) return fail(FLB_ERR_INVALID, "null handle");
  for (void* p : h->adj_ckpt) cudaFree(p);
  for (void* p : h->adj_seg) cudaFree(p);
  h->adj_ckpt.clear();
  h->adj_seg.clear();
  for (auto& p : h->adj_lam)
    if (p) {
      cudaFree(p);
      p = nullptr;
    }
  if (h->adj_galpha) cudaFree(h->adj_galpha);
  h->adj_galpha = nullptr;
  if (h->adj_gpart) cudaFree(h->adj_gpart);
  h->adj_gpart = nullptr;
  h->adj_gpart_n = 0;
  h->adj_T = h->adj_k = 0;
  return FLB_OK;
}

static int adjoint_supported(flb_lattice* h) {
  if (h->blocks.size() != 1 || h->mode >= 0)
    return fail(FLB_ERR_UNSUPPORTED, "the adjoint runs on single-block handles");
  if (h->desc.storage == FLB_STORAGE_FP16S)
    return fail(FLB_ERR_UNSUPPORTED, "the adjoint is built for FP32, FP32S and FP64 storage");
  if (h->desc.model != FLB_MODEL_BGK && h->desc.model != FLB_MODEL_BRINKMAN &&
      h->desc.model != FLB_MODEL_MRT)
    return fail(FLB_ERR_UNSUPPORTED, "the adjoint covers BGK, BRINKMAN and MRT bulk models");
  for (int t = 0; t < h->desc.ntasks; ++t)
    if (h->desc.task_ops[t] == FLB_OP_FIELD_BGK)
      return fail(FLB_ERR_UNSUPPORTED, "the adjoint does not cover FIELD_BGK cells");
  return FLB_OK;
}

int flb_adjoint_forward(flb_lattice* h, int nsteps, int every, double* J, void* stream) {
  if (!h) return fail(FLB_ERR_INVALID, "null handle");
  FLB_TRY(adjoint_supported(h));
  if (nsteps < 1 || every < 1) return fail(FLB_ERR_INVALID, "nsteps and checkpoint_every >= 1");
  cudaStream_t st = as_stream(stream);
  const size_t bytes = size_t(Q) * size_t(h->dstride) * h->elem_bytes;
  const int nck = (nsteps + every - 1) / every;
  // a previous pair of the same shape leaves its buffers for this one (no
  // allocation when gradients are evaluated repeatedly); any other shape
  // starts afresh
  if ((int)h->adj_ckpt.size() != nck || (int)h->adj_seg.size() != every - 1)
    flb_adjoint_release(h);
  for (int c = int(h->adj_ckpt.size()); c < nck; ++c) {
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
      flb_adjoint_release(h);
      return fail(FLB_ERR_OOM, "checkpoint %d of %d (%zu bytes): %s", c, nck, bytes,
                  cudaGetErrorString(e));
    }
    h->adj_ckpt.push_back(p);
  }
  h->adj_T = nsteps;
  h->adj_k = every;
  // the backward sweep's buffers, allocated here so that it allocates nothing:
  // lambda (two arrays), dJ/dalpha and the every - 1 recompute slots
  for (auto& p : h->adj_lam)
    if (!p) FLB_CUDA(cudaMalloc(&p, bytes));
  if (!h->adj_galpha)
    FLB_CUDA(cudaMalloc((void**)&h->adj_galpha, size_t(h->dstride) * sizeof(double)));
  while ((int)h->adj_seg.size() < every - 1) {
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
      flb_adjoint_release(h);
      return fail(FLB_ERR_OOM, "recompute slot (%zu bytes): %s", bytes, cudaGetErrorString(e));
    }
    h->adj_seg.push_back(p);
  }
  for (int t = 0; t < nsteps; ++t) {
    if (t % every == 0)
      FLB_CUDA(cudaMemcpyAsync(h->adj_ckpt[t / every], h->pops[h->cur], bytes,
                               cudaMemcpyDeviceToDevice, st));
    FLB_TRY(step_any(h, 1, st));
  }
  if (J) FLB_TRY(flb_objective_u2(h, J, stream));
  return FLB_OK;
}

}  // extern "C"

template <typename S, typename R>
static int adjoint_backward_t(flb_lattice* h, double* dJ_dalpha, double* dJ_dtau,
                              double* dJ_dulid, cudaStream_t st) {
  constexpr int V = std::is_same<R, double>::value ? 1 : 2;
  constexpr bool DEV = std::is_same<S, dev32>::value;  // forward states are FP32S deviations
  const HostBlock& b = h->blocks[0];
  const size_t ds = size_t(h->dstride);
  const size_t qbytes = size_t(Q) * ds * h->elem_bytes;
  const size_t lbytes = size_t(Q) * ds * sizeof(R);
  for (auto& p : h->adj_lam)
    if (!p) FLB_CUDA(cudaMalloc(&p, lbytes));
  if (!h->adj_galpha) FLB_CUDA(cudaMalloc((void**)&h->adj_galpha, ds * sizeof(double)));
  FLB_CUDA(cudaMemsetAsync(h->adj_galpha, 0, ds * sizeof(double), st));
  const int k = h->adj_k;
  while ((int)h->adj_seg.size() < k - 1) {
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, qbytes);
    if (e != cudaSuccess)
      return fail(FLB_ERR_OOM, "recompute slot (%zu bytes): %s", qbytes, cudaGetErrorString(e));
    h->adj_seg.push_back(p);
  }
  // seed lambda_T = dJ/dR_T and the direct dJ/dalpha term (the J partials are unused)
  k_objective<S, R><<<grid_1d(b.padded()), 256, 0, st>>>(
      b.L, geom_of(b), static_cast<const S*>(h->pops[h->cur]), h->sp,
      static_cast<R*>(h->adj_lam[0]), h->alpha ? h->adj_galpha : nullptr, h->red, true);
  FLB_CUDA(cudaGetLastError());
  int cur = 0;
  const long long chunks = (long long)(b.L.pitch / V) * b.L.ny * b.L.nz;
  const dim3 block(32 * h->tile_y);
  const dim3 grid(unsigned((chunks + block.x - 1) / block.x));
  const size_t npart = 2 * size_t(grid.x);
  if (h->adj_gpart_n < npart) {
    if (h->adj_gpart) cudaFree(h->adj_gpart);
    h->adj_gpart = nullptr;
    h->adj_gpart_n = 0;
    FLB_CUDA(cudaMalloc((void**)&h->adj_gpart, npart * sizeof(double)));
    h->adj_gpart_n = npart;
  }
  FLB_CUDA(cudaMemsetAsync(h->adj_gpart, 0, npart * sizeof(double), st));
  AdjParams a{};
  a.galpha = h->adj_galpha;
  a.gpart = h->adj_gpart;
  const int T = h->adj_T;
  const int nseg = (T + k - 1) / k;
  for (int sgi = nseg - 1; sgi >= 0; --sgi) {
    const int t0 = sgi * k, t1 = std::min(T, t0 + k);
    // states Q_t0 .. Q_{t1-1}: slot 0 is the checkpoint, the rest recomputed
    std::vector<const void*> q(t1 - t0);
    q[0] = h->adj_ckpt[sgi];
    for (int t = t0 + 1; t < t1; ++t) {
      FLB_TRY(step_between(h, q[t - 1 - t0], h->adj_seg[t - 1 - t0], st));
      q[t - t0] = h->adj_seg[t - 1 - t0];
    }
    for (int t = t1 - 1; t >= t0; --t) {
      a.lam_in = h->adj_lam[cur];
      a.lam_out = h->adj_lam[cur ^ 1];
      a.q = q[t - t0];
      if (h->desc.model == FLB_MODEL_MRT)
        k_adjoint_step<R, V, MODEL_MRT, DEV><<<grid, block, 0, st>>>(h->sp, a);
      else
        k_adjoint_step<R, V, MODEL_BGK, DEV><<<grid, block, 0, st>>>(h->sp, a);
      cur ^= 1;
    }
    FLB_CUDA(cudaGetLastError());
  }
  std::vector<double> part(npart);
  FLB_CUDA(cudaMemcpyAsync(part.data(), h->adj_gpart, npart * sizeof(double),
                           cudaMemcpyDeviceToHost, st));
  if (dJ_dalpha) {
    const LayoutParams& L = b.L;
    FLB_CUDA(cudaMemcpy2DAsync(dJ_dalpha, L.nx * sizeof(double), h->adj_galpha,
                               L.pitch * sizeof(double), L.nx * sizeof(double),
                               size_t(L.ny) * L.nz, cudaMemcpyDeviceToHost, st));
  }
  FLB_CUDA(cudaStreamSynchronize(st));
  double sc[2] = {0, 0};
  for (size_t b2 = 0; b2 < npart; b2 += 2) {
    sc[0] += part[b2];
    sc[1] += part[b2 + 1];
  }
  if (dJ_dtau) *dJ_dtau = sc[0];
  if (dJ_dulid) *dJ_dulid = sc[1];
  return FLB_OK;
}

extern "C" {

int flb_adjoint_backward(flb_lattice* h, double* dJ_dalpha, double* dJ_dtau, double* dJ_dulid,
                         void* stream) {
  if (!h) return fail(FLB_ERR_INVALID, "null handle");
  FLB_TRY(adjoint_supported(h));
  if (h->adj_T < 1 || h->adj_ckpt.empty())
    return fail(FLB_ERR_STATE, "flb_adjoint_backward needs a preceding flb_adjoint_forward");
  if (dJ_dalpha && !h->alpha)
    return fail(FLB_ERR_STATE, "dJ/dalpha needs the BRINKMAN model (ALPHA field)");
  cudaStream_t st = as_stream(stream);
  if (h->desc.storage == FLB_STORAGE_FP64)
    return adjoint_backward_t<double, double>(h, dJ_dalpha, dJ_dtau, dJ_dulid, st);
  if (h->desc.storage == FLB_STORAGE_FP32S)
    return adjoint_backward_t<dev32, float>(h, dJ_dalpha, dJ_dtau, dJ_dulid, st);
  return adjoint_backward_t<float, float>(h, dJ_dalpha, dJ_dtau, dJ_dulid, st);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// VTK DataArray bodies of device fields (flb_vtk.h)

template <typename R, typename O>
static int vtk_launch(const VtkArgs& a, unsigned* d_out, cudaStream_t st) {
  const long long groups = (a.nbytes + 2) / 3;
  long long blocks = (groups + 255) / 256;
  if (blocks < 1) blocks = 1;
  if (blocks > 148LL * 64) blocks = 148LL * 64;
  k_vtk_base64<R, O><<<unsigned(blocks), 256, 0, st>>>(a, d_out);
  FLB_CUDA(cudaGetLastError());
  return FLB_OK;
}

extern "C" {

int flb_vtk_field_base64(flb_lattice* h, int block, int field, int overlap, int out_dtype,
                         int map, double scale, double offset, char* out, size_t cap,
                         size_t* len, void* stream) {
  if (!h || !len) return fail(FLB_ERR_INVALID, "flb_vtk_field_base64: null argument");
  if (block < 0 || block >= int(h->blocks.size()))
    return fail(FLB_ERR_INVALID, "flb_vtk_field_base64: block %d of %d", block,
                int(h->blocks.size()));
  const HostBlock& b = h->blocks[block];
  const LayoutParams& L = b.L;
  if (overlap < 0 || 2 * overlap >= L.nx || 2 * overlap >= L.ny || 2 * overlap >= L.nz)
    return fail(FLB_ERR_INVALID, "flb_vtk_field_base64: overlap %d too large", overlap);
  const bool dbl = h->desc.storage == FLB_STORAGE_FP64;
  const size_t rsize = dbl ? 8 : 4;
  VtkArgs a{};
  a.comp_stride = h->dstride;
  a.pitch = L.pitch;
  a.plane = L.plane;
  a.sx = L.nx - 2 * overlap;
  a.sy = L.ny - 2 * overlap;
  a.sz = L.nz - 2 * overlap;
  a.ox = a.oy = a.oz = overlap;
  a.ncomp = 1;
  a.map = map ? 1 : 0;
  a.scale = scale;
  a.offset = offset;
  size_t osize = 1;
  if (field == FLB_VTK_FLAG) {
    a.src = h->flags + b.base;
    osize = 1;
  } else {
    if (out_dtype != FLB_DTYPE_F32 && out_dtype != FLB_DTYPE_F64)
      return fail(FLB_ERR_INVALID, "flb_vtk_field_base64: out_dtype %d", out_dtype);
    osize = out_dtype == FLB_DTYPE_F64 ? 8 : 4;
    const char* base = nullptr;
    if (field == FLB_FIELD_RHO) base = static_cast<const char*>(h->rho);
    else if (field == FLB_FIELD_VELOCITY) base = static_cast<const char*>(h->vel), a.ncomp = 3;
    else if (field == FLB_FIELD_ALPHA) base = static_cast<const char*>(h->alpha);
    else return fail(FLB_ERR_INVALID, "flb_vtk_field_base64: unknown field %d", field);
    if (!base) return fail(FLB_ERR_STATE, "flb_vtk_field_base64: field %d not allocated", field);
    a.src = base + size_t(b.base) * rsize;
  }
  const long long nelem = (long long)a.sx * a.sy * a.sz * a.ncomp;
  a.nbytes = nelem * (long long)osize;
  const size_t nchar = 8 + 4 * size_t((a.nbytes + 2) / 3);
  *len = nchar;
  if (!out) return FLB_OK;
  if (cap < nchar)
    return fail(FLB_ERR_INVALID, "flb_vtk_field_base64: buffer of %zu characters, need %zu", cap,
                nchar);
  cudaStream_t st = as_stream(stream);
  unsigned* d_out = nullptr;
  FLB_CUDA(cudaMalloc((void**)&d_out, (nchar + 3) & ~size_t(3)));
  int rc = FLB_OK;
  if (field == FLB_VTK_FLAG) rc = vtk_launch<uint8_t, uint8_t>(a, d_out, st);
  else if (dbl && osize == 8) rc = vtk_launch<double, double>(a, d_out, st);
  else if (dbl) rc = vtk_launch<double, float>(a, d_out, st);
  else if (osize == 8) rc = vtk_launch<float, double>(a, d_out, st);
  else rc = vtk_launch<float, float>(a, d_out, st);
  cudaError_t e = cudaSuccess;
  if (rc == FLB_OK) e = cudaMemcpyAsync(out, d_out, nchar, cudaMemcpyDeviceToHost, st);
  if (rc == FLB_OK && e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(d_out);
  if (rc) return rc;
  if (e != cudaSuccess)
    return fail(FLB_ERR_CUDA, "flb_vtk_field_base64: %s", cudaGetErrorString(e));
  return FLB_OK;
}

}  // extern "C"
