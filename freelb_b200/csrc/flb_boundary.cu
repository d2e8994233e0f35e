// flb_boundary.cu -- post-stream halfway bounce-back managers and the fixed
// periodic boundary manager on the device.
//
// The reference's BBLikeFixedBlockBdManager (src/boundary/boundary.h:86-140)
// visits, after Stream(), every inner cell whose flag matches `cell_flag` and,
// for each direction k whose neighbour x + c_k carries `void_flag`
// (BlockFixedBoundary::addtoBd, basic_boundary.h:196-211), sets the outflow
// j = opp(k) from prev = getPrevious(k), the population k the cell held
// before streaming, and the cell's RHO and VELOCITY fields
// (bounce_back_boundary.h:167-256):
//   normal         f_j = prev
//   movingwall     f_j = prev + 2 InvCs2 w_j rho (u . c_j)
//   anti_simple    f_j = 2 rho w_j - prev
//   anti_O1        f_j = 2 w_j rho (1 + InvCs2 u . c_j) - prev
//   anti_O2        f_j = 2 feq2_j(rho, u) - prev
//   anti_pressure  f_j = 2 rho w_j (1 + (uw . c_j)^2 InvCs4 / 2
//                                   - |uw|^2 InvCs2 / 2) - prev,
//                  uw = u + (u - u(x + c_k)) / 2.
//
// In the device convention (the lattice stores P with R = stream(P)) prev at x
// is P_k(x) and R_j(x) lives in P_j(x + c_k), so each link reads one
// population of a boundary cell and writes one population slot of its void
// neighbour: no link reads a slot another link writes.  Links are found once,
// on the host, from the lattice's flags; the manager is built on the public C
// ABI (flb_device_pointers, flb_get_layout).
#include <cuda_runtime.h>

#include <cstdio>
#include <new>
#include <vector>

#include "../../include/flb_boundary.h"
#include "flb_pull.cuh"

using namespace flb;

namespace flb {
int report_error(int code, const char* msg);       // flb_api.cu
int lattice_storage(const flb_lattice* h);         // flb_api.cu
}

struct flb_bb {
  int kind = FLB_BB_NORMAL;
  int storage = FLB_STORAGE_FP32;
  double rho0 = 1.0;
  flb_layout layout{};
  long long ncells = 0;
  long long nlinks = 0;
  long long* d_cell = nullptr;  // padded cell offset of each link's boundary cell
  int* d_dir = nullptr;         // direction k pointing at the void neighbour
};

namespace {

struct BBArgs {
  const long long* cell;
  const int* dir;
  long long n;
  Geom g;
  long long dstride;
  const void* rho;  // RHO field (arithmetic type), all kinds but normal
  const void* vel;  // VELOCITY field, 3 SoA planes of dstride
  float shift[Q];
  float scale, inv_scale;
};

template <typename R>
__device__ __forceinline__ R dot_c(R ux, R uy, R uz, int j) {
  return ux * R(cx(j)) + uy * R(cy(j)) + uz * R(cz(j));
}

template <typename S, typename R, int KIND>
__global__ void k_bb(BBArgs a, S* pops) {
  const R* rho = static_cast<const R*>(a.rho);
  const R* vel = static_cast<const R*>(a.vel);
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < a.n;
       r += (long long)gridDim.x * blockDim.x) {
    const long long c = a.cell[r];
    const int k = a.dir[r];
    const int j = opp(k);
    const long long zz = c / a.g.plane;
    const long long rem = c - zz * a.g.plane;
    const int y = int(rem / a.g.pitch), x = int(rem - (long long)y * a.g.pitch);
    const long long dst = wrap_off(a.g, x, y, int(zz), cx(k), cy(k), cz(k));
    const R prev = Storage<S, R>::load(pops + k * a.dstride + c, a.shift[k], a.inv_scale);
    const R w = weight<R>(j);
    R v = prev;
    if constexpr (KIND != FLB_BB_NORMAL) {
      const R rc = rho[c];
      const R ux = vel[c], uy = vel[c + a.dstride], uz = vel[c + 2 * a.dstride];
      if constexpr (KIND == FLB_BB_MOVINGWALL) {
        v = prev + R(2) * R(3) * w * rc * dot_c(ux, uy, uz, j);
      } else if constexpr (KIND == FLB_BB_ANTI_SIMPLE) {
        v = R(2) * rc * w - prev;
      } else if constexpr (KIND == FLB_BB_ANTI_O1) {
        v = R(2) * (w * rc * (R(1) + R(3) * dot_c(ux, uy, uz, j))) - prev;
      } else if constexpr (KIND == FLB_BB_ANTI_O2) {
        const R uc = dot_c(ux, uy, uz, j);
        const R u2 = ux * ux + uy * uy + uz * uz;
        v = R(2) * (w * rc * (R(1) + R(3) * uc + uc * uc * R(0.5) * R(9) - R(3) * u2 * R(0.5))) -
            prev;
      } else {  // FLB_BB_ANTI_PRESSURE: velocity of the neighbour x + c_k
        const R wx = ux + R(0.5) * (ux - vel[dst]);
        const R wy = uy + R(0.5) * (uy - vel[dst + a.dstride]);
        const R wz = uz + R(0.5) * (uz - vel[dst + 2 * a.dstride]);
        const R uc = dot_c(wx, wy, wz, j);
        const R u2 = wx * wx + wy * wy + wz * wz;
        v = R(2) * rc * w * (R(1) + uc * uc * R(0.5) * R(9) - u2 * R(0.5) * R(3)) - prev;
      }
    }
    Storage<S, R>::store(pops + j * a.dstride + dst, v, a.shift[j], a.scale);
  }
}

template <typename S, typename R>
int launch(flb_bb* bb, flb_lattice* lat, cudaStream_t st) {
  void *pops = nullptr, *rho = nullptr, *vel = nullptr;
  int rc = flb_device_pointers(lat, &pops, nullptr, &rho, &vel);
  if (rc) return rc;
  BBArgs a{};
  a.cell = bb->d_cell;
  a.dir = bb->d_dir;
  a.n = bb->nlinks;
  const flb_layout& L = bb->layout;
  a.g = Geom{L.nx, L.ny, L.nz, L.pitch_x, (long long)L.plane, 0};
  a.dstride = (long long)L.dir_stride;
  a.rho = rho;
  a.vel = vel;
  for (int i = 0; i < Q; ++i) {
    const double w = i == 0 ? 1.0 / 3.0 : (i < 7 ? 1.0 / 18.0 : 1.0 / 36.0);
    a.shift[i] = float(bb->rho0 * w);
  }
  a.scale = 1024.0f;
  a.inv_scale = 1.0f / 1024.0f;
  long long blocks = (a.n + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  if (blocks < 1) blocks = 1;
  S* p = static_cast<S*>(pops);
  switch (bb->kind) {
    case FLB_BB_NORMAL: k_bb<S, R, FLB_BB_NORMAL><<<unsigned(blocks), 256, 0, st>>>(a, p); break;
    case FLB_BB_MOVINGWALL:
      k_bb<S, R, FLB_BB_MOVINGWALL><<<unsigned(blocks), 256, 0, st>>>(a, p);
      break;
    case FLB_BB_ANTI_SIMPLE:
      k_bb<S, R, FLB_BB_ANTI_SIMPLE><<<unsigned(blocks), 256, 0, st>>>(a, p);
      break;
    case FLB_BB_ANTI_O1: k_bb<S, R, FLB_BB_ANTI_O1><<<unsigned(blocks), 256, 0, st>>>(a, p); break;
    case FLB_BB_ANTI_O2: k_bb<S, R, FLB_BB_ANTI_O2><<<unsigned(blocks), 256, 0, st>>>(a, p); break;
    default: k_bb<S, R, FLB_BB_ANTI_PRESSURE><<<unsigned(blocks), 256, 0, st>>>(a, p); break;
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    char m[160];
    std::snprintf(m, sizeof m, "flb_bb_apply: %s", cudaGetErrorString(e));
    return report_error(FLB_ERR_CUDA, m);
  }
  return FLB_OK;
}

// ---------------------------------------------------------------------------
// Fixed periodic boundary: population copies between two boxes.

// getCommPopDir (parallel/communicator.h:74-150): the directions entering a
// cell across each face named in `dir`, sorted.
std::vector<int> comm_pop_dirs(int dir) {
  std::vector<int> out;
  for (int i = 0; i < Q; ++i) {
    const bool xs = (dir & FLB_NBR_XN) ? cx(i) > 0 : ((dir & FLB_NBR_XP) ? cx(i) < 0 : false);
    const bool ys = (dir & FLB_NBR_YN) ? cy(i) > 0 : ((dir & FLB_NBR_YP) ? cy(i) < 0 : false);
    const bool zs = (dir & FLB_NBR_ZN) ? cz(i) > 0 : ((dir & FLB_NBR_ZP) ? cz(i) < 0 : false);
    if (xs || ys || zs) out.push_back(i);
  }
  return out;
}

// Cells of an inclusive box clamped to the mesh, z, y, x order (getCellIdx);
// false when the box misses the interior [1, n-2] of some axis.
bool box_cells(const flb_layout& L, const int* b, std::vector<long long>& cells) {
  const int n[3] = {L.nx, L.ny, L.nz};
  int lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    if (b[2 * a] > n[a] - 2 || b[2 * a + 1] < 1 || b[2 * a] > b[2 * a + 1]) return false;
    lo[a] = b[2 * a] < 0 ? 0 : b[2 * a];
    hi[a] = b[2 * a + 1] > n[a] - 1 ? n[a] - 1 : b[2 * a + 1];
  }
  for (int z = lo[2]; z <= hi[2]; ++z)
    for (int y = lo[1]; y <= hi[1]; ++y)
      for (int x = lo[0]; x <= hi[0]; ++x)
        cells.push_back(x + (long long)y * L.pitch_x + (long long)z * (long long)L.plane);
  return true;
}

template <typename E>
__global__ void k_gather(const long long* __restrict__ src, long long n, const E* pops, E* stage) {
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n;
       r += (long long)gridDim.x * blockDim.x)
    stage[r] = pops[src[r]];
}
template <typename E>
__global__ void k_scatter(const long long* __restrict__ dst, long long n, const E* stage, E* pops) {
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n;
       r += (long long)gridDim.x * blockDim.x)
    pops[dst[r]] = stage[r];
}

template <typename E>
int periodic_launch(flb_periodic* per, void* pops, cudaStream_t st);

}  // namespace

struct flb_periodic {
  flb_layout layout{};
  long long npairs = 0;
  long long ncopies = 0;
  long long* d_src = nullptr;  // element offset of each copy's source slot
  long long* d_dst = nullptr;  // and of its destination slot
  void* d_stage = nullptr;     // ncopies elements
};

namespace {
template <typename E>
int periodic_launch(flb_periodic* per, void* pops, cudaStream_t st) {
  const long long n = per->ncopies;
  const unsigned grid = unsigned(n / 256 + 1 < 4096 ? n / 256 + 1 : 4096);
  k_gather<E><<<grid, 256, 0, st>>>(per->d_src, n, static_cast<const E*>(pops),
                                    static_cast<E*>(per->d_stage));
  k_scatter<E><<<grid, 256, 0, st>>>(per->d_dst, n, static_cast<const E*>(per->d_stage),
                                     static_cast<E*>(pops));
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    char m[160];
    std::snprintf(m, sizeof m, "flb_periodic_apply: %s", cudaGetErrorString(e));
    return report_error(FLB_ERR_CUDA, m);
  }
  return FLB_OK;
}
}  // namespace

extern "C" {

int flb_periodic_create(flb_lattice* lat, const int box0[6], int dir0, const int box1[6],
                        int dir1, uint8_t cell_flag, flb_periodic** out) {
  if (!lat || !box0 || !box1 || !out)
    return report_error(FLB_ERR_INVALID, "flb_periodic_create: null argument");
  *out = nullptr;
  if (dir0 < 0 || dir0 > 63 || dir1 < 0 || dir1 > 63)
    return report_error(FLB_ERR_INVALID, "flb_periodic_create: direction outside the FLB_NBR_* bits");
  int nblocks = 0;
  int rc = flb_block_count(lat, &nblocks);
  if (rc) return rc;
  if (nblocks != 1)
    return report_error(FLB_ERR_UNSUPPORTED, "flb_periodic_create: single-block lattices only");
  flb_layout L{};
  if ((rc = flb_get_layout(lat, &L))) return rc;
  const long long N = (long long)L.nx * L.ny * L.nz;
  std::vector<uint8_t> flags(static_cast<size_t>(N));
  if ((rc = flb_download_flags(lat, flags.data(), nullptr))) return rc;
  bool any = false;  // NonLocalBoundary::Setup (basic_boundary.h:395-420): the block's BdCells
  for (long long id = 0; id < N && !any; ++id) any = (flags[size_t(id)] & cell_flag) != 0;
  std::vector<long long> c0, c1, src, dst;
  if (any && box_cells(L, box0, c0) && box_cells(L, box1, c1)) {
    if (c0.size() != c1.size())
      return report_error(FLB_ERR_INVALID, "flb_periodic_create: the boxes hold different cell counts");
    const long long ds = (long long)L.dir_stride;
    for (int k : comm_pop_dirs(dir0))
      for (size_t p = 0; p < c0.size(); ++p) {
        src.push_back(k * ds + c1[p]);
        dst.push_back(k * ds + c0[p]);
      }
    for (int k : comm_pop_dirs(dir1))
      for (size_t p = 0; p < c0.size(); ++p) {
        src.push_back(k * ds + c0[p]);
        dst.push_back(k * ds + c1[p]);
      }
  } else {
    c0.clear();
  }
  flb_periodic* per = new (std::nothrow) flb_periodic();
  if (!per) return report_error(FLB_ERR_OOM, "flb_periodic_create: host allocation");
  per->layout = L;
  per->npairs = (long long)c0.size();
  per->ncopies = (long long)src.size();
  if (per->ncopies > 0) {
    cudaError_t e = cudaMalloc((void**)&per->d_src, src.size() * sizeof(long long));
    if (e == cudaSuccess) e = cudaMalloc((void**)&per->d_dst, dst.size() * sizeof(long long));
    if (e == cudaSuccess) e = cudaMalloc(&per->d_stage, src.size() * size_t(L.elem_bytes));
    if (e == cudaSuccess)
      e = cudaMemcpy(per->d_src, src.data(), src.size() * sizeof(long long), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemcpy(per->d_dst, dst.data(), dst.size() * sizeof(long long), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      flb_periodic_destroy(per);
      char m[160];
      std::snprintf(m, sizeof m, "flb_periodic_create: %s", cudaGetErrorString(e));
      return report_error(FLB_ERR_OOM, m);
    }
  }
  *out = per;
  return FLB_OK;
}

int flb_periodic_count(const flb_periodic* per, long long* pairs, long long* copies) {
  if (!per) return report_error(FLB_ERR_INVALID, "flb_periodic_count: null handle");
  if (pairs) *pairs = per->npairs;
  if (copies) *copies = per->ncopies;
  return FLB_OK;
}

int flb_periodic_apply(flb_periodic* per, flb_lattice* lat, void* stream) {
  if (!per || !lat) return report_error(FLB_ERR_INVALID, "flb_periodic_apply: null argument");
  if (per->ncopies == 0) return FLB_OK;
  flb_layout L{};
  int rc = flb_get_layout(lat, &L);
  if (rc) return rc;
  if (L.nx != per->layout.nx || L.ny != per->layout.ny || L.nz != per->layout.nz ||
      L.pitch_x != per->layout.pitch_x || L.elem_bytes != per->layout.elem_bytes ||
      L.dir_stride != per->layout.dir_stride)
    return report_error(FLB_ERR_INVALID, "flb_periodic_apply: lattice differs from the one at creation");
  void* pops = nullptr;
  if ((rc = flb_device_pointers(lat, &pops, nullptr, nullptr, nullptr))) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (L.elem_bytes == 2) return periodic_launch<unsigned short>(per, pops, st);
  if (L.elem_bytes == 8) return periodic_launch<unsigned long long>(per, pops, st);
  return periodic_launch<unsigned>(per, pops, st);
}

int flb_periodic_destroy(flb_periodic* per) {
  if (!per) return FLB_OK;
  if (per->d_src) cudaFree(per->d_src);
  if (per->d_dst) cudaFree(per->d_dst);
  if (per->d_stage) cudaFree(per->d_stage);
  delete per;
  return FLB_OK;
}

int flb_bb_create(flb_lattice* lat, uint8_t cell_flag, uint8_t void_flag, int kind, double rho0,
                  flb_bb** out) {
  if (!lat || !out) return report_error(FLB_ERR_INVALID, "flb_bb_create: null argument");
  *out = nullptr;
  if (kind < FLB_BB_NORMAL || kind > FLB_BB_ANTI_PRESSURE)
    return report_error(FLB_ERR_INVALID, "flb_bb_create: unknown kind");
  int nblocks = 0;
  int rc = flb_block_count(lat, &nblocks);
  if (rc) return rc;
  if (nblocks != 1)
    return report_error(FLB_ERR_UNSUPPORTED, "flb_bb_create: single-block lattices only");
  flb_layout L{};
  if ((rc = flb_get_layout(lat, &L))) return rc;
  const long long N = (long long)L.nx * L.ny * L.nz;
  std::vector<uint8_t> flags(static_cast<size_t>(N));
  if ((rc = flb_download_flags(lat, flags.data(), nullptr))) return rc;
  std::vector<long long> cell;
  std::vector<int> dir;
  long long ncells = 0;
  // BlockFixedBoundary::Setup (basic_boundary.h:213-262): inner cells only
  for (int z = 1; z < L.nz - 1; ++z)
    for (int y = 1; y < L.ny - 1; ++y)
      for (int x = 1; x < L.nx - 1; ++x) {
        const long long id = x + (long long)L.nx * (y + (long long)L.ny * z);
        if (!(flags[size_t(id)] & cell_flag)) continue;
        bool any = false;
        for (int k = 1; k < Q; ++k) {
          const long long nb = (x + cx(k)) + (long long)L.nx * ((y + cy(k)) + (long long)L.ny * (z + cz(k)));
          if (flags[size_t(nb)] & void_flag) {
            cell.push_back(x + (long long)y * L.pitch_x + (long long)z * (long long)L.plane);
            dir.push_back(k);
            any = true;
          }
        }
        ncells += any ? 1 : 0;
      }
  flb_bb* bb = new (std::nothrow) flb_bb();
  if (!bb) return report_error(FLB_ERR_OOM, "flb_bb_create: host allocation");
  bb->kind = kind;
  bb->rho0 = rho0;
  bb->layout = L;
  bb->storage = flb::lattice_storage(lat);
  bb->ncells = ncells;
  bb->nlinks = (long long)cell.size();
  if (bb->nlinks > 0) {
    cudaError_t e = cudaMalloc((void**)&bb->d_cell, cell.size() * sizeof(long long));
    if (e == cudaSuccess) e = cudaMalloc((void**)&bb->d_dir, dir.size() * sizeof(int));
    if (e == cudaSuccess)
      e = cudaMemcpy(bb->d_cell, cell.data(), cell.size() * sizeof(long long), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemcpy(bb->d_dir, dir.data(), dir.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      flb_bb_destroy(bb);
      char m[160];
      std::snprintf(m, sizeof m, "flb_bb_create: %s", cudaGetErrorString(e));
      return report_error(FLB_ERR_OOM, m);
    }
  }
  *out = bb;
  return FLB_OK;
}

int flb_bb_count(const flb_bb* bb, long long* ncells, long long* nlinks) {
  if (!bb) return report_error(FLB_ERR_INVALID, "flb_bb_count: null handle");
  if (ncells) *ncells = bb->ncells;
  if (nlinks) *nlinks = bb->nlinks;
  return FLB_OK;
}

int flb_bb_apply(flb_bb* bb, flb_lattice* lat, void* stream) {
  if (!bb || !lat) return report_error(FLB_ERR_INVALID, "flb_bb_apply: null argument");
  if (bb->nlinks == 0) return FLB_OK;
  flb_layout L{};
  int rc = flb_get_layout(lat, &L);
  if (rc) return rc;
  if (L.nx != bb->layout.nx || L.ny != bb->layout.ny || L.nz != bb->layout.nz ||
      L.pitch_x != bb->layout.pitch_x || L.elem_bytes != bb->layout.elem_bytes ||
      flb::lattice_storage(lat) != bb->storage)
    return report_error(FLB_ERR_INVALID, "flb_bb_apply: lattice differs from the one at creation");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (bb->storage == FLB_STORAGE_FP64) return launch<double, double>(bb, lat, st);
  if (bb->storage == FLB_STORAGE_FP16S) return launch<__half, float>(bb, lat, st);
  if (bb->storage == FLB_STORAGE_FP32S) return launch<dev32, float>(bb, lat, st);
  return launch<float, float>(bb, lat, st);
}

int flb_bb_destroy(flb_bb* bb) {
  if (!bb) return FLB_OK;
  if (bb->d_cell) cudaFree(bb->d_cell);
  if (bb->d_dir) cudaFree(bb->d_dir);
  delete bb;
  return FLB_OK;
}

}  // extern "C"
