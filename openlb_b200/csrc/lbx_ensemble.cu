// Ensemble engine: many independent box cavities, one persistent kernel.
//
// Each admitted request owns a region of one device slab: Q population columns of period P
// (its padded cell count rounded up to 64; the periodic-shift layout of lbx_kernels.cuh, the
// ghost layer being the walls) and a velocity snapshot for the convergence residual.  A tile
// is up to `threads` consecutive core cells of one lattice; the persistent kernel runs
// `steps` steps, in each of which its blocks stride over the tile list, and two grid-wide
// barriers per step separate the steps from the per-lattice bookkeeping done by block 0
// (column shifts of the next step, step count, residual, state).  Lattices stop on their own
// residual and are retired by the host between runs while the others keep going, so requests
// of different sizes and ages are stepped together.
//
// Walls: halfway bounce-back on every face, applied when a boundary cell loads its
// populations: the population arriving from a wall direction k is the one the cell sent the
// step before, f_opp(k)(x_b) = f_k(x_b + c_k) - 2 t_k (c_k . u_w) / c_s^2 (the post-stream
// BouzidiVelocityPostProcessor with q = 1/2, boundary/setBouzidiBoundary.h:129-162, evaluated
// one step later: the collision sees identical values, only the stored between-step state of
// the boundary cells differs, and lbx_ensemble_moments applies the same rule).
//
// Memory ordering inside the persistent kernel: populations written by one block are read by
// another block in the next step (a streamed population crosses tile boundaries), so every
// load of shared state bypasses L1 (ld.global.cg) and the barrier fences.  The barrier waits
// are bounded: after ~4 s a block records an error and the kernel returns.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/lbx.h"
#include "lbx_kernels.cuh"

namespace lbx {
int set_error(int code, const std::string& msg);
}

namespace {

using namespace lbx;

constexpr int kMaxQ = 27;

struct EnsLattice {
  void* pop;        // column 0; column i starts at element i * P
  float* snap;      // velocity snapshot [3][ncore]
  uint32_t P;
  int32_t nx, ny, nz;
  int32_t sx, sy;   // padded strides
  int32_t ncore;
  int32_t dynamics;
  int32_t state;
  int32_t pad0;
  int64_t steps, maxSteps;
  double tol, residual;
  float omega, magic;
  float delta[kMaxQ];        // wall term of the links leaving through the moving lid
  uint32_t shift[2][kMaxQ];  // column shifts, double-buffered by global step parity
};

struct EnsArgs {
  EnsLattice* lat;
  const int2* tiles;       // {slot, first core cell}
  const int* nTiles;
  const int2* range;       // per slot {first tile, tile count}
  double* tilePart;        // {sum |du|^2, sum |u|^2} per tile at check steps
  unsigned* barrier;       // {arrived, generation}
  int* err;
  long long* globalStep;
  int maxLattices;
  int steps;
  int check;
};

template <typename S> struct CgLoad;
template <> struct CgLoad<double> { static __device__ __forceinline__ double ld(const double* p) { return __ldcg(p); } };
template <> struct CgLoad<float> { static __device__ __forceinline__ float ld(const float* p) { return __ldcg(p); } };
template <> struct CgLoad<__half> {
  static __device__ __forceinline__ float ld(const __half* p) {
    return __half2float(__ushort_as_half(__ldcg(reinterpret_cast<const unsigned short*>(p))));
  }
};
template <> struct CgLoad<__nv_bfloat16> {
  static __device__ __forceinline__ float ld(const __nv_bfloat16* p) {
    return __bfloat162float(__ushort_as_bfloat16(__ldcg(reinterpret_cast<const unsigned short*>(p))));
  }
};

__device__ __forceinline__ uint32_t wrap32(uint32_t a, uint32_t P) { return a >= P ? a - P : a; }

// Grid-wide barrier for a co-resident grid (cooperative launch).  Returns false when another
// block gave up or this block waited longer than the bound; the kernel then returns.
__device__ bool grid_barrier(unsigned* barrier, int* err) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* gen = barrier + 1;
    const unsigned my = *gen;
    __threadfence();
    if (atomicAdd(barrier, 1u) == gridDim.x - 1) {
      atomicExch(barrier, 0u);
      __threadfence();
      atomicAdd(barrier + 1, 1u);
    } else {
      long long spins = 0;
      while (*gen == my) {
        __nanosleep(64);
        if (++spins > (1ll << 26) || *reinterpret_cast<volatile int*>(err)) {
          atomicExch(err, 1);
          break;
        }
      }
    }
    __threadfence();
    ok = *reinterpret_cast<volatile int*>(err) == 0;
  }
  __syncthreads();
  return ok != 0;
}

template <int Q, typename S>
__global__ void __launch_bounds__(256) k_ensemble(EnsArgs a) {
  using R = typename Storage<S>::R;
  using D = Desc<Q>;
  __shared__ uint32_t sShift[Q];
  __shared__ float sDelta[Q];
  __shared__ double red[2][8];
  const int tid = threadIdx.x;
  for (int step = 0; step < a.steps; ++step) {
    const long long g = *reinterpret_cast<volatile long long*>(a.globalStep);
    const int par = int(g & 1);
    const int nTiles = *a.nTiles;
    for (int tile = blockIdx.x; tile < nTiles; tile += gridDim.x) {
      const int2 t = a.tiles[tile];
      EnsLattice* L = a.lat + t.x;
      const int state = __ldcg(&L->state);
      if (state != LBX_SLOT_RUNNING) continue;  // uniform over the block
      const int64_t steps = __ldcg(reinterpret_cast<const long long*>(&L->steps));
      const bool check = ((steps + 1) % a.check) == 0;
      __syncthreads();  // the previous tile's readers of sShift/sDelta are done
      if (tid < Q) {
        sShift[tid] = __ldcg(&L->shift[par][tid]);
        sDelta[tid] = __ldcg(&L->delta[tid]);
      }
      __syncthreads();
      const uint32_t P = L->P;
      const int nx = L->nx, ny = L->ny, nz = L->nz, sx = L->sx, sy = L->sy, ncore = L->ncore;
      S* pop = static_cast<S*>(L->pop);
      double du2 = 0.0, u2 = 0.0;
      const int c = t.y + tid;
      if (c < ncore) {
        const int z = c % nz;
        const int y = (c / nz) % ny;
        const int x = c / (nz * ny);
        const uint32_t n = uint32_t((x + 1) * sx + (y + 1) * sy + z + 1);
        R f[Q];
        static_for<Q>([&](auto I) { f[I] = CgLoad<S>::ld(pop + I * int64_t(P) + wrap32(n + sShift[I], P)); });
        // halfway bounce-back on load for the links that leave the core
        if (x == 0 || x == nx - 1 || y == 0 || y == ny - 1 || z == 0 || z == nz - 1) {
          static_for<Q>([&](auto K) {
            constexpr int cx = D::C[K][0], cy = D::C[K][1], cz = D::C[K][2];
            if constexpr (cx != 0 || cy != 0 || cz != 0) {
              const int tx = x + cx, ty = y + cy, tz = z + cz;
              if (tx < 0 || tx >= nx || ty < 0 || ty >= ny || tz < 0 || tz >= nz) {
                const uint32_t nb = uint32_t(int(n) + cx * sx + cy * sy + cz);
                const R v = CgLoad<S>::ld(pop + K * int64_t(P) + wrap32(nb + sShift[K], P));
                f[D::OPP[K]] = v - (ty == ny ? R(sDelta[K]) : R(0));
              }
            }
          });
        }
        if (check) {
          R rho, u[3];
          moments<Q, R, false>(f, nullptr, rho, u);
          float* snap = L->snap;
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            const double cur = double(u[d]);
            const double dd = cur - double(__ldcg(snap + int64_t(d) * ncore + c));
            du2 += dd * dd;
            u2 += cur * cur;
            snap[int64_t(d) * ncore + c] = float(cur);
          }
        }
        CollisionParams<R> cp;
        cp.omega = R(L->omega);
        cp.magic = R(L->magic);
        cp.smagorinsky = R(0);
        cp.force[0] = cp.force[1] = cp.force[2] = R(0);
        R rho, usq;
        if (L->dynamics == LBX_TRT) collide<Q, R, DYN_TRT>(f, cp, rho, usq);
        else collide<Q, R, DYN_BGK>(f, cp, rho, usq);
        if (!(usq == usq) || usq > R(1)) du2 = __longlong_as_double(0x7ff8000000000000ll);  // NaN flags divergence
        static_for<Q>([&](auto I) { Storage<S>::store(pop + I * int64_t(P) + wrap32(n + sShift[I], P), f[I]); });
      }
      if (check) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          du2 += __shfl_xor_sync(0xffffffffu, du2, o);
          u2 += __shfl_xor_sync(0xffffffffu, u2, o);
        }
        if ((tid & 31) == 0) {
          red[0][tid >> 5] = du2;
          red[1][tid >> 5] = u2;
        }
        __syncthreads();
        if (tid == 0) {
          double s0 = 0, s1 = 0;
          for (int w = 0; w < int(blockDim.x >> 5); ++w) {
            s0 += red[0][w];
            s1 += red[1][w];
          }
          a.tilePart[2 * int64_t(tile)] = s0;
          a.tilePart[2 * int64_t(tile) + 1] = s1;
        }
      }
    }
    if (!grid_barrier(a.barrier, a.err)) return;
    if (blockIdx.x == 0) {
      for (int s = tid; s < a.maxLattices; s += blockDim.x) {
        EnsLattice* L = a.lat + s;
        if (__ldcg(&L->state) != LBX_SLOT_RUNNING) continue;
        const int64_t steps = __ldcg(reinterpret_cast<const long long*>(&L->steps));
        const bool check = ((steps + 1) % a.check) == 0;
        L->steps = steps + 1;
        const uint32_t P = L->P;
        const int sx = L->sx, sy = L->sy;
        static_for<Q>([&](auto I) {
          const int64_t off = D::C[I][0] * int64_t(sx) + D::C[I][1] * int64_t(sy) + D::C[I][2];
          int64_t ns = (int64_t(__ldcg(&L->shift[par][I])) - off) % int64_t(P);
          if (ns < 0) ns += P;
          L->shift[par ^ 1][I] = uint32_t(ns);
        });
        int state = LBX_SLOT_RUNNING;
        if (check) {
          const int2 r = a.range[s];
          double s0 = 0, s1 = 0;
          for (int k = 0; k < r.y; ++k) {
            s0 += __ldcg(a.tilePart + 2 * int64_t(r.x + k));
            s1 += __ldcg(a.tilePart + 2 * int64_t(r.x + k) + 1);
          }
          const double res = s1 > 0 ? sqrt(s0 / s1) : (s0 > 0 ? INFINITY : 0.0);
          L->residual = res;
          if (!(res == res) || !(s1 == s1) || isinf(s1)) state = LBX_SLOT_DIVERGED;
          else if (res < L->tol) state = LBX_SLOT_CONVERGED;
        }
        if (state == LBX_SLOT_RUNNING && steps + 1 >= L->maxSteps) state = LBX_SLOT_MAX_STEPS;
        if (state != LBX_SLOT_RUNNING) L->state = state;
      }
      if (tid == 0) *a.globalStep = g + 1;
    }
    if (!grid_barrier(a.barrier, a.err)) return;
  }
}

// rho and u of one lattice's core cells with the wall links applied (FP64 out).
template <int Q, typename S>
__global__ void k_ensemble_moments(const EnsLattice* __restrict__ lat, const long long* globalStep, double* rho,
                                   double* u) {
  using R = typename Storage<S>::R;
  using D = Desc<Q>;
  const EnsLattice& L = *lat;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= L.ncore) return;
  const int par = int(*globalStep & 1);
  const uint32_t P = L.P;
  const int nx = L.nx, ny = L.ny, nz = L.nz, sx = L.sx, sy = L.sy;
  const int z = c % nz, y = (c / nz) % ny, x = c / (nz * ny);
  const uint32_t n = uint32_t((x + 1) * sx + (y + 1) * sy + z + 1);
  const S* pop = static_cast<const S*>(L.pop);
  R f[Q];
  static_for<Q>([&](auto I) { f[I] = Storage<S>::load(pop + I * int64_t(P) + wrap32(n + L.shift[par][I], P)); });
  static_for<Q>([&](auto K) {
    constexpr int cx = D::C[K][0], cy = D::C[K][1], cz = D::C[K][2];
    if constexpr (cx != 0 || cy != 0 || cz != 0) {
      const int tx = x + cx, ty = y + cy, tz = z + cz;
      if (tx < 0 || tx >= nx || ty < 0 || ty >= ny || tz < 0 || tz >= nz) {
        const uint32_t nb = uint32_t(int(n) + cx * sx + cy * sy + cz);
        f[D::OPP[K]] = Storage<S>::load(pop + K * int64_t(P) + wrap32(nb + L.shift[par][K], P)) -
                       (ty == ny ? R(L.delta[K]) : R(0));
      }
    }
  });
  R r, uu[3];
  moments<Q, R, false>(f, nullptr, r, uu);
  if (rho) rho[c] = double(r);
  if (u)
    for (int d = 0; d < 3; ++d) u[int64_t(d) * L.ncore + c] = double(uu[d]);
}

size_t elem_bytes(int storage) {
  switch (storage) {
  case LBX_F64: return 8;
  case LBX_F32: return 4;
  case LBX_F16DEV: case LBX_BF16DEV: return 2;
  default: return 0;
  }
}

int64_t region_bytes(int q, int storage, const lbx_ensemble_request* r, uint32_t* period) {
  const int64_t padded = int64_t(r->core[0] + 2) * (r->core[1] + 2) * (r->core[2] + 2);
  const int64_t P = (padded + 63) / 64 * 64;
  if (period) *period = uint32_t(P);
  const int64_t ncore = int64_t(r->core[0]) * r->core[1] * r->core[2];
  const int64_t popBytes = (int64_t(q) * P * int64_t(elem_bytes(storage)) + 255) / 256 * 256;
  const int64_t snapBytes = (3 * ncore * 4 + 255) / 256 * 256;
  return popBytes + snapBytes;
}

using KernelFn = void (*)(EnsArgs);
using MomentsFn = void (*)(const EnsLattice*, const long long*, double*, double*);

template <int Q, typename S>
void pick(KernelFn& k, MomentsFn& m) {
  k = k_ensemble<Q, S>;
  m = k_ensemble_moments<Q, S>;
}

bool kernels_for(int q, int storage, KernelFn& k, MomentsFn& m) {
  switch (q * 4 + storage) {
  case 19 * 4 + LBX_F64: pick<19, double>(k, m); return true;
  case 19 * 4 + LBX_F32: pick<19, float>(k, m); return true;
  case 19 * 4 + LBX_F16DEV: pick<19, __half>(k, m); return true;
  case 19 * 4 + LBX_BF16DEV: pick<19, __nv_bfloat16>(k, m); return true;
  case 27 * 4 + LBX_F64: pick<27, double>(k, m); return true;
  case 27 * 4 + LBX_F32: pick<27, float>(k, m); return true;
  case 27 * 4 + LBX_F16DEV: pick<27, __half>(k, m); return true;
  case 27 * 4 + LBX_BF16DEV: pick<27, __nv_bfloat16>(k, m); return true;
  default: return false;
  }
}

#define ENS_TRY(expr)                                                                         \
  do {                                                                                        \
    cudaError_t e_ = (expr);                                                                  \
    if (e_ != cudaSuccess)                                                                    \
      return lbx::set_error(e_ == cudaErrorMemoryAllocation ? LBX_ERR_OUT_OF_MEMORY : LBX_ERR_CUDA, \
                            std::string(#expr) + ": " + cudaGetErrorString(e_));            \
  } while (0)

struct DeviceScope {
  int prev = -1;
  explicit DeviceScope(int d) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != d) cudaSetDevice(d);
  }
  ~DeviceScope() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

}  // namespace

struct lbx_ensemble_s {
  int q = 19, storage = LBX_F32, device = 0, maxLattices = 0;
  char* slab = nullptr;
  int64_t slabBytes = 0;
  std::map<int64_t, int64_t> freeList;  // offset -> bytes, coalesced
  std::vector<int64_t> slotOffset, slotBytes;
  std::vector<int> slotUsed;
  std::vector<int32_t> slotCells;
  EnsLattice* dLat = nullptr;
  int2* dTiles = nullptr;
  int2* dRange = nullptr;
  int* dNTiles = nullptr;
  double* dTilePart = nullptr;
  int tileCapacity = 0;
  unsigned* dBarrier = nullptr;
  int* dErr = nullptr;
  long long* dGlobalStep = nullptr;
  bool dirty = true;
  int threads = 256, blocksPerSM = 0, check = 100;
  int grid = 0;
  KernelFn kernel = nullptr;
  MomentsFn momentsKernel = nullptr;
  std::map<int, cudaGraphExec_t> graphs;
  cudaGraph_t graphTemplate = nullptr;
};

namespace {

int64_t take_space(lbx_ensemble_s* E, int64_t bytes) {
  for (auto it = E->freeList.begin(); it != E->freeList.end(); ++it) {
    if (it->second >= bytes) {
      const int64_t off = it->first, rest = it->second - bytes;
      E->freeList.erase(it);
      if (rest > 0) E->freeList[off + bytes] = rest;
      return off;
    }
  }
  return -1;
}

void give_space(lbx_ensemble_s* E, int64_t off, int64_t bytes) {
  auto it = E->freeList.emplace(off, bytes).first;
  auto next = std::next(it);
  if (next != E->freeList.end() && it->first + it->second == next->first) {
    it->second += next->second;
    E->freeList.erase(next);
  }
  if (it != E->freeList.begin()) {
    auto prev = std::prev(it);
    if (prev->first + prev->second == it->first) {
      prev->second += it->second;
      E->freeList.erase(it);
    }
  }
}

void drop_graphs(lbx_ensemble_s* E) {
  for (auto& kv : E->graphs) cudaGraphExecDestroy(kv.second);
  E->graphs.clear();
}

int ensure_grid(lbx_ensemble_s* E) {
  if (E->grid > 0) return LBX_OK;
  int perSM = 0, sms = 0;
  ENS_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, E->kernel, E->threads, 0));
  ENS_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, E->device));
  if (E->blocksPerSM > 0) perSM = std::min(perSM, E->blocksPerSM);
  if (perSM < 1) return lbx::set_error(LBX_ERR_UNSUPPORTED, "ensemble kernel does not fit on an SM");
  E->grid = perSM * sms;
  return LBX_OK;
}

// Tile list and per-slot tile ranges of the admitted lattices (running or finished, not yet retired).
int upload_tiles(lbx_ensemble_s* E, cudaStream_t s) {
  std::vector<int2> tiles;
  std::vector<int2> range(size_t(E->maxLattices), int2{0, 0});
  for (int slot = 0; slot < E->maxLattices; ++slot) {
    if (!E->slotUsed[size_t(slot)]) continue;
    const int first = int(tiles.size());
    for (int c = 0; c < E->slotCells[size_t(slot)]; c += E->threads) tiles.push_back(int2{slot, c});
    range[size_t(slot)] = int2{first, int(tiles.size()) - first};
  }
  if (int(tiles.size()) > E->tileCapacity) {
    const int cap = std::max<int>(int(tiles.size()), 2 * E->tileCapacity);
    cudaFree(E->dTiles);
    cudaFree(E->dTilePart);
    E->dTiles = nullptr;
    E->dTilePart = nullptr;
    E->tileCapacity = 0;
    ENS_TRY(cudaMalloc(&E->dTiles, size_t(cap) * sizeof(int2)));
    ENS_TRY(cudaMalloc(&E->dTilePart, size_t(cap) * 2 * sizeof(double)));
    E->tileCapacity = cap;
    drop_graphs(E);  // the graphs captured the old pointers
  }
  const int n = int(tiles.size());
  if (n) ENS_TRY(cudaMemcpyAsync(E->dTiles, tiles.data(), size_t(n) * sizeof(int2), cudaMemcpyHostToDevice, s));
  ENS_TRY(cudaMemcpyAsync(E->dRange, range.data(), range.size() * sizeof(int2), cudaMemcpyHostToDevice, s));
  ENS_TRY(cudaMemcpyAsync(E->dNTiles, &n, sizeof(int), cudaMemcpyHostToDevice, s));
  ENS_TRY(cudaStreamSynchronize(s));  // the host vectors go out of scope
  E->dirty = false;
  return LBX_OK;
}

}  // namespace

extern "C" {

int lbx_ensemble_footprint(int32_t q, int32_t storage, const lbx_ensemble_request* req, int64_t* bytes) {
  if (!req || !bytes) return lbx::set_error(LBX_ERR_INVALID, "null argument");
  if (elem_bytes(storage) == 0) return lbx::set_error(LBX_ERR_INVALID, "unknown storage");
  if (q != 19 && q != 27) return lbx::set_error(LBX_ERR_UNSUPPORTED, "ensembles are D3Q19 or D3Q27");
  for (int a = 0; a < 3; ++a)
    if (req->core[a] < 1 || req->core[a] > 4096) return lbx::set_error(LBX_ERR_INVALID, "core extent out of range");
  *bytes = region_bytes(q, storage, req, nullptr);
  return LBX_OK;
}

int lbx_ensemble_create(int32_t q, int32_t storage, int64_t slab_bytes, int32_t max_lattices, int32_t device,
                        lbx_ensemble* out) {
  if (!out) return lbx::set_error(LBX_ERR_INVALID, "null argument");
  *out = nullptr;
  if (q != 19 && q != 27) return lbx::set_error(LBX_ERR_UNSUPPORTED, "ensembles are D3Q19 or D3Q27");
  if (elem_bytes(storage) == 0) return lbx::set_error(LBX_ERR_INVALID, "unknown storage");
  if (slab_bytes < (1 << 20) || max_lattices < 1 || max_lattices > 65536)
    return lbx::set_error(LBX_ERR_INVALID, "slab must hold >= 1 MiB and 1..65536 lattices");
  if (lbx_device_count() <= device || device < 0) return lbx::set_error(LBX_ERR_NO_DEVICE, "no sm_100 device at that index");
  DeviceScope scope(device);
  auto* E = new lbx_ensemble_s();
  E->q = q;
  E->storage = storage;
  E->device = device;
  E->maxLattices = max_lattices;
  E->slabBytes = slab_bytes / 256 * 256;
  E->slotOffset.assign(size_t(max_lattices), -1);
  E->slotBytes.assign(size_t(max_lattices), 0);
  E->slotUsed.assign(size_t(max_lattices), 0);
  E->slotCells.assign(size_t(max_lattices), 0);
  kernels_for(q, storage, E->kernel, E->momentsKernel);
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&E->slab), size_t(E->slabBytes));
  if (e == cudaSuccess) e = cudaMalloc(&E->dLat, size_t(max_lattices) * sizeof(EnsLattice));
  if (e == cudaSuccess) e = cudaMemset(E->dLat, 0, size_t(max_lattices) * sizeof(EnsLattice));
  if (e == cudaSuccess) e = cudaMalloc(&E->dRange, size_t(max_lattices) * sizeof(int2));
  if (e == cudaSuccess) e = cudaMalloc(&E->dNTiles, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(E->dNTiles, 0, sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&E->dBarrier, 2 * sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMemset(E->dBarrier, 0, 2 * sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMalloc(&E->dErr, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(E->dErr, 0, sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&E->dGlobalStep, sizeof(long long));
  if (e == cudaSuccess) e = cudaMemset(E->dGlobalStep, 0, sizeof(long long));
  if (e != cudaSuccess) {
    const std::string msg = std::string("ensemble allocation failed: ") + cudaGetErrorString(e);
    lbx_ensemble_destroy(E);
    return lbx::set_error(e == cudaErrorMemoryAllocation ? LBX_ERR_OUT_OF_MEMORY : LBX_ERR_CUDA, msg);
  }
  E->freeList[0] = E->slabBytes;
  *out = E;
  return LBX_OK;
}

int lbx_ensemble_destroy(lbx_ensemble E) {
  if (!E) return LBX_OK;
  DeviceScope scope(E->device);
  cudaDeviceSynchronize();
  drop_graphs(E);
  cudaFree(E->slab);
  cudaFree(E->dLat);
  cudaFree(E->dTiles);
  cudaFree(E->dRange);
  cudaFree(E->dNTiles);
  cudaFree(E->dTilePart);
  cudaFree(E->dBarrier);
  cudaFree(E->dErr);
  cudaFree(E->dGlobalStep);
  delete E;
  return LBX_OK;
}

int lbx_ensemble_set_config(lbx_ensemble E, int32_t threads, int32_t blocks_per_sm, int32_t check_interval) {
  if (!E) return lbx::set_error(LBX_ERR_INVALID, "null ensemble");
  if (threads < 32 || threads > 256 || threads % 32) return lbx::set_error(LBX_ERR_INVALID, "threads must be 32..256, multiple of 32");
  if (blocks_per_sm < 0 || check_interval < 1) return lbx::set_error(LBX_ERR_INVALID, "bad blocks_per_sm or check interval");
  DeviceScope scope(E->device);
  cudaDeviceSynchronize();
  E->threads = threads;
  E->blocksPerSM = blocks_per_sm;
  E->check = check_interval;
  E->grid = 0;
  E->dirty = true;
  drop_graphs(E);
  return LBX_OK;
}

int lbx_ensemble_admit(lbx_ensemble E, const lbx_ensemble_request* req, int32_t* slot) {
  if (!E || !req || !slot) return lbx::set_error(LBX_ERR_INVALID, "null argument");
  int64_t bytes = 0;
  if (int rc = lbx_ensemble_footprint(E->q, E->storage, req, &bytes)) return rc;
  if (req->dynamics != LBX_BGK && req->dynamics != LBX_TRT) return lbx::set_error(LBX_ERR_UNSUPPORTED, "ensembles run BGK or TRT");
  if (!(req->params.omega > 0 && req->params.omega < 2)) return lbx::set_error(LBX_ERR_INVALID, "omega must lie in (0, 2)");
  if (req->dynamics == LBX_TRT && !(req->params.magic > 0)) return lbx::set_error(LBX_ERR_INVALID, "TRT magic parameter must be > 0");
  if (!std::isfinite(req->lid_velocity) || std::fabs(req->lid_velocity) > 0.4)
    return lbx::set_error(LBX_ERR_INVALID, "lid velocity must be finite and below 0.4 in lattice units");
  if (!(req->tolerance >= 0) || req->max_steps < 1) return lbx::set_error(LBX_ERR_INVALID, "bad tolerance or max_steps");
  int s = -1;
  for (int i = 0; i < E->maxLattices; ++i)
    if (!E->slotUsed[size_t(i)]) { s = i; break; }
  if (s < 0) return lbx::set_error(LBX_ERR_OUT_OF_MEMORY, "no free lattice slot");
  const int64_t off = take_space(E, bytes);
  if (off < 0) return lbx::set_error(LBX_ERR_OUT_OF_MEMORY, "slab has no room for " + std::to_string(bytes) + " bytes");
  DeviceScope scope(E->device);
  uint32_t P = 0;
  region_bytes(E->q, E->storage, req, &P);
  EnsLattice L;
  std::memset(&L, 0, sizeof(L));
  L.pop = E->slab + off;
  const int64_t popBytes = (int64_t(E->q) * P * int64_t(elem_bytes(E->storage)) + 255) / 256 * 256;
  L.snap = reinterpret_cast<float*>(E->slab + off + popBytes);
  L.P = P;
  L.nx = req->core[0];
  L.ny = req->core[1];
  L.nz = req->core[2];
  L.sy = req->core[2] + 2;
  L.sx = (req->core[1] + 2) * L.sy;
  L.ncore = req->core[0] * req->core[1] * req->core[2];
  L.dynamics = req->dynamics;
  L.state = LBX_SLOT_RUNNING;
  L.steps = 0;
  L.maxSteps = req->max_steps;
  L.tol = req->tolerance;
  L.residual = INFINITY;
  L.omega = float(req->params.omega);
  L.magic = float(req->params.magic);
  for (int k = 0; k < E->q; ++k) {
    const int* c = E->q == 19 ? Desc<19>::C[k] : Desc<27>::C[k];
    const double w = E->q == 19 ? double(Desc<19>::WN[k]) / Desc<19>::WD[k] : double(Desc<27>::WN[k]) / Desc<27>::WD[k];
    // 2 * veloTerm with veloTerm = (c_k . u_w) t_k / c_s^2 for the links through the lid
    L.delta[k] = c[1] == 1 ? float(2.0 * (c[0] * req->lid_velocity * w * 3.0)) : 0.f;
  }
  cudaError_t e = cudaMemset(E->slab + off, 0, size_t(bytes));  // rest state (f - w = 0) and snapshot
  if (e == cudaSuccess) e = cudaMemcpy(E->dLat + s, &L, sizeof(L), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    give_space(E, off, bytes);
    return lbx::set_error(LBX_ERR_CUDA, std::string("admit failed: ") + cudaGetErrorString(e));
  }
  E->slotUsed[size_t(s)] = 1;
  E->slotOffset[size_t(s)] = off;
  E->slotBytes[size_t(s)] = bytes;
  E->slotCells[size_t(s)] = L.ncore;
  E->dirty = true;
  *slot = s;
  return LBX_OK;
}

int lbx_ensemble_retire(lbx_ensemble E, int32_t slot) {
  if (!E || slot < 0 || slot >= E->maxLattices || !E->slotUsed[size_t(slot)])
    return lbx::set_error(LBX_ERR_INVALID, "not an admitted slot");
  DeviceScope scope(E->device);
  ENS_TRY(cudaDeviceSynchronize());
  const int32_t freeState = LBX_SLOT_FREE;
  ENS_TRY(cudaMemcpy(reinterpret_cast<char*>(E->dLat + slot) + offsetof(EnsLattice, state), &freeState,
                     sizeof(freeState), cudaMemcpyHostToDevice));
  give_space(E, E->slotOffset[size_t(slot)], E->slotBytes[size_t(slot)]);
  E->slotUsed[size_t(slot)] = 0;
  E->slotOffset[size_t(slot)] = -1;
  E->dirty = true;
  return LBX_OK;
}

int lbx_ensemble_run(lbx_ensemble E, int32_t steps, void* stream) {
  if (!E || steps < 1) return lbx::set_error(LBX_ERR_INVALID, "bad ensemble or step count");
  DeviceScope scope(E->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (int rc = ensure_grid(E)) return rc;
  if (E->dirty)
    if (int rc = upload_tiles(E, s)) return rc;
  auto it = E->graphs.find(steps);
  if (it == E->graphs.end()) {
    EnsArgs a;
    a.lat = E->dLat;
    a.tiles = E->dTiles;
    a.nTiles = E->dNTiles;
    a.range = E->dRange;
    a.tilePart = E->dTilePart;
    a.barrier = E->dBarrier;
    a.err = E->dErr;
    a.globalStep = E->dGlobalStep;
    a.maxLattices = E->maxLattices;
    a.steps = steps;
    a.check = E->check;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(unsigned(E->grid));
    cfg.blockDim = dim3(unsigned(E->threads));
    cfg.stream = nullptr;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    // capture { reset the error flag; persistent kernel } once per step count and replay it
    cudaStream_t cap;
    ENS_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cfg.stream = cap;
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) e = cudaMemsetAsync(E->dErr, 0, sizeof(int), cap);
    if (e == cudaSuccess) e = cudaLaunchKernelEx(&cfg, E->kernel, a);
    cudaError_t e2 = cudaStreamEndCapture(cap, &graph);
    cudaStreamDestroy(cap);
    if (e == cudaSuccess) e = e2;
    cudaGraphExec_t exec = nullptr;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      // no graph for this launch shape: launch directly (same kernel, same arguments)
      cudaGetLastError();
      cfg.stream = s;
      ENS_TRY(cudaMemsetAsync(E->dErr, 0, sizeof(int), s));
      ENS_TRY(cudaLaunchKernelEx(&cfg, E->kernel, a));
      return LBX_OK;
    }
    it = E->graphs.emplace(steps, exec).first;
  }
  ENS_TRY(cudaGraphLaunch(it->second, s));
  return LBX_OK;
}

int lbx_ensemble_statuses(lbx_ensemble E, lbx_ensemble_status* out, int32_t n, void* stream) {
  if (!E || !out || n < 0) return lbx::set_error(LBX_ERR_INVALID, "null argument");
  DeviceScope scope(E->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int m = std::min<int>(n, E->maxLattices);
  std::vector<EnsLattice> h(size_t(std::max(m, 1)));
  int err = 0;
  if (m > 0) ENS_TRY(cudaMemcpyAsync(h.data(), E->dLat, size_t(m) * sizeof(EnsLattice), cudaMemcpyDeviceToHost, s));
  ENS_TRY(cudaMemcpyAsync(&err, E->dErr, sizeof(int), cudaMemcpyDeviceToHost, s));
  ENS_TRY(cudaStreamSynchronize(s));
  if (err) return lbx::set_error(LBX_ERR_CUDA, "ensemble kernel grid barrier timed out (blocks not co-resident)");
  for (int i = 0; i < n; ++i) {
    lbx_ensemble_status st{};
    if (i < m && E->slotUsed[size_t(i)]) {
      st.state = h[size_t(i)].state;
      st.steps = h[size_t(i)].steps;
      st.residual = h[size_t(i)].residual;
    }
    out[i] = st;
  }
  return LBX_OK;
}

int lbx_ensemble_moments(lbx_ensemble E, int32_t slot, double* rho, double* u, void* stream) {
  if (!E || slot < 0 || slot >= E->maxLattices || !E->slotUsed[size_t(slot)])
    return lbx::set_error(LBX_ERR_INVALID, "not an admitted slot");
  DeviceScope scope(E->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int64_t n = E->slotCells[size_t(slot)];
  double* dev = nullptr;
  ENS_TRY(cudaMalloc(&dev, size_t(n) * 4 * sizeof(double)));
  E->momentsKernel<<<unsigned((n + 255) / 256), 256, 0, s>>>(E->dLat + slot, E->dGlobalStep, dev, dev + n);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && rho) e = cudaMemcpyAsync(rho, dev, size_t(n) * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && u) e = cudaMemcpyAsync(u, dev + n, size_t(n) * 3 * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(dev);
  ENS_TRY(e);
  return LBX_OK;
}

}  // extern "C"
