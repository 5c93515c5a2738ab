// Ensemble engine: many independent box cavities, one persistent kernel.
//
// Each admitted request owns a region of one device slab: Q population columns of period P
// (its padded cell count rounded up to 64; the periodic-shift layout of lbx_kernels.cuh, the
// ghost layer being the walls) and a velocity snapshot for the convergence residual.  A tile
// is up to 512 consecutive core cells of one lattice; the persistent kernel runs `steps`
// steps, in each of which its warps claim tiles from a counter and step them, and two
// grid-wide barriers per step separate the steps from the per-lattice bookkeeping done by
// block 0 (column shifts of the next step, step count, residual, state).  Lattices stop on their own
// residual and are retired by the host between runs while the others keep going, so requests
// of different sizes and ages are stepped together.
//
// Walls: halfway bounce-back on every face, fused into the store of the boundary cells: the
// population a cell sends into a wall direction k comes back as the opposite one,
// f_opp(k)(x_b) = f_k(x_b) - 2 t_k (c_k . u_w) / c_s^2 (the post-stream
// BouzidiVelocityPostProcessor with q = 1/2, boundary/setBouzidiBoundary.h:129-162), written to
// the slot the next step's load of x_b reads: in periodic-shift storage that is the slot of the
// ghost cell x_b + c_k in column opp(k) at the current shift, the same slot the single-lattice
// link kernel writes after its stream, so both paths hold identical populations between steps.
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
#include "lbx_test.h"

namespace lbx {
int set_error(int code, const std::string& msg);
}

namespace {

using namespace lbx;

constexpr int kMaxQ = 27;
constexpr int kTileCells = 512;  // cells per tile, independent of the launch shape

struct EnsLattice {
  void* pop;        // column 0; column i starts at element i * P
  float* snap;      // velocity snapshot [3][ncore]
  uint32_t P;
  int32_t nx, ny, nz;
  int32_t sx, sy;   // padded strides
  int32_t ncore;
  uint32_t mz, my;  // round-up multipliers for division by nz and ny (FastDiv)
  int32_t lz, ly;   // and their shifts
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
  int* tileCounter;        // tiles claimed so far in this step
  unsigned* barrier;       // {arrived, generation}
  int* err;
  long long* globalStep;
  int maxLattices;
  int steps;
  int check;
  long long spinLimit;     // polls of a grid-barrier wait before it gives up
  int faultBlock;          // test hook (lbx_test_fault): this block leaves without arriving (-1: none)
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

// Division by an invariant divisor d >= 1 for dividends below 2^31 (the round-up method of
// Granlund and Montgomery, "Division by invariant integers using multiplication", 1994):
// l = ceil(log2 d), m = floor(2^32 (2^l - d) / d) + 1, n / d = (umulhi(m, n) + n) >> l.
struct FastDiv {
  static void make(uint32_t d, uint32_t& m, int32_t& l) {
    l = 0;
    while ((uint64_t(1) << l) < d) ++l;
    m = uint32_t(((uint64_t(1) << 32) * ((uint64_t(1) << l) - d)) / d + 1);
  }
  static __device__ __forceinline__ uint32_t div(uint32_t n, uint32_t m, int32_t l) {
    return (__umulhi(m, n) + n) >> l;
  }
};

// Grid-wide barrier for a co-resident grid (cooperative launch).  Returns false when another
// block gave up or this block waited longer than the bound; the kernel then returns.
__device__ bool grid_barrier(unsigned* barrier, int* err, long long spinLimit) {
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
        if (++spins > spinLimit || *reinterpret_cast<volatile int*>(err)) {
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

// Resident 256-thread blocks per SM the register budget is cut for: one cell per thread, three
// for the 32- and 16-bit D3Q19 forms (80 registers); two cells per thread, two blocks (128
// registers); the compiler's choice otherwise.
template <int Q, typename S, int K> struct EnsOccupancy { static constexpr int blocks = 1; };
template <> struct EnsOccupancy<19, float, 1> { static constexpr int blocks = 3; };
template <> struct EnsOccupancy<19, __half, 1> { static constexpr int blocks = 3; };
template <> struct EnsOccupancy<19, __nv_bfloat16, 1> { static constexpr int blocks = 3; };
template <> struct EnsOccupancy<19, float, 2> { static constexpr int blocks = 2; };
template <> struct EnsOccupancy<19, __half, 2> { static constexpr int blocks = 2; };
template <> struct EnsOccupancy<19, __nv_bfloat16, 2> { static constexpr int blocks = 2; };

// Loads of populations inside a step: through L1 when every step is its own launch (the L1
// starts clean at each launch), around it (ld.global.cg) in the persistent kernel, where a
// line another block wrote in the previous step may still sit in this SM's L1.
template <typename S, bool CACHED> struct EnsLoad {
  static __device__ __forceinline__ typename Storage<S>::R ld(const S* p) {
    if constexpr (CACHED) return Storage<S>::load(p);
    else return CgLoad<S>::ld(p);
  }
};

// Per-warp scratch of the tile loop: each warp steps whole tiles on its own.
template <int Q, typename S> struct EnsWarp {
  // column i's base pointer with the shift folded in, valid for every cell of the tile when no
  // column's cyclic wrap point falls inside the tile's index range ("straight" tiles)
  S* col[Q];
  uint32_t shift[Q];
  float delta[Q];
};
constexpr int kMaxWarps = 8;  // 256 threads

// Core faces a cell lies on: bit 2a for the low face of axis a, bit 2a + 1 for the high one.
__device__ __forceinline__ int face_mask(int x, int y, int z, int nx, int ny, int nz) {
  return int(x == 0) | (int(x == nx - 1) << 1) | (int(y == 0) << 2) | (int(y == ny - 1) << 3) | (int(z == 0) << 4) |
         (int(z == nz - 1) << 5);
}
// Faces through which direction (cx, cy, cz) leaves the core from a cell lying on them.
constexpr int leaving_faces(int cx, int cy, int cz) {
  return (cx < 0 ? 1 : 0) | (cx > 0 ? 2 : 0) | (cy < 0 ? 4 : 0) | (cy > 0 ? 8 : 0) | (cz < 0 ? 16 : 0) |
         (cz > 0 ? 32 : 0);
}

// One step of every running lattice.  Each warp claims tiles from a shared counter until the
// list is exhausted and steps each claimed tile alone (no block-wide barrier): its lanes read
// the lattice's column shifts into the warp's scratch, then the warp walks the tile in 32-cell
// slots, K consecutive slots per round, lane l holding cell l of each, so every load and store
// instruction covers 32 consecutive cells.  Each slot's residual terms are reduced by a fixed
// shuffle tree and summed over the tile in slot order: neither the populations nor the residual
// depend on the launch shape, K or which warp stepped which tile.
template <int Q, typename S, bool CACHED, int K>
__device__ __forceinline__ void ensemble_tiles(const EnsArgs& a, int par, int nTiles, EnsWarp<Q, S>& w) {
  using R = typename Storage<S>::R;
  using D = Desc<Q>;
  const int lane = threadIdx.x & 31;
  for (;;) {
    int tile = 0;
    if (lane == 0) tile = atomicAdd(a.tileCounter, 1);
    tile = __shfl_sync(0xffffffffu, tile, 0);
    if (tile >= nTiles) break;
    const int2 t = a.tiles[tile];
    EnsLattice* L = a.lat + t.x;
    if (__ldcg(&L->state) != LBX_SLOT_RUNNING) continue;  // uniform over the warp
    const int64_t steps = __ldcg(reinterpret_cast<const long long*>(&L->steps));
    const bool check = ((steps + 1) % a.check) == 0;
    __syncwarp();  // the previous tile's readers of the scratch are done
    bool wraps = false;
    if (lane < Q) {
      const uint32_t sh = __ldcg(&L->shift[par][lane]);
      w.shift[lane] = sh;
      w.delta[lane] = __ldcg(&L->delta[lane]);
      // padded index range of the tile's cells: rows of the first and the last cell
      const int c0 = t.y, c1 = min(t.y + kTileCells, L->ncore) - 1;
      const uint32_t q0 = FastDiv::div(uint32_t(c0), L->mz, L->lz), q1 = FastDiv::div(uint32_t(c1), L->mz, L->lz);
      const uint32_t x0 = FastDiv::div(q0, L->my, L->ly), x1 = FastDiv::div(q1, L->my, L->ly);
      const uint32_t lo = (x0 + 1) * uint32_t(L->sx) + (q0 - x0 * uint32_t(L->ny) + 1) * uint32_t(L->sy) +
                          (uint32_t(c0) - q0 * uint32_t(L->nz)) + 1;
      const uint32_t hi = (x1 + 1) * uint32_t(L->sx) + (q1 - x1 * uint32_t(L->ny) + 1) * uint32_t(L->sy) +
                          (uint32_t(c1) - q1 * uint32_t(L->nz)) + 1;
      const uint32_t P = L->P;
      // the bounce-back stores reach one padded row beyond the tile's range on either side
      const uint32_t span = uint32_t(L->sx) + uint32_t(L->sy) + 1;
      const int64_t a0 = int64_t(lo) - span + sh, b0 = int64_t(hi) + span + sh;
      int64_t off = 0;
      if (b0 < int64_t(P) && a0 >= 0) off = sh;
      else if (a0 >= int64_t(P)) off = int64_t(sh) - int64_t(P);
      else wraps = true;
      w.col[lane] = static_cast<S*>(L->pop) + int64_t(lane) * int64_t(P) + off;
    }
    const bool straight = !__any_sync(0xffffffffu, wraps);
    __syncwarp();
    const uint32_t P = L->P;
    const int nx = L->nx, ny = L->ny, nz = L->nz, sx = L->sx, sy = L->sy;
    const uint32_t mz = L->mz, my = L->my;
    const int32_t lz = L->lz, ly = L->ly;
    const int last = min(kTileCells, L->ncore - t.y);  // cells of this tile
    const int ncore = L->ncore;
    S* pop = static_cast<S*>(L->pop);
    CollisionParams<R> cp;
    cp.omega = R(L->omega);
    cp.magic = R(L->magic);
    cp.smagorinsky = R(0);
    cp.force[0] = cp.force[1] = cp.force[2] = R(0);
    cp.avgSrc = nullptr;
    const int dyn = L->dynamics;
    const int slots = (last + 31) / 32;
    double tileDu2 = 0.0, tileU2 = 0.0;  // the tile's sums, slot by slot
    for (int g = 0; g < slots; g += K) {
      // The warp walks the tile round by round, each round a batch of loads that waits on the
      // previous one: lane i < Q first prefetches column i's run of the next round's cells into
      // L2 (one bulk prefetch), so that batch finds its populations there.  Straight tiles only
      // (the run is contiguous); widened to 16-byte bounds, which stay inside the lattice's
      // region of the slab (regions are multiples of 256 bytes).  On the eight-cavity mix this
      // raised the kernel from 28.0k to 28.6k MLUPS (graph mode) and 27.2k to 27.8k (persistent).
      if (straight && lane < Q && g + K < slots) {
        const int f0 = t.y + (g + K) * 32, f1 = t.y + min((g + 2 * K) * 32, last) - 1;
        auto padded = [&](int c) {
          const uint32_t xy = FastDiv::div(uint32_t(c), mz, lz);
          const uint32_t px = FastDiv::div(xy, my, ly);
          return (px + 1) * uint32_t(sx) + (xy - px * uint32_t(ny) + 1) * uint32_t(sy) + (uint32_t(c) - xy * uint32_t(nz)) + 1;
        };
        const S* col = w.col[lane];
        const uintptr_t p0 = reinterpret_cast<uintptr_t>(col + padded(f0)) & ~uintptr_t(15);
        const uintptr_t p1 = (reinterpret_cast<uintptr_t>(col + padded(f1) + 1) + 15) & ~uintptr_t(15);
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(p0), "r"(uint32_t(p1 - p0)) : "memory");
      }
      uint32_t n[K];
      int fm[K];  // face mask of the lane's cell in slot g + k; -1: no cell
      double du2[K], u2[K];
#pragma unroll
      for (int k = 0; k < K; ++k) {
        du2[k] = 0.0;
        u2[k] = 0.0;
        n[k] = 0;
        fm[k] = -1;
        const int cl = (g + k) * 32 + lane;
        if (cl < last) {
          const int c = t.y + cl;
          const uint32_t xy = FastDiv::div(uint32_t(c), mz, lz);
          const int z = c - int(xy) * nz;
          const int x = int(FastDiv::div(xy, my, ly));
          const int y = int(xy) - x * ny;
          n[k] = uint32_t((x + 1) * sx + (y + 1) * sy + z + 1);
          fm[k] = face_mask(x, y, z, nx, ny, nz);
        }
      }
      R f[K][Q];
      if (straight) {
        static_for<Q>([&](auto I) {
          const S* col = w.col[I];
#pragma unroll
          for (int k = 0; k < K; ++k)
            if (fm[k] >= 0) f[k][I] = EnsLoad<S, CACHED>::ld(col + n[k]);
        });
      } else {
        static_for<Q>([&](auto I) {
          const uint32_t sh = w.shift[I];
#pragma unroll
          for (int k = 0; k < K; ++k)
            if (fm[k] >= 0) f[k][I] = EnsLoad<S, CACHED>::ld(pop + I * int64_t(P) + wrap32(n[k] + sh, P));
        });
      }
#pragma unroll
      for (int k = 0; k < K; ++k) {
        if (fm[k] < 0) continue;
        if (check) {
          R rho, u[3];
          moments<Q, R, false>(f[k], nullptr, rho, u);
          float* snap = L->snap;
          const int c = t.y + (g + k) * 32 + lane;
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            const double cur = double(u[d]);
            const double dd = cur - double(__ldcg(snap + int64_t(d) * ncore + c));
            du2[k] += dd * dd;
            u2[k] += cur * cur;
            snap[int64_t(d) * ncore + c] = float(cur);
          }
        }
        R rho, usq;
        if (dyn == LBX_TRT) collide<Q, R, DYN_TRT>(f[k], cp, rho, usq);
        else collide<Q, R, DYN_BGK>(f[k], cp, rho, usq);
        if (!(usq == usq) || usq > R(1)) du2[k] = __longlong_as_double(0x7ff8000000000000ll);  // NaN flags divergence
      }
      // store addresses re-read from shared memory (volatile: not kept live in registers
      // across the collision, which would cost two registers per population)
      if (straight) {
        static_for<Q>([&](auto I) {
          S* col = *reinterpret_cast<S* volatile*>(&w.col[I]);
#pragma unroll
          for (int k = 0; k < K; ++k)
            if (fm[k] >= 0) Storage<S>::store(col + n[k], f[k][I]);
        });
      } else {
        static_for<Q>([&](auto I) {
          const uint32_t sh = *reinterpret_cast<volatile uint32_t*>(&w.shift[I]);
#pragma unroll
          for (int k = 0; k < K; ++k)
            if (fm[k] >= 0) Storage<S>::store(pop + I * int64_t(P) + wrap32(n[k] + sh, P), f[k][I]);
        });
      }
      // Halfway bounce-back of the links that leave the core: the population sent into the
      // wall comes back as the opposite one, written where the next step's load of this cell
      // finds it (the slot of ghost cell x + c_J in column opp(J) at this step's shift).
#pragma unroll
      for (int k = 0; k < K; ++k) {
        if (fm[k] <= 0) continue;
        static_for<Q>([&](auto J) {
          constexpr int cx = D::C[J][0], cy = D::C[J][1], cz = D::C[J][2];
          constexpr int leaves = leaving_faces(cx, cy, cz);
          if constexpr (leaves != 0) {
            if (fm[k] & leaves) {
              constexpr int O = D::OPP[J];
              const uint32_t gh = uint32_t(int(n[k]) + cx * sx + cy * sy + cz);
              // through the +y face: the moving lid
              const R v = f[k][J] - ((cy > 0 && (fm[k] & 8)) ? R(w.delta[J]) : R(0));
              if (straight) {
                Storage<S>::store(*reinterpret_cast<S* volatile*>(&w.col[O]) + gh, v);
              } else {
                const uint32_t sh = *reinterpret_cast<volatile uint32_t*>(&w.shift[O]);
                Storage<S>::store(pop + O * int64_t(P) + wrap32(gh + sh, P), v);
              }
            }
          }
        });
      }
      if (check) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) {
            du2[k] += __shfl_xor_sync(0xffffffffu, du2[k], o);
            u2[k] += __shfl_xor_sync(0xffffffffu, u2[k], o);
          }
          if (g + k < slots) {
            tileDu2 += du2[k];
            tileU2 += u2[k];
          }
        }
      }
    }
    if (check && lane == 0) {
      a.tilePart[2 * int64_t(tile)] = tileDu2;
      a.tilePart[2 * int64_t(tile) + 1] = tileU2;
    }
  }
}

// Per-lattice bookkeeping after a step (one block, a warp per lattice): step count, the next
// step's column shifts, and at check steps the residual and the state.  The residual sums the
// lattice's tile partials in a fixed order (lane l takes tiles l, l + 32, ..., then a shuffle
// tree), which depends on neither the block size nor the launch mode.  Thread 0 also resets the
// tile counter for the next step.
template <int Q>
__device__ __forceinline__ void ensemble_book(const EnsArgs& a, int par) {
  using D = Desc<Q>;
  const int lane = threadIdx.x & 31;
  if (threadIdx.x == 0) *a.tileCounter = 0;
  for (int s = threadIdx.x >> 5; s < a.maxLattices; s += blockDim.x >> 5) {
    EnsLattice* L = a.lat + s;
    if (__ldcg(&L->state) != LBX_SLOT_RUNNING) continue;  // uniform over the warp
    const int64_t steps = __ldcg(reinterpret_cast<const long long*>(&L->steps));
    const bool check = ((steps + 1) % a.check) == 0;
    const uint32_t P = L->P;
    const int sx = L->sx, sy = L->sy;
    static_for<Q>([&](auto I) {
      if (lane == I) {
        const int64_t off = D::C[I][0] * int64_t(sx) + D::C[I][1] * int64_t(sy) + D::C[I][2];
        int64_t ns = (int64_t(__ldcg(&L->shift[par][I])) - off) % int64_t(P);
        if (ns < 0) ns += P;
        L->shift[par ^ 1][I] = uint32_t(ns);
      }
    });
    int state = LBX_SLOT_RUNNING;
    double res = 0.0;
    if (check) {
      const int2 r = a.range[s];
      double s0 = 0, s1 = 0;
      for (int k = lane; k < r.y; k += 32) {
        s0 += __ldcg(a.tilePart + 2 * int64_t(r.x + k));
        s1 += __ldcg(a.tilePart + 2 * int64_t(r.x + k) + 1);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
      }
      res = s1 > 0 ? sqrt(s0 / s1) : (s0 > 0 ? INFINITY : 0.0);
      if (!(res == res) || !(s1 == s1) || isinf(s1)) state = LBX_SLOT_DIVERGED;
      else if (res < L->tol) state = LBX_SLOT_CONVERGED;
    }
    if (state == LBX_SLOT_RUNNING && steps + 1 >= L->maxSteps) state = LBX_SLOT_MAX_STEPS;
    __syncwarp();  // every lane has read the step count and the state
    if (lane == 0) {
      L->steps = steps + 1;
      if (check) L->residual = res;
      if (state != LBX_SLOT_RUNNING) L->state = state;
    }
  }
}

template <int Q, typename S, int K>
__global__ void __launch_bounds__(256, EnsOccupancy<Q, S, K>::blocks) k_ensemble(EnsArgs a) {
  __shared__ EnsWarp<Q, S> scratch[kMaxWarps];
  for (int step = 0; step < a.steps; ++step) {
    const long long g = *reinterpret_cast<volatile long long*>(a.globalStep);
    const int par = int(g & 1);
    ensemble_tiles<Q, S, false, K>(a, par, *a.nTiles, scratch[threadIdx.x >> 5]);
    if (int(blockIdx.x) == a.faultBlock) return;  // test hook: never arrives at the barrier
    if (!grid_barrier(a.barrier, a.err, a.spinLimit)) return;
    if (blockIdx.x == 0) {
      ensemble_book<Q>(a, par);
      if (threadIdx.x == 0) *a.globalStep = g + 1;
    }
    if (!grid_barrier(a.barrier, a.err, a.spinLimit)) return;
  }
}

// The same step as one ordinary launch (launch mode 1: a CUDA graph chains step and
// bookkeeping launches; the launch boundaries order the blocks, so no grid barrier is needed).
template <int Q, typename S, int K>
__global__ void __launch_bounds__(256, EnsOccupancy<Q, S, K>::blocks) k_ensemble_step(EnsArgs a) {
  __shared__ EnsWarp<Q, S> scratch[kMaxWarps];
  const long long g = *a.globalStep;
  ensemble_tiles<Q, S, true, K>(a, int(g & 1), *a.nTiles, scratch[threadIdx.x >> 5]);
}

template <int Q>
__global__ void __launch_bounds__(256) k_ensemble_book(EnsArgs a) {
  const long long g = *a.globalStep;
  ensemble_book<Q>(a, int(g & 1));
  __syncthreads();
  if (threadIdx.x == 0) *a.globalStep = g + 1;
}

// rho and u of one lattice's core cells (FP64 out); the wall links were applied by the step that
// wrote them.
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
  const int ny = L.ny, nz = L.nz, sx = L.sx, sy = L.sy;
  const int z = c % nz, y = (c / nz) % ny, x = c / (nz * ny);
  const uint32_t n = uint32_t((x + 1) * sx + (y + 1) * sy + z + 1);
  const S* pop = static_cast<const S*>(L.pop);
  R f[Q];
  static_for<Q>([&](auto I) { f[I] = Storage<S>::load(pop + I * int64_t(P) + wrap32(n + L.shift[par][I], P)); });
  R r, uu[3];
  moments<Q, R, false>(f, nullptr, r, uu);
  if (rho) rho[c] = double(r);
  if (u)
    for (int d = 0; d < 3; ++d) u[int64_t(d) * L.ncore + c] = double(uu[d]);
}

// Admission: the links through the moving lid start as if the rest state had been bounced once
// (the reference applies its post-processors once at initialisation): population opp(K) of a
// top-layer cell becomes 0 - delta_K, in the cell's own slot (the initial shifts are zero and
// the first step loads the cell's populations where they are).
template <int Q, typename S>
__global__ void k_ensemble_init_links(const EnsLattice* __restrict__ lat) {
  using R = typename Storage<S>::R;
  using D = Desc<Q>;
  const EnsLattice& L = *lat;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= L.nx * L.nz) return;
  const int x = i / L.nz, z = i % L.nz, y = L.ny - 1;
  const uint32_t n = uint32_t((x + 1) * L.sx + (y + 1) * L.sy + z + 1);
  S* pop = static_cast<S*>(L.pop);
  static_for<Q>([&](auto K) {
    constexpr int cy = D::C[K][1];
    if constexpr (cy == 1) {
      constexpr int O = D::OPP[K];
      Storage<S>::store(pop + O * int64_t(L.P) + n, R(0) - R(L.delta[K]));
    }
  });
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
using InitFn = void (*)(const EnsLattice*);
using BookFn = void (*)(EnsArgs);

// Kernels of one (Q, storage) pair; persistent[k] and step[k] take k + 1 cells per thread.
struct EnsKernels {
  KernelFn persistent[2] = {nullptr, nullptr};
  KernelFn step[2] = {nullptr, nullptr};
  MomentsFn moments = nullptr;
  InitFn init = nullptr;
  BookFn book = nullptr;
};

template <int Q, typename S>
void pick(EnsKernels& k) {
  k.persistent[0] = k_ensemble<Q, S, 1>;
  k.persistent[1] = k_ensemble<Q, S, 2>;
  k.step[0] = k_ensemble_step<Q, S, 1>;
  k.step[1] = k_ensemble_step<Q, S, 2>;
  k.moments = k_ensemble_moments<Q, S>;
  k.init = k_ensemble_init_links<Q, S>;
  k.book = k_ensemble_book<Q>;
}

bool kernels_for(int q, int storage, EnsKernels& k) {
  switch (q * 4 + storage) {
  case 19 * 4 + LBX_F64: pick<19, double>(k); return true;
  case 19 * 4 + LBX_F32: pick<19, float>(k); return true;
  case 19 * 4 + LBX_F16DEV: pick<19, __half>(k); return true;
  case 19 * 4 + LBX_BF16DEV: pick<19, __nv_bfloat16>(k); return true;
  case 27 * 4 + LBX_F64: pick<27, double>(k); return true;
  case 27 * 4 + LBX_F32: pick<27, float>(k); return true;
  case 27 * 4 + LBX_F16DEV: pick<27, __half>(k); return true;
  case 27 * 4 + LBX_BF16DEV: pick<27, __nv_bfloat16>(k); return true;
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
  std::vector<double> slotLid;  // lid velocity of each admitted request (for its checkpoint)
  EnsLattice* dLat = nullptr;
  int2* dTiles = nullptr;
  int2* dRange = nullptr;
  int* dNTiles = nullptr;
  int* dTileCounter = nullptr;
  double* dTilePart = nullptr;
  int tileCapacity = 0;
  unsigned* dBarrier = nullptr;
  int* dErr = nullptr;
  long long* dGlobalStep = nullptr;
  bool dirty = true;
  int threads = 256, blocksPerSM = 0, check = 100;
  int grid = 0;
  EnsKernels kern;
  int mode = 0;   // 0: persistent cooperative kernel, 1: per-step launches and a bookkeeping
                  // launch each, chained in a CUDA graph
  int cells = 1;  // cells per thread of the tile loop (1 or 2)
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

KernelFn launch_kernel(const lbx_ensemble_s* E) {
  return E->mode ? E->kern.step[E->cells - 1] : E->kern.persistent[E->cells - 1];
}

int ensure_grid(lbx_ensemble_s* E) {
  if (E->grid > 0) return LBX_OK;
  int perSM = 0, sms = 0;
  ENS_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, launch_kernel(E), E->threads, 0));
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
    for (int c = 0; c < E->slotCells[size_t(slot)]; c += kTileCells) tiles.push_back(int2{slot, c});
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
  if (int64_t(req->core[0] + 2) * (req->core[1] + 2) * (req->core[2] + 2) >= (int64_t(1) << 31) - 64)
    return lbx::set_error(LBX_ERR_UNSUPPORTED, "an ensemble lattice holds fewer than 2^31 padded cells");
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
  E->slotLid.assign(size_t(max_lattices), 0.0);
  kernels_for(q, storage, E->kern);
  cudaError_t e = lbx::test_allocation_fails() ? cudaErrorMemoryAllocation  // lbx_test_fault
                                               : cudaMalloc(reinterpret_cast<void**>(&E->slab), size_t(E->slabBytes));
  if (e == cudaSuccess) e = cudaMalloc(&E->dLat, size_t(max_lattices) * sizeof(EnsLattice));
  if (e == cudaSuccess) e = cudaMemset(E->dLat, 0, size_t(max_lattices) * sizeof(EnsLattice));
  if (e == cudaSuccess) e = cudaMalloc(&E->dRange, size_t(max_lattices) * sizeof(int2));
  if (e == cudaSuccess) e = cudaMalloc(&E->dNTiles, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(E->dNTiles, 0, sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&E->dTileCounter, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(E->dTileCounter, 0, sizeof(int));
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
  cudaFree(E->dTileCounter);
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

int lbx_ensemble_set_launch_mode(lbx_ensemble E, int32_t mode) {
  if (!E) return lbx::set_error(LBX_ERR_INVALID, "null ensemble");
  if (mode != 0 && mode != 1) return lbx::set_error(LBX_ERR_INVALID, "launch mode must be 0 or 1");
  DeviceScope scope(E->device);
  cudaDeviceSynchronize();
  E->mode = mode;
  E->grid = 0;
  drop_graphs(E);
  return LBX_OK;
}

int lbx_ensemble_set_cells_per_thread(lbx_ensemble E, int32_t cells) {
  if (!E) return lbx::set_error(LBX_ERR_INVALID, "null ensemble");
  if (cells != 1 && cells != 2) return lbx::set_error(LBX_ERR_INVALID, "cells per thread must be 1 or 2");
  DeviceScope scope(E->device);
  cudaDeviceSynchronize();
  E->cells = cells;
  E->grid = 0;
  drop_graphs(E);
  return LBX_OK;
}

int lbx_ensemble_autotune(lbx_ensemble E, int32_t steps, lbx_tune_entry* out, int32_t capacity, int32_t* n_out,
                          void* stream) {
  if (!E) return lbx::set_error(LBX_ERR_INVALID, "null ensemble");
  if (steps < 1 || capacity < 0 || (capacity > 0 && !out)) return lbx::set_error(LBX_ERR_INVALID, "bad steps or output array");
  int64_t hi = 0;
  for (int i = 0; i < E->maxLattices; ++i)
    if (E->slotUsed[size_t(i)]) hi = std::max(hi, E->slotOffset[size_t(i)] + E->slotBytes[size_t(i)]);
  if (hi == 0) return lbx::set_error(LBX_ERR_STATE, "autotune needs at least one admitted lattice");
  DeviceScope scope(E->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // Candidates: both launch modes, one or two cells per thread, block sizes 64..256, resident
  // blocks per SM from 1 to the occupancy maximum (the grid, and with it the cost of each grid
  // barrier, grows with both).
  struct Cand { int mode, cells, threads, perSM; };
  std::vector<Cand> cands;
  for (int mode = 0; mode <= 1; ++mode)
    for (int cells = 1; cells <= 2; ++cells)
      for (int threads = 64; threads <= 256; threads *= 2) {
        int maxPerSM = 0;
        KernelFn fn = mode ? E->kern.step[cells - 1] : E->kern.persistent[cells - 1];
        ENS_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&maxPerSM, fn, threads, 0));
        for (int b = 1; b <= std::min(maxPerSM, 8); b *= 2) cands.push_back({mode, cells, threads, b});
        if (maxPerSM > 8) cands.push_back({mode, cells, threads, maxPerSM});
      }
  if (n_out) *n_out = int32_t(cands.size());
  const Cand keep{E->mode, E->cells, E->threads, E->blocksPerSM};
  const size_t latBytes = size_t(E->maxLattices) * sizeof(EnsLattice);
  char* saved = nullptr;
  cudaError_t e = cudaMalloc(&saved, size_t(hi) + latBytes + sizeof(long long));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return lbx::set_error(e == cudaErrorMemoryAllocation ? LBX_ERR_OUT_OF_MEMORY : LBX_ERR_CUDA,
                          std::string("autotune state copy: ") + cudaGetErrorString(e));
  }
  auto copy_state = [&](bool save) -> cudaError_t {
    char* a = save ? saved : E->slab;
    const char* b = save ? E->slab : saved;
    cudaError_t r = cudaMemcpyAsync(a, b, size_t(hi), cudaMemcpyDeviceToDevice, s);
    char* la = save ? saved + hi : reinterpret_cast<char*>(E->dLat);
    const char* lb = save ? reinterpret_cast<const char*>(E->dLat) : saved + hi;
    if (r == cudaSuccess) r = cudaMemcpyAsync(la, lb, latBytes, cudaMemcpyDeviceToDevice, s);
    char* ga = save ? saved + hi + latBytes : reinterpret_cast<char*>(E->dGlobalStep);
    const char* gb = save ? reinterpret_cast<const char*>(E->dGlobalStep) : saved + hi + latBytes;
    if (r == cudaSuccess) r = cudaMemcpyAsync(ga, gb, sizeof(long long), cudaMemcpyDeviceToDevice, s);
    return r;
  };
  e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = copy_state(true);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  int best = -1, rc = LBX_OK;
  float bestMs = 0.f;
  auto apply = [&](const Cand& c) {
    E->mode = c.mode;
    E->cells = c.cells;
    E->threads = c.threads;
    E->blocksPerSM = c.perSM;
    E->grid = 0;
    E->dirty = true;
    drop_graphs(E);
  };
  for (size_t i = 0; i < cands.size() && e == cudaSuccess && rc == LBX_OK; ++i) {
    const Cand& c = cands[i];
    float ms = -1.f;
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    apply(c);
    if (e == cudaSuccess) e = copy_state(false);
    if (e == cudaSuccess) rc = lbx_ensemble_run(E, steps, stream);  // warm-up, captures the graph
    if (e == cudaSuccess && rc == LBX_OK) e = copy_state(false);
    if (e == cudaSuccess && rc == LBX_OK) e = cudaEventRecord(e0, s);
    if (e == cudaSuccess && rc == LBX_OK) rc = lbx_ensemble_run(E, steps, stream);
    if (e == cudaSuccess && rc == LBX_OK) e = cudaEventRecord(e1, s);
    if (e == cudaSuccess && rc == LBX_OK) e = cudaEventSynchronize(e1);
    int kerr = 0;
    if (e == cudaSuccess && rc == LBX_OK) e = cudaMemcpy(&kerr, E->dErr, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && rc == LBX_OK && kerr == 0) {
      e = cudaEventElapsedTime(&ms, e0, e1);
      ms /= float(steps);
      if (e == cudaSuccess && (best < 0 || ms < bestMs)) {
        best = int(i);
        bestMs = ms;
      }
    } else if (kerr != 0) {
      ms = -1.f;
    }
    if (out && int32_t(i) < capacity) out[i] = lbx_tune_entry{c.mode, 0, 0, c.cells, c.threads, c.perSM, double(ms)};
  }
  const std::string err = rc != LBX_OK ? std::string(lbx_last_error()) : std::string();
  cudaError_t e2 = cudaStreamSynchronize(s);
  if (e2 == cudaSuccess) e2 = copy_state(false);
  if (e2 == cudaSuccess) e2 = cudaMemsetAsync(E->dErr, 0, sizeof(int), s);
  if (e2 == cudaSuccess) e2 = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = e2;
  cudaFree(saved);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  apply(best >= 0 ? cands[size_t(best)] : keep);
  if (rc != LBX_OK) return lbx::set_error(rc, "autotune: " + err);
  if (e != cudaSuccess) return lbx::set_error(LBX_ERR_CUDA, std::string("autotune: ") + cudaGetErrorString(e));
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
  FastDiv::make(uint32_t(L.nz), L.mz, L.lz);
  FastDiv::make(uint32_t(L.ny), L.my, L.ly);
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
  if (e == cudaSuccess) {
    const int lid = L.nx * L.nz;
    E->kern.init<<<(lid + 255) / 256, 256>>>(E->dLat + s);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    give_space(E, off, bytes);
    return lbx::set_error(LBX_ERR_CUDA, std::string("admit failed: ") + cudaGetErrorString(e));
  }
  E->slotUsed[size_t(s)] = 1;
  E->slotOffset[size_t(s)] = off;
  E->slotBytes[size_t(s)] = bytes;
  E->slotCells[size_t(s)] = L.ncore;
  E->slotLid[size_t(s)] = req->lid_velocity;
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

// ---- checkpoint of one slot (pre-emption) ---------------------------------------------------
// Header, then the slot's raw population columns (q columns of period P at the saved shifts)
// and its velocity snapshot.  The request is re-admitted on restore and its state written over
// the fresh region, so the resumed lattice continues bit for bit.
struct EnsCheckpointHeader {
  char magic[8];  // "LBXENS01"
  int32_t q, storage;
  int32_t core[3];
  int32_t dynamics, state, pad;
  int64_t steps, maxSteps;
  double tol, residual, lid, omega, magicParam;
  uint32_t P;
  uint32_t shift[kMaxQ];  // the column shifts the next step reads
  int64_t popBytes, snapBytes;
};

namespace {
int64_t slot_pop_bytes(const lbx_ensemble_s* E, uint32_t P) { return int64_t(E->q) * int64_t(P) * int64_t(elem_bytes(E->storage)); }
int64_t slot_snap_bytes(int64_t ncore) { return 3 * ncore * int64_t(sizeof(float)); }
}  // namespace

int lbx_ensemble_checkpoint_bytes(lbx_ensemble E, int32_t slot, int64_t* bytes) {
  if (!E || !bytes || slot < 0 || slot >= E->maxLattices || !E->slotUsed[size_t(slot)])
    return lbx::set_error(LBX_ERR_INVALID, "not an admitted slot");
  DeviceScope scope(E->device);
  EnsLattice L;
  ENS_TRY(cudaMemcpy(&L, E->dLat + slot, sizeof(L), cudaMemcpyDeviceToHost));
  *bytes = int64_t(sizeof(EnsCheckpointHeader)) + slot_pop_bytes(E, L.P) + slot_snap_bytes(L.ncore);
  return LBX_OK;
}

int lbx_ensemble_save_slot(lbx_ensemble E, int32_t slot, void* host, int64_t bytes, void* stream) {
  if (!E || !host || slot < 0 || slot >= E->maxLattices || !E->slotUsed[size_t(slot)])
    return lbx::set_error(LBX_ERR_INVALID, "not an admitted slot");
  DeviceScope scope(E->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  ENS_TRY(cudaStreamSynchronize(s));
  EnsLattice L;
  long long g = 0;
  ENS_TRY(cudaMemcpy(&L, E->dLat + slot, sizeof(L), cudaMemcpyDeviceToHost));
  ENS_TRY(cudaMemcpy(&g, E->dGlobalStep, sizeof(g), cudaMemcpyDeviceToHost));
  EnsCheckpointHeader h;
  std::memset(&h, 0, sizeof(h));
  std::memcpy(h.magic, "LBXENS01", 8);
  h.q = E->q;
  h.storage = E->storage;
  h.core[0] = L.nx;
  h.core[1] = L.ny;
  h.core[2] = L.nz;
  h.dynamics = L.dynamics;
  h.state = L.state;
  h.steps = L.steps;
  h.maxSteps = L.maxSteps;
  h.tol = L.tol;
  h.residual = L.residual;
  h.omega = L.omega;
  h.magicParam = L.magic;
  h.lid = E->slotLid[size_t(slot)];
  h.P = L.P;
  for (int k = 0; k < E->q; ++k) h.shift[k] = L.shift[g & 1][k];
  h.popBytes = slot_pop_bytes(E, L.P);
  h.snapBytes = slot_snap_bytes(L.ncore);
  const int64_t need = int64_t(sizeof(h)) + h.popBytes + h.snapBytes;
  if (bytes < need) return lbx::set_error(LBX_ERR_INVALID, "checkpoint buffer holds " + std::to_string(bytes) +
                                                            " bytes, the slot needs " + std::to_string(need));
  char* out = static_cast<char*>(host);
  std::memcpy(out, &h, sizeof(h));
  ENS_TRY(cudaMemcpyAsync(out + sizeof(h), L.pop, size_t(h.popBytes), cudaMemcpyDeviceToHost, s));
  ENS_TRY(cudaMemcpyAsync(out + sizeof(h) + h.popBytes, L.snap, size_t(h.snapBytes), cudaMemcpyDeviceToHost, s));
  ENS_TRY(cudaStreamSynchronize(s));
  return LBX_OK;
}

int lbx_ensemble_restore_slot(lbx_ensemble E, const void* host, int64_t bytes, int32_t* slot, void* stream) {
  if (!E || !host || !slot) return lbx::set_error(LBX_ERR_INVALID, "null argument");
  if (bytes < int64_t(sizeof(EnsCheckpointHeader))) return lbx::set_error(LBX_ERR_INVALID, "checkpoint shorter than its header");
  EnsCheckpointHeader h;
  std::memcpy(&h, host, sizeof(h));
  if (std::memcmp(h.magic, "LBXENS01", 8) != 0) return lbx::set_error(LBX_ERR_INVALID, "not an ensemble slot checkpoint");
  if (h.q != E->q || h.storage != E->storage)
    return lbx::set_error(LBX_ERR_INVALID, "checkpoint was taken from an ensemble of another descriptor or storage");
  if (bytes < int64_t(sizeof(h)) + h.popBytes + h.snapBytes) return lbx::set_error(LBX_ERR_INVALID, "checkpoint truncated");
  lbx_ensemble_request req;
  std::memset(&req, 0, sizeof(req));
  for (int a = 0; a < 3; ++a) req.core[a] = h.core[a];
  req.dynamics = h.dynamics;
  req.params.omega = h.omega;
  req.params.magic = h.magicParam;
  req.lid_velocity = h.lid;
  req.tolerance = h.tol;
  req.max_steps = h.maxSteps;
  int32_t s0 = -1;
  if (int rc = lbx_ensemble_admit(E, &req, &s0)) return rc;
  DeviceScope scope(E->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  EnsLattice L;
  cudaError_t e = cudaMemcpy(&L, E->dLat + s0, sizeof(L), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && (L.P != h.P || slot_pop_bytes(E, L.P) != h.popBytes || slot_snap_bytes(L.ncore) != h.snapBytes)) {
    lbx_ensemble_retire(E, s0);
    return lbx::set_error(LBX_ERR_INVALID, "checkpoint does not match the lattice its request describes");
  }
  const char* in = static_cast<const char*>(host) + sizeof(h);
  if (e == cudaSuccess) e = cudaMemcpyAsync(L.pop, in, size_t(h.popBytes), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(L.snap, in + h.popBytes, size_t(h.snapBytes), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) {
    L.state = h.state;
    L.steps = h.steps;
    L.residual = h.residual;
    // both parities: whichever this ensemble's next step reads
    for (int k = 0; k < E->q; ++k) L.shift[0][k] = L.shift[1][k] = h.shift[k];
    e = cudaMemcpyAsync(E->dLat + s0, &L, sizeof(L), cudaMemcpyHostToDevice, s);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    lbx_ensemble_retire(E, s0);
    return lbx::set_error(LBX_ERR_CUDA, std::string("restore failed: ") + cudaGetErrorString(e));
  }
  *slot = s0;
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
    a.tileCounter = E->dTileCounter;
    a.barrier = E->dBarrier;
    a.err = E->dErr;
    a.globalStep = E->dGlobalStep;
    a.maxLattices = E->maxLattices;
    a.steps = steps;
    a.check = E->check;
    const lbx::TestFault& tf = lbx::test_fault();
    const bool fault = tf.kind == LBX_TEST_ENSEMBLE_BARRIER;
    a.spinLimit = (fault && tf.param > 0) ? tf.param : (1ll << 26);
    a.faultBlock = fault ? 0 : -1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(unsigned(E->grid));
    cfg.blockDim = dim3(unsigned(E->threads));
    cfg.stream = nullptr;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    // capture once per step count and replay: mode 0 { reset the error flag; persistent
    // kernel }, mode 1 { step launch; bookkeeping launch } x steps
    cudaStream_t cap;
    ENS_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cfg.stream = cap;
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) e = cudaMemsetAsync(E->dErr, 0, sizeof(int), cap);
    if (e == cudaSuccess) e = cudaMemsetAsync(E->dTileCounter, 0, sizeof(int), cap);
    // a run that gave up leaves the barrier count behind: every run starts from a clear barrier
    if (e == cudaSuccess) e = cudaMemsetAsync(E->dBarrier, 0, 2 * sizeof(unsigned), cap);
    if (E->mode == 0) {
      if (e == cudaSuccess) e = cudaLaunchKernelEx(&cfg, launch_kernel(E), a);
    } else {
      for (int k = 0; k < steps && e == cudaSuccess; ++k) {
        launch_kernel(E)<<<unsigned(E->grid), unsigned(E->threads), 0, cap>>>(a);
        E->kern.book<<<1, 256, 0, cap>>>(a);
        e = cudaGetLastError();
      }
    }
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
      ENS_TRY(cudaMemsetAsync(E->dTileCounter, 0, sizeof(int), s));
      ENS_TRY(cudaMemsetAsync(E->dBarrier, 0, 2 * sizeof(unsigned), s));
      if (E->mode == 0) {
        ENS_TRY(cudaLaunchKernelEx(&cfg, launch_kernel(E), a));
      } else {
        for (int k = 0; k < steps; ++k) {
          launch_kernel(E)<<<unsigned(E->grid), unsigned(E->threads), 0, s>>>(a);
          E->kern.book<<<1, 256, 0, s>>>(a);
        }
        ENS_TRY(cudaGetLastError());
      }
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
  E->kern.moments<<<unsigned((n + 255) / 256), 256, 0, s>>>(E->dLat + slot, E->dGlobalStep, dev, dev + n);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && rho) e = cudaMemcpyAsync(rho, dev, size_t(n) * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && u) e = cudaMemcpyAsync(u, dev + n, size_t(n) * 3 * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(dev);
  ENS_TRY(e);
  return LBX_OK;
}

}  // extern "C"
