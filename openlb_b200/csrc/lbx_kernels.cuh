// Kernels of the B200 lattice Boltzmann hot path.
//
// Storage (HBM): one population column per direction, Q columns of `stride` elements, each
// column a cyclic array over the N cells of the padded block (pad = 1).  Cell index
// n = (x+1)*sx + (y+1)*sy + (z+pz) (z fastest; 2D: sy = 1, pz = 0), as the reference's
// BlockStructure orders cells (src/core/blockStructure.h:71).  Population i of cell n lives
// at column_i[(n + shift_i) mod N]: the periodic-shift (PS) pattern of the reference's
// CyclicColumn (src/core/platform/cpu/sisd/column.h:128-221, core/platform/gpu/cuda/column.h:100-171).
// Streaming is the rotation shift_i -= c_i . (sx, sy, 1) done on the host between launches
// (ConcreteBlockLattice::stream, core/blockLattice.hh:316-338): no population moves.
//
// The fused step kernel therefore reads and writes every population of a core cell exactly
// once, in place (2 Q elements per lattice update).  On periodic axes the ghost layer has to
// carry the post-collision populations of the opposite face before the rotation (the
// reference's PostCollide overlap copy, core/superLattice.hh:150-155, core/platform/gpu/cuda/
// communicator.hh:111-124); the step kernel writes those few values itself, so a periodic
// step is a single launch.
#pragma once

#include <atomic>
#include <cstring>
#include <type_traits>

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "lbx_collision.cuh"

namespace lbx {

// ---- storage formats -----------------------------------------------------------------
template <typename S> struct Storage;
template <> struct Storage<double> {
  using R = double;
  static __device__ __forceinline__ R load(const double* p) { return *p; }
  static __device__ __forceinline__ void store(double* p, R v) { *p = v; }
};
template <> struct Storage<float> {
  using R = float;
  static __device__ __forceinline__ R load(const float* p) { return *p; }
  static __device__ __forceinline__ void store(float* p, R v) { *p = v; }
};
template <> struct Storage<__half> {
  using R = float;
  static __device__ __forceinline__ R load(const __half* p) { return __half2float(*p); }
  static __device__ __forceinline__ void store(__half* p, R v) { *p = __float2half_rn(v); }
};
template <> struct Storage<__nv_bfloat16> {
  using R = float;
  static __device__ __forceinline__ R load(const __nv_bfloat16* p) { return __bfloat162float(*p); }
  static __device__ __forceinline__ void store(__nv_bfloat16* p, R v) { *p = __float2bfloat16_rn(v); }
};

// ---- geometry of one lattice as the kernels see it -------------------------------------
struct Geometry {
  int64_t n;       // padded cells N (column length)
  int64_t stride;  // elements between column starts
  int64_t sx, sy;  // padded strides of x and y (z stride 1)
  int32_t nx, ny, nz;
  int32_t pz;      // 1 in 3D (z is padded), 0 in 2D
  int32_t pmask;   // periodic axes, bit a for axis a
};

template <int Q>
struct Shifts {
  int64_t s[Q];
};

__device__ __forceinline__ int64_t wrap_add(int64_t a, int64_t s, int64_t n) {
  const int64_t r = a + s;
  return r >= n ? r - n : r;
}

// Cell kinds of the device cell map: the public ids (0 no dynamics, 1 bulk, 2 bounce-back,
// 3 velocity / pressure boundary, 4 bounce-back with a wall velocity) plus 7, a bulk cell some of
// whose populations leave towards a resting halfway bounce-back wall; the K-cells step kernel
// writes those populations back into the cell's opposite slots itself (see
// k_collide_stream_groups), the other kernels treat 7 as 1.  Kinds 3 and 4 are collided by their
// own kernels after the bulk kernel, which neither loads nor stores them.
constexpr uint8_t kCellBulkLinked = 7;
constexpr uint8_t kCellBounceBackVelocity = 4;
// 8, 9, 10: bulk cells colliding with the parameters of class 1, 2, 3 (lbx_set_dynamics_class;
// stepped by the one-cell-per-thread kernel only, which a lattice with classes always uses)
constexpr uint8_t kCellClassFirst = 8, kCellClassLast = 10;
__device__ __forceinline__ bool bulk_kind(uint8_t k) {
  return k == 1 || k == kCellBulkLinked || (k >= kCellClassFirst && k <= kCellClassLast);
}
// the kinds the K-cells step kernel loads, collides and stores itself
__device__ __forceinline__ bool stepped_kind(uint8_t k) { return bulk_kind(k) || k == 2; }


// Block partial of the lattice statistics {sum rho, sum |u|^2, max |u|^2, count}: a warp
// butterfly, then the warps in index order, written to part[4 * block] without atomics.  With
// k_stats_finalize summing the partials in a fixed order, the statistics are bitwise
// reproducible from run to run.
__device__ __forceinline__ void block_partial(double a, double b, double m, double c, double* __restrict__ part) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
    m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    c += __shfl_xor_sync(0xffffffffu, c, o);
  }
  __shared__ double red[4][32];
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  const int nwarps = (blockDim.x * blockDim.y + 31) >> 5;
  if ((tid & 31) == 0) {
    red[0][tid >> 5] = a;
    red[1][tid >> 5] = b;
    red[2][tid >> 5] = m;
    red[3][tid >> 5] = c;
  }
  __syncthreads();
  if (tid == 0) {
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    for (int w = 0; w < nwarps; ++w) {
      s0 += red[0][w];
      s1 += red[1][w];
      s2 = fmax(s2, red[2][w]);
      s3 += red[3][w];
    }
    const int64_t bid = blockIdx.x + int64_t(gridDim.x) * (blockIdx.y + int64_t(gridDim.y) * blockIdx.z);
    part[4 * bid + 0] = s0;
    part[4 * bid + 1] = s1;
    part[4 * bid + 2] = s2;
    part[4 * bid + 3] = s3;
  }
}

// The block partials summed in a fixed order into the StatAcc the host reads: thread t adds
// partials t, t + 1024, ... in index order (eight loads in flight per thread), then a fixed
// shared-memory tree.  One block of 1024 threads; the result depends only on the partials.
constexpr int kFinalizeThreads = 1024;
static __global__ void __launch_bounds__(kFinalizeThreads) k_stats_finalize(const double* __restrict__ part,
                                                                           int64_t nblocks,
                                                                           StatAcc* __restrict__ out) {
  double a = 0, b = 0, m = 0, c = 0;
  constexpr int U = 8;
  int64_t i = threadIdx.x;
  for (; i + int64_t(U - 1) * kFinalizeThreads < nblocks; i += int64_t(U) * kFinalizeThreads) {
    double4 v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) v[u] = *reinterpret_cast<const double4*>(part + 4 * (i + int64_t(u) * kFinalizeThreads));
#pragma unroll
    for (int u = 0; u < U; ++u) {
      a += v[u].x;
      b += v[u].y;
      m = fmax(m, v[u].z);
      c += v[u].w;
    }
  }
  for (; i < nblocks; i += kFinalizeThreads) {
    a += part[4 * i + 0];
    b += part[4 * i + 1];
    m = fmax(m, part[4 * i + 2]);
    c += part[4 * i + 3];
  }
  __shared__ double s[4][kFinalizeThreads];
  s[0][threadIdx.x] = a;
  s[1][threadIdx.x] = b;
  s[2][threadIdx.x] = m;
  s[3][threadIdx.x] = c;
  __syncthreads();
  for (int stride = kFinalizeThreads / 2; stride > 0; stride >>= 1) {
    if (threadIdx.x < stride) {
      s[0][threadIdx.x] += s[0][threadIdx.x + stride];
      s[1][threadIdx.x] += s[1][threadIdx.x + stride];
      s[2][threadIdx.x] = fmax(s[2][threadIdx.x], s[2][threadIdx.x + stride]);
      s[3][threadIdx.x] += s[3][threadIdx.x + stride];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out->sum[0] = s[0][0];
    out->sum[1] = s[1][0];
    out->count = (unsigned long long)s[3][0];
    out->maxbits = (unsigned long long)__double_as_longlong(s[2][0]);
  }
}

// Deterministic 4-component block reduction for the FP64 field reductions: component k is a
// sum, or a max when bit k of MAXMASK is set.  Warp butterfly, then the warps in index order;
// one entry of 4 doubles per block, no atomics.
template <int MAXMASK>
__device__ __forceinline__ void block_partial4(double v0, double v1, double v2, double v3, double* __restrict__ part) {
  double v[4] = {v0, v1, v2, v3};
#pragma unroll
  for (int k = 0; k < 4; ++k)
    for (int o = 16; o > 0; o >>= 1) {
      const double w = __shfl_xor_sync(0xffffffffu, v[k], o);
      v[k] = ((MAXMASK >> k) & 1) ? fmax(v[k], w) : v[k] + w;
    }
  __shared__ double red[4][32];
  const int tid = threadIdx.x;
  const int nwarps = (blockDim.x + 31) >> 5;
  if ((tid & 31) == 0)
    for (int k = 0; k < 4; ++k) red[k][tid >> 5] = v[k];
  __syncthreads();
  if (tid < 4) {
    double a = 0.0;
    for (int w = 0; w < nwarps; ++w) a = ((MAXMASK >> tid) & 1) ? fmax(a, red[tid][w]) : a + red[tid][w];
    part[4 * int64_t(blockIdx.x) + tid] = a;
  }
}

// The block entries combined in a fixed order (thread t: entries t, t + 1024, ...; then a fixed
// tree) into out[0..3].
template <int MAXMASK>
static __global__ void __launch_bounds__(kFinalizeThreads) k_finalize4(const double* __restrict__ part, int64_t n,
                                                                      double* __restrict__ out) {
  double v[4] = {0, 0, 0, 0};
  for (int64_t i = threadIdx.x; i < n; i += kFinalizeThreads) {
    const double4 p = *reinterpret_cast<const double4*>(part + 4 * i);
    const double q[4] = {p.x, p.y, p.z, p.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = ((MAXMASK >> k) & 1) ? fmax(v[k], q[k]) : v[k] + q[k];
  }
  __shared__ double s[4][kFinalizeThreads];
  for (int k = 0; k < 4; ++k) s[k][threadIdx.x] = v[k];
  __syncthreads();
  for (int stride = kFinalizeThreads / 2; stride > 0; stride >>= 1) {
    if (threadIdx.x < stride)
      for (int k = 0; k < 4; ++k)
        s[k][threadIdx.x] = ((MAXMASK >> k) & 1) ? fmax(s[k][threadIdx.x], s[k][threadIdx.x + stride])
                                                : s[k][threadIdx.x] + s[k][threadIdx.x + stride];
    __syncthreads();
  }
  if (threadIdx.x < 4) out[threadIdx.x] = s[threadIdx.x][0];
}

// ---- fused collide + PS stream --------------------------------------------------------
// One thread per core cell; threadIdx.x runs along the fastest core axis (z in 3D, y in 2D)
// so that every population load and store of a warp is one contiguous run.
// The parameters of the three classes of a lattice (lbx_set_dynamics_class); `used` is 0 when the
// lattice has none.
template <typename R> struct ClassParams {
  CollisionParams<R> p[3];
  int dyn[3];  // the class's dynamics when it is not the lattice's (DYN_*), else 0
  int used;
};

// One collision of any bulk dynamics chosen at run time: the cells of a parameter class whose
// dynamics differ in kind from the lattice's (BGK beside TRT, say).  Out of line: one copy per
// descriptor and precision serves every kernel, and only those cells pay for the call.
template <int Q, typename R>
__device__ __noinline__ void collide_kind(int dyn, R (&f)[Q], const CollisionParams<R>& p, R& rho, R& usq) {
  switch (dyn) {
    case DYN_TRT: collide<Q, R, DYN_TRT>(f, p, rho, usq); break;
    case DYN_SMAGORINSKY: collide<Q, R, DYN_SMAGORINSKY>(f, p, rho, usq); break;
    case DYN_FORCED_BGK: collide<Q, R, DYN_FORCED_BGK>(f, p, rho, usq); break;
    case DYN_FORCED_SMAGORINSKY: collide<Q, R, DYN_FORCED_SMAGORINSKY>(f, p, rho, usq); break;
    default: collide<Q, R, DYN_BGK>(f, p, rho, usq); break;
  }
}
// Class c's parameters by value selects (no indexing into the parameter space).
template <typename R>
__device__ __forceinline__ CollisionParams<R> class_params(const ClassParams<R>& cls, int c) {
  CollisionParams<R> r = c == 0 ? cls.p[0] : (c == 1 ? cls.p[1] : cls.p[2]);
  return r;
}

template <int Q, typename S, int DYN>
__global__ void __launch_bounds__(256) k_collide_stream(S* __restrict__ pop, Geometry g, Shifts<Q> sh,
                                                        CollisionParams<typename Storage<S>::R> p,
                                                        const uint8_t* __restrict__ cellDyn,
                                                        double* __restrict__ statPart,
                                                        ClassParams<typename Storage<S>::R> cls) {
  using R = typename Storage<S>::R;
  using D = Desc<Q>;
  int x, y, z;
  bool inside;
  {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    const int m = blockIdx.y * blockDim.y + threadIdx.y;
    if constexpr (D::d == 3) {
      z = f; y = m; x = blockIdx.z;
      inside = z < g.nz && y < g.ny;
    } else {
      y = f; x = m; z = 0;
      inside = y < g.ny && x < g.nx;
    }
  }
  R rho = R(-1), usq = R(-1);
  bool valid = false;
  if (inside) {
    const int64_t n = int64_t(x + 1) * g.sx + int64_t(y + 1) * g.sy + (z + g.pz);
    const uint8_t kind = cellDyn ? cellDyn[n] : uint8_t(1);
    R f[Q];
    const bool needPops = kind != 0;
    if (needPops) {
      static_for<Q>([&](auto I) { f[I] = Storage<S>::load(pop + I * g.stride + wrap_add(n, sh.s[I], g.n)); });
    }
    if (bulk_kind(kind)) {
      if (cls.used && kind >= kCellClassFirst) {
        const int c = int(kind) - kCellClassFirst;
        const CollisionParams<R> pc = class_params(cls, c);
        const int cd = c == 0 ? cls.dyn[0] : (c == 1 ? cls.dyn[1] : cls.dyn[2]);
        if (cd == 0 || cd == DYN) collide<Q, R, DYN>(f, pc, rho, usq);
        else collide_kind<Q, R>(cd, f, pc, rho, usq);
      } else {
        collide<Q, R, DYN>(f, p, rho, usq);
      }
      valid = true;
    } else if (kind == 2) {
      revert<Q, R>(f);
    }
    if (kind != 0) {
      static_for<Q>([&](auto I) { Storage<S>::store(pop + I * g.stride + wrap_add(n, sh.s[I], g.n), f[I]); });
    }

  }

  if (statPart) block_partial(valid ? double(rho) : 0.0, valid ? double(usq) : 0.0, valid ? double(usq) : 0.0,
                              valid ? 1.0 : 0.0, statPart);
}

// ---- fused collide + PS stream, pipelined shared-memory tiles --------------------------
// A tile is TILE consecutive cells of the flat padded index space (ghost and spare cells
// included; only core cells are computed and stored).  Every population column is shifted by
// its own amount, so the TILE values of population i sit at a per-population offset in HBM.
// The tile's span of each population is copied as aligned 16-byte chunks into shared memory
// (one extra chunk absorbs the misalignment), computed there, and written back as aligned
// 16-byte chunks; only chunks that straddle a non-core cell fall back to element stores, so
// no slot owned by another tile is ever written.  The column period P is a multiple of the
// vector width and every tile starts at a multiple of it, so the misalignment of population
// i is s_i mod V for every tile and a chunk never straddles the cyclic wrap.
//
// Blocks are persistent and run a STAGES-deep cp.async pipeline: while tile k is computed
// and stored, the loads of tiles k+1 .. k+STAGES-1 are in flight, which keeps enough bytes
// outstanding per SM to saturate HBM independently of the register count.
constexpr int TILE = 256;

template <typename S> struct Vec;
template <> struct Vec<double> { static constexpr int V = 2; using T = double2; };
template <> struct Vec<float> { static constexpr int V = 4; using T = float4; };
template <> struct Vec<__half> { static constexpr int V = 8; using T = uint4; };
template <> struct Vec<__nv_bfloat16> { static constexpr int V = 8; using T = uint4; };

template <int Q, typename S>
struct TileCfg {
  static constexpr int V = Vec<S>::V;
  static constexpr int NCH = TILE / V + 1;  // 16-byte chunks per population span
  static constexpr int SPAN = NCH * V;      // elements per population per stage
  static constexpr int STAGE_BYTES = Q * SPAN * int(sizeof(S));
  static constexpr int STAGES = (4 * STAGE_BYTES <= 100 * 1024) ? 4 : ((3 * STAGE_BYTES <= 120 * 1024) ? 3 : 2);
  static constexpr int SMEM = STAGES * STAGE_BYTES;
};

// Post-collision values that leave the core across a periodic face are written into the ghost
// cell from which the next rotation carries them into the opposite face (the reference's
// PostCollide overlap copy, core/superLattice.hh:150-155, core/platform/gpu/cuda/communicator.hh:111-124).
template <int Q, typename S>
__device__ __forceinline__ void periodic_ghost_writes(S* __restrict__ pop, const Geometry& g, const Shifts<Q>& sh,
                                                      int x, int y, int z, const typename Storage<S>::R (&f)[Q]) {
  using D = Desc<Q>;
  const bool edge = ((g.pmask & 1) && (x == 0 || x == g.nx - 1)) || ((g.pmask & 2) && (y == 0 || y == g.ny - 1)) ||
                    (D::d == 3 && (g.pmask & 4) && (z == 0 || z == g.nz - 1));
  if (!edge) return;
  static_for<Q>([&](auto I) {
    constexpr int cx = D::C[I][0], cy = D::C[I][1], cz = D::C[I][2];
    int tx = x + cx, ty = y + cy, tz = z + cz;
    bool crossed = false, lost = false;
    if (tx < 0 || tx >= g.nx) { if (g.pmask & 1) { tx = tx < 0 ? tx + g.nx : tx - g.nx; crossed = true; } else lost = true; }
    if (ty < 0 || ty >= g.ny) { if (g.pmask & 2) { ty = ty < 0 ? ty + g.ny : ty - g.ny; crossed = true; } else lost = true; }
    if constexpr (D::d == 3) {
      if (tz < 0 || tz >= g.nz) { if (g.pmask & 4) { tz = tz < 0 ? tz + g.nz : tz - g.nz; crossed = true; } else lost = true; }
    }
    if (crossed && !lost) {
      const int64_t gn = int64_t(tx - cx + 1) * g.sx + int64_t(ty - cy + 1) * g.sy + (tz - cz + g.pz);
      Storage<S>::store(pop + I * g.stride + wrap_add(gn, sh.s[I], g.n), f[I]);
    }
  });
}

// Core coordinates of flat padded cell n (< 2^32: checked at lattice creation).
__device__ __forceinline__ bool decode_cell(const Geometry& g, int64_t n, int64_t nFlat, int& x, int& y, int& z) {
  if (n >= nFlat) return false;
  const unsigned un = unsigned(n), usx = unsigned(g.sx), usy = unsigned(g.sy);
  const unsigned px = un / usx;
  const unsigned rem = un - px * usx;
  const unsigned py = rem / usy;
  x = int(px) - 1;
  y = int(py) - 1;
  z = int(rem - py * usy) - g.pz;
  return x >= 0 && x < g.nx && y >= 0 && y < g.ny && z >= 0 && z < g.nz;
}

template <int Q, typename S, int DYN>
__global__ void __launch_bounds__(TILE) k_collide_stream_tiled(S* __restrict__ pop, Geometry g, Shifts<Q> sh,
                                                               int64_t base, int64_t nFlat, int64_t nTiles,
                                                               CollisionParams<typename Storage<S>::R> p,
                                                               const uint8_t* __restrict__ cellDyn,
                                                               double* __restrict__ statPart) {
  using R = typename Storage<S>::R;
  using C = TileCfg<Q, S>;
  using VT = typename Vec<S>::T;
  constexpr int V = C::V, NCH = C::NCH, SPAN = C::SPAN, STAGES = C::STAGES;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  S* sm = reinterpret_cast<S*>(smem_raw);  // [STAGES][Q][SPAN]
  __shared__ int64_t sShift[Q];
  __shared__ int sR[Q];
  __shared__ uint8_t sCore[STAGES][TILE];

  const int tid = threadIdx.x;
  static_for<Q>([&](auto I) {
    if (tid == I) {
      sShift[I] = sh.s[I];
      sR[I] = int(sh.s[I] % V);
    }
  });
  __syncthreads();

  // issue the cp.async copies of one tile into one stage (an empty group past the last tile)
  auto issue = [&](int64_t tile, int st) {
    if (tile < nTiles) {
      const int64_t t0 = base + tile * TILE;
      int x, y, z;
      sCore[st][tid] = decode_cell(g, t0 + tid, nFlat, x, y, z) ? 1 : 0;
      S* stage = sm + st * (Q * SPAN);
      for (int c = tid; c < Q * NCH; c += TILE) {
        const int i = c / NCH;
        const int k = c - i * NCH;
        int64_t a = wrap_add(t0, sShift[i], g.n) - sR[i] + int64_t(k) * V;
        if (a >= g.n) a -= g.n;
        const unsigned dst = unsigned(__cvta_generic_to_shared(stage + i * SPAN + k * V));
        const S* src = pop + i * g.stride + a;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
      }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };

  double accRho = 0.0, accUsq = 0.0, accMax = 0.0;
  unsigned accCount = 0;

  const int64_t stride = gridDim.x;
  for (int s = 0; s < STAGES - 1; ++s) issue(blockIdx.x + s * stride, s);

  int k = 0;
  for (int64_t tile = blockIdx.x; tile < nTiles; tile += stride, ++k) {
    const int st = k % STAGES;
    issue(tile + (STAGES - 1) * stride, (k + STAGES - 1) % STAGES);
    asm volatile("cp.async.wait_group %0;\n" ::"n"(STAGES - 1) : "memory");
    __syncthreads();

    S* stage = sm + st * (Q * SPAN);
    const int64_t n = base + tile * TILE + tid;
    int x, y, z;
    if (decode_cell(g, n, nFlat, x, y, z)) {
      const uint8_t kind = cellDyn ? cellDyn[n] : uint8_t(1);
      R f[Q];
      static_for<Q>([&](auto I) { f[I] = Storage<S>::load(stage + I * SPAN + sR[I] + tid); });
      if (bulk_kind(kind)) {
        R rho, usq;
        collide<Q, R, DYN>(f, p, rho, usq);
        accRho += double(rho);
        accUsq += double(usq);
        accMax = fmax(accMax, double(usq));
        ++accCount;
      } else if (kind == 2) {
        revert<Q, R>(f);
      }
      if (kind != 0) {
        static_for<Q>([&](auto I) { Storage<S>::store(stage + I * SPAN + sR[I] + tid, f[I]); });
      }
    }
    __syncthreads();

    const int64_t t0 = base + tile * TILE;
    for (int c = tid; c < Q * NCH; c += TILE) {
      const int i = c / NCH;
      const int kk = c - i * NCH;
      const int j0 = kk * V - sR[i];
      int64_t a = wrap_add(t0, sShift[i], g.n) - sR[i] + int64_t(kk) * V;
      if (a >= g.n) a -= g.n;
      const S* src = stage + i * SPAN + kk * V;
      S* dst = pop + i * g.stride + a;
      bool full = j0 >= 0 && j0 + V <= TILE;
      if (full) {
#pragma unroll
        for (int e = 0; e < V; ++e) full = full && sCore[st][j0 + e];
      }
      if (full) {
        *reinterpret_cast<VT*>(dst) = *reinterpret_cast<const VT*>(src);
      } else {
#pragma unroll
        for (int e = 0; e < V; ++e) {
          const int j = j0 + e;
          if (j >= 0 && j < TILE && sCore[st][j]) dst[e] = src[e];
        }
      }
    }
    __syncthreads();
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");

  if (statPart) block_partial(accRho, accUsq, accMax, double(accCount), statPart);
}

// ---- fused collide + PS stream, whole tiles moved by the TMA bulk-copy engine ------------
// Variant 3.  A tile is BT consecutive cells of the flat padded index space.  In periodic-shift
// storage the slots of those cells in column i are one contiguous run (no wrap with doubled
// columns), so each tile is brought into shared memory with one 1D bulk copy per population
// (cp.async.bulk, completion on an mbarrier), computed in place, and written back with one bulk
// store per population for the 16-byte-aligned interior of the run plus element stores for the
// unaligned head and tail (at most 15 bytes each), so no slot outside the tile is written.
// Two stages per block: the next tile's copies are in flight while the current one is computed.
// Ghost and spare cells inside a tile are written back unchanged; the periodic overlap copy
// (k_periodic_halo) runs after this kernel and overwrites the ghost slots it owns.
// Memory requests: 2 * Q bulk operations per tile instead of 2 * Q * BT / 32 warp accesses,
// which is what the 16-bit forms are limited by on the SM -> L2 path.
// Division of flat cell indices (< 2^31) by the padded strides sx and sy: round-up multiplier and
// shift (Granlund and Montgomery, "Division by invariant integers using multiplication", 1994):
// n / d = (umulhi(m, n) + n) >> l with l = ceil(log2 d), m = floor(2^32 (2^l - d) / d) + 1.
struct FlatDiv {
  uint32_t mx, my;
  int32_t lx, ly;
  static void make(uint32_t d, uint32_t& m, int32_t& l) {
    l = 0;
    while ((uint64_t(1) << l) < d) ++l;
    m = uint32_t(((uint64_t(1) << 32) * ((uint64_t(1) << l) - d)) / d + 1);
  }
};

template <int Q, typename S> struct BulkCfg {
  static constexpr int ES = int(sizeof(S));
  static constexpr int BT = (36864 / (Q * ES)) / 64 * 64;  // cells per tile: ~36 KB of populations
  static constexpr int COL_BYTES = BT * ES + 32;           // one column's run + alignment slack
  static constexpr int STAGE_BYTES = Q * COL_BYTES;
  static constexpr int SMEM = 2 * STAGE_BYTES + 64;        // two stages + the mbarriers
  static constexpr int THREADS = 256;
  static constexpr int BLOCKS = 3;                          // resident blocks per SM (registers <= 85)
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}
__device__ __forceinline__ void bulk_s2g(void* dst, const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n" ::"l"(dst), "r"(smem_addr(src)),
               "r"(bytes)
               : "memory");
}

// Bounded wait on an mbarrier phase; false (and the error flag set) if it did not complete.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int* err, int limit) {
  for (int it = 0; it < limit; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if (it > 64) __nanosleep(64);
  }
  atomicExch(err, 1);
  return false;
}

template <int Q, typename S, int DYN>
__global__ void __launch_bounds__(BulkCfg<Q, S>::THREADS, BulkCfg<Q, S>::BLOCKS) k_collide_stream_bulk(
    S* __restrict__ pop, Geometry g, Shifts<Q> sh, int64_t base, int64_t nFlat, int64_t nTiles,
    CollisionParams<typename Storage<S>::R> p, const uint8_t* __restrict__ cellDyn, double* __restrict__ statPart,
    int* __restrict__ err, FlatDiv dv, int waitLimit, int faultSkip) {
  using R = typename Storage<S>::R;
  using C = BulkCfg<Q, S>;
  constexpr int ES = C::ES, BT = C::BT, NT = C::THREADS, VE = 16 / ES;
  constexpr int COL = C::COL_BYTES / ES;  // elements per column buffer
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + 2 * C::STAGE_BYTES);
  __shared__ int sHead[2][Q];  // per stage and column: elements from the aligned run start to the tile
  __shared__ int sAbort;
  const int tid = threadIdx.x;
  int issued[2] = {0, 0}, waited[2] = {0, 0};  // bulk-load phases per stage (thread 0's view)
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    sAbort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();

  // the bulk loads of `tile` into stage `st` (thread 0)
  auto issue = [&](int64_t tile, int st) {
    const int64_t t0 = base + tile * BT;
    const int64_t cells = (t0 + BT <= nFlat) ? BT : nFlat - t0;
    uint32_t total = 0;
    for (int i = 0; i < Q; ++i) {
      const int64_t first = (t0 + sh.s[i]) * ES;
      const int64_t a0 = first & ~int64_t(15), a1 = (first + cells * ES + 15) & ~int64_t(15);
      sHead[st][i] = int((first - a0) / ES);
      total += uint32_t(a1 - a0);
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    mbar_expect_tx(&bar[st], total);
    unsigned char* stage = smem_raw + st * C::STAGE_BYTES;
    for (int i = 0; i < Q; ++i) {
      const int64_t first = (t0 + sh.s[i]) * ES;
      const int64_t a0 = first & ~int64_t(15), a1 = (first + cells * ES + 15) & ~int64_t(15);
      // test hook (lbx_test_fault): block 0 leaves its first tile's column 0 unrequested, so that
      // its bounded wait runs out
      if (faultSkip && blockIdx.x == 0 && tile == int64_t(blockIdx.x) && i == 0) continue;
      bulk_g2s(stage + i * C::COL_BYTES, reinterpret_cast<const unsigned char*>(pop + i * g.stride) + a0,
               uint32_t(a1 - a0), &bar[st]);
    }
    ++issued[st];
  };

  double accRho = 0.0, accUsq = 0.0, accMax = 0.0, accCount = 0.0;
  const int64_t stride = gridDim.x;
  int k = 0;
  if (tid == 0 && int64_t(blockIdx.x) < nTiles) issue(blockIdx.x, 0);
  for (int64_t tile = blockIdx.x; tile < nTiles; tile += stride, ++k) {
    const int st = k & 1;
    __syncthreads();  // every thread is done with stage st ^ 1 (the previous tile)
    if (tid == 0) {
      asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");  // its bulk stores have read it
      if (tile + stride < nTiles) issue(tile + stride, st ^ 1);
    }
    if (!mbar_wait_bounded(&bar[st], uint32_t((k >> 1) & 1), err, waitLimit)) sAbort = 1;
    else if (tid == 0) ++waited[st];
    __syncthreads();
    if (sAbort) break;
    const int64_t t0 = base + tile * BT;
    const int cells = int((t0 + BT <= nFlat) ? BT : nFlat - t0);
    S* stage = reinterpret_cast<S*>(smem_raw + st * C::STAGE_BYTES);
    for (int j = tid; j < cells; j += NT) {
      // core test of flat cell t0 + j by multiply-high division (the divisors sx, sy are fixed)
      const uint32_t un = uint32_t(t0 + j);
      const uint32_t px = (__umulhi(un, dv.mx) + un) >> dv.lx;
      const uint32_t rem = un - px * uint32_t(g.sx);
      const uint32_t py = (__umulhi(rem, dv.my) + rem) >> dv.ly;
      const int x = int(px) - 1, y = int(py) - 1, z = int(rem - py * uint32_t(g.sy)) - g.pz;
      if (!(x >= 0 && x < g.nx && y >= 0 && y < g.ny && z >= 0 && z < g.nz)) continue;
      const uint8_t kind = cellDyn ? cellDyn[t0 + j] : uint8_t(1);
      if (!bulk_kind(kind) && kind != 2) continue;
      R f[Q];
      static_for<Q>([&](auto I) { f[I] = Storage<S>::load(stage + I * COL + sHead[st][I] + j); });
      if (bulk_kind(kind)) {
        R rho, usq;
        collide<Q, R, DYN>(f, p, rho, usq);
        accRho += double(rho);
        accUsq += double(usq);
        accMax = fmax(accMax, double(usq));
        accCount += 1.0;
      } else {
        revert<Q, R>(f);
      }
      static_for<Q>([&](auto I) { Storage<S>::store(stage + I * COL + sHead[st][I] + j, f[I]); });
    }
    // the new stage contents become visible to the bulk-copy (async) proxy, then go back: the
    // 16-byte-aligned interior of each column's run by one bulk store, the unaligned head and
    // tail (fewer than 16 bytes each) by element stores
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      for (int i = 0; i < Q; ++i) {
        const int64_t first = (t0 + sh.s[i]) * ES;
        const int64_t b0 = (first + 15) & ~int64_t(15), b1 = (first + int64_t(cells) * ES) & ~int64_t(15);
        if (b1 > b0)
          bulk_s2g(reinterpret_cast<unsigned char*>(pop + i * g.stride) + b0,
                   reinterpret_cast<unsigned char*>(stage) + i * C::COL_BYTES + (b0 - (first & ~int64_t(15))),
                   uint32_t(b1 - b0));
      }
      asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
    }
    for (int c = tid; c < Q * 2 * VE; c += NT) {
      const int i = c / (2 * VE), e = c - i * (2 * VE);
      const int64_t first = (t0 + sh.s[i]) * ES;
      const int64_t b0 = (first + 15) & ~int64_t(15), b1 = (first + int64_t(cells) * ES) & ~int64_t(15);
      int jj;
      bool ok;
      if (b1 > b0) {
        const int head = int((b0 - first) / ES), tail = int((b1 - first) / ES);
        jj = e < VE ? e : tail + (e - VE);
        ok = e < VE ? jj < head : jj < cells;
      } else {  // run shorter than 32 bytes: every element by an element store
        jj = e;
        ok = jj < cells;
      }
      if (ok) pop[i * g.stride + t0 + sh.s[i] + jj] = stage[i * COL + sHead[st][i] + jj];
    }
  }
  if (tid == 0) {
    asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
    // after an abort: let the loads still in flight land before the block exits (bounded)
    for (int st = 0; st < 2; ++st)
      while (waited[st] < issued[st]) {
        mbar_wait_bounded(&bar[st], uint32_t(waited[st] & 1), err, waitLimit);
        ++waited[st];
      }
  }
  if (statPart) block_partial(accRho, accUsq, accMax, accCount, statPart);
}

// ---- fused collide + PS stream, warp-specialised bulk-copy pipeline -----------------------
// Variant 4.  The tile scheme of variant 3 (BT consecutive flat cells; per population one
// contiguous run, brought in by one 1D bulk copy), rebuilt so that no block-wide barrier sits on
// the path of a tile:
//   - warp 0 is the producer: its lane 0 issues the bulk loads of a tile into a ring of NS
//     stages (completion: the stage's `full` mbarrier, by bytes), and, once the consumers have
//     released a stage (its `empty` mbarrier, one arrival per consumer warp), the bulk stores of
//     the 16-byte-aligned interior of every column's run; the stage is loaded again when those
//     stores have read it (the store group one behind the newest), so NS - 1 tiles are in flight
//     ahead of the one being computed;
//   - warps 1..16 are consumers: each waits for its tile's `full` phase, collides its cells in
//     shared memory (16-bit BGK pairs with the packed two-cell collision), writes the unaligned
//     head and tail elements of each run straight to their slots, makes its shared-memory
//     writes visible to the bulk-copy proxy and arrives on the stage's `empty` barrier.
// A fast consumer warp runs ahead into the next loaded stage instead of waiting for the block.
// Ghost and spare cells of a tile go back unchanged; the periodic overlap copy runs afterwards
// (k_periodic_halo), as for variant 3.  Every wait is bounded: a wait that gives up sets the
// error flag and the abort word, and every warp leaves its loop; the producer then waits
// (bounded) for its loads still in flight and its stores before the block exits.
template <int Q, typename S> struct WsCfg {
  static constexpr int ES = int(sizeof(S));
  // cells per tile: ~40 KB of populations, so that each bulk copy moves 1-4 KB (the per-copy
  // cost of the copy engine, not the bytes, bounded the first form with 20 KB tiles)
  static constexpr int BT = (40960 / (Q * ES)) / 64 * 64;
  static constexpr int COL_BYTES = BT * ES + 32;           // one column's run + alignment slack
  static constexpr int STAGE_BYTES = Q * COL_BYTES;
  static constexpr int NS = 4;                              // stages in the ring
  static constexpr int CONSUMER_WARPS = 16;
  static constexpr int THREADS = 32 * (1 + CONSUMER_WARPS);
  static constexpr int SMEM = NS * STAGE_BYTES + 2 * NS * 8;  // stages, then the full and empty mbarriers
  static constexpr int BLOCKS = 1;                          // resident blocks per SM
  static_assert(BT >= 64 && COL_BYTES % 16 == 0 && STAGE_BYTES % 16 == 0, "tile layout");
  static_assert(BT <= 4095, "packed run bounds hold 12 bits");
};

// Bounded wait without sleeping: try_wait itself suspends the thread for a while before it
// reports an incomplete phase, so the pipeline's waits need no back-off of their own.
__device__ __forceinline__ bool mbar_wait_spin(uint64_t* bar, uint32_t parity, int* err, int limit) {
  for (int it = 0; it < limit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  atomicExch(err, 1);
  return false;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_addr(bar)) : "memory");
}

template <int Q, typename S, int DYN>
__global__ void __launch_bounds__(WsCfg<Q, S>::THREADS, WsCfg<Q, S>::BLOCKS) k_collide_stream_ws(
    S* __restrict__ pop, Geometry g, Shifts<Q> sh, int64_t base, int64_t nFlat, int64_t nTiles,
    CollisionParams<typename Storage<S>::R> p, const uint8_t* __restrict__ cellDyn, double* __restrict__ statPart,
    int* __restrict__ err, FlatDiv dv, int waitLimit) {
  using R = typename Storage<S>::R;
  using C = WsCfg<Q, S>;
  constexpr int ES = C::ES, BT = C::BT, NS = C::NS;
  constexpr int COL = C::COL_BYTES / ES;      // elements per column buffer
  constexpr int NCT = 32 * C::CONSUMER_WARPS;  // consumer threads
  constexpr bool PACKED = sizeof(R) == 4 && sizeof(S) == 2 && DYN == DYN_BGK;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + NS * C::STAGE_BYTES);
  uint64_t* empty = full + NS;
  // per stage and column: bits 0-3 the elements from the aligned run start to the tile's first
  // cell, bits 4-15 the cells of the unaligned head, bits 16-27 the first cell of the tail
  __shared__ uint32_t sRun[NS][Q];
  __shared__ volatile int sAbort;
  const int warp = int(threadIdx.x) >> 5, lane = int(threadIdx.x) & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < NS; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], C::CONSUMER_WARPS);
    }
    sAbort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  const int64_t grid = gridDim.x;
  const int64_t nloc = int64_t(blockIdx.x) < nTiles ? (nTiles - int64_t(blockIdx.x) + grid - 1) / grid : 0;
  auto tile_first = [&](int64_t k) { return base + (int64_t(blockIdx.x) + k * grid) * BT; };
  auto tile_cells = [&](int64_t t0) { return int((t0 + BT <= nFlat) ? BT : nFlat - t0); };
  double accRho = 0.0, accUsq = 0.0, accMax = 0.0, accCount = 0.0;

  if (warp == 0) {
    // the whole producer warp: lane i < Q looks after column i (its run bounds, its bulk load and
    // its bulk store), lane 0 alone arms the stage's barrier with the total byte count
    const bool col = lane < Q;
    int64_t shift = 0;  // this lane's column shift (a select: no indexing into the parameters)
    static_for<Q>([&](auto I) {
      if (int(I) == lane) shift = sh.s[I];
    });
    const S* srcCol = pop + int64_t(col ? lane : 0) * g.stride;
    int64_t issued = 0;
    auto issue = [&](int64_t k) {
      const int s = int(k % NS);
      const int64_t t0 = tile_first(k);
      const int cells = tile_cells(t0);
      uint32_t bytes = 0;
      int64_t a0 = 0;
      if (col) {
        const int64_t first = (t0 + shift) * ES, last = first + int64_t(cells) * ES;
        a0 = first & ~int64_t(15);
        const int64_t a1 = (last + 15) & ~int64_t(15);
        const int64_t b0 = (first + 15) & ~int64_t(15), b1 = last & ~int64_t(15);
        const uint32_t head = b1 > b0 ? uint32_t((b0 - first) / ES) : uint32_t(cells);
        const uint32_t tail = b1 > b0 ? uint32_t((b1 - first) / ES) : uint32_t(cells);
        sRun[s][lane] = uint32_t((first - a0) / ES) | (head << 4) | (tail << 16);
        bytes = uint32_t(a1 - a0);
      }
      uint32_t total = bytes;
      for (int o = 16; o > 0; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
      __syncwarp();  // the lanes' run bounds precede lane 0's arrival, which releases them
      if (lane == 0) {
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        mbar_expect_tx(&full[s], total);
      }
      __syncwarp();
      if (col)
        bulk_g2s(smem_raw + s * C::STAGE_BYTES + lane * C::COL_BYTES,
                 reinterpret_cast<const unsigned char*>(srcCol) + a0, bytes, &full[s]);
      ++issued;
    };
    while (issued < nloc && issued < NS) issue(issued);
    for (int64_t k = 0; k < nloc; ++k) {
      const int s = int(k % NS);
      const bool ok = mbar_wait_spin(&empty[s], uint32_t((k / NS) & 1), err, waitLimit);
      if (!__all_sync(0xffffffffu, ok)) {
        sAbort = 1;
        break;
      }
      const int64_t t0 = tile_first(k);
      const int cells = tile_cells(t0);
      if (col) {
        const int64_t first = (t0 + shift) * ES;
        const int64_t b0 = (first + 15) & ~int64_t(15), b1 = (first + int64_t(cells) * ES) & ~int64_t(15);
        if (b1 > b0)
          bulk_s2g(reinterpret_cast<unsigned char*>(const_cast<S*>(srcCol)) + b0,
                   smem_raw + s * C::STAGE_BYTES + lane * C::COL_BYTES + (b0 - (first & ~int64_t(15))),
                   uint32_t(b1 - b0));
        asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
      }
      // the stage is free again once every lane's stores have read it; the next tile for it is
      // then NS - 1 tiles ahead of the consumers
      if (issued < nloc) {
        if (col) asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");
        if (__any_sync(0xffffffffu, sAbort != 0)) break;  // the same decision in every lane
        issue(issued);
      }
    }
    if (col) asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
    // loads still in flight (after an abort) land before the block exits: the phase of the
    // last load issued into each stage (no later phase follows it)
    if (lane == 0)
      for (int s = 0; s < NS; ++s)
        if (issued > s) {
          const int64_t kl = s + ((issued - 1 - s) / NS) * NS;
          mbar_wait_spin(&full[s], uint32_t((kl / NS) & 1), err, waitLimit);
        }
  } else {
    const int ct = int(threadIdx.x) - 32;
    for (int64_t k = 0; k < nloc; ++k) {
      if (sAbort) break;
      const int s = int(k % NS);
      if (!mbar_wait_spin(&full[s], uint32_t((k / NS) & 1), err, waitLimit)) {
        sAbort = 1;
        break;
      }
      const int64_t t0 = tile_first(k);
      const int cells = tile_cells(t0);
      S* stage = reinterpret_cast<S*>(smem_raw + s * C::STAGE_BYTES);
      for (int j0 = ct; j0 < cells; j0 += 2 * NCT) {
        int jj[2] = {j0, j0 + NCT};
        bool act[2];
        bool bulk[2];
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          const int j = jj[c];
          act[c] = false;
          bulk[c] = false;
          if (j >= cells) continue;
          // core test of flat cell t0 + j by multiply-high division (the divisors sx, sy are fixed)
          const uint32_t un = uint32_t(t0 + j);
          const uint32_t px = (__umulhi(un, dv.mx) + un) >> dv.lx;
          const uint32_t rem = un - px * uint32_t(g.sx);
          const uint32_t py = (__umulhi(rem, dv.my) + rem) >> dv.ly;
          const int x = int(px) - 1, y = int(py) - 1, z = int(rem - py * uint32_t(g.sy)) - g.pz;
          if (!(x >= 0 && x < g.nx && y >= 0 && y < g.ny && z >= 0 && z < g.nz)) continue;
          const uint8_t kind = cellDyn ? cellDyn[t0 + j] : uint8_t(1);
          bulk[c] = bulk_kind(kind);
          act[c] = bulk[c] || kind == 2;
        }
        R f[2][Q];
#pragma unroll
        for (int c = 0; c < 2; ++c)
          static_for<Q>([&](auto I) {
            f[c][I] = act[c] ? Storage<S>::load(stage + I * COL + (sRun[s][I] & 15u) + jj[c]) : R(0);
          });
        bool packedDone = false;
        if constexpr (PACKED) {
          if (bulk[0] && bulk[1]) {
            float rr[2], uu[2];
            collide_bgk_x2<Q>(f, p.omega, rr, uu);
#pragma unroll
            for (int c = 0; c < 2; ++c) {
              accRho += double(rr[c]);
              accUsq += double(uu[c]);
              accMax = fmax(accMax, double(uu[c]));
              accCount += 1.0;
            }
            packedDone = true;
          }
        }
        if (!packedDone) {
#pragma unroll
          for (int c = 0; c < 2; ++c) {
            if (bulk[c]) {
              R rho, usq;
              collide<Q, R, DYN>(f[c], p, rho, usq);
              accRho += double(rho);
              accUsq += double(usq);
              accMax = fmax(accMax, double(usq));
              accCount += 1.0;
            } else if (act[c]) {
              revert<Q, R>(f[c]);
            }
          }
        }
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          if (!act[c]) continue;
          const int j = jj[c];
          static_for<Q>([&](auto I) {
            const uint32_t run = sRun[s][I];
            Storage<S>::store(stage + I * COL + (run & 15u) + j, f[c][I]);
            if (uint32_t(j) < ((run >> 4) & 0xfffu) || uint32_t(j) >= (run >> 16))
              Storage<S>::store(pop + I * g.stride + t0 + sh.s[I] + j, f[c][I]);
          });
        }
      }
      // this warp's shared-memory writes become visible to the bulk stores the producer issues
      // after the stage's empty barrier completes
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
    }
  }
  if (statPart) block_partial(accRho, accUsq, accMax, accCount, statPart);
}

// ---- fused collide + PS stream, K cells per thread ---------------------------------------
// One thread owns K cells a warp (32 cells) apart along the fastest core axis (z in 3D, y in
// 2D).  For every population it forms ONE wrapped column index; the K values are then reached
// with constant offsets (a separate per-element wrap is only needed in the rare group that
// straddles the cyclic end of the column).  All K*Q loads are issued before the first
// collision.  Periodic faces are handled by k_periodic_halo after this kernel, so the hot
// kernel carries no face logic.  Column indices are 32-bit: the column period is < 2^31.
template <int Q>
struct ColumnBases {
  void* base[Q];   // start of population column i (doubled columns: start + shift)
  uint32_t s[Q];   // current shift of column i (doubled columns: 0)
};

// Resident blocks per SM the step kernel is compiled for: the 16-bit forms move half the
// bytes per request, so they need more warps in flight to keep HBM busy.  D3Q27 at one cell
// per thread (16-bit and FP32): four blocks (64 registers, no spills; for the 16-bit forms
// 24-38 % faster than the compiler's 96-142 registers for TRT and Smagorinsky-forced BGK); at
// six blocks its 27 values spill.
template <int Q, typename S, int K> struct StepOccupancy { static constexpr int blocks = 1; };
template <> struct StepOccupancy<19, __half, 1> { static constexpr int blocks = 6; };
template <> struct StepOccupancy<19, __nv_bfloat16, 1> { static constexpr int blocks = 6; };
template <> struct StepOccupancy<27, float, 1> { static constexpr int blocks = 4; };
// FP64 D3Q19, one cell per thread: three blocks (80 registers) run 2-3 % faster than the
// compiler's choice (FP32 at two cells per thread is fastest with its own 96 registers)
template <> struct StepOccupancy<19, double, 1> { static constexpr int blocks = 3; };
template <> struct StepOccupancy<27, __half, 1> { static constexpr int blocks = 4; };
template <> struct StepOccupancy<27, __nv_bfloat16, 1> { static constexpr int blocks = 4; };
template <> struct StepOccupancy<9, __half, 1> { static constexpr int blocks = 6; };
template <> struct StepOccupancy<9, __nv_bfloat16, 1> { static constexpr int blocks = 6; };
// two cells per thread (the packed two-cell collision): 80 registers (three blocks); at four
// blocks the packed form spills and runs 8 % slower
template <> struct StepOccupancy<19, __half, 2> { static constexpr int blocks = 3; };
template <> struct StepOccupancy<19, __nv_bfloat16, 2> { static constexpr int blocks = 3; };
template <> struct StepOccupancy<9, __half, 2> { static constexpr int blocks = 4; };
template <> struct StepOccupancy<9, __nv_bfloat16, 2> { static constexpr int blocks = 4; };
// four cells per thread: 128 registers (two blocks)
template <> struct StepOccupancy<19, __half, 4> { static constexpr int blocks = 2; };
template <> struct StepOccupancy<19, __nv_bfloat16, 4> { static constexpr int blocks = 2; };
template <> struct StepOccupancy<9, __half, 4> { static constexpr int blocks = 2; };
template <> struct StepOccupancy<9, __nv_bfloat16, 4> { static constexpr int blocks = 2; };

// Load of one stored population of a 16-bit form with an L2 prefetch-size hint of 256 bytes: a
// warp-wide load reads 64 bytes of a column, and the hint lets L2 fetch the following warps'
// bytes of the same column with the same DRAM access.  (The line stays in L1: the second cell of
// a thread, 32 cells on, reads the other half of it; loads that skip L1 ran 23 % slower.)  Wider
// forms load plainly.
template <typename S> __device__ __forceinline__ S ld_column(const S* p) {
  if constexpr (sizeof(S) == 2) {
    unsigned short v;
    asm("ld.global.L2::256B.b16 %0, [%1];" : "=h"(v) : "l"(p));
    S r;
    memcpy(&r, &v, sizeof(v));
    return r;
  } else {
    return *p;
  }
}

template <int Q, typename S, int DYN, int K, bool DOUBLED, bool MAPPED>
__global__ void __launch_bounds__(256, StepOccupancy<Q, S, K>::blocks) k_collide_stream_groups(ColumnBases<Q> cols, Geometry g,
                                                               CollisionParams<typename Storage<S>::R> p,
                                                               const uint8_t* __restrict__ cellDyn,
                                                               const uint32_t* __restrict__ linkMask,
                                                               double* __restrict__ statPart, int ahead) {
  using R = typename Storage<S>::R;
  using D = Desc<Q>;
  const uint32_t P = uint32_t(g.n);
  // L2 prefetch of the block `ahead` blocks later in launch order (about one wave of resident
  // blocks on): its Q column runs, one cp.async.bulk.prefetch per column and row, issued by the
  // first Q x rows threads.  That block then finds its populations in L2 instead of waiting on
  // DRAM latency.  Doubled columns only (every run is contiguous); a prefetch changes no value.
  // The runs are widened to 16-byte bounds, which stay inside the column's two mappings.
  // Launch variant 5 passes ahead > 0 (one wave), variant 2 passes 0.  On periodic D3Q19 boxes
  // with one-row blocks it was within -4 % .. +4 % of variant 2 from box to box, on lattices with
  // a cell map and on D3Q27 it lost 12-26 % (solid cells are prefetched but never loaded), so the
  // autotuner decides.
  if constexpr (DOUBLED) {
    const unsigned tid = threadIdx.y * blockDim.x + threadIdx.x;
    if (ahead > 0 && (blockDim.x & 31u) == 0 && tid < unsigned(Q) * blockDim.y) {
      const uint64_t t = blockIdx.x + uint64_t(gridDim.x) * (blockIdx.y + uint64_t(gridDim.y) * blockIdx.z) +
                         uint64_t(ahead);
      if (t < uint64_t(gridDim.x) * gridDim.y * gridDim.z) {
        const uint32_t bx = uint32_t(t % gridDim.x);
        const uint64_t r = t / gridDim.x;
        const uint32_t by = uint32_t(r % gridDim.y), bz = uint32_t(r / gridDim.y);
        const int col = int(tid % unsigned(Q));
        const int row = int(by * blockDim.y + tid / unsigned(Q));  // y (3D) or x (2D)
        const int nf = D::d == 3 ? g.nz : g.ny, nrows = D::d == 3 ? g.ny : g.nx;
        const int zlo = int(bx * blockDim.x) * K;  // the block's cells along the fastest axis
        const int zhi = min(nf, zlo + int(blockDim.x) * K);
        if (row < nrows && zlo < zhi) {
          const uint32_t nlo = (D::d == 3) ? uint32_t((int(bz) + 1) * g.sx + (row + 1) * g.sy + zlo + 1)
                                           : uint32_t((row + 1) * g.sx + zlo + 1);
          const S* base = nullptr;
          static_for<Q>([&](auto I) {
            if (int(I) == col) base = static_cast<const S*>(cols.base[I]);
          });
          const uintptr_t a0 = reinterpret_cast<uintptr_t>(base + nlo) & ~uintptr_t(15);
          const uintptr_t a1 = (reinterpret_cast<uintptr_t>(base + nlo + (zhi - zlo)) + 15) & ~uintptr_t(15);
          asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(a0), "r"(uint32_t(a1 - a0)) : "memory");
        }
      }
    }
  }
  // The K cells of a thread lie a warp apart along the fastest axis (z0, z0 + 32, ...): each
  // warp-wide load or store then covers one contiguous run of 32 cells, which a 16-bit column
  // moves in two full sectors, instead of every instruction touching twice the sectors it uses.
  constexpr int W = 32;
  int x, y, z0, nvalid;  // nvalid: cells k < nvalid of this thread lie in the core
  bool inside;
  {
    const int gi = blockIdx.x * blockDim.x + threadIdx.x;
    const int m = blockIdx.y * blockDim.y + threadIdx.y;
    z0 = (gi / W) * (W * K) + gi % W;
    const int nf = D::d == 3 ? g.nz : g.ny;
    if constexpr (D::d == 3) {
      y = m; x = blockIdx.z;
      inside = z0 < g.nz && y < g.ny;
    } else {
      x = m; y = 0;
      inside = z0 < g.ny && x < g.nx;
    }
    nvalid = (nf - z0 + W - 1) / W;
  }
  double accRho = 0.0, accUsq = 0.0, accMax = 0.0;
  unsigned accCount = 0;
  if (inside) {
    // 3D: (x+1)*sx + (y+1)*sy + z0 + 1; 2D: the fast axis is y (sy = 1), z absent; cell k of
    // the thread is n0 + W k
    const uint32_t n0 = (D::d == 3) ? uint32_t((x + 1) * g.sx + (y + 1) * g.sy + z0 + 1)
                                    : uint32_t((x + 1) * g.sx + z0 + 1);
    // the cell kinds first: a cell without dynamics is neither loaded nor stored, so the solid
    // part of a porous medium costs no population traffic (boundary cells of kinds 3 and 4 are
    // loaded and stored by their own kernels)
    // (MAPPED: the lattice has a cell map; without one every core cell is bulk and the kernel
    // compiles to plain loads)
    uint8_t kinds[K];
    bool act[K];  // this kernel loads, collides and stores cell k
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if constexpr (MAPPED) {
        kinds[k] = (k < nvalid) ? cellDyn[n0 + W * k] : uint8_t(0);
        act[k] = stepped_kind(kinds[k]);
      } else {
        kinds[k] = (k < nvalid) ? uint8_t(1) : uint8_t(0);
        act[k] = k < nvalid;
      }
    }
    // raw loads next, all in straight-line code (the wrap is a select, not a branch), so every
    // load of the thread is in flight before the first value is used
    S raw[K][Q];
    static_for<Q>([&](auto I) {
      const S* col = static_cast<const S*>(cols.base[I]);
      if constexpr (DOUBLED) {
#pragma unroll
        for (int k = 0; k < K; ++k)
          if (act[k]) raw[k][I] = ld_column(col + n0 + W * k);
      } else {
        uint32_t idx = n0 + cols.s[I];
        idx = idx >= P ? idx - P : idx;
#pragma unroll
        for (int k = 0; k < K; ++k) {
          uint32_t ik = idx + W * k;
          if (k > 0) ik = ik >= P ? ik - P : ik;
          if (act[k]) raw[k][I] = ld_column(col + ik);
        }
      }
    });
    R f[K][Q];
#pragma unroll
    for (int k = 0; k < K; ++k)
      static_for<Q>([&](auto I) { f[k][I] = act[k] ? Storage<S>::load(&raw[k][I]) : R(0); });
    // pairs of bulk BGK cells of a 16-bit form: one packed (f32x2) collision per pair, the same
    // bits as two scalar ones.  The 16-bit forms are limited by instruction issue, where the
    // packed form halves the collision's arithmetic; the FP32 form waits on HBM, and there the
    // packed form's extra registers cost more than they save.
    constexpr bool PACKED = K >= 2 && sizeof(R) == 4 && sizeof(S) == 2 && DYN == DYN_BGK;
#pragma unroll
    for (int pr = 0; pr < (K + 1) / 2; ++pr) {
      const int k0 = 2 * pr, k1 = 2 * pr + 1;
      bool packedDone = false;
      if constexpr (PACKED) {
        if (k1 < K && bulk_kind(kinds[k0]) && bulk_kind(kinds[k1])) {
          float rr[2], uu[2];
          collide_bgk_x2<Q>(*reinterpret_cast<float(*)[2][Q]>(&f[k0]), p.omega, rr, uu);
#pragma unroll
          for (int k = 0; k < 2; ++k) {
            accRho += double(rr[k]);
            accUsq += double(uu[k]);
            accMax = fmax(accMax, double(uu[k]));
            ++accCount;
          }
          packedDone = true;
        }
      }
      if (!packedDone) {
#pragma unroll
        for (int k = k0; k <= k1; ++k) {
          if (k >= K) break;
          if (bulk_kind(kinds[k])) {
            R rho, usq;
            collide<Q, R, DYN>(f[k], p, rho, usq);
            accRho += double(rho);
            accUsq += double(usq);
            accMax = fmax(accMax, double(usq));
            ++accCount;
          } else if (kinds[k] == 2) {
            revert<Q, R>(f[k]);
          }
        }
      }
    }
    // periodic overlap (the reference's PostCollide copy, done here so a step is one launch):
    //  - rows on a periodic slower face (whole warps, ~1% of the rows) copy every leaving
    //    population to its ghost slot with the full wrap, edges and corners included;
    //  - other rows copy only what leaves across the fastest axis, which lands in the same
    //    row's ghost cell at the other end (n -+ nf).
    const int nf = D::d == 3 ? g.nz : g.ny;
    const bool slowFace = ((g.pmask & 1) && (x == 0 || x == g.nx - 1)) ||
                          (D::d == 3 && (g.pmask & 2) && (y == 0 || y == g.ny - 1));
    auto ghost_store = [&](auto I, int k, uint32_t slot) {
      S* col = static_cast<S*>(cols.base[I]);
      if constexpr (DOUBLED) {
        Storage<S>::store(col + slot, f[k][I]);
      } else {
        uint32_t idx = slot + cols.s[I];
        idx = idx >= P ? idx - P : idx;
        Storage<S>::store(col + idx, f[k][I]);
      }
    };
    if (slowFace) {
#pragma unroll
      for (int k = 0; k < K; ++k) {
        // no dynamics: nothing to carry across (see linkMask); boundary cells: their own kernels
        if (!act[k]) continue;
        const int cz0 = D::d == 3 ? z0 + W * k : 0;
        const int cy0 = D::d == 3 ? y : z0 + W * k;
        static_for<Q>([&](auto I) {
          constexpr int cx = D::C[I][0], cy = D::C[I][1], cz = D::C[I][2];
          int tx = x + cx, ty = cy0 + cy, tz = cz0 + cz;
          bool crossed = false, lost = false;
          if (tx < 0 || tx >= g.nx) { if (g.pmask & 1) { tx = tx < 0 ? tx + g.nx : tx - g.nx; crossed = true; } else lost = true; }
          if (ty < 0 || ty >= g.ny) { if (g.pmask & 2) { ty = ty < 0 ? ty + g.ny : ty - g.ny; crossed = true; } else lost = true; }
          if constexpr (D::d == 3) {
            if (tz < 0 || tz >= g.nz) { if (g.pmask & 4) { tz = tz < 0 ? tz + g.nz : tz - g.nz; crossed = true; } else lost = true; }
          }
          if (crossed && !lost) {
            const int64_t gn = int64_t(tx - cx + 1) * g.sx + int64_t(ty - cy + 1) * g.sy + (tz - cz + g.pz);
            ghost_store(I, k, uint32_t(gn));
          }
        });
      }
    } else if (g.pmask & (D::d == 3 ? 4 : 2)) {
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const int fk = z0 + W * k;
        if (!act[k] || (fk != 0 && fk != nf - 1)) continue;
        static_for<Q>([&](auto I) {
          constexpr int cf = D::d == 3 ? D::C[I][2] : D::C[I][1];
          if constexpr (cf != 0) {
            if ((cf > 0 && fk == nf - 1) || (cf < 0 && fk == 0)) {
              constexpr int cx = D::C[I][0], cy = D::C[I][1];
              bool inside = x + cx >= 0 && x + cx < g.nx;
              if constexpr (D::d == 3) inside = inside && y + cy >= 0 && y + cy < g.ny;
              if (inside) ghost_store(I, k, n0 + W * k - uint32_t(cf * nf));
            }
          }
        });
      }
    }
    // resting halfway bounce-back (BouzidiPostProcessor with q = 1/2 and a wall at rest,
    // boundary/setBouzidiBoundary.h:48-77), fused into the store: a population f_k that leaves the
    // cell towards a solid neighbour x_s = x_b + c_k is also written into the slot of x_s's
    // opposite population, which the rotation of this step carries into f_opp(k)(x_b) -- the value
    // the link kernel would copy there after the stream.  The solid cell has no dynamics, so no
    // other thread writes that slot (cells without dynamics make no stores, ghost ones included).
    if (MAPPED && linkMask) {
#pragma unroll
      for (int k = 0; k < K; ++k) {
        if (kinds[k] != kCellBulkLinked) continue;
        const uint32_t mk = linkMask[n0 + W * k];
        static_for<Q>([&](auto I) {
          if ((mk >> int(I)) & 1u) {
            constexpr int O = D::OPP[I];
            const int32_t off = int32_t(D::C[I][0] * g.sx + D::C[I][1] * g.sy + D::C[I][2]);
            S* col = static_cast<S*>(cols.base[O]);
            const uint32_t slot = n0 + W * k + uint32_t(off);
            if constexpr (DOUBLED) {
              Storage<S>::store(col + slot, f[k][I]);
            } else {
              uint32_t idx = slot + cols.s[O];
              idx = idx >= P ? idx - P : idx;
              Storage<S>::store(col + idx, f[k][I]);
            }
          }
        });
      }
    }
    static_for<Q>([&](auto I) {
      S* col = static_cast<S*>(cols.base[I]);
      if constexpr (DOUBLED) {
#pragma unroll
        for (int k = 0; k < K; ++k)
          if (act[k]) Storage<S>::store(col + n0 + W * k, f[k][I]);
      } else {
        uint32_t idx = n0 + cols.s[I];
        idx = idx >= P ? idx - P : idx;
#pragma unroll
        for (int k = 0; k < K; ++k) {
          uint32_t ik = idx + W * k;
          if (k > 0) ik = ik >= P ? ik - P : ik;
          if (act[k]) Storage<S>::store(col + ik, f[k][I]);
        }
      }
    });
  }
  if (statPart) block_partial(accRho, accUsq, accMax, double(accCount), statPart);
}

// ---- periodic overlap copy (PostCollide) --------------------------------------------------
// After the collision, every population that leaves the core across a periodic face is
// copied into the ghost cell from which the next rotation carries it into the opposite face
// -- the single-block form of the reference's periodic overlap communication
// (core/superLattice.hh:150-155, core/platform/gpu/cuda/communicator.hh:111-124).  One thread per (face
// cell, leaving population); the threads are ordered (axis, side, population, cell) so that a
// warp copies one population of consecutive face cells.  A population leaving across two faces
// at once (an edge) is copied by both faces' threads to the same ghost slot with the same value.
template <int Q> struct FaceCount { static constexpr int n = Q == 9 ? 3 : (Q == 19 ? 5 : 9); };

template <int Q, typename S>
__global__ void __launch_bounds__(256) k_periodic_halo(S* __restrict__ pop, Geometry g, Shifts<Q> sh,
                                                       int64_t cntX, int64_t cntY, int64_t cntZ) {
  using D = Desc<Q>;
  constexpr int NF = FaceCount<Q>::n;
  int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  int axis;
  int64_t plane;
  if (t < cntX) {
    axis = 0;
    plane = int64_t(g.ny) * g.nz;
  } else if ((t -= cntX) < cntY) {
    axis = 1;
    plane = int64_t(g.nx) * g.nz;
  } else if ((t -= cntY) < cntZ) {
    axis = 2;
    plane = int64_t(g.nx) * g.ny;
  } else {
    return;
  }
  const int64_t perSide = plane * NF;
  const int side = t >= perSide ? 1 : -1;  // -1: the low face (leaving with c_axis = -1)
  const int64_t rs = t >= perSide ? t - perSide : t;
  const int j = int(rs / plane);
  const int64_t cell = rs - int64_t(j) * plane;
  int x, y, z;
  if (axis == 0) {
    x = side < 0 ? 0 : g.nx - 1;
    y = int(cell / g.nz);
    z = int(cell % g.nz);
  } else if (axis == 1) {
    y = side < 0 ? 0 : g.ny - 1;
    x = int(cell / g.nz);
    z = int(cell % g.nz);
  } else {
    z = side < 0 ? 0 : g.nz - 1;
    x = int(cell / g.ny);
    y = int(cell % g.ny);
  }
  const int64_t n = int64_t(x + 1) * g.sx + int64_t(y + 1) * g.sy + (z + g.pz);
  int count = 0;
  static_for<Q>([&](auto I) {
    constexpr int cx = D::C[I][0], cy = D::C[I][1], cz = D::C[I][2];
    const int ca = axis == 0 ? cx : (axis == 1 ? cy : cz);
    if (ca != side) return;
    if (count++ != j) return;
    int tx = x + cx, ty = y + cy, tz = z + cz;
    bool lost = false;
    if (tx < 0 || tx >= g.nx) { if (g.pmask & 1) tx = tx < 0 ? tx + g.nx : tx - g.nx; else lost = true; }
    if (ty < 0 || ty >= g.ny) { if (g.pmask & 2) ty = ty < 0 ? ty + g.ny : ty - g.ny; else lost = true; }
    if constexpr (D::d == 3) {
      if (tz < 0 || tz >= g.nz) { if (g.pmask & 4) tz = tz < 0 ? tz + g.nz : tz - g.nz; else lost = true; }
    }
    if (!lost) {
      const int64_t gn = int64_t(tx - cx + 1) * g.sx + int64_t(ty - cy + 1) * g.sy + (tz - cz + g.pz);
      S* col = pop + I * g.stride;
      col[wrap_add(gn, sh.s[I], g.n)] = col[wrap_add(n, sh.s[I], g.n)];
    }
  });
}

// ---- halfway bounce-back links (PostStream) ---------------------------------------------
// f_opp(k)(x_b) = f_k(x_b + c_k) - delta, delta = 2 (c_k . u_w) t_k / c_s^2.
template <int Q, typename S>
__global__ void __launch_bounds__(256) k_bouzidi(S* __restrict__ pop, Geometry g, Shifts<Q> sh,
                                                 const uint32_t* __restrict__ cell,
                                                 const uint8_t* __restrict__ dir,
                                                 const typename Storage<S>::R* __restrict__ delta,
                                                 int64_t nLinks) {
  using R = typename Storage<S>::R;
  using D = Desc<Q>;
  const int64_t l = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (l >= nLinks) return;
  const int64_t xb = cell[l];
  const int k = dir[l];
  int64_t off = 0;
  int kopp = 0;
  static_for<Q>([&](auto I) {
    if (I == k) {
      off = D::C[I][0] * g.sx + D::C[I][1] * g.sy + D::C[I][2];
      kopp = D::OPP[I];
    }
  });
  const int64_t xs = xb + off;
  const R v = Storage<S>::load(pop + int64_t(k) * g.stride + wrap_add(xs, sh.s[k], g.n));
  Storage<S>::store(pop + int64_t(kopp) * g.stride + wrap_add(xb, sh.s[kopp], g.n),
                    v - (delta ? delta[l] : R(0)));
}

// ---- velocity / pressure boundaries (Interpolated and Local Velocity / Pressure) ----------
// A boundary cell carries a meta word (FdMeta: the cell type -- 0 flat velocity, 1 flat
// pressure, 2 external edge (3D) with imposed velocity, 3 external corner with imposed
// velocity, 4 / 5 flat velocity / pressure of a local boundary -- and the outward discrete
// normal) and four values: the imposed velocity, or {rho, tangential velocity}.  Reference: the boundary
// momenta mixed into BGKdynamics for the collision (momenta::BasicDirichletVelocityBoundaryTuple
// / BasicDirichletPressureBoundaryTuple on flat faces, FixedVelocityBoundaryTuple on edges and
// corners, dynamics/momenta/aliases.h:173-220), and the post-stream processors
// PlaneFdBoundaryProcessor3D / StraightFdBoundaryProcessor2D (boundary/boundaryPostProcessors3D.hh:
// 39-93, boundaryPostProcessors2D.hh:39-76), OuterVelocityEdgeProcessor3D (3D.hh:164-238) and
// OuterVelocityCornerProcessor3D / 2D (3D.hh:240-294, 2D.hh:276-323).
// Types 4 and 5 are the flat cells of the local boundaries (LocalVelocity / LocalPressure with
// BGK mixed in): regularised in their collision (CombinedRLBdynamics, dynamics/dynamics.h:
// 470-523), no post-processor.  Types 6 and 7 are the internal (concave) edges and corners of a
// velocity boundary, interpolated or local alike: CombinedRLBdynamics with InnerEdgeVelocityTuple3D
// / InnerCornerVelocityTuple2D / 3D (boundary/interpolatedVelocity3D.h:56-67,
// interpolatedVelocity2D.h:59-62, dynamics/momenta/aliases.h:224-243), no post-processor.
enum FdType {
  FD_FLAT_VELOCITY = 0, FD_FLAT_PRESSURE = 1, FD_EDGE_VELOCITY = 2, FD_CORNER_VELOCITY = 3,
  FD_FLAT_VELOCITY_LOCAL = 4, FD_FLAT_PRESSURE_LOCAL = 5, FD_INNER_EDGE_VELOCITY = 6, FD_INNER_CORNER_VELOCITY = 7
};

// Meta word of a boundary cell: bits 0-2 the type, bits 3-8 the outward discrete normal, two bits
// per axis (0: 0, 1: +1, 2: -1), bit 9 the RLB mixin.
struct FdMeta {
  int type;
  int n[3];         // outward normal
  int dir, orient;  // flat cells: the normal axis and its sign
  int pressure;     // flat pressure cell (interpolated or local)
  int local;        // regularised in its collision, no post-processor (types 4 to 7)
  int flat;
  int inner;        // internal edge or corner
  int rlb;          // collided by RLB (the default mixin of LocalVelocity / LocalPressure), not BGK
  __host__ __device__ __forceinline__ explicit FdMeta(uint16_t m)
      : type(m & 7), dir(0), orient(0), pressure((m & 7) == 1 || (m & 7) == 5), local((m & 7) >= 4),
        flat((m & 7) <= 1 || (m & 7) == 4 || (m & 7) == 5), inner((m & 7) >= 6), rlb((m >> 9) & 1) {
    for (int a = 0; a < 3; ++a) {
      const int code = (m >> (3 + 2 * a)) & 3;
      n[a] = code == 1 ? 1 : (code == 2 ? -1 : 0);
    }
    for (int a = 2; a >= 0; --a)
      if (n[a] != 0) {
        dir = a;
        orient = n[a];
      }
  }
  static __host__ __device__ __forceinline__ uint16_t encode(int type, const int* normal, int rlb = 0) {
    unsigned m = unsigned(type & 7) | (rlb ? 1u << 9 : 0u);
    for (int a = 0; a < 3; ++a) m |= unsigned(normal[a] == 1 ? 1 : (normal[a] == -1 ? 2 : 0)) << (3 + 2 * a);
    return uint16_t(m);
  }
};

// Plain rho = sum f + 1 (lbm::computeRho, dynamics/lbm.h:289-297: BulkDensity).
template <int Q, typename R>
__device__ __forceinline__ R bulk_rho(const R (&f)[Q]) {
  R rho = R(0);
  static_for<Q>([&](auto I) { rho += f[I]; });
  return rho + R(1);
}

// velocityBMRho (dynamics/momenta/elements.h:54-71) along axis `dir` with outward sign `orient`
template <int Q, typename R>
__device__ __forceinline__ R bm_rho(const R (&f)[Q], int dir, int orient, const R (&u)[3]) {
  using D = Desc<Q>;
  R onWall = R(0), normal = R(0);
  static_for<Q>([&](auto I) {
    constexpr int c0 = D::C[I][0], c1 = D::C[I][1], c2 = D::C[I][2];
    const int c = dir == 0 ? c0 : (dir == 1 ? c1 : c2);
    if (c == 0) onWall += f[I];
  });
  static_for<Q>([&](auto I) {
    constexpr int c0 = D::C[I][0], c1 = D::C[I][1], c2 = D::C[I][2];
    const int c = dir == 0 ? c0 : (dir == 1 ? c1 : c2);
    if (c == orient) normal += f[I];
  });
  return (R(2) * normal + onWall + R(1)) / (R(1) + R(orient) * u[dir]);
}

// rho and u of a boundary cell from its momenta.  Flat velocity: u imposed, rho = velocityBMRho
// (dynamics/momenta/elements.h:54-71) with rho_onWall summing the populations with c_d = 0 and
// rho_normal those with c_d = orientation, each in index order.  Flat pressure: rho imposed,
// the tangential velocity imposed and u_d from the populations (FixedPressureMomentum::computeU,
// elements.h:653-690).  Edge and corner: u imposed, rho = sum f + 1 (BulkDensity).  Internal
// edge and corner: u imposed, rho the mean of velocityBMRho along the normal axes
// (InnerEdgeDensity3D: the two axes after the edge axis; InnerCornerDensity2D / 3D: x, y (, z);
// elements.h:406-483).
template <int Q, typename R>
__device__ __forceinline__ void fd_momenta(const R (&f)[Q], FdMeta m, const double* __restrict__ v, R& rho,
                                           R (&u)[3]) {
  using D = Desc<Q>;
  u[0] = u[1] = u[2] = R(0);
  if (m.inner) {
    static_for<D::d>([&](auto A) { u[A] = R(v[A]); });
    if (m.type == FD_INNER_EDGE_VELOCITY) {
      int plane = 0;
      for (int a = 0; a < 3; ++a)
        if (m.n[a] == 0) plane = a;
      const int a1 = (plane + 1) % 3, a2 = (plane + 2) % 3;
      rho = (bm_rho<Q, R>(f, a1, m.n[a1], u) + bm_rho<Q, R>(f, a2, m.n[a2], u)) / R(2);
    } else if constexpr (D::d == 3) {
      rho = (bm_rho<Q, R>(f, 0, m.n[0], u) + bm_rho<Q, R>(f, 1, m.n[1], u) + bm_rho<Q, R>(f, 2, m.n[2], u)) / R(3);
    } else {
      rho = (bm_rho<Q, R>(f, 0, m.n[0], u) + bm_rho<Q, R>(f, 1, m.n[1], u)) / R(2);
    }
    return;
  }
  if (!m.flat) {
    static_for<D::d>([&](auto A) { u[A] = R(v[A]); });
    rho = bulk_rho<Q, R>(f);
    return;
  }
  R onWall = R(0), normal = R(0);
  static_for<Q>([&](auto I) {
    constexpr int c0 = D::C[I][0], c1 = D::C[I][1], c2 = D::C[I][2];
    const int c = m.dir == 0 ? c0 : (m.dir == 1 ? c1 : c2);
    if (c == 0) onWall += f[I];
  });
  static_for<Q>([&](auto I) {
    constexpr int c0 = D::C[I][0], c1 = D::C[I][1], c2 = D::C[I][2];
    const int c = m.dir == 0 ? c0 : (m.dir == 1 ? c1 : c2);
    if (c == m.orient) normal += f[I];
  });
  if (!m.pressure) {
    static_for<D::d>([&](auto A) { u[A] = R(v[A]); });
    rho = (R(2) * normal + onWall + R(1)) / (R(1) + R(m.orient) * u[m.dir]);
  } else {
    static_for<D::d>([&](auto A) { u[A] = R(v[1 + A]); });
    rho = R(v[0]);
    u[m.dir] = R(m.orient) * ((R(2) * normal + onWall + R(1)) / rho - R(1));
  }
}

// f_i^eq - w_i in the reference's generic operation order for every precision (the boundary
// cells are few; their float arithmetic is left unfused).
template <int Q, int I, typename R>
__device__ __forceinline__ R equilibrium_plain(R rho, const R (&u)[3], R uSqr) {
  constexpr R t = weight<Q, R>(I);
  const R cu = c_dot<Q, I>(u);
  return rho * t * (R(1) + R(3) * cu + R(4.5) * cu * cu - R(1.5) * uSqr) - t;
}

// u of a bulk cell through its momenta: j / rho (BulkMomentum::computeU, dynamics/momenta/
// elements.h:500-508), plus F / 2 for the forced dynamics (ForcedMomentum, elements.h:1600-1608;
// halfF is zero otherwise).
template <int Q, typename R>
__device__ __forceinline__ void bulk_velocity(const R (&f)[Q], const R (&halfF)[3], R (&u)[3]) {
  using D = Desc<Q>;
  const R rho = bulk_rho<Q, R>(f);
  u[0] = u[1] = u[2] = R(0);
  static_for<Q>([&](auto I) {
    static_for<D::d>([&](auto A) {
      constexpr int c = D::C[I][A];
      if constexpr (c == 1) u[A] += f[I];
      else if constexpr (c == -1) u[A] -= f[I];
    });
  });
  static_for<D::d>([&](auto A) {
    u[A] /= rho;
    u[A] += halfF[A];
  });
}

__device__ __forceinline__ void fd_decode(const Geometry& g, int64_t n, int& x, int& y, int& z) {
  x = int(n / g.sx) - 1;
  const int64_t r = n - int64_t(x + 1) * g.sx;
  y = int(r / g.sy) - 1;
  z = int(r - int64_t(y + 1) * g.sy) - int(g.pz);
}

// Pi of a flat local boundary cell: RegularizedBoundaryStress (BoundaryHelpers::computeStress,
// boundary/helper.h:31-81): f^neq of the populations with c_d = 0, none for i = 0, and of those
// with c_d = orientation, the latter counted twice, summed in index order.
template <int Q, typename R>
__device__ __forceinline__ void flat_stress(const R (&f)[Q], FdMeta m, R rho, const R (&u)[3], R (&pi)[6]) {
  using D = Desc<Q>;
  R uSqr = R(0);
  static_for<D::d>([&](auto A) { uSqr += u[A] * u[A]; });
  R fneq[Q];
  static_for<Q>([&](auto I) {
    constexpr int c0 = D::C[I][0], c1 = D::C[I][1], c2 = D::C[I][2];
    const int c = m.dir == 0 ? c0 : (m.dir == 1 ? c1 : c2);
    fneq[I] = (int(I) != 0 && (c == 0 || c == m.orient)) ? f[I] - equilibrium_plain<Q, I>(rho, u, uSqr) : R(0);
  });
  int iPi = 0;
  static_for<D::d>([&](auto A) {
    static_for<D::d>([&](auto B) {
      if constexpr (int(B) >= int(A)) {
        R p = R(0);
        static_for<Q>([&](auto I) {
          constexpr int cc = D::C[I][A] * D::C[I][B];
          constexpr int c0 = D::C[I][0], c1 = D::C[I][1], c2 = D::C[I][2];
          const int c = m.dir == 0 ? c0 : (m.dir == 1 ? c1 : c2);
          if (c == 0) p += R(cc) * fneq[I];
        });
        static_for<Q>([&](auto I) {
          constexpr int cc = 2 * D::C[I][A] * D::C[I][B];
          constexpr int c0 = D::C[I][0], c1 = D::C[I][1], c2 = D::C[I][2];
          const int c = m.dir == 0 ? c0 : (m.dir == 1 ? c1 : c2);
          if (c == m.orient) p += R(cc) * fneq[I];
        });
        pi[iPi++] = p;
      }
    });
  });
}

// Pi from the second moment of populations h (lbm::computeStress, dynamics/lbm.h:333-351:
// sum c_a c_b h - rho u_a u_b, less (rho - 1) / 3 on the diagonal): BulkStress (the external
// edges and corners of a local boundary), and the internal edges' and corners' completed cell.
template <int Q, typename R>
__device__ __forceinline__ void moment_stress(const R (&h)[Q], R rho, const R (&u)[3], R (&pi)[6]) {
  using D = Desc<Q>;
  int iPi = 0;
  static_for<D::d>([&](auto A) {
    static_for<D::d>([&](auto B) {
      if constexpr (int(B) >= int(A)) {
        R p = R(0);
        static_for<Q>([&](auto I) {
          constexpr int cc = D::C[I][A] * D::C[I][B];
          if constexpr (cc != 0) p += R(cc) * h[I];
        });
        p -= rho * u[A] * u[B];
        if constexpr (int(A) == int(B)) p -= R(1) / R(3) * (rho - R(1));
        pi[iPi++] = p;
      }
    });
  });
}

// Pi of an internal edge or corner (InnerEdgeStress3D / InnerCornerStress2D / 3D,
// dynamics/momenta/elements.h:1814-1897): the second moment of a copy of the cell whose unknown
// populations -- c equal to -n along every normal axis of the edge (the two axes after the edge
// axis) or corner -- are replaced by f_opp - f^eq_opp + f^eq_i.
template <int Q, typename R>
__device__ __forceinline__ void inner_stress(const R (&f)[Q], FdMeta m, R rho, const R (&u)[3], R (&pi)[6]) {
  using D = Desc<Q>;
  R uSqr = R(0);
  static_for<D::d>([&](auto A) { uSqr += u[A] * u[A]; });
  int plane = -1;  // the edge axis, none for a corner
  if (m.type == FD_INNER_EDGE_VELOCITY)
    for (int a = 0; a < 3; ++a)
      if (m.n[a] == 0) plane = a;
  R h[Q];
  static_for<Q>([&](auto I) {
    bool unknown = true;
    static_for<D::d>([&](auto A) {
      constexpr int c = D::C[I][A];
      if (int(A) != plane && c != -m.n[A]) unknown = false;
    });
    constexpr int O = D::OPP[I];
    h[I] = unknown ? f[O] - equilibrium_plain<Q, O>(rho, u, uSqr) + equilibrium_plain<Q, I>(rho, u, uSqr) : f[I];
  });
  moment_stress<Q, R>(h, rho, u, pi);
}

// Pi of a boundary cell through its momenta: flat local cells RegularizedBoundaryStress, internal
// edges and corners their inner stress, external edges and corners BulkStress
// (momenta::FixedVelocityBoundaryTuple, aliases.h:215-220).
template <int Q, typename R>
__device__ __forceinline__ void boundary_stress(const R (&f)[Q], FdMeta m, R rho, const R (&u)[3], R (&pi)[6]) {
  if (m.flat) flat_stress<Q, R>(f, m, rho, u, pi);
  else if (m.inner) inner_stress<Q, R>(f, m, rho, u, pi);
  else moment_stress<Q, R>(f, rho, u, pi);
}

// fromPiToFneq(i, Pi) (dynamics/lbm.h:247-270)
template <int Q, int I, typename R>
__device__ __forceinline__ R fneq_of_pi(const R (&pi)[6]) {
  using D = Desc<Q>;
  constexpr R t = weight<Q, R>(I);
  R fn = R(0);
  int iPi = 0;
  static_for<D::d>([&](auto A) {
    static_for<D::d>([&](auto B) {
      if constexpr (int(B) >= int(A)) {
        R toAdd = R(D::C[I][A] * D::C[I][B]);
        if constexpr (int(A) == int(B)) toAdd -= R(1) / R(3);
        else toAdd *= R(2);
        toAdd *= pi[iPi++];
        fn += toAdd;
      }
    });
  });
  fn *= t * R(3) * R(3) / R(2);
  return fn;
}

// The regularisation of a local boundary cell -- flat, or an internal edge or corner of any
// velocity boundary -- before its mixed-in collision (CombinedRLBdynamics::collide,
// dynamics/dynamics.h:505-516): Pi from the boundary momenta, then
// f_i = f_i^eq(rho, u) + fromPiToFneq(i, Pi).
template <int Q, typename R>
__device__ __forceinline__ void local_regularize(R (&f)[Q], FdMeta m, R rho, const R (&u)[3]) {
  using D = Desc<Q>;
  R uSqr = R(0);
  static_for<D::d>([&](auto A) { uSqr += u[A] * u[A]; });
  R pi[6];
  boundary_stress<Q, R>(f, m, rho, u, pi);
  static_for<Q>([&](auto I) { f[I] = equilibrium_plain<Q, I>(rho, u, uSqr) + fneq_of_pi<Q, I, R>(pi); });
}

// The RLB collision with the boundary momenta (collision::RLB, dynamics/collision.h:82-112), the
// default mixed-in dynamics of LocalVelocity / LocalPressure: f_i = f_i^eq(rho, u) +
// (1 - omega) fromPiToFneq(i, Pi), Pi from the momenta's stress.  Returns |u|^2.
template <int Q, typename R>
__device__ __forceinline__ R rlb_relax(R (&f)[Q], FdMeta m, R rho, const R (&u)[3], R omega) {
  using D = Desc<Q>;
  R uSqr = R(0);
  static_for<D::d>([&](auto A) { uSqr += u[A] * u[A]; });
  R pi[6];
  boundary_stress<Q, R>(f, m, rho, u, pi);
  static_for<Q>([&](auto I) {
    f[I] = equilibrium_plain<Q, I>(rho, u, uSqr) + (R(1) - omega) * fneq_of_pi<Q, I, R>(pi);
  });
  return uSqr;
}

// Collision of the boundary cells: BGKdynamics with the boundary momenta
// (collision::BGK::apply with lbm::bgkCollision, dynamics/collision.h:68-78, lbm.h:395-403),
// in place at the current shifts, after the bulk step kernel left these cells untouched.  A cell
// on a periodic face also refreshes the ghost slots of its leaving populations (the bulk
// kernel wrote them before this collision).  Statistics partials go after the bulk kernel's.
template <int Q, typename S>
__global__ void __launch_bounds__(256) k_fd_collide(S* __restrict__ pop, Geometry g, Shifts<Q> sh, double omega,
                                                    int64_t nFd, const uint32_t* __restrict__ fdCell,
                                                    const uint16_t* __restrict__ fdMeta,
                                                    const double* __restrict__ fdValue, double* __restrict__ statPart) {
  using R = typename Storage<S>::R;
  using D = Desc<Q>;
  const int64_t b = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  double aR = 0.0, aU = 0.0, aC = 0.0;
  if (b < nFd) {
    const int64_t n = fdCell[b];
    const FdMeta m(fdMeta[b]);
    R f[Q];
    static_for<Q>([&](auto I) { f[I] = Storage<S>::load(pop + I * g.stride + wrap_add(n, sh.s[I], g.n)); });
    R rho, u[3];
    fd_momenta<Q, R>(f, m, fdValue + 4 * b, rho, u);
    if (m.local) {  // regularised first, then collided with the momenta of the rebuilt cell
      local_regularize<Q, R>(f, m, rho, u);
      fd_momenta<Q, R>(f, m, fdValue + 4 * b, rho, u);
    }
    R uSqr = R(0);
    const R w = R(omega);
    if (m.rlb) {  // the RLB mixin of a local boundary
      uSqr = rlb_relax<Q, R>(f, m, rho, u, w);
    } else {
      static_for<D::d>([&](auto A) { uSqr += u[A] * u[A]; });
      static_for<Q>([&](auto I) {
        f[I] *= R(1) - w;
        f[I] += w * equilibrium_plain<Q, I>(rho, u, uSqr);
      });
    }
    static_for<Q>([&](auto I) { Storage<S>::store(pop + I * g.stride + wrap_add(n, sh.s[I], g.n), f[I]); });
    if (g.pmask) {
      int x, y, z;
      fd_decode(g, n, x, y, z);
      static_for<Q>([&](auto I) {
        constexpr int cx = D::C[I][0], cy = D::C[I][1], cz = D::C[I][2];
        int tx = x + cx, ty = y + cy, tz = z + cz;
        bool crossed = false, lost = false;
        if (tx < 0 || tx >= g.nx) { if (g.pmask & 1) { tx = tx < 0 ? tx + g.nx : tx - g.nx; crossed = true; } else lost = true; }
        if (ty < 0 || ty >= g.ny) { if (g.pmask & 2) { ty = ty < 0 ? ty + g.ny : ty - g.ny; crossed = true; } else lost = true; }
        if constexpr (D::d == 3) {
          if (tz < 0 || tz >= g.nz) { if (g.pmask & 4) { tz = tz < 0 ? tz + g.nz : tz - g.nz; crossed = true; } else lost = true; }
        }
        if (crossed && !lost) {
          const int64_t gn = int64_t(tx - cx + 1) * g.sx + int64_t(ty - cy + 1) * g.sy + (tz - cz + g.pz);
          Storage<S>::store(pop + I * g.stride + wrap_add(gn, sh.s[I], g.n), f[I]);
        }
      });
    }
    aR = double(rho);
    aU = double(uSqr);
    aC = 1.0;
  }
  if (statPart) block_partial(aR, aU, aU, aC, statPart);
}

// BounceBack with a wall velocity (BounceBackVelocity, dynamics/dynamics.h:629-637): the
// populations swapped (collision::Revert, collision.h:465-484), then the Nguyen-Ladd correction
// (NguyenLaddCorrection, collision.h:495-521) f_i += 2 rho u_a c_ia t_i c_s^-2 for i >= 1, one axis
// after the other, with the cell's fixed density and velocity (momenta::
// ExternalVelocityFixedDensityTuple, dynamics/momenta/aliases.h:86-91); the cell counts in the
// statistics with {rho, |u|^2}.  In place at the current shifts after the bulk step kernel, with
// the ghost slots of a cell on a periodic face refreshed as k_fd_collide does; value[4 b ...] =
// {rho, u}.  Statistics partials go after the boundary kernel's.
template <int Q, typename S>
__global__ void __launch_bounds__(256) k_bbv_collide(S* __restrict__ pop, Geometry g, Shifts<Q> sh, int64_t nB,
                                                     const uint32_t* __restrict__ bCell,
                                                     const double* __restrict__ bValue, double* __restrict__ statPart) {
  using R = typename Storage<S>::R;
  using D = Desc<Q>;
  const int64_t b = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  double aR = 0.0, aU = 0.0, aC = 0.0;
  if (b < nB) {
    const int64_t n = bCell[b];
    R f[Q];
    static_for<Q>([&](auto I) { f[I] = Storage<S>::load(pop + I * g.stride + wrap_add(n, sh.s[I], g.n)); });
    revert<Q, R>(f);
    const R rho = R(bValue[4 * b]);
    R u[3] = {R(0), R(0), R(0)};
    static_for<D::d>([&](auto A) { u[A] = R(bValue[4 * b + 1 + A]); });
    static_for<Q>([&](auto I) {
      if constexpr (I >= 1) {
        constexpr R t = weight<Q, R>(I);
        static_for<D::d>([&](auto A) { f[I] += R(2) * rho * u[A] * R(D::C[I][A]) * t * R(3); });
      }
    });
    static_for<Q>([&](auto I) { Storage<S>::store(pop + I * g.stride + wrap_add(n, sh.s[I], g.n), f[I]); });
    if (g.pmask) {
      int x, y, z;
      fd_decode(g, n, x, y, z);
      static_for<Q>([&](auto I) {
        constexpr int cx = D::C[I][0], cy = D::C[I][1], cz = D::C[I][2];
        int tx = x + cx, ty = y + cy, tz = z + cz;
        bool crossed = false, lost = false;
        if (tx < 0 || tx >= g.nx) { if (g.pmask & 1) { tx = tx < 0 ? tx + g.nx : tx - g.nx; crossed = true; } else lost = true; }
        if (ty < 0 || ty >= g.ny) { if (g.pmask & 2) { ty = ty < 0 ? ty + g.ny : ty - g.ny; crossed = true; } else lost = true; }
        if constexpr (D::d == 3) {
          if (tz < 0 || tz >= g.nz) { if (g.pmask & 4) { tz = tz < 0 ? tz + g.nz : tz - g.nz; crossed = true; } else lost = true; }
        }
        if (crossed && !lost) {
          const int64_t gn = int64_t(tx - cx + 1) * g.sx + int64_t(ty - cy + 1) * g.sy + (tz - cz + g.pz);
          Storage<S>::store(pop + I * g.stride + wrap_add(gn, sh.s[I], g.n), f[I]);
        }
      });
    }
    R uSqr = R(0);
    static_for<D::d>([&](auto A) { uSqr += u[A] * u[A]; });
    aR = double(rho);
    aU = double(uSqr);
    aC = 1.0;
  }
  if (statPart) block_partial(aR, aU, aU, aC, statPart);
}

// Post-stream pass 1: every boundary cell's velocity and density from its momenta, and its
// bulk velocity (what a neighbour reached across a periodic face sees: the reference's overlap
// copy of the cell, which carries bulk dynamics), from the populations before any cell is
// rewritten.  fdMom[7 b ...] = {u, u_bulk, rho}.
template <int Q, typename S>
__global__ void __launch_bounds__(256) k_fd_momenta(const S* __restrict__ pop, Geometry g, Shifts<Q> sh, int64_t nFd,
                                                    const uint32_t* __restrict__ fdCell,
                                                    const uint16_t* __restrict__ fdMeta,
                                                    const double* __restrict__ fdValue, double hfx, double hfy,
                                                    double hfz, double* __restrict__ fdMom) {
  using R = typename Storage<S>::R;
  const int64_t b = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (b >= nFd) return;
  const int64_t n = fdCell[b];
  R f[Q];
  static_for<Q>([&](auto I) { f[I] = Storage<S>::load(pop + I * g.stride + wrap_add(n, sh.s[I], g.n)); });
  R rho, u[3], ub[3];
  const R halfF[3] = {R(hfx), R(hfy), R(hfz)};
  fd_momenta<Q, R>(f, FdMeta(fdMeta[b]), fdValue + 4 * b, rho, u);
  bulk_velocity<Q, R>(f, halfF, ub);
  double* out = fdMom + 7 * b;
  for (int a = 0; a < 3; ++a) {
    out[a] = double(u[a]);
    out[3 + a] = double(ub[a]);
  }
  out[6] = double(rho);
}

// Post-stream passes 2 and 3: the regularised populations f_i = f_i^eq(rho, u) +
// fromPiToFneq(i, Pi) (dynamics/lbm.h:247-270) with Pi = -rho / (c_s^-2 omega) (grad u + grad u^T)
// of every boundary cell.  Velocity gradients by fd::DirectedGradients (utilities/
// finiteDifference3D.h:74-210, finiteDifference2D.h): along a non-zero normal component n_a the
// one-sided -n_a (-3 u0 + 4 u1 - u2) / 2 from the cell and the two cells inward, along the other
// axes the central (u(+1) - u(-1)) / 2.  rho: a flat cell's own (momenta); an edge extrapolates
// 2/3 (rho_B1 + rho_A1) - 1/6 (rho_B2 + rho_A2) from the cells one and two steps inward along its
// two normal axes A < B in the cyclic order after the edge axis (OuterVelocityEdgeProcessor3D::
// getNeighborRho), a 2D corner the same with A = x, B = y, a 3D corner
// 4/9 (rho_z1 + rho_y1 + rho_x1) - 1/9 (rho_z2 + rho_y2 + rho_x2).
// Pass 2 (`corners` = 0) rebuilds the flat and edge cells, whose processors have priority 0;
// pass 3 (`corners` = 1) the corners, priority 1, after them, as the reference orders the
// post-processors of a stage.  Neighbour velocities come from pass 1 (boundary cells: their
// momenta; the imposed velocity of velocity cells does not depend on the order) or from the
// populations (bulk cells, never rewritten here); cells without dynamics or with plain
// bounce-back, and padding cells, read u = 0, rho = 1 (ZeroMomentum with OneDensity /
// FixedDensity), bounce-back cells with a wall velocity their fixed velocity and density.  Neighbour densities in pass 2 come from pass 1; in pass 3 from the current
// populations, i.e. those the priority-0 processors left, as the reference's corner processor
// reads them.
template <int Q, typename S>
__global__ void __launch_bounds__(256) k_fd_regularize(S* __restrict__ pop, Geometry g, Shifts<Q> sh, double omega,
                                                       int64_t nFd, const uint32_t* __restrict__ fdCell,
                                                       const uint16_t* __restrict__ fdMeta,
                                                       const double* __restrict__ fdValue,
                                                       const uint8_t* __restrict__ cellDyn, double hfx, double hfy,
                                                       double hfz, const double* __restrict__ fdMom, int corners,
                                                       int64_t nBbv, const uint32_t* __restrict__ bbvCell,
                                                       const double* __restrict__ bbvValue,
                                                       const int32_t* __restrict__ bIdx) {
  using R = typename Storage<S>::R;
  using D = Desc<Q>;
  // One thread per boundary cell, its neighbour lookups in stages so that the loads of every
  // stage are in flight together: the boundary-list entries of all neighbours, then the cell
  // kinds of those not on the list, then the momenta of the listed ones and the fixed values,
  // then the populations of the bulk neighbours two cells at a time.  Slots 0 .. 2d-1 are the
  // velocities of the gradient (slot 2a the first neighbour along axis a, 2a + 1 the second),
  // slots 6 .. 11 the densities of an edge or corner extrapolation.  (Against one lookup after
  // the other this took the pass from 22 to 19 us a launch on a 128 x 64 x 64 channel; a warp per
  // cell, every lane repeating the cell's arithmetic, was slower at 26 us.)
  const int64_t b = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (b >= nFd) return;
  const FdMeta m(fdMeta[b]);
  if (m.local) return;  // local boundaries have no post-processor
  if ((m.type == FD_CORNER_VELOCITY) != (corners != 0)) return;
  const int64_t n = fdCell[b];
  int pos[3];
  fd_decode(g, n, pos[0], pos[1], pos[2]);
  const int ext[3] = {g.nx, g.ny, g.nz};
  const R halfF[3] = {R(hfx), R(hfy), R(hfz)};
  const double* own = fdMom + 7 * b;
  const bool flatRho = m.type == FD_FLAT_VELOCITY || m.type == FD_FLAT_PRESSURE;
  const bool edgeRule = !flatRho && (m.type == FD_EDGE_VELOCITY || D::d == 2);
  // the two normal axes A < B (in the cyclic order after the edge axis) of an edge; x, y in 2D
  int A = 0, B = 1;
  if (D::d == 3 && edgeRule) {
    int plane = 0;
    for (int a = 0; a < 3; ++a)
      if (m.n[a] == 0) plane = a;
    A = (plane + 1) % 3;
    B = (plane + 2) % 3;
  }
  constexpr int NS = 12;
  int64_t nn[NS];
  bool use[NS], wrapped[6];
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    int p[3] = {pos[0], pos[1], pos[2]};
    use[s] = false;
    if (s < 6) {
      wrapped[s] = false;
      const int a = s >> 1, second = s & 1;
      if (a < D::d) {
        use[s] = true;
        if (m.n[a] != 0) {
          p[a] -= (second ? 2 : 1) * m.n[a];
        } else {
          // across a periodic face the partner cell is read (its overlap copy carries bulk
          // dynamics); across a non-periodic one the padding cell, which has none
          const bool per = (g.pmask >> a) & 1;
          if (!second) {
            p[a] += 1;
            wrapped[s] = per && p[a] >= ext[a];
            if (wrapped[s]) p[a] -= ext[a];
          } else {
            p[a] -= 1;
            wrapped[s] = per && p[a] < 0;
            if (wrapped[s]) p[a] += ext[a];
          }
        }
      }
    } else if (!flatRho) {
      // density at the cell `step` cells inward along axis `ax`: edges (A, 1), (B, 1), (A, 2),
      // (B, 2); 3D corners (x, 1), (y, 1), (z, 1), (x, 2), (y, 2), (z, 2)
      const int r = s - 6;
      int ax = -1, step = 1;
      if (edgeRule) {
        if (r < 4) {
          ax = (r & 1) ? B : A;
          step = 1 + (r >> 1);
        }
      } else {
        ax = r % 3;
        step = 1 + r / 3;
      }
      if (ax >= 0) {
        use[s] = true;
        p[ax] -= step * m.n[ax];
      }
    }
    nn[s] = int64_t(p[0] + 1) * g.sx + int64_t(p[1] + 1) * g.sy + (p[2] + g.pz);
  }
  int32_t bi[NS];  // boundary-list entries (see lbx_lattice_s::bIdx)
#pragma unroll
  for (int s = 0; s < NS; ++s) bi[s] = use[s] ? bIdx[nn[s]] : -1;
  uint8_t kind[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) kind[s] = (use[s] && bi[s] < 0 && cellDyn) ? cellDyn[nn[s]] : uint8_t(1);
  R nv[6][3], nr[6];
  bool pend[NS];  // the value comes from the cell's populations
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    pend[s] = false;
    const int64_t jb = bi[s] <= -2 ? int64_t(-2 - bi[s]) : -1;  // bounce-back-with-velocity entry
    if (s < 6) {
      nv[s][0] = nv[s][1] = nv[s][2] = R(0);
      if (!use[s]) continue;
      if (bi[s] >= 0) {
        const double* mm = fdMom + 7 * int64_t(bi[s]) + (wrapped[s] ? 3 : 0);
        nv[s][0] = R(mm[0]);
        nv[s][1] = R(mm[1]);
        nv[s][2] = R(mm[2]);
      } else if (bulk_kind(kind[s])) {
        pend[s] = true;
      } else if (kind[s] == kCellBounceBackVelocity && jb >= 0) {  // FixedVelocityMomentum
        for (int a = 0; a < D::d; ++a) nv[s][a] = R(bbvValue[4 * jb + 1 + a]);
      }
    } else {
      nr[s - 6] = R(0);
      if (!use[s]) continue;
      if (bi[s] >= 0) {
        if (!corners) nr[s - 6] = R(fdMom[7 * int64_t(bi[s]) + 6]);
        else pend[s] = true;  // the populations the flat and edge pass left
      } else if (kind[s] == kCellBounceBackVelocity) {  // FixedDensity
        nr[s - 6] = jb >= 0 ? R(bbvValue[4 * jb]) : R(1);
      } else if (!bulk_kind(kind[s])) {
        nr[s - 6] = R(1);
      } else {
        pend[s] = true;
      }
    }
  }
  auto finish = [&](int s, const R (&f)[Q]) {
    if (s < 6) {
      bulk_velocity<Q, R>(f, halfF, nv[s]);
    } else if (bi[s] >= 0) {
      R r, v[3];
      fd_momenta<Q, R>(f, FdMeta(fdMeta[bi[s]]), fdValue + 4 * int64_t(bi[s]), r, v);
      nr[s - 6] = r;
    } else {
      nr[s - 6] = bulk_rho<Q, R>(f);
    }
  };
#pragma unroll
  for (int s0 = 0; s0 < NS; s0 += 2) {
    if (!(pend[s0] || pend[s0 + 1])) continue;
    R f0[Q], f1[Q];
    static_for<Q>([&](auto I) {
      f0[I] = pend[s0] ? Storage<S>::load(pop + I * g.stride + wrap_add(nn[s0], sh.s[I], g.n)) : R(0);
      f1[I] = pend[s0 + 1] ? Storage<S>::load(pop + I * g.stride + wrap_add(nn[s0 + 1], sh.s[I], g.n)) : R(0);
    });
    if (pend[s0]) finish(s0, f0);
    if (pend[s0 + 1]) finish(s0 + 1, f1);
  }
  R u[3] = {R(own[0]), R(own[1]), R(own[2])};
  R rho;
  if (flatRho) {
    rho = R(own[6]);
  } else if (edgeRule) {
    const R r10 = nr[0], r01 = nr[1], r20 = nr[2], r02 = nr[3];
    rho = R(2) / R(3) * (r01 + r10) - R(1) / R(6) * (r02 + r20);
  } else {
    const R r100 = nr[0], r010 = nr[1], r001 = nr[2];
    const R r200 = nr[3], r020 = nr[4], r002 = nr[5];
    rho = R(4) / R(9) * (r001 + r010 + r100) - R(1) / R(9) * (r002 + r020 + r200);
  }
  R grad[3][3] = {{R(0), R(0), R(0)}, {R(0), R(0), R(0)}, {R(0), R(0), R(0)}};
#pragma unroll
  for (int a = 0; a < D::d; ++a) {
    const R* ua = nv[2 * a];
    const R* ub = nv[2 * a + 1];
    if (m.n[a] != 0) {
      const int o = m.n[a];
      for (int iD = 0; iD < D::d; ++iD)
        grad[a][iD] = R(-o) * (((R(-3) * u[iD] + R(4) * ua[iD]) - R(1) * ub[iD]) / R(2));
    } else {
      for (int iD = 0; iD < D::d; ++iD) grad[a][iD] = (ua[iD] - ub[iD]) / R(2);
    }
  }
  const R sToPi = -rho / R(3) / R(omega);
  R pi[6];
  if constexpr (D::d == 3) {
    pi[0] = R(2) * grad[0][0] * sToPi;
    pi[3] = R(2) * grad[1][1] * sToPi;
    pi[5] = R(2) * grad[2][2] * sToPi;
    pi[1] = (grad[0][1] + grad[1][0]) * sToPi;
    pi[2] = (grad[0][2] + grad[2][0]) * sToPi;
    pi[4] = (grad[1][2] + grad[2][1]) * sToPi;
  } else {
    pi[0] = R(2) * grad[0][0] * sToPi;
    pi[2] = R(2) * grad[1][1] * sToPi;
    pi[1] = (grad[0][1] + grad[1][0]) * sToPi;
  }
  R uSqr = R(0);
  static_for<D::d>([&](auto AX) { uSqr += u[AX] * u[AX]; });
  static_for<Q>([&](auto I) {
    constexpr R t = weight<Q, R>(I);
    R fneq = R(0);
    int ip = 0;
    static_for<D::d>([&](auto AL) {
      static_for<D::d>([&](auto BE) {
        if constexpr (BE >= AL) {
          constexpr int ca = D::C[I][AL], cb = D::C[I][BE];
          R add = R(ca) * R(cb);
          if constexpr (AL == BE) add -= R(1) / R(3);
          else add *= R(2);
          add *= pi[ip++];
          fneq += add;
        }
      });
    });
    fneq *= t * R(3) * R(3) / R(2);
    Storage<S>::store(pop + I * g.stride + wrap_add(n, sh.s[I], g.n), equilibrium_plain<Q, I>(rho, u, uSqr) + fneq);
  });
}

// ---- host <-> column transfers (one population at a time through a staging buffer) -----
template <typename S, typename H>
__global__ void k_scatter_pop(S* __restrict__ col, Geometry g, int64_t shift, const H* __restrict__ src) {
  const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t ncore = int64_t(g.nx) * g.ny * g.nz;
  if (c >= ncore) return;
  const int z = int(c % g.nz);
  const int y = int((c / g.nz) % g.ny);
  const int x = int(c / (int64_t(g.nz) * g.ny));
  const int64_t n = int64_t(x + 1) * g.sx + int64_t(y + 1) * g.sy + (z + g.pz);
  Storage<S>::store(col + wrap_add(n, shift, g.n), typename Storage<S>::R(src[c]));
}

template <typename S, typename H>
__global__ void k_gather_pop(const S* __restrict__ col, Geometry g, int64_t shift, H* __restrict__ dst) {
  const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t ncore = int64_t(g.nx) * g.ny * g.nz;
  if (c >= ncore) return;
  const int z = int(c % g.nz);
  const int y = int((c / g.nz) % g.ny);
  const int x = int(c / (int64_t(g.nz) * g.ny));
  const int64_t n = int64_t(x + 1) * g.sx + int64_t(y + 1) * g.sy + (z + g.pz);
  dst[c] = H(Storage<S>::load(col + wrap_add(n, shift, g.n)));
}

// f^eq - w from moment fields (BlockLattice::iniEquilibrium, core/blockLattice.hh:201-219)
template <int Q, typename S>
__global__ void k_ini_equilibrium(S* __restrict__ pop, Geometry g, Shifts<Q> sh,
                                  const double* __restrict__ rho, const double* __restrict__ u) {
  using R = typename Storage<S>::R;
  using D = Desc<Q>;
  const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t ncore = int64_t(g.nx) * g.ny * g.nz;
  if (c >= ncore) return;
  const int z = int(c % g.nz);
  const int y = int((c / g.nz) % g.ny);
  const int x = int(c / (int64_t(g.nz) * g.ny));
  const int64_t n = int64_t(x + 1) * g.sx + int64_t(y + 1) * g.sy + (z + g.pz);
  const R r = R(rho[c]);
  R uu[3] = {R(0), R(0), R(0)};
  static_for<D::d>([&](auto A) { uu[A] = R(u[A * ncore + c]); });
  R usq = R(0);
  static_for<D::d>([&](auto A) { usq += uu[A] * uu[A]; });
  static_for<Q>([&](auto I) {
    Storage<S>::store(pop + I * g.stride + wrap_add(n, sh.s[I], g.n), equilibrium<Q, I>(r, uu, usq));
  });
}

// rho and u of every core cell, FP64 out (forced dynamics: u = j/rho + F/2)
template <int Q, typename S>
__global__ void k_moments(const S* __restrict__ pop, Geometry g, Shifts<Q> sh, int forced,
                          double fx, double fy, double fz, double* __restrict__ rho,
                          double* __restrict__ u) {
  using R = typename Storage<S>::R;
  using D = Desc<Q>;
  const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t ncore = int64_t(g.nx) * g.ny * g.nz;
  if (c >= ncore) return;
  const int z = int(c % g.nz);
  const int y = int((c / g.nz) % g.ny);
  const int x = int(c / (int64_t(g.nz) * g.ny));
  const int64_t n = int64_t(x + 1) * g.sx + int64_t(y + 1) * g.sy + (z + g.pz);
  R f[Q];
  static_for<Q>([&](auto I) { f[I] = Storage<S>::load(pop + I * g.stride + wrap_add(n, sh.s[I], g.n)); });
  R r, uu[3];
  const R F[3] = {R(fx), R(fy), R(fz)};
  if (forced) moments<Q, R, true>(f, F, r, uu);
  else moments<Q, R, false>(f, F, r, uu);
  if (rho) rho[c] = double(r);
  if (u) static_for<D::d>([&](auto A) { u[A * ncore + c] = double(uu[A]); });
}

// FP64 mass and momentum over the bulk cells: block entries {sum rho, sum j_x, sum j_y, sum j_z}
template <int Q, typename S>
__global__ void __launch_bounds__(256) k_mass_momentum(const S* __restrict__ pop, Geometry g, Shifts<Q> sh,
                                                       const uint8_t* __restrict__ cellDyn,
                                                       double* __restrict__ part) {
  using R = typename Storage<S>::R;
  using D = Desc<Q>;
  const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t ncore = int64_t(g.nx) * g.ny * g.nz;
  double v[4] = {0, 0, 0, 0};
  if (c < ncore) {
    const int z = int(c % g.nz);
    const int y = int((c / g.nz) % g.ny);
    const int x = int(c / (int64_t(g.nz) * g.ny));
    const int64_t n = int64_t(x + 1) * g.sx + int64_t(y + 1) * g.sy + (z + g.pz);
    if (!cellDyn || bulk_kind(cellDyn[n])) {
      double r = 1.0;
      static_for<Q>([&](auto I) {
        const double fi = double(Storage<S>::load(pop + I * g.stride + wrap_add(n, sh.s[I], g.n)));
        r += fi;
        static_for<D::d>([&](auto A) {
          constexpr int cc = D::C[I][A];
          if constexpr (cc != 0) v[1 + A] += cc * fi;
        });
      });
      v[0] = r;
    }
  }
  block_partial4<0>(v[0], v[1], v[2], v[3], part);
}

// Momentum exchange over the bounce-back links after the PostStream step, in the convention of
// the reference's boundary-force functor (BlockLatticePhysBoundaryForce3D::operator(),
// functors/lattice/latticePhysBoundaryForce3D.hh:85-113): for every solid cell x_s and direction
// k towards a fluid cell x_f = x_s + c_k, F -= c_k (f_k(x_f) + f_opp(k)(x_s)) on the stored values
// f - w.  A link (x_b, j) with x_b + c_j = x_s is that pair with k = opp(j), x_f = x_b, so it
// contributes c_j (f_opp(j)(x_b) + f_j(x_s)): the population the link kernel wrote back and the
// one that streamed into the solid cell.  Links whose group is not `want` (want >= 0) are skipped.
template <int Q, typename S>
__global__ void __launch_bounds__(256) k_link_force(const S* __restrict__ pop, Geometry g, Shifts<Q> sh,
                                                    const uint32_t* __restrict__ cell,
                                                    const uint8_t* __restrict__ dir,
                                                    const uint8_t* __restrict__ group, int want, int64_t nLinks,
                                                    double* __restrict__ part) {
  using D = Desc<Q>;
  const int64_t l = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  double fx = 0, fy = 0, fz = 0;
  if (l < nLinks && (want < 0 || (group && int(group[l]) == want) || (!group && want == 0))) {
    const int64_t xb = cell[l];
    const int k = dir[l];
    int64_t off = 0;
    int kopp = 0;
    double cx = 0, cy = 0, cz = 0;
    static_for<Q>([&](auto I) {
      if (I == k) {
        off = D::C[I][0] * g.sx + D::C[I][1] * g.sy + D::C[I][2];
        kopp = D::OPP[I];
        cx = D::C[I][0]; cy = D::C[I][1]; cz = D::C[I][2];
      }
    });
    const double fb = double(Storage<S>::load(pop + int64_t(kopp) * g.stride + wrap_add(xb, sh.s[kopp], g.n)));
    const double fs = double(Storage<S>::load(pop + int64_t(k) * g.stride + wrap_add(xb + off, sh.s[k], g.n)));
    const double s = fb + fs;
    fx = cx * s; fy = cy * s; fz = cz * s;
  }
  block_partial4<0>(fx, fy, fz, 0.0, part);
}

// Velocity residual against a snapshot: block entries {sum |du|^2, sum |u|^2, max |du|}; the
// snapshot is refreshed with the current velocity.
template <int Q, typename S>
__global__ void __launch_bounds__(256) k_residual(const S* __restrict__ pop, Geometry g, Shifts<Q> sh,
                                                  const uint8_t* __restrict__ cellDyn, int forced,
                                                  float fx, float fy, float fz, float* __restrict__ snap,
                                                  double* __restrict__ part) {
  using R = typename Storage<S>::R;
  using D = Desc<Q>;
  const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t ncore = int64_t(g.nx) * g.ny * g.nz;
  double du2 = 0, u2 = 0;
  if (c < ncore) {
    const int z = int(c % g.nz);
    const int y = int((c / g.nz) % g.ny);
    const int x = int(c / (int64_t(g.nz) * g.ny));
    const int64_t n = int64_t(x + 1) * g.sx + int64_t(y + 1) * g.sy + (z + g.pz);
    if (!cellDyn || bulk_kind(cellDyn[n])) {
      R f[Q];
      static_for<Q>([&](auto I) { f[I] = Storage<S>::load(pop + I * g.stride + wrap_add(n, sh.s[I], g.n)); });
      R r, uu[3];
      const R F[3] = {R(fx), R(fy), R(fz)};
      if (forced) moments<Q, R, true>(f, F, r, uu);
      else moments<Q, R, false>(f, F, r, uu);
      static_for<D::d>([&](auto A) {
        const double cur = double(uu[A]);
        const double d = cur - double(snap[A * ncore + c]);
        du2 += d * d;
        u2 += cur * cur;
        snap[A * ncore + c] = float(cur);
      });
    }
  }
  block_partial4<4>(du2, u2, sqrt(du2), 0.0, part);
}

// ---- launchers (instantiated once per storage type) ------------------------------------
struct LaunchArgs {
  void* pop;
  Geometry g;
  int64_t shift[27];
  int32_t dynamics;
  double omega, magic, smagorinsky, force[3];
  const uint8_t* cellDyn;
  StatAcc* stats;       // statistics of this step requested: totals land here
  const StatAcc* avgSrc;  // ConstRhoBGK: statistics of the previous step (average density)
  const int32_t* bIdx;      // per padded cell: boundary-list entry (lbx_lattice_s::bIdx)
  int classes;              // parameter classes in use (then the step runs kernel 1)
  double classParam[3][6];  // per class: omega, magic, smagorinsky, force[3]
  int classDyn[3];          // per class: its dynamics (DYN_*), 0 for the lattice's own
  double* statPart;     // block partials of the statistics (4 doubles per block)
  int64_t statCapacity; // blocks statPart can hold
  int blockX, blockY;
  int kernel;          // 0: pipelined shared-memory tiles, 1: one cell per thread, 2: K cells per thread
  int cellsPerThread;  // K of kernel 2 (1, 2 or 4)
  int doubled;         // columns mapped twice back to back: index n + shift needs no wrap
  int64_t flatBase;    // first tile start (multiple of 8) and end of the flat cell range
  int64_t flatEnd;
  int64_t nFd;               // velocity/pressure boundary cells
  const uint32_t* fdCell;    // their padded indices, ascending
  const uint16_t* fdMeta;    // type and outward normal (FdMeta)
  const double* fdValue;     // 4 imposed values per cell
  double* fdMom;             // 7 doubles per cell of scratch (k_fd_momenta)
  int64_t nFdCorners;        // how many of them are corners (regularised in a second pass)
  const uint32_t* linkMask;  // per padded cell: directions of resting bounce-back links (kind 7 cells)
  int64_t nBbv;              // bounce-back cells with a wall velocity
  const uint32_t* bbvCell;   // their padded indices
  const double* bbvValue;    // {rho, u} per cell
  int* err;                  // device flag: a bounded wait of a step kernel gave up
  int waitLimit;             // polls of a bounded wait before it gives up
  int faultBulk;             // test hook: the bulk-copy kernel leaves one copy unrequested
};

// Threads along the fastest axis of the K-cells step kernel: whole warps of 32 threads, each
// thread K cells a warp apart (k_collide_stream_groups).
inline int k_cells_threads(int nf, int K) { return K == 1 ? nf : (nf + 32 * K - 1) / (32 * K) * 32; }

// Blocks of 256 threads the boundary-cell collision adds to a step's statistics partials.
inline int64_t fd_blocks(int64_t nFd) { return (nFd + 255) / 256; }

// How far ahead in launch order the step kernel prefetches into L2: one wave of resident blocks
// (the block that takes over a finishing block's SM).  `cache` belongs to one kernel: per device,
// the block size it was computed for (high 32 bits) and the resident blocks (low 32 bits) in one
// atomic word, so host threads launching at once read a consistent pair.
template <typename F>
int l2_ahead_blocks(F kern, int threads, std::atomic<uint64_t> (&cache)[64]) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  const uint64_t v = cache[dev & 63].load(std::memory_order_relaxed);
  if (uint32_t(v >> 32) == uint32_t(threads)) return int(uint32_t(v));
  int perSM = 0, sms = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kern, threads, 0) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  const int blocks = perSM * sms;
  cache[dev & 63].store((uint64_t(uint32_t(threads)) << 32) | uint32_t(blocks), std::memory_order_relaxed);
  return blocks;
}

template <int Q, typename S>
cudaError_t launch_step(const LaunchArgs& a, cudaStream_t stream);
template <int Q, typename S>
cudaError_t launch_halo(const LaunchArgs& a, cudaStream_t stream);
template <int Q, typename S>
cudaError_t launch_fd_boundary(const LaunchArgs& a, cudaStream_t stream);
template <int Q, typename S>
cudaError_t launch_bouzidi(const LaunchArgs& a, const uint32_t* cell, const uint8_t* dir,
                           const void* delta, int64_t nLinks, cudaStream_t stream);
template <int Q, typename S>
cudaError_t launch_transfer(const LaunchArgs& a, int pop, const void* stage, int hostType, bool toColumns,
                            cudaStream_t stream);
template <int Q, typename S>
cudaError_t launch_ini_equilibrium(const LaunchArgs& a, const double* rho, const double* u, cudaStream_t stream);
template <int Q, typename S>
cudaError_t launch_moments(const LaunchArgs& a, double* rho, double* u, cudaStream_t stream);
// FP64 reductions: per-block entries into `part` (4 doubles per block, sized by
// reduce_blocks), combined in a fixed order into out[0..3].
inline int64_t reduce_blocks(int64_t items) { return (items + 255) / 256; }
template <int Q, typename S>
cudaError_t launch_mass_momentum(const LaunchArgs& a, double* part, double* out, cudaStream_t stream);
template <int Q, typename S>
cudaError_t launch_link_force(const LaunchArgs& a, const uint32_t* cell, const uint8_t* dir, const uint8_t* group,
                              int want, int64_t nLinks, double* part, double* out, cudaStream_t stream);
template <int Q, typename S>
cudaError_t launch_residual(const LaunchArgs& a, float* snap, double* part, double* out, cudaStream_t stream);
// Slab faces (lbx_slabs_*): gather = true copies the listed slots of this lattice into buf,
// false copies buf into the listed slots; slot e is population dir[e] of padded cell cell[e] at
// the lattice's current shift.
template <int Q, typename S>
cudaError_t launch_face_copy(const LaunchArgs& a, void* buf, const uint32_t* cell, const uint8_t* dir, int64_t n,
                             bool gather, cudaStream_t stream);

template <int Q>
inline Shifts<Q> shifts_of(const LaunchArgs& a) {
  Shifts<Q> s;
  for (int i = 0; i < Q; ++i) s.s[i] = a.shift[i];
  return s;
}

template <typename R>
inline CollisionParams<R> params_of(const LaunchArgs& a) {
  CollisionParams<R> p;
  p.omega = R(a.omega);
  p.magic = R(a.magic);
  p.smagorinsky = R(a.smagorinsky);
  for (int k = 0; k < 3; ++k) p.force[k] = R(a.force[k]);
  p.avgSrc = a.avgSrc;
  return p;
}

inline int64_t ncore_of(const Geometry& g) { return int64_t(g.nx) * g.ny * g.nz; }

#ifdef LBX_KERNEL_TU
// Launcher bodies: compiled only in the per-storage instantiation units.
template <int Q, typename S, int DYN>
cudaError_t launch_step_dyn(const LaunchArgs& a, cudaStream_t stream) {
  using R = typename Storage<S>::R;
  const Geometry& g = a.g;
  const auto sh = shifts_of<Q>(a);
  const auto p = params_of<R>(a);
  S* pop = static_cast<S*>(a.pop);
  int64_t nblocks = 0;
  if (a.kernel == 0) {
    constexpr int smem = TileCfg<Q, S>::SMEM;
    static unsigned long long configured = 0;  // one bit per device ordinal
    static int residentBlocks[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (!(configured >> (dev & 63) & 1ull)) {
      cudaError_t e = cudaFuncSetAttribute(k_collide_stream_tiled<Q, S, DYN>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
      if (e != cudaSuccess) return e;
      int perSM = 0, sms = 0;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k_collide_stream_tiled<Q, S, DYN>, TILE, smem);
      if (e != cudaSuccess) return e;
      e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      if (e != cudaSuccess) return e;
      residentBlocks[dev & 63] = (perSM > 0 ? perSM : 1) * sms;
      configured |= 1ull << (dev & 63);
    }
    const int64_t tiles = (a.flatEnd - a.flatBase + TILE - 1) / TILE;
    const int64_t grid = tiles < residentBlocks[dev & 63] ? tiles : residentBlocks[dev & 63];
    if (a.stats && grid > a.statCapacity) return cudaErrorInvalidValue;
    k_collide_stream_tiled<Q, S, DYN><<<unsigned(grid), TILE, smem, stream>>>(pop, g, sh, a.flatBase, a.flatEnd,
                                                                               tiles, p, a.cellDyn,
                                                                               a.stats ? a.statPart : nullptr);
    nblocks = grid;
  } else if (a.kernel == 3) {
    using BC = BulkCfg<Q, S>;
    static unsigned long long configured = 0;  // one bit per device ordinal
    static int residentBlocks[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (!(configured >> (dev & 63) & 1ull)) {
      cudaError_t e = cudaFuncSetAttribute(k_collide_stream_bulk<Q, S, DYN>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, BC::SMEM);
      if (e != cudaSuccess) return e;
      int perSM = 0, sms = 0;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k_collide_stream_bulk<Q, S, DYN>, BC::THREADS, BC::SMEM);
      if (e != cudaSuccess) return e;
      e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      if (e != cudaSuccess) return e;
      residentBlocks[dev & 63] = (perSM > 0 ? perSM : 1) * sms;
      configured |= 1ull << (dev & 63);
    }
    if (!a.doubled) return cudaErrorInvalidValue;  // bulk runs need the doubled columns (no wrap)
    const int64_t tiles = (a.flatEnd - a.flatBase + BC::BT - 1) / BC::BT;
    const int64_t grid = tiles < residentBlocks[dev & 63] ? tiles : residentBlocks[dev & 63];
    if (a.stats && grid > a.statCapacity) return cudaErrorInvalidValue;
    FlatDiv dv;
    FlatDiv::make(uint32_t(g.sx), dv.mx, dv.lx);
    FlatDiv::make(uint32_t(g.sy), dv.my, dv.ly);
    k_collide_stream_bulk<Q, S, DYN><<<unsigned(grid), BC::THREADS, BC::SMEM, stream>>>(
        pop, g, sh, a.flatBase, a.flatEnd, tiles, p, a.cellDyn, a.stats ? a.statPart : nullptr, a.err, dv,
        a.waitLimit, a.faultBulk);
    nblocks = grid;
  } else if (a.kernel == 4) {
    using WC = WsCfg<Q, S>;
    static unsigned long long configured = 0;  // one bit per device ordinal
    static int residentBlocks[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (!(configured >> (dev & 63) & 1ull)) {
      cudaError_t e = cudaFuncSetAttribute(k_collide_stream_ws<Q, S, DYN>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, WC::SMEM);
      if (e != cudaSuccess) return e;
      int perSM = 0, sms = 0;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k_collide_stream_ws<Q, S, DYN>, WC::THREADS, WC::SMEM);
      if (e != cudaSuccess) return e;
      e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      if (e != cudaSuccess) return e;
      residentBlocks[dev & 63] = (perSM > 0 ? perSM : 1) * sms;
      configured |= 1ull << (dev & 63);
    }
    if (!a.doubled) return cudaErrorInvalidValue;  // bulk runs need the doubled columns (no wrap)
    const int64_t tiles = (a.flatEnd - a.flatBase + WC::BT - 1) / WC::BT;
    const int64_t grid = tiles < residentBlocks[dev & 63] ? tiles : residentBlocks[dev & 63];
    if (a.stats && grid > a.statCapacity) return cudaErrorInvalidValue;
    FlatDiv dv;
    FlatDiv::make(uint32_t(g.sx), dv.mx, dv.lx);
    FlatDiv::make(uint32_t(g.sy), dv.my, dv.ly);
    k_collide_stream_ws<Q, S, DYN><<<unsigned(grid), WC::THREADS, WC::SMEM, stream>>>(
        pop, g, sh, a.flatBase, a.flatEnd, tiles, p, a.cellDyn, a.stats ? a.statPart : nullptr, a.err, dv,
        a.waitLimit);
    nblocks = grid;
  } else if (a.kernel == 1) {
    dim3 block(a.blockX, a.blockY, 1);
    dim3 grid;
    if (Desc<Q>::d == 3) grid = dim3((g.nz + a.blockX - 1) / a.blockX, (g.ny + a.blockY - 1) / a.blockY, g.nx);
    else grid = dim3((g.ny + a.blockX - 1) / a.blockX, (g.nx + a.blockY - 1) / a.blockY, 1);
    nblocks = int64_t(grid.x) * grid.y * grid.z;
    if (a.stats && nblocks > a.statCapacity) return cudaErrorInvalidValue;
    ClassParams<R> cls;
    cls.used = a.classes;
    for (int c = 0; c < 3; ++c) cls.dyn[c] = a.classDyn[c];
    for (int c = 0; c < 3; ++c) {
      cls.p[c] = p;
      cls.p[c].omega = R(a.classParam[c][0]);
      cls.p[c].magic = R(a.classParam[c][1]);
      cls.p[c].smagorinsky = R(a.classParam[c][2]);
      for (int k = 0; k < 3; ++k) cls.p[c].force[k] = R(a.classParam[c][3 + k]);
    }
    k_collide_stream<Q, S, DYN><<<grid, block, 0, stream>>>(pop, g, sh, p, a.cellDyn, a.stats ? a.statPart : nullptr,
                                                            cls);
  } else {
    ColumnBases<Q> cols;
    for (int i = 0; i < Q; ++i) {
      cols.base[i] = pop + int64_t(i) * g.stride + (a.doubled ? a.shift[i] : 0);
      cols.s[i] = a.doubled ? 0u : uint32_t(a.shift[i]);
    }
    const int K = a.cellsPerThread;
    const int nf = Desc<Q>::d == 3 ? g.nz : g.ny;
    const int groups = k_cells_threads(nf, K);
    dim3 block(a.blockX, a.blockY, 1);
    dim3 grid;
    if (Desc<Q>::d == 3) grid = dim3((groups + a.blockX - 1) / a.blockX, (g.ny + a.blockY - 1) / a.blockY, g.nx);
    else grid = dim3((groups + a.blockX - 1) / a.blockX, (g.nx + a.blockY - 1) / a.blockY, 1);
    nblocks = int64_t(grid.x) * grid.y * grid.z;
    if (a.stats && nblocks > a.statCapacity) return cudaErrorInvalidValue;
    double* part = a.stats ? a.statPart : nullptr;
    auto go = [&](auto kk, auto doubled, auto mapped) {
      auto kern =
          k_collide_stream_groups<Q, S, DYN, decltype(kk)::value, decltype(doubled)::value, decltype(mapped)::value>;
      static std::atomic<uint64_t> aheadCache[64] = {};  // one per instantiation of this lambda, i.e. per kernel
      int ahead = 0;
      if constexpr (decltype(doubled)::value)
        if (a.kernel == 5) ahead = l2_ahead_blocks(kern, int(block.x * block.y), aheadCache);
      kern<<<grid, block, 0, stream>>>(cols, g, p, a.cellDyn, a.linkMask, part, ahead);
    };
    auto go_k = [&](auto kk) {
      if (a.doubled) {
        if (a.cellDyn) go(kk, std::true_type{}, std::true_type{});
        else go(kk, std::true_type{}, std::false_type{});
      } else {
        if (a.cellDyn) go(kk, std::false_type{}, std::true_type{});
        else go(kk, std::false_type{}, std::false_type{});
      }
    };
    switch (K) {
    case 1: go_k(std::integral_constant<int, 1>{}); break;
    case 2: go_k(std::integral_constant<int, 2>{}); break;
    case 4:
      // four cells per thread: the 16-bit forms only (their per-cell arithmetic, not HBM, is
      // what limits them; four cells share one thread's index and address work)
      if constexpr (sizeof(S) == 2) {
        go_k(std::integral_constant<int, 4>{});
        break;
      }
      return cudaErrorInvalidValue;
    default: return cudaErrorInvalidValue;
    }
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  int64_t fdb = 0;
  if (a.nFd > 0) {
    fdb = fd_blocks(a.nFd);
    if (a.stats && nblocks + fdb > a.statCapacity) return cudaErrorInvalidValue;
    k_fd_collide<Q, S><<<unsigned(fdb), 256, 0, stream>>>(pop, g, sh, a.omega, a.nFd, a.fdCell, a.fdMeta, a.fdValue,
                                                          a.stats ? a.statPart + 4 * nblocks : nullptr);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  int64_t bbb = 0;
  if (a.nBbv > 0) {
    bbb = fd_blocks(a.nBbv);
    if (a.stats && nblocks + fdb + bbb > a.statCapacity) return cudaErrorInvalidValue;
    k_bbv_collide<Q, S><<<unsigned(bbb), 256, 0, stream>>>(pop, g, sh, a.nBbv, a.bbvCell, a.bbvValue,
                                                           a.stats ? a.statPart + 4 * (nblocks + fdb) : nullptr);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (!a.stats) return cudaSuccess;
  k_stats_finalize<<<1, kFinalizeThreads, 0, stream>>>(a.statPart, nblocks + fdb + bbb, a.stats);
  return cudaGetLastError();
}
// Post-stream regularisation of the boundary cells: momenta, then flat faces and edges, then
// corners (see k_fd_regularize).
template <int Q, typename S>
cudaError_t launch_fd_boundary(const LaunchArgs& a, cudaStream_t stream) {
  if (a.nFd <= 0) return cudaSuccess;
  const unsigned blocks = unsigned(fd_blocks(a.nFd));
  S* pop = static_cast<S*>(a.pop);
  const auto sh = shifts_of<Q>(a);
  // forced bulk neighbours report j / rho + F / 2 (ForcedMomentum)
  const bool forced = a.dynamics == DYN_FORCED_BGK || a.dynamics == DYN_FORCED_SMAGORINSKY;
  const double hf[3] = {forced ? 0.5 * a.force[0] : 0.0, forced ? 0.5 * a.force[1] : 0.0, forced ? 0.5 * a.force[2] : 0.0};
  k_fd_momenta<Q, S><<<blocks, 256, 0, stream>>>(pop, a.g, sh, a.nFd, a.fdCell, a.fdMeta, a.fdValue, hf[0], hf[1],
                                                 hf[2], a.fdMom);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  for (int corners = 0; corners < (a.nFdCorners > 0 ? 2 : 1); ++corners) {
    k_fd_regularize<Q, S><<<blocks, 256, 0, stream>>>(pop, a.g, sh, a.omega, a.nFd, a.fdCell, a.fdMeta, a.fdValue,
                                                      a.cellDyn, hf[0], hf[1], hf[2], a.fdMom, corners, a.nBbv,
                                                      a.bbvCell, a.bbvValue, a.bIdx);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}
// Periodic overlap copy after the collision (no launch for a lattice without periodic axes).
template <int Q, typename S>
cudaError_t launch_halo(const LaunchArgs& a, cudaStream_t stream) {
  const Geometry& g = a.g;
  if (g.pmask == 0) return cudaSuccess;
  const auto sh = shifts_of<Q>(a);
  S* pop = static_cast<S*>(a.pop);
  constexpr int NF = FaceCount<Q>::n;
  // the K-cells step kernel (variant 2) does the whole overlap copy itself
  if (a.kernel == 2 || a.kernel == 5) return cudaSuccess;
  const int mask = g.pmask;
  const int64_t cntX = (mask & 1) ? 2 * NF * int64_t(g.ny) * g.nz : 0;
  const int64_t cntY = (mask & 2) ? 2 * NF * int64_t(g.nx) * g.nz : 0;
  const int64_t cntZ = (mask & 4) ? 2 * NF * int64_t(g.nx) * g.ny : 0;
  const int64_t total = cntX + cntY + cntZ;
  k_periodic_halo<Q, S><<<unsigned((total + 255) / 256), 256, 0, stream>>>(pop, g, sh, cntX, cntY, cntZ);
  return cudaGetLastError();
}
template <int Q, typename S>
cudaError_t launch_step(const LaunchArgs& a, cudaStream_t stream) {
  switch (a.dynamics) {
  case DYN_BGK: return launch_step_dyn<Q, S, DYN_BGK>(a, stream);
  case DYN_TRT: return launch_step_dyn<Q, S, DYN_TRT>(a, stream);
  case DYN_SMAGORINSKY: return launch_step_dyn<Q, S, DYN_SMAGORINSKY>(a, stream);
  case DYN_FORCED_BGK: return launch_step_dyn<Q, S, DYN_FORCED_BGK>(a, stream);
  case DYN_FORCED_SMAGORINSKY: return launch_step_dyn<Q, S, DYN_FORCED_SMAGORINSKY>(a, stream);
  case DYN_CONST_RHO: return launch_step_dyn<Q, S, DYN_CONST_RHO>(a, stream);
  default: return cudaErrorInvalidValue;
  }
}
template <int Q, typename S>
cudaError_t launch_bouzidi(const LaunchArgs& a, const uint32_t* cell, const uint8_t* dir,
                                 const void* delta, int64_t nLinks, cudaStream_t stream) {
  using R = typename Storage<S>::R;
  if (nLinks <= 0) return cudaSuccess;
  const int64_t blocks = (nLinks + 255) / 256;
  k_bouzidi<Q, S><<<unsigned(blocks), 256, 0, stream>>>(static_cast<S*>(a.pop), a.g, shifts_of<Q>(a), cell, dir,
                                                        static_cast<const R*>(delta), nLinks);
  return cudaGetLastError();
}
template <int Q, typename S>
cudaError_t launch_transfer(const LaunchArgs& a, int i, const void* stage, int hostType, bool toColumns,
                                  cudaStream_t stream) {
  const int64_t nc = ncore_of(a.g);
  const unsigned blocks = unsigned((nc + 255) / 256);
  S* col = static_cast<S*>(a.pop) + int64_t(i) * a.g.stride;
  if (toColumns) {
    if (hostType == 0) k_scatter_pop<S, double><<<blocks, 256, 0, stream>>>(col, a.g, a.shift[i], static_cast<const double*>(stage));
    else k_scatter_pop<S, float><<<blocks, 256, 0, stream>>>(col, a.g, a.shift[i], static_cast<const float*>(stage));
  } else {
    if (hostType == 0) k_gather_pop<S, double><<<blocks, 256, 0, stream>>>(col, a.g, a.shift[i], static_cast<double*>(const_cast<void*>(stage)));
    else k_gather_pop<S, float><<<blocks, 256, 0, stream>>>(col, a.g, a.shift[i], static_cast<float*>(const_cast<void*>(stage)));
  }
  return cudaGetLastError();
}
template <int Q, typename S>
cudaError_t launch_ini_equilibrium(const LaunchArgs& a, const double* rho, const double* u,
                                         cudaStream_t stream) {
  const unsigned blocks = unsigned((ncore_of(a.g) + 255) / 256);
  k_ini_equilibrium<Q, S><<<blocks, 256, 0, stream>>>(static_cast<S*>(a.pop), a.g, shifts_of<Q>(a), rho, u);
  return cudaGetLastError();
}
template <int Q, typename S>
cudaError_t launch_moments(const LaunchArgs& a, double* rho, double* u, cudaStream_t stream) {
  const unsigned blocks = unsigned((ncore_of(a.g) + 255) / 256);
  const int forced = (a.dynamics == DYN_FORCED_BGK || a.dynamics == DYN_FORCED_SMAGORINSKY);
  k_moments<Q, S><<<blocks, 256, 0, stream>>>(static_cast<const S*>(a.pop), a.g, shifts_of<Q>(a), forced,
                                              a.force[0], a.force[1], a.force[2], rho, u);
  return cudaGetLastError();
}
template <int Q, typename S>
cudaError_t launch_mass_momentum(const LaunchArgs& a, double* part, double* out, cudaStream_t stream) {
  const int64_t blocks = reduce_blocks(ncore_of(a.g));
  k_mass_momentum<Q, S><<<unsigned(blocks), 256, 0, stream>>>(static_cast<const S*>(a.pop), a.g, shifts_of<Q>(a),
                                                              a.cellDyn, part);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_finalize4<0><<<1, kFinalizeThreads, 0, stream>>>(part, blocks, out);
  return cudaGetLastError();
}
template <int Q, typename S>
cudaError_t launch_link_force(const LaunchArgs& a, const uint32_t* cell, const uint8_t* dir, const uint8_t* group,
                              int want, int64_t nLinks, double* part, double* out, cudaStream_t stream) {
  const int64_t blocks = reduce_blocks(nLinks);
  if (nLinks > 0) {
    k_link_force<Q, S><<<unsigned(blocks), 256, 0, stream>>>(static_cast<const S*>(a.pop), a.g, shifts_of<Q>(a), cell,
                                                             dir, group, want, nLinks, part);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  k_finalize4<0><<<1, kFinalizeThreads, 0, stream>>>(part, blocks, out);
  return cudaGetLastError();
}
template <int Q, typename S>
cudaError_t launch_residual(const LaunchArgs& a, float* snap, double* part, double* out, cudaStream_t stream) {
  const int64_t blocks = reduce_blocks(ncore_of(a.g));
  const int forced = (a.dynamics == DYN_FORCED_BGK || a.dynamics == DYN_FORCED_SMAGORINSKY);
  k_residual<Q, S><<<unsigned(blocks), 256, 0, stream>>>(static_cast<const S*>(a.pop), a.g, shifts_of<Q>(a), a.cellDyn,
                                                         forced, float(a.force[0]), float(a.force[1]),
                                                         float(a.force[2]), snap, part);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_finalize4<4><<<1, kFinalizeThreads, 0, stream>>>(part, blocks, out);
  return cudaGetLastError();
}
// One thread per listed slot of a slab face: gather (populations -> buffer) on the lattice that
// sends, scatter (buffer -> populations) on the lattice that receives.  The shift of each
// population is taken from the kernel's parameters, so the lists hold cells, not addresses.
template <int Q, typename S>
__global__ void __launch_bounds__(256) k_face_copy(S* __restrict__ pop, int64_t stride, int64_t period, Shifts<Q> sh,
                                                   S* __restrict__ buf, const uint32_t* __restrict__ cell,
                                                   const uint8_t* __restrict__ dir, int64_t n, int gather) {
  const int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const int i = dir[e];
  int64_t shift = 0;
  static_for<Q>([&](auto I) {
    if (int(I) == i) shift = sh.s[I];
  });
  S* slot = pop + int64_t(i) * stride + wrap_add(int64_t(cell[e]), shift, period);
  if (gather) buf[e] = *slot;
  else *slot = buf[e];
}
template <int Q, typename S>
cudaError_t launch_face_copy(const LaunchArgs& a, void* buf, const uint32_t* cell, const uint8_t* dir, int64_t n,
                             bool gather, cudaStream_t stream) {
  if (n <= 0) return cudaSuccess;
  k_face_copy<Q, S><<<unsigned((n + 255) / 256), 256, 0, stream>>>(static_cast<S*>(a.pop), a.g.stride, a.g.n,
                                                                    shifts_of<Q>(a), static_cast<S*>(buf), cell, dir,
                                                                    n, gather ? 1 : 0);
  return cudaGetLastError();
}
// Explicit instantiation of every launcher for one (descriptor, storage) pair.
#define LBX_INSTANTIATE(Q, S)                                                                          \
  template cudaError_t launch_step<Q, S>(const LaunchArgs&, cudaStream_t);                            \
  template cudaError_t launch_halo<Q, S>(const LaunchArgs&, cudaStream_t);                            \
  template cudaError_t launch_fd_boundary<Q, S>(const LaunchArgs&, cudaStream_t);                     \
  template cudaError_t launch_bouzidi<Q, S>(const LaunchArgs&, const uint32_t*, const uint8_t*,       \
                                            const void*, int64_t, cudaStream_t);                      \
  template cudaError_t launch_transfer<Q, S>(const LaunchArgs&, int, const void*, int, bool, cudaStream_t); \
  template cudaError_t launch_ini_equilibrium<Q, S>(const LaunchArgs&, const double*, const double*, cudaStream_t); \
  template cudaError_t launch_moments<Q, S>(const LaunchArgs&, double*, double*, cudaStream_t);       \
  template cudaError_t launch_mass_momentum<Q, S>(const LaunchArgs&, double*, double*, cudaStream_t); \
  template cudaError_t launch_link_force<Q, S>(const LaunchArgs&, const uint32_t*, const uint8_t*,    \
                                               const uint8_t*, int, int64_t, double*, double*,         \
                                               cudaStream_t);                                          \
  template cudaError_t launch_residual<Q, S>(const LaunchArgs&, float*, double*, double*, cudaStream_t); \
  template cudaError_t launch_face_copy<Q, S>(const LaunchArgs&, void*, const uint32_t*, const uint8_t*, int64_t, \
                                              bool, cudaStream_t);
#endif  // LBX_KERNEL_TU

}  // namespace lbx
