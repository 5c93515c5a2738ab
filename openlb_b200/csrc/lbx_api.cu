// C ABI of liblbx.so: lattice handles, host-side setters and the step driver.
// The kernels live in lbx_kernels.cuh and are instantiated per storage type in
// lbx_inst_*.cu.  See include/lbx.h for the contract of every entry point.
#include <cuda.h>  // driver-API types; the functions are resolved at run time (no libcuda link)
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/lbx.h"
#include "lbx_kernels.cuh"
#include "lbx_test.h"

using namespace lbx;

namespace {

thread_local std::string g_error;

int fail(int code, const std::string& msg) {
  g_error = msg;
  return code;
}

#define LBX_CUDA_TRY(expr)                                                                   \
  do {                                                                                       \
    cudaError_t e_ = (expr);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return fail(e_ == cudaErrorMemoryAllocation ? LBX_ERR_OUT_OF_MEMORY : LBX_ERR_CUDA,    \
                  std::string(#expr) + ": " + cudaGetErrorString(e_));                       \
  } while (0)

// Makes the lattice's device current for the duration of a call and restores the caller's.
struct DeviceGuard {
  int previous = -1;
  bool ok = false;
  explicit DeviceGuard(int device) {
    if (cudaGetDevice(&previous) != cudaSuccess) previous = -1;
    ok = (previous == device) || (cudaSetDevice(device) == cudaSuccess);
  }
  ~DeviceGuard() {
    if (previous >= 0) cudaSetDevice(previous);
  }
};

size_t storage_bytes(int storage) {
  switch (storage) {
  case LBX_F64: return 8;
  case LBX_F32: return 4;
  case LBX_F16DEV: return 2;
  case LBX_BF16DEV: return 2;
  default: return 0;
  }
}

const int* velocity(int q, int i) {
  static const int c9[9][3] = {{0, 0, 0},  {-1, 1, 0}, {-1, 0, 0}, {-1, -1, 0}, {0, -1, 0},
                               {1, -1, 0}, {1, 0, 0},  {1, 1, 0},  {0, 1, 0}};
  switch (q) {
  case 9: return c9[i];
  case 19: return Desc<19>::C[i];
  default: return Desc<27>::C[i];
  }
}
double weight_of(int q, int i) {
  switch (q) {
  case 9: return double(Desc<9>::WN[i]) / double(Desc<9>::WD[i]);
  case 19: return double(Desc<19>::WN[i]) / double(Desc<19>::WD[i]);
  default: return double(Desc<27>::WN[i]) / double(Desc<27>::WD[i]);
  }
}

}  // namespace

namespace lbx {
int set_error(int code, const std::string& msg) { return fail(code, msg); }

// lbx_test_fault's setting (process-wide; for tests only)
TestFault& test_fault() {
  static TestFault f;
  return f;
}
bool test_allocation_fails() {
  TestFault& f = test_fault();
  if (f.kind != LBX_TEST_ALLOCATION || f.param <= 0) return false;
  --f.param;
  return true;
}
// launch variants that run the K-cells step kernel (variant 5 adds its L2 prefetch)
inline bool groups_kernel(int variant) { return variant == 2 || variant == 5; }
// lbx_normals.cu
int discrete_normals(int q, const int32_t core[3], const int32_t periodic[3], const int32_t* material,
                     int32_t boundary, int32_t n_fluid, const int32_t* fluid, int32_t n_outside,
                     const int32_t* outside, std::vector<int64_t>& cells, std::vector<int32_t>& types,
                     std::vector<int32_t>& normals);
}  // namespace lbx

// A velocity / pressure boundary cell as set through the ABI.
struct FdHostCell {
  int64_t core = 0;
  int32_t kind = 0, type = 0;
  int32_t n[3] = {0, 0, 0};
  double v[4] = {0, 0, 0, 0};
};

struct lbx_lattice_s {
  int q = 0, d = 0, storage = 0, device = 0;
  int core[3] = {1, 1, 1};
  int padded[3] = {1, 1, 1};
  int periodic[3] = {0, 0, 0};
  int64_t n = 0, stride = 0, period = 0, ncore = 0;
  bool doubled = false;                      // columns mapped twice back to back (see alloc_columns)
  unsigned long long vmmHandles[27] = {};
  unsigned long long vmmBase = 0, vmmBytes = 0;
  int64_t shift[27] = {};
  void* pop = nullptr;
  uint8_t* cellDyn = nullptr;
  uint32_t* linkCell = nullptr;
  uint8_t* linkDir = nullptr;
  void* linkDelta = nullptr;
  uint8_t* linkGroup = nullptr;             // per link: index of the solid it faces
  int64_t nLinks = 0;
  // host copies: the cell map as set (public ids incl. the boundary list's marks; empty = bulk
  // everywhere) and the links (padded cell, direction, wall term) in their device order
  std::vector<uint8_t> hostMap;
  uint64_t mapVersion = 0;  // counts refresh_cell_map calls (slab face lists depend on the map)
  std::vector<uint32_t> linkHostCell;
  std::vector<uint8_t> linkHostDir;
  std::vector<double> linkHostDelta;
  // resting links fused into the K-cells step kernel (one direction bit per padded cell) and the
  // links the link kernel still applies after that kernel (moving walls, unusual neighbours)
  // bounce-back cells with a wall velocity (lbx_set_bounce_back_velocity): padded cells ascending
  // and {rho, u} per cell
  int64_t nBbv = 0;
  uint32_t* bbvCell = nullptr;
  double* bbvValue = nullptr;
  std::vector<uint32_t> bbvHostCells;
  // per padded cell: its index in the boundary list (>= 0), -2 - its index in the bounce-back
  // velocity list, or -1 (the boundary kernels' neighbour lookups); null without such cells
  int32_t* bIdx = nullptr;
  uint32_t* linkMask = nullptr;
  uint32_t* restCell = nullptr;
  uint8_t* restDir = nullptr;
  void* restDelta = nullptr;
  int64_t nRest = 0;
  // flat-face velocity / pressure boundary cells (lbx_set_fd_boundaries)
  int64_t nFd = 0;
  uint32_t* fdCell = nullptr;
  uint16_t* fdMeta = nullptr;
  double* fdValue = nullptr;
  double* fdMom = nullptr;
  std::vector<uint32_t> fdHostCells;  // padded indices, to re-mark after lbx_set_cell_dynamics
  std::vector<FdHostCell> fdHost;     // the list as set (core cells ascending)
  int64_t nFdCorners = 0;             // corner cells among them (second regularisation pass)
  StatAcc* stats = nullptr;
  double* statPart = nullptr;        // per-block statistics partials
  int64_t statCapacity = 0;          // blocks statPart holds
  double* reduceAcc = nullptr;       // 8 doubles + 1 ull of scratch for reductions
  double* reducePart = nullptr;      // per-block entries of the FP64 reductions (4 doubles each)
  int* devErr = nullptr;             // set by a step kernel whose bounded wait gave up
  int64_t reducePartCapacity = 0;    // blocks reducePart holds
  float* residualSnap = nullptr;
  void* stage = nullptr;             // ncore doubles
  int dynamics = LBX_BGK;
  lbx_params params{1.0, 0.25, 0.12, {0, 0, 0}};
  // parameter classes 1..3 of the bulk dynamics (lbx_set_dynamics_class): bit c - 1 set when
  // class c is defined
  int classMask = 0;
  lbx_params classParams[3] = {};
  int classDyn[3] = {0, 0, 0};  // a class's own dynamics (lbx_set_dynamics_class_kind), 0: the lattice's
  int blockX = 256, blockY = 1;
  int kernel = 2;
  int cellsPerThread = 1;
  int64_t bytes = 0;
  // optional per-kernel event timing (lbx_set_kernel_timing)
  bool timing = false;
  std::vector<cudaEvent_t> eventPool;
  std::vector<cudaEvent_t> pending;  // groups of 4: before/after collision, after halo, after links
  double timedMs[3] = {0, 0, 0};
  int64_t timedLaunches[3] = {0, 0, 0};
};

namespace {

Geometry geometry_of(const lbx_lattice_s* L) {
  Geometry g;
  g.n = L->period;  // cyclic period of every column (>= padded cells)
  g.stride = L->stride;
  g.sy = (L->d == 3) ? L->padded[2] : 1;
  g.sx = int64_t(L->padded[1]) * ((L->d == 3) ? L->padded[2] : 1);
  g.nx = L->core[0];
  g.ny = L->core[1];
  g.nz = (L->d == 3) ? L->core[2] : 1;
  g.pz = (L->d == 3) ? 1 : 0;
  g.pmask = (L->periodic[0] ? 1 : 0) | (L->periodic[1] ? 2 : 0) | ((L->d == 3 && L->periodic[2]) ? 4 : 0);
  return g;
}

LaunchArgs args_of(const lbx_lattice_s* L) {
  LaunchArgs a{};
  a.pop = L->pop;
  a.g = geometry_of(L);
  for (int i = 0; i < L->q; ++i) a.shift[i] = L->shift[i];
  a.dynamics = L->dynamics;
  a.omega = L->params.omega;
  a.magic = L->params.magic;
  a.smagorinsky = L->params.smagorinsky;
  for (int k = 0; k < 3; ++k) a.force[k] = L->params.force[k];
  a.cellDyn = L->cellDyn;
  a.stats = nullptr;
  a.avgSrc = L->dynamics == LBX_CONST_RHO_BGK ? L->stats : nullptr;
  a.blockX = L->blockX;
  a.blockY = L->blockY;
  a.kernel = L->kernel;
  a.doubled = L->doubled ? 1 : 0;
  a.cellsPerThread = L->cellsPerThread;
  const Geometry& g = a.g;
  const int64_t first = g.sx + g.sy + g.pz;
  const int64_t last = int64_t(g.nx) * g.sx + int64_t(g.ny) * g.sy + (g.nz - 1 + g.pz);
  a.flatBase = first / 8 * 8;
  a.flatEnd = last + 1;
  a.nFd = L->nFd;
  a.fdCell = L->fdCell;
  a.fdMeta = L->fdMeta;
  a.fdValue = L->fdValue;
  a.fdMom = L->fdMom;
  a.nFdCorners = L->nFdCorners;
  a.linkMask = groups_kernel(L->kernel) ? L->linkMask : nullptr;
  a.nBbv = L->nBbv;
  a.bbvCell = L->bbvCell;
  a.bbvValue = L->bbvValue;
  a.bIdx = L->bIdx;
  a.err = L->devErr;
  const TestFault& tf = test_fault();
  a.waitLimit = (tf.kind == LBX_TEST_BULK_COPY && tf.param > 0) ? tf.param : (1 << 22);
  a.faultBulk = tf.kind == LBX_TEST_BULK_COPY ? 1 : 0;
  a.classes = L->classMask != 0 ? 1 : 0;
  for (int c = 0; c < 3; ++c) {  // a class never defined collides with the lattice's own parameters
    const lbx_params& pc = (L->classMask >> c & 1) ? L->classParams[c] : L->params;
    a.classParam[c][0] = pc.omega;
    a.classParam[c][1] = pc.magic;
    a.classParam[c][2] = pc.smagorinsky;
    for (int k = 0; k < 3; ++k) a.classParam[c][3 + k] = pc.force[k];
    a.classDyn[c] = (L->classMask >> c & 1) ? L->classDyn[c] : 0;
  }
  return a;
}

// Dispatch a launcher template on (Q, storage).
#define LBX_DISPATCH(L, CALL)                                                                     \
  [&]() -> cudaError_t {                                                                          \
    switch ((L)->q * 4 + (L)->storage) {                                                          \
    case 9 * 4 + LBX_F64: { constexpr int Q = 9; using S = double; return CALL; }                 \
    case 9 * 4 + LBX_F32: { constexpr int Q = 9; using S = float; return CALL; }                  \
    case 9 * 4 + LBX_F16DEV: { constexpr int Q = 9; using S = __half; return CALL; }              \
    case 9 * 4 + LBX_BF16DEV: { constexpr int Q = 9; using S = __nv_bfloat16; return CALL; }      \
    case 19 * 4 + LBX_F64: { constexpr int Q = 19; using S = double; return CALL; }               \
    case 19 * 4 + LBX_F32: { constexpr int Q = 19; using S = float; return CALL; }                \
    case 19 * 4 + LBX_F16DEV: { constexpr int Q = 19; using S = __half; return CALL; }            \
    case 19 * 4 + LBX_BF16DEV: { constexpr int Q = 19; using S = __nv_bfloat16; return CALL; }    \
    case 27 * 4 + LBX_F64: { constexpr int Q = 27; using S = double; return CALL; }               \
    case 27 * 4 + LBX_F32: { constexpr int Q = 27; using S = float; return CALL; }                \
    case 27 * 4 + LBX_F16DEV: { constexpr int Q = 27; using S = __half; return CALL; }            \
    case 27 * 4 + LBX_BF16DEV: { constexpr int Q = 27; using S = __nv_bfloat16; return CALL; }    \
    default: return cudaErrorInvalidValue;                                                        \
    }                                                                                             \
  }()

int64_t core_index_to_padded(const lbx_lattice_s* L, int64_t c) {
  const int nz = (L->d == 3) ? L->core[2] : 1;
  const int64_t z = c % nz;
  const int64_t y = (c / nz) % L->core[1];
  const int64_t x = c / (int64_t(nz) * L->core[1]);
  const Geometry g = geometry_of(L);
  return (x + 1) * g.sx + (y + 1) * g.sy + (z + g.pz);
}

void rotate_all(lbx_lattice_s* L) {
  const Geometry g = geometry_of(L);
  for (int i = 0; i < L->q; ++i) {
    const int* c = velocity(L->q, i);
    const int64_t off = c[0] * g.sx + c[1] * g.sy + ((L->d == 3) ? c[2] : 0);
    int64_t s = (L->shift[i] - off) % L->period;
    if (s < 0) s += L->period;
    L->shift[i] = s;
  }
}

// Threads along the fastest core axis, filled up to 256 per block; the rest of the block
// spans the next axis.
void block_shape_for(int nf, int cellsPerThread, int& bx, int& by) {
  const int groups = lbx::k_cells_threads(nf, cellsPerThread);
  bx = 32;
  while (bx < groups && bx < 256) bx *= 2;
  by = 256 / bx;
}

void default_block_shape(lbx_lattice_s* L) {
  const int nf = (L->d == 3) ? L->core[2] : L->core[1];
  L->cellsPerThread = 1;
  L->kernel = (L->period < (int64_t(1) << 31)) ? 2 : 1;
  if (L->kernel == 1) L->cellsPerThread = 1;
  block_shape_for(nf, L->cellsPerThread, L->blockX, L->blockY);
}

// Blocks the step kernel of the current launch configuration runs (the statistics partials
// hold one entry per block).
int64_t step_blocks(const lbx_lattice_s* L) {
  const Geometry g = geometry_of(L);
  const int nf = (L->d == 3) ? g.nz : g.ny;
  const int nm = (L->d == 3) ? g.ny : g.nx;
  const int ns = (L->d == 3) ? g.nx : 1;
  if (L->kernel == 0) {
    const LaunchArgs a = args_of(L);
    return (a.flatEnd - a.flatBase + TILE - 1) / TILE;
  }
  if (L->kernel == 3 || L->kernel == 4) {  // at most one persistent block per tile (the grid is capped by residency)
    const LaunchArgs a = args_of(L);
    int64_t bt = 0;
    switch (L->q * 4 + L->storage) {
#define LBX_BT(QQ, SS, ST) \
  case QQ * 4 + ST: bt = L->kernel == 3 ? BulkCfg<QQ, SS>::BT : WsCfg<QQ, SS>::BT; break;
      LBX_BT(9, double, LBX_F64) LBX_BT(9, float, LBX_F32) LBX_BT(9, __half, LBX_F16DEV) LBX_BT(9, __nv_bfloat16, LBX_BF16DEV)
      LBX_BT(19, double, LBX_F64) LBX_BT(19, float, LBX_F32) LBX_BT(19, __half, LBX_F16DEV) LBX_BT(19, __nv_bfloat16, LBX_BF16DEV)
      LBX_BT(27, double, LBX_F64) LBX_BT(27, float, LBX_F32) LBX_BT(27, __half, LBX_F16DEV) LBX_BT(27, __nv_bfloat16, LBX_BF16DEV)
#undef LBX_BT
      default: bt = 64;
    }
    return (a.flatEnd - a.flatBase + bt - 1) / bt;
  }
  const int64_t groups = groups_kernel(L->kernel) ? lbx::k_cells_threads(nf, L->cellsPerThread) : nf;
  return ((groups + L->blockX - 1) / L->blockX) * int64_t((nm + L->blockY - 1) / L->blockY) * ns;
}

int ensure_stat_capacity(lbx_lattice_s* L) {
  const int64_t need = step_blocks(L) + fd_blocks(L->nFd) + fd_blocks(L->nBbv);
  if (need > L->statCapacity) {
    cudaFree(L->statPart);
    L->statPart = nullptr;
    L->statCapacity = 0;
    LBX_CUDA_TRY(cudaMalloc(&L->statPart, size_t(need) * 4 * sizeof(double)));
    L->statCapacity = need;
  }
  return LBX_OK;
}

int ensure_stage(lbx_lattice_s* L) {
  if (!L->stage) LBX_CUDA_TRY(cudaMalloc(&L->stage, size_t(L->ncore) * sizeof(double)));
  return LBX_OK;
}

// ---- population columns in doubled virtual mappings -------------------------------------
// Each column's physical memory (one allocation of C bytes) is mapped twice, back to back,
// into one reserved virtual range: element j and element j + P alias.  A population index
// n + shift (< 2P) then never needs the modulo of the periodic-shift pattern, which removes
// the wrap arithmetic from every access of the step kernel.  This is the technique of the
// reference's CUDA CyclicColumn (core/platform/gpu/cuda/column.hh:217-256), built here on the CUDA VMM
// API.  Without it (entry points missing, or any step failing) the columns fall back to one
// plain allocation and the kernels wrap explicitly.
namespace vmm {
using FnGran = CUresult (*)(size_t*, const CUmemAllocationProp*, CUmemAllocationGranularity_flags);
using FnCreate = CUresult (*)(CUmemGenericAllocationHandle*, size_t, const CUmemAllocationProp*, unsigned long long);
using FnRelease = CUresult (*)(CUmemGenericAllocationHandle);
using FnReserve = CUresult (*)(CUdeviceptr*, size_t, size_t, CUdeviceptr, unsigned long long);
using FnAddrFree = CUresult (*)(CUdeviceptr, size_t);
using FnMap = CUresult (*)(CUdeviceptr, size_t, size_t, CUmemGenericAllocationHandle, unsigned long long);
using FnUnmap = CUresult (*)(CUdeviceptr, size_t);
using FnAccess = CUresult (*)(CUdeviceptr, size_t, const CUmemAccessDesc*, size_t);

struct Api {
  FnGran gran = nullptr;
  FnCreate create = nullptr;
  FnRelease release = nullptr;
  FnReserve reserve = nullptr;
  FnAddrFree addrFree = nullptr;
  FnMap map = nullptr;
  FnUnmap unmap = nullptr;
  FnAccess access = nullptr;
  bool ok = false;
};

template <typename F>
bool entry(const char* name, F& fn) {
  void* p = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess || !p) {
    cudaGetLastError();
    return false;
  }
  fn = reinterpret_cast<F>(p);
  return true;
}

const Api& api() {
  static Api a = [] {
    Api r;
    r.ok = entry("cuMemGetAllocationGranularity", r.gran) && entry("cuMemCreate", r.create) &&
           entry("cuMemRelease", r.release) && entry("cuMemAddressReserve", r.reserve) &&
           entry("cuMemAddressFree", r.addrFree) && entry("cuMemMap", r.map) && entry("cuMemUnmap", r.unmap) &&
           entry("cuMemSetAccess", r.access);
    return r;
  }();
  return a;
}
}  // namespace vmm

void release_columns(lbx_lattice_s* L) {
  if (L->doubled) {
    const auto& a = vmm::api();
    if (L->vmmBase) a.unmap(CUdeviceptr(L->vmmBase), size_t(L->vmmBytes));
    for (int i = 0; i < L->q; ++i)
      if (L->vmmHandles[i]) a.release(CUmemGenericAllocationHandle(L->vmmHandles[i]));
    if (L->vmmBase) a.addrFree(CUdeviceptr(L->vmmBase), size_t(L->vmmBytes));
    L->vmmBase = 0;
    L->doubled = false;
  } else {
    cudaFree(L->pop);
  }
  L->pop = nullptr;
}

bool try_doubled_columns(lbx_lattice_s* L, size_t es) {
  const auto& a = vmm::api();
  if (!a.ok) return false;
  CUmemAllocationProp prop{};
  prop.type = CU_MEM_ALLOCATION_TYPE_PINNED;
  prop.location.type = CU_MEM_LOCATION_TYPE_DEVICE;
  prop.location.id = L->device;
  size_t gran = 0;
  if (a.gran(&gran, &prop, CU_MEM_ALLOC_GRANULARITY_MINIMUM) != CUDA_SUCCESS || gran == 0) return false;
  const size_t colBytes = (size_t(L->n) * es + gran - 1) / gran * gran;
  const size_t total = size_t(L->q) * 2 * colBytes;
  CUdeviceptr base = 0;
  if (a.reserve(&base, total, gran, 0, 0) != CUDA_SUCCESS) return false;
  L->vmmBase = base;
  L->vmmBytes = total;
  L->doubled = true;
  bool ok = true;
  for (int i = 0; i < L->q && ok; ++i) {
    CUmemGenericAllocationHandle h;
    if (a.create(&h, colBytes, &prop, 0) != CUDA_SUCCESS) { ok = false; break; }
    L->vmmHandles[i] = h;
    ok = a.map(base + CUdeviceptr(2 * i * colBytes), colBytes, 0, h, 0) == CUDA_SUCCESS &&
         a.map(base + CUdeviceptr((2 * i + 1) * colBytes), colBytes, 0, h, 0) == CUDA_SUCCESS;
  }
  if (ok) {
    CUmemAccessDesc acc{};
    acc.location.type = CU_MEM_LOCATION_TYPE_DEVICE;
    acc.location.id = L->device;
    acc.flags = CU_MEM_ACCESS_FLAGS_PROT_READWRITE;
    ok = a.access(base, total, &acc, 1) == CUDA_SUCCESS;
  }
  if (!ok) {
    // unmap whatever was mapped: unmapping the whole range is allowed only if fully mapped, so
    // unmap column by column
    for (int i = 0; i < L->q; ++i) {
      if (!L->vmmHandles[i]) continue;
      a.unmap(base + CUdeviceptr(2 * i * colBytes), colBytes);
      a.unmap(base + CUdeviceptr((2 * i + 1) * colBytes), colBytes);
      a.release(CUmemGenericAllocationHandle(L->vmmHandles[i]));
      L->vmmHandles[i] = 0;
    }
    a.addrFree(base, total);
    L->vmmBase = 0;
    L->doubled = false;
    cudaGetLastError();
    return false;
  }
  L->pop = reinterpret_cast<void*>(base);
  L->period = int64_t(colBytes / es);
  L->stride = 2 * L->period;
  L->bytes = int64_t(size_t(L->q) * colBytes);
  return true;
}

// Allocate the Q population columns: doubled mappings when the VMM API is available, one plain
// allocation otherwise.  Contents start at zero.
cudaError_t alloc_columns(lbx_lattice_s* L) {
  if (test_allocation_fails()) return cudaErrorMemoryAllocation;  // lbx_test_fault
  const size_t es = storage_bytes(L->storage);
  if (!std::getenv("LBX_PLAIN_COLUMNS") && try_doubled_columns(L, es)) {
    // zero the first copy of every column (the second aliases it)
    for (int i = 0; i < L->q; ++i) {
      cudaError_t e = cudaMemset(static_cast<char*>(L->pop) + size_t(i) * size_t(L->stride) * es, 0,
                                 size_t(L->period) * es);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  L->period = (L->n + 127) / 128 * 128;
  L->stride = L->period;
  const size_t bytes = size_t(L->q) * size_t(L->stride) * es;
  cudaError_t e = cudaMalloc(&L->pop, bytes);
  if (e == cudaSuccess) e = cudaMemset(L->pop, 0, bytes);
  L->bytes = int64_t(bytes);
  return e;
}

cudaEvent_t take_event(lbx_lattice_s* L) {
  if (!L->eventPool.empty()) {
    cudaEvent_t e = L->eventPool.back();
    L->eventPool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) e = nullptr;
  return e;
}

// Fold the recorded groups into the totals (waits for them) and recycle their events.
void drain_timing(lbx_lattice_s* L) {
  for (size_t g = 0; g + 4 <= L->pending.size(); g += 4) {
    cudaEvent_t* e = &L->pending[g];
    float ms = 0.f;
    if (cudaEventSynchronize(e[3]) == cudaSuccess) {
      if (cudaEventElapsedTime(&ms, e[0], e[1]) == cudaSuccess) { L->timedMs[0] += ms; ++L->timedLaunches[0]; }
      if ((L->periodic[0] || L->periodic[1] || L->periodic[2]) && !groups_kernel(L->kernel)) {  // variants 2, 5: no copy launch
        if (cudaEventElapsedTime(&ms, e[1], e[2]) == cudaSuccess) { L->timedMs[1] += ms; ++L->timedLaunches[1]; }
      }
      if (L->nLinks > 0) {
        if (cudaEventElapsedTime(&ms, e[2], e[3]) == cudaSuccess) { L->timedMs[2] += ms; ++L->timedLaunches[2]; }
      }
    }
    for (int k = 0; k < 4; ++k) L->eventPool.push_back(e[k]);
  }
  L->pending.clear();
  cudaGetLastError();
}


bool device_ok(int device, std::string& why) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    why = "no CUDA device";
    return false;
  }
  if (device < 0 || device >= count) {
    why = "device index out of range";
    return false;
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
    why = "cudaGetDeviceProperties failed";
    return false;
  }
  if (prop.major != 10) {
    why = "device is compute capability " + std::to_string(prop.major) + "." + std::to_string(prop.minor) +
          "; liblbx is built for sm_100a only";
    return false;
  }
  return true;
}


// Composes the device cell map from the map as set and the links, and splits the links: a link
// from a bulk cell (x_b, k) towards a cell without dynamics, at rest (no wall term), is fused
// into the K-cells step kernel (bit k of linkMask[x_b], x_b marked kCellBulkLinked); every other
// link stays with the link kernel, which with the other kernel variants applies all links.
// The per-cell boundary index (lbx_lattice_s::bIdx) from the two boundary lists.
int refresh_boundary_index(lbx_lattice_s* L) {
  cudaFree(L->bIdx);
  L->bIdx = nullptr;
  if (L->fdHostCells.empty() && L->bbvHostCells.empty()) return LBX_OK;
  std::vector<int32_t> idx(static_cast<size_t>(L->n), -1);
  for (size_t j = 0; j < L->fdHostCells.size(); ++j) idx[L->fdHostCells[j]] = int32_t(j);
  for (size_t j = 0; j < L->bbvHostCells.size(); ++j) idx[L->bbvHostCells[j]] = -2 - int32_t(j);
  LBX_CUDA_TRY(cudaMalloc(&L->bIdx, idx.size() * sizeof(int32_t)));
  LBX_CUDA_TRY(cudaMemcpy(L->bIdx, idx.data(), idx.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  return LBX_OK;
}

int refresh_cell_map(lbx_lattice_s* L) {
  ++L->mapVersion;
  if (int rc = refresh_boundary_index(L)) return rc;
  const bool need = !L->hostMap.empty() || L->nLinks > 0;
  cudaFree(L->linkMask);
  cudaFree(L->restCell);
  cudaFree(L->restDir);
  cudaFree(L->restDelta);
  L->linkMask = nullptr;
  L->restCell = nullptr;
  L->restDir = nullptr;
  L->restDelta = nullptr;
  L->nRest = 0;
  if (!need) {
    cudaFree(L->cellDyn);
    L->cellDyn = nullptr;
    return LBX_OK;
  }
  std::vector<uint8_t> map = L->hostMap;
  if (map.empty()) {
    map.assign(static_cast<size_t>(L->n), 0);
    for (int64_t c = 0; c < L->ncore; ++c) map[size_t(core_index_to_padded(L, c))] = LBX_CELL_BULK;
  }
  std::vector<uint32_t> mask;
  std::vector<uint32_t> rc;
  std::vector<uint8_t> rd;
  std::vector<double> rdelta;
  bool restWall = false;
  if (L->nLinks > 0) {
    mask.assign(static_cast<size_t>(L->n), 0u);
    const Geometry g = geometry_of(L);
    const int64_t ext[3] = {g.nx, g.ny, g.nz};
    for (size_t l = 0; l < L->linkHostCell.size(); ++l) {
      const uint32_t src = L->linkHostCell[l];
      const int k = L->linkHostDir[l];
      // core coordinates of the solid neighbour, across a periodic face to its image
      int64_t p[3];
      p[0] = int64_t(src) / g.sx - 1;
      const int64_t r = int64_t(src) - (p[0] + 1) * g.sx;
      p[1] = r / g.sy - 1;
      p[2] = r - (p[1] + 1) * g.sy - g.pz;
      const int* c = velocity(L->q, k);
      bool inside = true;
      for (int a = 0; a < L->d; ++a) {
        p[a] += c[a];
        if (p[a] < 0 || p[a] >= ext[a]) {
          if (L->periodic[a]) p[a] = (p[a] + ext[a]) % ext[a];
          else inside = false;
        }
      }
      const int64_t tgt = inside ? (p[0] + 1) * g.sx + (p[1] + 1) * g.sy + (p[2] + g.pz) : -1;
      const bool fuse = L->linkHostDelta[l] == 0.0 && map[src] == LBX_CELL_BULK && tgt >= 0 &&
                        map[size_t(tgt)] == LBX_CELL_NONE;
      if (fuse) {
        mask[src] |= 1u << k;
      } else {
        rc.push_back(src);
        rd.push_back(uint8_t(k));
        rdelta.push_back(L->linkHostDelta[l]);
        restWall = restWall || L->linkHostDelta[l] != 0.0;
      }
    }
    bool any = false;
    for (size_t n = 0; n < mask.size(); ++n)
      if (mask[n]) {
        map[n] = kCellBulkLinked;
        any = true;
      }
    if (any) {
      LBX_CUDA_TRY(cudaMalloc(&L->linkMask, mask.size() * sizeof(uint32_t)));
      LBX_CUDA_TRY(cudaMemcpy(L->linkMask, mask.data(), mask.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    }
    // the links the link kernel applies after the K-cells kernel
    const int64_t nr = int64_t(rc.size());
    if (nr > 0) {
      LBX_CUDA_TRY(cudaMalloc(&L->restCell, size_t(nr) * sizeof(uint32_t)));
      LBX_CUDA_TRY(cudaMalloc(&L->restDir, size_t(nr)));
      LBX_CUDA_TRY(cudaMemcpy(L->restCell, rc.data(), size_t(nr) * sizeof(uint32_t), cudaMemcpyHostToDevice));
      LBX_CUDA_TRY(cudaMemcpy(L->restDir, rd.data(), size_t(nr), cudaMemcpyHostToDevice));
      if (restWall) {
        if (L->storage == LBX_F64) {
          LBX_CUDA_TRY(cudaMalloc(&L->restDelta, size_t(nr) * sizeof(double)));
          LBX_CUDA_TRY(cudaMemcpy(L->restDelta, rdelta.data(), size_t(nr) * sizeof(double), cudaMemcpyHostToDevice));
        } else {
          std::vector<float> df(rdelta.begin(), rdelta.end());
          LBX_CUDA_TRY(cudaMalloc(&L->restDelta, size_t(nr) * sizeof(float)));
          LBX_CUDA_TRY(cudaMemcpy(L->restDelta, df.data(), size_t(nr) * sizeof(float), cudaMemcpyHostToDevice));
        }
      }
      L->nRest = nr;
    }
  }
  if (!L->cellDyn) LBX_CUDA_TRY(cudaMalloc(&L->cellDyn, size_t(L->n)));
  LBX_CUDA_TRY(cudaMemcpy(L->cellDyn, map.data(), size_t(L->n), cudaMemcpyHostToDevice));
  return LBX_OK;
}

// Validates a boundary list, sorts it by cell and uploads it (lbx_set_fd_boundaries,
// lbx_set_boundary_cells, lbx_set_interpolated_boundary).  The listed cells become
// LBX_CELL_FD_BOUNDARY in the cell map; cells of the previous list that are not listed again
// become bulk.
int install_boundary_list(lbx_lattice_s* L, std::vector<FdHostCell> list) {
  DeviceGuard guard(L->device);
  const int64_t n = int64_t(list.size());
  for (const FdHostCell& c : list) {
    if (c.core < 0 || c.core >= L->ncore) return fail(LBX_ERR_INVALID, "boundary cell out of range");
    if (c.kind < LBX_FD_VELOCITY || c.kind > LBX_FD_LOCAL_PRESSURE_RLB) return fail(LBX_ERR_INVALID, "unknown boundary kind");
    if (c.type < LBX_NORMAL_FLAT || c.type > LBX_NORMAL_INTERNAL_EDGE) return fail(LBX_ERR_INVALID, "unknown normal type");
    const bool edge = c.type == LBX_NORMAL_EXTERNAL_EDGE || c.type == LBX_NORMAL_INTERNAL_EDGE;
    if (edge && L->d != 3) return fail(LBX_ERR_INVALID, "edges exist in 3D only");
    const bool pressure =
        c.kind == LBX_FD_PRESSURE || c.kind == LBX_FD_LOCAL_PRESSURE || c.kind == LBX_FD_LOCAL_PRESSURE_RLB;
    if (pressure && c.type != LBX_NORMAL_FLAT)
      return fail(LBX_ERR_UNSUPPORTED, "pressure boundaries are provided on flat faces only");
    int nonzero = 0;
    for (int a = 0; a < 3; ++a) {
      if (c.n[a] < -1 || c.n[a] > 1 || (a >= L->d && c.n[a] != 0)) return fail(LBX_ERR_INVALID, "normal components must be -1, 0 or 1");
      nonzero += c.n[a] != 0;
    }
    const int want = c.type == LBX_NORMAL_FLAT ? 1 : (edge ? 2 : L->d);
    if (nonzero != want) return fail(LBX_ERR_INVALID, "the normal does not match the normal type");
    const int64_t ny = L->core[1], nz = (L->d == 3) ? L->core[2] : 1;
    const int p[3] = {int(c.core / (ny * nz)), int((c.core / nz) % ny), int(c.core % nz)};
    for (int a = 0; a < L->d; ++a) {
      if (c.n[a] == 0) continue;
      if (L->periodic[a]) return fail(LBX_ERR_INVALID, "a boundary normal cannot lie along a periodic axis");
      const int in2 = p[a] - 2 * c.n[a];
      if (in2 < 0 || in2 >= L->core[a])
        return fail(LBX_ERR_INVALID, "a boundary cell needs two cells inward along each normal component");
    }
    for (int k = 0; k < 4; ++k)
      if (!std::isfinite(c.v[k])) return fail(LBX_ERR_INVALID, "boundary values must be finite");
    if (pressure && !(c.v[0] > 0)) return fail(LBX_ERR_INVALID, "boundary density must be > 0");
  }
  std::sort(list.begin(), list.end(), [](const FdHostCell& x, const FdHostCell& y) { return x.core < y.core; });
  for (int64_t i = 1; i < n; ++i)
    if (list[size_t(i)].core == list[size_t(i - 1)].core) return fail(LBX_ERR_INVALID, "duplicate boundary cell");
  std::vector<uint32_t> hc(static_cast<size_t>(n));
  std::vector<uint16_t> hm(static_cast<size_t>(n));
  std::vector<double> hv(static_cast<size_t>(4 * n));
  int64_t corners = 0;
  for (int64_t k = 0; k < n; ++k) {
    const FdHostCell& c = list[size_t(k)];
    hc[size_t(k)] = uint32_t(core_index_to_padded(L, c.core));
    int t = FD_FLAT_VELOCITY;
    if (c.type == LBX_NORMAL_FLAT) {
      switch (c.kind) {
        case LBX_FD_PRESSURE: t = FD_FLAT_PRESSURE; break;
        case LBX_FD_LOCAL_VELOCITY:
        case LBX_FD_LOCAL_VELOCITY_RLB: t = FD_FLAT_VELOCITY_LOCAL; break;
        case LBX_FD_LOCAL_PRESSURE:
        case LBX_FD_LOCAL_PRESSURE_RLB: t = FD_FLAT_PRESSURE_LOCAL; break;
        default: t = FD_FLAT_VELOCITY;
      }
    }
    else if (c.type == LBX_NORMAL_EXTERNAL_EDGE) t = FD_EDGE_VELOCITY;
    else if (c.type == LBX_NORMAL_INTERNAL_EDGE) t = FD_INNER_EDGE_VELOCITY;
    else if (c.type == LBX_NORMAL_INTERNAL_CORNER) t = FD_INNER_CORNER_VELOCITY;
    else t = FD_CORNER_VELOCITY;
    corners += t == FD_CORNER_VELOCITY;
    const bool rlb = c.kind == LBX_FD_LOCAL_VELOCITY_RLB || c.kind == LBX_FD_LOCAL_PRESSURE_RLB;
    hm[size_t(k)] = FdMeta::encode(t, c.n, rlb ? 1 : 0);
    for (int v = 0; v < 4; ++v) hv[size_t(4 * k + v)] = c.v[v];
  }
  cudaDeviceSynchronize();
  cudaFree(L->fdCell);
  cudaFree(L->fdMeta);
  cudaFree(L->fdValue);
  cudaFree(L->fdMom);
  L->fdCell = nullptr;
  L->fdMeta = nullptr;
  L->fdValue = nullptr;
  L->fdMom = nullptr;
  L->nFd = 0;
  L->nFdCorners = 0;
  // cell map: the listed cells become LBX_CELL_FD_BOUNDARY, the ones of an old list bulk
  if (L->hostMap.empty()) {
    L->hostMap.assign(static_cast<size_t>(L->n), 0);
    for (int64_t c = 0; c < L->ncore; ++c) L->hostMap[size_t(core_index_to_padded(L, c))] = LBX_CELL_BULK;
  }
  for (uint32_t old : L->fdHostCells) L->hostMap[old] = LBX_CELL_BULK;
  for (uint32_t c : hc) L->hostMap[c] = LBX_CELL_FD_BOUNDARY;
  L->fdHostCells = hc;
  L->fdHost = list;
  if (int rc = refresh_cell_map(L)) return rc;
  if (n == 0) return LBX_OK;
  LBX_CUDA_TRY(cudaMalloc(&L->fdCell, size_t(n) * sizeof(uint32_t)));
  LBX_CUDA_TRY(cudaMalloc(&L->fdMeta, size_t(n) * sizeof(uint16_t)));
  LBX_CUDA_TRY(cudaMalloc(&L->fdValue, size_t(4 * n) * sizeof(double)));
  LBX_CUDA_TRY(cudaMalloc(&L->fdMom, size_t(7 * n) * sizeof(double)));
  LBX_CUDA_TRY(cudaMemcpy(L->fdCell, hc.data(), size_t(n) * sizeof(uint32_t), cudaMemcpyHostToDevice));
  LBX_CUDA_TRY(cudaMemcpy(L->fdMeta, hm.data(), size_t(n) * sizeof(uint16_t), cudaMemcpyHostToDevice));
  LBX_CUDA_TRY(cudaMemcpy(L->fdValue, hv.data(), size_t(4 * n) * sizeof(double), cudaMemcpyHostToDevice));
  L->nFd = n;
  L->nFdCorners = corners;
  return LBX_OK;
}
// Installs a link list (lbx_set_bouzidi_links, lbx_set_bouzidi_from_materials); groups[l] tags
// link l with the solid it faces (NULL: every link in group 0).
int set_links_impl(lbx_lattice_s* L, int64_t n, const int64_t* cells, const int32_t* dirs, const double* wall,
                   const uint8_t* groups) {
  if (!L) return fail(LBX_ERR_INVALID, "null lattice");
  if (n < 0 || (n > 0 && (!cells || !dirs))) return fail(LBX_ERR_INVALID, "bad link arrays");
  DeviceGuard guard(L->device);
  cudaFree(L->linkCell);
  cudaFree(L->linkDir);
  cudaFree(L->linkDelta);
  cudaFree(L->linkGroup);
  L->linkGroup = nullptr;
  L->linkCell = nullptr;
  L->linkDir = nullptr;
  L->linkDelta = nullptr;
  L->nLinks = 0;
  L->linkHostCell.clear();
  L->linkHostDir.clear();
  L->linkHostDelta.clear();
  if (n == 0) return refresh_cell_map(L);
  std::vector<uint32_t> hc(static_cast<size_t>(n));
  std::vector<uint8_t> hd(static_cast<size_t>(n));
  std::vector<double> delta(static_cast<size_t>(n));
  std::vector<uint8_t> hg(static_cast<size_t>(n), 0);
  bool anyWall = false;
  for (int64_t l = 0; l < n; ++l) {
    if (cells[l] < 0 || cells[l] >= L->ncore) return fail(LBX_ERR_INVALID, "link cell out of range");
    if (dirs[l] < 1 || dirs[l] >= L->q) return fail(LBX_ERR_INVALID, "link direction out of range");
    hc[size_t(l)] = uint32_t(core_index_to_padded(L, cells[l]));
    hd[size_t(l)] = uint8_t(dirs[l]);
    if (groups) hg[size_t(l)] = groups[l];
    // 2 * veloTerm, veloTerm = (c_k . u_w) * t_k * invCs2 (setBouzidiBoundary.h:146)
    delta[size_t(l)] = wall ? 2.0 * (wall[l] * weight_of(L->q, dirs[l]) * 3.0) : 0.0;
    if (delta[size_t(l)] != 0.0) anyWall = true;
  }
  // Links ordered by direction, then cell: neighbouring threads of the link kernel then read
  // and write the same population column at nearby cells and share DRAM sectors, instead of
  // touching q different columns for one cell.  Every link reads and writes its own slots, so
  // the order does not change any result.
  {
    std::vector<int64_t> order(static_cast<size_t>(n));
    for (int64_t l = 0; l < n; ++l) order[size_t(l)] = l;
    std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) {
      return hd[size_t(a)] != hd[size_t(b)] ? hd[size_t(a)] < hd[size_t(b)] : hc[size_t(a)] < hc[size_t(b)];
    });
    std::vector<uint32_t> sc(hc.size());
    std::vector<uint8_t> sd(hd.size());
    std::vector<double> sdelta(delta.size());
    std::vector<uint8_t> sg(hg.size());
    for (size_t i = 0; i < order.size(); ++i) {
      sc[i] = hc[size_t(order[i])];
      sd[i] = hd[size_t(order[i])];
      sdelta[i] = delta[size_t(order[i])];
      sg[i] = hg[size_t(order[i])];
    }
    hc.swap(sc);
    hd.swap(sd);
    delta.swap(sdelta);
    hg.swap(sg);
  }
  LBX_CUDA_TRY(cudaMalloc(&L->linkCell, size_t(n) * sizeof(uint32_t)));
  LBX_CUDA_TRY(cudaMalloc(&L->linkDir, size_t(n)));
  LBX_CUDA_TRY(cudaMemcpy(L->linkCell, hc.data(), size_t(n) * sizeof(uint32_t), cudaMemcpyHostToDevice));
  LBX_CUDA_TRY(cudaMemcpy(L->linkDir, hd.data(), size_t(n), cudaMemcpyHostToDevice));
  LBX_CUDA_TRY(cudaMalloc(&L->linkGroup, size_t(n)));
  LBX_CUDA_TRY(cudaMemcpy(L->linkGroup, hg.data(), size_t(n), cudaMemcpyHostToDevice));
  if (anyWall) {
    if (L->storage == LBX_F64) {
      LBX_CUDA_TRY(cudaMalloc(&L->linkDelta, size_t(n) * sizeof(double)));
      LBX_CUDA_TRY(cudaMemcpy(L->linkDelta, delta.data(), size_t(n) * sizeof(double), cudaMemcpyHostToDevice));
    } else {
      std::vector<float> df(delta.begin(), delta.end());
      LBX_CUDA_TRY(cudaMalloc(&L->linkDelta, size_t(n) * sizeof(float)));
      LBX_CUDA_TRY(cudaMemcpy(L->linkDelta, df.data(), size_t(n) * sizeof(float), cudaMemcpyHostToDevice));
    }
  }
  L->nLinks = n;
  L->linkHostCell = hc;
  L->linkHostDir = hd;
  L->linkHostDelta = delta;
  return refresh_cell_map(L);
}

// One step in two phases, so that a decomposed lattice can exchange its slab faces between
// them (lbx_slabs_collide_and_stream): the collision with the fused stores, the periodic overlap
// copy and the shift rotation; then the post-stream links and boundary cells.
// ConstRhoBGK reads the previous step's average density, so its statistics are kept on every
// step, as the reference keeps them whenever statistics are enabled (its default).
int step_collide(lbx_lattice_s* L, bool statistics, cudaStream_t s, cudaEvent_t (&ev)[4]) {
  LaunchArgs a = args_of(L);
  if (statistics || L->dynamics == LBX_CONST_RHO_BGK) {
    if (int rc = ensure_stat_capacity(L)) return rc;
    a.stats = L->stats;
    a.statPart = L->statPart;
    a.statCapacity = L->statCapacity;
  }
  if (L->timing) {
    if (L->pending.size() >= 4 * 2048) drain_timing(L);
    for (auto& e : ev) e = take_event(L);
    if (ev[0]) cudaEventRecord(ev[0], s);
  }
  LBX_CUDA_TRY(LBX_DISPATCH(L, (launch_step<Q, S>(a, s))));
  if (ev[1]) cudaEventRecord(ev[1], s);
  LBX_CUDA_TRY(LBX_DISPATCH(L, (launch_halo<Q, S>(a, s))));
  if (ev[2]) cudaEventRecord(ev[2], s);
  rotate_all(L);
  return LBX_OK;
}

int step_post_stream(lbx_lattice_s* L, cudaStream_t s) {
  if (L->nLinks > 0 || L->nFd > 0) {
    const LaunchArgs b = args_of(L);
    // the K-cells kernel applied the resting links itself (linkMask); the link kernel does
    // the rest, or all of them after the other kernel variants
    if (b.linkMask) {
      if (L->nRest > 0)
        LBX_CUDA_TRY(LBX_DISPATCH(L, (launch_bouzidi<Q, S>(b, L->restCell, L->restDir, L->restDelta, L->nRest, s))));
    } else if (L->nLinks > 0) {
      LBX_CUDA_TRY(LBX_DISPATCH(L, (launch_bouzidi<Q, S>(b, L->linkCell, L->linkDir, L->linkDelta, L->nLinks, s))));
    }
    if (L->nFd > 0) LBX_CUDA_TRY(LBX_DISPATCH(L, (launch_fd_boundary<Q, S>(b, s))));
  }
  return LBX_OK;
}

}  // namespace

extern "C" {

const char* lbx_last_error(void) { return g_error.c_str(); }

int lbx_abi_version(void) { return LBX_ABI_VERSION; }

int lbx_test_fault(int32_t kind, int32_t param) {
  if (kind < LBX_TEST_NONE || kind > LBX_TEST_ALLOCATION) return fail(LBX_ERR_INVALID, "unknown test fault");
  if (param < 0) return fail(LBX_ERR_INVALID, "the parameter must be >= 0");
  test_fault().kind = kind;
  test_fault().param = param;
  return LBX_OK;
}

int lbx_device_count(void) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  int usable = 0;
  for (int d = 0; d < count; ++d) {
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, d) == cudaSuccess && prop.major == 10) ++usable;
  }
  return usable;
}

int lbx_lattice_create(int32_t q, const int32_t core[3], const int32_t periodic[3], int32_t storage,
                       int32_t device, lbx_lattice* out) {
  if (!out || !core) return fail(LBX_ERR_INVALID, "null argument");
  *out = nullptr;
  if (q != 9 && q != 19 && q != 27) return fail(LBX_ERR_UNSUPPORTED, "descriptor must be D2Q9, D3Q19 or D3Q27");
  if (storage_bytes(storage) == 0) return fail(LBX_ERR_INVALID, "unknown storage");
  const int d = (q == 9) ? 2 : 3;
  if (core[0] < 1 || core[1] < 1 || core[2] < 1) return fail(LBX_ERR_INVALID, "core extents must be >= 1");
  if (d == 2 && core[2] != 1) return fail(LBX_ERR_INVALID, "D2Q9 lattices have core[2] == 1");
  if (core[0] > 65535 || core[1] > 65535 * 256 || core[2] > (1 << 30))
    return fail(LBX_ERR_INVALID, "core extent too large");
  std::string why;
  if (!device_ok(device, why)) return fail(LBX_ERR_NO_DEVICE, why);
  DeviceGuard guard(device);
  if (!guard.ok) return fail(LBX_ERR_CUDA, "cudaSetDevice failed");

  auto* L = new lbx_lattice_s();
  L->q = q;
  L->d = d;
  L->storage = storage;
  L->device = device;
  for (int a = 0; a < 3; ++a) {
    L->core[a] = core[a];
    L->periodic[a] = periodic ? (periodic[a] != 0) : 0;
  }
  if (d == 2) L->periodic[2] = 0;
  L->padded[0] = core[0] + 2;
  L->padded[1] = core[1] + 2;
  L->padded[2] = (d == 3) ? core[2] + 2 : 1;
  L->n = int64_t(L->padded[0]) * L->padded[1] * L->padded[2];
  if (L->n >= (int64_t(1) << 32)) {
    delete L;
    return fail(LBX_ERR_INVALID, "padded block exceeds 2^32 cells");
  }
  L->ncore = int64_t(core[0]) * core[1] * core[2];
  cudaError_t e = alloc_columns(L);
  default_block_shape(L);
  if (e == cudaSuccess) e = cudaMalloc(&L->stats, sizeof(StatAcc));
  if (e == cudaSuccess) e = cudaMemset(L->stats, 0, sizeof(StatAcc));
  if (e == cudaSuccess) e = cudaMalloc(&L->reduceAcc, 8 * sizeof(double) + sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc(&L->devErr, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(L->devErr, 0, sizeof(int));
  if (e != cudaSuccess) {
    const std::string msg = std::string("allocation failed: ") + cudaGetErrorString(e);
    release_columns(L);
    cudaFree(L->stats);
    cudaFree(L->reduceAcc);
    delete L;
    return fail(e == cudaErrorMemoryAllocation ? LBX_ERR_OUT_OF_MEMORY : LBX_ERR_CUDA, msg);
  }
  *out = L;
  return LBX_OK;
}

int lbx_lattice_destroy(lbx_lattice L) {
  if (!L) return LBX_OK;
  DeviceGuard guard(L->device);
  cudaDeviceSynchronize();
  drain_timing(L);
  for (cudaEvent_t e : L->eventPool) cudaEventDestroy(e);
  release_columns(L);
  cudaFree(L->cellDyn);
  cudaFree(L->linkCell);
  cudaFree(L->linkDir);
  cudaFree(L->linkDelta);
  cudaFree(L->linkGroup);
  cudaFree(L->linkMask);
  cudaFree(L->restCell);
  cudaFree(L->restDir);
  cudaFree(L->restDelta);
  cudaFree(L->bIdx);
  cudaFree(L->bbvCell);
  cudaFree(L->bbvValue);
  cudaFree(L->fdCell);
  cudaFree(L->fdMeta);
  cudaFree(L->fdValue);
  cudaFree(L->fdMom);
  cudaFree(L->stats);
  cudaFree(L->statPart);
  cudaFree(L->reduceAcc);
  cudaFree(L->reducePart);
  cudaFree(L->devErr);
  cudaFree(L->residualSnap);
  cudaFree(L->stage);
  delete L;
  return LBX_OK;
}

int lbx_get_info(lbx_lattice L, lbx_info* info) {
  if (!L || !info) return fail(LBX_ERR_INVALID, "null argument");
  std::memset(info, 0, sizeof(*info));
  info->q = L->q;
  info->d = L->d;
  for (int a = 0; a < 3; ++a) {
    info->core[a] = L->core[a];
    info->padded[a] = L->padded[a];
    info->periodic[a] = L->periodic[a];
  }
  info->pad = 1;
  info->storage = L->storage;
  info->n_cells = L->n;
  info->n_core = L->ncore;
  info->column_stride = L->stride;
  info->column_period = L->period;
  info->bytes = L->bytes;
  info->n_links = L->nLinks;
  return LBX_OK;
}

int lbx_set_dynamics(lbx_lattice L, int32_t dynamics, const lbx_params* params) {
  if (!L || !params) return fail(LBX_ERR_INVALID, "null argument");
  if (dynamics < LBX_BGK || dynamics > LBX_CONST_RHO_BGK) return fail(LBX_ERR_UNSUPPORTED, "unknown dynamics");
  if (!(params->omega > 0.0 && params->omega < 2.0)) return fail(LBX_ERR_INVALID, "omega must lie in (0, 2)");
  if (dynamics == LBX_TRT && !(params->magic > 0.0)) return fail(LBX_ERR_INVALID, "TRT magic parameter must be > 0");
  if ((dynamics == LBX_SMAGORINSKY_BGK || dynamics == LBX_SMAGORINSKY_FORCED_BGK) && !(params->smagorinsky >= 0.0))
    return fail(LBX_ERR_INVALID, "Smagorinsky constant must be >= 0");
  for (int k = 0; k < 3; ++k)
    if (!std::isfinite(params->force[k])) return fail(LBX_ERR_INVALID, "force must be finite");
  if (dynamics == LBX_CONST_RHO_BGK && L->classMask)
    return fail(LBX_ERR_UNSUPPORTED, "ConstRhoBGK couples every cell to one average density; no classes");
  L->dynamics = dynamics;
  L->params = *params;
  return LBX_OK;
}

int lbx_set_dynamics_class(lbx_lattice L, int32_t cls, const lbx_params* params) {
  if (!L) return fail(LBX_ERR_INVALID, "null lattice");
  if (cls < 1 || cls > 3) return fail(LBX_ERR_INVALID, "parameter class must be 1, 2 or 3");
  if (!params) {
    L->classMask &= ~(1 << (cls - 1));
    return LBX_OK;
  }
  if (!(params->omega > 0.0 && params->omega < 2.0)) return fail(LBX_ERR_INVALID, "omega must lie in (0, 2)");
  if (L->dynamics == LBX_CONST_RHO_BGK)
    return fail(LBX_ERR_UNSUPPORTED, "ConstRhoBGK couples every cell to one average density; no classes");
  L->classParams[cls - 1] = *params;
  L->classDyn[cls - 1] = 0;
  L->classMask |= 1 << (cls - 1);
  // the classes run on the one-cell-per-thread step kernel
  L->kernel = 1;
  L->cellsPerThread = 1;
  return LBX_OK;
}

int lbx_set_dynamics_class_kind(lbx_lattice L, int32_t cls, int32_t dynamics, const lbx_params* params) {
  if (!L) return fail(LBX_ERR_INVALID, "null lattice");
  if (!params) return lbx_set_dynamics_class(L, cls, nullptr);
  if (dynamics < LBX_BGK || dynamics > LBX_SMAGORINSKY_FORCED_BGK)
    return fail(LBX_ERR_UNSUPPORTED, "a class's dynamics must be BGK, TRT, Smagorinsky-BGK or a forced one");
  if (int rc = lbx_set_dynamics_class(L, cls, params)) return rc;
  L->classDyn[cls - 1] = dynamics == L->dynamics ? 0 : dynamics;
  return LBX_OK;
}

int lbx_set_cell_dynamics(lbx_lattice L, const uint8_t* ids) {
  if (!L) return fail(LBX_ERR_INVALID, "null lattice");
  DeviceGuard guard(L->device);
  std::vector<uint8_t> padded(static_cast<size_t>(L->n), 0);
  for (int64_t c = 0; c < L->ncore; ++c) {
    const uint8_t id = ids ? ids[c] : uint8_t(LBX_CELL_BULK);
    if (id > LBX_CELL_FD_BOUNDARY && (id < LBX_CELL_BULK_CLASS_1 || id > LBX_CELL_BULK_CLASS_3))
      return fail(LBX_ERR_INVALID, "cell dynamics id out of range (boundary cells are set by their own calls)");
    padded[size_t(core_index_to_padded(L, c))] = id;
  }
  for (uint32_t n : L->fdHostCells) padded[n] = LBX_CELL_FD_BOUNDARY;  // the boundary lists win
  for (uint32_t n : L->bbvHostCells) padded[n] = LBX_CELL_BOUNCE_BACK_VELOCITY;
  if (!ids && L->fdHostCells.empty() && L->bbvHostCells.empty()) padded.clear();  // bulk everywhere: no map
  L->hostMap.swap(padded);
  cudaDeviceSynchronize();
  return refresh_cell_map(L);
}

int lbx_set_fd_boundaries(lbx_lattice L, int64_t n, const int64_t* cells, const int32_t* kinds,
                          const int32_t* dirs, const int32_t* orients, const double* values) {
  if (!L) return fail(LBX_ERR_INVALID, "null lattice");
  if (n < 0 || (n > 0 && (!cells || !kinds || !dirs || !orients || !values)))
    return fail(LBX_ERR_INVALID, "bad boundary arrays");
  std::vector<FdHostCell> list(static_cast<size_t>(n));
  for (int64_t i = 0; i < n; ++i) {
    FdHostCell& c = list[size_t(i)];
    c.core = cells[i];
    c.kind = kinds[i];
    c.type = LBX_NORMAL_FLAT;
    if (dirs[i] < 0 || dirs[i] >= L->d) return fail(LBX_ERR_INVALID, "normal axis out of range");
    if (orients[i] != 1 && orients[i] != -1) return fail(LBX_ERR_INVALID, "orientation must be +1 or -1");
    c.n[dirs[i]] = orients[i];
    for (int k = 0; k < 4; ++k) c.v[k] = values[4 * i + k];
  }
  return install_boundary_list(L, std::move(list));
}

int lbx_set_boundary_cells(lbx_lattice L, int64_t n, const int64_t* cells, const int32_t* kinds, const int32_t* types,
                           const int32_t* normals, const double* values) {
  if (!L) return fail(LBX_ERR_INVALID, "null lattice");
  if (n < 0 || (n > 0 && (!cells || !kinds || !types || !normals || !values)))
    return fail(LBX_ERR_INVALID, "bad boundary arrays");
  std::vector<FdHostCell> list(static_cast<size_t>(n));
  for (int64_t i = 0; i < n; ++i) {
    FdHostCell& c = list[size_t(i)];
    c.core = cells[i];
    c.kind = kinds[i];
    c.type = types[i];
    for (int a = 0; a < 3; ++a) c.n[a] = normals[3 * i + a];
    for (int k = 0; k < 4; ++k) c.v[k] = values[4 * i + k];
  }
  return install_boundary_list(L, std::move(list));
}

int lbx_set_interpolated_boundary(lbx_lattice L, int32_t kind, const int32_t* material, int32_t boundary,
                                  int32_t n_fluid, const int32_t* fluid, int32_t n_outside, const int32_t* outside,
                                  const double* values) {
  if (!L || !material || !values) return fail(LBX_ERR_INVALID, "null argument");
  if (kind < LBX_FD_VELOCITY || kind > LBX_FD_LOCAL_PRESSURE_RLB) return fail(LBX_ERR_INVALID, "unknown boundary kind");
  const bool pressureKind = kind == LBX_FD_PRESSURE || kind == LBX_FD_LOCAL_PRESSURE || kind == LBX_FD_LOCAL_PRESSURE_RLB;
  const int32_t defFluid = 1, defOutside = 0;
  if (n_fluid == 0) {
    fluid = &defFluid;
    n_fluid = 1;
  }
  if (n_outside == 0) {
    outside = &defOutside;
    n_outside = 1;
  }
  std::vector<int64_t> cells;
  std::vector<int32_t> types, normals;
  if (int rc = discrete_normals(L->q, L->core, L->periodic, material, boundary, n_fluid, fluid, n_outside, outside,
                                cells, types, normals))
    return rc;
  std::vector<FdHostCell> add;
  for (size_t k = 0; k < cells.size(); ++k) {
    const int t = types[k];
    const int* nn = &normals[3 * k];
    if (t < 0) return fail(LBX_ERR_INVALID, "the boundary material is also a fluid or outside material");
    const bool zero = nn[0] == 0 && nn[1] == 0 && nn[2] == 0;
    if (pressureKind && (t != LBX_NORMAL_FLAT || zero)) {
      if (zero) return fail(LBX_ERR_UNSUPPORTED, "could not set boundary: a pressure cell has no discrete normal");
      if (kind == LBX_FD_LOCAL_PRESSURE || kind == LBX_FD_LOCAL_PRESSURE_RLB)
        return fail(LBX_ERR_UNSUPPORTED, "LocalPressure: no valid discrete normal (flat faces only)");
      continue;  // InterpolatedPressure installs nothing on edges and corners
    }
    if (zero) return fail(LBX_ERR_UNSUPPORTED, "could not set boundary: a velocity cell has no discrete normal");
    FdHostCell c;
    c.core = cells[k];
    c.kind = kind;
    c.type = t;
    for (int a = 0; a < 3; ++a) c.n[a] = nn[a];
    for (int v = 0; v < 4; ++v) c.v[v] = values[4 * cells[k] + v];
    add.push_back(c);
  }
  // merge with the cells already set: a cell set again takes the new entry
  std::vector<FdHostCell> list;
  {
    std::vector<char> taken(static_cast<size_t>(L->ncore), 0);
    for (const FdHostCell& c : add) taken[size_t(c.core)] = 1;
    for (const FdHostCell& c : L->fdHost)
      if (!taken[size_t(c.core)]) list.push_back(c);
    list.insert(list.end(), add.begin(), add.end());
  }
  return install_boundary_list(L, std::move(list));
}

int lbx_set_bounce_back_velocity(lbx_lattice L, int64_t n, const int64_t* cells, const double* rho, const double* u) {
  if (!L) return fail(LBX_ERR_INVALID, "null lattice");
  if (n < 0 || (n > 0 && (!cells || !u))) return fail(LBX_ERR_INVALID, "bad bounce-back arrays");
  DeviceGuard guard(L->device);
  std::vector<int64_t> order(static_cast<size_t>(n));
  for (int64_t i = 0; i < n; ++i) {
    order[size_t(i)] = i;
    if (cells[i] < 0 || cells[i] >= L->ncore) return fail(LBX_ERR_INVALID, "bounce-back cell out of range");
    const double r = rho ? rho[i] : 1.0;
    if (!(r > 0) || !std::isfinite(r)) return fail(LBX_ERR_INVALID, "bounce-back density must be finite and > 0");
    for (int a = 0; a < 3; ++a)
      if (!std::isfinite(u[3 * i + a])) return fail(LBX_ERR_INVALID, "bounce-back velocity must be finite");
  }
  std::sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return cells[a] < cells[b]; });
  std::vector<uint32_t> hc(static_cast<size_t>(n));
  std::vector<double> hv(static_cast<size_t>(4 * n));
  for (int64_t k = 0; k < n; ++k) {
    const int64_t i = order[size_t(k)];
    if (k > 0 && cells[i] == cells[order[size_t(k - 1)]]) return fail(LBX_ERR_INVALID, "duplicate bounce-back cell");
    hc[size_t(k)] = uint32_t(core_index_to_padded(L, cells[i]));
    hv[size_t(4 * k)] = rho ? rho[i] : 1.0;
    for (int a = 0; a < 3; ++a) hv[size_t(4 * k + 1 + a)] = (a < L->d) ? u[3 * i + a] : 0.0;
  }
  for (uint32_t c : hc)
    for (uint32_t f : L->fdHostCells)
      if (c == f) return fail(LBX_ERR_INVALID, "a cell cannot be a velocity / pressure boundary and a bounce-back cell");
  cudaDeviceSynchronize();
  cudaFree(L->bbvCell);
  cudaFree(L->bbvValue);
  L->bbvCell = nullptr;
  L->bbvValue = nullptr;
  L->nBbv = 0;
  if (L->hostMap.empty()) {
    L->hostMap.assign(static_cast<size_t>(L->n), 0);
    for (int64_t c = 0; c < L->ncore; ++c) L->hostMap[size_t(core_index_to_padded(L, c))] = LBX_CELL_BULK;
  }
  for (uint32_t old : L->bbvHostCells) L->hostMap[old] = LBX_CELL_NONE;
  for (uint32_t c : hc) L->hostMap[c] = LBX_CELL_BOUNCE_BACK_VELOCITY;
  L->bbvHostCells = hc;
  if (n > 0) {
    LBX_CUDA_TRY(cudaMalloc(&L->bbvCell, size_t(n) * sizeof(uint32_t)));
    LBX_CUDA_TRY(cudaMalloc(&L->bbvValue, size_t(4 * n) * sizeof(double)));
    LBX_CUDA_TRY(cudaMemcpy(L->bbvCell, hc.data(), size_t(n) * sizeof(uint32_t), cudaMemcpyHostToDevice));
    LBX_CUDA_TRY(cudaMemcpy(L->bbvValue, hv.data(), size_t(4 * n) * sizeof(double), cudaMemcpyHostToDevice));
    L->nBbv = n;
  }
  return refresh_cell_map(L);
}

int lbx_set_bouzidi_links(lbx_lattice L, int64_t n, const int64_t* cells, const int32_t* dirs, const double* wall) {
  return set_links_impl(L, n, cells, dirs, wall, nullptr);
}

int lbx_build_bouzidi_links(int32_t q, const int32_t core[3], const int32_t periodic[3], const int32_t* material,
                            int32_t fluid, int32_t n_solid, const int32_t* solid, const double* wall_velocity,
                            int64_t cap, int64_t* cells, int32_t* dirs, double* wall, int64_t* n_out) {
  if (!core || !material || !n_out || (n_solid > 0 && !solid)) return fail(LBX_ERR_INVALID, "null argument");
  if (q != 9 && q != 19 && q != 27) return fail(LBX_ERR_UNSUPPORTED, "descriptor must be D2Q9, D3Q19 or D3Q27");
  const int d = (q == 9) ? 2 : 3;
  const int64_t nx = core[0], ny = core[1], nz = (d == 3) ? core[2] : 1;
  if (nx < 1 || ny < 1 || nz < 1) return fail(LBX_ERR_INVALID, "core extents must be >= 1");
  int64_t count = 0;
  for (int64_t x = 0; x < nx; ++x)
    for (int64_t y = 0; y < ny; ++y)
      for (int64_t z = 0; z < nz; ++z) {
        const int64_t cb = (x * ny + y) * nz + z;
        if (material[cb] != fluid) continue;
        for (int k = 1; k < q; ++k) {
          const int* c = velocity(q, k);
          int64_t s[3] = {x + c[0], y + c[1], z + ((d == 3) ? c[2] : 0)};
          const int64_t ext[3] = {nx, ny, nz};
          bool inside = true;
          for (int a = 0; a < d; ++a) {
            if (s[a] < 0 || s[a] >= ext[a]) {
              if (periodic && periodic[a]) s[a] = (s[a] + ext[a]) % ext[a];
              else inside = false;
            }
          }
          if (!inside) continue;
          const int64_t cs = (s[0] * ny + s[1]) * nz + s[2];
          int which = -1;
          for (int j = 0; j < n_solid; ++j)
            if (material[cs] == solid[j]) { which = j; break; }
          if (which < 0) continue;
          if (count < cap) {
            if (cells) cells[count] = cb;
            if (dirs) dirs[count] = k;
            if (wall) {
              double cu = 0.0;
              if (wall_velocity)
                for (int a = 0; a < d; ++a) cu += c[a] * wall_velocity[which * 3 + a];
              wall[count] = cu;
            }
          }
          ++count;
        }
      }
  *n_out = count;
  return LBX_OK;
}

int lbx_set_bouzidi_from_materials(lbx_lattice L, const int32_t* material, int32_t fluid, int32_t n_solid,
                                   const int32_t* solid, const double* wall_velocity) {
  if (!L) return fail(LBX_ERR_INVALID, "null lattice");
  int64_t n = 0;
  int rc = lbx_build_bouzidi_links(L->q, L->core, L->periodic, material, fluid, n_solid, solid, wall_velocity, 0,
                                   nullptr, nullptr, nullptr, &n);
  if (rc != LBX_OK) return rc;
  std::vector<int64_t> cells(static_cast<size_t>(n));
  std::vector<int32_t> dirs(static_cast<size_t>(n));
  std::vector<double> wall(static_cast<size_t>(n));
  rc = lbx_build_bouzidi_links(L->q, L->core, L->periodic, material, fluid, n_solid, solid, wall_velocity, n,
                               cells.data(), dirs.data(), wall.data(), &n);
  if (rc != LBX_OK) return rc;
  if (n_solid > 255) return fail(LBX_ERR_INVALID, "at most 255 solid materials");
  // group of each link: the index in `solid` of the material of the solid neighbour
  std::vector<uint8_t> groups(static_cast<size_t>(n), 0);
  {
    const int64_t ny = L->core[1], nz = (L->d == 3) ? L->core[2] : 1;
    for (int64_t l = 0; l < n; ++l) {
      const int* c = velocity(L->q, dirs[size_t(l)]);
      int64_t p[3] = {cells[size_t(l)] / (ny * nz), (cells[size_t(l)] / nz) % ny, cells[size_t(l)] % nz};
      const int64_t ext[3] = {L->core[0], ny, nz};
      for (int a = 0; a < L->d; ++a) p[a] = ((p[a] + c[a]) % ext[a] + ext[a]) % ext[a];
      const int32_t m = material[(p[0] * ny + p[1]) * nz + p[2]];
      for (int32_t j = 0; j < n_solid; ++j)
        if (solid[j] == m) {
          groups[size_t(l)] = uint8_t(j);
          break;
        }
    }
  }
  return set_links_impl(L, n, cells.data(), dirs.data(), wall_velocity ? wall.data() : nullptr, groups.data());
}

int lbx_upload_populations(lbx_lattice L, const void* host, int32_t host_type, void* stream) {
  if (!L || !host) return fail(LBX_ERR_INVALID, "null argument");
  if (host_type != 0 && host_type != 1) return fail(LBX_ERR_INVALID, "host_type must be 0 (double) or 1 (float)");
  DeviceGuard guard(L->device);
  if (int rc = ensure_stage(L)) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const LaunchArgs a = args_of(L);
  const size_t es = host_type == 0 ? sizeof(double) : sizeof(float);
  for (int i = 0; i < L->q; ++i) {
    const char* src = static_cast<const char*>(host) + size_t(i) * size_t(L->ncore) * es;
    LBX_CUDA_TRY(cudaMemcpyAsync(L->stage, src, size_t(L->ncore) * es, cudaMemcpyHostToDevice, s));
    LBX_CUDA_TRY(LBX_DISPATCH(L, (launch_transfer<Q, S>(a, i, L->stage, host_type, true, s))));
  }
  return LBX_OK;
}

int lbx_download_populations(lbx_lattice L, void* host, int32_t host_type, void* stream) {
  if (!L || !host) return fail(LBX_ERR_INVALID, "null argument");
  if (host_type != 0 && host_type != 1) return fail(LBX_ERR_INVALID, "host_type must be 0 (double) or 1 (float)");
  DeviceGuard guard(L->device);
  if (int rc = ensure_stage(L)) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const LaunchArgs a = args_of(L);
  const size_t es = host_type == 0 ? sizeof(double) : sizeof(float);
  for (int i = 0; i < L->q; ++i) {
    char* dst = static_cast<char*>(host) + size_t(i) * size_t(L->ncore) * es;
    LBX_CUDA_TRY(LBX_DISPATCH(L, (launch_transfer<Q, S>(a, i, L->stage, host_type, false, s))));
    LBX_CUDA_TRY(cudaMemcpyAsync(dst, L->stage, size_t(L->ncore) * es, cudaMemcpyDeviceToHost, s));
  }
  LBX_CUDA_TRY(cudaStreamSynchronize(s));
  return LBX_OK;
}

// ---- checkpoint / resume ------------------------------------------------------------------
// Header of a checkpoint buffer (128 bytes, host byte order), then [q][core cells] populations
// of the exchange layout: FP64 for the FP64 form, FP32 for the others (exact for every form).
struct CheckpointHeader {
  char magic[8];          // "LBXCKPT1"
  int32_t version;        // 1
  int32_t q, d, storage;
  int32_t core[3], periodic[3];
  int64_t ncore;
  StatAcc stats;          // accumulator of the last statistics step (lbx_get_statistics)
  int32_t valueBytes;     // 8 or 4
  int32_t pad[9];
};
static_assert(sizeof(CheckpointHeader) == 128, "checkpoint header is 128 bytes");

static int64_t checkpoint_value_bytes(const lbx_lattice_s* L) { return L->storage == LBX_F64 ? 8 : 4; }

int lbx_checkpoint_bytes(lbx_lattice L, int64_t* bytes) {
  if (!L || !bytes) return fail(LBX_ERR_INVALID, "null argument");
  *bytes = int64_t(sizeof(CheckpointHeader)) + int64_t(L->q) * L->ncore * checkpoint_value_bytes(L);
  return LBX_OK;
}

int lbx_save_checkpoint(lbx_lattice L, void* host, int64_t bytes, void* stream) {
  if (!L || !host) return fail(LBX_ERR_INVALID, "null argument");
  int64_t need = 0;
  lbx_checkpoint_bytes(L, &need);
  if (bytes < need) return fail(LBX_ERR_INVALID, "checkpoint buffer holds " + std::to_string(bytes) +
                                                     " bytes, the lattice needs " + std::to_string(need));
  DeviceGuard guard(L->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  CheckpointHeader h;
  std::memset(&h, 0, sizeof(h));
  std::memcpy(h.magic, "LBXCKPT1", 8);
  h.version = 1;
  h.q = L->q;
  h.d = L->d;
  h.storage = L->storage;
  for (int a = 0; a < 3; ++a) {
    h.core[a] = L->core[a];
    h.periodic[a] = L->periodic[a];
  }
  h.ncore = L->ncore;
  h.valueBytes = int32_t(checkpoint_value_bytes(L));
  LBX_CUDA_TRY(cudaMemcpyAsync(&h.stats, L->stats, sizeof(StatAcc), cudaMemcpyDeviceToHost, s));
  LBX_CUDA_TRY(cudaStreamSynchronize(s));
  std::memcpy(host, &h, sizeof(h));
  return lbx_download_populations(L, static_cast<char*>(host) + sizeof(h), h.valueBytes == 8 ? 0 : 1, stream);
}

int lbx_load_checkpoint(lbx_lattice L, const void* host, int64_t bytes, void* stream) {
  if (!L || !host) return fail(LBX_ERR_INVALID, "null argument");
  if (bytes < int64_t(sizeof(CheckpointHeader))) return fail(LBX_ERR_INVALID, "checkpoint shorter than its header");
  CheckpointHeader h;
  std::memcpy(&h, host, sizeof(h));
  if (std::memcmp(h.magic, "LBXCKPT1", 8) != 0 || h.version != 1) return fail(LBX_ERR_INVALID, "not a checkpoint of this format");
  bool same = h.q == L->q && h.d == L->d && h.storage == L->storage && h.ncore == L->ncore &&
              h.valueBytes == checkpoint_value_bytes(L);
  for (int a = 0; a < 3; ++a) same = same && h.core[a] == L->core[a] && h.periodic[a] == L->periodic[a];
  if (!same) return fail(LBX_ERR_INVALID, "checkpoint was taken from a lattice of another descriptor, storage, extent or periodicity");
  int64_t need = 0;
  lbx_checkpoint_bytes(L, &need);
  if (bytes < need) return fail(LBX_ERR_INVALID, "checkpoint truncated");
  DeviceGuard guard(L->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (int rc = lbx_upload_populations(L, static_cast<const char*>(host) + sizeof(h), h.valueBytes == 8 ? 0 : 1, stream))
    return rc;
  StatAcc st = h.stats;
  LBX_CUDA_TRY(cudaMemcpyAsync(L->stats, &st, sizeof(StatAcc), cudaMemcpyHostToDevice, s));
  LBX_CUDA_TRY(cudaStreamSynchronize(s));
  return LBX_OK;
}

int lbx_ini_equilibrium(lbx_lattice L, const double* rho, const double* u, void* stream) {
  if (!L || !rho || !u) return fail(LBX_ERR_INVALID, "null argument");
  DeviceGuard guard(L->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t nb = size_t(L->ncore) * sizeof(double);
  double* dev = nullptr;
  LBX_CUDA_TRY(cudaMalloc(&dev, nb * size_t(1 + L->d)));
  cudaError_t e = cudaMemcpyAsync(dev, rho, nb, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dev + L->ncore, u, nb * size_t(L->d), cudaMemcpyHostToDevice, s);
  const LaunchArgs a = args_of(L);
  if (e == cudaSuccess) e = LBX_DISPATCH(L, (launch_ini_equilibrium<Q, S>(a, dev, dev + L->ncore, s)));
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(dev);
  LBX_CUDA_TRY(e);
  return LBX_OK;
}

int lbx_collide_and_stream(lbx_lattice L, int64_t steps, uint32_t flags, void* stream) {
  if (!L) return fail(LBX_ERR_INVALID, "null lattice");
  if (steps < 0) return fail(LBX_ERR_INVALID, "steps must be >= 0");
  DeviceGuard guard(L->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  for (int64_t k = 0; k < steps; ++k) {
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    if (int rc = step_collide(L, ((flags & LBX_STEP_STATISTICS) && k == steps - 1), s, ev)) return rc;
    if (int rc = step_post_stream(L, s)) return rc;
    if (ev[3]) {
      cudaEventRecord(ev[3], s);
      if (ev[0] && ev[1] && ev[2]) {
        for (auto e : ev) L->pending.push_back(e);
      }
    }
  }
  return LBX_OK;
}

int lbx_post_process(lbx_lattice L, void* stream) {
  if (!L) return fail(LBX_ERR_INVALID, "null lattice");
  if (L->nLinks == 0 && L->nFd == 0) return LBX_OK;
  DeviceGuard guard(L->device);
  const LaunchArgs b = args_of(L);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (L->nLinks > 0)
    LBX_CUDA_TRY(LBX_DISPATCH(L, (launch_bouzidi<Q, S>(b, L->linkCell, L->linkDir, L->linkDelta, L->nLinks, s))));
  if (L->nFd > 0) LBX_CUDA_TRY(LBX_DISPATCH(L, (launch_fd_boundary<Q, S>(b, s))));
  return LBX_OK;
}

int lbx_set_kernel_timing(lbx_lattice L, int32_t enable) {
  if (!L) return fail(LBX_ERR_INVALID, "null lattice");
  DeviceGuard guard(L->device);
  drain_timing(L);
  L->timing = enable != 0;
  for (int k = 0; k < 3; ++k) {
    L->timedMs[k] = 0;
    L->timedLaunches[k] = 0;
  }
  return LBX_OK;
}

int lbx_get_kernel_timing(lbx_lattice L, double out[6]) {
  if (!L || !out) return fail(LBX_ERR_INVALID, "null argument");
  DeviceGuard guard(L->device);
  drain_timing(L);
  for (int k = 0; k < 3; ++k) {
    out[k] = L->timedMs[k];
    out[3 + k] = double(L->timedLaunches[k]);
  }
  return LBX_OK;
}

int lbx_get_statistics(lbx_lattice L, double out[4], void* stream) {
  if (!L || !out) return fail(LBX_ERR_INVALID, "null argument");
  DeviceGuard guard(L->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  StatAcc h;
  int kerr = 0;
  LBX_CUDA_TRY(cudaMemcpyAsync(&h, L->stats, sizeof(StatAcc), cudaMemcpyDeviceToHost, s));
  LBX_CUDA_TRY(cudaMemcpyAsync(&kerr, L->devErr, sizeof(int), cudaMemcpyDeviceToHost, s));
  LBX_CUDA_TRY(cudaStreamSynchronize(s));
  if (kerr) {
    cudaMemset(L->devErr, 0, sizeof(int));
    return fail(LBX_ERR_CUDA, "a step kernel gave up waiting for its bulk copies; results of that step are invalid");
  }
  double mx;
  std::memcpy(&mx, &h.maxbits, sizeof(double));
  const double cnt = double(h.count);
  out[0] = h.count ? h.sum[0] / cnt : 1.0;
  out[1] = h.count ? 0.5 * h.sum[1] / cnt : 1.0;
  out[2] = std::sqrt(mx);
  out[3] = cnt;
  return LBX_OK;
}

int lbx_compute_moments(lbx_lattice L, double* rho, double* u, void* stream) {
  if (!L) return fail(LBX_ERR_INVALID, "null lattice");
  if (!rho && !u) return LBX_OK;
  DeviceGuard guard(L->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t nb = size_t(L->ncore) * sizeof(double);
  double* dev = nullptr;
  LBX_CUDA_TRY(cudaMalloc(&dev, nb * size_t(1 + L->d)));
  const LaunchArgs a = args_of(L);
  cudaError_t e = LBX_DISPATCH(L, (launch_moments<Q, S>(a, dev, dev + L->ncore, s)));
  if (e == cudaSuccess && rho) e = cudaMemcpyAsync(rho, dev, nb, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && u) e = cudaMemcpyAsync(u, dev + L->ncore, nb * size_t(L->d), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(dev);
  LBX_CUDA_TRY(e);
  return LBX_OK;
}

int lbx_reduce(lbx_lattice L, int32_t what, double* out, void* stream) {
  if (!L || !out) return fail(LBX_ERR_INVALID, "null argument");
  if (what != LBX_REDUCE_MASS_MOMENTUM && what != LBX_REDUCE_DRAG && what != LBX_REDUCE_RESIDUAL)
    return fail(LBX_ERR_INVALID, "unknown reduction");
  DeviceGuard guard(L->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const LaunchArgs a = args_of(L);
  // per-block entries (4 doubles per block of 256 cells or links), then a fixed-order sum
  const int64_t need = reduce_blocks(std::max<int64_t>(L->ncore, L->nLinks)) + 1;
  if (need > L->reducePartCapacity) {
    cudaFree(L->reducePart);
    L->reducePart = nullptr;
    L->reducePartCapacity = 0;
    LBX_CUDA_TRY(cudaMalloc(&L->reducePart, size_t(need) * 4 * sizeof(double)));
    L->reducePartCapacity = need;
  }
  double h[4] = {};
  switch (what) {
  case LBX_REDUCE_MASS_MOMENTUM:
    LBX_CUDA_TRY(LBX_DISPATCH(L, (launch_mass_momentum<Q, S>(a, L->reducePart, L->reduceAcc, s))));
    break;
  case LBX_REDUCE_DRAG:
    LBX_CUDA_TRY(LBX_DISPATCH(L, (launch_link_force<Q, S>(a, L->linkCell, L->linkDir, L->linkGroup, -1, L->nLinks,
                                                          L->reducePart, L->reduceAcc, s))));
    break;
  default:
    if (!L->residualSnap) {
      LBX_CUDA_TRY(cudaMalloc(&L->residualSnap, size_t(L->ncore) * size_t(L->d) * sizeof(float)));
      LBX_CUDA_TRY(cudaMemsetAsync(L->residualSnap, 0, size_t(L->ncore) * size_t(L->d) * sizeof(float), s));
    }
    LBX_CUDA_TRY(LBX_DISPATCH(L, (launch_residual<Q, S>(a, L->residualSnap, L->reducePart, L->reduceAcc, s))));
  }
  LBX_CUDA_TRY(cudaMemcpyAsync(h, L->reduceAcc, 4 * sizeof(double), cudaMemcpyDeviceToHost, s));
  LBX_CUDA_TRY(cudaStreamSynchronize(s));
  switch (what) {
  case LBX_REDUCE_MASS_MOMENTUM:
    for (int k = 0; k < 4; ++k) out[k] = h[k];
    break;
  case LBX_REDUCE_DRAG:
    for (int k = 0; k < 3; ++k) out[k] = h[k];
    break;
  default:
    out[0] = std::sqrt(h[0]);
    out[1] = std::sqrt(h[1]);
    out[2] = h[2];
  }
  return LBX_OK;
}

int lbx_boundary_force(lbx_lattice L, int32_t group, double out[3], void* stream) {
  if (!L || !out) return fail(LBX_ERR_INVALID, "null argument");
  if (group < -1 || group > 254) return fail(LBX_ERR_INVALID, "group must be -1 (all links) or a solid index");
  DeviceGuard guard(L->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const LaunchArgs a = args_of(L);
  const int64_t need = reduce_blocks(std::max<int64_t>(L->ncore, L->nLinks)) + 1;
  if (need > L->reducePartCapacity) {
    cudaFree(L->reducePart);
    L->reducePart = nullptr;
    L->reducePartCapacity = 0;
    LBX_CUDA_TRY(cudaMalloc(&L->reducePart, size_t(need) * 4 * sizeof(double)));
    L->reducePartCapacity = need;
  }
  double h[4] = {};
  LBX_CUDA_TRY(LBX_DISPATCH(L, (launch_link_force<Q, S>(a, L->linkCell, L->linkDir, L->linkGroup, group, L->nLinks,
                                                        L->reducePart, L->reduceAcc, s))));
  LBX_CUDA_TRY(cudaMemcpyAsync(h, L->reduceAcc, 4 * sizeof(double), cudaMemcpyDeviceToHost, s));
  LBX_CUDA_TRY(cudaStreamSynchronize(s));
  for (int k = 0; k < 3; ++k) out[k] = h[k];
  return LBX_OK;
}

int lbx_population_shift(lbx_lattice L, int32_t pop, int64_t* shift) {
  if (!L || !shift) return fail(LBX_ERR_INVALID, "null argument");
  if (pop < 0 || pop >= L->q) return fail(LBX_ERR_INVALID, "population index out of range");
  *shift = L->shift[pop];
  return LBX_OK;
}

int lbx_population_ptr(lbx_lattice L, int32_t pop, void** ptr, int64_t* shift) {
  if (!L || !ptr || !shift) return fail(LBX_ERR_INVALID, "null argument");
  if (pop < 0 || pop >= L->q) return fail(LBX_ERR_INVALID, "population index out of range");
  char* column = static_cast<char*>(L->pop) + size_t(pop) * size_t(L->stride) * storage_bytes(L->storage);
  if (L->doubled) {  // the second mapping makes [shift, shift + period) one contiguous run
    *ptr = column + size_t(L->shift[pop]) * storage_bytes(L->storage);
    *shift = 0;
  } else {
    *ptr = column;
    *shift = L->shift[pop];
  }
  return LBX_OK;
}

int lbx_rotate(lbx_lattice L, int32_t pop, int64_t offset) {
  if (!L) return fail(LBX_ERR_INVALID, "null lattice");
  if (pop < 0 || pop >= L->q) return fail(LBX_ERR_INVALID, "population index out of range");
  int64_t s = (L->shift[pop] - offset) % L->period;
  if (s < 0) s += L->period;
  L->shift[pop] = s;
  return LBX_OK;
}

int lbx_set_launch_config(lbx_lattice L, int32_t variant, int32_t block_x, int32_t block_y,
                          int32_t cells_per_thread) {
  if (!L) return fail(LBX_ERR_INVALID, "null lattice");
  if (variant < 0 || variant > 5) return fail(LBX_ERR_INVALID, "variant must be 0, 1, 2, 3, 4 or 5");
  if (L->classMask && variant != 1)
    return fail(LBX_ERR_UNSUPPORTED, "a lattice with parameter classes steps with launch variant 1");
  if ((variant == 3 || variant == 4) && (!L->doubled || L->period >= (int64_t(1) << 31)))
    return fail(LBX_ERR_UNSUPPORTED, "variants 3 and 4 (bulk copies) need the doubled column mapping and fewer than 2^31 cells");
  if (groups_kernel(variant) && L->period >= (int64_t(1) << 31))
    return fail(LBX_ERR_UNSUPPORTED, "variants 2 and 5 need a column period below 2^31 cells");
  if (groups_kernel(variant) && cells_per_thread != 1 && cells_per_thread != 2 &&
      !(cells_per_thread == 4 && storage_bytes(L->storage) == 2))
    return fail(LBX_ERR_INVALID, "cells_per_thread must be 1 or 2 (or 4 for 16-bit storage)");
  if (variant != 0) {
    if (block_x < 1 || block_y < 1 || block_x * block_y > 256 || (block_x * block_y) % 32 != 0)
      return fail(LBX_ERR_INVALID, "block must hold a multiple of 32 and at most 256 threads");
    L->blockX = block_x;
    L->blockY = block_y;
  }
  L->cellsPerThread = groups_kernel(variant) ? cells_per_thread : 1;
  L->kernel = variant;
  return LBX_OK;
}


int lbx_autotune(lbx_lattice L, int32_t steps, lbx_tune_entry* out, int32_t capacity, int32_t* n_out, void* stream) {
  if (!L) return fail(LBX_ERR_INVALID, "null lattice");
  if (steps < 1 || capacity < 0 || (capacity > 0 && !out)) return fail(LBX_ERR_INVALID, "bad steps or output array");
  DeviceGuard guard(L->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // Candidates: the three kernels, block shapes along the fastest axis from 32 to 256 cells,
  // full (256-thread) and half (128-thread) blocks, one or two cells per thread for variant 2.
  struct Cand { int variant, bx, by, k; };
  std::vector<Cand> cands;
  const int nf = (L->d == 3) ? L->core[2] : L->core[1];
  const int maxK = storage_bytes(L->storage) == 2 ? 4 : 2;
  for (int k = 1; k <= maxK && !L->classMask; k *= 2)
    for (int bx = 32; bx <= 256; bx *= 2) {
      if (bx > 32 && bx >= 2 * lbx::k_cells_threads(nf, k)) break;  // wider blocks only idle more threads
      for (int threads = 256; threads >= 128; threads /= 2)
        if (threads / bx >= 1) cands.push_back({2, bx, threads / bx, k});
      // variant 5 (the L2 prefetch) with one row a block: the shapes where it can pay
      if (L->doubled && bx >= 128) cands.push_back({5, bx, 1, k});
    }
  {
    int bx, by;
    block_shape_for(nf, 1, bx, by);
    cands.push_back({1, bx, by, 1});
    if (L->classMask) {  // the classes run on variant 1 only: its block shapes
      for (int bx1 = 32; bx1 <= 256; bx1 *= 2)
        if (bx1 != bx) cands.push_back({1, bx1, 256 / bx1, 1});
    }
    if (!L->classMask) cands.push_back({0, 256, 1, 1});
    if (!L->classMask && L->doubled && L->period < (int64_t(1) << 31)) {
      cands.push_back({3, 256, 1, 1});
      cands.push_back({4, 256, 1, 1});
    }
  }
  if (n_out) *n_out = int32_t(cands.size());
  const Cand keep{L->kernel, L->blockX, L->blockY, L->cellsPerThread};
  // saved state: every column's period of populations and the shifts
  const size_t es = storage_bytes(L->storage);
  const size_t colBytes = size_t(L->period) * es, pitch = size_t(L->stride) * es;
  void* saved = nullptr;
  cudaError_t e = cudaMalloc(&saved, colBytes * size_t(L->q));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? LBX_ERR_OUT_OF_MEMORY : LBX_ERR_CUDA,
                std::string("autotune state copy: ") + cudaGetErrorString(e));
  }
  int64_t shift0[27];
  std::memcpy(shift0, L->shift, sizeof(shift0));
  // the statistics too: ConstRhoBGK reads the last step's average density from them
  StatAcc stats0;
  cudaError_t estat = cudaMemcpyAsync(&stats0, L->stats, sizeof(StatAcc), cudaMemcpyDeviceToHost, s);
  if (estat == cudaSuccess) estat = cudaStreamSynchronize(s);
  if (estat != cudaSuccess) {
    cudaFree(saved);
    return fail(LBX_ERR_CUDA, std::string("autotune state copy: ") + cudaGetErrorString(estat));
  }
  const bool timing0 = L->timing;
  if (timing0) drain_timing(L);
  L->timing = false;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  auto restore = [&]() -> cudaError_t {
    std::memcpy(L->shift, shift0, sizeof(shift0));
    cudaError_t r = cudaMemcpyAsync(L->stats, &stats0, sizeof(StatAcc), cudaMemcpyHostToDevice, s);
    if (r != cudaSuccess) return r;
    return cudaMemcpy2DAsync(L->pop, pitch, saved, colBytes, colBytes, size_t(L->q), cudaMemcpyDeviceToDevice, s);
  };
  e = cudaMemcpy2DAsync(saved, colBytes, L->pop, pitch, colBytes, size_t(L->q), cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  int best = -1;
  float bestMs = 0.f;
  int rc = LBX_OK;
  for (size_t i = 0; i < cands.size() && e == cudaSuccess && rc == LBX_OK; ++i) {
    const Cand& c = cands[i];
    float ms = -1.f;
    if (lbx_set_launch_config(L, c.variant, c.bx, c.by, c.k) == LBX_OK) {
      e = restore();
      if (e == cudaSuccess) rc = lbx_collide_and_stream(L, 1, 0, stream);  // warm-up
      if (e == cudaSuccess && rc == LBX_OK) e = cudaEventRecord(e0, s);
      if (e == cudaSuccess && rc == LBX_OK) rc = lbx_collide_and_stream(L, steps, 0, stream);
      if (e == cudaSuccess && rc == LBX_OK) e = cudaEventRecord(e1, s);
      if (e == cudaSuccess && rc == LBX_OK) e = cudaEventSynchronize(e1);
      if (e == cudaSuccess && rc == LBX_OK) e = cudaEventElapsedTime(&ms, e0, e1);
      if (e == cudaSuccess && rc == LBX_OK) {
        ms /= float(steps);
        if (best < 0 || ms < bestMs) {
          best = int(i);
          bestMs = ms;
        }
      }
    }
    if (out && int32_t(i) < capacity) out[i] = lbx_tune_entry{c.variant, c.bx, c.by, c.k, 0, 0, double(ms)};
  }
  const std::string err = rc != LBX_OK ? std::string(lbx_last_error()) : std::string();
  cudaError_t e2 = restore();
  if (e2 == cudaSuccess) e2 = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = e2;
  cudaFree(saved);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  L->timing = timing0;
  const Cand pick = best >= 0 ? cands[size_t(best)] : keep;
  L->kernel = pick.variant;
  L->blockX = pick.bx;
  L->blockY = pick.by;
  L->cellsPerThread = pick.k;
  if (rc != LBX_OK) return fail(rc, "autotune: " + err);
  if (e != cudaSuccess) return fail(LBX_ERR_CUDA, std::string("autotune: ") + cudaGetErrorString(e));
  return LBX_OK;
}

}  // extern "C"

// ---- slab decomposition (lbx_slabs_*) -----------------------------------------------------
// One lattice cut along x into slabs, each an lbx_lattice of its own (on one device, or on
// several devices of this process), stepped in lock-step with one face exchange per step between
// the collision and the post-stream phase -- the single-process form of the reference's block
// decomposition and overlap communication (core/superLattice.hh:150-155,
// core/platform/gpu/cuda/communicator.hh:355-510).
//
// After a slab's collision and shift rotation, every population that left the slab across an x
// face sits in the slab's own ghost plane (x = -1 or nx): the plain store of the step kernel put
// it at the slot that the rotation then associates with the ghost cell.  The exchange copies it
// into the neighbour slab's first (or last) plane, at the target cell the population reaches in
// the whole lattice (across periodic y and z faces too).  Copies come only from cells that are
// stepped: the population of a cell without dynamics is supplied by the link that faces it, as
// in the whole lattice.  Each directed face is a list of (source slot, target slot) pairs made on
// the host from the slabs' cell maps (remade when a map changes); per step the sending slab
// gathers the listed slots into a face buffer (its own memory), the buffer crosses to the
// receiving device by cudaMemcpyPeerAsync when the slabs sit on different devices, and the
// receiving slab scatters it into its slots.  Each slab runs on a stream of its own; events order
// a gather after the sender's collision, the scatter after the receiver's collision, and the
// next gather into the buffer after the last scatter from it.
namespace {

struct SlabFace {
  int src = 0, dst = 0;             // slab indices
  int64_t n = 0;                    // listed slots
  uint32_t* srcCell = nullptr;      // on the sender's device
  uint8_t* srcDir = nullptr;
  uint32_t* dstCell = nullptr;      // on the receiver's device
  uint8_t* dstDir = nullptr;
  void* sendBuf = nullptr;          // sender's device
  void* recvBuf = nullptr;          // receiver's device (nullptr: same device, scatter reads sendBuf)
  cudaEvent_t sent = nullptr;       // recorded on the sender's stream after the gather
  cudaEvent_t consumed = nullptr;   // recorded on the receiver's stream after the scatter
};

void free_face(SlabFace& f, const std::vector<lbx_lattice_s*>& slabs) {
  {
    DeviceGuard g(slabs[size_t(f.src)]->device);
    cudaFree(f.srcCell);
    cudaFree(f.srcDir);
    cudaFree(f.sendBuf);
    if (f.sent) cudaEventDestroy(f.sent);
  }
  {
    DeviceGuard g(slabs[size_t(f.dst)]->device);
    cudaFree(f.dstCell);
    cudaFree(f.dstDir);
    cudaFree(f.recvBuf);
    if (f.consumed) cudaEventDestroy(f.consumed);
  }
  f = SlabFace{};
}

}  // namespace

struct lbx_slabs_s {
  int q = 19, d = 3, storage = LBX_F32;
  int core[3] = {0, 0, 0}, periodic[3] = {0, 0, 0};
  std::vector<lbx_lattice_s*> slab;
  std::vector<int> x0;
  std::vector<cudaStream_t> stream;
  std::vector<SlabFace> face;
  std::vector<uint64_t> versions;  // the slabs' map versions the face lists were made from
  bool facesBuilt = false;
};

namespace {

// Whether padded cell n of a slab is stepped by its own kernels (any kind but "no dynamics").
bool slab_stepped(const lbx_lattice_s* L, int64_t n) {
  return L->hostMap.empty() ? true : L->hostMap[size_t(n)] != LBX_CELL_NONE;
}

// The (source slot, target slot) pairs of the face from slab `a` to its neighbour `b`; side +1:
// b lies at higher x (populations with c_x = +1 enter b's plane x = 0), -1: at lower x.
void face_pairs(const lbx_lattice_s* A, const lbx_lattice_s* B, int side, std::vector<uint32_t>& sc,
                std::vector<uint8_t>& sd, std::vector<uint32_t>& dc, std::vector<uint8_t>& dd) {
  const Geometry ga = geometry_of(A), gb = geometry_of(B);
  const int ny = ga.ny, nz = ga.nz;
  const int xs = side > 0 ? ga.nx - 1 : 0, xt = side > 0 ? 0 : gb.nx - 1;
  auto pad = [](const Geometry& g, int x, int y, int z) {
    return int64_t(x + 1) * g.sx + int64_t(y + 1) * g.sy + (z + g.pz);
  };
  for (int i = 1; i < A->q; ++i) {
    const int* c = velocity(A->q, i);
    if (c[0] != side) continue;
    const int cy = c[1], cz = A->d == 3 ? c[2] : 0;
    for (int yt = 0; yt < ny; ++yt)
      for (int zt = 0; zt < nz; ++zt) {
        int ys = yt - cy, zs = zt - cz;
        if (ys < 0 || ys >= ny) {
          if (!A->periodic[1]) continue;
          ys = (ys + ny) % ny;
        }
        if (zs < 0 || zs >= nz) {
          if (A->d != 3 || !A->periodic[2]) continue;
          zs = (zs + nz) % nz;
        }
        if (!slab_stepped(A, pad(ga, xs, ys, zs))) continue;
        sc.push_back(uint32_t(pad(ga, xs + side, ys + cy, zs + cz)));
        sd.push_back(uint8_t(i));
        dc.push_back(uint32_t(pad(gb, xt, yt, zt)));
        dd.push_back(uint8_t(i));
      }
  }
}

template <typename T>
cudaError_t upload_vec(T** dst, const std::vector<T>& v) {
  *dst = nullptr;
  if (v.empty()) return cudaSuccess;
  cudaError_t e = cudaMalloc(dst, v.size() * sizeof(T));
  if (e == cudaSuccess) e = cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
  return e;
}

int build_faces(lbx_slabs_s* S) {
  for (auto& f : S->face) free_face(f, S->slab);
  S->face.clear();
  const int ns = int(S->slab.size());
  for (int k = 0; k < ns; ++k) {
    const int up = k + 1 < ns ? k + 1 : (S->periodic[0] ? 0 : -1);
    if (up < 0 || up == k) continue;
    for (int side : {+1, -1}) {
      SlabFace f;
      f.src = side > 0 ? k : up;
      f.dst = side > 0 ? up : k;
      std::vector<uint32_t> sc, dc;
      std::vector<uint8_t> sd, dd;
      face_pairs(S->slab[size_t(f.src)], S->slab[size_t(f.dst)], side, sc, sd, dc, dd);
      f.n = int64_t(sc.size());
      const lbx_lattice_s* A = S->slab[size_t(f.src)];
      const lbx_lattice_s* B = S->slab[size_t(f.dst)];
      const size_t bytes = size_t(std::max<int64_t>(f.n, 1)) * size_t(storage_bytes(A->storage));
      cudaError_t e;
      {
        DeviceGuard g(A->device);
        e = upload_vec(&f.srcCell, sc);
        if (e == cudaSuccess) e = upload_vec(&f.srcDir, sd);
        if (e == cudaSuccess) e = cudaMalloc(&f.sendBuf, bytes);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&f.sent, cudaEventDisableTiming);
      }
      if (e == cudaSuccess) {
        DeviceGuard g(B->device);
        e = upload_vec(&f.dstCell, dc);
        if (e == cudaSuccess) e = upload_vec(&f.dstDir, dd);
        if (e == cudaSuccess && B->device != A->device) e = cudaMalloc(&f.recvBuf, bytes);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&f.consumed, cudaEventDisableTiming);
      }
      S->face.push_back(f);
      if (e != cudaSuccess)
        return fail(e == cudaErrorMemoryAllocation ? LBX_ERR_OUT_OF_MEMORY : LBX_ERR_CUDA,
                    std::string("slab face set-up: ") + cudaGetErrorString(e));
    }
  }
  S->versions.clear();
  for (auto* L : S->slab) S->versions.push_back(L->mapVersion);
  S->facesBuilt = true;
  return LBX_OK;
}

bool faces_stale(const lbx_slabs_s* S) {
  if (!S->facesBuilt) return true;
  for (size_t k = 0; k < S->slab.size(); ++k)
    if (S->versions[k] != S->slab[k]->mapVersion) return true;
  return false;
}

void destroy_slabs(lbx_slabs_s* S) {
  for (auto& f : S->face) free_face(f, S->slab);
  for (size_t k = 0; k < S->slab.size(); ++k) {
    if (k < S->stream.size() && S->stream[k]) {
      DeviceGuard g(S->slab[k]->device);
      cudaStreamDestroy(S->stream[k]);
    }
    lbx_lattice_destroy(S->slab[k]);
  }
  delete S;
}

}  // namespace

extern "C" {

int lbx_slabs_create(int32_t q, const int32_t core[3], const int32_t periodic[3], int32_t storage, int32_t n_slabs,
                     const int32_t* devices, lbx_slabs* out) {
  if (!out || !core) return fail(LBX_ERR_INVALID, "null argument");
  *out = nullptr;
  if (n_slabs < 1) return fail(LBX_ERR_INVALID, "n_slabs must be >= 1");
  if (core[0] < 2 * n_slabs) return fail(LBX_ERR_INVALID, "every slab needs at least two x planes");
  auto* S = new lbx_slabs_s();
  S->q = q;
  S->d = q == 9 ? 2 : 3;
  S->storage = storage;
  for (int a = 0; a < 3; ++a) {
    S->core[a] = core[a];
    S->periodic[a] = periodic ? (periodic[a] != 0) : 0;
  }
  int x = 0;
  for (int k = 0; k < n_slabs; ++k) {
    const int nx = core[0] / n_slabs + (k < core[0] % n_slabs ? 1 : 0);
    const int32_t sc[3] = {nx, core[1], core[2]};
    // x is periodic inside a slab only when it is the whole lattice
    const int32_t sp[3] = {n_slabs == 1 ? S->periodic[0] : 0, S->periodic[1], S->periodic[2]};
    lbx_lattice L = nullptr;
    if (int rc = lbx_lattice_create(q, sc, sp, storage, devices ? devices[k] : 0, &L)) {
      const std::string msg = g_error;
      destroy_slabs(S);
      return fail(rc, "slab " + std::to_string(k) + ": " + msg);
    }
    S->slab.push_back(L);
    S->x0.push_back(x);
    x += nx;
    cudaStream_t st = nullptr;
    DeviceGuard g(L->device);
    cudaError_t e = cudaStreamCreate(&st);
    S->stream.push_back(st);
    if (e != cudaSuccess) {
      destroy_slabs(S);
      return fail(LBX_ERR_CUDA, std::string("slab stream: ") + cudaGetErrorString(e));
    }
  }
  // slabs on different devices read nothing of each other (the face buffers cross by copies),
  // but direct peer copies need peer access where the devices offer it
  for (size_t a = 0; a < S->slab.size(); ++a)
    for (size_t b = 0; b < S->slab.size(); ++b) {
      const int da = S->slab[a]->device, db = S->slab[b]->device;
      if (da == db) continue;
      int can = 0;
      if (cudaDeviceCanAccessPeer(&can, da, db) == cudaSuccess && can) {
        DeviceGuard g(da);
        if (cudaDeviceEnablePeerAccess(db, 0) != cudaSuccess) cudaGetLastError();  // already enabled
      }
    }
  *out = S;
  return LBX_OK;
}

int lbx_slabs_destroy(lbx_slabs S) {
  if (!S) return LBX_OK;
  for (size_t k = 0; k < S->slab.size(); ++k) {
    DeviceGuard g(S->slab[k]->device);
    cudaStreamSynchronize(S->stream[k]);
  }
  destroy_slabs(S);
  return LBX_OK;
}

int lbx_slabs_get(lbx_slabs S, int32_t k, lbx_lattice* lattice, int32_t* x0, int32_t* nx) {
  if (!S || k < 0 || k >= int32_t(S->slab.size())) return fail(LBX_ERR_INVALID, "no such slab");
  if (lattice) *lattice = S->slab[size_t(k)];
  if (x0) *x0 = S->x0[size_t(k)];
  if (nx) *nx = S->slab[size_t(k)]->core[0];
  return LBX_OK;
}

int lbx_slabs_collide_and_stream(lbx_slabs SL, int64_t steps, uint32_t flags) {
  if (!SL) return fail(LBX_ERR_INVALID, "null slabs");
  if (steps < 0) return fail(LBX_ERR_INVALID, "steps must be >= 0");
  for (auto* L : SL->slab)
    if (L->dynamics == LBX_CONST_RHO_BGK)
      return fail(LBX_ERR_UNSUPPORTED, "ConstRhoBGK couples every cell to the whole lattice's density; not on slabs");
  if (faces_stale(SL))
    if (int rc = build_faces(SL)) return rc;
  const size_t ns = SL->slab.size();
  for (int64_t k = 0; k < steps; ++k) {
    const bool stats = (flags & LBX_STEP_STATISTICS) && k == steps - 1;
    for (size_t j = 0; j < ns; ++j) {
      lbx_lattice_s* L = SL->slab[j];
      DeviceGuard g(L->device);
      cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
      const bool timing = L->timing;
      L->timing = false;  // per-kernel timing is a single-lattice tool
      const int rc = step_collide(L, stats, SL->stream[j], ev);
      L->timing = timing;
      if (rc) return rc;
    }
    for (auto& f : SL->face) {
      lbx_lattice_s* A = SL->slab[size_t(f.src)];
      lbx_lattice_s* B = SL->slab[size_t(f.dst)];
      cudaStream_t sa = SL->stream[size_t(f.src)], sb = SL->stream[size_t(f.dst)];
      const size_t bytes = size_t(f.n) * size_t(storage_bytes(A->storage));
      {
        DeviceGuard g(A->device);
        // the buffer is free once the previous step's scatter has read it
        if (f.consumed && k > 0) LBX_CUDA_TRY(cudaStreamWaitEvent(sa, f.consumed, 0));
        const LaunchArgs a = args_of(A);
        LBX_CUDA_TRY(LBX_DISPATCH(A, (launch_face_copy<Q, S>(a, f.sendBuf, f.srcCell, f.srcDir, f.n, true, sa))));
        LBX_CUDA_TRY(cudaEventRecord(f.sent, sa));
      }
      {
        DeviceGuard g(B->device);
        LBX_CUDA_TRY(cudaStreamWaitEvent(sb, f.sent, 0));
        void* in = f.sendBuf;
        if (f.recvBuf) {
          if (bytes) LBX_CUDA_TRY(cudaMemcpyPeerAsync(f.recvBuf, B->device, f.sendBuf, A->device, bytes, sb));
          in = f.recvBuf;
        }
        const LaunchArgs b = args_of(B);
        LBX_CUDA_TRY(LBX_DISPATCH(B, (launch_face_copy<Q, S>(b, in, f.dstCell, f.dstDir, f.n, false, sb))));
        LBX_CUDA_TRY(cudaEventRecord(f.consumed, sb));
      }
    }
    for (size_t j = 0; j < ns; ++j) {
      lbx_lattice_s* L = SL->slab[j];
      DeviceGuard g(L->device);
      if (int rc = step_post_stream(L, SL->stream[j])) return rc;
    }
  }
  return LBX_OK;
}

int lbx_slabs_synchronize(lbx_slabs S) {
  if (!S) return fail(LBX_ERR_INVALID, "null slabs");
  for (size_t k = 0; k < S->slab.size(); ++k) {
    DeviceGuard g(S->slab[k]->device);
    LBX_CUDA_TRY(cudaStreamSynchronize(S->stream[k]));
  }
  return LBX_OK;
}

int lbx_slabs_get_statistics(lbx_slabs S, double out[4]) {
  if (!S || !out) return fail(LBX_ERR_INVALID, "null argument");
  if (int rc = lbx_slabs_synchronize(S)) return rc;
  double sumRho = 0.0, sumE = 0.0, maxU = 0.0, cells = 0.0;
  for (auto* L : S->slab) {
    double st[4];
    if (int rc = lbx_get_statistics(L, st, nullptr)) return rc;
    sumRho += st[0] * st[3];
    sumE += st[1] * st[3];
    maxU = std::max(maxU, st[2]);
    cells += st[3];
  }
  out[0] = cells > 0 ? sumRho / cells : 1.0;
  out[1] = cells > 0 ? sumE / cells : 1.0;
  out[2] = maxU;
  out[3] = cells;
  return LBX_OK;
}

}  // extern "C"
