// lbx_mass_momentum_noalloc: the mass/momentum reduction for callers that cannot allocate
// device memory.
//
// The regular reduction (lbx_reduce with LBX_REDUCE_MASS_MOMENTUM) accumulates into scratch
// that the lattice handle obtained from cudaMalloc.  Some host programs cannot make that call:
// code running while a memory pool or arena owns all device memory, code inside a callback or
// a region where the driver allocator must not be entered, or an embedding that only hands out
// device buffers it already owns.  This unit gives them a reduction whose scratch lives in a
// file-scope __device__ array instead: the per-block partial sums go into g_partials, a second
// pass sums them in a fixed order, and the four totals are copied into the caller's host array.
//
// Limits and sharing (also stated in include/lbx.h):
//   - at most LBX_NOALLOC_MAX_BLOCKS blocks of LBX_NOALLOC_CELLS_PER_BLOCK cells, i.e.
//     LBX_NOALLOC_MAX_CELLS cells per call; larger arrays are rejected before any device work;
//   - g_partials (8192 blocks x 4 doubles = 256 KiB) exists on every GPU that loads the library
//     and is held until the process exits;
//   - every call uses the same array, so calls whose kernels overlap on the GPU (different
//     streams, or different host threads on one device) race and must be serialised by the
//     caller; each call writes every partial it later reads, so nothing needs clearing;
//   - every call looks up the device address of g_partials on the current device (see
//     partials_address) and synchronises the stream, so it must not be called while the stream
//     is being captured into a graph.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/lbx.h"
#include "lbx_kernels.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kCellsPerThread = LBX_NOALLOC_CELLS_PER_BLOCK / kThreads;
static_assert(LBX_NOALLOC_CELLS_PER_BLOCK % kThreads == 0, "cells per block must fill the threads");

// Scratch: {sum rho, sum j_x, sum j_y, sum j_z} per block, then the four totals.
static __device__ __align__(256) double g_partials[(LBX_NOALLOC_MAX_BLOCKS + 1) * 4];

}  // namespace

namespace lbx {
int set_error(int code, const std::string& msg);  // lbx_api.cu: the message lbx_last_error returns
}

namespace {

int noalloc_fail(int code, const std::string& msg) { return lbx::set_error(code, msg); }

// Device address of g_partials on the current device.  In host code the name g_partials only
// stands for the symbol; a kernel given &g_partials would touch host memory.  The address is
// looked up on every call, with the caller's device current: nothing is cached, so the call
// stays correct after a device reset and needs no locking between host threads.
cudaError_t partials_address(double** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_partials);
  if (e != cudaSuccess) return e;
  *out = static_cast<double*>(p);
  return cudaSuccess;
}

// Pass 1: block b sums rho = sum_i f_i + 1 and j = sum_i c_i f_i over its slice of cells.
template <int Q, typename S>
__global__ void __launch_bounds__(kThreads) k_noalloc_partials(const S* __restrict__ pop, int64_t n,
                                                               int64_t stride, double* __restrict__ partials) {
  using D = lbx::Desc<Q>;
  double v[4] = {0, 0, 0, 0};
  const int64_t first = int64_t(blockIdx.x) * LBX_NOALLOC_CELLS_PER_BLOCK;
#pragma unroll 1
  for (int r = 0; r < kCellsPerThread; ++r) {
    const int64_t c = first + int64_t(r) * kThreads + threadIdx.x;
    if (c >= n) break;
    double rho = 1.0;
    lbx::static_for<Q>([&](auto I) {
      const double fi = double(lbx::Storage<S>::load(pop + I * stride + c));
      rho += fi;
      lbx::static_for<D::d>([&](auto A) {
        constexpr int cc = D::C[I][A];
        if constexpr (cc != 0) v[1 + A] += cc * fi;
      });
    });
    v[0] += rho;
  }
  __shared__ double red[4][kThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    double a = v[k];
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) red[k][warp] = a;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double a = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) a += red[threadIdx.x][w];
    partials[int64_t(blockIdx.x) * 4 + threadIdx.x] = a;
  }
}

// Pass 2: the totals, summed over the blocks in index order (deterministic).
__global__ void k_noalloc_total(double* __restrict__ partials, int blocks) {
  if (threadIdx.x < 4) {
    double a = 0.0;
    for (int b = 0; b < blocks; ++b) a += partials[int64_t(b) * 4 + threadIdx.x];
    partials[int64_t(LBX_NOALLOC_MAX_BLOCKS) * 4 + threadIdx.x] = a;
  }
}

template <int Q, typename S>
cudaError_t launch_noalloc(const void* pop, int64_t n, int64_t stride, double* partials, int blocks,
                           cudaStream_t s) {
  k_noalloc_partials<Q, S><<<blocks, kThreads, 0, s>>>(static_cast<const S*>(pop), n, stride, partials);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_noalloc_total<<<1, 32, 0, s>>>(partials, blocks);
  return cudaGetLastError();
}

}  // namespace

extern "C" int lbx_mass_momentum_noalloc(int32_t q, int32_t storage, const void* populations, int64_t n_cells,
                                         int64_t column_stride, double out[4], void* stream) {
  if (!out) return noalloc_fail(LBX_ERR_INVALID, "out is null");
  if (q != 9 && q != 19 && q != 27) return noalloc_fail(LBX_ERR_UNSUPPORTED, "descriptor must be D2Q9, D3Q19 or D3Q27");
  if (storage < LBX_F64 || storage > LBX_BF16DEV) return noalloc_fail(LBX_ERR_INVALID, "unknown storage");
  if (n_cells < 1) return noalloc_fail(LBX_ERR_INVALID, "n_cells must be >= 1");
  if (n_cells > LBX_NOALLOC_MAX_CELLS)
    return noalloc_fail(LBX_ERR_INVALID, "n_cells " + std::to_string(n_cells) + " exceeds the static scratch limit of " +
                                             std::to_string(int64_t(LBX_NOALLOC_MAX_CELLS)) + " cells per call");
  if (column_stride < n_cells) return noalloc_fail(LBX_ERR_INVALID, "column_stride must be >= n_cells");
  if (!populations) return noalloc_fail(LBX_ERR_INVALID, "populations is null");
  double* partials = nullptr;
  cudaError_t e = partials_address(&partials);
  if (e != cudaSuccess) return noalloc_fail(LBX_ERR_CUDA, std::string("scratch set-up failed: ") + cudaGetErrorString(e));
  const int blocks = int((n_cells + LBX_NOALLOC_CELLS_PER_BLOCK - 1) / LBX_NOALLOC_CELLS_PER_BLOCK);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  switch (q * 4 + storage) {
  case 9 * 4 + LBX_F64: e = launch_noalloc<9, double>(populations, n_cells, column_stride, partials, blocks, s); break;
  case 9 * 4 + LBX_F32: e = launch_noalloc<9, float>(populations, n_cells, column_stride, partials, blocks, s); break;
  case 9 * 4 + LBX_F16DEV: e = launch_noalloc<9, __half>(populations, n_cells, column_stride, partials, blocks, s); break;
  case 9 * 4 + LBX_BF16DEV: e = launch_noalloc<9, __nv_bfloat16>(populations, n_cells, column_stride, partials, blocks, s); break;
  case 19 * 4 + LBX_F64: e = launch_noalloc<19, double>(populations, n_cells, column_stride, partials, blocks, s); break;
  case 19 * 4 + LBX_F32: e = launch_noalloc<19, float>(populations, n_cells, column_stride, partials, blocks, s); break;
  case 19 * 4 + LBX_F16DEV: e = launch_noalloc<19, __half>(populations, n_cells, column_stride, partials, blocks, s); break;
  case 19 * 4 + LBX_BF16DEV: e = launch_noalloc<19, __nv_bfloat16>(populations, n_cells, column_stride, partials, blocks, s); break;
  case 27 * 4 + LBX_F64: e = launch_noalloc<27, double>(populations, n_cells, column_stride, partials, blocks, s); break;
  case 27 * 4 + LBX_F32: e = launch_noalloc<27, float>(populations, n_cells, column_stride, partials, blocks, s); break;
  case 27 * 4 + LBX_F16DEV: e = launch_noalloc<27, __half>(populations, n_cells, column_stride, partials, blocks, s); break;
  case 27 * 4 + LBX_BF16DEV: e = launch_noalloc<27, __nv_bfloat16>(populations, n_cells, column_stride, partials, blocks, s); break;
  default: return noalloc_fail(LBX_ERR_INVALID, "bad descriptor/storage");
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out, partials + int64_t(LBX_NOALLOC_MAX_BLOCKS) * 4, 4 * sizeof(double),
                        cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return noalloc_fail(LBX_ERR_CUDA, std::string("reduction failed: ") + cudaGetErrorString(e));
  return LBX_OK;
}
