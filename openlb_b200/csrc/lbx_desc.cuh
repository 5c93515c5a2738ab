// Velocity-set traits for the B200 kernels.
//
// The tables restate the reference descriptors (src/descriptor/definition/common.h: D2Q9
// :91-109, D3Q19 :167-196, D3Q27 :360-399).  The population ordering (c_i = -c_{i+(q-1)/2},
// common.h:30-40), opposites and weights must be identical to the reference's because the
// stored arrays and the C ABI exchange populations in that order.  Every table access in
// device code happens at a compile-time index (static_for below), so the tables fold into
// immediates and never live in memory.
#pragma once

#include <cstdint>
#include <utility>

namespace lbx {

template <int Q> struct Desc;

template <> struct Desc<9> {
  static constexpr int q = 9;
  static constexpr int d = 2;
  static constexpr int C[9][3] = {{0, 0, 0},  {-1, 1, 0}, {-1, 0, 0}, {-1, -1, 0}, {0, -1, 0},
                                  {1, -1, 0}, {1, 0, 0},  {1, 1, 0},  {0, 1, 0}};
  static constexpr int OPP[9] = {0, 5, 6, 7, 8, 1, 2, 3, 4};
  static constexpr int WN[9] = {4, 1, 1, 1, 1, 1, 1, 1, 1};
  static constexpr int WD[9] = {9, 36, 9, 36, 9, 36, 9, 36, 9};
};

template <> struct Desc<19> {
  static constexpr int q = 19;
  static constexpr int d = 3;
  static constexpr int C[19][3] = {{0, 0, 0},   {-1, 0, 0}, {0, -1, 0}, {0, 0, -1}, {-1, -1, 0},
                                   {-1, 1, 0},  {-1, 0, -1}, {-1, 0, 1}, {0, -1, -1}, {0, -1, 1},
                                   {1, 0, 0},   {0, 1, 0},  {0, 0, 1},  {1, 1, 0},  {1, -1, 0},
                                   {1, 0, 1},   {1, 0, -1}, {0, 1, 1},  {0, 1, -1}};
  static constexpr int OPP[19] = {0, 10, 11, 12, 13, 14, 15, 16, 17, 18, 1, 2, 3, 4, 5, 6, 7, 8, 9};
  static constexpr int WN[19] = {1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1};
  static constexpr int WD[19] = {3, 18, 18, 18, 36, 36, 36, 36, 36, 36, 18, 18, 18, 36, 36, 36, 36, 36, 36};
};

template <> struct Desc<27> {
  static constexpr int q = 27;
  static constexpr int d = 3;
  static constexpr int C[27][3] = {
      {0, 0, 0},   {-1, 0, 0},  {0, -1, 0},  {0, 0, -1}, {-1, -1, 0}, {-1, 1, 0},  {-1, 0, -1},
      {-1, 0, 1},  {0, -1, -1}, {0, -1, 1},  {-1, -1, -1}, {-1, -1, 1}, {-1, 1, -1}, {-1, 1, 1},
      {1, 0, 0},   {0, 1, 0},   {0, 0, 1},   {1, 1, 0},  {1, -1, 0},  {1, 0, 1},   {1, 0, -1},
      {0, 1, 1},   {0, 1, -1},  {1, 1, 1},   {1, 1, -1}, {1, -1, 1},  {1, -1, -1}};
  static constexpr int OPP[27] = {0, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24, 25, 26,
                                  1, 2,  3,  4,  5,  6,  7,  8,  9,  10, 11, 12, 13};
  static constexpr int WN[27] = {8, 2, 2, 2, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1,
                                 2, 2, 2, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1};
  static constexpr int WD[27] = {27, 27, 27, 27, 54, 54, 54, 54, 54, 54, 216, 216, 216, 216,
                                 27, 27, 27, 54, 54, 54, 54, 54, 54, 216, 216, 216, 216};
};

// Compile-time loop: f(std::integral_constant<int, I>) for I = 0 .. N-1.
template <class F, int... Is>
__host__ __device__ __forceinline__ void static_for_impl(F&& f, std::integer_sequence<int, Is...>) {
  (f(std::integral_constant<int, Is>{}), ...);
}
template <int N, class F>
__host__ __device__ __forceinline__ void static_for(F&& f) {
  static_for_impl(f, std::make_integer_sequence<int, N>{});
}

// Weight t_i in the arithmetic R, computed as R(num) / R(den) like the reference's Fraction
// conversion (descriptors::t<V,DESCRIPTOR>).
template <int Q, typename R>
__host__ __device__ constexpr R weight(int i) {
  return R(Desc<Q>::WN[i]) / R(Desc<Q>::WD[i]);
}

}  // namespace lbx
