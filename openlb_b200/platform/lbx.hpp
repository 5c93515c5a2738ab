// lbx.hpp -- C++ host layer over the C ABI of liblbx.so (include/lbx.h).
//
// A new OpenLB platform binds the C ABI from C++. This header holds what that binding needs,
// written once:
//   - RAII ownership of a lattice handle;
//   - errors turned into exceptions, as the reference's CUDA platform does with device::check
//     (core/platform/gpu/cuda/device.hh:48-53): std::runtime_error, and std::domain_error for a combination
//     the library does not provide (the reference throws that for unsupported dynamics);
//   - compile-time mapping of dynamics and parameter tags to the ABI's ids.
// The names follow the reference's SuperLattice / BlockLattice API, so setup code reads like
// an OpenLB example:
//   defineDynamics<BGK>, setParameter<OMEGA>, setBouzidiBoundary, iniEquilibrium, initialize,
//   collideAndStream, getStatistics.
// No CUDA header is needed: streams are passed as void*.
#pragma once

#include <array>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "lbx.h"

namespace lbx {

// ---- errors ---------------------------------------------------------------------------------
inline void check(int rc, const char* where) {
  if (rc == LBX_OK) return;
  std::string msg = std::string(where) + ": " + lbx_last_error();
  if (rc == LBX_ERR_UNSUPPORTED) throw std::domain_error(msg);
  throw std::runtime_error(msg);
}

// ---- storage: the lattice's value type T (double, float) or a 16-bit deviation form ------------
struct Half {};      // f_i - w_i stored as IEEE binary16, collision in float
struct BFloat16 {};  // f_i - w_i stored as bfloat16, collision in float
template <typename S> struct storage_id;
template <> struct storage_id<double> { static constexpr int value = LBX_F64; };
template <> struct storage_id<float> { static constexpr int value = LBX_F32; };
template <> struct storage_id<Half> { static constexpr int value = LBX_F16DEV; };
template <> struct storage_id<BFloat16> { static constexpr int value = LBX_BF16DEV; };

// ---- descriptors ------------------------------------------------------------------------------
struct D2Q9 { static constexpr int q = 9, d = 2; };
struct D3Q19 { static constexpr int q = 19, d = 3; };
struct D3Q27 { static constexpr int q = 27, d = 3; };

// ---- bulk dynamics (dynamics/dynamics.h:89,223,529; smagorinskyBGKdynamics.h:39,67) ------------
struct BGKdynamics { static constexpr int id = LBX_BGK; };
struct TRTdynamics { static constexpr int id = LBX_TRT; };
struct SmagorinskyBGKdynamics { static constexpr int id = LBX_SMAGORINSKY_BGK; };
struct ForcedBGKdynamics { static constexpr int id = LBX_FORCED_BGK; };
struct SmagorinskyForcedBGKdynamics { static constexpr int id = LBX_SMAGORINSKY_FORCED_BGK; };
struct ConstRhoBGKdynamics { static constexpr int id = LBX_CONST_RHO_BGK; };
// cell kinds without a fluid dynamics (defineDynamics over a material)
struct NoDynamics { static constexpr int id = -LBX_CELL_NONE - 1; };
struct BounceBack { static constexpr int id = -LBX_CELL_BOUNCE_BACK - 1; };

// boundary::set<...> kinds over a material (lbx_set_interpolated_boundary)
enum class BoundaryKind : int32_t {
  InterpolatedVelocity = LBX_FD_VELOCITY,
  InterpolatedPressure = LBX_FD_PRESSURE,
  LocalVelocityBGK = LBX_FD_LOCAL_VELOCITY,
  LocalPressureBGK = LBX_FD_LOCAL_PRESSURE,
  LocalVelocity = LBX_FD_LOCAL_VELOCITY_RLB,
  LocalPressure = LBX_FD_LOCAL_PRESSURE_RLB,
};

// ---- parameters (descriptors::OMEGA, collision::TRT::MAGIC, collision::LES::SMAGORINSKY) ------
struct OMEGA {};
struct MAGIC {};
struct SMAGORINSKY {};
struct FORCE {};

// ---- per-cell dynamics ids (BlockDynamicsMap role) ----------------------------------------------
enum class CellDynamics : uint8_t {
  None = LBX_CELL_NONE,
  Bulk = LBX_CELL_BULK,
  BounceBack = LBX_CELL_BOUNCE_BACK,
};

struct LatticeStatistics {
  double averageRho = 0, averageEnergy = 0, maxU = 0;
  uint64_t cells = 0;
  double getAverageRho() const { return averageRho; }
  double getAverageEnergy() const { return averageEnergy; }
  double getMaxU() const { return maxU; }
};

struct FdBoundaryCell {
  int64_t cell;             // core cell index (x * ny + y) * nz + z
  int axis;                 // normal axis
  int orientation;          // +1 or -1: direction of the outward normal along the axis
  std::array<double, 3> u;  // velocity cells: the imposed velocity; pressure cells: tangential velocity
  double rho = 1.0;         // pressure cells: the imposed density
};

// One block lattice on one B200 (the ConcreteBlockLattice of the new platform).
template <typename DESCRIPTOR, typename S = float>
class BlockLattice {
 public:
  static constexpr int q = DESCRIPTOR::q;
  static constexpr int d = DESCRIPTOR::d;

  BlockLattice(std::array<int, 3> core, std::array<bool, 3> periodic = {false, false, false}, int device = 0)
      : core_(core) {
    if constexpr (d == 2) core_[2] = 1;
    const int32_t c[3] = {core_[0], core_[1], core_[2]};
    const int32_t p[3] = {periodic[0], periodic[1], d == 3 && periodic[2]};
    check(lbx_lattice_create(q, c, p, storage_id<S>::value, device, &h_), "lbx_lattice_create");
    params_ = lbx_params{1.0, 0.25, 0.12, {0.0, 0.0, 0.0}};
  }
  ~BlockLattice() {
    if (h_) lbx_lattice_destroy(h_);
  }
  BlockLattice(const BlockLattice&) = delete;
  BlockLattice& operator=(const BlockLattice&) = delete;
  BlockLattice(BlockLattice&& o) noexcept
      : h_(std::exchange(o.h_, nullptr)), core_(o.core_), dyn_(o.dyn_), params_(o.params_),
        fluidDefined_(o.fluidDefined_), cellMap_(std::move(o.cellMap_)) {
    for (int c = 0; c < 3; ++c) classDyn_[c] = o.classDyn_[c];
  }

  lbx_lattice handle() const { return h_; }
  int64_t coreCells() const { return int64_t(core_[0]) * core_[1] * core_[2]; }
  int64_t cellIndex(int x, int y, int z = 0) const { return (int64_t(x) * core_[1] + y) * core_[2] + z; }

  // defineDynamics<DYNAMICS>(...): the bulk dynamics of every LBX_CELL_BULK cell
  template <typename DYN>
  void defineDynamics() {
    dyn_ = DYN::id;
    check(lbx_set_dynamics(h_, dyn_, &params_), "lbx_set_dynamics");
  }
  // setParameter<OMEGA | MAGIC | SMAGORINSKY>(value), setParameter<FORCE>({fx, fy, fz})
  template <typename PARAM>
  void setParameter(double v) {
    if constexpr (std::is_same_v<PARAM, OMEGA>) params_.omega = v;
    else if constexpr (std::is_same_v<PARAM, MAGIC>) params_.magic = v;
    else if constexpr (std::is_same_v<PARAM, SMAGORINSKY>) params_.smagorinsky = v;
    else static_assert(sizeof(PARAM) == 0, "unknown scalar parameter");
    applyParameters();
  }
  template <typename PARAM>
  void setParameter(std::array<double, 3> v) {
    static_assert(std::is_same_v<PARAM, FORCE>, "only FORCE is a vector parameter");
    for (int a = 0; a < 3; ++a) params_.force[a] = v[a];
    applyParameters();
  }

  // defineDynamics<DYNAMICS>(material, m) (SuperLattice::defineDynamics over a material
  // indicator, core/superLattice.hh): the cells of material m get DYNAMICS.  The first fluid
  // dynamics becomes the lattice's; another kind becomes a parameter class of its own
  // (lbx_set_dynamics_class_kind, at most three); NoDynamics and BounceBack mark the cells.
  // Parameters are shared by every dynamics, as the reference's setParameter sets them.
  template <typename DYN>
  void defineDynamics(const std::vector<int32_t>& material, int32_t m) {
    if (int64_t(material.size()) != coreCells()) throw std::invalid_argument("material map must cover the core cells");
    if (cellMap_.empty()) cellMap_.assign(size_t(coreCells()), uint8_t(LBX_CELL_NONE));
    uint8_t id;
    if constexpr (DYN::id < 0) {
      id = uint8_t(-DYN::id - 1);
    } else {
      if (!fluidDefined_) {
        dyn_ = DYN::id;
        fluidDefined_ = true;
        check(lbx_set_dynamics(h_, dyn_, &params_), "lbx_set_dynamics");
      }
      id = LBX_CELL_BULK;
      if (DYN::id != dyn_) {
        int cls = 0;
        for (int c = 0; c < 3; ++c)
          if (classDyn_[c] == DYN::id || (cls == 0 && classDyn_[c] == 0)) {
            cls = c + 1;
            if (classDyn_[c] == DYN::id) break;
          }
        if (cls == 0) throw std::domain_error("more than four fluid dynamics in one block");
        classDyn_[cls - 1] = DYN::id;
        check(lbx_set_dynamics_class_kind(h_, cls, DYN::id, &params_), "lbx_set_dynamics_class_kind");
        id = uint8_t(LBX_CELL_BULK_CLASS_1 + cls - 1);
      }
    }
    for (size_t c = 0; c < material.size(); ++c)
      if (material[c] == m) cellMap_[c] = id;
    check(lbx_set_cell_dynamics(h_, cellMap_.data()), "lbx_set_cell_dynamics");
  }

  // boundary::set<KIND>(lattice, geometry, m) with the default fluid (1) and outside (0)
  // materials (boundary/setBoundary.h:112-121), then the values an application gives with
  // setVelocity / defineRho: values[4 c ...] = velocity, or {rho, tangential velocity}, of core
  // cell c (only the boundary cells' entries are read).
  void setBoundary(BoundaryKind kind, const std::vector<int32_t>& material, int32_t m,
                   const std::vector<double>& values) {
    if (int64_t(material.size()) != coreCells() || int64_t(values.size()) != 4 * coreCells())
      throw std::invalid_argument("material [cells] and values [4 * cells]");
    check(lbx_set_interpolated_boundary(h_, int32_t(kind), material.data(), m, 0, nullptr, 0, nullptr, values.data()),
          "lbx_set_interpolated_boundary");
  }

  void setCellDynamics(const std::vector<CellDynamics>& ids) {
    if (int64_t(ids.size()) != coreCells()) throw std::invalid_argument("cell dynamics map must cover the core cells");
    check(lbx_set_cell_dynamics(h_, reinterpret_cast<const uint8_t*>(ids.data())), "lbx_set_cell_dynamics");
  }

  // setBouzidiBoundary + setBouzidiVelocity with q = 1/2 (boundary/setBouzidiBoundary.h:193-420):
  // material per core cell; links from `fluid` cells into cells of the `solid` materials; the
  // wall velocity of each solid material (resting walls when empty).
  void setBouzidiBoundary(const std::vector<int32_t>& material, int32_t fluid, const std::vector<int32_t>& solid,
                          const std::vector<std::array<double, 3>>& wallVelocity = {}) {
    if (int64_t(material.size()) != coreCells()) throw std::invalid_argument("material map must cover the core cells");
    std::vector<double> wv;
    for (const auto& v : wallVelocity) wv.insert(wv.end(), v.begin(), v.end());
    if (!wallVelocity.empty() && wallVelocity.size() != solid.size())
      throw std::invalid_argument("one wall velocity per solid material");
    check(lbx_set_bouzidi_from_materials(h_, material.data(), fluid, int32_t(solid.size()), solid.data(),
                                         wv.empty() ? nullptr : wv.data()),
          "lbx_set_bouzidi_from_materials");
  }

  // boundary::set<InterpolatedVelocity> / <InterpolatedPressure> on flat faces
  void setInterpolatedBoundaries(const std::vector<FdBoundaryCell>& velocity, const std::vector<FdBoundaryCell>& pressure) {
    std::vector<int64_t> cells;
    std::vector<int32_t> kinds, dirs, orients;
    std::vector<double> values;
    auto add = [&](const FdBoundaryCell& b, int kind) {
      cells.push_back(b.cell);
      kinds.push_back(kind);
      dirs.push_back(b.axis);
      orients.push_back(b.orientation);
      if (kind == LBX_FD_VELOCITY) values.insert(values.end(), {b.u[0], b.u[1], b.u[2], 0.0});
      else values.insert(values.end(), {b.rho, b.u[0], b.u[1], b.u[2]});
    };
    for (const auto& b : velocity) add(b, LBX_FD_VELOCITY);
    for (const auto& b : pressure) add(b, LBX_FD_PRESSURE);
    check(lbx_set_fd_boundaries(h_, int64_t(cells.size()), cells.data(), kinds.data(), dirs.data(), orients.data(),
                                values.data()),
          "lbx_set_fd_boundaries");
  }

  // Cell::iniEquilibrium over the core: rho [cells], u [d][cells]
  void iniEquilibrium(const std::vector<double>& rho, const std::vector<double>& u, void* stream = nullptr) {
    if (int64_t(rho.size()) != coreCells() || int64_t(u.size()) != d * coreCells())
      throw std::invalid_argument("rho [cells], u [d][cells]");
    check(lbx_ini_equilibrium(h_, rho.data(), u.data(), stream), "lbx_ini_equilibrium");
  }
  // SuperLattice::initialize(): the post-processors applied once
  void initialize(void* stream = nullptr) { check(lbx_post_process(h_, stream), "lbx_post_process"); }

  // SuperLattice::collideAndStream(), `steps` times, statistics of the last step kept
  void collideAndStream(int64_t steps = 1, bool statistics = true, void* stream = nullptr) {
    check(lbx_collide_and_stream(h_, steps, statistics ? LBX_STEP_STATISTICS : 0u, stream), "lbx_collide_and_stream");
  }
  LatticeStatistics getStatistics(void* stream = nullptr) const {
    double out[4];
    check(lbx_get_statistics(h_, out, stream), "lbx_get_statistics");
    return LatticeStatistics{out[0], out[1], out[2], uint64_t(out[3])};
  }

  // populations [q][cells] (setProcessingContext(Simulation / Evaluation))
  void setPopulations(const std::vector<double>& f, void* stream = nullptr) {
    if (int64_t(f.size()) != q * coreCells()) throw std::invalid_argument("populations [q][cells]");
    check(lbx_upload_populations(h_, f.data(), 0, stream), "lbx_upload_populations");
  }
  std::vector<double> getPopulations(void* stream = nullptr) const {
    std::vector<double> f(static_cast<size_t>(q * coreCells()));
    check(lbx_download_populations(h_, f.data(), 0, stream), "lbx_download_populations");
    return f;
  }
  // SuperLattice::save / load, into and from a byte buffer (Serializer::save(buffer) / load)
  std::vector<uint8_t> save(void* stream = nullptr) const {
    int64_t n = 0;
    check(lbx_checkpoint_bytes(h_, &n), "lbx_checkpoint_bytes");
    std::vector<uint8_t> buf(static_cast<size_t>(n));
    check(lbx_save_checkpoint(h_, buf.data(), n, stream), "lbx_save_checkpoint");
    return buf;
  }
  void load(const std::vector<uint8_t>& buf, void* stream = nullptr) {
    check(lbx_load_checkpoint(h_, buf.data(), int64_t(buf.size()), stream), "lbx_load_checkpoint");
  }
  // SuperLatticeDensity / SuperLatticeVelocity: rho [cells], u [d][cells]
  std::pair<std::vector<double>, std::vector<double>> computeRhoU(void* stream = nullptr) const {
    std::vector<double> rho(static_cast<size_t>(coreCells())), u(static_cast<size_t>(d * coreCells()));
    check(lbx_compute_moments(h_, rho.data(), u.data(), stream), "lbx_compute_moments");
    return {std::move(rho), std::move(u)};
  }
  // FP64 {sum rho, sum j} over the bulk cells
  std::array<double, 4> massMomentum(void* stream = nullptr) const {
    double out[8];
    check(lbx_reduce(h_, LBX_REDUCE_MASS_MOMENTUM, out, stream), "lbx_reduce");
    return {out[0], out[1], out[2], out[3]};
  }
  // momentum-exchange force on the bounce-back links
  std::array<double, 3> drag(void* stream = nullptr) const {
    double out[8];
    check(lbx_reduce(h_, LBX_REDUCE_DRAG, out, stream), "lbx_reduce");
    return {out[0], out[1], out[2]};
  }
  // fastest step launch shape for this lattice (populations left as they were)
  void autotune(int32_t steps = 10, void* stream = nullptr) {
    int32_t n = 0;
    check(lbx_autotune(h_, steps, nullptr, 0, &n, stream), "lbx_autotune");
  }

 private:
  void applyParameters() {
    check(lbx_set_dynamics(h_, dyn_, &params_), "lbx_set_dynamics");
    for (int c = 0; c < 3; ++c)
      if (classDyn_[c] != 0)
        check(lbx_set_dynamics_class_kind(h_, c + 1, classDyn_[c], &params_), "lbx_set_dynamics_class_kind");
  }

  lbx_lattice h_ = nullptr;
  std::array<int, 3> core_;
  int dyn_ = LBX_BGK;
  lbx_params params_{};
  bool fluidDefined_ = false;
  int classDyn_[3] = {0, 0, 0};      // the dynamics of parameter classes 1..3 (0: unused)
  std::vector<uint8_t> cellMap_;   // per core cell: lbx_cell_dynamics (defineDynamics over materials)
};

}  // namespace lbx
