// Lid-driven cavity in 3D on the B200 path, set up the way OpenLB's cavity examples are
// (examples/laminar/cavity3dBenchmark: prepareGeometry / prepareLattice / simulate), through
// the C++ host layer lbx.hpp over liblbx.so.
//
//   cavity3d [N] [steps] [storage: f64|f32|f16] [Re]
//
// An N^3 fluid box inside a one-cell solid shell.  The walls are halfway bounce-back.  The top
// layer moves in +x with u_lid = 0.05.  The lid takes the edges.  nu = u_lid N / Re.
// Prints one JSON line with the lattice statistics of the last step and the wall-clock MLUPS.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "lbx.hpp"

namespace {

template <typename S>
int simulate(int n, long steps, double re) {
  const double uLid = 0.05;
  const double nu = uLid * n / re;
  const double omega = 1.0 / (3.0 * nu + 0.5);
  const int e = n + 2;  // fluid plus the solid shell

  // prepareGeometry: material 1 fluid, 2 resting wall, 3 moving lid (the whole top layer)
  lbx::BlockLattice<lbx::D3Q19, S> lattice({e, e, e});
  std::vector<int32_t> material(size_t(lattice.coreCells()), 2);
  std::vector<lbx::CellDynamics> cellDyn(material.size(), lbx::CellDynamics::None);
  for (int x = 0; x < e; ++x)
    for (int y = 0; y < e; ++y)
      for (int z = 0; z < e; ++z) {
        const int64_t c = lattice.cellIndex(x, y, z);
        const bool inside = x > 0 && x < e - 1 && y > 0 && y < e - 1 && z > 0 && z < e - 1;
        if (y == e - 1) material[size_t(c)] = 3;
        else if (inside) {
          material[size_t(c)] = 1;
          cellDyn[size_t(c)] = lbx::CellDynamics::Bulk;
        }
      }

  // prepareLattice: BGK on the fluid, NoDynamics + halfway bounce-back on the walls
  lattice.template defineDynamics<lbx::BGKdynamics>();
  lattice.template setParameter<lbx::OMEGA>(omega);
  lattice.setCellDynamics(cellDyn);
  lattice.setBouzidiBoundary(material, 1, {2, 3}, {{0.0, 0.0, 0.0}, {uLid, 0.0, 0.0}});
  lattice.initialize();

  // simulate
  const auto t0 = std::chrono::steady_clock::now();
  lattice.collideAndStream(steps, true);
  const lbx::LatticeStatistics st = lattice.getStatistics();  // synchronises
  const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  const auto mm = lattice.massMomentum();
  std::printf("{\"n\": %d, \"steps\": %ld, \"omega\": %.17g, \"average_rho\": %.17g, \"average_energy\": %.17g, "
              "\"max_u\": %.17g, \"cells\": %llu, \"mass\": %.17g, \"mlups\": %.6g}\n",
              n, steps, omega, st.getAverageRho(), st.getAverageEnergy(), st.getMaxU(),
              static_cast<unsigned long long>(st.cells), mm[0], double(n) * n * n * steps / sec / 1e6);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  const int n = argc > 1 ? std::atoi(argv[1]) : 64;
  const long steps = argc > 2 ? std::atol(argv[2]) : 1000;
  const std::string storage = argc > 3 ? argv[3] : "f32";
  const double re = argc > 4 ? std::atof(argv[4]) : 100.0;
  try {
    if (storage == "f64") return simulate<double>(n, steps, re);
    if (storage == "f32") return simulate<float>(n, steps, re);
    if (storage == "f16") return simulate<lbx::Half>(n, steps, re);
    std::fprintf(stderr, "storage must be f64, f32 or f16\n");
    return 2;
  } catch (const std::exception& ex) {
    std::fprintf(stderr, "cavity3d: %s\n", ex.what());
    return 1;
  }
}
