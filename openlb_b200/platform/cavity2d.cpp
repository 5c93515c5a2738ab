// Lid-driven cavity in 2D on the B200 path, set up the way OpenLB's examples/laminar/cavity2d
// sets it up (prepareGeometry / prepareLattice / setBoundaryValues / simulate), through the C++
// host layer lbx.hpp over liblbx.so: BGK on the fluid (material 1), InterpolatedVelocity on the
// resting walls (2) and on the lid (3, the top row with its corners), initialised at rest and
// then SuperLattice::initialize().
//
//   cavity2d [nx] [ny] [steps] [storage: f64|f32] [omega] [u_lid]
//
// Prints one JSON line with the lattice statistics of the last step.
#include <cstdio>
#include <cstdlib>
#include <exception>
#include <string>
#include <vector>

#include "lbx.hpp"

namespace {

template <typename S>
int simulate(int nx, int ny, long steps, double omega, double uLid) {
  lbx::BlockLattice<lbx::D2Q9, S> lattice({nx, ny, 1});

  // prepareGeometry: the outer layer 2, the top row 3 (corners included), the inside 1
  std::vector<int32_t> material(size_t(lattice.coreCells()), 2);
  for (int x = 0; x < nx; ++x)
    for (int y = 0; y < ny; ++y) {
      const int64_t c = lattice.cellIndex(x, y);
      if (y == ny - 1) material[size_t(c)] = 3;
      else if (x > 0 && x < nx - 1 && y > 0) material[size_t(c)] = 1;
    }

  // prepareLattice: BGK on the fluid, InterpolatedVelocity on walls and lid
  lattice.template setParameter<lbx::OMEGA>(omega);
  lattice.template defineDynamics<lbx::BGKdynamics>(material, 1);
  std::vector<double> values(size_t(4 * lattice.coreCells()), 0.0);
  for (size_t c = 0; c < material.size(); ++c)
    if (material[c] == 3) values[4 * c] = uLid;
  lattice.setBoundary(lbx::BoundaryKind::InterpolatedVelocity, material, 2, values);
  lattice.setBoundary(lbx::BoundaryKind::InterpolatedVelocity, material, 3, values);

  // at rest: rho = 1, u = 0 (iniEquilibrium), then SuperLattice::initialize(): the boundary
  // post-processors once, which give the lid cells their velocity
  std::vector<double> rho(size_t(lattice.coreCells()), 1.0), u(size_t(2 * lattice.coreCells()), 0.0);
  lattice.iniEquilibrium(rho, u);
  lattice.initialize();

  lattice.collideAndStream(steps, true);
  const lbx::LatticeStatistics st = lattice.getStatistics();
  std::printf("{\"nx\": %d, \"ny\": %d, \"steps\": %ld, \"average_rho\": %.17g, \"average_energy\": %.17g, "
              "\"max_u\": %.17g, \"cells\": %llu}\n",
              nx, ny, steps, st.getAverageRho(), st.getAverageEnergy(), st.getMaxU(),
              static_cast<unsigned long long>(st.cells));
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  const int nx = argc > 1 ? std::atoi(argv[1]) : 14;
  const int ny = argc > 2 ? std::atoi(argv[2]) : 12;
  const long steps = argc > 3 ? std::atol(argv[3]) : 150;
  const std::string storage = argc > 4 ? argv[4] : "f64";
  const double omega = argc > 5 ? std::atof(argv[5]) : 1.3;
  const double uLid = argc > 6 ? std::atof(argv[6]) : 0.1;
  try {
    if (storage == "f64") return simulate<double>(nx, ny, steps, omega, uLid);
    if (storage == "f32") return simulate<float>(nx, ny, steps, omega, uLid);
    std::fprintf(stderr, "storage must be f64 or f32\n");
    return 2;
  } catch (const std::exception& ex) {
    std::fprintf(stderr, "cavity2d: %s\n", ex.what());
    return 1;
  }
}
