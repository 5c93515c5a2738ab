/*  Reference-side driver (test infrastructure, never part of the shipped path).
 *
 *  Runs the reference implementation's OWN CPU code (SuperLattice / dynamics::Tuple /
 *  post-processors, compiled from the reference sources by oracle/Makefile) on a
 *  synthetic case and dumps the core-cell populations, so that the CUDA path and the
 *  C restatement in oracle/lbm_oracle.c can be checked against it.
 *
 *  API used (paths relative to the reference project):
 *    SuperLattice ctor / collideAndStream     src/core/superLattice.h:88, superLattice.hh:664-725
 *    defineDynamics<...>                      src/core/superLattice.h (BlockLattice::defineDynamics blockLattice.hh:274)
 *    BGKdynamics / TRTdynamics / ForcedBGK    src/dynamics/dynamics.h:89,223,529
 *    SmagorinskyBGK / SmagorinskyForcedBGK    src/dynamics/smagorinskyBGKdynamics.h:39,67
 *    ConstRhoBGKdynamics                      src/dynamics/dynamics.h:209-215
 *    BounceBack (Revert) / NoDynamics         src/dynamics/dynamics.h:51,557
 *    setBouzidiBoundary / setBouzidiVelocity  src/boundary/setBouzidiBoundary.h:193-420
 *    boundary::set<InterpolatedVelocity/Pressure>  src/boundary/setBoundary.h:80-160,
 *                                             interpolatedVelocity3D.h, interpolatedPressure3D.h
 *    Cell::iniEquilibrium                     src/core/cell.h:202
 *    LatticeStatistics                        src/core/latticeStatistics.h:91-93
 *
 *  Build-time selection: REF_T (double|float), REF_Q (9|19|27), REF_NO_FORCE (descriptor
 *  without the FORCE field; used by the timing build of plain BGK).
 *
 *  Usage:
 *    lbref <periodic|cavity|porous|channel> [--n NX NY [NZ]] [--dyn bgk|trt|smag|fbgk|fsmag|constrho]
 *          [--omega W] [--magic L] [--cs C] [--force FX FY [FZ]] [--steps S]
 *          [--init tgv|random|rest] [--u0 U] [--amp A] [--seed K] [--ulid U]
 *          [--walls bouzidi|bounceback] [--solid-frac P] [--out PREFIX]
 *          [--time W K] [--stats]
 *    lbref geo --mat FILE --n NX NY [NZ] [--periodic PX PY [PZ]] [--dyn ...] [--omega W] ...
 *          [--bouzidi M,...] [--lid M --ulid U] [--bounceback M,...] [--outside M,...]
 *          [--ivel M,... (--poiseuille UMAX | --uconst UX UY [UZ])] [--ivel-lid M] [--ipres M --rho R]
 *          [--bbvel M] [--local] [--local-rlb] [--bgk-mat M] [--trt-mat M]
 *          [--classify M] [--classify-only] [--force-mat M --force-every K] [--moments]
 *          [--no-pops] [--steps S] [--out PREFIX]
 *  The geo case reads the int32 materials of the core cells from FILE (x slowest, z fastest)
 *  and sets the lattice up through the reference's own setters: bulk dynamics on material 1,
 *  NoDynamics elsewhere; setBouzidiBoundary (q = 1/2) from fluid 1 towards the --bouzidi and
 *  --lid materials, setBouzidiVelocity (x velocity U) on the lid; BounceBack dynamics on the
 *  --bounceback materials, BounceBackVelocity with velocity (--ulid, 0, 0) on the --bbvel
 *  material; boundary::set<InterpolatedVelocity> / <InterpolatedPressure> on the
 *  --ivel / --ivel-lid / --ipres materials with fluid 1 and outside {0, --outside...}, which
 *  classifies every cell with computeBoundaryTypeAndNormal itself.  The imposed velocity of an
 *  --ivel material is RectanglePoiseuille3D over it (one --ivel material) with the zero-velocity
 *  planes half a cell outside it (peak UMAX along +x), or a constant; the --ivel-lid material
 *  moves with (--ulid, 0, 0).  Populations start at rest (all zero) or random (--init random).
 *  --local sets boundary::LocalVelocity / LocalPressure with BGK as the mixed-in dynamics on the
 *  --ivel / --ivel-lid / --ipres materials instead (src/boundary/localVelocity3D.h:47-115,
 *  localPressure3D.h, localVelocity2D.h: CombinedRLBdynamics on flat faces, the interpolated
 *  boundary's edges and corners); --local-rlb sets them with their default mixed-in dynamics,
 *  RLBdynamics (boundary/localVelocity.h:44-49, localPressure.h:31-36).
 *  --bgk-mat M puts BGKdynamics on material M beside the --dyn dynamics of material 1.
 *  --classify M writes PREFIX.normals.bin (int32 {core cell, type, n0, n1, n2} per cell of
 *  material M, fluid 1, outside {0, --outside...}); --classify-only stops there.
 *  --force-mat M writes PREFIX.force.txt: "step Fx Fy Fz" every K steps, the sum of
 *  SuperLatticePhysBoundaryForce3D over material M (lattice units).  --moments writes
 *  PREFIX.mom.bin (double rho, u [1 + d][ext...] from each cell's own computeRhoU) after the
 *  run; --no-pops skips the population and boundary-value dumps.  PREFIX.bclass.bin holds, for every cell the
 *  velocity / pressure setters equipped, int32 {core cell, kind (1 velocity, 2 pressure), normal
 *  type, n0, n1, n2} as computeBoundaryTypeAndNormal gave them.
 *  Output (with --out): PREFIX.f0.bin / PREFIX.fS.bin  raw T populations [Q][ext...] of the
 *  core cells after initialize() and after S steps; PREFIX.mat.bin int32 materials [ext...];
 *  PREFIX.stats.txt per-step "avgRho avgEnergy maxU"; PREFIX.json the case description.
 *  The channel case (x: a bounce-back layer, the velocity inlet, NX fluid layers ... the
 *  pressure outlet and a bounce-back layer, i.e. NX + 2 cells along x; periodic in the other
 *  axes, so every boundary cell is on a flat face) also writes PREFIX.bnd.bin: per
 *  boundary cell {core cell index, kind (1 velocity, 2 pressure), direction, orientation,
 *  value[4]} as doubles, value = the imposed velocity, or {rho, tangential velocity}.
 */

#include "olb.h"

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <fstream>
#ifdef PARALLEL_MODE_OMP
#include <omp.h>
#endif
#include <memory>
#include <string>
#include <vector>

using namespace olb;
using namespace olb::descriptors;

#ifndef REF_T
#define REF_T double
#endif
using T = REF_T;

#if REF_Q == 9
#  ifdef REF_NO_FORCE
using DESCRIPTOR = D2Q9<>;
#  else
using DESCRIPTOR = D2Q9<FORCE>;
#  endif
#elif REF_Q == 19
#  ifdef REF_NO_FORCE
using DESCRIPTOR = D3Q19<>;
#  else
using DESCRIPTOR = D3Q19<FORCE>;
#  endif
#elif REF_Q == 27
#  ifdef REF_NO_FORCE
using DESCRIPTOR = D3Q27<>;
#  else
using DESCRIPTOR = D3Q27<FORCE>;
#  endif
#else
#  error "REF_Q must be 9, 19 or 27"
#endif

constexpr int D = DESCRIPTOR::d;
constexpr int Q = DESCRIPTOR::q;

namespace {

struct Options {
  std::string kase = "periodic";
  int n[3] = {16, 16, 16};
  std::string dyn = "bgk";
  double omega = 1.0;
  double magic = 0.25;
  double cs = 0.12;
  double force[3] = {0, 0, 0};
  long steps = 10;
  std::string init = "random";
  double u0 = 0.05;
  double amp = 0.02;
  std::uint64_t seed = 1;
  double ulid = 0.1;
  std::string walls = "bouzidi";
  double solidFrac = 0.2;
  std::string out;
  long timeWarm = -1;
  long timeSteps = 0;
  bool stats = false;
  // geo case
  std::string matFile;
  int periodicFlags[3] = {0, 0, 0};
  std::vector<int> bouzidiMats, bouncebackMats, outsideMats;
  std::vector<int> ivelMats;
  int lidMat = -1, ivelLidMat = -1, ipresMat = -1, classifyMat = -1, forceMat = -1, bbvelMat = -1;
  long forceEvery = 0;
  double poiseuille = -1.0, uconst[3] = {0, 0, 0}, rhoOut = 1.0;
  bool classifyOnly = false, moments = false, noPops = false;
  bool local = false;  // --local: LocalVelocity / LocalPressure (BGK mixin) instead of the interpolated ones
  bool localRlb = false;  // --local-rlb: the same with their default RLB mixin
  int bgkMat = -1;     // --bgk-mat M: BGKdynamics on material M beside the --dyn dynamics on material 1
  int trtMat = -1;     // --trt-mat M: TRTdynamics on material M beside the --dyn dynamics on material 1
};

std::vector<int> parseList(const char* s) {
  std::vector<int> out;
  std::string t(s);
  std::size_t p = 0;
  while (p < t.size()) {
    std::size_t q = t.find(',', p);
    if (q == std::string::npos) q = t.size();
    out.push_back(std::atoi(t.substr(p, q - p).c_str()));
    p = q + 1;
  }
  return out;
}

/// splitmix64: deterministic per-(cell, population) values shared with the Python tests.
std::uint64_t mix(std::uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
double unit(std::uint64_t seed, std::uint64_t a, std::uint64_t b) {
  return double(mix(seed * 0x100000001B3ull ^ mix(a * 64 + b)) >> 11) * (1.0 / 9007199254740992.0);
}

/// Indicator whose distance queries always fail: setBouzidiBoundary then falls back to
/// q = 1/2 on every link (setBouzidiBoundary.h:262-278), i.e. halfway bounce-back.
template <int DIM> struct Nowhere;
template <> struct Nowhere<2> : public IndicatorF2D<T> {
  Nowhere() { this->_myMin = Vector<T,2>(-1e9); this->_myMax = Vector<T,2>(1e9); }
  bool operator()(bool output[], const T input[]) override { output[0] = false; return true; }
  bool distance(T& d, const Vector<T,2>&, const Vector<T,2>&, int) override { return false; }
};
template <> struct Nowhere<3> : public IndicatorF3D<T> {
  Nowhere() { this->_myMin = Vector<T,3>(-1e9); this->_myMax = Vector<T,3>(1e9); }
  bool operator()(bool output[], const T input[]) override { output[0] = false; return true; }
  bool distance(T& d, const Vector<T,3>&, const Vector<T,3>&, int) override { return false; }
};

template <typename F>
void forCore(const int ext[3], F f) {
  const int ez = (D == 3) ? ext[2] : 1;
  for (int x = 0; x < ext[0]; ++x)
    for (int y = 0; y < ext[1]; ++y)
      for (int z = 0; z < ez; ++z)
        f(x, y, z);
}

LatticeR<D> loc(int x, int y, int z) {
  if constexpr (D == 3) { return LatticeR<D>{x, y, z}; }
  else { return LatticeR<D>{x, y}; }
}

Options parse(int argc, char** argv) {
  Options o;
  if (argc > 1) o.kase = argv[1];
  for (int i = 2; i < argc; ++i) {
    std::string a = argv[i];
    auto next = [&]() -> const char* {
      if (i + 1 >= argc) { std::fprintf(stderr, "missing value for %s\n", a.c_str()); std::exit(2); }
      return argv[++i];
    };
    if (a == "--n") { for (int d = 0; d < D; ++d) o.n[d] = std::atoi(next()); }
    else if (a == "--dyn") o.dyn = next();
    else if (a == "--omega") o.omega = std::atof(next());
    else if (a == "--magic") o.magic = std::atof(next());
    else if (a == "--cs") o.cs = std::atof(next());
    else if (a == "--force") { for (int d = 0; d < D; ++d) o.force[d] = std::atof(next()); }
    else if (a == "--steps") o.steps = std::atol(next());
    else if (a == "--init") o.init = next();
    else if (a == "--u0") o.u0 = std::atof(next());
    else if (a == "--amp") o.amp = std::atof(next());
    else if (a == "--seed") o.seed = std::strtoull(next(), nullptr, 10);
    else if (a == "--ulid") o.ulid = std::atof(next());
    else if (a == "--walls") o.walls = next();
    else if (a == "--solid-frac") o.solidFrac = std::atof(next());
    else if (a == "--out") o.out = next();
    else if (a == "--time") { o.timeWarm = std::atol(next()); o.timeSteps = std::atol(next()); }
    else if (a == "--stats") o.stats = true;
    else if (a == "--mat") o.matFile = next();
    else if (a == "--periodic") { for (int d = 0; d < D; ++d) o.periodicFlags[d] = std::atoi(next()); }
    else if (a == "--bouzidi") o.bouzidiMats = parseList(next());
    else if (a == "--bounceback") o.bouncebackMats = parseList(next());
    else if (a == "--outside") o.outsideMats = parseList(next());
    else if (a == "--lid") o.lidMat = std::atoi(next());
    else if (a == "--ivel") o.ivelMats = parseList(next());
    else if (a == "--ivel-lid") o.ivelLidMat = std::atoi(next());
    else if (a == "--bbvel") o.bbvelMat = std::atoi(next());
    else if (a == "--local") o.local = true;
    else if (a == "--local-rlb") o.local = o.localRlb = true;
    else if (a == "--bgk-mat") o.bgkMat = std::atoi(next());
    else if (a == "--trt-mat") o.trtMat = std::atoi(next());
    else if (a == "--ipres") o.ipresMat = std::atoi(next());
    else if (a == "--poiseuille") o.poiseuille = std::atof(next());
    else if (a == "--uconst") { for (int d = 0; d < D; ++d) o.uconst[d] = std::atof(next()); }
    else if (a == "--rho") o.rhoOut = std::atof(next());
    else if (a == "--classify") o.classifyMat = std::atoi(next());
    else if (a == "--classify-only") o.classifyOnly = true;
    else if (a == "--force-mat") o.forceMat = std::atoi(next());
    else if (a == "--force-every") o.forceEvery = std::atol(next());
    else if (a == "--moments") o.moments = true;
    else if (a == "--no-pops") o.noPops = true;
    else { std::fprintf(stderr, "unknown option %s\n", a.c_str()); std::exit(2); }
  }
  return o;
}

template <typename DYN>
void defineFluid(SuperLattice<T,DESCRIPTOR>& lat, SuperGeometry<T,D>& geo) {
  lat.template defineDynamics<DYN>(geo, 1);
}

void dumpPopulations(SuperLattice<T,DESCRIPTOR>& lat, const int ext[3], const std::string& path) {
  auto& block = lat.getBlock(0);
  std::size_t nCells = std::size_t(ext[0]) * ext[1] * ((D == 3) ? ext[2] : 1);
  std::vector<T> buf(std::size_t(Q) * nCells);
  std::size_t c = 0;
  forCore(ext, [&](int x, int y, int z) {
    auto cell = block.get(loc(x, y, z));
    for (int i = 0; i < Q; ++i) buf[std::size_t(i) * nCells + c] = cell[i];
    ++c;
  });
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char*>(buf.data()), buf.size() * sizeof(T));
}


/// The geo case (see the usage note at the top of this file).
int runGeo(const Options& o) {
  int ext[3] = {1, 1, 1};
  for (int d = 0; d < D; ++d) ext[d] = o.n[d];
  const std::size_t nCore = std::size_t(ext[0]) * ext[1] * ext[2];
  std::vector<std::int32_t> mat(nCore);
  {
    std::ifstream f(o.matFile, std::ios::binary);
    f.read(reinterpret_cast<char*>(mat.data()), mat.size() * sizeof(std::int32_t));
    if (!f) { std::fprintf(stderr, "cannot read %zu materials from %s\n", nCore, o.matFile.c_str()); return 2; }
  }
  Vector<T,D> origin(T(0));
  Vector<int,D> extent;
  for (int d = 0; d < D; ++d) extent[d] = ext[d];
  CuboidDecomposition<T,D> cuboids(origin, T(1), extent, 1);
  {
    Vector<bool,D> per;
    for (int d = 0; d < D; ++d) per[d] = o.periodicFlags[d] != 0;
    cuboids.setPeriodicity(per);
  }
  HeuristicLoadBalancer<T> balancer(cuboids);
  SuperGeometry<T,D> geo(cuboids, balancer, 2);
  {
    auto& bg = geo.getBlockGeometry(0);
    std::size_t c = 0;
    forCore(ext, [&](int x, int y, int z) { bg.set(loc(x, y, z), mat[c++]); });
    geo.rename(1000, 1001);
    geo.communicate();
  }
  std::vector<int> outside{0};
  outside.insert(outside.end(), o.outsideMats.begin(), o.outsideMats.end());

  if (o.classifyMat >= 0) {
    auto fluidI = geo.getMaterialIndicator(1);
    auto outsideI = geo.getMaterialIndicator(std::vector<int>(outside));
    auto& fb = fluidI->getBlockIndicatorF(0);
    auto& ob = outsideI->getBlockIndicatorF(0);
    std::vector<std::int32_t> rows;
    std::size_t c = 0;
    forCore(ext, [&](int x, int y, int z) {
      if (mat[c] == o.classifyMat) {
        auto [type, n] = computeBoundaryTypeAndNormal(fb, ob, loc(x, y, z));
        rows.push_back(std::int32_t(c));
        rows.push_back(std::int32_t(static_cast<int>(type)));
        for (int d = 0; d < 3; ++d) rows.push_back(d < D ? std::int32_t(n[d]) : 0);
      }
      ++c;
    });
    std::ofstream f(o.out + ".normals.bin", std::ios::binary);
    f.write(reinterpret_cast<const char*>(rows.data()), rows.size() * sizeof(std::int32_t));
    if (o.classifyOnly) return 0;
  }

  // The set-up runs on one thread: with several, the OpenMP build's setBouzidiBoundary gives
  // results that vary from run to run (a race in the set-up, not in the steps).
#ifdef PARALLEL_MODE_OMP
  const int stepThreads = omp_get_max_threads();
  omp_set_num_threads(1);
#endif
  SuperLattice<T,DESCRIPTOR> lat(geo);
  const T nu = (T(1) / T(o.omega) - T(0.5)) / T(3);
  const UnitConverter<T,DESCRIPTOR> converter(T(1), T(1), T(1), T(1), nu, T(1));
  lat.setUnitConverter(converter);
  {
    std::vector<int> seen;
    for (std::int32_t m : mat)
      if (m != 1 && std::find(seen.begin(), seen.end(), m) == seen.end()) seen.push_back(m);
    lat.template defineDynamics<NoDynamics>(geo, 0);
    for (int m : seen) lat.template defineDynamics<NoDynamics>(geo, m);
  }
  if (o.dyn == "bgk") defineFluid<BGKdynamics<T,DESCRIPTOR>>(lat, geo);
  else if (o.dyn == "trt") defineFluid<TRTdynamics<T,DESCRIPTOR>>(lat, geo);
  else if (o.dyn == "smag") defineFluid<SmagorinskyBGKdynamics<T,DESCRIPTOR>>(lat, geo);
  else if (o.dyn == "constrho") defineFluid<ConstRhoBGKdynamics<T,DESCRIPTOR>>(lat, geo);
#ifndef REF_NO_FORCE
  else if (o.dyn == "fbgk") defineFluid<ForcedBGKdynamics<T,DESCRIPTOR>>(lat, geo);
  else if (o.dyn == "fsmag") defineFluid<SmagorinskyForcedBGKdynamics<T,DESCRIPTOR>>(lat, geo);
#endif
  else { std::fprintf(stderr, "unsupported --dyn %s\n", o.dyn.c_str()); return 2; }
  // a second fluid dynamics on one material (a block with two dynamics, as an application sets
  // them per material with dynamics::set)
  if (o.bgkMat >= 0) lat.template defineDynamics<BGKdynamics<T,DESCRIPTOR>>(geo, o.bgkMat);
  if (o.trtMat >= 0) lat.template defineDynamics<TRTdynamics<T,DESCRIPTOR>>(geo, o.trtMat);

  Nowhere<D> nowhere;
  if (o.lidMat >= 0) {
    std::vector<int> walls = o.bouzidiMats;
    walls.push_back(o.lidMat);
    setBouzidiBoundary<T,DESCRIPTOR,BouzidiVelocityPostProcessor>(
      lat, geo.getMaterialIndicator(std::vector<int>(walls)), geo.getMaterialIndicator({1}), nowhere);
    Vector<T,D> uw(T(0));
    uw[0] = T(o.ulid);
    AnalyticalConst<D,T,T> lidU(uw);
    setBouzidiVelocity<T,DESCRIPTOR>(lat, geo.getMaterialIndicator({o.lidMat}), geo.getMaterialIndicator({1}), lidU);
  } else if (!o.bouzidiMats.empty()) {
    setBouzidiBoundary<T,DESCRIPTOR,BouzidiPostProcessor>(
      lat, geo.getMaterialIndicator(std::vector<int>(o.bouzidiMats)), geo.getMaterialIndicator({1}), nowhere);
  }
  for (int m : o.bouncebackMats) lat.template defineDynamics<BounceBack>(geo, m);
  if (o.bbvelMat >= 0) lat.template defineDynamics<BounceBackVelocity>(geo, o.bbvelMat);
  std::vector<int> ivelAll = o.ivelMats;
  if (o.ivelLidMat >= 0) ivelAll.push_back(o.ivelLidMat);
  for (int m : ivelAll) {
    if (o.localRlb)
      boundary::set<T, DESCRIPTOR, boundary::LocalVelocity<T,DESCRIPTOR>>(
        lat, geo.getMaterialIndicator({m}), geo.getMaterialIndicator({1}), geo.getMaterialIndicator(std::vector<int>(outside)));
    else if (o.local)
      boundary::set<T, DESCRIPTOR, boundary::LocalVelocity<T,DESCRIPTOR,BGKdynamics<T,DESCRIPTOR>>>(
        lat, geo.getMaterialIndicator({m}), geo.getMaterialIndicator({1}), geo.getMaterialIndicator(std::vector<int>(outside)));
    else
      boundary::set<T, DESCRIPTOR, boundary::InterpolatedVelocity<T,DESCRIPTOR>>(
        lat, geo.getMaterialIndicator({m}), geo.getMaterialIndicator({1}), geo.getMaterialIndicator(std::vector<int>(outside)));
  }
  auto isIvel = [&](int m) { return std::find(ivelAll.begin(), ivelAll.end(), m) != ivelAll.end(); };
  if (o.ipresMat >= 0) {
    if (o.localRlb)
      boundary::set<T, DESCRIPTOR, boundary::LocalPressure<T,DESCRIPTOR>>(
        lat, geo.getMaterialIndicator({o.ipresMat}), geo.getMaterialIndicator({1}), geo.getMaterialIndicator(std::vector<int>(outside)));
    else if (o.local)
      boundary::set<T, DESCRIPTOR, boundary::LocalPressure<T,DESCRIPTOR,BGKdynamics<T,DESCRIPTOR>>>(
        lat, geo.getMaterialIndicator({o.ipresMat}), geo.getMaterialIndicator({1}), geo.getMaterialIndicator(std::vector<int>(outside)));
    else
      boundary::set<T, DESCRIPTOR, boundary::InterpolatedPressure<T,DESCRIPTOR>>(
        lat, geo.getMaterialIndicator({o.ipresMat}), geo.getMaterialIndicator({1}), geo.getMaterialIndicator(std::vector<int>(outside)));
  }

  // the classification boundary::set gave every cell it set up: rows {cell, kind (1 velocity,
  // 2 pressure), type, n0, n1, n2}; pressure cells only where the reference installs a condition
  // (flat faces)
  std::vector<std::int32_t> bclass;
  {
    auto fluidI = geo.getMaterialIndicator(1);
    auto outsideI = geo.getMaterialIndicator(std::vector<int>(outside));
    auto& fb = fluidI->getBlockIndicatorF(0);
    auto& ob = outsideI->getBlockIndicatorF(0);
    std::size_t c = 0;
    forCore(ext, [&](int x, int y, int z) {
      const bool vel = isIvel(mat[c]), pres = mat[c] == o.ipresMat;
      if (vel || pres) {
        auto [type, n] = computeBoundaryTypeAndNormal(fb, ob, loc(x, y, z));
        if (vel || static_cast<int>(type) == 0) {
          bclass.push_back(std::int32_t(c));
          bclass.push_back(vel ? 1 : 2);
          bclass.push_back(std::int32_t(static_cast<int>(type)));
          for (int d = 0; d < 3; ++d) bclass.push_back(d < D ? std::int32_t(n[d]) : 0);
        }
      }
      ++c;
    });
  }

  lat.template setParameter<descriptors::OMEGA>(T(o.omega));
  if (o.dyn == "trt" || o.trtMat >= 0) lat.template setParameter<collision::TRT::MAGIC>(T(o.magic));
  if (o.dyn == "smag" || o.dyn == "fsmag") lat.template setParameter<collision::LES::SMAGORINSKY>(T(o.cs));

  // imposed values: values[4 * c ...] = velocity (inlet) or {rho, 0, 0, 0} (outlet)
  std::vector<double> vals(4 * nCore, 0.0);
#if REF_Q != 9
  std::unique_ptr<RectanglePoiseuille3D<T>> profile;
  std::vector<T> umax{T(o.poiseuille), T(0), T(0)};
  if (o.ivelMats.size() == 1 && o.poiseuille >= 0)
    profile.reset(new RectanglePoiseuille3D<T>(geo, o.ivelMats[0], umax, T(0.5), T(0.5), T(0.5)));
#endif
  {
    auto& block = lat.getBlock(0);
    std::size_t c = 0;
    forCore(ext, [&](int x, int y, int z) {
      auto cell = block.get(loc(x, y, z));
      for (int i = 0; i < Q; ++i) cell[i] = T(0);
#ifndef REF_NO_FORCE
      if (mat[c] == 1) {
        Vector<T,D> fv;
        for (int d = 0; d < D; ++d) fv[d] = T(o.force[d]);
        cell.template setField<FORCE>(fv);
      }
#endif
      if (o.init == "random" && (mat[c] == 1 || isIvel(mat[c]) || mat[c] == o.ipresMat || mat[c] == o.bgkMat ||
                                 mat[c] == o.trtMat)) {
        T rho = T(1.0 + o.amp * (unit(o.seed, c, 60) - 0.5));
        T u[D] = {};
        for (int d = 0; d < D; ++d) u[d] = T(o.u0 * (unit(o.seed, c, 61 + d) - 0.5));
        cell.iniEquilibrium(rho, u);
        for (int i = 0; i < Q; ++i) cell[i] += T(o.amp * descriptors::t<double,DESCRIPTOR>(i) * (unit(o.seed, c, i) - 0.5));
      }
      if (isIvel(mat[c])) {
        T u[3] = {T(o.uconst[0]), T(o.uconst[1]), T(o.uconst[2])};
        if (mat[c] == o.ivelLidMat) {
          u[0] = T(o.ulid);
          u[1] = u[2] = T(0);
        }
#if REF_Q != 9
        if (profile && mat[c] != o.ivelLidMat) {
          const T at[3] = {T(x), T(y), T(z)};
          (*profile)(u, at);
        }
#endif
        Vector<T,D> uv;
        for (int d = 0; d < D; ++d) {
          uv[d] = u[d];
          vals[4 * c + d] = double(u[d]);
        }
        cell.defineU(uv.data());
      } else if (mat[c] == o.ipresMat) {
        cell.defineRho(T(o.rhoOut));
        vals[4 * c] = double(T(o.rhoOut));
      } else if (mat[c] == o.bbvelMat) {  // moving bounce-back wall: (--ulid, 0, 0), rho 1
        Vector<T,D> uv(T(0));
        uv[0] = T(o.ulid);
        cell.defineU(uv.data());
        vals[4 * c] = 1.0;
        vals[4 * c + 1] = double(uv[0]);
      }
      ++c;
    });
  }
  lat.initialize();
#ifdef PARALLEL_MODE_OMP
  omp_set_num_threads(stepThreads);
#endif

  std::FILE* statsFile = nullptr;
  std::FILE* forceFile = nullptr;
#if REF_Q != 9
  std::unique_ptr<SuperLatticePhysBoundaryForce3D<T,DESCRIPTOR>> forceF;
  std::unique_ptr<SuperSum3D<T,T>> sumF;
  if (o.forceMat >= 0) {
    forceF.reset(new SuperLatticePhysBoundaryForce3D<T,DESCRIPTOR>(lat, geo.getMaterialIndicator(o.forceMat), converter));
    sumF.reset(new SuperSum3D<T,T>(*forceF, geo.getMaterialIndicator(o.forceMat)));
  }
#endif
  if (!o.out.empty()) {
    if (!o.noPops) dumpPopulations(lat, ext, o.out + ".f0.bin");
    std::ofstream m(o.out + ".mat.bin", std::ios::binary);
    m.write(reinterpret_cast<const char*>(mat.data()), mat.size() * sizeof(std::int32_t));
    if (!o.noPops) {  // the large runs need neither the values nor the populations
      std::ofstream v(o.out + ".vals.bin", std::ios::binary);
      v.write(reinterpret_cast<const char*>(vals.data()), vals.size() * sizeof(double));
    }
    std::ofstream bc(o.out + ".bclass.bin", std::ios::binary);
    bc.write(reinterpret_cast<const char*>(bclass.data()), bclass.size() * sizeof(std::int32_t));
    statsFile = std::fopen((o.out + ".stats.txt").c_str(), "w");
    if (o.forceMat >= 0) forceFile = std::fopen((o.out + ".force.txt").c_str(), "w");
  }
  auto writeForce = [&](long step) {
#if REF_Q != 9
    if (!forceFile || !sumF) return;
    T sum[4] = {};
    int in[1] = {0};
    (*sumF)(sum, in);
    std::fprintf(forceFile, "%ld %.17g %.17g %.17g\n", step, double(sum[0]), double(sum[1]), double(sum[2]));
    std::fflush(forceFile);
#else
    (void)step;
#endif
  };
  const auto t0 = std::chrono::steady_clock::now();
  for (long s = 0; s < o.steps; ++s) {
    lat.collideAndStream();
    if (statsFile) {
      auto& st = lat.getStatistics();
      std::fprintf(statsFile, "%.17g %.17g %.17g\n", double(st.getAverageRho()), double(st.getAverageEnergy()), double(st.getMaxU()));
    }
    if (o.forceEvery > 0 && (s + 1) % o.forceEvery == 0) writeForce(s + 1);
  }
  const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (o.forceEvery <= 0) writeForce(o.steps);
  if (!o.out.empty()) {
    std::fclose(statsFile);
    if (forceFile) std::fclose(forceFile);
    if (!o.noPops) dumpPopulations(lat, ext, o.out + ".fS.bin");
    if (o.moments) {
      auto& block = lat.getBlock(0);
      std::vector<double> mom(std::size_t(1 + D) * nCore);
      std::size_t c = 0;
      forCore(ext, [&](int x, int y, int z) {
        auto cell = block.get(loc(x, y, z));
        T rho, u[D];
        cell.computeRhoU(rho, u);
        mom[c] = double(rho);
        for (int d = 0; d < D; ++d) mom[(1 + d) * nCore + c] = double(u[d]);
        ++c;
      });
      std::ofstream f(o.out + ".mom.bin", std::ios::binary);
      f.write(reinterpret_cast<const char*>(mom.data()), mom.size() * sizeof(double));
    }
    std::ofstream j(o.out + ".json");
    j.precision(17);
    j << "{\"case\": \"geo\", \"q\": " << Q << ", \"d\": " << D << ", \"ext\": [" << ext[0] << ", " << ext[1] << ", "
      << ext[2] << "], \"periodic\": [" << o.periodicFlags[0] << ", " << o.periodicFlags[1] << ", "
      << o.periodicFlags[2] << "], \"dyn\": \"" << o.dyn << "\", \"omega\": " << o.omega << ", \"magic\": " << o.magic
      << ", \"cs\": " << o.cs << ", \"force\": [" << o.force[0] << ", " << o.force[1] << ", " << o.force[2] << "]"
      << ", \"steps\": " << o.steps << ", \"init\": \"" << o.init << "\", \"ulid\": " << o.ulid
      << ", \"poiseuille\": " << o.poiseuille << ", \"rho_out\": " << o.rhoOut << ", \"seconds\": " << sec
      << ", \"bytes\": " << sizeof(T) << "}\n";
  }
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  olb::initialize(&argc, &argv);
  Options o = parse(argc, argv);
  OstreamManager clout(std::cout, "lbref");
  if (o.kase == "geo") return runGeo(o);

  const bool periodic = (o.kase == "periodic" || o.kase == "porous");
  const bool channel = o.kase == "channel";
  int ext[3] = {1, 1, 1};
  for (int d = 0; d < D; ++d) ext[d] = o.n[d] + (o.kase == "cavity" || (o.kase == "channel" && d == 0) ? 2 : 0);

  Vector<T,D> origin(T(0));
  Vector<int,D> extent;
  for (int d = 0; d < D; ++d) extent[d] = ext[d];
  CuboidDecomposition<T,D> cuboids(origin, T(1), extent, 1);
  if (periodic || channel) {
    Vector<bool,D> per;
    for (int d = 0; d < D; ++d) per[d] = !(channel && d == 0);
    cuboids.setPeriodicity(per);
  }
  HeuristicLoadBalancer<T> balancer(cuboids);
  SuperGeometry<T,D> geo(cuboids, balancer, 2);

  // --- materials: 1 fluid, 2 solid wall, 3 moving lid --------------------------------
  std::vector<std::int32_t> mat(std::size_t(ext[0]) * ext[1] * ((D == 3) ? ext[2] : 1), 1);
  {
    std::size_t c = 0;
    forCore(ext, [&](int x, int y, int z) {
      int m = 1;
      if (o.kase == "cavity") {
        const bool wall = x == 0 || x == ext[0] - 1 || y == 0 || (D == 3 && (z == 0 || z == ext[2] - 1));
        if (y == ext[1] - 1) m = 3;  // lid: the whole top layer, edges included
        else if (wall) m = 2;
      } else if (o.kase == "porous") {
        if (unit(o.seed ^ 0xABCDEFull, c, 63) < o.solidFrac) m = 2;
      } else if (channel) {
        if (x == 0 || x == ext[0] - 1) m = 2;  // bounce-back layer behind the open faces
        else if (x == 1) m = 3;                // velocity inlet
        else if (x == ext[0] - 2) m = 4;       // pressure outlet
      }
      mat[c++] = m;
    });
    auto& bg = geo.getBlockGeometry(0);
    c = 0;
    forCore(ext, [&](int x, int y, int z) { bg.set(loc(x, y, z), mat[c++]); });
    // BlockGeometry::set does not flag the overlap as stale; a rename between two unused
    // material numbers does (superGeometry.hh:221), so communicate() fills the periodic overlap.
    geo.rename(1000, 1001);
    geo.communicate();
  }

  SuperLattice<T,DESCRIPTOR> lat(geo);
  {
    // Lattice units throughout: dx = dt = 1, nu = (1/omega - 1/2) / 3.
    const T nu = (T(1) / T(o.omega) - T(0.5)) / T(3);
    const UnitConverter<T,DESCRIPTOR> converter(T(1), T(1), T(1), T(1), nu, T(1));
    lat.setUnitConverter(converter);
  }
  if (!o.stats && o.timeWarm >= 0) lat.setStatisticsOff();
  lat.template defineDynamics<NoDynamics>(geo, 0);

  if (o.dyn == "bgk") defineFluid<BGKdynamics<T,DESCRIPTOR>>(lat, geo);
  else if (o.dyn == "trt") defineFluid<TRTdynamics<T,DESCRIPTOR>>(lat, geo);
  else if (o.dyn == "smag") defineFluid<SmagorinskyBGKdynamics<T,DESCRIPTOR>>(lat, geo);
  else if (o.dyn == "constrho") defineFluid<ConstRhoBGKdynamics<T,DESCRIPTOR>>(lat, geo);
#ifndef REF_NO_FORCE
  else if (o.dyn == "fbgk") defineFluid<ForcedBGKdynamics<T,DESCRIPTOR>>(lat, geo);
  else if (o.dyn == "fsmag") defineFluid<SmagorinskyForcedBGKdynamics<T,DESCRIPTOR>>(lat, geo);
#endif
  else { std::fprintf(stderr, "unsupported --dyn %s\n", o.dyn.c_str()); return 2; }

  Nowhere<D> nowhere;
  if (o.kase == "cavity") {
    if (o.walls == "bouzidi") {
      lat.template defineDynamics<NoDynamics>(geo, 2);
      lat.template defineDynamics<NoDynamics>(geo, 3);
      setBouzidiBoundary<T,DESCRIPTOR,BouzidiVelocityPostProcessor>(
        lat, geo.getMaterialIndicator({2, 3}), geo.getMaterialIndicator({1}), nowhere);
      Vector<T,D> uw(T(0));
      uw[0] = T(o.ulid);
      AnalyticalConst<D,T,T> lidU(uw);
      setBouzidiVelocity<T,DESCRIPTOR>(lat, geo.getMaterialIndicator({3}), geo.getMaterialIndicator({1}), lidU);
    } else if (o.walls == "bounceback") {
      lat.template defineDynamics<BounceBack>(geo, 2);
      lat.template defineDynamics<BounceBack>(geo, 3);
    } else { std::fprintf(stderr, "unsupported --walls\n"); return 2; }
  } else if (o.kase == "porous") {
    if (o.walls == "bouzidi") {
      lat.template defineDynamics<NoDynamics>(geo, 2);
      setBouzidiBoundary<T,DESCRIPTOR,BouzidiPostProcessor>(
        lat, geo.getMaterialIndicator({2}), geo.getMaterialIndicator({1}), nowhere);
    } else {
      lat.template defineDynamics<BounceBack>(geo, 2);
    }
  }

  // inlet profile and outlet density of the channel (lattice units)
  const double twoPiC = 2.0 * 3.14159265358979323846;
  auto inletU = [&](int y, int z, T u[3]) {
    const double Y = twoPiC * y / ext[1], Z = (D == 3) ? twoPiC * z / ext[2] : 0.0;
    u[0] = T(o.u0 * (1.0 + 0.5 * std::sin(Y)) * (1.0 + 0.3 * std::cos(Z)));
    u[1] = T(0.2 * o.u0 * std::cos(Y));
    u[2] = T(0.1 * o.u0 * std::sin(Z));
  };
  const T rhoOut = T(1.0 - 0.2 * o.u0);
  if (channel) {
    lat.template defineDynamics<BGKdynamics<T,DESCRIPTOR>>(geo, 3);
    lat.template defineDynamics<BGKdynamics<T,DESCRIPTOR>>(geo, 4);
    // The layer behind each open face is bounce-back (material 2), so that the populations
    // the faces receive from outside are defined; it is the "outside" of the discrete
    // normals.
    lat.template defineDynamics<BounceBack>(geo, 2);
    boundary::set<T, DESCRIPTOR, boundary::InterpolatedVelocity<T,DESCRIPTOR>>(lat, geo.getMaterialIndicator({3}),
                                                  geo.getMaterialIndicator({1}), geo.getMaterialIndicator({0, 2}));
    boundary::set<T, DESCRIPTOR, boundary::InterpolatedPressure<T,DESCRIPTOR>>(lat, geo.getMaterialIndicator({4}),
                                                  geo.getMaterialIndicator({1}), geo.getMaterialIndicator({0, 2}));
  }

  lat.template setParameter<descriptors::OMEGA>(T(o.omega));
  if (o.dyn == "trt") lat.template setParameter<collision::TRT::MAGIC>(T(o.magic));
  if (o.dyn == "smag" || o.dyn == "fsmag") lat.template setParameter<collision::LES::SMAGORINSKY>(T(o.cs));

  // --- initial populations --------------------------------------------------------------
  {
    auto& block = lat.getBlock(0);
    std::size_t c = 0;
    const double twoPi = 2.0 * 3.14159265358979323846;
    forCore(ext, [&](int x, int y, int z) {
      auto cell = block.get(loc(x, y, z));
#ifndef REF_NO_FORCE
      if (mat[c] == 1) {
        Vector<T,D> fv;
        for (int d = 0; d < D; ++d) fv[d] = T(o.force[d]);
        cell.template setField<FORCE>(fv);
      }
#endif
      T rho = 1;
      T u[D] = {};
      if (o.init == "tgv") {
        const double X = twoPi * x / ext[0], Y = twoPi * y / ext[1], Z = (D == 3) ? twoPi * z / ext[2] : 0.0;
        u[0] = T(o.u0 * std::sin(X) * std::cos(Y) * std::cos(Z));
        u[1] = T(-o.u0 * std::cos(X) * std::sin(Y) * std::cos(Z));
      } else if (o.init == "random") {
        rho = T(1.0 + o.amp * (unit(o.seed, c, 60) - 0.5));
        for (int d = 0; d < D; ++d) u[d] = T(o.u0 * (unit(o.seed, c, 61 + d) - 0.5));
      }
      if (mat[c] == 1 || mat[c] == 3 || mat[c] == 4) {
        cell.iniEquilibrium(rho, u);
        if (o.init == "random") {
          for (int i = 0; i < Q; ++i) {
            cell[i] += T(o.amp * descriptors::t<double,DESCRIPTOR>(i) * (unit(o.seed, c, i) - 0.5));
          }
        }
      } else {
        for (int i = 0; i < Q; ++i) cell[i] = T(0);
      }
      ++c;
    });
  }
  std::vector<double> bnd;
  if (channel) {
    auto& block = lat.getBlock(0);
    std::size_t c = 0;
    forCore(ext, [&](int x, int y, int z) {
      auto cell = block.get(loc(x, y, z));
      if (mat[c] == 3) {
        T u[3];
        inletU(y, z, u);
        Vector<T,D> uv;
        for (int d = 0; d < D; ++d) uv[d] = u[d];
        cell.defineU(uv.data());
        const double row[8] = {double(c), 1, 0, -1, double(u[0]), double(u[1]), D == 3 ? double(u[2]) : 0.0, 0};
        bnd.insert(bnd.end(), row, row + 8);
      } else if (mat[c] == 4) {
        cell.defineRho(rhoOut);
        const double row[8] = {double(c), 2, 0, 1, double(rhoOut), 0, 0, 0};
        bnd.insert(bnd.end(), row, row + 8);
      }
      ++c;
    });
  }
  lat.initialize();

  const std::size_t nCore = std::size_t(ext[0]) * ext[1] * ((D == 3) ? ext[2] : 1);

  if (o.timeWarm >= 0) {
    for (long s = 0; s < o.timeWarm; ++s) lat.collideAndStream();
    auto t0 = std::chrono::steady_clock::now();
    for (long s = 0; s < o.timeSteps; ++s) lat.collideAndStream();
    auto t1 = std::chrono::steady_clock::now();
    const double sec = std::chrono::duration<double>(t1 - t0).count();
    int threads = 1;
#ifdef PARALLEL_MODE_OMP
    threads = singleton::omp().getSize();
#endif
    std::printf("{\"cells\": %zu, \"steps\": %ld, \"seconds\": %.9g, \"mlups\": %.9g, \"threads\": %d, \"q\": %d, \"bytes\": %zu}\n",
                nCore, o.timeSteps, sec, double(nCore) * o.timeSteps / sec / 1e6, threads, Q, sizeof(T));
    return 0;
  }

  std::FILE* statsFile = nullptr;
  if (!o.out.empty()) {
    dumpPopulations(lat, ext, o.out + ".f0.bin");
    std::ofstream m(o.out + ".mat.bin", std::ios::binary);
    m.write(reinterpret_cast<const char*>(mat.data()), mat.size() * sizeof(std::int32_t));
    statsFile = std::fopen((o.out + ".stats.txt").c_str(), "w");
    if (channel) {
      std::ofstream b(o.out + ".bnd.bin", std::ios::binary);
      b.write(reinterpret_cast<const char*>(bnd.data()), bnd.size() * sizeof(double));
    }
  }
  for (long s = 0; s < o.steps; ++s) {
    lat.collideAndStream();
    if (statsFile) {
      auto& st = lat.getStatistics();
      std::fprintf(statsFile, "%.17g %.17g %.17g\n", double(st.getAverageRho()), double(st.getAverageEnergy()), double(st.getMaxU()));
    }
  }
  if (!o.out.empty()) {
    std::fclose(statsFile);
    dumpPopulations(lat, ext, o.out + ".fS.bin");
    std::ofstream j(o.out + ".json");
    j.precision(17);
    j << "{\"case\": \"" << o.kase << "\", \"q\": " << Q << ", \"d\": " << D
      << ", \"ext\": [" << ext[0] << ", " << ext[1] << ", " << ((D == 3) ? ext[2] : 1) << "]"
      << ", \"dyn\": \"" << o.dyn << "\", \"omega\": " << o.omega << ", \"magic\": " << o.magic
      << ", \"cs\": " << o.cs << ", \"force\": [" << o.force[0] << ", " << o.force[1] << ", " << o.force[2] << "]"
      << ", \"steps\": " << o.steps << ", \"init\": \"" << o.init << "\", \"walls\": \"" << o.walls
      << "\", \"ulid\": " << o.ulid << ", \"bytes\": " << sizeof(T) << "}\n";
  }
  return 0;
}
