/* lbx.h -- C ABI of the B200 lattice Boltzmann hot path (liblbx.so, sm_100a).
 *
 * This is the boundary a new single-GPU platform of the reference (OpenLB 1.8r1,
 * src/core/platform) binds.  Every entry point names the reference interface it replaces
 * (paths relative to the reference project).  Conventions:
 *   - every function returns LBX_OK (0) or a negative lbx_status; lbx_last_error() gives a
 *     thread-local message.  Nothing throws across the ABI.  The reference's CUDA platform
 *     turns a failed call into std::runtime_error (core/platform/gpu/cuda/device.hh:48-53); the C++ host
 *     layer above this ABI does the same.
 *   - device memory is owned by the lattice handle; host buffers are caller-owned and only
 *     used during the call.
 *   - `stream` is a cudaStream_t passed as void* (NULL = the legacy default stream); all
 *     device work of a call is ordered on it.  One host thread drives one handle at a time;
 *     calls on different handles are independent.
 *   - no CPU fallback: without a usable sm_100 device lbx_lattice_create fails with
 *     LBX_ERR_NO_DEVICE.
 *
 * Populations are exchanged in the reference convention: the stored value is f_i - w_i
 * (src/dynamics/lbm.h:57-63, 296), descriptor ordering of src/descriptor/definition/common.h,
 * host arrays laid out [q][core cells] with cell = (x * ny + y) * nz + z (z fastest, as
 * BlockStructure orders cells, src/core/blockStructure.h:71).
 */
#ifndef LBX_H
#define LBX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBX_ABI_VERSION 1

typedef enum {
  LBX_OK = 0,
  LBX_ERR_INVALID = -1,     /* bad argument */
  LBX_ERR_NO_DEVICE = -2,   /* no CUDA device of compute capability 10.x */
  LBX_ERR_CUDA = -3,        /* a CUDA runtime call failed */
  LBX_ERR_UNSUPPORTED = -4, /* combination not provided (reference: std::domain_error) */
  LBX_ERR_OUT_OF_MEMORY = -5,
  LBX_ERR_STATE = -6        /* call not valid in the handle's current state */
} lbx_status;

/* Velocity sets (src/descriptor/definition/common.h:76-109, 152-193, 345-400). */
typedef enum { LBX_D2Q9 = 9, LBX_D3Q19 = 19, LBX_D3Q27 = 27 } lbx_descriptor;

/* Population storage.  F16DEV / BF16DEV hold f_i - w_i in binary16 / bfloat16 with the
 * collision in float registers; reductions are FP64 in every form. */
typedef enum { LBX_F64 = 0, LBX_F32 = 1, LBX_F16DEV = 2, LBX_BF16DEV = 3 } lbx_storage;

/* Bulk dynamics of a lattice (the lattice's own; the per-cell map below selects it, plain
 * bounce-back, no dynamics or one of up to three parameter classes per cell, and a class may
 * carry another of these dynamics, lbx_set_dynamics_class_kind). */
typedef enum {
  LBX_BGK = 1,                   /* BGKdynamics            dynamics/dynamics.h:89-99 */
  LBX_TRT = 2,                   /* TRTdynamics            dynamics/dynamics.h:529-536 */
  LBX_SMAGORINSKY_BGK = 3,       /* SmagorinskyBGKdynamics smagorinskyBGKdynamics.h:39-44 */
  LBX_FORCED_BGK = 4,            /* ForcedBGKdynamics      dynamics/dynamics.h:223-230 */
  LBX_SMAGORINSKY_FORCED_BGK = 5, /* SmagorinskyForcedBGKdynamics smagorinskyBGKdynamics.h:67-73 */
  LBX_CONST_RHO_BGK = 6          /* ConstRhoBGKdynamics    dynamics/dynamics.h:209-215,
                                    collision.h:322-351; AVERAGE_RHO is the previous step's
                                    average density (superLattice.hh:675-677), 1 before the
                                    first step, and statistics are kept on every step */
} lbx_dynamics;

/* Per-cell dynamics ids (the role of BlockDynamicsMap, core/blockDynamicsMap.h:264-416). */
typedef enum {
  LBX_CELL_NONE = 0,        /* NoDynamics (dynamics.h:51-63) */
  LBX_CELL_BULK = 1,        /* the lattice's bulk dynamics */
  LBX_CELL_BOUNCE_BACK = 2, /* BounceBack = collision::Revert (collision.h:465-484) */
  LBX_CELL_FD_BOUNDARY = 3, /* a cell of the lbx_set_fd_boundaries list (set by that call) */
  LBX_CELL_BOUNCE_BACK_VELOCITY = 4, /* BounceBackVelocity (set by lbx_set_bounce_back_velocity) */
  LBX_CELL_BULK_CLASS_1 = 8,  /* the bulk dynamics with the parameters of class 1, 2, 3 */
  LBX_CELL_BULK_CLASS_2 = 9,  /* (lbx_set_dynamics_class) */
  LBX_CELL_BULK_CLASS_3 = 10
} lbx_cell_dynamics;

/* Kinds of velocity / pressure boundary cells (lbx_set_fd_boundaries, lbx_set_boundary_cells,
 * lbx_set_interpolated_boundary). */
typedef enum {
  LBX_FD_VELOCITY = 1,       /* boundary::InterpolatedVelocity, boundary/interpolatedVelocity3D.h:45-52 */
  LBX_FD_PRESSURE = 2,       /* boundary::InterpolatedPressure, boundary/interpolatedPressure3D.h:48-90 */
  /* boundary::LocalVelocity / LocalPressure with BGKdynamics as the mixed-in dynamics
   * (boundary/localVelocity3D.h:47-115, localVelocity2D.h, localPressure3D.h): a flat cell is
   * CombinedRLBdynamics (dynamics/dynamics.h:470-523) -- its populations are rebuilt in the
   * collision as f^eq(rho, u) + fromPiToFneq(Pi) with Pi from RegularizedBoundaryStress
   * (boundary/helper.h:31-81), then collided by BGK with the same boundary momenta -- and has no
   * post-processor; velocity edges and corners are those of InterpolatedVelocity; pressure cells
   * exist on flat faces only (the reference throws elsewhere). */
  LBX_FD_LOCAL_VELOCITY = 3,
  LBX_FD_LOCAL_PRESSURE = 4,
  /* the same with their default mixed-in dynamics, RLBdynamics (boundary/localVelocity.h:44-49,
   * localPressure.h:31-36; collision::RLB, dynamics/collision.h:82-112): every cell of the
   * boundary, external edges and corners included, is collided by RLB with its momenta */
  LBX_FD_LOCAL_VELOCITY_RLB = 5,
  LBX_FD_LOCAL_PRESSURE_RLB = 6
} lbx_fd_kind;

/* Parameters of the bulk dynamics (the ParametersD fields OMEGA, TRT::MAGIC,
 * LES::SMAGORINSKY and the FORCE field, here uniform over the lattice). */
typedef struct {
  double omega;        /* descriptors::OMEGA */
  double magic;        /* collision::TRT::MAGIC (collision.h:382) */
  double smagorinsky;  /* collision::LES::SMAGORINSKY (collisionLES.h:69) */
  double force[3];     /* descriptors::FORCE, acceleration in lattice units */
} lbx_params;

typedef struct {
  int32_t q, d;
  int32_t core[3];       /* nx, ny, nz (nz = 1 in 2D) */
  int32_t padded[3];     /* core + 2 * pad in each spatial direction (pad = 1; 2D: nz' = 1) */
  int32_t pad;
  int32_t periodic[3];
  int32_t storage;
  int64_t n_cells;       /* padded cell count */
  int64_t n_core;        /* core cell count */
  int64_t column_stride; /* elements between column starts */
  int64_t bytes;         /* device bytes held by the population columns */
  int64_t n_links;       /* halfway bounce-back links */
  int64_t column_period; /* cyclic period of a column (= column_stride, or half of it when
                            every column is mapped twice back to back) */
} lbx_info;

typedef struct lbx_lattice_s* lbx_lattice;

/* Thread-local message of the last failing call on this thread. */
const char* lbx_last_error(void);
int lbx_abi_version(void);
/* Number of usable devices (compute capability 10.x); 0 without a GPU. */
int lbx_device_count(void);

/* Create a block lattice of `core` cells (ConcreteBlockLattice ctor, core/blockLattice.h:462;
 * population storage ImplementationOf<AbstractCyclicColumn>, core/platform/gpu/cuda/column.h:100-171).
 * periodic[3] flags make the block periodic along that axis (CuboidDecomposition::
 * setPeriodicity, geometry/cuboidDecomposition.hh:182 plus the PostCollide overlap copy,
 * core/superLattice.hh:150-155).  Populations start at 0 (= rest equilibrium at rho = 1). */
int lbx_lattice_create(int32_t q, const int32_t core[3], const int32_t periodic[3],
                       int32_t storage, int32_t device, lbx_lattice* out);
int lbx_lattice_destroy(lbx_lattice lattice);
int lbx_get_info(lbx_lattice lattice, lbx_info* info);

/* Select the bulk dynamics and its parameters (BlockDynamicsMap::set + setParameter,
 * core/blockLattice.h:559-576; ConcreteParametersD H2D, core/platform/gpu/cuda/context.hh:412-467). */
int lbx_set_dynamics(lbx_lattice lattice, int32_t dynamics, const lbx_params* params);

/* A second (third, fourth) fluid dynamics in one lattice: parameter classes 1..3 of the bulk
 * dynamics.  A reference block may carry different dynamics per material (dynamics::set,
 * core/blockDynamicsMap.h:264-310 keeps one collision operator per dynamics type); here the
 * cells marked LBX_CELL_BULK_CLASS_c in the cell map collide with the lattice's dynamics but
 * with these parameters (omega, TRT magic, Smagorinsky constant, force).  That covers a block
 * whose dynamics differ in their parameters, e.g. BGKdynamics beside ForcedBGKdynamics (the
 * forced dynamics with force 0 in one class) or regions of different viscosity.  A lattice with
 * classes steps with launch variant 1 (one cell per thread; lbx_set_launch_config refuses the
 * others and the autotuner tries only its block shapes), and its halfway bounce-back links all
 * run in the link kernel.  The moments, the residual and the velocity of a class cell seen by a
 * neighbouring velocity / pressure boundary cell use the lattice's own force.  params = NULL
 * removes class `cls` (its cells then use the lattice's parameters).  ConstRhoBGK takes no
 * classes (LBX_ERR_UNSUPPORTED). */
int lbx_set_dynamics_class(lbx_lattice lattice, int32_t cls, const lbx_params* params);

/* lbx_set_dynamics_class with a dynamics of its own for class `cls` (LBX_BGK ..
 * LBX_SMAGORINSKY_FORCED_BGK; ConstRhoBGK returns LBX_ERR_UNSUPPORTED): a block whose
 * materials carry dynamics of different kinds, e.g. TRTdynamics on one material beside
 * BGKdynamics on another (dynamics::set per material, core/blockDynamicsMap.h:264-310).  The
 * class's cells collide with that dynamics and these parameters; params = NULL removes the
 * class. */
int lbx_set_dynamics_class_kind(lbx_lattice lattice, int32_t cls, int32_t dynamics, const lbx_params* params);

/* Per-cell dynamics ids for the core cells ([core cells], lbx_cell_dynamics); NULL resets
 * to "bulk everywhere" (defineDynamics over a material, core/blockLattice.hh:274-286). */
int lbx_set_cell_dynamics(lbx_lattice lattice, const uint8_t* ids);

/* Flat-face velocity and pressure boundaries: what boundary::set<InterpolatedVelocity> and
 * boundary::set<InterpolatedPressure> install on a flat face (boundary/setBoundary.h:80-100):
 * the cell collides with BGKdynamics whose momenta are the boundary's
 * (momenta::BasicDirichletVelocityBoundaryTuple / BasicDirichletPressureBoundaryTuple,
 * dynamics/momenta/aliases.h:173-198; velocity: u imposed, rho from velocityBMRho; pressure:
 * rho imposed, u_normal from the populations, the tangential velocity imposed), and after each
 * stream PlaneFdBoundaryProcessor3D / StraightFdBoundaryProcessor2D
 * (boundary/boundaryPostProcessors3D.hh:39-93, boundaryPostProcessors2D.hh:39-76) rebuilds all
 * its populations as f^eq(rho, u) + f^neq(Pi) with Pi from finite-difference velocity gradients.
 * cells: core cell indices; kinds: lbx_fd_kind; dirs: normal axis; orients: +1 or -1, the
 * direction of the outward normal along that axis; values[4 * i ...]: the imposed velocity
 * (velocity cells) or {rho, tangential velocity} (pressure cells).  Every cell needs two cells
 * inward along its normal inside the core.  Its neighbours along the face contribute the
 * velocity their own dynamics give (computeU): a boundary cell of the list its momenta, a bulk
 * cell j / rho, a cell without dynamics or with plain bounce-back (and a padding cell beyond a
 * non-periodic face) zero.  Edges and corners take lbx_set_boundary_cells.  The cells become
 * LBX_CELL_FD_BOUNDARY in the cell dynamics map and keep that id through later
 * lbx_set_cell_dynamics calls; n = 0 removes the list.  A neighbour reached across a periodic
 * face contributes its j / rho, as the reference's overlap copy of that cell does (it carries
 * bulk dynamics). */
int lbx_set_fd_boundaries(lbx_lattice lattice, int64_t n, const int64_t* cells, const int32_t* kinds,
                          const int32_t* dirs, const int32_t* orients, const double* values);

/* Discrete normal types of a boundary cell (DiscreteNormalType, geometry/discreteNormals.h:33-39). */
typedef enum {
  LBX_NORMAL_FLAT = 0,
  LBX_NORMAL_EXTERNAL_CORNER = 1,
  LBX_NORMAL_INTERNAL_CORNER = 2,
  LBX_NORMAL_EXTERNAL_EDGE = 3,   /* 3D only */
  LBX_NORMAL_INTERNAL_EDGE = 4    /* 3D only */
} lbx_normal_type;

/* Discrete normal of every core cell of material `boundary` (computeBoundaryTypeAndNormal,
 * geometry/discreteNormals.hh:31-172 in 2D and 176-1191 in 3D, as boundary::set calls it,
 * boundary/setBoundary.h:80-99): a cell that is neither fluid nor outside is classified from
 * the fluid / outside state of its neighbours; the outward normal points away from the fluid.
 * A fluid cell is one whose material is in fluid[0..n_fluid), an outside cell one whose
 * material is in outside[0..n_outside); cells beyond a non-periodic face of the block count as
 * material 0, across a periodic face the partner cell is read.  A cell that matches no pattern
 * comes back as LBX_NORMAL_FLAT with a zero normal.  Returns the number of boundary-material
 * cells through n_out and, up to `cap` of them in ascending core-cell order, their core index,
 * type and normal (normals[3 * k + a]; arrays may be NULL to count only).  Host only. */
int lbx_discrete_normals(int32_t q, const int32_t core[3], const int32_t periodic[3], const int32_t* material,
                         int32_t boundary, int32_t n_fluid, const int32_t* fluid, int32_t n_outside,
                         const int32_t* outside, int64_t cap, int64_t* cells, int32_t* types, int32_t* normals,
                         int64_t* n_out);

/* Velocity / pressure boundary cells with their discrete normals: flat faces, external and
 * internal edges and corners, what boundary::set<InterpolatedVelocity> / <InterpolatedPressure>
 * install for each normal type (boundary/interpolatedVelocity3D.h:45-90,
 * interpolatedVelocity2D.h:45-80, interpolatedPressure3D.h:48-90):
 *   flat, velocity or pressure: as lbx_set_fd_boundaries (PlaneFdBoundaryProcessor3D /
 *     StraightFdBoundaryProcessor2D);
 *   external edge (3D), velocity: BGKdynamics with momenta::FixedVelocityBoundaryTuple
 *     (rho = sum f + 1, u imposed; dynamics/momenta/aliases.h:215-220) and after each stream
 *     OuterVelocityEdgeProcessor3D (boundary/boundaryPostProcessors3D.hh:164-238);
 *   external corner, velocity: the same momenta and OuterVelocityCornerProcessor3D
 *     (boundaryPostProcessors3D.hh:240-294) / OuterVelocityCornerProcessor2D
 *     (boundaryPostProcessors2D.hh:278-323), run after the flat and edge processors as their
 *     priority 1 orders them;
 *   internal edge (3D) and internal corner, velocity (interpolated or local alike):
 *     CombinedRLBdynamics with momenta::InnerEdgeVelocityTuple3D / InnerCornerVelocityTuple2D /
 *     InnerCornerVelocityTuple3D (dynamics/momenta/aliases.h:224-243): u imposed, rho the mean of
 *     velocityBMRho along the normal axes, Pi from the cell with its unknown populations bounced
 *     back in non-equilibrium; regularised in the collision, no post-processor.
 * kinds: lbx_fd_kind; types: lbx_normal_type; normals[3 * i + a]: outward normal components in
 * {-1, 0, 1} (a flat cell has one non-zero component, an edge two, a corner d); values[4 * i]:
 * the imposed velocity, or {rho, tangential velocity} of a pressure cell.  Every cell needs the
 * two cells inward along each non-zero normal component inside the core, and no normal
 * component may lie along a periodic axis.  Pressure cells that are not flat return
 * LBX_ERR_UNSUPPORTED.  A neighbour that carries no dynamics or plain
 * bounce-back (and a padding cell beyond a non-periodic face, the reference's NoDynamics
 * overlap) reads as u = 0, rho = 1 in the finite differences, as their momenta
 * (momenta::ZeroMomentum, OneDensity / FixedDensity) give it.  Replaces the boundary list of
 * lbx_set_fd_boundaries; n = 0 removes it. */
int lbx_set_boundary_cells(lbx_lattice lattice, int64_t n, const int64_t* cells, const int32_t* kinds,
                           const int32_t* types, const int32_t* normals, const double* values);

/* boundary::set<InterpolatedVelocity> (kind LBX_FD_VELOCITY) or <InterpolatedPressure>
 * (LBX_FD_PRESSURE), or <LocalVelocity> / <LocalPressure> (LBX_FD_LOCAL_VELOCITY /
 * LBX_FD_LOCAL_PRESSURE; a local pressure cell that is not flat returns LBX_ERR_UNSUPPORTED, as
 * the reference's "No valid discrete normal found"), over the core cells of material `boundary`, with the given fluid and outside
 * material lists, or (n_fluid = 0, n_outside = 0) those of the reference's default overload
 * (boundary/setBoundary.h:112-121: fluid 1, outside 0), followed by the values the application
 * would give them with
 * momenta::setVelocity / defineU or defineRho: values[4 * c ...] for core cell c (only the
 * entries of the boundary cells are read).  Pressure cells that are not flat are left out, as
 * the reference installs neither dynamics nor post-processor there; a velocity cell with no
 * discrete normal fails as the reference's "Could not set Boundary." does
 * (boundary/setBoundary3D.h:204-226).  The cells are added to those already set (a cell set
 * twice takes the later call). */
int lbx_set_interpolated_boundary(lbx_lattice lattice, int32_t kind, const int32_t* material, int32_t boundary,
                                  int32_t n_fluid, const int32_t* fluid, int32_t n_outside, const int32_t* outside,
                                  const double* values);

/* Bounce-back cells with a wall velocity: BounceBackVelocity (dynamics/dynamics.h:629-637), the
 * populations swapped (collision::Revert, collision.h:465-484) and then corrected by Nguyen-Ladd,
 * f_i += 2 rho u . c_i t_i / c_s^2 (NguyenLaddCorrection, collision.h:495-521), with the cell's
 * fixed density rho[i] (NULL: 1, FixedDensity's initial value) and velocity u[3 * i ...]
 * (momenta::ExternalVelocityFixedDensityTuple, dynamics/momenta/aliases.h:86-91; defineU).  The
 * cells count in the statistics with {rho, |u|^2} and become LBX_CELL_BOUNCE_BACK_VELOCITY in the
 * cell map, keeping that id through later lbx_set_cell_dynamics calls; cells of an earlier list
 * that are not listed again become cells without dynamics.  n = 0 removes the list.  A velocity /
 * pressure boundary cell reads such a neighbour's fixed velocity and density. */
int lbx_set_bounce_back_velocity(lbx_lattice lattice, int64_t n, const int64_t* cells, const double* rho,
                                 const double* u);

/* Halfway bounce-back links: BouzidiVelocityPostProcessor with q = 1/2
 * (boundary/setBouzidiBoundary.h:129-162), applied after streaming.  Link l acts on core
 * cell cells[l] (x_b) and direction dirs[l] (x_b + c_k is the solid neighbour); wall[l] is
 * c_k . u_wall (BOUZIDI_VELOCITY, setBouzidiBoundary.h:386-410), NULL for resting walls.
 * Replaces any previous link set.  n = 0 removes them. */
int lbx_set_bouzidi_links(lbx_lattice lattice, int64_t n, const int64_t* cells,
                          const int32_t* dirs, const double* wall);

/* Host-side setter: derive the links from a material map exactly as setBouzidiBoundary
 * (q = 1/2 fallback, setBouzidiBoundary.h:236-330) and setBouzidiVelocity (:386-410) do:
 * for every cell whose material is in solid[0..n_solid) and every direction, a neighbour of
 * material `fluid` gets a link; wall_velocity[j*3 + a] is the wall velocity of solid[j]
 * (NULL: resting).  Runs on the host; needs no device work beyond the upload. */
int lbx_set_bouzidi_from_materials(lbx_lattice lattice, const int32_t* material,
                                   int32_t fluid, int32_t n_solid, const int32_t* solid,
                                   const double* wall_velocity);
/* The same derivation without a lattice (for host tools and tests); returns the link count
 * through n_out and fills the arrays when they are not NULL (capacity `cap`). */
int lbx_build_bouzidi_links(int32_t q, const int32_t core[3], const int32_t periodic[3],
                            const int32_t* material, int32_t fluid, int32_t n_solid,
                            const int32_t* solid, const double* wall_velocity,
                            int64_t cap, int64_t* cells, int32_t* dirs, double* wall,
                            int64_t* n_out);

/* Populations of the core cells, host layout [q][core cells] of doubles (host_type 0) or
 * floats (host_type 1), f_i - w_i.  The Simulation/Evaluation context switches of the
 * population columns (core/platform/gpu/cuda/column.hh:285-296), restricted to the core cells. */
int lbx_upload_populations(lbx_lattice lattice, const void* host, int32_t host_type, void* stream);
int lbx_download_populations(lbx_lattice lattice, void* host, int32_t host_type, void* stream);

/* Checkpoint and resume (SuperLattice::save / load into a buffer, core/serializer.h:77-79 and
 * 187-189; a CUDA column serialises its data with its periodic-shift offset,
 * core/platform/gpu/cuda/column.hh:305-321).  A checkpoint is a host buffer of lbx_checkpoint_bytes bytes: a
 * 128-byte header (format tag, descriptor, storage form, core extent, periodic axes, the
 * statistics of the last statistics step) followed by the core cells' populations in the
 * layout of lbx_download_populations, FP64 for the FP64 form and FP32 for the others, which is
 * exact for every form.  The shift is not stored: populations are written in logical order and
 * load into a lattice at any shift, and the steps after a load give the same bits as steps
 * that were never interrupted.  Dynamics, boundaries and launch shape are set-up rather than
 * state: the caller applies them to the lattice it loads into, as an application re-runs its
 * set-up before SuperLattice::load.  A load checks that descriptor, storage, extent and
 * periodicity match (LBX_ERR_INVALID otherwise).  Both calls synchronise the stream. */
int lbx_checkpoint_bytes(lbx_lattice lattice, int64_t* bytes);
int lbx_save_checkpoint(lbx_lattice lattice, void* host, int64_t bytes, void* stream);
int lbx_load_checkpoint(lbx_lattice lattice, const void* host, int64_t bytes, void* stream);

/* Equilibrium initialisation from moment fields (BlockLattice::iniEquilibrium,
 * core/blockLattice.hh:201-219): rho [core cells], u [d][core cells], doubles. */
int lbx_ini_equilibrium(lbx_lattice lattice, const double* rho, const double* u, void* stream);

/* One or more fused collide-and-stream steps (SuperLattice::collideAndStream,
 * core/superLattice.hh:664-725): collision of every core cell by its dynamics, the
 * periodic overlap copy, the periodic-shift rotation of every population column
 * (ConcreteBlockLattice::stream, core/blockLattice.hh:316-338) and the PostStream
 * bounce-back links.  With LBX_STEP_STATISTICS the last step also accumulates the lattice
 * statistics (StatisticsPostProcessor, core/platform/gpu/cuda/statistics.hh:80-117) in FP64. */
#define LBX_STEP_STATISTICS 1u
int lbx_collide_and_stream(lbx_lattice lattice, int64_t steps, uint32_t flags, void* stream);

/* Run the PostStream post-processors once (the bounce-back links) without a step: what
 * BlockLattice::postProcess does (core/blockLattice.hh:483-489) and what the reference's
 * SuperLattice::initialize() runs once before the first collideAndStream. */
int lbx_post_process(lbx_lattice lattice, void* stream);

/* Statistics of the last step run with LBX_STEP_STATISTICS: {average rho, average energy
 * (= mean |u|^2 / 2), max |u|, cell count} (LatticeStatistics, core/latticeStatistics.hh:
 * 60-90).  Synchronises the stream. */
int lbx_get_statistics(lbx_lattice lattice, double out[4], void* stream);

/* Moment fields of the core cells, FP64 (the functor path: BlockLatticeDensity/Velocity via
 * cell.computeRhoU, functors/lattice/latticeVelocity3D.hh:66).  rho [core], u [d][core];
 * either may be NULL.  Forced dynamics report u = j/rho + F/2 (momenta::ForcedMomentum). */
int lbx_compute_moments(lbx_lattice lattice, double* rho, double* u, void* stream);

/* FP64 device reductions over the cells with bulk dynamics (SuperLatticeFieldReductionO,
 * core/superLatticeFieldReductionO.h; host functors SuperLpNorm3D, SuperLatticePhysDrag3D):
 *   LBX_REDUCE_MASS_MOMENTUM  out = {sum rho, sum j_x, sum j_y, sum j_z}
 *   LBX_REDUCE_DRAG           out = {F_x, F_y, F_z} momentum exchange over all links, in the
 *                             convention of lbx_boundary_force
 *   LBX_REDUCE_RESIDUAL       out = {||u - u_prev||_2, ||u||_2, max |u - u_prev|} against
 *                             the velocity snapshot of the previous RESIDUAL call, then
 *                             refreshes the snapshot (ValueTracer-style convergence). */
#define LBX_REDUCE_MASS_MOMENTUM 1
#define LBX_REDUCE_DRAG 2
#define LBX_REDUCE_RESIDUAL 3
int lbx_reduce(lbx_lattice lattice, int32_t what, double* out, void* stream);

/* Force on the solid behind a group of halfway bounce-back links, lattice units, FP64: the sum of
 * the reference's boundary-force functor over that solid (SuperLatticePhysBoundaryForce3D summed
 * by SuperSum3D; BlockLatticePhysBoundaryForce3D::operator(), functors/lattice/
 * latticePhysBoundaryForce3D.hh:85-113): for every solid cell x_s and direction k towards a fluid
 * cell, F -= c_k (f_k(x_s + c_k) + f_opp(k)(x_s)) on the stored values f - w, read after the last
 * step's post-processing.  group: the index in `solid` of lbx_set_bouzidi_from_materials of the
 * material whose force is wanted (links set by lbx_set_bouzidi_links are group 0), -1 for every
 * link.  The drag coefficient of SuperLatticePhysDrag3D is 2 F / (rho U^2 A) of this force.
 * Synchronises the stream. */
int lbx_boundary_force(lbx_lattice lattice, int32_t group, double out[3], void* stream);

/* Periodic-shift bookkeeping for a platform that keeps the reference's split collide /
 * stream calls: the device base of population column i at the current shift
 * (CyclicColumn::operator[] / deviceData, core/platform/gpu/cuda/column.h:100-171) and a column rotation
 * by `offset` cells (CyclicColumn::rotate, core/platform/gpu/cuda/column.h:144-154). */
int lbx_population_shift(lbx_lattice lattice, int32_t pop, int64_t* shift);
/* Device address of population column `pop` for code outside this library that works on the
 * populations in place (ConcreteBlockLattice::getPopulationPointers, core/blockLattice.h:134,
 * 676-681; CyclicColumn::deviceData, core/platform/gpu/cuda/column.h:100-171).  Population i of padded cell n
 * (n = (x + 1) * padded[1] * padded[2] + (y + 1) * padded[2] + z + 1 in 3D, see lbx_info) is at
 * ((S*)*ptr)[(n + *shift) % column_period], S the storage type.  With the columns mapped twice
 * (the default layout) *shift is 0 and the index needs no wrap; a plain layout returns the
 * column start and its shift.  The address stays valid until the lattice is destroyed; the
 * shift changes with every step (lbx_collide_and_stream, lbx_rotate). */
int lbx_population_ptr(lbx_lattice lattice, int32_t pop, void** ptr, int64_t* shift);
int lbx_rotate(lbx_lattice lattice, int32_t pop, int64_t offset);

/* Launch configuration of the step kernel, the knob the autotuner turns (no reference
 * counterpart; the reference's CUDA platform launches fixed 32-thread blocks,
 * core/platform/gpu/cuda/operator.hh:425-441).  variant 0: pipelined shared-memory tiles of 256 cells;
 * variant 1: one cell per thread in (block_x, block_y) blocks; variant 2 (default):
 * cells_per_thread (1 or 2; 4 for 16-bit storage) cells a warp apart per thread in
 * (block_x, block_y) blocks, block_x along the fastest axis; variant 3: tiles moved by TMA bulk
 * copies, two stages per block; variant 4: tiles moved by TMA bulk copies through a ring of
 * four stages, one producer warp and sixteen consumer warps per block (block_x, block_y and
 * cells_per_thread are ignored by 0, 3 and 4); variant 5: variant 2 plus an L2 bulk prefetch,
 * at the start of each block, of the populations of the block one wave of resident blocks later
 * in launch order.  Variants 3, 4 and 5 need the doubled column layout (variant 5 without it
 * runs as variant 2).  Every variant computes identical populations. */
int lbx_set_launch_config(lbx_lattice lattice, int32_t variant, int32_t block_x, int32_t block_y,
                          int32_t cells_per_thread);

/* Per-kernel device timing of lbx_collide_and_stream, for profiling and the roofline (no
 * reference counterpart; the reference's util::Timer times whole steps on the host,
 * utilities/timer.hh:55-86).  enable != 0 records CUDA events around the kernels of every
 * following step and clears the totals; lbx_get_kernel_timing synchronises and returns the
 * summed device milliseconds of the collision, periodic-overlap and bounce-back-link kernels in
 * out[0..2] and their launch counts in out[3..5]. */
int lbx_set_kernel_timing(lbx_lattice lattice, int32_t enable);
int lbx_get_kernel_timing(lbx_lattice lattice, double out[6]);

/* ---- ensemble engine: many independent lattices stepped together ----------------------
 * No reference counterpart (the reference steps one SuperLattice at a time).  An ensemble owns
 * one slab of device memory; each admitted request is a box cavity of its own size: all core
 * cells fluid with the given bulk dynamics, halfway bounce-back walls on every face, the +y
 * face moving in +x with lid_velocity (setBouzidiBoundary + setBouzidiVelocity semantics with
 * q = 1/2, boundary/setBouzidiBoundary.h:129-162, the lid taking the edges).  A persistent kernel
 * steps every running lattice through a tile -> lattice map, checks the relative L2 velocity
 * residual ||u(t) - u(t - check)|| / ||u(t)|| every `check_interval` steps and stops a lattice
 * when it falls below `tolerance` or after `max_steps`. */
typedef struct lbx_ensemble_s* lbx_ensemble;

typedef struct {
  int32_t core[3];        /* nx, ny, nz */
  int32_t dynamics;       /* LBX_BGK or LBX_TRT */
  lbx_params params;      /* omega (and magic for TRT) */
  double lid_velocity;    /* x velocity of the +y wall */
  double tolerance;       /* stop at residual < tolerance */
  int64_t max_steps;      /* stop after this many steps */
} lbx_ensemble_request;

typedef enum {
  LBX_SLOT_FREE = 0,
  LBX_SLOT_RUNNING = 1,
  LBX_SLOT_CONVERGED = 2,
  LBX_SLOT_MAX_STEPS = 3,
  LBX_SLOT_DIVERGED = 4     /* residual or velocity not finite */
} lbx_slot_state;

typedef struct {
  int32_t state;          /* lbx_slot_state */
  int32_t pad;
  int64_t steps;          /* steps taken */
  double residual;        /* last checked residual */
} lbx_ensemble_status;

/* Slab bytes a request needs (populations + velocity snapshot). */
int lbx_ensemble_footprint(int32_t q, int32_t storage, const lbx_ensemble_request* req, int64_t* bytes);
int lbx_ensemble_create(int32_t q, int32_t storage, int64_t slab_bytes, int32_t max_lattices, int32_t device,
                        lbx_ensemble* out);
int lbx_ensemble_destroy(lbx_ensemble ens);
/* Admit a request (populations at rest, rho = 1).  LBX_ERR_OUT_OF_MEMORY when the slab has no
 * room or all slots are taken: the caller retries after retiring finished lattices. */
int lbx_ensemble_admit(lbx_ensemble ens, const lbx_ensemble_request* req, int32_t* slot);
/* Run `steps` steps of every running lattice in one persistent launch (replayed from a CUDA
 * graph after the first call with the same step count), ordered on `stream`. */
int lbx_ensemble_run(lbx_ensemble ens, int32_t steps, void* stream);
/* Status of every slot (synchronises the stream); n = number of entries in `out`. */
int lbx_ensemble_statuses(lbx_ensemble ens, lbx_ensemble_status* out, int32_t n, void* stream);
/* rho [cells] and u [3][cells] of a slot's core cells, FP64 (with the wall links applied). */
int lbx_ensemble_moments(lbx_ensemble ens, int32_t slot, double* rho, double* u, void* stream);
/* Free a slot and its slab space (no effect on the others). */
int lbx_ensemble_retire(lbx_ensemble ens, int32_t slot);
/* Pre-emption: a running (or finished) slot saved to a host buffer and restored later, in this
 * or another ensemble of the same descriptor and storage, as a newly admitted slot that
 * continues exactly where it stopped: populations at their shifts, velocity snapshot, step
 * count, residual and state (the ensemble form of SuperLattice::save / load,
 * core/serializer.h:77-79).  The buffer holds a header and the slot's slab region;
 * lbx_ensemble_checkpoint_bytes gives its size.  Saving synchronises the stream and leaves the
 * slot admitted: retire it to free its memory.  Restoring admits by footprint like
 * lbx_ensemble_admit (LBX_ERR_OUT_OF_MEMORY when it does not fit yet). */
int lbx_ensemble_checkpoint_bytes(lbx_ensemble ens, int32_t slot, int64_t* bytes);
int lbx_ensemble_save_slot(lbx_ensemble ens, int32_t slot, void* host, int64_t bytes, void* stream);
int lbx_ensemble_restore_slot(lbx_ensemble ens, const void* host, int64_t bytes, int32_t* slot, void* stream);
/* Launch shape of the persistent kernel (the autotuner's knob): threads per block (multiple of
 * 32, <= 256; a tile is 512 cells whatever the block size, so results and residuals do not
 * depend on it), resident blocks per SM (0: occupancy maximum), and the residual check interval
 * in steps. */
int lbx_ensemble_set_config(lbx_ensemble ens, int32_t threads, int32_t blocks_per_sm, int32_t check_interval);
/* How a run is launched: 0 (default) one persistent cooperative kernel per run, steps separated
 * by grid-wide barriers; 1 one launch per step plus a one-block bookkeeping launch, chained in a
 * CUDA graph (the launch boundaries order the steps, and populations may then be read through
 * L1).  Both give identical results. */
int lbx_ensemble_set_launch_mode(lbx_ensemble ens, int32_t mode);
/* Cells per thread of the tile loop, 1 (default) or 2: a warp steps 32 * cells consecutive
 * cells of a tile per round, keeping that many loads in flight per thread.  Both give identical
 * results. */
int lbx_ensemble_set_cells_per_thread(lbx_ensemble ens, int32_t cells);

/* ---- autotuner ----------------------------------------------------------------------------
 * No reference counterpart (the reference's CUDA platform launches fixed 32-thread blocks,
 * core/platform/gpu/cuda/operator.hh:425-441).  Both calls time every candidate launch shape on the caller's
 * own data with CUDA events on `stream`, each candidate starting from the same saved state, then
 * keep the fastest and put the state back as it was: populations, column shifts (and for an
 * ensemble every lattice's step count, residual and state) are unchanged on return, and since
 * every launch shape computes identical bits the tuned run continues exactly as an untuned one
 * would.  The saved state is a temporary device copy (populations of the lattice, or the used
 * part of the ensemble slab); LBX_ERR_OUT_OF_MEMORY if it does not fit, config unchanged.
 * out[0 .. min(capacity, candidates) - 1] lists what was tried, *n_out the number of candidates;
 * ms_per_step < 0 marks a shape the device or the lattice does not accept. */
typedef struct {
  int32_t variant, block_x, block_y, cells_per_thread;  /* lbx_autotune: lbx_set_launch_config;
                                                           lbx_ensemble_autotune: variant = launch
                                                           mode, cells_per_thread as set by
                                                           lbx_ensemble_set_cells_per_thread */
  int32_t threads, blocks_per_sm;                       /* lbx_ensemble_autotune: set_config */
  double ms_per_step;
} lbx_tune_entry;
/* Tunes the step kernel of one lattice over `steps` timed steps per candidate. */
int lbx_autotune(lbx_lattice lattice, int32_t steps, lbx_tune_entry* out, int32_t capacity, int32_t* n_out,
                 void* stream);
/* Tunes the persistent kernel over `steps` timed steps of the admitted lattices (at least one). */
int lbx_ensemble_autotune(lbx_ensemble ens, int32_t steps, lbx_tune_entry* out, int32_t capacity,
                          int32_t* n_out, void* stream);

/* ---- slab decomposition -------------------------------------------------------------------
 * One lattice cut along x into n_slabs slabs (as equal as the extent allows, each at least two
 * planes thick), each an lbx_lattice of its own on devices[k] (NULL: all on device 0), stepped in
 * lock-step with one face exchange per step between the collision and the post-stream links and
 * boundary cells: the single-process form of the reference's block decomposition and overlap
 * communication (core/superLattice.hh:150-155, core/platform/gpu/cuda/communicator.hh:355-510).  Every
 * population that leaves a slab across an x face is copied into the plane of the neighbour slab
 * it streams into (periodic x joins the last slab to the first); slabs on different devices send
 * their face buffers by cudaMemcpyPeerAsync.  A decomposed lattice computes the populations of
 * the undivided one bit for bit.
 * Set-up goes through each slab's handle (lbx_slabs_get: the handle, its first x and its
 * extent; cell k of a slab is global cell (x0 + x, y, z)): dynamics, cell maps, links and boundary
 * cells as for any lattice, with two rules: a link whose solid neighbour lies in the next slab is
 * given to the slab of its fluid cell (its neighbour then lies in that slab's ghost plane), and a
 * velocity / pressure boundary cell must have two planes of its own slab on each side that meets
 * another slab (its finite differences and neighbour momenta stay inside its slab).  ConstRhoBGK is refused (LBX_ERR_UNSUPPORTED).
 * lbx_slabs_collide_and_stream returns once the work is queued (one stream per slab, ordered
 * with the default stream); lbx_slabs_get_statistics waits and combines the slabs' statistics. */
typedef struct lbx_slabs_s* lbx_slabs;
int lbx_slabs_create(int32_t q, const int32_t core[3], const int32_t periodic[3], int32_t storage, int32_t n_slabs,
                     const int32_t* devices, lbx_slabs* out);
int lbx_slabs_destroy(lbx_slabs slabs);
int lbx_slabs_get(lbx_slabs slabs, int32_t k, lbx_lattice* lattice, int32_t* x0, int32_t* nx);
int lbx_slabs_collide_and_stream(lbx_slabs slabs, int64_t steps, uint32_t flags);
int lbx_slabs_synchronize(lbx_slabs slabs);
int lbx_slabs_get_statistics(lbx_slabs slabs, double out[4]);

/* ---- test hook -------------------------------------------------------------------------
 * No reference counterpart.  Off by default; for tests of the error paths: it makes a bounded
 * wait of the library's own kernels run out, or an allocation fail, without any GPU fault, so
 * that the status the caller reads can be checked.
 *   LBX_TEST_NONE              normal operation (param ignored)
 *   LBX_TEST_ENSEMBLE_BARRIER  the persistent ensemble kernel's block 0 leaves before the first
 *                              grid barrier; the other blocks give up after `param` polls (0: the
 *                              normal bound), set the error flag and return, and
 *                              lbx_ensemble_statuses reports LBX_ERR_CUDA.  Applies to the runs
 *                              an ensemble prepares after the call (a new step count).
 *   LBX_TEST_BULK_COPY         the bulk-copy step kernel (launch variant 3) of block 0 leaves one
 *                              copy of its first tile unrequested; its wait gives up after `param`
 *                              polls, and lbx_get_statistics reports LBX_ERR_CUDA.
 *   LBX_TEST_ALLOCATION        the next `param` population-column or ensemble-slab allocations
 *                              fail as cudaMalloc does when memory is short (LBX_ERR_OUT_OF_MEMORY).
 * Process-wide; not for concurrent use. */
typedef enum {
  LBX_TEST_NONE = 0,
  LBX_TEST_ENSEMBLE_BARRIER = 1,
  LBX_TEST_BULK_COPY = 2,
  LBX_TEST_ALLOCATION = 3
} lbx_test_fault_kind;
int lbx_test_fault(int32_t kind, int32_t param);

/* Mass/momentum sums for callers that cannot allocate device memory.  No counterpart in the
 * reference.  lbx_reduce(LBX_REDUCE_MASS_MOMENTUM) needs a lattice handle, whose creation
 * calls cudaMalloc; a host program whose device memory is all owned by its own pool or arena,
 * or that must not enter the CUDA allocator where it runs, can still reduce populations it
 * already holds on the device with this entry point.  It allocates nothing: its scratch is a
 * static device array of (LBX_NOALLOC_MAX_BLOCKS + 1) * 4 doubles (256 KiB), present on every
 * GPU that loads the library until the process exits.
 *   populations  device array in the exchange layout, column i starting at element
 *                i * column_stride, n_cells cells per column, values f_i - w_i of `storage`;
 *   out          host array {sum rho, sum j_x, sum j_y, sum j_z} (rho = sum_i f_i + 1), FP64;
 *   n_cells      at most LBX_NOALLOC_MAX_CELLS, otherwise LBX_ERR_INVALID before any device work.
 * Runs on the current device and `stream`; every call looks up the scratch's device address on
 * the current device and synchronises the stream, so it must not be called while that stream is
 * being captured.  All calls share the one scratch array: calls that overlap on the GPU race, so
 * serialise them. */
#define LBX_NOALLOC_MAX_BLOCKS 8192
#define LBX_NOALLOC_CELLS_PER_BLOCK 4096
#define LBX_NOALLOC_MAX_CELLS ((int64_t)LBX_NOALLOC_MAX_BLOCKS * LBX_NOALLOC_CELLS_PER_BLOCK)
int lbx_mass_momentum_noalloc(int32_t q, int32_t storage, const void* populations, int64_t n_cells,
                              int64_t column_stride, double out[4], void* stream);

#ifdef __cplusplus
}
#endif

#endif
