/* CPU oracle for the lattice Boltzmann hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference algorithm (OpenLB 1.8r1) for one fused
 * collide-and-stream step plus the halfway bounce-back post-processor and the lattice
 * statistics.  Only tests/, the smoke check and bench.py's cpu_baseline leg may load it;
 * the shipped CUDA path never calls it.  Each routine cites the reference file:line it
 * restates (paths relative to the reference project).  It is pinned against dumps of the
 * reference's own CPU code (oracle/ref_driver.cpp) committed under tests/golden/.
 *
 * Population layout: f[i * ncells + cell], cell = (x * ny + y) * nz + z (z fastest, the
 * reference's BlockStructure order, src/core/blockStructure.h:71), holding f_i - w_i
 * (src/dynamics/lbm.h:57-63, 296).
 */
#ifndef LBM_ORACLE_H
#define LBM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum lbo_dynamics {
  LBO_BGK = 0,        /* BGKdynamics                 src/dynamics/dynamics.h:89-99 */
  LBO_TRT = 1,        /* TRTdynamics                 src/dynamics/dynamics.h:529-536 */
  LBO_SMAGORINSKY = 2,/* SmagorinskyBGKdynamics      src/dynamics/smagorinskyBGKdynamics.h:39-44 */
  LBO_FORCED_BGK = 3, /* ForcedBGKdynamics (Guo)     src/dynamics/dynamics.h:223-230 */
  LBO_FORCED_SMAGORINSKY = 4, /* SmagorinskyForcedBGKdynamics smagorinskyBGKdynamics.h:67-73 */
  LBO_CONST_RHO_BGK = 5       /* ConstRhoBGKdynamics dynamics.h:209-215, collision.h:322-351 */
};

enum lbo_material {
  LBO_SOLID = 0,      /* NoDynamics: left untouched (dynamics.h:51-63) */
  LBO_FLUID = 1,      /* the case's bulk dynamics */
  LBO_BOUNCE_BACK = 4,/* BounceBack = collision::Revert (collision.h:465-484) */
  LBO_FD_BOUNDARY = 5, /* velocity / pressure boundary cell: BGK with boundary momenta (fd_* below) */
  LBO_BOUNCE_BACK_VELOCITY = 6, /* BounceBackVelocity (dynamics.h:629-637): bbv_value below */
  /* the case's bulk dynamics with the parameters of class 1, 2 or 3 (class_params below): a
   * second fluid dynamics of the same kind in one block, e.g. BGK beside ForcedBGK (class force
   * 0) as dynamics::set gives them per material */
  LBO_FLUID_CLASS_1 = 8,
  LBO_FLUID_CLASS_2 = 9,
  LBO_FLUID_CLASS_3 = 10
};

typedef struct {
  int32_t q;             /* 9, 19 or 27 */
  int32_t nx, ny, nz;    /* core extents; nz = 1 for D2Q9 */
  int32_t periodic;      /* bit a set: periodic along axis a (1 x, 2 y, 4 z) */
  int32_t dynamics;      /* enum lbo_dynamics */
  double omega, magic, smagorinsky;
  double force[3];       /* body force (acceleration) of the forced dynamics */
  const int32_t* material;   /* per cell, enum lbo_material; NULL = all fluid */
  int64_t n_links;           /* halfway bounce-back links (Bouzidi q = 1/2) */
  const int64_t* link_cell;  /* fluid boundary cell x_b */
  const int32_t* link_dir;   /* k: direction from x_b into the solid neighbour x_b + c_k */
  const double* link_wall;   /* c_k . u_wall per link (NULL: resting walls) */
  /* Flat-face velocity / pressure boundary cells (boundary::InterpolatedVelocity and
   * boundary::InterpolatedPressure on faces whose tangential axes are periodic):
   * src/boundary/interpolatedVelocity3D.h:45-52,78-80, interpolatedPressure3D.h:48-90. */
  int64_t n_fd;
  const int64_t* fd_cell;    /* core cell, ascending */
  const int32_t* fd_kind;    /* 1 velocity, 2 pressure (interpolated); 3 velocity, 4 pressure
                                (local: boundary::LocalVelocity / LocalPressure with BGK mixed
                                in; flat cells regularised in the collision, no post-processor;
                                src/boundary/localVelocity3D.h:47-115, localPressure3D.h,
                                dynamics/dynamics.h:470-523); 5 velocity, 6 pressure (local with
                                their default RLB mixin, src/dynamics/collision.h:82-112) */
  const int32_t* fd_dir;     /* normal axis */
  const int32_t* fd_orient;  /* outward normal sign, -1 or +1 */
  const double* fd_value;    /* 4 per cell: the velocity, or {rho, tangential velocity} */
  /* Optional (NULL: every cell flat with the normal of fd_dir / fd_orient): the discrete normal
   * type (0 flat, 1 external corner, 2 internal corner, 3 external edge, 4 internal edge;
   * geometry/discreteNormals.h:33-39) and the outward normal, 3 per cell.  Edges and corners
   * carry an imposed velocity (boundary/interpolatedVelocity3D.h:45-90,
   * interpolatedVelocity2D.h:45-80); internal ones are regularised in their collision
   * (CombinedRLBdynamics with the inner edge / corner momenta, no post-processor). */
  const int32_t* fd_type;
  const int32_t* fd_normal;
  /* {rho, u_x, u_y, u_z} per cell (all cells; read for the LBO_BOUNCE_BACK_VELOCITY ones) */
  const double* bbv_value;
  /* {omega, magic, smagorinsky, force_x, force_y, force_z} of classes 1..3 (read for the
   * LBO_FLUID_CLASS_* cells) */
  const double* class_params;
  /* Optional (NULL: the case's own dynamics for every class): the dynamics of classes 1..3
   * (enum lbo_dynamics, -1: the case's own), e.g. TRTdynamics on one material beside
   * BGKdynamics on another (dynamics::set per material, core/blockDynamicsMap.h:264-310) */
  const int32_t* class_dynamics;
} lbo_case;

/* Run `steps` collide-and-stream steps in place.  stats (may be NULL) receives per step
 * {average rho, average energy, max |u|} as the reference's LatticeStatistics reports them
 * (src/core/latticeStatistics.hh:60-90).  Returns 0, or a negative code on bad input. */
int lbo_run_f64(const lbo_case* c, double* f, int64_t steps, double* stats);
int lbo_run_f32(const lbo_case* c, float* f, int64_t steps, double* stats);

/* Reduced-precision storage: f_i - w_i held as IEEE binary16 (storage = 1) or bfloat16
 * (storage = 2), round-to-nearest-even on every store, collision in float. */
int lbo_run_half(const lbo_case* c, uint16_t* f, int32_t storage, int64_t steps, double* stats);

/* f_i^eq - w_i for density rho and velocity u (equilibrium::secondOrder, lbm.h:50-64). */
void lbo_equilibrium_f64(int32_t q, double rho, const double* u, double* feq);

/* Conversions used by the reduced-precision storage (round to nearest even). */
uint16_t lbo_float_to_half(float v);
float lbo_half_to_float(uint16_t h);
uint16_t lbo_float_to_bf16(float v);
float lbo_bf16_to_float(uint16_t h);

#ifdef __cplusplus
}
#endif

#endif
