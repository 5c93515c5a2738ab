/* Body of the oracle step, included by lbm_oracle.c once per storage/compute type.
 * Expects: REAL (compute type), STORE_T (storage type), LOAD(x), STORE(x), FN(name).
 * TEST INFRASTRUCTURE ONLY (see lbm_oracle.h). */

/* Collision of one fluid cell in place on g[0..q-1] (values f_i - w_i).
 * Returns the cell statistic {rho, |u|^2} through rho_out/usq_out. */
static void FN(collide)(const lbo_desc* d, const lbo_case* c, REAL* g, REAL avg_rho, REAL* rho_out, REAL* usq_out)
{
  const int q = d->q, dim = d->d;
  const REAL invCs2 = (REAL)3;
  REAL t[27];
  for (int i = 0; i < q; ++i) t[i] = (REAL)d->tn[i] / (REAL)d->td[i];

  const int forced = (c->dynamics == LBO_FORCED_BGK || c->dynamics == LBO_FORCED_SMAGORINSKY);
  const REAL F[3] = {(REAL)c->force[0], (REAL)c->force[1], (REAL)c->force[2]};

  /* lbm::computeRho / computeJ / computeRhoU (src/dynamics/lbm.h:289-330) */
  REAL rho = 0;
  for (int i = 0; i < q; ++i) rho += g[i];
  rho += (REAL)1;
  REAL u[3] = {0, 0, 0};
  for (int i = 0; i < q; ++i)
    for (int a = 0; a < dim; ++a) u[a] += g[i] * (REAL)d->c[i][a];
  for (int a = 0; a < dim; ++a) u[a] /= rho;
  /* ForcedMomentum::computeU: u += F/2 (src/dynamics/momenta/elements.h:1600-1608) */
  if (forced)
    for (int a = 0; a < dim; ++a) u[a] += F[a] * (REAL)0.5;
  REAL uSqr = 0;
  for (int a = 0; a < dim; ++a) uSqr += u[a] * u[a];

  REAL omega = (REAL)c->omega;

  if (c->dynamics == LBO_SMAGORINSKY || c->dynamics == LBO_FORCED_SMAGORINSKY) {
    /* SmagorinskyEffectiveOmega::computeEffectiveOmega (src/dynamics/collisionLES.h:59-80)
     * with Pi^neq from lbm::computeStress (lbm.h:333-352), or ForcedStress for the forced
     * variant (momenta/elements.h:1947-1970), and its norm (momenta/interface.h:164-173). */
    REAL us[3] = {u[0], u[1], u[2]};
    if (forced)
      for (int a = 0; a < dim; ++a) us[a] = u[a] - (REAL)0.5 * F[a];
    REAL pi[6];
    int ip = 0;
    for (int a = 0; a < dim; ++a) {
      for (int b = a; b < dim; ++b) {
        REAL s = 0;
        for (int i = 0; i < q; ++i) s += (REAL)d->c[i][a] * (REAL)d->c[i][b] * g[i];
        s -= rho * us[a] * us[b];
        if (a == b) s -= (REAL)1 / invCs2 * (rho - (REAL)1);
        pi[ip++] = s;
      }
    }
    if (forced) {
      ip = 0;
      for (int a = 0; a < dim; ++a)
        for (int b = a; b < dim; ++b)
          pi[ip++] += (REAL)0.5 * rho * (F[a] * us[b] + us[a] * F[b]);
    }
    REAL n2 = pi[0] * pi[0] + (REAL)2 * pi[1] * pi[1] + pi[2] * pi[2];
    if (dim == 3) n2 += pi[2] * pi[2] + pi[3] * pi[3] + (REAL)2 * pi[4] * pi[4] + pi[5] * pi[5];
    const REAL cs = (REAL)c->smagorinsky;
    const REAL piNeqNorm = (REAL)sqrt((double)n2);
    const REAL pre = cs * cs * invCs2 * invCs2 * (REAL)2 * (REAL)sqrt(2.0);
    const REAL tauMol = (REAL)1 / omega;
    const REAL tauTurb = (REAL)0.5 * ((REAL)sqrt((double)(tauMol * tauMol + pre / rho * piNeqNorm)) - tauMol);
    omega = (REAL)1 / (tauMol + tauTurb);
  }

  /* equilibrium::secondOrder (src/dynamics/lbm.h:50-64) */
  REAL feq[27];
  for (int i = 0; i < q; ++i) {
    REAL cu = 0;
    for (int a = 0; a < dim; ++a) cu += (REAL)d->c[i][a] * u[a];
    feq[i] = rho * t[i] * ((REAL)1 + invCs2 * cu + invCs2 * invCs2 * (REAL)0.5 * cu * cu
                           - invCs2 * (REAL)0.5 * uSqr) - t[i];
  }

  if (c->dynamics == LBO_TRT) {
    /* collision::TRT::apply (src/dynamics/collision.h:393-416) */
    REAL fp[27], fm[27], ep[27], em[27];
    for (int i = 0; i < q; ++i) {
      fp[i] = (REAL)0.5 * (g[i] + g[d->opp[i]]);
      fm[i] = (REAL)0.5 * (g[i] - g[d->opp[i]]);
      ep[i] = (REAL)0.5 * (feq[i] + feq[d->opp[i]]);
      em[i] = (REAL)0.5 * (feq[i] - feq[d->opp[i]]);
    }
    const REAL magic = (REAL)c->magic;
    const REAL omega2 = (REAL)1 / (magic / ((REAL)1 / omega - (REAL)0.5) + (REAL)0.5);
    for (int i = 0; i < q; ++i) g[i] -= omega * (fp[i] - ep[i]) + omega2 * (fm[i] - em[i]);
  } else if (c->dynamics == LBO_CONST_RHO_BGK) {
    /* collision::ConstRhoBGK::apply (src/dynamics/collision.h:336-349): the equilibrium is
     * rescaled so that the lattice's average density returns to 1; avg_rho is the
     * AVERAGE_RHO parameter, the statistics' average density of the previous step. */
    const REAL deltaRho = (REAL)1 - avg_rho;
    const REAL ratioRho = (REAL)1 + deltaRho / rho;
    for (int i = 0; i < q; ++i)
      g[i] = ratioRho * (feq[i] + t[i]) - t[i] + ((REAL)1 - omega) * (g[i] - feq[i]);
    *rho_out = rho + deltaRho;
    *usq_out = uSqr;
    return;
  } else {
    /* collision::BGK::apply (src/dynamics/collision.h:68-78) */
    for (int i = 0; i < q; ++i) {
      g[i] *= (REAL)1 - omega;
      g[i] += omega * feq[i];
    }
  }

  if (forced) {
    /* lbm::addExternalForce (src/dynamics/lbm.h:568-588), called by forcing::PlainGuo /
     * forcing::Guo after the collision with the (effective) omega (forcing.h:58-64,141-147) */
    const REAL invCs4 = invCs2 * invCs2;
    for (int i = 0; i < q; ++i) {
      REAL cu = 0;
      for (int a = 0; a < dim; ++a) cu += (REAL)d->c[i][a] * u[a];
      cu *= invCs4;
      REAL ft = 0;
      for (int a = 0; a < dim; ++a)
        ft += (((REAL)d->c[i][a] - u[a]) * invCs2 + cu * (REAL)d->c[i][a]) * F[a];
      ft *= rho * ((REAL)1 - omega * (REAL)0.5) * t[i];
      g[i] += ft;
    }
  }
  *rho_out = rho;
  *usq_out = uSqr;
}

/* Type and outward normal of boundary cell b (see lbo_case). */
static void FN(fd_meta)(const lbo_case* c, int64_t b, int* type, int n[3])
{
  n[0] = n[1] = n[2] = 0;
  if (c->fd_normal) {
    *type = c->fd_type ? c->fd_type[b] : 0;
    for (int a = 0; a < 3; ++a) n[a] = c->fd_normal[3 * b + a];
  } else {
    *type = 0;
    n[c->fd_dir[b]] = c->fd_orient[b];
  }
}

/* Density and velocity of a boundary cell from its momenta
 * (src/dynamics/momenta/aliases.h:173-220):
 *  flat velocity (BasicDirichletVelocityBoundaryTuple): u = imposed (FixedVelocityMomentumGeneric,
 *            elements.h:603-630), rho from velocityBMRho (elements.h:54-71)
 *            = (2 rho_normal + rho_onWall + 1) / (1 + o u_d);
 *  flat pressure (BasicDirichletPressureBoundaryTuple): rho = imposed (FixedDensity,
 *            elements.h:270-280), u = imposed tangential velocity with
 *            u_d = o ((2 rho_normal + rho_onWall + 1) / rho - 1) (FixedPressureMomentum::computeU,
 *            elements.h:653-690);
 *  external edge / corner (FixedVelocityBoundaryTuple): u = imposed, rho = sum f + 1 (BulkDensity);
 *  internal edge / corner (InnerEdgeVelocityTuple3D, InnerCornerVelocityTuple2D / 3D,
 *            aliases.h:224-243): u = imposed, rho = the mean of velocityBMRho along the normal
 *            axes (InnerEdgeDensity3D: axes (plane+1)%3 and (plane+2)%3, plane the edge axis;
 *            InnerCornerDensity2D / 3D: x, y (, z); elements.h:406-483).
 * rho_onWall sums the populations with c_d = 0, rho_normal those with c_d = o, in index order. */
static REAL FN(bm_rho)(const lbo_desc* d, const REAL* g, int dir, int orient, const REAL* u)
{
  REAL onWall = 0, normal = 0;
  for (int i = 0; i < d->q; ++i)
    if (d->c[i][dir] == 0) onWall += g[i];
  for (int i = 0; i < d->q; ++i)
    if (d->c[i][dir] == orient) normal += g[i];
  return ((REAL)2 * normal + onWall + (REAL)1) / ((REAL)1 + (REAL)orient * u[dir]);
}

static void FN(fd_momenta)(const lbo_desc* d, const REAL* g, int kind, int type, const int* nrm,
                           const double* value, REAL* rho, REAL* u)
{
  const int q = d->q, dim = d->d;
  if (type == 2 || type == 4) {
    for (int a = 0; a < dim; ++a) u[a] = (REAL)value[a];
    if (type == 4) {
      int plane = 0;
      for (int a = 0; a < 3; ++a)
        if (nrm[a] == 0) plane = a;
      const int a1 = (plane + 1) % 3, a2 = (plane + 2) % 3;
      *rho = (FN(bm_rho)(d, g, a1, nrm[a1], u) + FN(bm_rho)(d, g, a2, nrm[a2], u)) / (REAL)2;
    } else if (dim == 3) {
      *rho = (FN(bm_rho)(d, g, 0, nrm[0], u) + FN(bm_rho)(d, g, 1, nrm[1], u) + FN(bm_rho)(d, g, 2, nrm[2], u)) /
             (REAL)3;
    } else {
      *rho = (FN(bm_rho)(d, g, 0, nrm[0], u) + FN(bm_rho)(d, g, 1, nrm[1], u)) / (REAL)2;
    }
    return;
  }
  if (type != 0) {
    REAL r = 0;
    for (int i = 0; i < q; ++i) r += g[i];
    *rho = r + (REAL)1;
    for (int a = 0; a < dim; ++a) u[a] = (REAL)value[a];
    return;
  }
  int dir = 0, orient = 0;
  for (int a = dim - 1; a >= 0; --a)
    if (nrm[a] != 0) { dir = a; orient = nrm[a]; }
  REAL onWall = 0, normal = 0;
  for (int i = 0; i < q; ++i)
    if (d->c[i][dir] == 0) onWall += g[i];
  for (int i = 0; i < q; ++i)
    if (d->c[i][dir] == orient) normal += g[i];
  if (kind == 1 || kind == 3 || kind == 5) {
    for (int a = 0; a < dim; ++a) u[a] = (REAL)value[a];
    *rho = ((REAL)2 * normal + onWall + (REAL)1) / ((REAL)1 + (REAL)orient * u[dir]);
  } else {
    for (int a = 0; a < dim; ++a) u[a] = (REAL)value[1 + a];
    *rho = (REAL)value[0];
    u[dir] = (REAL)orient * (((REAL)2 * normal + onWall + (REAL)1) / *rho - (REAL)1);
  }
}

/* f_i^eq - t_i: equilibrium::secondOrder (src/dynamics/lbm.h) with c.u summed axis by axis. */
static REAL FN(second_order)(const lbo_desc* d, int i, REAL rho, const REAL* u, REAL uSqr)
{
  const REAL invCs2 = (REAL)3;
  const REAL t = (REAL)d->tn[i] / (REAL)d->td[i];
  REAL cu = 0;
  for (int a = 0; a < d->d; ++a) cu += (REAL)d->c[i][a] * u[a];
  return rho * t * ((REAL)1 + invCs2 * cu + invCs2 * invCs2 * (REAL)0.5 * cu * cu - invCs2 * (REAL)0.5 * uSqr) - t;
}

/* Pi of a flat local boundary cell: RegularizedBoundaryStress (BoundaryHelpers::computeStress,
 * src/boundary/helper.h:31-81): f^neq of the populations with c_d = 0 (none for i = 0) and of
 * those with c_d = o, the latter counted twice. */
static void FN(flat_stress)(const lbo_desc* d, const REAL* g, REAL rho, const REAL* u, const int* nrm, REAL* pi)
{
  const int q = d->q, dim = d->d;
  int dir = 0, orient = 0;
  for (int a = dim - 1; a >= 0; --a)
    if (nrm[a] != 0) { dir = a; orient = nrm[a]; }
  REAL uSqr = 0;
  for (int a = 0; a < dim; ++a) uSqr += u[a] * u[a];
  REAL fneq[27];
  for (int i = 0; i < q; ++i) fneq[i] = 0;
  for (int i = 1; i < q; ++i)
    if (d->c[i][dir] == 0) fneq[i] = g[i] - FN(second_order)(d, i, rho, u, uSqr);
  for (int i = 0; i < q; ++i)
    if (d->c[i][dir] == orient) fneq[i] = g[i] - FN(second_order)(d, i, rho, u, uSqr);
  int iPi = 0;
  for (int a = 0; a < dim; ++a)
    for (int b = a; b < dim; ++b) {
      pi[iPi] = 0;
      for (int i = 0; i < q; ++i)
        if (d->c[i][dir] == 0) pi[iPi] += (REAL)(d->c[i][a] * d->c[i][b]) * fneq[i];
      for (int i = 0; i < q; ++i)
        if (d->c[i][dir] == orient) pi[iPi] += (REAL)(2 * d->c[i][a] * d->c[i][b]) * fneq[i];
      ++iPi;
    }
}

/* Pi from the second moment of populations h (lbm::computeStress, src/dynamics/lbm.h:333-351:
 * sum_i c_ia c_ib h_i - rho u_a u_b - (rho - 1) / c_s^-2 on the diagonal): BulkStress, and the
 * inner edge / corner stress on their completed cell. */
static void FN(moment_stress)(const lbo_desc* d, const REAL* h, REAL rho, const REAL* u, REAL* pi)
{
  const int q = d->q, dim = d->d;
  const REAL invCs2 = (REAL)3;
  int iPi = 0;
  for (int a = 0; a < dim; ++a)
    for (int b = a; b < dim; ++b) {
      pi[iPi] = 0;
      for (int i = 0; i < q; ++i) pi[iPi] += (REAL)(d->c[i][a] * d->c[i][b]) * h[i];
      pi[iPi] -= rho * u[a] * u[b];
      if (a == b) pi[iPi] -= (REAL)1 / invCs2 * (rho - (REAL)1);
      ++iPi;
    }
}

/* Pi of an internal edge or corner (InnerEdgeStress3D / InnerCornerStress2D / 3D, src/dynamics/
 * momenta/elements.h:1814-1897): a copy of the cell whose unknown populations -- c equal to -n
 * along every normal axis of the edge (the two axes after the edge axis) or corner -- are
 * replaced by f_opp - f^eq_opp + f^eq_i, then its second moment. */
static void FN(inner_stress)(const lbo_desc* d, const REAL* g, REAL rho, const REAL* u, int type, const int* nrm,
                             REAL* pi)
{
  const int q = d->q, dim = d->d;
  REAL uSqr = 0;
  for (int a = 0; a < dim; ++a) uSqr += u[a] * u[a];
  int axes[3], na = 0;
  if (type == 4) {
    int plane = 0;
    for (int a = 0; a < 3; ++a)
      if (nrm[a] == 0) plane = a;
    axes[na++] = (plane + 1) % 3;
    axes[na++] = (plane + 2) % 3;
  } else {
    for (int a = 0; a < dim; ++a) axes[na++] = a;
  }
  REAL h[27];
  for (int i = 0; i < q; ++i) h[i] = g[i];
  for (int i = 0; i < q; ++i) {
    int unknown = 1;
    for (int k = 0; k < na; ++k)
      if (d->c[i][axes[k]] != -nrm[axes[k]]) unknown = 0;
    if (unknown) {
      const int o = d->opp[i];
      h[i] = g[o] - FN(second_order)(d, o, rho, u, uSqr) + FN(second_order)(d, i, rho, u, uSqr);
    }
  }
  FN(moment_stress)(d, h, rho, u, pi);
}

/* fromPiToFneq(i, Pi) (src/dynamics/lbm.h:247-270). */
static REAL FN(fneq_of_pi)(const lbo_desc* d, int i, const REAL* pi)
{
  const int dim = d->d;
  const REAL invCs2 = (REAL)3;
  const REAL t = (REAL)d->tn[i] / (REAL)d->td[i];
  REAL fn = 0;
  int iPi = 0;
  for (int a = 0; a < dim; ++a)
    for (int b = a; b < dim; ++b) {
      REAL toAdd = (REAL)(d->c[i][a] * d->c[i][b]);
      if (a == b) toAdd -= (REAL)1 / invCs2;
      else toAdd *= (REAL)2;
      toAdd *= pi[iPi++];
      fn += toAdd;
    }
  fn *= t * invCs2 * invCs2 / (REAL)2;
  return fn;
}

/* Pi of boundary cell with normal type `type` and kind `kind` through its momenta: flat local
 * cells RegularizedBoundaryStress, internal edges and corners their inner stress, external edges
 * and corners BulkStress (momenta::FixedVelocityBoundaryTuple). */
static void FN(boundary_stress)(const lbo_desc* d, const REAL* g, REAL rho, const REAL* u, int type,
                                const int* nrm, REAL* pi)
{
  if (type == 0) FN(flat_stress)(d, g, rho, u, nrm, pi);
  else if (type == 2 || type == 4) FN(inner_stress)(d, g, rho, u, type, nrm, pi);
  else FN(moment_stress)(d, g, rho, u, pi);
}

/* The regularisation of a local boundary cell, flat or an internal edge or corner
 * (CombinedRLBdynamics::collide, src/dynamics/dynamics.h:505-516, before the mixed-in
 * collision): rho, u and Pi from the boundary momenta, then f_i = f_i^eq(rho, u) +
 * fromPiToFneq(i, Pi). */
static void FN(local_regularize)(const lbo_desc* d, REAL rho, const REAL* u, int type, const int* nrm, REAL* g)
{
  const int q = d->q, dim = d->d;
  REAL uSqr = 0;
  for (int a = 0; a < dim; ++a) uSqr += u[a] * u[a];
  REAL pi[6];
  FN(boundary_stress)(d, g, rho, u, type, nrm, pi);
  for (int i = 0; i < q; ++i) g[i] = FN(second_order)(d, i, rho, u, uSqr) + FN(fneq_of_pi)(d, i, pi);
}

/* RLB collision with the boundary momenta (collision::RLB, src/dynamics/collision.h:82-112):
 * f_i = f_i^eq(rho, u) + (1 - omega) fromPiToFneq(i, Pi), Pi from the momenta's stress. */
static REAL FN(rlb_with)(const lbo_desc* d, REAL omega, REAL rho, const REAL* u, int type, const int* nrm, REAL* g)
{
  const int q = d->q, dim = d->d;
  REAL uSqr = 0;
  for (int a = 0; a < dim; ++a) uSqr += u[a] * u[a];
  REAL pi[6];
  FN(boundary_stress)(d, g, rho, u, type, nrm, pi);
  for (int i = 0; i < q; ++i)
    g[i] = FN(second_order)(d, i, rho, u, uSqr) + ((REAL)1 - omega) * FN(fneq_of_pi)(d, i, pi);
  return uSqr;
}

/* BGK collision with given rho, u: lbm::bgkCollision (src/dynamics/lbm.h:395-403). */
static REAL FN(bgk_with)(const lbo_desc* d, REAL omega, REAL rho, const REAL* u, REAL* g)
{
  const int q = d->q, dim = d->d;
  const REAL invCs2 = (REAL)3;
  REAL uSqr = 0;
  for (int a = 0; a < dim; ++a) uSqr += u[a] * u[a];
  for (int i = 0; i < q; ++i) {
    const REAL t = (REAL)d->tn[i] / (REAL)d->td[i];
    REAL cu = 0;
    for (int a = 0; a < dim; ++a) cu += (REAL)d->c[i][a] * u[a];
    const REAL feq = rho * t * ((REAL)1 + invCs2 * cu + invCs2 * invCs2 * (REAL)0.5 * cu * cu
                                - invCs2 * (REAL)0.5 * uSqr) - t;
    g[i] *= (REAL)1 - omega;
    g[i] += omega * feq;
  }
  return uSqr;
}

/* u of a bulk cell: BulkMomentum::computeU (elements.h:500-508) = j / rho, plus F / 2 for the
 * forced dynamics (ForcedMomentum, elements.h:1600-1608). */
static void FN(bulk_u)(const lbo_desc* d, const lbo_case* c, const REAL* g, REAL* u)
{
  const int q = d->q, dim = d->d;
  for (int a = 0; a < dim; ++a) u[a] = 0;
  for (int i = 0; i < q; ++i)
    for (int a = 0; a < dim; ++a) u[a] += g[i] * (REAL)d->c[i][a];
  REAL rho = 0;
  for (int i = 0; i < q; ++i) rho += g[i];
  rho += (REAL)1;
  const int forced = (c->dynamics == LBO_FORCED_BGK || c->dynamics == LBO_FORCED_SMAGORINSKY);
  for (int a = 0; a < dim; ++a) {
    u[a] /= rho;
    if (forced) u[a] += (REAL)c->force[a] * (REAL)0.5;
  }
}

/* Cell index of p, -1 beyond a non-periodic face; *wrapped set when a periodic face was crossed. */
static int64_t FN(fd_index)(const lbo_case* c, int64_t p0, int64_t p1, int64_t p2, int* wrapped)
{
  const int64_t ext[3] = {c->nx, c->ny, c->nz};
  int64_t p[3] = {p0, p1, p2};
  *wrapped = 0;
  for (int a = 0; a < 3; ++a) {
    if (p[a] >= 0 && p[a] < ext[a]) continue;
    if (!((c->periodic >> a) & 1)) return -1;
    p[a] = (p[a] + ext[a]) % ext[a];
    *wrapped = 1;
  }
  return (p[0] * ext[1] + p[1]) * ext[2] + p[2];
}

/* Velocity the finite differences read at cell m (cell.computeU through its dynamics): a
 * boundary cell of the list its momenta on the current (in-place updated) populations, a bulk
 * cell j / rho, a cell without dynamics or with plain bounce-back zero (ZeroMomentum), and so a
 * cell beyond a non-periodic face (the reference's overlap carries NoDynamics there).  A
 * neighbour reached across a periodic face is the overlap copy of the partner cell, which the
 * post-stream communication filled with the partner's populations before any post-processor ran
 * (core/superLattice.hh:800-820, boundary/setBoundary3D.h:56-110) and which carries the
 * partner's dynamics as defined before boundary::set (boundary::set skips the overlap,
 * setBoundary.h:83-86): bulk for a boundary cell. */
static void FN(fd_u_of)(const lbo_desc* d, const lbo_case* c, const STORE_T* f, const STORE_T* pre,
                        const int64_t* fdIndex, int64_t m, int wrapped, REAL* u)
{
  const int q = d->q;
  const int64_t n = (int64_t)c->nx * c->ny * c->nz;
  REAL g[27];
  u[0] = u[1] = u[2] = 0;
  if (m < 0) return;
  const int mat = c->material ? c->material[m] : LBO_FLUID;
  if (mat == LBO_SOLID || mat == LBO_BOUNCE_BACK) return;
  if (mat == LBO_BOUNCE_BACK_VELOCITY) { /* FixedVelocityMomentum */
    for (int a = 0; a < d->d; ++a) u[a] = (REAL)c->bbv_value[4 * m + 1 + a];
    return;
  }
  if (wrapped) {
    for (int i = 0; i < q; ++i) g[i] = LOAD(pre[i * n + m]);
    FN(bulk_u)(d, c, g, u);
    return;
  }
  for (int i = 0; i < q; ++i) g[i] = LOAD(f[i * n + m]);
  const int64_t b = fdIndex[m];
  if (b >= 0) {
    REAL rho;
    int type, nrm[3];
    FN(fd_meta)(c, b, &type, nrm);
    FN(fd_momenta)(d, g, c->fd_kind[b], type, nrm, c->fd_value + 4 * b, &rho, u);
  } else {
    FN(bulk_u)(d, c, g, u);
  }
}

/* Density at cell m (cell.computeRho through its dynamics), on the current populations. */
static REAL FN(fd_rho_of)(const lbo_desc* d, const lbo_case* c, const STORE_T* f, const int64_t* fdIndex, int64_t m)
{
  const int q = d->q;
  const int64_t n = (int64_t)c->nx * c->ny * c->nz;
  if (m < 0) return (REAL)1;
  const int mat = c->material ? c->material[m] : LBO_FLUID;
  if (mat == LBO_SOLID || mat == LBO_BOUNCE_BACK) return (REAL)1;
  if (mat == LBO_BOUNCE_BACK_VELOCITY) return (REAL)c->bbv_value[4 * m]; /* FixedDensity */
  REAL g[27];
  for (int i = 0; i < q; ++i) g[i] = LOAD(f[i * n + m]);
  const int64_t b = fdIndex[m];
  if (b >= 0) {
    REAL rho, u[3] = {0, 0, 0};
    int type, nrm[3];
    FN(fd_meta)(c, b, &type, nrm);
    FN(fd_momenta)(d, g, c->fd_kind[b], type, nrm, c->fd_value + 4 * b, &rho, u);
    return rho;
  }
  REAL r = 0;
  for (int i = 0; i < q; ++i) r += g[i];
  return r + (REAL)1;
}

/* The post-stream boundary processors, one cell after the other in ascending cell order and in
 * place, as the CPU post-processor loop runs them (core/platform/cpu/sisd/operator.h:368-385),
 * by priority: the flat faces (PlaneFdBoundaryProcessor3D::apply, src/boundary/
 * boundaryPostProcessors3D.hh:39-93; StraightFdBoundaryProcessor2D::apply,
 * boundaryPostProcessors2D.hh:39-76) and the external edges (OuterVelocityEdgeProcessor3D,
 * boundaryPostProcessors3D.hh:164-238) at priority 0, then the external corners
 * (OuterVelocityCornerProcessor3D / 2D, 3D.hh:240-294, 2D.hh:276-323) at priority 1.  Velocity
 * gradients by fd::DirectedGradients (utilities/finiteDifference3D.h:74-210: one-sided second
 * order along each non-zero normal component, central along the other axes); rho: the cell's
 * momenta on a flat face, 2/3 (rho_01 + rho_10) - 1/6 (rho_02 + rho_20) on an edge or a 2D corner
 * (the cells one and two steps inward along its normal axes), 4/9 (rho_001 + rho_010 + rho_100)
 * - 1/9 (rho_002 + rho_020 + rho_200) on a 3D corner; Pi = -rho / (c_s^-2 omega)
 * (grad u + grad u^T), and f_i = f_i^eq(rho, u) + fromPiToFneq(i, Pi) (dynamics/lbm.h:247-270). */
static void FN(fd_postprocess)(const lbo_desc* d, const lbo_case* c, STORE_T* f, const STORE_T* pre,
                               const int64_t* fdIndex)
{
  const int q = d->q, dim = d->d;
  const int64_t ny = c->ny, nz = c->nz, n = (int64_t)c->nx * ny * nz;
  const REAL invCs2 = (REAL)3;
  const REAL omega = (REAL)c->omega;
  for (int pass = 0; pass < 2; ++pass) {
    for (int64_t b = 0; b < c->n_fd; ++b) {
      int type, nrm[3];
      FN(fd_meta)(c, b, &type, nrm);
      if ((type == 1) != (pass == 1)) continue;
      if (c->fd_kind[b] >= 3 && type == 0) continue;  /* local flat cells: no post-processor */
      if (type == 2 || type == 4) continue;              /* internal edges and corners: none either */
      const int64_t cell = c->fd_cell[b];
      const int64_t pos[3] = {cell / (ny * nz), (cell / nz) % ny, cell % nz};
      REAL g[27], rho, u[3] = {0, 0, 0};
      for (int i = 0; i < q; ++i) g[i] = LOAD(f[i * n + cell]);
      FN(fd_momenta)(d, g, c->fd_kind[b], type, nrm, c->fd_value + 4 * b, &rho, u);
      if (type != 0) {
        /* densities of the cells one (r1) and two (r2) steps inward along each normal axis */
        REAL r1[3] = {0, 0, 0}, r2[3] = {0, 0, 0};
        for (int a = 0; a < dim; ++a) {
          if (nrm[a] == 0) continue;
          for (int k = 1; k <= 2; ++k) {
            int64_t p[3] = {pos[0], pos[1], pos[2]};
            p[a] -= k * nrm[a];
            int w;
            const REAL r = FN(fd_rho_of)(d, c, f, fdIndex, FN(fd_index)(c, p[0], p[1], p[2], &w));
            if (k == 1) r1[a] = r; else r2[a] = r;
          }
        }
        if (dim == 3 && type == 1) {
          rho = (REAL)4 / (REAL)9 * (r1[2] + r1[1] + r1[0]) - (REAL)1 / (REAL)9 * (r2[2] + r2[1] + r2[0]);
        } else {
          int A = 0, B = 1;
          if (dim == 3) {
            int plane = 0;
            for (int a = 0; a < 3; ++a)
              if (nrm[a] == 0) plane = a;
            A = (plane + 1) % 3;
            B = (plane + 2) % 3;
          }
          rho = (REAL)2 / (REAL)3 * (r1[B] + r1[A]) - (REAL)1 / (REAL)6 * (r2[B] + r2[A]);
        }
      }
      REAL grad[3][3] = {{0}};  /* grad[a][iD] = d u_iD / d x_a */
      for (int a = 0; a < dim; ++a) {
        REAL ua[3] = {0, 0, 0}, ub[3] = {0, 0, 0};
        if (nrm[a] != 0) {
          const int o = nrm[a];
          for (int k = 1; k <= 2; ++k) {
            int64_t p[3] = {pos[0], pos[1], pos[2]};
            p[a] -= k * o;
            int w;
            const int64_t m = FN(fd_index)(c, p[0], p[1], p[2], &w);
            FN(fd_u_of)(d, c, f, pre, fdIndex, m, 0, k == 1 ? ua : ub);
          }
          for (int iD = 0; iD < dim; ++iD)
            grad[a][iD] = (REAL)(-o) * (((REAL)-3 * u[iD] + (REAL)4 * ua[iD]) - (REAL)1 * ub[iD]) / (REAL)2;
        } else {
          for (int k = 0; k < 2; ++k) {
            int64_t p[3] = {pos[0], pos[1], pos[2]};
            p[a] += k == 0 ? 1 : -1;
            int wrapped;
            const int64_t m = FN(fd_index)(c, p[0], p[1], p[2], &wrapped);
            FN(fd_u_of)(d, c, f, pre, fdIndex, m, wrapped, k == 0 ? ua : ub);
          }
          for (int iD = 0; iD < dim; ++iD) grad[a][iD] = (ua[iD] - ub[iD]) / (REAL)2;
        }
      }
      const REAL sToPi = -rho / invCs2 / omega;
      REAL pi[6];
      if (dim == 3) {
        pi[0] = (REAL)2 * grad[0][0] * sToPi;             /* xx */
        pi[3] = (REAL)2 * grad[1][1] * sToPi;             /* yy */
        pi[5] = (REAL)2 * grad[2][2] * sToPi;             /* zz */
        pi[1] = (grad[0][1] + grad[1][0]) * sToPi;        /* xy */
        pi[2] = (grad[0][2] + grad[2][0]) * sToPi;        /* xz */
        pi[4] = (grad[1][2] + grad[2][1]) * sToPi;        /* yz */
      } else {
        pi[0] = (REAL)2 * grad[0][0] * sToPi;             /* xx */
        pi[2] = (REAL)2 * grad[1][1] * sToPi;             /* yy */
        pi[1] = (grad[0][1] + grad[1][0]) * sToPi;        /* xy */
      }
      REAL uSqr = 0;
      for (int a = 0; a < dim; ++a) uSqr += u[a] * u[a];
      for (int i = 0; i < q; ++i) {
        const REAL t = (REAL)d->tn[i] / (REAL)d->td[i];
        REAL cu = 0;
        for (int a = 0; a < dim; ++a) cu += (REAL)d->c[i][a] * u[a];
        const REAL feq = rho * t * ((REAL)1 + invCs2 * cu + invCs2 * invCs2 * (REAL)0.5 * cu * cu
                                    - invCs2 * (REAL)0.5 * uSqr) - t;
        REAL fneq = 0;
        int ip = 0;
        for (int al = 0; al < dim; ++al) {
          for (int be = al; be < dim; ++be) {
            REAL add = (REAL)d->c[i][al] * (REAL)d->c[i][be];
            if (al == be) add -= (REAL)1 / invCs2;
            else add *= (REAL)2;
            add *= pi[ip++];
            fneq += add;
          }
        }
        fneq *= t * invCs2 * invCs2 / (REAL)2;
        f[i * n + cell] = STORE(feq + fneq);
      }
    }
  }
}

static int FN(run)(const lbo_case* c, STORE_T* f, int64_t steps, double* stats)
{
  const lbo_desc* d = lbo_get_desc(c->q);
  if (!d || c->nx <= 0 || c->ny <= 0 || c->nz <= 0 || (d->d == 2 && c->nz != 1)) return -1;
  const int q = d->q;
  const int64_t nx = c->nx, ny = c->ny, nz = c->nz;
  const int64_t n = nx * ny * nz;
  STORE_T* tmp = (STORE_T*)malloc(sizeof(STORE_T) * (size_t)(q * n));
  REAL* cellRho = (REAL*)malloc(sizeof(REAL) * (size_t)n);
  REAL* cellUsq = (REAL*)malloc(sizeof(REAL) * (size_t)n);
  int64_t* fdIndex = (int64_t*)malloc(sizeof(int64_t) * (size_t)n);
  STORE_T* pre = c->n_fd > 0 ? (STORE_T*)malloc(sizeof(STORE_T) * (size_t)(q * n)) : NULL;
  if (!tmp || !cellRho || !cellUsq || !fdIndex || (c->n_fd > 0 && !pre)) {
    free(tmp); free(cellRho); free(cellUsq); free(fdIndex); free(pre);
    return -2;
  }
  for (int64_t x = 0; x < n; ++x) fdIndex[x] = -1;
  for (int64_t b = 0; b < c->n_fd; ++b) fdIndex[c->fd_cell[b]] = b;

  /* AVERAGE_RHO: the superlattice statistics' average density, 1 before the first step
   * (latticeStatistics.hh:137), set before every collision (superLattice.hh:675-677) */
  REAL avgRho = (REAL)1;
  const int constRho = c->dynamics == LBO_CONST_RHO_BGK;
  for (int64_t s = 0; s < steps; ++s) {
    /* collide (ConcreteBlockCollisionO<..CPU_SISD..>::apply, cpu/sisd/operator.h:143-228) */
#pragma omp parallel for schedule(static) if (n > 200000)
    for (int64_t x = 0; x < n; ++x) {
      const int m = c->material ? c->material[x] : LBO_FLUID;
      cellRho[x] = (REAL)-1;
      cellUsq[x] = (REAL)-1;
      if (m == LBO_FLUID || (m >= LBO_FLUID_CLASS_1 && m <= LBO_FLUID_CLASS_3 && c->class_params)) {
        lbo_case cc = *c;
        if (m != LBO_FLUID) {
          const double* cp = c->class_params + 6 * (m - LBO_FLUID_CLASS_1);
          if (c->class_dynamics && c->class_dynamics[m - LBO_FLUID_CLASS_1] >= 0)
            cc.dynamics = c->class_dynamics[m - LBO_FLUID_CLASS_1];
          cc.omega = cp[0];
          cc.magic = cp[1];
          cc.smagorinsky = cp[2];
          for (int a = 0; a < 3; ++a) cc.force[a] = cp[3 + a];
        }
        REAL g[27];
        for (int i = 0; i < q; ++i) g[i] = LOAD(f[i * n + x]);
        FN(collide)(d, &cc, g, avgRho, &cellRho[x], &cellUsq[x]);
        for (int i = 0; i < q; ++i) f[i * n + x] = STORE(g[i]);
      } else if (m == LBO_FD_BOUNDARY && fdIndex[x] >= 0) {
        /* BGKdynamics with the boundary momenta exchanged in (collision::BGK::apply,
         * collision.h:68-78, with MOMENTA::computeRhoU of the tuple above) */
        const int64_t b = fdIndex[x];
        REAL g[27], rho, u[3] = {0, 0, 0};
        int type, nrm[3];
        FN(fd_meta)(c, b, &type, nrm);
        for (int i = 0; i < q; ++i) g[i] = LOAD(f[i * n + x]);
        FN(fd_momenta)(d, g, c->fd_kind[b], type, nrm, c->fd_value + 4 * b, &rho, u);
        if ((c->fd_kind[b] >= 3 && type == 0) || type == 2 || type == 4) {
          /* local flat cell, internal edge / corner: CombinedRLBdynamics, regularised first, then
           * the mixed-in collision with the momenta of the rebuilt cell */
          FN(local_regularize)(d, rho, u, type, nrm, g);
          FN(fd_momenta)(d, g, c->fd_kind[b], type, nrm, c->fd_value + 4 * b, &rho, u);
        }
        /* the mixed-in dynamics: RLB for kinds 5 and 6, BGK otherwise */
        if (c->fd_kind[b] >= 5) cellUsq[x] = FN(rlb_with)(d, (REAL)c->omega, rho, u, type, nrm, g);
        else cellUsq[x] = FN(bgk_with)(d, (REAL)c->omega, rho, u, g);
        cellRho[x] = rho;
        for (int i = 0; i < q; ++i) f[i * n + x] = STORE(g[i]);
      } else if (m == LBO_BOUNCE_BACK) {
        for (int i = 1; i <= q / 2; ++i) {
          STORE_T a = f[i * n + x];
          f[i * n + x] = f[d->opp[i] * n + x];
          f[d->opp[i] * n + x] = a;
        }
      } else if (m == LBO_BOUNCE_BACK_VELOCITY) {
        /* collision::Revert, then NguyenLaddCorrection (collision.h:495-521):
         * f_i += 2 rho u_a c_ia t_i invCs2, axis after axis; statistic {rho, |u|^2} */
        REAL g[27];
        for (int i = 0; i < q; ++i) g[i] = LOAD(f[i * n + x]);
        for (int i = 1; i <= q / 2; ++i) {
          const REAL a = g[i];
          g[i] = g[d->opp[i]];
          g[d->opp[i]] = a;
        }
        const double* v = c->bbv_value + 4 * x;
        const REAL rho = (REAL)v[0];
        REAL u[3] = {0, 0, 0};
        for (int a = 0; a < d->d; ++a) u[a] = (REAL)v[1 + a];
        for (int i = 1; i < q; ++i) {
          const REAL t = (REAL)d->tn[i] / (REAL)d->td[i];
          for (int a = 0; a < d->d; ++a) g[i] += (REAL)2 * rho * u[a] * (REAL)d->c[i][a] * t * (REAL)3;
        }
        for (int i = 0; i < q; ++i) f[i * n + x] = STORE(g[i]);
        REAL uSqr = 0;
        for (int a = 0; a < d->d; ++a) uSqr += u[a] * u[a];
        cellRho[x] = rho;
        cellUsq[x] = uSqr;
      }
    }
    /* statistics, accumulated in cell order (latticeStatistics.hh:183-192, 60-90) */
    if (stats || constRho) {
      double sr = 0, se = 0, mx = 0;
      int64_t cnt = 0;
      REAL sumR = 0, sumE = 0, maxE = 0;
      for (int64_t x = 0; x < n; ++x) {
        if (cellRho[x] != (REAL)-1 && cellUsq[x] != (REAL)-1) {
          sumR += cellRho[x];
          sumE += cellUsq[x];
          if (cellUsq[x] > maxE) maxE = cellUsq[x];
          ++cnt;
        }
      }
      sr = (double)sumR; se = (double)sumE; mx = (double)maxE;
      if (stats) {
        stats[3 * s + 0] = cnt ? sr / (double)cnt : 1.0;
        stats[3 * s + 1] = cnt ? 0.5 * se / (double)cnt : 1.0;
        stats[3 * s + 2] = sqrt(mx);
      }
      if (cnt) {
        /* the block average, then the superlattice's cell-count-weighted mean of the block
         * averages (superLattice.hh:61-106; one block of spacing 1: weight = cell count) */
        const REAL w = (REAL)cnt;
        const REAL avgBlock = sumR / w;
        avgRho = avgBlock * w / w;
      }
    }
    /* stream: f_i(x) <- f_i(x - c_i).  This is what the reference's periodic-shift rotation
     * (ConcreteBlockLattice::stream, core/blockLattice.hh:316-338) plus the periodic overlap
     * copy amount to for the core cells.  Sources outside a non-periodic domain are 0. */
    memcpy(tmp, f, sizeof(STORE_T) * (size_t)(q * n));
    for (int i = 0; i < q; ++i) {
      const int cx = d->c[i][0], cy = d->c[i][1], cz = (d->d == 3) ? d->c[i][2] : 0;
#pragma omp parallel for schedule(static) if (n > 200000)
      for (int64_t x = 0; x < nx; ++x) {
        for (int64_t y = 0; y < ny; ++y) {
          for (int64_t z = 0; z < nz; ++z) {
            int64_t sx = x - cx, sy = y - cy, sz = z - cz;
            STORE_T v = STORE((REAL)0);
            if (c->periodic & 1) sx = (sx + nx) % nx;
            if (c->periodic & 2) sy = (sy + ny) % ny;
            if (c->periodic & 4) sz = (sz + nz) % nz;
            if (sx >= 0 && sx < nx && sy >= 0 && sy < ny && sz >= 0 && sz < nz) {
              v = tmp[i * n + (sx * ny + sy) * nz + sz];
            }
            f[i * n + (x * ny + y) * nz + z] = v;
          }
        }
      }
    }
    /* halfway bounce-back: BouzidiVelocityPostProcessor::apply with q = 1/2
     * (src/boundary/setBouzidiBoundary.h:129-162): f_opp(k)(x_b) = f_k(x_b + c_k)
     * - 2 * (c_k . u_w) * t_k * invCs2 */
    for (int64_t l = 0; l < c->n_links; ++l) {
      const int64_t xb = c->link_cell[l];
      const int k = c->link_dir[l];
      int64_t bx = xb / (ny * nz), by = (xb / nz) % ny, bz = xb % nz;
      int64_t sx = bx + d->c[k][0], sy = by + d->c[k][1], sz = bz + ((d->d == 3) ? d->c[k][2] : 0);
      if (c->periodic & 1) sx = (sx + nx) % nx;
      if (c->periodic & 2) sy = (sy + ny) % ny;
      if (c->periodic & 4) sz = (sz + nz) % nz;
      if (sx < 0 || sx >= nx || sy < 0 || sy >= ny || sz < 0 || sz >= nz) continue;
      const int64_t xs = (sx * ny + sy) * nz + sz;
      const REAL tk = (REAL)d->tn[k] / (REAL)d->td[k];
      const REAL veloTerm = (c->link_wall ? (REAL)c->link_wall[l] : (REAL)0) * tk * (REAL)3;
      f[d->opp[k] * n + xb] = STORE(LOAD(f[k * n + xs]) - (REAL)2 * veloTerm);
    }
    if (c->n_fd > 0) {
      memcpy(pre, f, sizeof(STORE_T) * (size_t)(q * n));
      FN(fd_postprocess)(d, c, f, pre, fdIndex);
    }
  }
  free(tmp); free(cellRho); free(cellUsq); free(fdIndex); free(pre);
  return 0;
}
