/* Body of the oracle step, included by lbm_oracle.c once per storage/compute type.
 * Expects: REAL (compute type), STORE_T (storage type), LOAD(x), STORE(x), FN(name).
 * TEST INFRASTRUCTURE ONLY (see lbm_oracle.h). */

/* Collision of one fluid cell in place on g[0..q-1] (values f_i - w_i).
 * Returns the cell statistic {rho, |u|^2} through rho_out/usq_out. */
static void FN(collide)(const lbo_desc* d, const lbo_case* c, REAL* g, REAL* rho_out, REAL* usq_out)
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
  if (!tmp || !cellRho || !cellUsq) { free(tmp); free(cellRho); free(cellUsq); return -2; }

  for (int64_t s = 0; s < steps; ++s) {
    /* collide (ConcreteBlockCollisionO<..CPU_SISD..>::apply, cpu/sisd/operator.h:143-228) */
#pragma omp parallel for schedule(static) if (n > 200000)
    for (int64_t x = 0; x < n; ++x) {
      const int m = c->material ? c->material[x] : LBO_FLUID;
      cellRho[x] = (REAL)-1;
      cellUsq[x] = (REAL)-1;
      if (m == LBO_FLUID) {
        REAL g[27];
        for (int i = 0; i < q; ++i) g[i] = LOAD(f[i * n + x]);
        FN(collide)(d, c, g, &cellRho[x], &cellUsq[x]);
        for (int i = 0; i < q; ++i) f[i * n + x] = STORE(g[i]);
      } else if (m == LBO_BOUNCE_BACK) {
        for (int i = 1; i <= q / 2; ++i) {
          STORE_T a = f[i * n + x];
          f[i * n + x] = f[d->opp[i] * n + x];
          f[d->opp[i] * n + x] = a;
        }
      }
    }
    /* statistics, accumulated in cell order (latticeStatistics.hh:183-192, 60-90) */
    if (stats) {
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
      stats[3 * s + 0] = cnt ? sr / (double)cnt : 1.0;
      stats[3 * s + 1] = cnt ? 0.5 * se / (double)cnt : 1.0;
      stats[3 * s + 2] = sqrt(mx);
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
  }
  free(tmp); free(cellRho); free(cellUsq);
  return 0;
}
