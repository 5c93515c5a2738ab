// Per-cell collision algebra of the bulk dynamics, in registers.
//
// Written from the reference's generic dynamics templates (paths relative to the reference
// project).  The floating-point operation order follows those templates so that the FP64
// kernels, compiled without FMA contraction, reproduce the reference's CPU_SISD results
// built with its DISABLE_CSE feature:
//   moments          lbm<>::computeRho/computeJ/computeRhoU   src/dynamics/lbm.h:289-330
//   forced velocity  momenta::ForcedMomentum::computeU        src/dynamics/momenta/elements.h:1600-1608
//   equilibrium      equilibrium<>::secondOrder               src/dynamics/lbm.h:50-64
//   BGK              collision::BGK::apply                    src/dynamics/collision.h:68-78
//   TRT              collision::TRT::apply                    src/dynamics/collision.h:393-416
//   Smagorinsky      SmagorinskyEffectiveOmega                src/dynamics/collisionLES.h:59-89
//                    Pi^neq: lbm<>::computeStress lbm.h:333-352, ForcedStress elements.h:1947-1970,
//                    norm momenta/interface.h:164-173
//   Guo forcing      forcing::PlainGuo / forcing::Guo         src/dynamics/forcing.h:35-65, 115-151
//                    lbm<>::addExternalForce                   src/dynamics/lbm.h:568-588
//   bounce-back      collision::Revert                        src/dynamics/collision.h:465-484
#pragma once

#include "lbx_desc.cuh"

namespace lbx {

enum Dyn : int {
  DYN_BGK = 1,
  DYN_TRT = 2,
  DYN_SMAGORINSKY = 3,
  DYN_FORCED_BGK = 4,
  DYN_FORCED_SMAGORINSKY = 5
};

template <typename R>
struct CollisionParams {
  R omega;
  R magic;
  R smagorinsky;
  R force[3];
};

template <int DYN> struct DynTraits {
  static constexpr bool forced = (DYN == DYN_FORCED_BGK || DYN == DYN_FORCED_SMAGORINSKY);
  static constexpr bool smagorinsky = (DYN == DYN_SMAGORINSKY || DYN == DYN_FORCED_SMAGORINSKY);
  static constexpr bool trt = (DYN == DYN_TRT);
};

// Density and velocity of a cell (forced dynamics: u = j/rho + F/2).
template <int Q, typename R, bool FORCED>
__device__ __forceinline__ void moments(const R (&f)[Q], const R* force, R& rho, R (&u)[3]) {
  using D = Desc<Q>;
  rho = R(0);
  static_for<Q>([&](auto I) { rho += f[I]; });
  rho += R(1);
  u[0] = u[1] = u[2] = R(0);
  static_for<Q>([&](auto I) {
    static_for<D::d>([&](auto A) {
      constexpr int c = D::C[I][A];
      if constexpr (c == 1) u[A] += f[I];
      else if constexpr (c == -1) u[A] -= f[I];
    });
  });
  if constexpr (sizeof(R) == 8) {
    static_for<D::d>([&](auto A) { u[A] /= rho; });  // FP64: the reference's exact division
  } else {
    const R inv = R(1) / rho;  // FP32 collision: one division, within the FP32 tolerance
    static_for<D::d>([&](auto A) { u[A] *= inv; });
  }
  if constexpr (FORCED) {
    static_for<D::d>([&](auto A) { u[A] += force[A] * R(0.5); });
  }
}

// c_i . u accumulated over the non-zero components in axis order (the reference loop adds
// c*u for every axis; the zero terms do not change the rounded sum).
template <int Q, int I, typename R>
__device__ __forceinline__ R c_dot(const R (&u)[3]) {
  using D = Desc<Q>;
  R cu = R(0);
  static_for<D::d>([&](auto A) {
    constexpr int c = D::C[I][A];
    if constexpr (c == 1) cu += u[A];
    else if constexpr (c == -1) cu -= u[A];
  });
  return cu;
}

// f_i^eq - w_i (second order).  FP64 keeps the reference's operation sequence (no fused
// operations: the FP64 unit is built with -fmad=false); the float arithmetic of the FP32 and
// reduced-precision forms uses explicit fused multiply-adds.  Every unit is built without
// implicit contraction, so each kernel variant and launch shape rounds identically.
template <int Q, int I, typename R>
__device__ __forceinline__ R equilibrium(R rho, const R (&u)[3], R uSqr) {
  constexpr R t = weight<Q, R>(I);
  const R cu = c_dot<Q, I>(u);
  if constexpr (sizeof(R) == 8) {
    return rho * t * (R(1) + R(3) * cu + R(4.5) * cu * cu - R(1.5) * uSqr) - t;
  } else {
    const R e = __fmaf_rn(R(4.5) * cu, cu, __fmaf_rn(R(3), cu, R(1) - R(1.5) * uSqr));
    return __fmaf_rn(rho * t, e, -t);
  }
}

// Effective relaxation frequency of the Smagorinsky model.
template <int Q, typename R, bool FORCED>
__device__ __forceinline__ R smagorinsky_omega(const R (&f)[Q], R rho, const R (&u)[3],
                                               const CollisionParams<R>& p) {
  using D = Desc<Q>;
  R us[3] = {u[0], u[1], u[2]};
  if constexpr (FORCED) {
    static_for<D::d>([&](auto A) { us[A] = u[A] - R(0.5) * p.force[A]; });
  }
  R pi[6];
  static_for<D::d>([&](auto A) {
    static_for<D::d>([&](auto B) {
      if constexpr (B >= A) {
        R s = R(0);
        static_for<Q>([&](auto I) {
          constexpr int cab = D::C[I][A] * D::C[I][B];
          if constexpr (cab == 1) s += f[I];
          else if constexpr (cab == -1) s -= f[I];
        });
        s -= rho * us[A] * us[B];
        if constexpr (A == B) s -= R(1) / R(3) * (rho - R(1));
        if constexpr (FORCED) {
          s += R(0.5) * rho * (p.force[A] * us[B] + us[A] * p.force[B]);
        }
        // (xx, xy, xz, yy, yz, zz) in 3D, (xx, xy, yy) in 2D
        constexpr int ip = A * D::d - (A * (A - 1)) / 2 + (B - A);
        pi[ip] = s;
      }
    });
  });
  R n2 = pi[0] * pi[0] + R(2) * pi[1] * pi[1] + pi[2] * pi[2];
  if constexpr (D::d == 3) {
    n2 += pi[2] * pi[2] + pi[3] * pi[3] + R(2) * pi[4] * pi[4] + pi[5] * pi[5];
  }
  const R cs = p.smagorinsky;
  const R piNeqNorm = sqrt(n2);
  const R pre = cs * cs * R(3) * R(3) * R(2) * R(1.4142135623730951);
  const R tauMol = R(1) / p.omega;
  const R tauTurb = R(0.5) * (sqrt(tauMol * tauMol + pre / rho * piNeqNorm) - tauMol);
  return R(1) / (tauMol + tauTurb);
}

// Collide one cell in place.  Returns the cell statistic {rho, |u|^2}.
template <int Q, typename R, int DYN>
__device__ __forceinline__ void collide(R (&f)[Q], const CollisionParams<R>& p, R& rhoOut, R& uSqrOut) {
  using D = Desc<Q>;
  using T = DynTraits<DYN>;
  R rho, u[3];
  moments<Q, R, T::forced>(f, p.force, rho, u);
  R uSqr = R(0);
  static_for<D::d>([&](auto A) { uSqr += u[A] * u[A]; });

  R omega = p.omega;
  if constexpr (T::smagorinsky) omega = smagorinsky_omega<Q, R, T::forced>(f, rho, u, p);

  if constexpr (T::trt) {
    const R omega2 = R(1) / (p.magic / (R(1) / omega - R(0.5)) + R(0.5));
    // pairs (i, opp(i)) for i = 1 .. q/2, plus the rest population
    {
      const R feq0 = equilibrium<Q, 0>(rho, u, uSqr);
      const R fp = R(0.5) * (f[0] + f[0]);
      const R fm = R(0.5) * (f[0] - f[0]);
      const R ep = R(0.5) * (feq0 + feq0);
      const R em = R(0.5) * (feq0 - feq0);
      f[0] -= omega * (fp - ep) + omega2 * (fm - em);
    }
    static_for<Q / 2>([&](auto K) {
      constexpr int i = K + 1;
      constexpr int j = D::OPP[i];
      const R ei = equilibrium<Q, i>(rho, u, uSqr);
      const R ej = equilibrium<Q, j>(rho, u, uSqr);
      const R fi = f[i], fj = f[j];
      const R fpi = R(0.5) * (fi + fj), fmi = R(0.5) * (fi - fj);
      const R fpj = R(0.5) * (fj + fi), fmj = R(0.5) * (fj - fi);
      const R epi = R(0.5) * (ei + ej), emi = R(0.5) * (ei - ej);
      const R epj = R(0.5) * (ej + ei), emj = R(0.5) * (ej - ei);
      f[i] = fi - (omega * (fpi - epi) + omega2 * (fmi - emi));
      f[j] = fj - (omega * (fpj - epj) + omega2 * (fmj - emj));
    });
  } else if constexpr (sizeof(R) == 8) {
    const R keep = R(1) - omega;
    static_for<Q>([&](auto I) {
      const R feq = equilibrium<Q, I>(rho, u, uSqr);
      f[I] *= keep;
      f[I] += omega * feq;
    });
  } else {
    // float: opposite directions share t_i and |c_i . u|, so their equilibria are
    // sym +- asym with sym = rho t (1 - 1.5 u^2 + 4.5 (c.u)^2) - t and asym = 3 rho t (c.u)
    const R keep = R(1) - omega;
    const R base = R(1) - R(1.5) * uSqr;
    {
      constexpr R t0 = weight<Q, R>(0);
      f[0] = __fmaf_rn(omega, __fmaf_rn(rho * t0, base, -t0), f[0] * keep);
    }
    static_for<Q / 2>([&](auto K) {
      constexpr int i = K + 1;
      constexpr int j = D::OPP[i];
      constexpr R t = weight<Q, R>(i);
      const R cu = c_dot<Q, i>(u);
      const R rt = rho * t;
      const R sym = __fmaf_rn(rt, __fmaf_rn(R(4.5) * cu, cu, base), -t);
      const R asym = (rho * R(3 * t)) * cu;
      f[i] = __fmaf_rn(omega, sym + asym, f[i] * keep);
      f[j] = __fmaf_rn(omega, sym - asym, f[j] * keep);
    });
  }

  if constexpr (T::forced) {
    const R om = rho * (R(1) - omega * R(0.5));
    static_for<Q>([&](auto I) {
      constexpr R t = weight<Q, R>(I);
      const R cu = c_dot<Q, I>(u) * R(9);
      R ft = R(0);
      static_for<D::d>([&](auto A) {
        constexpr int c = D::C[I][A];
        ft += ((R(c) - u[A]) * R(3) + cu * R(c)) * p.force[A];
      });
      ft *= om * t;
      f[I] += ft;
    });
  }
  rhoOut = rho;
  uSqrOut = uSqr;
}

template <int Q, typename R>
__device__ __forceinline__ void revert(R (&f)[Q]) {
  using D = Desc<Q>;
  static_for<Q / 2>([&](auto K) {
    constexpr int i = K + 1;
    constexpr int j = D::OPP[i];
    const R a = f[i];
    f[i] = f[j];
    f[j] = a;
  });
}

}  // namespace lbx
