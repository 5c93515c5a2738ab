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
//   ConstRhoBGK      collision::ConstRhoBGK::apply            src/dynamics/collision.h:322-351
#pragma once

#include "lbx_desc.cuh"

namespace lbx {

enum Dyn : int {
  DYN_BGK = 1,
  DYN_TRT = 2,
  DYN_SMAGORINSKY = 3,
  DYN_FORCED_BGK = 4,
  DYN_FORCED_SMAGORINSKY = 5,
  DYN_CONST_RHO = 6
};

// Statistics accumulator: {sum rho, sum |u|^2} in FP64, {count, max |u|^2 bits}.
struct StatAcc {
  double sum[2];
  unsigned long long count;
  unsigned long long maxbits;
};

template <typename R>
struct CollisionParams {
  R omega;
  R magic;
  R smagorinsky;
  R force[3];
  // ConstRhoBGK: the statistics of the previous step, whose average density is the
  // AVERAGE_RHO parameter (1 while no step has been counted)
  const StatAcc* avgSrc;
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
// FP32 BGK, written so that no product is ever an operand of a separate add: the sums of the
// populations and of the momentum are plain adds, every product that meets an add does so inside
// an explicit fused multiply-add.  The packed two-cell form (collide_bgk_x2) repeats this
// sequence lane by lane, and since nothing here is left for the compiler to contract, the
// two give the same bits.
template <int Q>
__device__ __forceinline__ void collide_bgk_f32(float (&f)[Q], float omega, float& rhoOut, float& uSqrOut) {
  using D = Desc<Q>;
  float rho = 0.f;
  static_for<Q>([&](auto I) { rho = __fadd_rn(rho, f[I]); });
  rho = __fadd_rn(rho, 1.f);
  float j[3] = {0.f, 0.f, 0.f};
  static_for<Q>([&](auto I) {
    static_for<D::d>([&](auto A) {
      constexpr int c = D::C[I][A];
      if constexpr (c == 1) j[A] = __fadd_rn(j[A], f[I]);
      else if constexpr (c == -1) j[A] = __fsub_rn(j[A], f[I]);
    });
  });
  const float inv = 1.f / rho;
  float u[3];
  static_for<D::d>([&](auto A) { u[A] = __fmul_rn(j[A], inv); });
  float uSqr = __fmul_rn(u[0], u[0]);
  static_for<D::d - 1>([&](auto A) { uSqr = __fmaf_rn(u[A + 1], u[A + 1], uSqr); });
  const float keep = 1.f - omega;
  const float base = __fmaf_rn(-1.5f, uSqr, 1.f);
  {
    constexpr float t0 = weight<Q, float>(0);
    f[0] = __fmaf_rn(omega, __fmaf_rn(__fmul_rn(rho, t0), base, -t0), __fmul_rn(f[0], keep));
  }
  static_for<Q / 2>([&](auto K) {
    constexpr int i = K + 1;
    constexpr int jj = D::OPP[i];
    constexpr float t = weight<Q, float>(i);
    float cj = 0.f;  // c_i . j over the non-zero components in axis order
    static_for<D::d>([&](auto A) {
      constexpr int c = D::C[i][A];
      if constexpr (c == 1) cj = __fadd_rn(cj, j[A]);
      else if constexpr (c == -1) cj = __fsub_rn(cj, j[A]);
    });
    const float cu = __fmul_rn(cj, inv);
    const float sym = __fmaf_rn(__fmul_rn(rho, t), __fmaf_rn(__fmul_rn(4.5f, cu), cu, base), -t);
    const float r3t = __fmul_rn(rho, 3 * t);
    const float plus = __fmaf_rn(r3t, cu, sym), minus = __fmaf_rn(-r3t, cu, sym);
    f[i] = __fmaf_rn(omega, plus, __fmul_rn(f[i], keep));
    f[jj] = __fmaf_rn(omega, minus, __fmul_rn(f[jj], keep));
  });
  rhoOut = rho;
  uSqrOut = uSqr;
}

template <int Q, typename R, int DYN>
__device__ __forceinline__ void collide(R (&f)[Q], const CollisionParams<R>& p, R& rhoOut, R& uSqrOut) {
  using D = Desc<Q>;
  using T = DynTraits<DYN>;
  if constexpr (DYN == DYN_BGK && sizeof(R) == 4) {
    collide_bgk_f32<Q>(f, p.omega, rhoOut, uSqrOut);
    return;
  }
  R rho, u[3];
  moments<Q, R, T::forced>(f, p.force, rho, u);
  R uSqr = R(0);
  static_for<D::d>([&](auto A) { uSqr += u[A] * u[A]; });

  R omega = p.omega;
  if constexpr (T::smagorinsky) omega = smagorinsky_omega<Q, R, T::forced>(f, rho, u, p);

  if constexpr (DYN == DYN_CONST_RHO) {
    // collision::ConstRhoBGK::apply (src/dynamics/collision.h:336-349): the equilibrium part
    // is rescaled by 1 + (1 - <rho>) / rho, which pulls the lattice's average density back to
    // 1; the cell reports rho + (1 - <rho>) to the statistics.
    double avg = 1.0;
    if (p.avgSrc) {
      const unsigned long long cnt = p.avgSrc->count;
      if (cnt) avg = p.avgSrc->sum[0] / double(cnt);
    }
    const R deltaRho = R(1) - R(avg);
    const R ratioRho = R(1) + deltaRho / rho;
    const R keep = R(1) - omega;
    static_for<Q>([&](auto I) {
      constexpr R t = weight<Q, R>(I);
      const R feq = equilibrium<Q, I>(rho, u, uSqr);
      if constexpr (sizeof(R) == 8) f[I] = ratioRho * (feq + t) - t + keep * (f[I] - feq);
      else f[I] = __fmaf_rn(keep, f[I] - feq, __fmaf_rn(ratioRho, feq + t, -t));
    });
    rhoOut = rho + deltaRho;
    uSqrOut = uSqr;
    return;
  }

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

// ---- two cells at once: packed FP32 pairs (sm_100 f32x2 arithmetic) ------------------------
// Each packed operation rounds every lane exactly as the scalar operation does, so a pair of
// cells computed here gets the same bits as two calls of the scalar float path below: the
// operation sequence of collide<Q, float, DYN_BGK> is kept step for step.
// The pairs are CUDA's float2 and the operations its sm_100 packed intrinsics, whose rounding per
// component is that of __fadd_rn, __fmul_rn and __fmaf_rn; the compiler keeps a pair in a
// register pair instead of packing two floats around every operation.
using F2 = float2;
__device__ __forceinline__ F2 f2(float v) { return make_float2(v, v); }
__device__ __forceinline__ F2 add2(F2 a, F2 b) { return __fadd2_rn(a, b); }
// a - b with one rounding, as __fsub_rn: b * (-1) is exact, so the fused form rounds a + (-b) once
__device__ __forceinline__ F2 sub2(F2 a, F2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ F2 mul2(F2 a, F2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ F2 fma2(F2 a, F2 b, F2 c) { return __ffma2_rn(a, b, c); }

// BGK collision of two cells (f[k][i], k = 0, 1) in place: collide_bgk_f32 on pairs, the same
// operation sequence (no product ever meets a separate add, so no contraction can differ).
template <int Q>
__device__ __forceinline__ void collide_bgk_x2(float (&f)[2][Q], float omega, float (&rhoOut)[2], float (&usqOut)[2]) {
  using D = Desc<Q>;
  F2 g[Q];
  static_for<Q>([&](auto I) { g[I] = F2{f[0][I], f[1][I]}; });
  F2 rho = f2(0.f);
  static_for<Q>([&](auto I) { rho = add2(rho, g[I]); });
  rho = add2(rho, f2(1.f));
  F2 j[3] = {f2(0.f), f2(0.f), f2(0.f)};
  static_for<Q>([&](auto I) {
    static_for<D::d>([&](auto A) {
      constexpr int c = D::C[I][A];
      if constexpr (c == 1) j[A] = add2(j[A], g[I]);
      else if constexpr (c == -1) j[A] = sub2(j[A], g[I]);
    });
  });
  const F2 inv{1.f / rho.x, 1.f / rho.y};
  F2 u[3];
  static_for<D::d>([&](auto A) { u[A] = mul2(j[A], inv); });
  F2 uSqr = mul2(u[0], u[0]);
  static_for<D::d - 1>([&](auto A) { uSqr = fma2(u[A + 1], u[A + 1], uSqr); });
  const F2 w = f2(omega);
  const F2 keep = f2(1.f - omega);
  const F2 base = fma2(f2(-1.5f), uSqr, f2(1.f));
  {
    constexpr float t0 = weight<Q, float>(0);
    g[0] = fma2(w, fma2(mul2(rho, f2(t0)), base, f2(-t0)), mul2(g[0], keep));
  }
  static_for<Q / 2>([&](auto K) {
    constexpr int i = K + 1;
    constexpr int jj = D::OPP[i];
    constexpr float t = weight<Q, float>(i);
    F2 cj = f2(0.f);
    static_for<D::d>([&](auto A) {
      constexpr int c = D::C[i][A];
      if constexpr (c == 1) cj = add2(cj, j[A]);
      else if constexpr (c == -1) cj = sub2(cj, j[A]);
    });
    const F2 cu = mul2(cj, inv);
    const F2 sym = fma2(mul2(rho, f2(t)), fma2(mul2(f2(4.5f), cu), cu, base), f2(-t));
    const F2 r3t = mul2(rho, f2(3 * t));
    const F2 plus = fma2(r3t, cu, sym), minus = fma2(F2{-r3t.x, -r3t.y}, cu, sym);
    g[i] = fma2(w, plus, mul2(g[i], keep));
    g[jj] = fma2(w, minus, mul2(g[jj], keep));
  });
  static_for<Q>([&](auto I) {
    f[0][I] = g[I].x;
    f[1][I] = g[I].y;
  });
  rhoOut[0] = rho.x;
  rhoOut[1] = rho.y;
  usqOut[0] = uSqr.x;
  usqOut[1] = uSqr.y;
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
