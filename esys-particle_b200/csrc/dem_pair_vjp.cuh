// Hand-written reverse (vector-Jacobian product) of the two dynamic pair laws, for the
// differentiable window's reverse sweep:
//   CElasticInteraction::calcForces        (Model/ElasticInteraction.cpp:54-71)
//   CRotFrictionInteraction::calcSimpleForces (Model/RotFricInteraction.cpp:171-231)
// Each function recomputes the law's forward values in FP64 in the law's operation order
// (so every branch -- touching, stick / slip -- is the one the forward took on the same
// state) and then runs the chain rule backwards, step for step.  Inputs are the adjoints of
// the law's outputs as the particles receive them; outputs are the adjoints of the law's
// inputs, including the scaled stiffnesses (the caller multiplies by the scaling factor).
#pragma once
#include "dem_laws.cuh"

namespace dem {

// d/dx l.(a x b) = b x l for a, and l x a for b.
__device__ __forceinline__ V cross_vjp_a(const V& b, const V& l) { return cross(b, l); }
__device__ __forceinline__ V cross_vjp_b(const V& a, const V& l) { return cross(l, a); }

struct ElasticVjp {
  V x1, x2;
  double k_eff;
  bool touching;
};

// F = D k_eff (|D| - r0) / |D| applied to p2 (p1 gets -F); aF = lambda_F2 - lambda_F1.
__device__ __forceinline__ void law_elastic_vjp(double k_eff, const V& x1, double r1, const V& x2, double r2,
                                                const V& aF, ElasticVjp& g) {
  const V D = x1 - x2;
  const double d2 = dot(D, D);
  const double r0 = r1 + r2;
  g.x1 = g.x2 = mk(0.0, 0.0, 0.0);
  g.k_eff = 0.0;
  g.touching = d2 < r0 * r0;
  if (!g.touching) return;
  const double dist = sqrt(d2);
  const double s = k_eff * (dist - r0) / dist;
  const double aFD = dot(aF, D);
  // s = k_eff (1 - r0 / dist): ds/dk_eff = (dist - r0) / dist, ds/ddist = k_eff r0 / dist^2
  g.k_eff = aFD * (dist - r0) / dist;
  const double a_dist = aFD * k_eff * r0 / (dist * dist);
  const V aD = s * aF + (a_dist / dist) * D;
  g.x1 = aD;
  g.x2 = -aD;
}

struct FricVjp {
  V x1, x2, v1, v2, w1, w2, H;
  double k_eff, ks_eff;
  bool touching;
};

// Adjoints in: a_fn of the normal force applied to p2 (p1 gets -fn): lambda_F2 - lambda_F1;
// a_Ff of the tangential force / next history (p1 gets +Ff, p2 gets -Ff): lambda_F1 -
// lambda_F2 + lambda_H; lM1, lM2 of the moments.
__device__ __forceinline__ void law_friction_vjp(double k_eff, double ks_eff, double mu_s, double mu_d, double dt,
                                                 const V& x1, double r1, const V& v1, const V& w1, const V& x2,
                                                 double r2, const V& v2, const V& w2, const V& H, bool slipping,
                                                 const V& a_fn, const V& a_Ff0, const V& lM1, const V& lM2,
                                                 FricVjp& g) {
  const V z = mk(0.0, 0.0, 0.0);
  g.x1 = g.x2 = g.v1 = g.v2 = g.w1 = g.w2 = g.H = z;
  g.k_eff = g.ks_eff = 0.0;
  const double mu_current = slipping ? mu_d : mu_s;
  const V D = x1 - x2;
  const double d2 = dot(D, D);
  const double eq = r1 + r2;
  g.touching = d2 < eq * eq;
  if (!g.touching) return;  // the history resets: nothing flows back
  // forward, in the law's order
  const double dist = sqrt(d2);
  const double s = k_eff * (dist - eq) / dist;
  const V force = D * s;
  const double c = r2 / eq;
  const V pos = x2 + c * D;
  const V arm1 = pos - x1, arm2 = pos - x2;
  const V vp1 = v1 + cross(w1, arm1);
  const V vp2 = v2 + cross(w2, arm2);
  const V u = (vp2 - vp1) * dt;
  const double p = dot(u, D), q = norm2(D);
  const double t = p / q;
  const V ds = u - t * D;
  const V Fp = H + ks_eff * ds;
  const double FpN = norm(Fp);
  const double fN = norm(force);
  const bool slip = FpN > fN * mu_current;
  const double gsc = slip ? (mu_d * fN) / FpN : 1.0;
  const V Ff = slip ? Fp * gsc : Fp;
  // reverse
  // M1 = arm1 x Ff, M2 = arm2 x (-Ff)
  V a_arm1 = cross_vjp_a(Ff, lM1);
  V a_arm2 = -cross_vjp_a(Ff, lM2);
  const V a_Ff = a_Ff0 + cross_vjp_b(arm1, lM1) - cross_vjp_b(arm2, lM2);
  V a_force = a_fn;
  V a_Fp = a_Ff;
  if (slip) {  // Ff = Fp mu_d fN / |Fp|
    const double aFFp = dot(a_Ff, Fp);
    a_Fp = gsc * a_Ff - (mu_d * fN * aFFp / (FpN * FpN * FpN)) * Fp;
    const double a_fN = mu_d * aFFp / FpN;
    a_force = a_force + (a_fN / fN) * force;
  }
  // Fp = H + ks_eff ds
  g.H = a_Fp;
  g.ks_eff = dot(a_Fp, ds);
  const V a_ds = ks_eff * a_Fp;
  // ds = u - (u.D / D.D) D
  const double aDs = dot(a_ds, D);
  const V a_u = a_ds - (aDs / q) * D;
  V aD = -t * a_ds - aDs * (u / q - (2.0 * p / (q * q)) * D);
  // u = (vp2 - vp1) dt
  const V a_vp2 = dt * a_u, a_vp1 = -dt * a_u;
  g.v1 = a_vp1;
  g.v2 = a_vp2;
  g.w1 = cross_vjp_a(arm1, a_vp1);
  g.w2 = cross_vjp_a(arm2, a_vp2);
  a_arm1 = a_arm1 + cross_vjp_b(w1, a_vp1);
  a_arm2 = a_arm2 + cross_vjp_b(w2, a_vp2);
  // arm1 = pos - x1, arm2 = pos - x2, pos = x2 + c D
  const V a_pos = a_arm1 + a_arm2;
  V ax1 = -a_arm1;
  V ax2 = a_pos - a_arm2;
  aD = aD + c * a_pos;
  // force = D s, s = k_eff (dist - eq) / dist
  const double a_s = dot(a_force, D);
  aD = aD + s * a_force;
  g.k_eff = a_s * (dist - eq) / dist;
  const double a_dist = a_s * k_eff * eq / (dist * dist);
  aD = aD + (a_dist / dist) * D;
  // D = x1 - x2
  g.x1 = ax1 + aD;
  g.x2 = ax2 - aD;
}

}  // namespace dem
