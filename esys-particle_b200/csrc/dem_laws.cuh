// Per-pair and per-particle force laws of the DEM step, FP64.
//
// Each law is evaluated in the canonical orientation (p1 = lower particle id,
// p2 = higher), with p2's position already replaced by its periodic image
// nearest p1.  A particle-centric kernel evaluates every pair from both
// sides; both sides call the same function on the same inputs, so both get
// bit-identical results and the pair's contributions cancel exactly.
#pragma once
#include "dem_math.cuh"

namespace dem {

using V = V3<double>;
using Qd = Quat<double>;

// CElasticInteraction ctor scaling (Model/ElasticInteraction.cpp:25-49).
template <class S>
__device__ __forceinline__ S elastic_k_t(S k, int scaling, double r1, double r2) {
  double effR = 1.0, effA = 1.0, effL = 1.0;
  double r0 = r1 + r2;
  if (scaling) { effR = 0.5 * r0; effL = r0; effA = effR * effR; }
  return k * effA / effL;
}
__device__ __forceinline__ double elastic_k(double k, int scaling, double r1, double r2) {
  return elastic_k_t<double>(k, scaling, r1, r2);
}

// CElasticInteraction::calcForces (Model/ElasticInteraction.cpp:54-71).
// Returns true when touching; F is the force applied to p2 (p1 gets -F).
template <class S>
__device__ __forceinline__ bool law_elastic_t(S k_eff, const V3<S>& x1, double r1, const V3<S>& x2, double r2,
                                              V3<S>& F) {
  V3<S> D = x1 - x2;
  S dist = dot(D, D);
  double eq_dist = r1 + r2;
  if (dist < (eq_dist * eq_dist)) {
    dist = sqrt(dist);
    F = D * (k_eff * (dist - eq_dist) / dist);
    return true;
  }
  return false;
}
__device__ __forceinline__ bool law_elastic(double k_eff, const V& x1, double r1, const V& x2, double r2, V& F) {
  return law_elastic_t<double>(k_eff, x1, r1, x2, r2, F);
}

// CRotFrictionInteraction ctor scaling (Model/RotFricInteraction.cpp:103-146).
template <class S>
__device__ __forceinline__ void friction_k_t(S k, S ks, int scaling, int meanR, double r1, double r2, S& k_eff,
                                             S& ks_eff) {
  double effR = 1.0, effL = 1.0, effA = 1.0;
  double r0 = r1 + r2;
  if (scaling) {
    if (meanR) effR = 0.5 * r0; else effR = fmin(r1, r2);
    effL = r0;
    effA = effR * effR;
  }
  k_eff = k * effA / effL;
  ks_eff = ks * effA / effL;
}
__device__ __forceinline__ void friction_k(double k, double ks, int scaling, int meanR, double r1, double r2,
                                           double& k_eff, double& ks_eff) {
  friction_k_t<double>(k, ks, scaling, meanR, r1, r2, k_eff, ks_eff);
}

template <class S>
struct FricOutT {
  V3<S> fn;     // normal force applied to p2 (p1 gets -fn)
  V3<S> Ffric;  // tangential force after the update (p1 gets +Ffric, p2 gets -Ffric)
  V3<S> M1, M2; // moments on p1, p2
  bool touching, slipping;
};
using FricOut = FricOutT<double>;

// CRotFrictionInteraction::calcSimpleForces (Model/RotFricInteraction.cpp:171-231).
template <class S>
__device__ __forceinline__ void law_friction_t(S k_eff, S ks_eff, double mu_s, double mu_d, double dt,
                                               const V3<S>& x1, double r1, const V3<S>& v1, const V3<S>& w1,
                                               const V3<S>& x2, double r2, const V3<S>& v2, const V3<S>& w2,
                                               V3<S> Ffric, bool slipping, FricOutT<S>& o) {
  using VS = V3<S>;
  double mu_current = slipping ? mu_d : mu_s;
  const VS D = x1 - x2;
  S dist = dot(D, D);
  const double eq_dist = r1 + r2;
  if (dist < (eq_dist * eq_dist)) {
    dist = sqrt(dist);
    const VS force = D * (k_eff * (dist - eq_dist) / dist);
    const VS pos = x2 + (r2 / eq_dist) * D;
    const VS vp1 = v1 + cross(w1, pos - x1);
    const VS vp2 = v2 + cross(w2, pos - x2);
    VS ds = (vp2 - vp1) * dt;
    ds -= ((dot(ds, D)) / (norm2(D))) * D;
    Ffric += ks_eff * ds;
    const S FfricNorm = norm(Ffric);
    const S forceNorm = norm(force);
    if (FfricNorm > forceNorm * mu_current) {
      Ffric = Ffric * ((mu_d * forceNorm) / FfricNorm);
      o.slipping = true;
    } else {
      o.slipping = false;
    }
    o.M1 = cross(pos - x1, Ffric);
    o.M2 = cross(pos - x2, -Ffric);
    o.fn = force;
    o.Ffric = Ffric;
    o.touching = true;
  } else {
    o.Ffric = mk(S(0.0), S(0.0), S(0.0));
    o.fn = o.Ffric;
    o.M1 = o.M2 = o.Ffric;
    o.slipping = false;
    o.touching = false;
  }
}
__device__ __forceinline__ void law_friction(double k_eff, double ks_eff, double mu_s, double mu_d, double dt,
                                             const V& x1, double r1, const V& v1, const V& w1, const V& x2, double r2,
                                             const V& v2, const V& w2, V Ffric, bool slipping, FricOut& o) {
  law_friction_t<double>(k_eff, ks_eff, mu_s, mu_d, dt, x1, r1, v1, w1, x2, r2, v2, w2, Ffric, slipping, o);
}

// CBondedInteraction (NRotBond): constructor scaling (Model/BondedInteraction.cpp:43-69) and
// calcForces (:126-140).  The rest length is r1 + r2; F is applied to p2, -F to p1 (no moments:
// CParticle::applyForce adds the force only, Model/Particle.cpp:391-400).
__device__ __forceinline__ double nbond_k(double k, int scaling, double r1, double r2) {
  double effR = 1.0, effA = 1.0, effL = 1.0;
  const double r0 = r1 + r2;
  if (scaling) {
    effR = 0.5 * r0;
    effL = r0;
    effA = effR * effR;
  }
  return k * effA / effL;
}
__device__ __forceinline__ void law_nbond(double k_eff, const V& x1, double r1, const V& x2, double r2, V& F,
                                          double& dist) {
  const V D = x1 - x2;
  const double r0 = r1 + r2;
  dist = sqrt(dot(D, D));
  F = D * (k_eff * (dist - r0) / dist);
}
// CBondedInteraction::broken (:101-114): extension beyond r0 * rbreak; rbreak < 0 marks the group
// unbreakable (ParallelInteractionStorage_EB::setUnbreakable, SubLattice.hpp:1818-1821).
__device__ __forceinline__ bool nbond_broken(double dist, double r1, double r2, double rbreak) {
  const double r0 = r1 + r2;
  return rbreak >= 0.0 && (dist - r0) > r0 * rbreak;
}

// CFrictionInteraction (NRotFriction): constructor scaling (Model/FrictionInteraction.cpp:57-75)
// and calcForces (:93-149): an elastic normal force and a tangential force from the relative
// translation only, one friction coefficient; forces only (no moments).
__device__ __forceinline__ void nfriction_k(double k, double ks, int scaling, double r1, double r2, double& k_eff,
                                            double& ks_eff) {
  double f = 1.0;
  if (scaling) f = 0.5 * (r1 + r2);
  k_eff = f * k;
  ks_eff = f * ks;
}
__device__ __forceinline__ void law_nfriction(double k_eff, double ks_eff, double mu, double dt, const V& x1, double r1,
                                              const V& v1, const V& x2, double r2, const V& v2, V Ffric,
                                              FricOut& o) {
  const V D = x1 - x2;
  const double eq_dist = r1 + r2;
  double dist = dot(D, D);
  if (dist < (eq_dist * eq_dist)) {
    dist = sqrt(dist);
    const V force = D * (k_eff * (dist - eq_dist) / dist);
    const V d1 = v1 * dt;
    const V d2 = v2 * dt;
    V ds = d2 - d1;
    ds -= ((dot(ds, D)) / (norm2(D))) * D;
    Ffric += ks_eff * ds;
    const double FfricNorm = norm(Ffric);
    const double forceNorm = norm(force);
    if (FfricNorm > forceNorm * mu) {
      Ffric = Ffric * ((mu * forceNorm) / FfricNorm);
      o.slipping = true;
    } else {
      o.slipping = false;
    }
    o.fn = force;
    o.Ffric = Ffric;
    o.M1 = o.M2 = mk(0.0, 0.0, 0.0);
    o.touching = true;
  } else {
    o.Ffric = o.fn = o.M1 = o.M2 = mk(0.0, 0.0, 0.0);
    o.slipping = false;
    o.touching = false;
  }
}

// CRotFrictionInteraction::isPersistent (Model/RotFricInteraction.cpp:345-351).
__device__ __forceinline__ bool friction_persistent(const V& x1, double r1, const V& x2, double r2) {
  V D = x1 - x2;
  double dist = dot(D, D);
  double eq_dist = r1 + r2;
  return dist <= (eq_dist * eq_dist);
}

// Scaled RotBond constants (ARotBondedInteraction.cpp:141-180 overridden by
// CRotBondedInteraction ctor, Model/RotBondedInteraction.cpp:122-161).  dist0 is
// |m_D|, the particle distance when the bond was created.
template <class S>
struct BondKT {
  S kr, ks, kb, kt;
  double max_n, max_s, max_b, max_t;
};
using BondK = BondKT<double>;
template <class S>
__device__ __forceinline__ BondKT<S> bond_k_t(S kr, S ks, S kt, S kb, double mn, double ms, double mt, double mb,
                                              int scaling, int meanR, double dist0, double r1, double r2) {
  double effR = 1.0, effL = 1.0, effA = 1.0, J = 1.0, I = 1.0;
  if (scaling) {
    if (meanR) effR = 0.5 * dist0; else effR = fmin(r1, r2);
    effL = dist0;
    effA = effR * effR;
    J = 0.5 * effR * effR * effR * effR;
    I = 0.5 * J;
  }
  BondKT<S> b;
  b.kr = kr * effA / effL;
  b.ks = ks * effA / effL;
  b.kb = kb * I / effL;
  b.kt = kt * J / effL;
  b.max_n = mn * effA;
  b.max_s = ms * effA;
  b.max_b = mb * I / effR;
  b.max_t = mt * J / effR;
  return b;
}
__device__ __forceinline__ BondK bond_k(double kr, double ks, double kt, double kb, double mn, double ms, double mt,
                                        double mb, int scaling, int meanR, double dist0, double r1, double r2) {
  return bond_k_t<double>(kr, ks, kt, kb, mn, ms, mt, mb, scaling, meanR, dist0, r1, r2);
}

// calc_angle (Model/ARotBondedInteraction.cpp:22-51).
template <class S>
__device__ __forceinline__ S calc_angle(const S& s_in, const S& c_os) {
  if (s_in > 0.0) return (c_os >= 1.0 || c_os <= -1.0) ? S(0.0) : acos(c_os);
  if (s_in == 0.0) return S(0.0);
  return (c_os >= 1.0 || c_os <= -1.0) ? S(0.0) : -acos(c_os);
}

template <class S>
struct BondOutT {
  V3<S> force;    // applied to p1 (p2 gets -force)
  V3<S> moment1;  // applied to p1
  V3<S> moment2;  // applied to p2
  S nF, shF, tM, bM;
};
using BondOut = BondOutT<double>;

// ARotBondedInteraction::calcForces (Model/ARotBondedInteraction.cpp:307-448).
// Templated on the scalar S: S = double for the step kernels, a forward-mode
// dual number for the adjoint (dem_adjoint.cu).
template <class S>
__device__ __forceinline__ void law_bond_t(const BondKT<S>& K, const V3<S>& m_D, const V3<S>& x1, double r1,
                                           const Quat<S>& q1, const V3<S>& x2, double r2, const Quat<S>& q2,
                                           BondOutT<S>& o) {
  using VS = V3<S>;
  using QS = Quat<S>;
  const double HALF_SQRT_2 = 0.5 * sqrt(2.0);
  S s_fai = 0.0, c_fai = 0.0, c_pasi2 = 0.0, s_pasi2 = 0.0, sita = 0.0, pasi = 0.0;
  const M3<S> mat0 = to_matrix(q1);
  const VS rbp = x2 - x1;
  const S rbpNorm = norm(rbp);
  const VS rb = mul(mat0, x2 - x1);
  const S rbNorm = norm(rb);
  const double r_0Norm = r1 + r2;
  const VS delta_r = (rbNorm - r_0Norm) * rb / rbNorm;
  const VS Fr = K.kr * delta_r;
  const S gama_cos = dot(rb, m_D) / (rbNorm * norm(m_D));
  S gama = 0.0;
  if (gama_cos < 1.0 && gama_cos > -1.0) gama = acos(gama_cos);
  const VS rb_0 = cross(rb, m_D);
  const VS rb_b0 = cross(rb, rb_0);
  const S rb_b0Norm = norm(rb_b0);
  VS Fst = mk(S(0.0), S(0.0), S(0.0));
  if (rb_b0Norm != 0) Fst = K.ks * r_0Norm * gama * rb_b0 / rb_b0Norm;
  VS Mst = mk(S(0.0), S(0.0), S(0.0));
  const S rb_0Norm = norm(rb_0);
  if (rb_0Norm != 0) Mst = -norm(Fst) * rb_0 / rb_0Norm;
  const S m0 = HALF_SQRT_2 * sqrt((rbNorm + rb.z) / rbNorm);
  S m1 = -HALF_SQRT_2 * sqrt((rbNorm - rb.z) / rbNorm);
  S m2 = -m1;
  const S m3 = 0.0;
  const S rbX2PlusRbY2 = rb.x * rb.x + rb.y * rb.y;
  if (rbX2PlusRbY2 != 0.0) {
    const S denomSqrt = sqrt(rbX2PlusRbY2);
    m1 = m1 * rb.y / denomSqrt;
    m2 = m2 * rb.x / denomSqrt;
  }
  const QS qm{m0, mk(m1, m2, m3)};
  const M3<S> mat = to_matrix(qm);
  const QS rp = qmul(qinv(q1), q2);
  const QS r = qmul(qmul(qinv(qm), rp), qm);
  const S temp0 = r.s * r.s + r.v.z * r.v.z;
  if (temp0 == 0.0) {
    pasi = 0.0;
  } else {
    const S sqrtTemp0 = sqrt(temp0);
    c_pasi2 = r.s / sqrtTemp0;
    s_pasi2 = r.v.z / sqrtTemp0;
    pasi = 2.0 * calc_angle(s_pasi2, c_pasi2);
  }
  const VS Mtp = mk(S(0.0), S(0.0), K.kt * pasi);
  const VS Mtr = mulT(mat, Mtp);
  const S temp2 = r.v.x * r.v.x + r.v.y * r.v.y;
  const S temp3 = r.v.x * r.v.z + r.s * r.v.y;
  const S temp4 = r.v.y * r.v.z - r.s * r.v.x;
  VS Mbr = mk(S(0.0), S(0.0), S(0.0)), Fsr = Mbr, Msr = Mbr;
  if (temp2 != 0.0) {
    const S temp1 = temp0 - temp2;
    if (temp1 >= 1.0 || temp1 <= -1.0) sita = 0.0; else sita = acos(temp1);
    if (temp0 == 0.0) {
      const S sqrtDenom = sqrt(temp2);
      c_fai = r.v.y / sqrtDenom;
      s_fai = -r.v.x / sqrtDenom;
    } else {
      const S sqrtDenom = sqrt(temp0 * temp2);
      c_fai = temp3 / sqrtDenom;
      s_fai = temp4 / sqrtDenom;
    }
    const VS Mbp = mk(-0.5 * K.kb * sita * s_fai, 0.5 * K.kb * sita * c_fai, S(0.0));
    Mbr = mulT(mat, Mbp);
    const VS Fsp = mk(-0.5 * K.ks * c_fai * sita * r_0Norm, -0.5 * K.ks * s_fai * sita * r_0Norm, S(0.0));
    Fsr = mulT(mat, Fsp);
    const VS Msp = mk(0.5 * K.ks * s_fai * sita * r_0Norm, -0.5 * K.ks * c_fai * sita * r_0Norm, S(0.0));
    Msr = mulT(mat, Msp);
  }
  const double eq_rad1 = r1 / (r1 + r2);
  const double eq_rad2 = r2 / (r1 + r2);
  o.force = mulT(mat0, Fr + Fst + Fsr);
  o.moment1 = mulT(mat0, Mbr + Mtr + Msr * eq_rad1 * rbpNorm + Mst * eq_rad1 * rbpNorm);
  o.moment2 = mulT(mat0, Msr * eq_rad2 * rbpNorm + Mst * eq_rad2 * rbpNorm - Mbr - Mtr);
  o.shF = norm(Fst + Fsr);
  o.tM = norm(Mtr);
  o.bM = norm(Mbr);
  const double r0 = r1 + r2;
  const VS D = x1 - x2;
  const S dist = sqrt(dot(D, D));
  o.nF = ((dist < r0) ? -1.0 : 1.0) * norm(Fr);
}

__device__ __forceinline__ void law_bond(const BondK& K, const V& m_D, const V& x1, double r1, const Qd& q1,
                                         const V& x2, double r2, const Qd& q2, BondOut& o) {
  law_bond_t<double>(K, m_D, x1, r1, q1, x2, r2, q2, o);
}

// CRotBondedInteraction::broken (Model/RotBondedInteraction.cpp:175-219), beta1 = beta2 = 1.
__device__ __forceinline__ bool bond_broken(const BondK& K, const BondOut& o, double truncated) {
  const double beta1 = 1.0, beta2 = 1.0;
  double shearStress = o.shF / K.max_s + beta2 * o.tM / K.max_t;
  double normalStress = o.nF / K.max_n + beta1 * o.bM / K.max_b;
  return (normalStress > truncated) || (shearStress > (1.0 - normalStress));
}

// BrittleBeamDZCInteraction::broken (Model/BrittleBeamDZC.cpp:122-139) with the effective beam
// section of its constructor (:99-102): radius half the bond's length at creation (dist0),
// area pi R^2, second moments pi R^4 / 4 and pi R^4 / 2.
__device__ __forceinline__ bool dzc_broken(const BondOut& o, double dist0, double cohesion, double tan_angle,
                                           double t_cutoff, double c_cutoff, double beta1, double beta2) {
  const double pi = 3.14159265358979323846;  // M_PI
  const double effR = 0.5 * dist0;
  const double effA = pi * effR * effR;
  const double effI = 0.25 * pi * effR * effR * effR * effR;
  const double effJ = 0.5 * pi * effR * effR * effR * effR;
  const double shearStress = o.shF / effA + beta2 * o.tM * effR / effJ;
  const double normalStress = -1. * (o.nF / effA + beta1 * o.bM * effR / effI);
  return (normalStress < -1. * t_cutoff) || (shearStress > c_cutoff) || (shearStress > (cohesion + normalStress * tan_angle));
}

// BrittleBeamSCInteraction::broken (Model/BrittleBeamSC.cpp:96-150): the bond axis n = (x2 - x1)/|x2 - x1|
// with two transverse axes, the symmetric part of the two particles' mean stress (CParticle::sigma:
// the stress sum over the particle's volume, Model/Particle.cpp:405-408) rotated into that frame, and a
// truncated Mohr-Coulomb test on its normal and shear components.  S1, S2: the stress sums m_sigma.
__device__ __forceinline__ bool sc_broken(const V& x1, double r1, const double* S1, const V& x2, double r2,
                                          const double* S2, double cohesion, double tan_angle, double sigma3) {
  const double pi = 3.14159265358979323846;  // M_PI
  const V d = x2 - x1;
  const V n = d / norm(d);
  V sx;
  if (n.x != 1.0 || n.y != 0.0 || n.z != 0.0) {
    const V c = cross(n, mk(1.0, 0.0, 0.0));
    sx = c / norm(c);
  } else {
    const V c = cross(n, mk(0.0, 1.0, 0.0));
    sx = c / norm(c);
  }
  const V t = cross(n, sx);
  const double dv1 = 1.0 / (4.0 / 3.0 * pi * r1 * r1 * r1), dv2 = 1.0 / (4.0 / 3.0 * pi * r2 * r2 * r2);
  double avg[9], sym[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) avg[k] = 0.5 * (S1[k] * dv1 + S2[k] * dv2);
#pragma unroll
  for (int p = 0; p < 3; ++p)
#pragma unroll
    for (int q = 0; q < 3; ++q) sym[3 * p + q] = 0.5 * (avg[3 * p + q] + avg[3 * q + p]);
  const double nv[3] = {n.x, n.y, n.z}, sv[3] = {sx.x, sx.y, sx.z}, tv[3] = {t.x, t.y, t.z};
  double sn = 0.0, tx = 0.0, ty = 0.0;  // rows n, s, t of the rotation: n.S.n, n.S.s, n.S.t
#pragma unroll
  for (int p = 0; p < 3; ++p)
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      sn += nv[p] * sym[3 * p + q] * nv[q];
      tx += nv[p] * sym[3 * p + q] * sv[q];
      ty += nv[p] * sym[3 * p + q] * tv[q];
    }
  const double tau = sqrt(tx * tx + ty * ty);
  return (sn < -1.0 * sigma3) || (tau > cohesion + sn * tan_angle);
}

// CElasticWallInteraction: ctor scaling (Model/EWallInteraction.hpp:26-36) and
// calcForces (:42-78).  Returns true when in contact; F is the force on the particle.
__device__ __forceinline__ bool law_wall(double k, const V& o, const V& n, const V& x, double r, V& F) {
  double f = 1.0;
  f *= 3.141592654 * r;
  const double m_k = f * k;
  double dist = dot(x - o, n);
  if (dist < r) {
    F = m_k * (r - dist) * n;
    return true;
  }
  return false;
}

// CDamping<T>::calcForces (Model/Damping.hpp:99-124) with v_ref = 0: returns the damping
// force for velocity v, accumulated force frc, inverse mass s and mass m.  The
// rotational form (Model/RotDamping.hpp:58-84) is the same iteration on (omega,
// moment, 1/I, I).
__device__ __forceinline__ V damping_force(const V& v, const V& frc, double s, double mass, double visc, double dt,
                                           int maxiter, int* iterations = nullptr) {
  const double s_limit2 = 1e-12;
  const V vref = mk(0.0, 0.0, 0.0);
  V v_rel = mk(0.0, 0.0, 0.0);
  double error = 1.0;
  int count = 0;
  while ((error * error > s_limit2) & (count < maxiter)) {
    count++;
    V v_old = v_rel;
    v_rel = v - vref + s * dt * (frc - v_rel * visc * mass);
    error = norm2(v_rel - v_old);
  }
  if (iterations) *iterations = count;
  if (count >= maxiter) v_rel = mk(0.0, 0.0, 0.0);
  return -1.0 * visc * v_rel * mass;
}

// CHertzMindlinInteraction::calcForces (Model/HertzMindlinInteraction.cpp:108-172): Hertz normal
// force 4/3 E sqrt(R) dn^1.5 along D/|D| with R = 1 / (1/r1 + 1/r2), Mindlin tangential stiffness
// on the relative translation, one friction coefficient; forces only.  Here fn is the force on p1
// (p2 gets -fn) and Ffric the tangential force on p1 (p2 gets -Ffric).
__device__ __forceinline__ void law_hertz_mindlin(double E, double nu, double mu, double dt, const V& x1, double r1,
                                                  const V& v1, const V& x2, double r2, const V& v2, V Ffric,
                                                  FricOut& o) {
  const V D = x1 - x2;
  double dist = dot(D, D);
  const double eq_dist = r1 + r2;
  if (dist < (eq_dist * eq_dist)) {
    const double R_ij = 1.0 / (1.0 / r1 + 1.0 / r2);
    dist = sqrt(dist);
    const double dn = eq_dist - dist;
    const V dir = D / norm(D);
    const double norm_fn = 4.0 / 3.0 * E * sqrt(R_ij) * pow(dn, 1.5);
    const V fn = dir * norm_fn;
    const V d1 = v1 * dt;
    const V d2 = v2 * dt;
    V ds = d2 - d1;
    ds -= dot(ds, dir) * dir;
    Ffric += 2.0 / 3.0 * 8.0 * E / 2.0 / (1.0 + nu) * sqrt(R_ij) * sqrt(dn) * ds;
    const double FfricNorm = norm(Ffric);
    const double forceNorm = norm(fn);
    if (FfricNorm > forceNorm * mu) {
      Ffric = Ffric * ((mu * forceNorm) / FfricNorm);
      o.slipping = true;
    } else {
      o.slipping = false;
    }
    o.fn = fn;
    o.Ffric = Ffric;
    o.M1 = o.M2 = mk(0.0, 0.0, 0.0);
    o.touching = true;
  } else {
    o.Ffric = o.fn = o.M1 = o.M2 = mk(0.0, 0.0, 0.0);
    o.slipping = false;
    o.touching = false;
  }
}

// CHertzMindlinViscoInteraction::calcForces (Model/HertzMindlinViscoInteraction.cpp:119-200): the Hertz
// normal force less a normal damping term, and a tangential force recomputed every step (no history)
// less a tangential damping term, both from the coefficient of restitution (Antypov 2011, as the
// reference writes it, with its 3.1415926).  fn here is the net normal force on p1 (p2 gets -fn),
// Ffric the tangential force on p1 (p2 gets -Ffric).
__device__ __forceinline__ void law_hertz_mindlin_visco(double E, double nu, double mu, double COR, double dt,
                                                        const V& x1, double r1, double m1, const V& v1, const V& x2,
                                                        double r2, double m2, const V& v2, FricOut& o) {
  const V D = x1 - x2;
  double dist = dot(D, D);
  const double eq_dist = r1 + r2;
  o.M1 = o.M2 = mk(0.0, 0.0, 0.0);
  if (!(dist < (eq_dist * eq_dist))) {
    o.Ffric = o.fn = mk(0.0, 0.0, 0.0);
    o.slipping = false;
    o.touching = false;
    return;
  }
  const double R_ij = 1.0 / (1.0 / r1 + 1.0 / r2);
  dist = sqrt(dist);
  const double dn = eq_dist - dist;
  const V dir = D / norm(D);
  const double norm_fn = 4.0 / 3.0 * E * sqrt(R_ij) * pow(dn, 1.5);
  const V fn = dir * norm_fn;
  const double M_ij = 1.0 / (1.0 / m1 + 1.0 / m2);
  const V v_rel = v2 - v1;
  const V v_nor = dot(v_rel, dir) * dir;
  const double lnCOR = log(COR);
  const V normal_damping = 2.0 * sqrt(5.0 / 3.0) * lnCOR / sqrt(pow(lnCOR, 2) + pow(3.1415926, 2)) * sqrt(M_ij * E) *
                           pow(R_ij, 0.25) * pow(dn, 0.25) * v_nor;
  const V d1 = v1 * dt;
  const V d2 = v2 * dt;
  V ds = d2 - d1;
  ds -= dot(ds, dir) * dir;
  V Ffric = 2.0 / 3.0 * 8.0 * E / 2.0 / (1.0 + nu) * sqrt(R_ij) * sqrt(dn) * ds;
  const V v_tan = v_rel - v_nor;
  const V tange_damping = sqrt(80.0 / 3.0) * lnCOR / sqrt(pow(lnCOR, 2) + pow(3.1415926, 2)) *
                          sqrt(M_ij * E / 2.0 / (1.0 + nu)) * pow(R_ij, 0.25) * pow(dn, 0.25) * v_tan;
  Ffric -= tange_damping;
  const double FfricNorm = norm(Ffric);
  const double forceNorm = norm(fn);
  o.slipping = FfricNorm > forceNorm * mu;
  if (o.slipping) Ffric = Ffric * ((mu * forceNorm) / FfricNorm);
  o.fn = fn - normal_damping;
  o.Ffric = Ffric;
  o.touching = true;
}

// CLocalDamping::calcForces (Model/LocalDamping.hpp:82-118) and CRotLocalDamping::calcForces
// (Model/RotLocalDamping.hpp:82-117): each component of the accumulated force (moment) with the
// sign of the velocity (spin) component, zero where that component is zero, times -visc.
__device__ __forceinline__ V local_damping_force(const V& v, const V& frc, double visc) {
  double fx = fabs(frc.x), fy = fabs(frc.y), fz = fabs(frc.z);
  if (v.x < 0) fx *= -1.;
  if (v.x == 0) fx = 0.0;
  if (v.y < 0) fy *= -1.;
  if (v.y == 0) fy = 0.0;
  if (v.z < 0) fz *= -1.;
  if (v.z == 0) fz = 0.0;
  return -1.0 * visc * mk(fx, fy, fz);
}

}  // namespace dem
