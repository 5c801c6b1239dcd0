// Pair laws of the FP32-force form: contact detection, the overlap and the
// pair's relative position vector stay in FP64 (so the contact set and the
// lever arms are those of the FP64 path); the force arithmetic that follows runs
// in FP32 on relative vectors; the stick-slip threshold is re-decided in FP64
// when the FP32 comparison falls inside a relative band of 1e-5.
#pragma once
#include "dem_laws.cuh"

namespace dem {

using Vf = V3<float>;

// Kahan-compensated FP32 accumulation of 3-vectors.
struct KSum3 {
  Vf s, c;
  __device__ __forceinline__ void zero() { s = mk(0.f, 0.f, 0.f); c = s; }
  __device__ __forceinline__ void add1(float& sum, float& comp, float v) {
    const float y = v - comp;
    const float t = sum + y;
    comp = (t - sum) - y;
    sum = t;
  }
  __device__ __forceinline__ void add(const Vf& v) { add1(s.x, c.x, v.x); add1(s.y, c.y, v.y); add1(s.z, c.z, v.z); }
  __device__ __forceinline__ V value() const {
    return mk((double)s.x - (double)c.x, (double)s.y - (double)c.y, (double)s.z - (double)c.z);
  }
};

// CElasticInteraction::calcForces in the FP32 form.  D = x1 - x2 in FP64.
__device__ __forceinline__ bool law_elastic_f32(double k_eff, const V& D, double r1, double r2, Vf& F) {
  const double dist2 = dot(D, D);
  const double eq_dist = r1 + r2;
  if (dist2 < eq_dist * eq_dist) {
    const double dist = sqrt(dist2);
    const float s = (float)(k_eff * (dist - eq_dist) / dist);
    F = cvt<float>(D) * s;
    return true;
  }
  return false;
}

struct FricOutF {
  Vf fn, Ffric, M1, M2;
  bool touching, slipping;
};

// CRotFrictionInteraction::calcSimpleForces in the FP32 form.  D = x1 - x2 (FP64);
// v, w are the FP32 copies of the particles' velocities and spins.
__device__ __forceinline__ void law_friction_f32(double k_eff, double ks_eff, double mu_s, double mu_d, float dt,
                                                 const V& D, double r1, double r2, const Vf& v1, const Vf& w1,
                                                 const Vf& v2, const Vf& w2, Vf Ff, bool slipping, FricOutF& o) {
  const double dist2 = dot(D, D);
  const double eq_dist = r1 + r2;
  if (dist2 < eq_dist * eq_dist) {
    const double dist = sqrt(dist2);
    const double over = dist - eq_dist;
    const Vf Df = cvt<float>(D);
    const Vf force = Df * (float)(k_eff * over / dist);
    // contact point x2 + r2/(r1+r2) D, as lever arms from each centre
    const float a2 = (float)(r2 / eq_dist);
    const Vf arm2 = Df * a2;
    const Vf arm1 = arm2 - Df;
    const Vf vp1 = v1 + cross(w1, arm1);
    const Vf vp2 = v2 + cross(w2, arm2);
    Vf ds = (vp2 - vp1) * dt;
    ds -= (dot(ds, Df) / dot(Df, Df)) * Df;
    Ff += (float)ks_eff * ds;
    const float FfN = norm(Ff);
    const float fN = norm(force);
    const double mu_cur = slipping ? mu_d : mu_s;
    const float thr = fN * (float)mu_cur;
    bool slip = FfN > thr;
    if (fabsf(FfN - thr) <= 1e-5f * thr) {  // inside the band: decide in FP64
      const V Ffd = cvt<double>(Ff);
      slip = norm(Ffd) > fabs(k_eff * over) * mu_cur;
    }
    if (slip) {
      Ff = Ff * (float)((mu_d * (double)fN) / (double)FfN);
      o.slipping = true;
    } else {
      o.slipping = false;
    }
    o.M1 = cross(arm1, Ff);
    o.M2 = cross(arm2, -Ff);
    o.fn = force;
    o.Ffric = Ff;
    o.touching = true;
  } else {
    o.Ffric = o.fn = o.M1 = o.M2 = mk(0.f, 0.f, 0.f);
    o.slipping = false;
    o.touching = false;
  }
}

}  // namespace dem
