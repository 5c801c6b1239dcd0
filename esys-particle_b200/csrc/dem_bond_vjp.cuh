// Hand-written reverse (vector-Jacobian product) of the RotBond law
// (ARotBondedInteraction::calcForces, Model/ARotBondedInteraction.cpp:307-448, as
// restated in law_bond_t): given the adjoints of the bond's force on p1 and of
// its two moments, the gradients with respect to both positions, both
// quaternions and the four scaled stiffnesses.  The forward is recomputed in
// the same operation order; every branch (the acos guards, the zero-norm guards,
// calc_angle's sign) is the one the forward takes; the derivative of sqrt at 0
// is taken as 0, as the forward-mode duals of dem_dual.cuh do, so both adjoints
// agree wherever the law is differentiable.
#pragma once
#include "dem_laws.cuh"

namespace dem {

struct BondVjp {
  V x1, x2;       // d/dx1, d/dx2 (x2: the periodic image used by the law)
  Qd q1, q2;      // d/dq1, d/dq2
  double kr, ks, kt, kb;  // d/d(scaled stiffness)
};

// c = a (x) b (Quaternion.hpp operator*): adjoints of a and b from that of c.
__device__ __forceinline__ void qmul_vjp(const Qd& a, const Qd& b, const Qd& c_, Qd& a_, Qd& b_) {
  a_.s += c_.s * b.s + dot(c_.v, b.v);
  a_.v += -c_.s * b.v + b.s * c_.v + cross(b.v, c_.v);
  b_.s += c_.s * a.s + dot(c_.v, a.v);
  b_.v += -c_.s * a.v + a.s * c_.v + cross(c_.v, a.v);
}

// Adjoint of q from that of R = to_matrix(q) (Quaternion::to_matrix).
__device__ __forceinline__ void to_matrix_vjp(const Qd& q, const M3<double>& R_, Qd& q_) {
  const double s = q.s, x = q.v.x, y = q.v.y, z = q.v.z;
  const double (*R)[3] = R_.m;
  q_.s += 2.0 * (s * (R[0][0] + R[1][1] + R[2][2]) + z * (R[0][1] - R[1][0]) + y * (R[2][0] - R[0][2]) +
                 x * (R[1][2] - R[2][1]));
  q_.v.x += 2.0 * (x * (R[0][0] - R[1][1] - R[2][2]) + y * (R[0][1] + R[1][0]) + z * (R[0][2] + R[2][0]) +
                   s * (R[1][2] - R[2][1]));
  q_.v.y += 2.0 * (y * (-R[0][0] + R[1][1] - R[2][2]) + x * (R[0][1] + R[1][0]) + z * (R[1][2] + R[2][1]) +
                   s * (R[2][0] - R[0][2]));
  q_.v.z += 2.0 * (z * (-R[0][0] - R[1][1] + R[2][2]) + s * (R[0][1] - R[1][0]) + x * (R[0][2] + R[2][0]) +
                   y * (R[1][2] + R[2][1]));
}

// y = M^T v: adjoint of v is M y_, adjoint of M[j][i] gets y_[i] v[j].
__device__ __forceinline__ void mulT_vjp(const M3<double>& M, const V& v, const V& y_, M3<double>& M_, V& v_) {
  v_ += mul(M, y_);
  const double vv[3] = {v.x, v.y, v.z}, yy[3] = {y_.x, y_.y, y_.z};
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) M_.m[j][i] += yy[i] * vv[j];
}

// u = a / |a| (|a| = n > 0): adjoint of a from that of u.
__device__ __forceinline__ V unit_vjp(const V& u, double n, const V& u_) { return (u_ - dot(u, u_) * u) / n; }

__device__ __forceinline__ double sqrt_d(double r) { return r > 0.0 ? 0.5 / r : 0.0; }  // d sqrt(u)/du at sqrt(u) = r

__device__ __forceinline__ void law_bond_vjp(const BondK& K, const V& mD, const V& x1, double r1, const Qd& q1,
                                             const V& x2, double r2, const Qd& q2, const V& f_, const V& m1_,
                                             const V& m2_, BondVjp& g) {
  const double HALF_SQRT_2 = 0.5 * sqrt(2.0);
  // ---------------- forward (law_bond_t, same operations) ----------------
  const M3<double> mat0 = to_matrix(q1);
  const V rbp = x2 - x1;
  const double rbpNorm = norm(rbp);
  const V rb = mul(mat0, x2 - x1);
  const double rbNorm = norm(rb);
  const double r_0Norm = r1 + r2;
  const V dr_v = (rbNorm - r_0Norm) * rb;
  const V delta_r = dr_v / rbNorm;
  const V Fr = K.kr * delta_r;
  const double mDn = norm(mD);
  const double gc_num = dot(rb, mD), gc_den = rbNorm * mDn;
  const double gama_cos = gc_num / gc_den;
  const bool gama_on = gama_cos < 1.0 && gama_cos > -1.0;
  const double gama = gama_on ? acos(gama_cos) : 0.0;
  const V rb_0 = cross(rb, mD);
  const V rb_b0 = cross(rb, rb_0);
  const double rb_b0Norm = norm(rb_b0);
  const bool fst_on = rb_b0Norm != 0;
  const double a_st = K.ks * r_0Norm * gama;
  V Fst = mk(0.0, 0.0, 0.0);
  if (fst_on) Fst = a_st * rb_b0 / rb_b0Norm;
  const double rb_0Norm = norm(rb_0);
  const bool mst_on = rb_0Norm != 0;
  const double nFst = norm(Fst);
  V Mst = mk(0.0, 0.0, 0.0);
  if (mst_on) Mst = -nFst * rb_0 / rb_0Norm;
  const double u0 = (rbNorm + rb.z) / rbNorm, u1 = (rbNorm - rb.z) / rbNorm;
  const double s0 = sqrt(u0), s1 = sqrt(u1);
  const double m0 = HALF_SQRT_2 * s0;
  const double m1a = -HALF_SQRT_2 * s1;
  const double m2a = -m1a;
  const double rxy2 = rb.x * rb.x + rb.y * rb.y;
  const bool xy_on = rxy2 != 0.0;
  const double dsq = xy_on ? sqrt(rxy2) : 1.0;
  double m1 = m1a, m2 = m2a;
  if (xy_on) {
    m1 = m1a * rb.y / dsq;
    m2 = m2a * rb.x / dsq;
  }
  const Qd qm{m0, mk(m1, m2, 0.0)};
  const M3<double> mat = to_matrix(qm);
  const Qd q1i = qinv(q1), qmi = qinv(qm);
  const Qd rp = qmul(q1i, q2);
  const Qd t = qmul(qmi, rp);
  const Qd r = qmul(t, qm);
  const double temp0 = r.s * r.s + r.v.z * r.v.z;
  double pasi = 0.0, c_pasi2 = 0.0, sq0 = 0.0, pasi_sign = 0.0;
  if (temp0 != 0.0) {
    sq0 = sqrt(temp0);
    c_pasi2 = r.s / sq0;
    const double s_pasi2 = r.v.z / sq0;
    const double ang = calc_angle(s_pasi2, c_pasi2);
    pasi = 2.0 * ang;
    const bool inside = !(c_pasi2 >= 1.0 || c_pasi2 <= -1.0);
    pasi_sign = (s_pasi2 > 0.0 && inside) ? 1.0 : ((s_pasi2 < 0.0 && inside) ? -1.0 : 0.0);
  }
  const V Mtp = mk(0.0, 0.0, K.kt * pasi);
  const V Mtr = mulT(mat, Mtp);
  const double temp2 = r.v.x * r.v.x + r.v.y * r.v.y;
  const double temp3 = r.v.x * r.v.z + r.s * r.v.y;
  const double temp4 = r.v.y * r.v.z - r.s * r.v.x;
  V Mbr = mk(0.0, 0.0, 0.0), Fsr = Mbr, Msr = Mbr, Mbp = Mbr, Fsp = Mbr, Msp = Mbr;
  double sita = 0.0, c_fai = 0.0, s_fai = 0.0, temp1 = 0.0, sd = 0.0;
  const bool b_on = temp2 != 0.0;
  bool sita_on = false;
  if (b_on) {
    temp1 = temp0 - temp2;
    sita_on = !(temp1 >= 1.0 || temp1 <= -1.0);
    sita = sita_on ? acos(temp1) : 0.0;
    if (temp0 == 0.0) {
      sd = sqrt(temp2);
      c_fai = r.v.y / sd;
      s_fai = -r.v.x / sd;
    } else {
      sd = sqrt(temp0 * temp2);
      c_fai = temp3 / sd;
      s_fai = temp4 / sd;
    }
    Mbp = mk(-0.5 * K.kb * sita * s_fai, 0.5 * K.kb * sita * c_fai, 0.0);
    Mbr = mulT(mat, Mbp);
    Fsp = mk(-0.5 * K.ks * c_fai * sita * r_0Norm, -0.5 * K.ks * s_fai * sita * r_0Norm, 0.0);
    Fsr = mulT(mat, Fsp);
    Msp = mk(0.5 * K.ks * s_fai * sita * r_0Norm, -0.5 * K.ks * c_fai * sita * r_0Norm, 0.0);
    Msr = mulT(mat, Msp);
  }
  const double eq_rad1 = r1 / (r1 + r2);
  const double eq_rad2 = r2 / (r1 + r2);
  const V A = Fr + Fst + Fsr;
  const V S = Msr + Mst;  // both enter the moments scaled by eq_rad * rbpNorm
  const V B1 = Mbr + Mtr + Msr * eq_rad1 * rbpNorm + Mst * eq_rad1 * rbpNorm;
  const V B2 = Msr * eq_rad2 * rbpNorm + Mst * eq_rad2 * rbpNorm - Mbr - Mtr;

  // ---------------- reverse ----------------
  M3<double> mat0_{}, mat_{};
  V A_ = mk(0.0, 0.0, 0.0), B1_ = A_, B2_ = A_;
  mulT_vjp(mat0, A, f_, mat0_, A_);
  mulT_vjp(mat0, B1, m1_, mat0_, B1_);
  mulT_vjp(mat0, B2, m2_, mat0_, B2_);
  const V Fr_ = A_, Fst_in = A_, Fsr_ = A_;
  const V Mbr_ = B1_ - B2_, Mtr_ = B1_ - B2_;
  const V S_ = (eq_rad1 * rbpNorm) * B1_ + (eq_rad2 * rbpNorm) * B2_;
  const V Msr_ = S_, Mst_ = S_;
  double rbpNorm_ = eq_rad1 * dot(S, B1_) + eq_rad2 * dot(S, B2_);

  double kr_ = 0.0, ks_ = 0.0, kt_ = 0.0, kb_ = 0.0;
  // bending / shear rotation terms
  double sita_ = 0.0, c_fai_ = 0.0, s_fai_ = 0.0;
  if (b_on) {
    V Mbp_ = mk(0.0, 0.0, 0.0), Fsp_ = Mbp_, Msp_ = Mbp_;
    mulT_vjp(mat, Mbp, Mbr_, mat_, Mbp_);
    mulT_vjp(mat, Fsp, Fsr_, mat_, Fsp_);
    mulT_vjp(mat, Msp, Msr_, mat_, Msp_);
    // Mbp = (-0.5 kb sita s, 0.5 kb sita c, 0)
    kb_ += Mbp_.x * (-0.5 * sita * s_fai) + Mbp_.y * (0.5 * sita * c_fai);
    sita_ += Mbp_.x * (-0.5 * K.kb * s_fai) + Mbp_.y * (0.5 * K.kb * c_fai);
    s_fai_ += Mbp_.x * (-0.5 * K.kb * sita);
    c_fai_ += Mbp_.y * (0.5 * K.kb * sita);
    // Fsp = (-0.5 ks c sita r0, -0.5 ks s sita r0, 0)
    ks_ += Fsp_.x * (-0.5 * c_fai * sita * r_0Norm) + Fsp_.y * (-0.5 * s_fai * sita * r_0Norm);
    c_fai_ += Fsp_.x * (-0.5 * K.ks * sita * r_0Norm);
    s_fai_ += Fsp_.y * (-0.5 * K.ks * sita * r_0Norm);
    sita_ += Fsp_.x * (-0.5 * K.ks * c_fai * r_0Norm) + Fsp_.y * (-0.5 * K.ks * s_fai * r_0Norm);
    // Msp = (0.5 ks s sita r0, -0.5 ks c sita r0, 0)
    ks_ += Msp_.x * (0.5 * s_fai * sita * r_0Norm) + Msp_.y * (-0.5 * c_fai * sita * r_0Norm);
    s_fai_ += Msp_.x * (0.5 * K.ks * sita * r_0Norm);
    c_fai_ += Msp_.y * (-0.5 * K.ks * sita * r_0Norm);
    sita_ += Msp_.x * (0.5 * K.ks * s_fai * r_0Norm) + Msp_.y * (-0.5 * K.ks * c_fai * r_0Norm);
  }
  // twist: Mtr = mat^T (0, 0, kt pasi)
  V Mtp_ = mk(0.0, 0.0, 0.0);
  mulT_vjp(mat, Mtp, Mtr_, mat_, Mtp_);
  kt_ += Mtp_.z * pasi;
  double pasi_ = Mtp_.z * K.kt;

  // r's scalar functions
  double rs_ = 0.0, rx_ = 0.0, ry_ = 0.0, rz_ = 0.0, temp0_ = 0.0, temp2_ = 0.0, temp3_ = 0.0, temp4_ = 0.0;
  if (b_on) {
    if (temp0 == 0.0) {  // c = r.y / sd, s = -r.x / sd, sd = sqrt(temp2)
      ry_ += c_fai_ / sd;
      rx_ += -s_fai_ / sd;
      const double sd_ = -(c_fai_ * r.v.y + s_fai_ * (-r.v.x)) / (sd * sd);
      temp2_ += sd_ * sqrt_d(sd);
    } else {             // c = temp3 / sd, s = temp4 / sd, sd = sqrt(temp0 temp2)
      temp3_ += c_fai_ / sd;
      temp4_ += s_fai_ / sd;
      const double sd_ = -(c_fai_ * temp3 + s_fai_ * temp4) / (sd * sd);
      const double prod_ = sd_ * sqrt_d(sd);
      temp0_ += prod_ * temp2;
      temp2_ += prod_ * temp0;
    }
    if (sita_on) {
      const double t1_ = sita_ * (-1.0 / sqrt(1.0 - temp1 * temp1));
      temp0_ += t1_;
      temp2_ -= t1_;
    }
  }
  // temp3 = rx rz + rs ry, temp4 = ry rz - rs rx, temp2 = rx^2 + ry^2
  rx_ += temp3_ * r.v.z - temp4_ * r.s + 2.0 * temp2_ * r.v.x;
  rz_ += temp3_ * r.v.x + temp4_ * r.v.y;
  rs_ += temp3_ * r.v.y - temp4_ * r.v.x;
  ry_ += temp3_ * r.s + temp4_ * r.v.z + 2.0 * temp2_ * r.v.y;
  if (temp0 != 0.0) {  // pasi = 2 (+-)acos(c), c = rs / sq0, sq0 = sqrt(temp0)
    const double c_ = pasi_ * 2.0 * pasi_sign * (pasi_sign != 0.0 ? -1.0 / sqrt(1.0 - c_pasi2 * c_pasi2) : 0.0);
    rs_ += c_ / sq0;
    const double sq0_ = -c_ * r.s / (sq0 * sq0);
    temp0_ += sq0_ * sqrt_d(sq0);
  }
  rs_ += 2.0 * temp0_ * r.s;
  rz_ += 2.0 * temp0_ * r.v.z;
  // r = t (x) qm, t = qm^-1 (x) rp, rp = q1^-1 (x) q2
  const Qd r_{rs_, mk(rx_, ry_, rz_)};
  Qd t_{0.0, mk(0.0, 0.0, 0.0)}, qm_ = t_, qmi_ = t_, rp_ = t_, q1i_ = t_, q2_ = t_;
  qmul_vjp(t, qm, r_, t_, qm_);
  qmul_vjp(qmi, rp, t_, qmi_, rp_);
  qmul_vjp(q1i, q2, rp_, q1i_, q2_);
  qm_.s += qmi_.s;
  qm_.v = qm_.v - qmi_.v;
  to_matrix_vjp(qm, mat_, qm_);
  // qm = (m0, (m1, m2, 0)) from rb
  V rb_ = mk(0.0, 0.0, 0.0);
  double rbNorm_ = 0.0;
  double m1a_ = 0.0, m2a_ = 0.0;
  if (xy_on) {
    m1a_ += qm_.v.x * rb.y / dsq;
    rb_.y += qm_.v.x * m1a / dsq;
    m2a_ += qm_.v.y * rb.x / dsq;
    rb_.x += qm_.v.y * m2a / dsq;
    const double dsq_ = -(qm_.v.x * m1a * rb.y + qm_.v.y * m2a * rb.x) / (dsq * dsq);
    const double rxy2_ = dsq_ * sqrt_d(dsq);
    rb_.x += 2.0 * rb.x * rxy2_;
    rb_.y += 2.0 * rb.y * rxy2_;
  } else {
    m1a_ += qm_.v.x;
    m2a_ += qm_.v.y;
  }
  m1a_ -= m2a_;
  const double u0_ = qm_.s * HALF_SQRT_2 * sqrt_d(s0);
  const double u1_ = m1a_ * (-HALF_SQRT_2) * sqrt_d(s1);
  // u0 = (rbN + rbz) / rbN, u1 = (rbN - rbz) / rbN
  rbNorm_ += u0_ * (-rb.z / (rbNorm * rbNorm)) + u1_ * (rb.z / (rbNorm * rbNorm));
  rb_.z += u0_ / rbNorm - u1_ / rbNorm;

  // Mst = -|Fst| rb_0 / |rb_0|
  V Fst_ = Fst_in;
  V rb_0_ = mk(0.0, 0.0, 0.0);
  if (mst_on) {
    const V w = rb_0 / rb_0Norm;
    const double nF_ = -dot(Mst_, w);
    const V w_ = -nFst * Mst_;
    rb_0_ += unit_vjp(w, rb_0Norm, w_);
    if (nFst > 0.0) Fst_ += (nF_ / nFst) * Fst;
  }
  // Fst = a u, u = rb_b0 / |rb_b0|, a = ks r0 gama
  double gama_ = 0.0;
  V rb_b0_ = mk(0.0, 0.0, 0.0);
  if (fst_on) {
    const V u = rb_b0 / rb_b0Norm;
    const double a_ = dot(Fst_, u);
    rb_b0_ += unit_vjp(u, rb_b0Norm, a_st * Fst_);
    ks_ += a_ * r_0Norm * gama;
    gama_ += a_ * K.ks * r_0Norm;
  }
  // rb_b0 = rb x rb_0, rb_0 = rb x mD
  rb_ += cross(rb_0, rb_b0_);
  rb_0_ += cross(rb_b0_, rb);
  rb_ += cross(mD, rb_0_);
  // gama = acos(gc), gc = (rb . mD) / (rbN |mD|)
  if (gama_on) {
    const double gc_ = gama_ * (-1.0 / sqrt(1.0 - gama_cos * gama_cos));
    rb_ += (gc_ / gc_den) * mD;
    rbNorm_ += -gc_ * gama_cos / gc_den * mDn;
  }
  // Fr = kr delta_r, delta_r = ((rbN - r0) rb) / rbN
  kr_ += dot(Fr_, delta_r);
  const V delta_ = K.kr * Fr_;
  const V drv_ = delta_ / rbNorm;
  rbNorm_ += -dot(delta_, dr_v) / (rbNorm * rbNorm);
  rbNorm_ += dot(drv_, rb);
  rb_ += (rbNorm - r_0Norm) * drv_;
  // rbN = |rb|, rb = mat0 rbp
  rb_ += (rbNorm_ / rbNorm) * rb;
  V rbp_ = mulT(mat0, rb_);
  {
    const double rr[3] = {rb_.x, rb_.y, rb_.z}, pp[3] = {rbp.x, rbp.y, rbp.z};
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) mat0_.m[i][j] += rr[i] * pp[j];
  }
  rbp_ += (rbpNorm_ / rbpNorm) * rbp;
  g.x2 = rbp_;
  g.x1 = -rbp_;
  Qd q1_{0.0, mk(0.0, 0.0, 0.0)};
  to_matrix_vjp(q1, mat0_, q1_);
  q1_.s += q1i_.s;
  q1_.v = q1_.v - q1i_.v;
  g.q1 = q1_;
  g.q2 = q2_;
  g.kr = kr_;
  g.ks = ks_;
  g.kt = kt_;
  g.kb = kb_;
}

}  // namespace dem
