// Reverse-mode kernels of the differentiable loading window (dem_window_adjoint).
//
// The window is the FP64 step with the contact topology and the bond state
// frozen: the pair lists of the dynamic groups, the intact bonds and the wall
// candidates are those of the forward pass, and every branch of a law (touching,
// slipping, acos guards, the damping iteration count) is the one the forward
// pass took.  The state of particle i at step t is (x, v, omega, q) and the
// friction history of each RotFriction pair; the outputs whose gradients are
// wanted are the platen reactions (CWall::m_force after each step).
//
// One reverse step takes lambda_{t+1}, the adjoint of the state after step t,
// to lambda_t, with the forward states of the step recomputed from checkpoints:
//   k_adj_pre   per particle, hand-written: quaternion normalisation and update
//               (CRotParticle::integrate + rescale, Model/RotParticle.cpp:277-321),
//               the Euler velocity / position update (Model/Particle.cpp:257-274),
//               the damping fixed point unrolled over the forward iteration count
//               (Model/Damping.hpp:99-124, Model/RotDamping.hpp:58-84), the
//               elastic walls (Model/EWallInteraction.hpp:42-78) and the loss
//               term of the reactions.  Produces lF, lM: the adjoint of the
//               force and moment sums before damping.
//   k_adj_bond  per bond: the RotBond law (Model/ARotBondedInteraction.cpp:307-448)
//               evaluated on 18-component dual numbers (x1, q1, x2, q2, kr, ks,
//               kt, kb) and contracted with lF / lM of its two particles.
//   k_adj_pair  per pair of a dynamic group: CElasticInteraction (7 components)
//               or CRotFrictionInteraction (23: x1, x2, v1, v2, w1, w2, the
//               tangential history, k, ks), contracted with lF / lM and the
//               adjoint of the pair's next history; writes the history adjoint.
//   k_adj_post  per particle: the bond and pair contributions gathered in
//               adjacency order (no atomics, run-to-run reproducible).
// Parameter gradients accumulate in per-bond / per-pair / per-particle slots
// across the window and are reduced once, in a fixed order, at the end.
#include "dem_adjoint.h"
#include "dem_common.cuh"
#include "dem_dual.cuh"
#include "dem_bond_vjp.cuh"
#include "dem_pair_vjp.cuh"
#include "dem_laws.cuh"

namespace dem {

__device__ __forceinline__ V xyzv(const double4& a) { return mk(a.x, a.y, a.z); }

// lambda_q . d[(0,w)(x)q]/dq and lambda_q . d[(0,w)(x)q]/dw (Quaternion.hpp operator*):
// (0,w)(x)q = ( -w.qv , qs w + w x qv ) is bilinear in (w, q).
__device__ __forceinline__ void omega_times_vjp(const V& w, const Qd& q, const Qd& lq, Qd& lq_out, V& lw_out) {
  lq_out.s = dot(lq.v, w);
  lq_out.v = -lq.s * w + cross(lq.v, w);
  lw_out = -lq.s * q.v + q.s * lq.v + cross(q.v, lq.v);
}

// G = sum_{k<c} (-a)^k (the c-th damping iterate is G u) and dG/da.
__device__ __forceinline__ void damp_series(double a, int c, double& G, double& dG) {
  G = 0.0;
  dG = 0.0;
  double p = 1.0;   // (-a)^k
  double dp = 0.0;  // d/da (-a)^k
  for (int k = 0; k < c; ++k) {
    G += p;
    dG += dp;
    dp = -(double)(k + 1) * p;
    p *= -a;
  }
}

// Reverse of one damping group on one particle: F_tot = F + D(v, F),
// D = -visc m G (v + s dt F) when the fixed point converged in c < maxiter iterations.
__device__ __forceinline__ void damping_vjp(const V& v, const V& F, double s, double m, double visc, double dt, int c,
                                            int maxiter, const V& lFtot, V& lF, V& lv, double& gvisc) {
  lF = lFtot;
  if (c >= maxiter) return;  // v_rel = 0: no damping force
  double G, dGa;
  damp_series(s * dt * visc * m, c, G, dGa);
  const V u = v + (s * dt) * F;
  lF = lFtot * (1.0 - visc * m * G * s * dt);
  lv = lv + (-visc * m * G) * lFtot;
  const double dGdvisc = dGa * s * dt * m;
  gvisc += dot(lFtot, (-m * (G + visc * dGdvisc)) * u);
}

__device__ __forceinline__ void adj_pre_one(const AdjArgs& A, int i) {
  const unsigned pf = A.pflags[i];
  if (!(pf & PF_ALIVE)) return;
  const double dt = A.dt;
  const double4 p4 = A.s0.pr[i], v4 = A.s0.vm[i];
  const bool dyn = pf & PF_DYN;
  const double m = v4.w;
  const double invm = m != 0.0 ? 1.0 / m : 0.0;  // as the step kernel forms it
  V lx = xyzv(A.lx[i]), lv = xyzv(A.lv[i]);

  // position and velocity: v1 = v + F_tot/m dt, x1 = x + v1 dt
  V lFtot = mk(0.0, 0.0, 0.0), lv_t = lv;
  if (dyn) {
    const V lv_tot = lv + dt * lx;
    lFtot = (invm * dt) * lv_tot;
    lv_t = lv_tot;
  }
  V lx_t = lx;
  V lF = lFtot;
  double gl = 0.0, gr = 0.0;
  if (A.damp_lin)
    damping_vjp(xyzv(v4), xyzv(A.f_int[i]), invm, m, A.visc_lin, A.dt_lin, A.iters[2 * i], A.iter_lin, lFtot, lF,
                lv_t, gl);

  V lM = mk(0.0, 0.0, 0.0), lw_t = lM;
  Qd lq_t{0.0, lM};
  if (A.rot) {
    const double4 w4 = A.s0.wi[i], q4 = A.s0.qq[i], w1 = A.s1.wi[i];
    const double I = w4.w, invI = 1.0 / I;
    const V lw = xyzv(A.lw[i]);
    const double4 lq4 = A.lq[i];
    const Qd lq1{lq4.x, mk(lq4.y, lq4.z, lq4.w)};
    const Qd q{q4.x, mk(q4.y, q4.z, q4.w)};
    const bool rot = pf & PF_ROT;
    // q' = q + dt/2 (0, w1) (x) q for rotating particles, then q1 = q' / |q'|
    Qd qp = q;
    const V wn = xyzv(w1);
    if (rot) {
      const Qd dq = qmul(Qd{0.0, wn}, q);
      const double c = dt / 2.0;
      qp.s = q.s + c * dq.s;
      qp.v = q.v + c * dq.v;
    }
    const double nq = sqrt(qp.s * qp.s + dot(qp.v, qp.v));
    const Qd qn{qp.s / nq, qp.v / nq};
    const double pr = qn.s * lq1.s + dot(qn.v, lq1.v);
    const Qd lqp{(lq1.s - qn.s * pr) / nq, (lq1.v - qn.v * pr) / nq};
    lq_t = lqp;
    if (rot) {
      Qd aq;
      V aw;
      omega_times_vjp(wn, q, lqp, aq, aw);
      const double c = dt / 2.0;
      lq_t.s += c * aq.s;
      lq_t.v += c * aq.v;
      // w1 = w + dt/I M_tot; w1 feeds the output spin and the quaternion update
      const V lw_tot = lw + c * aw;
      const V lMtot = (dt * invI) * lw_tot;
      lw_t = lw_tot;
      lM = lMtot;
      if (A.damp_rot)
        damping_vjp(xyzv(w4), xyzv(A.m_int[i]), invI, I, A.visc_rot, A.dt_rot, A.iters[2 * i + 1], A.iter_rot, lMtot,
                    lM, lw_t, gr);
    }
  }

  // elastic walls: f = k' (r - d) n for d = (x - o).n < r; inner candidates feed the reactions
  const V x = xyzv(p4);
  for (int w = 0; w < A.nwall; ++w) {
    if (!(pf & (1u << (PF_WALL_SHIFT + w)))) continue;
    const WallDev W = A.walls[w];
    const V o = mk(W.ox, W.oy, W.oz), nn = mk(W.nx, W.ny, W.nz);
    const double d = dot(x - o, nn);
    if (!(d < p4.w)) continue;
    double f = 1.0;
    f *= 3.141592654 * p4.w;
    const double mk_ = f * W.k;
    V lf = lF;
    if (pf & (1u << (PF_INNER_SHIFT + w))) lf = lf + mk(A.gR[3 * w], A.gR[3 * w + 1], A.gR[3 * w + 2]);
    lx_t = lx_t + (-mk_ * dot(nn, lf)) * nn;
  }
  A.lx[i] = d4(lx_t, 0.0);
  A.lv[i] = d4(lv_t, 0.0);
  A.lF[i] = d4(lF, 0.0);
  if (A.rot) {
    A.lw[i] = d4(lw_t, 0.0);
    A.lq[i] = make_double4(lq_t.s, lq_t.v.x, lq_t.v.y, lq_t.v.z);
    A.lM[i] = d4(lM, 0.0);
  }
  A.gvisc[2 * i] += gl;
  A.gvisc[2 * i + 1] += gr;
}

__global__ void k_adj_pre(const AdjArgs A) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < A.n) adj_pre_one(A, i);
}

// Tangent slot of input gi in the pass whose inputs are [base, base + N): a unit tangent there,
// a constant elsewhere (the slot index is compared, never used as an array index, so the dual
// stays in registers).
template <int N>
__device__ __forceinline__ Dual<N> seed_in(double v, int gi, int base) {
  Dual<N> r(v);
#pragma unroll
  for (int s = 0; s < N; ++s) r.d[s] = (gi - base == s) ? 1.0 : 0.0;
  return r;
}

// RotBond VJP by forward-mode duals, NT tangents per pass over the 18 inputs (x1, q1, x2, q2,
// kr, ks, kt, kb): narrow duals keep the law's intermediates in registers.
template <int NT>
__global__ void __launch_bounds__(128) k_adj_bond(const AdjArgs A, int gi) {
  const AdjBond& B = A.bond[gi];
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B.nb) return;
  double4* out = B.gb + 3 * (size_t)b;
  if (B.broken_step[b] <= A.step) {  // removed before this step
    out[0] = out[1] = out[2] = make_double4(0.0, 0.0, 0.0, 0.0);
    return;
  }
  const int2 e = B.ends[b];
  const double4 p1 = A.s0.pr[e.x], p2 = A.s0.pr[e.y], qa = A.s0.qq[e.x], qb = A.s0.qq[e.y];
  const V x1d = xyzv(p1), x2d = image_of(A.g, x1d, xyzv(p2));
  const double4 D0 = B.D0[b];
  const double dist0 = sqrt(D0.x * D0.x + D0.y * D0.y + D0.z * D0.z);
  // p1 gets +force and moment1, p2 gets -force and moment2
  const V lFd = xyzv(A.lF[e.x]) - xyzv(A.lF[e.y]);
  const V lM1 = xyzv(A.lM[e.x]), lM2 = xyzv(A.lM[e.y]);
  double g[18];
#pragma unroll 1
  for (int base = 0; base < 18; base += NT) {
    using DN = Dual<NT>;
    const V3<DN> x1 = mk(seed_in<NT>(x1d.x, 0, base), seed_in<NT>(x1d.y, 1, base), seed_in<NT>(x1d.z, 2, base));
    const Quat<DN> q1{seed_in<NT>(qa.x, 3, base),
                      mk(seed_in<NT>(qa.y, 4, base), seed_in<NT>(qa.z, 5, base), seed_in<NT>(qa.w, 6, base))};
    const V3<DN> x2 = mk(seed_in<NT>(x2d.x, 7, base), seed_in<NT>(x2d.y, 8, base), seed_in<NT>(x2d.z, 9, base));
    const Quat<DN> q2{seed_in<NT>(qb.x, 10, base),
                      mk(seed_in<NT>(qb.y, 11, base), seed_in<NT>(qb.z, 12, base), seed_in<NT>(qb.w, 13, base))};
    const V3<DN> mD = mk(DN(D0.x), DN(D0.y), DN(D0.z));
    const BondKT<DN> K = bond_k_t<DN>(seed_in<NT>(B.kr, 14, base), seed_in<NT>(B.ks, 15, base),
                                      seed_in<NT>(B.kt, 16, base), seed_in<NT>(B.kb, 17, base), B.mn, B.ms, B.mt,
                                      B.mb, B.scaling, B.meanR, dist0, p1.w, p2.w);
    BondOutT<DN> o;
    law_bond_t<DN>(K, mD, x1, p1.w, q1, x2, p2.w, q2, o);
    const DN w = o.force.x * lFd.x + o.force.y * lFd.y + o.force.z * lFd.z + o.moment1.x * lM1.x +
                 o.moment1.y * lM1.y + o.moment1.z * lM1.z + o.moment2.x * lM2.x + o.moment2.y * lM2.y +
                 o.moment2.z * lM2.z;
#pragma unroll
    for (int k = 0; k < NT; ++k)
      if (base + k < 18) g[base + k] = w.d[k];
  }
  // the law depends on x2 - x1 only: d/dx2 = -d/dx1 (not stored)
  out[0] = make_double4(g[0], g[1], g[2], g[3]);
  out[1] = make_double4(g[4], g[5], g[6], g[10]);
  out[2] = make_double4(g[11], g[12], g[13], 0.0);
  double* gp = B.gpar + 4 * (size_t)b;
  gp[0] += g[14];
  gp[1] += g[15];
  gp[2] += g[16];
  gp[3] += g[17];
}


// RotBond VJP by the hand-written reverse of the law (dem_bond_vjp.cuh).
__device__ __forceinline__ void adj_bond_rev_one(const AdjArgs& A, int gi, int b) {
  const AdjBond& B = A.bond[gi];
  double4* out = B.gb + 3 * (size_t)b;
  if (B.broken_step[b] <= A.step) {  // removed before this step
    out[0] = out[1] = out[2] = make_double4(0.0, 0.0, 0.0, 0.0);
    return;
  }
  const int2 e = B.ends[b];
  const double4 p1 = A.s0.pr[e.x], p2 = A.s0.pr[e.y], qa = A.s0.qq[e.x], qb = A.s0.qq[e.y];
  const V x1 = xyzv(p1), x2 = image_of(A.g, x1, xyzv(p2));
  const double4 D0 = B.D0[b];
  const V mD = xyzv(D0);
  const double dist0 = sqrt(D0.x * D0.x + D0.y * D0.y + D0.z * D0.z);
  const BondK K = bond_k(B.kr, B.ks, B.kt, B.kb, B.mn, B.ms, B.mt, B.mb, B.scaling, B.meanR, dist0, p1.w, p2.w);
  const BondK U = bond_k(1.0, 1.0, 1.0, 1.0, B.mn, B.ms, B.mt, B.mb, B.scaling, B.meanR, dist0, p1.w, p2.w);
  const V lFd = xyzv(A.lF[e.x]) - xyzv(A.lF[e.y]);
  const V lM1 = xyzv(A.lM[e.x]), lM2 = xyzv(A.lM[e.y]);
  BondVjp g;
  law_bond_vjp(K, mD, x1, p1.w, Qd{qa.x, mk(qa.y, qa.z, qa.w)}, x2, p2.w, Qd{qb.x, mk(qb.y, qb.z, qb.w)}, lFd, lM1,
               lM2, g);
  // the law depends on x2 - x1 only: d/dx2 = -d/dx1 (not stored)
  out[0] = make_double4(g.x1.x, g.x1.y, g.x1.z, g.q1.s);
  out[1] = make_double4(g.q1.v.x, g.q1.v.y, g.q1.v.z, g.q2.s);
  out[2] = make_double4(g.q2.v.x, g.q2.v.y, g.q2.v.z, 0.0);
  double* gp = B.gpar + 4 * (size_t)b;  // the scaled stiffness is the group's times a constant factor
  gp[0] += g.kr * U.kr;
  gp[1] += g.ks * U.ks;
  gp[2] += g.kt * U.kt;
  gp[3] += g.kb * U.kb;
}

__global__ void __launch_bounds__(128, 3) k_adj_bond_rev(const AdjArgs A, int gi) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < A.bond[gi].nb) adj_bond_rev_one(A, gi, b);
}

using D7 = Dual<7>;
using D23 = Dual<23>;

__device__ __forceinline__ V3<D23> seed3(const V& a, int k) {
  return mk(D23::seed(a.x, k), D23::seed(a.y, k + 1), D23::seed(a.z, k + 2));
}
__device__ __forceinline__ D23 dotd(const V3<D23>& a, const V& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// DUALS selects the VJP form at compile time: the dual-number form's registers would otherwise
// set the hand-written form's occupancy too.
template <bool DUALS>
__device__ __forceinline__ void adj_pair_one(const AdjArgs& A, int gi, int k) {
  const AdjDyn& G = A.dyn[gi];
  const unsigned long long key = G.keys[k];
  const int s1 = (int)(key >> 32), s2 = (int)(key & 0xffffffffu);
  // Record of a touching pair: (d/dx1, d/dv1.x), (d/dv1.yz, d/dw1.xy), (d/dw1.z, d/dw2); the laws
  // depend on x1 - x2 and v1 - v2 only, so d/dx2 = -d/dx1 and d/dv2 = -d/dv1.  gact[k] = 0 marks a
  // pair with nothing to gather (not touching, or held by its excluding bond): no record written.
  double4* out = G.gpair + 3 * (size_t)k;
  G.gact[k] = 0;
  if (G.xbond) {  // a pair skipped by the step while its excluding bond holds
    const int xb = G.xbond[k];
    if (xb >= 0 && A.bond[xb >> 28].broken_step[xb & 0x0fffffff] > A.step) {
      if (G.kind == 1) G.lH[k] = make_double4(0.0, 0.0, 0.0, 0.0);
      return;
    }
  }
  const double4 pa = A.s0.pr[s1], pb = A.s0.pr[s2];
  const V x1d = xyzv(pa), x2d = image_of(A.g, x1d, xyzv(pb));
  const V lF1 = xyzv(A.lF[s1]), lF2 = xyzv(A.lF[s2]);
  if (!DUALS) {  // hand-written reverse of the law (dem_pair_vjp.cuh), the default
    if (G.kind == 0) {
      ElasticVjp e;
      law_elastic_vjp(elastic_k(G.k, G.scaling, pa.w, pb.w), x1d, pa.w, x2d, pb.w, lF2 - lF1, e);
      if (!e.touching) return;
      out[0] = d4(e.x1, 0.0);
      G.gact[k] = 1;
      G.gpar[2 * (size_t)k] += e.k_eff * elastic_k(1.0, G.scaling, pa.w, pb.w);  // k_eff = k x factor
      return;
    }
    double4 h;
    if (G.hist32_in) {
      const float4 f = G.hist32_in[k];
      h = make_double4(f.x, f.y, f.z, f.w);
    } else {
      h = G.hist_in[k];
    }
    double keff, kseff, uk, uks;
    friction_k(G.k, G.ks, G.scaling, G.meanR, pa.w, pb.w, keff, kseff);
    friction_k(1.0, 1.0, G.scaling, G.meanR, pa.w, pb.w, uk, uks);
    const V lH = xyzv(G.lH[k]);
    const V lM1 = xyzv(A.lM[s1]), lM2 = xyzv(A.lM[s2]);
    FricVjp f;
    law_friction_vjp(keff, kseff, G.mu_s, G.mu_d, G.dt, x1d, pa.w, xyzv(A.s0.vm[s1]), xyzv(A.s0.wi[s1]), x2d, pb.w,
                     xyzv(A.s0.vm[s2]), xyzv(A.s0.wi[s2]), xyzv(h), (((int)h.w) & 1) != 0, lF2 - lF1,
                     lF1 - lF2 + lH, lM1, lM2, f);
    if (!f.touching) {  // the history is reset: nothing flows back through it
      G.lH[k] = make_double4(0.0, 0.0, 0.0, 0.0);
      return;
    }
    out[0] = make_double4(f.x1.x, f.x1.y, f.x1.z, f.v1.x);
    out[1] = make_double4(f.v1.y, f.v1.z, f.w1.x, f.w1.y);
    out[2] = make_double4(f.w1.z, f.w2.x, f.w2.y, f.w2.z);
    G.gact[k] = 1;
    G.lH[k] = d4(f.H, 0.0);
    G.gpar[2 * (size_t)k] += f.k_eff * uk;
    G.gpar[2 * (size_t)k + 1] += f.ks_eff * uks;
    return;
  }
  if (G.kind == 0) {
    // CElasticInteraction: p2 gets F, p1 gets -F
    const V3<D7> x1 = mk(D7::seed(x1d.x, 0), D7::seed(x1d.y, 1), D7::seed(x1d.z, 2));
    const V3<D7> x2 = mk(D7::seed(x2d.x, 3), D7::seed(x2d.y, 4), D7::seed(x2d.z, 5));
    const D7 keff = elastic_k_t<D7>(D7::seed(G.k, 6), G.scaling, pa.w, pb.w);
    V3<D7> F;
    if (!law_elastic_t<D7>(keff, x1, pa.w, x2, pb.w, F)) return;
    const V l = lF2 - lF1;
    const D7 w = F.x * l.x + F.y * l.y + F.z * l.z;
    out[0] = make_double4(w.d[0], w.d[1], w.d[2], 0.0);
    G.gact[k] = 1;
    G.gpar[2 * (size_t)k] += w.d[6];
    return;
  }
  // CRotFrictionInteraction
  double4 h;
  if (G.hist32_in) {
    const float4 f = G.hist32_in[k];
    h = make_double4(f.x, f.y, f.z, f.w);
  } else {
    h = G.hist_in[k];
  }
  const V lH = xyzv(G.lH[k]);
  const V3<D23> x1 = seed3(x1d, 0), x2 = seed3(x2d, 3);
  const V3<D23> v1 = seed3(xyzv(A.s0.vm[s1]), 6), v2 = seed3(xyzv(A.s0.vm[s2]), 9);
  const V3<D23> w1 = seed3(xyzv(A.s0.wi[s1]), 12), w2 = seed3(xyzv(A.s0.wi[s2]), 15);
  const V3<D23> H = seed3(xyzv(h), 18);
  D23 keff, kseff;
  friction_k_t<D23>(D23::seed(G.k, 21), D23::seed(G.ks, 22), G.scaling, G.meanR, pa.w, pb.w, keff, kseff);
  FricOutT<D23> o;
  law_friction_t<D23>(keff, kseff, G.mu_s, G.mu_d, G.dt, x1, pa.w, v1, w1, x2, pb.w, v2, w2, H,
                      (((int)h.w) & 1) != 0, o);
  if (!o.touching) {  // the history is reset: nothing flows back through it
    G.lH[k] = make_double4(0.0, 0.0, 0.0, 0.0);
    return;
  }
  // p1 gets -fn + Ffric and M1, p2 gets fn - Ffric and M2; the next history is Ffric
  const V lM1 = xyzv(A.lM[s1]), lM2 = xyzv(A.lM[s2]);
  const D23 w = dotd(o.fn, lF2 - lF1) + dotd(o.Ffric, lF1 - lF2 + lH) + dotd(o.M1, lM1) + dotd(o.M2, lM2);
  out[0] = make_double4(w.d[0], w.d[1], w.d[2], w.d[6]);
  out[1] = make_double4(w.d[7], w.d[8], w.d[12], w.d[13]);
  out[2] = make_double4(w.d[14], w.d[15], w.d[16], w.d[17]);
  G.gact[k] = 1;
  G.lH[k] = make_double4(w.d[18], w.d[19], w.d[20], 0.0);
  G.gpar[2 * (size_t)k] += w.d[21];
  G.gpar[2 * (size_t)k + 1] += w.d[22];
}

template <bool DUALS>
__global__ void __launch_bounds__(128, DUALS ? 1 : 4) k_adj_pair(const AdjArgs A, int gi) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < A.dyn[gi].m) adj_pair_one<DUALS>(A, gi, k);
}

__device__ __forceinline__ void adj_post_one(const AdjArgs& A, int i) {
  if (!(A.pflags[i] & PF_ALIVE)) return;
  double4 gx = make_double4(0.0, 0.0, 0.0, 0.0), gv = gx, gw = gx, gq = gx;
  for (int d = 0; d < A.ndyn; ++d) {
    const AdjDyn& G = A.dyn[d];
    for (int e = G.adj_start[i]; e < G.adj_start[i + 1]; ++e) {
      const int2 en = G.adj[e];
      const int k = en.y & kAdjIndex;
      if (!G.gact[k]) continue;
      const double4* r = G.gpair + 3 * (size_t)k;
      const double4 r0 = r[0];
      const double sg = en.y < 0 ? 1.0 : -1.0;  // this particle is p1 (d/dx1) or p2 (d/dx2 = -d/dx1)
      gx.x += sg * r0.x; gx.y += sg * r0.y; gx.z += sg * r0.z;
      if (G.kind == 1) {
        const double4 r1 = r[1], r2 = r[2];
        gv.x += sg * r0.w; gv.y += sg * r1.x; gv.z += sg * r1.y;
        if (en.y < 0) { gw.x += r1.z; gw.y += r1.w; gw.z += r2.x; }
        else { gw.x += r2.y; gw.y += r2.z; gw.z += r2.w; }
      }
    }
  }
  for (int d = 0; d < A.nbond; ++d) {
    const AdjBond& B = A.bond[d];
    for (int e = B.adj_start[i]; e < B.adj_start[i + 1]; ++e) {
      const int2 en = B.adj[e];
      const int k = en.y & 0x7fffffff;
      const double4* r = B.gb + 3 * (size_t)k;
      const double4 r0 = r[0], r1 = r[1];
      if (en.y < 0) {  // p1: d/dx1, d/dq1
        gx.x += r0.x; gx.y += r0.y; gx.z += r0.z;
        gq.x += r0.w; gq.y += r1.x; gq.z += r1.y; gq.w += r1.z;
      } else {         // p2: d/dx2 = -d/dx1, d/dq2
        const double4 r2 = r[2];
        gx.x -= r0.x; gx.y -= r0.y; gx.z -= r0.z;
        gq.x += r1.w; gq.y += r2.x; gq.z += r2.y; gq.w += r2.z;
      }
    }
  }
  double4 t = A.lx[i];
  A.lx[i] = make_double4(t.x + gx.x, t.y + gx.y, t.z + gx.z, 0.0);
  t = A.lv[i];
  A.lv[i] = make_double4(t.x + gv.x, t.y + gv.y, t.z + gv.z, 0.0);
  if (A.rot) {
    t = A.lw[i];
    A.lw[i] = make_double4(t.x + gw.x, t.y + gw.y, t.z + gw.z, 0.0);
    t = A.lq[i];
    A.lq[i] = make_double4(t.x + gq.x, t.y + gq.y, t.z + gq.z, t.w + gq.w);
  }
}

__global__ void k_adj_post(const AdjArgs A) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < A.n) adj_post_one(A, i);
}

// acc[c] += sum over rows r of data[r * cols + c], in a fixed order (one block).
__global__ void k_reduce_cols(const double* data, int rows, int cols, double* acc) {
  __shared__ double red[32];
  for (int c = 0; c < cols; ++c) {
    double s = 0.0;
    for (int r = threadIdx.x; r < rows; r += blockDim.x) s += data[(size_t)r * cols + c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += red[k];
      acc[c] += t;
    }
    __syncthreads();
  }
}

void launch_adjoint_step(const AdjArgs& A, cudaStream_t s) {
  const int nb = (A.n + 255) / 256;
  if (nb == 0) return;
  k_adj_pre<<<nb, 256, 0, s>>>(A);
  for (int d = 0; d < A.nbond; ++d)
    if (A.bond[d].nb) {
      const int g = (A.bond[d].nb + 127) / 128;
      switch (A.bond_tangents) {  // 0: hand-written reverse; else tangents per dual pass (18 = one pass)
        case 0: k_adj_bond_rev<<<g, 128, 0, s>>>(A, d); break;
        case 3: k_adj_bond<3><<<g, 128, 0, s>>>(A, d); break;
        case 6: k_adj_bond<6><<<g, 128, 0, s>>>(A, d); break;
        case 9: k_adj_bond<9><<<g, 128, 0, s>>>(A, d); break;
        default: k_adj_bond<18><<<g, 128, 0, s>>>(A, d); break;
      }
    }
  for (int d = 0; d < A.ndyn; ++d)
    if (A.dyn[d].m) {
      if (A.pair_duals) k_adj_pair<true><<<(A.dyn[d].m + 127) / 128, 128, 0, s>>>(A, d);
      else k_adj_pair<false><<<(A.dyn[d].m + 127) / 128, 128, 0, s>>>(A, d);
    }
  if (A.nbond || A.ndyn) k_adj_post<<<nb, 256, 0, s>>>(A);
}

void launch_reduce_cols(const double* data, int rows, int cols, double* acc, cudaStream_t s) {
  if (rows > 0) k_reduce_cols<<<1, 1024, 0, s>>>(data, rows, cols, acc);
}

// ---- batched ensemble windows ----------------------------------------------------------

__device__ __forceinline__ ParticleBuf win_view(const WinSpec& w, int j) {
  const size_t n = (size_t)w.n;
  double4* b = w.st + (size_t)j * 4 * n;
  return ParticleBuf{b, b + n, b + 2 * n, b + 3 * n, w.st_vw ? w.st_vw + (size_t)j * 2 * (n > 0 ? n : 1) : nullptr};
}

// One thread per specimen: the base arguments with step j's buffers, and the wall planes
// step j starts from (the recompute moves them through the wall loaders as the forward did).
__global__ void k_window_step_expand(const StepArgs* base, StepArgs* out, const WinSpec* ws, int nspec, int j) {
  const int sp = blockIdx.x * blockDim.x + threadIdx.x;
  if (sp >= nspec) return;
  const WinSpec& w = ws[sp];
  StepArgs a = base[sp];
  const size_t n = (size_t)w.n;
  a.P.buf[0] = win_view(w, j);
  a.P.buf[1] = win_view(w, j + 1);
  a.cur = 0;
  for (int d = 0; d < a.ndyn; ++d) {
    const size_t h = (size_t)w.hstride[d];
    if (w.st_hist32[d]) {
      a.dyn[d].hist32_in = w.st_hist32[d] + j * h;
      a.dyn[d].hist32_out = w.st_hist32[d] + (j + 1) * h;
    } else if (w.st_hist[d]) {
      a.dyn[d].hist_in = w.st_hist[d] + j * h;
      a.dyn[d].hist_out = w.st_hist[d] + (j + 1) * h;
    }
  }
  a.f_int = w.st_f + j * n;
  a.m_int = w.st_m + j * n;
  a.damp_iters = w.st_it + j * 2 * n;
  a.pf_log = w.st_pf ? w.st_pf + j * n : nullptr;
  a.store_forces = 0;
  a.replay = 1;
  a.wall_hist = nullptr;
  out[2 * sp] = a;
  out[2 * sp + 1] = a;
  for (int k = 0; k < w.nwall; ++k) w.st_walls[(size_t)j * kMaxWalls + k] = w.walls[k];
}

__global__ void k_window_adj_expand(const AdjArgs* base, AdjArgs* out, const WinSpec* ws, int nspec, int c, int j) {
  const int sp = blockIdx.x * blockDim.x + threadIdx.x;
  if (sp >= nspec) return;
  const WinSpec& w = ws[sp];
  AdjArgs A = base[sp];
  const size_t n = (size_t)w.n;
  A.step = w.t0 + (long long)c * w.K + j + 1;
  A.s0 = win_view(w, j);
  A.s1 = win_view(w, j + 1);
  A.f_int = w.st_f + j * n;
  A.m_int = w.st_m + j * n;
  A.iters = w.st_it + j * 2 * n;
  A.walls = w.st_walls + (size_t)j * kMaxWalls;
  if (w.st_pf) A.pflags = w.st_pf + j * n;
  A.gR = w.gR + ((size_t)c * w.K + j) * kMaxWalls * 3;
  for (int d = 0; d < A.ndyn; ++d) {
    const size_t h = (size_t)w.hstride[d];
    A.dyn[d].hist_in = w.st_hist[d] ? w.st_hist[d] + j * h : nullptr;
    A.dyn[d].hist32_in = w.st_hist32[d] ? w.st_hist32[d] + j * h : nullptr;
  }
  out[sp] = A;
}

void launch_window_step_expand(const StepArgs* base, StepArgs* out, const WinSpec* ws, int nspec, int j,
                               cudaStream_t s) {
  if (nspec > 0) k_window_step_expand<<<(nspec + 63) / 64, 64, 0, s>>>(base, out, ws, nspec, j);
}
void launch_window_adj_expand(const AdjArgs* base, AdjArgs* out, const WinSpec* ws, int nspec, int c, int j,
                              cudaStream_t s) {
  if (nspec > 0) k_window_adj_expand<<<(nspec + 63) / 64, 64, 0, s>>>(base, out, ws, nspec, c, j);
}

// The item (specimen, or specimen x group) whose tile range holds `tile`: the last item whose
// first tile is <= tile (items without tiles share their successor's first tile).
__device__ __forceinline__ int batch_item(const int* start, int items, int tile) {
  int lo = 0, hi = items;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(start + mid) <= tile) lo = mid; else hi = mid;
  }
  return lo;
}

__global__ void __launch_bounds__(256) k_adj_pre_batch(const AdjBatch B) {
  for (int tile = blockIdx.x; tile < B.total_ptiles; tile += gridDim.x) {
    const int sp = batch_item(B.ptile_start, B.nspec, tile);
    const AdjArgs& A = B.args[sp];
    const int i = (tile - __ldg(B.ptile_start + sp)) * 256 + threadIdx.x;
    if (i < A.n) adj_pre_one(A, i);
  }
}

__global__ void __launch_bounds__(256) k_adj_post_batch(const AdjBatch B) {
  for (int tile = blockIdx.x; tile < B.total_ptiles; tile += gridDim.x) {
    const int sp = batch_item(B.ptile_start, B.nspec, tile);
    const AdjArgs& A = B.args[sp];
    const int i = (tile - __ldg(B.ptile_start + sp)) * 256 + threadIdx.x;
    if (i < A.n) adj_post_one(A, i);
  }
}

__global__ void __launch_bounds__(128, 3) k_adj_bond_rev_batch(const AdjBatch B) {
  for (int tile = blockIdx.x; tile < B.total_btiles; tile += gridDim.x) {
    const int it = batch_item(B.btile_start, B.nspec * kMaxBond, tile);
    const int sp = it / kMaxBond, gi = it % kMaxBond;
    const AdjArgs& A = B.args[sp];
    const int b = (tile - __ldg(B.btile_start + it)) * 128 + threadIdx.x;
    if (gi < A.nbond && b < A.bond[gi].nb) adj_bond_rev_one(A, gi, b);
  }
}

template <bool DUALS>
__global__ void __launch_bounds__(128, DUALS ? 1 : 4) k_adj_pair_batch(const AdjBatch B) {
  for (int tile = blockIdx.x; tile < B.total_dtiles; tile += gridDim.x) {
    const int it = batch_item(B.dtile_start, B.nspec * kMaxDyn, tile);
    const int sp = it / kMaxDyn, gi = it % kMaxDyn;
    const AdjArgs& A = B.args[sp];
    const int k = (tile - __ldg(B.dtile_start + it)) * 128 + threadIdx.x;
    if (gi < A.ndyn && k < A.dyn[gi].m) adj_pair_one<DUALS>(A, gi, k);
  }
}

// Grids of one tile per block up to a cap; the kernels stride over any remainder.
static inline int batch_grid(int tiles) { return tiles < 1048576 ? tiles : 1048576; }

void launch_adjoint_step_batch(const AdjBatch& B, bool bonds, bool pairs, cudaStream_t s) {
  if (B.total_ptiles <= 0) return;
  k_adj_pre_batch<<<batch_grid(B.total_ptiles), 256, 0, s>>>(B);
  if (bonds && B.total_btiles > 0) k_adj_bond_rev_batch<<<batch_grid(B.total_btiles), 128, 0, s>>>(B);
  if (pairs && B.total_dtiles > 0) {
    if (B.pair_duals) k_adj_pair_batch<true><<<batch_grid(B.total_dtiles), 128, 0, s>>>(B);
    else k_adj_pair_batch<false><<<batch_grid(B.total_dtiles), 128, 0, s>>>(B);
  }
  if (bonds || pairs) k_adj_post_batch<<<batch_grid(B.total_ptiles), 256, 0, s>>>(B);
}

}  // namespace dem
