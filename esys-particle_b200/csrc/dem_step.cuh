// The timestep kernel k_step, shared by the FP64 form (dem_kernels.cu, built
// with --fmad=false) and the FP32-force form (dem_step_fp32.cu).
//
// One launch = one CLatticeMaster::runOneStep force + integration phase for all
// particles (TSubLattice::zeroForces / calcForces / integrate,
// Parallel/SubLattice.hpp:2066-2236) plus the neighbour check of the next step
// (checkNeighbors, :2473-2519).
//
// Template parameters:
//   ROT   RotSphere (CRotParticle) vs NRotSphere (CParticle)
//   TPP   lanes per particle (1, 2, 4, 8): they stride over the particle's
//         adjacency and combine with a fixed-order butterfly
//   FEAT  interaction families compiled in (F_ELASTIC, F_FRIC, F_BOND)
//   FP32  pair forces in FP32 (positions, contact detection, overlap and
//         integration in FP64; Kahan-compensated FP32 accumulation)
//   EVAL  FP32 evaluation-only pass: forces of the current state into
//         force_eval / moment_eval, nothing else written (precision check)
#pragma once
#include <map>
#include <mutex>

#include "dem_common.cuh"
#include "dem_laws.cuh"
#include "dem_laws_f32.cuh"

namespace dem {

template <int TPP>
__device__ __forceinline__ double lane_sum(double v) {
#pragma unroll
  for (int o = 1; o < TPP; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
template <int TPP>
__device__ __forceinline__ float lane_sumf(float v) {
#pragma unroll
  for (int o = 1; o < TPP; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
template <int TPP>
__device__ __forceinline__ V lane_sum(V v) {
  return mk(lane_sum<TPP>(v.x), lane_sum<TPP>(v.y), lane_sum<TPP>(v.z));
}
template <int TPP>
__device__ __forceinline__ Vf lane_sumf(Vf v) {
  return mk(lane_sumf<TPP>(v.x), lane_sumf<TPP>(v.y), lane_sumf<TPP>(v.z));
}

constexpr int kStepThreads = 256;
constexpr int kStepWarps = kStepThreads / 32;
#ifndef DEM_FP32_BLOCKS
#define DEM_FP32_BLOCKS 3
#endif
constexpr int kFp32Blocks = DEM_FP32_BLOCKS;  // resident blocks per SM targeted by the FP32 pair instances
// Adjacency entries each lane of the pair loop fetches before using them.
#ifndef DEM_KBATCH
#define DEM_KBATCH 1
#endif
// 1: the fused step runs one persistent wave of blocks striding over the particle tiles;
// 0: one block per tile, the hardware scheduler balancing blocks across the SMs.
#ifndef DEM_STEP_PERSISTENT
#define DEM_STEP_PERSISTENT 1
#endif
// 1: the fused step is launched as a programmatic dependent of the stream's previous kernel.
#ifndef DEM_STEP_PDL
#define DEM_STEP_PDL 1
#endif
// 1: while a tile is processed, the records of the block's next tile are prefetched into L2.
#ifndef DEM_STEP_PREFETCH_NEXT
#define DEM_STEP_PREFETCH_NEXT 0
#endif

// Lanes per particle of a threads_per_particle setting, in units of kStepThreads per tile:
// the tiled kernels (kTiled, dem_tiled.cuh) give each particle one thread of a block of
// kTileThreads, i.e. a tile of kTileThreads particles.
__host__ __device__ __forceinline__ int tile_lanes(int tpp) {
  return tpp == kTiled ? kStepThreads / kTileThreads : (tpp == kWarpCoop ? 1 : tpp);
}

__host__ __device__ __forceinline__ int step_tiles(int n, int tpp) {
  tpp = tile_lanes(tpp);
  long long t = (long long)(n > 0 ? n : 1) * tpp;
  return (int)((t + kStepThreads - 1) / kStepThreads);
}

// Interaction families compiled into a k_step instance (the host picks the
// smallest instance that covers the groups present, so a friction-only run
// does not carry the registers of the bond law).
// F_BGATHER: bonds were evaluated by the bond pass (k_bond_pass, once per bond); the particle
// gathers their forces and moments in its adjacency order instead of evaluating the law.
// F_NFRIC: NRotFriction and HertzMindlin groups (FP64 only).
// F_STRESS: each particle's stress sum (CParticle::m_sigma) is accumulated and stored in a.sig
// (BrittleBeamSC groups read it in their failure test).
enum : int { F_ELASTIC = 1, F_FRIC = 2, F_BOND = 4, F_BGATHER = 8, F_NFRIC = 16, F_STRESS = 32 };

// Instances the warp-cooperative pair sums cover: the dynamic groups' contact laws (Elastic,
// RotFriction) with gathered bond records; the widened laws, in-line bonds and stress sums keep
// the lane loop.
template <int FEAT>
struct WarpCoopSupported {
  static constexpr bool value = (FEAT & (F_NFRIC | F_BOND | F_STRESS)) == 0;
};

// Device bond hand-off: whether adjacency entry .y = ey of group G is skipped at this step
// because the intact bond that excluded its pair when the list was built still holds.  Only
// bond failures set Particles::flagged, and under the hand-off nothing clears it while a list
// stands, so a particle whose flag is clear still has every bond the list's exclusions name and
// only a flagged one reads the bond's failure step.  A failure in the current step keeps its
// pair held until the next step whether or not its flag is seen set.
// Instances without bond groups (FEAT without F_BOND / F_BGATHER) hold no pair and carry none of this.
template <int FEAT>
__device__ __forceinline__ bool handoff_held(const StepArgs& a, const DynDev& G, int ey, bool self_flagged,
                                             long long step) {
  if constexpr ((FEAT & (F_BOND | F_BGATHER)) == 0) return false;
  if (!G.xbond || !(ey & kAdjHeld)) return false;
  if (!self_flagged) return true;
  const int xb = __ldg(G.xbond + (ey & kAdjIndex));
  return a.bond[xb >> 28].broken_step[xb & 0x0fffffff] > step;
}

// The flag that handoff_held takes for particle i (read only under the hand-off).
template <int FEAT>
__device__ __forceinline__ bool handoff_flag(const StepArgs& a, int i) {
  if constexpr ((FEAT & (F_BOND | F_BGATHER)) == 0) return false;
  return a.handoff && a.P.flagged[i] != 0;
}

// CParticle::applyForce's stress update (Model/Particle.cpp:392-401): m_sigma(i,j) -= f[i] * (pos - x)[j].
__device__ __forceinline__ void stress_add(double* S, const V& f, const V& pos, const V& x) {
  const V r = pos - x;
  const double fv[3] = {f.x, f.y, f.z}, rv[3] = {r.x, r.y, r.z};
#pragma unroll
  for (int p = 0; p < 3; ++p)
#pragma unroll
    for (int q = 0; q < 3; ++q) S[3 * p + q] -= fv[p] * rv[q];
}

// Sum of the pair-group and bond contributions on particle i (all TPP lanes of
// the particle call this; on return every lane holds the combined sums).  The
// order is fixed: each lane adds its entries in adjacency order, then a
// butterfly combines the lanes.
template <bool ROT, int TPP, int FEAT, bool FP32, bool EVAL>
__device__ __forceinline__ void pair_sums(const StepArgs& a, const ParticleBuf& in, int i, int lane, bool alive,
                                          long long step, const double4& p4, const double4& q4, V& Fp, V& Mp,
                                          double* gross = nullptr, double* stress = nullptr) {
  constexpr bool STRESS = !FP32 && (FEAT & F_STRESS) != 0;
  Fp = mk(0.0, 0.0, 0.0);
  Mp = mk(0.0, 0.0, 0.0);
  double Gs = 0.0;  // evaluation pass: sum of the contributions' magnitudes (the particle's force scale)
  // 3. dynamic pair groups (PIS_NE / PIS_ED::calcForces).  Contact is tested first from the
  //    positions alone; the partner's velocity / spin and the pair's history are gathered only
  //    for touching pairs (a non-touching RotFriction pair just resets its history).  Each lane
  //    takes one adjacency entry per pass (kBatch = 1); the gathers in flight come from the TPP
  //    lanes of a particle and the warps resident on the SM, not from batching within a thread.
  //    kBatch > 1 would fetch that many entries and partner positions per lane before use.
  KSum3 Fk, Mk;                                      // FP32 form
  Fk.zero();
  Mk.zero();
  if ((FEAT & (F_ELASTIC | F_FRIC | F_NFRIC)) && alive) {
    constexpr int kBatch = DEM_KBATCH;
    Vf vself = mk(0.f, 0.f, 0.f), wself = vself;
    double4 v4 = make_double4(0.0, 0.0, 0.0, 0.0), w4 = v4;
    if (FP32) {
      if (ROT && (FEAT & F_FRIC)) {  // the FP32 form's velocity and spin: the FP64 records rounded
        const double4 a0 = ldg4(in.vm + i), a1 = ldg4(in.wi + i);
        vself = mk((float)a0.x, (float)a0.y, (float)a0.z);
        wself = mk((float)a1.x, (float)a1.y, (float)a1.z);
      }
    } else if (FEAT & (F_FRIC | F_NFRIC)) {
      v4 = ldg4(in.vm + i);
      if (ROT) w4 = ldg4(in.wi + i);
    }
    const bool flg = handoff_flag<FEAT>(a, i);
    for (int d = 0; d < a.ndyn; ++d) {
      const DynDev& G = a.dyn[d];
      const int e0 = __ldg(G.adj_start + i), e1 = __ldg(G.adj_start + i + 1);
      for (int e = e0 + lane; e < e1; e += TPP * kBatch) {
        int2 en[kBatch];
        double4 pjs[kBatch];
#pragma unroll
        for (int b = 0; b < kBatch; ++b) {
          const int eb = e + b * TPP;
          en[b] = eb < e1 ? __ldg(G.adj + eb) : make_int2(-1, 0);
        }
        // device bond hand-off: a pair is skipped while the bond that excluded it holds, and its
        // partner record is not fetched
        bool held[kBatch];
#pragma unroll
        for (int b = 0; b < kBatch; ++b) held[b] = en[b].x >= 0 && handoff_held<FEAT>(a, G, en[b].y, flg, step);
#pragma unroll
        for (int b = 0; b < kBatch; ++b)
          pjs[b] = (en[b].x >= 0 && !held[b]) ? ldg4(in.pr + en[b].x) : make_double4(0.0, 0.0, 0.0, 0.0);
#pragma unroll
        for (int b = 0; b < kBatch; ++b) {
          if (en[b].x < 0) continue;
          const int j = en[b].x;
          const bool isp1 = en[b].y < 0;
          const int k = en[b].y & kAdjIndex;
          if (held[b]) {
            if (isp1 && !EVAL) {
              if (FP32) G.hist32_out[k] = make_float4(0.f, 0.f, 0.f, 0.f);
              else G.hist_out[k] = make_double4(0.0, 0.0, 0.0, 0.0);
            }
            continue;
          }
          const double4 pj = pjs[b];
          // canonical orientation: p1 = lower id
          const double4 pa = isp1 ? p4 : pj, pb = isp1 ? pj : p4;
          const V x1 = xyz(pa), x2 = image_of(a.g, x1, xyz(pb));
          const V D = x1 - x2;
          const double eq_dist = pa.w + pb.w;
          const bool touching = dot(D, D) < (eq_dist * eq_dist);  // the laws' contact test
          if (G.kind == 0) {
            if constexpr ((FEAT & F_ELASTIC) != 0) {
              if (!touching) continue;
              if constexpr (!FP32) {
                V f;
                if (law_elastic(elastic_k(G.k, G.scaling, pa.w, pb.w), x1, pa.w, x2, pb.w, f)) {
                  if (isp1) Fp += -1.0 * f; else Fp += f;
                  if constexpr (STRESS) {  // CElasticInteraction::calcForces: at x2 + r2 / (r1 + r2) D
                    const V pos = x2 + (pb.w / eq_dist) * D;
                    stress_add(stress, isp1 ? -1.0 * f : f, pos, isp1 ? x1 : x2);
                  }
                }
              } else {
                Vf f;
                if (law_elastic_f32(elastic_k(G.k, G.scaling, pa.w, pb.w), D, pa.w, pb.w, f)) {
                  Fk.add(isp1 ? -f : f);
                  if (EVAL) Gs += (double)norm(f);
                }
              }
            }
          } else if (G.kind >= 2) {
            // NRotFriction (CFrictionInteraction::calcForces) or HertzMindlin
            // (CHertzMindlinInteraction::calcForces): forces only, history of the tangential force
            if constexpr (!FP32 && (FEAT & F_NFRIC) != 0) {
              if (!touching) {
                if (isp1 && !EVAL) G.hist_out[k] = make_double4(0.0, 0.0, 0.0, 0.0);
                continue;
              }
              const double4 vj = ldg4(in.vm + j);
              const double4 va = isp1 ? v4 : vj, vb = isp1 ? vj : v4;
              const double4 h = ldg4(G.hist_in + k);
              FricOut o;
              if (G.kind == 2) {
                double keff, kseff;
                nfriction_k(G.k, G.ks, G.scaling, pa.w, pb.w, keff, kseff);
                law_nfriction(keff, kseff, G.mu_s, G.dt, x1, pa.w, xyz(va), x2, pb.w, xyz(vb), mk(h.x, h.y, h.z), o);
              } else if (G.kind == 3) {  // E in k, nu in ks; the normal force on p1 is +fn: negated for the common form
                law_hertz_mindlin(G.k, G.ks, G.mu_s, G.dt, x1, pa.w, xyz(va), x2, pb.w, xyz(vb), mk(h.x, h.y, h.z), o);
                o.fn = -1.0 * o.fn;
              } else {  // HertzMindlinVisco: E, nu, mu, restitution in k, ks, mu_s, mu_d; masses in the w's
                law_hertz_mindlin_visco(G.k, G.ks, G.mu_s, G.mu_d, G.dt, x1, pa.w, va.w, xyz(va), x2, pb.w, vb.w, xyz(vb),
                                        o);
                o.fn = -1.0 * o.fn;
              }
              if constexpr (STRESS) {
                const V pos = x2 + (pb.w / eq_dist) * D;
                const V xs = isp1 ? x1 : x2;
                stress_add(stress, isp1 ? -1.0 * o.fn : o.fn, pos, xs);
                stress_add(stress, isp1 ? o.Ffric : -1.0 * o.Ffric, pos, xs);
              }
              if (isp1) {  // p1: -force, then +Ffric; p2: +force, then -Ffric
                Fp += -1.0 * o.fn;
                Fp += o.Ffric;
                if (!EVAL)
                  G.hist_out[k] = make_double4(o.Ffric.x, o.Ffric.y, o.Ffric.z,
                                               (o.slipping ? 1.0 : 0.0) + (o.touching ? 2.0 : 0.0));
              } else {
                Fp += o.fn;
                Fp += -1.0 * o.Ffric;
              }
              if (EVAL) Gs += norm(o.fn) + norm(o.Ffric);
            }
          } else {
            if constexpr (ROT && (FEAT & F_FRIC) != 0) {
              if (!touching) {  // CRotFrictionInteraction::calcSimpleForces, no-contact branch
                if (isp1 && !EVAL) {
                  if (FP32) G.hist32_out[k] = make_float4(0.f, 0.f, 0.f, 0.f);
                  else G.hist_out[k] = make_double4(0.0, 0.0, 0.0, 0.0);
                }
                continue;
              }
              double keff, kseff;
              friction_k(G.k, G.ks, G.scaling, G.meanR, pa.w, pb.w, keff, kseff);
              if constexpr (!FP32) {
                const double4 vj = ldg4(in.vm + j), wj = ldg4(in.wi + j);
                const double4 va = isp1 ? v4 : vj, vb = isp1 ? vj : v4;
                const double4 wa = isp1 ? w4 : wj, wb = isp1 ? wj : w4;
                const double4 h = ldg4(G.hist_in + k);
                FricOut o;
                law_friction(keff, kseff, G.mu_s, G.mu_d, G.dt, x1, pa.w, xyz(va), xyz(wa), x2, pb.w, xyz(vb),
                             xyz(wb), mk(h.x, h.y, h.z), (((int)h.w) & 1) != 0, o);
                if constexpr (STRESS) {  // CRotFrictionInteraction::calcSimpleForces: both forces at the contact
                  const V pos = x2 + (pb.w / eq_dist) * D;
                  const V xs = isp1 ? x1 : x2;
                  stress_add(stress, isp1 ? -1.0 * o.fn : o.fn, pos, xs);
                  stress_add(stress, isp1 ? o.Ffric : -1.0 * o.Ffric, pos, xs);
                }
                if (isp1) {
                  Fp += -1.0 * o.fn;
                  Mp += o.M1;
                  Fp += o.Ffric;
                  G.hist_out[k] = make_double4(o.Ffric.x, o.Ffric.y, o.Ffric.z,
                                               (o.slipping ? 1.0 : 0.0) + (o.touching ? 2.0 : 0.0));
                } else {
                  Fp += o.fn;
                  Mp += o.M2;
                  Fp += -1.0 * o.Ffric;
                }
              } else {
                const double4 b0 = ldg4(in.vm + j), b1 = ldg4(in.wi + j);
                const Vf vj = mk((float)b0.x, (float)b0.y, (float)b0.z), wj = mk((float)b1.x, (float)b1.y, (float)b1.z);
                Vf hF;
                bool hs;
                if (EVAL) {  // evaluation pass of an FP64 run: its FP64 history
                  const double4 h = ldg4(G.hist_in + k);
                  hF = mk((float)h.x, (float)h.y, (float)h.z);
                  hs = (((int)h.w) & 1) != 0;
                } else {
                  const float4 h = __ldg(G.hist32_in + k);
                  hF = mk(h.x, h.y, h.z);
                  hs = (((int)h.w) & 1) != 0;
                }
                FricOutF o;
                law_friction_f32(keff, kseff, G.mu_s, G.mu_d, (float)G.dt, D, pa.w, pb.w, isp1 ? vself : vj,
                                 isp1 ? wself : wj, isp1 ? vj : vself, isp1 ? wj : wself, hF, hs, o);
                if (isp1) {
                  Fk.add(-o.fn);
                  Fk.add(o.Ffric);
                  Mk.add(o.M1);
                  if (EVAL) Gs += (double)norm(o.fn) + (double)norm(o.Ffric);
                  if (!EVAL)
                    G.hist32_out[k] = make_float4(o.Ffric.x, o.Ffric.y, o.Ffric.z,
                                                  (o.slipping ? 1.f : 0.f) + (o.touching ? 2.f : 0.f));
                } else {
                  Fk.add(o.fn);
                  Fk.add(-o.Ffric);
                  Mk.add(o.M2);
                  if (EVAL) Gs += (double)norm(o.fn) + (double)norm(o.Ffric);
                }
              }
            }
          }
        }
      }
    }
  }

  // 4. bonded groups (PIS_EB::calcForces) + failure test (PIS_EB::update at the next step)
  if constexpr ((FEAT & F_BGATHER) != 0) {
    if (alive) {
      for (int d = 0; d < a.nbond; ++d) {
        const BondDev& B = a.bond[d];
        const int e0 = __ldg(B.adj_start + i), e1 = __ldg(B.adj_start + i + 1);
        for (int e = e0 + lane; e < e1; e += TPP) {
          const int2 en = __ldg(B.adj + e);
          const int k = en.y & 0x7fffffff;
          // a bond removed by an earlier update carries zero records (bond_pass_one writes them)
          if constexpr (FP32 && !EVAL) {
            const float4* rf = B.bf32 + 4 * (size_t)k + (en.y < 0 ? 0 : 2);
            const float4 a0 = __ldg(rf), a1 = __ldg(rf + 1);
            Fp += mk((double)a0.x, (double)a0.y, (double)a0.z);
            if (ROT) Mp += mk((double)a0.w, (double)a1.x, (double)a1.y);
            continue;
          }
          const double4* r = B.bf + 3 * (size_t)k;
          if (en.y < 0) {
            Fp += xyz(ldg4(r));
            if (ROT) Mp += xyz(ldg4(r + 1));
          } else {
            Fp += -1.0 * xyz(ldg4(r));
            if (ROT) Mp += xyz(ldg4(r + 2));
          }
          if constexpr (STRESS) {  // bonds apply their force at x2 + r2 / (r1 + r2) (x1 - x2)
            const double4 pj = ldg4(in.pr + en.x);
            const bool isp1 = en.y < 0;
            const double4 pa = isp1 ? p4 : pj, pb = isp1 ? pj : p4;
            const V x1 = xyz(pa), x2 = image_of(a.g, x1, xyz(pb));
            const V pos = x2 + (pb.w / (pa.w + pb.w)) * (x1 - x2);
            const V f1 = xyz(ldg4(r));
            stress_add(stress, isp1 ? f1 : -1.0 * f1, pos, isp1 ? x1 : x2);
          }
          if (EVAL) Gs += norm(xyz(ldg4(r)));
        }
      }
    }
  }
  if constexpr (ROT && (FEAT & F_BOND) != 0) {
    if (alive) {
      for (int d = 0; d < a.nbond; ++d) {
        const BondDev& B = a.bond[d];
        const int e0 = __ldg(B.adj_start + i), e1 = __ldg(B.adj_start + i + 1);
        for (int e = e0 + lane; e < e1; e += TPP) {
          const int2 en = __ldg(B.adj + e);
          const int k = en.y & 0x7fffffff;
          if (B.broken_step[k] <= step) continue;  // removed by an earlier update
          const int j = en.x;
          const bool isp1 = en.y < 0;
          const double4 pj = ldg4(in.pr + j), qj = ldg4(in.qq + j);
          const double4 pa = isp1 ? p4 : pj, pb = isp1 ? pj : p4;
          const double4 qa = isp1 ? q4 : qj, qb = isp1 ? qj : q4;
          const V x1 = xyz(pa), x2 = image_of(a.g, x1, xyz(pb));
          const double4 D0 = ldg4(B.D0 + k);
          const V mD = xyz(D0);
          const double dist0 = sqrt(dot(mD, mD));
          const BondK K = bond_k(B.kr, B.ks, B.kt, B.kb, B.mn, B.ms, B.mt, B.mb, B.scaling, B.meanR, dist0, pa.w, pb.w);
          BondOut o;
          law_bond(K, mD, x1, pa.w, Qd{qa.x, mk(qa.y, qa.z, qa.w)}, x2, pb.w, Qd{qb.x, mk(qb.y, qb.z, qb.w)}, o);
          if (EVAL) Gs += norm(o.force);
          if (isp1) {
            Fp += o.force;
            Mp += o.moment1;
            const bool brk = B.kind == 2   ? dzc_broken(o, dist0, B.cohesion, B.tan_angle, B.t_cutoff, B.c_cutoff,
                                                        B.beta1, B.beta2)
                             : B.kind == 3 ? false
                                           : bond_broken(K, o, B.truncated);
            if (!EVAL && brk) {
              B.broken_step[k] = (int)(step + 1);
              a.P.flagged[i] = 1;
              a.P.flagged[j] = 1;
              if (!a.replay) {
                int slot = atomicAdd(B.nevents, 1);
                if (slot < B.cap_events) {
                  B.events[3 * slot] = a.P.id[i];
                  B.events[3 * slot + 1] = a.P.id[j];
                  B.events[3 * slot + 2] = (int)(step + 1);
                } else {
                  atomicOr(a.ctrl, CTRL_OVERFLOW);
                }
                atomicOr(a.ctrl, CTRL_BROKE);
              }
              if (a.handoff) a.brk_step[step & 1] = (int)step;
            }
          } else {
            Fp += -1.0 * o.force;
            Mp += o.moment2;
          }
        }
      }
    }
  }

  if (TPP > 1) {
    if (FP32) {
      Fk.s = lane_sumf<TPP>(Fk.s);
      Fk.c = lane_sumf<TPP>(Fk.c);
      Mk.s = lane_sumf<TPP>(Mk.s);
      Mk.c = lane_sumf<TPP>(Mk.c);
    }
    Fp = lane_sum<TPP>(Fp);
    Mp = lane_sum<TPP>(Mp);
    if (EVAL) Gs = lane_sum<TPP>(Gs);
    if constexpr (STRESS) {
#pragma unroll
      for (int c = 0; c < 9; ++c) stress[c] = lane_sum<TPP>(stress[c]);
    }
  }
  if (FP32) {
    // FP64-form sums (bonds) are added after the compensated FP32 pair sums
    Fp = Fk.value() + Fp;
    Mp = Mk.value() + Mp;
  }
  if (EVAL && gross) *gross = Gs;
}

// Warp-cooperative pair sums (threads_per_particle = kWarpCoop), for the particle layout of
// TPP = 1: one thread per particle, 32 consecutive particle slots per warp.  The warp's
// adjacency entries of a group are one contiguous range of the CSR (the particles' ranges in
// lane order); the warp takes them 32 at a time, one entry per lane, so the adjacency reads
// are coalesced and each lane has one partner gather in flight per batch however the entries
// are spread over the particles (a lane of the one-lane loop walks its own particle's entries
// one dependent gather after another, and its warp waits for the longest list).  The owner of
// an entry is the last lane whose range starts at or before it.  A touching entry's
// contributions go to the owner's lane in entry order (lanes in order within a batch, batches
// in order), so every particle adds the contributions the one-lane loop adds, in the same
// order: the sums are those of TPP = 1.
template <bool ROT, int FEAT, bool FP32, bool EVAL>
__device__ __forceinline__ void pair_sums_warp(const StepArgs& a, const ParticleBuf& in, int i, bool valid, bool alive,
                                               long long step, const double4& p4, V& Fp, V& Mp, double* gross) {
  static_assert(WarpCoopSupported<FEAT>::value, "instance outside the warp-cooperative pair sums");
  constexpr unsigned kFull = 0xffffffffu;
  const int wl = threadIdx.x & 31;
  Fp = mk(0.0, 0.0, 0.0);
  Mp = mk(0.0, 0.0, 0.0);
  double Gs = 0.0;
  KSum3 Fk, Mk;
  Fk.zero();
  Mk.zero();
  if constexpr ((FEAT & (F_ELASTIC | F_FRIC)) != 0) {
    // the owner-side records the friction law reads (as the one-lane loop loads them)
    Vf vself = mk(0.f, 0.f, 0.f), wself = vself;
    double4 v4 = make_double4(0.0, 0.0, 0.0, 0.0), w4 = v4;
    if (ROT && (FEAT & F_FRIC) && alive) {
      v4 = ldg4(in.vm + i);
      w4 = ldg4(in.wi + i);
      if (FP32) {  // the FP32 form's velocity and spin: the FP64 records rounded
        vself = mk((float)v4.x, (float)v4.y, (float)v4.z);
        wself = mk((float)w4.x, (float)w4.y, (float)w4.z);
      }
    }
    const int flg = valid && alive && handoff_flag<FEAT>(a, i) ? 1 : 0;
    for (int d = 0; d < a.ndyn; ++d) {
      const DynDev& G = a.dyn[d];
      int s0 = valid ? __ldg(G.adj_start + i) : 0;
      const int s1 = valid ? __ldg(G.adj_start + i + 1) : 0;
      const int w1 = __reduce_max_sync(kFull, s1);
      if (!valid) s0 = w1;  // lanes past the last particle: empty ranges at the warp's end
      const int w0 = __reduce_min_sync(kFull, s0);
      for (int base = w0; base < w1; base += 32) {
        const int e = base + wl;
        const bool has = e < w1;
        int o = 0;  // owner lane: the last lane whose range starts at or before e
#pragma unroll
        for (int st = 16; st > 0; st >>= 1) {
          const int sv = __shfl_sync(kFull, s0, o + st);
          if (sv <= e) o += st;
        }
        const int oi = __shfl_sync(kFull, i, o);
        const bool oalive = __shfl_sync(kFull, (int)alive, o) != 0;
        const bool oflg = __shfl_sync(kFull, flg, o) != 0;
        const double4 po = make_double4(__shfl_sync(kFull, p4.x, o), __shfl_sync(kFull, p4.y, o),
                                        __shfl_sync(kFull, p4.z, o), __shfl_sync(kFull, p4.w, o));
        const bool act = has && oalive;
        const int2 en = act ? __ldg(G.adj + e) : make_int2(-1, 0);
        const int j = en.x;
        const bool isp1 = en.y < 0;
        const int k = en.y & kAdjIndex;
        bool live = act;
        if (act && handoff_held<FEAT>(a, G, en.y, oflg, step)) {  // device bond hand-off
          if (isp1 && !EVAL) {
            if (FP32) G.hist32_out[k] = make_float4(0.f, 0.f, 0.f, 0.f);
            else G.hist_out[k] = make_double4(0.0, 0.0, 0.0, 0.0);
          }
          live = false;
        }
        const double4 pj = live ? ldg4(in.pr + j) : make_double4(0.0, 0.0, 0.0, 0.0);
        // canonical orientation: p1 = lower id
        const double4 pa = isp1 ? po : pj, pb = isp1 ? pj : po;
        const V x1 = xyz(pa), x2 = image_of(a.g, x1, xyz(pb));
        const V D = x1 - x2;
        const double eq_dist = pa.w + pb.w;
        const bool touching = live && dot(D, D) < (eq_dist * eq_dist);  // the laws' contact test
        if (live && !touching && G.kind == 1 && isp1 && !EVAL) {  // CRotFrictionInteraction: no-contact branch
          if (FP32) G.hist32_out[k] = make_float4(0.f, 0.f, 0.f, 0.f);
          else G.hist_out[k] = make_double4(0.0, 0.0, 0.0, 0.0);
        }
        if (!__any_sync(kFull, touching)) continue;
        // the owner's velocity and spin for the friction law
        Vf vo = vself, wo = wself;
        double4 vo4 = v4, wo4 = w4;
        if (ROT && (FEAT & F_FRIC)) {
          if (FP32) {
            vo = mk(__shfl_sync(kFull, vself.x, o), __shfl_sync(kFull, vself.y, o), __shfl_sync(kFull, vself.z, o));
            wo = mk(__shfl_sync(kFull, wself.x, o), __shfl_sync(kFull, wself.y, o), __shfl_sync(kFull, wself.z, o));
          } else {
            vo4 = make_double4(__shfl_sync(kFull, v4.x, o), __shfl_sync(kFull, v4.y, o), __shfl_sync(kFull, v4.z, o), 0.0);
            wo4 = make_double4(__shfl_sync(kFull, w4.x, o), __shfl_sync(kFull, w4.y, o), __shfl_sync(kFull, w4.z, o), 0.0);
          }
        }
        // this entry's contributions to its owner, in the order the one-lane loop adds them:
        // forces c0 then c1 (c1 only for friction), moment cm
        int nf = 0;
        bool hm = false;
        V c0 = mk(0.0, 0.0, 0.0), c1 = c0, cm = c0;
        Vf f0 = mk(0.f, 0.f, 0.f), f1 = f0, fm = f0;
        double g = 0.0;
        if (touching) {
          if (G.kind == 0) {
            if constexpr ((FEAT & F_ELASTIC) != 0) {
              if constexpr (!FP32) {
                V f;
                if (law_elastic(elastic_k(G.k, G.scaling, pa.w, pb.w), x1, pa.w, x2, pb.w, f)) {
                  c0 = isp1 ? -1.0 * f : f;
                  nf = 1;
                }
              } else {
                Vf f;
                if (law_elastic_f32(elastic_k(G.k, G.scaling, pa.w, pb.w), D, pa.w, pb.w, f)) {
                  f0 = isp1 ? -f : f;
                  nf = 1;
                  if (EVAL) g = (double)norm(f);
                }
              }
            }
          } else {
            if constexpr (ROT && (FEAT & F_FRIC) != 0) {
              double keff, kseff;
              friction_k(G.k, G.ks, G.scaling, G.meanR, pa.w, pb.w, keff, kseff);
              if constexpr (!FP32) {
                const double4 vj = ldg4(in.vm + j), wj = ldg4(in.wi + j);
                const double4 va = isp1 ? vo4 : vj, vb = isp1 ? vj : vo4;
                const double4 wa = isp1 ? wo4 : wj, wb = isp1 ? wj : wo4;
                const double4 h = ldg4(G.hist_in + k);
                FricOut fo;
                law_friction(keff, kseff, G.mu_s, G.mu_d, G.dt, x1, pa.w, xyz(va), xyz(wa), x2, pb.w, xyz(vb),
                             xyz(wb), mk(h.x, h.y, h.z), (((int)h.w) & 1) != 0, fo);
                if (isp1) {
                  c0 = -1.0 * fo.fn;
                  c1 = fo.Ffric;
                  cm = fo.M1;
                  if (!EVAL)
                    G.hist_out[k] = make_double4(fo.Ffric.x, fo.Ffric.y, fo.Ffric.z,
                                                 (fo.slipping ? 1.0 : 0.0) + (fo.touching ? 2.0 : 0.0));
                } else {
                  c0 = fo.fn;
                  c1 = -1.0 * fo.Ffric;
                  cm = fo.M2;
                }
                nf = 2;
                hm = true;
              } else {
                const double4 b0 = ldg4(in.vm + j), b1 = ldg4(in.wi + j);
                const Vf vj = mk((float)b0.x, (float)b0.y, (float)b0.z), wj = mk((float)b1.x, (float)b1.y, (float)b1.z);
                Vf hF;
                bool hs;
                if (EVAL) {  // evaluation pass of an FP64 run: its FP64 history
                  const double4 h = ldg4(G.hist_in + k);
                  hF = mk((float)h.x, (float)h.y, (float)h.z);
                  hs = (((int)h.w) & 1) != 0;
                } else {
                  const float4 h = __ldg(G.hist32_in + k);
                  hF = mk(h.x, h.y, h.z);
                  hs = (((int)h.w) & 1) != 0;
                }
                FricOutF fo;
                law_friction_f32(keff, kseff, G.mu_s, G.mu_d, (float)G.dt, D, pa.w, pb.w, isp1 ? vo : vj,
                                 isp1 ? wo : wj, isp1 ? vj : vo, isp1 ? wj : wo, hF, hs, fo);
                if (isp1) {
                  f0 = -fo.fn;
                  f1 = fo.Ffric;
                  fm = fo.M1;
                  if (!EVAL)
                    G.hist32_out[k] = make_float4(fo.Ffric.x, fo.Ffric.y, fo.Ffric.z,
                                                  (fo.slipping ? 1.f : 0.f) + (fo.touching ? 2.f : 0.f));
                } else {
                  f0 = fo.fn;
                  f1 = -fo.Ffric;
                  fm = fo.M2;
                }
                nf = 2;
                hm = true;
                if (EVAL) g = (double)norm(fo.fn) + (double)norm(fo.Ffric);
              }
            }
          }
        }
        // deliver, source lanes in order
        unsigned m = __ballot_sync(kFull, nf > 0);
        while (m) {
          const int src = __ffs(m) - 1;
          m &= m - 1;
          const int dst = __shfl_sync(kFull, o, src);
          const int snf = __shfl_sync(kFull, nf, src);
          const bool shm = __shfl_sync(kFull, (int)hm, src) != 0;
          if constexpr (FP32) {
            const Vf a0 = mk(__shfl_sync(kFull, f0.x, src), __shfl_sync(kFull, f0.y, src), __shfl_sync(kFull, f0.z, src));
            const Vf a1 = mk(__shfl_sync(kFull, f1.x, src), __shfl_sync(kFull, f1.y, src), __shfl_sync(kFull, f1.z, src));
            const Vf am = mk(__shfl_sync(kFull, fm.x, src), __shfl_sync(kFull, fm.y, src), __shfl_sync(kFull, fm.z, src));
            const double ag = EVAL ? __shfl_sync(kFull, g, src) : 0.0;
            if (wl == dst) {
              Fk.add(a0);
              if (snf > 1) Fk.add(a1);
              if (shm) Mk.add(am);
              if (EVAL) Gs += ag;
            }
          } else {
            const V a0 = mk(__shfl_sync(kFull, c0.x, src), __shfl_sync(kFull, c0.y, src), __shfl_sync(kFull, c0.z, src));
            const V a1 = mk(__shfl_sync(kFull, c1.x, src), __shfl_sync(kFull, c1.y, src), __shfl_sync(kFull, c1.z, src));
            const V am = mk(__shfl_sync(kFull, cm.x, src), __shfl_sync(kFull, cm.y, src), __shfl_sync(kFull, cm.z, src));
            if (wl == dst) {
              Fp += a0;
              if (shm) Mp += am;
              if (snf > 1) Fp += a1;
            }
          }
        }
      }
    }
  }

  // bonds evaluated by the bond pass: their records gathered in adjacency order
  if constexpr ((FEAT & F_BGATHER) != 0) {
    if (alive) {
      for (int d = 0; d < a.nbond; ++d) {
        const BondDev& B = a.bond[d];
        const int e0 = __ldg(B.adj_start + i), e1 = __ldg(B.adj_start + i + 1);
        for (int e = e0; e < e1; ++e) {
          const int2 en = __ldg(B.adj + e);
          const int k = en.y & 0x7fffffff;
          if constexpr (FP32 && !EVAL) {
            const float4* rf = B.bf32 + 4 * (size_t)k + (en.y < 0 ? 0 : 2);
            const float4 a0 = __ldg(rf), a1 = __ldg(rf + 1);
            Fp += mk((double)a0.x, (double)a0.y, (double)a0.z);
            if (ROT) Mp += mk((double)a0.w, (double)a1.x, (double)a1.y);
            continue;
          }
          const double4* r = B.bf + 3 * (size_t)k;
          if (en.y < 0) {
            Fp += xyz(ldg4(r));
            if (ROT) Mp += xyz(ldg4(r + 1));
          } else {
            Fp += -1.0 * xyz(ldg4(r));
            if (ROT) Mp += xyz(ldg4(r + 2));
          }
          if (EVAL) Gs += norm(xyz(ldg4(r)));
        }
      }
    }
  }
  if (FP32) {
    // FP64-form sums (bonds) are added after the compensated FP32 pair sums
    Fp = Fk.value() + Fp;
    Mp = Mk.value() + Mp;
  }
  if (EVAL && gross) *gross = Gs;
}

// Walls, body force, the pair sums, damping and the integration of particle i
// (TSubLattice::calcForces group order, then integrate + rescale).  Every thread
// of the block calls this: the wall reactions are reduced across the block.
template <bool ROT, int TPP, bool FP32, bool EVAL>
__device__ __forceinline__ void finish_particle(const StepArgs& a, long long step, const ParticleBuf& in,
                                                const ParticleBuf& out, int i, int lane, int wlane, int warp,
                                                unsigned pf, bool alive,
                                                const double4& p4, double4 q4, bool q_loaded, const V& Fp, const V& Mp,
                                                double (*s_red)[kMaxWalls][3]) {
  double4 v4 = make_double4(0.0, 0.0, 0.0, 0.0), w4 = v4;
  if (alive) {
    v4 = ldg4(in.vm + i);
    if (ROT) w4 = ldg4(in.wi + i);
  }
  const V xi = xyz(p4);
  V F = mk(0.0, 0.0, 0.0), M = mk(0.0, 0.0, 0.0);

  // 0. device bond hand-off: the step after a bond failure refreshes wall candidacy the way
  //    CEWallInteractionGroup::Update does in that step's updateInteractions
  //    (EWallInteractionGroup.hpp:57-82, NeighborTable::getParticlesAtPlane ntable.hpp:674-690)
  if (a.handoff && alive) {
    if (a.brk_step[(step - 1) & 1] == (int)(step - 1)) {
      pf &= ~(0xffffu << PF_WALL_SHIFT);
      const bool inner = inner_of(a.g, p4.x, p4.y, p4.z);
      for (int w = 0; w < a.nwall; ++w) {
        const WallDev W = a.walls[w];
        const double dist = dot(xi - mk(W.ox, W.oy, W.oz), mk(W.nx, W.ny, W.nz));
        if (fabs(dist) < a.g.dim) {
          pf |= 1u << (PF_WALL_SHIFT + w);
          if (inner) pf |= 1u << (PF_INNER_SHIFT + w);
        }
      }
      if (lane == 0 && !EVAL) a.P.pflags[i] = pf;
    }
  }
  if (a.pf_log && lane == 0 && i < a.P.n) a.pf_log[i] = pf;

  // 1. elastic walls, in group-name order (TSubLattice::calcForces, SubLattice.hpp:2116-2120).
  //    The walls' reactions are reduced in a fixed order: warp shuffle, then warps, then blocks.
  for (int w = 0; w < a.nwall; ++w) {
    V c = mk(0.0, 0.0, 0.0);
    if (alive && lane == 0 && (pf & (1u << (PF_WALL_SHIFT + w)))) {
      const WallDev W = a.walls[w];
      V f;
      if (law_wall(W.k, mk(W.ox, W.oy, W.oz), mk(W.nx, W.ny, W.nz), xi, p4.w, f)) {
        F += f;
        if (pf & (1u << (PF_INNER_SHIFT + w))) c = f;  // CWall::addForce(-F): m_force -= -F
      }
    }
    if (!EVAL) {
      double cx = c.x, cy = c.y, cz = c.z;
      if (__any_sync(0xffffffffu, cx != 0.0 || cy != 0.0 || cz != 0.0)) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          cx += __shfl_down_sync(0xffffffffu, cx, o);
          cy += __shfl_down_sync(0xffffffffu, cy, o);
          cz += __shfl_down_sync(0xffffffffu, cz, o);
        }
      }
      if (wlane == 0) { s_red[warp][w][0] += cx; s_red[warp][w][1] += cy; s_red[warp][w][2] += cz; }
    }
  }

  // 2. body forces (BodyForceGroup::calcForces, BodyForceGroup.hpp:54-65): F += g * m
  if (alive && lane == 0)
    for (int k = 0; k < a.ngrav; ++k) F += mk(a.grav[k][0], a.grav[k][1], a.grav[k][2]) * v4.w;

  if (alive && lane == 0) {
    F += Fp;
    M += Mp;
    // 1/m and 1/I as the particle constructors compute them (Particle.cpp:95-99, RotParticle.cpp:35)
    const double2 iv = make_double2(v4.w != 0.0 ? 1.0 / v4.w : 0.0, 1.0 / w4.w);
    if (a.f_int) {
      a.f_int[i] = d4(F, 0.0);
      a.m_int[i] = d4(M, 0.0);
    }
    // 5. damping, last (SubLattice.hpp:2140-2145), in the damping map's name order: on the force
    //    "Damping" and a LocalDamping group (by its own name); on the moment "RotDamping" then
    //    "RotLocalDamping"
    int it_lin = 0, it_rot = 0;
    if (a.damp_loc && a.loc_before_lin) F += local_damping_force(xyz(v4), F, a.visc_loc);
    if (a.damp_lin) F += damping_force(xyz(v4), F, iv.x, v4.w, a.visc_lin, a.dt_lin, a.iter_lin, &it_lin);
    if (a.damp_loc && !a.loc_before_lin) F += local_damping_force(xyz(v4), F, a.visc_loc);
    if (ROT && a.damp_rot) M += damping_force(xyz(w4), M, iv.y, w4.w, a.visc_rot, a.dt_rot, a.iter_rot, &it_rot);
    if (ROT && a.damp_rotloc) M += local_damping_force(xyz(w4), M, a.visc_rotloc);
    if (a.damp_iters) {
      a.damp_iters[2 * i] = (unsigned char)(it_lin > 255 ? 255 : it_lin);
      a.damp_iters[2 * i + 1] = (unsigned char)(it_rot > 255 ? 255 : it_rot);
    }
    if (EVAL) {
      a.P.force_eval[i] = d4(F, 0.0);
      if (ROT) a.P.moment_eval[i] = d4(M, 0.0);
    } else {
      // 6. integration (CRotParticle::integrate + rescale, RotParticle.cpp:277-321; Particle.cpp:257-274)
      const double dt = a.dt;
      V v = xyz(v4), x = xi;
      V w = xyz(w4);
      if (ROT) {
        if (!q_loaded) q4 = ldg4(in.qq + i);
        Qd q{q4.x, mk(q4.y, q4.z, q4.w)};
        if (pf & PF_ROT) {
          w += (dt * iv.y) * M;
          const Qd dq = qmul(Qd{0.0, w}, q);
          const double c = dt / 2.0;
          q.s += c * dq.s;
          q.v += c * dq.v;
        } else {
          w = mk(0.0, 0.0, 0.0);
        }
        const double module = sqrt(q.s * q.s + q.v.x * q.v.x + q.v.y * q.v.y + q.v.z * q.v.z);
        if (module != 0.0) {
          const double inverse = 1.0 / module;
          q.s = inverse * q.s;
          q.v = inverse * q.v;
        }
        out.wi[i] = d4(w, w4.w);
        out.qq[i] = make_double4(q.s, q.v.x, q.v.y, q.v.z);
      }
      if (pf & PF_DYN) {
        v += F * iv.x * dt;
        x += v * dt;
      }
      out.pr[i] = d4(x, p4.w);
      out.vm[i] = d4(v, v4.w);
      if (FP32 && !a.skip_vw) {
        out.vw[2 * i] = make_float4((float)v.x, (float)v.y, (float)v.z, (float)w.x);
        out.vw[2 * i + 1] = make_float4((float)w.y, (float)w.z, 0.f, 0.f);
      }
      if (a.store_forces && (a.force_step < 0 || step == a.force_step)) {
        a.P.force[i] = d4(F, 0.0);
        if (ROT) a.P.moment[i] = d4(M, 0.0);
      }
      // 7. displacement check for the next step (TSubLattice::checkNeighbors): |x - oldpos| >
      //    verletDist/2, evaluated exactly whenever the running bound of it (this step's
      //    displacement added to the bound, in FP32 rounded up) does not already rule it out.
      //    The difference of a position before and after one step is exact (the two are close),
      //    so the bound only has to cover the norm's rounding.
      const V sd = mk(x.x - xi.x, x.y - xi.y, x.z - xi.z);
      const float b = __fadd_ru(a.P.dbound[i], __fmul_ru(__double2float_ru(sqrt(dot(sd, sd))), 1.0000005f));
      a.P.dbound[i] = b;
      if ((double)b * (double)b >= a.half_alpha_sq * 0.999999) {
        const double4 op = ldg4(a.P.oldpos + i);
        const V dd = mk(x.x - op.x, x.y - op.y, x.z - op.z);
        if (dot(dd, dd) > a.half_alpha_sq) atomicOr(a.ctrl, CTRL_REBUILD);
      }
    }
  }
}

// Totals of the wall reactions from the nparts per-block (or per-tile) partials, in
// the last block of a launch: component wc = 3 w + c is summed by warp wc % (warps of the
// block), lane l adding partials l, l + 32, ... in order, then a fixed butterfly; all
// components at once, so the launch's serial tail is one round of loads.
__device__ __forceinline__ void wall_totals(const StepArgs& a, long long step, int nparts, int wlane, int warp) {
  const int nw3 = a.nwall * 3;
  const int nwarps = (int)(blockDim.x >> 5);
  for (int wc = warp; wc < nw3; wc += nwarps) {
    const int w = wc / 3, c = wc % 3;
    double acc = 0.0;
#pragma unroll 4
    for (int b = wlane; b < nparts; b += 32) acc += __ldcg(a.wall_partial + ((size_t)b * kMaxWalls + w) * 3 + c);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (wlane == 0) {
      a.wall_force[3 * w + c] = acc;
      if (a.wall_hist) a.wall_hist[(size_t)(step - a.wall_hist_t0 - 1) * (kMaxWalls * 3) + 3 * w + c] = acc;
    }
  }
}

// This block's wall partials (fixed order over warps) into slot `part`, then the
// last-arriving block of the `nparts` is detected on `counter`.  Returns true in that block.
// All threads of the block call this.
__device__ __forceinline__ bool block_partials(const StepArgs& a, int part, int nparts, unsigned* counter,
                                               double (*s_red)[kMaxWalls][3], bool* s_last) {
  const int nw3 = a.nwall * 3;
  __syncthreads();
  if (threadIdx.x < nw3) {
    const int w = threadIdx.x / 3, c = threadIdx.x % 3;
    double acc = 0.0;
    for (int k = 0; k < kStepWarps; ++k) acc += s_red[k][w][c];
    a.wall_partial[((size_t)part * kMaxWalls + w) * 3 + c] = acc;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();  // the block's partials and control bits before its arrival
    const unsigned prev = atomicInc(counter, (unsigned)nparts - 1u);
    *s_last = (prev == (unsigned)nparts - 1u);
  }
  __syncthreads();
  if (!*s_last) return false;
  __threadfence();
  return true;
}

// The end of a timestep, run by the last block: wall totals, native wall loaders (one
// thread per wall: origin += v dt, WallLoaderRunnable), the step counter and the stop word.
// The control word is read first, so its load overlaps the totals'.
__device__ __forceinline__ void launch_tail(const StepArgs& a, long long step, int nparts, int wlane, int warp) {
  int ctrl = 0;
  if (threadIdx.x == 0) ctrl = *(volatile int*)a.ctrl;
  wall_totals(a, step, nparts, wlane, warp);
  if ((int)threadIdx.x < a.nwall) {
    const int w = threadIdx.x;
    const double vx = a.wall_vel[3 * w], vy = a.wall_vel[3 * w + 1], vz = a.wall_vel[3 * w + 2];
    if (vx != 0.0 || vy != 0.0 || vz != 0.0) {
      WallDev* W = a.walls + w;
      W->ox += vx * a.dt;
      W->oy += vy * a.dt;
      W->oz += vz * a.dt;
    }
  }
  if (threadIdx.x == 0) {
    *a.step_counter = step;
    if (ctrl & ~a.stop_skip) *a.stop = 1;
  }
}

// Per-block wall reactions, then the last block of the launch finishes the step.  All
// threads of the block call this.
__device__ __forceinline__ void step_epilogue(const StepArgs& a, long long step, int wlane, int warp,
                                              double (*s_red)[kMaxWalls][3], bool* s_last) {
  if (!block_partials(a, blockIdx.x, gridDim.x, a.block_counter, s_red, s_last)) return;
  launch_tail(a, step, gridDim.x, wlane, warp);
}


// Bond pass: bond k of group d evaluated once, in its canonical orientation, for the
// particle pass to gather (F_BGATHER); the failure test and its records as the p1 side of
// the in-line evaluation writes them.  The same law and operation order as in pair_sums,
// so the gathered values equal what either side would compute.
// The bond pass's records of bond k: f the force on p1, m1 / m2 the moments on p1 / p2.
__device__ __forceinline__ void store_bond(const BondDev& B, int k, const V& f, const V& m1, const V& m2) {
  if (B.bf32) {
    float4* r = B.bf32 + 4 * (size_t)k;
    r[0] = make_float4((float)f.x, (float)f.y, (float)f.z, (float)m1.x);
    r[1] = make_float4((float)m1.y, (float)m1.z, 0.f, 0.f);
    r[2] = make_float4((float)(-f.x), (float)(-f.y), (float)(-f.z), (float)m2.x);
    r[3] = make_float4((float)m2.y, (float)m2.z, 0.f, 0.f);
  } else {
    double4* r = B.bf + 3 * (size_t)k;
    r[0] = d4(f, 0.0);
    r[1] = d4(m1, 0.0);
    r[2] = d4(m2, 0.0);
  }
}

template <bool EVAL>
__device__ __forceinline__ void bond_pass_one(const StepArgs& a, const BondDev& B, int k, long long step) {
  if (B.broken_step[k] <= step) {  // removed by an earlier update: zero records, so gathers need no test
    const V z = mk(0.0, 0.0, 0.0);
    store_bond(B, k, z, z, z);
    return;
  }
  const ParticleBuf in = a.P.buf[a.cur];
  const int2 e = __ldg(B.ends + k);
  if (B.kind == 1) {  // NRotBond: force on p2 F, on p1 -F, no moments
    const double4 pa = ldg4(in.pr + e.x), pb = ldg4(in.pr + e.y);
    const V x1 = xyz(pa), x2 = image_of(a.g, x1, xyz(pb));
    V F;
    double dist;
    law_nbond(nbond_k(B.knb, B.scaling, pa.w, pb.w), x1, pa.w, x2, pb.w, F, dist);
    const V z = mk(0.0, 0.0, 0.0);
    store_bond(B, k, -1.0 * F, z, z);
    if (!EVAL && nbond_broken(dist, pa.w, pb.w, B.rbreak)) {
      B.broken_step[k] = (int)(step + 1);
      a.P.flagged[e.x] = 1;
      a.P.flagged[e.y] = 1;
      if (!a.replay) {
        const int slot = atomicAdd(B.nevents, 1);
        if (slot < B.cap_events) {
          B.events[3 * slot] = a.P.id[e.x];
          B.events[3 * slot + 1] = a.P.id[e.y];
          B.events[3 * slot + 2] = (int)(step + 1);
        } else {
          atomicOr(a.ctrl, CTRL_OVERFLOW);
        }
        atomicOr(a.ctrl, CTRL_BROKE);
      }
      if (a.handoff) a.brk_step[step & 1] = (int)step;
    }
    return;
  }
  const double4 pa = ldg4(in.pr + e.x), pb = ldg4(in.pr + e.y);
  const double4 qa = ldg4(in.qq + e.x), qb = ldg4(in.qq + e.y);
  const V x1 = xyz(pa), x2 = image_of(a.g, x1, xyz(pb));
  const double4 D0 = ldg4(B.D0 + k);
  const V mD = xyz(D0);
  const double dist0 = sqrt(dot(mD, mD));
  const BondK K = bond_k(B.kr, B.ks, B.kt, B.kb, B.mn, B.ms, B.mt, B.mb, B.scaling, B.meanR, dist0, pa.w, pb.w);
  BondOut o;
  law_bond(K, mD, x1, pa.w, Qd{qa.x, mk(qa.y, qa.z, qa.w)}, x2, pb.w, Qd{qb.x, mk(qb.y, qb.z, qb.w)}, o);
  store_bond(B, k, o.force, o.moment1, o.moment2);
  // BrittleBeamSC: tested at the update that opens the step (k_sc_check), not on the forces
  const bool brk = B.kind == 2   ? dzc_broken(o, dist0, B.cohesion, B.tan_angle, B.t_cutoff, B.c_cutoff, B.beta1, B.beta2)
                   : B.kind == 3 ? false
                                 : bond_broken(K, o, B.truncated);
  if (!EVAL && brk) {
    const int i = e.x, j = e.y;
    B.broken_step[k] = (int)(step + 1);
    a.P.flagged[i] = 1;
    a.P.flagged[j] = 1;
    if (!a.replay) {
      const int slot = atomicAdd(B.nevents, 1);
      if (slot < B.cap_events) {
        B.events[3 * slot] = a.P.id[i];
        B.events[3 * slot + 1] = a.P.id[j];
        B.events[3 * slot + 2] = (int)(step + 1);
      } else {
        atomicOr(a.ctrl, CTRL_OVERFLOW);
      }
      atomicOr(a.ctrl, CTRL_BROKE);
    }
    if (a.handoff) a.brk_step[step & 1] = (int)step;
  }
}

template <bool EVAL, bool FP32>  // FP32: instance of the FP32-force form's translation unit
__global__ void __launch_bounds__(kBondPassThreads, 4) k_bond_pass(const StepArgs a, int d, int nb) {
  if (!EVAL && *a.stop) return;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nb) return;
  bond_pass_one<EVAL>(a, a.bond[d], k, *a.step_counter + 1);
}

// Fused step: pair sums and integration in one launch (small systems).
template <bool ROT, int TPP, int FEAT, bool FP32, bool EVAL>
__global__ void __launch_bounds__(kStepThreads, (FEAT & F_BOND) ? 1
                                                : ((FEAT & F_NFRIC) ? 2 : ((FEAT & F_BGATHER) ? 4 : (FP32 ? kFp32Blocks : 2))))
    k_step(const StepArgs a) {
  __shared__ double s_red[kStepWarps][kMaxWalls][3];
  __shared__ bool s_last;
  constexpr int LT = TPP == kWarpCoop ? 1 : TPP;  // lanes per particle of the particle's own work
  const int lane = threadIdx.x % LT;
  const int wlane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const ParticleBuf in = a.P.buf[a.cur];
  const ParticleBuf out = a.P.buf[a.cur ^ 1];
  for (int k = threadIdx.x; k < kStepWarps * kMaxWalls * 3; k += kStepThreads) (&s_red[0][0][0])[k] = 0.0;
  // Launched as a programmatic dependent of the previous step (launch_fused): everything the
  // previous step wrote is read after this wait, which returns once that grid has completed.
  grid_dependency_wait();
  __syncthreads();
  if (!EVAL && *a.stop) return;  // an earlier step of this chunk asked the host to intervene
  const long long step = *a.step_counter + 1;
  // Persistent grid: one wave of blocks strides over tiles of kStepThreads / LT particles.
  const int ntiles = step_tiles(a.P.n, TPP);
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int i = (tile * kStepThreads + threadIdx.x) / LT;
    const bool valid = i < a.P.n;
    // All of the particle's own loads are issued at once: the flags and position into
    // registers, the records needed after the pair loop into L1.
    unsigned pf = 0u;
    double4 p4 = make_double4(0, 0, 0, 0), q4 = make_double4(1, 0, 0, 0);
    if (valid) {
      pf = __ldg(a.P.pflags + i);
      p4 = ldg4(in.pr + i);
      if (lane == 0) {
        prefetch_l1(in.vm + i);
        if (ROT) { prefetch_l1(in.wi + i); prefetch_l1(in.qq + i); }
        for (int d = 0; d < a.ndyn; ++d) prefetch_l1(a.dyn[d].adj_start + i);
      }
      if (ROT && (FEAT & F_BOND)) q4 = ldg4(in.qq + i);
    }
#if DEM_STEP_PREFETCH_NEXT
    {  // the records of this thread's particle in the block's next tile, into L2
      const int inext = ((tile + gridDim.x) * kStepThreads + threadIdx.x) / LT;
      if (lane == 0 && inext < a.P.n) {
        if (DEM_STEP_PREFETCH_NEXT == 2) prefetch_l1(in.pr + inext);
        else prefetch_l2(in.pr + inext);
        prefetch_l2(in.vm + inext);
        if (ROT) { prefetch_l2(in.wi + inext); prefetch_l2(in.qq + inext); }
        for (int d = 0; d < a.ndyn; ++d) {
          if (DEM_STEP_PREFETCH_NEXT == 2) prefetch_l1(a.dyn[d].adj_start + inext);
          else prefetch_l2(a.dyn[d].adj_start + inext);
        }
      }
    }
#endif
    const bool alive = valid && (pf & PF_ALIVE);
    V Fp, Mp;
    double gross = 0.0;
    double Sg[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) Sg[c] = 0.0;
    if constexpr (TPP == kWarpCoop)
      pair_sums_warp<ROT, FEAT, FP32, EVAL>(a, in, i, valid, alive, step, p4, Fp, Mp, &gross);
    else
      pair_sums<ROT, TPP, FEAT, FP32, EVAL>(a, in, i, lane, alive, step, p4, q4, Fp, Mp, &gross, Sg);
    finish_particle<ROT, LT, FP32, EVAL>(a, step, in, out, i, lane, wlane, warp, pf, alive, p4, q4,
                                         ROT && (FEAT & F_BOND), Fp, Mp, s_red);
    if constexpr (!FP32 && !EVAL && (FEAT & F_STRESS) != 0) {
      if (alive && lane == 0) {
        const V xi = xyz(p4);
        for (int w = 0; w < a.nwall; ++w) {  // CElasticWallInteraction: at x - dist n
          if (!(pf & (1u << (PF_WALL_SHIFT + w)))) continue;
          const WallDev W = a.walls[w];
          const V o = mk(W.ox, W.oy, W.oz), nrm = mk(W.nx, W.ny, W.nz);
          V f;
          if (law_wall(W.k, o, nrm, xi, p4.w, f)) {
            const double dist = dot(xi - o, nrm);
            stress_add(Sg, f, xi - dist * nrm, xi);
          }
        }
        double* out_s = a.sig + 9 * (size_t)i;
#pragma unroll
        for (int c = 0; c < 9; ++c) out_s[c] = Sg[c];
      }
    }
    // evaluation pass: the particle's contact-force scale beside its force (w of the record)
    if (EVAL && alive && lane == 0) reinterpret_cast<double*>(a.P.force_eval + i)[3] = gross;
  }
  // the next step may start launching once every block is past its tiles (it waits for this
  // grid's completion before reading anything)
  grid_dependents_launch();
  if (EVAL) return;
  step_epilogue(a, step, wlane, warp, s_red, &s_last);
}

// Split step, part 1: pair and bond sums of every particle into P.sum_f / P.sum_m
// (no particle state written besides friction history and bond records).
template <bool ROT, int TPP, int FEAT, bool FP32>
__global__ void __launch_bounds__(kStepThreads, (FEAT & F_BOND) ? 1 : (FP32 ? 3 : 2)) k_pairs(const StepArgs a) {
  if (*a.stop) return;
  const long long step = *a.step_counter + 1;
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) / TPP;
  const int lane = threadIdx.x % TPP;
  const bool valid = i < a.P.n;
  const unsigned pf = valid ? __ldg(a.P.pflags + i) : 0u;
  const bool alive = valid && (pf & PF_ALIVE);
  const ParticleBuf in = a.P.buf[a.cur];
  double4 p4 = make_double4(0, 0, 0, 0), q4 = make_double4(1, 0, 0, 0);
  if (alive) {
    p4 = ldg4(in.pr + i);
    if (ROT && (FEAT & F_BOND)) q4 = ldg4(in.qq + i);
  }
  V Fp, Mp;
  pair_sums<ROT, TPP, FEAT, FP32, false>(a, in, i, lane, alive, step, p4, q4, Fp, Mp);
  if (alive && lane == 0) {
    a.P.sum_f[i] = d4(Fp, 0.0);
    if (ROT) a.P.sum_m[i] = d4(Mp, 0.0);
  }
}

// Split step, part 2: walls, body forces, the stored pair sums, damping,
// integration and the block/launch epilogue; one thread per particle.
template <bool ROT, bool FP32>
__global__ void __launch_bounds__(kStepThreads, 3) k_integrate(const StepArgs a) {
  __shared__ double s_red[kStepWarps][kMaxWalls][3];
  __shared__ bool s_last;
  if (*a.stop) return;
  const long long step = *a.step_counter + 1;
  for (int k = threadIdx.x; k < kStepWarps * kMaxWalls * 3; k += kStepThreads) (&s_red[0][0][0])[k] = 0.0;
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int wlane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool valid = i < a.P.n;
  const unsigned pf = valid ? a.P.pflags[i] : 0u;
  const bool alive = valid && (pf & PF_ALIVE);
  const ParticleBuf in = a.P.buf[a.cur];
  const ParticleBuf out = a.P.buf[a.cur ^ 1];
  double4 p4 = make_double4(0, 0, 0, 0);
  V Fp = mk(0.0, 0.0, 0.0), Mp = Fp;
  if (alive) {
    p4 = ldg4(in.pr + i);
    Fp = xyz(ldg4(a.P.sum_f + i));
    if (ROT) Mp = xyz(ldg4(a.P.sum_m + i));
  }
  finish_particle<ROT, 1, FP32, false>(a, step, in, out, i, 0, wlane, warp, pf, alive, p4, make_double4(1, 0, 0, 0), false,
                                       Fp, Mp, s_red);
  step_epilogue(a, step, wlane, warp, s_red, &s_last);
}

inline int step_blocks(int n, int tpp) {
  tpp = tile_lanes(tpp);
  long long t = (long long)(n > 0 ? n : 1) * tpp;
  return (int)((t + kStepThreads - 1) / kStepThreads);
}

// Blocks of one wave of kernel K on the current device, cached per kernel (every
// instance of k_step shares one function type, so the cache is keyed by address).
template <class K>
inline int one_wave(K kernel, int threads = kStepThreads) {
  static std::mutex mu;
  static std::map<const void*, int> cache;
  std::lock_guard<std::mutex> lock(mu);
  const void* key = reinterpret_cast<const void*>(kernel);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0);
  const int v = (sms > 0 ? sms : 1) * (per_sm > 0 ? per_sm : 1);
  cache[key] = v;
  return v;
}

template <bool R, int FEAT, bool FP32>
inline void launch_split_tpp(const StepArgs& a, int tpp, cudaStream_t s) {
  tpp = tile_lanes(tpp);
  const int grid = step_blocks(a.P.n, tpp);
  switch (tpp) {
    case 1: k_pairs<R, 1, FEAT, FP32><<<grid, kStepThreads, 0, s>>>(a); break;
    case 2: k_pairs<R, 2, FEAT, FP32><<<grid, kStepThreads, 0, s>>>(a); break;
    case 4: k_pairs<R, 4, FEAT, FP32><<<grid, kStepThreads, 0, s>>>(a); break;
    default: k_pairs<R, 8, FEAT, FP32><<<grid, kStepThreads, 0, s>>>(a); break;
  }
  k_integrate<R, FP32><<<step_blocks(a.P.n, 1), kStepThreads, 0, s>>>(a);
}

template <bool R, int T, int FEAT, bool FP32, bool EVAL>
inline void launch_fused(const StepArgs& a, cudaStream_t s) {
  const int tiles = step_blocks(a.P.n, T);
#if DEM_STEP_PERSISTENT
  const int wave = one_wave(k_step<R, T, FEAT, FP32, EVAL>);
  const int grid = tiles < wave ? tiles : wave;
#else
  const int grid = tiles;
#endif
#if DEM_STEP_PDL
  // programmatic dependent launch: the step's blocks are scheduled while the previous kernel
  // of the stream finishes (its last block's epilogue), and wait in grid_dependency_wait
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kStepThreads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, k_step<R, T, FEAT, FP32, EVAL>, a);
#else
  k_step<R, T, FEAT, FP32, EVAL><<<grid, kStepThreads, 0, s>>>(a);
#endif
}

template <bool EVAL, bool FP32>
inline void launch_bond_pass(const StepArgs& a, cudaStream_t s) {
  for (int d = 0; d < a.nbond; ++d) {
    const int nb = a.bond[d].nb_launch;
    if (nb > 0)
      k_bond_pass<EVAL, FP32><<<(nb + kBondPassThreads - 1) / kBondPassThreads, kBondPassThreads, 0, s>>>(a, d, nb);
  }
}

}  // namespace dem
