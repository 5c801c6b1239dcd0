// Arguments of the reverse step of the differentiable window (dem_adjoint.cu).
#pragma once
#include "dem_device.cuh"

namespace dem {

// One dynamic group (NRotElastic or RotFriction) in the reverse step.
struct AdjDyn {
  int kind;  // 0 elastic, 1 rot friction
  double k, ks, mu_s, mu_d, dt;
  int scaling, meanR;
  int m;                              // pairs (frozen over the window)
  const unsigned long long* keys;     // (p1 slot << 32) | p2 slot, p1 = lower id
  const int* adj_start;               // per-particle adjacency over the pairs
  const int2* adj;
  const double4* hist_in;             // friction history read by this step (forward recompute)
  const float4* hist32_in;            // the same when the window runs the FP32-force form
  const int* xbond;                   // device bond hand-off: excluding bond of each pair (else null)
  double4* lH;                        // adjoint of the history: in after step t, out before it
  double4* gpair;                     // [m][3]: d/dx1, d/dv1, d/dw1, d/dw2 of this step, packed (d/dx2 = -d/dx1,
                                      // d/dv2 = -d/dv1)
  unsigned char* gact;                // [m]: 1 when this step's record was written (a touching pair)
  double* gpar;                       // [m][2]: d/dk, d/dks accumulated over the window
};

// One RotBond group in the reverse step.
struct AdjBond {
  double kr, ks, kt, kb, mn, ms, mt, mb;
  int scaling, meanR;
  int nb;
  const int2* ends;                   // (p1 slot, p2 slot)
  const double4* D0;
  const int* broken_step;
  const int* adj_start;
  const int2* adj;
  double4* gb;                        // [nb][3]: d/dx1, d/dq1, d/dq2 of this step, packed (d/dx2 = -d/dx1)
  double* gpar;                       // [nb][4]: d/dkr, d/dks, d/dkt, d/dkb accumulated
};

struct AdjArgs {
  Grid g;
  int n;
  int rot;
  double dt;
  long long step;                     // timestep number of the step being reversed (1-based)
  const unsigned* pflags;
  ParticleBuf s0;                     // state before the step
  ParticleBuf s1;                     // state after the step
  const double4* f_int;               // force / moment sums before damping (forward recompute)
  const double4* m_int;
  const unsigned char* iters;         // damping iterations (lin, rot) per particle
  int damp_lin, damp_rot, iter_lin, iter_rot;
  double visc_lin, visc_rot, dt_lin, dt_rot;
  int nwall;
  const WallDev* walls;               // wall planes during the step
  const double* gR;                   // [kMaxWalls][3]: dLoss / d(reaction of each wall group) at this step
  double4 *lx, *lv, *lw, *lq;         // state adjoint: in lambda_{t+1}, out lambda_t
  double4 *lF, *lM;                   // adjoint of the force / moment sums before damping
  double* gvisc;                      // [n][2]: d/d(linear, rotational viscosity) accumulated
  int ndyn;
  AdjDyn dyn[kMaxDyn];
  int nbond;
  AdjBond bond[kMaxBond];
  int bond_tangents;                  // RotBond VJP: 0 hand-written reverse, else dual tangents per pass (3, 6, 9, 18)
  int pair_duals;                     // pair-law VJPs: 0 hand-written reverse, 1 forward-mode duals
};

void launch_adjoint_step(const AdjArgs& A, cudaStream_t s);

// ---- batched ensemble windows: every specimen's reverse step in one launch per kernel ----
// One specimen's window buffers, indexed by the step j of the segment being reversed.
struct WinSpec {
  int n;                          // particles
  int K;                          // checkpoint interval
  long long t0;                   // step counter at the window's start
  double4* st;                    // [K + 1][4 n] recomputed states (pr, vm, wi, qq blocks)
  float4* st_vw;                  // [K + 1][2 n] FP32 velocity shadows (FP32 form, else null)
  double4* st_f;                  // [K][n] pre-damping force sums
  double4* st_m;                  // [K][n] pre-damping moment sums
  unsigned char* st_it;           // [K][2 n] damping iterations
  WallDev* st_walls;              // [K][kMaxWalls] wall planes during each step
  unsigned* st_pf;                // [K][n] wall candidacy per step (bond failures inside the window, else null)
  double4* st_hist[kMaxDyn];      // [K + 1][hstride] friction histories (FP64 form)
  float4* st_hist32[kMaxDyn];     // the same in the FP32 form
  int hstride[kMaxDyn];           // max(pairs, 1)
  const double* gR;               // [T][kMaxWalls][3] loss gradient of the reactions
  const WallDev* walls;           // live wall planes (their state before each recomputed step)
  int nwall;
};

struct AdjBatch {
  int nspec;
  const AdjArgs* args;            // [nspec]: this step's reverse arguments
  const int* ptile_start;         // [nspec + 1]: particle tiles of 256
  int total_ptiles;
  const int* btile_start;         // [nspec * kMaxBond + 1]: bond tiles of 128 per (specimen, group)
  int total_btiles;
  const int* dtile_start;         // [nspec * kMaxDyn + 1]: pair tiles of 128 per (specimen, group)
  int total_dtiles;
  int pair_duals;                 // pair-law VJPs by forward-mode duals (else hand-written), as AdjArgs
};

// Step j's recompute arguments (both buffer parities) and wall planes, from each specimen's base.
void launch_window_step_expand(const StepArgs* base, StepArgs* out, const WinSpec* ws, int nspec, int j,
                               cudaStream_t s);
// Step j of segment c's reverse arguments, from each specimen's base.
void launch_window_adj_expand(const AdjArgs* base, AdjArgs* out, const WinSpec* ws, int nspec, int c, int j,
                              cudaStream_t s);
void launch_adjoint_step_batch(const AdjBatch& B, bool bonds, bool pairs, cudaStream_t s);
void launch_reduce_cols(const double* data, int rows, int cols, double* acc, cudaStream_t s);

}  // namespace dem
