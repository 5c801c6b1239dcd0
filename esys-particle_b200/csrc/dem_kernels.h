// Launch wrappers of the DEM kernels (dem_kernels.cu), called by the host
// simulation object (dem_sim.cu).  All launches are asynchronous on stream s.
#pragma once
#include "dem_device.cuh"

namespace dem {

void launch_scan(const int* in, int* out, int n, int* total, int* tmp, cudaStream_t s);
int scan_tmp_ints(int n);
void launch_bin(const Grid& g, const Particles& P, int cur, int* cell_count, cudaStream_t s);
void launch_scatter_cells(const Particles& P, const int* cell_start, int* cursor, int* cell_list, cudaStream_t s);
void launch_sort_cells(int ncell, const int* cell_start, int* cell_list, cudaStream_t s);
void launch_pairs_count(const Grid& g, const Particles& P, int cur, const int* cs, const int* cl, const ExclDev& ex,
                        int* count, cudaStream_t s);
template <class H>
void launch_pairs_write(const Grid& g, const Particles& P, int cur, const int* cs, const int* cl, const ExclDev& ex,
                        const int* start, unsigned long long* keys, int kind, const unsigned long long* old_keys,
                        int old_n, const H* old_hist, H* hist, cudaStream_t s);
void launch_adj(const unsigned long long* keys, int m, int n, int* adj_count, int* p1_start, int* adj_start,
                int* adj_cursor, int2* adj, int* total, int* tmp, cudaStream_t s);
void launch_newlist_count(const Grid& g, const Particles& P, const int* cs, const int* cl, const ExclDev& ex,
                          const unsigned long long* keys, int m, int check_in, int* count, cudaStream_t s);
void launch_newlist_write(const Grid& g, const Particles& P, const int* cs, const int* cl, const ExclDev& ex,
                          const unsigned long long* keys, int m, int check_in, const int* start,
                          unsigned long long* out, cudaStream_t s);
template <class H>
void launch_merge(const unsigned long long* A, const H* Ah, int m, const unsigned long long* B, int nb,
                  unsigned long long* out, H* outh, int kind, cudaStream_t s);
void launch_sync_vw(const Particles& P, int cur, cudaStream_t s);
void launch_hist_convert(int m, const double4* d, float4* f, bool to_f32, cudaStream_t s);
void launch_clear_flags(int n, unsigned char* flagged, cudaStream_t s);
void launch_pairs_alive(const unsigned long long* keys, int m, const unsigned* pflags, int* keep, cudaStream_t s);
void launch_compact(const unsigned long long* keys, const double4* hist, int m, const int* keep, const int* pos,
                    unsigned long long* okeys, double4* ohist, int kind, cudaStream_t s);
void launch_bonds_rebuild(int nb, const int2* ends, const unsigned* pflags, int* broken_step, cudaStream_t s);
void launch_bonds_init(int nb, const int2* ends, const double4* pr, double4* D0, cudaStream_t s);
void launch_wall_update(const Grid& g, const Particles& P, int cur, int nwall, const WallDev* walls, int* ncand,
                        cudaStream_t s);
void launch_set_state(const Particles& P, int cur, int cnt, const int* slots, const double* pos, const double* vel,
                      const double* angvel, const double* quat, cudaStream_t s);
void launch_alive_flags(const Particles& P, int* flags, cudaStream_t s);
void launch_set_alive(const Particles& P, int cnt, const int* slots, cudaStream_t s);
void launch_pack_particles(const Particles& P, int cur, int rot, const int* rows, int* id, double* pos, double* vel,
                           double* angvel, double* quat, double* force, double* moment, cudaStream_t s);
void launch_check_disp(const Particles& P, int cur, double half_alpha_sq, int* ctrl, cudaStream_t s);
void launch_move_tagged(const Particles& P, int cur, int tag, const double* d, cudaStream_t s);
// idx: scratch of at least P.n ints (each servo thread's candidate list)
void launch_wall_servo(const Particles& P, int cur, int w, WallDev* walls, const double* F, int* idx, cudaStream_t s);
void launch_pairs_xbond(const unsigned long long* keys, int m, const ExclDev& ex, int* xbond, cudaStream_t s);
void launch_adj_mark_held(int ne, const int* xbond, int2* adj, cudaStream_t s);
void launch_count_candidates(int n, const unsigned* pflags, int* ncand, cudaStream_t s);
void launch_particle_field(const Particles& P, int cur, int rot, int field, double* out, cudaStream_t s);
void launch_particle_vector_field(const Particles& P, int cur, int field, const double* initpos, double* out,
                                  cudaStream_t s);
void launch_pair_field(const Grid& g, const Particles& P, int prev, const unsigned long long* keys, int m, int kind,
                       double k, double ks, int scaling, int meanR, const double4* hist, const float4* hist32,
                       int field, double* out, cudaStream_t s);
void launch_bond_field(const Grid& g, const Particles& P, int prev, long long t, const BondDev& B, int nb, int field,
                       double* out, cudaStream_t s);
int step_grid(int n, int tpp);
void launch_step(const StepArgs& a, bool rot, int tpp, bool split, cudaStream_t s);
void launch_bond_pass_f64(const StepArgs& a, bool eval, cudaStream_t s);
void launch_step_fp32(const StepArgs& a, bool rot, int tpp, bool eval, bool split, cudaStream_t s);

// batched ensemble (dem_batch.cu, dem_batch_fp32.cu)
void launch_batch_step(const BatchArgs& B, bool rot, bool el, bool fr, bool bd, bool gather, int tpp, cudaStream_t s);
void launch_batch_step_fp32(const BatchArgs& B, bool rot, bool el, bool fr, bool bd, bool gather, int tpp,
                            cudaStream_t s);
void launch_batch_bond_pass(const BatchArgs& B, cudaStream_t s);
void launch_batch_reset(const StepArgs* args, int nspec, cudaStream_t s);
void launch_batch_status(const StepArgs* args, int nspec, long long* t, int* ctrl, cudaStream_t s);
void launch_batch_sync_vw(const StepArgs* args, const int* base_cur, int nspec, cudaStream_t s);

}  // namespace dem
