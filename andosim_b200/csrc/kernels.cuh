// kernels.cuh -- kernel entry points of the step (definitions in kernels.cu / pcg.cu).
#pragma once

#include "common.cuh"

namespace ando {

struct RigidDev {
  int nv, nt;
  const double* local;  // 3nv
  const int* tris;      // 3nt
  double* world;        // 3nv (written per step)
  double pos[3], R[9], Iinv_body[9], mass, lin[3], ang[3];
};

// setup
void launch_elastic_slots(const MeshDev& m, double mu, double thickness, int semantics, double* el_a, double* el_b, cudaStream_t s);
void launch_elastic_gradient(const MeshDev& m, const double* mesh_vertices, double mu, double thickness, double* g_el, cudaStream_t s);
void launch_arap_gradient(const MeshDev& m, const double* X, double mu, double thickness, double* g, cudaStream_t s);
// per face: the data of the projected exact membrane Hessian at X (MFACE doubles each)
void launch_membrane_face(const MeshDev& m, const double* X, double mu, double thickness, double* out, cudaStream_t s);

// per step
void launch_predict(int V, const double* x, const double* v, double dt, double* x_old, double* x_hat, cudaStream_t s);
void launch_gravity(int V, double* x, double* v, double gx, double gy, double gz, double dt, cudaStream_t s);
void launch_rigid_world(RigidDev* bodies_dev, const RigidDev* bodies_host, int nb, cudaStream_t s);
// contact detection: count per (PT vertex) + (rigid body, vertex); literal PT only when T == 1.
void launch_detect_count(const MeshDev& m, const double* x, const RigidDev* bodies, int nb, int literal_pt, double thresh, int* counts, cudaStream_t s);
void launch_detect_write(const MeshDev& m, const double* x, const RigidDev* bodies, int nb, int literal_pt, double thresh, const int* offsets, ContactDev* out, cudaStream_t s);
void launch_contact_prep(const MeshDev& m, ContactDev* c, int nc, const StepParams& p, cudaStream_t s);
void launch_contact_entries(const ContactDev* c, int nc, int V, int friction, int* keys, ContactEntry* ents, cudaStream_t s);
void launch_vertex_ranges(const int* sorted_keys, int n, int V, int* begin, int* end, cudaStream_t s);
void launch_contact_vertex(const MeshDev& m, const ContactDev* c, const ContactEntry* ents, const int* begin, const int* end,
                           const StepParams& p, const double* g_base, double* g_const, double* diag_const, cudaStream_t s);
void launch_extra_flags(const ContactEntry* ents, const int* keys, int n, int* flags, cudaStream_t s);

// Newton iteration
void launch_ctrl_reset(Ctrl* ctrl, cudaStream_t s);
void launch_strain_face(const MeshDev& m, const double* x, const StepParams& p, unsigned char* flags, StrainSV* sv, Ctrl* ctrl, cudaStream_t s);
void launch_gradient(const MeshDev& m, const double* x, const double* x_hat, const double* x_prev, const double* g_const,
                     const double* diag_const, const unsigned char* sflags, const StrainSV* sv,
                     const int* pin_vertex, const int* pin_head, const double* pin_target, int num_pins, const WallDev* walls,
                     const ContactDev* contacts, const ContactEntry* ents, const int* ebegin, const int* eend,
                     const StepParams& p, const unsigned char* fixed, double* g, float* b, double* diag_extra, Ctrl* ctrl, cudaStream_t s);
void launch_check(Ctrl* ctrl, double tol, cudaStream_t s);
void launch_pin_heads(const int* pin_vertex, int num_pins, int* pin_head, cudaStream_t s);
void launch_assemble(const MeshDev& m, const unsigned char* sflags, const StrainSV* sv, const double* diag_extra, int enable_strain,
                     const unsigned char* fixed, float* val, float* precond, const Ctrl* ctrl, cudaStream_t s);
// scaled system (CORRECTED): L = chol(A_ii), A^ = L^-1 A L^-T (kernels.cu)
// tpb: threads per block (a tuning knob; one thread per vertex / slot, so the
// results do not depend on it)
void launch_diag_factor(const MeshDev& m, const unsigned char* sflags, const StrainSV* sv, const double* diag_extra, int enable_strain,
                        const unsigned char* fixed, const double* g, double* Linv, float* Lf, float* bhat, unsigned char* chol_ok,
                        const Ctrl* ctrl, cudaStream_t s, int tpb = 256);
// With the SELL-32 slice offsets (chunk_off) and the widest slice's column
// slots (wmax <= ASM_SLICE_WMAX), one CTA per slice stages the slice in
// shared memory and writes with coalesced stores (tpb then sizes nothing);
// otherwise one thread per slot with tpb threads per block. Both write the
// same values: always the SELL copy, val (unscaled) and valh (scaled, CSR
// order) only when non-null.
constexpr int ASM_SLICE_TPB = 128, ASM_SLICE_WMAX = 32;
inline size_t asm_slice_smem(int wmax, int copies) { return size_t(copies) * 9 * 32 * wmax * sizeof(float); }
void launch_assemble_scaled(const MeshDev& m, const unsigned char* sflags, const StrainSV* sv, const double* diag_extra, int enable_strain,
                            const unsigned char* fixed, const double* Linv, const unsigned char* chol_ok, float* val, float* valh,
                            const int* sell_base, float* valh_sell, const Ctrl* ctrl, cudaStream_t s, int tpb = 256,
                            const int* chunk_off = nullptr, int wmax = 0);
void launch_extra_key64(const ContactEntry* xent, const int* xkeys, int n, unsigned long long* key, int* idx, cudaStream_t s);
void launch_run_heads(const unsigned long long* key, int n, int* flags, cudaStream_t s);
void launch_extra_merge(const ContactDev* c, const ContactEntry* xent, const unsigned long long* key, const int* idx, const int* heads, int nu,
                        int n, const unsigned char* fixed, const StepParams& p, const double* Linv, int* xrow, int* xcols, float* xval,
                        float* xvalh, cudaStream_t s);
void launch_ls_wall(int V, const double* x, const float* d, WallDev w, Ctrl* ctrl, cudaStream_t s);
void launch_ls_contacts(const ContactDev* c, int nc, const double* x, const float* d, Ctrl* ctrl, cudaStream_t s);
void launch_update(int V, double* x, const float* d, Ctrl* ctrl, cudaStream_t s);

// end of step
void launch_velocity(int V, const double* x, const double* x_old, double beta_dt, double damp_scale, double* v, cudaStream_t s);
void launch_restitution_contacts(const ContactDev* c, int nc, const double* mass, int V, double e, double gap_limit,
                                 RigidDev* bodies, int nb, double* v, cudaStream_t s);
void launch_restitution_walls(int V, const double* x, const WallDev* walls, int nw, double e, double gap_max, double* v, cudaStream_t s);
void launch_rigid_coupling(const MeshDev& m, const ContactDev* c, int nc, const StepParams& p, RigidDev* bodies, int nb,
                           const int* offsets, long long units, double dt, cudaStream_t s);

// whole-frame CUDA graph control (kernels.cu)
void launch_ctl_init(StepCtl* c, double beta_max, int max_it, cudaGraphConditionalHandle outer, cudaStream_t s);
void launch_inner_begin(StepCtl* c, cudaGraphConditionalHandle newton, cudaStream_t s);
void launch_newton_ctl(StepCtl* c, const Ctrl* ctrl, cudaGraphConditionalHandle newton, cudaStream_t s);
void launch_outer_ctl(StepCtl* c, double beta_max, cudaGraphConditionalHandle outer, cudaStream_t s);
void launch_velocity_ctl(int V, const double* x, const double* x_old, double dt, double damp_scale, double* v, const StepCtl* c, cudaStream_t s);

// CORRECTED semantics (corrected.cu)
void launch_drive_extent(const int* pin_vertex, const double* pin_target, int num_pins, const double* x, const double* v, int V, double dt,
                         unsigned long long* out, cudaStream_t s);
void launch_pin_gather(const int* pin_vertex, int num_pins, const double* x, double* start, cudaStream_t s);
void launch_pin_interp(int num_pins, const double* start, const double* fin, double f, double* target, cudaStream_t s);
void launch_pairs_to_contacts(const int2* vt, int nvt, const int2* ee, int nee, const int* tris, const int* edges, const double* x,
                              double gap_max, ContactDev* out, cudaStream_t s);
void launch_swept_end(int V, const double* x, const float* d, const unsigned char* fixed, double scale, double lmax,
                      double* x1, double* ext, cudaStream_t s);
void launch_toi_reset(unsigned long long* toi, cudaStream_t s);
void launch_toi_walls(int V, const double* x, const double* ext, const WallDev* walls, int nw, unsigned long long* toi, cudaStream_t s);
void launch_toi_rigid(int V, const double* x, const double* ext, const RigidDev* bodies, int nb, unsigned long long* toi, cudaStream_t s);
void launch_update_toi(int V, double* x, const double* ext, double scale, const unsigned char* fixed, Ctrl* ctrl,
                       const unsigned long long* toi, cudaStream_t s);

// PCG (pcg.cu)
struct PcgArgs {
  int V;
  const int* rowptr; const int* cols; const float* val;
  const int* xbegin; const int* xend; const int* xcols; const float* xval;  // extra contact segment
  const float* P;     // block-Jacobi inverse, 9V
  const float* b;
  float *x, *r, *z, *p0, *p1, *Ap;
  double* partials;   // 3 * grid
  Ctrl* ctrl;
  float tol; int max_iters;
};
int pcg_grid_size(int device);

// CG on the block-scaled system (pcg.cu): identity (= block-Jacobi on A) or
// the learned approximate inverse S of the scaled system.
struct PcgScaledArgs {
  int V;
  const int* chunk_off; const int* sell_col; const float* valh;               // A^ on the static pattern (SELL-32, pcg.cu)
  const int* xbegin; const int* xend; const int* xcols; const float* xvalh;  // A^ extra contact segment
  // learned solves only: S_ij = coef * A^_ij off the diagonal (coef per SELL
  // slot, at the positions of sell_col) and S_ii = Sdiag (9 per vertex)
  const float* coef; const float* Sdiag;
  const double* Linv;   // 6V packed L^-1
  const float* Lf;      // 6V packed L
  const float* bhat;    // 3V  L^-1 b
  float* d;             // 3V  output: L^-T x^
  double* xh;           // 3V  scaled iterate x^ (FP64)
  float *r, *r2, *z, *p0, *p1, *Ap;
  double* partials;     // pcg_scaled_partials(V): three per-slice arrays
  Ctrl* ctrl;
  float tol; int max_iters; int stall_window;
  // block-Jacobi solves only: snapshot k of (r^, x^) after 2^k - 1 iterations, k < snap_max
  float* snap_r; double* snap_x; int snap_max;
  // block-Jacobi only: 1 = the fallback of the learned solve just before it
  // on the stream; returns at once when that solve ended PCG_OK (or timed out)
  int fallback = 0;
};
// Launch shape of the scaled PCG (threads per CTA, CTAs, column slots loaded
// ahead per thread). A tuning knob only: every shape gives the same bits.
struct PcgShape { int tpb = 0, grid = 0, unroll = 1; };
size_t pcg_scaled_partials(int V);
int pcg_scaled_shapes(int device, int V, bool learned, PcgShape* out, int max);
cudaError_t launch_pcg_scaled(const PcgScaledArgs& a, bool learned, const PcgShape& sh, cudaStream_t s);
cudaError_t launch_pcg(const PcgArgs& a, int grid, cudaStream_t s);

}  // namespace ando
