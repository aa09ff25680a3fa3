// Internal declarations shared by the host orchestration (lee_capi.cu), the FP64
// setup kernels (lee_setup.cu) and the time-advance kernels (lee_step.cu).
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "../../include/lee_b200.h"

namespace lee {

constexpr int kMaxZones = 8;  // sponge zones per block read by the stage kernel
constexpr int kMaxVars = 5;   // s', u'(1..num_dim), p'
constexpr int kMaxScalars = 8;  // passive scalars Z_k' (PHYSICAL_MODEL = LEE_SCALAR)

// Compile-time traits of a block's coefficient layout, chosen at setup (stage kernels):
constexpr int kTrJmField = 1;  // J*metrics vary over the block (else kernel constants)
constexpr int kTrUniform = 2;  // uniform mean flow: u_bar, p_bar, rho_bar constant, zero gradients
constexpr int kTrSponge = 4;   // sponge strengths summed into one per-point field (else the zone loop)
constexpr int kTrGeneric = kTrJmField;  // every coefficient checked at run time
// Launch-time traits of the TMA stage kernel (blocks without holes), added to the layout traits:
constexpr int kTrTma = 8;       // no holes; with kTrJmField every J*metrics entry is a per-point field;
                                // 32-bit point offsets
constexpr int kKindShift = 4;   // bits 4..6: the stage's kind; 0 reads p.stage and p.last at run time
constexpr int kKindRuntime = 0, kKindRhs = 1, kKindFirst = 2, kKindMid = 3, kKindLast = 4;
// the last stage of the compensated form writing the step's increment alone (no y_n read, no
// y_pre / error written): the fused filter forms y_pre = y_n + increment as the exact two-float
// sum itself (TMA kernels only)
constexpr int kKindLastIncrement = 5;

// One directional operator: interior stencil c[l+h] (l = -h..h), closure rows
// B[row][s] (row < nb, s < S) and the right-boundary sign (-1 difference, +1 filter).
// Values are those of the reference's StandardCentral / StandardCentralFilter /
// OptimizedCentral* classes (camille src/solver/spatial_discretization.cpp:28-492).
struct OpTable {
  int h, nb, S;
  double c[11];
  double B[5][9];
  double mfac;
};

// Closure code of a point along one direction, precomputed on the host by running
// the reference's per-line scan (StandardCentral::apply_spatial_discretization and
// iblank_correction, src/solver/spatial_discretization.cpp:1078-1652):
//   0        interior stencil
//   1 + r    left closure row r, anchored r points to the left
//  -(1 + r)  right closure row r (mirrored), anchored r points to the right
//   kZero    the value is zero (a hole following a hole)
constexpr int8_t kCodeZero = 100;

// A per-point coefficient: a device field, or a constant when the field is uniform
// over the block (checked in FP64 at setup). `zero` marks an identically-zero term.
template <typename T>
struct Coef {
  const T* p;
  T c;
  int zero;
};

// A sponge zone: inclusive index box and its strengths (box-shaped, i fastest); `ref`, when
// set, holds the state the zone relaxes toward (V box fields one after the other, the
// time-harmonic wave at the stage time), else it relaxes toward zero.
template <typename T>
struct Zone {
  int lo[3], hi[3];
  const T* sig;
  const T* ref;
};

// The time-harmonic wave of lee_set_harmonic_wave: type LEE_WAVE_*, form LEE_WAVEFORM_*, the
// propagation direction, amplitude, wavenumber k = 2 pi / wavelength, the Gaussian exponent
// factor -ln 2 / halfwidth^2 and the ambient pressure 1/gamma.
struct Wave {
  int type, form, dir;
  double amp, k, gfac, p0;
};

// The wave at coordinates x and time t as bc::bc_dirichlet_harmonicwave evaluates it
// (src/solver/boundary_condition.cpp:232-344): the entropy, velocity (along dir) and pressure
// fluctuations. Unknown combinations are refused on the host.
__host__ __device__ inline void wave_eval(const Wave& w, const double x[3], double t, double* s, double* u,
                                          double* p) {
  double pf = 0.0, vf = 0.0, sf = 0.0;
  if (w.form == LEE_WAVEFORM_PLANE) {
    pf = w.amp * w.p0 * sin(w.k * (x[w.dir] - 1.0 * t));
    vf = pf;
  } else if (w.type == LEE_WAVE_ACOUSTIC) {
    pf = w.amp * w.p0 * sin(w.k * 1.0 * t);
    vf = pf;
  } else {
    sf = w.amp * (1.0 + sin(w.k * 1.0 * t));
    if (w.form == LEE_WAVEFORM_GAUSSIAN_ROUNDJET) {
      const double a = x[w.dir == 0 ? 1 : 0], b = x[w.dir == 2 ? 1 : 2];
      sf *= exp(w.gfac * (a * a + b * b));
    }
  }
  *s = sf;
  *u = vf / (1.0 * 1.0);
  *p = pf;
}

// Everything one stage kernel launch needs for one block.
template <typename T>
struct StageParams {
  int nx, ny, nz, dim, V;
  // RK stage
  int stage, last;        // stage index, 1 on the last stage
  T h, b, a;              // step size, b_i and a_{i+1,i} of the Butcher tableau
  const T* zin[kMaxVars];   // stage input (read with neighbours)
  const T* yn[kMaxVars];    // y_n
  T* acc[kMaxVars];         // FP64: running y_next; compensated: running increment
  T* zout[kMaxVars];        // next stage input, or (last stage, compensated) y_pre
  T* comp[kMaxVars];        // compensated form: carried rounding error of y
  // coefficients (physical gradient d/dx_i f = sum_l JM[l][i] D_l f)
  Coef<T> jm[9];            // J * metrics[l][i] at l*3+i
  Coef<T> ubar[3], pbar, rhobar_inv;
  Coef<T> gs[3], gu[9], gp[3];  // mean gradients: d s_bar/dx_j, d u_bar_i/dx_j at i*3+j, d p_bar/dx_j
  int need_rho;                 // 1 when some d u_bar_i/dx_j is nonzero
  int increment;                // last stage of the compensated form: write the increment alone
  const T* rho_prev;            // rho'/rho_bar of the previous step's pre-filter state, read by the
                                // first stage and by a right-hand-side evaluation (null: from q)
  T gamma, inv_gamma;
  // sponges: per zone (generic kernels) or summed into one per-point field (TMA kernels)
  int nzones;
  Zone<T> zones[kMaxZones];
  const T* sigma;
  // axisymmetric term of the pressure equation (2-D): the r coordinate (y) when on
  int axisym;
  const double* ry;
  // monopole source: rhs[p] += amp * g, g on a box (src_lo..src_hi), i fastest; amp is src_amp,
  // or, in a replayed step graph, amp_tab[*step_ctr * nstages + stage]
  int has_src;
  T src_amp;
  const T* amp_tab;
  const int* step_ctr;
  int nstages;
  int src_lo[3], src_hi[3];
  const T* src_g;
  // holes and closure codes (nullptr when the block has no holes)
  const int8_t* code[3];
  const int* iblank;
  OpTable fd;
};

template <typename T>
struct FilterParams {
  int nx, ny, nz, V, dir, first, last;
  const T* in[kMaxVars];
  T* out[kMaxVars];
  // FP64: y0 for the blend on the last pass; compensated: see lee_step.cu
  const T* y0[kMaxVars];
  T* dsum[kMaxVars];
  const T* dsum_in[kMaxVars];
  T* comp[kMaxVars];
  const T* err[kMaxVars];
  T blend;
  const int8_t* code;
  const int* iblank;
  OpTable op;
};

// One BC line applied to a stage output (lee_bc.cu).
template <typename T>
struct BcParams {
  int kind, dir, end, nd, V;
  int lo[3], nb[3];           // the end face of the line's box (nb[dir] = 1)
  int nx, ny;
  long long sd;               // index stride along dir
  int S;                      // closure row width
  double c0[9];               // row 0 of the difference operator's left closure
  T* y[kMaxVars];
  T* e[kMaxVars];             // rounding errors of a compensated pair, or null
  const double* met[9];       // metrics, inverse metrics and Jacobian (slip wall)
  const double* minv[9];
  const double* jac;
  const int* iblank;
  // harmonic wave: the wave, the coordinates and the time of the boundary update (t, or in a
  // replayed step graph t_tab[*ctr * t_stride])
  Wave wave;
  const double* xyz[3];
  double t;
  const double* t_tab;
  const int* ctr;
  int t_stride;
};

// The time-harmonic wave on a sponge zone's box (lee_bc.cu): V box fields, zero in holes.
template <typename T>
struct WaveRefParams {
  int lo[3], nb[3], nx, ny, nd, V;
  Wave wave;
  const double* xyz[3];
  const int* iblank;
  double t;                   // the stage time, or in a replayed step graph t_tab[*ctr * t_stride]
  const double* t_tab;
  const int* ctr;
  int t_stride;
  T* out;
};

// Overset interpolation of a stage output over all blocks (lee_bc.cu): receiver r of block
// rb[r], linear index rl[r], takes the weighted sum of the donor stencil with lower-left
// corner dl[r] in block db[r] (weights wt[r*W..], zeta outermost, xi innermost). With
// `fused` (no stencil reads a receiver) the sums are written straight to the receivers;
// otherwise they go through buf first, as overset::interpolate gathers every sum before it
// overwrites any receiver.
constexpr int kMaxOvsBlocks = 8;
template <typename T>
struct OvsParams {
  int n, W, V, fused;
  int w[3];
  const int* rb;
  const long long* rl;
  const int* db;
  const long long* dl;
  const double* wt;
  double* buf;               // n x V, when not fused
  T* y[kMaxOvsBlocks][kMaxVars];
  T* e[kMaxOvsBlocks][kMaxVars];  // compensated pair errors, or null
  int nx[kMaxOvsBlocks], ny[kMaxOvsBlocks];
  int pair;
};

template <typename T>
cudaError_t launch_overset(const OvsParams<T>& p, cudaStream_t s);

template <typename T>
cudaError_t launch_bc(const BcParams<T>& p, cudaStream_t s);
template <typename T>
cudaError_t launch_wave_ref(const WaveRefParams<T>& p, cudaStream_t s);
// out = p'/(gamma p_bar) - s' of the state y (+ e when e is non-null)
template <typename T>
cudaError_t launch_rho(long long n, int V, T* const* y, T* const* e, const double* pbar, double gamma, T* out,
                       cudaStream_t s);

// ---- discrete adjoint (lee_adjoint.cu) ----------------------------------------------------
// The transpose of one directional operator (difference or filter) with its boundary closures:
// out_i = sum_t w[t] in_{i+t}, t = -H..H, with w the interior row `in`, or a class row for
// the E outputs nearest each end (lt[r]: position r; rt[r]: position n-1-r).
constexpr int kTH = 8;
constexpr int kTE = 16;
struct TransOp {
  int H, E;
  double in[2 * kTH + 1];
  double lt[kTE][2 * kTH + 1];
  double rt[kTE][2 * kTH + 1];
};

// One adjoint RK stage s (processed from the last stage down): zbar = L^T kin, with L the
// uniform-mean LEE operator (chain rule through J*metrics, sponge); ybar accumulates zbar
// (first processed stage: ybar = mu + zbar), and the next input is
// kout = hb_next * mu + ha_next * zbar. The distributed source's box field gathers
// amp * kin[p'] (kin = hb_in * mu on the first processed stage).
template <typename T>
struct AdjStageParams {
  int nx, ny, nz, V;
  int first, has_next;
  T hb_in, hb_next, ha_next;
  const T* kin[kMaxVars];
  const T* mu[kMaxVars];
  T* ybar[kMaxVars];
  T* kout[kMaxVars];
  Coef<T> jm[9];
  T ubar[3];
  T gpb, rbi;
  const T* sigma;
  double* gbar;
  double amp;
  int src_lo[3], src_hi[3];
  TransOp op;
};

// One direction of the transposed filter; the last pass blends (1 - beta) lam + beta F^T(...).
template <typename T>
struct AdjFilterParams {
  int nx, ny, nz, V, dir, last;
  const T* in[kMaxVars];
  T* out[kMaxVars];
  const T* lam[kMaxVars];
  T blend;
  TransOp op;
};

template <typename T>
cudaError_t launch_adj_stage(const AdjStageParams<T>& p, int dim, cudaStream_t s);
template <typename T>
cudaError_t launch_adj_filter(const AdjFilterParams<T>& p, cudaStream_t s);
// trace[row * n + m] = p'(l0[m]) (+ its carried error), row = *ctr + *base in a replayed
// graph, else `row`
template <typename T>
cudaError_t launch_trace(int n, const long long* l0, const T* p, const T* e, double* trace, const int* ctr,
                         const int* base, int row, cudaStream_t s);
// lam_p[l0[m]] += scale * trace[row * n + m]
template <typename T>
cudaError_t launch_mic_force(int n, const long long* l0, T* lam_p, const double* trace, int row, double scale,
                             cudaStream_t s);

// ---- passive scalars (lee_scalar.cu) -------------------------------------------------------
// One RK stage of the n scalar slots of a block: dZ'/dt = -u_bar . grad Z' - u' . grad Z_bar
// minus the sponges, with the stage update of the LEE slots (hole bypass, FP64 or compensated).
// u' is the LEE stage input at the point.
template <typename T>
struct ScalarParams {
  int nx, ny, nz, dim, n;
  int stage, last;
  T h, b, a;
  const T* zin[kMaxScalars];
  const T* yn[kMaxScalars];
  T* acc[kMaxScalars];
  T* zout[kMaxScalars];
  T* comp[kMaxScalars];
  const T* uin[3];
  Coef<T> jm[9], ubar[3];
  Coef<T> gz[kMaxScalars][3];   // d Z_bar_k / dx_j
  int nzones;
  Zone<T> zones[kMaxZones];
  const int8_t* code[3];
  const int* iblank;
  OpTable fd;
};

template <typename T>
cudaError_t launch_scalar_stage(const ScalarParams<T>& p, int comp, cudaStream_t s);

// ---- the general discrete adjoint (lee_adjoint_gen.cu) ------------------------------------
// One transposed RK stage of one block: zbar = L^T w, w = scale * kin, with the forward stage's
// coefficients, sponge zones, closure codes and source box in `f` (fill_stage_common).
template <typename T>
struct AdjGenParams {
  StageParams<T> f;
  T scale;
  const T* kin[kMaxVars];
  T* g[3][kMaxVars];         // the fluxes G^d (flux kernel out, stage kernel in)
  T* zbar[kMaxVars];
  T* rbar;                   // the adjoint of rho_prev when the forward stage read it, else null
  double* gbar;              // the source box's gradient (null: none)
  double amp;
};

// One transposed filter pass (reverse order of the forward's passes): the first reads M lam
// (mask_in), the last blends (1 - beta) M lam + beta F^T(...) and adds R^T rb.
template <typename T>
struct AdjGenFilterParams {
  int nx, ny, nz, V, dir, last, mask_in;
  const T* in[kMaxVars];
  T* out[kMaxVars];
  const T* lam[kMaxVars];
  T blend;
  OpTable op;
  const int8_t* code;        // the filter's closure codes along dir (null: by position)
  const int* iblank;         // holes (null: none)
  const T* rb;               // adjoint of rho'/rho_bar of Y (null: none)
  const double* pbar;
  T inv_gamma;
};

// Pointwise operands: mask (and R^T rb) of `in` into `out`, or the stage combine
// nu = M in; ybar += nu; out = hb mu + ha nu (out[0] null: ybar += in unmasked).
template <typename T>
struct AdjGenPoint {
  const T* in[kMaxVars];
  T* out[kMaxVars];
  const T* mu[kMaxVars];
  T* ybar[kMaxVars];
  const int* iblank;
  const T* rb;
  const double* pbar;
  T inv_gamma;
};

// The transposed overset interpolation: n receivers (block rb, point rl) are taken out into
// tmp (n x V), then nd donor points (block ub, point ul) gather cw * tmp over their receiver
// lists off[u]..off[u+1] (receiver cr).
template <typename T>
struct AdjGenOvs {
  int n, nd, V;
  const int* rb;
  const long long* rl;
  const int* ub;
  const long long* ul;
  const int* off;
  const double* cw;
  const int* cr;
  double* tmp;
  T* y[kMaxOvsBlocks][kMaxVars];
};

template <typename T>
cudaError_t launch_adjg_stage(const AdjGenParams<T>& p, cudaStream_t s);
template <typename T>
cudaError_t launch_adjg_filter(const AdjGenFilterParams<T>& p, cudaStream_t s);
template <typename T>
cudaError_t launch_adjg_mask(long long n, int V, const AdjGenPoint<T>& p, cudaStream_t s);
template <typename T>
cudaError_t launch_adjg_combine(long long n, int V, const AdjGenPoint<T>& p, double hb, double ha, cudaStream_t s);
template <typename T>
cudaError_t launch_adjg_bc(const BcParams<T>& p, cudaStream_t s);
template <typename T>
cudaError_t launch_adjg_overset(const AdjGenOvs<T>& p, cudaStream_t s);

// ---- batches of 2-D blocks (lee_batch.cu) ------------------------------------------------
// Per-block filter operands of the batched filter: pre-filter state x (FP64: y_next;
// compensated: y_pre, with its rounding error err), outputs y (and the new error comp).
template <typename T>
struct BatchFilterInst {
  int nx, ny;
  const T* x[4];
  const T* err[4];
  T* y[4];
  T* comp[4];
};

constexpr int kBatchShapes = 7;
void batch_shape(int shape, int* tx, int* ty);
// A shape the persistent step launch takes (one column per stage thread: shapes 0..4).
bool batch_step_shape(int shape);
// The whole batched step (ns stages, then the filter) in one persistent cooperative launch over
// the work items of `shape` (lee_batch.cu): gbar is a two-word barrier, err the device flag that
// a barrier wait giving up after wait_ns sets.
template <typename T>
cudaError_t launch_batch_step(const StageParams<T>* prm, int nbk, int ns, const BatchFilterInst<T>* inst,
                              const int4* items, int n, int shape, int comp, const OpTable& op, double blend,
                              unsigned* gbar, int* err, unsigned long long wait_ns, cudaStream_t s);
// one launch over the tile list (int4: block, x0, y0, 0) with the blocks' stage parameters
template <typename T>
cudaError_t launch_batch_stage(const StageParams<T>* prm, const int4* tiles, int ntiles, int shape, int comp,
                               int grid, cudaStream_t s);
template <typename T>
cudaError_t launch_batch_filter(const BatchFilterInst<T>* inst, const int4* tiles, int ntiles, int shape, int comp,
                                int grid, const OpTable& op, double blend, cudaStream_t s);
template <typename T>
int batch_stage_occupancy(int shape, int comp);
template <typename T>
int batch_filter_occupancy(int shape, int comp);

// lee_step.cu
template <typename T>
cudaError_t launch_stage(const StageParams<T>& p, int comp, cudaStream_t s);
template <typename T>
cudaError_t launch_filter_pass(const FilterParams<T>& p, int comp, cudaStream_t s);
cudaError_t launch_hole_zero(int n, int V, double** f, const int* iblank, cudaStream_t s);
cudaError_t launch_hole_zero_f(int n, int V, float** f, const int* iblank, cudaStream_t s);

// lee_capi.cu helpers shared with lee_static.cu
bool filter_table(OpTable* o, int scheme, int order, double strength);
void set_global_error(const char* msg);

// lee_setup.cu (FP64, no FMA contraction)
cudaError_t setup_apply_dir(const OpTable& op, int nx, int ny, int nz, int dir, const double* f, double* out,
                            const int8_t* code, int zero_if_one_cell, cudaStream_t s);
cudaError_t setup_axpby(int n, double* out, double a, const double* x, double b, const double* y,
                        cudaStream_t s);  // out = a*x + b*y (y may be null)
cudaError_t setup_mul(int n, double* out, const double* x, const double* y, cudaStream_t s);
cudaError_t setup_jacobian(int n, int dim, double* const* xx, double* invjac, double* jac, cudaStream_t s);
cudaError_t setup_inverse_metrics(int n, int dim, double* const* met, double* const* minv, cudaStream_t s);
cudaError_t setup_grad_accum(int n, double* sum, const double* m, const double* d, cudaStream_t s);
cudaError_t setup_scale(int n, double* out, const double* sum, const double* jac, cudaStream_t s);
cudaError_t setup_sigma(int nx, int ny, int nz, const double* const* xyz, const int lo[3], const int hi[3], int dir,
                        int end, int order, double constant, double* sig, cudaStream_t s);
cudaError_t setup_minmax(int n, const double* f, double* d_out2, cudaStream_t s);
cudaError_t setup_state_minmax(long long n, const void* y, const void* e, bool fp32, double* d_out2, cudaStream_t s);
cudaError_t setup_cfl(int n, int dim, const double* const* met, const double* jac, const double* const* ubar,
                      const double* pbar, const double* sbar, const int* iblank, double gamma, double dt,
                      double* d_max, cudaStream_t s);
cudaError_t setup_rho_ratio(int n, int V, double gamma, const double* sv, const double* p, const double* pbar,
                            double* out, cudaStream_t s);
cudaError_t setup_monopole_g(int nx, int ny, const double* const* xyz, const int lo[3], const int hi[3],
                             double x0, double y0, double z0, double ef, double* g, cudaStream_t s);

}  // namespace lee
