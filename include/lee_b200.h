/*
 * lee_b200.h -- C ABI of the B200 linearized-Euler (LEE) time-advance path.
 *
 * This library replaces the RK loop of the camille solver: the seam is
 * solver::solve(UserInput*, StructuredGrid*, StructuredBlock*, State*)
 * (camille src/solver/solver.h:21, src/solver/solver.cpp:41-89), called once by
 * simulation::run (src/core/simulation.cpp:256) after the deck, grids, mean
 * flow, BC file and restart file have been read. A replacement solve() marshals
 * the reference's host arrays through the calls below; every array crosses the
 * boundary as plain float64/int32 pointers in the reference's own layout:
 * one array per variable, index l = i + nxi*(j + neta*k), i fastest
 * (src/geometry/geometry.h:131-136). The library copies host buffers on every
 * set/upload/download call; the caller keeps ownership of them.
 *
 * Conventions
 *  - Every entry point returns LEE_OK (0) or an LEE_ERR_* code; the message of
 *    the last failure on a context is lee_last_error(ctx). The reference has no
 *    status codes (it calls mpi::graceful_exit, src/parallel/parallel.cpp:90-96).
 *  - A context is single-threaded and owns one CUDA stream on its device. All
 *    blocks of a context are resident in that GPU's memory; block-halo and
 *    overset exchanges happen on the device.
 *  - State variables follow the reference's LEE slots (src/core/param.h:67-80):
 *    0 = s' (entropy), 1..3 = u', v', w', 4 = p'. The mean flow has the same
 *    slots (s_bar, u_bar, v_bar, w_bar, p_bar). In 2-D the w' slot must be zero
 *    on upload and is zero on download (in the reference it only ever carries
 *    the sponge term acting on a zero field).
 *  - There is no CPU fallback: lee_create fails with LEE_ERR_NODEVICE when no
 *    CUDA device is usable.
 */
#ifndef LEE_B200_H
#define LEE_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define LEE_ABI_VERSION 1

/* status codes */
#define LEE_OK 0
#define LEE_ERR_ARG 1          /* invalid argument */
#define LEE_ERR_STATE 2        /* call made in the wrong order */
#define LEE_ERR_CUDA 3         /* CUDA runtime error */
#define LEE_ERR_NOMEM 4        /* device or host allocation failed */
#define LEE_ERR_UNSUPPORTED 5  /* combination not implemented */
#define LEE_ERR_NONFINITE 6    /* NaN/Inf detected in the state */
#define LEE_ERR_NODEVICE 7     /* no usable CUDA device */
#define LEE_ERR_TIMEOUT 8      /* a bounded device-side wait gave up */

/* SPATIAL_SCHEME (src/core/input.cpp:147-150) */
#define LEE_FD_STANDARD_CENTRAL 1  /* with fd_order 2 or 4 (src/solver/spatial_discretization.cpp:28-109) */
#define LEE_FD_FDO11P 11           /* Bogey & Bailly 11-point (:228-344) */
/* SPATIAL_FILTER (src/core/input.cpp:152-165) */
#define LEE_FILTER_NONE 0
#define LEE_FILTER_STANDARD_CENTRAL 1  /* with filter_order 4 or 8 (:113-224) */
#define LEE_FILTER_SFO11P 11           /* with filter_strength (:348-492) */
/* TEMPORAL_SCHEME (src/solver/temporal_discretization.cpp:33-85) */
#define LEE_RK2 2
#define LEE_RK4 4
/* arithmetic form of the time advance */
#define LEE_FP64 0                /* the reference's own FP64 arithmetic */
#define LEE_FP32_COMPENSATED 1    /* FP32 state/stencils, compensated RK sum */

/* boundary kinds: the reference's codes (src/core/param.h:99-114) */
#define LEE_BC_DIRICHLET_ALLZERO 1         /* every slot 0 (bc_dirichlet_allzero) */
#define LEE_BC_DIRICHLET_HARMONICWAVE 2    /* the harmonic wave of lee_set_harmonic_wave */
#define LEE_BC_NEUMANN 100
#define LEE_BC_WALL_SLIP_KINEMATIC 201
#define LEE_BC_CENTERLINE_CART_NORM2X 900  /* Neumann, then u' = 0 (v' for 901, w' for 902) */
#define LEE_BC_CENTERLINE_CART_NORM2Y 901
#define LEE_BC_CENTERLINE_CART_NORM2Z 902
#define LEE_BC_CENTERLINE_AXISYM 903       /* Neumann, then u_r' (v') = 0 */
#define LEE_SPONGE_FREUND_AMBIENT 1000
#define LEE_SPONGE_FREUND_HARMONICWAVE 1002  /* relaxes toward the harmonic wave */

/* time-harmonic wave (HARMONIC_WAVE deck line, src/core/input.cpp:219-231) */
#define LEE_WAVE_NONE 0
#define LEE_WAVE_ACOUSTIC 1             /* WAVE_ACOUSTIC */
#define LEE_WAVE_ENTROPY 2              /* WAVE_ENTROPY */
#define LEE_WAVEFORM_PLANE 0            /* WAVEFORM_PLANE (acoustic) */
#define LEE_WAVEFORM_HOMOGENEOUS 1      /* WAVEFORM_HOMOGENEOUS (acoustic or entropy) */
#define LEE_WAVEFORM_GAUSSIAN_ROUNDJET 2 /* WAVEFORM_GAUSSIAN_ROUNDJET (entropy) */

/* physical sources */
#define LEE_SOURCE_NONE 0
#define LEE_SOURCE_MONOPOLE 1  /* params: x0, y0, z0, amplitude, omega, halfwidth, ramp_time */
/* Distributed monopole (no reference counterpart: the reference cannot express it): on block
 * `block`, rhs[p'] += (gamma - 1) sin(omega t) S(l), with S the trilinear prolongation of a
 * coarse amplitude lattice of cx x cy x cz nodes whose node (p, q, r) sits at the fractional
 * grid index (ox + p hx, oy + q hy, oz + r hz); S is zero outside the lattice's box.
 * params: block, omega, cx, cy, cz, ox, oy, oz, hx, hy, hz, then cx*cy*cz amplitudes
 * (p fastest). In 2-D, cz = 1. */
#define LEE_SOURCE_DISTRIBUTED 2
/* The pressure source of SIMULATION = CASE_2DJET_WITH_A_HARMONIC_SOURCE (source::apply_physicalSource,
 * src/solver/source.cpp:27-58), no params: rhs[p'] += exp(-(Bx x^2 + By y^2)) A cos(2 pi f t) with
 * the reference's constants made non-dimensional by b = 1.3, c_inf = sqrt(gamma 287 300),
 * rho_inf = 1.184 (A = 0.001 b / (rho_inf c_inf^3), f = 76 b / (2 pi c_inf), Bx = 0.04 ln 2 b^2,
 * By = 0.32 ln 2 b^2). */
#define LEE_SOURCE_JET2D_HARMONIC 3

/* lee_get_setup selectors: products of the one-time setup, per block */
#define LEE_SETUP_METRICS 0     /* 9 fields, metrics[l][i] = (1/J) dxi_l/dx_i, row-major (l*3+i) */
#define LEE_SETUP_JACOBIAN 1    /* 1 field, J */
#define LEE_SETUP_MEAN_GRADIENT 2 /* 5*num_dim fields, d(mean_v)/dx_j at v*num_dim + j */
#define LEE_SETUP_SPONGE 3      /* 1 field, sum of the Freund sponge strengths at each point */

typedef struct lee_ctx lee_ctx;

typedef struct {
  int num_dim;            /* DIMENSION: 2 or 3 */
  int num_blocks;         /* number of structured blocks */
  double gamma;           /* GAMMA_SPECIFICHEAT */
  int fd_scheme;          /* LEE_FD_* */
  int fd_order;           /* ORDER_ACCURACY of STANDARD_CENTRAL: 2 or 4 */
  int filter_scheme;      /* LEE_FILTER_* */
  int filter_order;       /* ORDER_ACCURACY of the standard filter: 4 or 8 */
  double filter_strength; /* SFO11P STRENGTH (the standard filter forces 1.0) */
  double filter_blend;    /* BLEND */
  int rk_scheme;          /* LEE_RK2 or LEE_RK4 */
  int precision;          /* LEE_FP64 or LEE_FP32_COMPENSATED */
  int sponge_order;       /* BUFFER_ZONE POLYNOMIAL_ORDER */
  double sponge_constant; /* BUFFER_ZONE CONSTANT */
  int device;             /* CUDA device ordinal */
} lee_config;

/* Create a context (replaces solver::initialize, src/solver/solver.cpp:8-15). */
int lee_create(const lee_config *cfg, lee_ctx **out);
/* Release every device and host resource of the context. */
void lee_destroy(lee_ctx *ctx);
/* Message of the last failure on ctx; with ctx NULL, of the calling thread's last failed call
 * without a context (lee_create, lee_filter_field_static). */
const char *lee_last_error(const lee_ctx *ctx);

/* Grid of block b: coordinates (io::read_grid, src/io/plot3d.cpp:443-671) and the
 * overset iblank (src/geometry/geometry.h:24-26; NULL = all NOTBLANKED). The
 * metrics and Jacobian are generated from these on the GPU in FP64 by
 * lee_prepare (metrics::compute, src/metrics/metrics.cpp:9-44). */
int lee_set_block(lee_ctx *ctx, int b, int nxi, int neta, int nzeta, const double *x, const double *y,
                  const double *z, const int *iblank);
/* Mean flow of block b, five fields (io::read_function, src/io/plot3d.cpp:881-989). */
int lee_set_mean(lee_ctx *ctx, int b, const double *const mean[5]);
/* One BC-file line (io::read_bc, src/io/io.cpp:957-1105): kind LEE_BC_* or
 * LEE_SPONGE_*, dir 0/1/2 (XI/ETA/ZETA), end 0 (left, "+dir") or 1 (right,
 * "-dir"), inclusive index box lo..hi. For sponges, sigma may hold the zone's
 * strengths (box-shaped, i fastest, as StructuredBufferZone::buffer_strength,
 * src/geometry/geometry.cpp:1126-1127); NULL computes them on the GPU. */
int lee_add_boundary(lee_ctx *ctx, int b, int kind, int dir, int end, const int lo[3], const int hi[3],
                     const double *sigma);
/* The time-harmonic wave read by LEE_BC_DIRICHLET_HARMONICWAVE lines and
 * LEE_SPONGE_FREUND_HARMONICWAVE zones (the deck's HARMONIC_WAVE line, src/core/input.cpp:219-231;
 * the wave of bc::bc_dirichlet_harmonicwave, src/solver/boundary_condition.cpp:232-344). type
 * LEE_WAVE_*, form LEE_WAVEFORM_*, dir 0/1/2 (X/Y/Z) the propagation direction, amplitude in
 * [0, 1] (check_consistency_wave, src/core/input.cpp:650-652), wavelength > 0, halfwidth > 0
 * for the Gaussian round jet (ignored otherwise). With k = 2 pi / wavelength, p_0 = 1/gamma and
 * x the coordinate along dir, the wave at time t is
 *   acoustic plane:        p' = u'_dir = amplitude p_0 sin(k (x - t)), s' = 0
 *   acoustic homogeneous:  p' = u'_dir = amplitude p_0 sin(k t),       s' = 0
 *   entropy homogeneous:   s' = amplitude (1 + sin(k t)),              u' = p' = 0
 *   entropy round jet:     s' = amplitude (1 + sin(k t)) exp(-ln 2 (a^2 + b^2) / halfwidth^2)
 * with a, b the two coordinates other than x; every other slot is 0. A BC line writes it on
 * its face at the time the reference's RungeKutta::integrate passes to update_boundary
 * (tn + c_{min(i+1, last)} h); a sponge zone adds -sigma (q - wave) at the stage time.
 * LEE_ERR_ARG for an unknown type or form, a form the type has no formula for, or a value out
 * of range (the reference stops at its first boundary update on a form the type has no formula
 * for); LEE_ERR_UNSUPPORTED for an acoustic wave along Z in 2-D (its w' has no slot here). */
int lee_set_harmonic_wave(lee_ctx *ctx, int type, int form, int dir, double amplitude, double wavelength,
                          double halfwidth);
/* AXISYMMETRY = TRUE with AXIS_OF_SYMMETRY = axis (src/core/input.cpp:105-108): the 2-D block is
 * the (x, r) half-plane with r = y, v' = u_r', and the pressure right-hand side gains
 * -gamma (p_bar v' + p' v_bar) / (y + 1e-99) (compute_RHS_linearized_Euler,
 * src/solver/spatial_discretization.cpp:2118-2126). Before lee_prepare; on = 0 turns it off.
 * LEE_ERR_ARG unless num_dim is 2 and axis is 0 (X) (check_consistency_dimension,
 * src/core/input.cpp:519-535). */
int lee_set_axisymmetric(lee_ctx *ctx, int on, int axis);
/* Physical source (source::apply_physicalSource, src/solver/source.cpp:22-107). */
int lee_set_source(lee_ctx *ctx, int kind, const double *params, int nparams);
/* A source for block b only (no reference counterpart: the reference applies its source to
 * every block): LEE_SOURCE_MONOPOLE with the 7 parameters of lee_set_source, or
 * LEE_SOURCE_NONE for a block without source. Used by batches of independent instances. */
int lee_set_block_source(lee_ctx *ctx, int b, int kind, const double *params, int nparams);
/* Overset donor maps, replacing overset::initialize_overset (src/overset/overset.cpp:56-84)
 * with the data of its Overture file (src/io/overture.cpp:473-680). n receivers, grouped by
 * block in block order: recv_block[r] and recv_ijk[3r..3r+2] (block-level indices), the donor
 * block and the lower-left corner donor_ijk of its stencil of width[0] x width[1] x width[2]
 * points, and the stencil weights (width product per receiver, zeta outermost, xi innermost),
 * which are normalised by their sum as initialize_donor does (:516-526). Holes are set
 * BLANKED (:683-751), then receivers INTERPOLATED (:755-790). After every boundary update
 * each receiver is overwritten with its stencil's weighted sum (overset::interpolate,
 * :820-845). Call after lee_set_block and before lee_prepare. */
int lee_set_overset(lee_ctx *ctx, int n, const int *recv_block, const int *recv_ijk, const int *donor_block,
                    const int *donor_ijk, const int width[3], const double *weights, int num_holes,
                    const int *hole_block, const int *hole_ijk);
/* Read the Overture overset file as read_overset_at_headrank does (src/io/overture.cpp:473-680;
 * the stencil width must be order_accuracy + 1, :609), then lee_set_overset. */
int lee_read_overset_file(lee_ctx *ctx, const char *path, int order_accuracy);
/* The maps as the time loop holds them (for the donor-map check; no reference counterpart):
 * per receiver its block and linear index i + nxi (j + neta k), the donor block and the
 * linear index of the stencil's lower-left corner, and the normalised weights. Any pointer
 * may be null. Arrays hold n (weights: n times the width product) entries. */
int lee_get_overset(lee_ctx *ctx, int *recv_block, long long *recv_l0, int *donor_block, long long *donor_l0,
                    double *weights);
/* Finish setup on the GPU: metrics, Jacobian, mean gradients (spatial::precompute_something,
 * src/solver/spatial_discretization.cpp:2250-2271), sponge strengths, hole closures,
 * and the per-point coefficient fields the kernels read. */
int lee_prepare(lee_ctx *ctx);

/* Restart state of block b with its step and time (io::read_solution, src/io/plot3d.cpp:715-835). */
int lee_upload_state(lee_ctx *ctx, int b, const double *const sol[5], int step, double time);
/* Current state of block b (State::sol, src/core/state.h:39). */
int lee_download_state(lee_ctx *ctx, int b, double *const sol[5], int *step, double *time);

/* Passive scalars (PHYSICAL_MODEL = LEE_SCALAR with NUMBER_SCALAR = n, src/core/input.cpp:113-119,
 * :768-773): n state slots Z_k' after p', with mean fields Z_bar_k, advanced by
 * dZ'/dt = -u_bar . grad Z' - u' . grad Z_bar (compute_RHS_linearized_Euler_scalar,
 * src/solver/spatial_discretization.cpp:2134-2158) plus the sponges (relaxing to zero); they
 * take the Neumann rows of every Neumann, slip-wall and centerline BC line, zero on Dirichlet
 * lines, and go through the overset interpolation, the filter and the hole mask with the other
 * slots. lee_set_scalars (0 <= n <= 8) comes before lee_set_block; the mean scalars before
 * lee_prepare; the state slots after it. Pointers: n fields of the block's points each. The
 * adjoint and the batched kernels do not take scalars. */
int lee_set_scalars(lee_ctx *ctx, int n);
int lee_set_mean_scalars(lee_ctx *ctx, int b, const double *const *zbar);
int lee_upload_scalars(lee_ctx *ctx, int b, const double *const *z);
int lee_download_scalars(lee_ctx *ctx, int b, double *const *z);

/* Time step for a target CFL (temporal::compute_CFL, src/solver/temporal_discretization.cpp:397-450),
 * including the reference's truncation of the convective term to an int (abs(double) resolving to
 * int abs(int) at :425): the first FIX_CFL step of solver::solve (src/solver/solver.cpp:54-64),
 * dt = 1e-6 * (cfl / cmax) with cmax the largest CFL over non-hole points at the dummy dt 1e-6. */
int lee_compute_dt(lee_ctx *ctx, double cfl, double *dt);
/* Largest CFL over all non-hole points at time step dt (temporal::compute_CFL,
 * src/solver/temporal_discretization.cpp:397-450): the value solver::solve reports and, under
 * FIX_CFL, rescales dt by at every step (src/solver/solver.cpp:54-68). */
int lee_compute_cfl(lee_ctx *ctx, double dt, double *cfl);
/* Minimum and maximum of each of the five solution slots over every point of every block
 * (ReportSolution::minmax, src/io/io.cpp:440-499), reduced on the GPU; a 2-D state's w' slot
 * reports 0 ~ 0. */
int lee_state_minmax(lee_ctx *ctx, double mn[5], double mx[5]);
/* Advance every block by nsteps RK steps of size dt (FIX_DT): per step the RK stages with
 * boundary conditions and overset updates, the filter and the hole mask
 * (temporal::time_advance, src/solver/temporal_discretization.cpp:334-374). */
int lee_advance(lee_ctx *ctx, int nsteps, double dt);

/* Inner seams, for operator-level parity checks. */
/* Right-hand side of the current state of block b at the given time (spatial::compute_RHS,
 * src/solver/spatial_discretization.cpp:1963-1990). */
int lee_eval_rhs(lee_ctx *ctx, int b, double time, double *const rhs[5]);
/* Apply the filter once to the current state of every block (spatial::apply_filter, :2191-2246). */
int lee_apply_filter(lee_ctx *ctx);
/* Copy a setup product of block b (LEE_SETUP_*) to host memory; out holds the selector's fields
 * back to back, each nxi*neta*nzeta long. */
int lee_get_setup(lee_ctx *ctx, int b, int what, double *out);

/* Batches (no reference counterpart): advance every block nsteps with its own time step
 * dt[b] and its own clock (lee_download_state returns each block's step and time). For
 * independent blocks only (no overset). A context whose blocks are all 2-D with a
 * uniform mean, the 4th-order difference, no BC lines or holes runs them through batched
 * kernels: one launch per RK stage and one per filter for the whole batch, over a work list
 * of tiles from every block, replayed as step graphs. */
int lee_advance_blocks(lee_ctx *ctx, int nsteps, const double *dt);
/* The FIX_CFL time step of every block on its own (dt[b], as lee_compute_dt would give for a
 * context holding block b alone). */
int lee_compute_dt_blocks(lee_ctx *ctx, double cfl, double *dt);
/* Override the batched launches' work-item shapes that lee_prepare picked by timing (index
 * 0..6; lee_info reports the strip of each): every shape gives the same results. */
int lee_set_batch_shapes(lee_ctx *ctx, int stage_shape, int filter_shape);
/* One launch per batched step (no reference counterpart; the same bits as the per-phase
 * launches): shape 0..4 (a work-item shape with one column per stage thread; lee_info's tiles
 * give the strips) runs every RK stage and the filter of lee_advance_blocks in one persistent
 * cooperative launch over that shape's work items, all of its CTAs resident, the phases separated
 * by device-wide barriers. A barrier wait gives up after the lee_set_wait_limit limit and the
 * call ends with LEE_ERR_TIMEOUT (the context stays usable); -1 (the default) goes back to one
 * launch per stage and per filter. Call after lee_prepare, on a context that runs batched
 * kernels. */
int lee_set_batch_persistent(lee_ctx *ctx, int shape);
/* Sizes and coefficient layout chosen by lee_prepare (no reference counterpart: the
 * reference has no timers or counters, finding F13). */
typedef struct {
  long long points;          /* grid points over all blocks */
  int state_vars;            /* active state variables per point (num_dim + 2) */
  int bytes_per_value;       /* 8 for LEE_FP64, 4 for LEE_FP32_COMPENSATED */
  int num_coef_fields;       /* per-point coefficient fields read by every stage; uniform
                                fields are folded into kernel constants at setup */
  long long device_bytes;    /* device memory held by the context */
  int tma_stage;             /* 1 when every block runs the TMA-staged stage kernel */
  int tma_filter;            /* 1 when every block runs the fused TMA-staged filter */
  int stage_chunk;           /* planes marched per CTA by the stage kernel (autotuned; block 0) */
  int filter_chunk;          /* planes marched per CTA by the filter kernel (autotuned; block 0) */
  int batched;               /* 1 when the blocks run through the batched kernels */
  int batch_stage_tile[2];   /* tile (xi, eta points) of the batched stage and filter launches, */
  int batch_filter_tile[2];  /* picked by timing the candidates at lee_prepare */
  int filter_kernel;         /* fused filter of block 0: 0 scalar, else the vector group width */
  int stage_kernel;          /* TMA stage kernel of block 0: points per thread */
  int filter_rows;           /* scalar fused filter of block 0: its form (lee_set_filter_form) */
  int increment_step;        /* 1 when every block's compensated step hands the increment to the filter */
} lee_info;
int lee_get_info(lee_ctx *ctx, lee_info *info);

/* Device-side timing of the last lee_advance, from CUDA events recorded on the
 * context's stream. Per-kernel times are collected only while timing is on. */
typedef struct {
  double advance_ms;         /* whole lee_advance */
  double stage_ms;           /* fused RK stage kernels */
  double filter_ms;          /* filter kernels */
  long long stage_launches;
  long long filter_launches;
  long long kernel_launches; /* every kernel this library launched in the last lee_advance */
} lee_stats;
int lee_set_timing(lee_ctx *ctx, int on);
/* Step graphs (no reference counterpart; on by default): lee_advance captures the launches
 * of a few steps once, until the buffer roles repeat, and replays them as one CUDA graph per
 * group of steps. Off, or while kernel timing is on, every launch is issued on its own. The
 * results are the same either way. */
int lee_set_graphs(lee_ctx *ctx, int on);
/* Multi-block contexts (no reference counterpart; results are the same bits either way):
 * lee_set_block_streams: on (default), the blocks' stage launches (with their BC lines) and filter
 * launches of one step go to side streams forked from the context stream and joined before the
 * overset update and the next stage, so blocks run side by side (parallel branches of a step
 * graph); off, one stream.
 * lee_set_batching (before lee_prepare): on (default), a context of 2-D uniform-mean blocks without
 * holes, BC lines or overset runs the batched kernels (one launch per stage for all blocks); off,
 * every block runs its own kernels (TMA-staged where the block allows), side by side. */
int lee_set_block_streams(lee_ctx *ctx, int on);
/* The compensated form's step (no reference counterpart; the same bits either way): on, on blocks
 * where nothing acts between the last RK stage and the filter (TMA-staged kernels, the one-row
 * fused filter, no BC lines, no overset, a uniform mean), the last stage writes the step's
 * increment alone and the fused filter forms y_pre = y_n + increment and its rounding error
 * itself: 2V fewer words of 4 bytes per point and step, but the filter then stages y_n and the
 * increment with their halos (twice the shared memory per plane), which costs it more time than
 * the stage saves on the B200. Off (default): the last stage writes y_pre and its error. On before
 * lee_prepare also keeps the fused filter to its one-row form (the form that takes the increment). */
int lee_set_increment_step(lee_ctx *ctx, int on);
int lee_set_batching(lee_ctx *ctx, int on);
/* Failure detection (no reference counterpart: camille keeps going on NaN, and its waits are MPI
 * calls, src/parallel/parallel.cpp:78-96).
 * lee_set_finite_check: after every `every` steps of lee_advance / lee_advance_blocks a sentinel
 * kernel checks that every state value is finite; a NaN or an infinity ends the call with
 * LEE_ERR_NONFINITE, the state left as it is (lee_download_state still works). 0 (default):
 * one check at the end of each call; -1: no check.
 * lee_set_wait_limit: the kernels stage their inputs with TMA copies and wait on them for at most
 * `seconds` (default 1 s, restored by a negative value; at most 10 s); a wait that gives up
 * ends the call with LEE_ERR_TIMEOUT after its CTA has drained its copies in flight, and the
 * context stays usable. 0 makes every such wait give up at once, landed or not: it exercises
 * that path in tests. */
int lee_set_finite_check(lee_ctx *ctx, int every);
int lee_set_wait_limit(lee_ctx *ctx, double seconds);
/* Kernel of the fused filter (no reference counterpart; results agree to rounding): -1 or 0
 * (default) the scalar kernel, 2 or 4 the kernel that gives each thread that many neighbouring
 * points along xi (4: FP32 only). LEE_ERR_UNSUPPORTED from lee_prepare when a block cannot run the
 * choice. Call before lee_prepare. */
int lee_set_filter_kernel(lee_ctx *ctx, int kind);
/* Form of the scalar fused filter (no reference counterpart; all forms give the same bits):
 * 0 (default) the fastest form, timed at lee_prepare; 1 one tile row per thread on tiles of 8
 * rows; 2 two rows per thread on tiles of 16 rows; 3 two neighbouring points per thread along xi
 * on tiles of 64 x 8 points (packed FP32 arithmetic: the compensated form on 3-D blocks of even
 * nxi). Forms 2 and 3 take no block with holes and not the vector kernel, form 3 nothing else
 * than its own case (LEE_ERR_UNSUPPORTED from lee_prepare), and with either the increment step
 * does not apply. Call before lee_prepare. */
int lee_set_filter_form(lee_ctx *ctx, int form);
/* Kernel of the RK stages on blocks that run the TMA stage kernel (no reference counterpart;
 * results agree to rounding): 1 one point per thread, 2 two neighbouring points per thread with
 * packed FP32 arithmetic (compensated form, uniform mean flow, even nxi); -1 (default) takes 2
 * where it applies, else 1. LEE_ERR_UNSUPPORTED from lee_prepare when a block cannot run the
 * choice. Call before lee_prepare. */
int lee_set_stage_kernel(lee_ctx *ctx, int kind);

/* ---- discrete adjoint (no reference counterpart: the reference has no adjoint) ----------
 * The step map of lee_advance is affine in the state; these entry points apply the exact
 * transpose of its linear part (transposed stencils and closures, transposed filter, reverse
 * RK stages) on any context lee_advance steps with one time step: every block, holes and their
 * closures, BC lines, sponges, overset interpolation (transposed receiver gather), non-uniform
 * mean flow and the axisymmetric term. A single-block, uniform-mean context without BC lines,
 * holes or overset runs the uniform-mean transposed kernels (plane-marching in 3-D); any other
 * the general per-point kernels. Sources and harmonic waves are the affine part and have no transpose. */
/* Objective J = weight * sum over steps n = 1..N of sum over microphones m of p'_n(l[m])^2,
 * p' of block b at linear indices l[m] (distinct) after every step. */
int lee_set_objective(lee_ctx *ctx, int b, int n, const long long *l, double weight);
/* Advance nsteps as lee_advance does and return J over those steps. */
int lee_eval_objective(lee_ctx *ctx, int nsteps, double dt, double *J);
/* Replace the uploaded state x (every block) by (M^T)^nsteps x, M^nsteps the linear part of
 * nsteps steps of lee_advance from an uploaded state (the dot-product test:
 * <l, M x> = <M^T l, x>; the first of those steps reads no rho'/rho_bar of a previous step). */
int lee_apply_adjoint(lee_ctx *ctx, int nsteps, double dt);
/* J over nsteps from the uploaded state and its gradient with respect to the amplitudes of
 * the LEE_SOURCE_DISTRIBUTED lattice (grad: cx*cy*cz values; the source's block and the
 * microphones' block may differ), by the discrete adjoint: the
 * forward pass records the microphone traces and keeps the state every checkpoint_every
 * steps; the reverse sweep goes segment by segment from the last. recompute = 1: each
 * segment's forward steps are run again from its checkpoint before its reverse sweep, and
 * *trace_mismatches counts recomputed trace values that differ from the first pass (0 when
 * the replay is bit-identical); recompute = 0: the first pass's traces drive the sweep (the
 * operator is linear, so the sweep needs no other forward state). On return the context
 * holds the state after nsteps. */
int lee_adjoint_gradient(lee_ctx *ctx, int nsteps, double dt, int checkpoint_every, int recompute, double *J,
                         double *grad, long long *trace_mismatches);
int lee_get_stats(lee_ctx *ctx, lee_stats *stats);

/* The filter of one field, with no device allocation (no counterpart in the reference: it
 * serves callers that cannot call cudaMalloc, such as a framework that owns the device
 * memory through its own allocator or a time loop that must not allocate). Applies the
 * dimension-split filter of spatial::apply_filter to one variable of one block without
 * holes: d_in and d_out are device arrays of nxi*neta*nzeta doubles (i fastest) that do not
 * overlap, owned by the caller and on the current device (as is `stream`); work is enqueued
 * on `stream` (a cudaStream_t, NULL for the default stream) and the call returns without
 * synchronizing. The intermediate passes use a
 * scratch array compiled into the library (2 x 2^20 doubles, held by every GPU that loads
 * the library until exit): fields above 2^20 points are refused with LEE_ERR_ARG. The first
 * call on each device looks up that array's device address; make it before any stream
 * capture. Calls share the array, so calls that overlap on the GPU race. Errors are
 * reported by lee_last_error(NULL). */
int lee_filter_field_static(int num_dim, int filter_scheme, int filter_order, double filter_strength,
                            double filter_blend, int nxi, int neta, int nzeta, const double *d_in, double *d_out,
                            void *stream);

#ifdef __cplusplus
}
#endif

#endif /* LEE_B200_H */
