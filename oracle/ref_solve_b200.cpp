// The replacement of the camille reference's src/solver/solver.cpp that hands the time advance to
// the B200 library through its C ABI (include/lee_b200.h): the reference-side binding a
// maintainer adds. It is compiled against the reference's own headers, linked with the rest of
// the reference (its main, deck reader, PLOT3D and BC-file I/O, reports and solution writes) and
// with camille_b200/liblee_b200.so by oracle/build_integration.py, and run by
// tests/test_integration_gpu.py on the reference's own input files.
//
// solver::initialize / finalize / precompute_something keep the reference's behaviour (they set
// up the temporal and spatial modules whose globals -- dt, the step counters, FIX_DT or FIX_CFL --
// the step loop reads); solver::solve (src/solver/solver.cpp:41-89) becomes:
//   lee_create / lee_set_block / lee_set_mean / one lee_add_boundary per sponge zone and BC line /
//   lee_prepare / lee_upload_state, then the reference's step loop with lee_compute_cfl for the
//   FIX_CFL rescale (the reference's CFL, integer truncation included), lee_advance over runs of
//   steps between reports, and at every report step lee_download_state followed by the
//   reference's own io::report_timeadvancing and io::write_solution_on_the_fly.
// One rank holding one whole block (no ghost cells); anything else stops with the reference's
// own graceful exit.
#include <cmath>
#include <cstdlib>
#include <string>
#include <vector>

#include "lee_b200.h"
#include "solver.h"

namespace solver {

void initialize(UserInput *myinput, Geometry::StructuredGrid *mygrid, State *mystate) {
  temporal::initialize(myinput, mystate);
  spatial::initialize(myinput, mygrid, mystate);
}

void finalize() {
  temporal::finalize();
  spatial::finalize();
}

void precompute_something(UserInput *myinput, Geometry::StructuredGrid *mygrid, State *mystate) {
  temporal::precompute_something(myinput, mygrid, mystate);
  spatial::precompute_something(myinput, mygrid, mystate);
}

namespace {

void check(lee_ctx *ctx, int rc, const char *what) {
  if (rc == LEE_OK) return;
  std::string msg = std::string("lee_b200: ") + what + ": " + lee_last_error(ctx);
  mpi::graceful_exit(msg);
}

int wave_type(const std::string &s) { return s == "WAVE_ACOUSTIC" ? LEE_WAVE_ACOUSTIC : LEE_WAVE_ENTROPY; }

int wave_form(const std::string &s) {
  if (s == "WAVEFORM_PLANE") return LEE_WAVEFORM_PLANE;
  if (s == "WAVEFORM_HOMOGENEOUS") return LEE_WAVEFORM_HOMOGENEOUS;
  return LEE_WAVEFORM_GAUSSIAN_ROUNDJET;
}

}  // namespace

void solve(UserInput *myinput, Geometry::StructuredGrid *mygrid, Geometry::StructuredBlock *block, State *mystate) {
  if (mpi::nprocs != 1 || myinput->do_overset)
    mpi::graceful_exit("lee_b200 binding: one rank holding one block (no overset) is supported");
  if (myinput->model_pde != "LEE" && myinput->model_pde != "LEE_SCALAR")
    mpi::graceful_exit("lee_b200 binding: PHYSICAL_MODEL = LEE or LEE_SCALAR");
  const int nsc = myinput->model_pde == "LEE_SCALAR" ? myinput->num_scalar : 0;  // slots after p'


  lee_config cfg = {};
  cfg.num_dim = myinput->num_dim;
  cfg.num_blocks = 1;
  cfg.gamma = myinput->gamma_specificheat;
  cfg.fd_scheme = myinput->spatial_scheme == "FDO11P" ? LEE_FD_FDO11P : LEE_FD_STANDARD_CENTRAL;
  cfg.fd_order = myinput->OA_spatial;
  cfg.filter_scheme = !myinput->do_filter                      ? LEE_FILTER_NONE
                      : myinput->filter_scheme == "SFO11P"     ? LEE_FILTER_SFO11P
                                                               : LEE_FILTER_STANDARD_CENTRAL;
  cfg.filter_order = myinput->OA_filter;
  cfg.filter_strength = myinput->filter_strength;
  cfg.filter_blend = myinput->filter_blend;
  cfg.rk_scheme = myinput->temporal_scheme == "RUNGE_KUTTA2" ? LEE_RK2 : LEE_RK4;
  const char *prec = std::getenv("LEE_B200_PRECISION");
  cfg.precision = prec && std::string(prec) == "fp32c" ? LEE_FP32_COMPENSATED : LEE_FP64;
  cfg.sponge_order = myinput->buffer_polynomial_order;
  cfg.sponge_constant = myinput->buffer_constant;
  cfg.device = 0;
  lee_ctx *ctx = nullptr;
  check(nullptr, lee_create(&cfg, &ctx), "lee_create");
  if (nsc) check(ctx, lee_set_scalars(ctx, nsc), "lee_set_scalars");

  // the block: one rank owns it whole, so the grid has no ghost cells (src/geometry/geometry.cpp:109-132)
  const int nx = mygrid->nXi, ny = mygrid->nEta, nz = mygrid->nZeta;
  const int n = mygrid->num_ocells;
  if (n != nx * ny * nz || mygrid->num_cells != n)
    mpi::graceful_exit("lee_b200 binding: the rank's grid carries ghost cells");
  std::vector<double> x(n), y(n), z(n);
  std::vector<int> ib(n);
  for (int l = 0; l < n; ++l) {  // GridPoint is an array of structures: gather xyz and iblank
    x[l] = mygrid->cell[l].xyz[XI];
    y[l] = mygrid->cell[l].xyz[ETA];
    z[l] = mygrid->cell[l].xyz[ZETA];
    ib[l] = mygrid->cell[l].iblank;
  }
  check(ctx, lee_set_block(ctx, 0, nx, ny, nz, x.data(), y.data(), z.data(), ib.data()), "lee_set_block");
  check(ctx, lee_set_mean(ctx, 0, mystate->sol_mean), "lee_set_mean");
  if (nsc) check(ctx, lee_set_mean_scalars(ctx, 0, mystate->sol_mean + 5), "lee_set_mean_scalars");
  // BC lines and sponge zones in the BC file's order; sponges pass the strengths the reference
  // computed (Geometry::StructuredBufferZone::buffer_strength, the zone box, xi fastest)
  for (int q = 0; q < mygrid->num_boundaryCondition_nonperiodic; ++q) {
    Geometry::StructuredBoundaryCondition *bc = &mygrid->boundaryCondition[q];
    check(ctx, lee_add_boundary(ctx, 0, bc->which_model, bc->which_dir, bc->which_end, bc->is_in_parent,
                                bc->ie_in_parent, nullptr),
          "lee_add_boundary (BC line)");
  }
  for (int q = 0; q < mygrid->num_bufferZones; ++q) {
    Geometry::StructuredBufferZone *bz = &mygrid->bufferZone[q];
    check(ctx, lee_add_boundary(ctx, 0, bz->which_model, bz->which_dir, bz->which_end, bz->is_in_parent,
                                bz->ie_in_parent, bz->buffer_strength),
          "lee_add_boundary (sponge)");
  }
  if (myinput->harmonicWave_waveType != "NONE")
    check(ctx,
          lee_set_harmonic_wave(ctx, wave_type(myinput->harmonicWave_waveType), wave_form(myinput->harmonicWave_waveForm),
                                myinput->harmonicWave_idir_propagation, myinput->harmonicWave_amplitude,
                                myinput->harmonicWave_wavelength, myinput->harmonicWave_halfWidth),
          "lee_set_harmonic_wave");
  if (myinput->axisym) check(ctx, lee_set_axisymmetric(ctx, 1, myinput->axis_of_sym), "lee_set_axisymmetric");
  if (mystate->simulation == "CASE_2DJET_WITH_A_HARMONIC_SOURCE")
    check(ctx, lee_set_source(ctx, LEE_SOURCE_JET2D_HARMONIC, nullptr, 0), "lee_set_source");
  check(ctx, lee_prepare(ctx), "lee_prepare");
  check(ctx, lee_upload_state(ctx, 0, mystate->sol, mystate->time_step, mystate->time_sol), "lee_upload_state");
  if (nsc) check(ctx, lee_upload_scalars(ctx, 0, mystate->sol + 5), "lee_upload_scalars");

  // solver::solve's loop (src/solver/solver.cpp:41-89): FIX_CFL rescales dt every step from the
  // CFL of the previous dt; FIX_DT advances whole runs of steps between reports
  const bool fix_cfl = temporal::fix_dt_or_cfl == "FIX_CFL";
  double dt = temporal::dt;
  for (int s = temporal::time_step_lastrun + 1; s <= temporal::num_time_steps;) {
    double cfl = 0.0;
    check(ctx, lee_compute_cfl(ctx, dt, &cfl), "lee_compute_cfl");
    if (fix_cfl) {
      dt *= temporal::cfl_max / cfl;
      temporal::dt = dt;
    } else {
      temporal::cfl_max = cfl;
    }
    const int next_report = ((s + myinput->report_freq - 1) / myinput->report_freq) * myinput->report_freq;
    const int steps = fix_cfl ? 1 : std::min(next_report, temporal::num_time_steps) - s + 1;
    check(ctx, lee_advance(ctx, steps, dt), "lee_advance");
    s += steps;
    const int done = s - 1;
    if (done % myinput->report_freq == 0 || done == temporal::num_time_steps) {
      check(ctx, lee_download_state(ctx, 0, mystate->sol, &mystate->time_step, &mystate->time_sol),
            "lee_download_state");
      if (nsc) check(ctx, lee_download_scalars(ctx, 0, mystate->sol + 5), "lee_download_scalars");
      temporal::time_step = mystate->time_step;
      temporal::time_sol = mystate->time_sol;
      if (done % myinput->report_freq == 0) {
        io::report_timeadvancing(temporal::time_step, temporal::time_sol, dt, cfl, myinput, mygrid, mystate);
        io::write_solution_on_the_fly(myinput, mygrid, block, mystate, temporal::num_time_steps);
      }
    }
  }
  lee_destroy(ctx);
}

}  // namespace solver
