// Oracle driver for the compiled camille reference (test infrastructure only).
//
// Replaces the reference's 9-line main (src/core/main.cpp:3-9) so that the
// oracle can (a) time the reference's own solver loop `solver::solve`
// (src/solver/solver.cpp:41-89) without setup or I/O, and (b) expose its inner
// seams one at a time: one right-hand side (spatial::compute_RHS,
// src/solver/spatial_discretization.cpp:1963-1990), one filter application
// (spatial::apply_filter, :2191-2246), and the setup products (metrics::compute,
// src/metrics/metrics.cpp:9-44; mean gradients, spatial_discretization.cpp:2250-2271;
// LEE auxiliaries, src/core/state.cpp:701-736).
//
// Controlled by environment variables (argv[1] stays the reference's restart file):
//   ORACLE_MODE = run | rhs | filter | setup | overset   (default run)
//   ORACLE_DUMP = path prefix; each rank writes <prefix>.<rank>.bin
// Dump layout: int32 magic 0x4C454532, block id, iso_in_parent[3], n_dir[3],
// nfields, time_step, is[3], ie[3] (the points this rank owns, local indices
// without ghost cells); float64 time_sol, dt; then nfields x N float64 fields,
// i fastest (the reference's idx1D, src/geometry/geometry.h:131-136).
//
// The reference exits 0 on fatal errors (src/parallel/parallel.cpp:78-96), so
// this driver prints "ORACLE_OK" last; harnesses treat its absence as failure.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "core/simulation.h"
#include "overset/overset.h"

namespace {

void dump(const char *prefix, const std::vector<double *> &fields) {
  if (!prefix) return;
  Geometry::StructuredGrid *g = simulation::grid;
  std::string path = std::string(prefix) + "." + std::to_string(mpi::irank) + ".bin";
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) {
    std::fprintf(stderr, "oracle driver: cannot open %s\n", path.c_str());
    std::exit(3);
  }
  int hdr[16];
  hdr[0] = 0x4C454532;
  hdr[1] = g->id_parent;
  for (int d = 0; d < 3; ++d) hdr[2 + d] = g->iso_in_parent[d];
  for (int d = 0; d < 3; ++d) hdr[5 + d] = g->num_ocells_dir[d];
  hdr[8] = (int)fields.size();
  hdr[9] = simulation::state.time_step;
  for (int d = 0; d < 3; ++d) hdr[10 + d] = g->is[d];
  for (int d = 0; d < 3; ++d) hdr[13 + d] = g->ie[d];
  std::fwrite(hdr, sizeof(int), 16, f);
  double td[2] = {simulation::state.time_sol, temporal::dt};
  std::fwrite(td, sizeof(double), 2, f);
  for (double *p : fields) std::fwrite(p, sizeof(double), (size_t)g->num_ocells, f);
  std::fclose(f);
}

}  // namespace

int main(int argc, char *argv[]) {
  const char *mode_env = std::getenv("ORACLE_MODE");
  std::string mode = mode_env ? mode_env : "run";
  const char *prefix = std::getenv("ORACLE_DUMP");

  simulation::initialize(argc, argv);
  State &st = simulation::state;
  Geometry::StructuredGrid *g = simulation::grid;
  int nv = st.num_vars_sol;
  int N = g->num_ocells;

  if (mode == "run") {
    MPI_Barrier(MPI_COMM_WORLD);
    auto t0 = std::chrono::steady_clock::now();
    simulation::run();
    MPI_Barrier(MPI_COMM_WORLD);
    auto t1 = std::chrono::steady_clock::now();
    double sec = std::chrono::duration<double>(t1 - t0).count();
    std::vector<double *> f(st.sol, st.sol + nv);
    dump(prefix, f);
    if (mpi::irank == 0)
      std::printf("ORACLE_RESULT {\"seconds\": %.9g, \"steps\": %d, \"time_sol\": %.17g, "
                  "\"dt\": %.17g, \"nprocs\": %d, \"cfl_max\": %.17g}\n",
                  sec, temporal::time_step - temporal::time_step_lastrun, st.time_sol, temporal::dt,
                  mpi::nprocs, temporal::cfl_max);
  } else if (mode == "rhs") {
    std::vector<double *> rhs((size_t)nv);
    for (auto &p : rhs) p = new double[(size_t)N];
    spatial::compute_RHS(&simulation::myinput, g, &st, st.sol, rhs.data(), st.time_sol);
    dump(prefix, rhs);
  } else if (mode == "filter") {
    spatial::apply_filter(nv, N, st.sol, g);
    std::vector<double *> f(st.sol, st.sol + nv);
    dump(prefix, f);
  } else if (mode == "setup") {
    int nd = st.num_dim;
    std::vector<double *> f;
    std::vector<std::vector<double>> store(12, std::vector<double>((size_t)N));
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c)
        for (int l = 0; l < N; ++l) store[(size_t)(r * 3 + c)][(size_t)l] = g->cell[l].metrics[r][c];
    for (int l = 0; l < N; ++l) store[9][(size_t)l] = g->cell[l].Jac;
    for (int l = 0; l < N; ++l) store[10][(size_t)l] = g->cell[l].invJac;
    for (int l = 0; l < N; ++l) store[11][(size_t)l] = (double)g->cell[l].iblank;
    for (int k = 0; k < 12; ++k) f.push_back(store[(size_t)k].data());
    for (int v = 0; v < st.num_vars_mean * nd; ++v) f.push_back(st.sol_meanGradient[v]);
    for (int v = 0; v < st.num_vars_aux; ++v) f.push_back(st.sol_aux[v]);
    // Sponge strength summed over zones, laid out on the grid.
    std::vector<double> sig((size_t)N, 0.0);
    for (int z = 0; z < g->num_bufferZones; ++z) {
      Geometry::StructuredBufferZone *bz = &g->bufferZone[z];
      for (int k = bz->is[ZETA]; k <= bz->ie[ZETA]; ++k)
        for (int j = bz->is[ETA]; j <= bz->ie[ETA]; ++j)
          for (int i = bz->is[XI]; i <= bz->ie[XI]; ++i) {
            int lb = bz->idx1D(i, j, k);
            int l0 = g->idx1D(i - bz->is[XI] + bz->is_in_parent[XI], j - bz->is[ETA] + bz->is_in_parent[ETA],
                              k - bz->is[ZETA] + bz->is_in_parent[ZETA]);
            sig[(size_t)l0] += bz->buffer_strength[lb];
          }
    }
    f.push_back(sig.data());
    dump(prefix, f);
    if (mpi::irank == 0)
      std::printf("ORACLE_SETUP {\"num_dim\": %d, \"n_mean_grad\": %d, \"n_aux\": %d, \"zones\": %d}\n", nd,
                  st.num_vars_mean * nd, st.num_vars_aux, g->num_bufferZones);
  } else if (mode == "overset") {
    // the donor and receiver maps this rank holds after overset::initialize_overset
    // (src/overset/overset.cpp:436-554): <prefix>.<rank>.ovs with int32 block id, int32
    // number of donor cells, per donor cell int32 l0, int32 num_coeffs and float64 coeffs
    // (normalised), then int32 number of receiver cells and their int32 l0
    if (prefix) {
      std::string path = std::string(prefix) + "." + std::to_string(mpi::irank) + ".ovs";
      FILE *f = std::fopen(path.c_str(), "wb");
      if (!f) return 3;
      int hdr[2] = {g->id_parent, overset::num_donorCells_in_this_grid};
      std::fwrite(hdr, sizeof(int), 2, f);
      for (int d = 0; d < overset::num_donorCells_in_this_grid; ++d) {
        int rec[2] = {overset::donorCells[d].l0, overset::donorCells[d].num_coeffs};
        std::fwrite(rec, sizeof(int), 2, f);
        std::fwrite(overset::donorCells[d].coeff, sizeof(double), (size_t)rec[1], f);
      }
      int nr = overset::total_num_donorCells_4mygrid;
      std::fwrite(&nr, sizeof(int), 1, f);
      for (int r = 0; r < nr; ++r) std::fwrite(&overset::receiverCells[r].l0, sizeof(int), 1, f);
      std::fclose(f);
    }
    std::vector<double> ib((size_t)N);
    for (int l = 0; l < N; ++l) ib[(size_t)l] = (double)g->cell[l].iblank;
    std::vector<double *> f(1, ib.data());
    dump(prefix, f);
  } else {
    std::fprintf(stderr, "oracle driver: unknown ORACLE_MODE %s\n", mode.c_str());
    return 2;
  }
  std::fflush(stdout);
  MPI_Barrier(MPI_COMM_WORLD);
  if (mpi::irank == 0) std::printf("ORACLE_OK\n");
  std::fflush(stdout);
  simulation::finalize();  // exits the process
  return 0;
}
