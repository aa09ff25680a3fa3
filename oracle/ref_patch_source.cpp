// Oracle patch P2: a parameterised monopole pressure source for the compiled
// camille reference (test infrastructure only).
//
// The reference has no source matching the overset and batched workloads; its
// closest case is the fixed Gaussian sin(8 pi t) source with a sin^2 ramp of
// CASE_SCATTERING_TWOCYLINDER (src/solver/source.cpp:60-92). This function adds
//   rhs[p'] += A (gamma - 1) ramp(t) exp(-ln2 r^2 / b^2) sin(omega t)
// with ramp(t) = sin^2(pi/2 t / T) for t < T (T <= 0 disables the ramp), where r
// is the distance to (x0, y0, z0). build_ref.py inserts one call to it into the
// otherwise empty CASE_KBK_COMBUSTOR branch of source::apply_physicalSource; it
// is active only when ORACLE_MONOPOLE="x0,y0,z0,A,omega,b,T" is set.
#include <cmath>
#include <cstdio>
#include <cstdlib>

#include "core/state.h"
#include "geometry/geometry.h"

void oracle_monopole_source(Geometry::StructuredGrid *mygrid, State *mystate, double **rhs, double time) {
  const char *env = std::getenv("ORACLE_MONOPOLE");
  if (!env) return;
  double x0, y0, z0, amp, omega, b, ramp_time;
  if (std::sscanf(env, "%lf,%lf,%lf,%lf,%lf,%lf,%lf", &x0, &y0, &z0, &amp, &omega, &b, &ramp_time) != 7) {
    std::fprintf(stderr, "ORACLE_MONOPOLE needs 7 comma-separated numbers\n");
    std::exit(4);
  }
  double ramp = 1.0;
  if (ramp_time > 0.0 && time < ramp_time) {
    double s = std::sin(0.5 * M_PI * time / ramp_time);
    ramp = s * s;
  }
  double fac = amp * (mystate->gamma_specificheat - 1.0) * ramp * std::sin(omega * time);
  double ef = -std::log(2.0) / (b * b);
  for (int l0 = 0; l0 < mystate->num_samples; ++l0) {
    double dx = mygrid->cell[l0].xyz[XDIR] - x0;
    double dy = mygrid->cell[l0].xyz[YDIR] - y0;
    double dz = mygrid->cell[l0].xyz[ZDIR] - z0;
    (rhs[IVAR_P])[l0] += fac * std::exp(ef * (dx * dx + dy * dy + dz * dz));
  }
}
