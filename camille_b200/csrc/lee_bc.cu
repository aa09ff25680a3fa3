// Boundary update of a stage output (BC lines, then overset interpolation) and the rho'/rho_bar
// field of the next step's first stage.
//
// spatial::update_boundary (camille src/solver/spatial_discretization.cpp:2162-2187) applies
// bc::apply_BC (src/solver/boundary_condition.cpp:46-209) to the stage output z (or to y_next
// after the last stage): each BC line overwrites the non-hole points of its box's end face.
//  - neumann (:348-444): q_b = -sum_{s>=1} c_0s q_s / c_00 from row 0 of the difference
//    operator's boundary closure, mirrored on a right end;
//  - wall_slip_kinematic (:448-494): s' and p' as Neumann; the velocity is taken to the
//    contravariant components with the metrics, the wall-normal one is set to zero, and it
//    is brought back with the inverse metrics times J;
//  - centerline_cart_norm2x/y/z and centerline_axisym (:141-156, :498-574): Neumann, then the
//    velocity component along x/y/z (u_r', the second one, on the axis) is set to zero;
//  - dirichlet_allzero (:213-228): every slot zero;
//  - dirichlet_harmonicwave (:232-344): the time-harmonic wave at the update's time
//    (tn + c_{min(i+1, last)} h, RungeKutta::integrate, src/solver/temporal_discretization.cpp:232-244).
// BC lines run one launch each, in the order they were added, so a later line sees what an
// earlier one wrote (corners). Within one line a face point reads only points off the face
// (and its own velocity), so the update is in place.
//
// The arithmetic is FP64 with explicit round-to-nearest products and sums, in the reference's
// order. A compensated last-stage output is a pair (y_pre, e): it is read as y_pre + e and
// written back as the rounded value and its rounding error.
#include "lee_internal.h"

namespace lee {

namespace {

template <typename T, bool PAIR>
__device__ __forceinline__ double ld(const BcParams<T>& p, int v, long long l) {
  double x = (double)p.y[v][l];
  if (PAIR) x = __dadd_rn(x, (double)p.e[v][l]);
  return x;
}

template <typename T, bool PAIR>
__device__ __forceinline__ double neumann(const BcParams<T>& p, int v, long long l) {
  double d = 0.0;
  if (p.end == 0) {
    for (int s = 1; s < p.S; ++s) d = __dsub_rn(d, __dmul_rn(p.c0[s], ld<T, PAIR>(p, v, l + p.sd * s)));
    d = __ddiv_rn(d, p.c0[0]);
  } else {
    for (int s = 1; s < p.S; ++s) d = __dadd_rn(d, __dmul_rn(p.c0[s], ld<T, PAIR>(p, v, l - p.sd * s)));
    d = __ddiv_rn(d, -p.c0[0]);
  }
  return d;
}

template <typename T, bool PAIR>
__global__ void k_bc(BcParams<T> p) {
  const long long n = (long long)p.nb[0] * p.nb[1] * p.nb[2];
  for (long long lb = blockIdx.x * (long long)blockDim.x + threadIdx.x; lb < n;
       lb += (long long)gridDim.x * blockDim.x) {
    const int i = p.lo[0] + (int)(lb % p.nb[0]);
    const int j = p.lo[1] + (int)((lb / p.nb[0]) % p.nb[1]);
    const int k = p.lo[2] + (int)(lb / ((long long)p.nb[0] * p.nb[1]));
    const long long l = i + (long long)p.nx * (j + (long long)p.ny * k);
    if (p.iblank && p.iblank[l] == 1) continue;
    const int P = p.nd + 1;
    double out[kMaxVars];
    if (p.kind == LEE_BC_NEUMANN) {
      for (int v = 0; v < p.V; ++v) out[v] = neumann<T, PAIR>(p, v, l);
    } else if (p.kind >= LEE_BC_CENTERLINE_CART_NORM2X && p.kind <= LEE_BC_CENTERLINE_AXISYM) {
      for (int v = 0; v < p.V; ++v) out[v] = neumann<T, PAIR>(p, v, l);
      // the velocity along x/y/z, or u_r' (IVAR_UR, the second component) on the axis
      const int d = p.kind == LEE_BC_CENTERLINE_AXISYM ? 1 : p.kind - LEE_BC_CENTERLINE_CART_NORM2X;
      if (d < p.nd) out[1 + d] = 0.0;
    } else if (p.kind == LEE_BC_DIRICHLET_ALLZERO) {
      for (int v = 0; v < p.V; ++v) out[v] = 0.0;
    } else if (p.kind == LEE_BC_DIRICHLET_HARMONICWAVE) {
      for (int v = 0; v < p.V; ++v) out[v] = 0.0;
      const double x[3] = {p.xyz[0][l], p.xyz[1][l], p.xyz[2][l]};
      const double t = p.t_tab ? p.t_tab[(long long)*p.ctr * p.t_stride] : p.t;
      double ws, wu, wp;
      wave_eval(p.wave, x, t, &ws, &wu, &wp);
      out[0] = ws;
      if (p.wave.dir < p.nd) out[1 + p.wave.dir] = wu;
      out[P] = wp;
    } else {
      out[0] = neumann<T, PAIR>(p, 0, l);
      out[P] = neumann<T, PAIR>(p, P, l);
      double vel[3] = {0.0, 0.0, 0.0}, vc[3] = {0.0, 0.0, 0.0};
      for (int q = 0; q < p.nd; ++q) vel[q] = ld<T, PAIR>(p, 1 + q, l);
      for (int a = 0; a < p.nd; ++a) {
        double s = 0.0;
        for (int q = 0; q < p.nd; ++q) s = __dadd_rn(s, __dmul_rn(p.met[a * 3 + q][l], vel[q]));
        vc[a] = s;
      }
      vc[p.dir] = 0.0;
      const double jac = p.jac[l];
      for (int q = 0; q < p.nd; ++q) {
        double s = 0.0;
        for (int a = 0; a < p.nd; ++a) s = __dadd_rn(s, __dmul_rn(p.minv[q * 3 + a][l], vc[a]));
        out[1 + q] = __dmul_rn(s, jac);
      }
    }
    for (int v = 0; v < p.V; ++v) {
      const T r = (T)out[v];
      p.y[v][l] = r;
      if (PAIR) p.e[v][l] = (T)__dsub_rn(out[v], (double)r);
    }
  }
}

// The reference state of a harmonic-wave sponge zone (source::apply_bufferZone_Freund_harmonicWave,
// src/solver/source.cpp:264-320, reading bc::bc_dirichlet_harmonicwave): the wave at the stage
// time on the zone's box, zero in hole points, in the working precision.
template <typename T>
__global__ void k_wave_ref(WaveRefParams<T> p) {
  const long long n = (long long)p.nb[0] * p.nb[1] * p.nb[2];
  const double t = p.t_tab ? p.t_tab[(long long)*p.ctr * p.t_stride] : p.t;
  for (long long lb = blockIdx.x * (long long)blockDim.x + threadIdx.x; lb < n;
       lb += (long long)gridDim.x * blockDim.x) {
    const int i = p.lo[0] + (int)(lb % p.nb[0]);
    const int j = p.lo[1] + (int)((lb / p.nb[0]) % p.nb[1]);
    const int k = p.lo[2] + (int)(lb / ((long long)p.nb[0] * p.nb[1]));
    const long long l = i + (long long)p.nx * (j + (long long)p.ny * k);
    double out[kMaxVars] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (!p.iblank || p.iblank[l] != 1) {
      const double x[3] = {p.xyz[0][l], p.xyz[1][l], p.xyz[2][l]};
      double ws, wu, wp;
      wave_eval(p.wave, x, t, &ws, &wu, &wp);
      out[0] = ws;
      if (p.wave.dir < p.nd) out[1 + p.wave.dir] = wu;
      out[p.nd + 1] = wp;
    }
    for (int v = 0; v < p.V; ++v) p.out[v * n + lb] = (T)out[v];
  }
}

// rho'/rho_bar = p'/(gamma p_bar) - s' (State::compute_auxiliary_variables_linear_Euler,
// src/core/state.cpp:701-736, divided by rho_bar).
template <typename T, bool PAIR>
__global__ void k_rho(long long n, const T* ys, const T* yp, const T* es, const T* ep, const double* pbar,
                      double inv_gamma, T* out) {
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < n; l += (long long)gridDim.x * blockDim.x) {
    double s = (double)ys[l], q = (double)yp[l];
    if (PAIR) {
      s += (double)es[l];
      q += (double)ep[l];
    }
    out[l] = (T)(q * inv_gamma * (1.0 / pbar[l]) - s);
  }
}

// overset::interpolate (src/overset/overset.cpp:820-845): compute_weighted_sum (:886-974) sums
// coeff * y over the stencil, zeta outermost and xi innermost, from 0.0 for every variable;
// update_each_grid (:1241-1278) overwrites the receivers. One thread per receiver.
template <typename T, bool PAIR>
__device__ __forceinline__ double ovs_ld(const OvsParams<T>& p, int b, int v, long long l) {
  double x = (double)p.y[b][v][l];
  if (PAIR) x = __dadd_rn(x, (double)p.e[b][v][l]);
  return x;
}

template <typename T, bool PAIR>
__device__ __forceinline__ void ovs_st(const OvsParams<T>& p, int b, int v, long long l, double x) {
  const T r = (T)x;
  p.y[b][v][l] = r;
  if (PAIR) p.e[b][v][l] = (T)__dsub_rn(x, (double)r);
}

template <typename T, bool PAIR>
__global__ void k_ovs_gather(OvsParams<T> p) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= p.n) return;
  const int d = p.db[r];
  const long long nx = p.nx[d], nxy = nx * p.ny[d];
  const long long base = p.dl[r];
  const double* cf = p.wt + (long long)r * p.W;
  double acc[kMaxVars] = {0.0, 0.0, 0.0, 0.0, 0.0};
  int st = 0;
  for (int w3 = 0; w3 < p.w[2]; ++w3)
    for (int w2 = 0; w2 < p.w[1]; ++w2)
      for (int w1 = 0; w1 < p.w[0]; ++w1) {
        const long long l1 = base + w1 + w2 * nx + w3 * nxy;
        const double c = cf[st++];
        for (int v = 0; v < p.V; ++v) acc[v] = __dadd_rn(acc[v], __dmul_rn(c, ovs_ld<T, PAIR>(p, d, v, l1)));
      }
  if (p.fused) {
    for (int v = 0; v < p.V; ++v) ovs_st<T, PAIR>(p, p.rb[r], v, p.rl[r], acc[v]);
  } else {
    for (int v = 0; v < p.V; ++v) p.buf[(long long)r * p.V + v] = acc[v];
  }
}

template <typename T, bool PAIR>
__global__ void k_ovs_scatter(OvsParams<T> p) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= p.n) return;
  for (int v = 0; v < p.V; ++v) ovs_st<T, PAIR>(p, p.rb[r], v, p.rl[r], p.buf[(long long)r * p.V + v]);
}

int grid_for(long long n) {
  long long g = (n + 255) / 256;
  return (int)(g < 1 ? 1 : (g > 148 * 16 ? 148 * 16 : g));
}

}  // namespace

template <typename T>
cudaError_t launch_bc(const BcParams<T>& p, cudaStream_t s) {
  const long long n = (long long)p.nb[0] * p.nb[1] * p.nb[2];
  if (p.e[0]) k_bc<T, true><<<grid_for(n), 256, 0, s>>>(p);
  else k_bc<T, false><<<grid_for(n), 256, 0, s>>>(p);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_rho(long long n, int V, T* const* y, T* const* e, const double* pbar, double gamma, T* out,
                       cudaStream_t s) {
  const int P = V - 1;
  if (e) k_rho<T, true><<<grid_for(n), 256, 0, s>>>(n, y[0], y[P], e[0], e[P], pbar, 1.0 / gamma, out);
  else k_rho<T, false><<<grid_for(n), 256, 0, s>>>(n, y[0], y[P], nullptr, nullptr, pbar, 1.0 / gamma, out);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_overset(const OvsParams<T>& p, cudaStream_t s) {
  if (p.n <= 0) return cudaSuccess;
  const int g = (p.n + 127) / 128;
  if (p.pair) {
    k_ovs_gather<T, true><<<g, 128, 0, s>>>(p);
    if (!p.fused) k_ovs_scatter<T, true><<<g, 128, 0, s>>>(p);
  } else {
    k_ovs_gather<T, false><<<g, 128, 0, s>>>(p);
    if (!p.fused) k_ovs_scatter<T, false><<<g, 128, 0, s>>>(p);
  }
  return cudaGetLastError();
}

template cudaError_t launch_overset<double>(const OvsParams<double>&, cudaStream_t);
template cudaError_t launch_overset<float>(const OvsParams<float>&, cudaStream_t);
template <typename T>
cudaError_t launch_wave_ref(const WaveRefParams<T>& p, cudaStream_t s) {
  const long long n = (long long)p.nb[0] * p.nb[1] * p.nb[2];
  k_wave_ref<T><<<grid_for(n), 256, 0, s>>>(p);
  return cudaGetLastError();
}

template cudaError_t launch_wave_ref<double>(const WaveRefParams<double>&, cudaStream_t);
template cudaError_t launch_wave_ref<float>(const WaveRefParams<float>&, cudaStream_t);
template cudaError_t launch_bc<double>(const BcParams<double>&, cudaStream_t);
template cudaError_t launch_bc<float>(const BcParams<float>&, cudaStream_t);
template cudaError_t launch_rho<double>(long long, int, double* const*, double* const*, const double*, double, double*,
                                        cudaStream_t);
template cudaError_t launch_rho<float>(long long, int, float* const*, float* const*, const double*, double, float*,
                                       cudaStream_t);

}  // namespace lee
