// One-time setup on the GPU in FP64: directional operators for the metric and
// mean-gradient generation, Thomas-Lombard products, Jacobian, inverse metrics,
// sponge strengths, CFL, and coefficient-field reductions.
//
// This translation unit is compiled with --fmad=false so that every product and
// sum rounds exactly as the reference's x86-64 build does (no contraction).
#include <cfloat>

#include "lee_internal.h"

namespace lee {
namespace {

constexpr int kThreads = 256;

inline int blocks_for(long long n) { return (int)((n + kThreads - 1) / kThreads); }

// Operator application at one point, in the reference's order of summation:
// interior stencil l = -h..h; closure rows s = 0..S-1 (src/solver/spatial_discretization.cpp:1094-1149,
// :1656-1745).
__device__ double op_point(const OpTable& op, const double* f, long long l0, int i, int n, long long sd, int code) {
  double acc = 0.0;
  if (code == kCodeZero) return 0.0;
  if (code == 0) {
    for (int l = -op.h; l <= op.h; ++l) acc += op.c[l + op.h] * f[l0 + l * sd];
    return acc;
  }
  if (code > 0) {
    int r = code - 1;
    long long a = l0 - r * sd;
    for (int s = 0; s < op.S; ++s) acc += op.B[r][s] * f[a + s * sd];
    return acc;
  }
  int r = -code - 1;
  long long a = l0 + r * sd;
  for (int s = 0; s < op.S; ++s) acc += op.mfac * op.B[r][s] * f[a - s * sd];
  return acc;
}

__global__ void k_apply_dir(OpTable op, int nx, int ny, int nz, int dir, const double* __restrict__ f,
                            double* __restrict__ out, const int8_t* __restrict__ code) {
  long long N = (long long)nx * ny * nz;
  for (long long l0 = blockIdx.x * (long long)blockDim.x + threadIdx.x; l0 < N;
       l0 += (long long)gridDim.x * blockDim.x) {
    int i = (int)(l0 % nx);
    int j = (int)((l0 / nx) % ny);
    int k = (int)(l0 / ((long long)nx * ny));
    int n = dir == 0 ? nx : (dir == 1 ? ny : nz);
    int p = dir == 0 ? i : (dir == 1 ? j : k);
    long long sd = dir == 0 ? 1 : (dir == 1 ? (long long)nx : (long long)nx * ny);
    int c;
    if (code) {
      c = code[l0];
    } else if (p >= op.h && p <= n - 1 - op.h) {
      c = 0;
    } else if (p < op.h) {
      c = 1 + p;
    } else {
      c = -(1 + (n - 1 - p));
    }
    out[l0] = op_point(op, f, l0, p, n, sd, c);
  }
}

__global__ void k_fill(long long n, double* out, double v) {
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < n; l += (long long)gridDim.x * blockDim.x)
    out[l] = v;
}

__global__ void k_copy(long long n, double* out, const double* in) {
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < n; l += (long long)gridDim.x * blockDim.x)
    out[l] = in[l];
}

__global__ void k_axpby(long long n, double* out, double a, const double* x, double b, const double* y) {
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < n; l += (long long)gridDim.x * blockDim.x)
    out[l] = y ? a * x[l] + b * y[l] : a * x[l];
}

__global__ void k_mul(long long n, double* out, const double* x, const double* y) {
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < n; l += (long long)gridDim.x * blockDim.x)
    out[l] = x[l] * y[l];
}

// metrics::compute_Jacobian (src/metrics/metrics.cpp:255-328), 3-D with oracle patch P1.
__global__ void k_jacobian(long long n, int dim, const double* const* xx, double* invjac, double* jac) {
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < n; l += (long long)gridDim.x * blockDim.x) {
    double v;
    if (dim == 2) {
      v = xx[0][l] * xx[4][l] - xx[1][l] * xx[3][l];
    } else {
      v = xx[0][l] * (xx[4][l] * xx[8][l] - xx[5][l] * xx[7][l])
        - xx[1][l] * (xx[3][l] * xx[8][l] - xx[5][l] * xx[6][l])
        + xx[2][l] * (xx[3][l] * xx[7][l] - xx[4][l] * xx[6][l]);
    }
    invjac[l] = v;
    jac[l] = 1.0 / v;
  }
}

// metrics::compute_metricsInverse (src/metrics/metrics.cpp:355-426).
__global__ void k_inverse(long long n, int dim, const double* const* m, double* const* mi) {
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < n; l += (long long)gridDim.x * blockDim.x) {
#define M(a, b) m[(a) * 3 + (b)][l]
    if (dim == 2) {
      mi[0][l] = M(1, 1);
      mi[1][l] = -M(0, 1);
      mi[3][l] = -M(1, 0);
      mi[4][l] = M(0, 0);
    } else {
      mi[0][l] = M(1, 1) * M(2, 2) - M(1, 2) * M(2, 1);
      mi[1][l] = M(0, 2) * M(2, 1) - M(0, 1) * M(2, 2);
      mi[2][l] = M(0, 1) * M(1, 2) - M(0, 2) * M(1, 1);
      mi[3][l] = M(1, 2) * M(2, 0) - M(1, 0) * M(2, 2);
      mi[4][l] = M(0, 0) * M(2, 2) - M(0, 2) * M(2, 0);
      mi[5][l] = M(0, 2) * M(1, 0) - M(0, 0) * M(1, 2);
      mi[6][l] = M(1, 0) * M(2, 1) - M(1, 1) * M(2, 0);
      mi[7][l] = M(0, 1) * M(2, 0) - M(0, 0) * M(2, 1);
      mi[8][l] = M(0, 0) * M(1, 1) - M(0, 1) * M(1, 0);
    }
#undef M
  }
}

__global__ void k_grad_accum(long long n, double* sum, const double* m, const double* d) {
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < n; l += (long long)gridDim.x * blockDim.x)
    sum[l] += m[l] * d[l];
}

__global__ void k_scale(long long n, double* out, const double* sum, const double* jac) {
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < n; l += (long long)gridDim.x * blockDim.x)
    out[l] = sum[l] * jac[l];
}

// Geometry::additionalInit_bufferZones (src/geometry/geometry.cpp:1028-1142): brute-force
// minimum distance to the zone's IN and OUT faces, sigma = C (d_in/(d_in+d_out))^order.
__global__ void k_sigma(int nx, int ny, const double* const* xyz, int lo0, int lo1, int lo2, int hi0, int hi1, int hi2,
                        int dir, int end, int order, double constant, double* sig) {
  int b0 = hi0 - lo0 + 1, b1 = hi1 - lo1 + 1, b2 = hi2 - lo2 + 1;
  long long nb = (long long)b0 * b1 * b2;
  int lo[3] = {lo0, lo1, lo2}, hi[3] = {hi0, hi1, hi2};
  int fin = end == 0 ? hi[dir] : lo[dir];
  int fout = end == 0 ? lo[dir] : hi[dir];
  for (long long lb = blockIdx.x * (long long)blockDim.x + threadIdx.x; lb < nb; lb += (long long)gridDim.x * blockDim.x) {
    int i = lo0 + (int)(lb % b0), j = lo1 + (int)((lb / b0) % b1), k = lo2 + (int)(lb / ((long long)b0 * b1));
    long long l0 = i + (long long)nx * (j + (long long)ny * k);
    double xb0 = xyz[0][l0], xb1 = xyz[1][l0], xb2 = xyz[2][l0];
    double dist[2];
    for (int side = 0; side < 2; ++side) {
      int flo[3] = {lo0, lo1, lo2}, fhi[3] = {hi0, hi1, hi2};
      flo[dir] = fhi[dir] = side == 0 ? fin : fout;
      double dmin = 1000000000.0;
      for (int kk = flo[2]; kk <= fhi[2]; ++kk)
        for (int jj = flo[1]; jj <= fhi[1]; ++jj)
          for (int ii = flo[0]; ii <= fhi[0]; ++ii) {
            long long lf = ii + (long long)nx * (jj + (long long)ny * kk);
            double d0 = xb0 - xyz[0][lf], d1 = xb1 - xyz[1][lf], d2 = xb2 - xyz[2][lf];
            double s = 0.0;
            s += d0 * d0;
            s += d1 * d1;
            s += d2 * d2;
            dmin = s < dmin ? s : dmin;
          }
      dist[side] = sqrt(dmin);
    }
    double rel = dist[0] / (dist[0] + dist[1]);
    double pw = 1.0;
    for (int q = 0; q < order; ++q) pw *= rel;
    sig[lb] = constant * pw;
  }
}

__device__ double atomic_max_double(double* addr, double v) {
  unsigned long long* a = (unsigned long long*)addr;
  unsigned long long old = *a, assumed;
  do {
    assumed = old;
    if (__longlong_as_double(assumed) >= v) break;
    old = atomicCAS(a, assumed, __double_as_longlong(v));
  } while (assumed != old);
  return __longlong_as_double(old);
}

__global__ void k_minmax(long long n, const double* f, double* out2) {
  __shared__ double smin[kThreads], smax[kThreads];
  double lo = DBL_MAX, hi = -DBL_MAX;
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < n; l += (long long)gridDim.x * blockDim.x) {
    double v = f[l];
    lo = v < lo ? v : lo;
    hi = v > hi ? v : hi;
  }
  smin[threadIdx.x] = lo;
  smax[threadIdx.x] = hi;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      smin[threadIdx.x] = fmin(smin[threadIdx.x], smin[threadIdx.x + s]);
      smax[threadIdx.x] = fmax(smax[threadIdx.x], smax[threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    atomic_max_double(&out2[0], -smin[0]);
    atomic_max_double(&out2[1], smax[0]);
  }
}

// Minimum and maximum of one state field, the value of a point being y (FP64) or fl64(y) + fl64(e)
// (a compensated FP32 pair): out2[0] collects -min and out2[1] max, both by atomic maximum.
template <typename T>
__global__ void k_state_minmax(long long n, const T* y, const T* e, double* out2) {
  __shared__ double smin[kThreads], smax[kThreads];
  double lo = DBL_MAX, hi = -DBL_MAX;
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < n; l += (long long)gridDim.x * blockDim.x) {
    const double v = e ? (double)y[l] + (double)e[l] : (double)y[l];
    lo = v < lo ? v : lo;
    hi = v > hi ? v : hi;
  }
  smin[threadIdx.x] = lo;
  smax[threadIdx.x] = hi;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      smin[threadIdx.x] = fmin(smin[threadIdx.x], smin[threadIdx.x + s]);
      smax[threadIdx.x] = fmax(smax[threadIdx.x], smax[threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    atomic_max_double(&out2[0], -smin[0]);
    atomic_max_double(&out2[1], smax[0]);
  }
}

// temporal::compute_CFL (src/solver/temporal_discretization.cpp:397-450), including the
// convective term's truncation to int (abs(double) resolving to int abs(int) at :425).
__global__ void k_cfl(long long n, int dim, const double* const* met, const double* jac, const double* const* ub,
                      const double* pbar, const double* sbar, const int* iblank, double gamma, double dt,
                      double* d_max) {
  __shared__ double sm[kThreads];
  double best = -1e300;
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < n; l += (long long)gridDim.x * blockDim.x) {
    if (iblank && iblank[l] != 0) continue;
    double vc[3] = {0, 0, 0};
    for (int a = 0; a < dim; ++a) {
      vc[a] = 0.0;
      for (int q = 0; q < dim; ++q) vc[a] += met[a * 3 + q][l] * ub[q][l];
    }
    double cfl = 0.0;
    for (int a = 0; a < dim; ++a)
      for (int q = 0; q < dim; ++q) {
        int t = (int)(vc[a] * met[a * 3 + q][l]);
        cfl += (double)(t < 0 ? -t : t);
      }
    double fac = 0.0;
    for (int a = 0; a < dim; ++a)
      for (int q = 0; q < dim; ++q) fac += met[a * 3 + q][l] * met[a * 3 + q][l];
    // State::compute_auxiliary_variables_linear_Euler (src/core/state.cpp:701-736)
    double g = gamma, gi = 1.0 / g, gg = g / (g - 1.0);
    double rhobar = pow(g * pbar[l], gi) * exp(-sbar[l]);
    double Tbar = pbar[l] * gg * (1.0 / rhobar);
    double sos = sqrt((gamma - 1.0) * Tbar);
    cfl += sos * sqrt(fac);
    cfl *= dt * jac[l];
    best = cfl > best ? cfl : best;
  }
  sm[threadIdx.x] = best;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) atomic_max_double(d_max, sm[0]);
}

// rho'/rho_bar = p'/(gamma p_bar) - s' (State::compute_auxiliary_variables_linear_Euler,
// src/core/state.cpp:701-736, divided by rho_bar).
__global__ void k_rho_ratio(long long n, double gi, const double* s, const double* p, const double* pbar, double* out) {
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < n; l += (long long)gridDim.x * blockDim.x)
    out[l] = p[l] * gi * (1.0 / pbar[l]) - s[l];
}

__global__ void k_monopole_g(int nx, int ny, const double* const* xyz, int lo0, int lo1, int lo2, int b0, int b1,
                             long long nb, double x0, double y0, double z0, double ef, double* g) {
  for (long long lb = blockIdx.x * (long long)blockDim.x + threadIdx.x; lb < nb; lb += (long long)gridDim.x * blockDim.x) {
    int i = lo0 + (int)(lb % b0), j = lo1 + (int)((lb / b0) % b1), k = lo2 + (int)(lb / ((long long)b0 * b1));
    long long l0 = i + (long long)nx * (j + (long long)ny * k);
    double dx = xyz[0][l0] - x0, dy = xyz[1][l0] - y0, dz = xyz[2][l0] - z0;
    g[lb] = exp(ef * (dx * dx + dy * dy + dz * dz));
  }
}

int grid_for(long long n) {
  long long b = (n + kThreads - 1) / kThreads;
  return (int)(b > 148 * 32 ? 148 * 32 : (b < 1 ? 1 : b));
}

}  // namespace

cudaError_t setup_apply_dir(const OpTable& op, int nx, int ny, int nz, int dir, const double* f, double* out,
                            const int8_t* code, int zero_if_one_cell, cudaStream_t s) {
  long long N = (long long)nx * ny * nz;
  int n = dir == 0 ? nx : (dir == 1 ? ny : nz);
  if (n == 1) {
    if (zero_if_one_cell)
      k_fill<<<grid_for(N), kThreads, 0, s>>>(N, out, 0.0);
    else
      k_copy<<<grid_for(N), kThreads, 0, s>>>(N, out, f);
    return cudaGetLastError();
  }
  k_apply_dir<<<grid_for(N), kThreads, 0, s>>>(op, nx, ny, nz, dir, f, out, code);
  return cudaGetLastError();
}

cudaError_t setup_axpby(int n, double* out, double a, const double* x, double b, const double* y, cudaStream_t s) {
  k_axpby<<<grid_for(n), kThreads, 0, s>>>(n, out, a, x, b, y);
  return cudaGetLastError();
}

cudaError_t setup_mul(int n, double* out, const double* x, const double* y, cudaStream_t s) {
  k_mul<<<grid_for(n), kThreads, 0, s>>>(n, out, x, y);
  return cudaGetLastError();
}

cudaError_t setup_jacobian(int n, int dim, double* const* xx, double* invjac, double* jac, cudaStream_t s) {
  k_jacobian<<<grid_for(n), kThreads, 0, s>>>(n, dim, xx, invjac, jac);
  return cudaGetLastError();
}

cudaError_t setup_inverse_metrics(int n, int dim, double* const* met, double* const* minv, cudaStream_t s) {
  k_inverse<<<grid_for(n), kThreads, 0, s>>>(n, dim, met, minv);
  return cudaGetLastError();
}

cudaError_t setup_grad_accum(int n, double* sum, const double* m, const double* d, cudaStream_t s) {
  k_grad_accum<<<grid_for(n), kThreads, 0, s>>>(n, sum, m, d);
  return cudaGetLastError();
}

cudaError_t setup_scale(int n, double* out, const double* sum, const double* jac, cudaStream_t s) {
  k_scale<<<grid_for(n), kThreads, 0, s>>>(n, out, sum, jac);
  return cudaGetLastError();
}

cudaError_t setup_sigma(int nx, int ny, int nz, const double* const* xyz, const int lo[3], const int hi[3], int dir,
                        int end, int order, double constant, double* sig, cudaStream_t s) {
  (void)nz;
  long long nb = (long long)(hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1);
  k_sigma<<<grid_for(nb), kThreads, 0, s>>>(nx, ny, xyz, lo[0], lo[1], lo[2], hi[0], hi[1], hi[2], dir, end, order,
                                            constant, sig);
  return cudaGetLastError();
}

cudaError_t setup_minmax(int n, const double* f, double* d_out2, cudaStream_t s) {
  k_minmax<<<grid_for(n), kThreads, 0, s>>>(n, f, d_out2);
  return cudaGetLastError();
}

cudaError_t setup_state_minmax(long long n, const void* y, const void* e, bool fp32, double* d_out2, cudaStream_t s) {
  if (fp32)
    k_state_minmax<float><<<grid_for(n), kThreads, 0, s>>>(n, (const float*)y, (const float*)e, d_out2);
  else
    k_state_minmax<double><<<grid_for(n), kThreads, 0, s>>>(n, (const double*)y, (const double*)e, d_out2);
  return cudaGetLastError();
}

cudaError_t setup_cfl(int n, int dim, const double* const* met, const double* jac, const double* const* ubar,
                      const double* pbar, const double* sbar, const int* iblank, double gamma, double dt,
                      double* d_max, cudaStream_t s) {
  k_cfl<<<grid_for(n), kThreads, 0, s>>>(n, dim, met, jac, ubar, pbar, sbar, iblank, gamma, dt, d_max);
  return cudaGetLastError();
}

cudaError_t setup_rho_ratio(int n, int V, double gamma, const double* sv, const double* p, const double* pbar,
                            double* out, cudaStream_t s) {
  (void)V;
  k_rho_ratio<<<grid_for(n), kThreads, 0, s>>>(n, 1.0 / gamma, sv, p, pbar, out);
  return cudaGetLastError();
}

cudaError_t setup_monopole_g(int nx, int ny, const double* const* xyz, const int lo[3], const int hi[3],
                             double x0, double y0, double z0, double ef, double* g, cudaStream_t s) {
  int b0 = hi[0] - lo[0] + 1, b1 = hi[1] - lo[1] + 1, b2 = hi[2] - lo[2] + 1;
  long long nb = (long long)b0 * b1 * b2;
  k_monopole_g<<<grid_for(nb), kThreads, 0, s>>>(nx, ny, xyz, lo[0], lo[1], lo[2], b0, b1, nb, x0, y0, z0, ef, g);
  return cudaGetLastError();
}

}  // namespace lee
