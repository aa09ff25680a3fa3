// Time-advance kernels: the fused RK stage (LEE right-hand side with metric chain
// rule, sponges, monopole source, hole mask and the Runge-Kutta stage update) and the
// dimension-split filter passes.
//
// Each stage kernel reads the stage input with its stencil neighbours once and
// writes the next stage input and the RK accumulator: the state crosses HBM once per
// stage (the reference makes 24/63 directional passes per stage in 2-D/3-D,
// src/solver/spatial_discretization.cpp:2053-2130).
#include <type_traits>

#include "lee_internal.h"
#include "lee_point.cuh"

namespace lee {
namespace {

// Operator value at one point: the interior stencil, or a closure row selected by
// position along the line or by the precomputed code (src/solver/spatial_discretization.cpp:1094-1149
// and the hole closures of :1656-1745).
template <typename T>
__device__ __forceinline__ T dop(const OpTable& op, const T* __restrict__ f, long long l0, int pos, int n,
                                 long long sd, const int8_t* __restrict__ code) {
  int c;
  if (code) {
    c = code[l0];
  } else if (pos >= op.h && pos <= n - 1 - op.h) {
    c = 0;
  } else if (pos < op.h) {
    c = 1 + pos;
  } else {
    c = -(1 + (n - 1 - pos));
  }
  T acc = T(0);
  if (c == 0) {
#pragma unroll 4
    for (int l = -op.h; l <= op.h; ++l) acc += T(op.c[l + op.h]) * __ldg(f + l0 + l * sd);
    return acc;
  }
  if (c == kCodeZero) return T(0);
  if (c > 0) {
    int r = c - 1;
    long long a = l0 - r * sd;
    for (int s = 0; s < op.S; ++s) acc += T(op.B[r][s]) * __ldg(f + a + s * sd);
    return acc;
  }
  int r = -c - 1;
  long long a = l0 + r * sd;
  for (int s = 0; s < op.S; ++s) acc += T(op.mfac * op.B[r][s]) * __ldg(f + a - s * sd);
  return acc;
}

template <typename T, int DIM, bool COMP>
__global__ void __launch_bounds__(256) k_stage(StageParams<T> p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= p.nx || j >= p.ny) return;
  constexpr int V = DIM + 2;
  const long long nxy = (long long)p.nx * p.ny;
  const long long l = i + (long long)p.nx * j + nxy * k;
  const int pos[3] = {i, j, k};
  const int nn[3] = {p.nx, p.ny, p.nz};
  const long long sd[3] = {1, p.nx, nxy};
  PointIn<T, DIM> in;
  gather<T, DIM, COMP, kTrGeneric>(p, l, in);
  T D[V][DIM], q[V];
#pragma unroll
  for (int v = 0; v < V; ++v) {
#pragma unroll
    for (int d = 0; d < DIM; ++d) D[v][d] = dop<T>(p.fd, p.zin[v], l, pos[d], nn[d], sd[d], p.code[d]);
    q[v] = p.zin[v][l];
  }
  rhs_update<T, DIM, COMP, kTrGeneric>(p, l, i, j, k, D, q, in);
}

// One direction of spatial::apply_filter (src/solver/spatial_discretization.cpp:2191-2246).
// FP64 form: out = F_dir(in); the last pass blends (1-beta) y0 + beta F(...) and zeroes holes
// (temporal::iblank_correction, src/solver/temporal_discretization.cpp:380-393).
// Compensated form: the filter is applied as y + D(y) with D = F - I, the increments D are
// summed over the passes, and the last pass adds beta * D + err to y_pre as an exact
// two-float sum, writing y and its new rounding error.
template <typename T, bool COMP>
__global__ void __launch_bounds__(256) k_filter(FilterParams<T> p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= p.nx || j >= p.ny) return;
  const long long nxy = (long long)p.nx * p.ny;
  const long long l = i + (long long)p.nx * j + nxy * k;
  const int pos = p.dir == 0 ? i : (p.dir == 1 ? j : k);
  const int n = p.dir == 0 ? p.nx : (p.dir == 1 ? p.ny : p.nz);
  const long long sd = p.dir == 0 ? 1 : (p.dir == 1 ? (long long)p.nx : nxy);
  const bool hole = p.last && p.iblank && p.iblank[l] == 1;
  // a hole after a hole: the reference writes F = 0 there, so the increment is D = -x, and a
  // later pass of a 3-D block reads the zero (the other codes give D = F - I directly)
  const bool zero = COMP && p.code && p.code[l] == kCodeZero;
  for (int v = 0; v < p.V; ++v) {
    const T f = zero ? -p.in[v][l] : dop<T>(p.op, p.in[v], l, pos, n, sd, p.code);
    if (!COMP) {
      T o = f;
      if (p.last) o = (T(1) - p.blend) * p.y0[v][l] + p.blend * f;
      p.out[v][l] = hole ? T(0) : o;
    } else {
      const T x = p.in[v][l];
      T dsum = p.first ? f : p.dsum_in[v][l] + f;
      if (!p.last) {
        p.out[v][l] = x + f;
        p.dsum[v][l] = dsum;
      } else {
        const T y0 = p.y0[v][l];
        const T t = p.blend * dsum + p.err[v][l];
        const T s = y0 + t;
        const T bb = s - y0;
        const T e = (y0 - (s - bb)) + (t - bb);
        p.out[v][l] = hole ? T(0) : s;
        p.comp[v][l] = hole ? T(0) : e;
      }
    }
  }
}

template <typename T>
__global__ void k_hole_zero(long long n, int V, T* f0, T* f1, T* f2, T* f3, T* f4, const int* iblank) {
  T* f[5] = {f0, f1, f2, f3, f4};
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < n; l += (long long)gridDim.x * blockDim.x)
    if (iblank[l] == 1)
      for (int v = 0; v < V; ++v) f[v][l] = T(0);
}

// One RK stage of a block's passive scalars (compute_RHS_linearized_Euler_scalar,
// src/solver/spatial_discretization.cpp:2134-2158): per direction x, r -= u_bar_x dZ/dx_x, then
// r -= u'_x dZ_bar/dx_x; the sponges (relaxing to zero, src/solver/source.cpp:174-201); then the
// stage update of the LEE slots (RungeKutta::integrate with the hole bypass).
template <typename T, int DIM, bool COMP>
__global__ void __launch_bounds__(256) k_scalar_stage(ScalarParams<T> p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= p.nx || j >= p.ny) return;
  const long long nxy = (long long)p.nx * p.ny;
  const long long l = i + (long long)p.nx * j + nxy * k;
  const int pos[3] = {i, j, k};
  const int nn[3] = {p.nx, p.ny, p.nz};
  const long long sd[3] = {1, p.nx, nxy};
  const bool first = p.stage == 0, last = p.last != 0;
  const bool hole = p.iblank && p.iblank[l] == 1;
  T jm[DIM][DIM], ub[DIM], u[DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d)
#pragma unroll
    for (int x = 0; x < DIM; ++x) jm[d][x] = p.jm[d * 3 + x].p ? __ldg(p.jm[d * 3 + x].p + l) : p.jm[d * 3 + x].c;
#pragma unroll
  for (int x = 0; x < DIM; ++x) {
    ub[x] = p.ubar[x].p ? __ldg(p.ubar[x].p + l) : p.ubar[x].c;
    u[x] = p.uin[x][l];
  }
  for (int q = 0; q < p.n; ++q) {
    const T z = p.zin[q][l];
    T r = T(0);
    T D[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) D[d] = dop<T>(p.fd, p.zin[q], l, pos[d], nn[d], sd[d], p.code[d]);
#pragma unroll
    for (int x = 0; x < DIM; ++x) {
      T g = T(0);
#pragma unroll
      for (int d = 0; d < DIM; ++d) g += jm[d][x] * D[d];
      r -= ub[x] * g;
      const Coef<T>& gz = p.gz[q][x];
      if (!gz.zero) r -= u[x] * (gz.p ? __ldg(gz.p + l) : gz.c);
    }
    for (int zi = 0; zi < p.nzones; ++zi) {
      const Zone<T>& zn = p.zones[zi];
      if (i < zn.lo[0] || i > zn.hi[0] || j < zn.lo[1] || j > zn.hi[1] || k < zn.lo[2] || k > zn.hi[2]) continue;
      const int b0 = zn.hi[0] - zn.lo[0] + 1, b1 = zn.hi[1] - zn.lo[1] + 1;
      const long long lb = (i - zn.lo[0]) + (long long)b0 * ((j - zn.lo[1]) + (long long)b1 * (k - zn.lo[2]));
      r += -zn.sig[lb] * (z - T(0));
    }
    if (hole) {
      p.acc[q][l] = T(0);
      if (!last || COMP) p.zout[q][l] = T(0);
      continue;
    }
    const T hk = r * p.h;
    const T yv = first ? z : p.yn[q][l];
    if (!COMP) {
      const T prev = first ? z : p.acc[q][l];
      p.acc[q][l] = prev + p.b * hk;
      if (!last) p.zout[q][l] = yv + p.a * hk;
    } else {
      const T inc = (first ? p.comp[q][l] : p.acc[q][l]) + p.b * hk;
      if (!last) {
        p.acc[q][l] = inc;
        p.zout[q][l] = yv + p.a * hk;
      } else {
        const T s = yv + inc;
        const T bb = s - yv;
        p.zout[q][l] = s;
        p.acc[q][l] = (yv - (s - bb)) + (inc - bb);
      }
    }
  }
}

}  // namespace

template <typename T>
cudaError_t launch_scalar_stage(const ScalarParams<T>& p, int comp, cudaStream_t s) {
  dim3 blk(32, 8, 1);
  dim3 grd((p.nx + 31) / 32, (p.ny + 7) / 8, p.nz);
  if (p.dim == 2) {
    if (comp) k_scalar_stage<T, 2, true><<<grd, blk, 0, s>>>(p);
    else k_scalar_stage<T, 2, false><<<grd, blk, 0, s>>>(p);
  } else {
    if (comp) k_scalar_stage<T, 3, true><<<grd, blk, 0, s>>>(p);
    else k_scalar_stage<T, 3, false><<<grd, blk, 0, s>>>(p);
  }
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_stage(const StageParams<T>& p, int comp, cudaStream_t s) {
  dim3 blk(32, 8, 1);
  dim3 grd((p.nx + 31) / 32, (p.ny + 7) / 8, p.nz);
  if (p.dim == 2) {
    if (comp) k_stage<T, 2, true><<<grd, blk, 0, s>>>(p);
    else k_stage<T, 2, false><<<grd, blk, 0, s>>>(p);
  } else {
    if (comp) k_stage<T, 3, true><<<grd, blk, 0, s>>>(p);
    else k_stage<T, 3, false><<<grd, blk, 0, s>>>(p);
  }
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_filter_pass(const FilterParams<T>& p, int comp, cudaStream_t s) {
  dim3 blk(32, 8, 1);
  dim3 grd((p.nx + 31) / 32, (p.ny + 7) / 8, p.nz);
  if (comp) k_filter<T, true><<<grd, blk, 0, s>>>(p);
  else k_filter<T, false><<<grd, blk, 0, s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_hole_zero(int n, int V, double** f, const int* iblank, cudaStream_t s) {
  k_hole_zero<double><<<(n + 255) / 256, 256, 0, s>>>(n, V, f[0], f[1], f[2], f[3], V > 4 ? f[4] : f[3], iblank);
  return cudaGetLastError();
}

cudaError_t launch_hole_zero_f(int n, int V, float** f, const int* iblank, cudaStream_t s) {
  k_hole_zero<float><<<(n + 255) / 256, 256, 0, s>>>(n, V, f[0], f[1], f[2], f[3], V > 4 ? f[4] : f[3], iblank);
  return cudaGetLastError();
}

template cudaError_t launch_stage<double>(const StageParams<double>&, int, cudaStream_t);
template cudaError_t launch_stage<float>(const StageParams<float>&, int, cudaStream_t);
template cudaError_t launch_filter_pass<double>(const FilterParams<double>&, int, cudaStream_t);
template cudaError_t launch_filter_pass<float>(const FilterParams<float>&, int, cudaStream_t);
template cudaError_t launch_scalar_stage<double>(const ScalarParams<double>&, int, cudaStream_t);
template cudaError_t launch_scalar_stage<float>(const ScalarParams<float>&, int, cudaStream_t);

}  // namespace lee
