// Discrete adjoint of the LEE time step: transposed RK stages, transposed filter, and the
// microphone objective's trace and forcing kernels.
//
// The step map of the reference's scheme (RungeKutta::integrate and spatial::apply_filter,
// camille src/solver/temporal_discretization.cpp:177-252, src/solver/spatial_discretization.cpp:2191-2246)
// is linear in the state: z_0 = y, k_s = L z_s + f_s, z_{s+1} = y + a_s h k_s,
// y_next = y + h sum_s b_s k_s, y_new = F y_next. Its transpose, for an adjoint lam of y_new:
//   mu = F^T lam;  kbar_{S-1} = h b_{S-1} mu;  zbar_s = L^T kbar_s;
//   kbar_{s-1} = h b_{s-1} mu + a_{s-1} h zbar_s;  ybar = mu + sum_s zbar_s,
// and a source f_s = amp_s S e_p' contributes amp_s kbar_s[p'] to the gradient of S.
//
// L^T: with the uniform-mean right-hand side r_v = sum_d sum_v' C^d_vv' D_d q_v' - sigma q_v
// (compute_RHS_linearized_Euler, spatial_discretization.cpp:2053-2130, and the Freund sponge,
// src/solver/source.cpp:174-201), (L^T w)_v' = sum_d D_d^T G^d_v' - sigma w_v' with the fluxes
//   G^d_s = -U^d w_s,  G^d_u_x = -U^d w_u_x - gamma p_bar JM[d][x] w_p,
//   G^d_p = -U^d w_p - (1/rho_bar) sum_a JM[d][a] w_u_a,  U^d = sum_x u_bar_x JM[d][x],
// where JM = J * metrics. D_d^T is the transposed difference operator with its transposed
// boundary closures (TransOp, built on the host from the forward tables).
#include "lee_internal.h"

namespace lee {
namespace {

template <typename T>
__device__ __forceinline__ T cval_a(const Coef<T>& c, long long l) {
  return c.p ? __ldg(c.p + l) : c.c;
}

__device__ __forceinline__ const double* trans_row(const TransOp& op, int pos, int n) {
  if (pos < op.E) return op.lt[pos];
  if (pos > n - 1 - op.E) return op.rt[n - 1 - pos];
  return op.in;
}

template <typename T, int DIM>
__global__ void __launch_bounds__(256) k_adj_stage(AdjStageParams<T> p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= p.nx || j >= p.ny) return;
  constexpr int V = DIM + 2;
  constexpr int P = DIM + 1;
  const long long nxy = (long long)p.nx * p.ny;
  const long long l = i + (long long)p.nx * j + nxy * k;
  const int pos[3] = {i, j, k};
  const int nn[3] = {p.nx, p.ny, p.nz};
  const long long sd[3] = {1, p.nx, nxy};
  const T scale = p.first ? p.hb_in : T(1);
  T acc[V];
#pragma unroll
  for (int v = 0; v < V; ++v) acc[v] = T(0);
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    const double* row = trans_row(p.op, pos[d], nn[d]);
    for (int t = -p.op.H; t <= p.op.H; ++t) {
      const T wgt = (T)row[t + p.op.H];
      if (wgt == T(0)) continue;
      const long long lq = l + t * sd[d];
      T w[V], jm[DIM];
#pragma unroll
      for (int v = 0; v < V; ++v) w[v] = scale * __ldg(p.kin[v] + lq);
      T U = T(0);
#pragma unroll
      for (int x = 0; x < DIM; ++x) {
        jm[x] = cval_a(p.jm[d * 3 + x], lq);
        U += p.ubar[x] * jm[x];
      }
      acc[0] += wgt * (-U * w[0]);
      T su = T(0);
#pragma unroll
      for (int x = 0; x < DIM; ++x) {
        acc[1 + x] += wgt * (-U * w[1 + x] - p.gpb * jm[x] * w[P]);
        su += jm[x] * w[1 + x];
      }
      acc[P] += wgt * (-U * w[P] - p.rbi * su);
    }
  }
  T wc[V];
#pragma unroll
  for (int v = 0; v < V; ++v) wc[v] = scale * p.kin[v][l];
  if (p.sigma) {
    const T sg = p.sigma[l];
#pragma unroll
    for (int v = 0; v < V; ++v) acc[v] -= sg * wc[v];
  }
#pragma unroll
  for (int v = 0; v < V; ++v) {
    const T m = p.mu[v][l];
    p.ybar[v][l] = p.first ? m + acc[v] : p.ybar[v][l] + acc[v];
    if (p.has_next) p.kout[v][l] = p.hb_next * m + p.ha_next * acc[v];
  }
  if (p.gbar && i >= p.src_lo[0] && i <= p.src_hi[0] && j >= p.src_lo[1] && j <= p.src_hi[1] && k >= p.src_lo[2] &&
      k <= p.src_hi[2]) {
    const int b0 = p.src_hi[0] - p.src_lo[0] + 1, b1 = p.src_hi[1] - p.src_lo[1] + 1;
    const long long lb = (i - p.src_lo[0]) + (long long)b0 * ((j - p.src_lo[1]) + (long long)b1 * (k - p.src_lo[2]));
    p.gbar[lb] += p.amp * (double)wc[P];
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_adj_filter(AdjFilterParams<T> p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= p.nx || j >= p.ny) return;
  const long long nxy = (long long)p.nx * p.ny;
  const long long l = i + (long long)p.nx * j + nxy * k;
  const int pos = p.dir == 0 ? i : (p.dir == 1 ? j : k);
  const int n = p.dir == 0 ? p.nx : (p.dir == 1 ? p.ny : p.nz);
  const long long sd = p.dir == 0 ? 1 : (p.dir == 1 ? (long long)p.nx : nxy);
  const double* row = trans_row(p.op, pos, n);
  for (int v = 0; v < p.V; ++v) {
    T f = T(0);
    for (int t = -p.op.H; t <= p.op.H; ++t) {
      const T wgt = (T)row[t + p.op.H];
      if (wgt != T(0)) f += wgt * __ldg(p.in[v] + l + t * sd);
    }
    p.out[v][l] = p.last ? (T(1) - p.blend) * p.lam[v][l] + p.blend * f : f;
  }
}

template <typename T>
__global__ void k_trace(int n, const long long* l0, const T* pp, const T* e, double* trace, const int* ctr,
                        const int* base, int row) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  const long long l = l0[m];
  double v = (double)pp[l];
  if (e) v += (double)e[l];
  trace[(long long)(ctr ? *ctr + *base : row) * n + m] = v;
}

template <typename T>
__global__ void k_mic_force(int n, const long long* l0, T* lam, const double* trace, int row, double scale) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  // microphones sit on distinct points, so the updates never collide
  lam[l0[m]] = (T)((double)lam[l0[m]] + scale * trace[(long long)row * n + m]);
}

}  // namespace

template <typename T>
cudaError_t launch_adj_stage(const AdjStageParams<T>& p, int dim, cudaStream_t s) {
  dim3 blk(32, 8, 1);
  dim3 grd((p.nx + 31) / 32, (p.ny + 7) / 8, p.nz);
  if (dim == 2) k_adj_stage<T, 2><<<grd, blk, 0, s>>>(p);
  else k_adj_stage<T, 3><<<grd, blk, 0, s>>>(p);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_adj_filter(const AdjFilterParams<T>& p, cudaStream_t s) {
  dim3 blk(32, 8, 1);
  dim3 grd((p.nx + 31) / 32, (p.ny + 7) / 8, p.nz);
  k_adj_filter<T><<<grd, blk, 0, s>>>(p);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_trace(int n, const long long* l0, const T* pp, const T* e, double* trace, const int* ctr,
                         const int* base, int row, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_trace<T><<<(n + 127) / 128, 128, 0, s>>>(n, l0, pp, e, trace, ctr, base, row);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_mic_force(int n, const long long* l0, T* lam, const double* trace, int row, double scale,
                             cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_mic_force<T><<<(n + 127) / 128, 128, 0, s>>>(n, l0, lam, trace, row, scale);
  return cudaGetLastError();
}

template cudaError_t launch_adj_stage<double>(const AdjStageParams<double>&, int, cudaStream_t);
template cudaError_t launch_adj_stage<float>(const AdjStageParams<float>&, int, cudaStream_t);
template cudaError_t launch_adj_filter<double>(const AdjFilterParams<double>&, cudaStream_t);
template cudaError_t launch_adj_filter<float>(const AdjFilterParams<float>&, cudaStream_t);
template cudaError_t launch_trace<double>(int, const long long*, const double*, const double*, double*, const int*,
                                          const int*, int, cudaStream_t);
template cudaError_t launch_trace<float>(int, const long long*, const float*, const float*, double*, const int*,
                                         const int*, int, cudaStream_t);
template cudaError_t launch_mic_force<double>(int, const long long*, double*, const double*, int, double,
                                              cudaStream_t);
template cudaError_t launch_mic_force<float>(int, const long long*, float*, const double*, int, double,
                                             cudaStream_t);

}  // namespace lee
