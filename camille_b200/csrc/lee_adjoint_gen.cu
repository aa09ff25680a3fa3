// The discrete adjoint of the general step: every block of a context, holes and their closure
// codes, BC lines, overset interpolation, non-uniform mean flow (the rho' term included),
// sponge zones and the axisymmetric term.
//
// One forward step of a block (lee_host_step.cu; RungeKutta::integrate, camille
// src/solver/temporal_discretization.cpp:177-252, then spatial::apply_filter and
// iblank_correction, :354-361), with M the hole mask, P = O B the boundary update (the BC lines
// of each block, then the overset interpolation over all blocks) and F the filter:
//   z_0 = y,  k_s = L_s z_s,  z_{s+1} = P M (y + a_s h k_s),  Y = P M (y + h sum_s b_s k_s),
//   y_new = M F Y.
// L_0 of a step after the first also reads rho'/rho_bar = R(Y_prev) of the previous step's Y
// (the rho' term of the non-uniform right-hand side, spatial_discretization.cpp:2080-2104).
// Its transpose, for an adjoint lam of y_new and rb, the adjoint of R(Y) carried from the next
// step:
//   Ybar = F^T M lam + R^T rb;  mu = M P^T Ybar;  kbar_{S-1} = h b_{S-1} mu;
//   zbar_s = L_s^T kbar_s;  nu_s = M P^T zbar_s;  kbar_{s-1} = h b_{s-1} mu + a_{s-1} h nu_s;
//   ybar = mu + sum_{s>=1} nu_s + zbar_0;  rb' = the rho' part of L_0^T kbar_0.
//
// L^T w at a point m is sum_d sum_l D_d[l][m] G^d(l) + B(m)^T w(m) - sigma(m) w(m): the fluxes
// G^d = (C^d)^T w of the gradient part r = sum_d C^d D_d q (C^d from J*metrics and the mean at
// the point), and the transposed pointwise part B (mean gradients, the rho' term, the
// axisymmetric term). D_d^T is applied in gather form: the rows of the points l within reach of
// m along the line are rebuilt from their closure code (or position), so the result does not
// depend on the order of any concurrent update.
#include "lee_internal.h"

namespace lee {
namespace {

template <typename T, typename I>
__device__ __forceinline__ T cv(const Coef<T>& c, I l) {
  return c.p ? __ldg(c.p + l) : c.c;
}

// The closure code of the point at position q of a line (dop() in lee_step.cu).
__device__ __forceinline__ int code_at(const OpTable& op, const int8_t* code, long long l, int q, int n) {
  if (code) return code[l];
  if (q >= op.h && q <= n - 1 - op.h) return 0;
  if (q < op.h) return 1 + q;
  return -(1 + (n - 1 - q));
}

// D[l][m] for the point l = m + t of the line: its row (interior, left closure row r anchored r
// points to the left, mirrored right row r anchored r points to the right, or zero) at m.
__device__ __forceinline__ double row_at(const OpTable& op, int c, int t) {
  if (c == 0) return (t >= -op.h && t <= op.h) ? op.c[-t + op.h] : 0.0;
  if (c == kCodeZero) return 0.0;
  if (c > 0) {
    const int s = -t + (c - 1);
    return (s >= 0 && s < op.S) ? op.B[c - 1][s] : 0.0;
  }
  const int r = -c - 1;
  const int s = t + r;
  return (s >= 0 && s < op.S) ? op.mfac * op.B[r][s] : 0.0;
}

// (D^T g)(m) along one line: m at position pos of n, index l0, stride sd.
template <typename T>
__device__ __forceinline__ T dop_t(const OpTable& op, const T* __restrict__ g, long long l0, int pos, int n,
                                   long long sd, const int8_t* __restrict__ code) {
  const int R = max(op.h, max(op.S - 1, op.nb - 1));
  T acc = T(0);
  for (int t = -R; t <= R; ++t) {
    const int q = pos + t;
    if (q < 0 || q >= n) continue;
    const long long l = l0 + t * sd;
    const int c = code_at(op, code, l, q, n);
    // the forward rounds each coefficient to T before use (dop); so does its transpose
    const T w = (T)row_at(op, c, t);
    if (w != T(0)) acc += w * __ldg(g + l);
  }
  return acc;
}

// G^d at every point: w = scale * kin, G^d_s = -U w_s, G^d_u_x = -U w_u_x - gamma p_bar JM[d][x] w_p,
// G^d_p = -U w_p - (1/rho_bar) sum_a JM[d][a] w_u_a, U = sum_x u_bar_x JM[d][x].
template <typename T, int DIM>
__global__ void __launch_bounds__(256) k_adjg_flux(AdjGenParams<T> p) {
  const StageParams<T>& f = p.f;
  const long long n = (long long)f.nx * f.ny * f.nz;
  constexpr int V = DIM + 2, P = DIM + 1;
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < n; l += (long long)gridDim.x * blockDim.x) {
    T w[V];
#pragma unroll
    for (int v = 0; v < V; ++v) w[v] = p.scale * p.kin[v][l];
    T ub[DIM];
#pragma unroll
    for (int x = 0; x < DIM; ++x) ub[x] = cv(f.ubar[x], l);
    const T gpb = f.gamma * cv(f.pbar, l);
    const T rbi = cv(f.rhobar_inv, l);
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      T jm[DIM];
      T U = T(0);
#pragma unroll
      for (int x = 0; x < DIM; ++x) {
        jm[x] = cv(f.jm[d * 3 + x], l);
        U += ub[x] * jm[x];
      }
      p.g[d][0][l] = -U * w[0];
      T su = T(0);
#pragma unroll
      for (int x = 0; x < DIM; ++x) {
        p.g[d][1 + x][l] = -U * w[1 + x] - gpb * jm[x] * w[P];
        su += jm[x] * w[1 + x];
      }
      p.g[d][P][l] = -U * w[P] - rbi * su;
    }
  }
}

// zbar = L^T w at every point, the source gradient on the source box, and the adjoint of
// rho_prev when the forward stage read it.
template <typename T, int DIM>
__global__ void __launch_bounds__(256) k_adjg_stage(AdjGenParams<T> p) {
  const StageParams<T>& f = p.f;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= f.nx || j >= f.ny) return;
  constexpr int V = DIM + 2, P = DIM + 1;
  const long long nxy = (long long)f.nx * f.ny;
  const long long l = i + (long long)f.nx * j + nxy * k;
  const int pos[3] = {i, j, k};
  const int nn[3] = {f.nx, f.ny, f.nz};
  const long long sd[3] = {1, f.nx, nxy};
  T acc[V];
#pragma unroll
  for (int v = 0; v < V; ++v) {
    T s = T(0);
#pragma unroll
    for (int d = 0; d < DIM; ++d) s += dop_t<T>(f.fd, p.g[d][v], l, pos[d], nn[d], sd[d], f.code[d]);
    acc[v] = s;
  }
  T w[V];
#pragma unroll
  for (int v = 0; v < V; ++v) w[v] = p.scale * p.kin[v][l];
  // B^T w: the mean-gradient terms of rhs_mean_terms (lee_point.cuh), transposed
#pragma unroll
  for (int x = 0; x < DIM; ++x) {
    if (!f.gs[x].zero) acc[1 + x] -= cv(f.gs[x], l) * w[0];
#pragma unroll
    for (int a = 0; a < DIM; ++a)
      if (!f.gu[a * 3 + x].zero) acc[1 + x] -= cv(f.gu[a * 3 + x], l) * w[1 + a];
    if (!f.gp[x].zero) acc[1 + x] -= cv(f.gp[x], l) * w[P];
    if (!f.gu[x * 3 + x].zero) acc[P] -= f.gamma * cv(f.gu[x * 3 + x], l) * w[P];
  }
  if (f.need_rho) {
    // r_u_a -= rr u_bar_x du_bar_a/dx_x: the adjoint of rr is -sum_a K_a w_u_a
    T rrb = T(0);
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
      T K = T(0);
#pragma unroll
      for (int x = 0; x < DIM; ++x)
        if (!f.gu[a * 3 + x].zero) K += cv(f.ubar[x], l) * cv(f.gu[a * 3 + x], l);
      rrb -= K * w[1 + a];
    }
    if (p.rbar) {
      p.rbar[l] = rrb;  // rr = rho_prev
    } else {
      // rr = p' / (gamma p_bar) - s'
      acc[P] += rrb * f.inv_gamma * (T(1) / cv(f.pbar, l));
      acc[0] -= rrb;
    }
  }
  if constexpr (DIM == 2) {
    if (f.axisym) {
      // r_p -= gamma (p_bar u_r' + p' u_r_bar) / (r + DUMMY_SMALL)
      const double rr = f.ry[l] + 1e-99;
      acc[2] -= (T)((double)f.gamma * (double)cv(f.pbar, l) / rr) * w[P];
      acc[P] -= (T)((double)f.gamma * (double)cv(f.ubar[1], l) / rr) * w[P];
    }
  }
  // sponges: -sigma w over every zone holding the point
  for (int z = 0; z < f.nzones; ++z) {
    const Zone<T>& zn = f.zones[z];
    if (i < zn.lo[0] || i > zn.hi[0] || j < zn.lo[1] || j > zn.hi[1] || k < zn.lo[2] || k > zn.hi[2]) continue;
    const int b0 = zn.hi[0] - zn.lo[0] + 1, b1 = zn.hi[1] - zn.lo[1] + 1;
    const long long lb = (i - zn.lo[0]) + (long long)b0 * ((j - zn.lo[1]) + (long long)b1 * (k - zn.lo[2]));
    const T sg = zn.sig[lb];
#pragma unroll
    for (int v = 0; v < V; ++v) acc[v] -= sg * w[v];
  }
#pragma unroll
  for (int v = 0; v < V; ++v) p.zbar[v][l] = acc[v];
  if (p.gbar && i >= f.src_lo[0] && i <= f.src_hi[0] && j >= f.src_lo[1] && j <= f.src_hi[1] && k >= f.src_lo[2] &&
      k <= f.src_hi[2]) {
    const int b0 = f.src_hi[0] - f.src_lo[0] + 1, b1 = f.src_hi[1] - f.src_lo[1] + 1;
    const long long lb = (i - f.src_lo[0]) + (long long)b0 * ((j - f.src_lo[1]) + (long long)b1 * (k - f.src_lo[2]));
    p.gbar[lb] += p.amp * (double)w[P];
  }
}

// One transposed filter pass along dir (F^T in gather form; the passes run in the reverse of the
// forward's order). The first pass reads M lam; the last writes (1 - beta) M lam + beta F^T(...)
// plus R^T rb (rho'/rho_bar = p'/(gamma p_bar) - s' of Y).
template <typename T>
__global__ void __launch_bounds__(256) k_adjg_filter(AdjGenFilterParams<T> p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= p.nx || j >= p.ny) return;
  const long long nxy = (long long)p.nx * p.ny;
  const long long l = i + (long long)p.nx * j + nxy * k;
  const int pos = p.dir == 0 ? i : (p.dir == 1 ? j : k);
  const int n = p.dir == 0 ? p.nx : (p.dir == 1 ? p.ny : p.nz);
  const long long sd = p.dir == 0 ? 1 : (p.dir == 1 ? (long long)p.nx : nxy);
  const int R = max(p.op.h, max(p.op.S - 1, p.op.nb - 1));
  for (int v = 0; v < p.V; ++v) {
    T acc = T(0);
    for (int t = -R; t <= R; ++t) {
      const int q = pos + t;
      if (q < 0 || q >= n) continue;
      const long long lq = l + t * sd;
      const T w = (T)row_at(p.op, code_at(p.op, p.code, lq, q, n), t);
      if (w == T(0)) continue;
      const T x = (p.mask_in && p.iblank[lq] == 1) ? T(0) : p.in[v][lq];
      acc += w * x;
    }
    if (p.last) {
      const T lm = (p.iblank && p.iblank[l] == 1) ? T(0) : p.lam[v][l];
      acc = (T(1) - p.blend) * lm + p.blend * acc;
    }
    p.out[v][l] = acc;
  }
  if (p.last && p.rb) {
    const T r = p.rb[l];
    p.out[p.V - 1][l] += r * p.inv_gamma * (T(1) / (T)p.pbar[l]);
    p.out[0][l] -= r;
  }
}

// out = M in + R^T rb (no filter), or M in alone (rb null); in place allowed.
template <typename T>
__global__ void k_adjg_mask(long long n, int V, AdjGenPoint<T> p) {
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < n; l += (long long)gridDim.x * blockDim.x) {
    const bool hole = p.iblank && p.iblank[l] == 1;
    for (int v = 0; v < V; ++v) p.out[v][l] = hole ? T(0) : p.in[v][l];
    if (p.rb) {
      const T r = p.rb[l];
      p.out[V - 1][l] += r * p.inv_gamma * (T(1) / (T)p.pbar[l]);
      p.out[0][l] -= r;
    }
  }
}

// nu = M zbar; ybar += nu; kout = hb mu + ha nu (kout null: the first stage, ybar += zbar unmasked)
template <typename T>
__global__ void k_adjg_combine(long long n, int V, AdjGenPoint<T> p, T hb, T ha) {
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < n; l += (long long)gridDim.x * blockDim.x) {
    const bool hole = p.iblank && p.iblank[l] == 1;
    for (int v = 0; v < V; ++v) {
      const T nu = hole ? T(0) : p.in[v][l];
      p.ybar[v][l] += nu;
      if (p.out[v]) p.out[v][l] = hb * p.mu[v][l] + ha * nu;
    }
  }
}

// The transpose of one BC line (k_bc in lee_bc.cu) on w, in place: a face point's adjoint moves
// to the points its Neumann row reads (its own normal line, never another face point of the
// line, so the face points of one launch touch disjoint points), the slip wall's velocity part
// is transposed at the point, and Dirichlet values are constants (no adjoint).
template <typename T>
__global__ void k_adjg_bc(BcParams<T> p) {
  const long long n = (long long)p.nb[0] * p.nb[1] * p.nb[2];
  for (long long lb = blockIdx.x * (long long)blockDim.x + threadIdx.x; lb < n;
       lb += (long long)gridDim.x * blockDim.x) {
    const int i = p.lo[0] + (int)(lb % p.nb[0]);
    const int j = p.lo[1] + (int)((lb / p.nb[0]) % p.nb[1]);
    const int k = p.lo[2] + (int)(lb / ((long long)p.nb[0] * p.nb[1]));
    const long long l = i + (long long)p.nx * (j + (long long)p.ny * k);
    if (p.iblank && p.iblank[l] == 1) continue;
    const int P = p.nd + 1;
    double tmp[kMaxVars];
    bool scat[kMaxVars];
    for (int v = 0; v < p.V; ++v) {
      tmp[v] = (double)p.y[v][l];
      scat[v] = false;
      p.y[v][l] = T(0);
    }
    if (p.kind == LEE_BC_NEUMANN) {
      for (int v = 0; v < p.V; ++v) scat[v] = true;
    } else if (p.kind >= LEE_BC_CENTERLINE_CART_NORM2X && p.kind <= LEE_BC_CENTERLINE_AXISYM) {
      for (int v = 0; v < p.V; ++v) scat[v] = true;
      const int d = p.kind == LEE_BC_CENTERLINE_AXISYM ? 1 : p.kind - LEE_BC_CENTERLINE_CART_NORM2X;
      if (d < p.nd) tmp[1 + d] = 0.0;
    } else if (p.kind == LEE_BC_DIRICHLET_ALLZERO || p.kind == LEE_BC_DIRICHLET_HARMONICWAVE) {
      // constants: nothing flows back
    } else {
      // slip wall: u_out = J Minv Z Met u (Z zeroes the wall-normal contravariant component);
      // its transpose Met^T Z Minv^T J acts on the velocity adjoint at the point
      scat[0] = scat[P] = true;
      const double jac = p.jac[l];
      double vc[3] = {0.0, 0.0, 0.0};
      for (int a = 0; a < p.nd; ++a) {
        double s = 0.0;
        for (int q = 0; q < p.nd; ++q) s += p.minv[q * 3 + a][l] * jac * tmp[1 + q];
        vc[a] = a == p.dir ? 0.0 : s;
      }
      for (int q = 0; q < p.nd; ++q) {
        double s = 0.0;
        for (int a = 0; a < p.nd; ++a) s += p.met[a * 3 + q][l] * vc[a];
        p.y[1 + q][l] = (T)s;
      }
    }
    const long long step = p.end == 0 ? p.sd : -p.sd;
    for (int s = 1; s < p.S; ++s) {
      const double alpha = -p.c0[s] / p.c0[0];
      const long long ls = l + step * s;
      for (int v = 0; v < p.V; ++v)
        if (scat[v]) p.y[v][ls] = (T)((double)p.y[v][ls] + alpha * tmp[v]);
    }
  }
}

// Overset transpose, first half: the receivers' adjoints are taken out (their forward values
// were overwritten) into tmp.
template <typename T>
__global__ void k_adjg_ovs_take(AdjGenOvs<T> p) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= p.n) return;
  const int b = p.rb[r];
  const long long l = p.rl[r];
  for (int v = 0; v < p.V; ++v) {
    p.tmp[(long long)r * p.V + v] = (double)p.y[b][v][l];
    p.y[b][v][l] = T(0);
  }
}

// Second half: every donor point gathers coeff * tmp over the receivers it donates to (a list
// per donor point in receiver order, so the sum does not depend on scheduling).
template <typename T>
__global__ void k_adjg_ovs_give(AdjGenOvs<T> p) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= p.nd) return;
  const int b = p.ub[u];
  const long long l = p.ul[u];
  double acc[kMaxVars] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int q = p.off[u]; q < p.off[u + 1]; ++q) {
    const double c = p.cw[q];
    const long long r = p.cr[q];
    for (int v = 0; v < p.V; ++v) acc[v] += c * p.tmp[r * p.V + v];
  }
  for (int v = 0; v < p.V; ++v) p.y[b][v][l] = (T)((double)p.y[b][v][l] + acc[v]);
}

int grid1(long long n) {
  long long g = (n + 255) / 256;
  return (int)(g < 1 ? 1 : (g > 148 * 16 ? 148 * 16 : g));
}

}  // namespace

template <typename T>
cudaError_t launch_adjg_stage(const AdjGenParams<T>& p, cudaStream_t s) {
  const long long n = (long long)p.f.nx * p.f.ny * p.f.nz;
  dim3 blk(32, 8, 1);
  dim3 grd((p.f.nx + 31) / 32, (p.f.ny + 7) / 8, p.f.nz);
  if (p.f.dim == 2) {
    k_adjg_flux<T, 2><<<grid1(n), 256, 0, s>>>(p);
    k_adjg_stage<T, 2><<<grd, blk, 0, s>>>(p);
  } else {
    k_adjg_flux<T, 3><<<grid1(n), 256, 0, s>>>(p);
    k_adjg_stage<T, 3><<<grd, blk, 0, s>>>(p);
  }
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_adjg_filter(const AdjGenFilterParams<T>& p, cudaStream_t s) {
  dim3 blk(32, 8, 1);
  dim3 grd((p.nx + 31) / 32, (p.ny + 7) / 8, p.nz);
  k_adjg_filter<T><<<grd, blk, 0, s>>>(p);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_adjg_mask(long long n, int V, const AdjGenPoint<T>& p, cudaStream_t s) {
  k_adjg_mask<T><<<grid1(n), 256, 0, s>>>(n, V, p);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_adjg_combine(long long n, int V, const AdjGenPoint<T>& p, double hb, double ha, cudaStream_t s) {
  k_adjg_combine<T><<<grid1(n), 256, 0, s>>>(n, V, p, (T)hb, (T)ha);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_adjg_bc(const BcParams<T>& p, cudaStream_t s) {
  const long long n = (long long)p.nb[0] * p.nb[1] * p.nb[2];
  k_adjg_bc<T><<<grid1(n), 256, 0, s>>>(p);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_adjg_overset(const AdjGenOvs<T>& p, cudaStream_t s) {
  if (p.n <= 0) return cudaSuccess;
  k_adjg_ovs_take<T><<<(p.n + 127) / 128, 128, 0, s>>>(p);
  if (p.nd > 0) k_adjg_ovs_give<T><<<(p.nd + 127) / 128, 128, 0, s>>>(p);
  return cudaGetLastError();
}

#define LEE_ADJG_INST(T)                                                                                 \
  template cudaError_t launch_adjg_stage<T>(const AdjGenParams<T>&, cudaStream_t);                       \
  template cudaError_t launch_adjg_filter<T>(const AdjGenFilterParams<T>&, cudaStream_t);                \
  template cudaError_t launch_adjg_mask<T>(long long, int, const AdjGenPoint<T>&, cudaStream_t);         \
  template cudaError_t launch_adjg_combine<T>(long long, int, const AdjGenPoint<T>&, double, double,     \
                                              cudaStream_t);                                             \
  template cudaError_t launch_adjg_bc<T>(const BcParams<T>&, cudaStream_t);                              \
  template cudaError_t launch_adjg_overset<T>(const AdjGenOvs<T>&, cudaStream_t);
LEE_ADJG_INST(double)
LEE_ADJG_INST(float)
#undef LEE_ADJG_INST

}  // namespace lee
