// Pointwise part of the fused RK stage, shared by every stage kernel: the LEE
// right-hand side from the physical gradients (compute_RHS_linearized_Euler,
// camille src/solver/spatial_discretization.cpp:2053-2130), the monopole source and
// the Freund sponges (src/solver/source.cpp:10-18, :174-201), then the Runge-Kutta
// stage update with the hole bypass (RungeKutta::integrate,
// src/solver/temporal_discretization.cpp:205-229).
#pragma once

#include "lee_internal.h"

namespace lee {

template <typename T, typename I>
__device__ __forceinline__ T cval(const Coef<T>& c, I l) {
  return c.p ? __ldg(c.p + l) : c.c;
}

// The stage's kind: from the traits when they fix it, else from p.stage and p.last.
template <int TR>
struct Kind {
  static constexpr int K = (TR >> kKindShift) & 7;
  template <typename T>
  __device__ __forceinline__ static bool rhs(const StageParams<T>& p) {
    return K == kKindRuntime ? p.stage < 0 : K == kKindRhs;
  }
  template <typename T>
  __device__ __forceinline__ static bool first(const StageParams<T>& p) {
    return K == kKindRuntime ? p.stage == 0 : K == kKindFirst;
  }
  template <typename T>
  __device__ __forceinline__ static bool last(const StageParams<T>& p) {
    return K == kKindRuntime ? p.last != 0 : (K == kKindLast || K == kKindLastIncrement);
  }
  // the last stage writes the increment alone (compile-time kinds only)
  static constexpr bool increment = K == kKindLastIncrement;
};

// Per-point inputs read from global memory, gathered before the arithmetic so that
// every load of the point is in flight at once.
template <typename T, int DIM>
struct PointIn {
  T jm[DIM][DIM];     // J * metrics[d][x]
  T yn[DIM + 2];      // y_n (stages after the first)
  T av[DIM + 2];      // accumulator (stages after the first) or carried error (compensated, first stage)
  T sg;               // sponge strength (kTrSponge)
};

template <typename T, int DIM, bool COMP, int TR, typename I>
__device__ __forceinline__ void gather(const StageParams<T>& p, I l, PointIn<T, DIM>& in) {
  constexpr int V = DIM + 2;
  using K = Kind<TR>;
#pragma unroll
  for (int d = 0; d < DIM; ++d)
#pragma unroll
    for (int x = 0; x < DIM; ++x) {
      const Coef<T>& c = p.jm[d * 3 + x];
      // TMA kernels: every entry is a field when any is
      in.jm[d][x] = (TR & kTrJmField) ? ((TR & kTrTma) ? __ldg(c.p + l) : cval(c, l)) : c.c;
    }
  const bool mid = !K::rhs(p) && !K::first(p);
  const bool need_yn = mid && (COMP || !K::last(p)) && !K::increment;
  const bool need_av = mid || (COMP && K::first(p));
#pragma unroll
  for (int v = 0; v < V; ++v) {
    in.yn[v] = need_yn ? p.yn[v][l] : T(0);
    in.av[v] = need_av ? (K::first(p) ? p.comp[v][l] : p.acc[v][l]) : T(0);
  }
  in.sg = (TR & kTrSponge) ? __ldg(p.sigma + l) : T(0);
}

template <typename T, int DIM, int TR, typename I>
__device__ __forceinline__ void rhs_mean_terms(const StageParams<T>& p, I l, const T (&g)[DIM + 2][DIM],
                                               const T (&q)[DIM + 2], const T (&ub)[DIM], T (&r)[DIM + 2]);
template <typename T, int DIM, bool COMP, int TR, typename I>
__device__ __forceinline__ void rk_update(const StageParams<T>& p, I l, const T (&q)[DIM + 2],
                                          const PointIn<T, DIM>& in, const T (&r)[DIM + 2]);

// D[v][d]: computational-space derivative of field v along direction d; q[v]: the
// stage input at the point; in: the gathered inputs. Writes the next stage input and
// the accumulator.
template <typename T, int DIM, bool COMP, int TR, typename I>
__device__ __forceinline__ void rhs_update(const StageParams<T>& p, I l, int i, int j, int k,
                                           const T (&D)[DIM + 2][DIM], const T (&q)[DIM + 2],
                                           const PointIn<T, DIM>& in) {
  constexpr int V = DIM + 2;
  constexpr int P = DIM + 1;
  // physical gradients g[v][x] = sum_d JM[d][x] D_d f_v (take_derivative_xyz, :1802-1826)
  T g[V][DIM];
#pragma unroll
  for (int x = 0; x < DIM; ++x) {
#pragma unroll
    for (int v = 0; v < V; ++v) {
      T s = T(0);
#pragma unroll
      for (int d = 0; d < DIM; ++d) s += in.jm[d][x] * D[v][d];
      g[v][x] = s;
    }
  }
  constexpr bool UNI = (TR & kTrUniform) != 0;
  T ub[DIM];
#pragma unroll
  for (int x = 0; x < DIM; ++x) ub[x] = UNI ? p.ubar[x].c : cval(p.ubar[x], l);
  T r[V];
  if (UNI) {
    // uniform mean flow: every mean-gradient term vanishes
    T rs = T(0);
#pragma unroll
    for (int x = 0; x < DIM; ++x) rs -= ub[x] * g[0][x];
    r[0] = rs;
    const T rbi = p.rhobar_inv.c;
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
      T ru = T(0);
#pragma unroll
      for (int x = 0; x < DIM; ++x) ru -= ub[x] * g[1 + a][x];
      ru -= g[P][a] * rbi;
      r[1 + a] = ru;
    }
    T rp = T(0);
    const T gpb = p.gamma * p.pbar.c;
#pragma unroll
    for (int x = 0; x < DIM; ++x) {
      rp -= ub[x] * g[P][x];
      rp -= gpb * g[1 + x][x];
    }
    r[P] = rp;
  } else {
    rhs_mean_terms<T, DIM, TR>(p, l, g, q, ub, r);
  }
  if constexpr (DIM == 2 && !(TR & kTrTma)) {
    if (p.axisym) {
      // -gamma (p_bar u_r' + p' u_r_bar) / (r + DUMMY_SMALL), in FP64 in the reference's order
      // (src/solver/spatial_discretization.cpp:2118-2126)
      const double pb = (double)cval(p.pbar, l), ur = (double)cval(p.ubar[1], l);
      const double num = __dadd_rn(__dmul_rn(pb, (double)q[2]), __dmul_rn((double)q[P], ur));
      r[P] -= (T)__ddiv_rn(__dmul_rn((double)p.gamma, num), __dadd_rn(p.ry[l], 1e-99));
    }
  }
  if (p.has_src && i >= p.src_lo[0] && i <= p.src_hi[0] && j >= p.src_lo[1] && j <= p.src_hi[1] &&
      k >= p.src_lo[2] && k <= p.src_hi[2]) {
    int b0 = p.src_hi[0] - p.src_lo[0] + 1, b1 = p.src_hi[1] - p.src_lo[1] + 1;
    long long lb = (i - p.src_lo[0]) + (long long)b0 * ((j - p.src_lo[1]) + (long long)b1 * (k - p.src_lo[2]));
    const T amp = p.amp_tab ? p.amp_tab[*p.step_ctr * p.nstages + p.stage] : p.src_amp;
    r[P] += amp * p.src_g[lb];
  }
  if (TR & kTrSponge) {
#pragma unroll
    for (int v = 0; v < V; ++v) r[v] += -in.sg * (q[v] - T(0));
  } else {
    for (int z = 0; z < p.nzones; ++z) {
      const Zone<T>& zn = p.zones[z];
      if (i < zn.lo[0] || i > zn.hi[0] || j < zn.lo[1] || j > zn.hi[1] || k < zn.lo[2] || k > zn.hi[2]) continue;
      int b0 = zn.hi[0] - zn.lo[0] + 1, b1 = zn.hi[1] - zn.lo[1] + 1;
      long long lb = (i - zn.lo[0]) + (long long)b0 * ((j - zn.lo[1]) + (long long)b1 * (k - zn.lo[2]));
      T sg = zn.sig[lb];
      if (zn.ref) {
        // source::apply_bufferZone_Freund_harmonicWave (src/solver/source.cpp:264-320): the
        // reference state is the wave at the stage time
        const long long nbz = (long long)b0 * b1 * (zn.hi[2] - zn.lo[2] + 1);
#pragma unroll
        for (int v = 0; v < V; ++v) r[v] += -sg * (q[v] - zn.ref[v * nbz + lb]);
        continue;
      }
#pragma unroll
      for (int v = 0; v < V; ++v) r[v] += -sg * (q[v] - T(0));
    }
  }
  rk_update<T, DIM, COMP, TR>(p, l, q, in, r);
}

// The LEE right-hand side of a non-uniform mean flow: every coefficient is read at the point
// when it varies, and terms whose mean gradient is identically zero are skipped.
template <typename T, int DIM, int TR, typename I>
__device__ __forceinline__ void rhs_mean_terms(const StageParams<T>& p, I l, const T (&g)[DIM + 2][DIM],
                                               const T (&q)[DIM + 2], const T (&ub)[DIM], T (&r)[DIM + 2]) {
  constexpr int P = DIM + 1;
  {
    T rs = T(0);
#pragma unroll
    for (int x = 0; x < DIM; ++x) {
      rs -= ub[x] * g[0][x];
      if (!p.gs[x].zero) rs -= q[1 + x] * cval(p.gs[x], l);
    }
    r[0] = rs;
  }
  T rr = T(0);
  if (p.need_rho) {
    if ((Kind<TR>::first(p) || Kind<TR>::rhs(p)) && p.rho_prev) {
      rr = p.rho_prev[l];
    } else {
      rr = q[P] * p.inv_gamma * (T(1) / cval(p.pbar, l)) - q[0];
    }
  }
  const T rbi = cval(p.rhobar_inv, l);
#pragma unroll
  for (int a = 0; a < DIM; ++a) {
    T ru = T(0);
#pragma unroll
    for (int x = 0; x < DIM; ++x) {
      ru -= ub[x] * g[1 + a][x];
      const Coef<T>& gu = p.gu[a * 3 + x];
      if (!gu.zero) ru -= (q[1 + x] + rr * ub[x]) * cval(gu, l);
    }
    ru -= g[P][a] * rbi;
    r[1 + a] = ru;
  }
  {
    T rp = T(0);
    const T pb = cval(p.pbar, l);
#pragma unroll
    for (int x = 0; x < DIM; ++x) {
      rp -= ub[x] * g[P][x];
      if (!p.gp[x].zero) rp -= q[1 + x] * cval(p.gp[x], l);
      rp -= p.gamma * pb * g[1 + x][x];
      const Coef<T>& gu = p.gu[x * 3 + x];
      if (!gu.zero) rp -= p.gamma * q[P] * cval(gu, l);
    }
    r[P] = rp;
  }
}

// The Runge-Kutta stage update of one point from its right-hand side r.
template <typename T, int DIM, bool COMP, int TR, typename I>
__device__ __forceinline__ void rk_update(const StageParams<T>& p, I l, const T (&q)[DIM + 2],
                                          const PointIn<T, DIM>& in, const T (&r)[DIM + 2]) {
  constexpr int V = DIM + 2;
  using K = Kind<TR>;
  if (K::rhs(p)) {  // right-hand side only (spatial::compute_RHS)
#pragma unroll
    for (int v = 0; v < V; ++v) p.zout[v][l] = r[v];
    return;
  }
  const bool first = K::first(p), last = K::last(p);
  const bool hole = p.iblank && p.iblank[l] == 1;  // null on blocks without holes
#pragma unroll
  for (int v = 0; v < V; ++v) {
    if (hole) {
      p.acc[v][l] = T(0);
      if (!last || COMP) p.zout[v][l] = T(0);
      continue;
    }
    const T hk = r[v] * p.h;
    if (!COMP) {
      // y_next = y_n + sum b_i h k_i; the next stage input y_n + a h k_i
      const T yv = first ? q[v] : in.yn[v];
      const T prev = first ? q[v] : in.av[v];
      p.acc[v][l] = prev + p.b * hk;
      if (!last) p.zout[v][l] = yv + p.a * hk;
    } else {
      // compensated form: acc carries the increment of y since y_n plus the carried
      // rounding error of y; the last stage forms y_pre = y_n + increment as an exact
      // two-float sum (y_pre in zout, its rounding error in acc)
      const T yv = first ? q[v] : in.yn[v];
      const T inc = in.av[v] + p.b * hk;
      if (!last) {
        p.acc[v][l] = inc;
        p.zout[v][l] = yv + p.a * hk;
      } else if (K::increment) {
        p.acc[v][l] = inc;  // the filter forms y_pre and its rounding error
      } else {
        const T s = yv + inc;
        const T bb = s - yv;
        const T e = (yv - (s - bb)) + (inc - bb);
        p.zout[v][l] = s;
        p.acc[v][l] = e;
      }
    }
  }
}

}  // namespace lee
