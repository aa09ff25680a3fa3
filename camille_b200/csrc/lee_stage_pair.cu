// Fused RK stage for the compensated FP32 form on uniform-mean blocks, two points per thread
// (sm_100a).
//
// The same stage as k_stage_tma (lee_tma.cu): a CTA owns a 32 x 8 tile in (i, j) and marches
// along k with the planes of every state field arriving in a shared-memory ring by TMA. Here each
// thread owns two neighbouring points along xi and computes them as a pair with the packed FP32
// instructions of sm_100 (__ffma2_rn, __fadd2_rn, __fmul2_rn): derivatives, chain rule, the LEE
// right-hand side (compute_RHS_linearized_Euler, src/solver/spatial_discretization.cpp:2053-2130,
// uniform mean: every mean-gradient term vanishes), the Freund sponge and the compensated RK
// update (RungeKutta::integrate, src/solver/temporal_discretization.cpp:205-229) issue once per
// pair, and shared and global memory move 8-byte pairs. Results are those of the one-point kernel
// up to FP32 rounding order.
//
// Every mbarrier wait is bounded (about one second); on expiry the CTA records the failure in the
// device flag, waits (bounded) for its own copies in flight and returns.
#include "lee_point.cuh"
#include "lee_tma.h"
#include "lee_tma_util.cuh"

namespace lee {
namespace {

using F2 = float2;

__device__ __forceinline__ F2 f2(float x) { return make_float2(x, x); }
__device__ __forceinline__ F2 add(F2 a, F2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ F2 mul(F2 a, F2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ F2 fma2(F2 a, F2 b, F2 c) { return __ffma2_rn(a, b, c); }
// a - b, exactly one rounding
__device__ __forceinline__ F2 sub(F2 a, F2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ F2 ld2(const float* p) { return *reinterpret_cast<const F2*>(p); }
__device__ __forceinline__ F2 ldg2(const float* p) { return __ldg(reinterpret_cast<const F2*>(p)); }
__device__ __forceinline__ void st2(float* p, F2 v) { *reinterpret_cast<F2*>(p) = v; }

// Pointwise inputs of a pair, gathered one plane ahead.
template <int DIM>
struct PairIn {
  F2 jm[DIM][DIM];  // J * metrics[d][x]
  F2 yn[DIM + 2];   // y_n (stages after the first)
  F2 av[DIM + 2];   // accumulator, or the carried rounding error (first stage)
  F2 sg;            // sponge strength
};

template <int DIM, int TR>
__device__ __forceinline__ void gather_pair(const StageParams<float>& p, unsigned l, PairIn<DIM>& in) {
  constexpr int V = DIM + 2;
  using K = Kind<TR>;
#pragma unroll
  for (int d = 0; d < DIM; ++d)
#pragma unroll
    for (int x = 0; x < DIM; ++x) in.jm[d][x] = (TR & kTrJmField) ? ldg2(p.jm[d * 3 + x].p + l) : f2(p.jm[d * 3 + x].c);
  const bool mid = !K::rhs(p) && !K::first(p);
  const bool need_av = mid || K::first(p);
#pragma unroll
  for (int v = 0; v < V; ++v) {
    in.yn[v] = (mid && !K::increment) ? ld2(p.yn[v] + l) : f2(0.f);
    in.av[v] = need_av ? (K::first(p) ? ld2(p.comp[v] + l) : ld2(p.acc[v] + l)) : f2(0.f);
  }
  in.sg = (TR & kTrSponge) ? ldg2(p.sigma + l) : f2(0.f);
}

template <int DIM, int TR>
__global__ void __launch_bounds__(128, 3)
    k_stage_pair(const __grid_constant__ FieldMaps zm, const __grid_constant__ TmaStageParams<float> P) {
  using T = float;
  constexpr int H = kFdHalf, TX = kTileX, TY = kTileY, V = DIM + 2, PV = DIM + 1;
  constexpr int HX = Box<T, H>::HX, BX = Box<T, H>::BX;
  constexpr int FB = Box<T, H>::FB, FBP = Box<T, H>::FBP;
  constexpr int NS = DIM == 3 ? 2 * H + 1 + StagePrefetch<T>::P : 1;
  static_assert(DIM == 2 || NS >= 2 * H + 2, "one barrier per plane needs a slot beyond the stencil");
  constexpr int PLANE = V * FBP;
  constexpr int LX = TX / 2;  // threads per row
  static_assert(HX % 2 == 0 && BX % 2 == 0, "pairs start on 8 bytes");
  using K = Kind<TR>;
  extern __shared__ __align__(128) unsigned char smem[];
  T* ring = reinterpret_cast<T*>(smem);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + sizeof(T) * NS * PLANE);

  const StageParams<T>& s = P.s;
  const int i0 = (int)(blockIdx.x % P.tiles_x) * TX, j0 = (int)(blockIdx.x / P.tiles_x) * TY;
  const int k0 = DIM == 3 ? (int)blockIdx.y * P.k_chunk : 0;
  const int k1 = DIM == 3 ? min(s.nz, k0 + P.k_chunk) : 1;
  const int tid = threadIdx.x, tx = tid % LX, ty = tid / LX;
  const int i = i0 + 2 * tx, j = j0 + ty;
  const bool active = i < s.nx && j < s.ny;  // nx is even: both points of the pair or neither
  const int plo = DIM == 3 ? max(0, k0 - H) : 0;
  const int phi = DIM == 3 ? min(s.nz - 1, k1 - 1 + H) : 0;

  if (tid == 0) {
    for (int q = 0; q < NS; ++q) mbar_init(&bar[q], 1);
    fence_mbar_init();
  }
  __syncthreads();
  int next_issue = plo;  // meaningful in thread 0 only
  auto issue_upto = [&](int last) {
    for (; next_issue <= min(phi, last); ++next_issue) {
      const int rel = next_issue - plo, slot = rel % NS;
      mbar_expect_tx(&bar[slot], (unsigned)(sizeof(T) * V * FB));
      for (int v = 0; v < V; ++v)
        tma_load_3d(ring + slot * PLANE + v * FBP, &zm.m[v], i0 - HX, j0 - H, next_issue, &bar[slot]);
    }
  };
  if (tid == 0) issue_upto(plo + NS - 1);

  const int c = (ty + H) * BX + (HX + 2 * tx);
  // derivative weights: along xi per point (closure classes), along eta per row
  F2 wx[2 * H + 1], wy[2 * H + 1];
  {
    const int cx0 = active ? cls_of(i, s.nx, H) : 0, cx1 = active ? cls_of(i + 1, s.nx, H) : 0;
    const int cy = active ? cls_of(j, s.ny, H) : 0;
#pragma unroll
    for (int o = 0; o <= 2 * H; ++o) {
      wx[o] = make_float2(P.w[cx0][o], P.w[cx1][o]);
      wy[o] = f2(P.w[cy][o]);
    }
  }
  // uniform mean flow, negated where the right-hand side subtracts
  F2 nub[DIM];
#pragma unroll
  for (int x = 0; x < DIM; ++x) nub[x] = f2(-s.ubar[x].c);
  const F2 nrbi = f2(-s.rhobar_inv.c), ngpb = f2(-(s.gamma * s.pbar.c));
  const F2 hh = f2(s.h), bb_ = f2(s.b), aa = f2(s.a);
  const unsigned nxy = (unsigned)s.nx * (unsigned)s.ny;
  const unsigned lij = (unsigned)i + (unsigned)s.nx * (unsigned)j;
  // monopole box test in (i, j), per point of the pair
  const bool src_ij0 = s.has_src && j >= s.src_lo[1] && j <= s.src_hi[1] && i + 1 >= s.src_lo[0] && i <= s.src_hi[0];

  PairIn<DIM> inA, inB;
  if (active) gather_pair<DIM, TR>(s, lij + nxy * (unsigned)k0, inA);
  int waited = plo;
  int sk = (k0 - plo) % NS;

  auto plane = [&](int k, PairIn<DIM>& cur, PairIn<DIM>& nxt) -> bool {
    const unsigned lk = lij + nxy * (unsigned)k;
    if (active && k + 1 < k1) gather_pair<DIM, TR>(s, lk + nxy, nxt);
    bool failed = false;
    const int need = DIM == 3 ? min(phi, k + H) : 0;
    // `waited` stays at a plane whose wait gave up, so the drain below starts there
    for (; waited <= need; ++waited) {
      const int rel = waited - plo;
      if (!mbar_wait(&bar[rel % NS], (unsigned)((rel / NS) & 1), P.wait_ns)) {
        failed = true;
        break;
      }
    }
    if (__syncthreads_or(failed)) {
      if (tid == 0) {
        atomicExch(P.err, 1);
        for (int w = waited; w < next_issue; ++w) mbar_wait(&bar[(w - plo) % NS], (unsigned)(((w - plo) / NS) & 1));
      }
      return false;
    }
    // every thread is past plane k-1, so the slot of plane k-1-H is free and takes the plane
    // NS ahead (the planes a barrier at the end of each plane would issue, one barrier per plane
    // fewer); with NS >= 2H+2 every plane up to k+H was issued at plane k-1, and the last plane
    // of the chunk issues nothing that it does not wait for
    if (DIM == 3 && tid == 0) issue_upto(k - H + NS - 1);
    if (active) {
      int zoff[2 * H + 1];
      F2 wz[2 * H + 1];
      if (DIM == 3) {
        const int cz = cls_of(k, s.nz, H);
#pragma unroll
        for (int o = -H; o <= H; ++o) {
          const int kk = min(max(k + o, plo), phi);
          int sl = sk + (kk - k);
          sl += sl < 0 ? NS : 0;
          sl -= sl >= NS ? NS : 0;
          zoff[o + H] = sl * PLANE + c;
          wz[o + H] = f2(P.w[cz][o + H]);
        }
      }
      const T* pk = ring + sk * PLANE;
      F2 D[V][DIM], q[V];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const T* f = pk + v * FBP + c;
        // xi: aligned pairs at offsets -2, 0, 2; the odd taps pair across them
        const F2 m2 = ld2(f - 2), z0 = ld2(f), p2 = ld2(f + 2);
        q[v] = z0;
        F2 dx = mul(wx[0], m2);
        dx = fma2(wx[2], z0, dx);
        dx = fma2(wx[4], p2, dx);
        dx.x = fmaf(wx[1].x, m2.y, dx.x);
        dx.y = fmaf(wx[1].y, z0.x, dx.y);
        dx.x = fmaf(wx[3].x, z0.y, dx.x);
        dx.y = fmaf(wx[3].y, p2.x, dx.y);
        F2 dy = mul(wy[0], ld2(f - 2 * BX));
#pragma unroll
        for (int o = -H + 1; o <= H; ++o) dy = fma2(wy[o + H], o == 0 ? z0 : ld2(f + o * BX), dy);
        D[v][0] = dx;
        D[v][1] = dy;
        if (DIM == 3) {
          F2 dz = mul(wz[0], ld2(ring + zoff[0] + v * FBP));
#pragma unroll
          for (int o = 1; o <= 2 * H; ++o) dz = fma2(wz[o], ld2(ring + zoff[o] + v * FBP), dz);
          D[v][DIM - 1] = dz;
        }
      }
      // physical gradients g[v][x] = sum_d JM[d][x] D_d f_v (take_derivative_xyz, :1802-1826)
      F2 g[V][DIM];
#pragma unroll
      for (int x = 0; x < DIM; ++x)
#pragma unroll
        for (int v = 0; v < V; ++v) {
          F2 t = mul(cur.jm[0][x], D[v][0]);
#pragma unroll
          for (int d = 1; d < DIM; ++d) t = fma2(cur.jm[d][x], D[v][d], t);
          g[v][x] = t;
        }
      // uniform mean flow: r_s = -u.grad s', r_u = -u.grad u' - grad p' / rho, r_p = -u.grad p' - gamma p div u'
      F2 r[V];
      {
        F2 t = mul(nub[0], g[0][0]);
#pragma unroll
        for (int x = 1; x < DIM; ++x) t = fma2(nub[x], g[0][x], t);
        r[0] = t;
      }
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        F2 t = mul(nub[0], g[1 + a][0]);
#pragma unroll
        for (int x = 1; x < DIM; ++x) t = fma2(nub[x], g[1 + a][x], t);
        r[1 + a] = fma2(g[PV][a], nrbi, t);
      }
      {
        F2 t = mul(nub[0], g[PV][0]);
#pragma unroll
        for (int x = 1; x < DIM; ++x) t = fma2(nub[x], g[PV][x], t);
#pragma unroll
        for (int x = 0; x < DIM; ++x) t = fma2(ngpb, g[1 + x][x], t);
        r[PV] = t;
      }
      // monopole: per point of the pair
      if (src_ij0 && k >= s.src_lo[2] && k <= s.src_hi[2]) {
        const T amp = s.amp_tab ? s.amp_tab[*s.step_ctr * s.nstages + s.stage] : s.src_amp;
        const int b0 = s.src_hi[0] - s.src_lo[0] + 1, b1 = s.src_hi[1] - s.src_lo[1] + 1;
        const long long row = (long long)b0 * ((j - s.src_lo[1]) + (long long)b1 * (k - s.src_lo[2]));
        if (i >= s.src_lo[0] && i <= s.src_hi[0]) r[PV].x += amp * s.src_g[row + (i - s.src_lo[0])];
        if (i + 1 >= s.src_lo[0] && i + 1 <= s.src_hi[0]) r[PV].y += amp * s.src_g[row + (i + 1 - s.src_lo[0])];
      }
      if (TR & kTrSponge) {
        const F2 nsg = mul(cur.sg, f2(-1.f));
#pragma unroll
        for (int v = 0; v < V; ++v) r[v] = fma2(nsg, q[v], r[v]);
      } else {
        for (int zz = 0; zz < s.nzones; ++zz) {
          const Zone<T>& zn = s.zones[zz];
          if (j < zn.lo[1] || j > zn.hi[1] || k < zn.lo[2] || k > zn.hi[2]) continue;
          const int b0 = zn.hi[0] - zn.lo[0] + 1, b1 = zn.hi[1] - zn.lo[1] + 1;
          const long long row = (long long)b0 * ((j - zn.lo[1]) + (long long)b1 * (k - zn.lo[2]));
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const int ii = i + e;
            if (ii < zn.lo[0] || ii > zn.hi[0]) continue;
            const T sg = zn.sig[row + (ii - zn.lo[0])];
#pragma unroll
            for (int v = 0; v < V; ++v) {
              if (e == 0) r[v].x += -sg * q[v].x;
              else r[v].y += -sg * q[v].y;
            }
          }
        }
      }
      // the compensated RK stage update (rk_update, lee_point.cuh)
      if (K::rhs(s)) {
#pragma unroll
        for (int v = 0; v < V; ++v) st2(s.zout[v] + lk, r[v]);
      } else {
        const bool first = K::first(s), last = K::last(s);
#pragma unroll
        for (int v = 0; v < V; ++v) {
          const F2 hk = mul(r[v], hh);
          const F2 yv = first ? q[v] : cur.yn[v];
          const F2 inc = fma2(bb_, hk, cur.av[v]);
          if (!last) {
            st2(s.acc[v] + lk, inc);
            st2(s.zout[v] + lk, fma2(aa, hk, yv));
          } else if (K::increment) {
            st2(s.acc[v] + lk, inc);  // the filter forms y_pre and its rounding error
          } else {
            const F2 sm = add(yv, inc);
            const F2 bv = sub(sm, yv);
            const F2 e = add(sub(yv, sub(sm, bv)), sub(inc, bv));
            st2(s.zout[v] + lk, sm);
            st2(s.acc[v] + lk, e);
          }
        }
      }
    }
    sk = sk + 1 == NS ? 0 : sk + 1;
    return true;
  };
  for (int k = k0; k < k1; k += 2) {
    if (!plane(k, inA, inB)) return;
    if (k + 1 < k1 && !plane(k + 1, inB, inA)) return;
  }
}

template <int DIM, int TR>
cudaError_t go_pair(const FieldMaps& z, const TmaStageParams<float>& p, int tiles, int chunks, cudaStream_t s) {
  constexpr int NS = DIM == 3 ? 2 * kFdHalf + 1 + StagePrefetch<float>::P : 1;
  const size_t sm = sizeof(float) * NS * (DIM + 2) * Box<float, kFdHalf>::FBP + NS * sizeof(uint64_t);
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k_stage_pair<DIM, TR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  k_stage_pair<DIM, TR><<<dim3(tiles, chunks), 128, sm, s>>>(z, p);
  return cudaGetLastError();
}

// layout traits (JmField, Sponge; Uniform is required) and the stage kind
template <int DIM, int KIND>
cudaError_t go_pair_layout(const FieldMaps& z, const TmaStageParams<float>& p, int tr, int tiles, int chunks,
                           cudaStream_t s) {
  constexpr int B = kTrTma | kTrUniform | (KIND << kKindShift);
  switch (tr & (kTrJmField | kTrSponge)) {
    case 0: return go_pair<DIM, B>(z, p, tiles, chunks, s);
    case kTrJmField: return go_pair<DIM, B | kTrJmField>(z, p, tiles, chunks, s);
    case kTrSponge: return go_pair<DIM, B | kTrSponge>(z, p, tiles, chunks, s);
    default: return go_pair<DIM, B | kTrJmField | kTrSponge>(z, p, tiles, chunks, s);
  }
}

template <int DIM>
cudaError_t go_pair_kind(const FieldMaps& z, const TmaStageParams<float>& p, int tr, int tiles, int chunks,
                         cudaStream_t s) {
  switch ((tr >> kKindShift) & 7) {
    case kKindRhs: return go_pair_layout<DIM, kKindRhs>(z, p, tr, tiles, chunks, s);
    case kKindFirst: return go_pair_layout<DIM, kKindFirst>(z, p, tr, tiles, chunks, s);
    case kKindMid: return go_pair_layout<DIM, kKindMid>(z, p, tr, tiles, chunks, s);
    case kKindLast: return go_pair_layout<DIM, kKindLast>(z, p, tr, tiles, chunks, s);
    case kKindLastIncrement: return go_pair_layout<DIM, kKindLastIncrement>(z, p, tr, tiles, chunks, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

bool stage_pair_applies(int traits, int nx) {
  return (traits & kTrTma) && (traits & kTrUniform) && ((traits >> kKindShift) & 7) != kKindRuntime && nx % 2 == 0;
}

cudaError_t launch_stage_pair(const FieldMaps& zin, const TmaStageParams<float>& p, int traits, int tiles, int chunks,
                              cudaStream_t s) {
  if (p.s.dim == 2) return go_pair_kind<2>(zin, p, traits, tiles, 1, s);
  return go_pair_kind<3>(zin, p, traits, tiles, chunks, s);
}

}  // namespace lee
