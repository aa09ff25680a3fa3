// Transposed RK stage of the discrete adjoint on 3-D blocks, staged through shared memory by TMA
// (sm_100a).
//
// zbar = L^T w with (L^T w)_v = sum_d D_d^T G^d_v(w) - sigma w_v (the fluxes G^d of lee_adjoint.cu,
// uniform mean flow). The generic kernel (k_adj_stage) rebuilds every neighbour's flux for every
// stencil tap; here a CTA owns a 32 x 8 tile in (i, j), marches along k, and builds each flux once:
// for every incoming plane (a TMA box of w and J*metrics with a two-point halo) each thread
// reads w and the nine J*metrics at its own tile point once and builds all three fluxes there;
// G^xi and G^eta go to shared memory, G^zeta to a register queue of five planes (the zeta
// stencil only reads the thread's own column). One warp adds G^xi two columns beyond the tile
// on each side of its rows and four warps G^eta two rows beyond it on each side of its columns.
// Then the transposed xi and eta stencils at the tile (kept per point in registers), and the
// plane two behind the incoming one is completed with the transposed zeta stencil. Each point's
// own work (the sponge, the ybar and next-input updates, the source gradient) is that of
// k_adj_stage. The transposed stencils must lie within two points of the row (TransOp.H == 2: the
// 4th-order difference); the host checks.
//
// Every mbarrier wait is bounded (about one second); on expiry the CTA records the failure in the
// device flag, waits (bounded) for its own copies in flight and returns.
#include "lee_tma.h"
#include "lee_tma_util.cuh"

namespace lee {
namespace {

constexpr int kAH = 2;  // halo of the fluxes along xi and eta, and of the zeta stencil

template <typename T>
struct AGeo {
  static constexpr int TX = 32, TY = 8;
  static constexpr int A = (int)(16 / sizeof(T));
  static constexpr int HX = ((kAH + A - 1) / A) * A;  // box halo along xi (16-byte aligned start)
  static constexpr int BX = TX + 2 * HX, BY = TY + 2 * kAH;
  static constexpr int FB = BX * BY;
  static constexpr int FBP = (int)((((size_t)FB * sizeof(T) + 127) / 128) * 128 / sizeof(T));
  static constexpr int NF = 14;        // boxes per plane: w (5) and J*metrics (9)
  static constexpr int NSL = 2;        // TMA slots: the plane in work and the next
  static constexpr int GXW = TX + 2 * kAH;  // G^xi row width
  static constexpr int GYH = TY + 2 * kAH;  // G^eta column height
  // the halo fluxes: G^xi at 2 kAH columns of the TY rows (one warp), G^eta at 2 kAH rows of the
  // TX columns (four warps)
  static_assert(2 * kAH * TY == 32 && 2 * kAH * TX == 128, "halo items of one and four warps");
  static constexpr int OFF_GX = NSL * NF * FBP;             // [2][5][TY][GXW]
  static constexpr int OFF_GY = OFF_GX + 2 * 5 * TY * GXW;  // [2][5][GYH][TX]
  static constexpr int OFF_BAR = OFF_GY + 2 * 5 * GYH * TX;
  static constexpr size_t BYTES = (size_t)OFF_BAR * sizeof(T) + NSL * sizeof(uint64_t);
  static_assert((OFF_BAR * sizeof(T)) % 8 == 0, "mbarrier alignment");
  static_assert((FBP * sizeof(T)) % 128 == 0, "box stride must be a multiple of 128 bytes");
};

// G^d(w) at one point, from w and the J*metrics row JM[d][.]: U = sum_x u_bar_x JM[d][x];
// G_s = -U w_s, G_u_x = -U w_u_x - gamma p_bar JM[d][x] w_p, G_p = -U w_p - (1/rho_bar) sum_a JM[d][a] w_u_a.
template <typename T>
__device__ __forceinline__ void flux(const T (&w)[5], const T (&jm)[3], const T (&ub)[3], T gpb, T rbi, T (&g)[5]) {
  const T U = ub[0] * jm[0] + ub[1] * jm[1] + ub[2] * jm[2];
  g[0] = -U * w[0];
  T su = T(0);
#pragma unroll
  for (int x = 0; x < 3; ++x) {
    g[1 + x] = -U * w[1 + x] - gpb * jm[x] * w[4];
    su += jm[x] * w[1 + x];
  }
  g[4] = -U * w[4] - rbi * su;
}

template <typename T, bool JMF>
__global__ void __launch_bounds__(256) k_adj_tma(const __grid_constant__ AdjMaps am,
                                                 const __grid_constant__ AdjTmaParams<T> P) {
  using G = AGeo<T>;
  constexpr int TX = G::TX, TY = G::TY, HX = G::HX, BX = G::BX, FBP = G::FBP, NF = G::NF;
  constexpr int GXW = G::GXW, GYH = G::GYH;
  extern __shared__ __align__(128) unsigned char smem[];
  T* ring = reinterpret_cast<T*>(smem);
  T* gxs = ring + G::OFF_GX;
  T* gys = ring + G::OFF_GY;
  uint64_t* bar = reinterpret_cast<uint64_t*>(ring + G::OFF_BAR);
  const AdjStageParams<T>& p = P.a;

  const int i0 = (int)(blockIdx.x % P.tiles_x) * TX, j0 = (int)(blockIdx.x / P.tiles_x) * TY;
  const int k0 = (int)blockIdx.y * P.k_chunk, k1 = min(p.nz, k0 + P.k_chunk);
  const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
  const int i = i0 + tx, j = j0 + ty;
  const bool active = i < p.nx && j < p.ny;
  const int plo = max(0, k0 - kAH), phi = min(p.nz - 1, k1 - 1 + kAH);
  const int nfl = JMF ? NF : 5;  // boxes a plane loads

  if (tid == 0) {
    for (int q = 0; q < G::NSL; ++q) mbar_init(&bar[q], 1);
    fence_mbar_init();
  }
  __syncthreads();
  int next_issue = plo;  // meaningful in thread 0 only
  auto issue_upto = [&](int last) {
    for (; next_issue <= min(phi, last); ++next_issue) {
      const int slot = (next_issue - plo) % G::NSL;
      mbar_expect_tx(&bar[slot], (unsigned)(sizeof(T) * G::FB * nfl));
      for (int f = 0; f < nfl; ++f)
        tma_load_3d(ring + (slot * NF + f) * FBP, &am.m[f], i0 - HX, j0 - kAH, next_issue, &bar[slot]);
    }
  };
  if (tid == 0) issue_upto(plo + G::NSL - 1);

  const T scale = p.first ? p.hb_in : T(1);
  const T ub[3] = {p.ubar[0], p.ubar[1], p.ubar[2]};
  // transposed stencil rows along xi and eta: fixed for a thread; the interior zeta row
  T rx[2 * kAH + 1], ry[2 * kAH + 1], rzi[2 * kAH + 1];
  {
    const int ci = min(i, p.nx - 1), cj = min(j, p.ny - 1);
    const double* ax = ci < p.op.E ? p.op.lt[ci] : (ci > p.nx - 1 - p.op.E ? p.op.rt[p.nx - 1 - ci] : p.op.in);
    const double* ay = cj < p.op.E ? p.op.lt[cj] : (cj > p.ny - 1 - p.op.E ? p.op.rt[p.ny - 1 - cj] : p.op.in);
#pragma unroll
    for (int t = 0; t <= 2 * kAH; ++t) {
      rx[t] = (T)ax[t + p.op.H - kAH];
      ry[t] = (T)ay[t + p.op.H - kAH];
      rzi[t] = (T)p.op.in[t + p.op.H - kAH];
    }
  }
  // w at a box point (scaled) and the J*metrics row of direction d there
  auto point = [&](const T* slot, int bx, int by, int d, T (&w)[5], T (&jm)[3]) {
    const int o = by * BX + bx;
#pragma unroll
    for (int v = 0; v < 5; ++v) w[v] = scale * slot[v * FBP + o];
#pragma unroll
    for (int x = 0; x < 3; ++x) jm[x] = JMF ? slot[(5 + d * 3 + x) * FBP + o] : p.jm[d * 3 + x].c;
  };

  const unsigned nxy = (unsigned)p.nx * (unsigned)p.ny;
  const unsigned lij = (unsigned)i + (unsigned)p.nx * (unsigned)j;
  // per-point results of the last planes: L^T restricted to xi and eta, and w at the point; and
  // G^zeta at the point over the planes the zeta stencil reads (zq[0] the oldest)
  T rq[kAH + 1][5], wq[kAH + 1][5], zq[2 * kAH + 1][5];
#pragma unroll
  for (int a = 0; a <= kAH; ++a)
#pragma unroll
    for (int v = 0; v < 5; ++v) rq[a][v] = wq[a][v] = T(0);
#pragma unroll
  for (int a = 0; a <= 2 * kAH; ++a)
#pragma unroll
    for (int v = 0; v < 5; ++v) zq[a][v] = T(0);

  for (int pl = k0 - kAH; pl <= k1 - 1 + kAH; ++pl) {
    const bool in_blk = pl >= plo && pl <= phi;
    const bool out_plane = pl >= k0 && pl < k1;
    const int kf = pl - kAH;  // the plane completed at the end of this iteration
    const bool fin = active && kf >= k0 && kf < k1;
    // the completed plane's point data, loaded early
    const unsigned lf = lij + nxy * (unsigned)max(kf, 0);
    T mu[5], yb[5], sg = T(0);
#pragma unroll
    for (int v = 0; v < 5; ++v) mu[v] = yb[v] = T(0);
    if (fin) {
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        mu[v] = p.mu[v][lf];
        yb[v] = p.first ? T(0) : p.ybar[v][lf];
      }
      if (p.sigma) sg = p.sigma[lf];
    }
    const int buf = pl & 1;
    T* gx = gxs + buf * (5 * TY * GXW);
    T* gy = gys + buf * (5 * GYH * TX);
    bool failed = false;
    T wc[5] = {T(0), T(0), T(0), T(0), T(0)};
    T gzc[5] = {T(0), T(0), T(0), T(0), T(0)};  // G^zeta at the point (zero beyond the block)
    if (in_blk) {
      const int rel = pl - plo;
      failed = !mbar_wait(&bar[rel % G::NSL], (unsigned)((rel / G::NSL) & 1), P.wait_ns);
      const T* slot = ring + (rel % G::NSL) * NF * FBP;
      T g[5];
      {
        // the tile point: w and the J*metrics rows of the three directions, read once
        const int o = (kAH + ty) * BX + HX + tx;
        T jm[3][3];
#pragma unroll
        for (int v = 0; v < 5; ++v) wc[v] = scale * slot[v * FBP + o];
#pragma unroll
        for (int d = 0; d < 3; ++d)
#pragma unroll
          for (int x = 0; x < 3; ++x) jm[d][x] = JMF ? slot[(5 + d * 3 + x) * FBP + o] : p.jm[d * 3 + x].c;
        flux(wc, jm[2], ub, p.gpb, p.rbi, gzc);
        if (out_plane) {
          flux(wc, jm[0], ub, p.gpb, p.rbi, g);
#pragma unroll
          for (int v = 0; v < 5; ++v) gx[(v * TY + ty) * GXW + tx + kAH] = g[v];
          flux(wc, jm[1], ub, p.gpb, p.rbi, g);
#pragma unroll
          for (int v = 0; v < 5; ++v) gy[(v * GYH + ty + kAH) * TX + tx] = g[v];
        }
      }
      if (out_plane && tid < 2 * kAH * (TY + TX)) {
        T w[5], jm[3];
        if (tid < 2 * kAH * TY) {
          // G^xi at columns i0-2, i0-1, i0+TX, i0+TX+1 of row r
          const int r = tid >> 2, c = tid & 3, cc = c < kAH ? c : TX + c;
          point(slot, HX - kAH + cc, kAH + r, 0, w, jm);
          flux(w, jm, ub, p.gpb, p.rbi, g);
#pragma unroll
          for (int v = 0; v < 5; ++v) gx[(v * TY + r) * GXW + cc] = g[v];
        } else {
          // G^eta at rows j0-2, j0-1, j0+TY, j0+TY+1 of column c
          const int q = tid - 2 * kAH * TY, r = q >> 5, c = q & 31, rr = r < kAH ? r : TY + r;
          point(slot, HX + c, rr, 1, w, jm);
          flux(w, jm, ub, p.gpb, p.rbi, g);
#pragma unroll
          for (int v = 0; v < 5; ++v) gy[(v * GYH + rr) * TX + c] = g[v];
        }
      }
    }
    if (__syncthreads_or(failed)) {
      if (tid == 0) {
        atomicExch(P.err, 1);
        for (int wv = pl; wv < next_issue; ++wv)
          mbar_wait(&bar[(wv - plo) % G::NSL], (unsigned)(((wv - plo) / G::NSL) & 1));
      }
      return;
    }
    // the slot of this plane has been read: load the plane after next into it
    if (tid == 0) issue_upto(pl + G::NSL);
    // shift the per-point queues; the new entries hold this plane's xi and eta terms and G^zeta
#pragma unroll
    for (int a = 0; a < kAH; ++a)
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        rq[a][v] = rq[a + 1][v];
        wq[a][v] = wq[a + 1][v];
      }
#pragma unroll
    for (int a = 0; a < 2 * kAH; ++a)
#pragma unroll
      for (int v = 0; v < 5; ++v) zq[a][v] = zq[a + 1][v];
#pragma unroll
    for (int v = 0; v < 5; ++v) zq[2 * kAH][v] = gzc[v];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      T acc = T(0);
      if (out_plane) {
#pragma unroll
        for (int t = 0; t <= 2 * kAH; ++t) {
          acc += rx[t] * gx[(v * TY + ty) * GXW + tx + t];
          acc += ry[t] * gy[(v * GYH + ty + t) * TX + tx];
        }
      }
      rq[kAH][v] = acc;
      wq[kAH][v] = wc[v];
    }
    if (fin) {
      // the zeta stencil of plane kf, then the point's own terms (k_adj_stage)
      const bool zin = kf >= p.op.E && kf <= p.nz - 1 - p.op.E;
      const double* az = kf < p.op.E ? p.op.lt[kf] : (kf > p.nz - 1 - p.op.E ? p.op.rt[p.nz - 1 - kf] : p.op.in);
      T acc[5];
#pragma unroll
      for (int v = 0; v < 5; ++v) acc[v] = rq[0][v];
      // planes kf-2..kf+2 are zq[0..4] (entries beyond the block are zero and carry zero weight)
#pragma unroll
      for (int t = 0; t <= 2 * kAH; ++t) {
        const T r = zin ? rzi[t] : (T)az[t + p.op.H - kAH];
#pragma unroll
        for (int v = 0; v < 5; ++v) acc[v] += r * zq[t][v];
      }
      const T(&wf)[5] = wq[0];
      if (p.sigma) {
#pragma unroll
        for (int v = 0; v < 5; ++v) acc[v] -= sg * wf[v];
      }
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        p.ybar[v][lf] = p.first ? mu[v] + acc[v] : yb[v] + acc[v];
        if (p.has_next) p.kout[v][lf] = p.hb_next * mu[v] + p.ha_next * acc[v];
      }
      if (p.gbar && i >= p.src_lo[0] && i <= p.src_hi[0] && j >= p.src_lo[1] && j <= p.src_hi[1] &&
          kf >= p.src_lo[2] && kf <= p.src_hi[2]) {
        const int b0 = p.src_hi[0] - p.src_lo[0] + 1, b1 = p.src_hi[1] - p.src_lo[1] + 1;
        const long long lb = (i - p.src_lo[0]) + (long long)b0 * ((j - p.src_lo[1]) + (long long)b1 * (kf - p.src_lo[2]));
        p.gbar[lb] += p.amp * (double)wf[4];
      }
    }
  }
}

template <typename T, bool JMF>
cudaError_t go_adj_tma(const AdjMaps& m, const AdjTmaParams<T>& p, int tiles, int chunks, cudaStream_t s) {
  using G = AGeo<T>;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k_adj_tma<T, JMF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::BYTES);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  k_adj_tma<T, JMF><<<dim3(tiles, chunks), 256, G::BYTES, s>>>(m, p);
  return cudaGetLastError();
}

}  // namespace

void adj_tma_box(size_t esz, int* bx, int* by, int* tx, int* ty) {
  const int a = (int)(16 / esz);
  const int hx = ((kAH + a - 1) / a) * a;
  *tx = 32;
  *ty = 8;
  *bx = 32 + 2 * hx;
  *by = 8 + 2 * kAH;
}

template <typename T>
cudaError_t launch_adj_tma(const AdjMaps& m, const AdjTmaParams<T>& p, bool jm_fields, int tiles, int chunks,
                           cudaStream_t s) {
  return jm_fields ? go_adj_tma<T, true>(m, p, tiles, chunks, s) : go_adj_tma<T, false>(m, p, tiles, chunks, s);
}

template cudaError_t launch_adj_tma<float>(const AdjMaps&, const AdjTmaParams<float>&, bool, int, int, cudaStream_t);
template cudaError_t launch_adj_tma<double>(const AdjMaps&, const AdjTmaParams<double>&, bool, int, int, cudaStream_t);

}  // namespace lee
