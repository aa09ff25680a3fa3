// TMA-staged, k-marching kernels (sm_100a). On a block with holes the closure class of each
// point along each direction comes from its closure code rather than its position, and the
// RK update and the filter's output take the hole mask.
//
// Stage kernel: a CTA owns a 32 x 8 tile in (i, j) and marches along k through a
// chunk of planes. Each plane of every state field arrives in shared memory as one
// box (tile plus stencil halo) through cp.async.bulk.tensor, completing on an
// mbarrier; a ring of 2h+2 planes holds the zeta stencil and one plane of prefetch,
// so HBM loads for plane k+h+1 overlap the arithmetic of plane k. Every point then
// takes its xi/eta/zeta derivatives from shared memory and runs the pointwise RHS and
// RK update (lee_point.cuh) with coalesced loads/stores of y_n, the accumulator and
// the coefficient fields.
//
// Filter kernel: the dimension-split filter of spatial::apply_filter
// (src/solver/spatial_discretization.cpp:2191-2246) fused into one pass per field:
// for each incoming plane, F_xi on the tile plus its eta halo (into shared memory),
// F_eta at the tile points, and a register queue of 2h+1 planes for F_zeta, so the
// pre-filter state is read once and the filtered state written once.
//
// Every mbarrier wait is bounded (about one second of %globaltimer); on expiry the
// CTA records the failure in a device flag, waits (bounded) for its own copies in
// flight and returns, and the host reports LEE_ERR_TIMEOUT.
#include "lee_point.cuh"
#include "lee_tma.h"
#include "lee_tma_util.cuh"

namespace lee {
namespace {

template <typename T, int DIM, bool COMP, int TR>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 3 : 2)
    k_stage_tma(const __grid_constant__ FieldMaps zm, const __grid_constant__ TmaStageParams<T> P) {
  constexpr int H = kFdHalf, TX = kTileX, TY = kTileY, V = DIM + 2;
  constexpr int HX = Box<T, H>::HX, BX = Box<T, H>::BX;
  constexpr int FB = Box<T, H>::FB;    // elements one box load writes
  constexpr int FBP = Box<T, H>::FBP;  // stride between boxes in shared memory
  constexpr int NS = DIM == 3 ? 2 * H + 1 + StagePrefetch<T>::P : 1;
  static_assert(DIM == 2 || NS >= 2 * H + 2, "one barrier per plane needs a slot beyond the stencil");
  constexpr int PLANE = V * FBP;
  extern __shared__ __align__(128) unsigned char smem[];
  T* ring = reinterpret_cast<T*>(smem);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + sizeof(T) * NS * PLANE);

  const StageParams<T>& s = P.s;
  const int i0 = (int)(blockIdx.x % P.tiles_x) * TX, j0 = (int)(blockIdx.x / P.tiles_x) * TY;
  const int k0 = DIM == 3 ? (int)blockIdx.y * P.k_chunk : 0;
  const int k1 = DIM == 3 ? min(s.nz, k0 + P.k_chunk) : 1;
  const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
  const int i = i0 + tx, j = j0 + ty;
  const bool active = i < s.nx && j < s.ny;
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

  const int c = (ty + H) * BX + (tx + HX);
  // closure-class weights along xi and eta: fixed for a thread by its position (kept in
  // registers), or on a block with holes read per plane from the closure codes
  const bool holes = s.code[0] != nullptr;
  T wx[2 * H + 1], wy[2 * H + 1];
  {
    const int cx = active && !holes ? cls_of(i, s.nx, H) : 0;
    const int cy = active && !holes ? cls_of(j, s.ny, H) : 0;
#pragma unroll
    for (int o = 0; o <= 2 * H; ++o) {
      wx[o] = P.w[cx][o];
      wy[o] = P.w[cy][o];
    }
  }
  // point offsets fit 32 bits (the host checks the block size)
  const unsigned nxy = (unsigned)s.nx * (unsigned)s.ny;
  const unsigned lij = (unsigned)i + (unsigned)s.nx * (unsigned)j;
  // pointwise inputs (y_n, accumulator, J*metrics, sponge): in FP32 they are software-pipelined
  // one plane ahead, so the loads for plane k+1 are in flight while plane k is computed; in
  // FP64 (twice the registers) they are issued at the top of the plane, before the wait
  constexpr bool PIPE = sizeof(T) == 4;
  PointIn<T, DIM> inA, inB;
  if (PIPE && active) gather<T, DIM, COMP, TR>(s, lij + nxy * (unsigned)k0, inA);
  int waited = plo;
  int sk = (k0 - plo) % NS;  // ring slot of plane k

  // one plane: `cur` holds its gathered inputs, `nxt` receives those of the next plane
  auto plane = [&](int k, PointIn<T, DIM>& cur, PointIn<T, DIM>& nxt) -> bool {
    const unsigned lk = lij + nxy * (unsigned)k;
    if (PIPE && active && k + 1 < k1) gather<T, DIM, COMP, TR>(s, lk + nxy, nxt);
    if (!PIPE && active) gather<T, DIM, COMP, TR>(s, lk, cur);
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
    // NS ahead; with NS >= 2H+2 every plane up to k+H was issued at plane k-1, and the last
    // plane of the chunk issues nothing that it does not wait for
    if (DIM == 3 && tid == 0) issue_upto(k - H + NS - 1);
    if (active) {
      if (holes) {
        const int cx = cls_of_code(s.code[0][lk], H), cy = cls_of_code(s.code[1][lk], H);
#pragma unroll
        for (int o = 0; o <= 2 * H; ++o) {
          wx[o] = P.w[cx][o];
          wy[o] = P.w[cy][o];
        }
      }
      // ring slots of planes k-H..k+H; planes outside [plo, phi] map to a loaded plane and
      // carry zero weight (their closure-class weights are zero)
      int zoff[2 * H + 1];
      T wz[2 * H + 1];
      if (DIM == 3) {
        const int cz = holes ? cls_of_code(s.code[2][lk], H) : cls_of(k, s.nz, H);
#pragma unroll
        for (int o = -H; o <= H; ++o) {
          const int kk = min(max(k + o, plo), phi);
          int sl = sk + (kk - k);
          sl += sl < 0 ? NS : 0;
          sl -= sl >= NS ? NS : 0;
          zoff[o + H] = sl * PLANE + c;
        }
#pragma unroll
        for (int o = 0; o <= 2 * H; ++o) wz[o] = P.w[cz][o];
      }
      const T* pk = ring + sk * PLANE;
      T D[V][DIM], q[V];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const T* f = pk + v * FBP + c;
        q[v] = f[0];
        T dx = T(0), dy = T(0);
#pragma unroll
        for (int o = -H; o <= H; ++o) {
          dx += wx[o + H] * f[o];
          dy += wy[o + H] * f[o * BX];
        }
        D[v][0] = dx;
        D[v][1] = dy;
        if (DIM == 3) {
          T dz = T(0);
#pragma unroll
          for (int o = 0; o <= 2 * H; ++o) dz += wz[o] * ring[zoff[o] + v * FBP];
          D[v][DIM - 1] = dz;
        }
      }
      rhs_update<T, DIM, COMP, TR>(s, lk, i, j, k, D, q, cur);
    }
    sk = sk + 1 == NS ? 0 : sk + 1;
    return true;
  };
  if (PIPE) {
    // planes in pairs, the two input sets alternating roles (no copies between them)
    for (int k = k0; k < k1; k += 2) {
      if (!plane(k, inA, inB)) return;
      if (k + 1 < k1 && !plane(k + 1, inB, inA)) return;
    }
  } else {
    for (int k = k0; k < k1; ++k)
      if (!plane(k, inA, inA)) return;
  }
}

// One tile row per thread row (the form of k_filter_tma with RY = 1, scheduled by the compiler
// without the per-row arrays).
// INC (compensated form): the step's last stage wrote its increment alone, and the filter's input
// is the pair y_n (ym) and increment (dm): each incoming plane's two boxes land in one ring slot,
// each thread forms its point's y_pre = y_n + increment and rounding error as the exact two-float
// sum the last stage would have formed, the other box points become fl(y_n + increment) (the same
// y_pre), and the rest is the filter of y_pre with its error: the same bits as the pair written by
// the last stage, with one read of y_n in place of the last stage's read of y_n and writes of
// y_pre and its error.
template <typename T, int DIM, bool COMP, int HF, bool INC = false, bool HOLES = false>
__global__ void __launch_bounds__(256) k_filter_tma_row(const __grid_constant__ FieldMaps ym,
                                                    const __grid_constant__ FieldMaps dm,
                                                    const __grid_constant__ TmaFilterParams<T> P) {
  static_assert(!INC || COMP, "the increment input is the compensated form's");
  static_assert(!(INC && HOLES), "the increment input is not taken on blocks with holes");
  constexpr int NB = INC ? 2 : 1;  // boxes per ring slot
  constexpr int TX = kTileX, TY = kTileY, NQ = 2 * HF + 1, NSF = kFilterSlots;
  constexpr int HX = Box<T, HF>::HX, BX = Box<T, HF>::BX, BY = Box<T, HF>::BY;
  constexpr int FB = Box<T, HF>::FB;    // elements one box load writes
  constexpr int FBP = Box<T, HF>::FBP;  // stride between boxes in shared memory
  extern __shared__ __align__(128) unsigned char smem[];
  T* ring = reinterpret_cast<T*>(smem);
  T* u1 = ring + NSF * NB * FBP;  // [BY][TX]
  uint64_t* bar = reinterpret_cast<uint64_t*>(u1 + BY * TX);

  const int v = blockIdx.z;
  const int i0 = (int)(blockIdx.x % P.tiles_x) * TX, j0 = (int)(blockIdx.x / P.tiles_x) * TY;
  const int k0 = DIM == 3 ? (int)blockIdx.y * P.k_chunk : 0;
  const int k1 = DIM == 3 ? min(P.nz, k0 + P.k_chunk) : 1;
  const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
  const int i = i0 + tx, j = j0 + ty;
  const bool active = i < P.nx && j < P.ny;
  const int plo = DIM == 3 ? max(0, k0 - HF) : 0;
  const int phi = DIM == 3 ? min(P.nz - 1, k1 - 1 + HF) : 0;

  if (tid == 0) {
    for (int q = 0; q < NSF; ++q) mbar_init(&bar[q], 1);
    fence_mbar_init();
  }
  __syncthreads();
  int next_issue = plo;
  auto issue_upto = [&](int last) {
    for (; next_issue <= min(phi, last); ++next_issue) {
      const int slot = (next_issue - plo) % NSF;
      mbar_expect_tx(&bar[slot], (unsigned)(sizeof(T) * FB * NB));
      tma_load_3d(ring + slot * NB * FBP, &ym.m[v], i0 - HX, j0 - HF, next_issue, &bar[slot]);
      if (INC) tma_load_3d(ring + (slot * NB + 1) * FBP, &dm.m[v], i0 - HX, j0 - HF, next_issue, &bar[slot]);
    }
  };
  if (tid == 0) issue_upto(plo + NSF - 1);

  // closure-class weights along xi and eta: fixed for a thread by its position (kept in
  // registers), or on a block with holes (HOLES: P.code and P.iblank set) read per plane from
  // the closure codes; the form without holes keeps none of that code
  constexpr bool holes = HOLES;
  T wx[NQ], wy[NQ];
  {
    const int cx = cls_of(min(i, P.nx - 1), P.nx, P.nb);
    const int cy = cls_of(min(j, P.ny - 1), P.ny, P.nb);
#pragma unroll
    for (int o = 0; o < NQ; ++o) {
      wx[o] = P.w[cx][o];
      wy[o] = P.w[cy][o];
    }
  }
  // the class of a point of plane kp from its code (0 outside the block: those box values are
  // the zero fill and feed nothing)
  auto code_cls = [&](int d, int ii, int jj, int kp) -> int {
    if (ii >= P.nx || jj < 0 || jj >= P.ny) return 0;
    return cls_of_code(P.code[d][ii + (long long)P.nx * (jj + (long long)P.ny * kp)], P.nb);
  };
  T uq[NQ], dq[HF + 1], xq[HF + 1], eq[INC ? HF + 1 : 1];
#pragma unroll
  for (int q = 0; q < NQ; ++q) uq[q] = T(0);
#pragma unroll
  for (int q = 0; q <= HF; ++q) dq[q] = xq[q] = T(0);
#pragma unroll
  for (int q = 0; q < (INC ? HF + 1 : 1); ++q) eq[q] = T(0);
  const int pstart = DIM == 3 ? k0 - HF : 0, pend = DIM == 3 ? k1 - 1 + HF : 0;
  for (int p = pstart; p <= pend; ++p) {
    T u2 = T(0), d12 = T(0), xc = T(0);
    const int kf = DIM == 3 ? p - HF : 0;  // the plane finalized at the end of this iteration
    const bool fin = active && kf >= k0 && kf < k1;
    const long long lf = i + (long long)P.nx * (j + (long long)P.ny * kf);
    const T ef = (COMP && !INC && fin) ? P.err[v][lf] : T(0);
    T ein = T(0);  // INC: the rounding error of y_pre at this thread's point of plane p
    if (p >= plo && p <= phi) {
      const int rel = p - plo;
      const bool ok = mbar_wait(&bar[rel % NSF], (unsigned)((rel / NSF) & 1), P.wait_ns);
      if (__syncthreads_or(!ok)) {
        if (tid == 0) {
          atomicExch(P.errflag, 1);
          // every copy still in flight, the one whose wait gave up included
          for (int w = p; w < next_issue; ++w) mbar_wait(&bar[(w - plo) % NSF], (unsigned)(((w - plo) / NSF) & 1));
        }
        return;
      }
      T* box = ring + (rel % NSF) * NB * FBP;
      if (INC) {
        // y_pre = y_n + increment and its rounding error at the thread's own point; fl(y_n +
        // increment) at the box's other points (the halo), then one barrier
        const T* dbox = box + FBP;
        const int c0 = (ty + HF) * BX + tx + HX;
        const T yv = box[c0], dv = dbox[c0];
        const T sm = yv + dv;
        const T bb = sm - yv;
        ein = (yv - (sm - bb)) + (dv - bb);
        box[c0] = sm;
        for (int q = tid; q < FB; q += TX * TY) {
          const int r = q / BX, cc = q - r * BX;
          if (r >= HF && r < HF + TY && cc >= HX && cc < HX + TX) continue;  // a tile point: its owner's
          box[q] = box[q] + dbox[q];
        }
        __syncthreads();
      }
      if (holes) {
        const int cx = code_cls(0, i, j, p), cy = code_cls(1, i, j, p);
#pragma unroll
        for (int o = 0; o < NQ; ++o) {
          wx[o] = P.w[cx][o];
          wy[o] = P.w[cy][o];
        }
      }
      // F_xi on the thread's own row (kept in registers) and on its share of the eta halo rows
      const T* fc = box + (ty + HF) * BX + tx + HX;
      xc = fc[0];
      T d1 = T(0);
#pragma unroll
      for (int o = -HF; o <= HF; ++o) d1 += wx[o + HF] * fc[o];
      const T u1c = COMP ? xc + d1 : d1;
      u1[(ty + HF) * TX + tx] = u1c;
      for (int r = ty; r < 2 * HF; r += TY) {
        const int row = r < HF ? r : r + TY;
        const T* f = box + row * BX + tx + HX;
        T wh[NQ];
        const int ch = holes ? code_cls(0, i, j0 - HF + row, p) : -1;
#pragma unroll
        for (int o = 0; o < NQ; ++o) wh[o] = ch < 0 ? wx[o] : P.w[ch][o];
        T d = T(0);
#pragma unroll
        for (int o = -HF; o <= HF; ++o) d += wh[o + HF] * f[o];
        u1[row * TX + tx] = COMP ? f[0] + d : d;
      }
      __syncthreads();
      // every thread is done with this plane's box: its slot takes the plane NSF ahead. The
      // eta pass below reads u1 only, and the next plane writes u1 after its own wait barrier,
      // which every thread reaches only once this pass is done
      if (tid == 0) issue_upto(p + NSF);
      T dy = T(0);
#pragma unroll
      for (int o = -HF; o <= HF; ++o) dy += wy[o + HF] * (o == 0 ? u1c : u1[(ty + HF + o) * TX + tx]);
      if (COMP) {
        u2 = u1c + dy;
        d12 = d1 + dy;
      } else {
        u2 = dy;
      }
    }
#pragma unroll
    for (int q = 0; q < NQ - 1; ++q) uq[q] = uq[q + 1];
    uq[NQ - 1] = u2;
#pragma unroll
    for (int q = 0; q < HF; ++q) {
      dq[q] = dq[q + 1];
      xq[q] = xq[q + 1];
    }
    dq[HF] = d12;
    xq[HF] = xc;
    if (INC) {
#pragma unroll
      for (int q = 0; q < HF; ++q) eq[q] = eq[q + 1];
      eq[HF] = ein;
    }
    const int k = kf;
    if (!fin) continue;
    T fz, x0, dsum;
    if (DIM == 3) {
      const int cz = holes ? code_cls(2, i, j, k) : cls_of(k, P.nz, P.nb);
      fz = T(0);
      if (cz == 0) {
        // interior plane: the loop-invariant interior weights
#pragma unroll
        for (int o = 0; o < NQ; ++o) fz += P.w[0][o] * uq[o];
      } else {
#pragma unroll
        for (int o = 0; o < NQ; ++o) fz += P.w[cz][o] * uq[o];
      }
      x0 = xq[0];
      dsum = dq[0];
    } else {
      fz = u2;
      x0 = xc;
      dsum = d12;
    }
    const T e0 = INC ? (DIM == 3 ? eq[0] : ein) : ef;
    const long long l = lf;
    const bool hole = HOLES && P.iblank[l] == 1;  // temporal::iblank_correction
    if (!COMP) {
      P.out[v][l] = hole ? T(0) : (T(1) - P.blend) * x0 + P.blend * fz;
    } else {
      const T D = DIM == 3 ? dsum + fz : dsum;
      const T t = P.blend * D + e0;
      const T sm = x0 + t;
      const T bb = sm - x0;
      P.out[v][l] = hole ? T(0) : sm;
      P.comp[v][l] = hole ? T(0) : (x0 - (sm - bb)) + (t - bb);
    }
  }
}

template <typename T, int DIM, bool COMP, int HF, int RY>
__global__ void __launch_bounds__(256) k_filter_tma(const __grid_constant__ FieldMaps ym,
                                                    const __grid_constant__ TmaFilterParams<T> P) {
  constexpr int TX = kTileX, TY = kTileY, TYE = kTileY * RY, NQ = 2 * HF + 1, NSF = kFilterSlots;
  using FBox = Box<T, HF, RY>;
  constexpr int HX = FBox::HX, BX = FBox::BX, BY = FBox::BY;
  constexpr int FB = FBox::FB;    // elements one box load writes
  constexpr int FBP = FBox::FBP;  // stride between boxes in shared memory
  extern __shared__ __align__(128) unsigned char smem[];
  T* ring = reinterpret_cast<T*>(smem);
  T* u1 = ring + NSF * FBP;  // [BY][TX]
  uint64_t* bar = reinterpret_cast<uint64_t*>(u1 + BY * TX);

  const int v = blockIdx.z;
  const int i0 = (int)(blockIdx.x % P.tiles_x) * TX, j0 = (int)(blockIdx.x / P.tiles_x) * TYE;
  const int k0 = DIM == 3 ? (int)blockIdx.y * P.k_chunk : 0;
  const int k1 = DIM == 3 ? min(P.nz, k0 + P.k_chunk) : 1;
  const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
  const int i = i0 + tx;
  // the thread's rows j0 + ty + TY r, r < RY
  int jr[RY];
  bool active[RY];
#pragma unroll
  for (int r = 0; r < RY; ++r) {
    jr[r] = j0 + ty + TY * r;
    active[r] = i < P.nx && jr[r] < P.ny;
  }
  const int plo = DIM == 3 ? max(0, k0 - HF) : 0;
  const int phi = DIM == 3 ? min(P.nz - 1, k1 - 1 + HF) : 0;

  if (tid == 0) {
    for (int q = 0; q < NSF; ++q) mbar_init(&bar[q], 1);
    fence_mbar_init();
  }
  __syncthreads();
  int next_issue = plo;
  auto issue_upto = [&](int last) {
    for (; next_issue <= min(phi, last); ++next_issue) {
      const int slot = (next_issue - plo) % NSF;
      mbar_expect_tx(&bar[slot], (unsigned)(sizeof(T) * FB));
      tma_load_3d(ring + slot * FBP, &ym.m[v], i0 - HX, j0 - HF, next_issue, &bar[slot]);
    }
  };
  if (tid == 0) issue_upto(plo + NSF - 1);

  // closure-class weights along xi and eta are fixed for a thread: keep them in registers
  T wx[NQ], wy[RY][NQ];
  {
    const int cx = cls_of(min(i, P.nx - 1), P.nx, P.nb);
#pragma unroll
    for (int o = 0; o < NQ; ++o) wx[o] = P.w[cx][o];
#pragma unroll
    for (int r = 0; r < RY; ++r) {
      const int cy = cls_of(min(jr[r], P.ny - 1), P.ny, P.nb);
#pragma unroll
      for (int o = 0; o < NQ; ++o) wy[r][o] = P.w[cy][o];
    }
  }
  T uq[RY][NQ], dq[RY][HF + 1], xq[RY][HF + 1];
#pragma unroll
  for (int r = 0; r < RY; ++r) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) uq[r][q] = T(0);
#pragma unroll
    for (int q = 0; q <= HF; ++q) dq[r][q] = xq[r][q] = T(0);
  }
  const int pstart = DIM == 3 ? k0 - HF : 0, pend = DIM == 3 ? k1 - 1 + HF : 0;
  for (int p = pstart; p <= pend; ++p) {
    T u2[RY], d12[RY], xc[RY];
    const int kf = DIM == 3 ? p - HF : 0;  // the plane finalized at the end of this iteration
    const bool kin = kf >= k0 && kf < k1;
    T ef[RY];
#pragma unroll
    for (int r = 0; r < RY; ++r) {
      u2[r] = d12[r] = xc[r] = T(0);
      ef[r] = (COMP && active[r] && kin) ? P.err[v][i + (long long)P.nx * (jr[r] + (long long)P.ny * kf)] : T(0);
    }
    if (p >= plo && p <= phi) {
      const int rel = p - plo;
      const bool ok = mbar_wait(&bar[rel % NSF], (unsigned)((rel / NSF) & 1), P.wait_ns);
      if (__syncthreads_or(!ok)) {
        if (tid == 0) {
          atomicExch(P.errflag, 1);
          // every copy still in flight, the one whose wait gave up included
          for (int w = p; w < next_issue; ++w) mbar_wait(&bar[(w - plo) % NSF], (unsigned)(((w - plo) / NSF) & 1));
        }
        return;
      }
      const T* box = ring + (rel % NSF) * FBP;
      // F_xi on the thread's own rows (kept in registers) and on its share of the eta halo rows
      T d1[RY], u1c[RY];
#pragma unroll
      for (int r = 0; r < RY; ++r) {
        const T* fc = box + (ty + TY * r + HF) * BX + tx + HX;
        xc[r] = fc[0];
        T d = T(0);
#pragma unroll
        for (int o = -HF; o <= HF; ++o) d += wx[o + HF] * fc[o];
        d1[r] = d;
        u1c[r] = COMP ? xc[r] + d : d;
        u1[(ty + TY * r + HF) * TX + tx] = u1c[r];
      }
      for (int rr = ty; rr < 2 * HF; rr += TY) {
        const int row = rr < HF ? rr : rr + TYE;
        const T* f = box + row * BX + tx + HX;
        T d = T(0);
#pragma unroll
        for (int o = -HF; o <= HF; ++o) d += wx[o + HF] * f[o];
        u1[row * TX + tx] = COMP ? f[0] + d : d;
      }
      __syncthreads();
      // the box is free for the plane NSF ahead; u1 is next written after the next wait barrier
      if (tid == 0) issue_upto(p + NSF);
#pragma unroll
      for (int r = 0; r < RY; ++r) {
        T dy = T(0);
#pragma unroll
        for (int o = -HF; o <= HF; ++o)
          dy += wy[r][o + HF] * (o == 0 ? u1c[r] : u1[(ty + TY * r + HF + o) * TX + tx]);
        if (COMP) {
          u2[r] = u1c[r] + dy;
          d12[r] = d1[r] + dy;
        } else {
          u2[r] = dy;
        }
      }
    }
    const int k = kf;
    int cz = 0;
    if (DIM == 3 && kin) cz = cls_of(k, P.nz, P.nb);
#pragma unroll
    for (int r = 0; r < RY; ++r) {
#pragma unroll
      for (int q = 0; q < NQ - 1; ++q) uq[r][q] = uq[r][q + 1];
      uq[r][NQ - 1] = u2[r];
#pragma unroll
      for (int q = 0; q < HF; ++q) {
        dq[r][q] = dq[r][q + 1];
        xq[r][q] = xq[r][q + 1];
      }
      dq[r][HF] = d12[r];
      xq[r][HF] = xc[r];
      if (!(active[r] && kin)) continue;
      T fz, x0, dsum;
      if (DIM == 3) {
        fz = T(0);
        if (cz == 0) {
          // interior plane: the loop-invariant interior weights
#pragma unroll
          for (int o = 0; o < NQ; ++o) fz += P.w[0][o] * uq[r][o];
        } else {
#pragma unroll
          for (int o = 0; o < NQ; ++o) fz += P.w[cz][o] * uq[r][o];
        }
        x0 = xq[r][0];
        dsum = dq[r][0];
      } else {
        fz = u2[r];
        x0 = xc[r];
        dsum = d12[r];
      }
      const long long l = i + (long long)P.nx * (jr[r] + (long long)P.ny * k);
      if (!COMP) {
        P.out[v][l] = (T(1) - P.blend) * x0 + P.blend * fz;
      } else {
        const T D = DIM == 3 ? dsum + fz : dsum;
        const T t = P.blend * D + ef[r];
        const T sm = x0 + t;
        const T bb = sm - x0;
        P.out[v][l] = sm;
        P.comp[v][l] = (x0 - (sm - bb)) + (t - bb);
      }
    }
  }
}

template <typename T, int DIM, bool COMP>
size_t stage_smem() {
  constexpr int NS = DIM == 3 ? 2 * kFdHalf + 1 + StagePrefetch<T>::P : 1;
  return sizeof(T) * NS * (DIM + 2) * Box<T, kFdHalf>::FBP + NS * sizeof(uint64_t);
}

template <typename T, int HF, int RY, int NB = 1>
size_t filter_smem() {
  return sizeof(T) * (kFilterSlots * NB * Box<T, HF, RY>::FBP + Box<T, HF, RY>::BY * kTileX) +
         kFilterSlots * sizeof(uint64_t);
}

template <typename T, int DIM, bool COMP, int TR>
cudaError_t go_stage(const FieldMaps& z, const TmaStageParams<T>& p, int tiles, int chunks, cudaStream_t s) {
  static bool attr = false;
  const size_t sm = stage_smem<T, DIM, COMP>();
  if (!attr) {
    cudaError_t e =
        cudaFuncSetAttribute(k_stage_tma<T, DIM, COMP, TR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  k_stage_tma<T, DIM, COMP, TR><<<dim3(tiles, chunks), 256, sm, s>>>(z, p);
  return cudaGetLastError();
}

// Traits are a run-time choice of the host (kTr* and the stage kind) mapped onto instantiations.
template <typename T, int DIM, bool COMP, int KIND>
cudaError_t go_stage_layout(const FieldMaps& z, const TmaStageParams<T>& p, int tr, int tiles, int chunks,
                            cudaStream_t s) {
  constexpr int B = kTrTma | (KIND << kKindShift);
  switch (tr & 7) {
    case 0: return go_stage<T, DIM, COMP, B | 0>(z, p, tiles, chunks, s);
    case 1: return go_stage<T, DIM, COMP, B | 1>(z, p, tiles, chunks, s);
    case 2: return go_stage<T, DIM, COMP, B | 2>(z, p, tiles, chunks, s);
    case 3: return go_stage<T, DIM, COMP, B | 3>(z, p, tiles, chunks, s);
    case 4: return go_stage<T, DIM, COMP, B | 4>(z, p, tiles, chunks, s);
    case 5: return go_stage<T, DIM, COMP, B | 5>(z, p, tiles, chunks, s);
    case 6: return go_stage<T, DIM, COMP, B | 6>(z, p, tiles, chunks, s);
    default: return go_stage<T, DIM, COMP, B | 7>(z, p, tiles, chunks, s);
  }
}

template <typename T, int DIM, bool COMP>
cudaError_t go_stage_tr(const FieldMaps& z, const TmaStageParams<T>& p, int tr, int tiles, int chunks,
                        cudaStream_t s) {
  switch ((tr >> kKindShift) & 7) {
    case kKindRhs: return go_stage_layout<T, DIM, COMP, kKindRhs>(z, p, tr, tiles, chunks, s);
    case kKindFirst: return go_stage_layout<T, DIM, COMP, kKindFirst>(z, p, tr, tiles, chunks, s);
    case kKindMid: return go_stage_layout<T, DIM, COMP, kKindMid>(z, p, tr, tiles, chunks, s);
    case kKindLast: return go_stage_layout<T, DIM, COMP, kKindLast>(z, p, tr, tiles, chunks, s);
    case kKindLastIncrement:
      if constexpr (COMP) return go_stage_layout<T, DIM, COMP, kKindLastIncrement>(z, p, tr, tiles, chunks, s);
      return cudaErrorInvalidValue;
    default: return go_stage_layout<T, DIM, COMP, kKindRuntime>(z, p, tr, tiles, chunks, s);
  }
}

template <typename T, int DIM, bool COMP, int HF>
cudaError_t go_filter(const FieldMaps& in, const TmaFilterParams<T>& p, int ry, int tiles, int chunks, cudaStream_t s) {
  if (p.code[0]) {
    // a block with holes: the one-row form with per-point classes and the hole mask
    if (ry != 1 || !p.iblank) return cudaErrorInvalidValue;
    k_filter_tma_row<T, DIM, COMP, HF, false, true><<<dim3(tiles, chunks, p.V), 256, filter_smem<T, HF, 1>(), s>>>(
        in, in, p);
  } else if (ry == 2) {
    k_filter_tma<T, DIM, COMP, HF, 2><<<dim3(tiles, chunks, p.V), 256, filter_smem<T, HF, 2>(), s>>>(in, p);
  } else {
    k_filter_tma_row<T, DIM, COMP, HF><<<dim3(tiles, chunks, p.V), 256, filter_smem<T, HF, 1>(), s>>>(in, in, p);
  }
  return cudaGetLastError();
}

}  // namespace

size_t stage_tma_smem(int dim, size_t esz) {
  if (esz == 8) return dim == 3 ? stage_smem<double, 3, false>() : stage_smem<double, 2, false>();
  return dim == 3 ? stage_smem<float, 3, true>() : stage_smem<float, 2, true>();
}

// The FP64 form runs uncompensated and the FP32 form compensated (lee_config.precision).
template <typename T>
cudaError_t launch_stage_tma(const FieldMaps& zin, const TmaStageParams<T>& p, int traits, int tiles, int chunks,
                             cudaStream_t s) {
  constexpr bool COMP = sizeof(T) == 4;
  if (p.s.dim == 2) return go_stage_tr<T, 2, COMP>(zin, p, traits, tiles, 1, s);
  return go_stage_tr<T, 3, COMP>(zin, p, traits, tiles, chunks, s);
}

template <typename T>
cudaError_t launch_filter_tma(const FieldMaps& in, const TmaFilterParams<T>& p, int hf, int dim, int comp, int ry,
                              int tiles, int chunks, cudaStream_t s) {
  if (ry != 1 && ry != 2) return cudaErrorInvalidValue;
#define LEE_FILTER_CASE(HF)                                                                      \
  if (hf == HF) {                                                                                \
    if (dim == 2)                                                                                \
      return comp ? go_filter<T, 2, true, HF>(in, p, ry, tiles, 1, s)                            \
                  : go_filter<T, 2, false, HF>(in, p, ry, tiles, 1, s);                          \
    return comp ? go_filter<T, 3, true, HF>(in, p, ry, tiles, chunks, s)                         \
                : go_filter<T, 3, false, HF>(in, p, ry, tiles, chunks, s);                       \
  }
  LEE_FILTER_CASE(2)
  LEE_FILTER_CASE(4)
  LEE_FILTER_CASE(5)
#undef LEE_FILTER_CASE
  return cudaErrorInvalidValue;
}

// The compensated one-row filter whose input is y_n and the last stage's increment.
cudaError_t launch_filter_tma_inc(const FieldMaps& y, const FieldMaps& inc, const TmaFilterParams<float>& p, int hf,
                                  int dim, int tiles, int chunks, cudaStream_t s) {
#define LEE_FILTER_INC(HF)                                                                                   \
  if (hf == HF) {                                                                                            \
    if (dim == 2)                                                                                            \
      k_filter_tma_row<float, 2, true, HF, true><<<dim3(tiles, 1, p.V), 256, filter_smem<float, HF, 1, 2>(), s>>>( \
          y, inc, p);                                                                                        \
    else                                                                                                     \
      k_filter_tma_row<float, 3, true, HF, true><<<dim3(tiles, chunks, p.V), 256, filter_smem<float, HF, 1, 2>(), \
                                                   s>>>(y, inc, p);                                          \
    return cudaGetLastError();                                                                               \
  }
  LEE_FILTER_INC(2)
  LEE_FILTER_INC(4)
  LEE_FILTER_INC(5)
#undef LEE_FILTER_INC
  return cudaErrorInvalidValue;
}

template cudaError_t launch_stage_tma<double>(const FieldMaps&, const TmaStageParams<double>&, int, int, int, cudaStream_t);
template cudaError_t launch_stage_tma<float>(const FieldMaps&, const TmaStageParams<float>&, int, int, int, cudaStream_t);
template cudaError_t launch_filter_tma<double>(const FieldMaps&, const TmaFilterParams<double>&, int, int, int, int, int, int,
                                               cudaStream_t);
template cudaError_t launch_filter_tma<float>(const FieldMaps&, const TmaFilterParams<float>&, int, int, int, int, int, int,
                                              cudaStream_t);

}  // namespace lee
