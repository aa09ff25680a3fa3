// Fused three-direction filter, vectorised along xi (sm_100a).
//
// spatial::apply_filter (src/solver/spatial_discretization.cpp:2191-2246) applies the filter
// line by line in xi, then eta, then zeta. This kernel does the three passes in one read of the
// pre-filter state and one write of the filtered state, as the scalar fused kernel does, but
// every thread owns a group of 16 bytes of consecutive points along xi (4 floats or 2 doubles):
// shared-memory traffic moves in 16-byte words, and FP32 arithmetic runs as packed pairs
// (__ffma2_rn and friends), which halves the instructions that the scalar form issues.
//
// A CTA owns a tile of TX = 32 groups along xi by 8 rows along eta and marches along zeta
// through a chunk of planes. Per incoming plane (one TMA box: tile plus halos):
//   A. F_xi on the tile's rows and the eta halo rows, each row done by one warp; interior
//      points use the symmetric interior stencil in registers, and the few lanes that hold a
//      block's xi closure points redo those points with their closure rows;
//   B. F_eta at the tile's rows, from the F_xi results in shared memory;
//   C. F_zeta from a register queue of the last 2h+1 planes (the plane loop is unrolled by
//      2h+1 so that the queue never moves), finishing the plane h behind the incoming one.
// The compensated form (FP32) carries the filter's increments, F - I, through the passes and
// adds blend * increment to the pre-filter value and its carried rounding error as an exact
// two-float sum, as the scalar kernels do.
//
// Every mbarrier wait is bounded (about one second); on expiry the CTA records the failure in
// the device flag, waits (bounded) for its own copies in flight and returns.
#include <type_traits>
#include <utility>

#include "lee_tma.h"
#include "lee_tma_util.cuh"

namespace lee {
namespace {

// Tile and shared-memory geometry of the vectorised filter for element type T, half-width HF and
// PX points per thread.
template <typename T, int DIM, bool COMP, int HF, int PX_>
struct FGeo {
  static constexpr int PX = PX_;                       // points per thread along xi
  static constexpr int LX = 32;                        // threads per row (one warp)
  static constexpr int TX = PX * LX;                   // tile width
  static constexpr int TY = 8;                         // tile rows (one per warp)
  static constexpr int NQ = 2 * HF + 1;                // stencil width
  static constexpr int A = (int)(16 / sizeof(T));      // elements in 16 bytes
  static constexpr int HXV = ((HF + A - 1) / A) * A;   // xi halo of the box: TMA starts on 16 bytes
  static constexpr int HXW = ((HF + PX - 1) / PX) * PX;  // xi halo of a thread's row window
  static constexpr int BX = TX + 2 * HXV;
  static constexpr int BY = TY + 2 * HF;
  static constexpr int FB = BX * BY;
  static constexpr int FBP = (int)((((size_t)FB * sizeof(T) + 127) / 128) * 128 / sizeof(T));
  static constexpr int PF = HF <= 4 ? 3 : 2;                        // planes of prefetch
  static constexpr int NSF = DIM == 3 ? HF + 1 + PF : 1;            // TMA ring slots
  static constexpr int ND = COMP ? (DIM == 3 ? HF + 2 : 1) : 0;     // increment ring planes
  static constexpr int NWG = (2 * HXW + PX) / PX;                   // groups in a row window
  // shared memory, in elements of T: ring | u1 (2 buffers) | increments | mbarriers
  static constexpr int OFF_U1 = NSF * FBP;
  static constexpr int OFF_D = OFF_U1 + 2 * BY * TX;
  static constexpr int OFF_BAR = OFF_D + ND * TY * TX;
  static constexpr size_t BYTES = (size_t)OFF_BAR * sizeof(T) + NSF * sizeof(uint64_t);
  static_assert((FBP * sizeof(T)) % 128 == 0, "box stride must be a multiple of 128 bytes");
  static_assert((OFF_BAR * sizeof(T)) % 8 == 0, "mbarriers need 8-byte alignment");
  static_assert(BX <= 256 && BY <= 256, "TMA box dimensions are at most 256");
  static_assert(HXV % PX == 0 && HXW <= HXV, "a row window lies inside the box row");
};

// A thread's group of PX points and the arithmetic on it: FP32 as packed pairs, FP64 as scalars.
// W is a weight broadcast to the group.
template <typename T, int PX>
struct Grp;

template <int PX>
struct Grp<float, PX> {
  static constexpr int NP = PX / 2;
  static_assert(PX == 2 || PX == 4, "FP32 groups hold 2 or 4 points");
  float2 p[NP];
  using W = float2;
  __device__ __forceinline__ static W w(float x) { return make_float2(x, x); }
  __device__ __forceinline__ static Grp zero() {
    Grp g;
#pragma unroll
    for (int h = 0; h < NP; ++h) g.p[h] = make_float2(0.f, 0.f);
    return g;
  }
  __device__ __forceinline__ static Grp load(const float* q) {
    Grp g;
    if constexpr (NP == 2) {
      const float4 v = *reinterpret_cast<const float4*>(q);
      g.p[0] = make_float2(v.x, v.y);
      g.p[1] = make_float2(v.z, v.w);
    } else {
      g.p[0] = *reinterpret_cast<const float2*>(q);
    }
    return g;
  }
  __device__ __forceinline__ void store(float* q) const {
    if constexpr (NP == 2)
      *reinterpret_cast<float4*>(q) = make_float4(p[0].x, p[0].y, p[1].x, p[1].y);
    else
      *reinterpret_cast<float2*>(q) = p[0];
  }
  __device__ __forceinline__ float get(int q) const { return (q & 1) ? p[q >> 1].y : p[q >> 1].x; }
  __device__ __forceinline__ static Grp of(const float (&e)[PX]) {
    Grp g;
#pragma unroll
    for (int h = 0; h < NP; ++h) g.p[h] = make_float2(e[2 * h], e[2 * h + 1]);
    return g;
  }
  __device__ __forceinline__ friend Grp operator+(Grp x, Grp y) {
#pragma unroll
    for (int h = 0; h < NP; ++h) x.p[h] = __fadd2_rn(x.p[h], y.p[h]);
    return x;
  }
  // x - y, exactly (one rounding)
  __device__ __forceinline__ friend Grp operator-(Grp x, Grp y) {
#pragma unroll
    for (int h = 0; h < NP; ++h) x.p[h] = __ffma2_rn(y.p[h], make_float2(-1.f, -1.f), x.p[h]);
    return x;
  }
  __device__ __forceinline__ friend Grp operator*(Grp x, W w) {
#pragma unroll
    for (int h = 0; h < NP; ++h) x.p[h] = __fmul2_rn(x.p[h], w);
    return x;
  }
  // x * w + c
  __device__ __forceinline__ static Grp fma(Grp x, W w, Grp c) {
#pragma unroll
    for (int h = 0; h < NP; ++h) c.p[h] = __ffma2_rn(x.p[h], w, c.p[h]);
    return c;
  }
};

template <>
struct Grp<double, 2> {
  double a, b;
  using W = double;
  __device__ __forceinline__ static W w(double x) { return x; }
  __device__ __forceinline__ static Grp zero() { return {0.0, 0.0}; }
  __device__ __forceinline__ static Grp load(const double* p) {
    const double2 v = *reinterpret_cast<const double2*>(p);
    return {v.x, v.y};
  }
  __device__ __forceinline__ void store(double* p) const { *reinterpret_cast<double2*>(p) = make_double2(a, b); }
  __device__ __forceinline__ double get(int q) const { return q == 0 ? a : b; }
  __device__ __forceinline__ static Grp of(const double (&e)[2]) { return {e[0], e[1]}; }
  __device__ __forceinline__ friend Grp operator+(Grp x, Grp y) { return {x.a + y.a, x.b + y.b}; }
  __device__ __forceinline__ friend Grp operator-(Grp x, Grp y) { return {x.a - y.a, x.b - y.b}; }
  __device__ __forceinline__ friend Grp operator*(Grp x, W w) { return {x.a * w, x.b * w}; }
  __device__ __forceinline__ static Grp fma(Grp x, W w, Grp c) { return {__fma_rn(x.a, w, c.a), __fma_rn(x.b, w, c.b)}; }
};


// The symmetric interior stencil along xi for the group whose points sit at win[C .. C+PX-1] of a
// row window: w0 x_c + sum_o w_o (x_{c-o} + x_{c+o}). FP32 pairs neighbouring points where the
// taps line up with register pairs (even o) and goes scalar for odd o.
template <int HF, int C, int PX, int NW>
__device__ __forceinline__ Grp<float, PX> xi_interior(const float (&win)[NW], const float2 (&wi)[HF + 1]) {
  Grp<float, PX> g;
#pragma unroll
  for (int h = 0; h < PX / 2; ++h) {
    const int c = C + 2 * h;
    float2 a = __fmul2_rn(make_float2(win[c], win[c + 1]), wi[0]);
#pragma unroll
    for (int o = 1; o <= HF; ++o) {
      if ((o & 1) == 0) {
        const float2 sum = __fadd2_rn(make_float2(win[c - o], win[c - o + 1]), make_float2(win[c + o], win[c + o + 1]));
        a = __ffma2_rn(sum, wi[o], a);
      } else {
        a.x = fmaf(win[c - o] + win[c + o], wi[o].x, a.x);
        a.y = fmaf(win[c + 1 - o] + win[c + 1 + o], wi[o].x, a.y);
      }
    }
    g.p[h] = a;
  }
  return g;
}

template <int HF, int C, int PX, int NW>
__device__ __forceinline__ Grp<double, 2> xi_interior(const double (&win)[NW], const double (&wi)[HF + 1]) {
  double d[2];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int c = C + q;
    double a = win[c] * wi[0];
#pragma unroll
    for (int o = 1; o <= HF; ++o) a = __fma_rn(win[c - o] + win[c + o], wi[o], a);
    d[q] = a;
  }
  return {d[0], d[1]};
}

template <typename T, int DIM, bool COMP, int HF, int PX>
__global__ void __launch_bounds__(256, PX * sizeof(T) == 16 ? 2 : 3)
    k_filter_vec(const __grid_constant__ FieldMaps ym, const __grid_constant__ TmaFilterParams<T> P) {
  using G = FGeo<T, DIM, COMP, HF, PX>;
  using V = Grp<T, PX>;
  using W = typename V::W;
  constexpr int TX = G::TX, TY = G::TY, NQ = G::NQ, HXV = G::HXV, HXW = G::HXW, BX = G::BX;
  constexpr int NSF = G::NSF, FBP = G::FBP;
  extern __shared__ __align__(128) unsigned char smem[];
  T* ring = reinterpret_cast<T*>(smem);
  T* u1s = ring + G::OFF_U1;   // [2][BY][TX]
  T* dsm = ring + G::OFF_D;    // [ND][TY][TX]: F_xi increments, then F_xi + F_eta increments
  uint64_t* bar = reinterpret_cast<uint64_t*>(ring + G::OFF_BAR);

  const int v = blockIdx.z;
  const int i0 = (int)(blockIdx.x % P.tiles_x) * TX, j0 = (int)(blockIdx.x / P.tiles_x) * TY;
  const int k0 = DIM == 3 ? (int)blockIdx.y * P.k_chunk : 0;
  const int k1 = DIM == 3 ? min(P.nz, k0 + P.k_chunk) : 1;
  const int tid = threadIdx.x, lane = tid & 31, wy_row = tid >> 5;
  const int gc = lane * PX;  // first column of the thread's group, in the tile
  const int i = i0 + gc, j = j0 + wy_row;
  const int plo = DIM == 3 ? max(0, k0 - HF) : 0;
  const int phi = DIM == 3 ? min(P.nz - 1, k1 - 1 + HF) : 0;

  if (tid == 0) {
    for (int q = 0; q < NSF; ++q) mbar_init(&bar[q], 1);
    fence_mbar_init();
  }
  __syncthreads();
  int next_issue = plo;  // meaningful in thread 0 only
  auto issue_upto = [&](int last) {
    for (; next_issue <= min(phi, last); ++next_issue) {
      const int slot = (next_issue - plo) % NSF;
      mbar_expect_tx(&bar[slot], (unsigned)(sizeof(T) * G::FB));
      tma_load_3d(ring + slot * FBP, &ym.m[v], i0 - HXV, j0 - HF, next_issue, &bar[slot]);
    }
  };
  if (tid == 0) issue_upto(plo + NSF - 1);

  // the symmetric interior stencil (F - I in the compensated form), shared by the directions
  W wi[HF + 1];
#pragma unroll
  for (int o = 0; o <= HF; ++o) wi[o] = V::w(P.w[0][HF + o]);
  const int cy = cls_of(min(j, P.ny - 1), P.ny, HF);
  const bool vec_io = (P.nx % PX) == 0;  // global groups are 16-byte aligned
  // xi closure points: the owner of a group skips them (cmask, bit q for point i + q), and after
  // the group stores each warp's lanes compute the closure points of the warp's rows, lane L
  // taking row task L / (2 HF) and closure point L % (2 HF) (left end first)
  constexpr int NR = (G::BY + TY - 1) / TY;  // row tasks of a warp
  unsigned cmask = 0;
#pragma unroll
  for (int q = 0; q < PX; ++q) {
    const int g = i + q;
    if (g < P.nx && (g < HF || g > P.nx - 1 - HF)) cmask |= 1u << q;
  }
  int fix_r = -1, fix_g = -1;  // this lane's closure point: row task and column
  {
    const int t = lane / (2 * HF), m = lane % (2 * HF);
    const int g = m < HF ? m : P.nx - HF + (m - HF);
    if (t < NR && wy_row + t * TY < G::BY && g >= i0 && g < i0 + TX) {
      fix_r = wy_row + t * TY;
      fix_g = g;
    }
  }

  // F_xi of the warp's box rows (r = wy_row + t TY): u1 into u1b, and for the tile's own rows the
  // increment into db
  auto xi_rows = [&](const T* box, T* u1b, T* db) {
    // row windows loaded in batches of NB rows before their arithmetic (NB = 1 where the
    // 11-point stencil's queue leaves no registers for more)
    constexpr int NB = HF >= 5 ? 1 : NR;
#pragma unroll
    for (int t0 = 0; t0 < NR; t0 += NB) {
      T win[NB][G::NWG * PX];
#pragma unroll
      for (int t = 0; t < NB; ++t) {
        const int r = wy_row + (t0 + t) * TY;
        if (t0 + t < NR && r < G::BY) {
#pragma unroll
          for (int g = 0; g < G::NWG; ++g) {
            const V x = V::load(box + r * BX + (HXV - HXW) + gc + g * PX);
#pragma unroll
            for (int q = 0; q < PX; ++q) win[t][g * PX + q] = x.get(q);
          }
        }
      }
#pragma unroll
      for (int t = 0; t < NB; ++t) {
        const int r = wy_row + (t0 + t) * TY;
        if (t0 + t >= NR || r >= G::BY) break;
        const bool own = COMP && r >= HF && r < HF + TY;
        const V dv = xi_interior<HF, HXW, PX>(win[t], wi);
        const V u1 = COMP ? V::of(*reinterpret_cast<const T(*)[PX]>(win[t] + HXW)) + dv : dv;
        if (cmask == 0) {
          u1.store(u1b + r * TX + gc);
          if (own) dv.store(db + (r - HF) * TX + gc);
        } else {
#pragma unroll
          for (int q = 0; q < PX; ++q)
            if (!((cmask >> q) & 1u)) {
              u1b[r * TX + gc + q] = u1.get(q);
              if (own) db[(r - HF) * TX + gc + q] = dv.get(q);
            }
        }
      }
    }
    if (fix_g >= 0) {
      // a closure point: its own weights, read by class
      const int cls = cls_of(fix_g, P.nx, HF);
      const T* cen = box + fix_r * BX + HXV + (fix_g - i0);
      T acc = T(0);
#pragma unroll
      for (int o = -HF; o <= HF; ++o) acc = fma(cen[o], P.w[cls][HF + o], acc);
      u1b[fix_r * TX + (fix_g - i0)] = COMP ? cen[0] + acc : acc;
      if (COMP && fix_r >= HF && fix_r < HF + TY) db[(fix_r - HF) * TX + (fix_g - i0)] = acc;
    }
  };

  V uq[NQ];
#pragma unroll
  for (int q = 0; q < NQ; ++q) uq[q] = V::zero();
  const int pstart = DIM == 3 ? k0 - HF : 0, pend = DIM == 3 ? k1 - 1 + HF : 0;
  int slot = (pstart - plo) % NSF;  // ring slot of plane p (planes below plo never load)
  if (slot < 0) slot += NSF;
  int dslot = 0;                    // increment ring plane of plane p
  bool stop = false;

  // one plane p; R = (p - pstart) % NQ names the queue entry that receives it
  auto plane = [&](int p, auto Rc) {
    constexpr int R = decltype(Rc)::value;
    const bool in_blk = p >= plo && p <= phi;
    // the finishing plane's point offset, and (compensated) its carried rounding error, loaded
    // before this plane's work so that the load's latency overlaps it
    const int kf = DIM == 3 ? p - HF : 0;
    const bool fin = kf >= k0 && kf < k1 && j < P.ny && i < P.nx;
    const unsigned long long l = (unsigned long long)i + (unsigned long long)P.nx * (j + (unsigned long long)P.ny * kf);
    const bool whole = vec_io && i + PX <= P.nx;
    V ef = V::zero();
    if (COMP && fin) {
      if (whole) {
        ef = V::load(P.err[v] + l);
      } else {
        T e[PX];
#pragma unroll
        for (int q = 0; q < PX; ++q) e[q] = i + q < P.nx ? P.err[v][l + q] : T(0);
        ef = V::of(e);
      }
    }
    const int buf = p & 1;
    T* u1b = u1s + buf * (G::BY * TX);
    T* db = COMP ? dsm + dslot * (TY * TX) : nullptr;
    const T* box = ring + slot * FBP;
    bool failed = false;
    if (in_blk) {
      const int rel = p - plo;
      failed = !mbar_wait(&bar[rel % NSF], (unsigned)((rel / NSF) & 1), P.wait_ns);
      // A: F_xi on the own rows (r = HF + wy_row) and the eta halo rows
      xi_rows(box, u1b, db);
    }
    if (__syncthreads_or(failed)) {
      if (tid == 0) {
        atomicExch(P.errflag, 1);
        for (int w = p; w < next_issue; ++w) mbar_wait(&bar[(w - plo) % NSF], (unsigned)(((w - plo) / NSF) & 1));
      }
      stop = true;
      return;
    }
    if (DIM == 3 && tid == 0) issue_upto(p + G::PF);
    // B: F_eta at the own row
    V u2 = V::zero();
    if (in_blk) {
      const T* col = u1b + gc;
      V dy = V::zero(), u1c = V::load(col + (HF + wy_row) * TX);
      if (cy == 0) {
        dy = u1c * wi[0];
#pragma unroll
        for (int o = 1; o <= HF; ++o)
          dy = V::fma(V::load(col + (HF + wy_row - o) * TX) + V::load(col + (HF + wy_row + o) * TX), wi[o], dy);
      } else {
#pragma unroll
        for (int o = -HF; o <= HF; ++o) dy = V::fma(V::load(col + (HF + wy_row + o) * TX), V::w(P.w[cy][HF + o]), dy);
      }
      if (COMP) {
        u2 = u1c + dy;
        T* dp = db + wy_row * TX + gc;
        (V::load(dp) + dy).store(dp);
      } else {
        u2 = dy;
      }
    }
    uq[R] = u2;
    // C: F_zeta and the blend for plane kf = p - HF
    if (fin) {
      V fz;
      if (DIM == 3) {
        const int cz = cls_of(kf, P.nz, HF);
        if (cz == 0) {
          fz = uq[(R + 1 + HF) % NQ] * wi[0];
#pragma unroll
          for (int o = 1; o <= HF; ++o) fz = V::fma(uq[(R + 1 + HF - o) % NQ] + uq[(R + 1 + HF + o) % NQ], wi[o], fz);
        } else {
          fz = V::zero();
#pragma unroll
          for (int o = 0; o < NQ; ++o) fz = V::fma(uq[(R + 1 + o) % NQ], V::w(P.w[cz][o]), fz);
        }
      } else {
        fz = u2;
      }
      // the pre-filter value: the plane's box is still in the ring (HF planes back)
      int fslot = slot - (DIM == 3 ? HF : 0);
      fslot += fslot < 0 ? NSF : 0;
      const V x0 = V::load(ring + fslot * FBP + (HF + wy_row) * BX + HXV + gc);
      if (!COMP) {
        const V out = V::fma(x0, V::w(T(1) - P.blend), fz * V::w(P.blend));
        if (whole) {
          out.store(P.out[v] + l);
        } else {
          for (int q = 0; q < PX && i + q < P.nx; ++q) P.out[v][l + q] = out.get(q);
        }
      } else {
        int ds = dslot - (DIM == 3 ? HF : 0);
        ds += ds < 0 ? G::ND : 0;
        const V dsum = V::load(dsm + ds * (TY * TX) + wy_row * TX + gc);
        const V D = DIM == 3 ? dsum + fz : dsum;
        const V t = V::fma(D, V::w(P.blend), ef);
        const V sm = x0 + t;
        const V bb = sm - x0;
        const V cm = (x0 - (sm - bb)) + (t - bb);
        if (whole) {
          sm.store(P.out[v] + l);
          cm.store(P.comp[v] + l);
        } else {
          for (int q = 0; q < PX && i + q < P.nx; ++q) {
            P.out[v][l + q] = sm.get(q);
            P.comp[v][l + q] = cm.get(q);
          }
        }
      }
    }
    slot = slot + 1 == NSF ? 0 : slot + 1;
    if (COMP) dslot = dslot + 1 == G::ND ? 0 : dslot + 1;
  };

  if (DIM == 2) {
    plane(0, std::integral_constant<int, 0>{});
  } else {
    for (int p0 = pstart; p0 <= pend && !stop; p0 += NQ) {
      static_for<NQ>([&](auto Rc) {
        constexpr int R = decltype(Rc)::value;
        if (!stop && p0 + R <= pend) plane(p0 + R, Rc);
      });
    }
  }
}

template <typename T, int DIM, bool COMP, int HF, int PX>
cudaError_t go_filter_vec(const FieldMaps& in, const TmaFilterParams<T>& p, int tiles, int chunks, cudaStream_t s) {
  using G = FGeo<T, DIM, COMP, HF, PX>;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k_filter_vec<T, DIM, COMP, HF, PX>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::BYTES);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  k_filter_vec<T, DIM, COMP, HF, PX><<<dim3(tiles, chunks, p.V), 256, G::BYTES, s>>>(in, p);
  return cudaGetLastError();
}

template <typename T, int PX>
cudaError_t go_filter_px(const FieldMaps& in, const TmaFilterParams<T>& p, int hf, int dim, int tiles, int chunks,
                         cudaStream_t s) {
  constexpr bool COMP = sizeof(T) == 4;
#define LEE_FILTER_VEC(HF)                                                                         \
  if (hf == HF)                                                                                    \
    return dim == 2 ? go_filter_vec<T, 2, COMP, HF, PX>(in, p, tiles, 1, s)                        \
                    : go_filter_vec<T, 3, COMP, HF, PX>(in, p, tiles, chunks, s);
  LEE_FILTER_VEC(2)
  LEE_FILTER_VEC(4)
  LEE_FILTER_VEC(5)
#undef LEE_FILTER_VEC
  return cudaErrorInvalidValue;
}

}  // namespace

int filter_vec_widths(size_t esz, int* px) {
  if (esz == 4) {
    px[0] = 4;
    px[1] = 2;
    return 2;
  }
  px[0] = 2;
  return 1;
}

void filter_vec_box(size_t esz, int hf, int px, int* bx, int* by, int* tx, int* ty) {
  const int a = (int)(16 / esz);
  const int hxv = ((hf + a - 1) / a) * a;
  *tx = 32 * px;
  *ty = 8;
  *bx = *tx + 2 * hxv;
  *by = *ty + 2 * hf;
}

template <typename T>
cudaError_t launch_filter_vec(const FieldMaps& in, const TmaFilterParams<T>& p, int hf, int px, int dim, int tiles,
                              int chunks, cudaStream_t s) {
  if constexpr (sizeof(T) == 4) {
    if (px == 4) return go_filter_px<T, 4>(in, p, hf, dim, tiles, chunks, s);
  }
  if (px == 2) return go_filter_px<T, 2>(in, p, hf, dim, tiles, chunks, s);
  return cudaErrorInvalidValue;
}

template cudaError_t launch_filter_vec<float>(const FieldMaps&, const TmaFilterParams<float>&, int, int, int, int, int,
                                              cudaStream_t);
template cudaError_t launch_filter_vec<double>(const FieldMaps&, const TmaFilterParams<double>&, int, int, int, int,
                                               int, cudaStream_t);

}  // namespace lee
