// Fused three-direction filter of the compensated FP32 form, two points per thread (sm_100a).
//
// spatial::apply_filter (src/solver/spatial_discretization.cpp:2191-2246) filters line by line in
// xi, then eta, then zeta, and the blend with the pre-filter state follows. This kernel fuses the
// three passes as k_filter_tma_row (lee_tma.cu) does, with each point's arithmetic in the same
// order (the same bits), but every thread owns two neighbouring points along xi:
//   - the pair's xi taps come from 8-byte shared-memory words, and the xi taps whose two values
//     lie in one word run as packed FP32 instructions (__ffma2_rn, with the pair's two weights
//     held in a register pair), as do the sums of pairs (__fadd2_rn);
//   - the per-plane work (the wait on the plane's copy, the barrier, addressing) is shared by the
//     two points, and the output moves in 8-byte words.
//
// A CTA owns 64 x 8 points in (i, j) and marches along k through a chunk of planes. Per incoming
// plane p (one TMA box: the tile plus its halos, in a ring of h + 4 slots):
//   xi:   F_xi - I at the thread's own row and at one eta halo row, from the box, into one of two
//         shared row buffers (u1, alternating by plane, so one barrier per plane suffices);
//   eta:  F_eta - I at the own row, from u1;
//   zeta: a register queue of the last 2h + 1 planes' F_eta F_xi values and a per-thread shared
//         ring of the last h + 1 planes' summed xi and eta increments finish plane p - h: F_zeta,
//         then the blend as the exact
//         two-float sum of the pre-filter value, blend * (sum of the increments) and the carried
//         rounding error. The pre-filter value comes from the ring, whose slot of plane p - h is
//         re-issued only after every thread has finished that plane.
// Each thread keeps its pair's xi weights (one closure class per point) in registers; rows near an
// eta end (one warp each) and planes near a zeta end take their class rows.
//
// Every mbarrier wait is bounded (about one second, or the context's limit); on expiry the CTA
// records the failure in the device flag, waits (bounded) for its own copies in flight and
// returns.
#include "lee_tma.h"
#include "lee_tma_util.cuh"

namespace lee {
namespace {

using F2 = float2;

__device__ __forceinline__ F2 add2(F2 a, F2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ F2 fma2(F2 a, F2 b, F2 c) { return __ffma2_rn(a, b, c); }
// w * a + c and a - b lane by lane (scalar instructions)
__device__ __forceinline__ F2 fmas(float w, F2 a, F2 c) { return make_float2(fmaf(w, a.x, c.x), fmaf(w, a.y, c.y)); }
__device__ __forceinline__ F2 subs(F2 a, F2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ F2 ld2(const float* p) { return *reinterpret_cast<const F2*>(p); }
__device__ __forceinline__ void st2(float* p, F2 v) { *reinterpret_cast<F2*>(p) = v; }

constexpr int kPairLX = 32;           // threads per tile row (one warp)
constexpr int kPairTX = 2 * kPairLX;  // points along i per CTA

// Geometry of the pair kernel for half-width HF.
template <int HF>
struct PairGeo {
  static constexpr int HX = ((HF + 3) / 4) * 4;  // xi halo of the box: every TMA row starts on 16 bytes
  static constexpr int BX = kPairTX + 2 * HX;
  static constexpr int BY = kTileY + 2 * HF;
  static constexpr int FB = BX * BY;
  static constexpr int FBP = ((FB * 4 + 127) / 128) * 128 / 4;  // box stride: 128-byte multiple
  static constexpr int PF = 3;                                   // planes of prefetch
  static constexpr int NS = HF + 1 + PF;                          // ring slots
  static constexpr int HP = (HF + 1) / 2;  // a pair's row window starts 2 HP points before it
  static constexpr int NW = 1 + 2 * HP;    // 8-byte words of the window
  static constexpr int U1 = BY * kPairTX;  // floats of one row buffer
  static constexpr int ND = HF + 1;        // planes of summed increments kept per point
  static constexpr int DP = kTileY * kPairTX;  // floats of one plane of them
  static constexpr size_t BYTES = ((size_t)NS * FBP + 2 * U1 + ND * DP) * 4 + NS * sizeof(uint64_t);
  static_assert(HX % 2 == 0 && BX % 2 == 0, "pairs start on 8 bytes");
  // the window of the last pair (column HX + kPairTX - 2) ends inside the box row
  static_assert(2 * HP <= HX && HX + kPairTX - 2 + 2 * HP + 1 < BX, "row window inside the box");
  static_assert(BX <= 256 && BY <= 256, "TMA box dimensions are at most 256");
  static_assert(((size_t)NS * FBP + 2 * U1 + ND * DP) * 4 % 8 == 0, "mbarriers need 8-byte alignment");
};

// COMP: the compensated form (the increments F - I, the carried rounding error in and out);
// otherwise the plain filter and blend (out = (1 - blend) x + blend F x, the adjoint's transposed
// filter, whose class rows are the transposed operator's).
template <int HF, bool COMP>
__global__ void __launch_bounds__(256, HF <= 4 ? 4 : 3) k_filter_pair(const __grid_constant__ FieldMaps ym,
                                                     const __grid_constant__ TmaFilterParams<float> P) {
  using G = PairGeo<HF>;
  constexpr int TY = kTileY, NQ = 2 * HF + 1, NS = G::NS, BX = G::BX, FBP = G::FBP, HP = G::HP, NW = G::NW;
  extern __shared__ __align__(128) unsigned char smem[];
  float* ring = reinterpret_cast<float*>(smem);
  float* u1s = ring + NS * FBP;  // [2][BY][kPairTX]
  // [ND][TY][kPairTX]: the summed xi and eta increments of the last h + 1 planes, each point's
  // own (written and read by its thread only)
  float* dsm = u1s + 2 * G::U1;
  uint64_t* bar = reinterpret_cast<uint64_t*>(dsm + G::ND * G::DP);

  const int v = blockIdx.z;
  const int i0 = (int)(blockIdx.x % P.tiles_x) * kPairTX, j0 = (int)(blockIdx.x / P.tiles_x) * TY;
  const int k0 = (int)blockIdx.y * P.k_chunk;
  const int k1 = min(P.nz, k0 + P.k_chunk);
  const int tid = threadIdx.x, tx = tid % kPairLX, ty = tid / kPairLX;
  const int i = i0 + 2 * tx, j = j0 + ty;
  const bool active = i < P.nx && j < P.ny;  // nx is even: both points of the pair or neither
  const int plo = max(0, k0 - HF), phi = min(P.nz - 1, k1 - 1 + HF);

  if (tid == 0) {
    for (int q = 0; q < NS; ++q) mbar_init(&bar[q], 1);
    fence_mbar_init();
  }
  __syncthreads();
  int next_issue = plo;  // meaningful in thread 0 only
  auto issue_upto = [&](int last) {
    for (; next_issue <= min(phi, last); ++next_issue) {
      const int slot = (next_issue - plo) % NS;
      mbar_expect_tx(&bar[slot], (unsigned)(sizeof(float) * G::FB));
      tma_load_3d(ring + slot * FBP, &ym.m[v], i0 - G::HX, j0 - HF, next_issue, &bar[slot]);
    }
  };
  if (tid == 0) issue_upto(plo + NS - 1);

  // closure classes: along xi per point of the pair (its weights kept in registers, one pair of
  // weights per tap), along eta per row (the warp's), along zeta per plane
  F2 wx[NQ];
  {
    const int cxa = cls_of(min(i, P.nx - 1), P.nx, P.nb), cxb = cls_of(min(i + 1, P.nx - 1), P.nx, P.nb);
#pragma unroll
    for (int o = 0; o < NQ; ++o) wx[o] = make_float2(P.w[cxa][o], P.w[cxb][o]);
  }
  const int cy = cls_of(min(j, P.ny - 1), P.ny, P.nb);
  const int c = G::HX + 2 * tx;  // column of the pair's first point in a box row

  // F_xi - I of the pair on one box row (brow: the row's first element); x receives the pair's values
  auto xi = [&](const float* brow, F2& x) -> F2 {
    F2 win[NW];
#pragma unroll
    for (int m = 0; m < NW; ++m) win[m] = ld2(brow + c - 2 * HP + 2 * m);
    x = win[HP];
    F2 d = make_float2(0.f, 0.f);
#pragma unroll
    for (int o = -HF; o <= HF; ++o) {
      const int t = o + 2 * HP;  // window position of the first point's tap
      if ((t & 1) == 0) {
        d = fma2(wx[o + HF], win[t >> 1], d);
      } else {
        d.x = fmaf(wx[o + HF].x, win[t >> 1].y, d.x);
        d.y = fmaf(wx[o + HF].y, win[(t >> 1) + 1].x, d.y);
      }
    }
    return d;
  };

  // point offsets fit 32 bits (the host checks the block size)
  const unsigned nxy = (unsigned)P.nx * (unsigned)P.ny;
  const unsigned lij = (unsigned)i + (unsigned)P.nx * (unsigned)j;
  // (the carried error may be read from and written to the same buffer: each point's error is
  // read by its owner before the owner writes the new one)
  const float* errp = P.err[v];
  float* outp = P.out[v];
  float* cmpp = P.comp[v];

  F2 uq[NQ];
#pragma unroll
  for (int q = 0; q < NQ; ++q) uq[q] = make_float2(0.f, 0.f);
  float* const dme = dsm + ty * kPairTX + 2 * tx;
  const int pstart = k0 - HF, pend = k1 - 1 + HF;
  int ds = 0;  // ring slot of plane p; advanced below, the slot of plane kf = p - h (h + 1 slots)
  for (int p = pstart; p <= pend; ++p) {
    const int rel = p - plo;  // negative for the planes before the block
    const int kf = p - HF;    // the plane finished at the end of this iteration
    const bool fin = active && kf >= k0 && kf < k1;
    const unsigned lf = lij + nxy * (unsigned)kf;
    F2 e0 = make_float2(0.f, 0.f);
    if (COMP && fin) e0 = ld2(errp + lf);
    F2 u2 = make_float2(0.f, 0.f), d12 = make_float2(0.f, 0.f);
    if (p >= plo && p <= phi) {
      const int slot = rel % NS;
      const bool ok = mbar_wait(&bar[slot], (unsigned)((rel / NS) & 1), P.wait_ns);
      // (a thread whose wait gave up reads a box in flight: values only, never used below)
      const float* box = ring + slot * FBP;
      float* u1 = u1s + (rel & 1) * G::U1;
      F2 xc;
      const F2 d1 = xi(box + (ty + HF) * BX, xc);
      const F2 u1c = COMP ? add2(xc, d1) : d1;
      st2(u1 + (ty + HF) * kPairTX + 2 * tx, u1c);
      // the eta halo rows, one per thread row (more than one for half-widths above 4)
#pragma unroll
      for (int r0 = 0; r0 < 2 * HF; r0 += TY) {
        const int r = r0 + ty;
        if (r < 2 * HF) {
          const int row = r < HF ? r : r + TY;
          F2 xh;
          const F2 dh = xi(box + row * BX, xh);
          st2(u1 + row * kPairTX + 2 * tx, COMP ? add2(xh, dh) : dh);
        }
      }
      // every thread is past plane p - 1 (so the ring slot of plane p - 1 - h, finished there, is
      // free) and has written its part of this plane's u1; the other buffer, read by plane p - 1,
      // is next written at plane p + 1, after the next barrier
      if (__syncthreads_or(!ok)) {
        if (tid == 0) {
          atomicExch(P.errflag, 1);
          // every copy still in flight, the one whose wait gave up included
          for (int w = p; w < next_issue; ++w) mbar_wait(&bar[(w - plo) % NS], (unsigned)(((w - plo) / NS) & 1));
        }
        return;
      }
      if (tid == 0) issue_upto(p + G::PF);
      // (eta and zeta taps as two scalar FMAs whose weight is an operand from the constant bank:
      // a packed FMA would first need the weight copied into both halves of a register pair)
      const float* col = u1 + (ty + HF) * kPairTX + 2 * tx;
      F2 dy = make_float2(0.f, 0.f);
      if (cy == 0) {
#pragma unroll
        for (int o = -HF; o <= HF; ++o) dy = fmas(P.w[0][o + HF], o == 0 ? u1c : ld2(col + o * kPairTX), dy);
      } else {
#pragma unroll
        for (int o = -HF; o <= HF; ++o) dy = fmas(P.w[cy][o + HF], o == 0 ? u1c : ld2(col + o * kPairTX), dy);
      }
      if (COMP) {
        u2 = add2(u1c, dy);
        d12 = add2(d1, dy);
      } else {
        u2 = dy;
      }
    }
#pragma unroll
    for (int q = 0; q < NQ - 1; ++q) uq[q] = uq[q + 1];
    uq[NQ - 1] = u2;
    if (COMP) {
      st2(dme + ds * G::DP, d12);
      ds = ds == HF ? 0 : ds + 1;
    }
    if (!fin) continue;
    const int cz = cls_of(kf, P.nz, P.nb);
    F2 fz = make_float2(0.f, 0.f);
    if (cz == 0) {
#pragma unroll
      for (int o = 0; o < NQ; ++o) fz = fmas(P.w[0][o], uq[o], fz);
    } else {
#pragma unroll
      for (int o = 0; o < NQ; ++o) fz = fmas(P.w[cz][o], uq[o], fz);
    }
    // the pre-filter pair of plane kf, still in its ring slot (kf >= plo)
    const F2 x0 = ld2(ring + ((rel - HF) % NS) * FBP + (ty + HF) * BX + c);
    if (!COMP) {
      // the one-row kernel's expression, lane by lane
      st2(outp + lf, make_float2((1.f - P.blend) * x0.x + P.blend * fz.x, (1.f - P.blend) * x0.y + P.blend * fz.y));
      continue;
    }
    const F2 D = add2(ld2(dme + ds * G::DP), fz);
    const F2 t = fmas(P.blend, D, e0);
    const F2 sm = add2(x0, t);
    const F2 bb = subs(sm, x0);
    const F2 cm = add2(subs(x0, subs(sm, bb)), subs(t, bb));
    st2(outp + lf, sm);
    st2(cmpp + lf, cm);
  }
}

template <int HF, bool COMP>
cudaError_t go_filter_pair(const FieldMaps& in, const TmaFilterParams<float>& p, int tiles, int chunks,
                           cudaStream_t s) {
  using G = PairGeo<HF>;
  static bool attr = false;
  if (!attr) {
    cudaError_t e =
        cudaFuncSetAttribute(k_filter_pair<HF, COMP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::BYTES);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  k_filter_pair<HF, COMP><<<dim3(tiles, chunks, p.V), 256, G::BYTES, s>>>(in, p);
  return cudaGetLastError();
}

}  // namespace

bool filter_pair_half_width(int hf) { return hf == 2 || hf == 4 || hf == 5; }

void filter_pair_box(int hf, int* bx, int* by, int* tx, int* ty) {
  const int hx = ((hf + 3) / 4) * 4;
  *bx = kPairTX + 2 * hx;
  *by = kTileY + 2 * hf;
  *tx = kPairTX;
  *ty = kTileY;
}

cudaError_t launch_filter_pair(const FieldMaps& in, const TmaFilterParams<float>& p, int hf, int comp, int tiles,
                               int chunks, cudaStream_t s) {
  if (p.nx % 2 != 0 || p.code[0] || (comp && (!p.err[0] || !p.comp[0]))) return cudaErrorInvalidValue;
#define LEE_PAIR_CASE(HF)                                                                            \
  if (hf == HF)                                                                                      \
    return comp ? go_filter_pair<HF, true>(in, p, tiles, chunks, s) : go_filter_pair<HF, false>(in, p, tiles, chunks, s);
  LEE_PAIR_CASE(2)
  LEE_PAIR_CASE(4)
  LEE_PAIR_CASE(5)
#undef LEE_PAIR_CASE
  return cudaErrorInvalidValue;
}

}  // namespace lee
