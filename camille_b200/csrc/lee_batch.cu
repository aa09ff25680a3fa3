// Batched kernels: many independent 2-D blocks (instances of uneven sizes) advance through one
// launch per RK stage and one per filter, over a work list of strips drawn from every block.
//
// A work item is a strip of columns of one block and a range of its rows; each CTA takes a
// run of consecutive items (a block's items are contiguous, so a CTA rarely changes block),
// copies the block's parameters (pointers, coefficients, time step, source) into shared memory
// when it does, and marches its strip along eta, streaming rows through a shared-memory ring
// with asynchronous copies issued a few rows ahead. The arithmetic is that of the per-block
// kernels (the generic operator order of lee_step.cu and the pointwise update of
// lee_point.cuh), so a block gives the same bits batched or alone.
#include <algorithm>
#include <type_traits>

#include "lee_internal.h"
#include "lee_point.cuh"
#include "lee_tma_util.cuh"

namespace lee {
namespace {

constexpr int kFdH = 2;   // the 4th-order difference: closure rows read 3 points, inside a halo of 2
constexpr int kFlH = 4;   // the 8th-order filter: closure rows read 7 points, inside a halo of 4

// An operator's weights in the working precision, converted once per CTA exactly as dop()
// converts them per use (T(c), T(B), T(mfac * B)), for a compile-time half-width HH and row
// width SS.
template <typename T, int HH, int SS>
struct SmOp {
  T c[2 * HH + 1];
  T bl[HH][SS];
  T br[HH][SS];
};

template <typename T, int HH, int SS>
__device__ __forceinline__ void load_op(SmOp<T, HH, SS>& w, const OpTable& op, int tid, int nthr) {
  for (int q = tid; q < 2 * HH + 1; q += nthr) w.c[q] = T(op.c[q]);
  for (int q = tid; q < HH * SS; q += nthr) {
    const int r = q / SS, s = q % SS;
    w.bl[r][s] = T(op.B[r][s]);
    w.br[r][s] = T(op.mfac * op.B[r][s]);
  }
}

// dop() of lee_step.cu on a line held in shared memory (same terms in the same order): f
// points at the element of position `pos` on a line of n points, stride ST.
template <typename T, int HH, int SS, int ST>
__device__ __forceinline__ T dop_c(const SmOp<T, HH, SS>& w, const T* f, int pos, int n) {
  T acc = T(0);
  if (pos >= HH && pos <= n - 1 - HH) {
#pragma unroll
    for (int l = -HH; l <= HH; ++l) acc += w.c[l + HH] * f[l * ST];
    return acc;
  }
  // closure rows: zero weights are skipped, so a row reads only the points within HH of its
  // own (the 8th-order filter's rows carry zeros out to 6 points, beyond the staged halo)
  if (pos < HH) {
    const int r = pos;
    const T* a = f - r * ST;
#pragma unroll
    for (int s = 0; s < SS; ++s)
      if (w.bl[r][s] != T(0)) acc += w.bl[r][s] * a[s * ST];
    return acc;
  }
  const int r = n - 1 - pos;
  const T* a = f + r * ST;
#pragma unroll
  for (int s = 0; s < SS; ++s)
    if (w.br[r][s] != T(0)) acc += w.br[r][s] * a[-s * ST];
  return acc;
}

// dop() along eta on rows held in a ring of NSL rows: row r of column `col` lives at
// ring[(r mod NSL) * rs + col]; so[] holds the ring offsets of rows j - HH .. j + HH.
template <typename T, int HH, int SS, int NSL>
__device__ __forceinline__ T dop_ring(const SmOp<T, HH, SS>& w, const T* ring, const int (&so)[2 * HH + 1], int rs,
                                      int col, int j, int n) {
  T acc = T(0);
  if (j >= HH && j <= n - 1 - HH) {
#pragma unroll
    for (int l = -HH; l <= HH; ++l) acc += w.c[l + HH] * ring[so[l + HH] + col];
    return acc;
  }
  if (j < HH) {
    const int r = j;
#pragma unroll
    for (int s = 0; s < SS; ++s)
      if (w.bl[r][s] != T(0)) acc += w.bl[r][s] * ring[((j - r + s + NSL) % NSL) * rs + col];
    return acc;
  }
  const int r = n - 1 - j;
#pragma unroll
  for (int s = 0; s < SS; ++s)
    if (w.br[r][s] != T(0)) acc += w.br[r][s] * ring[((j + r - s + 2 * NSL) % NSL) * rs + col];
  return acc;
}

// Copy a parameter struct from global to shared memory with all threads.
template <typename P>
__device__ __forceinline__ void copy_params(P* dst, const P* src, int tid, int nthr) {
  static_assert(sizeof(P) % 4 == 0, "parameter block size");
  const int* s = reinterpret_cast<const int*>(src);
  int* d = reinterpret_cast<int*>(dst);
  for (int q = tid; q < (int)(sizeof(P) / 4); q += nthr) d[q] = s[q];
}

// Asynchronous global -> shared copies of one element (4 or 8 bytes), grouped per row.
template <typename T>
__device__ __forceinline__ void cp_async(T* dst, const T* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  if (sizeof(T) == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
  else asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Row r of a strip (columns x0 - H .. x0 + TX + H - 1) of V fields into ring slot `slot`, by
// NT threads: cp.async inside the block, zeros outside it; one commit group per row (empty
// when the row is outside the block, so the group count stays one per row).
template <typename T, int V, int TX, int H, int NT = TX>
__device__ __forceinline__ void issue_row(T* ring, int slot, const T* const* fields, int r, int x0, int nx, int ny,
                                          int tid) {
  constexpr int W = TX + 2 * H;
  if (r >= 0 && r < ny) {
#pragma unroll
    for (int v = 0; v < V; ++v) {
      T* dst = ring + ((long long)slot * V + v) * W;
      const T* src = fields[v] + (long long)r * nx;
      for (int cc = tid; cc < W; cc += NT) {
        const int gx = x0 - H + cc;
        if (gx >= 0 && gx < nx) cp_async(dst + cc, src + gx);
        else dst[cc] = T(0);
      }
    }
  }
  cp_commit();
}

// The stage kernel of a batch, marching along eta: a CTA of TX threads owns CX * TX columns of
// a block (columns tid + m TX of the strip for m < CX) and rows [ys, ye) of them. Rows of the stage input (with a xi halo)
// stream through a ring of 2H + 2 + PF rows in shared memory, PF rows ahead of the row being
// computed; the pointwise inputs of the next row are loaded into registers while this row is
// computed. A work item is int4 (block, x0, ys, ye); a CTA takes `per` consecutive items.
template <typename T, bool COMP, int TX, int PF, int CX>
__device__ __forceinline__ void batch_stage_run(const StageParams<T>* __restrict__ prm,
                                                const int4* __restrict__ items, int t0, int t1) {
  constexpr int V = 4;
  constexpr int H = kFdH;
  constexpr int SW = CX * TX;  // strip width
  constexpr int W = SW + 2 * H;
  constexpr int NS = 2 * H + 2 + PF;
  constexpr int TR = kTrJmField | kTrUniform | kTrSponge;
  extern __shared__ __align__(16) unsigned char dsm[];
  T* ring = reinterpret_cast<T*>(dsm);  // [NS][V][W]
  __shared__ __align__(16) StageParams<T> P;
  __shared__ SmOp<T, kFdH, 3> w;
  __shared__ int cur;
  const int tid = threadIdx.x;
  if (tid == 0) cur = -1;
  load_op(w, prm[0].fd, tid, TX);
  for (int t = t0; t < t1; ++t) {
    const int4 it = items[t];
    __syncthreads();  // every thread is done with the previous item's ring and parameters
    if (it.x != cur) {
      copy_params(&P, prm + it.x, tid, TX);
      __syncthreads();
      if (tid == 0) cur = it.x;
    }
    const int nx = P.nx, ny = P.ny, x0 = it.y, ys = it.z, ye = it.w;
    const T* const* zin = P.zin;
    // prologue: rows ys - H .. ys + H + PF - 1
    for (int r = ys - H; r < ys + H + PF; ++r)
      issue_row<T, V, SW, H, TX>(ring, (r + NS) % NS, zin, r, x0, nx, ny, tid);
    PointIn<T, 2> in_cur[CX], in_nxt[CX];
#pragma unroll
    for (int m = 0; m < CX; ++m)
      if (x0 + tid + m * TX < nx) gather<T, 2, COMP, TR>(P, (long long)ys * nx + x0 + tid + m * TX, in_cur[m]);
    for (int j = ys; j < ye; ++j) {
      issue_row<T, V, SW, H, TX>(ring, (j + H + PF + NS) % NS, zin, j + H + PF, x0, nx, ny, tid);
#pragma unroll
      for (int m = 0; m < CX; ++m)
        if (x0 + tid + m * TX < nx && j + 1 < ye)
          gather<T, 2, COMP, TR>(P, (long long)(j + 1) * nx + x0 + tid + m * TX, in_nxt[m]);
      cp_wait<PF>();
      __syncthreads();
      int so[2 * H + 1];
#pragma unroll
      for (int l = -H; l <= H; ++l) so[l + H] = ((j + l + NS) % NS) * (V * W);
#pragma unroll
      for (int m = 0; m < CX; ++m) {
        const int cl = tid + m * TX, i = x0 + cl;
        if (i < nx) {
          T D[V][2], q[V];
#pragma unroll
          for (int v = 0; v < V; ++v) {
            const T* c0 = ring + so[H] + v * W + cl + H;
            D[v][0] = dop_c<T, kFdH, 3, 1>(w, c0, i, nx);
            D[v][1] = dop_ring<T, kFdH, 3, NS>(w, ring, so, V * W, v * W + cl + H, j, ny);
            q[v] = *c0;
          }
          rhs_update<T, 2, COMP, TR>(P, (long long)j * nx + i, i, j, 0, D, q, in_cur[m]);
        }
        in_cur[m] = in_nxt[m];
      }
    }
    cp_wait<0>();
  }
}

// The filter of a batch, marching along eta: rows of the pre-filter state (with a xi halo of
// 4) stream through a shared-memory ring; each thread applies F_xi to its column of every row
// as it arrives and keeps the results of the last 2H + 1 rows in a register queue, from which
// F_eta of the row H behind follows without another pass through shared memory. The
// arithmetic is that of the per-block passes (xi pass, then eta pass with the blend, or the
// increment form with the two-float sum), term for term. Fields are independent: a CTA takes
// VF of them (fields blockIdx.y * VF ...), which keeps the register queues short.
template <typename T, bool COMP, int TX, int PF, int VF>
__device__ __forceinline__ void batch_filter_run(const BatchFilterInst<T>* __restrict__ inst,
                                                 const int4* __restrict__ items, int t0, int t1, const OpTable& op,
                                                 T blend, int vb) {
  constexpr int V = VF;
  constexpr int H = kFlH;
  constexpr int S = 7;
  constexpr int W = TX + 2 * H;
  constexpr int NX = H + PF + 2;  // state rows r - H - 1 .. r + PF around the row r being filtered in xi
  extern __shared__ __align__(16) unsigned char dsm[];
  T* X = reinterpret_cast<T*>(dsm);  // [NX][VF][W]
  __shared__ __align__(16) BatchFilterInst<T> P;
  __shared__ SmOp<T, kFlH, S> w;
  __shared__ int cur;
  const int tid = threadIdx.x;
  if (tid == 0) cur = -1;
  load_op(w, op, tid, TX);
  for (int t = t0; t < t1; ++t) {
    const int4 it = items[t];
    __syncthreads();
    if (it.x != cur) {
      copy_params(&P, inst + it.x, tid, TX);
      __syncthreads();
      if (tid == 0) cur = it.x;
    }
    const int nx = P.nx, ny = P.ny, x0 = it.y, ys = it.z, ye = it.w;
    const T* const* xf = P.x + vb;
    const int i = x0 + tid;
    const bool col = i < nx;
    T fq[V][2 * H + 1];  // xi-pass values (x + D_xi x when compensated) of rows r - 2H .. r
    T dq[V][H + 1];      // compensated: D_xi x of rows r - H .. r
#pragma unroll
    for (int v = 0; v < V; ++v) {
#pragma unroll
      for (int q = 0; q <= 2 * H; ++q) fq[v][q] = T(0);
#pragma unroll
      for (int q = 0; q <= H; ++q) dq[v][q] = T(0);
    }
    T err_nxt[V];
    for (int r = ys - H; r < ys - H + PF; ++r) issue_row<T, V, TX, H>(X, (r + NX) % NX, xf, r, x0, nx, ny, tid);
    for (int r = ys - H; r < ye + H; ++r) {
      issue_row<T, V, TX, H>(X, (r + PF + NX) % NX, xf, r + PF, x0, nx, ny, tid);
      const int j = r - H;  // the row finished in this iteration
      if (COMP && col && j >= ys && j < ye) {
#pragma unroll
        for (int v = 0; v < V; ++v) err_nxt[v] = P.err[vb + v][(long long)j * nx + i];
      }
      cp_wait<PF>();
      __syncthreads();  // state row r landed for every thread
      const bool rin = r >= 0 && r < ny;
#pragma unroll
      for (int v = 0; v < V; ++v) {
        T o = T(0), fx = T(0);
        if (rin && col) {
          const T* f = X + ((long long)((r + NX) % NX) * V + v) * W + tid + H;
          fx = dop_c<T, kFlH, S, 1>(w, f, i, nx);
          o = COMP ? *f + fx : fx;
        }
#pragma unroll
        for (int q = 0; q < 2 * H; ++q) fq[v][q] = fq[v][q + 1];
        fq[v][2 * H] = o;
        if (COMP) {
#pragma unroll
          for (int q = 0; q < H; ++q) dq[v][q] = dq[v][q + 1];
          dq[v][H] = fx;
        }
      }
      if (col && j >= ys && j < ye) {
        const long long l = (long long)j * nx + i;
        const T* xrow = X + (long long)((j + NX) % NX) * V * W + tid + H;
#pragma unroll
        for (int v = 0; v < V; ++v) {
          // F_eta at row j from the queue (entry H + q holds row j + q), in dop()'s order
          T fy = T(0);
          if (j >= H && j <= ny - 1 - H) {
#pragma unroll
            for (int q = -H; q <= H; ++q) fy += w.c[q + H] * fq[v][q + H];
          } else if (j < H) {  // left closure row j reads rows s = 0 .. S-1, i.e. q = s - j
#pragma unroll
            for (int q = -H; q <= H; ++q) {
              const int sidx = j + q;
              if (sidx >= 0 && sidx < S && w.bl[j][sidx] != T(0)) fy += w.bl[j][sidx] * fq[v][q + H];
            }
          } else {  // right closure row rr reads rows ny-1-s, s = 0 .. S-1, i.e. q = rr - s (s ascending)
            const int rr = ny - 1 - j;
#pragma unroll
            for (int q = H; q >= -H; --q) {
              const int sidx = rr - q;
              if (sidx >= 0 && sidx < S && w.br[rr][sidx] != T(0)) fy += w.br[rr][sidx] * fq[v][q + H];
            }
          }
          const T xc = xrow[v * W];
          if (!COMP) {
            P.y[vb + v][l] = (T(1) - blend) * xc + blend * fy;
          } else {
            const T dsum = dq[v][0] + fy;
            const T tt = blend * dsum + err_nxt[v];
            const T s2 = xc + tt;
            const T bb = s2 - xc;
            const T e = (xc - (s2 - bb)) + (tt - bb);
            P.y[vb + v][l] = s2;
            P.comp[vb + v][l] = e;
          }
        }
      }
    }
    cp_wait<0>();
  }
}

// The launches of one stage and of the filter: each CTA takes a run of `per` consecutive items
// (the filter's CTAs in blockIdx.y take fields blockIdx.y * VF ...).
template <typename T, bool COMP, int TX, int PF, int CX>
__global__ void __launch_bounds__(TX) k_batch_stage(const StageParams<T>* __restrict__ prm,
                                                    const int4* __restrict__ items, int nitems, int per) {
  const int t0 = blockIdx.x * per;
  batch_stage_run<T, COMP, TX, PF, CX>(prm, items, t0, min(t0 + per, nitems));
}

template <typename T, bool COMP, int TX, int PF, int VF>
__global__ void __launch_bounds__(TX) k_batch_filter(const BatchFilterInst<T>* __restrict__ inst,
                                                     const int4* __restrict__ items, int nitems, int per, OpTable op,
                                                     T blend) {
  const int t0 = blockIdx.x * per;
  batch_filter_run<T, COMP, TX, PF, VF>(inst, items, t0, min(t0 + per, nitems), op, blend, (int)blockIdx.y * VF);
}

// Fields per filter CTA (of the four of a 2-D block).
constexpr int kFilterVF = 1;

// Barrier of all CTAs of a persistent launch (co-resident: the launch is cooperative). The
// counter gb[0] and generation gb[1] start at zero (the host clears them before each launch). A
// CTA's writes before the barrier are visible to every CTA after it (CTA barrier, then a
// device-scope fence around the arrival and the wait). The wait is bounded: after `limit_ns`
// nanoseconds (at once for 0) the CTA records the failure in the device flag and the barrier
// returns false, and the CTA leaves the kernel, so the others give up at this barrier or the
// next: nothing waits for ever.
__device__ __forceinline__ bool grid_barrier(unsigned* gb, unsigned nblk, unsigned long long limit_ns, int* err) {
  __syncthreads();
  int ok = 1;
  if (threadIdx.x == 0) {
    volatile unsigned* gen = gb + 1;
    const unsigned g = *gen;  // the current generation: it moves only once this CTA has arrived
    __threadfence();
    if (atomicAdd(gb, 1u) == nblk - 1) {
      atomicExch(gb, 0u);  // reset before the release: no CTA arrives again before it sees it
      __threadfence();
      atomicAdd(gb + 1, 1u);
    } else if (limit_ns == 0) {
      ok = 0;
    } else {
      const unsigned long long t0 = gtimer();
      for (unsigned it = 1; *gen == g; ++it)
        if ((it & 63u) == 0u && gtimer() - t0 > limit_ns) {
          ok = 0;
          break;
        }
    }
    __threadfence();
    if (!ok) atomicExch(err, 1);
  }
  return __syncthreads_and(ok) != 0;
}

// One whole batched step in one launch: the ns RK stages over the work list, each followed by a
// grid barrier, then the filter over the same work list (each field of each item one unit). A
// CTA takes the same run of items in every stage. The per-point arithmetic is that of the
// per-phase launches (the same bodies), so the results are the same bits.
template <typename T, bool COMP, int TX>
__global__ void __launch_bounds__(TX) k_batch_step(const StageParams<T>* __restrict__ prm, int nbk, int ns,
                                                   const BatchFilterInst<T>* __restrict__ inst,
                                                   const int4* __restrict__ items, int nitems, OpTable op, T blend,
                                                   unsigned* gbar, int* err, unsigned long long wait_ns) {
  const int G = (int)gridDim.x, b = (int)blockIdx.x;
  const int per = (nitems + G - 1) / G;
  const int t0 = min(b * per, nitems), t1 = min(t0 + per, nitems);
  for (int s = 0; s < ns; ++s) {
    batch_stage_run<T, COMP, TX, 2, 1>(prm + (size_t)s * nbk, items, t0, t1);
    if (!grid_barrier(gbar, (unsigned)G, wait_ns, err)) return;
  }
  constexpr int FG = 4 / kFilterVF;
  const int nu = FG * nitems, pu = (nu + G - 1) / G;
  const int u1 = min(nu, (b + 1) * pu);
  for (int u = min(nu, b * pu); u < u1;) {
    const int fg = u / nitems, i0 = u - fg * nitems, i1 = min(nitems, i0 + (u1 - u));
    batch_filter_run<T, COMP, TX, 2, kFilterVF>(inst, items, i0, i1, op, blend, fg * kFilterVF);
    u += i1 - i0;
  }
}

template <typename T, int SW>
size_t stage_smem() {
  return sizeof(T) * 4 * (2 * kFdH + 2 + 2) * (SW + 2 * kFdH);
}

// TX threads, each with CX columns of the strip
template <typename T, bool COMP, int TX, int CX>
cudaError_t go_stage(const StageParams<T>* prm, const int4* items, int n, int grid, cudaStream_t s) {
  const size_t smem = stage_smem<T, TX * CX>();
  cudaError_t e = cudaFuncSetAttribute(k_batch_stage<T, COMP, TX, 2, CX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  const int per = (n + grid - 1) / grid;
  k_batch_stage<T, COMP, TX, 2, CX><<<(n + per - 1) / per, TX, smem, s>>>(prm, items, n, per);
  return cudaGetLastError();
}

template <typename T, int TX>
size_t filter_smem() {
  return sizeof(T) * kFilterVF * (kFlH + 2 + 2) * (TX + 2 * kFlH);
}

template <typename T, bool COMP, int TX>
cudaError_t go_filter(const BatchFilterInst<T>* inst, const int4* items, int n, int grid, const OpTable& op, T blend,
                      cudaStream_t s) {
  const size_t smem = filter_smem<T, TX>();
  cudaError_t e = cudaFuncSetAttribute(k_batch_filter<T, COMP, TX, 2, kFilterVF>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  // `grid` CTAs in all: the items are shared out over grid / (4 / VF) CTAs per field group
  constexpr int G = 4 / kFilterVF;
  const int gx = std::max(1, grid / G);
  const int per = (n + gx - 1) / gx;
  k_batch_filter<T, COMP, TX, 2, kFilterVF><<<dim3((n + per - 1) / per, G), TX, smem, s>>>(inst, items, n, per, op,
                                                                                          blend);
  return cudaGetLastError();
}

template <typename T, bool COMP, int TX, int CX>
int occupancy_stage_of() {
  const size_t smem = stage_smem<T, TX * CX>();
  cudaFuncSetAttribute(k_batch_stage<T, COMP, TX, 2, CX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch_stage<T, COMP, TX, 2, CX>, TX, smem);
  return n > 0 ? n : 1;
}

template <typename T, bool COMP>
int occupancy_stage(int width, int cx) {
  if (cx == 2) return width == 128 ? occupancy_stage_of<T, COMP, 64, 2>() : occupancy_stage_of<T, COMP, 128, 2>();
  if (width == 64) return occupancy_stage_of<T, COMP, 64, 1>();
  if (width == 128) return occupancy_stage_of<T, COMP, 128, 1>();
  return occupancy_stage_of<T, COMP, 256, 1>();
}

}  // namespace

// Work-item shapes, by index: columns x rows of a strip, and the stage kernel's columns per
// thread (the filter has one thread per column).
namespace {
const int kShapes[kBatchShapes][3] = {{64, 16, 1}, {128, 16, 1}, {128, 32, 1}, {256, 16, 1},
                                      {64, 32, 1},  {128, 16, 2}, {256, 16, 2}};
}  // namespace

void batch_shape(int shape, int* tx, int* ty) {
  *tx = kShapes[shape][0];
  *ty = kShapes[shape][1];
}

template <typename T>
cudaError_t launch_batch_stage(const StageParams<T>* prm, const int4* items, int n, int shape, int comp, int grid,
                               cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  int tx, ty;
  batch_shape(shape, &tx, &ty);
  const int cx = kShapes[shape][2];
  if (comp) {
    if (cx == 2) return tx == 128 ? go_stage<T, true, 64, 2>(prm, items, n, grid, s)
                                  : go_stage<T, true, 128, 2>(prm, items, n, grid, s);
    if (tx == 64) return go_stage<T, true, 64, 1>(prm, items, n, grid, s);
    if (tx == 128) return go_stage<T, true, 128, 1>(prm, items, n, grid, s);
    return go_stage<T, true, 256, 1>(prm, items, n, grid, s);
  }
  if (cx == 2) return tx == 128 ? go_stage<T, false, 64, 2>(prm, items, n, grid, s)
                                : go_stage<T, false, 128, 2>(prm, items, n, grid, s);
  if (tx == 64) return go_stage<T, false, 64, 1>(prm, items, n, grid, s);
  if (tx == 128) return go_stage<T, false, 128, 1>(prm, items, n, grid, s);
  return go_stage<T, false, 256, 1>(prm, items, n, grid, s);
}

template <typename T>
cudaError_t launch_batch_filter(const BatchFilterInst<T>* inst, const int4* items, int n, int shape, int comp,
                                int grid, const OpTable& op, double blend, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  int tx, ty;
  batch_shape(shape, &tx, &ty);
  const T b = (T)blend;
  if (comp) {
    if (tx == 64) return go_filter<T, true, 64>(inst, items, n, grid, op, b, s);
    if (tx == 128) return go_filter<T, true, 128>(inst, items, n, grid, op, b, s);
    return go_filter<T, true, 256>(inst, items, n, grid, op, b, s);
  }
  if (tx == 64) return go_filter<T, false, 64>(inst, items, n, grid, op, b, s);
  if (tx == 128) return go_filter<T, false, 128>(inst, items, n, grid, op, b, s);
  return go_filter<T, false, 256>(inst, items, n, grid, op, b, s);
}

template <typename T>
int batch_stage_occupancy(int shape, int comp) {
  int tx, ty;
  batch_shape(shape, &tx, &ty);
  const int cx = kShapes[shape][2];
  return comp ? occupancy_stage<T, true>(tx, cx) : occupancy_stage<T, false>(tx, cx);
}

template <typename T, bool COMP>
int occupancy_filter(int tx) {
  int n = 0;
  if (tx == 64)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch_filter<T, COMP, 64, 2, kFilterVF>, 64, filter_smem<T, 64>());
  else if (tx == 128)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch_filter<T, COMP, 128, 2, kFilterVF>, 128, filter_smem<T, 128>());
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch_filter<T, COMP, 256, 2, kFilterVF>, 256, filter_smem<T, 256>());
  return n > 0 ? n : 1;
}

template <typename T>
int batch_filter_occupancy(int shape, int comp) {
  int tx, ty;
  batch_shape(shape, &tx, &ty);
  // the dynamic shared memory limit must be raised before the occupancy query counts it
  const size_t smem = tx == 64 ? filter_smem<T, 64>() : tx == 128 ? filter_smem<T, 128>() : filter_smem<T, 256>();
  if (comp) {
    cudaFuncSetAttribute(tx == 64 ? k_batch_filter<T, true, 64, 2, kFilterVF> : tx == 128 ? k_batch_filter<T, true, 128, 2, kFilterVF>
                                                                                : k_batch_filter<T, true, 256, 2, kFilterVF>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    return occupancy_filter<T, true>(tx);
  }
  cudaFuncSetAttribute(tx == 64 ? k_batch_filter<T, false, 64, 2, kFilterVF> : tx == 128 ? k_batch_filter<T, false, 128, 2, kFilterVF>
                                                                               : k_batch_filter<T, false, 256, 2, kFilterVF>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  return occupancy_filter<T, false>(tx);
}

// The whole step in one persistent launch (work items of a shape with one column per stage
// thread): as many CTAs as fit on the device at once, launched cooperatively so that they are
// all resident (the launch fails rather than waits otherwise).
template <typename T, bool COMP, int TX>
cudaError_t go_step(const StageParams<T>* prm, int nbk, int ns, const BatchFilterInst<T>* inst, const int4* items,
                    int n, const OpTable& op, T blend, unsigned* gbar, int* err, unsigned long long wait_ns,
                    cudaStream_t s) {
  const size_t smem = std::max(stage_smem<T, TX>(), filter_smem<T, TX>());
  auto kern = k_batch_step<T, COMP, TX>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0, nsm = 0, per_sm = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, TX, smem)) != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  const int grid = std::max(1, std::min(per_sm * nsm, n));
  if ((e = cudaMemsetAsync(gbar, 0, 2 * sizeof(unsigned), s)) != cudaSuccess) return e;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(TX);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, prm, nbk, ns, inst, items, n, op, blend, gbar, err, wait_ns);
}

bool batch_step_shape(int shape) { return shape >= 0 && shape < kBatchShapes && kShapes[shape][2] == 1; }

template <typename T>
cudaError_t launch_batch_step(const StageParams<T>* prm, int nbk, int ns, const BatchFilterInst<T>* inst,
                              const int4* items, int n, int shape, int comp, const OpTable& op, double blend,
                              unsigned* gbar, int* err, unsigned long long wait_ns, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  if (!batch_step_shape(shape)) return cudaErrorInvalidValue;
  const int tx = kShapes[shape][0];
  const T b = (T)blend;
#define LEE_STEP_CASE(C, X)                                                                     \
  if (comp == (C ? 1 : 0) && tx == X)                                                           \
    return go_step<T, C, X>(prm, nbk, ns, inst, items, n, op, b, gbar, err, wait_ns, s);
  LEE_STEP_CASE(true, 64)
  LEE_STEP_CASE(true, 128)
  LEE_STEP_CASE(true, 256)
  LEE_STEP_CASE(false, 64)
  LEE_STEP_CASE(false, 128)
  LEE_STEP_CASE(false, 256)
#undef LEE_STEP_CASE
  return cudaErrorInvalidValue;
}

template cudaError_t launch_batch_step<double>(const StageParams<double>*, int, int, const BatchFilterInst<double>*,
                                               const int4*, int, int, int, const OpTable&, double, unsigned*, int*,
                                               unsigned long long, cudaStream_t);
template cudaError_t launch_batch_step<float>(const StageParams<float>*, int, int, const BatchFilterInst<float>*,
                                              const int4*, int, int, int, const OpTable&, double, unsigned*, int*,
                                              unsigned long long, cudaStream_t);
template cudaError_t launch_batch_stage<double>(const StageParams<double>*, const int4*, int, int, int, int,
                                                cudaStream_t);
template cudaError_t launch_batch_stage<float>(const StageParams<float>*, const int4*, int, int, int, int,
                                               cudaStream_t);
template cudaError_t launch_batch_filter<double>(const BatchFilterInst<double>*, const int4*, int, int, int, int,
                                                 const OpTable&, double, cudaStream_t);
template cudaError_t launch_batch_filter<float>(const BatchFilterInst<float>*, const int4*, int, int, int, int,
                                                const OpTable&, double, cudaStream_t);
template int batch_stage_occupancy<double>(int, int);
template int batch_stage_occupancy<float>(int, int);
template int batch_filter_occupancy<double>(int, int);
template int batch_filter_occupancy<float>(int, int);

}  // namespace lee
