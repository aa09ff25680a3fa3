// Batched kernels: many independent 2-D blocks (instances of uneven sizes) advance through one
// launch per RK stage and one per filter, over a work list of tiles drawn from every block.
//
// Each CTA is persistent: it walks the tile list with a stride of the grid size. A tile
// names its block and its origin; the block's stage parameters (pointers, coefficients, time
// step, source) are copied into shared memory when the CTA moves to another block, and the
// tile's stage input with its stencil halo is staged in shared memory by coalesced row loads.
// The arithmetic is that of the per-block kernels (the generic operator order of lee_step.cu
// and the pointwise update of lee_point.cuh), so a block gives the same bits batched or alone.
#include <type_traits>

#include "lee_internal.h"
#include "lee_point.cuh"

namespace lee {
namespace {

constexpr int kFdH = 2;   // the 4th-order difference: closure rows read 3 points, inside a halo of 2
constexpr int kFlH = 4;   // the 8th-order filter: closure rows read 7 points, inside a halo of 4

// dop() of lee_step.cu on a line held in shared memory: f points at the line's element for
// position `pos`, stride `st`.
template <typename T>
__device__ __forceinline__ T dop_sm(const OpTable& op, const T* f, int st, int pos, int n) {
  int c;
  if (pos >= op.h && pos <= n - 1 - op.h) c = 0;
  else if (pos < op.h) c = 1 + pos;
  else c = -(1 + (n - 1 - pos));
  T acc = T(0);
  if (c == 0) {
#pragma unroll
    for (int l = -op.h; l <= op.h; ++l) acc += T(op.c[l + op.h]) * f[l * st];
    return acc;
  }
  if (c > 0) {
    const int r = c - 1;
    const T* a = f - r * st;
    for (int s = 0; s < op.S; ++s) acc += T(op.B[r][s]) * a[s * st];
    return acc;
  }
  const int r = -c - 1;
  const T* a = f + r * st;
  for (int s = 0; s < op.S; ++s) acc += T(op.mfac * op.B[r][s]) * a[-s * st];
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

template <typename T, bool COMP, int TX, int TY>
__global__ void __launch_bounds__(TX* TY) k_batch_stage(const StageParams<T>* __restrict__ prm,
                                                        const int4* __restrict__ tiles, int ntiles) {
  constexpr int V = 4;
  constexpr int H = kFdH;
  constexpr int W = TX + 2 * H, R = TY + 2 * H;
  // J*metrics read per point where a block keeps them as fields (cval falls back to the
  // constant otherwise); uniform mean; summed sponge field
  constexpr int TR = kTrJmField | kTrUniform | kTrSponge;
  __shared__ __align__(16) StageParams<T> P;
  __shared__ T sm[V][R][W];
  __shared__ int cur;
  const int tid = threadIdx.x, nthr = TX * TY;
  const int tx = tid % TX, ty = tid / TX;
  if (tid == 0) cur = -1;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int4 td = tiles[t];
    __syncthreads();  // the previous tile's readers are done with P and sm
    if (td.x != cur) {
      copy_params(&P, prm + td.x, tid, nthr);
      __syncthreads();
      if (tid == 0) cur = td.x;
    }
    const int nx = P.nx, ny = P.ny, x0 = td.y, y0 = td.z;
    for (int q = tid; q < V * R * W; q += nthr) {
      const int v = q / (R * W), rr = (q / W) % R, cc = q % W;
      const int gx = x0 - H + cc, gy = y0 - H + rr;
      sm[v][rr][cc] = (gx >= 0 && gx < nx && gy >= 0 && gy < ny) ? P.zin[v][(long long)gy * nx + gx] : T(0);
    }
    __syncthreads();
    const int i = x0 + tx, j = y0 + ty;
    if (i < nx && j < ny) {
      const long long l = (long long)j * nx + i;
      PointIn<T, 2> in;
      gather<T, 2, COMP, TR>(P, l, in);
      T D[V][2], q[V];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const T* c0 = &sm[v][ty + H][tx + H];
        D[v][0] = dop_sm<T>(P.fd, c0, 1, i, nx);
        D[v][1] = dop_sm<T>(P.fd, c0, W, j, ny);
        q[v] = *c0;
      }
      rhs_update<T, 2, COMP, TR>(P, l, i, j, 0, D, q, in);
    }
  }
}

template <typename T, bool COMP, int TX, int TY>
__global__ void __launch_bounds__(TX* TY) k_batch_filter(const BatchFilterInst<T>* __restrict__ inst,
                                                         const int4* __restrict__ tiles, int ntiles, OpTable op,
                                                         T blend) {
  constexpr int V = 4;
  constexpr int H = kFlH;
  constexpr int W = TX + 2 * H, R = TY + 2 * H;
  extern __shared__ __align__(16) unsigned char dsm[];
  T* X = reinterpret_cast<T*>(dsm);              // [V][R][W]: pre-filter state with halo
  T* O = X + V * R * W;                          // [V][R][TX]: after the xi pass
  __shared__ __align__(16) BatchFilterInst<T> P;
  __shared__ int cur;
  const int tid = threadIdx.x, nthr = TX * TY;
  const int tx = tid % TX, ty = tid / TX;
  if (tid == 0) cur = -1;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int4 td = tiles[t];
    __syncthreads();
    if (td.x != cur) {
      copy_params(&P, inst + td.x, tid, nthr);
      __syncthreads();
      if (tid == 0) cur = td.x;
    }
    const int nx = P.nx, ny = P.ny, x0 = td.y, y0 = td.z;
    for (int q = tid; q < V * R * W; q += nthr) {
      const int v = q / (R * W), rr = (q / W) % R, cc = q % W;
      const int gx = x0 - H + cc, gy = y0 - H + rr;
      X[q] = (gx >= 0 && gx < nx && gy >= 0 && gy < ny) ? P.x[v][(long long)gy * nx + gx] : T(0);
    }
    __syncthreads();
    // xi pass on every row of the tile and its eta halo, tile columns only
    for (int q = tid; q < V * R * TX; q += nthr) {
      const int v = q / (R * TX), rr = (q / TX) % R, cc = q % TX;
      const int gx = x0 + cc, gy = y0 - H + rr;
      T o = T(0);
      if (gx < nx && gy >= 0 && gy < ny) {
        const T* f = X + ((long long)v * R + rr) * W + (cc + H);
        const T fx = dop_sm<T>(op, f, 1, gx, nx);
        o = COMP ? *f + fx : fx;  // compensated: the increment form, x + (F - I) x
      }
      O[q] = o;
    }
    __syncthreads();
    const int i = x0 + tx, j = y0 + ty;
    if (i < nx && j < ny) {
      const long long l = (long long)j * nx + i;
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const T* col = O + ((long long)v * R + (ty + H)) * TX + tx;
        const T fy = dop_sm<T>(op, col, TX, j, ny);
        const T xc = X[((long long)v * R + (ty + H)) * W + (tx + H)];
        if (!COMP) {
          P.y[v][l] = (T(1) - blend) * xc + blend * fy;
        } else {
          // the xi increment again at the centre (as the per-block first pass keeps it), then
          // y = y_pre + beta (D_xi + D_eta) + err as an exact two-float sum
          const T dx = dop_sm<T>(op, X + ((long long)v * R + (ty + H)) * W + (tx + H), 1, i, nx);
          const T dsum = dx + fy;
          const T tt = blend * dsum + P.err[v][l];
          const T s = xc + tt;
          const T bb = s - xc;
          const T e = (xc - (s - bb)) + (tt - bb);
          P.y[v][l] = s;
          P.comp[v][l] = e;
        }
      }
    }
  }
}

template <typename T, bool COMP, int TX, int TY>
cudaError_t go_stage(const StageParams<T>* prm, const int4* tiles, int ntiles, int grid, cudaStream_t s) {
  k_batch_stage<T, COMP, TX, TY><<<grid, TX * TY, 0, s>>>(prm, tiles, ntiles);
  return cudaGetLastError();
}

template <typename T, int TX, int TY>
size_t filter_smem() {
  return sizeof(T) * 4 * ((TY + 2 * kFlH) * (TX + 2 * kFlH) + (TY + 2 * kFlH) * TX);
}

template <typename T, bool COMP, int TX, int TY>
cudaError_t go_filter(const BatchFilterInst<T>* inst, const int4* tiles, int ntiles, int grid, const OpTable& op,
                      T blend, cudaStream_t s) {
  const size_t smem = filter_smem<T, TX, TY>();
  cudaError_t e = cudaFuncSetAttribute(k_batch_filter<T, COMP, TX, TY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  k_batch_filter<T, COMP, TX, TY><<<grid, TX * TY, smem, s>>>(inst, tiles, ntiles, op, blend);
  return cudaGetLastError();
}

template <typename T, bool COMP>
int occupancy_stage(int shape) {
  int n = 0;
  switch (shape) {
    case 0: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch_stage<T, COMP, 32, 8>, 256, 0); break;
    case 1: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch_stage<T, COMP, 64, 4>, 256, 0); break;
    case 2: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch_stage<T, COMP, 64, 8>, 512, 0); break;
    case 3: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch_stage<T, COMP, 32, 16>, 512, 0); break;
    default: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch_stage<T, COMP, 128, 4>, 512, 0); break;
  }
  return n > 0 ? n : 1;
}

}  // namespace

// Tile shapes, by index: 0 = 32x8, 1 = 64x4, 2 = 64x8, 3 = 32x16, 4 = 128x4 (stage and filter).
void batch_shape(int shape, int* tx, int* ty) {
  static const int s[5][2] = {{32, 8}, {64, 4}, {64, 8}, {32, 16}, {128, 4}};
  *tx = s[shape][0];
  *ty = s[shape][1];
}

template <typename T>
cudaError_t launch_batch_stage(const StageParams<T>* prm, const int4* tiles, int ntiles, int shape, int comp,
                               int grid, cudaStream_t s) {
  if (ntiles <= 0) return cudaSuccess;
  if (comp) {
    switch (shape) {
      case 0: return go_stage<T, true, 32, 8>(prm, tiles, ntiles, grid, s);
      case 1: return go_stage<T, true, 64, 4>(prm, tiles, ntiles, grid, s);
      case 2: return go_stage<T, true, 64, 8>(prm, tiles, ntiles, grid, s);
      case 3: return go_stage<T, true, 32, 16>(prm, tiles, ntiles, grid, s);
      default: return go_stage<T, true, 128, 4>(prm, tiles, ntiles, grid, s);
    }
  }
  switch (shape) {
    case 0: return go_stage<T, false, 32, 8>(prm, tiles, ntiles, grid, s);
    case 1: return go_stage<T, false, 64, 4>(prm, tiles, ntiles, grid, s);
    case 2: return go_stage<T, false, 64, 8>(prm, tiles, ntiles, grid, s);
    case 3: return go_stage<T, false, 32, 16>(prm, tiles, ntiles, grid, s);
    default: return go_stage<T, false, 128, 4>(prm, tiles, ntiles, grid, s);
  }
}

template <typename T>
cudaError_t launch_batch_filter(const BatchFilterInst<T>* inst, const int4* tiles, int ntiles, int shape, int comp,
                                int grid, const OpTable& op, double blend, cudaStream_t s) {
  if (ntiles <= 0) return cudaSuccess;
  const T b = (T)blend;
  if (comp) {
    switch (shape) {
      case 0: return go_filter<T, true, 32, 8>(inst, tiles, ntiles, grid, op, b, s);
      case 1: return go_filter<T, true, 64, 4>(inst, tiles, ntiles, grid, op, b, s);
      case 2: return go_filter<T, true, 64, 8>(inst, tiles, ntiles, grid, op, b, s);
      case 3: return go_filter<T, true, 32, 16>(inst, tiles, ntiles, grid, op, b, s);
      default: return go_filter<T, true, 128, 4>(inst, tiles, ntiles, grid, op, b, s);
    }
  }
  switch (shape) {
    case 0: return go_filter<T, false, 32, 8>(inst, tiles, ntiles, grid, op, b, s);
    case 1: return go_filter<T, false, 64, 4>(inst, tiles, ntiles, grid, op, b, s);
    case 2: return go_filter<T, false, 64, 8>(inst, tiles, ntiles, grid, op, b, s);
    case 3: return go_filter<T, false, 32, 16>(inst, tiles, ntiles, grid, op, b, s);
    default: return go_filter<T, false, 128, 4>(inst, tiles, ntiles, grid, op, b, s);
  }
}

template <typename T>
int batch_stage_occupancy(int shape, int comp) {
  return comp ? occupancy_stage<T, true>(shape) : occupancy_stage<T, false>(shape);
}

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

}  // namespace lee
