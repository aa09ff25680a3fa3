// TMA-staged stage and filter kernels (lee_tma.cu): declarations shared with the host.
#pragma once

#include <cuda.h>

#include "lee_internal.h"

namespace lee {

constexpr int kTileX = 32;  // points along i per CTA (one warp row)
constexpr int kTileY = 8;   // points along j per CTA
constexpr int kFdHalf = 2;  // the TMA stage kernel handles the 4th-order difference
constexpr int kFilterSlots = 4;  // planes in the filter kernel's ring (three in flight)

// One tensor map per state field of a buffer (passed as a __grid_constant__ parameter).
struct __align__(64) FieldMaps {
  CUtensorMap m[kMaxVars];
};

template <typename T>
struct TmaStageParams {
  StageParams<T> s;
  int tiles_x, k_chunk;
  // derivative weights by closure class: 0 interior, 1..2 left rows, 3..4 right rows, 5 zero
  // (a hole after a hole); offsets -2..2 from the point (the reference's stencil tables
  // rewritten per class). On a block with holes (s.code set) each point's class along each
  // direction comes from its closure code, else from its position.
  T w[6][5];
  int* err;  // set when a bounded wait gives up
  unsigned long long wait_ns;  // limit of the waits on staged data (the drains keep the default)
};

template <typename T>
struct TmaFilterParams {
  int nx, ny, nz, V, tiles_x, k_chunk;
  int nb;  // class rows per line end: class 0 interior, 1..nb from the left, nb+1..2nb from the right
  // filter weights by class (interior, left rows, right rows, then the zero class 1 + 2 nb of a
  // hole after a hole), offsets -hf..hf; the compensated form uses F - I
  T w[1 + 2 * kTE][11];
  // a block with holes: the filter's closure codes per direction (classes from them, not from
  // positions) and the hole mask of the output; null otherwise
  const int8_t* code[3];
  const int* iblank;
  T blend;
  const T* err[kMaxVars];  // compensated: rounding error of the pre-filter state
  T* out[kMaxVars];
  T* comp[kMaxVars];
  int* errflag;
  unsigned long long wait_ns;  // limit of the waits on staged data (the drains keep the default)
};

// Shared-memory box geometry: halo along i rounded up so every TMA row starts on 16 bytes;
// consecutive boxes in shared memory are FBP elements apart, a multiple of 128 bytes, because
// a cp.async.bulk.tensor destination must be 128-byte aligned.
// RY: rows of the tile per thread row (the tile is kTileY * RY rows high).
template <typename T, int H, int RY = 1>
struct Box {
  static constexpr int A = (int)(16 / sizeof(T));
  static constexpr int HX = ((H + A - 1) / A) * A;
  static constexpr int BX = kTileX + 2 * HX;
  static constexpr int BY = kTileY * RY + 2 * H;
  static constexpr int FB = BX * BY;
  static constexpr int FBP = (int)((((size_t)FB * sizeof(T) + 127) / 128) * 128 / sizeof(T));
  static_assert((FBP * sizeof(T)) % 128 == 0, "box stride must be a multiple of 128 bytes");
};

// Planes of prefetch in the stage kernel's ring (beyond the 2h+1 stencil planes).
template <typename T>
struct StagePrefetch {
  static constexpr int P = sizeof(T) == 4 ? 2 : 1;
};

size_t stage_tma_smem(int dim, size_t esz);
template <typename T>
cudaError_t launch_stage_tma(const FieldMaps& zin, const TmaStageParams<T>& p, int traits, int tiles, int chunks,
                             cudaStream_t s);
// ry: tile rows per thread row, 1 or 2 (the same arithmetic for every point either way)
template <typename T>
cudaError_t launch_filter_tma(const FieldMaps& in, const TmaFilterParams<T>& p, int hf, int dim, int comp, int ry,
                              int tiles, int chunks, cudaStream_t s);
// The compensated one-row fused filter with the input y_n and the last stage's increment (the
// kernel forms y_pre and its rounding error; same bits as the pair the last stage would write).
cudaError_t launch_filter_tma_inc(const FieldMaps& y, const FieldMaps& inc, const TmaFilterParams<float>& p, int hf,
                                  int dim, int tiles, int chunks, cudaStream_t s);
// The FP32 fused filter with two neighbouring points per thread along xi (lee_filter_pair.cu):
// 3-D blocks without holes of even nx, half-widths 2, 4 and 5; the compensated form gives the same
// bits as the one-row scalar filter. Its TMA box (bx x by) and tile (tx x ty), and the launch.
bool filter_pair_half_width(int hf);
void filter_pair_box(int hf, int* bx, int* by, int* tx, int* ty);
// comp: the compensated form, else the plain filter and blend (the adjoint's transposed filter).
cudaError_t launch_filter_pair(const FieldMaps& in, const TmaFilterParams<float>& p, int hf, int comp, int tiles,
                               int chunks, cudaStream_t s);
// The plane-marching adjoint stage (lee_adjoint_tma.cu): tensor maps of w (5 fields) then the
// nine J*metrics fields, and its parameters.
struct __align__(64) AdjMaps {
  CUtensorMap m[14];
};
template <typename T>
struct AdjTmaParams {
  AdjStageParams<T> a;
  int tiles_x, k_chunk;
  int* err;  // set when a bounded wait gives up
  unsigned long long wait_ns;  // limit of the waits on staged data (the drains keep the default)
};
void adj_tma_box(size_t esz, int* bx, int* by, int* tx, int* ty);
template <typename T>
cudaError_t launch_adj_tma(const AdjMaps& m, const AdjTmaParams<T>& p, bool jm_fields, int tiles, int chunks,
                           cudaStream_t s);

// The FP32 stage kernel with two points per thread (lee_stage_pair.cu): compensated form,
// uniform mean flow, TMA blocks of even width, a fixed stage kind.
bool stage_pair_applies(int traits, int nx);
cudaError_t launch_stage_pair(const FieldMaps& zin, const TmaStageParams<float>& p, int traits, int tiles, int chunks,
                              cudaStream_t s);

// The vectorised fused filter (lee_filter.cu): the group widths (points per thread) it offers for
// an element size, its TMA box (bx x by) and tile (tx x ty) for one width, and the launch.
int filter_vec_widths(size_t esz, int* px);
void filter_vec_box(size_t esz, int hf, int px, int* bx, int* by, int* tx, int* ty);
template <typename T>
cudaError_t launch_filter_vec(const FieldMaps& in, const TmaFilterParams<T>& p, int hf, int px, int dim, int tiles,
                              int chunks, cudaStream_t s);

}  // namespace lee
