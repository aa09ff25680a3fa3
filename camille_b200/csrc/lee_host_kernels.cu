// Kernel selection and launch: tensor maps of the TMA-staged kernels, the stage and filter
// launches of one block (TMA, two-point or generic), the plane-chunk autotuner, boundary-line
// and harmonic-wave updates, microphone traces, and the device error flag of the bounded waits.
#include <algorithm>
#include "lee_host.h"

using namespace lee;

namespace lee {

// Dimension-split filter of `in` (spatial::apply_filter, src/solver/spatial_discretization.cpp:2191-2246).
// The passes alternate between the two free buffers f0/f1; *result names the buffer that holds the
// filtered state. FP64: the last pass blends (1-beta) in + beta F(in). Compensated: `in` is y_pre, `err`
// its rounding error; the increments D = F - I are summed over the passes and the last pass writes
// y = y_pre + beta D + err as a two-float sum, its new rounding error going to comp_out.
template <typename T>
int run_filter(lee_ctx* c, BlockData& b, void** in, void** err, void** comp_out, void** f0, void** f1,
               void*** result) {
  int dims[3] = {b.nx, b.ny, b.nz};
  int passes[3], np = 0;
  for (int d = 0; d < c->cfg.num_dim; ++d)
    if (dims[d] > 1) passes[np++] = d;
  void** fr[2] = {f0, f1};
  void** src = in;
  for (int q = 0; q < np; ++q) {
    FilterParams<T> fp;
    memset(&fp, 0, sizeof fp);
    fp.nx = b.nx; fp.ny = b.ny; fp.nz = b.nz;
    fp.V = c->V;
    fp.dir = passes[q];
    fp.first = q == 0;
    fp.last = q == np - 1;
    fp.blend = (T)c->cfg.filter_blend;
    fp.code = b.has_holes ? b.d_code_flt[passes[q]] : nullptr;
    fp.iblank = b.has_holes ? b.d_iblank : nullptr;
    fp.op = c->comp ? c->fltd : c->flt;
    void** dst = fr[q % 2];
    for (int v = 0; v < c->V; ++v) {
      fp.in[v] = (const T*)src[v];
      fp.out[v] = (T*)dst[v];
      fp.y0[v] = (const T*)in[v];
      fp.dsum[v] = (T*)b.dsum[v];
      fp.dsum_in[v] = (const T*)b.dsum[v];
      fp.comp[v] = comp_out ? (T*)comp_out[v] : nullptr;
      fp.err[v] = err ? (const T*)err[v] : nullptr;
    }
    int e0 = mark(c);
    CK(launch_filter_pass<T>(fp, c->comp ? 1 : 0, c->stream));
    int e1 = mark(c);
    span(c, 1, e0, e1);
    c->stats.filter_launches += 1;
    c->stats.kernel_launches += 1;
    src = dst;
  }
  *result = np > 0 ? fr[(np - 1) % 2] : in;
  return LEE_OK;
}

void swap_fields(int V, void** a, void** b) {
  if (a == b) return;
  for (int v = 0; v < V; ++v) std::swap(a[v], b[v]);
}

int ensure_encoder(lee_ctx* c) {
  if (c->encode) return LEE_OK;
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
  if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
    return fail(c, LEE_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
  c->encode = reinterpret_cast<EncodeTiledFn>(fn);
  return LEE_OK;
}

// Tensor maps (box bx x by x 1) of n fields of a block, cached per device pointer.
int encode_maps(lee_ctx* c, const BlockData& b, const void* const* fields, int n, int bx, int by, CUtensorMap* out) {
  int rc = ensure_encoder(c);
  if (rc) return rc;
  for (int v = 0; v < n; ++v) {
    MapKey key{const_cast<void*>(fields[v]), bx, by};
    auto it = c->tmaps.find(key);
    if (it == c->tmaps.end()) {
      CUtensorMap m;
      cuuint64_t dims[3] = {(cuuint64_t)b.nx, (cuuint64_t)b.ny, (cuuint64_t)b.nz};
      cuuint64_t strides[2] = {(cuuint64_t)b.nx * c->esz, (cuuint64_t)b.nx * b.ny * c->esz};
      cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
      cuuint32_t es[3] = {1, 1, 1};
      CUresult r = c->encode(&m, c->esz == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                             const_cast<void*>(fields[v]), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      if (r != CUDA_SUCCESS) return fail(c, LEE_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
      MapBytes mb;
      memcpy(mb.b, &m, sizeof m);
      it = c->tmaps.emplace(key, mb).first;
    }
    memcpy(&out[v], it->second.b, sizeof(CUtensorMap));
  }
  return LEE_OK;
}

// Tensor maps of the V fields of a buffer.
int field_maps(lee_ctx* c, const BlockData& b, void* const* fields, int bx, int by, FieldMaps* out) {
  return encode_maps(c, b, const_cast<const void* const*>(fields), c->V, bx, by, out->m);
}

bool increment_step_applies(const lee_ctx* c, const BlockData& b) {
  if (!c->comp || !c->increment_step || c->batch.active || c->ovs.n > 0 || b.has_holes) return false;
  if (c->cfg.filter_scheme == LEE_FILTER_NONE || !b.tma || !b.tma_filter || b.filter_px > 0 || b.filter_ry != 1 ||
      b.filter_pair)
    return false;
  if (b.need_rho) return false;  // rho'/rho_bar is formed from y_pre after the last stage
  for (const auto& z : b.bnd)
    if (is_bc_line(z.kind)) return false;  // BC lines update y_pre after the last stage
  return true;
}

// Tile rows per thread row of a form of the scalar fused filter (1 or 2).
int filter_form_rows(int form) { return form == 2 ? 2 : 1; }

// The fused filter's box (tile of kTileX x kTileY * rows points with a halo of h) and its tiles.
int filter_box(const lee_ctx* c, int h, int form, int* bx, int* by) {
  const int A = (int)(16 / c->esz);
  const int hx = ((h + A - 1) / A) * A;
  *bx = kTileX + 2 * hx;
  *by = kTileY * filter_form_rows(form) + 2 * h;
  return LEE_OK;
}

int filter_tiles_form(const BlockData& b, int ry) {
  const int ty = kTileY * filter_form_rows(ry);
  return b.tiles_x * ((b.ny + ty - 1) / ty);
}

int filter_tiles(const BlockData& b) { return filter_tiles_form(b, b.filter_ry); }

// Tiles of the vectorised filter at the block's group width, and of the two-point filter.
void set_filter_tiles(const lee_ctx* c, BlockData& b) {
  if (b.filter_pair_ok) {
    int bx, by, tx, ty;
    filter_pair_box(c->hf, &bx, &by, &tx, &ty);
    b.ptiles_x = (b.nx + tx - 1) / tx;
    b.ptiles_y = (b.ny + ty - 1) / ty;
  }
  if (b.filter_px <= 0) return;
  int bx, by, tx, ty;
  filter_vec_box(c->esz, c->hf, b.filter_px, &bx, &by, &tx, &ty);
  b.vtiles_x = (b.nx + tx - 1) / tx;
  b.vtiles_y = (b.ny + ty - 1) / ty;
}

template <typename T>
int launch_stage_any(lee_ctx* c, BlockData& b, const StageParams<T>& p, void* const* zin, int chunk_override) {
  if (!b.tma) {
    CK(launch_stage<T>(p, c->comp ? 1 : 0, c->stream));
    return LEE_OK;
  }
  TmaStageParams<T> tp;
  memset(&tp, 0, sizeof tp);
  tp.s = p;
  tp.tiles_x = b.tiles_x;
  tp.k_chunk = chunk_override ? chunk_override : b.stage_chunk;
  for (int a = 0; a < 6; ++a)
    for (int o = 0; o < 5; ++o) tp.w[a][o] = (T)c->wst[a][o];
  tp.err = c->d_err;
  tp.wait_ns = c->wait_ns;
  FieldMaps fm;
  int rc = field_maps(c, b, zin, Box<T, kFdHalf>::BX, Box<T, kFdHalf>::BY, &fm);
  if (rc) return rc;
  const int chunks = c->cfg.num_dim == 3 ? (b.nz + tp.k_chunk - 1) / tp.k_chunk : 1;
  // the stage's kind selects a specialised kernel; a first stage that is also the last (no
  // such tableau here) reads p.stage and p.last at run time
  const int kind = p.stage < 0 ? kKindRhs
                   : p.stage == 0 ? (p.last ? kKindRuntime : kKindFirst)
                                  : (p.last ? (p.increment ? kKindLastIncrement : kKindLast) : kKindMid);
  const int tr = b.traits | (kind << kKindShift);
  if constexpr (sizeof(T) == 4) {
    if (b.stage_px == 2 && stage_pair_applies(tr, b.nx)) {
      CK(launch_stage_pair(fm, tp, tr, b.tiles_x * b.tiles_y, chunks, c->stream));
      return LEE_OK;
    }
  }
  CK(launch_stage_tma<T>(fm, tp, tr, b.tiles_x * b.tiles_y, chunks, c->stream));
  return LEE_OK;
}

// Fused filter (all directions, one read and one write of the state): in -> out.
template <typename T>
int launch_filter_fused(lee_ctx* c, BlockData& b, void* const* in, void* const* err, void* const* out,
                        void* const* comp_out, int chunk_override, void* const* inc) {
  TmaFilterParams<T> fp;
  memset(&fp, 0, sizeof fp);
  fp.nx = b.nx; fp.ny = b.ny; fp.nz = b.nz;
  fp.V = c->V;
  fp.tiles_x = b.tiles_x;
  fp.k_chunk = chunk_override ? chunk_override : b.filter_chunk;
  fp.nb = c->hf;
  for (int a = 0; a < 12; ++a)
    for (int o = 0; o < 11; ++o) fp.w[a][o] = (T)c->wfl[a][o];
  if (b.has_holes) {
    for (int d = 0; d < 3; ++d) fp.code[d] = b.d_code_flt[d];
    fp.iblank = b.d_iblank;
  }
  fp.blend = (T)c->cfg.filter_blend;
  for (int v = 0; v < c->V; ++v) {
    fp.err[v] = err ? (const T*)err[v] : nullptr;
    fp.out[v] = (T*)out[v];
    fp.comp[v] = comp_out ? (T*)comp_out[v] : nullptr;
  }
  fp.errflag = c->d_err;
  fp.wait_ns = c->wait_ns;
  int bx, by, tx, ty;
  const bool pair = b.filter_pair && !inc;
  if (pair) {
    filter_pair_box(c->hf, &bx, &by, &tx, &ty);
    fp.tiles_x = b.ptiles_x;
  } else if (b.filter_px > 0) {
    filter_vec_box(c->esz, c->hf, b.filter_px, &bx, &by, &tx, &ty);
    fp.tiles_x = b.vtiles_x;
  } else {
    filter_box(c, c->hf, b.filter_ry, &bx, &by);
  }
  FieldMaps fm;
  int rc = field_maps(c, b, in, bx, by, &fm);
  if (rc) return rc;
  const int chunks = c->cfg.num_dim == 3 ? (b.nz + fp.k_chunk - 1) / fp.k_chunk : 1;
  FieldMaps im;
  if (inc && (rc = field_maps(c, b, inc, bx, by, &im))) return rc;
  int e0 = mark(c);
  if (inc) {
    if constexpr (sizeof(T) == 4) {
      CK(launch_filter_tma_inc(fm, im, fp, c->hf, c->cfg.num_dim, filter_tiles(b), chunks, c->stream));
    } else {
      return fail(c, LEE_ERR_UNSUPPORTED, "the increment step is the compensated form's");
    }
  } else if (pair) {
    if constexpr (sizeof(T) == 4) {
      CK(launch_filter_pair(fm, fp, c->hf, 1, b.ptiles_x * b.ptiles_y, chunks, c->stream));
    } else {
      return fail(c, LEE_ERR_UNSUPPORTED, "the two-point filter is the compensated form's");
    }
  } else if (b.filter_px > 0) {
    CK(launch_filter_vec<T>(fm, fp, c->hf, b.filter_px, c->cfg.num_dim, b.vtiles_x * b.vtiles_y, chunks, c->stream));
  } else {
    CK(launch_filter_tma<T>(fm, fp, c->hf, c->cfg.num_dim, c->comp ? 1 : 0, b.filter_ry, filter_tiles(b), chunks,
                            c->stream));
  }
  int e1 = mark(c);
  span(c, 1, e0, e1);
  c->stats.filter_launches += 1;
  c->stats.kernel_launches += 1;
  return LEE_OK;
}

// Pick the k-chunk (planes marched by one CTA) of the stage and filter kernels by timing
// the candidates on this block: short chunks give more CTAs, long chunks re-load fewer
// halo planes. Runs at setup on the (not yet uploaded) state buffers.
template <typename T>
int autotune(lee_ctx* c, BlockData& b) {
  if (!b.tma && !b.tma_filter) return LEE_OK;
  const bool d3 = c->cfg.num_dim == 3;
  // plane chunks: a fixed ladder (stage kernels), and for the filter also the near-equal splits
  // of the block's planes into 1..24 chunks (ceil(nz / c): every chunk but the last of the same
  // length, so that CTA counts that fill whole waves of the GPU are among the candidates)
  const std::vector<int> ladder = {8, 16, 24, 32, 48, 64, 96, 128, 192, 256};
  std::vector<int> splits = ladder;
  for (int q = 1; q <= 24; ++q) splits.push_back((b.nz + q - 1) / q);
  std::sort(splits.begin(), splits.end());
  splits.erase(std::unique(splits.begin(), splits.end()), splits.end());
  const std::vector<int> cands2 = {1};
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  const bool saved = c->timing;
  c->timing = false;
  // the kernels are fixed at this point (lee_set_stage_kernel, lee_set_filter_kernel or the
  // defaults); only the plane chunk, which leaves the arithmetic unchanged, is timed
  const int kinds[1] = {b.filter_px}, nkinds = 1;
  const int skinds[1] = {b.stage_px}, nskinds = 1;
  for (int which = 0; which < 2; ++which) {
    if ((which == 0 && !b.tma) || (which == 1 && !b.tma_filter)) continue;
    if (which == 0 && !d3 && nskinds == 1) continue;  // nothing to choose
    float best = 1e30f;
    int best_chunk = b.nz, best_kind = which == 0 ? b.stage_px : b.filter_px, best_ry = b.filter_ry;
    bool best_pair = b.filter_pair;
    // the best scalar form (one or two rows) and its chunk, kept for the transposed filter of
    // the adjoint, which the two-point kernel does not run
    float best_scalar = 1e30f;
    int best_scalar_chunk = b.nz, best_scalar_ry = b.filter_ry;
    // the scalar filter's forms (1: one tile row per thread row, 2: two rows, 3: two points per
    // thread) are timed with the chunk: each point's arithmetic is the same in all three
    const int nry = which == 1 && c->filter_form == 0 ? 3 : 1;
    for (int kq = 0; kq < (which == 1 ? nkinds : nskinds) * nry; ++kq) {
      if (which == 0) {
        b.stage_px = skinds[kq];
      } else {
        b.filter_px = kinds[kq / nry];
        const int form = c->filter_form > 0 ? c->filter_form : 1 + kq % nry;
        // the one-row form alone takes holes and the increment step's input (a form set by
        // lee_set_filter_form is kept, and the increment step then does not apply)
        if (c->filter_form == 0 && (b.filter_px > 0 || b.has_holes || (c->comp && c->increment_step)) && form > 1)
          continue;
        if (form == 3 && !b.filter_pair_ok) continue;
        b.filter_ry = form == 2 ? 2 : 1;
        b.filter_pair = form == 3;
        set_filter_tiles(c, b);
      }
      for (int ch : (d3 ? (which == 1 ? splits : ladder) : cands2)) {
        if (d3 && ch > b.nz) continue;
        float tsum = 0.f;
        for (int rep = 0; rep < 4; ++rep) {  // the first run warms up
          CK(cudaEventRecord(e0, c->stream));
          int rc;
          if (which == 0) {
            StageParams<T> p;
            fill_stage_common<T>(c, b, p);
            p.stage = 1;
            p.last = 0;
            p.h = (T)1e-3;
            p.b = (T)(1.0 / 3.0);
            p.a = (T)0.5;
            for (int v = 0; v < c->V; ++v) {
              p.zin[v] = (const T*)b.zb[0][v];
              p.yn[v] = (const T*)b.y[v];
              p.acc[v] = (T*)b.acc[v];
              p.zout[v] = (T*)b.zb[1][v];
              p.comp[v] = (T*)b.comp[v];
            }
            rc = launch_stage_any<T>(c, b, p, b.zb[0], d3 ? ch : 0);
          } else {
            const int chunk = d3 ? ch : 0;
            rc = c->comp ? launch_filter_fused<T>(c, b, b.zb[1], b.acc, b.zb[0], b.comp, chunk)
                         : launch_filter_fused<T>(c, b, b.acc, nullptr, b.zb[0], nullptr, chunk);
          }
          if (rc) return rc;
          CK(cudaEventRecord(e1, c->stream));
          CK(cudaEventSynchronize(e1));
          float ms = 0.f;
          CK(cudaEventElapsedTime(&ms, e0, e1));
          if (rep > 0) tsum += ms;
        }
        if (which == 1 && !b.filter_pair && tsum < best_scalar) {
          best_scalar = tsum;
          best_scalar_chunk = d3 ? ch : b.nz;
          best_scalar_ry = b.filter_ry;
        }
        if (tsum < best) {
          best = tsum;
          best_chunk = d3 ? ch : b.nz;
          best_kind = which == 0 ? b.stage_px : b.filter_px;
          best_ry = b.filter_ry;
          best_pair = b.filter_pair;
        }
      }
    }
    if (which == 0) {
      b.stage_chunk = best_chunk;
      b.stage_px = best_kind;
    } else {
      b.filter_chunk = best_chunk;
      b.filter_px = best_kind;
      b.filter_ry = best_ry;
      b.filter_pair = best_pair;
      b.tfilter_chunk = best_scalar < 1e30f ? best_scalar_chunk : best_chunk;
      b.tfilter_ry = best_scalar < 1e30f ? best_scalar_ry : (best_pair ? 1 : best_ry);
      set_filter_tiles(c, b);
    }
  }
  c->timing = saved;
  c->stats = lee_stats{};
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return check_device_error(c);
}

int check_device_error(lee_ctx* c) {
  int h[2] = {0, 0};
  CK(cudaMemcpyAsync(h, c->d_err, sizeof h, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (h[0] || h[1]) {
    CK(cudaMemsetAsync(c->d_err, 0, sizeof h, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (h[0]) return fail(c, LEE_ERR_TIMEOUT, "a bounded wait on a TMA transfer gave up (device flag %d)", h[0]);
    return fail(c, LEE_ERR_NONFINITE, "the state holds a non-finite value after step %d", c->step);
  }
  return LEE_OK;
}

// The non-finite sentinel: every value of the state is checked (the carried rounding error of
// the compensated form follows the state); any NaN or infinity sets d_err[1].
int check_finite(lee_ctx* c) {
  for (auto& b : c->blk) CK(launch_nonfinite(c->stream, b.N, c->V, c->esz, b.y, nullptr, c->d_err + 1));
  return LEE_OK;
}

// The launch parameters of one BC line on the fields f (e: the errors of a compensated pair);
// the update's time is the caller's.
template <typename T>
void fill_bc_params(lee_ctx* c, const BlockData& b, const Boundary& z, void** f, void** e, BcParams<T>& p) {
  memset(&p, 0, sizeof p);
  p.kind = z.kind; p.dir = z.dir; p.end = z.end;
  p.nd = c->cfg.num_dim; p.V = c->V;
  for (int d = 0; d < 3; ++d) {
    p.lo[d] = z.lo[d];
    p.nb[d] = z.hi[d] - z.lo[d] + 1;
  }
  p.lo[z.dir] = z.end == 0 ? z.lo[z.dir] : z.hi[z.dir];
  p.nb[z.dir] = 1;
  p.nx = b.nx; p.ny = b.ny;
  p.sd = z.dir == 0 ? 1 : z.dir == 1 ? (long long)b.nx : (long long)b.nx * b.ny;
  p.S = c->fd.S;
  for (int q = 0; q < c->fd.S; ++q) p.c0[q] = c->fd.B[0][q];
  for (int v = 0; v < c->V; ++v) {
    p.y[v] = (T*)f[v];
    p.e[v] = e ? (T*)e[v] : nullptr;
  }
  for (int q = 0; q < 9; ++q) { p.met[q] = b.d_met[q]; p.minv[q] = b.d_minv[q]; }
  p.jac = b.d_jac;
  p.iblank = b.has_holes ? b.d_iblank : nullptr;
  p.wave = c->wave;
  for (int d = 0; d < 3; ++d) p.xyz[d] = b.d_xyz[d];
}

// Every BC line of a block, in the order they were added, on the fields f (with the
// rounding errors e of a compensated pair, or null).
template <typename T>
int apply_bcs(lee_ctx* c, BlockData& b, void** f, void** e, double t, const double* t_tab, const int* ctr,
              int t_stride) {
  for (auto& z : b.bnd) {
    if (!is_bc_line(z.kind)) continue;
    BcParams<T> p;
    fill_bc_params<T>(c, b, z, f, e, p);
    p.t = t;
    p.t_tab = t_tab;
    p.ctr = ctr;
    p.t_stride = t_stride;
    CK(launch_bc<T>(p, c->stream));
    c->stats.kernel_launches += 1;
  }
  return LEE_OK;
}

// The reference states of the block's harmonic-wave sponge zones at a stage's time (t, or in a
// replayed step graph t_tab[*ctr * t_stride]), read by the stage kernel's zone loop.
template <typename T>
int wave_refs(lee_ctx* c, BlockData& b, double t, const double* t_tab, const int* ctr, int t_stride) {
  for (auto& z : b.bnd) {
    if (z.kind != LEE_SPONGE_FREUND_HARMONICWAVE) continue;
    WaveRefParams<T> p;
    memset(&p, 0, sizeof p);
    for (int d = 0; d < 3; ++d) {
      p.lo[d] = z.lo[d];
      p.nb[d] = z.hi[d] - z.lo[d] + 1;
    }
    p.nx = b.nx; p.ny = b.ny;
    p.nd = c->cfg.num_dim; p.V = c->V;
    p.wave = c->wave;
    for (int d = 0; d < 3; ++d) p.xyz[d] = b.d_xyz[d];
    p.iblank = b.has_holes ? b.d_iblank : nullptr;
    p.t = t;
    p.t_tab = t_tab;
    p.ctr = ctr;
    p.t_stride = t_stride;
    p.out = (T*)z.d_ref;
    CK(launch_wave_ref<T>(p, c->stream));
    c->stats.kernel_launches += 1;
  }
  return LEE_OK;
}

// p' at the microphones after a step (the objective's trace), in FP64.
template <typename T>
int trace_step(lee_ctx* c, const int* ctr) {
  if (!c->adj.trace_on) return LEE_OK;
  BlockData& b = c->blk[(size_t)c->adj.mic_block];
  const int P = c->V - 1;
  CK(launch_trace<T>((int)c->adj.mic.size(), c->adj.d_mic, (const T*)b.y[P], c->comp ? (const T*)b.comp[P] : nullptr,
                     c->adj.d_trace, ctr, ctr ? c->adj.d_base : nullptr, c->adj.host_row, c->stream));
  c->stats.kernel_launches += 1;
  if (!ctr) c->adj.host_row += 1;
  return LEE_OK;
}

// the host translation units use both precisions
template int run_filter<float>(lee_ctx* c, BlockData& b, void** in, void** err, void** comp_out, void** f0, void** f1,
               void*** result);
template int run_filter<double>(lee_ctx* c, BlockData& b, void** in, void** err, void** comp_out, void** f0, void** f1,
               void*** result);
template int launch_stage_any<float>(lee_ctx* c, BlockData& b, const StageParams<float>& p, void* const* zin, int chunk_override);
template int launch_stage_any<double>(lee_ctx* c, BlockData& b, const StageParams<double>& p, void* const* zin, int chunk_override);
template int launch_filter_fused<float>(lee_ctx* c, BlockData& b, void* const* in, void* const* err, void* const* out,
                        void* const* comp_out, int chunk_override, void* const* inc);
template int launch_filter_fused<double>(lee_ctx* c, BlockData& b, void* const* in, void* const* err, void* const* out,
                        void* const* comp_out, int chunk_override, void* const* inc);
template int autotune<float>(lee_ctx* c, BlockData& b);
template int autotune<double>(lee_ctx* c, BlockData& b);
template void fill_bc_params<float>(lee_ctx*, const BlockData&, const Boundary&, void**, void**, BcParams<float>&);
template void fill_bc_params<double>(lee_ctx*, const BlockData&, const Boundary&, void**, void**, BcParams<double>&);
template int apply_bcs<float>(lee_ctx* c, BlockData& b, void** f, void** e, double t, const double* t_tab, const int* ctr,
              int t_stride);
template int apply_bcs<double>(lee_ctx* c, BlockData& b, void** f, void** e, double t, const double* t_tab, const int* ctr,
              int t_stride);
template int wave_refs<float>(lee_ctx* c, BlockData& b, double t, const double* t_tab, const int* ctr, int t_stride);
template int wave_refs<double>(lee_ctx* c, BlockData& b, double t, const double* t_tab, const int* ctr, int t_stride);
template int trace_step<float>(lee_ctx* c, const int* ctr);
template int trace_step<double>(lee_ctx* c, const int* ctr);

}  // namespace lee
