// Batches of independent 2-D blocks (lee_advance_blocks): eligibility, the strip work lists,
// per-block stage parameters and the batched stage and filter launches of one step.
#include "lee_host.h"

using namespace lee;

namespace lee {

// ---- batches of independent 2-D blocks ----------------------------------------------------

// Blocks the batched kernels cover: 2-D, uniform mean, no holes,
// BC lines or overset (sponges allowed), the 4th-order difference and the 8th-order filter.
// Every nonzero closure weight of row r lies within h points of the row's own point (the batched
// kernels stage h points of halo and skip zero weights).
bool closures_within_halo(const OpTable& op) {
  for (int r = 0; r < op.h; ++r)
    for (int s = 0; s < op.S; ++s)
      if (op.B[r][s] != 0.0 && std::abs(s - r) > op.h) return false;
  return true;
}

bool batch_eligible(const lee_ctx* c) {
  if (c->cfg.num_dim != 2 || c->ovs.n > 0 || c->axisym || c->nsc > 0) return false;
  if (!(c->fd.h == 2 && c->fd.S == 3)) return false;
  if (c->cfg.filter_scheme != LEE_FILTER_STANDARD_CENTRAL || c->cfg.filter_order != 8) return false;
  if (!(c->flt.h == 4 && c->flt.S == 7 && c->fltd.h == 4 && c->fltd.S == 7)) return false;
  if (!closures_within_halo(c->fd) || !closures_within_halo(c->flt) || !closures_within_halo(c->fltd)) return false;
  for (auto& b : c->blk) {
    if (b.has_iblank || b.need_rho) return false;
    for (auto& z : b.bnd)
      if (z.kind != LEE_SPONGE_FREUND_AMBIENT) return false;
    auto is_const = [&](const Coef<double>& d, const Coef<float>& f) { return c->comp ? !f.p : !d.p; };
    auto is_zero = [&](const Coef<double>& d, const Coef<float>& f) { return c->comp ? f.zero != 0 : d.zero != 0; };
    bool uni = is_const(b.cd_pb, b.cf_pb) && is_const(b.cd_rbi, b.cf_rbi);
    for (int q = 0; q < 3; ++q)
      uni = uni && is_const(b.cd_ub[q], b.cf_ub[q]) && is_zero(b.cd_gs[q], b.cf_gs[q]) && is_zero(b.cd_gp[q], b.cf_gp[q]);
    for (int q = 0; q < 9; ++q) uni = uni && is_zero(b.cd_gu[q], b.cf_gu[q]);
    if (!uni) return false;
  }
  return true;
}

// Work items of a shape: (block, x0, ys, ye) strips of tx columns and ty rows.
std::vector<int4> batch_tiles(const lee_ctx* c, int shape) {
  int tx, ty;
  batch_shape(shape, &tx, &ty);
  std::vector<int4> t;
  for (size_t b = 0; b < c->blk.size(); ++b)
    for (int x0 = 0; x0 < c->blk[b].nx; x0 += tx)
      for (int y0 = 0; y0 < c->blk[b].ny; y0 += ty)
        t.push_back(make_int4((int)b, x0, y0, std::min(y0 + ty, c->blk[b].ny)));
  return t;
}

// The stage parameters of every block for every stage, [stage][block]: `stage_override` >= 0
// builds right-hand-side-only parameters (the autotuner's harmless launches).
template <typename T>
std::vector<StageParams<T>> batch_params(lee_ctx* c, const std::vector<double>& dts, bool graph, int rhs_only) {
  const Tableau tb = tableau(c->cfg.rk_scheme);
  const int ns = tb.ns, nbk = (int)c->blk.size();
  std::vector<StageParams<T>> out((size_t)ns * nbk);
  const bool src = c->src_kind != LEE_SOURCE_NONE;
  for (int s = 0; s < ns; ++s)
    for (int q = 0; q < nbk; ++q) {
      BlockData& b = c->blk[(size_t)q];
      StageParams<T>& p = out[(size_t)s * nbk + q];
      fill_stage_common<T>(c, b, p);
      const double dt = dts[(size_t)q];
      p.stage = rhs_only ? -1 : s;
      p.last = s == ns - 1;
      p.h = (T)dt;
      p.b = (T)tb.b[s];
      p.a = (T)tb.a[s];
      p.src_amp = (T)(src ? source_amp(c, b, b.time + tb.c[s] * dt) : 0.0);
      if (graph && src) {
        p.amp_tab = (const T*)c->graph.d_amp + (size_t)q * ns;
        p.step_ctr = c->graph.d_ctr;
        p.nstages = nbk * ns;
      }
      void** zin = s == 0 ? b.y : b.zb[(s + 1) % 2];
      void** zout = rhs_only ? b.zb[0] : b.zb[s % 2];
      if (rhs_only) zin = b.y;
      for (int v = 0; v < c->V; ++v) {
        p.zin[v] = (const T*)zin[v];
        p.yn[v] = (const T*)b.y[v];
        p.acc[v] = (T*)b.acc[v];
        p.zout[v] = (T*)zout[v];
        p.comp[v] = (T*)b.comp[v];
      }
      p.rho_prev = nullptr;
    }
  return out;
}

// Filter operands of every block; `scratch` sends the outputs to buffers that are free between
// steps (the autotuner's harmless launches).
template <typename T>
std::vector<BatchFilterInst<T>> batch_filter_inst(lee_ctx* c, bool scratch) {
  const Tableau tb = tableau(c->cfg.rk_scheme);
  std::vector<BatchFilterInst<T>> out;
  for (auto& b : c->blk) {
    BatchFilterInst<T> f;
    memset(&f, 0, sizeof f);
    f.nx = b.nx;
    f.ny = b.ny;
    void** last_out = b.zb[(tb.ns - 1) % 2];
    void** other = b.zb[tb.ns % 2];
    for (int v = 0; v < c->V; ++v) {
      f.x[v] = (const T*)(c->comp ? last_out[v] : b.acc[v]);
      f.err[v] = c->comp ? (const T*)b.acc[v] : nullptr;
      f.y[v] = (T*)(scratch ? other[v] : b.y[v]);
      f.comp[v] = c->comp ? (T*)(scratch ? b.dsum[v] : b.comp[v]) : nullptr;
    }
    out.push_back(f);
  }
  return out;
}

template <typename T>
int batch_launch_stage(lee_ctx* c, const void* prm, const int4* tiles, int nt, int shape, int grid) {
  CK(launch_batch_stage<T>((const StageParams<T>*)prm, tiles, nt, shape, c->comp ? 1 : 0, grid, c->stream));
  return LEE_OK;
}

template <typename T>
int batch_launch_filter(lee_ctx* c, const void* inst, const int4* tiles, int nt, int shape, int grid) {
  CK(launch_batch_filter<T>((const BatchFilterInst<T>*)inst, tiles, nt, shape, c->comp ? 1 : 0, grid,
                            c->comp ? c->fltd : c->flt, c->cfg.filter_blend, c->stream));
  return LEE_OK;
}

// Setup of the batched path at lee_prepare: operand arrays, sponge fields, and the tile shapes
// of the stage and filter launches picked by timing every candidate (right-hand-side-only
// stage launches and filter launches into scratch buffers, so the state is left alone).
template <typename T>
int batch_setup(lee_ctx* c) {
  auto& bt = c->batch;
  const int nbk = (int)c->blk.size();
  const Tableau tb = tableau(c->cfg.rk_scheme);
  int rc;
  for (auto& b : c->blk)
    if (!b.d_sigma_field && (rc = build_sigma_field(c, b))) return rc;
  const size_t pbytes = sizeof(StageParams<T>) * (size_t)tb.ns * nbk;
  if ((rc = dev_alloc(c, &bt.d_prm_graph, pbytes)) || (rc = dev_alloc(c, &bt.d_prm_direct, pbytes))) return rc;
  std::vector<BatchFilterInst<T>> fi = batch_filter_inst<T>(c, false);
  if ((rc = dev_alloc(c, &bt.d_finst, fi.size() * sizeof(fi[0])))) return rc;
  CK(cudaMemcpyAsync(bt.d_finst, fi.data(), fi.size() * sizeof(fi[0]), cudaMemcpyHostToDevice, c->stream));
  // scratch operands for the timing runs
  const std::vector<double> dts((size_t)nbk, 1e-3);
  std::vector<StageParams<T>> pr = batch_params<T>(c, dts, false, 1);
  std::vector<BatchFilterInst<T>> fs = batch_filter_inst<T>(c, true);
  void *d_pr = nullptr, *d_fs = nullptr;
  int4* d_t = nullptr;
  CK(cudaMalloc(&d_pr, pr.size() * sizeof(pr[0])));
  CK(cudaMalloc(&d_fs, fs.size() * sizeof(fs[0])));
  CK(cudaMemcpy(d_pr, pr.data(), pr.size() * sizeof(pr[0]), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_fs, fs.data(), fs.size() * sizeof(fs[0]), cudaMemcpyHostToDevice));
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->cfg.device);
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  float best_s = 1e30f, best_f = 1e30f;
  std::vector<int4> tiles_s, tiles_f;
  for (int shape = 0; shape < kBatchShapes; ++shape) {
    std::vector<int4> t = batch_tiles(c, shape);
    CK(cudaMalloc(&d_t, t.size() * sizeof(int4)));
    CK(cudaMemcpy(d_t, t.data(), t.size() * sizeof(int4), cudaMemcpyHostToDevice));
    const int nt = (int)t.size();
    const int gs = std::min(nt, nsm * batch_stage_occupancy<T>(shape, c->comp ? 1 : 0));
    // (the filter's CTAs each take a share of the items for some of the four fields)
    const int gf = std::min(4 * nt, nsm * batch_filter_occupancy<T>(shape, c->comp ? 1 : 0));
    float ms_s = 0.f, ms_f = 0.f;
    for (int pass = 0; pass < 2; ++pass) {  // the first pass warms up
      CK(cudaEventRecord(e0, c->stream));
      for (int r = 0; r < 3; ++r)
        if ((rc = batch_launch_stage<T>(c, (const StageParams<T>*)d_pr + nbk, d_t, nt, shape, gs))) return rc;
      CK(cudaEventRecord(e1, c->stream));
      CK(cudaEventSynchronize(e1));
      CK(cudaEventElapsedTime(&ms_s, e0, e1));
      CK(cudaEventRecord(e0, c->stream));
      for (int r = 0; r < 3; ++r)
        if ((rc = batch_launch_filter<T>(c, d_fs, d_t, nt, shape, gf))) return rc;
      CK(cudaEventRecord(e1, c->stream));
      CK(cudaEventSynchronize(e1));
      CK(cudaEventElapsedTime(&ms_f, e0, e1));
    }
    if (ms_s < best_s) {
      best_s = ms_s;
      bt.sshape = shape;
      bt.sgrid = gs;
      tiles_s = t;
    }
    if (ms_f < best_f) {
      best_f = ms_f;
      bt.fshape = shape;
      bt.fgrid = gf;
      tiles_f = t;
    }
    CK(cudaFree(d_t));
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  CK(cudaFree(d_pr));
  CK(cudaFree(d_fs));
  if ((rc = dalloc(c, &bt.d_stiles, tiles_s.size())) || (rc = dalloc(c, &bt.d_ftiles, tiles_f.size()))) return rc;
  CK(cudaMemcpy(bt.d_stiles, tiles_s.data(), tiles_s.size() * sizeof(int4), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(bt.d_ftiles, tiles_f.data(), tiles_f.size() * sizeof(int4), cudaMemcpyHostToDevice));
  bt.nst = (int)tiles_s.size();
  bt.nft = (int)tiles_f.size();
  // the timing runs wrote right-hand sides and filtered values into scratch buffers only
  bt.active = true;
  return LEE_OK;
}

// One batched step (see step_impl): ns stage launches and one filter launch for every block.
template <typename T>
int batch_step(lee_ctx* c, const std::vector<double>& dts, bool graph) {
  auto& bt = c->batch;
  const Tableau tb = tableau(c->cfg.rk_scheme);
  const int nbk = (int)c->blk.size();
  const void* prm = bt.d_prm_graph;
  if (!graph) {
    std::vector<StageParams<T>> pr = batch_params<T>(c, dts, false, 0);
    CK(cudaMemcpyAsync(bt.d_prm_direct, pr.data(), pr.size() * sizeof(pr[0]), cudaMemcpyHostToDevice, c->stream));
    prm = bt.d_prm_direct;
  }
  if (bt.pshape >= 0) {
    // the whole step in one persistent launch (stages and filter separated by grid barriers)
    int e0 = mark(c);
    CK(launch_batch_step<T>((const StageParams<T>*)prm, nbk, tb.ns, (const BatchFilterInst<T>*)bt.d_finst, bt.d_ptiles,
                            bt.npt, bt.pshape, c->comp ? 1 : 0, c->comp ? c->fltd : c->flt, c->cfg.filter_blend,
                            bt.d_gbar, c->d_err,
                            c->wait_ns, c->stream));
    int e1 = mark(c);
    span(c, 0, e0, e1);
    c->stats.stage_launches += 1;
    c->stats.kernel_launches += 1;
    return LEE_OK;
  }
  for (int s = 0; s < tb.ns; ++s) {
    int e0 = mark(c);
    int rc = batch_launch_stage<T>(c, (const StageParams<T>*)prm + (size_t)s * nbk, bt.d_stiles, bt.nst, bt.sshape,
                                   bt.sgrid);
    if (rc) return rc;
    int e1 = mark(c);
    span(c, 0, e0, e1);
    c->stats.stage_launches += 1;
    c->stats.kernel_launches += 1;
  }
  int e0 = mark(c);
  int rc = batch_launch_filter<T>(c, bt.d_finst, bt.d_ftiles, bt.nft, bt.fshape, bt.fgrid);
  if (rc) return rc;
  int e1 = mark(c);
  span(c, 1, e0, e1);
  c->stats.filter_launches += 1;
  c->stats.kernel_launches += 1;
  return LEE_OK;
}

// the host translation units use both precisions
template std::vector<StageParams<float>> batch_params<float>(lee_ctx* c, const std::vector<double>& dts, bool graph, int rhs_only);
template std::vector<StageParams<double>> batch_params<double>(lee_ctx* c, const std::vector<double>& dts, bool graph, int rhs_only);
template std::vector<BatchFilterInst<float>> batch_filter_inst<float>(lee_ctx* c, bool scratch);
template std::vector<BatchFilterInst<double>> batch_filter_inst<double>(lee_ctx* c, bool scratch);
template int batch_setup<float>(lee_ctx* c);
template int batch_setup<double>(lee_ctx* c);
template int batch_step<float>(lee_ctx* c, const std::vector<double>& dts, bool graph);
template int batch_step<double>(lee_ctx* c, const std::vector<double>& dts, bool graph);

}  // namespace lee

extern "C" {

int lee_set_batch_shapes(lee_ctx* c, int stage_shape, int filter_shape) {
  if (!c) return LEE_ERR_ARG;
  if (!c->prepared || !c->batch.active) return fail(c, LEE_ERR_STATE, "the context does not run batched kernels");
  if (stage_shape < 0 || stage_shape >= kBatchShapes || filter_shape < 0 || filter_shape >= kBatchShapes)
    return fail(c, LEE_ERR_ARG, "shape index");
  CK(cudaSetDevice(c->cfg.device));
  auto& bt = c->batch;
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->cfg.device);
  const std::vector<int4> ts = batch_tiles(c, stage_shape), tf = batch_tiles(c, filter_shape);
  int rc;
  if ((rc = dalloc(c, &bt.d_stiles, ts.size())) || (rc = dalloc(c, &bt.d_ftiles, tf.size()))) return rc;
  CK(cudaMemcpy(bt.d_stiles, ts.data(), ts.size() * sizeof(int4), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(bt.d_ftiles, tf.data(), tf.size() * sizeof(int4), cudaMemcpyHostToDevice));
  bt.nst = (int)ts.size();
  bt.nft = (int)tf.size();
  bt.sshape = stage_shape;
  bt.fshape = filter_shape;
  const int occs = c->comp ? batch_stage_occupancy<float>(stage_shape, 1) : batch_stage_occupancy<double>(stage_shape, 0);
  const int occf = c->comp ? batch_filter_occupancy<float>(filter_shape, 1)
                           : batch_filter_occupancy<double>(filter_shape, 0);
  bt.sgrid = std::min(bt.nst, nsm * occs);
  bt.fgrid = std::min(4 * bt.nft, nsm * occf);
  if (c->graph.exec) {  // captured launches name the old work lists
    cudaGraphExecDestroy(c->graph.exec);
    c->graph.exec = nullptr;
  }
  return LEE_OK;
}

int lee_set_batch_persistent(lee_ctx* c, int shape) {
  if (!c) return LEE_ERR_ARG;
  if (!c->prepared || !c->batch.active) return fail(c, LEE_ERR_STATE, "the context does not run batched kernels");
  if (shape != -1 && !batch_step_shape(shape))
    return fail(c, LEE_ERR_ARG, "persistent batch shape %d (one column per stage thread: 0 .. 4)", shape);
  CK(cudaSetDevice(c->cfg.device));
  auto& bt = c->batch;
  int rc;
  if (shape >= 0) {
    const std::vector<int4> t = batch_tiles(c, shape);
    if ((rc = dalloc(c, &bt.d_ptiles, t.size()))) return rc;
    CK(cudaMemcpy(bt.d_ptiles, t.data(), t.size() * sizeof(int4), cudaMemcpyHostToDevice));
    bt.npt = (int)t.size();
    if (!bt.d_gbar && (rc = dalloc(c, &bt.d_gbar, 2))) return rc;
  }
  bt.pshape = shape;
  if (c->graph.exec) {  // captured launches name the old schedule
    cudaGraphExecDestroy(c->graph.exec);
    c->graph.exec = nullptr;
  }
  return LEE_OK;
}

}  // extern "C"
