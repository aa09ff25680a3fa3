// The discrete adjoint: transposed operators, the reverse RK sweep of one step, microphone
// traces and the objective, checkpoints with segment recompute, and their entry points. The
// reference has no adjoint.
#include "lee_host.h"

using namespace lee;

namespace {

// out = fl32(y + e)
__global__ void k_add_pair(long long n, float* out, const float* y, const float* e) {
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < n; l += (long long)gridDim.x * blockDim.x)
    out[l] = (float)((double)y[l] + (double)e[l]);
}

}  // namespace

namespace lee {

// ---- discrete adjoint --------------------------------------------------------------------

// The transpose of a directional operator as dop() applies it (closure row r at the r-th point
// from either end, the mirrored right rows scaled by mfac, the interior stencil elsewhere),
// built densely on a line long enough to hold both ends and an interior, then read back as
// an interior row and E class rows per end within a window of H points on either side.
bool build_transpose(const OpTable& op, TransOp* t) {
  const int h = op.h, S = op.S;
  const int n = 4 * (h + S) + 2 * kTE + 1;
  std::vector<double> D((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) {
    if (i < h) {
      for (int s = 0; s < S; ++s) D[(size_t)i * n + s] += op.B[i][s];
    } else if (i > n - 1 - h) {
      const int r = n - 1 - i;
      for (int s = 0; s < S; ++s) D[(size_t)i * n + (n - 1 - s)] += op.mfac * op.B[r][s];
    } else {
      for (int l = -h; l <= h; ++l) D[(size_t)i * n + i + l] += op.c[l + h];
    }
  }
  auto DT = [&](int i, int j) { return (j < 0 || j >= n) ? 0.0 : D[(size_t)j * n + i]; };
  int H = 0;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j)
      if (DT(i, j) != 0.0) H = std::max(H, std::abs(j - i));
  if (H > kTH) return false;
  const int mid = n / 2;
  auto interior_like = [&](int i) {
    for (int q = -H; q <= H; ++q)
      if (DT(i, i + q) != DT(mid, mid + q)) return false;
    return true;
  };
  int E = 0;
  while (E < n / 2 && !interior_like(E)) ++E;
  int Er = 0;
  while (Er < n / 2 && !interior_like(n - 1 - Er)) ++Er;
  E = std::max(std::max(E, Er), H);
  if (E > kTE) return false;
  for (int i = E; i <= n - 1 - E; ++i)
    if (!interior_like(i)) return false;
  memset(t, 0, sizeof *t);
  t->H = H;
  t->E = E;
  for (int q = -H; q <= H; ++q) t->in[q + H] = DT(mid, mid + q);
  for (int r = 0; r < E; ++r)
    for (int q = -H; q <= H; ++q) {
      t->lt[r][q + H] = DT(r, r + q);
      t->rt[r][q + H] = DT(n - 1 - r, n - 1 - r + q);
    }
  return true;
}

// Checks and buffers of the adjoint path: the uniform-mean single-block path when it applies,
// else the general path (lee_host_adjoint_gen.cu).
int adjoint_setup(lee_ctx* c) {
  auto& a = c->adj;
  if (a.ready) return LEE_OK;
  if (c->nsc) return fail(c, LEE_ERR_UNSUPPORTED, "the adjoint has no passive scalars");
  if (!adjoint_fast_applies(c, nullptr)) return adjoint_gen_setup(c);
  BlockData& b = c->blk[0];
  // the class-row transposes need rows within reach and lines that keep the two ends' class
  // rows apart (n >= 2E, n >= E + H + h); otherwise the general path's per-point rows serve
  if (!build_transpose(c->fd, &a.dT)) return adjoint_gen_setup(c);
  if (c->cfg.filter_scheme != LEE_FILTER_NONE && !build_transpose(c->flt, &a.fT)) return adjoint_gen_setup(c);
  const int n[3] = {b.nx, b.ny, b.nz};
  int need = std::max(2 * a.dT.E, a.dT.E + a.dT.H + c->fd.h);
  if (c->cfg.filter_scheme != LEE_FILTER_NONE) need = std::max(need, std::max(2 * a.fT.E, a.fT.E + a.fT.H + c->flt.h));
  for (int d = 0; d < c->cfg.num_dim; ++d)
    if (n[d] < need) return adjoint_gen_setup(c);
  // the plane-marching stage kernel: 3-D, transposed stencils within two points, rows of 16-byte
  // multiples, 32-bit point offsets, J*metrics all fields or all constants
  {
    int nf = 0;
    for (int q = 0; q < 9; ++q) nf += (c->comp ? (const void*)b.cf_jm[q].p : (const void*)b.cd_jm[q].p) != nullptr;
    a.tma = c->cfg.num_dim == 3 && a.dT.H == 2 && ((size_t)b.nx * c->esz) % 16 == 0 &&
            (unsigned long long)b.N < (1ull << 32) && (nf == 0 || nf == 9);
    a.tma_jm = nf == 9;
    // the transposed filter through the fused filter kernel: its instantiated widths, rows of
    // 16-byte multiples (the TMA box), class rows within the parameter table
    const int H = a.fT.H;
    a.fused_filter = c->cfg.filter_scheme != LEE_FILTER_NONE && (H == 2 || H == 4 || H == 5) &&
                     a.fT.E <= kTE && ((size_t)b.nx * c->esz) % 16 == 0 && (unsigned long long)b.N < (1ull << 32);
  }
  int rc;
  if ((rc = alloc_fields(c, a.lam, b.N)) || (rc = alloc_fields(c, a.mu, b.N)) || (rc = alloc_fields(c, a.kb[0], b.N)) ||
      (rc = alloc_fields(c, a.kb[1], b.N)) || (rc = alloc_fields(c, a.ybar, b.N)))
    return rc;
  bool spg = false;
  for (auto& z : b.bnd) spg |= z.kind == LEE_SPONGE_FREUND_AMBIENT;
  if (spg && !b.d_sigma_field && (rc = build_sigma_field(c, b))) return rc;
  if (!a.d_base && (rc = dalloc(c, &a.d_base, 1))) return rc;
  a.ready = true;
  return LEE_OK;
}

// One transposed step: lam (adjoint of y_{n+1}) -> lam (adjoint of y_n); amps[s] are the
// source amplitudes of the forward step's stages (gbar null: no source gradient).
template <typename T>
int adjoint_step(lee_ctx* c, double dt, const double* amps, double* gbar) {
  auto& a = c->adj;
  BlockData& b = c->blk[0];
  const Tableau tb = tableau(c->cfg.rk_scheme);
  const int V = c->V;
  // mu = F^T lam: the directions commute, each is transposed, the last pass blends
  void** mu = a.lam;
  if (c->cfg.filter_scheme != LEE_FILTER_NONE && a.fused_filter) {
    // the fused filter kernel with the transposed rows as its class weights: one read of lam,
    // one write of mu = (1 - beta) lam + beta F^T lam
    TmaFilterParams<T> fp;
    memset(&fp, 0, sizeof fp);
    fp.nx = b.nx; fp.ny = b.ny; fp.nz = b.nz;
    fp.V = V;
    fp.tiles_x = b.tiles_x;
    // the scalar fused filter's form and chunk (the forward filter may run the two-point kernel)
    const int ry = b.tfilter_ry;
    fp.k_chunk = b.tfilter_chunk > 0 ? b.tfilter_chunk : (b.filter_chunk > 0 ? b.filter_chunk : b.nz);
    fp.nb = a.fT.E;
    const int H = a.fT.H;
    for (int o = 0; o <= 2 * H; ++o) {
      fp.w[0][o] = (T)a.fT.in[o];
      for (int r = 0; r < a.fT.E; ++r) {
        fp.w[1 + r][o] = (T)a.fT.lt[r][o];
        fp.w[1 + a.fT.E + r][o] = (T)a.fT.rt[r][o];
      }
    }
    fp.blend = (T)c->cfg.filter_blend;
    for (int v = 0; v < V; ++v) fp.out[v] = (T*)a.mu[v];
    fp.errflag = c->d_err;
    fp.wait_ns = c->wait_ns;
    // where the forward filter runs the two-point kernel (FP32, 3-D, no holes, even nxi), so does
    // the transposed filter, in its plain form, with the forward's tuned chunk
    const bool pair = sizeof(T) == 4 && b.filter_pair && filter_pair_half_width(H);
    int bx, by, ptx, pty;
    if (pair) {
      filter_pair_box(H, &bx, &by, &ptx, &pty);
      fp.tiles_x = b.ptiles_x;
      fp.k_chunk = b.filter_chunk > 0 ? b.filter_chunk : b.nz;
    } else {
      filter_box(c, H, ry, &bx, &by);
    }
    FieldMaps fm;
    int rc = field_maps(c, b, a.lam, bx, by, &fm);
    if (rc) return rc;
    const int chunks = c->cfg.num_dim == 3 ? (b.nz + fp.k_chunk - 1) / fp.k_chunk : 1;
    bool done = false;
    if constexpr (sizeof(T) == 4) {
      if (pair) {
        CK(launch_filter_pair(fm, fp, H, 0, b.ptiles_x * b.ptiles_y, chunks, c->stream));
        done = true;
      }
    }
    if (!done) CK(launch_filter_tma<T>(fm, fp, H, c->cfg.num_dim, 0, ry, filter_tiles_form(b, ry), chunks, c->stream));
    c->stats.kernel_launches += 1;
    mu = a.mu;
  } else if (c->cfg.filter_scheme != LEE_FILTER_NONE) {
    const int n[3] = {b.nx, b.ny, b.nz};
    int dirs[3], nd = 0;
    for (int d = 0; d < c->cfg.num_dim; ++d)
      if (n[d] > 1) dirs[nd++] = d;
    void** src = a.lam;
    for (int q = 0; q < nd; ++q) {
      AdjFilterParams<T> fp;
      memset(&fp, 0, sizeof fp);
      fp.nx = b.nx; fp.ny = b.ny; fp.nz = b.nz; fp.V = V; fp.dir = dirs[q]; fp.last = q == nd - 1;
      void** dst = fp.last ? a.mu : a.kb[q % 2];
      for (int v = 0; v < V; ++v) {
        fp.in[v] = (const T*)src[v];
        fp.out[v] = (T*)dst[v];
        fp.lam[v] = (const T*)a.lam[v];
      }
      fp.blend = (T)c->cfg.filter_blend;
      fp.op = a.fT;
      CK(launch_adj_filter<T>(fp, c->stream));
      c->stats.kernel_launches += 1;
      src = dst;
    }
    mu = a.mu;
  }
  const bool dbl = std::is_same<T, double>::value;
  AdjStageParams<T> p;
  memset(&p, 0, sizeof p);
  p.nx = b.nx; p.ny = b.ny; p.nz = b.nz; p.V = V;
  const Coef<T>* jm = dbl ? (const Coef<T>*)b.cd_jm : (const Coef<T>*)b.cf_jm;
  for (int q = 0; q < 9; ++q) p.jm[q] = jm[q];
  for (int x = 0; x < 3; ++x) p.ubar[x] = dbl ? (T)b.cd_ub[x].c : (T)b.cf_ub[x].c;
  const T pb = dbl ? (T)b.cd_pb.c : (T)b.cf_pb.c;
  p.gpb = (T)c->cfg.gamma * pb;
  p.rbi = dbl ? (T)b.cd_rbi.c : (T)b.cf_rbi.c;
  p.sigma = (const T*)b.d_sigma_field;
  p.gbar = gbar;
  for (int d = 0; d < 3; ++d) { p.src_lo[d] = b.src_lo[d]; p.src_hi[d] = b.src_hi[d]; }
  p.op = a.dT;
  const int ns = tb.ns;
  int cur = 0;
  for (int s = ns - 1; s >= 0; --s) {
    p.first = s == ns - 1;
    p.has_next = s > 0;
    p.hb_in = (T)(dt * tb.b[ns - 1]);
    p.hb_next = s > 0 ? (T)(dt * tb.b[s - 1]) : T(0);
    p.ha_next = s > 0 ? (T)(tb.a[s - 1] * dt) : T(0);
    p.amp = amps ? amps[s] : 0.0;
    for (int v = 0; v < V; ++v) {
      p.kin[v] = (const T*)(p.first ? mu[v] : a.kb[cur][v]);
      p.mu[v] = (const T*)mu[v];
      p.ybar[v] = (T*)a.ybar[v];
      p.kout[v] = (T*)a.kb[1 - cur][v];
    }
    if (a.tma) {
      // the plane-marching kernel: maps of w (this stage's input) and the J*metrics fields
      AdjMaps am;
      int bx, by, tx, ty;
      adj_tma_box(c->esz, &bx, &by, &tx, &ty);
      const void* f[14];
      for (int v = 0; v < 5; ++v) f[v] = p.kin[v];
      for (int q = 0; q < 9; ++q) f[5 + q] = p.jm[q].p;
      int rc = encode_maps(c, b, f, a.tma_jm ? 14 : 5, bx, by, am.m);
      if (rc) return rc;
      AdjTmaParams<T> tp;
      tp.a = p;
      tp.tiles_x = (b.nx + tx - 1) / tx;
      // 32 planes per CTA: a grid of several waves leaves room for the forward recompute that runs
      // beside the reverse sweep (one wave of longer marches, 96 planes at 192^3, took the
      // recompute mode from 3.04x to 3.54x the forward)
      tp.k_chunk = std::min(b.nz, 32);
      tp.err = c->d_err;
      tp.wait_ns = c->wait_ns;
      const int tiles = tp.tiles_x * ((b.ny + ty - 1) / ty);
      CK(launch_adj_tma<T>(am, tp, a.tma_jm, tiles, (b.nz + tp.k_chunk - 1) / tp.k_chunk, c->stream));
    } else {
      CK(launch_adj_stage<T>(p, c->cfg.num_dim, c->stream));
    }
    c->stats.kernel_launches += 1;
    if (!p.first) cur = 1 - cur;
    else cur = 1;  // the first processed stage wrote kb[1]
  }
  swap_fields(V, a.lam, a.ybar);
  return LEE_OK;
}

// Trace rows for nsteps steps (reallocated when too short).
int ensure_trace(lee_ctx* c, size_t rows) {
  auto& a = c->adj;
  if (a.trace_rows >= rows) return LEE_OK;
  int rc = dalloc(c, &a.d_trace, rows * a.mic.size());
  if (rc) return rc;
  a.trace_rows = rows;
  return LEE_OK;
}

// Advance nsteps with the microphone traces written from row 0.
int advance_traced(lee_ctx* c, int nsteps, double dt, int row0) {
  auto& a = c->adj;
  a.trace_on = true;
  a.host_row = row0;
  const std::vector<double> dts(c->blk.size(), dt);
  int rc = c->comp ? advance_impl<float>(c, nsteps, dts) : advance_impl<double>(c, nsteps, dts);
  a.trace_on = false;
  return rc;
}

double objective_of(const lee_ctx* c, const std::vector<double>& tr) {
  double J = 0.0;
  for (double v : tr) J += v * v;
  return c->adj.weight * J;
}

// The adjoint fields of block bi (the uniform path keeps one block's).
void** lam_of(lee_ctx* c, int bi) { return c->adj.gen ? c->adj.gb[(size_t)bi].lam : c->adj.lam; }

// One transposed step on whichever path the context set up, in its working precision.
int adjoint_step_any(lee_ctx* c, double dt, const double* amps, double* gbar, bool rho_in) {
  if (c->adj.gen)
    return c->comp ? adjoint_step_gen<float>(c, dt, amps, gbar, rho_in) : adjoint_step_gen<double>(c, dt, amps, gbar, rho_in);
  return c->comp ? adjoint_step<float>(c, dt, amps, gbar) : adjoint_step<double>(c, dt, amps, gbar);
}

// the host translation units use both precisions
template int adjoint_step<float>(lee_ctx* c, double dt, const double* amps, double* gbar);
template int adjoint_step<double>(lee_ctx* c, double dt, const double* amps, double* gbar);

}  // namespace lee

extern "C" {

int lee_set_objective(lee_ctx* c, int b, int n, const long long* l0, double weight) {
  if (!c) return LEE_ERR_ARG;
  if (!c->prepared) return fail(c, LEE_ERR_STATE, "lee_prepare first");
  if (b < 0 || b >= (int)c->blk.size()) return fail(c, LEE_ERR_ARG, "objective block");
  if (n < 1 || !l0) return fail(c, LEE_ERR_ARG, "the objective needs microphones");
  const BlockData& bk = c->blk[(size_t)b];
  std::vector<long long> mic(l0, l0 + n);
  std::vector<long long> sorted = mic;
  std::sort(sorted.begin(), sorted.end());
  for (size_t m = 0; m < sorted.size(); ++m) {
    if (sorted[m] < 0 || sorted[m] >= bk.N) return fail(c, LEE_ERR_ARG, "microphone %zu outside the block", m);
    if (m && sorted[m] == sorted[m - 1]) return fail(c, LEE_ERR_ARG, "two microphones on one point");
  }
  CK(cudaSetDevice(c->cfg.device));
  auto& a = c->adj;
  if (a.mic.size() != mic.size()) {
    int rc = dalloc(c, &a.d_mic, mic.size());
    if (rc) return rc;
  }
  a.mic = mic;
  a.mic_block = b;
  a.weight = weight;
  CK(cudaMemcpyAsync(a.d_mic, a.mic.data(), a.mic.size() * sizeof(long long), cudaMemcpyHostToDevice, c->stream));
  if (!a.d_base) {
    int rc = dalloc(c, &a.d_base, 1);
    if (rc) return rc;
  }
  CK(cudaStreamSynchronize(c->stream));
  return LEE_OK;
}

int lee_eval_objective(lee_ctx* c, int nsteps, double dt, double* J) {
  if (!c || !J) return LEE_ERR_ARG;
  if (!c->prepared || !c->uploaded) return fail(c, LEE_ERR_STATE, "lee_prepare and lee_upload_state first");
  if (c->adj.mic.empty()) return fail(c, LEE_ERR_STATE, "lee_set_objective first");
  if (nsteps < 1 || !(dt > 0.0)) return fail(c, LEE_ERR_ARG, "nsteps >= 1 and dt > 0");
  CK(cudaSetDevice(c->cfg.device));
  memset(&c->stats, 0, sizeof c->stats);
  int rc = ensure_trace(c, (size_t)nsteps);
  if (rc) return rc;
  if ((rc = advance_traced(c, nsteps, dt, 0))) return rc;
  std::vector<double> tr((size_t)nsteps * c->adj.mic.size());
  CK(cudaMemcpyAsync(tr.data(), c->adj.d_trace, tr.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *J = objective_of(c, tr);
  return check_device_error(c);
}

int lee_apply_adjoint(lee_ctx* c, int nsteps, double dt) {
  if (!c) return LEE_ERR_ARG;
  if (!c->prepared || !c->uploaded) return fail(c, LEE_ERR_STATE, "lee_prepare and lee_upload_state first");
  if (nsteps < 0 || !(dt > 0.0)) return fail(c, LEE_ERR_ARG, "nsteps >= 0 and dt > 0");
  CK(cudaSetDevice(c->cfg.device));
  int rc = adjoint_setup(c);
  if (rc) return rc;
  auto& a = c->adj;
  // the state slots of every block hold the adjoint variable (with a compensated state, y + e rounded)
  for (size_t bi = 0; bi < c->blk.size(); ++bi) {
    BlockData& b = c->blk[bi];
    void** lam = lam_of(c, (int)bi);
    const size_t bytes = (size_t)b.N * c->esz;
    for (int v = 0; v < c->V; ++v) {
      if (c->comp) {
        k_add_pair<<<grid1d(b.N), 256, 0, c->stream>>>(b.N, (float*)lam[v], (const float*)b.y[v],
                                                        (const float*)b.comp[v]);
        CK(cudaGetLastError());
      } else {
        CK(cudaMemcpyAsync(lam[v], b.y[v], bytes, cudaMemcpyDeviceToDevice, c->stream));
      }
    }
  }
  a.rb_live = false;
  // the transposed map of nsteps forward steps from an uploaded state: the first of them reads no
  // rho'/rho_bar of a previous step
  for (int it = 0; it < nsteps; ++it) {
    const bool rho_in = nsteps - it >= 2;
    rc = adjoint_step_any(c, dt, nullptr, nullptr, rho_in);
    if (rc) return rc;
  }
  for (size_t bi = 0; bi < c->blk.size(); ++bi) {
    BlockData& b = c->blk[bi];
    void** lam = lam_of(c, (int)bi);
    const size_t bytes = (size_t)b.N * c->esz;
    for (int v = 0; v < c->V; ++v) {
      CK(cudaMemcpyAsync(b.y[v], lam[v], bytes, cudaMemcpyDeviceToDevice, c->stream));
      if (c->comp) CK(cudaMemsetAsync(b.comp[v], 0, bytes, c->stream));
    }
    b.rho_valid = false;
  }
  CK(cudaStreamSynchronize(c->stream));
  return check_device_error(c);
}

int lee_adjoint_gradient(lee_ctx* c, int nsteps, double dt, int checkpoint_every, int recompute, double* J,
                         double* grad, long long* trace_mismatches) {
  if (!c || !J || !grad) return LEE_ERR_ARG;
  if (!c->prepared || !c->uploaded) return fail(c, LEE_ERR_STATE, "lee_prepare and lee_upload_state first");
  if (c->adj.mic.empty()) return fail(c, LEE_ERR_STATE, "lee_set_objective first");
  if (c->src_kind != LEE_SOURCE_DISTRIBUTED) return fail(c, LEE_ERR_STATE, "the gradient is for a distributed source");
  if (nsteps < 1 || checkpoint_every < 1 || !(dt > 0.0)) return fail(c, LEE_ERR_ARG, "nsteps, checkpoint_every, dt");
  CK(cudaSetDevice(c->cfg.device));
  memset(&c->stats, 0, sizeof c->stats);
  int rc = adjoint_setup(c);
  if (rc) return rc;
  auto& a = c->adj;
  const int V = c->V;
  const int nbk = (int)c->blk.size();
  const int sb = (int)c->dsrc[0];
  BlockData& bs = c->blk[(size_t)sb];
  const int K = checkpoint_every;
  const int nseg = (nsteps + K - 1) / K;
  // what a checkpoint holds: every block's state (and carried errors), and rho'/rho_bar of the
  // blocks whose first stage reads it
  struct Slot {
    int b, kind, v;  // kind 0 y, 1 comp, 2 rho
  };
  std::vector<Slot> slots;
  bool rho0 = false;
  std::vector<char> rho_start((size_t)nbk, 0);
  for (int bi = 0; bi < nbk; ++bi) {
    BlockData& b = c->blk[(size_t)bi];
    for (int v = 0; v < V; ++v) slots.push_back({bi, 0, v});
    if (c->comp)
      for (int v = 0; v < V; ++v) slots.push_back({bi, 1, v});
    if (b.need_rho) {
      slots.push_back({bi, 2, 0});
      rho_start[(size_t)bi] = b.rho_valid ? 1 : 0;
      rho0 |= b.rho_valid;
    }
  }
  auto field = [&](const Slot& q) -> void* {
    BlockData& b = c->blk[(size_t)q.b];
    return q.kind == 0 ? b.y[q.v] : q.kind == 1 ? b.comp[q.v] : b.rho;
  };
  auto bytes_of = [&](const Slot& q) { return (size_t)c->blk[(size_t)q.b].N * c->esz; };
  const size_t fields = slots.size();
  if (a.ckpt_slots < (size_t)nseg || a.ckpt.size() < (size_t)nseg * fields) {
    for (size_t q = a.ckpt.size(); q < (size_t)nseg * fields; ++q) {
      void* p = nullptr;
      if ((rc = dev_alloc(c, &p, bytes_of(slots[q % fields])))) return rc;
      a.ckpt.push_back(p);
    }
    a.ckpt_slots = (size_t)nseg;
  }
  if ((rc = ensure_trace(c, (size_t)nsteps))) return rc;
  auto save = [&](int seg) -> int {
    for (size_t q = 0; q < fields; ++q)
      CK(cudaMemcpyAsync(a.ckpt[(size_t)seg * fields + q], field(slots[q]), bytes_of(slots[q]), cudaMemcpyDeviceToDevice,
                         c->stream));
    return LEE_OK;
  };
  auto restore = [&](int seg) -> int {
    for (size_t q = 0; q < fields; ++q)
      CK(cudaMemcpyAsync(field(slots[q]), a.ckpt[(size_t)seg * fields + q], bytes_of(slots[q]), cudaMemcpyDeviceToDevice,
                         c->stream));
    // a segment after the first starts on the rho'/rho_bar its previous step wrote
    for (int bi = 0; bi < nbk; ++bi)
      if (c->blk[(size_t)bi].need_rho) c->blk[(size_t)bi].rho_valid = seg > 0 || rho_start[(size_t)bi];
    return LEE_OK;
  };
  // forward pass: checkpoints, traces, the stage times of every step
  const int step_start = c->step;
  std::vector<double> seg_time((size_t)nseg);
  for (int seg = 0; seg < nseg; ++seg) {
    const int n = std::min(K, nsteps - seg * K);
    seg_time[(size_t)seg] = c->time;
    if ((rc = save(seg))) return rc;
    if ((rc = advance_traced(c, n, dt, seg * K))) return rc;
  }
  std::vector<double> tr((size_t)nsteps * a.mic.size());
  CK(cudaMemcpyAsync(tr.data(), a.d_trace, tr.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *J = objective_of(c, tr);
  // final state, kept aside while segments are recomputed
  const double t_end = c->time;
  const int step_end = c->step;
  std::vector<void*> fin;
  std::vector<char> rho_end((size_t)nbk, 0);
  if (recompute) {
    for (size_t q = 0; q < fields; ++q) {
      void* p = nullptr;
      CK(cudaMallocAsync(&p, bytes_of(slots[q]), c->stream));
      fin.push_back(p);
      CK(cudaMemcpyAsync(p, field(slots[q]), bytes_of(slots[q]), cudaMemcpyDeviceToDevice, c->stream));
    }
    for (int bi = 0; bi < nbk; ++bi) rho_end[(size_t)bi] = c->blk[(size_t)bi].rho_valid ? 1 : 0;
  }
  // reverse sweep
  const size_t nbox = (size_t)(bs.src_hi[0] - bs.src_lo[0] + 1) * (bs.src_hi[1] - bs.src_lo[1] + 1) *
                      (bs.src_hi[2] - bs.src_lo[2] + 1);
  if (a.gbar_n < nbox) {
    if ((rc = dalloc(c, &a.d_gbar, nbox))) return rc;
    a.gbar_n = nbox;
  }
  CK(cudaMemsetAsync(a.d_gbar, 0, nbox * sizeof(double), c->stream));
  for (int bi = 0; bi < nbk; ++bi) {
    void** lam = lam_of(c, bi);
    for (int v = 0; v < V; ++v) CK(cudaMemsetAsync(lam[v], 0, (size_t)c->blk[(size_t)bi].N * c->esz, c->stream));
  }
  a.rb_live = false;
  const Tableau tb = tableau(c->cfg.rk_scheme);
  const size_t M = a.mic.size();
  const double scale = 2.0 * a.weight;
  const int P = V - 1;
  long long mismatches = 0;
  // With recompute, the reverse sweep runs on a stream of its own: segment s's reverse steps
  // wait for s's recomputed traces, and the recompute of segment s - 1 (forward buffers, its
  // own trace rows) runs beside them. The reverse sweep reads the adjoint buffers, the
  // coefficient fields and trace rows of its segment only, and the forward steps never touch
  // those, so the two overlap on the GPU with no other ordering.
  cudaStream_t main_stream = c->stream;
  if (recompute) {
    if (!a.rev) CK(cudaStreamCreateWithFlags(&a.rev, cudaStreamNonBlocking));
    if (!a.ev_fwd) CK(cudaEventCreateWithFlags(&a.ev_fwd, cudaEventDisableTiming));
    if (!a.ev_rev) CK(cudaEventCreateWithFlags(&a.ev_rev, cudaEventDisableTiming));
    CK(cudaEventRecord(a.ev_fwd, main_stream));  // lam and gbar zeroed above
    CK(cudaStreamWaitEvent(a.rev, a.ev_fwd, 0));
  }
  for (int seg = nseg - 1; seg >= 0; --seg) {
    const int n0 = seg * K, n = std::min(K, nsteps - n0);
    if (recompute && seg < nseg - 1) {
      // the segment's forward steps again, from its checkpoint; their traces must repeat (checked
      // against the first pass once every segment is done). The last segment is where the
      // forward pass ended: its traces were just recorded, so the reverse sweep starts on them.
      if ((rc = restore(seg))) return rc;
      set_clock(c, seg_time[(size_t)seg], step_start + n0);
      if ((rc = advance_traced(c, n, dt, n0))) return rc;
      CK(cudaEventRecord(a.ev_fwd, main_stream));
      CK(cudaStreamWaitEvent(a.rev, a.ev_fwd, 0));
    }
    // stage times of each step of the segment, advanced as the forward steps advance them
    std::vector<double> amps((size_t)n * tb.ns);
    double t = seg_time[(size_t)seg];
    for (int k = 0; k < n; ++k) {
      t += dt;
      for (int s = 0; s < tb.ns; ++s) amps[(size_t)k * tb.ns + s] = source_amp(c, bs, t + tb.c[s] * dt);
    }
    // the reverse steps go to the reverse stream (every launch below reads c->stream)
    if (recompute) c->stream = a.rev;
    void** lam_mic = lam_of(c, a.mic_block);
    for (int k = n - 1; k >= 0 && !rc; --k) {
      const int step = n0 + k;  // 0-based: this transposed step maps the adjoint of y_{step+1} to y_step
      cudaError_t e = c->comp
                          ? launch_mic_force<float>((int)M, a.d_mic, (float*)lam_mic[P], a.d_trace, step, scale, c->stream)
                          : launch_mic_force<double>((int)M, a.d_mic, (double*)lam_mic[P], a.d_trace, step, scale,
                                                     c->stream);
      if (e != cudaSuccess) rc = fail(c, LEE_ERR_CUDA, "microphone forcing: %s", cudaGetErrorString(e));
      if (!rc) rc = adjoint_step_any(c, dt, &amps[(size_t)k * tb.ns], a.d_gbar, step > 0 || rho0);
      lam_mic = lam_of(c, a.mic_block);
    }
    c->stream = main_stream;
    if (rc) {
      if (recompute) cudaStreamSynchronize(a.rev);
      return rc;
    }
  }
  if (recompute) {
    // the reverse sweep ends before the gradient is read and the final state put back
    CK(cudaEventRecord(a.ev_rev, a.rev));
    CK(cudaStreamWaitEvent(main_stream, a.ev_rev, 0));
    std::vector<double> tr2(tr.size());
    CK(cudaMemcpyAsync(tr2.data(), a.d_trace, tr2.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (size_t q = 0; q < tr2.size(); ++q) mismatches += tr2[q] != tr[q];
  }
  // source-box gradient -> lattice gradient
  std::vector<double> gbox(nbox);
  CK(cudaMemcpyAsync(gbox.data(), a.d_gbar, nbox * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  restrict_to_lattice(c->dsrc, c->cfg.num_dim, bs.src_lo, bs.src_hi, gbox.data(), grad);
  if (recompute) {
    for (size_t q = 0; q < fields; ++q) {
      CK(cudaMemcpyAsync(field(slots[q]), fin[q], bytes_of(slots[q]), cudaMemcpyDeviceToDevice, c->stream));
      CK(cudaFreeAsync(fin[q], c->stream));
    }
    for (int bi = 0; bi < nbk; ++bi) c->blk[(size_t)bi].rho_valid = rho_end[(size_t)bi] != 0;
    set_clock(c, t_end, step_end);
  }
  CK(cudaStreamSynchronize(c->stream));
  if (trace_mismatches) *trace_mismatches = mismatches;
  return check_device_error(c);
}

}  // extern "C"
