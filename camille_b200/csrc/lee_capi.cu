// Host side of the C ABI (include/lee_b200.h): context creation and configuration, block,
// mean-flow, boundary and source inputs, state upload and download, the CFL time step and the
// report reductions. The setup (lee_host_setup.cu), the time-advance schedule (lee_host_step.cu),
// batches (lee_host_batch.cu), the adjoint (lee_host_adjoint.cu) and overset maps
// (lee_host_overset.cu) have files of their own.
#include "lee_host.h"

using namespace lee;

namespace {

// FP64 -> (y, e) with y = fl32(x) and e = fl32(x - y): the compensated pair of an uploaded state
__global__ void k_split(long long n, float* y, float* e, const double* in) {
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < n; l += (long long)gridDim.x * blockDim.x) {
    const float r = (float)in[l];
    y[l] = r;
    e[l] = (float)(in[l] - (double)r);
  }
}

}  // namespace

namespace lee {

// FP64 staging field of the compensated form's uploads, downloads and right-hand sides, as large
// as the largest block; allocated once, on first use.
int staging(lee_ctx* c, double** out) {
  if (!c->d_staging) {
    long long n = 0;
    for (const auto& b : c->blk) n = std::max(n, b.N);
    const int rc = dalloc(c, &c->d_staging, (size_t)n);
    if (rc) return rc;
  }
  *out = c->d_staging;
  return LEE_OK;
}

// CFL maxima (temporal::compute_CFL) at time step dt0 of every block, or of all blocks.
int cfl_max(lee_ctx* c, bool per_block, std::vector<double>& out, double dt0) {
  CK(cudaSetDevice(c->cfg.device));
  double* d_max = nullptr;
  CK(cudaMallocAsync((void**)&d_max, sizeof(double), c->stream));
  const double init = -1e308;
  out.clear();
  CK(cudaMemcpyAsync(d_max, &init, sizeof init, cudaMemcpyHostToDevice, c->stream));
  for (auto& b : c->blk) {
    double** d_m = nullptr;
    double** d_u = nullptr;
    CK(cudaMallocAsync((void**)&d_m, 9 * sizeof(double*), c->stream));
    CK(cudaMallocAsync((void**)&d_u, 3 * sizeof(double*), c->stream));
    CK(cudaMemcpyAsync(d_m, b.d_met, 9 * sizeof(double*), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(d_u, b.d_mean + 1, 3 * sizeof(double*), cudaMemcpyHostToDevice, c->stream));
    CK(setup_cfl((int)b.N, c->cfg.num_dim, d_m, b.d_jac, d_u, b.d_mean[4], b.d_mean[0],
                 b.has_iblank ? b.d_iblank : nullptr, c->cfg.gamma, dt0, d_max, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaFreeAsync(d_m, c->stream));
    CK(cudaFreeAsync(d_u, c->stream));
    if (per_block) {
      double m = 0.0;
      CK(cudaMemcpyAsync(&m, d_max, sizeof m, cudaMemcpyDeviceToHost, c->stream));
      CK(cudaMemcpyAsync(d_max, &init, sizeof init, cudaMemcpyHostToDevice, c->stream));
      CK(cudaStreamSynchronize(c->stream));
      out.push_back(m);
    }
  }
  if (!per_block) {
    double m = 0.0;
    CK(cudaMemcpyAsync(&m, d_max, sizeof m, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    out.push_back(m);
  }
  CK(cudaFreeAsync(d_max, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return LEE_OK;
}

// The reference's dummy initial dt (src/core/input.cpp:131).
constexpr double kDummyDt = 1e-6;

// The FIX_CFL rescale of solver::solve (src/solver/solver.cpp:58-64) from the dummy dt.
double rescale(double cfl, double cmax) {
  double ratio = cfl / cmax;
  double d = kDummyDt;
  d *= ratio;
  return d;
}


}  // namespace lee

extern "C" {

int lee_create(const lee_config* cfg, lee_ctx** out) {
  lee_ctx* c = nullptr;
  if (!cfg || !out) return fail(nullptr, LEE_ERR_ARG, "null argument");
  *out = nullptr;
  if (cfg->num_dim != 2 && cfg->num_dim != 3) return fail(nullptr, LEE_ERR_ARG, "num_dim must be 2 or 3");
  if (cfg->num_blocks < 1 || cfg->num_blocks > 64) return fail(nullptr, LEE_ERR_ARG, "num_blocks out of range");
  if (cfg->rk_scheme != LEE_RK4 && cfg->rk_scheme != LEE_RK2) return fail(nullptr, LEE_ERR_ARG, "rk_scheme");
  if (cfg->precision != LEE_FP64 && cfg->precision != LEE_FP32_COMPENSATED)
    return fail(nullptr, LEE_ERR_ARG, "precision");
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0)
    return fail(nullptr, LEE_ERR_NODEVICE, "no CUDA device: %s", cudaGetErrorString(e));
  if (cfg->device < 0 || cfg->device >= ndev) return fail(nullptr, LEE_ERR_ARG, "device ordinal");
  c = new lee_ctx();
  c->cfg = *cfg;
  c->V = cfg->num_dim + 2;
  c->comp = cfg->precision == LEE_FP32_COMPENSATED;
  c->esz = c->comp ? 4 : 8;
  if (!make_fd(&c->fd, cfg->fd_scheme, cfg->fd_order)) {
    delete c;
    return fail(nullptr, LEE_ERR_UNSUPPORTED, "spatial scheme %d order %d", cfg->fd_scheme, cfg->fd_order);
  }
  if (cfg->filter_scheme != LEE_FILTER_NONE) {
    double strength = cfg->filter_scheme == LEE_FILTER_STANDARD_CENTRAL ? 1.0 : cfg->filter_strength;
    if (strength < 0.0 || strength > 1.0 || cfg->filter_blend < 0.0 || cfg->filter_blend > 1.0 ||
        !make_filter(&c->flt, cfg->filter_scheme, cfg->filter_order, strength)) {
      delete c;
      return fail(nullptr, LEE_ERR_UNSUPPORTED, "filter scheme %d order %d", cfg->filter_scheme, cfg->filter_order);
    }
    c->fltd = minus_identity(c->flt);
    c->hf = c->flt.h;
    c->wfl_ok = c->hf <= 5 && class_weights(c->comp ? c->fltd : c->flt, c->hf, &c->wfl[0][0], 11);
    // the zero class of a hole after a hole: F = 0, so the increment form's row is -1 at the point
    if (c->wfl_ok) c->wfl[1 + 2 * c->flt.nb][c->hf] = c->comp ? -1.0 : 0.0;
    c->wfl_sym = c->wfl_ok && (c->hf == 2 || c->hf == 4 || c->hf == 5);
    for (int o = 1; o <= c->hf && c->wfl_sym; ++o) c->wfl_sym = c->wfl[0][c->hf - o] == c->wfl[0][c->hf + o];
  }
  c->wst_ok = c->fd.h == kFdHalf && class_weights(c->fd, kFdHalf, &c->wst[0][0], 5);
  c->blk.resize((size_t)cfg->num_blocks);
  e = cudaSetDevice(cfg->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->d_err, 2 * sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(c->d_err, 0, 2 * sizeof(int));
  if (e != cudaSuccess) {
    if (c->d_err) cudaFree(c->d_err);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return fail(nullptr, LEE_ERR_CUDA, "stream creation failed: %s", cudaGetErrorString(e));
  }
  c->allocs.push_back(c->d_err);
  *out = c;
  return LEE_OK;
}

void lee_destroy(lee_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->cfg.device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->graph.exec) cudaGraphExecDestroy(c->graph.exec);
  for (auto e : c->ev_pool) cudaEventDestroy(e);
  if (c->adj.rev) {
    cudaStreamSynchronize(c->adj.rev);
    cudaStreamDestroy(c->adj.rev);
  }
  for (auto sd : c->side) {
    cudaStreamSynchronize(sd);
    cudaStreamDestroy(sd);
  }
  for (auto e : c->side_ev) cudaEventDestroy(e);
  if (c->adj.ev_fwd) cudaEventDestroy(c->adj.ev_fwd);
  if (c->adj.ev_rev) cudaEventDestroy(c->adj.ev_rev);
  for (void* p : c->allocs) cudaFree(p);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

const char* lee_last_error(const lee_ctx* c) { return c ? c->err.c_str() : g_create_error; }

int lee_set_block(lee_ctx* c, int b, int nx, int ny, int nz, const double* x, const double* y, const double* z,
                  const int* iblank) {
  if (!c) return LEE_ERR_ARG;
  if (c->prepared) return fail(c, LEE_ERR_STATE, "lee_set_block after lee_prepare");
  if (b < 0 || b >= (int)c->blk.size()) return fail(c, LEE_ERR_ARG, "block index %d", b);
  if (!x || !y || !z) return fail(c, LEE_ERR_ARG, "null coordinates");
  int need = std::max(2 * c->fd.h + 1, c->fd.S);
  if (c->cfg.filter_scheme != LEE_FILTER_NONE) need = std::max(need, std::max(2 * c->flt.h + 1, c->flt.S));
  int dims[3] = {nx, ny, nz};
  for (int d = 0; d < 3; ++d) {
    if (dims[d] < 1) return fail(c, LEE_ERR_ARG, "dimension %d is %d", d, dims[d]);
    if (d < c->cfg.num_dim && dims[d] < need)
      return fail(c, LEE_ERR_ARG, "direction %d has %d points; the stencils need at least %d", d, dims[d], need);
  }
  if (c->cfg.num_dim == 2 && nz != 1) return fail(c, LEE_ERR_ARG, "2-D blocks have nzeta = 1");
  BlockData& bk = c->blk[(size_t)b];
  bk.nx = nx; bk.ny = ny; bk.nz = nz;
  bk.N = (long long)nx * ny * nz;
  bk.hx.assign(x, x + bk.N);
  bk.hy.assign(y, y + bk.N);
  bk.hz.assign(z, z + bk.N);
  bk.hib.clear();
  bk.has_holes = bk.has_iblank = false;
  if (iblank) {
    bk.hib.assign(iblank, iblank + bk.N);
    for (int v : bk.hib) {
      if (v != 0 && v != 1 && v != -1) return fail(c, LEE_ERR_ARG, "iblank values are 0, 1 or -1");
      if (v == 1) bk.has_holes = true;
      if (v != 0) bk.has_iblank = true;
    }
  }
  bk.set = true;
  return LEE_OK;
}

int lee_set_mean(lee_ctx* c, int b, const double* const mean[5]) {
  if (!c) return LEE_ERR_ARG;
  if (c->prepared) return fail(c, LEE_ERR_STATE, "lee_set_mean after lee_prepare");
  if (b < 0 || b >= (int)c->blk.size() || !c->blk[(size_t)b].set) return fail(c, LEE_ERR_STATE, "lee_set_block first");
  BlockData& bk = c->blk[(size_t)b];
  for (int v = 0; v < 5; ++v) {
    if (!mean[v]) return fail(c, LEE_ERR_ARG, "null mean field");
    bk.hmean[v].assign(mean[v], mean[v] + bk.N);
  }
  for (long long l = 0; l < bk.N; ++l)
    if (!(bk.hmean[4][(size_t)l] > 0.0)) return fail(c, LEE_ERR_ARG, "mean pressure must be positive");
  bk.has_mean = true;
  return LEE_OK;
}

int lee_add_boundary(lee_ctx* c, int b, int kind, int dir, int end, const int lo[3], const int hi[3],
                     const double* sigma) {
  if (!c) return LEE_ERR_ARG;
  if (c->prepared) return fail(c, LEE_ERR_STATE, "lee_add_boundary after lee_prepare");
  if (b < 0 || b >= (int)c->blk.size() || !c->blk[(size_t)b].set) return fail(c, LEE_ERR_STATE, "lee_set_block first");
  BlockData& bk = c->blk[(size_t)b];
  if (!is_sponge(kind) && !is_bc_line(kind))
    return fail(c, LEE_ERR_UNSUPPORTED, "boundary kind %d is not supported", kind);
  if (dir < 0 || dir >= c->cfg.num_dim || (end != 0 && end != 1)) return fail(c, LEE_ERR_ARG, "dir/end");
  int dims[3] = {bk.nx, bk.ny, bk.nz};
  Boundary z;
  z.kind = kind; z.dir = dir; z.end = end;
  for (int d = 0; d < 3; ++d) {
    if (lo[d] < 0 || hi[d] >= dims[d] || lo[d] > hi[d]) return fail(c, LEE_ERR_ARG, "boundary box outside block");
    z.lo[d] = lo[d];
    z.hi[d] = hi[d];
  }
  if (reads_inward(kind)) {
    // the face's closure row reads S-1 points inward along dir
    const int S = c->fd.S, f = end == 0 ? lo[dir] : hi[dir];
    if ((end == 0 && f + S - 1 > dims[dir] - 1) || (end == 1 && f - (S - 1) < 0))
      return fail(c, LEE_ERR_ARG, "boundary face %d in direction %d lacks the %d points its closure row reads", f,
                  dir, S);
  }
  int nzones = 0;
  for (auto& q : bk.bnd) nzones += is_sponge(q.kind);
  if (is_sponge(kind) && nzones >= kMaxZones)
    return fail(c, LEE_ERR_UNSUPPORTED, "more than %d sponge zones in a block", kMaxZones);
  if (sigma && is_sponge(kind)) {
    size_t nb = (size_t)(hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1);
    z.sigma.assign(sigma, sigma + nb);
  }
  bk.bnd.push_back(std::move(z));
  return LEE_OK;
}

int lee_set_harmonic_wave(lee_ctx* c, int type, int form, int dir, double amplitude, double wavelength,
                          double halfwidth) {
  if (!c) return LEE_ERR_ARG;
  if (c->prepared) return fail(c, LEE_ERR_STATE, "lee_set_harmonic_wave after lee_prepare");
  if (type == LEE_WAVE_NONE) {
    c->wave = Wave{};
    return LEE_OK;
  }
  const bool ok = (type == LEE_WAVE_ACOUSTIC && (form == LEE_WAVEFORM_PLANE || form == LEE_WAVEFORM_HOMOGENEOUS)) ||
                  (type == LEE_WAVE_ENTROPY &&
                   (form == LEE_WAVEFORM_HOMOGENEOUS || form == LEE_WAVEFORM_GAUSSIAN_ROUNDJET));
  if (!ok) return fail(c, LEE_ERR_ARG, "unknown type of wave for this wave form (type %d, form %d)", type, form);
  if (dir < 0 || dir > 2) return fail(c, LEE_ERR_ARG, "wave direction %d", dir);
  if (!(amplitude >= 0.0 && amplitude <= 1.0)) return fail(c, LEE_ERR_ARG, "the wave amplitude should be between 0 and 1");
  if (!(wavelength > 0.0)) return fail(c, LEE_ERR_ARG, "the wavelength must be positive");
  if (form == LEE_WAVEFORM_GAUSSIAN_ROUNDJET && !(halfwidth > 0.0))
    return fail(c, LEE_ERR_ARG, "the round jet's half-width must be positive");
  if (type == LEE_WAVE_ACOUSTIC && dir >= c->cfg.num_dim)
    return fail(c, LEE_ERR_UNSUPPORTED, "an acoustic wave along direction %d of a %d-D case", dir, c->cfg.num_dim);
  Wave w{};
  w.type = type;
  w.form = form;
  w.dir = dir;
  w.amp = amplitude;
  w.k = 2.0 * acos(-1.0) / wavelength;  // math_constants::twopi (src/math/math.cpp:7-8)
  w.gfac = form == LEE_WAVEFORM_GAUSSIAN_ROUNDJET ? -log(2.0) / (halfwidth * halfwidth) : 0.0;
  w.p0 = 1.0 / c->cfg.gamma;
  c->wave = w;
  return LEE_OK;
}

int lee_set_axisymmetric(lee_ctx* c, int on, int axis) {
  if (!c) return LEE_ERR_ARG;
  if (c->prepared) return fail(c, LEE_ERR_STATE, "lee_set_axisymmetric after lee_prepare");
  if (!on) {
    c->axisym = false;
    return LEE_OK;
  }
  if (c->cfg.num_dim != 2) return fail(c, LEE_ERR_ARG, "Axisymmetry requires 2-D.");
  if (axis != 0) return fail(c, LEE_ERR_ARG, "The axis of symmetry should be x by definition of the coordinate system.");
  c->axisym = true;
  return LEE_OK;
}

int lee_set_source(lee_ctx* c, int kind, const double* params, int nparams) {
  if (!c) return LEE_ERR_ARG;
  if (c->prepared) return fail(c, LEE_ERR_STATE, "lee_set_source after lee_prepare");
  if (kind == LEE_SOURCE_NONE) {
    c->src_kind = kind;
    return LEE_OK;
  }
  if (kind == LEE_SOURCE_JET2D_HARMONIC) {
    for (auto& b : c->blk)
      if (b.src_mode == 1) return fail(c, LEE_ERR_UNSUPPORTED, "a block has its own monopole");
    c->src_kind = kind;
    return LEE_OK;
  }
  if (kind == LEE_SOURCE_DISTRIBUTED) {
    if (!params || nparams < 11) return fail(c, LEE_ERR_ARG, "distributed source takes 11 + lattice params");
    const int b = (int)params[0], cx = (int)params[2], cy = (int)params[3], cz = (int)params[4];
    if (b < 0 || b >= (int)c->blk.size()) return fail(c, LEE_ERR_ARG, "distributed source block");
    if (cx < 2 || cy < 2 || cz < 1 || (c->cfg.num_dim == 3 && cz < 2) || (c->cfg.num_dim == 2 && cz != 1))
      return fail(c, LEE_ERR_ARG, "distributed source lattice %d x %d x %d", cx, cy, cz);
    if ((long long)nparams != 11 + (long long)cx * cy * cz) return fail(c, LEE_ERR_ARG, "distributed source size");
    if (!(params[8] > 0.0 && params[9] > 0.0 && (cz == 1 || params[10] > 0.0)))
      return fail(c, LEE_ERR_ARG, "distributed source spacing must be positive");
    c->src_kind = kind;
    c->dsrc.assign(params, params + nparams);
    return LEE_OK;
  }
  if (kind != LEE_SOURCE_MONOPOLE || !params || nparams != 7) return fail(c, LEE_ERR_ARG, "monopole takes 7 params");
  if (!(params[5] > 0.0)) return fail(c, LEE_ERR_ARG, "monopole half-width must be positive");
  c->src_kind = kind;
  for (int q = 0; q < 7; ++q) c->src[q] = params[q];
  return LEE_OK;
}

int lee_set_block_source(lee_ctx* c, int b, int kind, const double* params, int nparams) {
  if (!c) return LEE_ERR_ARG;
  if (c->prepared) return fail(c, LEE_ERR_STATE, "lee_set_block_source after lee_prepare");
  if (b < 0 || b >= (int)c->blk.size()) return fail(c, LEE_ERR_ARG, "block index");
  if (c->src_kind == LEE_SOURCE_DISTRIBUTED) return fail(c, LEE_ERR_UNSUPPORTED, "a distributed source is set");
  BlockData& bk = c->blk[(size_t)b];
  if (kind == LEE_SOURCE_NONE) {
    bk.src_mode = 2;
    return LEE_OK;
  }
  if (kind != LEE_SOURCE_MONOPOLE || !params || nparams != 7) return fail(c, LEE_ERR_ARG, "monopole takes 7 params");
  if (!(params[5] > 0.0)) return fail(c, LEE_ERR_ARG, "monopole half-width must be positive");
  if (c->src_kind == LEE_SOURCE_JET2D_HARMONIC) return fail(c, LEE_ERR_UNSUPPORTED, "the 2-D jet source is set");
  bk.src_mode = 1;
  for (int q = 0; q < 7; ++q) bk.own_src[q] = params[q];
  if (c->src_kind == LEE_SOURCE_NONE) c->src_kind = LEE_SOURCE_MONOPOLE;  // other blocks keep none
  return LEE_OK;
}

int lee_upload_state(lee_ctx* c, int b, const double* const sol[5], int step, double time) {
  if (!c) return LEE_ERR_ARG;
  if (!c->prepared) return fail(c, LEE_ERR_STATE, "lee_prepare first");
  if (b < 0 || b >= (int)c->blk.size()) return fail(c, LEE_ERR_ARG, "block index");
  BlockData& bk = c->blk[(size_t)b];
  CK(cudaSetDevice(c->cfg.device));
  if (c->cfg.num_dim == 2)
    for (long long l = 0; l < bk.N; ++l)
      if (sol[3][l] != 0.0) return fail(c, LEE_ERR_ARG, "2-D state must have w' = 0");
  double* tmp = nullptr;
  if (c->comp) {
    const int rc = staging(c, &tmp);
    if (rc) return rc;
  }
  for (int v = 0; v < c->V; ++v) {
    if (!c->comp) {
      CK(cudaMemcpyAsync(bk.y[v], sol[slot_of(c->V, v)], (size_t)bk.N * 8, cudaMemcpyHostToDevice, c->stream));
    } else {
      CK(cudaMemcpyAsync(tmp, sol[slot_of(c->V, v)], (size_t)bk.N * 8, cudaMemcpyHostToDevice, c->stream));
      k_split<<<grid1d(bk.N), 256, 0, c->stream>>>(bk.N, (float*)bk.y[v], (float*)bk.comp[v], tmp);
      CK(cudaGetLastError());
    }
  }
  CK(cudaStreamSynchronize(c->stream));
  bk.rho_valid = false;  // the first stage takes rho'/rho_bar from the uploaded state
  bk.step = step;
  bk.time = time;
  c->step = c->blk[0].step;
  c->time = c->blk[0].time;
  c->uploaded = true;
  return LEE_OK;
}

int lee_download_state(lee_ctx* c, int b, double* const sol[5], int* step, double* time) {
  if (!c) return LEE_ERR_ARG;
  if (!c->prepared) return fail(c, LEE_ERR_STATE, "lee_prepare first");
  if (b < 0 || b >= (int)c->blk.size()) return fail(c, LEE_ERR_ARG, "block index");
  BlockData& bk = c->blk[(size_t)b];
  CK(cudaSetDevice(c->cfg.device));
  double* tmp = nullptr;
  if (c->comp) {
    const int rc = staging(c, &tmp);
    if (rc) return rc;
  }
  for (int v = 0; v < c->V; ++v) {
    if (!c->comp) {
      CK(cudaMemcpyAsync(sol[slot_of(c->V, v)], bk.y[v], (size_t)bk.N * 8, cudaMemcpyDeviceToHost, c->stream));
    } else {
      launch_to_double<float>(c->stream, bk.N, tmp, (const float*)bk.y[v],
                                                             (const float*)bk.comp[v]);
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(sol[slot_of(c->V, v)], tmp, (size_t)bk.N * 8, cudaMemcpyDeviceToHost, c->stream));
    }
  }
  CK(cudaStreamSynchronize(c->stream));
  if (c->cfg.num_dim == 2) memset(sol[3], 0, (size_t)bk.N * 8);
  if (step) *step = bk.step;
  if (time) *time = bk.time;
  return LEE_OK;
}

int lee_compute_dt(lee_ctx* c, double cfl, double* dt) {
  if (!c || !dt) return LEE_ERR_ARG;
  if (!c->prepared) return fail(c, LEE_ERR_STATE, "lee_prepare first");
  if (!(cfl > 0.0)) return fail(c, LEE_ERR_ARG, "cfl must be positive");
  std::vector<double> m;
  int rc = cfl_max(c, false, m, kDummyDt);
  if (rc) return rc;
  *dt = rescale(cfl, m[0]);
  return LEE_OK;
}

int lee_compute_cfl(lee_ctx* c, double dt, double* cfl) {
  if (!c || !cfl) return LEE_ERR_ARG;
  if (!c->prepared) return fail(c, LEE_ERR_STATE, "lee_prepare first");
  if (!(dt > 0.0)) return fail(c, LEE_ERR_ARG, "dt must be positive");
  std::vector<double> m;
  int rc = cfl_max(c, false, m, dt);
  if (rc) return rc;
  *cfl = m[0];
  return LEE_OK;
}

int lee_state_minmax(lee_ctx* c, double* mn, double* mx) {
  if (!c || !mn || !mx) return LEE_ERR_ARG;
  if (!c->prepared) return fail(c, LEE_ERR_STATE, "lee_prepare first");
  CK(cudaSetDevice(c->cfg.device));
  if (!c->d_report) {
    int rc = dalloc(c, &c->d_report, 10);
    if (rc) return rc;
  }
  double init[10];
  for (int q = 0; q < 10; ++q) init[q] = -DBL_MAX;
  CK(cudaMemcpyAsync(c->d_report, init, sizeof init, cudaMemcpyHostToDevice, c->stream));
  for (auto& bk : c->blk)
    for (int v = 0; v < c->V; ++v)
      CK(setup_state_minmax(bk.N, bk.y[v], c->comp ? bk.comp[v] : nullptr, c->comp, c->d_report + 2 * slot_of(c->V, v),
                            c->stream));
  double out[10];
  CK(cudaMemcpyAsync(out, c->d_report, sizeof out, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int q = 0; q < 5; ++q) {
    mn[q] = -out[2 * q];
    mx[q] = out[2 * q + 1];
  }
  if (c->cfg.num_dim == 2) mn[3] = mx[3] = 0.0;  // the w' slot of a 2-D state holds zeros
  return LEE_OK;
}

int lee_compute_dt_blocks(lee_ctx* c, double cfl, double* dt) {
  if (!c || !dt) return LEE_ERR_ARG;
  if (!c->prepared) return fail(c, LEE_ERR_STATE, "lee_prepare first");
  if (!(cfl > 0.0)) return fail(c, LEE_ERR_ARG, "cfl must be positive");
  std::vector<double> m;
  int rc = cfl_max(c, true, m, kDummyDt);
  if (rc) return rc;
  for (size_t b = 0; b < m.size(); ++b) dt[b] = rescale(cfl, m[b]);
  return LEE_OK;
}

int lee_get_info(lee_ctx* c, lee_info* info) {
  if (!c || !info) return LEE_ERR_ARG;
  if (!c->prepared) return fail(c, LEE_ERR_STATE, "lee_prepare first");
  memset(info, 0, sizeof *info);
  for (auto& b : c->blk) {
    info->points += b.N;
    info->num_coef_fields = std::max(info->num_coef_fields, b.n_coef_fields);
  }
  info->state_vars = c->V;
  info->bytes_per_value = (int)c->esz;
  info->device_bytes = c->device_bytes;
  info->tma_stage = 1;
  info->tma_filter = c->cfg.filter_scheme != LEE_FILTER_NONE ? 1 : 0;
  for (auto& b : c->blk) {
    info->tma_stage &= b.tma ? 1 : 0;
    info->tma_filter &= b.tma_filter ? 1 : 0;
  }
  info->stage_chunk = c->blk.empty() ? 0 : c->blk[0].stage_chunk;
  info->filter_chunk = c->blk.empty() ? 0 : c->blk[0].filter_chunk;
  info->filter_kernel = c->blk.empty() ? 0 : c->blk[0].filter_px;
  info->stage_kernel = c->blk.empty() ? 0 : c->blk[0].stage_px;
  info->filter_rows = c->blk.empty() ? 0 : (c->blk[0].filter_pair ? 3 : c->blk[0].filter_ry);
  info->increment_step = c->blk.empty() ? 0 : 1;
  for (const auto& b : c->blk) info->increment_step &= increment_step_applies(c, b) ? 1 : 0;
  info->batched = c->batch.active ? 1 : 0;
  if (c->batch.active) {
    batch_shape(c->batch.sshape, &info->batch_stage_tile[0], &info->batch_stage_tile[1]);
    batch_shape(c->batch.fshape, &info->batch_filter_tile[0], &info->batch_filter_tile[1]);
  }
  return LEE_OK;
}

int lee_set_stage_kernel(lee_ctx* c, int kind) {
  if (!c) return LEE_ERR_ARG;
  if (c->prepared) return fail(c, LEE_ERR_STATE, "lee_set_stage_kernel before lee_prepare");
  if (kind != -1 && kind != 1 && kind != 2) return fail(c, LEE_ERR_ARG, "stage kernel %d", kind);
  c->stage_kernel = kind;
  return LEE_OK;
}

int lee_set_filter_form(lee_ctx* c, int form) {
  if (!c) return LEE_ERR_ARG;
  if (c->prepared) return fail(c, LEE_ERR_STATE, "lee_set_filter_form before lee_prepare");
  if (form < 0 || form > 3) return fail(c, LEE_ERR_ARG, "filter form %d", form);
  c->filter_form = form;
  return LEE_OK;
}

int lee_set_filter_kernel(lee_ctx* c, int kind) {
  if (!c) return LEE_ERR_ARG;
  if (c->prepared) return fail(c, LEE_ERR_STATE, "lee_set_filter_kernel before lee_prepare");
  if (kind < -1) return fail(c, LEE_ERR_ARG, "filter kernel %d", kind);
  c->filter_kernel = kind;
  return LEE_OK;
}

int lee_get_setup(lee_ctx* c, int b, int what, double* out) {
  if (!c || !out) return LEE_ERR_ARG;
  if (!c->prepared) return fail(c, LEE_ERR_STATE, "lee_prepare first");
  if (b < 0 || b >= (int)c->blk.size()) return fail(c, LEE_ERR_ARG, "block index");
  BlockData& bk = c->blk[(size_t)b];
  const size_t N = (size_t)bk.N;
  CK(cudaSetDevice(c->cfg.device));
  if (what == LEE_SETUP_METRICS) {
    for (int q = 0; q < 9; ++q) CK(cudaMemcpyAsync(out + q * N, bk.d_met[q], N * 8, cudaMemcpyDeviceToHost, c->stream));
  } else if (what == LEE_SETUP_JACOBIAN) {
    CK(cudaMemcpyAsync(out, bk.d_jac, N * 8, cudaMemcpyDeviceToHost, c->stream));
  } else if (what == LEE_SETUP_MEAN_GRADIENT) {
    for (int q = 0; q < 5 * c->cfg.num_dim; ++q)
      CK(cudaMemcpyAsync(out + q * N, bk.d_grad[q], N * 8, cudaMemcpyDeviceToHost, c->stream));
  } else if (what == LEE_SETUP_SPONGE) {
    CK(cudaStreamSynchronize(c->stream));
    memset(out, 0, N * 8);
    for (auto& z : bk.bnd) {
      if (!is_sponge(z.kind)) continue;
      int b0 = z.hi[0] - z.lo[0] + 1, b1 = z.hi[1] - z.lo[1] + 1, b2 = z.hi[2] - z.lo[2] + 1;
      std::vector<double> h((size_t)b0 * b1 * b2);
      CK(cudaMemcpy(h.data(), z.d_sigma, h.size() * 8, cudaMemcpyDeviceToHost));
      for (int k = 0; k < b2; ++k)
        for (int j = 0; j < b1; ++j)
          for (int i = 0; i < b0; ++i)
            out[(size_t)(z.lo[0] + i) + (size_t)bk.nx * ((size_t)(z.lo[1] + j) + (size_t)bk.ny * (size_t)(z.lo[2] + k))] +=
                h[(size_t)i + (size_t)b0 * ((size_t)j + (size_t)b1 * (size_t)k)];
    }
  } else {
    return fail(c, LEE_ERR_ARG, "unknown setup selector %d", what);
  }
  CK(cudaStreamSynchronize(c->stream));
  return LEE_OK;
}

}  // extern "C"
