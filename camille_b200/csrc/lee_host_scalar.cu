// Passive scalars (PHYSICAL_MODEL = LEE_SCALAR): n slots Z_k' after p' (camille
// src/core/input.cpp:113-119, :768-773). Their right-hand side (compute_RHS_linearized_Euler_scalar,
// src/solver/spatial_discretization.cpp:2134-2158) reads the LEE slots only through u' at the
// point, and nothing in the LEE slots reads them, so they run beside the LEE kernels: one scalar
// stage launch after each LEE stage launch, their BC rows after the LEE slots' (Neumann rows for
// the Neumann, slip-wall and centerline lines, bc::apply_BC src/solver/boundary_condition.cpp:
// 116-160; zero on the Dirichlet lines, :213-228 and :264-265), the overset interpolation
// (num_vars_2interpolate = num_vars_sol, src/overset/overset.cpp:62) and the filter
// (spatial::apply_filter over num_vars_sol, src/solver/temporal_discretization.cpp:358) with the
// generic kernels, in chunks of up to V fields. The scalar buffers keep fixed roles.
#include "lee_host.h"

using namespace lee;

namespace {

__global__ void k_split_sc(long long n, float* y, float* e, const double* in) {
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < n; l += (long long)gridDim.x * blockDim.x) {
    const float r = (float)in[l];
    y[l] = r;
    e[l] = (float)(in[l] - (double)r);
  }
}

int dev_field(lee_ctx* c, void** f, long long N) {
  int rc = dev_alloc(c, f, (size_t)N * c->esz);
  if (rc) return rc;
  CK(cudaMemsetAsync(*f, 0, (size_t)N * c->esz, c->stream));
  return LEE_OK;
}

}  // namespace

namespace lee {

// Mean scalars on the device, their physical gradients as the LEE means' (FP64, with the hole
// closures: spatial::precompute_something, src/solver/spatial_discretization.cpp:2250-2271), the
// coefficient form of the gradients, and the slots' buffers.
int scalar_setup(lee_ctx* c, BlockData& b) {
  if (!c->nsc) return LEE_OK;
  if (b.hzmean.size() != (size_t)c->nsc * (size_t)b.N) return fail(c, LEE_ERR_STATE, "lee_set_mean_scalars first");
  const int dim = c->cfg.num_dim;
  const int N = (int)b.N;
  cudaStream_t s = c->stream;
  int rc;
  double *sum = nullptr, *tmp = nullptr;
  if ((rc = dalloc(c, &sum, (size_t)N)) || (rc = dalloc(c, &tmp, (size_t)N))) return rc;
  double jscale = 0.0;
  for (int l = 0; l < dim; ++l)
    for (int x = 0; x < dim; ++x) {
      double lo, hi;
      bool u, z;
      if ((rc = classify(c, b.d_jm[l * 3 + x], b.N, 1e300, &lo, &hi, &u, &z))) return rc;
      jscale = fmax(jscale, fmax(fabs(lo), fabs(hi)));
    }
  for (int k = 0; k < c->nsc; ++k) {
    std::vector<double> h(b.hzmean.begin() + (size_t)k * b.N, b.hzmean.begin() + (size_t)(k + 1) * b.N);
    if ((rc = upload(c, &b.d_zmean[k], h))) return rc;
    double lo, hi;
    bool u, z;
    if ((rc = classify(c, b.d_zmean[k], b.N, 1e300, &lo, &hi, &u, &z))) return rc;
    const double mscale = fmax(fmax(fabs(lo), fabs(hi)), 1e-300) * jscale;
    for (int j = 0; j < dim; ++j) {
      if ((rc = dalloc(c, &b.d_zgrad[k * 3 + j], (size_t)N))) return rc;
      CK(cudaMemsetAsync(sum, 0, (size_t)N * 8, s));
      for (int l = 0; l < dim; ++l) {
        CK(setup_apply_dir(c->fd, b.nx, b.ny, b.nz, l, b.d_zmean[k], tmp, b.has_holes ? b.d_code_fd[l] : nullptr, 1,
                           s));
        CK(setup_grad_accum(N, sum, b.d_met[l * 3 + j], tmp, s));
      }
      CK(setup_scale(N, b.d_zgrad[k * 3 + j], sum, b.d_jac, s));
    }
    for (int j = 0; j < 3; ++j) {
      b.cd_gz[k][j] = Coef<double>{nullptr, 0.0, 1};
      b.cf_gz[k][j] = Coef<float>{nullptr, 0.0f, 1};
    }
    for (int j = 0; j < dim; ++j) {
      rc = c->comp ? make_coef<float>(c, b, b.d_zgrad[k * 3 + j], mscale, &b.cf_gz[k][j])
                   : make_coef<double>(c, b, b.d_zgrad[k * 3 + j], mscale, &b.cd_gz[k][j]);
      if (rc) return rc;
    }
    if ((rc = dev_field(c, &b.zy[k], b.N)) || (rc = dev_field(c, &b.zacc[k], b.N)) ||
        (rc = dev_field(c, &b.zzb[0][k], b.N)) || (rc = dev_field(c, &b.zzb[1][k], b.N)) ||
        (rc = dev_field(c, &b.zf[k], b.N)))
      return rc;
    if (c->comp && ((rc = dev_field(c, &b.zcomp[k], b.N)) || (rc = dev_field(c, &b.zdsum[k], b.N)))) return rc;
  }
  CK(cudaStreamSynchronize(s));
  return LEE_OK;
}

template <typename T>
int scalar_stage(lee_ctx* c, BlockData& b, int s, int ns, double h, double bcoef, double acoef, void* const* lee_zin) {
  if (!c->nsc) return LEE_OK;
  const bool dbl = std::is_same<T, double>::value;
  ScalarParams<T> p;
  memset(&p, 0, sizeof p);
  p.nx = b.nx; p.ny = b.ny; p.nz = b.nz;
  p.dim = c->cfg.num_dim;
  p.n = c->nsc;
  p.stage = s;
  p.last = s == ns - 1;
  p.h = (T)h; p.b = (T)bcoef; p.a = (T)acoef;
  void* const* zin = s == 0 ? b.zy : b.zzb[(s + 1) % 2];
  for (int k = 0; k < c->nsc; ++k) {
    p.zin[k] = (const T*)zin[k];
    p.yn[k] = (const T*)b.zy[k];
    p.acc[k] = (T*)b.zacc[k];
    p.zout[k] = (T*)b.zzb[s % 2][k];
    p.comp[k] = (T*)b.zcomp[k];
    for (int j = 0; j < 3; ++j) p.gz[k][j] = dbl ? *(const Coef<T>*)&b.cd_gz[k][j] : *(const Coef<T>*)&b.cf_gz[k][j];
  }
  for (int x = 0; x < p.dim; ++x) p.uin[x] = (const T*)lee_zin[1 + x];
  const Coef<T>* jm = dbl ? (const Coef<T>*)b.cd_jm : (const Coef<T>*)b.cf_jm;
  const Coef<T>* ub = dbl ? (const Coef<T>*)b.cd_ub : (const Coef<T>*)b.cf_ub;
  for (int q = 0; q < 9; ++q) p.jm[q] = jm[q];
  for (int q = 0; q < 3; ++q) p.ubar[q] = ub[q];
  for (auto& z : b.bnd) {
    if (!is_sponge(z.kind)) continue;
    Zone<T>& zn = p.zones[p.nzones++];
    for (int d = 0; d < 3; ++d) { zn.lo[d] = z.lo[d]; zn.hi[d] = z.hi[d]; }
    zn.sig = dbl ? (const T*)z.d_sigma : (const T*)z.d_sigma_t;
    zn.ref = nullptr;  // the scalars relax to zero
  }
  for (int d = 0; d < 3; ++d) p.code[d] = b.has_holes ? b.d_code_fd[d] : nullptr;
  p.iblank = b.has_holes ? b.d_iblank : nullptr;
  p.fd = c->fd;
  CK(launch_scalar_stage<T>(p, c->comp ? 1 : 0, c->stream));
  c->stats.kernel_launches += 1;
  return LEE_OK;
}

// The stage output of the scalar slots: z_{s+1}, or after the last stage y_next (FP64) or the
// pair (y_pre, e) (compensated).
template <typename T>
static void scalar_target(lee_ctx* c, BlockData& b, int s, int ns, void** f, void** e) {
  const bool last = s == ns - 1;
  for (int k = 0; k < c->nsc; ++k) {
    f[k] = (last && !c->comp) ? b.zacc[k] : b.zzb[s % 2][k];
    e[k] = (last && c->comp) ? b.zacc[k] : nullptr;
  }
}

template <typename T>
int scalar_bcs(lee_ctx* c, BlockData& b, int s, int ns) {
  if (!c->nsc) return LEE_OK;
  void* f[kMaxScalars] = {};
  void* e[kMaxScalars] = {};
  scalar_target<T>(c, b, s, ns, f, e);
  for (auto& z : b.bnd) {
    if (!is_bc_line(z.kind)) continue;
    const bool dir = z.kind == LEE_BC_DIRICHLET_ALLZERO || z.kind == LEE_BC_DIRICHLET_HARMONICWAVE;
    for (int k0 = 0; k0 < c->nsc; k0 += c->V) {
      const int nk = std::min(c->V, c->nsc - k0);
      BcParams<T> p;
      fill_bc_params<T>(c, b, z, f, nullptr, p);  // the fields are set below
      p.kind = dir ? LEE_BC_DIRICHLET_ALLZERO : LEE_BC_NEUMANN;
      p.V = nk;
      for (int v = 0; v < kMaxVars; ++v) {
        p.y[v] = v < nk ? (T*)f[k0 + v] : nullptr;
        p.e[v] = v < nk ? (T*)e[k0 + v] : nullptr;
      }
      CK(launch_bc<T>(p, c->stream));
      c->stats.kernel_launches += 1;
    }
  }
  return LEE_OK;
}

template <typename T>
int scalar_overset(lee_ctx* c, int s, int ns) {
  if (!c->nsc || c->ovs.n <= 0) return LEE_OK;
  // chunks of at most V fields: the interpolants' buffer holds V per receiver
  for (int k0 = 0; k0 < c->nsc; k0 += c->V) {
    const int nk = std::min(c->V, c->nsc - k0);
    OvsParams<T> op;
    memset(&op, 0, sizeof op);
    op.n = c->ovs.n; op.W = c->ovs.W; op.V = nk; op.fused = c->ovs.fused ? 1 : 0;
    for (int d = 0; d < 3; ++d) op.w[d] = c->ovs.w[d];
    op.rb = c->ovs.d_rb; op.rl = c->ovs.d_rl; op.db = c->ovs.d_db; op.dl = c->ovs.d_dl;
    op.wt = c->ovs.d_wt; op.buf = c->ovs.d_buf;
    op.pair = (s == ns - 1 && c->comp) ? 1 : 0;
    for (size_t bi = 0; bi < c->blk.size(); ++bi) {
      BlockData& b = c->blk[bi];
      void* f[kMaxScalars] = {};
      void* e[kMaxScalars] = {};
      scalar_target<T>(c, b, s, ns, f, e);
      for (int v = 0; v < nk; ++v) {
        op.y[bi][v] = (T*)f[k0 + v];
        op.e[bi][v] = (T*)e[k0 + v];
      }
      op.nx[bi] = b.nx;
      op.ny[bi] = b.ny;
    }
    CK(launch_overset<T>(op, c->stream));
    c->stats.kernel_launches += op.fused ? 1 : 2;
  }
  return LEE_OK;
}

// The filter of the scalar slots after the last stage, into y (and, compensated, its carried
// error), with the hole mask on the last pass; without a filter, y_next (or the pair) is y.
template <typename T>
int scalar_filter(lee_ctx* c, BlockData& b, int ns) {
  if (!c->nsc) return LEE_OK;
  const size_t bytes = (size_t)b.N * c->esz;
  void** pre = c->comp ? b.zzb[(ns - 1) % 2] : b.zacc;  // y_next, or y_pre of the pair
  if (c->cfg.filter_scheme == LEE_FILTER_NONE) {
    for (int k = 0; k < c->nsc; ++k) {
      CK(cudaMemcpyAsync(b.zy[k], pre[k], bytes, cudaMemcpyDeviceToDevice, c->stream));
      if (c->comp) CK(cudaMemcpyAsync(b.zcomp[k], b.zacc[k], bytes, cudaMemcpyDeviceToDevice, c->stream));
    }
    return LEE_OK;
  }
  const int dims[3] = {b.nx, b.ny, b.nz};
  int passes[3], np = 0;
  for (int d = 0; d < c->cfg.num_dim; ++d)
    if (dims[d] > 1) passes[np++] = d;
  for (int k0 = 0; k0 < c->nsc; k0 += c->V) {
    const int nk = std::min(c->V, c->nsc - k0);
    void** src = pre + k0;
    for (int q = 0; q < np; ++q) {
      FilterParams<T> fp;
      memset(&fp, 0, sizeof fp);
      fp.nx = b.nx; fp.ny = b.ny; fp.nz = b.nz;
      fp.V = nk;
      fp.dir = passes[q];
      fp.first = q == 0;
      fp.last = q == np - 1;
      fp.blend = (T)c->cfg.filter_blend;
      fp.code = b.has_holes ? b.d_code_flt[passes[q]] : nullptr;
      fp.iblank = b.has_holes ? b.d_iblank : nullptr;
      fp.op = c->comp ? c->fltd : c->flt;
      // the last pass writes y; the ones before alternate so that no pass reads what it writes
      void** dst = ((np - 1 - q) % 2 == 0) ? b.zy + k0 : b.zf + k0;
      for (int v = 0; v < nk; ++v) {
        fp.in[v] = (const T*)src[v];
        fp.out[v] = (T*)dst[v];
        fp.y0[v] = (const T*)pre[k0 + v];
        fp.dsum[v] = (T*)b.zdsum[k0 + v];
        fp.dsum_in[v] = (const T*)b.zdsum[k0 + v];
        fp.comp[v] = c->comp ? (T*)b.zcomp[k0 + v] : nullptr;
        fp.err[v] = c->comp ? (const T*)b.zacc[k0 + v] : nullptr;
      }
      CK(launch_filter_pass<T>(fp, c->comp ? 1 : 0, c->stream));
      c->stats.kernel_launches += 1;
      src = dst;
    }
  }
  return LEE_OK;
}

template int scalar_stage<float>(lee_ctx*, BlockData&, int, int, double, double, double, void* const*);
template int scalar_stage<double>(lee_ctx*, BlockData&, int, int, double, double, double, void* const*);
template int scalar_bcs<float>(lee_ctx*, BlockData&, int, int);
template int scalar_bcs<double>(lee_ctx*, BlockData&, int, int);
template int scalar_overset<float>(lee_ctx*, int, int);
template int scalar_overset<double>(lee_ctx*, int, int);
template int scalar_filter<float>(lee_ctx*, BlockData&, int);
template int scalar_filter<double>(lee_ctx*, BlockData&, int);

}  // namespace lee

extern "C" {

int lee_set_scalars(lee_ctx* c, int n) {
  if (!c) return LEE_ERR_ARG;
  if (n < 0 || n > kMaxScalars) return fail(c, LEE_ERR_ARG, "0 <= n <= %d scalars", kMaxScalars);
  for (auto& b : c->blk)
    if (b.set) return fail(c, LEE_ERR_STATE, "lee_set_scalars before lee_set_block");
  c->nsc = n;
  return LEE_OK;
}

int lee_set_mean_scalars(lee_ctx* c, int b, const double* const* zbar) {
  if (!c) return LEE_ERR_ARG;
  if (c->prepared) return fail(c, LEE_ERR_STATE, "lee_set_mean_scalars after lee_prepare");
  if (b < 0 || b >= (int)c->blk.size() || !c->blk[(size_t)b].set) return fail(c, LEE_ERR_STATE, "lee_set_block first");
  if (!c->nsc || !zbar) return fail(c, LEE_ERR_ARG, "no scalars");
  BlockData& bk = c->blk[(size_t)b];
  bk.hzmean.resize((size_t)c->nsc * (size_t)bk.N);
  for (int k = 0; k < c->nsc; ++k) {
    if (!zbar[k]) return fail(c, LEE_ERR_ARG, "null mean scalar field");
    std::copy(zbar[k], zbar[k] + bk.N, bk.hzmean.begin() + (size_t)k * bk.N);
  }
  return LEE_OK;
}

int lee_upload_scalars(lee_ctx* c, int b, const double* const* z) {
  if (!c) return LEE_ERR_ARG;
  if (!c->prepared) return fail(c, LEE_ERR_STATE, "lee_prepare first");
  if (b < 0 || b >= (int)c->blk.size()) return fail(c, LEE_ERR_ARG, "block index");
  if (!c->nsc || !z) return fail(c, LEE_ERR_ARG, "no scalars");
  BlockData& bk = c->blk[(size_t)b];
  CK(cudaSetDevice(c->cfg.device));
  double* tmp = nullptr;
  if (c->comp) {
    const int rc = staging(c, &tmp);
    if (rc) return rc;
  }
  for (int k = 0; k < c->nsc; ++k) {
    if (!z[k]) return fail(c, LEE_ERR_ARG, "null scalar field");
    if (!c->comp) {
      CK(cudaMemcpyAsync(bk.zy[k], z[k], (size_t)bk.N * 8, cudaMemcpyHostToDevice, c->stream));
    } else {
      CK(cudaMemcpyAsync(tmp, z[k], (size_t)bk.N * 8, cudaMemcpyHostToDevice, c->stream));
      k_split_sc<<<grid1d(bk.N), 256, 0, c->stream>>>(bk.N, (float*)bk.zy[k], (float*)bk.zcomp[k], tmp);
      CK(cudaGetLastError());
    }
  }
  CK(cudaStreamSynchronize(c->stream));
  return LEE_OK;
}

int lee_download_scalars(lee_ctx* c, int b, double* const* z) {
  if (!c) return LEE_ERR_ARG;
  if (!c->prepared) return fail(c, LEE_ERR_STATE, "lee_prepare first");
  if (b < 0 || b >= (int)c->blk.size()) return fail(c, LEE_ERR_ARG, "block index");
  if (!c->nsc || !z) return fail(c, LEE_ERR_ARG, "no scalars");
  BlockData& bk = c->blk[(size_t)b];
  CK(cudaSetDevice(c->cfg.device));
  double* tmp = nullptr;
  if (c->comp) {
    const int rc = staging(c, &tmp);
    if (rc) return rc;
  }
  for (int k = 0; k < c->nsc; ++k) {
    if (!c->comp) {
      CK(cudaMemcpyAsync(z[k], bk.zy[k], (size_t)bk.N * 8, cudaMemcpyDeviceToHost, c->stream));
    } else {
      launch_to_double<float>(c->stream, bk.N, tmp, (const float*)bk.zy[k], (const float*)bk.zcomp[k]);
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(z[k], tmp, (size_t)bk.N * 8, cudaMemcpyDeviceToHost, c->stream));
    }
  }
  CK(cudaStreamSynchronize(c->stream));
  return LEE_OK;
}

}  // extern "C"
