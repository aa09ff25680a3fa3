// One-time setup on the GPU (lee_prepare): FP64 metrics, Jacobian and mean gradients
// (metrics::compute, camille src/metrics/metrics.cpp:9-44; spatial::precompute_something,
// src/solver/spatial_discretization.cpp:2250-2271), sponge strengths, coefficient fields in the
// working precision, TMA eligibility and the kernel autotuning.
#include "lee_host.h"

using namespace lee;

namespace {

__global__ void k_add_box(int nx, int ny, int lo0, int lo1, int lo2, int b0, int b1, long long nb, const double* sig,
                          double* field) {
  for (long long lb = blockIdx.x * (long long)blockDim.x + threadIdx.x; lb < nb; lb += (long long)gridDim.x * blockDim.x) {
    const int i = lo0 + (int)(lb % b0), j = lo1 + (int)((lb / b0) % b1), k = lo2 + (int)(lb / ((long long)b0 * b1));
    field[i + (long long)nx * (j + (long long)ny * k)] += sig[lb];
  }
}

template <typename T>
__global__ void k_fill_const(long long n, T* out, T v) {
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < n; l += (long long)gridDim.x * blockDim.x)
    out[l] = v;
}

}  // namespace

namespace lee {

// metrics::compute with Thomas-Lombard products (src/metrics/metrics.cpp:9-251), the
// Jacobian (:255-328; 3-D determinant of oracle patch P1) and inverse metrics (:355-426).
int compute_metrics(lee_ctx* c, BlockData& b) {
  int dim = c->cfg.num_dim;
  int N = (int)b.N;
  cudaStream_t s = c->stream;
  double* xx[9] = {};
  int rc;
  for (int q = 0; q < 9; ++q) {
    if ((rc = dalloc(c, &b.d_met[q], (size_t)N))) return rc;
    if ((rc = dalloc(c, &b.d_minv[q], (size_t)N))) return rc;
    if ((rc = dalloc(c, &xx[q], (size_t)N))) return rc;
    CK(cudaMemsetAsync(b.d_met[q], 0, (size_t)N * 8, s));
    CK(cudaMemsetAsync(b.d_minv[q], 0, (size_t)N * 8, s));
  }
  if ((rc = dalloc(c, &b.d_jac, (size_t)N))) return rc;
  if ((rc = dalloc(c, &b.d_invjac, (size_t)N))) return rc;
  for (int ip = 0; ip < dim; ++ip)
    for (int ic = 0; ic < dim; ++ic)
      CK(setup_apply_dir(c->fd, b.nx, b.ny, b.nz, ic, b.d_xyz[ip], xx[ip * 3 + ic], nullptr, 1, s));
  double** m = b.d_met;
#define XX(p, q) xx[(p) * 3 + (q)]
#define MT(l, i) m[(l) * 3 + (i)]
  if (dim == 2) {
    CK(setup_axpby(N, MT(0, 0), 1.0, XX(1, 1), 0.0, nullptr, s));
    CK(setup_axpby(N, MT(0, 1), -1.0, XX(0, 1), 0.0, nullptr, s));
    CK(setup_axpby(N, MT(1, 0), -1.0, XX(1, 0), 0.0, nullptr, s));
    CK(setup_axpby(N, MT(1, 1), 1.0, XX(0, 0), 0.0, nullptr, s));
  } else {
    double *func = nullptr, *tmp = nullptr;
    if ((rc = dalloc(c, &func, (size_t)N))) return rc;
    if ((rc = dalloc(c, &tmp, (size_t)N))) return rc;
    double* const* z = b.d_xyz;
    // (product of a grid derivative and a coordinate, derivative direction,
    //  target metric, sign, assign (1) or accumulate (0)), in the order of
    //  compute_ThomasLombard_3D (src/metrics/metrics.cpp:133-251).
    struct Term { int pa, pb, cz, dir, tl, ti; double sign; int assign; };
    const Term terms[] = {
        {1, 1, 2, 2, 0, 0, 1.0, 1}, {1, 1, 2, 0, 2, 0, -1.0, 1},
        {0, 1, 2, 2, 0, 1, -1.0, 1}, {0, 1, 2, 0, 2, 1, 1.0, 1},
        {0, 1, 1, 2, 0, 2, 1.0, 1}, {0, 1, 1, 0, 2, 2, -1.0, 1},
        {1, 0, 2, 2, 1, 0, -1.0, 1}, {1, 0, 2, 1, 2, 0, 1.0, 0},
        {0, 0, 2, 2, 1, 1, 1.0, 1}, {0, 0, 2, 1, 2, 1, -1.0, 0},
        {0, 0, 1, 2, 1, 2, -1.0, 1}, {0, 0, 1, 1, 2, 2, 1.0, 0},
        {1, 2, 2, 1, 0, 0, -1.0, 0}, {1, 2, 2, 0, 1, 0, 1.0, 0},
        {0, 2, 2, 1, 0, 1, 1.0, 0}, {0, 2, 2, 0, 1, 1, -1.0, 0},
        {0, 2, 1, 1, 0, 2, -1.0, 0}, {0, 2, 1, 0, 1, 2, 1.0, 0},
    };
    for (size_t t = 0; t < sizeof terms / sizeof terms[0]; ++t) {
      const Term& T = terms[t];
      if (t % 2 == 0) CK(setup_mul(N, func, XX(T.pa, T.pb), z[T.cz], s));
      CK(setup_apply_dir(c->fd, b.nx, b.ny, b.nz, T.dir, func, tmp, nullptr, 1, s));
      if (T.assign)
        CK(setup_axpby(N, MT(T.tl, T.ti), T.sign, tmp, 0.0, nullptr, s));
      else
        CK(setup_axpby(N, MT(T.tl, T.ti), 1.0, MT(T.tl, T.ti), T.sign, tmp, s));
    }
  }
#undef XX
#undef MT
  double** d_xx = nullptr;
  double** d_mm = nullptr;
  double** d_mi = nullptr;
  if ((rc = dalloc(c, &d_xx, 9))) return rc;
  if ((rc = dalloc(c, &d_mm, 9))) return rc;
  if ((rc = dalloc(c, &d_mi, 9))) return rc;
  CK(cudaMemcpyAsync(d_xx, xx, sizeof xx, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_mm, b.d_met, sizeof b.d_met, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_mi, b.d_minv, sizeof b.d_minv, cudaMemcpyHostToDevice, s));
  CK(setup_jacobian(N, dim, d_xx, b.d_invjac, b.d_jac, s));
  CK(setup_inverse_metrics(N, dim, d_mm, d_mi, s));
  CK(cudaStreamSynchronize(s));
  return LEE_OK;
}

// Sum of the sponge strengths of every zone at each point (zones are added one after the
// other, so overlapping corners accumulate as in source::apply_bufferZone), in the working
// precision of the stage kernels.
int build_sigma_field(lee_ctx* c, BlockData& b) {
  double* f = nullptr;
  int rc = dalloc(c, &f, (size_t)b.N);
  if (rc) return rc;
  CK(cudaMemsetAsync(f, 0, (size_t)b.N * 8, c->stream));
  for (auto& z : b.bnd) {
    if (!is_sponge(z.kind)) continue;
    const int b0 = z.hi[0] - z.lo[0] + 1, b1 = z.hi[1] - z.lo[1] + 1, b2 = z.hi[2] - z.lo[2] + 1;
    const long long nb = (long long)b0 * b1 * b2;
    k_add_box<<<grid1d(nb), 256, 0, c->stream>>>(b.nx, b.ny, z.lo[0], z.lo[1], z.lo[2], b0, b1, nb, z.d_sigma, f);
    CK(cudaGetLastError());
  }
  if (!c->comp) {
    b.d_sigma_field = f;
    return LEE_OK;
  }
  float* g = nullptr;
  if ((rc = dalloc(c, &g, (size_t)b.N))) return rc;
  launch_convert<float>(c->stream, b.N, g, f);
  CK(cudaGetLastError());
  b.d_sigma_field = g;
  return LEE_OK;
}


}  // namespace lee

extern "C" {

int lee_prepare(lee_ctx* c) {
  if (!c) return LEE_ERR_ARG;
  if (c->prepared) return fail(c, LEE_ERR_STATE, "lee_prepare called twice");
  CK(cudaSetDevice(c->cfg.device));
  const int dim = c->cfg.num_dim;
  cudaStream_t s = c->stream;
  int rc;
  c->wave_time = false;
  for (auto& b : c->blk)
    for (auto& z : b.bnd) c->wave_time |= reads_wave(z.kind);
  if (c->wave_time && c->wave.type == LEE_WAVE_NONE)
    return fail(c, LEE_ERR_STATE, "a harmonic-wave boundary needs lee_set_harmonic_wave");
  for (auto& b : c->blk) {
    if (!b.set || !b.has_mean) return fail(c, LEE_ERR_STATE, "every block needs lee_set_block and lee_set_mean");
    const int N = (int)b.N;
    if ((rc = upload(c, &b.d_xyz[0], b.hx))) return rc;
    if ((rc = upload(c, &b.d_xyz[1], b.hy))) return rc;
    if ((rc = upload(c, &b.d_xyz[2], b.hz))) return rc;
    for (int v = 0; v < 5; ++v)
      if ((rc = upload(c, &b.d_mean[v], b.hmean[v]))) return rc;
    if ((rc = compute_metrics(c, b))) return rc;
    if (b.has_iblank) {
      if ((rc = dalloc(c, &b.d_iblank, (size_t)N))) return rc;
      CK(cudaMemcpyAsync(b.d_iblank, b.hib.data(), (size_t)N * sizeof(int), cudaMemcpyHostToDevice, s));
      CK(cudaStreamSynchronize(s));
    }
    // hole closures (receivers alone leave every closure as it is)
    if (b.has_holes) {
      std::vector<int8_t> code;
      int dims[3] = {b.nx, b.ny, b.nz};
      for (int d = 0; d < dim; ++d) {
        if (dims[d] == 1) continue;
        if (!closure_codes(c->fd, b, d, code)) return fail(c, LEE_ERR_ARG, "hole closure lacks fluid support");
        if ((rc = dalloc(c, &b.d_code_fd[d], (size_t)N))) return rc;
        CK(cudaMemcpyAsync(b.d_code_fd[d], code.data(), (size_t)N, cudaMemcpyHostToDevice, s));
        CK(cudaStreamSynchronize(s));
        if (c->cfg.filter_scheme != LEE_FILTER_NONE) {
          if (!closure_codes(c->flt, b, d, code))
            return fail(c, LEE_ERR_ARG, "filter hole closure lacks fluid support");
          if ((rc = dalloc(c, &b.d_code_flt[d], (size_t)N))) return rc;
          CK(cudaMemcpyAsync(b.d_code_flt[d], code.data(), (size_t)N, cudaMemcpyHostToDevice, s));
          CK(cudaStreamSynchronize(s));
        }
      }
    }
    // mean gradients (spatial::precompute_something, src/solver/spatial_discretization.cpp:2250-2271)
    double *sum = nullptr, *tmp = nullptr;
    if ((rc = dalloc(c, &sum, (size_t)N))) return rc;
    if ((rc = dalloc(c, &tmp, (size_t)N))) return rc;
    for (int v = 0; v < 5; ++v)
      for (int j = 0; j < dim; ++j) {
        if ((rc = dalloc(c, &b.d_grad[v * dim + j], (size_t)N))) return rc;
        CK(cudaMemsetAsync(sum, 0, (size_t)N * 8, s));
        for (int l = 0; l < dim; ++l) {
          CK(setup_apply_dir(c->fd, b.nx, b.ny, b.nz, l, b.d_mean[v], tmp, b.has_holes ? b.d_code_fd[l] : nullptr,
                             1, s));
          CK(setup_grad_accum(N, sum, b.d_met[l * 3 + j], tmp, s));
        }
        CK(setup_scale(N, b.d_grad[v * dim + j], sum, b.d_jac, s));
      }
    // J * metrics products read by the stage kernels
    for (int l = 0; l < dim; ++l)
      for (int x = 0; x < dim; ++x) {
        if ((rc = dalloc(c, &b.d_jm[l * 3 + x], (size_t)N))) return rc;
        CK(setup_mul(N, b.d_jm[l * 3 + x], b.d_jac, b.d_met[l * 3 + x], s));
      }
    // 1 / rho_bar with rho_bar = (gamma p_bar)^(1/gamma) exp(-s_bar) (src/core/state.cpp:712-714),
    // evaluated on the host with the reference's libm calls
    {
      if ((rc = dalloc(c, &b.d_rbi, (size_t)N))) return rc;
      std::vector<double> rbi((size_t)N);
      double g = c->cfg.gamma, gi = 1.0 / g;
      for (int l = 0; l < N; ++l) rbi[(size_t)l] = 1.0 / (pow(g * b.hmean[4][(size_t)l], gi) * exp(-b.hmean[0][(size_t)l]));
      CK(cudaMemcpyAsync(b.d_rbi, rbi.data(), (size_t)N * 8, cudaMemcpyHostToDevice, s));
      CK(cudaStreamSynchronize(s));
    }
    // sponge strengths
    double** d_xyzp = nullptr;
    if ((rc = dalloc(c, &d_xyzp, 3))) return rc;
    CK(cudaMemcpyAsync(d_xyzp, b.d_xyz, sizeof b.d_xyz, cudaMemcpyHostToDevice, s));
    for (auto& z : b.bnd) {
      if (!is_sponge(z.kind)) continue;
      size_t nb = (size_t)(z.hi[0] - z.lo[0] + 1) * (z.hi[1] - z.lo[1] + 1) * (z.hi[2] - z.lo[2] + 1);
      if ((rc = dalloc(c, &z.d_sigma, nb))) return rc;
      if (!z.sigma.empty()) {
        CK(cudaMemcpyAsync(z.d_sigma, z.sigma.data(), nb * 8, cudaMemcpyHostToDevice, s));
      } else {
        CK(setup_sigma(b.nx, b.ny, b.nz, d_xyzp, z.lo, z.hi, z.dir, z.end, c->cfg.sponge_order,
                       c->cfg.sponge_constant, z.d_sigma, s));
      }
      if (c->comp) {
        float* f = nullptr;
        if ((rc = dalloc(c, &f, nb))) return rc;
        launch_convert<float>(s, (long long)nb, f, z.d_sigma);
        CK(cudaGetLastError());
        z.d_sigma_t = f;
      }
      if (z.kind == LEE_SPONGE_FREUND_HARMONICWAVE) {
        if ((rc = dev_alloc(c, &z.d_ref, nb * (size_t)c->V * c->esz))) return rc;
        CK(cudaMemsetAsync(z.d_ref, 0, nb * (size_t)c->V * c->esz, s));
      }
    }
    // monopole spatial factor on the box where exp() is nonzero in FP64
    if (const double* mp = monopole_of(c, b)) {
      double ef = -log(2.0) / (mp[5] * mp[5]);
      double rmax = sqrt(746.0 / -ef);
      int lo[3] = {b.nx, b.ny, b.nz}, hi[3] = {-1, -1, -1};
      for (long long l = 0; l < b.N; ++l) {
        double dx = b.hx[(size_t)l] - mp[0], dy = b.hy[(size_t)l] - mp[1], dz = b.hz[(size_t)l] - mp[2];
        if (dx * dx + dy * dy + dz * dz <= rmax * rmax) {
          int ijk[3] = {(int)(l % b.nx), (int)((l / b.nx) % b.ny), (int)(l / ((long long)b.nx * b.ny))};
          for (int d = 0; d < 3; ++d) {
            lo[d] = std::min(lo[d], ijk[d]);
            hi[d] = std::max(hi[d], ijk[d]);
          }
        }
      }
      if (hi[0] >= 0) {
        size_t nb = (size_t)(hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1);
        if ((rc = dalloc(c, &b.d_src_g, nb))) return rc;
        CK(setup_monopole_g(b.nx, b.ny, d_xyzp, lo, hi, mp[0], mp[1], mp[2], ef, b.d_src_g, s));
        for (int d = 0; d < 3; ++d) { b.src_lo[d] = lo[d]; b.src_hi[d] = hi[d]; }
        if (c->comp) {
          float* f = nullptr;
          if ((rc = dalloc(c, &f, nb))) return rc;
          launch_convert<float>(s, (long long)nb, f, b.d_src_g);
          CK(cudaGetLastError());
          b.d_src_g_t = f;
        }
      }
    }
    if (c->src_kind == LEE_SOURCE_JET2D_HARMONIC && b.src_mode == 0) {
      // exp(-(Bx x x + By y y)) on the box where it is nonzero in FP64, computed here in FP64
      double amp, om, bx, by;
      jet2d_constants(c->cfg.gamma, &amp, &om, &bx, &by);
      auto arg = [&](long long l) {
        const double x = b.hx[(size_t)l], y = b.hy[(size_t)l];
        return -(bx * x * x + by * y * y);
      };
      int lo[3] = {b.nx, b.ny, b.nz}, hi[3] = {-1, -1, -1};
      for (long long l = 0; l < b.N; ++l)
        if (exp(arg(l)) != 0.0) {
          int ijk[3] = {(int)(l % b.nx), (int)((l / b.nx) % b.ny), (int)(l / ((long long)b.nx * b.ny))};
          for (int d = 0; d < 3; ++d) {
            lo[d] = std::min(lo[d], ijk[d]);
            hi[d] = std::max(hi[d], ijk[d]);
          }
        }
      if (hi[0] >= 0) {
        std::vector<double> g((size_t)(hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1));
        size_t q = 0;
        for (int k = lo[2]; k <= hi[2]; ++k)
          for (int j = lo[1]; j <= hi[1]; ++j)
            for (int i = lo[0]; i <= hi[0]; ++i) g[q++] = exp(arg(i + (long long)b.nx * (j + (long long)b.ny * k)));
        if ((rc = upload(c, &b.d_src_g, g))) return rc;
        for (int d = 0; d < 3; ++d) { b.src_lo[d] = lo[d]; b.src_hi[d] = hi[d]; }
        if (c->comp) {
          float* f = nullptr;
          if ((rc = dalloc(c, &f, g.size()))) return rc;
          launch_convert<float>(s, (long long)g.size(), f, b.d_src_g);
          CK(cudaGetLastError());
          b.d_src_g_t = f;
        }
      }
    }
    if (c->src_kind == LEE_SOURCE_DISTRIBUTED && (int)(&b - &c->blk[0]) == (int)c->dsrc[0]) {
      int lo[3], hi[3];
      std::vector<double> g;
      if (!distributed_box(c->dsrc, c->cfg.num_dim, b.nx, b.ny, b.nz, lo, hi))
        return fail(c, LEE_ERR_ARG, "the distributed source lattice covers no grid point");
      prolong(c->dsrc, c->cfg.num_dim, lo, hi, c->dsrc.data() + 11, g);
      if ((rc = upload(c, &b.d_src_g, g))) return rc;
      for (int d = 0; d < 3; ++d) { b.src_lo[d] = lo[d]; b.src_hi[d] = hi[d]; }
      if (c->comp) {
        float* f = nullptr;
        if ((rc = dalloc(c, &f, g.size()))) return rc;
        launch_convert<float>(s, (long long)g.size(), f, b.d_src_g);
        CK(cudaGetLastError());
        b.d_src_g_t = f;
      }
    }
    CK(cudaStreamSynchronize(s));
    // coefficient fields: constant ones become kernel constants
    b.n_coef_fields = 0;
    double jscale = 0.0;
    for (int l = 0; l < dim; ++l)
      for (int x = 0; x < dim; ++x) {
        double lo, hi;
        bool u, z;
        if ((rc = classify(c, b.d_jm[l * 3 + x], b.N, 1e300, &lo, &hi, &u, &z))) return rc;
        jscale = fmax(jscale, fmax(fabs(lo), fabs(hi)));
      }
    double mscale[5];
    for (int v = 0; v < 5; ++v) {
      double lo, hi;
      bool u, z;
      if ((rc = classify(c, b.d_mean[v], b.N, 1e300, &lo, &hi, &u, &z))) return rc;
      mscale[v] = fmax(fmax(fabs(lo), fabs(hi)), 1e-300) * jscale;
    }
    auto coef = [&](const double* f, double scale, Coef<double>* cd, Coef<float>* cf) -> int {
      if (c->comp) return make_coef<float>(c, b, f, scale, cf);
      return make_coef<double>(c, b, f, scale, cd);
    };
    for (int q = 0; q < 9; ++q) {
      b.cd_jm[q] = Coef<double>{nullptr, 0.0, 1};
      b.cf_jm[q] = Coef<float>{nullptr, 0.0f, 1};
      b.cd_gu[q] = Coef<double>{nullptr, 0.0, 1};
      b.cf_gu[q] = Coef<float>{nullptr, 0.0f, 1};
    }
    for (int q = 0; q < 3; ++q) {
      b.cd_ub[q] = b.cd_gs[q] = b.cd_gp[q] = Coef<double>{nullptr, 0.0, 1};
      b.cf_ub[q] = b.cf_gs[q] = b.cf_gp[q] = Coef<float>{nullptr, 0.0f, 1};
    }
    for (int l = 0; l < dim; ++l)
      for (int x = 0; x < dim; ++x)
        if ((rc = coef(b.d_jm[l * 3 + x], 1e-300, &b.cd_jm[l * 3 + x], &b.cf_jm[l * 3 + x]))) return rc;
    for (int x = 0; x < dim; ++x)
      if ((rc = coef(b.d_mean[1 + x], 1e-300, &b.cd_ub[x], &b.cf_ub[x]))) return rc;
    if ((rc = coef(b.d_mean[4], 1e-300, &b.cd_pb, &b.cf_pb))) return rc;
    if ((rc = coef(b.d_rbi, 1e-300, &b.cd_rbi, &b.cf_rbi))) return rc;
    for (int x = 0; x < dim; ++x) {
      if ((rc = coef(b.d_grad[0 * dim + x], mscale[0], &b.cd_gs[x], &b.cf_gs[x]))) return rc;
      if ((rc = coef(b.d_grad[4 * dim + x], mscale[4], &b.cd_gp[x], &b.cf_gp[x]))) return rc;
      for (int a = 0; a < dim; ++a)
        if ((rc = coef(b.d_grad[(1 + a) * dim + x], mscale[1 + a], &b.cd_gu[a * 3 + x], &b.cf_gu[a * 3 + x])))
          return rc;
    }
    b.need_rho = 0;
    for (int q = 0; q < 9; ++q) b.need_rho |= c->comp ? !b.cf_gu[q].zero : !b.cd_gu[q].zero;
    if (b.need_rho && (rc = dev_alloc(c, &b.rho, (size_t)b.N * c->esz))) return rc;
    b.rho_valid = false;
    if ((rc = scalar_setup(c, b))) return rc;
    // state buffers
    if ((rc = alloc_fields(c, b.y, b.N))) return rc;
    if ((rc = alloc_fields(c, b.acc, b.N))) return rc;
    if ((rc = alloc_fields(c, b.zb[0], b.N))) return rc;
    if ((rc = alloc_fields(c, b.zb[1], b.N))) return rc;
    if (c->comp) {
      if ((rc = alloc_fields(c, b.comp, b.N))) return rc;
      if ((rc = alloc_fields(c, b.dsum, b.N))) return rc;
    }
    // TMA-staged kernels: the 4th-order difference, rows of 16-byte multiples; on a block with
    // holes the classes come from the closure codes (one-point stage kernel, one-row filter)
    const bool rows16 = ((size_t)b.nx * c->esz) % 16 == 0;
    b.tiles_x = (b.nx + kTileX - 1) / kTileX;
    b.tiles_y = (b.ny + kTileY - 1) / kTileY;
    // (the TMA stage kernel addresses points with 32-bit offsets)
    // (and the harmonic-wave sponge, an RHS term of the generic kernel's zone loop, is absent)
    bool wave_zone = false;
    for (auto& z : b.bnd) wave_zone |= z.kind == LEE_SPONGE_FREUND_HARMONICWAVE;
    b.tma = c->wst_ok && rows16 && (unsigned long long)b.N < (1ull << 32) && !wave_zone && !c->axisym;
    b.tma_filter = c->wfl_ok && rows16 && c->cfg.filter_scheme != LEE_FILTER_NONE &&
                   (unsigned long long)b.N < (1ull << 32) && (!b.has_holes || 1 + 2 * c->flt.nb < 12);
    // the kernels are a fixed choice (they round differently, and two contexts of one case give
    // the same bits): the scalar fused filter unless another is asked for
    b.filter_vec = b.tma_filter && c->wfl_sym && !b.has_holes;
    b.filter_px = 0;
    if (c->filter_kernel >= 0 && b.tma_filter) {
      int px[2];
      const int n = filter_vec_widths(c->esz, px);
      bool ok = c->filter_kernel == 0;
      for (int q = 0; q < n; ++q) ok |= b.filter_vec && c->filter_kernel == px[q];
      if (!ok)
        return fail(c, LEE_ERR_UNSUPPORTED, "filter kernel %d is not available for block %d", c->filter_kernel,
                    (int)(&b - c->blk.data()));
      b.filter_px = c->filter_kernel;
    }
    b.filter_ry = 1;
    // the two-point form: compensated FP32, 3-D, no holes, even nxi, the scalar kernel's place
    b.filter_pair_ok = b.tma_filter && c->comp && c->cfg.num_dim == 3 && !b.has_holes && b.nx % 2 == 0 &&
                       b.filter_px == 0 && filter_pair_half_width(c->hf);
    b.filter_pair = false;
    if (c->filter_form > 0 && b.tma_filter) {
      // the two-row and two-point forms take neither holes nor the vector kernel's groups
      if ((c->filter_form == 2 && (b.filter_px > 0 || b.has_holes)) || (c->filter_form == 3 && !b.filter_pair_ok))
        return fail(c, LEE_ERR_UNSUPPORTED, "filter form %d is not available for block %d", c->filter_form,
                    (int)(&b - c->blk.data()));
      b.filter_ry = c->filter_form == 2 ? 2 : 1;
      b.filter_pair = c->filter_form == 3;
    }
    b.tfilter_ry = b.filter_ry;
    b.tfilter_chunk = 0;
    set_filter_tiles(c, b);
    if (b.tma) {
      // coefficient-layout traits of the stage kernel
      bool jmf = false, uni = true, spg = false;
      for (int q = 0; q < 9; ++q) jmf |= (c->comp ? b.cf_jm[q].p : (const void*)b.cd_jm[q].p) != nullptr;
      auto is_const = [&](const Coef<double>& d, const Coef<float>& f) { return c->comp ? !f.p : !d.p; };
      auto is_zero = [&](const Coef<double>& d, const Coef<float>& f) { return c->comp ? f.zero : d.zero; };
      for (int q = 0; q < 3; ++q) {
        uni &= is_const(b.cd_ub[q], b.cf_ub[q]);
        uni &= is_zero(b.cd_gs[q], b.cf_gs[q]) != 0 && is_zero(b.cd_gp[q], b.cf_gp[q]) != 0;
      }
      for (int q = 0; q < 9; ++q) uni &= is_zero(b.cd_gu[q], b.cf_gu[q]) != 0;
      uni &= is_const(b.cd_pb, b.cf_pb) && is_const(b.cd_rbi, b.cf_rbi) && !b.need_rho;
      for (auto& z : b.bnd) spg |= is_sponge(z.kind);
      b.traits = kTrTma | (jmf ? kTrJmField : 0) | (uni ? kTrUniform : 0) | (spg ? kTrSponge : 0);
      b.stage_pair = c->comp && uni && b.nx % 2 == 0 && !b.has_holes;
      b.stage_px = b.stage_pair ? 2 : 1;
      if (c->stage_kernel > 0) {
        if (c->stage_kernel != 1 && !(c->stage_kernel == 2 && b.stage_pair))
          return fail(c, LEE_ERR_UNSUPPORTED, "stage kernel %d is not available for block %d", c->stage_kernel,
                      (int)(&b - c->blk.data()));
        b.stage_px = c->stage_kernel;
      }
      if (spg && (rc = build_sigma_field(c, b))) return rc;
      if (jmf) {
        // the TMA kernel reads every J*metrics entry as a field when one is: constant entries
        // become fields holding their constant
        for (int l = 0; l < dim; ++l)
          for (int x = 0; x < dim; ++x) {
            const int q = l * 3 + x;
            if (c->comp && !b.cf_jm[q].p) {
              float* f = nullptr;
              if ((rc = dalloc(c, &f, (size_t)b.N))) return rc;
              k_fill_const<float><<<grid1d(b.N), 256, 0, c->stream>>>(b.N, f, b.cf_jm[q].c);
              CK(cudaGetLastError());
              b.cf_jm[q].p = f;
            } else if (!c->comp && !b.cd_jm[q].p) {
              double* f = nullptr;
              if ((rc = dalloc(c, &f, (size_t)b.N))) return rc;
              k_fill_const<double><<<grid1d(b.N), 256, 0, c->stream>>>(b.N, f, b.cd_jm[q].c);
              CK(cudaGetLastError());
              b.cd_jm[q].p = f;
            }
          }
      }
    }
    b.stage_chunk = b.filter_chunk = b.nz;
    if ((b.tma || b.tma_filter) && (rc = ensure_encoder(c))) return rc;
    if ((rc = c->comp ? autotune<float>(c, b) : autotune<double>(c, b))) return rc;
  }
  if (c->blk.size() > 1 && c->batching && batch_eligible(c)) {
    rc = c->comp ? batch_setup<float>(c) : batch_setup<double>(c);
    if (rc) return rc;
  }
  if (c->ovs.n > 0) {
    auto& o = c->ovs;
    const size_t n = (size_t)o.n;
    if ((rc = dalloc(c, &o.d_rb, n)) || (rc = dalloc(c, &o.d_db, n)) || (rc = dalloc(c, &o.d_rl, n)) ||
        (rc = dalloc(c, &o.d_dl, n)) || (rc = dalloc(c, &o.d_wt, n * o.W)) || (rc = dalloc(c, &o.d_buf, n * c->V)))
      return rc;
    CK(cudaMemcpyAsync(o.d_rb, o.rb.data(), n * sizeof(int), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(o.d_db, o.db.data(), n * sizeof(int), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(o.d_rl, o.rl.data(), n * sizeof(long long), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(o.d_dl, o.dl.data(), n * sizeof(long long), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(o.d_wt, o.wt.data(), n * o.W * sizeof(double), cudaMemcpyHostToDevice, s));
    // one kernel is enough when no stencil reads a receiver: the sums then cannot see a value
    // written in the same update
    o.fused = true;
    for (size_t r = 0; r < n && o.fused; ++r) {
      const BlockData& dk = c->blk[(size_t)o.db[r]];
      if (dk.hib.empty()) continue;
      for (int w3 = 0; w3 < o.w[2] && o.fused; ++w3)
        for (int w2 = 0; w2 < o.w[1] && o.fused; ++w2)
          for (int w1 = 0; w1 < o.w[0]; ++w1) {
            const long long l1 = o.dl[r] + w1 + (long long)w2 * dk.nx + (long long)w3 * dk.nx * dk.ny;
            if (dk.hib[(size_t)l1] == -1) {
              o.fused = false;
              break;
            }
          }
    }
  }
  CK(cudaStreamSynchronize(s));
  if (c->blk.size() > 1 && c->side.empty()) {
    const size_t S = std::min<size_t>(c->blk.size(), 8);
    for (size_t q = 0; q < S; ++q) {
      cudaStream_t sd = nullptr;
      CK(cudaStreamCreateWithFlags(&sd, cudaStreamNonBlocking));
      c->side.push_back(sd);
    }
    for (size_t q = 0; q <= S; ++q) {
      cudaEvent_t e = nullptr;
      CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      c->side_ev.push_back(e);
    }
  }
  c->prepared = true;
  return LEE_OK;
}

}  // extern "C"
