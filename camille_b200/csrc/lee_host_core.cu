// Host helpers shared by the C ABI's translation units: error reporting, device allocation, the
// difference and filter operator tables with their closure codes, per-launch timing marks, the
// classification of FP64 coefficient fields into per-point fields or constants, the fields of one
// stage launch, and the source terms' time factors.
#include "lee_host.h"

using namespace lee;

namespace {

template <typename T>
__global__ void k_convert(long long n, T* out, const double* in) {
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < n; l += (long long)gridDim.x * blockDim.x)
    out[l] = (T)in[l];
}

// flag = 1 when some element of the fields is not finite (vector loads: the fields are
// cudaMalloc'd, and n is a multiple of the vector width or the tail is read one by one)
template <typename T>
__global__ void k_nonfinite(long long n, int nf, const T* f0, const T* f1, const T* f2, const T* f3, const T* f4,
                            const T* f5, const T* f6, const T* f7, const T* f8, const T* f9, int* flag) {
  const T* f[10] = {f0, f1, f2, f3, f4, f5, f6, f7, f8, f9};
  using V4 = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
  constexpr int W = (int)(sizeof(V4) / sizeof(T));
  const long long nv = n / W;
  bool bad = false;
  for (int q = 0; q < nf; ++q) {
    const V4* v = reinterpret_cast<const V4*>(f[q]);
    for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < nv; l += (long long)gridDim.x * blockDim.x) {
      const V4 x = v[l];
      const T* e = reinterpret_cast<const T*>(&x);
#pragma unroll
      for (int w = 0; w < W; ++w) bad |= !isfinite(e[w]);
    }
    for (long long l = nv * W + blockIdx.x * (long long)blockDim.x + threadIdx.x; l < n;
         l += (long long)gridDim.x * blockDim.x)
      bad |= !isfinite(f[q][l]);
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicExch(flag, 1);
}

template <typename T>
__global__ void k_to_double(long long n, double* out, const T* y, const T* comp) {
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < n; l += (long long)gridDim.x * blockDim.x)
    out[l] = comp ? (double)y[l] + (double)comp[l] : (double)y[l];
}

}  // namespace

namespace lee {

// Message of the calling thread's last failure outside a context (lee_create and the
// context-free entry points); one buffer per host thread, so callers on several threads do
// not overwrite each other's messages.
thread_local char g_create_error[512] = "";

int fail(lee_ctx* c, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (c)
    c->err = buf;
  else
    snprintf(g_create_error, sizeof g_create_error, "%s", buf);
  return code;
}

// Kinds of boundary lines: sponge zones (RHS terms) and BC lines (boundary updates).
bool is_sponge(int kind) { return kind == LEE_SPONGE_FREUND_AMBIENT || kind == LEE_SPONGE_FREUND_HARMONICWAVE; }

bool is_bc_line(int kind) {
  return kind == LEE_BC_NEUMANN || kind == LEE_BC_WALL_SLIP_KINEMATIC || kind == LEE_BC_DIRICHLET_ALLZERO ||
         kind == LEE_BC_DIRICHLET_HARMONICWAVE ||
         (kind >= LEE_BC_CENTERLINE_CART_NORM2X && kind <= LEE_BC_CENTERLINE_AXISYM);
}

// BC lines whose face values come from the closure row of the difference operator
bool reads_inward(int kind) {
  return kind == LEE_BC_NEUMANN || kind == LEE_BC_WALL_SLIP_KINEMATIC ||
         (kind >= LEE_BC_CENTERLINE_CART_NORM2X && kind <= LEE_BC_CENTERLINE_AXISYM);
}

bool reads_wave(int kind) { return kind == LEE_BC_DIRICHLET_HARMONICWAVE || kind == LEE_SPONGE_FREUND_HARMONICWAVE; }

int dev_alloc(lee_ctx* c, void** p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes ? bytes : 8);
  if (e != cudaSuccess) return fail(c, LEE_ERR_NOMEM, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
  c->allocs.push_back(*p);
  c->device_bytes += (long long)bytes;
  return LEE_OK;
}

// Coefficient tables (src/solver/spatial_discretization.cpp:28-492); the numbers are the
// published tables (Lele 1992; Bogey & Bailly 2004; Berland et al. 2007).
bool make_fd(OpTable* o, int scheme, int order) {
  memset(o, 0, sizeof *o);
  o->mfac = -1.0;
  if (scheme == LEE_FD_STANDARD_CENTRAL && order == 4) {
    o->h = 2; o->nb = 2; o->S = 3;
    o->c[3] = 8.0 / 12.0; o->c[4] = -1.0 / 12.0;
    o->B[0][0] = -3.0 / 2.0; o->B[0][1] = 4.0 / 2.0; o->B[0][2] = -1.0 / 2.0;
    o->B[1][0] = -1.0 / 2.0; o->B[1][1] = 0.0; o->B[1][2] = 1.0 / 2.0;
  } else if (scheme == LEE_FD_FDO11P) {
    o->h = 5; o->nb = 5; o->S = 9;
    const double in[6] = {0.0, 0.872756993962, -0.286511173973, 0.090320001280, -0.020779405824, 0.002484594688};
    for (int k = 0; k <= 5; ++k) o->c[5 + k] = in[k];
    const double r0[7] = {-2.225833963270, 4.827779580575, -5.001388453836, 3.911103941646,
                          -2.115267458633, 0.718882784412, -0.115276430894};
    const double r1[7] = {-0.212932721951, -1.060320390770, 2.078926116439, -1.287179452384,
                          0.685176395471, -0.245320613994, 0.041650667189};
    const double r2[5] = {1.0 / 12.0, -8.0 / 12.0, 0.0, 8.0 / 12.0, -1.0 / 12.0};
    const double r3[7] = {-0.02625099337517627, 0.18833730683403838, -0.797921633542548, 0.0,
                          0.797921633542548, -0.18833730683403838, 0.02625099337517627};
    const double r4[9] = {0.007650904064, -0.059463584768, 0.244678631765, -0.841570125482, 0.0,
                          0.841570125482, -0.244678631765, 0.059463584768, -0.007650904064};
    for (int s = 0; s < 7; ++s) { o->B[0][s] = r0[s]; o->B[1][s] = r1[s]; o->B[3][s] = r3[s]; }
    for (int s = 0; s < 5; ++s) o->B[2][s] = r2[s];
    for (int s = 0; s < 9; ++s) o->B[4][s] = r4[s];
  } else {
    return false;
  }
  for (int k = 1; k <= o->h; ++k) o->c[o->h - k] = -o->c[o->h + k];
  return true;
}

bool make_filter(OpTable* o, int scheme, int order, double strength) {
  memset(o, 0, sizeof *o);
  o->mfac = 1.0;
  const double r2[5] = {(-1.0 / 8.0) / 2.0, (1.0 / 2.0) / 2.0, 5.0 / 8.0, (1.0 / 2.0) / 2.0, (-1.0 / 8.0) / 2.0};
  const double r3[7] = {(1.0 / 32.0) / 2.0, (-3.0 / 16.0) / 2.0, (15.0 / 32.0) / 2.0, 11.0 / 16.0,
                        (15.0 / 32.0) / 2.0, (-3.0 / 16.0) / 2.0, (1.0 / 32.0) / 2.0};
  if (scheme == LEE_FILTER_STANDARD_CENTRAL && order == 4) {
    o->h = 2; o->nb = 2; o->S = 3;
    o->c[2] = 5.0 / 8.0; o->c[3] = (1.0 / 2.0) / 2.0; o->c[4] = (-1.0 / 8.0) / 2.0;
    o->B[0][0] = 1.0; o->B[1][1] = 1.0;
  } else if (scheme == LEE_FILTER_STANDARD_CENTRAL && order == 8) {
    o->h = 4; o->nb = 4; o->S = 7;
    o->c[4] = 1.0 - strength * (35.0 / 128.0);
    const double d[4] = {-7.0 / 32.0, 7.0 / 64.0, -1.0 / 32.0, 1.0 / 256.0};
    for (int k = 1; k <= 4; ++k) o->c[4 + k] = d[k - 1] * -strength;
    o->B[0][0] = 1.0; o->B[1][1] = 1.0;
    for (int s = 0; s < 5; ++s) o->B[2][s] = r2[s];
    for (int s = 0; s < 7; ++s) o->B[3][s] = r3[s];
  } else if (scheme == LEE_FILTER_SFO11P) {
    o->h = 5; o->nb = 5; o->S = 9;
    const double d[6] = {0.215044884112, -0.187772883589, 0.123755948787, -0.059227575576, 0.018721609157,
                         -0.002999540835};
    o->c[5] = 1.0 - strength * d[0];
    for (int k = 1; k <= 5; ++k) o->c[5 + k] = d[k] * -strength;
    o->B[0][0] = 1.0; o->B[1][1] = 1.0;
    for (int s = 0; s < 5; ++s) o->B[2][s] = r2[s];
    for (int s = 0; s < 7; ++s) o->B[3][s] = r3[s];
    const double r4[9] = {0.008228661760, -0.045211119360, 0.120007591680, -0.204788880640, 0.243527493120,
                          -0.204788880640, 0.120007591680, -0.045211119360, 0.008228661760};
    for (int s = 0; s < 9; ++s) o->B[4][s] = (s == 4) ? 1.0 - strength * r4[s] : r4[s] * -strength;
  } else {
    return false;
  }
  for (int k = 1; k <= o->h; ++k) o->c[o->h - k] = o->c[o->h + k];
  return true;
}

// F - I of a filter table: the increment form used by the compensated time advance.
OpTable minus_identity(const OpTable& f) {
  OpTable d = f;
  d.c[d.h] -= 1.0;
  for (int r = 0; r < d.nb; ++r) d.B[r][r] -= 1.0;
  return d;
}

// Closure codes of one direction: the reference's per-line scan (see lee_internal.h).
// Returns false when a hole closure would lack fluid support (the reference asserts,
// src/solver/spatial_discretization.cpp:1749-1798).
bool closure_codes(const OpTable& op, const BlockData& b, int d, std::vector<int8_t>& code) {
  int n[3] = {b.nx, b.ny, b.nz};
  long long st[3] = {1, b.nx, (long long)b.nx * b.ny};
  int o1 = d == 0 ? 1 : 0, o2 = d == 2 ? 1 : 2;
  int nd = n[d];
  code.assign((size_t)b.N, 0);
  for (int b2 = 0; b2 < n[o2]; ++b2)
    for (int b1 = 0; b1 < n[o1]; ++b1) {
      long long base = b1 * st[o1] + b2 * st[o2];
      auto at = [&](int p) { return base + p * st[d]; };
      for (int p = 0; p < nd; ++p) {
        int c = 0;
        if (p < op.h) c = 1 + p;
        else if (p > nd - 1 - op.h) c = -(1 + (nd - 1 - p));
        code[(size_t)at(p)] = (int8_t)c;
      }
      int last = b.hib[(size_t)at(0)];
      for (int p = 0; p < nd; ++p) {
        int my = b.hib[(size_t)at(p)];
        if (my == 1) {
          if (last == 1) {
            code[(size_t)at(p)] = kCodeZero;
          } else if (last == -1 && p > 0) {  // `last_iblank /= BLANKED` (:1391) is true only after -1
            for (int ib = 0; ib < op.nb; ++ib) {
              int q = p - 1 - ib;
              if (q < 0 || b.hib[(size_t)at(q)] > 0) return false;
            }
            if (p - 1 - (op.S - 1) < 0) return false;  // the mirrored rows read S points to the left
            for (int ib = 0; ib < op.nb; ++ib) code[(size_t)at(p - 1 - ib)] = (int8_t)(-(1 + ib));
          }
        } else if (last == 1) {
          for (int ib = 0; ib < op.nb; ++ib) {
            int q = p + ib;
            if (q > nd - 1 || b.hib[(size_t)at(q)] > 0) return false;
          }
          if (p + op.S - 1 > nd - 1) return false;  // the rows read S points to the right
          for (int ib = 0; ib < op.nb; ++ib) code[(size_t)at(p + ib)] = (int8_t)(1 + ib);
        }
        last = my;
      }
    }
  return true;
}

// Record an event on the context stream (timing on); returns its index or -1.
int mark(lee_ctx* c) {
  if (!c->timing) return -1;
  if (c->ev_used == c->ev_pool.size()) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return -1;
    c->ev_pool.push_back(e);
  }
  cudaEventRecord(c->ev_pool[c->ev_used], c->stream);
  return (int)c->ev_used++;
}

void span(lee_ctx* c, int kind, int a, int b) {
  if (a >= 0 && b >= 0) c->ev_marks.push_back({kind, a});
  (void)b;
}

int grid1d(long long n) {
  long long b = (n + 255) / 256;
  return (int)(b > 148 * 32 ? 148 * 32 : (b < 1 ? 1 : b));
}

// Decide whether an FP64 field is uniform over the block (then the kernels use a constant).
int classify(lee_ctx* c, const double* d_field, long long N, double scale, double* lo, double* hi, bool* uniform,
             bool* zero) {
  double* d_mm = nullptr;
  CK(cudaMallocAsync((void**)&d_mm, 2 * sizeof(double), c->stream));
  double init[2] = {-1e308, -1e308};
  CK(cudaMemcpyAsync(d_mm, init, sizeof init, cudaMemcpyHostToDevice, c->stream));
  CK(setup_minmax((int)N, d_field, d_mm, c->stream));
  double h[2];
  CK(cudaMemcpyAsync(h, d_mm, sizeof h, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaFreeAsync(d_mm, c->stream));
  *lo = -h[0];
  *hi = h[1];
  double mag = fmax(fabs(*lo), fabs(*hi));
  *zero = mag <= 1e-12 * scale;
  *uniform = *zero || (*hi - *lo) <= 1e-12 * mag;
  return LEE_OK;
}

template <typename T>
int make_coef(lee_ctx* c, BlockData& b, const double* d_field, double scale, Coef<T>* out) {
  double lo, hi;
  bool uni, zero;
  int rc = classify(c, d_field, b.N, scale, &lo, &hi, &uni, &zero);
  if (rc) return rc;
  out->zero = zero ? 1 : 0;
  if (uni) {
    out->p = nullptr;
    out->c = zero ? T(0) : (T)(0.5 * (lo + hi));
    return LEE_OK;
  }
  b.n_coef_fields += 1;
  if (std::is_same<T, double>::value) {
    out->p = reinterpret_cast<const T*>(d_field);
  } else {
    T* d = nullptr;
    rc = dalloc(c, &d, (size_t)b.N);
    if (rc) return rc;
    launch_convert<T>(c->stream, b.N, d, d_field);
    CK(cudaGetLastError());
    out->p = d;
  }
  out->c = T(0);
  return LEE_OK;
}

int upload(lee_ctx* c, double** d, const std::vector<double>& h) {
  int rc = dalloc(c, d, h.size());
  if (rc) return rc;
  CK(cudaMemcpyAsync(*d, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  return LEE_OK;
}

int alloc_fields(lee_ctx* c, void** f, long long N) {
  for (int v = 0; v < c->V; ++v) {
    int rc = dev_alloc(c, &f[v], (size_t)N * c->esz);
    if (rc) return rc;
    CK(cudaMemsetAsync(f[v], 0, (size_t)N * c->esz, c->stream));
  }
  return LEE_OK;
}

// Map the reference's five slots (s', u', v', w', p') to the V device fields.
int slot_of(int V, int v) { return v == V - 1 ? 4 : v; }

template <typename T>
void fill_stage_common(lee_ctx* c, BlockData& b, StageParams<T>& p) {
  memset(&p, 0, sizeof p);
  p.nx = b.nx; p.ny = b.ny; p.nz = b.nz;
  p.dim = c->cfg.num_dim;
  p.V = c->V;
  const bool dbl = std::is_same<T, double>::value;
  const Coef<T>* jm = dbl ? (const Coef<T>*)b.cd_jm : (const Coef<T>*)b.cf_jm;
  const Coef<T>* ub = dbl ? (const Coef<T>*)b.cd_ub : (const Coef<T>*)b.cf_ub;
  const Coef<T>* gs = dbl ? (const Coef<T>*)b.cd_gs : (const Coef<T>*)b.cf_gs;
  const Coef<T>* gu = dbl ? (const Coef<T>*)b.cd_gu : (const Coef<T>*)b.cf_gu;
  const Coef<T>* gp = dbl ? (const Coef<T>*)b.cd_gp : (const Coef<T>*)b.cf_gp;
  for (int q = 0; q < 9; ++q) { p.jm[q] = jm[q]; p.gu[q] = gu[q]; }
  for (int q = 0; q < 3; ++q) { p.ubar[q] = ub[q]; p.gs[q] = gs[q]; p.gp[q] = gp[q]; }
  p.pbar = dbl ? *(const Coef<T>*)&b.cd_pb : *(const Coef<T>*)&b.cf_pb;
  p.rhobar_inv = dbl ? *(const Coef<T>*)&b.cd_rbi : *(const Coef<T>*)&b.cf_rbi;
  p.need_rho = b.need_rho;
  p.gamma = (T)c->cfg.gamma;
  p.inv_gamma = (T)(1.0 / c->cfg.gamma);
  p.nzones = 0;
  for (auto& z : b.bnd) {
    if (!is_sponge(z.kind)) continue;
    Zone<T>& zn = p.zones[p.nzones++];
    for (int d = 0; d < 3; ++d) { zn.lo[d] = z.lo[d]; zn.hi[d] = z.hi[d]; }
    zn.sig = dbl ? (const T*)z.d_sigma : (const T*)z.d_sigma_t;
    zn.ref = (const T*)z.d_ref;
  }
  p.axisym = c->axisym ? 1 : 0;
  p.ry = b.d_xyz[1];
  p.has_src = b.d_src_g != nullptr;
  for (int d = 0; d < 3; ++d) { p.src_lo[d] = b.src_lo[d]; p.src_hi[d] = b.src_hi[d]; }
  p.src_g = dbl ? (const T*)b.d_src_g : (const T*)b.d_src_g_t;
  for (int d = 0; d < 3; ++d) p.code[d] = b.has_holes ? b.d_code_fd[d] : nullptr;
  p.iblank = b.has_holes ? b.d_iblank : nullptr;
  p.fd = c->fd;
  p.sigma = (const T*)b.d_sigma_field;
}

// Distributed source: the grid box covered by the lattice, and the trilinear prolongation of
// coarse amplitudes A onto it (box-shaped, i fastest) or its transpose (restriction of a box
// field onto the lattice). p = block, omega, cx, cy, cz, ox, oy, oz, hx, hy, hz, ...
bool distributed_box(const std::vector<double>& p, int dim, int nx, int ny, int nz, int lo[3], int hi[3]) {
  const int n[3] = {nx, ny, nz};
  for (int d = 0; d < 3; ++d) {
    if (d >= dim) {
      lo[d] = hi[d] = 0;
      continue;
    }
    const int cn = (int)p[2 + d];
    const double o = p[5 + d], h = p[8 + d];
    lo[d] = std::max(0, (int)std::ceil(o));
    hi[d] = std::min(n[d] - 1, (int)std::floor(o + (cn - 1) * h));
    if (hi[d] < lo[d]) return false;
  }
  return true;
}

// Corner weights of fine index i along one lattice direction: node p0 and weight of p0 + 1.
void lattice_weights(double i, double o, double h, int cn, int* p0, double* f) {
  const double u = (i - o) / h;
  int q = (int)std::floor(u);
  if (q > cn - 2) q = cn - 2;
  if (q < 0) q = 0;
  *p0 = q;
  *f = u - q;
}

void prolong(const std::vector<double>& p, int dim, const int lo[3], const int hi[3], const double* A,
             std::vector<double>& g) {
  const int cx = (int)p[2], cy = (int)p[3], cz = (int)p[4];
  const size_t nb = (size_t)(hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1);
  g.assign(nb, 0.0);
  size_t lb = 0;
  for (int k = lo[2]; k <= hi[2]; ++k)
    for (int j = lo[1]; j <= hi[1]; ++j)
      for (int i = lo[0]; i <= hi[0]; ++i, ++lb) {
        int q[3] = {0, 0, 0};
        double f[3] = {0.0, 0.0, 0.0};
        lattice_weights(i, p[5], p[8], cx, &q[0], &f[0]);
        lattice_weights(j, p[6], p[9], cy, &q[1], &f[1]);
        if (dim == 3) lattice_weights(k, p[7], p[10], cz, &q[2], &f[2]);
        double sum = 0.0;
        for (int c2 = 0; c2 < (dim == 3 ? 2 : 1); ++c2)
          for (int c1 = 0; c1 < 2; ++c1)
            for (int c0 = 0; c0 < 2; ++c0) {
              const double w = (c0 ? f[0] : 1.0 - f[0]) * (c1 ? f[1] : 1.0 - f[1]) *
                               (dim == 3 ? (c2 ? f[2] : 1.0 - f[2]) : 1.0);
              sum += w * A[(q[0] + c0) + (size_t)cx * ((q[1] + c1) + (size_t)cy * (q[2] + c2))];
            }
        g[lb] = sum;
      }
  (void)cz;
}

void restrict_to_lattice(const std::vector<double>& p, int dim, const int lo[3], const int hi[3], const double* gbar,
                         double* abar) {
  const int cx = (int)p[2], cy = (int)p[3], cz = (int)p[4];
  std::fill(abar, abar + (size_t)cx * cy * cz, 0.0);
  size_t lb = 0;
  for (int k = lo[2]; k <= hi[2]; ++k)
    for (int j = lo[1]; j <= hi[1]; ++j)
      for (int i = lo[0]; i <= hi[0]; ++i, ++lb) {
        int q[3] = {0, 0, 0};
        double f[3] = {0.0, 0.0, 0.0};
        lattice_weights(i, p[5], p[8], cx, &q[0], &f[0]);
        lattice_weights(j, p[6], p[9], cy, &q[1], &f[1]);
        if (dim == 3) lattice_weights(k, p[7], p[10], cz, &q[2], &f[2]);
        for (int c2 = 0; c2 < (dim == 3 ? 2 : 1); ++c2)
          for (int c1 = 0; c1 < 2; ++c1)
            for (int c0 = 0; c0 < 2; ++c0) {
              const double w = (c0 ? f[0] : 1.0 - f[0]) * (c1 ? f[1] : 1.0 - f[1]) *
                               (dim == 3 ? (c2 ? f[2] : 1.0 - f[2]) : 1.0);
              abar[(q[0] + c0) + (size_t)cx * ((q[1] + c1) + (size_t)cy * (q[2] + c2))] += w * gbar[lb];
            }
      }
}

// Amplitude of the monopole at time t (oracle patch P2, modelled on src/solver/source.cpp:60-92).
// The monopole parameters that apply to block b, or null when it has no monopole.
const double* monopole_of(const lee_ctx* c, const BlockData& b) {
  if (b.src_mode == 1) return b.own_src;
  if (b.src_mode == 0 && c->src_kind == LEE_SOURCE_MONOPOLE && c->src[5] > 0.0) return c->src;
  return nullptr;
}

// The constants of CASE_2DJET_WITH_A_HARMONIC_SOURCE's source (src/solver/source.cpp:30-49), in
// the reference's order: amplitude, angular frequency, Bx, By.
void jet2d_constants(double gamma, double* amp, double* omega, double* bx, double* by) {
  const double twopi = 2.0 * acos(-1.0), inverse_twopi = 1.0 / twopi;  // src/math/math.cpp:7-10
  double amplitude = 0.001, frequency = 76.0, Bx = 0.04 * log(2.0), By = 0.32 * log(2.0);
  const double b = 1.3, R = 287.0, rhoinfty = 1.184, Tinfty = 300.0;
  const double cinfty = sqrt(gamma * R * Tinfty);
  amplitude /= rhoinfty * pow(cinfty, 2) / (b / cinfty);
  frequency *= inverse_twopi * (b / cinfty);
  Bx *= pow(b, 2);
  By *= pow(b, 2);
  *amp = amplitude;
  *omega = frequency * twopi;
  *bx = Bx;
  *by = By;
}

double source_amp(const lee_ctx* c, const BlockData& b, double t) {
  if (c->src_kind == LEE_SOURCE_DISTRIBUTED) return (c->cfg.gamma - 1.0) * sin(c->dsrc[1] * t);
  if (c->src_kind == LEE_SOURCE_JET2D_HARMONIC && b.src_mode == 0) {
    double amp, om, bx, by;
    jet2d_constants(c->cfg.gamma, &amp, &om, &bx, &by);
    return amp * cos(om * t);
  }
  const double* m = monopole_of(c, b);
  if (!m) return 0.0;
  double T = m[6];
  double ramp = 1.0;
  if (T > 0.0 && t < T) {
    double sn = sin(0.5 * M_PI * t / T);
    ramp = sn * sn;
  }
  return m[3] * (c->cfg.gamma - 1.0) * ramp * sin(m[4] * t);
}

// Weights of an operator by closure class for offsets -H..H (see lee_tma.h); false when a
// nonzero coefficient falls outside the window.
// `stride` is the row length of the destination table (>= 2H+1).
bool class_weights(const OpTable& op, int H, double* w, int stride) {
  const int nb = op.nb;
  for (int q = 0; q < (1 + 2 * nb) * stride; ++q) w[q] = 0.0;
  if (op.h > H || 2 * H + 1 > stride) return false;
  for (int o = -op.h; o <= op.h; ++o) w[0 * stride + H + o] = op.c[o + op.h];
  for (int r = 0; r < nb; ++r)
    for (int s = 0; s < op.S; ++s) {
      if (op.B[r][s] == 0.0) continue;
      int ol = s - r, orr = r - s;
      if (ol < -H || ol > H || orr < -H || orr > H) return false;
      w[(1 + r) * stride + H + ol] += op.B[r][s];
      w[(1 + nb + r) * stride + H + orr] += op.mfac * op.B[r][s];
    }
  return true;
}

Tableau tableau(int rk) {
  Tableau t{};
  if (rk == LEE_RK4) {
    t.ns = 4;
    t.b[0] = 1.0 / 6.0; t.b[1] = 1.0 / 3.0; t.b[2] = 1.0 / 3.0; t.b[3] = 1.0 / 6.0;
    t.c[0] = 0.0; t.c[1] = 1.0 / 2.0; t.c[2] = 1.0 / 2.0; t.c[3] = 1.0;
    t.a[0] = 1.0 / 2.0; t.a[1] = 1.0 / 2.0; t.a[2] = 1.0; t.a[3] = 0.0;
  } else {
    t.ns = 2;
    t.b[0] = 1.0 / 2.0; t.b[1] = 1.0 / 2.0;
    t.c[0] = 0.0; t.c[1] = 1.0;
    t.a[0] = 1.0; t.a[1] = 0.0;
  }
  return t;
}

// Filter coefficient table and the context-free error message, for lee_static.cu.
bool filter_table(OpTable* o, int scheme, int order, double strength) {
  return make_filter(o, scheme, order, strength);
}
void set_global_error(const char* msg) { snprintf(g_create_error, sizeof g_create_error, "%s", msg); }

// the host translation units use both precisions
template int make_coef<float>(lee_ctx* c, BlockData& b, const double* d_field, double scale, Coef<float>* out);
template int make_coef<double>(lee_ctx* c, BlockData& b, const double* d_field, double scale, Coef<double>* out);
template void fill_stage_common<float>(lee_ctx* c, BlockData& b, StageParams<float>& p);
template void fill_stage_common<double>(lee_ctx* c, BlockData& b, StageParams<double>& p);

// Launches of the conversion kernels for the other host translation units.
template <typename T>
void launch_convert(cudaStream_t s, long long n, T* out, const double* in) {
  k_convert<T><<<grid1d(n), 256, 0, s>>>(n, out, in);
}
template <typename T>
void launch_to_double(cudaStream_t s, long long n, double* out, const T* y, const T* comp) {
  k_to_double<T><<<grid1d(n), 256, 0, s>>>(n, out, y, comp);
}
template void launch_convert<float>(cudaStream_t, long long, float*, const double*);
template void launch_convert<double>(cudaStream_t, long long, double*, const double*);
template void launch_to_double<float>(cudaStream_t, long long, double*, const float*, const float*);
template void launch_to_double<double>(cudaStream_t, long long, double*, const double*, const double*);

cudaError_t launch_nonfinite(cudaStream_t s, long long n, int V, size_t esz, void* const* f, void* const* e,
                             int* flag) {
  const void* p[10] = {};
  int nf = 0;
  for (int v = 0; v < V; ++v) p[nf++] = f[v];
  if (e)
    for (int v = 0; v < V; ++v) p[nf++] = e[v];
  const int grid = grid1d(n / 4 + 1);
  if (esz == 4) {
    const float* q[10];
    for (int k = 0; k < 10; ++k) q[k] = static_cast<const float*>(p[k]);
    k_nonfinite<float><<<grid, 256, 0, s>>>(n, nf, q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7], q[8], q[9], flag);
  } else {
    const double* q[10];
    for (int k = 0; k < 10; ++k) q[k] = static_cast<const double*>(p[k]);
    k_nonfinite<double><<<grid, 256, 0, s>>>(n, nf, q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7], q[8], q[9], flag);
  }
  return cudaGetLastError();
}

}  // namespace lee
