// Host side of the C ABI (include/lee_b200.h): context, device memory, one-time
// setup on the GPU, and the time-advance schedule.
//
// Schedule of one step (temporal::time_advance, camille src/solver/temporal_discretization.cpp:334-374):
//   time += dt (solver::solve increments before advancing, src/solver/solver.cpp:72)
//   for each RK stage s: one fused stage kernel per block (RHS + RK update, reading the
//     stage input with its stencil neighbours and writing the next stage input and the
//     accumulator), then the boundary conditions of the stage output
//   filter passes (dimension split, src/solver/spatial_discretization.cpp:2191-2246)
//   hole mask (temporal::iblank_correction, :380-393)
#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include <algorithm>
#include <map>
#include <memory>

#include "lee_internal.h"
#include "lee_tma.h"

using namespace lee;

namespace {

char g_create_error[512] = "";

struct Boundary {
  int kind, dir, end, lo[3], hi[3];
  std::vector<double> sigma;  // host copy when given by the caller
  double* d_sigma = nullptr;  // FP64 strengths
  void* d_sigma_t = nullptr;  // strengths in the working precision
  void* d_ref = nullptr;      // harmonic-wave sponge: the wave on the box, V fields (working precision)
};

struct BlockData {
  int nx = 0, ny = 0, nz = 0;
  long long N = 0;
  bool set = false, has_mean = false;
  std::vector<double> hx, hy, hz;
  std::vector<int> hib;
  std::vector<double> hmean[5];
  std::vector<Boundary> bnd;
  // FP64 setup products
  double* d_xyz[3] = {};
  double* d_mean[5] = {};
  double* d_met[9] = {};
  double* d_minv[9] = {};
  double* d_jac = nullptr;
  double* d_invjac = nullptr;
  double* d_grad[15] = {};
  double* d_jm[9] = {};
  double* d_rbi = nullptr;
  int* d_iblank = nullptr;
  int8_t* d_code_fd[3] = {};
  int8_t* d_code_flt[3] = {};
  bool has_holes = false;   // some point is BLANKED: hole closures and hole bypass
  bool has_iblank = false;  // some point is not NOTBLANKED (holes or receivers): CFL skips them
  // per-block clock (blocks advanced with their own time steps keep their own time)
  double time = 0.0;
  int step = 0;
  // source of this block: 0 the context's, 1 its own monopole (own_src), 2 none
  int src_mode = 0;
  double own_src[7] = {0, 0, 0, 0, 0, 0, 0};
  // monopole factor on a box
  int src_lo[3] = {0, 0, 0}, src_hi[3] = {-1, -1, -1};
  double* d_src_g = nullptr;
  void* d_src_g_t = nullptr;
  // coefficients in the working precision
  Coef<double> cd_jm[9], cd_ub[3], cd_pb, cd_rbi, cd_gs[3], cd_gu[9], cd_gp[3];
  Coef<float> cf_jm[9], cf_ub[3], cf_pb, cf_rbi, cf_gs[3], cf_gu[9], cf_gp[3];
  int need_rho = 0;
  int n_coef_fields = 0;
  // state buffers (element size 8 or 4), V fields each
  void* y[kMaxVars] = {};
  void* acc[kMaxVars] = {};
  void* zb[2][kMaxVars] = {};
  void* comp[kMaxVars] = {};
  void* dsum[kMaxVars] = {};
  void* rho = nullptr;      // rho'/rho_bar of the last pre-filter state (non-uniform mean velocity)
  bool rho_valid = false;   // false until a step or a filter call has written it
  // TMA-staged kernels (blocks without holes, 4th-order difference)
  bool tma = false, tma_filter = false;
  bool filter_vec = false;           // the vectorised fused filter (lee_filter.cu) applies
  int filter_px = 0;                 // the fused filter's kernel: 0 scalar, else the vector group width
  int stage_px = 1;                  // points per thread of the TMA stage kernel (2: lee_stage_pair.cu)
  bool stage_pair = false;           // the two-point stage kernel applies
  int vtiles_x = 0, vtiles_y = 0;    // tiles of the vectorised kernel at that width
  int traits = kTrGeneric;          // coefficient-layout traits of the TMA stage kernel
  void* d_sigma_field = nullptr;    // summed sponge strengths per point (working precision)
  int tiles_x = 0, tiles_y = 0;
  int stage_chunk = 0, filter_chunk = 0;
  int filter_ry = 1;                  // rows per thread row of the scalar fused filter (1 or 2)
};

struct MapKey {
  const void* p;
  int bx, by;
  bool operator<(const MapKey& o) const {
    if (p != o.p) return p < o.p;
    if (bx != o.bx) return bx < o.bx;
    return by < o.by;
  }
};

struct MapBytes {
  unsigned char b[sizeof(CUtensorMap)];
};

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

}  // namespace

struct lee_ctx {
  lee_config cfg;
  int V = 0;
  size_t esz = 8;
  bool comp = false;
  OpTable fd{}, flt{}, fltd{};
  std::vector<BlockData> blk;
  cudaStream_t stream = nullptr;
  int src_kind = LEE_SOURCE_NONE;
  double src[7] = {0, 0, 0, 0, 0, 0, 0};
  Wave wave{};               // lee_set_harmonic_wave (type LEE_WAVE_NONE until set)
  bool wave_time = false;    // some BC line or sponge zone reads the wave (from lee_prepare)
  bool axisym = false;       // lee_set_axisymmetric
  std::vector<double> dsrc;  // distributed source parameters (LEE_SOURCE_DISTRIBUTED)
  bool prepared = false, uploaded = false;
  int step = 0;
  double time = 0.0;
  std::vector<void*> allocs;
  long long device_bytes = 0;
  std::string err;
  // timing
  bool timing = false;
  lee_stats stats{};
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<int, int>> ev_marks;  // (kind, event index pair start); kind 0 stage, 1 filter
  size_t ev_used = 0;
  // TMA: tensor maps per field buffer, weight tables by closure class, device error flag
  EncodeTiledFn encode = nullptr;
  std::map<MapKey, MapBytes> tmaps;
  double wst[5][5] = {};
  double wfl[11][11] = {};
  int hf = 0;
  bool wst_ok = false, wfl_ok = false;
  bool wfl_sym = false;  // symmetric interior filter stencil: the vectorised filter kernel applies
  int filter_kernel = -1;  // lee_set_filter_kernel: -1/0 scalar, else vector group width
  int stage_kernel = -1;   // lee_set_stage_kernel: -1 default, else points per thread
  int* d_err = nullptr;
  double* d_report = nullptr;  // -min and max of the five state slots (lee_state_minmax)
  double* d_staging = nullptr;  // FP64 field of compensated uploads and downloads
  // overset maps (host copies, then device arrays from lee_prepare)
  struct {
    int n = 0, W = 1, w[3] = {1, 1, 1};
    bool fused = false;
    std::vector<int> rb, db;
    std::vector<long long> rl, dl;
    std::vector<double> wt;
    int *d_rb = nullptr, *d_db = nullptr;
    long long *d_rl = nullptr, *d_dl = nullptr;
    double *d_wt = nullptr, *d_buf = nullptr;
  } ovs;
  // replayed step graph: a few steps captured once (until the buffer roles repeat) and
  // launched as one graph; keyed by dt, precision and the buffer layout it was captured on
  struct {
    bool enabled = true;
    cudaGraphExec_t exec = nullptr;
    std::vector<double> dts;       // the time step of every block
    int steps = 0;                 // steps per replay
    std::vector<void*> layout;
    long long launches = 0, stage_launches = 0, filter_launches = 0;  // per replay
    void* d_amp = nullptr;         // monopole amplitudes, [step][stage], working precision
    size_t amp_cap = 0;            // entries
    int* d_ctr = nullptr;          // steps of the current chunk done so far
    double* d_ttab = nullptr;      // stage times, [step][block][stage] (harmonic-wave lines and zones)
  } graph;
  // batched kernels for many independent 2-D blocks (lee_advance_blocks)
  struct {
    bool active = false;
    int sshape = 0, fshape = 0, sgrid = 0, fgrid = 0;
    int4* d_stiles = nullptr;
    int nst = 0;
    int4* d_ftiles = nullptr;
    int nft = 0;
    void* d_prm_graph = nullptr;   // StageParams [stage][block], monopole amplitudes from the graph table
    void* d_prm_direct = nullptr;  // the same with the amplitudes of the step being launched
    void* d_finst = nullptr;       // BatchFilterInst [block]
    std::vector<double> graph_dts;  // time steps d_prm_graph was built for
  } batch;
  // discrete adjoint (single block, uniform mean, no BC lines, holes or overset)
  struct {
    bool ready = false;
    TransOp dT{}, fT{};                    // transposed difference and filter operators
    void *lam[kMaxVars] = {}, *mu[kMaxVars] = {}, *kb[2][kMaxVars] = {}, *ybar[kMaxVars] = {};
    int mic_block = 0;
    double weight = 0.0;
    std::vector<long long> mic;
    long long* d_mic = nullptr;
    bool trace_on = false;
    double* d_trace = nullptr;             // rows of p' at the microphones, one per step
    size_t trace_rows = 0;
    int* d_base = nullptr;                 // trace row of the first step of a replayed chunk
    int host_row = 0;                      // trace row of the next directly launched step
    double* d_gbar = nullptr;              // gradient of the distributed source's box field
    std::vector<void*> ckpt;               // checkpoints: V (+ V carried errors) fields each
    size_t ckpt_slots = 0;
    bool tma = false;                      // the plane-marching stage kernel (lee_adjoint_tma.cu)
    bool tma_jm = false;                   // ... with J*metrics fields (else constants)
    bool fused_filter = false;             // F^T by the fused filter kernel (lee_tma.cu)
  } adj;
};

namespace {

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

#define CK(call)                                                                       \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return fail(c, LEE_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));   \
  } while (0)

int dev_alloc(lee_ctx* c, void** p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes ? bytes : 8);
  if (e != cudaSuccess) return fail(c, LEE_ERR_NOMEM, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
  c->allocs.push_back(*p);
  c->device_bytes += (long long)bytes;
  return LEE_OK;
}

template <typename P>
int dalloc(lee_ctx* c, P** p, size_t count) {
  return dev_alloc(c, reinterpret_cast<void**>(p), count * sizeof(P));
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

template <typename T>
__global__ void k_convert(long long n, T* out, const double* in) {
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < n; l += (long long)gridDim.x * blockDim.x)
    out[l] = (T)in[l];
}

// FP64 -> (y, e) with y = fl32(x) and e = fl32(x - y): the compensated pair of an uploaded state
__global__ void k_split(long long n, float* y, float* e, const double* in) {
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < n; l += (long long)gridDim.x * blockDim.x) {
    const float r = (float)in[l];
    y[l] = r;
    e[l] = (float)(in[l] - (double)r);
  }
}

// out = fl32(y + e)
__global__ void k_add_pair(long long n, float* out, const float* y, const float* e) {
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < n; l += (long long)gridDim.x * blockDim.x)
    out[l] = (float)((double)y[l] + (double)e[l]);
}

template <typename T>
__global__ void k_to_double(long long n, double* out, const T* y, const T* comp) {
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < n; l += (long long)gridDim.x * blockDim.x)
    out[l] = comp ? (double)y[l] + (double)comp[l] : (double)y[l];
}

template <typename T>
__global__ void k_fill_const(long long n, T* out, T v) {
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < n; l += (long long)gridDim.x * blockDim.x)
    out[l] = v;
}

__global__ void k_zero_bytes(long long n, unsigned char* p) {
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < n; l += (long long)gridDim.x * blockDim.x)
    p[l] = 0;
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
    k_convert<T><<<grid1d(b.N), 256, 0, c->stream>>>(b.N, d, d_field);
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

template <typename T>
void** as_void(T** p) {
  return reinterpret_cast<void**>(p);
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

// The fused filter's box (tile of kTileX x kTileY * ry points with a halo of h) and its tiles.
int filter_box(const lee_ctx* c, int h, int ry, int* bx, int* by) {
  const int A = (int)(16 / c->esz);
  const int hx = ((h + A - 1) / A) * A;
  *bx = kTileX + 2 * hx;
  *by = kTileY * ry + 2 * h;
  return LEE_OK;
}

int filter_tiles(const BlockData& b) { return b.tiles_x * ((b.ny + kTileY * b.filter_ry - 1) / (kTileY * b.filter_ry)); }

// Tiles of the vectorised filter at the block's group width.
void set_filter_tiles(const lee_ctx* c, BlockData& b) {
  if (b.filter_px <= 0) return;
  int bx, by, tx, ty;
  filter_vec_box(c->esz, c->hf, b.filter_px, &bx, &by, &tx, &ty);
  b.vtiles_x = (b.nx + tx - 1) / tx;
  b.vtiles_y = (b.ny + ty - 1) / ty;
}

template <typename T>
int launch_stage_any(lee_ctx* c, BlockData& b, const StageParams<T>& p, void* const* zin, int chunk_override = 0) {
  if (!b.tma) {
    CK(launch_stage<T>(p, c->comp ? 1 : 0, c->stream));
    return LEE_OK;
  }
  TmaStageParams<T> tp;
  memset(&tp, 0, sizeof tp);
  tp.s = p;
  tp.tiles_x = b.tiles_x;
  tp.k_chunk = chunk_override ? chunk_override : b.stage_chunk;
  for (int a = 0; a < 5; ++a)
    for (int o = 0; o < 5; ++o) tp.w[a][o] = (T)c->wst[a][o];
  tp.err = c->d_err;
  FieldMaps fm;
  int rc = field_maps(c, b, zin, Box<T, kFdHalf>::BX, Box<T, kFdHalf>::BY, &fm);
  if (rc) return rc;
  const int chunks = c->cfg.num_dim == 3 ? (b.nz + tp.k_chunk - 1) / tp.k_chunk : 1;
  // the stage's kind selects a specialised kernel; a first stage that is also the last (no
  // such tableau here) reads p.stage and p.last at run time
  const int kind = p.stage < 0 ? kKindRhs
                   : p.stage == 0 ? (p.last ? kKindRuntime : kKindFirst)
                                  : (p.last ? kKindLast : kKindMid);
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
                        void* const* comp_out, int chunk_override = 0) {
  TmaFilterParams<T> fp;
  memset(&fp, 0, sizeof fp);
  fp.nx = b.nx; fp.ny = b.ny; fp.nz = b.nz;
  fp.V = c->V;
  fp.tiles_x = b.tiles_x;
  fp.k_chunk = chunk_override ? chunk_override : b.filter_chunk;
  fp.nb = c->hf;
  for (int a = 0; a < 11; ++a)
    for (int o = 0; o < 11; ++o) fp.w[a][o] = (T)c->wfl[a][o];
  fp.blend = (T)c->cfg.filter_blend;
  for (int v = 0; v < c->V; ++v) {
    fp.err[v] = err ? (const T*)err[v] : nullptr;
    fp.out[v] = (T*)out[v];
    fp.comp[v] = comp_out ? (T*)comp_out[v] : nullptr;
  }
  fp.errflag = c->d_err;
  int bx, by, tx, ty;
  if (b.filter_px > 0) {
    filter_vec_box(c->esz, c->hf, b.filter_px, &bx, &by, &tx, &ty);
    fp.tiles_x = b.vtiles_x;
  } else {
    filter_box(c, c->hf, b.filter_ry, &bx, &by);
  }
  FieldMaps fm;
  int rc = field_maps(c, b, in, bx, by, &fm);
  if (rc) return rc;
  const int chunks = c->cfg.num_dim == 3 ? (b.nz + fp.k_chunk - 1) / fp.k_chunk : 1;
  int e0 = mark(c);
  if (b.filter_px > 0)
    CK(launch_filter_vec<T>(fm, fp, c->hf, b.filter_px, c->cfg.num_dim, b.vtiles_x * b.vtiles_y, chunks, c->stream));
  else
    CK(launch_filter_tma<T>(fm, fp, c->hf, c->cfg.num_dim, c->comp ? 1 : 0, b.filter_ry, filter_tiles(b), chunks,
                            c->stream));
  int e1 = mark(c);
  span(c, 1, e0, e1);
  c->stats.filter_launches += 1;
  c->stats.kernel_launches += 1;
  return LEE_OK;
}

int check_device_error(lee_ctx* c);

// Pick the k-chunk (planes marched by one CTA) of the stage and filter kernels by timing
// the candidates on this block: short chunks give more CTAs, long chunks re-load fewer
// halo planes. Runs at setup on the (not yet uploaded) state buffers.
template <typename T>
int autotune(lee_ctx* c, BlockData& b) {
  if (!b.tma && !b.tma_filter) return LEE_OK;
  const bool d3 = c->cfg.num_dim == 3;
  const int cands3[] = {8, 16, 24, 32, 48, 64, 96, 128, 192, 256};
  const int cands2[] = {1};
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
    // the scalar filter's rows per thread row are timed with the chunk: each point's
    // arithmetic is the same for either
    const int nry = which == 1 ? 2 : 1;
    for (int kq = 0; kq < (which == 1 ? nkinds : nskinds) * nry; ++kq) {
      if (which == 0) {
        b.stage_px = skinds[kq];
      } else {
        b.filter_px = kinds[kq / nry];
        b.filter_ry = 1 + kq % nry;
        if (b.filter_px > 0 && b.filter_ry > 1) continue;
        set_filter_tiles(c, b);
      }
      for (int ch : (d3 ? std::vector<int>(std::begin(cands3), std::end(cands3))
                        : std::vector<int>(std::begin(cands2), std::end(cands2)))) {
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
        if (tsum < best) {
          best = tsum;
          best_chunk = d3 ? ch : b.nz;
          best_kind = which == 0 ? b.stage_px : b.filter_px;
          best_ry = b.filter_ry;
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
      set_filter_tiles(c, b);
    }
  }
  c->timing = saved;
  c->stats = lee_stats{};
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return check_device_error(c);
}

__global__ void k_add_box(int nx, int ny, int lo0, int lo1, int lo2, int b0, int b1, long long nb, const double* sig,
                          double* field) {
  for (long long lb = blockIdx.x * (long long)blockDim.x + threadIdx.x; lb < nb; lb += (long long)gridDim.x * blockDim.x) {
    const int i = lo0 + (int)(lb % b0), j = lo1 + (int)((lb / b0) % b1), k = lo2 + (int)(lb / ((long long)b0 * b1));
    field[i + (long long)nx * (j + (long long)ny * k)] += sig[lb];
  }
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
  k_convert<float><<<grid1d(b.N), 256, 0, c->stream>>>(b.N, g, f);
  CK(cudaGetLastError());
  b.d_sigma_field = g;
  return LEE_OK;
}

int check_device_error(lee_ctx* c) {
  int h = 0;
  CK(cudaMemcpyAsync(&h, c->d_err, sizeof h, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (h) {
    CK(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream));
    return fail(c, LEE_ERR_TIMEOUT, "a bounded wait on a TMA transfer gave up (device flag %d)", h);
  }
  return LEE_OK;
}

// Every BC line of a block, in the order they were added, on the fields f (with the
// rounding errors e of a compensated pair, or null).
template <typename T>
int apply_bcs(lee_ctx* c, BlockData& b, void** f, void** e, double t, const double* t_tab, const int* ctr,
              int t_stride) {
  for (auto& z : b.bnd) {
    if (!is_bc_line(z.kind)) continue;
    BcParams<T> p;
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

// The Butcher tableau of RungeKutta::initialize (src/solver/temporal_discretization.cpp:33-85).
struct Tableau {
  int ns;
  double b[4], c[4], a[4];
};

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
  if (c->cfg.num_dim != 2 || c->ovs.n > 0 || c->axisym) return false;
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

// One time step (temporal::time_advance with RungeKutta::integrate) enqueued on the context
// stream: the time is incremented first (solver::solve, src/solver/solver.cpp:72), then every
// stage runs on every block, the boundary update (BC lines, overset) follows each stage, and
// the filter closes the step. amp_tab/t_tab/ctr: the monopole amplitudes and stage times of a
// replayed step graph, [step][block][stage] (null: passed by value).
template <typename T>
int step_impl(lee_ctx* c, const std::vector<double>& dts, const T* amp_tab, const double* t_tab, const int* ctr) {
  const Tableau tb = tableau(c->cfg.rk_scheme);
  const int ns = tb.ns;
  const int nbk = (int)c->blk.size();
  const double *bi = tb.b, *ci = tb.c, *aij = tb.a;
  {
    for (int q = 0; q < nbk; ++q) {
      c->blk[(size_t)q].time += dts[(size_t)q];
      c->blk[(size_t)q].step += 1;
    }
    c->time = c->blk[0].time;
    c->step = c->blk[0].step;
    if (c->batch.active) {
      int rc = batch_step<T>(c, dts, ctr != nullptr);
      if (rc) return rc;
      return trace_step<T>(c, ctr);
    }
    for (int s = 0; s < ns; ++s) {
      for (auto& b : c->blk) {
        const size_t bix = (size_t)(&b - &c->blk[0]);
        const double dt = dts[bix];
        StageParams<T> p;
        fill_stage_common<T>(c, b, p);
        p.stage = s;
        p.last = s == ns - 1;
        p.h = (T)dt;
        p.b = (T)bi[s];
        p.a = (T)aij[s];
        p.src_amp = (T)(c->src_kind != LEE_SOURCE_NONE ? source_amp(c, b, b.time + ci[s] * dt) : 0.0);
        // the replayed graph's amplitude table holds [step][block][stage]
        p.amp_tab = amp_tab ? amp_tab + bix * ns : nullptr;
        p.step_ctr = ctr;
        p.nstages = nbk * ns;
        if (c->wave_time) {
          int rc = wave_refs<T>(c, b, b.time + ci[s] * dt, t_tab ? t_tab + bix * ns + s : nullptr, ctr, nbk * ns);
          if (rc) return rc;
        }
        void** zin = s == 0 ? b.y : b.zb[(s + 1) % 2];
        void** zout = b.zb[s % 2];
        for (int v = 0; v < c->V; ++v) {
          p.zin[v] = (const T*)zin[v];
          p.yn[v] = (const T*)b.y[v];
          p.acc[v] = (T*)b.acc[v];
          p.zout[v] = (T*)zout[v];
          p.comp[v] = (T*)b.comp[v];
        }
        p.rho_prev = b.rho_valid ? (const T*)b.rho : nullptr;
        int e0 = mark(c);
        int rc = launch_stage_any<T>(c, b, p, zin);
        if (rc) return rc;
        int e1 = mark(c);
        span(c, 0, e0, e1);
        c->stats.stage_launches += 1;
        c->stats.kernel_launches += 1;
      }
      // boundary update of the stage output (spatial::update_boundary): z, or y_next after the
      // last stage (FP64: the accumulator; compensated: the pair y_pre, e)
      const bool last = s == ns - 1;
      auto target = [&](BlockData& b) -> void** { return (last && !c->comp) ? b.acc : b.zb[s % 2]; };
      auto errors = [&](BlockData& b) -> void** { return (last && c->comp) ? b.acc : nullptr; };
      // the update's time is that of the next stage, the last stage's on the last
      // (RungeKutta::integrate, src/solver/temporal_discretization.cpp:232-244)
      const int sb = std::min(s + 1, ns - 1);
      for (auto& b : c->blk) {
        const size_t bix = (size_t)(&b - &c->blk[0]);
        int rc = apply_bcs<T>(c, b, target(b), errors(b), b.time + ci[sb] * dts[bix],
                              t_tab ? t_tab + bix * ns + sb : nullptr, ctr, nbk * ns);
        if (rc) return rc;
      }
      // overset interpolation over all blocks, from their post-BC values (overset::interpolate)
      if (c->ovs.n > 0) {
        OvsParams<T> op;
        memset(&op, 0, sizeof op);
        op.n = c->ovs.n; op.W = c->ovs.W; op.V = c->V; op.fused = c->ovs.fused ? 1 : 0;
        for (int d = 0; d < 3; ++d) op.w[d] = c->ovs.w[d];
        op.rb = c->ovs.d_rb; op.rl = c->ovs.d_rl; op.db = c->ovs.d_db; op.dl = c->ovs.d_dl;
        op.wt = c->ovs.d_wt; op.buf = c->ovs.d_buf;
        op.pair = (last && c->comp) ? 1 : 0;
        for (size_t bi = 0; bi < c->blk.size(); ++bi) {
          BlockData& b = c->blk[bi];
          void** t = target(b);
          void** e = errors(b);
          for (int v = 0; v < c->V; ++v) {
            op.y[bi][v] = (T*)t[v];
            op.e[bi][v] = e ? (T*)e[v] : nullptr;
          }
          op.nx[bi] = b.nx;
          op.ny[bi] = b.ny;
        }
        CK(launch_overset<T>(op, c->stream));
        c->stats.kernel_launches += op.fused ? 1 : 2;
      }
      for (auto& b : c->blk) {
        void** tgt = target(b);
        void** err = errors(b);
        if (last && b.need_rho) {
          // rho'/rho_bar of the pre-filter state, read by the next step's first stage: the
          // reference recomputes its auxiliary fields after the boundary update and not after
          // the filter (temporal_discretization.cpp:236-242)
          CK(launch_rho<T>(b.N, c->V, (T* const*)tgt, (T* const*)err, b.d_mean[4], c->cfg.gamma, (T*)b.rho,
                           c->stream));
          b.rho_valid = true;
          c->stats.kernel_launches += 1;
        }
      }
    }
    for (auto& b : c->blk) {
      void** last_out = b.zb[(ns - 1) % 2];
      void** other = b.zb[ns % 2];
      if (c->cfg.filter_scheme != LEE_FILTER_NONE && b.tma_filter) {
        // pre-filter state (FP64: acc; compensated: y_pre with its error in acc) -> y
        int rc = c->comp ? launch_filter_fused<T>(c, b, last_out, b.acc, b.y, b.comp)
                         : launch_filter_fused<T>(c, b, b.acc, nullptr, b.y, nullptr);
        if (rc) return rc;
      } else if (c->cfg.filter_scheme != LEE_FILTER_NONE) {
        void** res = nullptr;
        int rc = c->comp ? run_filter<T>(c, b, last_out, b.acc, b.comp, other, b.y, &res)
                         : run_filter<T>(c, b, b.acc, nullptr, nullptr, last_out, other, &res);
        if (rc) return rc;
        swap_fields(c->V, b.y, res);
      } else if (!c->comp) {
        swap_fields(c->V, b.y, b.acc);
      } else {
        swap_fields(c->V, b.y, last_out);
        swap_fields(c->V, b.comp, b.acc);
      }
    }
  }
  return trace_step<T>(c, ctr);
}

__global__ void k_tick(int* ctr) { *ctr += 1; }

// The buffer roles of every block (they rotate when a step ends with a swap) and whether each
// block's rho'/rho_bar field is live: a captured step sequence replays only on the same layout.
std::vector<void*> layout_of(lee_ctx* c) {
  std::vector<void*> l;
  for (auto& b : c->blk) {
    for (int v = 0; v < c->V; ++v) {
      l.push_back(b.y[v]); l.push_back(b.acc[v]); l.push_back(b.zb[0][v]); l.push_back(b.zb[1][v]);
      l.push_back(b.comp[v]); l.push_back(b.dsum[v]);
    }
    l.push_back((void*)(uintptr_t)(b.rho_valid ? 1 : 0));
  }
  l.push_back((void*)(uintptr_t)(c->adj.trace_on ? 1 : 0));
  l.push_back(c->adj.d_trace);  // buffers a captured step reads through baked-in pointers
  l.push_back(c->adj.d_base);
  l.push_back(c->adj.d_mic);
  return l;
}

struct SavedRoles {
  std::vector<std::vector<void*>> f;
};

SavedRoles save_roles(lee_ctx* c) {
  SavedRoles r;
  for (auto& b : c->blk) {
    std::vector<void*> v;
    for (int q = 0; q < c->V; ++q) {
      v.push_back(b.y[q]); v.push_back(b.acc[q]); v.push_back(b.zb[0][q]); v.push_back(b.zb[1][q]);
      v.push_back(b.comp[q]); v.push_back(b.dsum[q]);
    }
    r.f.push_back(v);
  }
  return r;
}

void restore_roles(lee_ctx* c, const SavedRoles& r) {
  for (size_t i = 0; i < c->blk.size(); ++i) {
    BlockData& b = c->blk[i];
    const std::vector<void*>& v = r.f[i];
    for (int q = 0; q < c->V; ++q) {
      b.y[q] = v[6 * q]; b.acc[q] = v[6 * q + 1]; b.zb[0][q] = v[6 * q + 2]; b.zb[1][q] = v[6 * q + 3];
      b.comp[q] = v[6 * q + 4]; b.dsum[q] = v[6 * q + 5];
    }
  }
}

struct Clocks {
  std::vector<double> t;
  std::vector<int> n;
};

Clocks save_clocks(const lee_ctx* c) {
  Clocks k;
  for (auto& b : c->blk) {
    k.t.push_back(b.time);
    k.n.push_back(b.step);
  }
  return k;
}

void restore_clocks(lee_ctx* c, const Clocks& k) {
  for (size_t i = 0; i < c->blk.size(); ++i) {
    c->blk[i].time = k.t[i];
    c->blk[i].step = k.n[i];
  }
  c->time = c->blk[0].time;
  c->step = c->blk[0].step;
}

// Every block at time t after `step` steps (the context's lockstep clock).
void set_clock(lee_ctx* c, double t, int step) {
  for (auto& b : c->blk) {
    b.time = t;
    b.step = step;
  }
  c->time = t;
  c->step = step;
}

// Capture steps into one graph until the buffer roles come back to where they started
// (at most 4 steps), with the monopole amplitudes read from the device table.
template <typename T>
int capture_steps(lee_ctx* c, const std::vector<double>& dts) {
  auto& g = c->graph;
  if (g.exec) {
    cudaGraphExecDestroy(g.exec);
    g.exec = nullptr;
  }
  const std::vector<void*> start = layout_of(c);
  const SavedRoles roles = save_roles(c);
  const Clocks clk = save_clocks(c);
  const lee_stats st0 = c->stats;
  memset(&c->stats, 0, sizeof c->stats);
  const bool src = c->src_kind != LEE_SOURCE_NONE;
  const bool tick = src || c->adj.trace_on || c->wave_time;
  CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed));
  int rc = LEE_OK, steps = 0;
  for (; steps < 4;) {
    rc = step_impl<T>(c, dts, src ? (const T*)g.d_amp : nullptr, c->wave_time ? g.d_ttab : nullptr,
                      tick ? g.d_ctr : nullptr);
    if (rc) break;
    if (tick) {
      k_tick<<<1, 1, 0, c->stream>>>(g.d_ctr);
      c->stats.kernel_launches += 1;
    }
    ++steps;
    if (layout_of(c) == start) break;
  }
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
  const bool repeat = rc == LEE_OK && layout_of(c) == start;
  const lee_stats per = c->stats;
  restore_roles(c, roles);
  restore_clocks(c, clk);
  c->stats = st0;
  if (rc) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (e != cudaSuccess) return fail(c, LEE_ERR_CUDA, "stream capture: %s", cudaGetErrorString(e));
  if (!repeat) {  // buffer roles that never come back: keep launching step by step
    cudaGraphDestroy(graph);
    g.steps = 0;
    return LEE_OK;
  }
  e = cudaGraphInstantiate(&g.exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    g.exec = nullptr;
    return fail(c, LEE_ERR_CUDA, "graph instantiation: %s", cudaGetErrorString(e));
  }
  g.dts = dts;
  g.steps = steps;
  g.layout = start;
  g.launches = per.kernel_launches;
  g.stage_launches = per.stage_launches;
  g.filter_launches = per.filter_launches;
  return LEE_OK;
}

// lee_advance: step by step when timing kernels (events between launches), else replays of a
// captured step graph; the remainder, and a first step whose rho'/rho_bar field is not yet
// live, run step by step. dts: the time step of every block.
template <typename T>
int advance_impl(lee_ctx* c, int nsteps, const std::vector<double>& dts) {
  auto& g = c->graph;
  int done = 0;
  auto direct = [&](int n) -> int {
    for (int k = 0; k < n; ++k) {
      int rc = step_impl<T>(c, dts, nullptr, nullptr, nullptr);
      if (rc) return rc;
    }
    done += n;
    return LEE_OK;
  };
  if (!g.enabled || c->timing || nsteps < 2) return direct(nsteps);
  bool need_rho = false, rho_live = true;
  for (auto& b : c->blk) {
    need_rho |= b.need_rho != 0;
    rho_live &= !b.need_rho || b.rho_valid;
  }
  if (need_rho && !rho_live) {
    int rc = direct(1);
    if (rc) return rc;
  }
  const bool src = c->src_kind != LEE_SOURCE_NONE;
  const bool tick = src || c->adj.trace_on || c->wave_time;
  const Tableau tb = tableau(c->cfg.rk_scheme);
  const size_t nbk = c->blk.size();
  constexpr size_t kTableSteps = 4096;  // amplitude table rows: steps per chunk of replays
  if (tick && !g.d_ctr) {
    int rc = dalloc(c, &g.d_ctr, 1);
    if (rc) return rc;
    void* p = nullptr;
    if ((rc = dev_alloc(c, &p, kTableSteps * 4 * nbk * sizeof(double)))) return rc;
    g.d_amp = p;
    g.amp_cap = kTableSteps * 4 * nbk;
  }
  if (c->wave_time && !g.d_ttab) {
    int rc = dalloc(c, &g.d_ttab, kTableSteps * 4 * nbk);
    if (rc) return rc;
  }
  if (!g.exec || g.dts != dts || g.layout != layout_of(c)) {
    if (c->batch.active) {
      // the stage parameters the captured batched launches read (amplitudes from the table)
      std::vector<StageParams<T>> pr = batch_params<T>(c, dts, true, 0);
      CK(cudaMemcpy(c->batch.d_prm_graph, pr.data(), pr.size() * sizeof(pr[0]), cudaMemcpyHostToDevice));
      c->batch.graph_dts = dts;
    }
    int rc = capture_steps<T>(c, dts);
    if (rc) return rc;
  }
  if (!g.exec || g.steps < 1) return direct(nsteps - done);
  const int P = g.steps;
  const size_t chunk_steps = (size_t)P * (kTableSteps / P);
  std::vector<T> amp;
  std::vector<double> ttab;
  while (nsteps - done >= P) {
    const int reps = (int)std::min<long long>((nsteps - done) / P, (long long)(chunk_steps / P));
    const int n = reps * P;
    if (src) {
      // amplitudes at the stage times of each step of each block, [step][block][stage], with
      // every block's time advanced as its steps advance it
      amp.assign((size_t)n * nbk * tb.ns, T(0));
      for (size_t q = 0; q < nbk; ++q) {
        double t = c->blk[q].time;
        for (int k = 0; k < n; ++k) {
          t += dts[q];
          for (int s = 0; s < tb.ns; ++s)
            amp[((size_t)k * nbk + q) * tb.ns + s] = (T)source_amp(c, c->blk[q], t + tb.c[s] * dts[q]);
        }
      }
      CK(cudaMemcpyAsync(g.d_amp, amp.data(), amp.size() * sizeof(T), cudaMemcpyHostToDevice, c->stream));
    }
    if (c->wave_time) {
      // the stage times themselves, in the same layout, for the harmonic wave
      ttab.assign((size_t)n * nbk * tb.ns, 0.0);
      for (size_t q = 0; q < nbk; ++q) {
        double t = c->blk[q].time;
        for (int k = 0; k < n; ++k) {
          t += dts[q];
          for (int s = 0; s < tb.ns; ++s) ttab[((size_t)k * nbk + q) * tb.ns + s] = t + tb.c[s] * dts[q];
        }
      }
      CK(cudaMemcpyAsync(g.d_ttab, ttab.data(), ttab.size() * 8, cudaMemcpyHostToDevice, c->stream));
    }
    if (tick) CK(cudaMemsetAsync(g.d_ctr, 0, sizeof(int), c->stream));
    if (c->adj.trace_on) {
      const int base = c->adj.host_row;
      CK(cudaMemcpyAsync(c->adj.d_base, &base, sizeof(int), cudaMemcpyHostToDevice, c->stream));
      CK(cudaStreamSynchronize(c->stream));  // `base` lives on this frame
      c->adj.host_row += n;
    }
    for (int r = 0; r < reps; ++r) CK(cudaGraphLaunch(g.exec, c->stream));
    for (size_t q = 0; q < nbk; ++q)
      for (int k = 0; k < n; ++k) {
        c->blk[q].time += dts[q];
        c->blk[q].step += 1;
      }
    c->time = c->blk[0].time;
    c->step = c->blk[0].step;
    for (auto& b : c->blk)
      if (b.need_rho) b.rho_valid = true;
    c->stats.kernel_launches += g.launches * reps;
    c->stats.stage_launches += g.stage_launches * reps;
    c->stats.filter_launches += g.filter_launches * reps;
    done += n;
  }
  return direct(nsteps - done);
}

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

// Checks and buffers of the adjoint path; the operators it transposes must be the
// uniform-mean, single-block, hole-free ones.
int adjoint_setup(lee_ctx* c) {
  auto& a = c->adj;
  if (a.ready) return LEE_OK;
  if (c->blk.size() != 1) return fail(c, LEE_ERR_UNSUPPORTED, "the adjoint covers single-block contexts");
  BlockData& b = c->blk[0];
  if (b.has_iblank || c->ovs.n > 0) return fail(c, LEE_ERR_UNSUPPORTED, "the adjoint has no holes or overset");
  if (c->axisym) return fail(c, LEE_ERR_UNSUPPORTED, "the adjoint has no axisymmetric term");
  for (auto& z : b.bnd) {
    if (z.kind == LEE_SPONGE_FREUND_HARMONICWAVE)
      return fail(c, LEE_ERR_UNSUPPORTED, "the adjoint has no harmonic-wave sponge");
    if (z.kind != LEE_SPONGE_FREUND_AMBIENT) return fail(c, LEE_ERR_UNSUPPORTED, "the adjoint has no BC lines");
  }
  auto is_const = [&](const Coef<double>& d, const Coef<float>& f) { return c->comp ? !f.p : !d.p; };
  auto is_zero = [&](const Coef<double>& d, const Coef<float>& f) { return c->comp ? f.zero != 0 : d.zero != 0; };
  bool uni = is_const(b.cd_pb, b.cf_pb) && is_const(b.cd_rbi, b.cf_rbi);
  for (int q = 0; q < 3; ++q)
    uni = uni && is_const(b.cd_ub[q], b.cf_ub[q]) && is_zero(b.cd_gs[q], b.cf_gs[q]) && is_zero(b.cd_gp[q], b.cf_gp[q]);
  for (int q = 0; q < 9; ++q) uni = uni && is_zero(b.cd_gu[q], b.cf_gu[q]);
  if (!uni) return fail(c, LEE_ERR_UNSUPPORTED, "the adjoint needs a uniform mean flow");
  if (!build_transpose(c->fd, &a.dT)) return fail(c, LEE_ERR_UNSUPPORTED, "difference operator too wide to transpose");
  if (c->cfg.filter_scheme != LEE_FILTER_NONE && !build_transpose(c->flt, &a.fT))
    return fail(c, LEE_ERR_UNSUPPORTED, "filter too wide to transpose");
  // a line must keep the two ends' class rows apart, and a class row must only meet closure
  // rows of its own end: n >= 2E and n >= E + H + h
  const int n[3] = {b.nx, b.ny, b.nz};
  int need = std::max(2 * a.dT.E, a.dT.E + a.dT.H + c->fd.h);
  if (c->cfg.filter_scheme != LEE_FILTER_NONE) need = std::max(need, std::max(2 * a.fT.E, a.fT.E + a.fT.H + c->flt.h));
  for (int d = 0; d < c->cfg.num_dim; ++d)
    if (n[d] < need) return fail(c, LEE_ERR_UNSUPPORTED, "the adjoint needs %d points per direction", need);
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
    fp.k_chunk = b.filter_chunk;
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
    int bx, by;
    filter_box(c, H, b.filter_ry, &bx, &by);
    FieldMaps fm;
    int rc = field_maps(c, b, a.lam, bx, by, &fm);
    if (rc) return rc;
    const int chunks = c->cfg.num_dim == 3 ? (b.nz + fp.k_chunk - 1) / fp.k_chunk : 1;
    CK(launch_filter_tma<T>(fm, fp, H, c->cfg.num_dim, 0, b.filter_ry, filter_tiles(b), chunks, c->stream));
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
      tp.k_chunk = std::min(b.nz, 32);
      tp.err = c->d_err;
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

}  // namespace

namespace lee {
// Filter coefficient table and the context-free error message, for lee_static.cu.
bool filter_table(OpTable* o, int scheme, int order, double strength) {
  return make_filter(o, scheme, order, strength);
}
void set_global_error(const char* msg) { snprintf(g_create_error, sizeof g_create_error, "%s", msg); }
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
    c->wfl_sym = c->wfl_ok && (c->hf == 2 || c->hf == 4 || c->hf == 5);
    for (int o = 1; o <= c->hf && c->wfl_sym; ++o) c->wfl_sym = c->wfl[0][c->hf - o] == c->wfl[0][c->hf + o];
  }
  c->wst_ok = c->fd.h == kFdHalf && class_weights(c->fd, kFdHalf, &c->wst[0][0], 5);
  c->blk.resize((size_t)cfg->num_blocks);
  e = cudaSetDevice(cfg->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->d_err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(c->d_err, 0, sizeof(int));
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

int lee_set_overset(lee_ctx* c, int n, const int* recv_block, const int* recv_ijk, const int* donor_block,
                    const int* donor_ijk, const int width[3], const double* weights, int num_holes,
                    const int* hole_block, const int* hole_ijk) {
  if (!c) return LEE_ERR_ARG;
  if (c->prepared) return fail(c, LEE_ERR_STATE, "lee_set_overset after lee_prepare");
  if (n < 0 || num_holes < 0 || !width) return fail(c, LEE_ERR_ARG, "negative count or null width");
  if (n > 0 && (!recv_block || !recv_ijk || !donor_block || !donor_ijk || !weights))
    return fail(c, LEE_ERR_ARG, "null receiver arrays");
  if (num_holes > 0 && (!hole_block || !hole_ijk)) return fail(c, LEE_ERR_ARG, "null hole arrays");
  const int nb = (int)c->blk.size();
  if (nb > kMaxOvsBlocks) return fail(c, LEE_ERR_UNSUPPORTED, "overset over more than %d blocks", kMaxOvsBlocks);
  for (int d = 0; d < 3; ++d)
    if (width[d] < 1 || (d >= c->cfg.num_dim && width[d] != 1)) return fail(c, LEE_ERR_ARG, "stencil width");
  const int W = width[0] * width[1] * width[2];
  auto& o = c->ovs;
  // validate everything before touching the blocks
  for (int q = 0; q < num_holes; ++q) {
    const int b = hole_block[q];
    if (b < 0 || b >= nb || !c->blk[(size_t)b].set) return fail(c, LEE_ERR_ARG, "hole %d: block %d", q, b);
    const BlockData& bk = c->blk[(size_t)b];
    const int* ijk = hole_ijk + 3 * (size_t)q;
    if (ijk[0] < 0 || ijk[0] >= bk.nx || ijk[1] < 0 || ijk[1] >= bk.ny || ijk[2] < 0 || ijk[2] >= bk.nz)
      return fail(c, LEE_ERR_ARG, "hole %d outside its block", q);
  }
  std::vector<int> rb((size_t)n), db((size_t)n);
  std::vector<long long> rl((size_t)n), dl((size_t)n);
  std::vector<double> wt((size_t)n * W);
  for (int r = 0; r < n; ++r) {
    const int b = recv_block[r], d = donor_block[r];
    if (b < 0 || b >= nb || d < 0 || d >= nb || !c->blk[(size_t)b].set || !c->blk[(size_t)d].set)
      return fail(c, LEE_ERR_ARG, "receiver %d: block %d or donor block %d", r, b, d);
    const BlockData &rk = c->blk[(size_t)b], &dk = c->blk[(size_t)d];
    const int* ri = recv_ijk + 3 * (size_t)r;
    const int* di = donor_ijk + 3 * (size_t)r;
    const int rn[3] = {rk.nx, rk.ny, rk.nz}, dn[3] = {dk.nx, dk.ny, dk.nz};
    for (int q = 0; q < 3; ++q) {
      if (ri[q] < 0 || ri[q] >= rn[q]) return fail(c, LEE_ERR_ARG, "receiver %d outside its block", r);
      // the stencil must lie within the donor grid (initialize_donor asserts it, :536-537)
      if (di[q] < 0 || di[q] + width[q] - 1 >= dn[q])
        return fail(c, LEE_ERR_ARG, "donor stencil of receiver %d outside block %d", r, d);
    }
    rb[(size_t)r] = b;
    db[(size_t)r] = d;
    rl[(size_t)r] = ri[0] + (long long)rk.nx * (ri[1] + (long long)rk.ny * ri[2]);
    dl[(size_t)r] = di[0] + (long long)dk.nx * (di[1] + (long long)dk.ny * di[2]);
    // normalised by the sum, accumulated left to right (initialize_donor, :516-526)
    double sum = 0.0;
    for (int q = 0; q < W; ++q) sum += weights[(size_t)r * W + q];
    sum = 1.0 / sum;
    for (int q = 0; q < W; ++q) wt[(size_t)r * W + q] = weights[(size_t)r * W + q] * sum;
  }
  // holes BLANKED, then receivers INTERPOLATED (override_iblank_4holeCells / _4interpolatedCells)
  auto touch = [&](BlockData& bk) {
    if (bk.hib.empty()) bk.hib.assign((size_t)bk.N, 0);
  };
  for (int q = 0; q < num_holes; ++q) {
    BlockData& bk = c->blk[(size_t)hole_block[q]];
    touch(bk);
    const int* ijk = hole_ijk + 3 * (size_t)q;
    bk.hib[(size_t)(ijk[0] + (long long)bk.nx * (ijk[1] + (long long)bk.ny * ijk[2]))] = 1;
  }
  for (int r = 0; r < n; ++r) {
    BlockData& bk = c->blk[(size_t)rb[(size_t)r]];
    touch(bk);
    bk.hib[(size_t)rl[(size_t)r]] = -1;
  }
  for (auto& bk : c->blk) {
    if (bk.hib.empty()) continue;
    bk.has_holes = bk.has_iblank = false;
    for (int v : bk.hib) {
      bk.has_holes |= v == 1;
      bk.has_iblank |= v != 0;
    }
  }
  o.n = n;
  o.W = W;
  for (int d = 0; d < 3; ++d) o.w[d] = width[d];
  o.rb.swap(rb); o.db.swap(db); o.rl.swap(rl); o.dl.swap(dl); o.wt.swap(wt);
  return LEE_OK;
}

int lee_read_overset_file(lee_ctx* c, const char* path, int order_accuracy) {
  if (!c || !path) return LEE_ERR_ARG;
  FILE* f = fopen(path, "rb");
  if (!f) return fail(c, LEE_ERR_ARG, "cannot open overset file %s", path);
  std::unique_ptr<FILE, int (*)(FILE*)> guard(f, fclose);
  auto rd = [&](void* p, size_t sz, size_t n) { return n == 0 || fread(p, sz, n, f) == n; };
  int nd = 0, nb = 0;
  if (!rd(&nd, 4, 1) || !rd(&nb, 4, 1)) return fail(c, LEE_ERR_ARG, "short overset file");
  if (nd != c->cfg.num_dim || nb != (int)c->blk.size())
    return fail(c, LEE_ERR_ARG, "overset file has %d dimensions and %d blocks", nd, nb);
  std::vector<int> cnt((size_t)nb);
  for (int b = 0; b < nb; ++b) {
    int np = 0;
    if (!rd(&np, 4, 1)) return fail(c, LEE_ERR_ARG, "short overset file");
    if (!c->blk[(size_t)b].set || np != c->blk[(size_t)b].N)
      return fail(c, LEE_ERR_ARG, "overset file: block %d has %d points", b, np);
  }
  if (!rd(cnt.data(), 4, (size_t)nb)) return fail(c, LEE_ERR_ARG, "short overset file");
  long long R = 0;
  for (int v : cnt) {
    if (v < 0) return fail(c, LEE_ERR_ARG, "overset file: negative receiver count");
    R += v;
  }
  if (R > (1LL << 30)) return fail(c, LEE_ERR_ARG, "overset file: too many receivers");
  std::vector<int> rb((size_t)R), db((size_t)R), rijk((size_t)R * 3, 0), dijk((size_t)R * 3, 0);
  if (!rd(rb.data(), 4, (size_t)R)) return fail(c, LEE_ERR_ARG, "short overset file");
  for (long long r = 0; r < R; ++r)
    if (!rd(&rijk[(size_t)r * 3], 4, (size_t)nd)) return fail(c, LEE_ERR_ARG, "short overset file");
  if (!rd(db.data(), 4, (size_t)R)) return fail(c, LEE_ERR_ARG, "short overset file");
  for (long long r = 0; r < R; ++r)
    if (!rd(&dijk[(size_t)r * 3], 4, (size_t)nd)) return fail(c, LEE_ERR_ARG, "short overset file");
  int width[3] = {1, 1, 1};
  std::vector<double> wt;
  size_t base = 0;
  for (int b = 0; b < nb; ++b) {
    if (!rd(width, 4, 3)) return fail(c, LEE_ERR_ARG, "short overset file");
    for (int d = 0; d < nd; ++d)
      if (width[d] - 1 != order_accuracy)  // overture.cpp:609
        return fail(c, LEE_ERR_ARG, "overset stencil width %d does not match order %d", width[d], order_accuracy);
    for (int d = 0; d < 3; ++d)
      if (width[d] < 1 || width[d] > 16) return fail(c, LEE_ERR_ARG, "overset stencil width %d", width[d]);
    const size_t W = (size_t)width[0] * width[1] * width[2];
    if (wt.empty()) wt.assign((size_t)R * W, 0.0);
    if (wt.size() != (size_t)R * W) return fail(c, LEE_ERR_UNSUPPORTED, "overset stencil widths differ by block");
    if (!rd(wt.data() + base * W, 8, (size_t)cnt[(size_t)b] * W)) return fail(c, LEE_ERR_ARG, "short overset file");
    base += (size_t)cnt[(size_t)b];
  }
  std::vector<int> hc((size_t)nb);
  if (!rd(hc.data(), 4, (size_t)nb)) return fail(c, LEE_ERR_ARG, "short overset file");
  std::vector<int> hb, hijk;
  for (int b = 0; b < nb; ++b) {
    if (hc[(size_t)b] < 0) return fail(c, LEE_ERR_ARG, "overset file: negative hole count");
    hb.insert(hb.end(), (size_t)hc[(size_t)b], b);
  }
  hijk.assign(hb.size() * 3, 0);
  if (!rd(hijk.data(), 4, hijk.size())) return fail(c, LEE_ERR_ARG, "short overset file");
  return lee_set_overset(c, (int)R, rb.data(), rijk.data(), db.data(), dijk.data(), width, wt.data(), (int)hb.size(),
                         hb.data(), hijk.data());
}

int lee_get_overset(lee_ctx* c, int* recv_block, long long* recv_l0, int* donor_block, long long* donor_l0,
                    double* weights) {
  if (!c) return LEE_ERR_ARG;
  auto& o = c->ovs;
  const size_t n = (size_t)o.n;
  if (!c->prepared || n == 0) {
    // the host copies (no device arrays yet)
    if (recv_block) std::copy(o.rb.begin(), o.rb.end(), recv_block);
    if (recv_l0) std::copy(o.rl.begin(), o.rl.end(), recv_l0);
    if (donor_block) std::copy(o.db.begin(), o.db.end(), donor_block);
    if (donor_l0) std::copy(o.dl.begin(), o.dl.end(), donor_l0);
    if (weights) std::copy(o.wt.begin(), o.wt.end(), weights);
    return LEE_OK;
  }
  // what the kernels read
  CK(cudaSetDevice(c->cfg.device));
  if (recv_block) CK(cudaMemcpyAsync(recv_block, o.d_rb, n * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  if (recv_l0) CK(cudaMemcpyAsync(recv_l0, o.d_rl, n * sizeof(long long), cudaMemcpyDeviceToHost, c->stream));
  if (donor_block) CK(cudaMemcpyAsync(donor_block, o.d_db, n * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  if (donor_l0) CK(cudaMemcpyAsync(donor_l0, o.d_dl, n * sizeof(long long), cudaMemcpyDeviceToHost, c->stream));
  if (weights) CK(cudaMemcpyAsync(weights, o.d_wt, n * o.W * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return LEE_OK;
}

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
        k_convert<float><<<grid1d((long long)nb), 256, 0, s>>>((long long)nb, f, z.d_sigma);
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
          k_convert<float><<<grid1d((long long)nb), 256, 0, s>>>((long long)nb, f, b.d_src_g);
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
          k_convert<float><<<grid1d((long long)g.size()), 256, 0, s>>>((long long)g.size(), f, b.d_src_g);
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
        k_convert<float><<<grid1d((long long)g.size()), 256, 0, s>>>((long long)g.size(), f, b.d_src_g);
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
    // state buffers
    if ((rc = alloc_fields(c, b.y, b.N))) return rc;
    if ((rc = alloc_fields(c, b.acc, b.N))) return rc;
    if ((rc = alloc_fields(c, b.zb[0], b.N))) return rc;
    if ((rc = alloc_fields(c, b.zb[1], b.N))) return rc;
    if (c->comp) {
      if ((rc = alloc_fields(c, b.comp, b.N))) return rc;
      if ((rc = alloc_fields(c, b.dsum, b.N))) return rc;
    }
    // TMA-staged kernels: no holes, the 4th-order difference, rows of 16-byte multiples
    const bool rows16 = ((size_t)b.nx * c->esz) % 16 == 0;
    b.tiles_x = (b.nx + kTileX - 1) / kTileX;
    b.tiles_y = (b.ny + kTileY - 1) / kTileY;
    // (the TMA stage kernel addresses points with 32-bit offsets)
    // (and the harmonic-wave sponge, an RHS term of the generic kernel's zone loop, is absent)
    bool wave_zone = false;
    for (auto& z : b.bnd) wave_zone |= z.kind == LEE_SPONGE_FREUND_HARMONICWAVE;
    b.tma = c->wst_ok && !b.has_holes && rows16 && (unsigned long long)b.N < (1ull << 32) && !wave_zone &&
            !c->axisym;
    b.tma_filter = c->wfl_ok && !b.has_holes && rows16 && c->cfg.filter_scheme != LEE_FILTER_NONE &&
                   (unsigned long long)b.N < (1ull << 32);
    // the kernels are a fixed choice (they round differently, and two contexts of one case give
    // the same bits): the scalar fused filter unless another is asked for
    b.filter_vec = b.tma_filter && c->wfl_sym;
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
      b.stage_pair = c->comp && uni && b.nx % 2 == 0;
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
  if (c->blk.size() > 1 && batch_eligible(c)) {
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
  c->prepared = true;
  return LEE_OK;
}

namespace {

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

}  // namespace

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
      k_to_double<float><<<grid1d(bk.N), 256, 0, c->stream>>>(bk.N, tmp, (const float*)bk.y[v],
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

namespace {

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

}  // namespace

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

namespace {

// lee_advance and lee_advance_blocks: K steps timed by events on the context stream.
int advance_timed(lee_ctx* c, int nsteps, const std::vector<double>& dts) {
  CK(cudaSetDevice(c->cfg.device));
  memset(&c->stats, 0, sizeof c->stats);
  c->ev_used = 0;
  c->ev_marks.clear();
  cudaEvent_t t0, t1;
  CK(cudaEventCreate(&t0));
  CK(cudaEventCreate(&t1));
  CK(cudaEventRecord(t0, c->stream));
  int rc = c->comp ? advance_impl<float>(c, nsteps, dts) : advance_impl<double>(c, nsteps, dts);
  CK(cudaEventRecord(t1, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, t0, t1));
  c->stats.advance_ms = ms;
  for (auto& m : c->ev_marks) {
    float d = 0.f;
    if (cudaEventElapsedTime(&d, c->ev_pool[(size_t)m.second], c->ev_pool[(size_t)m.second + 1]) == cudaSuccess) {
      if (m.first == 0) c->stats.stage_ms += d;
      else c->stats.filter_ms += d;
    }
  }
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  if (rc) return rc;
  return check_device_error(c);
}

}  // namespace

int lee_advance(lee_ctx* c, int nsteps, double dt) {
  if (!c) return LEE_ERR_ARG;
  if (!c->prepared || !c->uploaded) return fail(c, LEE_ERR_STATE, "lee_prepare and lee_upload_state first");
  if (nsteps < 0 || !(dt > 0.0)) return fail(c, LEE_ERR_ARG, "nsteps >= 0 and dt > 0");
  return advance_timed(c, nsteps, std::vector<double>(c->blk.size(), dt));
}

int lee_advance_blocks(lee_ctx* c, int nsteps, const double* dt) {
  if (!c || !dt) return LEE_ERR_ARG;
  if (!c->prepared || !c->uploaded) return fail(c, LEE_ERR_STATE, "lee_prepare and lee_upload_state first");
  if (nsteps < 0) return fail(c, LEE_ERR_ARG, "nsteps >= 0");
  if (c->ovs.n > 0) return fail(c, LEE_ERR_UNSUPPORTED, "overset blocks advance with one time step");
  std::vector<double> dts(dt, dt + c->blk.size());
  for (double d : dts)
    if (!(d > 0.0)) return fail(c, LEE_ERR_ARG, "every block needs dt > 0");
  return advance_timed(c, nsteps, dts);
}

int lee_eval_rhs(lee_ctx* c, int b, double time, double* const rhs[5]) {
  if (!c) return LEE_ERR_ARG;
  if (!c->prepared || !c->uploaded) return fail(c, LEE_ERR_STATE, "lee_prepare and lee_upload_state first");
  if (b < 0 || b >= (int)c->blk.size()) return fail(c, LEE_ERR_ARG, "block index");
  CK(cudaSetDevice(c->cfg.device));
  BlockData& bk = c->blk[(size_t)b];
  double* tmp = nullptr;
  {
    const int rc = staging(c, &tmp);
    if (rc) return rc;
  }
  if (!c->comp) {
    StageParams<double> p;
    fill_stage_common<double>(c, bk, p);
    p.stage = -1;
    p.src_amp = c->src_kind != LEE_SOURCE_NONE ? source_amp(c, bk, time) : 0.0;
    if (int rc = wave_refs<double>(c, bk, time, nullptr, nullptr, 0)) return rc;
    p.rho_prev = bk.rho_valid ? (const double*)bk.rho : nullptr;
    for (int v = 0; v < c->V; ++v) {
      p.zin[v] = (const double*)bk.y[v];
      p.zout[v] = (double*)bk.zb[0][v];
    }
    int rc = launch_stage_any<double>(c, bk, p, bk.y);
    if (rc) return rc;
    for (int v = 0; v < c->V; ++v)
      CK(cudaMemcpyAsync(rhs[slot_of(c->V, v)], bk.zb[0][v], (size_t)bk.N * 8, cudaMemcpyDeviceToHost, c->stream));
  } else {
    StageParams<float> p;
    fill_stage_common<float>(c, bk, p);
    p.stage = -1;
    p.src_amp = (float)(c->src_kind != LEE_SOURCE_NONE ? source_amp(c, bk, time) : 0.0);
    if (int rc = wave_refs<float>(c, bk, time, nullptr, nullptr, 0)) return rc;
    p.rho_prev = bk.rho_valid ? (const float*)bk.rho : nullptr;
    for (int v = 0; v < c->V; ++v) {
      p.zin[v] = (const float*)bk.y[v];
      p.zout[v] = (float*)bk.zb[0][v];
    }
    int rc = launch_stage_any<float>(c, bk, p, bk.y);
    if (rc) return rc;
    for (int v = 0; v < c->V; ++v) {
      k_to_double<float><<<grid1d(bk.N), 256, 0, c->stream>>>(bk.N, tmp, (const float*)bk.zb[0][v], nullptr);
      CK(cudaMemcpyAsync(rhs[slot_of(c->V, v)], tmp, (size_t)bk.N * 8, cudaMemcpyDeviceToHost, c->stream));
    }
  }
  CK(cudaStreamSynchronize(c->stream));
  if (c->cfg.num_dim == 2) memset(rhs[3], 0, (size_t)bk.N * 8);
  return LEE_OK;
}

int lee_apply_filter(lee_ctx* c) {
  if (!c) return LEE_ERR_ARG;
  if (!c->prepared || !c->uploaded) return fail(c, LEE_ERR_STATE, "lee_prepare and lee_upload_state first");
  if (c->cfg.filter_scheme == LEE_FILTER_NONE) return LEE_OK;
  CK(cudaSetDevice(c->cfg.device));
  for (auto& b : c->blk) {
    if (b.need_rho && !b.rho_valid) {
      // the auxiliary fields keep describing the state from before the filter
      if (c->comp)
        CK(launch_rho<float>(b.N, c->V, (float* const*)b.y, (float* const*)b.comp, b.d_mean[4], c->cfg.gamma,
                             (float*)b.rho, c->stream));
      else
        CK(launch_rho<double>(b.N, c->V, (double* const*)b.y, nullptr, b.d_mean[4], c->cfg.gamma, (double*)b.rho,
                              c->stream));
      b.rho_valid = true;
    }
    if (b.tma_filter) {
      // y (and its carried error) -> zb[0], then the buffers swap roles
      int rc = c->comp ? launch_filter_fused<float>(c, b, b.y, b.comp, b.zb[0], b.comp)
                       : launch_filter_fused<double>(c, b, b.y, nullptr, b.zb[0], nullptr);
      if (rc) return rc;
      swap_fields(c->V, b.y, b.zb[0]);
      continue;
    }
    void** res = nullptr;
    int rc = c->comp ? run_filter<float>(c, b, b.y, b.comp, b.comp, b.zb[0], b.zb[1], &res)
                     : run_filter<double>(c, b, b.y, nullptr, nullptr, b.zb[0], b.zb[1], &res);
    if (rc) return rc;
    swap_fields(c->V, b.y, res);
  }
  CK(cudaStreamSynchronize(c->stream));
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
  info->filter_rows = c->blk.empty() ? 0 : c->blk[0].filter_ry;
  info->batched = c->batch.active ? 1 : 0;
  if (c->batch.active) {
    batch_shape(c->batch.sshape, &info->batch_stage_tile[0], &info->batch_stage_tile[1]);
    batch_shape(c->batch.fshape, &info->batch_filter_tile[0], &info->batch_filter_tile[1]);
  }
  return LEE_OK;
}

int lee_set_timing(lee_ctx* c, int on) {
  if (!c) return LEE_ERR_ARG;
  c->timing = on != 0;
  return LEE_OK;
}

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

namespace {

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

}  // namespace

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
  BlockData& b = c->blk[0];
  auto& a = c->adj;
  const size_t bytes = (size_t)b.N * c->esz;
  // the state slots hold the adjoint variable (with a compensated state, y + e rounded)
  for (int v = 0; v < c->V; ++v) {
    if (c->comp) {
      k_add_pair<<<grid1d(b.N), 256, 0, c->stream>>>(b.N, (float*)a.lam[v], (const float*)b.y[v],
                                                      (const float*)b.comp[v]);
      CK(cudaGetLastError());
    } else {
      CK(cudaMemcpyAsync(a.lam[v], b.y[v], bytes, cudaMemcpyDeviceToDevice, c->stream));
    }
  }
  for (int it = 0; it < nsteps; ++it) {
    rc = c->comp ? adjoint_step<float>(c, dt, nullptr, nullptr) : adjoint_step<double>(c, dt, nullptr, nullptr);
    if (rc) return rc;
  }
  for (int v = 0; v < c->V; ++v) {
    CK(cudaMemcpyAsync(b.y[v], a.lam[v], bytes, cudaMemcpyDeviceToDevice, c->stream));
    if (c->comp) CK(cudaMemsetAsync(b.comp[v], 0, bytes, c->stream));
  }
  b.rho_valid = false;
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
  if (c->adj.mic_block != 0) return fail(c, LEE_ERR_ARG, "objective block");
  CK(cudaSetDevice(c->cfg.device));
  memset(&c->stats, 0, sizeof c->stats);
  int rc = adjoint_setup(c);
  if (rc) return rc;
  auto& a = c->adj;
  BlockData& b = c->blk[0];
  const int V = c->V;
  const size_t bytes = (size_t)b.N * c->esz;
  const int K = checkpoint_every;
  const int nseg = (nsteps + K - 1) / K;
  const int fields = c->comp ? 2 * V : V;
  // checkpoint slots: the state at the start of every segment
  if (a.ckpt_slots < (size_t)nseg) {
    for (size_t q = a.ckpt.size(); q < (size_t)nseg * fields; ++q) {
      void* p = nullptr;
      if ((rc = dev_alloc(c, &p, bytes))) return rc;
      a.ckpt.push_back(p);
    }
    a.ckpt_slots = (size_t)nseg;
  }
  if ((rc = ensure_trace(c, (size_t)nsteps))) return rc;
  auto save = [&](int seg) -> int {
    for (int v = 0; v < V; ++v) {
      CK(cudaMemcpyAsync(a.ckpt[(size_t)seg * fields + v], b.y[v], bytes, cudaMemcpyDeviceToDevice, c->stream));
      if (c->comp)
        CK(cudaMemcpyAsync(a.ckpt[(size_t)seg * fields + V + v], b.comp[v], bytes, cudaMemcpyDeviceToDevice,
                           c->stream));
    }
    return LEE_OK;
  };
  auto restore = [&](int seg) -> int {
    for (int v = 0; v < V; ++v) {
      CK(cudaMemcpyAsync(b.y[v], a.ckpt[(size_t)seg * fields + v], bytes, cudaMemcpyDeviceToDevice, c->stream));
      if (c->comp)
        CK(cudaMemcpyAsync(b.comp[v], a.ckpt[(size_t)seg * fields + V + v], bytes, cudaMemcpyDeviceToDevice,
                           c->stream));
    }
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
  const long long fwd_launches = c->stats.kernel_launches;
  std::vector<double> tr((size_t)nsteps * a.mic.size());
  CK(cudaMemcpyAsync(tr.data(), a.d_trace, tr.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *J = objective_of(c, tr);
  // final state, kept aside while segments are recomputed
  const double t_end = c->time;
  const int step_end = c->step;
  std::vector<void*> fin;
  if (recompute) {
    for (int q = 0; q < fields; ++q) {
      void* p = nullptr;
      CK(cudaMallocAsync(&p, bytes, c->stream));
      fin.push_back(p);
      CK(cudaMemcpyAsync(p, q < V ? b.y[q] : b.comp[q - V], bytes, cudaMemcpyDeviceToDevice, c->stream));
    }
  }
  // reverse sweep
  const size_t nbox = (size_t)(b.src_hi[0] - b.src_lo[0] + 1) * (b.src_hi[1] - b.src_lo[1] + 1) *
                      (b.src_hi[2] - b.src_lo[2] + 1);
  if (!a.d_gbar && (rc = dalloc(c, &a.d_gbar, nbox))) return rc;
  CK(cudaMemsetAsync(a.d_gbar, 0, nbox * sizeof(double), c->stream));
  for (int v = 0; v < V; ++v) CK(cudaMemsetAsync(a.lam[v], 0, bytes, c->stream));
  const Tableau tb = tableau(c->cfg.rk_scheme);
  const size_t M = a.mic.size();
  const double scale = 2.0 * a.weight;
  const int P = V - 1;
  long long mismatches = 0;
  std::vector<double> tr2;
  for (int seg = nseg - 1; seg >= 0; --seg) {
    const int n0 = seg * K, n = std::min(K, nsteps - n0);
    if (recompute) {
      // the segment's forward steps again, from its checkpoint; their traces must repeat
      if ((rc = restore(seg))) return rc;
      set_clock(c, seg_time[(size_t)seg], step_start + n0);
      if ((rc = advance_traced(c, n, dt, n0))) return rc;
      tr2.assign((size_t)n * M, 0.0);
      CK(cudaMemcpyAsync(tr2.data(), a.d_trace + (size_t)n0 * M, tr2.size() * sizeof(double), cudaMemcpyDeviceToHost,
                         c->stream));
      CK(cudaStreamSynchronize(c->stream));
      for (size_t q = 0; q < tr2.size(); ++q) mismatches += tr2[q] != tr[(size_t)n0 * M + q];
    }
    // stage times of each step of the segment, advanced as the forward steps advance them
    std::vector<double> amps((size_t)n * tb.ns);
    double t = seg_time[(size_t)seg];
    for (int k = 0; k < n; ++k) {
      t += dt;
      for (int s = 0; s < tb.ns; ++s) amps[(size_t)k * tb.ns + s] = source_amp(c, b, t + tb.c[s] * dt);
    }
    for (int k = n - 1; k >= 0; --k) {
      const int step = n0 + k;  // 0-based: this transposed step maps the adjoint of y_{step+1} to y_step
      if (c->comp)
        CK(launch_mic_force<float>((int)M, a.d_mic, (float*)a.lam[P], a.d_trace, step, scale, c->stream));
      else
        CK(launch_mic_force<double>((int)M, a.d_mic, (double*)a.lam[P], a.d_trace, step, scale, c->stream));
      rc = c->comp ? adjoint_step<float>(c, dt, &amps[(size_t)k * tb.ns], a.d_gbar)
                   : adjoint_step<double>(c, dt, &amps[(size_t)k * tb.ns], a.d_gbar);
      if (rc) return rc;
    }
  }
  // source-box gradient -> lattice gradient
  std::vector<double> gbox(nbox);
  CK(cudaMemcpyAsync(gbox.data(), a.d_gbar, nbox * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  restrict_to_lattice(c->dsrc, c->cfg.num_dim, b.src_lo, b.src_hi, gbox.data(), grad);
  if (recompute) {
    for (int q = 0; q < fields; ++q) {
      CK(cudaMemcpyAsync(q < V ? b.y[q] : b.comp[q - V], fin[(size_t)q], bytes, cudaMemcpyDeviceToDevice, c->stream));
      CK(cudaFreeAsync(fin[(size_t)q], c->stream));
    }
    set_clock(c, t_end, step_end);
  }
  CK(cudaStreamSynchronize(c->stream));
  (void)fwd_launches;
  if (trace_mismatches) *trace_mismatches = mismatches;
  return check_device_error(c);
}

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

int lee_set_stage_kernel(lee_ctx* c, int kind) {
  if (!c) return LEE_ERR_ARG;
  if (c->prepared) return fail(c, LEE_ERR_STATE, "lee_set_stage_kernel before lee_prepare");
  if (kind != -1 && kind != 1 && kind != 2) return fail(c, LEE_ERR_ARG, "stage kernel %d", kind);
  c->stage_kernel = kind;
  return LEE_OK;
}

int lee_set_filter_kernel(lee_ctx* c, int kind) {
  if (!c) return LEE_ERR_ARG;
  if (c->prepared) return fail(c, LEE_ERR_STATE, "lee_set_filter_kernel before lee_prepare");
  if (kind < -1) return fail(c, LEE_ERR_ARG, "filter kernel %d", kind);
  c->filter_kernel = kind;
  return LEE_OK;
}

int lee_set_graphs(lee_ctx* c, int on) {
  if (!c) return LEE_ERR_ARG;
  c->graph.enabled = on != 0;
  if (!c->graph.enabled && c->graph.exec) {
    cudaSetDevice(c->cfg.device);
    cudaStreamSynchronize(c->stream);
    cudaGraphExecDestroy(c->graph.exec);
    c->graph.exec = nullptr;
  }
  return LEE_OK;
}

int lee_get_stats(lee_ctx* c, lee_stats* st) {
  if (!c || !st) return LEE_ERR_ARG;
  *st = c->stats;
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
