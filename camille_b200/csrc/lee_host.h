// Host side of the C ABI: the context (lee_ctx), its blocks, and the helpers that the host
// translation units (lee_capi.cu, lee_host_*.cu) share.
#pragma once

#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include <algorithm>
#include <map>
#include <memory>

#include "lee_internal.h"
#include "lee_tma.h"

using namespace lee;

namespace lee {

// the kernels' default limit of a wait on staged data: one second
constexpr unsigned long long kDefaultWaitNs = 1000000000ull;

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
  bool filter_pair_ok = false;        // the two-point compensated filter (lee_filter_pair.cu) applies
  bool filter_pair = false;           // ... and runs the block's fused filter (form 3)
  int ptiles_x = 0, ptiles_y = 0;     // its tiles
  int tfilter_ry = 1, tfilter_chunk = 0;  // the scalar form and chunk of the adjoint's transposed filter
  // passive scalars (LEE_SCALAR): mean fields and their gradients, and the slots' buffers with
  // the LEE slots' roles (y, acc, two stage buffers, carried error, filter increments) plus a
  // filter scratch; fixed roles, nothing swaps
  std::vector<double> hzmean;         // n x N host copy
  double* d_zmean[kMaxScalars] = {};
  double* d_zgrad[kMaxScalars * 3] = {};
  Coef<double> cd_gz[kMaxScalars][3];
  Coef<float> cf_gz[kMaxScalars][3];
  void* zy[kMaxScalars] = {};
  void* zacc[kMaxScalars] = {};
  void* zzb[2][kMaxScalars] = {};
  void* zcomp[kMaxScalars] = {};
  void* zdsum[kMaxScalars] = {};
  void* zf[kMaxScalars] = {};
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

}  // namespace lee

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
  int nsc = 0;               // lee_set_scalars: passive scalar slots
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
  double wst[6][5] = {};   // stage classes: interior, 2 left, 2 right, the zero class (holes)
  double wfl[12][11] = {};  // filter classes: interior, nb left, nb right, the zero class (holes)
  int hf = 0;
  bool wst_ok = false, wfl_ok = false;
  bool wfl_sym = false;  // symmetric interior filter stencil: the vectorised filter kernel applies
  int filter_kernel = -1;  // lee_set_filter_kernel: -1/0 scalar, else vector group width
  int stage_kernel = -1;   // lee_set_stage_kernel: -1 default, else points per thread
  int filter_form = 0;     // lee_set_filter_form: 0 timed at setup, else the scalar filter's form
  // blocks of a multi-block context run their stage and filter launches on side streams, forked
  // from the context stream and joined before whatever couples the blocks (overset, the clock)
  bool concurrent = true;       // lee_set_block_streams
  bool batching = true;         // lee_set_batching: eligible batches run the batched kernels
  bool increment_step = false;  // lee_set_increment_step (measured slower on the B200: off)
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> side_ev;  // [0] the fork, [1 + q] the join of side stream q
  int* d_err = nullptr;          // [0] a bounded wait gave up, [1] a non-finite state value was found
  unsigned long long wait_ns = kDefaultWaitNs;  // limit of the kernels' waits on staged data
  int finite_every = 0;          // lee_set_finite_check: steps between checks (0: end of each advance, -1: off)
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
    // lee_set_batch_persistent: -1 the per-phase launches, else the shape of the one persistent
    // launch per step, its work list and its grid barrier (two words)
    int pshape = -1;
    int4* d_ptiles = nullptr;
    int npt = 0;
    unsigned* d_gbar = nullptr;
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
    size_t gbar_n = 0;
    std::vector<void*> ckpt;               // checkpoints: V (+ V carried errors) fields each
    size_t ckpt_slots = 0;
    bool tma = false;                      // the plane-marching stage kernel (lee_adjoint_tma.cu)
    bool tma_jm = false;                   // ... with J*metrics fields (else constants)
    bool fused_filter = false;             // F^T by the fused filter kernel (lee_tma.cu)
    cudaStream_t rev = nullptr;            // the reverse sweep's stream when segments are recomputed
    cudaEvent_t ev_fwd = nullptr, ev_rev = nullptr;
    // the general path (lee_adjoint_gen.cu): every block, holes, BC lines, overset, any mean flow
    bool gen = false;
    struct GenBlock {
      void *lam[kMaxVars] = {}, *mu[kMaxVars] = {}, *kb[2][kMaxVars] = {}, *ybar[kMaxVars] = {};
      void *nu[kMaxVars] = {}, *g[3][kMaxVars] = {};
      void* rb[2] = {};                    // adjoint of rho'/rho_bar: [0] carried in, [1] produced
    };
    std::vector<GenBlock> gb;
    bool rb_live = false;                  // gb[].rb[0] holds the next step's rho' adjoint
    int ovs_nd = 0;                        // donor points of the transposed overset gather
    int *d_ub = nullptr, *d_off = nullptr, *d_cr = nullptr;
    long long* d_ul = nullptr;
    double *d_cw = nullptr, *d_otmp = nullptr;
    std::vector<void*> rho_ckpt;           // rho'/rho_bar at each checkpoint (blocks that need it)
  } adj;
};

#define CK(call)                                                                       \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return fail(c, LEE_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));   \
  } while (0)

namespace lee {

// message of the calling thread's last failure outside a context
extern thread_local char g_create_error[512];

// The Butcher tableau of RungeKutta::initialize (src/solver/temporal_discretization.cpp:33-85).
struct Tableau {
  int ns;
  double b[4], c[4], a[4];
};

struct SavedRoles {
  std::vector<std::vector<void*>> f;
};

struct Clocks {
  std::vector<double> t;
  std::vector<int> n;
};

int fail(lee_ctx* c, int code, const char* fmt, ...);
bool is_sponge(int kind);
bool is_bc_line(int kind);
bool reads_inward(int kind);
bool reads_wave(int kind);
int dev_alloc(lee_ctx* c, void** p, size_t bytes);
bool make_fd(OpTable* o, int scheme, int order);
bool make_filter(OpTable* o, int scheme, int order, double strength);
OpTable minus_identity(const OpTable& f);
bool closure_codes(const OpTable& op, const BlockData& b, int d, std::vector<int8_t>& code);
int mark(lee_ctx* c);
void span(lee_ctx* c, int kind, int a, int b);
int grid1d(long long n);
int classify(lee_ctx* c, const double* d_field, long long N, double scale, double* lo, double* hi, bool* uniform,
             bool* zero);
template <typename T>
int make_coef(lee_ctx* c, BlockData& b, const double* d_field, double scale, Coef<T>* out);
int upload(lee_ctx* c, double** d, const std::vector<double>& h);
int alloc_fields(lee_ctx* c, void** f, long long N);
int slot_of(int V, int v);
template <typename T>
void fill_stage_common(lee_ctx* c, BlockData& b, StageParams<T>& p);
bool distributed_box(const std::vector<double>& p, int dim, int nx, int ny, int nz, int lo[3], int hi[3]);
void lattice_weights(double i, double o, double h, int cn, int* p0, double* f);
void prolong(const std::vector<double>& p, int dim, const int lo[3], const int hi[3], const double* A,
             std::vector<double>& g);
void restrict_to_lattice(const std::vector<double>& p, int dim, const int lo[3], const int hi[3], const double* gbar,
                         double* abar);
const double* monopole_of(const lee_ctx* c, const BlockData& b);
void jet2d_constants(double gamma, double* amp, double* omega, double* bx, double* by);
double source_amp(const lee_ctx* c, const BlockData& b, double t);
bool class_weights(const OpTable& op, int H, double* w, int stride);
Tableau tableau(int rk);
int compute_metrics(lee_ctx* c, BlockData& b);
int build_sigma_field(lee_ctx* c, BlockData& b);
template <typename T>
int run_filter(lee_ctx* c, BlockData& b, void** in, void** err, void** comp_out, void** f0, void** f1,
               void*** result);
void swap_fields(int V, void** a, void** b);
int ensure_encoder(lee_ctx* c);
int encode_maps(lee_ctx* c, const BlockData& b, const void* const* fields, int n, int bx, int by, CUtensorMap* out);
int field_maps(lee_ctx* c, const BlockData& b, void* const* fields, int bx, int by, FieldMaps* out);
int filter_form_rows(int form);
int filter_box(const lee_ctx* c, int h, int form, int* bx, int* by);
int filter_tiles(const BlockData& b);
int filter_tiles_form(const BlockData& b, int ry);  // the scalar fused filter's tiles in form ry (1 or 2)
void set_filter_tiles(const lee_ctx* c, BlockData& b);
template <typename T>
int launch_stage_any(lee_ctx* c, BlockData& b, const StageParams<T>& p, void* const* zin, int chunk_override = 0);
template <typename T>
int launch_filter_fused(lee_ctx* c, BlockData& b, void* const* in, void* const* err, void* const* out,
                        void* const* comp_out, int chunk_override = 0, void* const* inc = nullptr);
// the compensated form's last stage may write the step's increment alone and leave y_pre to the
// fused filter (lee_set_increment_step): on blocks where nothing acts between the two
bool increment_step_applies(const lee_ctx* c, const BlockData& b);
template <typename T>
int autotune(lee_ctx* c, BlockData& b);
int check_device_error(lee_ctx* c);
int check_finite(lee_ctx* c);
int fork_sides(lee_ctx* c);
int join_sides(lee_ctx* c);
template <typename T>
void fill_bc_params(lee_ctx* c, const BlockData& b, const Boundary& z, void** f, void** e, BcParams<T>& p);
template <typename T>
int apply_bcs(lee_ctx* c, BlockData& b, void** f, void** e, double t, const double* t_tab, const int* ctr,
              int t_stride);
template <typename T>
int wave_refs(lee_ctx* c, BlockData& b, double t, const double* t_tab, const int* ctr, int t_stride);
template <typename T>
int trace_step(lee_ctx* c, const int* ctr);
bool batch_eligible(const lee_ctx* c);
std::vector<int4> batch_tiles(const lee_ctx* c, int shape);
template <typename T>
std::vector<StageParams<T>> batch_params(lee_ctx* c, const std::vector<double>& dts, bool graph, int rhs_only);
template <typename T>
std::vector<BatchFilterInst<T>> batch_filter_inst(lee_ctx* c, bool scratch);
template <typename T>
int batch_launch_stage(lee_ctx* c, const void* prm, const int4* tiles, int nt, int shape, int grid);
template <typename T>
int batch_launch_filter(lee_ctx* c, const void* inst, const int4* tiles, int nt, int shape, int grid);
template <typename T>
int batch_setup(lee_ctx* c);
template <typename T>
int batch_step(lee_ctx* c, const std::vector<double>& dts, bool graph);
template <typename T>
int step_impl(lee_ctx* c, const std::vector<double>& dts, const T* amp_tab, const double* t_tab, const int* ctr);
std::vector<void*> layout_of(lee_ctx* c);
SavedRoles save_roles(lee_ctx* c);
void restore_roles(lee_ctx* c, const SavedRoles& r);
Clocks save_clocks(const lee_ctx* c);
void restore_clocks(lee_ctx* c, const Clocks& k);
void set_clock(lee_ctx* c, double t, int step);
template <typename T>
int capture_steps(lee_ctx* c, const std::vector<double>& dts);
template <typename T>
int advance_impl(lee_ctx* c, int nsteps, const std::vector<double>& dts);
int advance_timed(lee_ctx* c, int nsteps, const std::vector<double>& dts);
int adjoint_setup(lee_ctx* c);
template <typename T>
int adjoint_step(lee_ctx* c, double dt, const double* amps, double* gbar);
// passive scalars (lee_host_scalar.cu): setup at lee_prepare, and per stage s of ns the update,
// BC rows and overset of the scalar slots (lee_zin: the LEE stage input, for u'), then the filter
int scalar_setup(lee_ctx* c, BlockData& b);
template <typename T>
int scalar_stage(lee_ctx* c, BlockData& b, int s, int ns, double h, double bcoef, double acoef, void* const* lee_zin);
template <typename T>
int scalar_bcs(lee_ctx* c, BlockData& b, int s, int ns);
template <typename T>
int scalar_overset(lee_ctx* c, int s, int ns);
template <typename T>
int scalar_filter(lee_ctx* c, BlockData& b, int ns);
// the general path (lee_host_adjoint_gen.cu)
bool adjoint_fast_applies(lee_ctx* c, const char** why);
int adjoint_gen_setup(lee_ctx* c);
// one transposed step of every block; rho_in: the forward step's first stage read rho'/rho_bar
// of the previous step (its adjoint is produced and carried to the next transposed step)
template <typename T>
int adjoint_step_gen(lee_ctx* c, double dt, const double* amps, double* gbar, bool rho_in);
int ensure_trace(lee_ctx* c, size_t rows);
int advance_traced(lee_ctx* c, int nsteps, double dt, int row0);
double objective_of(const lee_ctx* c, const std::vector<double>& tr);

// FP64 staging field of compensated uploads, downloads and right-hand sides (lee_capi.cu)
int staging(lee_ctx* c, double** out);

template <typename P>
int dalloc(lee_ctx* c, P** p, size_t count) {
  return dev_alloc(c, reinterpret_cast<void**>(p), count * sizeof(P));
}

template <typename T>
void** as_void(T** p) {
  return reinterpret_cast<void**>(p);
}

template <typename T>
void launch_convert(cudaStream_t s, long long n, T* out, const double* in);
template <typename T>
void launch_to_double(cudaStream_t s, long long n, double* out, const T* y, const T* comp);
// flag = 1 when some value of the V fields f (and e, when given) of n elements of esz bytes is
// not finite
cudaError_t launch_nonfinite(cudaStream_t s, long long n, int V, size_t esz, void* const* f, void* const* e,
                             int* flag);

}  // namespace lee
