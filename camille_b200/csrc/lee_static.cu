// lee_filter_field_static: the filter of one field with no device allocation.
//
// Some callers cannot call cudaMalloc: a host framework that owns the whole device
// memory budget through its own caching allocator (a cudaMalloc behind its back
// fragments its pool or fails against its reservation), a solver loop that must not pay
// allocation latency or synchronization inside a time step, or code running in a
// partition with a fixed memory quota. lee_apply_filter needs a context, whose buffers
// are allocated by lee_prepare; this entry point applies the same dimension-split filter
// (spatial::apply_filter for one variable, camille src/solver/spatial_discretization.cpp:2191-2246,
// without holes) to a field the caller already holds on the device, writing a field the
// caller provides, and keeps the intermediate passes in a scratch array that is part of
// the library image: a file-scope __device__ array of kStaticFilterPoints doubles per pass
// (2 x 8 MiB), which every GPU that loads the library holds until the process exits.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "lee_internal.h"

namespace lee {
namespace {

constexpr long long kStaticFilterPoints = 1LL << 20;  // largest field (points) the scratch holds

// Intermediate results of the xi and eta passes.
static __device__ __align__(256) double g_filter_scratch[2][kStaticFilterPoints];

// Device address of g_filter_scratch per device: in host code the symbol is only a
// host-side stand-in, so its address is looked up once per device, with that device current.
constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_addr[kMaxDevices] = {};

// The device a pointer's memory lives on, or -1 when CUDA does not know it as device memory.
int device_of(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    (void)cudaGetLastError();  // the lookup's error is not sticky: clear it
    return -1;
  }
  return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) ? a.device : -1;
}

int scratch_for_current_device(const void* d_in, const void* d_out, double** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0) {
    set_global_error("lee_filter_field_static: no current CUDA device");
    return LEE_ERR_NODEVICE;
  }
  if (dev >= kMaxDevices) {
    char msg[128];
    snprintf(msg, sizeof msg, "lee_filter_field_static: device %d is beyond the %d devices the library serves", dev,
             kMaxDevices);
    set_global_error(msg);
    return LEE_ERR_UNSUPPORTED;
  }
  if (device_of(d_in) != dev || device_of(d_out) != dev) {
    set_global_error("lee_filter_field_static: d_in and d_out must be device memory of the current device");
    return LEE_ERR_ARG;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_filter_scratch);
    if (e != cudaSuccess || !p) {
      char msg[256];
      snprintf(msg, sizeof msg, "lee_filter_field_static: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
      set_global_error(msg);
      return LEE_ERR_CUDA;
    }
    g_scratch_addr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_addr[dev];
  return LEE_OK;
}

}  // namespace
}  // namespace lee

using namespace lee;

extern "C" int lee_filter_field_static(int num_dim, int filter_scheme, int filter_order, double filter_strength,
                                       double filter_blend, int nxi, int neta, int nzeta, const double* d_in,
                                       double* d_out, void* stream) {
  char msg[256];
  if (!d_in || !d_out || d_in == d_out) {
    set_global_error("lee_filter_field_static: distinct non-null device input and output are required");
    return LEE_ERR_ARG;
  }
  if ((num_dim != 2 && num_dim != 3) || (num_dim == 2 && nzeta != 1)) {
    set_global_error("lee_filter_field_static: num_dim must be 2 (nzeta = 1) or 3");
    return LEE_ERR_ARG;
  }
  OpTable op;
  const double strength = filter_scheme == LEE_FILTER_STANDARD_CENTRAL ? 1.0 : filter_strength;
  if (filter_scheme == LEE_FILTER_NONE || !(strength >= 0.0 && strength <= 1.0) ||
      !(filter_blend >= 0.0 && filter_blend <= 1.0) || !filter_table(&op, filter_scheme, filter_order, strength)) {
    set_global_error("lee_filter_field_static: unsupported filter scheme, order, strength or blend");
    return LEE_ERR_UNSUPPORTED;
  }
  const long long n = (long long)nxi * neta * nzeta;
  const int dims[3] = {nxi, neta, nzeta};
  const int need = std::max(2 * op.h + 1, op.S);
  for (int d = 0; d < 3; ++d) {
    if (dims[d] < 1 || (d < num_dim && dims[d] < need)) {
      snprintf(msg, sizeof msg, "lee_filter_field_static: direction %d has %d points, the filter needs %d", d,
               dims[d], need);
      set_global_error(msg);
      return LEE_ERR_ARG;
    }
  }
  if (n > kStaticFilterPoints) {
    snprintf(msg, sizeof msg,
             "lee_filter_field_static: %lld points exceed the static scratch of %lld points; use lee_apply_filter",
             n, kStaticFilterPoints);
    set_global_error(msg);
    return LEE_ERR_ARG;
  }
  // input and output ranges must not share any element: the passes read neighbours of
  // every point of d_in while the last one writes d_out
  const uintptr_t a0 = (uintptr_t)d_in, a1 = a0 + (uintptr_t)n * sizeof(double);
  const uintptr_t b0 = (uintptr_t)d_out, b1 = b0 + (uintptr_t)n * sizeof(double);
  if (a0 < b1 && b0 < a1) {
    set_global_error("lee_filter_field_static: the input and output ranges overlap");
    return LEE_ERR_ARG;
  }
  double* scratch = nullptr;
  int rc = scratch_for_current_device(d_in, d_out, &scratch);
  if (rc) return rc;
  // Every pass writes each scratch element it hands to the next pass, so nothing needs
  // clearing between calls. Calls that overlap on the GPU share the scratch and race.
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const double* src = d_in;
  for (int d = 0; d < num_dim; ++d) {
    FilterParams<double> fp;
    memset(&fp, 0, sizeof fp);
    fp.nx = nxi;
    fp.ny = neta;
    fp.nz = nzeta;
    fp.V = 1;
    fp.dir = d;
    fp.first = d == 0;
    fp.last = d == num_dim - 1;
    fp.blend = filter_blend;
    fp.op = op;
    double* dst = fp.last ? d_out : scratch + (size_t)(d % 2) * (size_t)kStaticFilterPoints;
    fp.in[0] = src;
    fp.out[0] = dst;
    fp.y0[0] = d_in;
    cudaError_t e = launch_filter_pass<double>(fp, 0, s);
    if (e != cudaSuccess) {
      snprintf(msg, sizeof msg, "lee_filter_field_static: launch failed: %s", cudaGetErrorString(e));
      set_global_error(msg);
      return LEE_ERR_CUDA;
    }
    src = dst;
  }
  return LEE_OK;
}
