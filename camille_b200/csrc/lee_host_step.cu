// The time-advance schedule (temporal::time_advance, camille src/solver/temporal_discretization.cpp:334-374):
// one step of all blocks, step graphs captured once per time step and buffer layout and replayed,
// and the advance, right-hand-side and filter entry points.
//
// Schedule of one step:
//   time += dt (solver::solve increments before advancing, src/solver/solver.cpp:72)
//   for each RK stage s: one fused stage kernel per block (RHS + RK update, reading the
//     stage input with its stencil neighbours and writing the next stage input and the
//     accumulator), then the boundary conditions of the stage output
//   filter passes (dimension split, src/solver/spatial_discretization.cpp:2191-2246)
//   hole mask (temporal::iblank_correction, :380-393)
#include "lee_host.h"

using namespace lee;

namespace {

__global__ void k_tick(int* ctr) { *ctr += 1; }

}  // namespace

namespace lee {

// The fork of the side streams from the context stream, and their join back into it (in a
// captured step graph these become the graph's parallel branches).
int fork_sides(lee_ctx* c) {
  CK(cudaEventRecord(c->side_ev[0], c->stream));
  for (auto sd : c->side) CK(cudaStreamWaitEvent(sd, c->side_ev[0], 0));
  return LEE_OK;
}

int join_sides(lee_ctx* c) {
  for (size_t q = 0; q < c->side.size(); ++q) {
    CK(cudaEventRecord(c->side_ev[1 + q], c->side[q]));
    CK(cudaStreamWaitEvent(c->stream, c->side_ev[1 + q], 0));
  }
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
    // blocks are independent within a stage (their BC lines included) and within the filter:
    // with several blocks each one's launches go to a side stream of their own
    const bool conc = c->concurrent && nbk > 1 && !c->timing && !c->side.empty();
    cudaStream_t origin = c->stream;
    for (int s = 0; s < ns; ++s) {
      const bool last = s == ns - 1;
      auto target = [&](BlockData& b) -> void** { return (last && !c->comp) ? b.acc : b.zb[s % 2]; };
      auto errors = [&](BlockData& b) -> void** { return (last && c->comp) ? b.acc : nullptr; };
      // the update's time is that of the next stage, the last stage's on the last
      // (RungeKutta::integrate, src/solver/temporal_discretization.cpp:232-244)
      const int sb = std::min(s + 1, ns - 1);
      if (conc) {
        int rc = fork_sides(c);
        if (rc) return rc;
      }
      for (auto& b : c->blk) {
        const size_t bix = (size_t)(&b - &c->blk[0]);
        const double dt = dts[bix];
        if (conc) c->stream = c->side[bix % c->side.size()];
        StageParams<T> p;
        fill_stage_common<T>(c, b, p);
        p.stage = s;
        p.last = s == ns - 1;
        p.increment = p.last && increment_step_applies(c, b) ? 1 : 0;
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
          if (rc) {
            c->stream = origin;
            return rc;
          }
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
        if (rc) {
          c->stream = origin;
          return rc;
        }
        int e1 = mark(c);
        span(c, 0, e0, e1);
        c->stats.stage_launches += 1;
        c->stats.kernel_launches += 1;
        // the passive scalars' stage reads u' of this stage's input
        if ((rc = scalar_stage<T>(c, b, s, ns, dt, bi[s], aij[s], zin))) {
          c->stream = origin;
          return rc;
        }
        // boundary update of the stage output (spatial::update_boundary): z, or y_next after the
        // last stage (FP64: the accumulator; compensated: the pair y_pre, e); BC lines touch their
        // own block only
        rc = apply_bcs<T>(c, b, target(b), errors(b), b.time + ci[sb] * dts[bix],
                          t_tab ? t_tab + bix * ns + sb : nullptr, ctr, nbk * ns);
        if (!rc) rc = scalar_bcs<T>(c, b, s, ns);
        c->stream = origin;
        if (rc) return rc;
      }
      if (conc) {
        int rc = join_sides(c);
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
        int rc = scalar_overset<T>(c, s, ns);
        if (rc) return rc;
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
    if (conc) {
      int rc = fork_sides(c);
      if (rc) return rc;
    }
    for (auto& b : c->blk) {
      void** last_out = b.zb[(ns - 1) % 2];
      void** other = b.zb[ns % 2];
      if (conc) c->stream = c->side[(size_t)(&b - &c->blk[0]) % c->side.size()];
      if (increment_step_applies(c, b)) {
        // the last stage left the increment in acc: y_n and the increment in, the filtered state
        // and its rounding error out (into the free stage buffer, which becomes y)
        int rc = launch_filter_fused<T>(c, b, b.y, nullptr, last_out, b.comp, 0, b.acc);
        if (rc) {
          c->stream = origin;
          return rc;
        }
        swap_fields(c->V, b.y, last_out);
      } else if (c->cfg.filter_scheme != LEE_FILTER_NONE && b.tma_filter) {
        // pre-filter state (FP64: acc; compensated: y_pre with its error in acc) -> y
        int rc = c->comp ? launch_filter_fused<T>(c, b, last_out, b.acc, b.y, b.comp)
                         : launch_filter_fused<T>(c, b, b.acc, nullptr, b.y, nullptr);
        if (rc) {
          c->stream = origin;
          return rc;
        }
      } else if (c->cfg.filter_scheme != LEE_FILTER_NONE) {
        void** res = nullptr;
        int rc = c->comp ? run_filter<T>(c, b, last_out, b.acc, b.comp, other, b.y, &res)
                         : run_filter<T>(c, b, b.acc, nullptr, nullptr, last_out, other, &res);
        if (rc) {
          c->stream = origin;
          return rc;
        }
        swap_fields(c->V, b.y, res);
      } else if (!c->comp) {
        swap_fields(c->V, b.y, b.acc);
      } else {
        swap_fields(c->V, b.y, last_out);
        swap_fields(c->V, b.comp, b.acc);
      }
      int rc = scalar_filter<T>(c, b, ns);
      c->stream = origin;
      if (rc) return rc;
    }
    if (conc) {
      int rc = join_sides(c);
      if (rc) return rc;
    }
  }
  return trace_step<T>(c, ctr);
}

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
  // chunks of lee_set_finite_check's interval, each followed by the non-finite sentinel; a
  // chunk that finds a NaN or an infinity ends the call (at the end of each call by default)
  const int every = c->finite_every > 0 ? c->finite_every : std::max(nsteps, 1);
  int rc = LEE_OK;
  for (int done = 0; done < nsteps && !rc;) {
    const int n = std::min(every, nsteps - done);
    rc = c->comp ? advance_impl<float>(c, n, dts) : advance_impl<double>(c, n, dts);
    done += n;
    if (rc || c->finite_every < 0) continue;
    rc = check_finite(c);
    if (!rc && done < nsteps) {
      int bad = 0;
      CK(cudaMemcpyAsync(&bad, c->d_err + 1, sizeof bad, cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
      if (bad) break;
    }
  }
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

// the host translation units use both precisions
template int step_impl<float>(lee_ctx* c, const std::vector<double>& dts, const float* amp_tab, const double* t_tab, const int* ctr);
template int step_impl<double>(lee_ctx* c, const std::vector<double>& dts, const double* amp_tab, const double* t_tab, const int* ctr);
template int capture_steps<float>(lee_ctx* c, const std::vector<double>& dts);
template int capture_steps<double>(lee_ctx* c, const std::vector<double>& dts);
template int advance_impl<float>(lee_ctx* c, int nsteps, const std::vector<double>& dts);
template int advance_impl<double>(lee_ctx* c, int nsteps, const std::vector<double>& dts);

}  // namespace lee

extern "C" {

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
      launch_to_double<float>(c->stream, bk.N, tmp, (const float*)bk.zb[0][v], nullptr);
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
    if (c->nsc) {
      // the scalar slots: y (and its carried error) take the pre-filter roles, then the filter
      const int ns = tableau(c->cfg.rk_scheme).ns;
      const size_t bytes = (size_t)b.N * c->esz;
      for (int k = 0; k < c->nsc; ++k) {
        CK(cudaMemcpyAsync(c->comp ? b.zzb[(ns - 1) % 2][k] : b.zacc[k], b.zy[k], bytes, cudaMemcpyDeviceToDevice,
                           c->stream));
        if (c->comp) CK(cudaMemcpyAsync(b.zacc[k], b.zcomp[k], bytes, cudaMemcpyDeviceToDevice, c->stream));
      }
      int rc = c->comp ? scalar_filter<float>(c, b, ns) : scalar_filter<double>(c, b, ns);
      if (rc) return rc;
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

int lee_set_timing(lee_ctx* c, int on) {
  if (!c) return LEE_ERR_ARG;
  c->timing = on != 0;
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

int lee_set_wait_limit(lee_ctx* c, double seconds) {
  if (!c) return LEE_ERR_ARG;
  if (!(seconds <= 10.0)) return fail(c, LEE_ERR_ARG, "wait limit %g s: at most 10 s", seconds);
  const unsigned long long ns = seconds < 0.0 ? kDefaultWaitNs : (unsigned long long)(seconds * 1e9);
  if (ns != c->wait_ns && c->graph.exec) {
    // captured launches hold the old limit in their parameters
    CK(cudaSetDevice(c->cfg.device));
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaGraphExecDestroy(c->graph.exec));
    c->graph.exec = nullptr;
  }
  c->wait_ns = ns;
  return LEE_OK;
}

int lee_set_increment_step(lee_ctx* c, int on) {
  if (!c) return LEE_ERR_ARG;
  if ((on != 0) != c->increment_step && c->graph.exec) {  // captured steps hold the old launches
    CK(cudaSetDevice(c->cfg.device));
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaGraphExecDestroy(c->graph.exec));
    c->graph.exec = nullptr;
  }
  c->increment_step = on != 0;
  return LEE_OK;
}

int lee_set_block_streams(lee_ctx* c, int on) {
  if (!c) return LEE_ERR_ARG;
  if ((on != 0) != c->concurrent && c->graph.exec) {  // captured graphs hold the old branches
    CK(cudaSetDevice(c->cfg.device));
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaGraphExecDestroy(c->graph.exec));
    c->graph.exec = nullptr;
  }
  c->concurrent = on != 0;
  return LEE_OK;
}

int lee_set_batching(lee_ctx* c, int on) {
  if (!c) return LEE_ERR_ARG;
  if (c->prepared) return fail(c, LEE_ERR_STATE, "lee_set_batching before lee_prepare");
  c->batching = on != 0;
  return LEE_OK;
}

int lee_set_finite_check(lee_ctx* c, int every) {
  if (!c) return LEE_ERR_ARG;
  if (every < -1) return fail(c, LEE_ERR_ARG, "finite-check interval %d", every);
  c->finite_every = every;
  return LEE_OK;
}

int lee_get_stats(lee_ctx* c, lee_stats* st) {
  if (!c || !st) return LEE_ERR_ARG;
  *st = c->stats;
  return LEE_OK;
}

}  // extern "C"
