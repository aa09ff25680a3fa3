// The general discrete adjoint's host side: per-block buffers, the transposed overset lists, and
// one transposed step of every block (the kernels and the algebra are in lee_adjoint_gen.cu).
// The reference has no adjoint.
#include "lee_host.h"

using namespace lee;

namespace lee {

// The uniform-mean single-block path (lee_adjoint.cu, lee_adjoint_tma.cu) applies: one block, no
// holes, receivers, BC lines, harmonic-wave sponge or axisymmetric term, a uniform mean flow.
bool adjoint_fast_applies(lee_ctx* c, const char** why) {
  auto no = [&](const char* w) {
    if (why) *why = w;
    return false;
  };
  if (c->blk.size() != 1) return no("several blocks");
  BlockData& b = c->blk[0];
  if (b.has_iblank || c->ovs.n > 0) return no("holes or overset");
  if (c->axisym) return no("the axisymmetric term");
  for (auto& z : b.bnd) {
    if (z.kind == LEE_SPONGE_FREUND_HARMONICWAVE) return no("a harmonic-wave sponge");
    if (z.kind != LEE_SPONGE_FREUND_AMBIENT) return no("BC lines");
  }
  auto is_const = [&](const Coef<double>& d, const Coef<float>& f) { return c->comp ? !f.p : !d.p; };
  auto is_zero = [&](const Coef<double>& d, const Coef<float>& f) { return c->comp ? f.zero != 0 : d.zero != 0; };
  bool uni = is_const(b.cd_pb, b.cf_pb) && is_const(b.cd_rbi, b.cf_rbi);
  for (int q = 0; q < 3; ++q)
    uni = uni && is_const(b.cd_ub[q], b.cf_ub[q]) && is_zero(b.cd_gs[q], b.cf_gs[q]) && is_zero(b.cd_gp[q], b.cf_gp[q]);
  for (int q = 0; q < 9; ++q) uni = uni && is_zero(b.cd_gu[q], b.cf_gu[q]);
  if (!uni) return no("a non-uniform mean flow");
  if (why) *why = nullptr;
  return true;
}

// Buffers of the general path: per block lam, mu, two stage adjoints, ybar, zbar and the fluxes
// G^d (V fields each), the rho' adjoints of blocks that read rho'/rho_bar; the overset transpose
// as lists per donor point, in receiver order.
int adjoint_gen_setup(lee_ctx* c) {
  auto& a = c->adj;
  const int nbk = (int)c->blk.size();
  if (nbk > kMaxOvsBlocks) return fail(c, LEE_ERR_UNSUPPORTED, "the adjoint covers up to %d blocks", kMaxOvsBlocks);
  a.gb.assign((size_t)nbk, {});
  int rc;
  for (int bi = 0; bi < nbk; ++bi) {
    BlockData& b = c->blk[(size_t)bi];
    auto& g = a.gb[(size_t)bi];
    if ((rc = alloc_fields(c, g.lam, b.N)) || (rc = alloc_fields(c, g.mu, b.N)) ||
        (rc = alloc_fields(c, g.kb[0], b.N)) || (rc = alloc_fields(c, g.kb[1], b.N)) ||
        (rc = alloc_fields(c, g.ybar, b.N)) || (rc = alloc_fields(c, g.nu, b.N)))
      return rc;
    for (int d = 0; d < c->cfg.num_dim; ++d)
      if ((rc = alloc_fields(c, g.g[d], b.N))) return rc;
    if (b.need_rho)
      for (int q = 0; q < 2; ++q) {
        if ((rc = dev_alloc(c, &g.rb[q], (size_t)b.N * c->esz))) return rc;
        CK(cudaMemsetAsync(g.rb[q], 0, (size_t)b.N * c->esz, c->stream));
      }
  }
  auto& o = c->ovs;
  if (o.n > 0) {
    // the receivers are distinct points (each forward value is overwritten once)
    std::vector<std::pair<int, long long>> recv((size_t)o.n);
    for (int r = 0; r < o.n; ++r) recv[(size_t)r] = {o.rb[(size_t)r], o.rl[(size_t)r]};
    std::sort(recv.begin(), recv.end());
    for (size_t q = 1; q < recv.size(); ++q)
      if (recv[q] == recv[q - 1]) return fail(c, LEE_ERR_UNSUPPORTED, "the adjoint needs distinct overset receivers");
    // (donor block, donor point, receiver, weight), grouped by donor point in receiver order
    struct Tap {
      int b;
      long long l;
      int r;
      double c;
    };
    std::vector<Tap> taps;
    taps.reserve((size_t)o.n * o.W);
    for (int r = 0; r < o.n; ++r) {
      const int db = o.db[(size_t)r];
      const long long nx = c->blk[(size_t)db].nx, nxy = nx * c->blk[(size_t)db].ny;
      int st = 0;
      for (int w3 = 0; w3 < o.w[2]; ++w3)
        for (int w2 = 0; w2 < o.w[1]; ++w2)
          for (int w1 = 0; w1 < o.w[0]; ++w1)
            taps.push_back({db, o.dl[(size_t)r] + w1 + w2 * nx + w3 * nxy, r, o.wt[(size_t)r * o.W + st++]});
    }
    std::stable_sort(taps.begin(), taps.end(), [](const Tap& x, const Tap& y) {
      if (x.b != y.b) return x.b < y.b;
      if (x.l != y.l) return x.l < y.l;
      return x.r < y.r;
    });
    std::vector<int> ub, off, cr;
    std::vector<long long> ul;
    std::vector<double> cw;
    for (size_t q = 0; q < taps.size(); ++q) {
      if (q == 0 || taps[q].b != taps[q - 1].b || taps[q].l != taps[q - 1].l) {
        ub.push_back(taps[q].b);
        ul.push_back(taps[q].l);
        off.push_back((int)q);
      }
      cr.push_back(taps[q].r);
      cw.push_back(taps[q].c);
    }
    off.push_back((int)taps.size());
    a.ovs_nd = (int)ub.size();
    if ((rc = dalloc(c, &a.d_ub, ub.size())) || (rc = dalloc(c, &a.d_ul, ul.size())) ||
        (rc = dalloc(c, &a.d_off, off.size())) || (rc = dalloc(c, &a.d_cr, cr.size())) ||
        (rc = dalloc(c, &a.d_cw, cw.size())) || (rc = dalloc(c, &a.d_otmp, (size_t)o.n * c->V)))
      return rc;
    CK(cudaMemcpyAsync(a.d_ub, ub.data(), ub.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(a.d_ul, ul.data(), ul.size() * sizeof(long long), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(a.d_off, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(a.d_cr, cr.data(), cr.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(a.d_cw, cw.data(), cw.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  a.rb_live = false;
  a.gen = true;
  a.ready = true;
  return LEE_OK;
}

namespace {

template <typename T>
AdjGenPoint<T> point_ops(lee_ctx* c, BlockData& b) {
  AdjGenPoint<T> p;
  memset(&p, 0, sizeof p);
  p.iblank = b.has_holes ? b.d_iblank : nullptr;
  p.pbar = b.d_mean[4];
  p.inv_gamma = (T)(1.0 / c->cfg.gamma);
  return p;
}

// w <- B^T O^T w on every block: the overset transpose over all blocks (the forward interpolates
// after every block's BC lines), then each block's BC lines in the reverse of their order.
template <typename T>
int boundary_t(lee_ctx* c, void** (*pick)(lee_ctx*, int, void*), void* ctx) {
  auto& a = c->adj;
  const int nbk = (int)c->blk.size();
  if (c->ovs.n > 0) {
    AdjGenOvs<T> op;
    memset(&op, 0, sizeof op);
    op.n = c->ovs.n;
    op.nd = a.ovs_nd;
    op.V = c->V;
    op.rb = c->ovs.d_rb;
    op.rl = c->ovs.d_rl;
    op.ub = a.d_ub;
    op.ul = a.d_ul;
    op.off = a.d_off;
    op.cw = a.d_cw;
    op.cr = a.d_cr;
    op.tmp = a.d_otmp;
    for (int bi = 0; bi < nbk; ++bi) {
      void** f = pick(c, bi, ctx);
      for (int v = 0; v < c->V; ++v) op.y[bi][v] = (T*)f[v];
    }
    CK(launch_adjg_overset<T>(op, c->stream));
    c->stats.kernel_launches += 2;
  }
  for (int bi = 0; bi < nbk; ++bi) {
    BlockData& b = c->blk[(size_t)bi];
    void** f = pick(c, bi, ctx);
    for (auto it = b.bnd.rbegin(); it != b.bnd.rend(); ++it) {
      if (!is_bc_line(it->kind)) continue;
      BcParams<T> p;
      fill_bc_params<T>(c, b, *it, f, nullptr, p);
      CK(launch_adjg_bc<T>(p, c->stream));
      c->stats.kernel_launches += 1;
    }
  }
  return LEE_OK;
}

void** pick_mu(lee_ctx* c, int bi, void*) { return c->adj.gb[(size_t)bi].mu; }
void** pick_nu(lee_ctx* c, int bi, void*) { return c->adj.gb[(size_t)bi].nu; }

}  // namespace

template <typename T>
int adjoint_step_gen(lee_ctx* c, double dt, const double* amps, double* gbar, bool rho_in) {
  auto& a = c->adj;
  const Tableau tb = tableau(c->cfg.rk_scheme);
  const int ns = tb.ns;
  const int V = c->V;
  const int nbk = (int)c->blk.size();
  const int src_blk = c->src_kind == LEE_SOURCE_DISTRIBUTED ? (int)c->dsrc[0] : -1;
  // mu = F^T M lam + R^T rb (the filter passes in the reverse of the forward's order)
  for (int bi = 0; bi < nbk; ++bi) {
    BlockData& b = c->blk[(size_t)bi];
    auto& g = a.gb[(size_t)bi];
    const T* rb = (a.rb_live && b.need_rho) ? (const T*)g.rb[0] : nullptr;
    const int n[3] = {b.nx, b.ny, b.nz};
    int dirs[3], nd = 0;
    for (int d = 0; d < c->cfg.num_dim; ++d)
      if (n[d] > 1) dirs[nd++] = d;
    if (c->cfg.filter_scheme != LEE_FILTER_NONE && nd > 0) {
      void** src = g.lam;
      for (int q = nd - 1; q >= 0; --q) {
        AdjGenFilterParams<T> fp;
        memset(&fp, 0, sizeof fp);
        fp.nx = b.nx; fp.ny = b.ny; fp.nz = b.nz; fp.V = V;
        fp.dir = dirs[q];
        fp.last = q == 0;
        fp.iblank = b.has_holes ? b.d_iblank : nullptr;
        fp.mask_in = (q == nd - 1 && fp.iblank) ? 1 : 0;
        fp.code = b.has_holes ? b.d_code_flt[dirs[q]] : nullptr;
        fp.op = c->flt;
        fp.blend = (T)c->cfg.filter_blend;
        fp.rb = fp.last ? rb : nullptr;
        fp.pbar = b.d_mean[4];
        fp.inv_gamma = (T)(1.0 / c->cfg.gamma);
        void** dst = fp.last ? g.mu : g.kb[q % 2];
        for (int v = 0; v < V; ++v) {
          fp.in[v] = (const T*)src[v];
          fp.out[v] = (T*)dst[v];
          fp.lam[v] = (const T*)g.lam[v];
        }
        CK(launch_adjg_filter<T>(fp, c->stream));
        c->stats.kernel_launches += 1;
        src = dst;
      }
    } else {
      AdjGenPoint<T> p = point_ops<T>(c, b);
      p.rb = rb;
      for (int v = 0; v < V; ++v) {
        p.in[v] = (const T*)g.lam[v];
        p.out[v] = (T*)g.mu[v];
      }
      CK(launch_adjg_mask<T>(b.N, V, p, c->stream));
      c->stats.kernel_launches += 1;
    }
  }
  // mu = M P^T mu, and ybar starts from it
  int rc = boundary_t<T>(c, pick_mu, nullptr);
  if (rc) return rc;
  for (int bi = 0; bi < nbk; ++bi) {
    BlockData& b = c->blk[(size_t)bi];
    auto& g = a.gb[(size_t)bi];
    if (b.has_holes) {
      AdjGenPoint<T> p = point_ops<T>(c, b);
      for (int v = 0; v < V; ++v) {
        p.in[v] = (const T*)g.mu[v];
        p.out[v] = (T*)g.mu[v];
      }
      CK(launch_adjg_mask<T>(b.N, V, p, c->stream));
      c->stats.kernel_launches += 1;
    }
    for (int v = 0; v < V; ++v)
      CK(cudaMemcpyAsync(g.ybar[v], g.mu[v], (size_t)b.N * c->esz, cudaMemcpyDeviceToDevice, c->stream));
  }
  // the stages, last to first: kbar_{S-1} = h b_{S-1} mu (as the scale of mu), then
  // zbar_s = L_s^T kbar_s, nu_s = M P^T zbar_s, kbar_{s-1} = h b_{s-1} mu + a_{s-1} h nu_s
  int cur = 0;
  for (int s = ns - 1; s >= 0; --s) {
    const bool top = s == ns - 1;
    for (int bi = 0; bi < nbk; ++bi) {
      BlockData& b = c->blk[(size_t)bi];
      auto& g = a.gb[(size_t)bi];
      AdjGenParams<T> p;
      memset(&p, 0, sizeof p);
      fill_stage_common<T>(c, b, p.f);
      p.f.stage = s;
      p.scale = top ? (T)(dt * tb.b[ns - 1]) : T(1);
      for (int v = 0; v < V; ++v) {
        p.kin[v] = (const T*)(top ? g.mu[v] : g.kb[cur][v]);
        p.zbar[v] = (T*)g.nu[v];
        for (int d = 0; d < c->cfg.num_dim; ++d) p.g[d][v] = (T*)g.g[d][v];
      }
      p.rbar = (s == 0 && rho_in && b.need_rho) ? (T*)g.rb[1] : nullptr;
      p.gbar = (bi == src_blk) ? gbar : nullptr;
      p.amp = amps ? amps[s] : 0.0;
      CK(launch_adjg_stage<T>(p, c->stream));
      c->stats.kernel_launches += 2;
    }
    if (s > 0) {
      if ((rc = boundary_t<T>(c, pick_nu, nullptr))) return rc;
    }
    for (int bi = 0; bi < nbk; ++bi) {
      BlockData& b = c->blk[(size_t)bi];
      auto& g = a.gb[(size_t)bi];
      AdjGenPoint<T> p = point_ops<T>(c, b);
      if (s == 0) p.iblank = nullptr;  // z_0 = y: no mask, no boundary update
      for (int v = 0; v < V; ++v) {
        p.in[v] = (const T*)g.nu[v];
        p.mu[v] = (const T*)g.mu[v];
        p.ybar[v] = (T*)g.ybar[v];
        p.out[v] = s > 0 ? (T*)g.kb[top ? 0 : 1 - cur][v] : nullptr;
      }
      const double hb = s > 0 ? dt * tb.b[s - 1] : 0.0;
      const double ha = s > 0 ? tb.a[s - 1] * dt : 0.0;
      CK(launch_adjg_combine<T>(b.N, V, p, hb, ha, c->stream));
      c->stats.kernel_launches += 1;
    }
    cur = top ? 0 : 1 - cur;
  }
  for (int bi = 0; bi < nbk; ++bi) {
    auto& g = a.gb[(size_t)bi];
    swap_fields(V, g.lam, g.ybar);
    if (rho_in) std::swap(g.rb[0], g.rb[1]);
  }
  a.rb_live = rho_in;
  return LEE_OK;
}

template int adjoint_step_gen<float>(lee_ctx* c, double dt, const double* amps, double* gbar, bool rho_in);
template int adjoint_step_gen<double>(lee_ctx* c, double dt, const double* amps, double* gbar, bool rho_in);

}  // namespace lee
