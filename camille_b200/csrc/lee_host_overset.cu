// Overset maps (overset::initialize_overset, camille src/overset/overset.cpp:56-84): from arrays or
// from the Overture file (read_overset_at_headrank, src/io/overture.cpp:473-680), and the maps the
// GPU holds.
#include "lee_host.h"

using namespace lee;

extern "C" {

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

}  // extern "C"
