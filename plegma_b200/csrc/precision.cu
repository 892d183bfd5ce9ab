// Split-FP16 form: orchestration of the FP32 site contraction and the
// tensor-core projection (project_split.cu) for one or more requests.
//
// Per chunk of time slices (from one or many requests):
//   1. per-slice exponents E_u, E_d from a strided sample of each propagator;
//   2. FP32 contraction of the inputs scaled by 2^-E, plus max |c_k| per slice;
//   3. hi+lo FP16 projection GEMM on tcgen05 with FP32 accumulation in TMEM;
//   4. FP64 reduction over site splits, pair recombination
//        S(+-h) = (Cc_re +- Cs_im) + i (Cc_im -+ Cs_re),
//      exact un-scaling by 2^(n_u E_u + n_d E_d - s_k), and the source phase
//      C(p) = exp(i p.x0) S(p).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "ctx.h"
#include "p2_common.cuh"

using namespace p2host;

namespace {

// powers (n_u, n_d) of the flavour scales carried by each component
std::vector<int> component_exponents(unsigned what) {
  std::vector<int> e;
  auto push = [&](int n, int nu, int nd) {
    for (int i = 0; i < n; i++) {
      e.push_back(nu);
      e.push_back(nd);
    }
  };
  for (unsigned bit : {(unsigned)P2_NUCLEON_CG5, (unsigned)P2_NUCLEON_NTOR, (unsigned)P2_NUCLEON_RTON,
                       (unsigned)P2_NUCLEON_RTOR})
    if (what & bit) {
      push(16, 2, 1);  // proton: u u d
      push(16, 1, 2);  // neutron: d d u
    }
  if (what & P2_DELTA_ISO12)
    for (int g = 0; g < 3; g++) {
      push(16, 2, 1);
      push(16, 1, 2);
    }
  if (what & P2_DELTA_ISO32)
    for (int g = 0; g < 3; g++) {
      push(16, 3, 0);
      push(16, 0, 3);
    }
  if (what & P2_MESON_G16) push(256, 1, 1);
  if (what & P2_MESON_ALL34) push(34, 1, 1);
  if (what & P2_MESON_NEW10) push(10, 1, 1);
  if (what & P2_MESON_DIAG10) {
    push(10, 2, 0);
    push(10, 0, 2);
  }
  return e;
}

struct PhaseRows {
  std::vector<int> reps;     // unique representatives, 3 ints each
  std::vector<int> row_h;    // per row: representative index
  std::vector<int> row_sin;  // per row: 0 cos, 1 sin
  std::vector<int> mom_row;  // per momentum: cos row, sin row, sign
  std::vector<int> mom_rep;  // per momentum: its representative
};

PhaseRows phase_rows(const std::vector<int>& moms) {
  PhaseRows pr;
  const int n = (int)moms.size() / 3;
  std::vector<int> cos_row, sin_row;
  for (int p = 0; p < n; p++) {
    int v[3] = {moms[3 * p], moms[3 * p + 1], moms[3 * p + 2]};
    int sg = 1;
    for (int d = 0; d < 3; d++)
      if (v[d] != 0) {
        sg = v[d] > 0 ? 1 : -1;
        break;
      }
    int h[3] = {sg * v[0], sg * v[1], sg * v[2]};
    int idx = -1;
    for (size_t q = 0; q < pr.reps.size() / 3; q++)
      if (pr.reps[3 * q] == h[0] && pr.reps[3 * q + 1] == h[1] && pr.reps[3 * q + 2] == h[2]) idx = (int)q;
    if (idx < 0) {
      idx = (int)pr.reps.size() / 3;
      pr.reps.insert(pr.reps.end(), h, h + 3);
      cos_row.push_back((int)pr.row_h.size());
      pr.row_h.push_back(idx);
      pr.row_sin.push_back(0);
      if (h[0] || h[1] || h[2]) {
        sin_row.push_back((int)pr.row_h.size());
        pr.row_h.push_back(idx);
        pr.row_sin.push_back(1);
      } else {
        sin_row.push_back(-1);
      }
    }
    pr.mom_row.push_back(cos_row[idx]);
    pr.mom_row.push_back(sin_row[idx]);
    pr.mom_row.push_back(sg);
    pr.mom_rep.push_back(idx);
  }
  return pr;
}

}  // namespace

namespace p2 {

// Phase tiles, momentum rows and component exponents, rebuilt only when the
// momentum list or the contraction set changes (the tiles have origin 0, so
// every source shares them).  what = 0: tiles and rows only.
p2_status split_prepare_tables(p2_ctx* c, const Plan& pl, unsigned what, int& nmtile, int& nkstep) {
  PhaseRows pr = phase_rows(pl.moms);
  const int nh = (int)pr.reps.size() / 3;
  const int nrows = (int)pr.row_h.size();
  nmtile = (nrows + 127) / 128;
  nkstep = (int)((c->V3 + 63) / 64);
  p2_status st;
  if (c->split_moms_key != pl.moms) {
    c->split_moms_key.clear();
    std::vector<double> tabh = phase_tables(c, pr.reps.data(), nh, -1, pl.Lmax);
    if ((st = upload_async(c, c->tab, tabh.data(), tabh.size() * sizeof(double), "phase table")) != P2_OK) return st;
    std::vector<int> rows(pr.row_h);
    rows.insert(rows.end(), pr.row_sin.begin(), pr.row_sin.end());
    if ((st = upload_async(c, c->rowtab, rows.data(), rows.size() * sizeof(int), "phase rows")) != P2_OK) return st;
    P2_TRY(c, c->phaseA.ensure((size_t)nmtile * nkstep * 2 * 128 * 64 * 2), "phase tiles alloc");
    p2::PhaseBuildArgs b{};
    b.tab = (const double*)c->tab.p;
    b.row_h = (const int*)c->rowtab.p;
    b.row_sin = (const int*)c->rowtab.p + nrows;
    b.nrows = nrows;
    b.nmtile = nmtile;
    b.nkstep = nkstep;
    b.V3 = (int)c->V3;
    b.Lx = c->Ll[0];
    b.Ly = c->Ll[1];
    b.Lmax = pl.Lmax;
    b.nh = nh;
    b.A = c->phaseA.p;
    {
      ProfScope ps(c, "build_phase_tiles");
      P2_TRY(c, p2::launch_build_phases(b, c->stream), "phase tiles");
    }
    // [nmom][6]: cos row, sin row, sign, p; then the momenta of each
    // representative (+h and -h share its rows): [nrep + 1] starts, [nmom] indices
    std::vector<int> mr;
    for (int p = 0; p < pl.nmom; p++) {
      for (int q = 0; q < 3; q++) mr.push_back(pr.mom_row[3 * p + q]);
      for (int q = 0; q < 3; q++) mr.push_back(pl.moms[3 * p + q]);
    }
    mr.push_back(0);
    for (int r = 0; r < nh; r++) {
      int cnt = 0;
      for (int p = 0; p < pl.nmom; p++) cnt += pr.mom_rep[p] == r;
      mr.push_back(mr.back() + cnt);
    }
    for (int r = 0; r < nh; r++)
      for (int p = 0; p < pl.nmom; p++)
        if (pr.mom_rep[p] == r) mr.push_back(p);
    c->split_nrep = nh;
    if ((st = upload_async(c, c->momrow, mr.data(), mr.size() * sizeof(int), "momentum rows")) != P2_OK) return st;
    c->split_moms_key = pl.moms;
  }
  if (what && c->split_what_key != what) {
    // [K][2] scale powers, then [K] unit phases i^q of the 16 x 16 mesons
    // that the contraction leaves out (g16_phase_deferred; with g16_raw the
    // components are colour products and the Gamma sums, phases included,
    // come after the reduction)
    std::vector<int> ke = component_exponents(what);
    const int K = (int)ke.size() / 2;
    ke.resize(3 * (size_t)K, 0);
    if (g16_phase_deferred(what) && !g16_raw(what)) {
      const int k0 = offsets_of(what).g16;
      for (int g1 = 0; g1 < 16; g1++)
        for (int g2 = 0; g2 < 16; g2++) ke[2 * K + k0 + 16 * g1 + g2] = meson_phase_q(g1, g2);
    }
    if ((st = upload_async(c, c->kexp, ke.data(), ke.size() * sizeof(int), "component exponents")) != P2_OK) return st;
    c->split_what_key = what;
  }
  return P2_OK;
}

// Projection of a chunk's FP32 position buffer c->cbuf ([n][K][V3], maxima in
// c->cmaxb) on the tensor cores, launch shape from the autotuner, then the
// FP64 reduction into the results of the slices dsl: per component k the
// un-scaling exponent is kexp[2k] (exps[2t] + eh_u) + kexp[2k+1] (exps[2t+1] + eh_d).
// With no blocks the results go to out[tau * oT + k * oK + p].
p2_status split_project(p2_ctx* c, const Plan& pl, int K, int n, int nmtile, int nkstep, const SliceDesc* dsl,
                        const int* exps, const int* kexp, const std::vector<ScatterBlock>& blocks, double* out,
                        long long oT, long long oK, const int* kphase) {
  // projection GEMM candidates (N-tile width NT <= project_split_max_nt()
  // components, a multiple of 8; number of N-tiles, site splits, k-steps per
  // split): the fewest N-tiles at ~2 waves first, then up to two more N-tiles
  // at 1, 2 and 4 waves, and for each N-tile count the two smallest split
  // counts whose last wave is at least 95 % full (the CTAs, one per SM, all
  // take about as long, so a launch lasts whole waves: at 32 slices of 4
  // N-tiles, 2, 3 or 5 splits fill 86 % of their last wave, 8 splits 99 %)
  std::vector<std::vector<int>> cands;
  const int maxnt = p2::project_split_max_nt();
  for (int ntile = (K + maxnt - 1) / maxnt, extra = 0; extra < 3; ntile++, extra++) {
    const int NT = ((K + ntile - 1) / ntile + 7) / 8 * 8;
    if ((ntile - 1) * NT >= K) continue;  // an empty N-tile
    const int per = ntile * nmtile * n;
    auto add = [&](int nsplit) {
      const int ks_per = (nkstep + nsplit - 1) / nsplit;
      nsplit = (nkstep + ks_per - 1) / ks_per;
      std::vector<int> v{NT, ntile, nsplit, ks_per};
      if (std::find(cands.begin(), cands.end(), v) == cands.end()) cands.push_back(v);
      return nsplit;
    };
    for (int waves : {2, 1, 4}) add(std::min(std::max(1, (waves * c->nsm + per - 1) / per), nkstep));
    for (int ns = 1, found = 0; ns <= std::min(nkstep, 64) && found < 2; ns++) {
      const double w = (double)per * ns / c->nsm;
      if (w < 1.0 || w > 16.0 || w / std::ceil(w) < 0.95) continue;
      if (add(ns) == ns) found++;
    }
  }
  size_t maxpart = 0;
  for (const auto& v : cands) maxpart = std::max(maxpart, (size_t)v[2] * v[1] * 2 * v[0]);
  P2_TRY(c, c->fpart.ensure((size_t)n * nmtile * 128 * maxpart * sizeof(float)), "partials alloc");
  p2::SplitGemmArgs g{};
  g.c = c->cbuf.p;
  g.cmax = (const int*)c->cmaxb.p;
  g.A = c->phaseA.p;
  g.ntau = n;
  g.K = K;
  g.V3 = (int)c->V3;
  g.nkstep = nkstep;
  g.nmtile = nmtile;
  g.part = (float*)c->fpart.p;
  g.err = (int*)c->errflag.p;
  g.wait_limit = 0;  // the kernel's default time limit
  auto set = [&](p2::SplitGemmArgs& q, const std::vector<int>& v) {
    q.NT = v[0];
    q.ntile = v[1];
    q.nsplit = v[2];
    q.ks_per_split = v[3];
  };
  char key[160];
  std::snprintf(key, sizeof(key), "project_split V3=%lld K=%d rows=%d n=%d", c->V3, K, nmtile * 128, n);
  std::vector<int> pick;
  P2_TRY(c,
         tune_choose(c->tuner.get(), key, cands, c->stream, !c->capturing,
                     [&](const std::vector<int>& v) {
                       p2::SplitGemmArgs q = g;
                       set(q, v);
                       return p2::launch_project_split(q, c->stream);
                     },
                     pick),
         "projection tuning");
  set(g, pick);
  if (c->wait_test) {  // p2_debug_wait_timeout: this launch's waits run out (after tuning, which launches normally)
    g.withhold = 1;
    g.wait_limit = 20000000;  // 20 ms
    c->wait_test = 0;
  }
  const int NT = g.NT, nsplit = g.nsplit;
  const int ncols = g.ntile * 2 * NT;
  {
    ProfScope ps(c, "project_split_tc");
    P2_TRY(c, p2::launch_project_split(g, c->stream), "tensor-core projection");
  }
  p2::SplitReduceArgs rd{};
  rd.part = (const float*)c->fpart.p;
  rd.ntau = n;
  rd.nsplit = nsplit;
  rd.nmtile = nmtile;
  rd.ncols = ncols;
  rd.NT = NT;
  rd.nmom = pl.nmom;
  rd.K = K;
  rd.mom_row = (const int*)c->momrow.p;
  rd.nrep = c->split_nrep;
  rd.rep_start = rd.mom_row + 6 * pl.nmom;
  rd.rep_moms = rd.rep_start + c->split_nrep + 1;
  for (int d = 0; d < 3; d++) rd.L[d] = c->g.L[d];
  rd.cmax = (const int*)c->cmaxb.p;
  rd.exps = exps;
  rd.kexp = kexp;
  rd.kphase = kphase;
  rd.sl = dsl;
  if (blocks.size() > (size_t)p2::kMaxBlocks) return c->fail(P2_ERR_INVALID_ARG, "too many result blocks");
  rd.nblocks = (int)blocks.size();
  for (size_t b = 0; b < blocks.size(); b++) rd.blk[b] = blocks[b];
  rd.out = out;
  rd.oT = oT;
  rd.oK = oK;
  {
    ProfScope ps(c, "split_reduce");
    P2_TRY(c, p2::launch_split_reduce(rd, c->stream), "split reduction");
  }
  return P2_OK;
}

p2_status precision_run_batch(p2_ctx* c, const p2_prop* props, const p2_request* reqs, const int* idx, int nidx,
                              const Plan& pl, double* const* outs) {
  if (!c->errflag.p) {
    P2_TRY(c, c->errflag.ensure(16), "error flag alloc");
    P2_TRY(c, cudaMemsetAsync(c->errflag.p, 0, 16, c->stream), "error flag clear");
  }
  if (c->project_split_smem_max < p2::project_split_smem_bytes(p2::project_split_max_nt()))
    return c->fail(P2_ERR_UNSUPPORTED, "device shared memory per block too small for the tensor-core projection");
  const p2_request& r0 = reqs[idx[0]];
  const unsigned what = r0.contractions;
  for (int q = 0; q < nidx; q++) {
    const p2_request& r = reqs[idx[q]];
    if (props[r.prop_u].precision != props[r.prop_d].precision)
      return c->fail(P2_ERR_UNSUPPORTED, "u and d must share a precision");
  }
  // FP64 views that all live on the host are converted to FP32 on the host
  // (the contraction computes in FP32 either way; half the bytes cross PCIe)
  bool all_host64 = true;
  for (int q = 0; q < nidx; q++) {
    const p2_request& r = reqs[idx[q]];
    for (int pi : {r.prop_u, r.prop_d})
      all_host64 = all_host64 && props[pi].location == P2_HOST && props[pi].precision == P2_FP64;
  }
  const int fp32_in = props[r0.prop_u].precision == P2_FP32;
  const int K = pl.K;
  int nmtile = 0, nkstep = 0;
  p2_status st = split_prepare_tables(c, pl, what, nmtile, nkstep);
  if (st != P2_OK) return st;

  // chunk of slices: FP32 position buffer within the workspace budget; a
  // chunk may hold slices of many requests (a batch of sources), so up to
  // all of the batch's slices go into one chunk
  const size_t per_slice = (size_t)K * c->V3 * 8;
  size_t nslices = 0;
  for (int q = 0; q < nidx; q++) nslices += (size_t)std::max(reqs[idx[q]].totalT, 0);
  int tc = (int)std::max<size_t>(1, std::min<size_t>(c->ws_budget / std::max<size_t>(per_slice, 1),
                                                   std::max<size_t>(nslices, 1)));
  if (all_host64) tc = std::min(tc, 4);  // short chunks: the host conversion pipeline fills and drains faster
  const Work w = make_work(c, props, reqs, idx, nidx, tc);
  if (w.sl.empty()) return P2_OK;
  const int mx = w.max_n;
  P2_TRY(c, c->cbuf.ensure((size_t)mx * per_slice), "position buffer alloc");
  P2_TRY(c, c->expb.ensure((size_t)2 * mx * sizeof(int)), "exponent alloc");
  P2_TRY(c, c->cmaxb.ensure((size_t)mx * K * sizeof(int)), "maxima alloc");
  Stager sg(c, props, reqs, w);
  sg.cvt32 = all_host64;
  if ((st = sg.prepare(outs)) != P2_OK) return st;

  for (int i = 0; i < 2; i++)
    if ((st = sg.issue(i)) != P2_OK) return st;
  for (size_t ci = 0; ci < w.chunks.size(); ci++) {
    const int n = w.chunks[ci].n;
    const SliceDesc* dsl = sg.desc((int)ci);
    if ((st = sg.wait((int)ci)) != P2_OK) return st;
    const int chunk_fp32 = fp32_in || sg.converts((int)ci);  // staged in FP32
    {
      ProfScope ps(c, "sample_exponents");
      p2::SampleArgs sa{dsl, chunk_fp32, (int)c->V3, n, (int*)c->expb.p};
      P2_TRY(c, p2::launch_sample_exponents(sa, c->stream), "exponent sample");
    }
    P2_TRY(c, cudaMemsetAsync(c->cmaxb.p, 0, (size_t)n * K * sizeof(int), c->stream), "maxima clear");
    p2::ContractArgs a{};
    a.sl = dsl;
    a.V3 = (int)c->V3;
    a.ntau = n;
    a.what = what;
    a.K = K;
    a.k = offsets_of(what);
    a.out = c->cbuf.p;
    a.exps = (const int*)c->expb.p;
    a.cmax = (int*)c->cmaxb.p;
    a.g16_raw = g16_raw(what) ? 1 : 0;
    {
      ProfScope ps(c, "contract_f32");
      P2_TRY(c, p2::launch_contract_f32(a, chunk_fp32, 2 * c->nsm, c->stream), "contract kernel");
    }
    if ((st = sg.release((int)ci)) != P2_OK) return st;
    if ((st = sg.issue((int)ci + 2)) != P2_OK) return st;
    const int* kexp = (const int*)c->kexp.p;
    if ((st = split_project(c, pl, K, n, nmtile, nkstep, dsl, (const int*)c->expb.p, kexp, pl.blocks, nullptr, 0,
                            0, g16_phase_deferred(what) ? kexp + 2 * K : nullptr)) != P2_OK)
      return st;
    if (g16_raw(what)) {
      // the Gamma sums of the 16 x 16 block on its projected colour products
      p2::MesonGammaArgs mg{};
      mg.sl = dsl;
      mg.ntau = n;
      mg.nmom = pl.nmom;
      bool found = false;
      for (const auto& b : pl.blocks)
        if (b.comps == 256) {
          mg.blk = b;
          found = true;
        }
      if (!found) return c->fail(P2_ERR_INVALID_ARG, "16 x 16 meson block missing from the plan");
      ProfScope ps(c, "meson_gamma");
      P2_TRY(c, p2::launch_meson_gamma(mg, c->stream), "meson Gamma sums");
    }
  }
  return P2_OK;
}

void precision_release(p2_ctx* c) {
  for (DevBuf* b : {&c->phaseA, &c->expb, &c->cmaxb, &c->momrow, &c->kexp, &c->fpart, &c->rowtab, &c->errflag})
    b->release();
  c->split_moms_key.clear();
  c->split_what_key = 0;
}

}  // namespace p2

extern "C" p2_status p2_debug_wait_timeout(p2_ctx* c) {
  if (!c) return P2_ERR_INVALID_ARG;
  if (c->host_only) return c->fail(P2_ERR_UNSUPPORTED, "host-only context");
  c->wait_test = 1;
  return P2_OK;
}
