// C ABI (include/plegma2pt.h): argument checks, workspaces, phase tables and
// the launch sequence of the hot path.  Every failure is returned as a
// p2_status with a message in the context; nothing here exits.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <emmintrin.h>
#include <omp.h>

#include "../../include/plegma2pt.h"
#include "kernels.cuh"
#include "ctx.h"
#include "synth_host.h"

using namespace p2host;

namespace p2host {

int components_of(unsigned what) {
  int k = 0;
  for (const auto& b : kBlocks)
    if (what & b.bit) k += b.groups * b.datasets * b.comps;
  return k;
}

p2::CompOffsets offsets_of(unsigned what) {
  p2::CompOffsets o{-1, -1, -1, -1, -1, -1, -1, -1, -1, -1};
  int k = 0;
  int* slot[] = {&o.nuc, &o.ntor, &o.rton, &o.rtor, &o.diso12, &o.diso32, &o.g16, &o.all34, &o.new10, &o.diag10};
  static_assert(sizeof(slot) / sizeof(slot[0]) == sizeof(kBlocks) / sizeof(kBlocks[0]), "one offset per block");
  for (int i = 0; i < 10; i++)
    if (what & kBlocks[i].bit) {
      *slot[i] = k;
      k += kBlocks[i].groups * kBlocks[i].datasets * kBlocks[i].comps;
    }
  return o;
}

std::vector<int> createMom(int q2max) {
  std::vector<int> m;
  for (int iq = 0; iq <= q2max; iq++)
    for (int nx = iq; nx >= -iq; nx--)
      for (int ny = iq; ny >= -iq; ny--)
        for (int nz = iq; nz >= -iq; nz--)
          if (nx * nx + ny * ny + nz * nz == iq) {
            m.push_back(nx);
            m.push_back(ny);
            m.push_back(nz);
          }
  return m;
}

// Per-dimension phase tables [3][nmom][Lmax] complex double:
// exp(sign * i * 2 pi * n_d * x_d / L_d) for the global coordinates x_d of
// the local sites (origin 0; the source's phase is applied per slice after
// the site sum).
std::vector<double> phase_tables(const p2_ctx* c, const int* moms, int nmom, int sign, int Lmax) {
  std::vector<double> t((size_t)3 * nmom * Lmax * 2, 0.0);
  for (int d = 0; d < 3; d++)
    for (int p = 0; p < nmom; p++)
      for (int xl = 0; xl < c->Ll[d]; xl++) {
        const long long xg = (long long)xl + (long long)c->g.coords[d] * c->Ll[d];
        // reduce n*x mod L exactly in integers before the division
        long long num = ((long long)moms[3 * p + d] * xg) % c->g.L[d];
        if (num < 0) num += c->g.L[d];
        const double ph = 2.0 * M_PI * (double)num / (double)c->g.L[d];
        const size_t i = ((size_t)(d * nmom + p) * Lmax + xl) * 2;
        t[i] = std::cos(ph);
        t[i + 1] = sign * std::sin(ph);
      }
  return t;
}

p2_status upload_async(p2_ctx* c, DevBuf& b, const void* src, size_t bytes, const char* what) {
  P2_TRY(c, b.ensure(std::max<size_t>(bytes, 16)), what);
  P2_TRY(c, cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, c->stream), what);
  return P2_OK;
}

}  // namespace p2host

namespace {

p2_status check_prop(p2_ctx* c, const p2_prop& p, const char* name) {
  if (!p.data) return c->fail(P2_ERR_INVALID_ARG, std::string(name) + ": null data");
  if (p.nt < 1 || p.nt > c->T) return c->fail(P2_ERR_INVALID_ARG, std::string(name) + ": nt out of range");
  if (p.t_first < 0 || p.t_first >= c->T)
    return c->fail(P2_ERR_INVALID_ARG, std::string(name) + ": t_first out of range");
  if (p.precision != P2_FP64 && p.precision != P2_FP32)
    return c->fail(P2_ERR_INVALID_ARG, std::string(name) + ": bad precision");
  if (p.location != P2_DEVICE && p.location != P2_HOST)
    return c->fail(P2_ERR_INVALID_ARG, std::string(name) + ": bad location");
  if (p.transform & ~0xFu) return c->fail(P2_ERR_INVALID_ARG, std::string(name) + ": unknown transform bits");
  if ((p.transform & P2_PROP_ROTATE_PLUS) && (p.transform & P2_PROP_ROTATE_MINUS))
    return c->fail(P2_ERR_INVALID_ARG, std::string(name) + ": both rotation signs");
  return P2_OK;
}

}  // namespace

namespace p2host {

Work make_work(const p2_ctx* c, const p2_prop* props, const p2_request* reqs, const int* idx, int nidx, int tc) {
  Work w;
  const int T = c->T;
  const int tl0 = c->g.coords[3] * c->Ll[3];
  for (int q = 0; q < nidx; q++) {
    const int ri = idx ? idx[q] : q;
    const p2_request& r = reqs[ri];
    const p2_prop& u = props[r.prop_u];
    const p2_prop& d = props[r.prop_d];
    for (int tau = 0; tau < r.totalT; tau++) {
      const int t = (r.source[3] + tau) % T;
      if (t < tl0 || t >= tl0 + c->Ll[3]) continue;  // another rank's time slab
      const int ju = ((t - u.t_first) % T + T) % T, jd = ((t - d.t_first) % T + T) % T;
      if (ju >= u.nt || jd >= d.nt) continue;  // not stored in the views
      w.sl.push_back({ri, tau, ju, jd});
    }
  }
  const int n = (int)w.sl.size();
  tc = std::max(1, tc);
  // equal chunks: ceil(n / tc) of them, sizes differing by at most one
  const int nch = (n + tc - 1) / tc;
  for (int i = 0, s0 = 0; i < nch; i++) {
    const int len = n / nch + (i < n % nch ? 1 : 0);
    w.chunks.push_back({s0, len});
    w.max_n = std::max(w.max_n, len);
    s0 += len;
  }
  return w;
}

Stager::Stager(p2_ctx* ctx, const p2_prop* pp, const p2_request* rr, const Work& work)
    : c(ctx), props(pp), reqs(rr), w(work) {
  for (const SliceRef& s : w.sl) {
    const p2_request& r = reqs[s.req];
    host |= props[r.prop_u].location == P2_HOST || props[r.prop_d].location == P2_HOST;
  }
}

namespace {
size_t esz_of(const p2_prop& p) { return p.precision == P2_FP64 ? 16 : 8; }

// Binary exponent e with max |Re|, |Im| < 2^e over component row 0 of slice j
// of an FP64 host view (0 for an all-zero row): the host conversion stores the
// slice times 2^-e, so its entries stay far inside FP32's range.
int host_slice_exponent(const p2_prop& p, int j, long long V3) {
  const double* row = (const double*)p.data + (size_t)j * V3 * 2;
  double m = 0.0;
  for (long long i = 0; i < 2 * V3; i++) m = std::max(m, std::fabs(row[i]));
  int e = 0;
  if (m > 0.0) std::frexp(m, &e);
  return e;
}

// dst[i] = (float)(src[i] * scale) for n doubles; scale a power of two, so
// the product is exact and the rounding is that of the plain conversion.
// Streaming stores when dst is 16-byte aligned (the pinned staging is read
// next by the copy engine, not by this core).
void convert_row(const double* src, float* dst, size_t n, double scale) {
  size_t i = 0;
  if (((uintptr_t)dst & 15) == 0) {
    const __m128d sc = _mm_set1_pd(scale);
    for (; i + 4 <= n; i += 4) {
      const __m128 lo = _mm_cvtpd_ps(_mm_mul_pd(_mm_loadu_pd(src + i), sc));
      const __m128 hi = _mm_cvtpd_ps(_mm_mul_pd(_mm_loadu_pd(src + i + 2), sc));
      _mm_stream_ps(dst + i, _mm_movelh_ps(lo, hi));
    }
  }
  for (; i < n; i++) dst[i] = (float)(src[i] * scale);
}
}  // namespace

// PropXf code of a view's load-time transform on global time t.
int prop_xf_code(const p2_prop& p, int t) {
  int code = 0;
  if (p.transform & P2_PROP_ROTATE_PLUS) code |= p2::PropXf::kRotPlus;
  if (p.transform & P2_PROP_ROTATE_MINUS) code |= p2::PropXf::kRotMinus;
  if (p.transform & P2_PROP_GAMMA5) code |= p2::PropXf::kGamma5;
  if ((p.transform & P2_PROP_BOUNDARY) && t < p.boundary_t0) code |= p2::PropXf::kNegate;
  return code;
}

namespace {
}  // namespace

p2_status Stager::prepare(double* const* outs) {
  if (w.sl.empty()) return P2_OK;
  size_t esz_max[2] = {0, 0};
  for (const SliceRef& s : w.sl) {
    const p2_request& r = reqs[s.req];
    for (int f = 0; f < 2; f++) {
      const p2_prop& p = props[f ? r.prop_d : r.prop_u];
      if (p.location == P2_HOST) esz_max[f] = std::max(esz_max[f], esz_of(p));
    }
  }
  if (host) {
    if (c->capturing) return c->fail(P2_ERR_UNSUPPORTED, "graphs need device-resident propagators");
    for (int slot = 0; slot < 2; slot++)
      for (int f = 0; f < 2; f++)
        if (esz_max[f])
          P2_TRY(c, (f ? c->stage_d2[slot] : c->stage_u2[slot]).ensure((size_t)144 * w.max_n * c->V3 * esz_max[f]),
                 "staging alloc");
    if (cvt32)
      for (int hs = 0; hs < p2_ctx::kHostSlots; hs++) {
        for (int f = 0; f < 2; f++)
          P2_TRY(c, (f ? c->hstage_d[hs] : c->hstage_u[hs]).ensure((size_t)144 * w.max_n * c->V3 * 8),
                 "pinned conversion buffer");
        if (!c->hcopied[hs])
          P2_TRY(c, cudaEventCreateWithFlags(&c->hcopied[hs], cudaEventDisableTiming), "conversion events");
      }
    if (!c->copy_stream) {
      P2_TRY(c, cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking), "copy stream");
      for (int i = 0; i < 2; i++) {
        P2_TRY(c, cudaEventCreateWithFlags(&c->copied[i], cudaEventDisableTiming), "copy events");
        P2_TRY(c, cudaEventCreateWithFlags(&c->consumed[i], cudaEventDisableTiming), "copy events");
      }
    }
    for (int i = 0; i < 2; i++) P2_TRY(c, cudaEventRecord(c->consumed[i], c->stream), "copy events");
  }
  // descriptors of every slice, in chunk order
  const size_t bytes = w.sl.size() * sizeof(p2::SliceDesc);
  if (!c->sdesc_copied)
    P2_TRY(c, cudaEventCreateWithFlags(&c->sdesc_copied, cudaEventDisableTiming), "descriptor event");
  else if (!c->capturing)
    P2_TRY(c, cudaEventSynchronize(c->sdesc_copied), "descriptor mirror");
  if (c->sdesc_host_n < bytes) {
    if (c->sdesc_host) cudaFreeHost(c->sdesc_host);
    c->sdesc_host = nullptr;
    c->sdesc_host_n = 0;
    P2_TRY(c, cudaMallocHost(&c->sdesc_host, bytes), "descriptor mirror");
    c->sdesc_host_n = bytes;
  }
  p2::SliceDesc* h = (p2::SliceDesc*)c->sdesc_host;
  for (size_t ci = 0; ci < w.chunks.size(); ci++) {
    const Chunk& ch = w.chunks[ci];
    const int slot = (int)(ci & 1);
    for (int i = 0; i < ch.n; i++) {
      const SliceRef& s = w.sl[ch.s0 + i];
      const p2_request& r = reqs[s.req];
      p2::SliceDesc& sd = h[ch.s0 + i];
      std::memset(&sd, 0, sizeof(sd));
      for (int f = 0; f < 2; f++) {
        const p2_prop& p = props[f ? r.prop_d : r.prop_u];
        const void* ptr = p.data;
        long long vol = c->V3 * p.nt, off = (long long)(f ? s.jd : s.ju) * c->V3;
        if (p.location == P2_HOST) {
          ptr = (f ? c->stage_d2[slot] : c->stage_u2[slot]).p;
          vol = c->V3 * ch.n;
          off = (long long)i * c->V3;
        }
        (f ? sd.d : sd.u) = ptr;
        (f ? sd.vol_d : sd.vol_u) = vol;
        (f ? sd.off_d : sd.off_u) = off;
      }
      sd.out = outs[s.req];
      sd.tau = s.tau;
      sd.totalT = r.totalT;
      for (int d = 0; d < 3; d++) sd.x0[d] = r.source[d];
      const int t = (r.source[3] + s.tau) % c->T;
      sd.xf[0] = prop_xf_code(props[r.prop_u], t);
      sd.xf[1] = prop_xf_code(props[r.prop_d], t);
    }
  }
  if (cvt32) {
    std::vector<int> conv;  // slices of the chunks converted on the host
    for (size_t ci = 0; ci < w.chunks.size(); ci++)
      if (converts((int)ci))
        for (int i = 0; i < w.chunks[ci].n; i++) conv.push_back(w.chunks[ci].s0 + i);
    const long long n = (long long)conv.size();
#pragma omp parallel for schedule(dynamic, 1)
    for (long long q = 0; q < 2 * n; q++) {
      const int si = conv[q >> 1];
      const SliceRef& s = w.sl[si];
      const int f = (int)(q & 1);
      const p2_request& r = reqs[s.req];
      h[si].eh[f] = host_slice_exponent(props[f ? r.prop_d : r.prop_u], f ? s.jd : s.ju, c->V3);
    }
  }
  P2_TRY(c, c->sdesc.ensure(bytes), "descriptor alloc");
  P2_TRY(c, cudaMemcpyAsync(c->sdesc.p, h, bytes, cudaMemcpyHostToDevice, c->stream), "descriptor upload");
  if (!c->capturing) P2_TRY(c, cudaEventRecord(c->sdesc_copied, c->stream), "descriptor event");
  dsl = (p2::SliceDesc*)c->sdesc.p;
  return P2_OK;
}

p2_status Stager::issue(int ci) {
  if (!host || ci >= (int)w.chunks.size()) return P2_OK;
  const int slot = ci & 1;
  const Chunk& ch = w.chunks[ci];
  P2_TRY(c, cudaStreamWaitEvent(c->copy_stream, c->consumed[slot], 0), "copy wait");
  if (converts(ci)) {
    // the previous upload from this pinned slot has finished; convert the
    // chunk into it (all host threads) and upload each flavour in one copy
    const int hs = host_slot(ci);
    P2_TRY(c, cudaEventSynchronize(c->hcopied[hs]), "conversion buffer reuse");
    const p2::SliceDesc* h = (const p2::SliceDesc*)c->sdesc_host + ch.s0;
    const long long V3 = c->V3;
    const long long rows = 2LL * 144 * ch.n;
#pragma omp parallel
    {
#pragma omp for schedule(static)
      for (long long q = 0; q < rows; q++) {
        const int f = (int)(q / (144LL * ch.n));
        const int comp = (int)((q / ch.n) % 144), i = (int)(q % ch.n);
        const SliceRef& s = w.sl[ch.s0 + i];
        const p2_request& r = reqs[s.req];
        const p2_prop& p = props[f ? r.prop_d : r.prop_u];
        const double* src = (const double*)p.data + ((size_t)comp * p.nt + (f ? s.jd : s.ju)) * V3 * 2;
        float* dst = (float*)(f ? c->hstage_d[hs] : c->hstage_u[hs]).p + ((size_t)comp * ch.n + i) * V3 * 2;
        convert_row(src, dst, (size_t)V3 * 2, std::ldexp(1.0, -h[i].eh[f]));
      }
      _mm_sfence();
    }
    ProfScope ps(c, "h2d_upload", c->copy_stream);
    for (int f = 0; f < 2; f++)
      P2_TRY(c,
             cudaMemcpyAsync((f ? c->stage_d2[slot] : c->stage_u2[slot]).p,
                             (f ? c->hstage_d[hs] : c->hstage_u[hs]).p, (size_t)144 * ch.n * V3 * 8,
                             cudaMemcpyHostToDevice, c->copy_stream),
             "host propagator upload");
    P2_TRY(c, cudaEventRecord(c->hcopied[hs], c->copy_stream), "copy event");
    P2_TRY(c, cudaEventRecord(c->copied[slot], c->copy_stream), "copy event");
    return P2_OK;
  }
  ProfScope ps(c, "h2d_upload", c->copy_stream);
  for (int f = 0; f < 2; f++) {
    // runs of slices that are consecutive in one host view: one contiguous
    // copy per component row and run (a strided 2-D copy of this shape runs
    // at a third of the link's bandwidth)
    int i = 0;
    while (i < ch.n) {
      const SliceRef& s = w.sl[ch.s0 + i];
      const p2_request& r = reqs[s.req];
      const int pi = f ? r.prop_d : r.prop_u;
      const p2_prop& p = props[pi];
      const int j0 = f ? s.jd : s.ju;
      int len = 1;
      while (i + len < ch.n) {
        const SliceRef& s2 = w.sl[ch.s0 + i + len];
        const p2_request& r2 = reqs[s2.req];
        if ((f ? r2.prop_d : r2.prop_u) != pi || (f ? s2.jd : s2.ju) != j0 + len) break;
        len++;
      }
      if (p.location == P2_HOST) {
        const size_t esz = esz_of(p);
        char* dst = (char*)(f ? c->stage_d2[slot] : c->stage_u2[slot]).p + (size_t)i * c->V3 * esz;
        const char* src = (const char*)p.data + (size_t)j0 * c->V3 * esz;
        const size_t width = (size_t)len * c->V3 * esz;
        const size_t spitch = (size_t)p.nt * c->V3 * esz, dpitch = (size_t)ch.n * c->V3 * esz;
        for (int comp = 0; comp < 144; comp++)
          P2_TRY(c,
                 cudaMemcpyAsync(dst + comp * dpitch, src + comp * spitch, width, cudaMemcpyHostToDevice,
                                 c->copy_stream),
                 "host propagator upload");
      }
      i += len;
    }
  }
  P2_TRY(c, cudaEventRecord(c->copied[slot], c->copy_stream), "copy event");
  return P2_OK;
}

p2_status Stager::wait(int ci) {
  if (host) P2_TRY(c, cudaStreamWaitEvent(c->stream, c->copied[ci & 1], 0), "compute wait");
  return P2_OK;
}

p2_status Stager::release(int ci) {
  if (host) P2_TRY(c, cudaEventRecord(c->consumed[ci & 1], c->stream), "consume event");
  return P2_OK;
}

p2_status make_plan(p2_ctx* c, const p2_request& r, Plan& pl) {
  if (r.contractions == 0 || (r.contractions & ~kAllBits))
    return c->fail(P2_ERR_INVALID_ARG, "contractions: empty or unknown bits");
  if (r.totalT < 1 || r.totalT > c->T) return c->fail(P2_ERR_INVALID_ARG, "totalT out of range");
  for (int d = 0; d < 4; d++)
    if (r.source[d] < 0 || r.source[d] >= c->g.L[d]) return c->fail(P2_ERR_INVALID_ARG, "source outside the lattice");
  if (r.moms) {
    if (r.nmom < 1) return c->fail(P2_ERR_INVALID_ARG, "nmom < 1 with an explicit momentum list");
    pl.moms.assign(r.moms, r.moms + 3 * r.nmom);
  } else {
    if (r.q2max < 0) return c->fail(P2_ERR_INVALID_ARG, "q2max < 0");
    pl.moms = createMom(r.q2max);
  }
  pl.nmom = (int)pl.moms.size() / 3;
  pl.K = components_of(r.contractions);
  pl.Lmax = std::max(c->Ll[0], std::max(c->Ll[1], c->Ll[2]));
  pl.totalT = r.totalT;
  pl.blocks.clear();
  int k = 0;
  for (const auto& b : kBlocks)
    if (r.contractions & b.bit) {
      p2::ScatterBlock sb;
      sb.k0 = k;
      sb.groups = b.groups;
      sb.datasets = b.datasets;
      sb.comps = b.comps;
      sb.base = k;  // the blocks before this one hold k components per (time, momentum)
      pl.blocks.push_back(sb);
      k += b.groups * b.datasets * b.comps;
    }
  pl.total = (size_t)k * r.totalT * pl.nmom;
  return P2_OK;
}

}  // namespace p2host

namespace {

int chunk_slices(p2_ctx* c, int K) {
  const size_t per = (size_t)K * c->V3 * 16;
  size_t n = c->ws_budget / std::max<size_t>(per, 1);
  return (int)std::max<size_t>(1, std::min<size_t>(n, (size_t)c->T));
}

// Plain FP64 form for requests reqs[idx[..]] that share contractions and
// momenta: FP64 site contraction, FP64 projection, deterministic reduction.
p2_status run_plain(p2_ctx* c, const p2_prop* props, const p2_request* reqs, const int* idx, int nidx,
                    const Plan& pl, double* const* outs) {
  for (int q = 0; q < nidx; q++) {
    const p2_request& r = reqs[idx[q]];
    if (props[r.prop_u].precision != P2_FP64 || props[r.prop_d].precision != P2_FP64)
      return c->fail(P2_ERR_UNSUPPORTED, "the plain FP64 form needs FP64 propagators");
  }
  const unsigned what = reqs[idx[0]].contractions;
  p2_status st;
  if (c->plain_moms_key != pl.moms) {  // phase tables have origin 0: one set per momentum list
    c->plain_moms_key.clear();
    std::vector<double> tabh = phase_tables(c, pl.moms.data(), pl.nmom, -1, pl.Lmax);
    if ((st = upload_async(c, c->ptab, tabh.data(), tabh.size() * sizeof(double), "phase table")) != P2_OK) return st;
    if ((st = upload_async(c, c->moms, pl.moms.data(), pl.moms.size() * sizeof(int), "momenta")) != P2_OK) return st;
    c->plain_moms_key = pl.moms;
  }

  const int tc = chunk_slices(c, pl.K);
  const Work w = make_work(c, props, reqs, idx, nidx, tc);
  if (w.sl.empty()) return P2_OK;
  P2_TRY(c, c->cbuf.ensure((size_t)w.max_n * pl.K * c->V3 * 16), "position buffer alloc");
  Stager sg(c, props, reqs, w);
  if ((st = sg.prepare(outs)) != P2_OK) return st;

  const int ptiles = (pl.nmom + 63) / 64;
  for (int i = 0; i < 2; i++)
    if ((st = sg.issue(i)) != P2_OK) return st;
  for (size_t ci = 0; ci < w.chunks.size(); ci++) {
    const int n = w.chunks[ci].n;
    if ((st = sg.wait((int)ci)) != P2_OK) return st;
    p2::ContractArgs a{};
    a.sl = sg.desc((int)ci);
    a.V3 = (int)c->V3;
    a.ntau = n;
    a.what = what;
    a.K = pl.K;
    a.k = offsets_of(what);
    a.out = c->cbuf.p;
    a.g16_raw = p2::g16_raw(what) ? 1 : 0;  // the projection is followed by k_meson_gamma
    {
      ProfScope ps(c, "contract_plain_fp64");
      P2_TRY(c, p2::launch_contract_plain(a, c->nsm, c->stream), "contract kernel");
    }
    if ((st = sg.release((int)ci)) != P2_OK) return st;
    if ((st = sg.issue((int)ci + 2)) != P2_OK) return st;

    p2::ProjArgs pa{};
    pa.c = c->cbuf.p;
    pa.sT = (long long)pl.K * c->V3;
    pa.sK = c->V3;
    pa.ntau = n;
    pa.K = pl.K;
    pa.V3 = (int)c->V3;
    pa.nmom = pl.nmom;
    pa.Lx = c->Ll[0];
    pa.Ly = c->Ll[1];
    pa.Lz = c->Ll[2];
    pa.Lmax = pl.Lmax;
    pa.tab = (const double*)c->ptab.p;
    // candidates (component tile, site splits): the least-waste tile at ~2
    // waves first, then other tiles at 1, 2 and 4 waves
    std::vector<std::vector<int>> cands;
    const int tk0 = p2::project_fp64_tk(pl.K, 0);
    for (int tk : {tk0, 8, 6, 4, 2})
      for (int waves : {2, 1, 4}) {
        const int ktiles = (pl.K + 16 * tk - 1) / (16 * tk);
        int nsplit = (waves * c->nsm + ptiles * ktiles * n - 1) / (ptiles * ktiles * n);
        nsplit = std::max(1, std::min(nsplit, (int)((c->V3 + 255) / 256)));
        const int chunk = (int)((((c->V3 + nsplit - 1) / nsplit) + 15) / 16 * 16);
        std::vector<int> v{tk, (int)((c->V3 + chunk - 1) / chunk), chunk};
        if (std::find(cands.begin(), cands.end(), v) == cands.end()) cands.push_back(v);
      }
    int maxsplit = 0;
    for (const auto& v : cands) maxsplit = std::max(maxsplit, v[1]);
    P2_TRY(c, c->part.ensure((size_t)w.max_n * maxsplit * pl.nmom * pl.K * 16), "partials alloc");
    pa.part = (double*)c->part.p;
    char key[160];
    std::snprintf(key, sizeof(key), "project_fp64 V3=%lld K=%d nmom=%d n=%d", c->V3, pl.K, pl.nmom, n);
    std::vector<int> pick;
    P2_TRY(c,
           tune_choose(c->tuner.get(), key, cands, c->stream, !c->capturing,
                       [&](const std::vector<int>& v) {
                         p2::ProjArgs q = pa;
                         q.tk = v[0];
                         q.nsplit = v[1];
                         q.chunk = v[2];
                         return p2::launch_project_fp64(q, c->stream);
                       },
                       pick),
           "projection tuning");
    pa.tk = pick[0];
    pa.nsplit = pick[1];
    pa.chunk = pick[2];
    {
      ProfScope ps(c, "project_fp64");
      P2_TRY(c, p2::launch_project_fp64(pa, c->stream), "projection kernel");
    }
    p2::ScatterArgs sa{};
    sa.part = (const double*)c->part.p;
    sa.ntau = n;
    sa.nsplit = pa.nsplit;
    sa.nmom = pl.nmom;
    sa.K = pl.K;
    if (pl.blocks.size() > (size_t)p2::kMaxBlocks) return c->fail(P2_ERR_INVALID_ARG, "too many result blocks");
    sa.nblocks = (int)pl.blocks.size();
    for (size_t b = 0; b < pl.blocks.size(); b++) sa.blk[b] = pl.blocks[b];
    sa.sl = sg.desc((int)ci);
    sa.moms = (const int*)c->moms.p;
    for (int d = 0; d < 3; d++) sa.L[d] = c->g.L[d];
    {
      ProfScope ps(c, "reduce_scatter");
      P2_TRY(c, p2::launch_scatter(sa, c->stream), "reduction kernel");
    }
    if (p2::g16_raw(what)) {
      // the Gamma sums of the 16 x 16 block on its projected colour products
      p2::MesonGammaArgs mg{};
      mg.sl = sg.desc((int)ci);
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

}  // namespace

cudaEvent_t p2_ctx::prof_begin(const char* name, int& slot, cudaStream_t on) {
  slot = -1;
  for (size_t i = 0; i < prof.size(); i++)
    if (prof[i].name == name) slot = (int)i;
  if (slot < 0) {
    prof.emplace_back();
    prof.back().name = name;
    slot = (int)prof.size() - 1;
  }
  cudaEvent_t e = nullptr;
  Prof& p = prof[slot];
  if (!p.pool.empty()) {
    e = p.pool.back();
    p.pool.pop_back();
  } else if (cudaEventCreate(&e) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  cudaEventRecord(e, on ? on : stream);
  return e;
}

void p2_ctx::prof_end(int slot, cudaEvent_t start, cudaStream_t on) {
  cudaEvent_t e = nullptr;
  Prof& p = prof[slot];
  if (!p.pool.empty()) {
    e = p.pool.back();
    p.pool.pop_back();
  } else if (cudaEventCreate(&e) != cudaSuccess) {
    cudaGetLastError();
    p.pool.push_back(start);
    return;
  }
  cudaEventRecord(e, on ? on : stream);
  p.pending.emplace_back(start, e);
}

void p2_ctx::prof_collect() {
  for (Prof& p : prof) {
    for (auto& ev : p.pending) {
      cudaEventSynchronize(ev.second);
      float ms = 0;
      if (cudaEventElapsedTime(&ms, ev.first, ev.second) == cudaSuccess) {
        p.ms += ms;
        p.launches++;
      }
      cudaGetLastError();
      p.pool.push_back(ev.first);
      p.pool.push_back(ev.second);
    }
    p.pending.clear();
  }
}

void p2_ctx::prof_clear() {
  prof_collect();
  for (Prof& p : prof) {
    p.ms = 0;
    p.launches = 0;
  }
}

extern "C" {

p2_status p2_profile_enable(p2_ctx* c, int on) {
  if (!c) return P2_ERR_INVALID_ARG;
  c->profiling = on != 0;
  return P2_OK;
}

int p2_profile_read(p2_ctx* c, p2_kernel_time* out, int max, int reset) {
  if (!c) return -1;
  c->prof_collect();
  int n = 0;
  for (const auto& p : c->prof) {
    if (out && n < max) {
      std::snprintf(out[n].name, sizeof(out[n].name), "%s", p.name.c_str());
      out[n].launches = p.launches;
      out[n].ms = p.ms;
    }
    n++;
  }
  if (reset) c->prof_clear();
  return n;
}

p2_status p2_ctx_create(const p2_geom* g, p2_ctx** out) {
  if (!g || !out) return P2_ERR_INVALID_ARG;
  *out = nullptr;
  for (int d = 0; d < 4; d++) {
    if (g->L[d] < 1 || g->procs[d] < 1 || g->L[d] % g->procs[d] != 0) return P2_ERR_INVALID_ARG;
    if (g->coords[d] < 0 || g->coords[d] >= g->procs[d]) return P2_ERR_INVALID_ARG;
  }
  p2_ctx* c = new p2_ctx();
  c->g = *g;
  for (int d = 0; d < 4; d++) c->Ll[d] = g->L[d] / g->procs[d];
  c->V3 = (long long)c->Ll[0] * c->Ll[1] * c->Ll[2];
  c->T = g->L[3];
  if (g->device < 0) {  // host-only context: argument checks and host helpers, no device work
    c->host_only = true;
    *out = c;
    return P2_OK;
  }
  if (cudaSetDevice(g->device) != cudaSuccess) {
    cudaGetLastError();
    delete c;
    return P2_ERR_CUDA;
  }
  int nsm = 0;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, g->device) == cudaSuccess && nsm > 0) c->nsm = nsm;
  cudaDeviceGetAttribute(&c->project_split_smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, g->device);
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    delete c;
    return P2_ERR_CUDA;
  }
  c->own_stream = true;
  size_t fr = 0, tot = 0;
  cudaMemGetInfo(&fr, &tot);
  c->ws_budget = std::min<size_t>((size_t)8 << 30, fr / 4);
  if (c->ws_budget < ((size_t)64 << 20)) c->ws_budget = (size_t)64 << 20;
  *out = c;
  return P2_OK;
}

p2_status p2_ctx_destroy(p2_ctx* c) {
  if (!c) return P2_ERR_INVALID_ARG;
  if (c->host_only) {
    delete c;
    return P2_OK;
  }
  cudaStreamSynchronize(c->stream);
  for (DevBuf* b : {&c->cbuf, &c->part, &c->tab, &c->res, &c->moms, &c->sdesc, &c->ptab, &c->ft_kexp}) b->release();
  if (c->sdesc_host) cudaFreeHost(c->sdesc_host);
  if (c->sdesc_copied) cudaEventDestroy(c->sdesc_copied);
  for (int i = 0; i < 2; i++) {
    c->stage_u2[i].release();
    c->stage_d2[i].release();
    if (c->copied[i]) cudaEventDestroy(c->copied[i]);
    if (c->consumed[i]) cudaEventDestroy(c->consumed[i]);
  }
  for (int i = 0; i < p2_ctx::kHostSlots; i++) {
    c->hstage_u[i].release();
    c->hstage_d[i].release();
    if (c->hcopied[i]) cudaEventDestroy(c->hcopied[i]);
  }
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  c->prof_collect();
  for (auto& p : c->prof)
    for (cudaEvent_t e : p.pool) cudaEventDestroy(e);
  if (c->own_stream) cudaStreamDestroy(c->stream);
  p2::precision_release(c);
  p2_udsc_release(c);
  delete c;
  return P2_OK;
}

const char* p2_last_error(const p2_ctx* c) { return c ? c->err.c_str() : "null context"; }

p2_status p2_sync(p2_ctx* c) {
  if (!c) return P2_ERR_INVALID_ARG;
  if (c->host_only) return c->fail(P2_ERR_UNSUPPORTED, "host-only context");
  P2_TRY(c, cudaStreamSynchronize(c->stream), "p2_sync");
  if (c->errflag.p) {
    int e = 0;
    P2_TRY(c, cudaMemcpy(&e, c->errflag.p, sizeof(int), cudaMemcpyDeviceToHost), "error flag read");
    if (e) {
      cudaMemset(c->errflag.p, 0, sizeof(int));
      return c->fail(P2_ERR_DEVICE_TIMEOUT, "a tensor-core pipeline wait gave up; results of the call are invalid");
    }
  }
  return P2_OK;
}

p2_status p2_set_stream(p2_ctx* c, void* s) {
  if (!c) return P2_ERR_INVALID_ARG;
  if (c->host_only) return c->fail(P2_ERR_UNSUPPORTED, "host-only context");
  if (c->own_stream) {
    cudaStreamSynchronize(c->stream);
    cudaStreamDestroy(c->stream);
    c->own_stream = false;
  }
  if (s) {
    c->stream = (cudaStream_t)s;
  } else {
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
      return c->fail(P2_ERR_CUDA, "stream create");
    c->own_stream = true;
  }
  return P2_OK;
}

p2_status p2_set_workspace(p2_ctx* c, size_t bytes) {
  if (!c) return P2_ERR_INVALID_ARG;
  if (bytes == 0) return c->fail(P2_ERR_INVALID_ARG, "p2_set_workspace: zero bytes");
  c->ws_budget = bytes;
  return P2_OK;
}

int p2_components(unsigned what) { return (what & ~kAllBits) ? -1 : components_of(what); }

int p2_mom_list(int q2max, int* moms) {
  if (q2max < 0) return -1;
  std::vector<int> m = createMom(q2max);
  if (moms) std::memcpy(moms, m.data(), m.size() * sizeof(int));
  return (int)m.size() / 3;
}

int p2_block_info(unsigned what, int totalT, int nmom, p2_block* blocks, int max_blocks, size_t* total) {
  if (what & ~kAllBits) return -1;
  int n = 0;
  size_t off = 0;
  for (const auto& b : kBlocks)
    if (what & b.bit) {
      if (blocks && n < max_blocks) {
        blocks[n].bit = b.bit;
        blocks[n].groups = b.groups;
        blocks[n].datasets = b.datasets;
        blocks[n].comps = b.comps;
        blocks[n].offset = off;
      }
      n++;
      off += (size_t)b.groups * b.datasets * b.comps * totalT * nmom;
    }
  if (total) *total = off;
  return n;
}

p2_status p2_contract_project(p2_ctx* c, const p2_prop* props, int nprops, const p2_request* reqs, int nreq) {
  if (!c) return P2_ERR_INVALID_ARG;
  if (!props || nprops < 1 || !reqs || nreq < 1) return c->fail(P2_ERR_INVALID_ARG, "empty props or requests");
  for (int i = 0; i < nprops; i++) {
    p2_status s = check_prop(c, props[i], "prop");
    if (s != P2_OK) return s;
  }
  std::vector<Plan> plans(nreq);
  for (int i = 0; i < nreq; i++) {
    const p2_request& r = reqs[i];
    if (r.prop_u < 0 || r.prop_u >= nprops || r.prop_d < 0 || r.prop_d >= nprops)
      return c->fail(P2_ERR_INVALID_ARG, "prop index out of range");
    if (!r.out) return c->fail(P2_ERR_INVALID_ARG, "null output");
    if (r.mode != P2_PLAIN_FP64 && r.mode != P2_SPLIT_FP16) return c->fail(P2_ERR_INVALID_ARG, "bad mode");
    if (r.out_location != P2_DEVICE && r.out_location != P2_HOST)
      return c->fail(P2_ERR_INVALID_ARG, "bad out_location");
    p2_status s = make_plan(c, r, plans[i]);
    if (s != P2_OK) return s;
  }
  if (c->host_only) return c->fail(P2_ERR_UNSUPPORTED, "host-only context");
  if (c->capturing)
    for (int i = 0; i < nreq; i++)
      if (reqs[i].out_location != P2_DEVICE) return c->fail(P2_ERR_UNSUPPORTED, "graphs need device-resident results");

  // requests that share form, contractions, momenta and input precision run as
  // one batch: each kernel launches once per chunk of slices from all of them
  std::vector<char> done(nreq, 0);
  for (int i = 0; i < nreq; i++) {
    if (done[i]) continue;
    std::vector<int> idx;
    const p2_request& ri = reqs[i];
    for (int j = i; j < nreq; j++) {
      const p2_request& rj = reqs[j];
      if (done[j] || rj.mode != ri.mode || rj.contractions != ri.contractions || plans[j].moms != plans[i].moms ||
          props[rj.prop_u].precision != props[ri.prop_u].precision ||
          props[rj.prop_d].precision != props[ri.prop_d].precision)
        continue;
      done[j] = 1;
      idx.push_back(j);
    }
    // a recorded graph holds one batch: its slice descriptors and tables are
    // uploaded once, from buffers a second batch would overwrite
    if (c->capturing && (int)idx.size() != nreq)
      return c->fail(P2_ERR_UNSUPPORTED,
                     "a graph records one batch: requests must share form, contractions, momenta and precision");
    // device result of each request; host results go through one device buffer
    std::vector<double*> outs(nreq, nullptr);
    size_t host_total = 0;
    for (int j : idx)
      if (reqs[j].out_location == P2_HOST) host_total += plans[j].total;
    if (host_total) {
      P2_TRY(c, c->res.ensure(host_total * 16), "result alloc");
      P2_TRY(c, cudaMemsetAsync(c->res.p, 0, host_total * 16, c->stream), "result clear");
    }
    size_t off = 0;
    for (int j : idx) {
      if (reqs[j].out_location == P2_HOST) {
        outs[j] = (double*)c->res.p + 2 * off;
        off += plans[j].total;
      } else {
        outs[j] = reqs[j].out;
      }
    }
    p2_status s = ri.mode == P2_PLAIN_FP64
                      ? run_plain(c, props, reqs, idx.data(), (int)idx.size(), plans[i], outs.data())
                      : p2::precision_run_batch(c, props, reqs, idx.data(), (int)idx.size(), plans[i], outs.data());
    if (s != P2_OK) return s;
    if (host_total) {
      for (int j : idx)
        if (reqs[j].out_location == P2_HOST)
          P2_TRY(c,
                 cudaMemcpyAsync(reqs[j].out, outs[j], plans[j].total * 16, cudaMemcpyDeviceToHost, c->stream),
                 "result download");
      P2_TRY(c, cudaStreamSynchronize(c->stream), "result download");
    }
  }
  return P2_OK;
}

int p2_local_taus(p2_ctx* c, const p2_prop* props, int nprops, const p2_request* r, int* taus, int max) {
  if (!c || !props || !r || nprops < 1) return -1;
  if (r->prop_u < 0 || r->prop_u >= nprops || r->prop_d < 0 || r->prop_d >= nprops) return -1;
  for (int i = 0; i < nprops; i++)
    if (check_prop(c, props[i], "prop") != P2_OK) return -1;
  Plan pl;
  if (make_plan(c, *r, pl) != P2_OK) return -1;
  const int idx = 0;
  const Work w = make_work(c, props, r, &idx, 1, c->T);
  const int n = (int)w.sl.size();
  for (int i = 0; taus && i < n && i < max; i++) taus[i] = w.sl[i].tau;
  return n;
}

p2_status p2_contract_position(p2_ctx* c, const p2_prop* props, int nprops, const p2_request* r) {
  if (!c) return P2_ERR_INVALID_ARG;
  if (!props || !r || nprops < 1) return c->fail(P2_ERR_INVALID_ARG, "empty props or request");
  for (int i = 0; i < nprops; i++) {
    p2_status s = check_prop(c, props[i], "prop");
    if (s != P2_OK) return s;
  }
  if (r->prop_u < 0 || r->prop_u >= nprops || r->prop_d < 0 || r->prop_d >= nprops)
    return c->fail(P2_ERR_INVALID_ARG, "prop index out of range");
  if (!r->out) return c->fail(P2_ERR_INVALID_ARG, "null output");
  if (r->contractions == 0 || (r->contractions & ~kAllBits))
    return c->fail(P2_ERR_INVALID_ARG, "contractions: empty or unknown bits");
  if (r->totalT < 1 || r->totalT > c->T) return c->fail(P2_ERR_INVALID_ARG, "totalT out of range");
  if (r->out_location != P2_DEVICE && r->out_location != P2_HOST)
    return c->fail(P2_ERR_INVALID_ARG, "bad out_location");
  const p2_prop& u = props[r->prop_u];
  const p2_prop& d = props[r->prop_d];
  if (u.precision != P2_FP64 || d.precision != P2_FP64)
    return c->fail(P2_ERR_UNSUPPORTED, "position-space output needs FP64 propagators");
  if (c->host_only) return c->fail(P2_ERR_UNSUPPORTED, "host-only context");
  const int K = components_of(r->contractions);
  const size_t slice = (size_t)K * c->V3;  // complex elements of one time slice
  const Work w = make_work(c, props, r, nullptr, 1, chunk_slices(c, K));
  if (w.sl.empty()) return P2_OK;
  P2_TRY(c, c->cbuf.ensure((size_t)w.max_n * slice * 16), "position buffer alloc");
  Stager sg(c, props, r, w);
  double* outs[1] = {r->out};
  p2_status st;
  if ((st = sg.prepare(outs)) != P2_OK) return st;
  for (int i = 0; i < 2; i++)
    if ((st = sg.issue(i)) != P2_OK) return st;
  for (size_t ci = 0; ci < w.chunks.size(); ci++) {
    const Chunk& ch = w.chunks[ci];
    if ((st = sg.wait((int)ci)) != P2_OK) return st;
    // slices of consecutive times go straight into a device result
    bool direct = r->out_location == P2_DEVICE;
    for (int i = 1; i < ch.n && direct; i++) direct = w.sl[ch.s0 + i].tau == w.sl[ch.s0].tau + i;
    p2::ContractArgs a{};
    a.sl = sg.desc((int)ci);
    a.V3 = (int)c->V3;
    a.ntau = ch.n;
    a.what = r->contractions;
    a.K = K;
    a.k = offsets_of(r->contractions);
    a.out = direct ? (void*)(r->out + 2 * slice * w.sl[ch.s0].tau) : c->cbuf.p;
    {
      ProfScope ps(c, "contract_plain_fp64");
      P2_TRY(c, p2::launch_contract_plain(a, c->nsm, c->stream), "contract kernel");
    }
    if ((st = sg.release((int)ci)) != P2_OK) return st;
    if ((st = sg.issue((int)ci + 2)) != P2_OK) return st;
    if (!direct)
      for (int i = 0; i < ch.n; i++)
        P2_TRY(c,
               cudaMemcpyAsync(r->out + 2 * slice * w.sl[ch.s0 + i].tau, (const double*)c->cbuf.p + 2 * slice * i,
                               slice * 16, cudaMemcpyDefault, c->stream),
               "position copy");
  }
  if (r->out_location == P2_HOST) P2_TRY(c, cudaStreamSynchronize(c->stream), "position download");
  return P2_OK;
}

p2_status p2_ft_apply_split(p2_ctx* c, const double* field, int dof, int nt, const int* moms, int nmom, int sign,
                            double* out, int out_location) {
  if (!c) return P2_ERR_INVALID_ARG;
  if (!field || !out || dof < 1 || nt < 1 || nt > c->Ll[3] || !moms || nmom < 1)
    return c->fail(P2_ERR_INVALID_ARG, "p2_ft_apply_split: bad arguments");
  if (sign != 1 && sign != -1) return c->fail(P2_ERR_INVALID_ARG, "p2_ft_apply_split: sign must be +1 or -1");
  if (out_location != P2_DEVICE && out_location != P2_HOST) return c->fail(P2_ERR_INVALID_ARG, "bad out_location");
  if (c->host_only) return c->fail(P2_ERR_UNSUPPORTED, "host-only context");
  if (c->project_split_smem_max < p2::project_split_smem_bytes(p2::project_split_max_nt()))
    return c->fail(P2_ERR_UNSUPPORTED, "device shared memory per block too small for the tensor-core projection");
  // exp(+i p.x) = exp(-i (-p).x): the projection's rows carry exp(-i p.x)
  Plan pl;
  pl.nmom = nmom;
  pl.moms.assign(moms, moms + 3 * nmom);
  if (sign == 1)
    for (int& m : pl.moms) m = -m;
  pl.Lmax = std::max(c->Ll[0], std::max(c->Ll[1], c->Ll[2]));
  pl.K = dof;
  pl.totalT = nt;
  if (!c->errflag.p) {
    P2_TRY(c, c->errflag.ensure(16), "error flag alloc");
    P2_TRY(c, cudaMemsetAsync(c->errflag.p, 0, 16, c->stream), "error flag clear");
  }
  int nmtile = 0, nkstep = 0;
  p2_status st = p2::split_prepare_tables(c, pl, 0, nmtile, nkstep);
  if (st != P2_OK) return st;
  const size_t total = (size_t)nt * dof * nmom;
  double* dst = out;
  if (out_location == P2_HOST) {
    P2_TRY(c, c->res.ensure(total * 16), "result alloc");
    dst = (double*)c->res.p;
  }
  // every component carries the slice scale once
  if (c->ft_kexp_n < dof) {
    std::vector<int> ke(2 * (size_t)dof, 0);
    for (int k = 0; k < dof; k++) ke[2 * k] = 1;
    if ((st = upload_async(c, c->ft_kexp, ke.data(), ke.size() * sizeof(int), "field exponents")) != P2_OK) return st;
    c->ft_kexp_n = dof;
  }
  const size_t per = (size_t)dof * c->V3 * 8;
  const int tc = (int)std::max<size_t>(1, std::min<size_t>(c->ws_budget / std::max<size_t>(per, 1), (size_t)nt));
  for (int t0 = 0; t0 < nt; t0 += tc) {
    const int n = std::min(tc, nt - t0);
    P2_TRY(c, c->cbuf.ensure((size_t)n * per), "position buffer alloc");
    P2_TRY(c, c->cmaxb.ensure((size_t)n * dof * sizeof(int)), "maxima alloc");
    P2_TRY(c, c->expb.ensure((size_t)2 * n * sizeof(int)), "exponent alloc");
    std::vector<p2::SliceDesc> desc(n);
    for (int i = 0; i < n; i++) {
      std::memset(&desc[i], 0, sizeof(p2::SliceDesc));
      desc[i].tau = t0 + i;
      desc[i].totalT = nt;
    }
    P2_TRY(c, c->sdesc.ensure((size_t)n * sizeof(p2::SliceDesc)), "descriptor alloc");
    P2_TRY(c,
           cudaMemcpyAsync(c->sdesc.p, desc.data(), (size_t)n * sizeof(p2::SliceDesc), cudaMemcpyHostToDevice,
                           c->stream),
           "descriptor upload");
    p2::FieldF32Args fa{};
    fa.field = field;
    fa.vol = c->V3 * nt;
    fa.t0 = t0;
    fa.ntau = n;
    fa.K = dof;
    fa.V3 = (int)c->V3;
    fa.exps = (int*)c->expb.p;
    fa.c = (float*)c->cbuf.p;
    fa.cmax = (int*)c->cmaxb.p;
    {
      ProfScope ps(c, "field_to_f32");
      P2_TRY(c, p2::launch_field_to_f32(fa, c->nsm, c->stream), "field conversion");
    }
    if ((st = p2::split_project(c, pl, dof, n, nmtile, nkstep, (const p2::SliceDesc*)c->sdesc.p,
                                (const int*)c->expb.p, (const int*)c->ft_kexp.p, {}, dst, (long long)dof * nmom,
                                nmom)) != P2_OK)
      return st;
  }
  if (out_location == P2_HOST) {
    P2_TRY(c, cudaMemcpyAsync(out, dst, total * 16, cudaMemcpyDeviceToHost, c->stream), "result download");
    P2_TRY(c, cudaStreamSynchronize(c->stream), "result download");
  }
  return P2_OK;
}

p2_status p2_ft_apply(p2_ctx* c, const double* field, int dof, int nt, const int* moms, int nmom, int sign,
                      double* out, int out_location) {
  if (!c) return P2_ERR_INVALID_ARG;
  if (!field || !out || dof < 1 || nt < 1 || nt > c->Ll[3] || !moms || nmom < 1)
    return c->fail(P2_ERR_INVALID_ARG, "p2_ft_apply: bad arguments");
  if (sign != 1 && sign != -1) return c->fail(P2_ERR_INVALID_ARG, "p2_ft_apply: sign must be +1 or -1");
  if (c->host_only) return c->fail(P2_ERR_UNSUPPORTED, "host-only context");
  const int Lmax = std::max(c->Ll[0], std::max(c->Ll[1], c->Ll[2]));
  std::vector<double> tabh = phase_tables(c, moms, nmom, sign, Lmax);
  P2_TRY(c, c->tab.ensure(tabh.size() * sizeof(double)), "phase table alloc");
  P2_TRY(c, cudaMemcpyAsync(c->tab.p, tabh.data(), tabh.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream),
         "phase table upload");
  p2::ProjArgs pa{};
  pa.c = field;
  pa.sT = c->V3;
  pa.sK = c->V3 * nt;
  pa.ntau = nt;
  pa.K = dof;
  pa.V3 = (int)c->V3;
  pa.nmom = nmom;
  pa.Lx = c->Ll[0];
  pa.Ly = c->Ll[1];
  pa.Lz = c->Ll[2];
  pa.Lmax = Lmax;
  pa.tab = (const double*)c->tab.p;
  const int ptiles = (nmom + 63) / 64, ktiles = (dof + 31) / 32;
  int nsplit = (2 * c->nsm + ptiles * ktiles * nt - 1) / (ptiles * ktiles * nt);
  nsplit = std::max(1, std::min(nsplit, (int)((c->V3 + 255) / 256)));
  pa.chunk = (int)((((c->V3 + nsplit - 1) / nsplit) + 15) / 16 * 16);
  pa.nsplit = (int)((c->V3 + pa.chunk - 1) / pa.chunk);
  P2_TRY(c, c->part.ensure((size_t)nt * pa.nsplit * nmom * dof * 16), "partials alloc");
  pa.part = (double*)c->part.p;
  {
        ProfScope ps(c, "project_fp64");
        P2_TRY(c, p2::launch_project_fp64(pa, c->stream), "projection kernel");
      }
  const size_t total = (size_t)nt * dof * nmom;
  double* dst = out;
  if (out_location == P2_HOST) {
    P2_TRY(c, c->res.ensure(total * 16), "result alloc");
    dst = (double*)c->res.p;
  }
  p2::ScatterArgs sa{};
  sa.part = (const double*)c->part.p;
  sa.ntau = nt;
  sa.nsplit = pa.nsplit;
  sa.nmom = nmom;
  sa.K = dof;
  sa.tau0 = 0;
  sa.nblocks = 0;
  sa.oT = (long long)dof * nmom;
  sa.oK = nmom;
  sa.out = dst;
  {
        ProfScope ps(c, "reduce_scatter");
        P2_TRY(c, p2::launch_scatter(sa, c->stream), "reduction kernel");
      }
  if (out_location == P2_HOST) {
    P2_TRY(c, cudaMemcpyAsync(out, dst, total * 16, cudaMemcpyDeviceToHost, c->stream), "result download");
    P2_TRY(c, cudaStreamSynchronize(c->stream), "result download");
  }
  return P2_OK;
}

p2_status p2_alloc(p2_ctx* c, size_t bytes, int location, void** ptr) {
  if (!c || !ptr || bytes == 0) return c ? c->fail(P2_ERR_INVALID_ARG, "p2_alloc: bad arguments") : P2_ERR_INVALID_ARG;
  *ptr = nullptr;
  if (c->host_only) return c->fail(P2_ERR_UNSUPPORTED, "host-only context");
  if (location == P2_DEVICE) return c->cuda(cudaMalloc(ptr, bytes), "p2_alloc device");
  if (location == P2_HOST) return c->cuda(cudaMallocHost(ptr, bytes), "p2_alloc host");
  return c->fail(P2_ERR_INVALID_ARG, "p2_alloc: bad location");
}

p2_status p2_free(p2_ctx* c, void* ptr, int location) {
  if (!c) return P2_ERR_INVALID_ARG;
  if (!ptr) return P2_OK;
  if (c->host_only) return c->fail(P2_ERR_UNSUPPORTED, "host-only context");
  if (location == P2_DEVICE) return c->cuda(cudaFree(ptr), "p2_free device");
  if (location == P2_HOST) return c->cuda(cudaFreeHost(ptr), "p2_free host");
  return c->fail(P2_ERR_INVALID_ARG, "p2_free: bad location");
}

p2_status p2_copy(p2_ctx* c, void* dst, const void* src, size_t bytes) {
  if (!c) return P2_ERR_INVALID_ARG;
  if (!dst || !src) return c->fail(P2_ERR_INVALID_ARG, "p2_copy: null pointer");
  if (c->host_only) return c->fail(P2_ERR_UNSUPPORTED, "host-only context");
  P2_TRY(c, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, c->stream), "p2_copy");
  return c->cuda(cudaStreamSynchronize(c->stream), "p2_copy");
}

p2_status p2_synth_propagator(p2_ctx* c, void* dst, int on_device, int precision, uint64_t seed, int flavour, int t0,
                              double decay, int t_first, int nt) {
  if (!c) return P2_ERR_INVALID_ARG;
  if (!dst || nt < 1 || nt > c->T || t_first < 0 || t_first >= c->T || t0 < 0 || t0 >= c->T)
    return c->fail(P2_ERR_INVALID_ARG, "p2_synth_propagator: bad arguments");
  if (precision != P2_FP64 && precision != P2_FP32) return c->fail(P2_ERR_INVALID_ARG, "bad precision");
  if (on_device) {
    if (c->host_only) return c->fail(P2_ERR_UNSUPPORTED, "host-only context");
    P2_TRY(c,
           p2::launch_synth(dst, precision == P2_FP32, seed, flavour, t0, decay, t_first, nt, c->g.L, c->Ll,
                            c->g.coords, c->stream),
           "synth kernel");
    return P2_OK;
  }
  p2::synth_host(dst, precision == P2_FP32, seed, flavour, t0, decay, t_first, nt, c->g.L, c->Ll, c->g.coords);
  return P2_OK;
}

}  // extern "C"
