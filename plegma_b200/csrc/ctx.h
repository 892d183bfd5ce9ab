// Context of the C ABI and the helpers shared by the plain (api.cu) and the
// split-FP16 (precision.cu) paths.
#pragma once
#include <memory>
#include <string>
#include <vector>

#include "../../include/plegma2pt.h"
#include "kernels.cuh"
#include "tuner.h"

namespace p2host {

// Pinned host buffer (cudaMallocHost), grown on demand.
struct HostBuf {
  void* p = nullptr;
  size_t n = 0;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= n) return cudaSuccess;
    if (p) cudaFreeHost(p);
    p = nullptr;
    n = 0;
    cudaError_t e = cudaMallocHost(&p, bytes);
    if (e == cudaSuccess) n = bytes;
    return e;
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    n = 0;
  }
};

struct DevBuf {
  void* p = nullptr;
  size_t n = 0;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= n) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e == cudaSuccess) n = bytes;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
};

struct BlockDef {
  unsigned bit;
  int groups, datasets, comps;
};
constexpr BlockDef kBlocks[] = {
    {P2_NUCLEON_CG5, 1, 2, 16},  {P2_NUCLEON_NTOR, 1, 2, 16}, {P2_NUCLEON_RTON, 1, 2, 16},
    {P2_NUCLEON_RTOR, 1, 2, 16}, {P2_DELTA_ISO12, 3, 2, 16},  {P2_DELTA_ISO32, 3, 2, 16},
    {P2_MESON_G16, 1, 1, 256},   {P2_MESON_ALL34, 1, 1, 34}, {P2_MESON_NEW10, 1, 1, 10},
    {P2_MESON_DIAG10, 1, 2, 10},
};
constexpr unsigned kAllBits = 0x3FFu;
// every block of a request has a slot in the reduction kernels' argument structs
static_assert(sizeof(kBlocks) / sizeof(kBlocks[0]) <= (size_t)p2::kMaxBlocks, "kMaxBlocks too small for kBlocks");

}  // namespace p2host

struct p2_udsc_cache;  // table-driven baryons: per-product lane plans (udsc.cu)

struct p2_ctx {
  p2_geom g{};
  int Ll[4]{};
  long long V3 = 0;
  int T = 0;
  int nsm = 148;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  bool host_only = false;  // created with device < 0
  std::string err = "no error";
  p2host::DevBuf cbuf, part, tab, res, moms;
  // slice descriptors of the current call and their pinned host mirror
  p2host::DevBuf sdesc;
  void* sdesc_host = nullptr;
  size_t sdesc_host_n = 0;
  cudaEvent_t sdesc_copied = nullptr;  // the mirror may be rewritten once this completes
  bool capturing = false;              // recording a graph: no host synchronisation
  // host-resident propagators: two staging slots per flavour, uploaded on a
  // copy stream while the previous chunk is contracted
  p2host::DevBuf ft_kexp;  // split field transform: (1, 0) per component
  int ft_kexp_n = 0;
  p2host::DevBuf stage_u2[2], stage_d2[2];
  // host-side FP32 conversion of host views (split form): pinned buffers and
  // the events of their last upload
  static constexpr int kHostSlots = 3;
  p2host::HostBuf hstage_u[kHostSlots], hstage_d[kHostSlots];
  cudaEvent_t hcopied[kHostSlots] = {nullptr, nullptr, nullptr};
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t copied[2] = {nullptr, nullptr}, consumed[2] = {nullptr, nullptr};
  // split form: phase tiles, per-slice exponents, component maxima, tables, partials, error flag
  p2host::DevBuf phaseA, expb, cmaxb, momrow, kexp, fpart, rowtab, errflag;
  std::vector<int> split_moms_key;  // momentum list the phase tiles and rows were built for
  int split_nrep = 0;                // representatives (+-h pairs) of that list
  unsigned split_what_key = 0;      // contraction set of the component exponents
  int project_split_smem_max = 0;  // opt-in shared memory per block of the device
  int wait_test = 0;               // p2_debug_wait_timeout armed for the next tensor-core projection
  size_t ws_budget = 0;
  // plain form: phase tables and momentum list, rebuilt when the momentum list changes
  p2host::DevBuf ptab;
  std::vector<int> plain_moms_key;
  p2_udsc_cache* udsc = nullptr;
  // launch-shape autotuner (shared with the context's graphs)
  std::shared_ptr<p2host::Tuner> tuner = std::make_shared<p2host::Tuner>();

  // kernel timing (p2_profile_enable)
  struct Prof {
    std::string name;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending;
    std::vector<cudaEvent_t> pool;
    double ms = 0;
    long long launches = 0;
  };
  bool profiling = false;
  std::vector<Prof> prof;
  cudaEvent_t prof_begin(const char* name, int& slot, cudaStream_t on = nullptr);
  void prof_end(int slot, cudaEvent_t start, cudaStream_t on = nullptr);
  void prof_collect();
  void prof_clear();

  p2_status fail(p2_status s, const std::string& m) {
    err = m;
    return s;
  }
  p2_status cuda(cudaError_t e, const char* where) {
    if (e == cudaSuccess) return P2_OK;
    cudaGetLastError();
    err = std::string(where) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? P2_ERR_OOM : P2_ERR_CUDA;
  }
};

// Brackets one kernel launch with events when profiling is on.
struct ProfScope {
  p2_ctx* c;
  cudaStream_t on;
  int slot = -1;
  cudaEvent_t start = nullptr;
  ProfScope(p2_ctx* ctx, const char* name, cudaStream_t s = nullptr) : c(ctx), on(s) {
    if (c->profiling) start = c->prof_begin(name, slot, on);
  }
  ~ProfScope() {
    if (start) c->prof_end(slot, start, on);
  }
};

#define P2_TRY(ctx, call, where)                 \
  do {                                           \
    p2_status _s = (ctx)->cuda((call), (where)); \
    if (_s != P2_OK) return _s;                  \
  } while (0)


namespace p2host {

struct Plan {
  int K, nmom, Lmax, totalT;
  std::vector<int> moms;
  std::vector<p2::ScatterBlock> blocks;  // base = block offset per unit of (totalT * nmom)
  size_t total;  // complex elements of the result
};

// One local time slice of one request: its source-relative time and the
// slice's index in the request's u and d views.
struct SliceRef {
  int req, tau, ju, jd;
};

// Slices [s0, s0 + n) of a work list, processed by one launch sequence.
struct Chunk {
  int s0, n;
};

struct Work {
  std::vector<SliceRef> sl;
  std::vector<Chunk> chunks;
  int max_n = 0;
};

// The local slices of requests reqs[idx[0..nidx)] in request order, cut into
// chunks of at most tc slices.
Work make_work(const p2_ctx* c, const p2_prop* props, const p2_request* reqs, const int* idx, int nidx, int tc);

// Device views and slice descriptors of a work list.  Device propagators are
// read in place; host propagators are uploaded chunk by chunk into two
// staging slots on a copy stream, so chunk i+1 crosses PCIe while chunk i is
// contracted.  All descriptors go to the device in one copy (prepare).
struct Stager {
  p2_ctx* c;
  const p2_prop* props;
  const p2_request* reqs;
  const Work& w;
  bool host = false;
  // split form with every view on the host in FP64: the host converts each
  // chunk to FP32 (times 2^-eh per slice and flavour, exact) into pinned
  // buffers and uploads half the bytes
  bool cvt32 = false;
  // with cvt32, every kRawEvery-th chunk (from the first) goes up unconverted
  // in FP64 instead: the link has room while the host cores convert, and the
  // first upload starts without waiting for a conversion
  static constexpr int kRawEvery = 6;
  bool converts(int ci) const { return cvt32 && ci % kRawEvery != 0; }
  // pinned buffer slot of converted chunk ci (the converted chunks before it, modulo the slots)
  int host_slot(int ci) const { return (ci - (ci + kRawEvery - 1) / kRawEvery) % p2_ctx::kHostSlots; }
  p2::SliceDesc* dsl = nullptr;
  Stager(p2_ctx* ctx, const p2_prop* pp, const p2_request* rr, const Work& work);
  // outs[req]: device result pointer of each request (indexed like reqs)
  p2_status prepare(double* const* outs);
  p2_status issue(int ci);    // start the upload of chunk ci
  p2_status wait(int ci);     // the compute stream waits for chunk ci's upload
  p2_status release(int ci);  // chunk ci's kernels are queued; its slot may be refilled
  const p2::SliceDesc* desc(int ci) const { return dsl + w.chunks[ci].s0; }
};

int components_of(unsigned what);
int prop_xf_code(const p2_prop& p, int t);
p2::CompOffsets offsets_of(unsigned what);
// [3][nmom][Lmax] complex exp(sign i 2 pi n_d x_d / L_d), x_d the global coordinate of local xl
std::vector<double> phase_tables(const p2_ctx* c, const int* moms, int nmom, int sign, int Lmax);
p2_status make_plan(p2_ctx* c, const p2_request& r, Plan& pl);
p2_status upload_async(p2_ctx* c, DevBuf& b, const void* src, size_t bytes, const char* what);

}  // namespace p2host

void p2_udsc_release(p2_ctx* c);

namespace p2 {
// split-FP16 path (precision.cu)
// requests reqs[idx[..]] share contractions, momenta (pl) and input precision;
// outs[j] is the device result of request j
p2_status precision_run_batch(p2_ctx* c, const p2_prop* props, const p2_request* reqs, const int* idx, int nidx,
                              const p2host::Plan& pl, double* const* outs);
void precision_release(p2_ctx* c);
// shared with the split form of the table-driven baryons (udsc.cu)
p2_status split_prepare_tables(p2_ctx* c, const p2host::Plan& pl, unsigned what, int& nmtile, int& nkstep);
p2_status split_project(p2_ctx* c, const p2host::Plan& pl, int K, int n, int nmtile, int nkstep, const SliceDesc* dsl,
                        const int* exps, const int* kexp, const std::vector<ScatterBlock>& blocks,
                        double* out = nullptr, long long oT = 0, long long oK = 0, const int* kphase = nullptr);
}  // namespace p2
