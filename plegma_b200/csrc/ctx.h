// Context of the C ABI and the helpers shared by the plain (api.cu) and the
// split-FP16 (precision.cu) paths.
#pragma once
#include <string>
#include <vector>

#include "../../include/plegma2pt.h"
#include "kernels.cuh"

namespace p2host {

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
    {P2_NUCLEON_CG5, 1, 2, 16},  {P2_DELTA_ISO12, 3, 2, 16}, {P2_DELTA_ISO32, 3, 2, 16},
    {P2_MESON_G16, 1, 1, 256},   {P2_MESON_ALL34, 1, 1, 34}, {P2_MESON_NEW10, 1, 1, 10},
    {P2_MESON_DIAG10, 1, 2, 10},
};
constexpr unsigned kAllBits = 0x7Fu;

}  // namespace p2host

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
  p2host::DevBuf cbuf, part, tab, res, stage_u, stage_d, scratch;
  // host-resident propagators: two staging slots per flavour, uploaded on a
  // copy stream while the previous chunk is contracted
  p2host::DevBuf stage_u2[2], stage_d2[2];
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t copied[2] = {nullptr, nullptr}, consumed[2] = {nullptr, nullptr};
  // split form: phase tiles, per-slice exponents, component maxima, tables, partials, error flag
  p2host::DevBuf phaseA, expb, cmaxb, momrow, kexp, fpart, rowtab, errflag;
  int project_split_smem_max = 0;  // opt-in shared memory per block of the device
  size_t ws_budget = 0;

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
  cudaEvent_t prof_begin(const char* name, int& slot);
  void prof_end(int slot, cudaEvent_t start);
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
  int slot = -1;
  cudaEvent_t start = nullptr;
  ProfScope(p2_ctx* ctx, const char* name) : c(ctx) {
    if (c->profiling) start = c->prof_begin(name, slot);
  }
  ~ProfScope() {
    if (start) c->prof_end(slot, start);
  }
};

#define P2_TRY(ctx, call, where)                 \
  do {                                           \
    p2_status _s = (ctx)->cuda((call), (where)); \
    if (_s != P2_OK) return _s;                  \
  } while (0)


namespace p2host {

// Consecutive source-relative times whose slices are stored contiguously in both views.
struct TauRun {
  int tau0, n;
};

struct Plan {
  int K, nmom, Lmax, totalT;
  std::vector<int> moms;
  std::vector<p2::ScatterBlock> blocks;
  size_t total;  // complex elements of the result
};

// A chunk of consecutive source-relative times processed by one launch sequence.
struct Chunk {
  int tau0, n, t_begin;
};

// Splits the local time runs of a request into chunks of at most `tc` slices.
std::vector<Chunk> make_chunks(const p2_ctx* c, const std::vector<TauRun>& runs, const int* src, int tc);

// Device views of (u, d) for each chunk.  Device propagators are used in
// place; host propagators are uploaded into two staging slots on a copy
// stream, so chunk i+1 crosses PCIe while chunk i is contracted.
struct Uploader {
  p2_ctx* c;
  const p2_prop& u;
  const p2_prop& d;
  bool host;
  Uploader(p2_ctx* ctx, const p2_prop& pu, const p2_prop& pd);
  p2_status issue(int slot, const Chunk& ch);                    // start the upload of a chunk
  p2_status view(int slot, const Chunk& ch, p2::ContractArgs& a);  // views for the compute stream
  p2_status release(int slot);                                   // the chunk's kernels are queued
};

int components_of(unsigned what);
p2::CompOffsets offsets_of(unsigned what);
std::vector<double> phase_tables(const p2_ctx* c, const int* moms, int nmom, const int* src, int sign, int Lmax);
std::vector<TauRun> local_runs(const p2_ctx* c, const p2_prop& u, const p2_prop& d, const int* src, int totalT);
p2_status make_plan(p2_ctx* c, const p2_request& r, Plan& pl);
p2_status chunk_view(p2_ctx* c, const p2_prop& p, DevBuf& stage, int t_begin, int n, p2::ContractArgs& a, bool is_u);

}  // namespace p2host

namespace p2 {
// split-FP16 path (precision.cu)
p2_status precision_run_batch(p2_ctx* c, const p2_prop* props, int nprops, const p2_request* reqs, int nreq);
void precision_release(p2_ctx* c);
}  // namespace p2
