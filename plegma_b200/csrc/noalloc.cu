// Momentum projection of a field without any allocation (p2_ft_apply_noalloc).
//
// Some callers cannot allocate device memory when they call the library: a
// host framework that reserves all device memory up front for its own pool
// and treats any further cudaMalloc/cudaFree as an error, or an embedded
// caller with a fixed device-memory budget that must not grow after start-up.
// For them the generic projection below keeps its scratch (the momentum list,
// the per-dimension phase tables and the per-block partial sums) in one
// file-scope device array of kNoAllocScratchBytes.  Every GPU that loads the
// library holds this array until the process exits.
//
// The array's device address is looked up once per device, with that device
// current, on the entry point's first call on the device; make that first
// call before any stream capture.  All calls share the array and it keeps the
// last call's contents: every byte a call reads is written earlier in the same
// call (momenta, tables, partials), so nothing needs clearing; calls whose work
// overlaps on the GPU (two streams or two threads at once) race on it.
#include <mutex>

#include "ctx.h"

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;  // 32 MiB
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

void* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mu;

constexpr size_t round256(size_t n) { return (n + 255) / 256 * 256; }

// [3][nmom][Lmax] complex double: exp(sign i 2 pi n_d x_d / L_d), x_d the global
// coordinate of local coordinate xl (origin at 0, as PLEGMA_FT::apply).
__global__ void k_noalloc_tables(const int* moms, int nmom, int l0, int l1, int l2, int o0, int o1, int o2, int L0,
                                 int L1, int L2, int Lmax, int sign, double* tab) {
  const int n = 3 * nmom * Lmax;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int d = i / (nmom * Lmax);
    const int p = (i / Lmax) % nmom;
    const int xl = i % Lmax;
    const int Ll = d == 0 ? l0 : d == 1 ? l1 : l2;
    const int Lg = d == 0 ? L0 : d == 1 ? L1 : L2;
    const int off = d == 0 ? o0 : d == 1 ? o1 : o2;
    double c = 0.0, s = 0.0;
    if (xl < Ll) {
      long long num = ((long long)moms[3 * p + d] * (long long)(xl + off)) % Lg;
      if (num < 0) num += Lg;
      sincospi(2.0 * (double)num / (double)Lg, &s, &c);
    }
    tab[2 * i] = c;
    tab[2 * i + 1] = sign * s;
  }
}

}  // namespace

extern "C" p2_status p2_ft_apply_noalloc(p2_ctx* c, const double* field, int dof, int nt, const int* moms, int nmom,
                                         int sign, double* out) {
  if (!c) return P2_ERR_INVALID_ARG;
  if (c->host_only) return c->fail(P2_ERR_UNSUPPORTED, "host-only context");
  if (!field || !out || dof < 1 || nt < 1 || nt > c->Ll[3] || !moms || nmom < 1)
    return c->fail(P2_ERR_INVALID_ARG, "p2_ft_apply_noalloc: bad arguments");
  if (sign != 1 && sign != -1) return c->fail(P2_ERR_INVALID_ARG, "p2_ft_apply_noalloc: sign must be +1 or -1");
  const int dev = c->g.device;
  if (dev < 0 || dev >= kMaxDevices) return c->fail(P2_ERR_UNSUPPORTED, "p2_ft_apply_noalloc: device ordinal too large");

  // scratch layout: momenta | phase tables | partials
  const int Lmax = c->Ll[0] > c->Ll[1] ? (c->Ll[0] > c->Ll[2] ? c->Ll[0] : c->Ll[2]) : (c->Ll[1] > c->Ll[2] ? c->Ll[1] : c->Ll[2]);
  const size_t mom_bytes = round256((size_t)3 * nmom * sizeof(int));
  const size_t tab_bytes = round256((size_t)3 * nmom * Lmax * 16);
  const size_t per_split = (size_t)nt * nmom * dof * 16;
  if (mom_bytes + tab_bytes + per_split > kNoAllocScratchBytes)
    return c->fail(P2_ERR_INVALID_ARG, "p2_ft_apply_noalloc: nt*nmom*dof*16 + tables exceeds the 32 MiB scratch");

  void* base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
      int prev = -1;
      cudaGetDevice(&prev);
      cudaError_t e = cudaSetDevice(dev);
      void* p = nullptr;
      if (e == cudaSuccess) e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (prev >= 0) cudaSetDevice(prev);
      if (e != cudaSuccess) return c->cuda(e, "p2_ft_apply_noalloc: scratch address");
      g_scratch_addr[dev] = p;
    }
    base = g_scratch_addr[dev];
  }
  int* dmoms = (int*)base;
  double* tab = (double*)((char*)base + mom_bytes);
  double* part = (double*)((char*)base + mom_bytes + tab_bytes);

  // as many site splits as fill the device, within the scratch
  const int ptiles = (nmom + 63) / 64, ktiles = (dof + 31) / 32;
  int nsplit = (2 * c->nsm + ptiles * ktiles * nt - 1) / (ptiles * ktiles * nt);
  const int fit = (int)((kNoAllocScratchBytes - mom_bytes - tab_bytes) / per_split);
  nsplit = nsplit < fit ? nsplit : fit;
  const int maxsplit = (int)((c->V3 + 255) / 256);
  nsplit = nsplit < maxsplit ? nsplit : maxsplit;
  if (nsplit < 1) nsplit = 1;

  P2_TRY(c, cudaMemcpyAsync(dmoms, moms, (size_t)3 * nmom * sizeof(int), cudaMemcpyHostToDevice, c->stream),
         "p2_ft_apply_noalloc: momenta");
  k_noalloc_tables<<<(3 * nmom * Lmax + 255) / 256, 256, 0, c->stream>>>(
      dmoms, nmom, c->Ll[0], c->Ll[1], c->Ll[2], c->g.coords[0] * c->Ll[0], c->g.coords[1] * c->Ll[1],
      c->g.coords[2] * c->Ll[2], c->g.L[0], c->g.L[1], c->g.L[2], Lmax, sign, tab);
  P2_TRY(c, cudaGetLastError(), "p2_ft_apply_noalloc: tables");

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
  pa.tab = tab;
  pa.chunk = (int)((((c->V3 + nsplit - 1) / nsplit) + 15) / 16 * 16);
  pa.nsplit = (int)((c->V3 + pa.chunk - 1) / pa.chunk);
  pa.part = part;
  P2_TRY(c, p2::launch_project_fp64(pa, c->stream), "p2_ft_apply_noalloc: projection");

  p2::ScatterArgs sa{};
  sa.part = part;
  sa.ntau = nt;
  sa.nsplit = pa.nsplit;
  sa.nmom = nmom;
  sa.K = dof;
  sa.tau0 = 0;
  sa.nblocks = 0;
  sa.oT = (long long)dof * nmom;
  sa.oK = nmom;
  sa.out = out;
  P2_TRY(c, p2::launch_scatter(sa, c->stream), "p2_ft_apply_noalloc: reduction");
  return P2_OK;
}
