// C entry point over the reference's own meson contraction kernels
// (lib/kernels/PLEGMA_mesons.cuh:10-65 contract_mesons_device,
// PLEGMA_mesonsAll.cuh:7-101 contract_mesons_all_device,
// PLEGMA_mesonsNew.cuh:5-60 contract_mesons_new_device) and their in-kernel
// momentum projection (lib/kernels/PLEGMA_kernel_utils.cuh:801-860 reduce +
// fourier_transform_3D), compiled from the reference sources as host code.
// oracle/build.py extracts those functions, the meson tables and the site
// index macro from the reference files into oracle/_ref/gen (never into the
// repository) and compiles this file against them and the reference's own
// gamma tables (lib/kernels/PLEGMA_gammas.cuh).
//
// The launch is emulated one block of one thread at a time (blockDim.x = 1,
// so the shared-memory tree of reduce() is empty and every block's partial
// is one site's projected value), then the per-block partials are summed on
// the host in block order, as the reference's host drivers do
// (PLEGMA_mesons.cuh:113-120, PLEGMA_mesonsAll.cuh:140-147).
// TEST INFRASTRUCTURE ONLY: used by tests/ to pin the oracle.
#include <vector>

#include "ref_shim/PLEGMA_kernel_utils.cuh"
#include <PLEGMA_gammas.cuh>
#include "ref_mesons_extract.h"

ShimDim3 gridDim, blockIdx, blockDim, threadIdx;
int DGC_localL[4], DGC_totalL[4], DGC_procPosition[4];
int DGC_localVolume3D;
int ext_shared_cache[4096];

extern "C" {

// Projected meson two-point functions of one local time slice j, as the
// reference's kernels compute them.
//   kind 0: contract_mesons_device (10 diagonal structures of S1 S1^+ then
//           S2 S2^+, 20 components), 1: contract_mesons_all_device (34 pairs),
//   2: contract_mesons_new_device (10 structures of S1 S2^+)
//   L[3], nt: local lattice (x, y, z extents) and slices held; u, d: SoA
//   [144][V3 nt] complex double; src[3]: spatial source position;
//   moms[nmom][3]; out[nmom][ncomp] complex.
// Returns the number of components, or -1 for an unknown kind.
int ref_meson_ft(int kind, const int* L, int nt, const double* u, const double* d, int j, const int* src,
                 const int* moms, int nmom, double* out) {
  const int ncomp = kind == 0 ? 2 * N_MESONS : kind == 1 ? N_PAIRS : kind == 2 ? N_MESONS : -1;
  if (ncomp < 0) return -1;
  const int V3 = L[0] * L[1] * L[2];
  for (int i = 0; i < 3; i++) {
    DGC_localL[i] = DGC_totalL[i] = L[i];
    DGC_procPosition[i] = 0;
  }
  DGC_localL[3] = DGC_totalL[3] = nt;
  DGC_procPosition[3] = 0;
  DGC_localVolume3D = V3;
  blockDim = {1, 1, 1};
  threadIdx = {0, 0, 0};
  gridDim = {(unsigned)V3, 1, 1};
  propTex<double> t1(u, (long)V3 * nt), t2(d, (long)V3 * nt);
  tex_mom_list ml{(size_t)nmom, moms};
  const int4 source{src[0], src[1], src[2], 0};
  // one time slice per launch (time_step 1, it = j) and no window wrap (maxT > j)
  std::vector<Float2<double>> part((size_t)nmom * ncomp * V3);
  for (int b = 0; b < V3; b++) {
    blockIdx = {(unsigned)b, 0, 0};
    if (kind == 0) contract_mesons_device<double, double, double>(t1, t2, part.data(), j, 1, nt + 1, source, true, ml);
    if (kind == 1)
      contract_mesons_all_device<double, double, double>(t1, t2, part.data(), j, 1, nt + 1, source, true, ml);
    if (kind == 2)
      contract_mesons_new_device<double, double, double>(t1, t2, part.data(), j, 1, nt + 1, source, true, ml);
  }
  for (int p = 0; p < nmom; p++)
    for (int c = 0; c < ncomp; c++) {
      Float2<double> acc(0.0, 0.0);
      for (int b = 0; b < V3; b++) acc = acc + part[((size_t)p * ncomp + c) * V3 + b];
      out[2 * (p * ncomp + c)] = acc.x;
      out[2 * (p * ncomp + c) + 1] = acc.y;
    }
  return ncomp;
}
}
