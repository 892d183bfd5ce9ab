// Plain FP64 site contraction: propagators staged through shared memory,
// one site per half-warp, results written to a position-space buffer that
// the direct phase sum (project_fp64.cu) consumes.
//
// Replaces the per-site part of contract_baryons_device / contract_NtoN_kernel
// (lib/kernels/PLEGMA_baryons.cuh:82-147, PLEGMA_baryons_NtoN.cu:6-46) and
// contract_mesons_{all,new,}_device (PLEGMA_mesonsAll.cuh:7-95,
// PLEGMA_mesonsNew.cuh:5-56, PLEGMA_mesons.cuh:10-65).
//
// Layout and schedule
//  - a CTA of 256 threads is persistent over tiles of 16 consecutive sites of
//    one time slice (tile = (tau, x0));
//  - each tile's 2 x 144 complex per site are copied with cp.async, 16 B per
//    copy, coalesced along the site axis of the SoA propagator, into
//    shared memory as [site][flavour*144 + component] (row padded to 289
//    complex so the 16 half-warps' rows start in different banks);
//  - two stages: tile i+1's copies are in flight while tile i is contracted;
//  - half-warp h contracts site h of the tile (site_contract.cuh).
#include "kernels.cuh"
#include "site_contract.cuh"

namespace p2 {

namespace {

constexpr int kThreads = 256;
constexpr int kSitesPerTile = 16;
constexpr int kRow = 289;  // complex per site row (2 * 144 + 1 pad)
constexpr int kStage = kSitesPerTile * kRow;

__device__ __forceinline__ void issue_tile(const ContractArgs& a, Cx<double>* st, long long tile, long long ntiles,
                                           int tiles_per_tau) {
  if (tile < ntiles) {
    const int tl = (int)(tile / tiles_per_tau);
    const int x0 = (int)(tile - (long long)tl * tiles_per_tau) * kSitesPerTile;
    const int t = (a.t0 + a.tau0 + tl) % a.T;
    const long long ju = (long long)((t - a.t_first_u + a.T) % a.T) * a.V3;
    const long long jd = (long long)((t - a.t_first_d + a.T) % a.T) * a.V3;
    const Cx<double>* U = (const Cx<double>*)a.u;
    const Cx<double>* D = (const Cx<double>*)a.d;
#pragma unroll 2
    for (int r = 0; r < (2 * 144 * kSitesPerTile) / kThreads; r++) {
      const int i = threadIdx.x + r * kThreads;
      const int s = i & (kSitesPerTile - 1);
      const int rest = i >> 4;
      const int f = rest >= 144;
      const int comp = rest - 144 * f;
      const int x = x0 + s;
      const bool ok = x < a.V3;
      const Cx<double>* src = f ? D + (long long)comp * a.vol_d + jd + (ok ? x : 0)
                                : U + (long long)comp * a.vol_u + ju + (ok ? x : 0);
      cp_async16(st + s * kRow + rest, src, ok ? 16 : 0);
    }
  }
  cp_async_commit();
}

// ALL34 / NEW10 / DIAG10 selection: index of a diagonal structure in the
// 10-structure list (1, g5, g1..g4, g5g1..g5g4), or -1.
__device__ __forceinline__ int diag10_slot(int g) {
  // structures 0, 5, 1, 2, 3, 4, 6, 7, 8, 9
  return g == 0 ? 0 : g == 5 ? 1 : (g >= 1 && g <= 4) ? g + 1 : (g >= 6 && g <= 9) ? g : -1;
}

__global__ void __launch_bounds__(kThreads, 1) k_contract_plain(const ContractArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cx<double>* sm = (Cx<double>*)smem_raw;
  const int tid = threadIdx.x;
  const int hw = tid >> 4, l = tid & 15;
  const unsigned mask = halfwarp_mask();
  const LaneTables lt = load_lane_tables(l);

  const int tiles_per_tau = (a.V3 + kSitesPerTile - 1) / kSitesPerTile;
  const long long ntiles = (long long)a.ntau * tiles_per_tau;
  long long tile = blockIdx.x;

  issue_tile(a, sm, tile, ntiles, tiles_per_tau);
  issue_tile(a, sm + kStage, tile + gridDim.x, ntiles, tiles_per_tau);

  for (int it = 0; tile < ntiles; tile += gridDim.x, it++) {
    Cx<double>* st = sm + (it & 1) * kStage;
    cp_async_wait<1>();
    __syncthreads();

    const int tl = (int)(tile / tiles_per_tau);
    const int x = (int)(tile - (long long)tl * tiles_per_tau) * kSitesPerTile + hw;
    if (x < a.V3) {
      const Cx<double>* U = st + hw * kRow;
      const Cx<double>* D = U + 144;
      Cx<double>* out = (Cx<double>*)a.out + (long long)tl * a.K * a.V3 + x;
      const long long V3 = a.V3;
      if (a.what & 1u) {
        Cx<double> p = nucleon_site<double>(U, D, lt, l, mask);
        Cx<double> n = nucleon_site<double>(D, U, lt, l, mask);
        out[(a.k.nuc + l) * V3] = p;
        out[(a.k.nuc + 16 + l) * V3] = n;
      }
      if (a.what & (8u | 16u | 32u)) {
        Cx<double> c[16];
        meson_site<double>(U, D, lt, l, mask, c);
        if (a.what & 8u) {
#pragma unroll
          for (int g2 = 0; g2 < 16; g2++) out[(a.k.g16 + l * 16 + g2) * V3] = c[g2];
        }
        if (a.what & 16u) {
          if (l == 0) out[(a.k.all34 + 0) * V3] = c[0];
          if (l == 5) out[(a.k.all34 + 1) * V3] = c[5];
          if (l >= 1 && l <= 4) {
#pragma unroll
            for (int g2 = 1; g2 <= 4; g2++) out[(a.k.all34 + 2 + (l - 1) * 4 + (g2 - 1)) * V3] = c[g2];
          }
          if (l >= 6 && l <= 9) {
#pragma unroll
            for (int g2 = 6; g2 <= 9; g2++) out[(a.k.all34 + 18 + (l - 6) * 4 + (g2 - 6)) * V3] = c[g2];
          }
        }
        if (a.what & 32u) {
          const int j = diag10_slot(l);
#pragma unroll
          for (int g2 = 0; g2 < 16; g2++)
            if (g2 == l && j >= 0) out[(a.k.new10 + j) * V3] = c[g2];
        }
      }
      if (a.what & 64u) {
        const int j = diag10_slot(l);
        Cx<double> c[16];
        meson_site<double>(U, U, lt, l, mask, c);
#pragma unroll
        for (int g2 = 0; g2 < 16; g2++)
          if (g2 == l && j >= 0) out[(a.k.diag10 + j) * V3] = c[g2];
        meson_site<double>(D, D, lt, l, mask, c);
#pragma unroll
        for (int g2 = 0; g2 < 16; g2++)
          if (g2 == l && j >= 0) out[(a.k.diag10 + 10 + j) * V3] = c[g2];
      }
    }
    __syncthreads();
    issue_tile(a, st, tile + 2LL * gridDim.x, ntiles, tiles_per_tau);
  }
  cp_async_wait<0>();
}

}  // namespace

int contract_plain_smem_bytes() { return 2 * kStage * (int)sizeof(Cx<double>); }

cudaError_t launch_contract_plain(const ContractArgs& a, int grid, cudaStream_t s) {
  const int smem = contract_plain_smem_bytes();
  cudaError_t e = cudaFuncSetAttribute(k_contract_plain, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  k_contract_plain<<<grid, kThreads, smem, s>>>(a);
  return cudaGetLastError();
}

}  // namespace p2
