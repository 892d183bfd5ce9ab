// Kernel argument blocks and launcher declarations shared by the kernels and
// the host orchestration (api.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace p2 {

constexpr int kMaxBlocks = 8;

// Where each contraction block's components sit inside the K components of a site.
struct CompOffsets {
  int nuc, diso12, diso32, g16, all34, new10, diag10;
};

struct ContractArgs {
  const void* u;
  const void* d;
  long long vol_u, vol_d;  // component stride of the views (V3 * nt)
  int t_first_u, t_first_d;
  int V3, T;
  int t0;
  int tau0, ntau;  // source-relative times of this chunk
  unsigned what;
  int K;
  CompOffsets k;
  void* out;  // [ntau][K][V3] complex (double for the plain form)
};

struct ProjArgs {
  const void* c;            // complex double, element (tau, k, x) at c[tau*sT + k*sK + x]
  long long sT, sK;
  int ntau, K, V3, nmom;
  int Lx, Ly, Lz, Lmax;
  const double* tab;        // [3][nmom][Lmax] complex: exp(sign i 2 pi n_d (x_d - x0_d) / L_d)
  int nsplit, chunk;        // site range per split (multiple of 16)
  double* part;             // [ntau][nsplit][nmom][K] complex
};

struct ScatterBlock {
  int k0;       // first component of the block inside K
  int groups, datasets, comps;
  long long base;  // offset (complex elements) of the block in the result
};

struct ScatterArgs {
  const double* part;  // [ntau][nsplit][nmom][K]
  int ntau, nsplit, nmom, K;
  int tau0, totalT;
  int nblocks;
  ScatterBlock blk[kMaxBlocks];
  // generic [t][dof][mom] layout when nblocks == 0: out[(tau0+tau)*oT + k*oK + p]
  long long oT, oK;
  double* out;
};

cudaError_t launch_contract_plain(const ContractArgs& a, int grid, cudaStream_t s);
cudaError_t launch_project_fp64(const ProjArgs& a, cudaStream_t s);
cudaError_t launch_scatter(const ScatterArgs& a, cudaStream_t s);
cudaError_t launch_synth(void* dst, int fp32, uint64_t seed, int flavour, int t0, double decay, int t_first, int nt,
                         const int* L, const int* Ll, const int* coords, cudaStream_t s);
int contract_plain_smem_bytes();

}  // namespace p2
