// Kernel argument blocks and launcher declarations shared by the kernels and
// the host orchestration (api.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace p2 {

constexpr int kMaxBlocks = 10;  // contraction blocks of a request (one per P2_* bit)

// Split form: the 16 x 16 meson outputs are staged through shared memory and
// written without their unit phases r_g1 r_g2 (every Gamma row is r times a
// Walsh character), which the projection's reduction applies per component,
// whenever the 16 x 16 block is requested without the 10 diagonal structures.
__host__ __device__ constexpr bool g16_phase_deferred(unsigned what) { return (what & 8u) && !(what & 64u); }
// ... and, when neither the 34 pairs nor the 10 diagonal structures of the
// same lanes are requested, no Gamma stage at all: the Gamma sums are linear
// and commute with the momentum projection, so the split contraction writes
// the 256 colour-traced products M_{a d}[b][z] = sum_colour u[a][b] conj(d[d][z])
// as the block's components (component 16 (4 a + d) + 4 b + z) and
// k_meson_gamma forms C[g1][g2] = sum G1[d][pi1(d)] G2[b][pi2(b)]
// M_{pi1(d) d}[b][pi2(b)] from their projections, per slice and momentum.
__host__ __device__ constexpr bool g16_raw(unsigned what) {
  return g16_phase_deferred(what) && !(what & (16u | 32u));
}

// Where each contraction block's components sit inside the K components of a site.
struct CompOffsets {
  int nuc, ntor, rton, rtor, diso12, diso32, g16, all34, new10, diag10;
};

// One time slice of one request, as the kernels see it.  A launch covers an
// array of slices, possibly from many sources with different windows.
struct SliceDesc {
  const void* u;           // propagator views (SoA [144][vol])
  const void* d;
  long long vol_u, vol_d;  // component strides of the views
  long long off_u, off_d;  // element offset of this slice inside the views (j * V3)
  double* out;             // result of the slice's request
  int tau;                 // source-relative time of the slice
  int totalT;              // window of the request (result layout)
  int x0[3];               // spatial source position of the request
  int xf[2];               // load-time transform of the u and d slice (prop_xf_code)
  int eh[2];               // staged u, d entries are the view's times 2^-eh (host-converted FP32 staging), else 0
};

// Load-time propagator transform of one slice, see P2_PROP_* in plegma2pt.h:
// bits 0-1 rotation (1: s = +1, 2: s = -1), bit 2 g5 from the left, bit 3 sign flip.
struct PropXf {
  static constexpr int kRotPlus = 1, kRotMinus = 2, kGamma5 = 4, kNegate = 8;
};

struct ContractArgs {
  const SliceDesc* sl;  // [ntau] slices of this launch
  int ntau;
  int V3;
  unsigned what;
  int K;
  CompOffsets k;
  void* out;  // [ntau][K][V3] complex (double for the plain form, float for the split form)
  // split form only: power-of-two scale exponents per slice and flavour
  // (input x 2^-E, exps[2 s + f]), and max(|Re|,|Im|) per (slice, component) as float bits
  const int* exps;
  int* cmax;  // [ntau][K]
  // 1: the 16 x 16 block's components are the colour products M of g16_raw
  // (its result goes through the projection and then k_meson_gamma)
  int g16_raw;
};

// Per-slice magnitude exponents of the u and d views, from a strided sample.
struct SampleArgs {
  const SliceDesc* sl;
  int fp32;
  int V3, ntau;
  int* exp_out;  // [ntau][2]
};

struct ProjArgs {
  const void* c;            // complex double, element (tau, k, x) at c[tau*sT + k*sK + x]
  long long sT, sK;
  int ntau, K, V3, nmom;
  int Lx, Ly, Lz, Lmax;
  const double* tab;        // [3][nmom][Lmax] complex: exp(sign i 2 pi n_d x_d / L_d)
  int nsplit, chunk;        // site range per split (multiple of 16)
  double* part;             // [ntau][nsplit][nmom][K] complex
  int tk;                   // component tile 16*tk (2, 4, 6 or 8); 0: the one that wastes least
};

struct ScatterBlock {
  int k0;       // first component of the block inside K
  int groups, datasets, comps;
  long long base;  // offset (complex elements) of the block in the result
};

struct ScatterArgs {
  const double* part;  // [ntau][nsplit][nmom][K]
  int ntau, nsplit, nmom, K;
  // block layout (nblocks > 0): slice tl goes to sl[tl].out at time sl[tl].tau
  // and is multiplied by the source phase exp(i p.x0) (phases have origin 0)
  int nblocks;
  ScatterBlock blk[kMaxBlocks];  // base = block offset per unit of (totalT * nmom)
  const SliceDesc* sl;
  const int* moms;  // [nmom][3]
  int L[3];
  // generic [t][dof][mom] layout when nblocks == 0: out[(tau0+tau)*oT + k*oK + p]
  int tau0;
  long long oT, oK;
  double* out;
};

// ---- split-FP16 projection ------------------------------------------------
// Phase rows: for every representative momentum h of a +-h pair, a cos row and
// (h != 0) a sin row; cos(h.x) and sin(h.x) over the sites (origin 0; the
// source's phase exp(i p.x0) is applied in the FP64 reduction), stored
// as hi+lo FP16 tiles of 128 rows x 64 sites in the tensor core's 128-byte
// swizzled K-major layout: A[mtile][kstep][hi, lo][128 x 64].
struct PhaseBuildArgs {
  const double* tab;  // [3][nh][Lmax] complex, exp(-i 2 pi h_d x_d / L_d)
  const int* row_h;   // [nrows] representative of each row
  const int* row_sin; // [nrows] 0 = cos row, 1 = sin row
  int nrows, nmtile, nkstep, V3, Lx, Ly, Lmax, nh;
  void* A;
};

struct SplitGemmArgs {
  const void* c;     // complex float [ntau][K][V3]
  const int* cmax;   // [ntau][K] max(|Re|,|Im|) as float bits
  const void* A;     // phase tiles (origin x = 0, shared by all sources)
  int ntau, K, V3, nkstep, nmtile;
  int NT, ntile;     // components per N-tile (multiple of 8, <= project_split_max_nt()), N-tiles
  int ks_per_split, nsplit;
  float* part;       // [ntau][nsplit][nmtile][128][ntile * 2 * NT]
  int* err;          // set to 1 if a bounded wait gave up
  long long wait_limit;  // nanoseconds (global timer) an mbarrier wait may take before it gives up; 0: 2 s
  int withhold;      // test hook: the converters never signal their B stages, so the waits run out
};

struct SplitReduceArgs {
  const float* part;
  int ntau, nsplit, nmtile, ncols, NT;
  int nmom, K;
  const int* mom_row;  // [nmom][6]: cos row, sin row (-1 for h = 0), sign (+1: p = h, -1: p = -h), p
  int nrep;             // representatives h; the momenta of h are rep_moms[rep_start[h] .. rep_start[h + 1])
  const int* rep_start;
  const int* rep_moms;
  int L[3];            // global spatial extents (source phase exp(i p.x0))
  const int* cmax;     // [ntau][K]
  const int* exps;     // [ntau][2]
  const int* kexp;     // [K][2]: powers of the u and d scales in component k
  const int* kphase;   // [K]: component k is multiplied by i^kphase[k], or null
  const SliceDesc* sl; // result location of each slice
  int nblocks;
  ScatterBlock blk[kMaxBlocks];  // base = block offset per unit of (totalT * nmom)
  // generic [t][K][mom] layout when nblocks == 0: out[sl[tl].tau * oT + k * oK + p]
  long long oT, oK;
  double* out;
};

// Generic field for the split projection: FP64 [K][V3 * nt] (slices t0 ..
// t0 + ntau - 1) to FP32 [ntau][K][V3] times 2^-exps[2t], exps[2t] the
// binary exponent of the largest entry of the slice; max |Re|, |Im| per
// (slice, component) into cmax.
struct FieldF32Args {
  const double* field;
  long long vol;  // component stride of the field (V3 * nt)
  int t0, ntau, K, V3;
  int* exps;      // [ntau][2]
  float* c;       // complex float
  int* cmax;      // [ntau][K]
};
cudaError_t launch_field_to_f32(const FieldF32Args& a, int nsm, cudaStream_t s);

cudaError_t launch_build_phases(const PhaseBuildArgs& a, cudaStream_t s);
cudaError_t launch_project_split(const SplitGemmArgs& a, cudaStream_t s);
cudaError_t launch_split_reduce(const SplitReduceArgs& a, cudaStream_t s);

// The 16 x 16 meson Gamma sums applied in place to the projected colour
// products of g16_raw requests: for every slice and momentum, the block's 256
// values M are replaced by C.  Result location as SplitReduceArgs (block
// layout: blk is the 16 x 16 block).
struct MesonGammaArgs {
  const SliceDesc* sl;
  int ntau, nmom;
  ScatterBlock blk;
};
cudaError_t launch_meson_gamma(const MesonGammaArgs& a, cudaStream_t s);
int project_split_smem_bytes(int NT);
int project_split_max_nt();  // widest N-tile (components) of the tensor-core projection

cudaError_t launch_contract_plain(const ContractArgs& a, int grid, cudaStream_t s);
// FP32 site contraction; fp32_in selects complex-float propagators.
cudaError_t launch_contract_f32(const ContractArgs& a, int fp32_in, int grid, cudaStream_t s);
cudaError_t launch_sample_exponents(const SampleArgs& a, cudaStream_t s);
cudaError_t launch_project_fp64(const ProjArgs& a, cudaStream_t s);
int project_fp64_tk(int K, int tk);  // component tile factor a launch with ProjArgs::tk uses
cudaError_t launch_scatter(const ScatterArgs& a, cudaStream_t s);
cudaError_t launch_synth(void* dst, int fp32, uint64_t seed, int flavour, int t0, double decay, int t_first, int nt,
                         const int* L, const int* Ll, const int* coords, cudaStream_t s);
int contract_plain_smem_bytes();

}  // namespace p2
