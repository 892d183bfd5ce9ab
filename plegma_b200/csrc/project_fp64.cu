// Direct FP64 phase sum and the deterministic cross-block reduction.
//
// C(t, p, k) = sum_x c_k(x, t) exp(sign * i p.(x - x0)), the reference's
// fourier_transform_3D (lib/kernels/PLEGMA_kernel_utils.cuh:820-860) and the
// host block sum after it (PLEGMA_baryons.cuh:146-155,198, PLEGMA_mesons*.cuh).
// Per time slice this is a complex [nmom x V3] . [V3 x K] product; the phase
// matrix is never stored: each entry is the product of three per-dimension
// phase tables (p.x = sum_d n_d x_d), built on the host in double precision.
//
// CTA tile 64 momenta x (16*TK) components, 256 threads, each thread a
// 4 x TK register tile; sites are consumed 16 at a time from shared memory,
// the next 16 sites' global loads in flight meanwhile.
// The site range of a slice is split over `nsplit` CTAs whose partial sums
// go to `part`; k_scatter adds them in a fixed order (bitwise reproducible)
// and writes the result layout.
#include "kernels.cuh"
#include "p2_common.cuh"

namespace p2 {

namespace {

constexpr int kThreads = 256;
constexpr int kXS = 16;  // sites per step
constexpr int kTP = 4;   // momenta per thread
constexpr int kPT = 16 * kTP;

// Shared-memory tiles of one 16-site step: phases sE[site][momentum] and
// site values sC[component][site ^ (component & 15)] (component-major like
// the global buffer, the site index XOR-swizzled so that the transposing
// store and the per-component reads of a quarter-warp both touch 8
// different 16-byte bank groups).  The next step's global loads are issued
// into registers before the current step's products (software pipeline).
// Tiles of up to 4 x 4 complex per thread fit in 128 registers: two CTAs per
// SM (16 warps) hide the loads without a register prefetch; the 4 x 6 tile
// runs one CTA per SM with the prefetch, the 4 x 8 tile with neither.
template <int TK>
__global__ void __launch_bounds__(kThreads, TK <= 4 ? 2 : 1) k_project_fp64(const ProjArgs a) {
  constexpr int KT = 16 * TK;
  constexpr int NE = (kXS * kPT) / kThreads;  // phase entries per thread per step
  constexpr int NC = (kXS * KT) / kThreads;   // site values per thread per step
  __shared__ Cx<double> sE[kXS][kPT];
  __shared__ Cx<double> sC[KT][kXS];
  const int tid = threadIdx.x;
  const int tp = tid >> 4, tk = tid & 15;
  const int ktiles = (a.K + KT - 1) / KT;
  const int p0 = (blockIdx.x / ktiles) * kPT;
  const int k0 = (blockIdx.x % ktiles) * KT;
  const int split = blockIdx.y;
  const int tau = blockIdx.z;
  const int xb = split * a.chunk;
  const int xe = min(a.V3, xb + a.chunk);
  const Cx<double>* c = (const Cx<double>*)a.c + (long long)tau * a.sT;
  const Cx<double>* tab = (const Cx<double>*)a.tab;
  const int LxLy = a.Lx * a.Ly;

  Cx<double> acc[kTP][TK];
#pragma unroll
  for (int i = 0; i < kTP; i++)
#pragma unroll
    for (int j = 0; j < TK; j++) acc[i][j] = czero<double>();

  // this thread's loads of a step: phase entries (xs = e / kPT, pp = e % kPT)
  // as three per-dimension factors, site values (xs = e % kXS, kk = e / kXS);
  // the 4 x 6 tile prefetches; the others load each step at its start
  constexpr bool kPrefetch = TK == 6;
  Cx<double> fx[NE], fy[NE], fz[NE], cv_next[NC];
  auto load_phases = [&](int xs0) {
#pragma unroll
    for (int r = 0; r < NE; r++) {
      const int e = tid + r * kThreads;
      const int xs = e / kPT, pp = e % kPT;
      const int p = p0 + pp, x = xs0 + xs;
      fx[r] = fy[r] = fz[r] = czero<double>();
      if (p < a.nmom && x < xe) {
        const int xx = x % a.Lx, yy = (x / a.Lx) % a.Ly, zz = x / LxLy;
        fx[r] = tab[(0 * a.nmom + p) * a.Lmax + xx];
        fy[r] = tab[(1 * a.nmom + p) * a.Lmax + yy];
        fz[r] = tab[(2 * a.nmom + p) * a.Lmax + zz];
      }
    }
  };
  auto load_step = [&](int xs0) {
    load_phases(xs0);
#pragma unroll
    for (int r = 0; r < NC; r++) {
      const int e = tid + r * kThreads;
      const int xs = e % kXS, kk = e / kXS;
      const int k = k0 + kk, x = xs0 + xs;
      cv_next[r] = czero<double>();
      if (k < a.K && x < xe) cv_next[r] = c[(long long)k * a.sK + x];
    }
  };
  if (kPrefetch && xb < xe) load_step(xb);
  for (int xs0 = xb; xs0 < xe; xs0 += kXS) {
    if (kPrefetch) {
#pragma unroll
      for (int r = 0; r < NE; r++) {
        const int e = tid + r * kThreads;
        sE[e / kPT][e % kPT] = cmul(cmul(fx[r], fy[r]), fz[r]);
      }
#pragma unroll
      for (int r = 0; r < NC; r++) {
        const int e = tid + r * kThreads;
        const int xs = e % kXS, kk = e / kXS;
        sC[kk][xs ^ (kk & 15)] = cv_next[r];
      }
    } else {
      // each entry straight from the global tables into shared memory (no register arrays live)
#pragma unroll
      for (int r = 0; r < NE; r++) {
        const int e = tid + r * kThreads;
        const int xs = e / kPT, pp = e % kPT;
        const int p = p0 + pp, x = xs0 + xs;
        Cx<double> v = czero<double>();
        if (p < a.nmom && x < xe) {
          const int xx = x % a.Lx, yy = (x / a.Lx) % a.Ly, zz = x / LxLy;
          v = cmul(cmul(tab[(0 * a.nmom + p) * a.Lmax + xx], tab[(1 * a.nmom + p) * a.Lmax + yy]),
                   tab[(2 * a.nmom + p) * a.Lmax + zz]);
        }
        sE[xs][pp] = v;
      }
#pragma unroll
      for (int r = 0; r < NC; r++) {
        const int e = tid + r * kThreads;
        const int xs = e % kXS, kk = e / kXS;
        const int k = k0 + kk, x = xs0 + xs;
        Cx<double> v = czero<double>();
        if (k < a.K && x < xe) v = c[(long long)k * a.sK + x];
        sC[kk][xs ^ (kk & 15)] = v;
      }
    }
    __syncthreads();
    if (kPrefetch && xs0 + kXS < xe) load_step(xs0 + kXS);  // in flight during the products
#pragma unroll 4
    for (int xs = 0; xs < kXS; xs++) {
      Cx<double> ev[kTP], cv[TK];
#pragma unroll
      for (int i = 0; i < kTP; i++) ev[i] = sE[xs][tp + 16 * i];
#pragma unroll
      for (int j = 0; j < TK; j++) cv[j] = sC[tk + 16 * j][xs ^ tk];  // (tk + 16 j) & 15 == tk
      // the two FMAs of each real and imaginary part in separate passes, so
      // that consecutive DFMAs update different accumulators (4 TK of them
      // between an accumulator's dependent pair)
#pragma unroll
      for (int i = 0; i < kTP; i++)
#pragma unroll
        for (int j = 0; j < TK; j++) {
          acc[i][j].x = fma(ev[i].x, cv[j].x, acc[i][j].x);
          acc[i][j].y = fma(ev[i].x, cv[j].y, acc[i][j].y);
        }
#pragma unroll
      for (int i = 0; i < kTP; i++)
#pragma unroll
        for (int j = 0; j < TK; j++) {
          acc[i][j].x = fma(-ev[i].y, cv[j].y, acc[i][j].x);
          acc[i][j].y = fma(ev[i].y, cv[j].x, acc[i][j].y);
        }
    }
    __syncthreads();
  }
  Cx<double>* part = (Cx<double>*)a.part + ((long long)tau * a.nsplit + split) * a.nmom * a.K;
#pragma unroll
  for (int i = 0; i < kTP; i++) {
    const int p = p0 + tp + 16 * i;
    if (p >= a.nmom) continue;
#pragma unroll
    for (int j = 0; j < TK; j++) {
      const int k = k0 + tk + 16 * j;
      if (k < a.K) part[(long long)p * a.K + k] = acc[i][j];
    }
  }
}

__global__ void k_scatter(const ScatterArgs a) {
  const long long n = (long long)a.ntau * a.nmom * a.K;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(i % a.K);
    const int p = (int)((i / a.K) % a.nmom);
    const int tau = (int)(i / ((long long)a.K * a.nmom));
    const Cx<double>* src = (const Cx<double>*)a.part + ((long long)tau * a.nsplit * a.nmom + p) * a.K + k;
    Cx<double> s = czero<double>();
    for (int sp = 0; sp < a.nsplit; sp++) s = s + src[(long long)sp * a.nmom * a.K];
    if (a.nblocks == 0) {
      ((Cx<double>*)a.out)[(long long)(a.tau0 + tau) * a.oT + (long long)k * a.oK + p] = s;
      continue;
    }
    const SliceDesc& sd = a.sl[tau];
    s = cmul(s, source_phase(a.moms + 3 * p, sd.x0, a.L));
    for (int b = 0; b < a.nblocks; b++) {
      const ScatterBlock& B = a.blk[b];
      const int rel = k - B.k0;
      if (rel >= 0 && rel < B.groups * B.datasets * B.comps) {
        const int comp = rel % B.comps;
        const int gd = rel / B.comps;  // group * datasets + dataset
        const long long o = B.base * sd.totalT * a.nmom +
                            (((long long)gd * sd.totalT + sd.tau) * a.nmom + p) * B.comps + comp;
        ((Cx<double>*)sd.out)[o] = s;
      }
    }
  }
}

}  // namespace

int project_fp64_tk(int K, int tk) {
  if (tk == 2 || tk == 4 || tk == 6 || tk == 8) return tk;
  // the component tile (16*TK) that wastes least
  int best = 1 << 30, pick = 8;
  for (int cand : {8, 6, 4, 2}) {
    const int kt = 16 * cand;
    const int waste = ((K + kt - 1) / kt) * kt - K;
    if (waste < best) {
      best = waste;
      pick = cand;
    }
  }
  return pick;
}

cudaError_t launch_project_fp64(const ProjArgs& a, cudaStream_t s) {
  const int tk = project_fp64_tk(a.K, a.tk);
  const int ptiles = (a.nmom + kPT - 1) / kPT;
  const int ktiles = (a.K + 16 * tk - 1) / (16 * tk);
  dim3 grid(ptiles * ktiles, a.nsplit, a.ntau);
  switch (tk) {
    case 2: k_project_fp64<2><<<grid, kThreads, 0, s>>>(a); break;
    case 4: k_project_fp64<4><<<grid, kThreads, 0, s>>>(a); break;
    case 6: k_project_fp64<6><<<grid, kThreads, 0, s>>>(a); break;
    default: k_project_fp64<8><<<grid, kThreads, 0, s>>>(a); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_scatter(const ScatterArgs& a, cudaStream_t s) {
  const long long n = (long long)a.ntau * a.nmom * a.K;
  int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
  if (blocks < 1) blocks = 1;
  k_scatter<<<blocks, 256, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace p2
