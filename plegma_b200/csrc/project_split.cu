// Split-FP16 momentum projection on the tcgen05 tensor cores.
//
// Per time slice the projection C(t,p,k) = sum_x c_k(x,t) exp(-i p.(x-x0))
// is a dense [nmom x V3] . [V3 x K] product (the reference computes it per
// site and momentum with cos/sin and a shared-memory tree,
// lib/kernels/PLEGMA_kernel_utils.cuh:820-860).  Here it runs as a real GEMM
//
//   D[row][n] = sum_x A[row][x] B[n][x]
//   rows: cos(h.x) and sin(h.x) for one representative h of every +-p pair
//         (123 momenta -> 123 rows, one M=128 tile), so each pair costs two
//         real rows instead of two complex rows; the rows have origin 0, so
//         every source shares them and the reduction applies exp(i p.x0);
//   n:    Re and Im of every component (2K columns).
//
// Both operands are split into FP16 hi + lo parts (hi = fp16(v), lo =
// fp16(v - hi)); three products Ah*Bh + Ah*Bl + Al*Bh accumulate in FP32 in
// TMEM.  B is scaled per (slice, component) by 2^(14 - e), e the exponent of
// max |c_k|, so the largest value sits just below 2^14.  The cross-CTA sum
// over site splits and the un-scaling are FP64 (k_split_reduce), in a fixed
// order.
//
// Accumulation precision.  Each tensor-core accumulation step D += A B
// (K = 16) loses about 2^-27 of |D| with a consistent sign (measured on B200:
// the error of a mean-dominated sum grows linearly with the number of MMAs
// accumulated into one TMEM tile, 3e-5 of the sum after ~2600 of them), so
// a k-step range must not accumulate in one TMEM tile.  The products go into
// one of two TMEM tiles D1a / D1b for kPromote k-steps (48 MMAs, <= ~3e-7),
// then the converter warps add that tile into an FP32 sum kept in a third
// TMEM region (CUDA-core adds, round to nearest) while the MMAs fill the
// other tile.  3 x 2NT TMEM columns: NT <= 80.
//
// CTA: 15 converter warps and one copy/MMA warp, one N-tile of NT
// components (2NT TMEM columns), a range of 64-site k-steps.  Per k-step the
// converters load c (coalesced along x, 16 bytes per thread and component),
// split it and store it swizzled into one of two B stages, then each warp
// arrives on the stage's "full" mbarrier; the MMA thread bulk-copies the two
// 16 KB phase tiles (prebuilt in the swizzled layout) one k-step ahead into
// one of three A stages, waits for A and B, issues 3 x 4 (x 2 N-halves)
// tcgen05.mma and commits to the stage's "done" mbarrier, which the
// converters wait for before refilling that stage two k-steps later.  No
// block-wide barrier inside the k-loop.
#include <cuda_fp16.h>

#include <climits>

#include "kernels.cuh"
#include "launch_util.h"
#include "p2_common.cuh"
#include "tc.cuh"

namespace p2 {

namespace {

constexpr int kConvWarps = 15;         // converter warps
constexpr int kThreads = 512;          // + the copy / MMA warp (16 warps; all 16 run the epilogue)
constexpr int kKS = 64;                   // sites per k-step
constexpr int kATile = 128 * kKS * 2;     // bytes of one 128 x 64 FP16 tile
#ifndef P2_PROMOTE_KSTEPS
#define P2_PROMOTE_KSTEPS 4
#endif
constexpr int kPromote = P2_PROMOTE_KSTEPS;  // k-steps accumulated in one TMEM tile before it is added to the sum
constexpr int kMaxNT = 80;                // 3 x 2NT TMEM columns <= 512

__host__ __device__ constexpr int b_tile_bytes(int NT) { return 2 * NT * kKS * 2; }
// Stage counts: B (converted operand) stages let the converters run ahead of
// the MMAs, phase (A) stages let each k-step's phase copy be issued ahead.
// Three A stages where they fit, and three B stages only beside them (N-tiles
// of up to 80 components): measured at 48^3 x 16 with 96-component tiles,
// three A stages beat three B stages (1.01 vs 1.08 ms at 123 momenta).
constexpr int kSmemMax = 232448;
constexpr int kBarBytes = 128;  // mbarriers, TMEM address, error flag
__host__ __device__ constexpr int stage_bytes(int NT, int nb, int na) {
  return nb * 2 * b_tile_bytes(NT) + na * 2 * kATile + kBarBytes + 1024;
}
// Preferred B and A stage counts (a build-time option, taken where they fit
// the shared memory; the mbarrier area holds up to kMaxNB and kMaxNA).  Two B
// and four A stages, the phase copies then two k-steps ahead, measured the
// same as three and three at 48^3 x 96 (6.65 vs 6.64 ms per step).
#ifndef P2_PROJ_NB
#define P2_PROJ_NB 3
#endif
#ifndef P2_PROJ_NA
#define P2_PROJ_NA 3
#endif
constexpr int kMaxNA = 4, kMaxNB = 3;
__host__ __device__ constexpr int b_stages(int NT) {
  return stage_bytes(NT, P2_PROJ_NB, P2_PROJ_NA) <= kSmemMax ? P2_PROJ_NB : stage_bytes(NT, 3, 3) <= kSmemMax ? 3 : 2;
}
__host__ __device__ constexpr int a_stages(int NT) {
  return stage_bytes(NT, P2_PROJ_NB, P2_PROJ_NA) <= kSmemMax ? P2_PROJ_NA
         : stage_bytes(NT, b_stages(NT), 3) <= kSmemMax ? 3 : 2;
}
__host__ __device__ constexpr int smem_bytes(int NT) { return stage_bytes(NT, b_stages(NT), a_stages(NT)); }
// two ping-pong accumulator tiles and the FP32 sum, 2NT columns each
__host__ __device__ constexpr int tmem_cols(int NT) {
  return 6 * NT <= 32 ? 32 : 6 * NT <= 64 ? 64 : 6 * NT <= 128 ? 128 : 6 * NT <= 256 ? 256 : 512;
}

__global__ void k_build_phases(const PhaseBuildArgs a) {
  const long long n = (long long)a.nmtile * a.nkstep * 128 * kKS;
  const Cx<double>* tab = (const Cx<double>*)a.tab;
  __half* A = (__half*)a.A;
  const int LxLy = a.Lx * a.Ly;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int xk = (int)(i % kKS);
    const int row = (int)((i / kKS) % 128);
    const long long ks = (i / (kKS * 128)) % a.nkstep;
    const int mt = (int)(i / ((long long)kKS * 128 * a.nkstep));
    const int r = mt * 128 + row;
    const long long x = ks * kKS + xk;
    double v = 0.0;
    if (r < a.nrows && x < a.V3) {
      const int h = a.row_h[r];
      const int xx = (int)(x % a.Lx), yy = (int)((x / a.Lx) % a.Ly), zz = (int)(x / LxLy);
      const Cx<double> e = cmul(cmul(tab[(0 * a.nh + h) * a.Lmax + xx], tab[(1 * a.nh + h) * a.Lmax + yy]),
                                tab[(2 * a.nh + h) * a.Lmax + zz]);
      v = a.row_sin[r] ? -e.y : e.x;  // e = cos(phi) - i sin(phi)
    }
    const __half hi = __double2half(v);
    const __half lo = __double2half(v - (double)__half2float(hi));
    unsigned char* tile = (unsigned char*)A + ((long long)mt * a.nkstep + ks) * 2 * kATile;
    const uint32_t off = tc::sw128_offset(row, xk);
    *(__half*)(tile + off) = hi;
    *(__half*)(tile + kATile + off) = lo;
  }
}

// Adds accumulator tile D1 (TMEM columns d1col..d1col + NR) into the FP32 sum
// (columns scol..), or copies it when `first`, for the 32 TMEM lanes of this
// warp's quarter: 4-column units j, j + nq, j + 2 nq, ... (warp-uniform).
template <int NR>
__device__ __forceinline__ void drain_tile(uint32_t tbase, int j, int nq, uint32_t d1col, uint32_t scol, bool first) {
  constexpr int NU = NR / 4;
  for (int u0 = j; u0 < NU; u0 += 2 * nq) {
    uint32_t r[16];
#pragma unroll
    for (int q = 0; q < 16; q++) r[q] = 0u;
    const int u1 = u0 + nq;
    tc::tmem_ld4(tbase + d1col + 4 * u0, r);
    if (!first) tc::tmem_ld4(tbase + scol + 4 * u0, r + 4);
    if (u1 < NU) {
      tc::tmem_ld4(tbase + d1col + 4 * u1, r + 8);
      if (!first) tc::tmem_ld4(tbase + scol + 4 * u1, r + 12);
    }
    tc::tmem_wait_ld16(r);
    uint32_t o0[4], o1[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      o0[q] = __float_as_uint(__uint_as_float(r[q]) + __uint_as_float(r[4 + q]));
      o1[q] = __float_as_uint(__uint_as_float(r[8 + q]) + __uint_as_float(r[12 + q]));
    }
    tc::tmem_st4(tbase + scol + 4 * u0, o0);
    if (u1 < NU) tc::tmem_st4(tbase + scol + 4 * u1, o1);
  }
  tc::tmem_wait_st();
}

template <int NT>
__global__ void __launch_bounds__(kThreads, 1) k_project_split(const SplitGemmArgs a) {
  constexpr int NR = 2 * NT;                 // B rows (Re, Im per component)
  constexpr int BT = b_tile_bytes(NT);
  constexpr int NA = a_stages(NT);
  constexpr int NB = b_stages(NT);
  static_assert(NT % 8 == 0 && NT <= kMaxNT, "N-tile width");
  static_assert(NA <= kMaxNA && NB <= kMaxNB && (kMaxNA + 2 * kMaxNB + 4) * 8 + 12 <= kBarBytes, "mbarrier area");
  constexpr uint32_t IDESC = tc::idesc_f16_f32(128, NR);
  constexpr int TCOLS = tmem_cols(NT);
  constexpr int NP = NB > kPromote ? NB : kPromote;  // k-steps per accumulator tile (>= NB: see the drain schedule)
  constexpr int JN = (NT + kConvWarps - 1) / kConvWarps;  // components per converter thread
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // the dynamic window is only guaranteed 16-byte aligned: round up to 1024
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* sA = smem + NB * 2 * BT;  // NA phase stages of 2 kATile (hi, lo) after the NB B stages
  uint64_t* fullA = (uint64_t*)(sA + NA * 2 * kATile);
  uint64_t* done = fullA + kMaxNA;
  uint64_t* fullB = done + kMaxNB;
  uint64_t* d1full = fullB + 3;  // accumulator tile b holds its group's complete sum (MMA commit)
  uint64_t* d1free = d1full + 2;  // accumulator tile b has been added to the sum (converter warps)
  uint32_t* tslot = (uint32_t*)(d1free + 2);
  int* flag = (int*)(tslot + 1);
  int* skipf = flag + 1;  // another CTA of the launch has already failed: do no work

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nti = blockIdx.x % a.ntile, mt = blockIdx.x / a.ntile;
  const int split = blockIdx.y, tau = blockIdx.z;
  const int k0 = nti * NT;
  const int ks0 = split * a.ks_per_split;
  const int nk = min(a.nkstep, ks0 + a.ks_per_split) - ks0;

  if (warp == 0) {
    tc::tmem_alloc(tslot, TCOLS);
    tc::tmem_relinquish();
  }
  if (tid == 0) {
    for (int j = 0; j < NA; j++) tc::mbar_init(&fullA[j], 1);
    for (int j = 0; j < NB; j++) {
      tc::mbar_init(&done[j], 1);
      tc::mbar_init(&fullB[j], kConvWarps);
    }
    for (int j = 0; j < 2; j++) {
      tc::mbar_init(&d1full[j], 1);
      tc::mbar_init(&d1free[j], kConvWarps);
    }
    tc::fence_mbar_init();
    *flag = 0;
    *skipf = *(volatile int*)a.err;
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tslot;
  const long long lim = a.wait_limit > 0 ? a.wait_limit : tc::kWaitLimitNs;
  const bool skip = *skipf != 0;
  const unsigned char* Ab = (const unsigned char*)a.A + (long long)mt * a.nkstep * 2 * kATile;
  bool failed = skip;

  if (skip) {
    // the launch's result is discarded: straight to the epilogue's error path
  } else if (warp == kConvWarps) {
    // ---- copy / MMA warp: lane 0 ----
    if (lane == 0 && nk > 0) {
      int issued = -1, committed = -1;
      // the phase tiles are re-read by every N-tile, slice and site split:
      // they stay in L2 ahead of the position buffer streamed past them
      const uint64_t keep_policy = tc::policy_evict_last();
      auto issue_a = [&](int i) {  // phase tiles of k-step i into A stage i % NA
        const int sa = i % NA;
        tc::mbar_expect_tx(&fullA[sa], 2 * kATile);
        tc::bulk_g2s_hint(sA + sa * 2 * kATile, Ab + (long long)(ks0 + i) * 2 * kATile, 2 * kATile, &fullA[sa],
                          keep_policy);
        issued = i;
      };
      issue_a(0);
      for (int i = 0; i < nk && !failed; i++) {
        // the phase copies up to k-step i + NA - 2 (NA - 2 k-steps ahead; this
        // k-step with two stages); the copy of k-step j reuses the stage of
        // k-step j - NA <= i - 2, whose MMAs must be complete
        const int next = min(i + NA - 2, nk - 1);
        while (issued < next) {
          const int j = issued + 1;
          if (j >= NA && !tc::mbar_wait(&done[(j - NA) % NB], ((j - NA) / NB) & 1, lim)) {
            failed = true;
            break;
          }
          issue_a(j);
        }
        if (failed) break;
        const int s = i % NB;
        const int grp = i / NP, b = grp & 1;
        // the first k-step of a group reuses accumulator tile b: the converters
        // must have added group grp - 2 into the sum
        if (i % NP == 0 && grp >= 2 && !tc::mbar_wait(&d1free[b], ((grp >> 1) - 1) & 1, lim)) {
          failed = true;
          break;
        }
        if (!tc::mbar_wait(&fullA[i % NA], (i / NA) & 1, lim) || !tc::mbar_wait(&fullB[s], (i / NB) & 1, lim)) {
          failed = true;
          break;
        }
        tc::tc_fence_after();
        const uint32_t a_hi = tc::smem_u32(sA + (i % NA) * 2 * kATile), a_lo = a_hi + kATile;
        const uint32_t b_hi = tc::smem_u32(smem + s * 2 * BT), b_lo = b_hi + BT;
        const uint32_t d1 = tmem + (uint32_t)(b * NR);
#pragma unroll
        for (int kk = 0; kk < kKS / 16; kk++) {
#pragma unroll
          for (int prod = 0; prod < 3; prod++) {
            const uint32_t aa = (prod == 2 ? a_lo : a_hi) + kk * 32;
            const uint32_t bb = (prod == 1 ? b_lo : b_hi) + kk * 32;
            const uint32_t acc = (i % NP > 0 || kk > 0 || prod > 0) ? 1u : 0u;
            tc::mma_f16(d1, tc::desc_sw128(aa), tc::desc_sw128(bb), IDESC, acc);
          }
        }
        tc::mma_commit(&done[s]);
        if (i % NP == NP - 1 || i == nk - 1) tc::mma_commit(&d1full[b]);
        committed = i;
      }
      // the accumulators are complete (or, after a failure, no MMA or phase
      // copy is still in flight) before the block moves on
      if (committed >= 0 && !tc::mbar_wait(&done[committed % NB], (committed / NB) & 1, lim)) failed = true;
      if (failed) {
        *flag = 1;
        for (int j = max(0, issued - NA + 1); j <= issued; j++)
          tc::mbar_wait(&fullA[j % NA], (j / NA) & 1, 100000000LL);  // in-flight copies: 0.1 s
      }
    }
    __syncwarp();
  } else {
    // ---- converters: site pair sp (sites 2sp, 2sp+1 of the k-step), components kg + 15 j ----
    const int sp = tid & 31, kg = tid >> 5;
    float sc[JN];
#pragma unroll
    for (int j = 0; j < JN; j++) {
      const int k = k0 + kg + kConvWarps * j;
      sc[j] = 0.f;
      if (kg + kConvWarps * j < NT && k < a.K) {
        const float mx = __int_as_float(a.cmax[(long long)tau * a.K + k]);
        int e = 0;
        if (mx > 0.f) frexpf(mx, &e);
        sc[j] = ldexpf(1.f, 14 - e);
      }
    }
    const Cx<float>* cb = (const Cx<float>*)a.c + (long long)tau * a.K * a.V3;
    const bool even = (a.V3 & 1) == 0;  // site pairs 16-byte aligned
    // swizzled byte offsets of this thread's (component, site pair) in a B
    // tile, fixed over the k-steps: the Re row 2 kk at
    //   256 kk + 16 ((sp >> 2) ^ 2 (kk & 3)) + 4 (sp & 3)   (tc::sw128_offset(2 kk, 2 sp)),
    // the Im row 2 kk + 1 a fixed 128 +- 16 bytes further
    uint32_t boff[JN];
#pragma unroll
    for (int j = 0; j < JN; j++) boff[j] = tc::sw128_offset(2 * (kg + kConvWarps * j), 2 * sp);
    const uint32_t dim = tc::sw128_offset(1, 2 * sp) - tc::sw128_offset(0, 2 * sp);
    // B values of two consecutive k-steps (register double buffer, the two
    // halves swapping roles every k-step: the loads of step i + 1 stay in
    // flight while step i is split)
    float4 b0[JN], b1[JN];
    // components this thread converts (bit j: component k0 + kg + 15 j exists)
    unsigned jok = 0;
#pragma unroll
    for (int j = 0; j < JN; j++)
      if (kg + kConvWarps * j < NT && k0 + kg + kConvWarps * j < a.K) jok |= 1u << j;
    const Cx<float>* cthr = cb + (long long)(k0 + kg) * a.V3 + 2 * sp;
    const long long cstride = (long long)kConvWarps * a.V3;
    const uint64_t stream_policy = tc::policy_evict_first();  // the position buffer is read once
    auto load_b = [&](int ks, float4 (&r)[JN]) {
      const long long x = (long long)ks * kKS + 2 * sp;
      const Cx<float>* cks = cthr + (long long)ks * kKS;
#pragma unroll
      for (int j = 0; j < JN; j++) {
        r[j] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (((jok >> j) & 1u) && x < a.V3) {
          const Cx<float>* src = cks + j * cstride;
          if (even) {
            r[j] = tc::ld_stream_f4(src, stream_policy);
          } else {
            r[j].x = src[0].x;
            r[j].y = src[0].y;
            if (x + 1 < a.V3) {
              r[j].z = src[1].x;
              r[j].w = src[1].y;
            }
          }
        }
      }
    };
    // one k-step; returns true when a wait timed out
    auto step = [&](int i, const float4 (&cur)[JN], float4 (&nxt)[JN]) -> bool {
      const int s = i % NB;
      if (i + 1 < nk) load_b(ks0 + i + 1, nxt);
      if (i >= NB && !tc::mbar_wait(&done[s], ((i / NB) - 1) & 1, lim)) return true;
      unsigned char* Bh = smem + s * 2 * BT;
      unsigned char* Bl = Bh + BT;
#pragma unroll
      for (int j = 0; j < JN; j++) {
        const int kk = kg + kConvWarps * j;
        if (kk >= NT) break;
        const float4 v = cur[j];
        const float r0 = v.x * sc[j], i0 = v.y * sc[j], r1 = v.z * sc[j], i1 = v.w * sc[j];
        const __half2 hr = __floats2half2_rn(r0, r1);
        const __half2 hi_ = __floats2half2_rn(i0, i1);
        const float2 fr = __half22float2(hr), fi = __half22float2(hi_);
        const __half2 lr = __floats2half2_rn(r0 - fr.x, r1 - fr.y);
        const __half2 li = __floats2half2_rn(i0 - fi.x, i1 - fi.y);
        const uint32_t ore = boff[j];
        const uint32_t oim = ore + dim;
        *(__half2*)(Bh + ore) = hr;
        *(__half2*)(Bh + oim) = hi_;
        *(__half2*)(Bl + ore) = lr;
        *(__half2*)(Bl + oim) = li;
      }
      tc::fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0 && !a.withhold) tc::mbar_arrive(&fullB[s]);
      return false;
    };
    // accumulator tile of group g (k-steps g NP .. g NP + NP - 1) into the
    // sum: converter warp w serves TMEM lane quarter w % 4 (warp 15, the MMA
    // warp, leaves quarter 3 to three converter warps)
    const int quarter = warp & 3, qj = warp >> 2, nq = quarter == 3 ? 3 : 4;
    const uint32_t tbase = tmem + ((uint32_t)(32 * quarter) << 16);
    int drained = 0;  // groups added to the sum so far
    auto drain = [&](int g) -> bool {
      const int b = g & 1;
      if (!tc::mbar_wait(&d1full[b], (g >> 1) & 1, lim)) return true;
      tc::tc_fence_after();
      drain_tile<NR>(tbase, qj, nq, (uint32_t)(b * NR), (uint32_t)(2 * NR), g == 0);
      tc::tc_fence_before();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&d1free[b]);
      drained = g + 1;
      return false;
    };
    if (nk > 0) load_b(ks0, b0);
    // the drain of group g comes before the converters wait for the MMAs of
    // k-step (g + 1) NP (converter step (g + 1) NP + NB), which need tile g+1's
    // predecessor drained; NP >= NB keeps the MMAs of group g + 2 from waiting
    // on it
    auto drain_due = [&](int i) -> bool {
      const int r = i - NB;
      return r >= NP && r % NP == 0 && drain(r / NP - 1);
    };
    for (int i = 0; i < nk; i += 2) {
      if (*(volatile int*)flag || drain_due(i) || step(i, b0, b1) ||
          (i + 1 < nk && (drain_due(i + 1) || step(i + 1, b1, b0)))) {
        failed = true;
        break;
      }
    }
    const int ngroups = (nk + NP - 1) / NP;
    while (!failed && drained < ngroups)
      if (drain(drained)) failed = true;
  }
  failed = __syncthreads_or(failed || *(volatile int*)flag);
  if (failed) {
    if (tid == 0) atomicExch(a.err, 1);
  } else {
    tc::tc_fence_after();
    // epilogue: warps w, w+4, w+8, w+12 share TMEM lanes 32*(w%4)..; 16-column
    // chunks are dealt round-robin among them
    const int row = 32 * (warp & 3) + lane;
    float* dst = a.part + ((((long long)tau * a.nsplit + split) * a.nmtile + mt) * 128 + row) * (long long)(a.ntile * NR) +
                 nti * NR;
#pragma unroll 1
    for (int c = (warp >> 2) * 16; c < NR; c += 64) {
      float v[16];
      tc::tmem_ld16(tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(2 * NR + c), v);
      float4* d4 = (float4*)(dst + c);
#pragma unroll
      for (int q = 0; q < 4; q++) d4[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, TCOLS);
}

// One thread per (slice, representative h, component): the cos and sin rows'
// partials of h are summed over the site splits once, in a fixed order, and
// give every momentum of h (+h and -h) its value.
__global__ void k_split_reduce(const SplitReduceArgs a) {
  const long long n = (long long)a.ntau * a.nrep * a.K;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(i % a.K);
    const int h = (int)((i / a.K) % a.nrep);
    const int tl = (int)(i / ((long long)a.K * a.nrep));
    const int j0 = a.rep_start[h], j1 = a.rep_start[h + 1];
    if (j0 == j1) continue;
    const int* mr0 = a.mom_row + 6 * a.rep_moms[j0];
    const int rc = mr0[0], rs = mr0[1];
    const int col = (k / a.NT) * 2 * a.NT + 2 * (k % a.NT);
    double cr = 0, ci = 0, sr = 0, si = 0;
    // fixed order over the splits; unrolled so that several splits' loads are in flight
#pragma unroll 4
    for (int sp = 0; sp < a.nsplit; sp++) {
      const float* base = a.part + ((long long)tl * a.nsplit + sp) * a.nmtile * 128 * (long long)a.ncols;
      const float* pc = base + (long long)rc * a.ncols + col;
      cr += (double)pc[0];
      ci += (double)pc[1];
      if (rs >= 0) {
        const float* ps = base + (long long)rs * a.ncols + col;
        sr += (double)ps[0];
        si += (double)ps[1];
      }
    }
    const float mx = __int_as_float(a.cmax[(long long)tl * a.K + k]);
    int e = 0;
    if (mx > 0.f) frexpf(mx, &e);
    const SliceDesc& sd = a.sl[tl];
    const int pw = a.kexp[2 * k] * (a.exps[2 * tl] + sd.eh[0]) + a.kexp[2 * k + 1] * (a.exps[2 * tl + 1] + sd.eh[1]) -
                   (14 - e);
    const double f = ldexp(1.0, pw);
    for (int j = j0; j < j1; j++) {
      const int p = a.rep_moms[j];
      const int* mr = a.mom_row + 6 * p;
      const int sg = mr[2];
      // S(p) = sum_x c e^{-i p.x}; the source phase: C(p) = e^{i p.x0} S(p), with
      // p.x0 / L reduced exactly in integers per dimension
      Cx<double> v = cmul(cx<double>((cr + sg * si) * f, (ci - sg * sr) * f), source_phase(mr + 3, sd.x0, a.L));
      if (a.kphase) {
        const int q = a.kphase[k];
        if (q & 1) v = cx<double>(-v.y, v.x);
        if (q & 2) v = cx<double>(-v.x, -v.y);
      }
      if (a.nblocks == 0) ((Cx<double>*)a.out)[(long long)sd.tau * a.oT + (long long)k * a.oK + p] = v;
      for (int b = 0; b < a.nblocks; b++) {
        const ScatterBlock& B = a.blk[b];
        const int rel = k - B.k0;
        if (rel >= 0 && rel < B.groups * B.datasets * B.comps) {
          const int comp = rel % B.comps;
          const int gd = rel / B.comps;
          const long long o = B.base * sd.totalT * a.nmom +
                              (((long long)gd * sd.totalT + sd.tau) * a.nmom + p) * B.comps + comp;
          ((Cx<double>*)sd.out)[o] = v;
        }
      }
    }
  }
}

// C[g1][g2] = sum_{d, b} G1[d][pi1(d)] G2[b][pi2(b)] M_{pi1(d) d}[b][pi2(b)]
// (PLEGMA_mesonsAll.cuh:58-76 with the spin sums moved after the projection:
// the Gamma sums are linear).  One block per (momentum, slice): the 256
// projected colour products of the 16 x 16 block are read into shared memory
// and replaced in place by the 256 C[g1][g2], component 16 g1 + g2.
__constant__ int c_gperm[16][4] = P2_INIT_GammaPerm;
__constant__ int c_gre[16][4] = P2_INIT_GammaRe;
__constant__ int c_gim[16][4] = P2_INIT_GammaIm;

__global__ void __launch_bounds__(256) k_meson_gamma(const MesonGammaArgs a) {
  __shared__ Cx<double> sm[256];
  const int p = blockIdx.x, tl = blockIdx.y, j = threadIdx.x;
  const SliceDesc& sd = a.sl[tl];
  Cx<double>* v = (Cx<double>*)sd.out + a.blk.base * sd.totalT * a.nmom + ((long long)sd.tau * a.nmom + p) * 256;
  sm[j] = v[j];
  __syncthreads();
  const int g1 = j >> 4, g2 = j & 15;
  Cx<double> acc = czero<double>();
#pragma unroll
  for (int d = 0; d < 4; d++) {
    const int al = c_gperm[g1][d];
    const Cx<double> v1 = cx<double>((double)c_gre[g1][d], (double)c_gim[g1][d]);
#pragma unroll
    for (int b = 0; b < 4; b++) {
      const int z = c_gperm[g2][b];
      const Cx<double> v2 = cx<double>((double)c_gre[g2][b], (double)c_gim[g2][b]);
      cmac(acc, cmul(v1, v2), sm[16 * (4 * al + d) + 4 * b + z]);
    }
  }
  v[j] = acc;
}

template <int NT>
cudaError_t launch_nt(const SplitGemmArgs& a, cudaStream_t s) {
  const int smem = smem_bytes(NT);
  cudaError_t e = ensure_smem((const void*)k_project_split<NT>, smem);
  if (e != cudaSuccess) return e;
  dim3 grid(a.ntile * a.nmtile, a.nsplit, a.ntau);
  k_project_split<NT><<<grid, kThreads, smem, s>>>(a);
  return cudaGetLastError();
}

}  // namespace

int project_split_max_nt() { return kMaxNT; }

int project_split_smem_bytes(int NT) { return smem_bytes(NT < 8 ? 8 : NT > kMaxNT ? kMaxNT : (NT + 7) / 8 * 8); }

cudaError_t launch_build_phases(const PhaseBuildArgs& a, cudaStream_t s) {
  const long long n = (long long)a.nmtile * a.nkstep * 128 * kKS;
  const int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 32);
  k_build_phases<<<blocks, 256, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_project_split(const SplitGemmArgs& a, cudaStream_t s) {
  static_assert(kMaxNT == 80, "instantiations below");
  switch (a.NT) {
    case 8: return launch_nt<8>(a, s);
    case 16: return launch_nt<16>(a, s);
    case 24: return launch_nt<24>(a, s);
    case 32: return launch_nt<32>(a, s);
    case 40: return launch_nt<40>(a, s);
    case 48: return launch_nt<48>(a, s);
    case 56: return launch_nt<56>(a, s);
    case 64: return launch_nt<64>(a, s);
    case 72: return launch_nt<72>(a, s);
    case 80: return launch_nt<80>(a, s);
    default: return cudaErrorInvalidValue;
  }
}

namespace {

// Blocks map to (component k, slice, site range): each reduces its range in
// shared memory and issues one atomic.
// Pass 1: binary exponent of the largest |Re|, |Im| of every slice.
__global__ void k_field_exponent(const FieldF32Args a, int xchunk) {
  __shared__ int red[256];
  const int k = blockIdx.x, tl = blockIdx.y;
  const long long x0 = (long long)blockIdx.z * xchunk, x1 = min((long long)a.V3, x0 + xchunk);
  const double2* row = (const double2*)a.field + (long long)k * a.vol + (long long)(a.t0 + tl) * a.V3;
  int emax = -100000;
  for (long long x = x0 + threadIdx.x; x < x1; x += blockDim.x) {
    const double2 v = row[x];
    int e;
    if (v.x != 0.0) {
      frexp(v.x, &e);
      emax = max(emax, e);
    }
    if (v.y != 0.0) {
      frexp(v.y, &e);
      emax = max(emax, e);
    }
  }
  red[threadIdx.x] = emax;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = max(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0 && red[0] != -100000) atomicMax(a.exps + 2 * tl, red[0]);
}

// Pass 2: the FP32 copy times 2^-E of its slice (exact) and the per-component maxima.
__global__ void k_field_to_f32(const FieldF32Args a, int xchunk) {
  __shared__ float red[256];
  const int k = blockIdx.x, tl = blockIdx.y;
  const long long x0 = (long long)blockIdx.z * xchunk, x1 = min((long long)a.V3, x0 + xchunk);
  const double2* row = (const double2*)a.field + (long long)k * a.vol + (long long)(a.t0 + tl) * a.V3;
  float2* dst = (float2*)a.c + ((long long)tl * a.K + k) * a.V3;
  const double sc = ldexp(1.0, -a.exps[2 * tl]);
  float m = 0.f;
  for (long long x = x0 + threadIdx.x; x < x1; x += blockDim.x) {
    const double2 v = row[x];
    const float2 f = make_float2((float)(v.x * sc), (float)(v.y * sc));
    dst[x] = f;
    m = fmaxf(m, fmaxf(fabsf(f.x), fabsf(f.y)));
  }
  red[threadIdx.x] = m;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = fmaxf(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicMax(a.cmax + (long long)tl * a.K + k, __float_as_int(red[0]));
}

// exponents before pass 1 (INT_MIN: none seen yet) and after it (an all-zero slice keeps scale 1)
__global__ void k_field_exps_init(int* exps, int ntau) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < ntau) {
    exps[2 * t] = INT_MIN;
    exps[2 * t + 1] = 0;
  }
}
__global__ void k_field_exps_zero(int* exps, int ntau) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < ntau && exps[2 * t] == INT_MIN) exps[2 * t] = 0;
}

}  // namespace

cudaError_t launch_field_to_f32(const FieldF32Args& a, int nsm, cudaStream_t s) {
  const int tb = (a.ntau + 255) / 256;
  k_field_exps_init<<<tb, 256, 0, s>>>(a.exps, a.ntau);
  cudaError_t e = cudaMemsetAsync(a.cmax, 0, (size_t)a.ntau * a.K * sizeof(int), s);
  if (e != cudaSuccess) return e;
  const long long rows = (long long)a.K * a.ntau;
  const int nx = (int)std::max<long long>(1, std::min<long long>((a.V3 + 4095) / 4096, (8LL * nsm + rows - 1) / rows));
  const int xchunk = (int)((a.V3 + nx - 1) / nx);
  const dim3 grid(a.K, a.ntau, nx);
  k_field_exponent<<<grid, 256, 0, s>>>(a, xchunk);
  k_field_exps_zero<<<tb, 256, 0, s>>>(a.exps, a.ntau);
  k_field_to_f32<<<grid, 256, 0, s>>>(a, xchunk);
  return cudaGetLastError();
}

cudaError_t launch_meson_gamma(const MesonGammaArgs& a, cudaStream_t s) {
  if (a.ntau < 1 || a.nmom < 1) return cudaSuccess;
  k_meson_gamma<<<dim3(a.nmom, a.ntau), 256, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_split_reduce(const SplitReduceArgs& a, cudaStream_t s) {
  const long long n = (long long)a.ntau * a.nrep * a.K;
  int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
  if (blocks < 1) blocks = 1;
  k_split_reduce<<<blocks, 256, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace p2
