// Site contraction kernels: propagators staged through shared memory, one
// site per half-warp, results written to a position-space buffer that the
// projection kernels consume.
//
// Replaces the per-site part of contract_baryons_device / contract_NtoN_kernel
// (lib/kernels/PLEGMA_baryons.cuh:31-96, PLEGMA_baryons_NtoN.cu:6-46) and
// contract_mesons_{all,new,}_device (PLEGMA_mesonsAll.cuh:7-95,
// PLEGMA_mesonsNew.cuh:5-56, PLEGMA_mesons.cuh:10-65).
//
// Two instantiations:
//  - plain:  FP64 propagators, FP64 arithmetic, complex-double output;
//  - split:  FP64 or FP32 propagators multiplied by 2^-E(slice, flavour)
//            (exact power-of-two scaling, so correlators that fall over ten
//            decades in t stay inside FP32's range), FP32 arithmetic,
//            complex-float output, plus max(|Re|,|Im|) per (slice, component)
//            for the FP16 split of the projection.
//
// Layout and schedule
//  - a CTA of 256 threads is persistent over tiles of 16 consecutive sites of
//    one time slice (tile = (tau, x0));
//  - each tile's 2 x 144 complex per site are copied with cp.async, coalesced
//    along the site axis of the SoA propagator, into shared memory as
//    [site][flavour*144 + component] (row padded to 289 complex);
//  - two stages: tile i+1's copies are in flight while tile i is contracted;
//  - half-warp h contracts site h of the tile (site_contract.cuh);
//  - split form: the tile is converted once into padded FP32 rows (component-
//    major staging, one buffer), and the 16 x 16 meson outputs go back through
//    the sites' rows to a tile-wide flush that writes 128-byte component rows;
//    when nothing else needs the lanes' Gamma stages (g16_raw) the outputs are
//    the colour-traced products M themselves and the Gamma sums run after the
//    projection.
#include "kernels.cuh"
#include "launch_util.h"
#include "site_contract.cuh"

namespace p2 {

namespace {

constexpr int kThreads = 256;
constexpr int kSitesPerTile = 16;
constexpr int kRow = 289;  // complex per site row (2 * 144 + 1 pad)
constexpr int kStage = kSitesPerTile * kRow;

// CM = false: site-major [site][kRow] (the plain kernel reads it directly);
// CM = true: component-major [flavour * 144 + component][16 sites], written
// without bank conflicts and transposed by the split kernel's conversion.
// Only the staging rows 144 f + component in [lo, hi) are copied (component-
// major staging; the site-major one always copies all).
template <typename Tin, bool CM = false>
__device__ __forceinline__ void issue_tile(const ContractArgs& a, Cx<Tin>* st, int tl, int x0, bool valid, int lo = 0,
                                           int hi = 288) {
  if (valid) {
    const int s = threadIdx.x & (kSitesPerTile - 1);
    const int x = x0 + s;
    const bool ok = x < a.V3;
    const SliceDesc* sd = a.sl + tl;
    // thread i copies component i/16 + 16 r of site i%16; with 256 threads
    // rows r < 9 are the u view's 144 components and r >= 9 the d view's
#pragma unroll
    for (int f = 0; f < 2; f++) {
      const long long vol = f ? sd->vol_d : sd->vol_u;
      const Cx<Tin>* src = (const Cx<Tin>*)(f ? sd->d : sd->u) + (f ? sd->off_d : sd->off_u) + (ok ? x : 0) +
                           (threadIdx.x >> 4) * vol;
      const long long step = 16 * vol;
#pragma unroll 3
      for (int r = 0; r < 9; r++) {
        const int comp = (threadIdx.x >> 4) + 16 * r;
        Cx<Tin>* dst = CM ? st + (144 * f + comp) * kSitesPerTile + s : st + s * kRow + 144 * f + comp;
        if (!CM || (144 * f + comp >= lo && 144 * f + comp < hi)) {
          if (sizeof(Tin) == 8)
            cp_async16(dst, src, ok ? 16 : 0);
          else
            cp_async8(dst, src, ok ? 8 : 0);
        }
        src += step;
      }
    }
  }
  cp_async_commit();
}

static_assert(kThreads == 256 && kSitesPerTile == 16, "issue_tile maps 256 threads onto 16 sites x 16 components");

// Index of a diagonal structure in the 10-structure list (1, g5, g1..g4,
// g5g1..g5g4) of contractMesons / contractMesonsNew, or -1.
__device__ __forceinline__ int diag10_slot(int g) {
  return g == 0 ? 0 : g == 5 ? 1 : (g >= 1 && g <= 4) ? g + 1 : (g >= 6 && g <= 9) ? g : -1;
}

// Split form: the per-component maxima of the current slice live in the spare
// slot of each FP32 tile block position (row s, position j holds components
// 2 (32 s + j) and 2 (32 s + j) + 1), which no load of the contraction reads,
// whichever block the position holds.
__device__ __forceinline__ int* smax_slot(Cx<float>* sf, int k) {
  const int p = k >> 1, s = p >> 5, j = p & 31;
  return reinterpret_cast<int*>(sf + s * kRow32 + 2 * row32_unit(j, 4) + 1) + (k & 1);
}

// Split form, 16 x 16 mesons: a half-warp reads only its own site's FP32 row,
// so once its contraction is done it stages the site's 256 outputs in that
// row (C[g1][g2] of lane g1, or with g16_raw the products M_{a d}[b][z] of lane
// l = 4 a + d in the slot of g1 = l, g2 = 4 b + z), in the eight data
// complex (units 0-3) of the row's 32 block positions (the colour-8 and spare
// slots keep their contents, the spare slots holding the per-component
// maxima).  The 16 outputs of one g2 go to positions b1 (g1 < 8) and b1 + 4
// (g1 >= 8), b1 = 8 (g2 >> 2) + (g2 & 3): their eight 16-byte units lie in
// eight different bank groups (4 positions = 20 units = 4 mod 8), and those
// of the warp's other site, whose row starts 161 units further, in the same
// eight shifted by one, so a warp-wide store takes the minimum two
// wavefronts.  The flush after the tile writes them to HBM, 128 contiguous
// bytes per component; direct stores from the lanes would touch 16 component
// rows per instruction.  The staging buffer stays free for the whole next
// tile's copies.
__device__ __forceinline__ int g16_slot(int g1, int g2) {
  const int pos = 8 * (g2 >> 2) + (g2 & 3) + 4 * (g1 >> 3);
  return 10 * pos + (g1 & 7);
}
// The nucleon's 32 outputs of a site staged beside them: component c in the
// colour-8 complex of block position c (complex 10 c + 8).
__device__ __forceinline__ int nuc_slot(int c) { return 10 * c + 8; }

// STG: the Delta outputs go to the tile's output staging (a compile-time
// choice: a run-time branch in the output path costs the Delta code ~3 %).
template <typename R, bool STG = false>
struct Writer {
  Cx<R>* out;
  long long V3;
  float* rmax;          // split form: this lane's running maxima of its nucleon outputs (slots 0, 1)
  Cx<float>* smax_base;  // split form: tile whose spare slots hold the per-component maxima, or null
  Cx<R>* g16;           // split form: this site's FP32 row, reused as its 16 x 16 meson staging (Delta
                        // instantiation: the tile's output staging); or null
  int h;                // the site's index in the tile (Delta output staging)
  __device__ __forceinline__ void put(int k, Cx<R> v) const {
    out[(long long)k * V3] = v;
    if (smax_base) {
      const float m = fmaxf(fabsf((float)v.x), fabsf((float)v.y));
      atomicMax(smax_slot(smax_base, k), __float_as_int(m));
    }
  }
  // Outputs whose component is fixed per lane: the maximum stays in a register
  // (slot) and reaches shared memory once per time slice.
  __device__ __forceinline__ void put_slot(int k, Cx<R> v, int slot) const {
    out[(long long)k * V3] = v;
    note_slot(v, slot);
  }
  // Delta instantiation: output row r of the tile's staging ([row][16 sites],
  // the site index XOR-swizzled by the row so that the 16 lanes of a store,
  // rows r0 + l, hit 16 different bank pairs), or component k straight to HBM
  // with its maximum
  __device__ __forceinline__ void dput(int r, int k, Cx<R> v) const {
    if constexpr (STG)
      g16[r * 16 + (h ^ (r & 15))] = v;
    else
      put(k, v);
  }
  // the maximum only (the value leaves through the staged flush)
  __device__ __forceinline__ void note_slot(Cx<R> v, int slot) const {
    if (rmax) rmax[slot] = fmaxf(rmax[slot], fmaxf(fabsf((float)v.x), fabsf((float)v.y)));
  }
};

// DELTA selects the instantiation: the Delta blocks and the second nucleon
// interpolator (true) or every other block (false); a request with both runs
// the two instantiations over the same tiles (the Delta part is ~5x the rest
// in arithmetic, so the second pass over the propagators is hidden under its
// compute).
template <bool DELTA, typename Row, typename W>
__device__ __forceinline__ void contract_site(const ContractArgs& a, const Row& row, const LaneTables& lt, int l,
                                              unsigned mask, const W& w) {
  typedef typename Row::R R;
  if (DELTA && (a.what & (128u | 256u | 512u))) {
    const int base[3] = {a.k.ntor, a.k.rton, a.k.rtor};
    light_nucleon_site(row, lt, l, mask, (a.what & 128u) != 0, (a.what & 256u) != 0, (a.what & 512u) != 0,
                       [&](int j, int ds, Cx<R> v) { w.put(base[j] + 16 * ds + l, v); });
  }
  if (DELTA && (a.what & (2u | 4u))) {
    // group g of each isospin block, datasets (u-rich, d-rich); the iso-1/2
    // partial sums of G^{ud} wait in a per-thread array (local memory, L1)
    // until the G^{uu} / G^{dd} terms complete them
    Cx<R> parked[3][2];
    delta_site(
        row, lt, l, mask,
        [&](int g, int j, Cx<R> v) {
          // staging rows: iso-1/2 0..95, iso-3/2 96..191
          if (j < 2 && (a.what & 2u)) w.dput((g * 2 + j) * 16 + l, a.k.diso12 + (g * 2 + j) * 16 + l, v);
          if (j >= 2 && (a.what & 4u)) w.dput(96 + (g * 2 + j - 2) * 16 + l, a.k.diso32 + (g * 2 + j - 2) * 16 + l, v);
        },
        [&](int g, int j, Cx<R> v) { parked[g][j] = v; }, [&](int g, int j) { return parked[g][j]; });
  }
  if (DELTA) return;
  // nucleon outputs: with staged 16 x 16 mesons they wait in registers until
  // the mesons have read the row, then go to its colour-8 slots and out
  // through the flush with the mesons (128-byte component rows instead of 16
  // scattered 16-byte segments per warp-wide store)
  const bool nuc = (a.what & 1u) != 0;
  Cx<R> pn[2];
  if (nuc) {
    nucleon_site(row, lt, l, mask, pn);
    if (w.g16) {
      w.note_slot(pn[0], 0);
      w.note_slot(pn[1], 1);
    } else {
      w.put_slot(a.k.nuc + l, pn[0], 0);
      w.put_slot(a.k.nuc + 16 + l, pn[1], 1);
    }
  }
  auto stage_nucleon = [&]() {
    if (nuc) {
      w.g16[nuc_slot(l)] = pn[0];
      w.g16[nuc_slot(16 + l)] = pn[1];
    }
  };
  const int g1 = lt.meson_g1();  // the sink Gamma of this lane's meson outputs
  if (a.g16_raw) {
    // the colour-traced products M_{al de}[b][z] of lane (al, de): no Gamma
    // stage here, k_meson_gamma forms the Gamma sums after the projection
    Cx<R> M[4][4];
    meson_M(row, kU, kD, l >> 2, l & 3, M);
    if (w.g16) {
      __syncwarp(mask);  // every lane of the half-warp has finished reading the row
#pragma unroll
      for (int b = 0; b < 4; b++)
#pragma unroll
        for (int z = 0; z < 4; z++) w.g16[g16_slot(l, 4 * b + z)] = M[b][z];
      stage_nucleon();
    } else {
#pragma unroll
      for (int b = 0; b < 4; b++)
#pragma unroll
        for (int z = 0; z < 4; z++) w.put(a.k.g16 + 16 * l + 4 * b + z, M[b][z]);
    }
  } else if (a.what & (8u | 16u | 32u)) {
    Cx<R> c[16];
    // staged 16 x 16 outputs leave their unit phases r_g1 r_g2 to the
    // projection's reduction (g16_phase_deferred); the other blocks get them here
    const bool phased = w.g16 == nullptr;
    meson_site(row, kU, kD, lt, l, mask, true, phased, c);
    auto val = [&](int g2) { return phased ? c[g2] : meson_phase(lt, g2, c[g2]); };
    if (a.what & 8u) {
      if (w.g16) {
        __syncwarp(mask);  // every lane of the half-warp has finished reading the row
#pragma unroll
        for (int g2 = 0; g2 < 16; g2++) w.g16[g16_slot(g1, g2)] = c[g2];
        stage_nucleon();
      } else {  // direct stores (plain form, or split form with the 10 diagonal structures: maxima in shared memory)
#pragma unroll
        for (int g2 = 0; g2 < 16; g2++) w.put(a.k.g16 + g1 * 16 + g2, c[g2]);
      }
    }
    if (a.what & 16u) {
      if (g1 == 0) w.put(a.k.all34 + 0, val(0));
      if (g1 == 5) w.put(a.k.all34 + 1, val(5));
      if (g1 >= 1 && g1 <= 4) {
#pragma unroll
        for (int g2 = 1; g2 <= 4; g2++) w.put(a.k.all34 + 2 + (g1 - 1) * 4 + (g2 - 1), val(g2));
      }
      if (g1 >= 6 && g1 <= 9) {
#pragma unroll
        for (int g2 = 6; g2 <= 9; g2++) w.put(a.k.all34 + 18 + (g1 - 6) * 4 + (g2 - 6), val(g2));
      }
    }
    if (a.what & 32u) {
      const int j = diag10_slot(g1);
#pragma unroll
      for (int g2 = 0; g2 < 16; g2++)
        if (g2 == g1 && j >= 0) w.put(a.k.new10 + j, val(g2));
    }
  }
  if (a.what & 64u) {
    const int j = diag10_slot(g1);
    Cx<R> c[16];
    meson_site(row, kU, kU, lt, l, mask, true, true, c);
#pragma unroll
    for (int g2 = 0; g2 < 16; g2++)
      if (g2 == g1 && j >= 0) w.put(a.k.diag10 + j, c[g2]);
    meson_site(row, kD, kD, lt, l, mask, true, true, c);
#pragma unroll
    for (int g2 = 0; g2 < 16; g2++)
      if (g2 == g1 && j >= 0) w.put(a.k.diag10 + 10 + j, c[g2]);
  }
}

// Plain FP64 form.
template <bool DELTA>
__global__ void __launch_bounds__(kThreads, 1) k_contract_plain(const ContractArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cx<double>* sm = (Cx<double>*)smem_raw;
  const int tid = threadIdx.x;
  const int hw = tid >> 4, l = tid & 15;
  const unsigned mask = halfwarp_mask();
  const LaneTables lt = load_lane_tables(l);

  const int tiles_per_tau = (a.V3 + kSitesPerTile - 1) / kSitesPerTile;
  TileCursor cur(blockIdx.x, gridDim.x, tiles_per_tau);
  TileCursor nx2 = cur.next();
  issue_tile<double>(a, sm, cur.tl, cur.x0(), cur.tl < a.ntau);
  issue_tile<double>(a, sm + kStage, nx2.tl, nx2.x0(), nx2.tl < a.ntau);

  for (int it = 0; cur.tl < a.ntau; cur = cur.next(), it++) {
    Cx<double>* st = sm + (it & 1) * kStage;
    cp_async_wait<1>();
    __syncthreads();
    const int tl = cur.tl;
    {
      // load-time transform of the staged tile, in place (uniform per tile)
      const int xfu = a.sl[tl].xf[0], xfd = a.sl[tl].xf[1];
      if (xfu | xfd) {
        const int s = tid & (kSitesPerTile - 1);
        for (int q = tid >> 4; q < 72; q += kThreads / kSitesPerTile) {
          const int f = q >= 36;
          int comp[4];
          prop_group_comps(q - 36 * f, comp);
          Cx<double>* r = st + s * kRow + 144 * f;
          prop_group_transform(r[comp[0]], r[comp[1]], r[comp[2]], r[comp[3]], f ? xfd : xfu);
        }
        __syncthreads();
      }
    }
    const int x = cur.x0() + hw;
    if (x < a.V3) {
      const RowF64 row{st + hw * kRow};
      const Writer<double> w{(Cx<double>*)a.out + (long long)tl * a.K * a.V3 + x, a.V3, nullptr, nullptr, nullptr, 0};
      contract_site<DELTA>(a, row, lt, l, mask, w);
    }
    __syncthreads();
    nx2 = nx2.next();  // two tiles ahead of the next iteration's
    issue_tile<double>(a, st, nx2.tl, nx2.x0(), nx2.tl < a.ntau);
  }
  cp_async_wait<0>();
}

// Split form: FP32 arithmetic on power-of-two scaled inputs.  One staging
// buffer in the input precision (component-major) plus an FP32 copy of the
// tile in the padded row layout of RowF32: the staging buffer is refilled
// with the whole next tile's cp.async as soon as the current one is
// converted, so the copies overlap the contraction, and two CTAs (16 warps)
// fit on an SM.
constexpr int kStage32 = kSitesPerTile * kRow32;

template <typename Tin, bool DELTA, bool DSTG = false>
__global__ void __launch_bounds__(kThreads, 2) k_contract_f32(const ContractArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cx<Tin>* st = (Cx<Tin>*)smem_raw;
  Cx<float>* sf = (Cx<float>*)(smem_raw + kSitesPerTile * 288 * sizeof(Cx<Tin>));
  // 16 x 16 meson outputs staged in the sites' own FP32 rows (not with the
  // 10 diagonal structures, whose second pass reads the rows again)
  const bool stage = !DELTA && g16_phase_deferred(a.what);
  // block layout of the FP32 rows: conflict-free lane-varying loads for the
  // nucleon and mesons; the Delta keeps the plain order (its registers are fuller)
  constexpr bool kPerm = !DELTA;
  // Delta instantiation with only the Delta blocks: its 192 outputs per site
  // (rows 0..95 iso-1/2, 96..191 iso-3/2) are staged in the last 24 KB of the
  // staging buffer, whose rows of the next tile are copied only after the
  // tile's output flush has read them; the flush writes 128-byte component
  // rows and takes the per-component maxima over the tile's sites (direct
  // stores from the lanes would touch 16 component rows per store, with a
  // shared-memory atomic per output)
  // (launched only for requests whose Delta pass holds the Delta blocks alone;
  // kept a run-time value: as a compile-time one ptxas spills 780 bytes here)
  const bool dstg = DELTA && DSTG && (a.what & (2u | 4u)) != 0;
  constexpr int kLate0 = 288 - 192 * kSitesPerTile * (int)sizeof(Cx<float>) / (kSitesPerTile * (int)sizeof(Cx<Tin>));
  Cx<float>* dstage = (Cx<float>*)(st + kLate0 * kSitesPerTile);
  const int tid = threadIdx.x;
  const int hw = tid >> 4, l = tid & 15;
  const unsigned mask = halfwarp_mask();
  const LaneTables lt = load_lane_tables(l);
  // the tile flush's thread -> (site, g1) map: lanes 0-7 / 8-15 / 16-23 / 24-31
  // of warp w take sites 0-7 / 0-7 / 8-15 / 8-15 of g1 = 2 w / 2 w + 1 / 2 w / 2 w + 1
  const int flush_s = (tid & 7) + ((tid >> 1) & 8), flush_g1 = 2 * (tid >> 5) + ((tid >> 3) & 1);

  const int tiles_per_tau = (a.V3 + kSitesPerTile - 1) / kSitesPerTile;
  TileCursor tc(blockIdx.x, gridDim.x, tiles_per_tau);
  for (int k = tid; k < a.K; k += kThreads) *smax_slot(sf, k) = 0;

  issue_tile<Tin, true>(a, st, tc.tl, tc.x0(), tc.tl < a.ntau);

  int cur = -1;  // slice whose maxima the spare slots hold
  // running maxima in registers: nucleon outputs of lane l (slots 0, 1) and
  // the staged meson outputs this thread writes out (slots 2 + g2); the
  // Delta instantiation tracks its maxima in shared memory only
  constexpr int kSlots = DELTA ? 1 : 18;
  float rmax[kSlots];
#pragma unroll
  for (int i = 0; i < kSlots; i++) rmax[i] = 0.f;
  // register maxima -> shared, once per time slice
  auto flush_lane = [&]() {
    if constexpr (!DELTA) {
      // nucleon: lane l of both half-warps holds components nuc + 16 i + l
#pragma unroll
      for (int i = 0; i < 2; i++) {
        const float m = fmaxf(rmax[i], __shfl_xor_sync(0xffffffffu, rmax[i], 16));
        rmax[i] = 0.f;
        if (!(tid & 16) && (a.what & 1u)) atomicMax(smax_slot(sf, a.k.nuc + 16 * i + l), __float_as_int(m));
      }
      // mesons: the 16 flush threads of g1 (lanes with the same bit 3 of a
      // warp) hold components g16 + 16 g1 + g2
#pragma unroll
      for (int i = 2; i < kSlots; i++) {
        float m = rmax[i];
        m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 1));
        m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 2));
        m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 4));
        m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 16));
        rmax[i] = 0.f;
        const int k = a.k.g16 + 16 * flush_g1 + (i - 2);
        if ((tid & 23) == 0 && stage) atomicMax(smax_slot(sf, k), __float_as_int(m));
      }
    }
  };
  for (; tc.tl < a.ntau; tc = tc.next()) {
    const int tl = tc.tl;
    if (tl != cur && cur >= 0) flush_lane();
    cp_async_wait<0>();
    __syncthreads();
    if (tl != cur) {
      if (cur >= 0)
        for (int k = tid; k < a.K; k += kThreads) {
          int* slot = smax_slot(sf, k);
          atomicMax(a.cmax + (long long)cur * a.K + k, *slot);
          *slot = 0;
        }
      cur = tl;
    }
    // scale by 2^-E per flavour and convert to FP32 once per tile: thread
    // (site s, groups g = c0 + 16 j of 40: 20 per flavour) reads the
    // component-major staging, applies the slice's load-time transform to the
    // group's four blocks b, b + 2, b + 8, b + 10 and writes the site's padded
    // row (exact power-of-two scales; products are formed in double so that
    // no intermediate leaves the representable range).  Groups 0..15 of a
    // flavour are (b, colour pair 2k, 2k + 1): one 16-byte store per block,
    // so the 8 sites of a quarter-warp write 8 different bank groups (rows are
    // 161 units apart); groups 16..19 are (b, colour 8).
    {
      const double su = ldexp(1.0, -a.exps[2 * tl]), sd = ldexp(1.0, -a.exps[2 * tl + 1]);
      const int xfu = a.sl[tl].xf[0], xfd = a.sl[tl].xf[1];
      const int s = tid & (kSitesPerTile - 1), c0 = tid >> 4;
      Cx<float>* row = sf + s * kRow32;
#pragma unroll
      for (int j = 0; j < 3; j++) {
        const int g = c0 + 16 * j;
        if (g < 40) {
          const int f = g >= 20, gf = g - 20 * f;
          const int bq = gf & 3, b = (bq >> 1) * 4 + (bq & 1);  // first block of the transform group: 0, 1, 4, 5
          const int xf = f ? xfd : xfu;
          const double sc = f ? sd : su;
          const Cx<Tin>* src = st + (144 * f + 9 * b) * kSitesPerTile + s;
          if (gf < 16) {
            const int k = gf >> 2;  // colours 2k, 2k + 1
            Cx<double> v[2][4];
#pragma unroll
            for (int c = 0; c < 2; c++)
#pragma unroll
              for (int i = 0; i < 4; i++) {
                const Cx<Tin> x = src[(9 * group_blk(i) + 2 * k + c) * kSitesPerTile];
                v[c][i] = cx<double>((double)x.x, (double)x.y);
              }
#pragma unroll
            for (int c = 0; c < 2; c++) prop_group_transform(v[c][0], v[c][1], v[c][2], v[c][3], xf);
#pragma unroll
            for (int i = 0; i < 4; i++)
              *reinterpret_cast<float4*>(row + 2 * row32_unit<kPerm>(16 * f + b + group_blk(i), k)) =
                  make_float4((float)(v[0][i].x * sc), (float)(v[0][i].y * sc), (float)(v[1][i].x * sc),
                              (float)(v[1][i].y * sc));
          } else {
            Cx<double> v[4];
#pragma unroll
            for (int i = 0; i < 4; i++) {
              const Cx<Tin> x = src[(9 * group_blk(i) + 8) * kSitesPerTile];
              v[i] = cx<double>((double)x.x, (double)x.y);
            }
            prop_group_transform(v[0], v[1], v[2], v[3], xf);
#pragma unroll
            for (int i = 0; i < 4; i++)
              row[2 * row32_unit<kPerm>(16 * f + b + group_blk(i), 4)] =
                  cx<float>((float)(v[i].x * sc), (float)(v[i].y * sc));
          }
        }
      }
    }
    __syncthreads();
    // the staged tile has been converted: refill the staging buffer while
    // contracting (with Delta output staging, all but its tail)
    const TileCursor nx = tc.next();
    issue_tile<Tin, true>(a, st, nx.tl, nx.x0(), nx.tl < a.ntau, 0, dstg ? kLate0 : 288);
    const int x0 = tc.x0();
    if (x0 + hw < a.V3) {
      const RowF32T<kPerm> row{sf + hw * kRow32};
      const Writer<float, DELTA && DSTG> w{(Cx<float>*)a.out + (long long)tl * a.K * a.V3 + x0 + hw, a.V3, DELTA ? nullptr : rmax, sf,
                            stage ? sf + hw * kRow32 : dstg ? dstage : nullptr, hw};
      contract_site<DELTA>(a, row, lt, l, mask, w);
    }
    if constexpr (DELTA) {
      if (dstg) {
        __syncthreads();  // every site's outputs are staged
        // half-warp q, lane s: staging rows q + 16 i of site s
        const int s = tid & 15, q = tid >> 4;
        const bool okx = x0 + s < a.V3;
#pragma unroll 1
        for (int i = 0; i < 12; i++) {
          const int r = q + 16 * i;
          if (!(r < 96 ? (a.what & 2u) : (a.what & 4u))) continue;  // uniform over the half-warp
          const int k = r < 96 ? a.k.diso12 + r : a.k.diso32 + r - 96;
          const Cx<float> v = dstage[r * 16 + (s ^ q)];
          float m = 0.f;
          if (okx) {
            ((Cx<float>*)a.out)[((long long)tl * a.K + k) * a.V3 + x0 + s] = v;
            m = fmaxf(fabsf(v.x), fabsf(v.y));
          }
          m = fmaxf(m, __shfl_xor_sync(mask, m, 1));
          m = fmaxf(m, __shfl_xor_sync(mask, m, 2));
          m = fmaxf(m, __shfl_xor_sync(mask, m, 4));
          m = fmaxf(m, __shfl_xor_sync(mask, m, 8));
          if (s == 0) atomicMax(smax_slot(sf, k), __float_as_int(m));
        }
        __syncthreads();  // the staging tail is read: the next tile's last rows may land there
        issue_tile<Tin, true>(a, st, nx.tl, nx.x0(), nx.tl < a.ntau, kLate0, 288);
      }
    }
    if constexpr (!DELTA) {
      if (stage) {
        __syncthreads();
        // thread (site s, g1 = flush_g1): components g16 + 16 g1 + g2, each a
        // 128-byte row segment over the tile's 16 sites written by the 16
        // threads of that g1; a half-warp reads 8 sites x the 2 adjacent
        // outputs of one 16-byte unit per site (rows 161 units apart: 8
        // different bank groups, one wavefront)
        const int s = flush_s;
        if (x0 + s < a.V3) {
          Cx<float>* o = (Cx<float>*)a.out + ((long long)tl * a.K + a.k.g16 + 16 * flush_g1) * a.V3 + x0 + s;
#pragma unroll
          for (int g2 = 0; g2 < 16; g2++) {
            const Cx<float> v = sf[s * kRow32 + g16_slot(flush_g1, g2)];
            o[(long long)g2 * a.V3] = v;
            rmax[2 + g2] = fmaxf(rmax[2 + g2], fmaxf(fabsf(v.x), fabsf(v.y)));
          }
          // nucleon components 2 g1, 2 g1 + 1 (maxima already taken by their lanes)
          if (a.what & 1u) {
            Cx<float>* on = (Cx<float>*)a.out + ((long long)tl * a.K + a.k.nuc + 2 * flush_g1) * a.V3 + x0 + s;
            on[0] = sf[s * kRow32 + nuc_slot(2 * flush_g1)];
            on[a.V3] = sf[s * kRow32 + nuc_slot(2 * flush_g1 + 1)];
          }
        }
      }
    }
  }
  cp_async_wait<0>();
  if (cur >= 0) flush_lane();
  __syncthreads();
  if (cur >= 0)
    for (int k = tid; k < a.K; k += kThreads) atomicMax(a.cmax + (long long)cur * a.K + k, *smax_slot(sf, k));
}

// Threads of the sampling kernel: the samples are scattered, so its time is
// the number of rounds of loads in flight per thread (21504 samples, 8 per
// thread and round).
constexpr int kSampleThreads = 512;

// Per-slice exponent E with max(|Re|,|Im|) < 2^E over a strided sample of
// sites and components (every 7th component, every 97th site), so that the
// scaled entries are O(1) in FP32.  Only the binary exponents are compared,
// so FP64 entries far below FP32's range are handled exactly.
__global__ void k_sample_exponents(const SampleArgs a) {
  __shared__ int red[kSampleThreads];
  const int tl = blockIdx.x, f = blockIdx.y;
  const SliceDesc& sd = a.sl[tl];
  const void* p = f ? sd.d : sd.u;
  const long long vol = f ? sd.vol_d : sd.vol_u;
  const long long j = f ? sd.off_d : sd.off_u;
  int emax = -100000;
  // 8 independent loads in flight per thread (the samples are scattered, so
  // each is a separate DRAM access)
  constexpr int kSamples = 21 * 1024, kBatch = 8;
  for (int i0 = threadIdx.x; i0 < kSamples; i0 += kBatch * blockDim.x) {
    double re[kBatch], im[kBatch];
#pragma unroll
    for (int u = 0; u < kBatch; u++) {
      const int i = i0 + u * blockDim.x;
      re[u] = im[u] = 0.0;
      if (i < kSamples) {
        const int comp = (i % 21) * 7;
        const long long x = ((long long)(i / 21) * 97) % a.V3;
        const long long idx = (long long)comp * vol + j + x;
        if (a.fp32) {
          const float2 v = ((const float2*)p)[idx];
          re[u] = v.x;
          im[u] = v.y;
        } else {
          const double2 v = ((const double2*)p)[idx];
          re[u] = v.x;
          im[u] = v.y;
        }
      }
    }
#pragma unroll
    for (int u = 0; u < kBatch; u++) {
      int e;
      if (re[u] != 0.0) {
        frexp(re[u], &e);
        emax = max(emax, e);
      }
      if (im[u] != 0.0) {
        frexp(im[u], &e);
        emax = max(emax, e);
      }
    }
  }
  red[threadIdx.x] = emax;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = max(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  // a rotation can double an entry: one more power of two of headroom
  if (threadIdx.x == 0) a.exp_out[2 * tl + f] = (red[0] == -100000 ? 0 : red[0]) + ((sd.xf[f] & 3) ? 1 : 0);
}

}  // namespace

int contract_plain_smem_bytes() { return 2 * kStage * (int)sizeof(Cx<double>); }

template <bool DELTA>
cudaError_t launch_plain_t(const ContractArgs& a, int grid, cudaStream_t s) {
  const int smem = contract_plain_smem_bytes();
  cudaError_t e = ensure_smem((const void*)k_contract_plain<DELTA>, smem);
  if (e != cudaSuccess) return e;
  k_contract_plain<DELTA><<<grid, kThreads, smem, s>>>(a);
  return cudaGetLastError();
}

template <typename Tin, bool DELTA, bool DSTG = false>
cudaError_t launch_f32_t(const ContractArgs& a, int grid, cudaStream_t s) {
  const int smem = kSitesPerTile * 288 * (int)sizeof(Cx<Tin>) + kStage32 * (int)sizeof(Cx<float>);
  if (a.K > 2 * 32 * kSitesPerTile) return cudaErrorInvalidValue;  // more components than spare slots
  cudaError_t e = ensure_smem((const void*)k_contract_f32<Tin, DELTA, DSTG>, smem);
  if (e != cudaSuccess) return e;
  k_contract_f32<Tin, DELTA, DSTG><<<grid, kThreads, smem, s>>>(a);
  return cudaGetLastError();
}

// the second instantiation: Delta and the second nucleon interpolator
constexpr unsigned kDeltaBits = 2u | 4u | 128u | 256u | 512u;

cudaError_t launch_contract_plain(const ContractArgs& a, int grid, cudaStream_t s) {
  cudaError_t e = cudaSuccess;
  if (a.what & ~kDeltaBits) e = launch_plain_t<false>(a, grid, s);
  if (e == cudaSuccess && (a.what & kDeltaBits)) e = launch_plain_t<true>(a, grid, s);
  return e;
}

cudaError_t launch_contract_f32(const ContractArgs& a, int fp32_in, int grid, cudaStream_t s) {
  cudaError_t e = cudaSuccess;
  if (a.what & ~kDeltaBits)
    e = fp32_in ? launch_f32_t<float, false>(a, grid, s) : launch_f32_t<double, false>(a, grid, s);
  if (e == cudaSuccess && (a.what & kDeltaBits)) {
    // the Delta pass with the Delta blocks alone stages its outputs
    const bool stg = !(a.what & (128u | 256u | 512u));
    if (stg)
      e = fp32_in ? launch_f32_t<float, true, true>(a, grid, s) : launch_f32_t<double, true, true>(a, grid, s);
    else
      e = fp32_in ? launch_f32_t<float, true>(a, grid, s) : launch_f32_t<double, true>(a, grid, s);
  }
  return e;
}

cudaError_t launch_sample_exponents(const SampleArgs& a, cudaStream_t s) {
  k_sample_exponents<<<dim3(a.ntau, 2), kSampleThreads, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace p2
