// Table-driven baryon two-point functions: the reference's UDSC set
// (contractBaryonsUDSC, lib/PLEGMA_Correlator.cu:137-189, kernels
// lib/kernels/PLEGMA_baryons_udsc.cu:85-309), plain FP64 form.
//
// A flavour product (e.g. "uud") has up to 16 datasets (interpolator and
// projector variants); dataset d of a site is
//   sum_entries w * sum_{eps eps'} P1[s0 s1][a a'] P2[s2 s3][b b'] P3[s4 s5][c c']
// over the spin tables of plegma_b200/udsc.py (weights in single precision
// like the reference's).  The colour sums factorise through the diquark
//   G_{s0 s1, s2 s3}[c][c'] = sum eps_abc eps_a'b'c' P1[a a'] P2[b b']
// (36 complex products), and an entry costs one 9-term product G . P3.
// Across a product's datasets only 112-256 distinct (s0 s1 s2 s3) tuples
// occur, so each G is computed once per site and shared by every entry of
// every dataset that uses it (the reference evaluates 36 x 3 products per
// entry).
//
// Layout: one site per half-warp; the three propagators of 16 sites are
// staged with cp.async in two stages ([site][3 x 144 + 1] complex double).
// The host assigns the distinct tuples to the 16 lanes (balanced by work)
// and encodes one instruction stream per lane:
//   per tuple: P1 block | P2 block << 8, four words of per-dataset entry
//   counts (one byte each), then per entry: P3 block, Re w, Im w (float bits).
// Each lane accumulates all datasets in registers; a half-warp reduce-scatter
// (lane d ends with dataset d) gives the site's values, written to a
// [slice][dataset][site] buffer that
// the FP64 projection (project_fp64.cu) and the deterministic reduction
// consume.
#include <algorithm>
#include <cstring>
#include <map>
#include <numeric>
#include <string>
#include <vector>

#include "ctx.h"
#include "launch_util.h"
#include "site_contract.cuh"
#include "udsc_tables.h"

using namespace p2host;

namespace p2 {
namespace {

constexpr int kThreadsU = 256;
constexpr int kSitesU = 16;
constexpr int kRowU = 3 * 144 + 1;  // complex per staged site row (P1, P2, P3 + pad)
constexpr int kStageU = kSitesU * kRowU;
constexpr int kMaxDs = 16;          // datasets per product (the reference's largest product has 16)

struct UdscSlice {
  long long off[3];  // element offset of the slice inside each of the three views
  int xf[3];         // load-time transform of each view on this slice (PropXf)
  int pad;
};

struct UdscArgs {
  const Cx<double>* p0;
  const Cx<double>* p1;
  const Cx<double>* p2;
  long long vol0, vol1, vol2;  // component strides of the views
  const UdscSlice* sl;
  int ntau, V3, nd;
  const int* plan;  // [16] lane offsets, then the lane streams
  Cx<double>* out;  // [ntau][nd][V3]
};

__device__ __forceinline__ void issue_tile_u(const UdscArgs& a, Cx<double>* st, const TileCursor& t, int ntau) {
  if (t.tl < ntau) {
    const int tl = t.tl;
    const int s = threadIdx.x & (kSitesU - 1);
    const int x = t.x0() + s;
    const bool ok = x < a.V3;
    const UdscSlice* sd = a.sl + tl;
    // thread i copies component i/16 + 16 r of site i%16: rows r < 9 are P1,
    // 9 <= r < 18 P2, 18 <= r < 27 P3
#pragma unroll
    for (int f = 0; f < 3; f++) {
      const Cx<double>* base = f == 0 ? a.p0 : f == 1 ? a.p1 : a.p2;
      const long long vol = f == 0 ? a.vol0 : f == 1 ? a.vol1 : a.vol2;
      const Cx<double>* src = base + sd->off[f] + (ok ? x : 0);
#pragma unroll 3
      for (int r = 0; r < 9; r++) {
        const int comp = (threadIdx.x >> 4) + 16 * r;
        cp_async16(st + s * kRowU + 144 * f + comp, src + comp * vol, ok ? 16 : 0);
      }
    }
  }
  cp_async_commit();
}

// Sum of the 16 lanes' dataset accumulators, lane l ending with dataset l:
// a reduce-scatter (8 + 4 + 2 + 1 exchanged values instead of 16 all-reduces).
template <typename R>
__device__ __forceinline__ Cx<R> reduce_scatter16(Cx<R> (&acc)[16], int l, unsigned mask) {
#pragma unroll
  for (int h = 8; h >= 1; h >>= 1) {
    const bool up = (l & h) != 0;
#pragma unroll
    for (int j = 0; j < h; j++) {
      const Cx<R> send = up ? acc[j] : acc[j + h];
      const Cx<R> keep = up ? acc[j + h] : acc[j];
      acc[j] = keep + shfl_xor16(send, h, mask);
    }
  }
  return acc[0];
}

__global__ void __launch_bounds__(kThreadsU, 1) k_contract_udsc(const UdscArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cx<double>* sm = (Cx<double>*)smem_raw;
  const int tid = threadIdx.x;
  const int hw = tid >> 4, l = tid & 15;
  const unsigned mask = halfwarp_mask();
  const int tiles_per_tau = (a.V3 + kSitesU - 1) / kSitesU;
  TileCursor cur(blockIdx.x, gridDim.x, tiles_per_tau);
  TileCursor nx2 = cur.next();
  const int* stream0 = a.plan + a.plan[l];

  issue_tile_u(a, sm, cur, a.ntau);
  issue_tile_u(a, sm + kStageU, nx2, a.ntau);
  for (int it = 0; cur.tl < a.ntau; cur = cur.next(), it++) {
    Cx<double>* st = sm + (it & 1) * kStageU;
    cp_async_wait<1>();
    __syncthreads();
    const int tl = cur.tl;
    {
      // load-time transforms of the staged tile, in place (uniform per tile)
      const UdscSlice& sd = a.sl[tl];
      if (sd.xf[0] | sd.xf[1] | sd.xf[2]) {
        const int s = tid & (kSitesU - 1);
        for (int q = tid >> 4; q < 108; q += kThreadsU / kSitesU) {
          const int f = q / 36;
          int comp[4];
          prop_group_comps(q - 36 * f, comp);
          Cx<double>* r = st + s * kRowU + 144 * f;
          prop_group_transform(r[comp[0]], r[comp[1]], r[comp[2]], r[comp[3]], sd.xf[f]);
        }
        __syncthreads();
      }
    }
    const int x = cur.x0() + hw;
    if (x < a.V3) {
      const RowF64 row{st + hw * kRowU};
      Cx<double> acc[kMaxDs];
#pragma unroll
      for (int d = 0; d < kMaxDs; d++) acc[d] = czero<double>();
      const int* q = stream0;
      const int ntup = *q++;
#pragma unroll 1
      for (int t = 0; t < ntup; t++) {
        const int head = q[0];
        const unsigned cnt[4] = {(unsigned)q[1], (unsigned)q[2], (unsigned)q[3], (unsigned)q[4]};
        q += 5;
        Cx<double> g[9];
#pragma unroll
        for (int i = 0; i < 9; i++) g[i] = czero<double>();
        // blocks: P1 at 0..15, P2 at 16..31 of the row (block offset kD), P3 at 32..47
        diquark_acc(row, head & 255, (head >> 8) & 255, 0, 0, 1.0, 0, 0, g);
#pragma unroll
        for (int d = 0; d < kMaxDs; d++) {
          if (d >= a.nd) break;
          const int n = (int)((cnt[d >> 2] >> (8 * (d & 3))) & 255u);
#pragma unroll 1
          for (int e = 0; e < n; e++) {
            const int blk = q[0];
            const Cx<double> w = cx<double>((double)__int_as_float(q[1]), (double)__int_as_float(q[2]));
            q += 3;
            Cx<double> z[9];
            row.load9(blk, z);
            Cx<double> dot = czero<double>();
#pragma unroll
            for (int i = 0; i < 9; i++) cmac(dot, g[i], z[i]);
            cmac(acc[d], w, dot);
          }
        }
      }
      Cx<double>* o = a.out + (long long)tl * a.nd * a.V3 + x;
      if (a.nd > 4) {
        static_assert(kMaxDs == 16, "the reduce-scatter spreads 16 datasets over the 16 lanes");
        const Cx<double> v = reduce_scatter16(acc, l, mask);
        if (l < a.nd) o[(long long)l * a.V3] = v;
      } else {
#pragma unroll
        for (int d = 0; d < 4; d++) {
          if (d >= a.nd) break;
          Cx<double> v = acc[d];
          v = v + shfl_xor16(v, 1, mask);
          v = v + shfl_xor16(v, 2, mask);
          v = v + shfl_xor16(v, 4, mask);
          v = v + shfl_xor16(v, 8, mask);
          if (l == d) o[(long long)d * a.V3] = v;
        }
      }
    }
    __syncthreads();
    nx2 = nx2.next();  // two tiles ahead of the next iteration's
    issue_tile_u(a, st, nx2, a.ntau);
  }
  cp_async_wait<0>();
}

cudaError_t launch_contract_udsc(const UdscArgs& a, int grid, cudaStream_t s) {
  const int smem = 2 * kStageU * (int)sizeof(Cx<double>);
  cudaError_t e = ensure_smem((const void*)k_contract_udsc, smem);
  if (e != cudaSuccess) return e;
  k_contract_udsc<<<grid, kThreadsU, smem, s>>>(a);
  return cudaGetLastError();
}

// ---- split form --------------------------------------------------------------
// The same lane streams in FP32 on the three views scaled by 2^-E (per slice
// and view, exact), the FP32 tile in the padded row layout of RowF32 with the
// views at blocks 0-15, 16-31, 32-47; per (slice, dataset) the maximum of
// |Re|, |Im| for the hi+lo FP16 split of the tensor-core projection.
constexpr int kRowU32 = 48 * 10 + 2;  // complex per FP32 site row (161 x 3 units: rows start in different bank groups)

struct UdscArgsF32 {
  const void* p[3];
  long long vol[3];  // component strides of the views
  const UdscSlice* sl;
  int ntau, V3, nd;
  const int* plan;
  int* e3;          // [ntau][3]: view v of slice t is staged times 2^-e3[3t+v]
  int* es;          // [ntau][2]: (sum of the slice's three exponents, 0), the un-scaling of every dataset
  Cx<float>* out;   // [ntau][nd][V3]
  int* cmax;        // [ntau][nd] max |Re|, |Im| as float bits
};

// Per slice and view the binary exponent of the largest of a strided sample
// (every 7th component, every 97th site), plus one when the view is rotated.
template <typename Tin>
__global__ void k_sample_udsc(const UdscArgsF32 a) {
  __shared__ int red[256];
  const int tl = blockIdx.x;
  const UdscSlice& sd = a.sl[tl];
  int total = 0;
  for (int f = 0; f < 3; f++) {
    const Cx<Tin>* p = (const Cx<Tin>*)a.p[f] + sd.off[f];
    int emax = -100000;
    for (int i = threadIdx.x; i < 21 * 1024; i += blockDim.x) {
      const int comp = (i % 21) * 7;
      const long long x = ((long long)(i / 21) * 97) % a.V3;
      const Cx<Tin> v = p[comp * a.vol[f] + x];
      int e;
      if (v.x != 0) {
        frexp((double)v.x, &e);
        emax = max(emax, e);
      }
      if (v.y != 0) {
        frexp((double)v.y, &e);
        emax = max(emax, e);
      }
    }
    red[threadIdx.x] = emax;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s) red[threadIdx.x] = max(red[threadIdx.x], red[threadIdx.x + s]);
      __syncthreads();
    }
    const int E = (red[0] == -100000 ? 0 : red[0]) + ((sd.xf[f] & 3) ? 1 : 0);
    total += E;
    if (threadIdx.x == 0) a.e3[3 * tl + f] = E;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    a.es[2 * tl] = total;
    a.es[2 * tl + 1] = 0;
  }
}

template <typename Tin>
__device__ __forceinline__ void issue_tile_u32(const UdscArgsF32& a, Cx<Tin>* st, const TileCursor& t, int ntau) {
  if (t.tl < ntau) {
    const int tl = t.tl;
    const int s = threadIdx.x & (kSitesU - 1);
    const int x = t.x0() + s;
    const bool ok = x < a.V3;
    const UdscSlice* sd = a.sl + tl;
    // component-major staging [view * 144 + component][16 sites]: thread i
    // copies component i/16 + 16 r of site i%16
#pragma unroll
    for (int f = 0; f < 3; f++) {
      const Cx<Tin>* src = (const Cx<Tin>*)a.p[f] + sd->off[f] + (ok ? x : 0);
#pragma unroll 3
      for (int r = 0; r < 9; r++) {
        const int comp = (threadIdx.x >> 4) + 16 * r;
        Cx<Tin>* dst = st + (144 * f + comp) * kSitesU + s;
        if (sizeof(Tin) == 8)
          cp_async16(dst, src + comp * a.vol[f], ok ? 16 : 0);
        else
          cp_async8(dst, src + comp * a.vol[f], ok ? 8 : 0);
      }
    }
  }
  cp_async_commit();
}

template <typename Tin>
__global__ void __launch_bounds__(kThreadsU, 1) k_contract_udsc_f32(const UdscArgsF32 a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cx<Tin>* st = (Cx<Tin>*)smem_raw;
  Cx<float>* sf = (Cx<float>*)(smem_raw + 3 * 144 * kSitesU * sizeof(Cx<Tin>));
  int* smx = (int*)(sf + kSitesU * kRowU32);  // [kMaxDs] maxima of the current slice
  const int tid = threadIdx.x;
  const int hw = tid >> 4, l = tid & 15;
  const unsigned mask = halfwarp_mask();
  const int tiles_per_tau = (a.V3 + kSitesU - 1) / kSitesU;
  TileCursor tc(blockIdx.x, gridDim.x, tiles_per_tau);
  const int* stream0 = a.plan + a.plan[l];
  if (tid < kMaxDs) smx[tid] = 0;

  issue_tile_u32<Tin>(a, st, tc, a.ntau);
  int cur = -1;
  for (; tc.tl < a.ntau; tc = tc.next()) {
    const int tl = tc.tl;
    cp_async_wait<0>();
    __syncthreads();
    if (tl != cur) {
      if (cur >= 0 && tid < a.nd) {
        atomicMax(a.cmax + (long long)cur * a.nd + tid, smx[tid]);
        smx[tid] = 0;
      }
      cur = tl;
    }
    // scale, transform and convert: thread (site s, transform groups
    // q = c0 + 16 j of 108: 36 per view) -> the site's FP32 row
    {
      const UdscSlice& sd = a.sl[tl];
      const int s = tid & (kSitesU - 1), c0 = tid >> 4;
      Cx<float>* row = sf + s * kRowU32;
#pragma unroll
      for (int j = 0; j < 7; j++) {
        const int q = c0 + 16 * j;
        if (q < 108) {
          const int f = q / 36;
          const double sc = ldexp(1.0, -a.e3[3 * tl + f]);
          int b, cc;
          prop_group_base(q - 36 * f, b, cc);
          const Cx<Tin>* src = st + (144 * f + 9 * b + cc) * kSitesU + s;
          Cx<double> v[4];
#pragma unroll
          for (int i = 0; i < 4; i++) {
            const Cx<Tin> x = src[9 * group_blk(i) * kSitesU];
            v[i] = cx<double>((double)x.x, (double)x.y);
          }
          prop_group_transform(v[0], v[1], v[2], v[3], sd.xf[f]);
#pragma unroll
          for (int i = 0; i < 4; i++)
            row[2 * row32_unit(16 * f + b + group_blk(i), cc >> 1) + (cc & 1)] =
                cx<float>((float)(v[i].x * sc), (float)(v[i].y * sc));
        }
      }
    }
    __syncthreads();
    issue_tile_u32<Tin>(a, st, tc.next(), a.ntau);
    const int x = tc.x0() + hw;
    if (x < a.V3) {
      const RowF32 row{sf + hw * kRowU32};
      Cx<float> acc[kMaxDs];
#pragma unroll
      for (int d = 0; d < kMaxDs; d++) acc[d] = czero<float>();
      const int* q = stream0;
      const int ntup = *q++;
#pragma unroll 1
      for (int t = 0; t < ntup; t++) {
        const int head = q[0];
        const unsigned cnt[4] = {(unsigned)q[1], (unsigned)q[2], (unsigned)q[3], (unsigned)q[4]};
        q += 5;
        Cx<float> g[9];
#pragma unroll
        for (int i = 0; i < 9; i++) g[i] = czero<float>();
        diquark_acc(row, head & 255, (head >> 8) & 255, 0, 0, 1.f, 0, 0, g);
#pragma unroll
        for (int d = 0; d < kMaxDs; d++) {
          if (d >= a.nd) break;
          const int n = (int)((cnt[d >> 2] >> (8 * (d & 3))) & 255u);
#pragma unroll 1
          for (int e = 0; e < n; e++) {
            const int blk = q[0];
            const Cx<float> w = cx<float>(__int_as_float(q[1]), __int_as_float(q[2]));
            q += 3;
            Cx<float> z[9];
            row.load9(blk, z);
            Cx<float> dot = czero<float>();
#pragma unroll
            for (int i = 0; i < 9; i++) cmac(dot, g[i], z[i]);
            cmac(acc[d], w, dot);
          }
        }
      }
      Cx<float>* o = a.out + (long long)tl * a.nd * a.V3 + x;
      if (a.nd > 4) {
        const Cx<float> v = reduce_scatter16(acc, l, mask);
        if (l < a.nd) {
          o[(long long)l * a.V3] = v;
          atomicMax(smx + l, __float_as_int(fmaxf(fabsf(v.x), fabsf(v.y))));
        }
      } else {
#pragma unroll
        for (int d = 0; d < 4; d++) {
          if (d >= a.nd) break;
          Cx<float> v = acc[d];
          v = v + shfl_xor16(v, 1, mask);
          v = v + shfl_xor16(v, 2, mask);
          v = v + shfl_xor16(v, 4, mask);
          v = v + shfl_xor16(v, 8, mask);
          if (l == d) {
            o[(long long)d * a.V3] = v;
            atomicMax(smx + d, __float_as_int(fmaxf(fabsf(v.x), fabsf(v.y))));
          }
        }
      }
    }
  }
  cp_async_wait<0>();
  __syncthreads();
  if (cur >= 0 && tid < a.nd) atomicMax(a.cmax + (long long)cur * a.nd + tid, smx[tid]);
}

template <typename Tin>
cudaError_t launch_udsc_split_t(const UdscArgsF32& a, int grid, cudaStream_t s) {
  k_sample_udsc<Tin><<<a.ntau, 256, 0, s>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const int smem = 3 * 144 * kSitesU * (int)sizeof(Cx<Tin>) + kSitesU * kRowU32 * (int)sizeof(Cx<float>) + 64;
  e = ensure_smem((const void*)k_contract_udsc_f32<Tin>, smem);
  if (e != cudaSuccess) return e;
  k_contract_udsc_f32<Tin><<<grid, kThreadsU, smem, s>>>(a);
  return cudaGetLastError();
}

// Per-lane instruction streams of one flavour product (see the file comment).
std::vector<int> build_plan(int prod) {
  const int d0 = kUdscDsBegin[prod], nd = kUdscDsBegin[prod + 1] - d0;
  // distinct (P1 block, P2 block) tuples in first-occurrence order, and per
  // tuple and dataset its entries (P3 block, weight)
  std::map<int, int> tix;
  std::vector<int> key;
  std::vector<std::vector<std::vector<int>>> ent;  // [tuple][dataset] -> (blk, wre bits, wim bits)...
  for (int d = 0; d < nd; d++)
    for (int e = kUdscEntBegin[d0 + d]; e < kUdscEntBegin[d0 + d + 1]; e++) {
      const signed char* m = kUdscIdx[e];
      const int k = (m[0] * 4 + m[1]) | ((16 + m[2] * 4 + m[3]) << 8);
      auto it = tix.find(k);
      int t;
      if (it == tix.end()) {
        t = (int)key.size();
        tix[k] = t;
        key.push_back(k);
        ent.emplace_back(nd);
      } else {
        t = it->second;
      }
      int wb[2];
      std::memcpy(wb, kUdscVal[e], sizeof(wb));
      auto& v = ent[t][d];
      v.push_back(32 + m[4] * 4 + m[5]);
      v.push_back(wb[0]);
      v.push_back(wb[1]);
    }
  // balance: largest tuples first, each to the least loaded lane (cost in
  // complex products: 36 for G, 9 per entry)
  const int nt = (int)key.size();
  std::vector<int> cost(nt), order(nt);
  for (int t = 0; t < nt; t++) {
    int n = 0;
    for (const auto& v : ent[t]) n += (int)v.size() / 3;
    cost[t] = 36 + 9 * n;
  }
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost[x] > cost[y]; });
  std::vector<std::vector<int>> lane(16);
  std::vector<int> load(16, 0);
  for (int t : order) {
    const int l = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    lane[l].push_back(t);
    load[l] += cost[t];
  }
  std::vector<int> plan(16, 0);
  for (int l = 0; l < 16; l++) {
    plan[l] = (int)plan.size();
    plan.push_back((int)lane[l].size());
    for (int t : lane[l]) {
      plan.push_back(key[t]);
      unsigned cnt[4] = {0, 0, 0, 0};
      for (int d = 0; d < nd; d++) cnt[d >> 2] |= (unsigned)(ent[t][d].size() / 3) << (8 * (d & 3));
      for (int i = 0; i < 4; i++) plan.push_back((int)cnt[i]);
      for (int d = 0; d < nd; d++) plan.insert(plan.end(), ent[t][d].begin(), ent[t][d].end());
    }
  }
  return plan;
}

// Products a request runs, in the reference's order and with its filters
// (lib/PLEGMA_Correlator.cu:152-177).
std::vector<int> products_of(const p2_udsc_request& r) {
  std::vector<int> todo;
  for (int i = 0; i < kUdscProducts; i++) {
    const std::string f = kUdscProduct[i];
    auto has = [&](char c) { return f.find(c) != std::string::npos; };
    if ((r.prop_u < 0 && has('u')) || (r.prop_d < 0 && has('d')) || (r.prop_s < 0 && has('s')) ||
        (r.prop_c < 0 && has('c')))
      continue;
    if (r.only_st && !has('s')) continue;
    if (r.only_ch && !has('c')) continue;
    todo.push_back(i);
  }
  return todo;
}

int prop_of(const p2_udsc_request& r, char f) {
  return f == 'u' ? r.prop_u : f == 'd' ? r.prop_d : f == 's' ? r.prop_s : r.prop_c;
}

}  // namespace
}  // namespace p2

struct p2_udsc_cache {
  std::vector<p2host::DevBuf> plan;  // per product, built on first use
  p2host::DevBuf slices, desc;
  p2host::DevBuf e3, es, kexp;  // split form: view exponents, un-scaling exponents, component multiplicities
  ~p2_udsc_cache() {
    for (auto& b : plan) b.release();
    for (p2host::DevBuf* b : {&slices, &desc, &e3, &es, &kexp}) b->release();
  }
};

void p2_udsc_release(p2_ctx* c) {
  delete c->udsc;
  c->udsc = nullptr;
}

extern "C" {

int p2_udsc_datasets(const p2_udsc_request* r, char* names, size_t cap) {
  if (!r) return -1;
  std::string s;
  int n = 0;
  for (int p : p2::products_of(*r))
    for (int d = kUdscDsBegin[p]; d < kUdscDsBegin[p + 1]; d++, n++) {
      s += kUdscName[d];
      s += '\n';
    }
  if (names && cap) {
    const size_t m = std::min(cap - 1, s.size());
    std::memcpy(names, s.data(), m);
    names[m] = 0;
  }
  return n;
}

p2_status p2_contract_udsc(p2_ctx* c, const p2_prop* props, int nprops, const p2_udsc_request* r) {
  using namespace p2;
  if (!c) return P2_ERR_INVALID_ARG;
  if (!props || nprops < 1 || !r) return c->fail(P2_ERR_INVALID_ARG, "p2_contract_udsc: empty props or request");
  for (int f : {r->prop_u, r->prop_d, r->prop_s, r->prop_c})
    if (f < -1 || f >= nprops) return c->fail(P2_ERR_INVALID_ARG, "p2_contract_udsc: prop index out of range");
  if (!r->out) return c->fail(P2_ERR_INVALID_ARG, "null output");
  if (r->out_location != P2_DEVICE && r->out_location != P2_HOST)
    return c->fail(P2_ERR_INVALID_ARG, "bad out_location");
  if (r->mode != P2_PLAIN_FP64 && r->mode != P2_SPLIT_FP16) return c->fail(P2_ERR_INVALID_ARG, "bad mode");
  const bool split = r->mode == P2_SPLIT_FP16;
  p2_request base{};
  std::memcpy(base.source, r->source, sizeof(base.source));
  base.totalT = r->totalT;
  base.moms = r->moms;
  base.nmom = r->nmom;
  base.q2max = r->q2max;
  base.contractions = P2_NUCLEON_CG5;  // any valid set: only the window and momenta are used
  Plan pl;
  p2_status st = make_plan(c, base, pl);
  if (st != P2_OK) return st;
  const std::vector<int> todo = products_of(*r);
  for (int p : todo)
    for (int k = 0; k < 3; k++) {
      const p2_prop& pr = props[prop_of(*r, kUdscProduct[p][k])];
      if (!pr.data || pr.nt < 1 || pr.nt > c->T || pr.t_first < 0 || pr.t_first >= c->T)
        return c->fail(P2_ERR_INVALID_ARG, "p2_contract_udsc: bad propagator view");
      if ((pr.transform & ~0xFu) || ((pr.transform & 1u) && (pr.transform & 2u)))
        return c->fail(P2_ERR_INVALID_ARG, "p2_contract_udsc: bad transform bits");
      if (pr.precision != P2_FP64 && !(split && pr.precision == P2_FP32))
        return c->fail(P2_ERR_UNSUPPORTED, "p2_contract_udsc: FP32 propagators need the split form");
      if (pr.precision != props[prop_of(*r, kUdscProduct[todo[0]][0])].precision)
        return c->fail(P2_ERR_UNSUPPORTED, "p2_contract_udsc: all propagators must share a precision");
      if (pr.location != P2_DEVICE)
        return c->fail(P2_ERR_UNSUPPORTED, "p2_contract_udsc needs device-resident propagators");
    }
  if (c->host_only) return c->fail(P2_ERR_UNSUPPORTED, "host-only context");
  int nds = 0;
  for (int p : todo) nds += kUdscDsBegin[p + 1] - kUdscDsBegin[p];
  const size_t total = (size_t)nds * r->totalT * pl.nmom;
  if (todo.empty()) return P2_OK;
  if (!c->udsc) c->udsc = new p2_udsc_cache();
  p2_udsc_cache& U = *c->udsc;
  if (U.plan.empty()) U.plan.resize(kUdscProducts);

  double* dres = r->out;
  if (r->out_location == P2_HOST) {
    P2_TRY(c, c->res.ensure(total * 16), "result alloc");
    P2_TRY(c, cudaMemsetAsync(c->res.p, 0, total * 16, c->stream), "result clear");
    dres = (double*)c->res.p;
  }
  int nmtile = 0, nkstep = 0;
  if (split) {
    if (c->project_split_smem_max < project_split_smem_bytes(project_split_max_nt()))
      return c->fail(P2_ERR_UNSUPPORTED, "device shared memory per block too small for the tensor-core projection");
    if (!c->errflag.p) {
      P2_TRY(c, c->errflag.ensure(16), "error flag alloc");
      P2_TRY(c, cudaMemsetAsync(c->errflag.p, 0, 16, c->stream), "error flag clear");
    }
    if ((st = split_prepare_tables(c, pl, 0, nmtile, nkstep)) != P2_OK) return st;
    if (!U.kexp.p) {  // every dataset carries each of its three views once: (1, 0) against es
      std::vector<int> ke(2 * kMaxDs, 0);
      for (int k = 0; k < kMaxDs; k++) ke[2 * k] = 1;
      if ((st = upload_async(c, U.kexp, ke.data(), ke.size() * sizeof(int), "udsc exponents")) != P2_OK) return st;
    }
  }
  // phase tables (origin 0; the scatter applies the source phase)
  if (!split && c->plain_moms_key != pl.moms) {
    c->plain_moms_key.clear();
    std::vector<double> tabh = phase_tables(c, pl.moms.data(), pl.nmom, -1, pl.Lmax);
    if ((st = upload_async(c, c->ptab, tabh.data(), tabh.size() * sizeof(double), "phase table")) != P2_OK)
      return st;
    if ((st = upload_async(c, c->moms, pl.moms.data(), pl.moms.size() * sizeof(int), "momenta")) != P2_OK)
      return st;
    c->plain_moms_key = pl.moms;
  }
  const int T = c->T, tl0 = c->g.coords[3] * c->Ll[3];
  int ds_off = 0;
  for (int p : todo) {
    const int nd = kUdscDsBegin[p + 1] - kUdscDsBegin[p];
    if (!U.plan[p].p) {
      const std::vector<int> plan = build_plan(p);
      if ((st = upload_async(c, U.plan[p], plan.data(), plan.size() * sizeof(int), "udsc plan")) != P2_OK) return st;
    }
    const p2_prop* v[3];
    for (int k = 0; k < 3; k++) v[k] = &props[prop_of(*r, kUdscProduct[p][k])];
    // local slices held by all three views
    std::vector<int> taus;
    std::vector<UdscSlice> sl;
    for (int tau = 0; tau < r->totalT; tau++) {
      const int t = (r->source[3] + tau) % T;
      if (t < tl0 || t >= tl0 + c->Ll[3]) continue;
      UdscSlice s{};
      bool ok = true;
      for (int k = 0; k < 3; k++) {
        const int j = ((t - v[k]->t_first) % T + T) % T;
        ok &= j < v[k]->nt;
        s.off[k] = (long long)j * c->V3;
        s.xf[k] = prop_xf_code(*v[k], t);
      }
      if (!ok) continue;
      taus.push_back(tau);
      sl.push_back(s);
    }
    const int n_all = (int)taus.size();
    if (split) {
      const bool f32 = v[0]->precision == P2_FP32;
      const size_t per32 = (size_t)nd * c->V3 * 8;
      const int tc = (int)std::max<size_t>(1, std::min<size_t>(c->ws_budget / std::max<size_t>(per32, 1), (size_t)T));
      for (int c0 = 0; c0 < n_all; c0 += tc) {
        const int n = std::min(tc, n_all - c0);
        P2_TRY(c, c->cbuf.ensure((size_t)n * per32), "position buffer alloc");
        P2_TRY(c, c->cmaxb.ensure((size_t)n * nd * sizeof(int)), "maxima alloc");
        P2_TRY(c, cudaMemsetAsync(c->cmaxb.p, 0, (size_t)n * nd * sizeof(int), c->stream), "maxima clear");
        P2_TRY(c, U.e3.ensure((size_t)n * 3 * sizeof(int)), "exponent alloc");
        P2_TRY(c, U.es.ensure((size_t)n * 2 * sizeof(int)), "exponent alloc");
        P2_TRY(c, U.slices.ensure((size_t)n * sizeof(UdscSlice)), "slice alloc");
        P2_TRY(c,
               cudaMemcpyAsync(U.slices.p, sl.data() + c0, (size_t)n * sizeof(UdscSlice), cudaMemcpyHostToDevice,
                               c->stream),
               "slice upload");
        std::vector<SliceDesc> desc(n);
        for (int i = 0; i < n; i++) {
          std::memset(&desc[i], 0, sizeof(SliceDesc));
          desc[i].out = dres;
          desc[i].tau = taus[c0 + i];
          desc[i].totalT = r->totalT;
          for (int d = 0; d < 3; d++) desc[i].x0[d] = r->source[d];
        }
        P2_TRY(c, U.desc.ensure((size_t)n * sizeof(SliceDesc)), "descriptor alloc");
        P2_TRY(c,
               cudaMemcpyAsync(U.desc.p, desc.data(), (size_t)n * sizeof(SliceDesc), cudaMemcpyHostToDevice,
                               c->stream),
               "descriptor upload");
        UdscArgsF32 a{};
        for (int k = 0; k < 3; k++) {
          a.p[k] = v[k]->data;
          a.vol[k] = c->V3 * v[k]->nt;
        }
        a.sl = (const UdscSlice*)U.slices.p;
        a.ntau = n;
        a.V3 = (int)c->V3;
        a.nd = nd;
        a.plan = (const int*)U.plan[p].p;
        a.e3 = (int*)U.e3.p;
        a.es = (int*)U.es.p;
        a.out = (Cx<float>*)c->cbuf.p;
        a.cmax = (int*)c->cmaxb.p;
        {
          ProfScope ps(c, "contract_udsc_f32");
          P2_TRY(c, f32 ? launch_udsc_split_t<float>(a, c->nsm, c->stream) : launch_udsc_split_t<double>(a, c->nsm, c->stream),
                 "udsc split contraction");
        }
        const std::vector<ScatterBlock> blocks{ScatterBlock{0, 1, nd, 1, (long long)ds_off}};
        if ((st = split_project(c, pl, nd, n, nmtile, nkstep, (const SliceDesc*)U.desc.p, (const int*)U.es.p,
                                (const int*)U.kexp.p, blocks)) != P2_OK)
          return st;
      }
      ds_off += nd;
      continue;
    }
    const size_t per = (size_t)nd * c->V3 * 16;
    const int tc = (int)std::max<size_t>(1, std::min<size_t>(c->ws_budget / std::max<size_t>(per, 1), (size_t)T));
    for (int c0 = 0; c0 < n_all; c0 += tc) {
      const int n = std::min(tc, n_all - c0);
      P2_TRY(c, c->cbuf.ensure((size_t)n * per), "position buffer alloc");
      P2_TRY(c, U.slices.ensure((size_t)n * sizeof(UdscSlice)), "slice alloc");
      P2_TRY(c,
             cudaMemcpyAsync(U.slices.p, sl.data() + c0, (size_t)n * sizeof(UdscSlice), cudaMemcpyHostToDevice,
                             c->stream),
             "slice upload");
      UdscArgs a{};
      a.p0 = (const Cx<double>*)v[0]->data;
      a.p1 = (const Cx<double>*)v[1]->data;
      a.p2 = (const Cx<double>*)v[2]->data;
      a.vol0 = c->V3 * v[0]->nt;
      a.vol1 = c->V3 * v[1]->nt;
      a.vol2 = c->V3 * v[2]->nt;
      a.sl = (const UdscSlice*)U.slices.p;
      a.ntau = n;
      a.V3 = (int)c->V3;
      a.nd = nd;
      a.plan = (const int*)U.plan[p].p;
      a.out = (Cx<double>*)c->cbuf.p;
      {
        ProfScope ps(c, "contract_udsc_fp64");
        P2_TRY(c, launch_contract_udsc(a, c->nsm, c->stream), "udsc contraction");
      }
      ProjArgs pa{};
      pa.c = c->cbuf.p;
      pa.sT = (long long)nd * c->V3;
      pa.sK = c->V3;
      pa.ntau = n;
      pa.K = nd;
      pa.V3 = (int)c->V3;
      pa.nmom = pl.nmom;
      pa.Lx = c->Ll[0];
      pa.Ly = c->Ll[1];
      pa.Lz = c->Ll[2];
      pa.Lmax = pl.Lmax;
      pa.tab = (const double*)c->ptab.p;
      const int ptiles = (pl.nmom + 63) / 64, ktiles = (nd + 31) / 32;
      int nsplit = (2 * c->nsm + ptiles * ktiles * n - 1) / (ptiles * ktiles * n);
      nsplit = std::max(1, std::min(nsplit, (int)((c->V3 + 255) / 256)));
      pa.chunk = (int)((((c->V3 + nsplit - 1) / nsplit) + 15) / 16 * 16);
      pa.nsplit = (int)((c->V3 + pa.chunk - 1) / pa.chunk);
      P2_TRY(c, c->part.ensure((size_t)n * pa.nsplit * pl.nmom * nd * 16), "partials alloc");
      pa.part = (double*)c->part.p;
      {
        ProfScope ps(c, "project_fp64");
        P2_TRY(c, launch_project_fp64(pa, c->stream), "projection kernel");
      }
      std::vector<SliceDesc> desc(n);
      for (int i = 0; i < n; i++) {
        std::memset(&desc[i], 0, sizeof(SliceDesc));
        desc[i].out = dres;
        desc[i].tau = taus[c0 + i];
        desc[i].totalT = r->totalT;
        for (int d = 0; d < 3; d++) desc[i].x0[d] = r->source[d];
      }
      P2_TRY(c, U.desc.ensure((size_t)n * sizeof(SliceDesc)), "descriptor alloc");
      P2_TRY(c,
             cudaMemcpyAsync(U.desc.p, desc.data(), (size_t)n * sizeof(SliceDesc), cudaMemcpyHostToDevice,
                             c->stream),
             "descriptor upload");
      ScatterArgs sa{};
      sa.part = (const double*)c->part.p;
      sa.ntau = n;
      sa.nsplit = pa.nsplit;
      sa.nmom = pl.nmom;
      sa.K = nd;
      sa.nblocks = 1;
      sa.blk[0] = ScatterBlock{0, 1, nd, 1, (long long)ds_off};
      sa.sl = (const SliceDesc*)U.desc.p;
      sa.moms = (const int*)c->moms.p;
      for (int d = 0; d < 3; d++) sa.L[d] = c->g.L[d];
      {
        ProfScope ps(c, "reduce_scatter");
        P2_TRY(c, launch_scatter(sa, c->stream), "reduction kernel");
      }
    }
    ds_off += nd;
  }
  if (r->out_location == P2_HOST) {
    P2_TRY(c, cudaMemcpyAsync(r->out, dres, total * 16, cudaMemcpyDeviceToHost, c->stream), "result download");
    P2_TRY(c, cudaStreamSynchronize(c->stream), "result download");
  }
  return P2_OK;
}

}  // extern "C"
