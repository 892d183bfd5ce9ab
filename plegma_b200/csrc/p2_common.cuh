// Shared device helpers: complex arithmetic in registers, the propagator
// index map, cp.async staging and half-warp shuffles.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "spin_tables.h"

namespace p2 {

template <typename R>
struct alignas(2 * sizeof(R)) Cx {
  R x, y;
};

template <typename R>
__device__ __forceinline__ Cx<R> cx(R x, R y) {
  Cx<R> c;
  c.x = x;
  c.y = y;
  return c;
}
template <typename R>
__device__ __forceinline__ Cx<R> czero() {
  return cx<R>(R(0), R(0));
}
template <typename R>
__device__ __forceinline__ Cx<R> operator+(Cx<R> a, Cx<R> b) {
  return cx<R>(a.x + b.x, a.y + b.y);
}
template <typename R>
__device__ __forceinline__ Cx<R> operator-(Cx<R> a, Cx<R> b) {
  return cx<R>(a.x - b.x, a.y - b.y);
}
template <typename R>
__device__ __forceinline__ Cx<R> cscale(Cx<R> a, R s) {
  return cx<R>(a.x * s, a.y * s);
}
// acc += a * b
template <typename R>
__device__ __forceinline__ void cmac(Cx<R>& acc, Cx<R> a, Cx<R> b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
}
// acc -= a * b
template <typename R>
__device__ __forceinline__ void cmsub(Cx<R>& acc, Cx<R> a, Cx<R> b) {
  acc.x = fma(-a.x, b.x, acc.x);
  acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(-a.x, b.y, acc.y);
  acc.y = fma(-a.y, b.x, acc.y);
}
// acc += a * conj(b)
template <typename R>
__device__ __forceinline__ void cmac_conj(Cx<R>& acc, Cx<R> a, Cx<R> b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(a.y, b.x, acc.y);
  acc.y = fma(-a.x, b.y, acc.y);
}
template <typename R>
__device__ __forceinline__ Cx<R> cmul(Cx<R> a, Cx<R> b) {
  return cx<R>(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
// a * (re + i im) for re, im in {-1, 0, 1}
template <typename R>
__device__ __forceinline__ Cx<R> cunit(Cx<R> a, int re, int im) {
  return cx<R>(R(re) * a.x - R(im) * a.y, R(re) * a.y + R(im) * a.x);
}

// Walsh factorisation of Gamma g (spin.gamma_walsh): G[d][d ^ m] = r (-1)^{popcount(s & d)}
// with m = pi(0), r = G[0][m] and s read off rows 1 and 2; checked for every row.
// Host side (device code indexes local copies of the tables).
constexpr int gamma_class(int g) { return kGammaPerm[g][0]; }
constexpr int gamma_char(int g) {
  return (kGammaRe[g][1] == -kGammaRe[g][0] && kGammaIm[g][1] == -kGammaIm[g][0] ? 1 : 0) |
         (kGammaRe[g][2] == -kGammaRe[g][0] && kGammaIm[g][2] == -kGammaIm[g][0] ? 2 : 0);
}
constexpr bool gamma_walsh_ok() {
  for (int g = 0; g < 16; g++)
    for (int d = 0; d < 4; d++) {
      const int sd = gamma_char(g) & d, sg = ((sd ^ (sd >> 1)) & 1) ? -1 : 1;
      if (kGammaPerm[g][d] != (d ^ gamma_class(g)) || kGammaRe[g][d] != sg * kGammaRe[g][0] ||
          kGammaIm[g][d] != sg * kGammaIm[g][0])
        return false;
    }
  return true;
}
static_assert(gamma_walsh_ok(), "a Gamma row is not a unit phase times a Walsh character");

// Phase r_g1 r_g2 of C[g1][g2] as i^q, q in 0..3 (the projection's reduction
// applies it when the contraction leaves it out).
constexpr int gamma_phase_q(int g) {
  return kGammaRe[g][0] == 1 ? 0 : kGammaIm[g][0] == 1 ? 1 : kGammaRe[g][0] == -1 ? 2 : 3;
}
constexpr int meson_phase_q(int g1, int g2) { return (gamma_phase_q(g1) + gamma_phase_q(g2)) & 3; }
// Packed float pairs for the paired FP32 FMA (fma.rn.f32x2): one instruction
// updates both halves of a register pair.
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 f2pack(float lo, float hi) {
  f32x2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void f2unpack(f32x2 v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f32x2 f2fma(f32x2 a, f32x2 b, f32x2 c) {
  f32x2 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

// Load-time propagator transform (PropXf codes) of the four spin blocks
// v0 = P[m][n], v1 = P[m][n+2], v2 = P[m+2][n], v3 = P[m+2][n+2] of one colour
// pair (m, n in {0, 1}): rotation P'[mu][nu] = (P[mu][nu] - P[mu+2][nu+2] +
// s i (P[mu][nu+2] + P[mu+2][nu])) / 2 (indices mod 4), then g5 P (P'[mu][nu] =
// P[mu+2][nu]), then the sign.
template <typename R>
__device__ __forceinline__ void prop_group_transform(Cx<R>& v0, Cx<R>& v1, Cx<R>& v2, Cx<R>& v3, int code) {
  const int rot = code & 3;
  if (rot) {
    const R s = rot == 1 ? R(1) : R(-1);
    auto is = [&](Cx<R> x) { return cx<R>(-s * x.y, s * x.x); };
    const Cx<R> a = cscale(v0 - v3 + is(v1 + v2), R(0.5));
    const Cx<R> b = cscale(v1 - v2 + is(v0 + v3), R(0.5));
    const Cx<R> c = cscale(v2 - v1 + is(v3 + v0), R(0.5));
    const Cx<R> d = cscale(v3 - v0 + is(v2 + v1), R(0.5));
    v0 = a;
    v1 = b;
    v2 = c;
    v3 = d;
  }
  if (code & 4) {
    const Cx<R> t0 = v0, t1 = v1;
    v0 = v2;
    v1 = v3;
    v2 = t0;
    v3 = t1;
  }
  if (code & 8) {
    v0 = cscale(v0, R(-1));
    v1 = cscale(v1, R(-1));
    v2 = cscale(v2, R(-1));
    v3 = cscale(v3, R(-1));
  }
}

// Components of transform group q (0..35) of one propagator: colour pair
// cc = q / 4, base (m, n) = ((q % 4) >> 1, q & 1); blocks b, b+2, b+8, b+10.
__device__ __forceinline__ void prop_group_comps(int q, int comp[4]) {
  const int cc = q >> 2, b = ((q & 3) >> 1) * 4 + (q & 1);
  comp[0] = b * 9 + cc;
  comp[1] = (b + 2) * 9 + cc;
  comp[2] = (b + 8) * 9 + cc;
  comp[3] = (b + 10) * 9 + cc;
}

// The same group as (first block b, colour cc): the four components are
// colour cc of blocks b + group_blk(i).
__host__ __device__ constexpr int group_blk(int i) { return i == 0 ? 0 : i == 1 ? 2 : i == 2 ? 8 : 10; }
__device__ __forceinline__ void prop_group_base(int q, int& b, int& cc) {
  cc = q >> 2;
  b = ((q & 3) >> 1) * 4 + (q & 1);
}

// Index of spin block (mu, nu) in a site's 144 components; colour (a, b) adds a*3 + b.
__host__ __device__ constexpr int sblk(int mu, int nu) { return (mu * 4 + nu) * 9; }

// Half-warp shuffles: lanes 0..15 of each half of a warp exchange among themselves.
__device__ __forceinline__ unsigned halfwarp_mask() {
  return (threadIdx.x & 16) ? 0xFFFF0000u : 0x0000FFFFu;
}
template <typename R>
__device__ __forceinline__ Cx<R> shfl_xor16(Cx<R> v, int m, unsigned mask) {
  return cx<R>(__shfl_xor_sync(mask, v.x, m, 16), __shfl_xor_sync(mask, v.y, m, 16));
}
template <typename R>
__device__ __forceinline__ Cx<R> shfl_idx16(Cx<R> v, int src, unsigned mask) {
  return cx<R>(__shfl_sync(mask, v.x, src, 16), __shfl_sync(mask, v.y, src, 16));
}

// Position (slice tl, tile rem of the slice) of a CTA's persistent walk over
// the tiles, advanced by the grid size without divisions: gridDim.x =
// q tiles_per_tau + r, so one step adds q slices and r tiles with a carry.
struct TileCursor {
  int tl, rem, q, r, tpt;
  __device__ __forceinline__ TileCursor(int start, int step, int tiles_per_tau)
      : tl(start / tiles_per_tau), rem(start % tiles_per_tau), q(step / tiles_per_tau), r(step % tiles_per_tau),
        tpt(tiles_per_tau) {}
  __device__ __forceinline__ TileCursor next() const {
    TileCursor n = *this;
    n.tl += q;
    n.rem += r;
    if (n.rem >= tpt) {
      n.rem -= tpt;
      n.tl++;
    }
    return n;
  }
  __device__ __forceinline__ int x0() const { return rem * 16; }  // first site of the 16-site tile
};

// Asynchronous global -> shared copies (LDGSTS).  Bytes beyond src_bytes are zero-filled.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, int src_bytes) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// exp(i 2 pi sum_d p_d x0_d / L_d): the phase that moves a projection with
// origin 0 to the source x0; each p_d x0_d is reduced mod L_d in integers.
__device__ __forceinline__ Cx<double> source_phase(const int* p, const int* x0, const int* L) {
  double frac = 0.0;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    int m = ((p[d] % L[d]) * x0[d]) % L[d];  // |p mod L| and x0 below L: no overflow
    if (m < 0) m += L[d];
    frac += (double)m / (double)L[d];
  }
  double sn, cs;
  sincospi(2.0 * frac, &sn, &cs);
  return cx<double>(cs, sn);
}

}  // namespace p2
