// Site-local contractions, one lattice site per half-warp (16 lanes).
//
// The reference evaluates every output component of a site in one thread,
// unfactorised (lib/kernels/PLEGMA_baryons_NtoN.cu:6-46: 16 (mu,mu') x 16 spin
// terms x 36 colour terms; PLEGMA_baryons_deltas.cu:7-110 likewise with 8 or 6
// Wick terms; PLEGMA_mesonsAll.cuh:34-82: 9 colour products per spin term per
// Gamma pair).  Here the same sums are regrouped so that the 16 lanes of a
// half-warp share one site and every lane does an equal share.
//
// Baryons (nucleon C g5, Delta C g_k).  Every Wick term is a product of three
// propagator lines X[nu][s1'] Y[lam][s2'] Z[mu][s3'] with the sink diquark
// (nu, lam) contracted with Gamma and the source spins (s1', s2', s3') a
// permutation of (nu', lam', mu') (lam', nu' contracted with Gamma-bar).
// Summing the sink diquark first gives, on lane (x', y') = (l >> 2, l & 3),
//   G^{XY}[c][e] = sum_{(nu,lam)} sA sum eps_abc eps_{c1 c2 e} X[nu][x'][a][c1] Y[lam][y'][b][c2]
// (144 complex products per lane), and every term is +-G contracted with Z:
//   mu' on X's source slot (slot 1): P[m] = f1 sum G[c][e] Z[m][z1][c][e], summed over y'
//   mu' on Y's source slot (slot 2): P[m] = f2 sum G[c][e] Z[m][z2][c][e], summed over x'
//   mu' on Z (type a):                D = sum over the 16 lanes of fa G, T = sum D Z[mu][mu']
// with f1 = -(c1A sA1 - c1B sB1), f2 = c2A sA2 - c2B sB2, fa = cN sN - cL sL from
// per-lane descriptors (spin.diquark_lane_tables) and the Wick coefficients c.
// Swapping the two diquark lines transposes the lanes: G^{YX}(y',x') =
// sign G^{XY}(x',y'), sign -1 for C g5 (antisymmetric), +1 for C g_k.
//   nucleon, per dataset: direct term = type a (cN = 1), exchange = slot 1 (c1A = -1)
//   -> 144 + 45 products per lane for the first dataset, 45 for the second
//   (formed on the transposed lanes, so G^{ud} never moves between lanes);
//   the reference spends ~1.1e5 per site and dataset.
// On the FP32 tile the colour sums run as paired FMAs (fma.rn.f32x2) with two
// accumulators per complex output: the shared-memory operand enters as its
// natural (Re, Im) pair and only the register operand is broadcast.
//
// Mesons, all 16 x 16 (G_sink, G_src):
//   C[g1][g2] = sum G1[d][a] A[a][b] G2[b][z] conj(B[d][z]) over spin and colour.
//   M_{a d}[b][z] = sum_{colour} A[a b] conj(B[d z])   (lane = (a, d), 144 products)
//   N_{a d}[g2]   = sum_b G2[b][pi2(b)] M_{a d}[b][pi2(b)]
//   C[g1][g2]     = sum_d G1[d][pi1(d)] N_{pi1(d) d}[g2]  (lane = g1, shuffles).
// Every Gamma row is a unit phase times a Walsh character
// (G[d][d ^ m] = r (-1)^{popcount(s & d)}), so both Gamma stages are 4-point
// Walsh-Hadamard transforms and the phases r_g1 r_g2 factor out of the sums.
#pragma once
#include "p2_common.cuh"

namespace p2 {

// Source-side descriptor of a diquark table for lane (x' = l >> 2, y' = l & 3).
struct DiquarkLane {
  int z1, sA1, sB1, z2, sA2, sB2, sN, sL;
};

// Per-lane table entries packed into registers (the tables are indexed by
// lane, so reading them from constant memory inside the site loop would
// serialise the half-warp): a diquark lane descriptor as 8 fields of 4 bits
// (value + 1), and the sink-Gamma stage of the mesons (spin.meson_lane_table):
// the lane's sink Gamma g1 (4 bits), then Re + 1, Im + 1 of its phase r_g1
// (2 bits each).
struct LaneTables {
  unsigned nuc;       // nucleon C g5 descriptor
  unsigned nucT;      // the same for the transposed lane ((l & 3) << 2) | (l >> 2)
  unsigned delta[3];  // Delta C g_k descriptors, k = 1..3
  unsigned light[3];  // NtoR, RtoN, RtoR descriptors (spin.light_lane_tables)
  unsigned lg5;       // their g5 signs, 2 bits each (value + 1)
  unsigned mes;       // meson stage
  __device__ __forceinline__ int meson_g1() const { return (int)(mes & 15u); }
};

__constant__ int c_nuc_lane[16][8] = P2_INIT_NucLane;
__constant__ int c_delta_lane[3][16][8] = P2_INIT_DeltaLane;
__constant__ int c_meson_lane[16][3] = P2_INIT_MesonLane;
__constant__ int c_light_lane[3][16][8] = P2_INIT_LightLane;
__constant__ int c_light_g5[16][3] = P2_INIT_LightG5;

// ---- shared-memory views of one site's two propagators --------------------
// Spin block b = mu * 4 + nu of flavour f is block 16 f + b; colour (a, b) is
// entry a * 3 + b of the block.
//
// Plain FP64 tile: row of 2 x 144 complex, block at 9 * block.
struct RowF64 {
  typedef double R;
  const Cx<double>* p;
  __device__ __forceinline__ void pair(int blk, int k, Cx<double>& v0, Cx<double>& v1) const {
    v0 = p[blk * 9 + 2 * k];
    v1 = p[blk * 9 + 2 * k + 1];
  }
  __device__ __forceinline__ Cx<double> last(int blk) const { return p[blk * 9 + 8]; }
  __device__ __forceinline__ void load9(int blk, Cx<double> v[9]) const {
#pragma unroll
    for (int i = 0; i < 9; i++) v[i] = p[blk * 9 + i];
  }
};

// Split-form FP32 tile: every block padded to 10 complex = five 16-byte units
// (colours 2k, 2k+1 in unit k, colour 8 and a spare slot in unit 4), so a
// block is four 16-byte loads and one 8-byte load at fixed offsets from a
// per-lane base.  Rows are 161 units apart (one unit of padding): the
// transposing writes of 16 sites then start in 8 different bank groups,
// and the two sites of a warp read disjoint bank groups.
constexpr int kRow32 = 322;  // complex per site row (32 blocks x 10 + 2)
// Position of spin block blk = 16 f + 4 mu + nu in the row.  PERM = false:
// position blk.  PERM = true: the blocks of a flavour are placed so that the
// four blocks of any fixed mu (nu = 0..3), of any fixed nu (mu = 0..3) and
// the eight of mu in {0, 1} or {2, 3} sit at positions distinct mod 8, i.e.
// in different bank groups (a position is 5 units and 5 is invertible mod
// 8): position (nu + 4 (mu & 1) + (mu >> 1)) mod 8 + 8 (mu >> 1).  The loads
// whose block varies over the lanes (the mesons' A[al][b] and B[de][z], the
// diquarks' X[nu][x'] and Y[lam][y'], the slot and type-a terms) then fetch
// their 4 or 8 distinct units without bank conflicts (ncu, nucleon + mesons
// at 32^3 x 16: shared-load bank conflicts 44.9 M -> 17.8 M per launch), at
// the price of per-lane position registers, so the Delta instantiation,
// whose registers are fuller, keeps PERM = false.
template <bool PERM>
__host__ __device__ __forceinline__ constexpr int row32_pos(int blk) {
  return PERM ? (blk & ~15) | ((((blk & 3) + 4 * ((blk >> 2) & 1) + ((blk >> 3) & 1)) & 7) + 8 * ((blk >> 3) & 1))
              : blk;
}
template <bool PERM = false>
__device__ __forceinline__ int row32_unit(int blk, int k) {
  return row32_pos<PERM>(blk) * 5 + k;
}

template <bool PERM>
struct RowF32T {
  typedef float R;
  static constexpr bool kPerm = PERM;
  const Cx<float>* p;
  __device__ __forceinline__ void pair(int blk, int k, Cx<float>& v0, Cx<float>& v1) const {
    const float4 q = *reinterpret_cast<const float4*>(p + 2 * row32_unit<PERM>(blk, k));
    v0 = cx<float>(q.x, q.y);
    v1 = cx<float>(q.z, q.w);
  }
  __device__ __forceinline__ Cx<float> last(int blk) const { return p[2 * row32_unit<PERM>(blk, 4)]; }
  __device__ __forceinline__ void load9(int blk, Cx<float> v[9]) const {
#pragma unroll
    for (int k = 0; k < 4; k++) pair(blk, k, v[2 * k], v[2 * k + 1]);
    v[8] = last(blk);
  }
};
using RowF32 = RowF32T<false>;

constexpr int kU = 0, kD = 16;  // block offsets of the u and d propagators in a row

__device__ __forceinline__ unsigned pack_diquark_lane(const int (*t)[8], int l) {
  unsigned v = 0;
#pragma unroll
  for (int f = 0; f < 8; f++) v |= (unsigned)(t[l][f] + 1) << (4 * f);
  return v;
}

__device__ __forceinline__ DiquarkLane unpack_diquark_lane(unsigned v) {
  DiquarkLane d;
  d.z1 = (int)((v >> 0) & 15u) - 1;
  d.sA1 = (int)((v >> 4) & 15u) - 1;
  d.sB1 = (int)((v >> 8) & 15u) - 1;
  d.z2 = (int)((v >> 12) & 15u) - 1;
  d.sA2 = (int)((v >> 16) & 15u) - 1;
  d.sB2 = (int)((v >> 20) & 15u) - 1;
  d.sN = (int)((v >> 24) & 15u) - 1;
  d.sL = (int)((v >> 28) & 15u) - 1;
  return d;
}

__device__ __forceinline__ LaneTables load_lane_tables(int l) {
  LaneTables t;
  t.nuc = pack_diquark_lane(c_nuc_lane, l);
  t.nucT = pack_diquark_lane(c_nuc_lane, ((l & 3) << 2) | (l >> 2));
#pragma unroll
  for (int g = 0; g < 3; g++) t.delta[g] = pack_diquark_lane(c_delta_lane[g], l);
#pragma unroll
  for (int j = 0; j < 3; j++) t.light[j] = pack_diquark_lane(c_light_lane[j], l);
  t.lg5 = (unsigned)(c_light_g5[l][0] + 1) | ((unsigned)(c_light_g5[l][1] + 1) << 2) |
          ((unsigned)(c_light_g5[l][2] + 1) << 4);
  t.mes = (unsigned)c_meson_lane[l][0] | ((unsigned)(c_meson_lane[l][1] + 1) << 4) |
          ((unsigned)(c_meson_lane[l][2] + 1) << 6);
  return t;
}

// q += sgn * P^{XY}_{(nu, lam)} for lane (x', y'):
//   P[c][e] = sum eps_abc eps_{c1 c2 e} X[nu][x'][a][c1] Y[lam][y'][b][c2]
// (36 complex products); X and Y are block offsets (kU, kD) of the two
// diquark lines in the site row.
template <typename Row>
__device__ __forceinline__ void diquark_acc(const Row& row, int X, int Y, int nu, int lam, typename Row::R sgn,
                                            int xp, int yp, Cx<typename Row::R> q[9]) {
  typedef typename Row::R R;
  Cx<R> a[9], b[9];
  row.load9(X + nu * 4 + xp, a);
  row.load9(Y + lam * 4 + yp, b);
#pragma unroll
  for (int i = 0; i < 9; i++) a[i] = cscale(a[i], sgn);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const int c1 = (c + 1) % 3, c2 = (c + 2) % 3;
#pragma unroll
    for (int e = 0; e < 3; e++) {
      const int e1 = (e + 1) % 3, e2 = (e + 2) % 3;
      Cx<R>& r = q[c * 3 + e];
      cmac(r, a[c1 * 3 + e1], b[c2 * 3 + e2]);
      cmsub(r, a[c1 * 3 + e2], b[c2 * 3 + e1]);
      cmsub(r, a[c2 * 3 + e1], b[c1 * 3 + e2]);
      cmac(r, a[c2 * 3 + e2], b[c1 * 3 + e1]);
    }
  }
}

// G^{XY} = sum over a sink table sink[iA] = (nu, lam, sA) of sA P^{XY}_{(nu, lam)},
// the table known at compile time (S = 0: nucleon C g5,
// 1..3: Delta C g_k, 4: C): signs fold into the products, block offsets into
// the load addresses.
__host__ __device__ constexpr int sink_entry(int S, int i, int f) {
  return S == 0 ? kNucSink[i][f] : S <= 3 ? kDeltaSink[S - 1][i][f] : kCSink[i][f];
}
template <int S, int iA, typename Row>
__device__ __forceinline__ void diquark_acc_ct(const Row& row, int X, int Y, int xp, int yp,
                                               Cx<typename Row::R> q[9]) {
  constexpr int nu = sink_entry(S, iA, 0), lam = sink_entry(S, iA, 1), sg = sink_entry(S, iA, 2);
  diquark_acc(row, X, Y, nu, lam, typename Row::R(sg), xp, yp, q);
}
// FP32 tile: the same products with paired FMAs and two accumulators per
// output, (ax bx, ax by) and (ay bx, ay by): b enters as its natural (Re, Im)
// pair (and its negation for the subtracted terms), a as broadcasts shared
// by its four terms.
template <int nu, int lam, int sg, typename Row>
__device__ __forceinline__ void dq_acc_f32(const Row& row, int X, int Y, int xp, int yp, f32x2 px[9], f32x2 py[9]) {
  Cx<float> a[9], b[9];
  row.load9(X + nu * 4 + xp, a);
  row.load9(Y + lam * 4 + yp, b);
  f32x2 bp[9], bn[9];
#pragma unroll
  for (int i = 0; i < 9; i++) {
    bp[i] = f2pack(b[i].x, b[i].y);
    bn[i] = f2pack(-b[i].x, -b[i].y);
  }
  auto term = [&](int o, int ia, int ib, int sign) {
    const f32x2 bb = sign * sg > 0 ? bp[ib] : bn[ib];
    px[o] = f2fma(f2pack(a[ia].x, a[ia].x), bb, px[o]);
    py[o] = f2fma(f2pack(a[ia].y, a[ia].y), bb, py[o]);
  };
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const int c1 = (c + 1) % 3, c2 = (c + 2) % 3;
#pragma unroll
    for (int e = 0; e < 3; e++) {
      const int e1 = (e + 1) % 3, e2 = (e + 2) % 3, o = c * 3 + e;
      term(o, c1 * 3 + e1, c2 * 3 + e2, 1);
      term(o, c1 * 3 + e2, c2 * 3 + e1, -1);
      term(o, c2 * 3 + e1, c1 * 3 + e2, -1);
      term(o, c2 * 3 + e2, c1 * 3 + e1, 1);
    }
  }
}

template <int S, int iA, typename Row>
__device__ __forceinline__ void diquark_acc_ct_f32(const Row& row, int X, int Y, int xp, int yp, f32x2 px[9],
                                                   f32x2 py[9]) {
  dq_acc_f32<sink_entry(S, iA, 0), sink_entry(S, iA, 1), sink_entry(S, iA, 2)>(row, X, Y, xp, yp, px, py);
}
__device__ __forceinline__ void dq_fin_f32(const f32x2 px[9], const f32x2 py[9], Cx<float> q[9]) {
#pragma unroll
  for (int i = 0; i < 9; i++) {
    float ax, ay, bx, by;
    f2unpack(px[i], ax, ay);  // (sum ax bx, sum ax by)
    f2unpack(py[i], bx, by);  // (sum ay bx, sum ay by)
    q[i] = cx<float>(ax - by, ay + bx);
  }
}

// q = s1 P^{XY}_{(nu1, lam1)} + s2 P^{XY}_{(nu2, lam2)} (the Delta's shared
// diagonal pairs), paired FMAs on the FP32 tile
template <int nu1, int lam1, int s1, int nu2, int lam2, int s2, typename Row>
__device__ __forceinline__ void diquark_pair_ct(const Row& row, int X, int Y, int xp, int yp,
                                                Cx<typename Row::R> q[9]) {
  typedef typename Row::R R;
  if constexpr (sizeof(R) == 4) {
    f32x2 px[9], py[9];
#pragma unroll
    for (int i = 0; i < 9; i++) px[i] = py[i] = f2pack(0.f, 0.f);
    dq_acc_f32<nu1, lam1, s1>(row, X, Y, xp, yp, px, py);
    dq_acc_f32<nu2, lam2, s2>(row, X, Y, xp, yp, px, py);
    dq_fin_f32(px, py, q);
  } else {
#pragma unroll
    for (int i = 0; i < 9; i++) q[i] = czero<R>();
    diquark_acc(row, X, Y, nu1, lam1, R(s1), xp, yp, q);
    diquark_acc(row, X, Y, nu2, lam2, R(s2), xp, yp, q);
  }
}

template <int S, typename Row>
__device__ __forceinline__ void diquark_G_ct(const Row& row, int X, int Y, int xp, int yp, Cx<typename Row::R> q[9]) {
  typedef typename Row::R R;
  if constexpr (sizeof(R) == 4) {
    f32x2 px[9], py[9];
#pragma unroll
    for (int i = 0; i < 9; i++) px[i] = py[i] = f2pack(0.f, 0.f);
    diquark_acc_ct_f32<S, 0>(row, X, Y, xp, yp, px, py);
    diquark_acc_ct_f32<S, 1>(row, X, Y, xp, yp, px, py);
    diquark_acc_ct_f32<S, 2>(row, X, Y, xp, yp, px, py);
    diquark_acc_ct_f32<S, 3>(row, X, Y, xp, yp, px, py);
    dq_fin_f32(px, py, q);
  } else {
#pragma unroll
    for (int i = 0; i < 9; i++) q[i] = czero<R>();
    diquark_acc_ct<S, 0>(row, X, Y, xp, yp, q);
    diquark_acc_ct<S, 1>(row, X, Y, xp, yp, q);
    diquark_acc_ct<S, 2>(row, X, Y, xp, yp, q);
    diquark_acc_ct<S, 3>(row, X, Y, xp, yp, q);
  }
}

// Type-a weights fa = cN sN - cL sL of every source table vanish outside one
// class {l0, l0 ^ 5, l0 ^ 10, l0 ^ 15} of lanes, so their sum over the
// half-warp takes two butterfly steps (xor 5, xor 10) and a broadcast from
// l0.  Under the lane transpose (x', y') -> (y', x') the weights are
// symmetric or antisymmetric (tau = +1 / -1), so for G^{YX} = s G^{XY}
// transposed the type-a sum is s tau times that of G^{XY}.  Both facts are
// checked on the generated tables at compile time.
__host__ __device__ constexpr int typea_lane(const int (&t)[16][8]) {
  for (int l = 0; l < 16; l++)
    if (t[l][6] || t[l][7]) return l;
  return 0;
}
__host__ __device__ constexpr bool typea_one_class(const int (&t)[16][8]) {
  const int l0 = typea_lane(t);
  for (int l = 0; l < 16; l++) {
    const int d = l ^ l0;
    if ((t[l][6] || t[l][7]) && d != 0 && d != 5 && d != 10 && d != 15) return false;
  }
  return true;
}
__host__ __device__ constexpr int typea_tau(const int (&t)[16][8]) {
  bool sym = true, anti = true;
  for (int l = 0; l < 16; l++) {
    const int lt = ((l & 3) << 2) | (l >> 2);
    for (int f = 6; f < 8; f++) {
      sym = sym && t[lt][f] == t[l][f];
      anti = anti && t[lt][f] == -t[l][f];
    }
  }
  return sym ? 1 : anti ? -1 : 0;
}
static_assert(typea_one_class(kNucLane) && typea_one_class(kDeltaLane[0]) && typea_one_class(kDeltaLane[1]) &&
                  typea_one_class(kDeltaLane[2]) && typea_one_class(kLightLane[0]) &&
                  typea_one_class(kLightLane[1]) && typea_one_class(kLightLane[2]),
              "type-a weights outside one lane class");
static_assert(typea_tau(kNucLane) == -1 && typea_tau(kLightLane[0]) == -1 && typea_tau(kLightLane[1]) == -1 &&
                  typea_tau(kLightLane[2]) == -1,
              "nucleon-type type-a weights not antisymmetric under the lane transpose");
static_assert(typea_tau(kDeltaLane[0]) == 1 && typea_tau(kDeltaLane[1]) == 1 && typea_tau(kDeltaLane[2]) == 1,
              "Delta type-a weights not symmetric under the lane transpose");
static_assert(typea_lane(kDeltaLane[0]) == 0 && typea_lane(kDeltaLane[1]) == 0 && typea_lane(kDeltaLane[2]) == 1,
              "Delta type-a lanes");

// sum_i g[i] z[i] over the 9 colour entries.  FP32: paired FMAs with two
// accumulators, (gx zx, gx zy) and (gy zx, gy zy), so that z enters as the
// natural (Re, Im) pair of its shared-memory load and only g is broadcast
// (once per g for all the dot products it takes part in).
template <typename R>
__device__ __forceinline__ Cx<R> cdot9(const Cx<R> g[9], const Cx<R> z[9]) {
  Cx<R> r = czero<R>();
#pragma unroll
  for (int i = 0; i < 9; i++) cmac(r, g[i], z[i]);
  return r;
}
template <>
__device__ __forceinline__ Cx<float> cdot9<float>(const Cx<float> g[9], const Cx<float> z[9]) {
  f32x2 px = f2pack(0.f, 0.f), py = f2pack(0.f, 0.f);
#pragma unroll
  for (int i = 0; i < 9; i++) {
    const f32x2 zz = f2pack(z[i].x, z[i].y);
    px = f2fma(f2pack(g[i].x, g[i].x), zz, px);
    py = f2fma(f2pack(g[i].y, g[i].y), zz, py);
  }
  float a, b, c, d;
  f2unpack(px, a, b);
  f2unpack(py, c, d);
  return cx<float>(a - d, b + c);
}

// G^{YX} from G^{XY}: move lane (y', x') to lane (x', y') with the table's sign.
template <typename R>
__device__ __forceinline__ void diquark_transpose(Cx<R> q[9], int l, unsigned mask, R sign) {
  const int src = ((l & 3) << 2) | (l >> 2);
#pragma unroll
  for (int i = 0; i < 9; i++) q[i] = cscale(shfl_idx16(q[i], src, mask), sign);
}

// Slot terms of one group of Wick terms sharing G and the third line Z (block
// offset in the site row); returns the lane's share of T[mu = l >> 2][mu' = l & 3].
//   slot 2: T[mu][mu'] = sum_{x'} f2 sum_ce G(x', mu')[c][e] Z[mu][z2][c][e]
//   slot 1: T[mu][mu'] = sum_{y'} f1 sum_ce G(mu', y')[c][e] Z[mu][z1][c][e]
template <bool S1, bool S2, typename Row>
__device__ __forceinline__ Cx<typename Row::R> diquark_slots(const Cx<typename Row::R> g[9], const Row& row, int Z,
                                                             const DiquarkLane& dl, int l, unsigned mask, int c1A,
                                                             int c1B, int c2A, int c2B) {
  typedef typename Row::R R;
  Cx<R> r = czero<R>();
  // the four m of a slot reduced over four lanes as a reduce-scatter: the lane
  // of bit b1 = bit hb of the lane index keeps m in {2 b1, 2 b1 + 1}, then the
  // lane of bit b0 = bit lb keeps m = 2 b1 + b0
  auto scatter = [&](Cx<R> (&P)[4], int hb, int lb) {
    const bool b1 = (l >> hb) & 1, b0 = (l >> lb) & 1;
    const Cx<R> s0 = b1 ? P[0] : P[2], s1 = b1 ? P[1] : P[3];
    Cx<R> k0 = b1 ? P[2] : P[0], k1 = b1 ? P[3] : P[1];
    k0 = k0 + shfl_xor16(s0, 1 << hb, mask);
    k1 = k1 + shfl_xor16(s1, 1 << hb, mask);
    const Cx<R> s = b0 ? k0 : k1;
    const Cx<R> k = b0 ? k1 : k0;
    return k + shfl_xor16(s, 1 << lb, mask);
  };
  if constexpr (sizeof(R) == 8) {
    // FP64: one m at a time (four m of FP64 sums held at once spill)
    const int mu = l >> 2, mup = l & 3;
    if (S2) {
      const R f2 = R(c2A * dl.sA2 - c2B * dl.sB2);
#pragma unroll 1
      for (int m = 0; m < 4; m++) {
        Cx<R> z[9];
        row.load9(Z + m * 4 + dl.z2, z);
        Cx<R> p2 = czero<R>();
#pragma unroll
        for (int i = 0; i < 9; i++) cmac(p2, g[i], z[i]);
        p2 = cscale(p2, f2);
        p2 = p2 + shfl_xor16(p2, 4, mask);
        p2 = p2 + shfl_xor16(p2, 8, mask);
        if (m == mu) r = r + p2;
      }
    }
    if (S1) {
      const R f1 = R(-(c1A * dl.sA1 - c1B * dl.sB1));
      const int src = mup << 2;
#pragma unroll 1
      for (int m = 0; m < 4; m++) {
        Cx<R> z[9];
        row.load9(Z + m * 4 + dl.z1, z);
        Cx<R> p1 = czero<R>();
#pragma unroll
        for (int i = 0; i < 9; i++) cmac(p1, g[i], z[i]);
        p1 = cscale(p1, f1);
        p1 = p1 + shfl_xor16(p1, 1, mask);
        p1 = p1 + shfl_xor16(p1, 2, mask);
        const Cx<R> v = shfl_idx16(p1, src, mask);
        if (m == mu) r = r + v;
      }
    }
    return r;
  }
  if (S2) {
    // slot 2 (sum over x'): lane (x', y' = mu') forms P[m] for T[m][mu'];
    // after the scatter over x' (lane bits 3, 2) lane (x', mu') holds T[x'][mu']
    const R f2 = R(c2A * dl.sA2 - c2B * dl.sB2);
    Cx<R> P[4];
#pragma unroll
    for (int m = 0; m < 4; m++) {
      Cx<R> z[9];
      row.load9(Z + m * 4 + dl.z2, z);
      P[m] = cscale(cdot9(g, z), f2);
    }
    r = r + scatter(P, 3, 2);
  }
  if (S1) {
    // slot 1 (sum over y'): lane (x' = mu', y') forms P[m] for T[m][mu'];
    // after the scatter over y' (lane bits 1, 0) lane (mu', y') holds
    // T[y'][mu'], which lane (mu, mu') takes from the transposed lane
    const R f1 = R(-(c1A * dl.sA1 - c1B * dl.sB1));
    Cx<R> P[4];
#pragma unroll
    for (int m = 0; m < 4; m++) {
      Cx<R> z[9];
      row.load9(Z + m * 4 + dl.z1, z);
      P[m] = cscale(cdot9(g, z), f1);
    }
    r = r + shfl_idx16(scatter(P, 1, 0), ((l & 3) << 2) | (l >> 2), mask);
  }
  return r;
}

// Slot-1 terms of the Wick-transposed diquark G^{YX}(x', y') = sign G^{XY}(y', x')
// without moving G: lane (a, b) holds G^{XY}(a, b) and forms the terms of
// the transposed lane (x', y') = (b, a) with that lane's descriptor dlT,
//   P[m] = f1(dlT) sign sum_ce G^{XY}(a, b)[c][e] Z[m][z1(dlT)][c][e];
// their sum over y' = a (lane bits 3, 2) leaves T[a][b] on lane (a, b),
// which is T[mu][mu'] of the lane itself.
template <typename Row>
__device__ __forceinline__ Cx<typename Row::R> diquark_slot1_transposed(const Cx<typename Row::R> g[9], const Row& row,
                                                                        int Z, const DiquarkLane& dlT, int l,
                                                                        unsigned mask, int c1A, int c1B,
                                                                        typename Row::R sign) {
  typedef typename Row::R R;
  const R f1 = sign * R(-(c1A * dlT.sA1 - c1B * dlT.sB1));
  if constexpr (sizeof(R) == 8) {
    const int mu = l >> 2;
    Cx<R> r = czero<R>();
#pragma unroll 1
    for (int m = 0; m < 4; m++) {
      Cx<R> z[9];
      row.load9(Z + m * 4 + dlT.z1, z);
      Cx<R> p = czero<R>();
#pragma unroll
      for (int i = 0; i < 9; i++) cmac(p, g[i], z[i]);
      p = cscale(p, f1);
      p = p + shfl_xor16(p, 4, mask);
      p = p + shfl_xor16(p, 8, mask);
      if (m == mu) r = r + p;
    }
    return r;
  } else {
    Cx<R> P[4];
#pragma unroll
    for (int m = 0; m < 4; m++) {
      Cx<R> z[9];
      row.load9(Z + m * 4 + dlT.z1, z);
      P[m] = cscale(cdot9(g, z), f1);
    }
    // reduce-scatter over lane bits 3, 2: lane (a, b) keeps m = a
    const bool b1 = (l >> 3) & 1, b0 = (l >> 2) & 1;
    const Cx<R> s0 = b1 ? P[0] : P[2], s1 = b1 ? P[1] : P[3];
    Cx<R> k0 = b1 ? P[2] : P[0], k1 = b1 ? P[3] : P[1];
    k0 = k0 + shfl_xor16(s0, 8, mask);
    k1 = k1 + shfl_xor16(s1, 8, mask);
    const Cx<R> sv = b0 ? k0 : k1;
    const Cx<R> kv = b0 ? k1 : k0;
    return kv + shfl_xor16(sv, 4, mask);
  }
}

// Type-a terms: D = sum over the 16 lanes of fa G (all lanes get D; fa is
// zero outside the lane class of l0), then the lane's
// T[mu][mu'] = sum_ce D[c][e] Z[mu][mu'][c][e].
template <typename R>
__device__ __forceinline__ void diquark_D(const Cx<R> g[9], R fa, unsigned mask, int l0, Cx<R> D[9]) {
#pragma unroll
  for (int i = 0; i < 9; i++) {
    Cx<R> d = cscale(g[i], fa);
    d = d + shfl_xor16(d, 5, mask);
    d = d + shfl_xor16(d, 10, mask);
    D[i] = shfl_idx16(d, l0, mask);
  }
}
template <typename Row>
__device__ __forceinline__ Cx<typename Row::R> diquark_typea(const Cx<typename Row::R> D[9], const Row& row, int Z,
                                                             int l) {
  typedef typename Row::R R;
  Cx<R> z[9];
  row.load9(Z + (l >> 2) * 4 + (l & 3), z);
  return cdot9(D, z);
}

// All Wick terms of one group: slot terms with the Wick coefficients
// (c1A, c1B, c2A, c2B) plus the type-a terms of the sum D.
template <bool S1, bool S2, typename Row>
__device__ __forceinline__ Cx<typename Row::R> diquark_eval(const Cx<typename Row::R> g[9], const Row& row, int Z,
                                                            const DiquarkLane& dl, int l, unsigned mask, int c1A,
                                                            int c1B, int c2A, int c2B, const Cx<typename Row::R> D[9]) {
  return diquark_slots<S1, S2>(g, row, Z, dl, l, mask, c1A, c1B, c2A, c2B) + diquark_typea(D, row, Z, l);
}

// Nucleon C g5, both datasets: out[0] = proton (u u d), out[1] = neutron (d d u),
// for lane (mu = l >> 2, mu' = l & 3).
template <typename Row>
__device__ __forceinline__ void nucleon_site(const Row& row, const LaneTables& lt, int l, unsigned mask,
                                             Cx<typename Row::R> out[2]) {
  typedef typename Row::R R;
  Cx<R> g[9], D[9];
  diquark_G_ct<0>(row, kU, kD, l >> 2, l & 3, g);  // G^{ud}
  const DiquarkLane dl = unpack_diquark_lane(lt.nuc);
  constexpr int l0 = typea_lane(kNucLane);
  diquark_D(g, R(dl.sN), mask, l0, D);  // cN = 1, cL = 0
  out[0] = diquark_eval<true, false>(g, row, kU, dl, l, mask, -1, 0, 0, 0, D);
  // G^{du}(x', y') = -G^{ud}(y', x'); its type-a sum is (-1)(tau = -1) D
  out[1] = diquark_slot1_transposed(g, row, kD, unpack_diquark_lane(lt.nucT), l, mask, -1, 0, R(-1)) +
           diquark_typea(D, row, kD, l);
}

// M_{al de}[b][z] = sum over colour of A[al][b] conj(B[de][z]).
template <typename Row>
__device__ __forceinline__ void meson_M(const Row& row, int A, int B, int al, int de,
                                        Cx<typename Row::R> M[4][4]) {
  typedef typename Row::R R;
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) M[i][j] = czero<R>();
  // colours in pairs (one 16-byte load per pair in the FP32 tile), then colour 8
#pragma unroll
  for (int k = 0; k < 4; k++) {
    Cx<R> u0[4], u1[4], d0[4], d1[4];
#pragma unroll
    for (int b = 0; b < 4; b++) row.pair(A + al * 4 + b, k, u0[b], u1[b]);
#pragma unroll
    for (int z = 0; z < 4; z++) row.pair(B + de * 4 + z, k, d0[z], d1[z]);
#pragma unroll
    for (int b = 0; b < 4; b++)
#pragma unroll
      for (int z = 0; z < 4; z++) {
        cmac_conj(M[b][z], u0[b], d0[z]);
        cmac_conj(M[b][z], u1[b], d1[z]);
      }
  }
  Cx<R> u[4], d[4];
#pragma unroll
  for (int b = 0; b < 4; b++) u[b] = row.last(A + al * 4 + b);
#pragma unroll
  for (int z = 0; z < 4; z++) d[z] = row.last(B + de * 4 + z);
#pragma unroll
  for (int b = 0; b < 4; b++)
#pragma unroll
    for (int z = 0; z < 4; z++) cmac_conj(M[b][z], u[b], d[z]);
}

// FP32 tile: the same sum with paired FMAs on (Re, Im) pairs,
//   M += (u.x, u.y) * (d.x, d.x) + (u.y, -u.x) * (d.y, d.y),
// two instructions per complex product instead of four.
template <bool PERM>
__device__ __forceinline__ void meson_M(const RowF32T<PERM>& row, int A, int B, int al, int de, Cx<float> Mo[4][4]) {
  f32x2 M[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) M[i][j] = f2pack(0.f, 0.f);
  auto colour = [&](const Cx<float> u[4], const Cx<float> d[4]) {
    f32x2 u1[4], u2[4];
#pragma unroll
    for (int b = 0; b < 4; b++) {
      u1[b] = f2pack(u[b].x, u[b].y);
      u2[b] = f2pack(u[b].y, -u[b].x);
    }
#pragma unroll
    for (int z = 0; z < 4; z++) {
      const f32x2 dx = f2pack(d[z].x, d[z].x), dy = f2pack(d[z].y, d[z].y);
#pragma unroll
      for (int b = 0; b < 4; b++) M[b][z] = f2fma(u2[b], dy, f2fma(u1[b], dx, M[b][z]));
    }
  };
#pragma unroll
  for (int k = 0; k < 4; k++) {
    Cx<float> u0[4], u1[4], d0[4], d1[4];
#pragma unroll
    for (int b = 0; b < 4; b++) row.pair(A + al * 4 + b, k, u0[b], u1[b]);
#pragma unroll
    for (int z = 0; z < 4; z++) row.pair(B + de * 4 + z, k, d0[z], d1[z]);
    colour(u0, d0);
    colour(u1, d1);
  }
  Cx<float> u[4], d[4];
#pragma unroll
  for (int b = 0; b < 4; b++) u[b] = row.last(A + al * 4 + b);
#pragma unroll
  for (int z = 0; z < 4; z++) d[z] = row.last(B + de * 4 + z);
  colour(u, d);
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) f2unpack(M[i][j], Mo[i][j].x, Mo[i][j].y);
}

// v * r_g2 * r_g1, g2 a compile-time constant after unrolling, g1 the lane's sink Gamma.
template <typename R>
__device__ __forceinline__ Cx<R> meson_phase(const LaneTables& lt, int g2, Cx<R> v) {
  constexpr int GR[16][4] = P2_INIT_GammaRe;
  constexpr int GI[16][4] = P2_INIT_GammaIm;
  const int rre = (int)((lt.mes >> 4) & 3u) - 1, rim = (int)((lt.mes >> 6) & 3u) - 1;
  return cunit(cunit(v, GR[g2][0], GI[g2][0]), rre, rim);
}

// Generic meson block of the lines A and B (block offsets): the lane gets
// C[g1][g2] for g2 = 0..15 in out[], g1 = lt.meson_g1() (a permutation of the
// lanes), times conj(r_g1 r_g2) when phased is false; with sink false the
// lane keeps its values before the sink stage.  Lane (al, de) first
// forms, per source class m2, the Walsh-Hadamard transform over b of
// M[b][b ^ m2] (N[g2] / r_g2 at index s_g2); the sink Gamma then runs as a
// Walsh-Hadamard transform over the 4 lanes of the lane's class (two
// butterflies, xor 5 and xor 10), which leaves C[g1][g2] / (r_g1 r_g2) on the
// lane whose spin index de is s_g1 (spin.meson_lane_table).
template <typename Row>
__device__ __forceinline__ void meson_site(const Row& row, int A, int B, const LaneTables& lt, int l, unsigned mask,
                                           bool sink, bool phased, Cx<typename Row::R> out[16]) {
  typedef typename Row::R R;
  const int al = l >> 2, de = l & 3;
  Cx<R> W[4][4];
  {
    Cx<R> M[4][4];
    meson_M(row, A, B, al, de, M);
#pragma unroll
    for (int m2 = 0; m2 < 4; m2++) {
      const Cx<R> a0 = M[0][m2] + M[1][1 ^ m2], a1 = M[0][m2] - M[1][1 ^ m2];
      const Cx<R> a2 = M[2][2 ^ m2] + M[3][3 ^ m2], a3 = M[2][2 ^ m2] - M[3][3 ^ m2];
      W[m2][0] = a0 + a2;
      W[m2][1] = a1 + a3;
      W[m2][2] = a0 - a2;
      W[m2][3] = a1 - a3;
    }
  }
  // local copies: the namespace-scope tables are not addressable in device code
  constexpr int GP[16][4] = P2_INIT_GammaPerm;
  constexpr int GR[16][4] = P2_INIT_GammaRe;
  constexpr int GI[16][4] = P2_INIT_GammaIm;
  auto source_value = [&](int g2) {
    const int ch = (GR[g2][1] == -GR[g2][0] && GI[g2][1] == -GI[g2][0] ? 1 : 0) |
                   (GR[g2][2] == -GR[g2][0] && GI[g2][2] == -GI[g2][0] ? 2 : 0);  // gamma_char(g2)
    return W[GP[g2][0]][ch];
  };
  if (!sink) {
#pragma unroll
    for (int g2 = 0; g2 < 16; g2++) out[g2] = source_value(g2);
    return;
  }
  const R s0 = (de & 1) ? R(-1) : R(1), s1 = (de & 2) ? R(-1) : R(1);
#pragma unroll
  for (int g2 = 0; g2 < 16; g2++) {
    Cx<R> x = source_value(g2);
    Cx<R> p = shfl_xor16(x, 5, mask);
    x = cx<R>(fma(s0, x.x, p.x), fma(s0, x.y, p.y));
    p = shfl_xor16(x, 10, mask);
    x = cx<R>(fma(s1, x.x, p.x), fma(s1, x.y, p.y));
    out[g2] = phased ? meson_phase(lt, g2, x) : x;
  }
}

// ---- Delta C g_k (PLEGMA_baryons_deltas.cu:7-110) ------------------------------
// Wick coefficients (c1A, c1B, c2A, c2B, cN, cL) per G, read off the reference's
// terms: with A the doubly represented flavour,
//   isospin 1/2, G^{AA}, Z = B: (0, 2, 0, -2, 1, -1)        x 1/3
//   isospin 1/2, G^{AB}, Z = A: (-4, 0, 2, -2, 4, 0)        x 1/3
//   isospin 3/2, G^{AA}, Z = A: (-1, 1, 1, -1, 1, -1)
// Both G^{AA} groups have cN = 1, cL = -1, so they share the type-a sum D.
//
// The three sink tables share products: C g_1 and C g_2 use the diagonal
// pairs (nu, nu) with signs (+ - - +) and (+ + - -), so with
// A = P00 - P22 and B = P11 - P33, G_1 = A - B and G_2 = A + B; C g_3 uses
// (0,1), (1,0), (2,3), (3,2) with signs (+ + - -), and for a single flavour
// P^{XX}_{(lam, nu)}(x', y') = P^{XX}_{(nu, lam)}(y', x'), so
// G_3^{XX} = Q + Q^T with Q = P01 - P23 (lane transpose).  For G^{uu} and
// G^{dd} that is 6 products instead of 12 (G^{ud} keeps 12): 24 per site and
// lane instead of 36.  The tables are pinned in the spin-table tests.
//
// For k = g + 1 and lane (mu, mu'), out(g, j, v) receives the final value of
// j = 0: iso-1/2 Delta+ (u,u,d), 1: iso-1/2 Delta0 (d,d,u), 2: iso-3/2
// Delta++ (u,u,u), 3: iso-3/2 Delta- (d,d,d); the G^{ud} part of the
// iso-1/2 values is parked first with part(g, j, v) and read back with
// part_get(g, j) (registers are the scarce resource here).
template <typename Row, typename Out, typename Part, typename PartGet>
__device__ __forceinline__ void delta_site(const Row& row, const LaneTables& lt, int l, unsigned mask, Out&& out,
                                           Part&& part, PartGet&& part_get) {
  typedef typename Row::R R;
  const int xp = l >> 2, yp = l & 3;
  const R third = R(1) / R(3);
  // iso-1/2 partial sums from G^{ud} / G^{du}, completed by the G^{uu} / G^{dd} terms
  // G^{ud} (A = u) and its lane transpose G^{du} (A = d; C g_k is symmetric)
  // C g_1 and C g_2 from the shared diagonal products ga = P00 - P22,
  // gb = P11 - P33 (8 products instead of 12).  FP64: ga and gb formed up
  // front; FP32 (registers are tighter): C g_3 first, then ga and gb, with
  // only C g_2's sum ga + gb held over C g_1's evaluation
  constexpr bool kShare = sizeof(R) == 8;
  Cx<R> ga[9], gb[9];
  if (kShare) {
#pragma unroll
    for (int i = 0; i < 9; i++) ga[i] = gb[i] = czero<R>();
    diquark_acc(row, kU, kD, 0, 0, R(1), xp, yp, ga);
    diquark_acc(row, kU, kD, 2, 2, R(-1), xp, yp, ga);
    diquark_acc(row, kU, kD, 1, 1, R(1), xp, yp, gb);
    diquark_acc(row, kU, kD, 3, 3, R(-1), xp, yp, gb);
  }
  Cx<R> q1[9];  // FP32: C g_2's G^{ud}, formed with C g_1's
#pragma unroll 1
  for (int it = 0; it < 3; it++) {
    const int g = kShare ? it : (it == 0 ? 2 : it - 1);
    Cx<R> q[9], D[9];
    if (kShare && g < 2) {
#pragma unroll
      for (int i = 0; i < 9; i++) q[i] = g == 0 ? ga[i] - gb[i] : ga[i] + gb[i];
    } else if (!kShare && it == 1) {
      diquark_pair_ct<0, 0, 1, 2, 2, -1>(row, kU, kD, xp, yp, q);
      diquark_pair_ct<1, 1, 1, 3, 3, -1>(row, kU, kD, xp, yp, q1);
#pragma unroll
      for (int i = 0; i < 9; i++) {
        const Cx<R> t = q[i];
        q[i] = t - q1[i];
        q1[i] = t + q1[i];
      }
    } else if (!kShare && it == 2) {
#pragma unroll
      for (int i = 0; i < 9; i++) q[i] = q1[i];
    } else {
      diquark_G_ct<3>(row, kU, kD, xp, yp, q);  // g = 2 (C g_3) in both forms
    }
    const DiquarkLane dl = unpack_diquark_lane(g == 0 ? lt.delta[0] : g == 1 ? lt.delta[1] : lt.delta[2]);
    diquark_D(q, R(4 * dl.sN), mask, g == 2 ? 1 : 0, D);  // cN = 4, cL = 0
    part(g, 0, cscale(diquark_eval<true, true>(q, row, kU, dl, l, mask, -4, 0, 2, -2, D), third));
    diquark_transpose<R>(q, l, mask, R(1));  // G^{du}; its type-a sum is (+1)(tau = +1) D
    part(g, 1, cscale(diquark_eval<true, true>(q, row, kD, dl, l, mask, -4, 0, 2, -2, D), third));
  }
  // G^{uu} (pair 0: Delta+ and Delta++) and G^{dd} (pair 1: Delta0 and Delta-)
#pragma unroll 1
  for (int pair = 0; pair < 2; pair++) {
    const int X = pair == 0 ? kU : kD;
    const int O = pair == 0 ? kD : kU;
    Cx<R> ga[9], gb[9];
    diquark_pair_ct<0, 0, 1, 2, 2, -1>(row, X, X, xp, yp, ga);
    diquark_pair_ct<1, 1, 1, 3, 3, -1>(row, X, X, xp, yp, gb);
#pragma unroll
    for (int i = 0; i < 9; i++) {
      const Cx<R> t = ga[i];
      ga[i] = t - gb[i];
      gb[i] = t + gb[i];
    }
#pragma unroll
    for (int g = 0; g < 3; g++) {
      Cx<R> q[9];
      if (g < 2) {
#pragma unroll
        for (int i = 0; i < 9; i++) q[i] = g == 0 ? ga[i] : gb[i];
      } else {
        diquark_pair_ct<0, 1, 1, 2, 3, -1>(row, X, X, xp, yp, q);
        Cx<R> t[9];
#pragma unroll
        for (int i = 0; i < 9; i++) t[i] = q[i];
        diquark_transpose<R>(t, l, mask, R(1));
#pragma unroll
        for (int i = 0; i < 9; i++) q[i] = q[i] + t[i];
      }
      const DiquarkLane dl = unpack_diquark_lane(g == 0 ? lt.delta[0] : g == 1 ? lt.delta[1] : lt.delta[2]);
      Cx<R> iso12 = diquark_slots<true, true>(q, row, O, dl, l, mask, 0, 2, 0, -2);
      Cx<R> iso32 = diquark_slots<true, true>(q, row, X, dl, l, mask, -1, 1, 1, -1);
      Cx<R> D[9];
      diquark_D(q, R(dl.sN + dl.sL), mask, g == 2 ? 1 : 0, D);  // cN = 1, cL = -1 for both groups
      iso12 = iso12 + diquark_typea(D, row, O, l);
      iso32 = iso32 + diquark_typea(D, row, X, l);
      out(g, pair, part_get(g, pair) + cscale(iso12, third));
      out(g, 2 + pair, iso32);
    }
  }
}

// ---- second nucleon interpolator (PLEGMA_baryons_NtoR.cu, _RtoN.cu, _RtoR.cu) ----
// N = eps (u^T C g5 d) u, R = eps (u^T C d) g5 u.  Each variant is the nucleon's
// Wick structure with the sink diquark of its sink interpolator (G^{ud} for
// C g5 or C), the source descriptors of its (sink, source) table, and a g5
// on the open spin of the third quark, which moves values between lanes:
// lane (mu, mu') takes T_NR from lane (mu, mu' ^ 2) (xor 2), T_RN from
// (mu ^ 2, mu') (xor 8), T_RR from (mu ^ 2, mu' ^ 2) (xor 10), with the signs
// of spin.light_lane_tables.  out(j, ds, v): j = 0 NtoR, 1 RtoN, 2 RtoR;
// ds 0 = proton (u u d), 1 = neutron (d d u).
template <typename Row, typename Out>
__device__ __forceinline__ void light_nucleon_site(const Row& row, const LaneTables& lt, int l, unsigned mask,
                                                   bool ntor, bool rton, bool rtor, Out&& out) {
  typedef typename Row::R R;
  constexpr int kCT[1] = P2_INIT_CTransposeSign;
  const R s_nr = R((int)(lt.lg5 & 3u) - 1), s_rn = R((int)((lt.lg5 >> 2) & 3u) - 1);
  const R s_rr = R((int)((lt.lg5 >> 4) & 3u) - 1);
  if (ntor) {
    Cx<R> g[9], D[9];
    diquark_G_ct<0>(row, kU, kD, l >> 2, l & 3, g);  // sink C g5
    const DiquarkLane dl = unpack_diquark_lane(lt.light[0]);
    constexpr int l0 = typea_lane(kLightLane[0]);
    diquark_D(g, R(dl.sN), mask, l0, D);
    const Cx<R> p = diquark_eval<true, false>(g, row, kU, dl, l, mask, -1, 0, 0, 0, D);
    diquark_transpose<R>(g, l, mask, R(-1));
    const Cx<R> n = diquark_eval<true, false>(g, row, kD, dl, l, mask, -1, 0, 0, 0, D);
    out(0, 0, cscale(shfl_xor16(p, 2, mask), s_nr));
    out(0, 1, cscale(shfl_xor16(n, 2, mask), s_nr));
  }
  if (rton || rtor) {
    Cx<R> g[9];
    diquark_G_ct<4>(row, kU, kD, l >> 2, l & 3, g);  // sink C
    const DiquarkLane drn = unpack_diquark_lane(lt.light[1]), drr = unpack_diquark_lane(lt.light[2]);
    constexpr int l0rn = typea_lane(kLightLane[1]), l0rr = typea_lane(kLightLane[2]);
    Cx<R> prn = czero<R>(), prr = czero<R>();
    {
      Cx<R> D[9];
      if (rton) {
        diquark_D(g, R(drn.sN), mask, l0rn, D);
        prn = diquark_eval<true, false>(g, row, kU, drn, l, mask, -1, 0, 0, 0, D);
      }
      if (rtor) {
        diquark_D(g, R(drr.sN), mask, l0rr, D);
        prr = diquark_eval<true, false>(g, row, kU, drr, l, mask, -1, 0, 0, 0, D);
      }
    }
    diquark_transpose<R>(g, l, mask, R(kCT[0]));
    if (rton) {
      Cx<R> D[9];
      diquark_D(g, R(drn.sN), mask, l0rn, D);
      const Cx<R> n = diquark_eval<true, false>(g, row, kD, drn, l, mask, -1, 0, 0, 0, D);
      out(1, 0, cscale(shfl_xor16(prn, 8, mask), s_rn));
      out(1, 1, cscale(shfl_xor16(n, 8, mask), s_rn));
    }
    if (rtor) {
      Cx<R> D[9];
      diquark_D(g, R(drr.sN), mask, l0rr, D);
      const Cx<R> n = diquark_eval<true, false>(g, row, kD, drr, l, mask, -1, 0, 0, 0, D);
      out(2, 0, cscale(shfl_xor16(prr, 10, mask), s_rr));
      out(2, 1, cscale(shfl_xor16(n, 10, mask), s_rr));
    }
  }
}

}  // namespace p2
