// Site-local contractions, one lattice site per half-warp (16 lanes).
//
// The reference evaluates every output component of a site in one thread,
// unfactorised (lib/kernels/PLEGMA_baryons_NtoN.cu:6-46: 16 (mu,mu') x 16 spin
// terms x 36 colour terms; PLEGMA_mesonsAll.cuh:34-82: 9 colour products per
// spin term per Gamma pair).  Here the same sums are regrouped so that the
// 16 lanes of a half-warp share one site and every lane does an equal share:
//
// Nucleon C g5 (per dataset, A = doubly represented flavour, B = the other):
//   tmp[mu][mu'] = sum_idx val_idx sum_{eps eps'} B[lam lam'][b b']
//                  ( A[nu nu'][a a'] A[mu mu'][c c'] - A[nu mu'][a c'] A[mu nu'][c a'] )
//   direct   : Q[c][c'] = sum_idx val sum_{a,a'} eps eps' A[nu nu'][a a'] B[lam lam'][b b']
//              (lane = idx, 36 complex products, butterfly over the 16 lanes),
//              then T1[mu][mu'] = sum_{c c'} Q[c][c'] A[mu mu'][c c'].
//   exchange : Z[c][a'] = sum_{(nu,lam)} val sum_{a,c'} eps eps' B[lam lam'][b b'] A[nu mu'][a c']
//              (lane = ((lam',nu'), mu'), 144 products, no reduction), then
//              P[mu] = sum_{c a'} Z[c][a'] A[mu nu'][c a'] and T2 = sum over the
//              four nu' lanes (two shuffle levels).
//   Per site and dataset: 3600 complex products instead of the reference's
//   ~1.1e5.
//
// Mesons, all 16 x 16 (G_sink, G_src):
//   C[g1][g2] = sum G1[d][a] A[a][b] G2[b][z] conj(B[d][z]) over spin and colour.
//   M_{a d}[b][z] = sum_{colour} A[a b] conj(B[d z])   (lane = (a, d), 144 products)
//   N_{a d}[g2]   = sum_b G2[b][pi2(b)] M_{a d}[b][pi2(b)]
//   C[g1][g2]     = sum_d G1[d][pi1(d)] N_{pi1(d) d}[g2]  (lane = g1, shuffles).
#pragma once
#include "p2_common.cuh"

namespace p2 {

// Per-lane copies of the table entries a lane needs with a lane-dependent index.
struct LaneTables {
  // nucleon table entry idx = lane: (nu, lam, lam', nu') and value
  int nu, lu, lup, nup, val;
  // exchange stage: lane = (iB = lane >> 2, mu' = lane & 3)
  int xlup, xnup;
  int xval[4];  // val(iA, iB) for iA = 0..3
  // meson stage: lane = g1, row d of G_g1: column pi1(d) and value
  int gsrc[4];  // source lane pi1(d)*4 + d
  int gre[4], gim[4];
};

__constant__ int c_nuc_idx[16][4] = P2_INIT_NucIdx;
__constant__ int c_nuc_val[16] = P2_INIT_NucVal;
__constant__ int c_gamma_perm[16][4] = P2_INIT_GammaPerm;
__constant__ int c_gamma_re[16][4] = P2_INIT_GammaRe;
__constant__ int c_gamma_im[16][4] = P2_INIT_GammaIm;

__device__ __forceinline__ LaneTables load_lane_tables(int l) {
  LaneTables t;
  t.nu = c_nuc_idx[l][0];
  t.lu = c_nuc_idx[l][1];
  t.lup = c_nuc_idx[l][2];
  t.nup = c_nuc_idx[l][3];
  t.val = c_nuc_val[l];
  const int iB = l >> 2;
  t.xlup = c_nuc_idx[iB][2];
  t.xnup = c_nuc_idx[iB][3];
#pragma unroll
  for (int iA = 0; iA < 4; iA++) t.xval[iA] = c_nuc_val[iA * 4 + iB];
#pragma unroll
  for (int d = 0; d < 4; d++) {
    t.gsrc[d] = c_gamma_perm[l][d] * 4 + d;
    t.gre[d] = c_gamma_re[l][d];
    t.gim[d] = c_gamma_im[l][d];
  }
  return t;
}

template <typename R>
__device__ __forceinline__ Cx<R> ld(const Cx<R>* p, int i) {
  return p[i];
}

// Nucleon C g5 for one dataset; returns tmp[lane >> 2][lane & 3].
template <typename R>
__device__ __forceinline__ Cx<R> nucleon_site(const Cx<R>* __restrict__ A, const Cx<R>* __restrict__ B,
                                              const LaneTables& lt, int l, unsigned mask) {
  // ---- direct term: Q[c][c'] ----
  Cx<R> Q[3][3];
  {
    const Cx<R>* An = A + sblk(lt.nu, lt.nup);
    const Cx<R>* Bl = B + sblk(lt.lu, lt.lup);
    Cx<R> a[9], b[9];
#pragma unroll
    for (int i = 0; i < 9; i++) {
      a[i] = An[i];
      b[i] = Bl[i];
    }
    const R v = R(lt.val);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const int c1 = (c + 1) % 3, c2 = (c + 2) % 3;
#pragma unroll
      for (int cp = 0; cp < 3; cp++) {
        const int d1 = (cp + 1) % 3, d2 = (cp + 2) % 3;
        Cx<R> q = czero<R>();
        cmac(q, a[c1 * 3 + d1], b[c2 * 3 + d2]);
        cmsub(q, a[c1 * 3 + d2], b[c2 * 3 + d1]);
        cmsub(q, a[c2 * 3 + d1], b[c1 * 3 + d2]);
        cmac(q, a[c2 * 3 + d2], b[c1 * 3 + d1]);
        Q[c][cp] = cscale(q, v);
      }
    }
  }
#pragma unroll
  for (int m = 1; m < 16; m <<= 1)
#pragma unroll
    for (int i = 0; i < 9; i++) Q[i / 3][i % 3] = Q[i / 3][i % 3] + shfl_xor16(Q[i / 3][i % 3], m, mask);

  const int mu = l >> 2, mup = l & 3;
  Cx<R> T1 = czero<R>();
  {
    const Cx<R>* Am = A + sblk(mu, mup);
#pragma unroll
    for (int i = 0; i < 9; i++) cmac(T1, Q[i / 3][i % 3], Am[i]);
  }

  // ---- exchange term: lane = (iB, mu'') with mu'' = l & 3 ----
  Cx<R> Z[9];
#pragma unroll
  for (int i = 0; i < 9; i++) Z[i] = czero<R>();
  {
    constexpr int NI[16][4] = P2_INIT_NucIdx;
    const int mpp = l & 3;
#pragma unroll
    for (int iA = 0; iA < 4; iA++) {
      const int nu = NI[iA * 4][0], lu = NI[iA * 4][1];
      const Cx<R>* Bq = B + sblk(lu, lt.xlup);
      const Cx<R>* Aq = A + sblk(nu, mpp);
      Cx<R> a[9], b[9];
#pragma unroll
      for (int i = 0; i < 9; i++) {
        a[i] = Aq[i];
        b[i] = cscale(Bq[i], R(lt.xval[iA]));
      }
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const int c1 = (c + 1) % 3, c2 = (c + 2) % 3;
#pragma unroll
        for (int ap = 0; ap < 3; ap++) {
          const int e1 = (ap + 1) % 3, e2 = (ap + 2) % 3;
          Cx<R>& z = Z[c * 3 + ap];
          cmac(z, a[c1 * 3 + e2], b[c2 * 3 + e1]);
          cmsub(z, a[c1 * 3 + e1], b[c2 * 3 + e2]);
          cmsub(z, a[c2 * 3 + e2], b[c1 * 3 + e1]);
          cmac(z, a[c2 * 3 + e1], b[c1 * 3 + e2]);
        }
      }
    }
  }
  Cx<R> P[4];
#pragma unroll
  for (int m = 0; m < 4; m++) {
    const Cx<R>* Am = A + sblk(m, lt.xnup);
    Cx<R> p = czero<R>();
#pragma unroll
    for (int i = 0; i < 9; i++) cmac(p, Z[i], Am[i]);
    P[m] = p;
  }
#pragma unroll
  for (int m = 0; m < 4; m++) {
    P[m] = P[m] + shfl_xor16(P[m], 4, mask);
    P[m] = P[m] + shfl_xor16(P[m], 8, mask);
  }
  // lane (mu = l >> 2, mu' = l & 3) holds T2[m][mu'] for all m; pick m = mu.
  Cx<R> T2 = P[0];
  T2 = (mu == 1) ? P[1] : T2;
  T2 = (mu == 2) ? P[2] : T2;
  T2 = (mu == 3) ? P[3] : T2;
  return T1 - T2;
}

// Generic meson block: lane g1 gets C[g1][g2] for g2 = 0..15 in out[].
template <typename R>
__device__ __forceinline__ void meson_site(const Cx<R>* __restrict__ A, const Cx<R>* __restrict__ B,
                                           const LaneTables& lt, int l, unsigned mask, Cx<R> out[16]) {
  const int al = l >> 2, de = l & 3;
  Cx<R> M[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) M[i][j] = czero<R>();
#pragma unroll
  for (int ab = 0; ab < 9; ab++) {
    Cx<R> u[4], d[4];
#pragma unroll
    for (int b = 0; b < 4; b++) u[b] = A[sblk(al, b) + ab];
#pragma unroll
    for (int z = 0; z < 4; z++) d[z] = B[sblk(de, z) + ab];
#pragma unroll
    for (int b = 0; b < 4; b++)
#pragma unroll
      for (int z = 0; z < 4; z++) cmac_conj(M[b][z], u[b], d[z]);
  }
  constexpr int GP[16][4] = P2_INIT_GammaPerm;
  constexpr int GR[16][4] = P2_INIT_GammaRe;
  constexpr int GI[16][4] = P2_INIT_GammaIm;
  Cx<R> N[16];
#pragma unroll
  for (int g2 = 0; g2 < 16; g2++) {
    Cx<R> n = czero<R>();
#pragma unroll
    for (int b = 0; b < 4; b++) n = n + cunit(M[b][GP[g2][b]], GR[g2][b], GI[g2][b]);
    N[g2] = n;
  }
#pragma unroll
  for (int g2 = 0; g2 < 16; g2++) {
    Cx<R> c = czero<R>();
#pragma unroll
    for (int d = 0; d < 4; d++) c = c + cunit(shfl_idx16(N[g2], lt.gsrc[d], mask), lt.gre[d], lt.gim[d]);
    out[g2] = c;
  }
}

// ---- Delta C g_k (PLEGMA_baryons_deltas.cu:7-110) ------------------------------
//
// All 14 Wick terms (8 of isospin 1/2, 6 of isospin 3/2) are products
//   X[nu][s1'] Y[lam][s2'] Z[mu][s3']  (colours a, b, c at the sink; the source
//   colour of a line follows its source spin slot),
// with Gamma = C g_k on (nu, lam) and Gamma-bar on (lam', nu').  Summing the
// sink diquark first gives, for the lane's source spins (x', y'),
//   G^{XY}[c][e] = sum_{(nu,lam)} sA sum eps_abc eps_{c1 c2 e} X[nu][x'][a][c1] Y[lam][y'][b][c2]
// (the same cofactor form as the nucleon's direct term), and every term is
// +-G contracted with the third line:
//   mu' on X's source slot (slot 1):  P[m] = f1 sum G[c][e] Z[m][z1][c][e], summed over y'
//   mu' on Y's source slot (slot 2):  P[m] = f2 sum G[c][e] Z[m][z2][c][e], summed over x'
//   mu' on Z (type a):                 D = sum over the 16 lanes of fa G, T = sum D Z[mu][mu']
// with f1 = -(c1A sA1 - c1B sB1), f2 = c2A sA2 - c2B sB2, fa = cN sN - cL sL from the
// per-lane descriptors (spin.diquark_lane_tables) and the Wick coefficients c.
struct DeltaLane {
  int z1, sA1, sB1, z2, sA2, sB2, sN, sL;
};

__constant__ int c_delta_lane[3][16][8] = P2_INIT_DeltaLane;

__device__ __forceinline__ DeltaLane load_delta_lane(int g, int l) {
  DeltaLane d;
  d.z1 = c_delta_lane[g][l][0];
  d.sA1 = c_delta_lane[g][l][1];
  d.sB1 = c_delta_lane[g][l][2];
  d.z2 = c_delta_lane[g][l][3];
  d.sA2 = c_delta_lane[g][l][4];
  d.sB2 = c_delta_lane[g][l][5];
  d.sN = c_delta_lane[g][l][6];
  d.sL = c_delta_lane[g][l][7];
  return d;
}

__constant__ int c_delta_sink[3][4][3] = P2_INIT_DeltaSink;

// G^{XY} for lane (x' = l >> 2, y' = l & 3) and table g (k = g + 1).
template <typename R>
__device__ __forceinline__ void delta_G(const Cx<R>* __restrict__ X, const Cx<R>* __restrict__ Y, int g, int xp,
                                        int yp, Cx<R> q[9]) {
#pragma unroll
  for (int i = 0; i < 9; i++) q[i] = czero<R>();
#pragma unroll 1
  for (int iA = 0; iA < 4; iA++) {
    const Cx<R>* Xb = X + sblk(c_delta_sink[g][iA][0], xp);
    const Cx<R>* Yb = Y + sblk(c_delta_sink[g][iA][1], yp);
    const R s = R(c_delta_sink[g][iA][2]);
    Cx<R> a[9], b[9];
#pragma unroll
    for (int i = 0; i < 9; i++) {
      a[i] = cscale(Xb[i], s);
      b[i] = Yb[i];
    }
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
}

// One group of Wick terms sharing G and the third line Z; returns the lane's
// share of T[mu = l >> 2][mu' = l & 3].
template <typename R>
__device__ __forceinline__ Cx<R> delta_eval(const Cx<R> g[9], const Cx<R>* __restrict__ Z, const DeltaLane& dl, int l,
                                            unsigned mask, int c1A, int c1B, int c2A, int c2B, int cN, int cL) {
  const R f1 = R(-(c1A * dl.sA1 - c1B * dl.sB1));
  const R f2 = R(c2A * dl.sA2 - c2B * dl.sB2);
  const R fa = R(cN * dl.sN - cL * dl.sL);
  const int mu = l >> 2, mup = l & 3;
  Cx<R> r = czero<R>();
  // slot 2 (reduce over x'): this lane's y' is mu'
#pragma unroll 1
  for (int m = 0; m < 4; m++) {
    const Cx<R>* Z2 = Z + sblk(m, dl.z2);
    Cx<R> p2 = czero<R>();
#pragma unroll
    for (int i = 0; i < 9; i++) cmac(p2, g[i], Z2[i]);
    p2 = cscale(p2, f2);
    p2 = p2 + shfl_xor16(p2, 4, mask);
    p2 = p2 + shfl_xor16(p2, 8, mask);
    if (m == mu) r = r + p2;
  }
  // slot 1 (reduce over y'): T[.][mu'] sits on lane (x' = mu', y' = 0)
  const int src = mup << 2;
#pragma unroll 1
  for (int m = 0; m < 4; m++) {
    const Cx<R>* Z1 = Z + sblk(m, dl.z1);
    Cx<R> p1 = czero<R>();
#pragma unroll
    for (int i = 0; i < 9; i++) cmac(p1, g[i], Z1[i]);
    p1 = cscale(p1, f1);
    p1 = p1 + shfl_xor16(p1, 1, mask);
    p1 = p1 + shfl_xor16(p1, 2, mask);
    const Cx<R> v = shfl_idx16(p1, src, mask);
    if (m == mu) r = r + v;
  }
  // type a
  const Cx<R>* Zm = Z + sblk(mu, mup);
#pragma unroll
  for (int i = 0; i < 9; i++) {
    Cx<R> d = cscale(g[i], fa);
    d = d + shfl_xor16(d, 1, mask);
    d = d + shfl_xor16(d, 2, mask);
    d = d + shfl_xor16(d, 4, mask);
    d = d + shfl_xor16(d, 8, mask);
    cmac(r, d, Zm[i]);
  }
  return r;
}

// Delta C g_k, k = g + 1: out = {iso-1/2 Delta+ (u,u,d), iso-1/2 Delta0 (d,d,u),
// iso-3/2 Delta++ (u,u,u), iso-3/2 Delta- (d,d,d)} for lane (mu, mu').
template <typename R>
__device__ __forceinline__ void delta_site(const Cx<R>* __restrict__ U, const Cx<R>* __restrict__ D, int g, int l,
                                           unsigned mask, Cx<R> out[4]) {
  const DeltaLane dl = load_delta_lane(g, l);
  const int xp = l >> 2, yp = l & 3;
  const R third = R(1) / R(3);
#pragma unroll
  for (int i = 0; i < 4; i++) out[i] = czero<R>();
  // flavour pairs (X, Y) of the two diquark lines: uu, dd, ud, du
#pragma unroll 1
  for (int pair = 0; pair < 4; pair++) {
    const Cx<R>* X = (pair == 0 || pair == 2) ? U : D;
    const Cx<R>* Y = (pair == 0 || pair == 3) ? U : D;
    Cx<R> q[9];
    delta_G<R>(X, Y, g, xp, yp, q);
    if (pair < 2) {
      // G^{AA}: isospin 1/2 with the other flavour on the third line, isospin 3/2 with the same
      const Cx<R> a = delta_eval<R>(q, pair == 0 ? D : U, dl, l, mask, 0, 2, 0, -2, 1, -1);
      const Cx<R> b = delta_eval<R>(q, pair == 0 ? U : D, dl, l, mask, -1, 1, 1, -1, 1, -1);
      out[pair] = out[pair] + cscale(a, third);
      out[2 + pair] = out[2 + pair] + b;
    } else {
      // G^{AB}: isospin 1/2 with A on the third line
      const Cx<R> a = delta_eval<R>(q, pair == 2 ? U : D, dl, l, mask, -4, 0, 2, -2, 4, 0);
      out[pair - 2] = out[pair - 2] + cscale(a, third);
    }
  }
}

}  // namespace p2
