// FP64 CPU oracle for the hadron two-point contraction + momentum projection.
//
// TEST INFRASTRUCTURE ONLY.  This file restates the reference algorithm on the
// CPU so that the CUDA kernels can be checked against it.  Only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg load it; the
// product library never links or calls it.
//
// Every loop follows the reference literally (same index order, same
// unfactorised sums), so this is a slow but faithful transcription:
//   nucleon      lib/kernels/PLEGMA_baryons_NtoN.cu:6-46, second interpolator
//                PLEGMA_baryons_NtoR.cu, _RtoN.cu, _RtoR.cu
//   Delta        lib/kernels/PLEGMA_baryons_deltas.cu:7-110
//   mesons       lib/kernels/PLEGMA_mesonsAll.cuh:34-82 (generic G1 S1 G2 S2^dag),
//                PLEGMA_mesons.cuh:29-53, PLEGMA_mesonsNew.cuh:27-45
//   projection   lib/kernels/PLEGMA_kernel_utils.cuh:820-860 (source-relative
//                phase, sign -1), evaluated in double precision
//   time window  include/PLEGMA_Correlator.h:53-79, PLEGMA_baryons.cuh:35-41
//   table-driven lib/kernels/PLEGMA_baryons_udsc.cu:85-134
// Spin tables come from plegma_b200/csrc/spin_tables.h, which is generated
// from the gamma matrices and pinned to the reference tables by digest.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../plegma_b200/csrc/spin_tables.h"

namespace {

struct cplx {
  double x, y;
};
inline cplx operator+(cplx a, cplx b) { return {a.x + b.x, a.y + b.y}; }
inline cplx operator-(cplx a, cplx b) { return {a.x - b.x, a.y - b.y}; }
inline cplx operator*(cplx a, cplx b) { return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
inline cplx operator*(double s, cplx a) { return {s * a.x, s * a.y}; }
inline cplx conj(cplx a) { return {a.x, -a.y}; }

typedef cplx Prop[4][4][3][3];

// Contraction-set bits; identical to include/plegma2pt.h.
enum : unsigned {
  NUCLEON_CG5 = 1u << 0,
  DELTA_ISO12 = 1u << 1,
  DELTA_ISO32 = 1u << 2,
  MESON_G16 = 1u << 3,
  MESON_ALL34 = 1u << 4,
  MESON_NEW10 = 1u << 5,
  MESON_DIAG10 = 1u << 6,
  NUCLEON_NTOR = 1u << 7,
  NUCLEON_RTON = 1u << 8,
  NUCLEON_RTOR = 1u << 9,
};

// Diagonal structures of contractMesons / contractMesonsNew, in output order.
constexpr int kMeson10[10] = {0, 5, 1, 2, 3, 4, 6, 7, 8, 9};

int components(unsigned what) {
  int k = 0;
  if (what & NUCLEON_CG5) k += 32;
  if (what & NUCLEON_NTOR) k += 32;
  if (what & NUCLEON_RTON) k += 32;
  if (what & NUCLEON_RTOR) k += 32;
  if (what & DELTA_ISO12) k += 96;
  if (what & DELTA_ISO32) k += 96;
  if (what & MESON_G16) k += 256;
  if (what & MESON_ALL34) k += 34;
  if (what & MESON_NEW10) k += 10;
  if (what & MESON_DIAG10) k += 20;
  return k;
}

inline cplx gam(int g, int row) { return {(double)p2::kGammaRe[g][row], (double)p2::kGammaIm[g][row]}; }

// Generic meson: sum G1[delta][alpha] S1[alpha][beta] G2[beta][zeta] conj(S2[delta][zeta]),
// PLEGMA_mesonsAll.cuh:58-76.
cplx meson_pair(const Prop& s1, const Prop& s2, int g1, int g2) {
  cplx acc = {0, 0};
  for (int is1 = 0; is1 < 4; is1++)
    for (int is2 = 0; is2 < 4; is2++) {
      int beta = is2, zeta = p2::kGammaPerm[g2][is2];
      int delta = is1, alpha = p2::kGammaPerm[g1][is1];
      cplx v1 = gam(g1, is1), v2 = gam(g2, is2);
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
          acc = acc + v1 * s1[alpha][beta][a][b] * v2 * conj(s2[delta][zeta][a][b]);
    }
  return acc;
}

// Nucleon C g5, both Wick terms; out[(ds*4+mu)*4+mup], ds 0 = proton, 1 = neutron.
void nucleon(const Prop& p1, const Prop& p2, cplx* out) {
  for (int mu = 0; mu < 4; mu++)
    for (int mup = 0; mup < 4; mup++) {
      cplx tmp[2] = {{0, 0}, {0, 0}};
      for (int idx = 0; idx < 16; idx++) {
        int nu = p2::kNucIdx[idx][0], lu = p2::kNucIdx[idx][1];
        int lup = p2::kNucIdx[idx][2], nup = p2::kNucIdx[idx][3];
        for (int cc1 = 0; cc1 < 6; cc1++) {
          int a = p2::kEps[cc1][0], b = p2::kEps[cc1][1], c = p2::kEps[cc1][2];
          for (int cc2 = 0; cc2 < 6; cc2++) {
            int a1 = p2::kEps[cc2][0], b1 = p2::kEps[cc2][1], c1 = p2::kEps[cc2][2];
            double f = (double)(p2::kEpsSign[cc1] * p2::kEpsSign[cc2] * p2::kNucVal[idx]);
            tmp[0] = tmp[0] + f * p2[lu][lup][b][b1] *
                                  (p1[nu][nup][a][a1] * p1[mu][mup][c][c1] - p1[nu][mup][a][c1] * p1[mu][nup][c][a1]);
            tmp[1] = tmp[1] + f * p1[lu][lup][b][b1] *
                                  (p2[nu][nup][a][a1] * p2[mu][mup][c][c1] - p2[nu][mup][a][c1] * p2[mu][nup][c][a1]);
          }
        }
      }
      out[(0 * 4 + mu) * 4 + mup] = tmp[0];
      out[(1 * 4 + mu) * 4 + mup] = tmp[1];
    }
}

// Delta isospin 1/2 (Delta+, Delta0) with C g_k, k = g+1.
void delta_iso12(const Prop& P1, const Prop& P2, int g, cplx* out) {
  for (int mu = 0; mu < 4; mu++)
    for (int mup = 0; mup < 4; mup++) {
      cplx tmp[2] = {{0, 0}, {0, 0}};
      for (int idx = 0; idx < 16; idx++) {
        int nu = p2::kDeltaIdx[g][idx][0], lu = p2::kDeltaIdx[g][idx][1];
        int lup = p2::kDeltaIdx[g][idx][2], nup = p2::kDeltaIdx[g][idx][3];
        for (int cc1 = 0; cc1 < 6; cc1++) {
          int a = p2::kEps[cc1][0], b = p2::kEps[cc1][1], c = p2::kEps[cc1][2];
          for (int cc2 = 0; cc2 < 6; cc2++) {
            int a1 = p2::kEps[cc2][0], b1 = p2::kEps[cc2][1], c1 = p2::kEps[cc2][2];
            double f = (1. / 3.) * (double)(p2::kEpsSign[cc1] * p2::kEpsSign[cc2] * p2::kDeltaVal[g][idx]);
            for (int s = 0; s < 2; s++) {
              const Prop& A = s ? P2 : P1;
              const Prop& B = s ? P1 : P2;
              cplx t = -4. * A[nu][mup][a][c1] * B[lu][lup][b][b1] * A[mu][nup][c][a1] +
                       2. * A[nu][lup][a][b1] * B[lu][mup][b][c1] * A[mu][nup][c][a1] +
                       2. * A[nu][mup][a][c1] * A[lu][nup][b][a1] * B[mu][lup][c][b1] -
                       2. * A[nu][nup][a][a1] * A[lu][mup][b][c1] * B[mu][lup][c][b1] -
                       2. * A[nu][nup][a][a1] * B[lu][mup][b][c1] * A[mu][lup][c][b1] -
                       1. * A[nu][lup][a][b1] * A[lu][nup][b][a1] * B[mu][mup][c][c1] +
                       1. * A[nu][nup][a][a1] * A[lu][lup][b][b1] * B[mu][mup][c][c1] +
                       4. * A[nu][nup][a][a1] * B[lu][lup][b][b1] * A[mu][mup][c][c1];
              tmp[s] = tmp[s] + f * t;
            }
          }
        }
      }
      out[(0 * 4 + mu) * 4 + mup] = tmp[0];
      out[(1 * 4 + mu) * 4 + mup] = tmp[1];
    }
}

// Delta isospin 3/2 (Delta++ from P1 only, Delta- from P2 only).
void delta_iso32(const Prop& P1, const Prop& P2, int g, cplx* out) {
  for (int mu = 0; mu < 4; mu++)
    for (int mup = 0; mup < 4; mup++) {
      cplx tmp[2] = {{0, 0}, {0, 0}};
      for (int idx = 0; idx < 16; idx++) {
        int nu = p2::kDeltaIdx[g][idx][0], lu = p2::kDeltaIdx[g][idx][1];
        int lup = p2::kDeltaIdx[g][idx][2], nup = p2::kDeltaIdx[g][idx][3];
        for (int cc1 = 0; cc1 < 6; cc1++) {
          int a = p2::kEps[cc1][0], b = p2::kEps[cc1][1], c = p2::kEps[cc1][2];
          for (int cc2 = 0; cc2 < 6; cc2++) {
            int a1 = p2::kEps[cc2][0], b1 = p2::kEps[cc2][1], c1 = p2::kEps[cc2][2];
            double f = (double)(p2::kEpsSign[cc1] * p2::kEpsSign[cc2] * p2::kDeltaVal[g][idx]);
            for (int s = 0; s < 2; s++) {
              const Prop& A = s ? P2 : P1;
              cplx t = A[nu][lup][a][b1] * A[lu][mup][b][c1] * A[mu][nup][c][a1] -
                       A[nu][mup][a][c1] * A[lu][lup][b][b1] * A[mu][nup][c][a1] +
                       A[nu][mup][a][c1] * A[lu][nup][b][a1] * A[mu][lup][c][b1] -
                       A[nu][nup][a][a1] * A[lu][mup][b][c1] * A[mu][lup][c][b1] -
                       A[nu][lup][a][b1] * A[lu][nup][b][a1] * A[mu][mup][c][c1] +
                       A[nu][nup][a][a1] * A[lu][lup][b][b1] * A[mu][mup][c][c1];
              tmp[s] = tmp[s] + f * t;
            }
          }
        }
      }
      out[(0 * 4 + mu) * 4 + mup] = tmp[0];
      out[(1 * 4 + mu) * 4 + mup] = tmp[1];
    }
}

// Second nucleon interpolator R = eps (u C d) g5 u against N and itself,
// out[(ds*4+mu)*4+mup]:
//   NtoR  lib/kernels/PLEGMA_baryons_NtoR.cu:6-52
//   RtoN  lib/kernels/PLEGMA_baryons_RtoN.cu:6-52
//   RtoR  lib/kernels/PLEGMA_baryons_RtoR.cu:6-46
// The index tables are the reference's (generated by plegma_b200/spin.py).
void nucleon_ntor(const Prop& p1, const Prop& p2, cplx* out) {
  for (int mu = 0; mu < 4; mu++) {
    cplx tmp[8] = {};
    for (int idx = 0; idx < 64; idx++) {
      const int* m = p2::kNtrIdx[idx];
      const int nu = m[0], lu = m[1], lup = m[2], nup = m[3], mup = m[4], rho = m[5];
      for (int cc1 = 0; cc1 < 6; cc1++) {
        int a = p2::kEps[cc1][0], b = p2::kEps[cc1][1], c = p2::kEps[cc1][2];
        for (int cc2 = 0; cc2 < 6; cc2++) {
          int a1 = p2::kEps[cc2][0], b1 = p2::kEps[cc2][1], c1 = p2::kEps[cc2][2];
          double f = (double)(p2::kEpsSign[cc1] * p2::kEpsSign[cc2] * p2::kNtrVal[idx]);
          tmp[mup] = tmp[mup] - f * p2[lu][lup][b][b1] *
                                    (p1[nu][nup][a][a1] * p1[mu][rho][c][c1] - p1[nu][rho][a][c1] * p1[mu][nup][c][a1]);
          tmp[4 + mup] = tmp[4 + mup] - f * p1[lu][lup][b][b1] *
                                            (p2[nu][nup][a][a1] * p2[mu][rho][c][c1] - p2[nu][rho][a][c1] * p2[mu][nup][c][a1]);
        }
      }
    }
    for (int i = 0; i < 2; i++)
      for (int mup = 0; mup < 4; mup++) out[(i * 4 + mu) * 4 + mup] = tmp[i * 4 + mup];
  }
}

void nucleon_rton(const Prop& p1, const Prop& p2, cplx* out) {
  for (int mup = 0; mup < 4; mup++) {
    cplx tmp[8] = {};
    for (int idx = 0; idx < 64; idx++) {
      const int* m = p2::kRtnIdx[idx];
      const int nu = m[0], lu = m[1], lup = m[2], nup = m[3], mu = m[4], rho = m[5];
      for (int cc1 = 0; cc1 < 6; cc1++) {
        int a = p2::kEps[cc1][0], b = p2::kEps[cc1][1], c = p2::kEps[cc1][2];
        for (int cc2 = 0; cc2 < 6; cc2++) {
          int a1 = p2::kEps[cc2][0], b1 = p2::kEps[cc2][1], c1 = p2::kEps[cc2][2];
          double f = (double)(p2::kEpsSign[cc1] * p2::kEpsSign[cc2] * p2::kRtnVal[idx]);
          tmp[mu] = tmp[mu] + f * p2[lu][lup][b][b1] *
                                  (p1[nu][nup][a][a1] * p1[rho][mup][c][c1] - p1[nu][mup][a][c1] * p1[rho][nup][c][a1]);
          tmp[4 + mu] = tmp[4 + mu] + f * p1[lu][lup][b][b1] *
                                          (p2[nu][nup][a][a1] * p2[rho][mup][c][c1] - p2[nu][mup][a][c1] * p2[rho][nup][c][a1]);
        }
      }
    }
    for (int i = 0; i < 2; i++)
      for (int mu = 0; mu < 4; mu++) out[(i * 4 + mu) * 4 + mup] = tmp[i * 4 + mu];
  }
}

void nucleon_rtor(const Prop& p1, const Prop& p2, cplx* out) {
  for (int i = 0; i < 32; i++) out[i] = {0, 0};
  for (int idx = 0; idx < 256; idx++) {
    const int* m = p2::kRtrIdx[idx];
    const int nu = m[0], lu = m[1], lup = m[2], nup = m[3], mu = m[4], rho = m[5], mup = m[6], rhop = m[7];
    for (int cc1 = 0; cc1 < 6; cc1++) {
      int a = p2::kEps[cc1][0], b = p2::kEps[cc1][1], c = p2::kEps[cc1][2];
      for (int cc2 = 0; cc2 < 6; cc2++) {
        int a1 = p2::kEps[cc2][0], b1 = p2::kEps[cc2][1], c1 = p2::kEps[cc2][2];
        double f = (double)(p2::kEpsSign[cc1] * p2::kEpsSign[cc2] * p2::kRtrVal[idx]);
        out[mu * 4 + mup] = out[mu * 4 + mup] - f * p2[lu][lup][b][b1] *
                                                    (p1[nu][nup][a][a1] * p1[rho][rhop][c][c1] -
                                                     p1[nu][rhop][a][c1] * p1[rho][nup][c][a1]);
        out[(4 + mu) * 4 + mup] = out[(4 + mu) * 4 + mup] - f * p1[lu][lup][b][b1] *
                                                                (p2[nu][nup][a][a1] * p2[rho][rhop][c][c1] -
                                                                 p2[nu][rhop][a][c1] * p2[rho][nup][c][a1]);
      }
    }
  }
}

// All requested components of one site, in block order.
void site_components(const Prop& u, const Prop& d, unsigned what, cplx* c) {
  int k = 0;
  if (what & NUCLEON_CG5) {
    nucleon(u, d, c + k);
    k += 32;
  }
  if (what & NUCLEON_NTOR) {
    nucleon_ntor(u, d, c + k);
    k += 32;
  }
  if (what & NUCLEON_RTON) {
    nucleon_rton(u, d, c + k);
    k += 32;
  }
  if (what & NUCLEON_RTOR) {
    nucleon_rtor(u, d, c + k);
    k += 32;
  }
  if (what & DELTA_ISO12) {
    for (int g = 0; g < 3; g++) delta_iso12(u, d, g, c + k + 32 * g);
    k += 96;
  }
  if (what & DELTA_ISO32) {
    for (int g = 0; g < 3; g++) delta_iso32(u, d, g, c + k + 32 * g);
    k += 96;
  }
  if (what & MESON_G16) {
    for (int g1 = 0; g1 < 16; g1++)
      for (int g2 = 0; g2 < 16; g2++) c[k + g1 * 16 + g2] = meson_pair(u, d, g1, g2);
    k += 256;
  }
  if (what & MESON_ALL34) {
    c[k + 0] = meson_pair(u, d, 0, 0);
    c[k + 1] = meson_pair(u, d, 5, 5);
    for (int ip = 0; ip < 2; ip++)
      for (int i1 = 0; i1 < 4; i1++)
        for (int i2 = 0; i2 < 4; i2++)
          c[k + 2 + i1 * 4 + i2 + 16 * ip] = meson_pair(u, d, 1 + i1 + 5 * ip, 1 + i2 + 5 * ip);
    k += 34;
  }
  if (what & MESON_NEW10) {
    for (int j = 0; j < 10; j++) c[k + j] = meson_pair(u, d, kMeson10[j], kMeson10[j]);
    k += 10;
  }
  if (what & MESON_DIAG10) {
    for (int j = 0; j < 10; j++) c[k + j] = meson_pair(u, u, kMeson10[j], kMeson10[j]);
    for (int j = 0; j < 10; j++) c[k + 10 + j] = meson_pair(d, d, kMeson10[j], kMeson10[j]);
    k += 20;
  }
}

struct View {
  const void* p;
  int fp32;       // 0: complex double, 1: complex float
  long vol;       // V3 * nt (component stride in complex elements)
};

inline cplx fetch(const View& v, int comp, long sid) {
  long i = (long)comp * v.vol + sid;
  if (v.fp32) {
    const float* f = (const float*)v.p;
    return {(double)f[2 * i], (double)f[2 * i + 1]};
  }
  const double* f = (const double*)v.p;
  return {f[2 * i], f[2 * i + 1]};
}

void gather(const View& v, long sid, Prop& P) {
  for (int mu = 0; mu < 4; mu++)
    for (int nu = 0; nu < 4; nu++)
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) P[mu][nu][a][b] = fetch(v, ((mu * 4 + nu) * 3 + a) * 3 + b, sid);
}

}  // namespace

extern "C" {

int orc_components(unsigned what) { return components(what); }

// Two-point functions for a list of source-relative times.
//   L[4]          lattice extents (x, y, z, t)
//   u, d          propagators, SoA [144][V3*nt] complex (re, im interleaved),
//                 covering global slices t_first .. t_first+nt-1 (mod T)
//   fp32          1 when the propagators are complex float
//   src[4]        source position; totalT the window
//   moms[nmom*3]  momenta (integers n, p = 2 pi n / L)
//   taus[ntau]    source-relative times to compute
//   out           [ntau][nmom][K] complex, K = orc_components(what)
//   abs_sum       [ntau][K] = sum_x |c_k(x,t)| (may be NULL)
//   pos           [ntau][K][V3] complex position-space values (may be NULL)
int orc_twopt(const int* L, int nt, int t_first, const void* u, const void* d, int fp32, const int* src,
              const int* moms, int nmom, unsigned what, const int* taus, int ntau, double* out, double* abs_sum,
              double* pos) {
  const int K = components(what);
  if (K == 0) return 1;
  const long V3 = (long)L[0] * L[1] * L[2];
  const int T = L[3];
  View vu{u, fp32, V3 * nt}, vd{d, fp32, V3 * nt};
  for (int it = 0; it < ntau; it++) {
    const int t = (src[3] + taus[it]) % T;
    const int j = ((t - t_first) % T + T) % T;
    if (j >= nt) return 2;
    cplx* o = (cplx*)out + (long)it * nmom * K;
    for (long i = 0; i < (long)nmom * K; i++) o[i] = {0, 0};
    std::vector<double> asum(K, 0.0);
#pragma omp parallel
    {
      std::vector<cplx> loc((size_t)nmom * K, cplx{0, 0});
      std::vector<double> locabs(K, 0.0);
      std::vector<cplx> c(K);
      Prop Pu, Pd;
#pragma omp for schedule(static)
      for (long x3 = 0; x3 < V3; x3++) {
        const long sid = x3 + V3 * j;
        gather(vu, sid, Pu);
        gather(vd, sid, Pd);
        site_components(Pu, Pd, what, c.data());
        const int id[3] = {(int)(x3 % L[0]), (int)((x3 / L[0]) % L[1]), (int)(x3 / ((long)L[0] * L[1]))};
        for (int k = 0; k < K; k++) locabs[k] += std::sqrt(c[k].x * c[k].x + c[k].y * c[k].y);
        if (pos) {
          cplx* pp = (cplx*)pos + (long)it * K * V3;
          for (int k = 0; k < K; k++) pp[(long)k * V3 + x3] = c[k];
        }
        for (int p = 0; p < nmom; p++) {
          double ph = 0;
          for (int i = 0; i < 3; i++) ph += (double)moms[3 * p + i] * (double)(id[i] - src[i]) / (double)L[i];
          ph *= 2.0 * M_PI;
          const cplx e = {std::cos(ph), -std::sin(ph)};
          for (int k = 0; k < K; k++) loc[(size_t)p * K + k] = loc[(size_t)p * K + k] + c[k] * e;
        }
      }
#pragma omp critical
      {
        for (long i = 0; i < (long)nmom * K; i++) o[i] = o[i] + loc[i];
        for (int k = 0; k < K; k++) asum[k] += locabs[k];
      }
    }
    if (abs_sum)
      for (int k = 0; k < K; k++) abs_sum[(long)it * K + k] = asum[k];
  }
  return 0;
}

// Site-local components only (no projection) for explicit per-site checks:
// u, d point at one site's 144 complex values each (component-major).
void orc_site(const double* u, const double* d, unsigned what, double* out) {
  Prop Pu, Pd;
  View vu{u, 0, 1}, vd{d, 0, 1};
  gather(vu, 0, Pu);
  gather(vd, 0, Pd);
  site_components(Pu, Pd, what, (cplx*)out);
}

// Generic field projection as PLEGMA_FT::apply(FT_NAIVE) with the source at
// the origin: field SoA [dof][V3*nt] complex; out [nt][dof][nmom] complex,
// lib/PLEGMA_FT.cu:122-134, lib/kernels/PLEGMA_FT.cuh:104-159.
int orc_ft(const int* L, int nt, const double* field, int dof, const int* moms, int nmom, int sign, double* out) {
  const long V3 = (long)L[0] * L[1] * L[2];
  const cplx* f = (const cplx*)field;
  cplx* o = (cplx*)out;
#pragma omp parallel for collapse(2) schedule(static)
  for (int t = 0; t < nt; t++)
    for (int df = 0; df < dof; df++) {
      for (int p = 0; p < nmom; p++) {
        cplx acc = {0, 0};
        for (long x3 = 0; x3 < V3; x3++) {
          const int id[3] = {(int)(x3 % L[0]), (int)((x3 / L[0]) % L[1]), (int)(x3 / ((long)L[0] * L[1]))};
          double ph = 0;
          for (int i = 0; i < 3; i++) ph += (double)moms[3 * p + i] * (double)id[i] / (double)L[i];
          ph *= 2.0 * M_PI;
          const cplx e = {std::cos(ph), sign * std::sin(ph)};
          acc = acc + f[(long)df * V3 * nt + (long)t * V3 + x3] * e;
        }
        o[((long)t * dof + df) * nmom + p] = acc;
      }
    }
  return 0;
}

// Table-driven three-propagator contraction (PLEGMA_baryons_udsc.cu:85-134):
// sum_i w_i sum_{eps eps'} P1[m0][m1][a][a'] P2[m2][m3][b][b'] P3[m4][m5][c][c']
// for one site; idx[n][6], w[n] complex.
void orc_udsc_site(const double* p1, const double* p2, const double* p3, int n, const short* idx, const double* w,
                   double* out) {
  Prop A, B, C;
  View va{p1, 0, 1}, vb{p2, 0, 1}, vc{p3, 0, 1};
  gather(va, 0, A);
  gather(vb, 0, B);
  gather(vc, 0, C);
  cplx acc = {0, 0};
  for (int i = 0; i < n; i++) {
    const short* m = idx + 6 * i;
    cplx wi = {w[2 * i], w[2 * i + 1]};
    for (int cc1 = 0; cc1 < 6; cc1++) {
      int a = p2::kEps[cc1][0], b = p2::kEps[cc1][1], c = p2::kEps[cc1][2];
      for (int cc2 = 0; cc2 < 6; cc2++) {
        int a1 = p2::kEps[cc2][0], b1 = p2::kEps[cc2][1], c1 = p2::kEps[cc2][2];
        cplx f = (double)(p2::kEpsSign[cc1] * p2::kEpsSign[cc2]) * wi;
        acc = acc + f * A[m[0]][m[1]][a][a1] * B[m[2]][m[3]][b][b1] * C[m[4]][m[5]][c][c1];
      }
    }
  }
  out[0] = acc.x;
  out[1] = acc.y;
}

}  // extern "C"

extern "C" {

// Table-driven baryon two-point functions of one flavour product
// (lib/kernels/PLEGMA_baryons_udsc.cu:85-134 per site, projected as
// lib/kernels/PLEGMA_kernel_utils.cuh:820-860):
//   p1, p2, p3   the product's three propagators (flavour-sorted roles)
//   ndata        datasets; dataset d has entries ent_begin[d] .. ent_begin[d+1]-1
//                of idx[][6] (spin indices) and w[][2] (single-precision weights)
//   out          [ntau][ndata][nmom] complex; abs_sum [ntau][ndata] (may be NULL)
int orc_udsc_twopt(const int* L, int nt, int t_first, const void* p1, const void* p2, const void* p3, int fp32,
                   const int* src, const int* moms, int nmom, int ndata, const int* ent_begin,
                   const signed char* idx, const float* w, const int* taus, int ntau, double* out,
                   double* abs_sum) {
  const long V3 = (long)L[0] * L[1] * L[2];
  const int T = L[3];
  View v1{p1, fp32, V3 * nt}, v2{p2, fp32, V3 * nt}, v3{p3, fp32, V3 * nt};
  for (int it = 0; it < ntau; it++) {
    const int t = (src[3] + taus[it]) % T;
    const int j = ((t - t_first) % T + T) % T;
    if (j >= nt) return 2;
    cplx* o = (cplx*)out + (long)it * ndata * nmom;
    for (long i = 0; i < (long)ndata * nmom; i++) o[i] = {0, 0};
    std::vector<double> asum(ndata, 0.0);
#pragma omp parallel
    {
      std::vector<cplx> loc((size_t)ndata * nmom, cplx{0, 0});
      std::vector<double> locabs(ndata, 0.0);
      Prop A, B, Cp;
#pragma omp for schedule(static)
      for (long x3 = 0; x3 < V3; x3++) {
        const long sid = x3 + V3 * j;
        gather(v1, sid, A);
        gather(v2, sid, B);
        gather(v3, sid, Cp);
        const int id[3] = {(int)(x3 % L[0]), (int)((x3 / L[0]) % L[1]), (int)(x3 / ((long)L[0] * L[1]))};
        for (int d = 0; d < ndata; d++) {
          cplx acc = {0, 0};
          for (int e = ent_begin[d]; e < ent_begin[d + 1]; e++) {
            const signed char* m = idx + 6 * e;
            const cplx we = {(double)w[2 * e], (double)w[2 * e + 1]};
            for (int cc1 = 0; cc1 < 6; cc1++) {
              const int a = p2::kEps[cc1][0], b = p2::kEps[cc1][1], c = p2::kEps[cc1][2];
              for (int cc2 = 0; cc2 < 6; cc2++) {
                const int a1 = p2::kEps[cc2][0], b1 = p2::kEps[cc2][1], c1 = p2::kEps[cc2][2];
                const cplx f = (double)(p2::kEpsSign[cc1] * p2::kEpsSign[cc2]) * we;
                acc = acc + f * A[m[0]][m[1]][a][a1] * B[m[2]][m[3]][b][b1] * Cp[m[4]][m[5]][c][c1];
              }
            }
          }
          locabs[d] += std::sqrt(acc.x * acc.x + acc.y * acc.y);
          for (int p = 0; p < nmom; p++) {
            double ph = 0;
            for (int i = 0; i < 3; i++) ph += (double)moms[3 * p + i] * (double)(id[i] - src[i]) / (double)L[i];
            ph *= 2.0 * M_PI;
            const cplx e = {std::cos(ph), -std::sin(ph)};
            loc[(size_t)d * nmom + p] = loc[(size_t)d * nmom + p] + acc * e;
          }
        }
      }
#pragma omp critical
      {
        for (long i = 0; i < (long)ndata * nmom; i++) o[i] = o[i] + loc[i];
        for (int d = 0; d < ndata; d++) asum[d] += locabs[d];
      }
    }
    if (abs_sum)
      for (int d = 0; d < ndata; d++) abs_sum[(long)it * ndata + d] = asum[d];
  }
  return 0;
}

}  // extern "C"
