// Stand-in for the reference's kernel utility header, used only to compile the
// reference's own contraction sources as host C++ (oracle/_ref).  It supplies
// the handful of types and globals those sources use: a complex pair, a
// propagator accessor over the SoA field, the Levi-Civita list, the CUDA
// launch coordinates (one thread per block: blockDim.x = 1) and the lattice
// geometry globals.  The Levi-Civita list comes from this project's generated
// tables (pinned to the reference's by digest), so nothing of the reference
// is copied here.
#pragma once
#include <cmath>
#include <cstddef>

#include "../../plegma_b200/csrc/spin_tables.h"

#define N_SPINS 4
#define N_COLS 3
#define DIM_T 3
#define PI 3.141592653589793

template <typename F>
struct Float2 {
  F x, y;
  Float2() = default;
  template <typename S>
  Float2(const S& r) : x((F)r), y((F)0) {}
  Float2(F a, F b) : x(a), y(b) {}
  template <typename G>
  Float2(const Float2<G>& o) : x((F)o.x), y((F)o.y) {}
  Float2 operator+(const Float2& b) const { return Float2(x + b.x, y + b.y); }
  Float2 operator-(const Float2& b) const { return Float2(x - b.x, y - b.y); }
  Float2 operator*(const Float2& b) const { return Float2(x * b.x - y * b.y, x * b.y + y * b.x); }
};
template <typename S, typename F>
inline Float2<F> operator*(const S& s, const Float2<F>& a) {
  return Float2<F>((F)(s * a.x), (F)(s * a.y));
}
template <typename F>
inline Float2<F> conj(const Float2<F>& a) {
  return Float2<F>(a.x, -a.y);
}

// Accessor over a propagator in the SoA layout [144][vol] (component
// ((mu*4 + nu)*3 + c1)*3 + c2, complex interleaved); get(P, vid) reads site vid.
// With vol = 1 and vid = 0 it reads one site's 144 consecutive values.
template <typename F>
struct propTex {
  const F* p;
  long vol;
  explicit propTex(const F* q, long v = 1) : p(q), vol(v) {}
  void get(Float2<F> P[4][4][3][3], long vid) const {
    for (int mu = 0; mu < 4; mu++)
      for (int nu = 0; nu < 4; nu++)
        for (int a = 0; a < 3; a++)
          for (int b = 0; b < 3; b++) {
            const long i = ((mu * 4 + nu) * 3 + a) * 3 + b;
            P[mu][nu][a][b] = Float2<F>(p[2 * (i * vol + vid)], p[2 * (i * vol + vid) + 1]);
          }
  }
};

static const int (&eps)[6][3] = p2::kEps;
static const int (&sgn_eps)[6] = p2::kEpsSign;

// CUDA launch coordinates and the lattice geometry of the emulated launch
// (defined in ref_mesons.cpp).
struct ShimDim3 {
  unsigned x, y, z;
};
struct int4 {
  int x, y, z, w;
};
extern ShimDim3 gridDim, blockIdx, blockDim, threadIdx;
extern int DGC_localL[4], DGC_totalL[4], DGC_procPosition[4];
extern int DGC_localVolume3D;
inline void __syncthreads() {}

// Momentum list as the kernels read it: get(i) returns (nx, ny, nz, 0).
struct tex_mom_list {
  size_t Nmoms;
  const int* m;
  int4 get(const size_t& i) const { return int4{m[3 * i], m[3 * i + 1], m[3 * i + 2], 0}; }
};
