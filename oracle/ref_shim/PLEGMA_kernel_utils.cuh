// Stand-in for the reference's kernel utility header, used only to compile the
// reference's own baryon contraction sources as host C++ (oracle/_ref).  It
// supplies the handful of types those sources use: a complex pair, a
// per-site propagator accessor and the Levi-Civita list.  The Levi-Civita list
// comes from this project's generated tables (pinned to the reference's by
// digest), so nothing of the reference is copied here.
#pragma once
#include "../../plegma_b200/csrc/spin_tables.h"

#define N_SPINS 4
#define N_COLS 3

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

// Accessor over one site's 144 complex values, component-major
// ((mu*4 + nu)*3 + c1)*3 + c2, the propagator's per-site order.
template <typename F>
struct propTex {
  const F* p;
  explicit propTex(const F* q) : p(q) {}
  void get(Float2<F> P[4][4][3][3], int) const {
    for (int mu = 0; mu < 4; mu++)
      for (int nu = 0; nu < 4; nu++)
        for (int a = 0; a < 3; a++)
          for (int b = 0; b < 3; b++) {
            int i = ((mu * 4 + nu) * 3 + a) * 3 + b;
            P[mu][nu][a][b] = Float2<F>(p[2 * i], p[2 * i + 1]);
          }
  }
};

static const int (&eps)[6][3] = p2::kEps;
static const int (&sgn_eps)[6] = p2::kEpsSign;
