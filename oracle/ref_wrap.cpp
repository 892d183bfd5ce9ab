// C entry points over the reference's own nucleon and Delta contraction
// functions (lib/kernels/PLEGMA_baryons_NtoN.cu, _NtoR.cu, _RtoN.cu, _RtoR.cu,
// PLEGMA_baryons_deltas.cu),
// compiled from the reference sources as host code by oracle/build.py.
// TEST INFRASTRUCTURE ONLY: used by tests/ to pin the oracle.
#include "ref_shim/PLEGMA_kernel_utils.cuh"

template <typename FloatA, typename FloatB, typename FloatC>
void contract_NtoN_kernel(propTex<FloatA>&, propTex<FloatB>&, Float2<FloatC>*, int);
template <typename FloatA, typename FloatB, typename FloatC>
void contract_NtoR_kernel(propTex<FloatA>&, propTex<FloatB>&, Float2<FloatC>*, int);
template <typename FloatA, typename FloatB, typename FloatC>
void contract_RtoN_kernel(propTex<FloatA>&, propTex<FloatB>&, Float2<FloatC>*, int);
template <typename FloatA, typename FloatB, typename FloatC>
void contract_RtoR_kernel(propTex<FloatA>&, propTex<FloatB>&, Float2<FloatC>*, int);
template <typename FloatA, typename FloatB, typename FloatC, int gamma>
void contract_deltas_iso1o2_kernel(propTex<FloatA>&, propTex<FloatB>&, Float2<FloatC>*, int);
template <typename FloatA, typename FloatB, typename FloatC, int gamma>
void contract_deltas_iso3o2_kernel(propTex<FloatA>&, propTex<FloatB>&, Float2<FloatC>*, int);

namespace {
void copy_out(const Float2<double>* a, int n, double* out) {
  for (int i = 0; i < n; i++) {
    out[2 * i] = a[i].x;
    out[2 * i + 1] = a[i].y;
  }
}
}  // namespace

extern "C" {
// u, d: one site's 144 complex doubles; out: 32 complex ([2][4][4]).
void ref_nucleon(const double* u, const double* d, double* out) {
  propTex<double> t1(u), t2(d);
  Float2<double> acc[32];
  contract_NtoN_kernel<double, double, double>(t1, t2, acc, 0);
  copy_out(acc, 32, out);
}

// which: 0 NtoR, 1 RtoN, 2 RtoR; out: 32 complex ([2][4][4]).
void ref_light(const double* u, const double* d, int which, double* out) {
  propTex<double> t1(u), t2(d);
  Float2<double> acc[32];
  for (int i = 0; i < 32; i++) acc[i] = Float2<double>(0., 0.);
  if (which == 0) contract_NtoR_kernel<double, double, double>(t1, t2, acc, 0);
  if (which == 1) contract_RtoN_kernel<double, double, double>(t1, t2, acc, 0);
  if (which == 2) contract_RtoR_kernel<double, double, double>(t1, t2, acc, 0);
  copy_out(acc, 32, out);
}

void ref_delta(const double* u, const double* d, int iso32, int g, double* out) {
  propTex<double> t1(u), t2(d);
  Float2<double> acc[32];
  if (!iso32) {
    if (g == 0) contract_deltas_iso1o2_kernel<double, double, double, 0>(t1, t2, acc, 0);
    if (g == 1) contract_deltas_iso1o2_kernel<double, double, double, 1>(t1, t2, acc, 0);
    if (g == 2) contract_deltas_iso1o2_kernel<double, double, double, 2>(t1, t2, acc, 0);
  } else {
    if (g == 0) contract_deltas_iso3o2_kernel<double, double, double, 0>(t1, t2, acc, 0);
    if (g == 1) contract_deltas_iso3o2_kernel<double, double, double, 1>(t1, t2, acc, 0);
    if (g == 2) contract_deltas_iso3o2_kernel<double, double, double, 2>(t1, t2, acc, 0);
  }
  copy_out(acc, 32, out);
}
}
