// Propagator pre-processing.  p2_prop_absorb builds a propagator column by
// column from the solver's spinor fields (PLEGMA_Propagator::absorb,
// lib/PLEGMA_Propagator.cu:33-95: there twelve blocking copies per column,
// here one launch).  p2_prop_transform applies, in place, the twisted-mass
// rotation to the physical basis, g5 P and the antiperiodic boundary sign of
// the reference's PLEGMA_Propagator (rotateToPhysicalBase_device,
// apply_gamma5, applyBoundaries_device; lib/kernels/PLEGMA_propagator_utils.cuh:
// 31-134).  The contraction kernels apply the same transforms while staging
// (p2_prop::transform), which saves a read and a write of the whole field;
// this kernel is for callers that need the transformed field itself.
//
// p2_prop_transform: one thread per (slice, site, transform group): the four spin blocks of a
// colour pair that the rotation mixes; consecutive threads take consecutive
// sites, so every load and store is coalesced along the site axis.  HBM
// bound: 2 x 2304 B per site (FP64) read and written once.
#include <algorithm>

#include "ctx.h"
#include "p2_common.cuh"

using namespace p2host;

namespace p2 {
namespace {

template <typename T>
__global__ void k_prop_transform(Cx<T>* p, long long V3, int nt, int t_first, int T_, int rot, int g5,
                                 int boundary, int bt0) {
  const long long n = 36LL * nt * V3;
  const long long vol = (long long)nt * V3;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long x = i % V3;
    const int j = (int)((i / V3) % nt);
    const int q = (int)(i / (V3 * nt));
    const int t = (t_first + j) % T_;
    const int code = rot | (g5 ? PropXf::kGamma5 : 0) | ((boundary && t < bt0) ? PropXf::kNegate : 0);
    int comp[4];
    prop_group_comps(q, comp);
    const long long sid = (long long)j * V3 + x;
    Cx<double> v[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const Cx<T> e = p[comp[k] * vol + sid];
      v[k] = cx<double>((double)e.x, (double)e.y);
    }
    prop_group_transform(v[0], v[1], v[2], v[3], code);
#pragma unroll
    for (int k = 0; k < 4; k++) p[comp[k] * vol + sid] = cx<T>((T)v[k].x, (T)v[k].y);
  }
}

// Column (nu, c2) of a propagator from a spinor field: component
// ((mu 4 + nu) 3 + c1) 3 + c2 of the propagator takes component mu 3 + c1 of
// the vector.  global_t < 0 copies the whole 4-D vector; otherwise the column
// is zero except slice global_t, taken from the vector's slice global_t (4-D)
// or from the 3-D vector.  Coalesced along sites, one pass.
template <typename T>
__global__ void k_prop_absorb(Cx<T>* p, const Cx<T>* v, long long V3, int nt, int t_first, int T_, int nu, int c2,
                              int vec_3d, int global_t) {
  const long long vol = (long long)nt * V3;
  const long long n = 12LL * vol;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long sid = i % vol;
    const int mc = (int)(i / vol);  // mu 3 + c1
    const int mu = mc / 3, c1 = mc % 3;
    Cx<T> e = cx<T>((T)0, (T)0);
    if (global_t < 0) {
      e = v[i];
    } else {
      const int j = (int)(sid / V3);
      if ((t_first + j) % T_ == global_t) e = vec_3d ? v[mc * V3 + sid % V3] : v[i];
    }
    p[(((mu * 4 + nu) * 3 + c1) * 3 + c2) * vol + sid] = e;
  }
}

}  // namespace
}  // namespace p2

extern "C" p2_status p2_prop_absorb(p2_ctx* c, void* prop, const void* vec, int precision, int t_first, int nt, int nu,
                                    int c2, int vec_3d, int global_t) {
  using namespace p2;
  if (!c) return P2_ERR_INVALID_ARG;
  if (c->host_only) return c->fail(P2_ERR_UNSUPPORTED, "host-only context");
  if (!prop || !vec || nt < 1 || nt > c->T || t_first < 0 || t_first >= c->T)
    return c->fail(P2_ERR_INVALID_ARG, "p2_prop_absorb: bad view");
  if (precision != P2_FP64 && precision != P2_FP32) return c->fail(P2_ERR_INVALID_ARG, "bad precision");
  if (nu < 0 || nu > 3 || c2 < 0 || c2 > 2) return c->fail(P2_ERR_INVALID_ARG, "p2_prop_absorb: nu or c2 out of range");
  if (global_t >= c->T) return c->fail(P2_ERR_INVALID_ARG, "The global time slice exceeds the temporal extent");
  if (vec_3d && global_t < 0) return c->fail(P2_ERR_INVALID_ARG, "p2_prop_absorb: a 3-D vector needs a time slice");
  const long long n = 12LL * nt * c->V3;
  const int blocks = (int)std::min<long long>((n + 255) / 256, (long long)c->nsm * 16);
  ProfScope ps(c, "prop_absorb");
  if (precision == P2_FP64)
    k_prop_absorb<double><<<blocks, 256, 0, c->stream>>>((Cx<double>*)prop, (const Cx<double>*)vec, c->V3, nt, t_first,
                                                         c->T, nu, c2, vec_3d != 0, global_t);
  else
    k_prop_absorb<float><<<blocks, 256, 0, c->stream>>>((Cx<float>*)prop, (const Cx<float>*)vec, c->V3, nt, t_first,
                                                        c->T, nu, c2, vec_3d != 0, global_t);
  return c->cuda(cudaGetLastError(), "p2_prop_absorb");
}

extern "C" p2_status p2_prop_transform(p2_ctx* c, void* data, int precision, int t_first, int nt, unsigned transform,
                                       int boundary_t0) {
  using namespace p2;
  if (!c) return P2_ERR_INVALID_ARG;
  if (c->host_only) return c->fail(P2_ERR_UNSUPPORTED, "host-only context");
  if (!data || nt < 1 || nt > c->T || t_first < 0 || t_first >= c->T)
    return c->fail(P2_ERR_INVALID_ARG, "p2_prop_transform: bad view");
  if (precision != P2_FP64 && precision != P2_FP32) return c->fail(P2_ERR_INVALID_ARG, "bad precision");
  if ((transform & ~0xFu) || ((transform & P2_PROP_ROTATE_PLUS) && (transform & P2_PROP_ROTATE_MINUS)))
    return c->fail(P2_ERR_INVALID_ARG, "p2_prop_transform: bad transform bits");
  if (!transform) return P2_OK;
  const int rot = (transform & P2_PROP_ROTATE_PLUS) ? PropXf::kRotPlus : (transform & P2_PROP_ROTATE_MINUS) ? PropXf::kRotMinus : 0;
  const long long n = 36LL * nt * c->V3;
  const int blocks = (int)std::min<long long>((n + 255) / 256, (long long)c->nsm * 16);
  ProfScope ps(c, "prop_transform");
  if (precision == P2_FP64)
    k_prop_transform<double><<<blocks, 256, 0, c->stream>>>((Cx<double>*)data, c->V3, nt, t_first, c->T, rot,
                                                            (transform & P2_PROP_GAMMA5) != 0,
                                                            (transform & P2_PROP_BOUNDARY) != 0, boundary_t0);
  else
    k_prop_transform<float><<<blocks, 256, 0, c->stream>>>((Cx<float>*)data, c->V3, nt, t_first, c->T, rot,
                                                           (transform & P2_PROP_GAMMA5) != 0,
                                                           (transform & P2_PROP_BOUNDARY) != 0, boundary_t0);
  return c->cuda(cudaGetLastError(), "p2_prop_transform");
}
