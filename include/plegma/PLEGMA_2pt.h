// Drop-in C++ surface of the two-point path: PLEGMA_init, site,
// PLEGMA_Field / PLEGMA_Propagator, PLEGMA_FT and PLEGMA_Correlator, with the
// reference's names, argument meanings and buffer layouts, implemented over
// the C ABI of plegma2pt.h (link with -lplegma2pt; no CUDA runtime needed in
// the caller).
//
// Reference interfaces mirrored:
//   PLEGMA_init                  lib/PLEGMA.cu:19-212 (one process; geometry only)
//   site                         include/global/PLEGMA_structs.h:4-13
//   PLEGMA_Field / Propagator    include/PLEGMA_Field.h:84-160, include/PLEGMA_Propagator.h:14-60
//   PLEGMA_FT                    include/PLEGMA_FT.h:10-135, lib/PLEGMA_FT.cu:14-182
//   PLEGMA_Correlator            include/PLEGMA_Correlator.h:18-215, lib/PLEGMA_Correlator.cu:25-189,721-807
//
// Differences, by design:
//   - argument errors throw plegma::PLEGMA_exception instead of aborting the
//     process (PLEGMA_error, include/global/PLEGMA_prints.hpp:49-81);
//   - writeFile(HDF5_FORMAT / DEFAULT_FORMAT) writes the same datasets as raw
//     little-endian binary plus a JSON sidecar (no HDF5 library here);
//   - contractions take an optional arithmetic mode (PLAIN_FP64 or SPLIT_FP16).
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../plegma2pt.h"

namespace plegma {

enum LATDIMS { DIM_X, DIM_Y, DIM_Z, DIM_T, N_DIMS };
enum CORR_SPACE { POSITION_SPACE, MOMENTUM_SPACE };
enum FILE_FORMAT { ASCII_FORMAT, HDF5_FORMAT, LIME_FORMAT, DEFAULT_FORMAT };
enum ALLOCATION_FLAG { EVERY = -1, NONE = 0, HOST, DEVICE, BOTH };
enum GHOST_FLAG { ALL_GHOSTS = -1, NO_GHOSTS, FIRST_SIDE, FIRST_CORNER, FIRST_VERTEX };
// FT_SPLIT (not in the reference): the tensor-core projection of p2_ft_apply_split.
enum FT_TYPE { FT_NAIVE, FT_GEMV, FT_FFT, FT_SPLIT };
enum GAMMAS { ONE, G1, G2, G3, G4, G5, G5G1, G5G2, G5G3, G5G4, S12, S13, S23, S41, S42, S43 };
enum CONTRACTION_MODE { PLAIN_FP64 = P2_PLAIN_FP64, SPLIT_FP16 = P2_SPLIT_FP16 };

struct PLEGMA_exception : std::runtime_error {
  using std::runtime_error::runtime_error;
};

struct site : std::array<int, N_DIMS> {
  site() = default;
  site(const std::array<int, N_DIMS>& v) : std::array<int, N_DIMS>(v) {}
  site(int x, int y, int z, int t) : std::array<int, N_DIMS>{{x, y, z, t}} {}
};

// The process-wide geometry and library context (the reference's HGC_* globals).
struct Runtime {
  p2_ctx* ctx = nullptr;
  std::array<int, 4> totalL{{0, 0, 0, 0}}, nProcs{{1, 1, 1, 1}}, procPosition{{0, 0, 0, 0}}, localL{{0, 0, 0, 0}};
  size_t localVolume3D = 0, localVolume = 0;
  static Runtime& get() {
    static Runtime r;
    return r;
  }
  static p2_ctx* context() {
    Runtime& r = get();
    if (!r.ctx) throw PLEGMA_exception("PLEGMA_init has not been called");
    return r.ctx;
  }
  static void check(p2_status s, const char* where) {
    if (s != P2_OK) {
      std::string m = std::string(where) + ": " + p2_last_error(get().ctx) + " (status " + std::to_string(s) + ")";
      throw PLEGMA_exception(m);
    }
  }
};

inline void PLEGMA_init(std::array<int, 4> totalL, std::array<int, 4> nProcs = {{1, 1, 1, 1}}, int device = 0,
                        std::array<int, 4> procPosition = {{0, 0, 0, 0}}) {
  Runtime& r = Runtime::get();
  if (r.ctx) p2_ctx_destroy(r.ctx);
  p2_geom g{};
  for (int d = 0; d < 4; d++) {
    g.L[d] = totalL[d];
    g.procs[d] = nProcs[d];
    g.coords[d] = procPosition[d];
  }
  g.device = device;
  if (p2_ctx_create(&g, &r.ctx) != P2_OK) throw PLEGMA_exception("PLEGMA_init: cannot create the library context");
  r.totalL = totalL;
  r.nProcs = nProcs;
  r.procPosition = procPosition;
  for (int d = 0; d < 4; d++) r.localL[d] = totalL[d] / nProcs[d];
  r.localVolume3D = (size_t)r.localL[0] * r.localL[1] * r.localL[2];
  r.localVolume = r.localVolume3D * r.localL[3];
}

inline void PLEGMA_finalize() {
  Runtime& r = Runtime::get();
  if (r.ctx) p2_ctx_destroy(r.ctx);
  r.ctx = nullptr;
}

template <typename Float>
constexpr int precision_of() {
  return sizeof(Float) == 8 ? P2_FP64 : P2_FP32;
}

// Complex field of `field_length` components per site, SoA [component][site].
template <typename Float>
class PLEGMA_Field {
 protected:
  ALLOCATION_FLAG alloc = NONE;
  int field_length = 0;
  size_t total_length = 0;
  Float* d_elem = nullptr;
  Float* h_elem = nullptr;

 public:
  PLEGMA_Field(ALLOCATION_FLAG a, int field_length, size_t total_length)
      : alloc(a), field_length(field_length), total_length(total_length) {
    p2_ctx* c = Runtime::context();
    const size_t bytes = bytes_();
    if (a == DEVICE || a == BOTH) Runtime::check(p2_alloc(c, bytes, P2_DEVICE, (void**)&d_elem), "create_device");
    if (a == HOST || a == BOTH) Runtime::check(p2_alloc(c, bytes, P2_HOST, (void**)&h_elem), "create_host");
  }
  PLEGMA_Field(const PLEGMA_Field&) = delete;
  PLEGMA_Field& operator=(const PLEGMA_Field&) = delete;
  virtual ~PLEGMA_Field() {
    p2_ctx* c = Runtime::get().ctx;
    if (c) {
      p2_free(c, d_elem, P2_DEVICE);
      p2_free(c, h_elem, P2_HOST);
    }
  }
  size_t bytes_() const { return (size_t)field_length * total_length * 2 * sizeof(Float); }
  Float* D_elem() const { return d_elem; }
  Float* H_elem() const { return h_elem; }
  ALLOCATION_FLAG getAllocation() const { return alloc; }
  int Field_length() const { return field_length; }
  size_t Total_length() const { return total_length; }
  void copyToDevice() {
    if (!d_elem || !h_elem) throw PLEGMA_exception("copyToDevice: field needs host and device storage");
    Runtime::check(p2_copy(Runtime::context(), d_elem, h_elem, bytes_()), "copyToDevice");
  }
  void copyToHost() {
    if (!d_elem || !h_elem) throw PLEGMA_exception("copyToHost: field needs host and device storage");
    Runtime::check(p2_copy(Runtime::context(), h_elem, d_elem, bytes_()), "copyToHost");
  }
};

// Spinor fields (12 components, [mu 3 + c1][site]): the solver's output that
// a propagator absorbs column by column (include/PLEGMA_Vector.h).
template <typename Float>
class PLEGMA_Vector : public PLEGMA_Field<Float> {
 public:
  explicit PLEGMA_Vector(ALLOCATION_FLAG a = BOTH, GHOST_FLAG = FIRST_SIDE)
      : PLEGMA_Field<Float>(a, 12, Runtime::get().localVolume) {}
};
template <typename Float>
class PLEGMA_Vector3D : public PLEGMA_Field<Float> {
 public:
  explicit PLEGMA_Vector3D(ALLOCATION_FLAG a = BOTH)
      : PLEGMA_Field<Float>(a, 12, Runtime::get().localVolume / Runtime::get().localL[DIM_T]) {}
};

template <typename Float>
class PLEGMA_Propagator : public PLEGMA_Field<Float> {
 public:
  explicit PLEGMA_Propagator(ALLOCATION_FLAG a = BOTH, GHOST_FLAG = FIRST_SIDE)
      : PLEGMA_Field<Float>(a, 144, Runtime::get().localVolume) {}
  // Seeded synthetic entries (Gaussian x exp(-decay |t - t0|)), generated where the field lives.
  void fillSynthetic(uint64_t seed, int flavour, int t0, double decay) {
    p2_ctx* c = Runtime::context();
    const int nt = Runtime::get().localL[DIM_T];
    const int t_first = Runtime::get().procPosition[DIM_T] * nt;
    if (this->d_elem)
      Runtime::check(p2_synth_propagator(c, this->d_elem, 1, precision_of<Float>(), seed, flavour, t0, decay, t_first, nt),
                     "fillSynthetic");
    if (this->h_elem) {
      if (this->d_elem)
        this->copyToHost();
      else
        Runtime::check(
            p2_synth_propagator(c, this->h_elem, 0, precision_of<Float>(), seed, flavour, t0, decay, t_first, nt),
            "fillSynthetic");
    }
  }
  // Column (nu, c2) from a spinor field, device to device
  // (lib/PLEGMA_Propagator.cu:33-95): the whole 4-D vector; or only global
  // slice global_it (from a 4-D or a 3-D vector), the rest of the column zero.
  void absorb(PLEGMA_Vector<Float>& vec, int nu, int c2) { absorb_(vec.D_elem(), 0, -1, nu, c2); }
  void absorb(PLEGMA_Vector<Float>& vec, int global_it, int nu, int c2) {
    absorb_(vec.D_elem(), 0, global_it, nu, c2);
  }
  void absorb(PLEGMA_Vector3D<Float>& vec, int global_it, int nu, int c2) {
    absorb_(vec.D_elem(), 1, global_it, nu, c2);
  }
  // In-place pre-processing on the device copy, as the reference's methods
  // (lib/PLEGMA_Propagator.cu:98-107,190-192): the physical-basis rotation
  // with sign +-1, g5 P, and the antiperiodic sign on global t < t0.
  void rotateToPhysicalBase_device(int sign) {
    if (sign != 1 && sign != -1) throw PLEGMA_exception("The sign can be only +-1");
    transform_(sign > 0 ? P2_PROP_ROTATE_PLUS : P2_PROP_ROTATE_MINUS, 0, "rotateToPhysicalBase_device");
  }
  void applyBoundaries_device(int t0) { transform_(P2_PROP_BOUNDARY, t0, "applyBoundaries_device"); }
  void apply_gamma5() { transform_(P2_PROP_GAMMA5, 0, "apply_gamma5"); }
  // The host copy: through the device copy (lib/PLEGMA_Propagator.cu:111-188
  // rotates on the host; the result is the same).
  void rotateToPhysicalBase_host(int sign) {
    if (sign != 1 && sign != -1) throw PLEGMA_exception("The sign can be only +-1");
    if (!this->h_elem || !this->d_elem)
      throw PLEGMA_exception("rotateToPhysicalBase_host: field needs host and device storage");
    this->copyToDevice();
    rotateToPhysicalBase_device(sign);
    this->copyToHost();
  }
  // The same transforms applied while contracting instead, leaving the stored
  // field as it is (no extra pass over the field): flags P2_PROP_*.
  void transformOnLoad(unsigned flags, int boundary_t0 = 0) {
    load_xf = flags;
    load_t0 = boundary_t0;
  }
  p2_prop view() const {
    p2_prop p{};
    p.transform = load_xf;
    p.boundary_t0 = load_t0;
    p.data = this->d_elem ? (const void*)this->d_elem : (const void*)this->h_elem;
    if (!p.data) throw PLEGMA_exception("propagator has no storage");
    p.precision = precision_of<Float>();
    p.location = this->d_elem ? P2_DEVICE : P2_HOST;
    p.t_first = Runtime::get().procPosition[DIM_T] * Runtime::get().localL[DIM_T];
    p.nt = Runtime::get().localL[DIM_T];
    return p;
  }

 private:
  unsigned load_xf = 0;
  int load_t0 = 0;
  void absorb_(const Float* v, int vec_3d, int global_it, int nu, int c2) {
    if (!this->d_elem || !v) throw PLEGMA_exception("absorb: propagator and vector need device storage");
    if (global_it >= Runtime::get().totalL[DIM_T])
      throw PLEGMA_exception("The global time slice you provided exceed the temporal extent");
    Runtime::check(p2_prop_absorb(Runtime::context(), this->d_elem, v, precision_of<Float>(),
                                  Runtime::get().procPosition[DIM_T] * Runtime::get().localL[DIM_T],
                                  Runtime::get().localL[DIM_T], nu, c2, vec_3d, global_it),
                   "absorb");
  }
  void transform_(unsigned flags, int t0, const char* what) {
    if (!this->d_elem) throw PLEGMA_exception(std::string(what) + ": propagator has no device storage");
    Runtime::check(p2_prop_transform(Runtime::context(), this->d_elem, precision_of<Float>(),
                                     Runtime::get().procPosition[DIM_T] * Runtime::get().localL[DIM_T],
                                     Runtime::get().localL[DIM_T], flags, t0),
                   what);
  }
};

template <typename Float>
class PLEGMA_FT {
  using VFloat = std::vector<Float>;
  using VVFloat = std::vector<VFloat>;
  int Q2_max = 0;
  VVFloat momList;
  int dof = 0, dims = 3, dimT = 0;
  bool accum = false;
  std::vector<Float> h;

 public:
  PLEGMA_FT(int Q2_max, int D3D4 = 3, bool accum = false, int dimT = -1)
      : Q2_max(Q2_max), dims(D3D4), dimT(dimT < 0 ? Runtime::get().localL[DIM_T] : dimT), accum(accum) {
    if (dims != 3) throw PLEGMA_exception("PLEGMA_FT: only 3-D transforms are supported");
    if (Q2_max < 0) throw PLEGMA_exception("The maximum number of Q2 cannot be negative");
    const int n = p2_mom_list(Q2_max, nullptr);
    std::vector<int> m(3 * n);
    p2_mom_list(Q2_max, m.data());
    for (int i = 0; i < n; i++) momList.push_back({(Float)m[3 * i], (Float)m[3 * i + 1], (Float)m[3 * i + 2]});
  }
  template <typename T>
  PLEGMA_FT(std::vector<std::vector<T>>& moms, int D3D4 = 3, bool accum = false, int dimT = -1)
      : dims(D3D4), dimT(dimT < 0 ? Runtime::get().localL[DIM_T] : dimT), accum(accum) {
    if (dims != 3) throw PLEGMA_exception("PLEGMA_FT: only 3-D transforms are supported");
    for (auto& m : moms) {
      if (m.size() != 3) throw PLEGMA_exception("The size of the momentum vector does not match the dimensionality");
      momList.push_back(VFloat(m.begin(), m.end()));
    }
  }
  // One momentum (lib/PLEGMA_FT.cu:23-31).
  template <typename T, typename = typename std::enable_if<std::is_arithmetic<T>::value>::type>
  PLEGMA_FT(std::vector<T> mom, int D3D4 = 3, bool accum = false, int dimT = -1)
      : dims(D3D4), dimT(dimT < 0 ? Runtime::get().localL[DIM_T] : dimT), accum(accum) {
    if (dims != 3) throw PLEGMA_exception("PLEGMA_FT: only 3-D transforms are supported");
    if (mom.size() != 3) throw PLEGMA_exception("The size of the momentum vector does not match the dimensionality of FT");
    momList.push_back(VFloat(mom.begin(), mom.end()));
  }
  int Nmoms() const { return (int)momList.size(); }
  VVFloat MomList() const { return momList; }
  int Dims() const { return dims; }
  int DimT() const { return dimT; }
  bool IsAccum() const { return accum; }
  Float* H_elem() { return h.empty() ? nullptr : h.data(); }
  std::vector<int> int_moms() const {
    std::vector<int> m;
    for (auto& v : momList)
      for (auto x : v) m.push_back((int)std::lround(x));
    return m;
  }
  void checkAllocation(int newDof) {
    dof = newDof;
    h.assign((size_t)Nmoms() * dimT * dof * 2, Float(0));
  }
  void zero() { std::fill(h.begin(), h.end(), Float(0)); }
  // PLEGMA_FT::apply: buffer [t][dof][mom] complex (lib/PLEGMA_FT.cu:155-162, PLEGMA_FT.cuh:149-157).
  void apply(const PLEGMA_Field<Float>& f, FT_TYPE type = FT_GEMV, int sign = -1) {
    if (type == FT_FFT) throw PLEGMA_exception("FT_FFT is not implemented (as in the reference)");
    if (sizeof(Float) != 8) throw PLEGMA_exception("PLEGMA_FT::apply: FP64 fields only");
    if (!f.D_elem()) throw PLEGMA_exception("PLEGMA_FT::apply: field has no device storage");
    const int nt = (int)(f.Total_length() / Runtime::get().localVolume3D);
    if (h.empty() || dof != f.Field_length() || nt != dimT) {
      dimT = nt;
      checkAllocation(f.Field_length());
    }
    std::vector<double> out((size_t)Nmoms() * dimT * dof * 2);
    std::vector<int> m = int_moms();
    Runtime::check((type == FT_SPLIT ? p2_ft_apply_split : p2_ft_apply)(Runtime::context(), (const double*)f.D_elem(),
                                                                        dof, dimT, m.data(), Nmoms(), sign,
                                                                        out.data(), P2_HOST),
                   "PLEGMA_FT::apply");
    for (size_t i = 0; i < out.size(); i++) h[i] = accum ? h[i] + (Float)out[i] : (Float)out[i];
  }
  // Constant source phase exp(sign i 2 pi p.src / L) (lib/PLEGMA_FT.cu:164-182).
  void mulConstMomentumPhases(std::vector<int> src, int sign) {
    if (src.size() != 3) throw PLEGMA_exception("src size is incompatible with the dimensionality of the FT");
    if (sign != 1 && sign != -1) throw PLEGMA_exception("Sign should be either +1 or -1");
    if (h.empty()) throw PLEGMA_exception("Apply first FT and then the const phases");
    const auto& L = Runtime::get().totalL;
    for (int p = 0; p < Nmoms(); p++) {
      double ph = 0;
      for (int i = 0; i < 3; i++) ph += (double)src[i] * momList[p][i] / (double)L[i];
      ph *= 2.0 * 3.14159265358979323846;
      const double c = std::cos(ph), s = sign * std::sin(ph);
      for (int d = 0; d < dof; d++)
        for (int t = 0; t < dimT; t++) {
          Float* z = &h[2 * ((size_t)t * dof * Nmoms() + (size_t)d * Nmoms() + p)];
          const double re = z[0], im = z[1];
          z[0] = (Float)(re * c - im * s);
          z[1] = (Float)(re * s + im * c);
        }
    }
  }
};

template <typename Float>
class PLEGMA_Correlator {
 protected:
  const site source;
  const int totalT;
  std::vector<int> shape;
  std::vector<std::string> datasets, groups;
  std::string description;
  const CORR_SPACE corr_space;
  std::shared_ptr<PLEGMA_FT<Float>> corr_mom_space;
  std::vector<Float> buf;  // reference buffer layout, see H_elem()
  CONTRACTION_MODE mode = PLAIN_FP64;

  static const Runtime& R() { return Runtime::get(); }

  // Runs the library and stores the result in the reference's host layout.
  void run(const PLEGMA_Propagator<Float>& p1, const PLEGMA_Propagator<Float>& p2, unsigned what, bool meson_diag) {
    p2_ctx* c = Runtime::context();
    const int lt = localT();
    if (corr_space == MOMENTUM_SPACE) {
      std::vector<int> m = corr_mom_space->int_moms();
      const int nmom = (int)m.size() / 3;
      size_t total = 0;
      p2_block blocks[8];
      const int nb = p2_block_info(what, totalT, nmom, blocks, 8, &total);
      std::vector<double> res(2 * total, 0.0);
      p2_prop props[2] = {p1.view(), p2.view()};
      p2_request r{};
      for (int d = 0; d < 4; d++) r.source[d] = source[d];
      r.totalT = totalT;
      r.moms = m.data();
      r.nmom = nmom;
      r.contractions = what;
      r.mode = mode;
      r.prop_u = 0;
      r.prop_d = 1;
      r.out = res.data();
      r.out_location = P2_HOST;
      Runtime::check(p2_contract_project(c, props, 2, &r, 1), "contract");
      buf.assign(getTotalSize() * 2, Float(0));
      size_t off = 0;  // running offset in the reference buffer (complex)
      for (int b = 0; b < nb; b++) {
        const p2_block& B = blocks[b];
        for (int g = 0; g < B.groups; g++)
          for (int ds = 0; ds < B.datasets; ds++)
            for (int i = 0; i < lt; i++) {
              const int tau = (i + startT()) % totalT;
              for (int p = 0; p < nmom; p++)
                for (int s = 0; s < B.comps; s++) {
                  const size_t src = B.offset + ((((size_t)g * B.datasets + ds) * totalT + tau) * nmom + p) * B.comps + s;
                  size_t dst;
                  if (meson_diag)  // contract_mesons stores [t][mom][dataset][10] (PLEGMA_mesons.cuh:113-120)
                    dst = (((size_t)i * nmom + p) * B.datasets + ds) * B.comps + s;
                  else
                    dst = off + ((((size_t)g * B.datasets + ds) * lt + i) * nmom + p) * B.comps + s;
                  buf[2 * dst] = (Float)res[2 * src];
                  buf[2 * dst + 1] = (Float)res[2 * src + 1];
                }
            }
        off += (size_t)B.groups * B.datasets * lt * nmom * B.comps;
      }
    } else {
      const int K = p2_components(what);
      const size_t V3 = R().localVolume3D;
      std::vector<double> res((size_t)2 * totalT * K * V3, 0.0);
      p2_prop props[2] = {p1.view(), p2.view()};
      p2_request r{};
      for (int d = 0; d < 4; d++) r.source[d] = source[d];
      r.totalT = totalT;
      r.contractions = what;
      r.prop_u = 0;
      r.prop_d = 1;
      r.out = res.data();
      r.out_location = P2_HOST;
      Runtime::check(p2_contract_position(c, props, 2, &r), "contract");
      // reference position-space layout: [group*dataset][t][x3][comp] for baryons
      // (PLEGMA_baryons.cuh:157-161,200-201), [t][x3][site] otherwise
      buf.assign(getTotalSize() * 2, Float(0));
      size_t total = 0;
      p2_block blocks[8];
      const int nb = p2_block_info(what, 1, 1, blocks, 8, &total);
      int k0 = 0;
      size_t off = 0;
      for (int b = 0; b < nb; b++) {
        const p2_block& B = blocks[b];
        const bool baryon = B.bit == P2_NUCLEON_CG5 || B.bit == P2_NUCLEON_NTOR || B.bit == P2_NUCLEON_RTON ||
                            B.bit == P2_NUCLEON_RTOR || B.bit == P2_DELTA_ISO12 || B.bit == P2_DELTA_ISO32;
        for (int gd = 0; gd < B.groups * B.datasets; gd++)
          for (int i = 0; i < lt; i++) {
            const int tau = (i + startT()) % totalT;
            for (size_t x = 0; x < V3; x++)
              for (int s = 0; s < B.comps; s++) {
                const size_t src = ((size_t)tau * K + k0 + gd * B.comps + s) * V3 + x;
                const size_t dst = baryon ? off + (((size_t)gd * lt + i) * V3 + x) * B.comps + s
                                          : off + ((size_t)i * V3 + x) * (B.groups * B.datasets * B.comps) +
                                                gd * B.comps + s;
                buf[2 * dst] = (Float)res[2 * src];
                buf[2 * dst + 1] = (Float)res[2 * src + 1];
              }
          }
        k0 += B.groups * B.datasets * B.comps;
        off += (size_t)B.groups * B.datasets * lt * V3 * B.comps;
      }
    }
  }

 public:
  PLEGMA_Correlator(CORR_SPACE corr_space, site source, int Q2_max = 0, int totalT = -1)
      : source(source), totalT(totalT < 0 ? Runtime::get().totalL[DIM_T] : totalT), corr_space(corr_space) {
    if (this->totalT < 1 || this->totalT > R().totalL[DIM_T]) throw PLEGMA_exception("totalT out of range");
    if (corr_space == MOMENTUM_SPACE) corr_mom_space.reset(new PLEGMA_FT<Float>(Q2_max, 3, false, localT()));
  }

  // include/PLEGMA_Correlator.h:41-79
  bool hasSource(int dir) const {
    if (dir < 0 || dir >= N_DIMS) return false;
    return (R().procPosition[dir] * R().localL[dir] <= source[dir]) &&
           (source[dir] < (R().procPosition[dir] + 1) * R().localL[dir]);
  }
  bool hasSource() const {
    bool ret = true;
    for (int d = 0; ret && d < N_DIMS; d++) ret &= hasSource(d);
    return ret;
  }
  int startT() const {
    const int start = (R().procPosition[DIM_T] * R().localL[DIM_T] + R().totalL[DIM_T] - source[DIM_T]) % R().totalL[DIM_T];
    return (start >= totalT) ? 0 : start;
  }
  int endT() const {
    const int start = startT();
    return start > 0 ? std::min(totalT, R().localL[DIM_T] + start) : 0;
  }
  int localT() const {
    if (hasSource(DIM_T)) {
      const int ts = source[DIM_T] % R().localL[DIM_T];
      return endT() - startT() + std::min(totalT, R().localL[DIM_T] - ts);
    }
    return endT() - startT();
  }

  void setMode(CONTRACTION_MODE m) { mode = m; }
  CORR_SPACE getCorrSpace() const { return corr_space; }
  Float* H_elem() { return buf.empty() ? nullptr : buf.data(); }
  site getSource() const { return source; }
  int getTotalT() const { return totalT; }
  size_t nDatasets() const { return std::max(datasets.size(), (size_t)1); }
  size_t nGroups() const { return std::max(groups.size(), (size_t)1); }
  size_t getSiteSize() const {
    size_t s = nDatasets() * nGroups();
    for (int n : shape) s *= n;
    return s;
  }
  size_t getVolSize() const {
    return corr_space == MOMENTUM_SPACE ? (size_t)corr_mom_space->Nmoms() * localT() : R().localVolume3D * localT();
  }
  size_t getTotalSize() const { return getSiteSize() * getVolSize(); }
  void setQ2max(int Q2_max) { corr_mom_space.reset(new PLEGMA_FT<Float>(Q2_max, 3, false, localT())); }
  void setFixMomList(std::vector<std::vector<int>>& l) {
    corr_mom_space.reset(new PLEGMA_FT<Float>(l, 3, false, localT()));
  }
  // One fixed momentum (include/PLEGMA_Correlator.h:135-138).
  void setFixMomVec(std::vector<int>& v) { corr_mom_space.reset(new PLEGMA_FT<Float>(v, 3, false, localT())); }
  std::vector<std::vector<int>> getMomList() const {
    std::vector<std::vector<int>> out;
    if (corr_space != MOMENTUM_SPACE) return out;
    for (auto& m : corr_mom_space->MomList()) {
      out.emplace_back();
      for (auto x : m) out.back().push_back((int)std::lround(x));
    }
    return out;
  }
  std::vector<std::string> getDatasets() const { return datasets; }
  std::vector<std::string> getGroups() const { return groups; }
  void setDatasets(std::vector<std::string> d) {
    if (datasets.size() == d.size() || (datasets.empty() && d.size() == 1))
      datasets = d;
    else
      throw PLEGMA_exception("Given vector size do not match. This would change the correlator size.");
  }
  void setGroups(std::vector<std::string> d) {
    if (groups.size() == d.size() || (groups.empty() && d.size() == 1))
      groups = d;
    else
      throw PLEGMA_exception("Given vector size do not match. This would change the correlator size.");
  }

  // lib/PLEGMA_Correlator.cu:43-55
  void contractMesons(PLEGMA_Propagator<Float>& p1, PLEGMA_Propagator<Float>& p2) {
    shape = {10};
    datasets = {"twop_meson_1", "twop_meson_2"};
    groups = {"mesons"};
    description = "pseudoscalar, scalar, g5g1, g5g2, g5g3, g5g4, g1, g2, g3, g4";
    run(p1, p2, P2_MESON_DIAG10, true);
  }
  // lib/PLEGMA_Correlator.cu:58-72
  void contractMesonsNew(PLEGMA_Propagator<Float>& p1, PLEGMA_Propagator<Float>& p2) {
    shape = {10};
    datasets = {"twop_meson"};
    groups = {"mesons"};
    description = "pseudoscalar, scalar, g5g1, g5g2, g5g3, g5g4, g1, g2, g3, g4";
    run(p1, p2, P2_MESON_NEW10, false);
  }
  // lib/PLEGMA_Correlator.cu:74-94
  void contractMesonsAll(PLEGMA_Propagator<Float>& p1, PLEGMA_Propagator<Float>& p2) {
    shape = {34};
    datasets = {"twop_meson"};
    groups = {"mesons"};
    description = "pseudoscalar, scalar";
    for (int p = 0; p < 2; p++) {
      std::string va = p ? "" : "g5";
      for (int i = 1; i < 5; i++)
        for (int j = 1; j < 5; j++)
          description += ", (" + va + "g" + std::to_string(i) + "," + va + "g" + std::to_string(j) + ")";
    }
    run(p1, p2, P2_MESON_ALL34, false);
  }
  // All 16 x 16 (Gamma_sink, Gamma_src) pairs of the generic insertion of PLEGMA_mesonsAll.cuh:52-76.
  void contractMesonsG16(PLEGMA_Propagator<Float>& p1, PLEGMA_Propagator<Float>& p2) {
    shape = {16, 16};
    datasets = {"twop_meson"};
    groups = {"mesons"};
    description = "(g_sink,g_src) over 1,g1,g2,g3,g4,g5,g5g1,g5g2,g5g3,g5g4,s12,s13,s23,s41,s42,s43";
    run(p1, p2, P2_MESON_G16, false);
  }
  // lib/PLEGMA_Correlator.cu:117-135: nucleon C g5 (proton, neutron); with
  // deltas, the Delta C g_k groups of the light-baryon build after it.
  // lib/PLEGMA_Correlator.cu:117-135; light_build = the reference built with
  // PLEGMA_LIGHT_BARYONS: the second nucleon interpolator and the Deltas too.
  void contractBaryons(PLEGMA_Propagator<Float>& p1, PLEGMA_Propagator<Float>& p2, bool light_build = false) {
    shape = {16};
    datasets = {"twop_baryon_1", "twop_baryon_2"};
    groups = {"baryons/nucl_nucl"};
    unsigned what = P2_NUCLEON_CG5;
    if (light_build) {
      for (const char* g : {"baryons/nucl_nucl2", "baryons/nucl2_nucl", "baryons/nucl2_nucl2",
                            "baryons/deltap_deltaz_11", "baryons/deltap_deltaz_22", "baryons/deltap_deltaz_33",
                            "baryons/deltapp_deltamm_11", "baryons/deltapp_deltamm_22", "baryons/deltapp_deltamm_33"})
        groups.push_back(g);
      what |= P2_NUCLEON_NTOR | P2_NUCLEON_RTON | P2_NUCLEON_RTOR | P2_DELTA_ISO12 | P2_DELTA_ISO32;
    }
    description = "1,g1,g2,g3,g4,g5,g5g1,g5g2,g5g3,g5g4,s12,s13,s23,s41,s42,s43";
    run(p1, p2, what, false);
  }

  // lib/PLEGMA_Correlator.cu:137-189: the table-driven baryon set over the u,
  // d, s, c propagators; a propagator created with NONE is not available and
  // the flavour products that need it are skipped.  One dataset per
  // (baryon, interpolator) with an empty shape.  Momentum space; FP64.
  void contractBaryonsUDSC(PLEGMA_Propagator<Float>& up, PLEGMA_Propagator<Float>& dn, PLEGMA_Propagator<Float>& st,
                           PLEGMA_Propagator<Float>& ch, bool only_st = false, bool only_ch = false) {
    if (corr_space != MOMENTUM_SPACE)
      throw PLEGMA_exception("contractBaryonsUDSC: position-space output is not supported");
    PLEGMA_Propagator<Float>* all[4] = {&up, &dn, &st, &ch};
    std::vector<p2_prop> props;
    int idx[4];
    for (int k = 0; k < 4; k++) {
      idx[k] = all[k]->getAllocation() == NONE ? -1 : (int)props.size();
      if (idx[k] >= 0) props.push_back(all[k]->view());
    }
    std::vector<int> m = corr_mom_space->int_moms();
    const int nmom = (int)m.size() / 3;
    p2_udsc_request r{};
    for (int d = 0; d < 4; d++) r.source[d] = source[d];
    r.totalT = totalT;
    r.moms = m.data();
    r.nmom = nmom;
    r.prop_u = idx[0];
    r.prop_d = idx[1];
    r.prop_s = idx[2];
    r.prop_c = idx[3];
    r.only_st = only_st;
    r.only_ch = only_ch;
    r.mode = mode;
    const int nd = p2_udsc_datasets(&r, nullptr, 0);
    std::vector<char> text((size_t)64 * (nd + 1), 0);
    p2_udsc_datasets(&r, text.data(), text.size());
    shape = {};
    groups = {};
    description = "";
    datasets.clear();
    std::string cur;
    for (char ch_ : std::string(text.data())) {
      if (ch_ == '\n') {
        datasets.push_back(cur);
        cur.clear();
      } else {
        cur += ch_;
      }
    }
    buf.assign(getTotalSize() * 2, Float(0));
    if (nd == 0) return;
    std::vector<double> res((size_t)2 * nd * totalT * nmom, 0.0);
    r.out = res.data();
    r.out_location = P2_HOST;
    Runtime::check(p2_contract_udsc(Runtime::context(), props.data(), (int)props.size(), &r), "contract");
    const int lt = localT();
    for (int d = 0; d < nd; d++)
      for (int i = 0; i < lt; i++) {
        const int tau = (i + startT()) % totalT;
        for (int p = 0; p < nmom; p++) {
          const size_t src = ((size_t)d * totalT + tau) * nmom + p;
          const size_t dst = ((size_t)d * lt + i) * nmom + p;
          buf[2 * dst] = (Float)res[2 * src];
          buf[2 * dst + 1] = (Float)res[2 * src + 1];
        }
      }
  }

  // ASCII writer of lib/PLEGMA_Correlator.cu:721-807 (momentum space, one process).
  void writeASCII(const std::string& filename_out) const {
    if (corr_space != MOMENTUM_SPACE) throw PLEGMA_exception("WriteASCII do not support writing in position space.");
    char suffix[64];
    std::snprintf(suffix, sizeof(suffix), "_sx%02dsy%02dsz%02dst%02d.dat", source[0], source[1], source[2], source[3]);
    FILE* f = std::fopen((filename_out + suffix).c_str(), "w");
    if (!f) throw PLEGMA_exception("Error opening file for writing");
    const int nmom = corr_mom_space->Nmoms();
    const int lt = localT();
    const size_t site_r = getSiteSize() / (nDatasets() * nGroups());
    auto moms = corr_mom_space->MomList();
    for (int it = 0; it < lt; it++) {
      const int i = ((it - startT()) % totalT + totalT) % totalT;  // buffer slot of source-relative time it
      for (int p = 0; p < nmom; p++) {
        std::fprintf(f, "%d  %+d  %+d  %+d ", it, (int)std::lround(moms[p][0]), (int)std::lround(moms[p][1]),
                     (int)std::lround(moms[p][2]));
        for (size_t d = 0; d < nDatasets(); d++)
          for (size_t g = 0; g < nGroups(); g++)
            for (size_t s = 0; s < site_r; s++) {
              const size_t idx = (((g * nDatasets() + d) * lt + i) * nmom + p) * site_r + s;
              std::fprintf(f, "%+e %+eI ", (double)buf[2 * idx], (double)buf[2 * idx + 1]);
            }
        std::fprintf(f, "\n");
      }
    }
    std::fclose(f);
  }

  // Stand-in for writeHDF5 (lib/PLEGMA_Correlator.cu:892-950): one raw binary
  // file per group/dataset with shape [totalT][Nmom][shape...][2] in
  // source-relative time, plus a JSON sidecar with groups, datasets, shapes,
  // the momentum list ("mvec") and the description.
  void writeBinary(const std::string& filename) const {
    const int nmom = corr_space == MOMENTUM_SPACE ? corr_mom_space->Nmoms() : 0;
    const int lt = localT();
    const size_t site_r = getSiteSize() / (nDatasets() * nGroups());
    const size_t per = (size_t)(corr_space == MOMENTUM_SPACE ? nmom : R().localVolume3D) * site_r;
    std::ostringstream js;
    char top[64];
    std::snprintf(top, sizeof(top), "sx%02dsy%02dsz%02dst%02d", source[0], source[1], source[2], source[3]);
    js << "{\"source\": \"" << top << "\", \"description\": \"" << description << "\", \"shape\": [" << lt;
    js << ", " << (corr_space == MOMENTUM_SPACE ? nmom : (int)R().localVolume3D);
    for (int s : shape) js << ", " << s;
    js << ", 2], \"datasets\": [";
    std::ofstream bin(filename + ".bin", std::ios::binary);
    bool first = true;
    for (size_t g = 0; g < nGroups(); g++)
      for (size_t d = 0; d < nDatasets(); d++) {
        for (int it = 0; it < lt; it++) {
          const int i = ((it - startT()) % totalT + totalT) % totalT;
          const size_t base = ((g * nDatasets() + d) * lt + i) * per;
          bin.write((const char*)&buf[2 * base], (std::streamsize)(2 * per * sizeof(Float)));
        }
        js << (first ? "" : ", ") << "\"" << (groups.empty() ? "" : groups[g]) << "/"
           << (datasets.empty() ? "arr" : datasets[d]) << "\"";
        first = false;
      }
    js << "], \"dtype\": \"" << (sizeof(Float) == 8 ? "float64" : "float32") << "\", \"mvec\": [";
    auto ml = getMomList();
    for (size_t p = 0; p < ml.size(); p++)
      js << (p ? ", " : "") << "[" << ml[p][0] << ", " << ml[p][1] << ", " << ml[p][2] << "]";
    js << "]}";
    std::ofstream(filename + ".json") << js.str();
  }

  void writeFile(const std::string& filename, FILE_FORMAT format) const {
    if (format == ASCII_FORMAT)
      writeASCII(filename);
    else if (format == LIME_FORMAT)
      throw PLEGMA_exception("LIME output is not supported for correlators");
    else
      writeBinary(filename);
  }
};

}  // namespace plegma
