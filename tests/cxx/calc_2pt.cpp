// A caller of the drop-in C++ surface, written the way the reference's
// production driver (plegma/Calc_2pt.cpp:73-131) uses PLEGMA_Correlator:
// two propagators, a momentum-space correlator per source, contractMesons*,
// contractBaryons, contractBaryonsUDSC, writeFile, and the propagator
// pre-processing (absorb, rotateToPhysicalBase_device, applyBoundaries_device,
// apply_gamma5).  The GPU tests compare what it writes with the C ABI
// results and the oracle.
//
//   calc_2pt Lx Ly Lz Lt sx sy sz st totalT q2max mode out_prefix
#include <cstdio>
#include <cstdlib>
#include <string>

#include "plegma/PLEGMA_2pt.h"

using namespace plegma;

int main(int argc, char** argv) {
  if (argc != 13) {
    std::fprintf(stderr, "usage: calc_2pt Lx Ly Lz Lt sx sy sz st totalT q2max mode out_prefix\n");
    return 2;
  }
  const std::array<int, 4> L{{std::atoi(argv[1]), std::atoi(argv[2]), std::atoi(argv[3]), std::atoi(argv[4])}};
  const site src(std::atoi(argv[5]), std::atoi(argv[6]), std::atoi(argv[7]), std::atoi(argv[8]));
  const int totalT = std::atoi(argv[9]), q2max = std::atoi(argv[10]);
  const CONTRACTION_MODE mode = std::atoi(argv[11]) ? SPLIT_FP16 : PLAIN_FP64;
  const std::string out = argv[12];
  try {
    PLEGMA_init(L);
    PLEGMA_Propagator<double> up(BOTH), dn(DEVICE);
    up.fillSynthetic(2024, 0, src[3], 0.5);
    dn.fillSynthetic(2024, 1, src[3], 0.5);

    PLEGMA_Correlator<double> mes(MOMENTUM_SPACE, src, q2max, totalT);
    mes.setMode(mode);
    mes.contractMesonsAll(up, dn);
    mes.writeFile(out + "_mesons_all", DEFAULT_FORMAT);
    mes.writeFile(out + "_mesons_all", ASCII_FORMAT);

    // one fixed momentum (the reference's setFixMomVec), nucleon
    PLEGMA_Correlator<double> fix(MOMENTUM_SPACE, src, q2max, totalT);
    std::vector<int> pfix{1, 0, -1};
    fix.setFixMomVec(pfix);
    fix.setMode(mode);
    fix.contractBaryons(up, dn, false);
    fix.writeFile(out + "_baryons_fixmom", DEFAULT_FORMAT);

    PLEGMA_Correlator<double> m10(MOMENTUM_SPACE, src, q2max, totalT);
    m10.setMode(mode);
    m10.contractMesons(up, dn);
    m10.writeFile(out + "_mesons10", DEFAULT_FORMAT);

    PLEGMA_Correlator<double> bar(MOMENTUM_SPACE, src, q2max, totalT);
    bar.setMode(mode);
    bar.contractBaryons(up, dn);
    bar.writeFile(out + "_baryons", DEFAULT_FORMAT);

    PLEGMA_Correlator<double> udsc(MOMENTUM_SPACE, src, q2max, totalT);
    PLEGMA_Propagator<double> st(NONE), ch(NONE);
    udsc.contractBaryonsUDSC(up, dn, st, ch);
    udsc.writeFile(out + "_udsc", DEFAULT_FORMAT);

    PLEGMA_Correlator<double> pos(POSITION_SPACE, src, 0, totalT);
    pos.contractBaryons(up, dn);
    pos.writeFile(out + "_baryons_pos", DEFAULT_FORMAT);

    // generic transform of the up propagator as a 144-component field
    PLEGMA_FT<double> ft(q2max);
    ft.apply(up, FT_GEMV, -1);
    FILE* f = std::fopen((out + "_ft_up.bin").c_str(), "wb");
    std::fwrite(ft.H_elem(), sizeof(double), (size_t)2 * ft.Nmoms() * ft.DimT() * 144, f);
    std::fclose(f);
    ft.apply(up, FT_SPLIT, -1);  // the same transform on the tensor cores
    f = std::fopen((out + "_ft_up_split.bin").c_str(), "wb");
    std::fwrite(ft.H_elem(), sizeof(double), (size_t)2 * ft.Nmoms() * ft.DimT() * 144, f);
    std::fclose(f);

    up.copyToHost();
    f = std::fopen((out + "_up.bin").c_str(), "wb");
    std::fwrite(up.H_elem(), sizeof(double), (size_t)2 * 144 * up.Total_length(), f);
    std::fclose(f);

    // pre-processing: in place (rotation +1, boundary at the source, g5) and
    // applied on load; the nucleon from both must agree
    PLEGMA_Propagator<double> rot(BOTH), lazy(DEVICE);
    rot.fillSynthetic(2024, 0, src[3], 0.5);
    lazy.fillSynthetic(2024, 0, src[3], 0.5);
    rot.rotateToPhysicalBase_device(+1);
    rot.applyBoundaries_device(src[3]);
    lazy.transformOnLoad(P2_PROP_ROTATE_PLUS | P2_PROP_BOUNDARY, src[3]);
    PLEGMA_Correlator<double> br(MOMENTUM_SPACE, src, q2max, totalT), bl(MOMENTUM_SPACE, src, q2max, totalT);
    br.setMode(mode);
    bl.setMode(mode);
    br.contractBaryons(rot, dn);
    bl.contractBaryons(lazy, dn);
    br.writeFile(out + "_baryons_rot", DEFAULT_FORMAT);
    bl.writeFile(out + "_baryons_lazy", DEFAULT_FORMAT);
    rot.apply_gamma5();
    rot.copyToHost();
    f = std::fopen((out + "_rot.bin").c_str(), "wb");
    std::fwrite(rot.H_elem(), sizeof(double), (size_t)2 * 144 * rot.Total_length(), f);
    std::fclose(f);

    // a propagator built from twelve spinor fields (absorb), and one slice of
    // another from a 3-D field; deterministic, exactly representable entries
    PLEGMA_Propagator<double> built(BOTH), sliced(BOTH);
    PLEGMA_Vector<double> vec(BOTH);
    PLEGMA_Vector3D<double> vec3(BOTH);
    for (int k = 0; k < 12; k++) {
      for (size_t i = 0; i < 12 * vec.Total_length(); i++) {
        vec.H_elem()[2 * i] = (double)((i * 7 + k * 13) % 101) / 16.0 - 3.0;
        vec.H_elem()[2 * i + 1] = (double)((i * 5 + k * 3) % 67) / 8.0;
      }
      vec.copyToDevice();
      built.absorb(vec, k / 3, k % 3);
    }
    for (size_t i = 0; i < 12 * vec3.Total_length(); i++) {
      vec3.H_elem()[2 * i] = (double)(i % 29) - 14.0;
      vec3.H_elem()[2 * i + 1] = (double)(i % 13) / 4.0;
    }
    vec3.copyToDevice();
    sliced.fillSynthetic(5, 0, 0, 0.5);
    sliced.absorb(vec3, src[3], 1, 2);
    built.copyToHost();
    sliced.copyToHost();
    f = std::fopen((out + "_absorb.bin").c_str(), "wb");
    std::fwrite(built.H_elem(), sizeof(double), (size_t)2 * 144 * built.Total_length(), f);
    std::fwrite(sliced.H_elem(), sizeof(double), (size_t)2 * 144 * sliced.Total_length(), f);
    std::fclose(f);
    PLEGMA_finalize();
  } catch (const PLEGMA_exception& e) {
    std::fprintf(stderr, "calc_2pt: %s\n", e.what());
    return 1;
  }
  return 0;
}
