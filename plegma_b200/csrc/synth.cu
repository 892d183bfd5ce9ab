// Synthetic propagators for benchmarks and tests: Re, Im ~ N(0,1) scaled by
// exp(-a |t - t0|), drawn from a counter-based stream so that any slice can
// be generated independently, on the host or on the device.
//
//   key   = splitmix64(seed ^ splitmix64(0x9E37 + flavour)) + 2 * (site * 144 + comp)
//   u1    = ((splitmix64(key) >> 11) + 1) * 2^-53      in (0, 1]
//   u2    =  (splitmix64(key + 1) >> 11) * 2^-53        in [0, 1)
//   value = sqrt(-2 ln u1) * (cos 2 pi u2, sin 2 pi u2) * exp(-a |t - t0|)
// with `site` the global 4-D site index x + Lx (y + Ly (z + Lz t)).
// Host and device draw identical integers; the transcendental functions are
// the host libm and the CUDA device library respectively (values agree to a
// few ulp, so tests always hand the oracle the exact bytes the GPU used).
#include <cmath>

#include "kernels.cuh"
#include "p2_common.cuh"
#include "synth_host.h"

namespace p2 {

__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__host__ __device__ __forceinline__ uint64_t synth_stream(uint64_t seed, int flavour) {
  return splitmix64(seed ^ splitmix64(0x9E37ull + (uint64_t)flavour));
}

namespace {

__global__ void k_synth(void* dst, int fp32, uint64_t stream, int t0, double decay, int t_first, int nt, int Lx, int Ly,
                        int Lz, int T, int lx, int ly, int lz, int ox, int oy, int oz) {
  const long long V3 = (long long)lx * ly * lz;
  const long long vol = V3 * nt;
  const long long n = vol * 144;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int comp = (int)(i / vol);
    const long long sid = i - comp * vol;
    const int j = (int)(sid / V3);
    const long long x3 = sid - (long long)j * V3;
    const int x = (int)(x3 % lx) + ox, y = (int)((x3 / lx) % ly) + oy, z = (int)(x3 / ((long long)lx * ly)) + oz;
    const int t = (t_first + j) % T;
    const uint64_t site = (uint64_t)x + (uint64_t)Lx * ((uint64_t)y + (uint64_t)Ly * ((uint64_t)z + (uint64_t)Lz * t));
    const uint64_t key = stream + 2ull * (site * 144ull + (uint64_t)comp);
    const double u1 = (double)((splitmix64(key) >> 11) + 1) * 0x1.0p-53;
    const double u2 = (double)(splitmix64(key + 1) >> 11) * 0x1.0p-53;
    const double r = sqrt(-2.0 * log(u1)) * exp(-decay * fabs((double)(t - t0)));
    double sn, cs;
    sincos(2.0 * M_PI * u2, &sn, &cs);
    if (fp32) {
      ((float2*)dst)[i] = make_float2((float)(r * cs), (float)(r * sn));
    } else {
      ((double2*)dst)[i] = make_double2(r * cs, r * sn);
    }
  }
}

}  // namespace

cudaError_t launch_synth(void* dst, int fp32, uint64_t seed, int flavour, int t0, double decay, int t_first, int nt,
                         const int* L, const int* Ll, const int* coords, cudaStream_t s) {
  k_synth<<<148 * 8, 256, 0, s>>>(dst, fp32, synth_stream(seed, flavour), t0, decay, t_first, nt, L[0], L[1], L[2],
                                   L[3], Ll[0], Ll[1], Ll[2], coords[0] * Ll[0], coords[1] * Ll[1], coords[2] * Ll[2]);
  return cudaGetLastError();
}

void synth_host(void* dst, int fp32, uint64_t seed, int flavour, int t0, double decay, int t_first, int nt,
                const int* L, const int* Ll, const int* coords) {
  const uint64_t stream = synth_stream(seed, flavour);
  const long long V3 = (long long)Ll[0] * Ll[1] * Ll[2];
  const long long vol = V3 * nt;
#pragma omp parallel for collapse(2) schedule(static)
  for (int comp = 0; comp < 144; comp++)
    for (long long sid = 0; sid < vol; sid++) {
      const long long i = (long long)comp * vol + sid;
      const int j = (int)(sid / V3);
      const long long x3 = sid - (long long)j * V3;
      const int x = (int)(x3 % Ll[0]) + coords[0] * Ll[0];
      const int y = (int)((x3 / Ll[0]) % Ll[1]) + coords[1] * Ll[1];
      const int z = (int)(x3 / ((long long)Ll[0] * Ll[1])) + coords[2] * Ll[2];
      const int t = (t_first + j) % L[3];
      const uint64_t site =
          (uint64_t)x + (uint64_t)L[0] * ((uint64_t)y + (uint64_t)L[1] * ((uint64_t)z + (uint64_t)L[2] * t));
      const uint64_t key = stream + 2ull * (site * 144ull + (uint64_t)comp);
      const double u1 = (double)((splitmix64(key) >> 11) + 1) * 0x1.0p-53;
      const double u2 = (double)(splitmix64(key + 1) >> 11) * 0x1.0p-53;
      const double r = std::sqrt(-2.0 * std::log(u1)) * std::exp(-decay * std::fabs((double)(t - t0)));
      const double ph = 2.0 * M_PI * u2;
      if (fp32) {
        ((float*)dst)[2 * i] = (float)(r * std::cos(ph));
        ((float*)dst)[2 * i + 1] = (float)(r * std::sin(ph));
      } else {
        ((double*)dst)[2 * i] = r * std::cos(ph);
        ((double*)dst)[2 * i + 1] = r * std::sin(ph);
      }
    }
}

}  // namespace p2
