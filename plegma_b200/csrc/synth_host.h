// Host half of the synthetic propagator generator (synth.cu).
#pragma once
#include <stdint.h>

namespace p2 {
void synth_host(void* dst, int fp32, uint64_t seed, int flavour, int t0, double decay, int t_first, int nt,
                const int* L, const int* Ll, const int* coords);
}
