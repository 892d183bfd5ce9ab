// Stand-in for the reference's complex-number header when its gamma tables
// (lib/kernels/PLEGMA_gammas.cuh) are compiled as host C++: the complex pair
// comes from the kernel-utility stand-in.
#pragma once
#include "PLEGMA_kernel_utils.cuh"
