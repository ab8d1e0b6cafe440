// Kernels of the D3Q19 lattice (instantiated from kernels_impl.cuh).
#define WK_Q 19
#include "kernels_impl.cuh"
