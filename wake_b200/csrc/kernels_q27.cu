// Kernels of the D3Q27 lattice (instantiated from kernels_impl.cuh).
#define WK_Q 27
#include "kernels_impl.cuh"
