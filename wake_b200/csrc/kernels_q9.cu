// Kernels of the D2Q9 lattice (instantiated from kernels_impl.cuh).
#define WK_Q 9
#include "kernels_impl.cuh"
