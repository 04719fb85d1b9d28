// Exact build: compiled with --fmad=false, so every multiply and add rounds
// separately as in the CPU reference (bit-for-bit parity mode).
#define BNZ_NS exact
#define BNZ_FAST_MATH 0
#include "bnz_kernels_impl.cuh"
BNZ_DEFINE_TABLE(exact)
