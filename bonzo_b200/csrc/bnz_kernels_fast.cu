// Fast build: compiled with --fmad=true (multiply-adds contract into DFMA).
#define BNZ_NS fast
#include "bnz_kernels_impl.cuh"
BNZ_DEFINE_TABLE(fast)
