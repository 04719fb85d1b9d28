// Fast build: compiled with --fmad=true (multiply-adds contract into DFMA).
#define BNZ_NS fast
// algebraically equal rewrites with fewer FP64 divisions and square roots
// (bnz_device.cuh, bnz_fused.cuh); the exact build keeps the reference's forms
#define BNZ_FAST_MATH 1
#include "bnz_kernels_impl.cuh"
BNZ_DEFINE_TABLE(fast)
