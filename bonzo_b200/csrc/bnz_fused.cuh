// bnz_fused.cuh -- fused tile kernels (filled in below).
#pragma once
namespace fused {}
