// MTTKRP kernels instantiated for rank R = 256 (FP32 and BF16 factors).
#include "mttkrp_kernels.cuh"

MMCSF_INSTANTIATE_R(256)
