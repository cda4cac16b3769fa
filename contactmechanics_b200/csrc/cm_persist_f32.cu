// FP32 instantiations of the persistent cooperative CCG kernel (cm_persist.cuh).
#include "cm_persist.cuh"

template const void* persist_kernel<float>(int);
