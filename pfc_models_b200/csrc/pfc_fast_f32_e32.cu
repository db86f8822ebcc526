// Power-of-two step kernels, float with 32 complex values per thread.
#include "pfc_fast_inst.cuh"

template struct pfc::FastInst<float, 32>;
