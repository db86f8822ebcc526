// Power-of-two step kernels, float with 8 complex values per thread.
#include "pfc_fast_inst.cuh"

template struct pfc::FastInst<float, 8>;
