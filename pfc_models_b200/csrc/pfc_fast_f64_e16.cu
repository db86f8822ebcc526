// Power-of-two step kernels, double with 16 complex values per thread.
#include "pfc_fast_inst.cuh"

template struct pfc::FastInst<double, 16>;
