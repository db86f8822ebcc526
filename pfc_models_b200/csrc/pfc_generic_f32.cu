// Mixed-radix kernels in float.
#include "pfc_generic_inst.cuh"

template struct pfc::GenericInst<float>;
