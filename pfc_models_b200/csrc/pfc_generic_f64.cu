// Mixed-radix kernels in double.
#include "pfc_generic_inst.cuh"

template struct pfc::GenericInst<double>;
