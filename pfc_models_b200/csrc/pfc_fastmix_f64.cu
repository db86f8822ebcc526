// Register-resident step kernels for N = ODD * 2^k transforms, double.
#include "pfc_fastmix_inst.cuh"

template struct pfc::MixInst<double>;
