// Kernel instantiations for order p = 6 (G = 7 Gauss points per direction).
#include "dsem_inst.cuh"
DSEM_INSTANTIATE(7)
