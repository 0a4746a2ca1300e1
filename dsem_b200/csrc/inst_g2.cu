// Kernel instantiations for order p = 1 (G = 2 Gauss points per direction).
#include "dsem_inst.cuh"
DSEM_INSTANTIATE(2)
