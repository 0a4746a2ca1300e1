// Kernel instantiations for order p = 7 (G = 8 Gauss points per direction).
#include "dsem_inst.cuh"
DSEM_INSTANTIATE(8)
