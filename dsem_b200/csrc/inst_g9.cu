// Kernel instantiations for order p = 8 (G = 9 Gauss points per direction).
#include "dsem_inst.cuh"
DSEM_INSTANTIATE(9)
