// Kernel instantiations for order p = 2 (G = 3 Gauss points per direction).
#include "dsem_inst.cuh"
DSEM_INSTANTIATE(3)
