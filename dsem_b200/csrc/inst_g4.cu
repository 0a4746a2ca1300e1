// Kernel instantiations for order p = 3 (G = 4 Gauss points per direction).
#include "dsem_inst.cuh"
DSEM_INSTANTIATE(4)
