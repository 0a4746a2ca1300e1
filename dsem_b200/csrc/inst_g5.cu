// Kernel instantiations for order p = 4 (G = 5 Gauss points per direction).
#include "dsem_inst.cuh"
DSEM_INSTANTIATE(5)
