// Kernel instantiations for order p = 5 (G = 6 Gauss points per direction).
#include "dsem_inst.cuh"
DSEM_INSTANTIATE(6)
