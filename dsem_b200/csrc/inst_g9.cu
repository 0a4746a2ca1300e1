// Kernel instantiations for order p = 8 (G = 9 Gauss points per direction).
#include "dsem_inst.cuh"
DSEM_INSTANTIATE(9)
#ifdef DSEM_PHASE_TIMING
extern "C" int dsem_debug_phase_cycles(unsigned long long *out, int reset) {
  cudaError_t e = cudaMemcpyFromSymbol(out, ::g_phase_cycles, sizeof(unsigned long long) * 32);
  if (reset) {
    unsigned long long z[32] = {};
    cudaMemcpyToSymbol(::g_phase_cycles, z, sizeof(z));
  }
  return (int)e;
}
#endif
