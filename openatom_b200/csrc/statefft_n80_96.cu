// Instantiation of the state FFT kernels for grid sizes 80 96.
#include "statefft_impl.cuh"
CPSTEP_INSTANTIATE_STATEFFT(80)
CPSTEP_INSTANTIATE_STATEFFT(96)
