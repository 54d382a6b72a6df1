// Instantiation of the state FFT kernels for grid sizes 32 40 42.
#include "statefft_impl.cuh"
CPSTEP_INSTANTIATE_STATEFFT(32)
CPSTEP_INSTANTIATE_STATEFFT(40)
CPSTEP_INSTANTIATE_STATEFFT(42)
