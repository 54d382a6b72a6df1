// Instantiation of the state FFT kernels for grid sizes 48 60 64.
#include "statefft_impl.cuh"
CPSTEP_INSTANTIATE_STATEFFT(48)
CPSTEP_INSTANTIATE_STATEFFT(60)
CPSTEP_INSTANTIATE_STATEFFT(64)
