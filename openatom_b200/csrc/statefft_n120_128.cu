// Instantiation of the state FFT kernels for grid sizes 120 128.
#include "statefft_impl.cuh"
CPSTEP_INSTANTIATE_STATEFFT(120)
CPSTEP_INSTANTIATE_STATEFFT(128)
