// Instantiation of the state FFT kernels for grid sizes 198 200.
#include "statefft_impl.cuh"
CPSTEP_INSTANTIATE_STATEFFT(198)
CPSTEP_INSTANTIATE_STATEFFT(200)
