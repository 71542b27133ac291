// ops_n6.cu -- kernel instances and launch wrappers for SU(6).
#include "sun_kernels.cuh"
template struct sunb::Ops<6>;
