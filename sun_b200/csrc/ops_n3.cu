// ops_n3.cu -- kernel instances and launch wrappers for SU(3).
#include "sun_kernels.cuh"
template struct sunb::Ops<3>;
