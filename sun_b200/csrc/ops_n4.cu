// ops_n4.cu -- kernel instances and launch wrappers for SU(4).
#include "sun_kernels.cuh"
template struct sunb::Ops<4>;
