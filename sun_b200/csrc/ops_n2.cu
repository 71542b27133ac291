// ops_n2.cu -- kernel instances and launch wrappers for SU(2).
#include "sun_kernels.cuh"
template struct sunb::Ops<2>;
