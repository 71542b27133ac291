/* Injected-uniform shim for compiling the reference's per-link update
 * functions (include/device_PHB_OVR.h: heatBathSUN, overrelaxationSUN) in
 * ref_link_probe.cu only.  It shadows the reference's random.h there so that
 * cuRNGState is a cursor into a caller buffer of uniforms instead of a cuRAND
 * state; Random<Real>() returns the next buffered value.  The reference
 * sources themselves are compiled unmodified. */
#ifndef RANDOM_GPU_H
#define RANDOM_GPU_H

#include <alloc.h>
#include <comm_mpi.h>
#include <cuda_runtime.h>

namespace CULQCD {
struct cuRNGState {
    const double* u;
    int pos, len;
    int* overrun;
};
template <class Real> __device__ inline Real Random(cuRNGState& s)
{
    if (s.pos >= s.len) {
        atomicOr(s.overrun, 1);
        return (Real)0.5;
    }
    return (Real)s.u[s.pos++];
}
// named (not called) by randomSU2 (device_PHB_OVR.h:633), which the probe
// never instantiates
__device__ inline unsigned int curand(cuRNGState*) { return 0u; }
template <class Real> __device__ inline Real Random(cuRNGState* s, Real a, Real b)
{
    return a + (b - a) * Random<Real>(*s);
}
}  // namespace CULQCD
#endif
