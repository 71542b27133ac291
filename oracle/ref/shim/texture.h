/* Build shim for compiling the reference (nmrcardoso/sun) with CUDA 12.x.
 *
 * The reference's include/texture.h declares legacy texture references,
 * which CUDA 12 removed.  Only its UseTex == false path is ever run here
 * (PARAMS::UseTex stays false), so every texture fetch is replaced by a stub
 * that is never reached.  This header shadows the reference's texture.h
 * through the include path; the reference sources are compiled unmodified. */
#ifndef TEXTURE_H
#define TEXTURE_H

#include <cuda.h>
#include <complex.h>

namespace CULQCD {
#define SUN_REF_TEX_STUB(NAME) \
    template <class Real> inline __device__ complex NAME(uint) { return complex::zero(); }
SUN_REF_TEX_STUB(TEXTURE_GAUGE)
SUN_REF_TEX_STUB(TEXTURE_GAUGE_CONJ)
SUN_REF_TEX_STUB(TEXTURE_DELTA)
SUN_REF_TEX_STUB(TEXTURE_DELTA_CONJ)
SUN_REF_TEX_STUB(TEXTURE_GX)
SUN_REF_TEX_STUB(TEXTURE_GX_CONJ)
SUN_REF_TEX_STUB(TEXTURE_LAMBDA)
#undef SUN_REF_TEX_STUB
}
#endif
