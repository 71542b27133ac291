// Build shim: no-op texture binding for the reference build (see
// shim/texture.h).  Declarations come from the reference's texture_host.h.
#include <texture_host.h>

namespace CULQCD {
#define SUN_REF_BIND_STUB(NAME)         \
    void NAME(complexs*, bool) {}       \
    void NAME(complexd*, bool) {}
#define SUN_REF_BIND1_STUB(NAME)        \
    void NAME(complexs*) {}             \
    void NAME(complexd*) {}
SUN_REF_BIND_STUB(GAUGE_TEXTURE)
SUN_REF_BIND_STUB(DELTA_TEXTURE)
SUN_REF_BIND_STUB(GX_TEXTURE)
SUN_REF_BIND_STUB(ILAMBDA_TEXTURE)
SUN_REF_BIND1_STUB(BIND_GAUGE_TEXTURE)
SUN_REF_BIND1_STUB(BIND_DELTA_TEXTURE)
SUN_REF_BIND1_STUB(BIND_GX_TEXTURE)
SUN_REF_BIND1_STUB(BIND_ILAMBDA_TEXTURE)
void UNBIND_ALL_TEXTURES() {}
}
