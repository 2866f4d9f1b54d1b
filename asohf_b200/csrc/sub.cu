// sub.cu -- SUBSTRUCTURE_PARTICLES (substructure.f:756-1697) on sm_100a.
#include "halo_dev.cuh"

extern "C" int asohf_substructure_particles(asohf_ctx* c, const asohf_consts* k, const asohf_mesh* mesh,
                                            asohf_catalogue* cat, int ir, const int32_t* subs_lev,
                                            int on_device) {
  if (!c || !k || !cat || !subs_lev) return ASOHF_ERR_INVALID;
  return ASOHF_ERR_UNSUPPORTED;
}
