// Precision form: fused k<=5 unitaries applied as BF16x3 tensor-core GEMMs.
#include "engine.cuh"

using namespace ncsim;

extern "C" ncsim_status ncsim_sv_run_fused(ncsim_state* s, const ncsim_circuit* c, ncsim_rng* rng, uint32_t max_fuse,
                                           uint8_t* rec, size_t cap, size_t* len, ncsim_fused_stats* stats) {
  (void)s, (void)c, (void)rng, (void)max_fuse, (void)rec, (void)cap, (void)len, (void)stats;
  return guarded([&] { throw Error(NCSIM_ERR_UNSUPPORTED, "the fused precision form is not built yet"); });
}
