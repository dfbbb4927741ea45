// lbx_particles.cu — rigid-sphere part of the hot path (placeholder until the
// particle kernels land): a context with max_particles > 0 is refused.
#include "lbx_ctx.h"

namespace lbx {
struct ParticleState {};
int particles_create(Ctx&) { return LBX_ERR_STATE; }
void particles_destroy(Ctx& c) { delete c.part; c.part = nullptr; }
int particles_step_pre(Ctx&) { return 0; }
int particles_step_post(Ctx&) { return 0; }
}  // namespace lbx
