// Fused two-pass RK3 stage (x pass + y pass); filled in below the operator
// path.
#include "common.cuh"

namespace mhd {
int fused_setup(Ctx *c) { (void)c; return MHDGPU_OK; }
void fused_free(Ctx *c) { (void)c; }
int fused_stage(Ctx *c, int iRK, int first, int last)
{
    (void)c; (void)iRK; (void)first; (void)last;
    return mhd_set_error(MHDGPU_ERR_UNSUPPORTED);
}
}  // namespace mhd

extern "C" int mhdgpu_steps_fused(mhdgpu_ctx *h, int nsteps, double dt_fixed, double *dt_io)
{
    (void)h; (void)nsteps; (void)dt_fixed; (void)dt_io;
    return mhd_set_error(MHDGPU_ERR_UNSUPPORTED);
}
