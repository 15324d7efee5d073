// pd_fast.cu -- throughput modes (PD_PREC_FP64, PD_PREC_FP32C).
#include "pd_env_impl.h"

namespace pd {

pd_status sync_state_to_fp64(pd_env *env) {
    (void)env;
    return PD_OK;
}

void fast_release(pd_env *env) { (void)env; }

pd_status fast_vv_steps(pd_env *env, int64_t nsteps) {
    (void)env;
    (void)nsteps;
    return fail(PD_ERR_UNSUPPORTED, "throughput modes are not built yet");
}

}  // namespace pd
