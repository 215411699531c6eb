// Instantiates the k-clique tier kernels for k = 7 and 8: counts and accounting (see clique_tiers.cuh).
#include "clique_tiers.cuh"

namespace jgpm {

int launch_tiers_k78(int k, int mode, const CliqueArgs& a, const TierPlan& p, int sms,
                     cudaStream_t s, int max_out) {
  if (k == 7)
    return mode == 1 ? launch_plan_k<7, true, false>(a, p, sms, s, max_out)
                     : launch_plan_k<7, false, false>(a, p, sms, s, max_out);
  return mode == 1 ? launch_plan_k<8, true, false>(a, p, sms, s, max_out)
                   : launch_plan_k<8, false, false>(a, p, sms, s, max_out);
}

}  // namespace jgpm
