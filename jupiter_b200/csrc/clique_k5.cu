// Instantiates the k-clique tier kernels for k = 5: counts and accounting (see clique_tiers.cuh).
#include "clique_tiers.cuh"

namespace jgpm {

int launch_tiers_k5(int mode, const CliqueArgs& a, const TierPlan& p, int sms, cudaStream_t s,
                    int max_out) {
  return mode == 1 ? launch_plan_k<5, true, false>(a, p, sms, s, max_out)
                   : launch_plan_k<5, false, false>(a, p, sms, s, max_out);
}

}  // namespace jgpm
