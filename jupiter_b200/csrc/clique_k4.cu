// Instantiates the k-clique tier kernels for k = 4: counts, accounting and the vertex-induced tailed triangle (see clique_tiers.cuh).
#include "clique_tiers.cuh"

namespace jgpm {

int launch_tiers_k4(int mode, const CliqueArgs& a, const TierPlan& p, int sms, cudaStream_t s,
                    int max_out) {
  if (mode == 4) return launch_plan_k<4, false, true, true, true>(a, p, sms, s, max_out);
  return mode == 1 ? launch_plan_k<4, true, false>(a, p, sms, s, max_out)
                   : launch_plan_k<4, false, false>(a, p, sms, s, max_out);
}

}  // namespace jgpm
