// Instantiates the k-clique tier kernels for k = 3: counts, accounting, edge triangles and diamond pairs (see clique_tiers.cuh).
#include "clique_tiers.cuh"

namespace jgpm {

int launch_tiers_k3(int mode, const CliqueArgs& a, const TierPlan& p, int sms, cudaStream_t s,
                    int max_out) {
  switch (mode) {
    case 1: return launch_plan_k<3, true, false>(a, p, sms, s, max_out);
    case 2: return launch_plan_k<3, false, true>(a, p, sms, s, max_out);
    case 3: return launch_plan_k<3, false, true, true>(a, p, sms, s, max_out);
    default: return launch_plan_k<3, false, false>(a, p, sms, s, max_out);
  }
}

}  // namespace jgpm
