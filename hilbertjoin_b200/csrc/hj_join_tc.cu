// hj_join_tc.cu -- tensor-core forms (placeholder until the tcgen05 kernel lands).
#include "hj_common.cuh"
#include "hj_internal.h"
#include "../../include/hj.h"

namespace hj {

void tc_band_constants(int form, uint32_t d, double maxabs, double *c_rel, double *c_abs) {
    (void)form; (void)d; (void)maxabs;
    *c_rel = 0;
    *c_abs = 0;
}

int launch_join_tc(const SortedSet &, const SortedSet &, bool, uint64_t, uint64_t, const TcParams &,
                   const IndexResult &, unsigned long long *, uint2 *, uint64_t, unsigned long long *, uint32_t *,
                   int, cudaStream_t, std::string *err) {
    *err = "tensor-core form not built";
    return 1;
}

void launch_recheck(const SortedSet &, const SortedSet &, double, const uint2 *, const unsigned long long *,
                    uint64_t, unsigned long long *, cudaStream_t) {}

}  // namespace hj
