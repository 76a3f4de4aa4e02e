// Batched decomposition of many graphs.
#include "device.h"

namespace fc {

// One graph after another through the single-graph path (plain launches):
// the baseline the persistent batched kernel is measured against.
static fc_status batch_plain(fc_graph* const* gs, uint32_t count, double beta,
                             uint32_t* const* tables, fc_densest_result* res, cudaStream_t s) {
    for (uint32_t i = 0; i < count; i++) {
        fc_graph* g = gs[i];
        if (!g) return FC_ERR_INVALID;
        FC_TRY(coreindex(g, tables ? tables[i] : nullptr, false, s));
        if (res) {
            if (g->n && g->L) {
                FC_TRY(densest(g, &beta, 1, res + i, s));
            } else {
                res[i] = fc_densest_result{};
                res[i].beta = beta;
            }
        }
    }
    return FC_OK;
}

fc_status batch_run(fc_graph* const* gs, uint32_t count, double beta, uint32_t* const* tables,
                    fc_densest_result* res, const fc_batch_options* opt, cudaStream_t s) {
    (void)opt;
    if (!cuda_available()) return FC_ERR_NO_DEVICE;
    return batch_plain(gs, count, beta, tables, res, s);
}

}  // namespace fc
