// bdc_factored.cu -- placeholder until the factored engine lands.
#include "bdc_engine.cuh"

namespace bdc {
bool factored_supports(int, int) { return false; }
bdc_status factored_init(bdc_handle*) { return fail(BDC_ERR_UNSUPPORTED, "factored engine not built"); }
void factored_free(bdc_handle*) {}
bdc_status factored_load_p(bdc_handle*) { return BDC_ERR_UNSUPPORTED; }
bdc_status factored_store_p(bdc_handle*, double*) { return BDC_ERR_UNSUPPORTED; }
bdc_status factored_iterate(bdc_handle*, int64_t, double, bdc_stats*) { return BDC_ERR_UNSUPPORTED; }
bdc_status factored_profile(bdc_handle*, int, bdc_profile_t*) { return BDC_ERR_UNSUPPORTED; }
}  // namespace bdc
