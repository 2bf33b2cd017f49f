// Entry points whose kernels are not built yet report GB_ERR_UNSUPPORTED.
#include "device_graph.cuh"

extern "C" {

int gb_ppr_forward(gb_graph*, uint32_t, const float*, float, float, uint32_t, float*, uint32_t*, gb_stats*,
                   void*) {
  GB_FAIL(GB_ERR_UNSUPPORTED, "gb_ppr_forward: not built");
}
int gb_ppr_backward(gb_graph*, uint32_t, const float*, const float*, float, float, uint32_t, float*, float*,
                    uint32_t*, gb_stats*, void*) {
  GB_FAIL(GB_ERR_UNSUPPORTED, "gb_ppr_backward: not built");
}
int gb_autotune(gb_graph*, const char*, uint32_t, const char*, gb_tuning*, void*) {
  GB_FAIL(GB_ERR_UNSUPPORTED, "gb_autotune: not built");
}

}  // extern "C"
