// Entry points whose kernels are not built yet report GB_ERR_UNSUPPORTED.
#include "device_graph.cuh"

extern "C" {

int gb_autotune(gb_graph*, const char*, uint32_t, const char*, gb_tuning*, void*) {
  GB_FAIL(GB_ERR_UNSUPPORTED, "gb_autotune: not built");
}

}  // extern "C"
