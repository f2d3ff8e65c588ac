// Split-precision (BF16x3) tensor-core path: placeholder until the tcgen05
// kernels land; operators with HB_PREC_BF16X3 report HB_ERR_UNSUPPORTED.
#include "common.cuh"

namespace hb {

hb_status prepare_split(Op* op) {
  (void)op;
  return fail(HB_ERR_UNSUPPORTED, "BF16x3 path not built");
}

hb_status launch_split(Op*, int, double, double, double, const void*, void*, void*,
                       const double*, const double*, const double*, cudaStream_t) {
  return fail(HB_ERR_UNSUPPORTED, "BF16x3 path not built");
}

void free_split(Op* op) { (void)op; }

}  // namespace hb
