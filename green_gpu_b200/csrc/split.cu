// Split-precision contraction engine (placeholder until the tcgen05 INT8 path lands).
#include "split.cuh"

namespace gg {

SplitGemm* split_engine(gg_context*) {
  throw Error(GG_ERR_ARG, "split precision (GG_PREC_SPLIT) is not available in this build");
}

int split_zgemm(SplitGemm*, const ZgemmDesc&, int, cudaStream_t) {
  throw Error(GG_ERR_ARG, "split precision (GG_PREC_SPLIT) is not available in this build");
}

}  // namespace gg
