// knn_tc.cu - tensor-core exact kNN (tcgen05).  Placeholder until the
// tcgen05 kernel lands: reports the path as unsupported so AUTO selects the
// plain FP32 kernel.
#include "kernels.cuh"

namespace umapb {

bool knn_tc_supported(int d, int k, int metric) {
    (void)d;
    (void)k;
    (void)metric;
    return false;
}

void knn_tc(const float*, int64_t, const float*, int64_t, int, int, int, int32_t*, float*,
            TcKnnStats*, cudaStream_t) {
    invalid("the tensor-core kNN path is not available in this build");
}

}  // namespace umapb
