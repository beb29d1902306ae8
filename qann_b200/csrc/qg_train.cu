// IVFIndex::train on the GPU (filled in below).
#include "qg_device.cuh"
#include "qg_ops.h"

namespace qg {

void train(IVFObj& o, const float* x, size_t n, size_t max_iters, int64_t seed, int clustering, size_t passes,
           cudaStream_t st) {
    (void)o; (void)x; (void)n; (void)max_iters; (void)seed; (void)clustering; (void)passes; (void)st;
    throw Error(kUnsupported, "train() is not available in this build");
}

} // namespace qg
