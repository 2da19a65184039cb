// tb_tensor.cu -- placeholder until the moment-tensor layout lands.
#include "tb_tensor.cuh"

namespace tb {
void MomentTensor::release() {
    if (d) cudaFree(d);
    d = nullptr;
}
int64_t tensor_bytes(int L, bool fp32, int64_t n) { return INT64_MAX; }
int build_tensor(const ChanDev&, const int32_t*, int64_t, int64_t, bool, MomentTensor&, cudaStream_t) {
    set_error("moment tensor layout not available");
    return TB_ERR_ARG;
}
int launch_collision_tensor(const ChanDev&, double, const MomentTensor&, const int32_t*, int64_t, int64_t,
                            const double*, double*, const int*, cudaStream_t) {
    set_error("moment tensor layout not available");
    return TB_ERR_ARG;
}
}  // namespace tb
