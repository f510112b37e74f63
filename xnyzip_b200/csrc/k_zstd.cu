// zstd frames decoded on the GPU, one frame per thread (zstd_dec.cuh), for callers that hold
// many container frames in device memory (the per-chunk workloads): no host round trip.
#include "kernels.h"
#include "zstd_dec.cuh"

namespace xnyz {
namespace dev {

namespace {

__global__ void __launch_bounds__(64) zstd_frames_kernel(const uint8_t* const* src, const uint64_t* src_len,
                                                         uint8_t* const* dst, const uint64_t* cap, long long* out_len,
                                                         zd::Workspace* ws, uint64_t count) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    out_len[i] = zd::decode_frame(src[i], src_len[i], dst[i], cap[i], ws[i]);
}

}  // namespace

size_t zstd_workspace_bytes() { return sizeof(zd::Workspace); }

void launch_zstd_frames(const uint8_t* const* src, const uint64_t* src_len, uint8_t* const* dst, const uint64_t* cap,
                        long long* out_len, void* workspace, uint64_t count, cudaStream_t st) {
    if (!count) return;
    const unsigned blocks = (unsigned)((count + 63) / 64);
    zstd_frames_kernel<<<blocks, 64, 0, st>>>(src, src_len, dst, cap, out_len,
                                              static_cast<zd::Workspace*>(workspace), count);
}

}  // namespace dev
}  // namespace xnyz
