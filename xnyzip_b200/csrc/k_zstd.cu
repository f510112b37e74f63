// zstd frames decoded on the GPU, one frame per warp (zstd_dec.cuh), for callers that hold
// many container frames in device memory: no host round trip.
#include "kernels.h"
#include "zstd_dec.cuh"

namespace xnyz {
namespace dev {

namespace {

// One frame per warp: the lanes decode it together (zd::WarpTeam).
__global__ void __launch_bounds__(128) zstd_frames_kernel(const uint8_t* const* src, const uint64_t* src_len,
                                                          uint8_t* const* dst, const uint64_t* cap, long long* out_len,
                                                          zd::Workspace* ws, uint64_t count) {
    const uint64_t f = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (f >= count) return;  // the same for every lane of the warp
    const zd::WarpTeam team{(int)(threadIdx.x & 31)};
    const long long r = zd::decode_frame(src[f], src_len[f], dst[f], cap[f], ws[f], team);
    if (team.rank == 0) out_len[f] = r;
}

}  // namespace

size_t zstd_workspace_bytes() { return sizeof(zd::Workspace); }

void launch_zstd_frames(const uint8_t* const* src, const uint64_t* src_len, uint8_t* const* dst, const uint64_t* cap,
                        long long* out_len, void* workspace, uint64_t count, cudaStream_t st) {
    if (!count) return;
    const unsigned blocks = (unsigned)((count + 3) / 4);  // four frames (warps) per block
    zstd_frames_kernel<<<blocks, 128, 0, st>>>(src, src_len, dst, cap, out_len,
                                              static_cast<zd::Workspace*>(workspace), count);
}

}  // namespace dev
}  // namespace xnyz
