// Exclusive prefix sums used by compaction and CSR construction: a
// two-level (recursive) block scan, 256 threads x 8 items per block, warp
// shuffles inside a block.
#include "device.cuh"

namespace asdm {

namespace {

constexpr int kThreads = 256;
constexpr int kItems = 8;
constexpr int kTile = kThreads * kItems;

template <typename Tin>
__global__ void __launch_bounds__(kThreads) scan_tiles(const Tin *__restrict__ in, uint64_t *__restrict__ out,
                                                     uint64_t *__restrict__ tile_sums, uint64_t n) {
    __shared__ uint64_t stage[kTile];
    __shared__ uint64_t warp_tot[kThreads / 32];
    const uint64_t base = (uint64_t)blockIdx.x * kTile;
    // coalesced load into shared memory
    for (int i = threadIdx.x; i < kTile; i += kThreads) {
        uint64_t idx = base + i;
        stage[i] = idx < n ? (uint64_t)in[idx] : 0ull;
    }
    __syncthreads();
    uint64_t v[kItems];
    uint64_t tsum = 0;
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        uint64_t t = stage[threadIdx.x * kItems + i];
        v[i] = tsum;
        tsum += t;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t x = tsum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint64_t w = lane < kThreads / 32 ? warp_tot[lane] : 0ull;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint64_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kThreads / 32) warp_tot[lane] = w;
    }
    __syncthreads();
    const uint64_t prefix = (warp > 0 ? warp_tot[warp - 1] : 0ull) + x - tsum;
#pragma unroll
    for (int i = 0; i < kItems; ++i) stage[threadIdx.x * kItems + i] = v[i] + prefix;
    __syncthreads();
    for (int i = threadIdx.x; i < kTile; i += kThreads) {
        uint64_t idx = base + i;
        if (idx < n) out[idx] = stage[i];
    }
    if (threadIdx.x == kThreads - 1) tile_sums[blockIdx.x] = prefix + tsum;
}

__global__ void add_tile_prefix(uint64_t *__restrict__ out, const uint64_t *__restrict__ tile_prefix, uint64_t n) {
    const uint64_t base = (uint64_t)blockIdx.x * kTile;
    const uint64_t add = tile_prefix[blockIdx.x];
    for (int i = threadIdx.x; i < kTile; i += blockDim.x) {
        uint64_t idx = base + i;
        if (idx < n) out[idx] += add;
    }
}

template <typename Tin>
int scan_impl(const Tin *in, uint64_t *out, uint64_t n, bool with_total, cudaStream_t s) {
    if (n == 0) {
        if (with_total) ASDM_CUDA(cudaMemsetAsync(out, 0, sizeof(uint64_t), s));
        return ASDM_OK;
    }
    const uint64_t ntiles = (n + kTile - 1) / kTile;
    uint64_t *sums = nullptr;
    ASDM_TRY(dalloc(&sums, ntiles + 1, s));
    scan_tiles<Tin><<<(unsigned)ntiles, kThreads, 0, s>>>(in, out, sums, n);
    ::asdm::count_launch();
    ASDM_CUDA(cudaGetLastError());
    int rc = ASDM_OK;
    uint64_t *prefix = nullptr;
    if (ntiles == 1) {
        // single tile: its sum is the total
        if (with_total) {
            cudaError_t e = cudaMemcpyAsync(out + n, sums, sizeof(uint64_t), cudaMemcpyDeviceToDevice, s);
            if (e != cudaSuccess) rc = fail(ASDM_ERR_CUDA, "scan total copy: %s", cudaGetErrorString(e));
        }
    } else {
        // exclusive scan of the tile sums, grand total in prefix[ntiles]
        rc = dalloc(&prefix, ntiles + 1, s);
        if (rc == ASDM_OK) rc = scan_impl<uint64_t>(sums, prefix, ntiles, true, s);
        if (rc == ASDM_OK) {
            add_tile_prefix<<<(unsigned)ntiles, kThreads, 0, s>>>(out, prefix, n);
            ::asdm::count_launch();
            if (cudaGetLastError() != cudaSuccess) rc = fail(ASDM_ERR_CUDA, "scan launch failed");
        }
        if (rc == ASDM_OK && with_total) {
            cudaError_t e = cudaMemcpyAsync(out + n, prefix + ntiles, sizeof(uint64_t), cudaMemcpyDeviceToDevice, s);
            if (e != cudaSuccess) rc = fail(ASDM_ERR_CUDA, "scan total copy: %s", cudaGetErrorString(e));
        }
    }
    dfree(prefix, s);
    dfree(sums, s);
    return rc;
}

}  // namespace

int scan_exclusive_u32(const uint32_t *in, uint64_t *out, uint64_t n, bool with_total, cudaStream_t s) {
    return scan_impl<uint32_t>(in, out, n, with_total, s);
}

int scan_exclusive_u64(const uint64_t *in, uint64_t *out, uint64_t n, bool with_total, cudaStream_t s) {
    return scan_impl<uint64_t>(in, out, n, with_total, s);
}

}  // namespace asdm
