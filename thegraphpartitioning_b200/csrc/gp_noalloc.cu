// gp_noalloc.cu -- edge cut and part weights without any allocation.
//
// gp_edge_cut_device() takes its scratch (the cut accumulator, the k part
// weight accumulators and a validation word) from the library's device
// workspace, which grows with cudaMalloc on first use.  Some callers cannot
// allow that: code inside a custom allocator or memory-pool callback (an
// allocation would re-enter the allocator), real-time loops that forbid
// allocation after start-up (an allocation can block or fail mid-loop), and
// hosts whose device memory is fully reserved by another framework.  gp_edge_cut_device_noalloc() is the
// same computation with its scratch in a fixed file-scope __device__ array.
//
// Limits and behaviour:
// * at most GP_NOALLOC_MAX_K parts (the scratch holds 1 + GP_NOALLOC_MAX_K
//   int64 accumulators and one validation word, about 8 KB per device);
//   larger k returns GP_EINVAL;
// * every call on a device shares that one array; calls whose work overlaps
//   on the GPU (different streams, or several host threads) race and give
//   wrong results -- serialize them;
// * every call looks up the array's device address (cudaGetSymbolAddress:
//   no allocation, no stream work), so a device reset or another context
//   never leaves a stale address behind;
// * no cudaMalloc, cudaFree, cudaMallocHost or other allocating routine is
//   called; results are copied into the caller's host memory.
#define GP_TU_ID 6   // site ids of the bounds-checked build
#include "gp_internal.cuh"


namespace gp {

// [0] directed cross weight, [1 .. k] part weights, [1 + GP_NOALLOC_MAX_K] error word
constexpr int kNoAllocWords = 2 + GP_NOALLOC_MAX_K;
static __device__ __align__(256) unsigned long long g_noalloc_scratch[kNoAllocWords];

__global__ void k_na_check(int64_t n, const int32_t* __restrict__ part, int32_t k,
                           unsigned long long* __restrict__ err) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const int32_t p = part[v];
        if (p < 0 || p >= k) atomicMin(err, (unsigned long long)v);
    }
}

// warp per row: directed cross weight; vertex weights into the part accumulators
__global__ void __launch_bounds__(256) k_na_cut(int64_t n, const int64_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                                const int32_t* __restrict__ ew, const int32_t* __restrict__ vw,
                                                const int32_t* __restrict__ part, int32_t k,
                                                unsigned long long* __restrict__ acc) {
    extern __shared__ unsigned long long s_pw[];
    __shared__ unsigned long long s_cross;
    for (int q = threadIdx.x; q < k; q += blockDim.x) s_pw[q] = 0;
    if (threadIdx.x == 0) s_cross = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    unsigned long long cross = 0;
    for (int64_t v = wid; v < n; v += nw) {
        const int32_t p = part[v];
        for (int64_t e = rp[v] + lane; e < rp[v + 1]; e += 32)
            if (part[ci[e]] != p) cross += ew ? (unsigned long long)ew[e] : 1ull;
        if (lane == 0) atomicAdd(&s_pw[p], vw ? (unsigned long long)vw[v] : 1ull);
    }
    for (int o = 16; o > 0; o >>= 1) cross += __shfl_xor_sync(0xffffffffu, cross, o);
    if (lane == 0 && cross) atomicAdd(&s_cross, cross);
    __syncthreads();
    if (threadIdx.x == 0 && s_cross) atomicAdd(&acc[0], s_cross);
    for (int q = threadIdx.x; q < k; q += blockDim.x)
        if (s_pw[q]) atomicAdd(&acc[1 + q], s_pw[q]);
}

// device address of the scratch array in the current context (looked up on
// every call: the module may have been reloaded at another address)
static unsigned long long* noalloc_scratch() {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
        throw GpError(GP_ECUDA, std::string("cudaGetSymbolAddress(no-allocation scratch): ") + cudaGetErrorString(e));
    return (unsigned long long*)p;
}

}  // namespace gp

using namespace gp;

extern "C" int gp_edge_cut_device_noalloc(int64_t n, const int64_t* d_rowptr, const int32_t* d_colidx,
                                          const int32_t* d_ewgt, const int32_t* d_vwgt, const int32_t* d_part,
                                          int32_t k, void* stream, int64_t* cut_out, int64_t* part_weights_out) {
    t_err.clear();
    try {
        if (n < 0) throw GpError(GP_EINVAL, "n must be >= 0");
        if (k < 1 || k > GP_NOALLOC_MAX_K)
            throw GpError(GP_EINVAL, "k must be in [1, " + std::to_string(GP_NOALLOC_MAX_K) +
                                         "]: the no-allocation scratch holds GP_NOALLOC_MAX_K part weights");
        if (!cut_out) throw GpError(GP_EINVAL, "null cut_out");
        if (n == 0) {
            *cut_out = 0;
            if (part_weights_out) for (int q = 0; q < k; ++q) part_weights_out[q] = 0;
            return GP_OK;
        }
        if (!d_rowptr || !d_colidx || !d_part) throw GpError(GP_EINVAL, "null array");
        int dev = 0;
        GP_CUDA(cudaGetDevice(&dev));
        unsigned long long* scratch = noalloc_scratch();
        unsigned long long* err = scratch + 1 + GP_NOALLOC_MAX_K;
        cudaStream_t s = (cudaStream_t)stream;
        int sms = 148;
        GP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        // accumulators start at zero, the error word at "none"; the array keeps
        // the previous call's contents otherwise
        GP_CUDA(cudaMemsetAsync(scratch, 0, sizeof(unsigned long long) * (1 + k), s));
        GP_CUDA(cudaMemsetAsync(err, 0xff, sizeof(unsigned long long), s));
        k_na_check<<<grid_for(n, 256, sms * 8), 256, 0, s>>>(n, d_part, k, err);
        GP_CUDA(cudaGetLastError());
        unsigned long long bad = ~0ull;
        GP_CUDA(cudaMemcpyAsync(&bad, err, sizeof bad, cudaMemcpyDeviceToHost, s));
        GP_CUDA(cudaStreamSynchronize(s));
        if (bad != ~0ull) throw GpError(GP_EINVAL, "part id out of range at vertex " + std::to_string(bad));
        k_na_cut<<<grid_for(n * 32, 256, sms * 8), 256, sizeof(unsigned long long) * k, s>>>(
            n, d_rowptr, d_colidx, d_ewgt, d_vwgt, d_part, k, scratch);
        GP_CUDA(cudaGetLastError());
        unsigned long long cross = 0;
        GP_CUDA(cudaMemcpyAsync(&cross, scratch, sizeof cross, cudaMemcpyDeviceToHost, s));
        if (part_weights_out)
            GP_CUDA(cudaMemcpyAsync(part_weights_out, scratch + 1, sizeof(int64_t) * k, cudaMemcpyDeviceToHost, s));
        GP_CUDA(cudaStreamSynchronize(s));
        *cut_out = (int64_t)(cross / 2);
        return GP_OK;
    } catch (const GpError& e) {
        t_err = e.what();
        return e.code;
    } catch (const std::exception& e) {
        t_err = e.what();
        return GP_EINTERNAL;
    }
}
