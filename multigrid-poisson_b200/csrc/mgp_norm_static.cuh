// mgp_norm_static.cuh -- max-norm of a caller-owned device array with no allocation.
//
// mgp_norm reduces into a scratch word that mgp_create allocated with the solver.  This
// variant serves callers that hold only a device pointer and must not allocate:
//  - a host code that couples to the solver through its own device buffers (the reference's
//    PoissonSolver is header-only and meant to sit inside a larger simulation) and checks a
//    norm from a region where its own pool allocator owns the device heap;
//  - a serving process that has committed device memory up to its reserve: a cudaMalloc
//    there can fail or, worse, take memory admission already promised to a request.
// Its scratch is a file-scope device array, so the only setup is looking up that array's
// address once per device; after that a call launches two kernels, copies 8 bytes back and
// synchronises the stream -- no cudaMalloc, cudaFree or allocating library call.
//
// Reduction: pass 1 gives block b the points [b*kNsChunk, (b+1)*kNsChunk) of the row-major
// (i, j, k) order and stores max |a| of that range (as the IEEE bit pattern of |a|, whose
// integer order is the order of the magnitudes; NaN sorts above every number, so a NaN
// propagates) into partial[b]; pass 2 is one block that reduces partial[0, nblk) into
// result.  Every slot that pass 2 reads was written by pass 1 of the same call, so nothing
// has to start at zero and no memset is issued.
#include <mutex>

namespace {

constexpr int kNsThreads = 256;
constexpr int kNsPerThread = 32;
constexpr long long kNsChunk = (long long)kNsThreads * kNsPerThread;  // points per block
constexpr int kNsMaxBlocks = 32768;                                    // 256 KB of partials
constexpr long long kNsMaxPoints = kNsChunk * kNsMaxBlocks;            // 2^28 points
constexpr int kNsMaxDevices = 64;

struct __align__(256) NormScratch {
    unsigned long long partial[kNsMaxBlocks];
    unsigned long long result;
};

static __device__ __align__(256) NormScratch g_norm_scratch;

// Block-wide max of v; the full result is valid in thread 0 only.
__device__ __forceinline__ unsigned long long ns_block_max(unsigned long long v) {
    __shared__ unsigned long long red[32];
    v = warp_max_u64(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        v = lane < nw ? red[lane] : 0ull;
        v = warp_max_u64(v);
    }
    return v;
}

template <typename T>
__global__ void __launch_bounds__(kNsThreads)
    k_norm_static_blocks(const T* __restrict__ a, int ny, int nz, long long sx, long long sy, long long n,
                         NormScratch* scratch) {
    const long long base = (long long)blockIdx.x * kNsChunk;
    unsigned long long mx = 0ull;
#pragma unroll 4
    for (int m = 0; m < kNsPerThread; m++) {
        const long long t = base + (long long)m * kNsThreads + threadIdx.x;
        if (t < n) {
            const int k = (int)(t % nz);
            const long long q = t / nz;
            const int j = (int)(q % ny);
            const long long i = q / ny;
            mx = max(mx, abs_bits(ldg(a + i * sx + (long long)j * sy + k)));
        }
    }
    mx = ns_block_max(mx);
    if (threadIdx.x == 0) scratch->partial[blockIdx.x] = mx;
}

__global__ void __launch_bounds__(1024) k_norm_static_final(int nblk, NormScratch* scratch) {
    unsigned long long mx = 0ull;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) mx = max(mx, scratch->partial[b]);
    mx = ns_block_max(mx);
    if (threadIdx.x == 0) scratch->result = mx;
}

// Address of g_norm_scratch on each device, looked up on the first call for that device.
std::mutex g_ns_mutex;
NormScratch* g_ns_addr[kNsMaxDevices] = {};

int ns_scratch(int device, NormScratch** out) {
    std::lock_guard<std::mutex> lock(g_ns_mutex);
    if (!g_ns_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_norm_scratch);
        if (e != cudaSuccess || !p)
            return fail(MGP_ERR_CUDA, "mgp_norm_device: cudaGetSymbolAddress of the static scratch on device %d: %s",
                        device, cudaGetErrorString(e));
        g_ns_addr[device] = (NormScratch*)p;
    }
    *out = g_ns_addr[device];
    return MGP_OK;
}

}  // namespace

extern "C" {

int mgp_norm_device(int device, const void* a, int dtype, const int64_t shape[3], const int64_t stride[2],
                    void* stream, double* out) {
    if (!shape || !stride || !out) return fail(MGP_ERR_INVALID_ARG, "mgp_norm_device: null shape, stride or out");
    if (dtype != MGP_F64 && dtype != MGP_F32) return fail(MGP_ERR_INVALID_ARG, "mgp_norm_device: bad dtype %d", dtype);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(MGP_ERR_NO_DEVICE, "mgp_norm_device: no CUDA device");
    if (device < 0 || device >= ndev || device >= kNsMaxDevices)
        return fail(MGP_ERR_INVALID_ARG, "mgp_norm_device: bad device %d", device);
    for (int d = 0; d < 3; d++)
        if (shape[d] < 0 || shape[d] > INT32_MAX)
            return fail(MGP_ERR_INVALID_ARG, "mgp_norm_device: bad extent %lld on axis %d", (long long)shape[d], d);
    const long long n = (long long)shape[0] * shape[1] * shape[2];
    if (n > kNsMaxPoints)
        return fail(MGP_ERR_INVALID_ARG,
                    "mgp_norm_device: %lld points exceed the static scratch limit of %lld points (%d blocks of %lld)",
                    n, kNsMaxPoints, kNsMaxBlocks, kNsChunk);
    if (n > 0) {
        if (!a) return fail(MGP_ERR_INVALID_ARG, "mgp_norm_device: null array");
        // rows must not overlap (stride[1] >= nz, stride[0] >= stride[1]*ny) and the last point's
        // offset must fit in 64 bits; products are checked for overflow before they are compared
        long long row = 0, last0 = 0, last1 = 0, last = 0;
        const bool ovf = __builtin_mul_overflow((long long)stride[1], (long long)shape[1], &row) ||
                         __builtin_mul_overflow((long long)stride[0], (long long)(shape[0] - 1), &last0) ||
                         __builtin_mul_overflow((long long)stride[1], (long long)(shape[1] - 1), &last1) ||
                         __builtin_add_overflow(last0, last1, &last) ||
                         __builtin_add_overflow(last, (long long)shape[2], &last);
        if (ovf || stride[1] < shape[2] || stride[0] < row)
            return fail(MGP_ERR_INVALID_ARG, "mgp_norm_device: strides {%lld, %lld} overlap rows of shape {%lld, %lld, %lld}"
                        " or overflow 64-bit offsets",
                        (long long)stride[0], (long long)stride[1], (long long)shape[0], (long long)shape[1],
                        (long long)shape[2]);
    }
    if (stream) {
        int sdev = -1;
        const cudaError_t e = cudaStreamGetDevice((cudaStream_t)stream, &sdev);
        if (e != cudaSuccess)
            return fail(MGP_ERR_INVALID_ARG, "mgp_norm_device: stream: %s", cudaGetErrorString(e));
        if (sdev != device)
            return fail(MGP_ERR_INVALID_ARG, "mgp_norm_device: the stream belongs to device %d, not %d", sdev, device);
    }
    DeviceGuard guard(device);
    NormScratch* scratch = nullptr;
    CKS(ns_scratch(device, &scratch));
    if (n == 0) {
        *out = 0.0;
        return MGP_OK;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const int nblk = (int)((n + kNsChunk - 1) / kNsChunk);
    const int ny = (int)shape[1], nz = (int)shape[2];
    if (dtype == MGP_F64)
        k_norm_static_blocks<double><<<nblk, kNsThreads, 0, st>>>((const double*)a, ny, nz, stride[0], stride[1], n,
                                                                  scratch);
    else
        k_norm_static_blocks<float><<<nblk, kNsThreads, 0, st>>>((const float*)a, ny, nz, stride[0], stride[1], n,
                                                                 scratch);
    CK(cudaGetLastError());
    k_norm_static_final<<<1, 1024, 0, st>>>(nblk, scratch);
    CK(cudaGetLastError());
    unsigned long long bits = 0ull;
    CK(cudaMemcpyAsync(&bits, &scratch->result, sizeof(bits), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    double v;
    memcpy(&v, &bits, sizeof(v));
    *out = v;
    return MGP_OK;
}

}  // extern "C"
