// noalloc.cu -- element-energy sum that performs no device allocation.
//
// Some callers cannot let a library call cudaMalloc: applications whose
// device memory is owned by their own pool or arena (a framework's caching
// allocator, a fixed budget on a shared GPU), and real-time loops, such as a
// robot controller, that must not allocate after start-up because an
// allocation can block or fail at an arbitrary moment.  For them this file
// provides sors_elem_energy_noalloc: the caller passes every input and the
// output as device pointers, and the only scratch the kernel needs (per-block
// partial sums and a completion counter) lives in a fixed-size array that is
// part of the library image itself.
//
// That array is a file-scope __device__ variable: every GPU that loads the
// library holds it (kNoAllocScratchBytes, 64 KiB + 256 B) until the process
// exits, and all calls share it.  Calls whose work overlaps on the GPU (two
// streams, or two host threads) therefore race on it and must be serialised
// by the caller.  Each call zeroes the completion counter before its kernel,
// and its kernel leaves it at zero again.
//
// In host code the array's name only stands for the variable; its device
// address comes from cudaGetSymbolAddress with the caller's device current.
// A call on a stream that is not being captured looks the address up afresh
// (so a device reset, which reloads the library's module at a possibly
// different address, is picked up by the next call) and remembers it per
// device; a call on a capturing stream uses the remembered address.  So the
// first call on each device should come before any stream capture, and after
// a device reset one uncaptured call must precede the next capture.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <string>

#include "../../include/sors_b200.h"
#include "fem_math.cuh"
#include "sors_internal.h"

namespace {

constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocPerThread = 4;
constexpr int kNoAllocElemsPerBlock = kNoAllocThreads * kNoAllocPerThread;  // 1024
constexpr int kNoAllocMaxBlocks = 8192;
constexpr long long kNoAllocMaxElems = (long long)kNoAllocMaxBlocks * kNoAllocElemsPerBlock;  // 8,388,608

// [0, kNoAllocMaxBlocks): block partial sums; [kNoAllocMaxBlocks]: completion counter
// (stored in the first 4 bytes of the slot), padded to 256 bytes.
constexpr size_t kNoAllocScratchBytes = (size_t)kNoAllocMaxBlocks * sizeof(double) + 256;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_addr[kMaxDevices] = {nullptr};

int noalloc_fail(int code, const std::string& msg) {
    sors::set_last_error(msg);  // reported by sors_last_error
    return code;
}

template <int NV>
__global__ void __launch_bounds__(kNoAllocThreads) k_elem_energy_noalloc(int E, const double* __restrict__ Xg,
                                                                         const double* __restrict__ qg,
                                                                         const int* __restrict__ conn,
                                                                         const double* __restrict__ youngs,
                                                                         const double* __restrict__ poisson,
                                                                         unsigned char* scratch, double* out) {
    double* partials = reinterpret_cast<double*>(scratch);
    unsigned* counter = reinterpret_cast<unsigned*>(scratch + (size_t)kNoAllocMaxBlocks * sizeof(double));
    __shared__ double sh[kNoAllocThreads / 32];
    __shared__ bool am_last;
    double acc = 0.0;
    const int e0 = blockIdx.x * kNoAllocElemsPerBlock;
    for (int k = 0; k < kNoAllocPerThread; k++) {
        const int e = e0 + k * kNoAllocThreads + threadIdx.x;
        if (e >= E) break;
        double X[NV][3], x[NV][3];
#pragma unroll
        for (int w = 0; w < NV; w++) {
            const int n = __ldg(conn + (size_t)e * NV + w);
#pragma unroll
            for (int r = 0; r < 3; r++) { X[w][r] = __ldg(Xg + 3 * (size_t)n + r); x[w][r] = qg[3 * (size_t)n + r]; }
        }
        // Lame parameters (cpp/src/energies/neoHookean.cpp:10-11)
        const double Ey = youngs[e], nu = poisson[e];
        const double lam = (Ey * nu) / ((1 + nu) * (1 - 2 * nu));
        const double mu = Ey / (2 * (1 + nu));
        double d[NV][3], F[9];
        if (NV == 4) {
            const double V = sors::tet_shape((const double(*)[3])X, (double(*)[3])d);
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    double s = 0.0;
#pragma unroll
                    for (int w = 0; w < NV; w++) s += x[w][r] * d[w][c];
                    F[r * 3 + c] = s;
                }
            acc += V * sors::nh_qp_energy(F, mu, lam);
        } else {
            const double V = sors::hex_volume((const double(*)[3])X);
            double a8 = 0.0;
            for (int s = 0; s < 8; s++) {
                sors::hex_shape((const double(*)[3])X, s, (double(*)[3])d);
#pragma unroll
                for (int r = 0; r < 3; r++)
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        double t = 0.0;
#pragma unroll
                        for (int w = 0; w < NV; w++) t += x[w][r] * d[w][c];
                        F[r * 3 + c] = t;
                    }
                a8 += sors::nh_qp_energy(F, mu, lam) * 0.125;
            }
            acc += V * a8;
        }
    }
    // block sum in a fixed order
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = acc;
    __syncthreads();
    if (w == 0) {
        double v = (l < kNoAllocThreads / 32) ? sh[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (l == 0) {
            partials[blockIdx.x] = v;
            __threadfence();
            am_last = (atomicAdd(counter, 1u) == gridDim.x - 1);
        }
    }
    __syncthreads();
    if (!am_last) return;
    // the last block to finish sums all partials in block order
    __threadfence();
    const volatile double* vp = partials;
    double t = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += kNoAllocThreads) t += vp[b];
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    __syncthreads();
    if (l == 0) sh[w] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < kNoAllocThreads / 32; k++) s += sh[k];
        *out = s;
        *counter = 0u;
    }
}

// Device address of the scratch array on the current device: looked up afresh
// unless `stream` is capturing, in which case the address remembered from the
// last uncaptured call on this device is used.
int scratch_address(int device, cudaStream_t stream, unsigned char** ptr) {
    if (device < 0 || device >= kMaxDevices) return noalloc_fail(SORS_ERR_ARG, "device ordinal out of range");
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(stream, &cap);
    if (e != cudaSuccess)
        return noalloc_fail(SORS_ERR_CUDA, std::string("cudaStreamIsCapturing: ") + cudaGetErrorString(e));
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (cap == cudaStreamCaptureStatusNone) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            return noalloc_fail(SORS_ERR_CUDA,
                                std::string("cudaGetSymbolAddress of the scratch array failed: ") + cudaGetErrorString(e));
        g_noalloc_addr[device] = p;
    } else if (!g_noalloc_addr[device]) {
        return noalloc_fail(SORS_ERR_ARG,
                            "sors_elem_energy_noalloc: the first call on a device must come before any stream capture");
    }
    *ptr = static_cast<unsigned char*>(g_noalloc_addr[device]);
    return SORS_OK;
}

}  // namespace

extern "C" {

int sors_elem_energy_noalloc(const double* X_device, const double* q_device, const int32_t* conn_device,
                             int32_t n_elems, int32_t nodes_per_elem, const double* youngs_device,
                             const double* poisson_device, double* out_device, void* stream) {
    if (nodes_per_elem != 4 && nodes_per_elem != 8) return noalloc_fail(SORS_ERR_ARG, "nodes_per_elem must be 4 or 8");
    if (!out_device || (n_elems > 0 && (!X_device || !q_device || !conn_device || !youngs_device || !poisson_device)))
        return noalloc_fail(SORS_ERR_ARG, "NULL device pointer");
    if (n_elems < 0) return noalloc_fail(SORS_ERR_ARG, "n_elems must be >= 0");
    if ((long long)n_elems > kNoAllocMaxElems)
        return noalloc_fail(SORS_ERR_ARG, "n_elems = " + std::to_string(n_elems) +
                                              " exceeds the capacity of the fixed scratch array (" +
                                              std::to_string(kNoAllocMaxElems) + " elements)");
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return noalloc_fail(SORS_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned char* scratch = nullptr;
    int st = scratch_address(device, s, &scratch);
    if (st) return st;
    if (n_elems == 0) {
        e = cudaMemsetAsync(out_device, 0, sizeof(double), s);
        if (e != cudaSuccess) return noalloc_fail(SORS_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
        return SORS_OK;
    }
    // the completion counter must start at zero
    e = cudaMemsetAsync(scratch + (size_t)kNoAllocMaxBlocks * sizeof(double), 0, sizeof(unsigned), s);
    if (e != cudaSuccess) return noalloc_fail(SORS_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
    const int blocks = (n_elems + kNoAllocElemsPerBlock - 1) / kNoAllocElemsPerBlock;
    if (nodes_per_elem == 4)
        k_elem_energy_noalloc<4><<<blocks, kNoAllocThreads, 0, s>>>(n_elems, X_device, q_device, conn_device,
                                                                    youngs_device, poisson_device, scratch, out_device);
    else
        k_elem_energy_noalloc<8><<<blocks, kNoAllocThreads, 0, s>>>(n_elems, X_device, q_device, conn_device,
                                                                    youngs_device, poisson_device, scratch, out_device);
    e = cudaGetLastError();
    if (e != cudaSuccess) return noalloc_fail(SORS_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    return SORS_OK;
}

}  // extern "C"
