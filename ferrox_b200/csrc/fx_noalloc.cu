// fx_noalloc.cu -- fx_mean_P_noalloc: the mean-polarization reduction on
// caller-owned device buffers, with its scratch in a static device array.
//
// Some callers cannot allocate device memory at the point where they need
// this number: code that runs while another component owns the CUDA memory
// pool (a fixed-budget allocator, a framework that pre-reserves all of HBM),
// or code that must not call cudaMalloc/cudaFree because those calls
// synchronise the device and would stall a pipeline of asynchronous work.
// This entry point allocates nothing.  Its scratch -- one partial sum pair per
// block and the last-block counter -- lives in `g_mean_p_scratch` below, a
// file-scope __device__ array of fixed size that every GPU which loads this
// library holds until the process exits.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/ferrox_b200.h"

namespace fx {
void set_free_error(const std::string& m);   // message for fx_create_error()
}

namespace {

constexpr int NA_THREADS = 256;
constexpr int NA_MAX_BLOCKS = 1024;
constexpr long long NA_CELLS_PER_THREAD = 64;
// largest n: every thread folds at most 64 cells into its register sum
constexpr long long NA_MAX_CELLS = (long long)NA_MAX_BLOCKS * NA_THREADS * NA_CELLS_PER_THREAD;

struct MeanPScratch {
    double part[4 * NA_MAX_BLOCKS];   // per-block sums of Px, Py, Pz and the cell count
    unsigned int counter;             // blocks finished; must be 0 when a launch starts
};

// 32 KB + 4 B on every device that loads the library
static __device__ __align__(256) MeanPScratch g_mean_p_scratch;

// host-side device addresses of g_mean_p_scratch, one per device.  In host
// code the symbol itself is only a stand-in, not a device address.
std::mutex g_mu;
constexpr int NA_MAX_DEVICES = 64;
MeanPScratch* g_addr[NA_MAX_DEVICES] = {};

__device__ double na_block_sum(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (w == 0) {
        r = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    __syncthreads();
    return r;
}

// mean of Px, Py, Pz over the cells whose mask is 0 (ferroelectric); the same
// fold as k_mean_p, with the block partials in the static scratch
__global__ void __launch_bounds__(NA_THREADS) k_mean_p_noalloc(const double* __restrict__ Px, const double* __restrict__ Py,
                                                               const double* __restrict__ Pz, const uint8_t* __restrict__ mask,
                                                               long long n, MeanPScratch* __restrict__ sc,
                                                               double* __restrict__ out) {
    __shared__ double sh[32];
    __shared__ bool last;
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        if (mask[c] == 0) {
            if (Px) s[0] += Px[c];
            if (Py) s[1] += Py[c];
            s[2] += Pz[c];
            s[3] += 1.0;
        }
    }
    double b[4];
    for (int q = 0; q < 4; ++q) b[q] = na_block_sum(s[q], sh);
    if (threadIdx.x == 0) {
        for (int q = 0; q < 4; ++q) sc->part[4 * blockIdx.x + q] = b[q];
        __threadfence();
        last = atomicAdd(&sc->counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last) {
        __threadfence();
        double t[4] = {0.0, 0.0, 0.0, 0.0};
        for (unsigned blk = threadIdx.x; blk < gridDim.x; blk += blockDim.x)
            for (int q = 0; q < 4; ++q) t[q] += ((volatile double*)sc->part)[4 * blk + q];
        for (int q = 0; q < 4; ++q) t[q] = na_block_sum(t[q], sh);
        if (threadIdx.x == 0) {
            for (int q = 0; q < 3; ++q) out[q] = t[3] > 0 ? t[q] / t[3] : 0.0;
            sc->counter = 0;
        }
    }
}

}  // namespace

extern "C" int fx_mean_P_noalloc(const double* d_Px, const double* d_Py, const double* d_Pz, const uint8_t* d_mask,
                                 size_t n, double* d_out, void* cuda_stream) {
    if (!d_Pz || !d_mask || !d_out || n == 0) {
        fx::set_free_error("fx_mean_P_noalloc: Pz, mask and out must be device pointers and n > 0");
        return FX_ERR_INVALID_ARGUMENT;
    }
    if ((long long)n > NA_MAX_CELLS) {
        fx::set_free_error("fx_mean_P_noalloc: n = " + std::to_string(n) + " exceeds the static scratch limit of " +
                           std::to_string(NA_MAX_CELLS) + " cells");
        return FX_ERR_INVALID_ARGUMENT;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= NA_MAX_DEVICES) {
        fx::set_free_error(std::string("fx_mean_P_noalloc: no current device: ") + cudaGetErrorString(e));
        return FX_ERR_CUDA;
    }
    MeanPScratch* sc = nullptr;
    {
        // first call on this device: look up the device address of the
        // static scratch (with this device current)
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_addr[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_mean_p_scratch);
            if (e != cudaSuccess || !p) {
                fx::set_free_error(std::string("fx_mean_P_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
                return FX_ERR_CUDA;
            }
            g_addr[dev] = static_cast<MeanPScratch*>(p);
        }
        sc = g_addr[dev];
    }
    cudaStream_t s = (cudaStream_t)cuda_stream;
    // the counter must start at 0; a call that was interrupted may have left it
    e = cudaMemsetAsync(&sc->counter, 0, sizeof(unsigned int), s);
    if (e != cudaSuccess) {
        fx::set_free_error(std::string("fx_mean_P_noalloc: ") + cudaGetErrorString(e));
        return FX_ERR_CUDA;
    }
    long long blocks = ((long long)n + (long long)NA_THREADS * NA_CELLS_PER_THREAD - 1) / ((long long)NA_THREADS * NA_CELLS_PER_THREAD);
    if (blocks < 1) blocks = 1;
    if (blocks > NA_MAX_BLOCKS) blocks = NA_MAX_BLOCKS;
    k_mean_p_noalloc<<<(unsigned)blocks, NA_THREADS, 0, s>>>(d_Px, d_Py, d_Pz, d_mask, (long long)n, sc, d_out);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        fx::set_free_error(std::string("fx_mean_P_noalloc: launch: ") + cudaGetErrorString(e));
        return FX_ERR_CUDA;
    }
    return FX_OK;
}
