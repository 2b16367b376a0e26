// lbm_check_noalloc: the check() residual reduction for callers that cannot
// allocate device memory.
//
// Who needs it.  Some callers own every byte of device memory themselves and
// cannot let a library call cudaMalloc:
//   * a Fortran host that keeps the flow fields in its own device arrays
//     (OpenACC `host_data use_device`, CUDA Fortran) inside a pool it reserved
//     up front, where a hidden allocation would break its accounting;
//   * codes that run the time loop with the allocator locked or exhausted by
//     design (a memory pool sized to the whole GPU);
//   * callers that must not pay an allocation's implicit device-wide
//     synchronisation inside their step loop.
// They pass their own device arrays in and get the residuals back; this
// entry point allocates nothing (no cudaMalloc, no cudaFree, no allocating
// library routine).
//
// How.  The per-block partial sums of the two-pass reduction go to a fixed
// array in device global memory, declared below at file scope.  Every GPU on
// which this library's kernels are loaded holds that array (256 KiB + 64 B)
// until the process exits.  Its size bounds the problem: one block reduces
// 8192 nodes and the array holds 8192 block results, so a call accepts at most
// LBM_NOALLOC_MAX_NODES = 8192 * 8192 = 67,108,864 nodes and rejects more with
// LBM_ERR_PARAM.
//
// Set-up.  Host code cannot use the array's name as a device address (in host
// code it names a host-side stand-in).  The first call on each device, with
// that device current, asks the runtime for the array's device address with
// cudaGetSymbolAddress, checks the result and keeps it; later calls reuse it.
// Make that first call on a device before any stream capture begins.
//
// Sharing.  All calls share the one array and it keeps what the last call left
// there.  Nothing in it needs to start at zero: each call overwrites every
// partial sum it later reads and the result slot.  Calls whose work overlaps
// on the GPU (e.g. on two streams at once) race on the array; serialise them.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <mutex>

#include "../../include/lbm_b200.h"

namespace lbm {
int set_error(int code, const char *fmt, ...);
extern int64_t g_launches;
}

namespace {

constexpr int kThreads = 256;
constexpr int64_t kChunk = 8192;  // nodes reduced by one block
constexpr int kMaxBlocks = 8192;  // block results the scratch array holds
static_assert((int64_t)kChunk * kMaxBlocks == LBM_NOALLOC_MAX_NODES, "limit and scratch size disagree");

// [0..3] the four sums of the last call, [4..7] unused, then 4 partial sums
// per block
static __device__ __align__(256) double g_check_scratch[8 + 4 * kMaxBlocks];

constexpr int kMaxDevices = 64;
double *g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mu;

// block-wide sum of NV values per thread, written by thread 0 to out[0..NV-1]
template <int NV>
__device__ __forceinline__ void block_sum(double (&acc)[NV], double *out)
{
    __shared__ double sh[NV][kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < NV; ++c) {
        double v = acc[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[c][warp] = v;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int c = 0; c < NV; ++c) {
            double v = lane < kThreads / 32 ? sh[c][lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) out[c] = v;
        }
    }
}

// check() of natural-convection_2dim_mono.f90:755-805 over one chunk of nodes:
// sums of |u - u_prev|^2, |u|^2, (T - T_prev)^2, T^2, then the previous fields
// take the current ones
__global__ void __launch_bounds__(kThreads)
k_check_chunk(const double *__restrict__ u, const double *__restrict__ v, const double *__restrict__ w,
              const double *__restrict__ T, double *__restrict__ up, double *__restrict__ vp,
              double *__restrict__ wp, double *__restrict__ Tp, int64_t n, double *__restrict__ partials)
{
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    const int64_t beg = (int64_t)blockIdx.x * kChunk;
    const int64_t end = beg + kChunk < n ? beg + kChunk : n;
    for (int64_t i = beg + threadIdx.x; i < end; i += kThreads) {
        const double ui = u[i], vi = v[i], Ti = T[i];
        const double du = ui - up[i], dv = vi - vp[i], dT = Ti - Tp[i];
        if (w) {
            const double wi = w[i], dw = wi - wp[i];
            acc[0] += du * du + dv * dv + dw * dw;
            acc[1] += ui * ui + vi * vi + wi * wi;
            wp[i] = wi;
        } else {
            acc[0] += du * du + dv * dv;
            acc[1] += ui * ui + vi * vi;
        }
        acc[2] += dT * dT;
        acc[3] += Ti * Ti;
        up[i] = ui;
        vp[i] = vi;
        Tp[i] = Ti;
    }
    block_sum<4>(acc, partials + (int64_t)blockIdx.x * 4);
}

// one block: the block results in block order -> res[0..3]
__global__ void __launch_bounds__(kThreads) k_check_total(const double *__restrict__ partials, int nb,
                                                          double *__restrict__ res)
{
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < nb; b += kThreads)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[c] += partials[(int64_t)b * 4 + c];
    block_sum<4>(acc, res);
}

// The device address of the scratch array on the current device, looked up
// once per device.
int scratch_on_current_device(double **out)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return lbm::set_error(LBM_ERR_CUDA, "lbm_check_noalloc: cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return lbm::set_error(LBM_ERR_PARAM, "lbm_check_noalloc: device %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_check_scratch);
        if (e != cudaSuccess || !p)
            return lbm::set_error(LBM_ERR_CUDA, "lbm_check_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        g_scratch_addr[dev] = (double *)p;
    }
    *out = g_scratch_addr[dev];
    return LBM_OK;
}

}  // namespace

extern "C" int lbm_check_noalloc(const double *u, const double *v, const double *w, const double *T, double *u_prev,
                                 double *v_prev, double *w_prev, double *T_prev, int64_t n, double *errU,
                                 double *errT, void *stream)
{
    if (!u || !v || !T || !u_prev || !v_prev || !T_prev || (w != nullptr) != (w_prev != nullptr))
        return lbm::set_error(LBM_ERR_PARAM, "lbm_check_noalloc: a field pointer is NULL (w and w_prev go together)");
    if (n <= 0) return lbm::set_error(LBM_ERR_PARAM, "lbm_check_noalloc: n must be > 0");
    if (n > LBM_NOALLOC_MAX_NODES)
        return lbm::set_error(LBM_ERR_PARAM,
                              "lbm_check_noalloc: %lld nodes exceed the fixed scratch limit of %lld nodes",
                              (long long)n, (long long)LBM_NOALLOC_MAX_NODES);
    double *scratch = nullptr;
    int st = scratch_on_current_device(&scratch);
    if (st) return st;
    cudaStream_t s = (cudaStream_t)stream;
    const int nb = (int)((n + kChunk - 1) / kChunk);
    k_check_chunk<<<nb, kThreads, 0, s>>>(u, v, w, T, u_prev, v_prev, w_prev, T_prev, n, scratch + 8);
    k_check_total<<<1, kThreads, 0, s>>>(scratch + 8, nb, scratch);
    lbm::g_launches += 2;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return lbm::set_error(LBM_ERR_CUDA, "lbm_check_noalloc: launch: %s", cudaGetErrorString(e));
    double sums[4];
    e = cudaMemcpyAsync(sums, scratch, sizeof sums, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return lbm::set_error(LBM_ERR_CUDA, "lbm_check_noalloc: %s", cudaGetErrorString(e));
    // errorU = sqrt(error1_all)/sqrt(error2_all), errorT likewise (2M:784, 798)
    if (errU) *errU = sqrt(sums[0]) / sqrt(sums[1]);
    if (errT) *errT = sqrt(sums[2]) / sqrt(sums[3]);
    for (double x : sums)
        if (!isfinite(x)) return lbm::set_error(LBM_ERR_NONFINITE, "lbm_check_noalloc: non-finite residual sum");
    return LBM_OK;
}
