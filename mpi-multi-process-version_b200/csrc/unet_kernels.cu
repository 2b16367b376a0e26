// Forward and backward kernels of the warm-start surrogate (a 4-level U-Net
// over NHWC bfloat16 images, FP32 accumulation).  No counterpart in the
// reference, which always starts from the conduction state of initial()
// (natural-convection_2dim_mono.f90:199-240).
//
// 3x3 convolutions are implicit GEMMs on the tensor cores (bf16 inputs, FP32
// accumulators, mma m16n8k16):
//   forward      M = pixels, N = Cout, K = 9 Cin;  A = im2col(x) gathered by
//                cp.async with zero fill at the image border, B = weights
//                [Cout][9][Cin] (K contiguous), two-stage shared-memory ring;
//   data grad    the same kernel on dL/dz with the flipped, transposed weights;
//   weight grad  M = Cout, N = 9 Cin, K = pixels, split over pixel ranges into
//                FP32 partials that a second kernel sums in a fixed order
//                (deterministic).
// Elementwise work (SiLU backward, pooling, upsampling, the 1x1 output layer,
// the loss, Adam) is plain CUDA-core code.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "../../include/lbm_b200.h"
#include "../../include/lbm_surrogate.h"

namespace lbm {
int set_error(int code, const char *fmt, ...);
extern int64_t g_launches;
}  // namespace lbm

namespace {

typedef __nv_bfloat16 bf16;

constexpr int kThreads = 256;

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int bytes)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// D += A * B for one 16x8x16 bf16 tile (A row-major, B column-major fragments)
__device__ __forceinline__ void mma16816(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t ld32(const bf16 *p) { return *reinterpret_cast<const uint32_t *>(p); }

__device__ __forceinline__ float silu(float z) { return z / (1.0f + expf(-z)); }
__device__ __forceinline__ float silu_grad(float z)
{
    const float s = 1.0f / (1.0f + expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

// ---------------------------------------------------------------------------
// 3x3 convolution (forward and data gradient)
// ---------------------------------------------------------------------------
constexpr int CBM = 128;       // pixels per block
constexpr int CBK = 32;        // input channels per K chunk (one tap)
constexpr int CLD = CBK + 8;   // shared-memory row stride: rows 80 B apart, conflict-free fragment loads

struct ConvArgs {
    const bf16 *x;
    int64_t xs;
    int xo;
    const bf16 *w;
    const float *bias;
    int B, H, W, Cin, Cout;
    float *of;
    int64_t os;
    int oo, acc;
    bf16 *oa;
    int64_t as;
    int ao, act;
};

// 8 warps: 4 along M (32 pixels each) x 2 along N (BN/2 channels each)
template <int BN>
__global__ void __launch_bounds__(kThreads) k_conv3x3(const ConvArgs a)
{
    __shared__ __align__(16) bf16 As[2][CBM * CLD];
    __shared__ __align__(16) bf16 Bs[2][BN * CLD];
    constexpr int NT = BN / 16;  // n8 tiles per warp
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp & 3, wn = warp >> 2;
    const int64_t M = (int64_t)a.B * a.H * a.W;
    const int64_t m0 = (int64_t)blockIdx.x * CBM;
    const int n0 = blockIdx.y * BN;
    const int cchunks = a.Cin / CBK;
    const int nk = 9 * cchunks;

    // the two 16-byte pieces of the A tile this thread gathers
    int ar[2], aq[2], ab[2], ay[2], ax[2];
    bool av[2];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const int v = tid + i * kThreads;
        ar[i] = v >> 2;
        aq[i] = v & 3;
        const int64_t m = m0 + ar[i];
        av[i] = m < M;
        const int64_t mm = av[i] ? m : 0;
        ax[i] = int(mm % a.W);
        ay[i] = int((mm / a.W) % a.H);
        ab[i] = int(mm / ((int64_t)a.W * a.H));
    }

    auto load = [&](int kc, int st) {
        const int tap = kc / cchunks, c0 = (kc % cchunks) * CBK;
        const int dy = tap / 3 - 1, dx = tap % 3 - 1;
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int yy = ay[i] + dy, xx = ax[i] + dx;
            const bool ok = av[i] && yy >= 0 && yy < a.H && xx >= 0 && xx < a.W;
            const bf16 *src =
                ok ? a.x + ((int64_t)(ab[i] * a.H + yy) * a.W + xx) * a.xs + a.xo + c0 + aq[i] * 8 : a.x;
            cp_async16(&As[st][ar[i] * CLD + aq[i] * 8], src, ok ? 16 : 0);
        }
        if (tid < BN * 4) {
            const int r = tid >> 2, q = tid & 3;
            const int n = n0 + r;
            const bool ok = n < a.Cout;
            const bf16 *src = ok ? a.w + ((int64_t)n * 9 + tap) * a.Cin + c0 + q * 8 : a.w;
            cp_async16(&Bs[st][r * CLD + q * 8], src, ok ? 16 : 0);
        }
        cp_commit();
    };

    float acc[2][NT][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.0f;

    const int g = lane >> 2, t = lane & 3;
    load(0, 0);
    for (int kc = 0; kc < nk; ++kc) {
        const int st = kc & 1;
        if (kc + 1 < nk) {
            load(kc + 1, st ^ 1);
            cp_wait<1>();
        } else {
            cp_wait<0>();
        }
        __syncthreads();
        const bf16 *as_ = As[st];
        const bf16 *bs_ = Bs[st];
#pragma unroll
        for (int ks = 0; ks < CBK; ks += 16) {
            const int col = ks + 2 * t;
            uint32_t af[2][4], bfr[NT][2];
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                const int row = wm * 32 + mt * 16 + g;
                af[mt][0] = ld32(as_ + row * CLD + col);
                af[mt][1] = ld32(as_ + (row + 8) * CLD + col);
                af[mt][2] = ld32(as_ + row * CLD + col + 8);
                af[mt][3] = ld32(as_ + (row + 8) * CLD + col + 8);
            }
#pragma unroll
            for (int nt = 0; nt < NT; ++nt) {
                const int nrow = wn * (BN / 2) + nt * 8 + g;
                bfr[nt][0] = ld32(bs_ + nrow * CLD + col);
                bfr[nt][1] = ld32(bs_ + nrow * CLD + col + 8);
            }
#pragma unroll
            for (int mt = 0; mt < 2; ++mt)
#pragma unroll
                for (int nt = 0; nt < NT; ++nt)
                    mma16816(acc[mt][nt], af[mt][0], af[mt][1], af[mt][2], af[mt][3], bfr[nt][0], bfr[nt][1]);
        }
        __syncthreads();
    }

#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < NT; ++nt)
#pragma unroll
            for (int h = 0; h < 2; ++h)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int64_t m = m0 + wm * 32 + mt * 16 + g + h * 8;
                    const int n = n0 + wn * (BN / 2) + nt * 8 + 2 * t + e;
                    if (m >= M || n >= a.Cout) continue;
                    float z = acc[mt][nt][h * 2 + e];
                    if (a.bias) z += a.bias[n];
                    if (a.of) {
                        float *p = a.of + m * a.os + a.oo + n;
                        *p = a.acc ? *p + z : z;
                    }
                    if (a.oa) a.oa[m * a.as + a.ao + n] = __float2bfloat16_rn(a.act ? silu(z) : z);
                }
}

__global__ void k_flip(const bf16 *__restrict__ w, bf16 *__restrict__ wt, int Cout, int Cin)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t n = (int64_t)Cout * 9 * Cin;
    if (i >= n) return;
    // i indexes wt[ci][tap][co]
    const int co = int(i % Cout);
    const int tap = int((i / Cout) % 9);
    const int ci = int(i / ((int64_t)Cout * 9));
    wt[i] = w[((int64_t)co * 9 + (8 - tap)) * Cin + ci];
}

// ---------------------------------------------------------------------------
// 3x3 weight gradient
// ---------------------------------------------------------------------------
constexpr int WBM = 64;       // output channels per block
constexpr int WBN = 32;       // input channels per block (one tap)
constexpr int WBK = 32;       // pixels per step
constexpr int WLD = WBK + 8;

// 8 warps: 4 along M (16 output channels) x 2 along N (16 input channels)
__global__ void __launch_bounds__(kThreads)
k_wgrad(const bf16 *__restrict__ dz, const bf16 *__restrict__ x, int64_t xs, int xo, int B, int H, int W, int Cin,
        int Cout, int64_t per, float *__restrict__ ws)
{
    __shared__ __align__(16) bf16 As[WBM * WLD];  // [co][p]
    __shared__ __align__(16) bf16 Bs[WBN * WLD];  // [ci][p]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp & 3, wn = warp >> 2;
    const int g = lane >> 2, t = lane & 3;
    const int cchunks = Cin / WBN;
    const int tap = blockIdx.x / cchunks, c0 = (blockIdx.x % cchunks) * WBN;
    const int dy = tap / 3 - 1, dx = tap % 3 - 1;
    const int co0 = blockIdx.y * WBM;
    const int64_t M = (int64_t)B * H * W;
    const int64_t p_beg = (int64_t)blockIdx.z * per;
    const int64_t p_end = p_beg + per < M ? p_beg + per : M;

    float acc[2][4];
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[j][e] = 0.0f;

    for (int64_t p0 = p_beg; p0 < p_end; p0 += WBK) {
        {   // dz rows: 32 pixels x 64 channels, 8 channels per thread
            const int pr = tid >> 3, cv = tid & 7;
            const int64_t p = p0 + pr;
            uint4 val = make_uint4(0, 0, 0, 0);
            if (p < p_end && co0 + cv * 8 < Cout)
                val = *reinterpret_cast<const uint4 *>(dz + p * Cout + co0 + cv * 8);
            const bf16 *e = reinterpret_cast<const bf16 *>(&val);
#pragma unroll
            for (int j = 0; j < 8; ++j) As[(cv * 8 + j) * WLD + pr] = e[j];
        }
        if (tid < 128) {   // x at the tap's offset: 32 pixels x 32 channels
            const int pr = tid >> 2, cv = tid & 3;
            const int64_t p = p0 + pr;
            uint4 val = make_uint4(0, 0, 0, 0);
            if (p < p_end) {
                const int xx = int(p % W) + dx;
                const int yy = int((p / W) % H) + dy;
                const int b = int(p / ((int64_t)W * H));
                if (yy >= 0 && yy < H && xx >= 0 && xx < W)
                    val = *reinterpret_cast<const uint4 *>(x + ((int64_t)(b * H + yy) * W + xx) * xs + xo + c0 + cv * 8);
            }
            const bf16 *e = reinterpret_cast<const bf16 *>(&val);
#pragma unroll
            for (int j = 0; j < 8; ++j) Bs[(cv * 8 + j) * WLD + pr] = e[j];
        }
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < WBK; ks += 16) {
            const int col = ks + 2 * t;
            const int row = wm * 16 + g;
            const uint32_t a0 = ld32(As + row * WLD + col), a1 = ld32(As + (row + 8) * WLD + col);
            const uint32_t a2 = ld32(As + row * WLD + col + 8), a3 = ld32(As + (row + 8) * WLD + col + 8);
#pragma unroll
            for (int nt = 0; nt < 2; ++nt) {
                const int nrow = wn * 16 + nt * 8 + g;
                mma16816(acc[nt], a0, a1, a2, a3, ld32(Bs + nrow * WLD + col), ld32(Bs + nrow * WLD + col + 8));
            }
        }
        __syncthreads();
    }
    const int64_t K9 = 9 * (int64_t)Cin;
#pragma unroll
    for (int nt = 0; nt < 2; ++nt)
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int co = co0 + wm * 16 + g + h * 8;
                const int ci = c0 + wn * 16 + nt * 8 + 2 * t + e;
                if (co < Cout) ws[((int64_t)blockIdx.z * Cout + co) * K9 + (int64_t)tap * Cin + ci] = acc[nt][h * 2 + e];
            }
}

// out[i] = sum_{s < S} ws[s*n + i], in order
__global__ void k_sum_splits(const float *__restrict__ ws, int S, int64_t n, float *__restrict__ out)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float s = 0.0f;
    for (int k = 0; k < S; ++k) s += ws[(int64_t)k * n + i];
    out[i] = s;
}

struct WgradPlan {
    int S;
    int64_t per;
};

WgradPlan wgrad_plan(int B, int H, int W, int Cin, int Cout)
{
    const int64_t M = (int64_t)B * H * W;
    const int64_t bps = (int64_t)(9 * Cin / WBN) * ((Cout + WBM - 1) / WBM);
    int64_t S = (1184 + bps - 1) / bps;                   // about 8 blocks per SM over 148 SMs
    const int64_t smax = (M + 255) / 256;                 // at least 256 pixels per split
    if (S > smax) S = smax;
    if (S < 1) S = 1;
    int64_t per = (M + S - 1) / S;
    per = (per + WBK - 1) / WBK * WBK;
    S = (M + per - 1) / per;
    return {int(S), per};
}

// ---------------------------------------------------------------------------
// column sums (bias gradient)
// ---------------------------------------------------------------------------
constexpr int64_t kColRows = 2048;

__global__ void k_colsum(const bf16 *__restrict__ a, int64_t P, int C, float *__restrict__ ws)
{
    __shared__ float sh[8][33];
    const int c = blockIdx.x * 32 + (threadIdx.x & 31);
    const int rl = threadIdx.x >> 5;
    const int64_t beg = (int64_t)blockIdx.y * kColRows;
    const int64_t end = beg + kColRows < P ? beg + kColRows : P;
    float s = 0.0f;
    if (c < C)
        for (int64_t p = beg + rl; p < end; p += 8) s += __bfloat162float(a[p * C + c]);
    sh[rl][threadIdx.x & 31] = s;
    __syncthreads();
    if (rl == 0 && c < C) {
        float tot = 0.0f;
        for (int r = 0; r < 8; ++r) tot += sh[r][threadIdx.x & 31];
        ws[(int64_t)blockIdx.y * C + c] = tot;
    }
}

// ---------------------------------------------------------------------------
// elementwise
// ---------------------------------------------------------------------------
__global__ void k_silu_bwd(const float *__restrict__ da, int64_t das, int dao, const float *__restrict__ z, int64_t P,
                           int C, bf16 *__restrict__ dz)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P * C) return;
    const int64_t p = i / C;
    const int c = int(i % C);
    dz[i] = __float2bfloat16_rn(da[p * das + dao + c] * silu_grad(z[i]));
}

__global__ void k_pool2(const bf16 *__restrict__ x, int64_t xs, int xo, int B, int H, int W, int C,
                        bf16 *__restrict__ y, int64_t ys, int yo)
{
    const int h = H / 2, w = W / 2;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)B * h * w * C) return;
    const int c = int(i % C);
    const int64_t q = i / C;
    const int X = int(q % w), Y = int((q / w) % h), b = int(q / ((int64_t)w * h));
    auto at = [&](int yy, int xx) { return __bfloat162float(x[((int64_t)(b * H + yy) * W + xx) * xs + xo + c]); };
    const float s = (at(2 * Y, 2 * X) + at(2 * Y, 2 * X + 1)) + (at(2 * Y + 1, 2 * X) + at(2 * Y + 1, 2 * X + 1));
    y[q * ys + yo + c] = __float2bfloat16_rn(0.25f * s);
}

__global__ void k_pool2_bwd(const float *__restrict__ dy, int64_t dys, int dyo, int B, int H, int W, int C,
                            float *__restrict__ dx, int64_t dxs, int dxo)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)B * H * W * C) return;
    const int c = int(i % C);
    const int64_t q = i / C;
    const int xx = int(q % W), yy = int((q / W) % H), b = int(q / ((int64_t)W * H));
    const int64_t src = ((int64_t)(b * (H / 2) + yy / 2) * (W / 2) + xx / 2) * dys + dyo + c;
    dx[q * dxs + dxo + c] += 0.25f * dy[src];
}

__global__ void k_up2(const bf16 *__restrict__ x, int64_t xs, int xo, int B, int h, int w, int C,
                      bf16 *__restrict__ y, int64_t ys, int yo)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int H = 2 * h, W = 2 * w;
    if (i >= (int64_t)B * H * W * C) return;
    const int c = int(i % C);
    const int64_t q = i / C;
    const int X = int(q % W), Y = int((q / W) % H), b = int(q / ((int64_t)W * H));
    y[q * ys + yo + c] = x[((int64_t)(b * h + Y / 2) * w + X / 2) * xs + xo + c];
}

__global__ void k_up2_bwd(const float *__restrict__ dy, int64_t dys, int dyo, int B, int h, int w, int C,
                          float *__restrict__ dx, int64_t dxs, int dxo, int accumulate)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)B * h * w * C) return;
    const int c = int(i % C);
    const int64_t q = i / C;
    const int X = int(q % w), Y = int((q / w) % h), b = int(q / ((int64_t)w * h));
    const int W = 2 * w, H = 2 * h;
    auto at = [&](int yy, int xx) { return dy[((int64_t)(b * H + yy) * W + xx) * dys + dyo + c]; };
    const float s = (at(2 * Y, 2 * X) + at(2 * Y, 2 * X + 1)) + (at(2 * Y + 1, 2 * X) + at(2 * Y + 1, 2 * X + 1));
    float *o = dx + q * dxs + dxo + c;
    *o = accumulate ? *o + s : s;
}

constexpr int kMaxJ = 8;

__global__ void k_head(const bf16 *__restrict__ a, int64_t as, int ao, const bf16 *__restrict__ wh,
                       const float *__restrict__ bh, int64_t P, int C, int J, float *__restrict__ y)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    float acc[kMaxJ];
    for (int j = 0; j < J; ++j) acc[j] = bh ? bh[j] : 0.0f;
    for (int c = 0; c < C; ++c) {
        const float v = __bfloat162float(a[p * as + ao + c]);
        for (int j = 0; j < J; ++j) acc[j] += v * __bfloat162float(wh[j * C + c]);
    }
    for (int j = 0; j < J; ++j) y[p * J + j] = acc[j];
}

__global__ void k_head_bwd_da(const float *__restrict__ dy, const bf16 *__restrict__ wh, int64_t P, int C, int J,
                              float *__restrict__ da, int64_t das, int dao)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P * C) return;
    const int64_t p = i / C;
    const int c = int(i % C);
    float s = 0.0f;
    for (int j = 0; j < J; ++j) s += dy[p * J + j] * __bfloat162float(wh[j * C + c]);
    da[p * das + dao + c] = s;
}

constexpr int64_t kHeadRows = 1024;

// per pixel range: items j*C + c (dwh) and J*C + j (dbh)
__global__ void k_head_bwd_w(const float *__restrict__ dy, const bf16 *__restrict__ a, int64_t as, int ao, int64_t P,
                             int C, int J, float *__restrict__ ws)
{
    const int items = J * C + J;
    const int64_t beg = (int64_t)blockIdx.x * kHeadRows;
    const int64_t end = beg + kHeadRows < P ? beg + kHeadRows : P;
    for (int it = threadIdx.x; it < items; it += blockDim.x) {
        float s = 0.0f;
        if (it < J * C) {
            const int j = it / C, c = it % C;
            for (int64_t p = beg; p < end; ++p) s += dy[p * J + j] * __bfloat162float(a[p * as + ao + c]);
        } else {
            const int j = it - J * C;
            for (int64_t p = beg; p < end; ++p) s += dy[p * J + j];
        }
        ws[(int64_t)blockIdx.x * items + it] = s;
    }
}

constexpr int kMseBlocks = 296;

__global__ void k_mse(const float *__restrict__ y, const float *__restrict__ t, const float *__restrict__ cw, int64_t P,
                      int J, float *__restrict__ dy, float *__restrict__ ws)
{
    __shared__ float sh[kThreads / 32];
    const int64_t n = P * J;
    const float inv = 1.0f / float(n);
    float s = 0.0f;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int j = int(i % J);
        const float d = y[i] - t[i];
        const float w = cw ? cw[j] : 1.0f;
        dy[i] = 2.0f * w * d * inv;
        s += w * d * d;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float tot = 0.0f;
        for (int k = 0; k < kThreads / 32; ++k) tot += sh[k];
        ws[blockIdx.x] = tot;
    }
}

__global__ void k_mse_final(const float *__restrict__ ws, int nb, int64_t n, float *__restrict__ loss)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    float s = 0.0f;
    for (int k = 0; k < nb; ++k) s += ws[k];
    *loss = s / float(n);
}

__global__ void k_adam(float *__restrict__ p, bf16 *__restrict__ pb, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, int64_t n, float lr, float b1, float b2, float eps, float c1, float c2,
                       float wd)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float pi = p[i] - lr * ((mi / c1) / (sqrtf(vi / c2) + eps) + wd * p[i]);
    p[i] = pi;
    if (pb) pb[i] = __float2bfloat16_rn(pi);
}

__global__ void k_to_bf16(const float *__restrict__ x, bf16 *__restrict__ y, int64_t n)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = __float2bfloat16_rn(x[i]);
}

unsigned blocks_for(int64_t n) { return unsigned((n + kThreads - 1) / kThreads); }

int launched(const char *what, int count = 1)
{
    lbm::g_launches += count;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return lbm::set_error(LBM_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    return LBM_OK;
}

bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }

// ---------------------------------------------------------------------------
// 3x3 convolution on the 5th-generation tensor cores (tcgen05, TMEM)
// ---------------------------------------------------------------------------
// Same implicit GEMM as k_conv3x3 (M = pixels, N = Cout, K = 9 Cin), with the
// accumulator tile (128 pixels x BN channels, FP32) held in tensor memory:
//   * 4 warps gather the im2col tile and the weight tile of each K chunk (one
//     tap, 32 input channels) with cp.async into a 4-stage ring, two chunks
//     ahead, in the no-swizzle K-major core-matrix layout (8 rows x 16 bytes
//     per core matrix; K-adjacent core matrices 128 B apart, 8-row groups
//     512 B apart);
//   * after a generic-to-async proxy fence and a CTA barrier, one thread issues
//     two tcgen05.mma (K = 16 each) and commits them to the stage's mbarrier,
//     which frees the stage for the copy of chunk kc + 4;
//   * the epilogue reads the accumulators back with tcgen05.ld (warp w owns
//     TMEM lanes 32w..32w+31, i.e. pixels 32w..32w+31 of the tile).
// Every mbarrier wait is bounded; on timeout the CTA counts the event in
// g_nn_timeouts (read by lbm_nn_timeouts), waits (bounded) for its own MMAs,
// frees its tensor memory and returns.
constexpr int TBM = 128, TBK = 32, TSTAGES = 4, TTHREADS = 128;
constexpr long long kNnWaitCycles = 2000000000LL;  // ~1 s at 1.9 GHz
__device__ int g_nn_timeouts;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void nn_mbar_init(uint64_t *b, uint32_t n)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(n) : "memory");
}

__device__ __forceinline__ bool nn_mbar_test(uint64_t *b, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool nn_mbar_wait(uint64_t *b, uint32_t parity)
{
    if (nn_mbar_test(b, parity)) return true;
    const long long t0 = clock64();
    while (!nn_mbar_test(b, parity))
        if (clock64() - t0 > kNnWaitCycles) return false;
    return true;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// shared-memory matrix descriptor: start address, leading / stride byte
// offsets (>> 4), descriptor version 1, base offset 0, no swizzle
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// instruction descriptor of kind::f16: FP32 accumulator, bf16 A and B, both
// K-major, N = BN, M = 128
template <int BN>
__host__ __device__ constexpr uint32_t umma_idesc()
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(TBM >> 4) << 24);
}

template <int BN>
struct TcLayout {
    static constexpr int A_BYTES = TBM * TBK * 2;  // 8 KB
    static constexpr int B_BYTES = BN * TBK * 2;
    static constexpr int STAGE = A_BYTES + B_BYTES;
    static constexpr int BAR = TSTAGES * STAGE;    // mbarriers, then the TMEM address
    static_assert(BAR >= TBM * 33 * 4, "the epilogue stages 128 x 33 floats in the ring");
    static_assert(BN == 32 || BN == 64 || BN == 128 || BN == 256, "TMEM allocations are powers of two >= 32");
    static constexpr int SMEM = BAR + 64 + 1024;   // + alignment slack
    // shared memory bounds the CTAs per SM, so their TMEM columns fit the SM's 512
    static_assert((228 * 1024 / SMEM) * BN <= 512, "TMEM oversubscription");
    // byte offset of element (row r, 16-byte piece q) in a K-major no-swizzle tile
    __device__ static int off(int r, int q) { return (r >> 3) * 512 + q * 128 + (r & 7) * 16; }
};

template <int BN>
__global__ void __launch_bounds__(TTHREADS) k_conv3x3_tc(const ConvArgs a)
{
    using Lt = TcLayout<BN>;
    extern __shared__ unsigned char tc_raw[];
    unsigned char *sm = tc_raw + ((1024u - (smem_u32(tc_raw) & 1023u)) & 1023u);
    uint64_t *bars = reinterpret_cast<uint64_t *>(sm + Lt::BAR);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + TSTAGES);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t M = (int64_t)a.B * a.H * a.W;
    const int64_t m0 = (int64_t)blockIdx.x * TBM;
    const int n0 = blockIdx.y * BN;
    const int cchunks = a.Cin / TBK;
    const int nk = 9 * cchunks;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < TSTAGES; ++s) nn_mbar_init(&bars[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    // the four A pieces of this thread: rows r = (tid + 128 i) / 4, 16-byte piece q
    int ab[4], ay[4], ax[4];
    bool av[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int r = (tid + i * TTHREADS) >> 2;
        const int64_t m = m0 + r;
        av[i] = m < M;
        const int64_t mm = av[i] ? m : 0;
        ax[i] = int(mm % a.W);
        ay[i] = int((mm / a.W) % a.H);
        ab[i] = int(mm / ((int64_t)a.W * a.H));
    }
    auto load = [&](int kc) {
        unsigned char *st = sm + (kc % TSTAGES) * Lt::STAGE;
        const int tap = kc / cchunks, c0 = (kc % cchunks) * TBK;
        const int dy = tap / 3 - 1, dx = tap % 3 - 1;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int v = tid + i * TTHREADS, r = v >> 2, q = v & 3;
            const int yy = ay[i] + dy, xx = ax[i] + dx;
            const bool ok = av[i] && yy >= 0 && yy < a.H && xx >= 0 && xx < a.W;
            const bf16 *src = ok ? a.x + ((int64_t)(ab[i] * a.H + yy) * a.W + xx) * a.xs + a.xo + c0 + q * 8 : a.x;
            cp_async16(st + Lt::off(r, q), src, ok ? 16 : 0);
        }
#pragma unroll
        for (int i = 0; i < BN / 32; ++i) {
            const int v = tid + i * TTHREADS, r = v >> 2, q = v & 3;
            const int n = n0 + r;
            const bool ok = n < a.Cout;
            const bf16 *src = ok ? a.w + ((int64_t)n * 9 + tap) * a.Cin + c0 + q * 8 : a.w;
            cp_async16(st + Lt::A_BYTES + Lt::off(r, q), src, ok ? 16 : 0);
        }
    };

    // K-direction core matrices 128 B apart, 8-row groups 512 B apart
    const uint32_t lbo = 128u, sbo = 512u;
    constexpr uint32_t idesc = umma_idesc<BN>();
    bool fail = false;
    int issued = 0;  // K chunks whose MMAs were issued (uniform over the CTA)
    // copies run two chunks ahead of the MMAs: the stage refilled at chunk kc
    // held chunk kc-2, whose MMAs were issued an iteration earlier and have
    // normally completed, so the wait below rarely stalls
    constexpr int AHEAD = TSTAGES - 2;
    for (int kc = 0; kc < AHEAD; ++kc) {
        if (kc < nk) load(kc);
        cp_commit();
    }
    for (int kc = 0; kc < nk; ++kc) {
        const int nxt = kc + AHEAD;
        if (nxt < nk) {
            if (kc >= 2 && !nn_mbar_wait(&bars[(kc - 2) % TSTAGES], uint32_t(((kc - 2) / TSTAGES) & 1))) fail = true;
            if (!fail) load(nxt);
        }
        cp_commit();
        cp_wait<AHEAD>();
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        if (__syncthreads_or(fail)) {
            fail = true;
            break;
        }
        tc_fence_after();
        if (tid == 0) {
            const uint32_t base = smem_u32(sm + (kc % TSTAGES) * Lt::STAGE);
#pragma unroll
            for (int ks = 0; ks < TBK; ks += 16) {
                const uint64_t da = umma_desc(base + (ks / 8) * 128, lbo, sbo);
                const uint64_t db = umma_desc(base + Lt::A_BYTES + (ks / 8) * 128, lbo, sbo);
                const uint32_t accum = (kc > 0 || ks > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(idesc), "r"(accum)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&bars[kc % TSTAGES]))
                         : "memory");
        }
        ++issued;
    }
    // every MMA of this CTA is complete once the commit of the last issued
    // chunk arrives (bounded: also on the failure path, before the tensor
    // memory is freed)
    bool done = true;
    if (issued > 0) done = nn_mbar_wait(&bars[(issued - 1) % TSTAGES], uint32_t(((issued - 1) / TSTAGES) & 1));
    cp_wait<0>();
    tc_fence_after();
    if (__syncthreads_or(fail || !done)) {
        if (tid == 0) atomicAdd(&g_nn_timeouts, 1);
    } else {
        // the ring is free now: stage each 32-column slice of the accumulator
        // (thread = pixel row) and write it out row by row with the lanes on
        // consecutive channels, so every store instruction is coalesced
        float *stg = reinterpret_cast<float *>(sm);   // 128 x 33 floats, fits the ring
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 32) {
            uint32_t r[32];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                  "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                  "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                : "r"(taddr)
                : "memory");
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            const int row = warp * 32 + lane;
#pragma unroll
            for (int j = 0; j < 32; ++j) stg[row * 33 + j] = __uint_as_float(r[j]);
            __syncthreads();
            const int n = n0 + c0 + lane;
            if (n < a.Cout) {
                const float bia = a.bias ? a.bias[n] : 0.0f;
#pragma unroll 4
                for (int rr = 0; rr < 32; ++rr) {
                    const int rl = warp * 32 + rr;
                    const int64_t m = m0 + rl;
                    if (m >= M) break;
                    const float z = stg[rl * 33 + lane] + bia;
                    if (a.of) {
                        float *p = a.of + m * a.os + a.oo + n;
                        *p = a.acc ? *p + z : z;
                    }
                    if (a.oa) a.oa[m * a.as + a.ao + n] = __float2bfloat16_rn(a.act ? silu(z) : z);
                }
            }
            __syncthreads();
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN) : "memory");
}

int g_use_tc = 0;          // 0: mma.sync (the default, faster on these layer sizes), 1: tcgen05 (lbm_nn_set_tensor_path)

}  // namespace

#define NN_REQUIRE(cond, ...)                                         \
    do {                                                              \
        if (!(cond)) return lbm::set_error(LBM_ERR_PARAM, __VA_ARGS__); \
    } while (0)

extern "C" int lbm_nn_conv3x3(const void *x, int64_t xs, int32_t xo, const void *w, const float *bias, int32_t B,
                              int32_t H, int32_t W, int32_t Cin, int32_t Cout, float *of, int64_t os, int32_t oo,
                              int32_t accumulate, void *oa, int64_t as, int32_t ao, int32_t act, void *stream)
{
    NN_REQUIRE(x && w, "lbm_nn_conv3x3: x and w are required");
    NN_REQUIRE(of || oa, "lbm_nn_conv3x3: no output");
    NN_REQUIRE(B > 0 && H > 0 && W > 0 && Cout > 0, "lbm_nn_conv3x3: empty shape");
    NN_REQUIRE(Cin > 0 && Cin % CBK == 0, "lbm_nn_conv3x3: Cin must be a positive multiple of 32");
    NN_REQUIRE(xs % 8 == 0 && xo % 8 == 0 && xo >= 0 && xo + Cin <= xs, "lbm_nn_conv3x3: bad input channel stride/offset");
    NN_REQUIRE(aligned16(x) && aligned16(w), "lbm_nn_conv3x3: x and w must be 16-byte aligned");
    NN_REQUIRE(!of || (oo >= 0 && oo + Cout <= os), "lbm_nn_conv3x3: bad FP32 output stride/offset");
    NN_REQUIRE(!oa || (ao >= 0 && ao + Cout <= as), "lbm_nn_conv3x3: bad bf16 output stride/offset");
    NN_REQUIRE(!accumulate || (!bias && !oa), "lbm_nn_conv3x3: accumulate takes no bias and no bf16 output");
    NN_REQUIRE(act == 0 || act == 1, "lbm_nn_conv3x3: act must be 0 or 1");
    ConvArgs a{(const bf16 *)x, xs, xo, (const bf16 *)w, bias, B, H, W, Cin, Cout, of, os, oo, accumulate,
               (bf16 *)oa, as, ao, act};
    const int64_t M = (int64_t)B * H * W;
    cudaStream_t s = (cudaStream_t)stream;
    if (g_use_tc) {
        const int bn = Cout <= 32 ? 32 : (Cout <= 64 ? 64 : (Cout <= 128 ? 128 : 256));
        dim3 grid(unsigned((M + TBM - 1) / TBM), unsigned((Cout + bn - 1) / bn));
        if (bn == 32) {
            cudaFuncSetAttribute(k_conv3x3_tc<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, TcLayout<32>::SMEM);
            k_conv3x3_tc<32><<<grid, TTHREADS, TcLayout<32>::SMEM, s>>>(a);
        } else if (bn == 64) {
            cudaFuncSetAttribute(k_conv3x3_tc<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, TcLayout<64>::SMEM);
            k_conv3x3_tc<64><<<grid, TTHREADS, TcLayout<64>::SMEM, s>>>(a);
        } else if (bn == 128) {
            cudaFuncSetAttribute(k_conv3x3_tc<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, TcLayout<128>::SMEM);
            k_conv3x3_tc<128><<<grid, TTHREADS, TcLayout<128>::SMEM, s>>>(a);
        } else {
            // 256 TMEM columns per CTA; its 97 KB of shared memory keep at most
            // two CTAs on an SM, within the SM's 512 columns
            cudaFuncSetAttribute(k_conv3x3_tc<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, TcLayout<256>::SMEM);
            k_conv3x3_tc<256><<<grid, TTHREADS, TcLayout<256>::SMEM, s>>>(a);
        }
        return launched("lbm_nn_conv3x3 (tcgen05)");
    }
    if (Cout <= 32) {
        dim3 grid(unsigned((M + CBM - 1) / CBM), unsigned((Cout + 31) / 32));
        k_conv3x3<32><<<grid, kThreads, 0, s>>>(a);
    } else {
        dim3 grid(unsigned((M + CBM - 1) / CBM), unsigned((Cout + 63) / 64));
        k_conv3x3<64><<<grid, kThreads, 0, s>>>(a);
    }
    return launched("lbm_nn_conv3x3");
}

extern "C" int lbm_nn_flip_weights(const void *w, void *wt, int32_t Cout, int32_t Cin, void *stream)
{
    NN_REQUIRE(w && wt && Cout > 0 && Cin > 0, "lbm_nn_flip_weights: bad arguments");
    const int64_t n = (int64_t)Cout * 9 * Cin;
    k_flip<<<blocks_for(n), kThreads, 0, (cudaStream_t)stream>>>((const bf16 *)w, (bf16 *)wt, Cout, Cin);
    return launched("lbm_nn_flip_weights");
}

extern "C" int64_t lbm_nn_wgrad_workspace(int32_t B, int32_t H, int32_t W, int32_t Cin, int32_t Cout)
{
    if (B <= 0 || H <= 0 || W <= 0 || Cin <= 0 || Cout <= 0) return 0;
    const WgradPlan pl = wgrad_plan(B, H, W, Cin, Cout);
    return (int64_t)pl.S * Cout * 9 * Cin;
}

extern "C" int lbm_nn_conv3x3_wgrad(const void *dz, const void *x, int64_t xs, int32_t xo, int32_t B, int32_t H,
                                    int32_t W, int32_t Cin, int32_t Cout, float *ws, int64_t ws_elems, float *dw,
                                    void *stream)
{
    NN_REQUIRE(dz && x && ws && dw, "lbm_nn_conv3x3_wgrad: NULL pointer");
    NN_REQUIRE(B > 0 && H > 0 && W > 0, "lbm_nn_conv3x3_wgrad: empty shape");
    NN_REQUIRE(Cin > 0 && Cin % WBN == 0, "lbm_nn_conv3x3_wgrad: Cin must be a positive multiple of 32");
    NN_REQUIRE(Cout > 0 && Cout % 8 == 0, "lbm_nn_conv3x3_wgrad: Cout must be a positive multiple of 8");
    NN_REQUIRE(xs % 8 == 0 && xo % 8 == 0 && xo >= 0 && xo + Cin <= xs, "lbm_nn_conv3x3_wgrad: bad channel stride/offset");
    NN_REQUIRE(aligned16(dz) && aligned16(x), "lbm_nn_conv3x3_wgrad: dz and x must be 16-byte aligned");
    const WgradPlan pl = wgrad_plan(B, H, W, Cin, Cout);
    const int64_t n = (int64_t)Cout * 9 * Cin;
    NN_REQUIRE(ws_elems >= (int64_t)pl.S * n, "lbm_nn_conv3x3_wgrad: workspace too small (%lld < %lld)",
               (long long)ws_elems, (long long)pl.S * n);
    cudaStream_t s = (cudaStream_t)stream;
    dim3 grid(unsigned(9 * Cin / WBN), unsigned((Cout + WBM - 1) / WBM), unsigned(pl.S));
    k_wgrad<<<grid, kThreads, 0, s>>>((const bf16 *)dz, (const bf16 *)x, xs, xo, B, H, W, Cin, Cout, pl.per, ws);
    k_sum_splits<<<blocks_for(n), kThreads, 0, s>>>(ws, pl.S, n, dw);
    return launched("lbm_nn_conv3x3_wgrad", 2);
}

extern "C" int64_t lbm_nn_colsum_workspace(int64_t P, int32_t C)
{
    if (P <= 0 || C <= 0) return 0;
    return ((P + kColRows - 1) / kColRows) * C;
}

extern "C" int lbm_nn_colsum(const void *a, int64_t P, int32_t C, float *ws, float *out, void *stream)
{
    NN_REQUIRE(a && ws && out && P > 0 && C > 0, "lbm_nn_colsum: bad arguments");
    const int64_t S = (P + kColRows - 1) / kColRows;
    cudaStream_t s = (cudaStream_t)stream;
    k_colsum<<<dim3(unsigned((C + 31) / 32), unsigned(S)), kThreads, 0, s>>>((const bf16 *)a, P, C, ws);
    k_sum_splits<<<blocks_for(C), kThreads, 0, s>>>(ws, int(S), C, out);
    return launched("lbm_nn_colsum", 2);
}

extern "C" int lbm_nn_silu_backward(const float *da, int64_t das, int32_t dao, const float *z, int64_t P, int32_t C,
                                    void *dz, void *stream)
{
    NN_REQUIRE(da && z && dz && P > 0 && C > 0 && dao >= 0 && dao + C <= das, "lbm_nn_silu_backward: bad arguments");
    k_silu_bwd<<<blocks_for(P * C), kThreads, 0, (cudaStream_t)stream>>>(da, das, dao, z, P, C, (bf16 *)dz);
    return launched("lbm_nn_silu_backward");
}

extern "C" int lbm_nn_pool2(const void *x, int64_t xs, int32_t xo, int32_t B, int32_t H, int32_t W, int32_t C,
                            void *y, int64_t ys, int32_t yo, void *stream)
{
    NN_REQUIRE(x && y && B > 0 && H > 1 && W > 1 && H % 2 == 0 && W % 2 == 0 && C > 0,
               "lbm_nn_pool2: bad shape (H, W even)");
    NN_REQUIRE(xo >= 0 && xo + C <= xs && yo >= 0 && yo + C <= ys, "lbm_nn_pool2: bad channel stride/offset");
    const int64_t n = (int64_t)B * (H / 2) * (W / 2) * C;
    k_pool2<<<blocks_for(n), kThreads, 0, (cudaStream_t)stream>>>((const bf16 *)x, xs, xo, B, H, W, C, (bf16 *)y, ys, yo);
    return launched("lbm_nn_pool2");
}

extern "C" int lbm_nn_pool2_backward(const float *dy, int64_t dys, int32_t dyo, int32_t B, int32_t H, int32_t W,
                                     int32_t C, float *dx, int64_t dxs, int32_t dxo, void *stream)
{
    NN_REQUIRE(dy && dx && B > 0 && H > 1 && W > 1 && H % 2 == 0 && W % 2 == 0 && C > 0,
               "lbm_nn_pool2_backward: bad shape");
    NN_REQUIRE(dyo >= 0 && dyo + C <= dys && dxo >= 0 && dxo + C <= dxs, "lbm_nn_pool2_backward: bad stride/offset");
    const int64_t n = (int64_t)B * H * W * C;
    k_pool2_bwd<<<blocks_for(n), kThreads, 0, (cudaStream_t)stream>>>(dy, dys, dyo, B, H, W, C, dx, dxs, dxo);
    return launched("lbm_nn_pool2_backward");
}

extern "C" int lbm_nn_up2(const void *x, int64_t xs, int32_t xo, int32_t B, int32_t h, int32_t w, int32_t C, void *y,
                          int64_t ys, int32_t yo, void *stream)
{
    NN_REQUIRE(x && y && B > 0 && h > 0 && w > 0 && C > 0, "lbm_nn_up2: bad shape");
    NN_REQUIRE(xo >= 0 && xo + C <= xs && yo >= 0 && yo + C <= ys, "lbm_nn_up2: bad channel stride/offset");
    const int64_t n = (int64_t)B * 4 * h * w * C;
    k_up2<<<blocks_for(n), kThreads, 0, (cudaStream_t)stream>>>((const bf16 *)x, xs, xo, B, h, w, C, (bf16 *)y, ys, yo);
    return launched("lbm_nn_up2");
}

extern "C" int lbm_nn_up2_backward(const float *dy, int64_t dys, int32_t dyo, int32_t B, int32_t h, int32_t w,
                                   int32_t C, float *dx, int64_t dxs, int32_t dxo, int32_t accumulate, void *stream)
{
    NN_REQUIRE(dy && dx && B > 0 && h > 0 && w > 0 && C > 0, "lbm_nn_up2_backward: bad shape");
    NN_REQUIRE(dyo >= 0 && dyo + C <= dys && dxo >= 0 && dxo + C <= dxs, "lbm_nn_up2_backward: bad stride/offset");
    const int64_t n = (int64_t)B * h * w * C;
    k_up2_bwd<<<blocks_for(n), kThreads, 0, (cudaStream_t)stream>>>(dy, dys, dyo, B, h, w, C, dx, dxs, dxo, accumulate);
    return launched("lbm_nn_up2_backward");
}

extern "C" int lbm_nn_head(const void *a, int64_t as, int32_t ao, const void *wh, const float *bh, int64_t P, int32_t C,
                           int32_t J, float *y, void *stream)
{
    NN_REQUIRE(a && wh && y && P > 0 && C > 0 && J > 0 && J <= kMaxJ, "lbm_nn_head: bad arguments (J <= 8)");
    NN_REQUIRE(ao >= 0 && ao + C <= as, "lbm_nn_head: bad channel stride/offset");
    k_head<<<blocks_for(P), kThreads, 0, (cudaStream_t)stream>>>((const bf16 *)a, as, ao, (const bf16 *)wh, bh, P, C, J, y);
    return launched("lbm_nn_head");
}

extern "C" int64_t lbm_nn_head_workspace(int64_t P, int32_t C, int32_t J)
{
    if (P <= 0 || C <= 0 || J <= 0) return 0;
    // per-split partials, then one row for their sums
    return ((P + kHeadRows - 1) / kHeadRows + 1) * ((int64_t)J * C + J);
}

extern "C" int lbm_nn_head_backward(const float *dy, const void *a, int64_t as, int32_t ao, const void *wh, int64_t P,
                                    int32_t C, int32_t J, float *da, int64_t das, int32_t dao, float *ws,
                                    int64_t ws_elems, float *dwh, float *dbh, void *stream)
{
    NN_REQUIRE(dy && a && wh && da && ws && dwh && dbh && P > 0 && C > 0 && J > 0 && J <= kMaxJ,
               "lbm_nn_head_backward: bad arguments");
    NN_REQUIRE(ao >= 0 && ao + C <= as && dao >= 0 && dao + C <= das, "lbm_nn_head_backward: bad stride/offset");
    const int64_t S = (P + kHeadRows - 1) / kHeadRows;
    const int items = J * C + J;
    NN_REQUIRE(ws_elems >= (S + 1) * items, "lbm_nn_head_backward: workspace too small");
    cudaStream_t s = (cudaStream_t)stream;
    k_head_bwd_da<<<blocks_for(P * C), kThreads, 0, s>>>(dy, (const bf16 *)wh, P, C, J, da, das, dao);
    k_head_bwd_w<<<unsigned(S), kThreads, 0, s>>>(dy, (const bf16 *)a, as, ao, P, C, J, ws);
    // each split's partials hold dwh (J*C) then dbh (J); their ordered sums go after them
    k_sum_splits<<<blocks_for(items), kThreads, 0, s>>>(ws, int(S), items, ws + S * items);
    int st = launched("lbm_nn_head_backward", 3);
    if (st) return st;
    cudaError_t e = cudaMemcpyAsync(dwh, ws + S * items, sizeof(float) * J * C, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dbh, ws + S * items + (int64_t)J * C, sizeof(float) * J, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return lbm::set_error(LBM_ERR_CUDA, "lbm_nn_head_backward: %s", cudaGetErrorString(e));
    return LBM_OK;
}

extern "C" int64_t lbm_nn_mse_workspace(int64_t P, int32_t J)
{
    (void)P;
    (void)J;
    return kMseBlocks;
}

extern "C" int lbm_nn_mse(const float *y, const float *t, const float *cw, int64_t P, int32_t J, float *dy, float *ws,
                          int64_t ws_elems, float *loss, void *stream)
{
    NN_REQUIRE(y && t && dy && ws && loss && P > 0 && J > 0, "lbm_nn_mse: bad arguments");
    NN_REQUIRE(ws_elems >= kMseBlocks, "lbm_nn_mse: workspace too small");
    cudaStream_t s = (cudaStream_t)stream;
    k_mse<<<kMseBlocks, kThreads, 0, s>>>(y, t, cw, P, J, dy, ws);
    k_mse_final<<<1, 32, 0, s>>>(ws, kMseBlocks, P * J, loss);
    return launched("lbm_nn_mse", 2);
}

extern "C" int lbm_nn_adam(float *p, void *pb, const float *g, float *m, float *v, int64_t n, float lr, float b1,
                           float b2, float eps, float c1, float c2, float wd, void *stream)
{
    NN_REQUIRE(p && g && m && v && n > 0, "lbm_nn_adam: bad arguments");
    NN_REQUIRE(c1 > 0.0f && c2 > 0.0f, "lbm_nn_adam: bias corrections must be > 0");
    k_adam<<<blocks_for(n), kThreads, 0, (cudaStream_t)stream>>>(p, (bf16 *)pb, g, m, v, n, lr, b1, b2, eps, c1, c2, wd);
    return launched("lbm_nn_adam");
}

extern "C" int lbm_nn_to_bf16(const float *x, void *y, int64_t n, void *stream)
{
    NN_REQUIRE(x && y && n > 0, "lbm_nn_to_bf16: bad arguments");
    k_to_bf16<<<blocks_for(n), kThreads, 0, (cudaStream_t)stream>>>(x, (bf16 *)y, n);
    return launched("lbm_nn_to_bf16");
}

extern "C" int lbm_nn_set_tensor_path(int32_t path)
{
    NN_REQUIRE(path == 0 || path == 1, "lbm_nn_set_tensor_path: path must be 0 (mma.sync) or 1 (tcgen05)");
    g_use_tc = path == 1;
    return LBM_OK;
}

extern "C" int lbm_nn_get_tensor_path(void) { return g_use_tc ? 1 : 0; }

extern "C" int lbm_nn_timeouts(int32_t *count, int32_t reset)
{
    NN_REQUIRE(count, "lbm_nn_timeouts: count is NULL");
    int v = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_nn_timeouts, sizeof v);
    if (e == cudaSuccess && reset) {
        const int zero = 0;
        e = cudaMemcpyToSymbol(g_nn_timeouts, &zero, sizeof zero);
    }
    if (e != cudaSuccess) return lbm::set_error(LBM_ERR_CUDA, "lbm_nn_timeouts: %s", cudaGetErrorString(e));
    *count = v;
    return LBM_OK;
}
