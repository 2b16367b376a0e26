// FP64 reductions and layout conversions.
//
// Reductions are deterministic: a fixed grid of blocks accumulates per-thread
// partial sums with a grid-stride loop, reduces them with warp shuffles and
// shared memory into one partial per block, and a single block then sums the
// partials in block order.  The result does not depend on timing, only on
// the grid size (fixed by the node count).
#include <math.h>
#include <stdint.h>

#include "lbm_internal.h"

namespace lbm {

int64_t g_launches = 0;

static constexpr int kRedBlocks = 592;  // 4 x 148 SMs
static constexpr int kRedThreads = 256;

template <int NV>
__device__ __forceinline__ void block_reduce_store(double (&acc)[NV], double *out)
{
    __shared__ double sh[NV][kRedThreads / 32];
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
            double v = lane < kRedThreads / 32 ? sh[c][lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) out[c] = v;
        }
    }
}

// sum partials[nb][NV] in block order -> res[0..NV-1]
template <int NV>
__global__ void k_final(const double *__restrict__ partials, int nb, double *__restrict__ res)
{
    double acc[NV];
#pragma unroll
    for (int c = 0; c < NV; ++c) acc[c] = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x)
#pragma unroll
        for (int c = 0; c < NV; ++c) acc[c] += partials[(int64_t)b * NV + c];
    block_reduce_store<NV>(acc, res);
}

// check(): 2M:755-805 / 3M:1027-1082.  sums of |du|^2, |u|^2, dT^2, T^2, then
// the previous fields take the current ones.  Block `blk` of kRedBlocks.
__device__ __forceinline__ void check_block(const Geo &G, const Bufs &B, int blk)
{
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    const int64_t stride = (int64_t)kRedBlocks * blockDim.x;
    // a slab: its own rows (2D) or z-slices (3D) only
    const bool d2 = G.dim == 2;
    const int lo = d2 ? G.jlo : G.klo, hi = d2 ? G.jhi : G.khi;
    const bool part = lo > 0 || hi < (d2 ? G.ny : G.nz);
    const int64_t layer = d2 ? (int64_t)G.nx : (int64_t)G.nx * G.ny;
    for (int64_t n = (int64_t)blk * blockDim.x + threadIdx.x; n < G.nnode; n += stride) {
        if (part) {
            const int64_t l = n / layer;
            if (l < lo || l >= hi) continue;
        }
        const double u = B.u[n], v = B.v[n], T = B.T[n];
        const double du = u - B.up[n], dv = v - B.vp[n], dT = T - B.Tp[n];
        if (G.dim == 2) {
            acc[0] += du * du + dv * dv;
            acc[1] += u * u + v * v;
        } else {
            const double w = B.w[n];
            const double dw = w - B.wp[n];
            acc[0] += du * du + dv * dv + dw * dw;
            acc[1] += u * u + v * v + w * w;
            B.wp[n] = w;
        }
        acc[2] += dT * dT;
        acc[3] += T * T;
        B.up[n] = u;
        B.vp[n] = v;
        B.Tp[n] = T;
    }
    block_reduce_store<4>(acc, B.partials + (int64_t)blk * 4);
}

__global__ void __launch_bounds__(kRedThreads) k_check(const Geo G, const Bufs B) { check_block(G, B, blockIdx.x); }

cudaError_t reduce_check(const Geo &g, const Bufs &b, cudaStream_t s)
{
    k_check<<<kRedBlocks, kRedThreads, 0, s>>>(g, b);
    k_final<4><<<1, kRedThreads, 0, s>>>(b.partials, kRedBlocks, b.scal + 0);
    g_launches += 2;
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// the stop test of a run on the device (lbm_run, lbm_batch_run)
// ---------------------------------------------------------------------------
// The sums are those of k_check / k_final (same blocks, same order), so the
// residuals are bit-identical to lbm_check's; errorU = sqrt(sum du^2) /
// sqrt(sum u^2), errorT likewise (2M:784, 798), and the loop continues while
// errorU > eps or errorT > eps (2M:307).
__device__ void run_decide(RunCtl *c, const double *sum, int period)
{
    const double eu = sqrt(sum[0]) / sqrt(sum[1]), et = sqrt(sum[2]) / sqrt(sum[3]);
    c->errU = eu;
    c->errT = et;
    c->steps += period;
    const bool sums_finite = isfinite(sum[0]) && isfinite(sum[1]) && isfinite(sum[2]) && isfinite(sum[3]);
    if (!c->stop_bad) {
        // single cavity (lbm_run): non-finite sums end the run as an error
        if (!sums_finite) {
            c->status = -2;
            c->active = 0;
        } else if (!(eu > c->eps || et > c->eps)) {
            c->status = 1;
            c->active = 0;
        }
        ++c->checks;
        return;
    }
    // batch member: a residual that stops being finite, or grows past growth x
    // its smallest value in this run, stops the member (status -1)
    const double r = eu < et ? et : eu;
    const bool bad = !sums_finite || !isfinite(r) || (c->growth > 0.0 && c->checks >= 2 && r > c->growth * c->best);
    if (!sums_finite && !(c->growth > 0.0)) {
        c->status = -2;
        c->active = 0;
        return;
    }
    ++c->checks;
    c->best = r < c->best ? r : c->best;
    if (bad) {
        c->status = -1;
        c->active = 0;
    } else if (!(eu > c->eps || et > c->eps)) {
        c->status = 1;
        c->active = 0;
    }
}

// the final sum of k_final<4>, then the decision, by one block
__device__ __forceinline__ void run_final_block(const Bufs &B, int period)
{
    __shared__ double sum[4];
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < kRedBlocks; b += blockDim.x)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[c] += B.partials[(int64_t)b * 4 + c];
    block_reduce_store<4>(acc, sum);
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int c = 0; c < 4; ++c) B.scal[c] = sum[c];
        run_decide(B.ctl, sum, period);
    }
}

__global__ void __launch_bounds__(kRedThreads) k_run_check(const Geo G, const Bufs B)
{
    if (!B.ctl->active) return;
    check_block(G, B, blockIdx.x);
}

__global__ void __launch_bounds__(kRedThreads) k_run_final(const Bufs B, int period)
{
    if (!B.ctl->active) return;
    run_final_block(B, period);
}

cudaError_t run_check(const Geo &g, const Bufs &b, int period, cudaStream_t s)
{
    k_run_check<<<kRedBlocks, kRedThreads, 0, s>>>(g, b);
    k_run_final<<<1, kRedThreads, 0, s>>>(b, period);
    g_launches += 2;
    return cudaGetLastError();
}

// batch: blockIdx.y (check) / blockIdx.x (final) picks the member idx[...]
__global__ void __launch_bounds__(kRedThreads) k_run_check_batch(const BatchDev D, const int *idx)
{
    const int m = idx[blockIdx.y];
    const Bufs &B = D.bufs[m];
    if (!B.ctl->active) return;
    check_block(D.geo[m], B, blockIdx.x);
}

__global__ void __launch_bounds__(kRedThreads) k_run_final_batch(const BatchDev D, const int *idx, int period)
{
    const Bufs &B = D.bufs[idx[blockIdx.x]];
    if (!B.ctl->active) return;
    run_final_block(B, period);
}

cudaError_t run_check_batch(const BatchDev &D, const int *idx, int n, int period, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    k_run_check_batch<<<dim3(kRedBlocks, n), kRedThreads, 0, s>>>(D, idx);
    k_run_final_batch<<<n, kRedThreads, 0, s>>>(D, idx, period);
    g_launches += 2;
    return cudaGetLastError();
}

// d/dn at the wall of the quadratic through (xw,Tw), (x1,T1), (x2,T2); the
// same expression as the CPU restatement's ora_wall_gradient
__device__ __forceinline__ double wall_gradient(double xw, double Tw, double x1, double T1, double x2, double T2)
{
    const double d0 = ((xw - x1) + (xw - x2)) / ((xw - x1) * (xw - x2));
    const double d1 = (xw - x2) / ((x1 - xw) * (x1 - x2));
    const double d2 = (xw - x1) / ((x2 - xw) * (x2 - x1));
    return d0 * Tw + d1 * T1 + d2 * T2;
}

// Wall-averaged Nusselt numbers: hot wall at the low end of the heated axis
// (x in 2D, y in 3D), cold wall at the high end.
__global__ void __launch_bounds__(kRedThreads) k_nusselt(const Geo G, const Bufs B)
{
    double acc[3] = {0.0, 0.0, 0.0};
    const double scale = -(G.length_LB - 1.0) / (G.Thot - G.Tcold);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    if (G.dim == 2) {
        const double *x = G.coord[0];
        const int nx = G.nx;
        const double xlo = x[1] - 0.5 * G.dt, xhi = x[nx] + 0.5 * G.dt;
        for (int64_t j = G.jlo + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < G.jhi; j += stride) {
            const double *T = B.T + j * nx;
            const double gh = wall_gradient(xlo, G.Thot, x[1], T[0], x[2], T[1]);
            const double gc = wall_gradient(xhi, G.Tcold, x[nx], T[nx - 1], x[nx - 1], T[nx - 2]);
            const double wy = G.cellw[1][j];
            acc[0] += scale * gh * wy;
            acc[1] += scale * gc * wy;
            acc[2] += wy;
        }
    } else {
        const double *y = G.coord[1];
        const int nx = G.nx, ny = G.ny;
        const double ylo = y[1] - 0.5 * G.dt, yhi = y[ny] + 0.5 * G.dt;
        const int64_t nwall = (int64_t)nx * (G.khi - G.klo);  // a slab's own z-slices
        for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nwall; t += stride) {
            const int i = int(t % nx), k = G.klo + int(t / nx);
            const double *T = B.T + (int64_t)k * nx * ny + i;
            const double gh = wall_gradient(ylo, G.Thot, y[1], T[0], y[2], T[nx]);
            const double gc = wall_gradient(yhi, G.Tcold, y[ny], T[(int64_t)(ny - 1) * nx],
                                            y[ny - 1], T[(int64_t)(ny - 2) * nx]);
            const double a = G.cellw[0][i] * G.cellw[2][k];
            acc[0] += scale * gh * a;
            acc[1] += scale * gc * a;
            acc[2] += a;
        }
    }
    block_reduce_store<3>(acc, B.partials + (int64_t)blockIdx.x * 3);
}

cudaError_t reduce_nusselt(const Geo &g, const Bufs &b, cudaStream_t s)
{
    k_nusselt<<<kRedBlocks, kRedThreads, 0, s>>>(g, b);
    k_final<3><<<1, kRedThreads, 0, s>>>(b.partials, kRedBlocks, b.scal + 4);
    g_launches += 2;
    return cudaGetLastError();
}

// mass = sum(rho dV), energy = sum(T dV)
__global__ void __launch_bounds__(kRedThreads) k_sums(const Geo G, const Bufs B)
{
    double acc[2] = {0.0, 0.0};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < G.nnode; n += stride) {
        const int i = int(n % G.nx);
        const int j = int((n / G.nx) % G.ny);
        const int k = int(n / ((int64_t)G.nx * G.ny));
        if (G.dim == 2 ? (j < G.jlo || j >= G.jhi) : (k < G.klo || k >= G.khi)) continue;  // a slab's ghosts
        const double vol = G.cellw[0][i] * G.cellw[1][j] * (G.dim == 3 ? G.cellw[2][k] : 1.0);
        acc[0] += B.rho[n] * vol;
        acc[1] += B.T[n] * vol;
    }
    block_reduce_store<2>(acc, B.partials + (int64_t)blockIdx.x * 2);
}

cudaError_t reduce_sums(const Geo &g, const Bufs &b, cudaStream_t s)
{
    k_sums<<<kRedBlocks, kRedThreads, 0, s>>>(g, b);
    k_final<2><<<1, kRedThreads, 0, s>>>(b.partials, kRedBlocks, b.scal + 7);
    g_launches += 2;
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// layout conversions between the Fortran f(0:Q-1, nx, ny[, nz]) order and the
// structure-of-arrays planes
// ---------------------------------------------------------------------------
// Reduced-precision storage keeps deviations: f - w (rho0 = 1) and g - wT*Tc
// with Tc the conduction profile at the node (tc_value).  Node n is packed,
// x fastest; the heated axis is x in 2D and y in 3D.
__device__ __forceinline__ double shift_of(const Geo &G, int q, int64_t n)
{
    if (G.dim == 2) {
        if (q < 9) return q == 0 ? 4.0 / 9.0 : (q < 5 ? 1.0 / 9.0 : 1.0 / 36.0);
        return (q == 9 ? 0.5 : 0.125) * tc_value(G, int(n % G.nx));
    }
    if (q < 19) return q == 0 ? 1.0 / 3.0 : (q < 7 ? 1.0 / 18.0 : 1.0 / 36.0);
    return (q == 19 ? 0.5 : 1.0 / 12.0) * tc_value(G, int((n / G.nx) % G.ny));
}

__device__ __forceinline__ int64_t pidx(const Geo &G, int64_t n)
{
    const int i = int(n % G.nx);
    const int j = int((n / G.nx) % G.ny);
    const int k = int(n / ((int64_t)G.nx * G.ny));
    return (int64_t)k * G.slab + (int64_t)j * G.pitch + i;
}

template <int ST>
__global__ void k_aos_to_planes(const Geo G, int q0, int nq, const double *__restrict__ aos, void *pop)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= G.nnode * nq) return;
    const int64_t n = e / nq;
    const int q = q0 + int(e % nq);
    const int64_t dst = (int64_t)q * G.plane + pidx(G, n);
    const double val = aos[e];
    if (ST == kF64) ((double *)pop)[dst] = val;
    else ((float *)pop)[dst] = float(val - shift_of(G, q, n));
}

template <int ST>
__global__ void k_planes_to_aos(const Geo G, int q0, int nq, const void *pop, double *__restrict__ aos)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= G.nnode * nq) return;
    const int64_t n = e / nq;
    const int q = q0 + int(e % nq);
    const int64_t src = (int64_t)q * G.plane + pidx(G, n);
    double val;
    if (ST == kF64) val = ((const double *)pop)[src];
    else val = double(((const float *)pop)[src]) + shift_of(G, q, n);
    aos[e] = val;
}

cudaError_t aos_to_planes(const Geo &g, int store, int q0, int nq, const double *aos, void *pop, cudaStream_t s)
{
    const int64_t n = g.nnode * nq;
    const unsigned nb = unsigned((n + 255) / 256);
    if (store == kF64) k_aos_to_planes<kF64><<<nb, 256, 0, s>>>(g, q0, nq, aos, pop);
    else k_aos_to_planes<kF32><<<nb, 256, 0, s>>>(g, q0, nq, aos, pop);
    ++g_launches;
    return cudaGetLastError();
}

cudaError_t planes_to_aos(const Geo &g, int store, int q0, int nq, const void *pop, double *aos, cudaStream_t s)
{
    const int64_t n = g.nnode * nq;
    const unsigned nb = unsigned((n + 255) / 256);
    if (store == kF64) k_planes_to_aos<kF64><<<nb, 256, 0, s>>>(g, q0, nq, pop, aos);
    else k_planes_to_aos<kF32><<<nb, 256, 0, s>>>(g, q0, nq, pop, aos);
    ++g_launches;
    return cudaGetLastError();
}

// Populations of one storage converted to another on the device (the value
// of a node's population is the same up to the target's rounding; deviation
// forms are undone and redone through shift_of).
template <int SRC, int DST>
__global__ void k_convert_planes(const Geo G, int nq, const void *src, void *dst)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= G.nnode * nq) return;
    const int64_t n = e / nq;
    const int q = int(e % nq);
    const int64_t a = (int64_t)q * G.plane + pidx(G, n);
    double val;
    if (SRC == kF64) val = ((const double *)src)[a];
    else val = double(((const float *)src)[a]) + shift_of(G, q, n);
    if (DST == kF64) ((double *)dst)[a] = val;
    else ((float *)dst)[a] = float(val - shift_of(G, q, n));
}

template <int SRC>
static void convert_from(const Geo &g, int dst_store, int nq, const void *src, void *dst, unsigned nb, cudaStream_t s)
{
    if (dst_store == kF64) k_convert_planes<SRC, kF64><<<nb, 256, 0, s>>>(g, nq, src, dst);
    else k_convert_planes<SRC, kF32><<<nb, 256, 0, s>>>(g, nq, src, dst);
}

// the carried force, one compute-type value per cell of a plane
__global__ void k_convert_force(int64_t n, int src8, int dst8, const void *src, void *dst)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const double v = src8 ? ((const double *)src)[e] : double(((const float *)src)[e]);
    if (dst8) ((double *)dst)[e] = v;
    else ((float *)dst)[e] = float(v);
}

cudaError_t convert_state(const Geo &g, int src_store, int dst_store, int nq, const void *pop_src, void *pop_dst,
                          const void *F_src, void *F_dst, cudaStream_t s)
{
    const int64_t n = g.nnode * nq;
    const unsigned nb = unsigned((n + 255) / 256);
    if (src_store == kF64) convert_from<kF64>(g, dst_store, nq, pop_src, pop_dst, nb, s);
    else convert_from<kF32>(g, dst_store, nq, pop_src, pop_dst, nb, s);
    k_convert_force<<<unsigned((g.plane + 255) / 256), 256, 0, s>>>(g.plane, src_store == kF64, dst_store == kF64,
                                                                    F_src, F_dst);
    g_launches += 2;
    return cudaGetLastError();
}

// macroscopic fields of loaded populations: rho = sum f, T = sum g, momentum
// over rho, with half the buoyancy force gbeta*T*rho of this state added to
// the gravity-axis velocity (v in 2D, w in 3D), as macro_u does (2M:734-735)
template <int ST>
__global__ void k_macro_from_pops(const Geo G, const void *pop, const Bufs B)
{
    const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= G.nnode) return;
    const int64_t id = pidx(G, n);
    const int Q = G.dim == 2 ? 9 : 19, QT = G.dim == 2 ? 5 : 7;
    auto ld = [&](int q) -> double {
        const int64_t a = (int64_t)q * G.plane + id;
        if (ST == kF64) return ((const double *)pop)[a];
        return double(((const float *)pop)[a]) + shift_of(G, q, n);
    };
    const int ex2[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
    const int ey2[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
    const int ex3[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
    const int ey3[19] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1};
    const int ez3[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};
    double rho = 0.0, jx = 0.0, jy = 0.0, jz = 0.0, T = 0.0;
    for (int q = 0; q < Q; ++q) {
        const double fq = ld(q);
        rho += fq;
        jx += (G.dim == 2 ? ex2[q] : ex3[q]) * fq;
        jy += (G.dim == 2 ? ey2[q] : ey3[q]) * fq;
        if (G.dim == 3) jz += ez3[q] * fq;
    }
    for (int q = 0; q < QT; ++q) T += ld(Q + q);
    const double F = G.gbeta * T * rho;
    B.rho[n] = rho;
    B.T[n] = T;
    B.u[n] = jx / rho;
    if (G.dim == 2) {
        B.v[n] = (jy + 0.5 * G.dt * F) / rho;
    } else {
        B.v[n] = jy / rho;
        B.w[n] = (jz + 0.5 * G.dt * F) / rho;
    }
}

cudaError_t macro_from_pops(const Geo &g, int store, const void *pop, const Bufs &b, cudaStream_t s)
{
    const unsigned nb = unsigned((g.nnode + 255) / 256);
    if (store == kF64) k_macro_from_pops<kF64><<<nb, 256, 0, s>>>(g, pop, b);
    else k_macro_from_pops<kF32><<<nb, 256, 0, s>>>(g, pop, b);
    ++g_launches;
    return cudaGetLastError();
}

}  // namespace lbm
