// Thermal LBM time-step kernels for sm_100a.
//
// This file is compiled twice:
//   LBM_NS=fast                      multiply-add contraction on, constant
//                                    divisions turned into reciprocal products;
//   LBM_NS=exact, LBM_EXACT=1, --fmad=false
//                                    every expression in the reference's operand
//                                    order with its divisions, no contraction:
//                                    FP64 results are bit-identical to the CPU
//                                    restatement of the reference.
//
// One fused kernel per time step replaces the reference's chain of sweeps
// collision_U -> collision_T -> update -> interpolate -> bounceback_u ->
// bounceback_T -> macro_u -> macro_t (natural-convection_2dim_mono.f90:309-325,
// natural-convection_3dim_mono.f90:375-391) with a pull formulation:
//   read post-collision populations of the previous step around the node,
//   interpolate (ISLBM streaming, 2M:591-660 / 3M:751-876),
//   apply the wall rules of the node (2B:731-801 / 3B:1053-1197),
//   form rho, u, T (2M:726-753 / 3M:988-1025) with the buoyancy force carried
//   from the previous collision,
//   collide (2M:431-569 / 3M:445-730) and write the new post-collision
//   populations and force.
// Populations live in structure-of-arrays planes: plane q holds population q of
// every node, rows of `pitch` elements, z-planes of `slab` elements.  Planes
// 0..Q-1 are f, Q..Q+QT-1 are g.
#include <cuda.h>
#include <stdint.h>

#include "lbm_internal.h"

#ifndef LBM_EXACT
#define LBM_EXACT 0
#endif

namespace lbm {
namespace LBM_NS {

// ---------------------------------------------------------------------------
// storage traits
// ---------------------------------------------------------------------------
template <int ST> struct Tr;
// kShift: flow populations stored and computed as f - w (deviation form);
// kDevT: thermal populations stored and computed as g - wT*Tc, Tc the
// conduction profile (tc_value)
template <> struct Tr<kF64> { using S = double; using C = double; static constexpr bool kShift = false, kDevT = false; };
template <> struct Tr<kF32> { using S = float;  using C = float;  static constexpr bool kShift = true, kDevT = true; };

__device__ __forceinline__ double tocomp(double x) { return x; }
__device__ __forceinline__ float tocomp(float x) { return x; }

template <class S> __device__ __forceinline__ S fromcomp(double x);
template <> __device__ __forceinline__ double fromcomp<double>(double x) { return x; }
template <class S> __device__ __forceinline__ S fromcompf(float x);
template <> __device__ __forceinline__ float fromcompf<float>(float x) { return x; }

template <class S, class C> __device__ __forceinline__ S tostore(C x);
template <> __device__ __forceinline__ double tostore<double, double>(double x) { return x; }
template <> __device__ __forceinline__ float tostore<float, float>(float x) { return x; }

// Reduced-precision storage (FP32) keeps f - w*rho0 (rho0 = 1)
// and g - wT*Tc (Tc: the linear conduction profile between the isothermal
// walls), and both stay in that deviation form through streaming and
// collision:
//   * velocities are small differences of O(w) populations: in FP32
//     arithmetic on the full populations their rounding (~1e-8) would hold the
//     check() residual above ~1e-5.  The interpolation weights sum to one and
//     bounce-back pairs directions of equal weight, so both commute with the
//     shift; the collision subtracts the rest state's moments;
//   * the wall Nusselt number amplifies temperature errors next to the wall
//     by ~L_LB/Nu (~400), so ~1e-7 of absolute rounding in T ~ 1 would bias
//     Nu by 1e-4.  Quadratic interpolation is exact on the linear profile, so
//     streaming the deviation only adds -wT e.grad(Tc) dt per direction; the
//     walls and the collision take Tc into their equilibria.
// lattice weights used as storage shifts
__device__ __forceinline__ float wU2(int q) { return q == 0 ? 4.0f / 9.0f : (q < 5 ? 1.0f / 9.0f : 1.0f / 36.0f); }
__device__ __forceinline__ float wT2(int q) { return q == 0 ? 0.5f : 0.125f; }
__device__ __forceinline__ float wU3(int q) { return q == 0 ? 1.0f / 3.0f : (q < 7 ? 1.0f / 18.0f : 1.0f / 36.0f); }
__device__ __forceinline__ float wT3(int q) { return q == 0 ? 0.5f : 1.0f / 12.0f; }

// division by a literal: a true division in the exact build, a product with
// the folded reciprocal in the fast build
#if LBM_EXACT
#define DV(a, c) ((a) / C(c))
#else
#define DV(a, c) ((a) * (C(1.0) / C(c)))
#endif

// three-point Lagrange interpolation with precomputed weights, in the operand
// order of interpolateF (2M:655-657): (w0*f0 + w1*f1) + w2*f2
template <class C>
__device__ __forceinline__ C ip(const C w[3], C a, C m, C b) { return w[0] * a + w[1] * m + w[2] * b; }

template <class C>
__device__ __forceinline__ void load_w(const double *__restrict__ tab, int n, C wp[3], C wm[3])
{
    const double *t = tab + (int64_t)n * 6;
    wp[0] = C(__ldg(t + 0)); wp[1] = C(__ldg(t + 1)); wp[2] = C(__ldg(t + 2));
    wm[0] = C(__ldg(t + 3)); wm[1] = C(__ldg(t + 4)); wm[2] = C(__ldg(t + 5));
}

// stencil offsets (in nodes) of inter_x(i,1) and inter_x(i,3) relative to i:
// (i+1, i+2) at the first node, (i-1, i-2) at the last, (i-1, i+1) inside
// (2B:246-296)
__device__ __forceinline__ int off_a(int i, int n) { (void)n; return i == 0 ? 1 : -1; }
__device__ __forceinline__ int off_b(int i, int n) { return i == 0 ? 2 : (i == n - 1 ? -2 : 1); }

// ---------------------------------------------------------------------------
// 2D: D2Q9 MRT + D2Q5
// ---------------------------------------------------------------------------

// collision_U (2M:431-520) and collision_T (2M:522-569) at one node.  DEV:
// f and fp are deviations from the rest state (rho is still the full density).
template <class C, bool DEV = false, bool DEVT = false>
__device__ __forceinline__ void collide2d(const C f[9], const C gg[5], C rho, C u, C v, C T,
                                          const Geo &G, C fp[9], C gp[5], C &Fy)
{
    const C Snu = C(G.Snu), Sq = C(G.Sq), dt = C(G.dt), gbeta = C(G.gbeta), sig_k = C(G.sig_k);
    C m[9], meq[9], mp[9];
    m[0] = f[0]+f[1]+f[2]+f[3]+f[4]+f[5]+f[6]+f[7]+f[8];
    m[1] = -C(4.0)*f[0]-f[1]-f[2]-f[3]-f[4]+C(2.0)*(f[5]+f[6]+f[7]+f[8]);
    m[2] = C(4.0)*f[0]-C(2.0)*(f[1]+f[2]+f[3]+f[4])+f[5]+f[6]+f[7]+f[8];
    m[3] = f[1]-f[3]+f[5]-f[6]-f[7]+f[8];
    m[4] = -C(2.0)*f[1]+C(2.0)*f[3]+f[5]-f[6]-f[7]+f[8];
    m[5] = f[2]-f[4]+f[5]+f[6]-f[7]-f[8];
    m[6] = -C(2.0)*f[2]+C(2.0)*f[4]+f[5]+f[6]-f[7]-f[8];
    m[7] = f[1]-f[2]+f[3]-f[4];
    m[8] = f[5]-f[6]+f[7]-f[8];

    meq[0] = rho;
    meq[1] = rho*( -C(2.0)+C(3.0)*(u*u+v*v) );
    meq[2] = rho*( C(1.0)-C(3.0)*(u*u+v*v) );
    meq[3] = rho*u;
    meq[4] = -rho*u;
    meq[5] = rho*v;
    meq[6] = -rho*v;
    meq[7] = rho*(u*u-v*v);
    meq[8] = rho*(u*v);
    if (DEV) {
        // minus the rest state's moments (1, -2, 1, 0, ...): rho - 1 = m[0]
        meq[0] = m[0];
        meq[1] = -C(2.0)*m[0]+C(3.0)*rho*(u*u+v*v);
        meq[2] = m[0]-C(3.0)*rho*(u*u+v*v);
    }

    Fy = gbeta*T*rho;
#if LBM_EXACT
    // the reference's source terms with Fx = 0 kept (2M:475-486)
    const C Fx = C(0.0);
    const C s1 = Snu, s2 = Snu, s4 = Sq, s6 = Sq, s7 = Snu, s8 = Snu;
    C src[9];
    src[0] = C(0.0);
    src[1] = (C(6.0)-C(3.0)*s1)*(u*Fx+v*Fy);
    src[2] = -(C(6.0)-C(3.0)*s2)*(u*Fx+v*Fy);
    src[3] = Fx;
    src[4] = -(C(1.0)-C(0.5)*s4)*Fx;
    src[5] = Fy;
    src[6] = -(C(1.0)-C(0.5)*s6)*Fy;
    src[7] = (C(2.0)-s7)*(u*Fx-v*Fy);
    src[8] = (C(1.0)-C(0.5)*s8)*(v*Fx+u*Fy);
    const C sv[9] = {C(0.0), Snu, Snu, C(0.0), Sq, C(0.0), Sq, Snu, Snu};
#pragma unroll
    for (int a = 0; a < 9; ++a) mp[a] = m[a]-sv[a]*(m[a]-meq[a])+src[a]*dt;
#else
    // Fx = 0: the Fx terms vanish
    const C vF = v*Fy, uF = u*Fy;
    mp[0] = m[0];
    mp[1] = m[1]-Snu*(m[1]-meq[1])+(C(6.0)-C(3.0)*Snu)*vF*dt;
    mp[2] = m[2]-Snu*(m[2]-meq[2])-(C(6.0)-C(3.0)*Snu)*vF*dt;
    mp[3] = m[3];
    mp[4] = m[4]-Sq*(m[4]-meq[4]);
    mp[5] = m[5]+Fy*dt;
    mp[6] = m[6]-Sq*(m[6]-meq[6])-(C(1.0)-C(0.5)*Sq)*Fy*dt;
    mp[7] = m[7]-Snu*(m[7]-meq[7])-(C(2.0)-Snu)*vF*dt;
    mp[8] = m[8]-Snu*(m[8]-meq[8])+(C(1.0)-C(0.5)*Snu)*uF*dt;
#endif

    fp[0] = DV( mp[0]-mp[1]+mp[2] , 9.0);
    fp[1] = DV(mp[0],9.0)-DV(mp[1],36.0)-DV(mp[2],18.0)+DV(mp[3],6.0)-DV(mp[4],6.0)+mp[7]*C(0.25);
    fp[2] = DV(mp[0],9.0)-DV(mp[1],36.0)-DV(mp[2],18.0)+DV(mp[5],6.0)-DV(mp[6],6.0)-mp[7]*C(0.25);
    fp[3] = DV(mp[0],9.0)-DV(mp[1],36.0)-DV(mp[2],18.0)-DV(mp[3],6.0)+DV(mp[4],6.0)+mp[7]*C(0.25);
    fp[4] = DV(mp[0],9.0)-DV(mp[1],36.0)-DV(mp[2],18.0)-DV(mp[5],6.0)+DV(mp[6],6.0)-mp[7]*C(0.25);
    fp[5] = DV(mp[0],9.0)+DV(mp[1],18.0)+DV(mp[2],36.0)+DV(mp[3],6.0)+DV(mp[4],12.0)
            +DV(mp[5],6.0)+DV(mp[6],12.0)+mp[8]*C(0.25);
    fp[6] = DV(mp[0],9.0)+DV(mp[1],18.0)+DV(mp[2],36.0)-DV(mp[3],6.0)-DV(mp[4],12.0)
            +DV(mp[5],6.0)+DV(mp[6],12.0)-mp[8]*C(0.25);
    fp[7] = DV(mp[0],9.0)+DV(mp[1],18.0)+DV(mp[2],36.0)-DV(mp[3],6.0)-DV(mp[4],12.0)
            -DV(mp[5],6.0)-DV(mp[6],12.0)+mp[8]*C(0.25);
    fp[8] = DV(mp[0],9.0)+DV(mp[1],18.0)+DV(mp[2],36.0)+DV(mp[3],6.0)+DV(mp[4],12.0)
            -DV(mp[5],6.0)-DV(mp[6],12.0)-mp[8]*C(0.25);

    // thermal D2Q5
    C n[5], np[5];
    n[0] = gg[0]+gg[1]+gg[2]+gg[3]+gg[4];
    n[1] = gg[1]-gg[3];
    n[2] = gg[2]-gg[4];
    n[3] = gg[1]+gg[2]+gg[3]+gg[4];
    n[4] = gg[1]-gg[2]+gg[3]-gg[4];
#if LBM_EXACT
    const C Qr[5] = {C(1.0), sig_k, sig_k, C(1.9), C(1.9)};
    const C neq[5] = {T, T*u, T*v, T*C(0.5), C(0.0)};
#pragma unroll
    for (int a = 0; a < 5; ++a) np[a] = n[a]-Qr[a]*(n[a]-neq[a]);
#else
    // DEVT: gg are deviations from wT*Tc, whose moments are (Tc, 0, 0, Tc/2, 0)
    const C Tn = DEVT ? n[0] : T;
    np[0] = Tn;  // n(0) - 1*(n(0) - T)
    np[1] = n[1]-sig_k*(n[1]-T*u);
    np[2] = n[2]-sig_k*(n[2]-T*v);
    np[3] = n[3]-C(1.9)*(n[3]-Tn*C(0.5));
    np[4] = n[4]-C(1.9)*n[4];
#endif
    gp[0] = np[0]-np[3];
    gp[1] = DV(np[1],2.0)+DV(np[3],4.0)+DV(np[4],4.0);
    gp[2] = DV(np[2],2.0)+DV(np[3],4.0)-DV(np[4],4.0);
    gp[3] = -DV(np[1],2.0)+DV(np[3],4.0)+DV(np[4],4.0);
    gp[4] = -DV(np[2],2.0)+DV(np[3],4.0)-DV(np[4],4.0);
}

// One node (i, j) of the fused 2D step.  KIND 0: fused step; KIND 1: stream
// + walls + macro only.  COHERENT: read the source through L2 (ld.global.cg)
// instead of the read-only path, for a kernel that wrote it itself earlier.
template <int ST, int KIND, bool COHERENT = false>
__device__ __forceinline__ void step2d_node(const Geo &G, const typename Tr<ST>::S *__restrict__ src,
                                            const typename Tr<ST>::C *__restrict__ Fin,
                                            typename Tr<ST>::S *__restrict__ dst, typename Tr<ST>::C *__restrict__ Fout,
                                            const Bufs &B, int write_macro, int i, int j)
{
    using S = typename Tr<ST>::S;
    using C = typename Tr<ST>::C;
    const int64_t P = G.plane;
    const int64_t id = (int64_t)j * G.pitch + i;
    const int xa = off_a(i, G.nx), xb = off_b(i, G.nx);
    const int64_t ya = (int64_t)off_a(j, G.ny) * G.pitch, yb = (int64_t)off_b(j, G.ny) * G.pitch;
    C xp[3], xm[3], yp[3], ym[3];
    load_w(G.wgt[0], i, xp, xm);
    load_w(G.wgt[1], j, yp, ym);

    auto LD = [&](int q, int64_t off) -> C {
        return tocomp(COHERENT ? __ldcg(src + q * P + id + off) : __ldg(src + q * P + id + off));
    };
    // y-interpolation of plane q on the column at x-offset c
    auto YI = [&](int q, const C w[3], int64_t c) -> C { return ip(w, LD(q, c + ya), LD(q, c), LD(q, c + yb)); };

    C f[9], gg[5];
    f[0] = LD(0, 0);
    f[1] = ip(xp, LD(1, xa), LD(1, 0), LD(1, xb));
    f[2] = ip(yp, LD(2, ya), LD(2, 0), LD(2, yb));
    f[3] = ip(xm, LD(3, xa), LD(3, 0), LD(3, xb));
    f[4] = ip(ym, LD(4, ya), LD(4, 0), LD(4, yb));
    f[5] = ip(xp, YI(5, yp, xa), YI(5, yp, 0), YI(5, yp, xb));
    f[6] = ip(xm, YI(6, yp, xa), YI(6, yp, 0), YI(6, yp, xb));
    f[7] = ip(xm, YI(7, ym, xa), YI(7, ym, 0), YI(7, ym, xb));
    f[8] = ip(xp, YI(8, ym, xa), YI(8, ym, 0), YI(8, ym, xb));
    gg[0] = LD(9, 0);
    gg[1] = ip(xp, LD(10, xa), LD(10, 0), LD(10, xb));
    gg[2] = ip(yp, LD(11, ya), LD(11, 0), LD(11, yb));
    gg[3] = ip(xm, LD(12, xa), LD(12, 0), LD(12, xb));
    gg[4] = ip(ym, LD(13, ya), LD(13, 0), LD(13, yb));
    // deviation from the conduction profile: the departure point of g1 / g3
    // lies dt behind / ahead along x
    C Tc = C(0.0);
    if (Tr<ST>::kDevT) {
        Tc = C(tc_value(G, i));
        const C sT = C(0.125 * G.dt * tc_gradient(G));
        gg[1] -= sT;
        gg[3] += sT;
    }

    // walls: bounceback_u (2B:731-768), bounceback_T (2B:770-801)
    const C two_wT = C(2.0) * C(0.125);
    if (i == 0) {
        f[1] = LD(3, 0); f[5] = LD(7, 0); f[8] = LD(6, 0);
        gg[1] = -LD(12, 0) + two_wT * (Tr<ST>::kDevT ? C(G.Thot) - Tc : C(G.Thot));
    }
    if (i == G.nx - 1) {
        f[3] = LD(1, 0); f[6] = LD(8, 0); f[7] = LD(5, 0);
        gg[3] = -LD(10, 0) + two_wT * (Tr<ST>::kDevT ? C(G.Tcold) - Tc : C(G.Tcold));
    }
    if (j == G.ny - 1) {
        f[4] = LD(2, 0); f[7] = LD(5, 0); f[8] = LD(6, 0);
        gg[4] = LD(11, 0);
    }
    if (j == 0) {
        f[2] = LD(4, 0); f[5] = LD(7, 0); f[6] = LD(8, 0);
        gg[2] = LD(13, 0);
    }

    // macro_u / macro_t (2M:726-753); the force is the one of the collision
    // that produced src
    const C Fy0 = COHERENT ? __ldcg(Fin + id) : Fin[id];
    const C dt = C(G.dt);
    const C rho = (Tr<ST>::kShift ? C(1.0) : C(0.0)) + (f[0]+f[1]+f[2]+f[3]+f[4]+f[5]+f[6]+f[7]+f[8]);
#if LBM_EXACT
    const C u = ( f[1]-f[3]+f[5]-f[6]-f[7]+f[8]+C(0.5)*dt*C(0.0))/rho;
    const C v = ( f[2]-f[4]+f[5]+f[6]-f[7]-f[8]+C(0.5)*dt*Fy0)/rho;
#else
    const C rinv = C(1.0) / rho;
    const C u = (f[1]-f[3]+f[5]-f[6]-f[7]+f[8])*rinv;
    const C v = (f[2]-f[4]+f[5]+f[6]-f[7]-f[8]+C(0.5)*dt*Fy0)*rinv;
#endif
    const C T = Tr<ST>::kDevT ? Tc + (gg[0]+gg[1]+gg[2]+gg[3]+gg[4]) : gg[0]+gg[1]+gg[2]+gg[3]+gg[4];

    if (write_macro || KIND == 1) {
        const int64_t mid = (int64_t)j * G.nx + i;
        B.rho[mid] = double(rho); B.u[mid] = double(u); B.v[mid] = double(v); B.T[mid] = double(T);
    }

    auto ST_ = [&](int q, C val) {
        dst[q * P + id] = tostore<S, C>(val);
    };
    if (KIND == 1) {
#pragma unroll
        for (int q = 0; q < 9; ++q) ST_(q, f[q]);
#pragma unroll
        for (int q = 0; q < 5; ++q) ST_(9 + q, gg[q]);
        return;
    }

    C fp[9], gp[5], Fy;
    collide2d<C, Tr<ST>::kShift, Tr<ST>::kDevT>(f, gg, rho, u, v, T, G, fp, gp, Fy);
    Fout[id] = Fy;
#pragma unroll
    for (int q = 0; q < 9; ++q) ST_(q, fp[q]);
#pragma unroll
    for (int q = 0; q < 5; ++q) ST_(9 + q, gp[q]);
}

template <int ST, int KIND>
__global__ void __launch_bounds__(256)
k_step2d(const Geo G, const typename Tr<ST>::S *__restrict__ src, const typename Tr<ST>::C *__restrict__ Fin,
         typename Tr<ST>::S *__restrict__ dst, typename Tr<ST>::C *__restrict__ Fout, const Bufs B,
         int write_macro)
{
    if (!B.ctl->active) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= G.nx || j < G.jlo || j >= G.jhi) return;  // a slab's ghost rows come from its neighbours
    step2d_node<ST, KIND>(G, src, Fin, dst, Fout, B, write_macro, i, j);
}

// Bounded grid-wide barrier for a cooperative launch (every block resident):
// sense by generation count.  False (and *err set) if the other blocks did
// not arrive within kGridWaitCycles.
static constexpr long long kGridWaitCycles = 2000000000LL;  // ~1 s

__device__ __forceinline__ bool grid_barrier(unsigned *count, unsigned *gen, unsigned nblocks, int *err)
{
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        const unsigned g0 = *(volatile unsigned *)gen;
        __threadfence();
        ok = 1;
        if (atomicAdd(count, 1u) + 1u == nblocks) {
            *(volatile unsigned *)count = 0u;
            __threadfence();
            atomicAdd(gen, 1u);
        } else {
            const long long t0 = clock64();
            while (*(volatile unsigned *)gen == g0)
                if (clock64() - t0 > kGridWaitCycles) {
                    atomicExch(err, 1);
                    ok = 0;
                    break;
                }
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

// nsteps fused 2D steps in one cooperative launch for domains that fit one
// wave (the per-step launch gap dominates there): step s reads buffer
// (cur + s) & 1, writes the other, and every block waits at the grid barrier
// before the next step reads what its neighbours wrote.  The macroscopic
// fields are written by the last step.
template <int ST>
__global__ void __launch_bounds__(256)
k_steps2d_resident(const Geo G, typename Tr<ST>::S *p0, typename Tr<ST>::S *p1, typename Tr<ST>::C *F0,
                   typename Tr<ST>::C *F1, const Bufs B, int cur, int nsteps, unsigned *bar, int *err)
{
    using S = typename Tr<ST>::S;
    using C = typename Tr<ST>::C;
    if (!B.ctl->active) return;
    const int64_t nn = (int64_t)G.nx * G.ny;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int s = 0; s < nsteps; ++s) {
        const int c = (cur + s) & 1;
        const S *src = c ? p1 : p0;
        S *dst = c ? p0 : p1;
        const C *Fin = c ? F1 : F0;
        C *Fout = c ? F0 : F1;
        const int wm = s == nsteps - 1;
        for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < nn; n += stride)
            step2d_node<ST, 0, true>(G, src, Fin, dst, Fout, B, wm, int(n % G.nx), int(n / G.nx));
        if (s + 1 < nsteps && !grid_barrier(bar, bar + 1, gridDim.x, err)) return;
    }
}

// ---------------------------------------------------------------------------
// 3D: D3Q19 MRT + D3Q7
// ---------------------------------------------------------------------------

// collision_U (3M:445-669) and collision_T (3M:671-730) at one node.  DEV:
// f and fp are deviations from the rest state (rho is still the full density).
template <class C, bool DEV = false, bool DEVT = false>
__device__ __forceinline__ void collide3d(const C f[19], const C gg[7], C rho, C u, C v, C w, C T,
                                          const Geo &G, C fp[19], C gp[7], C &Fz)
{
    const C Snu = C(G.Snu), Sq = C(G.Sq), dt = C(G.dt), gbeta = C(G.gbeta), sig_k = C(G.sig_k);
    const C Vsquare = u*u+v*v+w*w;
    C m[19], meq[19], mp[19];
    m[0]=f[0]+f[1]+f[2]+f[3]+f[4]+f[5]+f[6]+f[7]+f[8]+f[9]+f[10]+f[11]+f[12]+f[13]+f[14]+f[15]+f[16]+f[17]+f[18];
    m[1]=-C(30.0)*f[0]-C(11.0)*(f[1]+f[2]+f[3]+f[4]+f[5]+f[6])+C(8.0)*(f[7]+f[8]+f[9]+f[10]+f[11]+f[12]+f[13]+f[14]+f[15]+f[16]+f[17]+f[18]);
    m[2]=C(12.0)*f[0]-C(4.0)*(f[1]+f[2]+f[3]+f[4]+f[5]+f[6])+(f[7]+f[8]+f[9]+f[10]+f[11]+f[12]+f[13]+f[14]+f[15]+f[16]+f[17]+f[18]);
    m[3]=f[1]-f[2]+f[7]-f[8]+f[9]-f[10]+f[11]-f[12]+f[13]-f[14];
    m[4]=C(4.0)*(-f[1]+f[2])+f[7]-f[8]+f[9]-f[10]+f[11]-f[12]+f[13]-f[14];
    m[5]=f[3]-f[4]+f[7]+f[8]-f[9]-f[10]+f[15]-f[16]+f[17]-f[18];
    m[6]=-C(4.0)*(f[3]-f[4])+f[7]+f[8]-f[9]-f[10]+f[15]-f[16]+f[17]-f[18];
    m[7]=f[5]-f[6]+f[11]+f[12]-f[13]-f[14]+f[15]+f[16]-f[17]-f[18];
    m[8]=-C(4.0)*(f[5]-f[6])+f[11]+f[12]-f[13]-f[14]+f[15]+f[16]-f[17]-f[18];
    m[9]=C(2.0)*(f[1]+f[2])-(f[3]+f[4]+f[5]+f[6])+f[7]+f[8]+f[9]+f[10]+f[11]+f[12]+f[13]+f[14]-C(2.0)*(f[15]+f[16]+f[17]+f[18]);
    m[10]=-C(4.0)*(f[1]+f[2])+C(2.0)*(f[3]+f[4]+f[5]+f[6])+f[7]+f[8]+f[9]+f[10]+f[11]+f[12]+f[13]+f[14]-C(2.0)*(f[15]+f[16]+f[17]+f[18]);
    m[11]=f[3]+f[4]-f[5]-f[6]+f[7]+f[8]+f[9]+f[10]-f[11]-f[12]-f[13]-f[14];
    m[12]=-C(2.0)*(f[3]+f[4]-f[5]-f[6])+f[7]+f[8]+f[9]+f[10]-f[11]-f[12]-f[13]-f[14];
    m[13]=f[7]-f[8]-f[9]+f[10];
    m[14]=f[15]-f[16]-f[17]+f[18];
    m[15]=f[11]-f[12]-f[13]+f[14];
    m[16]=f[7]-f[8]+f[9]-f[10]-f[11]+f[12]-f[13]+f[14];
    m[17]=-f[7]-f[8]+f[9]+f[10]+f[15]-f[16]+f[17]-f[18];
    m[18]=f[11]+f[12]-f[13]-f[14]-f[15]-f[16]+f[17]+f[18];

    meq[0]=rho;
    meq[1]=-C(11.0)*rho+C(19.0)*rho*Vsquare;
    meq[2]=C(3.0)*rho-C(5.5)*rho*Vsquare;
    meq[3]=rho*u;
    meq[4]=DV(-C(2.0)*rho*u, 3.0);
    meq[5]=rho*v;
    meq[6]=DV(-C(2.0)*rho*v, 3.0);
    meq[7]=rho*w;
    meq[8]=DV(-C(2.0)*rho*w, 3.0);
    meq[9]=C(3.0)*rho*(u*u)-rho*Vsquare;
    meq[10]=-C(0.5)*(C(3.0)*rho*(u*u)-rho*Vsquare);
    meq[11]=rho*((v*v)-(w*w));
    meq[12]=-C(0.5)*rho*((v*v)-(w*w));
    meq[13]=rho*u*v;
    meq[14]=rho*v*w;
    meq[15]=rho*u*w;
    if (DEV) {
        // minus the rest state's moments (1, -11, 3, 0, ...): rho - 1 = m[0]
        meq[0]=m[0];
        meq[1]=-C(11.0)*m[0]+C(19.0)*rho*Vsquare;
        meq[2]=C(3.0)*m[0]-C(5.5)*rho*Vsquare;
    }

    Fz = gbeta*T*rho;
#if LBM_EXACT
    const C sv[19] = {C(0.0), Snu, Snu, C(0.0), Sq, C(0.0), Sq, C(0.0), Sq, Snu, Snu, Snu, Snu, Snu, Snu, Snu, Sq, Sq, Sq};
    meq[16]=C(0.0); meq[17]=C(0.0); meq[18]=C(0.0);
    C src[19];
    src[0] = C(0.0);
    src[1] = (C(38.0)-C(19.0)*sv[1])*w*Fz;
    src[2] = -(C(11.0)-C(5.5)*sv[2])*w*Fz;
    src[3] = C(0.0); src[4] = C(0.0); src[5] = C(0.0); src[6] = C(0.0);
    src[7] = (C(1.0)-C(0.5)*sv[7])*Fz;
    src[8] = -C(2.0)*(C(1.0)-C(0.5)*sv[8])*Fz/C(3.0);
    src[9] = (-C(2.0)+sv[9])*w*Fz;
    src[10] = (C(1.0)-C(0.5)*sv[10])*w*Fz;
    src[11] = -(C(2.0)-sv[11])*w*Fz;
    src[12] = (C(1.0)-C(0.5)*sv[12])*w*Fz;
    src[13] = C(0.0);
    src[14] = (C(1.0)-C(0.5)*sv[14])*v*Fz;
    src[15] = (C(1.0)-C(0.5)*sv[15])*u*Fz;
    src[16] = C(0.0); src[17] = C(0.0); src[18] = C(0.0);
#pragma unroll
    for (int a = 0; a < 19; ++a) mp[a] = m[a]-sv[a]*(m[a]-meq[a])+src[a]*dt;
#else
    const C wF = w*Fz*dt;
    const C hNu = C(1.0)-C(0.5)*Snu;
    mp[0] = m[0];
    mp[1] = m[1]-Snu*(m[1]-meq[1])+(C(38.0)-C(19.0)*Snu)*wF;
    mp[2] = m[2]-Snu*(m[2]-meq[2])-(C(11.0)-C(5.5)*Snu)*wF;
    mp[3] = m[3];
    mp[4] = m[4]-Sq*(m[4]-meq[4]);
    mp[5] = m[5];
    mp[6] = m[6]-Sq*(m[6]-meq[6]);
    mp[7] = m[7]+Fz*dt;
    mp[8] = m[8]-Sq*(m[8]-meq[8])-DV(C(2.0)*(C(1.0)-C(0.5)*Sq)*Fz*dt, 3.0);
    mp[9] = m[9]-Snu*(m[9]-meq[9])+(-C(2.0)+Snu)*wF;
    mp[10] = m[10]-Snu*(m[10]-meq[10])+hNu*wF;
    mp[11] = m[11]-Snu*(m[11]-meq[11])-(C(2.0)-Snu)*wF;
    mp[12] = m[12]-Snu*(m[12]-meq[12])+hNu*wF;
    mp[13] = m[13]-Snu*(m[13]-meq[13]);
    mp[14] = m[14]-Snu*(m[14]-meq[14])+hNu*v*Fz*dt;
    mp[15] = m[15]-Snu*(m[15]-meq[15])+hNu*u*Fz*dt;
    mp[16] = m[16]-Sq*m[16];
    mp[17] = m[17]-Sq*m[17];
    mp[18] = m[18]-Sq*m[18];
#endif

    fp[0]=DV(mp[0],19.0)-DV(C(5.0)*mp[1],399.0)+DV(mp[2],21.0);
    fp[1]=DV(mp[0],19.0)-DV(C(11.0)*mp[1],2394.0)-DV(mp[2],63.0)+DV(mp[3],10.0)-DV(mp[4],10.0)+DV(mp[9],18.0)-DV(mp[10],18.0);
    fp[2]=DV(mp[0],19.0)-DV(C(11.0)*mp[1],2394.0)-DV(mp[2],63.0)-DV(mp[3],10.0)+DV(mp[4],10.0)+DV(mp[9],18.0)-DV(mp[10],18.0);
    fp[3]=DV(mp[0],19.0)-DV(C(11.0)*mp[1],2394.0)-DV(mp[2],63.0)+DV(mp[5],10.0)-DV(mp[6],10.0)-DV(mp[9],36.0)+DV(mp[10],36.0)+DV(mp[11],12.0)-DV(mp[12],12.0);
    fp[4]=DV(mp[0],19.0)-DV(C(11.0)*mp[1],2394.0)-DV(mp[2],63.0)-DV(mp[5],10.0)+DV(mp[6],10.0)-DV(mp[9],36.0)+DV(mp[10],36.0)+DV(mp[11],12.0)-DV(mp[12],12.0);
    fp[5]=DV(mp[0],19.0)-DV(C(11.0)*mp[1],2394.0)-DV(mp[2],63.0)+DV(mp[7],10.0)-DV(mp[8],10.0)-DV(mp[9],36.0)+DV(mp[10],36.0)-DV(mp[11],12.0)+DV(mp[12],12.0);
    fp[6]=DV(mp[0],19.0)-DV(C(11.0)*mp[1],2394.0)-DV(mp[2],63.0)-DV(mp[7],10.0)+DV(mp[8],10.0)-DV(mp[9],36.0)+DV(mp[10],36.0)-DV(mp[11],12.0)+DV(mp[12],12.0);
    fp[7]=DV(mp[0],19.0)+DV(C(4.0)*mp[1],1197.0)+DV(mp[2],252.0)+DV(mp[3],10.0)+DV(mp[4],40.0)+DV(mp[5],10.0)+DV(mp[6],40.0)+DV(mp[9],36.0)+DV(mp[10],72.0)
          +DV(mp[11],12.0)+DV(mp[12],24.0)+DV(mp[13],4.0)+DV(mp[16],8.0)-DV(mp[17],8.0);
    fp[8]=DV(mp[0],19.0)+DV(C(4.0)*mp[1],1197.0)+DV(mp[2],252.0)-DV(mp[3],10.0)-DV(mp[4],40.0)+DV(mp[5],10.0)+DV(mp[6],40.0)+DV(mp[9],36.0)+DV(mp[10],72.0)
          +DV(mp[11],12.0)+DV(mp[12],24.0)-DV(mp[13],4.0)-DV(mp[16],8.0)-DV(mp[17],8.0);
    fp[9]=DV(mp[0],19.0)+DV(C(4.0)*mp[1],1197.0)+DV(mp[2],252.0)+DV(mp[3],10.0)+DV(mp[4],40.0)-DV(mp[5],10.0)-DV(mp[6],40.0)+DV(mp[9],36.0)+DV(mp[10],72.0)
          +DV(mp[11],12.0)+DV(mp[12],24.0)-DV(mp[13],4.0)+DV(mp[16],8.0)+DV(mp[17],8.0);
    fp[10]=DV(mp[0],19.0)+DV(C(4.0)*mp[1],1197.0)+DV(mp[2],252.0)-DV(mp[3],10.0)-DV(mp[4],40.0)-DV(mp[5],10.0)-DV(mp[6],40.0)+DV(mp[9],36.0)+DV(mp[10],72.0)
          +DV(mp[11],12.0)+DV(mp[12],24.0)+DV(mp[13],4.0)-DV(mp[16],8.0)+DV(mp[17],8.0);
    fp[11]=DV(mp[0],19.0)+DV(C(4.0)*mp[1],1197.0)+DV(mp[2],252.0)+DV(mp[3],10.0)+DV(mp[4],40.0)+DV(mp[7],10.0)+DV(mp[8],40.0)+DV(mp[9],36.0)+DV(mp[10],72.0)
          -DV(mp[11],12.0)-DV(mp[12],24.0)+DV(mp[15],4.0)-DV(mp[16],8.0)+DV(mp[18],8.0);
    fp[12]=DV(mp[0],19.0)+DV(C(4.0)*mp[1],1197.0)+DV(mp[2],252.0)-DV(mp[3],10.0)-DV(mp[4],40.0)+DV(mp[7],10.0)+DV(mp[8],40.0)+DV(mp[9],36.0)+DV(mp[10],72.0)
          -DV(mp[11],12.0)-DV(mp[12],24.0)-DV(mp[15],4.0)+DV(mp[16],8.0)+DV(mp[18],8.0);
    fp[13]=DV(mp[0],19.0)+DV(C(4.0)*mp[1],1197.0)+DV(mp[2],252.0)+DV(mp[3],10.0)+DV(mp[4],40.0)-DV(mp[7],10.0)-DV(mp[8],40.0)+DV(mp[9],36.0)+DV(mp[10],72.0)
          -DV(mp[11],12.0)-DV(mp[12],24.0)-DV(mp[15],4.0)-DV(mp[16],8.0)-DV(mp[18],8.0);
    fp[14]=DV(mp[0],19.0)+DV(C(4.0)*mp[1],1197.0)+DV(mp[2],252.0)-DV(mp[3],10.0)-DV(mp[4],40.0)-DV(mp[7],10.0)-DV(mp[8],40.0)+DV(mp[9],36.0)+DV(mp[10],72.0)
          -DV(mp[11],12.0)-DV(mp[12],24.0)+DV(mp[15],4.0)+DV(mp[16],8.0)-DV(mp[18],8.0);
    fp[15]=DV(mp[0],19.0)+DV(C(4.0)*mp[1],1197.0)+DV(mp[2],252.0)+DV(mp[5],10.0)+DV(mp[6],40.0)+DV(mp[7],10.0)+DV(mp[8],40.0)-DV(mp[9],18.0)-DV(mp[10],36.0)
          +DV(mp[14],4.0)+DV(mp[17],8.0)-DV(mp[18],8.0);
    fp[16]=DV(mp[0],19.0)+DV(C(4.0)*mp[1],1197.0)+DV(mp[2],252.0)-DV(mp[5],10.0)-DV(mp[6],40.0)+DV(mp[7],10.0)+DV(mp[8],40.0)-DV(mp[9],18.0)-DV(mp[10],36.0)
          -DV(mp[14],4.0)-DV(mp[17],8.0)-DV(mp[18],8.0);
    fp[17]=DV(mp[0],19.0)+DV(C(4.0)*mp[1],1197.0)+DV(mp[2],252.0)+DV(mp[5],10.0)+DV(mp[6],40.0)-DV(mp[7],10.0)-DV(mp[8],40.0)-DV(mp[9],18.0)-DV(mp[10],36.0)
          -DV(mp[14],4.0)+DV(mp[17],8.0)+DV(mp[18],8.0);
    fp[18]=DV(mp[0],19.0)+DV(C(4.0)*mp[1],1197.0)+DV(mp[2],252.0)-DV(mp[5],10.0)-DV(mp[6],40.0)-DV(mp[7],10.0)-DV(mp[8],40.0)-DV(mp[9],18.0)-DV(mp[10],36.0)
          +DV(mp[14],4.0)-DV(mp[17],8.0)+DV(mp[18],8.0);

    // thermal D3Q7
    C n[7], np[7];
    n[0] = gg[0]+gg[1]+gg[2]+gg[3]+gg[4]+gg[5]+gg[6];
    n[1] = gg[1]-gg[2];
    n[2] = gg[3]-gg[4];
    n[3] = gg[5]-gg[6];
    n[4] = gg[1]+gg[2]+gg[3]+gg[4]+gg[5]+gg[6];
    n[5] = gg[1]+gg[2]-gg[3]-gg[4];
    n[6] = gg[1]+gg[2]-gg[5]-gg[6];
#if LBM_EXACT
    const C Qr[7] = {C(1.0), sig_k, sig_k, sig_k, C(1.2), C(1.2), C(1.2)};
    const C neq[7] = {T, T*u, T*v, T*w, T*C(0.5), C(0.0), C(0.0)};
#pragma unroll
    for (int a = 0; a < 7; ++a) np[a] = n[a]-Qr[a]*(n[a]-neq[a]);
#else
    // DEVT: gg are deviations from wT*Tc, whose moments are (Tc, 0, 0, 0, Tc/2, 0, 0)
    const C Tn = DEVT ? n[0] : T;
    np[0] = Tn;
    np[1] = n[1]-sig_k*(n[1]-T*u);
    np[2] = n[2]-sig_k*(n[2]-T*v);
    np[3] = n[3]-sig_k*(n[3]-T*w);
    np[4] = n[4]-C(1.2)*(n[4]-Tn*C(0.5));
    np[5] = n[5]-C(1.2)*n[5];
    np[6] = n[6]-C(1.2)*n[6];
#endif
    gp[0] = np[0]-np[4];
    gp[1] = DV(np[1],2.0)+DV(np[4],6.0)+DV(np[5],6.0)+DV(np[6],6.0);
    gp[2] = -DV(np[1],2.0)+DV(np[4],6.0)+DV(np[5],6.0)+DV(np[6],6.0);
    gp[3] = DV(np[2],2.0)+DV(np[4],6.0)-DV(np[5],3.0)+DV(np[6],6.0);
    gp[4] = -DV(np[2],2.0)+DV(np[4],6.0)-DV(np[5],3.0)+DV(np[6],6.0);
    gp[5] = DV(np[3],2.0)+DV(np[4],6.0)+DV(np[5],6.0)-DV(np[6],3.0);
    gp[6] = -DV(np[3],2.0)+DV(np[4],6.0)+DV(np[5],6.0)-DV(np[6],3.0);
}

#if !LBM_EXACT
// Fast-path 3D node update: the same collision as collide3d (3M:445-730) with
// shared subexpressions.  Moments are built from pairwise sums and
// differences of the +- populations, rho and momentum are taken from the
// moments (the reference's macro_u sums are the same sums), and the inverse
// transform groups the +- symmetric populations; ~45 % fewer FP64 operations
// and shorter dependency chains.  Fz0 is the force carried from the previous
// collision (macro_u's half-force term).  Writes rho, u, v, w, T.
template <class C, bool DEV = false, bool DEVT = false>
__device__ __forceinline__ void node3d_fast(const C f[19], const C gg[7], C Fz0, const Geo &G, C fp[19], C gp[7],
                                            C &Fz, C &rho, C &u, C &v, C &w, C &T, C Tc = C(0.0))
{
    const C Snu = C(G.Snu), Sq = C(G.Sq), dt = C(G.dt), gbeta = C(G.gbeta), sig_k = C(G.sig_k);
    // pairwise sums / differences
    const C a12 = f[1] + f[2], d12 = f[1] - f[2];
    const C a34 = f[3] + f[4], d34 = f[3] - f[4];
    const C a56 = f[5] + f[6], d56 = f[5] - f[6];
    const C p78 = f[7] + f[8], q78 = f[7] - f[8], p910 = f[9] + f[10], q910 = f[9] - f[10];
    const C p1112 = f[11] + f[12], q1112 = f[11] - f[12], p1314 = f[13] + f[14], q1314 = f[13] - f[14];
    const C p1516 = f[15] + f[16], q1516 = f[15] - f[16], p1718 = f[17] + f[18], q1718 = f[17] - f[18];
    const C s_xy = p78 + p910, xy_x = q78 + q910, xy_y = p78 - p910;
    const C s_xz = p1112 + p1314, xz_x = q1112 + q1314, xz_z = p1112 - p1314;
    const C s_yz = p1516 + p1718, yz_y = q1516 + q1718, yz_z = p1516 - p1718;
    const C sA = a12 + (a34 + a56), sD = s_xy + (s_xz + s_yz);
    const C xsum = xy_x + xz_x, ysum = xy_y + yz_y, zsum = xz_z + yz_z;
    C m[19];
    m[0] = f[0] + sA + sD;
    m[1] = C(-30.0) * f[0] - C(11.0) * sA + C(8.0) * sD;
    m[2] = C(12.0) * f[0] - C(4.0) * sA + sD;
    m[3] = d12 + xsum;
    m[4] = C(-4.0) * d12 + xsum;
    m[5] = d34 + ysum;
    m[6] = C(-4.0) * d34 + ysum;
    m[7] = d56 + zsum;
    m[8] = C(-4.0) * d56 + zsum;
    const C a3456 = a34 + a56, sxyxz = s_xy + s_xz;
    m[9] = C(2.0) * a12 - a3456 + sxyxz - C(2.0) * s_yz;
    m[10] = C(-4.0) * a12 + C(2.0) * a3456 + sxyxz - C(2.0) * s_yz;
    const C a34m56 = a34 - a56, sxymxz = s_xy - s_xz;
    m[11] = a34m56 + sxymxz;
    m[12] = C(-2.0) * a34m56 + sxymxz;
    m[13] = q78 - q910;
    m[14] = q1516 - q1718;
    m[15] = q1112 - q1314;
    m[16] = xy_x - xz_x;
    m[17] = yz_y - xy_y;
    m[18] = xz_z - yz_z;

    // macro_u / macro_t (3M:988-1025); DEV: m[0] = rho - 1
    rho = DEV ? C(1.0) + m[0] : m[0];
    const C rinv = C(1.0) / rho;
    u = m[3] * rinv;
    v = m[5] * rinv;
    w = (m[7] + C(0.5) * dt * Fz0) * rinv;
    const C Tn = gg[0] + (gg[1] + gg[2]) + (gg[3] + gg[4]) + (gg[5] + gg[6]);  // DEVT: T - Tc
    T = DEVT ? Tc + Tn : Tn;

    // equilibria and relaxation (3M:522-587)
    const C uu = u * u, vv = v * v, ww = w * w;
    const C Vs = uu + vv + ww;
    const C ru = rho * u, rv = rho * v, rw = rho * w;
    Fz = gbeta * T * rho;
    const C wF = w * Fz * dt;
    const C hNu = C(1.0) - C(0.5) * Snu;
    const C e9 = C(3.0) * rho * uu - rho * Vs;
    const C e11 = rho * (vv - ww);
    C mp[19];
    mp[0] = m[0];
    // DEV: the equilibria minus the rest state's moments (1, -11, 3, 0, ...)
    const C r1 = DEV ? m[0] : rho;
    mp[1] = m[1] - Snu * (m[1] - (C(-11.0) * r1 + C(19.0) * rho * Vs)) + (C(38.0) - C(19.0) * Snu) * wF;
    mp[2] = m[2] - Snu * (m[2] - (C(3.0) * r1 - C(5.5) * rho * Vs)) - (C(11.0) - C(5.5) * Snu) * wF;
    mp[3] = m[3];
    mp[4] = m[4] - Sq * (m[4] - C(-2.0 / 3.0) * ru);
    mp[5] = m[5];
    mp[6] = m[6] - Sq * (m[6] - C(-2.0 / 3.0) * rv);
    mp[7] = m[7] + Fz * dt;
    mp[8] = m[8] - Sq * (m[8] - C(-2.0 / 3.0) * rw) - (C(2.0 / 3.0) * (C(1.0) - C(0.5) * Sq)) * Fz * dt;
    mp[9] = m[9] - Snu * (m[9] - e9) + (Snu - C(2.0)) * wF;
    mp[10] = m[10] - Snu * (m[10] + C(0.5) * e9) + hNu * wF;
    mp[11] = m[11] - Snu * (m[11] - e11) - (C(2.0) - Snu) * wF;
    mp[12] = m[12] - Snu * (m[12] + C(0.5) * e11) + hNu * wF;
    mp[13] = m[13] - Snu * (m[13] - ru * v);
    mp[14] = m[14] - Snu * (m[14] - rv * w) + hNu * v * Fz * dt;
    mp[15] = m[15] - Snu * (m[15] - ru * w) + hNu * u * Fz * dt;
    const C oSq = C(1.0) - Sq;
    mp[16] = oSq * m[16];
    mp[17] = oSq * m[17];
    mp[18] = oSq * m[18];

    // inverse transform (3M:589-655), grouped by symmetric pairs
    const C D0 = mp[0] * C(1.0 / 19.0);
    fp[0] = D0 - mp[1] * C(5.0 / 399.0) + mp[2] * C(1.0 / 21.0);
    const C A = D0 - mp[1] * C(11.0 / 2394.0) - mp[2] * C(1.0 / 63.0);
    const C D = D0 + mp[1] * C(4.0 / 1197.0) + mp[2] * C(1.0 / 252.0);
    const C h910 = (mp[9] - mp[10]);
    const C h1112 = (mp[11] - mp[12]);
    {
        const C c = A + h910 * C(1.0 / 18.0), o = (mp[3] - mp[4]) * C(0.1);
        fp[1] = c + o; fp[2] = c - o;
    }
    {
        const C c = A - h910 * C(1.0 / 36.0) + h1112 * C(1.0 / 12.0), o = (mp[5] - mp[6]) * C(0.1);
        fp[3] = c + o; fp[4] = c - o;
    }
    {
        const C c = A - h910 * C(1.0 / 36.0) - h1112 * C(1.0 / 12.0), o = (mp[7] - mp[8]) * C(0.1);
        fp[5] = c + o; fp[6] = c - o;
    }
    const C X = mp[3] * C(0.1) + mp[4] * C(0.025);
    const C Y = mp[5] * C(0.1) + mp[6] * C(0.025);
    const C Z = mp[7] * C(0.1) + mp[8] * C(0.025);
    const C e9b = mp[9] * C(1.0 / 36.0) + mp[10] * C(1.0 / 72.0);
    const C e11b = mp[11] * C(1.0 / 12.0) + mp[12] * C(1.0 / 24.0);
    const C r16 = mp[16] * C(0.125), r17 = mp[17] * C(0.125), r18 = mp[18] * C(0.125);
    {   // xy plane: 7 (+,+), 8 (-,+), 9 (+,-), 10 (-,-)
        const C DE = D + e9b + e11b, c = mp[13] * C(0.25);
        const C P = X + r16, Qy = Y - r17;
        const C s1 = DE + c, s2 = DE - c;
        fp[7] = s1 + (P + Qy); fp[10] = s1 - (P + Qy);
        fp[8] = s2 - (P - Qy); fp[9] = s2 + (P - Qy);
    }
    {   // xz plane: 11 (+,+), 12 (-,+), 13 (+,-), 14 (-,-)
        const C DE = D + e9b - e11b, c = mp[15] * C(0.25);
        const C P = X - r16, Qz = Z + r18;
        const C s1 = DE + c, s2 = DE - c;
        fp[11] = s1 + (P + Qz); fp[14] = s1 - (P + Qz);
        fp[12] = s2 - (P - Qz); fp[13] = s2 + (P - Qz);
    }
    {   // yz plane: 15 (+,+), 16 (-,+), 17 (+,-), 18 (-,-)
        const C DE = D - mp[9] * C(1.0 / 18.0) - mp[10] * C(1.0 / 36.0), c = mp[14] * C(0.25);
        const C P = Y + r17, Qz = Z - r18;
        const C s1 = DE + c, s2 = DE - c;
        fp[15] = s1 + (P + Qz); fp[18] = s1 - (P + Qz);
        fp[16] = s2 - (P - Qz); fp[17] = s2 + (P - Qz);
    }

    // thermal D3Q7 (3M:671-730)
    const C b12 = gg[1] + gg[2], b34 = gg[3] + gg[4], b56 = gg[5] + gg[6];
    const C n1 = gg[1] - gg[2], n2 = gg[3] - gg[4], n3 = gg[5] - gg[6];
    const C n4 = b12 + b34 + b56, n5 = b12 - b34, n6 = b12 - b56;
    const C np1 = n1 - sig_k * (n1 - T * u);
    const C np2 = n2 - sig_k * (n2 - T * v);
    const C np3 = n3 - sig_k * (n3 - T * w);
    const C np4 = n4 - C(1.2) * (n4 - Tn * C(0.5));
    const C np5 = C(-0.2) * n5, np6 = C(-0.2) * n6;
    gp[0] = Tn - np4;
    const C t4 = np4 * C(1.0 / 6.0), t5 = np5 * C(1.0 / 6.0), t6 = np6 * C(1.0 / 6.0);
    {
        const C c = t4 + t5 + t6, o = np1 * C(0.5);
        gp[1] = c + o; gp[2] = c - o;
    }
    {
        const C c = t4 - C(2.0) * t5 + t6, o = np2 * C(0.5);
        gp[3] = c + o; gp[4] = c - o;
    }
    {
        const C c = t4 + t5 - C(2.0) * t6, o = np3 * C(0.5);
        gp[5] = c + o; gp[6] = c - o;
    }
}
#endif

// macro_u / macro_t (3M:988-1025) in the reference's operation order
template <class C, bool DEV = false, bool DEVT = false>
__device__ __forceinline__ void macro3d(const C f[19], const C gg[7], C Fz0, const Geo &G, C &rho, C &u, C &v,
                                        C &w, C &T, C Tc = C(0.0))
{
    const C dt = C(G.dt);
    rho = (DEV ? C(1.0) : C(0.0)) + f[0]+f[1]+f[2]+f[3]+f[4]+f[5]+f[6]+f[7]+f[8]+f[9]+f[10]+f[11]+f[12]+f[13]+f[14]+f[15]+f[16]+f[17]+f[18];
#if LBM_EXACT
    u = (f[1]-f[2]+f[7]-f[8]+f[9]-f[10]+f[11]-f[12]+f[13]-f[14])/rho;
    v = (f[3]-f[4]+f[7]+f[8]-f[9]-f[10]+f[15]-f[16]+f[17]-f[18])/rho;
    w = (f[5]-f[6]+f[11]+f[12]-f[13]-f[14]+f[15]+f[16]-f[17]-f[18]+C(0.5)*dt*Fz0)/rho;
#else
    const C rinv = C(1.0) / rho;
    u = (f[1]-f[2]+f[7]-f[8]+f[9]-f[10]+f[11]-f[12]+f[13]-f[14])*rinv;
    v = (f[3]-f[4]+f[7]+f[8]-f[9]-f[10]+f[15]-f[16]+f[17]-f[18])*rinv;
    w = (f[5]-f[6]+f[11]+f[12]-f[13]-f[14]+f[15]+f[16]-f[17]-f[18]+C(0.5)*dt*Fz0)*rinv;
#endif
    T = DEVT ? Tc + (gg[0]+gg[1]+gg[2]+gg[3]+gg[4]+gg[5]+gg[6]) : gg[0]+gg[1]+gg[2]+gg[3]+gg[4]+gg[5]+gg[6];
}

// macro + collision of one node: the reference's order in the exact build,
// the shared-subexpression form in the fast build
template <class C, bool DEV = false, bool DEVT = false>
__device__ __forceinline__ void node3d(const C f[19], const C gg[7], C Fz0, const Geo &G, C fp[19], C gp[7], C &Fz,
                                       C &rho, C &u, C &v, C &w, C &T, C Tc = C(0.0))
{
#if LBM_EXACT
    macro3d<C, DEV, DEVT>(f, gg, Fz0, G, rho, u, v, w, T, Tc);
    collide3d<C, DEV, DEVT>(f, gg, rho, u, v, w, T, G, fp, gp, Fz);
#else
    node3d_fast<C, DEV, DEVT>(f, gg, Fz0, G, fp, gp, Fz, rho, u, v, w, T, Tc);
#endif
}

template <int ST, int KIND>
__global__ void __launch_bounds__(256)
k_step3d(const Geo G, const typename Tr<ST>::S *__restrict__ src, const typename Tr<ST>::C *__restrict__ Fin,
         typename Tr<ST>::S *__restrict__ dst, typename Tr<ST>::C *__restrict__ Fout, const Bufs B,
         int write_macro)
{
    using S = typename Tr<ST>::S;
    using C = typename Tr<ST>::C;
    if (!B.ctl->active) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = G.klo + blockIdx.z;  // a slab's ghost slices come from its neighbours
    if (i >= G.nx || j >= G.ny) return;
    const int64_t P = G.plane;
    const int64_t id = (int64_t)k * G.slab + (int64_t)j * G.pitch + i;
    const int64_t xa = off_a(i, G.nx), xb = off_b(i, G.nx);
    const int64_t ya = (int64_t)off_a(j, G.ny) * G.pitch, yb = (int64_t)off_b(j, G.ny) * G.pitch;
    const int64_t za = (int64_t)off_a(k, G.nz) * G.slab, zb = (int64_t)off_b(k, G.nz) * G.slab;
    C xp[3], xm[3], yp[3], ym[3], zp[3], zm[3];
    load_w(G.wgt[0], i, xp, xm);
    load_w(G.wgt[1], j, yp, ym);
    load_w(G.wgt[2], k, zp, zm);

    auto LD = [&](int q, int64_t off) -> C {
        C val = tocomp(__ldg(src + q * P + id + off));
        return val;
    };
    auto YI = [&](int q, const C w[3], int64_t c) -> C { return ip(w, LD(q, c + ya), LD(q, c), LD(q, c + yb)); };
    auto ZI = [&](int q, const C w[3], int64_t c) -> C { return ip(w, LD(q, c + za), LD(q, c), LD(q, c + zb)); };

    C f[19], gg[7];
    f[0] = LD(0, 0);
    // axis directions: one-dimensional interpolation (the zero-shift axis
    // weights of the reference's in-plane scheme are exactly (0, 1, 0))
    f[1] = ip(xp, LD(1, xa), LD(1, 0), LD(1, xb));
    f[2] = ip(xm, LD(2, xa), LD(2, 0), LD(2, xb));
    f[3] = ip(yp, LD(3, ya), LD(3, 0), LD(3, yb));
    f[4] = ip(ym, LD(4, ya), LD(4, 0), LD(4, yb));
    f[5] = ip(zp, LD(5, za), LD(5, 0), LD(5, zb));
    f[6] = ip(zm, LD(6, za), LD(6, 0), LD(6, zb));
    // xoy plane (3M:807-824): y-interpolation on three x-columns, then x
    f[7] = ip(xp, YI(7, yp, xa), YI(7, yp, 0), YI(7, yp, xb));
    f[8] = ip(xm, YI(8, yp, xa), YI(8, yp, 0), YI(8, yp, xb));
    f[9] = ip(xp, YI(9, ym, xa), YI(9, ym, 0), YI(9, ym, xb));
    f[10] = ip(xm, YI(10, ym, xa), YI(10, ym, 0), YI(10, ym, xb));
    // xoz plane (3M:787-804): z-interpolation on three x-columns, then x
    f[11] = ip(xp, ZI(11, zp, xa), ZI(11, zp, 0), ZI(11, zp, xb));
    f[12] = ip(xm, ZI(12, zp, xa), ZI(12, zp, 0), ZI(12, zp, xb));
    f[13] = ip(xp, ZI(13, zm, xa), ZI(13, zm, 0), ZI(13, zm, xb));
    f[14] = ip(xm, ZI(14, zm, xa), ZI(14, zm, 0), ZI(14, zm, xb));
    // yoz plane (3M:767-784): z-interpolation on three y-rows, then y
    f[15] = ip(yp, ZI(15, zp, ya), ZI(15, zp, 0), ZI(15, zp, yb));
    f[16] = ip(ym, ZI(16, zp, ya), ZI(16, zp, 0), ZI(16, zp, yb));
    f[17] = ip(yp, ZI(17, zm, ya), ZI(17, zm, 0), ZI(17, zm, yb));
    f[18] = ip(ym, ZI(18, zm, ya), ZI(18, zm, 0), ZI(18, zm, yb));
    // D3Q7 (3M:831-859)
    gg[0] = LD(19, 0);
    gg[1] = ip(xp, LD(20, xa), LD(20, 0), LD(20, xb));
    gg[2] = ip(xm, LD(21, xa), LD(21, 0), LD(21, xb));
    gg[3] = ip(yp, LD(22, ya), LD(22, 0), LD(22, yb));
    gg[4] = ip(ym, LD(23, ya), LD(23, 0), LD(23, yb));
    gg[5] = ip(zp, LD(24, za), LD(24, 0), LD(24, zb));
    gg[6] = ip(zm, LD(25, za), LD(25, 0), LD(25, zb));
    // deviation from the conduction profile along y (the heated axis)
    C Tc = C(0.0);
    if (Tr<ST>::kDevT) {
        Tc = C(tc_value(G, j));
        const C sT = C((1.0 / 12.0) * G.dt * tc_gradient(G));
        gg[3] -= sT;
        gg[4] += sT;
    }

    // walls: bounceback_u (3B:1053-1136), bounceback_T (3B:1138-1197)
    const C two_wT = C(2.0) * (C(1.0) / C(12.0));
    if (j == 0) {
        f[3] = LD(4, 0); f[7] = LD(10, 0); f[8] = LD(9, 0); f[15] = LD(18, 0); f[17] = LD(16, 0);
        gg[3] = -LD(23, 0) + two_wT * (Tr<ST>::kDevT ? C(G.Thot) - Tc : C(G.Thot));
    }
    if (j == G.ny - 1) {
        f[4] = LD(3, 0); f[9] = LD(8, 0); f[10] = LD(7, 0); f[16] = LD(17, 0); f[18] = LD(15, 0);
        gg[4] = -LD(22, 0) + two_wT * (Tr<ST>::kDevT ? C(G.Tcold) - Tc : C(G.Tcold));
    }
    if (i == 0) {
        f[1] = LD(2, 0); f[9] = LD(8, 0); f[7] = LD(10, 0); f[13] = LD(12, 0); f[11] = LD(14, 0);
        gg[1] = LD(21, 0);
    }
    if (i == G.nx - 1) {
        f[2] = LD(1, 0); f[8] = LD(9, 0); f[10] = LD(7, 0); f[12] = LD(13, 0); f[14] = LD(11, 0);
        gg[2] = LD(20, 0);
    }
    if (k == 0) {
        f[5] = LD(6, 0); f[11] = LD(14, 0); f[12] = LD(13, 0); f[15] = LD(18, 0); f[16] = LD(17, 0);
        gg[5] = LD(25, 0);
    }
    if (k == G.nz - 1) {
        f[6] = LD(5, 0); f[13] = LD(12, 0); f[14] = LD(11, 0); f[17] = LD(16, 0); f[18] = LD(15, 0);
        gg[6] = LD(24, 0);
    }

    // macro_u / macro_t (3M:988-1025) and the collision
    const C Fz0 = Fin[id];
    C rho, u, v, w, T, fp[19], gp[7], Fz;
    if (LBM_EXACT || KIND == 1) {
        macro3d<C, Tr<ST>::kShift, Tr<ST>::kDevT>(f, gg, Fz0, G, rho, u, v, w, T, Tc);
        if (KIND == 0) collide3d<C, Tr<ST>::kShift, Tr<ST>::kDevT>(f, gg, rho, u, v, w, T, G, fp, gp, Fz);
    } else {
        node3d<C, Tr<ST>::kShift, Tr<ST>::kDevT>(f, gg, Fz0, G, fp, gp, Fz, rho, u, v, w, T, Tc);
    }
    if (write_macro || KIND == 1) {
        const int64_t mid = ((int64_t)k * G.ny + j) * G.nx + i;
        B.rho[mid] = double(rho); B.u[mid] = double(u); B.v[mid] = double(v);
        B.w[mid] = double(w); B.T[mid] = double(T);
    }
    auto ST_ = [&](int q, C val) {
        dst[q * P + id] = tostore<S, C>(val);
    };
    if (KIND == 1) {
#pragma unroll
        for (int q = 0; q < 19; ++q) ST_(q, f[q]);
#pragma unroll
        for (int q = 0; q < 7; ++q) ST_(19 + q, gg[q]);
        return;
    }
    Fout[id] = Fz;
#pragma unroll
    for (int q = 0; q < 19; ++q) ST_(q, fp[q]);
#pragma unroll
    for (int q = 0; q < 7; ++q) ST_(19 + q, gp[q]);
}

// ---------------------------------------------------------------------------
// initial equilibrium (2M:227-240, 3M:286-301) and the first collision
// ---------------------------------------------------------------------------
// d/dc at c = xm of the quadratic through (xa, qa), (xm, qm), (xb, qb)
__device__ __forceinline__ double slope3(double xa, double qa, double xm, double qm, double xb, double qb)
{
    const double la = (xm - xb) / ((xa - xm) * (xa - xb));
    const double lm = ((xm - xa) + (xm - xb)) / ((xm - xa) * (xm - xb));
    const double lb = (xm - xa) / ((xb - xa) * (xb - xm));
    return (qa * la + qm * lm) + qb * lb;
}

// gradient of a packed field q at node n = (i, j, k) (0-based) along the
// three-node interpolation stencil of each axis (one-sided at both ends)
__device__ __forceinline__ void grad3(const Geo &G, const double *__restrict__ q, int64_t n, int i, int j, int k,
                                      double out[3])
{
    const int64_t sx = 1, sy = G.nx, sz = (int64_t)G.nx * G.ny;
    const int ii[3] = {i, j, k};
    const int nn[3] = {G.nx, G.ny, G.nz};
    const int64_t st[3] = {sx, sy, sz};
    for (int ax = 0; ax < 3; ++ax) {
        if (ax == 2 && G.dim != 3) {
            out[2] = 0.0;
            break;
        }
        const int m = ii[ax] + 1;  // 1-based node of the coordinate table
        int a, b;
        if (m == 1) { a = m + 1; b = m + 2; }
        else if (m == nn[ax]) { a = m - 1; b = m - 2; }
        else { a = m - 1; b = m + 1; }
        const double *c = G.coord[ax];
        out[ax] = slope3(c[a], q[n + (a - m) * st[ax]], c[m], q[n], c[b], q[n + (b - m) * st[ax]]);
    }
}

// Equilibrium populations of initial() (2M:227-240 / 3M:286-301) from the
// macroscopic fields in B; with neq != 0 plus the first-order Chapman-Enskog
// non-equilibrium part from the fields' gradients (warm starts):
//   f_a -= (cf w_a rho) (e_a e_a : grad u - div u / 3),  cf = 3 tau_f dt
//   g_a -= (ct wT_a) (e_a . grad T),                     ct = dt / sig_k
template <int ST>
__global__ void k_equilibrium(const Geo G, typename Tr<ST>::S *__restrict__ pop, const Bufs B, int neq, double cf,
                              double ct)
{
    using S = typename Tr<ST>::S;
    using C = typename Tr<ST>::C;
    const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= G.nnode) return;
    const int i = int(n % G.nx);
    const int j = int((n / G.nx) % G.ny);
    const int k = int(n / ((int64_t)G.nx * G.ny));
    const int64_t id = (int64_t)k * G.slab + (int64_t)j * G.pitch + i;
    const int64_t P = G.plane;
    // FP64 here in every storage mode: the initial state is formed once
    const double rho = B.rho[n], u = B.u[n], v = B.v[n], T = B.T[n];
    const double w = G.dim == 3 ? B.w[n] : 0.0;
    if (G.dim == 2) {
        const int ex[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
        const int ey[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
        const double wU[9] = {4.0/9.0, 1.0/9.0, 1.0/9.0, 1.0/9.0, 1.0/9.0, 1.0/36.0, 1.0/36.0, 1.0/36.0, 1.0/36.0};
        const double wT[5] = {1.0/2.0, 1.0/8.0, 1.0/8.0, 1.0/8.0, 1.0/8.0};
        const double velocitySquare = u*u+v*v;
        double gu[3] = {0.0, 0.0, 0.0}, gv[3] = {0.0, 0.0, 0.0}, gT[3] = {0.0, 0.0, 0.0};
        if (neq) {
            grad3(G, B.u, n, i, j, k, gu);
            grad3(G, B.v, n, i, j, k, gv);
            grad3(G, B.T, n, i, j, k, gT);
        }
        const double div = (gu[0] + gv[1]) + 0.0;
        for (int a = 0; a < 9; ++a) {
            const double un = u*ex[a]+v*ey[a];
            double fa = rho*wU[a]*(1.0+3.0*un+4.5*un*un-1.5*velocitySquare);
            if (neq) {
                const double exa = ex[a], eya = ey[a];
                double qq = (exa * exa) * gu[0] + (exa * eya) * (gv[0] + gu[1]) + (eya * eya) * gv[1];
                qq = qq - div / 3.0;
                fa = fa - ((cf * wU[a]) * rho) * qq;
            }
            if (Tr<ST>::kShift) fa -= wU[a];
            pop[a * P + id] = tostore<S, C>(C(fa));
        }
        for (int a = 0; a < 5; ++a) {
            const double un = u*ex[a]+v*ey[a];
            double ga = wT[a]*T*(1.0+4.0*un);
            if (neq) {
                const double en = (ex[a] * gT[0] + ey[a] * gT[1]) + 0 * gT[2];
                ga = ga - (ct * wT[a]) * en;
            }
            if (Tr<ST>::kDevT) ga -= wT[a] * tc_value(G, i);
            pop[(9 + a) * P + id] = tostore<S, C>(C(ga));
        }
    } else {
        const int ex[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
        const int ey[19] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1};
        const int ez[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};
        const double us2 = u*u+v*v+w*w;
        double gu[3] = {0.0, 0.0, 0.0}, gv[3] = {0.0, 0.0, 0.0}, gw[3] = {0.0, 0.0, 0.0}, gT[3] = {0.0, 0.0, 0.0};
        if (neq) {
            grad3(G, B.u, n, i, j, k, gu);
            grad3(G, B.v, n, i, j, k, gv);
            grad3(G, B.w, n, i, j, k, gw);
            grad3(G, B.T, n, i, j, k, gT);
        }
        const double div = (gu[0] + gv[1]) + gw[2];
        for (int a = 0; a < 19; ++a) {
            const double wa = a == 0 ? 1.0/3.0 : (a < 7 ? 1.0/18.0 : 1.0/36.0);
            const double un = u*ex[a]+v*ey[a]+w*ez[a];
            double fa = wa*rho*(1.0+3.0*un+4.5*un*un-1.5*us2);
            if (neq) {
                const double exa = ex[a], eya = ey[a], eza = ez[a];
                double qq = (exa * exa) * gu[0] + (exa * eya) * (gv[0] + gu[1]) + (eya * eya) * gv[1];
                qq = ((qq + (eza * eza) * gw[2]) + (exa * eza) * (gw[0] + gu[2])) + (eya * eza) * (gw[1] + gv[2]);
                qq = qq - div / 3.0;
                fa = fa - ((cf * wa) * rho) * qq;
            }
            if (Tr<ST>::kShift) fa -= wa;
            pop[a * P + id] = tostore<S, C>(C(fa));
        }
        for (int a = 0; a < 7; ++a) {
            const double wa = a == 0 ? 1.0/2.0 : 1.0/12.0;
            const double un = u*ex[a]+v*ey[a]+w*ez[a];
            double ga = wa*T*(1.0+6.0*un);
            if (neq) {
                const double en = (ex[a] * gT[0] + ey[a] * gT[1]) + ez[a] * gT[2];
                ga = ga - (ct * wa) * en;
            }
            if (Tr<ST>::kDevT) ga -= wa * tc_value(G, j);
            pop[(19 + a) * P + id] = tostore<S, C>(C(ga));
        }
    }
}

// The first collision of a run, from pre-collision populations and the
// macroscopic fields held in B (what the reference's loop starts from).
template <int ST>
__global__ void k_collide(const Geo G, const typename Tr<ST>::S *__restrict__ in,
                          typename Tr<ST>::S *__restrict__ out, typename Tr<ST>::C *__restrict__ Fout,
                          const Bufs B)
{
    using S = typename Tr<ST>::S;
    using C = typename Tr<ST>::C;
    const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= G.nnode) return;
    const int i = int(n % G.nx);
    const int j = int((n / G.nx) % G.ny);
    const int k = int(n / ((int64_t)G.nx * G.ny));
    const int64_t id = (int64_t)k * G.slab + (int64_t)j * G.pitch + i;
    const int64_t P = G.plane;
    const int Q = G.dim == 2 ? 9 : 19, QT = G.dim == 2 ? 5 : 7;
    C f[19], gg[7], fp[19], gp[7], F;
    // reduced-precision storage: the populations stay deviations (see the storage note above)
    for (int q = 0; q < Q; ++q) f[q] = tocomp(in[q * P + id]);
    for (int q = 0; q < QT; ++q) gg[q] = tocomp(in[(Q + q) * P + id]);
    const C rho = C(B.rho[n]), u = C(B.u[n]), v = C(B.v[n]), T = C(B.T[n]);
    if (G.dim == 2) {
        collide2d<C, Tr<ST>::kShift, Tr<ST>::kDevT>(f, gg, rho, u, v, T, G, fp, gp, F);
    } else {
        const C w = C(B.w[n]);
        collide3d<C, Tr<ST>::kShift, Tr<ST>::kDevT>(f, gg, rho, u, v, w, T, G, fp, gp, F);
    }
    Fout[id] = F;
    for (int q = 0; q < Q; ++q) out[q * P + id] = tostore<S, C>(fp[q]);
    for (int q = 0; q < QT; ++q) out[(Q + q) * P + id] = tostore<S, C>(gp[q]);
}

#include "lbm_march.cuh"

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
template <int ST>
static cudaError_t launch_step(const Geo &g, const void *pin, const void *Fin, void *pout, void *Fout,
                               const Bufs &b, int wm, int kind, cudaStream_t s)
{
    using S = typename Tr<ST>::S;
    using C = typename Tr<ST>::C;
    dim3 blk(32, 8, 1);
    if (g.dim == 2) {
        dim3 grd((g.nx + 31) / 32, (g.ny + 7) / 8, 1);
        if (kind == 0)
            k_step2d<ST, 0><<<grd, blk, 0, s>>>(g, (const S *)pin, (const C *)Fin, (S *)pout, (C *)Fout, b, wm);
        else
            k_step2d<ST, 1><<<grd, blk, 0, s>>>(g, (const S *)pin, (const C *)Fin, (S *)pout, (C *)Fout, b, wm);
    } else {
        dim3 grd((g.nx + 31) / 32, (g.ny + 7) / 8, g.khi - g.klo);
        if (kind == 0)
            k_step3d<ST, 0><<<grd, blk, 0, s>>>(g, (const S *)pin, (const C *)Fin, (S *)pout, (C *)Fout, b, wm);
        else
            k_step3d<ST, 1><<<grd, blk, 0, s>>>(g, (const S *)pin, (const C *)Fin, (S *)pout, (C *)Fout, b, wm);
    }
    ++g_launches;
    return cudaGetLastError();
}

#if LBM_EXACT
#define LBM_DISPATCH(store, CALL)                          \
    switch (store) {                                       \
    case kF64: return CALL(kF64);                          \
    default: return cudaErrorNotSupported;                 \
    }
#else
#define LBM_DISPATCH(store, CALL)                          \
    switch (store) {                                       \
    case kF64: return CALL(kF64);                          \
    case kF32: return CALL(kF32);                          \
    default: return cudaErrorNotSupported;                 \
    }
#endif

cudaError_t step(const Geo &g, int store, const void *pop_in, const void *F_in, void *pop_out, void *F_out,
                 const Bufs &b, int write_macro, cudaStream_t s)
{
#define CALL(ST) launch_step<ST>(g, pop_in, F_in, pop_out, F_out, b, write_macro, 0, s)
    LBM_DISPATCH(store, CALL)
#undef CALL
}

template <int ST>
static cudaError_t launch_resident(const Geo &g, void *const pop[2], void *const F[2], const Bufs &b, int cur,
                                   int nsteps, unsigned *bar, int *err, int nblocks, cudaStream_t s)
{
    using S = typename Tr<ST>::S;
    using C = typename Tr<ST>::C;
    S *p0 = (S *)pop[0], *p1 = (S *)pop[1];
    C *F0 = (C *)F[0], *F1 = (C *)F[1];
    Geo gg = g;
    Bufs bb = b;
    void *args[] = {&gg, &p0, &p1, &F0, &F1, &bb, &cur, &nsteps, &bar, &err};
    ++g_launches;
    return cudaLaunchCooperativeKernel((const void *)k_steps2d_resident<ST>, dim3(nblocks), dim3(256), args, 0, s);
}

cudaError_t steps_resident(const Geo &g, int store, void *const pop[2], void *const F[2], const Bufs &b, int cur,
                           int nsteps, unsigned *bar, int *err, int nblocks, cudaStream_t s)
{
#define CALL(ST) launch_resident<ST>(g, pop, F, b, cur, nsteps, bar, err, nblocks, s)
    LBM_DISPATCH(store, CALL)
#undef CALL
}

int resident_blocks(const Geo &g, int store, int device)
{
    int bps = 0, sms = 0;
    cudaError_t e = cudaErrorNotSupported;
    switch (store) {
    case kF64: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_steps2d_resident<kF64>, 256, 0); break;
    case kF32: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_steps2d_resident<kF32>, 256, 0); break;
    default: break;
    }
    if (e != cudaSuccess || bps <= 0) return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
    const int64_t need = ((int64_t)g.nx * g.ny + 255) / 256;
    const int64_t cap = (int64_t)bps * sms;
    return (int)(need < cap ? need : cap);
}

cudaError_t stream_only(const Geo &g, int store, const void *pop_in, const void *F_in, void *pop_out,
                        const Bufs &b, cudaStream_t s)
{
#define CALL(ST) launch_step<ST>(g, pop_in, F_in, pop_out, nullptr, b, 1, 1, s)
    LBM_DISPATCH(store, CALL)
#undef CALL
}

template <int ST>
static cudaError_t launch_eq(const Geo &g, void *pop, const Bufs &b, int neq, double cf, double ct, cudaStream_t s)
{
    const int64_t n = g.nnode;
    k_equilibrium<ST><<<unsigned((n + 255) / 256), 256, 0, s>>>(g, (typename Tr<ST>::S *)pop, b, neq, cf, ct);
    ++g_launches;
    return cudaGetLastError();
}

cudaError_t equilibrium(const Geo &g, int store, void *pop, const Bufs &b, int neq, double cf, double ct,
                        cudaStream_t s)
{
#define CALL(ST) launch_eq<ST>(g, pop, b, neq, cf, ct, s)
    LBM_DISPATCH(store, CALL)
#undef CALL
}

template <int ST>
static cudaError_t launch_collide(const Geo &g, const void *in, void *out, void *Fout, const Bufs &b,
                                  cudaStream_t s)
{
    const int64_t n = g.nnode;
    k_collide<ST><<<unsigned((n + 127) / 128), 128, 0, s>>>(g, (const typename Tr<ST>::S *)in,
                                                          (typename Tr<ST>::S *)out,
                                                          (typename Tr<ST>::C *)Fout, b);
    ++g_launches;
    return cudaGetLastError();
}

cudaError_t collide(const Geo &g, int store, const void *pop_in, void *pop_out, void *F_out, const Bufs &b,
                    cudaStream_t s)
{
#define CALL(ST) launch_collide<ST>(g, pop_in, pop_out, F_out, b, s)
    LBM_DISPATCH(store, CALL)
#undef CALL
}

// Launch of a march kernel.  With `pdl` the launch carries the
// programmatic-serialization attribute: the kernel's CTAs may be scheduled
// while the stream's previous kernel drains (its CTAs call dep_launch at
// their start) and wait in dep_wait, after their set-up, for that kernel's
// completion.  Consecutive steps then overlap one kernel's launch and set-up
// with the previous one's tail.
template <typename... KArgs, typename... Args>
static cudaError_t launch_k(void (*k)(KArgs...), int grid, int block, int smem, cudaStream_t s, bool pdl,
                            Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = (size_t)smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = pdl ? at : nullptr;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, k, args...);
}

template <int ST, int TY>
static cudaError_t prepare_march3d()
{
    static bool done = false;
    if (!done) {
        cudaError_t e = cudaFuncSetAttribute(k_march3d<ST, TY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             L3<ST, TY>::smem());
        if (e != cudaSuccess) return e;
        done = true;
    }
    return cudaSuccess;
}

template <int ST, class L>
static cudaError_t prepare_march2d()
{
    static bool done = false;
    if (!done) {
        cudaError_t e = cudaFuncSetAttribute(k_march2d<ST, L>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             L::smem());
        if (e != cudaSuccess) return e;
        done = true;
    }
    return cudaSuccess;
}

template <int ST, int TY>
static int mbps3(void)
{
    if (prepare_march3d<ST, TY>() != cudaSuccess) return 0;
    int n = 0;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_march3d<ST, TY>, L3<ST, TY>::NT,
                                                         L3<ST, TY>::smem()) == cudaSuccess
               ? n
               : 0;
}

template <int ST, class L>
static int mbps2(void)
{
    if (prepare_march2d<ST, L>() != cudaSuccess) return 0;
    int n = 0;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_march2d<ST, L>, L::NT, L::smem()) == cudaSuccess ? n
                                                                                                             : 0;
}

template <int ST>
static int mbps(const Geo &g, int ty)
{
    if (g.dim == 3) return ty == 4 ? mbps3<ST, 4>() : mbps3<ST, 8>();
    return g.nnode >= kDeepRingNodes ? mbps2<ST, L2d<ST>>() : mbps2<ST, L2s<ST>>();
}

int march_blocks_per_sm(const Geo &g, int store, int ty)
{
#define CALL(ST) mbps<ST>(g, ty)
    LBM_DISPATCH(store, CALL)
#undef CALL
}

template <int ST, int TY>
static cudaError_t launch_march3d(const Geo &g, const TmapSet &m, const void *Fin, void *pout, void *Fout,
                                  const Bufs &b, int wm, const int4 *segs, const int *segoff, int nblocks,
                                  bool pdl, cudaStream_t s)
{
    using S = typename Tr<ST>::S;
    using C = typename Tr<ST>::C;
    cudaError_t e = prepare_march3d<ST, TY>();
    if (e != cudaSuccess) return e;
    return launch_k(k_march3d<ST, TY>, nblocks, L3<ST, TY>::NT, L3<ST, TY>::smem(), s, pdl, m, g, (const C *)Fin,
                    (S *)pout, (C *)Fout, b, wm, segs, segoff, b.err);
}

template <int ST, class L>
static cudaError_t launch_march2d(const Geo &g, const TmapSet &m, const void *Fin, void *pout, void *Fout,
                                  const Bufs &b, int wm, int nblocks, bool pdl, cudaStream_t s)
{
    using S = typename Tr<ST>::S;
    using C = typename Tr<ST>::C;
    cudaError_t e = prepare_march2d<ST, L>();
    if (e != cudaSuccess) return e;
    const int64_t total = (int64_t)((g.nx + L::TX - 1) / L::TX) * (g.jhi - g.jlo);
    const int nb = int(nblocks < total ? nblocks : total);
    return launch_k(k_march2d<ST, L>, nb, L::NT, L::smem(), s, pdl, m, g, (const C *)Fin, (S *)pout, (C *)Fout, b,
                    wm, total, b.err);
}

template <int ST>
static cudaError_t launch_march(const Geo &g, const TmapSet &m, const void *Fin, void *pout, void *Fout,
                                const Bufs &b, int wm, int nblocks, int ty, const int4 *segs, const int *segoff,
                                bool pdl, cudaStream_t s)
{
    using S = typename Tr<ST>::S;
    using C = typename Tr<ST>::C;
    cudaError_t e;
    if (g.dim == 3) {
        e = ty == 4 ? launch_march3d<ST, 4>(g, m, Fin, pout, Fout, b, wm, segs, segoff, nblocks, pdl, s)
                    : launch_march3d<ST, 8>(g, m, Fin, pout, Fout, b, wm, segs, segoff, nblocks, pdl, s);
    } else {
        e = g.nnode >= kDeepRingNodes ? launch_march2d<ST, L2d<ST>>(g, m, Fin, pout, Fout, b, wm, nblocks, pdl, s)
                                      : launch_march2d<ST, L2s<ST>>(g, m, Fin, pout, Fout, b, wm, nblocks, pdl, s);
    }
    ++g_launches;
    return e;
}

cudaError_t march(const Geo &g, int store, const TmapSet &src, const void *F_in, void *pop_out, void *F_out,
                  const Bufs &b, int write_macro, int nblocks, int ty, const int4 *segs, const int *segoff,
                  bool pdl, cudaStream_t s)
{
#define CALL(ST) launch_march<ST>(g, src, F_in, pop_out, F_out, b, write_macro, nblocks, ty, segs, segoff, pdl, s)
    LBM_DISPATCH(store, CALL)
#undef CALL
}

template <int ST, int TX>
static cudaError_t prepare_batch()
{
    static bool done = false;
    if (!done) {
        cudaError_t e = cudaFuncSetAttribute(k_march2d_batch<ST, TX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             L2<ST, TX>::smem());
        if (e != cudaSuccess) return e;
        done = true;
    }
    return cudaSuccess;
}

template <int ST, int TX>
static cudaError_t launch_batch(const BatchDev &D, int nblocks, int cur, int wm, int *err, bool pdl, cudaStream_t s)
{
    cudaError_t e = prepare_batch<ST, TX>();
    if (e != cudaSuccess) return e;
    ++g_launches;
    return launch_k(k_march2d_batch<ST, TX>, nblocks, TX, L2<ST, TX>::smem(), s, pdl, D, cur, wm, err);
}

template <int ST, int TX>
static int batch_bps()
{
    if (prepare_batch<ST, TX>() != cudaSuccess) return 0;
    int n = 0;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_march2d_batch<ST, TX>, TX, L2<ST, TX>::smem()) ==
                   cudaSuccess
               ? n
               : 0;
}

template <int ST>
static cudaError_t launch_batch_tx(int TX, const BatchDev &D, int nblocks, int cur, int wm, int *err, bool pdl,
                                   cudaStream_t s)
{
    switch (TX) {
    case 32: return launch_batch<ST, 32>(D, nblocks, cur, wm, err, pdl, s);
    case 64: return launch_batch<ST, 64>(D, nblocks, cur, wm, err, pdl, s);
    case 128: return launch_batch<ST, 128>(D, nblocks, cur, wm, err, pdl, s);
    default: return cudaErrorInvalidValue;
    }
}

template <int ST>
static int batch_bps_tx(int TX)
{
    switch (TX) {
    case 32: return batch_bps<ST, 32>();
    case 64: return batch_bps<ST, 64>();
    case 128: return batch_bps<ST, 128>();
    default: return 0;
    }
}

cudaError_t march_batch(int store, int TX, const BatchDev &D, int nblocks, int cur, int write_macro, int *err,
                        bool pdl, cudaStream_t s)
{
#define CALL(ST) launch_batch_tx<ST>(TX, D, nblocks, cur, write_macro, err, pdl, s)
    LBM_DISPATCH(store, CALL)
#undef CALL
}

int march_batch_blocks_per_sm(int store, int TX)
{
#define CALL(ST) batch_bps_tx<ST>(TX)
    LBM_DISPATCH(store, CALL)
#undef CALL
}

template <int ST>
static cudaError_t prepare_batch3d()
{
    static bool done = false;
    if (!done) {
        cudaError_t e = cudaFuncSetAttribute(k_march3d_batch<ST, kBatchTileY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             L3<ST, kBatchTileY>::smem());
        if (e != cudaSuccess) return e;
        done = true;
    }
    return cudaSuccess;
}

template <int ST>
static cudaError_t launch_batch3d(const BatchDev &D, int nblocks, int cur, int wm, int *err, bool pdl,
                                  cudaStream_t s)
{
    cudaError_t e = prepare_batch3d<ST>();
    if (e != cudaSuccess) return e;
    ++g_launches;
    return launch_k(k_march3d_batch<ST, kBatchTileY>, nblocks, L3<ST, kBatchTileY>::NT, L3<ST, kBatchTileY>::smem(),
                    s, pdl, D, cur, wm, err);
}

template <int ST>
static int batch3d_bps()
{
    if (prepare_batch3d<ST>() != cudaSuccess) return 0;
    int n = 0;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_march3d_batch<ST, kBatchTileY>, L3<ST, kBatchTileY>::NT,
                                                         L3<ST, kBatchTileY>::smem()) == cudaSuccess
               ? n
               : 0;
}

cudaError_t march_batch3d(int store, const BatchDev &D, int nblocks, int cur, int write_macro, int *err,
                          bool pdl, cudaStream_t s)
{
#define CALL(ST) launch_batch3d<ST>(D, nblocks, cur, write_macro, err, pdl, s)
    LBM_DISPATCH(store, CALL)
#undef CALL
}

int march_batch3d_blocks_per_sm(int store)
{
#define CALL(ST) batch3d_bps<ST>()
    LBM_DISPATCH(store, CALL)
#undef CALL
}

cudaError_t set_wait_limit(long long cycles)
{
    if (cycles <= 0) cycles = kWaitCycles;
    return cudaMemcpyToSymbol(g_wait_limit, &cycles, sizeof cycles);
}

}  // namespace LBM_NS

#if !LBM_EXACT
// tile shapes of the march kernels, for the host's tensor-map encoding
MarchShape march_shape(int dim, int store, int tx, int ty)
{
    MarchShape m{};
    auto fill = [&](auto layout, int dims) {
        using L = decltype(layout);
        m.TX = L::TX;
        m.TY = dims == 3 ? (ty == 4 ? 4 : 8) : 1;
        m.HX = L::HX;
        m.threads = L::NT;
        m.smem = L::smem();
    };
    if (dim == 3) {
        if (ty == 4) {
            switch (store) {
            case kF64: fill(fast::L3<kF64, 4>{}, 3); break;
            case kF32: fill(fast::L3<kF32, 4>{}, 3); break;
            default: fill(fast::L3<kF32, 4>{}, 3); break;
            }
        } else {
            switch (store) {
            case kF64: fill(fast::L3<kF64, 8>{}, 3); break;
            case kF32: fill(fast::L3<kF32, 8>{}, 3); break;
            default: fill(fast::L3<kF32, 8>{}, 3); break;
            }
        }
        for (int c = 0; c < 4; ++c) {
            m.bx[c] = m.TX + ((c & 1) ? 2 * m.HX : 0);
            m.by[c] = m.TY + ((c & 2) ? 2 : 0);
        }
    } else {
#define LBM_FILL2(...)                                                    \
        switch (store) {                                                  \
        case kF64: fill(fast::L2<kF64, __VA_ARGS__>{}, 2); break;         \
        case kF32: fill(fast::L2<kF32, __VA_ARGS__>{}, 2); break;         \
        default: fill(fast::L2<kF32, __VA_ARGS__>{}, 2); break;           \
        }
        if (tx == 32) { LBM_FILL2(32) }
        else if (tx == 64) { LBM_FILL2(64) }
        else { LBM_FILL2(128) }
#undef LBM_FILL2
        for (int c = 0; c < 4; ++c) {
            m.bx[c] = m.TX + ((c & 1) ? 2 * m.HX : 0);
            m.by[c] = 1;
        }
    }
    return m;
}
#endif

}  // namespace lbm
