// Internal interface between the C ABI (lbm_capi.cu) and the kernels
// (lbm_kernels.cu, compiled once per arithmetic mode).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

namespace lbm {

// Geometry and physics constants a kernel needs, passed by value.
struct Geo {
    int dim, nx, ny, nz;
    int jlo, jhi;    // 2D: the rows the step kernels compute and the reductions sum, [jlo, jhi):
                     // 0, ny for a whole cavity; a slab (lbm_create_slab) leaves out its ghost rows
    int klo, khi;    // 3D: the z-slices the step kernels compute and the reductions sum, [klo, khi):
                     // 0, nz for a whole cavity; a 3D slab leaves out its ghost slices
    int64_t pitch;   // elements between rows of a population plane
    int64_t slab;    // elements between z-planes (pitch * ny)
    int64_t plane;   // elements between population planes
    int64_t nnode;   // nx*ny*nz: packed macro arrays, x fastest
    double Snu, Sq, sig_k, gbeta, dt, Thot, Tcold, T0, length_LB;
    double tc_lo, tc_grad;   // conduction profile: hot wall position and dTc per lattice unit (tc_setup)
    const double *wgt[3];    // per axis: weights [n][2 signs][3], sign 0 = +1, 1 = -1
    const double *coord[3];  // per axis: coordinates c(0:n+1)
    const double *cellw[3];  // per axis: cell widths of nodes 1..n
};

// The conduction profile between the isothermal walls along the heated axis
// (x in 2D, y in 3D; the walls lie dt/2 outside the end nodes): linear in the
// physical coordinate, Tc = Thot at the hot wall and Tcold at the cold one.
// Reduced-precision storage keeps the thermal populations as g - wT * Tc.
// tc_setup fills the two Geo fields from the host copy of the coordinates.
inline void tc_setup(Geo &G, const double *c_heated)
{
    const int n = G.dim == 2 ? G.nx : G.ny;
    G.tc_lo = c_heated[1] - 0.5 * G.dt;
    G.tc_grad = (G.Tcold - G.Thot) / ((c_heated[n] + 0.5 * G.dt) - G.tc_lo);
}

__host__ __device__ inline double tc_gradient(const Geo &G) { return G.tc_grad; }

// Tc at node m (0-based) of the heated axis
__host__ __device__ inline double tc_value(const Geo &G, int m)
{
    return G.Thot + G.tc_grad * (G.coord[G.dim == 2 ? 0 : 1][m + 1] - G.tc_lo);
}


// Device-side state of a run to a stop criterion (lbm_run, lbm_batch_run):
// the check kernels write it after every check, and while `active` is 0 the
// step and check kernels of the cavity do nothing, so graph replays queued
// past the stop cost only their launch.  Outside runs active = 1.
struct RunCtl {
    int active;        // 1: keep stepping
    int status;        // 0 running, 1 criterion met, -1 residual stopped being finite or grew (growth),
                       // -2 non-finite residual sums (the check's own error)
    int checks;        // checks done in this run
    int pad0_;
    long long steps;   // iterations up to the last check of this run
    double errU, errT; // residuals of the last check
    double best;       // smallest max(errU, errT) of this run
    double eps;        // stop when errU <= eps and errT <= eps
    double growth;     // > 0: stop (status -1) when max(errU, errT) > growth x best after 2 checks
    int stop_bad;      // batch rule: a residual that is not finite, or grew (growth), stops the
                       // member with status -1; non-finite sums give -1 with growth > 0, else -2
    int pad1_;
};

// Device buffers of one cavity.
struct Bufs {
    void *pop[2];          // ping-pong population buffers, (Q+QT) planes each
    void *F[2];            // carried buoyancy force, one value per node
    double *rho, *u, *v, *w, *T;   // macroscopic fields, packed
    double *up, *vp, *wp, *Tp;     // fields at the previous check
    double *partials;      // reduction partials
    double *scal;          // reduction results
    int *err;              // device error flag (bounded waits that gave up)
    RunCtl *ctl;           // run state; the step kernels return at once while ctl->active is 0
};

// TMA descriptors of one population buffer (one per box class) and of the
// carried-force array that goes with it
struct alignas(64) TmapSet {
    CUtensorMap m[4];
    CUtensorMap fmap;
};

// Per-cavity tables of a batch of cavities (device memory)
struct BatchDev {
    const Geo *geo;          // [ncav]
    const TmapSet *maps;     // [ncav][2]: descriptors of pop[0], pop[1] (+ their force arrays)
    const Bufs *bufs;        // [ncav]
    const int4 *segs;        // all segments: 2D (cavity, i0, ja, jb); 3D (tile, z0, z1, cavity)
    const int *seg_off;      // [nblocks + 1]
};

// shape of the march kernels' tiles for a lattice and storage (host side)
struct MarchShape {
    int TX, TY, HX, threads, smem;
    int bx[4], by[4];
};

enum Store { kF64 = 0, kF32 = 1 };

// tile rows of the 3D batch kernel (its tiles are 32 x kBatchTileY)
constexpr int kBatchTileY = 4;

// kernel launchers; one set per arithmetic mode
#define LBM_DECLARE_LAUNCHERS(NS)                                                             \
    namespace NS {                                                                            \
    /* init: equilibrium populations from the macroscopic fields into pop; neq != 0 adds  */ \
    /* the first-order non-equilibrium part, cf = 3 tau_f dt, ct = dt / sig_k              */ \
    cudaError_t equilibrium(const Geo &g, int store, void *pop, const Bufs &b, int neq, double cf, double ct, \
                            cudaStream_t s);                                                   \
    /* nsteps 2D fused steps in one cooperative launch (domains of one wave); bar: two    */ \
    /* zeroed unsigned of device memory, err: device flag set on a barrier timeout        */ \
    cudaError_t steps_resident(const Geo &g, int store, void *const pop[2], void *const F[2], \
                               const Bufs &b, int cur, int nsteps, unsigned *bar, int *err,    \
                               int nblocks, cudaStream_t s);                                   \
    /* resident grid of steps_resident for this domain (0: not available) */                  \
    int resident_blocks(const Geo &g, int store, int device);                                  \
    /* first collision of a run: pre-collision pop_in -> post-collision pop_out, F_out */     \
    cudaError_t collide(const Geo &g, int store, const void *pop_in, void *pop_out,           \
                        void *F_out, const Bufs &b, cudaStream_t s);                          \
    /* fused step: stream + walls + macro + collide.  write_macro != 0 also stores rho,u,T */ \
    cudaError_t step(const Geo &g, int store, const void *pop_in, const void *F_in,           \
                     void *pop_out, void *F_out, const Bufs &b, int write_macro,              \
                     cudaStream_t s);                                                         \
    /* stream + walls + macro only: pre-collision populations into pop_out, macro fields */  \
    cudaError_t stream_only(const Geo &g, int store, const void *pop_in, const void *F_in,    \
                            void *pop_out, const Bufs &b, cudaStream_t s);                    \
    /* fused step through the TMA-fed persistent march kernel; 3D: tile rows ty (4 or 8)  */ \
    /* and the blocks' segment lists segs[segoff[b] .. segoff[b+1]) (device memory);       */ \
    /* pdl: programmatic dependent launch (overlaps the previous kernel's tail)            */ \
    cudaError_t march(const Geo &g, int store, const TmapSet &src, const void *F_in,          \
                      void *pop_out, void *F_out, const Bufs &b, int write_macro, int nblocks,\
                      int ty, const int4 *segs, const int *segoff, bool pdl, cudaStream_t s); \
    /* resident blocks per SM of the march kernel (0 if it cannot launch) */                  \
    int march_blocks_per_sm(const Geo &g, int store, int ty);                                 \
    /* one step of every cavity of a 2D batch (tile width TX = 32, 64 or 128) */              \
    cudaError_t march_batch(int store, int TX, const BatchDev &D, int nblocks, int cur,       \
                            int write_macro, int *err, bool pdl, cudaStream_t s);             \
    int march_batch_blocks_per_sm(int store, int TX);                                         \
    /* one step of every cavity of a 3D batch (segments: tile, z0, z1, cavity; 32 x 4 tiles) */\
    cudaError_t march_batch3d(int store, const BatchDev &D, int nblocks, int cur,             \
                              int write_macro, int *err, bool pdl, cudaStream_t s);           \
    int march_batch3d_blocks_per_sm(int store);                                               \
    /* limit of the march kernels' per-step waits on this device, in clock cycles */          \
    cudaError_t set_wait_limit(long long cycles);                                             \
    }

LBM_DECLARE_LAUNCHERS(fast)
LBM_DECLARE_LAUNCHERS(exact)

// mode-independent kernels (lbm_reduce.cu)
cudaError_t reduce_check(const Geo &g, const Bufs &b, cudaStream_t s);      // scal[0..3]
cudaError_t reduce_nusselt(const Geo &g, const Bufs &b, cudaStream_t s);    // scal[4..6]
cudaError_t reduce_sums(const Geo &g, const Bufs &b, cudaStream_t s);       // scal[7..8]
// check() of a run: the same sums as reduce_check, then the stop test on the
// device (b.ctl); does nothing while b.ctl->active is 0.  period: iterations
// since the previous check
cudaError_t run_check(const Geo &g, const Bufs &b, int period, cudaStream_t s);
// the same for the batch members idx[0..n-1] (tables of D), in one pair of launches
cudaError_t run_check_batch(const BatchDev &D, const int *idx, int n, int period, cudaStream_t s);
// AoS (Fortran f(0:Q-1,nodes)) <-> SoA planes, for FP64/FP32 storage
cudaError_t aos_to_planes(const Geo &g, int store, int q0, int nq, const double *aos,
                          void *pop, cudaStream_t s);
cudaError_t planes_to_aos(const Geo &g, int store, int q0, int nq, const void *pop,
                          double *aos, cudaStream_t s);
// a state's populations (nq planes) and carried force in another storage
cudaError_t convert_state(const Geo &g, int src_store, int dst_store, int nq, const void *pop_src, void *pop_dst,
                          const void *F_src, void *F_dst, cudaStream_t s);
// macro fields from populations (used by set_populations)
cudaError_t macro_from_pops(const Geo &g, int store, const void *pop, const Bufs &b,
                            cudaStream_t s);

extern int64_t g_launches;  // kernels launched by this library

// record a message for lbm_last_error() and return code
int set_error(int code, const char *fmt, ...);

// tile shape of the march kernels (identical in both arithmetic modes); tx
// selects the tile width of the 2D kernels (0: the single-cavity default),
// ty the tile rows of the 3D kernel (4 or 8; 0: 8)
MarchShape march_shape(int dim, int store, int tx = 0, int ty = 0);

// Work plan of the 3D march kernel: for `nblocks` persistent blocks over
// `ntiles` tile columns of nz slices, the segments (tile, z0, z1, 0) of each
// block, block b owning segs[off[b] .. off[b+1]).  kind 0: balanced z-lockstep
// (every tile column in equal chunks run side by side, the blocks left over
// take the chunks' last slices in lockstep rounds); 1: contiguous equal
// shares of the (tile-major, slice-minor) items.  Returns the blocks used.
int plan_march3d(int ntiles, int nz, int nblocks, int kind, std::vector<int4> &segs, std::vector<int> &off);

}  // namespace lbm
