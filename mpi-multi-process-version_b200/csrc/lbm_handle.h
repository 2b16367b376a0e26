// Internal: the cavity handle behind the C ABI, shared by lbm_capi.cu and
// lbm_batch.cu.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "../../include/lbm_b200.h"
#include "lbm_internal.h"

struct Derived {
    double viscosity_LB, kappa, gbeta, tauf, Snu, Sq, sig_k;
};


// ---------------------------------------------------------------------------
// handle
// ---------------------------------------------------------------------------
struct lbm_handle {
    using Geo = lbm::Geo;
    using Bufs = lbm::Bufs;
    using TmapSet = lbm::TmapSet;
    lbm_params p;
    Derived d;
    int Q, QT;
    int device;
    size_t esize, csize;      // storage / compute element size
    Geo geo;
    Bufs bufs;
    std::vector<double> coord[3];
    double *d_wgt[3] = {nullptr, nullptr, nullptr};
    double *d_coord[3] = {nullptr, nullptr, nullptr};
    double *d_cellw[3] = {nullptr, nullptr, nullptr};
    void *staging = nullptr;     // population planes for stream-only output
    double *aos = nullptr;       // Fortran-layout staging
    cudaStream_t stream = nullptr;
    bool owns_stream = true;     // false for members of a batch (the batch's stream)
    bool owns_ctl = true;        // false for members of a batch (bufs.ctl points into the batch's array)
    TmapSet tmaps[2];            // TMA descriptors of pop[0] and pop[1]
    bool march_ok = false;       // tile shape and descriptors usable
    int kernel_opt = 0;          // LBM_OPT_KERNEL as set
    int use_march = 0;           // resolved choice
    int nblocks_opt = 0;         // LBM_OPT_NBLOCKS as set
    int nblocks = 0;             // resolved persistent grid
    int tiley_opt = 0;           // LBM_OPT_TILEY as set (0: automatic)
    int tiley = 4;               // resolved tile rows of the 3D march kernel (4 or 8)
    int plan_opt = 0;            // LBM_OPT_PLAN: 0 balanced z-lockstep, 1 contiguous shares
    int64_t wait_limit = 0;      // LBM_OPT_WAIT_LIMIT as last set through this handle
    int pdl = 1;                 // LBM_OPT_PDL: programmatic dependent launch of march steps
    int4 *d_msegs = nullptr;     // 3D march work plan: segments (tile, z0, z1, -)
    int *d_msegoff = nullptr;    // and each block's first segment
    size_t msegs_cap = 0, msegoff_cap = 0;
    int l2promo = 0;             // LBM_OPT_L2PROMO
    int use_graphs = 1;          // LBM_OPT_GRAPHS
    int resident_opt = 0;        // LBM_OPT_RESIDENT as set (opt-in)
    int resident = 0;            // resolved: blocks of the resident multi-step launch (0: off)
    unsigned *d_bar = nullptr;   // grid barrier of the resident launch (two counters)
    cudaGraphExec_t graph[2] = {nullptr, nullptr};  // 8-step graphs (kGraphSteps) from cur = 0 / 1
    cudaGraphExec_t run_graph[2] = {nullptr, nullptr};  // check periods of lbm_run from cur = 0 / 1
    int run_graph_period = 0;    // their length
    int cur = 0;                 // buffer holding the newest populations
    int phase = 0;               // 0: not initialised, 1: pre-collision, 2: post-collision
    int64_t itc = 0;
    int64_t bytes = 0;
};


// helpers of lbm_capi.cu used by the batch
namespace lbm {
// encode the TMA descriptors of h's two population buffers for the march
// kernel with tile width tx (0: the single-cavity default); false if TMA
// cannot be used
bool encode_maps_tx(const lbm_handle *h, int tx, lbm::TmapSet out[2]);
// the first collision of a run if h is still in its pre-collision state
int first_collision(lbm_handle *h);
// synchronise h's stream and report a kernel's bounded wait that gave up
int sync_handle(lbm_handle *h);
// release the captured step graphs (kernel choice or buffers changed)
void drop_graphs(lbm_handle *h);
// device-side runs (lbm_run, lbm_batch_run): initialise h's RunCtl, read it
// back after a synchronisation (with the bounded-wait check), and set it
// active again when the run is over
int run_begin(lbm_handle *h, double eps, double growth, int stop_bad);
int run_read(lbm_handle *h, RunCtl *out);
int run_end(lbm_handle *h);
// population storage of h converted in place (buffers, descriptors, kernel);
// target >= 0: the state lands in ping-pong buffer `target` (h->cur becomes it)
int change_storage(lbm_handle *h, int storage, int target = -1);
}  // namespace lbm
