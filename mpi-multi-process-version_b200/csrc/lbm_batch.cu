// Batches of independent cavities (the parameter-sweep use of the time step).
//
// The reference runs one cavity per program (natural-convection_2dim_mono.f90
// `program main`, 283-380).  A batch holds many cavities of different size and
// parameters and advances all of them at once:
//   * 2D batches: one persistent TMA march kernel per step (k_march2d_batch)
//     walks a work list of segments -- (cavity, column strip, row range) --
//     that splits the total work into equal contiguous shares, one per block;
//     the per-cavity geometry, TMA descriptors and buffers come from tables
//     in device memory;
//   * steps between checks are replayed from 2-step CUDA graphs;
//   * lbm_batch_run applies the reference's stop test per cavity (errorU and
//     errorT at most eps at a check, 2M:307) and drops stopped cavities
//     from the work list;
//   * lbm_batch_tune times the tile widths and grid sizes on the batch itself
//     and keeps the fastest;
//   * 3D batches: one persistent TMA march kernel per step too
//     (k_march3d_batch), over segments (tile, first slice, end slice,
//     cavity) that split the (tile column, slice) items into equal shares;
//   * with the persistent kernel switched off (or a 3D member the march
//     kernel does not cover), every cavity steps with its own launch;
//   * lbm_batch_run and lbm_batch_run_masked test the stop criterion on the
//     device and read the members' run state once every few checks.
// Every member is an ordinary lbm_handle (lbm_batch_cavity) sharing the
// batch's stream, so initialisation, checks and getters are the single-
// cavity entry points.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "lbm_handle.h"

using namespace lbm;

#define BCU(call)                                                                                        \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess)                                                                           \
            return set_error(e_ == cudaErrorMemoryAllocation ? LBM_ERR_NOMEM : LBM_ERR_CUDA, "%s: %s (%s:%d)", \
                             #call, cudaGetErrorString(e_), __FILE__, __LINE__);                         \
    } while (0)

struct lbm_batch {
    int n = 0;
    int dim = 2, storage = 0, mode = 0, device = 0;
    std::vector<lbm_handle *> cav;
    std::vector<char> active;
    cudaStream_t stream = nullptr;
    int tile_opt = 0, tile = 64;   // tile width of the 2D batch kernel (32, 64, 128)
    int nblocks_opt = 0, nblocks = 0;
    int persistent = 1;            // 0: one launch per cavity
    bool march_ok = true;          // every member can run in the persistent kernel (3D: tile rows fit)
    int use_graphs = 1;
    double growth = 0.0;           // residual growth factor that stops a member in lbm_batch_run (0: off)
    int storages = 0;              // LBM_BATCH_OPT_STORAGES: storages lbm_batch_tune may pick (0: the current)
    int pdl = 1;                   // LBM_BATCH_OPT_PDL: programmatic dependent launch of the step kernels
    Geo *d_geo = nullptr;
    TmapSet *d_maps = nullptr;
    Bufs *d_bufs = nullptr;
    // one work list per population storage (members may differ while a
    // mixed-precision run hands them from FP32 to FP64 one by one)
    struct WorkList {
        int4 *d_segs = nullptr;
        int *d_segoff = nullptr;
        size_t segs_cap = 0, segoff_cap = 0;
        int nblocks = 0;   // the list's grid (fixed while graphs replay it)
        int tx = 0;        // the tile width its kernel was captured with
        BatchDev dev{};
    } wl[2];
    bool run_both = false;         // a mixed run: both storages' kernels launch every step
    cudaStream_t stream2 = nullptr;  // the second branch when both storages' kernels run
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    int *d_err = nullptr;
    BatchDev dev{};                // the tables (segment fields unused) for the batched check
    bool dirty = true;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    cudaGraphExec_t run_graph[2] = {nullptr, nullptr};  // check periods of lbm_batch_run from cur = 0 / 1
    int run_graph_period = 0;
    int64_t run_graph_launches = 0;  // kernels one replay of a check-period graph launches
    int64_t graph_launches = 0;      // kernels one replay of a 2-step graph launches
    int64_t active_nodes = 0;
    RunCtl *d_ctl = nullptr;       // run state of every member (member i's bufs.ctl = d_ctl + i)
    int *d_idx = nullptr;          // the members of a run (its mask), for the batched check
    int nidx = 0;
};

static void drop_graphs(lbm_batch *b)
{
    for (auto &g : b->graph)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
    for (auto &g : b->run_graph)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
}

extern "C" int lbm_batch_destroy(lbm_batch *b)
{
    if (!b) return LBM_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_graphs(b);
    for (lbm_handle *h : b->cav) lbm_destroy(h);
    void *ptrs[] = {b->d_geo, b->d_maps,        b->d_bufs,         b->d_err,        b->d_ctl,
                    b->d_idx, b->wl[0].d_segs,  b->wl[0].d_segoff, b->wl[1].d_segs, b->wl[1].d_segoff};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    if (b->ev_join) cudaEventDestroy(b->ev_join);
    if (b->stream2) cudaStreamDestroy(b->stream2);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return LBM_OK;
}

extern "C" int lbm_batch_create(int32_t n, const lbm_params *params, const double *const *x, const double *const *y,
                                const double *const *z, lbm_batch **out)
{
    if (!out) return set_error(LBM_ERR_PARAM, "out is NULL");
    *out = nullptr;
    if (n < 1 || !params || !x || !y) return set_error(LBM_ERR_PARAM, "lbm_batch_create: need n >= 1, params, x, y");
    for (int i = 1; i < n; ++i)
        if (params[i].dim != params[0].dim || params[i].storage != params[0].storage ||
            params[i].mode != params[0].mode || params[i].device != params[0].device)
            return set_error(LBM_ERR_PARAM, "lbm_batch_create: cavity %d differs in dim/storage/mode/device", i);
    if (params[0].dim == 3 && !z) return set_error(LBM_ERR_PARAM, "lbm_batch_create: z is required in 3D");
    lbm_batch *b = new lbm_batch();
    b->n = n;
    b->dim = params[0].dim;
    b->storage = params[0].storage;
    b->mode = params[0].mode;
    b->device = params[0].device;
    auto bail = [&](int code) {
        lbm_batch_destroy(b);
        return code;
    };
    {
        cudaError_t e = cudaSetDevice(b->device);
        if (e != cudaSuccess) return bail(set_error(LBM_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e)));
        e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream2, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming);
        if (e != cudaSuccess) return bail(set_error(LBM_ERR_CUDA, "stream: %s", cudaGetErrorString(e)));
    }
    for (int i = 0; i < n; ++i) {
        lbm_handle *h = nullptr;
        int st = lbm_create(&params[i], x[i], y[i], z ? z[i] : nullptr, &h);
        if (st) return bail(st);
        cudaStreamDestroy(h->stream);
        h->stream = b->stream;
        h->owns_stream = false;
        h->resident_opt = 0;  // members step one iteration per launch (or in the batch kernel)
        h->resident = 0;
        b->cav.push_back(h);
    }
    b->active.assign(n, 1);
    {
        // one run-state array for all members, so a run reads every member's state in one copy
        cudaError_t e = cudaMalloc(&b->d_ctl, sizeof(RunCtl) * n);
        if (e == cudaSuccess) e = cudaMalloc(&b->d_idx, sizeof(int) * n);
        std::vector<RunCtl> c(n);
        for (auto &x : c) x.active = 1;
        if (e == cudaSuccess) e = cudaMemcpy(b->d_ctl, c.data(), sizeof(RunCtl) * n, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return bail(set_error(LBM_ERR_NOMEM, "batch run state: %s", cudaGetErrorString(e)));
        for (int i = 0; i < n; ++i) {
            lbm_handle *h = b->cav[i];
            cudaFree(h->bufs.ctl);
            h->bytes -= (int64_t)sizeof(RunCtl);
            h->bufs.ctl = b->d_ctl + i;
            h->owns_ctl = false;
        }
    }
    {
        cudaError_t e = cudaMalloc(&b->d_geo, sizeof(Geo) * n);
        if (e == cudaSuccess) e = cudaMalloc(&b->d_bufs, sizeof(Bufs) * n);
        if (e == cudaSuccess) e = cudaMalloc(&b->d_maps, sizeof(TmapSet) * 2 * n);
        if (e == cudaSuccess) e = cudaMalloc(&b->d_err, 16);
        if (e == cudaSuccess) e = cudaMemset(b->d_err, 0, 16);
        if (e != cudaSuccess) return bail(set_error(LBM_ERR_NOMEM, "batch tables: %s", cudaGetErrorString(e)));
        std::vector<Geo> geo(n);
        std::vector<Bufs> bufs(n);
        for (int i = 0; i < n; ++i) {
            geo[i] = b->cav[i]->geo;
            bufs[i] = b->cav[i]->bufs;
        }
        e = cudaMemcpy(b->d_geo, geo.data(), sizeof(Geo) * n, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(b->d_bufs, bufs.data(), sizeof(Bufs) * n, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return bail(set_error(LBM_ERR_CUDA, "batch tables: %s", cudaGetErrorString(e)));
    }
    // the 3D batch kernel has 32 x kBatchTileY tiles: a last tile row of a
    // single y-row (its one-sided stencil would reach two rows below the box)
    // is not covered
    if (b->dim == 3)
        for (int i = 0; i < n; ++i)
            if (b->cav[i]->geo.ny % kBatchTileY == 1 || b->cav[i]->tiley != kBatchTileY) b->march_ok = false;
    *out = b;
    return LBM_OK;
}

// descriptors for the tile width, and the work lists of the active cavities.
// A column is one march: 2D a TX-wide strip of rows, 3D a 32 x kBatchTileY tile
// of slices.  Each storage's list keeps a fixed grid (a full wave, or the
// caller's nblocks) and fixed device arrays sized for every member's columns,
// so a change of the active members or of a member's storage only rewrites
// the arrays' contents and captured graphs stay valid; blocks without work
// return at once.
static int build_tables(lbm_batch *b)
{
    const bool d3 = b->dim == 3;
    const int TX = d3 ? 32 : b->tile;
    std::vector<TmapSet> maps(2 * (size_t)b->n);
    for (int i = 0; i < b->n; ++i)
        if (!encode_maps_tx(b->cav[i], d3 ? 0 : TX, &maps[2 * (size_t)i]))
            return set_error(LBM_ERR_UNSUPPORTED, "batch: TMA descriptors for cavity %d could not be encoded", i);
    BCU(cudaMemcpyAsync(b->d_maps, maps.data(), sizeof(TmapSet) * maps.size(), cudaMemcpyHostToDevice, b->stream));
    {
        // the members' buffers (a storage change gives a member new ones)
        std::vector<Bufs> bufs(b->n);
        for (int i = 0; i < b->n; ++i) bufs[i] = b->cav[i]->bufs;
        BCU(cudaMemcpyAsync(b->d_bufs, bufs.data(), sizeof(Bufs) * b->n, cudaMemcpyHostToDevice, b->stream));
    }

    struct Col {
        int cav, pos, ny;  // pos: 2D the strip's x-offset, 3D the tile index; ny: items (rows or slices)
    };
    std::vector<Col> cols;
    size_t ncols_all = 0;  // the columns of every member, active or not: the lists' capacity
    b->active_nodes = 0;
    for (int i = 0; i < b->n; ++i) {
        const Geo &g = b->cav[i]->geo;
        const int nc = d3 ? ((g.nx + 31) / 32) * ((g.ny + kBatchTileY - 1) / kBatchTileY) : (g.nx + TX - 1) / TX;
        ncols_all += nc;
        if (!b->active[i]) continue;
        for (int c = 0; c < nc; ++c) cols.push_back({i, d3 ? c : c * TX, d3 ? g.nz : g.ny});
        b->active_nodes += g.nnode;
    }
    int sms = 0;
    BCU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
    bool regraph = false;
    b->nblocks = 0;
    for (int sto = 0; sto < 2; ++sto) {
        lbm_batch::WorkList &W = b->wl[sto];
        // this storage's columns
        std::vector<Col> sc;
        int64_t stotal = 0;
        for (const Col &c : cols)
            if (b->cav[c.cav]->p.storage == sto) {
                sc.push_back(c);
                stotal += c.ny;
            }
        const bool present = !sc.empty() || (b->run_both && b->mode != LBM_MODE_EXACT);
        if (!present) {
            if (W.nblocks) regraph = true;
            W.nblocks = 0;
            continue;
        }
        const int bps = d3 ? (b->mode == LBM_MODE_EXACT ? exact::march_batch3d_blocks_per_sm(sto)
                                                         : fast::march_batch3d_blocks_per_sm(sto))
                           : (b->mode == LBM_MODE_EXACT ? exact::march_batch_blocks_per_sm(sto, TX)
                                                        : fast::march_batch_blocks_per_sm(sto, TX));
        if (bps <= 0) return set_error(LBM_ERR_UNSUPPORTED, "batch kernel with tile %d cannot be resident", TX);
        const int64_t G = b->nblocks_opt > 0 ? b->nblocks_opt : (int64_t)bps * sms;
        // equal contiguous shares of the (column, item) items; blocks past the work get none
        std::vector<int4> segs;
        std::vector<int> off(G + 1, 0);
        size_t c = 0;
        int64_t colbase = 0;  // first item of column c
        for (int64_t blk = 0; blk < G; ++blk) {
            off[blk] = (int)segs.size();
            const int64_t lo = stotal * blk / G, hi = stotal * (blk + 1) / G;
            int64_t u = lo;
            while (u < hi) {
                while (c < sc.size() && colbase + sc[c].ny <= u) colbase += sc[c++].ny;
                const int64_t end = std::min<int64_t>(hi, colbase + sc[c].ny);
                if (d3)
                    segs.push_back(make_int4(sc[c].pos, (int)(u - colbase), (int)(end - colbase), sc[c].cav));
                else
                    segs.push_back(make_int4(sc[c].cav, sc[c].pos, (int)(u - colbase), (int)(end - colbase)));
                u = end;
            }
        }
        off[G] = (int)segs.size();
        const size_t seg_need = (size_t)G + ncols_all + 16;
        if (W.segs_cap < seg_need) {
            if (W.d_segs) cudaFree(W.d_segs);
            W.d_segs = nullptr;
            W.segs_cap = seg_need;
            BCU(cudaMalloc(&W.d_segs, sizeof(int4) * W.segs_cap));
            regraph = true;
        }
        if (W.segoff_cap < off.size()) {
            if (W.d_segoff) cudaFree(W.d_segoff);
            W.d_segoff = nullptr;
            W.segoff_cap = off.size();
            BCU(cudaMalloc(&W.d_segoff, sizeof(int) * W.segoff_cap));
            regraph = true;
        }
        if (!segs.empty())
            BCU(cudaMemcpyAsync(W.d_segs, segs.data(), sizeof(int4) * segs.size(), cudaMemcpyHostToDevice,
                                b->stream));
        BCU(cudaMemcpyAsync(W.d_segoff, off.data(), sizeof(int) * off.size(), cudaMemcpyHostToDevice, b->stream));
        if (W.nblocks != (int)G || W.tx != TX) regraph = true;
        W.nblocks = (int)G;
        W.tx = TX;
        W.dev = BatchDev{b->d_geo, b->d_maps, b->d_bufs, W.d_segs, W.d_segoff};
        b->nblocks += (int)G;
    }
    BCU(cudaStreamSynchronize(b->stream));
    b->dev = BatchDev{b->d_geo, b->d_maps, b->d_bufs, nullptr, nullptr};
    if (regraph) drop_graphs(b);
    b->dirty = false;
    return LBM_OK;
}

// one step of every member on the work lists: one persistent kernel per
// population storage present; pdl: launched as a programmatic dependent of the
// stream's previous kernel
static cudaError_t launch_list(lbm_batch *b, int sto, int cur, int wm, bool pdl, cudaStream_t s)
{
    const lbm_batch::WorkList &W = b->wl[sto];
    if (b->dim == 3)
        return b->mode == LBM_MODE_EXACT ? exact::march_batch3d(sto, W.dev, W.nblocks, cur, wm, b->d_err, pdl, s)
                                         : fast::march_batch3d(sto, W.dev, W.nblocks, cur, wm, b->d_err, pdl, s);
    return b->mode == LBM_MODE_EXACT ? exact::march_batch(sto, W.tx, W.dev, W.nblocks, cur, wm, b->d_err, pdl, s)
                                     : fast::march_batch(sto, W.tx, W.dev, W.nblocks, cur, wm, b->d_err, pdl, s);
}

// with both storages present the two kernels run side by side (a fork onto
// the second stream and a join), so a step costs one kernel's latency; a
// single list's kernels follow one another as programmatic dependents
static cudaError_t launch_step(lbm_batch *b, int cur, int wm)
{
    const bool a = b->wl[0].nblocks > 0, c = b->wl[1].nblocks > 0;
    if (a && c) {
        cudaError_t e = cudaEventRecord(b->ev_fork, b->stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream2, b->ev_fork, 0);
        if (e == cudaSuccess) e = launch_list(b, 1, cur, wm, false, b->stream2);
        if (e == cudaSuccess) e = launch_list(b, 0, cur, wm, false, b->stream);
        if (e == cudaSuccess) e = cudaEventRecord(b->ev_join, b->stream2);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, b->ev_join, 0);
        return e;
    }
    if (a) return launch_list(b, 0, cur, wm, b->pdl != 0, b->stream);
    if (c) return launch_list(b, 1, cur, wm, b->pdl != 0, b->stream);
    return cudaSuccess;
}

// a 2-step graph starting from buffer `cur`
static int get_graph(lbm_batch *b, int cur, cudaGraphExec_t *out)
{
    if (!b->graph[cur]) {
        cudaGraph_t g = nullptr;
        const int64_t launches0 = g_launches;
        BCU(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t e1 = launch_step(b, cur, 0);
        cudaError_t e2 = launch_step(b, 1 - cur, 0);
        cudaError_t e3 = cudaStreamEndCapture(b->stream, &g);
        b->graph_launches = g_launches - launches0;
        g_launches = launches0;  // counted when replayed
        if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return set_error(LBM_ERR_CUDA, "batch graph capture failed: %s",
                             cudaGetErrorString(e1 != cudaSuccess ? e1 : (e2 != cudaSuccess ? e2 : e3)));
        }
        cudaError_t e = cudaGraphInstantiate(&b->graph[cur], g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return set_error(LBM_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    }
    *out = b->graph[cur];
    return LBM_OK;
}

extern "C" int lbm_batch_step(lbm_batch *b, int32_t nsteps)
{
    if (!b) return set_error(LBM_ERR_PARAM, "batch is NULL");
    if (nsteps < 0) return set_error(LBM_ERR_PARAM, "nsteps < 0");
    BCU(cudaSetDevice(b->device));
    if (nsteps == 0) return LBM_OK;
    for (int i = 0; i < b->n; ++i)
        if (b->active[i] && b->cav[i]->phase == 0)
            return set_error(LBM_ERR_STATE, "batch: cavity %d stepped before an init call", i);
    if (!b->persistent || !b->march_ok) {
        for (int i = 0; i < b->n; ++i)
            if (b->active[i]) {
                int st = lbm_step(b->cav[i], nsteps);
                if (st) return st;
            }
        return LBM_OK;
    }
    int cur = -1;
    for (int i = 0; i < b->n; ++i) {
        if (!b->active[i]) continue;
        int st = first_collision(b->cav[i]);
        if (st) return st;
        if (cur < 0) cur = b->cav[i]->cur;
        if (b->cav[i]->cur != cur)
            return set_error(LBM_ERR_STATE, "batch: cavity %d is out of step with the others", i);
    }
    if (cur < 0) return LBM_OK;  // nothing active
    if (b->dirty) {
        int st = build_tables(b);
        if (st) return st;
    }
    int done = 0;
    // whole 2-step graphs for all but the last step, then the last step with the macroscopic output
    if (b->use_graphs) {
        while (nsteps - done > 2) {
            cudaGraphExec_t g;
            int st = get_graph(b, cur, &g);
            if (st) return st;
            BCU(cudaGraphLaunch(g, b->stream));
            g_launches += b->graph_launches;
            done += 2;
        }
    }
    while (done < nsteps) {
        BCU(launch_step(b, cur, done == nsteps - 1));
        cur = 1 - cur;
        ++done;
    }
    // each graph replay flips the buffers twice, each single launch once
    const int final_cur = cur;
    for (int i = 0; i < b->n; ++i)
        if (b->active[i]) {
            b->cav[i]->cur = final_cur;
            b->cav[i]->itc += nsteps;
        }
    return LBM_OK;
}

extern "C" int lbm_batch_synchronize(lbm_batch *b)
{
    if (!b) return set_error(LBM_ERR_PARAM, "batch is NULL");
    BCU(cudaSetDevice(b->device));
    BCU(cudaStreamSynchronize(b->stream));
    if (b->d_err) {
        int flag = 0;
        BCU(cudaMemcpy(&flag, b->d_err, sizeof(int), cudaMemcpyDeviceToHost));
        if (flag) {
            BCU(cudaMemset(b->d_err, 0, sizeof(int)));
            return set_error(LBM_ERR_TIMEOUT, "batch kernel: a bounded wait for TMA copies gave up");
        }
    }
    return LBM_OK;
}

extern "C" int lbm_batch_size(const lbm_batch *b, int32_t *n)
{
    if (!b || !n) return set_error(LBM_ERR_PARAM, "NULL argument");
    *n = b->n;
    return LBM_OK;
}

extern "C" int lbm_batch_cavity(lbm_batch *b, int32_t i, lbm_handle **h)
{
    if (!b || !h || i < 0 || i >= b->n) return set_error(LBM_ERR_PARAM, "lbm_batch_cavity: bad index");
    *h = b->cav[i];
    return LBM_OK;
}

extern "C" int lbm_batch_init_reference(lbm_batch *b)
{
    if (!b) return set_error(LBM_ERR_PARAM, "batch is NULL");
    for (lbm_handle *h : b->cav) {
        int st = lbm_init_reference(h);
        if (st) return st;
    }
    b->active.assign(b->n, 1);
    b->dirty = true;
    return LBM_OK;
}

extern "C" int lbm_batch_check(lbm_batch *b, double *errU, double *errT)
{
    if (!b || !errU || !errT) return set_error(LBM_ERR_PARAM, "NULL argument");
    int st = lbm_batch_synchronize(b);
    if (st) return st;
    for (int i = 0; i < b->n; ++i) {
        st = lbm_check(b->cav[i], &errU[i], &errT[i]);
        if (st) return st;
    }
    return LBM_OK;
}

extern "C" int lbm_batch_nusselt(lbm_batch *b, double *nu_hot, double *nu_cold)
{
    if (!b || !nu_hot || !nu_cold) return set_error(LBM_ERR_PARAM, "NULL argument");
    int st = lbm_batch_synchronize(b);
    if (st) return st;
    for (int i = 0; i < b->n; ++i) {
        st = lbm_nusselt(b->cav[i], &nu_hot[i], &nu_cold[i]);
        if (st) return st;
    }
    return LBM_OK;
}

// One check period of a persistent batch as a graph: `period` steps of every
// member on the work list, the last writing the macroscopic fields, then the
// batched check with the stop test on the device.
static int batch_period_graph(lbm_batch *b, int cur, int period, cudaGraphExec_t *out)
{
    if (b->run_graph_period != period) {
        for (auto &g : b->run_graph)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
        b->run_graph_period = period;
    }
    if (!b->run_graph[cur]) {
        cudaGraph_t g = nullptr;
        const int64_t launches0 = g_launches;
        BCU(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = cudaSuccess;
        for (int i = 0; i < period && e == cudaSuccess; ++i) e = launch_step(b, (cur + i) & 1, i == period - 1);
        if (e == cudaSuccess) e = run_check_batch(b->dev, b->d_idx, b->nidx, period, b->stream);
        const cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
        b->run_graph_launches = g_launches - launches0;
        g_launches = launches0;  // counted when replayed
        if (e != cudaSuccess || e2 != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return set_error(LBM_ERR_CUDA, "batch check-period graph capture: %s",
                             cudaGetErrorString(e != cudaSuccess ? e : e2));
        }
        e = cudaGraphInstantiate(&b->run_graph[cur], g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return set_error(LBM_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    }
    *out = b->run_graph[cur];
    return LBM_OK;
}

// check periods a batch run queues between two reads of the members' run state
static constexpr int kBatchPeriodsPerRead = 4;

// The batch's run loop.  Every member on the mask runs the reference's stop
// test on the device after each check (run_decide).  Single phase
// (two_phase false): criterion eps1.  Two phases (mixed precision): every
// member starts in FP32 storage with criterion eps1; when it meets it, the host
// (at its next read) converts that member alone to FP64 in place, into the
// batch's current ping-pong buffer, and it goes on with criterion eps2 while
// the others continue in FP32: each member's FP64 finish overlaps the other
// members' FP32 transients.  max_steps bounds each member's iterations.
static int batch_run(lbm_batch *b, const int32_t *mask, int32_t max_steps, int32_t check_every, double eps1,
                     double eps2, bool two_phase, int32_t *converged, int64_t *steps_done, int64_t *steps_low)
{
    if (!b) return set_error(LBM_ERR_PARAM, "batch is NULL");
    if (max_steps < 0 || check_every < 1) return set_error(LBM_ERR_PARAM, "need max_steps >= 0, check_every >= 1");
    if (two_phase && b->mode == LBM_MODE_EXACT)
        return set_error(LBM_ERR_UNSUPPORTED, "mixed precision: exact mode computes in FP64 storage only");
    BCU(cudaSetDevice(b->device));
    const int n = b->n;
    int remaining = 0;
    for (int i = 0; i < n; ++i) {
        const bool on = !mask || mask[i] != 0;
        if (converged) converged[i] = 0;
        if (steps_done) steps_done[i] = 0;
        if (steps_low) steps_low[i] = 0;
        b->active[i] = on ? 1 : 0;
        remaining += on ? 1 : 0;
    }
    for (int i = 0; i < n; ++i)
        if (b->active[i] && b->cav[i]->phase == 0)
            return set_error(LBM_ERR_STATE, "batch: cavity %d run before an init call", i);
    for (int i = 0; i < n; ++i)
        if (b->active[i]) {
            int st = first_collision(b->cav[i]);
            if (st) return st;
            if (two_phase && (st = change_storage(b->cav[i], LBM_STORE_F32))) return st;
        }
    if (two_phase) {
        std::vector<Bufs> bufs(n);
        for (int i = 0; i < n; ++i) bufs[i] = b->cav[i]->bufs;
        BCU(cudaMemcpy(b->d_bufs, bufs.data(), sizeof(Bufs) * n, cudaMemcpyHostToDevice));
    }
    // the common parity of the members on the mask
    int cur = -1;
    for (int i = 0; i < n; ++i)
        if (b->active[i]) {
            if (cur < 0) cur = b->cav[i]->cur;
            if (b->cav[i]->cur != cur)
                return set_error(LBM_ERR_STATE, "batch: cavity %d is out of step with the others", i);
        }
    auto fresh = [&](double eps) {
        RunCtl c{};
        c.active = 1;
        c.errU = c.errT = 100.0;
        c.best = INFINITY;
        c.eps = eps;
        c.growth = b->growth;
        c.stop_bad = 1;
        return c;
    };
    std::vector<RunCtl> ctl(n);
    for (int i = 0; i < n; ++i) {
        ctl[i] = fresh(eps1);
        ctl[i].active = b->active[i];  // members off the mask stay out of the batched check
    }
    BCU(cudaMemcpyAsync(b->d_ctl, ctl.data(), sizeof(RunCtl) * n, cudaMemcpyHostToDevice, b->stream));
    {
        // the batched check covers the run's members; stopped ones return at once
        std::vector<int> idx;
        for (int i = 0; i < n; ++i)
            if (b->active[i]) idx.push_back(i);
        b->nidx = (int)idx.size();
        if (!idx.empty())
            BCU(cudaMemcpyAsync(b->d_idx, idx.data(), sizeof(int) * idx.size(), cudaMemcpyHostToDevice, b->stream));
    }
    BCU(cudaStreamSynchronize(b->stream));
    drop_graphs(b);  // the check covers this run's members
    b->run_both = two_phase;
    std::vector<int64_t> itc0(n), base_steps(n, 0);
    std::vector<int> base_cur(n), phase(n, 1);
    for (int i = 0; i < n; ++i) {
        itc0[i] = b->cav[i]->itc;
        base_cur[i] = b->cav[i]->cur;
    }
    b->dirty = true;
    const bool persistent = b->persistent && b->march_ok;
    int64_t steps = 0;
    int periods = 0;
    int st = LBM_OK;
    while (steps < max_steps && remaining > 0) {
        const int k = (int)std::min<int64_t>(check_every, max_steps - steps);
        if (persistent) {
            if (b->dirty && (st = build_tables(b))) break;
            if (b->use_graphs && k >= 2) {
                cudaGraphExec_t g;
                if ((st = batch_period_graph(b, cur, k, &g))) break;
                cudaError_t e = cudaGraphLaunch(g, b->stream);
                if (e != cudaSuccess) {
                    st = set_error(LBM_ERR_CUDA, "cudaGraphLaunch: %s", cudaGetErrorString(e));
                    break;
                }
                g_launches += b->run_graph_launches;
            } else {
                for (int i = 0; i < k && !st; ++i) {
                    cudaError_t e = launch_step(b, (cur + i) & 1, i == k - 1);
                    if (e != cudaSuccess) st = set_error(LBM_ERR_CUDA, "batch step: %s", cudaGetErrorString(e));
                }
                if (st) break;
                cudaError_t e = run_check_batch(b->dev, b->d_idx, b->nidx, k, b->stream);
                if (e != cudaSuccess) {
                    st = set_error(LBM_ERR_CUDA, "batch check: %s", cudaGetErrorString(e));
                    break;
                }
            }
            for (int i = 0; i < n; ++i)
                if (b->active[i]) {
                    b->cav[i]->cur = (cur + k) & 1;
                    b->cav[i]->itc += k;
                }
        } else {
            // one launch per member (the persistent kernel switched off)
            for (int i = 0; i < n && !st; ++i)
                if (b->active[i]) {
                    lbm_handle *h = b->cav[i];
                    if (h->cur != cur) {  // a member that waited for the host: realign its buffers
                        if ((st = change_storage(h, h->p.storage, cur))) break;
                    }
                    if ((st = lbm_step(h, k))) break;
                    cudaError_t e = run_check(h->geo, h->bufs, k, b->stream);
                    if (e != cudaSuccess) st = set_error(LBM_ERR_CUDA, "batch check: %s", cudaGetErrorString(e));
                }
            if (st) break;
        }
        cur = (cur + k) & 1;
        steps += k;
        if (++periods % kBatchPeriodsPerRead != 0 && steps < max_steps) continue;
        // read every member's run state: one copy, one synchronisation
        BCU(cudaMemcpyAsync(ctl.data(), b->d_ctl, sizeof(RunCtl) * n, cudaMemcpyDeviceToHost, b->stream));
        if ((st = lbm_batch_synchronize(b))) break;
        bool changed = false;
        std::vector<int> moved;
        for (int i = 0; i < n; ++i) {
            if (!b->active[i]) continue;
            if (ctl[i].status == -2) {
                st = set_error(LBM_ERR_NONFINITE, "check: non-finite residual sum (cavity %d)", i);
                break;
            }
            if (ctl[i].active) continue;
            if (two_phase && phase[i] == 1 && ctl[i].status == 1) {
                // met the FP32 criterion: on to FP64, in the batch's current buffer
                lbm_handle *h = b->cav[i];
                h->cur = (int)((base_cur[i] + (ctl[i].steps - base_steps[i])) & 1);
                if ((st = change_storage(h, LBM_STORE_F64, cur))) break;
                if (steps_low) steps_low[i] = ctl[i].steps;
                base_cur[i] = cur;
                base_steps[i] = ctl[i].steps;
                phase[i] = 2;
                RunCtl c = fresh(eps2);
                c.steps = ctl[i].steps;
                ctl[i] = c;
                moved.push_back(i);
                changed = true;
                continue;
            }
            b->active[i] = 0;
            --remaining;
            changed = true;
        }
        if (st) break;
        for (int i : moved)
            BCU(cudaMemcpyAsync(b->d_ctl + i, &ctl[i], sizeof(RunCtl), cudaMemcpyHostToDevice, b->stream));
        if (!moved.empty()) {
            std::vector<Bufs> bufs(n);
            for (int i = 0; i < n; ++i) bufs[i] = b->cav[i]->bufs;
            BCU(cudaMemcpyAsync(b->d_bufs, bufs.data(), sizeof(Bufs) * n, cudaMemcpyHostToDevice, b->stream));
            BCU(cudaStreamSynchronize(b->stream));
        }
        if (changed) b->dirty = true;
    }
    // the final state: iterations each member ran (every period ends with a
    // check, so the device count is exact), its parity and counter
    cudaError_t e = cudaMemcpyAsync(ctl.data(), b->d_ctl, sizeof(RunCtl) * n, cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess && !st) st = set_error(LBM_ERR_CUDA, "batch run state: %s", cudaGetErrorString(e));
    for (int i = 0; i < n; ++i) {
        const bool on = !mask || mask[i] != 0;
        if (!on) continue;
        lbm_handle *h = b->cav[i];
        const int64_t ran = ctl[i].steps;
        h->itc = itc0[i] + ran;
        h->cur = (int)((base_cur[i] + (ran - base_steps[i])) & 1);
        if (steps_done) steps_done[i] = ran;
        if (steps_low && two_phase && phase[i] == 1) steps_low[i] = ran;
        const bool done = !ctl[i].active && (!two_phase || phase[i] == 2 || ctl[i].status != 1);
        if (converged) converged[i] = done ? (ctl[i].status == 1 ? 1 : (ctl[i].status == -1 ? -1 : 0)) : 0;
        if (!st && ctl[i].status == -2) st = set_error(LBM_ERR_NONFINITE, "check: non-finite residual sum (cavity %d)", i);
    }
    // members in different storages leave their buffers in different parities;
    // bring every member on the mask to the same one for the next steps
    if (!st) {
        int c0 = -1;
        for (int i = 0; i < n && !st; ++i) {
            if (!(!mask || mask[i] != 0)) continue;
            if (c0 < 0) c0 = b->cav[i]->cur;
            if (b->cav[i]->cur != c0) st = change_storage(b->cav[i], b->cav[i]->p.storage, c0);
        }
        if (!st) {
            std::vector<Bufs> bufs(n);
            for (int i = 0; i < n; ++i) bufs[i] = b->cav[i]->bufs;
            e = cudaMemcpy(b->d_bufs, bufs.data(), sizeof(Bufs) * n, cudaMemcpyHostToDevice);
            if (e != cudaSuccess) st = set_error(LBM_ERR_CUDA, "batch tables: %s", cudaGetErrorString(e));
        }
    }
    for (auto &c : ctl) c.active = 1;
    e = cudaMemcpyAsync(b->d_ctl, ctl.data(), sizeof(RunCtl) * n, cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess && !st) st = set_error(LBM_ERR_CUDA, "batch run state: %s", cudaGetErrorString(e));
    // the batch's storage: the members' common one
    if (two_phase) {
        bool all64 = true;
        for (int i = 0; i < n; ++i) all64 = all64 && b->cav[i]->p.storage == LBM_STORE_F64;
        b->storage = all64 ? LBM_STORE_F64 : -1;
    }
    b->run_both = false;
    b->active.assign(n, 1);
    b->dirty = true;
    return st;
}

extern "C" int lbm_batch_run_masked(lbm_batch *b, const int32_t *mask, int32_t max_steps, int32_t check_every,
                                    double eps, int32_t *converged, int64_t *steps_done)
{
    return batch_run(b, mask, max_steps, check_every, eps, eps, false, converged, steps_done, nullptr);
}

extern "C" int lbm_batch_run_mixed(lbm_batch *b, const int32_t *mask, int32_t max_steps, int32_t check_every,
                                   double switch_eps, double eps, int32_t *converged, int64_t *steps_done,
                                   int64_t *steps_low)
{
    return batch_run(b, mask, max_steps, check_every, switch_eps, eps, true, converged, steps_done, steps_low);
}

extern "C" int lbm_batch_run(lbm_batch *b, int32_t max_steps, int32_t check_every, double eps, int32_t *converged,
                             int64_t *steps_done)
{
    return lbm_batch_run_masked(b, nullptr, max_steps, check_every, eps, converged, steps_done);
}

extern "C" int lbm_batch_set_storage(lbm_batch *b, int32_t storage)
{
    if (!b) return set_error(LBM_ERR_PARAM, "batch is NULL");
    if (storage == b->storage) return LBM_OK;
    BCU(cudaSetDevice(b->device));
    BCU(cudaStreamSynchronize(b->stream));
    drop_graphs(b);
    for (int i = 0; i < b->n; ++i) {
        int st = change_storage(b->cav[i], storage);
        if (st) return st;
    }
    b->storage = storage;
    std::vector<Bufs> bufs(b->n);
    for (int i = 0; i < b->n; ++i) bufs[i] = b->cav[i]->bufs;
    BCU(cudaMemcpy(b->d_bufs, bufs.data(), sizeof(Bufs) * b->n, cudaMemcpyHostToDevice));
    b->dirty = true;
    return LBM_OK;
}

static int tune_storage(lbm_batch *b, int32_t steps, int32_t *tile, int32_t *nblocks, double *mlups);

// The autotuner: every storage the caller's accuracy rule allows
// (LBM_BATCH_OPT_STORAGES; the current one if none is set) x tile width x
// grid size, timed on the batch itself; the batch keeps the fastest.
extern "C" int lbm_batch_tune(lbm_batch *b, int32_t steps, int32_t *tile, int32_t *nblocks, double *mlups)
{
    if (!b) return set_error(LBM_ERR_PARAM, "batch is NULL");
    if (b->storage < 0) {  // members in different storages after a mixed run: FP64 is always allowed
        int st = lbm_batch_set_storage(b, LBM_STORE_F64);
        if (st) return st;
    }
    const int mask = b->storages ? b->storages : (1 << b->storage);
    const int user_nb = b->nblocks_opt;  // a grid the caller set stays
    double best = -1.0;
    int best_store = b->storage, best_tile = 0, best_nb = 0;
    // the current storage first, so a single-storage rule converts nothing
    int order[3] = {b->storage, -1, -1}, no = 1;
    for (int s = 0; s < 3; ++s)
        if (s != b->storage && (mask >> s) & 1) order[no++] = s;
    for (int k = 0; k < no; ++k) {
        if (!((mask >> order[k]) & 1)) continue;
        int st = lbm_batch_set_storage(b, order[k]);
        if (st) return st;
        int t = 0, nb = 0;
        double v = 0.0;
        b->nblocks_opt = user_nb;
        if ((st = tune_storage(b, steps, &t, &nb, &v))) return st;
        if (v > best) {
            best = v;
            best_store = order[k];
            best_tile = t;
            best_nb = nb;
        }
    }
    int st = lbm_batch_set_storage(b, best_store);
    if (st) return st;
    if (b->dim == 2) b->tile = b->tile_opt = best_tile;
    b->nblocks_opt = user_nb > 0 ? user_nb : best_nb;
    b->dirty = true;
    if (tile) *tile = best_tile;
    if (nblocks) *nblocks = best_nb;
    if (mlups) *mlups = best;
    return LBM_OK;
}

// tile width x grid size for the batch's current storage
static int tune_storage(lbm_batch *b, int32_t steps, int32_t *tile, int32_t *nblocks, double *mlups)
{
    if (!b->persistent || !b->march_ok)
        return set_error(LBM_ERR_UNSUPPORTED, "lbm_batch_tune: the batch does not use the persistent kernel");
    if (steps < 2) steps = 2;
    BCU(cudaSetDevice(b->device));
    int sms = 0;
    BCU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
    const int tiles2[3] = {32, 64, 128}, tiles3[1] = {32};  // 3D: the tile is fixed at 32 x kBatchTileY
    const int *tiles = b->dim == 3 ? tiles3 : tiles2;
    const int ntile = b->dim == 3 ? 1 : 3;
    double best = -1.0;
    int best_tile = b->tile, best_nb = 0;
    cudaEvent_t e0, e1;
    BCU(cudaEventCreate(&e0));
    BCU(cudaEventCreate(&e1));
    const int keep_nb = b->nblocks_opt;
    for (int ti = 0; ti < ntile; ++ti) {
        const int t = tiles[ti];
        const int bps = b->dim == 3 ? (b->mode == LBM_MODE_EXACT ? exact::march_batch3d_blocks_per_sm(b->storage)
                                                                 : fast::march_batch3d_blocks_per_sm(b->storage))
                                    : (b->mode == LBM_MODE_EXACT ? exact::march_batch_blocks_per_sm(b->storage, t)
                                                                 : fast::march_batch_blocks_per_sm(b->storage, t));
        if (bps <= 0) continue;
        const int cands[2] = {bps, bps > 1 ? bps / 2 : 0};
        for (int c : cands) {
            if (c <= 0) continue;
            b->tile = t;
            b->nblocks_opt = c * sms;
            b->dirty = true;
            int st = lbm_batch_step(b, 2);  // warm-up, builds the tables
            if (st) return st;
            BCU(cudaEventRecord(e0, b->stream));
            st = lbm_batch_step(b, steps);
            if (st) return st;
            BCU(cudaEventRecord(e1, b->stream));
            st = lbm_batch_synchronize(b);
            if (st) return st;
            float ms = 0.f;
            BCU(cudaEventElapsedTime(&ms, e0, e1));
            const double v = (double)b->active_nodes * steps / (ms * 1e-3) / 1e6;
            if (v > best) {
                best = v;
                best_tile = t;
                best_nb = b->nblocks_opt;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->tile = best_tile;
    b->tile_opt = best_tile;
    b->nblocks_opt = keep_nb > 0 ? keep_nb : best_nb;
    b->dirty = true;
    if (tile) *tile = best_tile;
    if (nblocks) *nblocks = best_nb;
    if (mlups) *mlups = best;
    return LBM_OK;
}

extern "C" int lbm_batch_set_option(lbm_batch *b, int32_t option, int64_t value)
{
    if (!b) return set_error(LBM_ERR_PARAM, "batch is NULL");
    switch (option) {
    case LBM_BATCH_OPT_TILE:
        if (value != 32 && value != 64 && value != 128) return set_error(LBM_ERR_PARAM, "tile must be 32, 64 or 128");
        b->tile = b->tile_opt = (int)value;
        break;
    case LBM_BATCH_OPT_NBLOCKS:
        if (value < 0 || value > (1 << 20)) return set_error(LBM_ERR_PARAM, "nblocks out of range");
        b->nblocks_opt = (int)value;
        break;
    case LBM_BATCH_OPT_PERSISTENT:
        b->persistent = value != 0;
        break;
    case LBM_BATCH_OPT_GRAPHS:
        b->use_graphs = value != 0;
        break;
    case LBM_BATCH_OPT_GROWTH:
        if (value < 0) return set_error(LBM_ERR_PARAM, "growth factor must be >= 0");
        b->growth = (double)value;
        break;
    case LBM_BATCH_OPT_STORAGES:
        if (value < 0 || value > 7) return set_error(LBM_ERR_PARAM, "storage mask must be 0..7");
        if (b->mode == LBM_MODE_EXACT && (value & ~1))
            return set_error(LBM_ERR_UNSUPPORTED, "exact mode computes in FP64 storage only");
        b->storages = (int)value;
        break;
    case LBM_BATCH_OPT_PDL:
        if (value != 0 && value != 1) return set_error(LBM_ERR_PARAM, "PDL must be 0 or 1");
        BCU(cudaSetDevice(b->device));
        BCU(cudaStreamSynchronize(b->stream));
        drop_graphs(b);
        b->pdl = (int)value;
        break;
    default:
        return set_error(LBM_ERR_PARAM, "unknown batch option %d", option);
    }
    b->dirty = true;
    return LBM_OK;
}

extern "C" int lbm_batch_get_option(const lbm_batch *b, int32_t option, int64_t *value)
{
    if (!b || !value) return set_error(LBM_ERR_PARAM, "NULL argument");
    switch (option) {
    case LBM_BATCH_OPT_TILE: *value = b->tile; return LBM_OK;
    case LBM_BATCH_OPT_NBLOCKS: *value = b->nblocks; return LBM_OK;
    case LBM_BATCH_OPT_PERSISTENT: *value = b->persistent; return LBM_OK;
    case LBM_BATCH_OPT_GRAPHS: *value = b->use_graphs; return LBM_OK;
    case LBM_BATCH_OPT_GROWTH: *value = (int64_t)b->growth; return LBM_OK;
    case LBM_BATCH_OPT_STORAGES: *value = b->storages; return LBM_OK;
    case LBM_BATCH_OPT_STORAGE: *value = b->storage; return LBM_OK;
    case LBM_BATCH_OPT_PDL: *value = b->pdl; return LBM_OK;
    default: return set_error(LBM_ERR_PARAM, "unknown batch option %d", option);
    }
}

extern "C" int lbm_batch_stream(const lbm_batch *b, void **stream)
{
    if (!b || !stream) return set_error(LBM_ERR_PARAM, "NULL argument");
    *stream = (void *)b->stream;
    return LBM_OK;
}
