// C ABI of the B200 thermal LBM step (declared in include/lbm_b200.h).
//
// Host side of the drop-in boundary: parameter derivation and mesh as in the
// reference's mesh() / initial() (natural-convection_2dim_mono.f90:74-281,
// natural-convection_3dim_mono.f90:122-345), the interpolation weight tables
// of interpolate() (2M:591-660), and the run state of the time loop
// (2M:307-330).  Host arithmetic is compiled without multiply-add contraction
// so the derived parameters and weights are the reference's to the bit.
#include <cuda_runtime.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <cmath>
#include <vector>

#include "../../include/lbm_b200.h"
#include "lbm_handle.h"

using namespace lbm;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string t_last_error;

static int fail(int code, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
static int fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    t_last_error = buf;
    return code;
}

#define CU(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(e_ == cudaErrorMemoryAllocation ? LBM_ERR_NOMEM : LBM_ERR_CUDA,   \
                        "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

// error reporting for the other translation units of the library
int lbm::set_error(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    t_last_error = buf;
    return code;
}

extern "C" int lbm_abi_version(void) { return LBM_ABI_VERSION; }

extern "C" const char *lbm_error_string(int status)
{
    switch (status) {
    case LBM_OK: return "ok";
    case LBM_ERR_PARAM: return "bad parameter";
    case LBM_ERR_CUDA: return "CUDA error";
    case LBM_ERR_NONFINITE: return "non-finite value";
    case LBM_ERR_DIVERGED: return "residual diverged";
    case LBM_ERR_TIMEOUT: return "device wait timed out";
    case LBM_ERR_STATE: return "call out of order";
    case LBM_ERR_NOMEM: return "out of device memory";
    case LBM_ERR_UNSUPPORTED: return "unsupported option";
    case LBM_ERR_NODEVICE: return "no CUDA device";
    default: return "unknown status";
    }
}

extern "C" const char *lbm_last_error(void) { return t_last_error.c_str(); }

extern "C" int64_t lbm_kernel_launches(void) { return g_launches; }

// ---------------------------------------------------------------------------
// mesh() and initial() host arithmetic
// ---------------------------------------------------------------------------
static void grid_raw(int kind, int n, double stretch, double *xr)
{
    // 2M:86-88 (erf, constA = stretch); tanh and uniform variants
    for (int i = 0; i <= n + 1; ++i) {
        double xi = (double)i / (double)(n + 1);
        if (kind == LBM_GRID_ERF)
            xr[i] = 0.5 * (erf(stretch * ((double)i / (double)(n + 1) - 0.5)) / erf(0.5 * stretch) + 1.0);
        else if (kind == LBM_GRID_TANH)
            xr[i] = 0.5 * (tanh(stretch * (2.0 * xi - 1.0)) / tanh(stretch) + 1.0);
        else
            xr[i] = xi;
    }
}

extern "C" int lbm_mesh(int32_t kind, double stretch, int32_t nx, int32_t ny, int32_t nz, double *x, double *y,
                        double *z, double *dx0_out, double *length_LB_out, double *dt_out)
{
    if (kind < 0 || kind > 2) return fail(LBM_ERR_PARAM, "lbm_mesh: unknown grid kind %d", kind);
    if (nx < 3 || ny < 3 || (z && nz < 3)) return fail(LBM_ERR_PARAM, "lbm_mesh: need >= 3 nodes per axis");
    if (!x || !y) return fail(LBM_ERR_PARAM, "lbm_mesh: x and y are required");
    if (kind != LBM_GRID_UNIFORM && !(stretch > 0.0))
        return fail(LBM_ERR_PARAM, "lbm_mesh: stretch must be > 0");
    grid_raw(kind, nx, stretch, x);
    grid_raw(kind, ny, stretch, y);
    if (z) grid_raw(kind, nz, stretch, z);
    // 2M:94-116: spacing of the first x cell sets the lattice unit
    const double dx1 = x[1] - x[0];
    const double dx0 = dx1, dt0 = dx0;
    const double length_LB = 1.0 / dx1;
    const double dt = dt0 * length_LB;
    for (int i = 1; i <= nx; ++i) x[i] = x[i] - dx0 / 2.0;
    for (int j = 1; j <= ny; ++j) y[j] = y[j] - dx0 / 2.0;
    if (z) for (int k = 1; k <= nz; ++k) z[k] = z[k] - dx0 / 2.0;
    for (int i = 0; i <= nx + 1; ++i) x[i] = x[i] * length_LB;
    for (int j = 0; j <= ny + 1; ++j) y[j] = y[j] * length_LB;
    if (z) for (int k = 0; k <= nz + 1; ++k) z[k] = z[k] * length_LB;
    if (dx0_out) *dx0_out = dx0;
    if (length_LB_out) *length_LB_out = length_LB;
    if (dt_out) *dt_out = dt;
    return LBM_OK;
}

extern "C" int lbm_mesh_box(int32_t kind, double stretch, int32_t nx, int32_t ny, int32_t nz, double lx, double ly,
                            double lz, double *x, double *y, double *z, double *dx0_out, double *length_LB_out,
                            double *dt_out)
{
    if (kind < 0 || kind > 2) return fail(LBM_ERR_PARAM, "lbm_mesh_box: unknown grid kind %d", kind);
    if (nx < 3 || ny < 3 || (z && nz < 3)) return fail(LBM_ERR_PARAM, "lbm_mesh_box: need >= 3 nodes per axis");
    if (!x || !y) return fail(LBM_ERR_PARAM, "lbm_mesh_box: x and y are required");
    if (!(lx > 0) || !(ly > 0) || (z && !(lz > 0))) return fail(LBM_ERR_PARAM, "lbm_mesh_box: lengths must be > 0");
    if (kind != LBM_GRID_UNIFORM && !(stretch > 0.0)) return fail(LBM_ERR_PARAM, "lbm_mesh_box: stretch must be > 0");
    grid_raw(kind, nx, stretch, x);
    grid_raw(kind, ny, stretch, y);
    if (z) grid_raw(kind, nz, stretch, z);
    if (lx != 1.0)
        for (int i = 0; i <= nx + 1; ++i) x[i] = x[i] * lx;
    if (ly != 1.0)
        for (int j = 0; j <= ny + 1; ++j) y[j] = y[j] * ly;
    if (z && lz != 1.0)
        for (int k = 0; k <= nz + 1; ++k) z[k] = z[k] * lz;
    // the finest first cell over the axes sets the lattice unit
    double dx1 = x[1] - x[0];
    if (y[1] - y[0] < dx1) dx1 = y[1] - y[0];
    if (z && z[1] - z[0] < dx1) dx1 = z[1] - z[0];
    const double dx0 = dx1, dt0 = dx0;
    const double length_LB = 1.0 / dx1;
    const double dt = dt0 * length_LB;
    for (int i = 1; i <= nx; ++i) x[i] = x[i] - dx0 / 2.0;
    for (int j = 1; j <= ny; ++j) y[j] = y[j] - dx0 / 2.0;
    if (z) for (int k = 1; k <= nz; ++k) z[k] = z[k] - dx0 / 2.0;
    for (int i = 0; i <= nx + 1; ++i) x[i] = x[i] * length_LB;
    for (int j = 0; j <= ny + 1; ++j) y[j] = y[j] * length_LB;
    if (z) for (int k = 0; k <= nz + 1; ++k) z[k] = z[k] * length_LB;
    if (dx0_out) *dx0_out = dx0;
    if (length_LB_out) *length_LB_out = length_LB;
    if (dt_out) *dt_out = dt;
    return LBM_OK;
}

static Derived derive(const lbm_params &p)
{
    // 2M:152-162 and 3M:207-229
    Derived d;
    d.viscosity_LB = (p.Ma * (p.length_LB - 1.0) * sqrt(p.Pr)) / sqrt(3.0 * p.Ra);
    d.kappa = d.viscosity_LB / p.Pr;
    const double L1 = p.length_LB - 1.0;
    d.gbeta = p.Ra * d.viscosity_LB * d.kappa / ((L1 * L1) * L1);
    d.tauf = d.viscosity_LB * 3.0 + 0.5;
    d.Snu = 1.0 / d.tauf;
    d.Sq = 8.0 * (2.0 - d.Snu) / (8.0 - d.Snu);
    if (p.dim == 2)
        d.sig_k = 1.0 / (0.5 + 4.0 * (1.0 / d.Snu - 0.5) / (3.0 * p.Pr));
    else
        d.sig_k = 1.0 / (0.5 + (1.0 / d.Snu - 0.5) / (0.5 * p.Pr));
    return d;
}

static int validate(const lbm_params *p)
{
    if (!p) return fail(LBM_ERR_PARAM, "params is NULL");
    if (p->dim != 2 && p->dim != 3) return fail(LBM_ERR_PARAM, "dim must be 2 or 3 (got %d)", p->dim);
    if (p->nx < 3 || p->ny < 3 || (p->dim == 3 && p->nz < 3))
        return fail(LBM_ERR_PARAM, "need >= 3 nodes per axis (got %d x %d x %d)", p->nx, p->ny, p->nz);
    const double lim = 1 << 24;
    if (p->nx > lim || p->ny > lim || (p->dim == 3 && p->nz > lim))
        return fail(LBM_ERR_PARAM, "axis too long");
    if (!(p->Ra > 0) || !(p->Pr > 0) || !(p->Ma > 0)) return fail(LBM_ERR_PARAM, "Ra, Pr, Ma must be > 0");
    if (!(p->dt > 0) || !isfinite(p->dt)) return fail(LBM_ERR_PARAM, "dt must be finite and > 0");
    if (!(p->length_LB > 1.0) || !isfinite(p->length_LB)) return fail(LBM_ERR_PARAM, "length_LB must be > 1");
    if (!isfinite(p->Thot) || !isfinite(p->Tcold) || p->Thot == p->Tcold)
        return fail(LBM_ERR_PARAM, "Thot and Tcold must be finite and differ");
    if (p->storage == LBM_STORE_F16S)
        return fail(LBM_ERR_UNSUPPORTED, "binary16 population storage is retired (inaccurate, not faster than FP32)");
    if (p->storage != LBM_STORE_F64 && p->storage != LBM_STORE_F32)
        return fail(LBM_ERR_PARAM, "unknown storage %d", p->storage);
    if (p->mode != LBM_MODE_FAST && p->mode != LBM_MODE_EXACT) return fail(LBM_ERR_PARAM, "unknown mode %d", p->mode);
    if (p->mode == LBM_MODE_EXACT && p->storage != LBM_STORE_F64)
        return fail(LBM_ERR_UNSUPPORTED, "exact mode needs FP64 storage");
    if (p->reserved != 0) return fail(LBM_ERR_PARAM, "reserved field must be 0");
    return LBM_OK;
}

extern "C" int lbm_derived_params(const lbm_params *p, double *out9)
{
    int st = validate(p);
    if (st) return st;
    if (!out9) return fail(LBM_ERR_PARAM, "out is NULL");
    Derived d = derive(*p);
    out9[0] = d.viscosity_LB; out9[1] = d.kappa; out9[2] = d.gbeta; out9[3] = d.tauf;
    out9[4] = d.Snu; out9[5] = d.Sq; out9[6] = d.sig_k; out9[7] = p->dt; out9[8] = p->length_LB;
    return LBM_OK;
}

// Interpolation weights of interpolateF (2M:649-660) for every node of one
// axis and both shift signs, in the stencil order of inter_x (2B:246-296):
// tab[(i-1)*6 + s*3 + c], s = 0 for a +dt shift, 1 for -dt.
static void axis_weights(const double *c, int n, double dt, double *tab)
{
    for (int i = 1; i <= n; ++i) {
        int a, m = i, b;
        if (i == 1) { a = i + 1; b = i + 2; }
        else if (i == n) { a = i - 1; b = i - 2; }
        else { a = i - 1; b = i + 1; }
        for (int s = 0; s < 2; ++s) {
            const double delta = (s == 0 ? 1.0 : -1.0) * dt;
            const double x0 = c[a] + delta, x1 = c[m] + delta, x2 = c[b] + delta, x = c[m];
            double *w = tab + (int64_t)(i - 1) * 6 + s * 3;
            w[0] = ((x - x1) * (x - x2)) / ((x0 - x1) * (x0 - x2));
            w[1] = ((x - x0) * (x - x2)) / ((x1 - x0) * (x1 - x2));
            w[2] = ((x - x0) * (x - x1)) / ((x2 - x0) * (x2 - x1));
        }
    }
}

// cell widths of nodes 1..n: the wall lies dt/2 outside the end nodes
static void cell_widths(const double *c, int n, double dt, double *wd)
{
    const double lo = c[1] - 0.5 * dt, hi = c[n] + 0.5 * dt;
    for (int i = 1; i <= n; ++i) {
        const double a = (i == 1) ? lo : 0.5 * (c[i - 1] + c[i]);
        const double b = (i == n) ? hi : 0.5 * (c[i] + c[i + 1]);
        wd[i - 1] = b - a;
    }
}

static int set_device(const lbm_handle *h)
{
    CU(cudaSetDevice(h->device));
    return LBM_OK;
}

template <class T>
static int dalloc(lbm_handle *h, T **ptr, size_t bytes)
{
    cudaError_t e = cudaMalloc((void **)ptr, bytes);
    if (e != cudaSuccess) {
        *ptr = nullptr;
        return fail(e == cudaErrorMemoryAllocation ? LBM_ERR_NOMEM : LBM_ERR_CUDA, "cudaMalloc(%zu): %s", bytes,
                    cudaGetErrorString(e));
    }
    h->bytes += (int64_t)bytes;
    return LBM_OK;
}

static void free_all(lbm_handle *h)
{
    lbm::drop_graphs(h);
    void *ptrs[] = {h->bufs.pop[0], h->bufs.pop[1], h->bufs.F[0], h->bufs.F[1], h->bufs.rho, h->bufs.u,
                    h->bufs.v, h->bufs.w, h->bufs.T, h->bufs.up, h->bufs.vp, h->bufs.wp, h->bufs.Tp,
                    h->bufs.partials, h->bufs.scal, h->d_wgt[0], h->d_wgt[1], h->d_wgt[2], h->d_coord[0],
                    h->d_coord[1], h->d_coord[2], h->d_cellw[0], h->d_cellw[1], h->d_cellw[2], h->staging,
                    h->aos, h->bufs.err, h->d_bar, h->d_msegs, h->d_msegoff, h->owns_ctl ? h->bufs.ctl : nullptr};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (h->stream && h->owns_stream) cudaStreamDestroy(h->stream);
}

extern "C" int lbm_destroy(lbm_handle *h)
{
    if (!h) return LBM_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    free_all(h);
    delete h;
    return LBM_OK;
}

// ---------------------------------------------------------------------------
// TMA descriptors for the march kernels
// ---------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    }
    return fn;
}

// Describe a population buffer as a (x, y, [z,] plane) tensor; one descriptor
// per box class of the march kernel.  Returns false if TMA cannot be used.
bool lbm::encode_maps_tx(const lbm_handle *h, int tx, TmapSet out[2])
{
    EncodeTiledFn enc = encode_fn();
    if (!enc) return false;
    const Geo &g = h->geo;
    const MarchShape ms = march_shape(g.dim, h->p.storage, tx, h->tiley);
    const CUtensorMapDataType dtype =
        h->p.storage == LBM_STORE_F64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    const cuuint64_t es = h->esize;
    const int nplanes = h->Q + h->QT;
    const CUtensorMapL2promotion promo = h->l2promo == 3   ? CU_TENSOR_MAP_L2_PROMOTION_L2_256B
                                         : h->l2promo == 2 ? CU_TENSOR_MAP_L2_PROMOTION_L2_128B
                                         : h->l2promo == 1 ? CU_TENSOR_MAP_L2_PROMOTION_L2_64B
                                                           : CU_TENSOR_MAP_L2_PROMOTION_NONE;
    for (int buf = 0; buf < 2; ++buf) {
        for (int c = 0; c < 4; ++c) {
            CUtensorMap *m = &out[buf].m[c];
            CUresult r;
            if (g.dim == 3) {
                const cuuint64_t dims[4] = {(cuuint64_t)g.nx, (cuuint64_t)g.ny, (cuuint64_t)g.nz, (cuuint64_t)nplanes};
                const cuuint64_t strides[3] = {(cuuint64_t)g.pitch * es, (cuuint64_t)g.slab * es,
                                               (cuuint64_t)g.plane * es};
                const cuuint32_t box[4] = {(cuuint32_t)ms.bx[c], (cuuint32_t)ms.by[c], 1, 1};
                const cuuint32_t estr[4] = {1, 1, 1, 1};
                r = enc(m, dtype, 4, h->bufs.pop[buf], dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_NONE, promo, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            } else {
                const int cc = c & 1;
                const cuuint64_t dims[3] = {(cuuint64_t)g.nx, (cuuint64_t)g.ny, (cuuint64_t)nplanes};
                const cuuint64_t strides[2] = {(cuuint64_t)g.pitch * es, (cuuint64_t)g.plane * es};
                const cuuint32_t box[3] = {(cuuint32_t)ms.bx[cc], 1, 1};
                const cuuint32_t estr[3] = {1, 1, 1};
                r = enc(m, dtype, 3, h->bufs.pop[buf], dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_NONE, promo, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            }
            if (r != CUDA_SUCCESS) return false;
        }
        // the carried force of this buffer: compute type, one value per node
        const CUtensorMapDataType ftype =
            h->csize == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
        const cuuint64_t cs = h->csize;
        CUresult r;
        if (g.dim == 3) {
            const cuuint64_t dims[3] = {(cuuint64_t)g.nx, (cuuint64_t)g.ny, (cuuint64_t)g.nz};
            const cuuint64_t strides[2] = {(cuuint64_t)g.pitch * cs, (cuuint64_t)g.slab * cs};
            const cuuint32_t box[3] = {(cuuint32_t)ms.TX, (cuuint32_t)ms.TY, 1};
            const cuuint32_t estr[3] = {1, 1, 1};
            r = enc(&out[buf].fmap, ftype, 3, h->bufs.F[buf], dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, promo, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        } else {
            const cuuint64_t dims[2] = {(cuuint64_t)g.nx, (cuuint64_t)g.ny};
            const cuuint64_t strides[1] = {(cuuint64_t)g.pitch * cs};
            const cuuint32_t box[2] = {(cuuint32_t)ms.TX, 1};
            const cuuint32_t estr[2] = {1, 1};
            r = enc(&out[buf].fmap, ftype, 2, h->bufs.F[buf], dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, promo, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        }
        if (r != CUDA_SUCCESS) return false;
    }
    return true;
}

static bool encode_maps(lbm_handle *h) { return lbm::encode_maps_tx(h, 0, h->tmaps); }

// The march kernel handles every size except, in 3D, a last tile row holding
// a single y-row (its one-sided stencil would reach two rows below the box).
static bool march_supported(const lbm_handle *h)
{
    if (!h->march_ok) return false;
    const MarchShape ms = march_shape(h->geo.dim, h->p.storage, 0, h->tiley);
    if (h->geo.dim == 3 && h->geo.ny % ms.TY == 1) return false;
    return true;
}

// tile rows of the 3D march kernel unless LBM_OPT_TILEY says otherwise: 32 x 4
// tiles run two blocks per SM; measured on B200 at 128^3 FP64 (balanced plan)
// 13.0 GLUPS against 12.0 GLUPS with 32 x 8 tiles and one block per SM
static constexpr int kDefaultTileY = 4;

// ---------------------------------------------------------------------------
// 3D march work plan
// ---------------------------------------------------------------------------
// Neighbouring tiles share halo rows and columns: when two neighbours are at
// the same slice at about the same time, the second reader finds those rows
// in L2.  A grid of (tile columns x equal z-chunks) blocks keeps every tile in
// lockstep with its neighbours but seldom fills the SMs: the 64 tile columns
// of a 128^3 cube on 148 SMs give 2 chunks, 128 blocks, and 20 idle SMs.  Here
// the left-over blocks take each chunk's last r slices ("tails"), round-robin
// over the tails in (chunk, tile) order, so each round is a patch of
// consecutive tiles that also run side by side.  r balances a main chunk (its
// length less r, plus one pipeline start) against the busiest tail block
// (one start and r slices per round).
int lbm::plan_march3d(int ntiles, int nz, int nblocks, int kind, std::vector<int4> &segs, std::vector<int> &off)
{
    segs.clear();
    off.clear();
    const int64_t total = (int64_t)ntiles * nz;
    int64_t G = nblocks < 1 ? 1 : nblocks;
    if (G > total) G = total;
    auto push = [&](int t, int z0, int z1) { segs.push_back(make_int4(t, z0, z1, 0)); };
    const int c = (int)(G / ntiles);
    if (kind == 1 || c < 1) {
        for (int64_t b = 0; b < G; ++b) {
            off.push_back((int)segs.size());
            int64_t u = total * b / G;
            const int64_t hi = total * (b + 1) / G;
            while (u < hi) {
                const int t = (int)(u / nz), z0 = (int)(u % nz);
                const int z1 = (int)std::min<int64_t>(nz, z0 + (hi - u));
                push(t, z0, z1);
                u += z1 - z0;
            }
        }
        off.push_back((int)segs.size());
        return (int)G;
    }
    const int E = (int)(G - (int64_t)c * ntiles);
    auto zb = [&](int k) { return (int)((int64_t)k * nz / c); };
    const int minL = nz / c;  // chunk lengths are minL or minL + 1
    int r = 0;
    if (E > 0 && minL >= 4) {
        const double start = 1.5;  // a segment's pipeline start, in slice times
        const int rounds = (c * ntiles + E - 1) / E;
        double best = (double)(minL + 1) + start;  // r = 0: the left-over blocks stay idle
        for (int rr = 1; rr < minL / 2; ++rr) {
            const double t = std::max((double)(minL + 1 - rr) + start, rounds * (rr + start));
            if (t < best - 1e-9) {
                best = t;
                r = rr;
            }
        }
    }
    for (int k = 0; k < c; ++k)
        for (int t = 0; t < ntiles; ++t) {
            off.push_back((int)segs.size());
            push(t, zb(k), zb(k + 1) - r);
        }
    if (r > 0) {
        const int ntail = c * ntiles;
        for (int e = 0; e < E; ++e) {
            off.push_back((int)segs.size());
            for (int i = e; i < ntail; i += E) push(i % ntiles, zb(i / ntiles + 1) - r, zb(i / ntiles + 1));
        }
    }
    off.push_back((int)segs.size());
    return (int)off.size() - 1;
}

// plan the 3D march for grid G and upload it; sets h->nblocks
static int upload_plan3d(lbm_handle *h, int G)
{
    CU(cudaStreamSynchronize(h->stream));  // no launch in flight reads the old plan
    const MarchShape ms = march_shape(3, h->p.storage, 0, h->tiley);
    const int ntiles = ((h->geo.nx + ms.TX - 1) / ms.TX) * ((h->geo.ny + ms.TY - 1) / ms.TY);
    std::vector<int4> segs;
    std::vector<int> off;
    // the slices the handle computes: all of them, or a slab's own [klo, khi)
    const int nb = lbm::plan_march3d(ntiles, h->geo.khi - h->geo.klo, G, h->plan_opt, segs, off);
    for (int4 &s : segs) {
        s.y += h->geo.klo;
        s.z += h->geo.klo;
    }
    if (segs.size() > h->msegs_cap) {
        if (h->d_msegs) cudaFree(h->d_msegs);
        h->d_msegs = nullptr;
        h->msegs_cap = 0;
        int st = dalloc(h, &h->d_msegs, sizeof(int4) * segs.size());
        if (st) return st;
        h->msegs_cap = segs.size();
    }
    if (off.size() > h->msegoff_cap) {
        if (h->d_msegoff) cudaFree(h->d_msegoff);
        h->d_msegoff = nullptr;
        h->msegoff_cap = 0;
        int st = dalloc(h, &h->d_msegoff, sizeof(int) * off.size());
        if (st) return st;
        h->msegoff_cap = off.size();
    }
    CU(cudaMemcpy(h->d_msegs, segs.data(), sizeof(int4) * segs.size(), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(h->d_msegoff, off.data(), sizeof(int) * off.size(), cudaMemcpyHostToDevice));
    h->nblocks = nb;
    return LBM_OK;
}

extern "C" int lbm_march_plan3d(int32_t ntiles, int32_t nz, int32_t nblocks, int32_t kind, int32_t *seg_count,
                                int32_t *segs, int32_t *off, int32_t *blocks_used)
{
    if (ntiles < 1 || nz < 3 || nblocks < 1 || (kind != 0 && kind != 1) || !seg_count)
        return fail(LBM_ERR_PARAM, "lbm_march_plan3d: bad arguments");
    std::vector<int4> sg;
    std::vector<int> of;
    const int nb = lbm::plan_march3d(ntiles, nz, nblocks, kind, sg, of);
    const int cap = *seg_count;
    *seg_count = (int32_t)sg.size();
    if (blocks_used) *blocks_used = nb;
    if (!segs || !off) return LBM_OK;  // size query
    if ((int)sg.size() > cap) return fail(LBM_ERR_PARAM, "lbm_march_plan3d: %d segments do not fit", (int)sg.size());
    for (size_t i = 0; i < sg.size(); ++i) {
        segs[3 * i] = sg[i].x;
        segs[3 * i + 1] = sg[i].y;
        segs[3 * i + 2] = sg[i].z;
    }
    for (size_t i = 0; i < of.size(); ++i) off[i] = of[i];
    return LBM_OK;
}

static int resolve_path(lbm_handle *h)
{
    lbm::drop_graphs(h);
    const bool ok = march_supported(h);
    if (h->kernel_opt == 2 && !ok)
        return fail(LBM_ERR_UNSUPPORTED, "march kernel not available for this shape / device");
    h->use_march = h->kernel_opt == 2 || (h->kernel_opt == 0 && ok && h->geo.nnode >= (1 << 15));
    if (h->use_march) {
        const int bps = h->p.mode == LBM_MODE_EXACT ? exact::march_blocks_per_sm(h->geo, h->p.storage, h->tiley)
                                                   : fast::march_blocks_per_sm(h->geo, h->p.storage, h->tiley);
        if (bps <= 0) {
            if (h->kernel_opt == 2) return fail(LBM_ERR_UNSUPPORTED, "march kernel cannot be resident");
            h->use_march = 0;
            return LBM_OK;
        }
        int sms = 0;
        CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
        const int slots = bps * sms;
        if (h->geo.dim == 3) {
            // one full wave, planned
            int st = upload_plan3d(h, h->nblocks_opt > 0 ? h->nblocks_opt : slots);
            if (st) return st;
        } else if (h->nblocks_opt > 0) {
            h->nblocks = h->nblocks_opt;
        } else {
            // z-lockstep grid: every tile column split into the same number of
            // chunks, so neighbouring tiles are processed at the same slice and
            // their shared halo rows are served from L2; used when it fills at
            // least 80 % of the resident slots, otherwise one full wave with an
            // equal share of tile-slices per block
            const MarchShape ms = march_shape(h->geo.dim, h->p.storage);
            const int64_t ntiles = (int64_t)((h->geo.nx + ms.TX - 1) / ms.TX) *
                                   (h->geo.dim == 3 ? (h->geo.ny + ms.TY - 1) / ms.TY : 1);
            const int64_t chunks = ntiles <= slots ? slots / ntiles : 0;
            if (chunks > 0 && ntiles * chunks * 5 >= (int64_t)slots * 4)
                h->nblocks = (int)(ntiles * chunks);
            else
                h->nblocks = slots;
        }
    }
    // small 2D domains: every iteration of an lbm_step call in one resident
    // cooperative launch (the per-iteration launch gap dominates there)
    h->resident = 0;
    if (!h->use_march && h->p.dim == 2 && h->resident_opt && h->owns_stream && h->d_bar && h->geo.jlo == 0 &&
        h->geo.jhi == h->geo.ny) {
        const int nb = h->p.mode == LBM_MODE_EXACT ? exact::resident_blocks(h->geo, h->p.storage, h->device)
                                                   : fast::resident_blocks(h->geo, h->p.storage, h->device);
        if (nb > 0 && (int64_t)nb * 256 >= h->geo.nnode) h->resident = nb;
    }
    return LBM_OK;
}

extern "C" int lbm_create(const lbm_params *p, const double *x, const double *y, const double *z, lbm_handle **out)
{
    if (!out) return fail(LBM_ERR_PARAM, "out is NULL");
    *out = nullptr;
    int st = validate(p);
    if (st) return st;
    if (!x || !y || (p->dim == 3 && !z)) return fail(LBM_ERR_PARAM, "coordinates missing");
    const int n[3] = {p->nx, p->ny, p->dim == 3 ? p->nz : 1};
    const double *c[3] = {x, y, z};
    for (int a = 0; a < p->dim; ++a) {
        for (int i = 0; i <= n[a] + 1; ++i)
            if (!isfinite(c[a][i])) return fail(LBM_ERR_PARAM, "axis %d: coordinate %d not finite", a, i);
        for (int i = 1; i < n[a]; ++i)
            if (!(c[a][i + 1] > c[a][i])) return fail(LBM_ERR_PARAM, "axis %d: nodes not increasing at %d", a, i);
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(LBM_ERR_NODEVICE, "no CUDA device");
    if (p->device < 0 || p->device >= ndev) return fail(LBM_ERR_PARAM, "device %d out of range", p->device);

    lbm_handle *h = new lbm_handle();
    h->p = *p;
    if (p->dim == 2) h->p.nz = 1;
    h->d = derive(h->p);
    h->device = p->device;
    h->Q = p->dim == 2 ? 9 : 19;
    h->QT = p->dim == 2 ? 5 : 7;
    h->esize = p->storage == LBM_STORE_F64 ? 8 : 4;
    h->csize = p->storage == LBM_STORE_F64 ? 8 : 4;

    auto bail = [&](int code) {
        free_all(h);
        delete h;
        return code;
    };
    if ((st = set_device(h))) return bail(st);
    {
        cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) return bail(fail(LBM_ERR_CUDA, "stream: %s", cudaGetErrorString(e)));
    }

    Geo &g = h->geo;
    memset(&g, 0, sizeof g);
    g.dim = p->dim;
    g.nx = h->p.nx; g.ny = h->p.ny; g.nz = h->p.nz;
    g.jlo = 0;
    g.jhi = g.ny;
    g.klo = 0;
    g.khi = g.nz;
    // rows padded to 16 bytes for every storage type (TMA stride rule)
    g.pitch = (g.nx + 7) / 8 * 8;
    g.slab = g.pitch * g.ny;
    const int64_t cells = g.slab * g.nz;
    g.plane = (cells + 127) / 128 * 128;
    g.nnode = (int64_t)g.nx * g.ny * g.nz;
    g.Snu = h->d.Snu; g.Sq = h->d.Sq; g.sig_k = h->d.sig_k; g.gbeta = h->d.gbeta;
    g.dt = p->dt; g.Thot = p->Thot; g.Tcold = p->Tcold; g.T0 = 0.5 * (p->Thot + p->Tcold);
    g.length_LB = p->length_LB;
    tc_setup(g, c[p->dim == 2 ? 0 : 1]);

    // coordinates, weights, cell widths
    for (int a = 0; a < 3; ++a) {
        const int na = n[a];
        h->coord[a].assign(na + 2, 0.0);
        if (a < p->dim) memcpy(h->coord[a].data(), c[a], sizeof(double) * (na + 2));
        std::vector<double> wt((size_t)na * 6, 0.0), cw((size_t)na, 1.0);
        if (a < p->dim) {
            axis_weights(h->coord[a].data(), na, p->dt, wt.data());
            cell_widths(h->coord[a].data(), na, p->dt, cw.data());
        }
        if ((st = dalloc(h, &h->d_wgt[a], wt.size() * 8))) return bail(st);
        if ((st = dalloc(h, &h->d_coord[a], h->coord[a].size() * 8))) return bail(st);
        if ((st = dalloc(h, &h->d_cellw[a], cw.size() * 8))) return bail(st);
        if (cudaMemcpy(h->d_wgt[a], wt.data(), wt.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(h->d_coord[a], h->coord[a].data(), h->coord[a].size() * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(h->d_cellw[a], cw.data(), cw.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess)
            return bail(fail(LBM_ERR_CUDA, "upload of axis tables failed"));
        g.wgt[a] = h->d_wgt[a];
        g.coord[a] = h->d_coord[a];
        g.cellw[a] = h->d_cellw[a];
    }

    // state
    Bufs &b = h->bufs;
    memset(&b, 0, sizeof b);
    const size_t popb = (size_t)(h->Q + h->QT) * (size_t)g.plane * h->esize;
    const size_t fb = (size_t)g.plane * h->csize;
    const size_t mb = (size_t)g.nnode * 8;
    if ((st = dalloc(h, &b.pop[0], popb)) || (st = dalloc(h, &b.pop[1], popb)) ||
        (st = dalloc(h, &b.F[0], fb)) || (st = dalloc(h, &b.F[1], fb)) || (st = dalloc(h, &b.rho, mb)) ||
        (st = dalloc(h, &b.u, mb)) || (st = dalloc(h, &b.v, mb)) || (st = dalloc(h, &b.w, mb)) ||
        (st = dalloc(h, &b.T, mb)) || (st = dalloc(h, &b.up, mb)) || (st = dalloc(h, &b.vp, mb)) ||
        (st = dalloc(h, &b.wp, mb)) || (st = dalloc(h, &b.Tp, mb)) ||
        (st = dalloc(h, &b.partials, 592 * 4 * 8)) || (st = dalloc(h, &b.scal, 16 * 8)))
        return bail(st);
    if ((st = dalloc(h, &b.err, 16))) return bail(st);
    if ((st = dalloc(h, &b.ctl, sizeof(RunCtl)))) return bail(st);
    {
        RunCtl c{};
        c.active = 1;
        if (cudaMemcpy(b.ctl, &c, sizeof c, cudaMemcpyHostToDevice) != cudaSuccess)
            return bail(fail(LBM_ERR_CUDA, "run state upload failed"));
    }
    if ((st = dalloc(h, &h->d_bar, 2 * sizeof(unsigned)))) return bail(st);
    if (cudaMemset(h->d_bar, 0, 2 * sizeof(unsigned)) != cudaSuccess)
        return bail(fail(LBM_ERR_CUDA, "memset failed"));
    if (cudaMemset(b.F[0], 0, fb) != cudaSuccess || cudaMemset(b.F[1], 0, fb) != cudaSuccess ||
        cudaMemset(b.w, 0, mb) != cudaSuccess || cudaMemset(b.wp, 0, mb) != cudaSuccess ||
        cudaMemset(b.err, 0, 16) != cudaSuccess || cudaMemset(b.pop[0], 0, popb) != cudaSuccess ||
        cudaMemset(b.pop[1], 0, popb) != cudaSuccess)
        return bail(fail(LBM_ERR_CUDA, "memset failed"));
    h->tiley = kDefaultTileY;
    h->march_ok = encode_maps(h);
    if ((st = resolve_path(h))) return bail(st);
    h->phase = 0;
    *out = h;
    return LBM_OK;
}

#define CHECK_H(h)                                                        \
    do {                                                                  \
        if (!(h)) return fail(LBM_ERR_PARAM, "handle is NULL");           \
        int st_ = set_device(h);                                          \
        if (st_) return st_;                                              \
    } while (0)

static cudaError_t launch_equilibrium(lbm_handle *h, void *pop, int neq = 0)
{
    // first-order non-equilibrium coefficients: 3 tau_f dt and tau_T dt with
    // tau_T = 1 / sig_k (the relaxation times of the stress and heat-flux moments)
    const double cf = 3.0 * h->d.tauf * h->p.dt;
    const double ct = (1.0 / h->d.sig_k) * h->p.dt;
    return h->p.mode == LBM_MODE_EXACT
               ? exact::equilibrium(h->geo, h->p.storage, pop, h->bufs, neq, cf, ct, h->stream)
               : fast::equilibrium(h->geo, h->p.storage, pop, h->bufs, neq, cf, ct, h->stream);
}

static int reset_run(lbm_handle *h)
{
    const size_t mb = (size_t)h->geo.nnode * 8;
    CU(cudaMemsetAsync(h->bufs.up, 0, mb, h->stream));
    CU(cudaMemsetAsync(h->bufs.vp, 0, mb, h->stream));
    CU(cudaMemsetAsync(h->bufs.wp, 0, mb, h->stream));
    CU(cudaMemsetAsync(h->bufs.Tp, 0, mb, h->stream));
    h->itc = 0;
    return LBM_OK;
}

static int upload_macro(lbm_handle *h, const double *rho, const double *u, const double *v, const double *w,
                        const double *T)
{
    const size_t mb = (size_t)h->geo.nnode * 8;
    if (rho) CU(cudaMemcpyAsync(h->bufs.rho, rho, mb, cudaMemcpyHostToDevice, h->stream));
    if (u) CU(cudaMemcpyAsync(h->bufs.u, u, mb, cudaMemcpyHostToDevice, h->stream));
    if (v) CU(cudaMemcpyAsync(h->bufs.v, v, mb, cudaMemcpyHostToDevice, h->stream));
    if (w && h->p.dim == 3) CU(cudaMemcpyAsync(h->bufs.w, w, mb, cudaMemcpyHostToDevice, h->stream));
    if (T) CU(cudaMemcpyAsync(h->bufs.T, T, mb, cudaMemcpyHostToDevice, h->stream));
    return LBM_OK;
}

extern "C" int lbm_init_reference(lbm_handle *h)
{
    CHECK_H(h);
    // initial(): rho = rho0, u = v = 0, T linear between the isothermal
    // walls (2M:200-212 in x; 3M:257-271 in y)
    const lbm_params &p = h->p;
    const int64_t N = h->geo.nnode;
    std::vector<double> rho((size_t)N, 1.0), zero((size_t)N, 0.0), T((size_t)N);
    for (int k = 0; k < p.nz; ++k)
        for (int j = 1; j <= p.ny; ++j)
            for (int i = 1; i <= p.nx; ++i) {
                const int64_t id = ((int64_t)k * p.ny + (j - 1)) * p.nx + (i - 1);
                if (p.dim == 2)
                    T[id] = (double)(i - 1) / (double)(p.nx - 1) * (p.Tcold - p.Thot) + p.Thot;
                else
                    T[id] = (double)(j - 1) / (double)(p.ny - 1) * (p.Tcold - p.Thot) + p.Thot;
            }
    int st = upload_macro(h, rho.data(), zero.data(), zero.data(), zero.data(), T.data());
    if (st) return st;
    CU(launch_equilibrium(h, h->bufs.pop[h->cur]));
    if ((st = reset_run(h))) return st;
    CU(cudaStreamSynchronize(h->stream));
    h->phase = 1;
    return LBM_OK;
}

extern "C" int lbm_init_equilibrium(lbm_handle *h, const double *rho, const double *u, const double *v,
                                    const double *w, const double *T)
{
    CHECK_H(h);
    if (!rho || !u || !v || !T) return fail(LBM_ERR_PARAM, "rho, u, v and T are required");
    const int64_t N = h->geo.nnode;
    std::vector<double> zero;
    if (h->p.dim == 3 && !w) {
        zero.assign((size_t)N, 0.0);
        w = zero.data();
    }
    int st = upload_macro(h, rho, u, v, w, T);
    if (st) return st;
    CU(launch_equilibrium(h, h->bufs.pop[h->cur]));
    if ((st = reset_run(h))) return st;
    CU(cudaStreamSynchronize(h->stream));
    h->phase = 1;
    return LBM_OK;
}

extern "C" int lbm_init_warm(lbm_handle *h, const double *rho, const double *u, const double *v, const double *w,
                             const double *T)
{
    CHECK_H(h);
    if (!rho || !u || !v || !T) return fail(LBM_ERR_PARAM, "rho, u, v and T are required");
    const int64_t N = h->geo.nnode;
    for (int64_t n = 0; n < N; ++n)
        if (!std::isfinite(rho[n]) || !std::isfinite(u[n]) || !std::isfinite(v[n]) || !std::isfinite(T[n]) ||
            (w && h->p.dim == 3 && !std::isfinite(w[n])))
            return fail(LBM_ERR_NONFINITE, "lbm_init_warm: non-finite field value at node %lld", (long long)n);
    std::vector<double> zero;
    if (h->p.dim == 3 && !w) {
        zero.assign((size_t)N, 0.0);
        w = zero.data();
    }
    int st = upload_macro(h, rho, u, v, w, T);
    if (st) return st;
    CU(launch_equilibrium(h, h->bufs.pop[h->cur], 1));
    if ((st = reset_run(h))) return st;
    CU(cudaStreamSynchronize(h->stream));
    h->phase = 1;
    return LBM_OK;
}

int lbm::first_collision(lbm_handle *h)
{
    if (h->phase != 1) return LBM_OK;
    // first collision of the run, from the pre-collision state
    const bool ex = h->p.mode == LBM_MODE_EXACT;
    Bufs &b = h->bufs;
    const int nxt = 1 - h->cur;
    CU(ex ? exact::collide(h->geo, h->p.storage, b.pop[h->cur], b.pop[nxt], b.F[nxt], b, h->stream)
          : fast::collide(h->geo, h->p.storage, b.pop[h->cur], b.pop[nxt], b.F[nxt], b, h->stream));
    h->cur = nxt;
    h->phase = 2;
    return LBM_OK;
}

// one fused step from buffer `cur` (asynchronous)
static cudaError_t launch_one(lbm_handle *h, int cur, int wm)
{
    const bool ex = h->p.mode == LBM_MODE_EXACT;
    Bufs &b = h->bufs;
    const int nxt = 1 - cur;
    if (h->use_march)
        return ex ? exact::march(h->geo, h->p.storage, h->tmaps[cur], b.F[cur], b.pop[nxt], b.F[nxt], b, wm,
                                 h->nblocks, h->tiley, h->d_msegs, h->d_msegoff, h->pdl != 0, h->stream)
                  : fast::march(h->geo, h->p.storage, h->tmaps[cur], b.F[cur], b.pop[nxt], b.F[nxt], b, wm,
                                h->nblocks, h->tiley, h->d_msegs, h->d_msegoff, h->pdl != 0, h->stream);
    return ex ? exact::step(h->geo, h->p.storage, b.pop[cur], b.F[cur], b.pop[nxt], b.F[nxt], b, wm, h->stream)
              : fast::step(h->geo, h->p.storage, b.pop[cur], b.F[cur], b.pop[nxt], b.F[nxt], b, wm, h->stream);
}

void lbm::drop_graphs(lbm_handle *h)
{
    for (auto &g : h->graph)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
    for (auto &g : h->run_graph)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
}

// steps per replayed graph in lbm_step (even: a replay leaves `cur` as it was);
// inside a graph consecutive march steps are programmatic dependents
static constexpr int kGraphSteps = 8;

// a kGraphSteps-step graph starting from buffer `cur`, captured once per kernel choice
static int step_graph(lbm_handle *h, int cur, cudaGraphExec_t *out)
{
    if (!h->graph[cur]) {
        cudaGraph_t g = nullptr;
        CU(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t e1 = cudaSuccess;
        for (int k = 0; k < kGraphSteps && e1 == cudaSuccess; ++k) e1 = launch_one(h, (cur + k) & 1, 0);
        const cudaError_t e3 = cudaStreamEndCapture(h->stream, &g);
        lbm::g_launches -= kGraphSteps;  // counted when replayed
        if (e1 != cudaSuccess || e3 != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return fail(LBM_ERR_CUDA, "step graph capture: %s", cudaGetErrorString(e1 != cudaSuccess ? e1 : e3));
        }
        const cudaError_t e = cudaGraphInstantiate(&h->graph[cur], g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return fail(LBM_ERR_CUDA, "step graph instantiate: %s", cudaGetErrorString(e));
    }
    *out = h->graph[cur];
    return LBM_OK;
}

extern "C" int lbm_step(lbm_handle *h, int32_t nsteps)
{
    CHECK_H(h);
    if (nsteps < 0) return fail(LBM_ERR_PARAM, "nsteps < 0");
    if (h->phase == 0) return fail(LBM_ERR_STATE, "lbm_step before an init call");
    if (nsteps == 0) return LBM_OK;
    int st = lbm::first_collision(h);
    if (st) return st;
    int done = 0;
    if (h->resident && nsteps > 4) {
        const bool ex = h->p.mode == LBM_MODE_EXACT;
        CU(cudaMemsetAsync(h->d_bar, 0, 2 * sizeof(unsigned), h->stream));
        CU(ex ? exact::steps_resident(h->geo, h->p.storage, h->bufs.pop, h->bufs.F, h->bufs, h->cur, nsteps, h->d_bar,
                                      h->bufs.err, h->resident, h->stream)
              : fast::steps_resident(h->geo, h->p.storage, h->bufs.pop, h->bufs.F, h->bufs, h->cur, nsteps, h->d_bar,
                                     h->bufs.err, h->resident, h->stream));
        h->cur = (h->cur + nsteps) & 1;
        h->itc += nsteps;
        return LBM_OK;
    }
    // replay kGraphSteps-step graphs for all but the last step(s) (small
    // domains are launch-bound), then single launches; the last step writes
    // the macroscopic fields
    if (h->use_graphs) {
        while (nsteps - done > kGraphSteps) {
            cudaGraphExec_t g;
            if ((st = step_graph(h, h->cur, &g))) return st;
            CU(cudaGraphLaunch(g, h->stream));
            lbm::g_launches += kGraphSteps;
            done += kGraphSteps;
        }
    }
    for (; done < nsteps; ++done) {
        CU(launch_one(h, h->cur, done == nsteps - 1));
        h->cur = 1 - h->cur;
    }
    h->itc += nsteps;
    return LBM_OK;
}

// ---------------------------------------------------------------------------
// runs to the reference's stop criterion with the test on the device
// ---------------------------------------------------------------------------
// The reference's loop (2M:307-330) iterates while errorU > eps or errorT > eps,
// calling check() every check_every iterations.  Here each check period (its
// steps, the check sums and the stop test) is queued without waiting for the
// previous one: the test runs on the device (run_check) and, once it fires,
// clears RunCtl::active, which turns the step and check kernels queued after it
// into no-ops.  The host reads the run state once every kRunPeriodsPerRead
// periods, so a run syncs once per that many checks instead of once per check.
static constexpr int kRunPeriodsPerRead = 4;

static int sync_and_check(lbm_handle *h);

int lbm::run_begin(lbm_handle *h, double eps, double growth, int stop_bad)
{
    RunCtl c{};
    c.active = 1;
    c.errU = c.errT = 100.0;
    c.best = INFINITY;
    c.eps = eps;
    c.growth = growth;
    c.stop_bad = stop_bad;
    CU(cudaMemcpyAsync(h->bufs.ctl, &c, sizeof c, cudaMemcpyHostToDevice, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    return LBM_OK;
}

int lbm::run_read(lbm_handle *h, RunCtl *out)
{
    CU(cudaMemcpyAsync(out, h->bufs.ctl, sizeof *out, cudaMemcpyDeviceToHost, h->stream));
    return sync_and_check(h);
}

int lbm::run_end(lbm_handle *h)
{
    static const int one = 1;
    CU(cudaMemcpyAsync(&h->bufs.ctl->active, &one, sizeof one, cudaMemcpyHostToDevice, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    return LBM_OK;
}

// one check period of `period` iterations from buffer `cur` as a graph
// (steps, the last writing the macroscopic fields, then the device check)
static int period_graph(lbm_handle *h, int cur, int period, cudaGraphExec_t *out)
{
    if (h->run_graph_period != period) {
        for (auto &g : h->run_graph)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
        h->run_graph_period = period;
    }
    if (!h->run_graph[cur]) {
        cudaGraph_t g = nullptr;
        CU(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = cudaSuccess;
        for (int i = 0; i < period && e == cudaSuccess; ++i) e = launch_one(h, (cur + i) & 1, i == period - 1);
        if (e == cudaSuccess) e = run_check(h->geo, h->bufs, period, h->stream);
        const cudaError_t e2 = cudaStreamEndCapture(h->stream, &g);
        lbm::g_launches -= period + 2;  // counted when replayed
        if (e != cudaSuccess || e2 != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return fail(LBM_ERR_CUDA, "check-period graph capture: %s", cudaGetErrorString(e != cudaSuccess ? e : e2));
        }
        e = cudaGraphInstantiate(&h->run_graph[cur], g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return fail(LBM_ERR_CUDA, "check-period graph instantiate: %s", cudaGetErrorString(e));
    }
    *out = h->run_graph[cur];
    return LBM_OK;
}

extern "C" int lbm_run(lbm_handle *h, int64_t max_steps, int32_t check_every, double eps, int64_t *steps_done,
                       double *errU, double *errT)
{
    CHECK_H(h);
    if (max_steps < 0 || check_every < 1) return fail(LBM_ERR_PARAM, "need max_steps >= 0 and check_every >= 1");
    if (h->phase == 0) return fail(LBM_ERR_STATE, "lbm_run before an init call");
    int st = lbm::first_collision(h);
    if (st) return st;
    if ((st = lbm::run_begin(h, eps, 0.0, 0))) return st;
    const int64_t itc0 = h->itc;
    const int cur0 = h->cur;
    int64_t launched = 0;
    int periods = 0;
    RunCtl c{};
    c.active = 1;
    c.errU = c.errT = 100.0;
    while (launched < max_steps) {
        const int64_t to_check = check_every - (h->itc % check_every);
        const int64_t k = std::min<int64_t>(to_check, max_steps - launched);
        if (k == to_check && k == check_every && h->use_graphs && !h->resident && k >= 2) {
            cudaGraphExec_t g;
            if ((st = period_graph(h, h->cur, (int)k, &g))) break;
            cudaError_t e = cudaGraphLaunch(g, h->stream);
            if (e != cudaSuccess) {
                st = fail(LBM_ERR_CUDA, "cudaGraphLaunch: %s", cudaGetErrorString(e));
                break;
            }
            lbm::g_launches += k + 2;
            h->cur = (int)((h->cur + k) & 1);
            h->itc += k;
        } else {
            if ((st = lbm_step(h, (int32_t)k))) break;
            if (k == to_check) {
                cudaError_t e = run_check(h->geo, h->bufs, (int)k, h->stream);
                if (e != cudaSuccess) {
                    st = fail(LBM_ERR_CUDA, "run check: %s", cudaGetErrorString(e));
                    break;
                }
            }
        }
        launched += k;
        if (k == to_check && ++periods % kRunPeriodsPerRead == 0) {
            if ((st = lbm::run_read(h, &c))) break;
            if (!c.active) break;
        }
    }
    int st2 = lbm::run_read(h, &c);
    if (!st) st = st2;
    // iterations that ran: up to the stopping check, or all that were queued
    const int64_t ran = c.active ? launched : c.steps;
    h->itc = itc0 + ran;
    h->cur = (int)((cur0 + ran) & 1);
    st2 = lbm::run_end(h);
    if (!st) st = st2;
    if (steps_done) *steps_done = ran;
    if (errU) *errU = c.errU;
    if (errT) *errT = c.errT;
    if (!st && c.status == -2) st = fail(LBM_ERR_NONFINITE, "check: non-finite residual sum");
    return st;
}

extern "C" int lbm_itc(const lbm_handle *h, int64_t *itc)
{
    if (!h || !itc) return fail(LBM_ERR_PARAM, "NULL argument");
    *itc = h->itc;
    return LBM_OK;
}

// Synchronise the handle's stream and report a kernel's bounded wait that gave up.
static int sync_and_check(lbm_handle *h)
{
    int flag = 0;
    CU(cudaMemcpyAsync(&flag, h->bufs.err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    if (flag) {
        CU(cudaMemsetAsync(h->bufs.err, 0, sizeof(int), h->stream));
        CU(cudaStreamSynchronize(h->stream));
        return fail(LBM_ERR_TIMEOUT, "a step kernel's bounded wait for its TMA copies gave up (code %d)", flag);
    }
    return LBM_OK;
}

int lbm::sync_handle(lbm_handle *h) { return sync_and_check(h); }

static int read_scal(lbm_handle *h, int first, int count, double *out)
{
    CU(cudaMemcpyAsync(out, h->bufs.scal + first, sizeof(double) * count, cudaMemcpyDeviceToHost, h->stream));
    return sync_and_check(h);
}

extern "C" int lbm_check(lbm_handle *h, double *errU, double *errT)
{
    CHECK_H(h);
    if (h->phase == 0) return fail(LBM_ERR_STATE, "lbm_check before an init call");
    CU(reduce_check(h->geo, h->bufs, h->stream));
    double s[4];
    int st = read_scal(h, 0, 4, s);
    if (st) return st;
    // errorU = sqrt(error1_all)/sqrt(error2_all) (2M:784), errorT likewise (2M:798)
    if (errU) *errU = sqrt(s[0]) / sqrt(s[1]);
    if (errT) *errT = sqrt(s[2]) / sqrt(s[3]);
    for (double v : s)
        if (!isfinite(v)) return fail(LBM_ERR_NONFINITE, "check: non-finite residual sum");
    return LBM_OK;
}

extern "C" int lbm_nusselt(lbm_handle *h, double *nu_hot, double *nu_cold)
{
    CHECK_H(h);
    if (h->phase == 0) return fail(LBM_ERR_STATE, "lbm_nusselt before an init call");
    CU(reduce_nusselt(h->geo, h->bufs, h->stream));
    double s[3];
    int st = read_scal(h, 4, 3, s);
    if (st) return st;
    if (nu_hot) *nu_hot = s[0] / s[2];
    if (nu_cold) *nu_cold = s[1] / s[2];
    if (!isfinite(s[0]) || !isfinite(s[1])) return fail(LBM_ERR_NONFINITE, "nusselt: non-finite");
    return LBM_OK;
}

// ---------------------------------------------------------------------------
// slabs: one domain split along its slowest axis (y in 2D, z in 3D) over
// several handles: the reference's slab decomposition with its per-step ghost
// exchange, `update` (2M:572-589 rows, 3M:732-749 z-planes)
// ---------------------------------------------------------------------------
extern "C" int lbm_create_slab(const lbm_params *p, const double *x, const double *y, const double *z, int32_t lo,
                               int32_t hi, lbm_handle **out)
{
    if (!out) return fail(LBM_ERR_PARAM, "out is NULL");
    *out = nullptr;
    if (!p) return fail(LBM_ERR_PARAM, "params NULL");
    int st = validate(p);
    if (st) return st;
    if (!x || !y || (p->dim == 3 && !z)) return fail(LBM_ERR_PARAM, "coordinates missing");
    const int n = p->dim == 2 ? p->ny : p->nz;  // the split axis
    if (lo < 0 || hi > n || hi - lo < 2) return fail(LBM_ERR_PARAM, "slab layers [%d, %d) of %d", lo, hi, n);
    // the slab's buffer: its layers plus one ghost layer on each side that has a neighbour
    const int b0 = lo > 0 ? lo - 1 : 0, b1 = hi < n ? hi + 1 : n;
    lbm_params q = *p;
    if (p->dim == 2) q.ny = b1 - b0;
    else q.nz = b1 - b0;
    st = p->dim == 2 ? lbm_create(&q, x, y + b0, nullptr, out) : lbm_create(&q, x, y, z + b0, out);
    if (st) return st;
    lbm_handle *h = *out;
    if (p->dim == 2) {
        h->geo.jlo = lo - b0;
        h->geo.jhi = hi - b0;
    } else {
        h->geo.klo = lo - b0;
        h->geo.khi = hi - b0;
    }
    st = resolve_path(h);
    if (st) {
        lbm_destroy(h);
        *out = nullptr;
    }
    return st;
}

// One layer of the newest state in every population plane: a row (2D) or a
// z-slice of pitch x ny elements, padding columns included (3D).
static size_t halo_layer(const Geo &g) { return g.dim == 2 ? (size_t)g.nx : (size_t)g.slab; }

extern "C" int lbm_halo_size(const lbm_handle *h, int64_t *bytes)
{
    CHECK_H(h);
    if (!bytes) return fail(LBM_ERR_PARAM, "bytes NULL");
    *bytes = (int64_t)((size_t)(h->Q + h->QT) * halo_layer(h->geo) * (size_t)h->esize);
    return LBM_OK;
}

// layer `r` (local) of every population plane of the newest state <-> a packed
// device buffer [Q + QT][layer] of the storage type, on the handle's stream
static int halo_copy(lbm_handle *h, int32_t side, void *buf, bool pack)
{
    CHECK_H(h);
    if (side != 0 && side != 1) return fail(LBM_ERR_PARAM, "side must be 0 (low end) or 1 (high end)");
    if (!buf) return fail(LBM_ERR_PARAM, "buffer NULL");
    if (h->phase == 0) return fail(LBM_ERR_STATE, "halo exchange before an init call");
    const Geo &g = h->geo;
    const bool d2 = g.dim == 2;
    const int lo = d2 ? g.jlo : g.klo, hi = d2 ? g.jhi : g.khi, n = d2 ? g.ny : g.nz;
    if (side == 0 ? lo == 0 : hi == n) return fail(LBM_ERR_PARAM, "no neighbour on side %d (a wall)", side);
    // pack: the slab's first / last own layer; unpack: the ghost layer below / above it
    const int r = pack ? (side == 0 ? lo : hi - 1) : (side == 0 ? lo - 1 : hi);
    const size_t es = (size_t)h->esize, w = halo_layer(g) * es;
    unsigned char *pop = (unsigned char *)h->bufs.pop[h->cur] + (size_t)r * (size_t)(d2 ? g.pitch : g.slab) * es;
    const size_t planes = (size_t)(h->Q + h->QT), pstride = (size_t)g.plane * es;
    CU(pack ? cudaMemcpy2DAsync(buf, w, pop, pstride, w, planes, cudaMemcpyDeviceToDevice, h->stream)
            : cudaMemcpy2DAsync(pop, pstride, buf, w, w, planes, cudaMemcpyDeviceToDevice, h->stream));
    return LBM_OK;
}

extern "C" int lbm_halo_pack(lbm_handle *h, int32_t side, void *dev_buf) { return halo_copy(h, side, dev_buf, true); }

extern "C" int lbm_halo_unpack(lbm_handle *h, int32_t side, const void *dev_buf)
{
    return halo_copy(h, side, const_cast<void *>(dev_buf), false);
}

extern "C" int lbm_check_sums(lbm_handle *h, double sums[4])
{
    CHECK_H(h);
    if (!sums) return fail(LBM_ERR_PARAM, "sums NULL");
    if (h->phase == 0) return fail(LBM_ERR_STATE, "lbm_check_sums before an init call");
    CU(reduce_check(h->geo, h->bufs, h->stream));
    return read_scal(h, 0, 4, sums);
}

extern "C" int lbm_nusselt_sums(lbm_handle *h, double sums[3])
{
    CHECK_H(h);
    if (!sums) return fail(LBM_ERR_PARAM, "sums NULL");
    if (h->phase == 0) return fail(LBM_ERR_STATE, "lbm_nusselt_sums before an init call");
    CU(reduce_nusselt(h->geo, h->bufs, h->stream));
    return read_scal(h, 4, 3, sums);
}

extern "C" int lbm_sums(lbm_handle *h, double *mass, double *energy)
{
    CHECK_H(h);
    if (h->phase == 0) return fail(LBM_ERR_STATE, "lbm_sums before an init call");
    CU(reduce_sums(h->geo, h->bufs, h->stream));
    double s[2];
    int st = read_scal(h, 7, 2, s);
    if (st) return st;
    if (mass) *mass = s[0];
    if (energy) *energy = s[1];
    if (!isfinite(s[0]) || !isfinite(s[1])) return fail(LBM_ERR_NONFINITE, "sums: non-finite");
    return LBM_OK;
}

extern "C" int lbm_get_macro(lbm_handle *h, double *rho, double *u, double *v, double *w, double *T)
{
    CHECK_H(h);
    if (h->phase == 0) return fail(LBM_ERR_STATE, "lbm_get_macro before an init call");
    const size_t mb = (size_t)h->geo.nnode * 8;
    if (rho) CU(cudaMemcpyAsync(rho, h->bufs.rho, mb, cudaMemcpyDeviceToHost, h->stream));
    if (u) CU(cudaMemcpyAsync(u, h->bufs.u, mb, cudaMemcpyDeviceToHost, h->stream));
    if (v) CU(cudaMemcpyAsync(v, h->bufs.v, mb, cudaMemcpyDeviceToHost, h->stream));
    if (w && h->p.dim == 3) CU(cudaMemcpyAsync(w, h->bufs.w, mb, cudaMemcpyDeviceToHost, h->stream));
    if (T) CU(cudaMemcpyAsync(T, h->bufs.T, mb, cudaMemcpyDeviceToHost, h->stream));
    return sync_and_check(h);
}

extern "C" int lbm_set_macro(lbm_handle *h, const double *rho, const double *u, const double *v, const double *w,
                             const double *T)
{
    CHECK_H(h);
    if (h->phase == 0) return fail(LBM_ERR_STATE, "lbm_set_macro before an init call");
    if (h->phase == 2)
        return fail(LBM_ERR_STATE, "lbm_set_macro after lbm_step: load populations first (lbm_set_populations)");
    int st = upload_macro(h, rho, u, v, w, T);
    if (st) return st;
    CU(cudaStreamSynchronize(h->stream));
    return LBM_OK;
}

static int ensure_staging(lbm_handle *h)
{
    if (!h->staging) {
        int st = dalloc(h, &h->staging, (size_t)(h->Q + h->QT) * (size_t)h->geo.plane * h->esize);
        if (st) return st;
    }
    if (!h->aos) {
        int st = dalloc(h, &h->aos, (size_t)h->geo.nnode * h->Q * 8);
        if (st) return st;
    }
    return LBM_OK;
}

extern "C" int lbm_get_populations(lbm_handle *h, double *f, double *g)
{
    CHECK_H(h);
    if (h->phase == 0) return fail(LBM_ERR_STATE, "lbm_get_populations before an init call");
    int st = ensure_staging(h);
    if (st) return st;
    const void *src = h->bufs.pop[h->cur];
    if (h->phase == 2) {
        // the newest buffer is one collision ahead; stream the previous one
        const int prv = 1 - h->cur;
        Bufs b = h->bufs;
        CU(h->p.mode == LBM_MODE_EXACT
               ? exact::stream_only(h->geo, h->p.storage, b.pop[prv], b.F[prv], h->staging, b, h->stream)
               : fast::stream_only(h->geo, h->p.storage, b.pop[prv], b.F[prv], h->staging, b, h->stream));
        src = h->staging;
    }
    const int64_t N = h->geo.nnode;
    if (f) {
        CU(planes_to_aos(h->geo, h->p.storage, 0, h->Q, src, h->aos, h->stream));
        CU(cudaMemcpyAsync(f, h->aos, (size_t)N * h->Q * 8, cudaMemcpyDeviceToHost, h->stream));
        CU(cudaStreamSynchronize(h->stream));
    }
    if (g) {
        CU(planes_to_aos(h->geo, h->p.storage, h->Q, h->QT, src, h->aos, h->stream));
        CU(cudaMemcpyAsync(g, h->aos, (size_t)N * h->QT * 8, cudaMemcpyDeviceToHost, h->stream));
        CU(cudaStreamSynchronize(h->stream));
    }
    return LBM_OK;
}

extern "C" int lbm_set_populations(lbm_handle *h, const double *f, const double *g)
{
    CHECK_H(h);
    if (!f || !g) return fail(LBM_ERR_PARAM, "f and g are required");
    if (h->phase == 0) return fail(LBM_ERR_STATE, "lbm_set_populations before an init call");
    int st = ensure_staging(h);
    if (st) return st;
    const int64_t N = h->geo.nnode;
    void *dst = h->bufs.pop[h->cur];
    CU(cudaMemcpyAsync(h->aos, f, (size_t)N * h->Q * 8, cudaMemcpyHostToDevice, h->stream));
    CU(aos_to_planes(h->geo, h->p.storage, 0, h->Q, h->aos, dst, h->stream));
    CU(cudaMemcpyAsync(h->aos, g, (size_t)N * h->QT * 8, cudaMemcpyHostToDevice, h->stream));
    CU(aos_to_planes(h->geo, h->p.storage, h->Q, h->QT, h->aos, dst, h->stream));
    CU(macro_from_pops(h->geo, h->p.storage, dst, h->bufs, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    h->phase = 1;
    return LBM_OK;
}

// Convert the cavity's state to another population storage in place: new
// buffers, the newest populations and carried force converted on the device,
// old buffers released, descriptors and kernel choice redone.
int lbm::change_storage(lbm_handle *h, int storage, int target)
{
    if (storage == h->p.storage && (target < 0 || target == h->cur)) return LBM_OK;
    if (storage == LBM_STORE_F16S)
        return fail(LBM_ERR_UNSUPPORTED, "binary16 population storage is retired (inaccurate, not faster than FP32)");
    if (storage != LBM_STORE_F64 && storage != LBM_STORE_F32) return fail(LBM_ERR_PARAM, "unknown storage %d", storage);
    if (h->p.mode == LBM_MODE_EXACT && storage != LBM_STORE_F64)
        return fail(LBM_ERR_UNSUPPORTED, "exact mode computes in FP64 storage only");
    CU(cudaStreamSynchronize(h->stream));
    const size_t es = storage == LBM_STORE_F64 ? 8 : 4;
    const size_t cs = storage == LBM_STORE_F64 ? 8 : 4;
    const size_t popb = (size_t)(h->Q + h->QT) * (size_t)h->geo.plane * es;
    const size_t fb = (size_t)h->geo.plane * cs;
    void *np[2] = {nullptr, nullptr}, *nF[2] = {nullptr, nullptr};
    int st = LBM_OK;
    for (int i = 0; i < 2 && !st; ++i) {
        st = dalloc(h, &np[i], popb);
        if (!st) st = dalloc(h, &nF[i], fb);
    }
    if (!st && h->phase == 0 &&
        (cudaMemset(nF[0], 0, fb) != cudaSuccess || cudaMemset(nF[1], 0, fb) != cudaSuccess ||
         cudaMemset(np[0], 0, popb) != cudaSuccess || cudaMemset(np[1], 0, popb) != cudaSuccess))
        st = fail(LBM_ERR_CUDA, "memset failed");
    if (!st && h->phase != 0) {
        // both buffers: the newest state, and the one before it (lbm_get_populations
        // streams that one to give the reference's pre-collision populations)
        const int c = h->cur, t = target < 0 ? c : target;
        cudaError_t e = convert_state(h->geo, h->p.storage, storage, h->Q + h->QT, h->bufs.pop[c], np[t],
                                      h->bufs.F[c], nF[t], h->stream);
        if (e == cudaSuccess)
            e = convert_state(h->geo, h->p.storage, storage, h->Q + h->QT, h->bufs.pop[1 - c], np[1 - t],
                              h->bufs.F[1 - c], nF[1 - t], h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) st = fail(LBM_ERR_CUDA, "storage conversion: %s", cudaGetErrorString(e));
    }
    if (st) {
        for (int i = 0; i < 2; ++i) {
            if (np[i]) cudaFree(np[i]);
            if (nF[i]) cudaFree(nF[i]);
        }
        return st;
    }
    const size_t old_popb = (size_t)(h->Q + h->QT) * (size_t)h->geo.plane * h->esize;
    const size_t old_fb = (size_t)h->geo.plane * h->csize;
    for (int i = 0; i < 2; ++i) {
        cudaFree(h->bufs.pop[i]);
        cudaFree(h->bufs.F[i]);
        h->bufs.pop[i] = np[i];
        h->bufs.F[i] = nF[i];
    }
    h->bytes -= (int64_t)(2 * (old_popb + old_fb));
    if (h->staging) {  // sized for the old storage; ensure_staging makes a new one
        cudaFree(h->staging);
        h->staging = nullptr;
        h->bytes -= (int64_t)old_popb;
    }
    h->p.storage = storage;
    h->esize = es;
    h->csize = cs;
    if (target >= 0) h->cur = target;
    lbm::drop_graphs(h);
    h->march_ok = encode_maps(h);
    return resolve_path(h);
}

extern "C" int lbm_set_storage(lbm_handle *h, int32_t storage)
{
    CHECK_H(h);
    if (!h->owns_ctl) return fail(LBM_ERR_STATE, "a batch member changes storage with lbm_batch_set_storage");
    return lbm::change_storage(h, storage);
}

extern "C" int lbm_synchronize(lbm_handle *h)
{
    CHECK_H(h);
    return sync_and_check(h);
}

extern "C" int lbm_set_option(lbm_handle *h, int32_t option, int64_t value)
{
    CHECK_H(h);
    switch (option) {
    case LBM_OPT_KERNEL: {
        if (value < 0 || value > 2) return fail(LBM_ERR_PARAM, "kernel option must be 0, 1 or 2");
        const int old = h->kernel_opt;
        h->kernel_opt = (int)value;
        int st = resolve_path(h);
        if (st) {
            h->kernel_opt = old;
            resolve_path(h);
            return st;
        }
        return LBM_OK;
    }
    case LBM_OPT_NBLOCKS:
        if (value < 0 || value > (1 << 20)) return fail(LBM_ERR_PARAM, "nblocks out of range");
        h->nblocks_opt = (int)value;
        return resolve_path(h);
    case LBM_OPT_GRAPHS:
        lbm::drop_graphs(h);
        h->use_graphs = value != 0;
        return LBM_OK;
    case LBM_OPT_RESIDENT:
        h->resident_opt = value != 0;
        return resolve_path(h);
    case LBM_OPT_L2PROMO:
        if (value < 0 || value > 3) return fail(LBM_ERR_PARAM, "L2 promotion must be 0..3");
        CU(cudaStreamSynchronize(h->stream));
        h->l2promo = (int)value;
        h->march_ok = encode_maps(h);
        return resolve_path(h);
    case LBM_OPT_TILEY:
        if (value != 0 && value != 4 && value != 8) return fail(LBM_ERR_PARAM, "tile rows must be 0, 4 or 8");
        CU(cudaStreamSynchronize(h->stream));
        h->tiley_opt = (int)value;
        h->tiley = value ? (int)value : kDefaultTileY;
        h->march_ok = encode_maps(h);
        return resolve_path(h);
    case LBM_OPT_PLAN:
        if (value != 0 && value != 1) return fail(LBM_ERR_PARAM, "plan must be 0 or 1");
        CU(cudaStreamSynchronize(h->stream));
        h->plan_opt = (int)value;
        return resolve_path(h);
    case LBM_OPT_WAIT_LIMIT:
        if (value < 0) return fail(LBM_ERR_PARAM, "wait limit must be >= 0");
        CU(cudaStreamSynchronize(h->stream));
        CU(fast::set_wait_limit(value));
        CU(exact::set_wait_limit(value));
        h->wait_limit = value;
        return LBM_OK;
    case LBM_OPT_PDL:
        if (value != 0 && value != 1) return fail(LBM_ERR_PARAM, "PDL must be 0 or 1");
        CU(cudaStreamSynchronize(h->stream));
        lbm::drop_graphs(h);
        h->pdl = (int)value;
        return LBM_OK;
    default:
        return fail(LBM_ERR_PARAM, "unknown option %d", option);
    }
}

extern "C" int lbm_get_option(const lbm_handle *h, int32_t option, int64_t *value)
{
    if (!h || !value) return fail(LBM_ERR_PARAM, "NULL argument");
    switch (option) {
    case LBM_OPT_KERNEL: *value = h->use_march ? 2 : 1; return LBM_OK;
    case LBM_OPT_NBLOCKS: *value = h->use_march ? h->nblocks : 0; return LBM_OK;
    case LBM_OPT_L2PROMO: *value = h->l2promo; return LBM_OK;
    case LBM_OPT_GRAPHS: *value = h->use_graphs; return LBM_OK;
    case LBM_OPT_RESIDENT: *value = h->resident > 0; return LBM_OK;
    case LBM_OPT_TILEY: *value = h->geo.dim == 3 ? h->tiley : 0; return LBM_OK;
    case LBM_OPT_PLAN: *value = h->plan_opt; return LBM_OK;
    case LBM_OPT_WAIT_LIMIT: *value = h->wait_limit; return LBM_OK;
    case LBM_OPT_PDL: *value = h->pdl; return LBM_OK;
    default: return fail(LBM_ERR_PARAM, "unknown option %d", option);
    }
}

extern "C" int lbm_stream(const lbm_handle *h, void **stream)
{
    if (!h || !stream) return fail(LBM_ERR_PARAM, "NULL argument");
    *stream = (void *)h->stream;
    return LBM_OK;
}

extern "C" int lbm_device_bytes(const lbm_handle *h, int64_t *bytes)
{
    if (!h || !bytes) return fail(LBM_ERR_PARAM, "NULL argument");
    *bytes = h->bytes;
    return LBM_OK;
}
