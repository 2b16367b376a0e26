// TMA-fed persistent "march" kernels for the fused time step.
//
// Included by lbm_kernels.cu inside namespace lbm::LBM_NS, so the arithmetic
// (ip, collide2d / collide3d, DV) is the same code as the direct-load kernels
// and is compiled in both the fast and the exact mode.
//
// Scheme (3D; 2D is the same one dimension down):
//   * the domain is cut into cross-section tiles of TX x TY nodes (x, y); a
//     work item is a tile at one z-slice.  In 3D each persistent CTA runs a
//     host-made list of segments (tile, first slice, end slice) and marches
//     along z through each; the host plans the lists so that neighbouring
//     tiles are at the same slice at the same time (their shared halo rows
//     then come from L2) while every SM has an equal share; in 2D each CTA
//     takes a contiguous, equal share of the (strip-major, row-minor) items;
//   * for every slice the CTA fetches one TMA box per population plane into
//     shared memory: a box covers the tile plus the in-plane halo the plane's
//     interpolation stencil needs (x +-HX columns, y +-1 rows);
//   * planes whose stencil reaches along z (D3Q19 5,6,11-18; D3Q7 5,6) live in
//     a 4-slot ring indexed by slice, fetched two slices ahead, so each slice
//     is read once per tile column and serves the steps k-1, k, k+1 (and the
//     one-sided stencils at the walls); the other planes use a 2-slot ring;
//   * one thread issues the copies (cp.async.bulk.tensor with an mbarrier
//     transaction count), every thread waits on the slot barriers it needs,
//     computes its node from shared memory and stores the new post-collision
//     populations straight to global memory; a __syncthreads ends each step
//     and frees the slots the next copies reuse;
//   * every wait is bounded: a step's waits by g_wait_limit (kWaitCycles
//     unless LBM_OPT_WAIT_LIMIT sets it), the final drain by kWaitCycles.  On
//     timeout the kernel records an error code in *err, stops issuing, lets
//     outstanding copies drain and returns; the host reports LBM_ERR_TIMEOUT.
// No copy uses cluster multicast; every copy reads this GPU's own buffers.

static constexpr long long kWaitCycles = 4000000000LL;  // ~2 s at 1.9 GHz

// limit of a step's waits, in clock cycles (set_wait_limit)
__device__ long long g_wait_limit = kWaitCycles;

__device__ __forceinline__ uint32_t saddr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *b, uint32_t n)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(b)), "r"(n) : "memory");
}

__device__ __forceinline__ void mbar_arrive_tx(uint64_t *b, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(b)), "r"(bytes) : "memory");
}

__device__ __forceinline__ uint32_t mbar_test(uint64_t *b, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(saddr(b)), "r"(parity)
        : "memory");
    return ok;
}

// non-blocking test of the phase of parity `parity` (try_wait may suspend
// the thread for a while before it reports an incomplete phase)
__device__ __forceinline__ uint32_t mbar_probe(uint64_t *b, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(saddr(b)), "r"(parity)
        : "memory");
    return ok;
}

// limits below this poll with mbar_probe, so that they can run out before a
// copy in flight lands (the error path's tests)
static constexpr long long kShortWait = 1000000LL;

// bounded wait for the phase of parity `parity`; false after `limit` cycles
__device__ __forceinline__ bool mbar_wait(uint64_t *b, uint32_t parity, long long limit = kWaitCycles)
{
    if (limit < kShortWait) {
        const long long t0 = clock64();
        while (!mbar_probe(b, parity))
            if (clock64() - t0 > limit) return false;
        return true;
    }
    if (mbar_test(b, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_test(b, parity))
        if (clock64() - t0 > limit) return false;
    return true;
}

__device__ __forceinline__ void tma_load4(void *dst, const CUtensorMap *m, uint64_t *bar, int c0, int c1, int c2,
                                          int c3)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(saddr(dst)),
        "l"(m), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(saddr(bar))
        : "memory");
}

__device__ __forceinline__ void tma_load3(void *dst, const CUtensorMap *m, uint64_t *bar, int c0, int c1, int c2)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(saddr(dst)),
        "l"(m), "r"(c0), "r"(c1), "r"(c2), "r"(saddr(bar))
        : "memory");
}

__device__ __forceinline__ void tma_load2(void *dst, const CUtensorMap *m, uint64_t *bar, int c0, int c1)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(saddr(dst)),
        "l"(m), "r"(c0), "r"(c1), "r"(saddr(bar))
        : "memory");
}

// plain bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned)
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     saddr(dst)),
                 "l"(src), "r"(bytes), "r"(saddr(bar))
                 : "memory");
}

// Programmatic dependent launch.  A march kernel launched with the
// programmatic-serialization attribute may start while the stream's previous
// kernel is still finishing: each CTA lets the next kernel's CTAs be scheduled
// as soon as it runs (dep_launch), sets up its barriers, reads its work list
// and geometry -- tables only the host writes -- and then waits (dep_wait) for
// the previous kernel to complete with its memory visible before it reads a
// run flag or a population.  Launched without the attribute, dep_wait has
// nothing to wait for.
__device__ __forceinline__ void dep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

__device__ __forceinline__ void fence_barrier_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// ---------------------------------------------------------------------------
// ring bookkeeping shared by the 2D and 3D kernels
// ---------------------------------------------------------------------------
// Slices needed at step k along a marching axis of n nodes: k-1..k+1, plus the
// far point of the one-sided stencils at the walls (k+2 at k = 0, k-2 at
// k = n-1): off_a / off_b give exactly these.
__device__ __forceinline__ int need_lo(int k, int n) { return k == n - 1 ? k - 2 : (k == 0 ? 0 : k - 1); }
__device__ __forceinline__ int need_hi(int k, int n) { return k == 0 ? 2 : (k == n - 1 ? k : k + 1); }

// ---------------------------------------------------------------------------
// 3D layout
// ---------------------------------------------------------------------------
// box classes: 0 tile only, 1 +-HX columns, 2 +-1 rows, 3 both
// Batch kernels copy the current segment's cavity geometry (Geo) into shared
// memory behind the ring barriers: the per-node arithmetic reads a dozen of its
// fields every step, and from the batch's table in global memory those reads
// miss the small L1 left beside the rings (each one an L2 round trip on the
// critical path of the step).  Single-cavity kernels take Geo as a kernel
// parameter and read it from the constant bank instead.
constexpr int kGeoStage = 256;
static_assert(sizeof(Geo) <= kGeoStage && sizeof(Geo) % 8 == 0, "staged Geo must fit its shared-memory slot");

// every thread of the CTA: copy *src into the shared slot dst (8-byte words),
// between two barriers (the slot's previous readers are done before it, the
// new readers start after it)
__device__ __forceinline__ const Geo *stage_geo(const Geo *src, Geo *dst)
{
    __syncthreads();
    const unsigned long long *s = (const unsigned long long *)src;
    unsigned long long *d = (unsigned long long *)dst;
    for (int w = threadIdx.x; w < (int)(sizeof(Geo) / 8); w += blockDim.x) d[w] = s[w];
    __syncthreads();
    return dst;
}

template <int ST, int TY_ = 8>
struct L3 {
    using S = typename Tr<ST>::S;
    using C = typename Tr<ST>::C;
    static constexpr int ES = sizeof(S);
    static constexpr int TX = 32, TY = TY_, NT = TX * TY;
    static constexpr int HX = 16 / ES;
    __host__ __device__ static constexpr int bx(int c) { return TX + ((c & 1) ? 2 * HX : 0); }
    __host__ __device__ static constexpr int by(int c) { return TY + ((c & 2) ? 2 : 0); }
    __host__ __device__ static constexpr int bytes(int c) { return bx(c) * by(c) * ES; }
    __host__ __device__ static constexpr int padded(int c) { return (bytes(c) + 127) / 128 * 128; }
    // z-ring planes: 5 6 | 11 12 13 14 | 15 16 17 18 | 24 25
    __host__ __device__ static constexpr int zq(int zi)
    {
        return zi < 2 ? 5 + zi : (zi < 10 ? 9 + zi : 14 + zi);
    }
    __host__ __device__ static constexpr int zc(int zi) { return zi < 2 ? 0 : (zi < 6 ? 1 : (zi < 10 ? 2 : 0)); }
    __host__ __device__ static constexpr int zoff(int zi)
    {
        int o = 0;
        for (int a = 0; a < zi; ++a) o += padded(zc(a));
        return o;
    }
    __host__ __device__ static constexpr int zslot() { return zoff(12); }
    __host__ __device__ static constexpr int ztx()
    {
        int b = 0;
        for (int a = 0; a < 12; ++a) b += bytes(zc(a));
        return b;
    }
    // n-ring planes: 0 | 1 2 | 3 4 | 7 8 9 10 | 19 | 20 21 | 22 23
    __host__ __device__ static constexpr int nq(int ni)
    {
        return ni < 5 ? ni : (ni < 9 ? ni + 2 : ni + 10);
    }
    __host__ __device__ static constexpr int nc(int ni)
    {
        return ni == 0 ? 0 : (ni < 3 ? 1 : (ni < 5 ? 2 : (ni < 9 ? 3 : (ni == 9 ? 0 : (ni < 12 ? 1 : 2)))));
    }
    __host__ __device__ static constexpr int noff(int ni)
    {
        int o = 0;
        for (int a = 0; a < ni; ++a) o += padded(nc(a));
        return o;
    }
    // after the planes: the carried-force box of the tile, then the slice's six
    // z-interpolation weights
    __host__ __device__ static constexpr int fbytes() { return TX * TY * (int)sizeof(C); }
    __host__ __device__ static constexpr int fo() { return noff(14); }
    __host__ __device__ static constexpr int wo() { return fo() + (fbytes() + 127) / 128 * 128; }
    __host__ __device__ static constexpr int nslot() { return wo() + 128; }
    __host__ __device__ static constexpr int ntx()
    {
        int b = 0;
        for (int a = 0; a < 14; ++a) b += bytes(nc(a));
        return b + fbytes() + 48;
    }
    // ring slots, 6 barriers and the abort flag, and slack for 128-byte alignment
    __host__ __device__ static constexpr int smem() { return 4 * zslot() + 2 * nslot() + 64 + kGeoStage + 128; }
};

// ---------------------------------------------------------------------------
// 3D march
// ---------------------------------------------------------------------------
// TY: tile rows (8: 256 threads, one CTA per SM in FP64; 4: 128 threads, two
// CTAs per SM).  A block runs segments segs[sbeg .. send), each (tile, first
// slice, end slice, cavity); tiles are numbered x-fastest within a cavity.
// `cavity(c, G, maps, dst, Fout, B)` yields cavity c's geometry, the TMA
// descriptors of the buffer read this step, the outputs and the buffers.
template <int ST, int TY_, bool kStage, class CavFn>
__device__ __forceinline__ void march3d_run(const int4 *__restrict__ segs, int sbeg, int send, CavFn cavity,
                                            int write_macro, int *err)
{
    using S = typename Tr<ST>::S;
    using C = typename Tr<ST>::C;
    using L = L3<ST, TY_>;
    constexpr int TX = L::TX, TY = L::TY, HX = L::HX;
    extern __shared__ unsigned char sm_raw[];
    unsigned char *sm = sm_raw + ((128u - (saddr(sm_raw) & 127u)) & 127u);
    uint64_t *zbar = (uint64_t *)(sm + 4 * L::zslot() + 2 * L::nslot());
    uint64_t *nbar = zbar + 4;
    volatile int &s_abort = *(volatile int *)(nbar + 2);
    Geo *sgeo = (Geo *)(sm + 4 * L::zslot() + 2 * L::nslot() + 64);

    const int tid = threadIdx.x;
    const int tx = tid % TX, ty = tid / TX;
    if (tid == 0) {
        for (int s = 0; s < 4; ++s) mbar_init(&zbar[s], 1);
        for (int s = 0; s < 2; ++s) mbar_init(&nbar[s], 1);
        fence_barrier_init();
        s_abort = 0;
    }
    dep_launch();
    __syncthreads();

    uint32_t znext = 0, nnext = 0;  // per-slot parity of the next copy
    int i0 = 0, j0 = 0;
    const Geo *Gp = nullptr;       // the current segment's cavity
    const TmapSet *Mp = nullptr;

    auto issue_z = [&](int s) {
        const int slot = s & 3;
        if (tid == 0) {
            uint64_t *bar = &zbar[slot];
            mbar_arrive_tx(bar, L::ztx());
            unsigned char *base = sm + slot * L::zslot();
#pragma unroll
            for (int zi = 0; zi < 12; ++zi) {
                const int c = L::zc(zi);
                tma_load4(base + L::zoff(zi), &Mp->m[c], bar, i0 - ((c & 1) ? HX : 0), j0 - ((c & 2) ? 1 : 0),
                          s, L::zq(zi));
            }
        }
        znext ^= 1u << slot;
    };
    auto issue_n = [&](int s) {
        const int slot = s & 1;
        if (tid == 0) {
            uint64_t *bar = &nbar[slot];
            mbar_arrive_tx(bar, L::ntx());
            unsigned char *base = sm + 4 * L::zslot() + slot * L::nslot();
#pragma unroll
            for (int ni = 0; ni < 14; ++ni) {
                const int c = L::nc(ni);
                tma_load4(base + L::noff(ni), &Mp->m[c], bar, i0 - ((c & 1) ? HX : 0), j0 - ((c & 2) ? 1 : 0),
                          s, L::nq(ni));
            }
            tma_load3(base + L::fo(), &Mp->fmap, bar, i0, j0, s);
            bulk_load(base + L::wo(), Gp->wgt[2] + (int64_t)s * 6, 48, bar);
        }
        nnext ^= 1u << slot;
    };
    const long long wlim = g_wait_limit;
    auto wait_z = [&](int s) -> bool { return mbar_wait(&zbar[s & 3], ((znext >> (s & 3)) & 1u) ^ 1u, wlim); };
    auto wait_n = [&](int s) -> bool { return mbar_wait(&nbar[s & 1], ((nnext >> (s & 1)) & 1u) ^ 1u, wlim); };

    bool aborted = false, waited = false;

    for (int si = sbeg; si < send && !aborted; ++si) {
        const int4 sg = segs[si];
        S *dst;
        C *Fout;
        const Bufs *Bp;
        cavity(sg.w, Gp, Mp, dst, Fout, Bp);
        if (kStage) Gp = stage_geo(Gp, sgeo);
        const RunCtl *ctl = Bp->ctl;
        if (!waited) {
            dep_wait();  // from here on: what earlier kernels wrote
            waited = true;
        }
        if (!ctl->active) continue;  // a cavity whose run has stopped
        const Geo &G = *Gp;
        const Bufs &B = *Bp;
        const int nz = G.nz;
        const int ntx = (G.nx + TX - 1) / TX;
        const int64_t P = G.plane;
        const int t = sg.x, ka = sg.y, kb = sg.z;
        i0 = (t % ntx) * TX;
        j0 = (t / ntx) * TY;
        // the segment's z-slices: the first step's needs, then one slice per step
        const int pre_lo = need_lo(ka, nz), pre_hi = need_hi(ka, nz);
        const int seg_hi = need_hi(kb - 1, nz) > pre_hi ? need_hi(kb - 1, nz) : pre_hi;
        for (int s = pre_lo; s <= pre_hi; ++s) issue_z(s);
        issue_n(ka);
        int zissued = pre_hi;

        const int i = i0 + tx, j = j0 + ty;
        const bool active = i < G.nx && j < G.ny;
        C xp[3], xm[3], yp[3], ym[3];
        int xa = 0, xb = 0, ya = 0, yb = 0;
        C Tcn = C(0.0), sTc = C(0.0);  // conduction profile at the node's y and its streaming shift
        if (active) {
            load_w(G.wgt[0], i, xp, xm);
            load_w(G.wgt[1], j, yp, ym);
            if (Tr<ST>::kDevT) {
                Tcn = C(tc_value(G, j));
                sTc = C((1.0 / 12.0) * G.dt * tc_gradient(G));
            }
            xa = off_a(i, G.nx); xb = off_b(i, G.nx);
            ya = off_a(j, G.ny); yb = off_b(j, G.ny);
        }

        for (int k = ka; k < kb; ++k) {
            // prefetch: z-slice k+2 (its slot held k-2, done last step), plane slice k+1
            if (zissued < seg_hi && k + 2 <= seg_hi && k + 2 > zissued) {
                issue_z(k + 2);
                zissued = k + 2;
            }
            if (k + 1 < kb) issue_n(k + 1);

            const int64_t id = (int64_t)k * G.slab + (int64_t)j * G.pitch + i;
            bool ok = true;
            for (int s = need_lo(k, nz); s <= need_hi(k, nz); ++s) ok = ok && wait_z(s);
            ok = ok && wait_n(k);
            if (!ok) {
                atomicExch(err, 1);
                s_abort = 1;
            }
            if (active && ok) {
                const int ka_ = k + off_a(k, nz), kb_ = k + off_b(k, nz);
                const unsigned char *nslot_k = sm + 4 * L::zslot() + (k & 1) * L::nslot();
                const C Fz0 = ((const C *)(nslot_k + L::fo()))[ty * TX + tx];
                const double *wz = (const double *)(nslot_k + L::wo());
                const C zp[3] = {C(wz[0]), C(wz[1]), C(wz[2])}, zm[3] = {C(wz[3]), C(wz[4]), C(wz[5])};
                auto SV = [&](const unsigned char *box, int idx, int q) -> C {
                    (void)q;
                    return tocomp(((const S *)box)[idx]);
                };
                auto ZB = [&](int zi, int s) -> const unsigned char * { return sm + (s & 3) * L::zslot() + L::zoff(zi); };
                auto NB = [&](int ni) -> const unsigned char * {
                    return sm + 4 * L::zslot() + (k & 1) * L::nslot() + L::noff(ni);
                };
                // element index of the thread's node in a box of class c, shifted by (dx, dy)
                auto ix = [&](int c, int dx, int dy) -> int {
                    return (ty + ((c & 2) ? 1 : 0) + dy) * L::bx(c) + tx + ((c & 1) ? HX : 0) + dx;
                };
                C f[19], gg[7];
                // in-plane planes (slice k)
                f[0] = SV(NB(0), ix(0, 0, 0), 0);
                f[1] = ip(xp, SV(NB(1), ix(1, xa, 0), 1), SV(NB(1), ix(1, 0, 0), 1), SV(NB(1), ix(1, xb, 0), 1));
                f[2] = ip(xm, SV(NB(2), ix(1, xa, 0), 2), SV(NB(2), ix(1, 0, 0), 2), SV(NB(2), ix(1, xb, 0), 2));
                f[3] = ip(yp, SV(NB(3), ix(2, 0, ya), 3), SV(NB(3), ix(2, 0, 0), 3), SV(NB(3), ix(2, 0, yb), 3));
                f[4] = ip(ym, SV(NB(4), ix(2, 0, ya), 4), SV(NB(4), ix(2, 0, 0), 4), SV(NB(4), ix(2, 0, yb), 4));
                // xoy (3M:807-824): y-interpolation on three x-columns, then x
                auto XY = [&](int ni, int q, const C *wx, const C *wy) -> C {
                    const unsigned char *b = NB(ni);
                    auto Y = [&](int dx) -> C {
                        return ip(wy, SV(b, ix(3, dx, ya), q), SV(b, ix(3, dx, 0), q), SV(b, ix(3, dx, yb), q));
                    };
                    return ip(wx, Y(xa), Y(0), Y(xb));
                };
                f[7] = XY(5, 7, xp, yp);
                f[8] = XY(6, 8, xm, yp);
                f[9] = XY(7, 9, xp, ym);
                f[10] = XY(8, 10, xm, ym);
                gg[0] = SV(NB(9), ix(0, 0, 0), 19);
                gg[1] = ip(xp, SV(NB(10), ix(1, xa, 0), 20), SV(NB(10), ix(1, 0, 0), 20), SV(NB(10), ix(1, xb, 0), 20));
                gg[2] = ip(xm, SV(NB(11), ix(1, xa, 0), 21), SV(NB(11), ix(1, 0, 0), 21), SV(NB(11), ix(1, xb, 0), 21));
                gg[3] = ip(yp, SV(NB(12), ix(2, 0, ya), 22), SV(NB(12), ix(2, 0, 0), 22), SV(NB(12), ix(2, 0, yb), 22));
                gg[4] = ip(ym, SV(NB(13), ix(2, 0, ya), 23), SV(NB(13), ix(2, 0, 0), 23), SV(NB(13), ix(2, 0, yb), 23));
                // z-reaching planes (slices ka_, k, kb_)
                auto Zc = [&](int zi, int q, const C *wz, int c, int dx, int dy) -> C {
                    const int e = ix(c, dx, dy);
                    return ip(wz, SV(ZB(zi, ka_), e, q), SV(ZB(zi, k), e, q), SV(ZB(zi, kb_), e, q));
                };
                f[5] = Zc(0, 5, zp, 0, 0, 0);
                f[6] = Zc(1, 6, zm, 0, 0, 0);
                // xoz (3M:787-804): z-interpolation on three x-columns, then x
                f[11] = ip(xp, Zc(2, 11, zp, 1, xa, 0), Zc(2, 11, zp, 1, 0, 0), Zc(2, 11, zp, 1, xb, 0));
                f[12] = ip(xm, Zc(3, 12, zp, 1, xa, 0), Zc(3, 12, zp, 1, 0, 0), Zc(3, 12, zp, 1, xb, 0));
                f[13] = ip(xp, Zc(4, 13, zm, 1, xa, 0), Zc(4, 13, zm, 1, 0, 0), Zc(4, 13, zm, 1, xb, 0));
                f[14] = ip(xm, Zc(5, 14, zm, 1, xa, 0), Zc(5, 14, zm, 1, 0, 0), Zc(5, 14, zm, 1, xb, 0));
                // yoz (3M:767-784): z-interpolation on three y-rows, then y
                f[15] = ip(yp, Zc(6, 15, zp, 2, 0, ya), Zc(6, 15, zp, 2, 0, 0), Zc(6, 15, zp, 2, 0, yb));
                f[16] = ip(ym, Zc(7, 16, zp, 2, 0, ya), Zc(7, 16, zp, 2, 0, 0), Zc(7, 16, zp, 2, 0, yb));
                f[17] = ip(yp, Zc(8, 17, zm, 2, 0, ya), Zc(8, 17, zm, 2, 0, 0), Zc(8, 17, zm, 2, 0, yb));
                f[18] = ip(ym, Zc(9, 18, zm, 2, 0, ya), Zc(9, 18, zm, 2, 0, 0), Zc(9, 18, zm, 2, 0, yb));
                gg[5] = Zc(10, 24, zp, 0, 0, 0);
                gg[6] = Zc(11, 25, zm, 0, 0, 0);
                // deviation from the conduction profile along y (the heated axis)
                if (Tr<ST>::kDevT) {
                    gg[3] -= sTc;
                    gg[4] += sTc;
                }

                // walls: bounceback_u / bounceback_T (3B:1053-1197), centre values of slice k
                auto CN = [&](int ni, int q) -> C { return SV(NB(ni), ix(L::nc(ni), 0, 0), q); };
                auto CZ = [&](int zi, int q) -> C { return SV(ZB(zi, k), ix(L::zc(zi), 0, 0), q); };
                const C two_wT = C(2.0) * (C(1.0) / C(12.0));
                if (j == 0) {
                    f[3] = CN(4, 4); f[7] = CN(8, 10); f[8] = CN(7, 9); f[15] = CZ(9, 18); f[17] = CZ(7, 16);
                    gg[3] = -CN(13, 23) + two_wT * (Tr<ST>::kDevT ? C(G.Thot) - Tcn : C(G.Thot));
                }
                if (j == G.ny - 1) {
                    f[4] = CN(3, 3); f[9] = CN(6, 8); f[10] = CN(5, 7); f[16] = CZ(8, 17); f[18] = CZ(6, 15);
                    gg[4] = -CN(12, 22) + two_wT * (Tr<ST>::kDevT ? C(G.Tcold) - Tcn : C(G.Tcold));
                }
                if (i == 0) {
                    f[1] = CN(2, 2); f[9] = CN(6, 8); f[7] = CN(8, 10); f[13] = CZ(3, 12); f[11] = CZ(5, 14);
                    gg[1] = CN(11, 21);
                }
                if (i == G.nx - 1) {
                    f[2] = CN(1, 1); f[8] = CN(7, 9); f[10] = CN(5, 7); f[12] = CZ(4, 13); f[14] = CZ(2, 11);
                    gg[2] = CN(10, 20);
                }
                if (k == 0) {
                    f[5] = CZ(1, 6); f[11] = CZ(5, 14); f[12] = CZ(4, 13); f[15] = CZ(9, 18); f[16] = CZ(8, 17);
                    gg[5] = CZ(11, 25);
                }
                if (k == nz - 1) {
                    f[6] = CZ(0, 5); f[13] = CZ(3, 12); f[14] = CZ(2, 11); f[17] = CZ(7, 16); f[18] = CZ(6, 15);
                    gg[6] = CZ(10, 24);
                }

                // macro_u / macro_t (3M:988-1025) and the collision
                C rho, u, v, w, T, fp[19], gp[7], Fz;
                node3d<C, Tr<ST>::kShift, Tr<ST>::kDevT>(f, gg, Fz0, G, fp, gp, Fz, rho, u, v, w, T, Tcn);
                if (write_macro) {
                    const int64_t mid = ((int64_t)k * G.ny + j) * G.nx + i;
                    B.rho[mid] = double(rho); B.u[mid] = double(u); B.v[mid] = double(v);
                    B.w[mid] = double(w); B.T[mid] = double(T);
                }
                Fout[id] = Fz;
#pragma unroll
                for (int q = 0; q < 19; ++q) {
                    dst[q * P + id] = tostore<S, C>(fp[q]);
                }
#pragma unroll
                for (int q = 0; q < 7; ++q) {
                    dst[(19 + q) * P + id] = tostore<S, C>(gp[q]);
                }
            }
            __syncthreads();
            if (s_abort) {
                aborted = true;
                break;
            }
        }
    }
    if (aborted && tid == 0) {
        // let copies still in flight land before the CTA's shared memory is released
        for (int s = 0; s < 4; ++s) mbar_wait(&zbar[s], ((znext >> s) & 1u) ^ 1u);
        for (int s = 0; s < 2; ++s) mbar_wait(&nbar[s], ((nnext >> s) & 1u) ^ 1u);
    }
}

template <int ST, int TY_>
__global__ void __launch_bounds__(32 * TY_, TY_ == 8 ? 1 : 2)
k_march3d(const __grid_constant__ TmapSet maps, const __grid_constant__ Geo G,
          const typename Tr<ST>::C *__restrict__ Fin, typename Tr<ST>::S *__restrict__ dst,
          typename Tr<ST>::C *__restrict__ Fout, const __grid_constant__ Bufs B, int write_macro,
          const int4 *__restrict__ segs, const int *__restrict__ seg_off, int *err)
{
    (void)Fin;
    using S = typename Tr<ST>::S;
    using C = typename Tr<ST>::C;
    auto cavity = [&](int, const Geo *&Gp, const TmapSet *&Mp, S *&d, C *&Fo, const Bufs *&Bp) {
        Gp = &G;
        Mp = &maps;
        d = dst;
        Fo = Fout;
        Bp = &B;
    };
    march3d_run<ST, TY_, false>(segs, seg_off[blockIdx.x], seg_off[blockIdx.x + 1], cavity, write_macro, err);
}

// many 3D cavities: segments (tile, z0, z1, cavity) of the batch's work list;
// `cur` is the ping-pong buffer holding the populations read this step
template <int ST, int TY_>
__global__ void __launch_bounds__(32 * TY_, TY_ == 8 ? 1 : 2)
k_march3d_batch(const BatchDev D, int cur, int write_macro, int *err)
{
    using S = typename Tr<ST>::S;
    using C = typename Tr<ST>::C;
    auto cavity = [&](int c, const Geo *&Gp, const TmapSet *&Mp, S *&d, C *&Fo, const Bufs *&Bp) {
        Gp = &D.geo[c];
        Mp = &D.maps[(int64_t)c * 2 + cur];
        Bp = &D.bufs[c];
        d = (S *)D.bufs[c].pop[1 - cur];
        Fo = (C *)D.bufs[c].F[1 - cur];
    };
    march3d_run<ST, TY_, true>(D.segs, D.seg_off[blockIdx.x], D.seg_off[blockIdx.x + 1], cavity, write_macro, err);
}

// ---------------------------------------------------------------------------
// 2D layout: a tile is TX nodes of one row; the march runs along y
// ---------------------------------------------------------------------------
// 2D layout.  Ring depths: the y-ring holds YS rows of the planes whose
// stencil reaches along y, the plane ring NS rows of the others; at row j the
// copies of rows up to j + YS - 2 (y-ring) and j + NS - 1 (plane ring) are in
// flight or landed, each refilling the slot of a row every thread has
// finished.  The batch kernel keeps 4 / 2 (more blocks per SM pay more on its
// short segments); the single-cavity kernel runs 6 / 4 (measured on B200 at
// 2048^2 FP64: 23,200 against 21,693 MLUPS; the batch loses 6-26 % with it).
template <int ST, int TX_ = 128, int YS_ = 4, int NS_ = 2>
struct L2 {
    static constexpr int YS = YS_, NS = NS_;
    static_assert(YS >= 4 && NS >= 2 && YS + NS <= 30, "2D ring depths");
    // the barriers (YS + NS) and the abort word, rounded up to 64 bytes
    static constexpr int BAR = ((YS + NS + 1) * 8 + 63) / 64 * 64;
    using S = typename Tr<ST>::S;
    using C = typename Tr<ST>::C;
    static constexpr int ES = sizeof(S);
    static constexpr int TX = TX_, NT = TX;
    static constexpr int HX = 16 / ES;
    __host__ __device__ static constexpr int bx(int c) { return TX + (c ? 2 * HX : 0); }
    __host__ __device__ static constexpr int bytes(int c) { return bx(c) * ES; }
    __host__ __device__ static constexpr int padded(int c) { return (bytes(c) + 127) / 128 * 128; }
    // y-ring planes: 2 4 | 5 6 7 8 | 11 13 ; classes 0 0 | 1 1 1 1 | 0 0
    __host__ __device__ static constexpr int yq(int yi)
    {
        return yi == 0 ? 2 : (yi == 1 ? 4 : (yi < 6 ? yi + 3 : (yi == 6 ? 11 : 13)));
    }
    __host__ __device__ static constexpr int yc(int yi) { return (yi >= 2 && yi < 6) ? 1 : 0; }
    __host__ __device__ static constexpr int yoff(int yi)
    {
        int o = 0;
        for (int a = 0; a < yi; ++a) o += padded(yc(a));
        return o;
    }
    __host__ __device__ static constexpr int yslot() { return yoff(8); }
    __host__ __device__ static constexpr int ytx()
    {
        int b = 0;
        for (int a = 0; a < 8; ++a) b += bytes(yc(a));
        return b;
    }
    // row planes: 0 1 3 9 10 12 ; classes 0 1 1 0 1 1
    __host__ __device__ static constexpr int nq(int ni)
    {
        return ni == 0 ? 0 : (ni == 1 ? 1 : (ni == 2 ? 3 : (ni == 3 ? 9 : (ni == 4 ? 10 : 12))));
    }
    __host__ __device__ static constexpr int nc(int ni) { return (ni == 0 || ni == 3) ? 0 : 1; }
    __host__ __device__ static constexpr int noff(int ni)
    {
        int o = 0;
        for (int a = 0; a < ni; ++a) o += padded(nc(a));
        return o;
    }
    __host__ __device__ static constexpr int fbytes() { return TX * (int)sizeof(C); }
    __host__ __device__ static constexpr int fo() { return noff(6); }
    __host__ __device__ static constexpr int wo() { return fo() + (fbytes() + 127) / 128 * 128; }
    __host__ __device__ static constexpr int nslot() { return wo() + 128; }
    __host__ __device__ static constexpr int ntx()
    {
        int b = 0;
        for (int a = 0; a < 6; ++a) b += bytes(nc(a));
        return b + fbytes() + 48;
    }
    __host__ __device__ static constexpr int smem() { return YS * yslot() + NS * nslot() + BAR + kGeoStage + 128; }
};

// the single-cavity 2D kernel's layouts: 128-node rows with 4 / 2 ring slots
// (four blocks per SM in FP64: lower latency per step, the faster choice up to
// a few hundred thousand nodes) or 6 / 4 (two blocks per SM, more rows in
// flight: the faster choice on large domains).  Measured on B200, FP64, per
// step: 256^2 4.87 us (4 / 2) against 5.70 us (6 / 4); 2048^2 21,666 against
// 23,400 MLUPS.
template <int ST>
using L2s = L2<ST, 128, 4, 2>;
template <int ST>
using L2d = L2<ST, 128, 6, 4>;
// nodes from which the single-cavity 2D kernel uses the deep ring
constexpr int64_t kDeepRingNodes = int64_t(1) << 20;

// One node of the 2D march at row j, from the ring slots in shared memory:
// interpolation, walls, macro, collision, stores.
template <int ST, class L>
__device__ __forceinline__ void march2d_node(const unsigned char *sm, const Geo &G, int tx, int i, int j, int xa,
                                             int xb, const typename Tr<ST>::C *xp, const typename Tr<ST>::C *xm,
                                             typename Tr<ST>::C Tcn, typename Tr<ST>::C sT,
                                             typename Tr<ST>::S *__restrict__ dst,
                                             typename Tr<ST>::C *__restrict__ Fout, const Bufs &B, int write_macro)
{
    using S = typename Tr<ST>::S;
    using C = typename Tr<ST>::C;
    constexpr int HX = L::HX;
    const int ny = G.ny;
    const int64_t P = G.plane;
    const int64_t id = (int64_t)j * G.pitch + i;
    const int ja_ = j + off_a(j, ny), jb_ = j + off_b(j, ny);
    const unsigned char *nslot_j = sm + L::YS * L::yslot() + (j % L::NS) * L::nslot();
    const C Fy0 = ((const C *)(nslot_j + L::fo()))[tx];
    const double *wy = (const double *)(nslot_j + L::wo());
    const C yp[3] = {C(wy[0]), C(wy[1]), C(wy[2])}, ym[3] = {C(wy[3]), C(wy[4]), C(wy[5])};
    auto SV = [&](const unsigned char *box, int idx, int q) -> C {
        (void)q;
        return tocomp(((const S *)box)[idx]);
    };
    auto YB = [&](int yi, int s) -> const unsigned char * { return sm + (s % L::YS) * L::yslot() + L::yoff(yi); };
    auto NB = [&](int ni) -> const unsigned char * { return nslot_j + L::noff(ni); };
    auto ix = [&](int c, int dx) -> int { return tx + (c ? HX : 0) + dx; };
    // y-interpolation of a y-ring plane at x-offset dx
    auto YI = [&](int yi, int q, const C *w, int dx) -> C {
        const int c = L::yc(yi);
        const int e = ix(c, dx);
        return ip(w, SV(YB(yi, ja_), e, q), SV(YB(yi, j), e, q), SV(YB(yi, jb_), e, q));
    };
    C f[9], gg[5];
    f[0] = SV(NB(0), ix(0, 0), 0);
    f[1] = ip(xp, SV(NB(1), ix(1, xa), 1), SV(NB(1), ix(1, 0), 1), SV(NB(1), ix(1, xb), 1));
    f[2] = YI(0, 2, yp, 0);
    f[3] = ip(xm, SV(NB(2), ix(1, xa), 3), SV(NB(2), ix(1, 0), 3), SV(NB(2), ix(1, xb), 3));
    f[4] = YI(1, 4, ym, 0);
    f[5] = ip(xp, YI(2, 5, yp, xa), YI(2, 5, yp, 0), YI(2, 5, yp, xb));
    f[6] = ip(xm, YI(3, 6, yp, xa), YI(3, 6, yp, 0), YI(3, 6, yp, xb));
    f[7] = ip(xm, YI(4, 7, ym, xa), YI(4, 7, ym, 0), YI(4, 7, ym, xb));
    f[8] = ip(xp, YI(5, 8, ym, xa), YI(5, 8, ym, 0), YI(5, 8, ym, xb));
    gg[0] = SV(NB(3), ix(0, 0), 9);
    gg[1] = ip(xp, SV(NB(4), ix(1, xa), 10), SV(NB(4), ix(1, 0), 10), SV(NB(4), ix(1, xb), 10));
    gg[2] = YI(6, 11, yp, 0);
    gg[3] = ip(xm, SV(NB(5), ix(1, xa), 12), SV(NB(5), ix(1, 0), 12), SV(NB(5), ix(1, xb), 12));
    gg[4] = YI(7, 13, ym, 0);
    // deviation from the conduction profile along x (the heated axis)
    // (Tcn: the conduction profile at the node's x, sT: its streaming shift;
    // both per column, computed once per segment)
    if (Tr<ST>::kDevT) {
        gg[1] -= sT;
        gg[3] += sT;
    }

    // walls (2B:731-801): centre values of row j
    auto CN = [&](int ni, int q) -> C { return SV(NB(ni), ix(L::nc(ni), 0), q); };
    auto CY = [&](int yi, int q) -> C { return SV(YB(yi, j), ix(L::yc(yi), 0), q); };
    const C two_wT = C(2.0) * C(0.125);
    if (i == 0) {
        f[1] = CN(2, 3); f[5] = CY(4, 7); f[8] = CY(3, 6);
        gg[1] = -CN(5, 12) + two_wT * (Tr<ST>::kDevT ? C(G.Thot) - Tcn : C(G.Thot));
    }
    if (i == G.nx - 1) {
        f[3] = CN(1, 1); f[6] = CY(5, 8); f[7] = CY(2, 5);
        gg[3] = -CN(4, 10) + two_wT * (Tr<ST>::kDevT ? C(G.Tcold) - Tcn : C(G.Tcold));
    }
    if (j == ny - 1) {
        f[4] = CY(0, 2); f[7] = CY(2, 5); f[8] = CY(3, 6);
        gg[4] = CY(6, 11);
    }
    if (j == 0) {
        f[2] = CY(1, 4); f[5] = CY(4, 7); f[6] = CY(5, 8);
        gg[2] = CY(7, 13);
    }

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
    const C T = Tr<ST>::kDevT ? Tcn + (gg[0]+gg[1]+gg[2]+gg[3]+gg[4]) : gg[0]+gg[1]+gg[2]+gg[3]+gg[4];
    if (write_macro) {
        const int64_t mid = (int64_t)j * G.nx + i;
        B.rho[mid] = double(rho); B.u[mid] = double(u); B.v[mid] = double(v); B.T[mid] = double(T);
    }
    C fp[9], gp[5], Fy;
    collide2d<C, Tr<ST>::kShift, Tr<ST>::kDevT>(f, gg, rho, u, v, T, G, fp, gp, Fy);
    Fout[id] = Fy;
#pragma unroll
    for (int q = 0; q < 9; ++q) dst[q * P + id] = tostore<S, C>(fp[q]);
#pragma unroll
    for (int q = 0; q < 5; ++q) dst[(9 + q) * P + id] = tostore<S, C>(gp[q]);
}

// The 2D march over a list of segments (a cavity, a TX-wide column strip at
// x-offset i0, rows [ja, jb)).  `seg(k, cav, i0, ja, jb)` yields the block's
// k-th segment; `cavity(cav, G, maps, dst, Fout, B)` yields the cavity's
// geometry, the TMA descriptors of its source buffer and its outputs.
template <int ST, class L, bool kStage, class SegFn, class CavFn>
__device__ __forceinline__ void march2d_run(int nseg, SegFn seg, CavFn cavity, int write_macro, int *err)
{
    using S = typename Tr<ST>::S;
    using C = typename Tr<ST>::C;
    constexpr int TX = L::TX;
    constexpr int HX = L::HX;
    extern __shared__ unsigned char sm_raw[];
    unsigned char *sm = sm_raw + ((128u - (saddr(sm_raw) & 127u)) & 127u);
    uint64_t *ybar = (uint64_t *)(sm + L::YS * L::yslot() + L::NS * L::nslot());
    uint64_t *nbar = ybar + L::YS;
    volatile int &s_abort = *(volatile int *)(nbar + L::NS);
    Geo *sgeo = (Geo *)(sm + L::YS * L::yslot() + L::NS * L::nslot() + L::BAR);

    const int tid = threadIdx.x;
    const int tx = tid;
    if (tid == 0) {
        for (int s = 0; s < L::YS; ++s) mbar_init(&ybar[s], 1);
        for (int s = 0; s < L::NS; ++s) mbar_init(&nbar[s], 1);
        fence_barrier_init();
        s_abort = 0;
    }
    dep_launch();
    __syncthreads();

    uint32_t ynext = 0, nnext = 0;
    bool aborted = false, waited = false;
    const long long wlim = g_wait_limit;
    for (int k = 0; k < nseg && !aborted; ++k) {
        int cav, i0, ja, jb;
        seg(k, cav, i0, ja, jb);
        const Geo *Gp;
        const CUtensorMap *maps;
        S *dst;
        C *Fout;
        const Bufs *Bp;
        cavity(cav, Gp, maps, dst, Fout, Bp);
        if (kStage) Gp = stage_geo(Gp, sgeo);
        const RunCtl *ctl = Bp->ctl;
        if (!waited) {
            dep_wait();  // from here on: what earlier kernels wrote
            waited = true;
        }
        if (!ctl->active) continue;  // a cavity whose run has stopped
        const Geo &G = *Gp;
        const int ny = G.ny;

        auto issue_y = [&](int s) {
            const int slot = s % L::YS;
            if (tid == 0) {
                uint64_t *bar = &ybar[slot];
                mbar_arrive_tx(bar, L::ytx());
                unsigned char *base = sm + slot * L::yslot();
#pragma unroll
                for (int yi = 0; yi < 8; ++yi) {
                    const int c = L::yc(yi);
                    tma_load3(base + L::yoff(yi), &maps[c], bar, i0 - (c ? HX : 0), s, L::yq(yi));
                }
            }
            ynext ^= 1u << slot;
        };
        auto issue_n = [&](int s) {
            const int slot = s % L::NS;
            if (tid == 0) {
                uint64_t *bar = &nbar[slot];
                mbar_arrive_tx(bar, L::ntx());
                unsigned char *base = sm + L::YS * L::yslot() + slot * L::nslot();
#pragma unroll
                for (int ni = 0; ni < 6; ++ni) {
                    const int c = L::nc(ni);
                    tma_load3(base + L::noff(ni), &maps[c], bar, i0 - (c ? HX : 0), s, L::nq(ni));
                }
                tma_load2(base + L::fo(), &maps[4], bar, i0, s);
                bulk_load(base + L::wo(), G.wgt[1] + (int64_t)s * 6, 48, bar);
            }
            nnext ^= 1u << slot;
        };
        auto wait_y = [&](int s) -> bool {
            return mbar_wait(&ybar[s % L::YS], ((ynext >> (s % L::YS)) & 1u) ^ 1u, wlim);
        };
        auto wait_n = [&](int s) -> bool {
            return mbar_wait(&nbar[s % L::NS], ((nnext >> (s % L::NS)) & 1u) ^ 1u, wlim);
        };

        // the segment's first copies: the y rows row ja needs and the rows
        // behind them up to ja + L::YS - 3, the plane rows ja .. ja + L::NS - 2
        const int pre_lo = need_lo(ja, ny), pre_hi = need_hi(ja, ny);
        const int seg_hi = need_hi(jb - 1, ny) > pre_hi ? need_hi(jb - 1, ny) : pre_hi;
        const int y0 = min(seg_hi, max(pre_hi, ja + L::YS - 3));
        for (int s = pre_lo; s <= y0; ++s) issue_y(s);
        const int n0 = min(jb - 1, ja + L::NS - 2);
        for (int s = ja; s <= n0; ++s) issue_n(s);
        int yissued = y0, nissued = n0;

        const int i = i0 + tx;
        const bool active = i < G.nx;
        C xp[3], xm[3];
        int xa = 0, xb = 0;
        C Tcn = C(0.0), sT = C(0.0);  // conduction profile at the column and its streaming shift
        if (active) {
            load_w(G.wgt[0], i, xp, xm);
            xa = off_a(i, G.nx); xb = off_b(i, G.nx);
            if (Tr<ST>::kDevT) {
                Tcn = C(tc_value(G, i));
                sT = C(0.125 * G.dt * tc_gradient(G));
            }
        }
        for (int j = ja; j < jb; ++j) {
            // refill the slots of rows every warp has finished (the barrier
            // that ended row j-1): y rows up to j + L::YS - 2, plane rows up to
            // j + L::NS - 1
            for (const int yt = min(seg_hi, j + L::YS - 2); yissued < yt;) issue_y(++yissued);
            for (const int nt = min(jb - 1, j + L::NS - 1); nissued < nt;) issue_n(++nissued);
            bool ok = true;
            for (int s = need_lo(j, ny); s <= need_hi(j, ny); ++s) ok = ok && wait_y(s);
            ok = ok && wait_n(j);
            if (!ok) {
                atomicExch(err, 1);
                s_abort = 1;
            }
            if (active && ok)
                march2d_node<ST, L>(sm, G, tx, i, j, xa, xb, xp, xm, Tcn, sT, dst, Fout, *Bp, write_macro);
            __syncthreads();
            if (s_abort) {
                aborted = true;
                break;
            }
        }
    }
    if (aborted && tid == 0) {
        for (int s = 0; s < L::YS; ++s) mbar_wait(&ybar[s], ((ynext >> s) & 1u) ^ 1u);
        for (int s = 0; s < L::NS; ++s) mbar_wait(&nbar[s], ((nnext >> s) & 1u) ^ 1u);
    }
}

// one cavity: each block takes an equal contiguous share of the
// (strip-major, row-minor) work items
template <int ST, class L>
__global__ void __launch_bounds__(128, 4)
k_march2d(const __grid_constant__ TmapSet maps, const Geo G, const typename Tr<ST>::C *__restrict__ Fin,
          typename Tr<ST>::S *__restrict__ dst, typename Tr<ST>::C *__restrict__ Fout, const Bufs B,
          int write_macro, int64_t total, int *err)
{
    (void)Fin;
    using S = typename Tr<ST>::S;
    using C = typename Tr<ST>::C;
    constexpr int TX = L::TX;
    // the rows the kernel computes, [jlo, jhi): all rows, or a slab's rows
    // without its ghost rows
    const int nr = G.jhi - G.jlo;
    const int64_t G_ = gridDim.x;
    const int64_t ubeg = total * blockIdx.x / G_, uend = total * (blockIdx.x + 1) / G_;
    // segments: the block's range split at strip boundaries
    const int nseg = ubeg >= uend ? 0 : int((uend - 1) / nr - ubeg / nr + 1);
    auto seg = [&](int k, int &cav, int &i0, int &ja, int &jb) {
        const int64_t t = ubeg / nr + k;
        const int64_t lo = t * nr > ubeg ? t * nr : ubeg;
        const int64_t hi = (t + 1) * nr < uend ? (t + 1) * nr : uend;
        cav = 0;
        i0 = int(t) * TX;
        ja = G.jlo + int(lo - t * nr);
        jb = G.jlo + int(hi - t * nr);
    };
    const CUtensorMap *mp = &maps.m[0];
    auto cavity = [&](int, const Geo *&Gp, const CUtensorMap *&m, S *&d, C *&Fo, const Bufs *&Bp) {
        Gp = &G;
        m = mp;
        d = dst;
        Fo = Fout;
        Bp = &B;
    };
    march2d_run<ST, L, false>(nseg, seg, cavity, write_macro, err);
}

// many cavities: block b runs segments seg_off[b] .. seg_off[b+1]-1; `cur`
// is the ping-pong buffer holding the populations read this step.  Blocks per
// SM: FP64 16 warps (shared memory bounds it there too), FP32 24 warps (80
// registers, no spills)
template <int ST, int TX>
__global__ void __launch_bounds__(TX, (ST == kF32 ? 768 : 512) / TX)
k_march2d_batch(const BatchDev D, int cur, int write_macro, int *err)
{
    using S = typename Tr<ST>::S;
    using C = typename Tr<ST>::C;
    const int s0 = D.seg_off[blockIdx.x], s1 = D.seg_off[blockIdx.x + 1];
    auto seg = [&](int k, int &cav, int &i0, int &ja, int &jb) {
        const int4 q = D.segs[s0 + k];
        cav = q.x;
        i0 = q.y;
        ja = q.z;
        jb = q.w;
    };
    auto cavity = [&](int c, const Geo *&Gp, const CUtensorMap *&m, S *&d, C *&Fo, const Bufs *&Bp) {
        Gp = &D.geo[c];
        m = &D.maps[(int64_t)c * 2 + cur].m[0];
        Bp = &D.bufs[c];
        d = (S *)D.bufs[c].pop[1 - cur];
        Fo = (C *)D.bufs[c].F[1 - cur];
    };
    march2d_run<ST, L2<ST, TX>, true>(s1 - s0, seg, cavity, write_macro, err);
}
