/*
 * lbm_b200.h -- C ABI of the B200 thermal lattice-Boltzmann time step.
 *
 * This is the drop-in boundary for the time step of the reference Fortran
 * solver (zzhao0930/MPI-Multi-Process-Version).  The reference has no API:
 * its step is a chain of argument-less subroutines that share `module
 * commondata` (natural-convection_2dim_mono.f90:1-72, 3dim_mono.f90:1-77) and
 * are called from the `do while` loop of `program main`
 * (2dim_mono.f90:307-330, 3dim_mono.f90:373-396).  Each entry point below
 * replaces one or more of those subroutines; the comment on each names them.
 * A Fortran caller binds these with `iso_c_binding` (`bind(C, name=...)`
 * interfaces over the same argument lists).
 *
 * Conventions
 *   - every function returns an int status: LBM_OK (0) or a negative
 *     LBM_ERR_* code; lbm_last_error() gives a one-line message;
 *   - host arrays are in the reference's Fortran layout: scalar fields
 *     a(nx, ny[, nz]) (x fastest), populations f(0:Q-1, nx, ny[, nz])
 *     (population index fastest), coordinates x(0:n+1) in lattice units;
 *   - all device work of a handle runs on the handle's own CUDA stream;
 *     lbm_step is asynchronous, the getters and reductions synchronise;
 *   - the library owns its device memory; the caller owns host arrays.
 */
#ifndef LBM_B200_H
#define LBM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBM_ABI_VERSION 1

/* status codes */
#define LBM_OK               0
#define LBM_ERR_PARAM       -1  /* a bad argument or parameter set */
#define LBM_ERR_CUDA        -2  /* a CUDA runtime call failed */
#define LBM_ERR_NONFINITE   -3  /* NaN or Inf found in a reduction */
#define LBM_ERR_DIVERGED    -4  /* residual grew past the allowed bound */
#define LBM_ERR_TIMEOUT     -5  /* a bounded device wait gave up */
#define LBM_ERR_STATE       -6  /* call out of order (e.g. step before init) */
#define LBM_ERR_NOMEM       -7  /* device allocation failed */
#define LBM_ERR_UNSUPPORTED -8  /* option not built into this library */
#define LBM_ERR_NODEVICE    -9  /* no CUDA device visible */

/* population storage precision */
#define LBM_STORE_F64   0  /* FP64 storage, FP64 arithmetic: the drop-in */
#define LBM_STORE_F32   1  /* FP32 storage and arithmetic on deviations: f - w*rho0 and
                              g - wT*Tc (Tc: the conduction profile between the walls) */
#define LBM_STORE_F16S  2  /* retired: the same deviations stored as binary16 gave Nu_avg errors
                              of order one against FP64 and no speed-up over FP32 storage on
                              B200; lbm_create rejects it with LBM_ERR_UNSUPPORTED */

/* arithmetic mode (FP64 storage only) */
#define LBM_MODE_FAST   0  /* multiply-add contraction, reciprocal constants */
#define LBM_MODE_EXACT  1  /* the reference's operation order, no contraction:
                              bit-identical to the CPU restatement */

/* options for lbm_set_option / lbm_get_option */
#define LBM_OPT_KERNEL   1  /* step kernel: 0 automatic, 1 direct-load, 2 TMA march */
#define LBM_OPT_NBLOCKS  2  /* persistent blocks of the march kernel (0 = automatic) */
#define LBM_OPT_L2PROMO  3  /* L2 fetch promotion of the march kernel's TMA boxes:
                               0 none, 1 64 B, 2 128 B, 3 256 B */
#define LBM_OPT_GRAPHS   4  /* 1 (default): lbm_step replays captured 8-step CUDA graphs */
#define LBM_OPT_RESIDENT 5  /* 0 (default) / 1: 2D domains of one resident wave run all iterations
                               of an lbm_step call in one cooperative launch with a bounded grid
                               barrier between iterations.  Measured at 128^2 on B200: 3.87 us per
                               iteration in FP32 (4.10 with graph-replayed launches) but 4.85 us
                               in FP64, hence opt-in.  Batch members always step per iteration. */
#define LBM_OPT_TILEY    6  /* 3D march kernel tile rows: 0 automatic (4), 4 (two blocks per SM) or 8 */
#define LBM_OPT_PLAN     7  /* 3D march work plan: 0 (default) every tile column in equal z-chunks
                               run side by side (neighbours share halo rows through L2), the blocks
                               left over taking the chunks' last slices in lockstep rounds;
                               1 contiguous equal shares of the (tile, slice) items */
#define LBM_OPT_WAIT_LIMIT 8 /* limit, in GPU clock cycles, of the march kernels' waits for their TMA
                               copies within a step, for every handle on the handle's device;
                               0 restores the default (4e9, about 2 s).  A wait that runs out sets
                               the device error flag: the next synchronising call returns
                               LBM_ERR_TIMEOUT and the populations are not valid until the next
                               init call.  For tests of that error path.  lbm_get_option reports
                               the value last set through this handle (0: default). */
#define LBM_OPT_PDL      9  /* 1 (default): consecutive march steps are launched as programmatic
                               dependents (CUDA programmatic dependent launch): a step's blocks are
                               scheduled while the previous step drains, set up, and wait for its
                               completion before reading the populations; 0: plain stream order.
                               Results are identical either way. */

/* grid kinds for lbm_mesh */
#define LBM_GRID_ERF     0  /* the reference's erf grid, constA = stretch (3.2) */
#define LBM_GRID_TANH    1  /* 0.5*(1 + tanh(b*(2*xi-1))/tanh(b)), b = stretch */
#define LBM_GRID_UNIFORM 2

typedef struct lbm_params {
    int32_t dim;            /* 2 (D2Q9 + D2Q5) or 3 (D3Q19 + D3Q7) */
    int32_t nx, ny, nz;     /* nodes per axis; nz ignored when dim == 2 */
    double Ra, Pr, Ma;      /* Rayleigh, Prandtl, Mach: commondata 2M:9-11 */
    double Thot, Tcold;     /* wall temperatures: 2M:12 */
    double dt;              /* time step in lattice units from mesh(): 2M:111 */
    double length_LB;       /* 1/dx(1) from mesh(): 2M:110 */
    int32_t storage;        /* LBM_STORE_* */
    int32_t mode;           /* LBM_MODE_* */
    int32_t device;         /* CUDA device ordinal */
    int32_t reserved;       /* must be 0 */
} lbm_params;

typedef struct lbm_handle lbm_handle;

/* Version of this ABI (LBM_ABI_VERSION). */
int lbm_abi_version(void);

/* Short text for a status code, and the last error message of this thread. */
const char *lbm_error_string(int status);
const char *lbm_last_error(void);

/* mesh(): the reference's grid construction, 2M:74-134 (3M:122-189).
 * Fills x(0:nx+1), y(0:ny+1) and, for nz > 0, z(0:nz+1) in lattice units and
 * returns dx0, length_LB and dt.  Host only; needs no GPU. */
int lbm_mesh(int32_t kind, double stretch, int32_t nx, int32_t ny, int32_t nz,
             double *x, double *y, double *z,
             double *dx0, double *length_LB, double *dt);

/* mesh() generalised to boxes of physical size lx x ly (x lz) with any node
 * counts (the reference assumes a unit square or cube with nx = ny = nz):
 * each axis gets the stretched raw grid on [0, l_axis]; the smallest first
 * spacing over the axes sets the lattice unit (dx0, length_LB = 1/dx0,
 * dt = dx0*length_LB); every axis is shifted by dx0/2 and scaled by
 * length_LB as in 2M:113-116.  With lx = ly (= lz) = 1 and equal node counts
 * this is exactly lbm_mesh. */
int lbm_mesh_box(int32_t kind, double stretch, int32_t nx, int32_t ny, int32_t nz,
                 double lx, double ly, double lz, double *x, double *y, double *z,
                 double *dx0, double *length_LB, double *dt);

/* The parameter block of initial() (2M:151-162, 3M:206-229) for a parameter
 * set: out[0..8] = viscosity_LB, kappa, gbeta, tauf, Snu, Sq, sig_k, dt,
 * length_LB.  Host only. */
int lbm_derived_params(const lbm_params *p, double *out9);

/* Create a cavity on p->device: allocates device state, derives the
 * parameters of initial() and the interpolation weights of interpolate()
 * (2M:591-660) from the coordinates.  x, y, z are x(0:n+1) as mesh() leaves
 * them; z may be NULL when dim == 2.  Replaces the allocations and the
 * parameter block of initial() (2M:143-197). */
int lbm_create(const lbm_params *p, const double *x, const double *y,
               const double *z, lbm_handle **out);

/* Free everything the handle owns (the deallocate block of main, 2M:347-375). */
int lbm_destroy(lbm_handle *h);

/* The reference's initial state (initial(), 2M:199-240 / 3M:256-301):
 * rho = 1, u = v = w = 0, T the linear conduction profile between the
 * isothermal walls, f and g at equilibrium; resets itc and the check state. */
int lbm_init_reference(lbm_handle *h);

/* Equilibrium initial state from host macroscopic fields a(nx,ny[,nz]) with
 * the equilibrium formulas of initial() (2M:227-240, 3M:286-301).  w may be
 * NULL (taken as 0).  Resets itc and the check state.  This is the entry
 * point of warm starts. */
int lbm_init_equilibrium(lbm_handle *h, const double *rho, const double *u,
                         const double *v, const double *w, const double *T);

/* Warm start (no counterpart in the reference, whose only initial state is
 * the one of initial()): like lbm_init_equilibrium, plus the first-order
 * Chapman-Enskog non-equilibrium part of the given fields,
 *   f_a -= 3 tau_f dt w_a rho (e_a e_a : grad u - div u / 3)
 *   g_a -= (dt / sig_k) wT_a (e_a . grad T)
 * with gradients from the slope of the quadratic through each node's
 * interpolation stencil (one-sided at the walls) on the stretched grid.
 * Rejects non-finite field values with LBM_ERR_NONFINITE. */
int lbm_init_warm(lbm_handle *h, const double *rho, const double *u,
                  const double *v, const double *w, const double *T);

/* Advance nsteps iterations of the reference loop body: collision_U,
 * collision_T, update (a no-op on one domain), interpolate, bounceback_u,
 * bounceback_T, macro_u, macro_t (2M:309-325, 3M:375-391).  Asynchronous. */
int lbm_step(lbm_handle *h, int32_t nsteps);

/* The reference's time loop (2M:307-330): lbm_step until, at a check every
 * check_every iterations (counted from the last init, as itc is), both
 * residuals of lbm_check are at most eps, or max_steps iterations were done.
 * Reports the iterations done and the last residuals; returns
 * LBM_ERR_NONFINITE if a residual sum stops being finite.  The stop test runs
 * on the device after each check (the same sums and residuals as lbm_check):
 * once it fires, the steps queued after it do nothing, and the host
 * synchronises once every four checks instead of at every check. */
int lbm_run(lbm_handle *h, int64_t max_steps, int32_t check_every, double eps,
            int64_t *steps_done, double *errU, double *errT);

/* Iterations done since the last init (the reference's itc). */
int lbm_itc(const lbm_handle *h, int64_t *itc);

/* check(): 2M:755-805 (3M:1027-1082).  errU = |u - u_prev| / |u|,
 * errT = |T - T_prev| / |T| in FP64 over all nodes; then u_prev = u,
 * T_prev = T.  Returns LBM_ERR_NONFINITE if a sum is not finite. */
int lbm_check(lbm_handle *h, double *errU, double *errT);

/* Wall-averaged Nusselt numbers at the hot and cold isothermal walls, FP64.
 * The reference has no such function (no counterpart to cite).
 * Local Nu = -(L_LB-1)/(Thot-Tcold) dT/dn from the quadratic through the
 * wall (dt/2 outside the first node) and the first two nodes; averaged with
 * node cell widths. */
int lbm_nusselt(lbm_handle *h, double *nu_hot, double *nu_cold);

/* Mass sum(rho*dV) and energy sum(T*dV) in FP64 (no counterpart). */
int lbm_sums(lbm_handle *h, double *mass, double *energy);

/* ------------------------------------------------------------------------ */
/* Slabs: one domain split along its slowest axis (y in 2D, z in 3D) over
 * several handles (on one GPU, on several GPUs of a process, or one per
 * rank).  Replaces the reference's slab decomposition (the ghost rows / planes
 * of f_post / g_post; natural-convection_2dim_mono.f90 and 3dim_mono.f90 split
 * y and z over ranks, StartEnd) and its per-step ghost exchange `update`
 * (natural-convection_2dim_mono.f90:572-589, 2dim_block.f90:602-658,
 * 3dim_mono.f90:732-749).
 *
 * lbm_create_slab: p and the coordinate arrays x(0:nx+1), y(0:ny+1) and, in
 * 3D, z(0:nz+1) describe the WHOLE domain (z NULL in 2D); the handle owns
 * layers [lo, hi) of the split axis (rows in 2D, z-slices in 3D; 0-based, at
 * least 2) plus one ghost layer on each side that has a neighbouring slab.
 * Every other call works on the handle as on a cavity of the slab's layers
 * plus ghosts (the fields of lbm_get_macro / lbm_init_* are (nx, rows incl.
 * ghosts) in 2D, (nx, ny, slices incl. ghosts) in 3D); its step kernels
 * compute only its own layers, lbm_check_sums / lbm_nusselt_sums sum only
 * them.  lbm_run and batches do not take slabs.
 *
 * After every lbm_step(h, 1) of all slabs, each interface is exchanged:
 * lbm_halo_pack(lower, 1, buf) and lbm_halo_pack(upper, 0, buf') copy the
 * slabs' boundary layers of every population plane into device buffers of
 * lbm_halo_size bytes (2D: (Q+QT) x nx values of the storage type, 14 x nx;
 * 3D: (Q+QT) x (padded row pitch x ny), 26 slices); once both copies are
 * complete (they run on each handle's stream), lbm_halo_unpack(upper, 0, buf)
 * and lbm_halo_unpack(lower, 1, buf') write them into the neighbours' ghost
 * layers.  The buffers may move between devices or ranks (peer copy, NCCL) in
 * between.  side 0 is the low end of the split axis, 1 the high end; a side
 * without a neighbour (a wall) is an error. */
int lbm_create_slab(const lbm_params *p, const double *x, const double *y, const double *z, int32_t lo, int32_t hi,
                    lbm_handle **out);
int lbm_halo_size(const lbm_handle *h, int64_t *bytes);
int lbm_halo_pack(lbm_handle *h, int32_t side, void *dev_buf);
int lbm_halo_unpack(lbm_handle *h, int32_t side, const void *dev_buf);

/* The sums behind lbm_check (sum |du|^2, sum |u|^2, sum dT^2, sum T^2, over
 * the handle's own layers; the previous fields are updated as by lbm_check) and
 * behind lbm_nusselt (sum Nu_hot w, sum Nu_cold w, sum w), so that slabs
 * combine them: errorU = sqrt(sum of the first) / sqrt(sum of the second)
 * (2M:784), Nu = sum / sum.  No counterpart beyond check() itself. */
int lbm_check_sums(lbm_handle *h, double sums[4]);
int lbm_nusselt_sums(lbm_handle *h, double sums[3]);

/* Copy the macroscopic fields to host arrays a(nx,ny[,nz]); any pointer may
 * be NULL; w is ignored in 2D.  Replaces gather_data (2M:807-816). */
int lbm_get_macro(lbm_handle *h, double *rho, double *u, double *v,
                  double *w, double *T);

/* Overwrite the macroscopic fields (an exact restart is set_populations
 * followed by set_macro with the saved fields).  NULL pointers keep the
 * current field. */
int lbm_set_macro(lbm_handle *h, const double *rho, const double *u,
                  const double *v, const double *w, const double *T);

/* Populations after the last completed iteration (post-streaming, post
 * boundary, pre-collision: the reference's f and g arrays) in the Fortran
 * layout f(0:Q-1,nx,ny[,nz]), g(0:QT-1,nx,ny[,nz]).  Either may be NULL. */
int lbm_get_populations(lbm_handle *h, double *f, double *g);

/* Load populations (same layout).  The macroscopic fields are recomputed
 * from them (rho = sum f, T = sum g, u from the momentum with half the
 * buoyancy force of the loaded state); call lbm_set_macro afterwards to
 * restore the exact carried state of a checkpoint. */
int lbm_set_populations(lbm_handle *h, const double *f, const double *g);

/* Tuning options of a handle (no counterpart in the reference): see
 * LBM_OPT_*.  lbm_get_option reports the value in effect (the kernel the
 * automatic choice picked, the block count used). */
int lbm_set_option(lbm_handle *h, int32_t option, int64_t value);
int lbm_get_option(const lbm_handle *h, int32_t option, int64_t *value);

/* Convert the cavity's state to another population storage (LBM_STORE_*) in
 * place, on the device: new buffers, the newest populations and carried
 * force converted, the check history kept (a mixed-precision run switches
 * from FP32 to FP64 this way).  Exact mode stays FP64; a batch member uses
 * lbm_batch_set_storage.  No counterpart in the reference (FP64 throughout). */
int lbm_set_storage(lbm_handle *h, int32_t storage);

/* Wait for all work of the handle; reports LBM_ERR_TIMEOUT if a kernel's
 * bounded wait gave up since the last synchronisation. */
int lbm_synchronize(lbm_handle *h);

/* The handle's CUDA stream as an opaque pointer (cudaStream_t). */
int lbm_stream(const lbm_handle *h, void **stream);

/* Device bytes the handle holds. */
int lbm_device_bytes(const lbm_handle *h, int64_t *bytes);

/* Number of kernels this library launched since load (all handles). */
int64_t lbm_kernel_launches(void);

/* ------------------------------------------------------------------------ */
/* Batches of independent cavities (no counterpart in the reference, which  */
/* runs one cavity per program; each member behaves as the reference's      */
/* program main would on its own parameters).                               */
/* ------------------------------------------------------------------------ */
typedef struct lbm_batch lbm_batch;

#define LBM_BATCH_OPT_TILE        1  /* tile width of the 2D batch kernel: 32, 64, 128 (3D: 32 x 4) */
#define LBM_BATCH_OPT_NBLOCKS     2  /* persistent blocks (0 = one full wave) */
#define LBM_BATCH_OPT_PERSISTENT  3  /* 1: one persistent kernel per step (2D and 3D; a 3D batch with a
                                        member whose ny % 4 == 1, or whose tile rows were changed,
                                        steps per member), 0: one launch per cavity */
#define LBM_BATCH_OPT_GRAPHS      4  /* 1: replay steps from CUDA graphs */
#define LBM_BATCH_OPT_GROWTH      5  /* lbm_batch_run stops a member whose residual is not finite or
                                        exceeds this factor x its smallest one in the run and reports
                                        it as converged = -1 (0, the default: off, a non-finite
                                        residual ends the run with LBM_ERR_NONFINITE) */
#define LBM_BATCH_OPT_STORAGES    6  /* the storages lbm_batch_tune may choose, as a mask of
                                        1 << LBM_STORE_*: the caller's accuracy rule (FP32 and FP64 for
                                        the transient of a run, FP64 alone to finish it); 0 (the
                                        default): the batch's current storage only */
#define LBM_BATCH_OPT_STORAGE     7  /* read only: the batch's current storage (LBM_STORE_*) */
#define LBM_BATCH_OPT_PDL         8  /* as LBM_OPT_PDL for the batch's step kernels (default 1; a step
                                        with both storages present forks onto two streams and is
                                        launched in plain stream order) */

/* Create n cavities (same dim, storage, mode and device; any size and
 * parameters).  x[i], y[i], z[i] are the coordinate arrays of cavity i as for
 * lbm_create; z may be NULL in 2D. */
int lbm_batch_create(int32_t n, const lbm_params *params, const double *const *x,
                     const double *const *y, const double *const *z, lbm_batch **out);
int lbm_batch_destroy(lbm_batch *b);
int lbm_batch_size(const lbm_batch *b, int32_t *n);
/* Member i as an ordinary handle (init, check, getters); it runs on the
 * batch's stream.  Do not destroy it. */
int lbm_batch_cavity(lbm_batch *b, int32_t i, lbm_handle **h);
/* lbm_init_reference on every member. */
int lbm_batch_init_reference(lbm_batch *b);
/* nsteps iterations of every member (lbm_step semantics; asynchronous). */
int lbm_batch_step(lbm_batch *b, int32_t nsteps);
/* Per-member check() residuals / Nusselt numbers into arrays of n. */
int lbm_batch_check(lbm_batch *b, double *errU, double *errT);
int lbm_batch_nusselt(lbm_batch *b, double *nu_hot, double *nu_cold);
/* The reference's loop for every member (2M:307-330): step check_every
 * iterations, check, and retire members whose errorU and errorT are both at
 * most eps; stop when all are retired or after max_steps.  converged[i] and
 * steps_done[i] (optional) report each member's outcome.  The stop test runs
 * on the device after each check: a stopped member's kernels become no-ops at
 * once, and the host reads all members' state (one copy, one
 * synchronisation) once every four checks to shrink the work list. */
int lbm_batch_run(lbm_batch *b, int32_t max_steps, int32_t check_every, double eps,
                  int32_t *converged, int64_t *steps_done);
/* lbm_batch_run over the members with mask[i] != 0 only (the others are not
 * stepped); mask NULL selects every member.  With LBM_BATCH_OPT_GROWTH set,
 * converged[i] = -1 marks a member stopped for a diverging residual (the
 * warm-start driver restarts those from the conduction state). */
int lbm_batch_run_masked(lbm_batch *b, const int32_t *mask, int32_t max_steps, int32_t check_every,
                         double eps, int32_t *converged, int64_t *steps_done);
/* Mixed precision, member by member: every member on the mask starts in FP32
 * storage and runs to errorU, errorT <= switch_eps; each member that gets
 * there is converted alone to FP64 in place (its FP64 finish overlaps the
 * others' FP32 transients) and runs on to eps, so its result is the FP64
 * fixed point.  max_steps bounds each member's iterations over both phases;
 * steps_low[i] (optional) reports its FP32 iterations; converged[] and
 * LBM_BATCH_OPT_GROWTH as lbm_batch_run_masked.  Members may end in different
 * storages (LBM_BATCH_OPT_STORAGE then reports -1).  Not in exact mode.  No
 * counterpart in the reference (FP64 throughout). */
int lbm_batch_run_mixed(lbm_batch *b, const int32_t *mask, int32_t max_steps, int32_t check_every,
                        double switch_eps, double eps, int32_t *converged, int64_t *steps_done,
                        int64_t *steps_low);
/* The autotuner: time each storage LBM_BATCH_OPT_STORAGES allows (the
 * batch's state is converted in place, lbm_batch_set_storage) x each tile
 * width and grid size on the batch itself (the timed steps advance the
 * members) and keep the fastest; reports the tile, grid and rate
 * (lbm_batch_get_option(LBM_BATCH_OPT_STORAGE) the storage).  No counterpart
 * in the reference. */
int lbm_batch_tune(lbm_batch *b, int32_t steps, int32_t *tile, int32_t *nblocks, double *mlups);
/* Convert every member's state to another population storage in place, on
 * the device (new buffers; the newest populations and carried force
 * converted; the check history kept).  Exact mode stays FP64.  No
 * counterpart in the reference (FP64 throughout). */
int lbm_batch_set_storage(lbm_batch *b, int32_t storage);
int lbm_batch_set_option(lbm_batch *b, int32_t option, int64_t value);
int lbm_batch_get_option(const lbm_batch *b, int32_t option, int64_t *value);
int lbm_batch_synchronize(lbm_batch *b);
int lbm_batch_stream(const lbm_batch *b, void **stream);

/* The check() residuals for callers that cannot allocate device memory.
 * No counterpart in the reference: it is check() (2M:755-805) on the
 * caller's own device arrays, for hosts that own all device memory (a
 * Fortran code keeping its fields in OpenACC / CUDA Fortran arrays inside a
 * reserved pool, a loop that must not trigger an allocation).  It allocates
 * nothing: the per-block partial sums go to a fixed 256 KiB array in device
 * memory that every GPU using this library holds until the process exits.
 * u, v, T (and w in 3D) are device arrays of n doubles; u_prev, v_prev, T_prev
 * (and w_prev) hold the fields of the previous check and are overwritten with
 * the current ones; w and w_prev are NULL in 2D.  n may be at most
 * LBM_NOALLOC_MAX_NODES; larger n is rejected with LBM_ERR_PARAM.  Work runs
 * on `stream` (a cudaStream_t, NULL for the default stream); the call waits
 * for it and writes errU, errT on the host.  The first call on each device
 * looks up the array's device address; make it before any stream capture.
 * Calls share the array: calls that overlap on the GPU race. */
#define LBM_NOALLOC_MAX_NODES 67108864LL
int lbm_check_noalloc(const double *u, const double *v, const double *w,
                      const double *T, double *u_prev, double *v_prev,
                      double *w_prev, double *T_prev, int64_t n,
                      double *errU, double *errT, void *stream);

/* The 3D march kernel's work plan (host code, no device needed), for tools
 * and tests that check it: ntiles tile columns of nz slices over `nblocks`
 * persistent blocks, kind as LBM_OPT_PLAN.  On entry *seg_count is the
 * capacity of segs (in segments); on return the number of segments.  segs
 * receives (tile, first slice, end slice) per segment, off (blocks_used + 1
 * entries) each block's first segment.  segs or off NULL: size query only.
 * No reference counterpart (the reference runs one MPI rank per subdomain). */
int lbm_march_plan3d(int32_t ntiles, int32_t nz, int32_t nblocks, int32_t kind,
                     int32_t *seg_count, int32_t *segs, int32_t *off,
                     int32_t *blocks_used);

#ifdef __cplusplus
}
#endif

#endif /* LBM_B200_H */
