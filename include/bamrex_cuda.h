/*
 * bamrex_cuda.h -- C ABI of libbamrex_cuda.so, the B200 (sm_100a) explicit
 * finite-volume path of BAMReX: MUSCL-Hancock reconstruction with half-step
 * evolution, HLLC / SLIC(FORCE) / FORCE / Lax-Friedrichs interface fluxes,
 * the split conservative update, boundary/ghost fill and the CFL reduction.
 *
 * Plain C types only: device pointers are `double *`, streams are `void *`
 * (a cudaStream_t; NULL = the legacy default stream).  Every entry point
 * returns an int status (BAMREX_OK = 0) and never throws; a human-readable
 * message for the last failure on the calling thread is available from
 * bamrex_last_error().  Reference citations are paths inside the BAMReX tree.
 */
#ifndef BAMREX_CUDA_H_
#define BAMREX_CUDA_H_

#if defined(__GNUC__)
#define BAMREX_API __attribute__((visibility("default")))
#else
#define BAMREX_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define BAMREX_ABI_VERSION 4
/* MAX_NCOMP = PUInd::size (Source/System/Parm.H:9) */
#define BAMREX_MAX_NCOMP 8

/* ---- status codes (the reference aborts instead: amrex::Abort / AMREX_ASSERT,
 *      Source/AmrLevelAdv_advance.cpp:133-137, 182-185) ---- */
enum {
    BAMREX_OK = 0,
    BAMREX_ERR_ARG = 1,         /* bad argument, box/fab geometry or layout */
    BAMREX_ERR_OOM = 2,         /* device or host allocation failed */
    BAMREX_ERR_NAN = 3,         /* non-finite wave speed / time step */
    BAMREX_ERR_TIMEOUT = 4,     /* a bounded device wait gave up */
    BAMREX_ERR_CUDA = 5,        /* a CUDA runtime call failed */
    BAMREX_ERR_UNSUPPORTED = 6, /* method/option not provided by this build */
    BAMREX_ERR_NOT_CONVERGED = 7 /* an iterative solve did not reach its tolerance */
};

/* ---- numerical method, same values as NumericalMethods::Method
 *      (Source/NumericalMethods.H:10-19) ---- */
enum {
    BAMREX_MUSCL_HANCOCK = 0,
    BAMREX_HLLC = 1,
    BAMREX_IMEX = 2, /* not a level method: the IMEX step is bamrex_imex (below) */
    BAMREX_RCM = 3,  /* not on this path: BAMREX_ERR_UNSUPPORTED */
    BAMREX_SLIC = 4,
    BAMREX_FORCE = 5,
    BAMREX_LAX_FRIEDRICHS = 6
};

/* ---- slope limiter, AMREX_ENUM(Limiter, ...) order (Source/Fluxes/Limiters.H:13) ---- */
enum { BAMREX_MINBEE = 0, BAMREX_VAN_LEER = 1, BAMREX_VAN_ALBADA = 2, BAMREX_SUPERBEE = 3 };

/* ---- domain boundary kind (BAMReXBCType; Source/BoundaryConditions/BCs.cpp:226-266):
 *      transmissive = foextrap, periodic = int_dir, reflective = reflect_even
 *      with reflect_odd on the normal momentum ---- */
enum { BAMREX_BC_TRANSMISSIVE = 0, BAMREX_BC_PERIODIC = 1, BAMREX_BC_REFLECTIVE = 2 };

/* ---- level state precision: FP64 (the drop-in), or FP32 storage with FP32
 *      fluxes (the CFL/dt reduction and the conserved sums stay FP64) ---- */
enum { BAMREX_FP64 = 0, BAMREX_FP32_STORAGE = 1 };

/* amrex::Box: cell-centred, inclusive lo/hi; unused dimensions are 0..0. */
typedef struct bamrex_box {
    int lo[3];
    int hi[3];
} bamrex_box;

/* amrex::Array4<Real>: element (i,j,k,n) lives at
 * p[(i-begin[0]) + (j-begin[1])*jstride + (k-begin[2])*kstride + n*nstride];
 * end[] is exclusive.  p is a device pointer. */
typedef struct bamrex_array4 {
    double *p;
    long long jstride;
    long long kstride;
    long long nstride;
    int begin[3];
    int end[3];
    int ncomp;
} bamrex_array4;

/* Parm POD (Source/System/Parm.H:14-61), field for field. */
typedef struct bamrex_parm {
    double adiabatic;
    double eos_mu;
    double Pr;
    double beta;
    double eta_prime;
    double T_prime;
    double S_eta;
    double epsilon;
    double Re;
    double R_spec;
    double cv;
    double cp;
    double adia[9];
    double Reinv;
    int limiter;
    unsigned int limiter_indices[BAMREX_MAX_NCOMP];
    unsigned char limit_on_primv[BAMREX_MAX_NCOMP];
    unsigned char need_primitive_for_limiting;
} bamrex_parm;

/* Library identity and errors. */
BAMREX_API int bamrex_abi_version(void);
/* Device memory of destroyed levels, couplings and bodies stays in the
 * library's pool for the next ones (blocks of 64 MiB and more kept whole, to
 * be handed out again as they are), and the pinned host buffer that stages
 * table uploads is kept too; this hands all of it that no live object uses
 * back to the driver (e.g. before a memory-hungry phase of the caller). */
BAMREX_API int bamrex_release_memory(void);
BAMREX_API const char *bamrex_last_error(void);
BAMREX_API const char *bamrex_status_string(int status);

/* Host-side region timers (the reference's BL_PROFILE scopes under AMReX's
 * TinyProfiler, e.g. Source/AmrLevelAdv_advance.cpp:24, Source/main.cpp:21):
 * wall time per named phase of level creation, regrid, coarse steps.  Off by
 * default; on with bamrex_profile_enable(1) or the environment variable
 * BAMREX_TINY_PROFILE=1.  enable returns the previous setting.  The report
 * is text, one region per line after a header, "name calls total_s avg_ms
 * max_ms", sorted by total time; *needed is its size with the terminating
 * NUL, and at most cap - 1 characters are written. */
BAMREX_API int bamrex_profile_enable(int on);
BAMREX_API int bamrex_profile_reset(void);
BAMREX_API int bamrex_profile_report(char *out, int cap, int *needed);

/* FluidSystem::set_parm_defaults (Source/System/FluidSystem.cpp:52-71) for a
 * spacedim-dimensional fluid (limiting variable = energy, UInd::E = 1+D). */
BAMREX_API int bamrex_parm_set_defaults(bamrex_parm *parm, int spacedim);
/* FluidSystem::init_parm (Source/System/FluidSystem.cpp:73-101): derived
 * quantities adia[], R_spec, cv, cp, Reinv, need_primitive_for_limiting. */
BAMREX_API int bamrex_parm_init(bamrex_parm *parm);

/* ------------------------------------------------------------------ */
/* Per-box flux and update (the Fluxes.H call surface)                 */
/* ------------------------------------------------------------------ */

/* compute_{MUSCL_hancock,HLLC,SLIC,force,LF}_flux(int dir, Real time,
 * const Box& bx, const Array4<Real>& flux, const Array4<const Real>& consv,
 * GpuArray<Real,D> const& dx, Real dt, const System*, const Parm* h_parm,
 * const Parm* d_parm)  -- Source/Fluxes/Fluxes.H:35-56, 98-119, 131-152,
 * 206-227, 237-257.  Selected by method (BAMREX_MUSCL_HANCOCK, BAMREX_HLLC,
 * BAMREX_SLIC, BAMREX_FORCE, BAMREX_LAX_FRIEDRICHS).
 * bx: the valid box; flux must cover surroundingNodes(bx, dir); consv must
 * cover bx grown by 2 (MUSCL-Hancock, SLIC) or 1 (first-order methods) in dir.
 * Asynchronous on `stream`. */
BAMREX_API int bamrex_compute_flux(int method, int dir, int spacedim, double time, const bamrex_box *bx,
                        bamrex_array4 flux, bamrex_array4 consv, const double dx[3], double dt,
                        const bamrex_parm *parm, void *stream);

/* compute_HLLC_flux_LR / compute_force_flux_LR with separate left/right
 * arrays (Source/Fluxes/Fluxes.H:79-87, 179-187): the face between i-1 and
 * i takes consv_L at i-1 and consv_R at i.  kind: BAMREX_HLLC or BAMREX_FORCE. */
BAMREX_API int bamrex_compute_flux_LR(int kind, int dir, int spacedim, double time, const bamrex_box *bx,
                           bamrex_array4 flux, bamrex_array4 consv_L, bamrex_array4 consv_R,
                           const double dx[3], double dt, const bamrex_parm *parm, void *stream);

/* The per-sweep conservative update of AmrLevelAdv::advance_explicit
 * (Source/AmrLevelAdv_advance.cpp:330-341):
 * Uout(i) = Uin(i) - (dt/dx[dir]) * (flux(i+1) - flux(i)) on bx. */
BAMREX_API int bamrex_sweep_update(int dir, int spacedim, const bamrex_box *bx, bamrex_array4 Uout,
                        bamrex_array4 Uin, bamrex_array4 flux, const double dx[3], double dt,
                        void *stream);

/* Unsplit conservative_update(bx, statein, fx, fy, fz, stateout, dt, idx)
 * (Source/Fluxes/Update.H:99-130); fluxes[d] for d < spacedim. */
BAMREX_API int bamrex_conservative_update(int spacedim, const bamrex_box *bx, bamrex_array4 out,
                               bamrex_array4 in, const bamrex_array4 *fluxes, double dt,
                               const double idx[3], void *stream);

/* Fused per-box sweep: the flux of `method` in direction dir and the sweep
 * update in one kernel (compute_*_flux + AmrLevelAdv_advance.cpp:330-341).
 * If flux.p is non-NULL the face fluxes are also written (reflux input). */
BAMREX_API int bamrex_sweep_box(int method, int dir, int spacedim, const bamrex_box *bx, bamrex_array4 Uout,
                     bamrex_array4 Uin, bamrex_array4 flux, const double dx[3], double dt,
                     const bamrex_parm *parm, void *stream);

/* ------------------------------------------------------------------ */
/* Level: every box of one AMR level in one device box table            */
/* ------------------------------------------------------------------ */

typedef struct bamrex_level bamrex_level;

typedef struct bamrex_level_desc {
    int spacedim;           /* 1, 2 or 3 */
    bamrex_box domain;      /* the level's index domain (Geometry::Domain) */
    double prob_lo[3];
    double prob_hi[3];
    int bc_lo[3];           /* BAMREX_BC_* per direction */
    int bc_hi[3];
    const bamrex_box *boxes; /* the level's BoxArray (disjoint, inside domain) */
    int nboxes;
    int ngrow;              /* ghost width of the state fabs, >= 2 (NUM_GROW) */
    int method;             /* BAMREX_MUSCL_HANCOCK ... (adv.num_method) */
    double cfl;             /* adv.cfl */
    bamrex_parm parm;
    int x_segment;          /* cells per warp item in x; 0 = automatic */
    int s_segment;          /* cells per thread item in y/z; 0 = automatic */
    int precision;          /* BAMREX_FP64 (0) or BAMREX_FP32_STORAGE */
    int x_mode;             /* BAMREX_XSWEEP_*: kernel of the x sweep; 0 = automatic */
    int staging;            /* BAMREX_STAGING_*: how sweeps stage their input; 0 = automatic */
    int staging_dir[3];     /* per direction, overriding `staging` where not 0 */
} bamrex_level_desc;

/* How a level's sweeps bring their input on chip and share the stencil.
 * REGISTERS: the marching and row kernels load through L2 and carry each
 * line's stencil in registers (every configuration).  TMA: a warp marches
 * 32 lines, its tiles (positions x 32 lines x components) arriving by tiled
 * tensor loads into shared memory, several in flight.  WAVE: a block of 8
 * warps walks 32 lines (8 rows in x) in passes, one position per thread,
 * its tiles arriving by tensor loads; cell stages and face fluxes pass
 * between threads through shared memory.  TMA and WAVE serve the fast
 * MUSCL-Hancock path in 2D and 3D (energy limiting, gamma with 1/z = 7);
 * other configurations refuse them with BAMREX_ERR_UNSUPPORTED.  AUTO: per
 * direction the kind with the least estimated time on the level's boxes (a
 * slot-step count, warm-up and idle lanes included, times a time per
 * slot-step measured on the B200).  All evaluate the same scheme per cell
 * (results agree to rounding). */
enum {
    BAMREX_STAGING_AUTO = 0,
    BAMREX_STAGING_REGISTERS = 1,
    BAMREX_STAGING_TMA = 2,
    BAMREX_STAGING_WAVE = 3
};

/* Kernel of a level's x sweep.  ROWS: a warp marches along a row segment,
 * lanes on consecutive cells (best for wide boxes: it spends two extra
 * 32-cell chunks per row segment).  MARCH: each thread marches one row,
 * lanes on 32 adjacent rows (best for levels of narrow boxes, such as
 * max_grid_size 32-128).  AUTO picks by an estimate of the lane slots each
 * spends on the level's boxes.  Both evaluate the same scheme per cell
 * (results agree to rounding: multiply-add contraction may differ). */
enum {
    BAMREX_XSWEEP_AUTO = 0,
    BAMREX_XSWEEP_ROWS = 1,
    BAMREX_XSWEEP_MARCH = 2
};

/* Build the level: allocates the state fabs (two time-level buffers with
 * ghost cells, 256-byte aligned rows), the device box table, ghost-fill
 * tables and a small scalar block, all at creation (no allocation per step).
 * Work is issued on `stream`; with stream NULL the level creates and owns a
 * non-blocking stream of its own (bamrex_level_stream returns it). */
BAMREX_API int bamrex_level_create(bamrex_level **out, const bamrex_level_desc *desc, void *stream);
BAMREX_API int bamrex_level_destroy(bamrex_level *level);
BAMREX_API const char *bamrex_level_last_error(const bamrex_level *level);

/* The stream the level issues its work on (the one given at creation, or
 * the level's own non-blocking stream when that was NULL). */
BAMREX_API void *bamrex_level_stream(const bamrex_level *level);

/* The x-sweep kernel the level runs: BAMREX_XSWEEP_ROWS or _MARCH. */
BAMREX_API int bamrex_level_x_mode(const bamrex_level *level);
/* The kernel of the sweep of direction dir: BAMREX_STAGING_REGISTERS, _TMA
 * or _WAVE (negative on a bad argument). */
BAMREX_API int bamrex_level_staging(const bamrex_level *level, int dir);

/* Number of valid cells, and the Array4 of box b of the current state.
 * bamrex_level_fab returns BAMREX_ERR_UNSUPPORTED for an FP32-storage level:
 * its fabs hold floats, and bamrex_array4 describes doubles only. */
BAMREX_API long long bamrex_level_num_cells(const bamrex_level *level);
BAMREX_API int bamrex_level_fab(const bamrex_level *level, int box, bamrex_array4 *out);

/* Copy the valid cells of every box in from / out to a packed buffer
 * (box-major; inside a box component-slowest, i-fastest; NCOMP*num_cells
 * doubles).  `src`/`dst` may be host (pinned or pageable) or device memory. */
BAMREX_API int bamrex_level_copy_in(bamrex_level *level, const double *src);
BAMREX_API int bamrex_level_copy_out(bamrex_level *level, double *dst);

/* Conserved totals sum(U) * cell volume per component over the valid cells
 * of the current state, accumulated in FP64 in a fixed order (per box, then
 * boxes in order), so repeated calls agree bit for bit.  totals: NCOMP
 * doubles.  Synchronises the stream. */
BAMREX_API int bamrex_level_conserved_sums(bamrex_level *level, double *totals);

/* The same totals for caller-owned fabs (box b's valid cells in fabs[b],
 * FP64), computed without any device allocation: this entry point has no
 * counterpart in the reference.  It serves callers that must not have a
 * library allocate device memory for them (a host code whose own arena owns
 * the GPU's memory, or an error path that no longer trusts the allocator).
 * All scratch lives in one fixed file-scope device array: at most 4096
 * boxes per call (larger counts are rejected with BAMREX_ERR_ARG).  The
 * first call on each device looks up that array's address
 * (cudaGetSymbolAddress) and must come before any stream capture; the
 * address is kept for the life of the process, so the function must not be
 * called after a cudaDeviceReset of that device.  Calls
 * that overlap in time share the array and race: serialise them.  Issues
 * its work on `stream` and synchronises it.  totals: NCOMP doubles, equal
 * bit for bit to bamrex_level_conserved_sums on a level's own fabs. */
BAMREX_API int bamrex_conserved_sums_noalloc(int spacedim, const bamrex_box *boxes, const bamrex_array4 *fabs,
                                             int nboxes, const double dx[3], double *totals, void *stream);

/* Wait for all work the level issued on its stream. */
/* One step of a host-resident state: host_in -> host_out (packed layout of
 * bamrex_level_copy_in/out; the same pointer for both is allowed), time step
 * dt, and the CFL estimate of the result in *dt_next (may be NULL) -- the
 * result of bamrex_level_copy_in + bamrex_level_advance + copy_out +
 * est_time_step.  Single-box levels (2D/3D, not periodic in the last
 * direction) are streamed in nslabs slabs along the last direction so that
 * uploads, sweeps and downloads overlap (pinned host buffers for the
 * overlap; one strided copy per slab and direction); nslabs <= 0 picks slabs
 * of at least 16 MiB per component (2 to 64 of them), since smaller copies
 * lose PCIe bandwidth when both directions run at once.  Other levels take
 * the plain sequence.  Synchronous. */
BAMREX_API int bamrex_level_step_host(bamrex_level *level, const double *host_in, double *host_out, double dt,
                                      int nslabs, double *dt_next);
/* nsteps steps of a host-resident state in place (host: packed layout),
 * each one a host round trip as bamrex_level_step_host, the first with time
 * step dt0 and the next ones with the CFL estimate of their input computed
 * on the device; step k + 1's upload of a slab starts as soon as step k has
 * downloaded it, so the copies of consecutive steps overlap.  *time_io
 * advances by the steps' dt; *dt_next (may be NULL) is the estimate for the
 * step after the last.  Levels that cannot be streamed take one plain host
 * step after the other.  Synchronous. */
BAMREX_API int bamrex_level_run_host(bamrex_level *level, double *host, int nsteps, double dt0, int nslabs,
                                     double *time_io, double *dt_next);
/* The number of slabs bamrex_level_step_host / bamrex_level_run_host stream
 * the level in for this nslabs (0: the level is not streamed and takes the
 * plain sequence).  No reference counterpart: the reference keeps its state
 * on the host and has no host round trip to schedule. */
BAMREX_API int bamrex_level_host_slabs(const bamrex_level *level, int nslabs, int *slabs);
BAMREX_API int bamrex_level_sync(bamrex_level *level);

/* bamrexBCData::fill_consv_boundary on the current state
 * (Source/BoundaryConditions/BCs.cpp:429-442): inter-box ghosts and
 * transmissive / periodic / reflective domain ghosts (all directions). */
BAMREX_API int bamrex_level_fill_boundary(bamrex_level *level);

/* AmrLevelAdv::advance(time, dt, iteration, ncycle) for the explicit methods
 * (Source/AmrLevelAdv.H:110-111, Source/AmrLevelAdv_advance.cpp:21-259,
 * 261-439): ghost fill, one split sweep per direction in x, y, z order with a
 * ghost fill after each, the result becoming the current state.  The
 * max wave speed of the new state is reduced inside the last sweep.
 * Asynchronous; returns the dt used in *dt_out (may be NULL). */
BAMREX_API int bamrex_level_advance(bamrex_level *level, double time, double dt, int iteration, int ncycle,
                         double *dt_out);

/* AmrLevelAdv::estTimeStep (Source/AmrLevelAdv.cpp:395-477) on the current
 * state: cfl * min_d dx_d / max(|u| + c).  Synchronises the stream.  On a
 * level with a rigid body it also reports what the fills since the last
 * call recorded: BAMREX_ERR_ARG when an interface's interpolation stencil
 * left the fab (ngrow too small), BAMREX_ERR_NOT_CONVERGED when an exact
 * Riemann solve at the interface took its 200 Newton iterations. */
BAMREX_API int bamrex_level_est_time_step(bamrex_level *level, double *dt_est);

/* The coarse-step loop of a single-level run (Amr::coarseTimeStep with
 * AmrLevelAdv::computeInitialDt / computeNewDt, Source/AmrLevelAdv.cpp:487-619):
 * up to nsteps steps, dt computed on the device after every step with the
 * stop-time clamp (stop_time < 0 disables it; steps stop once time reaches
 * it).  With use_graph != 0 one step is captured as a CUDA graph and
 * replayed.  On return (stream synchronised) *time_io holds the new time and
 * *steps_done the number of steps taken.  *time_io is the start time on entry. */
BAMREX_API int bamrex_level_run(bamrex_level *level, int nsteps, double stop_time, int use_graph, double *time_io,
                     int *steps_done);

/* The same loop split in two: bamrex_level_run_async issues the steps and
 * returns at once (no host synchronisation); bamrex_level_run_wait
 * synchronises the stream and reports the time and steps taken.  Between
 * the two calls the caller may record its own events on the level's stream. */
BAMREX_API int bamrex_level_run_async(bamrex_level *level, int nsteps, double stop_time, int use_graph,
                                      double start_time);
BAMREX_API int bamrex_level_run_wait(bamrex_level *level, double *time_out, int *steps_done);

/* Kernel accounting for measurement: kernels launched by the level since
 * creation / the last reset, and (when timing is enabled) the summed
 * CUDA-event time of the sweep kernels and their count. */
BAMREX_API int bamrex_level_set_timing(bamrex_level *level, int enable);
BAMREX_API int bamrex_level_counters(bamrex_level *level, long long *launches, double *sweep_ms, long long *sweep_launches);
BAMREX_API int bamrex_level_reset_counters(bamrex_level *level);
/* The timed sweep kernels split by direction: summed milliseconds and
 * launches for x, y, z (arrays of 3). */
BAMREX_API int bamrex_level_sweep_times(bamrex_level *level, double *ms_by_dir, long long *launches_by_dir);

/* ------------------------------------------------------------------ */
/* A level split over processes (one GPU per rank)                      */
/* ------------------------------------------------------------------ */

/* A level created with only this rank's boxes fills the ghosts those boxes
 * can fill themselves (copies between local boxes, physical boundaries);
 * the cells that come from other ranks' boxes travel through these buffers.
 * This is the FillBoundary step of bamrexBCData::fill_consv_boundary, run
 * after every sweep (Source/AmrLevelAdv_advance.cpp:356), across ranks. */
typedef struct bamrex_region {
    int box;            /* index into the level's boxes */
    int lo[3], hi[3];   /* cells of that box's fab (valid or ghost) */
    long long offset;   /* first cell in the buffer; regions are packed in order */
} bamrex_region;

/* Direction dir's send regions (valid cells read into the send buffer) and
 * receive regions (ghost cells written from the receive buffer).  A buffer
 * holds, region after region, NCOMP x (region cells) doubles, component
 * slowest: value (cell c, component n) of a region at offset o is at
 * buf[o*NCOMP + n*cells + c]. */
BAMREX_API int bamrex_level_set_halo(bamrex_level *level, int dir, const bamrex_region *send, int nsend,
                                     const bamrex_region *recv, int nrecv);
/* Device buffers, asynchronous on the level's stream. */
BAMREX_API int bamrex_level_halo_pack(bamrex_level *level, int dir, double *sendbuf);
BAMREX_API int bamrex_level_halo_unpack(bamrex_level *level, int dir, const double *recvbuf);
/* The step one piece at a time: ghost fill of direction dir, then its sweep
 * (reduce_ws != 0 also reduces the max wave speed of the result); after the
 * last direction the level's current state is the new time level. */
BAMREX_API int bamrex_level_fill_dir(bamrex_level *level, int dir);
BAMREX_API int bamrex_level_sweep_dir(bamrex_level *level, int dir, double dt, int reduce_ws);
/* Max wave speed |u| + c over this rank's valid cells (from the last sweep
 * that reduced it, else computed); synchronises the stream. */
BAMREX_API int bamrex_level_wave_speed(bamrex_level *level, double *ws);

/* The split step with the time step kept on the device, so a host driver
 * never waits inside a run.  dist_begin uploads the start time and the stop
 * time (< 0: none) and reduces this rank's max wave speed; per step the
 * driver enqueues, in order: wave_speed_async (this rank's max wave speed,
 * a double, copied to dst_device on the level's stream), an all-reduce MAX
 * of that buffer over the ranks (e.g. NCCL on the level's stream), dist_dt
 * (dt from the global max: estTimeStep with the stop-time clamp of
 * computeInitialDt / computeNewDt, Source/AmrLevelAdv.cpp:395-477,
 * 513-523, 600-611; first != 0 before the first step, 0 after each step,
 * which also advances the time and step count), then for every direction
 * the halo exchange, fill_dir_device and sweep_dir_device (the last with
 * reduce_ws != 0).  dist_end waits and returns the time, the next dt and
 * the steps taken; it reports a non-finite or non-positive dt the device
 * met.  Steps enqueued past the stop time do nothing. */
BAMREX_API int bamrex_level_dist_begin(bamrex_level *level, double time, double stop_time);
BAMREX_API int bamrex_level_wave_speed_async(bamrex_level *level, double *dst_device);
BAMREX_API int bamrex_level_dist_dt(bamrex_level *level, const double *ws_device, int first);
BAMREX_API int bamrex_level_fill_dir_device(bamrex_level *level, int dir);
BAMREX_API int bamrex_level_sweep_dir_device(bamrex_level *level, int dir, int reduce_ws);
/* Interior sweeps while halos travel (the MPI overlap of FillBoundary with
 * the MFIter loop of advance_explicit, Source/AmrLevelAdv_advance.cpp:356).
 * set_sweep_split lists the boxes (local indices) whose ghost cells in
 * direction dir come from other ranks; sweep_dir_device_part then sweeps
 * part 0 (every other box: no remote ghost cells, so it can run while the
 * exchange is in flight) or part 1 (the listed boxes, after the unpack),
 * with the arithmetic and kernels of bamrex_level_sweep_dir_device; part 1
 * completes the direction.  The split is set up once (synchronous). */
BAMREX_API int bamrex_level_set_sweep_split(bamrex_level *level, int dir, const int *boxes, int nboxes);
BAMREX_API int bamrex_level_sweep_dir_device_part(bamrex_level *level, int dir, int reduce_ws, int part);
BAMREX_API int bamrex_level_dist_end(bamrex_level *level, double *time, double *dt, int *steps);

/* ------------------------------------------------------------------ */
/* Rigid bodies by the ghost-fluid method                               */
/* ------------------------------------------------------------------ */

/* Signed-distance shapes (Source/Geometry/PlaneSDF.H, SphereSDF.H,
 * CylinderSDF.H); the level set is > 0 in the body, < 0 in the fluid. */
enum { BAMREX_SDF_PLANE = 0, BAMREX_SDF_SPHERE = 1, BAMREX_SDF_CYLINDER = 2 };
/* Two shapes combined (UnionSDF.H, IntersectionSDF.H). */
enum { BAMREX_SDF_UNION = 0, BAMREX_SDF_INTERSECTION = 1 };
/* RigidBodyBCType (Source/BoundaryConditions/BCTypes.H:50-57). */
enum { BAMREX_RB_REFLECTIVE = 0, BAMREX_RB_NO_SLIP = 1, BAMREX_RB_FOEXTRAP = 2 };
/* GFMFlag bits (Source/GFM/GFMFlag.H:10-21). */
enum { BAMREX_GFM_GHOST = 1, BAMREX_GFM_INTERFACE = 2, BAMREX_GFM_FILL = 4 };

typedef struct bamrex_sdf {
    int kind;          /* BAMREX_SDF_* */
    double center[3];  /* plane: a point of the plane; sphere, cylinder: centre */
    double axis[3];    /* plane: normal pointing out of the body; cylinder: axis (normalised here) */
    double radius;     /* sphere, cylinder */
    int fluid_inside;  /* sphere, cylinder: has_fluid_inside */
} bamrex_sdf;

typedef struct bamrex_body_desc {
    int nshapes;        /* 1 or 2 */
    int combine;        /* BAMREX_SDF_UNION / _INTERSECTION of shapes[0] and shapes[1] */
    bamrex_sdf shapes[2];
    int rb_bc;          /* BAMREX_RB_* (the reference default: reflective) */
    int stencil;        /* GFMFillInfo::stencil, 1..ngrow (default 2) */
    int fill_diagonals; /* GFMFillInfo::fill_diagonals */
} bamrex_body_desc;

/* Give the level a static rigid body (AmrLevelAdv::init_levelset + the
 * build_gfm_flags calls of AmrLevelAdv::initData, Source/AmrLevelAdv_LSinit.cpp:37-64,
 * Source/AmrLevelAdv.cpp:250-269): the level set on every cell of every fab
 * (fill_from_IF, cell centres), its normals on the fabs shrunk by one
 * (fill_ls_normals, Source/Geometry/Normals.cpp:12-54) and the GFM flags of the
 * valid cells (Source/GFM/GFMFlag.cpp:60-83), all on the device.  From then
 * on every bamrex_level_advance / _run starts with the rigid-body ghost fill
 * below (AmrLevelAdv_advance.cpp:110-116).  desc == NULL removes the body.
 * On a coupled AMR level the fill leaves the coarse/fine ghost cells as the
 * coupling's fill_patch set them. */
BAMREX_API int bamrex_level_set_body(bamrex_level *level, const bamrex_body_desc *desc); /* ngrow >= 4 */

/* The rigid-body ghost fill on the current state (FluidSystem::FillRBGhostCells
 * = fill_ghost_rb, Source/GFM/RigidBody.cpp:24-170, then fill_consv_boundary):
 * all ghost cells filled; interface ghost cells set from the state
 * interpolated at their reflection 1.5 dx into the fluid (reflective: exact
 * Riemann problem of the reflected normal velocity; no_slip: velocity
 * negated; foextrap: as interpolated); inter-box fill; spacedim + 1 rounds of
 * fast-sweeping extrapolation into the other body cells
 * (Source/GFM/Extrapolate.cc:9-37, Extrapolate.H, FastSweep.H), each followed
 * by the inter-box fill; then the boundary fill again.  Interface cells read
 * the state from before the fill (the reference writes them in place). */
BAMREX_API int bamrex_level_fill_body_ghosts(bamrex_level *level);

/* The level set (which = 0), normal component d (which = 1 + d) or the GFM
 * flags (which = -1) of every valid cell, as doubles in the packed order of
 * bamrex_level_copy_out.  Synchronises the stream. */
BAMREX_API int bamrex_level_body_field(bamrex_level *level, int which, double *out);

/* Interface ghost cells, and body cells swept by the extrapolation, of the level. */
BAMREX_API int bamrex_level_body_counts(const bamrex_level *level, long long *interface_cells, long long *swept_cells);

/* ------------------------------------------------------------------ */
/* AMR: coarse/fine coupling of two levels                              */
/* ------------------------------------------------------------------ */

/* Error estimation of AmrLevelAdv::errorEst (Source/AmrLevelAdv.cpp:711-832)
 * on the current state: grad_error (Source/Src_K/tagging_K.H:21-60) on
 * component grad_var (of the primitive vector if grad_var_is_primv) with the
 * relative threshold grad_threshold (skipped if <= 0), and state_error
 * (tagging_K.H:9-19) on err_var >= phierr (skipped if do_err == 0).  Ghost
 * cells one deep must be valid: the call fills the level's own inter-box and
 * physical ghosts; coarse/fine ghosts come from bamrex_coupling_fill_patch.
 * tags: num_cells chars (1 = refine) in the packed order of
 * bamrex_level_copy_out.  Synchronises the stream. */
BAMREX_API int bamrex_level_tag(bamrex_level *level, int grad_var, int grad_var_is_primv, double grad_threshold,
                                int do_err, int err_var, int err_var_is_primv, double phierr, char *tags);

/* Every criterion of AmrLevelAdv::errorEst (Source/AmrLevelAdv.cpp:711-832):
 * state_error and grad_error as bamrex_level_tag; box_error
 * (tagging_K.H:87-103): cells whose centre lies in [box_lo, box_hi] in every
 * direction; interface_error (tagging_K.H:62-72), on a level with a rigid
 * body: cells at the interface or with |level set| <= lstol.  On a level
 * with a rigid body, ghost_error (tagging_K.H:74-84) then clears the tags of
 * ghost (solid) cells not at the interface, as the reference does whenever
 * rigid bodies are enabled (bamrex_level_tag does the same). */
typedef struct bamrex_tag_desc {
    int do_err, err_var, err_var_is_primv;
    double phierr;
    int do_grad, grad_var, grad_var_is_primv;
    double phigrad;                  /* relative threshold */
    int do_box;
    double box_lo[3], box_hi[3];     /* physical coordinates (tagging.box_x/y/z) */
    int do_interface;
    double lstol;
} bamrex_tag_desc;
BAMREX_API int bamrex_level_tag_ex(bamrex_level *level, const bamrex_tag_desc *desc, char *tags);

/* The coupling of a coarse level and the next finer level (refinement ratio
 * 2 or 4).  It stands for the AMReX pieces the reference calls between two
 * AmrLevelAdv levels: the FluxRegister (FineAdd / CrseInit in
 * AmrLevelAdv::advance, Source/AmrLevelAdv_advance.cpp:236-254, Reflux in
 * AmrLevelAdv::reflux, Source/AmrLevelAdv.cpp:918-945), FillPatch /
 * FillPatcherFill with cell_cons_interp for the fine level's coarse/fine ghost
 * cells (AmrLevelAdv_advance.cpp:108), FillCoarsePatch for new fine data
 * (AmrLevelAdv.cpp:371), and average_down (AmrLevelAdv.cpp:947-987).
 *
 * Creation checks proper nesting (every coarse cell the fine level needs is a
 * valid coarse cell) and builds all tables.  From then on, every
 * bamrex_level_advance of the coarse level stores -dt*area*F at the
 * coarse/fine faces (CrseInit) and every advance of the fine level adds
 * dt*area*F of its faces (FineAdd), in the same kernels' stream order.  Both
 * levels must use the same stream.  Destroy the coupling before either
 * level. */
typedef struct bamrex_coupling bamrex_coupling;
BAMREX_API int bamrex_coupling_create(bamrex_coupling **out, bamrex_level *crse, bamrex_level *fine, int ref_ratio);
BAMREX_API int bamrex_coupling_destroy(bamrex_coupling *c);

/* Keep a copy of the coarse level's current state as its old time level
 * (StateData::swapTimeLevels at the start of AmrLevelAdv::advance) with the
 * times it spans, for time interpolation of fine ghost cells. */
BAMREX_API int bamrex_coupling_save_coarse_old(bamrex_coupling *c, double t_old, double t_new);

/* Fill the fine level's coarse/fine ghost cells (both state buffers) at
 * `time`: coarse data interpolated in time between the saved old state and
 * the current coarse state, then conservatively interpolated in space. */
BAMREX_API int bamrex_coupling_fill_patch(bamrex_coupling *c, double time);

/* Every valid fine cell from the current coarse state (FillCoarsePatch, for
 * a newly created fine level). */
BAMREX_API int bamrex_coupling_fill_coarse_patch(bamrex_coupling *c);

/* Reflux (AmrLevelAdv::reflux) and average_down (AmrLevelAdv::avgDown) on
 * the current coarse state. */
BAMREX_API int bamrex_coupling_reflux(bamrex_coupling *c);
BAMREX_API int bamrex_coupling_avg_down(bamrex_coupling *c);

/* Sums of the current coarse state over the coarse cells covered by the
 * fine level, times the coarse cell volume (NCOMP doubles; synchronises).
 * A composite total is sum over levels of (level totals - covered sums). */
BAMREX_API int bamrex_coupling_covered_sums(bamrex_coupling *c, double *sums);

/* Number of flux-register slots (coarse faces) in direction dir, and a copy
 * of the register (NCOMP * nslots doubles, component-major; reg may be NULL
 * to query the count).  Synchronises the stream. */
BAMREX_API int bamrex_coupling_register(bamrex_coupling *c, int dir, double *reg, int *nslots);

/* Grid generation for a new level l+1 from tags on level l (the role of
 * AMReX Amr::grid_places): tags buffered by n_error_buf cells, restricted to
 * cells n_proper cells inside level l's boxes (domain faces excepted),
 * coarsened by blocking_factor / ref_ratio, clustered by Berger-Rigoutsos
 * with efficiency grid_eff, chopped to max_grid_size and refined.  domain and
 * boxes are level l's; tags in the packed order of bamrex_level_tag;
 * periodic[d] != 0 for periodic directions.  Output: level l+1 boxes.  Host
 * only (no device work). */
BAMREX_API int bamrex_cluster_tags(int spacedim, const bamrex_box *domain, const int *periodic,
                                   const bamrex_box *boxes, int nboxes, const char *tags, int ref_ratio,
                                   int blocking_factor, int max_grid_size, int n_error_buf, int n_proper,
                                   double grid_eff, bamrex_box *out, int max_out, int *nout);

/* ------------------------------------------------------------------ */
/* AMR hierarchy with subcycling (the Amr time loop around AmrLevelAdv)  */
/* ------------------------------------------------------------------ */

#define BAMREX_MAX_LEVELS 8

typedef struct bamrex_amr bamrex_amr;

typedef struct bamrex_amr_desc {
    bamrex_level_desc base;   /* level 0; finer levels share its parameters */
    int max_level;            /* amr.max_level */
    int ref_ratio;            /* amr.ref_ratio (2 or 4, every level) */
    int blocking_factor;      /* amr.blocking_factor (fine cells; multiple of 2*ref_ratio) */
    int max_grid_size;        /* amr.max_grid_size (fine cells; multiple of blocking_factor) */
    int n_error_buf;          /* amr.n_error_buf */
    int n_proper;             /* amr.n_proper (coarse cells) */
    double grid_eff;          /* amr.grid_eff */
    int regrid_int;           /* amr.regrid_int (coarse steps; 0 = never) */
    int do_reflux;            /* adv.do_reflux */
    int phigrad_var, phigrad_var_is_primv;
    double phigrad[BAMREX_MAX_LEVELS];   /* tagging.phigrad per level */
    int max_phigrad_lev;                 /* tagging.max_phigrad_lev */
    int phierr_var, phierr_var_is_primv;
    double phierr[BAMREX_MAX_LEVELS];    /* tagging.phierr per level */
    int max_phierr_lev;                  /* tagging.max_phierr_lev */
    int max_int_lev;                     /* tagging.max_int_lev: interface tagging on levels below it */
    double lstol[BAMREX_MAX_LEVELS];     /* tagging.lstol per level */
    int max_box_lev;                     /* tagging.max_box_lev: box tagging on levels below it */
    double box_lo[3], box_hi[3];         /* tagging.box_x / box_y / box_z */
} bamrex_amr_desc;

BAMREX_API int bamrex_amr_create(bamrex_amr **out, const bamrex_amr_desc *desc, void *stream);
BAMREX_API int bamrex_amr_destroy(bamrex_amr *amr);
BAMREX_API const char *bamrex_amr_last_error(const bamrex_amr *amr);
BAMREX_API int bamrex_amr_finest_level(const bamrex_amr *amr);
/* The level object (owned by the hierarchy: valid until the next regrid). */
BAMREX_API bamrex_level *bamrex_amr_level(bamrex_amr *amr, int lev);
BAMREX_API int bamrex_amr_boxes(const bamrex_amr *amr, int lev, bamrex_box *out, int max_out, int *nout);
/* Replace level lev (1 <= lev <= finest + 1, lev <= max_level) by the given
 * boxes: new data from the old level where it overlaps, from coarse
 * interpolation elsewhere.  The next finer level stays (with its data) when
 * it is still properly nested in the new boxes; otherwise it and the levels
 * above it are removed. */
BAMREX_API int bamrex_amr_set_level_boxes(bamrex_amr *amr, int lev, const bamrex_box *boxes, int nboxes);
/* Regrid levels lbase+1 .. from tags (errorEst) on levels lbase .. at `time`. */
BAMREX_API int bamrex_amr_regrid(bamrex_amr *amr, int lbase, double time);
/* average_down from the finest level to level 0 (AmrLevelAdv::post_init). */
BAMREX_API int bamrex_amr_avg_down_all(bamrex_amr *amr);
/* One coarse step of the subcycled hierarchy (Amr::coarseTimeStep with
 * AmrLevelAdv's computeInitialDt / computeNewDt, Source/AmrLevelAdv.cpp:487-619,
 * timeStep recursion, and post_timestep reflux + avgDown, :624-652).  Regrids
 * first when regrid_int divides the coarse steps taken.  *time_io is the time
 * on entry and the new time on return; *dt_out the coarse dt taken. */
BAMREX_API int bamrex_amr_coarse_step(bamrex_amr *amr, double stop_time, double *time_io, double *dt_out);
/* Coarse steps as CUDA graphs (default on).  Once the levels have taken a
 * coarse step as they are, and when regrids are at least 4 coarse steps
 * apart (or never come), a coarse step without a regrid runs as: the stale
 * levels' max wave speeds, the coarse dt computed on the device (the same
 * operations as the host path, so the same dt bit for bit) and read back,
 * then the whole subcycled recursion (coarse/fine fills with their time
 * weights taken from device times, every level's sweeps and flux
 * registers with their dt read on the device, reflux, average_down) as one
 * graph replay, captured once per state of the levels' buffers.  The
 * result equals the host-driven step bit for bit.  No reference
 * counterpart: the reference steps its levels from the host. */
BAMREX_API int bamrex_amr_set_graph(bamrex_amr *amr, int use_graph);
/* Graphs captured, coarse steps replayed, and kernel nodes in the current
 * levels' graph (any pointer may be NULL). */
BAMREX_API int bamrex_amr_graph_stats(const bamrex_amr *amr, int *captures, long long *replays, long long *kernels);
/* Change amr.regrid_int (0: no more regrids). */
BAMREX_API int bamrex_amr_set_regrid_int(bamrex_amr *amr, int regrid_int);
/* A static rigid body on every level of the hierarchy, present and future
 * (bamrex_level_set_body on each; each level computes its level set at its
 * own resolution, as every AmrLevelAdv level does in initData); NULL
 * removes it.  The fill runs after each level's coarse/fine ghost fill
 * (FillPatcherFill, then FillRBGhostCells). */
BAMREX_API int bamrex_amr_set_body(bamrex_amr *amr, const bamrex_body_desc *desc);
/* dt of every level after the last computeInitialDt / computeNewDt. */
BAMREX_API int bamrex_amr_dt_level(const bamrex_amr *amr, double *dt_level);

/* The stepping state a checkpoint keeps besides the levels' boxes and
 * states (Amr::checkPoint's level steps and dt_level behind
 * amr.checkPoint(), Source/main.cpp:96-99, with AmrLevelAdv::checkPoint /
 * restart, Source/AmrLevelAdv.cpp:95-113): the coarse steps taken (they
 * time the regrids), whether a time step has been set, and the time step
 * of every level.  A restart rebuilds the levels and their states, then
 * sets this; the next coarse step then continues the run bit for bit. */
typedef struct bamrex_amr_stepping {
    int coarse_steps;
    int have_dt;
    int nlevels;                           /* entries of dt_level in use */
    double dt_level[BAMREX_MAX_LEVELS];
} bamrex_amr_stepping;
BAMREX_API int bamrex_amr_get_stepping(const bamrex_amr *amr, bamrex_amr_stepping *out);
BAMREX_API int bamrex_amr_set_stepping(bamrex_amr *amr, const bamrex_amr_stepping *in);
/* Composite conserved totals: every level's sums minus those of its cells
 * covered by the next finer level (NCOMP doubles; synchronises). */
BAMREX_API int bamrex_amr_conserved_sums(bamrex_amr *amr, double *totals);

/* ------------------------------------------------------------------ */
/* Pressure Helmholtz operator and solver (IMEX path)                    */
/* ------------------------------------------------------------------ */

/* Domain boundary types of the linear operator (amrex::LinOpBCType as set
 * by set_pressure_domain_BC, Source/IMEX/IMEX_O1.cpp:663-690): periodic,
 * homogeneous Neumann, homogeneous Dirichlet on the domain face. */
enum { BAMREX_LINOP_PERIODIC = 0, BAMREX_LINOP_NEUMANN = 1, BAMREX_LINOP_DIRICHLET = 2 };

typedef struct bamrex_helmholtz bamrex_helmholtz;

typedef struct bamrex_helmholtz_desc {
    int spacedim;          /* 2 or 3 */
    int n[3];              /* cells per direction: one box covering the domain */
    double prob_lo[3];
    double prob_hi[3];
    int bc_lo[3];          /* BAMREX_LINOP_* */
    int bc_hi[3];
    int max_levels;        /* multigrid levels including the finest; 0 = coarsen while every n is even and >= 4 */
    int nu1, nu2;          /* red+black sweeps before / after the coarse correction (0 = 2) */
    int bottom_sweeps;     /* sweeps on the coarsest level (0 = 16) */
} bamrex_helmholtz_desc;

/* The operator of MLABecLaplacianGrad (Source/LinearSolver/MLALaplacianGrad.H):
 *   y = A a x - B div(b grad x) + C c . grad x
 * with Fapply = mlalapgrad_adotx (MLALapGrad_2D_K.H:9-33, MLALapGrad_3D_K.H:9-38)
 * and Fsmooth = alapgrad_gsrb (MLALapGrad_2D_K.H:180-230, MLALapGrad_3D_K.H:258-324).
 * Vectors are dense arrays of n[0]*n[1]*n[2] doubles, i fastest; face
 * coefficients b[d] have one more entry along d.  Every pointer argument may
 * be host or device memory.  Coefficients default to a = 1, b = 1, no c,
 * scalars (A, B, C) = (1, 1, 0). */
BAMREX_API int bamrex_helmholtz_create(bamrex_helmholtz **out, const bamrex_helmholtz_desc *desc, void *stream);
BAMREX_API int bamrex_helmholtz_destroy(bamrex_helmholtz *h);
BAMREX_API const char *bamrex_helmholtz_last_error(const bamrex_helmholtz *h);
BAMREX_API int bamrex_helmholtz_num_levels(const bamrex_helmholtz *h);
/* setScalars(A, B, C) (MLALaplacianGrad.H:380) */
BAMREX_API int bamrex_helmholtz_set_scalars(bamrex_helmholtz *h, double a, double b, double c);
/* setACoeffs: a cell field, or the constant alpha_const when alpha is NULL */
BAMREX_API int bamrex_helmholtz_set_acoeffs(bamrex_helmholtz *h, const double *alpha, double alpha_const);
/* setBCoeffs: face fields per direction */
BAMREX_API int bamrex_helmholtz_set_bcoeffs(bamrex_helmholtz *h, const double *bx, const double *by, const double *bz);
/* setBCoeffs from a cell field by average_cellcenter_to_face
 * (IMEX_O1.cpp:599-609): b = (cell left + cell right) / 2, the boundary
 * cell itself outside a non-periodic face. */
BAMREX_API int bamrex_helmholtz_set_bcoeffs_from_cell(bamrex_helmholtz *h, const double *beta_cc);
/* setCCoeffs: spacedim cell fields (component-major), or NULL for none */
BAMREX_API int bamrex_helmholtz_set_ccoeffs(bamrex_helmholtz *h, const double *c);
/* y = A x on the finest level (Fapply) */
BAMREX_API int bamrex_helmholtz_apply(bamrex_helmholtz *h, const double *x, double *y);
/* One colour (redblack 0 or 1) of the Gauss-Seidel smoother (Fsmooth) */
BAMREX_API int bamrex_helmholtz_smooth(bamrex_helmholtz *h, double *phi, const double *rhs, int redblack);
/* z = one multigrid V-cycle applied to r from a zero initial guess */
BAMREX_API int bamrex_helmholtz_vcycle(bamrex_helmholtz *h, double *z, const double *r);
/* Solve A x = rhs by BiCGStab preconditioned with one V-cycle, from the
 * initial x, until ||rhs - A x||_2 <= max(tol_rel ||rhs||_2, tol_abs) or
 * max_iter iterations (solve_pressure, IMEX_O1.cpp:616-640).  use_graph != 0
 * replays each iteration as one CUDA graph. */
BAMREX_API int bamrex_helmholtz_solve(bamrex_helmholtz *h, double *x, const double *rhs, double tol_rel,
                                      double tol_abs, int max_iter, int use_graph, int *iters, double *rel_res);
/* Kernels launched by the operator so far (graph replays excluded). */
BAMREX_API long long bamrex_helmholtz_launches(const bamrex_helmholtz *h);

/* ------------------------------------------------------------------ */
/* Learned preconditioner (no counterpart in the reference)             */
/* ------------------------------------------------------------------ */

/* A 2D convolutional network M(r) ~ A^{-1} r for the pressure solve: four
 * resolution levels, 16 channels, 3x3 kernels, periodic padding, BF16
 * weights with FP32 accumulation; inputs (r / rms(r), log beta) per cell,
 * output the correction scaled by dx^2 / B.  Trained on the device with the
 * library's own forward, backward and Adam kernels. */
typedef struct bamrex_precnet bamrex_precnet;
BAMREX_API int bamrex_precnet_create(bamrex_precnet **out, int nx, int ny, int batch, unsigned long long seed,
                                     void *stream);
BAMREX_API int bamrex_precnet_destroy(bamrex_precnet *net);
BAMREX_API const char *bamrex_precnet_last_error(const bamrex_precnet *net);
BAMREX_API int bamrex_precnet_num_params(const bamrex_precnet *net);
/* Change the grid (sides multiples of 8) and batch of the workspace. */
BAMREX_API int bamrex_precnet_resize(bamrex_precnet *net, int nx, int ny, int batch);
/* FP32 master weights (num_params floats). */
BAMREX_API int bamrex_precnet_get_weights(bamrex_precnet *net, float *w);
BAMREX_API int bamrex_precnet_set_weights(bamrex_precnet *net, const float *w);
/* in: batch x 2 x ny x nx floats; out: batch x ny x nx floats. */
BAMREX_API int bamrex_precnet_forward(bamrex_precnet *net, const float *in, float *out);
/* Parameter gradient of sum(out * dout) after a forward on the same input. */
BAMREX_API int bamrex_precnet_backward(bamrex_precnet *net, const float *dout, float *grad);
/* Where inference forwards (bamrex_precnet_forward and the learned solve)
 * run the 16 -> 16 channel convolutions: on = 1 (the default) the tensor
 * cores with BF16 operands and FP32 accumulators -- tcgen05.mma with the
 * accumulators in tensor memory on levels whose width is a multiple of 128,
 * mma.sync on the others whose width is a multiple of 32 and height of 4,
 * the FP32 CUDA cores elsewhere; on = 2 mma.sync only (where it applies);
 * on = 0 the FP32 CUDA cores.  Training always uses the FP32 path. */
BAMREX_API int bamrex_precnet_set_tensor_cores(bamrex_precnet *net, int on);
/* One Adam step on the relative squared error ||out - target||^2 / ||target||^2
 * averaged over the batch; *loss is the value before the step. */
BAMREX_API int bamrex_precnet_train_step(bamrex_precnet *net, const float *in, const float *target, float lr,
                                         double *loss);

/* Preconditioners of the flexible solve: the network alone; the network
 * followed by one V-cycle on the residual it leaves (z = N(v) + V(v - A N(v)));
 * the V-cycle alone (the same solve without the network); or the V-cycle
 * followed by the network on what it left (z = V(v) + N(v - A V(v))). */
enum {
    BAMREX_PRECOND_NETWORK = 0,
    BAMREX_PRECOND_NETWORK_VCYCLE = 1,
    BAMREX_PRECOND_VCYCLE = 2,
    BAMREX_PRECOND_VCYCLE_NETWORK = 3
};

/* Solve A x = rhs by restarted flexible GMRES(restart) with the chosen
 * preconditioner (the network sized to the operator's grid, batch 1; NULL
 * for BAMREX_PRECOND_VCYCLE; periodic domains); if it has not reached the
 * tolerance after max_iter iterations, the plain BiCGStab/multigrid solve
 * continues from its iterate (*fell_back = 1).  Same stopping rule as
 * bamrex_helmholtz_solve; *iters counts the GMRES iterations and
 * *plain_iters the fallback's. */
BAMREX_API int bamrex_helmholtz_solve_learned(bamrex_helmholtz *h, bamrex_precnet *net, int mode, double *x,
                                              const double *rhs, double tol_rel, double tol_abs, int max_iter,
                                              int restart, int *iters, int *plain_iters, double *rel_res,
                                              int *fell_back);

/* ------------------------------------------------------------------ */
/* The IMEX step (advance_imex_rk with the linearised pressure equation,   */
/* Source/IMEX/IMEX_RK.cpp:23-86, Source/IMEX/IMEX_O1.cpp:19-176) on one    */
/* box covering the domain                                                  */
/* ------------------------------------------------------------------ */

typedef struct bamrex_imex bamrex_imex;

/* IMEXSettings (Source/IMEX/IMEXSettings.H:6-79) */
enum { BAMREX_IMEX_RUSANOV = 0, BAMREX_IMEX_MUSCL_RUSANOV = 1 };
enum {
    BAMREX_IMEX_ENTH_REUSE_PRESSURE = 0,
    BAMREX_IMEX_ENTH_CONSERVATIVE = 1,
    BAMREX_IMEX_ENTH_CONSERVATIVE_EX = 2
};
enum { BAMREX_IMEX_KE_CONSERVATIVE = 0, BAMREX_IMEX_KE_EX = 1, BAMREX_IMEX_KE_SPLIT = 2 };
/* imex.butcher_tableau (IMEXButcherTableau::TableauType, ButcherTableau.cpp) */
enum {
    BAMREX_IMEX_SP111 = 0,
    BAMREX_IMEX_SSP222 = 1,
    BAMREX_IMEX_SASSP322 = 2,
    BAMREX_IMEX_SASSP332 = 3,
    BAMREX_IMEX_SSP433 = 4
};

typedef struct bamrex_imex_desc {
    int spacedim;            /* 2 or 3 */
    int n[3];                /* cells per direction (one box: the domain) */
    double prob_lo[3];
    double prob_hi[3];
    int bc_lo[3];            /* BAMREX_BC_TRANSMISSIVE / PERIODIC / REFLECTIVE; the */
    int bc_hi[3];            /* pressure operator takes Neumann for the last two    */
    bamrex_parm parm;        /* adiabatic (gamma) and epsilon are used */
    int advection_flux;      /* imex.advection_flux */
    int enthalpy_method;     /* imex.enthalpy_method */
    int ke_method;           /* imex.ke_method */
    double cfl;              /* adv.cfl (0 = 0.5) */
    double tol_rel, tol_abs; /* pressure solve; 0 = 1e-12 / 1e-15 as solve_pressure */
    int max_iter;            /* 0 = 1000 as solve_pressure */
    int tableau;             /* BAMREX_IMEX_SP111 ... SSP433 */
} bamrex_imex_desc;

/* Allocates the state (with ghost cells), the intermediate fields and the
 * pressure operator at creation; a step allocates nothing.  Work is issued on
 * `stream` (NULL: the object's own non-blocking stream). */
BAMREX_API int bamrex_imex_create(bamrex_imex **out, const bamrex_imex_desc *desc, void *stream);
BAMREX_API int bamrex_imex_destroy(bamrex_imex *h);
BAMREX_API const char *bamrex_imex_last_error(const bamrex_imex *h);
/* The state: (D+2) components of n[0]*n[1]*n[2] doubles each, component-
 * major, i fastest (host or device memory).  p: the pressure (same cell
 * order), or NULL to take (gamma-1)(E - eps |m|^2 / (2 rho)) (copy_pressure). */
BAMREX_API int bamrex_imex_set_state(bamrex_imex *h, const double *U, const double *p);
BAMREX_API int bamrex_imex_get_state(bamrex_imex *h, double *U, double *p);
/* cfl / max (|m_x|/dx + |m_y|/dy [+ |m_z|/dz]) / rho: estTimeStep for IMEX
 * after the acoustic start-up (Source/AmrLevelAdv.cpp:417-468,
 * Source/System/Euler/Euler.cpp:107-129). */
BAMREX_API int bamrex_imex_est_time_step(bamrex_imex *h, double *dt);
/* One step of size dt (every stage of the tableau); *iters and *rel_res
 * report the pressure solves (total iterations, largest relative residual).
 * A solve that does not reach its tolerance returns BAMREX_ERR_NOT_CONVERGED
 * and leaves the state unchanged. */
BAMREX_API int bamrex_imex_step(bamrex_imex *h, double dt, int *iters, double *rel_res);
/* Solve the pressure equation with one FGMRES cycle preconditioned by the
 * network (bamrex_helmholtz_solve_learned; the plain solve continues from
 * its iterate when that cycle does not reach the tolerance) instead of
 * BiCGStab + multigrid; net NULL restores the plain solve.  The cycle's
 * iterations are capped at twice the last plain solve's (at least 2, at most
 * 30); after two cycles in a row fall back, steps solve plainly and try the
 * network again on every 16th solve. */
BAMREX_API int bamrex_imex_set_precnet(bamrex_imex *h, bamrex_precnet *net, int mode);
/* The pressure operator of the step (its coefficients are those of the last
 * step). */
BAMREX_API bamrex_helmholtz *bamrex_imex_operator(bamrex_imex *h);
/* Intermediate fields of the last stage, for checking (FLUX_d is the
 * tableau-weighted sum of the stage fluxes): *count receives the
 * number of doubles (out NULL: size query).  UEX and ENTHALPY cover the
 * valid box grown by one cell in every direction; KE, RHS and PRESSURE the
 * valid box; FLUX_d the faces of direction d of the valid box ((D+2)
 * components, one more entry along d). */
enum {
    BAMREX_IMEX_FIELD_UEX = 0,
    BAMREX_IMEX_FIELD_ENTHALPY = 1,
    BAMREX_IMEX_FIELD_KE = 2,
    BAMREX_IMEX_FIELD_RHS = 3,
    BAMREX_IMEX_FIELD_PRESSURE = 4,
    BAMREX_IMEX_FIELD_FLUX_X = 5,
    BAMREX_IMEX_FIELD_FLUX_Y = 6,
    BAMREX_IMEX_FIELD_FLUX_Z = 7
};
BAMREX_API int bamrex_imex_field(bamrex_imex *h, int which, double *out, long long *count);
/* Kernels launched by the step object (the pressure operator's excluded). */
BAMREX_API long long bamrex_imex_launches(const bamrex_imex *h);

#ifdef __cplusplus
}
#endif

#endif /* BAMREX_CUDA_H_ */
