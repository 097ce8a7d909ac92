/*
 * gazpart_gpu.h -- C ABI of the B200 implementation of GAZPART's frozen-flow
 * ellipsoidal-particle step (ADV_PARTICLE_ELLP followed by COLLISION).
 *
 * Every entry point replaces one Fortran routine of the reference; the routine and
 * its file:line (relative to the reference's source/ directory) are given beside it.
 * A Fortran host program binds these through ISO_C_BINDING interfaces with the reference's
 * argument lists (scalars by VALUE, arrays by reference); the module-level inputs the
 * reference reads implicitly (VISC, RHOF, DTIME, EMAJ_PART, ...) live in the context.
 *
 * Conventions
 *  - All functions return an int status: GP_OK (0) or one of the GP_E* codes.  The
 *    reference `stop`s where these report an error; a Fortran wrapper turns a nonzero
 *    status into `error stop` with the reference's message.
 *  - A context owns one CUDA stream on the current device and is not thread safe.
 *    Calls that return host data synchronise the stream before returning.
 *  - Arrays flagged `on_device` are device pointers on the context's device;
 *    otherwise host pointers (pinned memory is fastest).
 *  - Indices: IG (class) and IDP (sub-class) are 1-based as in the reference.
 *  - Particle state columns, in this order (GP_NSTATE = 13):
 *      x y z  u v w  qa qb qc qd  ox oy oz
 *    (PARTTYPE XP..ZP, UP..WP, ELLQUAT%a..d, OMEGAX..Z; mod_particle_parallel.f90:17-47).
 *  - Per-particle property columns (GP_NPROP = 6): emaj apr rhop ipxx ipyy ipzz
 *    (EMAJ_PART, APR_PART, RHOP, IPXX..IPZZ of the particle's class; every particle
 *    may carry its own values).
 */
#ifndef GAZPART_GPU_H
#define GAZPART_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GP_NSTATE 13
#define GP_NPROP 6
#define GP_NFLUID 6

/* status codes */
enum {
    GP_OK = 0,
    GP_ENAN_FORCE = 1,      /* 'In Fluid force'           fluid_force_ellipsoid.f90:150-159 */
    GP_ENAN_TORQUE = 2,     /* NaN angular velocity       fluid_torque_ellipsoid.f90:178-188 */
    GP_EENERGY = 3,         /* kinetic-energy balance     collision_response.f90:408-436,
                                                          wall_ellipsoid_rebound.f90:372-385 */
    GP_ESINGULAR = 4,       /* 'Matrix is numerically singular!' invert_ndim3_matrix.f90:19-21 */
    GP_EPAIR_OVERFLOW = 5,  /* candidate/contact buffer full (the reference has no check) */
    GP_EOUT_OF_GRID = 6,    /* particle outside the box grid collision_detection_connectivity.f90:81-89,
                               or outside the interpolation stencil range */
    GP_ETIMEOUT = 7,        /* a bounded device loop or host wait gave up */
    GP_ECUDA = 8,           /* CUDA runtime error */
    GP_EBADARG = 9,         /* invalid argument / unsupported configuration */
    GP_ENOMEM = 10,         /* device allocation or HBM budget refused */
    GP_EIO = 11,            /* a file could not be opened, read or written, or is truncated */
    GP_ERECORD = 12,        /* a read asked for more than the record holds (gfortran's
                               'I/O past end of record'), or a record marker is inconsistent */
    GP_EEOF = 13            /* end of file where a record was expected */
};

/* precision modes */
enum {
    GP_PREC_FP64 = 0,   /* plain path: FP64 field, FP64 everything */
    GP_PREC_MIXED = 1   /* FP32 field and stencil weights with compensated FP32 sums,
                           FP32 drag/lift/torque coefficients; FP64 integration,
                           quaternion renormalisation and FP64 contact solve */
};

/* field source layouts for gp_set_field */
enum {
    GP_LAYOUT_INTERIOR = 0,   /* (NX, NY, NZ), x fastest */
    GP_LAYOUT_REFERENCE = 1   /* (NX, NY+4, NZ+4) with ghost planes, x fastest
                                 (allocate_arrays.f90:93-118, NGHTCELL=2) */
};
/* ghost-plane modes for GP_LAYOUT_INTERIOR sources */
enum {
    GP_GHOST_PERIODIC = 0,    /* FLUIDCOMM on one rank (MPI_structures.f90:84-132) */
    GP_GHOST_ZERO = 1         /* never exchanged: the reference's vorticity arrays (main.f90:255-259) */
};
/* field components */
enum { GP_U = 0, GP_V = 1, GP_W = 2, GP_VORTX = 3, GP_VORTY = 4, GP_VORTZ = 5 };

/* Module-level inputs of the hot path (mod_param_phys.f90:14-113, mod_dns_dim.f90,
 * collision variables mod_collision.f90:5-38, readparam.f90). */
typedef struct {
    int32_t nx, ny, nz;          /* NX, NY, NZ; DX = LXMAX/real(NX-1) (meshing.f90:43-45) */
    double lx, ly, lz;           /* LXMAX, LYMAX, LZMAX */
    double visc, rhof;           /* VISC, RHOF */
    double dtime;                /* DTIME */
    double gravity;              /* GRAVITY(IG) */
    double ecp, mup;             /* ECP(IG), MUP(IG) */
    double ecw, muw;             /* ECW, MUW */
    int32_t periodicity;         /* PERIODICITY */
    int32_t wall_boundary;       /* WALL_BOUNDARY (stencil x mirror) */
    int32_t interp_scheme;       /* INTERP_SCHEME, must be 3 */
    int32_t frozen_flow;         /* FROZEN_FLOW: 1-3 = a frozen field; 3 = channel: after the
                                    advance only y and z wrap (adv_particle_new.f90:685-686) */
    int32_t precision;           /* GP_PREC_FP64 or GP_PREC_MIXED */
    int32_t store_fluid;         /* 1: write the interpolated field at each particle
                                    (PART%UFAP..VORTZAP) every step */
    int64_t max_particles;       /* particle capacity of the context (0: set by upload) */
} gp_params;

typedef struct gp_ctx gp_ctx;

/* ---------------------------------------------------------------- context ---- */
/* Allocates a context bound to the current CUDA device with one ensemble (class) and
 * one field slot described by *params.  Replaces the set-up that INIT_RUN/MESHING/
 * ALLOCATE_ARRAYS/COLLISION_INITIATION perform for the hot path (main.f90:125-340). */
int gp_ctx_create(const gp_params *params, gp_ctx **out);
int gp_ctx_destroy(gp_ctx *ctx);
/* First error recorded on the device since the last gp_clear_status: code and the
 * particle (or pair home) index that raised it. */
int gp_status(gp_ctx *ctx, int32_t *code, int64_t *first_id);
/* Counters of the last gp_collision call (accumulated over all steps since then when
 * stepping through graphs), GP_NCOUNTER values in this order: pairs within bounding
 * and centre-line reach, pairs handed to the contact stage, contact solves run (pairs
 * not proven disjoint), contacts, colliding pairs (NVREL < ZERO), accepted pairs,
 * function evaluations of the solves, largest evaluation count of one solve.  No
 * counterpart in the reference, which reports none of these. */
#define GP_NCOUNTER 8
int gp_collision_counters(gp_ctx *ctx, int64_t *vals);
/* Class (IG, 1-based) of the particle that raised the first error, 0 if none. */
int gp_status_class(gp_ctx *ctx, int32_t *ig);
/* ------------------------------------------------------------- statistics ---- */
/* Polydisperse index of each particle of class ig (PART(I,IG)%IDP): n values in
 * 1..ngroups, in the class's own particle order (host array), or NULL for all 1
 * (ngroups = 1).  The statistics below are kept per index, as the reference keeps
 * them per (IG, IDP). */
#define GP_STAT_MAX_GROUPS 8
int gp_set_class_groups(gp_ctx *ctx, int32_t ig, int32_t ngroups, const int32_t *idp);

/* STAT_PARTFLUID (stat_partfluid.f90:1-472) for class ig on the device: for each
 * index g, the sums over the class's particles of the 35 quantities the reference
 * averages (in its order: Re_p, C_D, C_L, F_drag xyz, F_lift xyz, |F_drag|, |F_lift|,
 * Re_R, C_T pitch, C_T rot, T_pitch xyz, T_rot xyz, |T_pitch|, |T_rot|, tau_p, gravity,
 * phi, symmetry axis xyz, 1/tau_p, u xyz, omega xyz) and the particle count:
 * out[g * GP_NSTAT_PARTFLUID + k], k < 35 the sums and k = 35 the count.  Dividing by
 * the count gives MEAN_PARTFLUID(:, IG, g+1).  The quantities use the fluid velocity
 * and vorticity the last step interpolated at each particle (PART%UFAP.., as the
 * reference's do), so the context must have stepped since its particles were last
 * uploaded or admitted (GP_EBADARG otherwise).  Synchronises the context's stream. */
#define GP_NSTAT_PARTFLUID 36
int gp_stat_partfluid(gp_ctx *ctx, int32_t ig, double *out);

/* Collision statistics of COLLISION_INTERACTION (collision_interaction.f90:171,
 * 330-345,397-398,423-450).  While on, every collision step adds, per class and pair of
 * indices (IDP of HOME, IDP of NEAR), over the pairs found in contact while both
 * particles were uncoloured: [0] their number, [1] the collisions among them
 * (NVREL < ZERO), [3] the overlap depth |EPT1-EPT2|, [5] NVREL, [6] |v_rel|,
 * [7] the collision angle acos(NVREL/|v_rel|).  gp_collision_stats returns class ig's
 * sums since the last reset, ngroups x ngroups x GP_NSTAT_COLLISION values, with the
 * reference's derived entries filled in from them: [2] = 2 [1] / DTIME per step
 * accumulated and [4] = [3] / [0]; *steps receives the number of collision steps
 * summed.  reset != 0 clears the sums afterwards.  Turning the statistics on or off
 * drops the captured step graphs. */
#define GP_NSTAT_COLLISION 8
int gp_collision_stats_enable(gp_ctx *ctx, int32_t on);
int gp_collision_stats(gp_ctx *ctx, int32_t ig, double *out, int64_t *steps, int32_t reset);
int gp_clear_status(gp_ctx *ctx);
int gp_sync(gp_ctx *ctx);

/* Class table used by the per-routine entry points that take IG/IDP:
 * EMAJ_PART(IG,IDP), APR_PART(IG), RHOP(IG,IDP); IPXX..IPZZ follow
 * initiation_particle_position.f90:609-634. */
int gp_set_class(gp_ctx *ctx, int32_t ig, int32_t idp, double emaj, double apr, double rhop);

/* Load one field component (UFLU, VFLU, WFLU, VORTICITY_X..Z;
 * mod_fluid_variable.f90:11-24) into the device layout. */
int gp_set_field(gp_ctx *ctx, int32_t comp, const double *src, int32_t src_layout,
                 int32_t ghost_mode, int32_t on_device);

/* Particle state (PART(1:N, IG)) in / out.  cols: GP_NSTATE column pointers;
 * props: GP_NPROP column pointers.  Download returns the caller's original order. */
int gp_upload_state(gp_ctx *ctx, int64_t n, const double *const *cols,
                    const double *const *props, int32_t on_device);
int gp_download_state(gp_ctx *ctx, int64_t n, double *const *cols, double *const *fluid,
                      int32_t on_device);

/* Several classes at once: PART(1:N(IG), IG) for IG = 1..nclass (the reference's NIG
 * classes, mod_particle_parallel.f90:103; each class collides only with itself,
 * collision.f90:7-200), all on the context's field.  counts: N(IG); cols/props are
 * arrays of sum(counts) values holding the classes one after another, and
 * gp_download_state/gp_put_state use the same concatenated order.  Every class gets
 * its own box grid (COLLISION_INITIATION from its own largest EMAJ) and search grid,
 * and one step advances and collides all classes in the same launches.
 * gp_upload_state(n, ...) is the one-class case. */
int gp_upload_classes(gp_ctx *ctx, int32_t nclass, const int64_t *counts, const double *const *cols,
                      const double *const *props, int32_t on_device);

/* ------------------------------------------------ resident fields and jobs ---- */
/* No counterpart in the reference.  Contact solves still running after `budget`
 * function evaluations are handed to a further pass of the contact kernel, which runs
 * them with every lane busy, under three times the budget, until a last pass without
 * one; the results do not change.  0 keeps every solve in one pass; at most 300
 * (MINPACK's maxfev). */
int gp_set_contact_tail(gp_ctx *ctx, int32_t budget);
int gp_get_contact_tail(gp_ctx *ctx, int32_t *budget);
/* No counterpart in the reference.  With the order on (the default), the contact solves
 * of a collision phase are handed to the lanes in decreasing predicted length, each pair
 * predicted from what its particles' solves took in the last collision phase, so that
 * solves of similar length share a warp; the results do not change.  The getter reports
 * whether the order is in use (on, with its buffers allocated). */
int gp_set_contact_order(gp_ctx *ctx, int32_t on);
int gp_get_contact_order(gp_ctx *ctx, int32_t *on);
/* No counterpart in the reference.  How the mixed form's stencil gather
 * (interp_lag3.f90:124-288) brings the field in: 0 (the default) loads each particle's
 * 16 stencil rows through L1; 1 stages each particle's 4x4x4-point box in shared memory
 * with the tensor-memory accelerator (one cp.async.bulk.tensor request per particle,
 * several particles in flight per warp).  Both give the same values bit for bit.  1 needs
 * the mixed precision and every class on one field, GP_EBADARG otherwise; should classes
 * later read several fields, the gather goes back to rows.  gp_autotune times both and
 * keeps the faster; the getter reports the staging in use. */
int gp_set_gather_staging(gp_ctx *ctx, int32_t mode);
int gp_get_gather_staging(gp_ctx *ctx, int32_t *mode);
/* Mesh (nx, ny, nz) of field slot `field`. */
int gp_field_shape(gp_ctx *ctx, int32_t field, int32_t dims[3]);
/* No counterpart in the reference (serving).  More resident fields beside the one of
 * gp_params: an (nx, ny, nz) mesh of the box (lx, ly, lz), same precision; *field
 * receives its slot (the context's own field is slot 0). */
int gp_add_field(gp_ctx *ctx, int32_t nx, int32_t ny, int32_t nz, double lx, double ly, double lz,
                 int32_t *field);
/* gp_set_field for field slot `field`. */
int gp_set_field_slot(gp_ctx *ctx, int32_t field, int32_t comp, const double *src, int32_t src_layout,
                      int32_t ghost_mode, int32_t on_device);
/* No counterpart in the reference (serving).  Admits one more class of n particles on
 * field slot `field` while others are resident: its particles join the pool (capacity
 * max_particles), it gets its own box and search grids, and from the next step on it is
 * advanced and collided (within itself) together with the others.  *ig receives its
 * class number (1-based, reused after gp_remove_class). */
int gp_add_class(gp_ctx *ctx, int32_t field, int64_t n, const double *const *cols,
                 const double *const *props, int32_t on_device, int32_t *ig);
/* One class's state columns in its own particle order (cols: GP_NSTATE pointers). */
int gp_download_class(gp_ctx *ctx, int32_t ig, double *const *cols, int32_t on_device);
/* Retires class ig, first downloading its state into cols unless cols is NULL; its
 * slots are reclaimed by the next advance. */
int gp_remove_class(gp_ctx *ctx, int32_t ig, double *const *cols, int32_t on_device);
/* Particles of class ig (0 once retired). */
int gp_class_count(gp_ctx *ctx, int32_t ig, int64_t *n);

/* No counterpart in the reference (serving).  One tracking job: a class of n particles
 * on resident field slot `field`, run for `steps` steps.  cols: GP_NSTATE host columns,
 * the initial state in and the final state out; props: GP_NPROP host columns. */
typedef struct {
    int32_t field;
    int32_t steps;
    int64_t n;
    double arrival_s;              /* arrival, seconds after gp_serve starts */
    double *const *cols;
    const double *const *props;
    double admitted_s, done_s;     /* out: admission and completion times (seconds) */
    int32_t status;                /* out: GP_OK, or the error that stopped this job */
    int32_t pad;
} gp_job;
/* Continuous batching over a job stream: jobs are admitted in arrival order as soon as
 * n * bytes_per_particle fits the HBM budget beside the running ones (and the pool,
 * capacity max_particles, has room); every iteration advances and collides all running
 * jobs in the same launches; finished jobs leave with their final state, and a job
 * whose particle raises an error leaves at once with that status while the others
 * continue.  Fields and particle state stay resident throughout.  *particle_steps:
 * the sum over steps of the particles stepped. */
int gp_serve(gp_ctx *ctx, gp_job *jobs, int32_t njobs, double hbm_budget, double bytes_per_particle,
             int64_t *particle_steps);

/* Replace the state columns of the resident particles (properties unchanged), caller
 * order.  The drop-in form of handing PART back to the device after host-side edits. */
int gp_put_state(gp_ctx *ctx, int64_t n, const double *const *cols, int32_t on_device);

/* One time step of an ensemble held in host memory, in one call: in_cols (the 13 state
 * columns, caller order) in, one ADV_PARTICLE_ELLP + COLLISION as gp_step(ctx, 1), the
 * state out to out_cols.  The results are those of gp_put_state, gp_step(ctx, 1) and
 * gp_download_state in turn, bit for bit; the copies overlap the step where the data
 * allow (the gather starts once the positions are in; positions and quaternions go out
 * during the collision phase).  in_cols and out_cols may be the same arrays.  The
 * reference's main loop with PART on the host (main.f90:496-509) maps to one call per
 * cycle. */
int gp_step_host(gp_ctx *ctx, int64_t n, const double *const *in_cols, double *const *out_cols);

/* ---------------------------------------------------------------- hot path ---- */
/* ADV_PARTICLE_ELLP(NCYCLE)  adv_particle_new.f90:7-704: interpolation of the six
 * fields at x_n, RK2 predictor/corrector with wall handling, BOUNDARY_PARTICLE's
 * periodic wrap (boundary_particle.f90:45-62).  State stays on the device. */
int gp_adv_particle_ellp(gp_ctx *ctx, int32_t ncycle);
/* COLLISION(NCYCLE, TIME)  collision.f90:7-200 with NPROC=1: detection
 * (collision_detection_connectivity.f90) and greedy interaction in list order
 * (collision_interaction.f90:190-419).  Optional counters: candidate pairs within
 * bounding distance, contacts, collisions (any may be NULL). */
int gp_collision(gp_ctx *ctx, int32_t ncycle, double time, int64_t *n_near,
                 int64_t *n_contact, int64_t *n_coll);
/* nsteps x (ADV_PARTICLE_ELLP + COLLISION) replayed from a captured CUDA graph. */
int gp_step(gp_ctx *ctx, int32_t nsteps);
/* Phases of one step, in launch order, as timed by gp_step_timed. */
enum {
    GP_PHASE_GATHER = 0,     /* stencil gather at x_n and the move into cell order */
    GP_PHASE_INTEGRATE = 1,  /* RK2 predictor/corrector, walls, periodic wrap */
    GP_PHASE_BIN = 2,        /* search-grid binning: count, scan, scatter */
    GP_PHASE_SEARCH = 3,     /* candidate pairs */
    GP_PHASE_CONTACT = 4,    /* contact solves and NVREL test */
    GP_PHASE_RESPONSE = 5,   /* greedy acceptance and impulse response */
    GP_NPHASE = 6
};
/* nsteps steps captured as one CUDA graph with timestamp nodes between the phases;
 * returns the total and, per step on average, each phase's duration in milliseconds
 * (phase_ms_avg: GP_NPHASE floats), and the number of kernels one step launches
 * (counted from the captured graph).  Any output pointer may be NULL.  No counterpart
 * in the reference (measurement). */
int gp_step_timed(gp_ctx *ctx, int32_t nsteps, float *total_ms, float *phase_ms_avg,
                  int32_t *kernels_per_step);
/* Launch grids (blocks per launch) that gp_autotune chooses, in this order. */
enum {
    GP_TUNE_GATHER = 0,      /* stencil gather */
    GP_TUNE_INTEGRATE = 1,   /* integrate */
    GP_TUNE_BIN = 2,         /* binning count and scatter */
    GP_TUNE_SEARCH = 3,      /* candidate-pair search */
    GP_NTUNE = 4
};
/* Autotuner: for each launch above, in turn, times one-step graphs of the resident
 * ensemble with 148 x {1,2,4,8,16} blocks and keeps the fastest; for the mixed form on
 * one field, also the gather's staging (gp_set_gather_staging); then times eight-step
 * graphs without and with the next step's gather run on a second stream beside the
 * contact solves, the latter also with the next step's integrate of the particles in
 * no candidate pair following the gather there (each also with the gather at 148 x 16
 * blocks), and keeps the fastest.  The particle state is saved first and restored
 * afterwards.  grids_out: GP_NTUNE + 1 ints (the grids, then 0: no overlap, 1: the
 * gather overlapped, 2: the gather and the speculative integrate overlapped) or NULL.
 * Every choice gives the same results bit for bit.  No counterpart in the reference. */
int gp_autotune(gp_ctx *ctx, int32_t *grids_out);
/* Sets the launch grids and the overlap choice (0, 1 or 2) directly (GP_NTUNE + 1 ints,
 * as gp_autotune reports them), e.g. to replay a tuned configuration.  Choice 2 needs
 * 4 bytes of device memory per pool slot; without them it returns GP_ENOMEM (and the
 * autotuner does not try it). */
int gp_set_launch(gp_ctx *ctx, const int32_t *grids);
/* Pair buffers.  The reference's candidate list is a static array of 1e8 pairs with no
 * check on it (collision.f90:35-37, collision_detection_connectivity.f90:171,189).  Here
 * the candidate-pair buffer starts at max(2^20, particle capacity) and the colliding-pair
 * buffer at a quarter of that.  A step whose candidates outgrow either one stops after
 * its advance (its search counts how many it needed), every later step of the same
 * graph does nothing, and the call that ran it grows both buffers to the counted need
 * plus a quarter, runs that step's collision phase again and carries on with the steps
 * that remain: gp_step, gp_collision, gp_step_host, gp_step_timed and gp_serve all
 * finish with the same states and pairs as with large enough buffers from the start.
 * (gp_collision_counters then counts that step's candidate pairs twice: its halted
 * search and the one that ran again.)
 * gp_set_pair_capacity sets both sizes (in pairs) directly, smaller or larger;
 * gp_pair_capacity reports them (either pointer may be NULL).  No counterpart in the
 * reference. */
int gp_set_pair_capacity(gp_ctx *ctx, int64_t cap_pairs, int64_t cap_coll);
int gp_pair_capacity(gp_ctx *ctx, int64_t *cap_pairs, int64_t *cap_coll);
/* Last step's accepted collisions as (home, near) original indices, in acceptance
 * (list) order; *count receives the total even if it exceeds cap. */
int gp_collision_pairs(gp_ctx *ctx, int64_t cap, int32_t *home, int32_t *near, int64_t *count);

/* COLLISION_BOX_CONNECTIVITY  collision_box_connectivity.f90:7-384 for the context's
 * box grid (COLLISION_INITIATION, collision_initiation.f90:44-103).  ncon: NBOX,
 * con: NBOX*27 (1-based box ids, zero-padded) host arrays; either may be NULL.
 * grid_out (optional, 3 ints + 6 doubles): NXBOX NYBOX NZBOX, DXBOX DYBOX DZBOX,
 * XMINBOX YMINBOX ZMINBOX. */
int gp_collision_box_connectivity(gp_ctx *ctx, int32_t *nbox, int32_t *ncon, int32_t *con,
                                  int32_t *grid_dims, double *grid_geom);

/* ------------------------------------------------------ per-routine drop-ins ---- */
/* INTERP_LAG3(XAIN,YAIN,ZAIN,UAIN,NINT,XINT,YINT,ZINT,UINT)  interp_lag3.f90:11-298
 * on the context's field component `comp` (the mesh is the context's). */
int gp_interp_lag3(gp_ctx *ctx, int32_t comp, int64_t nint, const double *xint,
                   const double *yint, const double *zint, double *uint, int32_t on_device);
/* FROZEN_INTERP_LAG3(XAIN,YAIN,ZAIN,NX,NY,NZ,UAIN,NINT,XINT,YINT,ZINT,UINT)
 * frozen_interp_lag3.f90:11-274 (mirror boundaries).  Host arrays. */
int gp_frozen_interp_lag3(gp_ctx *ctx, const double *xain, const double *yain,
                          const double *zain, int32_t nx, int32_t ny, int32_t nz,
                          const double *uain, int64_t nint, const double *xint,
                          const double *yint, const double *zint, double *uint);
/* FLUID_FORCE_ELLIPSOID(IG,IDP,UPART,VPART,WPART,UFLUID,VFLUID,WFLUID,quat,FDRAG,FLIFT)
 * fluid_force_ellipsoid.f90:1-161 */
int gp_fluid_force_ellipsoid(gp_ctx *ctx, int32_t ig, int32_t idp, double upart, double vpart,
                             double wpart, double ufluid, double vfluid, double wfluid,
                             const double quat[4], double fdrag[3], double flift[3]);
/* batched form: n particles, arrays of length n (quat n*4, outputs n*3, row major) */
int gp_fluid_force_ellipsoid_batch(gp_ctx *ctx, int64_t n, const int32_t *ig, const int32_t *idp,
                                   const double *up, const double *uf, const double *quat,
                                   double *fdrag, double *flift, int32_t on_device);
/* FLUID_TORQUE_ELLIPSOID(I,IG,IDP,OX,OY,OZ,QUAT,TORQUE_PITCHING,TORQUE_ROTATION)
 * fluid_torque_ellipsoid.f90:1-190.  The reference reads PART(I,IG)%UP..WP,
 * %UFAP..WFAP and %VORTXAP..VORTZAP from its module; they are passed explicitly. */
int gp_fluid_torque_ellipsoid(gp_ctx *ctx, int32_t ig, int32_t idp, double ox, double oy,
                              double oz, const double quat[4], const double part_up[3],
                              const double part_ufap[3], const double part_vort[3],
                              double tpitch[3], double trot[3]);
int gp_fluid_torque_ellipsoid_batch(gp_ctx *ctx, int64_t n, const int32_t *ig,
                                    const int32_t *idp, const double *omega, const double *quat,
                                    const double *part_up, const double *part_ufap,
                                    const double *part_vort, double *tpitch, double *trot,
                                    int32_t on_device);
/* QUATERNION_INTEGRATION(qp_n, omgx, omgy, omgz, dt)  adv_quaternion.f90:1-117 */
int gp_quaternion_integration(gp_ctx *ctx, double quat[4], double omgx, double omgy,
                              double omgz, double dt);
int gp_quaternion_integration_batch(gp_ctx *ctx, int64_t n, double *quat, const double *omega,
                                    double dt, int32_t on_device);
/* EULER_INTEGRATION(IG, IDP, omgx, omgy, omgz)  adv_angular_velocity.f90:1-168 */
int gp_euler_integration(gp_ctx *ctx, int32_t ig, int32_t idp, double *omgx, double *omgy,
                         double *omgz);
/* ellipsoid_contact_detection(IG,IDP1,IDP2,IXP,IYP,IZP,IQUAT,JXP,JYP,JZP,JQUAT,
 * flag,EPT1,EPT2,cnormal)  ellipsoid_contact_detection.f90:1-187 (lmder1 inside). */
int gp_ellipsoid_contact_detection(gp_ctx *ctx, int32_t ig, int32_t idp1, int32_t idp2,
                                   double ixp, double iyp, double izp, const double iquat[4],
                                   double jxp, double jyp, double jzp, const double jquat[4],
                                   int32_t *flag, double ept1[3], double ept2[3],
                                   double cnormal[3]);
/* batched form with explicit shapes: per pair emaj1 apr1 emaj2 apr2 (n*4), centres
 * (n*6: b1,b2), quaternions (n*8: q1,q2).  Outputs flag n, ept1/ept2/cnormal n*3. */
int gp_ellipsoid_contact_detection_batch(gp_ctx *ctx, int64_t n, const double *shapes,
                                         const double *centres, const double *quats,
                                         int32_t *flag, double *ept1, double *ept2,
                                         double *cnormal, int32_t on_device);
/* No counterpart in the reference.  The batched contact detection above for callers
 * that cannot allocate device memory (a solver whose particle pool has filled HBM, a
 * real-time loop that cannot take the device-wide synchronisation of cudaFree, a host
 * program whose memory plan forbids allocation after start-up).  Same arguments and
 * results as gp_ellipsoid_contact_detection_batch, without a context; `stream` is a
 * cudaStream_t (NULL: the default stream) on the current device.  It calls no
 * allocator: inputs and results pass through one static device array of
 * GP_NOALLOC_MAX_PAIRS pairs (220 bytes per pair), and n above that returns GP_EBADARG
 * without doing any work.  The array is shared by all calls on a device and keeps the
 * last call's contents; calls that can overlap on the GPU race on it and must be
 * ordered by the caller.  The first call on each device (and the first after the
 * device's context is replaced) looks up the array with that device current and may
 * load this library's device code.  Synchronises `stream` before returning; a stream
 * that is being captured is refused with GP_EBADARG before any work is enqueued. */
#define GP_NOALLOC_MAX_PAIRS 32768
int gp_ellipsoid_contact_detection_batch_noalloc(int64_t n, const double *shapes,
                                                 const double *centres, const double *quats,
                                                 int32_t *flag, double *ept1, double *ept2,
                                                 double *cnormal, int32_t on_device,
                                                 void *stream);
/* COLLISION_RESPONSE(IG,IDP,part1,part2,R_impact1,R_impact2,normal)
 * collision_response.f90:1-437.  partK: 10 doubles in/out (UP VP WP, OMEGAX..Z,
 * ELLQUAT a..d); inertia of class (IG,IDP) for both bodies as in the reference. */
int gp_collision_response(gp_ctx *ctx, int32_t ig, int32_t idp, double part1[10],
                          double part2[10], const double r_impact1[3],
                          const double r_impact2[3], const double normal[3]);

/* ------------------------------------------------------------ live fluid ---- */
/* The periodic pseudo-spectral solver of the reference's DNS mode (SOLVE_FLUID = 1),
 * on the device with cuFFT.  A solver holds the velocity on the NX x NY x NZ mesh of
 * *params (interior arrays [z][y][x], x fastest; NX, NY, NZ even), the wavenumbers of
 * meshing.f90:96-140 (KFIRST = 2 pi / LX for every direction) and the aliasing filter of
 * meshing.f90:144-180: aliascontrol 0 none, 1 sharp, 2 smooth with RTRUNC = rtrunc (the
 * reference uses 2 and 8/9).  No stochastic forcing (STEADY = .false.). */
typedef struct gp_dns gp_dns;
int gp_dns_create(const gp_params *params, int32_t aliascontrol, double rtrunc, gp_dns **out);
int gp_dns_destroy(gp_dns *dns);
int gp_dns_set_velocity(gp_dns *dns, const double *u, const double *v, const double *w, int32_t on_device);
int gp_dns_get_velocity(gp_dns *dns, double *u, double *v, double *w, int32_t on_device);
/* ADV_FLUID(NCYCLE) (adv_fluid.f90:1-271): one step of the two-stage scheme with the
 * viscous integrating factor, the rotational nonlinear term projected onto the
 * divergence-free plane (nonlinear_terms.f90), PROJ_DIVFREE and the filter. */
int gp_adv_fluid(gp_dns *dns, int32_t ncycle);
/* Vorticity of the current velocity, spectrally (i k x u, as nonlinear_terms.f90:81-99
 * forms it). */
int gp_dns_vorticity(gp_dns *dns, double *ox, double *oy, double *oz, int32_t on_device);
/* The velocity into field slot `field` of a context, with periodic y and z ghosts as
 * FLUIDCOMM leaves them (main.f90:499-505), so that the next particle step interpolates
 * the live field.  with_vorticity != 0 also writes the spectral vorticity (zero ghosts);
 * the reference leaves its vorticity arrays as initialised in DNS mode. */
int gp_dns_couple(gp_dns *dns, gp_ctx *ctx, int32_t field, int32_t with_vorticity);

#ifdef __cplusplus
}
#endif
#endif /* GAZPART_GPU_H */
