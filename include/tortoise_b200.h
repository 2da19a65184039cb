/*
 * tortoise_b200.h -- C ABI of the B200 (sm_100a) collision operator and
 * Dormand-Prince 5(4) time stepper for TORTOISE-style Boltzmann transport on
 * P1 discontinuous-Galerkin simplex meshes in 2D k-space.
 *
 * Plain C types only: pointers, sizes, doubles.  No exceptions cross this
 * boundary; every entry point returns a tb_status code and tb_last_error()
 * gives a one-line message for the calling thread.
 *
 * State layout (the "status" vector).  All bands are concatenated in band
 * order.  Band b occupies Ne_b * 3 doubles starting at tb_band_offset(b);
 * inside a band the layout is element-major, basis-minor:
 *     f[off_b + 3*e + 0] = f(v0)            (value at the element's first vertex)
 *     f[off_b + 3*e + 1] = f(v1) - f(v0)
 *     f[off_b + 3*e + 2] = f(v2) - f(v0)
 * which is the linear-form layout of the reference's Function<2>::vec
 * (src/Geometry/Structured/FunctionSpace/Function.cpp:60-68,
 *  include/Geometry/Structured/FunctionSpace/Function.hpp:352-369).
 *
 * Element numbering follows Mesh<2>::elemID (src/Geometry/Structured/
 * DirectSpace/Mesh.cpp:407-411): e = 2*(sx + sy*nx) + elemInSection, with
 * element 0 of a section spanning section-relative vertices (0,0),(1,0),(1,1)
 * and element 1 spanning (0,0),(0,1),(1,1).
 */
#ifndef TORTOISE_B200_H
#define TORTOISE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
typedef enum tb_status {
    TB_OK              = 0,
    TB_ERR_BAD_DESC    = 1,  /* malformed problem description               */
    TB_ERR_OOM         = 2,  /* device or host allocation failed            */
    TB_ERR_CUDA        = 3,  /* a CUDA runtime call failed                  */
    TB_ERR_DT_UNDERFLOW= 4,  /* DP45 step below denseStep/1e4 (reference's
                                "step size has become too small")           */
    TB_ERR_NONFINITE   = 5,  /* NaN/Inf met in the state or error norm      */
    TB_ERR_TIMEOUT     = 6,  /* bounded device wait ran out                 */
    TB_ERR_NO_DEVICE   = 7,  /* no CUDA device / library built without it   */
    TB_ERR_ARG         = 8,  /* bad argument (index out of range, NULL ...)  */
    TB_ERR_CAPACITY    = 9   /* an output buffer was too small              */
} tb_status;

/* scattLegDirection of the reference (include/Geometry/GeometryCore/Geometry.hpp:119) */
#define TB_IN   1
#define TB_OUT (-1)
/* statisticType of the reference (include/Physics/Material/Material.hpp:51) */
#define TB_FERMION (-1)
#define TB_BOSON     1

#define TB_MAX_LEGS 4

/* ------------------------------------------------------ problem description */
/* Region<2> (include/Geometry/Structured/DirectSpace/Region.hpp): origin and
 * the two side vectors, stored column-major: gvec[0..1] = side 0, gvec[2..3] = side 1. */
typedef struct tb_region {
    double origin[2];
    double gvec[4];
} tb_region;

/* Mesh<2>(region, relativeOrigin, relativeSize, nSecSplits)
 * (src/Geometry/Structured/DirectSpace/Mesh.cpp:319-347). */
typedef struct tb_mesh_desc {
    double  rel_origin[2];
    double  rel_size[2];
    int32_t nsplit[2];
} tb_mesh_desc;

/* Band<2> (include/Physics/Material/Band.hpp:49-113).  The dispersion is
 * given as linear-form coefficients (Ne*3 doubles, layout above); the crystal
 * momentum functions kx, ky are rebuilt from the mesh exactly as
 * costructCrystalMomentum<2> does (src/Physics/Material/Band.cpp:45-56). */
typedef struct tb_band_desc {
    int32_t       mesh;            /* index into tb_problem_desc.meshes        */
    double        charge;
    double        statistics;      /* TB_FERMION or TB_BOSON                   */
    const double* dispersion;      /* [Ne*3] linear-form coefficients          */
    double        abs_tol;         /* absoluteErrorTolerance  (Band.hpp:77)    */
    double        rel_tol;         /* relativeErrorTolerance  (Band.hpp:78)    */
    double        penalisation;    /* penalisationUnphysicalPopulation (:82)   */
    int32_t       constrained;     /* Band::constrained (Band.hpp:66)          */
    const double* constrained_population; /* [Ne*3] time-independent
                                     constrainedPopulation, or NULL            */
    double        drift_velocity[2]; /* dk/dt of the Vlasov drift term for this
                                     band (Vlasov<2>::vlasovFlux velocity,
                                     include/Physics/Transport/Vlasov.hpp:69);
                                     (0,0) disables drift for the band         */
} tb_band_desc;

/* ScatteringChannel<2,L> (include/Physics/Scattering/ScatteringChannel.hpp:54-192). */
typedef struct tb_channel_desc {
    int32_t        nlegs;              /* 2, 3 or 4                               */
    int32_t        band[TB_MAX_LEGS];  /* legBandNumber                           */
    int32_t        dir[TB_MAX_LEGS];   /* legDirection: TB_IN / TB_OUT            */
    double         amplitude;          /* amplitude (functAmplitude == 1)         */
    int32_t        n_mc;               /* numMCPoints                             */
    double         min_det;            /* minimumDeterminant                      */
    double         threshold;          /* scattElemeThreshold                     */
    int32_t        n_umklapp;          /* columns of umklappUnitVectors           */
    const double*  umklapp;            /* [n_umklapp*2], in units of region gvec  */
    /* Monte-Carlo table (ScatteringChannel::mCPoints, ScatteringChannel.cpp:677-688)
     * as an explicit seeded input, point-major: n_mc rows of R = 2*(L-2)+1
     * doubles: (L-2) points of the reference triangle followed by one
     * coordinate in [0,1] for the partially constrained leg.               */
    const double*  mc_points;
    /* Points for the tuple-survival test of precalculateIndices
     * (ScatteringChannel.cpp:476-504 via IntegratorCore.hpp:382-388); same
     * shape.  NULL: reuse mc_points.                                        */
    const double*  mc_points_precalc;
    /* Optional caller-supplied tuple list (the content of a .scattIndices
     * cache, ScatteringChannel.cpp:421-458).  n_tuples == 0: enumerate.     */
    int64_t        n_tuples;
    const int32_t* tuples;             /* [n_tuples*L] element ids              */
    const int32_t* tuple_umklapp;      /* [n_tuples] umklapp column index       */
} tb_channel_desc;

typedef struct tb_problem_desc {
    tb_region              region;
    int32_t                n_meshes;
    const tb_mesh_desc*    meshes;
    int32_t                n_bands;
    const tb_band_desc*    bands;
    int32_t                n_channels;
    const tb_channel_desc* channels;
} tb_problem_desc;


/* ------------------------------------------------------------ entry points */
typedef struct tb_handle tb_handle;

/* Collision-kernel layouts (tb_options.layout / tb_channel_info) */
#define TB_LAYOUT_AUTO   0  /* per channel: fastest layout that fits the budget  */
#define TB_LAYOUT_MC64   1  /* Monte-Carlo quadrature per tuple, FP64 (TypeB)    */
#define TB_LAYOUT_T64    2  /* precomputed moment tensor, FP64 storage            */
#define TB_LAYOUT_T32    3  /* precomputed moment tensor, FP32 storage, FP64 accumulate */
#define TB_LAYOUT_T40    4  /* moment tensor, upper 40 bits of FP64 (5 B, 2^-29 relative), FP64 accumulate */
#define TB_LAYOUT_T48    5  /* moment tensor, upper 48 bits of FP64 (6 B, 2^-37 relative), FP64 accumulate */
#define TB_LAYOUT_STREAM 6  /* Monte-Carlo quadrature over the points inside the simplices with the tuples
                               enumerated again in every evaluation: no stored list (tb_options.stream_legs) */

typedef struct tb_options {
    int32_t device;               /* CUDA device ordinal                            */
    int32_t layout;               /* TB_LAYOUT_*                                    */
    int32_t allow_fp32;           /* AUTO for 2- and 3-leg channels: 0 -> T64, 1 -> T32, 2 -> T40, 3 -> T48 */
    int64_t tensor_budget_bytes;  /* cap on precomputed-tensor memory (0: 60% free) */
    int32_t verbose;
    int32_t autotune;             /* 1: time the contraction schedules at creation, keep the fastest */
    int32_t shard_rank;           /* tuple sharding (tb_shard_connect): this process's part ... */
    int32_t shard_count;          /* ... of shard_count parts; 0 or 1: no sharding  */
    int32_t deterministic;        /* 1: bit-reproducible sums.  The collision, rate and VJP
                                     kernels add their per-tuple results into exact 192-bit
                                     fixed-point accumulators (units of 2^-112, integer
                                     atomics) that are rounded to FP64 once per evaluation,
                                     instead of FP64 atomics, so a result depends on the
                                     per-tuple values only -- not on thread arrival order,
                                     launch geometry or the contraction schedule.  Slower;
                                     24 more bytes of device memory per dof (and per slot of
                                     a run-minor group's accumulator).  A non-finite
                                     contribution makes the whole evaluation NaN; a finite one
                                     of magnitude 2^64 or more is clamped to that range (the
                                     huge trial stage of a step that its error norm rejects),
                                     and tb_rhs, tb_scattering_rates, tb_synchronize, the VJP
                                     and the adjoint sweep then return TB_ERR_NONFINITE.  The
                                     reference's TBB reduce (ScatteringChannel.cpp:651-670) is
                                     itself not reproducible across thread schedules. */
    int32_t stream_legs;          /* 2..4: every channel with at least this many legs whose tuples the
                                     library enumerates (n_tuples == 0) keeps no tuple list: each
                                     evaluation walks the candidates of precalculateIndices
                                     (ScatteringChannel.hpp:205-255, ScatteringChannel.cpp:476-504) on
                                     the device again and integrates the survivors on the spot
                                     (TB_LAYOUT_STREAM), for lists too large for device memory (four-leg
                                     e-e on fine meshes).  Same per-tuple sums as the stored list, for the
                                     operator, the rates and the adjoint's VJP.  Such channels have no
                                     tuple list to read or save and take no functAmplitude;
                                     tb_channel_info reports the counts of their last evaluation
                                     outside an integration.  0: every list is stored. */
} tb_options;

/* Pointer flags */
#define TB_PTR_HOST       1   /* f / out / dense buffers are host memory (copies inside) */
#define TB_NO_DRIFT       2   /* skip the Vlasov drift term                            */
#define TB_NO_COLLISIONS  4   /* skip all scattering channels                          */

typedef struct tb_dp45_stats {
    double  t;            /* time reached                                   */
    double  dt;           /* next step size                                 */
    double  last_err;     /* last normalised error                          */
    int64_t attempts, accepted, rejected, rhs_evals;
    int64_t n_dense;      /* dense outputs produced                         */
    int32_t status;       /* tb_status of the integration                   */
    int32_t done;         /* 1 once t >= t_final or the integration failed  */
} tb_dp45_stats;

const char* tb_last_error(void);

/* Builds device tables, enumerates (or uploads) the tuple lists and, for the
 * tensor layouts, precomputes the moment tensors.  Replaces the setup half of
 * Material::addScatteringChannelsWildcards (src/Physics/Material/Material.cpp:
 * 209-364: findUmklappVectors -> constructMCPoints -> precalculateIndices). */
int tb_create(tb_handle** h, const tb_problem_desc* desc, const tb_options* opts);
int tb_destroy(tb_handle* h);

/* Batched ensemble: n_runs independent runs (different initial conditions,
 * temperatures, coupling constants, meshes ...) in one handle and one state
 * vector (runs concatenated in order).  Runs whose structure is identical
 * (region, meshes, dispersions, statistics, channels, Monte-Carlo tables)
 * share one tuple list and one moment tensor: the collision kernels stream
 * each tuple tile once and contract it against every such run.  Every run
 * keeps its own amplitudes, tolerances, constraints, drift, state and, in the
 * integrator, its own adaptive step size and accept/reject sequence.  Bands
 * and channels are numbered globally in run order (tb_run_info gives each
 * run's first band and channel).  No counterpart in the reference (one
 * Material per process there). */
int tb_create_batch(tb_handle** h, const tb_problem_desc* const* runs, int n_runs, const tb_options* opts);
int tb_num_runs(const tb_handle* h);
int tb_run_info(const tb_handle* h, int run, int64_t* dof_offset, int64_t* ndofs, int32_t* first_band,
                int32_t* first_channel);

int64_t tb_num_dofs(const tb_handle* h);
int64_t tb_band_offset(const tb_handle* h, int band);
int     tb_num_channels(const tb_handle* h);
/* tuples kept, tuples passing the element energy window, tuples passing the
 * determinant filter, and the collision layout chosen for the channel.  On a
 * sharded handle the tuples kept (and tb_get_tuples) are this handle's part. */
int tb_channel_info(const tb_handle* h, int ch, int64_t* n_tuples, int64_t* n_prefilter, int64_t* n_det,
                    int32_t* layout);
/* Copies a channel's tuple list to host memory: ids[n*L] (tuple-major), umk[n]. */
int tb_get_tuples(const tb_handle* h, int ch, int32_t* ids, int32_t* umk);
/* A channel's k-dependent matrix element: ScatteringChannel::functAmplitude
 * (include/Physics/Scattering/ScatteringChannel.hpp:74), evaluated as
 * constructAmplitude does (src/Physics/Scattering/ScatteringChannel.cpp:
 * 399-415): once per tuple, at the barycentres of the tuple's elements
 * (Mesh<2>::elemCentre, src/Geometry/Structured/DirectSpace/Mesh.cpp:533-535),
 * fullAmplitude = amplitude * volumes * functAmplitude.  fn(user, n, nlegs,
 * barycentres, out) gets n tuples at a time -- barycentres[(i*nlegs + l)*2 +
 * {0,1}] = k_x, k_y of leg l's element of tuple i -- writes out[n] and returns
 * 0.  It is called inside this call only.  The factors belong to the
 * channel's structure group (every run of a batch that shares the tuple list);
 * the moment tensor, if any, is rebuilt with them folded in.  As in the
 * reference, the tuple list itself was chosen with functAmplitude = 1.  fn =
 * NULL returns to 1.  No state is kept of fn. */
typedef int (*tb_amplitude_fn)(void* user, int64_t n, int32_t nlegs, const double* barycentres, double* out);
int tb_set_channel_amplitude_fn(tb_handle* h, int ch, tb_amplitude_fn fn, void* user);

/* ScatteringChannel::amplitude (coupling constant); 0 disables the channel
 * like MaterialStatus::propagate does (MaterialStatus.cpp:149). */
int tb_set_amplitude(tb_handle* h, int ch, double amplitude);

/* dfdt = sum over channels of ScatteringChannel::propagate(f) (each including
 * M^-1) plus the Vlasov drift of bands with nonzero drift velocity.
 * Replaces MaterialStatus<2>::propagate() (src/Physics/Status/MaterialStatus.cpp:146-161). */
int tb_rhs(tb_handle* h, const double* f, double* dfdt, int flags);

/* One channel: ScatteringChannel<2,L>::propagate (src/Physics/Scattering/
 * ScatteringChannel.cpp:651-670), M^-1 included. */
int tb_channel_propagate(tb_handle* h, int ch, const double* f, double* out, int flags);

/* MaterialStatus::relativeError(err, pop) (MaterialStatus.cpp:189-196), one
 * value per run: result[n_runs]. */
int tb_relative_error(tb_handle* h, const double* err, const double* pop, double* result, int flags);

/* MaterialStatus::applyConstraints for time-independent constraints (refused
 * while a constraint callback is set: use tb_apply_constraints_at). */
int tb_apply_constraints(tb_handle* h, double* f, int flags);

/* Time-dependent constrained populations: Band::constrainedPopulation
 * (include/Physics/Material/Band.hpp:70-74), a std::function<Function(Real)>
 * in the reference, as a C callback.  fn(user, band, t, population) writes the
 * Ne*3 linear-form coefficients of constrained band `band` (global band index)
 * at time t and returns 0 (non-zero: failure, the integration stops with
 * TB_ERR_ARG).  While it is set, every enforceValue of the integrator
 * (MaterialStatus::applyConstraints(time), MaterialStatus.cpp:198-206) takes
 * the constrained bands from it -- at the stage times t + c_i dt, at t + dt and
 * at the dense-output times -- and MaterialTimeStatus::timeStepVetoer
 * (src/Physics/Status/MaterialTimeStatus.cpp:60-100) limits the step at the
 * start and after every accepted step, as DormandPrince54.hpp:554, 638-640 do.
 * The callback runs on a CUDA host thread between the kernels of an attempt:
 * it must not call CUDA.  At most TB_TC_DENSE_PER_STEP dense outputs per step
 * (TB_ERR_CAPACITY beyond).  The adjoint and tb_dp45_replay refuse a handle
 * with a callback.  fn = NULL returns to the constant populations of the
 * description. */
typedef int (*tb_constraint_fn)(void* user, int32_t band, double t, double* population);
#define TB_TC_DENSE_PER_STEP 8
int tb_set_constraint_fn(tb_handle* h, tb_constraint_fn fn, void* user);

/* MaterialStatus::applyConstraints(t): the constrained bands of f take their
 * populations at time t (the callback's, else the constant ones). */
int tb_apply_constraints_at(tb_handle* h, double* f, double t, int flags);

/* Dormand-Prince 5(4) from t0 to t_final with dense output every dense_step,
 * entirely on the device: Algorithms::dormandPrince54 (include/Generics/
 * Algorithms/DormandPrince54.hpp:479-665) as called by MaterialTimeStatus::
 * propagate (src/Physics/Status/MaterialTimeStatus.cpp:102-137).
 * f_inout: state at t0 on entry, state at the last accepted step on exit.
 * dense_out[max_dense*ndofs], dense_times[max_dense] receive the dense outputs;
 * for a batch, run r's block (max_dense slots of its own ndofs) follows run
 * r-1's, and dense_times holds max_dense entries per run. */
int tb_dp45_integrate(tb_handle* h, double* f_inout, double t0, double t_final, double dense_step,
                      double* dense_out, double* dense_times, int64_t max_dense, tb_dp45_stats* stats,
                      int flags);

/* The same integration in pieces: begin, advance by whole attempts (one CUDA
 * graph launch each, asynchronous; attempts after the end are no-ops), poll,
 * end.  max_dense == 0 keeps no dense output. */
int tb_dp45_begin(tb_handle* h, const double* f0, double t0, double t_final, double dense_step, int64_t max_dense,
                  int flags);
/* Per-run start time, end time and dense step (arrays of n_runs). */
int tb_dp45_begin_batch(tb_handle* h, const double* f0, const double* t0, const double* t_final,
                        const double* dense_step, int64_t max_dense, int flags);
/* Statistics of one run as of the last tb_dp45_poll / tb_dp45_end. */
int tb_dp45_run_stats(tb_handle* h, int run, tb_dp45_stats* stats);
int tb_dp45_advance(tb_handle* h, int64_t n_attempts);
/* stats of run 0; stats->done = 1 once every run is done. */
int tb_dp45_poll(tb_handle* h, tb_dp45_stats* stats);
int tb_dp45_end(tb_handle* h, double* f_out, double* dense_out, double* dense_times, int64_t max_dense,
                tb_dp45_stats* stats, int flags);

/* Synchronises the handle's stream; TB_ERR_TIMEOUT when a contraction's
 * bounded wait ran out since the last synchronising call. */
int tb_synchronize(tb_handle* h);

/* Poll limit of the moment-tensor contractions' wait for each staged tile of
 * moments (default 2^22 polls, far above any real copy).  A wait that runs
 * out makes its thread block record the failure, wait (with its own bound)
 * for the copies it still has in flight, and leave its tiles out; the next
 * synchronising call (tb_rhs / tb_scattering_rates with host buffers,
 * tb_synchronize, tb_dp45_poll / tb_dp45_end / tb_dp45_integrate, the
 * adjoint sweeps) returns TB_ERR_TIMEOUT, and the handle stays usable.
 * polls = 0 gives up at once, which exercises that path.  The reference has
 * no device waits (its only failure signal is the step-size underflow of
 * DormandPrince54.hpp:532, 658-661). */
int tb_set_copy_wait_limit(tb_handle* h, int64_t polls);

/* The cudaStream_t every launch of this handle goes to (for event timing). */
void* tb_get_stream(tb_handle* h);

/* acc += collision terms before M^-1 (device pointers): the scatter-adds of
 * singleScatteringPropagator (ScatteringChannel.cpp:649) for one channel, or
 * all channels with ch = -1.  The bare collision kernels, for timing and for
 * callers that compose their own right-hand side. */
int tb_collision_accumulate(tb_handle* h, int ch, const double* f, double* acc);

/* The tuple cache of the reference, byte for byte: what
 * ScatteringChannel::precalculateIndices writes to and reads from
 * "<scatteringName>.scattIndices" (src/Physics/Scattering/
 * ScatteringChannel.cpp:421-458, 516-534): int32 nSecSplits of every leg's
 * mesh (x, y), uint64 tuple count, then per tuple the legs' element ids and
 * the umklapp column as int32.  tb_write_scatt_indices saves a channel's
 * tuple list (enumerated on the device or supplied); tb_read_scatt_indices
 * reads one for tb_channel_desc.tuples: nsplit (2 * nlegs values, or NULL
 * to skip the check) must match the header as in the reference; with ids ==
 * umk == NULL it only returns the count. */
int tb_write_scatt_indices(const tb_handle* h, int ch, const char* path);
int tb_read_scatt_indices(const char* path, int nlegs, const int32_t* nsplit, int64_t* n_tuples, int32_t* ids,
                          int32_t* umk, int64_t capacity);

/* Contraction schedule of a channel's moment-tensor group: bulk-copy
 * pipeline stages (1 or 2); the instance schedule in `pair` -- 0 one
 * instance per thread, 1 two instances share each moment read, 2 / 3 / 4 / 5
 * run-minor (one lane per run, 32 / 8 / 4 / 16 runs per tuple and 1 / 4 / 8 /
 * 2 tuples per warp, for groups shared by many runs of a batch); and, after
 * tb_options.autotune, the fastest measured launch time in seconds (0 when
 * not tuned).  Monte-Carlo channels report stages 0, 0 seconds and pair 6
 * when the quadrature visits only the points inside the simplices (a list
 * of the tuples with such points and a 64-bit mask per tuple, built at
 * creation when the channel has at most 64 Monte-Carlo points; same sums as
 * the full quadrature for finite f), else 0 (every point of every tuple).
 * No counterpart in the reference. */
int tb_channel_schedule(const tb_handle* h, int ch, int32_t* stages, int32_t* pair, double* seconds);

/* Monte-Carlo channels: the tuples with at least one point inside the
 * simplices and the number of such (tuple, point) pairs, i.e. the work the
 * quadrature does per instance; -1, -1 when the channel has no such list
 * (moment-tensor layout, or more than 64 Monte-Carlo points).  On a sharded
 * handle, this handle's part.  No counterpart in the reference. */
int tb_channel_points_inside(const tb_handle* h, int ch, int64_t* n_tuples, int64_t* n_points);

/* Pins the contraction schedule of a channel's moment-tensor group (every
 * channel of that group): stages 1..2, pair as tb_channel_schedule reports it
 * (2..5 only for groups of 8..1024 runs with at most 3 legs).  Monte-Carlo
 * groups take stages 0 with pair 0 (every point) or 6 (points inside only).  The result is
 * the same up to FP64 summation order; the time is not.  No counterpart in the
 * reference. */
int tb_set_channel_schedule(tb_handle* h, int ch, int32_t stages, int32_t pair);

/* Out-scattering rates, state-shaped, M^-1 applied (replaces
 * ScatteringChannel::scatteringRates(status, which), src/Physics/Scattering/
 * ScatteringChannel.cpp:544-612, and MaterialStatus::scatteringRates,
 * src/Physics/Status/MaterialStatus.cpp:170-187): for every selected leg the
 * forms of that leg become the constant in / out unit forms and its block,
 * with the opposite sign of propagate, lands in the leg's band.
 * ch = -1: every channel (channels with zero amplitude contribute nothing);
 * leg = -1: every leg.  rates is overwritten.  flags: TB_PTR_HOST. */
int tb_scattering_rates(tb_handle* h, int ch, int leg, const double* f, double* rates, int flags);

/* ---------------------------------------------------------------- adjoint
 * No counterpart in the reference, which has no derivatives.  The right-hand
 * side is F(f) = M^-1 (sum_c amplitude_c C_c(f) + V f) (ScatteringChannel::
 * propagate and Vlasov::propagate followed by Function::applyInverseMass).
 * grad_amp arrays have tb_num_channels(h) entries in channel order and are
 * HOST memory whatever the flags say. */

typedef struct tb_adjoint_stats {
    double  t_obs;            /* time of the observable (the last dense output)   */
    double  dense_s;          /* its fraction inside the step that produced it    */
    int64_t steps;            /* accepted steps up to and including that step     */
    int64_t attempts;         /* forward attempts (accepted + rejected)           */
    int64_t checkpoints;      /* states stored by the forward sweep               */
    int64_t rhs_evals;        /* right-hand sides: forward + recomputation        */
    int64_t vjp_evals;        /* transposed right-hand sides of the reverse sweep */
    int32_t status;
    int32_t checkpoint_every;
} tb_adjoint_stats;

/* grad_f = (dF/df)^T theta at f, grad_amp[c] = <theta, dF/d amplitude_c>.
 * flags: TB_PTR_HOST for f, theta, grad_f; TB_NO_DRIFT; TB_NO_COLLISIONS. */
int tb_adjoint_rhs_vjp(tb_handle* h, const double* f, const double* theta, double* grad_f, double* grad_amp,
                       int flags);

/* Forward sweep of a differentiable integration (single-run handles): the
 * same adaptive integration as tb_dp45_integrate from t0 to t1 with dense
 * step dense_step, which also logs every accepted step (t, dt) and stores
 * f after every `checkpoint_every`-th accepted step in device memory.
 * max_steps bounds the accepted steps (TB_ERR_CAPACITY beyond); the
 * checkpoints take (max_steps / checkpoint_every + 2) * ndofs doubles.
 * f_obs (may be NULL) receives f at the last dense output time. */
int tb_adjoint_forward(tb_handle* h, const double* f0, double t0, double t1, double dense_step,
                       int checkpoint_every, int64_t max_steps, double* f_obs, tb_adjoint_stats* st, int flags);

/* Reverse sweep for the observable J = <lambda_T, f(t_obs)>: grad_f0 = dJ/df0
 * and grad_amp[c] = dJ/d amplitude_c of the step sequence the forward sweep
 * chose (step sizes frozen; their dependence on f is not differentiated).
 * Recomputes each segment of checkpoint_every steps from its checkpoint. */
int tb_adjoint_backward(tb_handle* h, const double* lambda_T, double* grad_f0, double* grad_amp,
                        tb_adjoint_stats* st, int flags);

/* tb_adjoint_forward followed by tb_adjoint_backward. */
int tb_adjoint_integrate(tb_handle* h, const double* f0, double t0, double t1, double dense_step,
                         int checkpoint_every, int64_t max_steps, const double* lambda_T, double* f_obs,
                         double* grad_f0, double* grad_amp, tb_adjoint_stats* st, int flags);

/* The frozen step sizes of the last forward sweep (up to cap of them), their
 * count and the dense fraction of the observable's step. */
int tb_adjoint_steps(tb_handle* h, double* dts, int64_t cap, int64_t* n_steps, double* dense_s);

/* Fixed-step Dormand-Prince: n_steps steps of sizes dts (HOST array) from f0,
 * then the dense output at fraction dense_s of the last step, into f_out.
 * The same arithmetic as the adaptive integration's accepted steps; replays
 * a logged step sequence (the map tb_adjoint_backward differentiates). */
int tb_dp45_replay(tb_handle* h, const double* f0, const double* dts, int64_t n_steps, double dense_s,
                   double* f_out, int flags);

/* The error norm of ONE band (what Band::relativeError computes for one
 * population) for callers that cannot call cudaMalloc when they need it -- a
 * host application whose device memory is fully reserved by its own pool
 * allocator, or code that must not risk the implicit device synchronisation of
 * cudaMalloc/cudaFree inside its own asynchronous work.  It needs no handle and
 * allocates nothing: err, pop (n_elements*3 doubles each, linear-form layout)
 * and result (one double) are device memory supplied by the caller, and the
 * per-block partial sums live in a fixed 64 KiB device array of the library
 * (held on every device that loads the library until the process exits).
 * Limit: n_elements <= 1,048,576 (TB_ERR_CAPACITY beyond).  The first call on
 * a device looks up that array's device address, so make it before any stream
 * capture.  The address is kept for the life of the process: a process that
 * resets the device (cudaDeviceReset) or otherwise tears down its primary
 * context must not call this entry point on that device again.  All calls
 * share the array: calls that overlap on the GPU race.
 * Launches on `stream` (a cudaStream_t, NULL = default stream) and does not
 * synchronise.  No counterpart in the reference. */
int tb_band_relative_error_noalloc(const double* err, const double* pop, int64_t n_elements, double elem_volume,
                                   double statistics, double rel_tol, double abs_tol, double penalisation,
                                   double* result, void* stream);

/* The device's FP64 fused multiply-add throughput in FMAs per second,
 * measured by a register-resident kernel (8 independent FMA chains per
 * thread, 8 blocks of 256 threads per SM) timed with CUDA events: the
 * roofline denominator of the FP64-bound kernels (the run-minor batched
 * contraction, the Monte-Carlo quadrature).  Takes a fraction of a second.
 * No counterpart in the reference. */
int tb_fp64_fma_rate(int device, double* fma_per_second);

/* ---------------------------------------------- tuple sharding across GPUs
 * One run split over shard_count processes, one GPU each: the process with
 * tb_options.shard_rank = r keeps the r-th contiguous part of every channel's
 * tuple list (tb_shard_range), so every tuple is evaluated by exactly one GPU
 * -- the work split that the TBB reduce of ScatteringChannel<2,L>::propagate
 * (src/Physics/Scattering/ScatteringChannel.cpp:651-670) makes across host
 * threads.  Each process then holds a partial collision accumulator.  Once the
 * handles are connected (tb_shard_connect), every collision evaluation ends
 * with one in-place FP64 sum all-reduce (NCCL) of that accumulator, before the
 * replicated drift term and M^-1: tb_rhs, tb_channel_propagate,
 * tb_collision_accumulate, tb_scattering_rates, every DP45 stage (inside the
 * captured attempt graph), the adjoint sweeps (the collision VJP and the
 * amplitude gradients) and tb_dp45_replay.  The state and the integrator are
 * replicated: the all-reduced accumulator is the same on every rank, so every
 * rank takes the same steps.  On a connected handle these calls are
 * collective: every rank makes the same calls in the same order.  Unconnected,
 * a sharded handle returns its partial sums (their sum over the ranks is the
 * full operator).  A sharded handle holds only its part of each tuple list, so
 * tb_write_scatt_indices refuses it.  NCCL (libnccl.so.2) is loaded on the
 * first tb_shard_* call that needs it.  No counterpart in the reference (one
 * process per Material there). */
#define TB_SHARD_ID_BYTES 128

/* The part [begin, end) of n_tuples tuples that rank `rank` of n_ranks keeps:
 * contiguous, in list order, boundaries on multiples of 128 tuples (whole
 * moment-tensor tiles), as even as that allows.  Host arithmetic only. */
int tb_shard_range(int64_t n_tuples, int rank, int n_ranks, int64_t* begin, int64_t* end);

/* A new communicator id (TB_SHARD_ID_BYTES bytes) into `id`.  One rank makes
 * it; the caller hands the bytes to the other ranks (a store, a broadcast). */
int tb_shard_unique_id(void* id);

/* Joins the handle to the communicator `id` as rank shard_rank of
 * shard_count (the handle's options).  Every rank calls it.  timeout_s bounds
 * this call and every later wait on the handle's stream: a wait that runs out
 * aborts the communicator and returns TB_ERR_TIMEOUT, and the handle's
 * collective calls fail from then on. */
int tb_shard_connect(tb_handle* h, const void* id, double timeout_s);

/* Channel ch's part on this handle: its first tuple's index in the full list
 * and the full list's length (begin 0 and the local count when unsharded). */
int tb_shard_info(const tb_handle* h, int ch, int64_t* begin, int64_t* n_total);

#ifdef __cplusplus
}
#endif

#endif /* TORTOISE_B200_H */
