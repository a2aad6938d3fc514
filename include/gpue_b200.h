/*
 * gpue_b200.h -- C ABI of the B200-native split-operator Gross-Pitaevskii step.
 *
 * This is the drop-in boundary for GPUE's time stepper.  Plain C types only
 * (pointers, sizes, PODs); every call returns a status code and never exits.
 * The entry points replace these GPUE interfaces (GPUE-group/GPUE):
 *
 *   gpue_ctx_create      init() + generate_fields()  src/init.cu:40-356,
 *                        src/operators.cu:722-992 (grids, K, A, V, operator
 *                        tables), with the Grid keys of include/ds.h:86-196
 *                        passed as a gpue_params POD
 *   gpue_set_operators   set_variables(par, ev_type)  src/init.cu:358-497
 *   gpue_set_wfc /
 *   gpue_get_wfc         the "wfc"/"wfc_gpu" Grid entries (src/init.cu:525-539,
 *                        src/evolution.cu:430, 906-907)
 *   gpue_evolve          evolve(par, numSteps, gstate, buffer)
 *                        include/evolution.h:54-57, src/evolution.cu:260-908
 *   gpue_energy          energy_calc(par, wfc)  src/split_op.cu:208-375
 *   gpue_observables_get the energy terms and moments computed from written
 *                        wavefunctions by julia/calc_energy.jl:32-66 and
 *                        py/en.py:44-66
 *   gpue_find_vortices   Tracker::findVortex  src/tracker.cu:102-166
 *   gpue_snapshot_*      binary counterpart of FileIO::writeOut/readIn
 *                        (src/fileIO.cu:13-72) for checkpoint and resume
 *   gpue_last_error      cudaHandleError/cudaCheckError/cufftHandleError
 *                        (src/split_op.cu:40-59) report-and-exit replaced by
 *                        status codes plus a message
 *
 * Units follow the caller: GPUE itself uses SI with the Rb-87 mass; hbar = m = 1
 * is equally valid.  Grids are square (2D) or cubic (3D), x fastest in memory
 * (index x + xDim*(y + yDim*z)), x_i = -xMax + i*dx with dx = xMax/(xDim/2),
 * as GPUE's generate_p_space lays them out.
 *
 * Threading: a context owns one CUDA stream; calls on one context must not
 * overlap; distinct contexts may be used from distinct threads.
 */
#ifndef GPUE_B200_H
#define GPUE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GPUE_B200_ABI_VERSION 2

typedef enum gpue_status {
    GPUE_OK = 0,
    GPUE_ERR_INVALID_ARG = 1,   /* bad size, pointer or flag */
    GPUE_ERR_UNSUPPORTED = 2,   /* grid length without a compiled FFT plan, ... */
    GPUE_ERR_CUDA = 3,          /* a CUDA runtime call failed (message in last_error) */
    GPUE_ERR_OUT_OF_MEMORY = 4, /* device allocation failed or budget exceeded */
    GPUE_ERR_AST = 5,           /* equation string did not parse */
    GPUE_ERR_STATE = 6,         /* call out of order (e.g. no wavefunction set) */
    GPUE_ERR_TIMEOUT = 7,       /* a bounded device wait gave up, or a served request's
                                   deadline passed */
    GPUE_ERR_CANCELLED = 8      /* a served request was cancelled (gpue_server_cancel) */
} gpue_status;

enum { GPUE_PREC_FP64 = 0, GPUE_PREC_FP32 = 1 };
enum { GPUE_MEM_HOST = 0, GPUE_MEM_DEVICE = 1 };
enum { GPUE_C128 = 0, GPUE_C64 = 1 };
/* gauge field presets (GPUE's -A flag, src/ds.cu:300-331) */
enum { GPUE_GAUGE_ROTATION = 0, GPUE_GAUGE_CONSTANT = 1 };

typedef struct gpue_ctx gpue_ctx;

/* The Grid keys evolve() and its callers read (src/evolution.cu:266-332). */
typedef struct gpue_params {
    int32_t dimnum;            /* 2 or 3 ("dimnum", -c) */
    int32_t xDim, yDim, zDim;  /* equal; zDim = 1 in 2D (-x -y -z) */
    double xMax, yMax, zMax;   /* half box widths ("xMax", -b) */
    double hbar, mass;         /* HBAR (include/constants.h:20), "mass" */
    double omegaX, omegaY, omegaZ, gammaY; /* trap (-X -Y -Z -G) */
    double x0_shift, y0_shift, z0_shift;   /* trap centre shifts (-U -V -Q) */
    double omega;              /* rotation rate scaling the gauge field (-w) */
    double interaction;        /* -i */
    double gDenConst;          /* nonlinear prefactor; gN = interaction*gDenConst */
    double gdt, dt;            /* imaginary / real time steps (-T -t) */
    int32_t gpe;               /* nonlinear term on (-s) */
    int32_t corotating;        /* gauge passes and L energy term on (-l) */
    int32_t gauge;             /* GPUE_GAUGE_* (-A) */
    int32_t ramp, ramp_type;   /* gauge ramp in imaginary time (-R) */
    int32_t precision;         /* GPUE_PREC_FP64 (plain) or GPUE_PREC_FP32 (fused) */
    int32_t device;            /* CUDA device ordinal (-C) */
    int32_t reserved[8];       /* zero */
} gpue_params;

typedef struct gpue_evolve_opts {
    int32_t energy_calc_steps;     /* energy every k steps (0: never), "-E thr k" */
    double energy_calc_threshold;  /* early-stop threshold (imaginary time) */
    int32_t threshold_abs;         /* 0: |E_old-E| < thr*E_old as GPUE, 1: |E_old-E| < thr */
    int32_t polish_steps;          /* FP64 steps after an FP32 imaginary-time run */
    int32_t graph_chunk;           /* steps per captured CUDA graph; 0 = automatic */
    int32_t no_sync;               /* 1: return once the steps are enqueued on the
                                      context stream (no energy checks allowed);
                                      result then holds steps_done and launches only */
    int32_t step_offset;           /* first step index (GPUE starts every evolve() at
                                      0); lets a run continue in slices with the same
                                      time = Dt*i and gauge order i%2 */
    int32_t norm_guard;            /* real time only: rescale to the starting norm each
                                      step (a no-op in exact arithmetic); -1 = on for
                                      the FP32 form, off for FP64; 0 off; 1 on */
    int32_t norm_guard_period;     /* guard every 1, 2 or 4 steps; 0 = default (2): the
                                      factor of a step's norm scales the next step's
                                      kinetic phase */
    int32_t reserved[3];
} gpue_evolve_opts;

typedef struct gpue_evolve_result {
    int32_t steps_done;
    int32_t early_stop;
    int32_t n_energies;
    int32_t reserved0;
    double energy;     /* last energy computed, NaN if none */
    double norm;       /* sum |psi|^2 dV of the final state */
    double device_ms;  /* device time of the step loop (CUDA events) */
    int64_t kernel_launches; /* kernels enqueued by this call */
} gpue_evolve_result;

int gpue_abi_version(void);

/* Defaults of GPUE's parseArgs (src/parser.cu:14-67) in the given units. */
gpue_status gpue_default_params(gpue_params* p);

/* init(): validates sizes, allocates the device state and builds the
 * per-axis operator tables.  Fails with GPUE_ERR_UNSUPPORTED for lengths with
 * no compiled FFT plan (see gpue_supported_length). */
gpue_status gpue_ctx_create(const gpue_params* p, gpue_ctx** out);
gpue_status gpue_ctx_destroy(gpue_ctx* ctx);
const char* gpue_last_error(const gpue_ctx* ctx);

/* 1 if an FFT plan is compiled for this line length in this precision. */
int gpue_supported_length(int32_t precision, int32_t n);

/* set_variables(): prepares the imaginary (0) or real (1) time operators. */
gpue_status gpue_set_operators(gpue_ctx* ctx, int32_t ev_type);

/* Wavefunction in/out, x fastest; mem = GPUE_MEM_*, dtype = GPUE_C128/C64.
 * Host pointers may be pageable or pinned; device pointers must be on the
 * context's device. */
gpue_status gpue_set_wfc(gpue_ctx* ctx, const void* psi, int32_t mem, int32_t dtype);
gpue_status gpue_get_wfc(gpue_ctx* ctx, void* psi, int32_t mem, int32_t dtype);

/* evolve(): nsteps split-operator steps, imaginary (gstate 0) or real (1)
 * time.  Step numbering restarts at 0 on every call as in GPUE (time = Dt*i,
 * gauge order alternates with i%2).  opts and result may be NULL. */
gpue_status gpue_evolve(gpue_ctx* ctx, int32_t nsteps, int32_t gstate,
                        const gpue_evolve_opts* opts, gpue_evolve_result* result);

/* energy_calc(): <psi|H|psi> dV of the current state (no division by the norm). */
gpue_status gpue_energy(gpue_ctx* ctx, double* energy);

/* sum |psi|^2 dV of the current state. */
gpue_status gpue_norm(gpue_ctx* ctx, double* norm);

/* Observables of the current state, one real-space pass plus the kinetic
 * passes of energy_calc.  Replaces the post-processing GPUE does on written
 * wavefunctions:
 *   - the energy split into its terms as julia/calc_energy.jl:32-66 prints
 *     them (kinetic, potential, internal, angular-momentum), with the terms
 *     formed exactly as energy_calc (src/split_op.cu:208-375) forms them:
 *     plain sums times dV, V including the m|A|^2/2 gauge term, and the
 *     gauge term through GPUE's forward difference derive()
 *     (src/kernels.cu:58-71, no periodic wrap);  e_kinetic + e_potential +
 *     e_interaction + e_rotation = energy = gpue_energy() up to rounding;
 *   - the density moments of py/en.py:44-50 (expectValueR with X, Y, R =
 *     X^2+Y^2 and Q = X^2-Y^2), integrated with np.trapz's weights (1/2 on
 *     the first and last point of each axis) times dV; x is the contiguous
 *     axis;
 *   - <L_z> = sum Re[conj(psi) (-i hbar)(x d+y psi - y d+x psi)] dV with the
 *     same forward differences, so e_rotation = -omega*omegaY * lz for the
 *     rotation gauge with omegaX = omegaY.
 * None of the values is divided by the norm. */
typedef struct gpue_observables {
    double norm;            /* sum |psi|^2 dV */
    double energy;          /* sum of the four terms below */
    double e_kinetic;       /* sum_k K |psi_k|^2 / N dV */
    double e_potential;     /* sum V |psi|^2 dV */
    double e_interaction;   /* sum gN/2 |psi|^4 dV (0 without the nonlinearity) */
    double e_rotation;      /* sum Re[conj(psi) i hbar A.d+ psi] dV (corotating only) */
    double x, y, z;         /* trapezoid <x>, <y>, <z> (0 for absent axes) */
    double r2;              /* trapezoid <x^2 + y^2> */
    double q;               /* trapezoid <x^2 - y^2> */
    double lz;              /* <L_z> */
    double reserved[4];
} gpue_observables;

gpue_status gpue_observables_get(gpue_ctx* ctx, gpue_observables* out);

/* Observables at the energy checks of gpue_evolve (the survey's "fused into
 * the check passes"): with an array set, every check runs the observables
 * reduction in place of energy_calc's real-space pass (one read of psi
 * either way; the energy it leaves is energy_calc's, summed per term) and
 * check k of each gpue_evolve call (k counted from 0; gpue_evolve_result
 * .n_energies of them) is stored in out[k] for k < cap.  out must stay valid
 * while it is set; NULL / 0 turns recording off.  Single contexts only: the
 * batch and server paths keep the plain energy check. */
gpue_status gpue_set_check_observables(gpue_ctx* ctx, gpue_observables* out, int32_t cap);

/* Binary snapshots for checkpoint and resume (GPUE only has the text dumps of
 * FileIO::writeOut/readIn, src/fileIO.cu:13-72, restarted with -r).  A
 * snapshot holds the state exactly as the context keeps it (the precision it
 * steps in, the imaginary-time renormalisation still pending, the energy of
 * the latest check that the next early-stop test compares with), the
 * gpue_params it belongs to, the caller's phase and step, and a checksum.
 * Loading it into a context with the same parameters (precision and device
 * may differ) and continuing with gpue_evolve's step_offset = step repeats
 * the uninterrupted run bit for bit in the same precision, except with the
 * real-time norm guard (on by default for FP32), which every gpue_evolve call
 * starts afresh from the norm it finds: then to FP32 round-off.  Field tables and
 * parameter-file fields are not part of a snapshot: install them again.
 * Saves write "<path>.tmp" and rename it over path.  Load fails with
 * GPUE_ERR_INVALID_ARG for another grid or parameters, a bad header, a short
 * file or a checksum mismatch. */
gpue_status gpue_snapshot_save(gpue_ctx* ctx, const char* path, int32_t gstate, int64_t step);
gpue_status gpue_snapshot_load(gpue_ctx* ctx, const char* path, int32_t* gstate,
                               int64_t* step);

/* 2D vortex finder: Tracker::findVortex (src/tracker.cu:102-166), which GPUE
 * runs on a host copy of the state at print steps in real time
 * (src/evolution.cu:430, 483-486), here on the resident state.  Plaquette
 * (i, j), i the row (y index) and j the column (x index), i, j < xDim-1, is
 * examined when sqrt(x_i^2 + x_j^2) < radius (GPUE's x grid on both axes) by
 * summing the wrapped phase steps around (i,j) -> (i+1,j) -> (i+1,j+1) ->
 * (i,j+1); a sum of magnitude >= 1.9 pi marks it with |lround(sum / 2 pi)|,
 * except that the in-radius plaquette visited right after a marked one (rows
 * in order, columns in order within a row) is never marked, as findVortex's
 * cond_x/cond_y counters have it.
 *   marker  xDim*yDim int32 in GPUE's layout (index i*xDim + j), zero except
 *           at marks; may be NULL; mem = GPUE_MEM_HOST or GPUE_MEM_DEVICE
 *           says where marker and list live;
 *   list    the first min(found, cap) marks in visiting order with the
 *           signed winding (x + i y around a point carries +1); may be NULL;
 *   found   number of marks (findVortex's return value).
 * 2D contexts only (GPUE_ERR_UNSUPPORTED otherwise).  The first call on a
 * context allocates a device workspace of about 13 bytes per grid point,
 * kept until gpue_ctx_destroy. */
typedef struct gpue_vortex {
    int32_t i, j;       /* row (y index), column (x index) of the plaquette corner */
    int32_t marker;     /* the value findVortex stores there */
    int32_t winding;    /* signed lround(sum / 2 pi) */
} gpue_vortex;

gpue_status gpue_find_vortices(gpue_ctx* ctx, double radius, int32_t* marker, int32_t mem,
                               gpue_vortex* list, int32_t cap, int32_t* found);

/* The context's cudaStream_t (as void*) for callers that time or order work. */
gpue_status gpue_ctx_stream(gpue_ctx* ctx, void** stream);

/* Parameter-file fields (GPUE's -I file: parse_param_file, src/dynamic.cu:187-222,
 * used by init() and generate_fields, src/init.cu:199-201,
 * src/operators.cu:472-618,808-830).  `text` holds "name = expr" lines in GPUE's
 * grammar; V, Ax, Ay, Az are evaluated once at t = 0 on the grid
 * (x = dx*i - xMax, ...) and replace the harmonic trap / preset gauge, with V
 * getting +0.5*mass*(Ax*Ax+Ay*Ay+Az*Az) unless it is the last entry, as GPUE
 * does.  time_mode 0 keeps GPUE's main() behaviour (static fields only);
 * time_mode 1 also evaluates every time-dependent entry (V, k, Ax, Ay, Az) per
 * point and step as evolve()'s AST kernels do (src/kernels.cu:391-422,632-665).
 * names/values add Grid doubles the expressions may use. */
gpue_status gpue_load_param_text(gpue_ctx* ctx, const char* text, int32_t time_mode,
                                 const char* const* names, const double* values,
                                 int32_t nvalues);

/* parse_eqn + tree_to_array (src/dynamic.cu:227-507) of one expression into
 * GPUE's flat EqnNode_gpu layout {double val; int32 is_dynamic; int32 var;
 * int32 left; int32 right; int32 op_num} (32 bytes each); no device work.
 * *count receives the node count; nodes_out may be NULL to query it. */
gpue_status gpue_ast_parse(const char* expr, const char* const* names, const double* values,
                           int32_t nvalues, void* nodes_out, int32_t cap, int32_t* count);

/* parse_param_file's host part (src/dynamic.cu:162-222, with parse_eqn and
 * tree_to_array, src/dynamic.cu:227-507) on the text of a parameter file:
 * entry `entry` (0-based, in file order) as GPUE's flat EqnNode_gpu array, as
 * allocate_eqn builds it before its device copy.  *nentries receives the number
 * of entries, `name` (name_cap bytes) the entry's name, *time_flag GPUE's
 * "<name>_time" flag (the entry uses t or names an earlier entry).  Lines
 * without '=' continue the previous entry and V gets
 * +0.5*mass*(Ax*Ax+Ay*Ay+Az*Az) unless it is the last entry.  nodes_out may be
 * NULL to query the sizes; no device work. */
gpue_status gpue_ast_parse_file(const char* text, const char* const* names,
                                const double* values, int32_t nvalues, int32_t entry,
                                char* name, int32_t name_cap, int32_t* time_flag,
                                void* nodes_out, int32_t cap, int32_t* count,
                                int32_t* nentries);

/* GPUE's file gauge (-A file: file_A and generate_gauge, src/operators.cu:259-270,
 * 505-520): full-field Ax, Ay, Az (host arrays of xDim*yDim*zDim doubles, x
 * fastest, already multiplied by omega as file_A does; NULL for a zero
 * component, Az ignored in 2D) replace the preset gauge.  V becomes the
 * harmonic trap plus m|A|^2/2 (kharmonic_V, src/operators.cu:994-1008) over
 * the full grid, and the gauge passes apply exp(-i A p dt) per point. */
gpue_status gpue_set_gauge_tables(gpue_ctx* ctx, const double* Ax, const double* Ay,
                                  const double* Az);

/* A full-field potential V (host array of xDim*yDim*zDim doubles, x fastest)
 * in place of the harmonic trap: GPUE's V_gpu as generate_fields leaves it
 * (src/operators.cu:800-831), e.g. ktorus_V for -v torus (src/operators.cu:
 * 1011-1029), including any m|A|^2/2 term.  Call it after
 * gpue_set_gauge_tables, which recomputes the harmonic V.  It also replaces
 * a parameter-file V expression. */
gpue_status gpue_set_potential_table(gpue_ctx* ctx, const double* V);

/* Device pointer of the resident wavefunction and its dtype (GPUE_C128/C64). */
gpue_status gpue_ctx_wfc_device(gpue_ctx* ctx, void** psi, int32_t* dtype);

/* No counterpart in GPUE (which hands its transforms to cuFFT plans,
 * src/ds.cu:11-79): choose, by timing on this device, the FFT radix plan and
 * the lines per CTA of every axis of the context's grid.  Each compiled plan
 * of the axis length and each lines-per-CTA count that fits is timed on four
 * time steps of the context's own schedule (the time kind its operators are
 * built for, imaginary if none), run on the state and then undone; the
 * fastest (by a clear margin over the default) is kept.  Choices are cached per (precision,
 * dimension, length, axis) for the process, so later contexts of the same
 * shape reuse them without timing; flags bit 0 re-times a cached shape.
 * Setting GPUE_AUTOTUNE=1 in the environment makes gpue_ctx_create do this. */
gpue_status gpue_autotune(gpue_ctx* ctx, int32_t flags);

typedef struct gpue_plan_info {
    int32_t n;                     /* line length */
    int32_t ra, rb, rc;            /* radix sequence (ra, [rb, [rc,]] ra) */
    int32_t threads_per_line;
    int32_t lines_per_cta;
    int32_t threads, blocks;       /* CTA size and persistent grid */
    int32_t tuned;                 /* 1 if chosen by gpue_autotune */
    float us, default_us;          /* step times (us) the tuner measured: chosen, default */
} gpue_plan_info;

/* The launch shape the context uses along an axis (0 = x). */
gpue_status gpue_get_plan(gpue_ctx* ctx, int32_t axis, gpue_plan_info* out);

/* The compiled plans of one line length (n, ra, rb, rc, threads_per_line set;
 * the first is the default).  *count receives how many exist; at most cap are
 * written. */
gpue_status gpue_list_plans(int32_t precision, int32_t n, gpue_plan_info* out, int32_t cap,
                            int32_t* count);

/* No counterpart in GPUE: the device time of each pass of a time step of the
 * context's schedule for gstate's time kind.  nsteps steps are run on the
 * state with a CUDA event pair around every pass launch (on the context's
 * stream, so no launch overlaps the next), and then undone: the state and the
 * scalar slots are saved first and put back after.  us[i] receives the mean
 * duration of pass i of a step, kinds[i] what the pass is: 0, 1, 2 a line
 * pass along x, y, z (2 also the z tile pass of a 3D complex64 step), 3 and
 * 4 the forward and inverse XY pass of a 3D complex64 step.  *npass receives
 * the passes per step; at most cap entries are written.  A measurement aid:
 * the results of later calls do not change. */
gpue_status gpue_time_passes(gpue_ctx* ctx, int32_t gstate, int32_t nsteps, float* us,
                             int32_t* kinds, int32_t cap, int32_t* npass);

/* Use the compiled plan (ra, rb, rc, threads_per_line) on one axis of the
 * context, with lines_per_cta lines per CTA (0: the default count).  Fails
 * with GPUE_ERR_INVALID_ARG when no such plan exists or the launch shape does
 * not fit the grid.  Results differ from another plan's only by round-off. */
gpue_status gpue_set_plan(gpue_ctx* ctx, int32_t axis, int32_t ra, int32_t rb, int32_t rc,
                          int32_t threads_per_line, int32_t lines_per_cta);

/* No counterpart in GPUE: sum |psi|^2 * dV of a wavefunction the caller owns
 * on the current device, written to *out (device memory the caller owns),
 * for callers that must not trigger any device allocation, such as a server
 * that reserved its whole memory budget up front.  The library allocates
 * nothing here: the reduction scratch is a fixed 1 MiB device array that
 * every GPU loading the library holds until exit, which caps npoints at
 * 2^28 (larger sizes return GPUE_ERR_INVALID_ARG with a message on stderr).
 * Asynchronous on `stream` (a cudaStream_t, may be NULL).  Every call looks
 * up the array's device address on the current device (a lookup, no
 * allocation); the first call on a device also loads the library's device code
 * there, so make that first call before any stream capture.  All calls share
 * the array, so calls whose kernels can overlap on the GPU race; order them on
 * one stream.  dtype is GPUE_C128 or
 * GPUE_C64. */
gpue_status gpue_norm_noalloc(const void* psi, int32_t dtype, int64_t npoints, double dV,
                              double* out, void* stream);

/* ---- batches of independent solves (no counterpart in GPUE, which runs one
 * solve per process): each context keeps its own state, operators and
 * parameters; solves with the same precision, dimension, grid and pass
 * schedule share one kernel launch per pass, the groups run side by side on
 * their own streams, and the whole run replays as captured CUDA graphs with
 * the energy check on the device.  Each solve stops independently: it is
 * frozen (its kernels skip it) from the check where it meets the early-stop
 * rule of gpue_evolve.  Contexts must live on one device and must not carry
 * parameter-file fields or a ramp; the batch does not own them, and they
 * must outlive it. */
typedef struct gpue_batch gpue_batch;

typedef struct gpue_batch_opts {
    int32_t energy_calc_steps;     /* check every k steps (k*i, as gpue_evolve); 0: none */
    double energy_calc_threshold;  /* early-stop threshold (imaginary time) */
    int32_t threshold_abs;         /* 1: |E_old-E| < thr; 0: |E_old-E| < thr*E_old */
    int32_t max_steps;             /* steps per solve at most (>= 1) */
    int32_t norm_guard;            /* as gpue_evolve_opts.norm_guard */
    int32_t segments_per_launch;   /* check segments per graph launch; 0 = automatic */
    int32_t autotune;              /* 1: gpue_autotune every solve first (cached per shape) */
    int32_t reserved[5];
} gpue_batch_opts;

typedef struct gpue_batch_result {
    int32_t steps_done;  /* steps this solve ran */
    int32_t early_stop;  /* 1 if it met the threshold */
    double energy;       /* energy of its last check, NaN if none */
} gpue_batch_result;

typedef struct gpue_batch_stats {
    double device_ms;         /* device time of the whole run (CUDA events) */
    int64_t kernel_launches;  /* kernels launched, graph nodes included */
    int64_t graph_launches;
    double point_steps;       /* sum over solves of grid points x steps run */
} gpue_batch_stats;

gpue_status gpue_batch_create(gpue_ctx* const* ctxs, int32_t n, gpue_batch** out);
gpue_status gpue_batch_destroy(gpue_batch* batch);
const char* gpue_batch_last_error(const gpue_batch* batch);
/* Runs every solve from its current state; results[i] belongs to ctxs[i];
 * results and stats may be NULL.  Afterwards each context holds its final
 * state as if gpue_evolve had run it alone. */
gpue_status gpue_batch_evolve(gpue_batch* batch, int32_t gstate, const gpue_batch_opts* opts,
                              gpue_batch_result* results, gpue_batch_stats* stats);

/* ---- serving (no counterpart in GPUE): a request loop on one device that
 * admits solves as HBM budget and slots free up, keeps each admitted solve's
 * wavefunction and operators resident, and steps all resident solves together
 * (continuous batching).  A worker thread runs ticks of check_steps steps:
 * every tick advances every resident solve by check_steps steps (solves of
 * one kind share launches as in gpue_batch_*), then checks each one's energy;
 * a solve leaves at the tick where it meets the threshold (imaginary time) or
 * reaches max_steps, and requests that arrived meanwhile are admitted before
 * the next tick.  A solve's arithmetic does not depend on the other solves
 * resident with it: its result is the same alone and in any mix. */
typedef struct gpue_server gpue_server;

typedef struct gpue_server_opts {
    int32_t device;
    int32_t precision;         /* form of every solve: GPUE_PREC_FP32 or GPUE_PREC_FP64 */
    int64_t hbm_budget_bytes;  /* device bytes resident solves may hold; 0: 90% of free */
    int32_t check_steps;       /* steps per tick and between energy checks (even, >= 2) */
    int32_t max_active;        /* resident solves at most; 0: no limit */
    double threshold;          /* imaginary-time stop between consecutive checks */
    int32_t threshold_abs;     /* 1: |E_old-E| < threshold; 0: |E_old-E| < threshold*E_old */
    int32_t autotune;          /* 1: gpue_autotune each admitted solve (cached per shape) */
    int32_t reserved[6];
} gpue_server_opts;

typedef struct gpue_request {
    gpue_params params;  /* grid and physics; precision and device are the server's */
    int32_t gstate;      /* 0: imaginary time until the threshold, 1: real time */
    int32_t max_steps;   /* a multiple of check_steps */
    const void* psi0;    /* host complex128, read when the solve is admitted */
    void* psi_out;       /* host complex128, written when it completes; may be NULL */
    int64_t tag;         /* returned with the result */
    double deadline_s;   /* 0: none; else the request fails with GPUE_ERR_TIMEOUT once this
                            many seconds have passed since its submission (checked while it
                            waits and after every tick; a resident solve's state at that
                            tick is written to psi_out) */
} gpue_request;

typedef struct gpue_server_result {
    int64_t tag;
    int32_t status;      /* gpue_status of this solve */
    int32_t steps_done;
    int32_t early_stop;
    int32_t reserved0;
    double energy;       /* energy at the last check */
    double t_submit, t_admit, t_done;  /* seconds on the server clock */
} gpue_server_result;

typedef struct gpue_server_stats {
    int64_t submitted, admitted, completed, failed;
    int32_t active, queued;
    int64_t bytes_resident, bytes_peak, bytes_budget;
    int64_t ticks, kernel_launches;
    double point_steps;  /* grid points x steps run by all ticks */
    double busy_s;       /* device time of the ticks (CUDA events) */
    double admit_s;      /* worker's host time admitting solves (context set-up) */
    double issue_s;      /* worker's host time planning and enqueuing ticks */
    double finish_s;     /* worker's host time returning finished solves */
    int64_t admitted_in_tick;  /* solves admitted while a tick ran on the device */
    int64_t timed_out, cancelled;
} gpue_server_stats;

gpue_status gpue_server_create(const gpue_server_opts* opts, gpue_server** out);
/* Stops the worker; queued and resident solves are dropped. */
gpue_status gpue_server_destroy(gpue_server* server);
const char* gpue_server_last_error(const gpue_server* server);
/* Queues a request (thread-safe); psi0 and psi_out must stay valid until its
 * result is polled. */
gpue_status gpue_server_submit(gpue_server* server, const gpue_request* req);
/* Cancels every queued or resident request with this tag: a queued one
 * leaves at once, a resident one after the tick in flight (its state at that
 * tick is written to psi_out); their results carry GPUE_ERR_CANCELLED.
 * GPUE_ERR_INVALID_ARG when no queued or resident request has the tag.
 * Replaces GPUE's only way to end a run early, the process exit
 * (src/split_op.cu:40-53). */
gpue_status gpue_server_cancel(gpue_server* server, int64_t tag);
/* Moves up to cap finished results into out (*n of them), waiting up to
 * timeout_s seconds when none is ready. */
gpue_status gpue_server_poll(gpue_server* server, gpue_server_result* out, int32_t cap,
                             int32_t* n, double timeout_s);
gpue_status gpue_server_get_stats(gpue_server* server, gpue_server_stats* stats);
/* Seconds since the server was created (the clock of the result times). */
double gpue_server_clock(const gpue_server* server);

#ifdef __cplusplus
}
#endif

#endif /* GPUE_B200_H */
