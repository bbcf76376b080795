/*
 * hydist_b200.h — C ABI of the B200 (sm_100a) ADI shallow-water + sediment library.
 *
 * The reference (GPU-hydist) has no C ABI: its operator surface is
 *   (1) the device structs Argument_Pointers / Array_Pointers (constant.cuh:6-29),
 *   (2) the compile-time case constants of constant.cuh:31-133, and
 *   (3) the Python host calls rep.gpu_init (rep.py:58-142) and
 *       Engine.hydraulic_Calculation (Engine.py:49-469).
 * Every entry point below names the piece of that surface it replaces.
 *
 * Conventions
 *   - All functions return 0 on success and a negative HYD_E* code on failure;
 *     hyd_last_error() then returns a human-readable message (thread-local).
 *   - Grid fields are host-owned, C-contiguous (N+3) x (M+3) arrays, row index i
 *     (x, dX, "N" direction) and column index j (y, dY, "M" direction), exactly
 *     the layout of Global_Variables.py:92-133.  The library copies them in and
 *     out; it never keeps host pointers.
 *   - The library owns all device memory and one CUDA stream per handle.  Calls
 *     on one handle are not thread-safe; separate handles are independent.
 */
#ifndef HYDIST_B200_H
#define HYDIST_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Maximum wet segments per grid line (constant.cuh:31 `segment_limit`). */
#define HYD_SEGMENT_LIMIT 20

/* Error codes. */
#define HYD_OK 0
#define HYD_EINVAL (-1)   /* bad argument */
#define HYD_ECUDA (-2)    /* CUDA runtime error */
#define HYD_ENOMEM (-3)   /* allocation failed */
#define HYD_ESTATE (-4)   /* call out of order (e.g. step before init) */
#define HYD_EDEVICE (-5)  /* a device-side check failed (see hyd_last_error) */

/* Boundary edges, in the order of Argument_Pointers' bc_up/bc_down/bc_left/bc_right
 * and of the rows of boundary_type (support_funcs.cu:632-665):
 *   up    = column j = M (location of vbt),   down  = column j = 2 (vbd),
 *   left  = row    i = 2 (ubt),               right = row    i = N (ubp). */
#define HYD_EDGE_UP 0
#define HYD_EDGE_DOWN 1
#define HYD_EDGE_LEFT 2
#define HYD_EDGE_RIGHT 3

/*
 * HydCaseParams — every __constant__ of the reference's case header
 * (constant.cuh:31-118) plus the run options that Engine.hydraulic_Calculation
 * takes as keywords (Engine.py:49-50).  It replaces "copy constant_<case>.cuh over
 * constant.cuh and recompile" (readme.md:13-15): the values are uploaded at run time.
 * The derived members (dXbp ... HaiChiadT) are stored explicitly because the
 * reference header spells them out as separate literals; hyd_params_derive()
 * recomputes them from dX, dY, dT.
 */
typedef struct HydCaseParams {
    /* grid spacing and time step (constant.cuh:32-47) */
    double dX, dY, dT;
    double dXbp, dX2, dYbp, dY2, dTchia2dX, dTchia2dY, QuyDoiTime, QuyDoiPi, HaiChiadT;
    /* wet/dry limits, wind, smoothing, friction exponent (constant.cuh:54-66) */
    double NANGDAY, H_TINH, Wind, huonggio, Zbandau, heso, mu_mn;
    /* concentrations (constant.cuh:70-74) */
    double NDnen, NDbphai, NDbtrai, NDbtren, NDbduoi;
    /* erosion/deposition and grain properties (constant.cuh:80-101) */
    double Tod, Toe, hstoe, ghtoe, Mbochat, ro, ros, dm, d90, muy, Dorong, Sx;
    /* depth counts, Coriolis, gravity, roughness height (constant.cuh:104-118) */
    double sohn, soha, sohn1, CORIOLIS_FORCE, g, Ks;
    /* run options (Engine.py:49-50, rep.py:152-156) */
    double sediment_start;   /* s; sediment ADI runs while t >= sediment_start (Engine.py:218,338) */
    double bed_change_start; /* s; source gate s_start (Engine.py:226,347) and Exner period (Engine.py:364) */
    int ketdinh;             /* 1 = cohesive source term (Engine.py:49 default True) */
    int kenhhepd;            /* channel mode, vertical channel (rep.py:37; Engine.py:68,156) */
    int kenhhepng;           /* channel mode, horizontal channel (rep.py:36; Engine.py:68,277) */
    int precision_mode;      /* HYD_PRECISION_FP64 (the reference's arithmetic) or HYD_PRECISION_MIXED */
    /* Morphodynamic feedback: no reference counterpart (the reference accumulates dH and
     * never applies it, Sediment_Transport.cu:504).  With bed_feedback = 0 every value
     * below is ignored but bed_period, and the step is the reference's. */
    double morfac;           /* morphological factor of each applied bed change */
    double bed_period;       /* s; Exner update every bed_period s from bed_change_start on;
                                0 = every bed_change_start s (Engine.py:364) */
    int bed_feedback;        /* 1 = apply each bed change to h and re-derive the depths */
    int bed_fixed;           /* the bed stays fixed within this many cells of the grid's edges
                                (the open boundaries' inlet and outlet sections) */
    double bed_min_depth;    /* m; the bed stays fixed where the water is shallower */
} HydCaseParams;

/* precision_mode values */
#define HYD_PRECISION_FP64 0
#define HYD_PRECISION_MIXED 1

/* Fill *p with the values of the reference's constant.cuh (constant.cuh:31-118)
 * and the Engine.hydraulic_Calculation defaults (Engine.py:49-50). */
void hyd_params_default(HydCaseParams* p);
/* Recompute dXbp, dX2, dYbp, dY2, dTchia2dX, dTchia2dY, QuyDoiTime, QuyDoiPi,
 * HaiChiadT from dX, dY, dT (the relations written out in constant.cuh:36-47). */
void hyd_params_derive(HydCaseParams* p);

typedef struct HydSim* hyd_handle;
typedef struct HydBatch* hyd_batch;

/* Message of the last failed call on this thread ("" if none). */
const char* hyd_last_error(void);

/* Library build string (architecture, precision). */
const char* hyd_version(void);

/*
 * Create a simulation of N x M interior cells on CUDA device `device`.
 * Replaces rep.gpu_init's context creation, Pointers.alloc/alloc_on_device_only
 * and the PointersStruct packing (rep.py:58-109, Pointers.py:15-81,169-191).
 * All device fields start zero-filled.
 */
int hyd_create(const HydCaseParams* p, int N, int M, int device, hyd_handle* out);

/* Release all device memory and the stream (replaces ctx.detach, rep.py:171). */
int hyd_destroy(hyd_handle h);

/*
 * Copy one field in from the host.  `name` is one of the Argument_Pointers
 * members that rep.py uploads (rep.py:110-111): "h", "hsnham", "VISCOIDX", "Fw",
 * "Tsxw", "Tsyw", "u", "v", "z", "FS", plus the state fields "t_u", "t_v", "t_z",
 * "H_moi", "htaiz", "Htdu", "Htdv", "dH", "tFS", "VTH", "Kx", "Ky", "Qbx", "Qby",
 * "Kx1", "Ky1" (double, (N+3)*(M+3) values) and "khouot" (int32, (N+3)*(M+3)).
 * `count` must equal the field's element count.  Replaces Pointers.toDevice
 * (Pointers.py:110-122).
 */
int hyd_set_field(hyd_handle h, const char* name, const void* host, size_t count);

/*
 * Copy one field out to the host (any name accepted by hyd_set_field, plus the
 * segment tables "daui","cuoii" (int32, (N+2)*20), "moci" (int32, N+2), "dauj",
 * "cuoij" ((M+2)*20), "mocj" (M+2), and "ubt","ubp" (M+2), "vbt","vbd" (N+2),
 * "hi" (2*(N+3)+2*(M+3)), "hmax" (4: the edge concentration scales 1/(ros*hmax) of
 * preprocess_data, up/down/left/right)).  Replaces Pointers.extract (Pointers.py:148-154).
 */
int hyd_get_field(hyd_handle h, const char* name, void* host, size_t count);

/*
 * Asynchronous read of a grid field of doubles ((N+3)x(M+3), e.g. "z" after a step): the
 * field is snapshotted on the device in order with the steps (two snapshots in turn),
 * and the snapshot is copied to `host` on a separate stream while later steps run, the
 * copies in call order.  `host` should be pinned (cudaHostAlloc / a pinned tensor) for
 * the copy to overlap, and must stay valid and untouched until the read is complete:
 * once hyd_wait_fields returns, or once the second hyd_get_field_async call after it has
 * returned.  No reference counterpart (the reference copies its output fields
 * synchronously, Engine.py:377-468).
 */
int hyd_get_field_async(hyd_handle h, const char* name, void* host, size_t count);

/* hyd_get_field into a DEVICE buffer of the handle's device (the same packed layout and
 * count): a device-to-device copy on the handle's stream, synchronous.  For callers that
 * keep their own device work (e.g. a network's input) beside the simulation. */
int hyd_get_field_device(hyd_handle h, const char* name, void* dst, size_t count);
int hyd_wait_fields(hyd_handle h);

/*
 * Host mirror of "z", "u" or "v": the library keeps two pinned host copies of the field
 * ((N+3)x(M+3) doubles, row-major like hyd_get_field) and hands them out in turn.
 * hyd_mirror_open fills both with the field as it is now.  hyd_mirror_update_async,
 * called after queued steps, brings the next copy up to date on the copy stream while
 * later steps run and returns it in *view: the copy is complete once the next update
 * call (or hyd_wait_fields) has returned, and stays valid until the second later update
 * call.  Between whole-grid events (the
 * set-up, any hyd_set_field / hyd_set_state / hyd_set_params, a step that ran whole-grid
 * passes, channel mode) a step changes the field only inside the rows x columns box of
 * the extended spans, so only that box is copied (*bytes, if given, receives the bytes
 * moved); after one, the whole field.  One mirror per handle; opening another closes
 * the first.  No reference counterpart (the reference keeps hourly host lists of u, v,
 * z, Engine.py:418-420).
 */
int hyd_mirror_open(hyd_handle h, const char* name);
int hyd_mirror_update_async(hyd_handle h, const double** view, size_t* bytes);
int hyd_mirror_close(hyd_handle h);

/*
 * Boundary tables for all four edges (Global_Variables.py:30-66):
 *   boundary_type: 4 x HYD_SEGMENT_LIMIT int32 (0 wall, 1 stage Z, 2 discharge Q);
 *   tables[e]:     nseg[e] x total_time hourly values of Q or Z (bc_up..bc_right);
 *   cc[e]:         nseg[e] x total_time hourly inflow concentrations (CC_u..CC_r).
 * bienQ is derived as in Global_Variables.py:56-66.  total_time must cover every
 * hour index the run reaches plus one (support_funcs.cu:565).
 */
int hyd_set_boundary(hyd_handle h, const int* boundary_type, const double* const* tables,
                     const double* const* cc, const int* nseg, int total_time);

/*
 * New values for the boundary tables set by hyd_set_boundary, of the same shapes
 * (tables[e], cc[e]: nseg[e] x total_time; edges with nseg 0 are skipped): a host that
 * drives the forcing as the run goes (a coupled model updating discharges, levels or
 * inflow concentrations) sends them here between steps.  The values are copied into the
 * library's pinned staging block at once (the caller's arrays are free on return) and
 * uploaded in one transfer queued on the handle's stream, in order with the steps.  No
 * reference counterpart (the reference loads its tables once, Global_Variables.py:39-47).
 */
int hyd_update_boundary(hyd_handle h, const double* const* tables, const double* const* cc);

/*
 * One-time initialisation (rep.py:126-139): Onetime_init, the wet-segment scans
 * Find_Calculation_limits_Horizontal/Vertical, Htuongdoi and preprocess_data
 * (support_funcs.cu:20-58, 230-354, 433-542).  Call after the fields and the
 * boundary tables are set; sets the simulation time to t_start.
 */
int hyd_init(hyd_handle h, double t_start);

/* hyd_init_pickup — hyd_init for a run picked up from saved fields (rep.py:126-131):
 * the wet/dry mask set with hyd_set_field("khouot", ...) before the call replaces the
 * one Onetime_init derives from h; then the segment scans, Htuongdoi and
 * preprocess_data run on it, as in the reference, which loads the pick-up files between
 * Onetime_init and the scans.  u, v, z, FS set before the call are kept (Onetime_init
 * does not touch them). */
int hyd_init_pickup(hyd_handle h, double t_start);

/*
 * Advance `nsteps` full ADI steps (two half-steps each, with the sediment ADI
 * and the Exner update when their start times are reached): the body of the
 * time loop of Engine.hydraulic_Calculation (Engine.py:144-366).  On return
 * *t_out (if not NULL) holds the simulation time.  Work is queued on the
 * handle's stream; the call returns after the launches are queued unless
 * `sync` is non-zero.
 */
int hyd_step(hyd_handle h, int nsteps, int sync, double* t_out);

/*
 * hyd_run — the time loop of Engine.hydraulic_Calculation (Engine.py:49-50, 144-412):
 * steps of dT while t < Tmax, and at every output time, a time t that is a whole multiple
 * of `interval` s (the reference's `int(t) % interval == 0` with t integral,
 * Engine.py:398; interval <= 0: only at the end), the reference's check of z, u, v (and
 * FS) for non-finite values (Engine.py:402-412), then cb(h, t, user) if cb is not NULL
 * (where the reference appends u, v, z to its output lists, the host reads fields with
 * hyd_get_field).  A non-finite value ends the run with HYD_EDEVICE and the time in the
 * message, the state left as it was then (the reference returns its lists there).  A
 * nonzero cb return ends the run with HYD_OK.  *t_out (if not NULL) receives the time
 * reached.  The run ends at the first step end with t >= Tmax, as the reference's loop.
 */
typedef int (*hyd_run_callback)(hyd_handle h, double t, void* user);
int hyd_run(hyd_handle h, double Tmax, double interval, hyd_run_callback cb, void* user, double* t_out);

/*
 * Replace the case parameters between steps (the run options of
 * Engine.hydraulic_Calculation, e.g. sediment_start, bed_change_start, ketdinh, are
 * keyword arguments there and may differ per call, Engine.py:49-50).  The grid size
 * cannot change.
 */
int hyd_set_params(hyd_handle h, const HydCaseParams* p);

/* Current simulation time (host mirror). */
int hyd_get_time(hyd_handle h, double* t);

/* Wait for all queued work on the handle and report device-side errors. */
int hyd_synchronize(hyd_handle h);

/*
 * Domain sums over interior cells i in [2,N], j in [2,M] with khouot == 0, in FP64:
 *   out[0] = sum(H_moi) * dX * dY   (water volume, m^3)
 *   out[1] = sum(FS * H_moi) * dX * dY   (suspended mass / ros scale as in FS)
 *   out[2] = sum(dH) * dX * dY      (accumulated bed change volume)
 *   out[3] = number of wet cells
 *   out[4] = number of non-finite values in z/u/v/FS (the reference's hourly NaN check,
 *            Engine.py:402)
 * n must be >= 5.
 */
int hyd_mass_balance(hyd_handle h, double* out, int n);

/*
 * Water volume budget since hyd_init, in FP64 (the reference has none: it only checks
 * for NaN once an hour, Engine.py:402-412).  Both sweeps' continuity
 * rows are in flux form (_uzSolver/_vzSolver_calculate_preindex,
 * UVZSolver_multithread.cu:345-349, 402-406): summed over the cells a sweep solves, the
 * faces between two solved cells cancel, so the domain's volume changes by the fluxes
 * through its edge faces and by the cells the wet/dry resets open and close
 * (support_funcs.cu:75-186).  The library accumulates exactly those terms on the device
 * every half-step (edge volumes as Kahan sums, one writer per edge):
 *   out[0] net volume into the domain through the four edges (m^3)
 *   out[1] gross inflow volume, out[2] gross outflow volume (m^3)
 *   out[3] volume of the cells opened by the wetting pass (m^3)
 *   out[4] volume of the cells closed by the drying pass (m^3)
 *   out[5] water volume the fed-back bed changes added to the wet cells' depths (m^3;
 *          0 without bed_feedback)
 *   out[6..9] net volume in through the up, down, left, right edge (m^3)
 *   out[10] water volume hyd_add_levels added (m^3; written when n >= 11)
 *   out[11] water volume the continuity rows moved out of the solved cells to wet cells
 *           the sweep did not solve, net, less the level change the stage boundary put on
 *           those cells (m^3; written when n >= 12): the segment scan skips a run starting
 *           at a line's last two cells (support_funcs.cu:230-335), while the neighbours'
 *           rows carry their face flux to it and the boundary still sets its level
 *           (support_funcs.cu:622-668)
 * Closure: between two times, the change of hyd_mass_balance's out[0] equals
 * d(out[0]) + d(out[3]) - d(out[4]) + d(out[5]) + d(out[10]) - d(out[11]).  n must be >= 10
 * (HYD_BUDGET_SLOTS for every slot).  No reference counterpart.
 */
#define HYD_BUDGET_SLOTS 12
int hyd_mass_budget(hyd_handle h, double* out, int n);

/*
 * hyd_mass_balance_noalloc — the sums of hyd_mass_balance (same out[0..4]) computed
 * without any allocation: the per-block partial sums live in a fixed device array of
 * HYD_MASS_NOALLOC_MAX_BLOCKS * 5 + 5 doubles (41 KB) instead of a per-call
 * cudaMallocAsync.  No counterpart in the reference (its hourly check copies whole
 * fields to the host, Engine.py:402).  For callers that must not touch the device
 * allocator between steps, e.g. a monitor running while another allocator (a framework's
 * caching pool) holds the device memory, where a per-call allocation can fail or force
 * the pool to trim mid-run.
 *   nblocks: number of partial-sum blocks, 1..HYD_MASS_NOALLOC_MAX_BLOCKS; HYD_EINVAL
 *            beyond.  nblocks = 148 sums in the order hyd_mass_balance uses.
 * Nothing in the array needs to start at zero (every partial is written before it is
 * read).  The array is one per device and process, shared by all handles on that
 * device: overlapping calls (from two threads, or on two streams not ordered with each
 * other) race on it and must be serialised by the caller.  hyd_create looks the array up
 * with cudaGetSymbolAddress on its device, which loads the module that holds it (with
 * CUDA's lazy module loading nothing loads it earlier), so calls on a handle's device
 * allocate nothing.  Only if that lookup was not possible there does the first call on
 * the device look it up and load the module itself (an allocation by the driver); such a
 * first call must not be made while a stream on that device is being captured.
 */
#define HYD_MASS_NOALLOC_MAX_BLOCKS 1024
int hyd_mass_balance_noalloc(hyd_handle h, int nblocks, double* out, int n);

/* Size in bytes of a checkpoint image, and checkpoint save/restore (replaces the
 * text pick-up of rep.py:43-55 with an exact binary image of every prognostic
 * field, the wet mask, the segment tables and the time). */
int hyd_state_size(hyd_handle h, size_t* bytes);
int hyd_get_state(hyd_handle h, void* buf, size_t bytes);
int hyd_set_state(hyd_handle h, const void* buf, size_t bytes);

/*
 * Quasi-steady support (no reference counterpart; the reference steps every dT through
 * Engine.py:144-366).  A morphodynamic run that needs only the hydraulics' equilibrium
 * between two bed updates can reach it by fewer steps from a predicted state, judged by
 * the plain step: these calls keep that loop on the device.
 *
 * hyd_checkpoint(h, 0) saves the whole device state (every field, the mask, the segment
 * tables, the spans, the water budget, the clock) into one device buffer of the handle
 * (allocated at the first save; the arena's size); hyd_checkpoint(h, 1) restores it, with
 * the time.  One slot per handle; a save replaces the previous one.
 *
 * hyd_set_time(h, t) moves the simulation time (the boundary tables' clock and the
 * sediment, bed-update and hourly table schedules) to t without touching any field.
 *
 * hyd_steady_residual(h, snapshot, out, n >= 2) compares the state with the snapshot
 * taken at the previous call with snapshot = 1, over the wet cells of [2,N] x [2,M]:
 *   out[0] = ||(u, v) - (u0, v0)||_2 / ||(u, v)||_2   (momentum: relative velocity change)
 *   out[1] = ||z - z0||_2 / ||H_moi||_2               (continuity: level change / depth)
 * each an FP64 sum added in a fixed order; HUGE_VAL before the first snapshot, with no
 * wet cell or no flow, and for a non-finite sum (so that such a state is never taken for
 * steady).  With snapshot = 1 the current u, v, z become the snapshot.  Synchronous.
 *
 * hyd_add_levels(h, du, dv, dz, i0, j0, rows, cols, ld) adds DEVICE arrays of FP32
 * increments (element r*ld + c belongs to cell (i0 + r, j0 + c) of the (N+3) x (M+3)
 * grid) to u, v and z on the wet cells of [2,N] x [2,M] (a cell whose depth would fall to
 * H_TINH or below keeps its level), and re-derives H_moi and the face depths Htdu, Htdv
 * there (update_h_moi, support_funcs.cu:60-73; Htuongdoi 338-354).  The water it adds is
 * kept in hyd_mass_budget's out[10].  Synchronous.
 */
int hyd_checkpoint(hyd_handle h, int restore);
int hyd_set_time(hyd_handle h, double t);
/*
 * hyd_quasi_steady_period: one bed period of the quasi-steady form with the calls above,
 * in the library (no host round trip between them): checkpoint; the optional jump
 * (du/dv/dz device arrays as hyd_add_levels; null for none); the last `warm` steps of the
 * period with the steady residual after each (from the min_warm-th on, both components
 * below `gate` and no non-finite value accept, and the period's last step, which makes
 * its bed update, is taken); a rejected jump retried once from the checkpoint without it
 * when `retry`; otherwise the checkpoint restored and the period stepped plainly.  A
 * failed device check in a warm step rejects the state.  result[0] = 1 if a warm start
 * was accepted, result[1] = 1 if that was the jump, result[2] = steps taken.  `period`
 * must be a whole number of steps, at least `warm`; the clock must stand on the period's
 * start.
 */
int hyd_quasi_steady_period(hyd_handle h, double period, int warm, int min_warm, double gate, const float* du,
                            const float* dv, const float* dz, int i0, int j0, int rows, int cols, long long ld,
                            int retry, int* result);
int hyd_steady_residual(hyd_handle h, int snapshot, double* out, int n);
int hyd_add_levels(hyd_handle h, const float* du, const float* dv, const float* dz, int i0, int j0, int rows,
                   int cols, long long ld);

/* Device status bits accumulated since creation (waits for the stream):
 *   1 = a line had more than 20 wet segments (the reference overflows its tables),
 *   2 = an edge concentration interpolation index left the grid (skipped),
 *   4 = a single-cell segment on an open edge was met (the reference solves a
 *       negative-size system on stale scratch there; this library solves nothing). */
int hyd_device_status(hyd_handle h, unsigned* status);

/* Number of kernels this library has launched in this process (instrumentation). */
int hyd_launch_count(hyd_handle h, long long* count);

/* The handle's CUDA stream (a cudaStream_t), so that callers can order their own work
 * and time the library with events on the stream it launches on. */
int hyd_get_stream(hyd_handle h, void** stream);

/* Per-phase device timing: while enabled, every phase of the step (boundary, the two
 * line sweeps, smoothing, explicit momentum, resets, state update, scans, sediment, bed,
 * the coefficient passes) is bracketed by CUDA events on the handle's stream.
 * hyd_timing_report() synchronizes and writes lines "name launches total_ms\n" into buf
 * (NUL-terminated), then clears the accumulators.  No reference counterpart (the
 * reference times whole steps on the host).
 *
 * hyd_set_timing_phases() brackets only the phases whose bit is set (bit k = phase k,
 * named by hyd_phase_name(k, &name); 0 turns timing off): each bracket adds two event
 * records to the step, so timing one phase alone disturbs the others least.
 * hyd_set_timing(h, 1) selects every phase. */
int hyd_set_timing(hyd_handle h, int enable);
int hyd_set_timing_phases(hyd_handle h, unsigned int phase_mask);
int hyd_phase_name(int phase, const char** name);
int hyd_timing_report(hyd_handle h, char* buf, size_t buflen);

/* Batches of independent reaches (the batched variant of the operator surface: a config-3
 * ensemble on one device).  hyd_batch_create makes `count` handles on `device`, member k
 * with params[k] and dims[2k] x dims[2k+1] cells; each member is then set up through its
 * own handle (hyd_batch_member: fields, boundary tables, hyd_init) like a single reach.
 * hyd_batch_step advances every member nsteps steps, one step of every member at a time;
 * the members' launches go to their own streams, so they run side by side on the device.
 * With sync, it waits for all members and reports the first device status error.  The
 * handles belong to the batch: hyd_batch_destroy frees them (do not hyd_destroy them).
 * No reference counterpart (the reference runs one reach per process). */
int hyd_batch_create(int count, const HydCaseParams* params, const int* dims, int device, hyd_batch* out);
int hyd_batch_size(hyd_batch b, int* count);
int hyd_batch_member(hyd_batch b, int k, hyd_handle* h);
int hyd_batch_step(hyd_batch b, int nsteps, int sync);
int hyd_batch_destroy(hyd_batch b);

/*
 * Batched launches (no reference counterpart): with hyd_batch_set_fused(b, 1) a batch
 * step whose members all allow it runs every phase of the step as ONE launch for all
 * members, each CTA working for one member (the line sweeps as one persistent launch over
 * every member's lines, one CTA per SM), the whole batch step captured as one CUDA graph
 * per step variant: about 20 launches per batch step instead of 20 per member.  The
 * members must be initialised, at the same time with the same time step and sediment /
 * bed schedule and precision, outside channel mode; a step that a member must take on its
 * own (whole-grid passes after a field was set, a rescan of every line) runs per member
 * and the batched form resumes after it.  Results are the same as the members' own steps
 * (every line and cell is computed by the same code).  hyd_batch_fused_steps reports how
 * many batch steps ran batched.
 */
int hyd_batch_set_fused(hyd_batch b, int on);
int hyd_batch_fused_steps(hyd_batch b, long long* steps);

/*
 * Launch shape of a handle's line sweeps: `ctas` persistent CTAs (0 or more than planned:
 * the planned number, one per SM), and with `wide` = 1 every line a warp's shared-memory
 * slice holds (up to 288 rows) swept by a warp rather than only lines of up to 96 rows.
 * Batch members start at ceil((max(N, M) + 3) / 16) CTAs, wide.  Changing the shape
 * drops the captured step graphs (the next step captures anew).  Results do not depend
 * on the shape beyond rounding (within the parity tolerance).  No reference counterpart
 * (the reference launches one block per line); hydist.tune picks shapes by timing.
 */
int hyd_set_sweep_shape(hyd_handle h, int ctas, int wide);
int hyd_get_sweep_shape(hyd_handle h, int* ctas, int* wide);

/*
 * Convolution kernels of the learned surrogate (BF16 operands on the tensor cores, FP32
 * accumulation in tensor memory).  No reference counterpart: the reference has no learned
 * part.  A layer is a 3x3 convolution over NHWC BF16 activations, output pixel p and tap
 * t = 3 (dy + 1) + (dx + 1) reading input pixel:
 *   HYD_CONV_SAME      (y + dy, x + dx)             same size
 *   HYD_CONV_SAME_ADJ  (y - dy, x - dx)             the adjoint of SAME
 *   HYD_CONV_DOWN      (2y + dy, 2x + dx)           stride 2 down
 *   HYD_CONV_UP        ((y - dy)/2, (x - dx)/2)     stride 2 up (where both are even),
 *                                                   the adjoint of DOWN
 * and zero outside the input.  The data gradient of a layer is hyd_conv_forward with the
 * adjoint mapping, the channel-transposed weights and the output gradient as input.
 *
 * hyd_conv_forward: y[p][n] = act(sum_{t,c} x[map(p,t)][c] w[n][t][c] + bias[n]), n < nout,
 *   times (mask[p][n] > 0) when mask is not null (the ReLU derivative of a data gradient).
 *   cin (16 or 48) channels per input pixel; ncol (16 or 48) the padded output channels the
 *   packed weights hold: w_packed is the tensor cores' shared-memory image, for K step
 *   s = (t cin + c) / 16 a block of ncol x 16 BF16 in which element (n, k) lies at byte
 *   (n / 8) 256 + (k / 8) 128 + (n % 8) 16 + (k % 8) 2.  relu: max(0, .); out_f32: FP32
 *   output instead of BF16.  *err is set to 1 if a wait on the tensor cores timed out.
 *   B x Hout x Wout must stay below 2^31 (HYD_EINVAL otherwise).
 * hyd_conv_wgrad: dw[n][t][c] += sum_p dy[p][n] x[map(p,t)][c] (FP32, n < nout), dy with
 *   ncol channels per pixel; map is the layer's forward mapping.
 * hyd_bias_grad: db[n] += sum_p dy[p][n].
 * hyd_mse_grad: loss += scale sum_p w[p] |pred[p] - target[p]|^2 over nc channels (FP32),
 *   dy[p][c] = 2 scale w[p] (pred - target) as BF16 with ncol channels (zero beyond nc).
 * All run on `stream` (a cudaStream_t) and return after queuing; pointers are device
 * memory, 16-byte aligned.
 */
#define HYD_CONV_SAME 0
#define HYD_CONV_SAME_ADJ 1
#define HYD_CONV_DOWN 2
#define HYD_CONV_UP 3
int hyd_conv_forward(const void* x, int B, int Hin, int Win, int cin, const void* w_packed, const float* bias,
                     int ncol, int nout, int mode, int relu, const void* mask, void* y, int Hout, int Wout,
                     int out_f32, int* err, void* stream);
int hyd_conv_wgrad(const void* x, int B, int Hin, int Win, int cin, int mode, const void* dy, int Hout, int Wout,
                   int ncol, int nout, float* dw, int* err, void* stream);
int hyd_bias_grad(const void* dy, long long npix, int ncol, int nout, float* db, void* stream);
int hyd_mse_grad(const float* pred, const float* target, const float* weight, long long npix, int nc, int ncol,
                 float scale, void* dy, float* loss, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* HYDIST_B200_H */
