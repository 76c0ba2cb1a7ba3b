/*
 * q2d_gpu.h — C ABI of the B200 (sm_100a) explicit finite-volume residual and
 * time-update path of Q2D.
 *
 * Drop-in granularity: one call of q2d_gpu_step() replaces one (or N) executions of the
 * body of Q2D's `Explicit_Step` for one grid level:
 *   src/lib/numerics/time/explicit/Mod_Explicit.f90:10-174
 * i.e. Compute_dt (Mod_dt.f90:10-106), Set_Global_dt (Mod_dt.f90:109-128), Copy_State
 * (Mod_Explicit.f90:177-197), the n_RK stages of {Fill_Ghost_Cell (Lib_Ghost.f90:16-140),
 * Fluxes (Mod_Fluxes.f90:97-234), BC_Fluxes (Mod_BC_Fluxes.f90:49-271), Compute_Sources
 * (Mod_Sources.f90:79-91), RK_Newstate (Lib_Newstate.f90:14-161)}, Compute_Residual
 * (Mod_Diagnostic.f90:438-469) and the TODO/stop logic (Mod_Explicit.f90:120-172).
 *
 * The per-face procedure pointers of the reference (Riemann, rlimiter, Fluxes, RK_Newstate,
 * bound in Assign_Setup.f90:40-62) become the scheme fields of q2d_options: the library
 * specialises its kernels on them once, at q2d_gpu_create().
 *
 * Conventions
 *   - All arrays are host arrays owned by the caller, read or written only during the call
 *     that receives them; no pointer is retained (ownership row of the boundary).
 *   - Block and cell indices in q2d_bc_rec are 1-based like bc.txt (IO_BC.f90:209-402);
 *     `b` is the 1-based index of the block inside its case, in q2d_gpu_add_block order.
 *   - nodes_xy: the reference array node(0:ni,0:nj)%c(2) in Fortran order, i.e. x,y of
 *     node (i,j) at nodes_xy[2*(i + (ni+1)*j) + {0,1}].
 *   - cross_section: nodal A(0:ni,0:nj), i fastest (Lib_Source_Areavariation.f90:53-101);
 *     NULL when the block has no area file.
 *   - P: the reference array P(nprim=4, 1-gc:ni+gc, 1-gc:nj+gc), gc=2, Fortran order
 *     (Mod_Allocate_Data.f90:122-123): variable v of cell (i,j) at
 *     P[v + 4*((i+1) + (ni+4)*(j+1))], i in [-1, ni+2], j in [-1, nj+2]; only the
 *     interior 1..ni x 1..nj is read or written. Variables: rho, u, v, p.
 *   - Every function returns a Q2D_* status; nothing aborts the process (the reference's
 *     `error stop`/`stop` sites map to Q2D_ERR_NONPHYSICAL / Q2D_ERR_NAN).
 *   - Threading: one host thread per context; calls on one context are stream-ordered and
 *     not re-entrant; separate contexts are independent.
 */
#ifndef Q2D_GPU_H
#define Q2D_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------ */
#define Q2D_OK               0
#define Q2D_ERR_BADARG       1   /* invalid argument or call order */
#define Q2D_ERR_OOM          2   /* device or host allocation failed */
#define Q2D_ERR_CUDA         3   /* CUDA runtime error (message in q2d_gpu_last_error) */
#define Q2D_ERR_NONPHYSICAL  4   /* non-physical interface state: Lib_Convective.f90:49-54 */
#define Q2D_ERR_NAN          5   /* NaN or p<0 after the update: Lib_Newstate.f90:327-331 */
#define Q2D_ERR_TIMEOUT      6   /* a bounded device wait ran out */
#define Q2D_ERR_UNSUPPORTED  7   /* option or BC type outside the built path */
#define Q2D_ERR_CAPACITY     8   /* request exceeds a fixed-size buffer or budget */

/* ---- scheme selectors (keywords of Mod_Space.f90:43-76 and Mod_Riemann.f90:25-109) --- */
#define Q2D_LIM_IORD       0   /* first order ('none' / unknown keyword)   Lib_Limiters.f90:26-33 */
#define Q2D_LIM_MINMOD     1   /* 'minmod'                                  :36-46 */
#define Q2D_LIM_VANLEER    2   /* 'vanleer'                                 :49-58 */
#define Q2D_LIM_VANALBADA  3   /* 'vanalbada'                               :61-70 */
#define Q2D_LIM_MC         4   /* 'mc'                                      :73-82 */
#define Q2D_LIM_SUPERBEE   5   /* 'superbee'                                :85-94 */
#define Q2D_LIM_LIMO3      6   /* 'LIMO3'                                   :98-110 */

#define Q2D_RIEMANN_HLLC   0   /* 'HLLC' (default)    Lib_Riemann_HLL.f90:34-123 */
#define Q2D_RIEMANN_HLLE   1   /* 'HLLE'              Lib_Riemann_HLL.f90:126-169 */
#define Q2D_RIEMANN_LLF    2   /* 'LLF' / 'Rusanov'   Lib_Riemann_LF.f90:11-40 */
#define Q2D_RIEMANN_SLAU   3   /* 'SLAU'              Lib_Riemann_SLAU.f90:10-91 */
#define Q2D_RIEMANN_SLAU2  4   /* 'SLAU2'             Lib_Riemann_SLAU.f90:10-53, 94-124 */
#define Q2D_RIEMANN_HLLCP  5   /* 'HLLC+'  HLLC / HLLE blend by the shock sensor,
                                            Lib_Riemann_HLL.f90:572-605 (computes the sensor) */
#define Q2D_RIEMANN_HLLEPP 6   /* 'HLLE++' Roe / HLLE eigenvalue blend by the shock sensor,
                                            Lib_Riemann_HLL.f90:437-533 (computes the sensor) */
#define Q2D_RIEMANN_HLLEM  7   /* 'HLLEM'             Lib_Riemann_HLL.f90:355-434 */
#define Q2D_RIEMANN_HLLC_ROTATED 8 /* 'HLLC Rotated' HLLE / HLLC on rotated normals,
                                            Lib_Riemann_HLL.f90:172-226 */
#define Q2D_RIEMANN_PLLF   9   /* 'PLLF'              Lib_Riemann_LF.f90:44-98 */
#define Q2D_RIEMANN_EXACT  10  /* 'exact' / 'Exact'   Lib_Riemann_Godunov.f90:14-248 */
#define Q2D_RIEMANN_HANEL  11  /* 'Hanel'             Lib_Riemann_AUSM.f90:18-70 */
#define Q2D_RIEMANN_AUSMP  12  /* 'AUSM+'             Lib_Riemann_AUSM.f90:73-128 */
#define Q2D_RIEMANN_AUSMP_UP  13 /* 'AUSM+-up'        Lib_Riemann_AUSM.f90:131-225 (riemann_minf > 0) */
#define Q2D_RIEMANN_AUSMP_UP2 14 /* 'AUSM+-up2'       Lib_Riemann_AUSM.f90:228-321 (riemann_minf > 0) */

#define Q2D_SRC_NONE       0
#define Q2D_SRC_AXI        1   /* [Q2D-Sources] active = axisymmetric   Lib_Source_Axisymmetry.f90:40-78 */
#define Q2D_SRC_AREA       2   /* [Q2D-Sources] active = area_variation Lib_Source_Areavariation.f90:104-144 */

#define Q2D_PREC_FP64      0   /* plain FP64 everywhere */
#define Q2D_PREC_FP32_FLUX 1   /* reconstruction, limiter, Riemann in FP32; state, flux sums,
                                  RK combination, positivity checks and norms in FP64 */

/* BC types served by the path (Mod_BC_Fluxes.f90:79-269 dispatch codes) */
#define Q2D_BC_CONNECTION  101
#define Q2D_BC_SYMMETRY    300
#define Q2D_BC_EXTRAP      400
#define Q2D_BC_STAGNATION  401
#define Q2D_BC_SUPERSONIC  405
#define Q2D_BC_OUTFLOW     406

/* q2d_step_info.todo, the reference's obj_sim_param%TODO (Mod_Explicit.f90:161-169) */
#define Q2D_TODO_CONTINUE  1
#define Q2D_TODO_IO        2
#define Q2D_TODO_END       3

typedef struct q2d_ctx q2d_ctx;

/* Numerics and run control. Mirrors the [Q2D-Numerics]/[Q2D-Parameters]/[Q2D-IO]/
 * [Q2D-Sources] keys read in Register_Numerics.f90:31-76, Register_Sim_Param.f90:26-29,
 * Register_IO.f90:26-35; defaults via q2d_options_default(). */
typedef struct q2d_options {
    int    limiter;         /* Q2D_LIM_*                       flux-limiter */
    int    riemann;         /* Q2D_RIEMANN_*                   riemann-solver */
    int    n_rk;            /* 1 ('euler'), 2 ('RK2'), 3 ('RK3') time-scheme */
    int    time_accurate;   /* 0/1                             time-accurate */
    int    source;          /* Q2D_SRC_*                       [Q2D-Sources] active */
    int    precision;       /* Q2D_PREC_*                      (no reference counterpart) */
    int    rampa_iter;      /* cfl-rise-threshold */
    int    res_diter;       /* res-diter */
    int    sol_diter;       /* sol-diter */
    int    res_relative;    /* 0: stop on residual(1) <= res_threshold (reference);
                               1: stop on residual(1) <= res_threshold * residual(1) of the
                                  first step of the case (relative drop, used by serving) */
    long long itermax;      /* iter-threshold */
    double cfl;             /* cfl */
    double res_threshold;   /* res-threshold */
    double time_threshold;  /* time-threshold */
    double sol_dtime;       /* sol-dtime */
    double gas_R;           /* specific gas constant R = Runiv/W of the single species */
    double gas_gamma;       /* ratio of specific heats of the calorically perfect closure */
    double irs_beta;        /* irs-beta: implicit residual smoothing when > 0 (Lib_IRS.f90:17-177,
                               Assign_Setup.f90:61); 0 by default */
    int    shock_detector;  /* 1: space-reconstruction = MUSCL-SD, the limited slopes of a face
                               scaled by the Tramel pressure sensor of its left / lower cell
                               (Mod_Space.f90:25-27, Mod_Fluxes.f90:132-204,
                               Lib_Shock_Detector.f90:14-38); 0 by default */
    double riemann_minf;    /* riemann-options-Minf: the reference Mach number of AUSM+-up /
                               AUSM+-up2, required > 0 by them (Register_Numerics.f90:76,
                               Assign_Setup.f90:108-112); 0 by default */
} q2d_options;

/* One boundary-cell record: the 5-integer header line of bc.txt plus its property line
 * (IO_BC.f90:209-402). Fields not used by a type are ignored. alpha >= 0.5*DBL_MAX means the
 * 'normal' keyword (parse_dir_tok sentinel, Lib_BC_Fluxes_Inflow.f90:552-560). */
typedef struct q2d_bc_rec {
    int    b, i, j, f, type;
    int    bs, is, js, fs, d11, d12, d21, d22;   /* 101: donor block/cell/face + orientation */
    double T0;        /* 401: total T; 405: static T */
    double p0;        /* 401: total p */
    double pamb;      /* 405: static p; 406: back pressure (<=0: extrapolation) */
    double mach;      /* 405: Mach */
    double alpha;     /* 401/405: flow angle [rad] or the 'normal' sentinel */
    double rel_fac;   /* 401/405/406: relaxation factor */
} q2d_bc_rec;

/* Per-case result of the last executed step (the reference's domain%dtglobal, %time,
 * %iter, obj_sim_param%residuotot and TODO) plus the first error seen. */
typedef struct q2d_step_info {
    double    dtglobal;
    double    time;
    long long iter;
    double    residual[4];   /* sqrt(sum over cells of |d rho|^2, |du|^2, |dv|^2, |dp|^2) */
    double    residual0;     /* residual[0] of the first step of the case */
    int       todo;          /* Q2D_TODO_* */
    int       err;           /* Q2D_OK, Q2D_ERR_NONPHYSICAL / Q2D_ERR_NAN, or Q2D_ERR_BADARG when a
                                stage kernel was launched with a layout it was not built for */
    int       err_b, err_i, err_j, err_stage;   /* where err was first raised (1-based) */
} q2d_step_info;

/* Fills *opt with the reference defaults (HLLC, first order, euler, cfl 0.5, res-threshold
 * 1e-10, time-threshold 1e30, iter-threshold 1e9, res-diter 1, R=287, gamma=1.4). */
void q2d_options_default(q2d_options* opt);

/* Creates a context on the current CUDA device. Replaces Assign_Setup (Assign_Setup.f90:11-117). */
int  q2d_gpu_create(q2d_ctx** out, const q2d_options* opt);

/* Adds an empty case (one Q2D domain: its blocks share dtglobal, time, iter, residual). */
int  q2d_gpu_add_case(q2d_ctx* ctx, int* case_id);

/* Adds a block to a case. Replaces Allocate_Block (Mod_Allocate_Data.f90:86-180) and the
 * node/Cross_Section reads (IO_Solution.f90:38-129, Lib_Source_Areavariation.f90:53-101). */
int  q2d_gpu_add_block(q2d_ctx* ctx, int case_id, int ni, int nj, const double* nodes_xy,
                       const double* cross_section, int* block_id);

/* Sets the boundary records of a case, sorted by block then face like bc.txt
 * (Read_BCfile, IO_BC.f90:163-440; ordering consumed by Mod_BC_Fluxes.f90:79-84). */
int  q2d_gpu_set_bcs(q2d_ctx* ctx, int case_id, const q2d_bc_rec* recs, int n);

/* Copies the interior of a block's primitive state host->device (Read_IC result). */
int  q2d_gpu_upload_prim(q2d_ctx* ctx, int block_id, const double* P);
/* Restart (newrun = false; Wrap_Setup.f90:132-149, Read_IC IO_Solution.f90:38-126): the physical
 * time a time-accurate case resumes from (SOLUTIONTIME of the restart field); the step and
 * iteration counters restart at 0 as in the reference. Before q2d_gpu_commit. */
int  q2d_gpu_set_case_time(q2d_ctx* ctx, int case_id, double time);

/* Thermally perfect single-species gas (replaces the constant-cp table of
 * FLINT_Lib_Thermodynamic for the path's routines: f_tabT_expr lerps at int(T) in roe_averages,
 * Lib_Riemann_HLL.f90:229-317, and in Compute_Prim_Residual, Lib_Newstate.f90:245-294; f_ss /
 * f_gamma / E0 / H0 / prim2cons / cons2prim of Lib_Newstate.f90:131-159 and the BC and source
 * routines): h(T) [J/kg] and cp(T) [J/(kg K)] at T = 0, 1, .., ntab-1 K, interpolated linearly
 * at int(T); gas constant options.gas_R, gamma(T) = cp/(cp - R). The state from the conserved
 * variables solves e(T) = h(T) - R T on the table, starting from the temperature before the
 * update. Plain FP64 form, HLLC / HLLE / LLF, no shock sensor, batch contexts only; before
 * q2d_gpu_commit. Q2D_ERR_BADARG otherwise, or when cp <= R or e(T) does not increase. */
int  q2d_gpu_set_thermo_table(q2d_ctx* ctx, int ntab, const double* h_tab, const double* cp_tab);

/* A case's own fixed end (no counterpart in the reference, whose domain has one iteration limit):
 * the case reports TODO = END once its iteration count reaches iter_end (0: none), besides the
 * context's limits. Usable before or after commit and on admitted serving cases; a served
 * request's end is set this way right after q2d_serve_admit. */
int  q2d_gpu_set_case_end(q2d_ctx* ctx, int case_id, long long iter_end);

/* Builds metrics (Setup_Metrics, Mod_Metrics.f90:11-148) and the device work lists.
 * Called implicitly by the first q2d_gpu_step(). */
int  q2d_gpu_commit(q2d_ctx* ctx);

/* Advances every running case by up to nsteps explicit steps (Explicit_Step). A case stops
 * early when its TODO becomes END, when it raises IO (sol-diter / sol-dtime), or on error.
 * out, when not NULL, receives q2d_gpu_num_cases() entries. Returns the first case error. */
int  q2d_gpu_step(q2d_ctx* ctx, int nsteps, q2d_step_info* out);

/* Asynchronous form of q2d_gpu_step: enqueues the steps on the context's stream and returns;
 * q2d_gpu_wait() synchronises and fills out (q2d_gpu_num_cases() entries, or NULL). */
int  q2d_gpu_step_async(q2d_ctx* ctx, int nsteps);
int  q2d_gpu_wait(q2d_ctx* ctx, q2d_step_info* out);

/* Builds (captures and instantiates) the CUDA graph of an nsteps call ahead of time, so that a
 * later q2d_gpu_step(ctx, nsteps, ...) only launches it. */
int  q2d_gpu_prepare(q2d_ctx* ctx, int nsteps);

/* Autotuner (no reference counterpart): times each candidate schedule of the stage kernels
 * (stage kernel and tile shape) for `steps` steps on this context's workload, keeps the fastest
 * and restores the state. *schedule gets the chosen candidate index, *ms_per_step its time
 * (either may be NULL). */
int  q2d_gpu_autotune(q2d_ctx* ctx, int steps, int* schedule, float* ms_per_step);

/* Pins the schedule of the stage kernels (the index the autotuner reports) without tuning:
 * 0-2 FP64 tile kernel on 32x10, 32x8, 64x4 tiles; 3-7 FP32-flux tile kernel on 32x10, 32x8,
 * 64x4 (256 threads) and 32x16, 64x8 (512 threads) tiles (FP32-flux form only); 8 FP32-flux tile
 * kernel in difference form on 32x8 tiles (FP32-flux form with HLLC, HLLE or LLF, without
 * MUSCL-SD or residual smoothing; the default of those options). q2d_gpu_get_schedule returns
 * the current one. */
int  q2d_gpu_set_schedule(q2d_ctx* ctx, int schedule);
int  q2d_gpu_get_schedule(const q2d_ctx* ctx);

/* Allocation-free residual norm. No counterpart in the reference: it serves callers that
 * cannot call cudaMalloc when they need the residual — a host whose device memory is owned
 * by its own pool allocator (for instance a Fortran driver that pre-allocates every array),
 * or a latency-critical path that cannot take the implicit synchronisation of an allocation.
 * It computes sqrt(sum over cells of |new - old|^2) for rho, u, v and p (Compute_Residual,
 * Mod_Diagnostic.f90:438-469, and the sqrt of Mod_Explicit.f90:132) from two caller-owned
 * device states stored as 4 planes (rho, u, v, p) of plane_stride doubles, cells
 * 0..ncells-1 of each plane, and writes the 4 norms to device memory at norms_out. The work
 * is enqueued on `stream` (a cudaStream_t; NULL is the legacy default stream) and the call
 * returns without synchronising. It allocates nothing: its scratch is a fixed device array of
 * Q2D_NOALLOC_MAX_PARTIALS x 4 doubles (256 KiB) that every GPU loading the library holds
 * until the process exits; ncells above Q2D_NOALLOC_MAX_PARTIALS *
 * Q2D_NOALLOC_CELLS_PER_PARTIAL (16,777,216) returns Q2D_ERR_CAPACITY. The first call on a
 * device looks up that array's device address on the current device, so make it before any
 * stream capture; host threads may make their first calls at the same time. The looked-up
 * address is kept for the life of the process: do not call this entry point on a device after
 * cudaDeviceReset. A CUDA error already pending when the call starts is returned as
 * Q2D_ERR_CUDA without launching anything and is left pending for the caller. All calls on one
 * device share the array and each call overwrites the part it uses: calls that overlap on the
 * GPU (concurrent streams) race. */
#define Q2D_NOALLOC_MAX_PARTIALS      8192
#define Q2D_NOALLOC_CELLS_PER_PARTIAL 2048
int  q2d_gpu_residual_norm_noalloc(const double* p_new, const double* p_old, long long ncells,
                                   long long plane_stride, double* norms_out, void* stream);

/* The CUDA stream (cudaStream_t) the context enqueues on, for event timing by callers. */
void* q2d_gpu_stream(const q2d_ctx* ctx);

/* Reads the current step info of one case. */
int  q2d_gpu_case_info(q2d_ctx* ctx, int case_id, q2d_step_info* out);

/* Copies the interior of a block's primitive state device->host. */
int  q2d_gpu_download_prim(q2d_ctx* ctx, int block_id, double* P);

/* Many-block forms of q2d_gpu_upload_prim / q2d_gpu_download_prim: block_ids[k] with the
 * ghosted array P[k], k < n. The host<->device copies of all blocks are queued back to back
 * through a 128 MiB device staging ring and the call synchronises once: what a host that reads
 * or writes every block of a batch (the loops over blocks of Read_IC, IO_Solution.f90:38-129,
 * and of the solution writers set up at IO_Solution.f90:132-231) should call. Upload copies
 * each whole array in one piece (its ghost values are read but not used); download writes the
 * interior only. Blocks of cases not on the device yet take the single-block path; download
 * requires every block to be on the device. Page-locked host arrays copy fastest. */
int  q2d_gpu_upload_prim_many(q2d_ctx* ctx, int n, const int* block_ids, const double* const* P);
int  q2d_gpu_download_prim_many(q2d_ctx* ctx, int n, const int* block_ids, double* const* P);

/* Number of cases (case slots of a serving context) and total interior cells of the cases
 * the context holds. */
int       q2d_gpu_num_cases(const q2d_ctx* ctx);
long long q2d_gpu_num_cells(const q2d_ctx* ctx);

/* ---- serving: continuous batching of independent cases (no reference counterpart) --------
 * The reference runs one domain per process from input files (main.f90:20-50). A serving
 * context holds up to max_cases independent cases in device pools sized from device_bytes
 * (state, metrics and face geometry: about 240 bytes per interior cell, 306 in the FP32-flux
 * form, which keeps FP32 copies of the geometry; the work lists and
 * per-case records are extra), all advanced together by q2d_gpu_step / step_async / wait, each
 * with its own time step, iteration count, residual, TODO state and error status.
 *
 * q2d_serve_admit adds a case between steps: nblocks blocks with the arguments of
 * q2d_gpu_add_block and q2d_gpu_upload_prim (P[b] in the ghosted Fortran layout) and the
 * boundary records of q2d_gpu_set_bcs (the arrays are read during the call only: the caller may
 * reuse them when it returns). It validates the input, computes the metrics and
 * reserves device memory on the host at once, and queues the copies of its device images on a
 * copy stream of the context right away (they overlap the steps in flight, into memory that no
 * listed case uses); its run state is started by the next step call. It returns
 * Q2D_ERR_CAPACITY when no slot is free or the pools cannot hold the case (nothing is kept).
 * The case starts at iteration 0 with a fresh residual reference; the other cases' results do
 * not depend on when it arrives.
 * q2d_serve_retire frees a case's slot and memory (its results are no longer readable); called
 * while steps are in flight it waits for them first.
 * q2d_serve_block_id maps (case, 1-based block) to the block id of download_prim / upload_prim.
 * q2d_serve_free_cells estimates how many more interior cells the pools can take. */
int  q2d_serve_create(q2d_ctx** out, const q2d_options* opt, unsigned long long device_bytes, int max_cases);
int  q2d_serve_admit(q2d_ctx* ctx, int nblocks, const int* ni, const int* nj, const double* const* nodes_xy,
                     const double* const* cross_sections, const double* const* P, const q2d_bc_rec* recs,
                     int nrecs, int* case_id);
int  q2d_serve_retire(q2d_ctx* ctx, int case_id);
int  q2d_serve_block_id(const q2d_ctx* ctx, int case_id, int b, int* block_id);
long long q2d_serve_free_cells(const q2d_ctx* ctx);

/* Number of kernel launches issued by this context since creation (instrumentation). */
long long q2d_gpu_launch_count(const q2d_ctx* ctx);

/* Text of a status code, and the last detailed error message of a context. */
const char* q2d_gpu_errstr(int status);
const char* q2d_gpu_last_error(const q2d_ctx* ctx);

void q2d_gpu_destroy(q2d_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif /* Q2D_GPU_H */
