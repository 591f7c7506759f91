/*
 * cmf_gpu.h -- C ABI of the B200 CaMa-Flood physics time step.
 *
 * Drop-in boundary: the call `CALL CMF_PHYSICS_ADVANCE` at src/cmf_drv_advance_mod.F90:101
 * is replaced by cmf_gpu_physics_advance() when the GPU switch is on.  Every pointer argument
 * is a plain host pointer to the reference's own module arrays, passed with ISO_C_BINDING c_loc:
 *   - (NSEQMAX,1) arrays are contiguous double[NSEQMAX] in sequence order;
 *   - (NSEQMAX,1,NLFP) arrays are double[NLFP][NSEQMAX] (layer-major);
 *   - (NPTHOUT,NPTHLEV) arrays are double[NPTHLEV][NPTHOUT];
 *   - 2-D index tables I1UPST(NSEQMAX,UPNMAX), I1P_OUT(NSEQMAX,ONMAX), I1P_INF(NSEQMAX,INMAX)
 *     are column-major int32 and hold 1-based indices, exactly as Fortran allocates them.
 * Sequence and path indices stay 1-based at the boundary (I1NEXT keeps the negative river-mouth
 * codes).  The library converts them once, in cmf_gpu_init, to its device layout.
 *
 * Ensembles: with nmembers > 1 every state, runoff and diagnostic array is member-major,
 * [nmembers][NSEQMAX] (or [nmembers][NPTHLEV][NPTHOUT]); maps are shared by all members and
 * each member runs its own adaptive time step.
 *
 * Status convention (no exceptions cross the ABI): 0 = ok; negative = configuration or
 * unsupported option (the Fortran shim writes cmf_gpu_strerror() to LOGNAM and STOPs 9, as
 * src/cmf_ctrl_nmlist_mod.F90:302 does); positive = device-side failure.
 * Threading: call from the serial part of the host program; one CUDA stream per context;
 * calls are synchronous from the caller's view except the *_async variants.
 */
#ifndef CMF_GPU_H
#define CMF_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CMF_GPU_ABI_VERSION 2

/* ---- status codes ------------------------------------------------------------------------ */
#define CMF_OK                0
#define CMF_E_ARG            -1  /* null pointer, bad size or inconsistent dimensions            */
#define CMF_E_UNSUPPORTED    -2  /* option combination the GPU path does not implement           */
#define CMF_E_STATE          -3  /* call out of order (no context, not initialised)              */
#define CMF_E_IO             -4  /* host model core: a map, table or namelist could not be read  */
#define CMF_E_CUDA            1  /* CUDA runtime error (message via cmf_gpu_last_error)          */
#define CMF_E_NT_CAP          2  /* adaptive sub-step count above the cap (non-finite DT_MIN)     */
#define CMF_E_NO_DEVICE       3  /* no CUDA device or the sm_100a kernels cannot run on it       */
#define CMF_E_NONFINITE       4  /* a sub-step produced a NaN/infinite storage (NaN runoff...)   */
#define CMF_E_BARRIER         5  /* a bounded device-side wait (persistent grid barrier) ran out */

/* ---- dimensions (src/yos_cmf_map.F90, src/yos_cmf_input.F90) ----------------------------- */
typedef struct cmf_dims {
    int32_t nseqall;    /* NSEQALL: river cells followed by river mouths                        */
    int32_t nseqriv;    /* NSEQRIV                                                               */
    int32_t nseqmax;    /* NSEQMAX (== NSEQALL for the single-region build)                      */
    int32_t nlfp;       /* NLFP floodplain layers                                                 */
    int32_t upnmax;     /* second extent of I1UPST                                                */
    int32_t npthout;    /* NPTHOUT (1 when LPTHOUT is off, as the reference allocates)           */
    int32_t npthlev;    /* NPTHLEV                                                                */
    int32_t onmax;      /* second extent of I1P_OUT                                               */
    int32_t inmax;      /* second extent of I1P_INF                                               */
    int32_t ndam;       /* NDAM (0 when LDAMOUT is off)                                          */
    int32_t nmembers;   /* ensemble members sharing the network (1 = the reference's single run) */
} cmf_dims;

/* ---- physical parameters (NPARAM, src/cmf_ctrl_nmlist_mod.F90:227-241) ------------------- */
typedef struct cmf_params {
    double pgrv;        /* PGRV                                                                   */
    double pmanfld;     /* PMANFLD                                                                */
    double pdstmth;     /* PDSTMTH                                                                */
    double pcadp;       /* PCADP                                                                  */
    double pminslp;     /* PMINSLP                                                                */
    double dfrcinc;     /* DFRCINC = NLFP**(-1)                                                   */
} cmf_params;

/* ---- options (NRUNVER logicals; 0/1) ----------------------------------------------------- */
typedef struct cmf_opts {
    int32_t ladpstp, lfldout, lpthout, ldamout, llevee, lspamat;
    /* options the GPU path refuses (cmf_gpu_init returns CMF_E_UNSUPPORTED when any is set) */
    int32_t lkine, lslpmix, lstg_es, lgdwdly, lrosplit, lwevap, lupsinf, lheatlink, ltrace, lslopemouth;
    int32_t ldamh22;     /* Hanazaki-2022 dam rule instead of the default Yamazaki-Funato rule   */
    int32_t ldamyby;     /* refused: year-by-year dam activation                                  */
    int32_t ldiag;       /* accumulate the CMF_DIAG_*_ADPSTP averages/maxima on the device       */
    int32_t launch_mode; /* 0: one CUDA graph per coupling step with a device-side sub-step loop;
                            1: host-driven launches (reads NT back before the sub-steps);
                            2: one persistent cooperative kernel per coupling step (grid barriers
                               between the phases, cell tiles interleaved over the CTAs)          */
    int32_t device;      /* CUDA device ordinal                                                   */
    int32_t block_size;  /* 0: the online autotuner picks the schedule (launch_mode 0); else
                            threads per block of the phase kernels (64..256)                     */
    int32_t ldiag_output;/* accumulate the output-interval averages/maxima (D2*_oAVG, D2*_oMAX) on
                            the device: CMF_DIAG_AVEMAX_OUTPUT after every outer step, as
                            CMF_DRV_ADVANCE calls it (src/cmf_drv_advance_mod.F90:114); needs ldiag */
} cmf_opts;

/* ---- static maps: Fortran module arrays (read-only, host memory) ------------------------- */
typedef struct cmf_map_ptrs {
    const int32_t *i1next;      /* I1NEXT(NSEQMAX)            1-based, mouth codes negative       */
    const int32_t *i1upst;      /* I1UPST(NSEQMAX,UPNMAX)     1-based, column-major               */
    const int32_t *i1upn;       /* I1UPN(NSEQMAX)                                                  */
    const int32_t *i2mask;      /* I2MASK(NSEQMAX,1)          0 normal, 1 dam-upstream, 2 dam      */
    const double *rivelv, *elevtn, *nxtdst, *rivwth, *rivhgt, *rivlen, *rivman, *grarea;
    const double *rivstomax;    /* D2RIVSTOMAX                                                     */
    const double *dwnelv;       /* D2DWNELV (downstream boundary elevation at the mouths)          */
    const double *fldstomax;    /* D2FLDSTOMAX(NSEQMAX,1,NLFP)                                     */
    const double *fldgrd;       /* D2FLDGRD(NSEQMAX,1,NLFP)                                        */
    const double *fldhgt;       /* D2FLDHGT(NSEQMAX,1,NLFP)   (levee scheme only)                 */
    /* bifurcation (LPTHOUT) */
    const int32_t *pth_upst, *pth_down;       /* PTH_UPST/PTH_DOWN(NPTHOUT) 1-based, <=0 outside  */
    const double *pth_dst;                    /* PTH_DST(NPTHOUT)                                */
    const double *pth_elv, *pth_wth;          /* PTH_ELV/PTH_WTH(NPTHOUT,NPTHLEV)                */
    const double *pth_man;                    /* PTH_MAN(NPTHLEV)                                */
    const int32_t *i1p_out, *i1p_outn, *i1p_inf, *i1p_infn;
    /* levee (LLEVEE), src/cmf_ctrl_levee_mod.F90:31-44 */
    const double *levhgt, *levfrc, *bashgt, *levdst, *levbassto, *levtopsto, *levfilsto;
    /* dams (LDAMOUT), src/cmf_ctrl_damout_mod.F90:45-74 */
    const int32_t *damseq;                    /* DamSeq(NDAM) 1-based or IMIS                    */
    const int32_t *damstat;                   /* DamStat(NDAM)                                   */
    const int32_t *i1dam;                     /* I1DAM(NSEQMAX)                                  */
    const double *dam_qn, *dam_qf, *dam_qa, *dam_convol, *dam_fldvol, *dam_emevol;
    const double *dam_norvol, *dam_adjvol, *dam_r_volupa;
} cmf_map_ptrs;

/* ---- prognostic state (src/yos_cmf_prog.F90); member-major when nmembers > 1 -------------- */
typedef struct cmf_state_ptrs {
    double *rivsto, *fldsto;                  /* P2RIVSTO, P2FLDSTO (FP64 storage)               */
    double *rivout, *fldout;                  /* D2RIVOUT, D2FLDOUT                              */
    double *rivout_pre, *fldout_pre;          /* D2RIVOUT_PRE, D2FLDOUT_PRE                      */
    double *rivdph_pre, *fldsto_pre;          /* D2RIVDPH_PRE, D2FLDSTO_PRE                      */
    double *pthflw, *pthflw_pre;              /* D1PTHFLW, D1PTHFLW_PRE (NPTHOUT,NPTHLEV)        */
    double *damsto, *daminf;                  /* P2DAMSTO, P2DAMINF                              */
    double *levsto;                           /* P2LEVSTO                                        */
} cmf_state_ptrs;

/* ---- diagnostics (src/yos_cmf_diag.F90); NULL entries are skipped ------------------------ */
typedef struct cmf_diag_ptrs {
    double *rivdph, *flddph, *fldfrc, *fldare, *sfcelv, *storge, *rivvel;
    double *rivinf, *fldinf, *pthout, *outflw, *pthflwsum, *levdph;
    /* adaptive-step averages and maxima after CMF_DIAG_GETAVE_ADPSTP (needs opts.ldiag) */
    double *rivout_aavg, *fldout_aavg, *outflw_aavg, *rivvel_aavg, *pthout_aavg;
    double *gdwrtn_aavg, *runoff_aavg, *rofsub_aavg, *daminf_aavg;
    double *storge_amax, *outflw_amax, *rivdph_amax;
    double *pthflw_aavg, *pthflwsum_aavg;
} cmf_diag_ptrs;

/* ---- output-interval averages and maxima (src/yos_cmf_diag.F90:82-103); NULL entries skipped */
typedef struct cmf_diag_out_ptrs {
    double *rivout_oavg, *fldout_oavg, *outflw_oavg, *rivvel_oavg, *pthout_oavg;
    double *gdwrtn_oavg, *runoff_oavg, *rofsub_oavg, *daminf_oavg;
    double *storge_omax, *outflw_omax, *rivdph_omax;
    double *pthflw_oavg;                      /* D1PTHFLW_oAVG (NPTHOUT,NPTHLEV)                 */
    double *nadd_out;                         /* NADD_out, one value per member                 */
} cmf_diag_out_ptrs;

/* ---- water budget of the last sub-step (CALC_WATBAL, src/cmf_ctrl_physics_mod.F90:216-248) */
typedef struct cmf_budget {
    double stopre, stonxt, stonew, rivinf, rivout;       /* P0GLB* written by CMF_CALC_STONXT      */
    double stopre2, stonew2, rivsto, fldsto, fldare;     /* P0GLB* written by the stage scheme     */
    double levsto;                                       /* P0GLBLEVSTO (levee scheme)             */
    double dam_miss;                                     /* DamMiss of CMF_DAMOUT_WATBAL           */
} cmf_budget;

typedef struct cmf_gpu_ctx cmf_gpu_ctx;

/* ======================================================================================== */
/* Context API (any number of contexts: regional domains, ensembles)                        */
/* ======================================================================================== */

/* Replaces the device-relevant part of CMF_DRV_INIT (src/cmf_drv_control_mod.F90:149-298):
 * uploads the static maps, builds the upstream/path CSR tables and validates the options. */
int cmf_gpu_create(const cmf_dims *dims, const cmf_params *params, const cmf_map_ptrs *maps,
                   const cmf_opts *opts, cmf_gpu_ctx **out);
int cmf_gpu_destroy(cmf_gpu_ctx *ctx);

/* Host -> device copy of the prognostic state (after CMF_PROG_INIT / CMF_RESTART_INIT /
 * CMF_DAMOUT_INIT, src/cmf_drv_control_mod.F90:237-252).  NULL members are left unchanged. */
int cmf_gpu_ctx_set_state(cmf_gpu_ctx *ctx, const cmf_state_ptrs *st);
/* Device -> host copy of the prognostic state (before output/restart,
 * src/cmf_drv_advance_mod.F90:121-152).  NULL members are skipped. */
int cmf_gpu_ctx_get_state(cmf_gpu_ctx *ctx, const cmf_state_ptrs *st);
/* Runoff after CMF_FORCING_PUT (src/MAIN_cmf.F90:105): D2RUNOFF [m3/s]; rofsub may be NULL. */
int cmf_gpu_ctx_put_runoff(cmf_gpu_ctx *ctx, const double *runoff, const double *rofsub);
/* One outer step, CMF_PHYSICS_ADVANCE (src/cmf_ctrl_physics_mod.F90:21-153).  dt_def is DT.
 * nt_out[nmembers], dt_out[nmembers] and budget_out[nmembers] may be NULL. */
int cmf_gpu_ctx_physics_advance(cmf_gpu_ctx *ctx, double dt_def, int32_t *nt_out, double *dt_out,
                                cmf_budget *budget_out);
int cmf_gpu_ctx_get_diag(cmf_gpu_ctx *ctx, const cmf_diag_ptrs *dg);

/* Pipelined host I/O for C, C++ and Python hosts (the Fortran shim keeps the calls above): the
 * next step's runoff is uploaded while the current step runs, and a finished step's diagnostics
 * are read back while the next one runs.  Host buffers should be pinned for the copies to overlap.
 *   put_runoff_async  copies D2RUNOFF of the next outer step into a device staging buffer on a
 *                     copy stream; the next advance (async or not) makes it D2RUNOFF;
 *   advance_async     launches one outer step and returns; at most two steps in flight, so the
 *                     next step is queued while the host handles the previous one;
 *   wait              finishes the oldest launched step (NT, DT, budgets, statuses as
 *                     physics_advance; after a failed step the device is drained before its error
 *                     word is cleared); physics_advance refuses while steps are in flight;
 *   get_diag_async    stages the named diagnostics as they stand after the steps enqueued so far
 *                     (device copies ordered before any later step), then copies them to the host
 *                     buffers on the copy stream (GDWRTN/ROFSUB not accepted);
 *   io_wait           blocks until every staged read-back has landed in the host buffers. */
int cmf_gpu_ctx_put_runoff_async(cmf_gpu_ctx *ctx, const double *runoff);
int cmf_gpu_ctx_advance_async(cmf_gpu_ctx *ctx, double dt_def);
int cmf_gpu_ctx_wait(cmf_gpu_ctx *ctx, int32_t *nt_out, double *dt_out, cmf_budget *budget_out);
int cmf_gpu_ctx_get_diag_async(cmf_gpu_ctx *ctx, const cmf_diag_ptrs *dg);
int cmf_gpu_ctx_io_wait(cmf_gpu_ctx *ctx);

/* Device-resident pipeline (no host round trip): runoff already in device memory, ksteps outer
 * steps enqueued on the context's stream; runoff_dev holds ksteps consecutive [nmembers][NSEQMAX]
 * fields (or one field reused when runoff_stride is 0).  With runoff_dev NULL the steps use the
 * context's D2RUNOFF, after applying a field staged by put_runoff_async; with runoff_dev given, a
 * staged field is discarded. */
int cmf_gpu_ctx_advance_device(cmf_gpu_ctx *ctx, double dt_def, int32_t ksteps,
                               const double *runoff_dev, int64_t runoff_stride);
int cmf_gpu_ctx_synchronize(cmf_gpu_ctx *ctx);
/* Per-member sub-step counts of the last outer step, read back from the device. */
int cmf_gpu_ctx_last_nt(cmf_gpu_ctx *ctx, int32_t *nt_out, double *dt_out);
/* CUDA stream (cudaStream_t) the context launches on, for event timing by the caller. */
void *cmf_gpu_ctx_stream(cmf_gpu_ctx *ctx);
/* Number of kernels this context launched so far (graph launches count their kernel nodes). */
int64_t cmf_gpu_ctx_kernel_launches(cmf_gpu_ctx *ctx);
/* Threads per block of the flux kernel in the current schedule. */
int32_t cmf_gpu_ctx_block_size(cmf_gpu_ctx *ctx);

/* Launch schedule of the outer step.  Every schedule computes the same bits (states, NT/DT and the
 * budgets, which are summed from per-warp partials), so it is a pure performance choice.  A
 * launch_mode 0 context with block_size 0 is tuned online: after 4 outer steps on a starting
 * schedule, each candidate (flux/rate block 128 or 256 x store block 128 or 256 x occupancy
 * profile, and the persistent kernel) runs 2 real outer steps timed with CUDA events (best time
 * per sub-step kept); the fastest is installed and cached per network shape for later contexts in
 * the process.  cmf_gpu_ctx_set_schedule fixes a schedule (and stops tuning). */
typedef struct cmf_schedule {
    int32_t mode;                 /* 0 graph of phase kernels, 2 persistent cooperative kernel     */
    int32_t flux_block, rate_block, store_block;   /* threads per block of the phase kernels     */
    int32_t profile;              /* 0 more resident warps (fewer registers), 1 fewer spills       */
    int32_t tuned;                /* 1 chosen by the autotuner, 0 fixed or cached, -1 still tuning  */
    int32_t candidates;           /* candidates the autotuner timed                                */
    double best_us_per_substep, worst_us_per_substep;
} cmf_schedule;
int cmf_gpu_ctx_get_schedule(cmf_gpu_ctx *ctx, cmf_schedule *out);
int cmf_gpu_ctx_set_schedule(cmf_gpu_ctx *ctx, const cmf_schedule *sched);
/* Forgets the cached schedules, so that the next contexts tune again. */
void cmf_gpu_schedule_cache_clear(void);
/* Device-side counters since creation: sum over outer steps and members of NT, sum over outer
 * steps of max NT (sub-step loop iterations) and the number of outer steps. */
int cmf_gpu_ctx_counters(cmf_gpu_ctx *ctx, int64_t *member_substeps, int64_t *loop_iters, int64_t *outer_steps);
/* Output-interval diagnostics on the device (needs opts.ldiag_output; src/cmf_calc_diag_mod.F90:
 * 222-356).  CMF_DIAG_AVEMAX_OUTPUT runs inside every outer step (fused into its last sub-step),
 * as CMF_DRV_ADVANCE calls it after every CMF_PHYSICS_ADVANCE (src/cmf_drv_advance_mod.F90:114).
 * op CMF_DIAG_OUT_GETAVE divides the sums by NADD_out in place (CMF_DIAG_GETAVE_OUTPUT, :123),
 * op CMF_DIAG_OUT_RESET zeroes them and NADD_out (CMF_DIAG_RESET_OUTPUT, :143).  Enqueued on the
 * context's stream.  cmf_gpu_ctx_get_diag_output copies the oAVG/oMAX arrays to the host
 * (synchronous; [nmembers][NSEQMAX], pthflw_oavg [nmembers][NPTHLEV][NPTHOUT]). */
#define CMF_DIAG_OUT_RESET  0
#define CMF_DIAG_OUT_GETAVE 2
int cmf_gpu_ctx_diag_output(cmf_gpu_ctx *ctx, int32_t op);
int cmf_gpu_ctx_get_diag_output(cmf_gpu_ctx *ctx, const cmf_diag_out_ptrs *dg);
/* Check of the persistent kernel's bounded waits (launch_mode 2 contexts, or any context whose
 * device can run it): launches the kernel with a grid barrier that one arrival short of its count
 * can never complete and a bound of wait_ns; every CTA gives up after about that time and the
 * kernel returns.  Returns CMF_E_BARRIER when the bound worked (the context stays usable: its
 * error word is cleared), another status otherwise.  No state changes. */
int cmf_gpu_ctx_persist_selftest(cmf_gpu_ctx *ctx, int64_t wait_ns);
/* The schedule the context runs: 0 graph, 1 host-driven, 2 persistent. */
int32_t cmf_gpu_ctx_launch_mode(cmf_gpu_ctx *ctx);
/* Adaptive-step statistics since creation: near_boundary = (outer step, member) pairs whose
 * DT_DEF/DT_MIN - 0.01 (the argument of INT in CALC_ADPSTP, src/cmf_ctrl_physics_mod.F90:205)
 * lay within 1e-12 (relative) of an integer, where NT depends on the last bits of DT_MIN;
 * hist[k] = pairs with NT == k for k < nbins-1, hist[nbins-1] = pairs with NT >= nbins-1.
 * Either pointer may be NULL. */
int cmf_gpu_ctx_nt_stats(cmf_gpu_ctx *ctx, int64_t *near_boundary, int64_t *hist, int32_t nbins);
/* Measurement helper: runs `reps` outer steps kernel by kernel with CUDA events between kernels
 * on the context's stream (advances the state), timing every sub-step.  ms_out[6] receives the mean
 * duration per launch of the stage/CFL and NT/DT kernels (once per outer step), of the flux, rate
 * and storage kernels (once per sub-step) and of the budget kernel (once per outer step). */
int cmf_gpu_ctx_time_phases(cmf_gpu_ctx *ctx, double dt_def, int32_t reps, double *ms_out);

/* Storage-only restart (LSTOONLY): the stage scheme, then CMF_CALC_OUTPRE
 * (src/cmf_opt_outflw_mod.F90:308-421) reconstructs D2RIVOUT_PRE, D2FLDOUT_PRE, D1PTHFLW_PRE and
 * D2RIVDPH_PRE of every member from the storage by the diffusive (Manning) wave, as CMF_DRV_INIT
 * does after a storage-only restart (src/cmf_drv_control_mod.F90:273-277).  Synchronous. */
int cmf_gpu_ctx_calc_outpre(cmf_gpu_ctx *ctx);
/* Downstream boundary of the mouths, CMF_BOUNDARY_UPDATE (src/cmf_ctrl_boundary_mod.F90:267-304):
 * D2DWNELV = D2ELEVTN (+ meansl when non-NULL) (+ sealev when non-NULL); host arrays [NSEQALL]
 * (sealev from CMF_BOUNDARY_GET_BIN's map via cmf_host_map_to_vec).  Synchronous. */
int cmf_gpu_ctx_update_boundary(cmf_gpu_ctx *ctx, const double *sealev, const double *meansl);

/* Runoff interpolation on the device, CMF_FORCING_PUT (src/cmf_ctrl_forcing_mod.F90:716-831).
 * cmf_gpu_ctx_set_runoff_map uploads the mapping once: linterp != 0 -> ROFF_INTERP with the input
 * matrix INPX/INPY/INPA(NSEQMAX,INPN) (column-major, i.e. [INPN][NSEQALL]; read from CINPMAT by
 * cmf_host_read_inpmat), runoff grid NXIN x NYIN; linterp == 0 -> CONV_RESOL with inpn == 1 and
 * inpx/inpy = I1SEQX/I1SEQY (grid == map, area D2GRAREA).  cmf_gpu_ctx_put_runoff_grid then turns
 * one runoff field per member, PBUFF(NXIN,NYIN) [mm/dt] laid out [nmembers][NYIN][NXIN] as fp64
 * (is_float == 0) or fp32 (promoted exactly), into D2RUNOFF [m3/s] of every member.  on_device:
 * grid is a device pointer (enqueued on the context's stream, asynchronous); else host memory
 * (copied, synchronous).  clean != 0 first applies CMF_FORCING_GET's NaN -> RMIS and max(., 0)
 * (:486-494). */
int cmf_gpu_ctx_set_runoff_map(cmf_gpu_ctx *ctx, int32_t linterp, int32_t nxin, int32_t nyin, int32_t inpn,
                               const int32_t *inpx, const int32_t *inpy, const double *inpa, double drofunit);
int cmf_gpu_ctx_put_runoff_grid(cmf_gpu_ctx *ctx, const void *grid, int32_t is_float, int32_t on_device,
                                int32_t clean);

/* Batch of contexts on one device -- regional domains of uneven size, each with its own members --
 * advanced by ONE graph launch per coupling step.  Each context's outer step (prologue + WHILE
 * sub-step loop) is an independent branch of the batch graph, so every domain and member keeps its
 * own adaptive DT (NT/DT per member as in CMF_PHYSICS_ADVANCE) and the branches run concurrently.
 * Results equal those of advancing each context alone.  Contexts must use launch_mode 0 and stay
 * alive while the batch exists.  cmf_gpu_batch_launch is asynchronous (ordered after each
 * context's earlier work, and each context's later work waits for it); cmf_gpu_batch_advance also
 * reads back NT/DT/budgets, concatenated over the contexts in batch order (sum of nmembers). */
typedef struct cmf_gpu_batch cmf_gpu_batch;
int cmf_gpu_batch_create(cmf_gpu_ctx *const *ctxs, int32_t nctx, cmf_gpu_batch **out);
int cmf_gpu_batch_launch(cmf_gpu_batch *batch, double dt_def);
int cmf_gpu_batch_advance(cmf_gpu_batch *batch, double dt_def, int32_t *nt_out, double *dt_out,
                          cmf_budget *budget_out);
int cmf_gpu_batch_synchronize(cmf_gpu_batch *batch);
void *cmf_gpu_batch_stream(cmf_gpu_batch *batch);
void cmf_gpu_batch_destroy(cmf_gpu_batch *batch);

/* Split outer step for basin-region sharding across GPUs (one 8-byte MIN all-reduce of DT_MIN
 * per outer step, src/cmf_ctrl_mpi_mod.F90:261-281): stage + local CFL minimum ... */
int cmf_gpu_ctx_stage(cmf_gpu_ctx *ctx, double dt_def, double *dt_min_local);
/* ... then the sub-steps with the globally reduced DT_MIN. */
int cmf_gpu_ctx_substeps(cmf_gpu_ctx *ctx, double dt_def, double dt_min_global, int32_t *nt_out,
                         double *dt_out, cmf_budget *budget_out);

/* Stage scheme + CFL minimum with no allocation by the library.  This entry point has no
 * counterpart in the reference: it serves hosts that cannot let a library allocate device memory
 * (a coupler whose pool owns all device memory, physics run during CUDA stream capture).  Every
 * pointer is a caller-owned DEVICE pointer on the current device; the library's only other global
 * memory is a fixed 64 KiB file-scope scratch array per GPU, held until process exit.  The
 * default stage scheme (CMF_CALC_FLDSTG_DEF) updates rivsto/fldsto in place and writes the six
 * diagnostics; *dt_min_out (device) receives min(DT, CFL minimum) of CALC_ADPSTP.  Limit:
 * NSEQALL <= 2,097,152 (larger returns CMF_E_ARG with a message).  The first call on a device
 * looks up the scratch array's address and must come before any stream capture.  All calls share
 * the scratch array: calls that overlap on the GPU (other streams, other host threads) race.
 * Enqueued on `stream` and asynchronous; no levee scheme in this variant. */
typedef struct cmf_stage_dev_args {
    int32_t nseqall, nseqriv, nlfp, ladpstp;
    double dt_def, pgrv, pdstmth, pcadp, dfrcinc;
    const double *rivstomax, *rivlen, *rivwth, *grarea, *rivelv, *nxtdst;
    const double *fldstomax, *fldgrd;        /* [NLFP][NSEQALL] */
    const int32_t *i2mask;
    double *rivsto, *fldsto;                 /* in/out */
    double *rivdph, *flddph, *fldfrc, *fldare, *sfcelv, *storge;   /* out */
    double *dt_min_out;                      /* out, one double */
    void *stream;                            /* cudaStream_t, may be NULL (legacy default stream) */
} cmf_stage_dev_args;
int cmf_gpu_stage_noalloc(const cmf_stage_dev_args *args);

/* ======================================================================================== */
/* Learned per-cell emulator (no counterpart in the reference): device building blocks       */
/* ======================================================================================== */
/* Device views of a context's network (next: 0-based downstream, -1 at mouths; upstream CSR in
 * the reference's I1UPST order) and the floodplain Manning coefficient.  qref (per-cell discharge
 * scale, m3/s) is set by the caller. */
typedef struct cmf_emu_net {
    int32_t nseqall, nseqriv;
    const int32_t *next, *up_ptr, *up_idx;
    const double *rivelv, *elevtn, *nxtdst, *rivwth, *rivhgt, *rivlen, *rivstomax, *qref, *rivman;
    double pmanfld;
} cmf_emu_net;
/* Device views of one member's state; qprev is the mean outflow of the last coupling step
 * (D2OUTFLW_aAVG of the physics, or the emulator's own prediction). */
typedef struct cmf_emu_member {
    double *rivsto, *fldsto, *levsto, *rivdph, *flddph, *fldfrc, *qprev, *runoff, *rivout_pre, *fldout_pre;
} cmf_emu_member;
int cmf_gpu_ctx_emu_views(cmf_gpu_ctx *ctx, int32_t member, cmf_emu_net *net, cmf_emu_member *mb);
/* Device-to-device copy of one member's prognostic state and last-step averages between two
 * contexts of the same network (hand-over between the emulator and the judging plain solver). */
int cmf_gpu_ctx_copy_member(cmf_gpu_ctx *dst, int32_t dst_member, cmf_gpu_ctx *src, int32_t src_member);
/* BF16 GEMM on the tcgen05 tensor cores (accumulator in tensor memory), fp32 accumulate:
 * C[M,N] (+)= op(A)[M,K] op(B)[K,N]; epilogue bias+ReLU, fp32 and/or bf16 output, or atomic
 * accumulation for split-K (ksplit > 1).  M,N % 64, K % 32, lda/ldb % 8, A and B 16-byte aligned.
 * A launch that gives up a bounded MMA wait reports through cmf_emu_mlp_tc_status. */
int cmf_emu_gemm(int M, int N, int K, const void *A, int lda, int transA, const void *B, int ldb, int transB,
                 float *C, int ldc, void *Cb, int ldcb, const float *bias, int relu, int accumulate, int ksplit,
                 void *stream);
/* Deterministic split-K on the same tensor cores: C[M,N] += op(A) op(B) with K split into
 * `ksplit` slices whose partial products go to `workspace` (at least
 * cmf_emu_gemm_splitk_ws_floats(M, N, K, ksplit) floats, 16-byte aligned) and are added to C in
 * slice order, so the result is the same bits on every run (the training's weight gradients). */
size_t cmf_emu_gemm_splitk_ws_floats(int M, int N, int K, int ksplit);
int cmf_emu_gemm_splitk(int M, int N, int K, const void *A, int lda, int transA, const void *B, int ldb, int transB,
                        float *C, int ldc, int ksplit, float *workspace, size_t workspace_floats, void *stream);
/* The same contract on the legacy mma.sync tiles (kept as the cross-check of cmf_emu_gemm). */
int cmf_emu_gemm_mma(int M, int N, int K, const void *A, int lda, int transA, const void *B, int ldb, int transB,
                     float *C, int ldc, void *Cb, int ldcb, const float *bias, int relu, int accumulate, int ksplit,
                     void *stream);
int cmf_emu_relu_bwd(int n, const float *dA, const void *act, void *dZ, float *dZf, void *stream);
int cmf_emu_colsum(int rows, int cols, const float *X, float *out, void *stream);
/* MSE gradient on column 0 of Y (rows padded, `valid` real rows): dY fp32 + bf16, loss partials
 * per 256-row block in loss_part[(rows+255)/256]. */
int cmf_emu_mse_grad(int rows, int valid, int ldy, const float *Y, const float *t, float *dY, void *dYb,
                     float *loss_part, void *stream);
int cmf_emu_adam(int n, float *w, void *wb, const float *grad, float *m, float *v, float lr, float b1, float b2,
                 float eps, int step, float wd, void *stream);
/* 14 local features + 2 channels x `hops` (<= 8) upstream messages + 2 Manning estimates -> the
 * first 32 columns of X rows (bf16, ldx % 8 == 0, X 16-byte aligned), for nmembers members whose
 * state arrays start at the member-0 views in mb (member-major [M][N]); member m's rows start at
 * m * rows_per_member.  planes: float scratch [2 * (hops + 1)][M * N]. */
int cmf_emu_features(const cmf_emu_net *net, const cmf_emu_member *mb, int nmembers, void *X, int ldx,
                     int rows_per_member, int hops, float *planes, void *stream);
/* Mass-conserving step from predicted transformed outflows y (column 0, stride ldy) for every
 * member with active_dev[m] != 0 (device int array); residual != 0: y is the change of
 * log1p(Q/qref) over the step, else its value; qout: double [M][N] scratch. */
int cmf_emu_rollout(const cmf_emu_net *net, const cmf_emu_member *mb, int nmembers, const int *active_dev,
                    const float *y, int ldy, int rows_per_member, double dt, int residual, double *qout, void *stream);
/* Fused inference of the 4-layer MLP.  cmf_emu_mlp_pack re-lays the bf16 weights (W0..W2 [K][128],
 * W3 [128][ldw3], row-major) into tensor-core fragment order in `pack` (cmf_emu_mlp_pack_bytes()
 * bytes, device memory); cmf_emu_mlp_fused then maps X rows (bf16, ldx >= 32 and even, columns
 * 32.. zero padding, rows % 16 == 0) to y[rows] (fp32) in one kernel with the activations kept in
 * registers.  y equals column 0 of the layer-by-layer forward built from cmf_emu_gemm bit for bit. */
size_t cmf_emu_mlp_pack_bytes(void);
int cmf_emu_mlp_pack(const void *W0, const void *W1, const void *W2, const void *W3, int ldw3, void *pack, void *stream);
int cmf_emu_mlp_fused(const void *X, int ldx, int rows, const void *pack, const float *b0, const float *b1,
                      const float *b2, const float *b3, float *y, void *stream);
/* The same fused inference on the 5th-generation tensor cores (tcgen05 MMA into tensor memory,
 * sm_100a): cmf_emu_mlp_tc_pack lays the four layers' weights out as one shared-memory image
 * (cmf_emu_mlp_tc_pack_bytes() bytes, 16-byte aligned device memory; W3 needs ldw3 >= 16 columns,
 * column 0 is the output); cmf_emu_mlp_tc maps X rows (bf16, ldx >= 32 and a multiple of 8, X
 * 16-byte aligned, columns 32.. ignored) to y[rows].  Rounding points as the layer-by-layer
 * chain; fp32 accumulation order is the tensor core's.  cmf_emu_mlp_tc_status() reports (after
 * the stream is synchronised) whether any launch since the last report gave up waiting for an MMA
 * (CMF_E_CUDA), and clears the report. */
size_t cmf_emu_mlp_tc_pack_bytes(void);
int cmf_emu_mlp_tc_pack(const void *W0, const void *W1, const void *W2, const void *W3, int ldw3, void *pack,
                        void *stream);
int cmf_emu_mlp_tc(const void *X, int ldx, int rows, const void *pack, const float *b0, const float *b1,
                   const float *b2, const float *b3, float *y, void *stream);
int cmf_emu_mlp_tc_status(void);
/* Diagnostic: bound (polls) of the MMA completion waits of later cmf_emu_mlp_tc launches; a
 * negative value restores the default.  With 0 every launch gives up at its first wait, reports
 * through cmf_emu_mlp_tc_status (which clears the report when it returns it) and still waits for
 * its MMA in flight, with the default bound, before releasing tensor memory. */
int cmf_emu_mlp_tc_set_wait_limit(int32_t limit);
const char *cmf_emu_last_error(void);

/* ======================================================================================== */
/* Default-context API bound by the Fortran ISO_C_BINDING shim                              */
/* ======================================================================================== */
int cmf_gpu_init(const cmf_dims *dims, const cmf_params *params, const cmf_map_ptrs *maps,
                 const cmf_opts *opts);
int cmf_gpu_set_state(const cmf_state_ptrs *st);
int cmf_gpu_get_state(const cmf_state_ptrs *st);
int cmf_gpu_put_runoff(const double *runoff, const double *rofsub);
int cmf_gpu_physics_advance(double dt_def, int32_t *nt_out, double *dt_out, cmf_budget *budget_out);
int cmf_gpu_get_diag(const cmf_diag_ptrs *dg);
/* replace CMF_DIAG_GETAVE_OUTPUT / CMF_DIAG_RESET_OUTPUT at src/cmf_drv_advance_mod.F90:123,143
 * (AVEMAX at :114 runs inside cmf_gpu_physics_advance when opts.ldiag_output is set) */
int cmf_gpu_diag_output(int32_t op);
int cmf_gpu_get_diag_output(const cmf_diag_out_ptrs *dg);
void cmf_gpu_finalize(void);
const char *cmf_gpu_strerror(int status);
const char *cmf_gpu_last_error(void);
int cmf_gpu_abi_version(void);
/* Diagnostic: evaluates on the current device the two depth powers of the flux formulas,
 * x**(-7._JPRB/3._JPRB) and x**(-4._JPRB/3._JPRB) (src/cmf_calc_outflw_mod.F90:74,106), exactly as
 * the sub-step kernels do, for n host values x; results into host arrays p73 and p43 (either may
 * be NULL).  Synchronous; allocates its own scratch. */
int cmf_gpu_depth_powers(const double *x, int32_t n, double *p73, double *p43);
/* Diagnostic: the CFL key of CALC_ADPSTP, PCADP*DDST*(PGRV*MAX(RIVDPH,0.01))**(-0.5)
 * (src/cmf_ctrl_physics_mod.F90:190-202), evaluated on the current device exactly as the stage
 * kernels do (the inverse square root correctly rounded), for n host values; key is a host
 * array.  Synchronous; allocates its own scratch. */
int cmf_gpu_cfl_keys(const double *rivdph, const double *ddst, int32_t n, double pgrv, double pcadp, double *key);

/* ======================================================================================== */
/* Host model core: the reference's CMF_DRV_INIT for a stand-alone (non-Fortran) host        */
/* ======================================================================================== */
typedef struct cmf_host_model cmf_host_model;

/* Reads input_cmf.nam (NRUNVER/NDIMTIME/NPARAM/NMAP/NLEVEE/NDAMOUT), diminfo and the binary
 * maps of casedir, then runs CMF_RIVMAP_INIT, CMF_TOPO_INIT, CMF_LEVEE_INIT, CMF_PROG_INIT,
 * CMF_PHYSICS_FLDSTG (host copy) and CMF_DAMOUT_INIT in the reference's order. */
int cmf_host_load(const char *casedir, const char *nmlfile, cmf_host_model **out);
void cmf_host_free(cmf_host_model *hm);
/* Fills the ABI structs with pointers into the host model (valid until cmf_host_free);
 * opts gets the namelist logicals and the GPU defaults; *dt gets DT. */
int cmf_host_describe(const cmf_host_model *hm, cmf_dims *dims, cmf_params *params,
                      cmf_map_ptrs *maps, cmf_opts *opts, double *dt);
/* Pointers to the host model's initialised prognostic arrays (single member). */
int cmf_host_state(cmf_host_model *hm, cmf_state_ptrs *st);
/* CONV_RESOL (src/cmf_ctrl_forcing_mod.F90:795-831): runoff map [mm/dt, NX*NY] -> m3/s. */
int cmf_host_conv_resol(const cmf_host_model *hm, const double *map, double *runoff_out);
/* Grid position of every sequence cell (I1SEQX/I1SEQY, 1-based) and the grid size. */
int cmf_host_grid(const cmf_host_model *hm, int32_t *nx, int32_t *ny, int32_t *i1seqx, int32_t *i1seqy);
/* CMF_INPMAT_INIT_BIN (src/cmf_ctrl_forcing_mod.F90:418-458): reads the input-matrix file (3*INPN
 * records of NX x NY 4-byte values: INPX int32 x INPN, INPY int32 x INPN, INPA float32 x INPN) into
 * sequence order, [INPN][NSEQMAX] each (INPA promoted to double). */
int cmf_host_read_inpmat(const cmf_host_model *hm, const char *file, int32_t inpn, int32_t *inpx, int32_t *inpy,
                         double *inpa);
/* DROFUNIT of the namelist NFORCE (runoff unit divisor, src/cmf_ctrl_forcing_mod.F90:59). */
double cmf_host_drofunit(const cmf_host_model *hm);
/* mapR2vecD (src/cmf_utils_mod.F90:282-303): an NX x NY float map (e.g. a sea-level record of
 * CMF_BOUNDARY_GET_BIN) to a double vector in sequence order. */
int cmf_host_map_to_vec(const cmf_host_model *hm, const float *map, double *vec);
/* Binary restart of one member's state in the reference's layout (CMF_RESTART_WRITE / WRTE_REST_BIN,
 * src/cmf_ctrl_restart_mod.F90:389-482; CMF_RESTART_INIT / READ_REST_BIN, :91-204): NX x NY map
 * records (FP64 when lrestdbl, else FP32; 1.E20 outside the sequence) rivsto, fldsto, [rivout_pre,
 * fldout_pre, rivdph_pre, fldsto_pre unless lstoonly], [damsto], [levsto], and <file>.pth with
 * D1PTHFLW_PRE.  The read zeroes every prognostic first and leaves rivout/fldout/pthflw at zero,
 * as the reference's binary path does; with lstoonly it sets fldsto_pre = fldsto.  The caller
 * names the file (the reference uses CRESTDIR//CVNREST//YYYYMMDDHH//'.bin'). */
int cmf_host_write_restart(const cmf_host_model *hm, const cmf_state_ptrs *st, const char *file, int32_t lrestdbl,
                           int32_t lstoonly);
int cmf_host_read_restart(const cmf_host_model *hm, const cmf_state_ptrs *st, const char *file, int32_t lrestdbl,
                          int32_t lstoonly);

#ifdef __cplusplus
}
#endif
#endif /* CMF_GPU_H */
