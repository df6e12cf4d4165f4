/*
 * cmscan_gpu.h -- C ABI of the B200 covariance-model scan library
 * (libcmscan_gpu.so).
 *
 * The library replaces the QDB-banded CYK / Inside window scanner of infernox
 * (src/cm_nohmm.rs) behind plain C entry points: POD structs, raw pointers and
 * sizes, int status codes, no exceptions and no torch types.  A Rust caller
 * binds these with an `extern "C"` block; the Python package `infernox_b200`
 * binds them with ctypes.
 *
 * Conventions
 *   - Every entry point returns CMGPU_OK (0) or a negative CMGPU_E* code;
 *     cmgpu_last_error() returns a message for the calling thread.
 *   - Digital sequences are "window frames" exactly as the reference passes
 *     them: dsq[0] = 255 (sentinel), dsq[1..n] residue codes 0..17
 *     (A0 C1 G2 U3, gap 4, IUPAC 5..15, nonresidue 16, missing 17),
 *     dsq[n+1] = 255.
 *   - Coordinates are 1-based window coordinates, as in the reference.
 *   - Scores are bits.  Integer Inside scores are the reference's
 *     INTSCALE=1000 fixed point with -INFTY = -987654321.
 *   - A model handle is read-only after upload and may be shared by threads;
 *     a workspace handle must be used by one thread at a time.
 */
#ifndef CMSCAN_GPU_H
#define CMSCAN_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CMGPU_OK 0
#define CMGPU_EINVAL (-1)     /* bad argument                                */
#define CMGPU_ENOMEM (-2)     /* host or device allocation failed            */
#define CMGPU_EDEVICE (-3)    /* CUDA error (message in cmgpu_last_error)    */
#define CMGPU_EOVERFLOW (-4)  /* caller's output array too small; *n_out set */
#define CMGPU_ERANGE (-5)     /* band calculation did not converge           */
#define CMGPU_ETIMEOUT (-6)   /* a device-side bounded wait gave up          */
#define CMGPU_ENOSPACE (-7)   /* request exceeds a fixed capacity            */

#define CMGPU_KP 18           /* digital alphabet size incl. degeneracies    */
#define CMGPU_MAXCONNECT 6    /* max children of a CM state                  */
#define CMGPU_ESC_STRIDE 324  /* per-state emission row: 18 (single), 18*18 (pair) */
#define CMGPU_INFTY 987654321

/* Semirings of the scanner (the reference's `generic_scan::<f32>` and
 * `generic_scan::<i32>`, src/cm_nohmm.rs:406). */
#define CMGPU_CYK_F32 0
#define CMGPU_INSIDE_I32 1
#define CMGPU_INSIDE_F32 2    /* float Inside (FLogsum): HMM-banded scans only */

/* Band sets (src/cm_nohmm.rs:261-262 SMX_QDB1_TIGHT / SMX_QDB2_LOOSE; 0 = the
 * `nonbanded` full d-range of the --max path, src/cm_nohmm.rs:431-437). */
#define CMGPU_NOQDB 0
#define CMGPU_QDB1 1
#define CMGPU_QDB2 2

/* Probability-level covariance model: structure + parameters, as read from a
 * CM file in global configuration (src/cm.rs:315-563).  Arrays are caller
 * owned.  t is [M][6], e is [M][16] (pairs a*4+b; singles use [0..4]). */
typedef struct cmgpu_cm_params {
    int32_t M, nodes, clen;
    const int8_t *sttype, *stid, *ndtype;
    const int32_t *ndidx, *cfirst, *cnum, *plast, *pnum, *nodemap;
    const float *t, *e;
    float null[4];
    float el_selfsc;      /* EL self-transition score (bits)               */
    float pbegin, pend;   /* local begin / end probabilities (0.05)        */
    float n3_omega;       /* null3 prior                                   */
} cmgpu_cm_params;

/* The scanner's view of a configured CM: exactly the fields generic_scan,
 * report_hits_greedily and the null3 correction read from `&CM`
 * (src/cm_nohmm.rs:406-812).  Arrays are caller owned; per-state rows:
 * tsc/itsc [M][6], oesc/ioesc [M][324]. */
typedef struct cmgpu_cm {
    int32_t M;
    int32_t W;            /* window length cm.w                            */
    uint32_t flags;       /* bit 10 = local begins (CMH_LOCAL_BEGIN)       */
    const int8_t *sttype, *stid;
    const int32_t *cfirst, *cnum;
    const float *tsc, *oesc, *endsc, *beginsc;
    float el_selfsc;
    const int32_t *itsc, *ioesc, *iendsc, *ibeginsc;
    int32_t iel_selfsc;
    const int32_t *dmin1, *dmax1, *dmin2, *dmax2;
    float null[4];
    float n3_omega;
} cmgpu_cm;

/* Output arrays filled by cmgpu_prep_configure (all caller allocated). */
typedef struct cmgpu_cm_scores {
    float *tsc, *oesc, *endsc, *beginsc;     /* [M*6], [M*324], [M], [M]   */
    int32_t *itsc, *ioesc, *iendsc, *ibeginsc;
    int32_t *dmin1, *dmax1, *dmin2, *dmax2;   /* [M] each                   */
    float *t_local;       /* [M*6] transition probs after localisation     */
    float el_selfsc;      /* out */
    int32_t iel_selfsc;   /* out */
    int32_t W;            /* out: dmax of ROOT at beta_W                   */
    uint32_t flags;       /* out */
} cmgpu_cm_scores;

typedef struct cmgpu_hit {
    int32_t i, j;         /* window coordinates                            */
    float score;          /* null3-corrected bit score                     */
    float bias;           /* null3 correction                              */
} cmgpu_hit;

typedef struct cmgpu_envelope {
    int32_t start, end;
} cmgpu_envelope;

/* One scan job of a batch: window [i0, j0] of the frame starting at byte
 * dsq_offset of the batch's residue buffer (frame[0] is the sentinel). */
typedef struct cmgpu_window {
    int64_t dsq_offset;
    int32_t i0, j0;
} cmgpu_window;

typedef struct cmgpu_batch_hit {
    int32_t win;          /* index of the window in the batch              */
    int32_t i, j;
    float score, bias;
} cmgpu_batch_hit;

/* Per-call counters (cells = (j,v,d) DP cells computed, terms = child
 * relaxations, both counted from the bands exactly as the oracle counts). */
typedef struct cmgpu_stats {
    double cells, terms, residues;
    int64_t work_items, candidates;
    float kernel_ms;      /* device time of the scan kernel(s)             */
    int32_t kernel_launches;
    int32_t deck_in_smem; /* 1 when the rolling decks live in shared memory */
    int32_t ctas;
    int32_t lanes;        /* work items per CTA                            */
    int32_t kernel;       /* CMGPU_KERNEL_LEVEL or CMGPU_KERNEL_SWEEP       */
} cmgpu_stats;

/* Scan kernels of the QDB scanner (cmgpu_workspace_set_kernel).  Both give
 * the same results.  LEVEL: one CTA scans up to 16 work items side by side,
 * state by state in dependency levels with CTA barriers (qdb_scan.cu).
 * SWEEP: one warp scans one work item node by node with no CTA barrier
 * (sweep_scan.cu); it needs W <= 255 and the node-local state topology of
 * CMs built by cmbuild.  AUTO picks LEVEL. */
#define CMGPU_KERNEL_AUTO 0
#define CMGPU_KERNEL_LEVEL 1
#define CMGPU_KERNEL_SWEEP 2

typedef struct cmgpu_model cmgpu_model;
typedef struct cmgpu_workspace cmgpu_workspace;

const char *cmgpu_last_error(void);
const char *cmgpu_version(void);

/* ---- host-side model preparation (no GPU needed) ------------------------
 * Configures a probability-level CM for scanning, as FaithfulSearcher::new
 * does (src/cm_search.rs:871-979): QDB bands and W on the global model
 * (cm_calc_qdb_bands, src/cm_nohmm.rs:374 -> band_calculation_engine,
 * src/cm_qdband.rs:258), then either the global scores
 * (cm_configure_scores_global, src/cm_nohmm.rs:264) or the local ones
 * (cm_configure_scores, src/cp9.rs:4538, plus build_integer_scores,
 * src/cm_nohmm.rs:279).  local=0/1.  W_in > 0 keeps a file W; 0 computes it. */
int cmgpu_prep_configure(const cmgpu_cm_params *p, int local, int32_t W_in,
                         double beta1, double beta2, double betaW,
                         cmgpu_cm_scores *out);

/* The CP9 HMM of a CM (cp9_build_and_configure, src/cp9.rs:2212-2232): the
 * profile HMM that HMM-banded search derives its bands from, built from the
 * global CM and put in local mode (begins and ends at pbegin, end-local
 * exits at pend).  Caller-allocated, M = the CM's consensus length:
 * mat / ins [(M+1)*4] emissions, t [(M+1)*10] transitions MM MI MD MEL IM II
 * ID DM DI DD, begin / end [M+1], msc / isc [(M+1)*18] integer emission
 * scores, otsc [(M+1)*12] integer transition scores in the DP's order MM IM
 * DM BM MI II DI MD ID DD ME MEL, has_el [M+1] (an end-local exit leaves
 * node k), hns2cs [(M+1)*3*2] the CM states behind node k's match, insert
 * and delete states (-1: none), el_pairs [nodes*2] the (source, destination)
 * HMM nodes of every end-local exit in CM node order (CPlan9InitEL's
 * el_from_idx lists, src/cp9.rs:1061-1075), their count in n_el. */
typedef struct cmgpu_cp9 {
    int32_t M;
    float *mat, *ins, *t, *begin, *end;
    int32_t *msc, *isc, *otsc;
    uint8_t *has_el;
    int32_t *hns2cs;
    int32_t *el_pairs;
    int32_t n_el;           /* out */
    float el_self;          /* out */
    int32_t el_selfsc;      /* out */
} cmgpu_cp9;
int cmgpu_prep_cp9(const cmgpu_cm_params *p, cmgpu_cp9 *out);

/* Inputs of the truncated scanners for a configured CM, all caller
 * allocated: the marginal emission scores (fill_marginal_emissions,
 * src/cp9.rs:4441) lmesc/rmesc and ilmesc/irmesc [M*18]; the truncated-begin
 * penalties of the local (local != 0) or global configuration
 * (TrPenalties::new, src/cm_trunc.rs:192, from the expected state occupancy
 * of src/cp9.rs:752 and the emit map of src/cp9.rs:144) as rows [3][M] --
 * 5'-and-3', 5'-only, 3'-only, the order of pty_idx_for_pass -- in pty (log2)
 * and ipty (Prob2Score); and the node span lpos/rpos [M] allow_truncation
 * reads for each state (src/cm_dpsearch_trunc.rs:2395-2406). */
typedef struct cmgpu_tr_prep {
    float *lmesc, *rmesc;
    int32_t *ilmesc, *irmesc;
    float *pty;
    int32_t *ipty;
    int32_t *lpos, *rpos;
} cmgpu_tr_prep;
int cmgpu_prep_truncated(const cmgpu_cm_params *p, int local, cmgpu_tr_prep *out);

/* ILogsum table (src/cp9.rs:28-44): tbl[0..n) with n <= 23000. */
int cmgpu_ilogsum_table(int32_t *tbl, int32_t n);
/* FLogsum table (src/cp9.rs:5391-5400). */
int cmgpu_flogsum_table(float *tbl, int32_t n);

/* ---- device model and workspace ---------------------------------------- */
int cmgpu_model_upload(const cmgpu_cm *cm, int device, cmgpu_model **out);
void cmgpu_model_free(cmgpu_model *m);
/* stream: a cudaStream_t or NULL for a library-owned stream. */
int cmgpu_workspace_create(int device, void *stream, cmgpu_workspace **out);
void cmgpu_workspace_free(cmgpu_workspace *ws);
int cmgpu_workspace_stats(const cmgpu_workspace *ws, cmgpu_stats *out);
/* Launch shape override for tuning (0 keeps the tuned value): CTAs per SM
 * (1..4), threads in {128,256,512}, residues per work item, work items
 * scanned side by side per CTA (1..8). */
int cmgpu_workspace_set_shape(cmgpu_workspace *ws, int ctas_per_sm, int threads, int chunk,
                              int lanes);
/* Kernel choice for the scans of this workspace (CMGPU_KERNEL_*).  A scan
 * with CMGPU_KERNEL_SWEEP on a model outside that kernel's scope fails with
 * CMGPU_EINVAL.  With SWEEP, set_shape's `lanes` is the warps per CTA (1..12)
 * and `chunk` the residues per work item. */
int cmgpu_workspace_set_kernel(cmgpu_workspace *ws, int kernel);

/* ---- scanner entry points ----------------------------------------------- */

/* generic_scan (src/cm_nohmm.rs:406-763): scan window [i0, j0] of dsq and
 * return the greedily reported, overlap-pruned hits (score order). */
int cmgpu_qdb_scan(const cmgpu_model *m, cmgpu_workspace *ws, int semiring,
                   int qdbidx, const uint8_t *dsq, int32_t n, int32_t i0,
                   int32_t j0, float cutoff, int do_null3, cmgpu_hit *hits,
                   int32_t cap, int32_t *n_out);

/* Window scan that allocates no device memory.  It has no counterpart in the
 * reference.  It serves callers that cannot call cudaMalloc or cudaFree: a
 * process whose device memory belongs to a framework's caching allocator or
 * to a fixed per-tenant budget, where a raw allocation fails or escapes the
 * accounting, and a process running other streams on the GPU that cannot
 * accept the device-wide synchronisation cudaFree implies.  Same arguments
 * and results as cmgpu_qdb_scan, minus the workspace; stream is a
 * cudaStream_t (NULL: the default stream).  The call waits for its stream
 * and returns with the scan finished; the calling thread's current device is
 * unchanged on return.  Its scratch -- a copy of the scan plan, the residues,
 * work items, counters, reportable cells and, when they do not fit in shared
 * memory, the decks -- lives in one 16 MiB `static __device__` array that
 * every GPU loading the library holds until the process exits.  Requests
 * that do not fit return CMGPU_ENOSPACE.  The first call on a device looks up
 * the array's address with cudaGetSymbolAddress (a one-time set-up).  All
 * calls on a device share the array: calls that overlap on the GPU race, so
 * serialise them.  The model must already be uploaded (cmgpu_model_upload). */
int cmgpu_qdb_scan_noalloc(const cmgpu_model *m, void *stream, int semiring, int qdbidx,
                           const uint8_t *dsq, int32_t n, int32_t i0, int32_t j0,
                           float cutoff, int do_null3, cmgpu_hit *hits, int32_t cap,
                           int32_t *n_out);

/* Test hook, the analogue of the reference's DUMP_* value dumps: every
 * reportable cell (j, d) of a generic_scan of [i0, j0] with bestsc >= cutoff,
 * sorted by (j, d), with its bit score, before null3 and greedy reporting. */
int cmgpu_qdb_scan_cells(const cmgpu_model *m, cmgpu_workspace *ws, int semiring,
                         int qdbidx, const uint8_t *dsq, int32_t n, int32_t i0,
                         int32_t j0, float cutoff, int32_t *cj, int32_t *cd,
                         float *csc, int32_t cap, int32_t *n_out);

/* cyk_seq_filter (src/cm_nohmm.rs:855-889): QDB1 CYK over [1, n] then hits
 * padded by W-1 and merged into envelopes (ascending end). */
int cmgpu_cyk_seq_filter(const cmgpu_model *m, cmgpu_workspace *ws,
                         const uint8_t *dsq, int32_t n, float cutoff,
                         int do_null3, cmgpu_envelope *envs, int32_t cap,
                         int32_t *n_out);

/* final_stage_inside_opt (src/cm_nohmm.rs:919-935): integer Inside over each
 * envelope (QDB2, or the full d-range when nonbanded != 0); hits of all
 * envelopes concatenated in envelope order. */
int cmgpu_final_stage_inside_opt(const cmgpu_model *m, cmgpu_workspace *ws,
                                 const uint8_t *dsq, int32_t n,
                                 const cmgpu_envelope *envs, int32_t nenv,
                                 float cutoff, int do_null3, int nonbanded,
                                 cmgpu_hit *hits, int32_t cap, int32_t *n_out);

/* Batched scan: every window is scanned as generic_scan would scan it on its
 * own (same hits, same order), but all windows of the batch share one
 * cost-ordered persistent launch.  dsq_all is host memory. */
int cmgpu_scan_batch(const cmgpu_model *m, cmgpu_workspace *ws, int semiring,
                     int qdbidx, const uint8_t *dsq_all, int64_t dsq_len,
                     const cmgpu_window *wins, int32_t nwin, float cutoff,
                     int do_null3, cmgpu_batch_hit *hits, int32_t cap,
                     int32_t *n_out);

/* As cmgpu_scan_batch with the residue buffer already resident in device
 * memory (d_dsq_all is a device pointer); windows and hits stay on the host. */
int cmgpu_scan_batch_device(const cmgpu_model *m, cmgpu_workspace *ws,
                            int semiring, int qdbidx, const uint8_t *d_dsq_all,
                            int64_t dsq_len, const cmgpu_window *wins,
                            int32_t nwin, float cutoff, int do_null3,
                            cmgpu_batch_hit *hits, int32_t cap, int32_t *n_out);

/* Plain comparator: one launch per window, one CTA per window, no work queue
 * and no sub-chunking.  Same results as cmgpu_scan_batch. */
int cmgpu_scan_plain(const cmgpu_model *m, cmgpu_workspace *ws, int semiring,
                     int qdbidx, const uint8_t *dsq_all, int64_t dsq_len,
                     const cmgpu_window *wins, int32_t nwin, float cutoff,
                     int do_null3, cmgpu_batch_hit *hits, int32_t cap,
                     int32_t *n_out);

/* ---- cmcalibrate (src/cm_calibrate.rs) ------------------------------------
 * The exponential-tail E-value fit of a CM in its four modes, indexed
 * GC, GI, LC, LI = glocal CYK, glocal Inside, local CYK, local Inside
 * (EXP_CM_*, src/cm_calibrate.rs:38-42). */
typedef struct cmgpu_calibrate_config {
    uint32_t seed;        /* generator seed (181)                              */
    double l_mb;          /* Mb of random sequence, in 10 kb sequences (1.6)   */
    double beta;          /* tail loss of both QDB band sets (1e-15)           */
    int32_t nonbanded;    /* full d-range instead of QDB bands                 */
    int32_t gtailn;       /* tail hits per Mb fitted, glocal modes (250)       */
    int32_t ltailn;       /* tail hits per Mb fitted, local modes (750)        */
    float tailp;          /* > 0: fixed tail mass instead of gtailn / ltailn   */
    int32_t do_null3;     /* null3 correction of the hit scores (1)            */
} cmgpu_calibrate_config;

/* ExpParams (src/evalue.rs:8-17) as set_exp_info fills it: mu is the
 * extrapolated location, mu_orig the fitted one. */
typedef struct cmgpu_exp_params {
    double lambda, mu, dbsize, mu_orig, tailp;
    int32_t nrandhits;
} cmgpu_exp_params;

typedef struct cmgpu_calibrate_result {
    cmgpu_exp_params exp[4];  /* GC, GI, LC, LI                               */
    int32_t nhits[4];         /* hits in each mode's histogram                */
    double dbsize;            /* residues scored per mode                     */
    double cells;             /* DP cells of the four scans                   */
    double terms;             /* child relaxations of the four scans          */
    float kernel_ms;          /* device time of the four scans                */
    int32_t launches;         /* scan kernel launches                         */
} cmgpu_calibrate_result;

/* generate_sequences / SampleGenomicSequenceFromHMM (src/cm_calibrate.rs:
 * 184-200, 1113-1124): nseq frames of L residues drawn from the five-state
 * genomic HMM with easel's Mersenne Twister seeded with `seed`, written
 * back to back as [255, L codes 0..3, 255].  No GPU. */
int cmgpu_genomic_sample(uint32_t seed, int32_t L, int32_t nseq, uint8_t *frames);

/* fit_histogram + SetExpInfo (src/cm_calibrate.rs:1000-1099): the tail mass
 * (tailp > 0, else the mode's tail hits per Mb of nseq x L residues), the
 * top floor(n * tailp) scores and the complete-data exponential fit.
 * CMGPU_ERANGE where the reference returns an error (too few tail points,
 * tailn too large, non-finite lambda or score).  No GPU. */
int cmgpu_exp_fit(const float *scores, int64_t n, int exp_mode, int32_t nseq, int32_t L, int32_t gtailn,
                  int32_t ltailn, float tailp, double dbsize, cmgpu_exp_params *out);

/* collect_scores's scan (src/cm_calibrate.rs:441-989): each window scanned
 * as cmcalibrate's generic_scan does -- cutoff -inf, local begins compared
 * in bit scores -- with the kept hits of every window, in window order.  The
 * device emits only the ROOT cells the greedy report could take. */
int cmgpu_calibrate_scan_batch(const cmgpu_model *m, cmgpu_workspace *ws, int semiring, int qdbidx,
                               const uint8_t *dsq_all, int64_t dsq_len, const cmgpu_window *wins,
                               int32_t nwin, int do_null3, cmgpu_batch_hit *hits, int32_t cap,
                               int32_t *n_out);

/* calibrate_cm (src/cm_calibrate.rs:1102-1182): a probability-level CM with
 * window length W; the global and local configurations with both band sets
 * at cfg->beta, the random sequences, one batched scan per mode on `device`
 * and the four fits.  The modes run on two host threads with a workspace
 * each, so one mode's host work overlaps another's scan; kernel_ms is the
 * sum of the four scans' device times. */
int cmgpu_calibrate(const cmgpu_cm_params *p, int32_t W, int device, const cmgpu_calibrate_config *cfg,
                    cmgpu_calibrate_result *out);

/* ---- HMM-banded (CP9-banded) scanners ------------------------------------
 * Bands of one envelope as CP9Bands holds them (src/cp9.rs:1450-1495): for
 * each CM state v, rows j = jmin[v]..jmax[v] (none when jmax < jmin), and for
 * row jp = j - jmin[v] the d-band hdmin..hdmax (empty when hdmax < hdmin),
 * stored at hdmin[hd_off[v] + jp] / hdmax[hd_off[v] + jp].  Every cell must
 * lie inside the envelope (i = j-d+1 >= i0, j <= j0, d >= 0); rows of
 * emitting states start at d >= 1 and END rows are non-empty, as
 * ij2d_bands (src/cp9.rs:3815) and the reference's wide-band test fixture
 * build them. */
typedef struct cmgpu_hb_bands {
    const int32_t *jmin, *jmax;   /* [M] */
    const int32_t *hd_off;        /* [M] */
    const int32_t *hdmin, *hdmax; /* rows */
} cmgpu_hb_bands;

/* One envelope of a batched HMM-banded scan: residues i0..j0 of the buffer
 * at dsq_offset (dsq_offset + x is residue x), its bands and cutoffs. */
typedef struct cmgpu_hb_task {
    int64_t dsq_offset;
    int32_t i0, j0;
    float env_cutoff, cutoff;
    cmgpu_hb_bands bands;
} cmgpu_hb_task;

/* Per-envelope result: vsc_root, the envelope of ROOT cells >= env_cutoff
 * (-1 when none), and the envelope's hits in hits[hit_first .. +nhits). */
typedef struct cmgpu_hb_result {
    float vsc_root;
    int32_t nhits;
    int64_t envi, envj;
    int64_t hit_first;
} cmgpu_hb_result;

/* fast_cyk_scan_hb (src/cp9.rs:4682): HMM-banded CYK filter scan of dsq's
 * residues i0..j0 (dsq = [255, codes.., 255] frame of n residues). */
int cmgpu_fast_cyk_scan_hb(const cmgpu_model *m, const cmgpu_hb_bands *bands, const uint8_t *dsq,
                           int32_t n, int32_t i0, int32_t j0, float env_cutoff, float *vsc_root,
                           int64_t *envi, int64_t *envj);
/* fast_fcyk_scan_hb (:4704, semiring CMGPU_CYK_F32) and fast_finside_scan_hb
 * (:5465, CMGPU_INSIDE_F32): the same plus the greedily reported hits (with
 * null3 when do_null3), before overlap removal, as the reference returns
 * them.  CMGPU_EOVERFLOW with the needed count in *n_out if cap is short. */
int cmgpu_hb_scan_hits(const cmgpu_model *m, int semiring, const cmgpu_hb_bands *bands,
                       const uint8_t *dsq, int32_t n, int32_t i0, int32_t j0, float env_cutoff,
                       float cutoff, int do_null3, float *vsc_root, int64_t *envi, int64_t *envj,
                       cmgpu_hit *hits, int32_t cap, int32_t *n_out);
/* Many envelopes (each with its own bands) in one call, one CTA per
 * envelope.  report_hits = 0 gives the filter form (no hits). */
int cmgpu_hb_scan_batch(const cmgpu_model *m, void *stream, int semiring, int report_hits, int do_null3,
                        const uint8_t *dsq_all, int64_t dsq_len, const cmgpu_hb_task *tasks,
                        int32_t ntask, cmgpu_hb_result *results, cmgpu_hit *hits, int64_t cap,
                        int64_t *n_out);
/* ---- truncated HMM-banded scanners (tr_cyk_scan_hb / ftr_inside_scan_hb) --
 * The per-pass inputs the reference's truncated scanner selects internally
 * (src/cm_dpsearch_trunc.rs:264-300): marginal emissions (CM.lmesc/rmesc,
 * src/cp9.rs:4441), the truncated-begin penalties of the pass and
 * configuration (TrPenalties l/g[pty_idx_for_pass(pass)], IMPOSSIBLE where
 * none), and the node span allow_truncation reads for each state (lpos of
 * the state's node, +1 unless MATP/MATL; rpos, -1 unless MATP/MATR). */
typedef struct cmgpu_tr_tables {
    const float *lmesc, *rmesc;   /* [M*18] */
    const float *pty;             /* [M] */
    const int32_t *lpos, *rpos;   /* [M] */
    int32_t clen;
    int32_t local;                /* truncation rules of local configurations */
    /* integer versions (CM.ilmesc/irmesc, TrPenalties il/ig), read only by
     * the integer Inside truncated QDB scan; may be NULL otherwise */
    const int32_t *ilmesc, *irmesc, *ipty;
} cmgpu_tr_tables;

/* TrHit (src/cm_dpsearch_trunc.rs:131-139): mode 3 J, 2 L, 1 R, 0 T;
 * root = the entry (truncated-begin) state. */
typedef struct cmgpu_tr_hit {
    int32_t i, j;
    float score, bias;
    int32_t mode, root;
} cmgpu_tr_hit;

/* One envelope of a batched truncated scan: as cmgpu_hb_task plus the
 * per-state J/L/R/T validity of its bands (CP9Bands jvalid..tvalid). */
typedef struct cmgpu_tr_task {
    int64_t dsq_offset;
    int32_t i0, j0;
    float env_cutoff, cutoff;
    cmgpu_hb_bands bands;
    const uint8_t *jvalid, *lvalid, *rvalid, *tvalid;  /* [M] */
} cmgpu_tr_task;

typedef struct cmgpu_tr_result {
    float vsc_root;
    int32_t vmode;
    int64_t envi, envj;
    int64_t hit_first;
    int32_t nhits, pad;
} cmgpu_tr_result;

/* tr_cyk_scan_hb (CMGPU_CYK_F32, src/cm_dpsearch_trunc.rs:264) and
 * ftr_inside_scan_hb (CMGPU_INSIDE_F32, :1055) of residues i0..j0 of dsq
 * in pass pass_idx (PLI_PASS_*: 2 5'-only, 3 3'-only, 4/5 5'-and-3'; other
 * passes return CMGPU_EINVAL, as the reference's truncated scanners refuse
 * them):
 * vsc_root and its mode, the envelope (-1 when none) and the hits after
 * overlap removal, as the reference returns them. */
int cmgpu_tr_scan_hb(const cmgpu_model *m, int semiring, const cmgpu_tr_tables *tt, const cmgpu_hb_bands *bands,
                     const uint8_t *jvalid, const uint8_t *lvalid, const uint8_t *rvalid, const uint8_t *tvalid,
                     const uint8_t *dsq, int32_t n, int32_t i0, int32_t j0, float cutoff, int do_null3,
                     int pass_idx, float env_cutoff, float *vsc_root, int32_t *vmode, int64_t *envi,
                     int64_t *envj, cmgpu_tr_hit *hits, int32_t cap, int32_t *n_out);
/* Many envelopes in one call, one CTA per envelope. */
int cmgpu_tr_scan_hb_batch(const cmgpu_model *m, void *stream, int semiring, const cmgpu_tr_tables *tt,
                           int pass_idx, int do_null3, const uint8_t *dsq_all, int64_t dsq_len,
                           const cmgpu_tr_task *tasks, int32_t ntask, cmgpu_tr_result *results,
                           cmgpu_tr_hit *hits, int64_t cap, int64_t *n_out);

/* ---- truncated QDB / non-banded scanner (generic_tr_scan) ---------------
 * ref_tr_cyk_scan (CMGPU_CYK_F32, src/cm_dpsearch_trunc.rs:207) and
 * ref_itr_inside_scan (CMGPU_INSIDE_I32, :226) of residues i0..j0 with the
 * QDB bands qdbidx (CMGPU_NOQDB / QDB1 / QDB2) in pass pass_idx: the hits
 * after overlap removal, vsc_root and its mode, and the best score spanning
 * the full window as the reference computes it (bsc_full).  The scan runs
 * the columns of a window in order on one CTA: its ROOT row carries over
 * from column to column as in the reference, so windows are not split. */
typedef struct cmgpu_trq_result {
    float vsc_root;
    int32_t vmode;
    float bsc_full;
    int32_t nhits;
    int64_t hit_first;
} cmgpu_trq_result;

int cmgpu_tr_qdb_scan(const cmgpu_model *m, int semiring, int qdbidx, const cmgpu_tr_tables *tt,
                      const uint8_t *dsq, int32_t n, int32_t i0, int32_t j0, float cutoff, int do_null3,
                      int pass_idx, float *vsc_root, int32_t *vmode, float *bsc_full, cmgpu_tr_hit *hits,
                      int32_t cap, int32_t *n_out);
/* Many windows in one call, one CTA per window. */
int cmgpu_tr_qdb_scan_batch(const cmgpu_model *m, void *stream, int semiring, int qdbidx,
                            const cmgpu_tr_tables *tt, int pass_idx, int do_null3, const uint8_t *dsq_all,
                            int64_t dsq_len, const cmgpu_window *wins, int32_t nwin, float cutoff,
                            cmgpu_trq_result *results, cmgpu_tr_hit *hits, int64_t cap, int64_t *n_out);
/* Test hook for failure detection: in the next truncated QDB call the warp
 * that runs column `column` (0-based within each window) never publishes its
 * progress, so the next column's bounded wait runs out (about a second) and
 * the call fails with CMGPU_ETIMEOUT instead of hanging; -1 clears it.  The
 * model stays usable. */
int cmgpu_tr_qdb_inject_stall(cmgpu_model *m, int32_t column);
/* Device memory the truncated QDB scan may hold in window decks at once
 * (each resident window has its own; the grid is cut to fit).  0 restores
 * the default, 4 GiB. */
int cmgpu_tr_qdb_set_deck_budget(cmgpu_model *m, int64_t bytes);
/* Device time, J-plane cells and launches of the last truncated QDB call. */
int cmgpu_tr_qdb_stats(const cmgpu_model *m, double *kernel_ms, int64_t *cells, int32_t *launches);

/* Device time and cells of the last HMM-banded call on this model. */
int cmgpu_hb_stats(const cmgpu_model *m, double *kernel_ms, int64_t *cells, int32_t *launches);

/* ---- P7 Viterbi filter (F2) ---------------------------------------------
 * A p7 filter profile as the reference's P7Profile holds it
 * (src/p7_hmm.rs:62-92): mat[k*4+x] match emissions for k = 1..M (row 0
 * unused), trans[k*7+t] transitions MM,MI,MD,IM,II,DM,DD for k = 0..M. */
typedef struct cmgpu_p7_profile {
    int32_t M;
    const float *mat;
    const float *trans;
} cmgpu_p7_profile;

typedef struct cmgpu_vit_filter cmgpu_vit_filter;

/* build_vit_filter (src/p7_vitfilter.rs:121-278): quantised int16 tables,
 * uploaded to `device` (device < 0: host tables only, for inspection). */
int cmgpu_vit_filter_build(const cmgpu_p7_profile *p, int device, cmgpu_vit_filter **out);
void cmgpu_vit_filter_free(cmgpu_vit_filter *f);
/* The filter's tables, [(M+1)][26]: emissions of the 18 codes, then local
 * entry, MM, IM, DM (row k-1 feeds position k), MI, II, MD, DD; specials =
 * {base_w, E move, E loop}.  For tests and inspection. */
int cmgpu_vit_filter_tables(const cmgpu_vit_filter *f, int16_t *tab, int32_t cap, int32_t *n_out,
                            int16_t *specials);
/* vit_score (src/p7_vitfilter.rs:292): the filter score in bits of residues
 * i0..j0 of every window; scored[w] = 0 where the reference returns None
 * (16-bit overflow, score NaN).  stream: cudaStream_t or NULL. */
int cmgpu_vit_score_batch(const cmgpu_vit_filter *f, void *stream, const uint8_t *dsq_all,
                          int64_t dsq_len, const cmgpu_window *wins, int32_t nwin, float *scores,
                          uint8_t *scored);

/* Device time, cells (residues x M) and launches of the last
 * cmgpu_vit_score_batch call on this filter. */
int cmgpu_vit_filter_stats(const cmgpu_vit_filter *f, double *kernel_ms, int64_t *cells, int32_t *launches);

/* ---- P7 MSV / SSV filter (F1) ------------------------------------------ */
typedef struct cmgpu_msv_filter cmgpu_msv_filter;

/* A candidate window of f1_msv_windows: residues start..end (1-based, in the
 * chunk's own coordinates) of chunk `chunk`, with the SSV diagonal score of
 * its first diagonal (src/cm_pipeline.rs:466-471). */
typedef struct cmgpu_f1_window {
    int64_t start, end;
    float score;
    int32_t chunk;
} cmgpu_f1_window;

/* One SSV diagonal as ssv_diagonals returns it (src/cm_pipeline.rs:455-462):
 * target start n, model length, model end k, score. */
typedef struct cmgpu_ssv_diagonal {
    int64_t n, length, k;
    float score;
    int32_t chunk;
} cmgpu_ssv_diagonal;

/* build_msv_filter (src/cm_pipeline.rs:201-340) with max_length = the
 * pipeline's maxW; lmmu / lmlambda are the profile's local MSV Gumbel
 * parameters (P7Profile.evparam).  device < 0: host tables only. */
int cmgpu_msv_filter_build(const cmgpu_p7_profile *p, int32_t max_length, double lmmu, double lmlambda,
                           int device, cmgpu_msv_filter **out);
void cmgpu_msv_filter_free(cmgpu_msv_filter *f);
/* The filter's tables: emission costs rbv[(M+1)*18], bytes5 = {base_b, bias_b,
 * tbm_b, tec_b, tjb_b}, prefix/suffix lengths [M+1], scale_b.  For tests. */
int cmgpu_msv_filter_tables(const cmgpu_msv_filter *f, uint8_t *rbv, int32_t cap, int32_t *n_out,
                            uint8_t *bytes5, float *prefix, float *suffix, float *scale_b);
/* The SSV trigger threshold sc_thresh of ssv_diagonals for F1 = f1. */
int cmgpu_ssv_threshold(const cmgpu_msv_filter *f, double f1, int32_t *thresh);
/* msv_score (src/cm_pipeline.rs:402, wlen == NULL) or msv_score_reconfig
 * (:410, length model of wlen[w] residues) of residues i0..j0 of every
 * window; scored[w] = 0 where the reference returns None (8-bit overflow). */
int cmgpu_msv_score_batch(const cmgpu_msv_filter *f, void *stream, const uint8_t *dsq_all, int64_t dsq_len,
                          const cmgpu_window *wins, int32_t nwin, const int32_t *wlen, float *scores,
                          uint8_t *scored);
/* f1_msv_windows (src/cm_pipeline.rs:842) on every chunk in one call: the
 * chunk's residues are i0..j0 of its window (local position 1 = i0).
 * Windows come back grouped by chunk, each chunk's in the reference's order.
 * CMGPU_EOVERFLOW with the needed count in *n_out when cap is too small. */
int cmgpu_f1_msv_windows(const cmgpu_msv_filter *f, void *stream, const uint8_t *dsq_all, int64_t dsq_len,
                         const cmgpu_window *chunks, int32_t nchunk, double f1, int64_t cmw,
                         cmgpu_f1_window *out, int32_t cap, int32_t *n_out);
/* ssv_diagonals (src/cm_pipeline.rs:521) on every chunk: the raw diagonals
 * before extension and merging (the reference's DUMP_SSV lines). */
int cmgpu_ssv_diagonals(const cmgpu_msv_filter *f, void *stream, const uint8_t *dsq_all, int64_t dsq_len,
                        const cmgpu_window *chunks, int32_t nchunk, double f1, cmgpu_ssv_diagonal *out,
                        int32_t cap, int32_t *n_out);
/* Device time, cells (rows x M, warm-up rows included) and kernel launches
 * of the last scoring or scanning call on this filter. */
int cmgpu_msv_filter_stats(const cmgpu_msv_filter *f, double *kernel_ms, int64_t *cells, int32_t *launches);

/* ---- P7 Forward filter (F3), composition bias (F3b), F1 -> F3b cascade -- */
typedef struct cmgpu_fwd_filter cmgpu_fwd_filter;

/* build_forward_filter (src/cm_pipeline.rs:969) and build_bias_filter
 * (:1683) from the p7 filter profile, its mean match composition compo[4]
 * (P7Profile.compo) and the local Forward exp-tail parameters (evparam
 * lftau, lflambda).  device < 0: host tables only. */
int cmgpu_fwd_filter_build(const cmgpu_p7_profile *p, const float *compo, double ftau, double flambda,
                           int device, cmgpu_fwd_filter **out);
void cmgpu_fwd_filter_free(cmgpu_fwd_filter *f);
/* The profile in natural order, for tests: rfv[(M+1)*18] match odds,
 * tr[(M+1)*8] = tBM, M->M, I->M, D->M (row k: into position k), M->I, I->I,
 * M->D, D->D (row k: out of position k); bias emission odds eo[18*2] and
 * state-1 transitions t1[3].  *m_out = M; cap = rows available (>= M+1). */
int cmgpu_fwd_filter_tables(const cmgpu_fwd_filter *f, float *rfv, float *tr, int32_t cap, int32_t *m_out,
                            float *eo, float *t1);
/* forward_filter_score (src/cm_pipeline.rs:1420; the striped engine) and
 * bias_filter_score (:1722) of residues i0..j0 of every window, in nats;
 * either output may be NULL. */
int cmgpu_fwd_score_batch(const cmgpu_fwd_filter *f, void *stream, const uint8_t *dsq_all, int64_t dsq_len,
                          const cmgpu_window *wins, int32_t nwin, float *fwd_scores, float *bias_scores);

/* The stages and thresholds of one f3_filter_sequence pass
 * (src/cm_pipeline.rs:1863-1887). */
typedef struct cmgpu_f3_config {
    double f1, f1b, f2, f2b, f3, f3b; /* P-value thresholds                  */
    int64_t cmw;                      /* the CM's W (SSV windows split at 2W) */
    int64_t maxw;                     /* do_msv == 0: 2*maxw-residue tiles    */
    int32_t do_msv, do_msvbias, do_vit, do_vitbias, do_fwd, do_fwdbias;
    double lmmu, lmlambda;            /* local MSV Gumbel (F1b)               */
    double lvmu, lvlambda;            /* local Viterbi Gumbel (F2, F2b)       */
} cmgpu_f3_config;

/* F1F3Acct (src/cm_pipeline.rs:1799-1814), summed over the chunks. */
typedef struct cmgpu_f3_acct {
    int64_t n_past_msv, pos_past_msv, n_past_msvbias, pos_past_msvbias;
    int64_t n_past_vit, pos_past_vit, n_past_vitbias, pos_past_vitbias;
    int64_t n_past_fwd, pos_past_fwd, n_past_fwdbias, pos_past_fwdbias;
} cmgpu_f3_acct;

/* f3_filter_sequence (src/cm_pipeline.rs:1863-2164) on every chunk (the
 * chunk's residues are i0..j0 of its window): SSV windows (mf) or tiles,
 * then the F1b MSV-bias (mf), F2 / F2b Viterbi (vf) and F3 / F3b Forward
 * gates, and the merge of the survivors.  Windows come back grouped by
 * chunk in chunk coordinates with the F3b bit score (the reference's wb).
 * mf may be NULL when do_msv and do_msvbias are 0, vf when do_vit is 0.
 * CMGPU_EOVERFLOW with the needed count in *n_out when cap is too small.
 * Device time and launches of the whole pass: cmgpu_fwd_filter_stats. */
int cmgpu_f3_filter(const cmgpu_fwd_filter *ff, const cmgpu_msv_filter *mf, const cmgpu_vit_filter *vf,
                    void *stream, const uint8_t *dsq_all, int64_t dsq_len, const cmgpu_window *chunks,
                    int32_t nchunk, const cmgpu_f3_config *cfg, cmgpu_f1_window *out, int32_t cap,
                    int32_t *n_out, cmgpu_f3_acct *acct);
/* Forward kernels (cmgpu_fwd_filter_set_kernel); both give the same bits.
 * AUTO keeps each lane's segment of the rows in registers where it fits
 * (nq = (M-1)/4+1 <= 32), else in shared memory; SHARED always uses the
 * shared-memory kernel. */
#define CMGPU_FWD_KERNEL_AUTO 0
#define CMGPU_FWD_KERNEL_SHARED 1
int cmgpu_fwd_filter_set_kernel(cmgpu_fwd_filter *f, int kernel);
/* Device time, Forward cells (residues x M) and launches of the last
 * scoring or filtering call on this filter. */
int cmgpu_fwd_filter_stats(const cmgpu_fwd_filter *f, double *kernel_ms, int64_t *cells, int32_t *launches);

/* Exact counts of cells and terms the reference scanner evaluates for a
 * window of length L (host only; used for Gcells/s). */
int cmgpu_count_work(const cmgpu_cm *cm, int semiring, int qdbidx, int32_t L,
                     double *cells, double *terms);

#ifdef __cplusplus
}
#endif
#endif /* CMSCAN_GPU_H */
