/*
 * qdb_oracle.c -- TEST INFRASTRUCTURE ONLY.  CPU restatement of the
 * reference's QDB-banded CYK / Inside window scanner, used as the parity
 * checker for the GPU path (tests, smoke check, and the CPU-baseline leg of
 * bench.py).  Nothing in the product library links or calls this file.
 *
 * It follows, loop for loop, infernox src/cm_nohmm.rs:
 *   generic_scan          :406-763  (rolling decks alpha[2][M][W+1] and
 *                                    alpha_begl[W+1][nbegl][W+1], j outer,
 *                                    v = M-1..1, d inner)
 *   reduce_c_order        :187-242  (integer Inside child order)
 *   report_hits_greedily  :769-812  (+ esl_vec_fnorm :815)
 *   cyk_seq_filter        :855-889  (pad by W-1, merge by end)
 *   final_stage_inside_opt:919-935
 * plus src/cp9.rs ilogsum (:28-75), flogsum (:5391-5413),
 * score_correction_null3 (:6516-6528) and remove_overlaps_greedy (:6544-6574).
 *
 * Two semirings are generated from one macro body, as the reference writes
 * the recursion once over `trait Sr`: f32 with ESL_MAX (CYK) and i32 with
 * wrapping adds and ILogsum (Inside).
 *
 * Build: make -C oracle  (gcc -O2 -ffp-contract=off, no fast-math).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/cmscan_gpu.h"

#define IMPOSSIBLE (-1.0e36f)
#define INFTY 987654321
#define LOGSUM_TBL 23000
#define KP 18
#define ESCW 324

enum { D_ST = 0, MP_ST, ML_ST, MR_ST, IL_ST, IR_ST, S_ST, E_ST, B_ST };
#define BEGL_S 3

/* cmcalibrate's copy of the scanner (src/cm_calibrate.rs:441-780) compares
 * local begins by their bit scores (S::scbits(a) < S::scbits(cand)); the
 * search scanner compares the raw values.  Set for oracle_calib_scan only. */
static int g_calib_begins = 0;

static int32_t g_ilog[LOGSUM_TBL];
static float g_flog[LOGSUM_TBL];
static int g_tables_ready = 0;

static void init_tables(void) {
    if (g_tables_ready) return;
    for (int i = 0; i < LOGSUM_TBL; i++) {
        /* src/cp9.rs:36-41: rint(1000*log2(1+2^(-i/1000))) */
        double v = 1000.0 * log2(1.0 + pow(2.0, -(double)i / 1000.0));
        g_ilog[i] = (int32_t)nearbyint(v);
        /* src/cp9.rs:5396-5398: sreLOG2(1+sreEXP2(-i/1000)) */
        double ex = exp((-(double)i / 1000.0) * 0.69314718);
        double x = 1.0 + ex;
        g_flog[i] = (float)(x > 0.0 ? log(x) * 1.44269504 : -1.0e36);
    }
    g_tables_ready = 1;
}

int oracle_ilogsum_table(int32_t *out, int n) {
    init_tables();
    if (n > LOGSUM_TBL) n = LOGSUM_TBL;
    memcpy(out, g_ilog, sizeof(int32_t) * (size_t)n);
    return n;
}

static inline int32_t ilogsum(int32_t s1, int32_t s2) {
    int32_t mx = s1 > s2 ? s1 : s2;
    if (mx < -INFTY) mx = -INFTY;
    int32_t mn = s1 < s2 ? s1 : s2;
    int32_t diff = mx - mn;
    if (mn <= -INFTY || (int64_t)diff >= LOGSUM_TBL) return mx;
    return mx + g_ilog[diff];
}

int32_t oracle_ilogsum(int32_t a, int32_t b) {
    init_tables();
    return ilogsum(a, b);
}

static inline float flogsum(float s1, float s2) {
    float mx = s1 > s2 ? s1 : s2; /* f32::max; no NaNs arise here */
    float mn = s1 < s2 ? s1 : s2;
    if (mn == -INFINITY || (mx - mn) >= 23.0f) return mx;
    return mx + g_flog[(size_t)((mx - mn) * 1000.0f)];
}

static inline int32_t wadd(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }
static inline float fmax_ge(float a, float b) { return a >= b ? a : b; }
static inline int32_t imax_ge(int32_t a, int32_t b) { return a >= b ? a : b; }
static inline int not_impossible(float x) { return x > IMPOSSIBLE + 1.0f; }
static inline float scorify(int32_t sc) { return sc == -INFTY ? IMPOSSIBLE : (float)((double)sc / 1000.0); }

static inline int state_delta(int st) {
    return st == MP_ST ? 2 : (st == ML_ST || st == MR_ST || st == IL_ST || st == IR_ST) ? 1 : 0;
}
static inline int right_delta(int st) { return (st == MP_ST || st == MR_ST || st == IR_ST); }
static inline int emitmode(int st) { /* 0 none, 1 left, 2 right, 3 pair */
    if (st == ML_ST || st == IL_ST) return 1;
    if (st == MR_ST || st == IR_ST) return 2;
    if (st == MP_ST) return 3;
    return 0;
}

/* ---- hit list helpers ---------------------------------------------------- */
typedef struct {
    cmgpu_hit *v;
    int n, cap;
} hitvec;

static void hv_push(hitvec *h, int32_t i, int32_t j, float sc, float bias) {
    if (h->n == h->cap) {
        h->cap = h->cap ? h->cap * 2 : 64;
        h->v = (cmgpu_hit *)realloc(h->v, sizeof(cmgpu_hit) * (size_t)h->cap);
    }
    h->v[h->n].i = i;
    h->v[h->n].j = j;
    h->v[h->n].score = sc;
    h->v[h->n].bias = bias;
    h->n++;
}

/* esl_vec_fnorm (src/cm_nohmm.rs:815-827) */
static void vec_fnorm(float *v, int n) {
    float sum = 0.0f;
    for (int i = 0; i < n; i++) sum += v[i];
    if (sum > 0.0f)
        for (int i = 0; i < n; i++) v[i] /= sum;
    else
        for (int i = 0; i < n; i++) v[i] = 1.0f / (float)n;
}

static inline double sre_log2d(double x) { return x > 0.0 ? log(x) * 1.44269504 : -1.0e36; }

/* score_correction_null3 (src/cp9.rs:6516-6528) */
static float null3_correction(const float *null0, const float *comp, int len, float omega) {
    float score = 0.0f;
    for (int a = 0; a < 4; a++) {
        double term = sre_log2d((double)(comp[a] / null0[a])) * (double)comp[a] * (double)len;
        score = (float)((double)score + term);
    }
    score = (float)((double)score + sre_log2d((double)omega));
    return flogsum(0.0f, score);
}

/* Candidate sink: every (j, d, bits) with bits >= cutoff, in scan order.  It
 * is the intermediate the GPU path emits, exposed for cell-level checks. */
typedef struct {
    int32_t *j, *d;
    float *sc;
    int n, cap;
} candvec;

static void cv_push(candvec *c, int32_t j, int32_t d, float sc) {
    if (!c) return;
    if (c->n == c->cap) {
        c->cap = c->cap ? c->cap * 2 : 256;
        c->j = (int32_t *)realloc(c->j, sizeof(int32_t) * (size_t)c->cap);
        c->d = (int32_t *)realloc(c->d, sizeof(int32_t) * (size_t)c->cap);
        c->sc = (float *)realloc(c->sc, sizeof(float) * (size_t)c->cap);
    }
    c->j[c->n] = j;
    c->d[c->n] = d;
    c->sc[c->n] = sc;
    c->n++;
}

/* report_hits_greedily (src/cm_nohmm.rs:769-812).  act holds cumulative
 * residue counts in a ring of W+1 as the reference keeps them. */
static void report_hits_greedily(const cmgpu_cm *cm, int32_t j, int32_t dmin, int32_t dmax,
                                 const float *bestsc, int w, const double (*act)[4], int32_t i0,
                                 float cutoff, hitvec *out) {
    if (dmin > dmax) return;
    float max_reported = IMPOSSIBLE;
    int32_t dlo = dmin > 1 ? dmin : 1;
    for (int32_t d = dlo; d <= dmax; d++) {
        int32_t i = j - d + 1;
        float hit_sc = bestsc[d];
        float bias = 0.0f;
        if (hit_sc > max_reported && hit_sc >= cutoff && not_impossible(hit_sc)) {
            int do_report = 1;
            if (act) {
                int ip = i - i0 + 1, jp = j - i0 + 1;
                float comp[4];
                for (int a = 0; a < 4; a++)
                    comp[a] = (float)(act[jp % (w + 1)][a] - act[(ip - 1) % (w + 1)][a]);
                vec_fnorm(comp, 4);
                float corr = null3_correction(cm->null, comp, d, cm->n3_omega);
                hit_sc -= corr;
                bias = corr;
                do_report = hit_sc > max_reported && hit_sc >= cutoff;
            }
            if (do_report) {
                hv_push(out, i, j, hit_sc, bias);
                max_reported = hit_sc;
            }
        }
    }
}

/* remove_overlaps_greedy (src/cp9.rs:6544-6574): stable sort by score desc,
 * start asc; a hit overlapping a kept higher-ranked one is removed. */
static int cmp_hit(const void *a, const void *b) {
    const cmgpu_hit *x = (const cmgpu_hit *)a, *y = (const cmgpu_hit *)b;
    if (x->score > y->score) return -1;
    if (x->score < y->score) return 1;
    if (x->i < y->i) return -1;
    if (x->i > y->i) return 1;
    return 0;
}

static void stable_sort_hits(cmgpu_hit *h, int n) {
    /* insertion-merge via index tiebreak keeps Rust's stable sort order */
    typedef struct {
        cmgpu_hit h;
        int k;
    } tagged;
    tagged *t = (tagged *)malloc(sizeof(tagged) * (size_t)(n ? n : 1));
    for (int k = 0; k < n; k++) {
        t[k].h = h[k];
        t[k].k = k;
    }
    /* simple stable merge sort */
    tagged *tmp = (tagged *)malloc(sizeof(tagged) * (size_t)(n ? n : 1));
    for (int width = 1; width < n; width *= 2) {
        for (int lo = 0; lo < n; lo += 2 * width) {
            int mid = lo + width < n ? lo + width : n;
            int hi = lo + 2 * width < n ? lo + 2 * width : n;
            int a = lo, b = mid, o = lo;
            while (a < mid && b < hi) {
                int c = cmp_hit(&t[a].h, &t[b].h);
                if (c <= 0)
                    tmp[o++] = t[a++];
                else
                    tmp[o++] = t[b++];
            }
            while (a < mid) tmp[o++] = t[a++];
            while (b < hi) tmp[o++] = t[b++];
        }
        memcpy(t, tmp, sizeof(tagged) * (size_t)n);
    }
    for (int k = 0; k < n; k++) h[k] = t[k].h;
    free(t);
    free(tmp);
}

static void remove_overlaps_greedy(hitvec *h) {
    int n = h->n;
    stable_sort_hits(h->v, n);
    char *removed = (char *)calloc((size_t)(n ? n : 1), 1);
    for (int i = 0; i < n; i++) {
        if (removed[i]) continue;
        int32_t si = h->v[i].i, ei = h->v[i].j;
        for (int j = i + 1; j < n; j++) {
            if (removed[j]) continue;
            int32_t sj = h->v[j].i, ej = h->v[j].j;
            if (!(ej < si) && !(ei < sj)) removed[j] = 1;
        }
    }
    int o = 0;
    for (int i = 0; i < n; i++)
        if (!removed[i]) h->v[o++] = h->v[i];
    h->n = o;
    free(removed);
}

/* c-order reduction (src/cm_nohmm.rs:187-242) */
#define REDUCE_C_ORDER(T, COMB, cnum, terms, init, out)                     \
    do {                                                                    \
        T s_;                                                               \
        switch (cnum) {                                                     \
        case 1: s_ = COMB(init, terms[0]); break;                           \
        case 2: s_ = COMB(COMB(terms[1], init), terms[0]); break;           \
        case 3: s_ = COMB(COMB(COMB(terms[2], terms[1]), init), terms[0]); break; \
        case 4:                                                             \
            s_ = COMB(terms[3], terms[2]);                                  \
            s_ = COMB(s_, init);                                            \
            s_ = COMB(s_, terms[1]);                                        \
            s_ = COMB(s_, terms[0]);                                        \
            break;                                                          \
        case 5:                                                             \
            s_ = COMB(terms[4], terms[3]);                                  \
            s_ = COMB(s_, init);                                            \
            s_ = COMB(s_, terms[1]);                                        \
            s_ = COMB(s_, terms[2]);                                        \
            s_ = COMB(s_, terms[0]);                                        \
            break;                                                          \
        case 6:                                                             \
            s_ = COMB(terms[5], init);                                      \
            s_ = COMB(s_, terms[4]);                                        \
            s_ = COMB(s_, terms[3]);                                        \
            s_ = COMB(s_, terms[2]);                                        \
            s_ = COMB(s_, terms[1]);                                        \
            s_ = COMB(s_, terms[0]);                                        \
            break;                                                          \
        default:                                                            \
            s_ = init;                                                      \
            for (int q_ = 0; q_ < (cnum); q_++) s_ = COMB(s_, terms[q_]);   \
        }                                                                   \
        out = s_;                                                           \
    } while (0)

typedef struct {
    double cells, terms;
} workcount;

/* The scanner body for one semiring.  T = cell type; ZERO = -inf sentinel;
 * COMB = child combine; VMAX = Viterbi max; ADDV = add; SCBITS = to bits;
 * POSSIBLE = begin gate; TSC/OESC/ENDSC/BEGINSC/ELSELF = score tables. */
#define DEFINE_SCAN(NAME, T, ZERO, COMB, VMAX, ADDV, SCBITS, POSSIBLE, TSC, OESC, ENDSC, BEGINSC, ELSELF) \
static void NAME(const cmgpu_cm *cm, const uint8_t *dsq, int32_t i0, int32_t j0, float cutoff,          \
                 int do_null3, int qdbidx, hitvec *out, candvec *cands, workcount *wc) {               \
    const int M = cm->M;                                                                                \
    const int local = (cm->flags & (1u << 10)) != 0;                                                    \
    const int32_t smx_w = cm->W;                                                                        \
    int32_t L = j0 - i0 + 1;                                                                            \
    int w = smx_w > L ? L : smx_w;                                                                      \
    const int32_t *dmin, *dmax;                                                                         \
    int32_t *fmin = NULL, *fmax = NULL;                                                                 \
    if (qdbidx == CMGPU_NOQDB) {                                                                        \
        fmin = (int32_t *)calloc((size_t)M, sizeof(int32_t));                                           \
        fmax = (int32_t *)malloc(sizeof(int32_t) * (size_t)M);                                          \
        for (int v = 0; v < M; v++) fmax[v] = smx_w;                                                    \
        dmin = fmin;                                                                                    \
        dmax = fmax;                                                                                    \
    } else if (qdbidx == CMGPU_QDB1) {                                                                  \
        dmin = cm->dmin1;                                                                               \
        dmax = cm->dmax1;                                                                               \
    } else {                                                                                            \
        dmin = cm->dmin2;                                                                               \
        dmax = cm->dmax2;                                                                               \
    }                                                                                                   \
    int32_t *dn_v = (int32_t *)malloc(sizeof(int32_t) * (size_t)M);                                     \
    int32_t *dxcap_v = (int32_t *)malloc(sizeof(int32_t) * (size_t)M);                                  \
    for (int v = 0; v < M; v++) {                                                                       \
        int32_t base = cm->sttype[v] == MP_ST ? 2 : 1;                                                  \
        int32_t dn = dmin[v] > base ? dmin[v] : base;                                                   \
        if (dn > smx_w) dn = smx_w;                                                                     \
        dn_v[v] = dn;                                                                                   \
        dxcap_v[v] = dmax[v] < smx_w ? dmax[v] : smx_w;                                                 \
    }                                                                                                   \
    int *begl_idx = (int *)malloc(sizeof(int) * (size_t)M);                                             \
    int nbegl = 0;                                                                                      \
    for (int v = 0; v < M; v++) begl_idx[v] = cm->stid[v] == BEGL_S ? nbegl++ : -1;                     \
    const size_t W1 = (size_t)w + 1;                                                                    \
    T *el_sca = (T *)malloc(sizeof(T) * W1);                                                            \
    el_sca[0] = (T)0;                                                                                   \
    for (size_t d = 1; d <= (size_t)w; d++) el_sca[d] = ADDV(el_sca[d - 1], ELSELF);                    \
    T *init_sc = (T *)malloc(sizeof(T) * (size_t)M * W1);                                               \
    for (int v = 0; v < M; v++) {                                                                       \
        T es = ENDSC[v];                                                                                \
        int ok = not_impossible(SCBITS(es));                                                            \
        for (size_t d = 0; d <= (size_t)w; d++) init_sc[(size_t)v * W1 + d] = ok ? ADDV(el_sca[d], es) : ZERO; \
    }                                                                                                   \
    T *alpha = (T *)malloc(sizeof(T) * 2 * (size_t)M * W1);                                             \
    for (size_t k = 0; k < 2 * (size_t)M * W1; k++) alpha[k] = ZERO;                                    \
    size_t nb = (size_t)(nbegl ? nbegl : 1);                                                            \
    T *abegl = (T *)malloc(sizeof(T) * W1 * nb * W1);                                                   \
    for (size_t k = 0; k < W1 * nb * W1; k++) abegl[k] = ZERO;                                          \
    /* cm_scan_mx_Initialize: d = 0 base cases, ESL_MAX for S/D/BEGL */                                 \
    for (int v = M - 1; v >= 0; v--) {                                                                  \
        int st = cm->sttype[v];                                                                         \
        if (cm->stid[v] != BEGL_S) {                                                                    \
            if (st == E_ST) {                                                                           \
                alpha[(0 * (size_t)M + v) * W1] = (T)0;                                                 \
                alpha[(1 * (size_t)M + v) * W1] = (T)0;                                                 \
            } else if (st == S_ST || st == D_ST) {                                                      \
                int y = cm->cfirst[v];                                                                  \
                T a0 = ENDSC[v];                                                                        \
                for (int yo = 0; yo < cm->cnum[v]; yo++)                                                \
                    a0 = VMAX(a0, ADDV(alpha[(0 * (size_t)M + y + yo) * W1], TSC[v * 6 + yo]));         \
                a0 = VMAX(a0, ZERO);                                                                    \
                alpha[(0 * (size_t)M + v) * W1] = a0;                                                   \
                alpha[(1 * (size_t)M + v) * W1] = a0;                                                   \
            } else if (st == B_ST) {                                                                    \
                int wl = cm->cfirst[v], y = cm->cnum[v];                                                \
                T a0 = ADDV(abegl[((size_t)0 * nb + begl_idx[wl]) * W1], alpha[(0 * (size_t)M + y) * W1]); \
                alpha[(0 * (size_t)M + v) * W1] = a0;                                                   \
                alpha[(1 * (size_t)M + v) * W1] = a0;                                                   \
            } else {                                                                                    \
                alpha[(1 * (size_t)M + v) * W1] = alpha[(0 * (size_t)M + v) * W1];                      \
            }                                                                                           \
        } else {                                                                                        \
            int bi = begl_idx[v], y = cm->cfirst[v];                                                    \
            T a0 = ENDSC[v];                                                                            \
            for (int yo = 0; yo < cm->cnum[v]; yo++)                                                    \
                a0 = VMAX(a0, ADDV(alpha[(0 * (size_t)M + y + yo) * W1], TSC[v * 6 + yo]));             \
            a0 = VMAX(a0, ZERO);                                                                        \
            for (size_t jj = 0; jj <= (size_t)w; jj++) abegl[(jj * nb + bi) * W1] = a0;                 \
        }                                                                                               \
    }                                                                                                   \
    double(*act)[4] = NULL;                                                                             \
    if (do_null3) act = (double(*)[4])calloc(W1, sizeof(double[4]));                                    \
    size_t *jp_wa = (size_t *)malloc(sizeof(size_t) * W1);                                              \
    T *sc_v = (T *)malloc(sizeof(T) * W1);                                                              \
    float *bestsc = (float *)malloc(sizeof(float) * W1);                                                \
    for (size_t d = 0; d <= (size_t)w; d++) bestsc[d] = IMPOSSIBLE;                                     \
    hitvec tmp = {0, 0, 0};                                                                             \
    for (int32_t j = i0; j <= j0; j++) {                                                                \
        size_t jp_g = (size_t)(j - i0 + 1);                                                             \
        size_t cur = (size_t)(j & 1), prv = (size_t)((j - 1) & 1);                                      \
        int32_t jrow = (int32_t)(jp_g < (size_t)w ? jp_g : (size_t)w);                                  \
        for (size_t d = 0; d <= (size_t)w; d++) {                                                       \
            int64_t r = ((int64_t)j - (int64_t)d) % (int64_t)W1;                                        \
            if (r < 0) r += (int64_t)W1;                                                                \
            jp_wa[d] = (size_t)r;                                                                       \
        }                                                                                               \
        if (act) {                                                                                      \
            size_t src = (jp_g - 1) % W1, dst = jp_g % W1;                                              \
            memcpy(act[dst], act[src], sizeof(double[4]));                                              \
            uint8_t dj = dsq[j];                                                                        \
            if (dj < 4) act[dst][dj] += 1.0;                                                            \
        }                                                                                               \
        for (int v = M - 1; v >= 1; v--) {                                                              \
            int st = cm->sttype[v];                                                                     \
            if (st == E_ST) continue;                                                                   \
            int sd = state_delta(st), em = emitmode(st);                                                \
            size_t jp_v = cm->stid[v] == BEGL_S ? (size_t)(((int64_t)j % (int64_t)W1 + (int64_t)W1) % (int64_t)W1) : cur; \
            size_t jp_y = right_delta(st) ? prv : cur;                                                  \
            int32_t dn = dn_v[v];                                                                       \
            int32_t dx = jrow < dxcap_v[v] ? jrow : dxcap_v[v];                                         \
            const T *esc_v = &OESC[(size_t)v * ESCW];                                                   \
            T esc_j = (st == IR_ST || st == MR_ST) ? esc_v[dsq[j]] : ZERO;                              \
            if (st == B_ST) {                                                                           \
                int wl = cm->cfirst[v], y = cm->cnum[v], bi = begl_idx[wl];                             \
                int32_t dn_y = dmin[y] < smx_w ? dmin[y] : smx_w, dx_y = dmax[y] < smx_w ? dmax[y] : smx_w; \
                int32_t dn_w = dmin[wl] < smx_w ? dmin[wl] : smx_w, dx_w = dmax[wl] < smx_w ? dmax[wl] : smx_w; \
                for (int32_t d = dn; d <= dx; d++) {                                                    \
                    int32_t kmin = dn_y > d - dx_w ? dn_y : d - dx_w;                                   \
                    if (kmin < 0) kmin = 0;                                                             \
                    int32_t kmax = dx_y < d - dn_w ? dx_y : d - dn_w;                                   \
                    T sc = init_sc[(size_t)v * W1 + (size_t)(d - sd)];                                  \
                    for (int32_t kk = kmin; kk <= kmax; kk++) {                                         \
                        T left = abegl[(jp_wa[kk] * nb + bi) * W1 + (size_t)(d - kk)];                   \
                        T right = alpha[(jp_y * (size_t)M + y) * W1 + (size_t)kk];                      \
                        sc = COMB(sc, ADDV(left, right));                                               \
                    }                                                                                   \
                    if (wc) { wc->cells += 1; wc->terms += (double)(kmax >= kmin ? kmax - kmin + 1 : 0); } \
                    alpha[(jp_v * (size_t)M + v) * W1 + (size_t)d] = sc;                                \
                }                                                                                       \
            } else if (cm->stid[v] == BEGL_S) {                                                         \
                int y = cm->cfirst[v], bi = begl_idx[v];                                                \
                for (int32_t d = dn; d <= dx; d++) {                                                    \
                    T sc = init_sc[(size_t)v * W1 + (size_t)(d - sd)];                                  \
                    for (int yo = 0; yo < cm->cnum[v]; yo++)                                            \
                        sc = COMB(sc, ADDV(alpha[(jp_y * (size_t)M + y + yo) * W1 + (size_t)(d - sd)], TSC[v * 6 + yo])); \
                    if (wc) { wc->cells += 1; wc->terms += cm->cnum[v]; }                               \
                    abegl[(jp_v * nb + bi) * W1 + (size_t)d] = sc;                                      \
                }                                                                                       \
            } else if (st == IL_ST || st == IR_ST) {                                                    \
                int y = cm->cfirst[v], cnum = cm->cnum[v];                                              \
                int32_t i = j - dn + 1, dp_y = dn - sd;                                                 \
                for (int32_t d = dn; d <= dx; d++) {                                                    \
                    T terms[6];                                                                         \
                    for (int yo = 0; yo < cnum; yo++)                                                   \
                        terms[yo] = ADDV(alpha[(jp_y * (size_t)M + y + yo) * W1 + (size_t)dp_y], TSC[v * 6 + yo]); \
                    T sc;                                                                               \
                    REDUCE_C_ORDER(T, COMB, cnum, terms, init_sc[(size_t)v * W1 + (size_t)dp_y], sc);   \
                    if (em == 1) { sc = ADDV(sc, esc_v[dsq[i]]); i--; }                                 \
                    else if (em == 2) sc = ADDV(sc, esc_j);                                             \
                    if (wc) { wc->cells += 1; wc->terms += cnum; }                                      \
                    alpha[(jp_v * (size_t)M + v) * W1 + (size_t)d] = sc;                                \
                    dp_y++;                                                                             \
                }                                                                                       \
            } else {                                                                                    \
                int y = cm->cfirst[v], cnum = cm->cnum[v];                                              \
                int32_t dp_y = dn - sd;                                                                 \
                for (int32_t d = dn; d <= dx; d++) {                                                    \
                    T terms[6];                                                                         \
                    for (int yo = 0; yo < cnum; yo++)                                                   \
                        terms[yo] = ADDV(alpha[(jp_y * (size_t)M + y + yo) * W1 + (size_t)dp_y], TSC[v * 6 + yo]); \
                    REDUCE_C_ORDER(T, COMB, cnum, terms, init_sc[(size_t)v * W1 + (size_t)dp_y], sc_v[d]); \
                    if (wc) { wc->cells += 1; wc->terms += cnum; }                                      \
                    dp_y++;                                                                             \
                }                                                                                       \
                T *dst = &alpha[(jp_v * (size_t)M + v) * W1];                                           \
                if (em == 1) {                                                                          \
                    int32_t i = j - dn + 1;                                                             \
                    for (int32_t d = dn; d <= dx; d++) { dst[d] = ADDV(sc_v[d], esc_v[dsq[i]]); i--; }   \
                } else if (em == 0) {                                                                   \
                    for (int32_t d = dn; d <= dx; d++) dst[d] = sc_v[d];                                \
                } else if (em == 2) {                                                                   \
                    for (int32_t d = dn; d <= dx; d++) dst[d] = ADDV(sc_v[d], esc_j);                   \
                } else {                                                                                \
                    int32_t i = j - dn + 1;                                                             \
                    for (int32_t d = dn; d <= dx; d++) {                                                \
                        dst[d] = ADDV(sc_v[d], esc_v[(size_t)dsq[i] * KP + dsq[j]]);                     \
                        i--;                                                                            \
                    }                                                                                   \
                }                                                                                       \
            }                                                                                           \
        }                                                                                               \
        /* ROOT_S: plain root transitions, then local begins (MAX in both semirings) */                \
        int32_t dn0 = dn_v[0];                                                                          \
        int32_t dx0 = jrow < dxcap_v[0] ? jrow : dxcap_v[0];                                            \
        int y0 = cm->cfirst[0];                                                                         \
        T *a0row = &alpha[(cur * (size_t)M + 0) * W1];                                                  \
        for (int32_t d = dn0; d <= dx0; d++) {                                                          \
            T a = COMB(ZERO, ADDV(alpha[(cur * (size_t)M + y0) * W1 + (size_t)d], TSC[0]));             \
            for (int yo = 1; yo < cm->cnum[0]; yo++)                                                    \
                a = COMB(a, ADDV(alpha[(cur * (size_t)M + y0 + yo) * W1 + (size_t)d], TSC[yo]));        \
            if (wc) { wc->cells += 1; wc->terms += cm->cnum[0]; }                                       \
            a0row[d] = a;                                                                               \
        }                                                                                               \
        if (local) {                                                                                    \
            for (int y = 1; y < M; y++) {                                                               \
                if (!(POSSIBLE(BEGINSC[y]))) continue;                                                  \
                int32_t dn = dn0 > dn_v[y] ? dn0 : dn_v[y];                                             \
                int32_t dxy = jrow < dxcap_v[y] ? jrow : dxcap_v[y];                                    \
                int32_t dx = dx0 < dxy ? dx0 : dxy;                                                     \
                if (cm->stid[y] == BEGL_S) {                                                            \
                    size_t jpy = jp_wa[0];                                                              \
                    int bi = begl_idx[y];                                                               \
                    for (int32_t d = dn; d <= dx; d++) {                                                \
                        T cand = ADDV(abegl[(jpy * nb + bi) * W1 + (size_t)d], BEGINSC[y]);             \
                        if (g_calib_begins ? SCBITS(a0row[d]) < SCBITS(cand) : a0row[d] < cand)         \
                            a0row[d] = cand;                                                            \
                        if (wc) wc->terms += 1;                                                         \
                    }                                                                                   \
                } else {                                                                                \
                    for (int32_t d = dn; d <= dx; d++) {                                                \
                        T cand = ADDV(alpha[(cur * (size_t)M + y) * W1 + (size_t)d], BEGINSC[y]);       \
                        if (g_calib_begins ? SCBITS(a0row[d]) < SCBITS(cand) : a0row[d] < cand)         \
                            a0row[d] = cand;                                                            \
                        if (wc) wc->terms += 1;                                                         \
                    }                                                                                   \
                }                                                                                       \
            }                                                                                           \
        }                                                                                               \
        for (int32_t d = dn0; d <= dx0; d++) {                                                          \
            bestsc[d] = SCBITS(a0row[d]);                                                               \
            if (cands && d >= 1 && bestsc[d] >= cutoff && not_impossible(bestsc[d])) cv_push(cands, j, d, bestsc[d]); \
        }                                                                                               \
        report_hits_greedily(cm, j, dn0, dx0, bestsc, w, (const double(*)[4])act, i0, cutoff, &tmp);  \
    }                                                                                                   \
    remove_overlaps_greedy(&tmp);                                                                       \
    for (int k = 0; k < tmp.n; k++) hv_push(out, tmp.v[k].i, tmp.v[k].j, tmp.v[k].score, tmp.v[k].bias); \
    free(tmp.v);                                                                                        \
    free(fmin); free(fmax); free(dn_v); free(dxcap_v); free(begl_idx); free(el_sca); free(init_sc);     \
    free(alpha); free(abegl); free(act); free(jp_wa); free(sc_v); free(bestsc);                         \
}

#define F_ZERO IMPOSSIBLE
#define F_COMB(a, b) fmax_ge((a), (b))
#define F_ADD(a, b) ((a) + (b))
#define F_BITS(a) (a)
#define F_POSSIBLE(a) not_impossible(a)
#define I_ZERO (-INFTY)
#define I_COMB(a, b) ilogsum((a), (b))
#define I_ADD(a, b) wadd((a), (b))
#define I_BITS(a) scorify(a)
#define I_POSSIBLE(a) ((a) != -INFTY)

DEFINE_SCAN(scan_cyk, float, F_ZERO, F_COMB, fmax_ge, F_ADD, F_BITS, F_POSSIBLE, cm->tsc, cm->oesc, cm->endsc,
            cm->beginsc, cm->el_selfsc)
DEFINE_SCAN(scan_inside, int32_t, I_ZERO, I_COMB, imax_ge, I_ADD, I_BITS, I_POSSIBLE, cm->itsc, cm->ioesc,
            cm->iendsc, cm->ibeginsc, cm->iel_selfsc)

/* ---- exported oracle entry points ---------------------------------------- */

/* generic_scan: hits after overlap removal; optional raw candidates. */
int oracle_qdb_scan(const cmgpu_cm *cm, int semiring, int qdbidx, const uint8_t *dsq, int32_t i0, int32_t j0,
                    float cutoff, int do_null3, cmgpu_hit *hits, int32_t cap, int32_t *n_out, int32_t *cand_j,
                    int32_t *cand_d, float *cand_sc, int32_t cand_cap, int32_t *n_cand, double *cells,
                    double *terms) {
    init_tables();
    hitvec out = {0, 0, 0};
    candvec cv = {0, 0, 0, 0, 0};
    workcount wc = {0.0, 0.0};
    if (j0 < i0) {
        *n_out = 0;
        if (n_cand) *n_cand = 0;
        return 0;
    }
    if (semiring == CMGPU_CYK_F32)
        scan_cyk(cm, dsq, i0, j0, cutoff, do_null3, qdbidx, &out, n_cand ? &cv : NULL, &wc);
    else
        scan_inside(cm, dsq, i0, j0, cutoff, do_null3, qdbidx, &out, n_cand ? &cv : NULL, &wc);
    int rc = 0;
    *n_out = out.n;
    if (out.n > cap)
        rc = CMGPU_EOVERFLOW;
    else if (out.n)
        memcpy(hits, out.v, sizeof(cmgpu_hit) * (size_t)out.n);
    if (n_cand) {
        *n_cand = cv.n;
        int m = cv.n < cand_cap ? cv.n : cand_cap;
        if (m > 0) {
            memcpy(cand_j, cv.j, sizeof(int32_t) * (size_t)m);
            memcpy(cand_d, cv.d, sizeof(int32_t) * (size_t)m);
            memcpy(cand_sc, cv.sc, sizeof(float) * (size_t)m);
        }
        if (cv.n > cand_cap) rc = CMGPU_EOVERFLOW;
    }
    if (cells) *cells = wc.cells;
    if (terms) *terms = wc.terms;
    free(out.v);
    free(cv.j);
    free(cv.d);
    free(cv.sc);
    return rc;
}

/* collect_scores's scan (src/cm_calibrate.rs:953-989): cutoff -inf and
 * local begins compared in bits; the kept hits of the window. */
int oracle_calib_scan(const cmgpu_cm *cm, int semiring, int qdbidx, const uint8_t *dsq, int32_t i0, int32_t j0,
                      int do_null3, cmgpu_hit *hits, int32_t cap, int32_t *n_out, double *cells) {
    g_calib_begins = 1;
    int rc = oracle_qdb_scan(cm, semiring, qdbidx, dsq, i0, j0, -INFINITY, do_null3, hits, cap, n_out, NULL, NULL,
                             NULL, 0, NULL, cells, NULL);
    g_calib_begins = 0;
    return rc;
}

typedef struct {
    int32_t a, b;
} envp;

static int cmp_env(const void *x, const void *y) {
    const envp *p = (const envp *)x, *q = (const envp *)y;
    if (p->b != q->b) return p->b < q->b ? -1 : 1;
    if (p->a != q->a) return p->a < q->a ? -1 : 1;
    return 0;
}

/* cyk_seq_filter (src/cm_nohmm.rs:855-889) */
int oracle_cyk_seq_filter(const cmgpu_cm *cm, const uint8_t *dsq, int32_t n, float cutoff, int do_null3,
                          cmgpu_envelope *envs, int32_t cap, int32_t *n_out) {
    init_tables();
    hitvec out = {0, 0, 0};
    scan_cyk(cm, dsq, 1, n, cutoff, do_null3, CMGPU_QDB1, &out, NULL, NULL);
    envp *pad = (envp *)malloc(sizeof(envp) * (size_t)(out.n ? out.n : 1));
    for (int k = 0; k < out.n; k++) {
        int32_t iw = out.v[k].j - (cm->W - 1);
        if (iw < 1) iw = 1;
        int32_t jw = out.v[k].i + (cm->W - 1);
        if (jw > n) jw = n;
        pad[k].a = iw;
        pad[k].b = jw;
    }
    qsort(pad, (size_t)out.n, sizeof(envp), cmp_env);
    int ne = 0, rc = 0;
    int h = 0;
    while (h < out.n) {
        int32_t iw = pad[h].a, jw = pad[h].b;
        while (h + 1 < out.n) {
            if (pad[h + 1].a <= jw) {
                h++;
                if (pad[h].b > jw) jw = pad[h].b;
            } else
                break;
        }
        if (ne < cap) {
            envs[ne].start = iw;
            envs[ne].end = jw;
        }
        ne++;
        h++;
    }
    if (ne > cap) rc = CMGPU_EOVERFLOW;
    *n_out = ne;
    free(pad);
    free(out.v);
    return rc;
}

/* final_stage_inside_opt (src/cm_nohmm.rs:919-935) */
int oracle_final_stage_inside_opt(const cmgpu_cm *cm, const uint8_t *dsq, const cmgpu_envelope *envs, int32_t nenv,
                                  float cutoff, int do_null3, int nonbanded, cmgpu_hit *hits, int32_t cap,
                                  int32_t *n_out) {
    init_tables();
    hitvec out = {0, 0, 0};
    for (int k = 0; k < nenv; k++)
        scan_inside(cm, dsq, envs[k].start, envs[k].end, cutoff, do_null3, nonbanded ? CMGPU_NOQDB : CMGPU_QDB2,
                    &out, NULL, NULL);
    *n_out = out.n;
    int rc = 0;
    if (out.n > cap)
        rc = CMGPU_EOVERFLOW;
    else if (out.n)
        memcpy(hits, out.v, sizeof(cmgpu_hit) * (size_t)out.n);
    free(out.v);
    return rc;
}

/* shared with hb_oracle.c */
float oracle_flogsum(float a, float b) {
    init_tables();
    return flogsum(a, b);
}

float oracle_null3(const float *null0, const float *comp, int len, float omega) {
    init_tables();
    return null3_correction(null0, comp, len, omega);
}
