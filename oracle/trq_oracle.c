/*
 * trq_oracle.c -- TEST INFRASTRUCTURE ONLY.  CPU restatement of the
 * reference's QDB / non-banded truncated scanner (src/cm_dpsearch_trunc.rs):
 *   generic_tr_scan<f32|i32>  :1800-2316  (ref_tr_cyk_scan :207 and
 *                                          ref_itr_inside_scan :226)
 * loop for loop: rolling planes J/L/R/T [2][M][W+1] and BEGL decks
 * [W+1][nbegl][W+1] for J/L/R, all initialised once; the d = 0 base cells
 * set once; local-end scores by repeated addition; `comb` = ESL_MAX (>=) for
 * CYK and ILogsum for Inside, `max2` = ESL_MAX in both; the ROOT row kept
 * across columns (never reset); the greedy truncated report with
 * allow_truncation and null3, then overlap removal.  Two semirings from one
 * macro body, as the reference writes the scan once over `trait TrSr`.
 * The parity checker for the GPU kernel of this scanner.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/cmscan_gpu.h"

#define IMPOSSIBLE (-1.0e36f)
#define INFTY 987654321
#define KP 18
#define ESCW 324

enum { D_ST = 0, MP_ST, ML_ST, MR_ST, IL_ST, IR_ST, S_ST, E_ST, B_ST };
enum { TRMODE_T = 0, TRMODE_R = 1, TRMODE_L = 2, TRMODE_J = 3, TRMODE_UNKNOWN = 4 };
#define BEGL_S 3
#define END_E 19

float oracle_flogsum(float a, float b);
float oracle_null3(const float *null0, const float *comp, int len, float omega);
int32_t oracle_ilogsum(int32_t a, int32_t b);

static inline int sdelta(int st) {
    return st == MP_ST ? 2 : (st == ML_ST || st == MR_ST || st == IL_ST || st == IR_ST) ? 1 : 0;
}
static inline int srdelta(int st) { return (st == MP_ST || st == MR_ST || st == IR_ST); }
static inline int emitmode(int st) {
    if (st == ML_ST || st == IL_ST) return 1;
    if (st == MR_ST || st == IR_ST) return 2;
    if (st == MP_ST) return 3;
    return 0;
}

typedef struct {
    int32_t i, j;
    float score, bias;
    int32_t mode, root;
} trhit;

/* f32 semiring */
static inline float f_comb(float a, float b) { return a >= b ? a : b; }
static inline float f_max2(float a, float b) { return a >= b ? a : b; }
static inline float f_add(float a, float b) { return a + b; }
static inline double f_ord(float a) { return (double)a; }
static inline float f_bits(float a) { return a; }
static inline int f_isimp(float a) { return !(a > IMPOSSIBLE + 1.0f); }
/* i32 semiring */
static inline int32_t i_comb(int32_t a, int32_t b) { return oracle_ilogsum(a, b); }
static inline int32_t i_max2(int32_t a, int32_t b) { return a >= b ? a : b; }
static inline int32_t i_add(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }
static inline double i_ord(int32_t a) { return (double)a; }
static inline float i_bits(int32_t a) { return a == -INFTY ? IMPOSSIBLE : (float)((double)a / 1000.0); }
static inline int i_isimp(int32_t a) { return a == -INFTY; }

static int allow_trunc(int pass_idx, int local, const int32_t *lpos, const int32_t *rpos, int clen, int64_t start,
                       int64_t stop, int64_t i0, int64_t j0, int mode, int b) {
    if (pass_idx == 1 || pass_idx == 5) return 1;
    if (start == i0 && stop == j0) return 1;
    if (local) {
        if (mode == TRMODE_J) return 1;
        if (mode == TRMODE_L) return stop == j0;
        if (mode == TRMODE_R) return start == i0;
        return 0;
    }
    if (mode == TRMODE_J) return lpos[b] == 1 && rpos[b] == clen;
    if (mode == TRMODE_L) return stop == j0 && lpos[b] == 1;
    if (mode == TRMODE_R) return start == i0 && rpos[b] == clen;
    return 0;
}

static void fnorm4(float *v) {
    float sum = 0.0f;
    for (int a = 0; a < 4; a++) sum += v[a];
    if (sum > 0.0f)
        for (int a = 0; a < 4; a++) v[a] /= sum;
    else
        for (int a = 0; a < 4; a++) v[a] = 0.25f;
}

typedef struct {
    trhit *v;
    int n, cap;
} trvec;
static void tv_push(trvec *t, trhit h) {
    if (t->n == t->cap) {
        t->cap = t->cap ? 2 * t->cap : 64;
        t->v = (trhit *)realloc(t->v, sizeof(trhit) * (size_t)t->cap);
    }
    t->v[t->n++] = h;
}

/* report_hits_greedily (src/cm_dpsearch_trunc.rs:2322) */
static void report_tr(const cmgpu_cm *cm, int pass_idx, int local, const int32_t *lpos, const int32_t *rpos,
                      int clen, int j, int dmin, int dmax, const float *bestsc, const int32_t *bestr,
                      const int32_t *bestmode, int w, const double (*act)[4], int i0, int j0, float cutoff,
                      trvec *out) {
    if (dmin > dmax) return;
    float max_rep = IMPOSSIBLE;
    for (int d = dmin > 1 ? dmin : 1; d <= dmax; d++) {
        const int i = j - d + 1, mode = bestmode[d];
        float hit = bestsc[d], bias = 0.0f;
        if (!(hit > max_rep && hit >= cutoff && hit > IMPOSSIBLE + 1.0f)) continue;
        int rep = allow_trunc(pass_idx, local, lpos, rpos, clen, i, j, i0, j0, mode, bestr[d]);
        if (rep && act) {
            const int ip = i - i0 + 1, jp = j - i0 + 1;
            float comp[4];
            for (int a = 0; a < 4; a++) comp[a] = (float)(act[jp % (w + 1)][a] - act[(ip - 1) % (w + 1)][a]);
            fnorm4(comp);
            const float corr = oracle_null3(cm->null, comp, d, cm->n3_omega);
            hit -= corr;
            bias = corr;
            rep = hit > max_rep && hit >= cutoff;
        }
        if (rep) {
            trhit h = {i, j, hit, bias, mode, bestr[d]};
            tv_push(out, h);
            max_rep = hit;
        }
    }
}

static int cmp_trhit(const trhit *x, const trhit *y) {
    if (x->score != y->score) return x->score > y->score ? -1 : 1;
    return (x->i > y->i) - (x->i < y->i);
}

static int finish_hits(trvec *t, trhit *out, int cap) {
    for (int a = 1; a < t->n; a++) { /* stable insertion sort */
        trhit x = t->v[a];
        int b = a - 1;
        while (b >= 0 && cmp_trhit(&t->v[b], &x) > 0) {
            t->v[b + 1] = t->v[b];
            b--;
        }
        t->v[b + 1] = x;
    }
    char *rm = (char *)calloc((size_t)t->n + 1, 1);
    int kept = 0;
    for (int a = 0; a < t->n; a++) {
        if (rm[a]) continue;
        for (int b = a + 1; b < t->n; b++)
            if (!rm[b] && !(t->v[b].j < t->v[a].i) && !(t->v[a].j < t->v[b].i)) rm[b] = 1;
    }
    for (int a = 0; a < t->n; a++)
        if (!rm[a]) {
            if (kept < cap) out[kept] = t->v[a];
            kept++;
        }
    free(rm);
    return kept;
}

#define IDX3(a, v, d) ((((size_t)(a) * (size_t)m) + (size_t)(v)) * (size_t)(w + 1) + (size_t)(d))
#define IDXB(jj, b, d) ((((size_t)(jj) * (size_t)nbegl) + (size_t)(b)) * (size_t)(w + 1) + (size_t)(d))

#define TRQ_SCAN(NAME, T, COMB, MAX2, ADD, ORD, BITS, ISIMP, ZERO, BASE0)                                            \
    static int NAME(const cmgpu_cm *cm, const T *tsc, const T *oesc, const T *lmesc, const T *rmesc,                 \
                    const T *endsc, T el_self, const T *pty, const int32_t *lpos, const int32_t *rpos, int clen,     \
                    const uint8_t *dsq, int i0, int j0, float cutoff, int do_null3, int qdbidx, int pass_idx,         \
                    int local, float *vsc_out, int32_t *vmode_out, float *bsc_full_out, trhit *hits, int cap) {        \
        const int m = cm->M, smx_w = cm->W, l = j0 - i0 + 1;                                                         \
        const int w = smx_w < l ? smx_w : l;                                                                         \
        const int fill_l = pass_idx == 3 || pass_idx == 4 || pass_idx == 5;                                          \
        const int fill_r = pass_idx == 2 || pass_idx == 4 || pass_idx == 5;                                          \
        const int fill_t = pass_idx == 4 || pass_idx == 5;                                                           \
        const int nonbanded = qdbidx == 0;                                                                           \
        int *dmax = (int *)malloc(sizeof(int) * (size_t)m), *dxcap = (int *)malloc(sizeof(int) * (size_t)m);         \
        for (int v = 0; v < m; v++) {                                                                                \
            dmax[v] = nonbanded ? smx_w : (qdbidx == 1 ? cm->dmax1[v] : cm->dmax2[v]);                               \
            dxcap[v] = dmax[v] < smx_w ? dmax[v] : smx_w;                                                            \
        }                                                                                                            \
        int *begl_idx = (int *)malloc(sizeof(int) * (size_t)m), nbegl = 0;                                           \
        for (int v = 0; v < m; v++) begl_idx[v] = cm->stid[v] == BEGL_S ? nbegl++ : -1;                              \
        T *el_sca = (T *)malloc(sizeof(T) * (size_t)(w + 1));                                                        \
        el_sca[0] = BASE0;                                                                                           \
        for (int d = 1; d <= w; d++) el_sca[d] = ADD(el_sca[d - 1], el_self);                                        \
        T *init_sc = (T *)malloc(sizeof(T) * (size_t)m * (size_t)(w + 1));                                          \
        for (int v = 0; v < m; v++)                                                                                  \
            for (int d = 0; d <= w; d++)                                                                             \
                init_sc[(size_t)v * (w + 1) + d] = ISIMP(endsc[v]) ? ZERO : ADD(el_sca[d], endsc[v]);                \
        const size_t n3 = (size_t)2 * m * (w + 1), nb = (size_t)(w + 1) * (nbegl ? nbegl : 1) * (w + 1);             \
        T *ja = (T *)malloc(sizeof(T) * n3), *la = (T *)malloc(sizeof(T) * n3), *ra = (T *)malloc(sizeof(T) * n3),    \
          *ta = (T *)malloc(sizeof(T) * n3);                                                                         \
        T *jb = (T *)malloc(sizeof(T) * nb), *lb = (T *)malloc(sizeof(T) * nb), *rb = (T *)malloc(sizeof(T) * nb);   \
        for (size_t q = 0; q < n3; q++) ja[q] = la[q] = ra[q] = ta[q] = ZERO;                                        \
        for (size_t q = 0; q < nb; q++) jb[q] = lb[q] = rb[q] = ZERO;                                                \
        for (int v = m - 1; v >= 0; v--) {                                                                           \
            const int st = cm->sttype[v];                                                                            \
            if (cm->stid[v] != BEGL_S) {                                                                             \
                if (st == E_ST) {                                                                                    \
                    for (int a = 0; a < 2; a++) {                                                                    \
                        ja[IDX3(a, v, 0)] = BASE0;                                                                   \
                        la[IDX3(a, v, 0)] = BASE0;                                                                   \
                        ra[IDX3(a, v, 0)] = BASE0;                                                                   \
                    }                                                                                                \
                } else if (st == S_ST || st == D_ST) {                                                               \
                    const int y = cm->cfirst[v];                                                                     \
                    T a0 = endsc[v];                                                                                 \
                    for (int yo = 0; yo < cm->cnum[v]; yo++) a0 = MAX2(a0, ADD(ja[IDX3(0, y + yo, 0)], tsc[v * 6 + yo])); \
                    a0 = MAX2(a0, ZERO);                                                                             \
                    ja[IDX3(0, v, 0)] = a0;                                                                          \
                    ja[IDX3(1, v, 0)] = a0;                                                                          \
                } else if (st == B_ST) {                                                                             \
                    const int wl = cm->cfirst[v], y = cm->cnum[v];                                                   \
                    const T a0 = ADD(jb[IDXB(0, begl_idx[wl], 0)], ja[IDX3(0, y, 0)]);                                \
                    ja[IDX3(0, v, 0)] = a0;                                                                          \
                    ja[IDX3(1, v, 0)] = a0;                                                                          \
                }                                                                                                    \
            } else {                                                                                                 \
                const int bi = begl_idx[v], y = cm->cfirst[v];                                                       \
                T a0 = endsc[v];                                                                                     \
                for (int yo = 0; yo < cm->cnum[v]; yo++) a0 = MAX2(a0, ADD(ja[IDX3(0, y + yo, 0)], tsc[v * 6 + yo]));    \
                a0 = MAX2(a0, ZERO);                                                                                 \
                for (int jj = 0; jj <= w; jj++) jb[IDXB(jj, bi, 0)] = a0;                                            \
            }                                                                                                        \
        }                                                                                                            \
        double(*act)[4] = (double(*)[4])calloc((size_t)w + 1, sizeof(double[4]));                                    \
        int *jp_wa = (int *)malloc(sizeof(int) * (size_t)(w + 1));                                                   \
        float *bestsc = (float *)malloc(sizeof(float) * (size_t)(w + 1));                                            \
        int32_t *bestr = (int32_t *)malloc(sizeof(int32_t) * (size_t)(w + 1));                                       \
        int32_t *bestmode = (int32_t *)malloc(sizeof(int32_t) * (size_t)(w + 1));                                    \
        float vsc = IMPOSSIBLE, bsc_full = IMPOSSIBLE;                                                               \
        int vmode = TRMODE_UNKNOWN;                                                                                  \
        trvec tmp = {0, 0, 0};                                                                                       \
        for (int j = i0; j <= j0; j++) {                                                                             \
            const int jp_g = j - i0 + 1, cur = j & 1, prv = (j - 1) & 1;                                             \
            const int jrow = jp_g < w ? jp_g : w;                                                                    \
            for (int d = 0; d <= w; d++) jp_wa[d] = (((j - d) % (w + 1)) + (w + 1)) % (w + 1);                       \
            if (do_null3) {                                                                                          \
                const int src = (jp_g - 1) % (w + 1), dst = jp_g % (w + 1);                                          \
                memcpy(act[dst], act[src], sizeof(double[4]));                                                       \
                if (dsq[j] < 4) act[dst][dsq[j]] += 1.0;                                                             \
            }                                                                                                        \
            for (int v = m - 1; v >= 1; v--) {                                                                       \
                const int st = cm->sttype[v];                                                                        \
                if (st == E_ST) continue;                                                                            \
                const int sd = sdelta(st), em = emitmode(st), is_begl = cm->stid[v] == BEGL_S;                       \
                const int jp_v = is_begl ? (((j % (w + 1)) + (w + 1)) % (w + 1)) : cur;                              \
                const int jp_y = srdelta(st) > 0 ? prv : cur, jq_y = srdelta(st) > 0 ? cur : prv;                    \
                const int dn = 1, dx = jrow < dxcap[v] ? jrow : dxcap[v];                                            \
                const T *esc = oesc + (size_t)v * ESCW, *ts = tsc + (size_t)v * 6;                                   \
                const T *lm = lmesc + (size_t)v * KP, *rm = rmesc + (size_t)v * KP;                                  \
                const T *isv = init_sc + (size_t)v * (w + 1);                                                        \
                const T esc_j = (st == IR_ST || st == MR_ST) ? esc[dsq[j]] : ZERO;                                   \
                const T rmesc_j = (st == IR_ST || st == MR_ST || st == MP_ST) ? rm[dsq[j]] : ZERO;                   \
                const int detached = cm->stid[v + 1] == END_E;                                                       \
                if (st == B_ST) {                                                                                    \
                    const int wl = cm->cfirst[v], y = cm->cnum[v], bi = begl_idx[wl];                                \
                    const int dx_y = dmax[y] < smx_w ? dmax[y] : smx_w, dx_w = dmax[wl] < smx_w ? dmax[wl] : smx_w;  \
                    for (int d = dn; d <= dx; d++) {                                                                 \
                        int kmin = 0, kmax = d;                                                                      \
                        if (!nonbanded) {                                                                            \
                            kmin = d - dx_w > 0 ? d - dx_w : 0;                                                      \
                            kmax = dx_y < d ? dx_y : d;                                                              \
                        }                                                                                            \
                        T jsc = isv[d - sd], lsc = fill_l ? isv[d - sd] : ZERO, rsc = fill_r ? isv[d - sd] : ZERO,   \
                          tsc2 = fill_t ? isv[d - sd] : ZERO;                                                        \
                        for (int k = kmin; k <= kmax; k++) {                                                         \
                            const T lft = jb[IDXB(jp_wa[k], bi, d - k)];                                             \
                            jsc = COMB(jsc, ADD(lft, ja[IDX3(jp_y, y, k)]));                                         \
                            if (fill_l) lsc = COMB(lsc, ADD(lft, la[IDX3(jp_y, y, k)]));                             \
                            if (fill_r) rsc = COMB(rsc, ADD(rb[IDXB(jp_wa[k], bi, d - k)], ja[IDX3(jp_y, y, k)]));   \
                        }                                                                                            \
                        if (fill_t) {                                                                                \
                            const int kn = kmin > 1 ? kmin : 1, kx = d - 1 < kmax ? d - 1 : kmax;                    \
                            for (int k = kn; k <= kx; k++)                                                           \
                                tsc2 = COMB(tsc2, ADD(rb[IDXB(jp_wa[k], bi, d - k)], la[IDX3(jp_y, y, k)]));         \
                        }                                                                                            \
                        ja[IDX3(jp_v, v, d)] = jsc;                                                                  \
                        if (fill_t) ta[IDX3(jp_v, v, d)] = tsc2;                                                     \
                        if (fill_l)                                                                                  \
                            la[IDX3(jp_v, v, d)] =                                                                   \
                                kmin == 0 ? COMB(lsc, MAX2(jb[IDXB(jp_wa[0], bi, d)], lb[IDXB(jp_wa[0], bi, d)]))  \
                                          : lsc;                                                                     \
                        if (fill_r)                                                                                  \
                            ra[IDX3(jp_v, v, d)] =                                                                   \
                                kmax == d ? COMB(rsc, MAX2(ja[IDX3(jp_y, y, d)], ra[IDX3(jp_y, y, d)])) : rsc;       \
                    }                                                                                                \
                } else if (is_begl) {                                                                                \
                    const int y = cm->cfirst[v], bi = begl_idx[v];                                                   \
                    for (int d = dn; d <= dx; d++) {                                                                 \
                        T jsc = isv[d - sd], lsc = fill_l ? isv[d - sd] : ZERO, rsc = fill_r ? isv[d - sd] : ZERO;   \
                        for (int yo = 0; yo < cm->cnum[v]; yo++) {                                                   \
                            jsc = COMB(jsc, ADD(ja[IDX3(jp_y, y + yo, d - sd)], ts[yo]));                            \
                            if (fill_l) lsc = COMB(lsc, ADD(la[IDX3(jp_y, y + yo, d - sd)], ts[yo]));                \
                            if (fill_r) rsc = COMB(rsc, ADD(ra[IDX3(jp_y, y + yo, d - sd)], ts[yo]));                \
                        }                                                                                            \
                        jb[IDXB(jp_v, bi, d)] = jsc;                                                                 \
                        if (fill_l) lb[IDXB(jp_v, bi, d)] = lsc;                                                     \
                        if (fill_r) rb[IDXB(jp_v, bi, d)] = rsc;                                                     \
                    }                                                                                                \
                } else if (em == 1) {                                                                                \
                    if (!detached) {                                                                                 \
                        const int y = cm->cfirst[v], ry0 = st == IL_ST ? 1 : 0;                                      \
                        int i = j - dn + 1;                                                                          \
                        for (int d = dn; d <= dx; d++) {                                                             \
                            T jsc = isv[d - sd], lsc = fill_l ? isv[d - sd] : ZERO;                                  \
                            if (fill_r) ra[IDX3(jp_v, v, d)] = isv[d];                                               \
                            for (int yo = 0; yo < cm->cnum[v]; yo++) {                                               \
                                jsc = COMB(jsc, ADD(ja[IDX3(jp_y, y + yo, d - sd)], ts[yo]));                        \
                                if (fill_l) lsc = COMB(lsc, ADD(la[IDX3(jp_y, y + yo, d - sd)], ts[yo]));            \
                            }                                                                                        \
                            const T e = esc[dsq[i]];                                                                 \
                            ja[IDX3(jp_v, v, d)] = ADD(jsc, e);                                                      \
                            if (fill_l) la[IDX3(jp_v, v, d)] = d >= 2 ? ADD(lsc, e) : e;                             \
                            if (fill_r) {                                                                            \
                                T rsc = ra[IDX3(jp_v, v, d)];                                                        \
                                for (int yo = ry0; yo < cm->cnum[v]; yo++)                                           \
                                    rsc = COMB(rsc, MAX2(ADD(ja[IDX3(jp_y, y + yo, d)], ts[yo]),                     \
                                                         ADD(ra[IDX3(jp_y, y + yo, d)], ts[yo])));                   \
                                ra[IDX3(jp_v, v, d)] = rsc;                                                          \
                            }                                                                                        \
                            i--;                                                                                     \
                        }                                                                                            \
                    }                                                                                                \
                } else if (em == 2) {                                                                                \
                    if (!detached) {                                                                                 \
                        const int y = cm->cfirst[v], ly0 = st == IR_ST ? 1 : 0;                                      \
                        for (int d = dn; d <= dx; d++) {                                                             \
                            T jsc = isv[d - sd], rsc = fill_r ? isv[d - sd] : ZERO;                                  \
                            if (fill_l) la[IDX3(jp_v, v, d)] = isv[d];                                               \
                            for (int yo = 0; yo < cm->cnum[v]; yo++) {                                               \
                                jsc = COMB(jsc, ADD(ja[IDX3(jp_y, y + yo, d - sd)], ts[yo]));                        \
                                if (fill_r) rsc = COMB(rsc, ADD(ra[IDX3(jp_y, y + yo, d - sd)], ts[yo]));            \
                            }                                                                                        \
                            ja[IDX3(jp_v, v, d)] = ADD(jsc, esc_j);                                                  \
                            if (fill_r) ra[IDX3(jp_v, v, d)] = d >= 2 ? ADD(rsc, esc_j) : esc_j;                     \
                            if (fill_l) {                                                                            \
                                T lsc = la[IDX3(jp_v, v, d)];                                                        \
                                for (int yo = ly0; yo < cm->cnum[v]; yo++)                                           \
                                    lsc = COMB(lsc, MAX2(ADD(ja[IDX3(jq_y, y + yo, d)], ts[yo]),                     \
                                                         ADD(la[IDX3(jq_y, y + yo, d)], ts[yo])));                   \
                                la[IDX3(jp_v, v, d)] = lsc;                                                          \
                            }                                                                                        \
                        }                                                                                            \
                    }                                                                                                \
                } else if (em == 3) {                                                                                \
                    const int y = cm->cfirst[v];                                                                     \
                    int i = j - dn + 1;                                                                              \
                    for (int d = dn; d <= dx; d++) {                                                                 \
                        T jsc = d >= 2 ? isv[d - sd] : ZERO, lsc = fill_l ? isv[d - 1] : ZERO,                       \
                          rsc = fill_r ? isv[d - 1] : ZERO;                                                          \
                        for (int yo = 0; yo < cm->cnum[v]; yo++) {                                                   \
                            if (d >= 2) jsc = COMB(jsc, ADD(ja[IDX3(jp_y, y + yo, d - 2)], ts[yo]));                 \
                            if (fill_l)                                                                              \
                                lsc = COMB(lsc, MAX2(ADD(ja[IDX3(jq_y, y + yo, d - 1)], ts[yo]),                     \
                                                     ADD(la[IDX3(jq_y, y + yo, d - 1)], ts[yo])));                   \
                            if (fill_r)                                                                              \
                                rsc = COMB(rsc, MAX2(ADD(ja[IDX3(jp_y, y + yo, d - 1)], ts[yo]),                     \
                                                     ADD(ra[IDX3(jp_y, y + yo, d - 1)], ts[yo])));                   \
                        }                                                                                            \
                        ja[IDX3(jp_v, v, d)] = d >= 2 ? ADD(jsc, esc[dsq[i] * KP + dsq[j]]) : ZERO;                  \
                        if (fill_l) la[IDX3(jp_v, v, d)] = d >= 2 ? ADD(lsc, lm[dsq[i]]) : lm[dsq[i]];               \
                        if (fill_r) ra[IDX3(jp_v, v, d)] = d >= 2 ? ADD(rsc, rmesc_j) : rmesc_j;                     \
                        i--;                                                                                         \
                    }                                                                                                \
                } else {                                                                                             \
                    const int y = cm->cfirst[v];                                                                     \
                    for (int d = dn; d <= dx; d++) {                                                                 \
                        T jsc = isv[d - sd], lsc = fill_l ? isv[d - sd] : ZERO, rsc = fill_r ? isv[d - sd] : ZERO;   \
                        for (int yo = 0; yo < cm->cnum[v]; yo++) {                                                   \
                            jsc = COMB(jsc, ADD(ja[IDX3(jp_y, y + yo, d - sd)], ts[yo]));                            \
                            if (fill_l) lsc = COMB(lsc, ADD(la[IDX3(jp_y, y + yo, d - sd)], ts[yo]));                \
                            if (fill_r) rsc = COMB(rsc, ADD(ra[IDX3(jp_y, y + yo, d - sd)], ts[yo]));                \
                        }                                                                                            \
                        ja[IDX3(jp_v, v, d)] = jsc;                                                                  \
                        if (fill_l) la[IDX3(jp_v, v, d)] = lsc;                                                      \
                        if (fill_r) ra[IDX3(jp_v, v, d)] = rsc;                                                      \
                    }                                                                                                \
                }                                                                                                    \
            }                                                                                                        \
            /* ROOT: truncated begins into the persistent row */                                                     \
            const int dn0 = 1, dx0 = jrow < dxcap[0] ? jrow : dxcap[0];                                              \
            for (int d = 0; d <= w; d++) {                                                                           \
                bestr[d] = 0;                                                                                        \
                bestsc[d] = IMPOSSIBLE;                                                                              \
                bestmode[d] = TRMODE_UNKNOWN;                                                                        \
            }                                                                                                        \
            for (int y = 1; y < m; y++) {                                                                            \
                const T pen = pty[y];                                                                                \
                if (ISIMP(pen)) continue;                                                                            \
                const int dxy = jrow < dxcap[y] ? jrow : dxcap[y];                                                   \
                const int dxm = dx0 < dxy ? dx0 : dxy;                                                               \
                T *P[4] = {ja, la, ra, ta};                                                                          \
                const int on[4] = {1, fill_l, fill_r, fill_t && cm->sttype[y] == B_ST};                              \
                const int md[4] = {TRMODE_J, TRMODE_L, TRMODE_R, TRMODE_T};                                          \
                for (int pl = 0; pl < 4; pl++) {                                                                     \
                    if (!on[pl]) continue;                                                                           \
                    for (int d = dn0; d <= dxm; d++) {                                                               \
                        const T sc = ADD(P[pl][IDX3(cur, y, d)], pen);                                               \
                        if (ORD(sc) > ORD(P[pl][IDX3(cur, 0, d)])) {                                                 \
                            P[pl][IDX3(cur, 0, d)] = sc;                                                             \
                            const float fsc = BITS(sc);                                                              \
                            if (fsc > bestsc[d]) {                                                                   \
                                bestsc[d] = fsc;                                                                     \
                                bestmode[d] = md[pl];                                                                \
                                bestr[d] = y;                                                                        \
                            }                                                                                        \
                        }                                                                                            \
                    }                                                                                                \
                }                                                                                                    \
            }                                                                                                        \
            for (int d = dn0; d <= dx0; d++)                                                                         \
                if (bestsc[d] > vsc) {                                                                               \
                    vsc = bestsc[d];                                                                                 \
                    vmode = bestmode[d];                                                                             \
                }                                                                                                    \
            if (j == j0 && j <= w && bestsc[j] > bsc_full) bsc_full = bestsc[j];                                     \
            report_tr(cm, pass_idx, local, lpos, rpos, clen, j, dn0, dx0, bestsc, bestr, bestmode, w,                \
                      do_null3 ? (const double(*)[4])act : NULL, i0, j0, cutoff, &tmp);                              \
        }                                                                                                            \
        const int kept = finish_hits(&tmp, hits, cap);                                                               \
        *vsc_out = vsc;                                                                                              \
        *vmode_out = vmode;                                                                                          \
        *bsc_full_out = bsc_full;                                                                                    \
        free(tmp.v);                                                                                                 \
        free(bestmode);                                                                                              \
        free(bestr);                                                                                                 \
        free(bestsc);                                                                                                \
        free(jp_wa);                                                                                                 \
        free(act);                                                                                                   \
        free(jb);                                                                                                    \
        free(lb);                                                                                                    \
        free(rb);                                                                                                    \
        free(ja);                                                                                                    \
        free(la);                                                                                                    \
        free(ra);                                                                                                    \
        free(ta);                                                                                                    \
        free(init_sc);                                                                                               \
        free(el_sca);                                                                                                \
        free(begl_idx);                                                                                              \
        free(dxcap);                                                                                                 \
        free(dmax);                                                                                                  \
        return kept;                                                                                                 \
    }

TRQ_SCAN(trq_scan_f, float, f_comb, f_max2, f_add, f_ord, f_bits, f_isimp, IMPOSSIBLE, 0.0f)
TRQ_SCAN(trq_scan_i, int32_t, i_comb, i_max2, i_add, i_ord, i_bits, i_isimp, (-INFTY), 0)

/* inside = 0: ref_tr_cyk_scan (float tables); 1: ref_itr_inside_scan
 * (integer tables: itsc/ioesc/iendsc/iel_selfsc of the CM, ilmesc/irmesc/ipty). */
int oracle_trq_scan(const cmgpu_cm *cm, int inside, const float *lmesc, const float *rmesc, const float *pty,
                    const int32_t *ilmesc, const int32_t *irmesc, const int32_t *ipty, const int32_t *lpos,
                    const int32_t *rpos, int32_t clen, const uint8_t *dsq, int32_t i0, int32_t j0, float cutoff,
                    int do_null3, int qdbidx, int pass_idx, int local, float *vsc, int32_t *vmode, float *bsc_full,
                    trhit *hits, int32_t cap) {
    if (inside)
        return trq_scan_i(cm, cm->itsc, cm->ioesc, ilmesc, irmesc, cm->iendsc, cm->iel_selfsc, ipty, lpos, rpos, clen,
                          dsq, i0, j0, cutoff, do_null3, qdbidx, pass_idx, local, vsc, vmode, bsc_full, hits, cap);
    return trq_scan_f(cm, cm->tsc, cm->oesc, lmesc, rmesc, cm->endsc, cm->el_selfsc, pty, lpos, rpos, clen, dsq, i0,
                      j0, cutoff, do_null3, qdbidx, pass_idx, local, vsc, vmode, bsc_full, hits, cap);
}
