/*
 * msv_oracle.c -- TEST INFRASTRUCTURE ONLY.  CPU restatement of the
 * reference's F1 MSV/SSV filter (src/cm_pipeline.rs):
 *   build_msv_filter (:201-340): byteified emission costs, bias, the B->M,
 *     E->C and J->B move costs, prefix/suffix window-extension lengths;
 *   msv_score_tjb (:412-452): full-sequence 8-bit MSV score, None on overflow;
 *   ssv_diagonals (:521-717): the SSV longtarget row scan with the trigger,
 *     backward recovery, forward extension, reset and skip;
 *   extend_and_merge (:722-815), split_windows (:817-840),
 *   f1_msv_windows (:842-857);
 *   esl_gumbel_invsurv (src/easel/gumbel.rs:168-179).
 * Natural-order scalar loops, unsigned 8-bit saturating arithmetic.  The
 * parity checker for the GPU MSV / SSV kernels.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define KP 18
static const double LN2 = 0.6931471805599453;

static uint8_t sadd8(uint8_t a, uint8_t b) {
    int s = (int)a + (int)b;
    return (uint8_t)(s > 255 ? 255 : s);
}
static uint8_t ssub8(uint8_t a, uint8_t b) { return (uint8_t)(a > b ? a - b : 0); }
static uint8_t max8(uint8_t a, uint8_t b) { return a > b ? a : b; }

/* unbiased_byteify (src/cm_pipeline.rs:146-150) */
static uint8_t unbiased_byteify(float scale_b, float sc) {
    float v = -roundf(scale_b * sc);
    if (v >= 255.0f) return 255;
    if (v <= 0.0f) return 0;
    return (uint8_t)v;
}

/* biased_byteify (src/cm_pipeline.rs:164-172) */
static uint8_t biased_byteify(float scale_b, uint8_t bias_b, float sc) {
    float v = -roundf(scale_b * sc);
    if (v > (float)(255 - (int)bias_b)) return 255;
    int b = (int)v + (int)bias_b;
    return (uint8_t)(b < 0 ? 0 : (b > 255 ? 255 : b));
}

static int degen(int code, int *out) {
    static const int sets[KP][5] = {{1, 0}, {1, 1}, {1, 2}, {1, 3}, {0},       {2, 0, 2},    {2, 1, 3},
                                    {2, 0, 1}, {2, 2, 3}, {2, 1, 2}, {2, 0, 3}, {3, 0, 1, 3}, {3, 1, 2, 3},
                                    {3, 0, 1, 2}, {3, 0, 2, 3}, {4, 0, 1, 2, 3}, {0}, {0}};
    for (int q = 0; q < sets[code][0]; q++) out[q] = sets[code][1 + q];
    return sets[code][0];
}

typedef struct {
    int m, max_length;
    float scale_b;
    uint8_t base_b, bias_b, tbm_b, tec_b, tjb_b;
    uint8_t *rbv; /* [m+1][KP] */
    float *prefix, *suffix;
    double mmu, mlambda;
} msvf;

static void msv_free(msvf *f) {
    free(f->rbv);
    free(f->prefix);
    free(f->suffix);
}

/* build_msv_filter; mat [m+1][4], trans [m+1][7] = MM,MI,MD,IM,II,DM,DD */
static void msv_build(int m, const float *mat, const float *trans, int max_length, double mmu, double mlambda,
                      msvf *f) {
    f->m = m;
    f->max_length = max_length;
    f->mmu = mmu;
    f->mlambda = mlambda;
    f->scale_b = (float)(3.0 / LN2);
    f->base_b = 190;
    float *msc = (float *)malloc(sizeof(float) * (size_t)(m + 1) * KP);
    for (int i = 0; i < (m + 1) * KP; i++) msc[i] = -INFINITY;
    float maxsc = 0.0f;
    for (int k = 1; k <= m; k++) {
        float *sc = msc + (size_t)k * KP;
        for (int x = 0; x < 4; x++) {
            sc[x] = (float)log((double)mat[k * 4 + x] / 0.25);
            if (sc[x] > maxsc) maxsc = sc[x];
        }
        for (int code = 4; code < KP; code++) {
            int set[4];
            int n = degen(code, set);
            if (n == 0) continue;
            float s = 0.0f;
            for (int q = 0; q < n; q++) s += sc[set[q]];
            sc[code] = s / (float)n;
        }
    }
    f->bias_b = unbiased_byteify(f->scale_b, -maxsc);
    f->rbv = (uint8_t *)malloc((size_t)(m + 1) * KP);
    memset(f->rbv, 255, (size_t)(m + 1) * KP);
    for (int k = 1; k <= m; k++)
        for (int x = 0; x < KP; x++)
            f->rbv[k * KP + x] = biased_byteify(f->scale_b, f->bias_b, msc[(size_t)k * KP + x]);
    free(msc);
    f->tbm_b = unbiased_byteify(f->scale_b, (float)log(2.0 / ((double)m * ((double)m + 1.0))));
    f->tec_b = unbiased_byteify(f->scale_b, logf(0.5f));
    f->tjb_b = unbiased_byteify(f->scale_b, (float)log(3.0 / ((double)max_length + 3.0)));

    /* prefix / suffix lengths (src/cm_pipeline.rs:292-325) */
    f->prefix = (float *)calloc((size_t)m + 1, sizeof(float));
    f->suffix = (float *)calloc((size_t)m + 1, sizeof(float));
    float sum = 0.0f;
    for (int k = 1; k < m; k++) {
        double t_mi = (double)trans[k * 7 + 1], t_ii = (double)trans[k * 7 + 4];
        float v;
        if (t_mi == 0.0) {
            v = 1.0f;
        } else {
            double lii = log(t_ii);
            if (lii == 0.0 || !isfinite(lii))
                v = 1.0f;
            else
                v = (float)(1.0 + trunc(log(1e-7 / t_mi) / lii));
        }
        f->prefix[k] = v;
        sum += v;
    }
    f->prefix[0] = 0.0f;
    f->prefix[m] = 0.0f;
    if (sum > 0.0f)
        for (int k = 1; k < m; k++) f->prefix[k] /= sum;
    f->suffix[m] = f->prefix[m - 1];
    for (int k = m - 1; k >= 1; k--) f->suffix[k] = f->suffix[k + 1] + f->prefix[k - 1];
    for (int k = 2; k < m; k++) f->prefix[k] += f->prefix[k - 1];
}

/* msv_score_tjb: returns 1 and the score, or 0 on overflow (None) */
static int msv_score_tjb(const msvf *f, const uint8_t *dsq, int l, uint8_t tjb_b, float *out) {
    const int m = f->m;
    const uint8_t bias = f->bias_b, tec = f->tec_b, base = f->base_b;
    const uint8_t tjbm = (uint8_t)(tjb_b + f->tbm_b); /* wrapping */
    uint8_t *dp = (uint8_t *)calloc((size_t)m + 1, 1);
    uint8_t xj = 0, xb = ssub8(base, tjbm);
    for (int i = 1; i <= l; i++) {
        int x = dsq[i];
        uint8_t xe = 0, mpv = 0;
        for (int k = 1; k <= m; k++) {
            uint8_t sv = max8(mpv, xb);
            sv = sadd8(sv, bias);
            sv = ssub8(sv, f->rbv[k * KP + x]);
            if (sv > xe) xe = sv;
            mpv = dp[k];
            dp[k] = sv;
        }
        if (sadd8(xe, bias) == 255) {
            free(dp);
            return 0;
        }
        xe = ssub8(xe, tec);
        xj = max8(xj, xe);
        xb = ssub8(max8(base, xj), tjbm);
    }
    free(dp);
    *out = ((float)((int)xj - (int)tjb_b) - (float)base) / f->scale_b - 3.0f;
    return 1;
}

/* esl_gumbel_invsurv */
static double gumbel_invsurv(double p, double mu, double lambda) {
    double log_part = p < 5e-9 ? (pow(p, p) - 1.0) / p : log(-log(1.0 - p));
    return mu - log_part / lambda;
}

typedef struct {
    int64_t n, length, k;
    float score;
} rawwin;

typedef struct {
    rawwin *v;
    int64_t n, cap;
} rawvec;

static void push_raw(rawvec *rv, rawwin w) {
    if (rv->n == rv->cap) {
        rv->cap = rv->cap ? rv->cap * 2 : 16;
        rv->v = (rawwin *)realloc(rv->v, sizeof(rawwin) * (size_t)rv->cap);
    }
    rv->v[rv->n++] = w;
}

/* ssv_diagonals: dsq 1-indexed with a sentinel at [0] */
static void ssv_diagonals(const msvf *f, const uint8_t *dsq, int64_t l, double f1, rawvec *out) {
    const int m = f->m;
    const double p1 = (double)f->max_length / ((double)f->max_length + 1.0);
    const double nullsc = (double)f->max_length * log(p1) + log(1.0 - p1);
    const double invp = gumbel_invsurv(f1, f->mmu, f->mlambda);
    const int sc_thresh = (int)ceil((nullsc + invp * LN2 + 3.0) * (double)f->scale_b + (double)f->base_b +
                                    (double)f->tec_b + (double)f->tjb_b);
    const uint8_t xb = ssub8(f->base_b, sadd8(f->tjb_b, f->tbm_b));
    uint8_t *rowa = (uint8_t *)calloc((size_t)m + 1, 1), *rowb = (uint8_t *)calloc((size_t)m + 1, 1);
    uint8_t *dp = rowa, *nw = rowb;
#define COST(kk, code) ((code) < KP ? f->rbv[(kk) * KP + (code)] : 255)
    int64_t i = 1;
    while (i <= l) {
        int x = dsq[i];
        uint8_t xe = 0;
        for (int k = 1; k <= m; k++) {
            uint8_t sv = ssub8(sadd8(max8(dp[k - 1], xb), f->bias_b), f->rbv[k * KP + x]);
            nw[k] = sv;
            if (sv > xe) xe = sv;
        }
        uint8_t *t = dp;
        dp = nw;
        nw = t;
        int end_k = 0;
        if ((int)xe >= sc_thresh) {
            uint8_t xe2 = 0;
            for (int k = 1; k <= m; k++)
                if (dp[k] > xe2) {
                    xe2 = dp[k];
                    end_k = k;
                }
        }
        if ((int)xe >= sc_thresh && end_k > 0) {
            const int baseline = (int)f->base_b - (int)f->tjb_b - (int)f->tbm_b;
            int64_t start = end_k, tstart = i;
            int rem = xe;
            while (rem > baseline && start >= 1 && tstart >= 1) {
                rem -= (int)f->bias_b - (int)COST(start, dsq[tstart]);
                start--;
                tstart--;
            }
            start++;
            tstart++;
            int sc2 = xe, max_sc = xe, since = 0;
            int64_t max_end = i, k = end_k + 1, n = i + 1;
            while (k < m && n <= l) {
                sc2 += (int)f->bias_b - (int)COST(k, dsq[n]);
                if (sc2 >= max_sc) {
                    max_sc = sc2;
                    max_end = n;
                    since = 0;
                } else {
                    since++;
                    if (since == 5) break;
                }
                k++;
                n++;
            }
            int64_t end_model = end_k + (max_end - i);
            float ret = ((float)(max_sc - (int)f->tjb_b) - (float)f->base_b) / f->scale_b - 3.0f;
            rawwin w = {tstart, end_model - start + 1, end_model, ret};
            push_raw(out, w);
            memset(dp, 0, (size_t)m + 1);
            i = max_end + 1;
            continue;
        }
        i++;
    }
#undef COST
    free(rowa);
    free(rowb);
}

typedef struct {
    int64_t start, end;
    float score;
} win;

/* extend_and_merge with pct_overlap = 0 (the value f1_msv_windows passes) */
static int64_t extend_and_merge(const msvf *f, rawvec *raws, int64_t target_len, win *out) {
    if (raws->n == 0) return 0;
    const double maxl = (double)f->max_length;
    for (int64_t q = 0; q < raws->n; q++) {
        rawwin *w = &raws->v[q];
        int64_t ks = w->k - w->length + 1, ke = w->k;
        ks = ks < 0 ? 0 : (ks > f->m ? f->m : ks);
        ke = ke < 0 ? 0 : (ke > f->m ? f->m : ke);
        double pref = (double)f->prefix[ks], suff = (double)f->suffix[ke];
        double ws = (double)w->n - maxl * (0.1 + pref);
        ws = ws > 1.0 ? ws : 1.0;
        double we = (double)w->n + (double)w->length + maxl * (0.1 + suff);
        we = we < (double)target_len ? we : (double)target_len;
        int64_t s = (int64_t)ws, e = (int64_t)we;
        w->n = s;
        w->length = e - s + 1;
    }
    int64_t nk = 0;
    rawwin *kept = (rawwin *)malloc(sizeof(rawwin) * (size_t)raws->n);
    kept[nk++] = raws->v[0];
    for (int64_t q = 1; q < raws->n; q++) {
        rawwin cur = raws->v[q];
        rawwin *prev = &kept[nk - 1];
        int64_t s = prev->n > cur.n ? prev->n : cur.n;
        int64_t pe = prev->n + prev->length - 1, ce = cur.n + cur.length - 1;
        int64_t e = pe < ce ? pe : ce;
        int64_t wl = e - s + 1;
        int64_t minlen = prev->length < cur.length ? prev->length : cur.length;
        if ((float)wl / (float)minlen > 0.0f) {
            int64_t ms = prev->n < cur.n ? prev->n : cur.n;
            int64_t me = pe > ce ? pe : ce;
            prev->n = ms;
            prev->length = me - ms + 1;
        } else {
            kept[nk++] = cur;
        }
    }
    for (int64_t q = 0; q < nk; q++) {
        out[q].start = kept[q].n;
        out[q].end = kept[q].n + kept[q].length - 1;
        out[q].score = kept[q].score;
    }
    free(kept);
    return nk;
}

/* split_windows; returns the count written (out sized by the caller) */
static int64_t split_windows(const win *in, int64_t n, int64_t cmw, win *out, int64_t cap) {
    int64_t c = 0;
    for (int64_t q = 0; q < n; q++) {
        win w = in[q];
        int64_t wlen = w.end - w.start + 1;
        if (wlen > 2 * cmw) {
            int64_t s = w.start, e = w.start + 2 * cmw - 1 < w.end ? w.start + 2 * cmw - 1 : w.end;
            if (c < cap) out[c] = (win){s, e, w.score};
            c++;
            while (e < w.end) {
                s = s + cmw < w.end ? s + cmw : w.end;
                e = e + cmw < w.end ? e + cmw : w.end;
                if (c < cap) out[c] = (win){s, e, w.score};
                c++;
            }
        } else {
            if (c < cap) out[c] = w;
            c++;
        }
    }
    return c;
}

/* ---------------- exported for tests ---------------- */

void oracle_msv_tables(int m, const float *mat, const float *trans, int max_length, uint8_t *rbv,
                       uint8_t *bytes6, float *prefix, float *suffix, float *scale_b) {
    msvf f;
    msv_build(m, mat, trans, max_length, 0.0, 1.0, &f);
    memcpy(rbv, f.rbv, (size_t)(m + 1) * KP);
    bytes6[0] = f.base_b;
    bytes6[1] = f.bias_b;
    bytes6[2] = f.tbm_b;
    bytes6[3] = f.tec_b;
    bytes6[4] = f.tjb_b;
    bytes6[5] = 0;
    memcpy(prefix, f.prefix, sizeof(float) * (size_t)(m + 1));
    memcpy(suffix, f.suffix, sizeof(float) * (size_t)(m + 1));
    *scale_b = f.scale_b;
    msv_free(&f);
}

/* msv_score (wlen == NULL) or msv_score_reconfig(f, dsq, l, wlen[w]) per
 * frame buf+offs[w] of lens[w] residues */
void oracle_msv_score_batch(int m, const float *mat, const float *trans, int max_length, const uint8_t *buf,
                            const int64_t *offs, const int32_t *lens, const int32_t *wlen, int32_t n, float *scores,
                            uint8_t *scored) {
    msvf f;
    msv_build(m, mat, trans, max_length, 0.0, 1.0, &f);
    for (int32_t w = 0; w < n; w++) {
        uint8_t tjb = wlen ? unbiased_byteify(f.scale_b, (float)log(3.0 / ((double)wlen[w] + 3.0))) : f.tjb_b;
        float s = 0.0f;
        scored[w] = (uint8_t)msv_score_tjb(&f, buf + offs[w], lens[w], tjb, &s);
        scores[w] = scored[w] ? s : NAN;
    }
    msv_free(&f);
}

/* f1_msv_windows on each chunk frame buf+offs[c] of lens[c] residues; out
 * rows (chunk, start, end) in int64 plus score; returns the total count
 * (entries beyond cap are not written). raw_out, if given, receives the
 * ssv_diagonals output (chunk, n, length, k) and raw_scores their scores. */
int64_t oracle_f1_msv_windows(int m, const float *mat, const float *trans, int max_length, double mmu,
                              double mlambda, const uint8_t *buf, const int64_t *offs, const int32_t *lens, int32_t n,
                              double f1, int64_t cmw, int64_t *out, float *out_scores, int64_t cap, int64_t *raw_out,
                              float *raw_scores, int64_t raw_cap, int64_t *n_raw) {
    msvf f;
    msv_build(m, mat, trans, max_length, mmu, mlambda, &f);
    int64_t total = 0, nr = 0;
    for (int32_t c = 0; c < n; c++) {
        rawvec rv = {0, 0, 0};
        ssv_diagonals(&f, buf + offs[c], lens[c], f1, &rv);
        for (int64_t q = 0; q < rv.n; q++) {
            if (raw_out && nr < raw_cap) {
                raw_out[nr * 4 + 0] = c;
                raw_out[nr * 4 + 1] = rv.v[q].n;
                raw_out[nr * 4 + 2] = rv.v[q].length;
                raw_out[nr * 4 + 3] = rv.v[q].k;
                raw_scores[nr] = rv.v[q].score;
            }
            nr++;
        }
        win *merged = (win *)malloc(sizeof(win) * (size_t)(rv.n + 1));
        int64_t nm = extend_and_merge(&f, &rv, lens[c], merged);
        int64_t ns = split_windows(merged, nm, cmw, NULL, 0);
        win *sp = (win *)malloc(sizeof(win) * (size_t)(ns + 1));
        split_windows(merged, nm, cmw, sp, ns);
        for (int64_t q = 0; q < ns; q++) {
            if (total < cap) {
                out[total * 3 + 0] = c;
                out[total * 3 + 1] = sp[q].start;
                out[total * 3 + 2] = sp[q].end;
                out_scores[total] = sp[q].score;
            }
            total++;
        }
        free(sp);
        free(merged);
        free(rv.v);
    }
    if (n_raw) *n_raw = nr;
    msv_free(&f);
    return total;
}

/* the SSV trigger threshold, for tests */
int oracle_ssv_threshold(int m, const float *mat, const float *trans, int max_length, double mmu, double mlambda,
                         double f1) {
    msvf f;
    msv_build(m, mat, trans, max_length, mmu, mlambda, &f);
    const double p1 = (double)f.max_length / ((double)f.max_length + 1.0);
    const double nullsc = (double)f.max_length * log(p1) + log(1.0 - p1);
    const double invp = gumbel_invsurv(f1, f.mmu, f.mlambda);
    int t = (int)ceil((nullsc + invp * LN2 + 3.0) * (double)f.scale_b + (double)f.base_b + (double)f.tec_b +
                      (double)f.tjb_b);
    msv_free(&f);
    return t;
}
