/*
 * fwd_oracle.c -- TEST INFRASTRUCTURE ONLY.  CPU restatement of the
 * reference's F3 / F3b filters (src/cm_pipeline.rs):
 *   build_forward_filter (:969-1120)       the odds-space local profile;
 *   forward_filter_score_striped (:1270-1418), the default Forward engine on
 *     x86: Farrar's striped layout with four lanes, emulated here lane by
 *     lane in scalar C with the same operation order (cell (q, z) is model
 *     position q + 1 + z * nq);
 *   build_bias_filter / bias_filter_score (:1683-1850), the two-state
 *     composition-bias null;
 *   the window gates of f3_filter_sequence (:1863-2164) live in oracle.py.
 * The parity checker for the GPU Forward and bias kernels.
 *
 * Built with -ffp-contract=off: every float multiply and add is rounded on
 * its own, as the reference's intrinsics and scalar code round them.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define KP 18
#define KC 4

static int fwd_degen(int code, int *out) {
    static const int sets[KP][5] = {{1, 0}, {1, 1}, {1, 2}, {1, 3}, {0},       {2, 0, 2},    {2, 1, 3},
                                    {2, 0, 1}, {2, 2, 3}, {2, 1, 2}, {2, 0, 3}, {3, 0, 1, 3}, {3, 1, 2, 3},
                                    {3, 0, 1, 2}, {3, 0, 2, 3}, {4, 0, 1, 2, 3}, {0}, {0}};
    int n = sets[code][0];
    for (int q = 0; q < n; q++) out[q] = sets[code][1 + q];
    return n;
}

/* natural-order arrays, index k = 0..m */
typedef struct {
    int m;
    float *rfv; /* [(m+1)][KP] emission odds */
    float *tbm, *amm, *aim, *adm, *tmi, *tii, *tmd, *tdd;
} fwdf;

static void fwd_free(fwdf *f) {
    free(f->rfv);
    free(f->tbm);
    free(f->amm);
    free(f->aim);
    free(f->adm);
    free(f->tmi);
    free(f->tii);
    free(f->tmd);
    free(f->tdd);
}

/* build_forward_filter (src/cm_pipeline.rs:969-1080): mat[k*4+x], trans[k*7+t]
 * with t = MM, MI, MD, IM, II, DM, DD. */
static void fwd_build(int m, const float *mat, const float *trans, fwdf *f) {
    f->m = m;
    f->rfv = (float *)calloc((size_t)(m + 1) * KP, sizeof(float));
    float **arr[8] = {&f->tbm, &f->amm, &f->aim, &f->adm, &f->tmi, &f->tii, &f->tmd, &f->tdd};
    for (int a = 0; a < 8; a++) *arr[a] = (float *)calloc((size_t)m + 1, sizeof(float));
    for (int k = 1; k <= m; k++) {
        float sc[KP];
        for (int x = 0; x < KP; x++) sc[x] = -INFINITY;
        for (int x = 0; x < KC; x++) sc[x] = (float)log((double)mat[k * 4 + x] / 0.25);
        for (int code = KC; code < KP; code++) {
            int set[4];
            int n = fwd_degen(code, set);
            if (n == 0) continue;
            float s = 0.0f;
            for (int q = 0; q < n; q++) s += sc[set[q]];
            sc[code] = s / (float)n;
        }
        for (int x = 0; x < KP; x++) f->rfv[k * KP + x] = expf(sc[x]);
    }
    /* occupancy (:1013-1024) and local entry (:1025-1040) */
    float *occ = (float *)calloc((size_t)m + 1, sizeof(float));
    if (m >= 1) occ[1] = trans[0 * 7 + 1] + trans[0 * 7 + 0];
    for (int k = 2; k <= m; k++)
        occ[k] = occ[k - 1] * (trans[(k - 1) * 7 + 0] + trans[(k - 1) * 7 + 1]) +
                 (1.0f - occ[k - 1]) * trans[(k - 1) * 7 + 5];
    float z = 0.0f;
    for (int k = 1; k <= m; k++) z += occ[k] * (float)(m - k + 1);
    for (int k = 1; k <= m; k++) f->tbm[k] = (float)exp(log((double)(occ[k] / z)));
    free(occ);
    for (int k = 1; k <= m; k++) {
        f->amm[k] = trans[(k - 1) * 7 + 0];
        f->aim[k] = trans[(k - 1) * 7 + 3];
        f->adm[k] = trans[(k - 1) * 7 + 5];
    }
    for (int k = 1; k < m; k++) {
        f->tmi[k] = trans[k * 7 + 1];
        f->tii[k] = trans[k * 7 + 4];
        f->tmd[k] = trans[k * 7 + 2];
        f->tdd[k] = trans[k * 7 + 6];
    }
}

static int fwd_nq(int m) {
    int nq = m >= 1 ? (m - 1) / 4 + 1 : 2;
    return nq < 2 ? 2 : nq;
}

static float at(const float *a, int m, int p) { return p <= m ? a[p] : 0.0f; }

/* lane z takes lane z-1's value, lane 0 takes zero (_mm_slli_si128 by 4) */
static void rsz(const float *v, float *out) {
    out[3] = v[2];
    out[2] = v[1];
    out[1] = v[0];
    out[0] = 0.0f;
}

/* forward_filter_score_striped (src/cm_pipeline.rs:1270-1418); also returns
 * the pieces of the score: the rescaling total and the final xC. */
static float fwd_score(const fwdf *f, const uint8_t *dsq, int L, float *ret_totscale, float *ret_xc) {
    const int m = f->m, nq = fwd_nq(m);
    const float nj = 1.0f;
    const float pmove = (2.0f + nj) / ((float)L + 2.0f + nj);
    const float ploop = 1.0f - pmove;
    const float xf_e_move = 0.5f, xf_e_loop = 0.5f;
    float *mm = (float *)calloc((size_t)4 * nq, sizeof(float));
    float *dm = (float *)calloc((size_t)4 * nq, sizeof(float));
    float *im = (float *)calloc((size_t)4 * nq, sizeof(float));
    float xn = 1.0f, xj = 0.0f, xb = pmove, xc = 0.0f, totscale = 0.0f;
    for (int i = 1; i <= L; i++) {
        const int x = dsq[i];
        float dcv[4] = {0, 0, 0, 0}, xev[4] = {0, 0, 0, 0};
        float mpv[4], dpv[4], ipv[4];
        rsz(mm + (nq - 1) * 4, mpv);
        rsz(dm + (nq - 1) * 4, dpv);
        rsz(im + (nq - 1) * 4, ipv);
        for (int q = 0; q < nq; q++) {
            for (int zz = 0; zz < 4; zz++) {
                const int p = q + 1 + zz * nq;
                float sv = xb * at(f->tbm, m, p);
                sv = sv + mpv[zz] * at(f->amm, m, p);
                sv = sv + ipv[zz] * at(f->aim, m, p);
                sv = sv + dpv[zz] * at(f->adm, m, p);
                sv = sv * (p <= m ? f->rfv[p * KP + x] : 0.0f);
                xev[zz] = xev[zz] + sv;
                mpv[zz] = mm[q * 4 + zz];
                dpv[zz] = dm[q * 4 + zz];
                ipv[zz] = im[q * 4 + zz];
                mm[q * 4 + zz] = sv;
                dm[q * 4 + zz] = dcv[zz];
                dcv[zz] = sv * at(f->tmd, m, p);
                float svi = mpv[zz] * at(f->tmi, m, p);
                im[q * 4 + zz] = svi + ipv[zz] * at(f->tii, m, p);
            }
        }
        /* DD paths: the obligatory pass */
        float t[4];
        rsz(dcv, t);
        memcpy(dcv, t, sizeof t);
        for (int zz = 0; zz < 4; zz++) dm[zz] = 0.0f;
        for (int q = 0; q < nq; q++)
            for (int zz = 0; zz < 4; zz++) {
                const int p = q + 1 + zz * nq;
                float d = dcv[zz] + dm[q * 4 + zz];
                dm[q * 4 + zz] = d;
                dcv[zz] = d * at(f->tdd, m, p);
            }
        for (int j = 1; j < 4; j++) {
            int changed = 0;
            rsz(dcv, t);
            memcpy(dcv, t, sizeof t);
            for (int q = 0; q < nq; q++)
                for (int zz = 0; zz < 4; zz++) {
                    const int p = q + 1 + zz * nq;
                    float old = dm[q * 4 + zz];
                    float d = dcv[zz] + old;
                    changed |= d > old;
                    dm[q * 4 + zz] = d;
                    dcv[zz] = dcv[zz] * at(f->tdd, m, p);
                }
            /* M >= 100: stop once a pass changes no cell (:1351-1380) */
            if (m >= 100 && !changed) break;
        }
        for (int q = 0; q < nq; q++)
            for (int zz = 0; zz < 4; zz++) xev[zz] = xev[zz] + dm[q * 4 + zz];
        float h[4];
        for (int zz = 0; zz < 4; zz++) h[zz] = xev[zz] + xev[(zz + 1) & 3];
        const float xe = h[0] + h[2];
        xn = xn * ploop;
        xc = (xc * ploop) + (xe * xf_e_move);
        xj = (xj * ploop) + (xe * xf_e_loop);
        xb = (xj * pmove) + (xn * pmove);
        if (xe > 1.0e4f) {
            const float inv = 1.0f / xe;
            xn *= inv;
            xc *= inv;
            xj *= inv;
            xb *= inv;
            for (int q = 0; q < 4 * nq; q++) {
                mm[q] = mm[q] * inv;
                dm[q] = dm[q] * inv;
                im[q] = im[q] * inv;
            }
            totscale += (float)log((double)xe);
        }
    }
    free(mm);
    free(dm);
    free(im);
    if (ret_totscale) *ret_totscale = totscale;
    if (ret_xc) *ret_xc = xc;
    return (float)((double)totscale + log((double)xc * (double)pmove));
}

#ifdef __SSE2__
#include <emmintrin.h>

/* The same engine on 128-bit vectors, as the reference runs it on x86: the
 * striped tables are packed once per profile (tmain[q][7][4] = BM, MM, IM,
 * DM, MD, MI, II; tdd[q][4]; rfv[x][q][4]) and every step above is one
 * packed op over the four lanes.  Bit-identical to fwd_score (the lanes are
 * independent except at the same shifts and sums); the timed CPU baseline. */
typedef struct {
    int m, nq;
    float *tmain, *tdd, *rfv;
} fwdv;

static void fwdv_build(const fwdf *f, fwdv *v) {
    const int m = f->m, nq = fwd_nq(m);
    v->m = m;
    v->nq = nq;
    v->tmain = (float *)aligned_alloc(16, sizeof(float) * (size_t)nq * 28);
    v->tdd = (float *)aligned_alloc(16, sizeof(float) * (size_t)nq * 4);
    v->rfv = (float *)aligned_alloc(16, sizeof(float) * (size_t)KP * nq * 4);
    const float *src[7] = {f->tbm, f->amm, f->aim, f->adm, f->tmd, f->tmi, f->tii};
    for (int q = 0; q < nq; q++)
        for (int zz = 0; zz < 4; zz++) {
            const int p = q + 1 + zz * nq;
            for (int t = 0; t < 7; t++) v->tmain[q * 28 + t * 4 + zz] = at(src[t], m, p);
            v->tdd[q * 4 + zz] = at(f->tdd, m, p);
            for (int x = 0; x < KP; x++) v->rfv[(x * nq + q) * 4 + zz] = p <= m ? f->rfv[p * KP + x] : 0.0f;
        }
}

static void fwdv_free(fwdv *v) {
    free(v->tmain);
    free(v->tdd);
    free(v->rfv);
}

static __m128 vshift(__m128 a) { return _mm_castsi128_ps(_mm_slli_si128(_mm_castps_si128(a), 4)); }

static float fwd_score_sse(const fwdv *v, const uint8_t *dsq, int L, float *ret_totscale, float *ret_xc) {
    const int m = v->m, nq = v->nq;
    const float nj = 1.0f;
    const float pmove = (2.0f + nj) / ((float)L + 2.0f + nj);
    const float ploop = 1.0f - pmove;
    __m128 *mm = (__m128 *)aligned_alloc(16, sizeof(__m128) * (size_t)nq);
    __m128 *dm = (__m128 *)aligned_alloc(16, sizeof(__m128) * (size_t)nq);
    __m128 *im = (__m128 *)aligned_alloc(16, sizeof(__m128) * (size_t)nq);
    const __m128 zero = _mm_setzero_ps();
    for (int q = 0; q < nq; q++) mm[q] = dm[q] = im[q] = zero;
    const __m128 *tm = (const __m128 *)v->tmain, *td = (const __m128 *)v->tdd;
    float xn = 1.0f, xj = 0.0f, xb = pmove, xc = 0.0f, totscale = 0.0f;
    for (int i = 1; i <= L; i++) {
        const __m128 *rf = (const __m128 *)v->rfv + (size_t)dsq[i] * nq;
        const __m128 xbv = _mm_set1_ps(xb);
        __m128 dcv = zero, xev = zero;
        __m128 mpv = vshift(mm[nq - 1]), dpv = vshift(dm[nq - 1]), ipv = vshift(im[nq - 1]);
        for (int q = 0; q < nq; q++) {
            const __m128 *t = tm + q * 7;
            __m128 sv = _mm_mul_ps(xbv, t[0]);
            sv = _mm_add_ps(sv, _mm_mul_ps(mpv, t[1]));
            sv = _mm_add_ps(sv, _mm_mul_ps(ipv, t[2]));
            sv = _mm_add_ps(sv, _mm_mul_ps(dpv, t[3]));
            sv = _mm_mul_ps(sv, rf[q]);
            xev = _mm_add_ps(xev, sv);
            mpv = mm[q];
            dpv = dm[q];
            ipv = im[q];
            mm[q] = sv;
            dm[q] = dcv;
            dcv = _mm_mul_ps(sv, t[4]);
            im[q] = _mm_add_ps(_mm_mul_ps(mpv, t[5]), _mm_mul_ps(ipv, t[6]));
        }
        dcv = vshift(dcv);
        dm[0] = zero;
        for (int q = 0; q < nq; q++) {
            dm[q] = _mm_add_ps(dcv, dm[q]);
            dcv = _mm_mul_ps(dm[q], td[q]);
        }
        for (int j = 1; j < 4; j++) {
            __m128 cv = zero;
            dcv = vshift(dcv);
            for (int q = 0; q < nq; q++) {
                const __m128 d = _mm_add_ps(dcv, dm[q]);
                cv = _mm_or_ps(cv, _mm_cmpgt_ps(d, dm[q]));
                dm[q] = d;
                dcv = _mm_mul_ps(dcv, td[q]);
            }
            if (m >= 100 && _mm_movemask_ps(cv) == 0) break;
        }
        for (int q = 0; q < nq; q++) xev = _mm_add_ps(xev, dm[q]);
        xev = _mm_add_ps(xev, _mm_shuffle_ps(xev, xev, 0x39));
        xev = _mm_add_ps(xev, _mm_shuffle_ps(xev, xev, 0x4E));
        const float xe = _mm_cvtss_f32(xev);
        xn = xn * ploop;
        xc = (xc * ploop) + (xe * 0.5f);
        xj = (xj * ploop) + (xe * 0.5f);
        xb = (xj * pmove) + (xn * pmove);
        if (xe > 1.0e4f) {
            const float inv = 1.0f / xe;
            xn *= inv;
            xc *= inv;
            xj *= inv;
            xb *= inv;
            const __m128 iv = _mm_set1_ps(inv);
            for (int q = 0; q < nq; q++) {
                mm[q] = _mm_mul_ps(mm[q], iv);
                dm[q] = _mm_mul_ps(dm[q], iv);
                im[q] = _mm_mul_ps(im[q], iv);
            }
            totscale += (float)log((double)xe);
        }
    }
    free(mm);
    free(dm);
    free(im);
    if (ret_totscale) *ret_totscale = totscale;
    if (ret_xc) *ret_xc = xc;
    return (float)((double)totscale + log((double)xc * (double)pmove));
}
#endif

/* build_bias_filter (src/cm_pipeline.rs:1683-1720) */
static void bias_build(const float *compo, int m, float *eo /* [KP][2] */, float *t1 /* [3] */) {
    const float bg = 0.25f;
    const float l1 = (float)m / 8.0f;
    for (int code = 0; code < KP; code++) {
        eo[code * 2 + 0] = 1.0f;
        int set[4];
        int n = fwd_degen(code, set);
        if (n == 0) {
            eo[code * 2 + 1] = 1.0f;
        } else {
            float num = 0.0f, den = 0.0f;
            for (int q = 0; q < n; q++) {
                num += compo[set[q]];
                den += bg;
            }
            eo[code * 2 + 1] = den > 0.0f ? num / den : 0.0f;
        }
    }
    t1[0] = 1.0f / (l1 + 1.0f);
    t1[1] = l1 / (l1 + 1.0f);
    t1[2] = 1.0f;
}

/* bias_filter_score (src/cm_pipeline.rs:1722-1790); *rows = the sum of the
 * per-row logs and the end term, before the length term. */
static float bias_score(const float *eo, const float *t1, const uint8_t *dsq, int L, float *rows) {
    if (L == 0) {
        if (rows) *rows = 0.0f;
        return 0.0f;
    }
    const float lf = (float)L;
    const float p1 = lf / (lf + 1.0f);
    const float t[2][3] = {{p1, 1.0f - p1, 1.0f}, {t1[0], t1[1], t1[2]}};
    const float pi[2] = {0.999f, 0.001f};
    float logsc = 0.0f;
    int x = dsq[1];
    float dp[2] = {eo[x * 2 + 0] * pi[0], eo[x * 2 + 1] * pi[1]};
    float mx = fmaxf(dp[0], dp[1]);
    dp[0] /= mx;
    dp[1] /= mx;
    logsc += (float)log((double)mx);
    for (int i = 2; i <= L; i++) {
        x = dsq[i];
        float nd[2];
        for (int k = 0; k < 2; k++) {
            float s = 0.0f;
            for (int mm = 0; mm < 2; mm++) s += dp[mm] * t[mm][k];
            nd[k] = s * eo[x * 2 + k];
        }
        mx = fmaxf(nd[0], nd[1]);
        dp[0] = nd[0] / mx;
        dp[1] = nd[1] / mx;
        logsc += (float)log((double)mx);
    }
    const float end = dp[0] * t[0][2] + dp[1] * t[1][2];
    logsc += (float)log((double)end);
    if (rows) *rows = logsc;
    return logsc + lf * logf(p1) + logf(1.0f - p1);
}

/* ---- exported ---------------------------------------------------------- */

/* the profile's natural arrays: rfv[(m+1)*KP], tr[(m+1)*8] = tbm, amm, aim,
 * adm, tmi, tii, tmd, tdd */
int oracle_fwd_tables(int m, const float *mat, const float *trans, float *rfv, float *tr) {
    fwdf f;
    fwd_build(m, mat, trans, &f);
    memcpy(rfv, f.rfv, sizeof(float) * (size_t)(m + 1) * KP);
    const float *arr[8] = {f.tbm, f.amm, f.aim, f.adm, f.tmi, f.tii, f.tmd, f.tdd};
    for (int k = 0; k <= m; k++)
        for (int a = 0; a < 8; a++) tr[k * 8 + a] = arr[a][k];
    fwd_free(&f);
    return 0;
}

/* forward_filter_score on residues 1..lens[w] of the frame at buf + offs[w]
 * (index 0 is the leading sentinel); totscale / xc may be NULL.  The
 * vectorised engine where the compiler has SSE2 (every x86-64), else the
 * lane-by-lane one; oracle_fwd_score_batch_scalar always the latter. */
int oracle_fwd_score_batch_scalar(int m, const float *mat, const float *trans, const uint8_t *buf,
                                  const int64_t *offs, const int32_t *lens, int32_t n, float *scores, float *totscale,
                                  float *xc) {
    fwdf f;
    fwd_build(m, mat, trans, &f);
    for (int32_t w = 0; w < n; w++)
        scores[w] = fwd_score(&f, buf + offs[w], lens[w], totscale ? totscale + w : NULL, xc ? xc + w : NULL);
    fwd_free(&f);
    return 0;
}

int oracle_fwd_score_batch(int m, const float *mat, const float *trans, const uint8_t *buf, const int64_t *offs,
                           const int32_t *lens, int32_t n, float *scores, float *totscale, float *xc) {
#ifdef __SSE2__
    fwdf f;
    fwdv v;
    fwd_build(m, mat, trans, &f);
    fwdv_build(&f, &v);
    for (int32_t w = 0; w < n; w++)
        scores[w] = fwd_score_sse(&v, buf + offs[w], lens[w], totscale ? totscale + w : NULL, xc ? xc + w : NULL);
    fwdv_free(&v);
    fwd_free(&f);
    return 0;
#else
    return oracle_fwd_score_batch_scalar(m, mat, trans, buf, offs, lens, n, scores, totscale, xc);
#endif
}

int oracle_bias_tables(const float *compo, int m, float *eo, float *t1) {
    bias_build(compo, m, eo, t1);
    return 0;
}

/* bias_filter_score per frame; rows (may be NULL) = the score before the
 * length term */
int oracle_bias_score_batch(const float *compo, int m, const uint8_t *buf, const int64_t *offs, const int32_t *lens,
                            int32_t n, float *scores, float *rows) {
    float eo[KP * 2], t1[3];
    bias_build(compo, m, eo, t1);
    for (int32_t w = 0; w < n; w++) scores[w] = bias_score(eo, t1, buf + offs[w], lens[w], rows ? rows + w : NULL);
    return 0;
}
