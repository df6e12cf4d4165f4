/*
 * p7_oracle.c -- TEST INFRASTRUCTURE ONLY.  CPU restatement of the
 * reference's P7 Viterbi filter (src/p7_vitfilter.rs): build_vit_filter
 * (:121-278) and the natural-order scalar scorer vit_score_scalar
 * (:305-385), 16-bit saturating arithmetic with -32768 as -infinity.
 * The parity checker for the GPU Viterbi filter kernel.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define KP 18
#define NEGINF (-32768)
static const double LOG2 = 0.6931471805599453;

static int16_t wordify(float scale_w, float sc) {
    if (sc == -INFINITY) return NEGINF;
    float v = roundf(scale_w * sc);
    if (v >= 32767.0f) return 32767;
    if (v <= -32768.0f) return NEGINF;
    return (int16_t)v;
}

static int16_t adds(int16_t a, int16_t b) {
    int s = (int)a + (int)b;
    return (int16_t)(s > 32767 ? 32767 : (s < -32768 ? -32768 : s));
}
static int16_t max16(int16_t a, int16_t b) { return a > b ? a : b; }
static int16_t min16(int16_t a, int16_t b) { return a < b ? a : b; }

static int degen_set(int code, int *out) {
    static const int sets[KP][5] = {{1, 0}, {1, 1}, {1, 2}, {1, 3}, {0},       {2, 0, 2},    {2, 1, 3},
                                    {2, 0, 1}, {2, 2, 3}, {2, 1, 2}, {2, 0, 3}, {3, 0, 1, 3}, {3, 1, 2, 3},
                                    {3, 0, 1, 2}, {3, 0, 2, 3}, {4, 0, 1, 2, 3}, {0}, {0}};
    int n = sets[code][0];
    for (int q = 0; q < n; q++) out[q] = sets[code][1 + q];
    return n;
}

typedef struct {
    int m;
    float scale_w;
    int16_t base_w, e_move, e_loop;
    int16_t *rwv; /* [m+1][KP] */
    int16_t *tmm, *tim, *tdm, *vbm, *tmi, *tii, *tmd, *tdd; /* [m+1] */
} vitf;

static void vit_free(vitf *f) {
    free(f->rwv);
    free(f->tmm);
    free(f->tim);
    free(f->tdm);
    free(f->vbm);
    free(f->tmi);
    free(f->tii);
    free(f->tmd);
    free(f->tdd);
}

/* build_vit_filter; mat [m+1][4], trans [m+1][7] = MM,MI,MD,IM,II,DM,DD */
static void vit_build(int m, const float *mat, const float *trans, vitf *f) {
    f->m = m;
    f->scale_w = (float)(500.0 / LOG2);
    f->base_w = 12000;
    f->rwv = (int16_t *)malloc(sizeof(int16_t) * (size_t)(m + 1) * KP);
    int16_t **arr[8] = {&f->tmm, &f->tim, &f->tdm, &f->vbm, &f->tmi, &f->tii, &f->tmd, &f->tdd};
    for (int a = 0; a < 8; a++) {
        *arr[a] = (int16_t *)malloc(sizeof(int16_t) * (size_t)(m + 1));
        for (int k = 0; k <= m; k++) (*arr[a])[k] = NEGINF;
    }
    for (int x = 0; x < KP; x++) f->rwv[x] = NEGINF;
    for (int k = 1; k <= m; k++) {
        float sc[KP];
        for (int x = 0; x < KP; x++) sc[x] = -INFINITY;
        for (int x = 0; x < 4; x++) sc[x] = (float)log((double)mat[k * 4 + x] / 0.25);
        for (int code = 4; code < KP; code++) {
            int set[4];
            int n = degen_set(code, set);
            if (n == 0) continue;
            float s = 0.0f;
            for (int q = 0; q < n; q++) s += sc[set[q]];
            sc[code] = s / (float)n;
        }
        for (int x = 0; x < KP; x++) f->rwv[k * KP + x] = wordify(f->scale_w, sc[x]);
    }
#define TR(j, t) trans[(j) * 7 + (t)]
    for (int j = 1; j < m; j++) {
        f->tmm[j] = min16(wordify(f->scale_w, (float)log((double)TR(j, 0))), 0);
        f->tim[j] = min16(wordify(f->scale_w, (float)log((double)TR(j, 3))), 0);
        f->tdm[j] = min16(wordify(f->scale_w, (float)log((double)TR(j, 5))), 0);
        f->tmi[j] = min16(wordify(f->scale_w, (float)log((double)TR(j, 1))), 0);
        f->tii[j] = min16(wordify(f->scale_w, (float)log((double)TR(j, 4))), -1);
        f->tmd[j] = min16(wordify(f->scale_w, (float)log((double)TR(j, 2))), 0);
        f->tdd[j] = min16(wordify(f->scale_w, (float)log((double)TR(j, 6))), 0);
    }
    float *occ = (float *)calloc((size_t)(m + 1), sizeof(float));
    occ[1] = TR(0, 1) + TR(0, 0);
    for (int k = 2; k <= m; k++)
        occ[k] = occ[k - 1] * (TR(k - 1, 0) + TR(k - 1, 1)) + (1.0f - occ[k - 1]) * TR(k - 1, 5);
    float z = 0.0f;
    for (int k = 1; k <= m; k++) z += occ[k] * (float)(m - k + 1);
    for (int k = 1; k <= m; k++) {
        float logv = (float)log((double)(occ[k] / z));
        f->vbm[k] = min16(wordify(f->scale_w, logv), 0);
    }
    free(occ);
#undef TR
    f->e_move = wordify(f->scale_w, -(float)LOG2);
    f->e_loop = wordify(f->scale_w, -(float)LOG2);
}

/* vit_score_scalar: returns 1 and *score, or 0 on overflow (None) */
static int vit_score(const vitf *f, const uint8_t *dsq, int l, float *score) {
    int m = f->m;
    float pmove = 3.0f / ((float)l + 3.0f);
    int16_t xw_move = wordify(f->scale_w, logf(pmove));
    size_t n = (size_t)(m + 1);
    int16_t *mp = (int16_t *)malloc(n * 2), *ip = (int16_t *)malloc(n * 2), *dp = (int16_t *)malloc(n * 2);
    int16_t *mc = (int16_t *)malloc(n * 2), *ic = (int16_t *)malloc(n * 2), *dc = (int16_t *)malloc(n * 2);
    for (size_t k = 0; k < n; k++) mp[k] = ip[k] = dp[k] = mc[k] = ic[k] = dc[k] = NEGINF;
    int16_t xn = f->base_w, xb = adds(xn, xw_move), xj = NEGINF, xc = NEGINF;
    int ok = 1;
    for (int i = 1; i <= l; i++) {
        int x = dsq[i];
        mc[0] = ic[0] = dc[0] = NEGINF;
        for (int k = 1; k <= m; k++) {
            int16_t sc = max16(max16(max16(adds(xb, f->vbm[k]), adds(mp[k - 1], f->tmm[k - 1])),
                                     adds(ip[k - 1], f->tim[k - 1])),
                               adds(dp[k - 1], f->tdm[k - 1]));
            mc[k] = adds(sc, f->rwv[k * KP + x]);
        }
        for (int k = 1; k <= m; k++) ic[k] = max16(adds(mp[k], f->tmi[k]), adds(ip[k], f->tii[k]));
        int16_t xe = NEGINF;
        for (int k = 1; k <= m; k++)
            if (mc[k] > xe) xe = mc[k];
        for (int k = 1; k <= m; k++) dc[k] = max16(adds(mc[k - 1], f->tmd[k - 1]), adds(dc[k - 1], f->tdd[k - 1]));
        if (xe >= 32767) {
            ok = 0;
            break;
        }
        xn = adds(xn, 0);
        xc = max16(xc, adds(xe, f->e_move));
        xj = max16(xj, adds(xe, f->e_loop));
        xb = max16(adds(xj, xw_move), adds(xn, xw_move));
        int16_t *t;
        t = mp; mp = mc; mc = t;
        t = ip; ip = ic; ic = t;
        t = dp; dp = dc; dc = t;
    }
    if (ok) {
        if (xc > NEGINF) {
            float ret = (float)xc + (float)xw_move - (float)f->base_w;
            ret /= f->scale_w;
            *score = ret - 3.0f;
        } else {
            *score = -INFINITY;
        }
    }
    free(mp); free(ip); free(dp); free(mc); free(ic); free(dc);
    return ok;
}

#ifdef __SSE2__
#include <emmintrin.h>

/* The same score on eight int16 lanes, striped the way the reference's SSE
 * engine lays a profile out (Q = max(2, (m-1)/8+1) vectors, lane z of vector
 * q = position q + 1 + z*Q, -32768 beyond m): M and I cells from the previous
 * row, D cells first from this row's M cells, then passes that carry D along
 * each lane and across lanes until no cell changes.  Every step is a
 * saturating add or an exact max, so the cells equal the scalar sweep's; the
 * timed CPU baseline. */
typedef struct {
    int m, q;
    __m128i *rw;                      /* [KP][Q] emissions */
    __m128i *bm, *mm, *im, *dm;       /* into position k: entry, and from k-1 */
    __m128i *mi, *ii, *md, *dd;       /* out of position k */
} vitv;

static void vitv_build(const vitf *f, vitv *v) {
    const int m = f->m, Q = m >= 1 ? ((m - 1) / 8 + 1 < 2 ? 2 : (m - 1) / 8 + 1) : 2;
    v->m = m;
    v->q = Q;
    __m128i **arr[9] = {&v->rw, &v->bm, &v->mm, &v->im, &v->dm, &v->mi, &v->ii, &v->md, &v->dd};
    for (int a = 0; a < 9; a++) *arr[a] = (__m128i *)aligned_alloc(16, sizeof(__m128i) * (size_t)Q * (a ? 1 : KP));
    for (int q = 0; q < Q; q++) {
        int16_t l[9][8], rw[KP][8];
        for (int z = 0; z < 8; z++) {
            const int k = q + 1 + z * Q;
            const int in = k <= m;
            l[1][z] = in ? f->vbm[k] : NEGINF;
            l[2][z] = in ? f->tmm[k - 1] : NEGINF;
            l[3][z] = in ? f->tim[k - 1] : NEGINF;
            l[4][z] = in ? f->tdm[k - 1] : NEGINF;
            l[5][z] = in ? f->tmi[k] : NEGINF;
            l[6][z] = in ? f->tii[k] : NEGINF;
            l[7][z] = in ? f->tmd[k] : NEGINF;
            l[8][z] = in ? f->tdd[k] : NEGINF;
            for (int x = 0; x < KP; x++) rw[x][z] = in ? f->rwv[k * KP + x] : NEGINF;
        }
        for (int a = 1; a < 9; a++) (*arr[a])[q] = _mm_loadu_si128((const __m128i *)l[a]);
        for (int x = 0; x < KP; x++) v->rw[x * Q + q] = _mm_loadu_si128((const __m128i *)rw[x]);
    }
}

static void vitv_free(vitv *v) {
    __m128i *arr[9] = {v->rw, v->bm, v->mm, v->im, v->dm, v->mi, v->ii, v->md, v->dd};
    for (int a = 0; a < 9; a++) free(arr[a]);
}

/* lane z takes lane z-1's value, lane 0 takes -infinity */
static __m128i vshift16(__m128i a) {
    return _mm_or_si128(_mm_slli_si128(a, 2), _mm_cvtsi32_si128(0x8000));
}

static int16_t hmax16(__m128i a) {
    a = _mm_max_epi16(a, _mm_shuffle_epi32(a, 0x4E));
    a = _mm_max_epi16(a, _mm_shuffle_epi32(a, 0xB1));
    a = _mm_max_epi16(a, _mm_shufflelo_epi16(a, 0xB1));
    return (int16_t)_mm_extract_epi16(a, 0);
}

static int vit_score_sse(const vitf *f, const vitv *v, const uint8_t *dsq, int l, float *score) {
    const int Q = v->q;
    const float pmove = 3.0f / ((float)l + 3.0f);
    const int16_t xw_move = wordify(f->scale_w, logf(pmove));
    __m128i *M = (__m128i *)aligned_alloc(16, sizeof(__m128i) * (size_t)Q * 3), *I = M + Q, *D = M + 2 * Q;
    const __m128i ninf = _mm_set1_epi16(NEGINF);
    for (int q = 0; q < Q; q++) M[q] = I[q] = D[q] = ninf;
    int16_t xn = f->base_w, xb = adds(xn, xw_move), xj = NEGINF, xc = NEGINF;
    int ok = 1;
    for (int i = 1; i <= l; i++) {
        const __m128i *rw = v->rw + (size_t)dsq[i] * Q;
        const __m128i xbv = _mm_set1_epi16(xb);
        __m128i mpv = vshift16(M[Q - 1]), ipv = vshift16(I[Q - 1]), dpv = vshift16(D[Q - 1]);
        __m128i dcv = ninf, xev = ninf;
        for (int q = 0; q < Q; q++) {
            __m128i sc = _mm_adds_epi16(xbv, v->bm[q]);
            sc = _mm_max_epi16(sc, _mm_adds_epi16(mpv, v->mm[q]));
            sc = _mm_max_epi16(sc, _mm_adds_epi16(ipv, v->im[q]));
            sc = _mm_max_epi16(sc, _mm_adds_epi16(dpv, v->dm[q]));
            sc = _mm_adds_epi16(sc, rw[q]);
            xev = _mm_max_epi16(xev, sc);
            mpv = M[q];
            ipv = I[q];
            dpv = D[q];
            M[q] = sc;
            I[q] = _mm_max_epi16(_mm_adds_epi16(mpv, v->mi[q]), _mm_adds_epi16(ipv, v->ii[q]));
            D[q] = dcv;
            dcv = _mm_adds_epi16(sc, v->md[q]);
        }
        /* D chains across the lanes: repeat until a pass changes nothing */
        for (int changed = 1; changed;) {
            changed = 0;
            dcv = vshift16(dcv);
            for (int q = 0; q < Q; q++) {
                const __m128i d = _mm_max_epi16(D[q], dcv);
                changed |= _mm_movemask_epi8(_mm_cmpeq_epi16(d, D[q])) != 0xFFFF;
                D[q] = d;
                dcv = _mm_adds_epi16(d, v->dd[q]);
            }
        }
        const int16_t xe = hmax16(xev);
        if (xe >= 32767) {
            ok = 0;
            break;
        }
        xn = adds(xn, 0);
        xc = max16(xc, adds(xe, f->e_move));
        xj = max16(xj, adds(xe, f->e_loop));
        xb = max16(adds(xj, xw_move), adds(xn, xw_move));
    }
    if (ok) {
        if (xc > NEGINF) {
            float ret = (float)xc + (float)xw_move - (float)f->base_w;
            ret /= f->scale_w;
            *score = ret - 3.0f;
        } else {
            *score = -INFINITY;
        }
    }
    free(M);
    return ok;
}
#endif

static int vit_batch(int m, const float *mat, const float *trans, const uint8_t *buf, const int64_t *offs,
                     const int32_t *lens, int32_t n, float *scores, uint8_t *scored, int scalar) {
    vitf f;
    vit_build(m, mat, trans, &f);
#ifdef __SSE2__
    vitv v;
    if (!scalar) vitv_build(&f, &v);
#endif
    for (int32_t q = 0; q < n; q++) {
        float s = NAN;
#ifdef __SSE2__
        scored[q] = (uint8_t)(scalar ? vit_score(&f, buf + offs[q], lens[q], &s)
                                     : vit_score_sse(&f, &v, buf + offs[q], lens[q], &s));
#else
        scored[q] = (uint8_t)vit_score(&f, buf + offs[q], lens[q], &s);
#endif
        scores[q] = scored[q] ? s : NAN;
    }
#ifdef __SSE2__
    if (!scalar) vitv_free(&v);
#endif
    vit_free(&f);
    return 0;
}

/* exported: score a batch of sequences (frames with sentinels); the
 * vectorised engine where the compiler has SSE2, the scalar sweep in
 * oracle_vit_score_batch_scalar */
int oracle_vit_score_batch(int m, const float *mat, const float *trans, const uint8_t *buf, const int64_t *offs,
                           const int32_t *lens, int32_t n, float *scores, uint8_t *scored) {
    return vit_batch(m, mat, trans, buf, offs, lens, n, scores, scored, 0);
}

int oracle_vit_score_batch_scalar(int m, const float *mat, const float *trans, const uint8_t *buf,
                                  const int64_t *offs, const int32_t *lens, int32_t n, float *scores,
                                  uint8_t *scored) {
    return vit_batch(m, mat, trans, buf, offs, lens, n, scores, scored, 1);
}

/* exported: the filter tables in the product's layout [(m+1)][26] */
int oracle_vit_tables(int m, const float *mat, const float *trans, int16_t *tab, int16_t *specials) {
    vitf f;
    vit_build(m, mat, trans, &f);
    for (int k = 0; k <= m; k++) {
        int16_t *r = tab + (size_t)k * 26;
        for (int x = 0; x < KP; x++) r[x] = k == 0 ? NEGINF : f.rwv[k * KP + x];
        r[18] = f.vbm[k];
        r[19] = f.tmm[k];
        r[20] = f.tim[k];
        r[21] = f.tdm[k];
        r[22] = f.tmi[k];
        r[23] = f.tii[k];
        r[24] = f.tmd[k];
        r[25] = f.tdd[k];
    }
    specials[0] = f.base_w;
    specials[1] = f.e_move;
    specials[2] = f.e_loop;
    vit_free(&f);
    return 0;
}
