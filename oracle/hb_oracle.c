/*
 * hb_oracle.c -- TEST INFRASTRUCTURE ONLY.  CPU restatement of the
 * reference's HMM-banded (CP9-banded) CM scanners, scalar branches
 * (src/cp9.rs):
 *   fast_cyk_scan_hb_core   :4717-5379  (F6 filter / --cyk final: CYK, MAX)
 *   fast_finside_scan_hb    :5465-6014  (F7: Inside, FLogsum)
 * over the banded matrix alpha[v][jp][dp] laid out as the reference lays it
 * out (row offsets roff(v, jp), rows of hdmax-hdmin+1 cells, IMPOSSIBLE
 * fill), states v = M-1..0, then the local begins, vsc_root, the envelope
 * and the greedy per-j report with null3 on ROOT.  Bands follow CP9Bands
 * (src/cp9.rs:1450-1495): jmin/jmax per state, hdmin/hdmax per (v, jp),
 * empty rows with hdmax < hdmin.  The parity checker for the GPU HB kernel.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/cmscan_gpu.h"

#define IMPOSSIBLE (-1.0e36f)
#define KP 18
#define ESCW 324

enum { D_ST = 0, MP_ST, ML_ST, MR_ST, IL_ST, IR_ST, S_ST, E_ST, B_ST };

float oracle_flogsum(float a, float b);
float oracle_null3(const float *null0, const float *comp, int len, float omega);

static inline int sdelta(int st) {
    return st == MP_ST ? 2 : (st == ML_ST || st == MR_ST || st == IL_ST || st == IR_ST) ? 1 : 0;
}
static inline int srdelta(int st) { return (st == MP_ST || st == MR_ST || st == IR_ST); }

/* esl_vec_fnorm of src/cp9.rs:464 (Kahan sum, sum != 0) */
static void fnorm_kahan(float *v, int n) {
    float sum = 0.0f, c = 0.0f;
    for (int i = 0; i < n; i++) {
        float y = v[i] - c;
        float t = sum + y;
        c = (t - sum) - y;
        sum = t;
    }
    if (sum != 0.0f)
        for (int i = 0; i < n; i++) v[i] /= sum;
    else
        for (int i = 0; i < n; i++) v[i] = 1.0f / (float)n;
}

typedef struct {
    const int32_t *jmin, *jmax, *hd_off, *hdmin, *hdmax;
} hbands;

#define HDMIN(v, jp) (b->hdmin[b->hd_off[v] + (jp)])
#define HDMAX(v, jp) (b->hdmax[b->hd_off[v] + (jp)])
#define ROFF(v, jp) (roff[roff_start[v] + (jp)])

static inline float comb(int inside, float cur, float cand) {
    if (inside) return oracle_flogsum(cur, cand);
    return cand > cur ? cand : cur;
}

/* returns the number of raw (not overlap-removed) hits; hits beyond cap are
 * counted, not written */
int oracle_hb_scan(const cmgpu_cm *cm, int inside, const int32_t *jmin, const int32_t *jmax, const int32_t *hd_off,
                   const int32_t *hdmin, const int32_t *hdmax, const uint8_t *dsq, int32_t i0, int32_t j0,
                   float env_cutoff, int report_hits, float cutoff, int do_null3, float *vsc_out, int64_t *envi_out,
                   int64_t *envj_out, cmgpu_hit *hits, int32_t cap) {
    const int m = cm->M;
    const hbands bb = {jmin, jmax, hd_off, hdmin, hdmax}, *b = &bb;
    const int w = j0 - i0 + 1;
    const float ninf = IMPOSSIBLE;
    int64_t *roff_start = (int64_t *)malloc(sizeof(int64_t) * (size_t)m);
    int64_t nrows = 0;
    for (int v = 0; v < m; v++) nrows += jmax[v] >= jmin[v] ? jmax[v] - jmin[v] + 1 : 0;
    int64_t *roff = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nrows + 1));
    int64_t ncells = 0, r = 0;
    for (int v = 0; v < m; v++) {
        int nj = jmax[v] >= jmin[v] ? jmax[v] - jmin[v] + 1 : 0;
        roff_start[v] = r;
        for (int jp = 0; jp < nj; jp++) {
            roff[r++] = ncells;
            int width = HDMAX(v, jp) - HDMIN(v, jp) + 1;
            if (width > 0) ncells += width;
        }
    }
    float *alpha = (float *)malloc(sizeof(float) * (size_t)(ncells + 1));
    for (int64_t q = 0; q < ncells; q++) alpha[q] = IMPOSSIBLE;
    float *el_sca = (float *)malloc(sizeof(float) * (size_t)(w + 1));
    for (int d = 0; d <= w; d++) el_sca[d] = cm->el_selfsc * (float)d;

    for (int v = m - 1; v >= 0; v--) {
        const int stt = cm->sttype[v], sd = sdelta(stt), sdr = srdelta(stt);
        const int cfirst = cm->cfirst[v], cnum = cm->cnum[v];
        const float *tsc = cm->tsc + (size_t)v * 6, *oesc = cm->oesc + (size_t)v * ESCW;
        if (cm->endsc[v] > -9.999e35f) {
            for (int j = jmin[v]; j <= jmax[v]; j++) {
                int jp = j - jmin[v], dpv = 0;
                for (int d = HDMIN(v, jp); d <= HDMAX(v, jp); d++, dpv++) {
                    int dp = d - sd > 0 ? d - sd : 0;
                    alpha[ROFF(v, jp) + dpv] = el_sca[dp] + cm->endsc[v];
                }
            }
        }
        if (stt == E_ST) {
            for (int j = jmin[v]; j <= jmax[v]; j++) alpha[ROFF(v, j - jmin[v])] = 0.0f;
        } else if (stt == IL_ST || stt == IR_ST) {
            for (int j = jmin[v]; j <= jmax[v]; j++) {
                const int jp = j - jmin[v], jsdr = j - sdr;
                for (int d = HDMIN(v, jp); d <= HDMAX(v, jp); d++) {
                    const int i = j - d + 1, dpv = d - HDMIN(v, jp);
                    float best = alpha[ROFF(v, jp) + dpv];
                    for (int yo = 0; yo < cnum; yo++) {
                        const int y = cfirst + yo;
                        if (jsdr < jmin[y] || jsdr > jmax[y]) continue;
                        const int jpy = jsdr - jmin[y];
                        if (d - sd >= HDMIN(y, jpy) && d - sd <= HDMAX(y, jpy))
                            best = comb(inside, best, alpha[ROFF(y, jpy) + (d - sd - HDMIN(y, jpy))] + tsc[yo]);
                    }
                    best += stt == IL_ST ? oesc[dsq[i]] : oesc[dsq[j]];
                    if (best < ninf) best = ninf;
                    alpha[ROFF(v, jp) + dpv] = best;
                }
            }
        } else if (stt != B_ST) {
            for (int yo = 0; yo < cnum; yo++) {
                const int y = cfirst + yo;
                const float t = tsc[yo];
                const int jn = jmin[v] > jmin[y] + sdr ? jmin[v] : jmin[y] + sdr;
                const int jx = jmax[v] < jmax[y] + sdr ? jmax[v] : jmax[y] + sdr;
                for (int j = jn; j <= jx; j++) {
                    const int jpv = j - jmin[v], jpy = j - jmin[y] - sdr;
                    const int dn = HDMIN(v, jpv) > HDMIN(y, jpy) + sd ? HDMIN(v, jpv) : HDMIN(y, jpy) + sd;
                    const int dx = HDMAX(v, jpv) < HDMAX(y, jpy) + sd ? HDMAX(v, jpv) : HDMAX(y, jpy) + sd;
                    for (int d = dn; d <= dx; d++) {
                        float *av = &alpha[ROFF(v, jpv) + (d - HDMIN(v, jpv))];
                        *av = comb(inside, *av, alpha[ROFF(y, jpy) + (d - sd - HDMIN(y, jpy))] + t);
                    }
                }
            }
            for (int j = jmin[v]; j <= jmax[v]; j++) {
                const int jp = j - jmin[v];
                for (int d = HDMIN(v, jp); d <= HDMAX(v, jp); d++) {
                    float *av = &alpha[ROFF(v, jp) + (d - HDMIN(v, jp))];
                    const int i = j - d + 1;
                    if (stt == ML_ST) *av += oesc[dsq[i]];
                    else if (stt == MR_ST) *av += oesc[dsq[j]];
                    else if (stt == MP_ST) *av += oesc[dsq[i] * KP + dsq[j]];
                    if (*av < ninf) *av = ninf;
                }
            }
        } else {
            const int y = cfirst, z = cnum;
            const int jn = jmin[v] > jmin[z] ? jmin[v] : jmin[z];
            const int jx = jmax[v] < jmax[z] ? jmax[v] : jmax[z];
            for (int j = jn; j <= jx; j++) {
                const int jpv = j - jmin[v], jpy = j - jmin[y], jpz = j - jmin[z];
                const int hz = HDMIN(z, jpz);
                int kn = j - jmax[y] > hz ? j - jmax[y] : hz;
                if (kn < 0) kn = 0;
                const int kx = jpy < HDMAX(z, jpz) ? jpy : HDMAX(z, jpz);
                for (int d = HDMIN(v, jpv); d <= HDMAX(v, jpv); d++) {
                    float *av = &alpha[ROFF(v, jpv) + (d - HDMIN(v, jpv))];
                    float cur = *av;
                    for (int k = kn; k <= kx; k++) {
                        const int jpyk = jpy - k;
                        if (k >= d - HDMAX(y, jpyk) && k <= d - HDMIN(y, jpyk)) {
                            float a = alpha[ROFF(y, jpyk) + (d - HDMIN(y, jpyk) - k)];
                            float c = alpha[ROFF(z, jpz) + (k - hz)];
                            cur = comb(inside, cur, a + c);
                        }
                    }
                    *av = cur;
                }
            }
        }
    }

    /* act: canonical residue counts over dsq[i0 .. i0+jp-1] */
    double(*act)[4] = (double(*)[4])calloc((size_t)w + 1, sizeof(double[4]));
    if (report_hits && do_null3)
        for (int jp = 1; jp <= w; jp++) {
            memcpy(act[jp], act[jp - 1], sizeof(double[4]));
            int res = dsq[i0 + jp - 1];
            if (res < 4) act[jp][res] += 1.0;
        }
    float vsc = ninf;
    int64_t envi = (int64_t)j0 + 1, envj = (int64_t)i0 - 1;
    const int local_begin = (cm->flags >> 10) & 1;
    int nh = 0;
    float *bestsc = (float *)malloc(sizeof(float) * (size_t)(w + 1));
    for (int d = 0; d <= w; d++) bestsc[d] = ninf;
    for (int j = jmin[0]; j <= jmax[0]; j++) {
        const int jp = j - jmin[0];
        if (local_begin)
            for (int y = 1; y < m; y++) {
                if (!(cm->beginsc[y] > -9.999e35f && j >= jmin[y] && j <= jmax[y])) continue;
                const int jpy = j - jmin[y];
                const int dn = HDMIN(0, jp) > HDMIN(y, jpy) ? HDMIN(0, jp) : HDMIN(y, jpy);
                const int dx = HDMAX(0, jp) < HDMAX(y, jpy) ? HDMAX(0, jp) : HDMAX(y, jpy);
                for (int d = dn; d <= dx; d++) {
                    float *av = &alpha[ROFF(0, jp) + (d - HDMIN(0, jp))];
                    float sc = alpha[ROFF(y, jpy) + (d - HDMIN(y, jpy))] + cm->beginsc[y];
                    if (sc > *av) *av = sc;
                }
            }
        for (int d = HDMIN(0, jp); d <= HDMAX(0, jp); d++) {
            float sc = alpha[ROFF(0, jp) + (d - HDMIN(0, jp))];
            if (report_hits) bestsc[d] = sc;
            if (sc > vsc) vsc = sc;
        }
        for (int d = HDMIN(0, jp); d <= HDMAX(0, jp); d++) {
            float sc = alpha[ROFF(0, jp) + (d - HDMIN(0, jp))];
            if (sc >= env_cutoff) {
                int i = j - d + 1;
                if (i < envi) envi = i;
                if (j > envj) envj = j;
            }
        }
        if (report_hits) {
            const int dmin = HDMIN(0, jp), dmax = HDMAX(0, jp);
            if (dmin <= dmax) {
                float max_rep = ninf;
                for (int d = dmin > 1 ? dmin : 1; d <= dmax; d++) {
                    const int i = j - d + 1;
                    float hit_sc = bestsc[d];
                    if (hit_sc > max_rep && hit_sc >= cutoff && hit_sc > -9.999e35f) {
                        int rep = 1;
                        float bias = 0.0f;
                        if (do_null3) {
                            float comp[4];
                            const int ip = i - i0 + 1, jq = j - i0 + 1;
                            for (int a = 0; a < 4; a++) comp[a] = (float)(act[jq][a] - act[ip - 1][a]);
                            fnorm_kahan(comp, 4);
                            float corr = oracle_null3(cm->null, comp, d, cm->n3_omega);
                            hit_sc -= corr;
                            bias = corr;
                            rep = hit_sc > max_rep && hit_sc >= cutoff;
                        }
                        if (rep) {
                            if (nh < cap) {
                                hits[nh].i = i;
                                hits[nh].j = j;
                                hits[nh].score = hit_sc;
                                hits[nh].bias = bias;
                            }
                            nh++;
                            max_rep = hit_sc;
                        }
                    }
                }
            }
            for (int d = 0; d <= w; d++) bestsc[d] = ninf;
        }
    }
    *vsc_out = vsc;
    *envi_out = envi == (int64_t)j0 + 1 ? -1 : envi;
    *envj_out = envj == (int64_t)i0 - 1 ? -1 : envj;
    free(bestsc);
    free(act);
    free(el_sca);
    free(alpha);
    free(roff);
    free(roff_start);
    return nh;
}
