/*
 * tr_oracle.c -- TEST INFRASTRUCTURE ONLY.  CPU restatement of the
 * reference's HMM-banded truncated scanners (src/cm_dpsearch_trunc.rs):
 *   tr_cyk_scan_hb        :264-1029  (TrCYK, ESL_MAX)
 *   ftr_inside_scan_hb    :1055-1799 (TrInside: FLogsum for every child,
 *                                     split and inherit combine; MAX for the
 *                                     ROOT truncated begins and vsc_root)
 *   report_hits_greedily  :2322-2374, allow_truncation :2376-2440,
 *   remove_overlaps_greedy_tr :2470-2496, fill_from_pass_idx :186-203.
 * Four planes J/L/R/T over the same banded layout as the standard HB scan
 * (row offsets, IMPOSSIBLE fill), states v = M-1..1 in the reference's loop
 * structure, then ROOT's truncated begins and the report.  The per-pass
 * inputs the reference selects inside the scanner (marginal emissions,
 * truncation penalties of the pass, the node spans allow_truncation reads,
 * the per-state J/L/R/T validity of the bands) are arguments.  The parity
 * checker for the GPU truncated kernel.
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
enum { TRMODE_T = 0, TRMODE_R = 1, TRMODE_L = 2, TRMODE_J = 3, TRMODE_UNKNOWN = 4 };

float oracle_flogsum(float a, float b);
float oracle_null3(const float *null0, const float *comp, int len, float omega);

static inline int sdelta(int st) {
    return st == MP_ST ? 2 : (st == ML_ST || st == MR_ST || st == IL_ST || st == IR_ST) ? 1 : 0;
}
static inline int srdelta(int st) { return (st == MP_ST || st == MR_ST || st == IR_ST); }
static inline int sldelta(int st) { return (st == MP_ST || st == ML_ST || st == IL_ST); }
static inline int notimp(float x) { return x > IMPOSSIBLE + 1.0f; }

static int g_ins;
/* the combine of a child / split / inherit term */
static inline void comb(float *a, float c) {
    if (g_ins)
        *a = oracle_flogsum(*a, c);
    else if (c > *a)
        *a = c;
}

typedef struct {
    int32_t i, j;
    float score, bias;
    int32_t mode, root;
} trhit;

static void fnorm4(float *v) {
    float sum = 0.0f;
    for (int a = 0; a < 4; a++) sum += v[a];
    if (sum > 0.0f)
        for (int a = 0; a < 4; a++) v[a] /= sum;
    else
        for (int a = 0; a < 4; a++) v[a] = 0.25f;
}

static int allow_trunc(int pass_idx, int local, const int32_t *lpos, const int32_t *rpos, int clen, int64_t start,
                       int64_t stop, int64_t i0, int64_t j0, int mode, int b) {
    if (pass_idx == 1 || pass_idx == 5) return 1; /* STD_ANY, 5P_AND_3P_ANY */
    if (start == i0 && stop == j0) return 1;
    const int lp = lpos[b], rp = rpos[b];
    if (local) {
        if (mode == TRMODE_J) return 1;
        if (mode == TRMODE_L) return stop == j0;
        if (mode == TRMODE_R) return start == i0;
        return 0;
    }
    if (mode == TRMODE_J) return lp == 1 && rp == clen;
    if (mode == TRMODE_L) return stop == j0 && lp == 1;
    if (mode == TRMODE_R) return start == i0 && rp == clen;
    return 0;
}

static int cmp_trhit(const void *a, const void *b) {
    const trhit *x = (const trhit *)a, *y = (const trhit *)b;
    if (x->score != y->score) return x->score > y->score ? -1 : 1;
    return (x->i > y->i) - (x->i < y->i);
}

/* stable sort by (score desc, i asc): insertion on an index-tagged copy */
static void sort_trhits(trhit *h, int n) {
    for (int a = 1; a < n; a++) {
        trhit t = h[a];
        int b = a - 1;
        while (b >= 0 && cmp_trhit(&h[b], &t) > 0) {
            h[b + 1] = h[b];
            b--;
        }
        h[b + 1] = t;
    }
}

#define HMN(v, jp) (hdmin[hd_off[v] + (jp)])
#define HMX(v, jp) (hdmax[hd_off[v] + (jp)])
#define RB(v, jp) (roff[roff_start[v] + (jp)])

/* returns the number of hits after overlap removal (written up to cap) */
int oracle_tr_hb_scan(const cmgpu_cm *cm, int inside, const float *lmesc, const float *rmesc, const float *pty,
                      const int32_t *lpos, const int32_t *rpos, int32_t clen, const uint8_t *jvalid,
                      const uint8_t *lvalid, const uint8_t *rvalid, const uint8_t *tvalid, const int32_t *jmin,
                      const int32_t *jmax, const int32_t *hd_off, const int32_t *hdmin, const int32_t *hdmax,
                      const uint8_t *dsq, int32_t i0, int32_t j0, float cutoff, int do_null3, int pass_idx,
                      float env_cutoff, int local, float *vsc_out, int32_t *vmode_out, int64_t *envi_out,
                      int64_t *envj_out, trhit *hits_out, int32_t cap) {
    g_ins = inside;
    const int m = cm->M;
    const int fill_l = pass_idx == 4 || pass_idx == 5 || pass_idx == 3;
    const int fill_r = pass_idx == 4 || pass_idx == 5 || pass_idx == 2;
    const int fill_t = pass_idx == 4 || pass_idx == 5;
    const int ww = j0 - i0 + 1;
    const float ninf = IMPOSSIBLE;
    float *el_sca = (float *)malloc(sizeof(float) * (size_t)(ww + 1));
    for (int d = 0; d <= ww; d++) el_sca[d] = cm->el_selfsc * (float)d;
    int64_t *roff_start = (int64_t *)malloc(sizeof(int64_t) * (size_t)m);
    int64_t nrows = 0;
    for (int v = 0; v < m; v++) nrows += jmax[v] >= jmin[v] ? jmax[v] - jmin[v] + 1 : 0;
    int64_t *roff = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nrows + 1));
    int64_t ncells = 0, r = 0;
    for (int v = 0; v < m; v++) {
        const int nj = jmax[v] >= jmin[v] ? jmax[v] - jmin[v] + 1 : 0;
        roff_start[v] = r;
        for (int jp = 0; jp < nj; jp++) {
            roff[r++] = ncells;
            const int width = HMX(v, jp) - HMN(v, jp) + 1;
            if (width > 0) ncells += width;
        }
    }
    float *ja = (float *)malloc(sizeof(float) * (size_t)(ncells + 1));
    float *la = (float *)malloc(sizeof(float) * (size_t)(ncells + 1));
    float *ra = (float *)malloc(sizeof(float) * (size_t)(ncells + 1));
    float *ta = (float *)malloc(sizeof(float) * (size_t)(ncells + 1));
    for (int64_t q = 0; q <= ncells; q++) ja[q] = la[q] = ra[q] = ta[q] = ninf;
    double(*act)[4] = (double(*)[4])calloc((size_t)ww + 1, sizeof(double[4]));
    if (do_null3)
        for (int j = i0; j <= j0; j++) {
            const int jp = j - i0 + 1;
            memcpy(act[jp], act[jp - 1], sizeof(double[4]));
            if (dsq[j] < 4) act[jp][dsq[j]] += 1.0;
        }

    for (int v = m - 1; v >= 1; v--) {
        const int stt = cm->sttype[v], sd = sdelta(stt), sdl = sldelta(stt), sdr = srdelta(stt);
        const int cfirst = cm->cfirst[v], cnum = cm->cnum[v];
        const float *esc = cm->oesc + (size_t)v * ESCW, *tsc = cm->tsc + (size_t)v * 6;
        const float *lm = lmesc + (size_t)v * KP, *rm = rmesc + (size_t)v * KP;
        const int do_j_v = jvalid[v], do_l_v = lvalid[v] && fill_l, do_r_v = rvalid[v] && fill_r,
                  do_t_v = tvalid[v] && fill_t;
        if (notimp(cm->endsc[v])) {
            for (int j = jmin[v]; j <= jmax[v]; j++) {
                const int jp = j - jmin[v];
                const int64_t base = RB(v, jp);
                const int hmn = HMN(v, jp), hmx = HMX(v, jp);
                if (do_j_v)
                    for (int d = hmn >= sd ? hmn : sd; d <= hmx; d++) ja[base + d - hmn] = el_sca[d - sd] + cm->endsc[v];
                if (do_l_v)
                    for (int d = hmn >= sdl ? hmn : sdl; d <= hmx; d++) la[base + d - hmn] = el_sca[d - sdl] + cm->endsc[v];
                if (do_r_v)
                    for (int d = hmn >= sdr ? hmn : sdr; d <= hmx; d++) ra[base + d - hmn] = el_sca[d - sdr] + cm->endsc[v];
            }
        }
        if (stt == E_ST) {
            for (int j = jmin[v]; j <= jmax[v]; j++) {
                const int64_t base = RB(v, j - jmin[v]);
                if (do_j_v) ja[base] = 0.0f;
                if (do_l_v) la[base] = 0.0f;
                if (do_r_v) ra[base] = 0.0f;
            }
        } else if (stt == ML_ST || stt == IL_ST) {
            for (int j = jmin[v]; j <= jmax[v]; j++) {
                const int jp = j - jmin[v], jsdr = j - sdr;
                const int64_t bv = RB(v, jp);
                const int hmn = HMN(v, jp);
                for (int d = hmn; d <= HMX(v, jp); d++) {
                    const int i = j - d + 1;
                    const int64_t c = bv + d - hmn;
                    if (do_j_v || do_l_v) {
                        for (int yo = 0; yo < cnum; yo++) {
                            const int y = cfirst + yo;
                            if (jsdr < jmin[y] || jsdr > jmax[y]) continue;
                            const int do_j_y = jvalid[y], do_l_y = lvalid[y] && fill_l;
                            if (!(do_j_y || do_l_y)) continue;
                            const int jpy = jsdr - jmin[y];
                            if (d - sd >= HMN(y, jpy) && d - sd <= HMX(y, jpy)) {
                                const int64_t cy = RB(y, jpy) + (d - sd - HMN(y, jpy));
                                if (do_j_v && do_j_y) comb(&ja[c], ja[cy] + tsc[yo]);
                                if (do_l_v && do_l_y) comb(&la[c], la[cy] + tsc[yo]);
                            }
                        }
                        if (do_j_v) {
                            ja[c] += esc[dsq[i]];
                            if (ja[c] < ninf) ja[c] = ninf;
                        }
                        if (do_l_v) {
                            const float e = esc[dsq[i]];
                            la[c] = d >= 2 ? la[c] + e : e;
                            if (la[c] < ninf) la[c] = ninf;
                        }
                    }
                    if (do_r_v) {
                        float rsc = ra[c];
                        for (int yo = 0; yo < cnum; yo++) {
                            const int y = cfirst + yo;
                            if (jsdr < jmin[y] || jsdr > jmax[y]) continue;
                            const int do_r_y = rvalid[y] && fill_r, do_j_y = jvalid[y];
                            if (!((do_j_y || do_r_y) && y != v)) continue;
                            const int jpy = jsdr - jmin[y];
                            if (d >= HMN(y, jpy) && d <= HMX(y, jpy)) {
                                const int64_t cy = RB(y, jpy) + (d - HMN(y, jpy));
                                if (do_j_y) comb(&rsc, ja[cy] + tsc[yo]);
                                if (do_r_y) comb(&rsc, ra[cy] + tsc[yo]);
                            }
                        }
                        ra[c] = rsc;
                    }
                }
            }
        } else if (stt == MR_ST || stt == IR_ST) {
            if (do_j_v || do_r_v)
                for (int j = jmin[v]; j <= jmax[v]; j++) {
                    const int jp = j - jmin[v], jsdr = j - sdr;
                    const int64_t bv = RB(v, jp);
                    const int hmn = HMN(v, jp);
                    for (int d = hmn; d <= HMX(v, jp); d++) {
                        const int64_t c = bv + d - hmn;
                        for (int yo = 0; yo < cnum; yo++) {
                            const int y = cfirst + yo;
                            if (jsdr < jmin[y] || jsdr > jmax[y]) continue;
                            const int do_j_y = jvalid[y], do_r_y = rvalid[y] && fill_r;
                            if (!(do_j_y || do_r_y)) continue;
                            const int jpy = jsdr - jmin[y];
                            if (d - sd >= HMN(y, jpy) && d - sd <= HMX(y, jpy)) {
                                const int64_t cy = RB(y, jpy) + (d - sd - HMN(y, jpy));
                                if (do_j_v && do_j_y) comb(&ja[c], ja[cy] + tsc[yo]);
                                if (do_r_v && do_r_y) comb(&ra[c], ra[cy] + tsc[yo]);
                            }
                        }
                        if (do_j_v) {
                            ja[c] += esc[dsq[j]];
                            if (ja[c] < ninf) ja[c] = ninf;
                        }
                        if (do_r_v) {
                            const float e = esc[dsq[j]];
                            ra[c] = d >= 2 ? ra[c] + e : e;
                            if (ra[c] < ninf) ra[c] = ninf;
                        }
                    }
                }
            if (do_l_v)
                for (int j = jmin[v]; j <= jmax[v]; j++) {
                    const int jp = j - jmin[v];
                    const int64_t bv = RB(v, jp);
                    const int hmn = HMN(v, jp);
                    for (int d = hmn; d <= HMX(v, jp); d++) {
                        const int64_t c = bv + d - hmn;
                        float lsc = la[c];
                        for (int yo = 0; yo < cnum; yo++) {
                            const int y = cfirst + yo;
                            if (y == v || j < jmin[y] || j > jmax[y]) continue;
                            const int do_l_y = lvalid[y] && fill_l, do_j_y = jvalid[y];
                            if (!(do_l_y || do_j_y)) continue;
                            const int jpy = j - jmin[y];
                            if (d >= HMN(y, jpy) && d <= HMX(y, jpy)) {
                                const int64_t cy = RB(y, jpy) + (d - HMN(y, jpy));
                                if (do_j_y) comb(&lsc, ja[cy] + tsc[yo]);
                                if (do_l_y) comb(&lsc, la[cy] + tsc[yo]);
                            }
                        }
                        la[c] = lsc;
                    }
                }
        } else if (stt == MP_ST) {
            for (int yo = 0; yo < cnum; yo++) {
                const int y = cfirst + yo;
                const int do_j_y = jvalid[y], do_l_y = lvalid[y] && fill_l, do_r_y = rvalid[y] && fill_r;
                const float t = tsc[yo];
                if ((do_j_v && do_j_y) || (do_r_v && (do_j_y || do_r_y))) {
                    const int jn = jmin[v] > jmin[y] + sdr ? jmin[v] : jmin[y] + sdr;
                    const int jx = jmax[v] < jmax[y] + sdr ? jmax[v] : jmax[y] + sdr;
                    for (int j = jn; j <= jx; j++) {
                        const int jpv = j - jmin[v], jpy = j - jmin[y] - sdr;
                        const int64_t bv = RB(v, jpv), by = RB(y, jpy);
                        if (do_j_v && do_j_y) {
                            const int dn = HMN(v, jpv) > HMN(y, jpy) + sd ? HMN(v, jpv) : HMN(y, jpy) + sd;
                            const int dx = HMX(v, jpv) < HMX(y, jpy) + sd ? HMX(v, jpv) : HMX(y, jpy) + sd;
                            for (int d = dn; d <= dx; d++)
                                comb(&ja[bv + d - HMN(v, jpv)], ja[by + d - sd - HMN(y, jpy)] + t);
                        }
                        if (do_r_v && (do_r_y || do_j_y)) {
                            const int dn = HMN(v, jpv) > HMN(y, jpy) + sdr ? HMN(v, jpv) : HMN(y, jpy) + sdr;
                            const int dx = HMX(v, jpv) < HMX(y, jpy) + sdr ? HMX(v, jpv) : HMX(y, jpy) + sdr;
                            for (int d = dn; d <= dx; d++) {
                                const int64_t cv = bv + d - HMN(v, jpv), cy = by + d - sdr - HMN(y, jpy);
                                if (do_j_y) comb(&ra[cv], ja[cy] + t);
                                if (do_r_y) comb(&ra[cv], ra[cy] + t);
                            }
                        }
                    }
                }
                if (do_l_v && (do_l_y || do_j_y)) {
                    const int jn = jmin[v] > jmin[y] ? jmin[v] : jmin[y];
                    const int jx = jmax[v] < jmax[y] ? jmax[v] : jmax[y];
                    for (int j = jn; j <= jx; j++) {
                        const int jpv = j - jmin[v], jpy = j - jmin[y];
                        const int dn = HMN(v, jpv) > HMN(y, jpy) + sdr ? HMN(v, jpv) : HMN(y, jpy) + sdr;
                        const int dx = HMX(v, jpv) < HMX(y, jpy) + sdr ? HMX(v, jpv) : HMX(y, jpy) + sdr;
                        const int64_t bv = RB(v, jpv), by = RB(y, jpy);
                        for (int d = dn; d <= dx; d++) {
                            const int64_t cv = bv + d - HMN(v, jpv), cy = by + d - sdr - HMN(y, jpy);
                            if (do_j_y) comb(&la[cv], ja[cy] + t);
                            if (do_l_y) comb(&la[cv], la[cy] + t);
                        }
                    }
                }
            }
            for (int j = jmin[v]; j <= jmax[v]; j++) {
                const int jp = j - jmin[v];
                const int64_t bv = RB(v, jp);
                for (int d = HMN(v, jp); d <= HMX(v, jp); d++) {
                    const int i = j - d + 1;
                    const int64_t c = bv + d - HMN(v, jp);
                    if (d >= 2) {
                        if (do_j_v) ja[c] += esc[dsq[i] * KP + dsq[j]];
                        if (do_l_v) la[c] += lm[dsq[i]];
                        if (do_r_v) ra[c] += rm[dsq[j]];
                    } else {
                        if (do_j_v) ja[c] = ninf;
                        if (do_l_v) la[c] = lm[dsq[i]];
                        if (do_r_v) ra[c] = rm[dsq[j]];
                    }
                    if (do_j_v && ja[c] < ninf) ja[c] = ninf;
                    if (do_l_v && la[c] < ninf) la[c] = ninf;
                    if (do_r_v && ra[c] < ninf) ra[c] = ninf;
                }
            }
        } else if (stt != B_ST) {
            for (int yo = 0; yo < cnum; yo++) {
                const int y = cfirst + yo;
                const int do_j_y = jvalid[y], do_l_y = lvalid[y] && fill_l, do_r_y = rvalid[y] && fill_r;
                const float t = tsc[yo];
                if (!((do_j_v && do_j_y) || (do_l_v && do_l_y) || (do_r_v && do_r_y))) continue;
                const int jn = jmin[v] > jmin[y] + sdr ? jmin[v] : jmin[y] + sdr;
                const int jx = jmax[v] < jmax[y] + sdr ? jmax[v] : jmax[y] + sdr;
                for (int j = jn; j <= jx; j++) {
                    const int jpv = j - jmin[v], jpy = j - jmin[y] - sdr;
                    const int dn = HMN(v, jpv) > HMN(y, jpy) + sd ? HMN(v, jpv) : HMN(y, jpy) + sd;
                    const int dx = HMX(v, jpv) < HMX(y, jpy) + sd ? HMX(v, jpv) : HMX(y, jpy) + sd;
                    const int64_t bv = RB(v, jpv), by = RB(y, jpy);
                    for (int d = dn; d <= dx; d++) {
                        const int64_t cv = bv + d - HMN(v, jpv), cy = by + d - sd - HMN(y, jpy);
                        if (do_j_v && do_j_y) comb(&ja[cv], ja[cy] + t);
                        if (do_l_v && do_l_y) comb(&la[cv], la[cy] + t);
                        if (do_r_v && do_r_y) comb(&ra[cv], ra[cy] + t);
                        if (d == dn && dn == 0) {
                            if (do_l_v) la[cv] = ninf;
                            if (do_r_v) ra[cv] = ninf;
                        }
                    }
                }
            }
        } else {
            const int y = cfirst, z = cnum;
            const int do_j_y = jvalid[y], do_l_y = lvalid[y] && fill_l, do_r_y = rvalid[y] && fill_r;
            const int do_j_z = jvalid[z], do_l_z = lvalid[z] && fill_l, do_r_z = rvalid[z] && fill_r;
            const int jn = jmin[v] > jmin[z] ? jmin[v] : jmin[z];
            const int jx = jmax[v] < jmax[z] ? jmax[v] : jmax[z];
            for (int j = jn; j <= jx; j++) {
                const int jpv = j - jmin[v], jpy = j - jmin[y], jpz = j - jmin[z];
                const int hz = HMN(z, jpz);
                int kn = j - jmax[y] > hz ? j - jmax[y] : hz;
                if (kn < 0) kn = 0;
                const int kx = jpy < HMX(z, jpz) ? jpy : HMX(z, jpz);
                const int64_t bv = RB(v, jpv), bz = RB(z, jpz);
                for (int d = HMN(v, jpv); d <= HMX(v, jpv); d++) {
                    const int64_t c = bv + d - HMN(v, jpv);
                    for (int k = kn; k <= kx; k++) {
                        const int jpyk = jpy - k;
                        if (!(k >= d - HMX(y, jpyk) && k <= d - HMN(y, jpyk))) continue;
                        const int64_t cy = RB(y, jpyk) + (d - HMN(y, jpyk) - k), cz = bz + (k - hz);
                        if (do_j_v && do_j_y && do_j_z) comb(&ja[c], ja[cy] + ja[cz]);
                        if (do_l_v && do_j_y && do_l_z) comb(&la[c], ja[cy] + la[cz]);
                        if (do_r_v && do_r_y && do_j_z) comb(&ra[c], ra[cy] + ja[cz]);
                        if (k != 0 && k != d && do_t_v && do_r_y && do_l_z) comb(&ta[c], ra[cy] + la[cz]);
                    }
                }
            }
            if (do_l_v && (do_j_y || do_l_y)) {
                const int jn2 = jmin[v] > jmin[y] ? jmin[v] : jmin[y];
                const int jx2 = jmax[v] < jmax[y] ? jmax[v] : jmax[y];
                for (int j = jn2; j <= jx2; j++) {
                    const int jpv = j - jmin[v], jpy = j - jmin[y];
                    const int dn = HMN(v, jpv) > HMN(y, jpy) ? HMN(v, jpv) : HMN(y, jpy);
                    const int dx = HMX(v, jpv) < HMX(y, jpy) ? HMX(v, jpv) : HMX(y, jpy);
                    for (int d = dn; d <= dx; d++) {
                        const int64_t cv = RB(v, jpv) + d - HMN(v, jpv), cy = RB(y, jpy) + d - HMN(y, jpy);
                        if (do_j_y) comb(&la[cv], ja[cy]);
                        if (do_l_y) comb(&la[cv], la[cy]);
                    }
                }
            }
            if (do_r_v && (do_j_z || do_r_z)) {
                const int jn2 = jmin[v] > jmin[z] ? jmin[v] : jmin[z];
                const int jx2 = jmax[v] < jmax[z] ? jmax[v] : jmax[z];
                for (int j = jn2; j <= jx2; j++) {
                    const int jpv = j - jmin[v], jpz = j - jmin[z];
                    const int dn = HMN(v, jpv) > HMN(z, jpz) ? HMN(v, jpv) : HMN(z, jpz);
                    const int dx = HMX(v, jpv) < HMX(z, jpz) ? HMX(v, jpv) : HMX(z, jpz);
                    for (int d = dn; d <= dx; d++) {
                        const int64_t cv = RB(v, jpv) + d - HMN(v, jpv), cz = RB(z, jpz) + d - HMN(z, jpz);
                        if (do_j_z) comb(&ra[cv], ja[cz]);
                        if (do_r_z) comb(&ra[cv], ra[cz]);
                    }
                }
            }
        }
    }

    /* ROOT: truncated begins (MAX) and the greedy report per j */
    const int do_j_0 = jvalid[0], do_l_0 = lvalid[0] && fill_l, do_r_0 = rvalid[0] && fill_r,
              do_t_0 = tvalid[0] && fill_t;
    float *bestsc = (float *)malloc(sizeof(float) * (size_t)(ww + 1));
    int32_t *bestr = (int32_t *)malloc(sizeof(int32_t) * (size_t)(ww + 1));
    int32_t *bestmode = (int32_t *)malloc(sizeof(int32_t) * (size_t)(ww + 1));
    int nh = 0, hcap = 64;
    trhit *tmp = (trhit *)malloc(sizeof(trhit) * (size_t)hcap);
    for (int j = jmin[0]; j <= jmax[0]; j++) {
        const int jp = j - jmin[0];
        const int64_t b0 = RB(0, jp);
        for (int d = 0; d <= ww; d++) {
            bestr[d] = 0;
            bestsc[d] = IMPOSSIBLE;
            bestmode[d] = TRMODE_UNKNOWN;
        }
        for (int y = 1; y < m; y++) {
            const float pen = pty[y];
            if (!(notimp(pen) && j >= jmin[y] && j <= jmax[y])) continue;
            const int do_j_y = jvalid[y], do_l_y = lvalid[y] && fill_l, do_r_y = rvalid[y] && fill_r,
                      do_t_y = tvalid[y] && fill_t;
            const int jpy = j - jmin[y];
            const int dn = HMN(0, jp) > HMN(y, jpy) ? HMN(0, jp) : HMN(y, jpy);
            const int dx = HMX(0, jp) < HMX(y, jpy) ? HMX(0, jp) : HMX(y, jpy);
            const int64_t cyb = RB(y, jpy);
            float *planes0[4] = {ja, la, ra, ta};
            const int dos[4] = {do_j_0 && do_j_y, do_l_0 && do_l_y, do_r_0 && do_r_y,
                                do_t_0 && do_t_y && cm->sttype[y] == B_ST};
            const int modes[4] = {TRMODE_J, TRMODE_L, TRMODE_R, TRMODE_T};
            for (int pl = 0; pl < 4; pl++) {
                if (!dos[pl]) continue;
                float *P = planes0[pl];
                for (int d = dn; d <= dx; d++) {
                    const float sc = P[cyb + d - HMN(y, jpy)] + pen;
                    float *a0 = &P[b0 + d - HMN(0, jp)];
                    if (sc > *a0) {
                        *a0 = sc;
                        if (sc > bestsc[d]) {
                            bestsc[d] = sc;
                            bestmode[d] = modes[pl];
                            bestr[d] = y;
                        }
                    }
                }
            }
        }
        const int dmin = HMN(0, jp), dmax = HMX(0, jp);
        if (dmin <= dmax) {
            float max_rep = IMPOSSIBLE;
            for (int d = dmin > 1 ? dmin : 1; d <= dmax; d++) {
                const int i = j - d + 1, mode = bestmode[d];
                float hit_sc = bestsc[d], bias = 0.0f;
                if (!(hit_sc > max_rep && hit_sc >= cutoff && notimp(hit_sc))) continue;
                int rep = allow_trunc(pass_idx, local, lpos, rpos, clen, i, j, i0, j0, mode, bestr[d]);
                if (rep && do_null3) {
                    float comp[4];
                    for (int a = 0; a < 4; a++) comp[a] = (float)(act[j - i0 + 1][a] - act[i - i0][a]);
                    fnorm4(comp);
                    const float corr = oracle_null3(cm->null, comp, d, cm->n3_omega);
                    hit_sc -= corr;
                    bias = corr;
                    rep = hit_sc > max_rep && hit_sc >= cutoff;
                }
                if (rep) {
                    if (nh == hcap) {
                        hcap *= 2;
                        tmp = (trhit *)realloc(tmp, sizeof(trhit) * (size_t)hcap);
                    }
                    tmp[nh].i = i;
                    tmp[nh].j = j;
                    tmp[nh].score = hit_sc;
                    tmp[nh].bias = bias;
                    tmp[nh].mode = mode;
                    tmp[nh].root = bestr[d];
                    nh++;
                    max_rep = hit_sc;
                }
            }
        }
    }
    float vsc = IMPOSSIBLE;
    int vmode = TRMODE_UNKNOWN;
    int64_t envi = (int64_t)j0 + 1, envj = (int64_t)i0 - 1;
    for (int j = jmin[0]; j <= jmax[0]; j++) {
        const int jp = j - jmin[0];
        const int64_t b0 = RB(0, jp);
        for (int d = HMN(0, jp); d <= HMX(0, jp); d++) {
            const int64_t c = b0 + d - HMN(0, jp);
            if (do_j_0 && ja[c] > vsc) { vsc = ja[c]; vmode = TRMODE_J; }
            if (do_l_0 && la[c] > vsc) { vsc = la[c]; vmode = TRMODE_L; }
            if (do_r_0 && ra[c] > vsc) { vsc = ra[c]; vmode = TRMODE_R; }
            if (do_t_0 && ta[c] > vsc) { vsc = ta[c]; vmode = TRMODE_T; }
        }
        for (int d = HMN(0, jp); d <= HMX(0, jp); d++) {
            const int64_t c = b0 + d - HMN(0, jp);
            if ((do_j_0 && ja[c] >= env_cutoff) || (do_l_0 && la[c] >= env_cutoff) ||
                (do_r_0 && ra[c] >= env_cutoff) || (do_t_0 && ta[c] >= env_cutoff)) {
                const int i = j - d + 1;
                if (i < envi) envi = i;
                if (j > envj) envj = j;
            }
        }
    }
    /* overlap removal */
    sort_trhits(tmp, nh);
    char *removed = (char *)calloc((size_t)nh + 1, 1);
    int kept = 0;
    for (int a = 0; a < nh; a++) {
        if (removed[a]) continue;
        for (int b = a + 1; b < nh; b++)
            if (!removed[b] && !(tmp[b].j < tmp[a].i) && !(tmp[a].j < tmp[b].i)) removed[b] = 1;
    }
    for (int a = 0; a < nh; a++)
        if (!removed[a]) {
            if (kept < cap) hits_out[kept] = tmp[a];
            kept++;
        }
    *vsc_out = vsc;
    *vmode_out = vmode;
    *envi_out = envi == (int64_t)j0 + 1 ? -1 : envi;
    *envj_out = envj == (int64_t)i0 - 1 ? -1 : envj;
    free(removed);
    free(tmp);
    free(bestmode);
    free(bestr);
    free(bestsc);
    free(act);
    free(ta);
    free(ra);
    free(la);
    free(ja);
    free(roff);
    free(roff_start);
    free(el_sca);
    return kept;
}
