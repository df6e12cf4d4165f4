/*
 * TEST INFRASTRUCTURE ONLY -- an independent restatement of the reference's
 * model-to-table builders, the checker of the library's host-side model
 * preparation (cmgpu_prep_configure, cmgpu_prep_truncated).  Shares no code
 * with the library.  Restated from (reference file:line):
 *   cm_config_local             src/cp9.rs:4193-4258
 *   cm_logoddsify + FCalcOptimizedEmitScores  src/cp9.rs:4263-4368
 *   build_integer_scores        src/cm_nohmm.rs:279-369
 *   cm_configure_scores(_global) src/cp9.rs:4538-4545, src/cm_nohmm.rs:264-276
 *   band_calculation_engine     src/cm_qdband.rs:258-549 (+ :150-185, :217-242)
 *   calculate_query_dependent_bands  src/cm_qdband.rs:554-592
 *   fill_marginal_emissions     src/cp9.rs:4441-4530 (+ expect scores :4370-4435)
 *   cm_expected_state_occupancy src/cp9.rs:752-838
 *   create_emit_map             src/cp9.rs:144-208
 *   TrPenalties::new            src/cm_trunc.rs:192-385 (+ :99-135)
 * Compiled with -ffp-contract=off (no fused multiply-add), like the Rust.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/cmscan_gpu.h"

#define PK 4            /* canonical alphabet */
#define PKP 18          /* digital alphabet with degeneracies */
#define PINF 987654321
#define PIMP (-1.0e36f)

enum { pD = 0, pMP, pML, pMR, pIL, pIR, pS, pE, pB };
enum { nBIF = 0, nMATP, nMATL, nMATR, nBEGL, nBEGR, nROOT, nEND };
enum { uMATP_MP = 6, uMATP_IL = 10, uMATL_ML = 12, uMATR_MR = 15, uBIF_B = 18, uEND_E = 19 };

/* which canonical residues each digital code stands for (src/cm.rs:24-43) */
static const unsigned char DEG[PKP][PK] = {
    {1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, 1, 0}, {0, 0, 0, 1}, {0, 0, 0, 0}, {1, 0, 1, 0},
    {0, 1, 0, 1}, {1, 1, 0, 0}, {0, 0, 1, 1}, {0, 1, 1, 0}, {1, 0, 0, 1}, {1, 1, 0, 1},
    {0, 1, 1, 1}, {1, 1, 1, 0}, {1, 0, 1, 1}, {1, 1, 1, 1}, {0, 0, 0, 0}, {0, 0, 0, 0}};

static int is_res(int x) { return x < PK || (x > PK && x < PKP - 2); }
static int ndeg(int x) {
    int n = 0;
    for (int i = 0; i < PK; i++) n += DEG[x][i];
    return n;
}
static float frac(int x, int l) { return DEG[x][l] ? 1.0f / (float)ndeg(x) : 0.0f; }
static double slog2(double x) { return x > 0.0 ? log(x) * 1.44269504 : -1.0e36; }
static int dlt(int st) { return st == pMP ? 2 : (st == pML || st == pMR || st == pIL || st == pIR) ? 1 : 0; }

/* Prob2Score of the scanner tables (src/cm_nohmm.rs:27-33) */
static int p2s_scan(float p, float nul) {
    if (p == 0.0f) return -PINF;
    return (int)floor(0.5 + 1000.0 * log2((double)p / (double)nul));
}
/* Prob2Score of the CP9 / truncation tables (src/cp9.rs:977-997) */
static int p2s_cp9(float p, float nul) {
    if (p == 0.0f) return -PINF;
    float r = p / nul;
    double v = floor(0.5 + 1000.0 * slog2((double)r));
    if (!isfinite(v)) return -PINF;
    if (v < -2147483648.0) v = -2147483648.0;
    if (v > 2147483647.0) v = 2147483647.0;
    int iv = (int)v;
    return iv < -PINF ? -PINF : iv;
}

/* A working copy of the probability-level model. */
typedef struct {
    const cmgpu_cm_params *p;
    int M, nodes;
    float *t;      /* [M][6], localised in place */
    float *begin, *end;
    uint32_t flags;
} pm;

static void pm_init(pm *m, const cmgpu_cm_params *p) {
    m->p = p;
    m->M = p->M;
    m->nodes = p->nodes;
    m->t = malloc(sizeof(float) * 6 * (size_t)p->M);
    memcpy(m->t, p->t, sizeof(float) * 6 * (size_t)p->M);
    m->begin = calloc((size_t)p->M, sizeof(float));
    m->end = calloc((size_t)p->M, sizeof(float));
    m->flags = 0;
}
static void pm_free(pm *m) {
    free(m->t);
    free(m->begin);
    free(m->end);
}

static int internal_start(int t) { return t == nMATP || t == nMATL || t == nMATR || t == nBIF; }

/* cm_config_local: local begins over internal node starts, state 0's
 * transitions zeroed, local ends with the Kahan-summed renormalisation. */
static void local_config(pm *m) {
    const cmgpu_cm_params *p = m->p;
    int ns = 0;
    for (int nd = 2; nd < p->nodes; nd++) ns += internal_start(p->ndtype[nd]);
    for (int v = 0; v < m->M; v++) m->begin[v] = 0.0f;
    m->begin[p->nodemap[1]] = 1.0f - p->pbegin;
    float share = p->pbegin / (float)ns;
    for (int nd = 2; nd < p->nodes; nd++)
        if (internal_start(p->ndtype[nd])) m->begin[p->nodemap[nd]] = share;
    for (int y = 0; y < p->cnum[0]; y++) m->t[y] = 0.0f;
    m->flags |= 1u << 10;
    int nx = 0;
    for (int nd = 1; nd < p->nodes; nd++) {
        int t = p->ndtype[nd];
        if ((t == nMATP || t == nMATL || t == nMATR || t == nBEGL || t == nBEGR) && p->ndtype[nd + 1] != nEND) nx++;
    }
    for (int v = 0; v < m->M; v++) m->end[v] = 0.0f;
    for (int nd = 1; nd < p->nodes; nd++) {
        int t = p->ndtype[nd];
        if (!((t == nMATP || t == nMATL || t == nMATR || t == nBEGL || t == nBEGR) && p->ndtype[nd + 1] != nEND))
            continue;
        int v = p->nodemap[nd];
        m->end[v] = p->pend / (float)nx;
        float s = 0.0f, comp = 0.0f;
        for (int x = 0; x < p->cnum[v]; x++) {
            float y = m->t[v * 6 + x] - comp;
            float tt = s + y;
            comp = (tt - s) - y;
            s = tt;
        }
        s += m->end[v];
        float inv = 1.0f / s;
        for (int x = 0; x < p->cnum[v]; x++) m->t[v * 6 + x] *= inv;
    }
    m->flags |= 1u << 11;
}

/* FAvgScore / IAvgScore of a degenerate code (src/cm.rs:84-117) */
static float favg(int x, const float *sc) {
    if (!is_res(x)) return 0.0f;
    float r = 0.0f;
    for (int i = 0; i < PK; i++)
        if (DEG[x][i]) r += sc[i];
    return r / (float)ndeg(x);
}
static int iavg(int x, const int *sc) {
    if (!is_res(x)) return 0;
    float r = 0.0f;
    for (int i = 0; i < PK; i++)
        if (DEG[x][i]) r += (float)sc[i];
    r /= (float)ndeg(x);
    return r < 0.0f ? (int)(r - 0.5f) : (int)(r + 0.5f);
}

/* Pair score of a code pair from the canonical 4x4 table, degenerate codes
 * marginalised with FCount fractions (FastPairScore*Degenerate). */
static float fpair(const float *esc, int a, int b) {
    float s = 0.0f;
    if (a > PK && b < PK) {
        for (int l = 0; l < PK; l++) s += esc[l * PK + b] * frac(a, l);
    } else if (a < PK && b > PK) {
        for (int r = 0; r < PK; r++) s += esc[a * PK + r] * frac(b, r);
    } else {
        for (int l = 0; l < PK; l++)
            for (int r = 0; r < PK; r++) s += esc[l * PK + r] * frac(a, l) * frac(b, r);
    }
    return s;
}
static int ipair(const int *iesc, int a, int b) {
    float s = 0.0f;
    if (a > PK && b < PK) {
        for (int l = 0; l < PK; l++) s += (float)iesc[l * PK + b] * frac(a, l);
    } else if (a < PK && b > PK) {
        for (int r = 0; r < PK; r++) s += (float)iesc[a * PK + r] * frac(b, r);
    } else {
        for (int l = 0; l < PK; l++)
            for (int r = 0; r < PK; r++) s += (float)iesc[l * PK + r] * frac(a, l) * frac(b, r);
    }
    return (int)s;
}

/* cm_logoddsify and build_integer_scores: tsc/oesc/beginsc/endsc and their
 * integer forms.  Unused entries keep IMPOSSIBLE / -INFTY. */
static void score_tables(const pm *m, float el_selfsc, cmgpu_cm_scores *o) {
    const cmgpu_cm_params *p = m->p;
    for (int v = 0; v < m->M; v++) {
        const int st = p->sttype[v];
        const float *e = p->e + (size_t)v * 16;
        for (int x = 0; x < 6; x++) {
            o->tsc[v * 6 + x] = PIMP;
            o->itsc[v * 6 + x] = -PINF;
        }
        for (int x = 0; x < 324; x++) {
            o->oesc[(size_t)v * 324 + x] = PIMP;
            o->ioesc[(size_t)v * 324 + x] = -PINF;
        }
        if (st != pB && st != pE)
            for (int x = 0; x < p->cnum[v]; x++) {
                o->tsc[v * 6 + x] = (float)slog2((double)m->t[v * 6 + x]);
                o->itsc[v * 6 + x] = p2s_scan(m->t[v * 6 + x], 1.0f);
            }
        if (st == pMP) {
            float esc[16];
            int iesc[16];
            for (int a = 0; a < PK; a++)
                for (int b = 0; b < PK; b++) {
                    esc[a * PK + b] = (float)slog2((double)(e[a * PK + b] / (p->null[a] * p->null[b])));
                    iesc[a * PK + b] = p2s_scan(e[a * PK + b], p->null[a] * p->null[b]);
                }
            for (int a = 0; a < PKP - 1; a++)
                for (int b = 0; b < PKP - 1; b++) {
                    if (a == PK || b == PK) continue;
                    float *fo = &o->oesc[(size_t)v * 324 + a * PKP + b];
                    int32_t *io = &o->ioesc[(size_t)v * 324 + a * PKP + b];
                    if (a < PK && b < PK) {
                        *fo = esc[a * PK + b];
                        *io = iesc[a * PK + b];
                    } else {
                        *fo = fpair(esc, a, b);
                        *io = ipair(iesc, a, b);
                    }
                }
        } else if (st == pML || st == pMR || st == pIL || st == pIR) {
            float esc[PK];
            int iesc[PK];
            for (int a = 0; a < PK; a++) {
                esc[a] = (float)slog2((double)(e[a] / p->null[a]));
                iesc[a] = p2s_scan(e[a], p->null[a]);
            }
            for (int a = 0; a < PKP - 1; a++) {
                if (a == PK) continue;
                o->oesc[(size_t)v * 324 + a] = a < PK ? esc[a] : favg(a, esc);
                o->ioesc[(size_t)v * 324 + a] = a < PK ? iesc[a] : iavg(a, iesc);
            }
        }
        o->beginsc[v] = (float)slog2((double)m->begin[v]);
        o->endsc[v] = (float)slog2((double)m->end[v]);
        o->ibeginsc[v] = p2s_scan(m->begin[v], 1.0f);
        o->iendsc[v] = p2s_scan(m->end[v], 1.0f);
    }
    o->iel_selfsc = p2s_scan(powf(2.0f, el_selfsc), 1.0f);
}

/* BandTruncationNegligible (src/cm_qdband.rs:217-242) */
static int trunc_ok(const double *dens, long b, long z) {
    if (b + 1 >= z) return 0;
    double c = 0.0;
    for (long i = b + 1; i <= z; i++) c += dens[i];
    double lb = (log(dens[z]) - log(dens[b + 1])) / (double)(z - b - 1);
    double beta = exp(lb);
    double d = (beta / (1.0 - beta)) * dens[z];
    return d < c * 2.220446049250313e-16;
}

/* band_calculation_engine on the global model: gamma_v(n) bottom-up, local
 * begins on into gamma_0, then dmin/dmax at beta1/beta2 and W at betaW.
 * Returns 0, or 1 when Z is too small. */
static int bands_at(const cmgpu_cm_params *p, long z, double b1, double b2, double bw, int *dmin1, int *dmax1,
                    int *dmin2, int *dmax2, int *W) {
    const int M = p->M;
    double maxb = bw > b1 ? bw : b1;
    maxb = maxb > b2 ? maxb : b2;
    float *bg = calloc((size_t)M, sizeof(float));
    int ns = 0;
    for (int nd = 2; nd < p->nodes; nd++) ns += internal_start(p->ndtype[nd]);
    if (p->nodes > 1) bg[p->nodemap[1]] = (float)(1.0 - (double)p->pbegin);
    if (ns > 0) {
        float sh = (float)((double)p->pbegin / (double)ns);
        for (int nd = 2; nd < p->nodes; nd++)
            if (internal_start(p->ndtype[nd])) bg[p->nodemap[nd]] = sh;
    }
    double *g = calloc((size_t)M * (size_t)(z + 1), sizeof(double));
#define G(v, n) g[(size_t)(v) * (size_t)(z + 1) + (size_t)(n)]
    int rc = 0, w = 0;
    for (int v = M - 1; v >= 0 && !rc; v--) {
        const int st = p->sttype[v];
        if (st == pE) {
            G(v, 0) = 1.0;
            dmin1[v] = dmax1[v] = dmin2[v] = dmax2[v] = 0;
            continue;
        }
        double pdf = 0.0;
        if (st == pB) {
            const int L = p->cfirst[v], R = p->cnum[v];
            for (long n = 0; n <= z; n++) {
                for (long k = 0; k <= n; k++) G(v, n) += G(L, k) * G(R, n - k);
                pdf += G(v, n);
            }
        } else if (v != 0) {
            const int d = dlt(st);
            for (long n = d; n <= z; n++) {
                for (int yo = 0; yo < p->cnum[v]; yo++)
                    G(v, n) += (double)p->t[v * 6 + yo] * G(p->cfirst[v] + yo, n - d);
                pdf += G(v, n);
            }
        }
        if (bg[v] > 0.0f && v != 0)
            for (long n = 0; n <= z; n++) G(0, n) += (double)bg[v] * G(v, n);
        if (v == 0) {
            pdf = 0.0;
            for (long n = 0; n <= z; n++) pdf += G(0, n);
        }
        if (pdf <= 0.999 || G(v, z) > maxb * 2.220446049250313e-16) {
            rc = 1;
            break;
        }
        if (pdf > 1.0)
            for (long n = 0; n <= z; n++) G(v, n) /= pdf;
        double cum = 0.0;
        int got2 = 0;
        for (long n = 0; n <= z; n++) {
            cum += G(v, n);
            if (!got2 && cum > b2) {
                dmin2[v] = (int)n;
                got2 = 1;
            }
            if (got2 && cum > b1) {
                dmin1[v] = (int)n;
                break;
            }
        }
        cum = 0.0;
        got2 = 0;
        for (long n = z; n >= 0; n--) {
            cum += G(v, n);
            if (!got2 && cum > b2) {
                dmax2[v] = (int)n;
                got2 = 1;
            }
            if (got2 && cum > b1) {
                dmax1[v] = (int)n;
                break;
            }
        }
        if (v == 0) {
            cum = 0.0;
            for (long n = z; n >= 0; n--) {
                cum += G(0, n);
                if (cum > bw) {
                    w = (int)n;
                    break;
                }
            }
        }
    }
    if (!rc) {
        double *g0 = &G(0, 0);
        if (!trunc_ok(g0, w, z) || !trunc_ok(g0, dmax1[0], z) || !trunc_ok(g0, dmax2[0], z)) rc = 1;
    }
#undef G
    free(g);
    free(bg);
    *W = w;
    return rc;
}

/* FaithfulSearcher's configuration of a CM for scanning: bands and W on the
 * global model (Z from 4 clen, doubled until the truncation is negligible),
 * then the local (cm_configure_scores) or global scores; el_selfsc clamped
 * so that el_selfsc * W stays above IMPOSSIBLE. */
int oracle_prep_configure(const cmgpu_cm_params *p, int local, int32_t W_in, double beta1, double beta2,
                          double betaW, cmgpu_cm_scores *o) {
    int W = 0;
    for (long z = 4L * p->clen;; z *= 2) {
        if (z > 1000L * p->clen) return -5;
        if (bands_at(p, z, beta1, beta2, betaW, o->dmin1, o->dmax1, o->dmin2, o->dmax2, &W) == 0) break;
    }
    if (W_in > 0) W = W_in;
    pm m;
    pm_init(&m, p);
    if (local) local_config(&m);
    float el = p->el_selfsc;
    if (el * (float)W < PIMP) el = PIMP / ((float)W + 1.0f);
    score_tables(&m, el, o);
    if (o->t_local) memcpy(o->t_local, m.t, sizeof(float) * 6 * (size_t)p->M);
    o->el_selfsc = el;
    o->W = W;
    o->flags = m.flags;
    pm_free(&m);
    return 0;
}

/* ExpectScore of a degenerate code under the background (src/cp9.rs:4370-4435) */
static float fexp_sc(int x, const float *sc, const float *bg) {
    if (!is_res(x)) return 0.0f;
    float num = 0.0f, den = 0.0f;
    for (int i = 0; i < PK; i++)
        if (DEG[x][i]) {
            num += sc[i] * bg[i];
            den += bg[i];
        }
    return num / den;
}
static int iexp_sc(int x, const int *sc, const float *bg) {
    if (!is_res(x)) return 0;
    float num = 0.0f, den = 0.0f;
    for (int i = 0; i < PK; i++)
        if (DEG[x][i]) {
            num += (float)sc[i] * bg[i];
            den += bg[i];
        }
    num /= den;
    return num < 0.0f ? (int)(num - 0.5f) : (int)(num + 0.5f);
}

/* fill_marginal_emissions: left / right marginal scores [M][18]. */
static void oracle_marginals(const cmgpu_cm_params *p, float *lm, float *rm, int32_t *ilm, int32_t *irm) {
    for (int v = 0; v < p->M; v++) {
        float *L = lm + (size_t)v * PKP, *R = rm + (size_t)v * PKP;
        int32_t *IL = ilm + (size_t)v * PKP, *IR = irm + (size_t)v * PKP;
        for (int x = 0; x < PKP; x++) {
            int dead = x == PK || x == PKP - 2 || x == PKP - 1;
            L[x] = R[x] = dead ? PIMP : 0.0f;
            IL[x] = IR[x] = dead ? -PINF : 0;
        }
        const int st = p->sttype[v];
        const float *e = p->e + (size_t)v * 16;
        if (st == pMP) {
            float sl[PK] = {0}, sr[PK] = {0};
            for (int a = 0; a < PK; a++)
                for (int b = 0; b < PK; b++) {
                    sl[a] += e[a * PK + b];
                    sr[b] += e[a * PK + b];
                }
            for (int a = 0; a < PK; a++) {
                IL[a] = p2s_cp9(sl[a], p->null[a]);
                IR[a] = p2s_cp9(sr[a], p->null[a]);
                L[a] = (float)slog2((double)(sl[a] / p->null[a]));
                R[a] = (float)slog2((double)(sr[a] / p->null[a]));
            }
            for (int x = PK + 1; x <= PKP - 3; x++) {
                L[x] = fexp_sc(x, L, p->null);
                R[x] = fexp_sc(x, R, p->null);
                IL[x] = iexp_sc(x, IL, p->null);
                IR[x] = iexp_sc(x, IR, p->null);
            }
        } else if (st == pML || st == pIL || st == pMR || st == pIR) {
            float *F = (st == pML || st == pIL) ? L : R;
            int32_t *I = (st == pML || st == pIL) ? IL : IR;
            for (int a = 0; a < PK; a++) {
                F[a] = (float)slog2((double)(e[a] / p->null[a]));
                I[a] = p2s_cp9(e[a], p->null[a]);
            }
            for (int x = PK + 1; x <= PKP - 3; x++) {
                F[x] = fexp_sc(x, F, p->null);
                I[x] = iexp_sc(x, I, p->null);
            }
        }
    }
}

/* cm_expected_state_occupancy of the global model.  The transition the
 * reference's transition map picks for parent x into v is v's offset among
 * x's children; -1 when a parent does not list v. */
static int occupancy(const cmgpu_cm_params *p, double *psi) {
    for (int v = 0; v < p->M; v++) {
        const int st = p->sttype[v];
        psi[v] = 0.0;
        if (st == pS) {
            psi[v] = 1.0;
            continue;
        }
        const int ins = st == pIL || st == pIR;
        for (int y = p->pnum[v] - 1; y >= ins; y--) {
            const int x = p->plast[v] - y, k = v - p->cfirst[x];
            if (k < 0 || k >= p->cnum[x]) return -1;
            psi[v] += psi[x] * (double)p->t[x * 6 + k];
        }
        if (ins) {
            const double s = (double)p->t[v * 6];
            psi[v] += psi[v] * (s / (1.0 - s));
        }
    }
    return 0;
}

/* create_emit_map: consensus columns per node by a depth-first walk of the
 * guide tree (left side down, right side on the way back). */
static void emitmap(const cmgpu_cm_params *p, int *lpos, int *rpos) {
    int *stk = malloc(sizeof(int) * 4 * (size_t)(p->nodes + 4));
    int top = 0, col = 0;
    for (int nd = 0; nd < p->nodes; nd++) lpos[nd] = rpos[nd] = -1;
    stk[top++] = 0;  /* left side of node 0 (encoded as 2*nd + side) */
    while (top > 0) {
        const int code = stk[--top], nd = code >> 1, right = code & 1, t = p->ndtype[nd];
        if (right) {
            rpos[nd] = col + 1;
            if (t == nMATP || t == nMATR) col++;
            continue;
        }
        if (t == nMATP || t == nMATL) col++;
        lpos[nd] = col;
        stk[top++] = 2 * nd + 1;
        if (t == nBIF) {
            const int b = p->nodemap[nd];
            stk[top++] = 2 * p->ndidx[p->cnum[b]];
            stk[top++] = 2 * p->ndidx[p->cfirst[b]];
        } else if (t != nEND) {
            stk[top++] = 2 * (nd + 1);
        }
    }
    free(stk);
}

/* Insert states of node nd (InsertsGivenNodeIndex) */
static void node_inserts(const cmgpu_cm_params *p, int nd, int *i1, int *i2) {
    *i1 = *i2 = -1;
    if (nd < 0) return;
    const int v = p->nodemap[nd];
    switch (p->ndtype[nd]) {
    case nMATP: *i1 = v + 4; *i2 = v + 5; break;
    case nMATL: case nMATR: *i1 = v + 2; break;
    case nBEGR: *i1 = v + 1; break;
    case nROOT: *i1 = v + 1; *i2 = v + 2; break;
    default: break;
    }
}

/* TrPenalties::new: the three truncated-begin rows (5'-and-3', 5'-only,
 * 3'-only) of the global (g, ig) and the local (l, il) configuration, [3][M]. */
static void penalties(const cmgpu_cm_params *p, const int *elp, const int *erp, const double *psi, float *g,
                      int32_t *ig, float *l, int32_t *il) {
    const int M = p->M, clen = p->clen;
    for (int k = 0; k < 3 * M; k++) {
        g[k] = l[k] = PIMP;
        ig[k] = il[k] = -PINF;
    }
    const float g53 = (float)(2.0 / (double)(clen * (clen + 1))), g1 = (float)(1.0 / (double)clen);
    float *bg = calloc((size_t)M, sizeof(float));
    int ns = 0;
    for (int nd = 2; nd < p->nodes; nd++) ns += internal_start(p->ndtype[nd]);
    if (p->nodes > 1) bg[p->nodemap[1]] = (float)(1.0 - (double)p->pbegin);
    const float sh = p->pbegin / (float)ns;
    for (int nd = 2; nd < p->nodes; nd++)
        if (internal_start(p->ndtype[nd])) bg[p->nodemap[nd]] = sh;
    float run5 = 0.0f, run3 = 0.0f, run53 = 0.0f;
    for (int nd = 0; nd < p->nodes; nd++) {
        const int t = p->ndtype[nd];
        const int lp = (t == nMATP || t == nMATL) ? elp[nd] : elp[nd] + 1;
        const int rp = (t == nMATP || t == nMATR) ? erp[nd] : erp[nd] - 1;
        if (t == nEND) {
            run5 = run3 = run53 = 0.0f;
            continue;
        }
        if (t == nBEGL || t == nBEGR) {
            const int b = p->plast[p->nodemap[nd]];
            run5 = t == nBEGL ? 0.0f : l[M + b];
            run3 = t == nBEGR ? 0.0f : l[2 * M + b];
            run53 = l[b];
            continue;
        }
        if (!internal_start(t)) continue;
        const int s = p->nodemap[nd];
        int i1, i2;
        node_inserts(p, nd - 1, &i1, &i2);
        const float ps = (float)psi[s], p1 = i1 >= 0 ? (float)psi[i1] : 0.0f, p2 = i2 >= 0 ? (float)psi[i2] : 0.0f;
        const float tot = ps + p1 + p2;
        float *rows[6] = {g, g + M, g + 2 * M, l, l + M, l + 2 * M};
        float probs[6];
        int use[6] = {1, rp == clen, lp == 1, 1, 1, 1};
        const int span = rp - lp + 1, n53 = (span * (span + 1)) / 2;
        const float c5 = bg[s] / (float)span + run5, c3 = bg[s] / (float)span + run3;
        const float c53 = bg[s] / (float)n53 + run53;
        probs[0] = g53;
        probs[1] = probs[2] = g1;
        probs[3] = c53;
        probs[4] = c5;
        probs[5] = c3;
        for (int r = 0; r < 6; r++) {
            if (!use[r]) continue;
            rows[r][s] = (ps / tot) * probs[r];
            if (i1 >= 0) rows[r][i1] = (p1 / tot) * probs[r];
            if (i2 >= 0) rows[r][i2] = (p2 / tot) * probs[r];
        }
        run5 = t == nMATL ? c5 : 0.0f;
        run3 = t == nMATR ? c3 : 0.0f;
        run53 = c53;
    }
    free(bg);
    for (int v = 0; v < M; v++) {
        const int id = p->stid[v], st = p->sttype[v];
        const int det = v + 1 < M && p->stid[v + 1] == uEND_E;
        if (!(id == uMATP_MP || id == uMATL_ML || id == uMATR_MR || id == uBIF_B || ((st == pIL || st == pIR) && !det)))
            continue;
        if (id == uMATP_IL && p->ndtype[p->ndidx[v] + 1] == nEND) continue;
        for (int r = 0; r < 3; r++) {
            if (g[r * M + v] > PIMP + 1.0f) {
                ig[r * M + v] = p2s_cp9(g[r * M + v], 1.0f);
                g[r * M + v] = (float)slog2((double)g[r * M + v]);
            }
            il[r * M + v] = p2s_cp9(l[r * M + v], 1.0f);
            l[r * M + v] = (float)slog2((double)l[r * M + v]);
        }
    }
}

/* The truncated scanners' inputs (the layout of cmgpu_prep_truncated). */
int oracle_prep_truncated(const cmgpu_cm_params *p, int local, cmgpu_tr_prep *o) {
    const int M = p->M;
    oracle_marginals(p, o->lmesc, o->rmesc, o->ilmesc, o->irmesc);
    int *elp = malloc(sizeof(int) * (size_t)p->nodes), *erp = malloc(sizeof(int) * (size_t)p->nodes);
    double *psi = malloc(sizeof(double) * (size_t)M);
    float *g = malloc(sizeof(float) * 3 * (size_t)M), *l = malloc(sizeof(float) * 3 * (size_t)M);
    int32_t *ig = malloc(sizeof(int32_t) * 3 * (size_t)M), *il = malloc(sizeof(int32_t) * 3 * (size_t)M);
    emitmap(p, elp, erp);
    int rc = occupancy(p, psi);
    if (rc == 0) {
        penalties(p, elp, erp, psi, g, ig, l, il);
        memcpy(o->pty, local ? l : g, sizeof(float) * 3 * (size_t)M);
        memcpy(o->ipty, local ? il : ig, sizeof(int32_t) * 3 * (size_t)M);
        for (int v = 0; v < M; v++) {
            const int nd = p->ndidx[v], t = p->ndtype[nd];
            o->lpos[v] = (t == nMATP || t == nMATL) ? elp[nd] : elp[nd] + 1;
            o->rpos[v] = (t == nMATP || t == nMATR) ? erp[nd] : erp[nd] - 1;
        }
    }
    free(elp);
    free(erp);
    free(psi);
    free(g);
    free(l);
    free(ig);
    free(il);
    return rc;
}

/* ---- the CP9 HMM of a CM (cp9_build_and_configure, src/cp9.rs:2212) ---- */

#define C9N 10 /* MM MI MD MEL IM II ID DM DI DD */
enum { cMM = 0, cMI, cMD, cMEL, cIM, cII, cID, cDM, cDI, cDD };

typedef struct {
    const cmgpu_cm_params *p;
    int H;
    int *nd2l, *nd2r, *pos2nd; /* [nodes], [nodes], [H+1] */
    int *hns;                  /* [H+1][3][2] */
    int *csn, *css;            /* [M+1][2] */
    const double *psi;
    float *mat, *ins, *t, *beg, *end; /* [H+1][4], [H+1][4], [H+1][10], [H+1], [H+1] */
} c9;

#define HNS(m, k, s, j) (m)->hns[((k) * 3 + (s)) * 2 + (j)]

static int c9_sttype(const c9 *m, int v) { return v < m->p->M ? m->p->sttype[v] : 9; /* EL */ }

/* map_helper (src/cp9.rs:247-273) */
static int c9_map(c9 *m, int k, int ks, int v) {
    if (ks == 1 && c9_sttype(m, v + 1) == pE) return 0; /* detached insert */
    if (m->csn[v * 2] == -1) {
        m->csn[v * 2] = k;
        m->css[v * 2] = ks;
    } else if (m->csn[v * 2 + 1] == -1) {
        m->csn[v * 2 + 1] = k;
        m->css[v * 2 + 1] = ks;
    } else
        return -1;
    if (HNS(m, k, ks, 0) == -1)
        HNS(m, k, ks, 0) = v;
    else if (HNS(m, k, ks, 1) == -1)
        HNS(m, k, ks, 1) = v;
    else
        return -1;
    return 0;
}

/* the insert for the column right of k (the MATP-right and MATR cases of
 * CP9_map_cm2hmm, src/cp9.rs:331-356, :383-404) */
static int c9_right_insert(c9 *m, int k) {
    const cmgpu_cm_params *p = m->p;
    if (k == m->H) return c9_map(m, k, 1, 2);
    int nn = m->pos2nd[k + 1];
    if (m->nd2l[nn] == k + 1) {
        int b = nn;
        while (b >= 0 && p->ndtype[b] != nBEGR) b--;
        if (b < 0) return -1;
        return c9_map(m, k, 1, p->nodemap[b] + 1);
    }
    if (m->nd2r[nn] == k + 1) {
        if (p->ndtype[nn] == nMATP) return c9_map(m, k, 1, p->nodemap[nn] + 5);
        if (p->ndtype[nn] == nMATR) return c9_map(m, k, 1, p->nodemap[nn] + 2);
    }
    return 0;
}

/* CP9_map_cm2hmm (src/cp9.rs:275-427) */
static int c9_mapping(c9 *m, const int *lpos, const int *rpos) {
    const cmgpu_cm_params *p = m->p;
    int rc = 0;
    for (int n = 0; n < p->nodes; n++) {
        m->nd2l[n] = m->nd2r[n] = -1;
        if (p->ndtype[n] == nMATP || p->ndtype[n] == nMATL) {
            m->nd2l[n] = lpos[n];
            m->pos2nd[lpos[n]] = n;
        }
        if (p->ndtype[n] == nMATP || p->ndtype[n] == nMATR) {
            m->nd2r[n] = rpos[n];
            m->pos2nd[rpos[n]] = n;
        }
    }
    rc |= c9_map(m, 0, 0, 0);
    rc |= c9_map(m, 0, 1, 1);
    for (int k = 1; k <= m->H && rc == 0; k++) {
        const int n = m->pos2nd[k], nm = p->nodemap[n], t = p->ndtype[n];
        if (t == nMATP && m->nd2l[n] == k) {
            rc |= c9_map(m, k, 0, nm);
            rc |= c9_map(m, k, 0, nm + 1);
            rc |= c9_map(m, k, 1, nm + 4);
            rc |= c9_map(m, k, 2, nm + 2);
            rc |= c9_map(m, k, 2, nm + 3);
        } else if (t == nMATP) {
            rc |= c9_map(m, k, 0, nm);
            rc |= c9_map(m, k, 0, nm + 2);
            rc |= c9_right_insert(m, k);
            const int pk = m->pos2nd[k - 1];
            if (m->nd2l[pk] == k - 1) {
                if (p->ndtype[pk] != nMATL && p->ndtype[pk] != nMATP) return -1;
                rc |= c9_map(m, k - 1, 1, nm + 5);
            }
            rc |= c9_map(m, k, 2, nm + 1);
            rc |= c9_map(m, k, 2, nm + 3);
        } else if (t == nMATL) {
            rc |= c9_map(m, k, 0, nm);
            rc |= c9_map(m, k, 1, nm + 2);
            rc |= c9_map(m, k, 2, nm + 1);
            if (k == m->H) rc |= c9_map(m, k, 1, 2);
        } else if (t == nMATR) {
            rc |= c9_map(m, k, 0, nm);
            rc |= c9_right_insert(m, k);
            if (m->nd2l[m->pos2nd[k - 1]] == k - 1) return -1;
            rc |= c9_map(m, k, 2, nm + 1);
        } else
            return -1;
    }
    return rc;
}

static float c9_emit(const c9 *m, int x, int i, int k) {
    const cmgpu_cm_params *p = m->p;
    const float *e = p->e + (size_t)x * 16;
    if (p->stid[x] != uMATP_MP) return e[i];
    float r = 0.0f;
    if (m->nd2l[m->pos2nd[k]] == k)
        for (int j = i * PK; j < (i + 1) * PK; j++) r += e[j];
    else
        for (int j = i; j < PK * PK; j += PK) r += e[j];
    return r;
}

static int c9_is_ins(const cmgpu_cm_params *p, int v) { return p->sttype[v] == pIL || p->sttype[v] == pIR; }

/* cm_sum_subpaths_cp9 (src/cp9.rs:2615-2693) */
static float c9_subpaths(const c9 *m, int start, int end, int k) {
    const cmgpu_cm_params *p = m->p;
    if (start == end) return c9_is_ins(p, start) ? p->t[start * 6] : 1.0f;
    double *sp = calloc((size_t)(end - start + 1), sizeof(double));
    sp[0] = 1.0;
    if (!c9_is_ins(p, start) && !c9_is_ins(p, end)) {
        double its = 0.0;
        const int h0 = HNS(m, k, 1, 0), h1 = HNS(m, k, 1, 1);
        if (h0 < start) its = m->psi[h0] * (double)c9_subpaths(m, h0, start, k);
        if (h1 != -1 && h1 < start) its += m->psi[h1] * (double)c9_subpaths(m, h1, start, k);
        sp[0] -= its / m->psi[start];
    }
    for (int v = start + 1; v <= end; v++) {
        const int vi = v - start, isi = c9_is_ins(p, v);
        if (p->sttype[v] == pS) sp[vi] = sp[vi - 1] * 1.0;
        if (v != end && isi && (m->csn[v * 2] == k || m->csn[v * 2 + 1] == k)) continue;
        for (int y = p->pnum[v] - 1; y >= isi; y--) {
            const int x = p->plast[v] - y;
            const int ti = p->sttype[x] == pB ? 0 : v - p->cfirst[x]; /* transition map */
            if (x - start >= 0) sp[vi] += sp[x - start] * (double)p->t[x * 6 + ti];
        }
        if (v != end && isi) sp[vi] += sp[vi] * ((double)p->t[v * 6] / (1.0 - (double)p->t[v * 6]));
    }
    const float r = (float)sp[end - start];
    free(sp);
    return r;
}

static void c9_add(c9 *m, int a, int b, int k, int idx) {
    if (a == -1 || b == -1) return;
    float *c = &m->t[k * C9N + idx];
    if (a <= b)
        *c = (float)((double)*c + m->psi[a] * (double)c9_subpaths(m, a, b, k));
    else
        *c = (float)((double)*c + m->psi[b] * (double)c9_subpaths(m, b, a, k));
}

static void c9_add4(c9 *m, int ka, int sa, int kb, int sb, int k, int idx) {
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) c9_add(m, HNS(m, ka, sa, i), HNS(m, kb, sb, j), k, idx);
}

/* the END_E state paired with nothing, as the second operand */
static void c9_add_end(c9 *m, int ka, int sa, int k, int idx) {
    for (int i = 0; i < 2; i++) c9_add(m, HNS(m, ka, sa, i), m->p->M - 1, k, idx);
}

static float c9_ksum(const float *v, int n) {
    float s = 0.0f, c = 0.0f;
    for (int i = 0; i < n; i++) {
        float y = v[i] - c, t = s + y;
        c = (t - s) - y;
        s = t;
    }
    return s;
}
static void c9_norm(float *v, int n) {
    const float s = c9_ksum(v, n);
    for (int i = 0; i < n; i++) v[i] = s != 0.0f ? v[i] / s : 1.0f / (float)n;
}
static void c9_scale(float *v, int n, float f) {
    for (int i = 0; i < n; i++) v[i] *= f;
}
static int c9_exit(const cmgpu_cm_params *p, int nd) {
    const int t = p->ndtype[nd];
    return (t == nMATP || t == nMATL || t == nMATR || t == nBEGL || t == nBEGR) && nd + 1 < p->nodes &&
           p->ndtype[nd + 1] != nEND;
}

static int c9_iexp(int x, const int *sc, const float *nul) {
    if (!is_res(x)) return 0;
    float r = 0.0f, d = 0.0f;
    for (int i = 0; i < PK; i++)
        if (DEG[x][i]) {
            r += (float)sc[i] * nul[i];
            d += nul[i];
        }
    r /= d;
    return r < 0.0f ? (int)(r - 0.5f) : (int)(r + 0.5f);
}

static void c9_scores(const float *pr, const float *nul, int32_t *out) {
    int sc[PKP];
    for (int x = 0; x < PK; x++) sc[x] = p2s_cp9(pr[x], nul[x]);
    sc[PK] = sc[PKP - 2] = sc[PKP - 1] = -PINF;
    for (int x = PK + 1; x <= PKP - 3; x++) sc[x] = c9_iexp(x, sc, nul);
    for (int x = 0; x < PKP; x++) out[x] = sc[x];
}

/* exported: cp9_build_and_configure into the product's cmgpu_cp9 layout */
int oracle_prep_cp9(const cmgpu_cm_params *p, cmgpu_cp9 *o) {
    const int M = p->M;
    int H = 0;
    for (int v = 0; v < M; v++) H += p->stid[v] == uMATP_MP ? 2 : (p->stid[v] == uMATL_ML || p->stid[v] == uMATR_MR);
    if (H != o->M) return -1;
    c9 m;
    m.p = p;
    m.H = H;
    m.nd2l = malloc(sizeof(int) * (size_t)p->nodes);
    m.nd2r = malloc(sizeof(int) * (size_t)p->nodes);
    m.pos2nd = malloc(sizeof(int) * (size_t)(H + 1));
    m.hns = malloc(sizeof(int) * 6 * (size_t)(H + 1));
    m.csn = malloc(sizeof(int) * 2 * (size_t)(M + 1));
    m.css = malloc(sizeof(int) * 2 * (size_t)(M + 1));
    for (int i = 0; i <= H; i++) m.pos2nd[i] = -1;
    for (int i = 0; i < 6 * (H + 1); i++) m.hns[i] = -1;
    for (int i = 0; i < 2 * (M + 1); i++) m.csn[i] = m.css[i] = -1;
    int *lpos = malloc(sizeof(int) * (size_t)p->nodes), *rpos = malloc(sizeof(int) * (size_t)p->nodes);
    double *psi = malloc(sizeof(double) * (size_t)M);
    emitmap(p, lpos, rpos);
    int rc = c9_mapping(&m, lpos, rpos);
    if (rc == 0) rc = occupancy(p, psi);
    for (int k = 0; rc == 0 && k <= H; k++)
        if (HNS(&m, k, 0, 0) == -1 || HNS(&m, k, 1, 0) == -1) rc = -1;
    m.psi = psi;
    m.mat = calloc((size_t)(H + 1) * 4, sizeof(float));
    m.ins = calloc((size_t)(H + 1) * 4, sizeof(float));
    m.t = calloc((size_t)(H + 1) * C9N, sizeof(float));
    m.beg = calloc((size_t)(H + 1), sizeof(float));
    m.end = calloc((size_t)(H + 1), sizeof(float));
    unsigned char *hel = calloc((size_t)(H + 1), 1);
    float nul[PK];
    if (rc == 0) {
        /* emissions (src/cp9.rs:2558-2612) */
        for (int i = 0; i < PK; i++) {
            nul[i] = p->null[i];
            m.ins[i] = p->e[1 * 16 + i];
        }
        for (int k = 1; k <= H; k++) {
            for (int i = 0; i < PK; i++) {
                for (int j = 0; j < 2; j++) {
                    const int a = HNS(&m, k, 0, j);
                    if (a != -1) m.mat[k * 4 + i] = (float)((double)m.mat[k * 4 + i] + psi[a] * (double)c9_emit(&m, a, i, k));
                }
            }
            for (int i = 0; i < PK; i++) {
                for (int j = 0; j < 2; j++) {
                    const int b = HNS(&m, k, 1, j);
                    if (b != -1) m.ins[k * 4 + i] = (float)((double)m.ins[k * 4 + i] + psi[b] * (double)c9_emit(&m, b, i, k));
                }
            }
        }
        /* end-local states (:1042-1077) */
        const float el_self = (float)exp((double)p->el_selfsc * 0.69314718);
        for (int nd = 0; nd < p->nodes; nd++)
            if (c9_exit(p, nd)) hel[lpos[nd]] = 1;
        /* transitions (:2742-2841) */
        float *T = m.t;
        c9_add4(&m, 0, 0, 1, 0, 0, cMM);
        m.beg[1] = T[cMM];
        T[cMM] = 0.0f;
        c9_add4(&m, 0, 0, 0, 1, 0, cMI);
        c9_add4(&m, 0, 0, 1, 2, 0, cMD);
        c9_add4(&m, 0, 1, 1, 0, 0, cIM);
        c9_add4(&m, 0, 1, 0, 1, 0, cII);
        c9_add4(&m, 0, 1, 1, 2, 0, cID);
        T[cDM] = T[cDI] = T[cDD] = 0.0f;
        float d = c9_ksum(m.beg + 1, H) + T[cMI] + T[cMD];
        c9_scale(m.beg + 1, H, 1.0f / d);
        T[cMI] /= d;
        T[cMD] /= d;
        c9_norm(T + cIM, 3);
        float *TH = m.t + H * C9N;
        c9_add_end(&m, H, 0, H, cMM);
        m.end[H] = TH[cMM];
        TH[cMM] = 0.0f;
        c9_add4(&m, H, 0, H, 1, H, cMI);
        TH[cMD] = 0.0f;
        c9_add_end(&m, H, 1, H, cIM);
        c9_add4(&m, H, 1, H, 1, H, cII);
        TH[cID] = 0.0f;
        c9_add_end(&m, H, 2, H, cDM);
        c9_add4(&m, H, 2, H, 1, H, cDI);
        TH[cDD] = 0.0f;
        d = c9_ksum(TH, 4) + m.end[H];
        c9_scale(TH, 4, 1.0f / d);
        m.end[H] /= d;
        c9_norm(TH + cIM, 3);
        c9_norm(TH + cDM, 3);
        for (int k = 1; k < H; k++) {
            float *Tk = m.t + k * C9N;
            c9_add4(&m, k, 0, k + 1, 0, k, cMM);
            c9_add4(&m, k, 0, k, 1, k, cMI);
            c9_add4(&m, k, 0, k + 1, 2, k, cMD);
            c9_add4(&m, k, 1, k + 1, 0, k, cIM);
            c9_add4(&m, k, 1, k, 1, k, cII);
            c9_add4(&m, k, 1, k + 1, 2, k, cID);
            c9_add4(&m, k, 2, k + 1, 0, k, cDM);
            c9_add4(&m, k, 2, k, 1, k, cDI);
            c9_add4(&m, k, 2, k + 1, 2, k, cDD);
            d = c9_ksum(Tk, 4) + m.end[k];
            c9_scale(Tk, 4, 1.0f / d);
            m.end[k] /= d;
            c9_norm(Tk + cIM, 3);
            c9_norm(Tk + cDM, 3);
        }
        /* CPlan9Renormalize (:1000-1040) */
        for (int i = 0; i < PK; i++) m.mat[i] = 0.0f;
        for (int k = 1; k <= H; k++) c9_norm(m.mat + k * 4, PK);
        for (int k = 0; k <= H; k++) c9_norm(m.ins + k * 4, PK);
        d = c9_ksum(m.beg + 1, H) + T[cMI] + T[cMD] + T[cMEL];
        c9_scale(m.beg + 1, H, 1.0f / d);
        T[cMI] /= d;
        T[cMD] /= d;
        T[cMEL] /= d;
        c9_norm(T + cIM, 3);
        T[cDM] = T[cDI] = T[cDD] = 0.0f;
        for (int k = 1; k <= H; k++) {
            float *Tk = m.t + k * C9N;
            const float dk = c9_ksum(Tk, 4) + m.end[k];
            c9_scale(Tk, 4, 1.0f / dk);
            m.end[k] /= dk;
            c9_norm(Tk + cIM, 3);
            c9_norm(Tk + cDM, 3);
        }
        c9_norm(nul, PK);
        /* local begins and ends, pentry = pexit = pbegin (:1097-1119, :1079) */
        const float pb = p->pbegin;
        const float s = T[cMI] + T[cMD] + T[cMEL];
        m.beg[1] = (1.0f - pb) * (1.0f - s);
        for (int k = 2; k <= H; k++) m.beg[k] = (pb * (1.0f - s)) / ((float)H - 1.0f);
        const float basep = pb / ((float)H - 1.0f);
        for (int k = 1; k < H; k++) m.end[k] = basep / (1.0f - basep * ((float)k - 1.0f));
        for (int k = 1; k < H; k++) {
            float *Tk = m.t + k * C9N;
            const float dk = c9_ksum(Tk, 4);
            c9_scale(Tk, 4, (1.0f - m.end[k]) / dk);
        }
        const float dm = TH[cMI] + TH[cMEL];
        if (fabsf(dm - 0.0f) >= 5e-9f) {
            const float f = (1.0f - m.end[H]) / dm;
            TH[cMI] *= f;
            TH[cMEL] *= f;
        }
        /* end-local exits (:1121-1147) */
        int nexits = 0;
        for (int nd = 1; nd < p->nodes; nd++) nexits += c9_exit(p, nd);
        const float to_el = p->pend / (float)nexits;
        T[cMEL] = 0.0f;
        for (int k = 1; k <= H; k++) {
            float *Tk = m.t + k * C9N;
            if (!hel[k]) continue;
            Tk[cMEL] = to_el;
            const float nf = 1.0f - (Tk[cMEL] / (1.0f - m.end[k]));
            Tk[cMM] *= nf;
            Tk[cMI] *= nf;
            Tk[cMD] *= nf;
        }
        /* CP9Logoddsify (:1176-1255) into the product's layout */
        for (int k = 0; k <= H; k++) {
            const float *Tk = m.t + k * C9N;
            memcpy(o->mat + k * 4, m.mat + k * 4, sizeof(float) * 4);
            memcpy(o->ins + k * 4, m.ins + k * 4, sizeof(float) * 4);
            memcpy(o->t + k * C9N, Tk, sizeof(float) * C9N);
            o->begin[k] = m.beg[k];
            o->end[k] = m.end[k];
            o->has_el[k] = hel[k];
            c9_scores(m.ins + k * 4, nul, o->isc + k * PKP);
            if (k == 0)
                for (int x = 0; x < PKP; x++) o->msc[x] = 0;
            else
                c9_scores(m.mat + k * 4, nul, o->msc + k * PKP);
            int32_t *ot = o->otsc + k * 12;
            ot[0] = p2s_cp9(Tk[cMM], 1.0f);
            ot[1] = p2s_cp9(Tk[cIM], 1.0f);
            ot[2] = k ? p2s_cp9(Tk[cDM], 1.0f) : -PINF;
            ot[3] = k ? p2s_cp9(m.beg[k], 1.0f) : -PINF;
            ot[4] = p2s_cp9(Tk[cMI], 1.0f);
            ot[5] = p2s_cp9(Tk[cII], 1.0f);
            ot[6] = k ? p2s_cp9(Tk[cDI], 1.0f) : -PINF;
            ot[7] = p2s_cp9(Tk[cMD], 1.0f);
            ot[8] = p2s_cp9(Tk[cID], 1.0f);
            ot[9] = k ? p2s_cp9(Tk[cDD], 1.0f) : -PINF;
            ot[10] = k ? p2s_cp9(m.end[k], 1.0f) : -PINF;
            ot[11] = p2s_cp9(Tk[cMEL], 1.0f);
            for (int s2 = 0; s2 < 3; s2++)
                for (int j = 0; j < 2; j++) o->hns2cs[(k * 3 + s2) * 2 + j] = HNS(&m, k, s2, j);
        }
        o->n_el = 0;
        for (int nd = 0; nd < p->nodes; nd++) {
            if (!c9_exit(p, nd)) continue;
            o->el_pairs[2 * o->n_el] = lpos[nd];
            o->el_pairs[2 * o->n_el + 1] = rpos[nd];
            o->n_el++;
        }
        o->el_self = el_self;
        o->el_selfsc = p2s_cp9(el_self, 1.0f);
    }
    free(m.nd2l);
    free(m.nd2r);
    free(m.pos2nd);
    free(m.hns);
    free(m.csn);
    free(m.css);
    free(lpos);
    free(rpos);
    free(psi);
    free(m.mat);
    free(m.ins);
    free(m.t);
    free(m.beg);
    free(m.end);
    free(hel);
    return rc;
}
