// Host-side model preparation: turns a probability-level CM into the score
// tables and query-dependent bands the scanner reads.
//
// Each routine follows the arithmetic of the reference routine it names
// (operand types, rounding points and loop order), because every score it
// produces feeds the bit-exact scan:
//   logoddsify          src/cp9.rs:4263-4368  (CMLogoddsify + FCalcOptimizedEmitScores)
//   integer scores      src/cm_nohmm.rs:279-369 (build_integer_scores)
//   localisation        src/cp9.rs:4193-4258  (cm_config_local)
//   QDB band engine     src/cm_qdband.rs:258-549, wrapper :554-592
//   ILogsum / FLogsum   src/cp9.rs:28-44, :5391-5400
//   CP9 HMM of a CM     src/cp9.rs:275-427, :1000-1255, :2212-2232, :2532-2841
// Compiled with -ffp-contract=off: no multiply-add is fused, as in Rust.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "cm_internal.h"
#include "../../include/cmscan_gpu.h"

using namespace cmx;

namespace cmx {
void set_error(const std::string &msg);
}

namespace {

// Prob2Score of cm_nohmm (src/cm_nohmm.rs:27-33): floor(0.5 + 1000*log2(p/null)).
int prob2score(float p, float null) {
    if (p == 0.0f) return -INFTY;
    return (int)std::floor(0.5 + INTSCALE * std::log2((double)p / (double)null));
}

// esl_abc_FAvgScore (src/cm.rs:84-96)
float favg_score(int x, const float *sc) {
    if (!is_residue(x)) return 0.0f;
    float r = 0.0f;
    for (int i = 0; i < K; i++)
        if (degen(x, i)) r += sc[i];
    return r / (float)ndegen(x);
}

// esl_abc_IAvgScore (src/cm.rs:101-117)
int iavg_score(int x, const int *sc) {
    if (!is_residue(x)) return 0;
    float r = 0.0f;
    for (int i = 0; i < K; i++)
        if (degen(x, i)) r += (float)sc[i];
    r /= (float)ndegen(x);
    return r < 0.0f ? (int)(r - 0.5f) : (int)(r + 0.5f);
}

// esl_vec_FSum with Kahan compensation (src/cp9.rs:451-461)
float kahan_fsum(const float *v, int n) {
    float sum = 0.0f, c = 0.0f;
    for (int i = 0; i < n; i++) {
        float y = v[i] - c;
        float t = sum + y;
        c = (t - sum) - y;
        sum = t;
    }
    return sum;
}

struct Model {
    int M, nodes, clen;
    std::vector<int8_t> sttype, stid, ndtype;
    std::vector<int32_t> cfirst, cnum, nodemap;
    std::vector<float> t, e, begin, end;
    float null[4];
    float el_selfsc, pbegin, pend;
    uint32_t flags = 0;
};

Model load(const cmgpu_cm_params *p) {
    Model m;
    m.M = p->M;
    m.nodes = p->nodes;
    m.clen = p->clen;
    m.sttype.assign(p->sttype, p->sttype + m.M);
    m.stid.assign(p->stid, p->stid + m.M);
    m.ndtype.assign(p->ndtype, p->ndtype + m.nodes);
    m.cfirst.assign(p->cfirst, p->cfirst + m.M);
    m.cnum.assign(p->cnum, p->cnum + m.M);
    m.nodemap.assign(p->nodemap, p->nodemap + m.nodes);
    m.t.assign(p->t, p->t + (size_t)m.M * MAXC);
    m.e.assign(p->e, p->e + (size_t)m.M * 16);
    m.begin.assign(m.M, 0.0f);
    m.end.assign(m.M, 0.0f);
    std::memcpy(m.null, p->null, sizeof(m.null));
    m.el_selfsc = p->el_selfsc;
    m.pbegin = p->pbegin;
    m.pend = p->pend;
    return m;
}

// cm_config_local (src/cp9.rs:4193-4258)
void config_local(Model &cm) {
    const float p_internal_start = cm.pbegin, p_internal_exit = cm.pend;
    int nstarts = 0;
    for (int nd = 2; nd < cm.nodes; nd++) {
        int t = cm.ndtype[nd];
        if (t == MATP_ND || t == MATL_ND || t == MATR_ND || t == BIF_ND) nstarts++;
    }
    std::fill(cm.begin.begin(), cm.begin.end(), 0.0f);
    cm.begin[cm.nodemap[1]] = 1.0f - p_internal_start;
    float p = p_internal_start / (float)nstarts;
    for (int nd = 2; nd < cm.nodes; nd++) {
        int t = cm.ndtype[nd];
        if (t == MATP_ND || t == MATL_ND || t == MATR_ND || t == BIF_ND) cm.begin[cm.nodemap[nd]] = p;
    }
    for (int y = 0; y < cm.cnum[0]; y++) cm.t[y] = 0.0f;  // state 0 row
    cm.flags |= 1u << 10;

    auto is_exit = [&](int nd) {
        int t = cm.ndtype[nd];
        return (t == MATP_ND || t == MATL_ND || t == MATR_ND || t == BEGL_ND || t == BEGR_ND) &&
               cm.ndtype[nd + 1] != END_ND;
    };
    int nexits = 0;
    for (int nd = 1; nd < cm.nodes; nd++)
        if (is_exit(nd)) nexits++;
    std::fill(cm.end.begin(), cm.end.end(), 0.0f);
    for (int nd = 1; nd < cm.nodes; nd++) {
        if (!is_exit(nd)) continue;
        int v = cm.nodemap[nd];
        cm.end[v] = p_internal_exit / (float)nexits;
        int cnum = cm.cnum[v];
        float denom = kahan_fsum(&cm.t[(size_t)v * MAXC], cnum);
        denom += cm.end[v];
        float inv = 1.0f / denom;
        for (int x = 0; x < cnum; x++) cm.t[(size_t)v * MAXC + x] *= inv;
    }
    cm.flags |= 1u << 11;
}

// cm_logoddsify (src/cp9.rs:4263-4368), scan-relevant outputs.
void logoddsify(const Model &cm, cmgpu_cm_scores *o) {
    for (int v = 0; v < cm.M; v++) {
        int st = cm.sttype[v];
        float *tsc = o->tsc + (size_t)v * MAXC;
        float *oesc = o->oesc + (size_t)v * ESC;
        for (int x = 0; x < MAXC; x++) tsc[x] = IMPOSSIBLE;
        for (int x = 0; x < ESC; x++) oesc[x] = IMPOSSIBLE;
        if (st != B_ST && st != E_ST) {
            for (int x = 0; x < cm.cnum[v]; x++)
                tsc[x] = (float)sre_log2((double)cm.t[(size_t)v * MAXC + x]);
        }
        const float *e = &cm.e[(size_t)v * 16];
        if (st == MP_ST) {
            float esc[16];
            for (int x = 0; x < K; x++)
                for (int y = 0; y < K; y++) {
                    float arg = e[x * K + y] / (cm.null[x] * cm.null[y]);
                    esc[x * K + y] = (float)sre_log2((double)arg);
                }
            for (int a = 0; a < K; a++)
                for (int b = 0; b < K; b++) oesc[a * KP + b] = esc[a * K + b];
            for (int a = K + 1; a < KP - 1; a++)
                for (int b = 0; b < K; b++) {
                    float sc = 0.0f;
                    for (int l = 0; l < K; l++) sc += esc[l * K + b] * fcount_frac(a, l);
                    oesc[a * KP + b] = sc;
                }
            for (int a = 0; a < K; a++)
                for (int b = K + 1; b < KP - 1; b++) {
                    float sc = 0.0f;
                    for (int r = 0; r < K; r++) sc += esc[a * K + r] * fcount_frac(b, r);
                    oesc[a * KP + b] = sc;
                }
            for (int a = K + 1; a < KP - 1; a++)
                for (int b = K + 1; b < KP - 1; b++) {
                    float sc = 0.0f;
                    for (int l = 0; l < K; l++)
                        for (int r = 0; r < K; r++)
                            sc += esc[l * K + r] * fcount_frac(a, l) * fcount_frac(b, r);
                    oesc[a * KP + b] = sc;
                }
        } else if (st == ML_ST || st == MR_ST || st == IL_ST || st == IR_ST) {
            float esc[K];
            for (int x = 0; x < K; x++) {
                float arg = e[x] / cm.null[x];
                esc[x] = (float)sre_log2((double)arg);
            }
            for (int a = 0; a < K; a++) oesc[a] = esc[a];
            for (int a = K + 1; a < KP - 1; a++) oesc[a] = favg_score(a, esc);
        }
        o->beginsc[v] = (float)sre_log2((double)cm.begin[v]);
        o->endsc[v] = (float)sre_log2((double)cm.end[v]);
    }
}

// build_integer_scores (src/cm_nohmm.rs:279-369)
void integer_scores(const Model &cm, float el_selfsc, cmgpu_cm_scores *o) {
    for (int v = 0; v < cm.M; v++) {
        int st = cm.sttype[v];
        int32_t *itsc = o->itsc + (size_t)v * MAXC;
        int32_t *ioesc = o->ioesc + (size_t)v * ESC;
        for (int x = 0; x < MAXC; x++) itsc[x] = -INFTY;
        for (int x = 0; x < ESC; x++) ioesc[x] = -INFTY;
        if (st != B_ST && st != E_ST)
            for (int x = 0; x < cm.cnum[v]; x++) itsc[x] = prob2score(cm.t[(size_t)v * MAXC + x], 1.0f);
        const float *e = &cm.e[(size_t)v * 16];
        if (st == MP_ST) {
            int iesc[16];
            for (int a = 0; a < K; a++)
                for (int b = 0; b < K; b++) iesc[a * K + b] = prob2score(e[a * K + b], cm.null[a] * cm.null[b]);
            for (int a = 0; a < K; a++)
                for (int b = 0; b < K; b++) ioesc[a * KP + b] = iesc[a * K + b];
            for (int a = K + 1; a < KP - 1; a++)
                for (int b = 0; b < K; b++) {
                    float sc = 0.0f;
                    for (int l = 0; l < K; l++) sc += (float)iesc[l * K + b] * fcount_frac(a, l);
                    ioesc[a * KP + b] = (int)sc;
                }
            for (int a = 0; a < K; a++)
                for (int b = K + 1; b < KP - 1; b++) {
                    float sc = 0.0f;
                    for (int r = 0; r < K; r++) sc += (float)iesc[a * K + r] * fcount_frac(b, r);
                    ioesc[a * KP + b] = (int)sc;
                }
            for (int a = K + 1; a < KP - 1; a++)
                for (int b = K + 1; b < KP - 1; b++) {
                    float sc = 0.0f;
                    for (int l = 0; l < K; l++)
                        for (int r = 0; r < K; r++)
                            sc += (float)iesc[l * K + r] * fcount_frac(a, l) * fcount_frac(b, r);
                    ioesc[a * KP + b] = (int)sc;
                }
        } else if (st == ML_ST || st == MR_ST || st == IL_ST || st == IR_ST) {
            int iesc[K];
            for (int a = 0; a < K; a++) iesc[a] = prob2score(e[a], cm.null[a]);
            for (int a = 0; a < K; a++) ioesc[a] = iesc[a];
            for (int a = K + 1; a < KP - 1; a++) ioesc[a] = iavg_score(a, iesc);
        }
        o->ibeginsc[v] = prob2score(cm.begin[v], 1.0f);
        o->iendsc[v] = prob2score(cm.end[v], 1.0f);
    }
    o->iel_selfsc = prob2score(std::pow(2.0f, el_selfsc), 1.0f);
}

// BandTruncationNegligible (src/cm_qdband.rs:217-242)
bool band_truncation_negligible(const std::vector<double> &density, size_t b, size_t z) {
    if (b + 1 >= z) return false;
    double c = 0.0;
    for (size_t i = b + 1; i <= z; i++) c += density[i];
    double logbeta = (std::log(density[z]) - std::log(density[b + 1])) / (double)(z - b - 1);
    double beta = std::exp(logbeta);
    double d = (beta / (1.0 - beta)) * density[z];
    return d < c * 2.220446049250313e-16;
}

struct BandResult {
    int W;
    std::vector<int32_t> dmin1, dmax1, dmin2, dmax2;
};

// band_calculation_engine (src/cm_qdband.rs:258-549) on a global-config
// model; returns 1 when Z is too small (the caller doubles Z), 0 on success.
int band_engine(const Model &cm, size_t z, double beta1, double beta2, double beta_w, BandResult &r) {
    const int m = cm.M;
    double max_beta = std::max(std::max(beta_w, beta1), beta2);
    std::vector<float> tc((size_t)m * MAXC, 0.0f);
    for (int v = 0; v < m; v++)
        for (int k = 0; k < std::min(cm.cnum[v], MAXC); k++) tc[(size_t)v * MAXC + k] = cm.t[(size_t)v * MAXC + k];
    // local begin probabilities (src/cm_qdband.rs:151-183)
    std::vector<float> begin_copy(m, 0.0f);
    {
        int nstarts = 0;
        for (int nd = 2; nd < cm.nodes; nd++) {
            int t = cm.ndtype[nd];
            if (t == MATP_ND || t == MATL_ND || t == MATR_ND || t == BIF_ND) nstarts++;
        }
        double pis = (double)cm.pbegin;
        if (cm.nodes > 1) begin_copy[cm.nodemap[1]] = (float)(1.0 - pis);
        if (nstarts > 0) {
            float p = (float)(pis / (double)nstarts);
            for (int nd = 2; nd < cm.nodes; nd++) {
                int t = cm.ndtype[nd];
                if (t == MATP_ND || t == MATL_ND || t == MATR_ND || t == BIF_ND) begin_copy[cm.nodemap[nd]] = p;
            }
        }
    }
    std::vector<std::vector<double>> gamma(m, std::vector<double>(z + 1, 0.0));
    gamma[m - 1][0] = 1.0;
    r.dmin1.assign(m, 0);
    r.dmin2.assign(m, 0);
    r.dmax1.assign(m, cm.clen * 2);
    r.dmax2.assign(m, cm.clen * 2);
    int w = 0;
    for (int v = m - 1; v >= 0; v--) {
        int st = cm.sttype[v];
        if (st == E_ST) {
            gamma[v][0] = 1.0;
            r.dmin1[v] = r.dmax1[v] = r.dmin2[v] = r.dmax2[v] = 0;
            continue;
        }
        double pdf = 0.0;
        std::vector<double> &gv = gamma[v];
        if (st == B_ST) {
            const std::vector<double> &gl = gamma[cm.cfirst[v]];
            const std::vector<double> &gr = gamma[cm.cnum[v]];
            for (size_t n = 0; n <= z; n++) {
                for (size_t ln = 0; ln <= n; ln++) gv[n] += gl[ln] * gr[n - ln];
                pdf += gv[n];
            }
        } else if (v != 0) {
            size_t dv = (size_t)state_delta(st);
            int cf = cm.cfirst[v], cn = cm.cnum[v];
            // Element-wise the accumulation is over yoffset ascending in both
            // forms of the reference (src/cm_qdband.rs:368-399).
            for (size_t n = dv; n <= z; n++) {
                for (int yo = 0; yo < cn; yo++) {
                    int y = cf + yo;
                    gv[n] += (double)tc[(size_t)v * MAXC + yo] * gamma[y][n - dv];
                }
                pdf += gv[n];
            }
        }
        if (begin_copy[v] > 0.0f && v != 0) {
            for (size_t n = 0; n <= z; n++) gamma[0][n] += (double)begin_copy[v] * gv[n];
        }
        if (v == 0) {
            pdf = 0.0;
            for (size_t n = 0; n <= z; n++) pdf += gamma[0][n];
        }
        if (pdf <= 0.999 || gv[z] > max_beta * 2.220446049250313e-16) return 1;
        if (pdf > 1.0)
            for (double &x : gv) x /= pdf;
        {
            double cum = 0.0;
            bool set2 = false;
            for (size_t n = 0; n <= z; n++) {
                cum += gv[n];
                if (!set2 && cum > beta2) {
                    r.dmin2[v] = (int)n;
                    set2 = true;
                }
                if (set2 && cum > beta1) {
                    r.dmin1[v] = (int)n;
                    break;
                }
            }
            cum = 0.0;
            set2 = false;
            for (size_t n = z + 1; n-- > 0;) {
                cum += gv[n];
                if (!set2 && cum > beta2) {
                    r.dmax2[v] = (int)n;
                    set2 = true;
                }
                if (set2 && cum > beta1) {
                    r.dmax1[v] = (int)n;
                    break;
                }
            }
        }
        if (v == 0) {
            double cum = 0.0;
            for (size_t n = z + 1; n-- > 0;) {
                cum += gamma[0][n];
                if (cum > beta_w) {
                    w = (int)n;
                    break;
                }
            }
        }
    }
    if (!band_truncation_negligible(gamma[0], (size_t)w, z)) return 1;
    if (!band_truncation_negligible(gamma[0], (size_t)r.dmax1[0], z)) return 1;
    if (!band_truncation_negligible(gamma[0], (size_t)r.dmax2[0], z)) return 1;
    r.W = w;
    return 0;
}

}  // namespace

extern "C" int cmgpu_prep_configure(const cmgpu_cm_params *p, int local, int32_t W_in, double beta1,
                                    double beta2, double betaW, cmgpu_cm_scores *out) {
    if (!p || !out || p->M < 2 || p->nodes < 2 || !p->sttype || !p->t || !p->e) {
        cmx::set_error("cmgpu_prep_configure: bad arguments");
        return CMGPU_EINVAL;
    }
    if (beta2 - beta1 > 1e-20) {
        cmx::set_error("cmgpu_prep_configure: beta1 must be >= beta2");
        return CMGPU_EINVAL;
    }
    Model cm = load(p);
    // QDB bands + W on the un-localised model (src/cm_search.rs:899-912,
    // src/cm_qdband.rs:554-592).
    BandResult br;
    size_t z = (size_t)cm.clen * 4;
    for (;;) {
        int rc = band_engine(cm, z, beta1, beta2, betaW, br);
        if (rc == 0) break;
        z *= 2;
        if (z > (size_t)cm.clen * 1000) {
            cmx::set_error("cmgpu_prep_configure: QDB band calculation: Z got insanely large (> 1000*clen)");
            return CMGPU_ERANGE;
        }
    }
    int W = W_in > 0 ? W_in : br.W;
    std::copy(br.dmin1.begin(), br.dmin1.end(), out->dmin1);
    std::copy(br.dmax1.begin(), br.dmax1.end(), out->dmax1);
    std::copy(br.dmin2.begin(), br.dmin2.end(), out->dmin2);
    std::copy(br.dmax2.begin(), br.dmax2.end(), out->dmax2);

    float el = cm.el_selfsc;
    if (local) {
        // cm_configure_scores (src/cp9.rs:4538-4545)
        config_local(cm);
    }
    if (el * (float)W < IMPOSSIBLE) el = IMPOSSIBLE / ((float)W + 1.0f);
    logoddsify(cm, out);
    integer_scores(cm, el, out);
    if (out->t_local) std::copy(cm.t.begin(), cm.t.end(), out->t_local);
    out->el_selfsc = el;
    out->W = W;
    out->flags = cm.flags;
    return CMGPU_OK;
}

// init_ilogsum (src/cp9.rs:28-44): rint(1000 * log2(1 + 2^(-i/1000))).
extern "C" int cmgpu_ilogsum_table(int32_t *tbl, int32_t n) {
    if (!tbl || n < 0 || n > LOGSUM_TBL) return CMGPU_EINVAL;
    for (int i = 0; i < n; i++) {
        double v = INTSCALE * std::log2(1.0 + std::pow(2.0, -(double)i / INTSCALE));
        tbl[i] = (int32_t)std::nearbyint(v);
    }
    return CMGPU_OK;
}

// flogsum_lookup (src/cp9.rs:5391-5400): sreLOG2(1 + sreEXP2(-i/1000)).
extern "C" int cmgpu_flogsum_table(float *tbl, int32_t n) {
    if (!tbl || n < 0 || n > LOGSUM_TBL) return CMGPU_EINVAL;
    for (int i = 0; i < n; i++) {
        double ex = std::exp((-(double)i / 1000.0) * 0.69314718);
        tbl[i] = (float)sre_log2(1.0 + ex);
    }
    return CMGPU_OK;
}

// ===========================================================================
// Truncated-scan inputs: marginal emission scores and truncated-begin
// penalties of a configured CM.
// ===========================================================================
namespace {

// unique state ids (src/constants.rs:46-81)
constexpr int ID_MATP_MP = 6, ID_MATP_IL = 10, ID_MATL_ML = 12, ID_MATR_MR = 15, ID_BIF_B = 18, ID_END_E = 19;

// Prob2Score of the CP9/truncation code (src/cp9.rs:977-997, src/cm_trunc.rs:
// 176-185): the ratio in f32, sreLOG2 in f64, -INFTY for p == 0 and for a
// non-finite result, never below -INFTY.
int prob2score_f(float p, float null) {
    if (p == 0.0f) return -INFTY;
    float ratio = p / null;
    double v = std::floor(0.5 + 1000.0 * sre_log2((double)ratio));
    if (!std::isfinite(v)) return -INFTY;
    double c = std::max(v, (double)INT32_MIN);
    c = std::min(c, (double)INT32_MAX);
    return std::max((int)c, -INFTY);
}

// esl_abc_FExpectScore / IExpectScore over the background (src/cp9.rs:4380-4420)
float fexpect(int x, const float *sc, const float *p) {
    if (!is_residue(x)) return 0.0f;
    float r = 0.0f, den = 0.0f;
    for (int i = 0; i < K; i++)
        if (degen(x, i)) {
            r += sc[i] * p[i];
            den += p[i];
        }
    return r / den;
}
int iexpect(int x, const int *sc, const float *p) {
    if (!is_residue(x)) return 0;
    float r = 0.0f, den = 0.0f;
    for (int i = 0; i < K; i++)
        if (degen(x, i)) {
            r += (float)sc[i] * p[i];
            den += p[i];
        }
    r /= den;
    return r < 0.0f ? (int)(r - 0.5f) : (int)(r + 0.5f);
}

// fill_marginal_emissions (src/cp9.rs:4441-4530): [M][18] left / right
// marginal scores, float and integer.
void marginals(const Model &cm, float *lm, float *rm, int32_t *ilm, int32_t *irm) {
    for (int v = 0; v < cm.M; v++) {
        float *L = lm + (size_t)v * KP, *R = rm + (size_t)v * KP;
        int32_t *IL = ilm + (size_t)v * KP, *IR = irm + (size_t)v * KP;
        for (int x = 0; x < KP; x++) {
            L[x] = R[x] = 0.0f;
            IL[x] = IR[x] = 0;
        }
        for (int x : {K, KP - 2, KP - 1}) {
            L[x] = R[x] = IMPOSSIBLE;
            IL[x] = IR[x] = -INFTY;
        }
        const int st = cm.sttype[v];
        const float *e = &cm.e[(size_t)v * 16];
        if (st == MP_ST) {
            float l4[K] = {0, 0, 0, 0}, r4[K] = {0, 0, 0, 0};
            for (int x = 0; x < K; x++)
                for (int y = 0; y < K; y++) {
                    l4[x] += e[x * K + y];
                    r4[y] += e[x * K + y];
                }
            for (int x = 0; x < K; x++) {
                IL[x] = prob2score_f(l4[x], cm.null[x]);
                IR[x] = prob2score_f(r4[x], cm.null[x]);
                L[x] = (float)sre_log2((double)(l4[x] / cm.null[x]));
                R[x] = (float)sre_log2((double)(r4[x] / cm.null[x]));
            }
            for (int x = K + 1; x <= KP - 3; x++) {
                L[x] = fexpect(x, L, cm.null);
                R[x] = fexpect(x, R, cm.null);
                IL[x] = iexpect(x, IL, cm.null);
                IR[x] = iexpect(x, IR, cm.null);
            }
        } else if (st == ML_ST || st == IL_ST || st == MR_ST || st == IR_ST) {
            const bool left = st == ML_ST || st == IL_ST;
            float *F = left ? L : R;
            int32_t *I = left ? IL : IR;
            for (int x = 0; x < K; x++) {
                F[x] = (float)sre_log2((double)(e[x] / cm.null[x]));
                I[x] = prob2score_f(e[x], cm.null[x]);
            }
            for (int x = K + 1; x <= KP - 3; x++) {
                F[x] = fexpect(x, F, cm.null);
                I[x] = iexpect(x, I, cm.null);
            }
        }
    }
}

// CreateEmitMap (src/cp9.rs:144-208): left / right consensus column per node.
void emit_map(const Model &cm, const std::vector<int32_t> &ndidx, std::vector<int> &lpos, std::vector<int> &rpos) {
    lpos.assign(cm.nodes, -1);
    rpos.assign(cm.nodes, -1);
    int cpos = 0;
    std::vector<std::pair<int, int>> stack{{0, 0}};  // (on_right, node)
    while (!stack.empty()) {
        auto [on_right, nd] = stack.back();
        stack.pop_back();
        const int t = cm.ndtype[nd];
        if (on_right) {
            rpos[nd] = cpos + 1;
            if (t == MATP_ND || t == MATR_ND) cpos++;
            continue;
        }
        if (t == MATP_ND || t == MATL_ND) cpos++;
        lpos[nd] = cpos;
        stack.push_back({1, nd});
        if (t == BIF_ND) {
            const int s = cm.nodemap[nd];
            stack.push_back({0, ndidx[cm.cnum[s]]});
            stack.push_back({0, ndidx[cm.cfirst[s]]});
        } else if (t != END_ND) {
            stack.push_back({0, nd + 1});
        }
    }
}

}  // namespace

namespace {

// cm_ExpectedStateOccupancy (src/cp9.rs:752-838) of the global CM: psi[v],
// the expected number of times a parse enters state v.  The transition from
// parent x to v is x's child offset of v (the reference's transition map
// gives the same index for every parent / child pair of a CM).
bool state_occupancy(const Model &cm, const int32_t *plast, const int32_t *pnum, std::vector<double> &psi) {
    psi.assign(cm.M, 0.0);
    for (int v = 0; v < cm.M; v++) {
        const int st = cm.sttype[v];
        if (st == S_ST) {
            psi[v] = 1.0;
            continue;
        }
        const int ins = (st == IL_ST || st == IR_ST) ? 1 : 0;
        for (int y = pnum[v] - 1; y >= ins; y--) {
            const int x = plast[v] - y;
            const int off = v - cm.cfirst[x];
            if (x < 0 || off < 0 || off >= cm.cnum[x]) return false;
            psi[v] += psi[x] * (double)cm.t[(size_t)x * MAXC + off];
        }
        if (ins) {
            const double t0 = (double)cm.t[(size_t)v * MAXC];
            psi[v] += psi[v] * (t0 / (1.0 - t0));
        }
    }
    return true;
}

// InsertsGivenNodeIndex (src/cm_trunc.rs:111-124)
std::pair<int, int> inserts_of(const Model &cm, int nd) {
    if (nd < 0) return {-1, -1};
    const int v = cm.nodemap[nd];
    switch (cm.ndtype[nd]) {
    case MATP_ND: return {v + 4, v + 5};
    case MATL_ND:
    case MATR_ND: return {v + 2, -1};
    case BEGR_ND: return {v + 1, -1};
    case ROOT_ND: return {v + 1, v + 2};
    default: return {-1, -1};
    }
}

// cm_tr_penalties_Create with ignore_inserts = FALSE (TrPenalties::new,
// src/cm_trunc.rs:192-385): truncated-begin penalties [3][M] (rows
// 5'-and-3', 5'-only, 3'-only), global g / ig and local l / il.
void tr_penalties(const Model &cm, const int32_t *ndidx, const int32_t *plast, const std::vector<int> &elpos,
                  const std::vector<int> &erpos, const std::vector<double> &psi, std::vector<float> &g,
                  std::vector<int32_t> &ig, std::vector<float> &l, std::vector<int32_t> &il) {
    const int M = cm.M, clen = cm.clen;
    g.assign((size_t)3 * M, IMPOSSIBLE);
    l.assign((size_t)3 * M, IMPOSSIBLE);
    ig.assign((size_t)3 * M, -INFTY);
    il.assign((size_t)3 * M, -INFTY);
    const float g53 = (float)(2.0 / (double)(clen * (clen + 1)));
    const float g5or3 = (float)(1.0 / (double)clen);
    // local begin probabilities with the C float / double mix
    std::vector<float> begin(M, 0.0f);
    int nstarts = 0;
    for (int nd = 2; nd < cm.nodes; nd++) {
        const int t = cm.ndtype[nd];
        if (t == MATP_ND || t == MATL_ND || t == MATR_ND || t == BIF_ND) nstarts++;
    }
    if (cm.nodes > 1) begin[cm.nodemap[1]] = (float)(1.0 - (double)cm.pbegin);
    const float pb = cm.pbegin / (float)nstarts;
    for (int nd = 2; nd < cm.nodes; nd++) {
        const int t = cm.ndtype[nd];
        if (t == MATP_ND || t == MATL_ND || t == MATR_ND || t == BIF_ND) begin[cm.nodemap[nd]] = pb;
    }
    float prv5 = 0.0f, prv3 = 0.0f, prv53 = 0.0f;
    for (int nd = 0; nd < cm.nodes; nd++) {
        const int t = cm.ndtype[nd];
        const int lpos = (t == MATP_ND || t == MATL_ND) ? elpos[nd] : elpos[nd] + 1;
        const int rpos = (t == MATP_ND || t == MATR_ND) ? erpos[nd] : erpos[nd] - 1;
        if (t == END_ND) {
            prv5 = prv3 = prv53 = 0.0f;
        } else if (t == BEGL_ND || t == BEGR_ND) {
            const int b = plast[cm.nodemap[nd]];
            prv5 = t == BEGL_ND ? 0.0f : l[(size_t)1 * M + b];
            prv3 = t == BEGR_ND ? 0.0f : l[(size_t)2 * M + b];
            prv53 = l[b];
        } else if (t == MATP_ND || t == MATL_ND || t == MATR_ND || t == BIF_ND) {
            const int m = cm.nodemap[nd];
            const auto ins = inserts_of(cm, nd - 1);
            const float m_psi = (float)psi[m];
            const float i1_psi = ins.first >= 0 ? (float)psi[ins.first] : 0.0f;
            const float i2_psi = ins.second >= 0 ? (float)psi[ins.second] : 0.0f;
            const float summed = m_psi + i1_psi + i2_psi;
            auto set = [&](std::vector<float> &a, int row, float prob) {
                a[(size_t)row * M + m] = (m_psi / summed) * prob;
                if (ins.first >= 0) a[(size_t)row * M + ins.first] = (i1_psi / summed) * prob;
                if (ins.second >= 0) a[(size_t)row * M + ins.second] = (i2_psi / summed) * prob;
            };
            set(g, 0, g53);
            if (rpos == clen) set(g, 1, g5or3);
            if (lpos == 1) set(g, 2, g5or3);
            const int sub = rpos - lpos + 1;
            const int nfrag53 = (sub * (sub + 1)) / 2;
            const float cur5 = begin[m] / (float)sub + prv5;
            const float cur3 = begin[m] / (float)sub + prv3;
            const float cur53 = begin[m] / (float)nfrag53 + prv53;
            set(l, 0, cur53);
            set(l, 1, cur5);
            set(l, 2, cur3);
            prv5 = t == MATL_ND ? cur5 : 0.0f;
            prv3 = t == MATR_ND ? cur3 : 0.0f;
            prv53 = cur53;
        }
    }
    for (int v = 0; v < M; v++) {
        const int id = cm.stid[v], st = cm.sttype[v];
        const bool detached = v + 1 < M && cm.stid[v + 1] == ID_END_E;
        const bool qualifies = id == ID_MATP_MP || id == ID_MATL_ML || id == ID_MATR_MR || id == ID_BIF_B ||
                               ((st == IL_ST || st == IR_ST) && !detached);
        if (!qualifies) continue;
        if (id == ID_MATP_IL && cm.ndtype[ndidx[v] + 1] == END_ND) continue;
        for (int r = 0; r < 3; r++) {
            float &x = g[(size_t)r * M + v];
            if (x > IMPOSSIBLE + 1.0f) {
                ig[(size_t)r * M + v] = prob2score_f(x, 1.0f);
                x = (float)sre_log2((double)x);
            }
            float &y = l[(size_t)r * M + v];
            il[(size_t)r * M + v] = prob2score_f(y, 1.0f);
            y = (float)sre_log2((double)y);
        }
    }
}

}  // namespace

extern "C" int cmgpu_prep_truncated(const cmgpu_cm_params *p, int local, cmgpu_tr_prep *out) {
    if (!p || !out || p->M < 2 || p->nodes < 2 || !p->sttype || !p->t || !p->e || !p->plast || !p->pnum ||
        !p->ndidx || !out->lmesc || !out->rmesc || !out->ilmesc || !out->irmesc || !out->pty || !out->ipty ||
        !out->lpos || !out->rpos) {
        cmx::set_error("cmgpu_prep_truncated: bad arguments");
        return CMGPU_EINVAL;
    }
    Model cm = load(p);
    marginals(cm, out->lmesc, out->rmesc, out->ilmesc, out->irmesc);
    std::vector<int32_t> ndidx(p->ndidx, p->ndidx + cm.M);
    std::vector<int> elpos, erpos;
    emit_map(cm, ndidx, elpos, erpos);
    std::vector<double> psi;
    if (!state_occupancy(cm, p->plast, p->pnum, psi)) {
        cmx::set_error("cmgpu_prep_truncated: a parent does not list the state among its children");
        return CMGPU_EINVAL;
    }
    std::vector<float> g, l;
    std::vector<int32_t> ig, il;
    tr_penalties(cm, p->ndidx, p->plast, elpos, erpos, psi, g, ig, l, il);
    const std::vector<float> &pt = local ? l : g;
    const std::vector<int32_t> &ipt = local ? il : ig;
    std::copy(pt.begin(), pt.end(), out->pty);
    std::copy(ipt.begin(), ipt.end(), out->ipty);
    for (int v = 0; v < cm.M; v++) {
        const int nd = ndidx[v], t = cm.ndtype[nd];
        out->lpos[v] = (t == MATP_ND || t == MATL_ND) ? elpos[nd] : elpos[nd] + 1;
        out->rpos[v] = (t == MATP_ND || t == MATR_ND) ? erpos[nd] : erpos[nd] - 1;
    }
    return CMGPU_OK;
}

// ---------------------------------------------------------------------------
// The CP9 HMM of a CM: the first step of HMM-banded search
// (cp9_build_and_configure, src/cp9.rs:2212-2232): the CM <-> HMM state map
// (CP9_map_cm2hmm, :275-427), occupancy-weighted emissions (:2558-2612) and
// transitions summed over CM subpaths (:2615-2841), renormalisation (:1000),
// end-local states (:1042), local begins and ends (:1097, :1121) and the
// integer log-odds scores (:1176-1255).
// ---------------------------------------------------------------------------
namespace {

constexpr int CT_MM = 0, CT_MI = 1, CT_MD = 2, CT_MEL = 3, CT_IM = 4, CT_II = 5, CT_ID = 6, CT_DM = 7, CT_DI = 8,
              CT_DD = 9, CT_N = 10;
constexpr int HM = 0, HI = 1, HD = 2;  // HMM match, insert, delete
constexpr int CP9_INFTY = 987654321;

struct Cp9Map {
    int hmm_m = 0;
    std::vector<int> nd2lpos, nd2rpos, pos2nd;
    std::vector<std::array<std::array<int, 2>, 3>> hns2cs;  // [k][ks][0..1]
    std::vector<std::array<int, 2>> cs2hn, cs2hs;          // [v][0..1]
};

struct Cp9 {
    int M = 0;
    std::vector<std::array<float, 4>> mat, ins;
    std::vector<std::array<float, CT_N>> t;
    std::vector<float> begin, end;
    std::vector<uint8_t> has_el;
    float null[4] = {};
    float el_self = 0.0f;
};

// Prob2Score of the CP9 (src/cp9.rs:977-998): the ratio in float, sreLOG2
// (ln x * 1.44269504) in double, floor(0.5 + 1000 x), never below -INFTY.
int cp9_prob2score(float p, float null) {
    if (p == 0.0f) return -CP9_INFTY;
    const float ratio = p / null;
    const double l2 = ratio > 0.0f ? std::log((double)ratio) * 1.44269504 : -1e36;
    const double v = std::floor(0.5 + 1000.0 * l2);
    if (!std::isfinite(v) || v <= -(double)CP9_INFTY) return -CP9_INFTY;
    return (int)v;
}

void fnorm_f(float *v, int n) {
    const float s = kahan_fsum(v, n);
    for (int i = 0; i < n; i++) v[i] = s != 0.0f ? v[i] / s : 1.0f / (float)n;
}

bool map_helper(const Model &cm, Cp9Map &m, int k, int ks, int v) {
    // a detached insert (the state after it an END_E) maps to no HMM state
    if (ks == HI && (v + 1 >= cm.M ? EL_ST : cm.sttype[v + 1]) == E_ST) return true;
    if (m.cs2hn[v][0] == -1) {
        m.cs2hn[v][0] = k;
        m.cs2hs[v][0] = ks;
    } else if (m.cs2hn[v][1] == -1) {
        m.cs2hn[v][1] = k;
        m.cs2hs[v][1] = ks;
    } else {
        return false;
    }
    auto &h = m.hns2cs[k][ks];
    if (h[0] == -1) {
        h[0] = v;
    } else if (h[1] == -1) {
        h[1] = v;
    } else {
        return false;
    }
    return true;
}

// the insert state modelling the column after HMM node k, looked up from the
// node of column k+1 (or ROOT_IR after the last column)
bool map_right_insert(const Model &cm, Cp9Map &m, int k) {
    if (k == m.hmm_m) return map_helper(cm, m, k, HI, 2);  // ROOT_IR
    const int nn = m.pos2nd[k + 1];
    if (m.nd2lpos[nn] == k + 1) {
        int b = nn;
        while (b >= 0 && cm.ndtype[b] != BEGR_ND) b--;
        if (b < 0) return false;
        return map_helper(cm, m, k, HI, cm.nodemap[b] + 1);  // BEGR_IL
    }
    if (m.nd2rpos[nn] == k + 1) {
        if (cm.ndtype[nn] == MATP_ND) return map_helper(cm, m, k, HI, cm.nodemap[nn] + 5);  // MATP_IR
        if (cm.ndtype[nn] == MATR_ND) return map_helper(cm, m, k, HI, cm.nodemap[nn] + 2);  // MATR_IR
    }
    return true;
}

bool map_cm2hmm(const Model &cm, const std::vector<int> &lpos, const std::vector<int> &rpos, Cp9Map &m) {
    m.hmm_m = 0;
    for (int v = 0; v < cm.M; v++) {
        if (cm.stid[v] == ID_MATP_MP) m.hmm_m += 2;
        else if (cm.stid[v] == ID_MATL_ML || cm.stid[v] == ID_MATR_MR) m.hmm_m += 1;
    }
    const int H = m.hmm_m;
    m.nd2lpos.assign(cm.nodes, -1);
    m.nd2rpos.assign(cm.nodes, -1);
    m.pos2nd.assign(H + 1, -1);
    std::array<std::array<int, 2>, 3> none;
    for (auto &a : none) a = {-1, -1};
    m.hns2cs.assign(H + 1, none);
    m.cs2hn.assign(cm.M + 1, {-1, -1});
    m.cs2hs.assign(cm.M + 1, {-1, -1});
    for (int n = 0; n < cm.nodes; n++) {
        const int t = cm.ndtype[n];
        if (t == MATP_ND || t == MATL_ND) {
            m.nd2lpos[n] = lpos[n];
            m.pos2nd[lpos[n]] = n;
        }
        if (t == MATP_ND || t == MATR_ND) {
            m.nd2rpos[n] = rpos[n];
            m.pos2nd[rpos[n]] = n;
        }
    }
    bool ok = map_helper(cm, m, 0, HM, 0) && map_helper(cm, m, 0, HI, 1);  // ROOT_S, ROOT_IL
    for (int k = 1; ok && k <= H; k++) {
        const int n = m.pos2nd[k];
        if (n < 0) return false;
        const int t = cm.ndtype[n], nm = cm.nodemap[n];
        if (t == MATP_ND && m.nd2lpos[n] == k) {
            ok = map_helper(cm, m, k, HM, nm) && map_helper(cm, m, k, HM, nm + 1) &&
                 map_helper(cm, m, k, HI, nm + 4) && map_helper(cm, m, k, HD, nm + 2) &&
                 map_helper(cm, m, k, HD, nm + 3);
        } else if (t == MATP_ND) {
            ok = map_helper(cm, m, k, HM, nm) && map_helper(cm, m, k, HM, nm + 2) && map_right_insert(cm, m, k);
            const int pk = m.pos2nd[k - 1];
            if (ok && m.nd2lpos[pk] == k - 1) {
                if (cm.ndtype[pk] != MATL_ND && cm.ndtype[pk] != MATP_ND) return false;
                ok = map_helper(cm, m, k - 1, HI, nm + 5);  // MATP_IR
            }
            ok = ok && map_helper(cm, m, k, HD, nm + 1) && map_helper(cm, m, k, HD, nm + 3);
        } else if (t == MATL_ND) {
            ok = map_helper(cm, m, k, HM, nm) && map_helper(cm, m, k, HI, nm + 2) &&
                 map_helper(cm, m, k, HD, nm + 1);
            if (ok && k == H) ok = map_helper(cm, m, k, HI, 2);  // ROOT_IR
        } else if (t == MATR_ND) {
            ok = map_helper(cm, m, k, HM, nm) && map_right_insert(cm, m, k);
            if (ok && m.nd2lpos[m.pos2nd[k - 1]] == k - 1) return false;
            ok = ok && map_helper(cm, m, k, HD, nm + 1);
        } else {
            return false;
        }
    }
    return ok;
}

// probability that CM state x emits residue i at HMM node k (a pair state
// marginalised over its other half), cm2hmm_emit_prob (src/cp9.rs:2532-2553)
float emit_prob(const Model &cm, const Cp9Map &m, int x, int i, int k) {
    const float *e = &cm.e[(size_t)x * 16];
    if (cm.stid[x] != ID_MATP_MP) return e[i];
    float r = 0.0f;
    if (m.nd2lpos[m.pos2nd[k]] == k) {
        for (int j = i * K; j < (i + 1) * K; j++) r += e[j];
    } else {
        for (int j = i; j < K * K; j += K) r += e[j];
    }
    return r;
}

void add_emission(float &cell, double psi, float p) { cell = (float)((double)cell + psi * (double)p); }

void cp9_emissions(const Model &cm, const Cp9Map &m, const std::vector<double> &psi, Cp9 &h) {
    const int H = m.hmm_m;
    for (int i = 0; i < K; i++) {
        h.null[i] = cm.null[i];
        h.ins[0][i] = cm.e[(size_t)1 * 16 + i];  // node 0's insert is ROOT_IL
    }
    for (int k = 1; k <= H; k++) {
        for (int ks : {HM, HI}) {
            const int a0 = m.hns2cs[k][ks][0], a1 = m.hns2cs[k][ks][1];
            auto &row = ks == HM ? h.mat[k] : h.ins[k];
            for (int i = 0; i < K; i++) {
                add_emission(row[i], psi[a0], emit_prob(cm, m, a0, i, k));
                if (a1 != -1) add_emission(row[i], psi[a1], emit_prob(cm, m, a1, i, k));
            }
        }
    }
}

// the nodes with an end-local exit: MATP/MATL/MATR/BEGL/BEGR not followed by END
bool has_exit(const Model &cm, int nd) {
    const int t = cm.ndtype[nd];
    return (t == MATP_ND || t == MATL_ND || t == MATR_ND || t == BEGL_ND || t == BEGR_ND) && nd + 1 < cm.nodes &&
           cm.ndtype[nd + 1] != END_ND;
}

// transition index from parent x to its child v (the reference's transition
// map: a bifurcation's two children are both its transition 0)
int child_index(const Model &cm, int x, int v) { return cm.sttype[x] == B_ST ? 0 : v - cm.cfirst[x]; }

// cm_sum_subpaths_cp9 (src/cp9.rs:2615-2693): summed probability of the CM
// subpaths from start to end
float sum_subpaths(const Model &cm, const int32_t *plast, const int32_t *pnum, const Cp9Map &m, int start, int end,
                   int k, const std::vector<double> &psi) {
    auto is_ins = [&](int v) { return cm.sttype[v] == IL_ST || cm.sttype[v] == IR_ST; };
    if (start == end) return is_ins(start) ? cm.t[(size_t)start * MAXC] : 1.0f;
    std::vector<double> sub(end - start + 1, 0.0);
    sub[0] = 1.0;
    if (!is_ins(start) && !is_ins(end)) {
        double to_start = 0.0;
        const int h0 = m.hns2cs[k][HI][0], h1 = m.hns2cs[k][HI][1];
        if (h0 < start) to_start = psi[h0] * (double)sum_subpaths(cm, plast, pnum, m, h0, start, k, psi);
        if (h1 != -1 && h1 < start)
            to_start += psi[h1] * (double)sum_subpaths(cm, plast, pnum, m, h1, start, k, psi);
        sub[0] -= to_start / psi[start];
    }
    for (int v = start + 1; v <= end; v++) {
        const int vi = v - start, ins = is_ins(v) ? 1 : 0;
        if (cm.sttype[v] == S_ST) sub[vi] = sub[vi - 1] * 1.0;
        if (v != end && ins && (m.cs2hn[v][0] == k || m.cs2hn[v][1] == k)) continue;
        for (int y = pnum[v] - 1; y >= ins; y--) {
            const int x = plast[v] - y;
            if (x - start >= 0) sub[vi] += sub[x - start] * (double)cm.t[(size_t)x * MAXC + child_index(cm, x, v)];
        }
        if (v != end && ins) {
            const double t0 = (double)cm.t[(size_t)v * MAXC];
            sub[vi] += sub[vi] * (t0 / (1.0 - t0));
        }
    }
    return (float)sub[end - start];
}

void add_trans(const Model &cm, const int32_t *plast, const int32_t *pnum, const Cp9Map &m, Cp9 &h, int a, int b,
               int k, int idx, const std::vector<double> &psi) {
    if (a == -1 || b == -1) return;
    const int lo = a <= b ? a : b, hi = a <= b ? b : a;
    const float sub = sum_subpaths(cm, plast, pnum, m, lo, hi, k, psi);
    h.t[k][idx] = (float)((double)h.t[k][idx] + psi[lo] * (double)sub);
}

void add4(const Model &cm, const int32_t *plast, const int32_t *pnum, const Cp9Map &m, Cp9 &h,
          const std::array<int, 2> &ap, const std::array<int, 2> &bp, int k, int idx, const std::vector<double> &psi) {
    for (int i : {0, 1})
        for (int j : {0, 1}) add_trans(cm, plast, pnum, m, h, ap[i], bp[j], k, idx, psi);
}

void fscale_f(float *v, int n, float s) {
    for (int i = 0; i < n; i++) v[i] *= s;
}

void cp9_transitions(const Model &cm, const int32_t *plast, const int32_t *pnum, const Cp9Map &m,
                     const std::vector<double> &psi, Cp9 &h) {
    const int H = m.hmm_m;
    auto &c = m.hns2cs;
    // into node 1 (src/cp9.rs:2742-2770)
    add4(cm, plast, pnum, m, h, c[0][HM], c[1][HM], 0, CT_MM, psi);
    h.begin[1] = h.t[0][CT_MM];
    h.t[0][CT_MM] = 0.0f;
    add4(cm, plast, pnum, m, h, c[0][HM], c[0][HI], 0, CT_MI, psi);
    add4(cm, plast, pnum, m, h, c[0][HM], c[1][HD], 0, CT_MD, psi);
    add4(cm, plast, pnum, m, h, c[0][HI], c[1][HM], 0, CT_IM, psi);
    add4(cm, plast, pnum, m, h, c[0][HI], c[0][HI], 0, CT_II, psi);
    add4(cm, plast, pnum, m, h, c[0][HI], c[1][HD], 0, CT_ID, psi);
    h.t[0][CT_DM] = h.t[0][CT_DI] = h.t[0][CT_DD] = 0.0f;
    float d = kahan_fsum(&h.begin[1], H) + h.t[0][CT_MI] + h.t[0][CT_MD];
    fscale_f(&h.begin[1], H, 1.0f / d);
    h.t[0][CT_MI] /= d;
    h.t[0][CT_MD] /= d;
    fnorm_f(&h.t[0][CT_IM], 3);
    // out of node M (:2772-2800)
    const std::array<int, 2> end_e{cm.M - 1, -1};
    add4(cm, plast, pnum, m, h, c[H][HM], end_e, H, CT_MM, psi);
    h.end[H] = h.t[H][CT_MM];
    h.t[H][CT_MM] = 0.0f;
    add4(cm, plast, pnum, m, h, c[H][HM], c[H][HI], H, CT_MI, psi);
    h.t[H][CT_MD] = 0.0f;
    add4(cm, plast, pnum, m, h, c[H][HI], end_e, H, CT_IM, psi);
    add4(cm, plast, pnum, m, h, c[H][HI], c[H][HI], H, CT_II, psi);
    h.t[H][CT_ID] = 0.0f;
    add4(cm, plast, pnum, m, h, c[H][HD], end_e, H, CT_DM, psi);
    add4(cm, plast, pnum, m, h, c[H][HD], c[H][HI], H, CT_DI, psi);
    h.t[H][CT_DD] = 0.0f;
    d = kahan_fsum(&h.t[H][0], 4) + h.end[H];
    fscale_f(&h.t[H][0], 4, 1.0f / d);
    h.end[H] /= d;
    fnorm_f(&h.t[H][CT_IM], 3);
    fnorm_f(&h.t[H][CT_DM], 3);
    // interior nodes (:2803-2826)
    for (int k = 1; k < H; k++) {
        const auto &hm = c[k][HM], &hi = c[k][HI], &hd = c[k][HD], &nm = c[k + 1][HM], &nd = c[k + 1][HD];
        add4(cm, plast, pnum, m, h, hm, nm, k, CT_MM, psi);
        add4(cm, plast, pnum, m, h, hm, hi, k, CT_MI, psi);
        add4(cm, plast, pnum, m, h, hm, nd, k, CT_MD, psi);
        add4(cm, plast, pnum, m, h, hi, nm, k, CT_IM, psi);
        add4(cm, plast, pnum, m, h, hi, hi, k, CT_II, psi);
        add4(cm, plast, pnum, m, h, hi, nd, k, CT_ID, psi);
        add4(cm, plast, pnum, m, h, hd, nm, k, CT_DM, psi);
        add4(cm, plast, pnum, m, h, hd, hi, k, CT_DI, psi);
        add4(cm, plast, pnum, m, h, hd, nd, k, CT_DD, psi);
        d = kahan_fsum(&h.t[k][0], 4) + h.end[k];
        fscale_f(&h.t[k][0], 4, 1.0f / d);
        h.end[k] /= d;
        fnorm_f(&h.t[k][CT_IM], 3);
        fnorm_f(&h.t[k][CT_DM], 3);
    }
}

// CPlan9Renormalize (src/cp9.rs:1000-1040)
void cp9_renormalize(Cp9 &h) {
    const int H = h.M;
    h.mat[0] = {0.0f, 0.0f, 0.0f, 0.0f};
    for (int k = 1; k <= H; k++) fnorm_f(h.mat[k].data(), K);
    for (int k = 0; k <= H; k++) fnorm_f(h.ins[k].data(), K);
    const float d = kahan_fsum(&h.begin[1], H) + h.t[0][CT_MI] + h.t[0][CT_MD] + h.t[0][CT_MEL];
    fscale_f(&h.begin[1], H, 1.0f / d);
    h.t[0][CT_MI] /= d;
    h.t[0][CT_MD] /= d;
    h.t[0][CT_MEL] /= d;
    fnorm_f(&h.t[0][CT_IM], 3);
    h.t[0][CT_DM] = h.t[0][CT_DI] = h.t[0][CT_DD] = 0.0f;
    for (int k = 1; k <= H; k++) {
        const float dk = kahan_fsum(&h.t[k][0], 4) + h.end[k];
        fscale_f(&h.t[k][0], 4, 1.0f / dk);
        h.end[k] /= dk;
        fnorm_f(&h.t[k][CT_IM], 3);
        fnorm_f(&h.t[k][CT_DM], 3);
    }
    fnorm_f(h.null, K);
}

// CPlan9InitEL, the score-relevant part (src/cp9.rs:1042-1077)
void cp9_init_el(const Model &cm, const std::vector<int> &lpos, Cp9 &h) {
    h.el_self = (float)std::exp((double)cm.el_selfsc * 0.69314718);
    std::fill(h.has_el.begin(), h.has_el.end(), 0);
    for (int nd = 0; nd < cm.nodes; nd++)
        if (has_exit(cm, nd)) h.has_el[lpos[nd]] = 1;
}

// cp9_renormalize_exits (src/cp9.rs:1079-1095)
void cp9_renormalize_exits(Cp9 &h) {
    const int H = h.M;
    for (int k = 1; k < H; k++) {
        const float d = kahan_fsum(&h.t[k][0], 4);
        fscale_f(&h.t[k][0], 4, (1.0f - h.end[k]) / d);
    }
    const float d = h.t[H][CT_MI] + h.t[H][CT_MEL];
    if (std::fabs(d - 0.0f) >= 5e-9f) {
        const float f = (1.0f - h.end[H]) / d;
        h.t[H][CT_MI] *= f;
        h.t[H][CT_MEL] *= f;
    }
}

// cp9_sw_config (src/cp9.rs:1097-1119), entry and exit pbegin
void cp9_sw_config(Cp9 &h, float pentry, float pexit) {
    const int H = h.M;
    const float s = h.t[0][CT_MI] + h.t[0][CT_MD] + h.t[0][CT_MEL];
    h.begin[1] = (1.0f - pentry) * (1.0f - s);
    const float val = (pentry * (1.0f - s)) / ((float)H - 1.0f);
    for (int k = 2; k <= H; k++) h.begin[k] = val;
    const float basep = pexit / ((float)H - 1.0f);
    for (int k = 1; k < H; k++) h.end[k] = basep / (1.0f - basep * ((float)k - 1.0f));
    cp9_renormalize_exits(h);
}

// cp9_EL_local_ends_config (src/cp9.rs:1121-1147), on the global CM
void cp9_el_local_ends(const Model &cm, Cp9 &h) {
    int nexits = 0;
    for (int nd = 1; nd < cm.nodes; nd++)
        if (has_exit(cm, nd)) nexits++;
    const float to_el = cm.pend / (float)nexits;
    h.t[0][CT_MEL] = 0.0f;
    for (int k = 1; k <= h.M; k++) {
        if (!h.has_el[k]) continue;
        h.t[k][CT_MEL] = to_el;
        const float nf = 1.0f - (h.t[k][CT_MEL] / (1.0f - h.end[k]));
        h.t[k][CT_MM] *= nf;
        h.t[k][CT_MI] *= nf;
        h.t[k][CT_MD] *= nf;
    }
}

// esl_abc_IExpectScore with the CP9's null (src/cp9.rs:1152-1173)
int cp9_iexpect(int x, const int *sc, const float *p) {
    if (!is_residue(x)) return 0;
    float r = 0.0f, den = 0.0f;
    for (int i = 0; i < K; i++)
        if (degen(x, i)) {
            r += (float)sc[i] * p[i];
            den += p[i];
        }
    r /= den;
    return r < 0.0f ? (int)(r - 0.5f) : (int)(r + 0.5f);
}

void cp9_emission_scores(const std::array<float, 4> &pr, const float *null, int32_t *out) {
    int sc[KP];
    for (int x = 0; x < K; x++) sc[x] = cp9_prob2score(pr[x], null[x]);
    sc[K] = sc[KP - 2] = sc[KP - 1] = -CP9_INFTY;
    for (int x = K + 1; x <= KP - 3; x++) sc[x] = cp9_iexpect(x, sc, null);
    std::copy(sc, sc + KP, out);
}

}  // namespace

extern "C" int cmgpu_prep_cp9(const cmgpu_cm_params *p, cmgpu_cp9 *out) {
    if (!p || !out || p->M < 2 || p->nodes < 2 || !p->sttype || !p->t || !p->e || !p->plast || !p->pnum ||
        !p->ndidx || !out->mat || !out->ins || !out->t || !out->begin || !out->end || !out->msc || !out->isc ||
        !out->otsc || !out->has_el || !out->hns2cs || !out->el_pairs || out->M != p->clen) {
        cmx::set_error("cmgpu_prep_cp9: bad arguments (out->M must be the CM's consensus length)");
        return CMGPU_EINVAL;
    }
    Model cm = load(p);
    std::vector<int32_t> ndidx(p->ndidx, p->ndidx + cm.M);
    std::vector<int> lpos, rpos;
    emit_map(cm, ndidx, lpos, rpos);
    Cp9Map m;
    if (!map_cm2hmm(cm, lpos, rpos, m) || m.hmm_m != p->clen || m.hmm_m < 2) {
        cmx::set_error("cmgpu_prep_cp9: the CM's nodes do not map onto a CP9 HMM");
        return CMGPU_EINVAL;
    }
    for (int k = 0; k <= m.hmm_m; k++)
        if (m.hns2cs[k][HI][0] == -1 || m.hns2cs[k][HM][0] == -1) {
            cmx::set_error("cmgpu_prep_cp9: HMM node " + std::to_string(k) + " has no CM match or insert state");
            return CMGPU_EINVAL;
        }
    std::vector<double> psi;
    if (!state_occupancy(cm, p->plast, p->pnum, psi)) {
        cmx::set_error("cmgpu_prep_cp9: a parent does not list the state among its children");
        return CMGPU_EINVAL;
    }
    const int H = m.hmm_m;
    Cp9 h;
    h.M = H;
    h.mat.assign(H + 1, {0.0f, 0.0f, 0.0f, 0.0f});
    h.ins.assign(H + 1, {0.0f, 0.0f, 0.0f, 0.0f});
    std::array<float, CT_N> zt{};
    h.t.assign(H + 1, zt);
    h.begin.assign(H + 1, 0.0f);
    h.end.assign(H + 1, 0.0f);
    h.has_el.assign(H + 1, 0);
    cp9_emissions(cm, m, psi, h);
    cp9_init_el(cm, lpos, h);
    cp9_transitions(cm, p->plast, p->pnum, m, psi, h);
    cp9_renormalize(h);
    cp9_sw_config(h, cm.pbegin, cm.pbegin);
    cp9_el_local_ends(cm, h);
    // CP9Logoddsify (src/cp9.rs:1176-1255), transitions in the DP's order
    for (int k = 0; k <= H; k++) {
        std::copy(h.mat[k].begin(), h.mat[k].end(), out->mat + (size_t)k * 4);
        std::copy(h.ins[k].begin(), h.ins[k].end(), out->ins + (size_t)k * 4);
        std::copy(h.t[k].begin(), h.t[k].end(), out->t + (size_t)k * CT_N);
        out->begin[k] = h.begin[k];
        out->end[k] = h.end[k];
        out->has_el[k] = h.has_el[k];
        cp9_emission_scores(h.ins[k], h.null, out->isc + (size_t)k * KP);
        if (k == 0) {
            std::fill(out->msc, out->msc + KP, 0);
        } else {
            cp9_emission_scores(h.mat[k], h.null, out->msc + (size_t)k * KP);
        }
        auto ts = [&](int c) { return cp9_prob2score(h.t[k][c], 1.0f); };
        const int bsc = k == 0 ? -CP9_INFTY : cp9_prob2score(h.begin[k], 1.0f);
        const int esc = k == 0 ? -CP9_INFTY : cp9_prob2score(h.end[k], 1.0f);
        const bool k0 = k == 0;
        int32_t *o = out->otsc + (size_t)k * 12;
        o[0] = ts(CT_MM);
        o[1] = ts(CT_IM);
        o[2] = k0 ? -CP9_INFTY : ts(CT_DM);
        o[3] = bsc;
        o[4] = ts(CT_MI);
        o[5] = ts(CT_II);
        o[6] = k0 ? -CP9_INFTY : ts(CT_DI);
        o[7] = ts(CT_MD);
        o[8] = ts(CT_ID);
        o[9] = k0 ? -CP9_INFTY : ts(CT_DD);
        o[10] = esc;
        o[11] = ts(CT_MEL);
        for (int ks = 0; ks < 3; ks++)
            for (int j = 0; j < 2; j++) out->hns2cs[((size_t)k * 3 + ks) * 2 + j] = m.hns2cs[k][ks][j];
    }
    out->n_el = 0;
    for (int nd = 0; nd < cm.nodes; nd++)
        if (has_exit(cm, nd)) {
            out->el_pairs[2 * out->n_el] = lpos[nd];
            out->el_pairs[2 * out->n_el + 1] = rpos[nd];
            out->n_el++;
        }
    out->el_self = h.el_self;
    out->el_selfsc = cp9_prob2score(h.el_self, 1.0f);
    return CMGPU_OK;
}
