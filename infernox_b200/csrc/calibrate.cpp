// cmcalibrate on the GPU: the exponential-tail E-value fit of a CM
// (calibrate_cm, src/cm_calibrate.rs:1102-1182).
//
// The reference scores N random "genomic" sequences of 10 kb with the CM in
// four modes -- glocal / local x CYK / integer Inside -- one sequence after
// another on one core (collect_scores, src/cm_calibrate.rs:953-989), and fits
// an exponential to the top of each mode's score histogram.  Here the random
// sequences are drawn on the host with the reference's generator (the
// Mersenne Twister of easel and the five-state genomic HMM), and each mode is
// ONE batched launch of the QDB scanner over all N sequences, in the
// calibration variant of the scan (local begins in bit-score order, cutoff
// -inf with the device-side report pre-filter).  The fit is host arithmetic
// in f64, in the reference's order.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/cmscan_gpu.h"

namespace cmx {
void set_error(const std::string &msg);
}
using cmx::set_error;

namespace {

// ---- easel's Mersenne Twister (src/easel/random.rs) ----------------------
class Mt19937 {
  public:
    explicit Mt19937(uint32_t seed) { reseed(seed); }
    // seeding: Knuth's LCG over the table, then one refill
    void reseed(uint32_t seed) {
        mt_[0] = seed;
        for (int z = 1; z < 624; z++) mt_[z] = 69069u * mt_[z - 1];
        refill();
    }
    // uniform deviate on [0, 1): the tempered word / 2^32
    double uniform() { return (double)next() / 4294967296.0; }

  private:
    uint32_t mt_[624];
    int idx_ = 0;
    static uint32_t mix(uint32_t hi, uint32_t lo, uint32_t far) {
        const uint32_t y = (hi & 0x80000000u) | (lo & 0x7fffffffu);
        return far ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
    }
    void refill() {
        for (int z = 0; z < 624; z++) mt_[z] = mix(mt_[z], mt_[(z + 1) % 624], mt_[(z + 397) % 624]);
        idx_ = 0;
    }
    uint32_t next() {
        if (idx_ >= 624) refill();
        uint32_t x = mt_[idx_++];
        x ^= x >> 11;
        x ^= (x << 7) & 0x9d2c5680u;
        x ^= (x << 15) & 0xefc60000u;
        x ^= x >> 18;
        return x;
    }
};

// ---- the genomic HMM (CreateGenomicHMM, src/cm_calibrate.rs:85-158) -------
// Five states fitted to genomic DNA; the rows are renormalised in f64 as the
// reference does (esl_vec_dnorm: divide by the left-to-right sum).
struct GenomicHmm {
    double start[5];
    double trans[5][5];
    double emit[5][4];
};

void dnorm(double *v, int n) {
    double s = 0.0;
    for (int i = 0; i < n; i++) s += v[i];
    for (int i = 0; i < n; i++) v[i] = s != 0.0 ? v[i] / s : 1.0 / n;
}

GenomicHmm genomic_hmm() {
    GenomicHmm h = {
        {0.157377049180328, 0.39344262295082, 0.265573770491803, 0.00327868852459016, 0.180327868852459},
        {{0.999483637183643, 0.000317942006440604, 0.000185401071732768, 2.60394763669618e-07,
          1.27593434198113e-05},
         {9.76333640771184e-05, 0.99980020511745, 9.191359010352e-05, 7.94413051888677e-08, 1.01684870641751e-05},
         {1.3223694798182e-07, 0.000155642887774602, 0.999700615549769, 9.15079680034191e-05, 5.21013575048369e-05},
         {0.994252873563218, 0.0014367816091954, 0.0014367816091954, 0.0014367816091954, 0.0014367816091954},
         {8.32138798088677e-06, 2.16356087503056e-05, 6.42411152124459e-05, 1.66427759617735e-07,
          0.999905635460297}},
        {{0.370906566523225, 0.129213995153577, 0.130511270043053, 0.369368168280145},
         {0.305194882571888, 0.194580936415687, 0.192343972160245, 0.307880208852179},
         {0.238484980800698, 0.261262845707113, 0.261810301531792, 0.238441871960397},
         {0.699280575539568, 0.00143884892086331, 0.00143884892086331, 0.297841726618705},
         {0.169064007664923, 0.331718611320207, 0.33045427183482, 0.16876310918005}},
    };
    dnorm(h.start, 5);
    for (int s = 0; s < 5; s++) {
        dnorm(h.trans[s], 5);
        dnorm(h.emit[s], 4);
    }
    return h;
}

// esl_rnd_DChoose (src/cm_calibrate.rs:163-182): the first index whose
// running sum / total exceeds one uniform draw
int choose(Mt19937 &r, const double *p, int n) {
    const double roll = r.uniform();
    double norm = 0.0;
    for (int i = 0; i < n; i++) norm += p[i];
    double sum = 0.0;
    for (int i = 0; i < n; i++) {
        sum += p[i];
        if (roll < sum / norm) return i;
    }
    return n - 1;
}

constexpr int32_t CHUNK = 10000;  // EXPTAIL_CHUNKLEN, src/cm_calibrate.rs:35
constexpr int EXP_GC = 0, EXP_GI = 1, EXP_LC = 2, EXP_LI = 3;

// Owner of one configured CM's tables and its cmgpu_cm view.
struct Configured {
    int32_t M = 0;
    std::vector<float> tsc, oesc, endsc, beginsc, t_local;
    std::vector<int32_t> itsc, ioesc, iendsc, ibeginsc, dmin1, dmax1, dmin2, dmax2;
    cmgpu_cm_scores sc{};
    cmgpu_cm view{};

    int build(const cmgpu_cm_params *p, int local, int32_t W, double beta, int nonbanded) {
        M = p->M;
        tsc.assign((size_t)M * 6, 0.0f);
        oesc.assign((size_t)M * 324, 0.0f);
        endsc.assign(M, 0.0f);
        beginsc.assign(M, 0.0f);
        t_local.assign((size_t)M * 6, 0.0f);
        itsc.assign((size_t)M * 6, 0);
        ioesc.assign((size_t)M * 324, 0);
        iendsc.assign(M, 0);
        ibeginsc.assign(M, 0);
        dmin1.assign(M, 0);
        dmax1.assign(M, 0);
        dmin2.assign(M, 0);
        dmax2.assign(M, 0);
        sc.tsc = tsc.data();
        sc.oesc = oesc.data();
        sc.endsc = endsc.data();
        sc.beginsc = beginsc.data();
        sc.t_local = t_local.data();
        sc.itsc = itsc.data();
        sc.ioesc = ioesc.data();
        sc.iendsc = iendsc.data();
        sc.ibeginsc = ibeginsc.data();
        sc.dmin1 = dmin1.data();
        sc.dmax1 = dmax1.data();
        sc.dmin2 = dmin2.data();
        sc.dmax2 = dmax2.data();
        // both band sets at the calibration beta (cm_calc_qdb_bands(cm, beta,
        // beta, w_beta) keeps the model's W), on the global transitions
        int rc = cmgpu_prep_configure(p, local, W, beta, beta, 1e-7, &sc);
        if (rc) return rc;
        if (nonbanded) {  // set_full_bands (src/cm_calibrate.rs:1224-1232)
            std::fill(dmin1.begin(), dmin1.end(), 0);
            std::fill(dmin2.begin(), dmin2.end(), 0);
            std::fill(dmax1.begin(), dmax1.end(), sc.W);
            std::fill(dmax2.begin(), dmax2.end(), sc.W);
        }
        view.M = M;
        view.W = sc.W;
        view.flags = sc.flags;
        view.sttype = p->sttype;
        view.stid = p->stid;
        view.cfirst = p->cfirst;
        view.cnum = p->cnum;
        view.tsc = tsc.data();
        view.oesc = oesc.data();
        view.endsc = endsc.data();
        view.beginsc = beginsc.data();
        view.el_selfsc = sc.el_selfsc;
        view.itsc = itsc.data();
        view.ioesc = ioesc.data();
        view.iendsc = iendsc.data();
        view.ibeginsc = ibeginsc.data();
        view.iel_selfsc = sc.iel_selfsc;
        view.dmin1 = dmin1.data();
        view.dmax1 = dmax1.data();
        view.dmin2 = dmin2.data();
        view.dmax2 = dmax2.data();
        for (int a = 0; a < 4; a++) view.null[a] = p->null[a];
        view.n3_omega = p->n3_omega;
        return CMGPU_OK;
    }
};

}  // namespace

extern "C" {

// generate_sequences + SampleGenomicSequenceFromHMM (src/cm_calibrate.rs:
// 184-200, 1113-1124): the generator is seeded once (a seed of 0 is used as
// it stands), then each sequence draws its start state, and per residue an
// emission and a transition.
int cmgpu_genomic_sample(uint32_t seed, int32_t L, int32_t nseq, uint8_t *frames) {
    if (L < 0 || nseq < 0 || (nseq > 0 && !frames)) return CMGPU_EINVAL;
    const GenomicHmm h = genomic_hmm();
    Mt19937 r(seed);
    for (int32_t s = 0; s < nseq; s++) {
        uint8_t *f = frames + (size_t)s * ((size_t)L + 2);
        f[0] = 255;
        f[L + 1] = 255;
        int st = choose(r, h.start, 5);
        for (int32_t x = 1; x <= L; x++) {
            f[x] = (uint8_t)choose(r, h.emit[st], 4);
            st = choose(r, h.trans[st], 5);
        }
    }
    return CMGPU_OK;
}

// fit_histogram + SetExpInfo (src/cm_calibrate.rs:1000-1099): the tail mass
// from the hits per Mb wanted (f32 arithmetic, as the reference), the top
// floor(n * tailp) scores of the ascending sort, and the complete-data
// exponential ML fit (mu = lowest tail score, lambda = 1 / mean excess).
int cmgpu_exp_fit(const float *scores, int64_t n, int exp_mode, int32_t n_seqs, int32_t L, int32_t gtailn,
                  int32_t ltailn, float tailp, double dbsize, cmgpu_exp_params *out) {
    if (!out || n < 0 || (n > 0 && !scores) || exp_mode < 0 || exp_mode > 3) return CMGPU_EINVAL;
    std::vector<double> x((size_t)n);
    for (int64_t k = 0; k < n; k++) {
        if (!std::isfinite(scores[k])) {
            set_error("cmgpu_exp_fit: histogram Add failed: score is not finite");
            return CMGPU_ERANGE;
        }
        x[(size_t)k] = (double)scores[k];
    }
    float tp = tailp;
    if (!(tailp > 0.0f)) {
        const float mb = ((float)n_seqs * (float)L) / 1000000.0f;
        const bool local = exp_mode == EXP_LC || exp_mode == EXP_LI;
        const float want = (float)(local ? ltailn : gtailn) * mb;
        tp = want / (float)n;
        if (tp > 1.0f) {
            set_error("cmgpu_exp_fit: tailn too large: too few hits per Mb in the histogram");
            return CMGPU_ERANGE;
        }
    }
    if (tp < 0.0f || tp > 1.0f) {
        set_error("cmgpu_exp_fit: tail mass outside [0, 1]");
        return CMGPU_EINVAL;
    }
    std::sort(x.begin(), x.end());
    const uint64_t nt = (uint64_t)((double)n * (double)tp);
    if (nt <= 1) {
        set_error("cmgpu_exp_fit: too few points in the tail fit");
        return CMGPU_ERANGE;
    }
    const double *t = x.data() + (n - (int64_t)nt);
    double mu = t[0];
    for (uint64_t k = 1; k < nt; k++)
        if (t[k] < mu) mu = t[k];
    double mean = 0.0;
    for (uint64_t k = 0; k < nt; k++) mean += t[k] - mu;
    mean /= (double)nt;
    const double lambda = 1.0 / mean;
    if (std::isnan(lambda) || std::isinf(lambda)) {
        set_error("cmgpu_exp_fit: exponential tail fit lambda is not finite");
        return CMGPU_ERANGE;
    }
    out->lambda = lambda;
    out->mu_orig = mu;
    out->mu = mu - std::log(1.0 / (double)tp) / lambda;
    out->dbsize = dbsize;
    out->nrandhits = (int32_t)n;
    out->tailp = (double)tp;
    return CMGPU_OK;
}

int cmgpu_calibrate(const cmgpu_cm_params *p, int32_t W, int device, const cmgpu_calibrate_config *cfg,
                    cmgpu_calibrate_result *out) {
    if (!p || !cfg || !out || W < 1) return CMGPU_EINVAL;
    std::memset(out, 0, sizeof(*out));
    // N = round(L_Mb * 1e6 / chunk) (src/cm_calibrate.rs:1105-1109)
    const int32_t nseq = (int32_t)(((cfg->l_mb * 1000000.0) / (double)(float)CHUNK) + 0.5);
    if (nseq < 1) {
        set_error("cmgpu_calibrate: -L too small: N < 1 sequence");
        return CMGPU_EINVAL;
    }
    const size_t flen = (size_t)CHUNK + 2;
    std::vector<uint8_t> frames(flen * (size_t)nseq);
    int rc = cmgpu_genomic_sample(cfg->seed, CHUNK, nseq, frames.data());
    if (rc) return rc;
    std::vector<cmgpu_window> wins(nseq);
    for (int32_t s = 0; s < nseq; s++) wins[s] = cmgpu_window{(int64_t)((size_t)s * flen), 1, CHUNK};
    const double dbsize = (double)CHUNK * (double)nseq;
    out->dbsize = dbsize;

    Configured g, l;
    if ((rc = g.build(p, 0, W, cfg->beta, cfg->nonbanded))) return rc;
    if ((rc = l.build(p, 1, W, cfg->beta, cfg->nonbanded))) return rc;
    cmgpu_model *gm = nullptr, *lm = nullptr;
    cmgpu_workspace *ws[2] = {nullptr, nullptr};
    auto done = [&](int code) {
        cmgpu_workspace_free(ws[0]);
        cmgpu_workspace_free(ws[1]);
        cmgpu_model_free(gm);
        cmgpu_model_free(lm);
        return code;
    };
    if ((rc = cmgpu_model_upload(&g.view, device, &gm))) return done(rc);
    if ((rc = cmgpu_model_upload(&l.view, device, &lm))) return done(rc);
    for (int w = 0; w < 2; w++)
        if ((rc = cmgpu_workspace_create(device, nullptr, &ws[w]))) return done(rc);
    // The four modes run on two host threads, each with its own workspace and
    // stream, taking modes from a shared counter (slowest first): one mode's
    // host work -- ordering the reportable cells, the greedy report with
    // null3, overlap removal, the fit -- overlaps another mode's scan.
    static const int ORDER[4] = {EXP_GI, EXP_LI, EXP_GC, EXP_LC};
    std::atomic<int> next{0};
    int rcs[2] = {CMGPU_OK, CMGPU_OK};
    std::string errs[2];
    cmgpu_stats stats[4] = {};
    auto worker = [&](int w) {
        // kept hits of a window are disjoint, so a window holds at most CHUNK
        std::vector<cmgpu_batch_hit> hits((size_t)nseq * CHUNK);
        std::vector<float> scores;
        cudaSetDevice(device);
        for (int q; (q = next.fetch_add(1)) < 4;) {
            const int mode = ORDER[q];
            const bool local = mode == EXP_LC || mode == EXP_LI;
            const int semiring = (mode == EXP_GI || mode == EXP_LI) ? CMGPU_INSIDE_I32 : CMGPU_CYK_F32;
            int32_t nh = 0;
            int r = cmgpu_calibrate_scan_batch(local ? lm : gm, ws[w], semiring, CMGPU_QDB2, frames.data(),
                                               (int64_t)frames.size(), wins.data(), nseq, cfg->do_null3, hits.data(),
                                               (int32_t)hits.size(), &nh);
            if (!r) {
                cmgpu_workspace_stats(ws[w], &stats[mode]);
                scores.resize((size_t)nh);
                for (int32_t k = 0; k < nh; k++) scores[k] = hits[k].score;
                out->nhits[mode] = nh;
                r = cmgpu_exp_fit(scores.data(), nh, mode, nseq, CHUNK, cfg->gtailn, cfg->ltailn, cfg->tailp,
                                  dbsize, &out->exp[mode]);
            }
            if (r) {
                rcs[w] = r;
                errs[w] = cmgpu_last_error();
                next.store(4);
                return;
            }
        }
    };
    std::thread other(worker, 1);
    worker(0);
    other.join();
    for (int w = 0; w < 2; w++)
        if (rcs[w]) {
            set_error(errs[w]);
            return done(rcs[w]);
        }
    for (int mode = 0; mode < 4; mode++) {
        out->cells += stats[mode].cells;
        out->terms += stats[mode].terms;
        out->kernel_ms += stats[mode].kernel_ms;
        out->launches += stats[mode].kernel_launches;
    }
    return done(CMGPU_OK);
}

}  // extern "C"
