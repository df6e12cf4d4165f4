/* Oracle (test infrastructure only): the host parts of cmcalibrate
 * restated from the reference -- easel's Mersenne Twister
 * (src/easel/random.rs:29-160), the genomic HMM and its sampler
 * (CreateGenomicHMM / esl_rnd_DChoose / SampleGenomicSequenceFromHMM,
 * src/cm_calibrate.rs:85-200), and fit_histogram + SetExpInfo
 * (src/cm_calibrate.rs:1000-1099, with esl_histogram_GetTailByMass and
 * esl_exp_FitComplete, src/easel/histogram.rs:334-355,
 * src/easel/exponential.rs:67-91).  The scan itself is oracle_calib_scan in
 * qdb_oracle.c.  Written loop for loop after the reference, sharing no code
 * with the library.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/cmscan_gpu.h"

typedef struct {
    uint32_t mt[624];
    int mti;
} mtrng;

static void mt_seed_table(mtrng *r, uint32_t seed) {
    r->mt[0] = seed;
    for (int z = 1; z < 624; z++) r->mt[z] = 69069u * r->mt[z - 1];
}

static void mt_fill_table(mtrng *r) {
    static const uint32_t mag01[2] = {0x0u, 0x9908b0dfu};
    uint32_t y;
    int z;
    for (z = 0; z < 227; z++) {
        y = (r->mt[z] & 0x80000000u) | (r->mt[z + 1] & 0x7fffffffu);
        r->mt[z] = r->mt[z + 397] ^ (y >> 1) ^ mag01[y & 0x1u];
    }
    for (z = 227; z < 623; z++) {
        y = (r->mt[z] & 0x80000000u) | (r->mt[z + 1] & 0x7fffffffu);
        r->mt[z] = r->mt[z - 227] ^ (y >> 1) ^ mag01[y & 0x1u];
    }
    y = (r->mt[623] & 0x80000000u) | (r->mt[0] & 0x7fffffffu);
    r->mt[623] = r->mt[396] ^ (y >> 1) ^ mag01[y & 0x1u];
    r->mti = 0;
}

static uint32_t mt_next(mtrng *r) {
    if (r->mti >= 624) mt_fill_table(r);
    uint32_t x = r->mt[r->mti++];
    x ^= (x >> 11);
    x ^= (x << 7) & 0x9d2c5680u;
    x ^= (x << 15) & 0xefc60000u;
    x ^= (x >> 18);
    return x;
}

static double mt_random(mtrng *r) { return (double)mt_next(r) / 4294967296.0; }

static void vec_dnorm(double *v, int n) {
    double sum = 0.0;
    for (int i = 0; i < n; i++) sum += v[i];
    if (sum != 0.0)
        for (int i = 0; i < n; i++) v[i] /= sum;
    else
        for (int i = 0; i < n; i++) v[i] = 1.0 / (double)n;
}

static int dchoose(mtrng *r, const double *p, int n) {
    double roll = mt_random(r);
    double norm = 0.0, sum = 0.0;
    for (int i = 0; i < n; i++) norm += p[i];
    for (int i = 0; i < n; i++) {
        sum += p[i];
        if (roll < (sum / norm)) return i;
    }
    return n - 1;
}

/* new(seed) seeds and fills; init(seed) does the same again. */
int oracle_genomic_sample(uint32_t seed, int32_t L, int32_t nseq, uint8_t *frames) {
    double s_a[5] = {0.157377049180328, 0.39344262295082, 0.265573770491803, 0.00327868852459016,
                     0.180327868852459};
    double t_aa[5][5] = {
        {0.999483637183643, 0.000317942006440604, 0.000185401071732768, 2.60394763669618e-07, 1.27593434198113e-05},
        {9.76333640771184e-05, 0.99980020511745, 9.191359010352e-05, 7.94413051888677e-08, 1.01684870641751e-05},
        {1.3223694798182e-07, 0.000155642887774602, 0.999700615549769, 9.15079680034191e-05, 5.21013575048369e-05},
        {0.994252873563218, 0.0014367816091954, 0.0014367816091954, 0.0014367816091954, 0.0014367816091954},
        {8.32138798088677e-06, 2.16356087503056e-05, 6.42411152124459e-05, 1.66427759617735e-07, 0.999905635460297},
    };
    double e_aa[5][4] = {
        {0.370906566523225, 0.129213995153577, 0.130511270043053, 0.369368168280145},
        {0.305194882571888, 0.194580936415687, 0.192343972160245, 0.307880208852179},
        {0.238484980800698, 0.261262845707113, 0.261810301531792, 0.238441871960397},
        {0.699280575539568, 0.00143884892086331, 0.00143884892086331, 0.297841726618705},
        {0.169064007664923, 0.331718611320207, 0.33045427183482, 0.16876310918005},
    };
    vec_dnorm(s_a, 5);
    for (int i = 0; i < 5; i++) vec_dnorm(t_aa[i], 5);
    for (int i = 0; i < 5; i++) vec_dnorm(e_aa[i], 4);
    mtrng r;
    mt_seed_table(&r, seed);
    mt_fill_table(&r);
    if (seed != 0) {
        mt_seed_table(&r, seed);
        mt_fill_table(&r);
    }
    for (int32_t s = 0; s < nseq; s++) {
        uint8_t *dsq = frames + (size_t)s * ((size_t)L + 2);
        dsq[0] = 255;
        dsq[L + 1] = 255;
        int si = dchoose(&r, s_a, 5);
        for (int32_t x = 1; x <= L; x++) {
            dsq[x] = (uint8_t)dchoose(&r, e_aa[si], 4);
            si = dchoose(&r, t_aa[si], 5);
        }
    }
    return 0;
}

static int cmp_double(const void *a, const void *b) {
    double x = *(const double *)a, y = *(const double *)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

/* fit_histogram (tail mass, GetTailByMass, FitComplete) + set_exp_info.
 * Returns 0, or -5 where the reference returns an error. */
int oracle_exp_fit(const float *scores, int64_t n_scores, int exp_mode, int32_t n_seqs, int32_t l, int32_t gtailn,
                   int32_t ltailn, float tailp_opt, double dbsize, cmgpu_exp_params *out) {
    double *x = (double *)malloc(sizeof(double) * (size_t)(n_scores > 0 ? n_scores : 1));
    for (int64_t k = 0; k < n_scores; k++) {
        if (!isfinite(scores[k])) {
            free(x);
            return -5;
        }
        x[k] = (double)scores[k];
    }
    uint64_t hn = (uint64_t)n_scores;
    float tailp;
    if (tailp_opt > 0.0f) {
        tailp = tailp_opt;
    } else {
        float mb = ((float)n_seqs * (float)l) / 1000000.0f;
        int local = exp_mode == 2 || exp_mode == 3;
        float nhits_to_fit = local ? (float)ltailn * mb : (float)gtailn * mb;
        float tp = nhits_to_fit / (float)hn;
        if (tp > 1.0f) {
            free(x);
            return -5;
        }
        tailp = tp;
    }
    qsort(x, (size_t)hn, sizeof(double), cmp_double);
    uint64_t nn = (uint64_t)((double)hn * (double)tailp);
    if (nn <= 1) {
        free(x);
        return -5;
    }
    const double *xv = x + (hn - nn);
    double mu = xv[0];
    for (uint64_t i = 1; i < nn; i++)
        if (xv[i] < mu) mu = xv[i];
    double mean = 0.0;
    for (uint64_t i = 0; i < nn; i++) mean += xv[i] - mu;
    mean /= (double)nn;
    double lambda = 1.0 / mean;
    free(x);
    if (isnan(lambda) || isinf(lambda)) return -5;
    out->lambda = lambda;
    out->mu_orig = mu;
    out->mu = mu - log(1.0 / (double)tailp) / lambda;
    out->dbsize = dbsize;
    out->nrandhits = (int32_t)hn;
    out->tailp = (double)tailp;
    return 0;
}
