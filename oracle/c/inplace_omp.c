/* ORACLE (test infrastructure; CPU baseline only).
 *
 * C + OpenMP restatement of the reference's one-buffer executor `execute_inplace`
 * (source/kernel_opt/inplace_plan.py:90-135) in complex128: per vertex step, every orbit of
 * 1, 2 or 4 entries is read before it is written, then the active entries are renormalised
 * by 2^-frexp(max|x|) and the exponent is added to the log scale.  The orbit formulas follow
 * the reference's kinds (inplace_gpu.py:29-58).  Never linked into the product.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

typedef double complex cplx;

/* byte address tables, as the reference's executors use (scan_plan.py:133-145):
 * c = XOR over bytes b of T[b][(x >> 8b) & 255] */
static void make_tables(const int *slots, int m, uint64_t T[8][256]) {
    for (int b = 0; b < 8; ++b)
        for (int v = 0; v < 256; ++v) {
            uint64_t acc = 0;
            for (int t = 0; t < 8; ++t) {
                const int i = 8 * b + t;
                if (i < m && ((v >> t) & 1)) acc |= 1ull << slots[i];
            }
            T[b][v] = acc;
        }
}

static inline uint64_t deposit_t(uint64_t x, uint64_t T[8][256], int nb) {
    uint64_t c = 0;
    for (int b = 0; b < nb; ++b) c ^= T[b][(x >> (8 * b)) & 255];
    return c;
}

static inline double sgn(uint64_t c, uint64_t beta, int ov) {
    return ((__builtin_popcountll(c & beta) & 1) ^ ov) ? -1.0 : 1.0;
}

static int mask_slots(uint64_t mask, int *slots) {
    int m = 0;
    for (int p = 0; p < 64; ++p)
        if ((mask >> p) & 1) slots[m++] = p;
    return m;
}

/* steps: per step 8 words: kind, K, Ka, beta, pivot_bit, enum_mask, out_mask, unused
 * params: per step 6 doubles: f0r f0i f1r f1i ov y.  Runs steps [first, first+count).
 * E: 2^maxslots complex128 (E[0] = 1 before the first step).  Returns the added log scale. */
double oracle_run_steps(const uint64_t *steps, const double *params, int first, int count, cplx *E) {
    double ls = 0.0;
    for (int s = first; s < first + count; ++s) {
        const uint64_t *d = steps + 8 * s;
        const int kind = (int)d[0];
        const uint64_t K = d[1], Ka = d[2], beta = d[3], pbit = d[4];
        const double *p = params + 6 * s;
        const cplx f0 = p[0] + I * p[1], f1 = p[2] + I * p[3];
        const int ov = (int)p[4], y = (int)p[5];
        int slots[64], oslots[64];
        const int m = mask_slots(d[5], slots);
        const int mo = mask_slots(d[6], oslots);
        const int64_t n = (int64_t)1 << m;
        static uint64_t Ti[8][256], To[8][256];
        make_tables(slots, m, Ti);
        make_tables(oslots, mo, To);
        const int nbi = (m + 7) / 8, nbo = (mo + 7) / 8;
#pragma omp parallel for schedule(static)
        for (int64_t x = 0; x < n; ++x) {
            const uint64_t c = deposit_t((uint64_t)x, Ti, nbi);
            const cplx a = E[c];
            switch (kind) {
                case 0: E[c] = f0 * a; E[c | pbit] = f1 * a * sgn(c, beta, ov); break;
                case 1: { const uint64_t dd = c ^ Ka; const cplx b = E[dd];
                          E[c] = f0 * a + f1 * sgn(dd, beta, ov) * b; E[dd] = f0 * b + f1 * sgn(c, beta, ov) * a; } break;
                case 2: E[c] = (f0 + f1 * sgn(c, beta, ov)) * a; break;
                case 3: { const uint64_t dd = c ^ K; const cplx b = E[dd];
                          E[c] = f0 * (a + b); E[dd] = f1 * (sgn(c, beta, ov) * a + sgn(dd, beta, ov) * b); } break;
                case 4: E[c] = (y ? f1 * sgn(c, beta, ov) : f0) * a; break;
                case 5: { const uint64_t dd = c ^ K; const cplx b = E[dd];
                          E[c] = y ? f1 * (sgn(c, beta, ov) * a + sgn(dd, beta, ov) * b) : f0 * (a + b); } break;
                case 6: { const uint64_t c1 = c ^ K, dd = c ^ Ka, d1 = dd ^ K;
                          const cplx b = E[c1], e = E[dd], g = E[d1];
                          E[c] = f0 * (a + b) + f1 * (sgn(dd, beta, ov) * e + sgn(d1, beta, ov) * g);
                          E[dd] = f0 * (e + g) + f1 * (sgn(c, beta, ov) * a + sgn(c1, beta, ov) * b); } break;
                default: { const uint64_t dd = c ^ K; const cplx b = E[dd];
                           E[c] = (f0 + f1 * sgn(c, beta, ov)) * a + (f0 + f1 * sgn(dd, beta, ov)) * b; } break;
            }
        }
        const int64_t no = (int64_t)1 << mo;
        double mx = 0.0;
#pragma omp parallel for reduction(max : mx) schedule(static)
        for (int64_t x = 0; x < no; ++x) {
            const double v = cabs(E[deposit_t((uint64_t)x, To, nbo)]);
            if (v > mx) mx = v;
        }
        if (mx > 0.0) {
            int e;
            frexp(mx, &e);
            const double sc = ldexp(1.0, -e);
#pragma omp parallel for schedule(static)
            for (int64_t x = 0; x < no; ++x) E[deposit_t((uint64_t)x, To, nbo)] *= sc;
            ls += e * log(2.0);
        }
    }
    return ls;
}

int oracle_threads(void) {
#ifdef _OPENMP
    extern int omp_get_max_threads(void);
    return omp_get_max_threads();
#else
    return 1;
#endif
}
