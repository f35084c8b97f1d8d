/*
 * bdc_oracle.c -- CPU restatement of the reference Blahut-Arimoto (BA) path for
 * the binary deletion channel BDC_{n,k}.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: it is loaded by tests/,
 * by __graft_entry__.smoke() and by the cpu_baseline / reference legs of
 * bench.py.  The product (the CUDA engine behind include/bdc_b200.h) never
 * links, loads or calls it.
 *
 * Every function follows one reference function, cited as file:line within the
 * reference project (Pintz45/BDC-Upper-Bounds-GPU):
 *   backend/BAA.cu               kernels and host drivers of one BA iteration
 *   backend/main_BAA.cu          canonical list, BA outer loop, stopping rule
 *   backend/generate_bit_transition_cache.cpp   the cache_n_k generator
 *
 * Strings are integers, MSB first: character i of an n-bit string x is bit
 * (n-1-i) of x (generate_bit_transition_cache.cpp:15, BAA.cu:271).
 *
 * Arithmetic: counts are exact uint32; probabilities and logs are double, with
 * per-x sums and the q accumulation in long double so that the oracle is at
 * least as accurate as the reference's own double arithmetic.
 *
 * Threads: OpenMP over canonical representatives ("reps").  The number of
 * threads is whatever the caller sets via oracle_set_threads() (default: all).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORACLE_MAX_N 32

/* ------------------------------------------------------------------------ */
/* threads                                                                  */
/* ------------------------------------------------------------------------ */
void oracle_set_threads(int t) {
#ifdef _OPENMP
    if (t > 0) omp_set_num_threads(t);
#else
    (void)t;
#endif
}

int oracle_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/* binomial  (BAA.cu:15-24)                                                 */
/* ------------------------------------------------------------------------ */
uint32_t oracle_nck(uint32_t n, uint32_t k) {
    if (k > n) return 0;
    if (k > n - k) k = n - k;
    uint64_t r = 1;
    for (uint32_t i = 1; i <= k; ++i) r = r * (n - i + 1) / i;
    return (uint32_t)r;
}

/* ------------------------------------------------------------------------ */
/* symmetry group {id, reverse, complement, reverse-complement}             */
/* (BAA.cu:195-258)                                                         */
/* ------------------------------------------------------------------------ */
static uint32_t rev_bits(uint32_t x, int len) {
    uint32_t r = 0;
    for (int i = 0; i < len; ++i) r |= ((x >> i) & 1u) << (len - 1 - i);
    return r;
}

static uint32_t cmp_bits(uint32_t x, int len) {
    uint32_t m = (len >= 32) ? 0xFFFFFFFFu : ((1u << len) - 1u);
    return x ^ m;
}

/* rep(x) = min over the orbit (BAA.cu:216-227) */
uint32_t oracle_rep(uint32_t x, int len) {
    uint32_t r = rev_bits(x, len), c = cmp_bits(x, len), rc = rev_bits(c, len);
    uint32_t m = x;
    if (r < m) m = r;
    if (c < m) m = c;
    if (rc < m) m = rc;
    return m;
}

/* |orbit(x)| = 2 if x is fixed by reverse or by reverse-complement, else 4
 * (BAA.cu:230-241) */
int oracle_orbit(uint32_t x, int len) {
    uint32_t r = rev_bits(x, len), rc = rev_bits(cmp_bits(x, len), len);
    return (x == r || x == rc) ? 2 : 4;
}

/* canonical list in ascending order (main_BAA.cu:46-50).  Returns the count;
 * writes at most cap entries to out (out may be NULL to only count). */
int64_t oracle_canonicals(int n, uint32_t* out, int64_t cap) {
    int64_t c = 0;
    uint64_t total = 1ull << n;
    for (uint64_t x = 0; x < total; ++x) {
        if (oracle_rep((uint32_t)x, n) != (uint32_t)x) continue;
        if (out && c < cap) out[c] = (uint32_t)x;
        ++c;
    }
    return c;
}

/* ------------------------------------------------------------------------ */
/* subsequence counts                                                        */
/* ------------------------------------------------------------------------ */
/* number of occurrences of y (k bits) as a subsequence of x (n bits):
 * the prefix DP of generate_bit_transition_cache.cpp:23-44 */
uint32_t oracle_count_dp(uint32_t x, int n, uint32_t y, int k) {
    uint32_t dp[ORACLE_MAX_N + 1];
    if (k > n) return 0;
    dp[0] = 1;
    for (int j = 1; j <= k; ++j) dp[j] = 0;
    for (int i = 1; i <= n; ++i) {
        uint32_t xi = (x >> (n - i)) & 1u;
        for (int j = (i < k ? i : k); j >= 1; --j) {
            uint32_t yj = (y >> (k - j)) & 1u;
            if (xi == yj) dp[j] += dp[j - 1];
        }
    }
    return dp[k];
}

/* the full table cache_{n,k}: out[(x << k) | y] = count (generate_bit_
 * transition_cache.cpp:46-77, layout of cache_io.h:17-26) */
void oracle_gen_cache(int n, int k, uint32_t* out) {
    int64_t nx = 1ll << n;
    int64_t ny = 1ll << k;
#pragma omp parallel for schedule(static)
    for (int64_t x = 0; x < nx; ++x)
        for (int64_t y = 0; y < ny; ++y)
            out[(x << k) | y] = oracle_count_dp((uint32_t)x, n, (uint32_t)y, k);
}

/* ---- per-x DP of distinct subsequences (BAA.cu:261-303) ---- */
typedef struct {
    uint8_t nextpos[ORACLE_MAX_N + 2][2];
    uint32_t cnt[ORACLE_MAX_N + 2][ORACLE_MAX_N + 2];
} dp_tables;

static void fill_dp(uint32_t x, int n, int k, dp_tables* t) {
    for (int b = 0; b < 2; ++b) {
        for (int i = 0; i <= n; ++i) t->nextpos[i][b] = (uint8_t)n;
        int last = n;
        for (int i = n - 1; i >= 0; --i) {
            uint32_t xi = (x >> (n - i - 1)) & 1u;
            if ((int)xi == b) last = i;
            t->nextpos[i][b] = (uint8_t)last;
        }
    }
    for (int i = 0; i <= n; ++i) {
        t->cnt[i][0] = 1;
        for (int r = 1; r <= k; ++r) t->cnt[i][r] = 0;
    }
    for (int i = n - 1; i >= 0; --i)
        for (int r = 1; r <= k; ++r) {
            uint32_t tot = 0;
            int j0 = t->nextpos[i][0], j1 = t->nextpos[i][1];
            if (j0 < n) tot += t->cnt[j0 + 1][r - 1];
            if (j1 < n) tot += t->cnt[j1 + 1][r - 1];
            t->cnt[i][r] = tot;
        }
}

/* j-th distinct length-k subsequence, 0 before 1 (BAA.cu:304-335) */
static uint32_t unrank(const dp_tables* t, int n, int k, uint32_t j) {
    int i = 0, rem = k;
    uint32_t y = 0;
    while (rem > 0) {
        int j0 = t->nextpos[i][0];
        uint32_t c0 = (j0 < n) ? t->cnt[j0 + 1][rem - 1] : 0;
        if (j < c0) { i = j0 + 1; --rem; continue; }
        j -= c0;
        int j1 = t->nextpos[i][1];
        y |= 1u << (rem - 1);
        i = j1 + 1;
        --rem;
    }
    return y;
}

/* number of distinct length-k subsequences of x */
uint32_t oracle_num_distinct(uint32_t x, int n, int k) {
    dp_tables t;
    fill_dp(x, n, k, &t);
    return t.cnt[0][k];
}

/* all distinct length-k subsequences of x in unrank order; returns count */
uint32_t oracle_distinct_subsequences(uint32_t x, int n, int k, uint32_t* out) {
    dp_tables t;
    fill_dp(x, n, k, &t);
    uint32_t c = t.cnt[0][k];
    for (uint32_t j = 0; j < c; ++j) out[j] = unrank(&t, n, k, j);
    return c;
}

/* N(x,y) by the split identity over half tables (BAA.cu:340-395):
 * n1 = ceil(n/2), n2 = n - n1; the left half uses cache_{n1, j}, the right
 * half cache_{n2, k-j}, and a half whose length equals its sub-word length is
 * an equality test.  The half tables are recomputed here by the prefix DP,
 * which is what the cache files hold. */
uint32_t oracle_total_transitions(uint32_t x, uint32_t y, int n, int k) {
    int n1 = (n + 1) / 2, n2 = n - n1;
    uint32_t x1 = x >> n2, x2 = x & ((1u << n2) - 1u);
    uint32_t tot = 0;
    for (int j = 0; j <= k; ++j) {
        if (j > n1 || (k - j) > n2) continue;
        uint32_t y1 = (k - j >= 32) ? 0 : (y >> (k - j));
        uint32_t y2 = y & (((k - j) >= 32) ? 0xFFFFFFFFu : ((1u << (k - j)) - 1u));
        uint32_t c1 = (j == n1) ? (x1 == y1) : oracle_count_dp(x1, n1, y1, j);
        uint32_t c2 = (k - j == n2) ? (x2 == y2) : oracle_count_dp(x2, n2, y2, k - j);
        tot += c1 * c2;
    }
    return tot;
}

/* ------------------------------------------------------------------------ */
/* one BA iteration, split as the reference splits it                        */
/* ------------------------------------------------------------------------ */
/* Table-driven N(x,y): the half tables are materialised once per call so the
 * per-pair cost matches the reference's lookup (BAA.cu:376-387). */
typedef struct {
    int n, k, n1, n2;
    uint32_t* t1[ORACLE_MAX_N + 1]; /* cache_{n1, j}, j < n1 */
    uint32_t* t2[ORACLE_MAX_N + 1]; /* cache_{n2, m}, m < n2 */
} half_tables;

static void ht_build(half_tables* h, int n, int k) {
    memset(h, 0, sizeof(*h));
    h->n = n; h->k = k; h->n1 = (n + 1) / 2; h->n2 = n - h->n1;
    for (int j = 0; j <= k && j < h->n1; ++j) {
        if (k - j > h->n2) continue;
        h->t1[j] = (uint32_t*)malloc(sizeof(uint32_t) << (h->n1 + j));
        oracle_gen_cache(h->n1, j, h->t1[j]);
    }
    for (int m = 0; m <= k && m < h->n2; ++m) {
        if (k - m > h->n1) continue;
        h->t2[m] = (uint32_t*)malloc(sizeof(uint32_t) << (h->n2 + m));
        oracle_gen_cache(h->n2, m, h->t2[m]);
    }
}

static void ht_free_all(half_tables* h) {
    for (int i = 0; i <= ORACLE_MAX_N; ++i) { free(h->t1[i]); free(h->t2[i]); }
    memset(h, 0, sizeof(*h));
}

/* The half tables of the last (n,k) stay cached between calls, so that
 * timing a pass does not re-time the table generation.  Not thread-safe
 * across concurrent callers (the oracle is driven from one host thread). */
static half_tables g_ht;
static int g_ht_valid = 0;

static void ht_get(half_tables* h, int n, int k) {
    if (!g_ht_valid || g_ht.n != n || g_ht.k != k) {
        if (g_ht_valid) ht_free_all(&g_ht);
        ht_build(&g_ht, n, k);
        g_ht_valid = 1;
    }
    *h = g_ht;
}

static void ht_free(half_tables* h) { (void)h; }

void oracle_release_tables(void) {
    if (g_ht_valid) ht_free_all(&g_ht);
    g_ht_valid = 0;
}

static inline uint32_t ht_count(const half_tables* h, uint32_t x, uint32_t y) {
    int n1 = h->n1, n2 = h->n2, k = h->k;
    uint32_t x1 = x >> n2, x2 = x & ((1u << n2) - 1u);
    uint32_t tot = 0;
    for (int j = 0; j <= k; ++j) {
        if (j > n1 || (k - j) > n2) continue;
        uint32_t y1 = y >> (k - j), y2 = y & ((1u << (k - j)) - 1u);
        uint32_t c1 = (j == n1) ? (x1 == y1) : h->t1[j][(x1 << j) | y1];
        uint32_t c2 = (k - j == n2) ? (x2 == y2) : h->t2[k - j][(x2 << (k - j)) | y2];
        tot += c1 * c2;
    }
    return tot;
}

/* counts for a list of (x, y) pairs through the split identity */
void oracle_counts_pairs(int n, int k, const uint32_t* xs, const uint32_t* ys,
                         int64_t npairs, uint32_t* out) {
    half_tables h;
    ht_get(&h, n, k);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < npairs; ++i) out[i] = ht_count(&h, xs[i], ys[i]);
    ht_free(&h);
}

/* dense rows N(x, .) for listed x: out[i * 2^k + y] */
void oracle_count_rows(int n, int k, const uint32_t* xs, int64_t nx, uint32_t* out) {
    half_tables h;
    ht_get(&h, n, k);
    int64_t ny = 1ll << k;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nx; ++i)
        for (int64_t y = 0; y < ny; ++y) out[i * ny + y] = ht_count(&h, xs[i], (uint32_t)y);
    ht_free(&h);
}

/* ln with the reference's convention that 0 stays 0 (BAA.cu:573-580) */
static inline double log_keep0(double v) { return v != 0.0 ? log(v) : 0.0; }

/* q-pass: ln q over the 2^{k-1} rep-value slots (BAA.cu:429-485 kernel,
 * 573-580 log, 642-724 host).  For each canonical x and each distinct y of x:
 *   q[rep(y)] += |O(x)| / |O(y)| * p(x) * N(x,y) / C(n,k)                   */
void oracle_log_q(int n, int k, const double* p, const uint32_t* reps, int64_t R,
                  double* lnq_out) {
    half_tables h;
    ht_get(&h, n, k);
    int64_t nq = 1ll << (k - 1 > 0 ? k - 1 : 0);
    if (k == 0) nq = 1;
    double inv_c = 1.0 / (double)oracle_nck(n, k); /* BAA.cu:108 */
    int nt = oracle_get_threads();
    long double* part = (long double*)calloc((size_t)nt * nq, sizeof(long double));
#pragma omp parallel
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        long double* mine = part + (size_t)tid * nq;
        dp_tables t;
#pragma omp for schedule(dynamic, 64)
        for (int64_t i = 0; i < R; ++i) {
            uint32_t x = reps[i];
            fill_dp(x, n, k, &t);
            double ox = (double)oracle_orbit(x, n);
            uint32_t cnt = t.cnt[0][k];
            for (uint32_t j = 0; j < cnt; ++j) {
                uint32_t y = unrank(&t, n, k, j);
                uint32_t ry = oracle_rep(y, k);
                double oy = (double)oracle_orbit(y, k);
                double w = p[i] * (double)ht_count(&h, x, y) * inv_c; /* BAA.cu:397-399 */
                mine[ry] += (long double)((ox / oy) * w);
            }
        }
    }
    for (int64_t s = 0; s < nq; ++s) {
        long double acc = 0.0L;
        for (int tt = 0; tt < nt; ++tt) acc += part[(size_t)tt * nq + s];
        lnq_out[s] = log_keep0((double)acc);
    }
    free(part);
    ht_free(&h);
}

/* per-x sum over distinct y of W * (ln W + lnp_x - lnq[rep y]) -- the
 * reference's log_W (BAA.cu:401-411, 487-530) when with_lnp != 0, and KL(x)
 * = D(x) (BAA.cu:413-425, 533-571) when with_lnp == 0 */
static void per_x_divergence(int n, int k, const double* p, const uint32_t* reps,
                             int64_t R, const double* lnq, int with_lnp, double* out) {
    half_tables h;
    ht_get(&h, n, k);
    double C = (double)oracle_nck(n, k);
    double inv_c = 1.0 / C;
    double neg_log_c = -log(C);
#pragma omp parallel
    {
        dp_tables t;
#pragma omp for schedule(dynamic, 64)
        for (int64_t i = 0; i < R; ++i) {
            uint32_t x = reps[i];
            fill_dp(x, n, k, &t);
            double lp = with_lnp ? log_keep0(p[i]) : 0.0;
            long double acc = 0.0L;
            uint32_t cnt = t.cnt[0][k];
            for (uint32_t j = 0; j < cnt; ++j) {
                uint32_t y = unrank(&t, n, k, j);
                uint32_t N = ht_count(&h, x, y);
                double W = (double)N * inv_c;
                double lW = log((double)N) + neg_log_c;
                acc += (long double)(W * (lW + lp - lnq[oracle_rep(y, k)]));
            }
            out[i] = (double)acc;
        }
    }
    ht_free(&h);
}

void oracle_log_w(int n, int k, const double* p, const double* lnq,
                  const uint32_t* reps, int64_t R, double* logw_out) {
    per_x_divergence(n, k, p, reps, R, lnq, 1, logw_out);
}

void oracle_kl(int n, int k, const double* lnq, const uint32_t* reps, int64_t R,
               double* kl_out) {
    per_x_divergence(n, k, NULL, reps, R, lnq, 0, kl_out);
}

/* normalised update p' = exp(logW - max) / sum |O| exp(logW - max)
 * (BAA.cu:590-639) */
void oracle_normalise(int n, const double* logw, const uint32_t* reps, int64_t R,
                      double* p_out) {
    double mx = -INFINITY;
    for (int64_t i = 0; i < R; ++i) if (logw[i] > mx) mx = logw[i];
    long double s = 0.0L;
    for (int64_t i = 0; i < R; ++i) {
        p_out[i] = exp(logw[i] - mx);
        s += (long double)oracle_orbit(reps[i], n) * (long double)p_out[i];
    }
    double sd = (double)s;
    for (int64_t i = 0; i < R; ++i) p_out[i] = p_out[i] / sd;
}

/* one BA iteration (BAA.cu:590-639); also returns lnq and logW if asked */
void oracle_ba_iteration(int n, int k, const double* p, const uint32_t* reps, int64_t R,
                         double* p_out, double* lnq_out, double* logw_out) {
    int64_t nq = (k >= 1) ? (1ll << (k - 1)) : 1;
    double* lnq = lnq_out ? lnq_out : (double*)malloc(sizeof(double) * nq);
    double* lw = logw_out ? logw_out : (double*)malloc(sizeof(double) * R);
    oracle_log_q(n, k, p, reps, R, lnq);
    oracle_log_w(n, k, p, lnq, reps, R, lw);
    oracle_normalise(n, lw, reps, R, p_out);
    if (!lnq_out) free(lnq);
    if (!logw_out) free(lw);
}

/* mx = max_i log2 p_i - log2 pb_i (BAA.cu:916-946) */
double oracle_max_deviation(const double* p, const double* pb, int64_t R) {
    double m = -INFINITY;
    for (int64_t i = 0; i < R; ++i) {
        double v = log2(p[i]) - log2(pb[i]);
        if (v > m || isnan(v)) m = (isnan(m) || isnan(v)) ? NAN : v;
    }
    return m;
}

/* I(p;W) in nats = sum |O| p KL (BAA.cu:820-913) */
double oracle_rate(int n, int k, const double* lnq, const double* p,
                   const uint32_t* reps, int64_t R) {
    double* kl = (double*)malloc(sizeof(double) * R);
    oracle_kl(n, k, lnq, reps, R, kl);
    long double s = 0.0L;
    for (int64_t i = 0; i < R; ++i)
        s += (long double)oracle_orbit(reps[i], n) * (long double)p[i] * (long double)kl[i];
    free(kl);
    return (double)s;
}

/* ------------------------------------------------------------------------ */
/* the BA outer loop (main_BAA.cu:39-131)                                    */
/* ------------------------------------------------------------------------ */
/* Runs `while (mx >= a)` from p (in place) for at most max_iters iterations.
 * Per iteration t it records mx_t, and the upper bound max_x D_t(x) in bits
 * computed from the iterate the step started from.  Returns iterations done;
 * *rate_bits gets I(p_final; W) with a fresh q (main_BAA.cu:123-125). */
int64_t oracle_run_ba(int n, int k, double* p, const uint32_t* reps, int64_t R,
                      double a, int64_t max_iters, double* mx_log, double* ub_log,
                      double* rate_bits, double* mx_final) {
    int64_t nq = (k >= 1) ? (1ll << (k - 1)) : 1;
    double* lnq = (double*)malloc(sizeof(double) * nq);
    double* lw = (double*)malloc(sizeof(double) * R);
    double* pn = (double*)malloc(sizeof(double) * R);
    double mx = a;
    int64_t it = 0;
    const double LN2 = 0.69314718055994530942;
    while (mx >= a && it < max_iters) {
        oracle_log_q(n, k, p, reps, R, lnq);
        oracle_log_w(n, k, p, lnq, reps, R, lw);
        if (ub_log) {
            double ub = -INFINITY;
            for (int64_t i = 0; i < R; ++i) {
                double d = lw[i] - log_keep0(p[i]);
                if (d > ub) ub = d;
            }
            ub_log[it] = ub / LN2;
        }
        oracle_normalise(n, lw, reps, R, pn);
        mx = oracle_max_deviation(pn, p, R);
        if (mx_log) mx_log[it] = mx;
        memcpy(p, pn, sizeof(double) * R);
        ++it;
    }
    if (rate_bits) {
        oracle_log_q(n, k, p, reps, R, lnq);
        *rate_bits = oracle_rate(n, k, lnq, p, reps, R) / LN2;
    }
    if (mx_final) *mx_final = mx;
    free(lnq); free(lw); free(pn);
    return it;
}
