/*
 * CPU oracle for exact brute-force Euclidean neighbour search.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product imports, links or calls
 * this file; it is the checker that tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py compare the CUDA library against.
 *
 * It restates the results contract of mlxlearn's neighbour path:
 *
 *  - kNN order is the exact real squared distance of the float32 coordinates,
 *    ties broken by the smaller training index
 *    (src/mlxlearn/_kernels/_neighbors_cpu_native.cpp:170-190,301-360;
 *     src/mlxlearn/_kernels/neighbors_cpu.py:1-15).
 *  - radius membership is exact: S(q,x) <= fl64(r*r)
 *    (src/mlxlearn/_kernels/radius_contract.py:1-25,129-217).
 *  - reported distances are sqrt of the canonical float64 value, a strictly
 *    sequential sum over features of (double(q_k) - double(x_k))^2 with no
 *    FMA (src/mlxlearn/_kernels/_radius_common.h:348-358); radius distances are
 *    sqrt(min(canonical, R2)) (src/mlxlearn/_kernels/radius_cpu.py:7-16).
 *
 * The exact comparison is written from the mathematics, not from the
 * reference's code: every float32 value is an integer multiple of 2^-149, so
 * each coordinate difference is an exact integer D_i in those units and
 * S * 2^298 = sum_i D_i^2 is an exact non-negative integer.  We form each D_i
 * as a multi-limb integer, square it, and add the square into a 640-bit
 * accumulator.  All terms are non-negative, so no borrow handling is needed.
 *
 * Parity of this oracle is pinned by tests/test_oracle.py against the
 * reference's own outputs (golden fixtures produced by tests/golden/
 * make_golden.py from the reference's CPU path) and against the known-answer
 * cases in the reference's tests.
 *
 * Build: oracle/Makefile  (gcc -O2 -ffp-contract=off -pthread -shared -fPIC).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define KEY_LIMBS 10 /* 640 bits: squares reach 2^556, sums of 2^31 terms 2^587 */

typedef struct {
    uint64_t w[KEY_LIMBS];
} okey;

typedef unsigned __int128 u128;

static uint32_t f32_bits(float v) {
    uint32_t b;
    memcpy(&b, &v, 4);
    return b;
}

/* v = (-1)^neg * m * 2^(e - 149), m < 2^24, 0 <= e <= 253. */
static void f32_decode(float v, uint64_t *m, int *e, int *neg) {
    uint32_t b = f32_bits(v);
    uint32_t ex = (b >> 23) & 255u;
    *m = (uint64_t)((b & 0x7fffffu) | (ex ? 0x800000u : 0u));
    *e = ex ? (int)ex - 1 : 0;
    *neg = (int)(b >> 31);
}

/* dst (n limbs) = src (up to 1 limb) << shift, shift < 64*n. */
static void big_from_shifted(uint64_t *dst, int n, uint64_t v, int shift) {
    memset(dst, 0, sizeof(uint64_t) * (size_t)n);
    int limb = shift >> 6, bit = shift & 63;
    dst[limb] = v << bit;
    if (bit && limb + 1 < n) dst[limb + 1] = v >> (64 - bit);
}

/* Compare two n-limb integers. */
static int big_cmp(const uint64_t *a, const uint64_t *b, int n) {
    for (int i = n - 1; i >= 0; --i) {
        if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
    }
    return 0;
}

/* r = a - b (a >= b), n limbs. */
static void big_sub(uint64_t *r, const uint64_t *a, const uint64_t *b, int n) {
    uint64_t borrow = 0;
    for (int i = 0; i < n; ++i) {
        uint64_t bi = b[i] + borrow;
        uint64_t nb = (bi < borrow) || (a[i] < bi);
        r[i] = a[i] - bi;
        borrow = nb;
    }
}

/* r = a + b, n limbs (no overflow by construction). */
static void big_add(uint64_t *r, const uint64_t *a, const uint64_t *b, int n) {
    uint64_t carry = 0;
    for (int i = 0; i < n; ++i) {
        u128 s = (u128)a[i] + b[i] + carry;
        r[i] = (uint64_t)s;
        carry = (uint64_t)(s >> 64);
    }
}

/* acc += v << shift (v has nv limbs). */
static void key_add_shifted(okey *acc, const uint64_t *v, int nv, int shift) {
    int base = shift >> 6, bit = shift & 63;
    uint64_t carry = 0;
    for (int i = 0; i + base < KEY_LIMBS; ++i) {
        uint64_t part = 0;
        if (i < nv) part = v[i] << bit;
        if (bit && i > 0 && i - 1 < nv) part |= v[i - 1] >> (64 - bit);
        u128 s = (u128)acc->w[i + base] + part + carry;
        acc->w[i + base] = (uint64_t)s;
        carry = (uint64_t)(s >> 64);
        if (i >= nv && !carry) break;
    }
}

/* S(q, x) * 2^298 as an exact 640-bit integer. */
static void exact_key(const float *q, const float *x, int64_t d, okey *out) {
    memset(out, 0, sizeof(*out));
    for (int64_t i = 0; i < d; ++i) {
        uint64_t ma, mb;
        int ea, eb, na, nb;
        f32_decode(q[i], &ma, &ea, &na);
        f32_decode(x[i], &mb, &eb, &nb);
        if (!ma && !mb) continue;
        int e0 = ea < eb ? ea : eb;
        /* |D| = | (-1)^na ma 2^(ea-e0) - (-1)^nb mb 2^(eb-e0) | in units 2^(e0-149) */
        uint64_t A[5], B[5], D[5];
        big_from_shifted(A, 5, ma, ea - e0);
        big_from_shifted(B, 5, mb, eb - e0);
        if (na == nb) {
            if (big_cmp(A, B, 5) >= 0) big_sub(D, A, B, 5);
            else big_sub(D, B, A, 5);
        } else {
            big_add(D, A, B, 5);
        }
        int nd = 5;
        while (nd > 0 && D[nd - 1] == 0) --nd;
        if (!nd) continue;
        /* D^2, schoolbook */
        uint64_t sq[10];
        memset(sq, 0, sizeof(sq));
        for (int a = 0; a < nd; ++a) {
            uint64_t carry = 0;
            for (int b = 0; b < nd; ++b) {
                u128 t = (u128)D[a] * D[b] + sq[a + b] + carry;
                sq[a + b] = (uint64_t)t;
                carry = (uint64_t)(t >> 64);
            }
            int pos = a + nd;
            while (carry && pos < 10) {
                u128 t = (u128)sq[pos] + carry;
                sq[pos] = (uint64_t)t;
                carry = (uint64_t)(t >> 64);
                ++pos;
            }
        }
        int ns = 2 * nd;
        while (ns > 0 && sq[ns - 1] == 0) --ns;
        key_add_shifted(out, sq, ns, 2 * e0);
    }
}

static int key_cmp(const okey *a, const okey *b) { return big_cmp(a->w, b->w, KEY_LIMBS); }

/* Canonical float64 squared distance: strictly sequential, no contraction. */
static double canonical_d2(const float *q, const float *x, int64_t d) {
    double s = 0.0;
    for (int64_t i = 0; i < d; ++i) {
        double t = (double)q[i] - (double)x[i];
        s = s + t * t;
    }
    return s;
}

/* ---------------------------------------------------------------- public */

/* Exact sign of S(q,a) - S(q,b): -1, 0, 1. */
int orc_exact_compare(const float *q, const float *a, const float *b, int64_t d) {
    okey ka, kb;
    exact_key(q, a, d, &ka);
    exact_key(q, b, d, &kb);
    return key_cmp(&ka, &kb);
}

/* Exact key as 10 little-endian uint64 limbs (units 2^-298). */
void orc_exact_key(const float *q, const float *x, int64_t d, uint64_t *out10) {
    okey k;
    exact_key(q, x, d, &k);
    memcpy(out10, k.w, sizeof(k.w));
}

void orc_canonical_d2(const float *q, const float *x, int64_t d, int64_t n, double *out) {
    for (int64_t j = 0; j < n; ++j) out[j] = canonical_d2(q, x + j * d, d);
}

/* ------------------------------------------------------------------ kNN */

typedef struct {
    double s, lo, hi;
    int64_t idx;
    int have_key;
    okey key;
} cand;

static int cand_cmp(cand *a, cand *b, const float *q, const float *X, int64_t d) {
    if (a->hi < b->lo) return -1;
    if (a->lo > b->hi) return 1;
    if (!(a->s == 0.0 && b->s == 0.0)) {
        if (!a->have_key) { exact_key(q, X + a->idx * d, d, &a->key); a->have_key = 1; }
        if (!b->have_key) { exact_key(q, X + b->idx * d, d, &b->key); b->have_key = 1; }
        int c = key_cmp(&a->key, &b->key);
        if (c) return c;
    }
    return a->idx < b->idx ? -1 : (a->idx > b->idx ? 1 : 0);
}

typedef struct {
    const float *X, *Q;
    int64_t n, d, m, k, q_offset;
    int exclude_self;
    double *dist; /* sqrt(canonical), may be NULL */
    int64_t *idx;
    int64_t begin, end;
} knn_job;

static void *knn_worker(void *arg) {
    knn_job *J = (knn_job *)arg;
    const double u = ldexp(1.0, -53);
    /* canonical sum of d non-negative terms: |s - S| <= g S, g = (d+2)u/(1-(d+2)u);
       the interval uses 2g for slack (radius_contract.py:16-25). */
    const double g = (double)(J->d + 2) * u / (1.0 - (double)(J->d + 2) * u);
    const double f_lo = 1.0 - 2.0 * g, f_hi = 1.0 + 2.0 * g;
    cand *best = (cand *)malloc(sizeof(cand) * (size_t)(J->k + 1));
    for (int64_t r = J->begin; r < J->end; ++r) {
        const float *q = J->Q + r * J->d;
        int64_t count = 0;
        for (int64_t j = 0; j < J->n; ++j) {
            if (J->exclude_self && j == J->q_offset + r) continue;
            cand c;
            c.s = canonical_d2(q, J->X + j * J->d, J->d);
            c.lo = c.s * f_lo;
            c.hi = c.s * f_hi;
            c.idx = j;
            c.have_key = 0;
            if (count == J->k) {
                if (c.lo > best[J->k - 1].hi) continue;
                if (cand_cmp(&c, &best[J->k - 1], q, J->X, J->d) >= 0) continue;
            }
            int64_t pos = count < J->k ? count : J->k - 1;
            while (pos > 0 && cand_cmp(&c, &best[pos - 1], q, J->X, J->d) < 0) {
                best[pos] = best[pos - 1];
                --pos;
            }
            best[pos] = c;
            if (count < J->k) ++count;
        }
        for (int64_t t = 0; t < J->k; ++t) {
            J->idx[r * J->k + t] = t < count ? best[t].idx : -1;
            if (J->dist) J->dist[r * J->k + t] = t < count ? sqrt(best[t].s) : INFINITY;
        }
    }
    free(best);
    return NULL;
}

static int run_jobs(void *(*fn)(void *), void *jobs, size_t job_size, int nthreads) {
    if (nthreads <= 1) {
        fn(jobs);
        return 0;
    }
    pthread_t *t = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)nthreads);
    int started = 0;
    for (int i = 0; i < nthreads; ++i) {
        if (pthread_create(&t[i], NULL, fn, (char *)jobs + job_size * (size_t)i) == 0) ++started;
        else fn((char *)jobs + job_size * (size_t)i);
    }
    for (int i = 0; i < started; ++i) pthread_join(t[i], NULL);
    free(t);
    return 0;
}

/* Exact kNN: rows ordered by (S, index); dist = sqrt(canonical d2). */
int orc_knn(const float *X, int64_t n, int64_t d, const float *Q, int64_t m, int64_t k,
            int exclude_self, int64_t q_offset, double *dist, int64_t *idx, int nthreads) {
    if (n <= 0 || d <= 0 || k <= 0 || k > n - (exclude_self ? 1 : 0) || m < 0) return -1;
    if (nthreads < 1) nthreads = 1;
    if ((int64_t)nthreads > m) nthreads = m > 0 ? (int)m : 1;
    knn_job *jobs = (knn_job *)calloc((size_t)nthreads, sizeof(knn_job));
    int64_t per = (m + nthreads - 1) / nthreads;
    for (int i = 0; i < nthreads; ++i) {
        jobs[i] = (knn_job){X, Q, n, d, m, k, q_offset, exclude_self, dist, idx, 0, 0};
        jobs[i].begin = i * per < m ? i * per : m;
        jobs[i].end = (i + 1) * per < m ? (i + 1) * per : m;
    }
    run_jobs(knn_worker, jobs, sizeof(knn_job), nthreads);
    free(jobs);
    return 0;
}

/* --------------------------------------------------------------- radius */

static double nd_down(double v) { return nextafter(v, -INFINITY); }
static double nd_up(double v) { return nextafter(v, INFINITY); }

typedef struct {
    double R2, f_in, f_out;
    int all, none_band;
    int r2_huge;  /* R2*2^298 exceeds every possible key */
    okey r2key;   /* floor(R2 * 2^298) */
} rthr;

/* Thresholds as in radius_contract.py:129-153 (outward rounded band). */
static void radius_thresholds(int64_t d, double R2, rthr *t) {
    memset(t, 0, sizeof(*t));
    t->R2 = R2;
    if (isinf(R2)) {
        t->all = 1;
        return;
    }
    const double u = ldexp(1.0, -53);
    double g = (double)(d + 2) * u / (1.0 - (double)(d + 2) * u);
    if (R2 == 0.0) {
        t->f_in = t->f_out = 0.0;
        t->none_band = 1;
    } else {
        double fin = nd_down(nd_down(R2 * nd_down(1.0 - 2.0 * g)));
        t->f_in = fin > 0.0 ? fin : 0.0;
        t->f_out = nd_up(nd_up(R2 * nd_up(1.0 + 2.0 * g)));
    }
    /* floor(R2 * 2^298): R2 = M * 2^E with M < 2^53 */
    int e2;
    double fr = frexp(R2, &e2); /* R2 = fr * 2^e2, fr in [0.5,1) */
    uint64_t M = (uint64_t)ldexp(fr, 53);
    int E = e2 - 53;
    int shift = E + 298;
    if (shift >= 0) {
        if (shift + 53 > 64 * KEY_LIMBS - 1) {
            t->r2_huge = 1;
        } else {
            big_from_shifted(t->r2key.w, KEY_LIMBS, M, 0);
            okey tmp;
            memset(&tmp, 0, sizeof(tmp));
            uint64_t mv[1] = {M};
            key_add_shifted(&tmp, mv, 1, shift);
            t->r2key = tmp;
        }
    } else {
        memset(&t->r2key, 0, sizeof(t->r2key));
        if (-shift < 64) t->r2key.w[0] = M >> (-shift);
    }
}

static int radius_member(const float *q, const float *x, int64_t d, double s, const rthr *t) {
    if (t->all) return 1;
    if (s <= t->f_in) return 1;
    if (!(s <= t->f_out)) return 0;
    if (t->r2_huge) return 1;
    okey k;
    exact_key(q, x, d, &k);
    return key_cmp(&k, &t->r2key) <= 0;
}

typedef struct {
    const float *X, *Q;
    int64_t n, d, q_offset;
    int exclude_self;
    const rthr *thr;
    int64_t begin, end;
    int64_t *counts;          /* pass 1 */
    const int64_t *indptr;    /* pass 2 */
    int64_t *indices;
    double *dist;
    int sort;
} rad_job;

static void *rad_count_worker(void *arg) {
    rad_job *J = (rad_job *)arg;
    for (int64_t r = J->begin; r < J->end; ++r) {
        const float *q = J->Q + r * J->d;
        int64_t c = 0;
        for (int64_t j = 0; j < J->n; ++j) {
            if (J->exclude_self && j == J->q_offset + r) continue;
            double s = J->thr->all ? 0.0 : canonical_d2(q, J->X + j * J->d, J->d);
            c += radius_member(q, J->X + j * J->d, J->d, s, J->thr);
        }
        J->counts[r] = c;
    }
    return NULL;
}

typedef struct {
    double v;
    int64_t i;
} dv;

static int dv_cmp(const void *a, const void *b) {
    const dv *x = (const dv *)a, *y = (const dv *)b;
    if (x->v < y->v) return -1;
    if (x->v > y->v) return 1;
    return x->i < y->i ? -1 : (x->i > y->i ? 1 : 0);
}

static void *rad_fill_worker(void *arg) {
    rad_job *J = (rad_job *)arg;
    for (int64_t r = J->begin; r < J->end; ++r) {
        const float *q = J->Q + r * J->d;
        int64_t o = J->indptr[r];
        int64_t start = o;
        for (int64_t j = 0; j < J->n; ++j) {
            if (J->exclude_self && j == J->q_offset + r) continue;
            double s = canonical_d2(q, J->X + j * J->d, J->d);
            if (radius_member(q, J->X + j * J->d, J->d, J->thr->all ? 0.0 : s, J->thr)) {
                J->indices[o] = j;
                if (J->dist) J->dist[o] = sqrt(s < J->thr->R2 ? s : J->thr->R2);
                ++o;
            }
        }
        if (J->sort && J->dist && o - start > 1) {
            int64_t len = o - start;
            dv *tmp = (dv *)malloc(sizeof(dv) * (size_t)len);
            for (int64_t t = 0; t < len; ++t) tmp[t] = (dv){J->dist[start + t], J->indices[start + t]};
            qsort(tmp, (size_t)len, sizeof(dv), dv_cmp);
            for (int64_t t = 0; t < len; ++t) {
                J->dist[start + t] = tmp[t].v;
                J->indices[start + t] = tmp[t].i;
            }
            free(tmp);
        }
    }
    return NULL;
}

static int rad_run(const float *X, int64_t n, int64_t d, const float *Q, int64_t m, double R2,
                   int exclude_self, int64_t q_offset, int64_t *counts, const int64_t *indptr,
                   int64_t *indices, double *dist, int sort, int nthreads, int pass) {
    if (n <= 0 || d <= 0 || m < 0 || !(R2 >= 0.0)) return -1;
    rthr thr;
    radius_thresholds(d, R2, &thr);
    if (nthreads < 1) nthreads = 1;
    if ((int64_t)nthreads > m) nthreads = m > 0 ? (int)m : 1;
    rad_job *jobs = (rad_job *)calloc((size_t)nthreads, sizeof(rad_job));
    int64_t per = (m + nthreads - 1) / nthreads;
    for (int i = 0; i < nthreads; ++i) {
        rad_job j = {X, Q, n, d, q_offset, exclude_self, &thr, 0, 0,
                     counts, indptr, indices, dist, sort};
        j.begin = i * per < m ? i * per : m;
        j.end = (i + 1) * per < m ? (i + 1) * per : m;
        jobs[i] = j;
    }
    run_jobs(pass == 1 ? rad_count_worker : rad_fill_worker, jobs, sizeof(rad_job), nthreads);
    free(jobs);
    return 0;
}

/* Pass 1: exact per-query neighbour counts. */
int orc_radius_count(const float *X, int64_t n, int64_t d, const float *Q, int64_t m, double R2,
                     int exclude_self, int64_t q_offset, int64_t *counts, int nthreads) {
    return rad_run(X, n, d, Q, m, R2, exclude_self, q_offset, counts, NULL, NULL, NULL, 0,
                   nthreads, 1);
}

/* Pass 2: CSR fill; rows ascend by index, or by (distance, index) with sort. */
int orc_radius_fill(const float *X, int64_t n, int64_t d, const float *Q, int64_t m, double R2,
                    int exclude_self, int64_t q_offset, const int64_t *indptr, int64_t *indices,
                    double *dist, int sort, int nthreads) {
    return rad_run(X, n, d, Q, m, R2, exclude_self, q_offset, NULL, indptr, indices, dist, sort,
                   nthreads, 2);
}

/* Exact S(q,x) <= R2 test, for tests of the boundary logic. */
int orc_exact_le(const float *q, const float *x, int64_t d, double R2) {
    rthr thr;
    radius_thresholds(d, R2, &thr);
    if (thr.all || thr.r2_huge) return 1;
    okey k;
    exact_key(q, x, d, &k);
    return key_cmp(&k, &thr.r2key) <= 0;
}
