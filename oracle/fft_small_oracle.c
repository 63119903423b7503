/*
    fft_small_oracle.c -- CPU restatement of the reference's small-prime
    NTT multiplication path.  TEST INFRASTRUCTURE ONLY: used by tests/ as the
    checker and by bench.py's cpu_baseline leg; the product never calls it.

    It follows the structure of FLINT's fft_small mpn_ctx route, step by step,
    with plain 64-bit integer arithmetic (unsigned __int128 products) instead
    of the reference's double-precision FMA kernels:

      * context: the 50-bit prime walk from DEFAULT_PRIME and the CRT data
        (src/fft_small/mpn_mul.c:1000-1016, 1076-1137; default_ctx.c:17);
      * chunk size / prime count: the profile table and the bound
        ceil(64 bn / bits) 2^(2 bits) <= prod primes (mpn_mul.c:46-119,
        152-184, 1171-1195) and the score of mpn_ctx_best_profile
        (mpn_mul.c:1248-1340) evaluated for one thread;
      * splitting limbs into bits-sized chunks reduced mod each prime
        (slow_mpn_to_fft, mpn_mul.c:422-481);
      * cyclic transform of length 2^depth, pointwise product with the
        normaliser (cop 2^depth)^-1 (mpn_mul.c:1505-1527, plan.c:127-149),
        inverse transform -- any exact transform gives the same residues, so
        a textbook iterative NTT stands in for sd_fft_trunc / sd_ifft_trunc
        (sd_fft.c:1230-1274, sd_ifft.c:1503-1533);
      * CRT of each coefficient as sum x_l (P / p_l) reduced below P, shifted
        by i*bits and added into the output with carries (_mpn_from_ffts_NP,
        mpn_mul.c:802-993; _convert_block, mpn_helpers.c:18-51);
      * nmod windows: reduce inputs mod each prime, convolve, CRT, reduce mod
        n (_nmod_poly_mul_mid_mpn_ctx, nmod_poly_mul.c:904-972; prime count
        from bn 2^(2 modbits) <= prod primes, plan.c:356-398).

    The reference's two-prime pipeline for max(an, bn) <= 40000
    (mpn_mul_np2.c:246-310) produces the same (unique) product and is not
    restated separately.

    Parity of this restatement is pinned in tests/ against the compiled
    reference (oracle/_ref), GMP's mpn_mul, Python integers and the golden
    fixtures under tests/golden/.
*/
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef uint64_t ulong_t;
typedef unsigned __int128 u128;

#define NCRTS 8
#define DEFAULT_PRIME 0x0003f00000000001ull

static ulong_t mulmod(ulong_t a, ulong_t b, ulong_t p) { return (ulong_t)(((u128)a * b) % p); }

static ulong_t powmod(ulong_t a, ulong_t e, ulong_t p)
{
    ulong_t r = 1 % p;
    a %= p;
    while (e) {
        if (e & 1) r = mulmod(r, a, p);
        a = mulmod(a, a, p);
        e >>= 1;
    }
    return r;
}

/* deterministic Miller-Rabin for 64-bit n */
static int is_prime(ulong_t n)
{
    static const ulong_t bases[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    if (n < 2) return 0;
    for (int i = 0; i < 12; i++) {
        if (n == bases[i]) return 1;
        if (n % bases[i] == 0) return 0;
    }
    ulong_t d = n - 1;
    int s = 0;
    while (!(d & 1)) { d >>= 1; s++; }
    for (int i = 0; i < 12; i++) {
        ulong_t x = powmod(bases[i], d, n);
        if (x == 1 || x == n - 1) continue;
        int ok = 0;
        for (int r = 1; r < s; r++) {
            x = mulmod(x, x, n);
            if (x == n - 1) { ok = 1; break; }
        }
        if (!ok) return 0;
    }
    return 1;
}

static int nbits(ulong_t x) { return x ? 64 - __builtin_clzll(x) : 0; }

/* next_fft_number (src/fft_small/mpn_mul.c:1000-1016) */
static ulong_t next_fft_number(ulong_t p)
{
    int bits = nbits(p);
    int l = __builtin_ctzll(p - 1);
    ulong_t q = p - (2ull << l);
    if (nbits(q) == bits) return q;
    if (l < 5) return (1ull << (bits - 2)) + 1;
    return (1ull << bits) - (1ull << (l - 1)) + 1;
}

/* ---- small multi-limb helpers (64-bit limbs) -------------------------- */
static ulong_t mpn_mul_1_(ulong_t *r, const ulong_t *x, int n, ulong_t m)
{
    ulong_t c = 0;
    for (int i = 0; i < n; i++) {
        u128 t = (u128)x[i] * m + c;
        r[i] = (ulong_t)t;
        c = (ulong_t)(t >> 64);
    }
    return c;
}

static void mpn_divexact_1_(ulong_t *q, const ulong_t *x, int n, ulong_t d)
{
    u128 r = 0;
    for (int i = n - 1; i >= 0; i--) {
        u128 t = (r << 64) | x[i];
        q[i] = (ulong_t)(t / d);
        r = t % d;
    }
}

static ulong_t mpn_mod_1_(const ulong_t *x, int n, ulong_t d)
{
    u128 r = 0;
    for (int i = n - 1; i >= 0; i--) r = ((r << 64) | x[i]) % d;
    return (ulong_t)r;
}

static int mpn_cmp_(const ulong_t *a, const ulong_t *b, int n)
{
    for (int i = n - 1; i >= 0; i--)
        if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
    return 0;
}

static void mpn_sub_n_(ulong_t *r, const ulong_t *a, const ulong_t *b, int n)
{
    ulong_t br = 0;
    for (int i = 0; i < n; i++) {
        ulong_t t = a[i] - b[i];
        ulong_t b1 = t > a[i];
        ulong_t t2 = t - br;
        ulong_t b2 = t2 > t;
        r[i] = t2;
        br = b1 | b2;
    }
}

/* add x[0..xn) into z[0..zn) starting at limb 0 with carry propagation */
static void mpn_add_into(ulong_t *z, long zn, const ulong_t *x, int xn)
{
    ulong_t c = 0;
    long i = 0;
    for (; i < xn && i < zn; i++) {
        u128 t = (u128)z[i] + x[i] + c;
        z[i] = (ulong_t)t;
        c = (ulong_t)(t >> 64);
    }
    for (; c && i < zn; i++) {
        z[i] += c;
        c = z[i] == 0;
    }
}

/* ---- context (mpn_ctx_init, src/fft_small/mpn_mul.c:1076-1137) -------- */
typedef struct {
    ulong_t p[NCRTS];
    int coeff_len[NCRTS];                 /* limbs of prod primes (with room) */
    ulong_t prod[NCRTS][NCRTS + 2];       /* product of the first i+1 primes */
    ulong_t cofac[NCRTS][NCRTS][NCRTS + 2];   /* prod / p_l */
    ulong_t cofac_red[NCRTS][NCRTS];      /* (prod / p_l) mod p_l */
} oracle_ctx;

static void ctx_init(oracle_ctx *R)
{
    ulong_t p = DEFAULT_PRIME;
    memset(R, 0, sizeof *R);
    for (int i = 0; i < NCRTS; i++) {
        if (i > 0) p = next_fft_number(p);
        while (!is_prime(p)) p = next_fft_number(p);
        R->p[i] = p;
    }
    R->coeff_len[0] = 1;
    R->prod[0][0] = R->p[0];
    R->cofac[0][0][0] = 1;
    R->cofac_red[0][0] = 1;
    for (int i = 1; i < NCRTS; i++) {
        int len = R->coeff_len[i - 1];
        ulong_t t[NCRTS + 2] = {0};
        t[len] = mpn_mul_1_(t, R->prod[i - 1], len, R->p[i]);
        len += 2;   /* room for (prod) * (number of primes) */
        ulong_t tt[NCRTS + 2] = {0};
        mpn_mul_1_(tt, t, len, i + 1);
        while (tt[len - 1] == 0) len--;
        R->coeff_len[i] = len;
        memcpy(R->prod[i], t, len * sizeof(ulong_t));
        for (int l = 0; l <= i; l++) {
            mpn_divexact_1_(R->cofac[i][l], t, len, R->p[l]);
            R->cofac_red[i][l] = mpn_mod_1_(R->cofac[i][l], len, R->p[l]);
        }
    }
}

static oracle_ctx *g_ctx = NULL;
static oracle_ctx *ctx(void)
{
    if (!g_ctx) {
        g_ctx = (oracle_ctx *)malloc(sizeof(oracle_ctx));
        ctx_init(g_ctx);
    }
    return g_ctx;
}

/* log2 of the product of the first np primes */
static double log2_prod(const oracle_ctx *R, int np)
{
    double s = 0;
    for (int i = 0; i < np; i++) s += __builtin_log2((double)R->p[i]);
    return s;
}

/* ceil(64 bn / bits) 2^(2 bits) <= prod primes (mpn_mul.c:92-119) */
static int bits_ok(const oracle_ctx *R, int np, int bits, ulong_t bn)
{
    ulong_t blen = (64 * bn + bits - 1) / bits;
    return __builtin_log2((double)blen) + 2.0 * bits + 1e-9 < log2_prod(R, np);
}

/* profile choice: the reference's table of (np, bits) and its score for one
   thread (mpn_mul.c:1171-1195, 1248-1340) */
static void choose_profile(const oracle_ctx *R, ulong_t an, ulong_t bn, int *np_out, int *bits_out)
{
    static const int prof[15][2] = {{4, 84}, {4, 88}, {4, 92}, {5, 112}, {5, 116}, {5, 120},
                                    {6, 136}, {6, 140}, {6, 144}, {7, 160}, {7, 164}, {7, 168},
                                    {8, 184}, {8, 188}, {8, 192}};
    double best = 1e300;
    int bnp = 8, bbits = 0;
    for (int i = 0; i < 15; i++) {
        int np = prof[i][0], bits = prof[i][1];
        if (!bits_ok(R, np, bits, bn)) continue;
        /* maximise bits within this np */
        if (i + 1 < 15 && prof[i + 1][0] == np && bits_ok(R, np, prof[i + 1][1], bn)) continue;
        ulong_t alen = (64 * an + bits - 1) / bits, blen = (64 * bn + bits - 1) / bits;
        ulong_t zlen = alen + blen - 1;
        ulong_t ztrunc = (zlen + 255) / 256 * 256;
        int depth = 8;
        while ((1ull << depth) < ztrunc) depth++;
        double ratio = (double)ztrunc / (double)(1ull << depth);
        double score = (1 - 0.25 * ratio) * 1e-6 * np * depth * (double)ztrunc;
        if (score < best) { best = score; bnp = np; bbits = bits; }
    }
    if (bbits == 0) {   /* beyond every profile: largest np, widest chunk that fits */
        bnp = 8;
        bbits = 66;
        while (bits_ok(R, 8, bbits + 1, bn)) bbits++;
    }
    *np_out = bnp;
    *bits_out = bbits;
}

/* chunk i of `bits` bits of x (slow_mpn_to_fft, mpn_mul.c:422-481) */
static void get_chunk(ulong_t *out, int ow, const ulong_t *x, ulong_t xn, ulong_t i, int bits)
{
    ulong_t bit0 = i * (ulong_t)bits;
    for (int w = 0; w < ow; w++) out[w] = 0;
    for (int b = 0; b < bits;) {
        ulong_t pos = bit0 + b;
        ulong_t limb = pos / 64;
        int off = (int)(pos % 64);
        if (limb >= xn) break;
        int take = 64 - off;
        if (take > bits - b) take = bits - b;
        ulong_t v = (x[limb] >> off) & (take == 64 ? ~0ull : ((1ull << take) - 1));
        int w = b / 64, wo = b % 64;
        out[w] |= v << wo;
        if (wo && wo + take > 64) out[w + 1] |= v >> (64 - wo);
        b += take;
    }
}

/* textbook iterative NTT mod p of length 2^k (bit-reversal + Cooley-Tukey) */
static ulong_t root_of_unity(ulong_t p, int k)
{
    ulong_t m = p - 1, f[64];
    int nf = 0;
    for (ulong_t q = 2; q * q <= m; q++)
        if (m % q == 0) { f[nf++] = q; while (m % q == 0) m /= q; }
    if (m > 1) f[nf++] = m;
    for (ulong_t g = 2;; g++) {
        int ok = 1;
        for (int i = 0; i < nf; i++)
            if (powmod(g, (p - 1) / f[i], p) == 1) { ok = 0; break; }
        if (ok) return powmod(g, (p - 1) >> k, p);
    }
}

static void ntt(ulong_t *x, int k, ulong_t w, ulong_t p)
{
    ulong_t n = 1ull << k;
    for (ulong_t i = 1, j = 0; i < n; i++) {
        ulong_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) { ulong_t t = x[i]; x[i] = x[j]; x[j] = t; }
    }
    for (ulong_t len = 2; len <= n; len <<= 1) {
        ulong_t wl = powmod(w, n / len, p);
        for (ulong_t i = 0; i < n; i += len) {
            ulong_t ww = 1;
            for (ulong_t j = 0; j < len / 2; j++) {
                ulong_t u = x[i + j], v = mulmod(x[i + j + len / 2], ww, p);
                x[i + j] = u + v >= p ? u + v - p : u + v;
                x[i + j + len / 2] = u >= v ? u - v : u + p - v;
                ww = mulmod(ww, wl, p);
            }
        }
    }
}

/* cyclic convolution mod p of length 2^depth with the normaliser folded into
   the pointwise product (mpn_mul.c:1505-1527) */
static void conv_mod_p(ulong_t *A, ulong_t *B, int depth, ulong_t p, ulong_t cop, int squaring)
{
    ulong_t n = 1ull << depth;
    ulong_t w = root_of_unity(p, depth);
    ntt(A, depth, w, p);
    if (!squaring) ntt(B, depth, w, p);
    ulong_t m = powmod(mulmod(cop % p, powmod(2, depth, p), p), p - 2, p);
    for (ulong_t i = 0; i < n; i++) A[i] = mulmod(mulmod(A[i], squaring ? A[i] : B[i], p), m, p);
    ntt(A, depth, powmod(w, p - 2, p), p);
}

/* z = a * b, an, bn >= 1 (mpn_ctx_mpn_mul, mpn_mul.c:1617-1983) */
int oracle_mpn_mul(ulong_t *z, const ulong_t *a, ulong_t an, const ulong_t *b, ulong_t bn)
{
    oracle_ctx *R = ctx();
    int np, bits;
    if (an == 0 || bn == 0) return 1;
    choose_profile(R, an, bn, &np, &bits);
    ulong_t alen = (64 * an + bits - 1) / bits, blen = (64 * bn + bits - 1) / bits;
    ulong_t zlen = alen + blen - 1;
    int depth = 0;
    while ((1ull << depth) < zlen) depth++;
    ulong_t N = 1ull << depth;
    int cw = (bits + 63) / 64 + 1;
    int squaring = (a == b) && (an == bn);
    ulong_t *res = (ulong_t *)calloc(N * np, sizeof(ulong_t));
    ulong_t *tmp = (ulong_t *)calloc(N, sizeof(ulong_t));
    ulong_t chunk[8];
    if (!res || !tmp) return 2;
    for (int l = 0; l < np; l++) {
        ulong_t p = R->p[l];
        ulong_t *A = res + (ulong_t)l * N;
        for (ulong_t i = 0; i < alen; i++) {
            get_chunk(chunk, cw, a, an, i, bits);
            A[i] = mpn_mod_1_(chunk, cw, p);
        }
        if (!squaring) {
            memset(tmp, 0, N * sizeof(ulong_t));
            for (ulong_t i = 0; i < blen; i++) {
                get_chunk(chunk, cw, b, bn, i, bits);
                tmp[i] = mpn_mod_1_(chunk, cw, p);
            }
        }
        conv_mod_p(A, tmp, depth, p, R->cofac_red[np - 1][l], squaring);
    }
    /* CRT + shifted add (mpn_mul.c:802-993) */
    int n = R->coeff_len[np - 1];
    memset(z, 0, (an + bn) * sizeof(ulong_t));
    ulong_t *s = (ulong_t *)calloc(n + 2, sizeof(ulong_t));
    ulong_t *sh = (ulong_t *)calloc(n + 3, sizeof(ulong_t));
    for (ulong_t i = 0; i < zlen; i++) {
        memset(s, 0, (n + 2) * sizeof(ulong_t));
        for (int l = 0; l < np; l++) {
            ulong_t x = res[(ulong_t)l * N + i];
            ulong_t t[NCRTS + 3] = {0};
            t[n] = mpn_mul_1_(t, R->cofac[np - 1][l], n, x);
            mpn_add_into(s, n + 1, t, n + 1);
        }
        while (s[n] != 0 || mpn_cmp_(s, R->prod[np - 1], n) >= 0) {
            ulong_t pp[NCRTS + 3] = {0};
            memcpy(pp, R->prod[np - 1], n * sizeof(ulong_t));
            mpn_sub_n_(s, s, pp, n + 1);
        }
        ulong_t bit0 = i * (ulong_t)bits;
        ulong_t limb = bit0 / 64;
        int off = (int)(bit0 % 64);
        memset(sh, 0, (n + 3) * sizeof(ulong_t));
        for (int w = 0; w < n; w++) {
            sh[w] |= off ? s[w] << off : s[w];
            if (off) sh[w + 1] |= s[w] >> (64 - off);
        }
        if (limb < an + bn) mpn_add_into(z + limb, (long)(an + bn - limb), sh, n + 1);
    }
    free(s);
    free(sh);
    free(res);
    free(tmp);
    return 0;
}

/* coefficients [zl, zh) of a * b mod n, inputs reduced mod n
   (_nmod_poly_mul_mid_mpn_ctx, nmod_poly_mul.c:904-972) */
int oracle_nmod_mul_mid(ulong_t *z, ulong_t zl, ulong_t zh, const ulong_t *a, ulong_t an,
                        const ulong_t *b, ulong_t bn, ulong_t mod)
{
    oracle_ctx *R = ctx();
    if (an == 0 || bn == 0 || mod == 0) return 1;
    if (zl >= zh) return 0;
    ulong_t zn = an + bn - 1;
    memset(z, 0, (zh - zl) * sizeof(ulong_t));
    if (zl >= zn) return 0;
    if (zh > zn) zh = zn;
    /* prime count: bn 2^(2 modbits) <= prod primes (plan.c:356-398) */
    int modbits = nbits(mod);
    ulong_t mn = an < bn ? an : bn;
    int np = 1;
    while (np < NCRTS && !(__builtin_log2((double)mn) + 2.0 * modbits + 1e-9 < log2_prod(R, np))) np++;
    int depth = 0;
    while ((1ull << depth) < zn) depth++;
    ulong_t N = 1ull << depth;
    int squaring = (a == b) && (an == bn);
    ulong_t *res = (ulong_t *)calloc(N * np, sizeof(ulong_t));
    ulong_t *tmp = (ulong_t *)calloc(N, sizeof(ulong_t));
    if (!res || !tmp) return 2;
    for (int l = 0; l < np; l++) {
        ulong_t p = R->p[l];
        ulong_t *A = res + (ulong_t)l * N;
        for (ulong_t i = 0; i < an; i++) A[i] = a[i] % p;
        memset(tmp, 0, N * sizeof(ulong_t));
        if (!squaring)
            for (ulong_t i = 0; i < bn; i++) tmp[i] = b[i] % p;
        conv_mod_p(A, tmp, depth, p, R->cofac_red[np - 1][l], squaring);
    }
    int n = R->coeff_len[np - 1];
    ulong_t *s = (ulong_t *)calloc(n + 2, sizeof(ulong_t));
    for (ulong_t k = zl; k < zh; k++) {
        memset(s, 0, (n + 2) * sizeof(ulong_t));
        for (int l = 0; l < np; l++) {
            ulong_t t[NCRTS + 3] = {0};
            t[n] = mpn_mul_1_(t, R->cofac[np - 1][l], n, res[(ulong_t)l * N + k]);
            mpn_add_into(s, n + 1, t, n + 1);
        }
        while (s[n] != 0 || mpn_cmp_(s, R->prod[np - 1], n) >= 0) {
            ulong_t pp[NCRTS + 3] = {0};
            memcpy(pp, R->prod[np - 1], n * sizeof(ulong_t));
            mpn_sub_n_(s, s, pp, n + 1);
        }
        z[k - zl] = mpn_mod_1_(s, n + 1, mod);
    }
    free(s);
    free(res);
    free(tmp);
    return 0;
}

/* the reference's prime set, for tests that compare the restated context */
ulong_t oracle_prime(int i) { return (i >= 0 && i < NCRTS) ? ctx()->p[i] : 0; }
