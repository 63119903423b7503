// Host side of the B200 small-prime NTT multiplication library: context
// set-up (primes, twiddle and CRT tables), plan selection, kernel launches
// and the C ABI declared in include/gpu_fft_small.h.
//
// Everything here is plain CUDA runtime + C++; no torch types cross the ABI.
#include "../../include/gpu_fft_small.h"
#include "mpn_kernels.cuh"
#include "nmod_kernels.cuh"
#include "fmpz_kernels.cuh"
#include "basecase_kernels.cuh"
#include "mlp_kernels.cuh"
#include "op_kernels.cuh"
#include "neg_kernels.cuh"
#include "mpn3_kernels.cuh"

#include <cuda_runtime.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <algorithm>
#include <atomic>
#include <mutex>
#include <string>
#include <vector>
#include <unordered_map>

using namespace fb;

// ---------------------------------------------------------------------------
// Prime set: every prime 2^30 < p < 2^31 with 2^25 | p - 1, largest first,
// plus the two smaller ones with the same 2-adic valuation.  Five of them
// hold coefficients of 64-bit-chunk products up to min(an, bn) ~ 2^24.3
// limbs; six go to ~2^53.
static const uint32_t PRIMES[MAX_NP] = {
    2113929217u, 2013265921u, 1811939329u, 1711276033u, 1107296257u,
    469762049u, 167772161u};

// ---------------------------------------------------------------------------
// errors
static thread_local std::string g_last_error;
static void (*g_throw_handler)(int, const char *) = nullptr;

static int set_error(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

static void raise_error(int code)
{
    if (g_throw_handler) {
        g_throw_handler(code, g_last_error.c_str());
        return;
    }
    fprintf(stderr, "gpu_fft_small: error %d: %s\n", code, g_last_error.c_str());
    fflush(stderr);
    abort();
}

#define CU(call)                                                              \
    do {                                                                      \
        cudaError_t e_ = (call);                                              \
        if (e_ != cudaSuccess)                                                \
            return set_error(GPU_FFT_SMALL_ECUDA, "%s: %s (%s:%d)", #call,    \
                             cudaGetErrorString(e_), __FILE__, __LINE__);     \
    } while (0)

// ---------------------------------------------------------------------------
// host number theory
// Smallest primitive root mod p (no heap use: the allocation-free entry
// point's set-up calls it too).
static uint32_t primitive_root(uint32_t p)
{
    uint32_t m = p - 1, f[32];
    int nf = 0;
    for (uint32_t q = 2; (uint64_t)q * q <= m; q++)
        if (m % q == 0) {
            f[nf++] = q;
            while (m % q == 0) m /= q;
        }
    if (m > 1) f[nf++] = m;
    for (uint32_t g = 2;; g++) {
        bool ok = true;
        for (int i = 0; i < nf; i++)
            if (h_powmod(g, (p - 1) / f[i], p) == 1) { ok = false; break; }
        if (ok) return g;
    }
}

// Constant-memory tables that every kernel of the module reads: the
// radix-32 twiddles w_32^k, w_32^-k of all MAX_NP primes (c_w32) and the
// opaque constants of fadd/fsub (c_one, c_minus_one).  Their values depend on
// nothing but the prime set, so they are written once per device, by
// whichever of context creation or the allocation-free entry point's set-up
// reaches the device first, and never rewritten while kernels may read them.
// (A cudaDeviceReset would discard them with the module; this library never
// resets a device.)
constexpr int CONST_MAX_DEVICES = 64;
static std::atomic<bool> g_const_ready[CONST_MAX_DEVICES];
static std::mutex g_const_lock;

static cudaError_t device_constants_ensure(int dev)
{
    if (dev >= 0 && dev < CONST_MAX_DEVICES && g_const_ready[dev].load(std::memory_order_acquire))
        return cudaSuccess;
    std::lock_guard<std::mutex> guard(g_const_lock);
    if (dev >= 0 && dev < CONST_MAX_DEVICES && g_const_ready[dev].load(std::memory_order_relaxed))
        return cudaSuccess;
    W32Table w32[MAX_NP];
    for (int j = 0; j < MAX_NP; j++) {
        const uint32_t p = PRIMES[j];
        const uint32_t w = h_powmod(primitive_root(p), (p - 1) >> LOG_MAXM, p);   // order 2^25
        const uint32_t w32f = h_powmod(w, 1u << (LOG_MAXM - 5), p), w32i = h_invmod(w32f, p);
        uint32_t x = 1, xi = 1;
        for (int k = 0; k < 16; k++) {
            w32[j].f[k] = make_uint2(x, shoup_companion(x, p));
            w32[j].i[k] = make_uint2(xi, shoup_companion(xi, p));
            x = h_mulmod(x, w32f, p);
            xi = h_mulmod(xi, w32i, p);
        }
    }
    const uint32_t one = 1, minus_one = 0xffffffffu;
    cudaError_t e = cudaMemcpyToSymbol(c_w32, w32, sizeof w32);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_one, &one, sizeof one);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_minus_one, &minus_one, sizeof minus_one);
    if (e == cudaSuccess && dev >= 0 && dev < CONST_MAX_DEVICES)
        g_const_ready[dev].store(true, std::memory_order_release);
    return e;
}

static uint2 shoup_pair(uint32_t w, uint32_t p)
{
    return make_uint2(w, shoup_companion(w, p));
}

// multiword helpers, 32-bit little-endian words
static void mw_mul_small(std::vector<uint32_t> &x, uint32_t m)
{
    uint64_t c = 0;
    for (auto &w : x) {
        uint64_t t = (uint64_t)w * m + c;
        w = (uint32_t)t;
        c = t >> 32;
    }
    if (c) x.push_back((uint32_t)c);
}

static std::vector<uint32_t> mw_div_small(const std::vector<uint32_t> &x, uint32_t d)
{
    std::vector<uint32_t> q(x.size());
    uint64_t r = 0;
    for (size_t i = x.size(); i-- > 0;) {
        uint64_t t = (r << 32) | x[i];
        q[i] = (uint32_t)(t / d);
        r = t % d;
    }
    while (q.size() > 1 && q.back() == 0) q.pop_back();
    return q;
}

static uint32_t mw_mod_small(const std::vector<uint32_t> &x, uint32_t d)
{
    uint64_t r = 0;
    for (size_t i = x.size(); i-- > 0;) r = ((r << 32) | x[i]) % d;
    return (uint32_t)r;
}

static double log2_product(int np)
{
    double s = 0;
    for (int j = 0; j < np; j++) s += log2((double)PRIMES[j]);
    return s;
}

// ---------------------------------------------------------------------------
// context

// Per-kernel timing record: events before the first and after each of the
// four kernels of one product (slot k spans ev[k] .. ev[k+1]).
constexpr int TIMING_SLOTS = 4;
constexpr size_t TIMING_RING = 512;
struct TimingRecord {
    cudaEvent_t ev[TIMING_SLOTS + 1];
    bool used;
};

struct Ctx;
static TimingRecord *timing_begin(Ctx *X, cudaStream_t st);
static void timing_mark(TimingRecord *r, int k, cudaStream_t st)
{
    if (r) cudaEventRecord(r->ev[k], st);
}

struct Ctx {
    int device = -1;
    int nsm = 148;                        // multiprocessors of the device
    gpu_ulong p0 = 0;
    cudaStream_t stream = nullptr;
    void *d_tables = nullptr;
    DevTables T{};
    uint32_t *d_scale = nullptr;          // [np][logM][MAX_NP] pointwise scales
    int *d_err = nullptr;
    int *h_err = nullptr;                 // pinned copy of *d_err, read after a host-pointer product
    unsigned long long *d_ticket = nullptr;
    unsigned long long ticket_base = 0;
    uint32_t *d_status = nullptr;
    size_t status_cap = 0;                // tiles
    uint32_t epoch = 0;
    uint32_t *d_res = nullptr;
    size_t res_cap = 0;                   // bytes
    uint64_t *d_io = nullptr;
    size_t io_cap = 0;                    // bytes
    int last_launches = 0;
    // opt-in per-kernel timing: a ring of event records, read lazily
    bool timing = false;
    std::vector<TimingRecord> rec;
    size_t rec_head = 0, rec_tail = 0;
    double kernel_ms[TIMING_SLOTS] = {0};
    long kernel_count[TIMING_SLOTS] = {0};
    CrtConst crt[MAX_NP + 1];
    uint32_t cof_red[MAX_NP + 1][MAX_NP]; // (P/p_j) mod p_j for each np
    // host-pointer products: a second stream for the copies that overlap
    // the kernels, and events to order the two
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_copy[9] = {nullptr};
    // configuration timing (autotuner): operand buffer and events kept
    // between calls, so a timing costs launches only
    uint64_t *d_time = nullptr;
    size_t time_cap = 0;                  // bytes
    cudaEvent_t ev_time[2] = {nullptr, nullptr};
};


static int grow(void **ptr, size_t *cap, size_t need)
{
    if (need <= *cap) return 0;
    if (*ptr) cudaFree(*ptr);
    *ptr = nullptr;
    *cap = 0;
    size_t sz = std::max(need, *cap + *cap / 8);
    CU(cudaMalloc(ptr, sz));
    *cap = sz;
    return 0;
}

// the timing buffer (at least `bytes`) and the two timing events
static int timing_scratch(Ctx *X, size_t bytes, uint64_t **buf)
{
    int rc = grow((void **)&X->d_time, &X->time_cap, bytes);
    if (rc) return rc;
    for (auto &e : X->ev_time)
        if (!e) CU(cudaEventCreate(&e));
    *buf = X->d_time;
    return 0;
}

static int ctx_build_tables(Ctx *X)
{
    const size_t n_twf = (size_t)MAX_NP * TW_SZ;
    const size_t n_th = (size_t)MAX_NP * TH_SZ;
    const size_t n_tl = (size_t)MAX_NP * TL_SZ;
    std::vector<PrimeInfo> pi(MAX_NP);
    std::vector<uint2> twf(n_twf), twi(n_twf), th(n_th), tl(n_tl), thi(n_th), tli(n_tl);
    for (int j = 0; j < MAX_NP; j++) {
        const uint32_t p = PRIMES[j];
        PrimeInfo &P = pi[j];
        memset(&P, 0, sizeof P);
        P.p = p;
        uint32_t inv = 1;                 // p^-1 mod 2^32 by Newton iteration
        for (int it = 0; it < 5; it++) inv *= 2 - p * inv;
        P.pneg_inv = 0u - inv;
        P.c32 = (uint32_t)((1ull << 32) % p);
        P.r2 = h_mulmod(P.c32, P.c32, p);
        P.finv = 1.0f / (float)p;
        const uint32_t g = primitive_root(p);
        const uint32_t w = h_powmod(g, (p - 1) >> LOG_MAXM, p);   // order 2^25
        const uint32_t wi = h_invmod(w, p);
        // local twiddles: entry h + jj = w_{2h}^jj, w_{2h} = w^(2^25 / 2h)
        twf[(size_t)j * TW_SZ] = make_uint2(1, 0);
        twi[(size_t)j * TW_SZ] = make_uint2(1, 0);
        for (int h = 1; h < TW_SZ; h <<= 1) {
            const int lh = __builtin_ctz(h);
            const uint32_t r = h_powmod(w, 1ull << (LOG_MAXM - lh - 1), p);
            const uint32_t ri = h_powmod(wi, 1ull << (LOG_MAXM - lh - 1), p);
            uint32_t x = 1, xi = 1;
            for (int jj = 0; jj < h; jj++) {
                twf[(size_t)j * TW_SZ + h + jj] = shoup_pair(x, p);
                twi[(size_t)j * TW_SZ + h + jj] = shoup_pair(xi, p);
                x = h_mulmod(x, r, p);
                xi = h_mulmod(xi, ri, p);
            }
        }
        // twist tables
        {
            const uint32_t step = h_powmod(w, 1u << 13, p), stepi = h_powmod(wi, 1u << 13, p);
            uint32_t x = 1, xi = 1;
            for (int t = 0; t < TH_SZ; t++) {
                th[(size_t)j * TH_SZ + t] = shoup_pair(x, p);
                thi[(size_t)j * TH_SZ + t] = shoup_pair(xi, p);
                x = h_mulmod(x, step, p);
                xi = h_mulmod(xi, stepi, p);
            }
            x = 1; xi = 1;
            for (int t = 0; t < TL_SZ; t++) {
                tl[(size_t)j * TL_SZ + t] = shoup_pair(x, p);
                tli[(size_t)j * TL_SZ + t] = shoup_pair(xi, p);
                x = h_mulmod(x, w, p);
                xi = h_mulmod(xi, wi, p);
            }
        }
    }
    // tables of the 3 2^k-point transforms (first NP3 primes): twist powers
    // of w3 of order 3 2^25, radix-3 stage twiddles omega^(+-e) / 2 with omega
    // of order 3 2^11, and the stage constants w - w^2, w^-1 - w^-2 (w of
    // order 3)
    const size_t n_th3 = (size_t)NP3 * TH3_SZ, n_tl3 = (size_t)NP3 * TL_SZ, n_tw3 = (size_t)NP3 * TW3_SZ;
    std::vector<uint2> th3(n_th3), tl3(n_tl3), th3i(n_th3), tl3i(n_tl3), tw3f(n_tw3), tw3i(n_tw3),
        w3c((size_t)NP3 * 2);
    for (int j = 0; j < NP3; j++) {
        const uint32_t p = PRIMES[j];
        const uint32_t w3 = h_powmod(primitive_root(p), (p - 1) / (3u << LOG_MAXM), p);
        const uint32_t w3i = h_invmod(w3, p);
        const uint32_t inv2 = (p + 1) / 2;
        uint32_t x = 1, xi = 1;
        const uint32_t st = h_powmod(w3, 1u << 13, p), sti = h_powmod(w3i, 1u << 13, p);
        for (int t = 0; t < TH3_SZ; t++) {
            th3[(size_t)j * TH3_SZ + t] = shoup_pair(x, p);
            th3i[(size_t)j * TH3_SZ + t] = shoup_pair(xi, p);
            x = h_mulmod(x, st, p);
            xi = h_mulmod(xi, sti, p);
        }
        x = 1; xi = 1;
        for (int t = 0; t < TL_SZ; t++) {
            tl3[(size_t)j * TL_SZ + t] = shoup_pair(x, p);
            tl3i[(size_t)j * TL_SZ + t] = shoup_pair(xi, p);
            x = h_mulmod(x, w3, p);
            xi = h_mulmod(xi, w3i, p);
        }
        const uint32_t om = h_powmod(w3, 1u << (LOG_MAXM - LOG_R3), p), omi = h_invmod(om, p);
        x = inv2; xi = inv2;
        for (int e = 0; e < TW3_SZ; e++) {
            tw3f[(size_t)j * TW3_SZ + e] = shoup_pair(x, p);
            tw3i[(size_t)j * TW3_SZ + e] = shoup_pair(xi, p);
            x = h_mulmod(x, om, p);
            xi = h_mulmod(xi, omi, p);
        }
        const uint32_t w = h_powmod(w3, 1u << LOG_MAXM, p), wi = h_invmod(w, p);
        const uint32_t c = (uint32_t)(((uint64_t)w + p - h_mulmod(w, w, p)) % p);
        const uint32_t ci = (uint32_t)(((uint64_t)wi + p - h_mulmod(wi, wi, p)) % p);
        w3c[(size_t)j * 2] = shoup_pair(c, p);
        w3c[(size_t)j * 2 + 1] = shoup_pair(ci, p);
    }
    // CRT constants for every prime count
    for (int np = 1; np <= MAX_NP; np++) {
        CrtConst &K = X->crt[np];
        memset(&K, 0, sizeof K);
        K.np = np;
        std::vector<uint32_t> P = {1};
        for (int j = 0; j < np; j++) mw_mul_small(P, PRIMES[j]);
        for (size_t w = 0; w < P.size() && w < (size_t)MAX_NP; w++) K.P[w] = P[w];
        for (int j = 0; j < np; j++) {
            std::vector<uint32_t> c = mw_div_small(P, PRIMES[j]);
            for (size_t w = 0; w < c.size() && w < (size_t)MAX_NP; w++) K.cof[j][w] = c[w];
            X->cof_red[np][j] = mw_mod_small(c, PRIMES[j]);
            K.finv[j] = 1.0f / (float)PRIMES[j];
        }
    }

    size_t off = 0;
    auto place = [&](size_t bytes) { size_t o = off; off += (bytes + 255) & ~(size_t)255; return o; };
    const size_t o_pi = place(sizeof(PrimeInfo) * MAX_NP);
    const size_t o_twf = place(sizeof(uint2) * n_twf), o_twi = place(sizeof(uint2) * n_twf);
    const size_t o_th = place(sizeof(uint2) * n_th), o_tl = place(sizeof(uint2) * n_tl);
    const size_t o_thi = place(sizeof(uint2) * n_th), o_tli = place(sizeof(uint2) * n_tl);
    const size_t o_th3 = place(sizeof(uint2) * n_th3), o_tl3 = place(sizeof(uint2) * n_tl3);
    const size_t o_th3i = place(sizeof(uint2) * n_th3), o_tl3i = place(sizeof(uint2) * n_tl3);
    const size_t o_tw3f = place(sizeof(uint2) * n_tw3), o_tw3i = place(sizeof(uint2) * n_tw3);
    const size_t o_w3c = place(sizeof(uint2) * NP3 * 2);
    CU(cudaMalloc(&X->d_tables, off));
    char *base = (char *)X->d_tables;
    CU(cudaMemcpy(base + o_pi, pi.data(), sizeof(PrimeInfo) * MAX_NP, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(base + o_twf, twf.data(), sizeof(uint2) * n_twf, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(base + o_twi, twi.data(), sizeof(uint2) * n_twf, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(base + o_th, th.data(), sizeof(uint2) * n_th, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(base + o_tl, tl.data(), sizeof(uint2) * n_tl, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(base + o_thi, thi.data(), sizeof(uint2) * n_th, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(base + o_tli, tli.data(), sizeof(uint2) * n_tl, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(base + o_th3, th3.data(), sizeof(uint2) * n_th3, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(base + o_tl3, tl3.data(), sizeof(uint2) * n_tl3, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(base + o_th3i, th3i.data(), sizeof(uint2) * n_th3, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(base + o_tl3i, tl3i.data(), sizeof(uint2) * n_tl3, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(base + o_tw3f, tw3f.data(), sizeof(uint2) * n_tw3, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(base + o_tw3i, tw3i.data(), sizeof(uint2) * n_tw3, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(base + o_w3c, w3c.data(), sizeof(uint2) * NP3 * 2, cudaMemcpyHostToDevice));
    X->T.pi = (const PrimeInfo *)(base + o_pi);
    X->T.twf = (const uint2 *)(base + o_twf);
    X->T.twi = (const uint2 *)(base + o_twi);
    X->T.th = (const uint2 *)(base + o_th);
    X->T.tl = (const uint2 *)(base + o_tl);
    X->T.thi = (const uint2 *)(base + o_thi);
    X->T.tli = (const uint2 *)(base + o_tli);
    X->T.th3 = (const uint2 *)(base + o_th3);
    X->T.tl3 = (const uint2 *)(base + o_tl3);
    X->T.th3i = (const uint2 *)(base + o_th3i);
    X->T.tl3i = (const uint2 *)(base + o_tl3i);
    X->T.tw3f = (const uint2 *)(base + o_tw3f);
    X->T.tw3i = (const uint2 *)(base + o_tw3i);
    X->T.w3c = (const uint2 *)(base + o_w3c);
    // constant memory belongs to the current device's module instance
    CU(device_constants_ensure(X->device));
    CU(cudaDeviceGetAttribute(&X->nsm, cudaDevAttrMultiProcessorCount, X->device));
    return 0;
}

// ---------------------------------------------------------------------------
// kernel dispatch by transform shape (column length 2^logR, row length 2^logC)
typedef void (*fwd_cols_fn)(DevTables, const uint64_t *, uint64_t, const uint64_t *, uint64_t,
                            uint32_t *, uint32_t *, int, int, const InstDesc *, int, FzShape,
                            const uint32_t *, int);
typedef void (*inv_cols_fn)(DevTables, uint32_t *, int, int, const InstDesc *, ChunkOut);
typedef void (*rows_fn)(DevTables, uint32_t *, const uint32_t *, int, int, int, const uint32_t *,
                        int, const InstDesc *, int, int);

template <int LOGR>
constexpr int tmpl_cols() { return LOGR >= 5 ? cols_per_tile(LOGR) : 0; }

#define FB_COLS(X, ...) X<0, tmpl_cols<0>() __VA_ARGS__>, X<1, tmpl_cols<1>() __VA_ARGS__>,        \
                        X<2, tmpl_cols<2>() __VA_ARGS__>, X<3, tmpl_cols<3>() __VA_ARGS__>,        \
                        X<4, tmpl_cols<4>() __VA_ARGS__>, X<5, tmpl_cols<5>() __VA_ARGS__>,        \
                        X<6, tmpl_cols<6>() __VA_ARGS__>, X<7, tmpl_cols<7>() __VA_ARGS__>,        \
                        X<8, tmpl_cols<8>() __VA_ARGS__>, X<9, tmpl_cols<9>() __VA_ARGS__>,        \
                        X<10, tmpl_cols<10>() __VA_ARGS__>, X<11, tmpl_cols<11>() __VA_ARGS__>
static const fwd_cols_fn FWD_COLS[12] = {FB_COLS(k_fwd_cols, , false)};
static const fwd_cols_fn FWD_COLS_FZ[12] = {FB_COLS(k_fwd_cols, , true)};
static const inv_cols_fn INV_COLS[12] = {FB_COLS(k_inv_cols)};
// constant-stride instances: 2^13-point rows under 2^9..2^11-point columns
// (index logR - 9) and 2^14-point rows under 2^11-point columns
static const fwd_cols_fn FWD_COLS_C13[3] = {k_fwd_cols<9, tmpl_cols<9>(), false, 13>,
                                            k_fwd_cols<10, tmpl_cols<10>(), false, 13>,
                                            k_fwd_cols<11, tmpl_cols<11>(), false, 13>};
static const fwd_cols_fn FWD_COLS_FZ_C13[3] = {k_fwd_cols<9, tmpl_cols<9>(), true, 13>,
                                               k_fwd_cols<10, tmpl_cols<10>(), true, 13>,
                                               k_fwd_cols<11, tmpl_cols<11>(), true, 13>};
static const inv_cols_fn INV_COLS_C13[3] = {k_inv_cols<9, tmpl_cols<9>(), 13>,
                                            k_inv_cols<10, tmpl_cols<10>(), 13>,
                                            k_inv_cols<11, tmpl_cols<11>(), 13>};
// narrow tiles (a quarter of the columns, 128 threads) for columns of 2^5 to
// 2^8 points (index logR - 5): small transforms get four times the CTAs
static const fwd_cols_fn FWD_COLS_S[4] = {k_fwd_cols<5, cols_per_tile(5) / 4, false>,
                                          k_fwd_cols<6, cols_per_tile(6) / 4, false>,
                                          k_fwd_cols<7, cols_per_tile(7) / 4, false>,
                                          k_fwd_cols<8, cols_per_tile(8) / 4, false>};
static const inv_cols_fn INV_COLS_S[4] = {k_inv_cols<5, cols_per_tile(5) / 4>, k_inv_cols<6, cols_per_tile(6) / 4>,
                                          k_inv_cols<7, cols_per_tile(7) / 4>, k_inv_cols<8, cols_per_tile(8) / 4>};
static const fwd_cols_fn FWD_COLS_C14 = k_fwd_cols<11, tmpl_cols<11>(), false, 14>;
static const fwd_cols_fn FWD_COLS_FZ_C14 = k_fwd_cols<11, tmpl_cols<11>(), true, 14>;
static const inv_cols_fn INV_COLS_C14 = k_inv_cols<11, tmpl_cols<11>(), 14>;

// columns of 3 2^r points, r = 5 .. 10 (index r - 5)
typedef void (*fwd_cols3_fn)(DevTables, const uint64_t *, uint64_t, const uint64_t *, uint64_t, uint32_t *,
                             uint32_t *, int, int, const uint32_t *, int, FzShape);
typedef void (*inv_cols3_fn)(DevTables, uint32_t *, int, int);
constexpr int LOG3_RMIN = 5, LOG3_RMAX = 10;
static const fwd_cols3_fn FWD_COLS3[6] = {
    k_fwd_cols3<5, cols_per_tile3(5)>, k_fwd_cols3<6, cols_per_tile3(6)>, k_fwd_cols3<7, cols_per_tile3(7)>,
    k_fwd_cols3<8, cols_per_tile3(8)>, k_fwd_cols3<9, cols_per_tile3(9)>, k_fwd_cols3<10, cols_per_tile3(10)>};
// the same for integer-polynomial operands
static const fwd_cols3_fn FWD_COLS3_FZ[6] = {
    k_fwd_cols3<5, cols_per_tile3(5), true>, k_fwd_cols3<6, cols_per_tile3(6), true>,
    k_fwd_cols3<7, cols_per_tile3(7), true>, k_fwd_cols3<8, cols_per_tile3(8), true>,
    k_fwd_cols3<9, cols_per_tile3(9), true>, k_fwd_cols3<10, cols_per_tile3(10), true>};
static const inv_cols3_fn INV_COLS3[6] = {
    k_inv_cols3<5, cols_per_tile3(5)>, k_inv_cols3<6, cols_per_tile3(6)>, k_inv_cols3<7, cols_per_tile3(7)>,
    k_inv_cols3<8, cols_per_tile3(8)>, k_inv_cols3<9, cols_per_tile3(9)>, k_inv_cols3<10, cols_per_tile3(10)>};

// the column kernels for a transform shape
static fwd_cols_fn fwd_cols_kernel(int logR, int logC, bool fz = false)
{
    if (logR == 11 && logC == 14) return fz ? FWD_COLS_FZ_C14 : FWD_COLS_C14;
    if (logR >= 9 && logR <= 11 && logC == 13) return (fz ? FWD_COLS_FZ_C13 : FWD_COLS_C13)[logR - 9];
    return (fz ? FWD_COLS_FZ : FWD_COLS)[logR];
}
static inv_cols_fn inv_cols_kernel(int logR, int logC)
{
    if (logR == 11 && logC == 14) return INV_COLS_C14;
    if (logR >= 9 && logR <= 11 && logC == 13) return INV_COLS_C13[logR - 9];
    return INV_COLS[logR];
}
// Rows run with 32 elements per thread (k_rows<LOGC, 5>) or 16 (k_rows<LOGC,
// 4>: twice the threads, 64 registers).  On the 2^24 product 16 is slower
// (1.88 against 1.74 ms: one more shared-memory pass, and the register cap);
// small transforms, whose row launch has only a few warps per SM and runs
// latency-bound, take 16 (rows_loge).
static const rows_fn ROWS[15] = {nullptr, nullptr, nullptr, nullptr, nullptr,
                                 k_rows<5>, k_rows<6>, k_rows<7>, k_rows<8>, k_rows<9>,
                                 k_rows<10>, k_rows<11>, k_rows<12>, k_rows<13>, k_rows<14>};
constexpr int ROWS16_MIN_LOGC = 9;
static const rows_fn ROWS16[15] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                                   nullptr, k_rows<9, 4>, k_rows<10, 4>, k_rows<11, 4>, k_rows<12, 4>,
                                   k_rows<13, 4>, k_rows<14, 4>};
#undef FB_COLS
typedef void (*rows_op_fn)(DevTables, uint32_t *, int, int, int, int);
static const rows_op_fn ROWS_FWD[15] = {nullptr, nullptr, nullptr, nullptr, nullptr,
                                        k_rows_fwd<5>, k_rows_fwd<6>, k_rows_fwd<7>, k_rows_fwd<8>,
                                        k_rows_fwd<9>, k_rows_fwd<10>, k_rows_fwd<11>, k_rows_fwd<12>,
                                        k_rows_fwd<13>, k_rows_fwd<14>};
static const rows_op_fn ROWS_INV[15] = {nullptr, nullptr, nullptr, nullptr, nullptr,
                                        k_rows_inv<5>, k_rows_inv<6>, k_rows_inv<7>, k_rows_inv<8>,
                                        k_rows_inv<9>, k_rows_inv<10>, k_rows_inv<11>, k_rows_inv<12>,
                                        k_rows_inv<13>, k_rows_inv<14>};

constexpr int MIN_LOGM = 5;

struct LaunchShape {
    MulShape S;
    int col_threads, col_grid;   // column kernels
    size_t col_smem;
    int nv, row_threads, row_grid;   // row_threads: at 32 elements per thread
    size_t row_smem;
    int loge = 0;                    // row elements per thread 2^loge; 0: rows_loge's rule
};

// Four-step split of a 2^logM transform: rows of 2^logC, columns of
// 2^(logM - logC); logC < 0 takes the longest rows (2^14), which leaves the
// shortest columns.
constexpr int LOG_MAXR = 11;
// Default row length: the whole transform up to 2^13 points; 2^5-point
// columns from 2^14 to 2^17 points and 2^6 at 2^18 (small transforms are
// latency-bound, and 32-point columns spread a product over the most CTAs:
// measured 2^15-point products 0.056 -> 0.030 ms, 2^17-point 0.062 -> 0.038
// ms); 2^13-point rows from 2^19 to 2^24 (more row items for mid sizes), 2^14
// at 2^25 where the columns reach their longest length.
static int default_logC(int logM)
{
    if (logM <= LOG_MAXC - 1) return logM;
    if (logM <= 17) return logM - 5;
    if (logM == 18) return 12;
    return std::max(LOG_MAXC - 1, logM - LOG_MAXR);
}
// Shortest row for a transform of 2^logM points: columns at most 2^11 long,
// and with 32 or more columns (the column kernel's 2^14-word tiles of
// 2^(14 - logR) columns) rows at least one tile wide, which below 2^14
// points means at most 16 columns.
static int min_logC(int logM)
{
    int lo = std::max(MIN_LOGM, logM - LOG_MAXR);
    if (logM < LOG_MAXC) lo = std::max(lo, logM - 4);
    return lo;
}
static bool valid_logC(int logM, int logC)
{
    return logC >= min_logC(logM) && logC <= std::min(logM, LOG_MAXC);
}

static LaunchShape make_shape(int logM, int logC = -1)
{
    LaunchShape L;
    L.S.logC = logC < 0 ? default_logC(logM) : logC;
    L.S.logR = logM - L.S.logC;
    const int R = 1 << L.S.logR, C = 1 << L.S.logC;
    if (L.S.logR >= 5) {
        L.S.G = cols_per_tile(L.S.logR);
        L.col_threads = std::min(512, L.S.G * R / 32);
    } else {
        L.S.G = std::min(C, (1 << 14) >> L.S.logR);
        L.col_threads = std::min(512, L.S.G);
    }
    L.col_grid = C / L.S.G;
    L.col_smem = (size_t)(padw(R * L.S.G) + 32) * sizeof(uint32_t);
    // rows per row-kernel CTA: up to 2^13 words per row buffer, so shorter rows
    // leave room for two CTAs per SM (measured: 2^13-point rows one per CTA
    // 13% faster than two per CTA; 2^12-point rows two per CTA 6% faster than
    // four)
    L.nv = std::min(R, 1 << std::max(0, LOG_MAXC - 1 - L.S.logC));
    L.row_threads = (L.nv * C) >> 5;
    L.row_grid = (R + L.nv - 1) / L.nv;                // items per prime; launch clamps
    L.row_smem = (size_t)3 * L.nv * padw(C) * sizeof(uint32_t);   // b and two a buffers
    return L;
}

// the three transform launches shared by every product type; with a batch
// descriptor array (ninst products of this shape) a, b, ra, rb are ignored;
// with fz the operands are integer polynomials (an, bn coefficients); with co
// the inverse column pass writes a split product's chunk (ChunkOut).  Returns
// the residue array that holds the product (ra, or rb for a large product
// whose b arrives late: b_ready)
static uint32_t *launch_transforms(const Ctx *X, const LaunchShape &L, int np, const uint64_t *a,
                              uint64_t an, const uint64_t *b, uint64_t bn, uint32_t *ra,
                              uint32_t *rb, bool sq, const uint32_t *d_scale, cudaStream_t st,
                              TimingRecord *tr, const InstDesc *desc = nullptr, int ninst = 1,
                              const FzShape *fz = nullptr, cudaEvent_t b_ready = nullptr,
                              const ChunkOut *co = nullptr);

static int upload_scales(Ctx *X);

static int configure_kernels()
{
    static bool done = false;
    if (done) return 0;
    for (int r = 0; r < 12; r++) {
        CU(cudaFuncSetAttribute(FWD_COLS[r], cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024));
        CU(cudaFuncSetAttribute(FWD_COLS_FZ[r], cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024));
        CU(cudaFuncSetAttribute(INV_COLS[r], cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024));
    }
    for (int r = 0; r < 3; r++) {
        CU(cudaFuncSetAttribute(FWD_COLS_C13[r], cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024));
        CU(cudaFuncSetAttribute(FWD_COLS_FZ_C13[r], cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024));
        CU(cudaFuncSetAttribute(INV_COLS_C13[r], cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024));
    }
    CU(cudaFuncSetAttribute(FWD_COLS_C14, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024));
    CU(cudaFuncSetAttribute(FWD_COLS_FZ_C14, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024));
    CU(cudaFuncSetAttribute(INV_COLS_C14, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024));
    for (int r = 0; r < 6; r++) {
        CU(cudaFuncSetAttribute(FWD_COLS3[r], cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024));
        CU(cudaFuncSetAttribute(FWD_COLS3_FZ[r], cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024));
        CU(cudaFuncSetAttribute(INV_COLS3[r], cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024));
    }
    for (int c = ROWS16_MIN_LOGC; c <= LOG_MAXC; c++)
        CU(cudaFuncSetAttribute(ROWS16[c], cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
    for (int c = 5; c <= LOG_MAXC; c++) {
        CU(cudaFuncSetAttribute(ROWS[c], cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
        CU(cudaFuncSetAttribute(ROWS_FWD[c], cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024));
        CU(cudaFuncSetAttribute(ROWS_INV[c], cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024));
    }
    done = true;
    return 0;
}

static int ctx_create(Ctx **out, gpu_ulong p)
{
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        return set_error(GPU_FFT_SMALL_ECUDA, "no CUDA device available (%s)",
                         e != cudaSuccess ? cudaGetErrorString(e) : "0 devices");
    Ctx *X = new Ctx();
    X->p0 = p;
    int rc = 0;
    if (cudaGetDevice(&X->device) != cudaSuccess) rc = set_error(GPU_FFT_SMALL_ECUDA, "cudaGetDevice failed");
    if (!rc && cudaStreamCreateWithFlags(&X->stream, cudaStreamNonBlocking) != cudaSuccess)
        rc = set_error(GPU_FFT_SMALL_ECUDA, "cudaStreamCreate failed");
    if (!rc) rc = configure_kernels();
    if (!rc) rc = ctx_build_tables(X);
    if (!rc) {
        cudaError_t e1 = cudaMalloc(&X->d_scale, sizeof(uint32_t) * (MAX_NP + 2) * (LOG_MAXM + 1) * MAX_NP);
        cudaError_t e2 = cudaMalloc(&X->d_err, sizeof(int));
        cudaError_t e3 = cudaMalloc(&X->d_ticket, sizeof(unsigned long long));
        cudaError_t e4 = cudaHostAlloc(&X->h_err, sizeof(int), cudaHostAllocDefault);
        if (e1 || e2 || e3 || e4) rc = set_error(GPU_FFT_SMALL_ECUDA, "cudaMalloc of context state failed");
        else {
            cudaMemset(X->d_err, 0, sizeof(int));
            cudaMemset(X->d_ticket, 0, sizeof(unsigned long long));
            *X->h_err = 0;
        }
    }
    if (!rc) rc = upload_scales(X);
    if (rc) {
        delete X;
        return rc;
    }
    *out = X;
    return 0;
}

// fold finished records into the per-kernel totals (blocks on pending ones)
static void timing_drain(Ctx *X)
{
    while (X->rec_tail != X->rec_head) {
        TimingRecord &r = X->rec[X->rec_tail % TIMING_RING];
        cudaEventSynchronize(r.ev[TIMING_SLOTS]);
        for (int k = 0; k < TIMING_SLOTS; k++) {
            float ms = 0;
            if (cudaEventElapsedTime(&ms, r.ev[k], r.ev[k + 1]) == cudaSuccess) {
                X->kernel_ms[k] += ms;
                X->kernel_count[k]++;
            }
        }
        X->rec_tail++;
    }
}

static TimingRecord *timing_begin(Ctx *X, cudaStream_t st)
{
    if (!X->timing) return nullptr;
    if (X->rec.empty()) {
        X->rec.resize(TIMING_RING);
        for (auto &r : X->rec) {
            for (auto &e : r.ev) cudaEventCreate(&e);
            r.used = true;
        }
    }
    if (X->rec_head - X->rec_tail >= TIMING_RING) {   // ring full: fold the oldest
        TimingRecord &r = X->rec[X->rec_tail % TIMING_RING];
        cudaEventSynchronize(r.ev[TIMING_SLOTS]);
        for (int k = 0; k < TIMING_SLOTS; k++) {
            float ms = 0;
            if (cudaEventElapsedTime(&ms, r.ev[k], r.ev[k + 1]) == cudaSuccess) {
                X->kernel_ms[k] += ms;
                X->kernel_count[k]++;
            }
        }
        X->rec_tail++;
    }
    TimingRecord *r = &X->rec[X->rec_head % TIMING_RING];
    X->rec_head++;
    cudaEventRecord(r->ev[0], st);
    return r;
}

static void ctx_destroy(Ctx *X)
{
    if (!X) return;
    if (X->stream) cudaStreamSynchronize(X->stream);
    for (auto &r : X->rec)
        for (auto &e : r.ev) cudaEventDestroy(e);
    cudaFree(X->d_tables);
    cudaFree(X->d_scale);
    cudaFree(X->d_err);
    if (X->h_err) cudaFreeHost(X->h_err);
    cudaFree(X->d_ticket);
    cudaFree(X->d_status);
    cudaFree(X->d_res);
    cudaFree(X->d_io);
    if (X->stream) cudaStreamDestroy(X->stream);
    if (X->copy_stream) {
        cudaStreamSynchronize(X->copy_stream);
        cudaStreamDestroy(X->copy_stream);
    }
    for (auto &e : X->ev_copy)
        if (e) cudaEventDestroy(e);
    for (auto &e : X->ev_time)
        if (e) cudaEventDestroy(e);
    cudaFree(X->d_time);
    delete X;
}

// ---------------------------------------------------------------------------
// plans
struct MulPlan {
    int np;
    int logM;
    LaunchShape L;
    int route;   // GPU_MUL_ROUTE_*
};

static int ceil_log2_u64(uint64_t x)
{
    int l = 0;
    while (((uint64_t)1 << l) < x) l++;
    return l;
}

// Plan under an explicit configuration (zero fields take the defaults of
// plan_mpn); every choice is checked against the exactness bound and the
// kernels' shape limits.
static int plan_mpn(uint64_t an, uint64_t bn, MulPlan *P);
static int three_length(uint64_t L, int np, int logM);
static int split_plan(uint64_t an, uint64_t bn, int logM);
static int plan_mpn_cfg(uint64_t an, uint64_t bn, const gpu_mul_config *cfg, MulPlan *P)
{
    int rc = plan_mpn(an, bn, P);
    if (rc || !cfg) return rc;
    if (cfg->route == GPU_MUL_ROUTE_BASECASE) {
        if (std::min(an, bn) > (uint64_t)BASECASE_MAX)
            return set_error(GPU_FFT_SMALL_EINVAL, "basecase route needs an operand of at most %d limbs",
                             BASECASE_MAX);
        if (cfg->np || cfg->logM || cfg->logC || cfg->flags)
            return set_error(GPU_FFT_SMALL_EINVAL, "basecase route takes no transform parameters");
        P->route = GPU_MUL_ROUTE_BASECASE;
        P->np = 0;
        P->logM = std::max(ceil_log2_u64(an + bn - 1), MIN_LOGM);
        return 0;
    }
    if (cfg->route != GPU_MUL_ROUTE_NTT) return set_error(GPU_FFT_SMALL_EINVAL, "unknown route %d", cfg->route);
    if (cfg->np) {
        if (cfg->np < P->np || cfg->np > 6)
            return set_error(GPU_FFT_SMALL_EINVAL, "prime count %d outside [%d, 6]", cfg->np, P->np);
        P->np = cfg->np;
    }
    if (cfg->logM) {
        if (cfg->logM < P->logM || cfg->logM > LOG_MAXM)
            return set_error(GPU_FFT_SMALL_EINVAL, "transform length 2^%d outside [2^%d, 2^%d]", cfg->logM,
                             P->logM, LOG_MAXM);
        P->logM = cfg->logM;
    }
    const int fl = cfg->flags;
    // a 3 2^k-point transform has rows of 2^LOGC3 points whatever logM is
    const int logC = (fl & GPU_MUL_FLAG_THREE) ? LOGC3 : cfg->logC ? cfg->logC : default_logC(P->logM);
    if (!(fl & GPU_MUL_FLAG_THREE) && !valid_logC(P->logM, logC))
        return set_error(GPU_FFT_SMALL_EINVAL, "row length 2^%d invalid for a 2^%d transform", logC, P->logM);
    P->L = make_shape(P->logM, (fl & GPU_MUL_FLAG_THREE) ? -1 : logC);
    if (fl & ~(GPU_MUL_FLAG_THREE | GPU_MUL_FLAG_SPLIT | GPU_MUL_FLAG_ROWS16 | GPU_MUL_FLAG_ROWS32))
        return set_error(GPU_FFT_SMALL_EINVAL, "unknown configuration flags 0x%x", fl);
    if ((fl & GPU_MUL_FLAG_ROWS16) && (fl & GPU_MUL_FLAG_ROWS32))
        return set_error(GPU_FFT_SMALL_EINVAL, "ROWS16 and ROWS32 exclude each other");
    if ((fl & GPU_MUL_FLAG_ROWS16) && ((fl & (GPU_MUL_FLAG_THREE | GPU_MUL_FLAG_SPLIT)) || logC < ROWS16_MIN_LOGC))
        return set_error(GPU_FFT_SMALL_EINVAL, "16 points per thread need rows of 2^%d points or more "
                         "and neither THREE nor SPLIT", ROWS16_MIN_LOGC);
    if (fl & GPU_MUL_FLAG_ROWS16) P->L.loge = 4;
    if (fl & GPU_MUL_FLAG_ROWS32) P->L.loge = 5;
    if ((fl & GPU_MUL_FLAG_THREE) && (fl & GPU_MUL_FLAG_SPLIT))
        return set_error(GPU_FFT_SMALL_EINVAL, "THREE and SPLIT exclude each other");
    if ((fl & GPU_MUL_FLAG_THREE) && !three_length(an + bn - 1, P->np, P->logM))
        return set_error(GPU_FFT_SMALL_EINVAL, "no 3 2^%d-point transform for a %llu x %llu product with %d primes",
                         P->logM - 2, (unsigned long long)an, (unsigned long long)bn, P->np);
    if ((fl & GPU_MUL_FLAG_THREE) && cfg->logC && cfg->logC != LOGC3)
        return set_error(GPU_FFT_SMALL_EINVAL, "3 2^k-point transforms use 2^%d-point rows", LOGC3);
    if ((fl & GPU_MUL_FLAG_SPLIT) && !split_plan(an, bn, P->logM))
        return set_error(GPU_FFT_SMALL_EINVAL, "a %llu x %llu product does not split",
                         (unsigned long long)an, (unsigned long long)bn);
    return 0;
}

static int plan_mpn(uint64_t an, uint64_t bn, MulPlan *P)
{
    if (an == 0 || bn == 0) return set_error(GPU_FFT_SMALL_EINVAL, "empty operand");
    const uint64_t L = an + bn - 1;
    const uint64_t mn = std::min(an, bn);
    // every coefficient is < mn 2^128; the CRT needs P > 2 * bound
    const double need = log2((double)mn) + 128.0 + 1.0 + 1e-3;
    int np = 0;
    for (int k = 1; k <= 6; k++)
        if (log2_product(k) > need) { np = k; break; }
    if (np == 0) return set_error(GPU_FFT_SMALL_ENOPRIMES, "operand length %llu beyond the prime set",
                                  (unsigned long long)mn);
    np = std::max(np, 5);
    int logM = std::max(ceil_log2_u64(L), MIN_LOGM);
    if (logM > LOG_MAXM)
        return set_error(GPU_FFT_SMALL_ETOOBIG, "product of %llu coefficients exceeds 2^%d",
                         (unsigned long long)L, LOG_MAXM);
    P->np = np;
    P->logM = logM;
    P->L = make_shape(logM);
    P->route = GPU_MUL_ROUTE_NTT;
    return 0;
}

// pointwise scale: M^-1 (P/p_j)^-1 2^128, see k_rows / limb_redc
static void fill_scale(const Ctx *X, int np, int logM, uint32_t *scale, int extra_redc)
{
    for (int j = 0; j < np; j++) {
        const uint32_t p = PRIMES[j];
        uint32_t s = h_invmod(h_powmod(2, logM, p), p);
        s = h_mulmod(s, h_invmod(X->cof_red[np][j], p), p);
        s = h_mulmod(s, h_powmod(2, 32 * (uint64_t)extra_redc, p), p);
        scale[j] = s;
    }
}

// pointwise scale of a 3 2^k-point transform: (3 2^k)^-1 (P/p_j)^-1 2^128
static void fill_scale3(const Ctx *X, int np, int k, uint32_t *scale)
{
    for (int j = 0; j < np; j++) {
        const uint32_t p = PRIMES[j];
        uint32_t s = h_invmod(h_mulmod(3, h_powmod(2, k, p), p), p);
        s = h_mulmod(s, h_invmod(X->cof_red[np][j], p), p);
        s = h_mulmod(s, h_powmod(2, 128, p), p);
        scale[j] = s;
    }
}

static int ensure_status(Ctx *X, size_t tiles)
{
    if (tiles <= X->status_cap) return 0;
    if (X->d_status) cudaFree(X->d_status);
    X->d_status = nullptr;
    X->status_cap = 0;
    CU(cudaMalloc(&X->d_status, tiles * sizeof(uint32_t)));
    CU(cudaMemsetAsync(X->d_status, 0, tiles * sizeof(uint32_t), X->stream));
    X->status_cap = tiles;
    return 0;
}

static const uint32_t *scale_ptr(const Ctx *X, int np, int logM)
{
    return X->d_scale + ((size_t)np * (LOG_MAXM + 1) + logM) * MAX_NP;
}
// scales of the 3 2^k-point transforms (NP3 primes), after the 2^logM ones
static const uint32_t *scale3_ptr(const Ctx *X, int k)
{
    return X->d_scale + ((size_t)(MAX_NP + 1) * (LOG_MAXM + 1) + k) * MAX_NP;
}

// pointwise scales for every (np, logM), uploaded once per context
static int upload_scales(Ctx *X)
{
    std::vector<uint32_t> tab((size_t)(MAX_NP + 2) * (LOG_MAXM + 1) * MAX_NP, 0);
    for (int np = 1; np <= MAX_NP; np++)
        for (int lm = 0; lm <= LOG_MAXM; lm++)
            fill_scale(X, np, lm, &tab[((size_t)np * (LOG_MAXM + 1) + lm) * MAX_NP], 4);
    for (int k = 0; k <= LOG_MAXM; k++)
        fill_scale3(X, NP3, k, &tab[((size_t)(MAX_NP + 1) * (LOG_MAXM + 1) + k) * MAX_NP]);
    CU(cudaMemcpy(X->d_scale, tab.data(), tab.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    return 0;
}

// Resident row CTAs per SM for a shape: 1 for long rows (512 threads, ~135 KB
// of shared memory), several for short ones.  The row launch depends on the
// row length and the rows per item.
static int rows_per_sm(const LaunchShape &L, int loge = 5)
{
    static int occ[2][LOG_MAXC + 1][LOG_MAXC + 1] = {{{0}}};
    const int c = L.S.logC, v = __builtin_ctz((unsigned)L.nv), e = loge == 4;
    if (occ[e][c][v] == 0) {
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, e ? ROWS16[c] : ROWS[c], (L.nv << c) >> loge,
                                                          L.row_smem) != cudaSuccess || n < 1)
            n = 1;
        occ[e][c][v] = n;
    }
    return occ[e][c][v];
}

// Row elements per thread (log2) for a launch of ninst products of np primes:
// the shape's choice, else 16 where 32 would give the launch fewer than 16
// warps per SM (measured on 2^15- to 2^18-point products, whose row items
// run latency-bound at 8 warps per CTA), else 32.
static int rows_loge(const Ctx *X, const LaunchShape &L, int np, int ninst)
{
    if (L.loge) return L.loge;
    if (L.S.logC < ROWS16_MIN_LOGC) return 5;
    const uint64_t warps = ((uint64_t)np * (uint64_t)ninst << (L.S.logR + L.S.logC)) >> 10;
    return warps < (uint64_t)X->nsm * 16 ? 4 : 5;
}

// The row launch of ninst products of np primes: rows per item as the
// shape has them (up to 2^13 points per CTA), halved while the launch would
// have fewer than two items per SM (small transforms).
static LaunchShape row_launch_shape(const Ctx *X, const LaunchShape &L, int np, int ninst)
{
    LaunchShape Lr = L;
    const int R = 1 << L.S.logR;
    while (Lr.nv > 1 && (int64_t)(R / Lr.nv) * np * ninst < 2 * (int64_t)X->nsm) Lr.nv >>= 1;
    Lr.row_grid = (R + Lr.nv - 1) / Lr.nv;
    Lr.row_smem = (size_t)3 * Lr.nv * padw(1 << L.S.logC) * sizeof(uint32_t);
    return Lr;
}

// A column launch: the shape's 2^14-word tiles, or narrow ones (a quarter of
// the columns) where the launch would have fewer than two CTAs per SM --
// small transforms, whose column passes are bound by latency, not by HBM.
struct ColLaunch {
    int G, grid, threads;
    size_t smem;
    bool narrow;
};
static ColLaunch col_launch(const Ctx *X, const LaunchShape &L, int np, int zdim, bool fz)
{
    const MulShape &S = L.S;
    ColLaunch c{S.G, L.col_grid, L.col_threads, L.col_smem, false};
    const int64_t want = 2 * (int64_t)X->nsm;
    if (!fz && S.logR >= 5 && S.logR <= 8 && (int64_t)L.col_grid * np * zdim < want) {
        c.G = S.G / 4;
        c.grid = L.col_grid * 4;
        c.threads = L.col_threads / 4;
        c.smem = (size_t)(padw((1 << S.logR) * c.G) + 32) * sizeof(uint32_t);
        c.narrow = true;
    } else if (S.logR < 5) {
        // short columns (one thread per column, tile width at run time):
        // halve the tile down to 128 columns
        const int C = 1 << S.logC;
        while (c.G > 128 && (int64_t)(C / c.G) * np * zdim < want) c.G >>= 1;
        c.grid = C / c.G;
        c.threads = std::min(512, c.G);
        c.smem = (size_t)(padw((1 << S.logR) * c.G) + 32) * sizeof(uint32_t);
    }
    return c;
}

static uint32_t *launch_transforms(const Ctx *X, const LaunchShape &L, int np, const uint64_t *a,
                                   uint64_t an, const uint64_t *b, uint64_t bn, uint32_t *ra,
                                   uint32_t *rb, bool sq, const uint32_t *d_scale, cudaStream_t st,
                                   TimingRecord *tr, const InstDesc *desc, int ninst, const FzShape *fz,
                                   cudaEvent_t b_ready, const ChunkOut *co)
{
    const MulShape &S = L.S;
    const int zdim = desc ? 2 * ninst : (sq ? 1 : 2);
    const int ni = desc ? ninst : 1;
    const ColLaunch cf = col_launch(X, L, np, zdim, fz != nullptr);
    const ColLaunch ci = col_launch(X, L, np, ni, false);
    const fwd_cols_fn fwd = cf.narrow ? FWD_COLS_S[S.logR - 5] : fwd_cols_kernel(S.logR, S.logC, fz != nullptr);
    const inv_cols_fn inv = ci.narrow ? INV_COLS_S[S.logR - 5] : inv_cols_kernel(S.logR, S.logC);
    const FzShape shape = fz ? *fz : FzShape{1, 1, 1};
    // Products of two operands whose columns are long enough for the
    // per-thread twist (2^5 points or more) fold the pointwise scale into
    // b's twist factors, so the row pass multiplies the spectra once instead
    // of twice; squarings keep the scale in the row pass.
    const bool fold = !(sq && !desc) && S.logR >= 5;
    const int R = 1 << S.logR;
    if (b_ready && !desc && !sq) {
        // b is still arriving: a's column pass first, b's after its copy
        fwd<<<dim3(np, cf.grid, 1), cf.threads, cf.smem, st>>>(X->T, a, an, a, an, ra, ra, S.logC, cf.G, nullptr,
                                                               np, shape, d_scale, 0);
        // A large product also runs a's forward row transforms before b has
        // arrived (k_rows_fwd); the row pass then transforms b alone and
        // multiplies it by a's spectrum (squaring mode 2, as the chunks of a
        // split product do), so less of the transform waits for b's upload.
        // The product ends in b's residues.
        const bool early = !fz && !co && fold && S.logR + S.logC >= 20;
        if (early) {
            const int C = 1 << S.logC, groups = (R + L.nv - 1) / L.nv;
            ROWS_FWD[S.logC]<<<groups * np, L.nv * C / 32, (size_t)L.nv * padw(C) * sizeof(uint32_t), st>>>(
                X->T, ra, S.logR, L.nv, np, R);
        }
        cudaStreamWaitEvent(st, b_ready, 0);
        const FzShape shb = fz ? FzShape{shape.S, shape.wb, shape.wb} : shape;
        fwd<<<dim3(np, cf.grid, 1), cf.threads, cf.smem, st>>>(X->T, b, bn, b, bn, rb, rb, S.logC, cf.G, nullptr,
                                                               np, shb, d_scale, fold ? 1 : 0);
        if (early) {
            timing_mark(tr, 1, st);
            ROWS[S.logC]<<<std::min(L.row_grid * np, X->nsm * rows_per_sm(L)), L.row_threads, L.row_smem, st>>>(
                X->T, rb, ra, S.logR, L.nv, np, nullptr, 2, nullptr, 1, R);
            timing_mark(tr, 2, st);
            inv<<<dim3(ci.grid, np, 1), ci.threads, ci.smem, st>>>(X->T, rb, S.logC, ci.G, nullptr,
                                                                   ChunkOut{nullptr, 0, 0, 0, 0});
            timing_mark(tr, 3, st);
            return rb;
        }
    } else {
        if (b_ready) cudaStreamWaitEvent(st, b_ready, 0);
        fwd<<<dim3(np, cf.grid, zdim), cf.threads, cf.smem, st>>>(X->T, a, an, b, bn, ra, rb, S.logC, cf.G, desc,
                                                                  np, shape, d_scale, fold ? 2 : 0);
    }
    timing_mark(tr, 1, st);
    const LaunchShape Lr = row_launch_shape(X, L, np, ni);
    const int items = Lr.row_grid * np * ni;
    const int loge = rows_loge(X, Lr, np, ni);
    (loge == 4 ? ROWS16 : ROWS)[S.logC]<<<std::min(items, X->nsm * rows_per_sm(Lr, loge)),
                                         (Lr.nv << S.logC) >> loge, Lr.row_smem, st>>>(
        X->T, ra, rb, S.logR, Lr.nv, np, fold ? nullptr : d_scale, (sq && !desc) ? 1 : 0, desc, ni, R);
    timing_mark(tr, 2, st);
    if (S.logR > 0)
        inv<<<dim3(ci.grid, np, ni), ci.threads, ci.smem, st>>>(X->T, ra, S.logC, ci.G, desc,
                                                                co ? *co : ChunkOut{nullptr, 0, 0, 0, 0});
    timing_mark(tr, 3, st);
    return ra;
}

// Transform of M = 3 2^k points (k - 13 in [LOG3_RMIN, LOG3_RMAX]): columns of
// 3 2^(k - 13) points with a radix-3 stage, 2^13-point rows; residue planes
// of 2^logMs words (logMs = k + 2).  The pointwise scale is folded into b's
// twist as in launch_transforms (squarings keep it in the row pass).  With fz
// the operands are integer polynomials (an, bn coefficients).
static void launch_transforms3(const Ctx *X, int k, int logMs, const uint64_t *a, uint64_t an,
                               const uint64_t *b, uint64_t bn, uint32_t *ra, uint32_t *rb, bool sq,
                               cudaStream_t st, TimingRecord *tr, cudaEvent_t b_ready,
                               const FzShape *fz = nullptr)
{
    const int np = NP3, r = k - LOGC3;
    const int G = cols_per_tile3(r);
    const int C = 1 << LOGC3, rows = 3 << r;
    const size_t smem = (size_t)(padw(3 * (1 << r) * G) + 32) * sizeof(uint32_t);
    const uint32_t *sc = scale3_ptr(X, k);
    if (b_ready) cudaStreamWaitEvent(st, b_ready, 0);
    (fz ? FWD_COLS3_FZ : FWD_COLS3)[r - LOG3_RMIN]<<<dim3(np, C / G, sq ? 1 : 2), 512, smem, st>>>(
        X->T, a, an, b, bn, ra, rb, logMs, k, sc, sq ? 0 : 2, fz ? *fz : FzShape{1, 1, 1});
    timing_mark(tr, 1, st);
    const LaunchShape L = make_shape(logMs, LOGC3);   // row launch shape (one 2^13-point row per item)
    const int items = rows * np;
    ROWS[LOGC3]<<<std::min(items, X->nsm * rows_per_sm(L)), L.row_threads, L.row_smem, st>>>(
        X->T, ra, rb, logMs - LOGC3, 1, np, sq ? sc : nullptr, sq ? 1 : 0, nullptr, 1, rows);
    timing_mark(tr, 2, st);
    INV_COLS3[r - LOG3_RMIN]<<<dim3(C / G, np), 512, smem, st>>>(X->T, ra, logMs, k);
    timing_mark(tr, 3, st);
}

// The 3 2^k-point length for a whole product of L coefficients on the
// default plan (np primes, 2^logM points), or 0 where the power of two stays
// (beyond 3 2^(logM - 2), other prime counts, sizes outside the kernels').
static int three_length(uint64_t L, int np, int logM)
{
    const int k = logM - 2;
    if (np != NP3 || k - LOGC3 < LOG3_RMIN || k - LOGC3 > LOG3_RMAX) return 0;
    return L <= (3ull << k) ? k : 0;
}

// Schoolbook route: column sums, then the carry kernel's direct mode.
static int mpn_mul_basecase_enqueue(Ctx *X, uint64_t *z, const uint64_t *a, uint64_t an,
                                    const uint64_t *b, uint64_t bn, int logM, cudaStream_t st)
{
    const uint64_t *x = a, *y = b;
    uint64_t xn = an, yn = bn;
    if (yn > xn) { std::swap(x, y); std::swap(xn, yn); }
    const uint64_t L = an + bn - 1, zn = an + bn;
    const size_t plane = (size_t)1 << logM;
    int rc = grow((void **)&X->d_res, &X->res_cap, 3 * plane * sizeof(uint64_t));
    if (rc) return rc;
    uint64_t *sums = (uint64_t *)X->d_res;
    constexpr int THREADS = 256, TILE = 4 * THREADS;
    const size_t tiles = (zn + TILE - 1) / TILE;
    rc = ensure_status(X, tiles);
    if (rc) return rc;
    X->epoch = (X->epoch + 1) & 0x0fffffffu;
    if (X->epoch == 0) {
        CU(cudaMemsetAsync(X->d_status, 0, X->status_cap * sizeof(uint32_t), st));
        X->epoch = 1;
    }
    TimingRecord *tr = timing_begin(X, st);
    // column sums split over positions and short-operand chunks, added into
    // zeroed planes (k_basecase_split)
    CU(cudaMemsetAsync(sums, 0, 3 * plane * sizeof(uint64_t), st));
    k_basecase_split<<<dim3((unsigned)((L + BC_POS - 1) / BC_POS), (unsigned)((yn + BC_JCH - 1) / BC_JCH)),
                       BC_THREADS, 0, st>>>(x, xn, y, yn, (unsigned long long *)sums, logM);
    timing_mark(tr, 1, st);
    timing_mark(tr, 2, st);
    timing_mark(tr, 3, st);
    k_crt_carry<0, THREADS><<<tiles, THREADS, 0, st>>>((const uint32_t *)sums, logM, L, zn, z, X->crt[5],
                                                       X->d_status, X->d_ticket, X->ticket_base, X->epoch,
                                                       X->d_err, nullptr, nullptr, 0ull);
    timing_mark(tr, 4, st);
    X->ticket_base += tiles;
    X->last_launches = 2;
    CU(cudaGetLastError());
    return 0;
}

// Cyclic length of a window product of limbs [lo, hi): coefficients
// lo - 3 .. hi - 1 must be free of wrap-around (M >= L - lo + 3) and
// addressable (M >= min(hi, L)), L = an + bn - 1.
static int window_logM(uint64_t an, uint64_t bn, uint64_t lo, uint64_t hi)
{
    const uint64_t L = an + bn - 1;
    const uint64_t need = std::max(std::min(hi, L), L + 3 > lo ? L + 3 - lo : 1);
    return std::max(ceil_log2_u64(need), MIN_LOGM);
}

// Enqueue z = limbs [lo, hi) of a * b on `st` with device pointers (cfg NULL:
// default plan; the default window is the whole product).  For lo > 0 the
// carry chain starts at limb lo: the coefficients below lo add their words
// that land in the window but not the carry that would ripple up from the
// limbs below, so the result is a lower approximation of floor(a b / 2^(64 lo))
// short by at most 2 units (and by 0 unless limb lo - 1 of the exact product
// is within 2 of 2^64 - 1).  That is the contract of the reference's
// _mpn_ctx_mpn_mul_range (lower approximation, deficit <= min(an, bn, lo)
// 2^64, exact for lo = 0), and the result depends on a, b and lo only, not on
// hi or the transform length.  A window far below the top uses a shorter
// cyclic transform (window_logM).
// A host-pointer product copies each CRT chunk back while the next one runs:
// after the launch of chunk k (limbs [l0, l1) of the output) the hook queues
// its copy.
struct CrtChunks {
    int chunks = 1;
    void (*hook)(void *arg, uint64_t l0, uint64_t l1) = nullptr;
    void *arg = nullptr;
};

// Chunk transform length for an unbalanced whole product (0: one transform).
// Chunks of the long operand of c = 2^Lc - yn + 1 limbs each multiply the
// short operand in a 2^Lc-point transform; the short operand is transformed
// once, so k chunks cost 2k + 1 transforms of Lc levels on 2^Lc points
// against 3 of logM levels on 2^logM, plus a fixed cost per chunk (its
// three launches and their tails: about 24 2^20 level-points, measured as
// ~0.04 ms per 2^20-point chunk on the B200).  Splitting is taken when that
// is at most 75% of the single transform's work (the margin covers the
// separate spectrum pass and the CRT, which costs the same either way), for
// products of 2^20 points or more and chunks of at least 2^20 points.
// Measured (split / single transform): 2^24 x 2^20 0.66, 2^22 x 3000 0.71,
// 2^23 x 7 10^5 0.70, 5 10^6 x 3 10^5 0.77, 2^24 x 2^22 0.90; without the
// chunk cost term 2^23 x 1 (8 chunks) 1.06 and 3 2^20 x 2^16 1.10, which
// now take the single transform.  (The reference truncates its transforms
// instead, src/fft_small/sd_fft.c:1230-1274.)
static int split_search(uint64_t xn, uint64_t yn, int Lmax, double *best_cost)
{
    int best = 0;
    for (int Lc = 20; Lc <= Lmax; Lc++) {
        const uint64_t Mc = (uint64_t)1 << Lc;
        if (Mc < 2 * yn) continue;
        const uint64_t c = Mc - yn + 1;
        const uint64_t k = (xn + c - 1) / c;
        const double cost = (double)(2 * k + 1) * Lc * (double)Mc + (double)k * (24u << 20);
        if (cost < *best_cost) { *best_cost = cost; best = Lc; }
    }
    return best;
}

static int split_plan(uint64_t an, uint64_t bn, int logM)
{
    if (logM < 20) return 0;
    double cost = 0.75 * 3.0 * logM * (double)((uint64_t)1 << logM);
    return split_search(std::max(an, bn), std::min(an, bn), logM - 1, &cost);
}

// Whole products beyond the longest transform (an + bn - 1 > 2^25 limbs)
// run split when the short operand leaves room for chunks of at most 2^25
// points: the chunk length is the cheapest by the same count, the residues
// of the whole product take 2^logM words per prime (logM <= LOG_MAX_SPLIT),
// and the prime count is the one the coefficient bound of the short operand
// asks for, as for any product.
constexpr int LOG_MAX_SPLIT = 30;

static int plan_mpn_oversize(uint64_t an, uint64_t bn, MulPlan *P, int *Lc)
{
    const uint64_t L = an + bn - 1, yn = std::min(an, bn);
    const int logM = ceil_log2_u64(L);
    if (logM > LOG_MAX_SPLIT)
        return set_error(GPU_FFT_SMALL_ETOOBIG, "product of %llu coefficients exceeds 2^%d",
                         (unsigned long long)L, LOG_MAX_SPLIT);
    double cost = 1e300;
    const int lc = split_search(std::max(an, bn), yn, LOG_MAXM, &cost);
    if (!lc)
        return set_error(GPU_FFT_SMALL_ETOOBIG, "product of %llu coefficients with a %llu-limb short operand "
                         "exceeds a 2^%d transform", (unsigned long long)L, (unsigned long long)yn, LOG_MAXM);
    MulPlan Q;
    int rc = plan_mpn(yn, yn, &Q);   // the prime count for a short operand of yn limbs
    if (rc) return rc;
    P->np = Q.np;
    P->logM = logM;
    P->route = GPU_MUL_ROUTE_NTT;
    *Lc = lc;
    return 0;
}

static int mpn_mul_enqueue(Ctx *X, uint64_t *z, const uint64_t *a, uint64_t an,
                           const uint64_t *b, uint64_t bn, cudaStream_t st,
                           const gpu_mul_config *cfg = nullptr, uint64_t lo = 0, uint64_t hi = ~0ull,
                           cudaEvent_t b_ready = nullptr, const CrtChunks *chunks = nullptr)
{
    MulPlan P;
    int rc = plan_mpn_cfg(an, bn, cfg, &P);
    const uint64_t zfull = an + bn;
    hi = std::min(hi, zfull);
    const bool window = lo > 0 || hi < zfull;
    // beyond the longest transform: a whole unbalanced product may still run split
    int Lover = 0;
    if (rc == GPU_FFT_SMALL_ETOOBIG && !cfg && !window && !(a == b && an == bn))
        rc = plan_mpn_oversize(an, bn, &P, &Lover);
    if (rc) return rc;
    if (lo >= hi) return 0;
    if (P.route == GPU_MUL_ROUTE_BASECASE) {
        if (window) return set_error(GPU_FFT_SMALL_EINVAL, "the basecase route computes whole products only");
        if (b_ready) CU(cudaStreamWaitEvent(st, b_ready, 0));
        rc = mpn_mul_basecase_enqueue(X, z, a, an, b, bn, P.logM, st);
        if (!rc && chunks && chunks->hook) chunks->hook(chunks->arg, 0, zfull);
        return rc;
    }
    // limbs [lo, hi): the carry chain starts at lo; a shorter cyclic
    // transform is used when the window allows one
    const uint64_t base = lo;
    if (lo > 0 && !(cfg && cfg->logM)) {
        const int lw = window_logM(an, bn, lo, hi);
        if (lw < P.logM) {
            const int loge = P.L.loge;
            P.logM = lw;
            P.L = make_shape(lw, cfg && cfg->logC && valid_logC(lw, cfg->logC) ? cfg->logC : -1);
            if (P.L.S.logC >= ROWS16_MIN_LOGC) P.L.loge = loge;
        }
    }
    const bool sq = (a == b) && (an == bn);
    const int np = P.np, logM = P.logM;
    const size_t M = (size_t)1 << logM;
    // an unbalanced whole product may run as chunks of the long operand
    // against the short one (split_plan): their residues are summed into
    // one array of the full length, then a single CRT/carry pass follows
    const int fl = cfg ? cfg->flags : 0;
    const int Lc = Lover ? Lover : ((!cfg || (fl & GPU_MUL_FLAG_SPLIT)) && !window && !sq) ? split_plan(an, bn, logM) : 0;
    // whole products between 2^(logM - 1) and 3 2^(logM - 2) coefficients on
    // the default plan (or under the THREE flag) run a 3 2^(logM - 2)-point
    // transform
    const int k3 = ((!cfg || (fl & GPU_MUL_FLAG_THREE)) && !window && !Lc) ? three_length(an + bn - 1, np, logM) : 0;
    const size_t Mc = Lc ? (size_t)1 << Lc : 0;
    const size_t res_bytes = Lc ? (size_t)np * (M + 2 * Mc) * sizeof(uint32_t)
                                : (sq ? 1 : 2) * (size_t)np * M * sizeof(uint32_t);
    rc = grow((void **)&X->d_res, &X->res_cap, res_bytes);
    if (rc) return rc;
    uint32_t *ra = X->d_res, *rb = X->d_res + (size_t)np * M;
    const uint64_t zn = hi;   // limbs produced: [base, hi)
    constexpr int THREADS = CRT_THREADS, TILE = CRT_TILE;
    const size_t tiles = (zn - base + TILE - 1) / TILE;
    rc = ensure_status(X, tiles);
    if (rc) return rc;
    X->epoch = (X->epoch + 1) & 0x0fffffffu;
    if (X->epoch == 0) {   // epoch wrapped: clear stale status words
        CU(cudaMemsetAsync(X->d_status, 0, X->status_cap * sizeof(uint32_t), st));
        X->epoch = 1;
    }
    const CrtConst &K = X->crt[np];

    int launches = 3;
    TimingRecord *tr = timing_begin(X, st);
    if (Lc) {
        // chunk i: x[i c, i c + c) times y, c = 2^Lc - yn + 1 (the chunk's
        // product fills the 2^Lc-point transform without wrapping); y's
        // spectrum is computed once (column pass, k_rows_fwd) and every
        // chunk's row pass transforms only its x part (squaring mode 2); the
        // chunk's residues land at i c in ra, added where chunk i - 1's end
        const uint64_t *x = a, *y = b;
        uint64_t xn = an, yn = bn;
        if (yn > xn) { std::swap(x, y); std::swap(xn, yn); }
        const uint64_t c = Mc - yn + 1;
        uint32_t *ca = ra + (size_t)np * M, *cb = ca + (size_t)np * Mc;
        const LaunchShape Ls = make_shape(Lc);
        const MulShape &S = Ls.S;
        const FzShape one{1, 1, 1};
        if (b_ready) CU(cudaStreamWaitEvent(st, b_ready, 0));
        fwd_cols_kernel(S.logR, S.logC)<<<dim3(np, Ls.col_grid, 1), Ls.col_threads, Ls.col_smem, st>>>(
            X->T, y, yn, y, yn, cb, cb, S.logC, S.G, nullptr, np, one, nullptr, 0);
        ROWS_FWD[S.logC]<<<((1 << S.logR) / Ls.nv) * np, Ls.nv * (1 << S.logC) / 32,
                           Ls.nv * padw(1 << S.logC) * sizeof(uint32_t), st>>>(X->T, cb, S.logR, Ls.nv, np,
                                                                              1 << S.logR);
        launches = 2;
        const int items = Ls.row_grid * np;
        for (uint64_t i = 0; i * c < xn; i++) {
            const uint64_t xi = std::min(c, xn - i * c);
            const ChunkOut co{ra, logM, i * c, i ? yn - 1 : 0, xi + yn - 1};
            fwd_cols_kernel(S.logR, S.logC)<<<dim3(np, Ls.col_grid, 1), Ls.col_threads, Ls.col_smem, st>>>(
                X->T, x + i * c, xi, x + i * c, xi, ca, ca, S.logC, S.G, nullptr, np, one, nullptr, 0);
            ROWS[S.logC]<<<std::min(items, X->nsm * rows_per_sm(Ls)), Ls.row_threads, Ls.row_smem, st>>>(
                X->T, ca, cb, S.logR, Ls.nv, np, scale_ptr(X, np, Lc), 2, nullptr, 1, 1 << S.logR);
            inv_cols_kernel(S.logR, S.logC)<<<dim3(Ls.col_grid, np, 1), Ls.col_threads, Ls.col_smem, st>>>(X->T, ca, S.logC, S.G,
                                                                                          nullptr, co);
            launches += 3;
        }
        timing_mark(tr, 1, st);
        timing_mark(tr, 2, st);
        timing_mark(tr, 3, st);
    } else if (k3) {
        launch_transforms3(X, k3, logM, a, an, b, bn, ra, rb, sq, st, tr, b_ready);
    } else {
        // the product's residues: ra, or rb when b arrived late (launch_transforms)
        ra = launch_transforms(X, P.L, np, a, an, b, bn, ra, rb, sq, scale_ptr(X, np, logM), st, tr, nullptr, 1,
                               nullptr, b_ready);
    }
    // tiles take their index from the ticket counter, so consecutive launches
    // with the same ticket base continue one carry chain: tile k's look-back
    // finds tile k - 1 finished by an earlier launch
    const int nch = (chunks && !window) ? std::max(1, std::min<int>(chunks->chunks, (int)tiles)) : 1;
    for (int c = 0; c < nch; c++) {
        const size_t t0 = tiles * c / nch, t1 = tiles * (c + 1) / nch;
        if (t1 == t0) continue;
        if (np == 5)
            k_crt_carry<5, THREADS><<<t1 - t0, THREADS, 0, st>>>(ra, logM, an + bn - 1, zn, z, K, X->d_status,
                                                                X->d_ticket, X->ticket_base, X->epoch, X->d_err,
                                                                nullptr, nullptr, base);
        else
            k_crt_carry<6, THREADS><<<t1 - t0, THREADS, 0, st>>>(ra, logM, an + bn - 1, zn, z, K, X->d_status,
                                                                X->d_ticket, X->ticket_base, X->epoch, X->d_err,
                                                                nullptr, nullptr, base);
        if (chunks && chunks->hook)
            chunks->hook(chunks->arg, base + t0 * TILE, std::min<uint64_t>(zn, base + t1 * TILE));
    }
    launches++;
    timing_mark(tr, 4, st);
    X->ticket_base += tiles;
    X->last_launches = launches;
    CU(cudaGetLastError());
    return 0;
}

static int check_device_error(Ctx *X)
{
    int err = 0;
    CU(cudaMemcpyAsync(&err, X->d_err, sizeof(int), cudaMemcpyDeviceToHost, X->stream));
    CU(cudaStreamSynchronize(X->stream));
    if (err) {
        cudaMemsetAsync(X->d_err, 0, sizeof(int), X->stream);
        return set_error(GPU_FFT_SMALL_ETIMEOUT, "carry look-back wait exceeded its limit");
    }
    return 0;
}

static int io_buffers(Ctx *X, size_t words, uint64_t **p)
{
    int rc = grow((void **)&X->d_io, &X->io_cap, words * sizeof(uint64_t));
    if (rc) return rc;
    *p = X->d_io;
    return 0;
}

static Ctx *get_ctx(gpu_mpn_ctx_t R) { return (Ctx *)R->impl; }

static int bind_device(Ctx *X)
{
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != X->device) CU(cudaSetDevice(X->device));
    return 0;
}

static int ensure_copy_stream(Ctx *X)
{
    if (X->copy_stream) return 0;
    CU(cudaStreamCreateWithFlags(&X->copy_stream, cudaStreamNonBlocking));
    for (auto &e : X->ev_copy) CU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return 0;
}

// Copy streams shared by several contexts (a pipeline): all uploads on one
// stream and all downloads on another, so each direction of the link moves
// one product at a time; per-product events order them with the kernels.
struct HostLinks {
    cudaStream_t up, down;
    cudaEvent_t a_in, b_in, done;   // a uploaded, b uploaded, last download queued
};

// Host-pointer product, queued: a's upload on the compute stream, b's on the
// copy stream (or both on links->up), the kernels, and the result's download
// in chunks on the copy stream (or links->down).  Returns once all of it is
// queued; mpn_mul_host_finish waits for the result and checks the device
// error flag.
static int mpn_mul_host_issue(Ctx *X, gpu_ulong *z, const gpu_ulong *a, gpu_ulong an,
                              const gpu_ulong *b, gpu_ulong bn, gpu_ulong lo, gpu_ulong hi,
                              const HostLinks *links = nullptr)
{
    if (!X) return set_error(GPU_FFT_SMALL_EINVAL, "context not initialised");
    if (an == 0 || bn == 0) return set_error(GPU_FFT_SMALL_EINVAL, "empty operand");
    int rc = bind_device(X);
    if (rc) return rc;
    const bool sq = (a == b) && (an == bn);
    const size_t zn = an + bn;
    const gpu_ulong top = std::min<gpu_ulong>(hi, zn);
    const size_t nz = top > lo ? top - lo : 0;
    uint64_t *buf;
    rc = io_buffers(X, (sq ? an : an + bn) + nz, &buf);
    if (rc) return rc;
    uint64_t *da = buf, *db = sq ? buf : buf + an, *dz = buf + (sq ? an : an + bn);
    if (nz) {
        rc = ensure_copy_stream(X);
        if (rc) return rc;
        cudaStream_t S = X->stream, C = X->copy_stream;
        const cudaStream_t down = links ? links->down : C;
        cudaEvent_t b_ready = nullptr;
        if (links) {
            CU(cudaMemcpyAsync(da, a, an * 8, cudaMemcpyHostToDevice, links->up));
            CU(cudaEventRecord(links->a_in, links->up));
            CU(cudaStreamWaitEvent(S, links->a_in, 0));
            if (!sq) {
                CU(cudaMemcpyAsync(db, b, bn * 8, cudaMemcpyHostToDevice, links->up));
                CU(cudaEventRecord(links->b_in, links->up));
                b_ready = links->b_in;
            }
        } else {
            // a on the compute stream; b on the copy stream once a is in (the
            // two copies share the link), while a's column pass runs
            CU(cudaMemcpyAsync(da, a, an * 8, cudaMemcpyHostToDevice, S));
            if (!sq) {
                CU(cudaEventRecord(X->ev_copy[0], S));
                CU(cudaStreamWaitEvent(C, X->ev_copy[0], 0));
                CU(cudaMemcpyAsync(db, b, bn * 8, cudaMemcpyHostToDevice, C));
                CU(cudaEventRecord(X->ev_copy[1], C));
                b_ready = X->ev_copy[1];
            }
        }
        // the result comes back in chunks on the download stream, each as
        // soon as its CRT launch has finished
        struct Back { Ctx *X; cudaStream_t down; uint64_t *z, *dz; uint64_t lo; int k; int rc; } bk{
            X, down, z, dz, lo, 0, 0};
        CrtChunks ch;
        ch.chunks = lo == 0 ? 4 : 1;
        ch.arg = &bk;
        ch.hook = [](void *p, uint64_t l0, uint64_t l1) {
            Back &B = *(Back *)p;
            if (B.rc || l1 <= l0) return;
            cudaEvent_t e = B.X->ev_copy[2 + (B.k++ % 7)];
            if (cudaEventRecord(e, B.X->stream) != cudaSuccess || cudaStreamWaitEvent(B.down, e, 0) != cudaSuccess ||
                cudaMemcpyAsync(B.z + (l0 - B.lo), B.dz + (l0 - B.lo), (l1 - l0) * 8, cudaMemcpyDeviceToHost,
                                B.down) != cudaSuccess)
                B.rc = set_error(GPU_FFT_SMALL_ECUDA, "result copy");
        };
        rc = mpn_mul_enqueue(X, dz, da, an, db, bn, S, nullptr, lo, top, b_ready, &ch);
        if (!rc) rc = bk.rc;
        // the error flag follows the result home (pinned word: no staging copy
        // that would queue behind other products' transfers)
        if (!rc && cudaMemcpyAsync(X->h_err, X->d_err, sizeof(int), cudaMemcpyDeviceToHost, down) != cudaSuccess)
            rc = set_error(GPU_FFT_SMALL_ECUDA, "error flag copy");
        if (!rc && links && cudaEventRecord(links->done, down) != cudaSuccess)
            rc = set_error(GPU_FFT_SMALL_ECUDA, "cudaEventRecord");
        if (rc) {
            if (links) cudaStreamSynchronize(links->up);
            cudaStreamSynchronize(S);
            cudaStreamSynchronize(down);
            return rc;
        }
    }
    return 0;
}

// The second half of a host-pointer product (same arguments as the issue):
// the download is the last work queued on the copy stream, after the
// kernels on the compute stream.
static int mpn_mul_host_finish(Ctx *X, gpu_ulong *z, gpu_ulong an, gpu_ulong bn, gpu_ulong lo, gpu_ulong hi,
                               const HostLinks *links = nullptr)
{
    int rc = 0;
    if (links) CU(cudaEventSynchronize(links->done));
    else if (X->copy_stream) CU(cudaStreamSynchronize(X->copy_stream));
    if (an + bn > lo && std::min<gpu_ulong>(hi, an + bn) > lo) {
        // the flag was copied behind the last download
        if (*X->h_err) {
            *X->h_err = 0;
            cudaMemsetAsync(X->d_err, 0, sizeof(int), X->stream);
            return set_error(GPU_FFT_SMALL_ETIMEOUT, "carry look-back wait exceeded its limit");
        }
    } else {
        rc = check_device_error(X);
        if (rc) return rc;
    }
    const gpu_ulong zn = an + bn;
    if (hi > zn) memset(z + (zn > lo ? zn - lo : 0), 0, (hi - std::max<gpu_ulong>(zn, lo)) * 8);
    return 0;
}

static int mpn_mul_host(Ctx *X, gpu_ulong *z, const gpu_ulong *a, gpu_ulong an,
                        const gpu_ulong *b, gpu_ulong bn, gpu_ulong lo, gpu_ulong hi)
{
    int rc = mpn_mul_host_issue(X, z, a, an, b, bn, lo, hi);
    if (rc) return rc;
    return mpn_mul_host_finish(X, z, an, bn, lo, hi);
}

// ---------------------------------------------------------------------------
// Pipelines of host-pointer products: a ring of `depth` contexts (slots),
// each with its own scratch and kernel stream, takes products in turn, so
// that one product's download, the next one's upload and a third one's
// kernels run at the same time (PCIe is full duplex; copies and kernels use
// different engines).  All uploads go through one stream and all downloads
// through another (HostLinks): each direction carries one product at a
// time, in submission order, at the full rate of the link, instead of
// several products' copies sharing it and all finishing late.  A submission
// to a busy slot first completes the product that slot holds (so its device
// buffers are free before the next upload into them is queued); the status
// of a completed product is kept until its ticket is waited for (once).
struct Pipe {
    std::vector<Ctx *> slot;
    cudaStream_t up = nullptr, down = nullptr;
    std::vector<HostLinks> links;         // per slot: the shared streams and its events
    std::vector<long long> cur;           // ticket in flight on the slot (-1: none)
    std::unordered_map<long long, int> finished;   // completed, not yet waited: status
    struct Pending { gpu_ulong *z; gpu_ulong an, bn; };
    std::vector<Pending> pend;
    long long next = 0;
};

static int pipe_complete(Pipe *P, int s)
{
    if (P->cur[s] < 0) return 0;
    Ctx *X = P->slot[s];
    const Pipe::Pending &q = P->pend[s];
    int rc = bind_device(X);
    if (!rc) rc = mpn_mul_host_finish(X, q.z, q.an, q.bn, 0, q.an + q.bn, &P->links[s]);
    P->finished[P->cur[s]] = rc;
    P->cur[s] = -1;
    return rc;
}

static void pipe_free(Pipe *P)
{
    for (Ctx *X : P->slot) ctx_destroy(X);
    for (HostLinks &L : P->links)
        for (cudaEvent_t e : {L.a_in, L.b_in, L.done})
            if (e) cudaEventDestroy(e);
    if (P->up) cudaStreamDestroy(P->up);
    if (P->down) cudaStreamDestroy(P->down);
    delete P;
}

// ---------------------------------------------------------------------------
// nmod polynomials
#include "nmod_host.inc"

// ---------------------------------------------------------------------------
// batches of uneven products
#include "batch_host.inc"

// ---------------------------------------------------------------------------
// integer polynomials
#include "fmpz_host.inc"

// ---------------------------------------------------------------------------
// cost model of the learned schedule
#include "mlp_host.inc"

// ---------------------------------------------------------------------------
// plans and transformed operands
#include "op_host.inc"

// ---------------------------------------------------------------------------
// precomputed transforms for nmod products and division
#include "precomp_host.inc"

// ---------------------------------------------------------------------------
// negacyclic products mod 2^N + 1
#include "neg_host.inc"

// ---------------------------------------------------------------------------
// C ABI
extern "C" {

int gpu_mpn_ctx_init_status(gpu_mpn_ctx_t R, gpu_ulong p)
{
    R->impl = nullptr;
    Ctx *X = nullptr;
    int rc = ctx_create(&X, p);
    if (rc) return rc;
    R->impl = X;
    return 0;
}

void gpu_mpn_ctx_init(gpu_mpn_ctx_t R, gpu_ulong p)
{
    int rc = gpu_mpn_ctx_init_status(R, p);
    if (rc) raise_error(rc);
}

void gpu_mpn_ctx_clear(gpu_mpn_ctx_t R)
{
    ctx_destroy(get_ctx(R));
    R->impl = nullptr;
}

int gpu_mpn_ctx_mpn_mul_status(gpu_mpn_ctx_t R, gpu_ulong *z, const gpu_ulong *a, gpu_ulong an,
                               const gpu_ulong *b, gpu_ulong bn)
{
    return mpn_mul_host(get_ctx(R), z, a, an, b, bn, 0, an + bn);
}

void gpu_mpn_ctx_mpn_mul(gpu_mpn_ctx_t R, gpu_ulong *z, const gpu_ulong *a, gpu_ulong an,
                         const gpu_ulong *b, gpu_ulong bn)
{
    int rc = gpu_mpn_ctx_mpn_mul_status(R, z, a, an, b, bn);
    if (rc) raise_error(rc);
}

int gpu_mpn_pipe_init(gpu_mpn_pipe_t R, int depth)
{
    R->impl = nullptr;
    if (depth < 1 || depth > GPU_MPN_PIPE_MAX_DEPTH)
        return set_error(GPU_FFT_SMALL_EINVAL, "pipeline depth %d outside 1..%d", depth, GPU_MPN_PIPE_MAX_DEPTH);
    Pipe *P = new Pipe;
    int rc = 0;
    for (int s = 0; s < depth && !rc; s++) {
        Ctx *X = nullptr;
        rc = ctx_create(&X, 0);
        if (!rc) rc = ensure_copy_stream(X);
        if (X) P->slot.push_back(X);
    }
    if (!rc && (cudaStreamCreateWithFlags(&P->up, cudaStreamNonBlocking) != cudaSuccess ||
                cudaStreamCreateWithFlags(&P->down, cudaStreamNonBlocking) != cudaSuccess))
        rc = set_error(GPU_FFT_SMALL_ECUDA, "cudaStreamCreate failed");
    for (int s = 0; s < depth && !rc; s++) {
        HostLinks L{P->up, P->down, nullptr, nullptr, nullptr};
        if (cudaEventCreateWithFlags(&L.a_in, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&L.b_in, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&L.done, cudaEventDisableTiming) != cudaSuccess)
            rc = set_error(GPU_FFT_SMALL_ECUDA, "cudaEventCreate failed");
        P->links.push_back(L);
    }
    if (rc) {
        pipe_free(P);
        return rc;
    }
    P->cur.assign(depth, -1);
    P->pend.assign(depth, Pipe::Pending{nullptr, 0, 0});
    R->impl = P;
    return 0;
}

int gpu_mpn_pipe_submit(gpu_mpn_pipe_t R, gpu_ulong *z, const gpu_ulong *a, gpu_ulong an,
                        const gpu_ulong *b, gpu_ulong bn, long long *ticket)
{
    Pipe *P = (Pipe *)R->impl;
    if (!P || !ticket) return set_error(GPU_FFT_SMALL_EINVAL, "pipeline not initialised");
    if (an == 0 || bn == 0) return set_error(GPU_FFT_SMALL_EINVAL, "empty operand");
    const int s = (int)(P->next % (long long)P->slot.size());
    pipe_complete(P, s);   // its status stays with its own ticket
    int rc = mpn_mul_host_issue(P->slot[s], z, a, an, b, bn, 0, an + bn, &P->links[s]);
    if (rc) return rc;
    P->cur[s] = P->next;
    P->pend[s] = Pipe::Pending{z, an, bn};
    *ticket = P->next++;
    return 0;
}

int gpu_mpn_pipe_wait(gpu_mpn_pipe_t R, long long ticket)
{
    Pipe *P = (Pipe *)R->impl;
    if (!P) return set_error(GPU_FFT_SMALL_EINVAL, "pipeline not initialised");
    if (ticket < 0 || ticket >= P->next) return set_error(GPU_FFT_SMALL_EINVAL, "unknown ticket %lld", ticket);
    const int s = (int)(ticket % (long long)P->slot.size());
    if (P->cur[s] == ticket) pipe_complete(P, s);
    auto it = P->finished.find(ticket);
    if (it == P->finished.end()) return set_error(GPU_FFT_SMALL_EINVAL, "ticket %lld already waited for", ticket);
    const int rc = it->second;
    P->finished.erase(it);
    return rc;
}

void gpu_mpn_pipe_clear(gpu_mpn_pipe_t R)
{
    Pipe *P = (Pipe *)R->impl;
    if (!P) return;
    for (size_t s = 0; s < P->slot.size(); s++) pipe_complete(P, (int)s);
    pipe_free(P);
    R->impl = nullptr;
}

void _gpu_mpn_ctx_mpn_mul_range(gpu_mpn_ctx_t R, gpu_ulong *z, gpu_ulong lo, gpu_ulong hi,
                                const gpu_ulong *a, gpu_ulong an, const gpu_ulong *b, gpu_ulong bn)
{
    if (lo >= hi) return;
    int rc = mpn_mul_host(get_ctx(R), z, a, an, b, bn, lo, hi);
    if (rc) raise_error(rc);
}

int gpu_mpn_mul_device(gpu_mpn_ctx_t R, uint64_t *z_dev, const uint64_t *a_dev, gpu_ulong an,
                       const uint64_t *b_dev, gpu_ulong bn, void *stream)
{
    Ctx *X = get_ctx(R);
    if (!X) return set_error(GPU_FFT_SMALL_EINVAL, "context not initialised");
    int rc = bind_device(X);
    if (rc) return rc;
    // NULL is CUDA's default stream, as everywhere in the runtime API
    return mpn_mul_enqueue(X, z_dev, a_dev, an, b_dev, bn, (cudaStream_t)stream);
}

// Scratch a whole product needs on the device (residue bytes, CRT tiles),
// following mpn_mul_enqueue's plan: split products hold the full residue
// array plus a chunk pair, the basecase route three 64-bit planes.
static int mpn_mul_scratch_need(uint64_t an, uint64_t bn, const gpu_mul_config *cfg, bool sq,
                                size_t *bytes, size_t *tiles)
{
    MulPlan P;
    int Lover = 0;
    int rc = plan_mpn_cfg(an, bn, cfg, &P);
    if (rc == GPU_FFT_SMALL_ETOOBIG && !cfg && !sq) rc = plan_mpn_oversize(an, bn, &P, &Lover);
    if (rc) return rc;
    const uint64_t zn = an + bn;
    if (P.route == GPU_MUL_ROUTE_BASECASE) {
        *bytes = 3 * ((size_t)1 << P.logM) * sizeof(uint64_t);
        *tiles = (zn + 1023) / 1024;
        return 0;
    }
    const size_t M = (size_t)1 << P.logM;
    const int Lc = Lover ? Lover : (!cfg && !sq) ? split_plan(an, bn, P.logM) : 0;
    const size_t Mc = Lc ? (size_t)1 << Lc : 0;
    *bytes = Lc ? (size_t)P.np * (M + 2 * Mc) * sizeof(uint32_t) : (sq ? 1 : 2) * (size_t)P.np * M * sizeof(uint32_t);
    *tiles = (zn + CRT_TILE - 1) / CRT_TILE;
    return 0;
}

int gpu_mpn_mul_device_list(gpu_mpn_ctx_t R, const gpu_mpn_mul_req *reqs, size_t n,
                            const gpu_mul_config *cfgs, void *stream)
{
    Ctx *X = get_ctx(R);
    if (!X) return set_error(GPU_FFT_SMALL_EINVAL, "context not initialised");
    if (n && !reqs) return set_error(GPU_FFT_SMALL_EINVAL, "null request list");
    size_t bytes = 0, tiles = 0;
    for (size_t i = 0; i < n; i++) {
        const gpu_mpn_mul_req &q = reqs[i];
        size_t b = 0, t = 0;
        int rc = (!q.z || !q.a || !q.b || q.an == 0 || q.bn == 0)
                     ? set_error(GPU_FFT_SMALL_EINVAL, "null pointer or empty operand")
                     : mpn_mul_scratch_need(q.an, q.bn, cfgs ? &cfgs[i] : nullptr, q.a == q.b && q.an == q.bn,
                                            &b, &t);
        if (rc) {
            const std::string msg = g_last_error;
            return set_error(rc, "request %zu: %s", i, msg.c_str());
        }
        bytes = std::max(bytes, b);
        tiles = std::max(tiles, t);
    }
    int rc = bind_device(X);
    if (!rc) rc = grow((void **)&X->d_res, &X->res_cap, bytes);
    if (!rc) rc = ensure_status(X, tiles);
    for (size_t i = 0; i < n && !rc; i++) {
        const gpu_mpn_mul_req &q = reqs[i];
        rc = mpn_mul_enqueue(X, q.z, q.a, q.an, q.b, q.bn, (cudaStream_t)stream, cfgs ? &cfgs[i] : nullptr);
    }
    return rc;
}

int gpu_mpn_mul_config_resolve(gpu_ulong an, gpu_ulong bn, gpu_mul_config *cfg)
{
    if (!cfg) return set_error(GPU_FFT_SMALL_EINVAL, "null configuration");
    MulPlan P;
    int rc = plan_mpn_cfg(an, bn, cfg, &P);
    if (rc) return rc;
    if (P.route == GPU_MUL_ROUTE_NTT) {
        cfg->np = P.np;
        cfg->logM = P.logM;
        cfg->logC = (cfg->flags & GPU_MUL_FLAG_THREE) ? LOGC3 : P.L.S.logC;
    }
    return 0;
}

// The reference's profile choice (mpn_ctx_best_profile, src/fft_small/
// mpn_mul.c:1248-1340) in this library's configuration space: among single
// transforms with the longest rows -- the fewest primes or one more, the
// shortest power-of-two length or, where the product fits it, the 3 2^k
// length (the counterpart of its truncated ztrunc) -- the least score
// (1 - ratio / 4) np depth L_t, with L_t the transform's points,
// depth = ceil(log2 L_t) and ratio = L_t / 2^depth (ties to fewer primes).
// The reference scores its own profiles (50-bit primes, chunk bit sizes,
// 256-point truncation); the formula is the same.
int gpu_mul_reference_rule(int kind, gpu_ulong an, gpu_ulong aw, gpu_ulong bn, gpu_ulong bw,
                           gpu_mul_config *cfg)
{
    if (!cfg) return set_error(GPU_FFT_SMALL_EINVAL, "null configuration");
    gpu_mul_config best{0, 0, 0, 0, 0};
    double best_score = -1.0;
    int rc = 0;
    for (int dnp = 0; dnp <= 1; dnp++)
        for (int fl = 0; fl <= GPU_MUL_FLAG_THREE; fl += GPU_MUL_FLAG_THREE) {
            gpu_mul_config c{GPU_MUL_ROUTE_NTT, 0, 0, 0, fl};
            rc = kind == 0 ? gpu_mpn_mul_config_resolve(an, bn, &c)
                           : gpu_fmpz_poly_mul_config_resolve(an, aw, bn, bw, &c);
            if (rc) continue;
            if (dnp) {
                c.np += 1;
                c.logC = 0;
                rc = kind == 0 ? gpu_mpn_mul_config_resolve(an, bn, &c)
                               : gpu_fmpz_poly_mul_config_resolve(an, aw, bn, bw, &c);
                if (rc) continue;
            }
            const double lt = fl ? 3.0 * ldexp(1.0, c.logM - 2) : ldexp(1.0, c.logM);
            const int depth = (int)ceil(log2(lt) - 1e-9);
            const double score = (1.0 - 0.25 * lt / ldexp(1.0, depth)) * c.np * depth * lt;
            if (best_score < 0 || score < best_score) {
                best = c;
                best_score = score;
            }
        }
    if (best_score < 0) return rc ? rc : set_error(GPU_FFT_SMALL_EINVAL, "no transform configuration");
    *cfg = best;
    return 0;
}

int gpu_mpn_mul_device_config(gpu_mpn_ctx_t R, uint64_t *z_dev, const uint64_t *a_dev, gpu_ulong an,
                              const uint64_t *b_dev, gpu_ulong bn, const gpu_mul_config *cfg,
                              void *stream)
{
    Ctx *X = get_ctx(R);
    if (!X) return set_error(GPU_FFT_SMALL_EINVAL, "context not initialised");
    int rc = bind_device(X);
    if (rc) return rc;
    return mpn_mul_enqueue(X, z_dev, a_dev, an, b_dev, bn, (cudaStream_t)stream, cfg);
}

int gpu_mpn_mul_range_device(gpu_mpn_ctx_t R, uint64_t *z_dev, gpu_ulong lo, gpu_ulong hi,
                             const uint64_t *a_dev, gpu_ulong an, const uint64_t *b_dev, gpu_ulong bn,
                             void *stream)
{
    Ctx *X = get_ctx(R);
    if (!X) return set_error(GPU_FFT_SMALL_EINVAL, "context not initialised");
    if (an == 0 || bn == 0) return set_error(GPU_FFT_SMALL_EINVAL, "empty operand");
    int rc = bind_device(X);
    if (rc) return rc;
    return mpn_mul_enqueue(X, z_dev, a_dev, an, b_dev, bn, (cudaStream_t)stream, nullptr, lo, hi);
}

void gpu_mpn_mulmid_default_mpn_ctx(gpu_ulong *z, const gpu_ulong *a, gpu_slong an, const gpu_ulong *b,
                                    gpu_slong bn, gpu_slong zlo, gpu_slong zhi)
{
    _gpu_mpn_ctx_mpn_mul_range(gpu_get_default_mpn_ctx(), z, (gpu_ulong)zlo, (gpu_ulong)zhi, a,
                               (gpu_ulong)an, b, (gpu_ulong)bn);
}

int _gpu_nmod_poly_mul_mid_status(gpu_ulong *z, gpu_ulong zl, gpu_ulong zh,
                                  const gpu_ulong *a, gpu_ulong an, const gpu_ulong *b, gpu_ulong bn,
                                  gpu_nmod_t mod, gpu_mpn_ctx_t R)
{
    return nmod_mul_mid_host(get_ctx(R), z, zl, zh, a, an, b, bn, mod.n);
}

int gpu_nmod_poly_mul_mid_device(gpu_mpn_ctx_t R, uint64_t *z_dev, gpu_ulong zl, gpu_ulong zh,
                                 const uint64_t *a_dev, gpu_ulong an, const uint64_t *b_dev, gpu_ulong bn,
                                 gpu_nmod_t mod, void *stream)
{
    Ctx *X = get_ctx(R);
    if (!X) return set_error(GPU_FFT_SMALL_EINVAL, "context not initialised");
    if (an == 0 || bn == 0) return set_error(GPU_FFT_SMALL_EINVAL, "empty operand");
    if (mod.n == 0) return set_error(GPU_FFT_SMALL_EINVAL, "modulus must be nonzero");
    if (zl >= zh) return 0;
    int rc = bind_device(X);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const gpu_ulong zn = an + bn - 1;
    // coefficients at or beyond the product's length are zero, as is
    // everything mod 1
    const gpu_ulong top = mod.n == 1 ? zl : std::min<gpu_ulong>(zh, std::max<gpu_ulong>(zn, zl));
    if (zh > top) CU(cudaMemsetAsync(z_dev + (top - zl), 0, (zh - top) * 8, st));
    if (top > zl) rc = nmod_mul_mid_enqueue(X, z_dev, zl, top, a_dev, an, b_dev, bn, mod.n, st);
    return rc;
}

int _gpu_nmod_poly_divrem_status(gpu_ulong *q, gpu_ulong *r, const gpu_ulong *a, gpu_ulong an,
                                 const gpu_ulong *b, gpu_ulong bn, gpu_nmod_t mod, gpu_mpn_ctx_t R)
{
    return nmod_divrem_host(get_ctx(R), q, r, a, an, b, bn, mod.n);
}

void _gpu_nmod_poly_divrem_mpn_ctx(gpu_ulong *q, gpu_ulong *r, const gpu_ulong *a, gpu_ulong an,
                                   const gpu_ulong *b, gpu_ulong bn, gpu_nmod_t mod, gpu_mpn_ctx_t R)
{
    int rc = _gpu_nmod_poly_divrem_status(q, r, a, an, b, bn, mod, R);
    if (rc) raise_error(rc);
}

void _gpu_nmod_poly_mul_mid_mpn_ctx(gpu_ulong *z, gpu_ulong zl, gpu_ulong zh,
                                    const gpu_ulong *a, gpu_ulong an, const gpu_ulong *b, gpu_ulong bn,
                                    gpu_nmod_t mod, gpu_mpn_ctx_t R)
{
    int rc = _gpu_nmod_poly_mul_mid_status(z, zl, zh, a, an, b, bn, mod, R);
    if (rc) raise_error(rc);
}

static thread_local gpu_mpn_ctx_struct g_default_ctx = {nullptr};

gpu_mpn_ctx_struct *gpu_get_default_mpn_ctx(void)
{
    // same starting prime as the reference's DEFAULT_PRIME
    if (!g_default_ctx.impl) gpu_mpn_ctx_init(&g_default_ctx, 0x0003f00000000001ull);
    return &g_default_ctx;
}

// the calling thread's default context is released here, as the cleanup
// hook mpn_ctx_cleanup (src/fft_small/default_ctx.c:19-27) does under
// flint_cleanup; a later use creates a new one
void gpu_default_mpn_ctx_cleanup(void)
{
    if (g_default_ctx.impl) gpu_mpn_ctx_clear(&g_default_ctx);
    g_default_ctx.impl = nullptr;
}

void gpu_mpn_mul_default_mpn_ctx(gpu_ulong *r1, const gpu_ulong *i1, gpu_slong n1,
                                 const gpu_ulong *i2, gpu_slong n2)
{
    gpu_mpn_ctx_mpn_mul(gpu_get_default_mpn_ctx(), r1, i1, (gpu_ulong)n1, i2, (gpu_ulong)n2);
}

void _gpu_nmod_poly_mul_mid_default_mpn_ctx(gpu_ulong *res, gpu_slong zl, gpu_slong zh,
                                            const gpu_ulong *a, gpu_slong an,
                                            const gpu_ulong *b, gpu_slong bn, gpu_nmod_t mod)
{
    _gpu_nmod_poly_mul_mid_mpn_ctx(res, (gpu_ulong)zl, (gpu_ulong)zh, a, (gpu_ulong)an, b,
                                   (gpu_ulong)bn, mod, gpu_get_default_mpn_ctx());
}

int _gpu_fmpz_poly_mul_mid_raw(gpu_ulong *z, gpu_ulong zw, gpu_ulong zl, gpu_ulong zh,
                               const gpu_ulong *a, gpu_ulong aw, gpu_ulong an,
                               const gpu_ulong *b, gpu_ulong bw, gpu_ulong bn, gpu_mpn_ctx_t R)
{
    return fmpz_mul_mid_host(get_ctx(R), z, zw, zl, zh, a, aw, an, b, bw, bn);
}

int gpu_fmpz_poly_mul_mid_device(gpu_mpn_ctx_t R, uint64_t *z_dev, gpu_ulong zw, gpu_ulong zl,
                                 gpu_ulong zh, const uint64_t *a_dev, gpu_ulong aw, gpu_ulong an,
                                 const uint64_t *b_dev, gpu_ulong bw, gpu_ulong bn, void *stream)
{
    Ctx *X = get_ctx(R);
    if (!X) return set_error(GPU_FFT_SMALL_EINVAL, "context not initialised");
    int rc = fmpz_check_args(zw, aw, an, bw, bn);
    if (rc) return rc;
    if (zl >= zh) return 0;
    rc = bind_device(X);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const gpu_ulong zn = an + bn - 1;
    if (zh > zn) {
        const gpu_ulong from = std::max(zl, zn);
        CU(cudaMemsetAsync(z_dev + (from - zl) * zw, 0, (zh - from) * zw * 8, st));
        if (zl >= zn) return 0;
        zh = zn;
    }
    return fmpz_mul_mid_enqueue(X, z_dev, zw, zl, zh, a_dev, aw, an, b_dev, bw, bn, st);
}

int gpu_fmpz_poly_mul_config_resolve(gpu_ulong an, gpu_ulong aw, gpu_ulong bn, gpu_ulong bw,
                                     gpu_mul_config *cfg)
{
    if (!cfg) return set_error(GPU_FFT_SMALL_EINVAL, "null configuration");
    FmpzPlan P;
    int rc = plan_fmpz_cfg(an, aw, bn, bw, cfg, &P);
    if (rc) return rc;
    cfg->np = P.np;
    cfg->logM = P.logM;
    cfg->logC = P.k3 ? LOGC3 : P.L.S.logC;
    return 0;
}

int gpu_fmpz_poly_mul_mid_device_list(gpu_mpn_ctx_t R, const gpu_fmpz_mul_req *reqs, size_t n,
                                      const gpu_mul_config *cfgs, void *stream)
{
    Ctx *X = get_ctx(R);
    if (!X) return set_error(GPU_FFT_SMALL_EINVAL, "context not initialised");
    if (n && !reqs) return set_error(GPU_FFT_SMALL_EINVAL, "null request list");
    size_t need = 0;
    for (size_t i = 0; i < n; i++) {
        const gpu_fmpz_mul_req &q = reqs[i];
        int rc = fmpz_check_args(q.zw, q.aw, q.an, q.bw, q.bn);
        if (!rc && (q.zl >= q.zh || q.zh > q.an + q.bn - 1))
            rc = set_error(GPU_FFT_SMALL_EINVAL, "window must lie inside the product");
        FmpzPlan P;
        if (!rc) rc = plan_fmpz_cfg(q.an, q.aw, q.bn, q.bw, cfgs ? &cfgs[i] : nullptr, &P);
        if (rc) {
            const std::string msg = g_last_error;
            return set_error(rc, "request %zu: %s", i, msg.c_str());
        }
        const bool sq = (q.a == q.b) && (q.an == q.bn) && (q.aw == q.bw);
        need = std::max(need, (sq ? 1 : 2) * (size_t)P.np * ((size_t)1 << P.logM) * sizeof(uint32_t));
    }
    int rc = bind_device(X);
    if (rc) return rc;
    rc = grow((void **)&X->d_res, &X->res_cap, need);
    if (rc) return rc;
    for (size_t i = 0; i < n; i++) {
        const gpu_fmpz_mul_req &q = reqs[i];
        rc = fmpz_mul_mid_enqueue(X, q.z, q.zw, q.zl, q.zh, q.a, q.aw, q.an, q.b, q.bw, q.bn,
                                  (cudaStream_t)stream, cfgs ? &cfgs[i] : nullptr);
        if (rc) return rc;
    }
    return 0;
}

int gpu_fmpz_poly_mul_mid_device_config(gpu_mpn_ctx_t R, uint64_t *z_dev, gpu_ulong zw, gpu_ulong zl,
                                        gpu_ulong zh, const uint64_t *a_dev, gpu_ulong aw, gpu_ulong an,
                                        const uint64_t *b_dev, gpu_ulong bw, gpu_ulong bn,
                                        const gpu_mul_config *cfg, void *stream)
{
    Ctx *X = get_ctx(R);
    if (!X) return set_error(GPU_FFT_SMALL_EINVAL, "context not initialised");
    int rc = fmpz_check_args(zw, aw, an, bw, bn);
    if (rc) return rc;
    if (zl >= zh || zh > an + bn - 1)
        return set_error(GPU_FFT_SMALL_EINVAL, "window must lie inside the product");
    rc = bind_device(X);
    if (rc) return rc;
    return fmpz_mul_mid_enqueue(X, z_dev, zw, zl, zh, a_dev, aw, an, b_dev, bw, bn, (cudaStream_t)stream,
                                cfg);
}

// device-side operand filler for the timing entry point (splitmix64)
__global__ void k_fill_limbs(uint64_t *p, uint64_t n, uint64_t seed)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        p[i] = (z ^ (z >> 31)) | (i + 1 == n ? 1ull : 0ull);
    }
}

int gpu_test_crt_lookback_timeout(gpu_mpn_ctx_t R)
{
    Ctx *X = get_ctx(R);
    if (!X) return set_error(GPU_FFT_SMALL_EINVAL, "context not initialised");
    int rc = bind_device(X);
    if (rc) return rc;
    // one tile of a 1024-coefficient product whose ticket makes it tile 1:
    // its look-back waits on tile 0's status word, which nothing publishes in
    // this epoch, until the spin limit; every access stays inside the
    // 5 x 1024 residues, the 1024-limb output and the two status words
    constexpr int logM = 10;
    const size_t M = (size_t)1 << logM;
    rc = grow((void **)&X->d_res, &X->res_cap, 5 * M * sizeof(uint32_t));
    if (!rc) rc = ensure_status(X, 2);
    uint64_t *dz = nullptr;
    if (!rc) rc = io_buffers(X, M, &dz);
    if (rc) return rc;
    cudaStream_t st = X->stream;
    CU(cudaMemsetAsync(X->d_res, 0, 5 * M * sizeof(uint32_t), st));
    X->epoch = (X->epoch + 1) & 0x0fffffffu;
    if (X->epoch == 0) {
        CU(cudaMemsetAsync(X->d_status, 0, X->status_cap * sizeof(uint32_t), st));
        X->epoch = 1;
    }
    k_crt_carry<5, CRT_THREADS><<<1, CRT_THREADS, 0, st>>>(X->d_res, logM, M - 1, M, dz, X->crt[5], X->d_status,
                                                          X->d_ticket, X->ticket_base - 1, X->epoch, X->d_err,
                                                          nullptr, nullptr, 0ull);
    CU(cudaGetLastError());
    X->ticket_base += 1;
    return check_device_error(X);
}

void *gpu_test_pipe_slot_ctx(gpu_mpn_pipe_t R, int slot)
{
    Pipe *P = (Pipe *)R->impl;
    if (!P || slot < 0 || slot >= (int)P->slot.size()) return nullptr;
    return P->slot[slot];
}

int gpu_test_set_device_error(gpu_mpn_ctx_t R)
{
    Ctx *X = get_ctx(R);
    if (!X) return set_error(GPU_FFT_SMALL_EINVAL, "context not initialised");
    int rc = bind_device(X);
    if (rc) return rc;
    CU(cudaMemsetAsync(X->d_err, 1, sizeof(int), X->stream));
    CU(cudaStreamSynchronize(X->stream));
    return 0;
}

int gpu_butterfly_rate(gpu_mpn_ctx_t R, double *per_s)
{
    Ctx *X = get_ctx(R);
    if (!X || !per_s) return set_error(GPU_FFT_SMALL_EINVAL, "context not initialised");
    int rc = bind_device(X);
    if (rc) return rc;
    const int blocks = X->nsm * 8, threads = 256;
    uint32_t *buf = nullptr;
    CU(cudaMalloc(&buf, (size_t)blocks * threads * 16 * sizeof(uint32_t)));
    cudaStream_t st = X->stream;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    std::vector<float> t(5);
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
        rc = set_error(GPU_FFT_SMALL_ECUDA, "cudaEventCreate");
    k_bfly_rate<<<blocks, threads, 0, st>>>(buf, X->T.twf, PRIMES[0], 17u);   // warm-up
    for (int r = 0; r < (int)t.size() && !rc; r++) {
        cudaEventRecord(e0, st);
        k_bfly_rate<<<blocks, threads, 0, st>>>(buf, X->T.twf, PRIMES[0], 19u + r);
        cudaEventRecord(e1, st);
        if (cudaEventSynchronize(e1) != cudaSuccess) rc = set_error(GPU_FFT_SMALL_ECUDA, "calibration sync");
        else cudaEventElapsedTime(&t[r], e0, e1);
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaStreamSynchronize(st);
    cudaFree(buf);
    if (rc) return rc;
    std::sort(t.begin(), t.end());
    // butterflies per launch: every thread runs CAL_ITERS x 4 levels x 8
    const double bfly = (double)blocks * threads * CAL_ITERS * 4 * 8;
    *per_s = bfly / (t[t.size() / 2] * 1e-3);
    return 0;
}

int gpu_mul_time_config(gpu_mpn_ctx_t R, int kind, gpu_ulong an, gpu_ulong aw, gpu_ulong bn, gpu_ulong bw,
                        const gpu_mul_config *cfg, int reps, double *ms)
{
    Ctx *X = get_ctx(R);
    if (!X) return set_error(GPU_FFT_SMALL_EINVAL, "context not initialised");
    if (reps < 1 || !ms || (kind != 0 && kind != 1)) return set_error(GPU_FFT_SMALL_EINVAL, "bad timing request");
    if (kind == 0) aw = bw = 1;
    int rc = bind_device(X);
    if (rc) return rc;
    // validate the configuration before allocating
    gpu_mul_config c = cfg ? *cfg : gpu_mul_config{0, 0, 0, 0};
    rc = kind == 0 ? gpu_mpn_mul_config_resolve(an, bn, &c) : gpu_fmpz_poly_mul_config_resolve(an, aw, bn, bw, &c);
    if (rc) return rc;
    const uint64_t zn = an + bn, zw = kind == 0 ? 1 : aw + bw + 1;
    const size_t na = an * aw, nb = bn * bw, nz = zn * zw;
    uint64_t *buf = nullptr;
    rc = timing_scratch(X, (na + nb + nz) * sizeof(uint64_t), &buf);
    if (rc) return rc;
    uint64_t *da = buf, *db = buf + na, *dz = buf + na + nb;
    cudaStream_t st = X->stream;
    k_fill_limbs<<<X->nsm * 4, 256, 0, st>>>(da, na, 0x1234567ull + an);
    k_fill_limbs<<<X->nsm * 4, 256, 0, st>>>(db, nb, 0x7654321ull + bn);
    auto call = [&]() -> int {
        return kind == 0 ? mpn_mul_enqueue(X, dz, da, an, db, bn, st, cfg)
                         : fmpz_mul_mid_enqueue(X, dz, zw, 0, an + bn - 1, da, aw, an, db, bw, bn, st, cfg);
    };
    std::vector<float> t(reps);
    cudaEvent_t e0 = X->ev_time[0], e1 = X->ev_time[1];
    rc = call();   // warm-up (allocations, first launch)
    for (int r = 0; r < reps && !rc; r++) {
        cudaEventRecord(e0, st);
        rc = call();
        cudaEventRecord(e1, st);
        if (!rc && cudaEventSynchronize(e1) != cudaSuccess) rc = set_error(GPU_FFT_SMALL_ECUDA, "timing sync");
        if (!rc) cudaEventElapsedTime(&t[r], e0, e1);
    }
    if (!rc) rc = check_device_error(X);
    cudaStreamSynchronize(st);
    if (rc) return rc;
    std::sort(t.begin(), t.end());
    *ms = t[reps / 2];
    return 0;
}

int gpu_mpn_mul_time_batched(gpu_mpn_ctx_t R, gpu_ulong an, gpu_ulong bn, const gpu_mul_config *cfg,
                             int copies, int reps, double *ms_per_product)
{
    Ctx *X = get_ctx(R);
    if (!X) return set_error(GPU_FFT_SMALL_EINVAL, "context not initialised");
    if (reps < 1 || copies < 1 || !ms_per_product) return set_error(GPU_FFT_SMALL_EINVAL, "bad timing request");
    int rc = bind_device(X);
    if (rc) return rc;
    gpu_mul_config c = cfg ? *cfg : gpu_mul_config{0, 0, 0, 0};
    rc = gpu_mpn_mul_config_resolve(an, bn, &c);
    if (rc) return rc;
    const size_t per = an + bn + (an + bn);
    uint64_t *buf = nullptr;
    rc = timing_scratch(X, per * copies * sizeof(uint64_t), &buf);
    if (rc) return rc;
    cudaStream_t st = X->stream;
    std::vector<gpu_mpn_mul_req> reqs(copies);
    std::vector<gpu_mul_config> cfgs(copies, cfg ? *cfg : gpu_mul_config{0, 0, 0, 0});
    for (int k = 0; k < copies; k++) {
        uint64_t *base = buf + per * k;
        k_fill_limbs<<<X->nsm, 256, 0, st>>>(base, an + bn, 0x9999ull + 77 * k);
        reqs[k] = gpu_mpn_mul_req{base + an + bn, base, an, base + an, bn};
    }
    Batch *B = new Batch();
    B->X = X;
    gpu_mpn_batch_options opt = {0, 4, 1};
    rc = batch_plan(B, reqs.data(), cfgs.data(), copies, &opt);
    std::vector<float> t(reps);
    cudaEvent_t e0 = X->ev_time[0], e1 = X->ev_time[1];
    if (!rc) rc = batch_run(B, st);   // warm-up and graph capture
    for (int r = 0; r < reps && !rc; r++) {
        cudaEventRecord(e0, st);
        rc = batch_run(B, st);
        cudaEventRecord(e1, st);
        if (!rc && cudaEventSynchronize(e1) != cudaSuccess) rc = set_error(GPU_FFT_SMALL_ECUDA, "timing sync");
        if (!rc) cudaEventElapsedTime(&t[r], e0, e1);
    }
    if (!rc) rc = check_device_error(X);
    cudaStreamSynchronize(st);
    batch_destroy(B);
    if (rc) return rc;
    std::sort(t.begin(), t.end());
    *ms_per_product = t[reps / 2] / copies;
    return 0;
}

int _gpu_fmpz_poly_mul_mid_mpn_ctx(gpu_slong *z, gpu_ulong zl, gpu_ulong zh, const gpu_slong *a,
                                   gpu_ulong an, const gpu_slong *b, gpu_ulong bn, gpu_mpn_ctx_t R)
{
    const int rc = fmpz_poly_mul_mid_fmpz(get_ctx(R), z, zl, zh, a, an, b, bn);
    if (rc < 0) {
        raise_error(-rc);
        return 0;
    }
    return rc;
}

int _gpu_fmpz_poly_mul_mid_default_mpn_ctx(gpu_slong *z, gpu_slong zl, gpu_slong zh,
                                           const gpu_slong *a, gpu_slong an, const gpu_slong *b,
                                           gpu_slong bn)
{
    return _gpu_fmpz_poly_mul_mid_mpn_ctx(z, (gpu_ulong)zl, (gpu_ulong)zh, a, (gpu_ulong)an, b,
                                          (gpu_ulong)bn, gpu_get_default_mpn_ctx());
}

void gpu_fmpz_set_signed_hook(void (*set_signed)(gpu_slong *f, const gpu_ulong *limbs, gpu_slong n))
{
    g_fmpz_set_signed = set_signed;
}

struct gpu_mpn_batch_struct {
    Batch *impl;
};

int gpu_mpn_batch_init(gpu_mpn_batch_t *out, gpu_mpn_ctx_t R, const gpu_mpn_mul_req *reqs, size_t n,
                       const gpu_mpn_batch_options *opt)
{
    return gpu_mpn_batch_init_config(out, R, reqs, nullptr, n, opt);
}

int gpu_mpn_batch_init_config(gpu_mpn_batch_t *out, gpu_mpn_ctx_t R, const gpu_mpn_mul_req *reqs,
                              const gpu_mul_config *cfgs, size_t n, const gpu_mpn_batch_options *opt)
{
    if (!out) return set_error(GPU_FFT_SMALL_EINVAL, "null batch handle");
    *out = nullptr;
    Ctx *X = get_ctx(R);
    if (!X) return set_error(GPU_FFT_SMALL_EINVAL, "context not initialised");
    if (n == 0 || !reqs) return set_error(GPU_FFT_SMALL_EINVAL, "empty batch");
    if (opt && (opt->promote_small < 0 || opt->max_streams < 0))
        return set_error(GPU_FFT_SMALL_EINVAL, "negative batch option");
    int rc = bind_device(X);
    if (rc) return rc;
    Batch *B = new Batch();
    B->X = X;
    rc = batch_plan(B, reqs, cfgs, n, opt);
    if (rc) {
        batch_destroy(B);
        return rc;
    }
    *out = new gpu_mpn_batch_struct{B};
    return 0;
}

int gpu_mpn_batch_run(gpu_mpn_batch_t B, void *stream)
{
    if (!B || !B->impl) return set_error(GPU_FFT_SMALL_EINVAL, "batch not initialised");
    return batch_run(B->impl, (cudaStream_t)stream);
}

int gpu_mpn_batch_check(gpu_mpn_batch_t B, void *stream)
{
    if (!B || !B->impl) return set_error(GPU_FFT_SMALL_EINVAL, "batch not initialised");
    Ctx *X = B->impl->X;
    int rc = bind_device(X);
    if (rc) return rc;
    CU(cudaStreamSynchronize((cudaStream_t)stream));
    return check_device_error(X);
}

int gpu_mpn_batch_launches(gpu_mpn_batch_t B)
{
    return (B && B->impl) ? B->impl->launches : 0;
}

int gpu_mpn_batch_classes(gpu_mpn_batch_t B)
{
    return (B && B->impl) ? (int)B->impl->cls.size() : 0;
}

void gpu_mpn_batch_clear(gpu_mpn_batch_t B)
{
    if (!B) return;
    batch_destroy(B->impl);
    delete B;
}

void gpu_fft_small_set_throw(void (*handler)(int code, const char *msg))
{
    g_throw_handler = handler;
}

const char *gpu_fft_small_last_error(void) { return g_last_error.c_str(); }

int gpu_mpn_mul_plan(gpu_ulong an, gpu_ulong bn, int *np, int *logM)
{
    MulPlan P;
    int rc = plan_mpn(an, bn, &P);
    if (rc) return rc;
    *np = P.np;
    *logM = P.logM;
    return 0;
}

int gpu_mpn_mul_split_plan(gpu_ulong an, gpu_ulong bn, int *chunk_logM)
{
    MulPlan P;
    int rc = plan_mpn(an, bn, &P);
    if (rc == GPU_FFT_SMALL_ETOOBIG && an != bn) return plan_mpn_oversize(an, bn, &P, chunk_logM);
    if (rc) return rc;
    *chunk_logM = P.route == GPU_MUL_ROUTE_NTT ? split_plan(an, bn, P.logM) : 0;
    return 0;
}

int gpu_mpn_mul_transform_points(gpu_ulong an, gpu_ulong bn, int square, gpu_ulong *points)
{
    if (!points) return set_error(GPU_FFT_SMALL_EINVAL, "null output");
    MulPlan P;
    int Lover = 0;
    int rc = plan_mpn(an, bn, &P);
    if (rc == GPU_FFT_SMALL_ETOOBIG && !square) rc = plan_mpn_oversize(an, bn, &P, &Lover);
    if (rc) return rc;
    if (P.route != GPU_MUL_ROUTE_NTT) {
        *points = 0;
        return 0;
    }
    const int Lc = Lover ? Lover : square ? 0 : split_plan(an, bn, P.logM);
    if (Lc) {
        *points = (gpu_ulong)1 << Lc;
        return 0;
    }
    const int k3 = three_length(an + bn - 1, P.np, P.logM);
    *points = k3 ? (gpu_ulong)3 << k3 : (gpu_ulong)1 << P.logM;
    return 0;
}

gpu_ulong gpu_fft_small_prime(int i)
{
    return (i >= 0 && i < MAX_NP) ? PRIMES[i] : 0;
}

int gpu_mpn_ctx_last_launches(gpu_mpn_ctx_t R)
{
    Ctx *X = get_ctx(R);
    return X ? X->last_launches : 0;
}

int gpu_mpn_ctx_set_timing(gpu_mpn_ctx_t R, int on)
{
    Ctx *X = get_ctx(R);
    if (!X) return set_error(GPU_FFT_SMALL_EINVAL, "context not initialised");
    timing_drain(X);
    for (int k = 0; k < TIMING_SLOTS; k++) {
        X->kernel_ms[k] = 0;
        X->kernel_count[k] = 0;
    }
    X->timing = on != 0;
    return 0;
}

int gpu_mpn_ctx_kernel_times(gpu_mpn_ctx_t R, double *ms, long *count, int max)
{
    Ctx *X = get_ctx(R);
    if (!X) return 0;
    timing_drain(X);
    const int n = std::min(max, TIMING_SLOTS);
    for (int k = 0; k < n; k++) {
        ms[k] = X->kernel_ms[k];
        count[k] = X->kernel_count[k];
    }
    return n;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free entry point.
//
// Some callers cannot call cudaMalloc: a host framework that owns every byte
// of device memory through its own pool and forbids outside allocations (an
// extra cudaMalloc would fragment or exceed its reservation), or a latency-
// critical pipeline that cannot afford cudaMalloc's implicit device-wide
// synchronisation in the middle of a run.  For them gpu_mpn_mul_device_noalloc
// computes a product from caller-owned device buffers using only storage that
// is part of this library's device image: the arrays below are allocated when
// the module is loaded on a device and kept until the process exits, on every
// GPU that loads the library.
//
// Limits: an + bn <= NA_MAX_LIMBS (transforms up to 2^18 points, five primes);
// larger products are rejected with GPU_FFT_SMALL_ETOOBIG.  All calls share the
// scratch, which keeps the last call's contents, so calls whose work overlaps on
// the GPU (different streams, or different host threads) race and must be
// serialised by the caller.
//
// The first call on a device sets the device up: it writes the module's
// constant tables unless a context did so already, launches the table kernel
// on CUDA's legacy default stream and synchronises the device.  Make that
// first call before any stream capture.  Later calls only queue kernels on
// the caller's stream and return; a device-side error (the carry look-back's
// bounded wait running out, which takes a GPU that stops scheduling the
// earlier tiles) is recorded in the scratch's error word but cannot be
// reported by the return code, which only covers argument checks, the set-up
// and the launches.
constexpr int NA_LOG_MAXM = 18;
constexpr uint64_t NA_MAX_LIMBS = ((uint64_t)1 << NA_LOG_MAXM) + 1;
constexpr int NA_NP = 5;
constexpr size_t NA_RES_WORDS = (size_t)2 * NA_NP << NA_LOG_MAXM;
constexpr int NA_TILES = (int)((NA_MAX_LIMBS + CRT_TILE - 1) / CRT_TILE);

// scratch: residues of both operands, look-back status, ticket, error flag
static __device__ __align__(256) uint32_t na_scratch[NA_RES_WORDS + NA_TILES + 8];
// constant tables, written once per device by the set-up kernel
static __device__ __align__(256) uint2 na_twf[NA_NP * TW_SZ];
static __device__ __align__(256) uint2 na_twi[NA_NP * TW_SZ];
static __device__ __align__(256) uint2 na_th[NA_NP * TH_SZ];
static __device__ __align__(256) uint2 na_tl[NA_NP * TL_SZ];
static __device__ __align__(256) uint2 na_thi[NA_NP * TH_SZ];
static __device__ __align__(256) uint2 na_tli[NA_NP * TL_SZ];
static __device__ __align__(256) PrimeInfo na_pi[MAX_NP];
static __device__ __align__(256) uint32_t na_scale[(NA_LOG_MAXM + 1) * MAX_NP];
__constant__ uint32_t c_na_primes[NA_NP];
__constant__ uint2 c_na_roots[NA_NP];   // (w, w^-1), w of order 2^25

__device__ uint32_t na_powmod(uint32_t a, uint32_t e, uint32_t p)
{
    uint64_t r = 1, x = a;
    while (e) {
        if (e & 1) r = r * x % p;
        x = x * x % p;
        e >>= 1;
    }
    return (uint32_t)r;
}

// twiddle and twist tables from the order-2^25 roots w[j] and their inverses
__global__ void k_na_tables(uint2* twf, uint2* twi, uint2* th, uint2* tl, uint2* thi, uint2* tli)
{
    const uint2* roots = c_na_roots;
    const int total = NA_NP * (TW_SZ + TH_SZ + TL_SZ);
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < total; f += gridDim.x * blockDim.x) {
        int r = f;
        int kind, j, t;
        if (r < NA_NP * TW_SZ) { kind = 0; j = r / TW_SZ; t = r % TW_SZ; }
        else if ((r -= NA_NP * TW_SZ) < NA_NP * TH_SZ) { kind = 1; j = r / TH_SZ; t = r % TH_SZ; }
        else { r -= NA_NP * TH_SZ; kind = 2; j = r / TL_SZ; t = r % TL_SZ; }
        const uint32_t p = c_na_primes[j];
        uint32_t e;
        if (kind == 0) {
            if (t == 0) { twf[r] = make_uint2(1, 0); twi[r] = make_uint2(1, 0); continue; }
            const int lh = 31 - __clz(t);                 // t = 2^lh + jj
            e = (uint32_t)(t - (1 << lh)) << (LOG_MAXM - lh - 1);
        } else if (kind == 1) {
            e = (uint32_t)t << 13;
        } else {
            e = (uint32_t)t;
        }
        const uint32_t wf = na_powmod(roots[j].x, e, p), wi = na_powmod(roots[j].y, e, p);
        const uint2 vf = make_uint2(wf, shoup_companion_dev(wf, p));
        const uint2 vi = make_uint2(wi, shoup_companion_dev(wi, p));
        if (kind == 0) { twf[j * TW_SZ + t] = vf; twi[j * TW_SZ + t] = vi; }
        else if (kind == 1) { th[j * TH_SZ + t] = vf; thi[j * TH_SZ + t] = vi; }
        else { tl[j * TL_SZ + t] = vf; tli[j * TL_SZ + t] = vi; }
    }
}

struct NaDevice {
    std::atomic<bool> ready{false};   // stored (release) after every field below is set
    Ctx ctx;                       // only T and nsm are used by the launches
    uint32_t *res = nullptr, *status = nullptr, *scale = nullptr;
    unsigned long long *ticket = nullptr;
    int *err = nullptr;
};
constexpr int NA_MAX_DEVICES = 64;
static NaDevice g_na[NA_MAX_DEVICES];
static std::mutex g_na_lock;

// 2^32-word product and cofactors of the first NA_NP primes, fixed-size
static void na_crt_constants(CrtConst &K, uint32_t *cof_red)
{
    uint32_t P[MAX_NP + 1] = {1};
    int n = 1;
    for (int j = 0; j < NA_NP; j++) {
        uint64_t c = 0;
        for (int w = 0; w < n; w++) {
            const uint64_t t = (uint64_t)P[w] * PRIMES[j] + c;
            P[w] = (uint32_t)t;
            c = t >> 32;
        }
        if (c) P[n++] = (uint32_t)c;
    }
    memset(&K, 0, sizeof K);
    K.np = NA_NP;
    for (int w = 0; w < n && w < MAX_NP; w++) K.P[w] = P[w];
    for (int j = 0; j < NA_NP; j++) {
        uint64_t r = 0;
        for (int w = n - 1; w >= 0; w--) {
            const uint64_t t = (r << 32) | P[w];
            K.cof[j][w] = (uint32_t)(t / PRIMES[j]);
            r = t % PRIMES[j];
        }
        uint64_t m = 0;
        for (int w = n - 1; w >= 0; w--) m = ((m << 32) | K.cof[j][w]) % PRIMES[j];
        cof_red[j] = (uint32_t)m;
        K.finv[j] = 1.0f / (float)PRIMES[j];
    }
}

// set-up runtime calls: no error message (that would allocate), just the code
#define NA_CU(call)                                                           \
    do {                                                                      \
        if ((call) != cudaSuccess) return GPU_FFT_SMALL_ECUDA;                \
    } while (0)

static int na_setup(int dev, NaDevice &D)
{
    // order-2^25 roots of unity (forward, inverse) per prime
    uint2 roots[NA_NP];
    PrimeInfo pi[MAX_NP];
    memset(pi, 0, sizeof pi);
    for (int j = 0; j < NA_NP; j++) {
        const uint32_t p = PRIMES[j];
        const uint32_t w = h_powmod(primitive_root(p), (p - 1) >> LOG_MAXM, p), wi = h_invmod(w, p);
        roots[j] = make_uint2(w, wi);
        PrimeInfo &P = pi[j];
        P.p = p;
        uint32_t inv = 1;
        for (int it = 0; it < 5; it++) inv *= 2 - p * inv;
        P.pneg_inv = 0u - inv;
        P.c32 = (uint32_t)((1ull << 32) % p);
        P.r2 = h_mulmod(P.c32, P.c32, p);
        P.finv = 1.0f / (float)p;
    }
    // device addresses of the image's arrays, taken with this device current
    void *scr = nullptr, *twf, *twi, *th, *tl, *thi, *tli, *pip, *sc;
    NA_CU(cudaGetSymbolAddress(&scr, na_scratch));
    NA_CU(cudaGetSymbolAddress(&twf, na_twf));
    NA_CU(cudaGetSymbolAddress(&twi, na_twi));
    NA_CU(cudaGetSymbolAddress(&th, na_th));
    NA_CU(cudaGetSymbolAddress(&tl, na_tl));
    NA_CU(cudaGetSymbolAddress(&thi, na_thi));
    NA_CU(cudaGetSymbolAddress(&tli, na_tli));
    NA_CU(cudaGetSymbolAddress(&pip, na_pi));
    NA_CU(cudaGetSymbolAddress(&sc, na_scale));
    for (int r = 0; r < 12; r++) {
        NA_CU(cudaFuncSetAttribute(FWD_COLS[r], cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024));
        NA_CU(cudaFuncSetAttribute(INV_COLS[r], cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024));
    }
    for (int r = 0; r < 3; r++) {
        NA_CU(cudaFuncSetAttribute(FWD_COLS_C13[r], cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024));
        NA_CU(cudaFuncSetAttribute(INV_COLS_C13[r], cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024));
    }
    for (int c = 5; c <= LOG_MAXC; c++)
        NA_CU(cudaFuncSetAttribute(ROWS[c], cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
    for (int c = ROWS16_MIN_LOGC; c <= LOG_MAXC; c++)
        NA_CU(cudaFuncSetAttribute(ROWS16[c], cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
    NA_CU(cudaMemcpyToSymbol(c_na_primes, PRIMES, sizeof(uint32_t) * NA_NP));
    NA_CU(cudaMemcpyToSymbol(c_na_roots, roots, sizeof roots));
    // the module-wide constant tables (all MAX_NP primes), unless a context
    // or an earlier set-up on this device has written them already
    NA_CU(device_constants_ensure(dev));
    NA_CU(cudaMemcpyToSymbol(na_pi, pi, sizeof pi));
    k_na_tables<<<256, 256>>>((uint2 *)twf, (uint2 *)twi, (uint2 *)th, (uint2 *)tl, (uint2 *)thi,
                              (uint2 *)tli);
    NA_CU(cudaGetLastError());
    // pointwise scales for five primes and every transform length
    CrtConst K;
    uint32_t cof_red[MAX_NP];
    na_crt_constants(K, cof_red);
    uint32_t scales[(NA_LOG_MAXM + 1) * MAX_NP];
    memset(scales, 0, sizeof scales);
    for (int lm = 0; lm <= NA_LOG_MAXM; lm++)
        for (int j = 0; j < NA_NP; j++) {
            const uint32_t p = PRIMES[j];
            uint32_t s = h_invmod(h_powmod(2, lm, p), p);
            s = h_mulmod(s, h_invmod(cof_red[j], p), p);
            scales[lm * MAX_NP + j] = h_mulmod(s, h_powmod(2, 128, p), p);
        }
    NA_CU(cudaMemcpyToSymbol(na_scale, scales, sizeof scales));
    NA_CU(cudaDeviceSynchronize());
    D.ctx.device = dev;
    NA_CU(cudaDeviceGetAttribute(&D.ctx.nsm, cudaDevAttrMultiProcessorCount, dev));
    D.ctx.T.pi = (const PrimeInfo *)pip;
    D.ctx.T.twf = (const uint2 *)twf;
    D.ctx.T.twi = (const uint2 *)twi;
    D.ctx.T.th = (const uint2 *)th;
    D.ctx.T.tl = (const uint2 *)tl;
    D.ctx.T.thi = (const uint2 *)thi;
    D.ctx.T.tli = (const uint2 *)tli;
    D.ctx.crt[NA_NP] = K;
    D.res = (uint32_t *)scr;
    D.status = D.res + NA_RES_WORDS;
    D.ticket = (unsigned long long *)(D.status + NA_TILES + (NA_TILES & 1));   // 8-byte aligned
    D.err = (int *)(D.ticket + 1);
    D.scale = (uint32_t *)sc;
    D.ready.store(true, std::memory_order_release);
    return 0;
}

extern "C" {

int gpu_mpn_mul_device_noalloc(uint64_t *z_dev, const uint64_t *a_dev, gpu_ulong an,
                               const uint64_t *b_dev, gpu_ulong bn, void *stream)
{
    if (an == 0 || bn == 0 || !z_dev || !a_dev || !b_dev) return GPU_FFT_SMALL_EINVAL;
    if (an > NA_MAX_LIMBS || bn > NA_MAX_LIMBS - an) return GPU_FFT_SMALL_ETOOBIG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NA_MAX_DEVICES)
        return GPU_FFT_SMALL_ECUDA;
    NaDevice &D = g_na[dev];
    if (!D.ready.load(std::memory_order_acquire)) {
        std::lock_guard<std::mutex> guard(g_na_lock);
        if (!D.ready.load(std::memory_order_relaxed) && na_setup(dev, D) != 0)
            return GPU_FFT_SMALL_ECUDA;
    }
    const cudaStream_t st = (cudaStream_t)stream;
    const uint64_t L = an + bn - 1;
    int logM = MIN_LOGM;
    while (((uint64_t)1 << logM) < L) logM++;
    const LaunchShape shape = make_shape(logM);
    const bool sq = (a_dev == b_dev) && (an == bn);
    const size_t M = (size_t)1 << logM;
    uint32_t *ra = D.res, *rb = D.res + (size_t)NA_NP * M;
    const uint64_t zn = an + bn;
    constexpr int THREADS = CRT_THREADS, TILE = CRT_TILE;
    const size_t tiles = (zn + TILE - 1) / TILE;
    // the scratch keeps the previous call's contents: clear the look-back
    // status, the tile ticket and the error flag
    if (cudaMemsetAsync(D.status, 0, (NA_TILES + 8) * sizeof(uint32_t), st) != cudaSuccess)
        return GPU_FFT_SMALL_ECUDA;
    launch_transforms(&D.ctx, shape, NA_NP, a_dev, an, b_dev, bn, ra, rb, sq,
                      D.scale + (size_t)logM * MAX_NP, st, nullptr);
    k_crt_carry<NA_NP, THREADS><<<tiles, THREADS, 0, st>>>(ra, logM, L, zn, z_dev, D.ctx.crt[NA_NP],
                                                          D.status, D.ticket, 0ull, 1u, D.err,
                                                          nullptr, nullptr, 0ull);
    return cudaGetLastError() == cudaSuccess ? GPU_FFT_SMALL_OK : GPU_FFT_SMALL_ECUDA;
}

}  // extern "C"
