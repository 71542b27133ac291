/*
 * sun_oracle.c -- FP64 CPU restatement of the CULQCD (nmrcardoso/sun) hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA engine and the timed CPU
 * baseline.  Nothing in the product links or calls this file.
 *
 * Each function cites the reference code it restates (paths relative to the
 * reference project root).  Build: gcc -O2 -fcx-limited-range -fopenmp -fPIC
 * -shared (see oracle/Makefile).  -fcx-limited-range only drops C99 Annex-G
 * inf/nan recovery from complex multiply; the arithmetic on finite values is
 * the textbook (ac-bd, ad+bc).
 */
#include "sun_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cplx;
#define TWO_PI 6.2831853071795864769252867665590
#define NMAX 8

/* ------------------------------------------------------------------------- */
/* Philox4x32-10 (Salmon et al., SC'11): 10 rounds of the 4x32 S-box with the
 * published multipliers and Weyl key increments. */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n1 = lo1;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        uint32_t n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        if (r < 9) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Per-link uniform stream.  Philox modes draw words from counter
 * (block, lex, mu | purpose << 8, pass); injected mode reads a buffer. */
typedef struct {
    int mode;
    uint32_t key[2];
    uint32_t ctr[4];
    uint32_t buf[4];
    int pos;           /* next word in buf (4 = empty) */
    const double *inj;
    int inj_len, inj_pos;
    int used;
    int overrun;
} stream_t;

static void stream_init(stream_t *s, int mode, uint64_t seed, int lex, int mu, int purpose,
                        uint32_t pass, const double *inj, int inj_len)
{
    s->mode = mode;
    s->key[0] = (uint32_t)(seed & 0xffffffffu);
    s->key[1] = (uint32_t)(seed >> 32);
    s->ctr[0] = 0;
    s->ctr[1] = (uint32_t)lex;
    s->ctr[2] = (uint32_t)(mu | (purpose << 8));
    s->ctr[3] = pass;
    s->pos = 4;
    s->inj = inj; s->inj_len = inj_len; s->inj_pos = 0;
    s->used = 0; s->overrun = 0;
}

static uint32_t stream_word(stream_t *s)
{
    if (s->pos == 4) {
        orc_philox4x32_10(s->ctr, s->key, s->buf);
        s->ctr[0]++;
        s->pos = 0;
    }
    return s->buf[s->pos++];
}

static double stream_uniform(stream_t *s)
{
    s->used++;
    if (s->mode == ORC_RNG_INJECTED) {
        if (s->inj_pos >= s->inj_len) { s->overrun = 1; return 0.5; }
        return s->inj[s->inj_pos++];
    }
    if (s->mode == ORC_RNG_PHILOX32) {
        uint32_t w = stream_word(s);
        return (double)((w >> 8) + 1u) * (1.0 / 16777216.0);
    }
    uint32_t a = stream_word(s);
    uint32_t b = stream_word(s);
    uint64_t k = ((uint64_t)(a >> 11) << 32) | (uint64_t)b;
    return (double)(k + 1u) * (1.0 / 9007199254740992.0);
}

void orc_uniforms(uint64_t seed, int lex, int mu, int purpose, uint32_t pass,
                  int fp64, int n, double *out)
{
    stream_t s;
    stream_init(&s, fp64 ? ORC_RNG_PHILOX64 : ORC_RNG_PHILOX32, seed, lex, mu, purpose, pass, 0, 0);
    for (int i = 0; i < n; ++i) out[i] = stream_uniform(&s);
}

/* ------------------------------------------------------------------------- */
/* SU(N) matrix helpers on cplx[N*N] row-major. */
static inline void mat_mul(int N, const cplx *A, const cplx *B, cplx *C)
{
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) {
            cplx s = 0;
            for (int k = 0; k < N; ++k) s += A[i * N + k] * B[k * N + j];
            C[i * N + j] = s;
        }
}
/* C = A * B^dagger */
static inline void mat_mul_nd(int N, const cplx *A, const cplx *B, cplx *C)
{
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) {
            cplx s = 0;
            for (int k = 0; k < N; ++k) s += A[i * N + k] * conj(B[j * N + k]);
            C[i * N + j] = s;
        }
}
/* C = A^dagger * B */
static inline void mat_mul_dn(int N, const cplx *A, const cplx *B, cplx *C)
{
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) {
            cplx s = 0;
            for (int k = 0; k < N; ++k) s += conj(A[k * N + i]) * B[k * N + j];
            C[i * N + j] = s;
        }
}
static inline void mat_dagger(int N, const cplx *A, cplx *B)
{
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) B[j * N + i] = conj(A[i * N + j]);
}
static inline void mat_unit(int N, cplx *A)
{
    for (int i = 0; i < N * N; ++i) A[i] = 0;
    for (int i = 0; i < N; ++i) A[i * N + i] = 1;
}
static inline cplx mat_trace(int N, const cplx *A)
{
    cplx t = 0;
    for (int i = 0; i < N; ++i) t += A[i * N + i];
    return t;
}

/* Determinant by Gaussian elimination with partial pivoting. */
static cplx mat_det(int N, const cplx *A)
{
    cplx b[NMAX * NMAX];
    memcpy(b, A, sizeof(cplx) * N * N);
    cplx det = 1;
    for (int k = 0; k < N; ++k) {
        int piv = k;
        double best = cabs(b[k * N + k]);
        for (int i = k + 1; i < N; ++i)
            if (cabs(b[i * N + k]) > best) { best = cabs(b[i * N + k]); piv = i; }
        if (best == 0.0) return 0;
        if (piv != k) {
            for (int j = 0; j < N; ++j) { cplx t = b[k * N + j]; b[k * N + j] = b[piv * N + j]; b[piv * N + j] = t; }
            det = -det;
        }
        det *= b[k * N + k];
        for (int i = k + 1; i < N; ++i) {
            cplx f = b[i * N + k] / b[k * N + k];
            for (int j = k; j < N; ++j) b[i * N + j] -= f * b[k * N + j];
        }
    }
    return det;
}

/* SU(2) subgroup enumeration: (0,1),(1,2),...,(N-2,N-1), then (0,2),(1,3),...
 * -- restates IndexBlock (include/constants.h:143-192). */
void orc_su2_index(int N, int block, int *p, int *q)
{
    int idx = -1;
    for (int del = 1; del < N; ++del)
        for (int i = 0; i < N - del; ++i) {
            ++idx;
            if (idx == block) { *p = i; *q = i + del; return; }
        }
    *p = -1; *q = -1;
}

/* Reunitarization -- restates reunit_link (include/reunitlink.h:16-88).
 * N == 3: normalise row 0, orthogonalise and normalise row 1, row 2 =
 * conj(row0 x row1).  N > 3: Gram-Schmidt over columns, then multiply the
 * last column by exp(-i arg det).  N == 2 (no reference build exists,
 * reunitlink.h:86 #error): normalise row 0 and set row 1 = (-conj u01, conj u00). */
static void reunit(int N, cplx *U)
{
    if (N == 2) {
        double n = sqrt(creal(U[0] * conj(U[0])) + creal(U[1] * conj(U[1])));
        U[0] /= n; U[1] /= n;
        U[2] = -conj(U[1]);
        U[3] = conj(U[0]);
        return;
    }
    if (N == 3) {
        double t1 = 0;
        for (int c = 0; c < 3; ++c) t1 += creal(U[c]) * creal(U[c]) + cimag(U[c]) * cimag(U[c]);
        t1 = 1.0 / sqrt(t1);
        for (int c = 0; c < 3; ++c) U[c] *= t1;
        cplx t2 = 0;
        for (int c = 0; c < 3; ++c) t2 += conj(U[c]) * U[3 + c];
        for (int c = 0; c < 3; ++c) U[3 + c] -= t2 * U[c];
        t1 = 0;
        for (int c = 0; c < 3; ++c) t1 += creal(U[3 + c]) * creal(U[3 + c]) + cimag(U[3 + c]) * cimag(U[3 + c]);
        t1 = 1.0 / sqrt(t1);
        for (int c = 0; c < 3; ++c) U[3 + c] *= t1;
        U[6] = conj(U[1] * U[5] - U[2] * U[4]);
        U[7] = conj(U[2] * U[3] - U[0] * U[5]);
        U[8] = conj(U[0] * U[4] - U[1] * U[3]);
        return;
    }
    double t1 = 0;
    for (int c = 0; c < N; ++c) t1 += creal(U[c * N]) * creal(U[c * N]) + cimag(U[c * N]) * cimag(U[c * N]);
    t1 = 1.0 / sqrt(t1);
    for (int c = 0; c < N; ++c) U[c * N] *= t1;
    for (int j = 1; j < N; ++j) {
        for (int i = 0; i < j; ++i) {
            cplx t2 = 0;
            for (int c = 0; c < N; ++c) t2 += conj(U[c * N + i]) * U[c * N + j];
            for (int c = 0; c < N; ++c) U[c * N + j] -= t2 * U[c * N + i];
        }
        t1 = 0;
        for (int c = 0; c < N; ++c) t1 += creal(U[c * N + j]) * creal(U[c * N + j]) + cimag(U[c * N + j]) * cimag(U[c * N + j]);
        t1 = 1.0 / sqrt(t1);
        for (int c = 0; c < N; ++c) U[c * N + j] *= t1;
    }
    cplx d = mat_det(N, U);
    double ph = atan2(cimag(d), creal(d));
    cplx f = cos(ph) - I * sin(ph);
    for (int c = 0; c < N; ++c) U[c * N + N - 1] *= f;
}

void orc_reunit_link(int N, double *U) { reunit(N, (cplx *)U); }

/* ------------------------------------------------------------------------- */
/* SU(2) heatbath draw -- restates generate_su2_matrix_milc
 * (include/device_PHB_OVR.h:163-223): Kennedy-Pendleton when alpha > 2,
 * Creutz otherwise, at most 20 retries each, 1e-10 inside the logs. */
static void su2_milc(double al, stream_t *s, double a[4])
{
    double xr1, xr2, xr3, xr4, d, r;
    double a0 = 0;
    xr1 = log(stream_uniform(s) + 1.e-10);
    xr2 = log(stream_uniform(s) + 1.e-10);
    xr3 = stream_uniform(s);
    xr4 = stream_uniform(s);
    xr3 = cos(TWO_PI * xr3);
    d = -(xr2 + xr1 * xr3 * xr3) / al;
    int accepted = (1.00 - 0.5 * d) > xr4 * xr4;
    if (!accepted && al > 2.0) {
        for (int k = 0; k < 20; ++k) {
            xr1 = log(stream_uniform(s) + 1.e-10);
            xr2 = log(stream_uniform(s) + 1.e-10);
            xr3 = stream_uniform(s);
            xr4 = stream_uniform(s);
            xr3 = cos(TWO_PI * xr3);
            d = -(xr2 + xr1 * xr3 * xr3) / al;
            if ((1.00 - 0.5 * d) > xr4 * xr4) break;
        }
    }
    if (!accepted && al <= 2.0) {
        xr3 = exp(-2.0 * al);
        xr4 = 1.0 - xr3;
        for (int k = 0; k < 20; ++k) {
            xr1 = stream_uniform(s);
            xr2 = stream_uniform(s);
            r = xr3 + xr4 * xr1;
            a0 = 1.00 + log(r) / al;
            if ((1.0 - a0 * a0) > xr2 * xr2) break;
        }
        d = 1.0 - a0;
    }
    a0 = 1.0 - d;
    xr3 = fabs(1.0 - a0 * a0);
    r = sqrt(xr3);
    a[0] = a0;
    a[3] = (2.0 * stream_uniform(s) - 1.0) * r;
    xr1 = sqrt(fabs(xr3 - a[3] * a[3]));
    xr2 = TWO_PI * stream_uniform(s);
    a[1] = xr1 * cos(xr2);
    a[2] = xr1 * sin(xr2);
}

void orc_su2_generate(double alpha, int mode, uint64_t seed, int lex, int mu,
                      uint32_t pass, const double *inj, int inj_len, double a[4], int *used)
{
    stream_t s;
    stream_init(&s, mode, seed, lex, mu, 0, pass, inj, inj_len);
    su2_milc(alpha, &s, a);
    if (used) *used = s.overrun ? -1 : s.used;
}

/* Block 4-vector of the (p,q) subgroup of M -- restates get_block_su2
 * (device_PHB_OVR.h:265-272). */
static inline void block_of(int N, const cplx *M, int p, int q, double r[4])
{
    r[0] = creal(M[p * N + p]) + creal(M[q * N + q]);
    r[1] = cimag(M[p * N + q]) + cimag(M[q * N + p]);
    r[2] = creal(M[p * N + q]) - creal(M[q * N + p]);
    r[3] = cimag(M[p * N + p]) - cimag(M[q * N + q]);
}

/* rows p,q of L <- su2(b) * rows p,q -- restates mul_block_sun
 * (device_PHB_OVR.h:296-303). */
static inline void apply_block(int N, cplx *L, int p, int q, const double b[4])
{
    cplx a00 = b[0] + I * b[3], a01 = b[2] + I * b[1];
    cplx a10 = -b[2] + I * b[1], a11 = b[0] - I * b[3];
    for (int j = 0; j < N; ++j) {
        cplx up = L[p * N + j], uq = L[q * N + j];
        L[p * N + j] = a00 * up + a01 * uq;
        L[q * N + j] = a10 * up + a11 * uq;
    }
}

/* a * r^dagger on 4-vectors -- restates mulsu2UVDagger (msu2.h:212-219). */
static inline void su2_mul_udag(const double a[4], const double r[4], double b[4])
{
    b[0] = a[0] * r[0] + a[1] * r[1] + a[2] * r[2] + a[3] * r[3];
    b[1] = a[1] * r[0] - a[0] * r[1] + a[2] * r[3] - a[3] * r[2];
    b[2] = a[2] * r[0] - a[0] * r[2] + a[3] * r[1] - a[1] * r[3];
    b[3] = a[3] * r[0] - a[0] * r[3] + a[1] * r[2] - a[2] * r[1];
}

/* (U F) restricted to rows p,q and columns p,q, for the SU(3) path that
 * recomputes the block from the current U (device_PHB_OVR.h:382-405). */
static inline void block_from_UF(int N, const cplx *U, const cplx *F, int p, int q, double r[4])
{
    cplx a0 = 0, a1 = 0, a2 = 0, a3 = 0;
    for (int j = 0; j < N; ++j) {
        a0 += U[p * N + j] * F[j * N + p];
        a1 += U[p * N + j] * F[j * N + q];
        a2 += U[q * N + j] * F[j * N + p];
        a3 += U[q * N + j] * F[j * N + q];
    }
    r[0] = creal(a0) + creal(a3);
    r[1] = cimag(a1) + cimag(a2);
    r[2] = creal(a1) - creal(a2);
    r[3] = cimag(a0) - cimag(a3);
}

/* Cabibbo-Marinari pseudo-heatbath -- restates heatBathSUN
 * (device_PHB_OVR.h:362-485).  N == 3 recomputes each block from U and F;
 * other N keep M = U F and update it alongside U. */
static void heatbath_link(int N, cplx *U, const cplx *F, double beta_over_n, stream_t *s)
{
    int nb = N * (N - 1) / 2;
    cplx M[NMAX * NMAX];
    if (N != 3) mat_mul(N, U, F, M);
    for (int blk = 0; blk < nb; ++blk) {
        int p, q;
        orc_su2_index(N, blk, &p, &q);
        double r[4], a[4], b[4];
        if (N == 3) block_from_UF(N, U, F, p, q, r);
        else block_of(N, M, p, q, r);
        double k = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + r[3] * r[3]);
        double ap = beta_over_n * k;
        k = 1.0 / k;
        for (int i = 0; i < 4; ++i) r[i] *= k;
        su2_milc(ap, s, a);
        su2_mul_udag(a, r, b);
        apply_block(N, U, p, q, b);
        if (N != 3) apply_block(N, M, p, q, b);
    }
}

/* Microcanonical overrelaxation -- restates overrelaxationSUN
 * (device_PHB_OVR.h:494-608): per subgroup, conj-normalise the block vector
 * and apply it twice. */
static void overrelax_link(int N, cplx *U, const cplx *F)
{
    int nb = N * (N - 1) / 2;
    cplx M[NMAX * NMAX];
    if (N != 3) mat_mul(N, U, F, M);
    for (int blk = 0; blk < nb; ++blk) {
        int p, q;
        orc_su2_index(N, blk, &p, &q);
        double r[4];
        if (N == 3) block_from_UF(N, U, F, p, q, r);
        else block_of(N, M, p, q, r);
        double n = 1.0 / sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + r[3] * r[3]);
        r[0] *= n; r[1] *= -n; r[2] *= -n; r[3] *= -n;
        apply_block(N, U, p, q, r);
        apply_block(N, U, p, q, r);
        if (N != 3) { apply_block(N, M, p, q, r); apply_block(N, M, p, q, r); }
    }
}

int orc_heatbath_link(int N, double *U, const double *F, double beta_over_n,
                      int mode, uint64_t seed, int lex, int mu, uint32_t pass,
                      const double *inj, int inj_len)
{
    stream_t s;
    stream_init(&s, mode, seed, lex, mu, 0, pass, inj, inj_len);
    heatbath_link(N, (cplx *)U, (const cplx *)F, beta_over_n, &s);
    return s.overrun ? -1 : s.used;
}

void orc_overrelax_link(int N, double *U, const double *F)
{
    overrelax_link(N, (cplx *)U, (const cplx *)F);
}

/* ------------------------------------------------------------------------- */
/* Geometry (canonical lexicographic order). */
static inline void lex_coords(const int X[4], int lex, int x[4])
{
    x[0] = lex % X[0]; lex /= X[0];
    x[1] = lex % X[1]; lex /= X[1];
    x[2] = lex % X[2];
    x[3] = lex / X[2];
}
static inline int coords_lex(const int X[4], const int x[4])
{
    return ((x[3] * X[2] + x[2]) * X[1] + x[1]) * X[0] + x[0];
}
static inline int shift(const int X[4], int lex, int mu, int d)
{
    int x[4];
    lex_coords(X, lex, x);
    x[mu] = (x[mu] + d + X[mu]) % X[mu];
    return coords_lex(X, x);
}
static inline const cplx *LINK(const cplx *U, int N, int lex, int mu)
{
    return U + ((size_t)lex * 4 + mu) * N * N;
}

/* Staple sum S = sum_{nu != mu} [ U_nu(x) U_mu(x+nu) U_nu(x+mu)^dagger
 *                               + U_nu(x-nu)^dagger U_mu(x-nu) U_nu(x-nu+mu) ]
 * in the reference's nu order, "up" then "down" (src/monte/monte.cu:64-80). */
static void staple(int N, const int X[4], const cplx *U, int lex, int mu, cplx *S)
{
    cplx T1[NMAX * NMAX], T2[NMAX * NMAX];
    for (int i = 0; i < N * N; ++i) S[i] = 0;
    int xpmu = shift(X, lex, mu, 1);
    for (int nu = 0; nu < 4; ++nu) {
        if (nu == mu) continue;
        int xpnu = shift(X, lex, nu, 1);
        int xmnu = shift(X, lex, nu, -1);
        int xmnu_pmu = shift(X, xmnu, mu, 1);
        mat_mul(N, LINK(U, N, lex, nu), LINK(U, N, xpnu, mu), T1);
        mat_mul_nd(N, T1, LINK(U, N, xpmu, nu), T2);
        for (int i = 0; i < N * N; ++i) S[i] += T2[i];
        mat_mul_dn(N, LINK(U, N, xmnu, nu), LINK(U, N, xmnu, mu), T1);
        mat_mul(N, T1, LINK(U, N, xmnu_pmu, nu), T2);
        for (int i = 0; i < N * N; ++i) S[i] += T2[i];
    }
}

void orc_staple(int N, const int X[4], const double *U, int lex, int mu, double *S)
{
    staple(N, X, (const cplx *)U, lex, mu, (cplx *)S);
}

static inline int site_parity(const int X[4], int lex)
{
    int x[4];
    lex_coords(X, lex, x);
    return (x[0] + x[1] + x[2] + x[3]) & 1;
}

/* One checkerboard phase: every link (x, mu) with parity(x) == parity is
 * replaced by its heatbath or overrelaxation update with F = staple^dagger
 * -- restates kernel_PHeatBath_evenodd (src/monte/monte.cu:44-88) and
 * kernel_overrelaxation_evenodd (src/monte/ovr.cu:41-80). */
int orc_update_phase(int N, const int X[4], double *Ud, int parity, int mu, int kind,
                     double beta, int mode, uint64_t seed, uint32_t pass,
                     const double *inj, int inj_stride, int nthreads)
{
    cplx *U = (cplx *)Ud;
    int V = X[0] * X[1] * X[2] * X[3];
    double bon = beta / N;
    int overruns = 0;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(static) num_threads(nthreads) reduction(+ : overruns)
#endif
    for (int lex = 0; lex < V; ++lex) {
        if (site_parity(X, lex) != parity) continue;
        cplx S[NMAX * NMAX], F[NMAX * NMAX];
        staple(N, X, U, lex, mu, S);
        mat_dagger(N, S, F);
        cplx *L = U + ((size_t)lex * 4 + mu) * N * N;
        if (kind == 0) {
            stream_t s;
            const double *ip = inj ? inj + ((size_t)lex * 4 + mu) * inj_stride : 0;
            stream_init(&s, mode, seed, lex, mu, 0, pass, ip, inj_stride);
            heatbath_link(N, L, F, bon, &s);
            overruns += s.overrun;
        } else {
            overrelax_link(N, L, F);
        }
    }
    (void)nthreads;
    return overruns;
}

void orc_reunitarize(int N, const int X[4], double *Ud)
{
    cplx *U = (cplx *)Ud;
    int V = X[0] * X[1] * X[2] * X[3];
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int l = 0; l < 4 * V; ++l) reunit(N, U + (size_t)l * N * N);
}

/* Sweeps as the reference composes them: HeatBath::Run then
 * OverRelaxation::Run, each 2 parities x 4 directions (monte.cu:205-206). */
void orc_sweeps(int N, const int X[4], double *U, double beta, int n_hb, int n_or,
                int n_sweeps, int reunit_every, int mode, uint64_t seed, uint32_t *pass,
                int nthreads)
{
    for (int s = 0; s < n_sweeps; ++s) {
        for (int h = 0; h < n_hb; ++h) {
            for (int p = 0; p < 2; ++p)
                for (int mu = 0; mu < 4; ++mu)
                    orc_update_phase(N, X, U, p, mu, 0, beta, mode, seed, *pass, 0, 0, nthreads);
            (*pass)++;
        }
        for (int o = 0; o < n_or; ++o)
            for (int p = 0; p < 2; ++p)
                for (int mu = 0; mu < 4; ++mu)
                    orc_update_phase(N, X, U, p, mu, 1, beta, mode, seed, *pass, 0, 0, nthreads);
        if (reunit_every > 0 && (s + 1) % reunit_every == 0) orc_reunitarize(N, X, U);
    }
}

/* Mean link trace / N and mean link determinant -- the sums of GaugeTraceCUB
 * (src/meas/linktrsum.cu:56, normalised :146 by 4 N V) and GaugeDetCUB
 * (src/meas/linkdetsum.cu:62, normalised :115 by 4 V).
 * out = {Re tr/N, Im tr/N, Re det, Im det}. */
void orc_link_trace_det(int N, const int X[4], const double *Ud, double out[4])
{
    const cplx *U = (const cplx *)Ud;
    int V = X[0] * X[1] * X[2] * X[3];
    cplx tr = 0, det = 0;
    for (int l = 0; l < 4 * V; ++l) {
        tr += mat_trace(N, U + (size_t)l * N * N);
        det += mat_det(N, U + (size_t)l * N * N);
    }
    out[0] = creal(tr) / (4.0 * N * V);
    out[1] = cimag(tr) / (4.0 * N * V);
    out[2] = creal(det) / (4.0 * V);
    out[3] = cimag(det) / (4.0 * V);
}

double orc_unitarity_violation(int N, const int X[4], const double *Ud)
{
    const cplx *U = (const cplx *)Ud;
    int V = X[0] * X[1] * X[2] * X[3];
    double worst = 0;
    for (int l = 0; l < 4 * V; ++l) {
        cplx P[NMAX * NMAX];
        mat_mul_dn(N, U + (size_t)l * N * N, U + (size_t)l * N * N, P);
        for (int i = 0; i < N; ++i)
            for (int j = 0; j < N; ++j) {
                double d = cabs(P[i * N + j] - (i == j ? 1.0 : 0.0));
                if (d > worst) worst = d;
            }
    }
    return worst;
}

/* ------------------------------------------------------------------------- */
/* Plaquette -- restates kernel_calc_plaquette_*_cub
 * (src/meas/plaquette_cub.cu:97-145) and its normalisation 1/(3 N V) (:234):
 * out[0] = spatial (nu < 3), out[1] = temporal (nu == 3). */
void orc_plaquette(int N, const int X[4], const double *Ud, double out[2])
{
    const cplx *U = (const cplx *)Ud;
    int V = X[0] * X[1] * X[2] * X[3];
    double sp = 0, tp = 0;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) reduction(+ : sp, tp)
#endif
    for (int lex = 0; lex < V; ++lex) {
        cplx A[NMAX * NMAX], B[NMAX * NMAX], C[NMAX * NMAX];
        for (int mu = 0; mu < 3; ++mu) {
            int xpmu = shift(X, lex, mu, 1);
            for (int nu = mu + 1; nu < 4; ++nu) {
                int xpnu = shift(X, lex, nu, 1);
                mat_mul(N, LINK(U, N, lex, mu), LINK(U, N, xpmu, nu), A);
                mat_mul(N, LINK(U, N, lex, nu), LINK(U, N, xpnu, mu), B);
                mat_mul_nd(N, A, B, C);
                double t = creal(mat_trace(N, C));
                if (nu == 3) tp += t; else sp += t;
            }
        }
    }
    out[0] = sp / (3.0 * N * V);
    out[1] = tp / (3.0 * N * V);
}

/* Polyakov loop -- restates kernel_calc_polyakovloop_evenodd
 * (src/meas/polyakovloop.cu:54-96): L(x) = U_3(x,0) U_3(x,1) ... U_3(x,T-1),
 * result sum tr L / (N V_3) (:761). */
void orc_polyakov(int N, const int X[4], const double *Ud, double out[2])
{
    const cplx *U = (const cplx *)Ud;
    int V3 = X[0] * X[1] * X[2];
    double re = 0, im = 0;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) reduction(+ : re, im)
#endif
    for (int s = 0; s < V3; ++s) {
        cplx L[NMAX * NMAX], T[NMAX * NMAX];
        mat_unit(N, L);
        for (int t = 0; t < X[3]; ++t) {
            mat_mul(N, L, LINK(U, N, s + t * V3, 3), T);
            memcpy(L, T, sizeof(cplx) * N * N);
        }
        cplx tr = mat_trace(N, L);
        re += creal(tr);
        im += cimag(tr);
    }
    out[0] = re / ((double)N * V3);
    out[1] = im / ((double)N * V3);
}

/* Planar R x T Wilson loops averaged over the 3 spatial directions --
 * restates kernel_WilsonLineSP / kernel_WilsonLoopSP
 * (src/meas/wilsonloop.cu:60-128): W(r,t) = tr[ L_mu(x,r) T(x+r mu,t)
 * L_mu(x+t e3,r)^dagger T(x,t)^dagger ], sum / (3 N V) (:525).
 * out[2*(t + r*(T+1)) + {0,1}] = (re, im). */
void orc_wilson_loops(int N, const int X[4], const double *Ud, int R, int T, double *out)
{
    const cplx *U = (const cplx *)Ud;
    int V = X[0] * X[1] * X[2] * X[3];
    int nres = (R + 1) * (T + 1);
    double *acc = calloc((size_t)2 * nres, sizeof(double));
#ifdef _OPENMP
#pragma omp parallel
#endif
    {
        double *loc = calloc((size_t)2 * nres, sizeof(double));
        cplx *Ls = malloc(sizeof(cplx) * (T + 1) * NMAX * NMAX);
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
        for (int lex = 0; lex < V; ++lex) {
            cplx T0[NMAX * NMAX], T1[NMAX * NMAX], P[NMAX * NMAX], Q[NMAX * NMAX], tmp[NMAX * NMAX];
            for (int mu = 0; mu < 3; ++mu) {
                for (int t = 0; t <= T; ++t) mat_unit(N, Ls + t * N * N);
                for (int r = 0; r <= R; ++r) {
                    if (r > 0)
                        for (int t = 0; t <= T; ++t) {
                            int y = shift(X, shift(X, lex, 3, t), mu, r - 1);
                            mat_mul(N, Ls + t * N * N, LINK(U, N, y, mu), tmp);
                            memcpy(Ls + t * N * N, tmp, sizeof(cplx) * N * N);
                        }
                    mat_unit(N, T0);
                    mat_unit(N, T1);
                    int xr = shift(X, lex, mu, r);
                    for (int t = 0; t <= T; ++t) {
                        /* tr[L0 T1 Lt^dag T0^dag] = sum_ij (L0 T1)_ij conj((T0 Lt)_ij) */
                        mat_mul(N, Ls, T1, P);
                        mat_mul(N, T0, Ls + t * N * N, Q);
                        cplx w = 0;
                        for (int i = 0; i < N * N; ++i) w += P[i] * conj(Q[i]);
                        loc[2 * (t + r * (T + 1))] += creal(w);
                        loc[2 * (t + r * (T + 1)) + 1] += cimag(w);
                        if (t < T) {
                            mat_mul(N, T0, LINK(U, N, shift(X, lex, 3, t), 3), tmp);
                            memcpy(T0, tmp, sizeof(cplx) * N * N);
                            mat_mul(N, T1, LINK(U, N, shift(X, xr, 3, t), 3), tmp);
                            memcpy(T1, tmp, sizeof(cplx) * N * N);
                        }
                    }
                }
            }
        }
#ifdef _OPENMP
#pragma omp critical
#endif
        for (int i = 0; i < 2 * nres; ++i) acc[i] += loc[i];
        free(loc);
        free(Ls);
    }
    for (int i = 0; i < 2 * nres; ++i) out[i] = acc[i] / (3.0 * N * V);
    free(acc);
}

/* ------------------------------------------------------------------------- */
/* Initial configurations.  Cold: identity (gaugearray.cu:278).  Hot: Haar
 * SU(N) per link -- a new definition (the reference's kernel_hot_start1,
 * gaugearray.cu:355, fills uniform entries and reunitarizes, which is not
 * Haar).  Each entry (i,j) is a complex Gaussian from Philox block i*N+j of
 * stream (lex, mu, purpose 1): Box-Muller on FP64 uniforms u1,u2 ->
 * sqrt(-2 ln u1) (cos 2 pi u2, sin 2 pi u2).  Modified Gram-Schmidt over
 * the columns gives the Haar-U(N) Q of a QR with positive diagonal R; the
 * phase exp(-i arg(det Q)/N) moves it onto SU(N). */
void orc_cold(int N, const int X[4], double *Ud)
{
    cplx *U = (cplx *)Ud;
    int V = X[0] * X[1] * X[2] * X[3];
    for (int l = 0; l < 4 * V; ++l) mat_unit(N, U + (size_t)l * N * N);
}

static void haar_link(int N, uint64_t seed, int lex, int mu, cplx *Q)
{
    stream_t s;
    stream_init(&s, ORC_RNG_PHILOX64, seed, lex, mu, 1, 0, 0, 0);
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) {
            double u1 = stream_uniform(&s);
            double u2 = stream_uniform(&s);
            double rad = sqrt(-2.0 * log(u1));
            double th = TWO_PI * u2;
            Q[i * N + j] = rad * cos(th) + I * (rad * sin(th));
        }
    for (int j = 0; j < N; ++j) {
        for (int i = 0; i < j; ++i) {
            cplx d = 0;
            for (int c = 0; c < N; ++c) d += conj(Q[c * N + i]) * Q[c * N + j];
            for (int c = 0; c < N; ++c) Q[c * N + j] -= d * Q[c * N + i];
        }
        double n = 0;
        for (int c = 0; c < N; ++c) n += creal(Q[c * N + j]) * creal(Q[c * N + j]) + cimag(Q[c * N + j]) * cimag(Q[c * N + j]);
        n = 1.0 / sqrt(n);
        for (int c = 0; c < N; ++c) Q[c * N + j] *= n;
    }
    cplx d = mat_det(N, Q);
    double ph = atan2(cimag(d), creal(d)) / N;
    cplx f = cos(ph) - I * sin(ph);
    for (int k = 0; k < N * N; ++k) Q[k] *= f;
}

void orc_hot(int N, const int X[4], double *Ud, uint64_t seed)
{
    cplx *U = (cplx *)Ud;
    int V = X[0] * X[1] * X[2] * X[3];
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int lex = 0; lex < V; ++lex)
        for (int mu = 0; mu < 4; ++mu) haar_link(N, seed, lex, mu, U + ((size_t)lex * 4 + mu) * N * N);
}

/* ------------------------------------------------------------------------- */
/* Device image -- restates the SoA addressing of GAUGE_SAVE / GAUGE_LOAD
 * (include/device_load_save.h:77-289): element e of link (site s, mu) lives at
 * complex index s + mu*V + e*4V, s the lexicographic index or, in even/odd
 * order, (lex >> 1) + parity * V/2.  SOA: e = row-major N*N.  SOA12 (N=3):
 * rows 0 and 1.  SOA8 (N=3): e01, e02, e10, (arg e00, arg e20). */
int orc_layout_elems(int N, int layout)
{
    if (layout == ORC_SOA12) return 6;
    if (layout == ORC_SOA8) return 4;
    return N * N;
}

static inline size_t img_site(const int X[4], int lex, int evenodd)
{
    if (!evenodd) return (size_t)lex;
    int V = X[0] * X[1] * X[2] * X[3];
    return (size_t)(lex >> 1) + (size_t)site_parity(X, lex) * (V / 2);
}

static inline void img_put(void *img, int fp64, size_t idx, cplx v)
{
    if (fp64) { ((double *)img)[2 * idx] = creal(v); ((double *)img)[2 * idx + 1] = cimag(v); }
    else { ((float *)img)[2 * idx] = (float)creal(v); ((float *)img)[2 * idx + 1] = (float)cimag(v); }
}
static inline cplx img_get(const void *img, int fp64, size_t idx)
{
    if (fp64) return ((const double *)img)[2 * idx] + I * ((const double *)img)[2 * idx + 1];
    return (double)((const float *)img)[2 * idx] + I * (double)((const float *)img)[2 * idx + 1];
}

void orc_pack(int N, const int X[4], const double *Ud, int layout, int evenodd, int fp64, void *img)
{
    const cplx *U = (const cplx *)Ud;
    int V = X[0] * X[1] * X[2] * X[3];
    size_t st = (size_t)4 * V;
    for (int lex = 0; lex < V; ++lex)
        for (int mu = 0; mu < 4; ++mu) {
            const cplx *A = LINK(U, N, lex, mu);
            size_t id = img_site(X, lex, evenodd) + (size_t)mu * V;
            if (layout == ORC_SOA) {
                for (int e = 0; e < N * N; ++e) img_put(img, fp64, id + e * st, A[e]);
            } else if (layout == ORC_SOA12) {
                for (int e = 0; e < 6; ++e) img_put(img, fp64, id + e * st, A[e]);
            } else {
                img_put(img, fp64, id, A[1]);
                img_put(img, fp64, id + st, A[2]);
                img_put(img, fp64, id + 2 * st, A[3]);
                img_put(img, fp64, id + 3 * st, carg(A[0]) + I * carg(A[6]));
            }
        }
}

/* SU(3) row 2 = conj(row0 x row1) -- restates reconstruct12p
 * (include/reconstruct_12p_8p.h:17-21). */
static void rebuild12(cplx *A)
{
    A[6] = conj(A[1] * A[5] - A[2] * A[4]);
    A[7] = conj(A[2] * A[3] - A[0] * A[5]);
    A[8] = conj(A[0] * A[4] - A[1] * A[3]);
}

/* SU(3) from e01, e02, e10 and the phases of e00, e20 -- restates
 * reconstruct8p (include/reconstruct_12p_8p.h:38-82).  With a = row 0,
 * b1 = e10, c1 = e20 and n = |a2|^2 + |a3|^2, unitarity and det = 1 give
 *   b2 = -(conj(a1) b1 a2 + conj(c1 a3)) / n,  b3 = (conj(c1 a2) - conj(a1) b1 a3) / n,
 *   c2 = (conj(b1 a3) - conj(a1) c1 a2) / n,   c3 = -(conj(b1 a2) + conj(a1) c1 a3) / n. */
static void rebuild8(cplx *A, double th0, double th2)
{
    double n = creal(A[1] * conj(A[1])) + creal(A[2] * conj(A[2]));
    double inv = 1.0 / n;
    double d = 1.0 - n;
    double m = sqrt(d >= 0 ? d : 0.0);
    A[0] = m * cos(th0) + I * (m * sin(th0));
    d = 1.0 - creal(A[0] * conj(A[0])) - creal(A[3] * conj(A[3]));
    m = sqrt(d >= 0 ? d : 0.0);
    A[6] = m * cos(th2) + I * (m * sin(th2));
    cplx a1 = A[0], a2 = A[1], a3 = A[2], b1 = A[3], c1 = A[6];
    A[4] = -(conj(a1) * b1 * a2 + conj(c1 * a3)) * inv;
    A[5] = (conj(c1 * a2) - conj(a1) * b1 * a3) * inv;
    A[7] = (conj(b1 * a3) - conj(a1) * c1 * a2) * inv;
    A[8] = -(conj(b1 * a2) + conj(a1) * c1 * a3) * inv;
}

void orc_unpack(int N, const int X[4], const void *img, int layout, int evenodd, int fp64, double *Ud)
{
    cplx *U = (cplx *)Ud;
    int V = X[0] * X[1] * X[2] * X[3];
    size_t st = (size_t)4 * V;
    for (int lex = 0; lex < V; ++lex)
        for (int mu = 0; mu < 4; ++mu) {
            cplx *A = U + ((size_t)lex * 4 + mu) * N * N;
            size_t id = img_site(X, lex, evenodd) + (size_t)mu * V;
            if (layout == ORC_SOA) {
                for (int e = 0; e < N * N; ++e) A[e] = img_get(img, fp64, id + e * st);
            } else if (layout == ORC_SOA12) {
                for (int e = 0; e < 6; ++e) A[e] = img_get(img, fp64, id + e * st);
                rebuild12(A);
            } else {
                A[1] = img_get(img, fp64, id);
                A[2] = img_get(img, fp64, id + st);
                A[3] = img_get(img, fp64, id + 2 * st);
                cplx th = img_get(img, fp64, id + 3 * st);
                rebuild8(A, creal(th), cimag(th));
            }
        }
}

/* ------------------------------------------------------------------------- */
/* Reference gauge file -- restates SaveBin_Gauge / ReadBin_Gauge
 * (src/io_gauge.cpp:429-583, 605-776).  Optional header: int32 grid[4], then
 * the leading sizeof(Real) bytes of the double beta (Real = the in-memory
 * precision of the saved array; header_fp64 selects it), then size_t
 * sizeof(save precision).  Body: sites t,z,y,x (x fastest), 4 directions,
 * N x N row-major complex in the save precision. */
int orc_save_bin(int N, const int X[4], const double *U, double beta, const char *path,
                 int save_fp64, int header_fp64, int with_header)
{
    FILE *f = fopen(path, "wb");
    if (!f) return -1;
    if (with_header) {
        int g[4] = {X[0], X[1], X[2], X[3]};
        fwrite(g, sizeof(int), 4, f);
        fwrite(&beta, header_fp64 ? 8 : 4, 1, f);
        size_t prec = save_fp64 ? 8 : 4;
        fwrite(&prec, sizeof(size_t), 1, f);
    }
    size_t n = (size_t)X[0] * X[1] * X[2] * X[3] * 4 * N * N * 2;
    int ok;
    if (save_fp64) ok = fwrite(U, sizeof(double), n, f) == n;
    else {
        float *tmp = malloc(n * sizeof(float));
        for (size_t i = 0; i < n; ++i) tmp[i] = (float)U[i];
        ok = fwrite(tmp, sizeof(float), n, f) == n;
        free(tmp);
    }
    fclose(f);
    return ok ? 0 : -2;
}

int orc_load_bin(int N, const int X[4], double *U, const char *path, int save_fp64,
                 int header_fp64, int with_header, int grid_out[4], double *beta_out)
{
    FILE *f = fopen(path, "rb");
    if (!f) return -1;
    if (with_header) {
        int g[4];
        double beta = 0;
        size_t prec = 0;
        if (fread(g, sizeof(int), 4, f) != 4) { fclose(f); return -2; }
        if (fread(&beta, header_fp64 ? 8 : 4, 1, f) != 1) { fclose(f); return -2; }
        if (fread(&prec, sizeof(size_t), 1, f) != 1) { fclose(f); return -2; }
        if (grid_out) memcpy(grid_out, g, sizeof g);
        if (beta_out) {
            if (header_fp64) *beta_out = beta;
            else { float fb; memcpy(&fb, &beta, 4); *beta_out = fb; }
        }
        if (prec != (size_t)(save_fp64 ? 8 : 4)) { fclose(f); return -3; }
    }
    size_t n = (size_t)X[0] * X[1] * X[2] * X[3] * 4 * N * N * 2;
    int ok;
    if (save_fp64) ok = fread(U, sizeof(double), n, f) == n;
    else {
        float *tmp = malloc(n * sizeof(float));
        ok = fread(tmp, sizeof(float), n, f) == n;
        for (size_t i = 0; ok && i < n; ++i) U[i] = tmp[i];
        free(tmp);
    }
    fclose(f);
    return ok ? 0 : -2;
}

/* smearing and multihit share this file's helpers */
#include "sun_oracle_smear.inc"
