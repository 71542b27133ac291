// sun_core.cuh -- counter-based random numbers, lattice geometry, the
// device link layouts and the per-link Monte Carlo updates of the engine.
#pragma once
#include "sun_math.cuh"

namespace sunb {

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), written from the
// published round function: per round
//   (c0,c1,c2,c3) <- (hi(M1*c2) ^ c1 ^ k0, lo(M1*c2), hi(M0*c0) ^ c3 ^ k1, lo(M0*c0))
// with M0 = 0xD2511F53, M1 = 0xCD9E8D57 and the key bumped by the Weyl
// constants (0x9E3779B9, 0xBB67AE85) between rounds.
SUN_HD void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
#ifdef __CUDA_ARCH__
        uint32_t hi0 = __umulhi(0xD2511F53u, c[0]), lo0 = 0xD2511F53u * c[0];
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c[2]), lo1 = 0xCD9E8D57u * c[2];
#else
        uint64_t p0 = (uint64_t)0xD2511F53u * c[0], p1 = (uint64_t)0xCD9E8D57u * c[2];
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
#endif
        uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
}

// Stream of uniforms of one link: Philox words from counter
// (block, lex_site, mu | purpose << 8, pass), key = seed.  FP32: one word per
// uniform, u = ((w >> 8) + 1) 2^-24 in (0,1].  FP64: two words a,b per
// uniform, u = ((((a >> 11) << 32) | b) + 1) 2^-53 in (0,1].
template <class R> struct PhiloxStream {
    uint32_t k0, k1, c1, c2, c3, blk;
    uint32_t buf[4];
    int pos;
    SUN_DEV void init(uint64_t seed, uint32_t lex, uint32_t mu_purpose, uint32_t pass)
    {
        k0 = (uint32_t)seed; k1 = (uint32_t)(seed >> 32);
        c1 = lex; c2 = mu_purpose; c3 = pass; blk = 0; pos = 4;
    }
    SUN_DEV uint32_t word()
    {
        if (pos == 4) {
            buf[0] = blk; buf[1] = c1; buf[2] = c2; buf[3] = c3;
            philox4x32_10(buf, k0, k1);
            ++blk;
            pos = 0;
        }
        uint32_t w = buf[0];
        // rotate so the next word is always buf[0] (keeps buf in registers)
        buf[0] = buf[1]; buf[1] = buf[2]; buf[2] = buf[3];
        ++pos;
        return w;
    }
    SUN_DEV R uniform();
};
// uniforms from a stream's words (FP32: one word, FP64: two)
template <class R> struct WordsToUniform;
template <> struct WordsToUniform<float> {
    template <class S> static SUN_DEV float get(S& s)
    {
        uint32_t w = s.word();
        return (float)((w >> 8) + 1u) * 5.9604644775390625e-08f;
    }
};
template <> struct WordsToUniform<double> {
    template <class S> static SUN_DEV double get(S& s)
    {
        uint32_t a = s.word();
        uint32_t b = s.word();
        uint64_t k = ((uint64_t)(a >> 11) << 32) | (uint64_t)b;
        return (double)(k + 1ull) * 1.1102230246251565e-16;
    }
};
template <class R> SUN_DEV R PhiloxStream<R>::uniform() { return WordsToUniform<R>::get(*this); }

// Uniforms read from a caller buffer (oracle-parity mode); running out sets
// an error flag and returns 0.5.
template <class R> struct InjectedStream {
    const double* p;
    int left;
    int* err;
    SUN_DEV R uniform()
    {
        if (left <= 0) { if (err) atomicOr(err, 1); return R(0.5); }
        --left;
        return (R)(*p++);
    }
};

// ---------------------------------------------------------------------------
// SU(2) heatbath draw -- generate_su2_matrix_milc
// (include/device_PHB_OVR.h:163-223): a first Kennedy-Pendleton try, then up
// to 20 more KP tries (alpha > 2) or up to 20 Creutz tries (alpha <= 2), then
// a random direction.  Draw order: xr1, xr2, xr3, xr4 per KP try, xr1, xr2
// per Creutz try, then one uniform for a3 and one for the azimuth.
template <class R> struct MathFns;
// FP32 draws use the hardware approximations (absolute error ~1e-6 on these
// arguments, below the FP32 storage rounding of the links they feed); the
// angle 2 pi u is shifted into [-pi, pi], where __sincosf is accurate:
// cos(2 pi u) = -cos(2 pi (u - 1/2)), sin(2 pi u) = -sin(2 pi (u - 1/2)).
template <> struct MathFns<float> {
    static SUN_DEV float log_(float x) { return __logf(x); }
    static SUN_DEV float exp_(float x) { return __expf(x); }
    static SUN_DEV float sqrt_(float x) { return sqrtf(x); }
    static SUN_DEV void sincos2pi(float u, float* s, float* c)
    {
        float ss, cc;
        __sincosf(6.28318530717958648f * (u - 0.5f), &ss, &cc);
        *s = -ss;
        *c = -cc;
    }
    static SUN_DEV float cos2pi(float u) { return -__cosf(6.28318530717958648f * (u - 0.5f)); }
};
template <> struct MathFns<double> {
    static SUN_DEV double log_(double x) { return log(x); }
    static SUN_DEV double exp_(double x) { return exp(x); }
    static SUN_DEV double sqrt_(double x) { return sqrt(x); }
    static SUN_DEV void sincos2pi(double u, double* s, double* c) { sincospi(2.0 * u, s, c); }
    static SUN_DEV double cos2pi(double u) { return cospi(2.0 * u); }
};

template <class R, class Stream> SUN_DEV void su2_heatbath_draw(R al, Stream& st, R a[4])
{
    typedef MathFns<R> M;
    const R tiny = R(1.e-10);
    R xr1 = M::log_(st.uniform() + tiny);
    R xr2 = M::log_(st.uniform() + tiny);
    R xr3 = M::cos2pi(st.uniform());
    R xr4 = st.uniform();
    R d = -fma(xr1 * xr3, xr3, xr2) / al;
    bool accepted = fma(R(-0.5), d, R(1)) > xr4 * xr4;
    if (!accepted) {
        if (al > R(2)) {
            for (int k = 0; k < 20; ++k) {
                xr1 = M::log_(st.uniform() + tiny);
                xr2 = M::log_(st.uniform() + tiny);
                xr3 = M::cos2pi(st.uniform());
                xr4 = st.uniform();
                d = -fma(xr1 * xr3, xr3, xr2) / al;
                if (fma(R(-0.5), d, R(1)) > xr4 * xr4) break;
            }
        } else {
            const R e = M::exp_(R(-2) * al);
            const R w = R(1) - e;
            R a0 = R(0);
            for (int k = 0; k < 20; ++k) {
                R u1 = st.uniform();
                R u2 = st.uniform();
                a0 = R(1) + M::log_(fma(w, u1, e)) / al;
                if (fma(-a0, a0, R(1)) > u2 * u2) break;
            }
            d = R(1) - a0;
        }
    }
    R a0 = R(1) - d;
    R rr = fabs(fma(-a0, a0, R(1)));
    a[0] = a0;
    a[3] = fma(R(2), st.uniform(), R(-1)) * M::sqrt_(rr);
    R x1 = M::sqrt_(fabs(fma(-a[3], a[3], rr)));
    R s, c;
    M::sincos2pi(st.uniform(), &s, &c);
    a[1] = x1 * c;
    a[2] = x1 * s;
}

// Arithmetic of the SU(2) draw in FP32 updates (SUN_F32_DRAW): 0 FP32 with
// the hardware log / exp / sincos approximations; 1 FP64 arithmetic on the
// same 24-bit uniforms (the accept/reject tests then see only the FP32
// rounding of alpha, not that of the transcendentals).
#ifndef SUN_F32_DRAW
#define SUN_F32_DRAW 0
#endif
template <class Stream> struct WideStream {
    Stream& s;
    SUN_DEV double uniform() { return (double)s.uniform(); }
};
template <class R, class Stream> SUN_DEV void su2_draw(R al, Stream& st, R a[4])
{
    if constexpr (sizeof(R) == 4 && SUN_F32_DRAW == 1) {
        WideStream<Stream> w{st};
        double ad[4];
        su2_heatbath_draw<double>((double)al, w, ad);
        a[0] = (R)ad[0]; a[1] = (R)ad[1]; a[2] = (R)ad[2]; a[3] = (R)ad[3];
    } else {
        su2_heatbath_draw<R>(al, st, a);
    }
}

// Cabibbo-Marinari pseudo-heatbath of U against the staple sum S (F = S^dag)
// -- heatBathSUN (include/device_PHB_OVR.h:362-485).  SU(3) recomputes each
// block from U and S like the reference; N >= 4 does the same (the
// reference keeps M = U S^dagger and updates it with U, which needs N^2 more
// live complex numbers); N = 2 keeps M.
// ROW2 false (SU(3) 12-parameter links, whose row 2 is not stored): the
// last subgroup, (0, 2), rotates row 0 only and row 2 is left as it was.
template <int N, class R, class Stream, bool ROW2 = true>
SUN_DEV void heatbath_update(Mat<N, R>& U, const Mat<N, R>& S, R beta_over_n, Stream& st)
{
    if constexpr (N == 3) {
        // one copy of the (large) SU(2) draw in a rolled loop over the three
        // subgroups; the block extraction and row update switch on the
        // subgroup so the matrices keep static (register) indexing
#pragma unroll 1
        for (int b = 0; b < 3; ++b) {
            R r[4], a[4], c[4];
            if (b == 0) su2_block_US<N, R>(U, S, 0, 1, r);
            else if (b == 1) su2_block_US<N, R>(U, S, 1, 2, r);
            else su2_block_US<N, R>(U, S, 0, 2, r);
            R k = sqrt(qnorm2(r));
            R ap = beta_over_n * k;
            k = R(1) / k;
            r[0] *= k; r[1] *= k; r[2] *= k; r[3] *= k;
            su2_draw<R>(ap, st, a);
            su2_mul_udag(a, r, c);
            if (b == 0) su2_apply<N, R>(U, 0, 1, c);
            else if (b == 1) su2_apply<N, R>(U, 1, 2, c);
            else if (ROW2) su2_apply<N, R>(U, 0, 2, c);
            else su2_apply_row_p<N, R>(U, 0, 2, c);
        }
    } else if constexpr (N >= 4) {
        // each block of U S^dagger recomputed from U and S instead of
        // keeping M = U S^dagger (N^2 fewer live complex numbers, no N^3
        // product up front; the same values up to rounding), one rolled copy
        // of the draw
#pragma unroll 1
        for (int b = 0; b < SubGroup<N>::count; ++b) {
            R r[4], a[4], c[4];
            with_subgroup<N>(b, [&](auto P, auto Q) { su2_block_US<N, R>(U, S, P(), Q(), r); });
            R k = sqrt(qnorm2(r));
            R ap = beta_over_n * k;
            k = R(1) / k;
            r[0] *= k; r[1] *= k; r[2] *= k; r[3] *= k;
            su2_draw<R>(ap, st, a);
            su2_mul_udag(a, r, c);
            with_subgroup<N>(b, [&](auto P, auto Q) { su2_apply<N, R>(U, P(), Q(), c); });
        }
    } else {
        Mat<N, R> M;
        mmul_nd<N, R>(U, S, M);
#pragma unroll
        for (int b = 0; b < SubGroup<N>::count; ++b) {
            const int p = SubGroup<N>::p(b), q = SubGroup<N>::q(b);
            R r[4], a[4], c[4];
            su2_block<N, R>(M, p, q, r);
            R k = sqrt(qnorm2(r));
            R ap = beta_over_n * k;
            k = R(1) / k;
            r[0] *= k; r[1] *= k; r[2] *= k; r[3] *= k;
            su2_draw<R>(ap, st, a);
            su2_mul_udag(a, r, c);
            su2_apply<N, R>(U, p, q, c);
            su2_apply<N, R>(M, p, q, c);
        }
    }
}

// Microcanonical overrelaxation -- overrelaxationSUN
// (include/device_PHB_OVR.h:494-608): per subgroup the conj-normalised block
// element a is applied twice.  Here its square is applied once: for the
// quaternion a = (a0, a1, a2, a3), a a = (a0^2 - |a_vec|^2, 2 a0 a_vec), the
// same SU(2) element with half the row arithmetic.
template <class R> SUN_DEV void su2_overrelax_element(const R r[4], R c[4])
{
    const R n2 = qnorm2(r);
    const R inv = R(1) / n2;
    // a = (r0, -r1, -r2, -r3)/|r|  ->  a^2 = ((r0^2 - |r_vec|^2), -2 r0 r_vec) / |r|^2
    const R t = R(-2) * r[0] * inv;
    c[0] = fma(r[0], r[0], -fma(r[3], r[3], fma(r[2], r[2], r[1] * r[1]))) * inv;
    c[1] = t * r[1];
    c[2] = t * r[2];
    c[3] = t * r[3];
}

// ROW2: as in heatbath_update.
template <int N, class R, bool ROW2 = true> SUN_DEV void overrelax_update(Mat<N, R>& U, const Mat<N, R>& S)
{
    if constexpr (N >= 3) {
        // blocks recomputed from U and S (for N >= 4 instead of the
        // reference's M = U S^dagger: the same values up to rounding)
#pragma unroll
        for (int b = 0; b < SubGroup<N>::count; ++b) {
            const int p = SubGroup<N>::p(b), q = SubGroup<N>::q(b);
            R r[4], c[4];
            su2_block_US<N, R>(U, S, p, q, r);
            su2_overrelax_element(r, c);
            if (ROW2 || N != 3 || b + 1 < SubGroup<N>::count) su2_apply<N, R>(U, p, q, c);
            else su2_apply_row_p<N, R>(U, p, q, c);
        }
    } else {
        Mat<N, R> M;
        mmul_nd<N, R>(U, S, M);
#pragma unroll
        for (int b = 0; b < SubGroup<N>::count; ++b) {
            const int p = SubGroup<N>::p(b), q = SubGroup<N>::q(b);
            R r[4], c[4];
            su2_block<N, R>(M, p, q, r);
            su2_overrelax_element(r, c);
            su2_apply<N, R>(U, p, q, c);
            su2_apply<N, R>(M, p, q, c);
        }
    }
}

// ---------------------------------------------------------------------------
// Geometry.  Canonical site index lex = x + X0 (y + X1 (z + X2 t)); even/odd
// index (lex >> 1) + parity V/2 (index.h:133-244; needs X0 even).
struct Geom {
    int X[4];
    int V, halfV;
};

SUN_DEV int lex_of(const Geom& g, const int x[4])
{
    return ((x[3] * g.X[2] + x[2]) * g.X[1] + x[1]) * g.X[0] + x[0];
}
SUN_DEV int eo_of(const Geom& g, const int x[4])
{
    return (lex_of(g, x) >> 1) + ((x[0] + x[1] + x[2] + x[3]) & 1) * g.halfV;
}
template <bool EO> SUN_DEV int site_of(const Geom& g, const int x[4])
{
    return EO ? eo_of(g, x) : lex_of(g, x);
}
// coordinates of half-site id of the given parity -- Index_4D_EO (index.h:133)
SUN_DEV void eo_coords(const Geom& g, int id, int parity, int x[4])
{
    int hx = g.X[0] >> 1;
    int za = id / hx;
    int zb = za / g.X[1];
    x[1] = za - zb * g.X[1];
    x[3] = zb / g.X[2];
    x[2] = zb - x[3] * g.X[2];
    int xodd = (x[1] + x[2] + x[3] + parity) & 1;
    x[0] = 2 * id + xodd - za * g.X[0];
}
SUN_DEV void lex_coords(const Geom& g, int lex, int x[4])
{
    int a = lex / g.X[0];
    x[0] = lex - a * g.X[0];
    int b = a / g.X[1];
    x[1] = a - b * g.X[1];
    x[3] = b / g.X[2];
    x[2] = b - x[3] * g.X[2];
}
SUN_DEV int wrap_up(int v, int L) { return v + 1 == L ? 0 : v + 1; }
SUN_DEV int wrap_dn(int v, int L) { return v == 0 ? L - 1 : v - 1; }

// ---------------------------------------------------------------------------
// Link layouts of the device image -- the SoA addressing of GAUGE_SAVE /
// GAUGE_LOAD (include/device_load_save.h:77-289): complex element e of link
// (site s, mu) at s + mu V + e 4V.  SOA: N*N row-major; SOA12 (SU(3)): rows
// 0,1, row 2 rebuilt in registers; SOA8 (SU(3)): e01, e02, e10 and
// (arg e00, arg e20).
enum Layout { L_SOA = 0, L_SOA12 = 1, L_SOA8 = 2 };

template <int N, int LAYOUT> struct LayoutInfo {
    static constexpr int elems = LAYOUT == L_SOA12 ? 6 : (LAYOUT == L_SOA8 ? 4 : N * N);
};

template <class R> struct Vec2;
template <> struct Vec2<float> { typedef float2 T; };
template <> struct Vec2<double> { typedef double2 T; };

// Load paths of a link element: LD_CA plain (coherent, L1-cached), LD_NC the
// read-only path (data constant for the kernel's lifetime), LD_CG L2 only.
// The update kernels, which overlap the previous phase's launch, read
// through L2 only: lines an SM's L1 held across the overlap were seen stale.
enum { LD_CA = 0, LD_NC = 1, LD_CG = 2 };
template <class R, int P> SUN_DEV cx<R> ld_elem(const cx<R>* p)
{
    typedef typename Vec2<R>::T V2;
    V2 v;
    if (P == LD_NC) v = __ldg(reinterpret_cast<const V2*>(p));
    else if (P == LD_CG) v = __ldcg(reinterpret_cast<const V2*>(p));
    else v = *reinterpret_cast<const V2*>(p);
    return mkc<R>(v.x, v.y);
}
template <class R> SUN_DEV void st_elem(cx<R>* p, cx<R> c)
{
    typedef typename Vec2<R>::T V2;
    V2 v;
    v.x = c.re; v.y = c.im;
    *reinterpret_cast<V2*>(p) = v;
}

// SU(3) from e01, e02, e10 and the phases of e00, e20 -- reconstruct8p
// (include/reconstruct_12p_8p.h:38-82).  With a = row 0, b1 = e10, c1 = e20
// and n = |a2|^2 + |a3|^2, unitarity and det = 1 give
//   b2 = -(conj(a1) b1 a2 + conj(c1 a3)) / n,  b3 = (conj(c1 a2) - conj(a1) b1 a3) / n,
//   c2 = (conj(b1 a3) - conj(a1) c1 a2) / n,   c3 = -(conj(b1 a2) + conj(a1) c1 a3) / n.
template <class R> SUN_DEV void rebuild8(Mat<3, R>& A, R th0, R th2)
{
    R n = cnorm2(A.e[0][1]) + cnorm2(A.e[0][2]);
    R inv = R(1) / n;
    R d = R(1) - n;
    R m = sqrt(d >= R(0) ? d : R(0));
    R s, c;
    sincos(th0, &s, &c);
    A.e[0][0] = mkc(m * c, m * s);
    d = R(1) - cnorm2(A.e[0][0]) - cnorm2(A.e[1][0]);
    m = sqrt(d >= R(0) ? d : R(0));
    sincos(th2, &s, &c);
    A.e[2][0] = mkc(m * c, m * s);
    const cx<R> a1 = A.e[0][0], a2 = A.e[0][1], a3 = A.e[0][2], b1 = A.e[1][0], c1 = A.e[2][0];
    const cx<R> ca1b1 = cconj(a1) * b1, ca1c1 = cconj(a1) * c1;
    A.e[1][1] = (R(-1) * inv) * (ca1b1 * a2 + cconj(c1 * a3));
    A.e[1][2] = inv * (cconj(c1 * a2) - ca1b1 * a3);
    A.e[2][1] = inv * (cconj(b1 * a3) - ca1c1 * a2);
    A.e[2][2] = (R(-1) * inv) * (cconj(b1 * a2) + ca1c1 * a3);
}

template <int N, class R, int LAYOUT> struct LinkIO {
    static constexpr int NE = LayoutInfo<N, LAYOUT>::elems;
    // SOA12: the two stored rows only, row 2 left unset
    template <int NC> static SUN_DEV void load_rows(const cx<R>* base, uint32_t idx, uint32_t stride, Mat<N, R>& A)
    {
        static_assert(LAYOUT == L_SOA12, "stored rows exist for SOA12 only");
#pragma unroll
        for (int e = 0; e < 6; ++e) A.e[e / 3][e % 3] = ld_elem<R, NC>(base + idx + e * stride);
    }
    template <int NC> static SUN_DEV void load(const cx<R>* base, uint32_t idx, uint32_t stride, Mat<N, R>& A)
    {
        if constexpr (LAYOUT == L_SOA) {
#pragma unroll
            for (int e = 0; e < N * N; ++e) A.e[e / N][e % N] = ld_elem<R, NC>(base + idx + e * stride);
        } else if constexpr (LAYOUT == L_SOA12) {
#pragma unroll
            for (int e = 0; e < 6; ++e) A.e[e / 3][e % 3] = ld_elem<R, NC>(base + idx + e * stride);
            rebuild12<R>(A);
        } else {
            A.e[0][1] = ld_elem<R, NC>(base + idx);
            A.e[0][2] = ld_elem<R, NC>(base + idx + stride);
            A.e[1][0] = ld_elem<R, NC>(base + idx + 2 * stride);
            cx<R> th = ld_elem<R, NC>(base + idx + 3 * stride);
            rebuild8<R>(A, th.re, th.im);
        }
    }
    // the same loads and store through element accessors: f(idx, e) returns
    // element e of the link at image index idx (complex element
    // idx + e stride of the image), w(idx, e, v) writes it
    template <class F> static SUN_DEV void load_rows_f(F&& f, uint32_t idx, uint32_t stride, Mat<N, R>& A)
    {
        static_assert(LAYOUT == L_SOA12, "stored rows exist for SOA12 only");
#pragma unroll
        for (int e = 0; e < 6; ++e) A.e[e / 3][e % 3] = f(idx, e);
    }
    template <class F> static SUN_DEV void load_f(F&& f, uint32_t idx, uint32_t stride, Mat<N, R>& A)
    {
        if constexpr (LAYOUT == L_SOA) {
#pragma unroll
            for (int e = 0; e < N * N; ++e) A.e[e / N][e % N] = f(idx, e);
        } else if constexpr (LAYOUT == L_SOA12) {
#pragma unroll
            for (int e = 0; e < 6; ++e) A.e[e / 3][e % 3] = f(idx, e);
            rebuild12<R>(A);
        } else {
            A.e[0][1] = f(idx, 0);
            A.e[0][2] = f(idx, 1);
            A.e[1][0] = f(idx, 2);
            cx<R> th = f(idx, 3);
            rebuild8<R>(A, th.re, th.im);
        }
    }
    template <class W> static SUN_DEV void store_f(W&& w, uint32_t idx, uint32_t stride, const Mat<N, R>& A)
    {
        if constexpr (LAYOUT == L_SOA) {
#pragma unroll
            for (int e = 0; e < N * N; ++e) w(idx, e, A.e[e / N][e % N]);
        } else if constexpr (LAYOUT == L_SOA12) {
#pragma unroll
            for (int e = 0; e < 6; ++e) w(idx, e, A.e[e / 3][e % 3]);
        } else {
            w(idx, 0, A.e[0][1]);
            w(idx, 1, A.e[0][2]);
            w(idx, 2, A.e[1][0]);
            w(idx, 3, mkc<R>(atan2(A.e[0][0].im, A.e[0][0].re), atan2(A.e[2][0].im, A.e[2][0].re)));
        }
    }
    static SUN_DEV void store(cx<R>* base, uint32_t idx, uint32_t stride, const Mat<N, R>& A)
    {
        if constexpr (LAYOUT == L_SOA) {
#pragma unroll
            for (int e = 0; e < N * N; ++e) st_elem<R>(base + idx + e * stride, A.e[e / N][e % N]);
        } else if constexpr (LAYOUT == L_SOA12) {
#pragma unroll
            for (int e = 0; e < 6; ++e) st_elem<R>(base + idx + e * stride, A.e[e / 3][e % 3]);
        } else {
            st_elem<R>(base + idx, A.e[0][1]);
            st_elem<R>(base + idx + stride, A.e[0][2]);
            st_elem<R>(base + idx + 2 * stride, A.e[1][0]);
            st_elem<R>(base + idx + 3 * stride,
                       mkc<R>(atan2(A.e[0][0].im, A.e[0][0].re), atan2(A.e[2][0].im, A.e[2][0].re)));
        }
    }
};

}  // namespace sunb
