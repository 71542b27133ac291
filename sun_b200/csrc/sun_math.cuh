// sun_math.cuh -- register-resident complex and SU(N) matrix algebra for the
// B200 engine.  Everything here is __forceinline__ and fully unrolled over N
// so that a link lives in registers; there is no local-memory matrix type.
//
// The algebra is the textbook one; where an operation restates a specific
// reference routine the reference file:line is given (paths relative to the
// nmrcardoso/sun project root).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#define SUN_DEV __device__ __forceinline__
#define SUN_HD __host__ __device__ __forceinline__

namespace sunb {

template <class R> struct cx { R re, im; };

template <class R> SUN_HD cx<R> mkc(R a, R b) { cx<R> c; c.re = a; c.im = b; return c; }
template <class R> SUN_HD cx<R> operator+(cx<R> a, cx<R> b) { return mkc(a.re + b.re, a.im + b.im); }
template <class R> SUN_HD cx<R> operator-(cx<R> a, cx<R> b) { return mkc(a.re - b.re, a.im - b.im); }
// The library is compiled without implicit multiply-add contraction
// (-fmad=false): every fused operation is written out as fma(), so each
// kernel rounds exactly as its source says and kernels that perform the same
// operations give the same bits, whatever the compiler does around them.
template <class R> SUN_HD cx<R> operator*(cx<R> a, cx<R> b)
{
    return mkc(fma(a.re, b.re, -(a.im * b.im)), fma(a.re, b.im, a.im * b.re));
}
template <class R> SUN_HD cx<R> operator*(R s, cx<R> a) { return mkc(s * a.re, s * a.im); }
template <class R> SUN_HD cx<R> cconj(cx<R> a) { return mkc(a.re, -a.im); }
template <class R> SUN_HD R cnorm2(cx<R> a) { return fma(a.re, a.re, a.im * a.im); }
// |r|^2 of a quaternion 4-vector
template <class R> SUN_HD R qnorm2(const R r[4]) { return fma(r[3], r[3], fma(r[2], r[2], fma(r[1], r[1], r[0] * r[0]))); }
// acc + a*b, acc + conj(a)*b, acc + a*conj(b) as FMA chains
template <class R> SUN_HD cx<R> cfma(cx<R> a, cx<R> b, cx<R> acc)
{
    acc.re = fma(a.re, b.re, acc.re); acc.re = fma(-a.im, b.im, acc.re);
    acc.im = fma(a.re, b.im, acc.im); acc.im = fma(a.im, b.re, acc.im);
    return acc;
}
template <class R> SUN_HD cx<R> cfma_cn(cx<R> a, cx<R> b, cx<R> acc)  // acc + conj(a) b
{
    acc.re = fma(a.re, b.re, acc.re); acc.re = fma(a.im, b.im, acc.re);
    acc.im = fma(a.re, b.im, acc.im); acc.im = fma(-a.im, b.re, acc.im);
    return acc;
}
template <class R> SUN_HD cx<R> cfma_nc(cx<R> a, cx<R> b, cx<R> acc)  // acc + a conj(b)
{
    acc.re = fma(a.re, b.re, acc.re); acc.re = fma(a.im, b.im, acc.re);
    acc.im = fma(a.im, b.re, acc.im); acc.im = fma(-a.re, b.im, acc.im);
    return acc;
}

// conj(p q - r s), each component one chain of a product and three FMAs
// (the 12-parameter third row: 8 operations per element against 10 for two
// products and a difference)
template <class R> SUN_HD cx<R> conj_det2(cx<R> p, cx<R> q, cx<R> r, cx<R> s)
{
    const R re = fma(p.re, q.re, fma(-p.im, q.im, fma(-r.re, s.re, r.im * s.im)));
    const R im = fma(-p.re, q.im, fma(-p.im, q.re, fma(r.re, s.im, r.im * s.re)));
    return mkc(re, im);
}

template <int N, class R> struct Mat { cx<R> e[N][N]; };

template <int N, class R> SUN_HD void mzero(Mat<N, R>& A)
{
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) A.e[i][j] = mkc<R>(0, 0);
}
template <int N, class R> SUN_HD void munit(Mat<N, R>& A)
{
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) A.e[i][j] = mkc<R>(i == j ? R(1) : R(0), 0);
}
// C = A B
template <int N, class R> SUN_HD void mmul(const Mat<N, R>& A, const Mat<N, R>& B, Mat<N, R>& C)
{
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) {
            cx<R> s = A.e[i][0] * B.e[0][j];
#pragma unroll
            for (int k = 1; k < N; ++k) s = cfma(A.e[i][k], B.e[k][j], s);
            C.e[i][j] = s;
        }
}
// C = A B^dagger
template <int N, class R> SUN_HD void mmul_nd(const Mat<N, R>& A, const Mat<N, R>& B, Mat<N, R>& C)
{
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) {
            cx<R> s = mkc<R>(0, 0);
#pragma unroll
            for (int k = 0; k < N; ++k) s = cfma_nc(A.e[i][k], B.e[j][k], s);
            C.e[i][j] = s;
        }
}
// C = A^dagger B
template <int N, class R> SUN_HD void mmul_dn(const Mat<N, R>& A, const Mat<N, R>& B, Mat<N, R>& C)
{
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) {
            cx<R> s = mkc<R>(0, 0);
#pragma unroll
            for (int k = 0; k < N; ++k) s = cfma_cn(A.e[k][i], B.e[k][j], s);
            C.e[i][j] = s;
        }
}
// S += A B^dagger
template <int N, class R> SUN_HD void macc_nd(const Mat<N, R>& A, const Mat<N, R>& B, Mat<N, R>& S)
{
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) {
            cx<R> s = S.e[i][j];
#pragma unroll
            for (int k = 0; k < N; ++k) s = cfma_nc(A.e[i][k], B.e[j][k], s);
            S.e[i][j] = s;
        }
}
// S += A B
template <int N, class R> SUN_HD void macc(const Mat<N, R>& A, const Mat<N, R>& B, Mat<N, R>& S)
{
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) {
            cx<R> s = S.e[i][j];
#pragma unroll
            for (int k = 0; k < N; ++k) s = cfma(A.e[i][k], B.e[k][j], s);
            S.e[i][j] = s;
        }
}
// S += A^dagger B
template <int N, class R> SUN_HD void macc_dn(const Mat<N, R>& A, const Mat<N, R>& B, Mat<N, R>& S)
{
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) {
            cx<R> s = S.e[i][j];
#pragma unroll
            for (int k = 0; k < N; ++k) s = cfma_cn(A.e[k][i], B.e[k][j], s);
            S.e[i][j] = s;
        }
}
// rows 0 and 1 of C = A B (only rows 0, 1 of A are read)
template <class R> SUN_HD void mmul_rows01(const Mat<3, R>& A, const Mat<3, R>& B, Mat<3, R>& C)
{
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            cx<R> s = A.e[i][0] * B.e[0][j];
            s = cfma(A.e[i][1], B.e[1][j], s);
            s = cfma(A.e[i][2], B.e[2][j], s);
            C.e[i][j] = s;
        }
}
// rows 0 and 1 of C = A B^dagger (only rows 0, 1 of A are read)
template <class R> SUN_HD void mmul_nd_rows01(const Mat<3, R>& A, const Mat<3, R>& B, Mat<3, R>& C)
{
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            cx<R> s = mkc<R>(0, 0);
#pragma unroll
            for (int k = 0; k < 3; ++k) s = cfma_nc(A.e[i][k], B.e[j][k], s);
            C.e[i][j] = s;
        }
}
// S += P
template <int N, class R> SUN_HD void madd(Mat<N, R>& S, const Mat<N, R>& P)
{
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) S.e[i][j] = S.e[i][j] + P.e[i][j];
}
// -- one row of the products above, for kernels that spread a matrix over N
// lanes (lane i owns row i).  Element (i, j) is formed by exactly the same
// operations, in the same order, as in the whole-matrix routine it names, so
// the two give the same bits.
// row r (runtime) of the first ROWS rows of A, by selects (no local memory)
template <int N, class R, int ROWS = N> SUN_DEV void mrow(const Mat<N, R>& A, int r, cx<R> out[N])
{
#pragma unroll
    for (int j = 0; j < N; ++j) {
        cx<R> v = A.e[0][j];
#pragma unroll
        for (int i = 1; i < ROWS; ++i)
            if (r == i) v = A.e[i][j];
        out[j] = v;
    }
}
// column c (runtime) of A
template <int N, class R> SUN_DEV void mcol(const Mat<N, R>& A, int c, cx<R> out[N])
{
#pragma unroll
    for (int k = 0; k < N; ++k) {
        cx<R> v = A.e[k][0];
#pragma unroll
        for (int i = 1; i < N; ++i)
            if (c == i) v = A.e[k][i];
        out[k] = v;
    }
}
// row of A B from the row a of A -- mmul (and mmul_rows01)
template <int N, class R> SUN_DEV void rmul(const cx<R> a[N], const Mat<N, R>& B, cx<R> c[N])
{
#pragma unroll
    for (int j = 0; j < N; ++j) {
        cx<R> s = a[0] * B.e[0][j];
#pragma unroll
        for (int k = 1; k < N; ++k) s = cfma(a[k], B.e[k][j], s);
        c[j] = s;
    }
}
// row i of A B^dagger from row i of A (a) -- mmul_nd, mmul_nd_rows01
template <int N, class R> SUN_DEV void rmul_nd(const cx<R> a[N], const Mat<N, R>& B, cx<R> c[N])
{
#pragma unroll
    for (int j = 0; j < N; ++j) {
        cx<R> s = mkc<R>(0, 0);
#pragma unroll
        for (int k = 0; k < N; ++k) s = cfma_nc(a[k], B.e[j][k], s);
        c[j] = s;
    }
}
// row i of A^dagger B from column i of A (a) -- mmul_dn
template <int N, class R> SUN_DEV void rmul_dn(const cx<R> a[N], const Mat<N, R>& B, cx<R> c[N])
{
#pragma unroll
    for (int j = 0; j < N; ++j) {
        cx<R> s = mkc<R>(0, 0);
#pragma unroll
        for (int k = 0; k < N; ++k) s = cfma_cn(a[k], B.e[k][j], s);
        c[j] = s;
    }
}
// row of S += A B^dagger from the row a of A -- macc_nd
template <int N, class R> SUN_DEV void racc_nd(const cx<R> a[N], const Mat<N, R>& B, cx<R> s[N])
{
#pragma unroll
    for (int j = 0; j < N; ++j) {
        cx<R> t = s[j];
#pragma unroll
        for (int k = 0; k < N; ++k) t = cfma_nc(a[k], B.e[j][k], t);
        s[j] = t;
    }
}
// row of S += A B from the row a of A -- macc
template <int N, class R> SUN_DEV void racc(const cx<R> a[N], const Mat<N, R>& B, cx<R> s[N])
{
#pragma unroll
    for (int j = 0; j < N; ++j) {
        cx<R> t = s[j];
#pragma unroll
        for (int k = 0; k < N; ++k) t = cfma(a[k], B.e[k][j], t);
        s[j] = t;
    }
}
// row i of S += A^dagger B from column i of A (a) -- macc_dn
template <int N, class R> SUN_DEV void racc_dn(const cx<R> a[N], const Mat<N, R>& B, cx<R> s[N])
{
#pragma unroll
    for (int j = 0; j < N; ++j) {
        cx<R> t = s[j];
#pragma unroll
        for (int k = 0; k < N; ++k) t = cfma_cn(a[k], B.e[k][j], t);
        s[j] = t;
    }
}
// The same four row routines with the right factor B read through an
// accessor B(k, j) (e.g. a matrix staged in shared memory): the same
// operations in the same order, so the same bits.
template <int N, class R, class G> SUN_DEV void rmul_g(const cx<R> a[N], G&& B, cx<R> c[N])
{
#pragma unroll
    for (int j = 0; j < N; ++j) {
        cx<R> s = a[0] * B(0, j);
#pragma unroll
        for (int k = 1; k < N; ++k) s = cfma(a[k], B(k, j), s);
        c[j] = s;
    }
}
template <int N, class R, class G> SUN_DEV void rmul_dn_g(const cx<R> a[N], G&& B, cx<R> c[N])
{
#pragma unroll
    for (int j = 0; j < N; ++j) {
        cx<R> s = mkc<R>(0, 0);
#pragma unroll
        for (int k = 0; k < N; ++k) s = cfma_cn(a[k], B(k, j), s);
        c[j] = s;
    }
}
template <int N, class R, class G> SUN_DEV void racc_nd_g(const cx<R> a[N], G&& B, cx<R> s[N])
{
#pragma unroll
    for (int j = 0; j < N; ++j) {
        cx<R> t = s[j];
#pragma unroll
        for (int k = 0; k < N; ++k) t = cfma_nc(a[k], B(j, k), t);
        s[j] = t;
    }
}
template <int N, class R, class G> SUN_DEV void racc_g(const cx<R> a[N], G&& B, cx<R> s[N])
{
#pragma unroll
    for (int j = 0; j < N; ++j) {
        cx<R> t = s[j];
#pragma unroll
        for (int k = 0; k < N; ++k) t = cfma(a[k], B(k, j), t);
        s[j] = t;
    }
}

// The same for RW rows at once: each element of B is read once for all RW
// rows, and each row goes through exactly the operations above.
template <int N, int RW, class R, class G> SUN_DEV void rmul_rows_g(const cx<R> (&a)[RW][N], G&& B, cx<R> (&c)[RW][N])
{
#pragma unroll
    for (int j = 0; j < N; ++j) {
        const cx<R> b0 = B(0, j);
        cx<R> s[RW];
#pragma unroll
        for (int r = 0; r < RW; ++r) s[r] = a[r][0] * b0;
#pragma unroll
        for (int k = 1; k < N; ++k) {
            const cx<R> bk = B(k, j);
#pragma unroll
            for (int r = 0; r < RW; ++r) s[r] = cfma(a[r][k], bk, s[r]);
        }
#pragma unroll
        for (int r = 0; r < RW; ++r) c[r][j] = s[r];
    }
}
template <int N, int RW, class R, class G>
SUN_DEV void rmul_dn_rows_g(const cx<R> (&a)[RW][N], G&& B, cx<R> (&c)[RW][N])
{
#pragma unroll
    for (int j = 0; j < N; ++j) {
        cx<R> s[RW];
#pragma unroll
        for (int r = 0; r < RW; ++r) s[r] = mkc<R>(0, 0);
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const cx<R> bk = B(k, j);
#pragma unroll
            for (int r = 0; r < RW; ++r) s[r] = cfma_cn(a[r][k], bk, s[r]);
        }
#pragma unroll
        for (int r = 0; r < RW; ++r) c[r][j] = s[r];
    }
}
template <int N, int RW, class R, class G>
SUN_DEV void racc_nd_rows_g(const cx<R> (&a)[RW][N], G&& B, cx<R> (&s)[RW][N])
{
#pragma unroll
    for (int j = 0; j < N; ++j)
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const cx<R> bjk = B(j, k);
#pragma unroll
            for (int r = 0; r < RW; ++r) s[r][j] = cfma_nc(a[r][k], bjk, s[r][j]);
        }
}
template <int N, int RW, class R, class G>
SUN_DEV void racc_rows_g(const cx<R> (&a)[RW][N], G&& B, cx<R> (&s)[RW][N])
{
#pragma unroll
    for (int j = 0; j < N; ++j)
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const cx<R> bkj = B(k, j);
#pragma unroll
            for (int r = 0; r < RW; ++r) s[r][j] = cfma(a[r][k], bkj, s[r][j]);
        }
}

// row 2 of an SU(3) matrix from rows 0, 1 -- rebuild12
template <class R> SUN_DEV void rebuild12_row(const cx<R> a[3], const cx<R> b[3], cx<R> c[3])
{
    c[0] = conj_det2(a[1], b[2], a[2], b[1]);
    c[1] = conj_det2(a[2], b[0], a[0], b[2]);
    c[2] = conj_det2(a[0], b[1], a[1], b[0]);
}

template <int N, class R> SUN_HD cx<R> mtrace(const Mat<N, R>& A)
{
    cx<R> t = A.e[0][0];
#pragma unroll
    for (int i = 1; i < N; ++i) t = t + A.e[i][i];
    return t;
}
// tr(A B^dagger) = sum_ij A_ij conj(B_ij)
template <int N, class R> SUN_HD cx<R> mtrace_nd(const Mat<N, R>& A, const Mat<N, R>& B)
{
    cx<R> t = mkc<R>(0, 0);
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) t = cfma_nc(A.e[i][j], B.e[i][j], t);
    return t;
}
template <int N, class Rd, class Rs> SUN_HD void mconvert(const Mat<N, Rs>& A, Mat<N, Rd>& B)
{
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) B.e[i][j] = mkc<Rd>((Rd)A.e[i][j].re, (Rd)A.e[i][j].im);
}

// SU(2) subgroup (p,q) of block b: (0,1),(1,2),...,(N-2,N-1),(0,2),(1,3),...
// -- the enumeration of IndexBlock (include/constants.h:143-192), resolved at
// compile time.
template <int N> struct SubGroup {
    static constexpr int count = N * (N - 1) / 2;
    static SUN_HD constexpr int p(int b)
    {
        int idx = 0;
        for (int del = 1; del < N; ++del)
            for (int i = 0; i < N - del; ++i, ++idx)
                if (idx == b) return i;
        return -1;
    }
    static SUN_HD constexpr int q(int b)
    {
        int idx = 0;
        for (int del = 1; del < N; ++del)
            for (int i = 0; i < N - del; ++i, ++idx)
                if (idx == b) return i + del;
        return -1;
    }
};

// Calls f(P, Q) with the (p, q) of subgroup b as compile-time constants
// (std::integral_constant), so the code in f indexes matrices statically,
// i.e. keeps them in registers, although b is a runtime loop index.
template <int N, int B = 0, class F> SUN_DEV void with_subgroup(int b, F&& f)
{
    if constexpr (B < SubGroup<N>::count) {
        if (b == B)
            f(std::integral_constant<int, SubGroup<N>::p(B)>{}, std::integral_constant<int, SubGroup<N>::q(B)>{});
        else
            with_subgroup<N, B + 1>(b, f);
    }
}

// Block 4-vector of M restricted to rows/cols (p,q) -- get_block_su2
// (include/device_PHB_OVR.h:265-272).
template <int N, class R> SUN_DEV void su2_block(const Mat<N, R>& M, int p, int q, R r[4])
{
    r[0] = M.e[p][p].re + M.e[q][q].re;
    r[1] = M.e[p][q].im + M.e[q][p].im;
    r[2] = M.e[p][q].re - M.e[q][p].re;
    r[3] = M.e[p][p].im - M.e[q][q].im;
}
// Block 4-vector of (U S^dagger) on rows/cols (p,q), S the staple sum; the
// SU(3) path of heatBathSUN / overrelaxationSUN recomputes it from the
// current U (device_PHB_OVR.h:382-405, :518-535).
template <int N, class R>
SUN_DEV void su2_block_US(const Mat<N, R>& U, const Mat<N, R>& S, int p, int q, R r[4])
{
    cx<R> a0 = mkc<R>(0, 0), a1 = a0, a2 = a0, a3 = a0;
#pragma unroll
    for (int j = 0; j < N; ++j) {
        a0 = cfma_nc(U.e[p][j], S.e[p][j], a0);
        a1 = cfma_nc(U.e[p][j], S.e[q][j], a1);
        a2 = cfma_nc(U.e[q][j], S.e[p][j], a2);
        a3 = cfma_nc(U.e[q][j], S.e[q][j], a3);
    }
    r[0] = a0.re + a3.re;
    r[1] = a1.im + a2.im;
    r[2] = a1.re - a2.re;
    r[3] = a0.im - a3.im;
}
// rows p,q of L <- su2(b) rows p,q -- mul_block_sun (device_PHB_OVR.h:296-303)
template <int N, class R> SUN_DEV void su2_apply(Mat<N, R>& L, int p, int q, const R b[4])
{
    const cx<R> a00 = mkc(b[0], b[3]), a01 = mkc(b[2], b[1]);
    const cx<R> a10 = mkc(-b[2], b[1]), a11 = mkc(b[0], -b[3]);
#pragma unroll
    for (int j = 0; j < N; ++j) {
        cx<R> up = L.e[p][j], uq = L.e[q][j];
        L.e[p][j] = cfma(a01, uq, a00 * up);
        L.e[q][j] = cfma(a11, uq, a10 * up);
    }
}
// row p only of su2_apply (the same operations), for a last subgroup whose
// row q is not needed afterwards
template <int N, class R> SUN_DEV void su2_apply_row_p(Mat<N, R>& L, int p, int q, const R b[4])
{
    const cx<R> a00 = mkc(b[0], b[3]), a01 = mkc(b[2], b[1]);
#pragma unroll
    for (int j = 0; j < N; ++j) L.e[p][j] = cfma(a01, L.e[q][j], a00 * L.e[p][j]);
}
// a * r^dagger on quaternion 4-vectors -- mulsu2UVDagger (msu2.h:212-219)
template <class R> SUN_DEV void su2_mul_udag(const R a[4], const R r[4], R b[4])
{
    b[0] = fma(a[3], r[3], fma(a[2], r[2], fma(a[1], r[1], a[0] * r[0])));
    b[1] = fma(-a[3], r[2], fma(a[2], r[3], fma(-a[0], r[1], a[1] * r[0])));
    b[2] = fma(-a[1], r[3], fma(a[3], r[1], fma(-a[0], r[2], a[2] * r[0])));
    b[3] = fma(-a[2], r[1], fma(a[1], r[2], fma(-a[0], r[3], a[3] * r[0])));
}

// SU(3) third row from the first two: row2 = conj(row0 x row1) --
// reconstruct12p (include/reconstruct_12p_8p.h:17-21).
template <class R> SUN_HD void rebuild12(Mat<3, R>& A)
{
    A.e[2][0] = conj_det2(A.e[0][1], A.e[1][2], A.e[0][2], A.e[1][1]);
    A.e[2][1] = conj_det2(A.e[0][2], A.e[1][0], A.e[0][0], A.e[1][2]);
    A.e[2][2] = conj_det2(A.e[0][0], A.e[1][1], A.e[0][1], A.e[1][0]);
}

SUN_DEV float rsq(float x) { return rsqrtf(x); }
SUN_DEV double rsq(double x) { return rsqrt(x); }

// The link a 12-parameter update rewrites: its rebuilt row 2 scaled to unit
// length.  The update rotates row 2 into the two stored rows.  Unscaled,
// |row2|^2 - 1 ~ (|row0|^2 - 1) + (|row1|^2 - 1) is fed back into them, and
// the storage error grows about 4x per sweep: FP32 links measured on B200
// reach |U^dag U - 1| ~ 0.5 in 9 sweeps and overflow in 13 without
// reunitarization (FP64: 1e-13 to 3e-5 in 16 sweeps).  The reference's
// reconstruction (reconstruct_12p_8p.h:17-21) grows the same way.  Scaled,
// each rotation shrinks the norm and orthogonality errors of the stored rows
// instead, and the error stays at the rounding level of full links.
template <class R> SUN_DEV void unit_row2(Mat<3, R>& A)
{
    const R s = rsq(cnorm2(A.e[2][0]) + cnorm2(A.e[2][1]) + cnorm2(A.e[2][2]));
#pragma unroll
    for (int j = 0; j < 3; ++j) A.e[2][j] = s * A.e[2][j];
}

// Determinant; N <= 3 by cofactors, larger N by Gaussian elimination with
// partial pivoting (used only by FP64 reunitarization and the hot start).
template <int N, class R> SUN_DEV cx<R> mdet(const Mat<N, R>& A)
{
    if constexpr (N == 2) return A.e[0][0] * A.e[1][1] - A.e[0][1] * A.e[1][0];
    else if constexpr (N == 3) {
        return A.e[0][0] * (A.e[1][1] * A.e[2][2] - A.e[1][2] * A.e[2][1]) -
               A.e[0][1] * (A.e[1][0] * A.e[2][2] - A.e[1][2] * A.e[2][0]) +
               A.e[0][2] * (A.e[1][0] * A.e[2][1] - A.e[1][1] * A.e[2][0]);
    } else {
    Mat<N, R> b = A;
    cx<R> det = mkc<R>(1, 0);
#pragma unroll
    for (int k = 0; k < N; ++k) {
        int piv = k;
        R best = cnorm2(b.e[k][k]);
#pragma unroll
        for (int i = k + 1; i < N; ++i)
            if (cnorm2(b.e[i][k]) > best) { best = cnorm2(b.e[i][k]); piv = i; }
        if (piv != k) {
#pragma unroll
            for (int i = k + 1; i < N; ++i)
                if (i == piv)
#pragma unroll
                    for (int j = 0; j < N; ++j) { cx<R> t = b.e[k][j]; b.e[k][j] = b.e[i][j]; b.e[i][j] = t; }
            det = mkc(-det.re, -det.im);
        }
        cx<R> d = b.e[k][k];
        det = det * d;
        R inv = R(1) / cnorm2(d);
        cx<R> dinv = mkc(d.re * inv, -d.im * inv);
#pragma unroll
        for (int i = k + 1; i < N; ++i) {
            cx<R> f = b.e[i][k] * dinv;
#pragma unroll
            for (int j = k; j < N; ++j) b.e[i][j] = b.e[i][j] - f * b.e[k][j];
        }
    }
    return det;
    }
}

// Reunitarization in the arithmetic of R -- reunit_link
// (include/reunitlink.h:16-88).  N == 3: normalise row 0, Gram-Schmidt row 1,
// row 2 = conj(row0 x row1).  N > 3: Gram-Schmidt over columns, then the last
// column times exp(-i arg det).  N == 2 has no reference counterpart
// (reunitlink.h:86 is an #error): normalise row 0, row 1 = (-conj u01, conj u00).
template <int N, class R> SUN_DEV void reunit(Mat<N, R>& U)
{
    if constexpr (N == 2) {
        R n = R(1) / sqrt(cnorm2(U.e[0][0]) + cnorm2(U.e[0][1]));
        U.e[0][0] = n * U.e[0][0];
        U.e[0][1] = n * U.e[0][1];
        U.e[1][0] = mkc(-U.e[0][1].re, U.e[0][1].im);
        U.e[1][1] = cconj(U.e[0][0]);
    } else if constexpr (N == 3) {
        R t1 = R(0);
#pragma unroll
        for (int c = 0; c < N; ++c) t1 += cnorm2(U.e[0][c]);
        t1 = R(1) / sqrt(t1);
#pragma unroll
        for (int c = 0; c < N; ++c) U.e[0][c] = t1 * U.e[0][c];
        cx<R> t2 = mkc<R>(0, 0);
#pragma unroll
        for (int c = 0; c < N; ++c) t2 = cfma_cn(U.e[0][c], U.e[1][c], t2);
#pragma unroll
        for (int c = 0; c < N; ++c) U.e[1][c] = U.e[1][c] - t2 * U.e[0][c];
        t1 = R(0);
#pragma unroll
        for (int c = 0; c < N; ++c) t1 += cnorm2(U.e[1][c]);
        t1 = R(1) / sqrt(t1);
#pragma unroll
        for (int c = 0; c < N; ++c) U.e[1][c] = t1 * U.e[1][c];
        rebuild12(U);
    } else {
    R t1 = R(0);
#pragma unroll
    for (int c = 0; c < N; ++c) t1 += cnorm2(U.e[c][0]);
    t1 = R(1) / sqrt(t1);
#pragma unroll
    for (int c = 0; c < N; ++c) U.e[c][0] = t1 * U.e[c][0];
#pragma unroll
    for (int j = 1; j < N; ++j) {
#pragma unroll
        for (int i = 0; i < j; ++i) {
            cx<R> t2 = mkc<R>(0, 0);
#pragma unroll
            for (int c = 0; c < N; ++c) t2 = cfma_cn(U.e[c][i], U.e[c][j], t2);
#pragma unroll
            for (int c = 0; c < N; ++c) U.e[c][j] = U.e[c][j] - t2 * U.e[c][i];
        }
        t1 = R(0);
#pragma unroll
        for (int c = 0; c < N; ++c) t1 += cnorm2(U.e[c][j]);
        t1 = R(1) / sqrt(t1);
#pragma unroll
        for (int c = 0; c < N; ++c) U.e[c][j] = t1 * U.e[c][j];
    }
    cx<R> d = mdet<N, R>(U);
    R ph = atan2(d.im, d.re);
    R s, c;
    sincos(ph, &s, &c);
    cx<R> f = mkc(c, -s);
#pragma unroll
    for (int r = 0; r < N; ++r) U.e[r][N - 1] = U.e[r][N - 1] * f;
    }
}

}  // namespace sunb
