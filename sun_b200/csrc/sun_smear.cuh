// sun_smear.cuh -- smearing and multihit kernels (src/smear/ape.cu, stout.cu,
// hyp.cu, multihit.cu, multihitsp.cu) and their Ops<N> launch wrappers.
// Included at the end of sun_kernels.cuh.
//
// Every kernel reads the unchanged field `src` and writes `dst` (distinct
// device images of one lattice's layout, order and precision), one thread per
// site and one grid row (blockIdx.y) per smeared direction or intermediate
// link, so a smearing step is one launch (three for HYP) whatever the
// directions.  The reference allows only normal-order SOA arrays here
// (src/smear/ape.cu:194-197); these kernels take any storage order and layout.
#pragma once

namespace sunb {

// direction of grid row `row` of a launch over the directions in dirmask
SUN_DEV int nth_dir(int dirmask, int row)
{
    int mu = 0;
#pragma unroll 1
    for (; mu < 4; ++mu)
        if ((dirmask >> mu) & 1) {
            if (row == 0) break;
            --row;
        }
    return mu;
}

// link (x, mu) of a device image
template <int N, class R, int LAYOUT>
SUN_DEV void ld_site(const LatDev& L, const Geom& g, const void* img, const int x[4], int mu, Mat<N, R>& A)
{
    LinkIO<N, R, LAYOUT>::template load<true>(reinterpret_cast<const cx<R>*>(img),
                                              (uint32_t)site_index(L, g, x) + (uint32_t)mu * (uint32_t)g.V,
                                              4u * (uint32_t)g.V, A);
}

// S += the "up" and "down" staples of a link in direction a in the plane
// (a, r):  R(x) A(x+r) R(x+a)^dag + R(x-r)^dag A(x-r) R(x-r+a), where
// get_r / get_a load the link-like matrices that play U_r and U_a at a site
// (the links themselves, or an intermediate HYP level).  The shape of
// CalcStaple (src/smear/hyp.cu:57, src/smear/multihit.cu:38).
template <int N, class R, class GR, class GA>
SUN_DEV void plane_staple(const Geom& g, const int x[4], int a, int r, GR get_r, GA get_a, Mat<N, R>& S)
{
    int xr[4], xa[4], xmr[4], xmra[4];
    shifted(g, x, r, 1, xr);
    shifted(g, x, a, 1, xa);
    shifted(g, x, r, -1, xmr);
    shifted(g, xmr, a, 1, xmra);
    Mat<N, R> A, B, C;
    get_r(x, A);
    get_a(xr, B);
    mmul(A, B, C);
    get_r(xa, A);
    macc_nd(C, A, S);
    get_r(xmr, A);
    get_a(xmr, B);
    mmul_dn(A, B, C);
    get_r(xmra, A);
    macc(C, A, S);
}

// staple of the link (x, mu) over the planes nu in numask (nu != mu), nu
// ascending -- kernel_APE_Space (src/smear/ape.cu:44) with numask = 7
template <int N, class R, int LAYOUT>
SUN_DEV void staple_planes(const LatDev& L, const Geom& g, const void* img, const int x[4], int mu, int numask,
                           Mat<N, R>& S)
{
    mzero(S);
    auto get_mu = [&](const int* y, Mat<N, R>& M) { ld_site<N, R, LAYOUT>(L, g, img, y, mu, M); };
#pragma unroll 1
    for (int nu = 0; nu < 4; ++nu) {
        if (nu == mu || !((numask >> nu) & 1)) continue;
        auto get_nu = [&](const int* y, Mat<N, R>& M) { ld_site<N, R, LAYOUT>(L, g, img, y, nu, M); };
        plane_staple<N, R>(g, x, mu, nu, get_nu, get_mu, S);
    }
}

// Re tr(W Q) = sum_ij W_ij Q_ji, the convergence measure of project_link
// (include/projectlink.h:20, realtraceUVdagger of w and the daggered q)
template <int N, class R> SUN_DEV R re_tr_nn(const Mat<N, R>& W, const Mat<N, R>& Q)
{
    R s = R(0);
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) s += W.e[i][j].re * Q.e[j][i].re - W.e[i][j].im * Q.e[j][i].im;
    return s;
}

// Projection onto SU(N): maximise Re tr(W Q^dagger) by Cabibbo-Marinari SU(2)
// hits starting from W -- project_link (include/projectlink.h:17): per
// subgroup the block of W Q^dagger is conj-normalised (a zero block counts as
// the unit element) and multiplied into rows p,q of W; with tol > 0 the hits
// stop once the relative change of Re tr(W Q)/N is <= tol.  SU3project
// (projectlink.h:119) is this iteration from W = 1 with tol = 0.
template <int N, class R> SUN_DEV void project_sun(Mat<N, R>& W, const Mat<N, R>& Q, int nhits, R tol)
{
    R conver = R(1), old_tr = R(0);
    if (tol > R(0)) old_tr = re_tr_nn(W, Q) / R(N);
#pragma unroll 1
    for (int h = 0; h < nhits && conver > tol; ++h) {
#pragma unroll
        for (int b = 0; b < SubGroup<N>::count; ++b) {
            const int p = SubGroup<N>::p(b), q = SubGroup<N>::q(b);
            R r[4], c[4];
            su2_block_US<N, R>(W, Q, p, q, r);
            R k = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + r[3] * r[3]);
            if (k == R(0)) { k = R(1); r[0] = R(1); }
            k = R(1) / k;
            c[0] = r[0] * k; c[1] = -r[1] * k; c[2] = -r[2] * k; c[3] = -r[3] * k;
            su2_apply<N, R>(W, p, q, c);
        }
        if (tol > R(0)) {
            const R nt = re_tr_nn(W, Q) / R(N);
            conver = (nt - old_tr) / old_tr;
            old_tr = nt;
        }
    }
}

// exp(iQ) for traceless Hermitian 3x3 Q as f0 + f1 Q + f2 Q^2, written from
// Morningstar and Peardon, Phys. Rev. D69 (2004) 054501, eqs. 19-34, in the
// regimes of get_fs_and_bs_from_Qs (src/smear/stout.cu:99): c0 = tr Q^3/3,
// c1 = tr Q^2/2; c1 < 4e-3 by the Taylor series of the f_j (from
// Q^3 = c1 Q + c0); theta by its series in eps = (c0max - |c0|)/c0max for
// eps < 1e-3; sin(w)/w by its series for |w| < 0.05; c0 < 0 through
// f_j(-c0) = (-1)^j conj(f_j(c0)).
template <class R> SUN_DEV void exp_iq3(const Mat<3, R>& Q, Mat<3, R>& E)
{
    Mat<3, R> QQ;
    mmul(Q, Q, QQ);
    R c0 = R(0);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int k = 0; k < 3; ++k) c0 += Q.e[i][k].re * QQ.e[k][i].re - Q.e[i][k].im * QQ.e[k][i].im;
    c0 = c0 / R(3);
    const R c1 = (QQ.e[0][0].re + QQ.e[1][1].re + QQ.e[2][2].re) * R(0.5);
    cx<R> f0, f1, f2;
    if (c1 < R(4.0e-3)) {
        f0 = mkc<R>(R(1) - c0 * c0 / R(720), -(c0 / R(6)) * (R(1) - (c1 / R(20)) * (R(1) - c1 / R(42))));
        f1 = mkc<R>(c0 / R(24) * (R(1) - c1 / R(15) * (R(1) - R(3) * c1 / R(112))),
                    R(1) - c1 / R(6) * (R(1) - c1 / R(20) * (R(1) - c1 / R(42))) - c0 * c0 / R(5040));
        f2 = mkc<R>(R(0.5) * (R(-1) + c1 / R(12) * (R(1) - c1 / R(30) * (R(1) - c1 / R(56))) + c0 * c0 / R(20160)),
                    R(0.5) * (c0 / R(60) * (R(1) - c1 / R(21) * (R(1) - c1 / R(48)))));
    } else {
        const R c0abs = fabs(c0);
        const R c13 = c1 / R(3);
        const R c0max = R(2) * c13 * sqrt(c13);
        const R eps = (c0max - c0abs) / c0max;
        R theta;
        if (eps < R(0)) theta = R(0);
        else if (eps < R(1.0e-3))
            theta = sqrt(R(2)) * sqrt(eps) *
                    (R(1) + ((R(1) / R(12)) +
                             ((R(3) / R(160)) +
                              ((R(5) / R(896)) + ((R(35) / R(18432)) + (R(63) / R(90112)) * eps) * eps) * eps) * eps) *
                                eps);
        else theta = acos(c0abs / c0max);
        const R u = sqrt(c13) * cos(theta / R(3));
        const R w = sqrt(c1) * sin(theta / R(3));
        const R u2 = u * u, w2 = w * w;
        const R xi0 = fabs(w) < R(0.05)
                          ? R(1) - (R(1) / R(6)) * w2 * (R(1) - (R(1) / R(20)) * w2 * (R(1) - (R(1) / R(42)) * w2))
                          : sin(w) / w;
        const R cu = cos(u), su = sin(u), cw = cos(w), c2u = cos(R(2) * u), s2u = sin(R(2) * u);
        const R den = R(9) * u2 - w2;
        f0 = mkc<R>(((u2 - w2) * c2u + cu * R(8) * u2 * cw + R(2) * u * su * (R(3) * u2 + w2) * xi0) / den,
                    ((u2 - w2) * s2u - su * R(8) * u2 * cw + R(2) * u * cu * (R(3) * u2 + w2) * xi0) / den);
        f1 = mkc<R>((R(2) * (u * c2u - u * cu * cw) + (R(3) * u2 - w2) * xi0 * su) / den,
                    (R(2) * (u * s2u + u * su * cw) + (R(3) * u2 - w2) * xi0 * cu) / den);
        f2 = mkc<R>((c2u - cu * cw - u * su * R(3) * xi0) / den, (s2u + su * cw - u * cu * R(3) * xi0) / den);
        if (c0 < R(0)) {
            f0.im = -f0.im;
            f1.re = -f1.re;
            f2.im = -f2.im;
        }
    }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) E.e[i][j] = f1 * Q.e[i][j] + f2 * QQ.e[i][j];
#pragma unroll
    for (int i = 0; i < 3; ++i) E.e[i][i] = E.e[i][i] + f0;
}

// ---------------------------------------------------------------------------
// APE: U'_mu = P[(U_mu + w S_mu) / (1 + 6 w)], S_mu over the spatial planes --
// kernel_APE_Space (src/smear/ape.cu:44).  SU(3): SU3project from 1
// (tol unused); other N: project_link from U_mu with tol.
template <int N, class R, int LAYOUT>
__global__ void __launch_bounds__(128) k_ape(BatchView bv, const void* src, void* dst, int dirmask, R w, int nhits,
                                             R tol)
{
    const int b = blockIdx.x;
    const int l = find_lat(bv, b);
    const LatDev& L = bv.lats[l];
    const Geom g = geom_of(L);
    const int site = (b - __ldg(bv.begin + l)) * blockDim.x + threadIdx.x;
    if (site >= g.V) return;
    const int mu = nth_dir(dirmask, blockIdx.y);
    int x[4];
    site_coords(L, g, site, x);
    Mat<N, R> S, U, W;
    staple_planes<N, R, LAYOUT>(L, g, src, x, mu, 7, S);
    ld_site<N, R, LAYOUT>(L, g, src, x, mu, U);
    const R inv = R(1) / (R(1) + R(6) * w);
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) {
            S.e[i][j].re = (U.e[i][j].re + S.e[i][j].re * w) * inv;
            S.e[i][j].im = (U.e[i][j].im + S.e[i][j].im * w) * inv;
        }
    if constexpr (N == 3) {
        munit(W);
        project_sun<N, R>(W, S, nhits, R(0));
    } else {
        W = U;
        project_sun<N, R>(W, S, nhits, tol);
    }
    LinkIO<N, R, LAYOUT>::store(reinterpret_cast<cx<R>*>(dst), (uint32_t)site + (uint32_t)mu * (uint32_t)g.V,
                                4u * (uint32_t)g.V, W);
}

// Stout (SU(3)): C = w S_mu (spatial planes), Omega = C U^dagger,
// Q = traceless part of (i/2)(Omega^dagger - Omega), U' = exp(iQ) U --
// kernel_Stout / stout_smear (src/smear/stout.cu:557, :521).
template <class R, int LAYOUT>
__global__ void __launch_bounds__(128) k_stout(BatchView bv, const void* src, void* dst, int dirmask, R w)
{
    const int b = blockIdx.x;
    const int l = find_lat(bv, b);
    const LatDev& L = bv.lats[l];
    const Geom g = geom_of(L);
    const int site = (b - __ldg(bv.begin + l)) * blockDim.x + threadIdx.x;
    if (site >= g.V) return;
    const int mu = nth_dir(dirmask, blockIdx.y);
    int x[4];
    site_coords(L, g, site, x);
    Mat<3, R> S, U, Om, Q, E;
    staple_planes<3, R, LAYOUT>(L, g, src, x, mu, 7, S);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) S.e[i][j] = w * S.e[i][j];
    ld_site<3, R, LAYOUT>(L, g, src, x, mu, U);
    mmul_nd(S, U, Om);
    // (i/2)(Om^dag - Om): entry ij = (i/2)(conj(Om_ji) - Om_ij)
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const cx<R> d = cconj(Om.e[j][i]) - Om.e[i][j];
            Q.e[i][j] = mkc<R>(R(-0.5) * d.im, R(0.5) * d.re);
        }
    const cx<R> tr = R(1) / R(3) * (Q.e[0][0] + Q.e[1][1] + Q.e[2][2]);
#pragma unroll
    for (int i = 0; i < 3; ++i) Q.e[i][i] = Q.e[i][i] - tr;
    exp_iq3<R>(Q, E);
    mmul(E, U, S);
    LinkIO<3, R, LAYOUT>::store(reinterpret_cast<cx<R>*>(dst), (uint32_t)site + (uint32_t)mu * (uint32_t)g.V,
                                4u * (uint32_t)g.V, S);
}

// ---------------------------------------------------------------------------
// HYP (src/smear/hyp.cu:88-190), one level per launch.  Levels 1 and 2 are
// kept in scratch images of 16 full N x N link slots per site: slot d * 4 + o
// at complex element ((slot * N*N + e) * V + site) -- Vbar_{d;o} (o the
// direction of its staple) and Vtil_{d;o} (o the excluded direction).
template <int N, class R>
SUN_DEV void ld_slot(const Geom& g, const void* B, int site, int slot, Mat<N, R>& A)
{
    const cx<R>* p = reinterpret_cast<const cx<R>*>(B) + (size_t)slot * N * N * g.V + site;
#pragma unroll
    for (int e = 0; e < N * N; ++e) A.e[e / N][e % N] = ld_elem<R, true>(p + (size_t)e * g.V);
}
template <int N, class R>
SUN_DEV void st_slot(const Geom& g, void* B, int site, int slot, const Mat<N, R>& A)
{
    cx<R>* p = reinterpret_cast<cx<R>*>(B) + (size_t)slot * N * N * g.V + site;
#pragma unroll
    for (int e = 0; e < N * N; ++e) st_elem<R>(p + (size_t)e * g.V, A.e[e / N][e % N]);
}

// level 1: Vbar_{m;e}(x) = P[(1 - a3) U_m(x) + a3/2 staple of U_m in plane (m, e)]
// (HYPSmearVbar, hyp.cu:88); grid row = m * 3 + (index of e among e != m)
template <int N, class R, int LAYOUT>
__global__ void __launch_bounds__(128) k_hyp1(BatchView bv, const void* src, void* B1, R a3, int nhits, R tol)
{
    const int b = blockIdx.x;
    const int l = find_lat(bv, b);
    const LatDev& L = bv.lats[l];
    const Geom g = geom_of(L);
    const int site = (b - __ldg(bv.begin + l)) * blockDim.x + threadIdx.x;
    if (site >= g.V) return;
    const int m = blockIdx.y / 3, j = blockIdx.y % 3, e = j + (j >= m ? 1 : 0);
    int x[4];
    site_coords(L, g, site, x);
    Mat<N, R> S, U;
    mzero(S);
    auto get_e = [&](const int* y, Mat<N, R>& M) { ld_site<N, R, LAYOUT>(L, g, src, y, e, M); };
    auto get_m = [&](const int* y, Mat<N, R>& M) { ld_site<N, R, LAYOUT>(L, g, src, y, m, M); };
    plane_staple<N, R>(g, x, m, e, get_e, get_m, S);
    ld_site<N, R, LAYOUT>(L, g, src, x, m, U);
    const R h = R(0.5) * a3, c = R(1) - a3;
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int k = 0; k < N; ++k) {
            S.e[i][k].re = S.e[i][k].re * h + U.e[i][k].re * c;
            S.e[i][k].im = S.e[i][k].im * h + U.e[i][k].im * c;
        }
    project_sun<N, R>(U, S, nhits, tol);
    st_slot<N, R>(g, B1, site, m * 4 + e, U);
}

// level 2: Vtil_{a;b}(x) = P[(1 - a2) U_a(x) + a2/4 sum_{r != a,b} staple of
// Vbar_{a;s} with Vbar_{r;s}, s the fourth direction] (HYPSmearVtil,
// hyp.cu:106); grid row = a * 3 + (index of b among b != a)
template <int N, class R, int LAYOUT>
__global__ void __launch_bounds__(128) k_hyp2(BatchView bv, const void* src, const void* B1, void* B2, R a2,
                                              int nhits, R tol)
{
    const int b = blockIdx.x;
    const int l = find_lat(bv, b);
    const LatDev& L = bv.lats[l];
    const Geom g = geom_of(L);
    const int site = (b - __ldg(bv.begin + l)) * blockDim.x + threadIdx.x;
    if (site >= g.V) return;
    const int a = blockIdx.y / 3, j = blockIdx.y % 3, bb = j + (j >= a ? 1 : 0);
    int x[4];
    site_coords(L, g, site, x);
    Mat<N, R> S, U;
    mzero(S);
#pragma unroll 1
    for (int r = 0; r < 4; ++r) {
        if (r == a || r == bb) continue;
        const int s = 6 - a - bb - r;
        auto get_r = [&](const int* y, Mat<N, R>& M) { ld_slot<N, R>(g, B1, site_index(L, g, y), r * 4 + s, M); };
        auto get_a = [&](const int* y, Mat<N, R>& M) { ld_slot<N, R>(g, B1, site_index(L, g, y), a * 4 + s, M); };
        plane_staple<N, R>(g, x, a, r, get_r, get_a, S);
    }
    ld_site<N, R, LAYOUT>(L, g, src, x, a, U);
    const R h = R(0.25) * a2, c = R(1) - a2;
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int k = 0; k < N; ++k) {
            S.e[i][k].re = S.e[i][k].re * h + U.e[i][k].re * c;
            S.e[i][k].im = S.e[i][k].im * h + U.e[i][k].im * c;
        }
    project_sun<N, R>(U, S, nhits, tol);
    st_slot<N, R>(g, B2, site, a * 4 + bb, U);
}

// level 3: V_m(x) = P[(1 - a1) U_m(x) + a1/6 sum_{n != m} staple of Vtil_{m;n}
// with Vtil_{n;m}] (HYPSmearV, hyp.cu:137); grid row = smeared direction
template <int N, class R, int LAYOUT>
__global__ void __launch_bounds__(128) k_hyp3(BatchView bv, const void* src, const void* B2, void* dst, int dirmask,
                                              R a1, int nhits, R tol)
{
    const int b = blockIdx.x;
    const int l = find_lat(bv, b);
    const LatDev& L = bv.lats[l];
    const Geom g = geom_of(L);
    const int site = (b - __ldg(bv.begin + l)) * blockDim.x + threadIdx.x;
    if (site >= g.V) return;
    const int m = nth_dir(dirmask, blockIdx.y);
    int x[4];
    site_coords(L, g, site, x);
    Mat<N, R> S, U;
    mzero(S);
#pragma unroll 1
    for (int n = 0; n < 4; ++n) {
        if (n == m) continue;
        auto get_n = [&](const int* y, Mat<N, R>& M) { ld_slot<N, R>(g, B2, site_index(L, g, y), n * 4 + m, M); };
        auto get_m = [&](const int* y, Mat<N, R>& M) { ld_slot<N, R>(g, B2, site_index(L, g, y), m * 4 + n, M); };
        plane_staple<N, R>(g, x, m, n, get_n, get_m, S);
    }
    ld_site<N, R, LAYOUT>(L, g, src, x, m, U);
    const R h = a1 / R(6), c = R(1) - a1;
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int k = 0; k < N; ++k) {
            S.e[i][k].re = S.e[i][k].re * h + U.e[i][k].re * c;
            S.e[i][k].im = S.e[i][k].im * h + U.e[i][k].im * c;
        }
    project_sun<N, R>(U, S, nhits, tol);
    LinkIO<N, R, LAYOUT>::store(reinterpret_cast<cx<R>*>(dst), (uint32_t)site + (uint32_t)m * (uint32_t)g.V,
                                4u * (uint32_t)g.V, U);
}

// ---------------------------------------------------------------------------
// Multihit of the temporal links -- kernel_multihit_1D_halfrng /
// kernel_evenodd (src/smear/multihit.cu:80, :117): U_3(x) of `dst` (SOA layout)
// becomes (U + U_1 + ... + U_nhit)/(nhit + 1), U_h the heatbath chain of
// U_3(x) against its full staple in `src`.  Random numbers: the Philox stream
// of link (lex, 3) with purpose 2, pass 0, drawn through all hits in order.
template <int N, class R, int LAYOUT>
__global__ void __launch_bounds__(128) k_multihit(BatchView bv, const void* src, void* dst, int nhit,
                                                  unsigned long long seed)
{
    const int b = blockIdx.x;
    const int l = find_lat(bv, b);
    const LatDev& L = bv.lats[l];
    const Geom g = geom_of(L);
    const int site = (b - __ldg(bv.begin + l)) * blockDim.x + threadIdx.x;
    if (site >= g.V) return;
    int x[4];
    site_coords(L, g, site, x);
    Mat<N, R> S, U, A;
    staple_planes<N, R, LAYOUT>(L, g, src, x, 3, 15, S);
    ld_site<N, R, LAYOUT>(L, g, src, x, 3, U);
    A = U;
    PhiloxStream<R> st;
    st.init(seed, (uint32_t)lex_of(g, x), 3u | (2u << 8), 0u);
    const R bon = (R)L.beta_over_n;
#pragma unroll 1
    for (int h = 0; h < nhit; ++h) {
        heatbath_update<N, R>(U, S, bon, st);
#pragma unroll
        for (int i = 0; i < N; ++i)
#pragma unroll
            for (int j = 0; j < N; ++j) A.e[i][j] = A.e[i][j] + U.e[i][j];
    }
    const R inv = R(1) / R(nhit + 1);
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) A.e[i][j] = inv * A.e[i][j];
    LinkIO<N, R, L_SOA>::store(reinterpret_cast<cx<R>*>(dst), (uint32_t)site + 3u * (uint32_t)g.V,
                               4u * (uint32_t)g.V, A);
}

// Spatial multihit by overrelaxation -- kernel_MultiHitSP_1D_halfrng
// (src/smear/multihitsp.cu:115): spatial U_m(x) of `dst` (SOA layout)
// becomes the mean of the nhit overrelaxation iterates of U_m(x) against its
// spatial staple in `src`; grid row = m.
template <int N, class R, int LAYOUT>
__global__ void __launch_bounds__(128) k_multihit_space(BatchView bv, const void* src, void* dst, int nhit)
{
    const int b = blockIdx.x;
    const int l = find_lat(bv, b);
    const LatDev& L = bv.lats[l];
    const Geom g = geom_of(L);
    const int site = (b - __ldg(bv.begin + l)) * blockDim.x + threadIdx.x;
    if (site >= g.V) return;
    const int m = blockIdx.y;
    int x[4];
    site_coords(L, g, site, x);
    Mat<N, R> S, U, A;
    staple_planes<N, R, LAYOUT>(L, g, src, x, m, 7, S);
    ld_site<N, R, LAYOUT>(L, g, src, x, m, U);
    mzero(A);
#pragma unroll 1
    for (int h = 0; h < nhit; ++h) {
        overrelax_update<N, R>(U, S);
#pragma unroll
        for (int i = 0; i < N; ++i)
#pragma unroll
            for (int j = 0; j < N; ++j) A.e[i][j] = A.e[i][j] + U.e[i][j];
    }
    const R inv = R(1) / R(nhit);
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) A.e[i][j] = inv * A.e[i][j];
    LinkIO<N, R, L_SOA>::store(reinterpret_cast<cx<R>*>(dst), (uint32_t)site + (uint32_t)m * (uint32_t)g.V,
                               4u * (uint32_t)g.V, A);
}

// ---------------------------------------------------------------------------
// launch wrappers
static inline int popcount4(int m) { return (m & 1) + ((m >> 1) & 1) + ((m >> 2) & 1) + ((m >> 3) & 1); }

template <int N>
cudaError_t Ops<N>::ape(int fp64, int layout, const BatchView& bv, int block, const void* src, void* dst,
                        int dirmask, double w, int nhits, double tol, cudaStream_t s)
{
    const dim3 grid(bv.nblocks, popcount4(dirmask));
#define CALL(R_, L_) k_ape<N, R_, L_><<<grid, block, 0, s>>>(bv, src, dst, dirmask, (R_)w, nhits, (R_)tol)
    SUN_DISPATCH(fp64, layout, CALL);
#undef CALL
    return cudaGetLastError();
}

template <int N>
cudaError_t Ops<N>::stout(int fp64, int layout, const BatchView& bv, int block, const void* src, void* dst,
                          int dirmask, double w, cudaStream_t s)
{
    if constexpr (N != 3) {
        return cudaErrorNotSupported;
    } else {
        const dim3 grid(bv.nblocks, popcount4(dirmask));
#define CALL(R_, L_) k_stout<R_, L_><<<grid, block, 0, s>>>(bv, src, dst, dirmask, (R_)w)
        SUN_DISPATCH(fp64, layout, CALL);
#undef CALL
        return cudaGetLastError();
    }
}

template <int N>
cudaError_t Ops<N>::hyp(int fp64, int layout, const BatchView& bv, int block, int level, const void* src, void* b1,
                        void* b2, void* dst, int dirmask, double alpha, int nhits, double tol, cudaStream_t s)
{
    const dim3 grid(bv.nblocks, level == 3 ? popcount4(dirmask) : 12);
#define CALL(R_, L_)                                                                                               \
    if (level == 1) k_hyp1<N, R_, L_><<<grid, block, 0, s>>>(bv, src, b1, (R_)alpha, nhits, (R_)tol);             \
    else if (level == 2) k_hyp2<N, R_, L_><<<grid, block, 0, s>>>(bv, src, b1, b2, (R_)alpha, nhits, (R_)tol);    \
    else k_hyp3<N, R_, L_><<<grid, block, 0, s>>>(bv, src, b2, dst, dirmask, (R_)alpha, nhits, (R_)tol)
    SUN_DISPATCH(fp64, layout, CALL);
#undef CALL
    return cudaGetLastError();
}

template <int N>
cudaError_t Ops<N>::multihit(int fp64, int layout, const BatchView& bv, int block, const void* src, void* dst,
                             int nhit, unsigned long long seed, int space, cudaStream_t s)
{
#define CALL(R_, L_)                                                                                 \
    if (space) k_multihit_space<N, R_, L_><<<dim3(bv.nblocks, 3), block, 0, s>>>(bv, src, dst, nhit); \
    else k_multihit<N, R_, L_><<<bv.nblocks, block, 0, s>>>(bv, src, dst, nhit, seed)
    SUN_DISPATCH(fp64, layout, CALL);
#undef CALL
    return cudaGetLastError();
}

}  // namespace sunb
