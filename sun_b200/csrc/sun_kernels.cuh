// sun_kernels.cuh -- the sm_100a kernels of the engine and the host launch
// wrappers Ops<N>.  Included only by ops_n{2,3,4,6}.cu, one translation unit
// per colour number N.
//
// Every launch covers a table of lattices of one (N, precision, layout)
// class; CTA b finds its lattice by a binary search over the table's CTA
// prefix (BatchView::begin), so one launch advances many uneven lattices.
#pragma once
#include "sun_core.cuh"
#include "sun_ops.h"

namespace sunb {

SUN_DEV int find_lat(const BatchView& bv, int b)
{
    int lo = 0, hi = bv.nlat - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(bv.begin + mid) <= b) lo = mid; else hi = mid - 1;
    }
    return lo;
}

SUN_DEV Geom geom_of(const LatDev& L)
{
    Geom g;
    g.X[0] = L.X[0]; g.X[1] = L.X[1]; g.X[2] = L.X[2]; g.X[3] = L.X[3];
    g.V = L.V; g.halfV = L.halfV;
    return g;
}

// lexicographic index one step (s = +1 / -1) along a direction with
// coordinate xc, extent Xc and lexicographic stride Sc, periodic
SUN_DEV int lex_step(int lex, int xc, int Xc, int Sc, int s)
{
    if (s > 0) return xc == Xc - 1 ? lex - (Xc - 1) * Sc : lex + Sc;
    return xc == 0 ? lex + (Xc - 1) * Sc : lex - Sc;
}

SUN_DEV int sel4(const int a[4], int i) { return i == 0 ? a[0] : (i == 1 ? a[1] : (i == 2 ? a[2] : a[3])); }

// y = x shifted by s (+1/-1) along direction d (d may be a runtime value)
SUN_DEV void shifted(const Geom& g, const int x[4], int d, int s, int y[4])
{
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        int v = x[k] + (k == d ? s : 0);
        v = v < 0 ? v + g.X[k] : (v >= g.X[k] ? v - g.X[k] : v);
        y[k] = v;
    }
}

// ---------------------------------------------------------------------------
// Register caps of the update kernel (CTAs of 128 threads that must fit on an
// SM).  The update is latency-bound at the register-limited occupancy.
// Measured fastest for SU(3) on B200, with the phases overlapped:
// overrelaxation FP32 12-parameter 64 registers (8 CTAs, 32 warps per SM; no
// spills; 1.2 % faster than 72 and 2.4 % than 80), FP32 full and
// 8-parameter links 72 registers (7 CTAs; 64 spills them); heatbath FP32 102
// registers (5 CTAs, 2.5 % faster than uncapped; 4 and 6 CTAs are slower);
// overrelaxation FP64 168 registers (3 CTAs, 2 % faster); the FP64 heatbath
// is fastest uncapped.
#ifndef SUN_OCC_F32_OR12
#define SUN_OCC_F32_OR12 8
#endif
#ifndef SUN_OCC_F32_OR
#define SUN_OCC_F32_OR 7
#endif
#ifndef SUN_OCC_F32_HB
#define SUN_OCC_F32_HB 5
#endif
#ifndef SUN_OCC_F64_OR
#define SUN_OCC_F64_OR 3
#endif
#ifndef SUN_OCC_F64_HB
#define SUN_OCC_F64_HB 1
#endif
// N >= 4 in FP32: a 168-register cap (3 CTAs per SM) measured 18-28 % faster
// than the uncapped kernels (208-255 registers, 1-2 CTAs) at 24^4; FP64 and
// N = 2 are fastest uncapped.
// Per mode (SUN_OCC_SUN_OR / _HB): a 128-register cap (4 CTAs) measured
// slower for SU(4) FP32, overrelaxation 24^4 49.2 against 43.1 us per
// launch, heatbath 71.8 against 60.5 us (spills).
#ifndef SUN_OCC_SUN_OR
#define SUN_OCC_SUN_OR 3
#endif
#ifndef SUN_OCC_SUN_HB
#define SUN_OCC_SUN_HB 3
#endif
template <int N, class R, int MODE, int LAYOUT> struct UpdateOccupancy {
    static constexpr int min_blocks =
        (N >= 4 && sizeof(R) == 4) ? (MODE == MODE_OR ? SUN_OCC_SUN_OR : SUN_OCC_SUN_HB) : 1;
};
template <class R, int MODE, int LAYOUT> struct UpdateOccupancy<3, R, MODE, LAYOUT> {
    static constexpr bool f32 = sizeof(R) == 4;
    static constexpr int min_blocks =
        MODE == MODE_OR ? (f32 ? (LAYOUT == L_SOA12 ? SUN_OCC_F32_OR12 : SUN_OCC_F32_OR) : SUN_OCC_F64_OR)
                        : (f32 ? SUN_OCC_F32_HB : SUN_OCC_F64_HB);
};

// ---------------------------------------------------------------------------
// Where an update waits for the phase before it.  That phase wrote the links
// of direction dep = mu - 1 (mod 4), which only the staples of nu = dep
// read: the staples before it are summed while the previous phase drains,
// and the update waits (Dep::wait) just before the staple of nu = dep.
// GdcDep: a launch that may be a programmatic dependent of the previous
// phase (pdl != 0).  griddepcontrol.wait waits for that launch to complete,
// and only after it the next phase may launch (launch_dependents), so a
// launch never runs beside the one two back.  The resident sweeps wait on
// their grid's arrival count instead (ResidentDep).
struct GdcDep {
    int pdl;
    SUN_DEV int dep(int mu) const { return pdl ? ((mu + 3) & 3) : -1; }
    SUN_DEV void start(int dep) const
    {
        if (dep < 0) asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    }
    SUN_DEV void wait() const
    {
        asm volatile("griddepcontrol.wait;" ::: "memory");
        asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    }
};

// One link update of the checkerboard phase (parity, mu): half-site id of
// lattice L.  ld(i, e) returns element e of the link at image index i
// (complex element i + 4 V e) and st(i, e, v) writes it; dp: where and how
// to wait for the previous phase.
template <int N, class R, int LAYOUT, int MODE, class Dep, class Ld, class St>
SUN_DEV void update_site(const Geom& g, const LatDev& L, int id, int parity, int mu, unsigned hb_offset,
                         const InjView& inj, const Dep& dp, Ld&& ld, St&& st)
{
    typedef LinkIO<N, R, LAYOUT> IO;
    const uint32_t V = (uint32_t)g.V, stride = 4u * V;

    int x[4];
    eo_coords(g, id, parity, x);
    const int H = g.halfV;
    const int sx = id + parity * H;
    // neighbours by lexicographic stepping: lex +- stride_d with the periodic
    // wrap, then even/odd index (lex >> 1) + parity * V/2
    const int st_[4] = {1, g.X[0], g.X[0] * g.X[1], g.X[0] * g.X[1] * g.X[2]};
    const int lex = x[0] + st_[1] * x[1] + st_[2] * x[2] + st_[3] * x[3];
    const int xm = mu == 0 ? x[0] : (mu == 1 ? x[1] : (mu == 2 ? x[2] : x[3]));
    const int Xm = mu == 0 ? g.X[0] : (mu == 1 ? g.X[1] : (mu == 2 ? g.X[2] : g.X[3]));
    const int Sm = mu == 0 ? st_[0] : (mu == 1 ? st_[1] : (mu == 2 ? st_[2] : st_[3]));
    const int other = (1 - parity) * H;
    const int sxpmu = (lex_step(lex, xm, Xm, Sm, 1) >> 1) + other;

    const int dep = dp.dep(mu);
    dp.start(dep);
    Mat<N, R> S;
    mzero(S);
    // N <= 4: nu = mu+1, mu+2, mu+3 (mod 4), the staple of the previous
    // phase's direction last, so two thirds of the sum overlap the previous
    // launch; N = 6 keeps the reference's order (nu ascending, whose FP32
    // rounding its parity tolerance is set for)
    constexpr bool kRot = N <= 4;
#pragma unroll
    for (int kk = kRot ? 1 : 0; kk < 4; ++kk) {
        const int nu = kRot ? ((mu + kk) & 3) : kk;
        if (!kRot && nu == mu) continue;
        if (nu == dep) dp.wait();
        const int xn_ = kRot ? sel4(x, nu) : x[kk], Xn_ = kRot ? sel4(g.X, nu) : g.X[kk],
                  Sn_ = kRot ? sel4(st_, nu) : st_[kk];
        const int lup = lex_step(lex, xn_, Xn_, Sn_, 1);
        const int ldn = lex_step(lex, xn_, Xn_, Sn_, -1);
        const int syp = (lup >> 1) + other;                               // x + nu
        const int sy = (ldn >> 1) + other;                                // x - nu
        const int sz = (lex_step(ldn, xm, Xm, Sm, 1) >> 1) + parity * H;  // x - nu + mu
        Mat<N, R> A, B, C;
        if constexpr (N == 3 && LAYOUT == L_SOA12) {
            // 12-parameter links: a product of SU(3) links is SU(3), so only
            // its rows 0, 1 are multiplied out (from the stored rows of the
            // left factor, which is not rebuilt) and row 2 is rebuilt as
            // conj(row0 x row1).  Up: rows 0, 1 of the whole staple from
            // rows 0, 1 of U_nu(x) U_mu(x+nu), then its row 2, then added
            IO::load_rows_f(ld, sx + nu * V, stride, A);
            IO::load_f(ld, syp + mu * V, stride, B);
            mmul_rows01(A, B, C);
            IO::load_f(ld, sxpmu + nu * V, stride, A);
            mmul_nd_rows01(C, A, B);
            rebuild12(B);
            madd(S, B);
            // down: U_nu(x-nu)^dagger [U_mu(x-nu) U_nu(x-nu+mu)]
            IO::load_rows_f(ld, sy + mu * V, stride, A);
            IO::load_f(ld, sz + nu * V, stride, B);
            mmul_rows01(A, B, C);
            rebuild12(C);
            IO::load_f(ld, sy + nu * V, stride, A);
            macc_dn(A, C, S);
        } else {
            // up: U_nu(x) U_mu(x+nu) U_nu(x+mu)^dagger
            IO::load_f(ld, sx + nu * V, stride, A);
            IO::load_f(ld, syp + mu * V, stride, B);
            mmul(A, B, C);
            IO::load_f(ld, sxpmu + nu * V, stride, A);
            macc_nd(C, A, S);
            // down: U_nu(x-nu)^dagger U_mu(x-nu) U_nu(x-nu+mu)
            IO::load_f(ld, sy + nu * V, stride, A);
            IO::load_f(ld, sy + mu * V, stride, B);
            mmul_dn(A, B, C);
            IO::load_f(ld, sz + nu * V, stride, A);
            macc(C, A, S);
        }
    }

    const uint32_t own = (uint32_t)sx + (uint32_t)mu * V;
    Mat<N, R> U;
    IO::load_f(ld, own, stride, U);
    if constexpr (N == 3 && LAYOUT == L_SOA12) unit_row2<R>(U);
    if constexpr (MODE == MODE_OR) {
        overrelax_update<N, R, !(N == 3 && LAYOUT == L_SOA12)>(U, S);
    } else {
        const R bon = (R)L.beta_over_n;
        if constexpr (MODE == MODE_HB) {
            PhiloxStream<R> ph;
            ph.init(L.seed, (uint32_t)lex, (uint32_t)mu, L.state[0] + hb_offset);
            heatbath_update<N, R, PhiloxStream<R>, !(N == 3 && LAYOUT == L_SOA12)>(U, S, bon, ph);
        } else {
            InjectedStream<R> is;
            is.p = inj.u + ((size_t)lex * 4 + mu) * inj.stride;
            is.left = inj.stride;
            is.err = inj.err;
            heatbath_update<N, R, InjectedStream<R>, !(N == 3 && LAYOUT == L_SOA12)>(U, S, bon, is);
        }
    }
    IO::store_f(st, own, stride, U);
}

// Checkerboard update of the links (x, mu) with parity(x) == parity --
// kernel_PHeatBath_evenodd (src/monte/monte.cu:44-88) and
// kernel_overrelaxation_evenodd (src/monte/ovr.cu:41-80).  One thread per
// half-lattice site; the staples are summed "up" then "down" per nu, nu in
// the reference's ascending order for N = 6 and in the order mu+1, mu+2,
// mu+3 (mod 4) for N <= 4 (see update_site); all links are read through L2
// only (LD_CG: the launch overlaps the previous phase's).
template <int N, class R, int LAYOUT, int MODE>
__global__ void __launch_bounds__(128, (UpdateOccupancy<N, R, MODE, LAYOUT>::min_blocks)) k_update(BatchView bv, int parity, int mu, unsigned hb_offset,
                                                InjView inj, int pdl)
{
    const int b = blockIdx.x;
    const int l = find_lat(bv, b);
    const LatDev& L = bv.lats[l];
    const Geom g = geom_of(L);
    const int id = (b - __ldg(bv.begin + l)) * blockDim.x + threadIdx.x;
    if (id >= g.halfV || lat_frozen(L)) return;
    cx<R>* base = reinterpret_cast<cx<R>*>(L.links);
    const uint32_t stride = 4u * (uint32_t)g.V;
    update_site<N, R, LAYOUT, MODE>(
        g, L, id, parity, mu, hb_offset, inj, GdcDep{pdl},
        [&](uint32_t i, int e) { return ld_elem<R, LD_CG>(base + i + e * stride); },
        [&](uint32_t i, int e, cx<R> v) { st_elem<R>(base + i + e * stride, v); });
}

template <class R> SUN_DEV cx<R> shfl_cx(cx<R> v, int src)
{
    return mkc<R>(__shfl_sync(0xffffffffu, v.re, src), __shfl_sync(0xffffffffu, v.im, src));
}

// Row-split k_update for small lattices of larger N.  The N lanes of a site
// (32/N sites per warp) each multiply out one row of every staple product,
// the full neighbour links loaded by every lane (the repeats served by L1);
// the lanes then exchange their rows of the staple sum by warp shuffles, all
// run the same update on the same inputs, and lane 0 stores the link.  Per
// lane this holds far fewer live values than one thread per site (SU(6)
// FP32: no spills against 3.7 KB) and, on a lattice too small to fill the
// GPU, shortens each site's chain of dependent instructions.  Every element
// goes through the same operations in the same order as in k_update (the row
// routines of sun_math.cuh), so both kernels give the same bits and either
// may run any lattice.
// The row-split update of the warp whose first half-site is `first` (<
// halfV); dp as in update_site.
template <int N, class R, int LAYOUT, int MODE, class Dep>
SUN_DEV void update_rows_warp(const Geom& g, const LatDev& L, int first, int parity, int mu, unsigned hb_offset,
                              const InjView& inj, const Dep& dp)
{
    constexpr int SPW = 32 / N;  // sites per warp; lanes 32 - 32 % N .. 31 shadow the last site
    const int lane = threadIdx.x & 31;
    const int grp = lane / N;
    const bool used = grp < SPW;
    const int slot = used ? grp : SPW - 1;
    const int r = used ? lane - grp * N : lane % N;
    const int lead = slot * N;  // the lane holding row 0 of this site
    const int id0 = first + slot;
    const bool valid = used && id0 < g.halfV;
    const int id = id0 < g.halfV ? id0 : g.halfV - 1;  // past the end: compute a copy, store nothing
    typedef LinkIO<N, R, LAYOUT> IO;
    const cx<R>* base = reinterpret_cast<const cx<R>*>(L.links);
    const uint32_t V = (uint32_t)g.V, stride = 4u * V;

    int x[4];
    eo_coords(g, id, parity, x);
    const int H = g.halfV;
    const int sx = id + parity * H;
    const int st[4] = {1, g.X[0], g.X[0] * g.X[1], g.X[0] * g.X[1] * g.X[2]};
    const int lex = x[0] + st[1] * x[1] + st[2] * x[2] + st[3] * x[3];
    const int xm = mu == 0 ? x[0] : (mu == 1 ? x[1] : (mu == 2 ? x[2] : x[3]));
    const int Xm = mu == 0 ? g.X[0] : (mu == 1 ? g.X[1] : (mu == 2 ? g.X[2] : g.X[3]));
    const int Sm = mu == 0 ? st[0] : (mu == 1 ? st[1] : (mu == 2 ? st[2] : st[3]));
    const int other = (1 - parity) * H;
    const int sxpmu = (lex_step(lex, xm, Xm, Sm, 1) >> 1) + other;

    const int dep = dp.dep(mu);
    dp.start(dep);
    cx<R> Sr[N];  // row r of the staple sum
#pragma unroll
    for (int j = 0; j < N; ++j) Sr[j] = mkc<R>(0, 0);
    // N <= 4: nu = mu+1, mu+2, mu+3 (mod 4), the staple of the previous
    // phase's direction last, so two thirds of the sum overlap the previous
    // launch; N = 6 keeps the reference's order (nu ascending, whose FP32
    // rounding its parity tolerance is set for)
    constexpr bool kRot = N <= 4;
#pragma unroll
    for (int kk = kRot ? 1 : 0; kk < 4; ++kk) {
        const int nu = kRot ? ((mu + kk) & 3) : kk;
        if (!kRot && nu == mu) continue;
        if (nu == dep) dp.wait();
        const int xn_ = kRot ? sel4(x, nu) : x[kk], Xn_ = kRot ? sel4(g.X, nu) : g.X[kk],
                  Sn_ = kRot ? sel4(st, nu) : st[kk];
        const int lup = lex_step(lex, xn_, Xn_, Sn_, 1);
        const int ldn = lex_step(lex, xn_, Xn_, Sn_, -1);
        const int syp = (lup >> 1) + other;
        const int sy = (ldn >> 1) + other;
        const int sz = (lex_step(ldn, xm, Xm, Sm, 1) >> 1) + parity * H;
        Mat<N, R> A, B;
        cx<R> a[N], c[N];
        if constexpr (N == 3 && LAYOUT == L_SOA12) {
            // up: rows 0, 1 of the two-link product and then of the whole
            // staple by lanes 0, 1 (lane 2 repeats row 0), the staple's row 2
            // rebuilt from them in every lane
            cx<R> c0[3], c1[3], c2[3];
            IO::template load_rows<LD_CG>(base, sx + nu * V, stride, A);
            IO::template load<LD_CG>(base, syp + mu * V, stride, B);
            mrow<3, R, 2>(A, r, a);
            rmul<3, R>(a, B, c);
            IO::template load<LD_CG>(base, sxpmu + nu * V, stride, A);
            rmul_nd<3, R>(c, A, a);
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                c0[j] = shfl_cx(a[j], lead);
                c1[j] = shfl_cx(a[j], lead + 1);
            }
            rebuild12_row<R>(c0, c1, c2);
#pragma unroll
            for (int j = 0; j < 3; ++j) Sr[j] = Sr[j] + (r == 0 ? c0[j] : (r == 1 ? c1[j] : c2[j]));
            // down: U_nu(x-nu)^dagger [U_mu(x-nu) U_nu(x-nu+mu)], the product
            // needed whole
            IO::template load_rows<LD_CG>(base, sy + mu * V, stride, A);
            IO::template load<LD_CG>(base, sz + nu * V, stride, B);
            mrow<3, R, 2>(A, r, a);
            rmul<3, R>(a, B, c);
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                c0[j] = shfl_cx(c[j], lead);
                c1[j] = shfl_cx(c[j], lead + 1);
            }
            rebuild12_row<R>(c0, c1, c2);
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                B.e[0][j] = c0[j];
                B.e[1][j] = c1[j];
                B.e[2][j] = c2[j];
            }
            IO::template load<LD_CG>(base, sy + nu * V, stride, A);
            mcol<3, R>(A, r, a);
            racc_dn<3, R>(a, B, Sr);
        } else {
            IO::template load<LD_CG>(base, sx + nu * V, stride, A);
            IO::template load<LD_CG>(base, syp + mu * V, stride, B);
            mrow<N, R>(A, r, a);
            rmul<N, R>(a, B, c);
            IO::template load<LD_CG>(base, sxpmu + nu * V, stride, A);
            racc_nd<N, R>(c, A, Sr);
            IO::template load<LD_CG>(base, sy + nu * V, stride, A);
            IO::template load<LD_CG>(base, sy + mu * V, stride, B);
            mcol<N, R>(A, r, a);
            rmul_dn<N, R>(a, B, c);
            IO::template load<LD_CG>(base, sz + nu * V, stride, A);
            racc<N, R>(c, A, Sr);
        }
    }

    Mat<N, R> S;
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) S.e[i][j] = shfl_cx(Sr[j], lead + i);

    cx<R>* wbase = reinterpret_cast<cx<R>*>(L.links);
    const uint32_t own = (uint32_t)sx + (uint32_t)mu * V;
    Mat<N, R> U;
    IO::template load<LD_CG>(wbase, own, stride, U);
    if constexpr (N == 3 && LAYOUT == L_SOA12) unit_row2<R>(U);
    if constexpr (MODE == MODE_OR) {
        overrelax_update<N, R, !(N == 3 && LAYOUT == L_SOA12)>(U, S);
    } else {
        const R bon = (R)L.beta_over_n;
        if constexpr (MODE == MODE_HB) {
            PhiloxStream<R> st;
            st.init(L.seed, (uint32_t)lex, (uint32_t)mu, L.state[0] + hb_offset);
            heatbath_update<N, R, decltype(st), !(N == 3 && LAYOUT == L_SOA12)>(U, S, bon, st);
        } else {
            InjectedStream<R> st;
            st.p = inj.u + ((size_t)lex * 4 + mu) * inj.stride;
            st.left = inj.stride;
            st.err = inj.err;
            heatbath_update<N, R, decltype(st), !(N == 3 && LAYOUT == L_SOA12)>(U, S, bon, st);
        }
    }
    if (valid && r == 0) IO::store(wbase, own, stride, U);
}

template <int N, class R, int LAYOUT, int MODE>
__global__ void __launch_bounds__(128) k_update_rows(BatchView bv, int parity, int mu, unsigned hb_offset,
                                                     InjView inj, int pdl)
{
    constexpr int SPW = 32 / N;
    const int b = blockIdx.x;
    const int l = find_lat(bv, b);
    const LatDev& L = bv.lats[l];
    const Geom g = geom_of(L);
    const int first = (b - __ldg(bv.begin + l)) * ((int)(blockDim.x >> 5) * SPW) + (int)(threadIdx.x >> 5) * SPW;
    if (first >= g.halfV || lat_frozen(L)) return;  // the whole warp is past the end, or the lattice done
    update_rows_warp<N, R, LAYOUT, MODE>(g, L, first, parity, mu, hb_offset, inj, GdcDep{pdl});
}

// ---------------------------------------------------------------------------
// Tiled update for N >= 4 (full links): a CTA of N / RW warps advances 32
// half-sites, one per lane, and warp w owns the RW rows i = w RW .. w RW +
// RW - 1 (tile_rpw).  Per staple, a warp loads its rows (up staple) or
// columns (down staple) of the first factor straight into registers, and the
// CTA stages the other two factors once in shared memory (each warp loads its
// rows of them), so every link element is read from L2 exactly once and every
// load is a 32-lane coalesced one.  Each warp then forms its rows of the six
// staple products with the row routines of k_update_rows (same operations,
// same order: the same bits as k_update; one shared-memory read serves all
// the warp's rows) and keeps its rows of the staple sum in registers.  The
// SU(2) subgroup updates run in warp 0, one lane per site, streaming rows p
// and q of U and S from shared memory, so no thread ever holds an N x N
// matrix: SU(6) needs no spills at a modest register count, where one thread
// per site spills kilobytes.
//
// Shared memory (dynamic, tile_smem_bytes): B and D staging, N*N complex x
// 32 sites each; once the staples are summed, U takes the place of B and
// the staple sum S that of D.  Element e of a matrix sits at [e][lane]: a
// warp's access to one element is 32 consecutive complex numbers (no bank
// conflicts).  Measured on B200 (SU(6) sweeps): with S in a third array,
// FP64 24^4 took 17.4 ms against 14.8 ms (FP32 7.86 against 7.75 ms);
// CTAs of one 32-site tile per warp, each warp then updating its own tile
// so that none waits for warp 0, took 8.73 ms (FP32) and 19.2 ms (FP64):
// other CTAs already fill those waits, and the larger CTAs fit fewer per SM.
constexpr int kTileSites = 32;
template <int N, class R> constexpr int tile_smem_bytes() { return 2 * N * N * kTileSites * (int)sizeof(cx<R>); }
// CTAs per SM the tiled kernel's registers are capped for (FP32; 0: no cap,
// the compiler's own choice -- 72 registers for overrelaxation, 96 for the
// heatbath; FP64 is uncapped).  Caps for 4 to 6 CTAs per SM measured no
// faster (SU(6) 16^4, 24^4): other CTAs already fill the barrier waits while
// warp 0 of a CTA runs its SU(2) updates, and the kernel is issue-bound.
#ifndef SUN_TILE_OCC_OR
#define SUN_TILE_OCC_OR 0
#endif
#ifndef SUN_TILE_OCC_HB
#define SUN_TILE_OCC_HB 0
#endif
template <class R, int MODE> struct TileOccupancy {
    static constexpr int min_blocks = sizeof(R) == 4 ? (MODE == MODE_OR ? SUN_TILE_OCC_OR : SUN_TILE_OCC_HB) : 0;
};
// Rows of the link matrices per warp (N / rows warps per CTA): each element
// staged in shared memory is read once for all of a warp's rows, so more
// rows per warp mean fewer shared-memory reads and fewer, fuller warps.
// Measured on B200 (SU(6) sweeps, ms, 1 / 2 / 3 rows per warp, S in a
// third array): FP32 16^4 2.01 / 1.71 / 1.95, 24^4 9.60 / 7.86 / 7.79; FP64
// 16^4 4.59 / 4.31 / 3.51, 24^4 21.8 / 20.9 / 17.4.  With S in D's place:
// FP32 2 / 3 rows 12^4 0.67 / 0.76, 16^4 1.68 / 1.91, 24^4 7.84 / 7.52; FP64
// 3 / 2 rows 16^4 3.10 / 4.30, 24^4 14.9 / 20.8.  All give the same bits.
#ifndef SUN_TILE_RPW_F32
#define SUN_TILE_RPW_F32 2
#endif
#ifndef SUN_TILE_RPW_F64
#define SUN_TILE_RPW_F64 3
#endif
template <int N, class R> constexpr int tile_rpw()
{
    constexpr int r = sizeof(R) == 4 ? SUN_TILE_RPW_F32 : SUN_TILE_RPW_F64;
    return N % r == 0 ? r : (N % 2 == 0 ? 2 : 1);
}

template <int N, class R, int MODE>
__global__ void __launch_bounds__(32 * N / tile_rpw<N, R>(), (TileOccupancy<R, MODE>::min_blocks)) k_update_tile(
    BatchView bv, int parity, int mu, unsigned hb_offset, InjView inj, int pdl)
{
    static_assert(N >= 4, "the tiled update serves N >= 4");
    constexpr int RW = tile_rpw<N, R>();  // rows w RW .. w RW + RW - 1 belong to warp w
    typedef cx<R> C;
    extern __shared__ __align__(16) unsigned char tile_raw[];
    C(*const Bs)[kTileSites] = reinterpret_cast<C(*)[kTileSites]>(tile_raw);
    C(*const Ds)[kTileSites] = Bs + N * N;
    C(*const Ss)[kTileSites] = Ds;  // after the staple sum
    C(*const Us)[kTileSites] = Bs;
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    const int b = blockIdx.x;
    const int l = find_lat(bv, b);
    const LatDev& L = bv.lats[l];
    const Geom g = geom_of(L);
    if (lat_frozen(L)) return;  // the whole CTA: no barrier reached yet
    const int id0 = (b - __ldg(bv.begin + l)) * kTileSites + lane;
    const bool valid = id0 < g.halfV;
    const int id = valid ? id0 : g.halfV - 1;  // past the end: compute a copy, store nothing
    const cx<R>* base = reinterpret_cast<const cx<R>*>(L.links);
    const uint32_t V = (uint32_t)g.V, stride = 4u * V;

    int x[4];
    eo_coords(g, id, parity, x);
    const int H = g.halfV;
    const int sx = id + parity * H;
    const int st[4] = {1, g.X[0], g.X[0] * g.X[1], g.X[0] * g.X[1] * g.X[2]};
    const int lex = x[0] + st[1] * x[1] + st[2] * x[2] + st[3] * x[3];
    const int xm = sel4(x, mu), Xm = sel4(g.X, mu), Sm = sel4(st, mu);
    const int other = (1 - parity) * H;
    const int sxpmu = (lex_step(lex, xm, Xm, Sm, 1) >> 1) + other;

    const int dep = pdl ? ((mu + 3) & 3) : -1;  // as in k_update
    if (dep < 0) asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    auto Bget = [&](int k, int j) { return Bs[k * N + j][lane]; };
    auto Dget = [&](int k, int j) { return Ds[k * N + j][lane]; };
    C Sr[RW][N];
#pragma unroll
    for (int r = 0; r < RW; ++r)
#pragma unroll
        for (int j = 0; j < N; ++j) Sr[r][j] = mkc<R>(0, 0);
    // the order over nu of k_update: rotated for N = 4, ascending for N = 6
    constexpr bool kRot = N <= 4;
#pragma unroll 1
    for (int kk = kRot ? 1 : 0; kk < 4; ++kk) {
        const int nu = kRot ? ((mu + kk) & 3) : kk;
        if (nu == mu) continue;
        if (nu == dep) {
            asm volatile("griddepcontrol.wait;" ::: "memory");
            asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
        }
        const int xn_ = sel4(x, nu), Xn_ = sel4(g.X, nu), Sn_ = sel4(st, nu);
        const int lup = lex_step(lex, xn_, Xn_, Sn_, 1);
        const int ldn = lex_step(lex, xn_, Xn_, Sn_, -1);
        const int syp = (lup >> 1) + other;                               // x + nu
        const int sy = (ldn >> 1) + other;                                // x - nu
        const int sz = (lex_step(ldn, xm, Xm, Sm, 1) >> 1) + parity * H;  // x - nu + mu
        C a[RW][N], c[RW][N];
        // up: rows i of U_nu(x) U_mu(x+nu) U_nu(x+mu)^dagger
#pragma unroll
        for (int r = 0; r < RW; ++r)
#pragma unroll
            for (int k = 0; k < N; ++k) {
                const int i = w * RW + r;
                const uint32_t e = (uint32_t)(i * N + k) * stride;
                a[r][k] = ld_elem<R, LD_CG>(base + (uint32_t)sx + nu * V + e);
                Bs[i * N + k][lane] = ld_elem<R, LD_CG>(base + (uint32_t)syp + mu * V + e);
                Ds[i * N + k][lane] = ld_elem<R, LD_CG>(base + (uint32_t)sxpmu + nu * V + e);
            }
        __syncthreads();
        rmul_rows_g<N, RW, R>(a, Bget, c);
        racc_nd_rows_g<N, RW, R>(c, Dget, Sr);
        __syncthreads();
        // down: rows i of U_nu(x-nu)^dagger U_mu(x-nu) U_nu(x-nu+mu)
#pragma unroll
        for (int r = 0; r < RW; ++r)
#pragma unroll
            for (int k = 0; k < N; ++k) {
                const int i = w * RW + r;
                const uint32_t e = (uint32_t)(i * N + k) * stride;
                a[r][k] = ld_elem<R, LD_CG>(base + (uint32_t)sy + nu * V + (uint32_t)(k * N + i) * stride);
                Bs[i * N + k][lane] = ld_elem<R, LD_CG>(base + (uint32_t)sy + mu * V + e);
                Ds[i * N + k][lane] = ld_elem<R, LD_CG>(base + (uint32_t)sz + nu * V + e);
            }
        __syncthreads();
        rmul_dn_rows_g<N, RW, R>(a, Bget, c);
        racc_rows_g<N, RW, R>(c, Dget, Sr);
        __syncthreads();
    }

    cx<R>* wbase = reinterpret_cast<cx<R>*>(L.links);
    const uint32_t own = (uint32_t)sx + (uint32_t)mu * V;
#pragma unroll
    for (int r = 0; r < RW; ++r)
#pragma unroll
        for (int j = 0; j < N; ++j) {
            const int i = w * RW + r;
            Ss[i * N + j][lane] = Sr[r][j];
            Us[i * N + j][lane] = ld_elem<R, LD_CG>(wbase + own + (uint32_t)(i * N + j) * stride);
        }
    __syncthreads();
    if (w == 0) {
        // the subgroup sequence of overrelax_update / heatbath_update (N >= 4:
        // blocks of U S^dagger recomputed from U and S), rows from shared memory
        PhiloxStream<R> ph;
        InjectedStream<R> is;
        if constexpr (MODE == MODE_HB) ph.init(L.seed, (uint32_t)lex, (uint32_t)mu, L.state[0] + hb_offset);
        if constexpr (MODE == MODE_HB_INJECTED) {
            is.p = inj.u + ((size_t)lex * 4 + mu) * inj.stride;
            is.left = inj.stride;
            is.err = inj.err;
        }
        const R bon = (R)L.beta_over_n;
#pragma unroll 1
        for (int del = 1; del < N; ++del)
#pragma unroll 1
            for (int p = 0; p < N - del; ++p) {
                const int q = p + del;
                C a0 = mkc<R>(0, 0), a1 = a0, a2 = a0, a3 = a0;
#pragma unroll
                for (int j = 0; j < N; ++j) {
                    const C up = Us[p * N + j][lane], uq = Us[q * N + j][lane];
                    const C sp = Ss[p * N + j][lane], sq = Ss[q * N + j][lane];
                    a0 = cfma_nc(up, sp, a0);
                    a1 = cfma_nc(up, sq, a1);
                    a2 = cfma_nc(uq, sp, a2);
                    a3 = cfma_nc(uq, sq, a3);
                }
                R r[4] = {a0.re + a3.re, a1.im + a2.im, a1.re - a2.re, a0.im - a3.im};
                R cq[4];
                if constexpr (MODE == MODE_OR) {
                    su2_overrelax_element(r, cq);
                } else {
                    R k = sqrt(qnorm2(r));
                    R ap = bon * k;
                    k = R(1) / k;
                    r[0] *= k; r[1] *= k; r[2] *= k; r[3] *= k;
                    R ad[4];
                    if constexpr (MODE == MODE_HB) su2_draw<R>(ap, ph, ad);
                    else su2_draw<R>(ap, is, ad);
                    su2_mul_udag(ad, r, cq);
                }
                // su2_apply on rows p, q
                const C m00 = mkc(cq[0], cq[3]), m01 = mkc(cq[2], cq[1]);
                const C m10 = mkc(-cq[2], cq[1]), m11 = mkc(cq[0], -cq[3]);
#pragma unroll
                for (int j = 0; j < N; ++j) {
                    const C up = Us[p * N + j][lane], uq = Us[q * N + j][lane];
                    Us[p * N + j][lane] = cfma(m01, uq, m00 * up);
                    Us[q * N + j][lane] = cfma(m11, uq, m10 * up);
                }
            }
    }
    __syncthreads();
    if (valid) {
#pragma unroll
        for (int r = 0; r < RW; ++r)
#pragma unroll
            for (int j = 0; j < N; ++j) {
                const int i = w * RW + r;
                st_elem<R>(wbase + own + (uint32_t)(i * N + j) * stride, Us[i * N + j][lane]);
            }
    }
}

// ---------------------------------------------------------------------------
// Link-wise kernels: work index w over 4V links, w = site * 4 + mu with
// `site` in the lattice's storage order.
template <int N, class R, int LAYOUT>
__global__ void __launch_bounds__(256) k_cold(BatchView bv)
{
    const int b = blockIdx.x;
    const int l = find_lat(bv, b);
    const LatDev& L = bv.lats[l];
    const int w = (b - __ldg(bv.begin + l)) * blockDim.x + threadIdx.x;
    if (w >= 4 * L.V) return;
    Mat<N, R> U;
    munit(U);
    LinkIO<N, R, LAYOUT>::store(reinterpret_cast<cx<R>*>(L.links), (uint32_t)w, 4u * L.V, U);
}

// Haar-random SU(N) link (a new definition; the reference's hot start,
// gaugearray.cu:355, is uniform entries + reunitarization, not Haar): a
// complex Gaussian matrix from Philox stream (lex, mu | 1 << 8, pass 0) --
// entry (i,j) by Box-Muller on FP64 uniforms u1, u2 -- then modified
// Gram-Schmidt over columns (QR with positive diagonal) and the phase
// exp(-i arg(det)/N) onto SU(N).  Computed in FP64, stored in R.
template <int N, class R, int LAYOUT>
__global__ void __launch_bounds__(128) k_hot(BatchView bv)
{
    const int b = blockIdx.x;
    const int l = find_lat(bv, b);
    const LatDev& L = bv.lats[l];
    const Geom g = geom_of(L);
    const int s = (b - __ldg(bv.begin + l)) * blockDim.x + threadIdx.x;
    if (s >= g.V) return;
    int x[4];
    int site;
    if (L.evenodd) {
        const int par = s >= g.halfV;
        eo_coords(g, s - par * g.halfV, par, x);
        site = s;
    } else {
        lex_coords(g, s, x);
        site = s;
    }
    const int lex = lex_of(g, x);
    for (int mu = 0; mu < 4; ++mu) {
        PhiloxStream<double> st;
        st.init(L.seed, (uint32_t)lex, (uint32_t)mu | (1u << 8), 0u);
        Mat<N, double> Q;
#pragma unroll
        for (int i = 0; i < N; ++i)
#pragma unroll
            for (int j = 0; j < N; ++j) {
                double u1 = st.uniform();
                double u2 = st.uniform();
                double rad = sqrt(-2.0 * log(u1));
                double sn, cs;
                sincospi(2.0 * u2, &sn, &cs);
                Q.e[i][j] = mkc(rad * cs, rad * sn);
            }
#pragma unroll
        for (int j = 0; j < N; ++j) {
#pragma unroll
            for (int i = 0; i < j; ++i) {
                cx<double> d = mkc(0.0, 0.0);
#pragma unroll
                for (int c = 0; c < N; ++c) d = cfma_cn(Q.e[c][i], Q.e[c][j], d);
#pragma unroll
                for (int c = 0; c < N; ++c) Q.e[c][j] = Q.e[c][j] - d * Q.e[c][i];
            }
            double n = 0.0;
#pragma unroll
            for (int c = 0; c < N; ++c) n += cnorm2(Q.e[c][j]);
            n = 1.0 / sqrt(n);
#pragma unroll
            for (int c = 0; c < N; ++c) Q.e[c][j] = n * Q.e[c][j];
        }
        cx<double> d = mdet<N, double>(Q);
        double ph = atan2(d.im, d.re) / N;
        double sn, cs;
        sincos(ph, &sn, &cs);
        const cx<double> f = mkc(cs, -sn);
#pragma unroll
        for (int i = 0; i < N; ++i)
#pragma unroll
            for (int j = 0; j < N; ++j) Q.e[i][j] = Q.e[i][j] * f;
        Mat<N, R> U;
        mconvert(Q, U);
        LinkIO<N, R, LAYOUT>::store(reinterpret_cast<cx<R>*>(L.links), (uint32_t)site + (uint32_t)mu * g.V,
                                    4u * g.V, U);
    }
}

// FP64 reunitarization of every link -- kernel_calc_reunitarize
// (src/reunitarize.cu:23-31), always in double arithmetic.  Link w (image
// index) of lattice L, loaded through path P.
template <int N, class R, int LAYOUT, int P> SUN_DEV void reunit_link(const LatDev& L, int w)
{
    cx<R>* base = reinterpret_cast<cx<R>*>(L.links);
    Mat<N, R> U;
    LinkIO<N, R, LAYOUT>::template load<P>(base, (uint32_t)w, 4u * L.V, U);
    Mat<N, double> D;
    mconvert(U, D);
    reunit<N, double>(D);
    mconvert(D, U);
    LinkIO<N, R, LAYOUT>::store(base, (uint32_t)w, 4u * L.V, U);
}
template <int N, class R, int LAYOUT>
__global__ void __launch_bounds__(256) k_reunit(BatchView bv, int only_due)
{
    const int b = blockIdx.x;
    const int l = find_lat(bv, b);
    const LatDev& L = bv.lats[l];
    if (only_due) {
        // due after a sweep that advanced the lattice (not after the sweeps
        // a lattice at its sweep limit sits out)
        if (L.reunit_every <= 0 || L.state[2] == 0u) return;
        const unsigned sw = L.state[1];
        if (sw == 0u || (sw % (unsigned)L.reunit_every) != 0u) return;
    }
    const int w = (b - __ldg(bv.begin + l)) * blockDim.x + threadIdx.x;
    if (w >= 4 * L.V) return;
    reunit_link<N, R, LAYOUT, LD_CA>(L, w);
}

// ---------------------------------------------------------------------------
// Deterministic FP64 reductions: Neumaier/TwoSum-compensated pairs, reduced
// in a fixed tree (warp shuffles, then one warp over the warp results).
struct DD { double s, c; };
SUN_DEV DD dd_add(DD a, DD b)
{
    double s = a.s + b.s;
    double bb = s - a.s;
    double e = (a.s - (s - bb)) + (b.s - bb);
    DD r;
    r.s = s;
    r.c = (a.c + b.c) + e;
    return r;
}
SUN_DEV DD dd_warp(DD d)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        DD t;
        t.s = __shfl_down_sync(0xffffffffu, d.s, o);
        t.c = __shfl_down_sync(0xffffffffu, d.c, o);
        d = dd_add(d, t);
    }
    return d;
}
// reduces v over the CTA; thread 0 writes (sum, comp) to out[0..1]
SUN_DEV void block_sum(double v, double* out, DD* sh)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    DD d;
    d.s = v; d.c = 0.0;
    d = dd_warp(d);
    if (lane == 0) sh[warp] = d;
    __syncthreads();
    if (warp == 0) {
        DD t;
        if (lane < nw) t = sh[lane]; else { t.s = 0.0; t.c = 0.0; }
        t = dd_warp(t);
        if (lane == 0) { out[0] = t.s; out[1] = t.c; }
    }
    __syncthreads();
}
// Finalize of lattice l's CTA partials, run by the last of its CTAs to
// finish (each CTA fences its partials, then counts itself in): the same
// lane-strided compensated sums and shuffle tree as k_finalize_sum, so the
// result is the same whichever CTA runs it.  The result goes straight to
// out (host-mapped memory allowed); the counter is left at zero.  slot (may
// be null): a device counter; the results go to row *slot of out (nlat *
// nvals doubles per row), so a replayed graph fills one row per replay.
// The sums of CTA partials b0 .. b1 - 1 (nvals values each), by one warp
// (lane = threadIdx.x < 32): lane-strided compensated sums, then the shuffle
// tree; lane 0 writes value v to dst[v].
SUN_DEV void finalize_partials(const double* partials, int b0, int b1, int nvals, double* dst)
{
    const int lane = threadIdx.x;
    for (int v = 0; v < nvals; ++v) {
        DD d;
        d.s = 0.0; d.c = 0.0;
        for (int b = b0 + lane; b < b1; b += 32) {
            DD t;
            t.s = __ldcg(partials + ((size_t)b * nvals + v) * 2);
            t.c = __ldcg(partials + ((size_t)b * nvals + v) * 2 + 1);
            d = dd_add(d, t);
        }
        d = dd_warp(d);
        if (lane == 0) dst[v] = d.s + d.c;
    }
}
// Returns (in every thread) whether this CTA was the one that finalized.
SUN_DEV bool finalize_if_last(const BatchView& bv, int l, const double* partials, int nvals, double* out,
                              unsigned* counters, const unsigned* slot)
{
    __shared__ int last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned n = (unsigned)(__ldg(bv.begin + l + 1) - __ldg(bv.begin + l));
        last = atomicAdd(counters + l, 1u) == n - 1u;
    }
    __syncthreads();
    const bool mine = last != 0;
    if (!mine || threadIdx.x >= 32) return mine;
    __threadfence();
    const size_t row = slot ? (size_t)__ldcg(slot) * (size_t)bv.nlat * nvals : 0;
    finalize_partials(partials, __ldg(bv.begin + l), __ldg(bv.begin + l + 1), nvals, out + row + (size_t)l * nvals);
    if (threadIdx.x == 0) counters[l] = 0u;
    return mine;
}

SUN_DEV void block_max(double v, double* out, double* sh)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    if (warp == 0) {
        double t = lane < nw ? sh[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t = fmax(t, __shfl_down_sync(0xffffffffu, t, o));
        if (lane == 0) { out[0] = t; out[1] = 0.0; }
    }
    __syncthreads();
}

// site w of a sites-launch -> coordinates (storage order of the lattice)
SUN_DEV void site_coords(const LatDev& L, const Geom& g, int w, int x[4])
{
    if (L.evenodd) {
        const int par = w >= g.halfV;
        eo_coords(g, w - par * g.halfV, par, x);
    } else {
        lex_coords(g, w, x);
    }
}
SUN_DEV int site_index(const LatDev& L, const Geom& g, const int x[4])
{
    return L.evenodd ? eo_of(g, x) : lex_of(g, x);
}

template <int N, class R, int LAYOUT, int P = LD_NC>
SUN_DEV void load_d(const LatDev& L, const Geom& g, const int x[4], int mu, Mat<N, double>& D)
{
    Mat<N, R> A;
    LinkIO<N, R, LAYOUT>::template load<P>(reinterpret_cast<const cx<R>*>(L.links),
                                              (uint32_t)site_index(L, g, x) + (uint32_t)mu * g.V,
                                              4u * g.V, A);
    mconvert(A, D);
}

// Plaquette -- kernel_calc_plaquette_evenodd_cub / _normal_cub
// (src/meas/plaquette_cub.cu:47-145): per site sum over mu < nu of
// Re tr[U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag], nu == 3 temporal.
// Links are widened to FP64 before the products.  Lattices below
// kPlaneSplitMaxV sites take one thread per (site, plane), warp-major (a
// warp holds one plane of 32 consecutive sites, so its loads coalesce): a
// small lattice's launch then lasts one plaquette instead of six.  Larger
// lattices take one thread per site.  Sites are walked in lexicographic
// order whatever the storage order, so the neighbours x + mu, x + nu that a
// CTA reads are read by the CTAs beside it at about the same time (walking
// one even/odd block after the other fetched every link from DRAM twice).
template <int N, class R, int LAYOUT, int LP = LD_NC>
SUN_DEV double plaquette_plane(const LatDev& L, const Geom& g, const int x[4], int mu, int nu)
{
    int xm[4], xn[4];
    shifted(g, x, mu, 1, xm);
    shifted(g, x, nu, 1, xn);
    Mat<N, double> A, B, P, Q;
    load_d<N, R, LAYOUT, LP>(L, g, x, mu, A);
    load_d<N, R, LAYOUT, LP>(L, g, xm, nu, B);
    mmul(A, B, P);
    load_d<N, R, LAYOUT, LP>(L, g, x, nu, A);
    load_d<N, R, LAYOUT, LP>(L, g, xn, mu, B);
    mmul(A, B, Q);
    return mtrace_nd(P, Q).re;
}

// plaquette work item w of lattice L (thread w of k_plaquette's CTAs over
// the lattice): its spatial and temporal sums, links loaded through path P
template <int N, class R, int LAYOUT, int P>
SUN_DEV void plaquette_item(const LatDev& L, const Geom& g, int w, double& sp, double& tp)
{
    sp = 0.0;
    tp = 0.0;
    if (g.V < kPlaneSplitMaxV) {
        const int chunk = w / 192, r = w - 192 * chunk, plane = r >> 5;
        const int site = chunk * 32 + (r & 31);
        if (site < g.V) {
            const int mu = plane < 3 ? 0 : (plane < 5 ? 1 : 2);
            const int nu = plane < 3 ? plane + 1 : (plane < 5 ? plane - 1 : 3);
            int x[4];
            lex_coords(g, site, x);
            const double t = plaquette_plane<N, R, LAYOUT, P>(L, g, x, mu, nu);
            if (nu == 3) tp = t; else sp = t;
        }
    } else if (w < g.V) {
        int x[4];
        lex_coords(g, w, x);
#pragma unroll 1
        for (int mu = 0; mu < 3; ++mu)
#pragma unroll 1
            for (int nu = mu + 1; nu < 4; ++nu) {
                const double t = plaquette_plane<N, R, LAYOUT, P>(L, g, x, mu, nu);
                if (nu == 3) tp += t; else sp += t;
            }
    }
}

template <int N, class R, int LAYOUT>
__global__ void __launch_bounds__(128) k_plaquette(BatchView bv, double* partials, double* out, unsigned* counters,
                                                    const unsigned* slot)
{
    __shared__ DD sh[32];
    const int b = blockIdx.x;
    const int l = find_lat(bv, b);
    const LatDev& L = bv.lats[l];
    const Geom g = geom_of(L);
    const int w = (b - __ldg(bv.begin + l)) * blockDim.x + threadIdx.x;
    double sp, tp;
    plaquette_item<N, R, LAYOUT, LD_NC>(L, g, w, sp, tp);
    block_sum(sp, partials + (size_t)b * 4, sh);
    block_sum(tp, partials + (size_t)b * 4 + 2, sh);
    if (out) finalize_if_last(bv, l, partials, 2, out, counters, slot);
}

template <int N> SUN_DEV void shfl_mat(Mat<N, double>& D, const Mat<N, double>& S, int src)
{
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j)
            D.e[i][j] = mkc(__shfl_sync(0xffffffffu, S.e[i][j].re, src), __shfl_sync(0xffffffffu, S.e[i][j].im, src));
}

// Polyakov loop -- kernel_calc_polyakovloop_evenodd
// (src/meas/polyakovloop.cu:54-96): L = U_3(x,0) U_3(x,1) ... U_3(x,T-1),
// trace summed over spatial sites.  kPolyLanes (8) consecutive lanes per
// spatial site: lane k multiplies the links t in [k T / 8, (k + 1) T / 8)
// (an empty range gives the unit matrix), then the lane products are joined
// in order by a shuffle tree, (P0 P1)(P2 P3)..., so the time chain is T / 8
// products plus three joins instead of T products.
// Polyakov work item w of lattice L (thread w of k_polyakov's CTAs; all
// lanes of the warp take part): the trace at the site of lane k == 0, links
// loaded through path P
template <int N, class R, int LAYOUT, int P>
SUN_DEV void polyakov_item(const LatDev& L, const Geom& g, int w, double& re, double& im)
{
    const int V3 = g.X[0] * g.X[1] * g.X[2];
    const int site = w / kPolyLanes, k = w - kPolyLanes * site;
    const bool valid = site < V3;
    Mat<N, double> Pm, A, T;
    munit(Pm);
    if (valid) {
        int x[4];
        x[0] = site % g.X[0];
        x[1] = (site / g.X[0]) % g.X[1];
        x[2] = site / (g.X[0] * g.X[1]);
        const int t0 = k * g.X[3] / kPolyLanes, t1 = (k + 1) * g.X[3] / kPolyLanes;
#pragma unroll 1
        for (int t = t0; t < t1; ++t) {
            x[3] = t;
            load_d<N, R, LAYOUT, P>(L, g, x, 3, A);
            mmul(Pm, A, T);
            Pm = T;
        }
    }
    // blockDim is a multiple of 32 and of kPolyLanes: a site's lanes share a
    // warp, every lane of the warp takes part in the shuffles
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int step = 1; step < kPolyLanes; step <<= 1) {
        shfl_mat<N>(A, Pm, lane + step < 32 ? lane + step : lane);
        if ((k & (2 * step - 1)) == 0) {
            mmul(Pm, A, T);
            Pm = T;
        }
    }
    re = 0.0;
    im = 0.0;
    if (valid && k == 0) {
        const cx<double> tr = mtrace(Pm);
        re = tr.re;
        im = tr.im;
    }
}

template <int N, class R, int LAYOUT>
__global__ void __launch_bounds__(128) k_polyakov(BatchView bv, double* partials, double* out, unsigned* counters,
                                                   const unsigned* slot)
{
    __shared__ DD sh[32];
    const int b = blockIdx.x;
    const int l = find_lat(bv, b);
    const LatDev& L = bv.lats[l];
    const Geom g = geom_of(L);
    const int w = (b - __ldg(bv.begin + l)) * blockDim.x + threadIdx.x;
    double re, im;
    polyakov_item<N, R, LAYOUT, LD_NC>(L, g, w, re, im);
    block_sum(re, partials + (size_t)b * 4, sh);
    block_sum(im, partials + (size_t)b * 4 + 2, sh);
    if (out) finalize_if_last(bv, l, partials, 2, out, counters, slot);
}

// The plaquette and the Polyakov loop in one launch (the measurements of a
// replayed sweep-and-measure graph): CTAs below vp.nblocks are k_plaquette's,
// the others k_polyakov's, with the same partials and finalize, so the same
// bits; the two run side by side.  Each part's last CTA per lattice writes
// row *slot; the last of all the finalizing CTAs (joint counts them) then
// advances *slot for the next replay and, with end_n_hb >= 0, ends the sweep
// (the counters, which the measurements do not read).
template <int N, class R, int LAYOUT>
__global__ void __launch_bounds__(128) k_plaq_poly(BatchView vp, BatchView vl, double* part_p, double* part_l,
                                                    double* out_p, double* out_l, unsigned* cnt_p, unsigned* cnt_l,
                                                    unsigned* slot, unsigned* joint, int end_n_hb)
{
    __shared__ DD sh[32];
    const bool plaq = (int)blockIdx.x < vp.nblocks;
    const BatchView& bv = plaq ? vp : vl;
    const int b = plaq ? (int)blockIdx.x : (int)blockIdx.x - vp.nblocks;
    const int l = find_lat(bv, b);
    const LatDev& L = bv.lats[l];
    const Geom g = geom_of(L);
    const int w = (b - __ldg(bv.begin + l)) * blockDim.x + threadIdx.x;
    double v0, v1;
    if (plaq) plaquette_item<N, R, LAYOUT, LD_NC>(L, g, w, v0, v1);
    else polyakov_item<N, R, LAYOUT, LD_NC>(L, g, w, v0, v1);
    double* part = plaq ? part_p : part_l;
    block_sum(v0, part + (size_t)b * 4, sh);
    block_sum(v1, part + (size_t)b * 4 + 2, sh);
    const bool fin = finalize_if_last(bv, l, part, 2, plaq ? out_p : out_l, plaq ? cnt_p : cnt_l, slot);
    if (fin && threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(joint, 1u) == 2u * (unsigned)vp.nlat - 1u) {
            *joint = 0u;
            *slot += 1u;
            if (end_n_hb >= 0)
                for (int i = 0; i < vp.nlat; ++i) advance_counters(vp.lats[i], (unsigned)end_n_hb, 1u);
        }
    }
}

// Planar Wilson loops W(r,t), r <= R, t <= T, averaged over the 3 spatial
// directions -- kernel_WilsonLineSP + kernel_WilsonLoopSP
// (src/meas/wilsonloop.cu:60-128), without the V*3*R temporary of spatial
// lines: each thread keeps the T+1 spatial lines of its site in local
// memory and builds the temporal lines on the fly.
#define SUN_WMAX 8
template <int N, class R, int LAYOUT>
__global__ void __launch_bounds__(64) k_wilson(BatchView bv, int RR, int TT, double* partials)
{
    __shared__ DD sh[32];
    const int b = blockIdx.x;
    const int l = find_lat(bv, b);
    const LatDev& L = bv.lats[l];
    const Geom g = geom_of(L);
    const int w = (b - __ldg(bv.begin + l)) * blockDim.x + threadIdx.x;
    const int nres = (RR + 1) * (TT + 1);
    double acc[2 * (SUN_WMAX + 1) * (SUN_WMAX + 1)];
    for (int i = 0; i < 2 * nres; ++i) acc[i] = 0.0;
    if (w < g.V) {
        int x[4];
        lex_coords(g, w, x);  // lexicographic walk, as in k_plaquette
        Mat<N, double> Ls[SUN_WMAX + 1];
#pragma unroll 1
        for (int mu = 0; mu < 3; ++mu) {
#pragma unroll 1
            for (int t = 0; t <= TT; ++t) munit(Ls[t]);
#pragma unroll 1
            for (int r = 0; r <= RR; ++r) {
                if (r > 0) {
#pragma unroll 1
                    for (int t = 0; t <= TT; ++t) {
                        int y[4] = {x[0], x[1], x[2], x[3]};
                        y[3] = (x[3] + t) % g.X[3];
                        int c = y[0] * (mu == 0) + y[1] * (mu == 1) + y[2] * (mu == 2);
                        c = (c + r - 1) % g.X[mu];
                        if (mu == 0) y[0] = c; else if (mu == 1) y[1] = c; else y[2] = c;
                        Mat<N, double> A, T2;
                        load_d<N, R, LAYOUT>(L, g, y, mu, A);
                        mmul(Ls[t], A, T2);
                        Ls[t] = T2;
                    }
                }
                int xr[4] = {x[0], x[1], x[2], x[3]};
                {
                    int c = x[0] * (mu == 0) + x[1] * (mu == 1) + x[2] * (mu == 2);
                    c = (c + r) % g.X[mu];
                    if (mu == 0) xr[0] = c; else if (mu == 1) xr[1] = c; else xr[2] = c;
                }
                Mat<N, double> T0, T1, P, Q, A;
                munit(T0);
                munit(T1);
#pragma unroll 1
                for (int t = 0; t <= TT; ++t) {
                    // tr[L0 T1 Lt^dag T0^dag] = sum_ij (L0 T1)_ij conj((T0 Lt)_ij)
                    mmul(Ls[0], T1, P);
                    mmul(T0, Ls[t], Q);
                    const cx<double> wv = mtrace_nd(P, Q);
                    acc[2 * (t + r * (TT + 1))] += wv.re;
                    acc[2 * (t + r * (TT + 1)) + 1] += wv.im;
                    if (t < TT) {
                        int y[4] = {x[0], x[1], x[2], (x[3] + t) % g.X[3]};
                        load_d<N, R, LAYOUT>(L, g, y, 3, A);
                        mmul(T0, A, P);
                        T0 = P;
                        int z[4] = {xr[0], xr[1], xr[2], (x[3] + t) % g.X[3]};
                        load_d<N, R, LAYOUT>(L, g, z, 3, A);
                        mmul(T1, A, P);
                        T1 = P;
                    }
                }
            }
        }
    }
    for (int i = 0; i < 2 * nres; ++i) block_sum(acc[i], partials + ((size_t)b * 2 * nres + i) * 2, sh);
}

// max over links of max_ij |(U^dag U - 1)_ij| (FP64)
template <int N, class R, int LAYOUT>
__global__ void __launch_bounds__(256) k_unitarity(BatchView bv, double* partials);

// Link diagnostics -- the sums of GaugeTraceCUB / GaugeDetCUB
// (src/meas/linktrsum.cu, src/meas/linkdetsum.cu): per link tr U and det U in
// FP64, four compensated sums (Re tr, Im tr, Re det, Im det) per CTA.
template <int N, class R, int LAYOUT>
__global__ void __launch_bounds__(256) k_linkstats(BatchView bv, double* partials)
{
    __shared__ DD sh[32];
    const int b = blockIdx.x;
    const int l = find_lat(bv, b);
    const LatDev& L = bv.lats[l];
    const int w = (b - __ldg(bv.begin + l)) * blockDim.x + threadIdx.x;
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    if (w < 4 * L.V) {
        Mat<N, R> A;
        LinkIO<N, R, LAYOUT>::template load<true>(reinterpret_cast<const cx<R>*>(L.links), (uint32_t)w, 4u * L.V,
                                                  A);
        Mat<N, double> D;
        mconvert(A, D);
        const cx<double> t = mtrace(D);
        const cx<double> d = mdet<N, double>(D);
        v[0] = t.re; v[1] = t.im; v[2] = d.re; v[3] = d.im;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) block_sum(v[k], partials + ((size_t)b * 4 + k) * 2, sh);
}

template <int N, class R, int LAYOUT>
__global__ void __launch_bounds__(256) k_unitarity(BatchView bv, double* partials)
{
    __shared__ double sh[32];
    const int b = blockIdx.x;
    const int l = find_lat(bv, b);
    const LatDev& L = bv.lats[l];
    const int w = (b - __ldg(bv.begin + l)) * blockDim.x + threadIdx.x;
    double worst = 0.0;
    if (w < 4 * L.V) {
        Mat<N, R> A;
        LinkIO<N, R, LAYOUT>::template load<true>(reinterpret_cast<const cx<R>*>(L.links), (uint32_t)w,
                                                  4u * L.V, A);
        Mat<N, double> D, P;
        mconvert(A, D);
        mmul_dn(D, D, P);
#pragma unroll
        for (int i = 0; i < N; ++i)
#pragma unroll
            for (int j = 0; j < N; ++j) {
                cx<double> e = P.e[i][j];
                if (i == j) e.re -= 1.0;
                worst = fmax(worst, sqrt(cnorm2(e)));
            }
    }
    block_max(worst, partials + (size_t)b * 2, sh);
}

// canonical FP64 (site lex, mu, N*N row-major) <-> device image; work over
// 4V links with w = lex*4 + mu
template <int N, class R, int LAYOUT>
__global__ void __launch_bounds__(256) k_pack(BatchView bv, const double2* canon)
{
    const int b = blockIdx.x;
    const int l = find_lat(bv, b);
    const LatDev& L = bv.lats[l];
    const Geom g = geom_of(L);
    const int w = (b - __ldg(bv.begin + l)) * blockDim.x + threadIdx.x;
    if (w >= 4 * g.V) return;
    const int lex = w >> 2, mu = w & 3;
    int x[4];
    lex_coords(g, lex, x);
    Mat<N, R> U;
    const double2* src = canon + (size_t)w * N * N;
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) {
            double2 v = src[i * N + j];
            U.e[i][j] = mkc<R>((R)v.x, (R)v.y);
        }
    LinkIO<N, R, LAYOUT>::store(reinterpret_cast<cx<R>*>(L.links),
                                (uint32_t)site_index(L, g, x) + (uint32_t)mu * g.V, 4u * g.V, U);
}

template <int N, class R, int LAYOUT>
__global__ void __launch_bounds__(256) k_unpack(BatchView bv, double2* canon)
{
    const int b = blockIdx.x;
    const int l = find_lat(bv, b);
    const LatDev& L = bv.lats[l];
    const Geom g = geom_of(L);
    const int w = (b - __ldg(bv.begin + l)) * blockDim.x + threadIdx.x;
    if (w >= 4 * g.V) return;
    const int lex = w >> 2, mu = w & 3;
    int x[4];
    lex_coords(g, lex, x);
    Mat<N, R> U;
    LinkIO<N, R, LAYOUT>::template load<false>(reinterpret_cast<const cx<R>*>(L.links),
                                               (uint32_t)site_index(L, g, x) + (uint32_t)mu * g.V,
                                               4u * g.V, U);
    double2* dst = canon + (size_t)w * N * N;
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) dst[i * N + j] = make_double2((double)U.e[i][j].re, (double)U.e[i][j].im);
}

// ---------------------------------------------------------------------------
// Resident sweeps: one cooperative launch advances a lattice through many
// sweeps and measures it after each, with grid barriers where the launched
// path has launch boundaries (a small lattice's phase is a few microseconds,
// so the boundaries are a large share of it).  Each stage walks the
// decomposition of the kernel it stands for (an update phase's virtual CTA
// v on CTA v mod P of the set running the phase, a whole-grid stage's on CTA
// v mod grid), and every stage reads the links through L2 only (their lines
// in an SM's L1 may be stale after a barrier), so the links, the counters
// and the measurements have the bits of the launched path.
SUN_DEV unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
SUN_DEV unsigned ld_relaxed(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
SUN_DEV void fence_acq_rel() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
// spins of one barrier wait at most (a second bound beside wait_ns)
constexpr unsigned kBarrierMaxSpins = 1u << 24;

// Split grid barriers on one arrival count: barrier k is complete once
// *a.bar >= G (k + 1), G the grid size (the count only grows during a
// launch, so nothing is reset between barriers).  A CTA arrives when its
// part of the stage is done (its threads' writes, then one release fence and
// an atomic add by thread 0) and waits only where it needs the stage
// complete -- an update just before the staple of the direction the
// previous phase wrote, as a programmatic dependent launch does.  A wait
// polls with relaxed loads and ends with an acquire fence; it is bounded by
// a.wait_ns and kBarrierMaxSpins: one that runs out sets *a.status, every
// later wait then returns at once, and each CTA leaves at its next
// arrival.  Returns the count seen (0 when the wait failed).
SUN_DEV unsigned wait_count(const unsigned* count, unsigned target, int* status, unsigned long long wait_ns)
{
    unsigned c = ld_relaxed(count);
    if (c < target) {
        const unsigned long long t0 = global_ns();
        for (unsigned it = 0;; ++it) {
            c = ld_relaxed(count);
            if (c >= target) break;
            if (ld_relaxed(reinterpret_cast<const unsigned*>(status)) != 0u) return 0u;
            if (it >= kBarrierMaxSpins || global_ns() - t0 > wait_ns) {
                atomicExch(status, 1);
                return 0u;
            }
            if (it >= 64) __nanosleep(32);
        }
    }
    fence_acq_rel();
    return c;
}
// The waits of one update phase of a resident launch: `pre` the arrival
// count at which the phase two back is complete (before any staple),
// `dep_target` the count at which the previous phase is complete (before
// the staple of its direction); 0: nothing to wait for.  Called by all lanes of a warp at
// once: lane 0 polls (unless the CTA has seen the count already, *seen),
// records the count seen, and the warp proceeds together.
struct ResidentDep {
    const unsigned* count;
    int* status;
    unsigned long long wait_ns;
    unsigned pre, dep_target;
    unsigned* seen;
    SUN_DEV void wait_for(unsigned target) const
    {
        if ((threadIdx.x & 31) == 0) {
            if (*reinterpret_cast<volatile unsigned*>(seen) >= target) {
                // another warp saw the count (its acquire fence, then the
                // write of *seen); this fence makes the read an acquire
                __threadfence_block();
            } else {
                const unsigned c = wait_count(count, target, status, wait_ns);
                if (c) atomicMax(seen, c);
            }
        }
        __syncwarp();
    }
    SUN_DEV int dep(int mu) const { return dep_target ? ((mu + 3) & 3) : -1; }
    SUN_DEV void start(int) const
    {
        if (pre) wait_for(pre);
    }
    SUN_DEV void wait() const { wait_for(dep_target); }
};
// this CTA arrives at the barrier of the stage it has finished (its
// threads' writes, then a release fence and the count), once the arrival
// count has reached `need` (the stage before complete: seen by one of its
// warps already, or waited for here), so the arrivals of one barrier never
// run ahead of the barrier before.  The test hook: the CTA a.skip_arrive
// leaves at its first arrival without arriving.  False: leave.
SUN_DEV bool cta_arrive(const ResidentArgs& a, unsigned need, unsigned* seen, bool& first)
{
    __shared__ int go;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = !((int)blockIdx.x == a.skip_arrive && first);
        if (ok && *seen < need) {
            const unsigned c = wait_count(a.bar, need, a.status, a.wait_ns);
            if (c) *seen = c;
            ok = c != 0u;
        }
        if (ok) {
            fence_acq_rel();
            atomicAdd(a.bar, 1u);
        }
        go = ok;
    }
    first = false;
    __syncthreads();
    return go != 0;
}
// the whole CTA waits until the arrival count reaches target.  False: leave.
SUN_DEV bool cta_wait(const ResidentArgs& a, unsigned target, unsigned* seen)
{
    __shared__ int go;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned c = *seen >= target ? *seen : wait_count(a.bar, target, a.status, a.wait_ns);
        if (c) *seen = c;
        go = c != 0u;
    }
    __syncthreads();
    return go != 0;
}

// one update phase over the update decomposition, on the CTAs of one set
// (CTA rank r of P in the set walks virtual CTAs r, r + P, ...): ROWS the
// row-split body of k_update_rows (CTAs of 4 warps, 32 / N half-sites per
// warp), else one thread per half-site as k_update
template <int N, class R, int LAYOUT, int MODE, bool ROWS>
SUN_DEV void resident_phase(const ResidentArgs& a, const Geom& g, const LatDev& L, int parity, int mu,
                            unsigned hb_offset, const ResidentDep& dp, int rank, int P)
{
    const InjView none{nullptr, 0, nullptr};
    cx<R>* base = reinterpret_cast<cx<R>*>(L.links);
    const uint32_t stride = 4u * (uint32_t)g.V;
    for (int vb = rank; vb < a.upd.nblocks; vb += P) {
        if constexpr (ROWS) {
            constexpr int SPW = 32 / N;
            const int first = vb * ((int)(blockDim.x >> 5) * SPW) + (int)(threadIdx.x >> 5) * SPW;
            if (first < g.halfV) update_rows_warp<N, R, LAYOUT, MODE>(g, L, first, parity, mu, hb_offset, none, dp);
        } else {
            // every lane of a warp with work runs the update (the waits are
            // warp-wide); a lane past the end computes a copy of the last
            // half-site and stores nothing
            const int id0 = vb * (int)blockDim.x + (int)threadIdx.x;
            if (id0 - (int)(threadIdx.x & 31) < g.halfV) {
                const bool valid = id0 < g.halfV;
                update_site<N, R, LAYOUT, MODE>(
                    g, L, valid ? id0 : g.halfV - 1, parity, mu, hb_offset, none, dp,
                    [&](uint32_t i, int e) { return ld_elem<R, LD_CG>(base + i + e * stride); },
                    [&](uint32_t i, int e, cx<R> v) {
                        if (valid) st_elem<R>(base + i + e * stride, v);
                    });
            }
        }
    }
}

// The grid is two sets of P CTAs that take the update phases in turn, as
// launched phases overlap under programmatic dependent launch: set j mod 2
// runs phase j, summing the staples that do not read the previous phase's
// direction while phase j - 1 still runs on the other set, and waiting for
// it only before the last staple.  Barrier arithmetic: every CTA tracks
// `done`, the arrival count at which the latest barrier completes, and
// `prev` the one before; a phase adds P arrivals, a stage run by the whole
// grid (reunitarization, measurements) adds 2 P.
template <int N, class R, int LAYOUT, bool ROWS>
__global__ void __launch_bounds__(128) k_sweeps_resident(ResidentArgs a)
{
    __shared__ DD sh[32];
    __shared__ unsigned seen;  // the largest arrival count this CTA has seen reached
    if (threadIdx.x == 0) seen = 0u;
    __syncthreads();
    const LatDev& L = a.upd.lats[0];
    const Geom g = geom_of(L);
    const unsigned P = gridDim.x / 2u;
    const int set = blockIdx.x >= P, rank = (int)blockIdx.x - set * (int)P;
    unsigned done = 0u, prev = 0u;
    bool first = true;
    // the counters stay as they were during the launch (the heatbath pass of
    // sweep i is the lattice's pass count plus i n_hb + h, as the launched
    // path counts it); CTA 0 advances them at the end
    const unsigned sweeps0 = __ldcg(L.state + 1);
    for (int sw = 0; sw < a.n_sweeps; ++sw) {
        int j = 0;  // phase of the sweep (8 per pass: an even count, so each sweep starts on set 0)
        for (int pass = 0; pass < a.n_hb + a.n_or; ++pass) {
            const bool hb = pass < a.n_hb;
            const unsigned off = hb ? (unsigned)(sw * a.n_hb + pass) : 0u;
            for (int par = 0; par < 2; ++par)
                for (int mu = 0; mu < 4; ++mu, ++j) {
                    if ((j & 1) == set) {
                        const ResidentDep dp{a.bar, a.status, a.wait_ns, prev, done, &seen};
                        if (hb) resident_phase<N, R, LAYOUT, MODE_HB, ROWS>(a, g, L, par, mu, off, dp, rank, (int)P);
                        else resident_phase<N, R, LAYOUT, MODE_OR, ROWS>(a, g, L, par, mu, 0u, dp, rank, (int)P);
                        if (!cta_arrive(a, done, &seen, first)) return;
                    }
                    prev = done;
                    done += P;
                }
        }
        // reunitarization on the lattice's schedule, as k_reunit(only_due)
        const unsigned swn = sweeps0 + (unsigned)sw + 1u;
        if (L.reunit_every > 0 && swn % (unsigned)L.reunit_every == 0u) {
            if (!cta_wait(a, done, &seen)) return;
            for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < 4 * g.V; w += gridDim.x * blockDim.x)
                reunit_link<N, R, LAYOUT, LD_CG>(L, w);
            if (!cta_arrive(a, done, &seen, first)) return;
            prev = done;
            done += gridDim.x;
        }
        // plaquette and Polyakov loop, partials of k_plaquette's and
        // k_polyakov's CTAs, finalized as their last CTA does
        if (!cta_wait(a, done, &seen)) return;
        double* ppart = a.partials + (size_t)a.plaq.nblocks * 4;
        for (int vb = blockIdx.x; vb < a.plaq.nblocks; vb += gridDim.x) {
            double sp, tp;
            plaquette_item<N, R, LAYOUT, LD_CG>(L, g, vb * (int)blockDim.x + (int)threadIdx.x, sp, tp);
            block_sum(sp, a.partials + (size_t)vb * 4, sh);
            block_sum(tp, a.partials + (size_t)vb * 4 + 2, sh);
        }
        for (int vb = blockIdx.x; vb < a.poly.nblocks; vb += gridDim.x) {
            double re, im;
            polyakov_item<N, R, LAYOUT, LD_CG>(L, g, vb * (int)blockDim.x + (int)threadIdx.x, re, im);
            block_sum(re, ppart + (size_t)vb * 4, sh);
            block_sum(im, ppart + (size_t)vb * 4 + 2, sh);
        }
        if (!cta_arrive(a, done, &seen, first)) return;
        prev = done;
        done += gridDim.x;
        if (!cta_wait(a, done, &seen)) return;
        // finalized by two CTAs of set 1, which starts the next sweep second;
        // the partials are written again only after the next sweep's
        // barriers, which these CTAs reach after their finalize
        if (blockIdx.x == P && threadIdx.x < 32) finalize_partials(a.partials, 0, a.plaq.nblocks, 2, a.out_plaq + 2 * sw);
        if (blockIdx.x == gridDim.x - 1 && threadIdx.x < 32) finalize_partials(ppart, 0, a.poly.nblocks, 2, a.out_poly + 2 * sw);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        L.state[0] += (unsigned)(a.n_sweeps * a.n_hb);
        L.state[1] += (unsigned)a.n_sweeps;
        L.state[2] = 1u;
    }
}

// ---------------------------------------------------------------------------
// Host launch wrappers: runtime (precision, layout) -> template instance.
// SOA12 and SOA8 exist for N == 3 only (the reference silently falls back to
// SOA for other N, gaugearray.h:127-137; the C ABI rejects them instead).
#define SUN_DISPATCH(FP64, LAYOUT, CALL)                                            \
    do {                                                                            \
        if constexpr (N == 3) {                                                     \
            if ((LAYOUT) == L_SOA12) {                                              \
                if (FP64) { CALL(double, L_SOA12); } else { CALL(float, L_SOA12); } \
            } else if ((LAYOUT) == L_SOA8) {                                        \
                if (FP64) { CALL(double, L_SOA8); } else { CALL(float, L_SOA8); }   \
            } else {                                                                \
                if (FP64) { CALL(double, L_SOA); } else { CALL(float, L_SOA); }     \
            }                                                                       \
        } else {                                                                    \
            if (FP64) { CALL(double, L_SOA); } else { CALL(float, L_SOA); }         \
        }                                                                           \
    } while (0)

// One update launch; pdl: as a programmatic dependent of the launch before
// it on the stream (which must be the previous update phase).
template <class K>
cudaError_t launch_phase(K kernel, const BatchView& bv, int block, int parity, int mu, unsigned hb_offset,
                         const InjView& inj, int pdl, cudaStream_t s, int smem = 0)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)bv.nblocks);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = (size_t)smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, bv, parity, mu, hb_offset, inj, pdl);
}

template <int N>
cudaError_t Ops<N>::update(int fp64, int layout, int mode, const BatchView& bv, int block, int parity, int mu,
                           unsigned hb_offset, const InjView& inj, int pdl, cudaStream_t s)
{
    cudaError_t e = cudaSuccess;
#define CALL(R_, L_)                                                                                          \
    if (mode == MODE_OR) e = launch_phase(k_update<N, R_, L_, MODE_OR>, bv, block, parity, mu, hb_offset, inj, pdl, s); \
    else if (mode == MODE_HB) e = launch_phase(k_update<N, R_, L_, MODE_HB>, bv, block, parity, mu, hb_offset, inj, pdl, s); \
    else e = launch_phase(k_update<N, R_, L_, MODE_HB_INJECTED>, bv, block, parity, mu, hb_offset, inj, pdl, s)
    SUN_DISPATCH(fp64, layout, CALL);
#undef CALL
    return e != cudaSuccess ? e : cudaGetLastError();
}

template <int N>
cudaError_t Ops<N>::update_rows(int fp64, int layout, int mode, const BatchView& bv, int block, int parity, int mu,
                                unsigned hb_offset, const InjView& inj, int pdl, cudaStream_t s)
{
    cudaError_t e = cudaSuccess;
#define CALL(R_, L_)                                                                                               \
    if (mode == MODE_OR) e = launch_phase(k_update_rows<N, R_, L_, MODE_OR>, bv, block, parity, mu, hb_offset, inj, pdl, s); \
    else if (mode == MODE_HB) e = launch_phase(k_update_rows<N, R_, L_, MODE_HB>, bv, block, parity, mu, hb_offset, inj, pdl, s); \
    else e = launch_phase(k_update_rows<N, R_, L_, MODE_HB_INJECTED>, bv, block, parity, mu, hb_offset, inj, pdl, s)
    SUN_DISPATCH(fp64, layout, CALL);
#undef CALL
    return e != cudaSuccess ? e : cudaGetLastError();
}

// the tiled update's instance for (R, MODE), its shared memory opted in once
template <int N, class R, int MODE> cudaError_t launch_tile(const BatchView& bv, int parity, int mu,
                                                            unsigned hb_offset, const InjView& inj, int pdl,
                                                            cudaStream_t s)
{
    constexpr int smem = tile_smem_bytes<N, R>();
    // the dynamic size opted in above 48 KB.  The shared-memory carve-out is
    // left to the driver: forcing the largest one measured slower (SU(6)
    // 24^4 FP64 21.7 -> 38.0 ms per sweep, FP32 9.6 -> 10.7 ms).
    static const cudaError_t attr =
        smem > 48 * 1024
            ? cudaFuncSetAttribute(k_update_tile<N, R, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)
            : cudaSuccess;
    if (attr != cudaSuccess) return attr;
    return launch_phase(k_update_tile<N, R, MODE>, bv, 32 * N / tile_rpw<N, R>(), parity, mu, hb_offset, inj, pdl, s,
                        smem);
}

template <int N>
cudaError_t Ops<N>::update_tile(int fp64, int layout, int mode, const BatchView& bv, int parity, int mu,
                                unsigned hb_offset, const InjView& inj, int pdl, cudaStream_t s)
{
    if constexpr (N < 4) {
        return cudaErrorInvalidValue;
    } else {
        if (layout != L_SOA) return cudaErrorInvalidValue;
        cudaError_t e;
        if (fp64) {
            if (mode == MODE_OR) e = launch_tile<N, double, MODE_OR>(bv, parity, mu, hb_offset, inj, pdl, s);
            else if (mode == MODE_HB) e = launch_tile<N, double, MODE_HB>(bv, parity, mu, hb_offset, inj, pdl, s);
            else e = launch_tile<N, double, MODE_HB_INJECTED>(bv, parity, mu, hb_offset, inj, pdl, s);
        } else {
            if (mode == MODE_OR) e = launch_tile<N, float, MODE_OR>(bv, parity, mu, hb_offset, inj, pdl, s);
            else if (mode == MODE_HB) e = launch_tile<N, float, MODE_HB>(bv, parity, mu, hb_offset, inj, pdl, s);
            else e = launch_tile<N, float, MODE_HB_INJECTED>(bv, parity, mu, hb_offset, inj, pdl, s);
        }
        return e != cudaSuccess ? e : cudaGetLastError();
    }
}

template <int N>
cudaError_t Ops<N>::sweeps_resident(int fp64, int layout, int rows, const ResidentArgs& a, int grid, cudaStream_t s)
{
    if constexpr (N > 4) {
        return cudaErrorInvalidValue;  // N = 6 runs the tiled update, which has no resident form
    } else {
        cudaError_t e = cudaSuccess;
        ResidentArgs args = a;
        void* params[] = {&args};
#define CALL(R_, L_)                                                                                             \
    e = rows ? cudaLaunchCooperativeKernel((const void*)k_sweeps_resident<N, R_, L_, true>, dim3(grid), dim3(128), \
                                           params, 0, s)                                                          \
             : cudaLaunchCooperativeKernel((const void*)k_sweeps_resident<N, R_, L_, false>, dim3(grid),          \
                                           dim3(128), params, 0, s)
        SUN_DISPATCH(fp64, layout, CALL);
#undef CALL
        return e != cudaSuccess ? e : cudaGetLastError();
    }
}

template <int N> int Ops<N>::resident_capacity(int fp64, int layout, int rows)
{
    if constexpr (N > 4) {
        return 0;
    } else {
        int dev = 0, sms = 0, per = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            return 0;
        cudaError_t e = cudaSuccess;
#define CALL(R_, L_)                                                                                            \
    e = rows ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_sweeps_resident<N, R_, L_, true>, 128, 0) \
             : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_sweeps_resident<N, R_, L_, false>, 128, 0)
        SUN_DISPATCH(fp64, layout, CALL);
#undef CALL
        return e == cudaSuccess ? per * sms : 0;
    }
}

template <int N> cudaError_t Ops<N>::cold(int fp64, int layout, const BatchView& bv, int block, cudaStream_t s)
{
#define CALL(R_, L_) k_cold<N, R_, L_><<<bv.nblocks, block, 0, s>>>(bv)
    SUN_DISPATCH(fp64, layout, CALL);
#undef CALL
    return cudaGetLastError();
}

template <int N> cudaError_t Ops<N>::hot(int fp64, int layout, const BatchView& bv, int block, cudaStream_t s)
{
#define CALL(R_, L_) k_hot<N, R_, L_><<<bv.nblocks, block, 0, s>>>(bv)
    SUN_DISPATCH(fp64, layout, CALL);
#undef CALL
    return cudaGetLastError();
}

template <int N>
cudaError_t Ops<N>::reunit(int fp64, int layout, const BatchView& bv, int block, int only_due, cudaStream_t s)
{
#define CALL(R_, L_) k_reunit<N, R_, L_><<<bv.nblocks, block, 0, s>>>(bv, only_due)
    SUN_DISPATCH(fp64, layout, CALL);
#undef CALL
    return cudaGetLastError();
}

template <int N>
cudaError_t Ops<N>::plaquette(int fp64, int layout, const BatchView& bv, int block, double* partials,
                              double* out, unsigned* counters, const unsigned* slot, cudaStream_t s)
{
#define CALL(R_, L_) k_plaquette<N, R_, L_><<<bv.nblocks, block, 0, s>>>(bv, partials, out, counters, slot)
    SUN_DISPATCH(fp64, layout, CALL);
#undef CALL
    return cudaGetLastError();
}

template <int N>
cudaError_t Ops<N>::polyakov(int fp64, int layout, const BatchView& bv, int block, double* partials,
                             double* out, unsigned* counters, const unsigned* slot, cudaStream_t s)
{
#define CALL(R_, L_) k_polyakov<N, R_, L_><<<bv.nblocks, block, 0, s>>>(bv, partials, out, counters, slot)
    SUN_DISPATCH(fp64, layout, CALL);
#undef CALL
    return cudaGetLastError();
}

template <int N>
cudaError_t Ops<N>::plaq_poly(int fp64, int layout, const BatchView& vp, const BatchView& vl, double* part_p,
                              double* part_l, double* out_p, double* out_l, unsigned* cnt_p, unsigned* cnt_l,
                              unsigned* slot, unsigned* joint, int end_n_hb, cudaStream_t s)
{
#define CALL(R_, L_)                                                                                          \
    k_plaq_poly<N, R_, L_><<<vp.nblocks + vl.nblocks, 128, 0, s>>>(vp, vl, part_p, part_l, out_p, out_l, cnt_p, \
                                                                    cnt_l, slot, joint, end_n_hb)
    SUN_DISPATCH(fp64, layout, CALL);
#undef CALL
    return cudaGetLastError();
}

template <int N>
cudaError_t Ops<N>::wilson(int fp64, int layout, const BatchView& bv, int block, int R, int T, double* partials,
                           cudaStream_t s)
{
#define CALL(R_, L_) k_wilson<N, R_, L_><<<bv.nblocks, block, 0, s>>>(bv, R, T, partials)
    SUN_DISPATCH(fp64, layout, CALL);
#undef CALL
    return cudaGetLastError();
}

template <int N>
cudaError_t Ops<N>::unitarity(int fp64, int layout, const BatchView& bv, int block, double* partials,
                              cudaStream_t s)
{
#define CALL(R_, L_) k_unitarity<N, R_, L_><<<bv.nblocks, block, 0, s>>>(bv, partials)
    SUN_DISPATCH(fp64, layout, CALL);
#undef CALL
    return cudaGetLastError();
}

template <int N>
cudaError_t Ops<N>::linkstats(int fp64, int layout, const BatchView& bv, int block, double* partials,
                              cudaStream_t s)
{
#define CALL(R_, L_) k_linkstats<N, R_, L_><<<bv.nblocks, block, 0, s>>>(bv, partials)
    SUN_DISPATCH(fp64, layout, CALL);
#undef CALL
    return cudaGetLastError();
}

template <int N>
cudaError_t Ops<N>::pack(int fp64, int layout, const BatchView& bv, int block, const void* canon, cudaStream_t s)
{
#define CALL(R_, L_) k_pack<N, R_, L_><<<bv.nblocks, block, 0, s>>>(bv, reinterpret_cast<const double2*>(canon))
    SUN_DISPATCH(fp64, layout, CALL);
#undef CALL
    return cudaGetLastError();
}

template <int N>
cudaError_t Ops<N>::unpack(int fp64, int layout, const BatchView& bv, int block, void* canon, cudaStream_t s)
{
#define CALL(R_, L_) k_unpack<N, R_, L_><<<bv.nblocks, block, 0, s>>>(bv, reinterpret_cast<double2*>(canon))
    SUN_DISPATCH(fp64, layout, CALL);
#undef CALL
    return cudaGetLastError();
}

}  // namespace sunb

#include "sun_smear.cuh"
