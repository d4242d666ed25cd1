// flow.cu -- shallow-water step on the staggered grid (flowstep,
// Wave_gpu.cu:1106-1403; kernels of Flow_kernel.cu) in four fused passes
// (k_flow_uv) or five (k_flow_u and k_flow_v apart).
// Each pass cuts where the reference reads a field that an earlier launch of
// the same step rewrote at a neighbouring cell; inside a pass, neighbour
// values of per-cell intermediates are recomputed instead of stored.
//
//   k_flow_a     udepthmomcont, vdepthmomcont, smago  -> hum hvm wetu wetv nuh
//   k_flow_u     wlevslopes(x), ududx_adv, vdudy_adv, viscou1+2, eulerustep,
//                latbnd(uu)                           -> uu*
//   k_flow_v     wlevslopes(y), vdvdy_adv, udvdx_adv, viscov1+2, eulervstep,
//                vvlatbnd                             -> vv*
//   k_flow_uv    k_flow_u and k_flow_v in one pass (uu* of the tile and its
//                ring in shared memory)               -> uu* vv*
//   k_flow_corr  wrkuu2Ocorr+uu2Ocorr, wrkvv2Ocorr+vv2Ocorr, then depthhu,
//                depthhv, CalcQFlow, continuity      -> uu vv hu hv qx qy zs* dzsdt
//   k_flow_final wrkzs2Ocorr+zs2Ocorr, latbnd(zs), hsbnd, calcuvvu, uvlatbnd
// (* = a per-step buffer).  viscovbnd (Flow_kernel.cu:1461) changes viscv only
// at rows 0 and ny-2, whose eulervstep results vvlatbnd then overwrites, so it
// has no effect on the state and is not evaluated.  Quotients by the grid
// spacing are products with its reciprocal (within an ulp of the reference's
// float division).
#include "xbg_common.cuh"

namespace xbg {

template <class R>
__device__ __forceinline__ R minmod(R d1, R d2) {   // Flow_kernel.cu:23-41
    R r = (R)0.0f;
    if (d1 * d2 > (R)0.0f) {
        if (d1 > (R)0.0f) r = DM<R>::fmin(d1, d2);
        if (d1 < (R)0.0f) r = DM<R>::fmax(d1, d2);
    }
    return r;
}

#define IDX(x, y) ((x) + (y) * nx)

// the block tile of the staged passes (32 x 8 cells) and its one-cell ring
constexpr int FT_X = 32, FT_Y = 8, FT_TX = FT_X + 2, FT_TY = FT_Y + 2, FT_N = FT_TX * FT_TY;
constexpr int FC_H = 3;   // tile halo of the momentum-correction pass

// smago (Flow_kernel.cu:1282-1316) from its inputs: depth and DR of the
// cell; uu at the cell and its left (xm), upper (yp), lower (ym), upper-left
// and lower-left neighbours; vv at the cell and its lower, right, left,
// lower-right and lower-left neighbours (mm/pp-clamped at the grid edges)
template <class R>
struct SmagoIn { R h, dr, u, uxm, uyp, uym, uxmyp, uxmym, v, vym, vxp, vxm, vxpym, vxmym; };
template <class R>
__device__ __forceinline__ R smago_of(const Konst<R>& K, const SmagoIn<R>& a) {
    R dx = K.dx, rdx = K.rdx, nuh = K.nuh, nuhfac = K.nuhfac, rho = K.rho;
    R b = nuhfac * a.h * DM<R>::pow13(a.dr / rho);
    if (K.usesmago == 1) {
        R dudx = (a.u - a.uxm) * rdx;
        R dudy = (R)0.50f * (a.uyp - a.uym + a.uxmyp - a.uxmym) * rdx;
        R dvdy = (a.v - a.vym) * rdx;
        R dvdx = (R)0.50f * (a.vxp - a.vxm + a.vxpym - a.vxmym) * rdx;
        R tau = DM<R>::sqrt((R)2.0f * dudx * dudx + (R)2.0f * dvdy * dvdy + (dudy + dvdx) * (dudy + dvdx));
        return DM<R>::fmax(nuh * nuh * dx * dx * tau, b);
    }
    return DM<R>::fmax(nuh, b);
}
// smago at cell (ix, iy)
template <class R>
__device__ __forceinline__ R smago_cell(const Dev<R>& S, const Konst<R>& K, int ix, int iy) {
    const int nx = K.nx, ny = K.ny;
    const R* uu = S.f[UU]; const R* vv = S.f[VV];
    int i = IDX(ix, iy), xm = mm(ix), xp = pp(ix, nx), ym = mm(iy), yp = pp(iy, ny);
    SmagoIn<R> a{};
    a.h = ld(S.f[HH] + i);
    a.dr = ld(S.f[DR] + i);
    if (K.usesmago == 1) {
        a.u = ld(uu + i); a.uxm = ld(uu + IDX(xm, iy)); a.uyp = ld(uu + IDX(ix, yp)); a.uym = ld(uu + IDX(ix, ym));
        a.uxmyp = ld(uu + IDX(xm, yp)); a.uxmym = ld(uu + IDX(xm, ym));
        a.v = ld(vv + i); a.vym = ld(vv + IDX(ix, ym)); a.vxp = ld(vv + IDX(xp, iy)); a.vxm = ld(vv + IDX(xm, iy));
        a.vxpym = ld(vv + IDX(xp, ym)); a.vxmym = ld(vv + IDX(xm, ym));
    }
    return smago_of(K, a);
}

// udepthmomcont / vdepthmomcont (Flow_kernel.cu:653-750) from the cell's
// depth, its right and upper neighbours' and the cell's hu, hv
template <class R>
struct DepthMom { R humi, hvmi; int wu, wv; };
template <class R>
__device__ __forceinline__ DepthMom<R> depthmom_of(const Konst<R>& K, R hh, R hhxp, R hhyp, R hu, R hv) {
    const R eps = K.eps;
    DepthMom<R> o;
    o.humi = (R)0.5f * (hh + hhxp);
    o.wu = (hu > eps && o.humi > eps) ? 1 : 0;
    o.hvmi = (R)0.5f * (hh + hhyp);
    o.wv = (hv > eps && o.hvmi > eps) ? 1 : 0;
    return o;
}

template <class R>
__device__ __forceinline__ void b_flow_a(const Dev<R>& S, const Konst<R>& K, const int bix, const int biy) {
    const bool off = halted(S.clk);   // tested before the first store (see halted())
    const int nx = K.nx, ny = K.ny;
    int ix = bix * blockDim.x + threadIdx.x, iy = biy * blockDim.y + threadIdx.y;
    if (ix >= nx || iy >= ny) return;
    int i = IDX(ix, iy);
    R eps = K.eps;
    R hh = ld(S.f[HH] + i);
    const DepthMom<R> d = depthmom_of(K, hh, ld(S.f[HH] + IDX(pp(ix, nx), iy)), ld(S.f[HH] + IDX(ix, pp(iy, ny))),
                                      ld(S.f[HU] + i), ld(S.f[HV] + i));
    const R nuh = smago_cell(S, K, ix, iy);
    loads_before_here();
    if (off) return;
    S.wetu[i] = d.wu;
    S.f[HUM][i] = DM<R>::fmax(d.humi, eps);
    S.wetv[i] = d.wv;
    S.f[HVM][i] = DM<R>::fmax(d.hvmi, eps);
    S.tmp[T_NUH][i] = nuh;
}
XBG_KERNELS(flow_a)

// The same pass over row segments (Seg: V cells of a row per thread, 16-byte
// loads, neighbours by lane shuffles), with the scalar pass's arithmetic
// (the same functions), so the results are bit-identical.
template <class R>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 4 : 1) k_flow_a_v(Dev<R> S, Konst<R> K) {
    using G = Seg<R>;
    constexpr int V = G::V;
    const bool off = halted(S.clk);
    const int nx = K.nx, ny = K.ny;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (iy >= ny) return;   // the whole warp: a warp is one row
    const G g(nx, blockIdx.x);
    const int ym = mm(iy), yp = pp(iy, ny);
    const typename G::U h = g.row(S.f[HH], iy), hyp = g.row(S.f[HH], yp), hu = g.row(S.f[HU], iy),
                        hv = g.row(S.f[HV], iy), dr = g.row(S.f[DR], iy);
    const R hr = g.right(h, S.f[HH], iy);
    typename G::U u{}, uyp{}, uym{}, v{}, vym{};
    R ul = 0, ulyp = 0, ulym = 0, vl = 0, vr = 0, vlym = 0, vrym = 0;
    const bool smago = K.usesmago == 1;   // uniform
    if (smago) {
        const R* uu = S.f[UU]; const R* vv = S.f[VV];
        u = g.row(uu, iy); uyp = g.row(uu, yp); uym = g.row(uu, ym); v = g.row(vv, iy); vym = g.row(vv, ym);
        ul = g.left(u, uu, iy); ulyp = g.left(uyp, uu, yp); ulym = g.left(uym, uu, ym);
        vl = g.left(v, vv, iy); vr = g.right(v, vv, iy); vlym = g.left(vym, vv, ym); vrym = g.right(vym, vv, ym);
    }
    const R eps = K.eps;
    typename G::U hum, hvm, nuh;
    typename G::W wu, wv;
#pragma unroll
    for (int k = 0; k < V; k++) {
        const DepthMom<R> d = depthmom_of(K, h.a[k], k < V - 1 ? h.a[k + 1] : hr, hyp.a[k], hu.a[k], hv.a[k]);
        SmagoIn<R> a{};
        a.h = h.a[k];
        a.dr = dr.a[k];
        if (smago) {
            a.u = u.a[k]; a.uxm = k > 0 ? u.a[k - 1] : ul; a.uyp = uyp.a[k]; a.uym = uym.a[k];
            a.uxmyp = k > 0 ? uyp.a[k - 1] : ulyp; a.uxmym = k > 0 ? uym.a[k - 1] : ulym;
            a.v = v.a[k]; a.vym = vym.a[k]; a.vxp = k < V - 1 ? v.a[k + 1] : vr; a.vxm = k > 0 ? v.a[k - 1] : vl;
            a.vxpym = k < V - 1 ? vym.a[k + 1] : vrym; a.vxmym = k > 0 ? vym.a[k - 1] : vlym;
        }
        nuh.a[k] = smago_of(K, a);
        hum.a[k] = DM<R>::fmax(d.humi, eps);
        hvm.a[k] = DM<R>::fmax(d.hvmi, eps);
        wu.a[k] = d.wu;
        wv.a[k] = d.wv;
    }
    loads_before_here();
    if (off || !g.act) return;
    g.put(S.wetu, iy, wu);
    g.put(S.f[HUM], iy, hum);
    g.put(S.wetv, iy, wv);
    g.put(S.f[HVM], iy, hvm);
    g.put(S.tmp[T_NUH], iy, nuh);
}

// eulerustep (Flow_kernel.cu:1487-1544) at an interior-x cell, with the
// advection (ududx_adv :752, vdudy_adv :887) and viscosity (viscou1 :1319,
// viscou2 :1358) terms evaluated in place.
template <class R>
__device__ R euler_u(const Dev<R>& S, const Konst<R>& K, int ix, int iy, R dtf, R wu) {
    const int nx = K.nx, ny = K.ny;
    const R* uu = S.f[UU]; const R* vv = S.f[VV]; const R* hu = S.f[HU]; const R* hv = S.f[HV];
    const R* hum = S.f[HUM]; const R* hvm = S.f[HVM]; const R* nuhg = S.tmp[T_NUH];
    const R* hh = S.f[HH];
    int i = IDX(ix, iy), xm = mm(ix), xp = pp(ix, nx), ym = mm(iy), yp = pp(iy, ny);
    R rdx = K.rdx, g = K.g, rho = K.rho;
    R uui = ld(uu + i);
    if (ld(S.wetu + i) != 1) return (R)0.0f;
    R humi = ld(hum + i);
    // wlevslopes, x
    R dzsdx = (ld(S.f[ZS] + IDX(xp, iy)) - ld(S.f[ZS] + i)) * rdx;
    // ududx_adv
    R uur = ld(uu + IDX(xp, iy)), uul = ld(uu + IDX(xm, iy));
    R ududx = (R)0.0f;
    R qin = (R)0.5f * (ld(hu + i) * uui + ld(hu + IDX(xm, iy)) * uul);
    R du = uui - uul;
    if (qin > (R)0.0f) {
        if (du > (R)0.5f) ududx = ududx + (R)0.5f * (uul + uui) * (uui - uul) * rdx;
        else ududx = ududx + qin / humi * (uui - uul) * rdx;
    }
    qin = (R)-0.5f * (ld(hu + i) * uui + ld(hu + IDX(xp, iy)) * uur);
    du = uur - uui;
    if (qin > (R)0.0f) {
        if (du > (R)0.5f) ududx = ududx - (R)0.5f * (uur + uui) * (uui - uur) * rdx;
        else ududx = ududx + qin / humi * (uui - uur) * rdx;
    }
    // vdudy_adv
    R uut = ld(uu + IDX(ix, yp)), uub = ld(uu + IDX(ix, ym));
    R vb = ld(vv + IDX(ix, ym)), vbr = ld(vv + IDX(xp, ym)), vi = ld(vv + i), vr = ld(vv + IDX(xp, iy));
    R vdudy = (R)0.0f;
    qin = (R)0.5f * (vb * ld(hv + IDX(ix, ym)) + vbr * ld(hv + IDX(xp, ym)));
    R dv = vi - vb;
    if (qin > (R)0.0f) {
        if (dv > (R)0.5f) vdudy = vdudy + (R)0.5f * (vb + vbr) * (uui - uub) * rdx;
        else vdudy = vdudy + qin / humi * (uui - uub) * rdx;
    }
    qin = (R)-0.5f * (vi * ld(hv + i) + vr * ld(hv + IDX(xp, iy)));
    dv = ld(vv + IDX(ix, yp)) - vi;
    if (qin > (R)0.0f) {
        if (dv > (R)0.5f) vdudy = vdudy - (R)0.5f * (vi + vr) * (uui - uut) * rdx;
        else vdudy = vdudy + qin / humi * (uui - uut) * rdx;
    }
    // viscou1 + viscou2
    R nuh1 = ld(nuhg + IDX(xp, iy)), nuh2 = ld(nuhg + i);
    R dudx1 = nuh1 * ld(hh + IDX(xp, iy)) * (uur - uui) * rdx;
    R dudx2 = nuh2 * ld(hh + i) * (uui - uul) * rdx;
    R visc = ((R)1.0f / humi) * ((dudx1 - dudx2) * rdx);
    nuh1 = (R)0.25f * (ld(nuhg + i) + ld(nuhg + IDX(xp, iy)) + ld(nuhg + IDX(xp, yp)) + ld(nuhg + IDX(ix, yp)));
    nuh2 = (R)0.25f * (ld(nuhg + i) + ld(nuhg + IDX(xp, iy)) + ld(nuhg + IDX(xp, ym)) + ld(nuhg + IDX(ix, ym)));
    R dudy1 = nuh1 * (R)0.5f * (ld(hvm + i) + ld(hvm + IDX(xp, iy))) * (uut - uui) * rdx;
    R dudy2 = nuh2 * (R)0.5f * (ld(hvm + IDX(ix, ym)) + ld(hvm + IDX(xp, ym))) * (uui - uub) * rdx;
    visc = visc + ((R)1.0f / humi) * ((dudy1 - dudy2) * rdx * (R)ld(S.wetu + IDX(ix, yp)) * (R)ld(S.wetu + IDX(ix, ym)));
    // eulerustep
    R hmin = (R)0.2;
    int sw = (wu > (R)0.0) - (wu < (R)0.0);
    R urms = ld(S.f[URMS] + i), vmag = ld(S.f[VMAGEU] + i);
    R taubx = ld(S.f[CFM] + i) * rho * ld(S.f[UEU] + i) * DM<R>::sqrt((R)1.3456f * urms * urms + vmag * vmag);
    return uui - dtf * (ududx + vdudy - visc + g * dzsdx + taubx / (rho * ld(hu + i)) -
                        ld(S.f[FX] + i) / (rho * DM<R>::fmax(humi, hmin)) -
                        (R)1.25f * K.Cd * (R)sw * wu * wu / (rho * humi) - K.fc * ld(S.f[VU] + i));
}

// uu* (eulerustep, then latbnd(uu): rows 0 / ny-1 take the updated rows
// 1 / ny-2) at cell (ix, iy)
template <class R>
__device__ __forceinline__ R ustar_cell(const Dev<R>& S, const Konst<R>& K, int ix, int iy, R dtf, R wu) {
    const int nx = K.nx, ny = K.ny;
    int sy = iy;
    if (iy == 0) sy = 1;
    if (iy == ny - 1) sy = ny - 2;
    return (ix > 0) ? euler_u(S, K, ix, sy, dtf, wu) : ld(S.f[UU] + IDX(ix, sy));
}

template <class R>
__device__ __forceinline__ void b_flow_u(const Dev<R>& S, const Konst<R>& K, const int bix, const int biy) {
    const Clock* clk = S.clk;
    const bool off = halted(clk);
    const int nx = K.nx, ny = K.ny;
    int ix = bix * blockDim.x + threadIdx.x, iy = biy * blockDim.y + threadIdx.y;
    if (ix >= nx || iy >= ny) return;
    const R u = ustar_cell(S, K, ix, iy, (R)clk->dt, (R)clk->windu);
    loads_before_here();
    if (off) return;
    S.tmp[T_UU][IDX(ix, iy)] = u;
}
XBG_KERNELS(flow_u)

// vdvdy_adv (Flow_kernel.cu:1024-1074) at a row that eulervstep updates.
template <class R>
__device__ __forceinline__ R vdvdy_cell(const Dev<R>& S, const Konst<R>& K, int ix, int iy) {
    const int nx = K.nx, ny = K.ny;
    const R* vv = S.f[VV]; const R* hv = S.f[HV];
    R r = (R)0.0f;
    if (ix > 0 && iy > 0 && iy < ny - 2) {
        int i = IDX(ix, iy), ym = mm(iy), yp = pp(iy, ny);
        R rdx = K.rdx, hvmi = ld(S.f[HVM] + i);
        R vi = ld(vv + i), vb = ld(vv + IDX(ix, ym)), vt = ld(vv + IDX(ix, yp));
        R qin = (R)0.5f * (vi * ld(hv + i) + vb * ld(hv + IDX(ix, ym)));
        R dv = vi - vb;
        if (qin > (R)0.0f) {
            if (dv > (R)0.5f) r = r + (R)0.5f * (vb - vi) * (vi - vb) * rdx;
            else r = r + qin / hvmi * (vi - vb) * rdx;
        }
        qin = (R)-0.5f * (ld(hv + i) * vi + ld(hv + IDX(ix, yp)) * vt);
        dv = vt - vi;
        if (qin > (R)0.0f) {
            if (dv > (R)0.5f) r = r - (R)0.5f * (vt + vi) * (vi - vt) * rdx;
            else r = r + qin / hvmi * (vi - vt) * rdx;
        }
    }
    return r;
}

// eulervstep (Flow_kernel.cu:1546-1599) at ix > 0, iy < ny-2, with udvdx_adv
// (:1159, on the updated uu*), vdvdy_adv and viscov1 + viscov2.  us(x, y)
// gives uu* at cell (x, y).
template <class R, class US>
__device__ R euler_v(const Dev<R>& S, const Konst<R>& K, int ix, int iy, R dtf, R wv, const US& us) {
    const int nx = K.nx, ny = K.ny;
    const R* vv = S.f[VV]; const R* hu = S.f[HU];
    const R* hum = S.f[HUM]; const R* hvm = S.f[HVM]; const R* nuhg = S.tmp[T_NUH];
    const R* hh = S.f[HH];
    int i = IDX(ix, iy), xm = mm(ix), xp = pp(ix, nx), ym = mm(iy), yp = pp(iy, ny);
    R rdx = K.rdx, g = K.g, rho = K.rho;
    R vvi = ld(vv + i);
    if (ld(S.wetv + i) != 1) return (R)0.0f;
    R hvmi = ld(hvm + i);
    R dzsdy = (ld(S.f[ZS] + IDX(ix, yp)) - ld(S.f[ZS] + i)) * rdx;
    R vdvdy = vdvdy_cell(S, K, ix, iy);
    // udvdx_adv
    R ul = us(xm, iy), ultl = us(xm, yp), ui = us(ix, iy), ur = us(xp, iy);
    R vl = ld(vv + IDX(xm, iy)), vr = ld(vv + IDX(xp, iy));
    R udvdx = (R)0.0f;
    R qin = (R)(0.5 * (double)(ul * ld(hu + IDX(xm, iy)) + ultl * ld(hu + IDX(xm, yp))));
    R du = ui - ul;
    if (qin > (R)0.0f) {
        if (du > (R)0.5f) udvdx = udvdx + (R)0.5f * (ul + ultl) * (vvi - vl) * rdx;
        else udvdx = udvdx + qin / hvmi * (vvi - vl) * rdx;
    }
    qin = (R)(-0.5 * (double)(ui * ld(hu + i) + us(ix, yp) * ld(hu + IDX(ix, yp))));
    du = ur - ui;
    if (qin > (R)0.0f) {
        if (du > (R)0.5f) udvdx = udvdx - (R)0.5f * (ui + ur) * (vvi - vr) * rdx;
        else udvdx = udvdx + qin / hvmi * (vvi - vr) * rdx;
    }
    // viscov1 + viscov2
    R vt = ld(vv + IDX(ix, yp)), vb = ld(vv + IDX(ix, ym));
    R nuh1 = ld(nuhg + IDX(ix, yp)), nuh2 = ld(nuhg + i);
    R dvdy1 = nuh1 * ld(hh + IDX(ix, yp)) * (vt - vvi) * rdx;
    R dvdy2 = nuh2 * ld(hh + i) * (vvi - vb) * rdx;
    R visc = ((R)1.0f / hvmi) * (dvdy1 - dvdy2) * rdx * (R)ld(S.wetv + IDX(ix, yp)) * (R)ld(S.wetv + IDX(ix, ym));
    nuh1 = (R)0.25f * (ld(nuhg + i) + ld(nuhg + IDX(xp, iy)) + ld(nuhg + IDX(xp, yp)) + ld(nuhg + IDX(ix, yp)));
    nuh2 = (R)0.25f * (ld(nuhg + i) + ld(nuhg + IDX(xm, iy)) + ld(nuhg + IDX(xm, yp)) + ld(nuhg + IDX(ix, yp)));
    R dvdx1 = nuh1 * (R)0.5f * (ld(hum + i) + ld(hum + IDX(ix, yp))) * (vr - vvi) * rdx;
    R dvdx2 = nuh2 * (R)0.5f * (ld(hum + IDX(xm, iy)) + ld(hum + IDX(xm, yp))) * (vvi - vl) * rdx;
    visc = visc + ((R)1.0f / hvmi) * ((dvdx1 - dvdx2) * rdx * (R)ld(S.wetv + IDX(xp, iy)) * (R)ld(S.wetv + IDX(xm, iy)));
    R hmin = (R)0.2;
    int sw = (wv > (R)0.0) - (wv < (R)0.0);
    R urms = ld(S.f[URMS] + i), vmag = ld(S.f[VMAGEV] + i);
    R tauby = ld(S.f[CFM] + i) * rho * ld(S.f[VEV] + i) * DM<R>::sqrt((R)1.3456f * urms * urms + vmag * vmag);
    return vvi - dtf * (udvdx + vdvdy - visc + g * dzsdy + tauby / (rho * ld(S.f[HV] + i)) -
                        ld(S.f[FY] + i) / (rho * DM<R>::fmax(hvmi, hmin)) + K.fc * ld(S.f[UV] + i) -
                        (R)1.25f * K.Cd * (R)sw * wv * wv / (rho * hvmi));
}

template <class R>
__device__ __forceinline__ void b_flow_v(const Dev<R>& S, const Konst<R>& K, const int bix, const int biy) {
    const Clock* clk = S.clk;
    const bool off = halted(clk);
    const int nx = K.nx, ny = K.ny;
    int ix = bix * blockDim.x + threadIdx.x, iy = biy * blockDim.y + threadIdx.y;
    if (ix >= nx || iy >= ny) return;
    R dtf = (R)clk->dt, wv = (R)clk->windv;
    // vvlatbnd: row 0 <- row 1, row ny-2 <- row ny-3; row ny-1 keeps its value
    int sy = iy;
    if (iy == 0) sy = 1;
    if (iy == ny - 2) sy = ny - 3;
    const R* us = S.tmp[T_UU];
    R v;
    if (sy < ny - 2 && ix > 0) v = euler_v(S, K, ix, sy, dtf, wv, [&](int x, int y) { return ld(us + IDX(x, y)); });
    else v = ld(S.f[VV] + IDX(ix, sy));
    loads_before_here();
    if (off) return;
    S.tmp[T_VV][IDX(ix, iy)] = v;
}
XBG_KERNELS(flow_v)

// flow_u and flow_v in one pass.  eulervstep reads uu* at the cell, its left,
// right and upper neighbours and the upper-left one, so the block first
// evaluates uu* over its 32 x 8 tile plus the column on each side and the row
// above (clamped like mm/pp) into shared memory, stores the tile's own
// values, and then evaluates vv* from there.  The one row outside that range
// (row ny-3 for the vvlatbnd copy into row ny-2, when ny-2 is the tile's
// first row) evaluates its uu* directly.  Results are bit-identical to the
// two passes.
constexpr int UV_TX = FT_X + 2, UV_TY = FT_Y + 1;

template <class R>
__device__ __forceinline__ void b_flow_uv(const Dev<R>& S, const Konst<R>& K, const int bix, const int biy) {
    const Clock* clk = S.clk;
    const bool off = halted(clk);
    __shared__ R sU[UV_TY * UV_TX];
    const int nx = K.nx, ny = K.ny;
    const int bx0 = bix * FT_X, by0 = biy * FT_Y;
    const R dtf = (R)clk->dt, wu = (R)clk->windu, wv = (R)clk->windv;
    for (int e = threadIdx.x + threadIdx.y * FT_X; e < UV_TX * UV_TY; e += FT_X * FT_Y) {
        const int gx = min(max(bx0 - 1 + e % UV_TX, 0), nx - 1), gy = min(by0 + e / UV_TX, ny - 1);
        sU[e] = ustar_cell(S, K, gx, gy, dtf, wu);
    }
    __syncthreads();
    const int ix = bx0 + threadIdx.x, iy = by0 + threadIdx.y;
    loads_before_here();
    if (off || ix >= nx || iy >= ny) return;
    S.tmp[T_UU][IDX(ix, iy)] = sU[threadIdx.y * UV_TX + threadIdx.x + 1];
    // vvlatbnd: row 0 <- row 1, row ny-2 <- row ny-3; row ny-1 keeps its value
    int sy = iy;
    if (iy == 0) sy = 1;
    if (iy == ny - 2) sy = ny - 3;
    R v;
    if (sy < ny - 2 && ix > 0) {
        // the accessed cells are clamped grid cells: x in [bx0-1, bx0+32], y in [sy, sy+1]
        v = euler_v(S, K, ix, sy, dtf, wv, [&](int x, int y) {
            const int ex = x - bx0 + 1, ey = y - by0;
            return (ey >= 0 && ey < UV_TY) ? sU[ey * UV_TX + ex] : ustar_cell(S, K, x, y, dtf, wu);
        });
    } else {
        v = ld(S.f[VV] + IDX(ix, sy));
    }
    S.tmp[T_VV][IDX(ix, iy)] = v;
}
XBG_KERNELS(flow_uv)

// depthhu / depthhv (Flow_kernel.cu:653-750) at a u (v) point from the levels
// and beds of the cell and its right (upper) neighbour and the velocity there
template <class R>
__device__ __forceinline__ R depth_face(R zsi, R zsn, R zbi, R zbn, R u, R eps) {
    const R b = DM<R>::fmax((R)-1.0f * zbi, (R)-1.0f * zbn);
    const R ummn = (R)0.0f;
    R h;
    if (u > ummn) h = zsi - b;
    else if (u < (R)-1.0f * ummn) h = zsn - b;
    else h = DM<R>::fmax(DM<R>::fmax(zsi, zsn) - b, eps);
    return DM<R>::fmax(h, (R)0.0f);
}

// Fields of the momentum-correction pass, in its shared-memory tile.
enum { C_ZS, C_ZB, C_UU, C_VV, C_UO, C_VO, C_QX, C_QY, C_NF };

// wrkuu2Ocorr (Flow_kernel.cu:1960-2044) at cell (ix, iy); a: field access
// around the cell (uu is the post-Euler uu*, uo the previous step's).
template <class R, class A>
__device__ __forceinline__ void wrk_u(const A& a, const Konst<R>& K, int ix, int iy, R& w1, R& w2) {
    const R eps2 = K.eps * (R)2.0f;
    w1 = (R)0.0f; w2 = (R)0.0f;
    if (ix > 0) {
        const Pair2<R> m1 = zz_min<R>(a, -2, 2, 0, 0);   // zs, zb over x-2 .. x+2
        if (m1.a + m1.b > eps2) {
            R qs = a(C_QX, 0, 0) + a(C_QX, -1, 0);
            if (qs > (R)0.0f) w1 = (R)0.5f * minmod(a(C_UU, 0, 0) - a(C_UO, -1, 0), a(C_UU, -1, 0) - a(C_UO, -2, 0));
            if (qs < (R)0.0f) w1 = (R)-0.5f * minmod(a(C_UO, 0, 0) - a(C_UU, -1, 0), a(C_UO, 1, 0) - a(C_UU, 0, 0));
        }
        if (iy > 0) {
            const Pair2<R> m2 = zz_min<R>(a, 0, 1, -1, 2);   // x, x+1 over y-1 .. y+2
            if (m2.a + m2.b > eps2) {
                R qs = a(C_QY, 1, 0) + a(C_QY, 0, 0);
                if (qs > (R)0.0f) w2 = (R)0.5f * minmod(a(C_UU, 0, 1) - a(C_UO, 0, 0), a(C_UU, 0, 0) - a(C_UO, 0, -1));
                if (qs < (R)0.0f) w2 = (R)-0.5f * minmod(a(C_UO, 0, 1) - a(C_UU, 0, 0), a(C_UO, 0, 2) - a(C_UU, 0, 1));
            }
        }
    }
}

// wrkvv2Ocorr (Flow_kernel.cu:2046-2128) at cell (ix, iy)
template <class R, class A>
__device__ __forceinline__ void wrk_v(const A& a, const Konst<R>& K, int ix, int iy, R& w1, R& w2) {
    const R eps2 = K.eps * (R)2.0f;
    w1 = (R)0.0f; w2 = (R)0.0f;
    if (ix > 0 && iy > 0 && iy < K.ny - 2) {
        const Pair2<R> m1 = zz_min<R>(a, 0, 0, -2, 2);   // y-2 .. y+2
        if (m1.a + m1.b > eps2) {
            R qs = a(C_QY, 0, 0) + a(C_QY, 0, -1);
            if (qs > (R)0.0f) w1 = (R)0.5f * minmod(a(C_VV, 0, 0) - a(C_VO, 0, -1), a(C_VV, 0, -1) - a(C_VO, 0, -2));
            if (qs < (R)0.0f) w1 = (R)-0.5f * minmod(a(C_VO, 0, 0) - a(C_VV, 0, -1), a(C_VO, 0, 1) - a(C_VV, 0, 0));
        }
        const Pair2<R> m2 = zz_min<R>(a, -1, 2, 0, 1);   // x-1 .. x+2 over y, y+1
        if (m2.a + m2.b > eps2) {
            R qs = a(C_QX, 0, 1) + a(C_QX, 0, 0);
            if (qs > (R)0.0f) w2 = (R)0.5f * minmod(a(C_VV, 1, 0) - a(C_VO, 0, 0), a(C_VV, 0, 0) - a(C_VO, -1, 0));
            if (qs < (R)0.0f) w2 = (R)-0.5f * minmod(a(C_VO, 1, 0) - a(C_VV, 0, 0), a(C_VO, 2, 0) - a(C_VV, 1, 0));
        }
    }
}

// uu2Ocorr + vv2Ocorr (Flow_kernel.cu:2210-2282), then depthhu/depthhv,
// CalcQFlow and continuity (:653-750, 1917, 1626-1681).  The eight input
// fields of the block's tile (halo 3) stream into shared memory first; the
// wrk values of the tile cells and a one-cell ring (the left, right, lower and
// upper neighbours the corrections read) are computed once from there.
// Continuity needs the corrected velocities of the left and lower
// neighbours: the block evaluates them once, for its cells and for the
// column to its left (u) and the row below it (v), in shared memory.

template <class R>
__device__ __forceinline__ void b_flow_corr(const Dev<R>& S, const Konst<R>& K, const int bix, const int biy) {
    const Clock* clk = S.clk;
    const bool off = halted(clk);
    using G = TileG<FC_H>;
    __shared__ __align__(16) R tile[C_NF * G::N];   // (level, bed) pairs, then planes
    __shared__ R sU1[FT_N], sU2[FT_N], sV1[FT_N], sV2[FT_N];
    const int nx = K.nx, ny = K.ny;
    const int bx0 = bix * FT_X, by0 = biy * FT_Y;
    const int ix = bx0 + threadIdx.x, iy = by0 + threadIdx.y;
    const bool inside = ix < nx && iy < ny;
    const int i = IDX(ix, iy);
    // the face depths the corrections divide by (the cell's, and those of the
    // extra column / row cells this thread corrects) are loaded first, so
    // their round trip overlaps the tile's
    const bool xrow = threadIdx.y == 0 && by0 > 0 && ix < nx;   // corrects v at (ix, by0-1)
    const bool xcol = threadIdx.y == 1 && threadIdx.x < FT_Y && bx0 > 0 && by0 + (int)threadIdx.x < ny;   // u at (bx0-1, by0+r)
    R hum_c = (R)1, hvm_c = (R)1, hvm_x = (R)1, hum_x = (R)1;
    if (inside) { hum_c = ld(S.f[HUM] + i); hvm_c = ld(S.f[HVM] + i); }
    if (xrow) hvm_x = ld(S.f[HVM] + i - nx);
    if (xcol) hum_x = ld(S.f[HUM] + IDX(bx0 - 1, by0 + (int)threadIdx.x));
    {
        const R* src[C_NF] = {S.f[ZS], S.f[ZB], S.tmp[T_UU], S.tmp[T_VV], S.f[UUOLD], S.f[VVOLD], S.f[QX], S.f[QY]};
        tile_load<R, FC_H, C_NF>(tile, src, bx0, by0, nx, ny);
    }
    for (int e = threadIdx.x + threadIdx.y * FT_X; e < FT_N; e += FT_X * FT_Y) {
        int gx, gy;
        int k = tile_centre<FC_H>(e % FT_TX + FC_H - 1, e / FT_TX + FC_H - 1, bx0, by0, nx, ny, gx, gy);
        TileAt<R, FC_H> a{tile, k};
        R w1, w2, v1, v2;
        wrk_u(a, K, gx, gy, w1, w2);
        wrk_v(a, K, gx, gy, v1, v2);
        sU1[e] = w1; sU2[e] = w2; sV1[e] = v1; sV2[e] = v2;
    }
    __syncthreads();
    R dtf = (R)clk->dt, rdx = K.rdx;
    const int kc = (threadIdx.y + FC_H) * G::TX + threadIdx.x + FC_H;
    const int c = (threadIdx.y + 1) * FT_TX + threadIdx.x + 1;
    // uu2Ocorr at the cell r (ring index) of tile slot k, grid cell (x, y) with
    // face depth hm: wrk at the cell, its right and lower neighbours
    auto ucorr = [&](int k, int r, int x, int y, R hm) -> R {
        TileAt<R, FC_H> a{tile, k};
        R u = a(C_UU, 0, 0);
        if (x > 0 && y > 0) {
            R w1i = sU1[r], w2i = sU2[r], w1r = sU1[r + 1], w2b = sU2[r - FT_TX];
            R qe = (R)0.5f * (a(C_QX, 1, 0) + a(C_QX, 0, 0));
            R qw = (R)0.5f * (a(C_QX, 0, 0) + a(C_QX, -1, 0));
            R qn = (R)0.5f * (a(C_QY, 0, -1) + a(C_QY, 1, -1));
            R qs = (R)0.5f * (a(C_QY, 0, 0) + a(C_QY, -1, 0));
            u = u - dtf / hm * ((qe * w1r - qw * w1i) * rdx + (qs * w2i - qn * w2b) * rdx);
        }
        return u;
    };
    // vv2Ocorr: wrk at the cell, its left and upper neighbours
    auto vcorr = [&](int k, int r, int x, int y, R hm) -> R {
        TileAt<R, FC_H> a{tile, k};
        R v = a(C_VV, 0, 0);
        if (x > 0 && y > 0) {
            R v1i = sV1[r], v2i = sV2[r], v2l = sV2[r - 1], v1t = sV1[r + FT_TX];
            R qe = (R)0.5f * (a(C_QX, 0, 1) + a(C_QX, 0, 0));
            R qw = (R)0.5f * (a(C_QX, -1, 0) + a(C_QX, -1, 1));
            R qn = (R)0.5f * (a(C_QY, 0, 0) + a(C_QY, 0, -1));
            R qs = (R)0.5f * (a(C_QY, 0, 1) + a(C_QY, 0, 0));
            v = v - dtf / hm * ((qe * v2i - qw * v2l) * rdx + (qs * v1t - qn * v1i) * rdx);
        }
        return v;
    };
    // corrected velocities once per cell: the tile's (u and v), the column to
    // its left (u) and the row below it (v) into shared memory for the
    // continuity of the neighbouring cells.  They take the tile planes of the
    // previous step's velocities, which only the ring pass above reads.
    static_assert(FT_Y * (FT_X + 1) <= G::N && (FT_Y + 1) * FT_X <= G::N, "corrected velocities fit a plane");
    R* sUc = tile + C_UO * G::N;   // [FT_Y][FT_X + 1], x = bx0-1 .. bx0+31
    R* sVc = tile + C_VO * G::N;   // [FT_Y + 1][FT_X], y = by0-1 .. by0+7
    R u = (R)0, v = (R)0;
    if (inside) {
        u = ucorr(kc, c, ix, iy, hum_c);
        v = vcorr(kc, c, ix, iy, hvm_c);
        sUc[threadIdx.y * (FT_X + 1) + threadIdx.x + 1] = u;
        sVc[(threadIdx.y + 1) * FT_X + threadIdx.x] = v;
    }
    if (xrow)   // (ix, by0-1)
        sVc[threadIdx.x] = vcorr(kc - G::TX, c - FT_TX, ix, by0 - 1, hvm_x);
    if (xcol) {   // (bx0-1, by0+r)
        const int r = threadIdx.x;
        sUc[r * (FT_X + 1)] = ucorr((r + FC_H) * G::TX + FC_H - 1, (r + 1) * FT_TX, bx0 - 1, by0 + r, hum_x);
    }
    __syncthreads();
    loads_before_here();
    if (off || !inside) return;
    S.f[UU][i] = u;
    S.f[VV][i] = v;
    // depthhu, depthhv, CalcQFlow (Flow_kernel.cu:653-750, 1917) and continuity
    // (:1626-1681) with the corrected velocities of the cell and of its left
    // (lower) neighbour; the tile is clamped like pp()
    TileAt<R, FC_H> a{tile, kc};
    const R eps = K.eps;
    const R hu = depth_face(a(C_ZS, 0, 0), a(C_ZS, 1, 0), a(C_ZB, 0, 0), a(C_ZB, 1, 0), u, eps);
    const R hv = depth_face(a(C_ZS, 0, 0), a(C_ZS, 0, 1), a(C_ZB, 0, 0), a(C_ZB, 0, 1), v, eps);
    const R qxi = u * hu, qyi = v * hv;
    R zs = a(C_ZS, 0, 0);
    R dzdt = (R)0;
    if (ix > 0) {
        const R ul = sUc[threadIdx.y * (FT_X + 1) + threadIdx.x];
        const R qxl = ul * depth_face(a(C_ZS, -1, 0), a(C_ZS, 0, 0), a(C_ZB, -1, 0), a(C_ZB, 0, 0), ul, eps);
        R qyb = qyi;
        if (iy > 0) {
            const R vb = sVc[threadIdx.y * FT_X + threadIdx.x];
            qyb = vb * depth_face(a(C_ZS, 0, -1), a(C_ZS, 0, 0), a(C_ZB, 0, -1), a(C_ZB, 0, 0), vb, eps);
        }
        dzdt = (qxl - qxi + qyb - qyi) * rdx;
        zs = zs + dzdt * dtf;
    }
    // the new fluxes go to per-step buffers: neighbouring blocks of this pass
    // still read the previous step's qx, qy (k_flow_final stores the final ones)
    S.f[HU][i] = hu; S.f[HV][i] = hv;
    S.tmp[T_QX][i] = qxi; S.tmp[T_QY][i] = qyi;
    if (ix > 0) S.f[DZSDT][i] = dzdt;
    S.tmp[T_ZS][i] = zs;
}
XBG_KERNELS(flow_corr)


// Fields of the final pass, in its shared-memory tile: the post-continuity
// level, bed, previous step's level, corrected velocities, Stokes drift inputs.
enum { Z_ZS, Z_ZB, Z_ZO, Z_UU, Z_VV, Z_UST, Z_THM, Z_NF };

// wrkzs2Ocorr (Flow_kernel.cu:2130-2208) at cell (ix, iy)
template <class R, class A>
__device__ __forceinline__ void wrk_z(const A& a, const Konst<R>& K, int ix, int iy, R& w1, R& w2) {
    const R eps2 = K.eps * (R)2.0f;
    w1 = (R)0.0f; w2 = (R)0.0f;
    if (ix > 0) {
        const Pair2<R> m1 = zz_min<R>(a, -1, 2, 0, 0);   // x-1 .. x+2
        if (m1.a + m1.b > eps2) {
            R u = a(Z_UU, 0, 0);
            if (u > (R)0.0f) w1 = u * (R)0.5f * minmod(a(Z_ZS, 1, 0) - a(Z_ZO, 0, 0), a(Z_ZS, 0, 0) - a(Z_ZO, -1, 0));
            if (u < (R)0.0f) w1 = (R)-1.0f * u * (R)0.5f * minmod(a(Z_ZO, 2, 0) - a(Z_ZS, 1, 0), a(Z_ZO, 1, 0) - a(Z_ZS, 0, 0));
        }
        if (iy > 0) {
            const Pair2<R> m2 = zz_min<R>(a, 0, 0, -1, 2);   // y-1 .. y+2
            if (m2.a + m2.b > eps2) {
                R v = a(Z_VV, 0, 0);
                if (v > (R)0.0f) w2 = v * (R)0.5f * minmod(a(Z_ZS, 0, 1) - a(Z_ZO, 0, 0), a(Z_ZS, 0, 0) - a(Z_ZO, 0, -1));
                if (v < (R)0.0f) w2 = v * (R)0.5f * minmod(a(Z_ZO, 0, 2) - a(Z_ZS, 0, 1), a(Z_ZO, 0, 1) - a(Z_ZS, 0, 0));
            }
        }
    }
}

// zs after zs2Ocorr (Flow_kernel.cu:2284-2317) at (ix, iy), every wrk
// evaluated from global memory (the one lateral cell the tile cannot serve).
template <class R>
__device__ R zs_corr_global(const Dev<R>& S, const Konst<R>& K, const R* zso, int ix, int iy, R dtf) {
    auto at = [&](int x, int y) {
        return GlobalAt<R, Z_NF>{{S.tmp[T_ZS], S.f[ZB], zso, S.f[UU], S.f[VV], S.f[UST], S.f[THM]}, x, y, K.nx, K.ny};
    };
    R w1, w2, w1l, w2b, t0, t1;
    wrk_z(at(ix, iy), K, ix, iy, w1, w2);
    R z = ld(S.tmp[T_ZS] + ix + iy * K.nx);
    if (ix > 0 && iy > 0) {
        wrk_z(at(ix - 1, iy), K, ix - 1, iy, w1l, t0);
        wrk_z(at(ix, iy - 1), K, ix, iy - 1, t1, w2b);
        z = z - dtf * ((w1 - w1l) * K.rdx + (w2 - w2b) * K.rdx);
    }
    return z;
}

// calcuvvu (Flow_kernel.cu:467-544) at (ix, iy); a: the final-pass tile around
// the cell; sS/sC hold ust*sin(thetamean) and ust*cos(thetamean) of the ring
// tile, k is the ring index of (ix, iy), whose right and top neighbours are
// k + 1 and k + FT_TX.
template <class R, class A>
__device__ __forceinline__ void uvvu_cell(const A& a, R wu, R wv, const R* sS, const R* sC, int k, R* o6) {
    R vu = (R)0.25f * (a(Z_VV, 0, -1) + a(Z_VV, 0, 0) + a(Z_VV, 1, -1) + a(Z_VV, 1, 0)) * wu;
    R uv = (R)0.25f * (a(Z_UU, -1, 0) + a(Z_UU, 0, 0) + a(Z_UU, -1, 1) + a(Z_UU, 0, 1)) * wv;
    R vsu = (R)0.5f * (sS[k] + sS[k + 1]) * wu;
    R usu = (R)0.5f * (sC[k] + sC[k + 1]) * wu;
    R ue = a(Z_UU, 0, 0) - usu;
    R ve = vu - vsu;
    R usv = (R)0.5f * (sC[k] + sC[k + FT_TX]) * wv;
    R vsv = (R)0.5f * (sS[k] + sS[k + FT_TX]) * wv;
    R vvv = a(Z_VV, 0, 0) - vsv;
    R uvv = uv - usv;
    o6[0] = vu; o6[1] = uv; o6[2] = ue; o6[3] = vvv;
    o6[4] = DM<R>::sqrt(ue * ue + ve * ve);
    o6[5] = DM<R>::sqrt(uvv * uvv + vvv * vvv);
}

// wrkzs2Ocorr + zs2Ocorr, latbnd(zs), hsbnd, calcuvvu + uvlatbnd.  The seven
// input fields of the block's tile (halo 3) stream into shared memory; the
// wrk values and Stokes-drift products of the tile cells and a one-cell ring
// are computed once from there.  The lateral row ny-1 takes zs of row ny-2
// (latbnd), whose lower neighbour is outside the ring when ny-1 is the block's
// first row: that one case evaluates zs from global memory.
template <class R>
__device__ __forceinline__ void b_flow_final(const Dev<R>& S, const Konst<R>& K, const int bix, const int biy) {
    const Clock* clk = S.clk;
    const bool off = halted(clk);
    using G = TileG<FC_H>;
    __shared__ __align__(16) R tile[Z_NF * G::N];   // (level, bed) pairs, then planes
    __shared__ R sW1[FT_N], sW2[FT_N], sS[FT_N], sC[FT_N];
    const R* zsold_in = S.zsold[clk->par ^ 1];
    R* zsold_out = S.zsold[clk->par];
    const int nx = K.nx, ny = K.ny;
    const int bx0 = bix * FT_X, by0 = biy * FT_Y;
    {
        const R* src[Z_NF] = {S.tmp[T_ZS], S.f[ZB], zsold_in, S.f[UU], S.f[VV], S.f[UST], S.f[THM]};
        tile_load<R, FC_H, Z_NF>(tile, src, bx0, by0, nx, ny);
    }
    for (int e = threadIdx.x + threadIdx.y * FT_X; e < FT_N; e += FT_X * FT_Y) {
        int gx, gy;
        int k = tile_centre<FC_H>(e % FT_TX + FC_H - 1, e / FT_TX + FC_H - 1, bx0, by0, nx, ny, gx, gy);
        TileAt<R, FC_H> a{tile, k};
        R w1, w2;
        wrk_z(a, K, gx, gy, w1, w2);
        R us = a(Z_UST, 0, 0), tm = a(Z_THM, 0, 0), sn, cs;
        DM<R>::sincos(tm, &sn, &cs);   // one range reduction for both
        sW1[e] = w1; sW2[e] = w2;
        sS[e] = us * sn;
        sC[e] = us * cs;
    }
    __syncthreads();
    int ix = bx0 + threadIdx.x, iy = by0 + threadIdx.y;
    if (ix >= nx || iy >= ny) return;
    int i = IDX(ix, iy);
    R dtf = (R)clk->dt;
    int sy = iy;
    if (iy == 0) sy = 1;
    if (iy == ny - 1) sy = ny - 2;
    const int k = (threadIdx.y + 1) * FT_TX + threadIdx.x + 1;
    const int ks = k + (sy - iy) * FT_TX;   // ring index of (ix, sy)
    const int kc = (threadIdx.y + FC_H) * G::TX + threadIdx.x + FC_H;
    TileAt<R, FC_H> a{tile, kc};                          // around (ix, iy)
    TileAt<R, FC_H> as{tile, kc + (sy - iy) * G::TX};     // around (ix, sy)
    auto zcorr = [&](const TileAt<R, FC_H>& c, int r, int y) {
        R z = c(Z_ZS, 0, 0);
        if (ix > 0 && y > 0) z = z - dtf * ((sW1[r] - sW1[r - 1]) * K.rdx + (sW2[r] - sW2[r - FT_TX]) * K.rdx);
        return z;
    };
    R zf = zcorr(a, k, iy);
    R qx = ld(S.tmp[T_QX] + i), qy = ld(S.tmp[T_QY] + i);
    R wu = (R)ld(S.wetu + IDX(ix, sy)), wv = (R)ld(S.wetv + IDX(ix, sy));
    if (sy != iy) {           // latbnd(zs)
        if (ks >= FT_TX) zf = zcorr(as, ks, sy);
        else zf = zs_corr_global(S, K, zsold_in, ix, sy, dtf);
    }
    R o6[6];
    uvvu_cell(as, wu, wv, sS, sC, ks, o6);   // calcuvvu + uvlatbnd
    // CalcQFlow's fluxes, with the zs2Ocorr update in the interior
    loads_before_here();
    if (off) return;
    S.f[QX][i] = (ix > 0 && iy > 0) ? qx + sW1[k] : qx;
    S.f[QY][i] = (ix > 0 && iy > 0) ? qy + sW2[k] : qy;
    S.f[ZS][i] = zf;
    S.f[HH][i] = DM<R>::fmax(a(Z_ZB, 0, 0) + zf, K.eps);   // hsbnd
    S.f[UUOLD][i] = a(Z_UU, 0, 0);
    S.f[VVOLD][i] = a(Z_VV, 0, 0);
    zsold_out[i] = zf;
    S.f[VU][i] = o6[0]; S.f[UV][i] = o6[1]; S.f[UEU][i] = o6[2]; S.f[VEV][i] = o6[3];
    S.f[VMAGEU][i] = o6[4]; S.f[VMAGEV][i] = o6[5];
}
XBG_KERNELS(flow_final)

// fuse_uv: the momentum steps as one pass (k_flow_uv) instead of two
// (k_flow_u, k_flow_v); wide: the pointwise passes (k_flow_a, k_flow_u,
// k_flow_v) in 64 x 4 blocks instead of 32 x 8 (their bodies index cells by
// the block's shape; the staged passes keep their 32 x 8 tiles)
template <class R>
int launch_flow(const Dev<R>& S, const Konst<R>& K, cudaStream_t st, Prof* pf, bool fuse_uv, bool wide,
                bool vec) {
    dim3 b(32, 8), g((K.nx + 31) / 32, (K.ny + 7) / 8);
    dim3 bp = wide ? dim3(64, 4) : b, gp = wide ? dim3((K.nx + 63) / 64, (K.ny + 3) / 4) : g;
    if (vec && K.nx % SegVec<R>::V == 0) {
        const int V = SegVec<R>::V;
        k_flow_a_v<R><<<dim3((K.nx / V + 31) / 32, (K.ny + 7) / 8), dim3(32, 8), 0, st>>>(S, K);
    } else {
        k_flow_a<R><<<gp, bp, 0, st>>>(S, K);
    }
    PMARK(pf, "k_flow_a");
    if (fuse_uv) {
        k_flow_uv<R><<<g, b, 0, st>>>(S, K);
        PMARK(pf, "k_flow_uv");
    } else {
        k_flow_u<R><<<gp, bp, 0, st>>>(S, K);
        PMARK(pf, "k_flow_u");
        k_flow_v<R><<<gp, bp, 0, st>>>(S, K);
        PMARK(pf, "k_flow_v");
    }
    k_flow_corr<R><<<g, b, 0, st>>>(S, K);
    PMARK(pf, "k_flow_corr");
    k_flow_final<R><<<g, b, 0, st>>>(S, K);
    PMARK(pf, "k_flow_final");
    return fuse_uv ? 4 : 5;
}
// the flow kernels over every scenario of a batch
template <class R>
int launch_flow_batch(const BatchTab<R>& T, const BatchLaunch& L, cudaStream_t st, Prof* pf, bool fuse_uv,
                      bool wide) {
    dim3 b(32, 8);
    const int2* it = L.items[BS_TILE];
    int n = L.n[BS_TILE], g = L.grid[BS_TILE];
    const int sp = wide ? BS_WIDE : BS_TILE;
    const dim3 bp = wide ? dim3(64, 4) : b;
    const int2* itp = L.items[sp];
    const int np = L.n[sp], gp = L.grid[sp];
    kb_flow_a<R><<<gp, bp, 0, st>>>(T, itp, np);
    PMARK(pf, "k_flow_a");
    if (fuse_uv) {
        kb_flow_uv<R><<<g, b, 0, st>>>(T, it, n);
        PMARK(pf, "k_flow_uv");
    } else {
        kb_flow_u<R><<<gp, bp, 0, st>>>(T, itp, np);
        PMARK(pf, "k_flow_u");
        kb_flow_v<R><<<gp, bp, 0, st>>>(T, itp, np);
        PMARK(pf, "k_flow_v");
    }
    kb_flow_corr<R><<<g, b, 0, st>>>(T, it, n);
    PMARK(pf, "k_flow_corr");
    kb_flow_final<R><<<g, b, 0, st>>>(T, it, n);
    PMARK(pf, "k_flow_final");
    return fuse_uv ? 4 : 5;
}
template int launch_flow_batch<float>(const BatchTab<float>&, const BatchLaunch&, cudaStream_t, Prof*, bool, bool);
template int launch_flow_batch<double>(const BatchTab<double>&, const BatchLaunch&, cudaStream_t, Prof*, bool, bool);

template int launch_flow<float>(const Dev<float>&, const Konst<float>&, cudaStream_t, Prof*, bool, bool, bool);
template int launch_flow<double>(const Dev<double>&, const Konst<double>&, cudaStream_t, Prof*, bool, bool, bool);

}  // namespace xbg
