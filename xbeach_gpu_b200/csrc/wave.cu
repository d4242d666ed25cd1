// wave.cu -- wave action balance of one step (wavestep, Wavestep.cu:755-1167;
// arithmetic of the reference's CPU judge, wave_CPU.cpp).
//
// Kernels (launch order):
//   k_disp       dispersion (wave_CPU.cpp:154-205) per cell -> k, c, cg
//   k_wave_fast  rows 1..ny-2, one thread per cell, bins streamed in order:
//                offshore boundary + sanity + action, x/y/theta second-order
//                upwind advection of ee and rr with the Euler step (in energy
//                units), then energint, roelvink|baldock, dissipation,
//                meandir, radstress.  Each bin's ee/rr plane tile (32 x 8
//                cells + 2-cell halo) streams into shared memory by cp.async
//                three bins ahead (five buffers, one barrier per bin), and
//                the cell's own bins for the theta fluxes come from the
//                resident tiles; ctheta
//                (propagtheta) is evaluated on the fly from per-cell slopes;
//                the theta-face flux is computed once and carried to the
//                next bin.  The threads of rows 1 and ny-2 then also
//                finish rows 0 and ny-1, whose ee/rr are copies of theirs
//                (rollerlatbnd, wave_CPU.cpp:830-870) around the
//                dissipation.  Emits the per-block WAVEDT minimum.
//   k_wave_force wavforce + twodimbnd(noix) + breakerdelay + twodimbnd(ust).
#include <type_traits>

#include "xbg_common.cuh"
#include "../../include/xbg.h"

namespace xbg {

// dispersion relation, wave_CPU.cpp:154-205 (golden-ratio relaxation)
template <class R>
__device__ void disp_cell(const Konst<R>& K, R sg, R h, R& k_, R& c_, R& cg_) {
    R g = K.g;
    R L0 = K.twopi * g / (sg * sg);
    R L1 = L0, L2, errdisp;
    // FP32: the relaxation in float (the reference promotes tanh's argument to
    // double through its pi; the stopping rule |L2 - L1| <= 1e-4 m bounds the
    // difference).  FP64: as written.
    const R kh0 = (R)(2 * XBG_PI) * h;
    for (int n = 1; n < 200; n++) {
        if constexpr (sizeof(R) == 4) L2 = L0 * tanhf(kh0 / L1);
        else L2 = (R)((double)L0 * ::tanh(2 * XBG_PI * (double)h / (double)L1));
        errdisp = DM<R>::fabs(L2 - L1);
        L1 = (L1 * K.aphi + L2 * K.bphi);
        if (errdisp <= 0.0001f) break;
        if (n == 199) {
            L1 = L0 * DM<R>::pow(DM<R>::tanh(DM<R>::pow(sg * sg * h / g, (R)(3.0f / 4.0f))), (R)(2.0f / 3.0f));
            break;
        }
    }
    R kk = (R)(2 * XBG_PI / (double)L1);
    k_ = kk;
    R cc = sg / kk;
    c_ = cc;
    R kkhh = cmin(kk * h, (R)10.0f);
    R s2kh = DM<R>::sinh((R)2.0f * kkhh);
    cg_ = cc * ((R)0.5f + kkhh / s2kh);
}

template <class R>
__device__ __forceinline__ void b_disp(const Dev<R>& S, const Konst<R>& K, const int bix, const int biy) {
    const bool off = wave_off(S.clk);   // tested once the cell's loads are issued (see halted())
    int i = bix * blockDim.x + threadIdx.x;
    if (i >= S.C) return;
    const R sg = (R)S.clk->sigm, h = ld(S.f[HH] + i);
    loads_before_here();
    if (off) return;
    R k_, c_, cg_;
    disp_cell(K, sg, h, k_, c_, cg_);
    S.f[WK][i] = k_;
    S.f[CC_][i] = c_;
    S.f[CG][i] = cg_;
}
XBG_KERNELS(disp)

// Per-cell slope terms of propagtheta (wave_CPU.cpp:226-306).
template <class R>
struct CthCoef { R s, dhdx, dhdy, dudx, dudy, dvdx, dvdy, wci, sg; };

template <class R>
__device__ __forceinline__ CthCoef<R> cth_coef(const Dev<R>& S, const Konst<R>& K, int ix, int iy, R sg) {
    const int nx = K.nx, ny = K.ny;
    const R* hh = S.f[HH]; const R* uu = S.f[UU]; const R* vv = S.f[VV];
    int xm = mm(ix), xp = pp(ix, nx), ym = mm(iy), yp = pp(iy, ny);
    R dxf = K.dx;
    R sx = (R)(xp - xm) * dxf, sy = (R)(yp - ym) * dxf;
    CthCoef<R> c;
    c.dhdx = (ld(hh + xp + iy * nx) - ld(hh + xm + iy * nx)) / sx;
    c.dudx = (ld(uu + xp + iy * nx) - ld(uu + xm + iy * nx)) / sx;
    c.dvdx = (ld(vv + xp + iy * nx) - ld(vv + xm + iy * nx)) / sx;
    c.dhdy = (ld(hh + ix + yp * nx) - ld(hh + ix + ym * nx)) / sy;
    c.dudy = (ld(uu + ix + yp * nx) - ld(uu + ix + ym * nx)) / sy;
    c.dvdy = (ld(vv + ix + yp * nx) - ld(vv + ix + ym * nx)) / sy;
    int i = ix + iy * nx;
    R h = ld(hh + i);
    R kh = cmin(ld(S.f[WK] + i) * h, (R)10.0f);
    c.s = sg / DM<R>::sinh((R)2.0f * kh);
    c.wci = K.wci * cmin(h / K.hwci, (R)1.0f);
    c.sg = sg;
    return c;
}
template <class R>
__device__ __forceinline__ R cth_eval(const CthCoef<R>& c, R cx, R sx) {
    R ctht = (c.s) * (c.dhdx * sx - c.dhdy * cx) +
             c.wci * (cx * (sx * c.dudx - cx * c.dudy) + sx * (sx * c.dvdx - cx * c.dvdy));
    return cmin(cmax(ctht, (R)(-0.25f * c.sg)), (R)(0.25f * c.sg));
}

template <class R>
__device__ __forceinline__ void block_min_store(R v, R* dst) {
    // warp shuffle, then one value per warp through shared memory
    for (int o = 16; o > 0; o >>= 1) v = DM<R>::fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    __shared__ R wmin[32];
    int tid = threadIdx.x + threadIdx.y * blockDim.x;
    int nw = (blockDim.x * blockDim.y + 31) / 32;
    if ((tid & 31) == 0) wmin[tid >> 5] = v;
    __syncthreads();
    if (tid < 32) {
        R m = tid < nw ? wmin[tid] : (R)3.0e38f;
        for (int o = 16; o > 0; o >>= 1) m = DM<R>::fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (tid == 0) *dst = m;
    }
}

#define WT_X 32
#define WT_Y 8
#define WT_TX (WT_X + 4)
#define WT_TY (WT_Y + 4)
#define WT_N (WT_TX * WT_TY)
// ------------------------------------------------------------------------
// Fast rows pass.  Same algorithm as k_wave_tile, arranged for instruction
// throughput (the pass is issue-bound, not HBM-bound):
//  - ee is advected in energy units: action (ee/sigm), the Euler step and
//    energy (*sigm) of the reference cancel for the uniform sigm, and the
//    upwind selection is scale invariant, so A*sigm = ee - dt*(fluxes of ee);
//  - upwind choices are selects instead of branches (no divergence);
//  - reciprocals of the uniform divisors (dtheta, idiv, D/E) multiply;
//  - WAVEDT's min over bins of a/|ctheta| is a/max|ctheta| (one division);
//  - the theta tables live in shared memory, plane pointers advance by C.
// Results agree with the reference arithmetic to a few ulps per operation.
template <class R>
__device__ __forceinline__ R upw(R a, R b) {   // 1.5a - 0.5b, first-order fallback
    R v = DM<R>::fma((R)1.5, a, (R)-0.5 * b);
    return v < (R)0 ? a : v;
}
// The upwind side is chosen first and one extrapolation evaluated (the same
// value as evaluating both sides and selecting).
template <class R>
__device__ __forceinline__ R flux2(R qm2, R qm, R qi, R qp, R qp2, R cf, R cfmin) {
    const bool pin = cf > (R)0, pmin = cfmin > (R)0;
    const R arrin = upw(pin ? qi : qp, pin ? qm : qp2) * cf;
    const R arrmin = upw(pmin ? qm : qi, pmin ? qm2 : qp) * cfmin;
    return arrin - arrmin;
}
// The same flux when the sign of the face speeds is known for the whole bin:
// the speeds cg and c are positive, so without wave-current interaction the
// face speed 0.5 (cg_i + cg_j) cos(theta) has the sign of cos(theta) (of
// sin(theta) for y), and a zero speed gives a zero flux on either side.  Only
// the two upwind taps at stride s are read.
template <class R, bool POS>
__device__ __forceinline__ R flux2s(const R* q, int s, R qi, R cf, R cfmin) {
    if (POS) {
        const R qm = q[-s], qm2 = q[-2 * s];
        const R arrin = upw(qi, qm) * cf;
        const R arrmin = upw(qm, qm2) * cfmin;
        return arrin - arrmin;
    } else {
        const R qp = q[s], qp2 = q[2 * s];
        const R arrin = upw(qp, qp2) * cf;
        const R arrmin = upw(qi, qp) * cfmin;
        return arrin - arrmin;
    }
}
// Without wave-current interaction every face speed of a bin is a cell
// constant times cos(theta) (x) or sin(theta) (y).  The cell constants carry
// dt / dx (kin, kmin: the face speeds 0.5 (cg_i + cg_j) dt / dx), so a bin's
// x or y flux difference is cos (sin) times fk(), and its Euler update
// A = e - (cos fk_x + sin fk_y + dt / dtheta (theta-face difference)).  The
// upwind side is the one of cos (sin): pos.  Both rows-pass kernels use
// these two (bit-identical results).
template <class R, bool POS>
__device__ __forceinline__ R flux2k(const R* q, int s, R qi, R kin, R kmin) {
    R ain, amin;
    if (POS) {
        const R qm = q[-s];
        ain = upw(qi, qm);
        amin = upw(qm, q[-2 * s]);
    } else {
        const R qp = q[s];
        ain = upw(qp, q[2 * s]);
        amin = upw(qi, qp);
    }
    return DM<R>::fma(ain, kin, -(amin * kmin));
}
template <class R>
__device__ __forceinline__ R flux2kv(R qm2, R qm, R qi, R qp, R qp2, bool pos, R kin, R kmin) {
    const R ain = upw(pos ? qi : qp, pos ? qm : qp2);
    const R amin = upw(pos ? qm : qi, pos ? qm2 : qp);
    return DM<R>::fma(ain, kin, -(amin * kmin));
}
template <class R>
__device__ __forceinline__ R euler_k(R e, R ct, R st, R fkx, R fky, R ft, R kth) {
    return e - DM<R>::fma(ct, fkx, DM<R>::fma(st, fky, ft * kth));
}

// theta-face flux between bins t and t+1 (the arrint of bin t, which is the
// arrmint of bin t+1): e(t-1), e(t), e(t+1), e(t+2), ctheta(t), ctheta(t+1)
template <class R>
__device__ __forceinline__ R theta_face(R em, R e0, R ep, R ep2, R c0, R cp) {
    const R cb = (R)0.5f * (c0 + cp);
    const bool p = cb > (R)0;
    const R a = p ? e0 : ep, b = p ? em : ep2;
    R u = DM<R>::fma((R)1.5f, a, DM<R>::mul((R)-0.5f, b));
    u = u < (R)0 ? a : u;
    return cb * u;
}

// The same arithmetic on (wave energy, roller energy) pairs with the packed
// FP32 instructions of sm_100 (fma / mul / add .f32x2): each lane rounds as
// the scalar operation it replaces, so the results are the scalar path's bit
// for bit, in half the floating-point instructions.  kminn is -kmin, and the
// Euler update is written with negated factors (exact under round-to-nearest).
__device__ __forceinline__ float2 upw2(float2 a, float2 b) {
    float2 v = __ffma2_rn(make_float2(1.5f, 1.5f), a, __fmul2_rn(make_float2(-0.5f, -0.5f), b));
    v.x = v.x < 0.f ? a.x : v.x;
    v.y = v.y < 0.f ? a.y : v.y;
    return v;
}
template <bool POS>
__device__ __forceinline__ float2 flux2k2(const float* qE, const float* qR, int s, float2 qi, float2 kin,
                                          float2 kminn) {
    float2 ain, amin;
    if (POS) {
        const float2 qm = make_float2(qE[-s], qR[-s]);
        ain = upw2(qi, qm);
        amin = upw2(qm, make_float2(qE[-2 * s], qR[-2 * s]));
    } else {
        const float2 qp = make_float2(qE[s], qR[s]);
        ain = upw2(qp, make_float2(qE[2 * s], qR[2 * s]));
        amin = upw2(qi, qp);
    }
    return __ffma2_rn(ain, kin, __fmul2_rn(amin, kminn));
}
__device__ __forceinline__ float2 theta_face2(float2 em, float2 e0, float2 ep, float2 ep2, float c0, float cp) {
    const float cb = 0.5f * (c0 + cp);
    const bool p = cb > 0.f;
    const float2 a = p ? e0 : ep, b = p ? em : ep2;
    float2 u = __ffma2_rn(make_float2(1.5f, 1.5f), a, __fmul2_rn(make_float2(-0.5f, -0.5f), b));
    u.x = u.x < 0.f ? a.x : u.x;
    u.y = u.y < 0.f ? a.y : u.y;
    return __fmul2_rn(make_float2(cb, cb), u);
}

// Direction tables of the bins in shared memory: (cos, sin) and
// (cos^2, sin^2, sin cos, theta), one vector load each.
template <class R> struct alignas(2 * sizeof(R)) Dir2 { R c, s; };
template <class R> struct alignas(4 * sizeof(R)) Dir4 { R c2, s2, cs, th; };

// energint + roelvink|baldock (wave_CPU.cpp:873-1028) of one cell from the sum
// over bins of its sanitised advected ee: 1/idiv, Dv and Dv / max(Eint, 1e-7).
template <class R>
__device__ __forceinline__ void wave_breaking(const Konst<R>& K, R esum, R hh, R k, R fw, R Trep, R& ridiv, R& Dv,
                                              R& Dq) {
    const R rho = K.rho, g = K.g;
    const R Etmp = esum * K.dtheta;
    R Htmp = DM<R>::sqrt(Etmp / (rho * g / (R)8.0f));
    const R hr = Htmp / (K.gammax * hh);
    const R idiv = DM<R>::fmax((R)1.0f, hr * hr);
    ridiv = (R)1 / idiv;
    Htmp = DM<R>::fmin(Htmp, K.gammax * hh);
    const R Eint = (rho * g * Htmp * Htmp) / (R)8.0f;
    if (K.breakmodel == 1) {   // roelvinkCPU
        R Ht = DM<R>::sqrt(Eint * (R)(8.0 / (double)rho / (double)g));
        R x = Ht / K.gammaa / hh;
        R Qb = (R)1 - DM<R>::exp(DM<R>::fmax(-DM<R>::pow(x, K.nexp), (R)-100));
        Qb = DM<R>::fmin(Qb, (R)1.0f);
        Dv = Qb * (R)2 * K.alpha / Trep * Eint * Ht / hh;
        R uorb = (R)XBG_PI * Ht / (Trep * DM<R>::sinh(DM<R>::fmin(k * hh, (R)10.0f)));
        Dv = Dv + (R)(0.66666666f / XBG_PI) * rho * fw * uorb * uorb * uorb;
    } else {                   // baldockCPU
        R khh = k * hh;
        R Hb = ((R)0.88f / k) * DM<R>::tanh(K.gammaa * khh / (R)0.88f);
        R Rr = Hb / DM<R>::fmax(Htmp, (R)0.00001f);
        R Qb = DM<R>::exp((R)-1.0f * Rr * Rr);
        Dv = (R)0.25f * K.alpha * Qb * rho * ((R)1.0f / Trep) * g * (Hb * Hb + Htmp * Htmp);
        R uorb = (R)XBG_PI * Htmp / (Trep * DM<R>::sinh(DM<R>::fmin(k * hh, (R)10.0f)));
        Dv = Dv + (R)(0.66666666f / XBG_PI) * rho * fw * uorb * uorb * uorb;
    }
    Dq = Dv / DM<R>::fmax(Eint, (R)0.0000001f);
}

// dissipationCPU's wave-energy part of one bin (wave_CPU.cpp:1258-1295): the
// sanitised advected energy a scaled by 1/idiv, its dissipation dd = e Dq,
// and the new energy max(e - dt dd, 0).  One definition for every kernel
// that forms it, so they round alike.
template <class R>
__device__ __forceinline__ R diss_ee(R a, R ridiv, R Dq, R dtf, R& dd) {
    const R eet = DM<R>::mul(DM<R>::fmax(a, (R)0.0f), ridiv);
    dd = DM<R>::mul(eet, Dq);
    return DM<R>::fmax(DM<R>::fma(-dtf, dd, eet), (R)0.0f);
}
// the roller energy of one bin after the roller's dissipation (rrd, the
// dissipation term) and the wave breaking dissipation dd it gains
template <class R>
__device__ __forceinline__ R diss_rr(R rrt, R rrd, R dd, R dtf) {
    return DM<R>::fmax(DM<R>::fma(dtf, dd - rrd, rrt), (R)0.0f);
}

// radstress (wave_CPU.cpp:1123-1162) of one cell from its bin sums: sum2 =
// sum ee, ec / es / ecs = sum (cos^2, sin^2, sin cos) ee, rc / rs / rcs the
// same for rr, n = cg / c.  Every product and fused product is written out,
// so the rounding is the same in every kernel that stores them.
template <class R>
__device__ __forceinline__ void radstress(R* sxx, R* sxy, R* syy, int i, R n, R sum2, R ec, R es, R ecs, R rc, R rs,
                                          R rcs, R dth) {
    const R half = DM<R>::mul((R)-0.5f, sum2);
    sxx[i] = DM<R>::fma(DM<R>::fma(n, sum2 + ec, half), dth, DM<R>::mul(rc, dth));
    syy[i] = DM<R>::fma(DM<R>::fma(n, sum2 + es, half), dth, DM<R>::mul(rs, dth));
    sxy[i] = DM<R>::fma(DM<R>::mul(n, ecs), dth, DM<R>::mul(rcs, dth));
}

// Row 0 or ny-1 (iyE), the lateral copy of row iyS = 1 or ny-2
// (rollerlatbnd, wave_CPU.cpp:830-870, around dissipationCPU): its advected
// ee and rr are the source row's times the wet mask, breaking and roller
// dissipation run with the edge cell's own depth and speeds, and after
// dissipation its ee is again the source row's (final) ee times the mask.
// Run by the thread of the source cell, which holds the advected bins in
// sA / sR; src_final(t) gives the source cell's final ee of bin t.  Returns
// the edge cell's WAVEDT.
template <class R, bool ROLLER, bool WCI, class SrcFinal>
__device__ __forceinline__ R wave_edge_cell(const Dev<R>& S, const Konst<R>& K, int ix, int iyE, const R* sA,
                                            const R* sR, const Dir2<R>* sCS2, const Dir4<R>* sMom, R esum, R sg,
                                            R dtf, R Trep, const R* rro, R* een, R* rrn, SrcFinal&& src_final) {
    const int nx = K.nx, nt = K.nt, C = S.C;
    const int ie = ix + iyE * nx;
    const R dth = K.dtheta, rho = K.rho, g = K.g;
    const R hE = ld(S.f[HH] + ie);
    const bool wet = hE > K.eps;
    const R w = wet ? (R)1.0f : (R)0.0f;
    // WAVEDT: cfl*dtheta over the largest |ctheta| of the edge cell's bins
    const CthCoef<R> ce = cth_coef(S, K, ix, iyE, sg);
    const R P = ce.s * ce.dhdx, Q = -(ce.s * ce.dhdy);
    R cab = (R)0;
    for (int t = 0; t < nt; t++) {
        const Dir2<R> d = sCS2[t];
        R c;
        if (WCI) c = cth_eval(ce, d.c, d.s);
        else c = cmin(cmax(DM<R>::fma(P, d.s, Q * d.c), (R)(-0.25f * ce.sg)), (R)(0.25f * ce.sg));
        cab = DM<R>::fmax(cab, DM<R>::fabs(c));
    }
    const R dtw = DM<R>::fmin(K.cfl * dth / cab, (R)9999999.9f);
    // sum of max(A * w, 0) over the bins: the source's sum, or 0 when dry
    R ridiv, Dv, Dq;
    wave_breaking(K, wet ? esum : (R)0, hE, ld(S.f[WK] + ie), ld(S.f[FWM] + ie), Trep, ridiv, Dv, Dq);
    const R cE = ld(S.f[CC_] + ie);
    const R twogb = (R)2.0f * g * K.beta;
    R uE = (R)0, vE = (R)0;
    if (WCI) {
        const R wc = K.wci * cmin(hE / K.hwci, (R)1.0f);
        uE = ld(S.f[UU] + ie) * wc;
        vE = wc * ld(S.f[VV] + ie);
    }
    const R rcoef = twogb / cE;
    const int tid = threadIdx.x + threadIdx.y * WT_X;
    R RR = (R)0, drr = (R)0, rc = (R)0, rs = (R)0, rcs = (R)0;
    for (int t = 0; t < nt; t++) {
        const R eet = DM<R>::fmax(sA[t * 256 + tid] * w, (R)0.0f) * ridiv;
        R rrt = ROLLER ? sR[t * 256 + tid] * w : ld(rro + ie + (size_t)t * C);
        const R dd = eet * Dq;
        R rrd;
        if (WCI) {
            const Dir2<R> d = sCS2[t];
            const R cx = cE * d.c + uE, cy = cE * d.s + vE;
            rrd = twogb * rrt / DM<R>::sqrt(cx * cx + cy * cy);
        } else {
            rrd = DM<R>::mul(rrt, rcoef);
        }
        rrt = wet ? diss_rr(rrt, rrd, dd, dtf) : (R)0;
        drr = wet ? drr + rrd : (R)0;
        RR = RR + rrt;
        rrn[ie + (size_t)t * C] = rrt;
        const Dir4<R> m = sMom[t];
        rc = DM<R>::fma(m.c2, rrt, rc);
        rs = DM<R>::fma(m.s2, rrt, rs);
        rcs = DM<R>::fma(m.cs, rrt, rcs);
    }
    // the second copy of ee: the source cell's final bins
    R sume = (R)0, sumethet = (R)0, ec = (R)0, es = (R)0, ecs = (R)0;
    for (int t = 0; t < nt; t++) {
        const R eet = src_final(t) * w;
        een[ie + (size_t)t * C] = eet;
        const Dir4<R> m = sMom[t];
        sume = sume + eet;
        sumethet = DM<R>::fma(eet, m.th, sumethet);
        ec = DM<R>::fma(m.c2, eet, ec);
        es = DM<R>::fma(m.s2, eet, es);
        ecs = DM<R>::fma(m.cs, eet, ecs);
    }
    const R sum2 = sume;
    sume = DM<R>::fmax(sume, (R)0.00001f);
    S.f[THM][ie] = sumethet / sume;
    S.f[E][ie] = sume * dth;
    S.f[H][ie] = DM<R>::sqrt(sume * dth / (rho * g / (R)8));
    S.f[D][ie] = Dv;
    S.f[ROL][ie] = RR * dth;
    S.f[DR][ie] = drr * dth;
    const R n = ld(S.f[CG] + ie) / cE;
    radstress(S.tmp[T_SXX], S.tmp[T_SXY], S.tmp[T_SYY], ie, n, sum2, ec, es, ecs, rc, rs, rcs, dth);
    return dtw;
}

// Plane tile buffers.  At bin t planes t, t+1 and t+2 are resident (the
// stencil of plane t; the cell's own values of planes t+1 and t+2 for the
// theta fluxes) and plane t+3 streams in; it goes into the buffer of plane
// t-2, which every thread finished reading before the previous barrier.
constexpr int WT_NB = 5;

template <class R, bool ROLLER, bool WCI>
__device__ __forceinline__ void b_wave_fast(const Dev<R>& S, const Konst<R>& K, const int bix, const int biy) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Clock* clk = S.clk;
    if (wave_off(clk)) return;
    const int nx = K.nx, ny = K.ny, nt = K.nt, C = S.C;
    const int tid = threadIdx.x + threadIdx.y * WT_X;
    R* tE = (R*)smem_raw;                 // [WT_NB][WT_N] plane tiles of ee
    R* tR = tE + WT_NB * WT_N;            // [WT_NB][WT_N] plane tiles of rr
    R* sA = tR + WT_NB * WT_N;            // [nt][256] advected ee (energy units)
    R* sR = sA + (size_t)nt * 256;        // [nt][256] advected rr
    Dir4<R>* sMom = reinterpret_cast<Dir4<R>*>(sR + (size_t)nt * 256);   // [nt]
    Dir2<R>* sCS2 = reinterpret_cast<Dir2<R>*>(sMom + nt);               // [nt]
    if (tid < nt) {
        const R c = K.cxsth[tid], sn = K.sxnth[tid];
        sCS2[tid] = Dir2<R>{c, sn};
        sMom[tid] = Dir4<R>{c * c, sn * sn, sn * c, K.theta[tid]};
    }
    const int bx0 = bix * WT_X, by0 = 1 + biy * WT_Y;
    const int ix = bx0 + threadIdx.x, iy = by0 + threadIdx.y;
    const bool active = ix < nx && iy <= ny - 2;
    const int par = clk->par;
    const R* eeo = S.ee[par ^ 1];
    const R* rro = S.rr[par ^ 1];
    const R dtf = (R)clk->dt;
    const R taper = (R)cmin((double)(R)clk->totaltime / 100.0, 1.0);
    const R* St = S.St;
    const R dth = K.dtheta;
    const R rdth = (R)1 / dth;
    const R rdx = (R)1 / K.dx;
    // tile elements of this thread (two at most): plane offsets, clamped as
    // mm()/pp()/mm2()/pp2() clamp; column 0 is the offshore boundary St*taper
    int eoff0 = -1, eoff1 = -1, ey0 = 0, ey1 = 0;
    bool ez0 = false, ez1 = false;
    {
        int e = tid, kx = e % WT_TX, ky = e / WT_TX;
        int gx = min(max(bx0 - 2 + kx, 0), nx - 1), gy = min(max(by0 - 2 + ky, 0), ny - 1);
        eoff0 = gx + gy * nx; ey0 = gy; ez0 = gx == 0;
        e = tid + 256;
        if (e < WT_N) {
            kx = e % WT_TX; ky = e / WT_TX;
            gx = min(max(bx0 - 2 + kx, 0), nx - 1); gy = min(max(by0 - 2 + ky, 0), ny - 1);
            eoff1 = gx + gy * nx; ey1 = gy; ez1 = gx == 0;
        }
    }
    // sources of this thread's tile elements in the next plane to issue
    const R* gE0 = eeo + eoff0; const R* gR0 = rro + eoff0; const R* gS0 = St + ey0;
    const R* gE1 = eeo + max(eoff1, 0); const R* gR1 = rro + max(eoff1, 0); const R* gS1 = St + ey1;
    // issue the copies of the next plane into buffer b (boundary column written directly)
    auto issue = [&](int b) {
        R* dE = tE + b * WT_N;
        R* dR = tR + b * WT_N;
        if (ez0) dE[tid] = DM<R>::fmax(*gS0 * taper, (R)0);
        else cp_async<sizeof(R)>(dE + tid, gE0);
        if (ROLLER) cp_async<sizeof(R)>(dR + tid, gR0);
        if (eoff1 >= 0) {
            if (ez1) dE[tid + 256] = DM<R>::fmax(*gS1 * taper, (R)0);
            else cp_async<sizeof(R)>(dE + tid + 256, gE1);
            if (ROLLER) cp_async<sizeof(R)>(dR + tid + 256, gR1);
        }
        cp_async_commit();
        gE0 += C; gR0 += C; gS0 += ny; gE1 += C; gR1 += C; gS1 += ny;
    };
    // sanity (ee = max(ee, 0)) on this thread's copied elements of buffer b
    auto fixup = [&](int b) {
        R* dE = tE + b * WT_N;
        if (!ez0) dE[tid] = DM<R>::fmax(dE[tid], (R)0);
        if (eoff1 >= 0 && !ez1) dE[tid + 256] = DM<R>::fmax(dE[tid + 256], (R)0);
    };
    // the cell's tile slot; the tile is clamped like mm()/pp()/mm2()/pp2(), so
    // its x/y neighbours are at fixed offsets +-1, +-2, +-WT_TX, +-2*WT_TX
    const int ctile = (iy - by0 + 2) * WT_TX + (ix - bx0 + 2);
    int i = 0;
    R hh = 0, uui = 0, vvi = 0;
    // face speeds as ct * A + B (x faces) and st * A + B (y faces), for cg (ee) and c (rr)
    R axp = 0, axm = 0, ayp = 0, aym = 0, rxp = 0, rxm = 0, ryp = 0, rym = 0;
    R bxp = 0, bxm = 0, byp = 0, bym = 0, cgi = 0, cci = 0;
    CthCoef<R> cc{};
    R we1 = 0, we2 = 0, we3 = 0, we4 = 0, wr1 = 0, wr2 = 0, wr3 = 0, wr4 = 0;   // bins t-1 .. t+2
    R c0 = 0, cpp = 0, Etmp = 0, cabs = 0, fte = 0, ftr = 0;
    // ctheta of a bin (propagtheta); without wave-current interaction only the
    // depth-refraction term remains: s (dhdx sin - dhdy cos)
    R cthP = 0, cthQ = 0;
    auto cth = [&](R cx, R sx) -> R {
        if (WCI) return cth_eval(cc, cx, sx);
        const R ctht = DM<R>::fma(cthP, sx, cthQ * cx);
        return cmin(cmax(ctht, (R)(-0.25f * cc.sg)), (R)(0.25f * cc.sg));
    };
    // planes 0, 1, 2 (empty groups past the last plane)
    issue(0);
    if (nt > 1) issue(1); else cp_async_commit();
    if (nt > 2) issue(2); else cp_async_commit();
    __syncthreads();   // theta tables
    if (active) {
        i = ix + iy * nx;
        const int xm = mm(ix), xp = pp(ix, nx);
        const int ym = mm(iy), yp = pp(iy, ny);
        hh = ld(S.f[HH] + i);
        R sg = (R)clk->sigm;
        cc = cth_coef(S, K, ix, iy, sg);
        const R wci = cc.wci;
        const R* cgp = S.f[CG];
        const R* cp = S.f[CC_];
        cgi = ld(cgp + i); cci = ld(cp + i);
        // without wave-current interaction the face speeds carry dt / dx
        // (flux2kv, euler_k: the arithmetic of the TMA rows pass)
        const R h = WCI ? (R)0.5f : (R)0.5f * (dtf * rdx);
        axp = h * (cgi + ld(cgp + xp + iy * nx)); axm = h * (cgi + ld(cgp + xm + iy * nx));
        ayp = h * (cgi + ld(cgp + ix + yp * nx)); aym = h * (cgi + ld(cgp + ix + ym * nx));
        rxp = h * (cci + ld(cp + xp + iy * nx)); rxm = h * (cci + ld(cp + xm + iy * nx));
        ryp = h * (cci + ld(cp + ix + yp * nx)); rym = h * (cci + ld(cp + ix + ym * nx));
        const R* uu = S.f[UU]; const R* vv = S.f[VV];
        uui = ld(uu + i) * wci; vvi = wci * ld(vv + i);
        bxp = h * (uui + ld(uu + xp + iy * nx) * wci); bxm = h * (uui + ld(uu + xm + iy * nx) * wci);
        byp = h * (vvi + wci * ld(vv + ix + yp * nx)); bym = h * (vvi + wci * ld(vv + ix + ym * nx));
        auto cl = [&](int t) { return t < 0 ? 0 : (t >= nt ? nt - 1 : t); };
        if (!WCI) { cthP = cc.s * cc.dhdx; cthQ = -(cc.s * cc.dhdy); }
        c0 = cth(sCS2[0].c, sCS2[0].s);
        cpp = cth(sCS2[cl(1)].c, sCS2[cl(1)].s);
    }
    cp_async_wait1();   // planes 0 and 1 have landed (this thread's copies)
    fixup(0);
    if (nt > 1) fixup(1);
    R* oA = sA + tid;
    R* oR = sR + tid;
    const R* oldR = rro + i;   // without the roller pass rr is carried unchanged
#pragma unroll 1
    for (int t = 0; t < nt; t++) {
        const int b = t % WT_NB;
        if (t + 3 < nt) issue((t + 3) % WT_NB);
        else cp_async_commit();
        cp_async_wait1();   // plane t+2 has landed (this thread's copies)
        if (t + 2 < nt) fixup((t + 2) % WT_NB);
        __syncthreads();    // ... and every thread's
        if (active) {
            const R* qE = tE + b * WT_N + ctile;
            const R* qR = tR + b * WT_N + ctile;
            // the cell's own bins t-1 .. t+2 (clamped to the last bin)
            if (t == 0) {
                const int b1 = (nt > 1 ? 1 : 0);
                we2 = qE[0]; we1 = we2; we3 = tE[b1 * WT_N + ctile];
                if (ROLLER) { wr2 = qR[0]; wr1 = wr2; wr3 = tR[b1 * WT_N + ctile]; }
            }
            const int b2 = (t + 2 < nt ? t + 2 : nt - 1) % WT_NB;
            we4 = tE[b2 * WT_N + ctile];
            if (ROLLER) wr4 = tR[b2 * WT_N + ctile];
            const Dir2<R> d = sCS2[t];
            const R ct = d.c, st = d.s;
            const bool last = t == nt - 1;
            cabs = DM<R>::fmax(cabs, DM<R>::fabs(c0));
            // theta flux: upper face computed here, lower face carried from bin t-1
            R fup = last ? (R)0 : theta_face(we1, we2, we3, we4, c0, cpp);
            R ft = fup - fte;
            fte = fup;
            R A;
            const bool px = ct > (R)0, py = st > (R)0;
            if (WCI) {
                R fx = flux2(qE[-2], qE[-1], we2, qE[1], qE[2], DM<R>::fma(ct, axp, bxp), DM<R>::fma(ct, axm, bxm));
                R fy = flux2(qE[-2 * WT_TX], qE[-WT_TX], we2, qE[WT_TX], qE[2 * WT_TX], DM<R>::fma(st, ayp, byp),
                             DM<R>::fma(st, aym, bym));
                A = we2 - dtf * ((fx + fy) * rdx + ft * rdth);
            } else {
                R fx = flux2kv(qE[-2], qE[-1], we2, qE[1], qE[2], px, axp, axm);
                R fy = flux2kv(qE[-2 * WT_TX], qE[-WT_TX], we2, qE[WT_TX], qE[2 * WT_TX], py, ayp, aym);
                A = euler_k(we2, ct, st, fx, fy, ft, dtf * rdth);
            }
            R Ar;
            if (!ROLLER) Ar = ld(oldR + (size_t)t * C);
            if (ROLLER) {
                R rup = last ? (R)0 : theta_face(wr1, wr2, wr3, wr4, c0, cpp);
                R rt = rup - ftr;
                ftr = rup;
                if (WCI) {
                    R rx = flux2(qR[-2], qR[-1], wr2, qR[1], qR[2], DM<R>::fma(ct, rxp, bxp),
                                 DM<R>::fma(ct, rxm, bxm));
                    R ry = flux2(qR[-2 * WT_TX], qR[-WT_TX], wr2, qR[WT_TX], qR[2 * WT_TX],
                                 DM<R>::fma(st, ryp, byp), DM<R>::fma(st, rym, bym));
                    Ar = wr2 - dtf * ((rx + ry) * rdx + rt * rdth);
                } else {
                    R rx = flux2kv(qR[-2], qR[-1], wr2, qR[1], qR[2], px, rxp, rxm);
                    R ry = flux2kv(qR[-2 * WT_TX], qR[-WT_TX], wr2, qR[WT_TX], qR[2 * WT_TX], py, ryp, rym);
                    Ar = euler_k(wr2, ct, st, rx, ry, rt, dtf * rdth);
                }
            }
            *oA = A;
            *oR = Ar;
            oA += 256; oR += 256;
            Etmp = Etmp + DM<R>::fmax(A, (R)0);
            const int t2 = t + 2 < nt ? t + 2 : nt - 1;
            we1 = we2; we2 = we3; we3 = we4;
            wr1 = wr2; wr2 = wr3; wr3 = wr4;
            const Dir2<R> d2 = sCS2[t2];
            c0 = cpp; cpp = cth(d2.c, d2.s);
        }
    }
    R dtw = (R)3.0e38f;
    if (active) {
        // WAVEDT: min over bins of cfl*dtheta/|ctheta| (Wave_kernel.cu:232-249)
        dtw = DM<R>::fmin(K.cfl * dth / cabs, (R)9999999.9f);
        R* een = S.ee[par];
        R* rrn = S.rr[par];
        const R Trep = (R)clk->Trep;
        const R rho = K.rho, g = K.g;
        R ridiv, Dv, Dq;
        wave_breaking(K, Etmp, hh, ld(S.f[WK] + i), ld(S.f[FWM] + i), Trep, ridiv, Dv, Dq);
        // dissipationCPU, meandir, radstress
        const R cc_i = cci;
        const R twogb = (R)2.0f * g * K.beta;
        const R rcoef = twogb / cc_i;   // without wave-current interaction |c (cos, sin)| = c
        const bool wet = hh > K.eps;
        R RR = (R)0.0f, drr = (R)0.0f, sume = (R)0, sumethet = (R)0;
        R ec = 0, es = 0, ecs = 0, rc = 0, rs = 0, rcs = 0;   // sums of cos^2, sin^2, sin cos times e / r
        R* pe_n = een + i;
        R* pr_n = rrn + i;
        if (wet) {
#pragma unroll 2
            for (int t = 0; t < nt; t++) {
                R dd;
                R eet = diss_ee(sA[t * 256 + tid], ridiv, Dq, dtf, dd);
                R rrt = sR[t * 256 + tid];
                R rrd;
                if (WCI) {
                    const Dir2<R> d = sCS2[t];
                    const R cx = cc_i * d.c + uui;
                    const R cy = cc_i * d.s + vvi;
                    rrd = twogb * rrt / DM<R>::sqrt(cx * cx + cy * cy);
                } else {
                    rrd = DM<R>::mul(rrt, rcoef);
                }
                rrt = diss_rr(rrt, rrd, dd, dtf);
                drr = drr + rrd;
                RR = RR + rrt;
                pe_n[(size_t)t * C] = eet;
                pr_n[(size_t)t * C] = rrt;
                const Dir4<R> m = sMom[t];
                sume = sume + eet;
                sumethet = DM<R>::fma(eet, m.th, sumethet);
                ec = DM<R>::fma(m.c2, eet, ec);
                es = DM<R>::fma(m.s2, eet, es);
                ecs = DM<R>::fma(m.cs, eet, ecs);
                rc = DM<R>::fma(m.c2, rrt, rc);
                rs = DM<R>::fma(m.s2, rrt, rs);
                rcs = DM<R>::fma(m.cs, rrt, rcs);
            }
        } else {   // dry: ee, rr and every sum are zero
            for (int t = 0; t < nt; t++) {
                pe_n[(size_t)t * C] = (R)0;
                pr_n[(size_t)t * C] = (R)0;
            }
        }
        const R sum2 = sume;
        sume = DM<R>::fmax(sume, (R)0.00001f);
        S.f[THM][i] = sumethet / sume;
        S.f[E][i] = sume * dth;
        S.f[H][i] = DM<R>::sqrt(sume * dth / (rho * g / (R)8));
        S.f[D][i] = Dv;
        S.f[ROL][i] = RR * dth;
        S.f[DR][i] = drr * dth;
        const R n = cgi / cc_i;
        // radstress: sum (1 + cos^2) e = sum e + sum cos^2 e, ...
        radstress(S.tmp[T_SXX], S.tmp[T_SXY], S.tmp[T_SYY], i, n, sum2, ec, es, ecs, rc, rs, rcs, dth);
        // the lateral rows 0 and ny-1, from rows 1 and ny-2
        const R sg = (R)clk->sigm;
        // the source cell's final bins: this thread's own stores, read back
        auto own = [&](int t) { return een[i + (size_t)t * C]; };
        if (iy == 1)
            dtw = DM<R>::fmin(dtw, wave_edge_cell<R, ROLLER, WCI>(S, K, ix, 0, sA, sR, sCS2, sMom, Etmp, sg, dtf, Trep,
                                                                  rro, een, rrn, own));
        if (iy == ny - 2)
            dtw = DM<R>::fmin(dtw, wave_edge_cell<R, ROLLER, WCI>(S, K, ix, ny - 1, sA, sR, sCS2, sMom, Etmp, sg, dtf,
                                                                  Trep, rro, een, rrn, own));
    }
    block_min_store<R>(dtw, S.part_wave + bix + biy * ((K.nx + 31) / 32));
}
template <class R, bool ROLLER, bool WCI>
__global__ void __launch_bounds__(256, 3) k_wave_fast(Dev<R> S, Konst<R> K) {
    b_wave_fast<R, ROLLER, WCI>(S, K, blockIdx.x, blockIdx.y);
}
template <class R, bool ROLLER, bool WCI>
__global__ void __launch_bounds__(256, 3) kb_wave_fast(BatchTab<R> T, const int2* items, int n) {
    batch_items<R>(T, items, n, [&](const Dev<R>& S, const Konst<R>& K, const BatchAux&, int bx, int by) {
        b_wave_fast<R, ROLLER, WCI>(S, K, bx, by);
    });
}
// the four variants (roller on/off, wave-current interaction on/off)
template <class R>
void launch_wave_fast(const Dev<R>& S, const Konst<R>& K, dim3 g, dim3 b, size_t smem, cudaStream_t st) {
    const bool w = K.wci != (R)0;
    if (K.roller == 1) {
        if (w) k_wave_fast<R, true, true><<<g, b, smem, st>>>(S, K);
        else k_wave_fast<R, true, false><<<g, b, smem, st>>>(S, K);
    } else {
        if (w) k_wave_fast<R, false, true><<<g, b, smem, st>>>(S, K);
        else k_wave_fast<R, false, false><<<g, b, smem, st>>>(S, K);
    }
}
template <class R>
void launch_wave_fast_batch(const BatchTab<R>& T, const BatchLaunch& L, int roller, int wci, size_t smem,
                            cudaStream_t st) {
    dim3 b(32, 8);
    const int g = L.grid[BS_WROWS], n = L.n[BS_WROWS];
    const int2* it = L.items[BS_WROWS];
    if (roller == 1) {
        if (wci) kb_wave_fast<R, true, true><<<g, b, smem, st>>>(T, it, n);
        else kb_wave_fast<R, true, false><<<g, b, smem, st>>>(T, it, n);
    } else {
        if (wci) kb_wave_fast<R, false, true><<<g, b, smem, st>>>(T, it, n);
        else kb_wave_fast<R, false, false><<<g, b, smem, st>>>(T, it, n);
    }
}
template <class R>
size_t wave_fast_smem(int nt) { return ((size_t)2 * WT_NB * WT_N + (size_t)2 * nt * 256 + 6 * nt) * sizeof(R); }

// ------------------------------------------------------------------------
// Rows pass with tensor-memory-accelerator (TMA) tiles: the same arithmetic
// as b_wave_fast (identical results), with the data movement moved off the
// threads.
//  - One elected thread loads each bin's ee and rr plane tile with one 2-D
//    box copy (cp.async.bulk.tensor, no multicast) into one of four
//    buffers, completion counted on the buffer's mbarrier; the box starts
//    4 columns left of the block (the 16-byte rule on x) and 2 rows below,
//    40 x 12 cells.  Cells outside the grid arrive as zeros; blocks at the
//    grid's edges rewrite those (and the offshore column, St * taper) with
//    the clamped values the reference reads through mm()/pp().
//  - ee in memory is never negative (every writer stores max(., 0), and
//    xbg_set_field clips what a caller sets), so the tile needs no sanity
//    pass.
//  - The new bins go to shared memory (in place of the advected ones) and
//    leave in two 3-D box stores (all bins of the block's 32 x 8 cells); the
//    store map ends at row ny-2, so rows 0 and ny-1 (rollerlatbnd copies,
//    written by the row 1 / ny-2 threads) are never touched by it.
//  - Every wait on an mbarrier is bounded; a block that gives up records
//    XBG_ERR_TIMEOUT in the clock, halts the step, waits (bounded) for its
//    copies in flight and leaves.
// Used for wave-current interaction off and nx a multiple of 4 (the row
// pitch of a tensor map is a multiple of 16 bytes); else b_wave_fast.
constexpr int TM_X = 40, TM_Y = 12, TM_N = TM_X * TM_Y, TM_NB = 4;
constexpr unsigned TM_WAIT_LIMIT = 1u << 20;   // mbarrier polls before a block gives up (copies land in microseconds)

__device__ __forceinline__ unsigned su32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void tm_mbar_init(unsigned a) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(a) : "memory");
}
__device__ __forceinline__ void tm_expect(unsigned a, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(a), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool tm_wait(unsigned a, unsigned parity) {
    for (unsigned it = 0; it < TM_WAIT_LIMIT; it++) {
        unsigned ok;
        asm volatile(
            "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}
__device__ __forceinline__ void tm_load3(unsigned dst, const CUtensorMap* m, int x, int y, int z, unsigned mbar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];\n" ::"r"(dst),
        "l"((unsigned long long)m), "r"(x), "r"(y), "r"(z), "r"(mbar)
        : "memory");
}
__device__ __forceinline__ void tm_store3(const CUtensorMap* m, int x, int y, int z, unsigned src) {
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];\n" ::"l"(
                     (unsigned long long)m),
                 "r"(x), "r"(y), "r"(z), "r"(src)
                 : "memory");
}
__device__ __forceinline__ void tm_fence_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

template <class R>
size_t wave_tma_smem(int nt) {
    return 128 + ((size_t)2 * TM_NB * TM_N + (size_t)2 * nt * 256 + 6 * nt) * sizeof(R);
}

// The state one thread keeps for one cell of the rows pass.
template <class R>
struct WCell {
    int i, ctile, cid, ix, iy;
    bool active;
    R hh, axp, axm, ayp, aym, rxp, rxm, ryp, rym, cgi, cci, cthP, cthQ;
    R we1, we2, we3, we4, wr1, wr2, wr3, wr4, c0, cpp, Etmp, cabs, fte, ftr;
    // the packed FP32 path: (ee, rr) window, face speeds (upper, lower negated),
    // the negated θ flux of the face below
    float2 p1, p2, p3, p4, kx, kxn, ky, kyn, ften;
};

// CPT cells per thread: the block is 32 x (8 / CPT) threads over the same
// 32 x 8 cells (thread row r owns cell rows r, r + 8/CPT, ...); with two,
// the per-bin work that does not depend on the cell (waits, barrier,
// direction table, loop control) is shared by both cells and the two
// cells' independent arithmetic interleaves.
template <class R, bool ROLLER, int CPT>
__device__ __forceinline__ void b_wave_tma(const Dev<R>& S, const Konst<R>& K, const WaveMaps& M, const int bix,
                                           const int biy) {
    constexpr int NTH = 256 / CPT, RPT = WT_Y / CPT;   // threads, thread rows
    constexpr bool PACKED = ROLLER && std::is_same<R, float>::value;   // (ee, rr) pairs in f32x2 instructions
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(8) unsigned long long mbar[TM_NB];
    Clock* clk = S.clk;
    if (wave_off(clk)) return;
    const int nx = K.nx, ny = K.ny, nt = K.nt, C = S.C;
    const int tid = threadIdx.x + threadIdx.y * WT_X;
    const unsigned base = (su32(smem_raw) + 127u) & ~127u;
    R* tE = reinterpret_cast<R*>(smem_raw + (base - su32(smem_raw)));   // [TM_NB][TM_N] plane tiles of ee
    R* tR = tE + TM_NB * TM_N;                                          // [TM_NB][TM_N] plane tiles of rr
    R* sA = tR + TM_NB * TM_N;           // [nt][256] advected ee (energy units), then the new ee
    R* sR = sA + (size_t)nt * 256;       // [nt][256] advected rr, then the new rr
    Dir4<R>* sMom = reinterpret_cast<Dir4<R>*>(sR + (size_t)nt * 256);
    Dir2<R>* sCS2 = reinterpret_cast<Dir2<R>*>(sMom + nt);
    if (tid < nt) {
        const R c = K.cxsth[tid], sn = K.sxnth[tid];
        sCS2[tid] = Dir2<R>{c, sn};
        sMom[tid] = Dir4<R>{c * c, sn * sn, sn * c, K.theta[tid]};
    }
    const int bx0 = bix * WT_X, by0 = 1 + biy * WT_Y;
    const int par = clk->par;
    const CUtensorMap* mE = &M.ld_e[par ^ 1];
    const CUtensorMap* mR = &M.ld_r[par ^ 1];
    const R* rro = S.rr[par ^ 1];
    const R dtf = (R)clk->dt;
    const R taper = (R)cmin((double)(R)clk->totaltime / 100.0, 1.0);
    const R dth = K.dtheta;
    const R rdth = (R)1 / dth;
    const R rdx = (R)1 / K.dx;
    const R sg = (R)clk->sigm;
    const R cmax_ = (R)(0.25f * sg), cmin_ = (R)(-0.25f * sg);   // propagtheta's clamp of ctheta
    const R kxy = dtf * rdx, kth = dtf * rdth;
    constexpr unsigned TBYTES = (ROLLER ? 2u : 1u) * TM_N * sizeof(R);
    if (tid == 0) {
        for (int b = 0; b < TM_NB; b++) tm_mbar_init(su32(&mbar[b]));
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        tm_fence_async();
    }
    __syncthreads();   // barriers initialised, theta tables written
    int issued = 0;             // planes issued so far (elected thread)
    auto issue = [&](int p) {   // elected thread: plane p into buffer p % 4
        issued = p + 1;
        const int b = p & (TM_NB - 1);
        const unsigned mb = su32(&mbar[b]);
        tm_expect(mb, TBYTES);
        tm_load3(su32(tE + b * TM_N), mE, bx0 - 4, by0 - 2, p, mb);
        if (ROLLER) tm_load3(su32(tR + b * TM_N), mR, bx0 - 4, by0 - 2, p, mb);
    };
    if (tid == 0)
        for (int p = 0; p < nt && p < TM_NB; p++) issue(p);
    auto wait_plane = [&](int p) { return tm_wait(su32(&mbar[p & (TM_NB - 1)]), (unsigned)(p >> 2) & 1u); };
    // blocks whose box reaches outside the grid or over the offshore column
    const bool edge = bx0 == 0 || bx0 + 35 > nx - 1 || by0 - 2 < 0 || by0 + 9 > ny - 1;
    // the clamped values of the box's out-of-grid cells, and St * taper on
    // column 0 (ee only): every rewritten cell reads an in-grid cell of
    // column >= 1 of the same box, which no thread rewrites
    auto fixup = [&](int p) {
        R* dE = tE + (p & (TM_NB - 1)) * TM_N;
        R* dR = tR + (p & (TM_NB - 1)) * TM_N;
        for (int e = tid; e < TM_N; e += NTH) {
            const int gx = bx0 - 4 + e % TM_X, gy = by0 - 2 + e / TM_X;
            const int cx = min(max(gx, 0), nx - 1), cy = min(max(gy, 0), ny - 1);
            const bool in = cx == gx && cy == gy;
            const int src = (cx - (bx0 - 4)) + (cy - (by0 - 2)) * TM_X;
            if (!(in && gx != 0)) dE[e] = cx == 0 ? DM<R>::fmax(S.St[cy + p * ny] * taper, (R)0) : dE[src];
            if (ROLLER && !in) dR[e] = dR[src];
        }
        tm_fence_async();   // these writes before the buffer's next box copy
    };
    auto cth = [&](const WCell<R>& w, R cx, R sx) -> R {
        const R ctht = DM<R>::fma(w.cthP, sx, w.cthQ * cx);
        return cmin(cmax(ctht, cmin_), cmax_);
    };
    WCell<R> cl[CPT];
#pragma unroll
    for (int c = 0; c < CPT; c++) {
        WCell<R>& w = cl[c];
        w = WCell<R>{};
        const int ty = threadIdx.y + c * RPT;
        w.ix = bx0 + threadIdx.x;
        w.iy = by0 + ty;
        w.cid = threadIdx.x + ty * WT_X;
        w.ctile = (ty + 2) * TM_X + (threadIdx.x + 4);
        w.active = w.ix < nx && w.iy <= ny - 2;
        w.i = 0;
        if (w.active) {
            const int ix = w.ix, iy = w.iy;
            const int i = ix + iy * nx;
            w.i = i;
            const int xm = mm(ix), xp = pp(ix, nx);
            const int ym = mm(iy), yp = pp(iy, ny);
            w.hh = ld(S.f[HH] + i);
            const CthCoef<R> cc = cth_coef(S, K, ix, iy, sg);
            const R* cgp = S.f[CG];
            const R* cp = S.f[CC_];
            w.cgi = ld(cgp + i); w.cci = ld(cp + i);
            // face speeds times dt / dx: without wave-current interaction the
            // current terms of the face speed are exactly zero
            const R h = (R)0.5f * kxy;
            w.axp = h * (w.cgi + ld(cgp + xp + iy * nx)); w.axm = h * (w.cgi + ld(cgp + xm + iy * nx));
            w.ayp = h * (w.cgi + ld(cgp + ix + yp * nx)); w.aym = h * (w.cgi + ld(cgp + ix + ym * nx));
            w.rxp = h * (w.cci + ld(cp + xp + iy * nx)); w.rxm = h * (w.cci + ld(cp + xm + iy * nx));
            w.ryp = h * (w.cci + ld(cp + ix + yp * nx)); w.rym = h * (w.cci + ld(cp + ix + ym * nx));
            if constexpr (PACKED) {
                w.kx = make_float2(w.axp, w.rxp); w.kxn = make_float2(-w.axm, -w.rxm);
                w.ky = make_float2(w.ayp, w.ryp); w.kyn = make_float2(-w.aym, -w.rym);
                w.ften = make_float2(0.f, 0.f);
            }
            w.cthP = cc.s * cc.dhdx; w.cthQ = -(cc.s * cc.dhdy);
            w.c0 = cth(w, sCS2[0].c, sCS2[0].s);
            const int t1 = nt > 1 ? 1 : 0;
            w.cpp = cth(w, sCS2[t1].c, sCS2[t1].s);
        }
    }
    bool ok = wait_plane(0) && (nt < 2 || wait_plane(1));
    if (edge) {
        fixup(0);
        if (nt > 1) fixup(1);
    }
    bool failed = false;
#pragma unroll 1
    for (int t = 0; t < nt; t++) {
        const int b = t & (TM_NB - 1);
        if (t + 2 < nt) {
            ok = ok && wait_plane(t + 2);
            if (edge) fixup(t + 2);
        }
        if (__syncthreads_or(!ok)) { failed = true; break; }   // fixups visible; plane t-1 read by all
        if (tid == 0 && t >= 1 && t + 3 < nt) issue(t + 3);    // into plane t-1's buffer
        const Dir2<R> d = sCS2[t];
        const R ct = d.c, st = d.s;
        const bool last = t == nt - 1;
        const int b2 = (t + 2 < nt ? t + 2 : nt - 1) & (TM_NB - 1);
        const Dir2<R> d2 = sCS2[t + 2 < nt ? t + 2 : nt - 1];
#pragma unroll
        for (int c = 0; c < CPT; c++) {
            WCell<R>& w = cl[c];
            if (!w.active) continue;
            const R* qE = tE + b * TM_N + w.ctile;
            const R* qR = tR + b * TM_N + w.ctile;
            if constexpr (PACKED) {
                if (t == 0) {
                    const int b1 = (nt > 1 ? 1 : 0);
                    w.p2 = make_float2(qE[0], qR[0]);
                    w.p1 = w.p2;
                    w.p3 = make_float2(tE[b1 * TM_N + w.ctile], tR[b1 * TM_N + w.ctile]);
                }
                w.p4 = make_float2(tE[b2 * TM_N + w.ctile], tR[b2 * TM_N + w.ctile]);
                w.cabs = DM<R>::fmax(w.cabs, DM<R>::fabs(w.c0));
                float2 fx, fy;
                auto xy2 = [&](auto px, auto py) {
                    constexpr bool PX = decltype(px)::value, PY = decltype(py)::value;
                    fx = flux2k2<PX>(qE, qR, 1, w.p2, w.kx, w.kxn);
                    fy = flux2k2<PY>(qE, qR, TM_X, w.p2, w.ky, w.kyn);
                };
                if (ct > (R)0) {
                    if (st > (R)0) xy2(std::true_type{}, std::true_type{}); else xy2(std::true_type{}, std::false_type{});
                } else {
                    if (st > (R)0) xy2(std::false_type{}, std::true_type{}); else xy2(std::false_type{}, std::false_type{});
                }
                const float2 fup = last ? make_float2(0.f, 0.f) : theta_face2(w.p1, w.p2, w.p3, w.p4, w.c0, w.cpp);
                const float2 ft = __fadd2_rn(fup, w.ften);
                w.ften = __fmul2_rn(fup, make_float2(-1.f, -1.f));
                const float2 A2 = __fadd2_rn(
                    w.p2, __ffma2_rn(make_float2(-ct, -ct), fx,
                                     __ffma2_rn(make_float2(-st, -st), fy, __fmul2_rn(ft, make_float2(-kth, -kth)))));
                sA[t * 256 + w.cid] = A2.x;
                sR[t * 256 + w.cid] = A2.y;
                w.Etmp = w.Etmp + DM<R>::fmax(A2.x, (R)0);
                w.p1 = w.p2; w.p2 = w.p3; w.p3 = w.p4;
                w.c0 = w.cpp; w.cpp = cth(w, d2.c, d2.s);
                continue;
            }
            if (t == 0) {
                const int b1 = (nt > 1 ? 1 : 0);
                w.we2 = qE[0]; w.we1 = w.we2; w.we3 = tE[b1 * TM_N + w.ctile];
                if (ROLLER) { w.wr2 = qR[0]; w.wr1 = w.wr2; w.wr3 = tR[b1 * TM_N + w.ctile]; }
            }
            w.we4 = tE[b2 * TM_N + w.ctile];
            if (ROLLER) w.wr4 = tR[b2 * TM_N + w.ctile];
            w.cabs = DM<R>::fmax(w.cabs, DM<R>::fabs(w.c0));
            // x and y fluxes with the upwind side of the bin (the sign of
            // cos and sin is the same for every cell of the bin)
            R fx, fy, rx = 0, ry = 0;
            auto xy = [&](auto px, auto py) {
                constexpr bool PX = decltype(px)::value, PY = decltype(py)::value;
                fx = flux2k<R, PX>(qE, 1, w.we2, w.axp, w.axm);
                fy = flux2k<R, PY>(qE, TM_X, w.we2, w.ayp, w.aym);
                if (ROLLER) {
                    rx = flux2k<R, PX>(qR, 1, w.wr2, w.rxp, w.rxm);
                    ry = flux2k<R, PY>(qR, TM_X, w.wr2, w.ryp, w.rym);
                }
            };
            using T_ = std::true_type;
            using F_ = std::false_type;
            if (ct > (R)0) {
                if (st > (R)0) xy(T_{}, T_{}); else xy(T_{}, F_{});
            } else {
                if (st > (R)0) xy(F_{}, T_{}); else xy(F_{}, F_{});
            }
            R fup = last ? (R)0 : theta_face(w.we1, w.we2, w.we3, w.we4, w.c0, w.cpp);
            R ft = fup - w.fte;
            w.fte = fup;
            R A = euler_k(w.we2, ct, st, fx, fy, ft, kth);
            R Ar;
            if (!ROLLER) Ar = ld(rro + w.i + (size_t)t * C);   // without the roller pass rr is carried unchanged
            if (ROLLER) {
                R rup = last ? (R)0 : theta_face(w.wr1, w.wr2, w.wr3, w.wr4, w.c0, w.cpp);
                R rt = rup - w.ftr;
                w.ftr = rup;
                Ar = euler_k(w.wr2, ct, st, rx, ry, rt, kth);
            }
            sA[t * 256 + w.cid] = A;
            sR[t * 256 + w.cid] = Ar;
            w.Etmp = w.Etmp + DM<R>::fmax(A, (R)0);
            w.we1 = w.we2; w.we2 = w.we3; w.we3 = w.we4;
            w.wr1 = w.wr2; w.wr2 = w.wr3; w.wr3 = w.wr4;
            w.c0 = w.cpp; w.cpp = cth(w, d2.c, d2.s);
        }
    }
    if (failed) {   // a copy never completed: record, halt, let the copies in flight land (bounded), leave
        if (tid == 0) {
            atomicExch(&clk->status, XBG_ERR_TIMEOUT);
            atomicExch(&clk->halt, 1);
            for (int p = issued - TM_NB < 0 ? 0 : issued - TM_NB; p < issued; p++)
                wait_plane(p);   // the last plane issued into each buffer
        }
        __syncthreads();
        return;
    }
    R dtw = (R)3.0e38f;
    R* een = S.ee[par];
    R* rrn = S.rr[par];
    const R Trep = (R)clk->Trep;
    const R rho = K.rho, g = K.g;
    const R twogb = (R)2.0f * g * K.beta;
#pragma unroll
    for (int c = 0; c < CPT; c++) {
        const WCell<R>& w = cl[c];
        if (!w.active) continue;
        const int i = w.i, cid = w.cid;
        dtw = DM<R>::fmin(dtw, DM<R>::fmin(K.cfl * dth / w.cabs, (R)9999999.9f));   // WAVEDT (Wave_kernel.cu:232-249)
        R ridiv, Dv, Dq;
        wave_breaking(K, w.Etmp, w.hh, ld(S.f[WK] + i), ld(S.f[FWM] + i), Trep, ridiv, Dv, Dq);
        const R cc_i = w.cci;
        const R rcoef = twogb / cc_i;
        const bool wet = w.hh > K.eps;
        // the lateral rows 0 and ny-1 first, while sA / sR still hold the
        // advected bins; the source cell's new ee is formed as below
        auto fin = [&](int t) {
            R dd;
            return wet ? diss_ee(sA[t * 256 + cid], ridiv, Dq, dtf, dd) : (R)0;
        };
        if (w.iy == 1)
            dtw = DM<R>::fmin(dtw, wave_edge_cell<R, ROLLER, false>(S, K, w.ix, 0, sA + (cid - tid), sR + (cid - tid),
                                                                   sCS2, sMom, w.Etmp, sg, dtf, Trep, rro, een, rrn,
                                                                   fin));
        if (w.iy == ny - 2)
            dtw = DM<R>::fmin(dtw, wave_edge_cell<R, ROLLER, false>(S, K, w.ix, ny - 1, sA + (cid - tid),
                                                                   sR + (cid - tid), sCS2, sMom, w.Etmp, sg, dtf,
                                                                   Trep, rro, een, rrn, fin));
        R RR = (R)0.0f, drr = (R)0.0f, sume = (R)0, sumethet = (R)0;
        R ec = 0, es = 0, ecs = 0, rc = 0, rs = 0, rcs = 0;
        R* pA = sA + cid;
        R* pR = sR + cid;
        if (wet && PACKED) {   // the (ee, rr) sums in f32x2 instructions, rounding as the scalar loop
            float2 sr = make_float2(0.f, 0.f), cc2 = sr, ss2 = sr, cs2 = sr;
#pragma unroll 2
            for (int t = 0; t < nt; t++) {
                float dd;
                const float eet = diss_ee((float)pA[t * 256], (float)ridiv, (float)Dq, (float)dtf, dd);
                float rrt = pR[t * 256];
                const float rrd = __fmul_rn(rrt, (float)rcoef);
                rrt = diss_rr(rrt, rrd, dd, (float)dtf);
                drr = drr + rrd;
                pA[t * 256] = eet;
                pR[t * 256] = rrt;
                const Dir4<R> m = sMom[t];
                const float2 er = make_float2(eet, rrt);
                sr = __fadd2_rn(sr, er);
                sumethet = DM<R>::fma(eet, m.th, sumethet);
                cc2 = __ffma2_rn(make_float2(m.c2, m.c2), er, cc2);
                ss2 = __ffma2_rn(make_float2(m.s2, m.s2), er, ss2);
                cs2 = __ffma2_rn(make_float2(m.cs, m.cs), er, cs2);
            }
            sume = sr.x; RR = sr.y;
            ec = cc2.x; rc = cc2.y; es = ss2.x; rs = ss2.y; ecs = cs2.x; rcs = cs2.y;
        } else if (wet) {
#pragma unroll 2
            for (int t = 0; t < nt; t++) {
                R dd;
                const R eet = diss_ee(pA[t * 256], ridiv, Dq, dtf, dd);
                R rrt = pR[t * 256];
                const R rrd = DM<R>::mul(rrt, rcoef);
                rrt = diss_rr(rrt, rrd, dd, dtf);
                drr = drr + rrd;
                RR = RR + rrt;
                pA[t * 256] = eet;
                pR[t * 256] = rrt;
                const Dir4<R> m = sMom[t];
                sume = sume + eet;
                sumethet = DM<R>::fma(eet, m.th, sumethet);
                ec = DM<R>::fma(m.c2, eet, ec);
                es = DM<R>::fma(m.s2, eet, es);
                ecs = DM<R>::fma(m.cs, eet, ecs);
                rc = DM<R>::fma(m.c2, rrt, rc);
                rs = DM<R>::fma(m.s2, rrt, rs);
                rcs = DM<R>::fma(m.cs, rrt, rcs);
            }
        } else {
            for (int t = 0; t < nt; t++) {
                pA[t * 256] = (R)0;
                pR[t * 256] = (R)0;
            }
        }
        const R sum2 = sume;
        sume = DM<R>::fmax(sume, (R)0.00001f);
        S.f[THM][i] = sumethet / sume;
        S.f[E][i] = sume * dth;
        S.f[H][i] = DM<R>::sqrt(sume * dth / (rho * g / (R)8));
        S.f[D][i] = Dv;
        S.f[ROL][i] = RR * dth;
        S.f[DR][i] = drr * dth;
        const R n = w.cgi / cc_i;
        radstress(S.tmp[T_SXX], S.tmp[T_SXY], S.tmp[T_SYY], i, n, sum2, ec, es, ecs, rc, rs, rcs, dth);
    }
    // the block's new bins of rows 1..ny-2 in two box stores
    tm_fence_async();
    __syncthreads();
    if (tid == 0) {
        tm_store3(&M.st_e[par], bx0, by0, 0, su32(sA));
        tm_store3(&M.st_r[par], bx0, by0, 0, su32(sR));
        asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
    }
    block_min_store<R>(dtw, S.part_wave + bix + biy * ((K.nx + 31) / 32));
    if (tid == 0) asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");   // shared memory read out
}
// FP32: 64 registers, four blocks (32 warps) per SM, which hides the pass's
// dependent-arithmetic latency better than three (-15 % at 2048 x 1024);
// FP64 (the error-oracle build) keeps room for its wider registers.
template <class R, bool ROLLER, int CPT>
__global__ void __launch_bounds__(256 / CPT, sizeof(R) == 4 ? 4 : 2)
    k_wave_tma(Dev<R> S, Konst<R> K, const __grid_constant__ WaveMaps M) {
    b_wave_tma<R, ROLLER, CPT>(S, K, M, blockIdx.x, blockIdx.y);
}
// every scenario of a batch: its tensor maps from a device array (written
// by the host before the first launch), one per scenario
template <class R, bool ROLLER, int CPT>
__global__ void __launch_bounds__(256 / CPT, sizeof(R) == 4 ? 4 : 2)
    kb_wave_tma(BatchTab<R> T, const WaveMaps* __restrict__ maps, const int2* items, int n) {
    batch_items<R>(T, items, n, [&](const Dev<R>& S, const Konst<R>& K, const BatchAux& A, int bx, int by) {
        b_wave_tma<R, ROLLER, CPT>(S, K, maps[A.scen], bx, by);
    });
}

// Tensor maps of the TMA rows pass: ee and rr of both plane sets as 3-D
// arrays [nt][ny][nx]; loads in 40 x 12 x 1 boxes, stores in 32 x 8 x nt
// boxes over rows 0..ny-2 (the map ends before row ny-1).  Encoded with the
// driver's cuTensorMapEncodeTiled (fetched through the runtime).
template <class R>
int wave_maps_make(const Dev<R>& S, const Konst<R>& K, WaveMaps* M) {
    if (K.nx % 4 != 0 || K.nt > 256) return 1;
    static PFN_cuTensorMapEncodeTiled_v12000 enc = nullptr;
    if (!enc) {
        cudaDriverEntryPointQueryResult q;
        void* fn = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return 1;
        enc = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    const CUtensorMapDataType dt = sizeof(R) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    const cuuint64_t es = sizeof(R);
    const cuuint32_t one[3] = {1, 1, 1};
    auto make = [&](CUtensorMap* m, const R* base, int rows, cuuint32_t bx, cuuint32_t by, cuuint32_t bz) {
        const cuuint64_t dims[3] = {(cuuint64_t)K.nx, (cuuint64_t)rows, (cuuint64_t)K.nt};
        const cuuint64_t strides[2] = {(cuuint64_t)K.nx * es, (cuuint64_t)K.nx * K.ny * es};
        const cuuint32_t box[3] = {bx, by, bz};
        return enc(m, dt, 3, (void*)base, dims, strides, box, one, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    };
    for (int k = 0; k < 2; k++) {
        if (make(&M->ld_e[k], S.ee[k], K.ny, TM_X, TM_Y, 1) != CUDA_SUCCESS ||
            make(&M->ld_r[k], S.rr[k], K.ny, TM_X, TM_Y, 1) != CUDA_SUCCESS ||
            make(&M->st_e[k], S.ee[k], K.ny - 1, WT_X, WT_Y, (cuuint32_t)K.nt) != CUDA_SUCCESS ||
            make(&M->st_r[k], S.rr[k], K.ny - 1, WT_X, WT_Y, (cuuint32_t)K.nt) != CUDA_SUCCESS)
            return 1;
    }
    return 0;
}

// wavforce (wave_CPU.cpp:1164-1238) from the radiation stresses around a
// cell (r: the right neighbour, t: the upper, b: the lower, l: the left, tr,
// br, tl: the diagonals), before the boundary copies
template <class R>
__device__ __forceinline__ void force_of(R dxf, R Sxxi, R Sxxr, R Sxyt, R Sxytr, R Sxyb, R Sxybr, R Syyi, R Syyt,
                                         R Sxyr, R Sxyl, R Sxytl, R& Fx, R& Fy) {
    Fx = (R)-1 * (Sxxr - Sxxi) / dxf - (R)0.5f * (Sxyt + Sxytr - Sxyb - Sxybr) / ((R)2.0f * dxf);
    Fy = (R)-1 * (Syyt - Syyi) / dxf - (R)0.5f * (Sxyr + Sxytr - Sxyl - Sxytl) / ((R)2.0f * dxf);
}
// ... at cell (ix, iy)
template <class R>
__device__ __forceinline__ void force_raw(const Dev<R>& S, const Konst<R>& K, int ix, int iy, R& Fx, R& Fy) {
    const int nx = K.nx, ny = K.ny;
    const R* Sxx = S.tmp[T_SXX]; const R* Sxy = S.tmp[T_SXY]; const R* Syy = S.tmp[T_SYY];
    int xm = mm(ix), xp = pp(ix, nx), ym = mm(iy), yp = pp(iy, ny);
    int i = ix + iy * nx;
    force_of(K.dx, ld(Sxx + i), ld(Sxx + xp + iy * nx), ld(Sxy + ix + yp * nx), ld(Sxy + xp + yp * nx),
             ld(Sxy + ix + ym * nx), ld(Sxy + xp + ym * nx), ld(Syy + i), ld(Syy + ix + yp * nx), ld(Sxy + xp + iy * nx),
             ld(Sxy + xm + iy * nx), ld(Sxy + xm + yp * nx), Fx, Fy);
}

// breakerdelayCPU (wave_CPU.cpp:1333-1368) from a cell's H, k, depth, c,
// roller energy and E
template <class R>
__device__ __forceinline__ void breaker_of(const Konst<R>& K, R Trep, R Hi, R ki, R hh, R c, R Rl, R Ei, R& urms,
                                           R& ust) {
    R hmin = (R)0.2;
    R g = K.g, rho = K.rho;
    R hhi = cmax(hh, hmin);
    R ci = cmax(c, DM<R>::sqrt(hmin * g));
    R uorb = (R)(XBG_PI * (double)Hi / (double)Trep / (double)DM<R>::sinh(cmin(cmax(ki, (R)0.01f) * hhi, (R)10.0f)));
    urms = uorb / (DM<R>::sqrt((R)2.0f));
    R ustw = Ei / ci / rho / hhi;
    R ustr = (R)2.0f * Rl / ci / rho / hhi;
    ust = ustw + ustr;
}
// ... at cell j
template <class R>
__device__ __forceinline__ void breaker_raw(const Dev<R>& S, const Konst<R>& K, int j, R Trep, R& urms, R& ust) {
    breaker_of(K, Trep, ld(S.f[H] + j), ld(S.f[WK] + j), ld(S.f[HH] + j), ld(S.f[CC_] + j), ld(S.f[ROL] + j),
               ld(S.f[E] + j), urms, ust);
}

template <class R>
__device__ __forceinline__ void b_wave_force(const Dev<R>& S, const Konst<R>& K, const int bix, const int biy) {
    const Clock* clk = S.clk;
    if (wave_off(clk)) return;
    const int nx = K.nx, ny = K.ny;
    int ix = bix * blockDim.x + threadIdx.x;
    int iy = biy * blockDim.y + threadIdx.y;
    if (ix >= nx || iy >= ny) return;
    int i = ix + iy * nx;
    R Trep = (R)clk->Trep;
    R w = ld(S.f[HH] + i) > K.eps ? (R)1.0f : (R)0.0f;
    // twodimbndnoixCPU(Fx): rows only; twodimbndCPU(Fy, ust): rows then ix = 0
    int sy = iy;
    if (iy == 0) sy = pp(0, ny);
    if (iy == ny - 1) sy = mm(ny - 1);
    int fx_src_x = ix, fx_src_y = sy;
    int fy_src_x = (ix == 0) ? pp(0, nx) : ix;
    int fy_src_y = (ix == 0) ? iy : sy;
    bool rowb = (iy == 0 || iy == ny - 1);
    bool anyb = rowb || ix == 0;
    R Fx, Fy, tmp;
    force_raw(S, K, fx_src_x, fx_src_y, Fx, tmp);
    if (rowb) Fx = Fx * w;
    force_raw(S, K, fy_src_x, fy_src_y, tmp, Fy);
    if (anyb) Fy = Fy * w;
    S.f[FX][i] = Fx;
    S.f[FY][i] = Fy;
    R urms, ust, u2;
    breaker_raw(S, K, i, Trep, urms, ust);
    if (anyb) {
        breaker_raw(S, K, fy_src_x + fy_src_y * nx, Trep, u2, ust);
        ust = ust * w;
    }
    S.f[URMS][i] = urms;
    S.f[UST][i] = ust;
}
XBG_KERNELS(wave_force)

// ---------------------------------------------------------------- launchers
template <class R>
int wave_parts(const Konst<R>& K) {
    return ((K.nx + 31) / 32) * ((K.ny - 2 + 7) / 8);
}

// join: an event of a concurrent branch (the boundary kernels) that the
// rows pass waits for after the dispersion kernel; null when sequential.
// maps: the tensor maps of the TMA rows pass, or null for the thread-copied
// tiles (b_wave_fast); the TMA pass has no wave-current interaction variant.
template <class R>
int launch_wave(const Dev<R>& S, const Konst<R>& K, cudaStream_t st, Prof* pf, cudaEvent_t join,
                const WaveMaps* maps, int cpt, bool wide) {
    int n = 0;
    k_disp<R><<<(S.C + 255) / 256, 256, 0, st>>>(S, K); n++;
    PMARK(pf, "k_disp");
    if (join) cudaStreamWaitEvent(st, join, 0);
    {
        dim3 b(32, 8), g((K.nx + 31) / 32, (K.ny - 2 + 7) / 8);
        if (maps && K.wci == (R)0) {
            const size_t smem = wave_tma_smem<R>(K.nt);
            if (cpt == 2) {
                const dim3 b2(32, 4);
                if (K.roller == 1) k_wave_tma<R, true, 2><<<g, b2, smem, st>>>(S, K, *maps);
                else k_wave_tma<R, false, 2><<<g, b2, smem, st>>>(S, K, *maps);
            } else {
                if (K.roller == 1) k_wave_tma<R, true, 1><<<g, b, smem, st>>>(S, K, *maps);
                else k_wave_tma<R, false, 1><<<g, b, smem, st>>>(S, K, *maps);
            }
            n++;
            PMARK(pf, "k_wave_tma");
        } else {
            launch_wave_fast(S, K, g, b, wave_fast_smem<R>(K.nt), st); n++;
            PMARK(pf, "k_wave_fast");
        }
    }
    // the force pass is pointwise: 32 x 8 or (wide) 64 x 4 blocks (a row-segment
    // form measured slower: 37.0 against 32.8 us at 2048 x 1024, 94 registers)
    if (wide) k_wave_force<R><<<dim3((K.nx + 63) / 64, (K.ny + 3) / 4), dim3(64, 4), 0, st>>>(S, K);
    else k_wave_force<R><<<dim3((K.nx + 31) / 32, (K.ny + 7) / 8), dim3(32, 8), 0, st>>>(S, K);
    n++;
    PMARK(pf, "k_wave_force");
    return n;
}

// the wave kernels over every scenario of a batch (one ntheta and roller
// setting for the whole batch)
// maps: the scenarios' tensor maps (device array) for the TMA rows pass, or
// null for the thread-copied tiles
template <class R>
int launch_wave_batch(const BatchTab<R>& T, const BatchLaunch& L, int nt, int roller, int wci, cudaStream_t st,
                      Prof* pf, cudaEvent_t join, const WaveMaps* maps, int cpt, bool wide) {
    kb_disp<R><<<L.grid[BS_LIN], 256, 0, st>>>(T, L.items[BS_LIN], L.n[BS_LIN]);
    PMARK(pf, "k_disp");
    if (join) cudaStreamWaitEvent(st, join, 0);
    if (maps && !wci) {
        const int g = L.grid[BS_WROWS], n = L.n[BS_WROWS];
        const int2* it = L.items[BS_WROWS];
        const size_t smem = wave_tma_smem<R>(nt);
        if (cpt == 2) {
            if (roller == 1) kb_wave_tma<R, true, 2><<<g, dim3(32, 4), smem, st>>>(T, maps, it, n);
            else kb_wave_tma<R, false, 2><<<g, dim3(32, 4), smem, st>>>(T, maps, it, n);
        } else {
            if (roller == 1) kb_wave_tma<R, true, 1><<<g, dim3(32, 8), smem, st>>>(T, maps, it, n);
            else kb_wave_tma<R, false, 1><<<g, dim3(32, 8), smem, st>>>(T, maps, it, n);
        }
        PMARK(pf, "k_wave_tma");
    } else {
        launch_wave_fast_batch(T, L, roller, wci, wave_fast_smem<R>(nt), st);
        PMARK(pf, "k_wave_fast");
    }
    const int sf = wide ? BS_WIDE : BS_TILE;
    kb_wave_force<R><<<L.grid[sf], wide ? dim3(64, 4) : dim3(32, 8), 0, st>>>(T, L.items[sf], L.n[sf]);
    PMARK(pf, "k_wave_force");
    return 3;
}
template int launch_wave_batch<float>(const BatchTab<float>&, const BatchLaunch&, int, int, int, cudaStream_t, Prof*,
                                      cudaEvent_t, const WaveMaps*, int, bool);
template int launch_wave_batch<double>(const BatchTab<double>&, const BatchLaunch&, int, int, int, cudaStream_t, Prof*,
                                       cudaEvent_t, const WaveMaps*, int, bool);

// One-time kernel attributes (dynamic shared memory above 48 KB for wide
// theta sets in FP64).
template <class R>
int wave_prepare(const Konst<R>& K) {
    const int smem = (int)wave_fast_smem<R>(K.nt);
    const int smem_tma = (int)wave_tma_smem<R>(K.nt);
    const cudaFuncAttribute a = cudaFuncAttributeMaxDynamicSharedMemorySize;
    if (cudaFuncSetAttribute(k_wave_tma<R, true, 1>, a, smem_tma) != cudaSuccess ||
        cudaFuncSetAttribute(k_wave_tma<R, false, 1>, a, smem_tma) != cudaSuccess ||
        cudaFuncSetAttribute(k_wave_tma<R, true, 2>, a, smem_tma) != cudaSuccess ||
        cudaFuncSetAttribute(k_wave_tma<R, false, 2>, a, smem_tma) != cudaSuccess ||
        cudaFuncSetAttribute(kb_wave_tma<R, true, 1>, a, smem_tma) != cudaSuccess ||
        cudaFuncSetAttribute(kb_wave_tma<R, false, 1>, a, smem_tma) != cudaSuccess ||
        cudaFuncSetAttribute(kb_wave_tma<R, true, 2>, a, smem_tma) != cudaSuccess ||
        cudaFuncSetAttribute(kb_wave_tma<R, false, 2>, a, smem_tma) != cudaSuccess)
        return 1;
    cudaError_t e[8] = {
        cudaFuncSetAttribute(k_wave_fast<R, true, true>, a, smem), cudaFuncSetAttribute(k_wave_fast<R, true, false>, a, smem),
        cudaFuncSetAttribute(k_wave_fast<R, false, true>, a, smem), cudaFuncSetAttribute(k_wave_fast<R, false, false>, a, smem),
        cudaFuncSetAttribute(kb_wave_fast<R, true, true>, a, smem), cudaFuncSetAttribute(kb_wave_fast<R, true, false>, a, smem),
        cudaFuncSetAttribute(kb_wave_fast<R, false, true>, a, smem), cudaFuncSetAttribute(kb_wave_fast<R, false, false>, a, smem)};
    for (auto x : e)
        if (x != cudaSuccess) return 1;
    return 0;
}
template int wave_prepare<float>(const Konst<float>&);
template int wave_prepare<double>(const Konst<double>&);

template int launch_wave<float>(const Dev<float>&, const Konst<float>&, cudaStream_t, Prof*, cudaEvent_t,
                                const WaveMaps*, int, bool);
template int launch_wave<double>(const Dev<double>&, const Konst<double>&, cudaStream_t, Prof*, cudaEvent_t,
                                 const WaveMaps*, int, bool);
template int wave_maps_make<float>(const Dev<float>&, const Konst<float>&, WaveMaps*);
template int wave_maps_make<double>(const Dev<double>&, const Konst<double>&, WaveMaps*);
template int wave_parts<float>(const Konst<float>&);
template int wave_parts<double>(const Konst<double>&);

}  // namespace xbg
