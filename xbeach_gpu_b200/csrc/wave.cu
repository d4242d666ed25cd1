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
//                one bin ahead (three buffers, one barrier per bin); ctheta
//                (propagtheta) is evaluated on the fly from per-cell slopes;
//                the theta-face flux is computed once and carried to the
//                next bin.  Emits the per-block WAVEDT minimum.
//   k_wave_edge  rows 0 and ny-1, whose ee/rr are copies of rows 1 / ny-2
//                (rollerlatbnd, wave_CPU.cpp:830-870) between the passes.
//   k_wave_force wavforce + twodimbnd(noix) + breakerdelay + twodimbnd(ust).
#include "xbg_common.cuh"

namespace xbg {

// ---------------------------------------------------------------- helpers
// (R)(1.5*(double)a - 0.5*(double)b): one rounding of the exact value, as the
// double literals of xadvecupwind2CPU give (wave_CPU.cpp:426-453).
template <class R> __device__ __forceinline__ R up2d(R a, R b) {
    return DM<R>::fma((R)1.5, a, (R)-0.5 * b);
}
// 1.5f*a - 0.5f*b with two roundings (thetaadvecuw2hoCPU, wave_CPU.cpp:747-790).
template <class R> __device__ __forceinline__ R up2f(R a, R b) {
    R x = (R)1.5f * a;
    R y = (R)0.5f * b;
    return x - y;
}

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
    if (halted(S.clk)) return;
    int i = bix * blockDim.x + threadIdx.x;
    if (i >= S.C) return;
    R sg = (R)S.clk->sigm;
    R k_, c_, cg_;
    disp_cell(K, sg, ld(S.f[HH] + i), k_, c_, cg_);
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

// x/y second-order upwind fluxes of one theta plane, xadvecupwind2CPU /
// yadvecupwind2CPU (wave_CPU.cpp:367-560).  q(-2..2) are the plane's values at
// the clamped neighbours mminus2, mminus, i, pplus, pplus2.
template <class R>
__device__ __forceinline__ R adv2(R qm2, R qm, R qi, R qp, R qp2, R cf, R cfmin, R dxplus_i) {
    R arrin, arrmin;
    if (cf > (R)0.0f) {
        arrin = up2d(qi, qm);
        if (arrin < (R)0.0f) arrin = qi;
        arrin = arrin * cf;
    } else {
        arrin = up2d(qp, qp2);
        if (arrin < (R)0.0f) arrin = qp;
        arrin = arrin * cf;
    }
    if (cfmin > (R)0.0f) {
        arrmin = up2d(qm, qm2);
        if (arrmin < (R)0.0f) arrmin = qm;
        arrmin = arrmin * cfmin;
    } else {
        arrmin = up2d(qi, qp);
        if (arrmin < (R)0.0f) arrmin = qi;
        arrmin = arrmin * cfmin;
    }
    return (arrin - arrmin) * dxplus_i;
}

// Advected field of one cell: q_new[t] = q[t] - dt*(xadv + yadv + thetaadv).
// loadq(ix, iy, t) returns the (transformed) plane value at a grid point.
template <class R, int NMAX, class LoadQ>
__device__ __forceinline__ void advect_cell(const Dev<R>& S, const Konst<R>& K, int ix, int iy,
                                            const R* speed, const R* cthv, LoadQ loadq, R dtf,
                                            R* out) {
    const int nx = K.nx, ny = K.ny, nt = K.nt;
    int i = ix + iy * nx;
    int xm = mm(ix), xp = pp(ix, nx), xm2 = mm2(ix), xp2 = pp2(ix, nx);
    int ym = mm(iy), yp = pp(iy, ny), ym2 = mm2(iy), yp2 = pp2(iy, ny);
    R dxplus_i = (R)1.0f / K.dx;
    R wci = K.wci * cmin(ld(S.f[HH] + i) / K.hwci, (R)1.0f);
    R ccg = ld(speed + i);
    R ccgxmin = ld(speed + xm + iy * nx), ccgxmax = ld(speed + xp + iy * nx);
    R ccgymin = ld(speed + ix + ym * nx), ccgymax = ld(speed + ix + yp * nx);
    const R* uu = S.f[UU]; const R* vv = S.f[VV];
    R uui = ld(uu + i) * wci;
    R uuixmin = ld(uu + xm + iy * nx) * wci;
    R uuixmax = ld(uu + xp + iy * nx) * wci;
    R vvi = wci * ld(vv + i);
    R vviymin = wci * ld(vv + ix + ym * nx);
    R vviymax = wci * ld(vv + ix + yp * nx);
    R own[NMAX];
#pragma unroll
    for (int t = 0; t < NMAX; t++) own[t] = (t < nt) ? loadq(ix, iy, t) : (R)0;
    R dth = K.dtheta;
#pragma unroll
    for (int t = 0; t < NMAX; t++) {
        if (t < nt) {
            R ct = K.cxsth[t], st = K.sxnth[t];
            R cgx = (R)0.5f * (ccg * ct + uui + ccgxmax * ct + uuixmax);
            R cgxmin = (R)0.5f * (ccg * ct + uui + ccgxmin * ct + uuixmin);
            R xa = adv2(loadq(xm2, iy, t), loadq(xm, iy, t), own[t], loadq(xp, iy, t), loadq(xp2, iy, t),
                        cgx, cgxmin, dxplus_i);
            R cgy = (R)0.5f * (ccg * st + vvi + ccgymax * st + vviymax);
            R cgymin = (R)0.5f * (ccg * st + vvi + ccgymin * st + vviymin);
            R ya = adv2(loadq(ix, ym2, t), loadq(ix, ym, t), own[t], loadq(ix, yp, t), loadq(ix, yp2, t),
                        cgy, cgymin, dxplus_i);
            // thetaadvecuw2hoCPU (wave_CPU.cpp:706-806) with clamped bins
            R ta = (R)0.0f;
            if (nt > 1) {
                const int tm = t > 0 ? t - 1 : 0;
                const int tm2 = t > 1 ? t - 2 : 0;
                const int t1 = (t + 1 < NMAX) ? t + 1 : t;
                const int t2 = (t + 2 < NMAX) ? t + 2 : t1;
                R e_p = (t + 1 < nt) ? own[t1] : own[t];
                R e_p2 = (t + 2 < nt) ? own[t2] : e_p;
                R c_p = (t + 1 < nt) ? cthv[t1] : cthv[t];
                R cthetab = (R)0.5f * (cthv[t] + c_p);
                R eupw;
                if (cthetab > (R)0.0f) {
                    eupw = up2f(own[t], own[tm]);
                    if (eupw < (R)0.0f) eupw = own[t];
                } else {
                    eupw = up2f(e_p, e_p2);
                    if (eupw < (R)0.0f) eupw = e_p;
                }
                R arrint = cthetab * eupw;
                cthetab = (R)0.5f * (cthv[tm] + cthv[t]);
                if (cthetab > (R)0.0f) {
                    eupw = up2f(own[tm], own[tm2]);
                    if (eupw < (R)0.0f) eupw = own[tm];
                } else {
                    eupw = up2f(own[t], e_p);
                    if (eupw < (R)0.0f) eupw = own[t];
                }
                R arrmint = cthetab * eupw;
                ta = (arrint - arrmint) / dth;
                if (t == nt - 1) ta = ((R)0.0f - arrmint) / dth;
                if (t == 0) ta = (arrint - (R)0.0f) / dth;
            }
            out[t] = own[t] - dtf * (xa + ya + ta);
        } else {
            out[t] = (R)0;
        }
    }
}

// Per-cell chain after advection: energy, energint, roelvink|baldock and
// dissipation (wave_CPU.cpp:873-1092).  e (advected ee with the row copy
// applied) and r (rr before dissipation) are updated in place.
template <class R>
struct CellOut { R E, H, D, R_, DR; };

template <class R, int NMAX>
__device__ __forceinline__ CellOut<R> chain_cell(const Dev<R>& S, const Konst<R>& K, int i, R sg, R dtf,
                                                 R Trep, R* e, R* r) {
    const int nt = K.nt;
    R rho = K.rho, g = K.g, dth = K.dtheta;
    R hh = ld(S.f[HH] + i);
    CellOut<R> o;
    // energyCPU
#pragma unroll
    for (int t = 0; t < NMAX; t++)
        if (t < nt) e[t] = cmax(e[t], (R)0.0f);   // advected ee arrive in energy units
    // energintCPU
    R Etmp = (R)0.0f;
#pragma unroll
    for (int t = 0; t < NMAX; t++)
        if (t < nt) Etmp = Etmp + e[t];
    Etmp = Etmp * dth;
    R Htmp = DM<R>::sqrt(Etmp / (rho * g / (R)8.0f));
    R idiv = cmax((R)1.0f, DM<R>::pow(Htmp / (K.gammax * hh), (R)2.0f));
#pragma unroll
    for (int t = 0; t < NMAX; t++)
        if (t < nt) e[t] = e[t] / idiv;
    Htmp = cmin(Htmp, K.gammax * hh);
    R Eint = (rho * g * Htmp * Htmp) / (R)8.0f;
    R k = ld(S.f[WK] + i);
    R fw = ld(S.f[FWM] + i);
    R Dv;
    if (K.breakmodel == 1) {
        // roelvinkCPU (wave_CPU.cpp:927-985): double arithmetic as there
        R fac = (R)(8.0 / (double)rho / (double)g);
        R Ht = DM<R>::sqrt(Eint * fac);
        R Qb = (R)(1.0 - ::exp(cmax(-1.0 * (double)DM<R>::pow((Ht / K.gammaa / hh), K.nexp), -100.0)));
        Qb = cmin(Qb, (R)1.0f);
        Dv = (R)((double)Qb * 2.0 * (double)K.alpha / (double)Trep * (double)Eint * (double)Ht / (double)hh);
        R uorb = (R)(XBG_PI * (double)Ht / (double)(Trep * DM<R>::sinh(cmin(k * hh, (R)10.0f))));
        Dv = (R)((double)Dv + (double)0.66666666f / XBG_PI * (double)rho * (double)fw * (double)uorb *
                                  (double)uorb * (double)uorb);
    } else {
        // baldockCPU (wave_CPU.cpp:987-1028)
        R khh = k * hh;
        R Hb = ((R)0.88f / k) * DM<R>::tanh(K.gammaa * khh / (R)0.88f);
        R Rr = Hb / cmax(Htmp, (R)0.00001f);
        R Qb = DM<R>::exp((R)-1.0f * Rr * Rr);
        Dv = (R)0.25f * K.alpha * Qb * rho * ((R)1.0f / Trep) * g * (Hb * Hb + Htmp * Htmp);
        R uorb = (R)(XBG_PI * (double)Htmp / (double)(Trep * DM<R>::sinh(cmin(k * hh, (R)10.0f))));
        Dv = (R)((double)Dv + (double)0.66666666f / XBG_PI * (double)rho * (double)fw * (double)uorb *
                                  (double)uorb * (double)uorb);
    }
    // dissipationCPU (wave_CPU.cpp:1030-1092)
    R wci = K.wci * cmin(hh / K.hwci, (R)1.0f);
    R cc = ld(S.f[CC_] + i);
    R uui = ld(S.f[UU] + i) * wci, vvi = ld(S.f[VV] + i) * wci;
    R RR = (R)0.0f, drr = (R)0.0f;
    R Emax = cmax(Eint, (R)0.0000001f);
    bool wet = hh > K.eps;
#pragma unroll
    for (int t = 0; t < NMAX; t++) {
        if (t < nt) {
            R cx = cc * K.cxsth[t] + uui;
            R cy = cc * K.sxnth[t] + vvi;
            R eet = e[t];
            R dd = eet * Dv / Emax;
            R rrt;
            if (wet) {
                rrt = r[t];
                R rrd = (R)2.0f * g * K.beta * rrt / DM<R>::sqrt(cx * cx + cy * cy);
                eet = cmax(eet - dtf * dd, (R)0.0f);
                rrt = cmax(rrt + dtf * (dd - rrd), (R)0.0f);
                drr = drr + rrd;
            } else {
                eet = (R)0.0f; rrt = (R)0.0f; drr = (R)0.0f;
            }
            RR = RR + rrt;
            e[t] = eet;
            r[t] = rrt;
        }
    }
    o.E = Eint; o.H = Htmp; o.D = Dv; o.R_ = RR * dth; o.DR = drr * dth;
    return o;
}

// meandir + radstress (wave_CPU.cpp:1095-1162) of the final ee (e) and rr (r);
// writes everything a cell owns at the end of the wave pass.
template <class R, int NMAX>
__device__ __forceinline__ void finish_cell(const Dev<R>& S, const Konst<R>& K, int i, const R* e,
                                            const R* r, const CellOut<R>& o, R* een, R* rrn) {
    const int nt = K.nt, C = S.C;
    R rho = K.rho, g = K.g, dth = K.dtheta;
    R sume = (R)0, sumethet = (R)0;
    R txx = 0, txy = 0, tyy = 0, rxx = 0, rxy = 0, ryy = 0, sum2 = 0;
#pragma unroll
    for (int t = 0; t < NMAX; t++) {
        if (t < nt) {
            R et = e[t], rt = r[t];
            R cx = K.cxsth[t], sx = K.sxnth[t];
            sume = sume + et;
            sumethet = sumethet + et * K.theta[t];
            sum2 = sum2 + et;
            txx = txx + (((R)1.0f + cx * cx) * et);
            tyy = tyy + (((R)1.0f + sx * sx) * et);
            txy = txy + (sx * cx * et);
            rxx = rxx + ((cx * cx) * rt);
            ryy = ryy + ((sx * sx) * rt);
            rxy = rxy + (sx * cx * rt);
            een[i + (size_t)t * C] = et;
            rrn[i + (size_t)t * C] = rt;
        }
    }
    sume = cmax(sume, (R)0.00001f);
    S.f[THM][i] = (sumethet / (R)nt) / (sume / (R)nt);
    S.f[E][i] = sume * dth;
    S.f[H][i] = DM<R>::sqrt(sume * dth / (rho * g / (R)8));
    S.f[D][i] = o.D;
    S.f[ROL][i] = o.R_;
    S.f[DR][i] = o.DR;
    R n = ld(S.f[CG] + i) / ld(S.f[CC_] + i);
    S.tmp[T_SXX][i] = (n * txx - (R)0.5f * sum2) * dth + rxx * dth;
    S.tmp[T_SYY][i] = (n * tyy - (R)0.5f * sum2) * dth + ryy * dth;
    S.tmp[T_SXY][i] = n * txy * dth + rxy * dth;
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

// ctheta of every bin of a cell and WAVEDT (Wave_kernel.cu:232-249):
// min over theta of cfl*dtheta/|ctheta|.
template <class R, int NMAX>
__device__ __forceinline__ R ctheta_cell(const Konst<R>& K, const CthCoef<R>& cc, R* cthv) {
    R mindt = (R)9999999.9f;
#pragma unroll
    for (int t = 0; t < NMAX; t++) {
        if (t < K.nt) {
            cthv[t] = cth_eval(cc, K.cxsth[t], K.sxnth[t]);
            mindt = DM<R>::fmin(K.cfl * K.dtheta / DM<R>::fabs(cthv[t]), mindt);
        } else {
            cthv[t] = (R)0;
        }
    }
    return mindt;
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
template <class R>
__device__ __forceinline__ R flux2(R qm2, R qm, R qi, R qp, R qp2, R cf, R cfmin) {
    R arrin = (cf > (R)0 ? upw(qi, qm) : upw(qp, qp2)) * cf;
    R arrmin = (cfmin > (R)0 ? upw(qm, qm2) : upw(qi, qp)) * cfmin;
    return arrin - arrmin;
}
// theta-face flux between bins t and t+1 (the arrint of bin t, which is the
// arrmint of bin t+1): e(t-1), e(t), e(t+1), e(t+2), ctheta(t), ctheta(t+1)
template <class R>
__device__ __forceinline__ R theta_face(R em, R e0, R ep, R ep2, R c0, R cp) {
    R cb = (R)0.5f * (c0 + cp);
    R u1 = (R)1.5f * e0 - (R)0.5f * em;   u1 = u1 < (R)0 ? e0 : u1;
    R u2 = (R)1.5f * ep - (R)0.5f * ep2;  u2 = u2 < (R)0 ? ep : u2;
    return cb * (cb > (R)0 ? u1 : u2);
}

constexpr int WT_NB = 3;   // plane tile buffers: plane t+1 streams in while t is used

template <class R, bool ROLLER, bool WCI>
__device__ __forceinline__ void b_wave_fast(const Dev<R>& S, const Konst<R>& K, const int bix, const int biy) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Clock* clk = S.clk;
    if (halted(clk)) return;
    const int nx = K.nx, ny = K.ny, nt = K.nt, C = S.C;
    const int tid = threadIdx.x + threadIdx.y * WT_X;
    R* tE = (R*)smem_raw;                 // [WT_NB][WT_N] plane tiles of ee
    R* tR = tE + WT_NB * WT_N;            // [WT_NB][WT_N] plane tiles of rr
    R* sA = tR + WT_NB * WT_N;            // [nt][256] advected ee (energy units)
    R* sR = sA + (size_t)nt * 256;        // [nt][256] advected rr
    R* sCos = sR + (size_t)nt * 256;      // [nt]
    R* sSin = sCos + nt;                  // [nt]
    R* sTh = sSin + nt;                   // [nt]
    R* sC2 = sTh + nt;                    // [nt] cos^2, sin^2, sin cos of the bins
    R* sS2 = sC2 + nt;
    R* sCS = sS2 + nt;
    if (tid < nt) {
        const R c = K.cxsth[tid], sn = K.sxnth[tid];
        sCos[tid] = c; sSin[tid] = sn; sTh[tid] = K.theta[tid];
        sC2[tid] = c * c; sS2[tid] = sn * sn; sCS[tid] = sn * c;
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
    const bool own_bnd = ix == 0;
    auto own_e = [&](int t) -> R {
        R v = own_bnd ? St[iy + t * ny] * taper : ld(eeo + i + (size_t)t * C);
        return DM<R>::fmax(v, (R)0);
    };
    const bool edge_row = active && (iy == 1 || iy == ny - 2);
    const int slot = (iy == 1) ? 0 : 1;
    issue(0);
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
        const R h = (R)0.5f;
        axp = h * (cgi + ld(cgp + xp + iy * nx)); axm = h * (cgi + ld(cgp + xm + iy * nx));
        ayp = h * (cgi + ld(cgp + ix + yp * nx)); aym = h * (cgi + ld(cgp + ix + ym * nx));
        rxp = h * (cci + ld(cp + xp + iy * nx)); rxm = h * (cci + ld(cp + xm + iy * nx));
        ryp = h * (cci + ld(cp + ix + yp * nx)); rym = h * (cci + ld(cp + ix + ym * nx));
        const R* uu = S.f[UU]; const R* vv = S.f[VV];
        uui = ld(uu + i) * wci; vvi = wci * ld(vv + i);
        bxp = h * (uui + ld(uu + xp + iy * nx) * wci); bxm = h * (uui + ld(uu + xm + iy * nx) * wci);
        byp = h * (vvi + wci * ld(vv + ix + yp * nx)); bym = h * (vvi + wci * ld(vv + ix + ym * nx));
        auto cl = [&](int t) { return t < 0 ? 0 : (t >= nt ? nt - 1 : t); };
        we2 = own_e(0); we1 = we2; we3 = own_e(cl(1)); we4 = own_e(cl(2));
        wr2 = ld(rro + i); wr1 = wr2;
        wr3 = ld(rro + i + (size_t)cl(1) * C); wr4 = ld(rro + i + (size_t)cl(2) * C);
        if (!WCI) { cthP = cc.s * cc.dhdx; cthQ = -(cc.s * cc.dhdy); }
        c0 = cth(sCos[0], sSin[0]);
        cpp = cth(sCos[cl(1)], sSin[cl(1)]);
    }
    // the cell's own bins ahead (window refill): plane min(t+3, nt-1)
    const R* wE = eeo + i + (size_t)min(3, nt - 1) * C;
    const R* wR = rro + i + (size_t)min(3, nt - 1) * C;
    const R* wS = St + iy + min(3, nt - 1) * ny;
    R* oA = sA + tid;
    R* oR = sR + tid;
    R* oEdge = S.edge + ix + (size_t)slot * nt * nx;
    const size_t edge_rr = (size_t)2 * nt * nx;
#pragma unroll 1
    for (int t = 0; t < nt; t++) {
        const int b = t % WT_NB;
        if (t + 1 < nt) issue((t + 1) % WT_NB);
        else cp_async_commit();
        cp_async_wait1();   // plane t has landed (this thread's copies)
        fixup(b);
        __syncthreads();    // ... and every thread's; buffer (t+1)%3 was last read two planes ago
        if (active) {
            const R* qE = tE + b * WT_N + ctile;
            const R* qR = tR + b * WT_N + ctile;
            const R ct = sCos[t], st = sSin[t];
            const bool last = t == nt - 1;
            cabs = DM<R>::fmax(cabs, DM<R>::fabs(c0));
            R fx = flux2(qE[-2], qE[-1], we2, qE[1], qE[2], DM<R>::fma(ct, axp, bxp), DM<R>::fma(ct, axm, bxm));
            R fy = flux2(qE[-2 * WT_TX], qE[-WT_TX], we2, qE[WT_TX], qE[2 * WT_TX], DM<R>::fma(st, ayp, byp),
                         DM<R>::fma(st, aym, bym));
            // theta flux: upper face computed here, lower face carried from bin t-1
            R fup = last ? (R)0 : theta_face(we1, we2, we3, we4, c0, cpp);
            R ft = fup - fte;
            fte = fup;
            R A = we2 - dtf * ((fx + fy) * rdx + ft * rdth);
            R Ar = wr2;
            if (ROLLER) {
                R rx = flux2(qR[-2], qR[-1], wr2, qR[1], qR[2], DM<R>::fma(ct, rxp, bxp), DM<R>::fma(ct, rxm, bxm));
                R ry = flux2(qR[-2 * WT_TX], qR[-WT_TX], wr2, qR[WT_TX], qR[2 * WT_TX], DM<R>::fma(st, ryp, byp),
                             DM<R>::fma(st, rym, bym));
                R rup = last ? (R)0 : theta_face(wr1, wr2, wr3, wr4, c0, cpp);
                R rt = rup - ftr;
                ftr = rup;
                Ar = wr2 - dtf * ((rx + ry) * rdx + rt * rdth);
            }
            *oA = A;
            *oR = Ar;
            oA += 256; oR += 256;
            if (edge_row) {
                oEdge[0] = A;
                oEdge[edge_rr] = Ar;
            }
            oEdge += nx;
            Etmp = Etmp + DM<R>::fmax(A, (R)0);
            const int t2 = t + 2 < nt ? t + 2 : nt - 1;
            we1 = we2; we2 = we3; we3 = we4;
            we4 = DM<R>::fmax(own_bnd ? *wS * taper : ld(wE), (R)0);
            wr1 = wr2; wr2 = wr3; wr3 = wr4; wr4 = ld(wR);
            if (t + 4 <= nt - 1) { wE += C; wR += C; wS += ny; }
            c0 = cpp; cpp = cth(sCos[t2], sSin[t2]);
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
        // energintCPU
        Etmp = Etmp * dth;
        R Htmp = DM<R>::sqrt(Etmp / (rho * g / (R)8.0f));
        R hr = Htmp / (K.gammax * hh);
        const R idiv = DM<R>::fmax((R)1.0f, hr * hr);
        const R ridiv = (R)1 / idiv;
        Htmp = DM<R>::fmin(Htmp, K.gammax * hh);
        const R Eint = (rho * g * Htmp * Htmp) / (R)8.0f;
        const R k = ld(S.f[WK] + i);
        const R fw = ld(S.f[FWM] + i);
        R Dv;
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
        // dissipationCPU, meandir, radstress
        const R cc_i = cci;
        const R Dq = Dv / DM<R>::fmax(Eint, (R)0.0000001f);
        const R twogb = (R)2.0f * g * K.beta;
        const R rcoef = twogb / cc_i;   // without wave-current interaction |c (cos, sin)| = c
        const bool wet = hh > K.eps;
        R RR = (R)0.0f, drr = (R)0.0f, sume = (R)0, sumethet = (R)0;
        R ec = 0, es = 0, ecs = 0, rc = 0, rs = 0, rcs = 0;   // sums of cos^2, sin^2, sin cos times e / r
        R* pe_n = een + i;
        R* pr_n = rrn + i;
#pragma unroll 2
        for (int t = 0; t < nt; t++) {
            R eet = DM<R>::fmax(sA[t * 256 + tid], (R)0.0f) * ridiv;
            R rrt = sR[t * 256 + tid];
            const R dd = eet * Dq;
            R rrd;
            if (WCI) {
                const R cx = cc_i * sCos[t] + uui;
                const R cy = cc_i * sSin[t] + vvi;
                rrd = twogb * rrt / DM<R>::sqrt(cx * cx + cy * cy);
            } else {
                rrd = rrt * rcoef;
            }
            eet = wet ? DM<R>::fmax(eet - dtf * dd, (R)0.0f) : (R)0;
            rrt = wet ? DM<R>::fmax(rrt + dtf * (dd - rrd), (R)0.0f) : (R)0;
            drr = wet ? drr + rrd : (R)0;
            RR = RR + rrt;
            pe_n[(size_t)t * C] = eet;
            pr_n[(size_t)t * C] = rrt;
            sume = sume + eet;
            sumethet = sumethet + eet * sTh[t];
            const R c2 = sC2[t], s2 = sS2[t], cs = sCS[t];
            ec = DM<R>::fma(c2, eet, ec);
            es = DM<R>::fma(s2, eet, es);
            ecs = DM<R>::fma(cs, eet, ecs);
            rc = DM<R>::fma(c2, rrt, rc);
            rs = DM<R>::fma(s2, rrt, rs);
            rcs = DM<R>::fma(cs, rrt, rcs);
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
        S.tmp[T_SXX][i] = (n * (sum2 + ec) - (R)0.5f * sum2) * dth + rc * dth;
        S.tmp[T_SYY][i] = (n * (sum2 + es) - (R)0.5f * sum2) * dth + rs * dth;
        S.tmp[T_SXY][i] = n * ecs * dth + rcs * dth;
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

template <class R, int NMAX>
__device__ __forceinline__ void b_wave_edge(const Dev<R>& S, const Konst<R>& K, const int bix, const int biy) {
    const Clock* clk = S.clk;
    if (halted(clk)) return;
    const int nx = K.nx, ny = K.ny, nt = K.nt, C = S.C;
    int ix = bix * blockDim.x + threadIdx.x;
    int iy = (biy == 0) ? 0 : ny - 1;
    R dtw = (R)3.0e38f;
    if (ix < nx) {
        int i = ix + iy * nx;
        int src = (iy == 0) ? pp(0, ny) : mm(ny - 1);
        int slot = (iy == 0) ? 0 : 1;
        int par = clk->par;
        const R* rro = S.rr[par ^ 1];
        R* een = S.ee[par];
        R* rrn = S.rr[par];
        R sg = (R)clk->sigm;
        R dtf = (R)clk->dt;
        R Trep = (R)clk->Trep;
        CthCoef<R> cc = cth_coef(S, K, ix, iy, sg);
        R cthv[NMAX];
        dtw = ctheta_cell<R, NMAX>(K, cc, cthv);
        R w = ld(S.f[HH] + i) > K.eps ? (R)1.0f : (R)0.0f;
        R e[NMAX], r[NMAX];
#pragma unroll
        for (int t = 0; t < NMAX; t++) {
            if (t < nt) {
                e[t] = S.edge[ix + (size_t)t * nx + (size_t)slot * nt * nx] * w;
                r[t] = (K.roller == 1) ? S.edge[ix + (size_t)t * nx + (size_t)(slot + 2) * nt * nx] * w
                                       : ld(rro + i + (size_t)t * C);
            } else {
                e[t] = (R)0; r[t] = (R)0;
            }
        }
        CellOut<R> o = chain_cell<R, NMAX>(S, K, i, sg, dtf, Trep, e, r);
        // second rollerlatbnd(ee) after dissipation: copy of the source row
#pragma unroll
        for (int t = 0; t < NMAX; t++)
            if (t < nt) e[t] = een[ix + src * nx + (size_t)t * C] * w;
        finish_cell<R, NMAX>(S, K, i, e, r, o, een, rrn);
    }
    block_min_store<R>(dtw, S.part_wave + ((K.nx + 31) / 32) * ((K.ny - 2 + 7) / 8) + bix + biy * ((K.nx + 127) / 128));
}
template <class R, int NMAX>
__global__ void __launch_bounds__(128) k_wave_edge(Dev<R> S, Konst<R> K) {
    b_wave_edge<R, NMAX>(S, K, blockIdx.x, blockIdx.y);
}
template <class R, int NMAX>
__global__ void __launch_bounds__(128) kb_wave_edge(BatchTab<R> T, const int2* items, int n) {
    batch_items<R>(T, items, n, [&](const Dev<R>& S, const Konst<R>& K, const BatchAux&, int bx, int by) {
        b_wave_edge<R, NMAX>(S, K, bx, by);
    });
}

// wavforce (wave_CPU.cpp:1164-1238) at cell j, before the boundary copies.
template <class R>
__device__ __forceinline__ void force_raw(const Dev<R>& S, const Konst<R>& K, int ix, int iy, R& Fx, R& Fy) {
    const int nx = K.nx, ny = K.ny;
    const R* Sxx = S.tmp[T_SXX]; const R* Sxy = S.tmp[T_SXY]; const R* Syy = S.tmp[T_SYY];
    int xm = mm(ix), xp = pp(ix, nx), ym = mm(iy), yp = pp(iy, ny);
    int i = ix + iy * nx;
    R dxf = K.dx;
    R Sxxi = ld(Sxx + i), Sxxr = ld(Sxx + xp + iy * nx), Sxyt = ld(Sxy + ix + yp * nx);
    R Sxytr = ld(Sxy + xp + yp * nx), Sxyb = ld(Sxy + ix + ym * nx), Sxybr = ld(Sxy + xp + ym * nx);
    R Syyi = ld(Syy + i), Syyt = ld(Syy + ix + yp * nx), Sxyr = ld(Sxy + xp + iy * nx);
    R Sxyl = ld(Sxy + xm + iy * nx), Sxytl = ld(Sxy + xm + yp * nx);
    Fx = (R)-1 * (Sxxr - Sxxi) / dxf - (R)0.5f * (Sxyt + Sxytr - Sxyb - Sxybr) / ((R)2.0f * dxf);
    Fy = (R)-1 * (Syyt - Syyi) / dxf - (R)0.5f * (Sxyr + Sxytr - Sxyl - Sxytl) / ((R)2.0f * dxf);
}

// breakerdelayCPU (wave_CPU.cpp:1333-1368) at cell j.
template <class R>
__device__ __forceinline__ void breaker_raw(const Dev<R>& S, const Konst<R>& K, int j, R Trep, R& urms, R& ust) {
    R hmin = (R)0.2;
    R g = K.g, rho = K.rho;
    R Hi = ld(S.f[H] + j), ki = ld(S.f[WK] + j);
    R hhi = cmax(ld(S.f[HH] + j), hmin);
    R ci = cmax(ld(S.f[CC_] + j), DM<R>::sqrt(hmin * g));
    R Rl = ld(S.f[ROL] + j);
    R uorb = (R)(XBG_PI * (double)Hi / (double)Trep / (double)DM<R>::sinh(cmin(cmax(ki, (R)0.01f) * hhi, (R)10.0f)));
    urms = uorb / (DM<R>::sqrt((R)2.0f));
    R ustw = ld(S.f[E] + j) / ci / rho / hhi;
    R ustr = (R)2.0f * Rl / ci / rho / hhi;
    ust = ustw + ustr;
}

template <class R>
__device__ __forceinline__ void b_wave_force(const Dev<R>& S, const Konst<R>& K, const int bix, const int biy) {
    const Clock* clk = S.clk;
    if (halted(clk)) return;
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
    int gx = (K.nx + 31) / 32, gy = (K.ny - 2 + 7) / 8;
    int ex = (K.nx + 127) / 128;
    return gx * gy + ex * 2;
}

template <class R, int NMAX>
void launch_wave_main(const Dev<R>& S, const Konst<R>& K, cudaStream_t st, Prof* pf) {
    dim3 b(32, 8), g((K.nx + 31) / 32, (K.ny - 2 + 7) / 8);
    launch_wave_fast(S, K, g, b, wave_fast_smem<R>(K.nt), st);
    PMARK(pf, "k_wave_fast");
    dim3 be(128), ge((K.nx + 127) / 128, 2);
    k_wave_edge<R, NMAX><<<ge, be, 0, st>>>(S, K);
    PMARK(pf, "k_wave_edge");
}

template <class R>
int launch_wave(const Dev<R>& S, const Konst<R>& K, cudaStream_t st, Prof* pf) {
    int n = 0;
    k_disp<R><<<(S.C + 255) / 256, 256, 0, st>>>(S, K); n++;
    PMARK(pf, "k_disp");
    if (K.nt <= 4) launch_wave_main<R, 4>(S, K, st, pf);
    else if (K.nt <= 8) launch_wave_main<R, 8>(S, K, st, pf);
    else if (K.nt <= 12) launch_wave_main<R, 12>(S, K, st, pf);
    else if (K.nt <= 16) launch_wave_main<R, 16>(S, K, st, pf);
    else if (K.nt <= 20) launch_wave_main<R, 20>(S, K, st, pf);
    else if (K.nt <= 24) launch_wave_main<R, 24>(S, K, st, pf);
    else launch_wave_main<R, 32>(S, K, st, pf);
    n += 2;
    dim3 b(32, 8), g((K.nx + 31) / 32, (K.ny + 7) / 8);
    k_wave_force<R><<<g, b, 0, st>>>(S, K); n++;
    PMARK(pf, "k_wave_force");
    return n;
}

// the wave kernels over every scenario of a batch (one ntheta and roller
// setting for the whole batch)
template <class R, int NMAX>
void launch_wave_main_batch(const BatchTab<R>& T, const BatchLaunch& L, int nt, int roller, int wci, cudaStream_t st,
                            Prof* pf) {
    launch_wave_fast_batch(T, L, roller, wci, wave_fast_smem<R>(nt), st);
    PMARK(pf, "k_wave_fast");
    kb_wave_edge<R, NMAX><<<L.grid[BS_EDGE], 128, 0, st>>>(T, L.items[BS_EDGE], L.n[BS_EDGE]);
    PMARK(pf, "k_wave_edge");
}

template <class R>
int launch_wave_batch(const BatchTab<R>& T, const BatchLaunch& L, int nt, int roller, int wci, cudaStream_t st,
                      Prof* pf) {
    kb_disp<R><<<L.grid[BS_LIN], 256, 0, st>>>(T, L.items[BS_LIN], L.n[BS_LIN]);
    PMARK(pf, "k_disp");
    if (nt <= 4) launch_wave_main_batch<R, 4>(T, L, nt, roller, wci, st, pf);
    else if (nt <= 8) launch_wave_main_batch<R, 8>(T, L, nt, roller, wci, st, pf);
    else if (nt <= 12) launch_wave_main_batch<R, 12>(T, L, nt, roller, wci, st, pf);
    else if (nt <= 16) launch_wave_main_batch<R, 16>(T, L, nt, roller, wci, st, pf);
    else if (nt <= 20) launch_wave_main_batch<R, 20>(T, L, nt, roller, wci, st, pf);
    else if (nt <= 24) launch_wave_main_batch<R, 24>(T, L, nt, roller, wci, st, pf);
    else launch_wave_main_batch<R, 32>(T, L, nt, roller, wci, st, pf);
    kb_wave_force<R><<<L.grid[BS_TILE], dim3(32, 8), 0, st>>>(T, L.items[BS_TILE], L.n[BS_TILE]);
    PMARK(pf, "k_wave_force");
    return 4;
}
template int launch_wave_batch<float>(const BatchTab<float>&, const BatchLaunch&, int, int, int, cudaStream_t, Prof*);
template int launch_wave_batch<double>(const BatchTab<double>&, const BatchLaunch&, int, int, int, cudaStream_t, Prof*);

// One-time kernel attributes (dynamic shared memory above 48 KB for wide
// theta sets in FP64).
template <class R>
int wave_prepare(const Konst<R>& K) {
    const int smem = (int)wave_fast_smem<R>(K.nt);
    const cudaFuncAttribute a = cudaFuncAttributeMaxDynamicSharedMemorySize;
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

template int launch_wave<float>(const Dev<float>&, const Konst<float>&, cudaStream_t, Prof*);
template int launch_wave<double>(const Dev<double>&, const Konst<double>&, cudaStream_t, Prof*);
template int wave_parts<float>(const Konst<float>&);
template int wave_parts<double>(const Konst<double>&);

}  // namespace xbg
