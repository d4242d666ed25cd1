// sed.cu -- sediment transport and bed update (sedimentstep,
// Wave_gpu.cu:1405-1635; kernels of Sediment_kernel.cu) in three passes.
//
//   k_sed_a  longturb (rolthick; kturb = 0, Sediment_kernel.cu:161), Sbvr,
//            Rvr, Erosus                      -> rolthick ceqsg Tsg* ua* facero*
//   k_sed_b  Susp, Conc, CClatbnd, bedupdate  -> C* zb* hh* stdep* dzb
//   k_sed_c  zblatbnd, avalanching (gathered per cell), updatezb, zblatbnd,
//            updatezom                        -> zb stdep zs hh dzb cfm fwm C
// (* = per-step buffer).  hardlayer and zblatbnd(Sout) (:824-879) feed only
// the bed-load divergence that bedupdate has commented out (:954) and are not
// evaluated.  All kernels skip the step unless sedtrans = 1 and t >= sedstart
// (Wave_gpu.cu:724), a flag the device clock sets.
#include "xbg_common.cuh"

namespace xbg {

#define IDX(x, y) ((x) + (y) * nx)

__device__ __forceinline__ bool sed_skip(const Clock* c) {
    return halted(c) || *((volatile const int*)&c->do_sed) == 0;
}

// longturb, Sbvr, Rvr, Erosus (Sediment_kernel.cu:27-531) of one cell from
// its inputs: ueu_l is ueu of the left neighbour (mm), vev_b vev of the one
// below (mm)
template <class R>
struct SedAIn { R c, H, stdep, cfm, rol, dr, urms, rolth, dzsdt, hh, ueu_l, ueu, vev_b, vev; };
template <class R>
struct SedAOut { R rolth, ceqsg, ceqbg, Tsg, ua, facero; };
template <class R>
__device__ __forceinline__ SedAOut<R> sed_a_of(const Konst<R>& K, R dtf, R Trep, const SedAIn<R>& in) {
    R rho = K.rho, g = K.g, eps = K.eps;
    const R c = in.c, Hi = in.H, stdep = in.stdep, cfm = in.cfm, rol = in.rol, dri = in.dr, urms = in.urms;
    // longturb (Sediment_kernel.cu:27-164)
    R rolth = in.rolth + dtf * (DM<R>::fabs(in.dzsdt) - K.beta * c);
    rolth = DM<R>::fmax(rolth, (R)0.0f);
    // Sbvr (:167-326); kturb is 0 after longturb
    R zo = (R)0.006f, sedcal = (R)1.0f, bulk = (R)1.0f;
    R D50 = K.D50, D90 = K.D90;
    const R drhog = K.sed_drhog;
    R hh = in.hh;
    R hhi = DM<R>::fmax(hh, (R)0.01f);
    R ue = (R)(0.5 * (double)(in.ueu_l + in.ueu));
    R ve = (R)(0.5 * (double)(in.vev_b + in.vev));
    R vmags = ue * ue + ve * ve;
    R ML = DM<R>::fmax(DM<R>::fmin(DM<R>::sqrt((R)2.0f * rol * Trep / (rho * c)), hhi), (R)0.01f);
    R dcfin = DM<R>::exp(DM<R>::fmin(hhi, (R)100.0f) / ML);
    R dcf = DM<R>::fmin((R)1 / (dcfin - (R)1), (R)1.0f);
    R kb = K.nuhfac * DM<R>::pow23(dri / rho) * dcf;
    R Urms2 = urms * urms + (R)1.45f * (kb + (R)0.0f);
    R Tsg = DM<R>::fmax((R)0.1f * hhi / K.wws, (R)0.5f);
    R Ucr;
    Ucr = K.sed_ucr * DM<R>::log10((R)4.0f * hhi / D90);
    R hdrag = DM<R>::fmax(hhi, (R)10.0f * zo);
    R Cd = (R)0.4f / (DM<R>::log(hdrag / zo) - (R)1.0f);
    Cd = Cd * Cd;
    R Asb = (R)0.005f * hhi * DM<R>::pow((R)1 / hhi / drhog, (R)1.2f);
    R Ass = K.sed_Ass;
    R T1 = vmags + (R)0.018f / Cd * Urms2;
    T1 = DM<R>::fmin(T1, (R)100000.0f * g / cfm * D50 * K.sed_drho);
    T1 = DM<R>::sqrt(T1);
    R wetz = hhi > eps ? (R)1 : (R)0;
    R T2 = (R)0.0f;
    if (T1 > Ucr && hhi > eps) T2 = DM<R>::pow(T1 - Ucr, (R)2.4f);
    R ceqb = Asb * T2;
    ceqb = DM<R>::fmin(ceqb / hhi, (R)0.05f);
    R ceqbg = ((R)1 - bulk) * ceqb * sedcal * wetz;
    R ceqs = DM<R>::fmin(Ass * T2 / hhi, (R)0.05f);
    R ceqsg = (ceqs + bulk * ceqb) * sedcal * wetz;
    // Rvr (:477-509)
    R ua;
    {
        R m1 = (R)0.0f, m2 = (R)0.7939f, m3 = (R)-0.6065f, m4 = (R)0.3539f, m5 = (R)0.6373f, m6 = (R)0.5995f;
        R alpha = K.rvr_alpha;
        R beta = K.rvr_beta;
        R k = (R)(2 * XBG_PI / (double)(c * Trep));
        R Ur = (R)3.0f / (R)8.0f * DM<R>::sqrt((R)2.0f) * Hi * k / ((k * hh) * (k * hh) * (k * hh));
        Ur = DM<R>::fmax(Ur, (R)0.00001f);
        R Bm = m1 + (m2 - m1) / ((R)1.0f + beta * DM<R>::pow(Ur, alpha));
        R B1 = (R)((double)((R)-90.0f + (R)90.0f * DM<R>::tanh(m5 / DM<R>::pow(Ur, m6))) * XBG_PI / 180.0f);
        R Sk = Bm * DM<R>::cos(B1);
        R As = Bm * DM<R>::sin(B1);
        ua = (K.facsk * Sk - K.facas * As) * urms;
    }
    // Erosus (:512-531)
    {
        R exp_ero = K.morfac * dtf / ((R)1.0f - K.por) * hh * (ceqsg * (R)1.0f / Tsg + ceqbg * (R)1.0f / dtf);
        R facero = DM<R>::fmin((R)1.0f, stdep * (R)1.0f / DM<R>::fmax((R)0.000001f, exp_ero));
        return SedAOut<R>{rolth, ceqsg, ceqbg, Tsg, ua, facero};
    }
}

template <class R>
__device__ __forceinline__ void b_sed_a(const Dev<R>& S, const Konst<R>& K, const int bix, const int biy) {
    const Clock* clk = S.clk;
    if (sed_skip(clk)) return;
    const int nx = K.nx, ny = K.ny;
    int ix = bix * blockDim.x + threadIdx.x, iy = biy * blockDim.y + threadIdx.y;
    if (ix >= nx || iy >= ny) return;
    int i = IDX(ix, iy), xm = mm(ix), ym = mm(iy);
    const R dtf = (R)clk->dt, Trep = (R)clk->Trep;
    // every input is loaded here, ahead of the arithmetic's branches, so that
    // the loads make one round trip to memory
    const SedAIn<R> in{ld(S.f[CC_] + i), ld(S.f[H] + i), ld(S.f[STDEP] + i), ld(S.f[CFM] + i), ld(S.f[ROL] + i),
                       ld(S.f[DR] + i), ld(S.f[URMS] + i), ld(S.f[ROLTHICK] + i), ld(S.f[DZSDT] + i),
                       ld(S.f[HH] + i), ld(S.f[UEU] + IDX(xm, iy)), ld(S.f[UEU] + i), ld(S.f[VEV] + IDX(ix, ym)),
                       ld(S.f[VEV] + i)};
    const SedAOut<R> o = sed_a_of(K, dtf, Trep, in);
    S.f[ROLTHICK][i] = o.rolth;
    S.f[KTURB][i] = (R)0.0f;
    S.f[CEQSG][i] = o.ceqsg;
    S.tmp[T_CEQBG][i] = o.ceqbg;
    S.tmp[T_TSG][i] = o.Tsg;
    S.tmp[T_UA][i] = o.ua;
    S.tmp[T_FACERO][i] = o.facero;
}
XBG_KERNELS(sed_a)

// The same pass over row segments (Seg), with the same arithmetic.
template <class R>
__global__ void __launch_bounds__(256) k_sed_a_v(Dev<R> S, Konst<R> K) {
    using G = Seg<R>;
    constexpr int V = G::V;
    const Clock* clk = S.clk;
    if (sed_skip(clk)) return;
    const int nx = K.nx, ny = K.ny;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (iy >= ny) return;   // the whole warp: a warp is one row
    const G g(nx, blockIdx.x);
    const int ym = mm(iy);
    const R dtf = (R)clk->dt, Trep = (R)clk->Trep;
    const typename G::U c = g.row(S.f[CC_], iy), Hs = g.row(S.f[H], iy), sd = g.row(S.f[STDEP], iy),
                        cf = g.row(S.f[CFM], iy), ro = g.row(S.f[ROL], iy), dr = g.row(S.f[DR], iy),
                        ur = g.row(S.f[URMS], iy), rt = g.row(S.f[ROLTHICK], iy), dz = g.row(S.f[DZSDT], iy),
                        hh = g.row(S.f[HH], iy), ue = g.row(S.f[UEU], iy), vb = g.row(S.f[VEV], ym),
                        ve = g.row(S.f[VEV], iy);
    const R uel = g.left(ue, S.f[UEU], iy);
    typename G::U o_rt, o_cs, o_cb, o_ts, o_ua, o_fe, zero;
#pragma unroll
    for (int k = 0; k < V; k++) {
        const SedAIn<R> in{c.a[k], Hs.a[k], sd.a[k], cf.a[k], ro.a[k], dr.a[k], ur.a[k], rt.a[k], dz.a[k], hh.a[k],
                           k > 0 ? ue.a[k - 1] : uel, ue.a[k], vb.a[k], ve.a[k]};
        const SedAOut<R> o = sed_a_of(K, dtf, Trep, in);
        o_rt.a[k] = o.rolth; o_cs.a[k] = o.ceqsg; o_cb.a[k] = o.ceqbg; o_ts.a[k] = o.Tsg; o_ua.a[k] = o.ua;
        o_fe.a[k] = o.facero; zero.a[k] = (R)0.0f;
    }
    if (!g.act) return;
    g.put(S.f[ROLTHICK], iy, o_rt);
    g.put(S.f[KTURB], iy, zero);
    g.put(S.f[CEQSG], iy, o_cs);
    g.put(S.tmp[T_CEQBG], iy, o_cb);
    g.put(S.tmp[T_TSG], iy, o_ts);
    g.put(S.tmp[T_UA], iy, o_ua);
    g.put(S.tmp[T_FACERO], iy, o_fe);
}

// Susp (Sediment_kernel.cu:534-719): suspended fluxes Sus, Svs at (ix, iy)
template <class R>
__device__ __forceinline__ void susp_cell(const Dev<R>& S, const Konst<R>& K, int ix, int iy, R& Sus, R& Svs) {
    const int nx = K.nx, ny = K.ny;
    int i = IDX(ix, iy), xp = pp(ix, nx), yp = pp(iy, ny);
    const R* ua = S.tmp[T_UA];
    R dx = K.dx, eps = K.eps, facsl = (R)1.6f;
    R hhi = ld(S.f[HH] + i), zbi = ld(S.f[ZB] + i), zbr = ld(S.f[ZB] + IDX(xp, iy)), zbt = ld(S.f[ZB] + IDX(ix, yp));
    R cci = ld(S.f[CSED] + i), ccr = ld(S.f[CSED] + IDX(xp, iy)), cct = ld(S.f[CSED] + IDX(ix, yp));
    R uui = ld(S.f[UU] + i), vvi = ld(S.f[VV] + i), tm = ld(S.f[THM] + i);
    const R hu = ld(S.f[HU] + i), hv = ld(S.f[HV] + i), dri = ld(S.f[DR] + i);   // ahead of the branches
    R uai = ld(ua + i), uar = ld(ua + IDX(xp, iy)), uat = ld(ua + IDX(ix, yp));
    double ctm = (double)DM<R>::cos(tm), stm = (double)DM<R>::sin(tm);
    R uau = (R)(0.5 * ctm * (double)(uai + uar));
    R uav = (R)(0.5 * stm * (double)(uar + uai));
    R uv = ld(S.f[UV] + i), vu = ld(S.f[VU] + i);
    R urep = ld(S.f[UEU] + i) + uau;
    R vmagu = DM<R>::sqrt((uui + uau) * (uui + uau) + (vu + uav) * (vu + uav));
    uau = (R)(0.5 * ctm * (double)(uai + uat));
    uav = (R)(0.5 * stm * (double)(uat + uai));
    R vrep = ld(S.f[VEV] + i) + uav;
    R vmagv = DM<R>::sqrt((uv + uau) * (uv + uau) + (vvi + uav) * (vvi + uav));
    R dzbdx = (R)-1.0f * (zbr - zbi) / dx;
    R dzbdy = (R)-1.0f * (zbt - zbi) / dx;
    R wu = hu > eps ? (R)1.0f : (R)0.0f;
    R wv = hv > eps ? (R)1.0f : (R)0.0f;
    R cu, cv;
    if (urep > (R)0.0f) cu = cci;
    else if (urep < (R)0.0f) cu = ccr;
    else cu = (R)0.50f * (cci + ccr);
    R dcsdx = (ccr - cci) / dx;
    if (vrep > (R)0.0f) cv = cci;
    else if (vrep < (R)0.0f) cv = cct;
    else cv = (R)0.50f * (cci + cct);
    R dcsdy = (cct - cci) / dx;
    R Dc = K.nuh + K.nuhfac * hhi * DM<R>::pow13(dri / K.rho);
    Sus = K.sus * (cu * urep * hu - Dc * hu * dcsdx - facsl * cu * vmagu * hu * dzbdx) * wu;
    Svs = K.sus * (cv * vrep * hv - Dc * hv * dcsdy - facsl * cv * vmagv * hv * dzbdy) * wv;
}

// Conc (Sediment_kernel.cu:721-780) at cell i from the suspended fluxes of
// the cell (Susi, Svsi), its left face neighbour (Susl) and the one below
// (Svsb): new C, ero, depo.
template <class R>
struct ConcIn { R hhi, Tsg, facero, ceqsg, csed; };
template <class R>
__device__ __forceinline__ ConcIn<R> conc_in(const Dev<R>& S, int i) {
    return ConcIn<R>{ld(S.f[HH] + i), ld(S.tmp[T_TSG] + i), ld(S.tmp[T_FACERO] + i), ld(S.f[CEQSG] + i),
                     ld(S.f[CSED] + i)};
}
template <class R>
__device__ __forceinline__ R conc_of(const Konst<R>& K, const ConcIn<R>& c, R dtf, R Susi, R Svsi, R Susl, R Svsb,
                                     R& ero, R& depo) {
    const R hhi = c.hhi, Tsg = c.Tsg;
    R wetz = hhi > K.eps ? (R)1.0f : (R)0.0f;
    ero = c.facero * hhi * c.ceqsg * (R)1.0f / Tsg;
    R dsusdx = (Susi - Susl) / K.dx;
    R dsvsdy = (Svsi - Svsb) / K.dx;
    R cs = (dtf * Tsg) / (dtf + Tsg) * (hhi * c.csed / dtf - (dsusdx + dsvsdy - ero)) * wetz;
    cs = DM<R>::fmax(cs, (R)0.0f);
    cs = DM<R>::fmin(cs, (R)0.1f * hhi);
    depo = cs / Tsg;
    return cs / hhi;
}
template <class R>
__device__ __forceinline__ R conc_from(const Dev<R>& S, const Konst<R>& K, int i, R dtf, R Susi, R Svsi, R Susl,
                                       R Svsb, R& ero, R& depo) {
    return conc_of(K, conc_in(S, i), dtf, Susi, Svsi, Susl, Svsb, ero, depo);
}

// Conc at (ix, iy) evaluating the three Susp it needs (lateral rows only).
template <class R>
__device__ __forceinline__ R conc_cell(const Dev<R>& S, const Konst<R>& K, int ix, int iy, R dtf, R& ero, R& depo) {
    R Susi, Svsi, Susl, t0, t1, Svsb;
    susp_cell(S, K, ix, iy, Susi, Svsi);
    int xm = mm(ix), ym = mm(iy);
    if (xm != ix) susp_cell(S, K, xm, iy, Susl, t0); else Susl = Susi;
    if (ym != iy) susp_cell(S, K, ix, ym, t1, Svsb); else Svsb = Svsi;
    return conc_from(S, K, ix + iy * K.nx, dtf, Susi, Svsi, Susl, Svsb, ero, depo);
}

// Susp once per cell of the block's 32 x 8 tile plus the column to its left
// and the row below it (clamped at the grid edge, where mm() maps a cell to
// itself), then Conc from shared memory.  The lateral rows 0 and ny-1 take
// Conc of rows 1 and ny-2 (CClatbnd), evaluated directly.
constexpr int SB_X = 32, SB_Y = 8, SB_TX = SB_X + 1, SB_TY = SB_Y + 1;

template <class R>
__device__ __forceinline__ void b_sed_b(const Dev<R>& S, const Konst<R>& K, const int bix, const int biy) {
    const Clock* clk = S.clk;
    // tested once the block's loads are in flight (see halted())
    const bool off = sed_skip(clk);
    __shared__ R sSus[SB_TY * SB_TX], sSvs[SB_TY * SB_TX];
    const int nx = K.nx, ny = K.ny;
    const int bx0 = bix * SB_X, by0 = biy * SB_Y;
    const int tid = threadIdx.x + threadIdx.y * SB_X;
    const int ix = bx0 + threadIdx.x, iy = by0 + threadIdx.y;
    const bool cell = ix < nx && iy < ny;
    const int i = IDX(ix, iy);
    const bool morph = K.morfac > (R)0.0f;
    // the cell's own inputs first, so that their round trip overlaps the tile's
    ConcIn<R> ci{};
    R zb0 = (R)0, sd0 = (R)0;
    if (cell) {
        ci = conc_in(S, i);
        if (morph) { zb0 = ld(S.f[ZB] + i); sd0 = ld(S.f[STDEP] + i); }
    }
    for (int e = tid; e < SB_TY * SB_TX; e += SB_X * SB_Y) {
        int kx = e % SB_TX, ky = e / SB_TX;
        int gx = min(max(bx0 - 1 + kx, 0), nx - 1), gy = min(max(by0 - 1 + ky, 0), ny - 1);
        R a, b;
        susp_cell(S, K, gx, gy, a, b);
        sSus[e] = a;
        sSvs[e] = b;
    }
    __syncthreads();
    if (!cell) return;
    R dtf = (R)clk->dt;
    R ero, depo, cnew;
    const int c = (threadIdx.y + 1) * SB_TX + threadIdx.x + 1;
    cnew = conc_of(K, ci, dtf, sSus[c], sSvs[c], sSus[c - 1], sSvs[c - SB_TX], ero, depo);
    // CClatbnd (Sediment_kernel.cu:782-821)
    if (iy == 0 || iy == ny - 1) {
        R e2, d2;
        cnew = conc_cell(S, K, ix, iy == 0 ? pp(0, ny) : mm(ny - 1), dtf, e2, d2);
    }
    if (ix == 0) cnew = (R)0.0f;
    loads_before_here();
    if (off) return;
    S.tmp[T_UU][i] = cnew;   // per-step buffer reused for the new C
    if (morph) {
        // bedupdate (:881-968), bed-load divergence commented out there
        R dzg = K.morfac * dtf / ((R)1.0f - K.por) * (ero - depo);
        S.tmp[T_ZB][i] = zb0 + dzg;
        S.tmp[T_HH][i] = ci.hhi + dzg;
        S.f[DZB][i] = (R)-1 * dzg;
        S.tmp[T_STDEP][i] = sd0 - dzg;
    }
}
XBG_KERNELS(sed_b)

// zblatbnd source cell (Sediment_kernel.cu:970-1018, pre-kernel reads)
__device__ __forceinline__ int zbl_src(int ix, int iy, int nx, int ny) {
    int sx = ix, sy = iy;
    if (iy == 0) sy = pp(iy, ny);
    if (iy == ny - 1) sy = mm(iy);
    if (ix == 0) { sx = pp(ix, nx); sy = iy; }
    return sx + sy * nx;
}

// the same source as a column and row
__device__ __forceinline__ void zbl_xy(int ix, int iy, int nx, int ny, int& sx, int& sy) {
    sx = ix; sy = iy;
    if (iy == 0) sy = pp(iy, ny);
    if (iy == ny - 1) sy = mm(iy);
    if (ix == 0) { sx = pp(ix, nx); sy = iy; }
}

// avalanching (Sediment_kernel.cu:1020-1137) transfers (dzbx, dzby) of (ix, iy)
template <class R>
__device__ __forceinline__ void aval_cell(const Dev<R>& S, const Konst<R>& K, int ix, int iy, R dtf, R& dzbx, R& dzby) {
    const int nx = K.nx, ny = K.ny;
    const R* zb = S.tmp[T_ZB]; const R* sd = S.tmp[T_STDEP];
    int xp = pp(ix, nx), yp = pp(iy, ny);
    R Zbi = ld(zb + zbl_src(ix, iy, nx, ny)), Zbt = ld(zb + zbl_src(ix, yp, nx, ny)), Zbr = ld(zb + zbl_src(xp, iy, nx, ny));
    R sti = ld(sd + zbl_src(ix, iy, nx, ny)), stt = ld(sd + zbl_src(ix, yp, nx, ny)), str = ld(sd + zbl_src(xp, iy, nx, ny));
    R dx = K.dx, maxchg = K.maxslpchg;
    R dzmax = ld(S.tmp[T_HH] + IDX(ix, iy)) > K.eps ? K.wetdzmax : K.drydzmax;
    dzbx = (R)0.0f; dzby = (R)0.0f;
    R dzbdx = (Zbr - Zbi) / dx;
    if (DM<R>::fabs(dzbdx) > dzmax) {
        R s = dzbdx / DM<R>::fabs(dzbdx);
        dzbx = s * (DM<R>::fabs(dzbdx) - dzmax) * dx;
        if (s > (R)0) {
            dzbx = DM<R>::fmin(dzbx, maxchg * dtf / dx);
            dzbx = DM<R>::fmin(dzbx, sti);
        } else {
            dzbx = DM<R>::fmax(dzbx, (R)-1.0f * maxchg * dtf / dx);
            dzbx = DM<R>::fmax(dzbx, (R)-1.0f * str);
        }
    }
    R dzbdy = (Zbt - Zbi) / dx;
    if (DM<R>::fabs(dzbdy) > dzmax) {
        R s = dzbdy / DM<R>::fabs(dzbdy);
        dzby = s * (DM<R>::fabs(dzbdy) - dzmax) * dx;
        if (s > (R)0) {
            dzby = DM<R>::fmin(dzby, maxchg * dtf / dx);
            dzby = DM<R>::fmin(dzby, sti);
        } else {
            dzby = DM<R>::fmax(dzby, (R)-1 * maxchg * dtf / dx);
            dzby = DM<R>::fmax(dzby, (R)-1 * stt);
        }
    }
}

// bed change of (ix, iy) gathered from its own and its neighbours' transfers,
// in the order a serial launch adds them: ((-dzby[below] - dzbx[left]) + dzbx) + dzby
template <class R>
__device__ __forceinline__ R ddzb_cell(const Dev<R>& S, const Konst<R>& K, int ix, int iy, R dtf) {
    R a = (R)0.0f, bx, by, t;
    if (iy > 0) { aval_cell(S, K, ix, iy - 1, dtf, t, by); a = a - by; }
    if (ix > 0) { aval_cell(S, K, ix - 1, iy, dtf, bx, t); a = a - bx; }
    aval_cell(S, K, ix, iy, dtf, bx, by);
    a = a + bx;
    a = a + by;
    return a;
}

// zblatbnd, avalanching, updatezb, zblatbnd, updatezom.  The transfers
// (dzbx, dzby) of every cell of the 32 x 8 tile, the column to its left and
// the row below it go to shared memory once; a boundary cell whose zblatbnd
// source lies elsewhere evaluates that source's bed change directly.
template <class R>
__device__ __forceinline__ void b_sed_c(const Dev<R>& S, const Konst<R>& K, const int bix, const int biy) {
    const Clock* clk = S.clk;
    if (sed_skip(clk)) return;
    __shared__ R sBx[SB_TY * SB_TX], sBy[SB_TY * SB_TX];
    const int nx = K.nx, ny = K.ny;
    const int bx0 = bix * SB_X, by0 = biy * SB_Y;
    const bool morph = K.morfac > (R)0.0f;
    const R dtf = (R)clk->dt;
    const int ix = bx0 + threadIdx.x, iy = by0 + threadIdx.y;
    const bool cell = ix < nx && iy < ny;
    const int i = IDX(ix, iy);
    // the cell's own inputs first, so that their round trip overlaps the tile's
    R cnew = (R)0, dzb0 = (R)0, zs0 = (R)0, hh0 = (R)0, zb1 = (R)0, sd1 = (R)0;
    int sx = ix, sy = iy;
    if (cell) {
        cnew = ld(S.tmp[T_UU] + i);
        if (morph) {
            dzb0 = ld(S.f[DZB] + i);
            zs0 = ld(S.f[ZS] + i);
            hh0 = ld(S.tmp[T_HH] + i);
            zbl_xy(ix, iy, nx, ny, sx, sy);
            int s1x, s1y;
            zbl_xy(sx, sy, nx, ny, s1x, s1y);
            zb1 = ld(S.tmp[T_ZB] + IDX(s1x, s1y));
            sd1 = ld(S.tmp[T_STDEP] + IDX(s1x, s1y));
        }
    }
    if (morph) {
        for (int e = threadIdx.x + threadIdx.y * SB_X; e < SB_TY * SB_TX; e += SB_X * SB_Y) {
            int gx = min(max(bx0 - 1 + e % SB_TX, 0), nx - 1), gy = min(max(by0 - 1 + e / SB_TX, 0), ny - 1);
            R a, b;
            aval_cell(S, K, gx, gy, dtf, a, b);
            sBx[e] = a;
            sBy[e] = b;
        }
    }
    __syncthreads();
    if (!cell) return;
    S.f[CSED][i] = cnew;
    if (morph) {
        // bed change gathered in the serial launch order:
        // ((-dzby[below] - dzbx[left]) + dzbx) + dzby
        const int c = (threadIdx.y + 1) * SB_TX + threadIdx.x + 1;
        R dd = (R)0.0f;
        if (iy > 0) dd = dd - sBy[c - SB_TX];
        if (ix > 0) dd = dd - sBx[c - 1];
        dd = dd + sBx[c];
        dd = dd + sBy[c];
        // updatezb (:1139-1160) at the own cell
        S.f[DZB][i] = dzb0 - dd;
        S.f[ZS][i] = zs0 - dd;
        S.f[HH][i] = hh0 - dd;
        // zb, stdep: updatezb at the zblatbnd source, then the copy
        const int s = IDX(sx, sy);
        R ds = (s == i) ? dd : ddzb_cell(S, K, sx, sy, dtf);
        R zbn = zb1 + ds;
        R sdn = sd1 - ds;
        S.f[ZB][i] = zbn;
        S.f[STDEP][i] = sdn;
        // updatezom (:1162-1190)
        if (sdn < (R)0.05f) { S.f[CFM][i] = K.cfreef; S.f[FWM][i] = K.fwreef; }
        else { S.f[CFM][i] = K.cfsand; S.f[FWM][i] = K.fwsand; }
    }
}
XBG_KERNELS(sed_c)

// wide: the pointwise first pass in 64 x 4 blocks instead of 32 x 8; vec: over
// row segments (where nx is a multiple of the segment width)
template <class R>
int launch_sed(const Dev<R>& S, const Konst<R>& K, cudaStream_t st, Prof* pf, bool wide, bool vec) {
    dim3 b(32, 8), g((K.nx + 31) / 32, (K.ny + 7) / 8);
    constexpr int V = SegVec<R>::V;
    if (vec && K.nx % V == 0) k_sed_a_v<R><<<dim3((K.nx / V + 31) / 32, (K.ny + 7) / 8), b, 0, st>>>(S, K);
    else if (wide) k_sed_a<R><<<dim3((K.nx + 63) / 64, (K.ny + 3) / 4), dim3(64, 4), 0, st>>>(S, K);
    else k_sed_a<R><<<g, b, 0, st>>>(S, K);
    PMARK(pf, "k_sed_a");
    k_sed_b<R><<<g, b, 0, st>>>(S, K);
    PMARK(pf, "k_sed_b");
    k_sed_c<R><<<g, b, 0, st>>>(S, K);
    PMARK(pf, "k_sed_c");
    return 3;
}
// the three sediment kernels over every scenario of a batch
template <class R>
int launch_sed_batch(const BatchTab<R>& T, const BatchLaunch& L, cudaStream_t st, Prof* pf, bool wide) {
    dim3 b(32, 8);
    const int2* it = L.items[BS_TILE];
    int n = L.n[BS_TILE], g = L.grid[BS_TILE];
    if (wide) kb_sed_a<R><<<L.grid[BS_WIDE], dim3(64, 4), 0, st>>>(T, L.items[BS_WIDE], L.n[BS_WIDE]);
    else kb_sed_a<R><<<g, b, 0, st>>>(T, it, n);
    PMARK(pf, "k_sed_a");
    kb_sed_b<R><<<g, b, 0, st>>>(T, it, n);
    PMARK(pf, "k_sed_b");
    kb_sed_c<R><<<g, b, 0, st>>>(T, it, n);
    PMARK(pf, "k_sed_c");
    return 3;
}
template int launch_sed_batch<float>(const BatchTab<float>&, const BatchLaunch&, cudaStream_t, Prof*, bool);
template int launch_sed_batch<double>(const BatchTab<double>&, const BatchLaunch&, cudaStream_t, Prof*, bool);

template int launch_sed<float>(const Dev<float>&, const Konst<float>&, cudaStream_t, Prof*, bool, bool);
template int launch_sed<double>(const Dev<double>&, const Konst<double>&, cudaStream_t, Prof*, bool, bool);

}  // namespace xbg
