// k4_adjoint.cu -- gradients of the FP32 far-field amplitudes (the adjoint).
//
// For one orientation the FP32 far-field sum (k2_fp32.cu) maps the facet
// vertices and the beam amplitude matrices to the amplitude grids
// ampl_far_beam / ampl_far_ext_diff.  Given the cotangents of those grids
// (dL/dRe + i dL/dIm, e.g. from a Mueller-matrix loss), this file computes
// dL/d(vertex coordinates) and dL/d(amplitude matrices): the vector-Jacobian
// product of the forward, with the beam topology (which facets emit, their
// propagation and e-perp directions, the anti-parallel sign and the
// field-of-view masks) held fixed.
//
// The forward is restated in terms of the facet centre c, the vertices in the
// aperture frame (xa_j, ya_j) and the frame R = [x; y; z] itself, where z = -n
// with n = unit((v1-c) x (v2-c)), x = unit(p - (p.n) n) and y = z x x: that is
// the frame the reference builds from angles (src/diff_mod.f90:200-289,
// 540-559).  Per facet x bin the kernel recomputes the forward quantities and
// back-propagates; everything that depends on the bin only through a linear
// map of per-facet data is accumulated as a per-facet sum over bins (36
// floats), so no facet x bin intermediate is stored.  A host pass in FP64 then
// maps those sums through the frame construction to the vertex gradients.
//
// Layout: one warp per record (4 per CTA), lanes striding over a range of
// bins with the 36 sums in registers; one warp reduction and one FP64 atomic
// per (record, bin range) at the end.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "frame.h"
#include "pbt_internal.h"

namespace pbt {

namespace {

constexpr int K4_WARPS = 4;     // records per CTA, one per warp
constexpr int64_t K4_MAX_LANE_BINS = 1024;  // FP32 terms per lane and accumulator
constexpr int K4_NACC = 36;     // per-record accumulators
constexpr double kTwoPi4 = 6.283185307179586;
constexpr double kInv2Pi4 = 0.15915494309189535;
constexpr double kMagic4 = 6755399441055744.0;
constexpr float kClampSq4 = (float)(1.0 - (double)0.999999f * (double)0.999999f);

// accumulator layout
enum {
    A_AMP = 0,     // 8: cotangent of amp' (re, im) x 4
    A_TKX = 8,     // 3: sum theta_bar_j * kxx
    A_TKY = 11,    // 3: sum theta_bar_j * kyy
    A_WU = 14,     // 9: sum w_bar (x) u   (row-major, R_bar contribution)
    A_EA = 23,     // 3: sum ea_bar
    A_P2 = 26,     // 3: prop2 cotangent
    A_INC = 29,    // 3: incidence-in-frame cotangent
    A_CU = 32,     // 3: sum of (c-direct coefficient) x u, the u-parallel part of c_bar
    A_CE = 35,     // 1: sum of the coefficient of 2 c / R^2 in c_bar
};

// packed accumulator pairs: (TKX_j, TKY_j) and (WU_i0, WU_i1)
// and the two Karczewski-Wolf bin sums (sum ee_bar s, sum X) that the
// record's constants scale into A_P2 at the end
enum { P_TK = 0, P_WU01 = 3, P_KW = 6, K4_NPAIR = 7 };

// Fields in groups of four floats on 16-byte boundaries, in the order the
// bin loop reads them, so that the shared-memory reads can be 16 bytes wide.
struct __align__(16) K4Rec {
    double kc[3];
    double pad0;
    float eps[3], b;
    float R[9], ea[3];
    float kp[2], kw1, hicf;  // kw1 = -p2z cf / 2, hicf = icf / 2
    float inc[3], kw2;       // kw2 = p2x p2y cf / 2
    float xa[3], ya[3], cf, icf;
    float p2[3], pad1;
    float amp[8];
};
static_assert(sizeof(K4Rec) == 208, "K4Rec layout");

// Per-bin input in HBM: the unit bin direction in FP64, 32 B (two 16-byte
// loads).  The forward-bodge direction (same phi, first row above 1 degree)
// is read from the same table inside the (rare) bodge branch.
struct __align__(16) K4Bin {
    double ux, uy, uz, pad;
};

struct Bin4 {
    double ux, uy, uz;
    float fx, fy, fz;
    bool pole;     // within reach of the forward bodge for some record (|uz| near 1)
    int64_t o;     // bin index
    float2 G[4];   // cotangent of S' (pre-T, common phase removed) for the record's kind,
                   // circular basis of the columns: H+_1, H-_1, H+_2, H-_2
    float2 Gm[4];  // -i G
};

__device__ __forceinline__ float2 bc2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }

__device__ __forceinline__ float rcp4(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// the special-function unit's approximations with subnormal inputs flushed
// to zero (phases and squared norms here, never subnormal)
__device__ __forceinline__ void sincos4(float x, float *sn, float *cs) {
    asm("sin.approx.ftz.f32 %0, %1;" : "=f"(*sn) : "f"(x));
    asm("cos.approx.ftz.f32 %0, %1;" : "=f"(*cs) : "f"(x));
}
__device__ __forceinline__ float rsqrt4(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// sinc(h) and sinc'(h) for h >= 0: series below 0.5, else sin(h)/h and
// (cos h - sinc h)/h with rh = 1/max(h, 0.5).  series (warp-uniform) is false
// when no lane of the warp has an argument below 0.5; the polynomials are
// then skipped.
__device__ __forceinline__ void sinc_d(float h, float rh, bool series, float &sc, float &dsc) {
    float s, c;
    sincos4(h, &s, &c);
    sc = s * rh;
    dsc = (c - sc) * rh;
    if (series) {
        const float h2 = h * h;
        const float ps = fmaf(
            h2, fmaf(h2, fmaf(h2, fmaf(h2, 2.7557319e-6f, -1.9841270e-4f), 8.3333333e-3f), -1.6666667e-1f),
            1.0f);
        // d/dh (sin h / h) = -h/3 + h^3/30 - h^5/840 + h^7/45360
        const float pd =
            h * fmaf(h2, fmaf(h2, fmaf(h2, 2.2045855e-5f, -1.1904762e-3f), 3.3333333e-2f), -0.33333333f);
        const bool small = h < 0.5f;
        sc = small ? ps : sc;
        dsc = small ? pd : dsc;
    }
}

// g, dg/dlo, dg/dhi from the series about mid, for phases within 0.25 rad
__device__ __forceinline__ void dd_series(float lo, float mid, float hi, float2 &g, float2 &dlo,
                                          float2 &dhi) {
    // series about mid: g = e^{i mid} sum_n c_n h_n(ya, yc), c_n = i^(n+2)/(n+2)!
    const float ya = lo - mid, yc = hi - mid;
    const float cr[8] = {-0.5f, 0.0f, 1.0f / 24.0f, 0.0f, -1.0f / 720.0f, 0.0f, 1.0f / 40320.0f, 0.0f};
    const float ci[8] = {0.0f, -1.0f / 6.0f, 0.0f, 1.0f / 120.0f, 0.0f, -1.0f / 5040.0f, 0.0f,
                         1.0f / 362880.0f};
    float hq = 1.0f, da = 0.0f, dc = 0.0f, yap = 1.0f;
    float2 sg = make_float2(cr[0], ci[0]), sa = make_float2(0, 0), sc = make_float2(0, 0);
#pragma unroll
    for (int n = 1; n < 8; n++) {
        dc = fmaf(yc, dc, hq);
        da = fmaf(yc, da, (float)n * yap);
        yap *= ya;
        hq = fmaf(yc, hq, yap);
        sg.x = fmaf(cr[n], hq, sg.x);
        sg.y = fmaf(ci[n], hq, sg.y);
        sa.x = fmaf(cr[n], da, sa.x);
        sa.y = fmaf(ci[n], da, sa.y);
        sc.x = fmaf(cr[n], dc, sc.x);
        sc.y = fmaf(ci[n], dc, sc.y);
    }
    float sm, cm;
    sincos4(mid, &sm, &cm);
    auto rot = [&](float2 z) { return make_float2(cm * z.x - sm * z.y, cm * z.y + sm * z.x); };
    g = rot(sg);
    dlo = rot(sa);
    dhi = rot(sc);
}

// g = second divided difference of e^{ix} at t0, t1, t2, and dg/dlo, dg/dhi
// for the smallest and largest phase (dg/dmid = i g - dg/dlo - dg/dhi, since
// g(t + s) = e^{is} g(t)).
__device__ __forceinline__ void dd_grad(float t0, float t1, float t2, float2 &g, float2 &dlo,
                                        float2 &dhi) {
    const float lo = fminf(fminf(t0, t1), t2), hi = fmaxf(fmaxf(t0, t1), t2);
    const float mid = fmaxf(fminf(t0, t1), fminf(fmaxf(t0, t1), t2));
    const float D = hi - lo;
    {
        const float h1 = 0.5f * (mid - lo), h2 = 0.5f * (hi - mid);
        float s1, c1, s2, c2;
        sincos4(lo + h1, &s1, &c1);
        sincos4(mid + h2, &s2, &c2);
        // 1/max(h1,.5), 1/max(h2,.5), 1/max(D,.25) from one reciprocal
        const float a1 = fmaxf(h1, 0.5f), a2 = fmaxf(h2, 0.5f), Dg = fmaxf(D, 0.25f);
        const float p12 = a1 * a2;
        const float r = rcp4(p12 * Dg);
        const float rD = Dg * r, iD = p12 * r;
        float sc1, dsc1, sc2, dsc2;
        // the lanes that reach here vote; a lane that needs the series is among them
        const bool series = __any_sync(__activemask(), fminf(h1, h2) < 0.5f);
        sinc_d(h1, a2 * rD, series, sc1, dsc1);
        sinc_d(h2, a1 * rD, series, sc2, dsc2);
        // E = i e^{ic} sinc(h) = sc n with n = i e^{ic} = (-s, c); dE/dc = i E = sc (i n),
        // i n = (-c, -s); dE/dh = dsc n.  g = (E2 - E1) / D,
        // dg/dlo = (g - (iE1 - H1)/2) / D, dg/dhi = ((iE2 + H2)/2 - g) / D
        const float2 n1 = make_float2(-s1, c1), n2 = make_float2(-s2, c2);
        const float2 in1 = make_float2(-c1, -s1), in2 = make_float2(-c2, -s2);
        const float2 iD2 = bc2(iD);
        g = mul2(fma2(bc2(sc2), n2, mul2(bc2(-sc1), n1)), iD2);
        dlo = mul2(fma2(bc2(0.5f * dsc1), n1, fma2(bc2(-0.5f * sc1), in1, g)), iD2);
        dhi = mul2(fma2(bc2(0.5f * dsc2), n2, fma2(bc2(0.5f * sc2), in2, make_float2(-g.x, -g.y))), iD2);
    }
    if (D < 0.25f) dd_series(lo, mid, hi, g, dlo, dhi);
}

// dd_grad for the main bin step: D unguarded (below 0.25 the series about mid
// replaces g, dlo and dhi, and D < 0.25 puts both half gaps below 0.5, inside
// the warp's series branch), sinc and sinc' below h = 0.5 from minimax fits to
// their relative error on [0, 0.5] (Lawson's iteration; 1.2e-7 and 3.3e-8),
// and the outputs formed in scalar arithmetic.
__device__ __forceinline__ void dd_grad_main(float t0, float t1, float t2, float2 &g, float2 &dlo,
                                             float2 &dhi) {
    const float lo = fminf(fminf(t0, t1), t2), hi = fmaxf(fmaxf(t0, t1), t2);
    const float mid = fmaxf(fminf(t0, t1), fminf(fmaxf(t0, t1), t2));
    const float D = hi - lo;
    const float h1 = 0.5f * (mid - lo), h2 = 0.5f * (hi - mid);
    float s1, c1, s2, c2, sn1, cs1, sn2, cs2;
    sincos4(lo + h1, &s1, &c1);
    sincos4(mid + h2, &s2, &c2);
    sincos4(h1, &sn1, &cs1);
    sincos4(h2, &sn2, &cs2);
    // 1/max(h1,.5), 1/max(h2,.5) and 1/D from one reciprocal
    const float a1 = fmaxf(h1, 0.5f), a2 = fmaxf(h2, 0.5f);
    const float p12 = a1 * a2;
    const float r = rcp4(p12 * D);
    const float rD = D * r, iD = p12 * r;
    const float rh1 = a2 * rD, rh2 = a1 * rD;
    float sc1 = sn1 * rh1, sc2 = sn2 * rh2;
    float dsc1 = (cs1 - sc1) * rh1, dsc2 = (cs2 - sc2) * rh2;
    const bool series = __any_sync(__activemask(), fminf(h1, h2) < 0.5f);
    if (series) {
        const float x1 = h1 * h1, x2 = h2 * h2;
        if (h1 < 0.5f) {
            sc1 = fmaf(x1, fmaf(x1, 8.264339e-3f, -1.6666131e-1f), 1.0f);
            dsc1 = h1 * fmaf(x1, fmaf(x1, -1.1822202e-3f, 3.3332558e-2f), -3.3333332e-1f);
        }
        if (h2 < 0.5f) {
            sc2 = fmaf(x2, fmaf(x2, 8.264339e-3f, -1.6666131e-1f), 1.0f);
            dsc2 = h2 * fmaf(x2, fmaf(x2, -1.1822202e-3f, 3.3332558e-2f), -3.3333332e-1f);
        }
    }
    // E = i e^{ic} sinc(h) = sc n with n = (-s, c), i n = (-c, -s), dE/dh = dsc n:
    // g = (E2 - E1) / D, dg/dlo = (g - (iE1 - H1)/2) / D, dg/dhi = ((iE2 + H2)/2 - g) / D
    const float gx = iD * fmaf(sc1, s1, -sc2 * s2), gy = iD * fmaf(sc2, c2, -sc1 * c1);
    g = make_float2(gx, gy);
    dlo = make_float2(iD * fmaf(0.5f, fmaf(sc1, c1, -dsc1 * s1), gx),
                      iD * fmaf(0.5f, fmaf(dsc1, c1, sc1 * s1), gy));
    dhi = make_float2(iD * fmaf(-0.5f, fmaf(dsc2, s2, sc2 * c2), -gx),
                      iD * fmaf(0.5f, fmaf(dsc2, c2, -sc2 * s2), -gy));
    if (series && D < 0.25f) dd_series(lo, mid, hi, g, dlo, dhi);
}

// Bin direction from the facet centre in the aperture frame (second order in c/R)
struct Dir4 {
    float a, b, opa, opa2, w[3], k[3];
};
__device__ __forceinline__ Dir4 dir4(const K4Rec &r, float fx, float fy, float fz) {
    Dir4 d;
    d.a = fmaf(fz, r.eps[2], fmaf(fy, r.eps[1], fx * r.eps[0]));
    d.b = r.b;
    d.opa = 1.0f + d.a;
    d.opa2 = fmaf(d.a, fmaf(1.5f, d.a, 1.0f), fmaf(-0.5f, r.b, 1.0f));
    for (int i = 0; i < 3; i++) {
        d.w[i] = fmaf(r.R[3 * i + 2], fz, fmaf(r.R[3 * i + 1], fy, r.R[3 * i] * fx));
        d.k[i] = fmaf(d.w[i], d.opa2, -r.ea[i] * d.opa);
    }
    return d;
}

// Back-propagate a cotangent kb of the aperture-frame direction into the
// frame outer product and ea accumulators; returns the cotangents of
// a = u.c/R (ab) and b = |c|^2/R^2 (bb) for the caller's c terms.
__device__ __forceinline__ void dir4_back(const K4Rec &r, const Dir4 &d, const float kb[3], float fx,
                                          float fy, float fz, float *acc, float2 *accP, float &ab,
                                          float &bb) {
    const float2 u01 = make_float2(fx, fy);
    float opa2b = 0.0f, opab = 0.0f;
    for (int i = 0; i < 3; i++) {
        const float wb = kb[i] * d.opa2;
        opa2b = fmaf(kb[i], d.w[i], opa2b);
        opab = fmaf(-kb[i], r.ea[i], opab);
        accP[P_WU01 + i] = fma2(bc2(wb), u01, accP[P_WU01 + i]);
        acc[A_WU + 3 * i + 2] = fmaf(wb, fz, acc[A_WU + 3 * i + 2]);
        acc[A_EA + i] = fmaf(-kb[i], d.opa, acc[A_EA + i]);
    }
    ab = opab + opa2b * fmaf(3.0f, d.a, 1.0f);
    bb = -0.5f * opa2b;
}

// Cotangents through the polarisation block and the amplitudes: g_bar, A_bar
// and B_bar from the bin's cotangent G, and the amplitude sums.
__device__ __forceinline__ void w_back(const K4Rec &r, const Bin4 &B, float2 g, float A, float Bm,
                                       float2 *accA, float2 &gb, float &Ab, float &Bb) {
    const float2 *u = reinterpret_cast<const float2 *>(r.amp);
    // H conj(u) = Re(u) H + Im(u) (-i H)
    const float2 Sp = fma2(bc2(u[0].x), B.G[0], fma2(bc2(u[0].y), B.Gm[0],
                           fma2(bc2(u[2].x), B.G[2], mul2(bc2(u[2].y), B.Gm[2]))));
    const float2 Sn = fma2(bc2(u[1].x), B.G[1], fma2(bc2(u[1].y), B.Gm[1],
                           fma2(bc2(u[3].x), B.G[3], mul2(bc2(u[3].y), B.Gm[3]))));
    const float2 Ss = add2(Sp, Sn), Sd = sub2(Sp, Sn);
    gb = make_float2(fmaf(A, Ss.x, -Bm * Sd.y), fmaf(A, Ss.y, Bm * Sd.x));
    Ab = fmaf(g.x, Ss.x, g.y * Ss.y);
    Bb = fmaf(g.y, Sd.x, -g.x * Sd.y);
    {
        const float gyB = g.y * Bm, gyA = g.y * A;
        // conj(g z+) and conj(g z-); H w = Re(w) H - Im(w) (-i H)
        const float wpr = fmaf(g.x, A, gyB), wpi = fmaf(g.x, Bm, -gyA);
        const float wnr = fmaf(g.x, A, -gyB), wni = fmaf(-g.x, Bm, -gyA);
        accA[0] = fma2(bc2(wpr), B.G[0], fma2(bc2(-wpi), B.Gm[0], accA[0]));
        accA[1] = fma2(bc2(wnr), B.G[1], fma2(bc2(-wni), B.Gm[1], accA[1]));
        accA[2] = fma2(bc2(wpr), B.G[2], fma2(bc2(-wpi), B.Gm[2], accA[2]));
        accA[3] = fma2(bc2(wnr), B.G[3], fma2(bc2(-wni), B.Gm[3], accA[3]));
    }
}

// Cotangents of the phases t_j, the aperture wave vector and the bin direction,
// given those of kx, ky, kz from the polarisation block (kxb, kyb, kzb).
__device__ __forceinline__ void phase_back(const K4Rec &r, const Bin4 &B, const Dir4 &d, float2 g,
                                           float2 dlo, float2 dhi, float2 gb, const float (&t)[3],
                                           float kxx, float kyy, float kxb, float kyb, float kzb,
                                           float k, float hkR, float iRf, float *acc, float2 *accP) {
    // phases: t_j = ph + kxx xa_j + kyy ya_j.  t_bar = Re(conj(g_bar) dg/dt),
    // assigned by rank (ties broken by index); phb = sum_j t_bar_j = Re(conj(g_bar) i g).
    const float tlo = fmaf(gb.x, dlo.x, gb.y * dlo.y), thi = fmaf(gb.x, dhi.x, gb.y * dhi.y);
    const float phb = fmaf(gb.y, g.x, -gb.x * g.y);
    const float tmid = phb - tlo - thi;
    // rank 0 (lowest) / 2 (highest) of each t_j, ties broken by index
    const bool c01 = t[1] < t[0], c02 = t[2] < t[0], c12 = t[2] < t[1];
    const bool is_lo[3] = {!c01 && !c02, c01 && !c12, c02 && c12};
    const bool is_hi[3] = {c01 && c02, !c01 && c12, !c02 && !c12};
    float kxxb = 0.0f, kyyb = 0.0f;
    const float2 kk2 = make_float2(kxx, kyy);
#pragma unroll
    for (int j = 0; j < 3; j++) {
        const float tb = is_lo[j] ? tlo : (is_hi[j] ? thi : tmid);
        kxxb = fmaf(tb, r.xa[j], kxxb);
        kyyb = fmaf(tb, r.ya[j], kyyb);
        accP[P_TK + j] = fma2(bc2(tb), kk2, accP[P_TK + j]);
    }
    // kxx = k p2x - k kx ; kyy = k p2y - k ky
    kxb = fmaf(-k, kxxb, kxb);
    kyb = fmaf(-k, kyyb, kyb);
    acc[A_P2 + 0] += kxxb;  // times k after the loop
    acc[A_P2 + 1] += kyyb;
    const float kb3[3] = {kxb, kyb, kzb};
    float ab, bb;
    dir4_back(r, d, kb3, B.fx, B.fy, B.fz, acc, accP, ab, bb);
    // ph = hkR (b - a^2)(1 + a) - rf with rf = k u.c (mod 2 pi), a = u.c/R, b = |c|^2/R^2:
    // c_bar = (ab + phb dph/da) u / R - phb k u + (bb + phb dph/db) 2 c / R^2
    const float dpa = hkR * fmaf(-2.0f * d.a, d.opa, fmaf(-d.a, d.a, r.b));
    const float dpb = hkR * d.opa;
    const float cu = fmaf(fmaf(phb, dpa, ab), iRf, -k * phb);
    acc[A_CU + 0] = fmaf(cu, B.fx, acc[A_CU + 0]);
    acc[A_CU + 1] = fmaf(cu, B.fy, acc[A_CU + 1]);
    acc[A_CU + 2] = fmaf(cu, B.fz, acc[A_CU + 2]);
    acc[A_CE] += fmaf(phb, dpb, bb);
}

// The bin step outside the clamps and the forward bodge (a bin away from the
// poles, |ky| <= 0.999999 and kx^2 + kz^2 above the floor): the general step
// below with kyc = ky, tt = kx^2 + kz^2 and q = k, its branches left out.
__device__ __forceinline__ void k4_main(const K4Rec &r, const Bin4 &B, const Dir4 &d, float kx,
                                        float ky, float kz, float kxx, float kyy,
                                        const float (&t)[3], float tt, float k, float hkR,
                                        float iRf, float *acc, float2 *accA, float2 *accP) {
    float2 g, dlo, dhi;
    dd_grad_main(t[0], t[1], t[2], g, dlo, dhi);
    const float rs = rsqrt4(tt), s = tt * rs;
    const float e = rs * r.hicf, kxky = kx * ky;
    const float dd = fmaf(r.kw1, s, -kz * e);
    const float ee = fmaf(r.kw2, s, -kxky * e);
    const float hr[3] = {fmaf(r.inc[1], kz, -r.inc[2] * ky), fmaf(r.inc[2], kx, -r.inc[0] * kz),
                         fmaf(r.inc[0], ky, -r.inc[1] * kx)};
    const float hn = rsqrt4(fmaf(hr[2], hr[2], fmaf(hr[1], hr[1], hr[0] * hr[0])));
    // hr is normal to k and |k| = 1 to third order in |c|/R, so the general
    // p = hn (hr1 s - (ky/s) hr . (kx, 0, kz)) is hn hr1 / s, the forward kernel's
    // form; rr = hn (hr2 kx - hr0 kz) / s.
    const float f = hn * rs;
    const float R0 = fmaf(hr[2], kx, -hr[0] * kz);
    const float pp = f * hr[1], rr = f * R0;
    const float A = fmaf(pp, dd, rr * ee), Bm = fmaf(pp, ee, -rr * dd);
    float2 gb;
    float Ab, Bb;
    w_back(r, B, g, A, Bm, accA, gb, Ab, Bb);
    const float ppb = fmaf(Ab, dd, Bb * ee), rrb = fmaf(Ab, ee, -Bb * dd);
    const float ddb = fmaf(Ab, pp, -Bb * rr), eeb = fmaf(Ab, rr, Bb * pp);
    // f = hn rs: f_bar = pp_bar hr1 + rr_bar R0; hn_bar = f_bar rs, rs_bar = f_bar hn
    const float fb = fmaf(ppb, hr[1], rrb * R0);
    const float R0b = rrb * f;
    const float hn3 = -(fb * rs) * (hn * hn * hn);  // d hn / d hr_i = -hn^3 hr_i
    const float hrb[3] = {fmaf(-R0b, kz, hn3 * hr[0]), fmaf(ppb, f, hn3 * hr[1]),
                          fmaf(R0b, kx, hn3 * hr[2])};
    float kxb = R0b * hr[2];
    float kzb = -R0b * hr[0];
    float kyb = 0.0f;
    const float sbm = -(fb * hn) * (rs * rs);  // rs = 1/s
    // h = inc x k
    kxb += hrb[1] * r.inc[2] - hrb[2] * r.inc[1];
    kyb += hrb[2] * r.inc[0] - hrb[0] * r.inc[2];
    kzb += hrb[0] * r.inc[1] - hrb[1] * r.inc[0];
    acc[A_INC + 0] += ky * hrb[2] - kz * hrb[1];
    acc[A_INC + 1] += kz * hrb[0] - kx * hrb[2];
    acc[A_INC + 2] += kx * hrb[1] - ky * hrb[0];
    // Karczewski-Wolf dd, ee (see k4_eval)
    const float dde = ddb * e, eee = eeb * e;
    kxb = fmaf(-eee, ky, kxb);
    kyb = fmaf(-eee, kx, kyb);
    kzb -= dde;
    const float X = fmaf(dde, kz, eee * kxky);
    const float sb = sbm + fmaf(ddb, r.kw1, fmaf(eeb, r.kw2, rs * X));
    acc[A_P2 + 2] = fmaf(ddb, s, acc[A_P2 + 2]);
    accP[P_KW].x = fmaf(eeb, s, accP[P_KW].x);
    accP[P_KW].y += X;
    const float ttb = 0.5f * sb * rs;  // s = sqrt(tt)
    kxb = fmaf(2.0f * kx, ttb, kxb);
    kzb = fmaf(2.0f * kz, ttb, kzb);
    phase_back(r, B, d, g, dlo, dhi, gb, t, kxx, kyy, kxb, kyb, kzb, k, hkR, iRf, acc, accP);
}

// Cotangent contributions of one (record, bin).
template <bool FAST>
__device__ __forceinline__ void k4_eval(const K4Rec &r, const Bin4 &B, float k, float hkR, float iRf,
                                        float cosfov, const float *p0, const K4Bin *__restrict__ bins,
                                        int64_t nphi, int64_t theta_i, float *acc, float2 *accA,
                                        float2 *accP) {
    // forward
    const double ka = fma(B.uz, r.kc[2], fma(B.uy, r.kc[1], B.ux * r.kc[0]));
    const double nq = fma(ka, kInv2Pi4, kMagic4) - kMagic4;
    const float rf = (float)fma(-nq, kTwoPi4, ka);
    const Dir4 d = dir4(r, B.fx, B.fy, B.fz);
    if (FAST) {
        const float dx = fmaf(B.fx, d.opa, -r.eps[0]), dy = fmaf(B.fy, d.opa, -r.eps[1]),
                    dz = fmaf(B.fz, d.opa, -r.eps[2]);
        if (fmaf(dz, p0[2], fmaf(dy, p0[1], dx * p0[0])) < cosfov) return;
    }
    const float ph = fmaf(hkR * fmaf(-d.a, d.a, r.b), d.opa, -rf);
    const float kx = d.k[0], ky = d.k[1], kz = d.k[2];
    const float kxx = fmaf(-k, kx, r.kp[0]), kyy = fmaf(-k, ky, r.kp[1]);
    float t[3];
    for (int j = 0; j < 3; j++) t[j] = fmaf(kyy, r.ya[j], fmaf(kxx, r.xa[j], ph));
    {
        const float tr = fmaf(kx, kx, kz * kz);
        if (!B.pole && tr > kClampSq4 && fabsf(ky) <= 0.999999f) {
            k4_main(r, B, d, kx, ky, kz, kxx, kyy, t, tr, k, hkR, iRf, acc, accA, accP);
            return;
        }
    }
    float2 g, dlo, dhi;
    dd_grad(t[0], t[1], t[2], g, dlo, dhi);
    const bool yclamp = !(fabsf(ky) <= 0.999999f);
    const float kyc = fminf(fmaxf(ky, -0.999999f), 0.999999f);
    const float traw = fmaf(kx, kx, kz * kz);
    const bool floored = !(traw > kClampSq4);
    const float tt = floored ? kClampSq4 : traw;
    const float rs = rsqrt4(tt), s = tt * rs;
    const float kyrs = kyc * rs;
    const float m[3] = {-kx * kyrs, s, -kz * kyrs};
    // dd = -Kz cf s / 2 - kz icf / (2 s), ee = Kx Ky cf s / 2 - kx ky icf / (2 s)
    const float e = rs * r.hicf, kxkyc = kx * kyc;
    const float dd = fmaf(r.kw1, s, -kz * e);
    const float ee = fmaf(r.kw2, s, -kxkyc * e);
    const float kc3[3] = {kx, kyc, kz};
    // the forward bodge (src/diff_mod.f90:630-633) can apply only in bins near the poles
    bool bodge = false;
    if (B.pole) {
        const float dinc = fmaf(r.inc[2], kz, fmaf(r.inc[1], kyc, r.inc[0] * kx));
        bodge = !(fabsf(dinc) < 0.999f);
    }
    Dir4 dh;
    float q[3] = {kx, kyc, kz};
    float hx = 0.0f, hy = 0.0f, hz = 0.0f;
    if (bodge) {
        const K4Bin hb = bins[B.o % nphi + nphi * theta_i];
        hx = (float)hb.ux;
        hy = (float)hb.uy;
        hz = (float)hb.uz;
        dh = dir4(r, hx, hy, hz);
        q[0] = dh.k[0];
        q[1] = dh.k[1];
        q[2] = dh.k[2];
    }
    const float hr[3] = {fmaf(r.inc[1], q[2], -r.inc[2] * q[1]), fmaf(r.inc[2], q[0], -r.inc[0] * q[2]),
                         fmaf(r.inc[0], q[1], -r.inc[1] * q[0])};
    const float hn = rsqrt4(fmaf(hr[2], hr[2], fmaf(hr[1], hr[1], hr[0] * hr[0])));
    // p = hc.m, rr = hc.evo2 with hc = hr hn.  Inside the clamp k is a unit
    // vector and evo2 = k x m = (-kz, 0, kx) / s, so p = hn (hy s - ky T1 / s),
    // T1 = hx kx + hz kz, and rr = hn (hz kx - hx kz) / s.
    float pp, rr, T1 = 0.0f, P0 = 0.0f, R0 = 0.0f;
    float hc[3], ev[3], vn = 1.0f;
    if (!floored) {
        T1 = fmaf(hr[0], kx, hr[2] * kz);
        P0 = fmaf(hr[1], s, -kyrs * T1);
        R0 = fmaf(hr[2], kx, -hr[0] * kz);
        pp = hn * P0;
        rr = hn * rs * R0;
    } else {
        for (int i = 0; i < 3; i++) hc[i] = hr[i] * hn;
        const float vr[3] = {fmaf(kyc, m[2], -kz * m[1]), fmaf(kz, m[0], -kx * m[2]),
                             fmaf(kx, m[1], -kyc * m[0])};
        vn = rsqrt4(fmaf(vr[2], vr[2], fmaf(vr[1], vr[1], vr[0] * vr[0])));
        for (int i = 0; i < 3; i++) ev[i] = vr[i] * vn;
        pp = fmaf(hc[2], m[2], fmaf(hc[1], m[1], hc[0] * m[0]));
        rr = fmaf(hc[2], ev[2], fmaf(hc[1], ev[1], hc[0] * ev[0]));
    }
    const float A = fmaf(pp, dd, rr * ee), Bm = fmaf(pp, ee, -rr * dd);
    // W = [[A, B], [-B, A]] amp' is diagonal in the circular basis:
    // W1j +- i W2j = z+- u+-_j with z+ = A - iB, z- = A + iB.  With the cotangent
    // H+-_j of the same basis and S+- = sum_j H+-_j conj(u+-_j):
    //   g_bar = conj(z+) S+ + conj(z-) S- = A (S+ + S-) + i B (S+ - S-)
    //   A_bar = Re conj(g) (S+ + S-),  B_bar = Im conj(g) (S- - S+)
    //   u+-_j_bar = H+-_j conj(g z+-)
    float2 gb;
    float Ab, Bb;
    w_back(r, B, g, A, Bm, accA, gb, Ab, Bb);
    // A = pp dd + rr ee, B = pp ee - rr dd
    const float ppb = fmaf(Ab, dd, Bb * ee), rrb = fmaf(Ab, ee, -Bb * dd);
    const float ddb = fmaf(Ab, pp, -Bb * rr), eeb = fmaf(Ab, rr, Bb * pp);
    float hrb[3], kxb, kycb, kzb, sbm;  // sbm: cotangent of s from p and rr
    if (!floored) {
        const float Pb = ppb * hn, Rb = rrb * hn * rs;
        const float hn3 = -fmaf(ppb, P0, rrb * rs * R0) * hn * hn * hn;
        const float T1b = -Pb * kyrs;
        hrb[0] = fmaf(T1b, kx, fmaf(-Rb, kz, hn3 * hr[0]));
        hrb[1] = fmaf(Pb, s, hn3 * hr[1]);
        hrb[2] = fmaf(T1b, kz, fmaf(Rb, kx, hn3 * hr[2]));
        kxb = fmaf(T1b, hr[0], Rb * hr[2]);
        kzb = fmaf(T1b, hr[2], -Rb * hr[0]);
        kycb = -Pb * rs * T1;
        sbm = fmaf(Pb, fmaf(kyc * T1, rs * rs, hr[1]), -Rb * R0 * rs);
    } else {
        float hcb[3], mb[3], evb[3];
        for (int i = 0; i < 3; i++) {
            hcb[i] = fmaf(ppb, m[i], rrb * ev[i]);
            mb[i] = ppb * hc[i];
            evb[i] = rrb * hc[i];
        }
        // ev = vr * vn ; vr = kc3 x m
        float vrb[3];
        {
            const float dp = evb[0] * ev[0] + evb[1] * ev[1] + evb[2] * ev[2];
            for (int i = 0; i < 3; i++) vrb[i] = (evb[i] - dp * ev[i]) * vn;
        }
        kxb = m[1] * vrb[2] - m[2] * vrb[1];
        kycb = m[2] * vrb[0] - m[0] * vrb[2];
        kzb = m[0] * vrb[1] - m[1] * vrb[0];
        mb[0] += vrb[1] * kc3[2] - vrb[2] * kc3[1];
        mb[1] += vrb[2] * kc3[0] - vrb[0] * kc3[2];
        mb[2] += vrb[0] * kc3[1] - vrb[1] * kc3[0];
        // hc = hr * hn
        const float dp = hcb[0] * hc[0] + hcb[1] * hc[1] + hcb[2] * hc[2];
        for (int i = 0; i < 3; i++) hrb[i] = (hcb[i] - dp * hc[i]) * hn;
        // m = (-kx kyc rs, s, -kz kyc rs)
        kxb += mb[0] * (-kyrs);
        kycb += mb[0] * (-kx * rs) + mb[2] * (-kz * rs);
        kzb += mb[2] * (-kyrs);
        sbm = mb[0] * (kx * kyrs * rs) + mb[2] * (kz * kyrs * rs) + mb[1];
    }
    float qb[3];
    qb[0] = hrb[1] * r.inc[2] - hrb[2] * r.inc[1];
    qb[1] = hrb[2] * r.inc[0] - hrb[0] * r.inc[2];
    qb[2] = hrb[0] * r.inc[1] - hrb[1] * r.inc[0];
    acc[A_INC + 0] += q[1] * hrb[2] - q[2] * hrb[1];
    acc[A_INC + 1] += q[2] * hrb[0] - q[0] * hrb[2];
    acc[A_INC + 2] += q[0] * hrb[1] - q[1] * hrb[0];
    if (bodge) {
        float abh, bbh;
        dir4_back(r, dh, qb, hx, hy, hz, acc, accP, abh, bbh);
        const float ch = abh * iRf;
        acc[A_CU + 0] = fmaf(ch, hx, acc[A_CU + 0]);
        acc[A_CU + 1] = fmaf(ch, hy, acc[A_CU + 1]);
        acc[A_CU + 2] = fmaf(ch, hz, acc[A_CU + 2]);
        acc[A_CE] += bbh;
    } else {
        kxb += qb[0];
        kycb += qb[1];
        kzb += qb[2];
    }
    // Karczewski-Wolf dd, ee as above.  With X = (dd_bar kz + ee_bar kx ky) e:
    //   s_bar += kw1 dd_bar + kw2 ee_bar + X / s
    //   p2_bar: z -cf/2 dd_bar s, x Ky cf/2 ee_bar s,
    //           y Kx cf/2 ee_bar s + Ky cf^2 (kw1 dd_bar s + kw2 ee_bar s + X)
    // (cf = 1/sqrt(1 - Ky^2)); the bin sums of dd_bar s, ee_bar s and X are
    // scaled by the record's constants after the loop.
    const float dde = ddb * e, eee = eeb * e;
    kxb = fmaf(-eee, kyc, kxb);
    kycb = fmaf(-eee, kx, kycb);
    kzb -= dde;
    const float X = fmaf(dde, kz, eee * kxkyc);
    const float sb = sbm + fmaf(ddb, r.kw1, fmaf(eeb, r.kw2, rs * X));
    acc[A_P2 + 2] = fmaf(ddb, s, acc[A_P2 + 2]);
    accP[P_KW].x = fmaf(eeb, s, accP[P_KW].x);
    accP[P_KW].y += X;
    if (!floored) {
        const float ttb = 0.5f * sb * rs;  // s = sqrt(tt)
        kxb = fmaf(2.0f * kx, ttb, kxb);
        kzb = fmaf(2.0f * kz, ttb, kzb);
    }
    float kyb = yclamp ? 0.0f : kycb;
    phase_back(r, B, d, g, dlo, dhi, gb, t, kxx, kyy, kxb, kyb, kzb, k, hkR, iRf, acc, accP);
}

// One warp per record, K4_WARPS records per CTA; blockIdx.y selects a range
// of bins.  Each lane walks the range with stride 32 and keeps the 36 sums of
// its record in registers (FP32, at most K4_MAX_LANE_BINS terms), so the warp
// reduction and the FP64 atomic into out[record][36] happen once per
// (record, range).  The warps of a CTA walk the same bins, which the L1 serves.
template <bool FAST, int MINB>
__global__ void __launch_bounds__(K4_WARPS * 32, MINB) k4_adjoint_kernel(
    const K4Rec *__restrict__ recs, const int *__restrict__ kinds, const float *__restrict__ fovdat,
    int64_t nrec, const K4Bin *__restrict__ bins, const float4 *__restrict__ gbin, int64_t nb,
    int64_t nphi, int64_t theta_i, int64_t chunk, float k, float hkR, float iRf, float pole_cos,
    double *__restrict__ out) {
    __shared__ K4Rec s_rec[K4_WARPS];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t rec = (int64_t)blockIdx.x * K4_WARPS + warp;
    if (rec >= nrec) return;  // whole warp; no block-wide barrier follows
    {
        const float *src = reinterpret_cast<const float *>(recs + rec);
        float *dst = reinterpret_cast<float *>(&s_rec[warp]);
        for (int i = lane; i < (int)(sizeof(K4Rec) / 4); i += 32) dst[i] = src[i];
        __syncwarp();
    }
    const K4Rec &r = s_rec[warp];
    const int kd = kinds[rec];
    const float4 *G = gbin + (int64_t)kd * 2 * nb;
    float cosfov = 0.0f, p0[3] = {0.0f, 0.0f, 0.0f};
    if (FAST) {
        p0[0] = fovdat[4 * rec];
        p0[1] = fovdat[4 * rec + 1];
        p0[2] = fovdat[4 * rec + 2];
        cosfov = fovdat[4 * rec + 3];
    }
    float acc[K4_NACC];
    float2 accA[4], accP[K4_NPAIR];
#pragma unroll
    for (int q = 0; q < K4_NACC; q++) acc[q] = 0.0f;
#pragma unroll
    for (int q = 0; q < K4_NPAIR; q++) accP[q] = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int q = 0; q < 4; q++) accA[q] = make_float2(0.0f, 0.0f);
    const int64_t o0 = (int64_t)blockIdx.y * chunk, o1 = min(nb, o0 + chunk);
    for (int64_t o = o0 + lane; o < o1; o += 32) {
        Bin4 B;
        const double2 *pb = reinterpret_cast<const double2 *>(bins + o);
        const double2 q0 = pb[0], q1 = pb[1];
        B.ux = q0.x;
        B.uy = q0.y;
        B.uz = q1.x;
        B.fx = (float)B.ux;
        B.fy = (float)B.uy;
        B.fz = (float)B.uz;
        B.pole = !(fabs(B.uz) < (double)pole_cos);
        B.o = o;
        const float4 *pg = G + 2 * o;
        const float4 g0 = pg[0], g1 = pg[1];
        B.G[0] = make_float2(g0.x, g0.y);
        B.G[1] = make_float2(g0.z, g0.w);
        B.G[2] = make_float2(g1.x, g1.y);
        B.G[3] = make_float2(g1.z, g1.w);
#pragma unroll
        for (int c = 0; c < 4; c++) B.Gm[c] = make_float2(B.G[c].y, -B.G[c].x);
        k4_eval<FAST>(r, B, k, hkR, iRf, cosfov, p0, bins, nphi, theta_i, acc, accA, accP);
    }
    // amplitude sums back from the circular basis: a1j_bar = u+_j_bar + u-_j_bar,
    // a2j_bar = i (u-_j_bar - u+_j_bar)
#pragma unroll
    for (int j = 0; j < 2; j++) {
        const float2 up = accA[2 * j], un = accA[2 * j + 1];
        acc[A_AMP + 4 * j] = up.x + un.x;
        acc[A_AMP + 4 * j + 1] = up.y + un.y;
        acc[A_AMP + 4 * j + 2] = up.y - un.y;
        acc[A_AMP + 4 * j + 3] = un.x - up.x;
    }
#pragma unroll
    for (int j = 0; j < 3; j++) {
        acc[A_TKX + j] = accP[P_TK + j].x;
        acc[A_TKY + j] = accP[P_TK + j].y;
        acc[A_WU + 3 * j] += accP[P_WU01 + j].x;
        acc[A_WU + 3 * j + 1] += accP[P_WU01 + j].y;
    }
    {
        // A_P2 held (sum kxx_bar, sum kyy_bar, sum dd_bar s) and P_KW (sum ee_bar s, sum X)
        const float cf = r.cf, Kx = r.p2[0], Ky = r.p2[1];
        const float q1 = acc[A_P2 + 2], q2 = accP[P_KW].x, q3 = accP[P_KW].y;
        acc[A_P2 + 0] = fmaf(k, acc[A_P2 + 0], 0.5f * Ky * cf * q2);
        acc[A_P2 + 1] = fmaf(k, acc[A_P2 + 1],
                             fmaf(0.5f * Kx * cf, q2, Ky * cf * cf * fmaf(r.kw1, q1, fmaf(r.kw2, q2, q3))));
        acc[A_P2 + 2] = -0.5f * cf * q1;
    }
#pragma unroll
    for (int q = 0; q < K4_NACC; q++) {
        float v = acc[q];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if (lane == (q & 31)) atomicAdd(&out[rec * K4_NACC + q], (double)v);
    }
}

// Per-bin inputs of the adjoint: the unit bin direction (FP64) and the
// cotangent of S' (pre-T, common phase removed): G' = conj(e^{ik|X|}) G T^T,
// per kind.
__global__ void k4_prep_kernel(const double *__restrict__ gafb, const double *__restrict__ gafe,
                               const double *__restrict__ xyz, const double *__restrict__ phitab,
                               int64_t nb, int64_t nphi, double k, K4Bin *__restrict__ bins,
                               float4 *__restrict__ gbin) {
    const int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= nb) return;
    const double cp = phitab[o % nphi], sp = phitab[nphi + o % nphi];
    const double X = xyz[o], Y = xyz[nb + o], Zc = xyz[2 * nb + o];
    const double rho = sqrt(X * X + Y * Y + Zc * Zc), ir = 1.0 / rho;
    K4Bin bn;
    bn.ux = X * ir;
    bn.uy = Y * ir;
    bn.uz = Zc * ir;
    bn.pad = 0.0;
    bins[o] = bn;
    double sK, cK;
    sincos(k * rho, &sK, &cK);
    const double T11 = -sp, T12 = -cp, T21 = cp, T22 = -sp;
    for (int kd = 0; kd < 2; kd++) {
        const double *Gc = kd ? gafe : gafb;
        double gr[4], gi[4];  // (1,1),(2,1),(1,2),(2,2), times conj(e^{iK})
        for (int c = 0; c < 4; c++) {
            const double re = Gc[2 * (o + nb * c)], im = Gc[2 * (o + nb * c) + 1];
            gr[c] = re * cK + im * sK;
            gi[c] = im * cK - re * sK;
        }
        // S = S' T  ->  S'_bar = S_bar T^T : S'(a,1) <- S(a,1) T11 + S(a,2) T12, S'(a,2) <- S(a,1) T21 + S(a,2) T22
        const double o11r = gr[0] * T11 + gr[2] * T12, o11i = gi[0] * T11 + gi[2] * T12;
        const double o21r = gr[1] * T11 + gr[3] * T12, o21i = gi[1] * T11 + gi[3] * T12;
        const double o12r = gr[0] * T21 + gr[2] * T22, o12i = gi[0] * T21 + gi[2] * T22;
        const double o22r = gr[1] * T21 + gr[3] * T22, o22i = gi[1] * T21 + gi[3] * T22;
        // in the circular basis of the columns: H+-_j = (G1j +- i G2j) / 2
        float4 *dst = gbin + (kd * nb + o) * 2;
        dst[0] = make_float4((float)(0.5 * (o11r - o21i)), (float)(0.5 * (o11i + o21r)),
                             (float)(0.5 * (o11r + o21i)), (float)(0.5 * (o11i - o21r)));
        dst[1] = make_float4((float)(0.5 * (o12r - o22i)), (float)(0.5 * (o12i + o22r)),
                             (float)(0.5 * (o12r + o22i)), (float)(0.5 * (o12i - o22r)));
    }
}

// Per-record data of the FP64 mapping: centre, vertex offsets, frame,
// propagation direction, signed area, anti-parallel sign, vertex indices.
struct Host4 {
    double c[3], e[3][3], R[3][3], p[3], As, sign;
    int64_t vi[3];
};

// Thread per record (beam outbeams, then external diffraction): the FP64
// set-up of the kernel record K4Rec (frame, aperture-frame vertices, the
// constants of the bin loop, the circular-basis amplitudes), of the
// field-of-view data and of the mapping data Host4.
__global__ void k4_setup_kernel(const pbt_outbeam *__restrict__ beam, int64_t nbeam,
                                const pbt_outbeam *__restrict__ ext, int64_t nrec,
                                const double *__restrict__ verts, int64_t nverts,
                                const int64_t *__restrict__ face_off, const int64_t *__restrict__ face_vi,
                                double k, double lambda, K4Rec *__restrict__ recs, int *__restrict__ kinds,
                                float *__restrict__ fovd, Host4 *__restrict__ H) {
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nrec) return;
    const double Rf = kFarR;
        const pbt_outbeam &ob = q < nbeam ? beam[q] : ext[q - nbeam];
        const int64_t fb = face_off[ob.fi - 1];
        double vx[3], vy[3], vz[3], rx[3], ry[3], rz[3];
        for (int i = 0; i < 3; i++) {
            const int64_t vi = face_vi[fb + i] - 1;
            H[q].vi[i] = vi;
            vx[i] = verts[vi];
            vy[i] = verts[vi + nverts];
            vz[i] = verts[vi + 2 * nverts];
        }
        FacetFrame fr;
        fr.sign = 1.0;
        facet_frame(vx, vy, vz, 3, ob.prop_out, ob.vk7, fr, rx, ry, rz);
        K4Rec &r = recs[q];
        Host4 &h = H[q];
        kinds[q] = q < nbeam ? 0 : 1;
        double ea[3], xa[3], ya[3];
        mv33(fr.R, fr.com, ea);
        for (int i = 0; i < 3; i++) {
            const double d[3] = {rx[i], ry[i], rz[i]};
            double a3[3];
            mv33(fr.R, d, a3);
            xa[i] = a3[0];
            ya[i] = a3[1];
            h.e[i][0] = rx[i];
            h.e[i][1] = ry[i];
            h.e[i][2] = rz[i];
        }
        const double As = 0.5 * ((xa[1] - xa[0]) * (ya[2] - ya[0]) - (xa[2] - xa[0]) * (ya[1] - ya[0]));
        const double cpre = 2.0 * As / lambda * fr.sign;
        for (int c = 0; c < 3; c++) {
            r.kc[c] = k * fr.com[c];
            r.eps[c] = (float)(fr.com[c] / Rf);
            r.ea[c] = (float)(ea[c] / Rf);
            r.p2[c] = (float)fr.prop2[c];
            r.inc[c] = (float)fr.inc2[c];
            r.xa[c] = (float)xa[c];
            r.ya[c] = (float)ya[c];
            h.c[c] = fr.com[c];
            h.p[c] = ob.prop_out[c];
        }
        r.b = (float)((fr.com[0] * fr.com[0] + fr.com[1] * fr.com[1] + fr.com[2] * fr.com[2]) / (Rf * Rf));
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) {
                r.R[3 * a + b] = (float)fr.R.m[a][b];
                h.R[a][b] = fr.R.m[a][b];
            }
        r.kp[0] = (float)(k * fr.prop2[0]);
        r.kp[1] = (float)(k * fr.prop2[1]);
        r.cf = (float)(1.0 / sqrt(1.0 - fr.prop2[1] * fr.prop2[1]));
        r.icf = (float)sqrt(1.0 - fr.prop2[1] * fr.prop2[1]);
        {
            const double cfd = 1.0 / sqrt(1.0 - fr.prop2[1] * fr.prop2[1]);
            r.kw1 = (float)(-0.5 * fr.prop2[2] * cfd);
            r.kw2 = (float)(0.5 * fr.prop2[0] * fr.prop2[1] * cfd);
            r.hicf = (float)(0.5 * sqrt(1.0 - fr.prop2[1] * fr.prop2[1]));
        }
        {
            // amp' = (2 i A / lambda) sign ampl in the order (1,1),(2,1),(1,2),(2,2),
            // stored as the columns in the circular basis u+-_j = a1j +- i a2j:
            // u+_1, u-_1, u+_2, u-_2
            double am[8];
            for (int c = 0; c < 4; c++) {
                am[2 * c] = -cpre * ob.ampl[2 * c + 1];
                am[2 * c + 1] = cpre * ob.ampl[2 * c];
            }
            const double uc[8] = {am[0] - am[3], am[1] + am[2], am[0] + am[3], am[1] - am[2],
                                  am[4] - am[7], am[5] + am[6], am[4] + am[7], am[5] - am[6]};
            for (int c = 0; c < 8; c++) r.amp[c] = (float)uc[c];
        }
        h.As = As;
        h.sign = fr.sign;
        const double fov = q < nbeam ? ob.fov : kPiRef / 2.0;
        fovd[4 * q + 0] = (float)ob.prop_out[0];
        fovd[4 * q + 1] = (float)ob.prop_out[1];
        fovd[4 * q + 2] = (float)ob.prop_out[2];
        fovd[4 * q + 3] = (float)cos(fov);
    }

// Thread per record: the record's 36 sums mapped through the frame
// construction (z = -n, x = unit(p - (p.n) n), y = z x x, n = unit(e0 x e1),
// c = mean(v)) to its three vertices (added with FP64 atomics) and to its
// amplitude (gamp: 8 doubles, the outbeam's ampl order).
__global__ void k4_map_kernel(const double *__restrict__ acc, const Host4 *__restrict__ H,
                              const pbt_outbeam *__restrict__ beam, int64_t nbeam,
                              const pbt_outbeam *__restrict__ ext, int64_t nrec, double lambda,
                              int64_t nverts, double *__restrict__ gbeam, double *__restrict__ gext,
                              double *__restrict__ gverts) {
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nrec) return;
    const double Rf = kFarR;
    const double inc[3] = {0, 0, -1};
        const double *A = &acc[q * K4_NACC];
        const Host4 &h = H[q];
        const pbt_outbeam &ob = q < nbeam ? beam[q] : ext[q - nbeam];
        // amplitude: amp' = i cpre ampl -> ampl_bar = conj(i cpre) amp'_bar = -i cpre amp'_bar
        const double cpre = 2.0 * h.As / lambda * h.sign;
        double *ga = q < nbeam ? gbeam + 8 * q : gext + 8 * (q - nbeam);
        double Asb = 0.0;  // d amp' / d As = i (2 sign / lambda) ampl
        for (int c = 0; c < 4; c++) {
            const double br = A[A_AMP + 2 * c], bi = A[A_AMP + 2 * c + 1];
            ga[2 * c] = cpre * bi;
            ga[2 * c + 1] = -cpre * br;
            // Re(conj(amp'_bar) * i (2 sign/lambda) ampl)
            const double ar = ob.ampl[2 * c], ai = ob.ampl[2 * c + 1];
            Asb += (2.0 * h.sign / lambda) * (br * (-ai) + bi * ar);
        }
        // aperture coordinates xa_j = x.e_j, ya_j = y.e_j
        double xab[3], yab[3];
        double xa[3], ya[3];
        for (int j = 0; j < 3; j++) {
            xa[j] = h.R[0][0] * h.e[j][0] + h.R[0][1] * h.e[j][1] + h.R[0][2] * h.e[j][2];
            ya[j] = h.R[1][0] * h.e[j][0] + h.R[1][1] * h.e[j][1] + h.R[1][2] * h.e[j][2];
        }
        // As = 0.5 ((x1-x0)(y2-y0) - (x2-x0)(y1-y0))
        const double dAx[3] = {0.5 * (ya[1] - ya[2]), 0.5 * (ya[2] - ya[0]), 0.5 * (ya[0] - ya[1])};
        const double dAy[3] = {0.5 * (xa[2] - xa[1]), 0.5 * (xa[0] - xa[2]), 0.5 * (xa[1] - xa[0])};
        for (int j = 0; j < 3; j++) {
            xab[j] = A[A_TKX + j] + Asb * dAx[j];
            yab[j] = A[A_TKY + j] + Asb * dAy[j];
        }
        // R_bar
        double Rb[3][3];
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++)
                Rb[a][b] = A[A_WU + 3 * a + b] + A[A_EA + a] * h.c[b] / Rf +
                           A[A_INC + a] * inc[b] + A[A_P2 + a] * h.p[b];
        double eb[3][3];
        for (int j = 0; j < 3; j++)
            for (int b = 0; b < 3; b++) {
                Rb[0][b] += xab[j] * h.e[j][b];
                Rb[1][b] += yab[j] * h.e[j][b];
                eb[j][b] = xab[j] * h.R[0][b] + yab[j] * h.R[1][b];
            }
        // c_bar = direct + R^T ea_bar / Rf
        double cb[3];
        for (int b = 0; b < 3; b++)
            cb[b] = A[A_CU + b] + A[A_CE] * 2.0 * h.c[b] / (Rf * Rf) +
                    (h.R[0][b] * A[A_EA + 0] + h.R[1][b] * A[A_EA + 1] + h.R[2][b] * A[A_EA + 2]) / Rf;
        // frame: z = -n, x = unit(p - (p.n) n), y = z x x
        double n[3] = {-h.R[2][0], -h.R[2][1], -h.R[2][2]}, xh[3] = {h.R[0][0], h.R[0][1], h.R[0][2]};
        double zb[3] = {Rb[2][0], Rb[2][1], Rb[2][2]}, xb[3] = {Rb[0][0], Rb[0][1], Rb[0][2]},
               yb[3] = {Rb[1][0], Rb[1][1], Rb[1][2]};
        double z[3] = {-n[0], -n[1], -n[2]};
        // y = z x x: z_bar += x x y_bar, x_bar += y_bar x z
        zb[0] += xh[1] * yb[2] - xh[2] * yb[1];
        zb[1] += xh[2] * yb[0] - xh[0] * yb[2];
        zb[2] += xh[0] * yb[1] - xh[1] * yb[0];
        xb[0] += yb[1] * z[2] - yb[2] * z[1];
        xb[1] += yb[2] * z[0] - yb[0] * z[2];
        xb[2] += yb[0] * z[1] - yb[1] * z[0];
        const double pn = h.p[0] * n[0] + h.p[1] * n[1] + h.p[2] * n[2];
        double w[3] = {h.p[0] - pn * n[0], h.p[1] - pn * n[1], h.p[2] - pn * n[2]};
        const double wl = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
        const double xdot = xb[0] * xh[0] + xb[1] * xh[1] + xb[2] * xh[2];
        double wb[3];
        for (int b = 0; b < 3; b++) wb[b] = (xb[b] - xdot * xh[b]) / wl;
        const double wbn = wb[0] * n[0] + wb[1] * n[1] + wb[2] * n[2];
        double nb_[3];
        for (int b = 0; b < 3; b++) nb_[b] = -zb[b] - wbn * h.p[b] - pn * wb[b];
        // n = N/|N|, N = e0 x e1
        const double N[3] = {h.e[0][1] * h.e[1][2] - h.e[0][2] * h.e[1][1],
                             h.e[0][2] * h.e[1][0] - h.e[0][0] * h.e[1][2],
                             h.e[0][0] * h.e[1][1] - h.e[0][1] * h.e[1][0]};
        const double Nl = sqrt(N[0] * N[0] + N[1] * N[1] + N[2] * N[2]);
        const double ndot = nb_[0] * n[0] + nb_[1] * n[1] + nb_[2] * n[2];
        double Nb[3];
        for (int b = 0; b < 3; b++) Nb[b] = (nb_[b] - ndot * n[b]) / Nl;
        // e0_bar += e1 x N_bar ; e1_bar += N_bar x e0
        eb[0][0] += h.e[1][1] * Nb[2] - h.e[1][2] * Nb[1];
        eb[0][1] += h.e[1][2] * Nb[0] - h.e[1][0] * Nb[2];
        eb[0][2] += h.e[1][0] * Nb[1] - h.e[1][1] * Nb[0];
        eb[1][0] += Nb[1] * h.e[0][2] - Nb[2] * h.e[0][1];
        eb[1][1] += Nb[2] * h.e[0][0] - Nb[0] * h.e[0][2];
        eb[1][2] += Nb[0] * h.e[0][1] - Nb[1] * h.e[0][0];
        // e_j = v_j - c, c = mean(v)
        double esum[3] = {0, 0, 0};
        for (int j = 0; j < 3; j++)
            for (int b = 0; b < 3; b++) esum[b] += eb[j][b];
        for (int j = 0; j < 3; j++)
            for (int b = 0; b < 3; b++)
                atomicAdd(&gverts[h.vi[j] + nverts * b], eb[j][b] + (cb[b] - esum[b]) / 3.0);
    }

}  // namespace

// Host side: the triangle check, the device set-up, the kernels, and the
// gradient copies.
int k4_adjoint(pbt_ctx *ctx, cudaStream_t st, const pbt_outbeam *beam, int64_t nbeam,
               const pbt_outbeam *ext, int64_t next, const double *verts, int64_t nverts,
               const int64_t *face_off, const int64_t *face_vi, int64_t nfaces, double lambda,
               int fast_diff, const double *gafb, const double *gafe, double *gverts,
               double *gbeam, double *gext) {
    pbt::NvtxRange nvtx_("pbt: adjoint");
    const GridCache &g = ctx->grid;
    const int64_t nb = g.nb, nphi = (int64_t)g.phi.size();
    const double k = 2.0 * kPiRef / lambda, Rf = kFarR;
    const int64_t nrec = nbeam + next;
    for (int64_t q = 0; q < nrec; q++) {
        const pbt_outbeam &ob = q < nbeam ? beam[q] : ext[q - nbeam];
        if (face_off[ob.fi] - face_off[ob.fi - 1] != 3) {
            set_error("the adjoint supports triangular facets only (outbeam %lld, face %lld)",
                      (long long)(q + 1), (long long)ob.fi);
            return PBT_EINVAL;
        }
    }
    // device buffers: recs | kinds | fov | gafb | gafe | bins | gbin | out | outbeams |
    // verts | face_off | face_vi | mapping data | vertex gradients | amplitude gradients
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const int64_t nvi = face_off[nfaces];
    const size_t ob = sizeof(pbt_outbeam);
    const size_t o_rec = 0, o_kind = al(nrec * sizeof(K4Rec)), o_fov = al(o_kind + nrec * 4),
                 o_ga = al(o_fov + 16 * nrec), o_gb = al(o_ga + 8 * nb * 8),
                 o_bin = al(o_gb + 8 * nb * 8), o_gbin = al(o_bin + nb * sizeof(K4Bin)),
                 o_out = al(o_gbin + 16 * nb * 4), o_ob = al(o_out + nrec * K4_NACC * 8),
                 o_vert = al(o_ob + nrec * ob), o_fo = al(o_vert + 3 * nverts * 8),
                 o_fv = al(o_fo + (nfaces + 1) * 8), o_h = al(o_fv + nvi * 8),
                 o_gv = al(o_h + nrec * sizeof(Host4)), o_gamp = al(o_gv + 3 * nverts * 8),
                 o_end = al(o_gamp + nrec * 8 * 8);
    PBT_TRY(ctx->d_ws.ensure(o_end));
    char *base = ctx->d_ws.as<char>();
    pbt_outbeam *d_ob = (pbt_outbeam *)(base + o_ob);
    Host4 *d_h = (Host4 *)(base + o_h);
    double *d_gv = (double *)(base + o_gv), *d_gamp = (double *)(base + o_gamp);
    PBT_CUDA_TRY(cudaMemsetAsync(d_gv, 0, 3 * nverts * 8, st));
    if (nrec > 0) {
        // the FP64 set-up of each record on the device (the same frame code as the
        // forward's set-up), one thread per record
        if (nbeam) PBT_CUDA_TRY(cudaMemcpyAsync(d_ob, beam, nbeam * ob, cudaMemcpyHostToDevice, st));
        if (next) PBT_CUDA_TRY(cudaMemcpyAsync(d_ob + nbeam, ext, next * ob, cudaMemcpyHostToDevice, st));
        PBT_CUDA_TRY(cudaMemcpyAsync(base + o_vert, verts, 3 * nverts * 8, cudaMemcpyHostToDevice, st));
        PBT_CUDA_TRY(cudaMemcpyAsync(base + o_fo, face_off, (nfaces + 1) * 8, cudaMemcpyHostToDevice, st));
        PBT_CUDA_TRY(cudaMemcpyAsync(base + o_fv, face_vi, nvi * 8, cudaMemcpyHostToDevice, st));
        k4_setup_kernel<<<(unsigned)((nrec + 127) / 128), 128, 0, st>>>(
            d_ob, nbeam, d_ob + nbeam, nrec, (const double *)(base + o_vert), nverts,
            (const int64_t *)(base + o_fo), (const int64_t *)(base + o_fv), k, lambda,
            (K4Rec *)(base + o_rec), (int *)(base + o_kind), (float *)(base + o_fov), d_h);
        PBT_CUDA_TRY(cudaMemsetAsync(base + o_out, 0, nrec * K4_NACC * 8, st));
    }
    PBT_CUDA_TRY(cudaMemcpyAsync(base + o_ga, gafb, 8 * nb * 8, cudaMemcpyHostToDevice, st));
    PBT_CUDA_TRY(cudaMemcpyAsync(base + o_gb, gafe, 8 * nb * 8, cudaMemcpyHostToDevice, st));
    k4_prep_kernel<<<(unsigned)((nb + 127) / 128), 128, 0, st>>>(
        (const double *)(base + o_ga), (const double *)(base + o_gb), g.xyz.as<double>(),
        g.phitab.as<double>(), nb, nphi, k, (K4Bin *)(base + o_bin),
        (float4 *)(base + o_gbin));
    // bin ranges: at most K4_MAX_LANE_BINS terms per lane, and enough CTAs
    // for a few waves when there are few records
    const int64_t ncta_rec = (nrec + K4_WARPS - 1) / K4_WARPS;
    int64_t nsplit = (nb + 32 * K4_MAX_LANE_BINS - 1) / (32 * K4_MAX_LANE_BINS);
    if (ncta_rec > 0) nsplit = std::max(nsplit, (int64_t)(8 * ctx->sm_count + ncta_rec - 1) / ncta_rec);
    nsplit = std::min(nsplit, std::max<int64_t>(1, nb / 256));
    nsplit = std::min<int64_t>(nsplit, 65535);
    const int64_t chunk = (((nb + nsplit - 1) / nsplit) + 31) / 32 * 32;
    nsplit = (nb + chunk - 1) / chunk;
    const dim3 grid((unsigned)ncta_rec, (unsigned)nsplit);
    // bins with |uz| below pole_cos are out of reach of the forward bodge: the
    // direction from a facet centre c differs from the bin direction by at most
    // 2 |c| / R, and |c| <= max |v| over the vertices
    double vmax2 = 0.0;
    for (int64_t i = 0; i < nverts; i++) {
        const double x = verts[i], y = verts[i + nverts], z = verts[i + 2 * nverts];
        vmax2 = std::max(vmax2, x * x + y * y + z * z);
    }
    const float pole_cos = (float)(0.999 - 2.0 * sqrt(vmax2) / Rf - 1e-5);
    timing_begin(ctx, st);
    // Minimum CTAs per SM for the register budget: 3 (168 registers, a few
    // bytes of spill) by default; PBT_K4_MINB=1|2|4 selects another build.
    static const int minb = [] {
        const char *e = getenv("PBT_K4_MINB");
        const int v = e ? atoi(e) : 3;
        return (v == 1 || v == 2 || v == 4) ? v : 3;
    }();
    if (nrec > 0) {
        auto launch = [&](auto kern) {
            kern<<<grid, K4_WARPS * 32, 0, st>>>(
                (const K4Rec *)(base + o_rec), (const int *)(base + o_kind), (const float *)(base + o_fov),
                nrec, (const K4Bin *)(base + o_bin), (const float4 *)(base + o_gbin), nb, nphi,
                g.theta_i, chunk, (float)k,
                (float)(0.5 * k * Rf), (float)(1.0 / Rf), pole_cos, (double *)(base + o_out));
        };
        if (fast_diff) {
            if (minb == 1) launch(k4_adjoint_kernel<true, 1>);
            else if (minb == 2) launch(k4_adjoint_kernel<true, 2>);
            else if (minb == 4) launch(k4_adjoint_kernel<true, 4>);
            else launch(k4_adjoint_kernel<true, 3>);
        } else {
            if (minb == 1) launch(k4_adjoint_kernel<false, 1>);
            else if (minb == 2) launch(k4_adjoint_kernel<false, 2>);
            else if (minb == 4) launch(k4_adjoint_kernel<false, 4>);
            else launch(k4_adjoint_kernel<false, 3>);
        }
    }
    timing_end(ctx, st);
    ctx->launches += nrec > 0 ? 2 : 1;
    PBT_CUDA_TRY(cudaGetLastError());
    // FP64 mapping of the per-record sums to the vertices and amplitudes, one
    // thread per record; the vertex cotangents are added with FP64 atomics
    if (nrec > 0)
        k4_map_kernel<<<(unsigned)((nrec + 127) / 128), 128, 0, st>>>(
            (const double *)(base + o_out), d_h, d_ob, nbeam, d_ob + nbeam, nrec, lambda, nverts,
            d_gamp, d_gamp + 8 * nbeam, d_gv);
    ctx->launches += nrec > 0 ? 2 : 0;
    PBT_CUDA_TRY(cudaGetLastError());
    PBT_CUDA_TRY(cudaMemcpyAsync(gverts, d_gv, 3 * nverts * 8, cudaMemcpyDeviceToHost, st));
    if (nbeam) PBT_CUDA_TRY(cudaMemcpyAsync(gbeam, d_gamp, nbeam * 8 * 8, cudaMemcpyDeviceToHost, st));
    if (next)
        PBT_CUDA_TRY(cudaMemcpyAsync(gext, d_gamp + 8 * nbeam, next * 8 * 8, cudaMemcpyDeviceToHost, st));
    PBT_CUDA_TRY(cudaStreamSynchronize(st));
    return PBT_OK;
}

}  // namespace pbt
