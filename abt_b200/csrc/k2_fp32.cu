// k2_fp32.cu -- batched far-field sum in FP32 with the phase formed in FP64.
//
// Pipeline for a batch of orientations (all on the GPU, no host round trip):
//   1. k2_count / CUB scan / k2_setup: one thread per outgoing facet forms the
//      facet's aperture frame in FP64 (frame.h, the reference's set-up of
//      src/diff_mod.f90:515-574) and writes nv-2 K2Rec triangle records.
//   2. k2_plan: per (orientation, beam|external) segment, the number of
//      work items = facet splits x bin tiles.
//   3. k2_main: a persistent kernel; each CTA claims work items with an
//      atomic counter, streams the item's facet records through shared memory
//      with 1-D bulk copies (cp.async.bulk + mbarrier, bounded waits), and
//      accumulates for each of its bins the 2x2 complex amplitude in FP32
//      (chunk sums carried in FP64), then adds it to the orientation's
//      amplitude workspace.
//   4. k2_epi: FP64 epilogue per bin over the orientations of the batch:
//      T(phi) rotation, Mueller matrix (ampl_to_mueller, src/outputs_mod.f90:
//      473-549), running orientation sum, and per-orientation weighted sums
//      that equal the reference's simpne phi/theta integrals of M11.
//   5. k2_final / k2_average: per-orientation parameters (finalise,
//      src/outputs_mod.f90:133-245) and the orientation average
//      (summation + divide_by_num_orientations).
//
// Per facet x bin arithmetic.  The reference evaluates, per edge, a contour
// term with a 1/(kxx kyy) coordinate singularity (src/diff_mod.f90:408-420).
// Summed over a triangle's edges it equals (-i/lambda) e^{iK} times the
// aperture integral, which for a triangle is -2A g[d1,d2,d3]: the second
// divided difference of e^{ix} at the three vertex phases.  That form has no
// coordinate singularity; it is evaluated from edge-midpoint phases and
// sinc((d_b - d_a)/2) (stable for every pair gap), with a Taylor series when
// all three phases lie within 0.25 rad.  The far-field phase
// k(|X - c| - |X|) = -k u.c + k(|c|^2 - (u.c)^2)(1 + u.c/R)/(2R) is formed
// with k u.c in FP64 and reduced mod 2 pi before the FP32 work; the common
// e^{ik|X|} is applied per bin only when amplitudes are returned.
#include <stdio.h>
#include <stdlib.h>

#include <cub/device/device_scan.cuh>

#include "frame.h"
#include "k2_common.cuh"
#include "pbt_internal.h"

namespace pbt {

namespace {

constexpr int K2_THREADS = 128;
constexpr int K2_CH = 32;   // records per shared-memory stage
constexpr int K2_NST = 3;   // stages
constexpr double kTwoPi = 6.283185307179586;
constexpr double kInv2Pi = 0.15915494309189535;
constexpr double kMagic = 6755399441055744.0;  // 1.5 * 2^52, round-to-integer constant
constexpr double kPi = 3.141592653589793;
constexpr double kInvPi = 0.3183098861837907;
// 1 - c^2 for the reference's clamp c = 0.999999 (a float literal)
constexpr float kOneMinusClampSq = (float)(1.0 - (double)0.999999f * (double)0.999999f);

struct BinDev {
    double ux, uy, uz;  // unit bin direction, FP64
    float fx, fy, fz;   // same, FP32
    float sz, sg;       // s = u + sg z: sz = uz + sg (rounded once from FP64), sg = +-1
    float hx, hy, hsz;  // the (phi_i, theta_i) bin of the forward bodge in the same form
    int64_t bin;        // bin index
};

// The field-of-view test of the FP64 drop-in for bin `bin` (src/diff_mod.f90:593-603):
// x1 = X - com, dot(x1/r1, prop0) >= cos(fov), each operation rounded once.
__device__ __forceinline__ bool fov_exact(const K2Fov &f, const double *__restrict__ xyz, int64_t nb,
                                       int64_t bin) {
    const double x1 = __dadd_rn(xyz[bin], -f.com[0]);
    const double y1 = __dadd_rn(xyz[nb + bin], -f.com[1]);
    const double z1 = __dadd_rn(xyz[2 * nb + bin], -f.com[2]);
    const double r1 =
        __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(x1, x1), __dmul_rn(y1, y1)), __dmul_rn(z1, z1)));
    const double v0 = __ddiv_rn(x1, r1), v1 = __ddiv_rn(y1, r1), v2 = __ddiv_rn(z1, r1);
    const double d = __dadd_rn(__dadd_rn(__dmul_rn(v0, f.p0d[0]), __dmul_rn(v1, f.p0d[1])),
                               __dmul_rn(v2, f.p0d[2]));
    return !(d < f.cos_fovd);
}

// ---------------------------------------------------------------- set-up

struct RefSrc {
    const pbt_outbeam *beam;
    const pbt_outbeam *ext;
    const int64_t *beam_off;  // device copies, norient+1
    const int64_t *ext_off;
    const int64_t *refbase;   // beam_off[o] + ext_off[o]
    int64_t norient;
};

__device__ __forceinline__ int64_t find_orient(const int64_t *base, int64_t n, int64_t g) {
    int64_t lo = 0, hi = n;  // largest o in [0, n) with base[o] <= g
    while (hi - lo > 1) {
        int64_t mid = (lo + hi) >> 1;
        if (base[mid] <= g)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

__device__ __forceinline__ const pbt_outbeam *ref_lookup(const RefSrc &S, int64_t g, int64_t &o,
                                                         int &kind) {
    o = find_orient(S.refbase, S.norient, g);
    const int64_t local = g - S.refbase[o];
    const int64_t nb = S.beam_off[o + 1] - S.beam_off[o];
    if (local < nb) {
        kind = 0;
        return S.beam + S.beam_off[o] + local;
    }
    kind = 1;
    return S.ext + S.ext_off[o] + (local - nb);
}

__global__ void k2_count_kernel(RefSrc S, int64_t nrefs, const int64_t *__restrict__ face_off,
                                int64_t nfaces, int64_t *__restrict__ cnt, int *__restrict__ err) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g > nrefs) return;
    if (g == nrefs) {
        cnt[g] = 0;
        return;
    }
    int64_t o;
    int kind;
    const pbt_outbeam *ob = ref_lookup(S, g, o, kind);
    const int64_t fi = ob->fi;
    if (fi < 1 || fi > nfaces) {
        atomicOr(err, 1);
        cnt[g] = 0;
        return;
    }
    cnt[g] = face_off[fi] - face_off[fi - 1] - 2;
}

// Write record r into half r % 2 of pair r / 2 (K2Pair's half-phase and
// scaled forms): kzc = -Kz / (1 - Ky^2) and the circular-basis amplitudes uc
// times sqrt(1 - Ky^2) / 4, both formed in FP64 by the caller.
__device__ __forceinline__ void store_pair_half(K2Pair *pairs, int64_t r, const K2Rec &rec,
                                                double kzc, const double (&uc)[8]) {
    K2Pair &P = pairs[r >> 1];
    const int h = (int)(r & 1);
    auto put = [h](float2 &dst, float v) {
        if (h)
            dst.y = v;
        else
            dst.x = v;
    };
    for (int c = 0; c < 3; c++) {
        P.kc[c][h] = 0.5 * rec.kc[c];
        put(P.eps[c], rec.eps[c]);
        put(P.nea[c], -rec.ea[c]);
        put(P.inc[c], rec.inc[c]);
        put(P.vx[c], rec.vx[c]);
        put(P.vy[c], rec.vy[c]);
    }
    put(P.b, rec.b);
    for (int q = 0; q < 9; q++) put(P.R[q], rec.R[q]);
    put(P.kp[0], 0.5f * rec.kp[0]);
    put(P.kp[1], 0.5f * rec.kp[1]);
    put(P.kzc, (float)kzc);
    for (int q = 0; q < 8; q++) put(P.amp[q], (float)uc[q]);
}

__global__ void k2_setup_kernel(RefSrc S, int64_t nrefs, const double *__restrict__ verts,
                                int64_t nverts, const int64_t *__restrict__ face_off,
                                const int64_t *__restrict__ face_vi, const int64_t *__restrict__ start,
                                double waveno, double lambda, int fast_diff,
                                K2Rec *__restrict__ recs, K2Pair *__restrict__ pairs,
                                K2Fov *__restrict__ fovs, float2 *__restrict__ rlo,
                                int *__restrict__ err, unsigned *__restrict__ epsmax) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nrefs) return;
    int64_t o;
    int kind;
    const pbt_outbeam *ob = ref_lookup(S, g, o, kind);
    const int64_t fi = ob->fi;
    if (fi < 1) return;  // reported by the count kernel
    const int64_t fb = face_off[fi - 1];
    const int nv = (int)(face_off[fi] - fb);
    const double *V = verts + o * 3 * nverts;
    constexpr int NVS = 16;  // vertices held in registers; larger faces re-read
    double vx[NVS], vy[NVS], vz[NVS];
    double prop0[3] = {ob->prop_out[0], ob->prop_out[1], ob->prop_out[2]};
    double perp0[3] = {ob->vk7[0], ob->vk7[1], ob->vk7[2]};
    if (nv > NVS) {
        atomicOr(err, 2);  // faces above 16 vertices are not supported in FP32
        return;
    }
    for (int i = 0; i < nv; i++) {
        const int64_t vi = face_vi[fb + i] - 1;
        vx[i] = V[vi];
        vy[i] = V[vi + nverts];
        vz[i] = V[vi + 2 * nverts];
    }
    FacetFrame fr;
    facet_frame(vx, vy, vz, nv, prop0, perp0, fr, nullptr, nullptr, nullptr);
    const double sign = fr.sign;
    const double *com = fr.com;
    const double R = kFarR;
    if (epsmax) {
        // an upper bound of |com| / R over the records (positive floats order as
        // unsigned integers)
        const double e = sqrt(com[0] * com[0] + com[1] * com[1] + com[2] * com[2]) / R;
        atomicMax(epsmax, __float_as_uint((float)(e * (1.0 + 1e-6)) + 1e-30f));
    }
    const double Ky = fr.prop2[1];
    const double cf = 1.0 / sqrt(1.0 - Ky * Ky);
    double ea[3];
    mv33(fr.R, com, ea);
    const int64_t r0 = start[g];
    for (int t = 0; t < nv - 2; t++) {
        const int iv[3] = {0, t + 1, t + 2};
        double xa[3], ya[3];
        for (int q = 0; q < 3; q++) {
            const double d[3] = {vx[iv[q]] - com[0], vy[iv[q]] - com[1], vz[iv[q]] - com[2]};
            double rr[3];
            mv33(fr.R, d, rr);
            xa[q] = rr[0];
            ya[q] = rr[1];
        }
        const double As = 0.5 * ((xa[1] - xa[0]) * (ya[2] - ya[0]) - (xa[2] - xa[0]) * (ya[1] - ya[0]));
        const double cpre = 2.0 * As / lambda * sign;  // amp' = i * cpre * ampl
        K2Rec rec;
        for (int c = 0; c < 3; c++) {
            rec.kc[c] = waveno * com[c];
            rec.eps[c] = (float)(com[c] / R);
            rec.ea[c] = (float)(ea[c] / R);
            rec.inc[c] = (float)fr.inc2[c];
            rec.vx[c] = (float)xa[c];
            rec.vy[c] = (float)ya[c];
        }
        rec.b = (float)((com[0] * com[0] + com[1] * com[1] + com[2] * com[2]) / (R * R));
        for (int q = 0; q < 9; q++) rec.R[q] = (float)fr.R.m[q / 3][q % 3];
        for (int i = 0; i < 3; i++) {
            // the low part of the y row, read only by lanes on the ky clamp
            float2 &l = rlo[((r0 + t) >> 1) * 3 + i];
            const float lo = (float)(fr.R.m[1][i] - (double)rec.R[3 + i]);
            if ((r0 + t) & 1)
                l.y = lo;
            else
                l.x = lo;
        }
        rec.kp[0] = (float)(waveno * fr.prop2[0]);
        rec.kp[1] = (float)(waveno * fr.prop2[1]);
        rec.hkz_cf = (float)(-0.5 * fr.prop2[2] * cf);
        rec.hicf = (float)(0.5 / cf);
        rec.hkxky_cf = (float)(0.5 * fr.prop2[0] * Ky * cf);
        double am[8];  // (2 i A / lambda) sign ampl: (1,1),(2,1),(1,2),(2,2) re/im
        for (int q = 0; q < 4; q++) {
            am[2 * q] = -cpre * ob->ampl[2 * q + 1];
            am[2 * q + 1] = cpre * ob->ampl[2 * q];
        }
        for (int q = 0; q < 8; q++) rec.amp[q] = (float)am[q];
        if (pairs) {
            // the packed kernel works on the columns in the circular basis
            // u+ = a1c + i a2c, u- = a1c - i a2c (formed in FP64), scaled by the
            // Karczewski-Wolf factor sqrt(1 - Ky^2) / 2 and the 1/2 of the
            // half-phase divided difference
            const double sk = 0.25 / cf;
            const double uc[8] = {sk * (am[0] - am[3]), sk * (am[1] + am[2]), sk * (am[0] + am[3]),
                                  sk * (am[1] - am[2]), sk * (am[4] - am[7]), sk * (am[5] + am[6]),
                                  sk * (am[4] + am[7]), sk * (am[5] - am[6])};
            store_pair_half(pairs, r0 + t, rec, -fr.prop2[2] * cf * cf, uc);
        } else {
            recs[r0 + t] = rec;
        }
        if (fast_diff) {
            K2Fov fv;
            const double fov = kind ? kPiRef / 2.0 : ob->fov;
            fv.p0[0] = (float)prop0[0];
            fv.p0[1] = (float)prop0[1];
            fv.p0[2] = (float)prop0[2];
            fv.cos_fov = (float)cos(fov);
            // the per-bin test uses the direction from the facet centre: it is
            // within |c|/R of the direction from the origin; 2|c|/R + 1e-5 rad
            // also covers the FP32 rounding of both tests
            const double cn = sqrt(fr.com[0] * fr.com[0] + fr.com[1] * fr.com[1] +
                                   fr.com[2] * fr.com[2]);
            const double fovm = fov + 2.0 * cn / kFarR + 1e-5;
            fv.fovm = (float)fovm;
            fv.cos_fovm = (float)cos(fovm);
            fv.sin_fovm = (float)sin(fovm);
            // FP32 test error: second-order parallax (< 3 |c/R|^2) and rounding (< 8e-7)
            const double e2 = (cn / kFarR) * (cn / kFarR);
            fv.tol = (float)(3.0 * e2 + 8e-7);
            for (int c = 0; c < 3; c++) {
                fv.com[c] = fr.com[c];
                fv.p0d[c] = prop0[c];
            }
            fv.cos_fovd = cos(fov);
            fv.pad = 0.0;
            fovs[r0 + t] = fv;
        }
    }
}

// Per orientation chunk [o0, o0+no): segment records and work-item prefix.
__global__ void k2_plan_kernel(const int64_t *__restrict__ start, const int64_t *__restrict__ refbase,
                               const int64_t *__restrict__ beam_off, int64_t o0, int64_t no,
                               int64_t rpi, int64_t ntiles, int64_t *__restrict__ seg_rec,
                               int64_t *__restrict__ item_pre, unsigned long long *__restrict__ counter) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int64_t q = 0; q < no; q++) {
        const int64_t o = o0 + q;
        const int64_t nbo = beam_off[o + 1] - beam_off[o];
        seg_rec[2 * q] = start[refbase[o]];
        seg_rec[2 * q + 1] = start[refbase[o] + nbo];
    }
    seg_rec[2 * no] = start[refbase[o0 + no]];
    int64_t p = 0;
    for (int64_t s = 0; s < 2 * no; s++) {
        item_pre[s] = p;
        const int64_t n = seg_rec[s + 1] - seg_rec[s];
        p += ((n + rpi - 1) / rpi) * ntiles;
    }
    item_pre[2 * no] = p;
    *counter = 0ull;
}

// ------------------------------------------------------------ main kernel

__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// sin(h)/h for h >= 0: Taylor series below 0.5, MUFU sine above
__device__ __forceinline__ float sinc_pos(float h) {
    const float h2 = h * h;
    const float p = fmaf(h2, fmaf(h2, fmaf(h2, fmaf(h2, 2.7557319e-6f, -1.9841270e-4f), 8.3333333e-3f),
                                  -1.6666667e-1f),
                         1.0f);
    const float q = __sinf(h) * rcp_approx(h);
    return h < 0.5f ? p : q;
}

// Second divided difference of e^{ix} at t1, t2, t3 (symmetric in its arguments).
__device__ __forceinline__ float2 tri_dd(float t1, float t2, float t3) {
    float lo = fminf(t1, t2), hi = fmaxf(t1, t2);
    const float mid = fmaxf(lo, fminf(hi, t3));
    lo = fminf(lo, t3);
    hi = fmaxf(hi, t3);
    const float D = hi - lo;
    float2 g;
    if (D >= 0.25f) {
        const float h1 = 0.5f * (mid - lo), h2 = 0.5f * (hi - mid);
        float s1, c1, s2, c2;
        __sincosf(lo + h1, &s1, &c1);
        __sincosf(mid + h2, &s2, &c2);
        const float sc1 = sinc_pos(h1), sc2 = sinc_pos(h2);
        const float iD = rcp_approx(D);
        g.x = (sc1 * s1 - sc2 * s2) * iD;
        g.y = (sc2 * c2 - sc1 * c1) * iD;
    } else {
        // e^{i mid} * sum_n i^(n+2)/(n+2)! h_n(ya, yc), h_n complete homogeneous
        const float ya = lo - mid, yc = hi - mid;
        const float h1 = ya + yc;
        const float ya2 = ya * ya;
        const float h2 = fmaf(yc, h1, ya2);
        const float ya3 = ya2 * ya;
        const float h3 = fmaf(yc, h2, ya3);
        const float ya4 = ya3 * ya;
        const float h4 = fmaf(yc, h3, ya4);
        const float h5 = fmaf(yc, h4, ya4 * ya);
        const float h6 = fmaf(yc, h5, ya4 * ya2);
        const float re = -0.5f + h2 * (1.0f / 24.0f) - h4 * (1.0f / 720.0f) + h6 * (1.0f / 40320.0f);
        const float im = -h1 * (1.0f / 6.0f) + h3 * (1.0f / 120.0f) - h5 * (1.0f / 5040.0f);
        float sm, cm;
        __sincosf(mid, &sm, &cm);
        g.x = cm * re - sm * im;
        g.y = cm * im + sm * re;
    }
    return g;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ uint64_t gtimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
        "l"(src), "r"(bytes), "r"(bar)
        : "memory");
}
// Bounded wait on an mbarrier phase: false after limit_ns of global time or
// 2^26 polls, whichever comes first.
constexpr uint64_t kWaitLimitNs = 2000000000ull;
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity,
                                          uint64_t limit_ns = kWaitLimitNs) {
    uint64_t t0 = 0;
    for (uint32_t it = 0; it < (1u << 26); ++it) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
        if (it == 0) t0 = gtimer();
        else if ((it & 255) == 0 && gtimer() - t0 > limit_ns) return false;
    }
    return false;
}

// Work items of one (segment, bin tile) are facet splits.  Each adds its FP64
// sums into the workspace after the previous split of the same tile: ticket
// tk counts the splits added so far (split s waits for tk >= s, adds, and sets
// tk = s + 1), so the sum over splits is in split order and the result is the
// same from run to run.  The item of split s - 1 has the lower item index, so
// it was claimed earlier by a running CTA and never waits on split s.  A wait
// that gives up (2 s of global time or 2^26 polls), or a CTA whose bulk copy
// timed out, sets the ticket to kTicketPoison: later splits of the tile then
// skip their add at once and the call reports PBT_ETIMEOUT.
constexpr unsigned kTicketPoison = 0xffffffffu;
__device__ __forceinline__ bool ticket_wait(const unsigned *tk, unsigned s) {
    uint64_t t0 = 0;
    for (uint32_t it = 0; it < (1u << 26); ++it) {
        unsigned v;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(tk) : "memory");
        if (v >= s) return v != kTicketPoison;
        if (it == 0) t0 = gtimer();
        else if ((it & 255) == 0 && gtimer() - t0 > kWaitLimitNs) return false;
    }
    return false;
}

// The item's sums (lin[bin][8], FP64) into the workspace in split order (see
// ticket_wait); every thread of the CTA calls this.
template <int BPT>
__device__ __forceinline__ void ordered_add(double *__restrict__ out, int64_t nb, unsigned *tk,
                                            unsigned split, const bool (&valid)[BPT],
                                            const int64_t (&bin)[BPT], const double (&lin)[BPT][8],
                                            int *s_ok, int *err) {
    if (threadIdx.x == 0) *s_ok = ticket_wait(tk, split);
    __syncthreads();
    const bool go = *s_ok != 0;
    if (go) {
        __threadfence();
#pragma unroll
        for (int q = 0; q < BPT; q++)
            if (valid[q])
#pragma unroll
                for (int cc = 0; cc < 8; cc++) {
                    double *o = out + cc * nb + bin[q];
                    *o = __ldcg(o) + lin[q][cc];
                }
        __threadfence();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (go) {
            atomicMax(tk, split + 1u);
        } else {
            atomicOr(err, 4);
            atomicMax(tk, kTicketPoison);
        }
    }
}

struct K2MainArgs {
    const K2Rec *recs;
    const K2Fov *fovs;
    const float2 *rlo;  // R_1 - (float)R_1, pair layout (3 per pair)
    const int64_t *seg_rec;
    const int64_t *item_pre;
    int64_t nseg;
    int64_t rpi;
    int64_t ntiles;
    const double *xyz;
    int64_t nb, nphi;
    int64_t theta_i;
    float k;      // wavenumber
    float hkR;    // k R / 2
    float sgh;    // +1 when the bodge row theta_i lies in the hemisphere of (0,0,-1), else -1
    double *ws;   // [seg][8][nb]
    unsigned *tickets;  // [seg][tile], splits added so far
    unsigned long long *counter;
    int *err;
};

// For a lane on the ky clamp: one component of v = u - sigma R_1, sigma the sign of
// ky and R_1 the aperture frame's y axis (rounded row hi, low part lo), formed from
// the FP64 bin direction.  On the clamp the reference divides kx and kz by
// s = sqrt(1 - 0.999999^2) = 1.4e-3 (m = (-kx ky / s, s, -kz ky / s),
// src/diff_mod.f90:151-158); formed in FP32 from u they are differences of O(1)
// terms with an absolute error near 1e-7, which that division makes 1e-4.  With
// R_0 . R_1 = 0, kx = R_0 . v opa2 + nea_0 opa and kz = R_2 . v opa2 + nea_2 opa,
// where v is small and known to FP32 precision (absolute error near 1e-10).
__device__ __forceinline__ float clamp_v(float hi, float lo, double u, float sigma) {
    return fmaf(-sigma, lo, (float)fma(-(double)sigma, (double)hi, u));
}

template <int BPT, bool FAST>
__device__ __forceinline__ void k2_record(const K2Rec &r, const K2Fov *fv, const BinDev (&bd)[BPT],
                                          const bool (&valid)[BPT], float (&acc)[BPT][8], float k,
                                          float hkR, float sgh, const double *__restrict__ xyz,
                                          int64_t nb, const float2 *__restrict__ rl, int half) {
    const double kc0 = r.kc[0], kc1 = r.kc[1], kc2 = r.kc[2];
#pragma unroll
    for (int q = 0; q < BPT; q++) {
        const BinDev &B = bd[q];
        // far-field phase: FP64 k u.c, reduced mod 2 pi
        const double ka = fma(B.uz, kc2, fma(B.uy, kc1, B.ux * kc0));
        const double nq = fma(ka, kInv2Pi, kMagic) - kMagic;
        const float rf = (float)fma(-nq, kTwoPi, ka);
        const float a = fmaf(B.fz, r.eps[2], fmaf(B.fy, r.eps[1], B.fx * r.eps[0]));
        const float ph = fmaf(hkR * fmaf(-a, a, r.b), 1.0f + a, -rf);
        // bin direction from the facet centre, in the aperture frame:
        // (u - e)/|u - e| = u (1 + a + 3a^2/2 - b/2) - e (1 + a) + O(|e|^3), e = c/R.
        // The second-order terms matter: near k ~ +-y the polarisation matrix
        // depends on 1 - ky^2 and amplifies direction errors by 1/(1 - ky^2).
        // With s = u + sg z and inc = -R z: k = ks + sg opa2 inc, ks = R s opa2 - ea opa,
        // and h = inc x k = inc x ks is formed from small vectors near the poles.
        const float opa = 1.0f + a;
        const float opa2 = fmaf(a, fmaf(1.5f, a, 1.0f), fmaf(-0.5f, r.b, 1.0f));
        const float w0 = fmaf(r.R[2], B.sz, fmaf(r.R[1], B.fy, r.R[0] * B.fx));
        const float w1 = fmaf(r.R[5], B.sz, fmaf(r.R[4], B.fy, r.R[3] * B.fx));
        const float w2 = fmaf(r.R[8], B.sz, fmaf(r.R[7], B.fy, r.R[6] * B.fx));
        const float ks0 = fmaf(w0, opa2, -r.ea[0] * opa);
        const float ks1 = fmaf(w1, opa2, -r.ea[1] * opa);
        const float ks2 = fmaf(w2, opa2, -r.ea[2] * opa);
        const float so = B.sg * opa2;
        const float kx = fmaf(so, r.inc[0], ks0);
        const float ky = fmaf(so, r.inc[1], ks1);
        const float kz = fmaf(so, r.inc[2], ks2);
        bool use = valid[q];
        if (FAST) {
            // lab-frame direction from the centre: u - eps + u a
            const float dx = fmaf(B.fx, opa, -r.eps[0]);
            const float dy = fmaf(B.fy, opa, -r.eps[1]);
            const float dz = fmaf(B.fz, opa, -r.eps[2]);
            const float dp = fmaf(dz, fv->p0[2], fmaf(dy, fv->p0[1], dx * fv->p0[0]));
            bool in = !(dp < fv->cos_fov);
            if (use && fabsf(dp - fv->cos_fov) < fv->tol) in = fov_exact(*fv, xyz, nb, B.bin);
            use = use && in;
        }
        // aperture integral
        const float kxx = fmaf(-k, kx, r.kp[0]);
        const float kyy = fmaf(-k, ky, r.kp[1]);
        const float t1 = fmaf(kyy, r.vy[0], fmaf(kxx, r.vx[0], ph));
        const float t2 = fmaf(kyy, r.vy[1], fmaf(kxx, r.vx[1], ph));
        const float t3 = fmaf(kyy, r.vy[2], fmaf(kxx, r.vx[2], ph));
        const float2 g = tri_dd(t1, t2, t3);
        // Karczewski-Wolf polarisation matrix [[d, e], [-e, d]].  1 - ky^2 is
        // formed as kx^2 + kz^2 (equal for a unit vector, without the
        // cancellation near |ky| = 1); the floor is the reference's clamp
        // |ky| <= 0.999999 (src/diff_mod.f90:151).
        const float kyc = fminf(fmaxf(ky, -0.999999f), 0.999999f);
        const float tr = fmaf(kx, kx, kz * kz);
        float kxv = kx, kzv = kz;  // kx, kz of the polarisation block
        if (tr <= kOneMinusClampSq) {
            auto lo = [&](int i) { return half ? rl[i].y : rl[i].x; };
            const float sig = ky < 0.0f ? -1.0f : 1.0f;
            const float v0 = clamp_v(r.R[3], lo(0), B.ux, sig), v1 = clamp_v(r.R[4], lo(1), B.uy, sig),
                        v2 = clamp_v(r.R[5], lo(2), B.uz, sig);
            kxv = fmaf(fmaf(r.R[2], v2, fmaf(r.R[1], v1, r.R[0] * v0)), opa2, -r.ea[0] * opa);
            kzv = fmaf(fmaf(r.R[8], v2, fmaf(r.R[7], v1, r.R[6] * v0)), opa2, -r.ea[2] * opa);
        }
        const float tt = fmaxf(tr, kOneMinusClampSq);
        const float rs = rsqrtf(tt);
        const float s = tt * rs;
        const float kyrs = kyc * rs;
        const float m0 = -kxv * kyrs, m1 = s, m2 = -kzv * kyrs;
        const float d = fmaf(r.hkz_cf, s, -(kzv * rs) * r.hicf);
        const float e = fmaf(r.hkxky_cf, s, -(kxv * kyrs) * r.hicf);
        // vector perpendicular to the scattering plane (forward bodge near the poles)
        // h = inc x (kx, kyc, kz) = inc x (ks0, ks1 + kyc - ky, ks2)
        float qx = ks0, qy = ks1 + (kyc - ky), qz = ks2;
        const float dinc = fmaf(r.inc[2], kzv, fmaf(r.inc[1], kyc, r.inc[0] * kxv));
        if (!(fabsf(dinc) < 0.999f)) {
            // bodge direction in the s form: uh . eps = hs . eps - sgh eps_z
            const float ah = fmaf(-sgh, r.eps[2],
                                  fmaf(B.hsz, r.eps[2], fmaf(B.hy, r.eps[1], B.hx * r.eps[0])));
            const float oh = 1.0f + ah;
            const float oh2 = fmaf(ah, fmaf(1.5f, ah, 1.0f), fmaf(-0.5f, r.b, 1.0f));
            qx = fmaf(fmaf(r.R[2], B.hsz, fmaf(r.R[1], B.hy, r.R[0] * B.hx)), oh2, -r.ea[0] * oh);
            qy = fmaf(fmaf(r.R[5], B.hsz, fmaf(r.R[4], B.hy, r.R[3] * B.hx)), oh2, -r.ea[1] * oh);
            qz = fmaf(fmaf(r.R[8], B.hsz, fmaf(r.R[7], B.hy, r.R[6] * B.hx)), oh2, -r.ea[2] * oh);
        }
        float hx = fmaf(r.inc[1], qz, -r.inc[2] * qy);
        float hy = fmaf(r.inc[2], qx, -r.inc[0] * qz);
        float hz = fmaf(r.inc[0], qy, -r.inc[1] * qx);
        const float hn = rsqrtf(fmaf(hz, hz, fmaf(hy, hy, hx * hx)));
        hx *= hn;
        hy *= hn;
        hz *= hn;
        float ex = fmaf(kyc, m2, -kzv * m1);
        float ey = fmaf(kzv, m0, -kxv * m2);
        float ez = fmaf(kxv, m1, -kyc * m0);
        if (tt <= kOneMinusClampSq) {
            // inside the clamp cone k and m are not unit vectors and the
            // reference's normalisation of k x m (src/diff_mod.f90:637) matters
            const float ne = rsqrtf(fmaf(ez, ez, fmaf(ey, ey, ex * ex)));
            ex *= ne;
            ey *= ne;
            ez *= ne;
        }
        const float p = fmaf(hz, m2, fmaf(hy, m1, hx * m0));
        const float rr = fmaf(hz, ez, fmaf(hy, ey, hx * ex));
        const float A = fmaf(p, d, rr * e);
        const float Bc = fmaf(p, e, -rr * d);
        // G = [[A, B], [-B, A]] . amp ; acc += g * G
        const float gx = use ? g.x : 0.0f, gy = use ? g.y : 0.0f;
        float G[8];
        G[0] = fmaf(A, r.amp[0], Bc * r.amp[2]);
        G[1] = fmaf(A, r.amp[1], Bc * r.amp[3]);
        G[2] = fmaf(A, r.amp[2], -Bc * r.amp[0]);
        G[3] = fmaf(A, r.amp[3], -Bc * r.amp[1]);
        G[4] = fmaf(A, r.amp[4], Bc * r.amp[6]);
        G[5] = fmaf(A, r.amp[5], Bc * r.amp[7]);
        G[6] = fmaf(A, r.amp[6], -Bc * r.amp[4]);
        G[7] = fmaf(A, r.amp[7], -Bc * r.amp[5]);
#pragma unroll
        for (int c = 0; c < 4; c++) {
            acc[q][2 * c] = fmaf(gx, G[2 * c], fmaf(-gy, G[2 * c + 1], acc[q][2 * c]));
            acc[q][2 * c + 1] = fmaf(gx, G[2 * c + 1], fmaf(gy, G[2 * c], acc[q][2 * c + 1]));
        }
    }
}

template <int BPT, bool FAST>
__global__ void __launch_bounds__(K2_THREADS, 2) k2_main_kernel(K2MainArgs P) {
    __shared__ __align__(128) K2Rec sbuf[K2_NST][K2_CH];
    __shared__ __align__(8) uint64_t bars[K2_NST];
    __shared__ long long s_item;
    __shared__ int s_ok;
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int s = 0; s < K2_NST; s++) mbar_init(smem_u32(&bars[s]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    uint32_t parity[K2_NST] = {0, 0, 0};
    const int64_t total = P.item_pre[P.nseg];
    constexpr int64_t TILE = (int64_t)K2_THREADS * BPT;
    for (;;) {
        if (tid == 0) s_item = (long long)atomicAdd(P.counter, 1ull);
        __syncthreads();
        const int64_t item = s_item;
        if (item >= total) break;
        // decode item -> (segment, split, tile)
        int64_t lo = 0, hi = P.nseg;
        while (hi - lo > 1) {
            const int64_t m = (lo + hi) >> 1;
            if (P.item_pre[m] <= item)
                lo = m;
            else
                hi = m;
        }
        const int64_t seg = lo;
        const int64_t local = item - P.item_pre[seg];
        const int64_t split = local / P.ntiles, tile = local % P.ntiles;
        const int64_t rbeg = P.seg_rec[seg] + split * P.rpi;
        const int64_t rend = min(rbeg + P.rpi, P.seg_rec[seg + 1]);
        // bins of this thread
        BinDev bd[BPT];
        bool valid[BPT];
        int64_t bin[BPT];
#pragma unroll
        for (int q = 0; q < BPT; q++) {
            bin[q] = tile * TILE + q * K2_THREADS + tid;
            valid[q] = bin[q] < P.nb;
            const int64_t o = valid[q] ? bin[q] : 0;
            const double X = P.xyz[o], Y = P.xyz[P.nb + o], Zc = P.xyz[2 * P.nb + o];
            const double ir = 1.0 / sqrt(X * X + Y * Y + Zc * Zc);
            bd[q].bin = o;
            bd[q].ux = X * ir;
            bd[q].uy = Y * ir;
            bd[q].uz = Zc * ir;
            bd[q].fx = (float)bd[q].ux;
            bd[q].fy = (float)bd[q].uy;
            bd[q].fz = (float)bd[q].uz;
            const double sg = bd[q].uz <= 0.0 ? 1.0 : -1.0;
            bd[q].sz = (float)(bd[q].uz + sg);
            bd[q].sg = (float)sg;
            const int64_t oh = (o % P.nphi) + P.nphi * P.theta_i;
            const double Xh = P.xyz[oh], Yh = P.xyz[P.nb + oh], Zh = P.xyz[2 * P.nb + oh];
            const double irh = 1.0 / sqrt(Xh * Xh + Yh * Yh + Zh * Zh);
            bd[q].hx = (float)(Xh * irh);
            bd[q].hy = (float)(Yh * irh);
            bd[q].hsz = (float)(Zh * irh + (double)P.sgh);
        }
        double acc64[BPT][8];
#pragma unroll
        for (int q = 0; q < BPT; q++)
#pragma unroll
            for (int c = 0; c < 8; c++) acc64[q][c] = 0.0;
        const int64_t nrec = rend - rbeg;
        const int64_t nchunk = (nrec + K2_CH - 1) / K2_CH;
        if (tid == 0) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            for (int64_t c = 0; c < nchunk && c < K2_NST; c++) {
                const int64_t n = min((int64_t)K2_CH, nrec - c * K2_CH);
                bulk_load(smem_u32(&sbuf[c][0]), P.recs + rbeg + c * K2_CH,
                          (uint32_t)(n * sizeof(K2Rec)), smem_u32(&bars[c]));
            }
        }
        bool timed_out = false;
        int64_t c_out = 0;
        for (int64_t c = 0; c < nchunk; c++) {
            const int st = (int)(c % K2_NST);
            const bool ok = mbar_wait(smem_u32(&bars[st]), parity[st]);
            parity[st] ^= 1u;
            if (__syncthreads_or(!ok)) {
                timed_out = true;
                c_out = c;
                break;
            }
            const int n = (int)min((int64_t)K2_CH, nrec - c * K2_CH);
            float acc[BPT][8];
#pragma unroll
            for (int q = 0; q < BPT; q++)
#pragma unroll
                for (int cc = 0; cc < 8; cc++) acc[q][cc] = 0.0f;
            const K2Fov *fv = FAST ? P.fovs + rbeg + c * K2_CH : nullptr;
            for (int j = 0; j < n; j++) {
                const int64_t ri = rbeg + c * K2_CH + j;
                k2_record<BPT, FAST>(sbuf[st][j], FAST ? fv + j : nullptr, bd, valid, acc, P.k,
                                     P.hkR, P.sgh, P.xyz, P.nb, P.rlo + (ri >> 1) * 3, (int)(ri & 1));
            }
#pragma unroll
            for (int q = 0; q < BPT; q++)
#pragma unroll
                for (int cc = 0; cc < 8; cc++) acc64[q][cc] += (double)acc[q][cc];
            __syncthreads();  // every thread is done with stage st
            if (tid == 0 && c + K2_NST < nchunk) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                const int64_t c2 = c + K2_NST;
                const int64_t n2 = min((int64_t)K2_CH, nrec - c2 * K2_CH);
                bulk_load(smem_u32(&sbuf[st][0]), P.recs + rbeg + c2 * K2_CH,
                          (uint32_t)(n2 * sizeof(K2Rec)), smem_u32(&bars[st]));
            }
        }
        unsigned *tk = P.tickets + seg * P.ntiles + tile;
        if (timed_out) {
            if (tid == 0) {
                atomicOr(P.err, 4);
                atomicMax(tk, kTicketPoison);
                // bounded wait for this CTA's bulk copies still in flight
                for (int64_t c2 = c_out; c2 < min(nchunk, c_out + K2_NST); c2++) {
                    const int s2 = (int)(c2 % K2_NST);
                    mbar_wait(smem_u32(&bars[s2]), c2 == c_out ? parity[s2] ^ 1u : parity[s2]);
                }
            }
            return;
        }
        ordered_add<BPT>(P.ws + seg * 8 * P.nb, P.nb, tk, (unsigned)split, valid, bin, acc64, &s_ok,
                         P.err);
    }
}

// ---------------------------------------------- packed two-facet main kernel
//
// Same arithmetic as k2_record, evaluated for two facets at once with packed
// FP32x2 instructions (FFMA2/FMUL2/FADD2 of sm_100): the x lane carries the
// even record of a K2Pair, the y lane the odd one.  The bin's data are
// loop-invariant broadcast pairs.  Special-function calls, the sort of the
// three phases and the FP64 phase stay per facet.

__device__ __forceinline__ float2 bc2(float v) { return make_float2(v, v); }
// the special-function unit's approximations with subnormal inputs flushed
// to zero (the arguments here are phases and squared norms, never subnormal)
__device__ __forceinline__ float sin_fz(float x) {
    float r;
    asm("sin.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float cos_fz(float x) {
    float r;
    asm("cos.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float rsqrt_fz(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 sel2(bool px, bool py, float2 a, float2 b) {
    return make_float2(px ? a.x : b.x, py ? a.y : b.y);
}

// A bin of the packed kernel.  The direction is held as s = u + sg z, sg = +1 in
// the hemisphere of the incidence direction (0,0,-1) and -1 in the other, so
// that sz = uz + sg (formed in FP64, rounded once) is small and exact to FP32
// precision near both poles; u = (fx, fy, sz - sg).  The forward-bodge bin
// direction, used near the poles only, is kept in shared memory (slot hslot of
// the kernel's bodge table) in the same form with the kernel's sgh.
struct BinPk {
    double ux, uy, uz;     // unit bin direction, FP64
    float2 fx, fy, sz, sg; // broadcast FP32 pairs
    int hslot;
    bool pole;             // within reach of the forward bodge (|uz| near 1) for some record
    int64_t bin;           // bin index
};
constexpr int K2P_HB = K2_THREADS * 2;  // bodge table slots (bins per thread <= 2)

// sin(h)/h below h = 0.5, where the MUFU sine's absolute error would be a large
// relative one: 1 + c1 h^2 + c2 h^4 with c1, c2 the minimax fit to the relative
// error on [0, 0.5] (Lawson's iteration: 1.2e-7, 1.6e-7 evaluated in FP32)
__device__ __forceinline__ float2 sinc_series(float2 h) {
    const float2 hh = mul2(h, h);
    return fma2(hh, fma2(hh, bc2(8.264339e-3f), bc2(-1.6666131e-1f)), bc2(1.0f));
}

// 2 sc g for each lane, g the second divided difference of e^{ix} at the full
// phases 2 t1, 2 t2, 2 t3, from the half phases t, and sc = 1 / (|h| tt) =
// rsqrt(hn2 tt^2) the normalisation of the polarisation block.  With the half
// phases sorted (lo <= mid <= hi) the edge midpoints of the full phases are
// lo + mid and mid + hi and the half gaps mid - lo and hi - mid, each one
// operation.  Formed in two halves: tri_front from the three half phases alone,
// tri_back with the polarisation block's |h|^2 and tt (for the shared reciprocal
// square root below).
struct TriF {
    float2 lo, mid, hi, Dh, h1, h2, s1, k1, s2, k2, p12, S1, S2;
};
__device__ __forceinline__ TriF tri_front(float2 t1, float2 t2, float2 t3) {
    TriF F;
    float2 lo, hi, mid;
    lo.x = fminf(t1.x, t2.x);
    hi.x = fmaxf(t1.x, t2.x);
    mid.x = fmaxf(lo.x, fminf(hi.x, t3.x));
    lo.x = fminf(lo.x, t3.x);
    hi.x = fmaxf(hi.x, t3.x);
    lo.y = fminf(t1.y, t2.y);
    hi.y = fmaxf(t1.y, t2.y);
    mid.y = fmaxf(lo.y, fminf(hi.y, t3.y));
    lo.y = fminf(lo.y, t3.y);
    hi.y = fmaxf(hi.y, t3.y);
    const float2 Dh = add2(hi, neg2(lo));  // half of the largest gap D
    const float2 h1 = add2(mid, neg2(lo));
    const float2 h2 = add2(hi, neg2(mid));
    const float2 c1 = add2(lo, mid), c2 = add2(mid, hi);
    float2 s1, k1, s2, k2;
    s1 = make_float2(sin_fz(c1.x), sin_fz(c1.y));
    k1 = make_float2(cos_fz(c1.x), cos_fz(c1.y));
    s2 = make_float2(sin_fz(c2.x), sin_fz(c2.y));
    k2 = make_float2(cos_fz(c2.x), cos_fz(c2.y));
    // With a1 = max(h1, .5) and a2 = max(h2, .5), 2 sc g = scr (S1 e^{i c1} -
    // S2 e^{i c2}) (imaginary unit and sign aside), S1 = sinc(h1) a1 a2,
    // S2 = sinc(h2) a1 a2 and scr = sc / (a1 a2 Dh): one reciprocal square root,
    // rsqrt(hn2 (tt a1 a2 Dh)^2), gives the polarisation block's normalisation,
    // 1/a1, 1/a2 and 2/D.  Where h >= 0.5, sinc(h1) a1 a2 = a2 sin(h1).
    const float2 a1 = make_float2(fmaxf(h1.x, 0.5f), fmaxf(h1.y, 0.5f));
    const float2 a2 = make_float2(fmaxf(h2.x, 0.5f), fmaxf(h2.y, 0.5f));
    const float2 p12 = mul2(a1, a2);
    F.lo = lo; F.mid = mid; F.hi = hi; F.Dh = Dh; F.h1 = h1; F.h2 = h2;
    F.s1 = s1; F.k1 = k1; F.s2 = s2; F.k2 = k2; F.p12 = p12;
    F.S1 = mul2(make_float2(sin_fz(h1.x), sin_fz(h1.y)), a2);
    F.S2 = mul2(make_float2(sin_fz(h2.x), sin_fz(h2.y)), a1);
    return F;
}

__device__ __forceinline__ void tri_back(const TriF &F, float2 hn2, float2 tt, float2 &gx, float2 &gy) {
    const float2 lo = F.lo, mid = F.mid, hi = F.hi, Dh = F.Dh, h1 = F.h1, h2 = F.h2;
    const float2 s1 = F.s1, k1 = F.k1, s2 = F.s2, k2 = F.k2, p12 = F.p12;
    const float2 q = mul2(mul2(p12, Dh), tt);
    const float2 hq = mul2(hn2, mul2(q, q));
    const float2 scr = make_float2(rsqrt_fz(hq.x), rsqrt_fz(hq.y));
    float2 S1 = F.S1, S2 = F.S2;
    // below h = 0.5 sinc(h) from its series, evaluated only when a lane of the
    // warp needs it (small gaps occur near a facet's specular and forward
    // directions), one vote for both
    const bool ax = h1.x < 0.5f, ay = h1.y < 0.5f, bx = h2.x < 0.5f, by = h2.y < 0.5f;
    if (__any_sync(0xffffffffu, ax || ay || bx || by)) {
        S1 = sel2(ax, ay, mul2(sinc_series(h1), p12), S1);
        S2 = sel2(bx, by, mul2(sinc_series(h2), p12), S2);
        gx = mul2(fma2(S1, s1, neg2(mul2(S2, s2))), scr);
        gy = mul2(fma2(S2, k2, neg2(mul2(S1, k1))), scr);
        if (Dh.x < 0.125f || Dh.y < 0.125f) {
            // all three full phases within 0.25 rad: Taylor series about the middle
            // phase, g = e^{2i mid} sum_n i^(n+2)/(n+2)! q_n(ya, yc) with the complete
            // homogeneous q_n of the full-phase offsets 2 ya, 2 yc (2^n folded into
            // the coefficients)
            const float2 ya = add2(lo, neg2(mid)), yc = add2(hi, neg2(mid));
            const float2 q1 = add2(ya, yc);
            const float2 ya2 = mul2(ya, ya);
            const float2 q2 = fma2(yc, q1, ya2);
            const float2 ya3 = mul2(ya2, ya);
            const float2 q3 = fma2(yc, q2, ya3);
            const float2 ya4 = mul2(ya3, ya);
            const float2 q4 = fma2(yc, q3, ya4);
            const float2 q5 = fma2(yc, q4, mul2(ya4, ya));
            const float2 q6 = fma2(yc, q5, mul2(ya4, ya2));
            const float2 ht = mul2(mul2(hn2, tt), tt);
            const float2 tsc = make_float2(2.0f * rsqrt_fz(ht.x), 2.0f * rsqrt_fz(ht.y));
            const float2 re = mul2(tsc, fma2(q6, bc2(1.0f / 630.0f),
                                             fma2(q4, bc2(-1.0f / 45.0f), fma2(q2, bc2(1.0f / 6.0f), bc2(-0.5f)))));
            const float2 im = mul2(tsc, fma2(q5, bc2(-2.0f / 315.0f),
                                             fma2(q3, bc2(1.0f / 15.0f), mul2(q1, bc2(-1.0f / 3.0f)))));
            const float2 m2 = add2(mid, mid);
            float2 sm, cm;
            sm = make_float2(sin_fz(m2.x), sin_fz(m2.y));
            cm = make_float2(cos_fz(m2.x), cos_fz(m2.y));
            const float2 sx = fma2(cm, re, neg2(mul2(sm, im)));
            const float2 sy = fma2(cm, im, mul2(sm, re));
            gx = sel2(Dh.x < 0.125f, Dh.y < 0.125f, sx, gx);
            gy = sel2(Dh.x < 0.125f, Dh.y < 0.125f, sy, gy);
        }
    } else {
        gx = mul2(fma2(S1, s1, neg2(mul2(S2, s2))), scr);
        gy = mul2(fma2(S2, k2, neg2(mul2(S1, k1))), scr);
    }
}

// Two adjacent float2 fields of a record pair from one 16-byte shared-memory load
// (every such field pair of K2Pair starts on a 16-byte boundary).
__device__ __forceinline__ void ld22(const float2 *p, float2 &a, float2 &b) {
    const float4 v = *reinterpret_cast<const float4 *>(p);
    a = make_float2(v.x, v.y);
    b = make_float2(v.z, v.w);
}

template <bool FAST>
__device__ __forceinline__ void k2_pair(const K2Pair &P, const K2Fov *fv, const BinPk &B,
                                        float2 (&acc)[8], float2 nkh, float2 hkRh, float2 sgh,
                                        const float (&hb)[3][K2P_HB], bool lo_ok, bool hi_ok,
                                        const double *__restrict__ xyz, int64_t nb,
                                        const float2 *__restrict__ rl) {
    // far-field half phase per facet: FP64 k u.c / 2, reduced mod pi
    float2 rf;
    {
        const double2 k0 = *reinterpret_cast<const double2 *>(&P.kc[0][0]);
        const double2 k1 = *reinterpret_cast<const double2 *>(&P.kc[1][0]);
        const double2 k2 = *reinterpret_cast<const double2 *>(&P.kc[2][0]);
        const double ka = fma(B.uz, k2.x, fma(B.uy, k1.x, B.ux * k0.x));
        const double nq = fma(ka, kInvPi, kMagic) - kMagic;
        rf.x = (float)fma(-nq, kPi, ka);
        const double kb = fma(B.uz, k2.y, fma(B.uy, k1.y, B.ux * k0.y));
        const double nb = fma(kb, kInvPi, kMagic) - kMagic;
        rf.y = (float)fma(-nb, kPi, kb);
    }
    const float2 one = bc2(1.0f);
    float2 eps0, eps1, eps2, pb;
    ld22(&P.eps[0], eps0, eps1);
    ld22(&P.eps[2], eps2, pb);
    // a = u . eps = s . eps - sg eps_z
    const float2 a = fma2(neg2(B.sg), eps2, fma2(B.sz, eps2, fma2(B.fy, eps1, mul2(B.fx, eps0))));
    // with y = b - a^2: half phase hkRh y (1 + a) - rf, and
    // opa2 = 1 + a + 1.5 a^2 - 0.5 b = (1 + a) - 0.5 y + a^2
    const float2 opa = add2(one, a);
    const float2 y = fma2(neg2(a), a, pb);
    const float2 ph = fma2(mul2(hkRh, y), opa, neg2(rf));
    const float2 opa2 = fma2(a, a, fma2(bc2(-0.5f), y, opa));
    // The bin direction enters through s = u + sg z (sg = +1 in the hemisphere of
    // the incidence direction (0,0,-1), -1 in the other), which is small and known
    // to full FP32 precision near both poles.  With inc = -R z (the incidence
    // direction in the aperture frame), k = R u opa2 + nea opa = ks + sg opa2 inc
    // with ks = R s opa2 + nea opa, and the normal of the scattering plane is
    // h = inc x k = inc x ks: no cancellation of nearly parallel unit vectors near
    // the forward and backward directions, where |h| is small.
    float2 ks0, ks1, ks2;
    {
        float2 r0, r1, r2, r3, r4, r5, r6, r7, r8, n0, n1, n2;
        ld22(&P.R[0], r0, r1);
        ld22(&P.R[2], r2, r3);
        ld22(&P.R[4], r4, r5);
        ld22(&P.R[6], r6, r7);
        ld22(&P.R[8], r8, n0);
        ld22(&P.nea[1], n1, n2);
        const float2 w0 = fma2(r2, B.sz, fma2(r1, B.fy, mul2(r0, B.fx)));
        const float2 w1 = fma2(r5, B.sz, fma2(r4, B.fy, mul2(r3, B.fx)));
        const float2 w2 = fma2(r8, B.sz, fma2(r7, B.fy, mul2(r6, B.fx)));
        ks0 = fma2(w0, opa2, mul2(n0, opa));
        ks1 = fma2(w1, opa2, mul2(n1, opa));
        ks2 = fma2(w2, opa2, mul2(n2, opa));
    }
    float2 kzc, inc0, inc1, inc2;
    ld22(&P.kzc, kzc, inc0);
    ld22(&P.inc[1], inc1, inc2);
    const float2 so = mul2(B.sg, opa2);
    float2 kx = fma2(so, inc0, ks0);
    const float2 ky = fma2(so, inc1, ks1);
    float2 kz = fma2(so, inc2, ks2);
    // aperture wave vector (halved with the phases)
    float2 kxx, kyy;
    {
        float2 kp0, kp1;
        ld22(&P.kp[0], kp0, kp1);
        kxx = fma2(nkh, kx, kp0);
        kyy = fma2(nkh, ky, kp1);
    }
    // the divided difference's phases, sort, sines and cosines: independent of
    // the polarisation block and its rare branch, so formed ahead of the branch
    // (one basic block with the direction arithmetic for the scheduler)
    TriF tf;
    {
        float2 vx0, vx1, vx2, vy0, vy1, vy2;
        ld22(&P.vx[0], vx0, vx1);
        ld22(&P.vx[2], vx2, vy0);
        ld22(&P.vy[1], vy1, vy2);
        const float2 t1 = fma2(kyy, vy0, fma2(kxx, vx0, ph));
        const float2 t2 = fma2(kyy, vy1, fma2(kxx, vx1, ph));
        const float2 t3 = fma2(kyy, vy2, fma2(kxx, vx2, ph));
        tf = tri_front(t1, t2, t3);
    }
    // Polarisation matrix [[d, e], [-e, d]] (see k2_record for the forms) and
    // the rotation into the scattering plane, with their normalisations folded
    // into one factor: with s = sqrt(tt) and hc = h / |h|,
    //   d = d1 / s, e = e1 / s, p = P1 / (|h| s), rr = R1 / (|h| s),
    // so A = p d + rr e = sc (P1 d1 + R1 e1) and B = sc (P1 e1 - R1 d1) with
    // sc = 1 / (|h| tt) = rsqrt(|h|^2 tt^2).  The in-plane rotation of the set-up
    // puts prop2 in the x-z plane (src/diff_mod.f90:540-559), so Ky = 0 up to
    // rounding and d1 = (sqrt(1 - Ky^2)/2) (kzc tt - kz), e1 = (sqrt(1 - Ky^2)/2)(-kx kyc)
    // (the Kx Ky term is below 1e-16 and left out); the common factor is in the
    // record's amplitudes and sc in the divided difference.
    // Main path: |ky| < 0.999999 (no clamp) and no forward bodge, so kyc = ky
    // and tt = kx^2 + kz^2; h = inc x (kx, ky, kz) = inc x ks.
    const float2 tr = fma2(kx, kx, mul2(kz, kz));
    float2 tt = tr;
    float2 d1 = fma2(kzc, tr, neg2(kz));
    float2 e1 = mul2(neg2(kx), ky);
    float2 hx = fma2(inc1, ks2, neg2(mul2(inc2, ks1)));
    float2 hy = fma2(inc2, ks0, neg2(mul2(inc0, ks2)));
    float2 hz = fma2(inc0, ks1, neg2(mul2(inc1, ks0)));
    // P1 = p |h| s = hy tt - kyc (hx kx + hz kz), from m = (-kx ky / s, s, -kz ky / s).
    // Where h is normal to q = (kx, kyc, kz), hx kx + hz kz = -hy kyc and
    // P1 = hy (tt + kyc^2) = hy |q|^2 = hy (|q| = 1 up to rounding; on the clamp
    // tt + kyc^2 = 1 - c^2 + c^2); the forward bodge takes the general form.
    // Inside the clamp evo2 = (-kz, 0, kx) / s, so R1 = rr |h| s = hz kx - hx kz.
    float2 P1 = hy, R1;
    const bool cx = tr.x <= kOneMinusClampSq, cy = tr.y <= kOneMinusClampSq;
    if (B.pole || cx || cy) {
        if (cx || cy) {
            // on the clamp: kx and kz from v = u - sigma R_1 (see clamp_v)
            float2 a0, a1, a2, a3, a4, a5, c6, c7, c8, n0, n1, n2;
            ld22(&P.R[0], a0, a1);
            ld22(&P.R[2], a2, a3);
            ld22(&P.R[4], a4, a5);
            ld22(&P.R[6], c6, c7);
            ld22(&P.R[8], c8, n0);
            ld22(&P.nea[1], n1, n2);
            const float2 l0 = rl[0], l1 = rl[1], l2 = rl[2];
            const float sx = ky.x < 0.0f ? -1.0f : 1.0f, sy = ky.y < 0.0f ? -1.0f : 1.0f;
            const float2 v0 = make_float2(clamp_v(a3.x, l0.x, B.ux, sx), clamp_v(a3.y, l0.y, B.ux, sy));
            const float2 v1 = make_float2(clamp_v(a4.x, l1.x, B.uy, sx), clamp_v(a4.y, l1.y, B.uy, sy));
            const float2 v2 = make_float2(clamp_v(a5.x, l2.x, B.uz, sx), clamp_v(a5.y, l2.y, B.uz, sy));
            const float2 kxa = fma2(fma2(a2, v2, fma2(a1, v1, mul2(a0, v0))), opa2, mul2(n0, opa));
            const float2 kza = fma2(fma2(c8, v2, fma2(c7, v1, mul2(c6, v0))), opa2, mul2(n2, opa));
            kx = sel2(cx, cy, kxa, kx);
            kz = sel2(cx, cy, kza, kz);
        }
        // near the poles (the forward bodge) or on the clamp: ky clamped to
        // +-0.999999 and tt to 1 - 0.999999^2 as in src/diff_mod.f90
        const float2 kyc = make_float2(fminf(fmaxf(ky.x, -0.999999f), 0.999999f),
                                       fminf(fmaxf(ky.y, -0.999999f), 0.999999f));
        tt = make_float2(fmaxf(tr.x, kOneMinusClampSq), fmaxf(tr.y, kOneMinusClampSq));
        d1 = fma2(kzc, tt, neg2(kz));
        e1 = mul2(neg2(kx), kyc);
        bool bx = false, by = false;
        if (B.pole) {
            // the forward bodge (src/diff_mod.f90:630-633) can apply only in bins near
            // the poles; dinc = inc . (kx, kyc, kz)
            const float2 dinc = fma2(inc2, kz, fma2(inc1, kyc, mul2(inc0, kx)));
            bx = !(fabsf(dinc.x) < 0.999f);
            by = !(fabsf(dinc.y) < 0.999f);
            if (bx || by) {
                // the bodge direction in the s form: hs = uh + sgh z, uh . eps = hs . eps - sgh eps_z,
                // h = inc x (R hs oh2 + nea oh)
                const float2 hx_ = bc2(hb[0][B.hslot]), hy_ = bc2(hb[1][B.hslot]),
                             hsz = bc2(hb[2][B.hslot]);
                float2 ah = fma2(hsz, eps2, fma2(hy_, eps1, mul2(hx_, eps0)));
                ah = fma2(neg2(sgh), eps2, ah);
                const float2 oh = add2(one, ah);
                const float2 oh2 = fma2(ah, fma2(bc2(1.5f), ah, one), fma2(bc2(-0.5f), pb, one));
                const float2 vx = fma2(fma2(P.R[2], hsz, fma2(P.R[1], hy_, mul2(P.R[0], hx_))), oh2,
                                       mul2(P.nea[0], oh));
                const float2 vy = fma2(fma2(P.R[5], hsz, fma2(P.R[4], hy_, mul2(P.R[3], hx_))), oh2,
                                       mul2(P.nea[1], oh));
                const float2 vz = fma2(fma2(P.R[8], hsz, fma2(P.R[7], hy_, mul2(P.R[6], hx_))), oh2,
                                       mul2(P.nea[2], oh));
                const float2 gx = fma2(inc1, vz, neg2(mul2(inc2, vy)));
                const float2 gy = fma2(inc2, vx, neg2(mul2(inc0, vz)));
                const float2 gz = fma2(inc0, vy, neg2(mul2(inc1, vx)));
                const float2 gP = fma2(gy, tt, neg2(mul2(kyc, fma2(gx, kx, mul2(gz, kz)))));
                hx = sel2(bx, by, gx, hx);
                hy = sel2(bx, by, gy, hy);
                hz = sel2(bx, by, gz, hz);
                P1 = sel2(bx, by, gP, P1);
            }
        }
        if (cx || cy) {
            // a lane on the clamp: outside the bodge, h = inc x (kx, kyc, kz) takes the
            // clamped ky (q_y = ks1 + kyc - ky); evo2 = normalise(k x m) with the clamped
            // ky, R1 = s (h . evo2)
            const float2 qy = add2(ks1, add2(kyc, neg2(ky)));
            const float2 fx = fma2(inc1, ks2, neg2(mul2(inc2, qy)));
            const float2 fz = fma2(inc0, qy, neg2(mul2(inc1, ks0)));
            const bool ux = cx && !bx, uy = cy && !by;
            hx = sel2(ux, uy, fx, hx);
            hz = sel2(ux, uy, fz, hz);
            const float2 rs = make_float2(rsqrtf(tt.x), rsqrtf(tt.y));
            const float2 s = mul2(tt, rs), kyrs = mul2(kyc, rs);
            const float2 m0 = neg2(mul2(kx, kyrs)), m1 = s, m2 = neg2(mul2(kz, kyrs));
            float2 ex = fma2(kyc, m2, neg2(mul2(kz, m1)));
            float2 ey = fma2(kz, m0, neg2(mul2(kx, m2)));
            float2 ez = fma2(kx, m1, neg2(mul2(kyc, m0)));
            const float2 en2 = fma2(ez, ez, fma2(ey, ey, mul2(ex, ex)));
            const float2 ne = make_float2(cx ? rsqrtf(en2.x) : 1.0f, cy ? rsqrtf(en2.y) : 1.0f);
            const float2 rc = mul2(mul2(s, ne), fma2(hz, ez, fma2(hy, ey, mul2(hx, ex))));
            R1 = sel2(cx, cy, rc, fma2(hz, kx, neg2(mul2(hx, kz))));
        } else {
            R1 = fma2(hz, kx, neg2(mul2(hx, kz)));
        }
    } else {
        R1 = fma2(hz, kx, neg2(mul2(hx, kz)));
    }
    const float2 hn2 = fma2(hz, hz, fma2(hy, hy, mul2(hx, hx)));
    const float2 A = fma2(P1, d1, mul2(R1, e1));
    const float2 Bc = fma2(P1, e1, neg2(mul2(R1, d1)));
    // aperture integral on the half phases, its second half (the normalisation
    // sc needs the polarisation block's |h| and tt): 2 sc g
    float2 gx, gy;
    tri_back(tf, hn2, tt, gx, gy);
    // [[A, B], [-B, A]] is diagonal in the circular basis: with z = A - iB the
    // columns' u+ take z, their u- take conj(z).  q+ = g z, q- = g conj(z).
    const float2 gyB = mul2(gy, Bc), gxB = mul2(gx, Bc);
    float2 qpr = fma2(gx, A, gyB), qmr = fma2(gx, A, neg2(gyB));
    float2 qpi = fma2(gy, A, neg2(gxB)), qmi = fma2(gy, A, gxB);
    bool ok_x = lo_ok, ok_y = hi_ok;
    if (FAST) {
        // the field-of-view test (direction from the facet centre, lab frame)
        const float2 dx = fma2(B.fx, opa, neg2(eps0));
        const float2 dy = fma2(B.fy, opa, neg2(eps1));
        const float2 dz = fma2(add2(B.sz, neg2(B.sg)), opa, neg2(eps2));
        const K2Fov &fa = fv[0], &fb = fv[1];
        const float dpx = fmaf(dz.x, fa.p0[2], fmaf(dy.x, fa.p0[1], dx.x * fa.p0[0]));
        const float dpy = fmaf(dz.y, fb.p0[2], fmaf(dy.y, fb.p0[1], dx.y * fb.p0[0]));
        bool in_x = !(dpx < fa.cos_fov), in_y = !(dpy < fb.cos_fov);
        if (ok_x && fabsf(dpx - fa.cos_fov) < fa.tol) in_x = fov_exact(fa, xyz, nb, B.bin);
        if (ok_y && fabsf(dpy - fb.cos_fov) < fb.tol) in_y = fov_exact(fb, xyz, nb, B.bin);
        ok_x = ok_x && in_x;
        ok_y = ok_y && in_y;
    }
    if (FAST || !lo_ok || !hi_ok) {
        // a lane outside the item or outside the field of view adds nothing
        qpr = sel2(ok_x, ok_y, qpr, bc2(0.0f));
        qmr = sel2(ok_x, ok_y, qmr, bc2(0.0f));
        qpi = sel2(ok_x, ok_y, qpi, bc2(0.0f));
        qmi = sel2(ok_x, ok_y, qmi, bc2(0.0f));
    }
    // acc: (U+ col 1, U- col 1, U+ col 2, U- col 2), re/im
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const float2 qr = (c & 1) ? qmr : qpr, qi = (c & 1) ? qmi : qpi;
        float2 ur, ui;
        ld22(&P.amp[2 * c], ur, ui);
        acc[2 * c] = fma2(qr, ur, fma2(neg2(qi), ui, acc[2 * c]));
        acc[2 * c + 1] = fma2(qr, ui, fma2(qi, ur, acc[2 * c + 1]));
    }
}

// Record pairs per shared-memory stage: 44 for the full sum (three stages, 44 KB,
// four CTAs per SM); 32 with the field-of-view cull, whose per-stage keep masks are
// two 32-bit ballot words of the stage's 64 records.
constexpr int K2P_CH_FULL = 44, K2P_CH_FOV = 32;

// The record's per-bin test passes no bin of the tile when the angle between
// prop0 and the tile centre exceeds fovm + psi (fovm includes the parallax
// and rounding margin); compared through cosines with a further 1e-6 margin.
__device__ __forceinline__ bool cone_culled(const K2Fov &f, const K2Cone &t) {
    if (!(f.fovm + t.psi < 3.14159f)) return false;
    const float d = fmaf(f.p0[2], t.c[2], fmaf(f.p0[1], t.c[1], f.p0[0] * t.c[0]));
    return d < fmaf(f.cos_fovm, t.cos_psi, -f.sin_fovm * t.sin_psi) - 1e-6f;
}

struct K2PkArgs {
    const float2 *rlo;  // R_1 - (float)R_1, pair layout (3 per pair)
    const K2Pair *pairs;
    const K2Fov *fovs;
    const int *perm;        // is_fast_diff: tile-major bin order (-1: padding)
    const K2Cone *cones;    // is_fast_diff: cone of each tile
    const int64_t *seg_rec;
    const int64_t *item_pre;
    int64_t nseg;
    int64_t rpi;
    int64_t ntiles;
    const double *xyz;
    int64_t nb, nphi;
    int64_t theta_i;
    float k;
    float hkR;
    float sgh;   // +1 when the bodge row theta_i lies in the hemisphere of (0,0,-1), else -1
    const unsigned *epsmax;  // float bits of a bound of |com| / R over the records
    double *ws;         // [seg][8][nb]
    unsigned *tickets;  // [seg][tile], splits added so far
    unsigned long long *counter;
    int *err;
};

template <int BPT, bool FAST>
__global__ void __launch_bounds__(K2_THREADS, BPT == 1 ? 4 : 0) k2_main_pk_kernel(K2PkArgs P) {
    constexpr int CH = FAST ? K2P_CH_FOV : K2P_CH_FULL;
    __shared__ __align__(128) K2Pair sbuf[K2_NST][CH];
    __shared__ __align__(8) uint64_t bars[K2_NST];
    __shared__ long long s_item;
    __shared__ unsigned s_keep[2];  // is_fast_diff: records of the stage not culled for the tile
    __shared__ float s_hb[3][K2P_HB];  // forward-bodge bin directions of this CTA's bins (s form)
    __shared__ int s_ok;
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int s = 0; s < K2_NST; s++) mbar_init(smem_u32(&bars[s]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    uint32_t parity = 0;  // bit s: phase of stage s
    const int64_t total = P.item_pre[P.nseg];
    constexpr int64_t TILE = (int64_t)K2_THREADS * BPT;
    // half phases: -k/2 and k R / 4
    const float2 nkh = bc2(-0.5f * P.k), hkRh = bc2(0.5f * P.hkR), sgh = bc2(P.sgh);
    // bins with |uz| below pole_cos are out of reach of the forward bodge for every
    // record: |inc . k - (-uz)| <= 2 |com| / R for the direction k from a facet centre
    const float pole_cos = 0.999f - 2.0f * __uint_as_float(*P.epsmax) - 1e-5f;
    for (;;) {
        if (tid == 0) s_item = (long long)atomicAdd(P.counter, 1ull);
        __syncthreads();
        const int64_t item = s_item;
        if (item >= total) break;
        int64_t lo = 0, hi = P.nseg;
        while (hi - lo > 1) {
            const int64_t m = (lo + hi) >> 1;
            if (P.item_pre[m] <= item)
                lo = m;
            else
                hi = m;
        }
        const int64_t seg = lo;
        const int64_t local = item - P.item_pre[seg];
        const int64_t split = local / P.ntiles, tile = local % P.ntiles;
        const int64_t rbeg = P.seg_rec[seg] + split * P.rpi;
        const int64_t rend = min(rbeg + P.rpi, P.seg_rec[seg + 1]);
        BinPk bd[BPT];
        bool valid[BPT];
        int64_t bin[BPT];
#pragma unroll
        for (int q = 0; q < BPT; q++) {
            const int64_t li = tile * TILE + q * K2_THREADS + tid;
            bin[q] = FAST ? (int64_t)P.perm[li] : li;
            valid[q] = FAST ? bin[q] >= 0 : bin[q] < P.nb;
            const int64_t o = valid[q] ? bin[q] : 0;
            const double X = P.xyz[o], Y = P.xyz[P.nb + o], Zc = P.xyz[2 * P.nb + o];
            const double ir = 1.0 / sqrt(X * X + Y * Y + Zc * Zc);
            bd[q].bin = o;
            bd[q].ux = X * ir;
            bd[q].uy = Y * ir;
            bd[q].uz = Zc * ir;
            bd[q].fx = bc2((float)bd[q].ux);
            bd[q].fy = bc2((float)bd[q].uy);
            const double sg = bd[q].uz <= 0.0 ? 1.0 : -1.0;
            bd[q].sz = bc2((float)(bd[q].uz + sg));
            bd[q].sg = bc2((float)sg);
            bd[q].pole = !(fabs(bd[q].uz) < (double)pole_cos);
            const int64_t oh = (o % P.nphi) + P.nphi * P.theta_i;
            const double Xh = P.xyz[oh], Yh = P.xyz[P.nb + oh], Zh = P.xyz[2 * P.nb + oh];
            const double irh = 1.0 / sqrt(Xh * Xh + Yh * Yh + Zh * Zh);
            bd[q].hslot = q * K2_THREADS + tid;
            s_hb[0][bd[q].hslot] = (float)(Xh * irh);
            s_hb[1][bd[q].hslot] = (float)(Yh * irh);
            s_hb[2][bd[q].hslot] = (float)(Zh * irh + (double)P.sgh);
        }
        double acc64[BPT][8];
#pragma unroll
        for (int q = 0; q < BPT; q++)
#pragma unroll
            for (int c = 0; c < 8; c++) acc64[q][c] = 0.0;
        K2Cone cone;
        if (FAST) cone = P.cones[tile];
        // record pairs [p0, p1) cover records [rbeg, rend)
        const int64_t p0 = rbeg >> 1, p1 = (rend + 1) >> 1;
        const int64_t npair = p1 - p0;
        const int64_t nchunk = (npair + CH - 1) / CH;
        if (tid == 0) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            for (int64_t c = 0; c < nchunk && c < K2_NST; c++) {
                const int64_t n = min((int64_t)CH, npair - c * CH);
                bulk_load(smem_u32(&sbuf[c][0]), P.pairs + p0 + c * CH,
                          (uint32_t)(n * sizeof(K2Pair)), smem_u32(&bars[c]));
            }
        }
        bool timed_out = false;
        int64_t c_out = 0;
        for (int64_t c = 0; c < nchunk; c++) {
            const int st = (int)(c % K2_NST);
            const bool ok = mbar_wait(smem_u32(&bars[st]), (parity >> st) & 1u);
            parity ^= 1u << st;
            const int n = (int)min((int64_t)CH, npair - c * CH);
            if (!FAST && ok && tid < 39) {
                // The item's first pair (odd rbeg) and last pair (odd rend) hold a
                // record of another item or the array's padding: that half takes a
                // copy of the pair's other record with zero amplitude, so the pair
                // loop needs no per-pair range test.  Threads 0-2 copy the FP64
                // phase, threads 3-38 the 36 float2 fields from eps on (the last 8
                // are the amplitudes); the barrier below publishes the copy.
                auto patch = [&](int j, int src, int dst) {
                    K2Pair &Q = sbuf[st][j];
                    if (tid < 3) {
                        Q.kc[tid][dst] = Q.kc[tid][src];
                    } else {
                        float2 *f = &Q.eps[0];
                        const int i = tid - 3;
                        const float v = i >= 28 ? 0.0f : (src ? f[i].y : f[i].x);
                        if (dst)
                            f[i].y = v;
                        else
                            f[i].x = v;
                    }
                };
                if (c == 0 && (rbeg & 1)) patch(0, 1, 0);
                if (c == nchunk - 1 && (rend & 1)) patch(n - 1, 0, 1);
            }
            if (__syncthreads_or(!ok)) {
                timed_out = true;
                c_out = c;
                break;
            }
            float2 acc[BPT][8];
#pragma unroll
            for (int q = 0; q < BPT; q++)
#pragma unroll
                for (int cc = 0; cc < 8; cc++) acc[q][cc] = bc2(0.0f);
            // only the item's first pair (odd rbeg) and last pair (odd rend) are partial
            const int j_lo = (c == 0 && (rbeg & 1)) ? 0 : -1;
            const int j_hi = (c == nchunk - 1 && (rend & 1)) ? n - 1 : -1;
            if (FAST) {
                // the tile cull of the stage's 2n records, one per thread of
                // warps 0 and 1: a record whose field of view misses the whole
                // tile adds nothing
                if (tid < 64) {
                    const bool keep =
                        tid < 2 * n && !cone_culled(P.fovs[2 * (p0 + c * CH) + tid], cone);
                    const unsigned m = __ballot_sync(0xffffffffu, keep);
                    if ((tid & 31) == 0) s_keep[tid >> 5] = m;
                }
                __syncthreads();
            }
            auto pair_step = [&](int j) {
                bool lo_ok = j != j_lo, hi_ok = j != j_hi;
                const K2Fov *fv = FAST ? P.fovs + 2 * (p0 + c * CH + j) : nullptr;
                if (FAST) {
                    const unsigned m = s_keep[j >> 4] >> (2 * (j & 15));
                    lo_ok = lo_ok && (m & 1u);
                    hi_ok = hi_ok && (m & 2u);
                    if (!lo_ok && !hi_ok) return;  // uniform over the CTA
                }
                // without the field-of-view test every lane adds (the edge pairs are
                // patched above; a bin beyond nb is never written out)
#pragma unroll
                for (int q = 0; q < BPT; q++)
                    k2_pair<FAST>(sbuf[st][j], fv, bd[q], acc[q], nkh, hkRh, sgh, s_hb,
                                  FAST ? (lo_ok && valid[q]) : true,
                                  FAST ? (hi_ok && valid[q]) : true, P.xyz, P.nb,
                                  P.rlo + (p0 + c * CH + j) * 3);
            };
            if (FAST) {
                // visit only the pairs with a record the tile cull kept: bit j of pm
                // is set when record 2j or 2j+1 is (the two ballot words compacted)
                auto pairs_of = [](unsigned x) {
                    x = (x | (x >> 1)) & 0x55555555u;
                    x = (x | (x >> 1)) & 0x33333333u;
                    x = (x | (x >> 2)) & 0x0F0F0F0Fu;
                    x = (x | (x >> 4)) & 0x00FF00FFu;
                    x = (x | (x >> 8)) & 0x0000FFFFu;
                    return x;
                };
                unsigned pm = pairs_of(s_keep[0]) | (pairs_of(s_keep[1]) << 16);
                while (pm) {
                    const int j = __ffs(pm) - 1;
                    pm &= pm - 1u;
                    pair_step(j);
                }
            } else {
                for (int j = 0; j < n; j++) pair_step(j);
            }
#pragma unroll
            for (int q = 0; q < BPT; q++)
#pragma unroll
                for (int cc = 0; cc < 8; cc++)
                    acc64[q][cc] += (double)acc[q][cc].x + (double)acc[q][cc].y;
            __syncthreads();
            if (tid == 0 && c + K2_NST < nchunk) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                const int64_t c2 = c + K2_NST;
                const int64_t n2 = min((int64_t)CH, npair - c2 * CH);
                bulk_load(smem_u32(&sbuf[st][0]), P.pairs + p0 + c2 * CH,
                          (uint32_t)(n2 * sizeof(K2Pair)), smem_u32(&bars[st]));
            }
        }
        unsigned *tk = P.tickets + seg * P.ntiles + tile;
        if (timed_out) {
            if (tid == 0) {
                atomicOr(P.err, 4);
                atomicMax(tk, kTicketPoison);
                // bounded wait for this CTA's bulk copies still in flight
                for (int64_t c2 = c_out; c2 < min(nchunk, c_out + K2_NST); c2++) {
                    const int s2 = (int)(c2 % K2_NST);
                    const uint32_t ph = (parity >> s2) & 1u;
                    mbar_wait(smem_u32(&bars[s2]), c2 == c_out ? ph ^ 1u : ph);
                }
            }
            return;
        }
        // back from the circular basis: a1 = (U+ + U-)/2, a2 = -i (U+ - U-)/2
        double lin[BPT][8];
#pragma unroll
        for (int q = 0; q < BPT; q++) {
            const double *u = acc64[q];
            lin[q][0] = 0.5 * (u[0] + u[2]);
            lin[q][1] = 0.5 * (u[1] + u[3]);
            lin[q][2] = 0.5 * (u[1] - u[3]);
            lin[q][3] = 0.5 * (u[2] - u[0]);
            lin[q][4] = 0.5 * (u[4] + u[6]);
            lin[q][5] = 0.5 * (u[5] + u[7]);
            lin[q][6] = 0.5 * (u[5] - u[7]);
            lin[q][7] = 0.5 * (u[6] - u[4]);
        }
        ordered_add<BPT>(P.ws + seg * 8 * P.nb, P.nb, tk, (unsigned)split, valid, bin, lin, &s_ok,
                         P.err);
    }
}

// --------------------------------------------------------------- epilogue

struct Zd {
    double re, im;
};
__device__ __forceinline__ double re_mc(Zd a, Zd b) { return a.re * b.re + a.im * b.im; }
__device__ __forceinline__ double im_mc(Zd a, Zd b) { return a.im * b.re - a.re * b.im; }

__device__ __forceinline__ void mueller16d(const Zd *S, double mu[16]) {
    const Zd a11 = S[0], a21 = S[1], a12 = S[2], a22 = S[3];
    const double p11 = re_mc(a11, a11), p12 = re_mc(a12, a12), p21 = re_mc(a21, a21),
                 p22 = re_mc(a22, a22);
    mu[0] = 0.5 * (p11 + p12 + p21 + p22);
    mu[1] = 0.5 * (p11 - p12 + p21 - p22);
    mu[2] = re_mc(a11, a12) + re_mc(a22, a21);
    mu[3] = im_mc(a11, a12) - im_mc(a22, a21);
    mu[4] = 0.5 * (p11 + p12 - p21 - p22);
    mu[5] = 0.5 * (p11 - p12 - p21 + p22);
    mu[6] = re_mc(a11, a12) - re_mc(a22, a21);
    mu[7] = im_mc(a11, a12) + im_mc(a22, a21);
    mu[8] = re_mc(a11, a21) + re_mc(a22, a12);
    mu[9] = re_mc(a11, a21) - re_mc(a22, a12);
    mu[10] = re_mc(a11, a22) + re_mc(a12, a21);
    mu[11] = im_mc(a11, a22) + im_mc(a21, a12);
    mu[12] = im_mc(a21, a11) + im_mc(a22, a12);
    mu[13] = im_mc(a21, a11) - im_mc(a22, a12);
    mu[14] = im_mc(a22, a11) - im_mc(a12, a21);
    mu[15] = re_mc(a22, a11) - re_mc(a12, a21);
}

// Amplitude of segment seg at bin o as reference-layout complex 2x2 (with
// T(phi) applied and scaled by sc), common phase e^{ik|X|} omitted.
__device__ __forceinline__ void ws_ampl(const double *ws, int64_t seg, int64_t nb, int64_t o, double cp,
                                        double sp, double sc, Zd S[4]) {
    const double *w = ws + seg * 8 * nb + o;
    Zd a[4];
#pragma unroll
    for (int c = 0; c < 4; c++) {
        a[c].re = w[(2 * c) * nb];
        a[c].im = w[(2 * c + 1) * nb];
    }
    // (S T)(a,b) = S(a,1) T(1,b) + S(a,2) T(2,b); T = [[-s, -c], [c, -s]]
    // order (1,1),(2,1),(1,2),(2,2): a[0]=S11 a[1]=S21 a[2]=S12 a[3]=S22
    const double T11 = -sp, T12 = -cp, T21 = cp, T22 = -sp;
    S[0] = {(a[0].re * T11 + a[2].re * T21) * sc, (a[0].im * T11 + a[2].im * T21) * sc};
    S[1] = {(a[1].re * T11 + a[3].re * T21) * sc, (a[1].im * T11 + a[3].im * T21) * sc};
    S[2] = {(a[0].re * T12 + a[2].re * T22) * sc, (a[0].im * T12 + a[2].im * T22) * sc};
    S[3] = {(a[1].re * T12 + a[3].re * T22) * sc, (a[1].im * T12 + a[3].im * T22) * sc};
}

__device__ __forceinline__ double block_sum(double v, double *red) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) s += red[i];
    __syncthreads();
    return s;
}

// Pre-pass of -scaling: per-orientation scatt_beam / scatt_ext sums.
// Per-orientation sums over the bins are reduced in two fixed-order steps (a
// block sum into part[(q K + k) nblk + block], then k2_part_sum_kernel over the
// blocks in order), so they are the same from run to run.
__global__ void k2_scatt_be_kernel(const double *__restrict__ ws, int64_t no, int64_t o0, int64_t nb,
                                   int64_t nphi, const double *__restrict__ phitab, double waveno,
                                   const double *__restrict__ wbin, double *__restrict__ part) {
    __shared__ double red[32];
    const int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = o < nb;
    const int64_t oo = in ? o : 0;
    const double cp = phitab[oo % nphi], sp = phitab[nphi + oo % nphi];
    const double W = in ? wbin[oo] / (waveno * waveno) : 0.0;
    for (int64_t q = 0; q < no; q++) {
        Zd Sb[4], Se[4];
        ws_ampl(ws, 2 * q, nb, oo, cp, sp, waveno, Sb);
        ws_ampl(ws, 2 * q + 1, nb, oo, cp, sp, waveno, Se);
        double mb[16], me[16];
        mueller16d(Sb, mb);
        mueller16d(Se, me);
        const double vb = block_sum(W * mb[0], red);
        const double ve = block_sum(W * me[0], red);
        if (threadIdx.x == 0) {
            part[(2 * q) * gridDim.x + blockIdx.x] = vb;
            part[(2 * q + 1) * gridDim.x + blockIdx.x] = ve;
        }
    }
    (void)o0;
}
// out[k0 + r] = sum over b of part[r nblk + b] in block order, r < nrow (one warp
// per row: lanes take blocks b = lane + 32 i in order, then a fixed shuffle tree).
__global__ void k2_part_sum_kernel(const double *__restrict__ part, int64_t nrow, int64_t nblk,
                                   double *__restrict__ out) {
    const int64_t r = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (r >= nrow) return;
    double v = 0.0;
    for (int64_t b = lane; b < nblk; b += 32) v += part[r * nblk + b];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if (lane == 0) out[r] = v;
}

// sqrt(scatt_part / energy_part) per orientation (src/outputs_mod.f90:151,154)
__global__ void k2_scale_kernel(double *__restrict__ scale, const pbt_output_params *__restrict__ pin,
                                int64_t o0, int64_t no) {
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= no) return;
    const int64_t o = o0 + q;
    scale[2 * o] = sqrt(scale[2 * o] / pin[o].beam_energy_out);
    scale[2 * o + 1] = sqrt(scale[2 * o + 1] / pin[o].ext_energy_out);
}

// Main epilogue: Mueller sum over the chunk's orientations and per-orientation
// weighted sums  red[o] = {scatt, scatt_beam, scatt_ext, g_num, g_num_beam, g_num_ext}.
__global__ void k2_epi_kernel(const double *__restrict__ ws, int64_t no, int64_t o0, int64_t nb,
                              int64_t nphi, const double *__restrict__ phitab,
                              const double *__restrict__ cth, double waveno,
                              const double *__restrict__ wbin, int64_t back_bin,
                              const double *__restrict__ scale, double *__restrict__ mu_sum,
                              double *__restrict__ part, double *__restrict__ bs) {
    __shared__ double red[32];
    const int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = o < nb;
    const int64_t oo = in ? o : 0;
    const int64_t i = oo % nphi, j = oo / nphi;
    const double cp = phitab[i], sp = phitab[nphi + i];
    const double W = in ? wbin[oo] / (waveno * waveno) : 0.0;
    const double ct = cth[j];
    double acc[16];
#pragma unroll
    for (int e = 0; e < 16; e++) acc[e] = 0.0;
    for (int64_t q = 0; q < no; q++) {
        const int64_t og = o0 + q;
        const double sb = scale ? 1.0 / scale[2 * og] : 1.0;
        const double se = scale ? 1.0 / scale[2 * og + 1] : 1.0;
        Zd Sb[4], Se[4], St[4];
        ws_ampl(ws, 2 * q, nb, oo, cp, sp, waveno * sb, Sb);
        ws_ampl(ws, 2 * q + 1, nb, oo, cp, sp, waveno * se, Se);
#pragma unroll
        for (int c = 0; c < 4; c++) St[c] = {Sb[c].re + Se[c].re, Sb[c].im + Se[c].im};
        double m[16];
        mueller16d(St, m);
#pragma unroll
        for (int e = 0; e < 16; e++) acc[e] += m[e];
        const double mb = 0.5 * (re_mc(Sb[0], Sb[0]) + re_mc(Sb[2], Sb[2]) + re_mc(Sb[1], Sb[1]) +
                                 re_mc(Sb[3], Sb[3]));
        const double me = 0.5 * (re_mc(Se[0], Se[0]) + re_mc(Se[2], Se[2]) + re_mc(Se[1], Se[1]) +
                                 re_mc(Se[3], Se[3]));
        double v[6] = {W * m[0], W * mb, W * me, W * ct * m[0], W * ct * mb, W * ct * me};
#pragma unroll
        for (int k = 0; k < 6; k++) {
            const double s = block_sum(v[k], red);
            if (threadIdx.x == 0) part[(6 * q + k) * gridDim.x + blockIdx.x] = s;
        }
        if (in && o == back_bin) bs[og] = m[0] * 4.0 * kPiRef / (waveno * waveno);
    }
    if (in)
#pragma unroll
        for (int e = 0; e < 16; e++) mu_sum[e * nb + o] += acc[e];
}

__global__ void k2_final_kernel(const double *__restrict__ redo, const double *__restrict__ bs,
                                const pbt_output_params *__restrict__ pin, int64_t norient,
                                pbt_output_params *__restrict__ pout) {
    const int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= norient) return;
    const double *r = redo + 6 * o;
    pbt_output_params p = pin[o];
    const double scatt = r[0], scatt_b = r[1], scatt_e = r[2];
    p.scatt = scatt;
    p.ext = p.abs + scatt;
    p.albedo = 1 - (p.ext - scatt) / p.ext;
    p.asymmetry = r[3] / scatt;
    p.abs_eff = p.abs / p.geo_cross_sec;
    p.scatt_eff = scatt / p.geo_cross_sec;
    p.ext_eff = p.ext / p.geo_cross_sec;
    p.back_scatt = bs[o];
    p.scatt_beam = scatt_b;
    p.scatt_ext_diff = scatt_e;
    p.asymmetry_beam = r[4] / scatt_b;
    p.asymmetry_ext_diff = r[5] / scatt_e;
    p.scatt_eff_beam = scatt_b / p.geo_cross_sec;
    p.scatt_eff_ext_diff = scatt_e / p.geo_cross_sec;
    pout[o] = p;
}

// Orientation average of the parameters (summation then divide), one thread per field.
__global__ void k2_param_avg_kernel(const pbt_output_params *__restrict__ per, int64_t norient,
                                    pbt_output_params *__restrict__ avg) {
    const int f = threadIdx.x;
    if (f >= 18) return;
    const double *src = reinterpret_cast<const double *>(per);
    double s = 0.0;
    for (int64_t o = 0; o < norient; o++) s = s + src[18 * o + f];
    // beam_energy_out / ext_energy_out are not summed by the reference
    reinterpret_cast<double *>(avg)[f] = (f == 10 || f == 11) ? 0.0 : s / (double)norient;
}

__global__ void k2_mu_avg_kernel(const double *__restrict__ mu_sum, int64_t n, double inv_n,
                                 double norient, double *__restrict__ mu_avg) {
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) mu_avg[q] = mu_sum[q] / norient;
    (void)inv_n;
}

__global__ void k2_phi_int_kernel(const double *__restrict__ mu, const double *__restrict__ wphi,
                                  int64_t nphi, int64_t ntheta, double *__restrict__ m1d) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 16 * ntheta) return;
    const int64_t j = t % ntheta, e = t / ntheta;
    const double *src = mu + e * nphi * ntheta + nphi * j;
    double s = 0.0;
    for (int64_t i = 0; i < nphi; i++) s += wphi[i] * src[i];
    m1d[j + ntheta * e] = s;
}

// FP32 diff_main output: reference-layout complex(8) grids, e^{ik|X|} S' T(phi).
__global__ void k2_ampl_out_kernel(const double *__restrict__ ws, int64_t nb, int64_t nphi,
                                   const double *__restrict__ phitab, const double *__restrict__ xyz,
                                   double waveno, double *__restrict__ afb, double *__restrict__ afe) {
    const int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= nb) return;
    const double cp = phitab[o % nphi], sp = phitab[nphi + o % nphi];
    const double X = xyz[o], Y = xyz[nb + o], Zc = xyz[2 * nb + o];
    double sK, cK;
    sincos(waveno * sqrt(X * X + Y * Y + Zc * Zc), &sK, &cK);
    for (int kind = 0; kind < 2; kind++) {
        Zd S[4];
        ws_ampl(ws, kind, nb, o, cp, sp, 1.0, S);
        double *dst = kind ? afe : afb;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            dst[2 * (o + nb * c)] = S[c].re * cK - S[c].im * sK;
            dst[2 * (o + nb * c) + 1] = S[c].re * sK + S[c].im * cK;
        }
    }
}

}  // namespace

// --------------------------------------------------------------- host side

namespace {

// Launch shape of the main kernel.  variant 1 = packed two-facet kernel over
// K2Pair records, 0 = one facet per step over K2Rec records.  bpt = bins per
// thread, rpi = facet records per work item.  PBT_K2_PLAN="variant,bpt,rpi"
// overrides the default (used by the tuner).
K2Plan k2_plan_for(const pbt_ctx *ctx) {
    K2Plan p;
    if (ctx->plan_variant >= 0) {
        p.variant = ctx->plan_variant;
        p.bpt = ctx->plan_bpt;
        p.rpi = ctx->plan_rpi;
        p.auto_rpi = false;
        return p;
    }
    if (const char *e = getenv("PBT_K2_PLAN")) {
        int v = 0, b = 0;
        long long r = 0;
        if (sscanf(e, "%d,%d,%lld", &v, &b, &r) == 3 && (v == 0 || v == 1) && (b == 1 || b == 2) &&
            r >= 32 && r <= (1 << 22)) {
            p.variant = v;
            p.bpt = b;
            p.rpi = r;
            p.auto_rpi = false;
        }
    }
    return p;
}

// Device-side set-up shared by the batched and single-orientation entry points.
struct K2Setup {
    K2Rec *recs = nullptr;
    K2Pair *pairs = nullptr;
    K2Fov *fovs = nullptr;
    float2 *rlo = nullptr;  // R_1 - (float)R_1 per record (the y row), pair layout (3 per pair)
    int64_t *start = nullptr;
    int64_t *refbase = nullptr;
    int64_t *beam_off = nullptr;
    int64_t *ext_off = nullptr;
    int *err = nullptr;
    unsigned *epsmax = nullptr;  // float bits of a bound of |com| / R over the records
};

size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }

int k2_prepare(pbt_ctx *ctx, cudaStream_t st, int64_t norient, const pbt_outbeam *d_beam,
               const int64_t *h_beam_off, const pbt_outbeam *d_ext, const int64_t *h_ext_off,
               const double *d_verts, int64_t nverts, const int64_t *d_face_off,
               const int64_t *d_face_vi, int64_t nfaces, int64_t max_nv, double lambda,
               int fast_diff, int variant, K2Setup &S) {
    pbt::NvtxRange nvtx_("pbt: set-up (records)");
    const int64_t nrefs = h_beam_off[norient] + h_ext_off[norient];
    const int64_t max_recs = std::max<int64_t>(1, nrefs * std::max<int64_t>(1, max_nv - 2));
    // scan temp size
    size_t scan_tmp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, scan_tmp, (int64_t *)nullptr, (int64_t *)nullptr,
                                  (int)(nrefs + 1), st);
    // d_in: cnt | start | refbase | beam_off | ext_off | err | scan tmp
    const size_t o_cnt = 0, o_start = align_up(o_cnt + (nrefs + 1) * 8),
                 o_rb = align_up(o_start + (nrefs + 1) * 8),
                 o_bo = align_up(o_rb + (norient + 1) * 8), o_eo = align_up(o_bo + (norient + 1) * 8),
                 o_err = align_up(o_eo + (norient + 1) * 8), o_tmp = align_up(o_err + 64),
                 o_end = align_up(o_tmp + scan_tmp);
    PBT_TRY(ctx->d_scan.ensure(o_end));
    char *base = ctx->d_scan.as<char>();
    int64_t *cnt = (int64_t *)(base + o_cnt);
    S.start = (int64_t *)(base + o_start);
    S.refbase = (int64_t *)(base + o_rb);
    S.beam_off = (int64_t *)(base + o_bo);
    S.ext_off = (int64_t *)(base + o_eo);
    S.err = (int *)(base + o_err);
    S.epsmax = (unsigned *)(base + o_err + 8);
    void *tmp = base + o_tmp;
    // records (or record pairs; an even count so the last pair is whole)
    const int64_t nrec2 = (max_recs + 1) & ~(int64_t)1;
    const size_t rec_bytes = variant ? (size_t)(nrec2 / 2) * sizeof(K2Pair) : (size_t)max_recs * sizeof(K2Rec);
    const size_t fov_bytes = fast_diff ? align_up(nrec2 * sizeof(K2Fov)) : 0;
    PBT_TRY(ctx->d_rec.ensure(align_up(rec_bytes) + fov_bytes + (size_t)(nrec2 / 2) * 3 * sizeof(float2)));
    S.recs = variant ? nullptr : ctx->d_rec.as<K2Rec>();
    S.pairs = variant ? ctx->d_rec.as<K2Pair>() : nullptr;
    S.fovs = fast_diff ? (K2Fov *)(ctx->d_rec.as<char>() + align_up(rec_bytes)) : nullptr;
    S.rlo = (float2 *)(ctx->d_rec.as<char>() + align_up(rec_bytes) + fov_bytes);
    // host-side offsets -> device (pinned staging; the previous call's copy
    // out of the staging buffer must have run before it is overwritten)
    if (ctx->stage_pending && !ctx->capturing) {
        PBT_CUDA_TRY(cudaEventSynchronize(ctx->stage_ev));
        ctx->stage_pending = false;
    }
    if (!ctx->stage_ev) PBT_CUDA_TRY(cudaEventCreateWithFlags(&ctx->stage_ev, cudaEventDisableTiming));
    PBT_TRY(ctx->h_stage.ensure(3 * (norient + 1) * 8));
    int64_t *hs = ctx->h_stage.as<int64_t>();
    for (int64_t o = 0; o <= norient; o++) {
        hs[o] = h_beam_off[o] + h_ext_off[o];
        hs[norient + 1 + o] = h_beam_off[o];
        hs[2 * (norient + 1) + o] = h_ext_off[o];
    }
    PBT_CUDA_TRY(cudaMemcpyAsync(S.refbase, hs, (norient + 1) * 8, cudaMemcpyHostToDevice, st));
    PBT_CUDA_TRY(cudaMemcpyAsync(S.beam_off, hs + norient + 1, (norient + 1) * 8,
                                 cudaMemcpyHostToDevice, st));
    PBT_CUDA_TRY(cudaMemcpyAsync(S.ext_off, hs + 2 * (norient + 1), (norient + 1) * 8,
                                 cudaMemcpyHostToDevice, st));
    if (!ctx->capturing) {
        PBT_CUDA_TRY(cudaEventRecord(ctx->stage_ev, st));
        ctx->stage_pending = true;
    }
    PBT_CUDA_TRY(cudaMemsetAsync(S.err, 0, 16, st));  // error flags and epsmax
    // rotation low parts: zero in a pair's unused half (an odd record count)
    PBT_CUDA_TRY(cudaMemsetAsync(S.rlo, 0, (size_t)(nrec2 / 2) * 3 * sizeof(float2), st));
    RefSrc src{d_beam, d_ext, S.beam_off, S.ext_off, S.refbase, norient};
    const int th = 256;
    k2_count_kernel<<<(unsigned)((nrefs + 1 + th - 1) / th), th, 0, st>>>(src, nrefs, d_face_off,
                                                                          nfaces, cnt, S.err);
    PBT_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp, scan_tmp, cnt, S.start, (int)(nrefs + 1), st));
    const double waveno = 2.0 * kPiRef / lambda;
    if (nrefs > 0)
        k2_setup_kernel<<<(unsigned)((nrefs + th - 1) / th), th, 0, st>>>(
            src, nrefs, d_verts, nverts, d_face_off, d_face_vi, S.start, waveno, lambda, fast_diff,
            S.recs, S.pairs, S.fovs, S.rlo, S.err, S.epsmax);
    ctx->launches += 3;
    PBT_CUDA_TRY(cudaGetLastError());
    return PBT_OK;
}

template <int BPT, bool FAST>
int k2_launch_main(pbt_ctx *ctx, cudaStream_t st, const K2MainArgs &A) {
    // resident CTAs per SM, computed once (thread-safe static initialisation)
    static const int occ = [] {
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k2_main_kernel<BPT, FAST>, K2_THREADS, 0) !=
            cudaSuccess)
            (void)cudaGetLastError();
        return n > 0 ? n : 1;
    }();
    const int grid = ctx->sm_count * occ;
    timing_begin(ctx, st);
    k2_main_kernel<BPT, FAST><<<grid, K2_THREADS, 0, st>>>(A);
    timing_end(ctx, st);
    ctx->launches++;
    PBT_CUDA_TRY(cudaGetLastError());
    return PBT_OK;
}

template <int BPT, bool FAST>
int k2_launch_pk(pbt_ctx *ctx, cudaStream_t st, const K2PkArgs &A) {
    static const int occ = [] {
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k2_main_pk_kernel<BPT, FAST>, K2_THREADS,
                                                          0) != cudaSuccess)
            (void)cudaGetLastError();
        return n > 0 ? n : 1;
    }();
    const int grid = ctx->sm_count * occ;
    timing_begin(ctx, st);
    k2_main_pk_kernel<BPT, FAST><<<grid, K2_THREADS, 0, st>>>(A);
    timing_end(ctx, st);
    ctx->launches++;
    PBT_CUDA_TRY(cudaGetLastError());
    return PBT_OK;
}

// One warp per tile: unit centre of the tile's bin directions and the
// largest angle of a bin from it (FP64).
__global__ void k2_cone_kernel(const int *__restrict__ perm, int64_t ntiles, int64_t tile,
                               const double *__restrict__ xyz, int64_t nb, K2Cone *__restrict__ cones) {
    const int64_t t = (int64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (t >= ntiles) return;
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int64_t i = lane; i < tile; i += 32) {
        const int o = perm[t * tile + i];
        if (o < 0) continue;
        const double X = xyz[o], Y = xyz[nb + o], Z = xyz[2 * nb + o];
        const double ir = 1.0 / sqrt(X * X + Y * Y + Z * Z);
        sx += X * ir;
        sy += Y * ir;
        sz += Z * ir;
    }
    for (int off = 16; off > 0; off >>= 1) {
        sx += __shfl_xor_sync(0xffffffffu, sx, off);
        sy += __shfl_xor_sync(0xffffffffu, sy, off);
        sz += __shfl_xor_sync(0xffffffffu, sz, off);
    }
    const double sn = sqrt(sx * sx + sy * sy + sz * sz);
    // a tile whose directions cancel gets psi > pi: never culled
    const bool ok = sn > 1e-9;
    const double cx = ok ? sx / sn : 0.0, cy = ok ? sy / sn : 0.0, cz = ok ? sz / sn : 1.0;
    double dmin = 1.0;
    for (int64_t i = lane; i < tile; i += 32) {
        const int o = perm[t * tile + i];
        if (o < 0) continue;
        const double X = xyz[o], Y = xyz[nb + o], Z = xyz[2 * nb + o];
        const double ir = 1.0 / sqrt(X * X + Y * Y + Z * Z);
        dmin = fmin(dmin, (X * cx + Y * cy + Z * cz) * ir);
    }
    for (int off = 16; off > 0; off >>= 1) dmin = fmin(dmin, __shfl_xor_sync(0xffffffffu, dmin, off));
    if (lane == 0) {
        const double psi = ok ? acos(fmax(-1.0, fmin(1.0, dmin))) + 1e-6 : 4.0;
        K2Cone c;
        c.c[0] = (float)cx;
        c.c[1] = (float)cy;
        c.c[2] = (float)cz;
        c.psi = (float)psi;
        c.cos_psi = (float)cos(psi);
        c.sin_psi = (float)sin(psi);
        c.pad[0] = c.pad[1] = 0.0f;
        cones[t] = c;
    }
}

// is_fast_diff tiles of `tile` bins: blocks of (tile/16) theta x 16 phi bins,
// so that a tile spans a small solid angle; cached with the bin grid.
int k2_fast_tiles(pbt_ctx *ctx, cudaStream_t st, int64_t tile) {
    GridCache &g = ctx->grid;
    if (g.fast_tile == tile) return PBT_OK;
    const int64_t nphi = (int64_t)g.phi.size(), ntheta = (int64_t)g.theta.size();
    const int64_t bp = 16, bt = tile / bp;
    const int64_t ntb = (ntheta + bt - 1) / bt, npb = (nphi + bp - 1) / bp;
    const int64_t ntiles = ntb * npb;
    std::vector<int> perm((size_t)(ntiles * tile), -1);
    for (int64_t a = 0; a < ntb; a++)
        for (int64_t b = 0; b < npb; b++) {
            const int64_t t = a * npb + b;
            int64_t i = 0;
            for (int64_t j = a * bt; j < std::min(ntheta, (a + 1) * bt); j++)
                for (int64_t q = b * bp; q < std::min(nphi, (b + 1) * bp); q++)
                    perm[(size_t)(t * tile + i++)] = (int)(q + nphi * j);
        }
    PBT_TRY(g.fast_perm.ensure(perm.size() * sizeof(int)));
    PBT_TRY(g.fast_cone.ensure((size_t)ntiles * sizeof(K2Cone)));
    PBT_CUDA_TRY(cudaMemcpyAsync(g.fast_perm.p, perm.data(), perm.size() * sizeof(int),
                                 cudaMemcpyHostToDevice, st));
    k2_cone_kernel<<<(unsigned)((ntiles + 3) / 4), 128, 0, st>>>(
        g.fast_perm.as<int>(), ntiles, tile, g.xyz.as<double>(), g.nb, g.fast_cone.as<K2Cone>());
    ctx->launches++;
    PBT_CUDA_TRY(cudaGetLastError());
    PBT_CUDA_TRY(cudaStreamSynchronize(st));  // perm (pageable) and cones ready before caching
    g.fast_tile = tile;
    g.fast_ntiles = ntiles;
    return PBT_OK;
}

// Records per work item of the default plan: about eight items per resident CTA
// (four per SM) for the call's records and bin tiles, in multiples of 64, between
// 256 and 2,048.  Fewer, larger items cost less per item on large lists; on small
// grids larger items leave the SMs short of work at the end of the launch (a
// 31,000-outbeam orientation on 16,290 bins: 2.95 ms at 1,024 records per item,
// 3.56 ms at 4,096).
int64_t k2_auto_rpi(int64_t nrec, int64_t ntiles, int nsm) {
    const int64_t want = (int64_t)8 * 4 * std::max(nsm, 1);
    int64_t r = nrec * ntiles / want;
    r = (r / 64) * 64;
    return std::min<int64_t>(2048, std::max<int64_t>(256, r));
}

int k2_run_chunk(pbt_ctx *ctx, cudaStream_t st, const K2Setup &S, int64_t o0, int64_t no,
                 int64_t nrefs, double lambda, int fast_diff, K2Plan plan, double *ws,
                 int64_t *seg_rec, int64_t *item_pre, unsigned long long *counter) {
    pbt::NvtxRange nvtx_("pbt: far-field sum (FP32)");
    const GridCache &g = ctx->grid;
    const int64_t tile = (int64_t)K2_THREADS * plan.bpt;
    int64_t ntiles = (g.nb + tile - 1) / tile;
    const bool cull = fast_diff && plan.variant == 1;
    if (cull) {
        PBT_TRY(k2_fast_tiles(ctx, st, tile));
        ntiles = g.fast_ntiles;
    }
    if (plan.auto_rpi) plan.rpi = k2_auto_rpi(nrefs, ntiles, ctx->sm_count);
    k2_plan_kernel<<<1, 32, 0, st>>>(S.start, S.refbase, S.beam_off, o0, no, plan.rpi, ntiles,
                                     seg_rec, item_pre, counter);
    ctx->launches++;
    PBT_CUDA_TRY(cudaMemsetAsync(ws, 0, (size_t)2 * no * 8 * g.nb * sizeof(double), st));
    // split tickets of every (segment, tile)
    const size_t tk_bytes = (size_t)2 * no * ntiles * sizeof(unsigned);
    PBT_TRY(ctx->d_tk.ensure(tk_bytes));
    PBT_CUDA_TRY(cudaMemsetAsync(ctx->d_tk.p, 0, tk_bytes, st));
    const double waveno = 2.0 * kPiRef / lambda;
    K2MainArgs A;
    A.recs = S.recs;
    A.fovs = S.fovs;
    A.rlo = S.rlo;
    A.seg_rec = seg_rec;
    A.item_pre = item_pre;
    A.nseg = 2 * no;
    A.rpi = plan.rpi;
    A.ntiles = ntiles;
    A.xyz = g.xyz.as<double>();
    A.nb = g.nb;
    A.nphi = (int64_t)g.phi.size();
    A.theta_i = g.theta_i;
    A.k = (float)waveno;
    A.hkR = (float)(0.5 * waveno * kFarR);
    A.sgh = -cos(g.theta[g.theta_i]) <= 0.0 ? 1.0f : -1.0f;  // sign rule of the bin set-up
    A.ws = ws;
    A.tickets = ctx->d_tk.as<unsigned>();
    A.counter = counter;
    A.err = S.err;
    if (plan.variant == 1) {
        K2PkArgs B;
        B.pairs = S.pairs;
        B.rlo = S.rlo;
        B.fovs = S.fovs;
        B.perm = cull ? g.fast_perm.as<int>() : nullptr;
        B.cones = cull ? g.fast_cone.as<K2Cone>() : nullptr;
        B.seg_rec = seg_rec;
        B.item_pre = item_pre;
        B.nseg = A.nseg;
        B.rpi = plan.rpi;
        B.ntiles = ntiles;
        B.xyz = A.xyz;
        B.nb = A.nb;
        B.nphi = A.nphi;
        B.theta_i = A.theta_i;
        B.k = A.k;
        B.hkR = A.hkR;
        B.sgh = A.sgh;
        B.epsmax = S.epsmax;
        B.ws = ws;
        B.tickets = A.tickets;
        B.counter = counter;
        B.err = S.err;
        if (plan.bpt == 1)
            return fast_diff ? k2_launch_pk<1, true>(ctx, st, B) : k2_launch_pk<1, false>(ctx, st, B);
        return fast_diff ? k2_launch_pk<2, true>(ctx, st, B) : k2_launch_pk<2, false>(ctx, st, B);
    }
    if (plan.bpt == 1)
        return fast_diff ? k2_launch_main<1, true>(ctx, st, A) : k2_launch_main<1, false>(ctx, st, A);
    return fast_diff ? k2_launch_main<2, true>(ctx, st, A) : k2_launch_main<2, false>(ctx, st, A);
}

int64_t max_face_nv(const int64_t *h_face_off, int64_t nfaces) {
    int64_t m = 3;
    for (int64_t f = 0; f < nfaces; f++) m = std::max(m, h_face_off[f + 1] - h_face_off[f]);
    return m;
}

}  // namespace

namespace {
// One CTA waits on an mbarrier that nothing arrives at: the bounded wait must
// give up after limit_ns and raise the timeout flag.
__global__ void k2_wait_selftest_kernel(uint64_t limit_ns, int *__restrict__ err) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(smem_u32(&bar), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const bool ok = mbar_wait(smem_u32(&bar), 0u, limit_ns);
    if (threadIdx.x == 0 && !ok) atomicOr(err, 4);
}
}  // namespace

int k2_wait_selftest(pbt_ctx *ctx, cudaStream_t st, uint64_t limit_ns) {
    PBT_TRY(ctx->d_misc.ensure(64));
    int *d_err = ctx->d_misc.as<int>();
    PBT_CUDA_TRY(cudaMemsetAsync(d_err, 0, sizeof(int), st));
    k2_wait_selftest_kernel<<<1, 32, 0, st>>>(limit_ns, d_err);
    ctx->launches = 1;
    PBT_CUDA_TRY(cudaGetLastError());
    return k2_check_err(ctx, st, d_err);
}

int k2_check_err(pbt_ctx *ctx, cudaStream_t st, const int *d_err) {
    (void)ctx;
    int h = 0;
    PBT_CUDA_TRY(cudaMemcpyAsync(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    PBT_CUDA_TRY(cudaStreamSynchronize(st));
    if (h & 1) {
        set_error("an outbeam face index fi is out of range");
        return PBT_EINVAL;
    }
    if (h & 2) {
        set_error("the FP32 path supports faces of up to 16 vertices");
        return PBT_EINVAL;
    }
    if (h & 4) {
        set_error("a bounded device wait timed out in the far-field kernel");
        return PBT_ETIMEOUT;
    }
    return PBT_OK;
}

// Batched FP32 orientation average in three steps: begin (the orientation
// sums and per-orientation results for norient orientations), add (a run of
// orientations [o0, o0+no): record set-up, the far-field sum and the
// epilogue into the sums), finish (averages and phi integrals).
// h_beam_off / h_ext_off (relative to the run) and h_face_off are host arrays;
// every other array is device memory.
namespace {
__global__ void k2_err_fold_kernel(const int *__restrict__ run_err, int *__restrict__ total) {
    if (threadIdx.x == 0 && *run_err) atomicOr(total, *run_err);
}
}  // namespace

int k2_batch_begin(pbt_ctx *ctx, cudaStream_t st, int64_t norient, int64_t max_run,
                   const pbt_output_params *d_params_per, K2Batch &B) {
    const GridCache &g = ctx->grid;
    const int64_t nb = g.nb;
    B.norient = norient;
    B.plan = k2_plan_for(ctx);
    // orientation chunks of the FP64 workspace, capped at 16 GiB
    const size_t per_orient = (size_t)2 * 8 * nb * sizeof(double);
    const size_t cap = (size_t)16 << 30;
    B.wchunk = std::max<int64_t>(1, std::min<int64_t>(max_run, (int64_t)(cap / per_orient)));
    const int64_t chunk = B.wchunk;
    // d_ws: workspace | mu_sum | per-orient red (6) | bs | scale (2) | per-orient params | seg/items
    const size_t o_ws = 0, o_mu = align_up(o_ws + chunk * per_orient),
                 o_red = align_up(o_mu + 16 * nb * 8), o_bs = align_up(o_red + 6 * norient * 8),
                 o_sc = align_up(o_bs + norient * 8), o_pp = align_up(o_sc + 2 * norient * 8),
                 o_seg = align_up(o_pp + norient * sizeof(pbt_output_params)),
                 o_it = align_up(o_seg + (2 * chunk + 1) * 8), o_cnt = align_up(o_it + (2 * chunk + 1) * 8),
                 o_err = align_up(o_cnt + 64),
                 o_part = align_up(o_err + 64),
                 o_end = align_up(o_part + (size_t)6 * chunk * ((nb + 255) / 256) * 8);
    PBT_TRY(ctx->d_ws.ensure(o_end));
    char *base = ctx->d_ws.as<char>();
    B.err = (int *)(base + o_err);
    B.part = (double *)(base + o_part);
    PBT_CUDA_TRY(cudaMemsetAsync(B.err, 0, sizeof(int), st));
    B.ws = (double *)(base + o_ws);
    B.mu_sum = (double *)(base + o_mu);
    B.redo = (double *)(base + o_red);
    B.bs = (double *)(base + o_bs);
    B.scale = (double *)(base + o_sc);
    B.pp = d_params_per ? const_cast<pbt_output_params *>(d_params_per) : (pbt_output_params *)(base + o_pp);
    B.seg_rec = (int64_t *)(base + o_seg);
    B.item_pre = (int64_t *)(base + o_it);
    B.counter = (unsigned long long *)(base + o_cnt);
    PBT_CUDA_TRY(cudaMemsetAsync(B.mu_sum, 0, 16 * nb * 8, st));
    PBT_CUDA_TRY(cudaMemsetAsync(B.redo, 0, 6 * norient * 8, st));
    PBT_CUDA_TRY(cudaMemsetAsync(B.bs, 0, norient * 8, st));
    PBT_CUDA_TRY(cudaMemsetAsync(B.scale, 0, 2 * norient * 8, st));
    return PBT_OK;
}

int k2_batch_add(pbt_ctx *ctx, cudaStream_t st, K2Batch &B, int64_t o0, int64_t no,
                 const pbt_outbeam *d_beam, const int64_t *h_beam_off, const pbt_outbeam *d_ext,
                 const int64_t *h_ext_off, const double *d_verts, int64_t nverts,
                 const int64_t *h_face_off, const int64_t *d_face_off, const int64_t *d_face_vi,
                 int64_t nfaces, double lambda, int fast_diff, int scaling,
                 const pbt_output_params *d_params_in) {
    const GridCache &g = ctx->grid;
    const int64_t nb = g.nb, nphi = (int64_t)g.phi.size(), ntheta = (int64_t)g.theta.size();
    K2Setup S;
    PBT_TRY(k2_prepare(ctx, st, no, d_beam, h_beam_off, d_ext, h_ext_off, d_verts, nverts,
                       d_face_off, d_face_vi, nfaces, max_face_nv(h_face_off, nfaces), lambda,
                       fast_diff, B.plan.variant, S));
    const double waveno = 2.0 * kPiRef / lambda;
    const double *phitab = g.phitab.as<double>(), *sth = g.thtab.as<double>(), *cth = sth + ntheta;
    (void)sth;
    const int64_t back_bin = 0 + nphi * g.back_i;
    const int eb = 256;
    const unsigned egrid = (unsigned)((nb + eb - 1) / eb);
    for (int64_t l0 = 0; l0 < no; l0 += B.wchunk) {
        const int64_t n = std::min(B.wchunk, no - l0);
        const int64_t nrefs =
            (h_beam_off[l0 + n] - h_beam_off[l0]) + (h_ext_off[l0 + n] - h_ext_off[l0]);
        PBT_TRY(k2_run_chunk(ctx, st, S, l0, n, nrefs, lambda, fast_diff, B.plan, B.ws, B.seg_rec,
                             B.item_pre, B.counter));
        const int64_t og = o0 + l0;  // global orientation of the workspace's first slot
        pbt::NvtxRange nvtx_epi("pbt: epilogue (Mueller, orientation sums)");
        if (scaling) {
            k2_scatt_be_kernel<<<egrid, eb, 0, st>>>(B.ws, n, og, nb, nphi, phitab, waveno,
                                                     g.wbin.as<double>(), B.part);
            k2_part_sum_kernel<<<(unsigned)((2 * n + 3) / 4), 128, 0, st>>>(B.part, 2 * n, egrid,
                                                                          B.scale + 2 * og);
            k2_scale_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(B.scale, d_params_in, og, n);
            ctx->launches += 3;
        }
        k2_epi_kernel<<<egrid, eb, 0, st>>>(B.ws, n, og, nb, nphi, phitab, cth, waveno,
                                            g.wbin.as<double>(), back_bin, scaling ? B.scale : nullptr,
                                            B.mu_sum, B.part, B.bs);
        k2_part_sum_kernel<<<(unsigned)((6 * n + 3) / 4), 128, 0, st>>>(B.part, 6 * n, egrid,
                                                                      B.redo + 6 * og);
        ctx->launches += 2;
        PBT_CUDA_TRY(cudaGetLastError());
    }
    // the run's error flags (its set-up buffer is reused by the next run)
    k2_err_fold_kernel<<<1, 32, 0, st>>>(S.err, B.err);
    ctx->launches++;
    PBT_CUDA_TRY(cudaGetLastError());
    return PBT_OK;
}

int k2_batch_finish(pbt_ctx *ctx, cudaStream_t st, K2Batch &B, const pbt_output_params *d_params_in,
                    double *d_mueller_avg, double *d_m1d_avg, pbt_output_params *d_params_avg,
                    int check_errors) {
    pbt::NvtxRange nvtx_("pbt: orientation average");
    const GridCache &g = ctx->grid;
    const int64_t nb = g.nb, nphi = (int64_t)g.phi.size(), ntheta = (int64_t)g.theta.size();
    const int64_t norient = B.norient;
    k2_final_kernel<<<(unsigned)((norient + 127) / 128), 128, 0, st>>>(B.redo, B.bs, d_params_in,
                                                                       norient, B.pp);
    k2_param_avg_kernel<<<1, 32, 0, st>>>(B.pp, norient, d_params_avg);
    k2_mu_avg_kernel<<<(unsigned)((16 * nb + 255) / 256), 256, 0, st>>>(
        B.mu_sum, 16 * nb, 1.0 / (double)norient, (double)norient, d_mueller_avg);
    k2_phi_int_kernel<<<(unsigned)((16 * ntheta + 127) / 128), 128, 0, st>>>(
        d_mueller_avg, g.wphi.as<double>(), nphi, ntheta, d_m1d_avg);
    ctx->launches += 4;
    PBT_CUDA_TRY(cudaGetLastError());
    if (check_errors) PBT_TRY(k2_check_err(ctx, st, B.err));
    return PBT_OK;
}

int k2_batch_impl(pbt_ctx *ctx, cudaStream_t st, int64_t norient, const pbt_outbeam *d_beam,
                  const int64_t *h_beam_off, const pbt_outbeam *d_ext, const int64_t *h_ext_off,
                  const double *d_verts, int64_t nverts, const int64_t *h_face_off,
                  const int64_t *d_face_off, const int64_t *d_face_vi, int64_t nfaces,
                  double lambda, int fast_diff, int scaling, const pbt_output_params *d_params_in,
                  double *d_mueller_avg, double *d_m1d_avg, pbt_output_params *d_params_avg,
                  pbt_output_params *d_params_per, int check_errors) {
    K2Batch B;
    PBT_TRY(k2_batch_begin(ctx, st, norient, norient, d_params_per, B));
    PBT_TRY(k2_batch_add(ctx, st, B, 0, norient, d_beam, h_beam_off, d_ext, h_ext_off, d_verts,
                         nverts, h_face_off, d_face_off, d_face_vi, nfaces, lambda, fast_diff,
                         scaling, d_params_in));
    return k2_batch_finish(ctx, st, B, d_params_in, d_mueller_avg, d_m1d_avg, d_params_avg,
                           check_errors);
}

// FP32 diff_main: one orientation, amplitude grids in the reference layout.
int k2_diff_main_impl(pbt_ctx *ctx, cudaStream_t st, const pbt_outbeam *d_beam, int64_t nbeam,
                      const pbt_outbeam *d_ext, int64_t next, const double *d_verts, int64_t nverts,
                      const int64_t *h_face_off, const int64_t *d_face_off,
                      const int64_t *d_face_vi, int64_t nfaces, double lambda, int fast_diff,
                      double *d_afb, double *d_afe) {
    const GridCache &g = ctx->grid;
    const int64_t nb = g.nb;
    const K2Plan plan = k2_plan_for(ctx);
    K2Setup S;
    const int64_t hbo[2] = {0, nbeam}, heo[2] = {0, next};
    PBT_TRY(k2_prepare(ctx, st, 1, d_beam, hbo, d_ext, heo, d_verts, nverts, d_face_off, d_face_vi,
                       nfaces, max_face_nv(h_face_off, nfaces), lambda, fast_diff, plan.variant, S));
    const size_t o_ws = 0, o_seg = align_up(o_ws + (size_t)2 * 8 * nb * sizeof(double)),
                 o_it = align_up(o_seg + 3 * 8), o_cnt = align_up(o_it + 3 * 8), o_end = align_up(o_cnt + 64);
    PBT_TRY(ctx->d_ws.ensure(o_end));
    char *base = ctx->d_ws.as<char>();
    double *ws = (double *)(base + o_ws);
    PBT_TRY(k2_run_chunk(ctx, st, S, 0, 1, nbeam + next, lambda, fast_diff, plan, ws,
                         (int64_t *)(base + o_seg), (int64_t *)(base + o_it),
                         (unsigned long long *)(base + o_cnt)));
    const double waveno = 2.0 * kPiRef / lambda;
    k2_ampl_out_kernel<<<(unsigned)((nb + 127) / 128), 128, 0, st>>>(
        ws, nb, (int64_t)g.phi.size(), g.phitab.as<double>(), g.xyz.as<double>(), waveno, d_afb,
        d_afe);
    ctx->launches++;
    PBT_CUDA_TRY(cudaGetLastError());
    return k2_check_err(ctx, st, S.err);
}

}  // namespace pbt
