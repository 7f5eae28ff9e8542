// k1_fp64.cu -- reference-exact FP64 far-field sum (the plain drop-in).
//
// One thread per far-field bin; each thread walks the facet list in order and
// adds every facet's 2x2 complex amplitude to its bin, so the sum has the
// reference's association ((0 + c_1) + c_2) + ... (src/diff_mod.f90:744-766).
// Per facet x bin the thread repeats the reference's arithmetic operation by
// operation: the bin translation/rotation (src/diff_mod.f90:576-618),
// karczewski (:124-198), the scattering-plane rotation (:628-658) and the
// contour integral (:357-428), then multiplies (:665-670).  The file is built
// with -fmad=false so no multiply-add is fused.  Facet frames come from the
// host (host_setup.cpp); the bin grid and cos/sin(phi) are libm values.
#include "frame.h"
#include "pbt_internal.h"

namespace pbt {

namespace {

struct Z {
    double re, im;
};
__device__ __forceinline__ Z zmul(Z a, Z b) {
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}

__device__ __forceinline__ void cross_n(const double a[3], const double b[3], double c[3]) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
    double nf = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
    c[0] = c[0] / nf;
    c[1] = c[1] / nf;
    c[2] = c[2] / nf;
}
__device__ __forceinline__ double dot_3(const double a[3], const double b[3]) {
    double s = 0.0;
    s = s + a[0] * b[0];
    s = s + a[1] * b[1];
    s = s + a[2] * b[2];
    return s;
}

__global__ void __launch_bounds__(128) k1_kernel(
    const K1Facet *__restrict__ fac, int64_t nf, const K1Edge *__restrict__ edges,
    const double *__restrict__ xyz, const double *__restrict__ phitab, int64_t nphi, int64_t nb,
    int64_t theta_i, double waveno, double lambda, int fast_diff, double *__restrict__ out) {
    const int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= nb) return;
    const int64_t i = o % nphi;
    const double X = xyz[o], Y = xyz[nb + o], Zc = xyz[2 * nb + o];
    const int64_t oh = i + nphi * theta_i;
    const double Xh = xyz[oh], Yh = xyz[nb + oh], Zh = xyz[2 * nb + oh];

    // getRotationMatrix(temp_rot1, -sin(phi), cos(phi), 0, 1,0,0, 0,0,-1) then
    // transpose, src/diff_mod.f90:646-650
    double T[2][2];
    {
        const double cp = phitab[i], sp = phitab[nphi + i];
        const double vk71 = -sp, vk72 = cp, vk73 = 0.0;
        const double ev11 = 1, ev12 = 0, ev13 = 0, ev31 = 0, ev32 = 0, ev33 = -1;
        const double mfa = vk71 * ev11 + vk72 * ev12 + vk73 * ev13;
        const double evo21 = ev32 * ev13 - ev33 * ev12;
        const double evo22 = ev33 * ev11 - ev31 * ev13;
        const double evo23 = ev31 * ev12 - ev32 * ev11;
        const double q = vk71 * evo21 + vk72 * evo22 + vk73 * evo23;
        T[0][0] = mfa;
        T[1][0] = -q;  // transpose of rot(1,2)
        T[0][1] = +q;  // transpose of rot(2,1)
        T[1][1] = mfa;
    }

    Z acc[4] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
    for (int64_t f = 0; f < nf; ++f) {
        const K1Facet *F = fac + f;
        const double c0 = F->com[0], c1 = F->com[1], c2 = F->com[2];
        const double x1 = X - c0, y1 = Y - c1, z1 = Zc - c2;
        const double r1 = sqrt(x1 * x1 + y1 * y1 + z1 * z1);
        if (fast_diff) {
            const double vec[3] = {x1 / r1, y1 / r1, z1 / r1};
            const double p0[3] = {F->prop0[0], F->prop0[1], F->prop0[2]};
            if (dot_3(vec, p0) < F->cos_fov) continue;  // outside the field of view
        }
        double R[9];
#pragma unroll
        for (int q = 0; q < 9; q++) R[q] = F->R[q];
        const double x3 = R[0] * x1 + R[1] * y1 + R[2] * z1;
        const double y3 = R[3] * x1 + R[4] * y1 + R[5] * z1;
        const double z3 = R[6] * x1 + R[7] * y1 + R[8] * z1;
        const double prop2[3] = {F->prop2[0], F->prop2[1], F->prop2[2]};
        const double inc2[3] = {F->inc2[0], F->inc2[1], F->inc2[2]};

        // karczewski
        double k[3], m[3], D[2][2];
        {
            k[0] = x3 / r1;
            k[1] = y3 / r1;
            k[2] = z3 / r1;
            if (fabs(k[1]) > kLit0_999999) k[1] = copysign(kLit0_999999, k[1]);
            const double Kx = prop2[0], Ky = prop2[1], Kz = prop2[2];
            const double sq = sqrt(1 - k[1] * k[1]);
            m[0] = -(k[0] * k[1] / sq);
            m[1] = sq;
            m[2] = -(k[1] * k[2] / sq);
            const double frac = sqrt((1 - k[1] * k[1]) / (1 - Ky * Ky));
            const double a1m = -Kz * frac;
            const double b2m = -k[2] / frac;
            const double b1m = -(k[0] * k[1] / frac) + Kx * Ky * frac;
            const double a2e = -b1m;
            D[0][0] = 0.5 * (a1m + b2m);
            D[0][1] = 0.5 * b1m;
            D[1][0] = 0.5 * a2e;
            D[1][1] = 0.5 * (b2m + a1m);
        }
        double hc[3], evo2[3];
        if (fabs(dot_3(inc2, k)) < kLit0_999) {
            cross_n(inc2, k, hc);
        } else {
            // forward bodge: the bin at the same phi and theta index theta_i
            const double xh = Xh - c0, yh = Yh - c1, zh = Zh - c2;
            const double rh = sqrt(xh * xh + yh * yh + zh * zh);
            const double x3h = R[0] * xh + R[1] * yh + R[2] * zh;
            const double y3h = R[3] * xh + R[4] * yh + R[5] * zh;
            const double z3h = R[6] * xh + R[7] * yh + R[8] * zh;
            const double my_k[3] = {x3h / rh, y3h / rh, z3h / rh};
            cross_n(inc2, my_k, hc);
        }
        cross_n(k, m, evo2);
        double rot4[2][2];
        rot4[0][0] = dot_3(hc, m);
        rot4[1][1] = dot_3(hc, m);
        rot4[0][1] = -dot_3(hc, evo2);
        rot4[1][0] = +dot_3(hc, evo2);

        // ampl_temp2 = rot4 . (diff_ampl . (ampl . T))
        Z A[2][2];
        A[0][0] = {F->ampl[0], F->ampl[1]};
        A[1][0] = {F->ampl[2], F->ampl[3]};
        A[0][1] = {F->ampl[4], F->ampl[5]};
        A[1][1] = {F->ampl[6], F->ampl[7]};
        Z P[2][2], Q[2][2], Rz[2][2];
#pragma unroll
        for (int a = 0; a < 2; a++)
#pragma unroll
            for (int b = 0; b < 2; b++) {
                Z s = {0, 0};
                s.re = s.re + A[a][0].re * T[0][b];
                s.im = s.im + A[a][0].im * T[0][b];
                s.re = s.re + A[a][1].re * T[1][b];
                s.im = s.im + A[a][1].im * T[1][b];
                P[a][b] = s;
            }
#pragma unroll
        for (int a = 0; a < 2; a++)
#pragma unroll
            for (int b = 0; b < 2; b++) {
                Z s = {0, 0};
                s.re = s.re + P[0][b].re * D[a][0];
                s.im = s.im + P[0][b].im * D[a][0];
                s.re = s.re + P[1][b].re * D[a][1];
                s.im = s.im + P[1][b].im * D[a][1];
                Q[a][b] = s;
            }
#pragma unroll
        for (int a = 0; a < 2; a++)
#pragma unroll
            for (int b = 0; b < 2; b++) {
                Z s = {0, 0};
                s.re = s.re + Q[0][b].re * rot4[a][0];
                s.im = s.im + Q[0][b].im * rot4[a][0];
                s.re = s.re + Q[1][b].re * rot4[a][1];
                s.im = s.im + Q[1][b].im * rot4[a][1];
                Rz[a][b] = s;
            }

        // contour_integral for this bin
        const double bvs = waveno * sqrt(x3 * x3 + y3 * y3 + z3 * z3);
        double kxx = F->kinc[0] - waveno * waveno * x3 / bvs;
        double kyy = F->kinc[1] - waveno * waveno * y3 / bvs;
        if (fabs(kxx) < kLit1em6) kxx = kLit1em6;
        if (fabs(kyy) < kLit1em6) kyy = kLit1em6;
        double sK, cK;
        sincos(bvs, &sK, &cK);
        const Z eK = {cK, sK};
        Z area = {0, 0};
        const K1Edge *E = edges + F->edge_off;
        const int64_t nv = F->nv;
        for (int64_t j = 0; j < nv; j++) {
            const double xj = E[j].xj, yj = E[j].yj, mj = E[j].mj, nj = E[j].nj;
            const double dx = E[j].dx, dy = E[j].dy;
            const double delta = kxx * xj + kyy * yj;
            const double delta1 = kyy * mj + kxx;
            const double delta2 = kxx * nj + kyy;
            const double omega1 = dx * delta1;
            const double omega2 = dy * delta2;
            const double alpha = 1 / (2 * kyy * delta1);
            const double beta = 1 / (2 * kxx * delta2);
            double s0, c0d, s1, c1d, s2, c2d;
            sincos(delta, &s0, &c0d);
            sincos(delta + omega1, &s1, &c1d);
            sincos(delta + omega2, &s2, &c2d);
            const double sumim = alpha * (c0d - c1d) - beta * (c0d - c2d);
            const double sumre = -(alpha * (s0 - s1)) + beta * (s0 - s2);
            Z t = zmul(eK, Z{sumre, sumim});
            t.re = t.re / lambda;
            t.im = t.im / lambda;
            area.re = area.re + t.re;
            area.im = area.im + t.im;
        }
        // amplC = ampl_temp2 * area; ampl_far += amplC
        const Z c11 = zmul(Rz[0][0], area), c21 = zmul(Rz[1][0], area);
        const Z c12 = zmul(Rz[0][1], area), c22 = zmul(Rz[1][1], area);
        acc[0].re = acc[0].re + c11.re;
        acc[0].im = acc[0].im + c11.im;
        acc[1].re = acc[1].re + c21.re;
        acc[1].im = acc[1].im + c21.im;
        acc[2].re = acc[2].re + c12.re;
        acc[2].im = acc[2].im + c12.im;
        acc[3].re = acc[3].re + c22.re;
        acc[3].im = acc[3].im + c22.im;
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
        out[2 * (o + nb * q)] = acc[q].re;
        out[2 * (o + nb * q) + 1] = acc[q].im;
    }
}

}  // namespace

int k1_launch(pbt_ctx *ctx, cudaStream_t st, const K1Facet *d_fac, int64_t nf,
              const K1Edge *d_edges, double lambda, int fast_diff, double *d_grid) {
    const GridCache &g = ctx->grid;
    const double waveno = 2.0 * kPiRef / lambda;
    const int threads = 128;
    const int64_t blocks = (g.nb + threads - 1) / threads;
    timing_begin(ctx, st);
    k1_kernel<<<(unsigned)blocks, threads, 0, st>>>(
        d_fac, nf, d_edges, g.xyz.as<double>(), g.phitab.as<double>(), (int64_t)g.phi.size(), g.nb,
        g.theta_i, waveno, lambda, fast_diff, d_grid);
    timing_end(ctx, st);
    ctx->launches++;
    PBT_CUDA_TRY(cudaGetLastError());
    return PBT_OK;
}

}  // namespace pbt
