// k3_finalise.cu -- reference-exact FP64 epilogue: finalise, summation and
// divide_by_num_orientations (src/outputs_mod.f90:13-43, 63-278, 407-549).
//
// Built with -fmad=false.  Pass 1 (one thread per bin) scales the amplitude
// grids by the wavenumber (:104-105), forms the total (:108) and the
// Bohren-Huffman Mueller matrix (ampl_to_mueller, :473-549).  Pass 2 (one
// thread per theta row and element) integrates over phi with simpne in the
// reference's sequential order (get_1d_mueller, :280-329).  Pass 3 (one
// thread) does the theta integrals and the output parameters (:133-245).
// With -scaling, passes 1-3 run twice, the second time with the energy
// scale factors that pass 3 wrote to device memory (:146-184).
#include "frame.h"
#include "pbt_internal.h"

namespace pbt {

namespace {

struct Z {
    double re, im;
};

// real(a*conjg(b)) and imag(a*conjg(b)) as gfortran evaluates them
__device__ __forceinline__ double re_mc(Z a, Z b) { return a.re * b.re - a.im * (-b.im); }
__device__ __forceinline__ double im_mc(Z a, Z b) { return a.re * (-b.im) + a.im * b.re; }

__device__ __forceinline__ void mueller16(Z a11, Z a21, Z a12, Z a22, double mu[16]) {
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

__device__ __forceinline__ double m11_of(Z a11, Z a21, Z a12, Z a22) {
    const double p11 = re_mc(a11, a11), p12 = re_mc(a12, a12), p21 = re_mc(a21, a21),
                 p22 = re_mc(a22, a22);
    return 0.5 * (p11 + p12 + p21 + p22);
}

// simpne, src/misc_submod.f90:2392-2531, with y given by a functor
template <class Y>
__device__ double simpne_dev(int64_t ntab, const double *x, Y y) {
    double del[3], g[3], pi1[3], e, f, feints, sum1, x1, x2, x3, result = 0.0;
    int64_t n = 1;
    for (;;) {
        x1 = x[n - 1];
        x2 = x[n];
        x3 = x[n + 1];
        e = x3 * x3 - x1 * x1;
        f = x3 * x3 * x3 - x1 * x1 * x1;
        feints = x3 - x1;
        del[0] = x3 - x2;
        del[1] = x1 - x3;
        del[2] = x2 - x1;
        g[0] = x2 + x3;
        g[1] = x1 + x3;
        g[2] = x1 + x2;
        pi1[0] = x2 * x3;
        pi1[1] = x1 * x3;
        pi1[2] = x1 * x2;
        sum1 = 0.0;
        for (int i = 1; i <= 3; i++)
            sum1 = sum1 + y(n - 2 + i) * del[i - 1] * (f / 3.0 - g[i - 1] * 0.5 * e + pi1[i - 1] * feints);
        result = result - sum1 / (del[0] * del[1] * del[2]);
        n = n + 2;
        if (ntab <= n + 1) break;
    }
    if (ntab % 2 != 0) return result;
    n = ntab - 2;
    x3 = x[ntab - 1];
    x2 = x[ntab - 2];
    x1 = x[ntab - 3];
    e = x3 * x3 - x2 * x2;
    f = x3 * x3 * x3 - x2 * x2 * x2;
    feints = x3 - x2;
    del[0] = x3 - x2;
    del[1] = x1 - x3;
    del[2] = x2 - x1;
    g[0] = x2 + x3;
    g[1] = x1 + x3;
    g[2] = x1 + x2;
    pi1[0] = x2 * x3;
    pi1[1] = x1 * x3;
    pi1[2] = x1 * x2;
    sum1 = 0.0;
    for (int i = 1; i <= 3; i++)
        sum1 = sum1 + y(n - 2 + i) * del[i - 1] * (f / 3.0 - g[i - 1] * 0.5 * e + pi1[i - 1] * feints);
    result = result - sum1 / (del[0] * del[1] * del[2]);
    return result;
}

// Pass 1: ampl -> Mueller (total, 16 elements) and M11 of the beam and
// external-diffraction parts.  scale: NULL, or [sb, se] energy scale factors.
__global__ void k3_mueller_kernel(const double *__restrict__ afb, const double *__restrict__ afe,
                                  int64_t nb, double waveno, const double *__restrict__ scale,
                                  double *__restrict__ mu, double *__restrict__ m11be) {
    const int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= nb) return;
    Z b[4], e[4], t[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        b[q].re = afb[2 * (o + nb * q)] * waveno;
        b[q].im = afb[2 * (o + nb * q) + 1] * waveno;
        e[q].re = afe[2 * (o + nb * q)] * waveno;
        e[q].im = afe[2 * (o + nb * q) + 1] * waveno;
    }
    if (scale) {
        const double sb = scale[0], se = scale[1];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            b[q].re = b[q].re / sb;
            b[q].im = b[q].im / sb;
            e[q].re = e[q].re / se;
            e[q].im = e[q].im / se;
        }
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
        t[q].re = b[q].re + e[q].re;
        t[q].im = b[q].im + e[q].im;
    }
    double m[16];
    mueller16(t[0], t[1], t[2], t[3], m);
#pragma unroll
    for (int q = 0; q < 16; q++) mu[o + nb * q] = m[q];
    m11be[o] = m11_of(b[0], b[1], b[2], b[3]);
    m11be[nb + o] = m11_of(e[0], e[1], e[2], e[3]);
}

// Pass 2: phi integration per theta row.  Thread (row j, element e): e < 16
// integrates the total Mueller element e; e = 16, 17 integrate M11 of the beam
// and external-diffraction parts.
__global__ void k3_phi_kernel(const double *__restrict__ mu, const double *__restrict__ m11be,
                              const double *__restrict__ phi, int64_t nphi, int64_t ntheta,
                              double *__restrict__ m1d, double *__restrict__ m1be) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntheta * 18) return;
    const int64_t j = t % ntheta, e = t / ntheta;
    const int64_t nb = nphi * ntheta;
    const double *src = (e < 16) ? mu + nb * e + nphi * j : m11be + nb * (e - 16) + nphi * j;
    const double r = simpne_dev(nphi, phi, [&](int64_t k) { return src[k]; });
    if (e < 16)
        m1d[j + ntheta * e] = r;
    else
        m1be[j + ntheta * (e - 16)] = r;
}

// Pass 3: theta integrals and output parameters.  With final == 0 this is the
// first pass of a -scaling run: only the energy scale factors are written.
__global__ void k3_params_kernel(const double *__restrict__ mu, const double *__restrict__ m1d,
                                 const double *__restrict__ m1be, const double *__restrict__ theta,
                                 const double *__restrict__ sth, const double *__restrict__ cth,
                                 int64_t ntheta, int64_t nphi, int64_t back_i, double waveno,
                                 const pbt_output_params pin, int final_pass,
                                 double *__restrict__ scale, double *__restrict__ pout) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double w2 = waveno * waveno;
    const double *m1b = m1be, *m1e = m1be + ntheta;
    const double scatt = simpne_dev(ntheta, theta, [&](int64_t j) { return m1d[j] * sth[j] / w2; });
    const double scatt_beam =
        simpne_dev(ntheta, theta, [&](int64_t j) { return m1b[j] * sth[j] / w2; });
    const double scatt_ext =
        simpne_dev(ntheta, theta, [&](int64_t j) { return m1e[j] * sth[j] / w2; });
    if (!final_pass) {
        scale[0] = sqrt(scatt_beam / pin.beam_energy_out);
        scale[1] = sqrt(scatt_ext / pin.ext_energy_out);
        return;
    }
    const double absorption = pin.abs;
    const double ext = absorption + scatt;
    const double albedo = 1 - (ext - scatt) / ext;
    const double asym =
        simpne_dev(ntheta, theta, [&](int64_t j) { return m1d[j] * sth[j] * cth[j] / scatt / w2; });
    const double asym_beam = simpne_dev(
        ntheta, theta, [&](int64_t j) { return m1b[j] * sth[j] * cth[j] / scatt_beam / w2; });
    const double asym_ext = simpne_dev(
        ntheta, theta, [&](int64_t j) { return m1e[j] * sth[j] * cth[j] / scatt_ext / w2; });
    const double back_scatt = mu[0 + nphi * back_i] * 4 * kPiRef / w2;
    pbt_output_params p = pin;
    p.scatt = scatt;
    p.abs = absorption;
    p.ext = ext;
    p.albedo = albedo;
    p.asymmetry = asym;
    p.abs_eff = absorption / p.geo_cross_sec;
    p.scatt_eff = scatt / p.geo_cross_sec;
    p.ext_eff = ext / p.geo_cross_sec;
    p.back_scatt = back_scatt;
    p.scatt_beam = scatt_beam;
    p.scatt_ext_diff = scatt_ext;
    p.asymmetry_beam = asym_beam;
    p.asymmetry_ext_diff = asym_ext;
    p.scatt_eff_beam = scatt_beam / p.geo_cross_sec;
    p.scatt_eff_ext_diff = scatt_ext / p.geo_cross_sec;
    const double *pp = reinterpret_cast<const double *>(&p);
    for (int q = 0; q < 18; q++) pout[q] = pp[q];
}

// summation, src/outputs_mod.f90:450-469
__global__ void k3_sum_kernel(double *__restrict__ t_mu, const double *__restrict__ mu, int64_t n2,
                              double *__restrict__ t_m1, const double *__restrict__ m1, int64_t n1,
                              double *__restrict__ t_p, const double *__restrict__ p) {
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n2) t_mu[q] = t_mu[q] + mu[q];
    if (q < n1) t_m1[q] = t_m1[q] + m1[q];
    if (q < 18) {
        // every component except beam_energy_out (10) and ext_energy_out (11)
        if (q != 10 && q != 11) t_p[q] = t_p[q] + p[q];
    }
}

// divide_by_num_orientations, src/outputs_mod.f90:23-41 (into copies)
__global__ void k3_div_kernel(const double *__restrict__ t_mu, double *__restrict__ mu, int64_t n2,
                              const double *__restrict__ t_m1, double *__restrict__ m1, int64_t n1,
                              const double *__restrict__ t_p, double *__restrict__ p, double n) {
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n2) mu[q] = t_mu[q] / n;
    if (q < n1) m1[q] = t_m1[q] / n;
    if (q < 18) p[q] = (q == 10 || q == 11) ? t_p[q] : t_p[q] / n;
}

}  // namespace

int totals_ensure(DevTotals &T, int64_t ntheta, int64_t nphi, cudaStream_t st) {
    if (T.count > 0 && (T.ntheta != ntheta || T.nphi != nphi)) {
        set_error("totals hold a %lldx%lld grid; reset them before changing the grid",
                  (long long)T.ntheta, (long long)T.nphi);
        return PBT_ESTATE;
    }
    if (T.ntheta != ntheta || T.nphi != nphi || !T.mu.p) {
        T.ntheta = ntheta;
        T.nphi = nphi;
        PBT_TRY(T.mu.ensure(16 * ntheta * nphi * sizeof(double)));
        PBT_TRY(T.m1.ensure(16 * ntheta * sizeof(double)));
        PBT_TRY(T.par.ensure(18 * sizeof(double)));
        PBT_TRY(totals_reset(T, st));
    }
    return PBT_OK;
}

int totals_reset(DevTotals &T, cudaStream_t st) {
    if (T.mu.p) {
        PBT_CUDA_TRY(cudaMemsetAsync(T.mu.p, 0, 16 * T.ntheta * T.nphi * sizeof(double), st));
        PBT_CUDA_TRY(cudaMemsetAsync(T.m1.p, 0, 16 * T.ntheta * sizeof(double), st));
        PBT_CUDA_TRY(cudaMemsetAsync(T.par.p, 0, 18 * sizeof(double), st));
    }
    T.count = 0;
    return PBT_OK;
}

int totals_add_device(pbt_ctx *ctx, DevTotals &T, cudaStream_t st, const double *d_mueller,
                      const double *d_m1d, const double *d_params) {
    const int64_t n2 = 16 * T.ntheta * T.nphi, n1 = 16 * T.ntheta;
    const int threads = 256;
    k3_sum_kernel<<<(unsigned)((n2 + threads - 1) / threads), threads, 0, st>>>(
        T.mu.as<double>(), d_mueller, n2, T.m1.as<double>(), d_m1d, n1, T.par.as<double>(),
        d_params);
    ctx->launches++;
    PBT_CUDA_TRY(cudaGetLastError());
    T.count++;
    return PBT_OK;
}

int totals_divide_device(pbt_ctx *ctx, DevTotals &T, cudaStream_t st, int64_t num_orients,
                         double *d_mu, double *d_m1, double *d_p) {
    const int64_t n2 = 16 * T.ntheta * T.nphi, n1 = 16 * T.ntheta;
    const int threads = 256;
    k3_div_kernel<<<(unsigned)((n2 + threads - 1) / threads), threads, 0, st>>>(
        T.mu.as<double>(), d_mu, n2, T.m1.as<double>(), d_m1, n1, T.par.as<double>(), d_p,
        (double)num_orients);
    ctx->launches++;
    PBT_CUDA_TRY(cudaGetLastError());
    return PBT_OK;
}

int k3_finalise(pbt_ctx *ctx, cudaStream_t st, const double *d_afb, const double *d_afe,
                double lambda, int scaling, const pbt_output_params *h_params_in,
                double *d_mueller, double *d_m1d, double *d_params, DevTotals *acc) {
    pbt::NvtxRange nvtx_("pbt: finalise");
    const GridCache &g = ctx->grid;
    const int64_t nb = g.nb, nphi = (int64_t)g.phi.size(), ntheta = (int64_t)g.theta.size();
    const double waveno = 2.0 * kPiRef / lambda;  // src/outputs_mod.f90:98
    // scratch: m11be (2 nb) | m1be (2 ntheta) | scale (2)
    PBT_TRY(ctx->d_misc.ensure((2 * nb + 2 * ntheta + 8) * sizeof(double)));
    double *m11be = ctx->d_misc.as<double>();
    double *m1be = m11be + 2 * nb;
    double *scale = m1be + 2 * ntheta;
    const double *sth = g.thtab.as<double>(), *cth = sth + ntheta, *th = sth + 2 * ntheta;
    const double *ph = th + ntheta;
    const int threads = 128;
    for (int pass = 0; pass < (scaling ? 2 : 1); pass++) {
        const bool final_pass = !scaling || pass == 1;
        k3_mueller_kernel<<<(unsigned)((nb + threads - 1) / threads), threads, 0, st>>>(
            d_afb, d_afe, nb, waveno, pass == 1 ? scale : nullptr, d_mueller, m11be);
        k3_phi_kernel<<<(unsigned)((18 * ntheta + 63) / 64), 64, 0, st>>>(d_mueller, m11be, ph,
                                                                          nphi, ntheta, d_m1d, m1be);
        k3_params_kernel<<<1, 32, 0, st>>>(d_mueller, d_m1d, m1be, th, sth, cth, ntheta, nphi,
                                           g.back_i, waveno, *h_params_in, final_pass ? 1 : 0,
                                           scale, d_params);
        ctx->launches += 3;
        PBT_CUDA_TRY(cudaGetLastError());
    }
    if (acc) PBT_TRY(totals_add_device(ctx, *acc, st, d_mueller, d_m1d, d_params));
    return PBT_OK;
}

}  // namespace pbt
