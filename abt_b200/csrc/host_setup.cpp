// host_setup.cpp -- host-side preparation for the far-field kernels.
//
// Built with the host compiler and -ffp-contract=off: the O(nbins) bin grid
// (make_far_field_bins, src/diff_mod.f90:827-855) and the O(nfacets)
// per-facet frames of the reference-exact FP64 path are formed here with the
// platform libm, exactly as the Fortran reference forms them, because these
// few transcendental calls per facet / per bin set the ~1e-9 rad phase floor
// of a phase k|x| ~ 1e7 rad.  Everything O(nfacets x nbins) runs on the GPU.
#include <float.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "frame.h"
#include "pbt_internal.h"

namespace pbt {

int validate_angles(const double *theta, int64_t ntheta, const double *phi, int64_t nphi) {
    if (!theta || !phi) {
        set_error("theta/phi must not be NULL");
        return PBT_EINVAL;
    }
    if (ntheta < 3 || nphi < 3) {
        // simpne needs at least 3 points (src/misc_submod.f90:2453-2459)
        set_error("need at least 3 theta and 3 phi values (got %lld, %lld)", (long long)ntheta,
                  (long long)nphi);
        return PBT_EINVAL;
    }
    if (ntheta > (1 << 20) || nphi > (1 << 20) || ntheta * nphi > (int64_t)1 << 31) {
        set_error("far-field grid too large (%lld x %lld)", (long long)ntheta, (long long)nphi);
        return PBT_EINVAL;
    }
    for (int64_t i = 0; i < ntheta; i++)
        if (!isfinite(theta[i])) {
            set_error("theta[%lld] is not finite", (long long)i);
            return PBT_EINVAL;
        }
    for (int64_t i = 0; i < nphi; i++)
        if (!isfinite(phi[i])) {
            set_error("phi[%lld] is not finite", (long long)i);
            return PBT_EINVAL;
        }
    return PBT_OK;
}

int validate_geometry(const double *verts, int64_t nverts, const int64_t *face_off,
                      const int64_t *face_vi, int64_t nfaces) {
    if (!verts || !face_off || !face_vi) {
        set_error("geometry arrays must not be NULL");
        return PBT_EINVAL;
    }
    if (nverts < 3 || nfaces < 1) {
        set_error("geometry needs >= 3 vertices and >= 1 face");
        return PBT_EINVAL;
    }
    if (face_off[0] != 0) {
        set_error("face_off[0] must be 0");
        return PBT_EINVAL;
    }
    for (int64_t f = 0; f < nfaces; f++) {
        int64_t nv = face_off[f + 1] - face_off[f];
        if (nv < 3 || nv > 4096) {
            set_error("face %lld has %lld vertices (need 3..4096)", (long long)(f + 1),
                      (long long)nv);
            return PBT_EINVAL;
        }
    }
    int64_t nvi = face_off[nfaces];
    // the first bad index and coordinate, found with all host threads
    int64_t bad_vi = nvi, bad_v = 3 * nverts;
#pragma omp parallel for reduction(min : bad_vi) schedule(static) if (nvi > 65536)
    for (int64_t q = 0; q < nvi; q++)
        if (face_vi[q] < 1 || face_vi[q] > nverts) bad_vi = std::min(bad_vi, q);
#pragma omp parallel for reduction(min : bad_v) schedule(static) if (nverts > 20000)
    for (int64_t q = 0; q < 3 * nverts; q++)
        if (!isfinite(verts[q])) bad_v = std::min(bad_v, q);
    for (int64_t q = bad_vi; q < nvi; q++)
        if (face_vi[q] < 1 || face_vi[q] > nverts) {
            set_error("face_vi[%lld] = %lld out of range 1..%lld", (long long)q,
                      (long long)face_vi[q], (long long)nverts);
            return PBT_EINVAL;
        }
    for (int64_t q = bad_v; q < 3 * nverts; q++)
        if (!isfinite(verts[q])) {
            set_error("vertex coordinate %lld is not finite", (long long)q);
            return PBT_EINVAL;
        }
    return PBT_OK;
}

// Coefficients c_i with simpne(x, y) = sum_i c_i y_i (simpne is linear in y,
// src/misc_submod.f90:2392-2531).  Used by the batched epilogue, which forms
// the phi/theta integrals as weighted sums.
static void simpne_weights(const double *x, int64_t ntab, double *w) {
    for (int64_t i = 0; i < ntab; i++) w[i] = 0;
    auto panel = [&](int64_t n0, double x1, double x2, double x3, double e, double f,
                     double feints) {
        double del[3] = {x3 - x2, x1 - x3, x2 - x1};
        double g[3] = {x2 + x3, x1 + x3, x1 + x2};
        double pi1[3] = {x2 * x3, x1 * x3, x1 * x2};
        double den = del[0] * del[1] * del[2];
        for (int i = 0; i < 3; i++)
            w[n0 + i] -= del[i] * (f / 3.0 - g[i] * 0.5 * e + pi1[i] * feints) / den;
    };
    int64_t n = 1;
    for (;;) {
        double x1 = x[n - 1], x2 = x[n], x3 = x[n + 1];
        panel(n - 1, x1, x2, x3, x3 * x3 - x1 * x1, x3 * x3 * x3 - x1 * x1 * x1, x3 - x1);
        n += 2;
        if (ntab <= n + 1) break;
    }
    if (ntab % 2 != 0) return;
    double x3 = x[ntab - 1], x2 = x[ntab - 2], x1 = x[ntab - 3];
    panel(ntab - 3, x1, x2, x3, x3 * x3 - x2 * x2, x3 * x3 * x3 - x2 * x2 * x2, x3 - x2);
}

// make_far_field_bins (src/diff_mod.f90:827-855) in meshgrid order, phi fastest
// (:846-853): X = R (sin t cos p, sin t sin p, -cos t), R = 1e6, libm values.
void far_field_bins(const double *theta, int64_t ntheta, const double *phi, int64_t nphi,
                    double *x, double *y, double *z) {
    const double r = kFarR;
    for (int64_t j = 0; j < ntheta; j++)
        for (int64_t i = 0; i < nphi; i++) {
            const int64_t o = i + nphi * j;
            x[o] = r * sin(theta[j]) * cos(phi[i]);
            y[o] = r * sin(theta[j]) * sin(phi[i]);
            z[o] = -(r * cos(theta[j]));
        }
}

int grid_prepare(pbt_ctx *ctx, const double *theta, int64_t ntheta, const double *phi,
                 int64_t nphi, cudaStream_t st) {
    GridCache &g = ctx->grid;
    if (g.valid && (int64_t)g.theta.size() == ntheta && (int64_t)g.phi.size() == nphi &&
        !memcmp(g.theta.data(), theta, ntheta * sizeof(double)) &&
        !memcmp(g.phi.data(), phi, nphi * sizeof(double)))
        return PBT_OK;
    g.valid = false;
    g.fast_tile = 0;
    g.theta.assign(theta, theta + ntheta);
    g.phi.assign(phi, phi + nphi);
    int64_t nb = ntheta * nphi;
    g.nb = nb;
    g.theta_i = -1;
    for (int64_t i = 0; i < ntheta; i++)
        if (theta[i] > 1 * kPiRef / 180) {  // src/diff_mod.f90:587
            g.theta_i = i;
            break;
        }
    g.back_i = 0;  // minloc(abs(theta_vals - 2*pi)), src/outputs_mod.f90:204
    double best = fabs(theta[0] - 2 * kPiRef);
    for (int64_t i = 1; i < ntheta; i++) {
        double d = fabs(theta[i] - 2 * kPiRef);
        if (d < best) {
            best = d;
            g.back_i = i;
        }
    }
    std::vector<double> xyz(3 * nb), pt(2 * nphi), tt(2 * ntheta), wb(nb), wph(nphi), wth(ntheta);
    far_field_bins(theta, ntheta, phi, nphi, xyz.data(), xyz.data() + nb, xyz.data() + 2 * nb);
    for (int64_t i = 0; i < nphi; i++) {
        pt[i] = cos(phi[i]);
        pt[nphi + i] = sin(phi[i]);
    }
    for (int64_t j = 0; j < ntheta; j++) {
        tt[j] = sin(theta[j]);
        tt[ntheta + j] = cos(theta[j]);
    }
    simpne_weights(phi, nphi, wph.data());
    simpne_weights(theta, ntheta, wth.data());
    for (int64_t j = 0; j < ntheta; j++)
        for (int64_t i = 0; i < nphi; i++) wb[i + nphi * j] = wph[i] * wth[j] * tt[j];
    PBT_TRY(g.xyz.ensure(3 * nb * sizeof(double)));
    PBT_TRY(g.phitab.ensure(2 * nphi * sizeof(double)));
    PBT_TRY(g.thtab.ensure(2 * ntheta * sizeof(double) + 2 * (ntheta + nphi) * sizeof(double)));
    PBT_TRY(g.wbin.ensure(nb * sizeof(double)));
    PBT_TRY(g.wphi.ensure(nphi * sizeof(double)));
    PBT_CUDA_TRY(cudaMemcpyAsync(g.xyz.p, xyz.data(), 3 * nb * sizeof(double),
                                 cudaMemcpyHostToDevice, st));
    PBT_CUDA_TRY(cudaMemcpyAsync(g.phitab.p, pt.data(), 2 * nphi * sizeof(double),
                                 cudaMemcpyHostToDevice, st));
    // thtab: sin(theta) | cos(theta) | theta | phi
    std::vector<double> th2(2 * ntheta + ntheta + nphi);
    std::copy(tt.begin(), tt.end(), th2.begin());
    std::copy(theta, theta + ntheta, th2.begin() + 2 * ntheta);
    std::copy(phi, phi + nphi, th2.begin() + 3 * ntheta);
    PBT_CUDA_TRY(cudaMemcpyAsync(g.thtab.p, th2.data(), th2.size() * sizeof(double),
                                 cudaMemcpyHostToDevice, st));
    PBT_CUDA_TRY(cudaMemcpyAsync(g.wbin.p, wb.data(), nb * sizeof(double),
                                 cudaMemcpyHostToDevice, st));
    PBT_CUDA_TRY(cudaMemcpyAsync(g.wphi.p, wph.data(), nphi * sizeof(double),
                                 cudaMemcpyHostToDevice, st));
    // the host vectors die at return: wait for the copies
    PBT_CUDA_TRY(cudaStreamSynchronize(st));
    g.valid = true;
    return PBT_OK;
}

int k1_build_facets(const pbt_outbeam *obs, int64_t n, double fov_override, const double *verts,
                    int64_t nverts, const int64_t *face_off, const int64_t *face_vi,
                    int64_t nfaces, double lambda, std::vector<K1Facet> &fac,
                    std::vector<K1Edge> &edges) {
    const double waveno = 2.0 * kPiRef / lambda;  // src/diff_mod.f90:332
    size_t f0 = fac.size(), e0 = edges.size();
    std::vector<int64_t> eoff(n + 1, 0);
    for (int64_t j = 0; j < n; j++) {
        const pbt_outbeam &ob = obs[j];
        if (ob.fi < 1 || ob.fi > nfaces) {
            set_error("outbeam %lld: face index fi=%lld out of range 1..%lld", (long long)(j + 1),
                      (long long)ob.fi, (long long)nfaces);
            return PBT_EINVAL;
        }
        for (int q = 0; q < 8; q++)
            if (!isfinite(ob.ampl[q])) {
                set_error("outbeam %lld: amplitude is not finite", (long long)(j + 1));
                return PBT_EINVAL;
            }
        for (int q = 0; q < 3; q++)
            if (!isfinite(ob.vk7[q]) || !isfinite(ob.prop_out[q])) {
                set_error("outbeam %lld: direction is not finite", (long long)(j + 1));
                return PBT_EINVAL;
            }
        eoff[j + 1] = eoff[j] + (face_off[ob.fi] - face_off[ob.fi - 1]);
    }
    fac.resize(f0 + n);
    edges.resize(e0 + eoff[n]);
#pragma omp parallel for schedule(static) if (n > 512)
    for (int64_t j = 0; j < n; j++) {
        const pbt_outbeam &ob = obs[j];
        const int64_t fb = face_off[ob.fi - 1];
        const int nv = (int)(face_off[ob.fi] - fb);
        std::vector<double> vb(6 * nv);
        double *vx = vb.data(), *vy = vx + nv, *vz = vx + 2 * nv;
        double *rx = vx + 3 * nv, *ry = vx + 4 * nv, *rz = vx + 5 * nv;
        for (int i = 0; i < nv; i++) {
            int64_t vi = face_vi[fb + i] - 1;
            vx[i] = verts[vi];
            vy[i] = verts[vi + nverts];
            vz[i] = verts[vi + 2 * nverts];
        }
        FacetFrame fr;
        fr.sign = 1.0;
        facet_frame(vx, vy, vz, nv, ob.prop_out, ob.vk7, fr, rx, ry, rz);
        K1Facet &F = fac[f0 + j];
        for (int c = 0; c < 3; c++) {
            F.com[c] = fr.com[c];
            F.prop2[c] = fr.prop2[c];
            F.inc2[c] = fr.inc2[c];
            F.prop0[c] = ob.prop_out[c];
        }
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) F.R[3 * a + b] = fr.R.m[a][b];
        for (int q = 0; q < 8; q++) F.ampl[q] = fr.sign < 0 ? -ob.ampl[q] : ob.ampl[q];
        double fov = fov_override >= 0 ? fov_override : ob.fov;
        F.cos_fov = cos(fov);  // src/diff_mod.f90:523
        F.kinc[0] = fr.prop2[0] * waveno;
        F.kinc[1] = fr.prop2[1] * waveno;
        F.edge_off = (int64_t)e0 + eoff[j];
        F.nv = nv;
        // contour_integral set-up, src/diff_mod.f90:334-354
        std::vector<double> xs(nv), ys(nv), ms(nv);
        for (int i = 0; i < nv; i++) {
            double c[3] = {rx[i], ry[i], rz[i]}, r[3];
            mv33(fr.R, c, r);
            xs[i] = r[0];
            ys[i] = r[1];
        }
        for (int i = 0; i < nv; i++) {
            int in = (i == nv - 1) ? 0 : i + 1;
            ms[i] = (ys[in] - ys[i]) / (xs[in] - xs[i]);
        }
        for (int i = 0; i < nv; i++) {
            double mj = ms[i], nj = 1 / ms[i];
            // slope clamps, in the reference's order, src/diff_mod.f90:379-382
            if (fabs(mj) > DBL_MAX) mj = 1e6;
            if (fabs(nj) > DBL_MAX) nj = 1e6;
            if (fabs(mj) < 1e-9) nj = 1e6;
            if (fabs(nj) < 1e-9) mj = 1e6;
            int in = (i == nv - 1) ? 0 : i + 1;
            K1Edge &E = edges[F.edge_off + i];
            E.xj = xs[i];
            E.yj = ys[i];
            E.mj = mj;
            E.nj = nj;
            E.dx = xs[in] - xs[i];
            E.dy = ys[in] - ys[i];
        }
    }
    return PBT_OK;
}

}  // namespace pbt

extern "C" int pbt_make_far_field_bins_c(const double *theta, int64_t ntheta, const double *phi,
                                         int64_t nphi, double *xfar, double *yfar, double *zfar) {
    pbt::clear_error();
    if (!theta || !phi || !xfar || !yfar || !zfar || ntheta < 1 || nphi < 1) {
        pbt::set_error("make_far_field_bins: NULL array or empty angle list");
        return PBT_EINVAL;
    }
    pbt::far_field_bins(theta, ntheta, phi, nphi, xfar, yfar, zfar);
    return PBT_OK;
}
