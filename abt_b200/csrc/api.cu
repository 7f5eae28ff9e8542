// api.cu -- the extern "C" entry points of libpbt_b200.so (include/pbt_diff.h).
//
// Each entry point validates its arguments on the host, stages host arrays to
// the context's device buffers on the context stream, runs the kernels and
// copies results back.  Calls on one context are serialised by its mutex.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <new>
#include <vector>

#include "frame.h"
#include "pbt_internal.h"

namespace pbt {

int validate_outbeams(const pbt_outbeam *obs, int64_t n, int64_t nfaces, const char *what) {
    if (n < 0) {
        set_error("%s: negative outbeam count", what);
        return PBT_EINVAL;
    }
    if (n > 0 && !obs) {
        set_error("%s: outbeam array is NULL", what);
        return PBT_EINVAL;
    }
    // find the first bad record with all host threads, then report it in order
    auto good = [nfaces](const pbt_outbeam &ob) {
        bool ok = ob.fi >= 1 && ob.fi <= nfaces && isfinite(ob.fov);
        for (int q = 0; q < 8; q++) ok = ok && isfinite(ob.ampl[q]);
        for (int q = 0; q < 3; q++) ok = ok && isfinite(ob.vk7[q]) && isfinite(ob.prop_out[q]);
        return ok;
    };
    int64_t first_bad = n;
#pragma omp parallel for reduction(min : first_bad) schedule(static) if (n > 65536)
    for (int64_t j = 0; j < n; j++)
        if (!good(obs[j])) first_bad = std::min(first_bad, j);
    for (int64_t j = first_bad; j < n; j++) {
        const pbt_outbeam &ob = obs[j];
        if (ob.fi < 1 || ob.fi > nfaces) {
            set_error("%s outbeam %lld: face index fi=%lld out of range 1..%lld", what,
                      (long long)(j + 1), (long long)ob.fi, (long long)nfaces);
            return PBT_EINVAL;
        }
        for (int q = 0; q < 8; q++)
            if (!isfinite(ob.ampl[q])) {
                set_error("%s outbeam %lld: amplitude is not finite", what, (long long)(j + 1));
                return PBT_EINVAL;
            }
        for (int q = 0; q < 3; q++)
            if (!isfinite(ob.vk7[q]) || !isfinite(ob.prop_out[q])) {
                set_error("%s outbeam %lld: direction is not finite", what, (long long)(j + 1));
                return PBT_EINVAL;
            }
        if (!isfinite(ob.fov)) {
            set_error("%s outbeam %lld: fov is not finite", what, (long long)(j + 1));
            return PBT_EINVAL;
        }
    }
    return PBT_OK;
}

}  // namespace pbt

using namespace pbt;

namespace {

int check_ctx(pbt_ctx *ctx) {
    if (!ctx) {
        set_error("context is NULL");
        return PBT_EINVAL;
    }
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) {
        set_error("cudaSetDevice(%d): %s", ctx->device, cudaGetErrorString(e));
        return PBT_ECUDA;
    }
    return PBT_OK;
}

int check_lambda(double lambda) {
    if (!(lambda > 0) || !isfinite(lambda)) {
        set_error("lambda must be positive and finite (got %g)", lambda);
        return PBT_EINVAL;
    }
    return PBT_OK;
}

int check_grid_ready(pbt_ctx *ctx) {
    if (ctx->grid.theta_i < 0) {
        // the reference leaves theta_i undefined when no theta exceeds 1 degree
        // (src/diff_mod.f90:583-591); refuse instead of reading out of range
        set_error("no theta value above 1 degree: the forward-bin fix of the reference needs one");
        return PBT_EINVAL;
    }
    return PBT_OK;
}

template <class T>
int upload(DevBuf &buf, const T *src, size_t n, cudaStream_t st, size_t off_bytes = 0) {
    PBT_TRY(buf.ensure(off_bytes + std::max<size_t>(n * sizeof(T), 16)));
    if (n) PBT_CUDA_TRY(cudaMemcpyAsync(buf.as<char>() + off_bytes, src, n * sizeof(T),
                                        cudaMemcpyHostToDevice, st));
    return PBT_OK;
}

size_t al(size_t x) { return (x + 255) & ~(size_t)255; }

// FP64 reference-exact amplitude grids of one orientation into d_afb / d_afe.
int fp64_diff_main_device(pbt_ctx *ctx, cudaStream_t st, const pbt_outbeam *beam, int64_t nbeam,
                          const pbt_outbeam *ext, int64_t next, const double *verts, int64_t nverts,
                          const int64_t *face_off, const int64_t *face_vi, int64_t nfaces,
                          double lambda, int fast_diff, double *d_afb, double *d_afe) {
    std::vector<K1Facet> fac;
    std::vector<K1Edge> edges;
    fac.reserve(nbeam + next);
    PBT_TRY(k1_build_facets(beam, nbeam, -1.0, verts, nverts, face_off, face_vi, nfaces, lambda,
                            fac, edges));
    // external diffraction: fov forced to pi/2, src/diff_mod.f90:797
    PBT_TRY(k1_build_facets(ext, next, kPiRef / 2.0, verts, nverts, face_off, face_vi, nfaces,
                            lambda, fac, edges));
    PBT_TRY(upload(ctx->d_fac, fac.data(), fac.size(), st));
    PBT_TRY(upload(ctx->d_edge, edges.data(), edges.size(), st));
    const K1Facet *df = ctx->d_fac.as<K1Facet>();
    PBT_TRY(k1_launch(ctx, st, df, nbeam, ctx->d_edge.as<K1Edge>(), lambda, fast_diff, d_afb));
    PBT_TRY(k1_launch(ctx, st, df + nbeam, next, ctx->d_edge.as<K1Edge>(), lambda, fast_diff, d_afe));
    // the host vectors are released at return: finish the copies first
    PBT_CUDA_TRY(cudaStreamSynchronize(st));
    return PBT_OK;
}

// Stage the geometry (face CSR + vertices) of norient orientations.
struct GeoDev {
    const double *verts;
    const int64_t *face_off;
    const int64_t *face_vi;
};

int upload_geometry(pbt_ctx *ctx, cudaStream_t st, const double *verts, int64_t nverts,
                    int64_t norient, const int64_t *face_off, const int64_t *face_vi,
                    int64_t nfaces, GeoDev &G) {
    const size_t nvi = (size_t)face_off[nfaces];
    const size_t o_fo = 0, o_fv = al((nfaces + 1) * 8), o_v = al(o_fv + nvi * 8),
                 o_end = al(o_v + (size_t)norient * 3 * nverts * 8);
    PBT_TRY(ctx->d_in.ensure(o_end));
    char *b = ctx->d_in.as<char>();
    PBT_CUDA_TRY(cudaMemcpyAsync(b + o_fo, face_off, (nfaces + 1) * 8, cudaMemcpyHostToDevice, st));
    PBT_CUDA_TRY(cudaMemcpyAsync(b + o_fv, face_vi, nvi * 8, cudaMemcpyHostToDevice, st));
    if (verts)  // else the caller copies the orientations' blocks
        PBT_CUDA_TRY(cudaMemcpyAsync(b + o_v, verts, (size_t)norient * 3 * nverts * 8,
                                     cudaMemcpyHostToDevice, st));
    G.face_off = (const int64_t *)(b + o_fo);
    G.face_vi = (const int64_t *)(b + o_fv);
    G.verts = (const double *)(b + o_v);
    return PBT_OK;
}

int check_offsets(const int64_t *off, int64_t norient, const char *what) {
    if (!off) {
        set_error("%s offsets are NULL", what);
        return PBT_EINVAL;
    }
    if (off[0] != 0) {
        set_error("%s_off[0] must be 0", what);
        return PBT_EINVAL;
    }
    for (int64_t o = 0; o < norient; o++)
        if (off[o + 1] < off[o]) {
            set_error("%s_off must be non-decreasing (orientation %lld)", what, (long long)(o + 1));
            return PBT_EINVAL;
        }
    return PBT_OK;
}

}  // namespace

#define API_ENTER(ctx)                              \
    clear_error();                                  \
    pbt::DeviceRestore dev_restore_;                \
    PBT_TRY(check_ctx(ctx));                        \
    std::lock_guard<std::mutex> lock_((ctx)->mu);   \
    (ctx)->launches = 0;                            \
    cudaStream_t st = (ctx)->stream

extern "C" int pbt_diff_main_c(pbt_ctx *ctx, const pbt_outbeam *beam, int64_t nbeam,
                               const pbt_outbeam *ext, int64_t next, const double *verts,
                               int64_t nverts, const int64_t *face_off, const int64_t *face_vi,
                               int64_t nfaces, const double *theta, int64_t ntheta,
                               const double *phi, int64_t nphi, double lambda, int32_t is_fast_diff,
                               int32_t precision, double *ampl_far_beam, double *ampl_far_ext_diff) {
    API_ENTER(ctx);
    PBT_TRY(check_lambda(lambda));
    if (!ampl_far_beam || !ampl_far_ext_diff) {
        set_error("output grids must not be NULL");
        return PBT_EINVAL;
    }
    if (precision != PBT_PREC_FP64 && precision != PBT_PREC_FP32) {
        set_error("unknown precision %d", precision);
        return PBT_EINVAL;
    }
    PBT_TRY(validate_angles(theta, ntheta, phi, nphi));
    PBT_TRY(validate_geometry(verts, nverts, face_off, face_vi, nfaces));
    PBT_TRY(validate_outbeams(beam, nbeam, nfaces, "beam"));
    PBT_TRY(validate_outbeams(ext, next, nfaces, "external diffraction"));
    PBT_TRY(grid_prepare(ctx, theta, ntheta, phi, nphi, st));
    PBT_TRY(check_grid_ready(ctx));
    const int64_t nb = ctx->grid.nb;
    PBT_TRY(ctx->d_out.ensure(2 * 8 * nb * sizeof(double)));
    double *d_afb = ctx->d_out.as<double>(), *d_afe = d_afb + 8 * nb;
    if (precision == PBT_PREC_FP64) {
        PBT_TRY(fp64_diff_main_device(ctx, st, beam, nbeam, ext, next, verts, nverts, face_off,
                                      face_vi, nfaces, lambda, is_fast_diff ? 1 : 0, d_afb, d_afe));
    } else {
        GeoDev G;
        PBT_TRY(upload_geometry(ctx, st, verts, nverts, 1, face_off, face_vi, nfaces, G));
        const size_t ob = sizeof(pbt_outbeam);
        PBT_TRY(ctx->d_fac.ensure(al((nbeam + 1) * ob) + (next + 1) * ob));
        pbt_outbeam *d_beam = ctx->d_fac.as<pbt_outbeam>();
        pbt_outbeam *d_ext = (pbt_outbeam *)(ctx->d_fac.as<char>() + al((nbeam + 1) * ob));
        if (nbeam) PBT_CUDA_TRY(cudaMemcpyAsync(d_beam, beam, nbeam * ob, cudaMemcpyHostToDevice, st));
        if (next) PBT_CUDA_TRY(cudaMemcpyAsync(d_ext, ext, next * ob, cudaMemcpyHostToDevice, st));
        PBT_TRY(k2_diff_main_impl(ctx, st, d_beam, nbeam, d_ext, next, G.verts, nverts, face_off,
                                  G.face_off, G.face_vi, nfaces, lambda, is_fast_diff ? 1 : 0, d_afb,
                                  d_afe));
    }
    PBT_CUDA_TRY(cudaMemcpyAsync(ampl_far_beam, d_afb, 8 * nb * sizeof(double),
                                 cudaMemcpyDeviceToHost, st));
    PBT_CUDA_TRY(cudaMemcpyAsync(ampl_far_ext_diff, d_afe, 8 * nb * sizeof(double),
                                 cudaMemcpyDeviceToHost, st));
    PBT_CUDA_TRY(cudaStreamSynchronize(st));
    return PBT_OK;
}

extern "C" int pbt_diffraction_c(pbt_ctx *ctx, const pbt_outbeam *outbeam, const double *verts,
                                 int64_t nverts, const int64_t *face_off, const int64_t *face_vi,
                                 int64_t nfaces, const double *theta, int64_t ntheta,
                                 const double *phi, int64_t nphi, double lambda,
                                 int32_t is_fast_diff, double *amplC) {
    API_ENTER(ctx);
    PBT_TRY(check_lambda(lambda));
    if (!outbeam || !amplC) {
        set_error("outbeam and amplC must not be NULL");
        return PBT_EINVAL;
    }
    PBT_TRY(validate_angles(theta, ntheta, phi, nphi));
    PBT_TRY(validate_geometry(verts, nverts, face_off, face_vi, nfaces));
    PBT_TRY(validate_outbeams(outbeam, 1, nfaces, "outbeam"));
    PBT_TRY(grid_prepare(ctx, theta, ntheta, phi, nphi, st));
    PBT_TRY(check_grid_ready(ctx));
    const int64_t nb = ctx->grid.nb;
    std::vector<K1Facet> fac;
    std::vector<K1Edge> edges;
    PBT_TRY(k1_build_facets(outbeam, 1, -1.0, verts, nverts, face_off, face_vi, nfaces, lambda, fac,
                            edges));
    PBT_TRY(upload(ctx->d_fac, fac.data(), fac.size(), st));
    PBT_TRY(upload(ctx->d_edge, edges.data(), edges.size(), st));
    PBT_TRY(ctx->d_out.ensure(8 * nb * sizeof(double)));
    PBT_TRY(k1_launch(ctx, st, ctx->d_fac.as<K1Facet>(), 1, ctx->d_edge.as<K1Edge>(), lambda,
                      is_fast_diff ? 1 : 0, ctx->d_out.as<double>()));
    PBT_CUDA_TRY(cudaMemcpyAsync(amplC, ctx->d_out.p, 8 * nb * sizeof(double),
                                 cudaMemcpyDeviceToHost, st));
    PBT_CUDA_TRY(cudaStreamSynchronize(st));
    return PBT_OK;
}

extern "C" int pbt_finalise_c(pbt_ctx *ctx, const double *ampl_far_beam,
                              const double *ampl_far_ext_diff, const double *theta, int64_t ntheta,
                              const double *phi, int64_t nphi, double lambda, int32_t scaling,
                              pbt_output_params *params, double *mueller, double *mueller_1d,
                              int32_t accumulate) {
    API_ENTER(ctx);
    PBT_TRY(check_lambda(lambda));
    if (!ampl_far_beam || !ampl_far_ext_diff || !params) {
        set_error("amplitude grids and params must not be NULL");
        return PBT_EINVAL;
    }
    PBT_TRY(validate_angles(theta, ntheta, phi, nphi));
    PBT_TRY(grid_prepare(ctx, theta, ntheta, phi, nphi, st));
    const int64_t nb = ctx->grid.nb;
    if (accumulate) PBT_TRY(totals_ensure(ctx->tot, ntheta, nphi, st));
    // d_out: afb | afe ; d_mu: mueller | m1d | params
    PBT_TRY(ctx->d_out.ensure(2 * 8 * nb * sizeof(double)));
    PBT_TRY(ctx->d_mu.ensure((16 * nb + 16 * ntheta + 18) * sizeof(double)));
    double *d_afb = ctx->d_out.as<double>(), *d_afe = d_afb + 8 * nb;
    double *d_mu = ctx->d_mu.as<double>(), *d_m1 = d_mu + 16 * nb, *d_p = d_m1 + 16 * ntheta;
    PBT_CUDA_TRY(cudaMemcpyAsync(d_afb, ampl_far_beam, 8 * nb * sizeof(double),
                                 cudaMemcpyHostToDevice, st));
    PBT_CUDA_TRY(cudaMemcpyAsync(d_afe, ampl_far_ext_diff, 8 * nb * sizeof(double),
                                 cudaMemcpyHostToDevice, st));
    const pbt_output_params pin = *params;
    PBT_TRY(k3_finalise(ctx, st, d_afb, d_afe, lambda, scaling ? 1 : 0, &pin, d_mu, d_m1, d_p,
                        accumulate ? &ctx->tot : nullptr));
    if (mueller)
        PBT_CUDA_TRY(cudaMemcpyAsync(mueller, d_mu, 16 * nb * sizeof(double),
                                     cudaMemcpyDeviceToHost, st));
    if (mueller_1d)
        PBT_CUDA_TRY(cudaMemcpyAsync(mueller_1d, d_m1, 16 * ntheta * sizeof(double),
                                     cudaMemcpyDeviceToHost, st));
    PBT_CUDA_TRY(cudaMemcpyAsync(params, d_p, sizeof(pbt_output_params), cudaMemcpyDeviceToHost, st));
    PBT_CUDA_TRY(cudaStreamSynchronize(st));
    return PBT_OK;
}

extern "C" int pbt_summation_c(pbt_ctx *ctx, const double *mueller, const double *mueller_1d,
                               const pbt_output_params *params, int64_t ntheta, int64_t nphi) {
    API_ENTER(ctx);
    if (!mueller || !mueller_1d || !params || ntheta < 1 || nphi < 1) {
        set_error("summation: bad arguments");
        return PBT_EINVAL;
    }
    PBT_TRY(totals_ensure(ctx->tot, ntheta, nphi, st));
    const int64_t nb = ntheta * nphi;
    PBT_TRY(ctx->d_mu.ensure((16 * nb + 16 * ntheta + 18) * sizeof(double)));
    double *d_mu = ctx->d_mu.as<double>(), *d_m1 = d_mu + 16 * nb, *d_p = d_m1 + 16 * ntheta;
    PBT_CUDA_TRY(cudaMemcpyAsync(d_mu, mueller, 16 * nb * 8, cudaMemcpyHostToDevice, st));
    PBT_CUDA_TRY(cudaMemcpyAsync(d_m1, mueller_1d, 16 * ntheta * 8, cudaMemcpyHostToDevice, st));
    PBT_CUDA_TRY(cudaMemcpyAsync(d_p, params, sizeof(pbt_output_params), cudaMemcpyHostToDevice, st));
    PBT_TRY(totals_add_device(ctx, ctx->tot, st, d_mu, d_m1, d_p));
    PBT_CUDA_TRY(cudaStreamSynchronize(st));
    return PBT_OK;
}

extern "C" int pbt_divide_by_num_orientations_c(pbt_ctx *ctx, int64_t num_orients,
                                                double *mueller_total, double *mueller_1d_total,
                                                pbt_output_params *params_total) {
    API_ENTER(ctx);
    if (num_orients < 1 || !mueller_total || !mueller_1d_total || !params_total) {
        set_error("divide: bad arguments");
        return PBT_EINVAL;
    }
    if (ctx->tot.count == 0 || !ctx->tot.mu.p) {
        set_error("divide: no orientation has been accumulated");
        return PBT_ESTATE;
    }
    const int64_t nb = ctx->tot.ntheta * ctx->tot.nphi, nt = ctx->tot.ntheta;
    PBT_TRY(ctx->d_mu.ensure((16 * nb + 16 * nt + 18) * sizeof(double)));
    double *d_mu = ctx->d_mu.as<double>(), *d_m1 = d_mu + 16 * nb, *d_p = d_m1 + 16 * nt;
    PBT_TRY(totals_divide_device(ctx, ctx->tot, st, num_orients, d_mu, d_m1, d_p));
    PBT_CUDA_TRY(cudaMemcpyAsync(mueller_total, d_mu, 16 * nb * 8, cudaMemcpyDeviceToHost, st));
    PBT_CUDA_TRY(cudaMemcpyAsync(mueller_1d_total, d_m1, 16 * nt * 8, cudaMemcpyDeviceToHost, st));
    PBT_CUDA_TRY(cudaMemcpyAsync(params_total, d_p, sizeof(pbt_output_params),
                                 cudaMemcpyDeviceToHost, st));
    PBT_CUDA_TRY(cudaStreamSynchronize(st));
    return PBT_OK;
}

extern "C" int pbt_totals_reset_c(pbt_ctx *ctx) {
    API_ENTER(ctx);
    PBT_TRY(totals_reset(ctx->tot, st));
    PBT_CUDA_TRY(cudaStreamSynchronize(st));
    return PBT_OK;
}

namespace {

int batch_common_checks(pbt_ctx *ctx, int64_t norient, const int64_t *beam_off,
                        const int64_t *ext_off, const int64_t *face_off, int64_t nfaces,
                        const double *theta, int64_t ntheta, const double *phi, int64_t nphi,
                        double lambda, int32_t precision, const void *mu_avg, const void *m1_avg,
                        const void *p_avg, const void *p_in) {
    (void)ctx;
    PBT_TRY(check_lambda(lambda));
    if (norient < 1) {
        set_error("norient must be >= 1");
        return PBT_EINVAL;
    }
    if (precision != PBT_PREC_FP64 && precision != PBT_PREC_FP32) {
        set_error("unknown precision %d", precision);
        return PBT_EINVAL;
    }
    if (!mu_avg || !m1_avg || !p_avg || !p_in) {
        set_error("batch: output arrays and params_in must not be NULL");
        return PBT_EINVAL;
    }
    PBT_TRY(check_offsets(beam_off, norient, "beam"));
    PBT_TRY(check_offsets(ext_off, norient, "ext"));
    if (!face_off || face_off[0] != 0 || nfaces < 1) {
        set_error("batch: bad face_off");
        return PBT_EINVAL;
    }
    PBT_TRY(validate_angles(theta, ntheta, phi, nphi));
    return PBT_OK;
}

}  // namespace

namespace {

// The host batch over per-orientation arrays: beams[o] (boff[o+1]-boff[o]
// records), exts[o], verts[o] (nverts x 3, column-major).  Both host batch
// entry points land here; consecutive orientations whose arrays are adjacent
// in memory are copied in one piece.
struct HostRuns {
    const pbt_outbeam *const *beam;
    const pbt_outbeam *const *ext;
    const double *const *verts;
    const int64_t *boff, *eoff;
};

// Copies orientations [o0, o1) of one kind into consecutive device records.
int copy_lists(const pbt_outbeam *const *src, const int64_t *off, int64_t o0, int64_t o1,
               pbt_outbeam *dst, cudaStream_t s) {
    int64_t o = o0;
    while (o < o1) {
        const pbt_outbeam *p = src[o];
        int64_t n = off[o + 1] - off[o], e = o + 1;
        while (e < o1 && src[e] == p + n) {
            n += off[e + 1] - off[e];
            e++;
        }
        if (n) PBT_CUDA_TRY(cudaMemcpyAsync(dst + (off[o] - off[o0]), p, n * sizeof(pbt_outbeam),
                                            cudaMemcpyHostToDevice, s));
        o = e;
    }
    return PBT_OK;
}

int host_batch(pbt_ctx *ctx, cudaStream_t st, int64_t norient, const HostRuns &H, int64_t nverts,
               const int64_t *face_off, const int64_t *face_vi, int64_t nfaces,
               const double *theta, int64_t ntheta, const double *phi, int64_t nphi,
               double lambda, int32_t is_fast_diff, int32_t scaling, int32_t precision,
               const pbt_output_params *params_in, double *mueller_avg, double *mueller_1d_avg,
               pbt_output_params *params_avg, pbt_output_params *params_per_orient) {
    const int64_t *beam_off = H.boff, *ext_off = H.eoff;
    PBT_TRY(batch_common_checks(ctx, norient, beam_off, ext_off, face_off, nfaces, theta, ntheta,
                                phi, nphi, lambda, precision, mueller_avg, mueller_1d_avg,
                                params_avg, params_in));
    for (int64_t o = 0; o < norient; o++) {
        PBT_TRY(validate_geometry(H.verts[o], nverts, face_off, face_vi, nfaces));
        PBT_TRY(validate_outbeams(H.beam[o], beam_off[o + 1] - beam_off[o], nfaces, "beam"));
        PBT_TRY(validate_outbeams(H.ext[o], ext_off[o + 1] - ext_off[o], nfaces,
                                  "external diffraction"));
    }
    PBT_TRY(grid_prepare(ctx, theta, ntheta, phi, nphi, st));
    PBT_TRY(check_grid_ready(ctx));
    const int64_t nb = ctx->grid.nb;
    if (precision == PBT_PREC_FP64) {
        // the per-orientation loop of src/pbt_seq_mod.f90:146-269 on the device
        DevTotals &T = ctx->btot;
        T.count = 0;
        PBT_TRY(totals_ensure(T, ntheta, nphi, st));
        PBT_TRY(totals_reset(T, st));
        PBT_TRY(ctx->d_out.ensure(2 * 8 * nb * sizeof(double)));
        PBT_TRY(ctx->d_mu.ensure((16 * nb + 16 * ntheta + 18) * sizeof(double)));
        double *d_afb = ctx->d_out.as<double>(), *d_afe = d_afb + 8 * nb;
        double *d_mu = ctx->d_mu.as<double>(), *d_m1 = d_mu + 16 * nb, *d_p = d_m1 + 16 * ntheta;
        for (int64_t o = 0; o < norient; o++) {
            PBT_TRY(fp64_diff_main_device(ctx, st, H.beam[o], beam_off[o + 1] - beam_off[o],
                                          H.ext[o], ext_off[o + 1] - ext_off[o], H.verts[o],
                                          nverts, face_off, face_vi, nfaces, lambda,
                                          is_fast_diff ? 1 : 0, d_afb, d_afe));
            PBT_TRY(k3_finalise(ctx, st, d_afb, d_afe, lambda, scaling ? 1 : 0, &params_in[o], d_mu,
                                d_m1, d_p, &T));
            if (params_per_orient)
                PBT_CUDA_TRY(cudaMemcpyAsync(&params_per_orient[o], d_p, sizeof(pbt_output_params),
                                             cudaMemcpyDeviceToHost, st));
        }
        PBT_TRY(totals_divide_device(ctx, T, st, norient, d_mu, d_m1, d_p));
        PBT_CUDA_TRY(cudaMemcpyAsync(mueller_avg, d_mu, 16 * nb * 8, cudaMemcpyDeviceToHost, st));
        PBT_CUDA_TRY(cudaMemcpyAsync(mueller_1d_avg, d_m1, 16 * ntheta * 8, cudaMemcpyDeviceToHost, st));
        PBT_CUDA_TRY(cudaMemcpyAsync(params_avg, d_p, sizeof(pbt_output_params),
                                     cudaMemcpyDeviceToHost, st));
        PBT_CUDA_TRY(cudaStreamSynchronize(st));
        return PBT_OK;
    }
    // FP32 batched path.  The orientations go in runs of about an eighth of the
    // outbeams each: run k+1's outbeams are copied on the copy stream into one
    // of two slots while run k computes on the compute stream.
    GeoDev G;
    {
        const bool contiguous = [&] {
            for (int64_t o = 1; o < norient; o++)
                if (H.verts[o] != H.verts[0] + o * 3 * nverts) return false;
            return true;
        }();
        PBT_TRY(upload_geometry(ctx, st, contiguous ? H.verts[0] : nullptr, nverts, norient,
                                face_off, face_vi, nfaces, G));
        if (!contiguous)
            for (int64_t o = 0; o < norient; o++)
                PBT_CUDA_TRY(cudaMemcpyAsync(const_cast<double *>(G.verts) + o * 3 * nverts,
                                             H.verts[o], 3 * nverts * 8, cudaMemcpyHostToDevice, st));
    }
    const size_t ob = sizeof(pbt_outbeam);
    const int64_t nbt = beam_off[norient], net = ext_off[norient];
    std::vector<int64_t> run{0};
    {
        const int64_t target = std::max<int64_t>((nbt + net) / 8, 262144);
        int64_t acc = 0;
        for (int64_t o = 0; o < norient; o++) {
            acc += (beam_off[o + 1] - beam_off[o]) + (ext_off[o + 1] - ext_off[o]);
            if (acc >= target && o + 1 < norient) {
                run.push_back(o + 1);
                acc = 0;
            }
        }
        run.push_back(norient);
    }
    const int64_t nrun = (int64_t)run.size() - 1;
    int64_t mb = 0, me = 0, mo = 0;
    for (int64_t k = 0; k < nrun; k++) {
        mb = std::max(mb, beam_off[run[k + 1]] - beam_off[run[k]]);
        me = std::max(me, ext_off[run[k + 1]] - ext_off[run[k]]);
        mo = std::max(mo, run[k + 1] - run[k]);
    }
    const int nslot = nrun > 1 ? 2 : 1;
    size_t o_slot[2][2], off = 0;
    for (int i = 0; i < nslot; i++) {
        o_slot[i][0] = off;
        off = al(off + (mb + 1) * ob);
        o_slot[i][1] = off;
        off = al(off + (me + 1) * ob);
    }
    const size_t o_pi = off, o_pp = al(o_pi + norient * sizeof(pbt_output_params)),
                 o_mu = al(o_pp + norient * sizeof(pbt_output_params)),
                 o_m1 = al(o_mu + 16 * nb * 8), o_pa = al(o_m1 + 16 * ntheta * 8),
                 o_end = al(o_pa + sizeof(pbt_output_params));
    PBT_TRY(ctx->d_fac.ensure(o_end));
    char *b = ctx->d_fac.as<char>();
    pbt_output_params *d_pin = (pbt_output_params *)(b + o_pi), *d_pp = (pbt_output_params *)(b + o_pp),
                      *d_pa = (pbt_output_params *)(b + o_pa);
    double *d_mu = (double *)(b + o_mu), *d_m1 = (double *)(b + o_m1);
    PBT_CUDA_TRY(cudaMemcpyAsync(d_pin, params_in, norient * sizeof(pbt_output_params),
                                 cudaMemcpyHostToDevice, st));
    cudaStream_t cs = st;
    if (nrun > 1) {
        if (!ctx->copy_stream)
            PBT_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
        for (int i = 0; i < 2; i++) {
            if (!ctx->up_ev[i]) PBT_CUDA_TRY(cudaEventCreateWithFlags(&ctx->up_ev[i], cudaEventDisableTiming));
            if (!ctx->done_ev[i]) PBT_CUDA_TRY(cudaEventCreateWithFlags(&ctx->done_ev[i], cudaEventDisableTiming));
        }
        cs = ctx->copy_stream;
        try {
            if (ctx->h_gather.size() < (size_t)(mb + me + 2) * ob) ctx->h_gather.resize((size_t)(mb + me + 2) * ob);
        } catch (...) {
            set_error("batch: out of host memory for the gather buffer");
            return PBT_ENOMEM;
        }
        // the slots (and the buffers before them) may still be read by earlier work on st
        PBT_CUDA_TRY(cudaEventRecord(ctx->done_ev[0], st));
        PBT_CUDA_TRY(cudaStreamWaitEvent(cs, ctx->done_ev[0], 0));
    }
    K2Batch B;
    PBT_TRY(k2_batch_begin(ctx, st, norient, mo, d_pp, B));
    std::vector<int64_t> hbo(mo + 1), heo(mo + 1);
    for (int64_t k = 0; k < nrun; k++) {
        const int slot = (int)(k % nslot);
        const int64_t o0 = run[k], no = run[k + 1] - run[k];
        const int64_t b0 = beam_off[o0], e0 = ext_off[o0];
        const int64_t nbk = beam_off[o0 + no] - b0, nek = ext_off[o0 + no] - e0;
        pbt_outbeam *d_beam = (pbt_outbeam *)(b + o_slot[slot][0]);
        pbt_outbeam *d_ext = (pbt_outbeam *)(b + o_slot[slot][1]);
        if (nrun > 1) {
            // gather the run on the host (threads), then one copy per kind; the
            // copy returns once the host buffer is staged, so one buffer serves
            char *hb = ctx->h_gather.data();
            pbt_outbeam *hbeam = (pbt_outbeam *)hb, *hext = (pbt_outbeam *)(hb + mb * ob);
#pragma omp parallel for schedule(dynamic, 8)
            for (int64_t o = o0; o < o0 + no; o++) {
                const int64_t nbo = beam_off[o + 1] - beam_off[o], neo = ext_off[o + 1] - ext_off[o];
                if (nbo) memcpy(hbeam + (beam_off[o] - b0), H.beam[o], nbo * ob);
                if (neo) memcpy(hext + (ext_off[o] - e0), H.ext[o], neo * ob);
            }
            if (k >= 2) PBT_CUDA_TRY(cudaStreamWaitEvent(cs, ctx->done_ev[slot], 0));
            if (nbk) PBT_CUDA_TRY(cudaMemcpyAsync(d_beam, hbeam, nbk * ob, cudaMemcpyHostToDevice, cs));
            if (nek) PBT_CUDA_TRY(cudaMemcpyAsync(d_ext, hext, nek * ob, cudaMemcpyHostToDevice, cs));
            PBT_CUDA_TRY(cudaEventRecord(ctx->up_ev[slot], cs));
            PBT_CUDA_TRY(cudaStreamWaitEvent(st, ctx->up_ev[slot], 0));
        } else {
            if (nbk) PBT_TRY(copy_lists(H.beam, beam_off, o0, o0 + no, d_beam, cs));
            if (nek) PBT_TRY(copy_lists(H.ext, ext_off, o0, o0 + no, d_ext, cs));
        }
        for (int64_t q = 0; q <= no; q++) {
            hbo[q] = beam_off[o0 + q] - b0;
            heo[q] = ext_off[o0 + q] - e0;
        }
        PBT_TRY(k2_batch_add(ctx, st, B, o0, no, d_beam, hbo.data(), d_ext, heo.data(),
                             G.verts + o0 * 3 * nverts, nverts, face_off, G.face_off, G.face_vi,
                             nfaces, lambda, is_fast_diff ? 1 : 0, scaling ? 1 : 0, d_pin));
        if (nrun > 1) PBT_CUDA_TRY(cudaEventRecord(ctx->done_ev[slot], st));
    }
    PBT_TRY(k2_batch_finish(ctx, st, B, d_pin, d_mu, d_m1, d_pa, 1));
    PBT_CUDA_TRY(cudaMemcpyAsync(mueller_avg, d_mu, 16 * nb * 8, cudaMemcpyDeviceToHost, st));
    PBT_CUDA_TRY(cudaMemcpyAsync(mueller_1d_avg, d_m1, 16 * ntheta * 8, cudaMemcpyDeviceToHost, st));
    PBT_CUDA_TRY(cudaMemcpyAsync(params_avg, d_pa, sizeof(pbt_output_params), cudaMemcpyDeviceToHost,
                                 st));
    if (params_per_orient)
        PBT_CUDA_TRY(cudaMemcpyAsync(params_per_orient, d_pp, norient * sizeof(pbt_output_params),
                                     cudaMemcpyDeviceToHost, st));
    PBT_CUDA_TRY(cudaStreamSynchronize(st));
    return PBT_OK;
}

}  // namespace

extern "C" int pbt_diff_batch_c(pbt_ctx *ctx, int64_t norient, const pbt_outbeam *beam,
                                const int64_t *beam_off, const pbt_outbeam *ext,
                                const int64_t *ext_off, const double *verts, int64_t nverts,
                                const int64_t *face_off, const int64_t *face_vi, int64_t nfaces,
                                const double *theta, int64_t ntheta, const double *phi,
                                int64_t nphi, double lambda, int32_t is_fast_diff, int32_t scaling,
                                int32_t precision, const pbt_output_params *params_in,
                                double *mueller_avg, double *mueller_1d_avg,
                                pbt_output_params *params_avg,
                                pbt_output_params *params_per_orient) {
    API_ENTER(ctx);
    if (norient < 1 || !verts) {
        set_error(norient < 1 ? "norient must be >= 1" : "batch: verts must not be NULL");
        return PBT_EINVAL;
    }
    PBT_TRY(check_offsets(beam_off, norient, "beam"));
    PBT_TRY(check_offsets(ext_off, norient, "ext"));
    std::vector<const pbt_outbeam *> pb(norient), pe(norient);
    std::vector<const double *> pv(norient);
    for (int64_t o = 0; o < norient; o++) {
        pb[o] = beam ? beam + beam_off[o] : nullptr;
        pe[o] = ext ? ext + ext_off[o] : nullptr;
        pv[o] = verts + o * 3 * nverts;
    }
    const HostRuns H{pb.data(), pe.data(), pv.data(), beam_off, ext_off};
    return host_batch(ctx, st, norient, H, nverts, face_off, face_vi, nfaces, theta, ntheta, phi,
                      nphi, lambda, is_fast_diff, scaling, precision, params_in, mueller_avg,
                      mueller_1d_avg, params_avg, params_per_orient);
}

extern "C" int pbt_diff_batch_list_c(pbt_ctx *ctx, int64_t norient,
                                     const pbt_outbeam *const *beams, const int64_t *nbeam,
                                     const pbt_outbeam *const *exts, const int64_t *next,
                                     const double *const *verts, int64_t nverts,
                                     const int64_t *face_off, const int64_t *face_vi,
                                     int64_t nfaces, const double *theta, int64_t ntheta,
                                     const double *phi, int64_t nphi, double lambda,
                                     int32_t is_fast_diff, int32_t scaling, int32_t precision,
                                     const pbt_output_params *params_in, double *mueller_avg,
                                     double *mueller_1d_avg, pbt_output_params *params_avg,
                                     pbt_output_params *params_per_orient) {
    API_ENTER(ctx);
    if (norient < 1 || !beams || !nbeam || !exts || !next || !verts) {
        set_error(norient < 1 ? "norient must be >= 1" : "batch: NULL list argument");
        return PBT_EINVAL;
    }
    std::vector<int64_t> boff(norient + 1, 0), eoff(norient + 1, 0);
    for (int64_t o = 0; o < norient; o++) {
        if (nbeam[o] < 0 || next[o] < 0 || !verts[o]) {
            set_error("batch: orientation %lld has a negative count or NULL vertices",
                      (long long)(o + 1));
            return PBT_EINVAL;
        }
        boff[o + 1] = boff[o] + nbeam[o];
        eoff[o + 1] = eoff[o] + next[o];
    }
    const HostRuns H{beams, exts, verts, boff.data(), eoff.data()};
    return host_batch(ctx, st, norient, H, nverts, face_off, face_vi, nfaces, theta, ntheta, phi,
                      nphi, lambda, is_fast_diff, scaling, precision, params_in, mueller_avg,
                      mueller_1d_avg, params_avg, params_per_orient);
}

namespace {

// Checks and enqueue of the device-pointer batch; copy_face_off = false when
// the face offsets are already on the device (a graph capture reuses them).
int dev_batch_enqueue(pbt_ctx *ctx, cudaStream_t st, int64_t norient, const pbt_outbeam *beam,
                      const int64_t *beam_off, const pbt_outbeam *ext, const int64_t *ext_off,
                      const double *verts, int64_t nverts, const int64_t *face_off,
                      const int64_t *face_vi, int64_t nfaces, const double *theta, int64_t ntheta,
                      const double *phi, int64_t nphi, double lambda, int32_t is_fast_diff,
                      int32_t scaling, int32_t precision, const pbt_output_params *params_in,
                      double *mueller_avg, double *mueller_1d_avg, pbt_output_params *params_avg,
                      pbt_output_params *params_per_orient, bool copy_face_off) {
    ctx->launches = 0;
    PBT_TRY(batch_common_checks(ctx, norient, beam_off, ext_off, face_off, nfaces, theta, ntheta,
                                phi, nphi, lambda, precision, mueller_avg, mueller_1d_avg,
                                params_avg, params_in));
    if (precision != PBT_PREC_FP32) {
        set_error("the device-pointer batch entry point runs the FP32 path only; use "
                  "pbt_diff_batch_c for the reference-exact FP64 path");
        return PBT_EINVAL;
    }
    if ((beam_off[norient] > 0 && !beam) || (ext_off[norient] > 0 && !ext) || !verts || !face_vi) {
        set_error("batch: device arrays must not be NULL");
        return PBT_EINVAL;
    }
    PBT_TRY(grid_prepare(ctx, theta, ntheta, phi, nphi, st));
    PBT_TRY(check_grid_ready(ctx));
    // the face offsets are needed on the device too
    PBT_TRY(ctx->d_items.ensure((nfaces + 1) * 8));
    if (copy_face_off)
        PBT_CUDA_TRY(cudaMemcpyAsync(ctx->d_items.p, face_off, (nfaces + 1) * 8,
                                     cudaMemcpyHostToDevice, st));
    return k2_batch_impl(ctx, st, norient, beam, beam_off, ext, ext_off, verts, nverts, face_off,
                         ctx->d_items.as<int64_t>(), face_vi, nfaces, lambda, is_fast_diff ? 1 : 0,
                         scaling ? 1 : 0, params_in, mueller_avg, mueller_1d_avg, params_avg,
                         params_per_orient, 0);
}

}  // namespace

extern "C" int pbt_diff_batch_dev_c(pbt_ctx *ctx, void *stream, int64_t norient,
                                    const pbt_outbeam *beam, const int64_t *beam_off,
                                    const pbt_outbeam *ext, const int64_t *ext_off,
                                    const double *verts, int64_t nverts, const int64_t *face_off,
                                    const int64_t *face_vi, int64_t nfaces, const double *theta,
                                    int64_t ntheta, const double *phi, int64_t nphi, double lambda,
                                    int32_t is_fast_diff, int32_t scaling, int32_t precision,
                                    const pbt_output_params *params_in, double *mueller_avg,
                                    double *mueller_1d_avg, pbt_output_params *params_avg,
                                    pbt_output_params *params_per_orient) {
    clear_error();
    PBT_TRY(check_ctx(ctx));
    std::lock_guard<std::mutex> lock_(ctx->mu);
    return dev_batch_enqueue(ctx, (cudaStream_t)stream, norient, beam, beam_off, ext, ext_off,
                             verts, nverts, face_off, face_vi, nfaces, theta, ntheta, phi, nphi,
                             lambda, is_fast_diff, scaling, precision, params_in, mueller_avg,
                             mueller_1d_avg, params_avg, params_per_orient, true);
}

// A CUDA graph of the device-pointer batch.  The graph owns a private context
// (its scratch buffers, bin tables and staged offsets), so nothing else
// writes what a replay reads; the caller's device arrays are baked in by
// address and read at every replay.
struct pbt_graph {
    pbt_ctx *gctx = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int64_t launches = 0;
    int device = 0;
};

extern "C" int pbt_diff_batch_dev_graph_c(pbt_ctx *ctx, void *stream, int64_t norient,
                                          const pbt_outbeam *beam, const int64_t *beam_off,
                                          const pbt_outbeam *ext, const int64_t *ext_off,
                                          const double *verts, int64_t nverts,
                                          const int64_t *face_off, const int64_t *face_vi,
                                          int64_t nfaces, const double *theta, int64_t ntheta,
                                          const double *phi, int64_t nphi, double lambda,
                                          int32_t is_fast_diff, int32_t scaling,
                                          const pbt_output_params *params_in,
                                          double *mueller_avg, double *mueller_1d_avg,
                                          pbt_output_params *params_avg,
                                          pbt_output_params *params_per_orient, pbt_graph **out) {
    clear_error();
    pbt::DeviceRestore dev_restore_;
    PBT_TRY(check_ctx(ctx));
    if (!out) {
        set_error("graph: out must not be NULL");
        return PBT_EINVAL;
    }
    *out = nullptr;
    PBT_CUDA_TRY(cudaSetDevice(ctx->device));
    pbt_ctx *g = nullptr;
    PBT_TRY(pbt_ctx_create(ctx->device, &g));
    g->plan_variant = ctx->plan_variant;
    g->plan_bpt = ctx->plan_bpt;
    g->plan_rpi = ctx->plan_rpi;
    cudaStream_t st = (cudaStream_t)stream;
    auto fail = [&](int rc) {
        pbt_ctx_destroy(g);
        return rc;
    };
    auto cfail = [&](const char *what, cudaError_t e) {
        set_error("%s failed: %s", what, cudaGetErrorString(e));
        return fail(e == cudaErrorMemoryAllocation ? PBT_ENOMEM : PBT_ECUDA);
    };
    cudaError_t e;
    // a plain run sizes every buffer, stages the offsets and fills the bin tables
    int rc = dev_batch_enqueue(g, st, norient, beam, beam_off, ext, ext_off, verts, nverts,
                               face_off, face_vi, nfaces, theta, ntheta, phi, nphi, lambda,
                               is_fast_diff, scaling, PBT_PREC_FP32, params_in, mueller_avg,
                               mueller_1d_avg, params_avg, params_per_orient, true);
    if (rc != PBT_OK) return fail(rc);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cfail("graph warm-up", e);
    cudaStream_t cs = nullptr;
    if ((e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking)) != cudaSuccess)
        return cfail("cudaStreamCreateWithFlags", e);
    g->capturing = true;
    cudaGraph_t graph = nullptr;
    if ((e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed)) != cudaSuccess) {
        g->capturing = false;
        cudaStreamDestroy(cs);
        return cfail("cudaStreamBeginCapture", e);
    }
    rc = dev_batch_enqueue(g, cs, norient, beam, beam_off, ext, ext_off, verts, nverts, face_off,
                           face_vi, nfaces, theta, ntheta, phi, nphi, lambda, is_fast_diff,
                           scaling, PBT_PREC_FP32, params_in, mueller_avg, mueller_1d_avg,
                           params_avg, params_per_orient, false);
    const cudaError_t ce = cudaStreamEndCapture(cs, &graph);
    g->capturing = false;
    cudaStreamDestroy(cs);
    if (rc != PBT_OK || ce != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        (void)cudaGetLastError();
        if (rc == PBT_OK) {
            set_error("graph capture failed: %s", cudaGetErrorString(ce));
            rc = PBT_ECUDA;
        }
        return fail(rc);
    }
    cudaGraphExec_t exec = nullptr;
    if ((e = cudaGraphInstantiate(&exec, graph, 0)) != cudaSuccess) {
        cudaGraphDestroy(graph);
        return cfail("cudaGraphInstantiate", e);
    }
    pbt_graph *G = new (std::nothrow) pbt_graph;
    if (!G) {
        cudaGraphExecDestroy(exec);
        cudaGraphDestroy(graph);
        set_error("graph: out of host memory");
        return fail(PBT_ENOMEM);
    }
    G->gctx = g;
    G->graph = graph;
    G->exec = exec;
    G->launches = g->launches;
    G->device = ctx->device;
    *out = G;
    return PBT_OK;
}

extern "C" int pbt_graph_launch_c(pbt_graph *G, void *stream) {
    clear_error();
    if (!G || !G->exec) {
        set_error("graph: NULL or destroyed graph");
        return PBT_EINVAL;
    }
    pbt::DeviceRestore dev_restore_;
    PBT_CUDA_TRY(cudaSetDevice(G->device));
    PBT_CUDA_TRY(cudaGraphLaunch(G->exec, (cudaStream_t)stream));
    return PBT_OK;
}

extern "C" int64_t pbt_graph_kernel_count(const pbt_graph *G) { return G ? G->launches : -1; }

extern "C" int pbt_graph_destroy_c(pbt_graph *G) {
    clear_error();
    if (!G) return PBT_OK;
    pbt::DeviceRestore dev_restore_;
    cudaSetDevice(G->device);
    if (G->exec) cudaGraphExecDestroy(G->exec);
    if (G->graph) cudaGraphDestroy(G->graph);
    pbt_ctx_destroy(G->gctx);
    delete G;
    return PBT_OK;
}

namespace pbt {
int k4_adjoint(pbt_ctx *ctx, cudaStream_t st, const pbt_outbeam *beam, int64_t nbeam,
               const pbt_outbeam *ext, int64_t next, const double *verts, int64_t nverts,
               const int64_t *face_off, const int64_t *face_vi, int64_t nfaces, double lambda,
               int fast_diff, const double *gafb, const double *gafe, double *gverts,
               double *gbeam, double *gext);
}

extern "C" int pbt_diff_adjoint_c(pbt_ctx *ctx, const pbt_outbeam *beam, int64_t nbeam,
                                  const pbt_outbeam *ext, int64_t next, const double *verts,
                                  int64_t nverts, const int64_t *face_off, const int64_t *face_vi,
                                  int64_t nfaces, const double *theta, int64_t ntheta,
                                  const double *phi, int64_t nphi, double lambda,
                                  int32_t is_fast_diff, const double *grad_ampl_far_beam,
                                  const double *grad_ampl_far_ext_diff, double *grad_verts,
                                  double *grad_beam_ampl, double *grad_ext_ampl) {
    API_ENTER(ctx);
    PBT_TRY(check_lambda(lambda));
    if (!grad_ampl_far_beam || !grad_ampl_far_ext_diff || !grad_verts ||
        (nbeam > 0 && !grad_beam_ampl) || (next > 0 && !grad_ext_ampl)) {
        set_error("adjoint: gradient arrays must not be NULL");
        return PBT_EINVAL;
    }
    PBT_TRY(validate_angles(theta, ntheta, phi, nphi));
    PBT_TRY(validate_geometry(verts, nverts, face_off, face_vi, nfaces));
    PBT_TRY(validate_outbeams(beam, nbeam, nfaces, "beam"));
    PBT_TRY(validate_outbeams(ext, next, nfaces, "external diffraction"));
    PBT_TRY(grid_prepare(ctx, theta, ntheta, phi, nphi, st));
    PBT_TRY(check_grid_ready(ctx));
    return k4_adjoint(ctx, st, beam, nbeam, ext, next, verts, nverts, face_off, face_vi, nfaces,
                      lambda, is_fast_diff ? 1 : 0, grad_ampl_far_beam, grad_ampl_far_ext_diff,
                      grad_verts, grad_beam_ampl, grad_ext_ampl);
}

// Failure-detection self-test: a device wait that nothing completes must end
// by itself within limit_ms and come back as PBT_ETIMEOUT with the context
// still usable.
extern "C" int pbt_selftest_bounded_wait_c(pbt_ctx *ctx, int32_t limit_ms) {
    API_ENTER(ctx);
    if (limit_ms < 1 || limit_ms > 5000) {
        set_error("self-test limit must be 1..5000 ms");
        return PBT_EINVAL;
    }
    return k2_wait_selftest(ctx, st, (uint64_t)limit_ms * 1000000ull);
}
