/* c_drop_in.c -- a plain C caller of libpbt_b200.so (include/pbt_diff.h).
 *
 * One triangular facet, one beam outbeam and one external-diffraction
 * outbeam: diff_main in FP64 and FP32, then finalise.  Prints
 * "ok <rel diff fp32/fp64> <scatt> <asymmetry>" and exits 0 on success.
 *
 *   gcc -O2 -I include c_drop_in.c -L abt_b200 -lpbt_b200 -Wl,-rpath,abt_b200 -lm
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "pbt_diff.h"

#define CHECK(call)                                                                  \
    do {                                                                             \
        int s_ = (call);                                                             \
        if (s_ != PBT_OK) {                                                          \
            fprintf(stderr, "%s -> %d: %s\n", #call, s_, pbt_last_error_string());   \
            return 1;                                                                \
        }                                                                            \
    } while (0)

int main(void) {
    const double pi = (double)3.14159265358979f;
    enum { NT = 91, NP = 90 };
    double theta[NT], phi[NP];
    for (int i = 0; i < NT; i++) theta[i] = (2.0 * i) * pi / 180.0;
    for (int i = 0; i < NP; i++) phi[i] = (4.0 * i) * pi / 180.0;
    /* v(3,3) column-major: x of the three vertices, then y, then z */
    double v[9] = {0.1, 1.3, 0.2, 0.2, 0.3, 1.4, 0.0, 0.1, -0.1};
    int64_t face_off[2] = {0, 3}, face_vi[3] = {1, 2, 3};
    pbt_outbeam ob[2] = {{{0}}};
    double amp[8] = {0.8, 0.1, 0.05, -0.02, 0.03, 0.01, 0.7, -0.2};
    for (int q = 0; q < 8; q++) ob[0].ampl[q] = ob[1].ampl[q] = amp[q];
    double p0[3] = {0.2, -0.1, -0.97}, n = sqrt(0.04 + 0.01 + 0.97 * 0.97);
    for (int c = 0; c < 3; c++) ob[0].prop_out[c] = p0[c] / n;
    ob[0].vk7[1] = 1.0;
    ob[0].vk7[2] = ob[0].prop_out[1] != 0 ? -ob[0].prop_out[1] / ob[0].prop_out[2] : 0.0;
    n = sqrt(ob[0].vk7[1] * ob[0].vk7[1] + ob[0].vk7[2] * ob[0].vk7[2]);
    ob[0].vk7[1] /= n;
    ob[0].vk7[2] /= n;
    ob[0].fov = 0.3;
    ob[0].fi = 1;
    ob[1].prop_out[2] = -1.0;
    ob[1].vk7[1] = 1.0;
    ob[1].fov = pi / 2;
    ob[1].fi = 1;
    const size_t ng = (size_t)8 * NT * NP;
    double *afb = malloc(ng * sizeof(double)), *afe = malloc(ng * sizeof(double));
    double *gfb = malloc(ng * sizeof(double)), *gfe = malloc(ng * sizeof(double));
    double *mu = malloc((size_t)16 * NT * NP * sizeof(double)), *mu1 = malloc(16 * NT * sizeof(double));
    pbt_ctx *ctx = NULL;
    CHECK(pbt_ctx_create(0, &ctx));
    CHECK(pbt_diff_main_c(ctx, &ob[0], 1, &ob[1], 1, v, 3, face_off, face_vi, 1, theta, NT, phi, NP,
                          0.532, 0, PBT_PREC_FP64, afb, afe));
    CHECK(pbt_diff_main_c(ctx, &ob[0], 1, &ob[1], 1, v, 3, face_off, face_vi, 1, theta, NT, phi, NP,
                          0.532, 0, PBT_PREC_FP32, gfb, gfe));
    double dmax = 0, amax = 0;
    for (size_t q = 0; q < ng; q++) {
        double d = fabs(gfb[q] + gfe[q] - afb[q] - afe[q]), a = fabs(afb[q] + afe[q]);
        if (d > dmax) dmax = d;
        if (a > amax) amax = a;
    }
    pbt_output_params p = {0};
    p.geo_cross_sec = 0.7;
    CHECK(pbt_finalise_c(ctx, afb, afe, theta, NT, phi, NP, 0.532, 0, &p, mu, mu1, 0));
    /* a bad face index is reported, not trapped */
    ob[0].fi = 5;
    int s = pbt_diff_main_c(ctx, &ob[0], 1, &ob[1], 1, v, 3, face_off, face_vi, 1, theta, NT, phi, NP,
                            0.532, 0, PBT_PREC_FP64, afb, afe);
    if (s != PBT_EINVAL) {
        fprintf(stderr, "expected PBT_EINVAL, got %d\n", s);
        return 1;
    }
    CHECK(pbt_ctx_destroy(ctx));
    printf("ok %.3e %.9f %.9f\n", dmax / amax, p.scatt, p.asymmetry);
    free(afb); free(afe); free(gfb); free(gfe); free(mu); free(mu1);
    return dmax / amax < 1e-4 ? 0 : 2;
}
