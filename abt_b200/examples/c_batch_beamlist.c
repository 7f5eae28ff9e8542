/* c_batch_beamlist.c -- a C host program that dumps per-orientation outbeam
 * lists to a beam-list file, reads them back and averages the orientations
 * with pbt_diff_batch_c (FP64 drop-in and FP32 batch).
 *
 * The particle is one triangle, rotated about z for each orientation; each
 * orientation has one outgoing beam and one external-diffraction outbeam.
 * Without a CUDA device the file and far-field-bin steps still run and the
 * program prints "ok-nodevice".  With a device it prints
 * "ok <Mueller M11 rel diff fp32/fp64> <scatt>".
 *
 *   gcc -O2 -std=c99 -I include c_batch_beamlist.c -L abt_b200 -lpbt_b200 \
 *       -Wl,-rpath,abt_b200 -lm
 *   ./a.out /tmp/orient.pbtb
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "pbt_diff.h"

#define CHECK(call)                                                                  \
    do {                                                                             \
        int s_ = (call);                                                             \
        if (s_ != PBT_OK) {                                                          \
            fprintf(stderr, "%s -> %d: %s\n", #call, s_, pbt_last_error_string());   \
            return 1;                                                                \
        }                                                                            \
    } while (0)

enum { NO = 3, NT = 46, NP = 45 };

int main(int argc, char **argv) {
    const char *path = argc > 1 ? argv[1] : "orient.pbtb";
    const double pi = (double)3.14159265358979f;
    double theta[NT], phi[NP];
    for (int i = 0; i < NT; i++) theta[i] = (4.0 * i) * pi / 180.0;
    for (int i = 0; i < NP; i++) phi[i] = (8.0 * i) * pi / 180.0;
    const double v0[3][3] = {{0.1, 0.2, 0.0}, {1.3, 0.3, 0.1}, {0.2, 1.4, -0.1}};
    int64_t face_off[2] = {0, 3}, face_vi[3] = {1, 2, 3};

    /* far-field bins, as the tracer's make_far_field_bins would give them */
    double *xf = malloc(sizeof(double) * NT * NP), *yf = malloc(sizeof(double) * NT * NP),
           *zf = malloc(sizeof(double) * NT * NP);
    CHECK(pbt_make_far_field_bins_c(theta, NT, phi, NP, xf, yf, zf));
    if (fabs(zf[0] + 1e6) > 1e-6 || fabs(xf[NP] - 1e6 * sin(theta[1])) > 1e-3) {
        fprintf(stderr, "unexpected far-field bins\n");
        return 1;
    }

    /* dump: one call per orientation, as beside diff_main in the tracer's loop */
    pbt_beamlist_writer *w = NULL;
    CHECK(pbt_beamlist_writer_open(path, theta, NT, phi, NP, 3, face_off, face_vi, 1, 0.532, &w));
    for (int o = 0; o < NO; o++) {
        const double a = 0.7 * o, c = cos(a), s = sin(a);
        double v[9];  /* v(3,3) column-major */
        for (int j = 0; j < 3; j++) {
            v[j] = c * v0[j][0] - s * v0[j][1];
            v[3 + j] = s * v0[j][0] + c * v0[j][1];
            v[6 + j] = v0[j][2];
        }
        pbt_outbeam ob[2];
        memset(ob, 0, sizeof(ob));
        const double amp[8] = {0.8, 0.1, 0.05, -0.02, 0.03, 0.01, 0.7, -0.2};
        for (int q = 0; q < 8; q++) ob[0].ampl[q] = amp[q];
        ob[0].prop_out[0] = 0.3 * c;
        ob[0].prop_out[1] = 0.3 * s;
        ob[0].prop_out[2] = -sqrt(1.0 - 0.09);
        ob[0].vk7[0] = -s;
        ob[0].vk7[1] = c;
        ob[0].fov = 0.4;
        ob[0].fi = 1;
        ob[1].ampl[0] = ob[1].ampl[6] = 1.0;
        ob[1].prop_out[2] = -1.0;
        ob[1].vk7[1] = 1.0;
        ob[1].fov = pi / 2;
        ob[1].fi = 1;
        pbt_output_params p;
        memset(&p, 0, sizeof(p));
        p.geo_cross_sec = 0.7;
        p.beam_energy_out = p.ext_energy_out = 1.0;
        CHECK(pbt_beamlist_writer_add(w, &ob[0], 1, &ob[1], 1, v, &p));
    }
    CHECK(pbt_beamlist_writer_close(w));

    /* replay */
    pbt_beamlist *bl = NULL;
    CHECK(pbt_beamlist_read(path, &bl));
    int64_t cnt[8];
    double lam;
    CHECK(pbt_beamlist_info(bl, cnt, &lam));
    if (cnt[0] != NO || cnt[4] != NT || cnt[5] != NP || cnt[6] != NO || cnt[7] != NO) {
        fprintf(stderr, "unexpected counts\n");
        return 1;
    }
    const double *th, *ph, *verts;
    const int64_t *fo, *fv, *boff, *eoff;
    const pbt_outbeam *beam, *ext;
    const pbt_output_params *pin;
    CHECK(pbt_beamlist_arrays(bl, &th, &ph, &fo, &fv, &verts, &boff, &beam, &eoff, &ext, &pin));

    pbt_ctx *ctx = NULL;
    if (pbt_ctx_create(0, &ctx) == PBT_ENODEV) {
        printf("ok-nodevice\n");
        pbt_beamlist_free(bl);
        return 0;
    }
    const size_t nm = (size_t)16 * NT * NP;
    double *mu64 = malloc(nm * sizeof(double)), *mu32 = malloc(nm * sizeof(double));
    double *m164 = malloc(16 * NT * sizeof(double)), *m132 = malloc(16 * NT * sizeof(double));
    pbt_output_params pa64, pa32;
    CHECK(pbt_diff_batch_c(ctx, cnt[0], beam, boff, ext, eoff, verts, cnt[1], fo, fv, cnt[2], th,
                           cnt[4], ph, cnt[5], lam, 0, 0, PBT_PREC_FP64, pin, mu64, m164, &pa64,
                           NULL));
    CHECK(pbt_diff_batch_c(ctx, cnt[0], beam, boff, ext, eoff, verts, cnt[1], fo, fv, cnt[2], th,
                           cnt[4], ph, cnt[5], lam, 0, 0, PBT_PREC_FP32, pin, mu32, m132, &pa32,
                           NULL));
    double dmax = 0, amax = 0;
    for (size_t q = 0; q < (size_t)NT * NP; q++) { /* M11: the first (nphi,ntheta) block */
        const double d = fabs(mu32[q] - mu64[q]);
        if (d > dmax) dmax = d;
        if (mu64[q] > amax) amax = mu64[q];
    }
    CHECK(pbt_ctx_destroy(ctx));
    pbt_beamlist_free(bl);
    printf("ok %.3e %.9f\n", dmax / amax, pa64.scatt);
    free(xf); free(yf); free(zf); free(mu64); free(mu32); free(m164); free(m132);
    return dmax / amax < 1e-4 ? 0 : 2;
}
