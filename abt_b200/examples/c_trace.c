/* c_trace.c -- the near-field tracer through the C ABI (host only, no GPU).
 *
 * Builds a smooth hexagonal prism (radius 5 um, length 10 um) of 24 triangles
 * (each rectangular side split in two, each hexagonal end a fan of 6) with its
 * 8 parent faces as apertures, traces one orientation at n = 1.31,
 * lambda = 0.532 um with the reference's default limits, and checks the
 * energy record: the external-diffraction energy equals the illuminated
 * geometric cross section.  (The beam energy falls well short of it on a mesh
 * this coarse: the reference's visibility test lights whole triangles by
 * their centroids, so it wants facets small against the particle.)  Prints
 * "ok <beam outbeams> <external outbeams> <beam energy / geo>".
 *
 *   gcc -std=c99 -I include abt_b200/examples/c_trace.c -L abt_b200 -lpbt_b200 \
 *       -Wl,-rpath,abt_b200 -lm
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "pbt_diff.h"

int main(void) {
    enum { NV = 14, NF = 24 };
    double v[NV * 3]; /* v(NV,3) column-major, as geometry%v */
    const double r = 5.0, h = 5.0, pi = 3.14159265358979323846;
    for (int k = 0; k < 6; k++) {
        const double a = k * pi / 3;
        v[k] = v[6 + k] = r * cos(a);
        v[NV + k] = v[NV + 6 + k] = r * sin(a);
        v[2 * NV + k] = h;      /* top ring: vertices 1..6 */
        v[2 * NV + 6 + k] = -h; /* bottom ring: 7..12 */
    }
    v[12] = v[NV + 12] = 0.0, v[2 * NV + 12] = h;  /* top centre: 13 */
    v[13] = v[NV + 13] = 0.0, v[2 * NV + 13] = -h; /* bottom centre: 14 */
    int64_t off[NF + 1], vi[3 * NF], ap[NF];
    int f = 0;
    for (int k = 0; k < 6; k++) { /* sides, counter-clockwise seen from outside */
        const int64_t a = k + 1, b = (k + 1) % 6 + 1;
        const int64_t tri[2][3] = {{a + 6, b + 6, b}, {a + 6, b, a}};
        for (int t = 0; t < 2; t++, f++) {
            for (int q = 0; q < 3; q++) vi[3 * f + q] = tri[t][q];
            ap[f] = k + 1;
        }
    }
    for (int k = 0; k < 6; k++, f++) { /* top fan */
        vi[3 * f] = 13, vi[3 * f + 1] = k + 1, vi[3 * f + 2] = (k + 1) % 6 + 1;
        ap[f] = 7;
    }
    for (int k = 0; k < 6; k++, f++) { /* bottom fan */
        vi[3 * f] = 14, vi[3 * f + 1] = (k + 1) % 6 + 7, vi[3 * f + 2] = k + 7;
        ap[f] = 8;
    }
    for (int i = 0; i <= NF; i++) off[i] = 3 * i;

    pbt_particle *p = NULL;
    if (pbt_particle_create(v, NV, off, vi, NF, ap, &p) != PBT_OK) {
        printf("particle: %s\n", pbt_last_error_string());
        return 1;
    }
    const double euler[3] = {0.4, 0.9, 1.3};
    pbt_trace_params prm = {0.532, 1.31, 0.0, 8, 10, 0.1, 1e-4};
    pbt_trace *t = NULL;
    if (pbt_trace_orientation_c(p, euler, &prm, &t) != PBT_OK) {
        printf("trace: %s\n", pbt_last_error_string());
        return 1;
    }
    int64_t nbeam = 0, next = 0;
    pbt_trace_sizes(t, &nbeam, &next);
    pbt_outbeam *beam = malloc(sizeof(pbt_outbeam) * (nbeam ? nbeam : 1));
    pbt_outbeam *ext = malloc(sizeof(pbt_outbeam) * (next ? next : 1));
    double rv[NV * 3];
    pbt_trace_energy e;
    pbt_trace_copy(t, beam, ext, rv, &e);
    int ok = nbeam > 0 && next > 0;
    ok = ok && fabs(e.ext_energy_out / e.geo_cross_sec - 1.0) < 1e-12;
    ok = ok && e.beam_energy_out > 0.0 && e.beam_energy_out < 1.05 * e.geo_cross_sec;
    for (int64_t i = 0; i < nbeam && ok; i++) ok = beam[i].fi >= 1 && beam[i].fi <= NF;
    /* a bad argument is a status and a message, not a crash */
    prm.rbi = 0.5;
    pbt_trace *bad = NULL;
    ok = ok && pbt_trace_orientation_c(p, euler, &prm, &bad) == PBT_EINVAL && bad == NULL;
    pbt_trace_destroy(t);
    pbt_particle_destroy(p);
    free(beam);
    free(ext);
    if (!ok) {
        printf("fail %lld %lld %.6f\n", (long long)nbeam, (long long)next,
               e.beam_energy_out / e.geo_cross_sec);
        return 1;
    }
    printf("ok %lld %lld %.17g\n", (long long)nbeam, (long long)next,
           e.beam_energy_out / e.geo_cross_sec);
    return 0;
}
