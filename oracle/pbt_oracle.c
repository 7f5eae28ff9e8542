/*
 * pbt_oracle.c -- CPU FP64 restatement of PBT's far-field diffraction stage.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: it is built and
 * called by tests/, by __graft_entry__.smoke() as the checker, and by bench.py's
 * CPU-baseline leg.  The product library (abt_b200/) never links or calls it.
 *
 * PARITY UNPINNED: the reference (Fortran, gfortran + libm) cannot be compiled
 * or run on this machine (no Fortran front end) and the reference ships no
 * golden far-field vectors, so this restatement is checked only against
 * closed-form known answers (tests/test_oracle_known_answers.py) and frozen
 * fixtures generated from it (tests/golden/).
 *
 * Every routine follows the reference operation by operation, in Fortran's
 * left-to-right evaluation order, without FMA contraction (build with
 * -ffp-contract=off), with the reference's single-precision literals widened
 * exactly as gfortran widens them:
 *
 *   pi      = 3.14159265358979 (a default-real literal)  src/misc_submod.f90:12
 *   0.999999, 1e-6, 0.999, 0.0001 are float literals       src/diff_mod.f90:151,364,630,563
 *
 * Citations are path:line inside the reference project.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* src/misc_submod.f90:12 -- a default-real (float) literal widened to real(8) */
#define PI_REF ((double)3.14159265358979f)
#define LIT_0_999999 ((double)0.999999f) /* src/diff_mod.f90:151 */
#define LIT_1EM6 ((double)1e-6f)         /* src/diff_mod.f90:364-365 */
#define LIT_0_999 ((double)0.999f)       /* src/diff_mod.f90:630 */
#define LIT_0_0001 ((double)0.0001f)     /* src/diff_mod.f90:563 */
#define FAR_R ((double)1e6f)             /* src/diff_mod.f90:848 */

typedef struct { double re, im; } zc;

/* Same memory layout as the library's pbt_outbeam record (128 bytes):
 * the fields of outbeamtype (src/types_mod.f90:8-17) that diffraction reads. */
typedef struct {
    double ampl[8];  /* ampl(1:2,1:2) complex(8), column-major: (1,1),(2,1),(1,2),(2,2); re,im */
    double vk7[3];
    double prop_out[3];
    double fov;
    int64_t fi;      /* 1-based face index */
} or_outbeam;

/* output_parameters_type, src/types_mod.f90:32-53, same component order */
typedef struct {
    double abs_, scatt, ext, albedo, asymmetry, abs_eff, scatt_eff, ext_eff,
        geo_cross_sec, back_scatt, beam_energy_out, ext_energy_out, scatt_beam,
        scatt_ext_diff, asymmetry_beam, asymmetry_ext_diff, scatt_eff_beam,
        scatt_eff_ext_diff;
} or_params;

static inline zc zmul(zc a, zc b) { zc r; r.re = a.re * b.re - a.im * b.im; r.im = a.re * b.im + a.im * b.re; return r; }
static inline zc zadd(zc a, zc b) { zc r; r.re = a.re + b.re; r.im = a.im + b.im; return r; }
static inline zc zscale(zc a, double s) { zc r; r.re = a.re * s; r.im = a.im * s; return r; }

/* matmul of 3x3 by 3x3: c(i,j) = sum_k a(i,k)*b(k,j), k in order, from 0 */
static void mm33(const double a[3][3], const double b[3][3], double c[3][3]) {
    double t[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double s = 0.0;
            s = s + a[i][0] * b[0][j];
            s = s + a[i][1] * b[1][j];
            s = s + a[i][2] * b[2][j];
            t[i][j] = s;
        }
    memcpy(c, t, sizeof t);
}
static void mv33(const double a[3][3], const double x[3], double y[3]) {
    double t[3];
    for (int i = 0; i < 3; i++) {
        double s = 0.0;
        s = s + a[i][0] * x[0];
        s = s + a[i][1] * x[1];
        s = s + a[i][2] * x[2];
        t[i] = s;
    }
    y[0] = t[0]; y[1] = t[1]; y[2] = t[2];
}
static inline double dot3(const double a[3], const double b[3]) {
    double s = 0.0;
    s = s + a[0] * b[0];
    s = s + a[1] * b[1];
    s = s + a[2] * b[2];
    return s;
}
/* cross, src/misc_submod.f90:2367-2390 (normalises unless told otherwise) */
static void cross3(const double a[3], const double b[3], double c[3], int normalise) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
    double nf = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
    if (!normalise) nf = 1;
    c[0] = c[0] / nf; c[1] = c[1] / nf; c[2] = c[2] / nf;
}

/* ------------------------------------------------------------------ angles */

/* make_angles, src/input_mod.f90:114-196.  vals_in/splits_in in degrees;
 * returns the number of angles written (degrees), or -1 on a bad split. */
int64_t oracle_make_angles(const double *vals_in, const double *splits_in,
                           int64_t counter, double *out, int64_t cap) {
    int64_t kint = 0;
    for (int64_t i = 0; i < counter - 1; i++) {
        double q = (vals_in[i + 1] - vals_in[i]) / splits_in[i];
        int64_t jmax = llround(q);
        double fr = fmod(q, 1.0);
        if (fr > (double)1e-3f && fr < (double)(1.0f - 1e-3f)) return -1;
        for (int64_t j = 0; j <= jmax; j++) {
            if (i != counter - 2 && j == jmax) continue;
            if (kint >= cap) return -2;
            out[kint++] = vals_in[i] + (double)j * splits_in[i];
        }
    }
    return kint;
}

/* theta_vals*pi/180d0, src/input_mod.f90:742,789 */
void oracle_deg_to_rad(double *a, int64_t n) {
    for (int64_t i = 0; i < n; i++) a[i] = a[i] * PI_REF / 180.0;
}

/* make_far_field_bins + meshgrid_real, src/diff_mod.f90:827-855,
 * src/misc_submod.f90:1743-1779.  Arrays are (nphi, ntheta), column-major. */
void oracle_make_far_field_bins(const double *theta, int64_t ntheta,
                                const double *phi, int64_t nphi,
                                double *x, double *y, double *z) {
    double r = FAR_R;
    for (int64_t j = 0; j < ntheta; j++)
        for (int64_t i = 0; i < nphi; i++) {
            int64_t o = i + nphi * j;
            x[o] = r * sin(theta[j]) * cos(phi[i]);
            y[o] = r * sin(theta[j]) * sin(phi[i]);
            z[o] = -(r * cos(theta[j]));
        }
}

/* --------------------------------------------------------------- diff_mod */

/* get_rotation_matrix2, src/diff_mod.f90:200-289 */
static void get_rotation_matrix2(const double *v0x, const double *v0y,
                                 const double *v0z, double rot[3][3]) {
    double a1[3] = {v0x[0], v0y[0], v0z[0]};
    double b1[3] = {v0x[1], v0y[1], v0z[1]};
    double t1 = atan(a1[0] / a1[1]);
    double rot1[3][3] = {{cos(t1), -sin(t1), 0}, {sin(t1), cos(t1), 0}, {0, 0, 1}};
    double a2[3], b2[3];
    mv33(rot1, a1, a2);
    mv33(rot1, b1, b2);
    double t2 = -atan(a2[2] / a2[1]);
    double rot2[3][3] = {{1, 0, 0}, {0, cos(t2), -sin(t2)}, {0, sin(t2), cos(t2)}};
    double a3[3], b3[3];
    mv33(rot2, a2, a3);
    mv33(rot2, b2, b3);
    double t3 = atan(b3[2] / b3[0]);
    double rot3[3][3] = {{cos(t3), 0, sin(t3)}, {0, 1, 0}, {-sin(t3), 0, cos(t3)}};
    double a4[3], b4[3];
    mv33(rot3, a3, a4);
    mv33(rot3, b3, b4);
    double r21[3][3], r321[3][3];
    mm33(rot2, rot1, r21);
    mm33(rot3, r21, r321);
    if (a4[0] * b4[1] - a4[1] * b4[0] > 0) {
        double rot4[3][3] = {{-1, 0, 0}, {0, 1, 0}, {0, 0, -1}};
        mm33(rot4, r321, rot);
    } else {
        memcpy(rot, r321, sizeof r321);
    }
}

/* karczewski, src/diff_mod.f90:124-198 */
static void karczewski(double D[2][2], double m[3], double k[3], const double prop2[3],
                       double x3, double y3, double z3, double r) {
    double bvs = r;
    k[0] = x3 / bvs;
    k[1] = y3 / bvs;
    k[2] = z3 / bvs;
    if (fabs(k[1]) > LIT_0_999999) k[1] = copysign(LIT_0_999999, k[1]);
    double Kx = prop2[0], Ky = prop2[1], Kz = prop2[2];
    m[0] = -(k[0] * k[1] / sqrt(1 - k[1] * k[1]));
    m[1] = sqrt(1 - k[1] * k[1]);
    m[2] = -(k[1] * k[2] / sqrt(1 - k[1] * k[1]));
    double frac = sqrt((1 - k[1] * k[1]) / (1 - Ky * Ky));
    double a1m = -Kz * frac;
    double b2m = -k[2] / frac;
    double a1e = b2m;
    double b2e = a1m;
    double b1m = -(k[0] * k[1] / frac) + Kx * Ky * frac;
    double a2e = -b1m;
    D[0][0] = 0.5 * (a1m + a1e);
    D[0][1] = 0.5 * b1m;
    D[1][0] = 0.5 * a2e;
    D[1][1] = 0.5 * (b2m + b2e);
}

typedef struct {
    int64_t nphi, ntheta;
    const double *theta, *phi;
    const double *xfar, *yfar, *zfar;
    double lambda;
    int is_fast_diff;
} or_grid;

typedef struct {
    int64_t nverts;
    const double *v;          /* v(nverts,3) column-major */
    const int64_t *face_off;  /* nfaces+1 */
    const int64_t *face_vi;   /* 1-based */
    int64_t nfaces;
} or_geom;

/* diffraction + contour_integral, src/diff_mod.f90:446-672 and :291-444.
 * amplC is (nphi, ntheta, 2, 2) complex, fully overwritten.  fov_override
 * replaces outbeam%fov when >= 0 (diff_main sets pi/2 for external
 * diffraction, src/diff_mod.f90:797).  Returns 0 or a negative error code. */
int oracle_diffraction(const or_grid *g, const or_geom *geo, const or_outbeam *ob,
                       double fov_override, zc *amplC) {
    const int64_t nphi = g->nphi, nth = g->ntheta, nb = nphi * nth;
    if (ob->fi < 1 || ob->fi > geo->nfaces) return -3;
    int64_t f = ob->fi - 1;
    int64_t v_beg = geo->face_off[f], nv = geo->face_off[f + 1] - geo->face_off[f];
    if (nv < 3) return -4;

    zc ampl[2][2];
    ampl[0][0].re = ob->ampl[0]; ampl[0][0].im = ob->ampl[1];
    ampl[1][0].re = ob->ampl[2]; ampl[1][0].im = ob->ampl[3];
    ampl[0][1].re = ob->ampl[4]; ampl[0][1].im = ob->ampl[5];
    ampl[1][1].re = ob->ampl[6]; ampl[1][1].im = ob->ampl[7];
    double perp0[3] = {ob->vk7[0], ob->vk7[1], ob->vk7[2]};
    double prop0[3] = {ob->prop_out[0], ob->prop_out[1], ob->prop_out[2]};
    double fov = fov_override >= 0 ? fov_override : ob->fov;
    for (int64_t q = 0; q < 4 * nb; q++) { amplC[q].re = 0; amplC[q].im = 0; }
    double cos_fov = cos(fov);

    double *v2x = malloc(sizeof(double) * 6 * nv);
    double *v2y = v2x + nv, *v2z = v2x + 2 * nv;
    double *v20x = v2x + 3 * nv, *v20y = v2x + 4 * nv, *v20z = v2x + 5 * nv;
    for (int64_t i = 0; i < nv; i++) {
        int64_t vi = geo->face_vi[v_beg + i] - 1;
        v2x[i] = geo->v[vi];
        v2y[i] = geo->v[vi + geo->nverts];
        v2z[i] = geo->v[vi + 2 * geo->nverts];
    }
    double com[3] = {0, 0, 0};
    for (int64_t i = 0; i < nv; i++) { com[0] = com[0] + v2x[i]; com[1] = com[1] + v2y[i]; com[2] = com[2] + v2z[i]; }
    com[0] = com[0] / (double)nv; com[1] = com[1] / (double)nv; com[2] = com[2] / (double)nv;
    for (int64_t i = 0; i < nv; i++) {
        v20x[i] = v2x[i] - com[0]; v20y[i] = v2y[i] - com[1]; v20z[i] = v2z[i] - com[2];
    }
    double rot[3][3];
    get_rotation_matrix2(v20x, v20y, v20z, rot);
    double prop1[3], perp1[3];
    mv33(rot, prop0, prop1);
    mv33(rot, perp0, perp1);
    double angle = -atan2(prop1[1], prop1[0]);
    double rot2[3][3] = {{cos(angle), -sin(angle), 0}, {sin(angle), cos(angle), 0}, {0, 0, 1}};
    double prop2[3], perp2[3], e_par2[3];
    mv33(rot2, prop1, prop2);
    mv33(rot2, perp1, perp2);
    cross3(perp2, prop2, e_par2, 1);
    if (e_par2[2] > LIT_0_0001) {
        for (int a = 0; a < 2; a++)
            for (int b = 0; b < 2; b++) { ampl[a][b].re = -ampl[a][b].re; ampl[a][b].im = -ampl[a][b].im; }
    }
    double incidence[3] = {0, 0, -1}, tmp3[3], incidence2[3];
    mv33(rot, incidence, tmp3);
    mv33(rot2, tmp3, incidence2);

    /* theta_i: first theta above 1 degree, src/diff_mod.f90:583-591 */
    int64_t theta_i = -1;
    for (int64_t i = 0; i < nth; i++)
        if (g->theta[i] > 1 * PI_REF / 180) { theta_i = i; break; }
    if (theta_i < 0) { free(v2x); return -5; }

    double *x1 = malloc(sizeof(double) * 7 * nb);
    double *y1 = x1 + nb, *z1 = x1 + 2 * nb, *r1 = x1 + 3 * nb;
    double *x3 = x1 + 4 * nb, *y3 = x1 + 5 * nb, *z3 = x1 + 6 * nb;
    unsigned char *in_fov = malloc(nb);
    zc *area = malloc(sizeof(zc) * nb);
    for (int64_t o = 0; o < nb; o++) {
        x1[o] = g->xfar[o] - com[0];
        y1[o] = g->yfar[o] - com[1];
        z1[o] = g->zfar[o] - com[2];
        r1[o] = sqrt(x1[o] * x1[o] + y1[o] * y1[o] + z1[o] * z1[o]);
        in_fov[o] = 1;
    }
    if (g->is_fast_diff) {
        for (int64_t o = 0; o < nb; o++) {
            double vec[3] = {x1[o] / r1[o], y1[o] / r1[o], z1[o] / r1[o]};
            if (dot3(vec, prop0) < cos_fov) in_fov[o] = 0;
        }
    }
    double R[3][3];
    mm33(rot2, rot, R);
    /* rotate_far_field_bins, src/diff_mod.f90:86-122 (masked bins + the theta_i row) */
    for (int64_t j = 0; j < nth; j++)
        for (int64_t i = 0; i < nphi; i++) {
            int64_t o = i + nphi * j;
            if (!in_fov[o] && j != theta_i) continue;
            x3[o] = R[0][0] * x1[o] + R[0][1] * y1[o] + R[0][2] * z1[o];
            y3[o] = R[1][0] * x1[o] + R[1][1] * y1[o] + R[1][2] * z1[o];
            z3[o] = R[2][0] * x1[o] + R[2][1] * y1[o] + R[2][2] * z1[o];
        }

    /* per-bin polarisation, src/diff_mod.f90:620-660 */
    for (int64_t j = 0; j < nth; j++)
        for (int64_t i = 0; i < nphi; i++) {
            int64_t o = i + nphi * j;
            if (!in_fov[o]) continue;
            double phi = g->phi[i];
            double D[2][2], m[3], k[3], hc[3], evo2[3];
            karczewski(D, m, k, prop2, x3[o], y3[o], z3[o], r1[o]);
            if (fabs(dot3(incidence2, k)) < LIT_0_999) {
                cross3(incidence2, k, hc, 1);
            } else {
                int64_t oi = i + nphi * theta_i;
                double my_k[3] = {x3[oi] / r1[oi], y3[oi] / r1[oi], z3[oi] / r1[oi]};
                cross3(incidence2, my_k, hc, 1);
            }
            cross3(k, m, evo2, 1);
            double rot4[2][2];
            rot4[0][0] = dot3(hc, m);
            rot4[1][1] = dot3(hc, m);
            rot4[0][1] = -dot3(hc, evo2);
            rot4[1][0] = +dot3(hc, evo2);
            /* getRotationMatrix, src/diff_mod.f90:14-37, then transposed (:650) */
            double tv[3] = {cos(phi), sin(phi), 0.0};
            double vk71 = -tv[1], vk72 = tv[0], vk73 = 0.0;
            double ev11 = 1, ev12 = 0, ev13 = 0, ev31 = 0, ev32 = 0, ev33 = -1;
            double mfa = vk71 * ev11 + vk72 * ev12 + vk73 * ev13;
            double evo21 = ev32 * ev13 - ev33 * ev12;
            double evo22 = ev33 * ev11 - ev31 * ev13;
            double evo23 = ev31 * ev12 - ev32 * ev11;
            double tr[2][2];
            tr[0][0] = mfa;
            tr[0][1] = -(vk71 * evo21 + vk72 * evo22 + vk73 * evo23);
            tr[1][0] = +(vk71 * evo21 + vk72 * evo22 + vk73 * evo23);
            tr[1][1] = mfa;
            double T[2][2] = {{tr[0][0], tr[1][0]}, {tr[0][1], tr[1][1]}};
            /* ampl_temp2 = rot4 . (diff_ampl . (ampl . T)) */
            zc P[2][2], Q[2][2], Rz[2][2];
            for (int a = 0; a < 2; a++)
                for (int b = 0; b < 2; b++) {
                    zc s = {0, 0};
                    s = zadd(s, zscale(ampl[a][0], T[0][b]));
                    s = zadd(s, zscale(ampl[a][1], T[1][b]));
                    P[a][b] = s;
                }
            for (int a = 0; a < 2; a++)
                for (int b = 0; b < 2; b++) {
                    zc s = {0, 0};
                    s = zadd(s, zscale(P[0][b], D[a][0]));
                    s = zadd(s, zscale(P[1][b], D[a][1]));
                    Q[a][b] = s;
                }
            for (int a = 0; a < 2; a++)
                for (int b = 0; b < 2; b++) {
                    zc s = {0, 0};
                    s = zadd(s, zscale(Q[0][b], rot4[a][0]));
                    s = zadd(s, zscale(Q[1][b], rot4[a][1]));
                    Rz[a][b] = s;
                }
            for (int a = 0; a < 2; a++)
                for (int b = 0; b < 2; b++) amplC[o + nb * (a + 2 * b)] = Rz[a][b];
        }

    /* contour_integral, src/diff_mod.f90:291-444 */
    {
        double waveno = 2.0 * PI_REF / g->lambda;
        double Rc[3][3];
        mm33(rot2, rot, Rc);
        double *xv = malloc(sizeof(double) * 4 * nv), *yv = xv + nv, *mv = xv + 2 * nv, *nvv = xv + 3 * nv;
        for (int64_t jv = 0; jv < nv; jv++) {
            double c[3] = {v20x[jv], v20y[jv], v20z[jv]}, r[3];
            mv33(Rc, c, r);
            xv[jv] = r[0]; yv[jv] = r[1];
        }
        double kinc[3] = {prop2[0] * waveno, prop2[1] * waveno, prop2[2] * waveno};
        for (int64_t jv = 0; jv < nv; jv++) {
            int64_t jn = (jv == nv - 1) ? 0 : jv + 1;
            mv[jv] = (yv[jn] - yv[jv]) / (xv[jn] - xv[jv]);
        }
        for (int64_t jv = 0; jv < nv; jv++) nvv[jv] = 1 / mv[jv];
        double *bvs = malloc(sizeof(double) * 3 * nb), *kxxs = bvs + nb, *kyys = bvs + 2 * nb;
        for (int64_t o = 0; o < nb; o++) { area[o].re = 0; area[o].im = 0; }
        for (int64_t o = 0; o < nb; o++) {
            if (!in_fov[o]) continue;
            bvs[o] = waveno * sqrt(x3[o] * x3[o] + y3[o] * y3[o] + z3[o] * z3[o]);
            kxxs[o] = kinc[0] - waveno * waveno * x3[o] / bvs[o];
            kyys[o] = kinc[1] - waveno * waveno * y3[o] / bvs[o];
            if (fabs(kxxs[o]) < LIT_1EM6) kxxs[o] = LIT_1EM6;
            if (fabs(kyys[o]) < LIT_1EM6) kyys[o] = LIT_1EM6;
        }
        for (int64_t jv = 0; jv < nv; jv++) {
            double mj = mv[jv], nj = nvv[jv], xj = xv[jv], yj = yv[jv];
            if (fabs(mj) > DBL_MAX) mj = 1e6;
            if (fabs(nj) > DBL_MAX) nj = 1e6;
            if (fabs(mj) < 1e-9) nj = 1e6;
            if (fabs(nj) < 1e-9) mj = 1e6;
            int64_t jn = (jv == nv - 1) ? 0 : jv + 1;
            double dx = xv[jn] - xj, dy = yv[jn] - yj;
            for (int64_t o = 0; o < nb; o++) {
                if (!in_fov[o]) continue;
                double K = bvs[o], kxx = kxxs[o], kyy = kyys[o];
                double delta = kxx * xj + kyy * yj;
                double delta1 = kyy * mj + kxx;
                double delta2 = kxx * nj + kyy;
                double omega1 = dx * delta1;
                double omega2 = dy * delta2;
                double alpha = 1 / (2 * kyy * delta1);
                double beta = 1 / (2 * kxx * delta2);
                double sumim = alpha * (cos(delta) - cos(delta + omega1)) - beta * (cos(delta) - cos(delta + omega2));
                double sumre = -(alpha * (sin(delta) - sin(delta + omega1))) + beta * (sin(delta) - sin(delta + omega2));
                zc e = {cos(K), sin(K)}, s = {sumre, sumim};
                zc t = zmul(e, s);
                t.re = t.re / g->lambda;
                t.im = t.im / g->lambda;
                area[o] = zadd(area[o], t);
            }
        }
        free(bvs);
        free(xv);
    }
    /* amplC(i,j,:,:) = amplC(i,j,:,:) * area_facs2(i,j), src/diff_mod.f90:665-670 */
    for (int64_t o = 0; o < nb; o++) {
        if (!in_fov[o]) continue;
        for (int q = 0; q < 4; q++) amplC[o + nb * q] = zmul(amplC[o + nb * q], area[o]);
    }
    free(area);
    free(in_fov);
    free(x1);
    free(v2x);
    return 0;
}

/* diff_main, src/diff_mod.f90:674-825.  Sequential facet order (the
 * reference's -mt 0 order).  Outputs are (nphi, ntheta, 2, 2) complex. */
int oracle_diff_main(const or_grid *g, const or_geom *geo,
                     const or_outbeam *beam, int64_t nbeam,
                     const or_outbeam *ext, int64_t next,
                     zc *ampl_far_beam, zc *ampl_far_ext_diff) {
    const int64_t n4 = 4 * g->nphi * g->ntheta;
    zc *amplC = malloc(sizeof(zc) * n4);
    int rc = 0;
    for (int64_t q = 0; q < n4; q++) { ampl_far_beam[q].re = 0; ampl_far_beam[q].im = 0; ampl_far_ext_diff[q] = ampl_far_beam[q]; }
    for (int64_t jb = 0; jb < nbeam && !rc; jb++) {
        rc = oracle_diffraction(g, geo, &beam[jb], -1.0, amplC);
        if (!rc) for (int64_t q = 0; q < n4; q++) ampl_far_beam[q] = zadd(ampl_far_beam[q], amplC[q]);
    }
    for (int64_t jb = 0; jb < next && !rc; jb++) {
        rc = oracle_diffraction(g, geo, &ext[jb], PI_REF / 2.0, amplC);
        if (!rc) for (int64_t q = 0; q < n4; q++) ampl_far_ext_diff[q] = zadd(ampl_far_ext_diff[q], amplC[q]);
    }
    free(amplC);
    return rc;
}

/* 1 when the library was compiled with OpenMP (the threaded loop below runs
 * on nthreads threads), 0 when it was compiled without (one thread). */
int oracle_openmp(void) {
#ifdef _OPENMP
    return 1;
#else
    return 0;
#endif
}

/* The reference's multithreaded loop shape (src/diff_mod.f90:739-816):
 * OpenMP worksharing over outbeams, each thread computing one outbeam's full
 * grid and adding it under a critical section.  Used only as the timed CPU
 * baseline; the summation order depends on thread timing. */
int oracle_diff_main_omp(const or_grid *g, const or_geom *geo,
                         const or_outbeam *beam, int64_t nbeam,
                         const or_outbeam *ext, int64_t next,
                         zc *ampl_far_beam, zc *ampl_far_ext_diff, int nthreads) {
    const int64_t n4 = 4 * g->nphi * g->ntheta;
    int rc = 0;
    for (int64_t q = 0; q < n4; q++) { ampl_far_beam[q].re = 0; ampl_far_beam[q].im = 0; ampl_far_ext_diff[q] = ampl_far_beam[q]; }
#pragma omp parallel num_threads(nthreads)
    {
        zc *amplC = malloc(sizeof(zc) * n4);
#pragma omp for
        for (int64_t jb = 0; jb < nbeam; jb++) {
            int r = oracle_diffraction(g, geo, &beam[jb], -1.0, amplC);
#pragma omp critical
            {
                if (r) rc = r;
                else for (int64_t q = 0; q < n4; q++) ampl_far_beam[q] = zadd(ampl_far_beam[q], amplC[q]);
            }
        }
#pragma omp for
        for (int64_t jb = 0; jb < next; jb++) {
            int r = oracle_diffraction(g, geo, &ext[jb], PI_REF / 2.0, amplC);
#pragma omp critical
            {
                if (r) rc = r;
                else for (int64_t q = 0; q < n4; q++) ampl_far_ext_diff[q] = zadd(ampl_far_ext_diff[q], amplC[q]);
            }
        }
        free(amplC);
    }
    return rc;
}

/* ------------------------------------------------------------ outputs_mod */

/* simpne, src/misc_submod.f90:2392-2531 (y read with stride ys) */
double oracle_simpne(int64_t ntab, const double *x, const double *y, int64_t ys) {
    double del[3], g[3], pi1[3], e, f, feints, sum1, x1, x2, x3, result = 0.0;
    if (ntab <= 2) return NAN;
    int64_t n = 1;
    for (;;) {
        x1 = x[n - 1]; x2 = x[n]; x3 = x[n + 1];
        e = x3 * x3 - x1 * x1;
        f = x3 * x3 * x3 - x1 * x1 * x1;
        feints = x3 - x1;
        del[0] = x3 - x2; del[1] = x1 - x3; del[2] = x2 - x1;
        g[0] = x2 + x3; g[1] = x1 + x3; g[2] = x1 + x2;
        pi1[0] = x2 * x3; pi1[1] = x1 * x3; pi1[2] = x1 * x2;
        sum1 = 0.0;
        for (int i = 1; i <= 3; i++)
            sum1 = sum1 + y[(n - 2 + i) * ys] * del[i - 1] * (f / 3.0 - g[i - 1] * 0.5 * e + pi1[i - 1] * feints);
        result = result - sum1 / (del[0] * del[1] * del[2]);
        n = n + 2;
        if (ntab <= n + 1) break;
    }
    if (ntab % 2 != 0) return result;
    n = ntab - 2;
    x3 = x[ntab - 1]; x2 = x[ntab - 2]; x1 = x[ntab - 3];
    e = x3 * x3 - x2 * x2;
    f = x3 * x3 * x3 - x2 * x2 * x2;
    feints = x3 - x2;
    del[0] = x3 - x2; del[1] = x1 - x3; del[2] = x2 - x1;
    g[0] = x2 + x3; g[1] = x1 + x3; g[2] = x1 + x2;
    pi1[0] = x2 * x3; pi1[1] = x1 * x3; pi1[2] = x1 * x2;
    sum1 = 0.0;
    for (int i = 1; i <= 3; i++)
        sum1 = sum1 + y[(n - 2 + i) * ys] * del[i - 1] * (f / 3.0 - g[i - 1] * 0.5 * e + pi1[i - 1] * feints);
    result = result - sum1 / (del[0] * del[1] * del[2]);
    return result;
}

static inline double re_mc(zc a, zc b) { return a.re * b.re - a.im * (-b.im); } /* real(a*conjg(b)) */
static inline double im_mc(zc a, zc b) { return a.re * (-b.im) + a.im * b.re; } /* imag(a*conjg(b)) */

/* ampl_to_mueller, src/outputs_mod.f90:473-549.  mueller is (nphi,ntheta,16). */
void oracle_ampl_to_mueller(int64_t nb, const zc *ampl, double *mu) {
    for (int64_t o = 0; o < nb; o++) {
        zc a11 = ampl[o], a21 = ampl[o + nb], a12 = ampl[o + 2 * nb], a22 = ampl[o + 3 * nb];
        double p11 = re_mc(a11, a11), p12 = re_mc(a12, a12), p21 = re_mc(a21, a21), p22 = re_mc(a22, a22);
        mu[o + nb * 0] = 0.5 * (p11 + p12 + p21 + p22);
        mu[o + nb * 1] = 0.5 * (p11 - p12 + p21 - p22);
        mu[o + nb * 2] = re_mc(a11, a12) + re_mc(a22, a21);
        mu[o + nb * 3] = im_mc(a11, a12) - im_mc(a22, a21);
        mu[o + nb * 4] = 0.5 * (p11 + p12 - p21 - p22);
        mu[o + nb * 5] = 0.5 * (p11 - p12 - p21 + p22);
        mu[o + nb * 6] = re_mc(a11, a12) - re_mc(a22, a21);
        mu[o + nb * 7] = im_mc(a11, a12) + im_mc(a22, a21);
        mu[o + nb * 8] = re_mc(a11, a21) + re_mc(a22, a12);
        mu[o + nb * 9] = re_mc(a11, a21) - re_mc(a22, a12);
        mu[o + nb * 10] = re_mc(a11, a22) + re_mc(a12, a21);
        mu[o + nb * 11] = im_mc(a11, a22) + im_mc(a21, a12);
        mu[o + nb * 12] = im_mc(a21, a11) + im_mc(a22, a12);
        mu[o + nb * 13] = im_mc(a21, a11) - im_mc(a22, a12);
        mu[o + nb * 14] = im_mc(a22, a11) - im_mc(a12, a21);
        mu[o + nb * 15] = re_mc(a22, a11) - re_mc(a12, a21);
    }
}

/* get_1d_mueller, src/outputs_mod.f90:280-329: mueller_1d is (ntheta,16) */
void oracle_get_1d_mueller(const double *mu, int64_t nphi, int64_t ntheta,
                           const double *phi, double *mu1d) {
    int64_t nb = nphi * ntheta;
    for (int64_t i = 0; i < ntheta; i++)
        for (int e = 0; e < 16; e++)
            mu1d[i + ntheta * e] = oracle_simpne(nphi, phi, mu + nb * e + nphi * i, 1);
}

/* finalise, src/outputs_mod.f90:63-278.  ampl_far_beam / ampl_far_ext_diff
 * are taken by value (copied); params_io carries abs, geo_cross_sec,
 * beam_energy_out and ext_energy_out in and receives the results. */
int oracle_finalise(const zc *afb_in, const zc *afe_in, int64_t nphi, int64_t ntheta,
                    const double *theta, const double *phi, double la, int scaling,
                    double *mueller, double *mueller_1d, or_params *P) {
    int64_t nb = nphi * ntheta;
    if (nphi <= 2 || ntheta <= 2) return -6;
    zc *afb = malloc(sizeof(zc) * 12 * nb), *afe = afb + 4 * nb, *af = afb + 8 * nb;
    double *mb = malloc(sizeof(double) * 32 * nb), *me = mb + 16 * nb;
    double *m1b = malloc(sizeof(double) * 32 * ntheta), *m1e = m1b + 16 * ntheta;
    double *yv = malloc(sizeof(double) * ntheta);
    double waveno = 2.0 * PI_REF / la;
    double w2 = waveno * waveno;
    for (int64_t q = 0; q < 4 * nb; q++) { afb[q] = zscale(afb_in[q], waveno); afe[q] = zscale(afe_in[q], waveno); }
    for (int64_t q = 0; q < 4 * nb; q++) af[q] = zadd(afb[q], afe[q]);
    oracle_ampl_to_mueller(nb, af, mueller);
    oracle_ampl_to_mueller(nb, afb, mb);
    oracle_ampl_to_mueller(nb, afe, me);
    oracle_get_1d_mueller(mueller, nphi, ntheta, phi, mueller_1d);
    oracle_get_1d_mueller(mb, nphi, ntheta, phi, m1b);
    oracle_get_1d_mueller(me, nphi, ntheta, phi, m1e);
#define THETA_INT(dst, m1, extra_div)                                              \
    do {                                                                           \
        for (int64_t j = 0; j < ntheta; j++) yv[j] = (m1)[j] * sin(theta[j]) extra_div / w2; \
        dst = oracle_simpne(ntheta, theta, yv, 1);                                 \
    } while (0)
    double scatt, scatt_beam, scatt_ext;
    THETA_INT(scatt, mueller_1d, );
    THETA_INT(scatt_beam, m1b, );
    THETA_INT(scatt_ext, m1e, );
    if (scaling) {
        double sb = sqrt(scatt_beam / P->beam_energy_out), se = sqrt(scatt_ext / P->ext_energy_out);
        for (int64_t q = 0; q < 4 * nb; q++) {
            afb[q].re = afb[q].re / sb; afb[q].im = afb[q].im / sb;
            afe[q].re = afe[q].re / se; afe[q].im = afe[q].im / se;
        }
        for (int64_t q = 0; q < 4 * nb; q++) af[q] = zadd(afb[q], afe[q]);
        oracle_ampl_to_mueller(nb, af, mueller);
        oracle_ampl_to_mueller(nb, afb, mb);
        oracle_ampl_to_mueller(nb, afe, me);
        oracle_get_1d_mueller(mueller, nphi, ntheta, phi, mueller_1d);
        oracle_get_1d_mueller(mb, nphi, ntheta, phi, m1b);
        oracle_get_1d_mueller(me, nphi, ntheta, phi, m1e);
        THETA_INT(scatt, mueller_1d, );
        THETA_INT(scatt_beam, m1b, );
        THETA_INT(scatt_ext, m1e, );
    }
    double absorption = P->abs_;
    double ext = absorption + scatt;
    double albedo = 1 - (ext - scatt) / ext;
    double asym, asym_beam, asym_ext;
    THETA_INT(asym, mueller_1d, * cos(theta[j]) / scatt);
    THETA_INT(asym_beam, m1b, * cos(theta[j]) / scatt_beam);
    THETA_INT(asym_ext, m1e, * cos(theta[j]) / scatt_ext);
#undef THETA_INT
    int64_t ib = 0;
    double best = fabs(theta[0] - 2 * PI_REF);
    for (int64_t j = 1; j < ntheta; j++) {
        double d = fabs(theta[j] - 2 * PI_REF);
        if (d < best) { best = d; ib = j; }
    }
    double back_scatt = mueller[0 + nphi * ib] * 4 * PI_REF / w2;
    P->scatt = scatt;
    P->abs_ = absorption;
    P->ext = ext;
    P->albedo = albedo;
    P->asymmetry = asym;
    P->abs_eff = absorption / P->geo_cross_sec;
    P->scatt_eff = scatt / P->geo_cross_sec;
    P->ext_eff = ext / P->geo_cross_sec;
    P->back_scatt = back_scatt;
    P->scatt_beam = scatt_beam;
    P->scatt_ext_diff = scatt_ext;
    P->asymmetry_beam = asym_beam;
    P->asymmetry_ext_diff = asym_ext;
    P->scatt_eff_beam = scatt_beam / P->geo_cross_sec;
    P->scatt_eff_ext_diff = scatt_ext / P->geo_cross_sec;
    free(yv); free(m1b); free(mb); free(afb);
    return 0;
}

/* summation, src/outputs_mod.f90:407-471 (totals must start zeroed) */
void oracle_summation(const double *mu, double *mu_tot, int64_t n2d,
                      const double *mu1d, double *mu1d_tot, int64_t n1d,
                      const or_params *p, or_params *t) {
    for (int64_t q = 0; q < n2d; q++) mu_tot[q] = mu_tot[q] + mu[q];
    for (int64_t q = 0; q < n1d; q++) mu1d_tot[q] = mu1d_tot[q] + mu1d[q];
    t->abs_ += p->abs_; t->scatt += p->scatt; t->back_scatt += p->back_scatt;
    t->ext += p->ext; t->albedo += p->albedo; t->asymmetry += p->asymmetry;
    t->abs_eff += p->abs_eff; t->scatt_eff += p->scatt_eff; t->ext_eff += p->ext_eff;
    t->geo_cross_sec += p->geo_cross_sec; t->scatt_beam += p->scatt_beam;
    t->scatt_ext_diff += p->scatt_ext_diff; t->asymmetry_beam += p->asymmetry_beam;
    t->asymmetry_ext_diff += p->asymmetry_ext_diff; t->scatt_eff_beam += p->scatt_eff_beam;
    t->scatt_eff_ext_diff += p->scatt_eff_ext_diff;
}

/* divide_by_num_orientations, src/outputs_mod.f90:13-43 */
void oracle_divide(double *mu_tot, int64_t n2d, double *mu1d_tot, int64_t n1d,
                   or_params *t, int64_t num_orients) {
    double n = (double)num_orients;
    for (int64_t q = 0; q < n2d; q++) mu_tot[q] = mu_tot[q] / n;
    for (int64_t q = 0; q < n1d; q++) mu1d_tot[q] = mu1d_tot[q] / n;
    t->abs_ /= n; t->scatt /= n; t->ext /= n; t->albedo /= n; t->asymmetry /= n;
    t->abs_eff /= n; t->scatt_eff /= n; t->ext_eff /= n; t->geo_cross_sec /= n;
    t->back_scatt /= n; t->scatt_beam /= n; t->scatt_ext_diff /= n;
    t->asymmetry_beam /= n; t->asymmetry_ext_diff /= n; t->scatt_eff_beam /= n;
    t->scatt_eff_ext_diff /= n;
}

/* ------------------------------------------------------ flat C entry points */

int oracle_diff_main_flat(const double *theta, int64_t ntheta, const double *phi, int64_t nphi,
                          double lambda, int is_fast_diff,
                          const double *verts, int64_t nverts, const int64_t *face_off,
                          const int64_t *face_vi, int64_t nfaces,
                          const void *beam, int64_t nbeam, const void *ext, int64_t next,
                          double *ampl_far_beam, double *ampl_far_ext_diff, int nthreads) {
    int64_t nb = nphi * ntheta;
    double *xyz = malloc(sizeof(double) * 3 * nb);
    oracle_make_far_field_bins(theta, ntheta, phi, nphi, xyz, xyz + nb, xyz + 2 * nb);
    or_grid g = {nphi, ntheta, theta, phi, xyz, xyz + nb, xyz + 2 * nb, lambda, is_fast_diff};
    or_geom geo = {nverts, verts, face_off, face_vi, nfaces};
    int rc;
    if (nthreads <= 0)
        rc = oracle_diff_main(&g, &geo, beam, nbeam, ext, next, (zc *)ampl_far_beam, (zc *)ampl_far_ext_diff);
    else
        rc = oracle_diff_main_omp(&g, &geo, beam, nbeam, ext, next, (zc *)ampl_far_beam,
                                  (zc *)ampl_far_ext_diff, nthreads);
    free(xyz);
    return rc;
}

int oracle_diffraction_flat(const double *theta, int64_t ntheta, const double *phi, int64_t nphi,
                            double lambda, int is_fast_diff,
                            const double *verts, int64_t nverts, const int64_t *face_off,
                            const int64_t *face_vi, int64_t nfaces,
                            const void *ob, double fov_override, double *amplC) {
    int64_t nb = nphi * ntheta;
    double *xyz = malloc(sizeof(double) * 3 * nb);
    oracle_make_far_field_bins(theta, ntheta, phi, nphi, xyz, xyz + nb, xyz + 2 * nb);
    or_grid g = {nphi, ntheta, theta, phi, xyz, xyz + nb, xyz + 2 * nb, lambda, is_fast_diff};
    or_geom geo = {nverts, verts, face_off, face_vi, nfaces};
    int rc = oracle_diffraction(&g, &geo, ob, fov_override, (zc *)amplC);
    free(xyz);
    return rc;
}

int oracle_finalise_flat(const double *afb, const double *afe, int64_t nphi, int64_t ntheta,
                         const double *theta, const double *phi, double la, int scaling,
                         double *mueller, double *mueller_1d, double *params18) {
    return oracle_finalise((const zc *)afb, (const zc *)afe, nphi, ntheta, theta, phi, la,
                           scaling, mueller, mueller_1d, (or_params *)params18);
}

void oracle_summation_flat(const double *mu, double *mu_tot, int64_t n2d, const double *mu1d,
                           double *mu1d_tot, int64_t n1d, const double *p, double *t) {
    oracle_summation(mu, mu_tot, n2d, mu1d, mu1d_tot, n1d, (const or_params *)p, (or_params *)t);
}

void oracle_divide_flat(double *mu_tot, int64_t n2d, double *mu1d_tot, int64_t n1d, double *t,
                        int64_t num_orients) {
    oracle_divide(mu_tot, n2d, mu1d_tot, n1d, (or_params *)t, num_orients);
}
