// frame.h -- the per-facet aperture frame of PBT's diffraction routine.
//
// One outgoing facet's set-up work, done once per facet before its far-field
// sum: centre of mass, the rotation into the aperture plane
// (get_rotation_matrix2, src/diff_mod.f90:200-289), the in-plane rotation
// that puts the propagation direction in the x-z plane (src/diff_mod.f90:
// 540-559), the anti-parallel amplitude flip (:561-571) and the rotated
// incidence direction (:573-574).  Operation order follows the reference
// exactly (left-to-right sums from zero, as gfortran's inline matmul); build
// without FMA contraction so the host copy reproduces the reference's
// rounding with the platform libm.
//
// Compiled twice: by the host compiler for the reference-exact FP64 path
// (libm atan/atan2/sin/cos) and by nvcc for the GPU set-up kernel of the
// batched path (CUDA libm).
#pragma once
#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define PBT_HD __host__ __device__ __forceinline__
#else
#define PBT_HD inline
#endif

namespace pbt {

// src/misc_submod.f90:12: pi is a default-real literal widened to real(8)
constexpr double kPiRef = (double)3.14159265358979f;
constexpr double kLit0_999999 = (double)0.999999f;  // src/diff_mod.f90:151
constexpr double kLit1em6 = (double)1e-6f;          // src/diff_mod.f90:364-365
constexpr double kLit0_999 = (double)0.999f;        // src/diff_mod.f90:630
constexpr double kLit0_0001 = (double)0.0001f;      // src/diff_mod.f90:563
constexpr double kFarR = 1e6;                       // src/diff_mod.f90:848

struct Mat3 {
    double m[3][3];
};

PBT_HD void mm33(const Mat3 &a, const Mat3 &b, Mat3 &c) {
    Mat3 t;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double s = 0.0;
            s = s + a.m[i][0] * b.m[0][j];
            s = s + a.m[i][1] * b.m[1][j];
            s = s + a.m[i][2] * b.m[2][j];
            t.m[i][j] = s;
        }
    c = t;
}

PBT_HD void mv33(const Mat3 &a, const double x[3], double y[3]) {
    double t[3];
    for (int i = 0; i < 3; i++) {
        double s = 0.0;
        s = s + a.m[i][0] * x[0];
        s = s + a.m[i][1] * x[1];
        s = s + a.m[i][2] * x[2];
        t[i] = s;
    }
    y[0] = t[0];
    y[1] = t[1];
    y[2] = t[2];
}

PBT_HD double dot3(const double a[3], const double b[3]) {
    double s = 0.0;
    s = s + a[0] * b[0];
    s = s + a[1] * b[1];
    s = s + a[2] * b[2];
    return s;
}

// cross, src/misc_submod.f90:2367-2390 (normalised)
PBT_HD void cross3n(const double a[3], const double b[3], double c[3]) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
    double nf = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
    c[0] = c[0] / nf;
    c[1] = c[1] / nf;
    c[2] = c[2] / nf;
}

// Result of the per-facet set-up.
struct FacetFrame {
    double com[3];    // aperture centre of mass
    Mat3 R;           // matmul(rot2, rot): lab -> aperture frame (src/diff_mod.f90:618, :334)
    double prop2[3];  // propagation direction in the aperture frame
    double inc2[3];   // incidence direction (0,0,-1) in the aperture frame
    double sign;      // -1 when the anti-parallel flip applies (src/diff_mod.f90:571)
};

// get_rotation_matrix2, src/diff_mod.f90:200-289.  a1/b1: first two vertices
// relative to the centre of mass.
PBT_HD void get_rotation_matrix2(const double a1[3], const double b1[3], Mat3 &rot) {
    double t1 = atan(a1[0] / a1[1]);
    Mat3 rot1 = {{{cos(t1), -sin(t1), 0}, {sin(t1), cos(t1), 0}, {0, 0, 1}}};
    double a2[3], b2[3];
    mv33(rot1, a1, a2);
    mv33(rot1, b1, b2);
    double t2 = -atan(a2[2] / a2[1]);
    Mat3 rot2 = {{{1, 0, 0}, {0, cos(t2), -sin(t2)}, {0, sin(t2), cos(t2)}}};
    double a3[3], b3[3];
    mv33(rot2, a2, a3);
    mv33(rot2, b2, b3);
    double t3 = atan(b3[2] / b3[0]);
    Mat3 rot3 = {{{cos(t3), 0, sin(t3)}, {0, 1, 0}, {-sin(t3), 0, cos(t3)}}};
    double a4[3], b4[3];
    mv33(rot3, a3, a4);
    mv33(rot3, b3, b4);
    Mat3 r21, r321;
    mm33(rot2, rot1, r21);
    mm33(rot3, r21, r321);
    if (a4[0] * b4[1] - a4[1] * b4[0] > 0) {
        Mat3 rot4 = {{{-1, 0, 0}, {0, 1, 0}, {0, 0, -1}}};
        mm33(rot4, r321, rot);
    } else {
        rot = r321;
    }
}

// Per-facet set-up of diffraction, src/diff_mod.f90:515-574 (+ the rotation
// product passed to rotate_far_field_bins, :618).  vx/vy/vz: the facet's nv
// vertices (lab frame).  Returns the frame; v20 (vertices relative to com) is
// written to rx/ry/rz when those are non-null.
PBT_HD void facet_frame(const double *vx, const double *vy, const double *vz, int nv,
                        const double prop0[3], const double perp0[3], FacetFrame &fr,
                        double *rx, double *ry, double *rz) {
    double com[3] = {0, 0, 0};
    for (int i = 0; i < nv; i++) {
        com[0] = com[0] + vx[i];
        com[1] = com[1] + vy[i];
        com[2] = com[2] + vz[i];
    }
    com[0] = com[0] / (double)nv;
    com[1] = com[1] / (double)nv;
    com[2] = com[2] / (double)nv;
    double a1[3] = {vx[0] - com[0], vy[0] - com[1], vz[0] - com[2]};
    double b1[3] = {vx[1] - com[0], vy[1] - com[1], vz[1] - com[2]};
    if (rx) {
        for (int i = 0; i < nv; i++) {
            rx[i] = vx[i] - com[0];
            ry[i] = vy[i] - com[1];
            rz[i] = vz[i] - com[2];
        }
    }
    Mat3 rot;
    get_rotation_matrix2(a1, b1, rot);
    double prop1[3], perp1[3];
    mv33(rot, prop0, prop1);
    mv33(rot, perp0, perp1);
    double angle = -atan2(prop1[1], prop1[0]);
    Mat3 rot2 = {{{cos(angle), -sin(angle), 0}, {sin(angle), cos(angle), 0}, {0, 0, 1}}};
    double prop2[3], perp2[3], e_par2[3];
    mv33(rot2, prop1, prop2);
    mv33(rot2, perp1, perp2);
    cross3n(perp2, prop2, e_par2);
    fr.sign = (e_par2[2] > kLit0_0001) ? -1.0 : 1.0;
    double inc[3] = {0, 0, -1}, t3[3];
    mv33(rot, inc, t3);
    mv33(rot2, t3, fr.inc2);
    mm33(rot2, rot, fr.R);
    for (int c = 0; c < 3; c++) {
        fr.com[c] = com[c];
        fr.prop2[c] = prop2[c];
    }
}

}  // namespace pbt
