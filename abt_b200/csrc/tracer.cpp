// tracer.cpp -- PBT's near-field beam tracer on the host (FP64, OpenMP): the
// per-orientation outbeam lists that the far-field stage consumes.
//
// What it restates (the reference's speed-priority orientation step):
//   * particle preparation after reading: aperture count, midpoints, areas,
//     centre of mass moved to the origin, normals, apertures
//     (src/input_mod.f90:2663-2680; helpers src/misc_submod.f90:65-230);
//   * the Euler rotation of one orientation and the recomputed midpoints,
//     normals and apertures (src/input_mod.f90:1705-1908, methods 'euler'
//     and 'multi' after their angles are formed);
//   * the incident beam: one square facet at z = 1000 along (0,0,-1) with
//     the identity amplitude and e-perp (1,0,0) (src/input_mod.f90:2112-2264);
//   * the beam loop (src/beam_loop_mod.f90:1626-1806): incidence
//     (recursion_inc :424-612), internal and external propagation
//     (recursion_int :614-812, recursion_ext :814-1008), the visibility tests
//     (find_vis_inc/int/ext :2037-2609 with the 4 x 4 beam-aligned buckets
//     :2668-2743), complex Snell's law (:342-383), refracted directions
//     (:1010-1051), the scattering-plane rotation (:2611-2638), beam-tree
//     growth with the area/energy thresholds (:1053-1465), beam rotation
//     (:1467-1526), outbeam emission with fov = 8 lambda / d (:2745-2794),
//     the geometric cross section (:2640-2666) and the energy checks
//     (:1528-1624).
//
// Arithmetic follows the reference's operation order (left-to-right sums,
// Fortran's default-real literals widened to double, libm trig, Smith's
// complex division as gfortran lowers a/b); the unit is built without FMA
// contraction.
//
// Provenance: the physics routines restate the reference project's
// algorithms (hballington12/abt, GPL-3.0) step by step and in its operation
// order, because the outbeam lists must agree with a run of the reference bit
// for bit.  The data layout, the bucket assignment of the visibility tests, the
// per-level parallel propagation with ordered appends, and the C interface
// are this file's own.
//
// Order of work.  The reference propagates the beams of one recursion level
// on OpenMP threads and appends their children and outbeams inside critical
// sections, so its list order depends on thread timing.  Here the beams of a
// level are propagated in parallel and their children and outbeams are
// appended afterwards in beam order -- the order of a single-threaded run of
// the reference -- so the lists are the same on any number of threads.
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "frame.h"
#include "pbt_diff.h"
#include "pbt_internal.h"

using pbt::kPiRef;
using pbt::Mat3;
using pbt::set_error;

namespace {

constexpr double kLit0_01 = (double)0.01f;  // aperture-facing tests, src/beam_loop_mod.f90:2345
constexpr double kLit1_1 = (double)1.1f;    // stretch factors, src/beam_loop_mod.f90:2681,
                                            // src/input_mod.f90:2160
constexpr double kLit1em5 = (double)1e-5f;  // near-normal refraction, src/beam_loop_mod.f90:1040
constexpr double kBeamZ = 1000.0;           // incident plane, src/input_mod.f90:2169
constexpr int kBB = 4;                      // bucket grid 4 x 4, src/beam_loop_mod.f90:2679-2680
constexpr int64_t kGridFaces = 256;  // find_vis: candidate sets from this size use the cell grid

// The cell-grid threshold; PBT_TRACER_GRID_MIN overrides it (a test compares the
// lists of both walks).
int64_t grid_min_faces() {
    static const int64_t v = [] {
        const char *e = getenv("PBT_TRACER_GRID_MIN");
        const long long x = e ? atoll(e) : -1;
        return x >= 0 ? (int64_t)x : kGridFaces;
    }();
    return v;
}
constexpr int64_t kMaxBeams = 20000000;     // guard against a runaway tree

// ------------------------------------------------------------------ complex

struct Z {
    double re, im;
};
inline Z zmul(Z a, Z b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline Z zadd(Z a, Z b) { return {a.re + b.re, a.im + b.im}; }
inline Z zsub(Z a, Z b) { return {a.re - b.re, a.im - b.im}; }
inline Z zscale(double s, Z a) { return {s * a.re, s * a.im}; }
// a / b with Smith's range reduction (R. L. Smith, Comm. ACM 5(8):435, 1962),
// the method gfortran uses for complex division
inline Z zdiv(Z a, Z b) {
    if (fabs(b.re) < fabs(b.im)) {
        const double r = b.re / b.im, den = b.re * r + b.im;
        return {(a.re * r + a.im) / den, (a.im * r - a.re) / den};
    }
    const double r = b.im / b.re, den = b.im * r + b.re;
    return {(a.im * r + a.re) / den, (a.im - a.re * r) / den};
}

// 2x2 complex amplitude matrix, A[i][j] = ampl(i+1, j+1)
struct Amp {
    Z a[2][2];
};
inline Amp amp_identity() {
    Amp m;
    m.a[0][0] = {1.0, 0.0};
    m.a[0][1] = {0.0, 0.0};
    m.a[1][0] = {0.0, 0.0};
    m.a[1][1] = {1.0, 0.0};
    return m;
}
// matmul(r, A) for a real 2x2 r (sums from zero, k ascending)
inline Amp rmatmul(const double r[2][2], const Amp &A) {
    Amp c;
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) {
            Z s = {0.0, 0.0};
            s = zadd(s, zscale(r[i][0], A.a[0][j]));
            s = zadd(s, zscale(r[i][1], A.a[1][j]));
            c.a[i][j] = s;
        }
    return c;
}
// matmul(F, A) for a complex 2x2 F
inline Amp zmatmul(const Z F[2][2], const Amp &A) {
    Amp c;
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) {
            Z s = {0.0, 0.0};
            s = zadd(s, zmul(F[i][0], A.a[0][j]));
            s = zadd(s, zmul(F[i][1], A.a[1][j]));
            c.a[i][j] = s;
        }
    return c;
}
inline Amp amp_times(const Amp &A, Z z) {
    Amp c;
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) c.a[i][j] = zmul(A.a[i][j], z);
    return c;
}
inline Amp amp_scale(const Amp &A, double s) {
    Amp c;
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) c.a[i][j] = {A.a[i][j].re * s, A.a[i][j].im * s};
    return c;
}
// real(0.5 * sum of |a_ij|^2) in the order (1,1), (1,2), (2,1), (2,2)
inline double intensity(const Amp &A) {
    auto p = [](Z z) { return z.re * z.re + z.im * z.im; };
    double s = p(A.a[0][0]);
    s = s + p(A.a[0][1]);
    s = s + p(A.a[1][0]);
    s = s + p(A.a[1][1]);
    return 0.5 * s;
}

// ------------------------------------------------------------------ vectors

inline double dot3(const double *a, const double *b) {
    double s = 0.0;
    s = s + a[0] * b[0];
    s = s + a[1] * b[1];
    s = s + a[2] * b[2];
    return s;
}
// cross(a, b, c, normalise) of src/misc_submod.f90:2367-2390
inline void cross3(const double *a, const double *b, double *c, bool normalise) {
    double t[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2],
                   a[0] * b[1] - a[1] * b[0]};
    double nf = sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
    if (!normalise) nf = 1.0;
    c[0] = t[0] / nf;
    c[1] = t[1] / nf;
    c[2] = t[2] / nf;
}
inline void normalise3(double *v) {
    const double nf = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    v[0] = v[0] / nf;
    v[1] = v[1] / nf;
    v[2] = v[2] / nf;
}
inline void matT_vec(const Mat3 &r, const double *x, double *y) {  // transpose(r) . x
    double t[3];
    for (int i = 0; i < 3; i++) {
        double s = 0.0;
        s = s + r.m[0][i] * x[0];
        s = s + r.m[1][i] * x[1];
        s = s + r.m[2][i] * x[2];
        t[i] = s;
    }
    y[0] = t[0];
    y[1] = t[1];
    y[2] = t[2];
}

// ------------------------------------------------------------------ geometry

// Vertices row-major (x, y, z per vertex); faces as a 0-based CSR; apertures
// 0-based per face.  Per-face and per-aperture data of one frame.
struct Shape {
    int64_t nv = 0, nf = 0, na = 0;
    std::vector<double> v;             // nv * 3
    std::vector<int64_t> off, vi;      // CSR
    std::vector<int64_t> ap;           // per face
    std::vector<double> area;          // per face (rotation invariant)
    std::vector<double> mid, n;        // per face * 3
    std::vector<double> apn, apmid;    // per aperture * 3
    std::vector<double> aparea;
};

// compute_geometry_midpoints (src/misc_submod.f90:199-209)
void shape_midpoints(Shape &g) {
    g.mid.assign(3 * g.nf, 0.0);
    for (int64_t f = 0; f < g.nf; f++) {
        const int64_t n = g.off[f + 1] - g.off[f];
        for (int c = 0; c < 3; c++) {
            double s = 0.0;
            for (int64_t q = g.off[f]; q < g.off[f + 1]; q++) s = s + g.v[3 * g.vi[q] + c];
            g.mid[3 * f + c] = s / (double)n;
        }
    }
}

// compute_geometry_areas (src/misc_submod.f90:172-197): fan from the midpoint
void shape_areas(Shape &g) {
    g.area.assign(g.nf, 0.0);
    for (int64_t f = 0; f < g.nf; f++) {
        const int64_t b = g.off[f], e = g.off[f + 1];
        double a = 0.0;
        for (int64_t q = b; q < e; q++) {
            const int64_t q2 = (q + 1 < e) ? q + 1 : b;
            double va[3], vb[3], c[3];
            for (int k = 0; k < 3; k++) {
                va[k] = g.v[3 * g.vi[q] + k] - g.mid[3 * f + k];
                vb[k] = g.v[3 * g.vi[q2] + k] - g.mid[3 * f + k];
            }
            cross3(va, vb, c, false);
            a = a + sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]) / 2;
        }
        g.area[f] = a;
    }
}

// compute_geometry_normals (src/misc_submod.f90:211-230): first three vertices
void shape_normals(Shape &g) {
    g.n.assign(3 * g.nf, 0.0);
    for (int64_t f = 0; f < g.nf; f++) {
        const double *v1 = &g.v[3 * g.vi[g.off[f]]], *v2 = &g.v[3 * g.vi[g.off[f] + 1]],
                     *v3 = &g.v[3 * g.vi[g.off[f] + 2]];
        double e12[3], e23[3];
        for (int k = 0; k < 3; k++) {
            e12[k] = v2[k] - v1[k];
            e23[k] = v3[k] - v2[k];
        }
        cross3(e12, e23, &g.n[3 * f], true);
    }
}

// compute_geometry_apertures (src/misc_submod.f90:141-170)
void shape_apertures(Shape &g) {
    g.apn.assign(3 * g.na, 0.0);
    g.apmid.assign(3 * g.na, 0.0);
    g.aparea.assign(g.na, 0.0);
    std::vector<int64_t> cnt(g.na, 0);
    for (int64_t f = 0; f < g.nf; f++) {  // faces in order within each aperture
        const int64_t a = g.ap[f];
        cnt[a]++;
        for (int k = 0; k < 3; k++) {
            g.apn[3 * a + k] = g.apn[3 * a + k] + g.n[3 * f + k];
            g.apmid[3 * a + k] = g.apmid[3 * a + k] + g.mid[3 * f + k];
        }
        g.aparea[a] = g.aparea[a] + g.area[f];
    }
    for (int64_t a = 0; a < g.na; a++) {
        for (int k = 0; k < 3; k++) g.apmid[3 * a + k] = g.apmid[3 * a + k] / (double)cnt[a];
        const double *n = &g.apn[3 * a];
        const double fac = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        for (int k = 0; k < 3; k++) g.apn[3 * a + k] = g.apn[3 * a + k] / fac;
    }
}

// The Euler matrix of PROT_MPI (src/input_mod.f90:1794-1812, 1864-1882)
Mat3 euler_matrix(const double e[3]) {
    const double s1 = sin(e[0]), s2 = sin(e[1]), s3 = sin(e[2]);
    const double c1 = cos(e[0]), c2 = cos(e[1]), c3 = cos(e[2]);
    Mat3 r;
    r.m[0][0] = c1 * c2 * c3 - s1 * s3;
    r.m[0][1] = -(c1 * c2 * s3) - s1 * c3;
    r.m[0][2] = c1 * s2;
    r.m[1][0] = s1 * c2 * c3 + c1 * s3;
    r.m[1][1] = -(s1 * c2 * s3) + c1 * c3;
    r.m[1][2] = s1 * s2;
    r.m[2][0] = -(s2 * c3);
    r.m[2][1] = s2 * s3;
    r.m[2][2] = c2;
    return r;
}

// ------------------------------------------------------------------ beams

struct FieldIn {
    int64_t fi;  // face (0-based); the incident beam's own facet is -1
    Amp ampl;
    double e_perp[3];
    bool is_outgoing;
};

struct FieldOut {
    int64_t fi, ap;
    Amp ampl_int, ampl_ext;
    double e_perp[3], prop_int[3], prop_ext[3];
    bool is_tir;
    double pr, pt;
};

struct Beam {
    double prop[3];
    std::vector<FieldIn> in;
    bool is_int;
    int64_t rec, refl;
    bool is_tir;
    double abs;
};

// The particle in one beam's frame (rot . orientation frame), the buckets of
// find_vis, and the visibility result per face.
struct Vis {
    std::vector<char> in_beam, is_shad;
    std::vector<int64_t> id_beam;  // index into the beam's field list
    std::vector<double> dist;
};

struct Rotated {
    std::vector<double> v, mid, n, apn;
};

// rotate (src/beam_loop_mod.f90:1467-1526): prop onto -z
Mat3 beam_rotation(const double *prop) {
    const double t1 = 2 * kPiRef - atan2(prop[1], prop[0]);
    Mat3 r1 = {{{cos(t1), -sin(t1), 0.0}, {sin(t1), cos(t1), 0.0}, {0.0, 0.0, 1.0}}};
    double tv[3];
    pbt::mv33(r1, prop, tv);
    normalise3(tv);
    const double t2 = acos(-tv[2]);
    Mat3 r2 = {{{cos(t2), 0.0, sin(t2)}, {0.0, 1.0, 0.0}, {-sin(t2), 0.0, cos(t2)}}};
    Mat3 r;
    pbt::mm33(r2, r1, r);
    return r;
}

// component i of matmul(r, x), summed as the full product does
inline double row_dot(const Mat3 &r, int i, const double *x) {
    double s = 0.0;
    s = s + r.m[i][0] * x[0];
    s = s + r.m[i][1] * x[1];
    s = s + r.m[i][2] * x[2];
    return s;
}

// The particle in a beam's frame.  The visibility test reads the vertices' x
// and y, the normals' z, and the midpoints and aperture normals whole; only
// those components are formed (each exactly as the full rotation forms it).
void rotate_shape(const Shape &g, const Mat3 &r, Rotated &o) {
    o.v.resize(3 * g.nv);
    o.mid.resize(3 * g.nf);
    o.n.resize(3 * g.nf);
    o.apn.resize(3 * g.na);
    for (int64_t i = 0; i < g.nv; i++) {
        o.v[3 * i] = row_dot(r, 0, &g.v[3 * i]);
        o.v[3 * i + 1] = row_dot(r, 1, &g.v[3 * i]);
    }
    for (int64_t f = 0; f < g.nf; f++) {
        o.n[3 * f + 2] = row_dot(r, 2, &g.n[3 * f]);
        pbt::mv33(r, &g.mid[3 * f], &o.mid[3 * f]);
    }
    for (int64_t a = 0; a < g.na; a++) pbt::mv33(r, &g.apn[3 * a], &o.apn[3 * a]);
}

enum VisKind { VIS_INC, VIS_INT, VIS_EXT };

// A triangle seen along -z as a possible blocker: corners, the edge normals of
// the reference's inside test (edge k from corner k to k+1), centroid height,
// and whether it faces the incidence (n_z >= 0.01, tested for incidence only)
struct Blocker {
    double x[3], y[3], en1[3], en2[3], z;
    bool up;
};

// find_vis_inc / find_vis_int / find_vis_ext (src/beam_loop_mod.f90:2037-2609).
// A face m is lit when its centroid, seen along -z, lies inside a face j of
// the beam (closest such j); another aperture's face in front of it blocks it.
// Candidate blockers are the faces with a vertex nearest to the 4 x 4 bucket
// nearest to m's centroid, visited in face order as the reference does.
void find_vis(const Shape &g, const Rotated &R, const Beam &beam, VisKind kind, bool par,
              Vis &out) {
    const int64_t nf = g.nf;
    // buckets (beam_aligned_bounding_boxes, :2668-2743), midpoints of 4 corners
    double mnx = R.v[0], mxx = R.v[0], mny = R.v[1], mxy = R.v[1];
    for (int64_t i = 1; i < g.nv; i++) {
        mnx = std::min(mnx, R.v[3 * i]);
        mxx = std::max(mxx, R.v[3 * i]);
        mny = std::min(mny, R.v[3 * i + 1]);
        mxy = std::max(mxy, R.v[3 * i + 1]);
    }
    double xs[kBB + 1], ys[kBB + 1];
    for (int i = 0; i <= kBB; i++) {
        xs[i] = kLit1_1 * (mnx + (mxx - mnx) / kBB * (double)i);
        ys[i] = kLit1_1 * (mny + (mxy - mny) / kBB * (double)i);  // the reference divides by the x count
    }
    // bucket (i,j), corners (i,j), (i,j+1), (i+1,j+1), (i+1,j): its centre's x
    // depends on i only and its y on j only
    double cx[kBB], cy[kBB];
    for (int i = 0; i < kBB; i++) {
        cx[i] = (((xs[i] + xs[i]) + xs[i + 1]) + xs[i + 1]) / 4.0;
        cy[i] = (((ys[i] + ys[i + 1]) + ys[i + 1]) + ys[i]) / 4.0;
    }
    // minloc over b = 4 i + j of sqrt((cx_i - x)^2 + (cy_j - y)^2), the
    // reference's distances.  Rounded addition is monotone in each term, so
    // the smallest sum pairs the smallest x and y terms; only sums within
    // rounding of it can tie after the (monotone) square root, and then the
    // first b with the smallest root wins, as minloc picks it.
    auto nearest = [&](double x, double y) {
        double dx2[kBB], dy2[kBB];
        for (int i = 0; i < kBB; i++) {
            const double dx = cx[i] - x, dy = cy[i] - y;
            dx2[i] = dx * dx;
            dy2[i] = dy * dy;
        }
        int im = 0, jm = 0;
        for (int i = 1; i < kBB; i++) {
            if (dx2[i] < dx2[im]) im = i;
            if (dy2[i] < dy2[jm]) jm = i;
        }
        const double smin = dx2[im] + dy2[jm], win = smin * (1.0 + 1e-14);
        bool alone = true;
        for (int i = 0; i < kBB; i++) {
            if (i != im && dx2[i] + dy2[jm] <= win) alone = false;
            if (i != jm && dx2[im] + dy2[i] <= win) alone = false;
        }
        if (alone) return im * kBB + jm;
        const double rmin = sqrt(smin);
        for (int b = 0; b < kBB * kBB; b++) {
            const double sb = dx2[b / kBB] + dy2[b % kBB];
            if (sb <= win && (sb == smin || sqrt(sb) == rmin)) return b;
        }
        return 0;  // not reached for finite coordinates
    };
    // scratch of the calling thread, reused from beam to beam (bound by
    // reference so that the threads of the loops below share this instance)
    thread_local std::vector<int> vb_tl;
    thread_local std::vector<Blocker> bl_tl;
    thread_local std::vector<char> is_vis_tl;
    thread_local std::vector<int64_t> map_tl, rel_tl;
    thread_local std::vector<uint16_t> memb_tl;
    thread_local std::vector<int64_t> members_tl[kBB * kBB];
    std::vector<int> &vb = vb_tl;
    std::vector<Blocker> &bl = bl_tl;
    std::vector<char> &is_vis = is_vis_tl;
    std::vector<int64_t> &map = map_tl;  // face -> index in the beam's field list
    std::vector<int64_t> &rel = rel_tl;
    std::vector<uint16_t> &memb = memb_tl;
    std::vector<int64_t>(&members)[kBB * kBB] = members_tl;
    vb.resize(g.nv);
    bl.resize(nf);
    memb.resize(nf);
    out.in_beam.assign(nf, kind == VIS_INC ? 1 : 0);
    out.is_shad.assign(nf, 0);
    out.id_beam.assign(nf, -1);
    out.dist.assign(nf, 0.0);
    is_vis.assign(nf, 1);
    map.assign(nf, -1);
    const double ex = std::max(mxx - mnx, mxy - mny), pad = 1e-12 * ex;
    // The faces that can be lit or block.  For the incident beam, every face.  For
    // a beam leaving the particle's faces, a lit centroid lies in the beam's extent
    // in x, y, and a blocker contains it: the faces whose outline (padded by 1e-12
    // of the particle's extent, far beyond the rounding of the inside test) meets
    // that extent -- about a tenth of a rough column's faces.  Their buckets,
    // outlines and bucket lists are formed, in face order; the others' would not
    // be read.
    rel.clear();
    if (kind != VIS_INC) {
        for (size_t i = 0; i < beam.in.size(); i++) map[beam.in[i].fi] = (int64_t)i;
        // beam extent in x, y (:2126-2160)
        const int64_t v0 = g.vi[g.off[beam.in[0].fi]];
        double bxmin = R.v[3 * v0], bxmax = bxmin, bymin = R.v[3 * v0 + 1], bymax = bymin;
        for (const FieldIn &fin : beam.in)
            for (int64_t q = g.off[fin.fi]; q < g.off[fin.fi + 1]; q++) {
                const double x = R.v[3 * g.vi[q]], y = R.v[3 * g.vi[q] + 1];
                if (x > bxmax) bxmax = x;
                if (x < bxmin) bxmin = x;
                if (y > bymax) bymax = y;
                if (y < bymin) bymin = y;
            }
        for (int64_t f = 0; f < nf; f++) {
            const double x = R.mid[3 * f], y = R.mid[3 * f + 1];
            if (x < bxmin || x > bxmax || y < bymin || y > bymax) is_vis[f] = 0;
        }
        const double ax0 = bxmin - pad, ax1 = bxmax + pad, ay0 = bymin - pad, ay1 = bymax + pad;
        for (int64_t f = 0; f < nf; f++) {
            const int64_t q0 = 3 * g.vi[g.off[f]], q1 = 3 * g.vi[g.off[f] + 1],
                          q2 = 3 * g.vi[g.off[f] + 2];
            const double x0 = std::min(std::min(R.v[q0], R.v[q1]), R.v[q2]);
            const double x1 = std::max(std::max(R.v[q0], R.v[q1]), R.v[q2]);
            const double y0 = std::min(std::min(R.v[q0 + 1], R.v[q1 + 1]), R.v[q2 + 1]);
            const double y1 = std::max(std::max(R.v[q0 + 1], R.v[q1 + 1]), R.v[q2 + 1]);
            if (!(x1 < ax0 || x0 > ax1 || y1 < ay0 || y0 > ay1)) rel.push_back(f);
        }
    }
    const bool all = kind == VIS_INC;
    const int64_t nrel = all ? nf : (int64_t)rel.size();
    auto rel_face = [&](int64_t i) { return all ? i : rel[i]; };
    // bucket of every vertex of those faces (a face's vertices are tested one by
    // one in the reference; the answer depends on the coordinates only)
    if (all) {
#pragma omp parallel for schedule(static) if (par && g.nv > 4096)
        for (int64_t q = 0; q < g.nv; q++) vb[q] = nearest(R.v[3 * q], R.v[3 * q + 1]);
    } else {
        // each shared vertex once: stamp[q] marks the calls that formed vb[q]
        thread_local std::vector<uint32_t> stamp_tl;
        thread_local uint32_t call_tl = 0;
        std::vector<uint32_t> &stamp = stamp_tl;
        if (stamp.size() != (size_t)g.nv || ++call_tl == 0) {
            stamp.assign(g.nv, 0);
            call_tl = 1;
        }
        const uint32_t call = call_tl;
        for (int64_t i = 0; i < nrel; i++)
            for (int k = 0; k < 3; k++) {
                const int64_t q = g.vi[g.off[rel[i]] + k];
                if (stamp[q] != call) {
                    stamp[q] = call;
                    vb[q] = nearest(R.v[3 * q], R.v[3 * q + 1]);
                }
            }
    }
#pragma omp parallel for schedule(static) if (par && nrel > 4096)
    for (int64_t i = 0; i < nrel; i++) {
        const int64_t f = rel_face(i);
        // the face as a blocker: its corners and edge normals in x, y
        Blocker &B = bl[f];
        for (int k = 0; k < 3; k++) {
            const double *v = &R.v[3 * g.vi[g.off[f] + k]];
            B.x[k] = v[0];
            B.y[k] = v[1];
        }
        for (int k = 0; k < 3; k++) {
            const int kn = k == 2 ? 0 : k + 1;
            B.en2[k] = -B.x[kn] + B.x[k];
            B.en1[k] = B.y[kn] - B.y[k];
        }
        B.z = R.mid[3 * f + 2];
        B.up = R.n[3 * f + 2] >= kLit0_01;
    }
    // bucket membership of those faces (bit b: a vertex in bucket b), and on small
    // meshes the members of every bucket in face order
    const bool use_grid = nrel >= grid_min_faces();
    if (!use_grid)
        for (int b = 0; b < kBB * kBB; b++) members[b].clear();
    for (int64_t i = 0; i < nrel; i++) {
        const int64_t f = rel_face(i);
        unsigned m = 0;
        for (int k = 0; k < 3; k++) m |= 1u << vb[g.vi[g.off[f] + k]];
        memb[f] = (uint16_t)m;
        if (!use_grid)
            for (; m; m &= m - 1) members[__builtin_ctz(m)].push_back(f);
    }
    // On large sets, a finer grid of the faces' outlines: cell c lists, in face
    // order, the faces whose bounding box (padded as above) meets it.  The
    // blockers of a centroid are the members of its bucket whose outline contains
    // it, all in the centroid's cell: the loop below visits the same faces in the
    // same order as a walk over the bucket's members, less the ones whose inside
    // test would fail.
    const int G = (int)std::min<int64_t>(128, std::max<int64_t>(4, (int64_t)sqrt((double)nrel / 2.0)));
    const double gx0 = mnx - pad, gy0 = mny - pad;
    const double csx = (mxx - mnx + 2 * pad) / G, csy = (mxy - mny + 2 * pad) / G;
    // (coordinates are at or above the padded origin, so truncation is the floor)
    auto cell_x = [&](double x) {
        const int c = (int)((x - gx0) / csx);
        return c < 0 ? 0 : (c >= G ? G - 1 : c);
    };
    auto cell_y = [&](double y) {
        const int c = (int)((y - gy0) / csy);
        return c < 0 ? 0 : (c >= G ? G - 1 : c);
    };
    thread_local std::vector<int> c_off_tl, c_rng_tl;
    thread_local std::vector<int64_t> c_item_tl;
    std::vector<int> &c_off = c_off_tl, &c_rng = c_rng_tl;
    std::vector<int64_t> &c_item = c_item_tl;
    if (use_grid) {
        c_off.assign((size_t)G * G + 1, 0);
        c_rng.resize(4 * nrel);
        for (int64_t i = 0; i < nrel; i++) {
            const Blocker &B = bl[rel_face(i)];
            const double x0 = std::min(std::min(B.x[0], B.x[1]), B.x[2]) - pad;
            const double x1 = std::max(std::max(B.x[0], B.x[1]), B.x[2]) + pad;
            const double y0 = std::min(std::min(B.y[0], B.y[1]), B.y[2]) - pad;
            const double y1 = std::max(std::max(B.y[0], B.y[1]), B.y[2]) + pad;
            int *r = &c_rng[4 * i];
            r[0] = cell_x(x0);
            r[1] = cell_x(x1);
            r[2] = cell_y(y0);
            r[3] = cell_y(y1);
            for (int a = r[0]; a <= r[1]; a++)
                for (int b = r[2]; b <= r[3]; b++) c_off[a * G + b + 1]++;
        }
        for (int c = 0; c < G * G; c++) c_off[c + 1] += c_off[c];
        c_item.resize(c_off[G * G]);
        thread_local std::vector<int> fill_tl;
        std::vector<int> &fill = fill_tl;
        fill.assign(c_off.begin(), c_off.end() - 1);
        for (int64_t i = 0; i < nrel; i++) {
            const int *r = &c_rng[4 * i];
            for (int a = r[0]; a <= r[1]; a++)
                for (int b = r[2]; b <= r[3]; b++) c_item[fill[a * G + b]++] = rel_face(i);
        }
    }
    for (int64_t f = 0; f < nf; f++) {
        const double nz = R.n[3 * f + 2];
        if (kind == VIS_INT ? nz >= 0 : nz <= 0) out.is_shad[f] = 1;
    }
    const double esign = kind == VIS_EXT ? -1.0 : 1.0;
#pragma omp parallel for schedule(dynamic, 64) if (par && nf > 256)
    for (int64_t m = 0; m < nf; m++) {
        if (!is_vis[m]) continue;
        const double apz = R.apn[3 * g.ap[m] + 2];
        const bool away = kind == VIS_INT ? apz > -kLit0_01 : apz < kLit0_01;
        if (away) {
            is_vis[m] = 0;
            if (kind == VIS_INC) out.in_beam[m] = 0;
            continue;
        }
        const double mx = R.mid[3 * m], my = R.mid[3 * m + 1], mz = R.mid[3 * m + 2];
        const int fb = nearest(mx, my);  // the centroid's bucket
        const unsigned bit = 1u << fb;
        const int cm = use_grid ? cell_x(mx) * G + cell_y(my) : 0;
        const int64_t nq = use_grid ? c_off[cm + 1] - c_off[cm] : (int64_t)members[fb].size();
        const int64_t *cand = use_grid ? &c_item[c_off[cm]] : members[fb].data();
        for (int64_t q = 0; q < nq; q++) {
            const int64_t j = cand[q];
            if (!(memb[j] & bit) || j == m) continue;  // not in m's bucket
            const Blocker &B = bl[j];
            if (kind == VIS_INC && !B.up) continue;  // down-facing blocker
            const double jz = B.z;
            if (mz > jz) continue;  // j behind m
            // m's centroid inside j's outline, edge by edge
            bool inside = true;
            for (int k = 0; k < 3 && inside; k++) {
                const double b1 = mx - B.x[k], b2 = my - B.y[k];
                if (esign * (b1 * B.en1[k] + b2 * B.en2[k]) > 0) inside = false;
            }
            if (!inside) continue;
            if (kind == VIS_INC) {
                if (g.ap[m] == g.ap[j]) {
                    out.is_shad[m] = 1;
                } else {
                    is_vis[m] = 0;
                    out.in_beam[m] = 0;
                }
                continue;
            }
            if (map[j] >= 0) {  // j emits this beam
                if (out.in_beam[m]) {
                    const double cz = R.mid[3 * beam.in[out.id_beam[m]].fi + 2];
                    if (jz < cz) {
                        out.id_beam[m] = map[j];
                        out.dist[m] = jz - mz;
                    }
                } else {
                    out.in_beam[m] = 1;
                    out.id_beam[m] = map[j];
                    out.dist[m] = jz - mz;
                }
            } else if (g.ap[m] != g.ap[j]) {  // another aperture in the way
                if (out.in_beam[m]) {
                    const double cz = R.mid[3 * beam.in[out.id_beam[m]].fi + 2];
                    if (jz > cz) continue;  // above the emitting surface
                }
                is_vis[m] = 0;
                out.in_beam[m] = 0;
                break;
            }
        }
    }
    if (kind == VIS_INC)
        for (int64_t m = 0; m < nf; m++)
            if (out.in_beam[m]) {
                out.dist[m] = kBeamZ - R.mid[3 * m + 2];
                out.id_beam[m] = 0;
            }
}

// Angle of refraction from medium m1 into m2 with complex indices: Macke's
// (1996) form of Snell's law for absorbing media, as get_theta_t_complex has
// it (src/beam_loop_mod.f90:342-383).  With kappa = Im/Re of each index, the
// relative index n_rel (1 + i kappa_rel) gives a complex
// c = 1 - sin^2(theta_i) (1 - kappa_rel^2 - 2 i kappa_rel) / (n_rel^2 (1 + kappa_rel^2)^2);
// the real effective index n_eff then satisfies sin(theta_t) = sin(theta_i) / n_eff.
// Operations in the reference's order.
double theta_t_complex(double theta_i, Z m1, Z m2) {
    const double kappa1 = m1.im / m1.re, kappa2 = m2.im / m2.re;
    const double kap_rel = (kappa2 - kappa1) / (1 + kappa1 * kappa2);
    const double n_rel = m2.re / m1.re * (1 + kappa1 * kappa2) / (1 + kappa1 * kappa1);
    const double n_rel2 = n_rel * n_rel, kap_rel2 = kap_rel * kap_rel;
    const double damp2 = (1 + kap_rel2) * (1 + kap_rel2);
    const double scale = n_rel2 * damp2 / (1 + kap_rel * kappa2) / (1 + kap_rel * kappa2);
    const double sin2_i = sin(theta_i) * sin(theta_i);
    const double c_re = 1 - (1 - kap_rel2) / n_rel2 / damp2 * sin2_i;
    const double c_im = 2 * kap_rel / n_rel2 / damp2 * sin2_i;
    const double c_abs2 = c_re * c_re + c_im * c_im;
    const double c_abs = sqrt(c_abs2);
    const double half_arg = acos(c_re / c_abs) / 2;
    const double proj = cos(half_arg) - kappa2 * sin(half_arg);
    const double proj2 = proj * proj;
    const double n_eff = sqrt(sin2_i + scale * c_abs * proj2);
    return asin(sin(theta_i) / n_eff);
}

// get_trans_prop (src/beam_loop_mod.f90:1010-1051)
void trans_prop(double theta_i, double theta_t, const double *prop_in, const double *norm,
                double *out) {
    const double alpha = kPiRef - theta_t;
    double a, b;
    if (theta_t < kLit1em5) {
        a = 0.25;
        b = 0.75;
    } else {
        a = sin(theta_t - theta_i) / sin(theta_i);
        b = sin(alpha) / sin(theta_i);
    }
    for (int k = 0; k < 3; k++) out[k] = b * prop_in[k] - a * norm[k];
    normalise3(out);
}

// get_rot_matrix (src/beam_loop_mod.f90:2611-2638)
void rot_matrix(const double *vk7, const double *ev1, const double *ev3, double r[2][2]) {
    const double c = dot3(vk7, ev1);
    double evo2[3];
    cross3(ev3, ev1, evo2, true);
    const double s = dot3(vk7, evo2);
    r[0][0] = c;
    r[0][1] = -s;
    r[1][0] = s;
    r[1][1] = c;
    const double det = r[0][0] * r[1][1] - r[0][1] * r[1][0];
    const double nrm = sqrt(fabs(det));
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) r[i][j] = r[i][j] / nrm;
}

inline Z expi(double x) { return {cos(x), sin(x)}; }

// Fresnel matrices for incidence from outside (facet angles), the forms of
// src/beam_loop_mod.f90:553-556 and :923-926
void fresnel_outside(double ti, double tt, Z m, Z fr[2][2], Z ft[2][2]) {
    const Z zero = {0.0, 0.0};
    fr[0][1] = fr[1][0] = ft[0][1] = ft[1][0] = zero;
    const Z ci = {cos(ti), 0.0}, ct = {cos(tt), 0.0};
    const Z mct = zmul(m, ct), mci = zmul(m, ci);
    const Z two_ci = {2 * cos(ti), 0.0};
    fr[1][1] = zdiv(zsub(ci, mct), zadd(ci, mct));
    ft[1][1] = zdiv(two_ci, zadd(ci, mct));
    fr[0][0] = zdiv(zsub(mci, ct), zadd(ct, mci));
    ft[0][0] = zdiv(two_ci, zadd(ct, mci));
}

struct Params {
    double lambda, rbi, ibi, thresh_area, thresh_energy;
    int64_t rec, refl;
    bool par;  // spread one orientation's work over the host threads
};

// recursion_inc (src/beam_loop_mod.f90:424-612): the incident beam on the
// lit faces; also the external-diffraction outbeams
void propagate_inc(const Shape &g, const Params &P, std::vector<FieldOut> &fo,
                   std::vector<pbt_outbeam> &ext) {
    const double waveno = 2 * kPiRef / P.lambda;
    const Z m_int = {P.rbi, P.ibi}, m_ext = {1.0, 0.0};
    Rotated R;
    R.v = g.v;
    R.mid = g.mid;
    R.n = g.n;
    R.apn = g.apn;
    Beam inc;
    inc.prop[0] = 0.0;
    inc.prop[1] = 0.0;
    inc.prop[2] = -1.0;
    Vis vis;
    find_vis(g, R, inc, VIS_INC, P.par, vis);
    const double prop[3] = {0.0, 0.0, -1.0}, e_perp_inc[3] = {1.0, 0.0, 0.0};
    for (int64_t i = 0; i < g.nf; i++) {
        if (!vis.in_beam[i]) continue;
        const int64_t ai = g.ap[i];
        const double *an = &g.apn[3 * ai], *ni = &g.n[3 * i];
        FieldOut o;
        o.fi = i;
        o.ap = ai;
        o.is_tir = false;
        o.prop_ext[0] = 0 + 2 * an[2] * an[0];
        o.prop_ext[1] = 0 + 2 * an[2] * an[1];
        o.prop_ext[2] = -1 + 2 * an[2] * an[2];
        cross3(ni, prop, o.e_perp, true);
        double rot2[2][2];
        rot_matrix(o.e_perp, e_perp_inc, prop, rot2);
        Amp ampl = amp_times(amp_identity(), expi(waveno * vis.dist[i]));
        ampl = rmatmul(rot2, ampl);
        const double theta_i = acos(an[2]);
        const double ti_f = vis.is_shad[i] ? theta_i : acos(ni[2]);
        const double tt_f = theta_t_complex(ti_f, m_ext, m_int);
        Z fr[2][2], ft[2][2];
        fresnel_outside(ti_f, tt_f, m_int, fr, ft);
        o.ampl_ext = zmatmul(fr, ampl);
        o.ampl_int = zmatmul(ft, ampl);
        const double int_i = intensity(o.ampl_int), ext_i = intensity(o.ampl_ext);
        const double theta_t = theta_t_complex(theta_i, m_ext, m_int);
        const double norm[3] = {-an[0], -an[1], -an[2]};
        trans_prop(theta_i, theta_t, prop, norm, o.prop_int);
        const double mn[3] = {-ni[0], -ni[1], -ni[2]};
        const double tt_f2 = acos(dot3(mn, o.prop_int));
        o.pr = ext_i * g.area[i] * cos(ti_f);
        o.pt = int_i * g.area[i] * P.rbi * cos(tt_f2);
        fo.push_back(o);
        pbt_outbeam e;
        // ampl(1,1), (2,1), (1,2), (2,2)
        const Z order[4] = {ampl.a[0][0], ampl.a[1][0], ampl.a[0][1], ampl.a[1][1]};
        for (int k = 0; k < 4; k++) {
            e.ampl[2 * k] = order[k].re;
            e.ampl[2 * k + 1] = order[k].im;
        }
        for (int k = 0; k < 3; k++) {
            e.vk7[k] = o.e_perp[k];
            e.prop_out[k] = prop[k];
        }
        e.fov = kPiRef / 2.0;
        e.fi = i + 1;
        ext.push_back(e);
    }
}

// recursion_int (src/beam_loop_mod.f90:614-812)
void propagate_int(const Shape &g, const Params &P, Beam &beam, std::vector<FieldOut> &fo) {
    const double waveno = 2 * kPiRef / P.lambda;
    const Z m_int = {P.rbi, P.ibi}, m_ext = {1.0, 0.0};
    const Mat3 rot = beam_rotation(beam.prop);
    thread_local Rotated R_tl;  // reused from beam to beam
    Rotated &R = R_tl;
    rotate_shape(g, rot, R);
    Vis vis;
    find_vis(g, R, beam, VIS_INT, P.par, vis);
    double prop_ext_prev[3] = {0.0, 0.0, 0.0};  // left over from the previous face on TIR
    for (int64_t i = 0; i < g.nf; i++) {
        if (!vis.in_beam[i]) continue;
        const int64_t ai = g.ap[i];
        const double *ran = &R.apn[3 * ai], *ni = &g.n[3 * i];
        const FieldIn &src = beam.in[vis.id_beam[i]];
        const double dist = vis.dist[i];
        FieldOut o;
        o.fi = i;
        o.ap = ai;
        double pr_[3] = {0 + 2 * ran[2] * ran[0], 0 + 2 * ran[2] * ran[1],
                         -1 + 2 * ran[2] * ran[2]};
        matT_vec(rot, pr_, o.prop_int);
        const double mni[3] = {-ni[0], -ni[1], -ni[2]};
        cross3(mni, beam.prop, o.e_perp, true);
        double rot2[2][2];
        rot_matrix(o.e_perp, src.e_perp, beam.prop, rot2);
        Amp ampl = rmatmul(rot2, src.ampl);
        ampl = amp_times(ampl, expi(waveno * P.rbi * dist));
        const double in_i = intensity(ampl);
        const double att = exp(-(2 * waveno * P.ibi * sqrt(dist)));
        const double abs_i = in_i * (1.0 - att * att);
        ampl = amp_scale(ampl, att);
        const double theta_i = acos(-ran[2]);
        const double ti_f = acos(-R.n[3 * i + 2]);
        Z fr[2][2], ft[2][2];
        const Z zero = {0.0, 0.0};
        fr[0][1] = fr[1][0] = ft[0][1] = ft[1][0] = zero;
        double theta_t = 0.0;
        if (beam.is_int && theta_i >= asin(1 / P.rbi)) {
            o.is_tir = true;
            fr[0][0] = fr[1][1] = {-1.0, 0.0};
            ft[0][0] = ft[1][1] = zero;
        } else {
            o.is_tir = false;
            theta_t = theta_t_complex(theta_i, m_int, m_ext);
            const Z ci = {cos(theta_i), 0.0}, ct = {cos(theta_t), 0.0};
            const Z mci = zmul(m_int, ci), mct = zmul(m_int, ct);
            const Z two_mci = zmul(zscale(2.0, m_int), ci);
            fr[1][1] = zdiv(zsub(mci, ct), zadd(mci, ct));
            ft[1][1] = zdiv(two_mci, zadd(mci, ct));
            fr[0][0] = zdiv(zsub(ci, mct), zadd(mct, ci));
            ft[0][0] = zdiv(two_mci, zadd(mct, ci));
        }
        o.ampl_int = zmatmul(fr, ampl);
        o.ampl_ext = zmatmul(ft, ampl);
        const double int_i = intensity(o.ampl_int), ext_i = intensity(o.ampl_ext);
        if (vis.is_shad[i]) o.ampl_ext = Amp{};  // a shadowed face transmits nothing
        beam.abs = beam.abs + abs_i * g.area[i] * cos(ti_f) * P.rbi;
        if (!o.is_tir) trans_prop(theta_i, theta_t, beam.prop, ni, prop_ext_prev);
        for (int k = 0; k < 3; k++) o.prop_ext[k] = prop_ext_prev[k];
        o.pr = int_i * g.area[i] * cos(ti_f) * P.rbi;
        o.pt = o.is_tir ? 0.0 : ext_i * g.area[i] * cos(theta_t);
        fo.push_back(o);
    }
}

// recursion_ext (src/beam_loop_mod.f90:814-1008); marks the beam's faces whose
// light hits the particle again as not outgoing
void propagate_ext(const Shape &g, const Params &P, Beam &beam, std::vector<FieldOut> &fo) {
    const double waveno = 2 * kPiRef / P.lambda;
    const Z m_int = {P.rbi, P.ibi}, m_ext = {1.0, 0.0};
    const Mat3 rot = beam_rotation(beam.prop);
    thread_local Rotated R_tl;  // reused from beam to beam
    Rotated &R = R_tl;
    rotate_shape(g, rot, R);
    Vis vis;
    find_vis(g, R, beam, VIS_EXT, P.par, vis);
    for (int64_t j = 0; j < g.nf; j++)
        if (vis.in_beam[j]) beam.in[vis.id_beam[j]].is_outgoing = false;
    for (int64_t i = 0; i < g.nf; i++) {
        if (!vis.in_beam[i]) continue;
        const int64_t ai = g.ap[i];
        const double *an = &g.apn[3 * ai], *ran = &R.apn[3 * ai], *ni = &g.n[3 * i];
        const FieldIn &src = beam.in[vis.id_beam[i]];
        FieldOut o;
        o.fi = i;
        o.ap = ai;
        o.is_tir = false;
        double pe[3] = {0 + 2 * ran[2] * ran[0], 0 + 2 * ran[2] * ran[1],
                        -1 + 2 * ran[2] * ran[2]};
        matT_vec(rot, pe, o.prop_ext);
        cross3(ni, beam.prop, o.e_perp, true);
        double rot2[2][2];
        rot_matrix(o.e_perp, src.e_perp, beam.prop, rot2);
        Amp ampl = rmatmul(rot2, src.ampl);
        ampl = amp_times(ampl, expi(waveno * vis.dist[i]));
        const double theta_i = acos(ran[2]);
        const double ti_f = acos(R.n[3 * i + 2]);
        const double tt_f = theta_t_complex(ti_f, m_ext, m_int);
        Z fr[2][2], ft[2][2];
        fresnel_outside(ti_f, tt_f, m_int, fr, ft);
        o.ampl_ext = zmatmul(fr, ampl);
        o.ampl_int = zmatmul(ft, ampl);
        const double int_i = intensity(o.ampl_int), ext_i = intensity(o.ampl_ext);
        const double theta_t = theta_t_complex(theta_i, m_ext, m_int);
        const double norm[3] = {-an[0], -an[1], -an[2]};
        trans_prop(theta_i, theta_t, beam.prop, norm, o.prop_int);
        const double mn[3] = {-ni[0], -ni[1], -ni[2]};
        const double tt_f2 = acos(dot3(mn, o.prop_int));
        o.pr = ext_i * g.area[i] * cos(ti_f);
        o.pt = int_i * g.area[i] * P.rbi * cos(tt_f2);
        fo.push_back(o);
    }
}

Beam new_beam(const Beam &parent, bool is_int) {
    Beam b;
    b.prop[0] = b.prop[1] = b.prop[2] = 0.0;
    b.is_int = is_int;
    b.rec = parent.rec + 1;
    b.refl = parent.refl;
    b.is_tir = false;
    b.abs = 0.0;
    return b;
}

// add_to_beam_tree_internal / _external (src/beam_loop_mod.f90:1053-1342):
// one internal and (unless totally internally reflected) one external child
// per aperture lit with enough area (and, from inside, enough energy)
void spawn(const Shape &g, const Params &P, const Beam &beam, bool parent_int,
           const std::vector<FieldOut> &fo, std::vector<Beam> &tree) {
    std::vector<double> ap_area(g.na, 0.0), ap_energy(g.na, 0.0);
    std::vector<char> tir(g.na, 0), create(g.na, 0);
    for (const FieldOut &o : fo) {
        ap_area[o.ap] = ap_area[o.ap] + g.area[o.fi];
        if (parent_int) ap_energy[o.ap] = ap_energy[o.ap] + o.pr;
        if (o.is_tir) tir[g.ap[o.fi]] = 1;
    }
    for (int64_t a = 0; a < g.na; a++)
        create[a] = parent_int ? (ap_area[a] > P.thresh_area && ap_energy[a] > P.thresh_energy)
                               : (ap_area[a] > P.thresh_area);
    std::vector<int64_t> slot(g.na, -1), nface(g.na, 0);
    for (const FieldOut &o : fo)
        if (create[o.ap]) nface[o.ap]++;
    for (int64_t a = 0; a < g.na; a++) {
        if (!create[a]) continue;
        slot[a] = (int64_t)tree.size();
        // each child's field list gets its final length at once (one allocation)
        tree.push_back(new_beam(beam, true));
        tree.back().in.reserve(nface[a]);
        if (!parent_int || !tir[a]) {
            tree.push_back(new_beam(beam, false));
            tree.back().in.reserve(nface[a]);
        }
    }
    for (const FieldOut &o : fo) {
        if (!create[o.ap]) continue;
        Beam &bi = tree[slot[o.ap]];
        FieldIn fi;
        fi.fi = o.fi;
        fi.ampl = o.ampl_int;
        for (int k = 0; k < 3; k++) fi.e_perp[k] = o.e_perp[k];
        fi.is_outgoing = false;
        bi.in.push_back(fi);
        for (int k = 0; k < 3; k++) bi.prop[k] = o.prop_int[k];
        if (parent_int && o.is_tir) {
            bi.refl = beam.refl + 1;
            bi.is_tir = true;
        }
        // total internal reflection is decided per aperture (its normal's
        // angle), so a face of a TIR aperture is TIR too and the external
        // child exists whenever this branch is taken
        if ((!parent_int || !o.is_tir) && slot[o.ap] + 1 < (int64_t)tree.size()) {
            Beam &be = tree[slot[o.ap] + 1];
            FieldIn fe;
            fe.fi = o.fi;
            fe.ampl = o.ampl_ext;
            for (int k = 0; k < 3; k++) fe.e_perp[k] = o.e_perp[k];
            fe.is_outgoing = true;
            be.in.push_back(fe);
            for (int k = 0; k < 3; k++) be.prop[k] = o.prop_ext[k];
        }
    }
}

// add_to_outbeam_tree (src/beam_loop_mod.f90:2745-2794)
void emit(const Shape &g, const Params &P, const Beam &beam, std::vector<pbt_outbeam> &out) {
    double area = 0.0;
    for (const FieldIn &f : beam.in) area = area + g.area[f.fi];
    const double d = 2 * sqrt(area / kPiRef);
    const double fov = P.lambda / d * 8;
    for (const FieldIn &f : beam.in) {
        if (!f.is_outgoing) continue;
        pbt_outbeam o;
        const Z order[4] = {f.ampl.a[0][0], f.ampl.a[1][0], f.ampl.a[0][1], f.ampl.a[1][1]};
        for (int k = 0; k < 4; k++) {
            o.ampl[2 * k] = order[k].re;
            o.ampl[2 * k + 1] = order[k].im;
        }
        for (int k = 0; k < 3; k++) {
            o.vk7[k] = f.e_perp[k];
            o.prop_out[k] = beam.prop[k];
        }
        o.fov = fov;
        o.fi = f.fi + 1;
        out.push_back(o);
    }
}

double outbeam_intensity(const pbt_outbeam &o) {
    double s = 0.0;
    const int order[4] = {0, 2, 1, 3};  // (1,1), (1,2), (2,1), (2,2)
    for (int k = 0; k < 4; k++) {
        const double re = o.ampl[2 * order[k]], im = o.ampl[2 * order[k] + 1];
        s = s + (re * re + im * im);
    }
    return 0.5 * s;
}

}  // namespace

struct pbt_particle {
    Shape g;
    double com[3];
};

struct pbt_trace {
    std::vector<pbt_outbeam> beam, ext;
    std::vector<double> verts;  // (nverts, 3) column-major, orientation frame
    pbt_trace_energy energy;
};

extern "C" int pbt_particle_create(const double *verts, int64_t nverts, const int64_t *face_off,
                                   const int64_t *face_vi, int64_t nfaces,
                                   const int64_t *face_ap, pbt_particle **out) {
    if (!out) {
        set_error("pbt_particle_create: NULL output handle");
        return PBT_EINVAL;
    }
    *out = nullptr;
    if (!verts || !face_off || !face_vi || nverts < 3 || nfaces < 1) {
        set_error("pbt_particle_create: need >= 3 vertices, >= 1 face and non-NULL arrays");
        return PBT_EINVAL;
    }
    if (face_off[0] != 0) {
        set_error("pbt_particle_create: face_off[0] must be 0");
        return PBT_EINVAL;
    }
    for (int64_t f = 0; f < nfaces; f++) {
        const int64_t n = face_off[f + 1] - face_off[f];
        if (n != 3) {
            set_error("pbt_particle_create: face %lld has %lld vertices (the tracer's visibility "
                      "test takes triangles)",
                      (long long)(f + 1), (long long)n);
            return PBT_EINVAL;
        }
    }
    for (int64_t q = 0; q < face_off[nfaces]; q++)
        if (face_vi[q] < 1 || face_vi[q] > nverts) {
            set_error("pbt_particle_create: face_vi[%lld] = %lld out of range 1..%lld",
                      (long long)q, (long long)face_vi[q], (long long)nverts);
            return PBT_EINVAL;
        }
    for (int64_t q = 0; q < 3 * nverts; q++)
        if (!isfinite(verts[q])) {
            set_error("pbt_particle_create: vertex coordinate %lld is not finite", (long long)q);
            return PBT_EINVAL;
        }
    std::unique_ptr<pbt_particle> p(new (std::nothrow) pbt_particle);
    if (!p) {
        set_error("pbt_particle_create: out of host memory");
        return PBT_ENOMEM;
    }
    Shape &g = p->g;
    g.nv = nverts;
    g.nf = nfaces;
    g.v.resize(3 * nverts);
    for (int64_t i = 0; i < nverts; i++)
        for (int c = 0; c < 3; c++) g.v[3 * i + c] = verts[i + nverts * c];
    g.off.assign(face_off, face_off + nfaces + 1);
    g.vi.resize(face_off[nfaces]);
    for (int64_t q = 0; q < face_off[nfaces]; q++) g.vi[q] = face_vi[q] - 1;
    g.ap.resize(nfaces);
    int64_t na = 0;
    for (int64_t f = 0; f < nfaces; f++) {
        // no aperture file: every face is its own aperture (src/input_mod.f90:2645-2648)
        const int64_t a = face_ap ? face_ap[f] : f + 1;
        if (a < 1) {
            set_error("pbt_particle_create: face %lld has aperture %lld (apertures are 1-based)",
                      (long long)(f + 1), (long long)a);
            return PBT_EINVAL;
        }
        g.ap[f] = a - 1;
        na = std::max(na, a);
    }
    g.na = na;
    std::vector<int64_t> used(na, 0);
    for (int64_t f = 0; f < nfaces; f++) used[g.ap[f]]++;
    for (int64_t a = 0; a < na; a++)
        if (!used[a]) {
            set_error("pbt_particle_create: aperture %lld has no faces", (long long)(a + 1));
            return PBT_EINVAL;
        }
    // src/input_mod.f90:2665-2680
    shape_midpoints(g);
    shape_areas(g);
    double com[3] = {0.0, 0.0, 0.0}, area = 0.0;
    for (int64_t f = 0; f < nfaces; f++) {
        for (int c = 0; c < 3; c++) com[c] = com[c] + g.mid[3 * f + c] * g.area[f];
        area = area + g.area[f];
    }
    for (int c = 0; c < 3; c++) {
        com[c] = com[c] / area;
        p->com[c] = com[c];
    }
    for (int64_t i = 0; i < nverts; i++)
        for (int c = 0; c < 3; c++) g.v[3 * i + c] = g.v[3 * i + c] - com[c];
    shape_midpoints(g);
    shape_normals(g);
    shape_apertures(g);
    for (int64_t f = 0; f < nfaces; f++)
        if (!isfinite(g.n[3 * f]) || !isfinite(g.n[3 * f + 1]) || !isfinite(g.n[3 * f + 2])) {
            set_error("pbt_particle_create: face %lld is degenerate (no normal)",
                      (long long)(f + 1));
            return PBT_EINVAL;
        }
    *out = p.release();
    return PBT_OK;
}

extern "C" int pbt_particle_info(const pbt_particle *p, int64_t *nverts, int64_t *nfaces,
                                 int64_t *napertures, double *com) {
    if (!p) {
        set_error("pbt_particle_info: NULL particle");
        return PBT_EINVAL;
    }
    if (nverts) *nverts = p->g.nv;
    if (nfaces) *nfaces = p->g.nf;
    if (napertures) *napertures = p->g.na;
    if (com)
        for (int c = 0; c < 3; c++) com[c] = p->com[c];
    return PBT_OK;
}

extern "C" int pbt_particle_verts(const pbt_particle *p, double *verts) {
    if (!p || !verts) {
        set_error("pbt_particle_verts: NULL argument");
        return PBT_EINVAL;
    }
    const int64_t nv = p->g.nv;
    for (int64_t i = 0; i < nv; i++)
        for (int c = 0; c < 3; c++) verts[i + nv * c] = p->g.v[3 * i + c];
    return PBT_OK;
}

extern "C" int pbt_particle_destroy(pbt_particle *p) {
    delete p;
    return PBT_OK;
}

namespace {

int check_trace_args(const pbt_particle *p, const double *euler, int64_t n,
                     const pbt_trace_params *prm, const char *who) {
    if (!p || (n > 0 && !euler) || !prm) {
        set_error("%s: NULL argument", who);
        return PBT_EINVAL;
    }
    if (!(prm->lambda > 0) || !isfinite(prm->lambda) || !(prm->rbi > 1.0) ||
        !isfinite(prm->rbi) || !(prm->ibi >= 0) || !isfinite(prm->ibi) || prm->rec < 0 ||
        prm->refl < 0 || !isfinite(prm->thresh_area) || !isfinite(prm->thresh_energy)) {
        set_error("%s: bad parameters (need lambda > 0, rbi > 1, ibi >= 0, rec >= 0, "
                  "refl >= 0, finite thresholds)",
                  who);
        return PBT_EINVAL;
    }
    for (int64_t k = 0; k < 3 * n; k++)
        if (!isfinite(euler[k])) {
            set_error("%s: Euler angle %lld of orientation %lld is not finite", who,
                      (long long)(k % 3 + 1), (long long)(k / 3 + 1));
            return PBT_EINVAL;
        }
    return PBT_OK;
}

Params make_params(const pbt_trace_params *prm, bool par) {
    Params P;
    P.lambda = prm->lambda;
    P.rbi = prm->rbi;
    P.ibi = prm->ibi;
    P.rec = prm->rec;
    P.refl = prm->refl;
    P.thresh_area = prm->thresh_area;
    P.thresh_energy = prm->thresh_energy;
    P.par = par;
    return P;
}

// One orientation: PROT_MPI, make_incident_beam, beam_loop_for_speed and
// energy_checks into tr.
int trace_one(const pbt_particle *p, const double *euler, const Params &P, pbt_trace *tr) {
    try {
        // PROT_MPI: rotate the vertices, recompute midpoints, normals, apertures
        Shape g = p->g;
        const Mat3 rot = euler_matrix(euler);
        for (int64_t i = 0; i < g.nv; i++) pbt::mv33(rot, &p->g.v[3 * i], &g.v[3 * i]);
        shape_midpoints(g);
        shape_normals(g);
        shape_apertures(g);
        // beam_loop_for_speed
        std::vector<FieldOut> fo_inc;
        propagate_inc(g, P, fo_inc, tr->ext);
        Beam inc;
        inc.prop[0] = 0.0;
        inc.prop[1] = 0.0;
        inc.prop[2] = -1.0;
        inc.is_int = false;
        inc.rec = 0;
        inc.refl = 0;
        inc.is_tir = false;
        inc.abs = 0.0;
        std::vector<Beam> tree;
        spawn(g, P, inc, false, fo_inc, tree);
        double geo = 0.0;  // get_geo_cross_section
        for (const FieldOut &o : fo_inc) geo = geo + g.area[o.fi] * g.n[3 * o.fi + 2];
        double abs_total = 0.0;
        size_t lo = 0;
        while (lo < tree.size()) {
            const size_t hi = tree.size();
            std::vector<std::vector<FieldOut>> fo(hi - lo);
            // many beams: one per thread; few: one at a time, each with
            // the visibility test spread over the threads
            const bool outer = P.par && hi - lo >= (size_t)omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) if (outer)
            for (size_t j = lo; j < hi; j++) {
                if (tree[j].is_int)
                    propagate_int(g, P, tree[j], fo[j - lo]);
                else
                    propagate_ext(g, P, tree[j], fo[j - lo]);
            }
            for (size_t j = lo; j < hi; j++) {
                // spawn appends to the tree, which may move its elements
                const Beam b = std::move(tree[j]);
                if (b.is_int) {
                    if (P.ibi > 0) abs_total = abs_total + b.abs;
                    if (b.rec < P.rec || (b.is_tir && b.refl < P.refl))
                        spawn(g, P, b, true, fo[j - lo], tree);
                } else {
                    if (b.rec < P.rec) spawn(g, P, b, false, fo[j - lo], tree);
                    emit(g, P, b, tr->beam);
                }
                if ((int64_t)tree.size() > kMaxBeams) {
                    set_error("tracer: beam tree exceeds %lld beams", (long long)kMaxBeams);
                    return PBT_ESTATE;
                }
            }
            lo = hi;
        }
        // energy_checks (src/beam_loop_mod.f90:1528-1624)
        double e_beam = 0.0, e_ext = 0.0;
        for (size_t i = 0; i < tr->beam.size(); i++) {
            const pbt_outbeam &o = tr->beam[i];
            const double oi = outbeam_intensity(o);
            if (isnan(oi)) {
                set_error("tracer: outbeam %lld has a NaN amplitude (a face normal parallel to "
                          "a beam direction leaves its e-perp undefined, e.g. an axis-aligned "
                          "orientation; the reference's 'euler' method lifts beta to 1e-4 "
                          "degree against this)",
                          (long long)(i + 1));
                return PBT_ESTATE;
            }
            const int64_t f = o.fi - 1;
            e_beam = e_beam + oi * g.area[f] * dot3(o.prop_out, &g.n[3 * f]);
        }
        for (const pbt_outbeam &o : tr->ext) {
            const int64_t f = o.fi - 1;
            e_ext = e_ext + outbeam_intensity(o) * g.area[f] * -dot3(o.prop_out, &g.n[3 * f]);
        }
        tr->energy.abs = abs_total;
        tr->energy.geo_cross_sec = geo;
        tr->energy.beam_energy_out = e_beam;
        tr->energy.ext_energy_out = e_ext;
        tr->energy.nbeams = (int64_t)tree.size();
        tr->verts.resize(3 * g.nv);
        for (int64_t i = 0; i < g.nv; i++)
            for (int c = 0; c < 3; c++) tr->verts[i + g.nv * c] = g.v[3 * i + c];
    } catch (const std::bad_alloc &) {
        set_error("tracer: out of host memory");
        return PBT_ENOMEM;
    }
    return PBT_OK;
}

}  // namespace

extern "C" int pbt_trace_orientation_c(const pbt_particle *p, const double *euler,
                                       const pbt_trace_params *prm, pbt_trace **out) {
    if (!out) {
        set_error("pbt_trace_orientation_c: NULL output handle");
        return PBT_EINVAL;
    }
    *out = nullptr;
    int st = check_trace_args(p, euler, 1, prm, "pbt_trace_orientation_c");
    if (st != PBT_OK) return st;
    std::unique_ptr<pbt_trace> tr(new (std::nothrow) pbt_trace);
    if (!tr) {
        set_error("pbt_trace_orientation_c: out of host memory");
        return PBT_ENOMEM;
    }
    st = trace_one(p, euler, make_params(prm, true), tr.get());
    if (st != PBT_OK) return st;
    *out = tr.release();
    return PBT_OK;
}

extern "C" int pbt_trace_batch_c(const pbt_particle *p, int64_t n, const double *euler,
                                 const pbt_trace_params *prm, pbt_trace **out) {
    if (!out || n < 0) {
        set_error("pbt_trace_batch_c: NULL output array or negative count");
        return PBT_EINVAL;
    }
    for (int64_t i = 0; i < n; i++) out[i] = nullptr;
    int st = check_trace_args(p, euler, n, prm, "pbt_trace_batch_c");
    if (st != PBT_OK) return st;
    const Params P = make_params(prm, false);
    std::vector<int> status(n, PBT_OK);
    std::vector<std::string> msg(n);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t i = 0; i < n; i++) {
        pbt_trace *tr = new (std::nothrow) pbt_trace;
        if (!tr) {
            status[i] = PBT_ENOMEM;
            msg[i] = "out of host memory";
            continue;
        }
        status[i] = trace_one(p, euler + 3 * i, P, tr);
        if (status[i] != PBT_OK) {
            msg[i] = pbt::last_error();
            delete tr;
        } else {
            out[i] = tr;
        }
    }
    for (int64_t i = 0; i < n; i++)
        if (status[i] != PBT_OK) {
            for (int64_t j = 0; j < n; j++) {
                delete out[j];
                out[j] = nullptr;
            }
            set_error("pbt_trace_batch_c: orientation %lld: %s", (long long)(i + 1),
                      msg[i].c_str());
            return status[i];
        }
    return PBT_OK;
}

extern "C" int pbt_trace_sizes(const pbt_trace *t, int64_t *nbeam, int64_t *next) {
    if (!t) {
        set_error("pbt_trace_sizes: NULL trace");
        return PBT_EINVAL;
    }
    if (nbeam) *nbeam = (int64_t)t->beam.size();
    if (next) *next = (int64_t)t->ext.size();
    return PBT_OK;
}

extern "C" int pbt_trace_copy(const pbt_trace *t, pbt_outbeam *beam, pbt_outbeam *ext,
                              double *verts, pbt_trace_energy *energy) {
    if (!t) {
        set_error("pbt_trace_copy: NULL trace");
        return PBT_EINVAL;
    }
    if (beam && !t->beam.empty()) memcpy(beam, t->beam.data(), t->beam.size() * sizeof(pbt_outbeam));
    if (ext && !t->ext.empty()) memcpy(ext, t->ext.data(), t->ext.size() * sizeof(pbt_outbeam));
    if (verts) memcpy(verts, t->verts.data(), t->verts.size() * sizeof(double));
    if (energy) *energy = t->energy;
    return PBT_OK;
}

extern "C" int pbt_trace_destroy(pbt_trace *t) {
    delete t;
    return PBT_OK;
}
