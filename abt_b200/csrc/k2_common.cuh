// k2_common.cuh -- record layout and device helpers of the batched FP32 path.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pbt {

// One triangular aperture prepared for the FP32 far-field sum.  A polygon
// facet becomes nv-2 records (a fan from its first vertex) that share the
// facet's centre of mass and aperture frame, so their sum is the polygon's
// contour integral.  176 bytes, a multiple of 16 for 1-D bulk copies.
struct __align__(16) K2Rec {
    double kc[3];    // k * com (lab frame), FP64: the far-field phase k r.c
    float eps[3];    // com / R
    float b;         // |com|^2 / R^2
    float R[9];      // lab -> aperture frame rotation, row-major
    float ea[3];     // R * com / R
    float kp[2];     // k * prop2 (x, y)
    float hkz_cf;    // -0.5 Kz / sqrt(1 - Ky^2)
    float hicf;      // 0.5 sqrt(1 - Ky^2)
    float hkxky_cf;  // 0.5 Kx Ky / sqrt(1 - Ky^2)
    float inc[3];    // incidence direction (0,0,-1) in the aperture frame
    float vx[3];     // triangle vertices (aperture frame, relative to com)
    float vy[3];
    float amp[8];    // (2 i A / lambda) * sign * ampl, (1,1),(2,1),(1,2),(2,2) re/im
};
static_assert(sizeof(K2Rec) == 176, "K2Rec must be 176 bytes");

// Per-record field-of-view test data (is_fast_diff only): prop0 and cos(fov)
// for the per-bin test; fovm = fov + a parallax margin with its cosine and
// sine for the per-tile cull (a tile whose cone lies beyond fovm is skipped).
// When the FP32 per-bin test is within tol of the threshold the FP64 test of
// the reference (facet centre com, prop0, cos(fov)) decides, with the same
// rounding as the FP64 drop-in.
struct __align__(16) K2Fov {
    float p0[3];
    float cos_fov;
    float cos_fovm, sin_fovm, fovm, tol;
    double com[3], p0d[3], cos_fovd, pad;
};
static_assert(sizeof(K2Fov) == 96, "K2Fov must be 96 bytes");

// Cone of a bin tile (is_fast_diff only): unit centre direction and the
// largest angle psi of a tile bin from it.
struct __align__(16) K2Cone {
    float c[3];
    float psi;
    float cos_psi, sin_psi, pad[2];
};
static_assert(sizeof(K2Cone) == 32, "K2Cone must be 32 bytes");

}  // namespace pbt

namespace pbt {

// Two triangle records interleaved field by field (x = even record, y = odd
// record), so that a shared-memory load of a float2 yields the operand pair of
// a packed FP32x2 instruction evaluating two facets at once.  The packed kernel
// works with half phases (kc and kp are halved) and with the Karczewski-Wolf
// block divided by its factor sqrt(1 - Ky^2) / 2, which goes into the
// amplitudes together with the 1/2 of the half-phase divided difference.
// Every pair of adjacent float2 fields from eps on starts on a 16-byte
// boundary, so the kernel reads them two at a time.  336 bytes.
struct __align__(16) K2Pair {
    double kc[3][2];  // k * com / 2, [component][half]
    float2 eps[3];
    float2 b;
    float2 R[9];
    float2 nea[3];    // -R * com / R
    float2 kp[2];     // k * prop2 (x, y) / 2
    float2 kzc;       // -Kz / (1 - Ky^2)
    float2 inc[3];
    float2 vx[3], vy[3];
    float2 amp[8];    // the amplitude columns in the circular basis, u+_1, u-_1, u+_2, u-_2
                      // (u+- = a1c +- i a2c of K2Rec::amp) times sqrt(1 - Ky^2) / 4, re/im
};
static_assert(sizeof(K2Pair) == 336, "K2Pair must be 336 bytes");

}  // namespace pbt
