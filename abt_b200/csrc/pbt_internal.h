// pbt_internal.h -- shared declarations of the library's host and device code.
#pragma once
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <stdint.h>

#include <mutex>
#include <string>
#include <vector>

#include "../../include/pbt_diff.h"

namespace pbt {

// A named NVTX range over a host-side stage (set-up, far-field sum, epilogue,
// finalise, adjoint), the counterpart of the reference's timing spans
// (src/diff_mod.f90:705-707, 740-742, 810-822).  NVTX is header-only and costs
// nothing unless a profiler is attached.
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

// ------------------------------------------------------------------ errors
void set_error(const char *fmt, ...);
void clear_error();
const char *last_error();

#define PBT_CUDA_TRY(call)                                                                  \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess) {                                                            \
            ::pbt::set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_),        \
                             __FILE__, __LINE__);                                           \
            return e_ == cudaErrorMemoryAllocation ? PBT_ENOMEM : PBT_ECUDA;                \
        }                                                                                   \
    } while (0)

#define PBT_TRY(call)                     \
    do {                                  \
        int rc_ = (call);                 \
        if (rc_ != PBT_OK) return rc_;    \
    } while (0)

// ------------------------------------------------------------ device memory
// Grow-only device buffer owned by a context.
// Restores the calling thread's current device when an entry point returns
// (entry points make their context's device current while they run).
struct DeviceRestore {
    int prev = -1;
    DeviceRestore() {
        if (cudaGetDevice(&prev) != cudaSuccess) {
            prev = -1;
            (void)cudaGetLastError();
        }
    }
    ~DeviceRestore() {
        if (prev >= 0) (void)cudaSetDevice(prev);
    }
    DeviceRestore(const DeviceRestore &) = delete;
    DeviceRestore &operator=(const DeviceRestore &) = delete;
};

struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
    int ensure(size_t bytes);
    void release();
    template <class T>
    T *as() const { return static_cast<T *>(p); }
};

// Grow-only pinned host staging buffer.
struct HostBuf {
    void *p = nullptr;
    size_t cap = 0;
    int ensure(size_t bytes);
    void release();
    template <class T>
    T *as() const { return static_cast<T *>(p); }
};

// ------------------------------------------- reference-exact FP64 records
// One outgoing facet, prepared for the FP64 kernel (all values formed in the
// reference's operation order).  272 bytes.
struct K1Facet {
    double com[3];
    double R[9];      // matmul(rot2, rot), row-major
    double prop2[3];
    double inc2[3];
    double kinc[2];   // prop2(1:2) * waveno  (src/diff_mod.f90:336)
    double ampl[8];   // amplitude after the anti-parallel flip: (1,1),(2,1),(1,2),(2,2) re/im
    double prop0[3];  // lab-frame propagation (field-of-view test)
    double cos_fov;
    int64_t edge_off;
    int64_t nv;
};
static_assert(sizeof(K1Facet) == 272, "K1Facet layout");

// One aperture edge after the slope clamps of src/diff_mod.f90:379-393.
struct K1Edge {
    double xj, yj, mj, nj, dx, dy;
};

// Far-field bin grid cached per (theta, phi) list.
struct GridCache {
    std::vector<double> theta, phi;  // radians, as given
    int64_t nb = 0;
    int64_t theta_i = -1;            // first theta above 1 degree (0-based), -1 if none
    int64_t back_i = 0;              // minloc(|theta - 2 pi|)
    DevBuf xyz;                      // xfar | yfar | zfar  (nb each), libm values
    DevBuf phitab;                   // cos(phi) | sin(phi)  (nphi each), libm values
    DevBuf thtab;                    // sin(theta) | cos(theta) (ntheta each), libm values
    DevBuf wbin;                     // simpne weights w_phi(i) * w_theta(j) * sin(theta_j)  (nb)
    DevBuf wphi;                     // simpne weights over phi (nphi)
    // is_fast_diff bin tiles: (theta x phi) blocks of fast_tile bins
    int64_t fast_tile = 0, fast_ntiles = 0;
    DevBuf fast_perm;                // tile-major bin indices (int32, -1 = padding)
    DevBuf fast_cone;                // K2Cone per tile
    bool valid = false;
};

// Device running totals of summation (src/outputs_mod.f90:407-471).
struct DevTotals {
    DevBuf mu, m1, par;  // (nphi,ntheta,16) | (ntheta,16) | 18 params
    int64_t ntheta = 0, nphi = 0, count = 0;
    void release() {
        mu.release();
        m1.release();
        par.release();
    }
};

}  // namespace pbt

struct pbt_ctx {
    int device = 0;
    std::mutex mu;
    cudaStream_t stream = nullptr;   // internal stream of the host-pointer entry points
    cudaStream_t copy_stream = nullptr;       // uploads of the next orientation run (batch)
    cudaEvent_t up_ev[2] = {nullptr, nullptr};    // run uploaded into slot i
    cudaEvent_t done_ev[2] = {nullptr, nullptr};  // compute done with slot i
    std::vector<char> h_gather;                // host gather buffer of one batch run
    pbt::GridCache grid;
    // scratch (grow-only)
    pbt::DevBuf d_fac, d_edge, d_out, d_mu, d_m1, d_misc, d_in, d_rec, d_ws, d_scan, d_items;
    pbt::DevBuf d_tk;  // split tickets of the FP32 kernel's (segment, tile) pairs
    pbt::DevBuf d_k1part;  // FP64 drop-in: partial grids of the facet splits (small grids)
    pbt::HostBuf h_stage;
    cudaEvent_t stage_ev = nullptr;  // last copy out of h_stage (wait before reuse)
    bool stage_pending = false;
    pbt::DevTotals tot;    // user-visible totals (pbt_summation_c / pbt_finalise_c accumulate)
    pbt::DevTotals btot;   // totals of the FP64 batch path
    int64_t launches = 0;            // kernel launches of the last compute call
    int sm_count = 0;
    // launch plan of the FP32 main kernel (-1: default / PBT_K2_PLAN)
    int plan_variant = -1, plan_bpt = 1;
    int64_t plan_rpi = 2048;
    // CUDA-event timing of the far-field kernels
    bool timing = false;
    std::vector<cudaEvent_t> ev;  // start/stop pairs
    // set while a graph captures this context's enqueue: no host waits, no events
    bool capturing = false;
    size_t ev_used = 0;
};

namespace pbt {

// ----------------------------------------------------------- host helpers
int validate_geometry(const double *verts, int64_t nverts, const int64_t *face_off,
                      const int64_t *face_vi, int64_t nfaces);
int validate_angles(const double *theta, int64_t ntheta, const double *phi, int64_t nphi);
int grid_prepare(pbt_ctx *ctx, const double *theta, int64_t ntheta, const double *phi,
                 int64_t nphi, cudaStream_t st);

// Reference-exact facet set-up on the host (libm).  Appends to fac/edges.
int k1_build_facets(const pbt_outbeam *obs, int64_t n, double fov_override, const double *verts,
                    int64_t nverts, const int64_t *face_off, const int64_t *face_vi,
                    int64_t nfaces, double lambda, std::vector<K1Facet> &fac,
                    std::vector<K1Edge> &edges);

// FP64 far-field sum of nf facets into a complex (nphi,ntheta,2,2) grid (overwritten).
int k1_launch(pbt_ctx *ctx, cudaStream_t st, const K1Facet *d_fac, int64_t nf,
              const K1Edge *d_edges, double lambda, int fast_diff, double *d_grid);

// Reference-exact finalise on device grids.  Writes mueller (nb*16),
// mueller_1d (ntheta*16) and params (18 doubles) to device memory; adds to the
// context totals when accumulate.
int k3_finalise(pbt_ctx *ctx, cudaStream_t st, const double *d_afb, const double *d_afe,
                double lambda, int scaling, const pbt_output_params *h_params_in,
                double *d_mueller, double *d_m1d, double *d_params, DevTotals *acc);
int totals_ensure(DevTotals &T, int64_t ntheta, int64_t nphi, cudaStream_t st);
int totals_reset(DevTotals &T, cudaStream_t st);
int totals_add_device(pbt_ctx *ctx, DevTotals &T, cudaStream_t st, const double *d_mueller,
                      const double *d_m1d, const double *d_params);

// Batched FP32 path.  h_beam_off / h_ext_off / h_face_off are host arrays,
// every other pointer is device memory.
// Batched FP32 average in steps (k2_batch_impl = begin + one add + finish).
struct K2Plan {
    int variant = 1;   // 0: one record per step, 1: two records packed (FP32x2)
    int bpt = 1;       // bins per thread
    int64_t rpi = 2048;  // facet records per work item
    bool auto_rpi = true;  // default plan: rpi sized per call from the records and bin tiles
};
struct K2Batch {
    int64_t norient = 0, wchunk = 1;
    K2Plan plan;
    double *ws = nullptr;
    double *mu_sum = nullptr, *redo = nullptr, *bs = nullptr, *scale = nullptr;
    double *part = nullptr;  // per-block partial sums of the epilogue (6 per orientation and block)
    pbt_output_params *pp = nullptr;
    int64_t *seg_rec = nullptr, *item_pre = nullptr;
    unsigned long long *counter = nullptr;
    int *err = nullptr;
};
int k2_batch_begin(pbt_ctx *ctx, cudaStream_t st, int64_t norient, int64_t max_run,
                   const pbt_output_params *d_params_per, K2Batch &B);
int k2_batch_add(pbt_ctx *ctx, cudaStream_t st, K2Batch &B, int64_t o0, int64_t no,
                 const pbt_outbeam *d_beam, const int64_t *h_beam_off, const pbt_outbeam *d_ext,
                 const int64_t *h_ext_off, const double *d_verts, int64_t nverts,
                 const int64_t *h_face_off, const int64_t *d_face_off, const int64_t *d_face_vi,
                 int64_t nfaces, double lambda, int fast_diff, int scaling,
                 const pbt_output_params *d_params_in);
int k2_batch_finish(pbt_ctx *ctx, cudaStream_t st, K2Batch &B, const pbt_output_params *d_params_in,
                    double *d_mueller_avg, double *d_m1d_avg, pbt_output_params *d_params_avg,
                    int check_errors);
int k2_batch_impl(pbt_ctx *ctx, cudaStream_t st, int64_t norient, const pbt_outbeam *d_beam,
                  const int64_t *h_beam_off, const pbt_outbeam *d_ext, const int64_t *h_ext_off,
                  const double *d_verts, int64_t nverts, const int64_t *h_face_off,
                  const int64_t *d_face_off, const int64_t *d_face_vi, int64_t nfaces,
                  double lambda, int fast_diff, int scaling, const pbt_output_params *d_params_in,
                  double *d_mueller_avg, double *d_m1d_avg, pbt_output_params *d_params_avg,
                  pbt_output_params *d_params_per, int check_errors);

// FP32 single-orientation amplitude grids (the fast diff_main).
int k2_diff_main_impl(pbt_ctx *ctx, cudaStream_t st, const pbt_outbeam *d_beam, int64_t nbeam,
                      const pbt_outbeam *d_ext, int64_t next, const double *d_verts, int64_t nverts,
                      const int64_t *h_face_off, const int64_t *d_face_off,
                      const int64_t *d_face_vi, int64_t nfaces, double lambda, int fast_diff,
                      double *d_afb, double *d_afe);
int k2_check_err(pbt_ctx *ctx, cudaStream_t st, const int *d_err);
// Launches a bounded wait that nothing completes (the failure-detection self-test).
int k2_wait_selftest(pbt_ctx *ctx, cudaStream_t st, uint64_t limit_ns);
int totals_divide_device(pbt_ctx *ctx, DevTotals &T, cudaStream_t st, int64_t num_orients,
                         double *d_mu, double *d_m1, double *d_p);
int validate_outbeams(const pbt_outbeam *obs, int64_t n, int64_t nfaces, const char *what);
// Bracket a far-field kernel launch with timing events (no-op unless enabled).
void timing_begin(pbt_ctx *ctx, cudaStream_t st);
void timing_end(pbt_ctx *ctx, cudaStream_t st);

}  // namespace pbt
