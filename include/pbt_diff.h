/*
 * pbt_diff.h -- C ABI of the B200 far-field diffraction library (libpbt_b200.so).
 *
 * Drop-in replacement for PBT's far-field stage: diff_mod (diffraction,
 * diff_main) and the outputs_mod epilogue (finalise, summation,
 * divide_by_num_orientations).  Every entry point is extern "C", takes plain
 * pointers and sizes, and returns an int status (PBT_OK = 0).  A non-zero
 * status leaves a message for pbt_last_error_string() in the calling thread.
 *
 * Array layouts are the reference's Fortran layouts, so a Fortran caller can
 * pass its arrays unchanged through iso_c_binding:
 *   amplitude grid  complex(8) ampl(nphi, ntheta, 2, 2), column-major,
 *                   element (i,j,a,b) at 2*((i-1)+nphi*((j-1)+ntheta*((a-1)+2*(b-1)))) doubles
 *   Mueller grid    real(8) mueller(nphi, ntheta, 16), column-major
 *   1-D Mueller     real(8) mueller_1d(ntheta, 16), column-major
 *   vertices        real(8) v(nverts, 3), column-major (geometry%v)
 *   faces           CSR: face_off(nfaces+1) 0-based offsets into face_vi,
 *                   face_vi 1-based vertex indices (geometry%f(:)%vi)
 *   angles          theta_vals / phi_vals in radians (job_params%theta_vals, %phi_vals)
 *
 * Citations are path:line inside the reference project (hballington12/abt).
 */
#ifndef PBT_DIFF_H
#define PBT_DIFF_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define PBT_OK 0
#define PBT_EINVAL 1   /* bad argument: sizes, indices, null pointers, non-finite input */
#define PBT_ENOMEM 2   /* device or pinned-host allocation failed */
#define PBT_ECUDA 3    /* a CUDA call failed */
#define PBT_ETIMEOUT 4 /* a bounded device-side wait ran out; results not written */
#define PBT_ENODEV 5   /* no usable sm_100 device */
#define PBT_ESTATE 6   /* call out of order (e.g. totals of an empty accumulation) */

/* arithmetic of the far-field sum */
#define PBT_PREC_FP64 0 /* reference-exact FP64 (the plain drop-in) */
#define PBT_PREC_FP32 1 /* FP32 with the far-field phase formed and range-reduced in FP64 */

/* One outgoing facet: the fields of outbeamtype (src/types_mod.f90:8-17) that
 * diffraction reads (src/diff_mod.f90:515-531).  128 bytes. */
typedef struct pbt_outbeam {
    double ampl[8];     /* ampl(1:2,1:2) complex(8) column-major: (1,1),(2,1),(1,2),(2,2), re/im */
    double vk7[3];      /* perpendicular e-field direction */
    double prop_out[3]; /* outgoing propagation direction */
    double fov;         /* field of view (rad), used when is_fast_diff */
    int64_t fi;         /* 1-based face index into the face CSR */
} pbt_outbeam;

/* output_parameters_type (src/types_mod.f90:32-53), same component order.
 * Inputs to finalise: abs, geo_cross_sec, beam_energy_out, ext_energy_out. */
typedef struct pbt_output_params {
    double abs, scatt, ext, albedo, asymmetry, abs_eff, scatt_eff, ext_eff, geo_cross_sec,
        back_scatt, beam_energy_out, ext_energy_out, scatt_beam, scatt_ext_diff, asymmetry_beam,
        asymmetry_ext_diff, scatt_eff_beam, scatt_eff_ext_diff;
} pbt_output_params;

typedef struct pbt_ctx pbt_ctx;

/* ---------------------------------------------------------------- lifecycle */

/* Create a context bound to CUDA device `device`.  The context owns device
 * buffers reused across calls; it is safe to share between host threads
 * (calls are serialised on an internal mutex).  PBT_DEVICE_LOCAL_RANK picks the
 * device from the process's node-local rank, as an MPI launcher (the
 * reference's MPI build, src/pbt_mpi_mod.f90) or torchrun exports it
 * (LOCAL_RANK, OMPI_COMM_WORLD_LOCAL_RANK, MV2_COMM_WORLD_LOCAL_RANK,
 * MPI_LOCALRANKID, SLURM_LOCALID or PMI_LOCAL_RANK, the first one set; 0 when
 * none is) modulo the number of visible devices, so that the ranks of one node
 * spread over its GPUs. */
#define PBT_DEVICE_LOCAL_RANK (-1)
int pbt_ctx_create(int device, pbt_ctx **out);
/* The CUDA device the context is bound to. */
int pbt_ctx_device(const pbt_ctx *ctx, int *device);
int pbt_ctx_destroy(pbt_ctx *ctx);
/* Message of the last failed call made by this thread ("" if none). */
const char *pbt_last_error_string(void);
/* ABI version: major*10000 + minor*100 + patch. */
int pbt_version(void);

/* --------------------------------------------------------------- diff_mod */

/* diff_main replacement, src/diff_mod.f90:674-825.
 * Sums every beam outbeam into ampl_far_beam and every external-diffraction
 * outbeam (with fov forced to pi/2, src/diff_mod.f90:797) into
 * ampl_far_ext_diff.  precision = PBT_PREC_FP64 reproduces the reference's
 * arithmetic (facet order 1..n, no FMA); PBT_PREC_FP32 is the fast form.
 * Both output grids are overwritten. */
int pbt_diff_main_c(pbt_ctx *ctx, const pbt_outbeam *beam, int64_t nbeam,
                    const pbt_outbeam *ext, int64_t next, const double *verts, int64_t nverts,
                    const int64_t *face_off, const int64_t *face_vi, int64_t nfaces,
                    const double *theta, int64_t ntheta, const double *phi, int64_t nphi,
                    double lambda, int32_t is_fast_diff, int32_t precision,
                    double *ampl_far_beam, double *ampl_far_ext_diff);

/* diffraction replacement, src/diff_mod.f90:446-672: the far-field amplitude
 * of one outbeam, as used by the -memory path (src/beam_loop_mod.f90:44,71).
 * amplC is overwritten (zero outside the field of view when is_fast_diff).
 * FP64, reference-exact. */
int pbt_diffraction_c(pbt_ctx *ctx, const pbt_outbeam *outbeam, const double *verts,
                      int64_t nverts, const int64_t *face_off, const int64_t *face_vi,
                      int64_t nfaces, const double *theta, int64_t ntheta, const double *phi,
                      int64_t nphi, double lambda, int32_t is_fast_diff, double *amplC);

/* make_far_field_bins, src/diff_mod.f90:827-855: the far-field points
 * X = R (sin t cos p, sin t sin p, -cos t), R = 1e6, for every (phi, theta),
 * written as xfar/yfar/zfar(nphi, ntheta) column-major (phi fastest), with the
 * platform libm as the reference computes them.  Host only. */
int pbt_make_far_field_bins_c(const double *theta, int64_t ntheta, const double *phi,
                              int64_t nphi, double *xfar, double *yfar, double *zfar);

/* pbt_diffraction_c for callers that cannot let a library allocate memory.
 * No counterpart in the reference.  Programs whose device memory is reserved
 * up front by their own pool allocator, or that may allocate nothing after
 * start-up, can call this instead: it computes the same FP64 amplitude of one
 * outbeam but keeps its device scratch in one fixed array built into the
 * library (about 5.6 MB on every GPU that loads it, held until exit) and
 * calls no allocation routine; it needs no context.  Limits: at most
 * PBT_NOALLOC_MAX_BINS bins (ntheta * nphi), PBT_NOALLOC_MAX_PHI phi values
 * and PBT_NOALLOC_MAX_VERTS vertices per face; larger inputs return
 * PBT_EINVAL.  The first call on a device loads the library's device code
 * there and commits the array, which makes the CUDA runtime allocate device
 * memory (and may create the device's primary context): make the first call
 * at start-up, before a pool reserves the device's memory and outside any
 * stream capture, or run with CUDA_MODULE_LOADING=EAGER.  Every call looks up
 * the array's address on the current device and runs on the calling thread's
 * per-thread default stream (cudaStreamPerThread), waiting for its work.  All
 * calls on a device share the array; calls in one process are serialised and
 * complete before returning, and calls that overlapped on the GPU would race.
 * The bin grid stays in the array: a call whose theta and phi are the same,
 * bit for bit, as the previous call's builds and uploads no grid (a tag stored
 * beside the grid, read back each call, tells whether this device holds it). */
#define PBT_NOALLOC_MAX_BINS 65536
#define PBT_NOALLOC_MAX_PHI 4096
#define PBT_NOALLOC_MAX_VERTS 64
int pbt_diffraction_noalloc_c(const pbt_outbeam *outbeam, const double *verts, int64_t nverts,
                              const int64_t *face_off, const int64_t *face_vi, int64_t nfaces,
                              const double *theta, int64_t ntheta, const double *phi,
                              int64_t nphi, double lambda, int32_t is_fast_diff, double *amplC);

/* Gradients of the FP32 far-field sum of one orientation: the vector-Jacobian
 * product of pbt_diff_main_c with PBT_PREC_FP32.  No counterpart in the
 * reference (it has no derivatives).  Inputs as pbt_diff_main_c plus the
 * cotangents of its two output grids (dL/dRe + i dL/dIm, reference layout);
 * outputs dL/dverts (nverts,3) and dL/dampl per outbeam (8 doubles, re/im of
 * ampl(1,1),(2,1),(1,2),(2,2)).  The beam topology (which facets emit, their
 * directions, anti-parallel sign and field-of-view masks) is held fixed.
 * Triangular facets only.  Phase terms are recomputed per facet x bin; no
 * facet x bin intermediate is stored. */
int pbt_diff_adjoint_c(pbt_ctx *ctx, const pbt_outbeam *beam, int64_t nbeam,
                       const pbt_outbeam *ext, int64_t next, const double *verts, int64_t nverts,
                       const int64_t *face_off, const int64_t *face_vi, int64_t nfaces,
                       const double *theta, int64_t ntheta, const double *phi, int64_t nphi,
                       double lambda, int32_t is_fast_diff, const double *grad_ampl_far_beam,
                       const double *grad_ampl_far_ext_diff, double *grad_verts,
                       double *grad_beam_ampl, double *grad_ext_ampl);

/* ------------------------------------------------------------ outputs_mod */

/* finalise replacement, src/outputs_mod.f90:63-278 (FP64, reference order).
 * params: in abs, geo_cross_sec, beam_energy_out, ext_energy_out; out all.
 * The amplitude grids are read only (the reference scales its copies in
 * place; the library does not).  When accumulate != 0 the orientation's
 * mueller, mueller_1d and params are also added to the context's device
 * totals (summation, src/outputs_mod.f90:407-471).  mueller / mueller_1d
 * may be NULL when only the totals are wanted. */
int pbt_finalise_c(pbt_ctx *ctx, const double *ampl_far_beam, const double *ampl_far_ext_diff,
                   const double *theta, int64_t ntheta, const double *phi, int64_t nphi,
                   double lambda, int32_t scaling, pbt_output_params *params, double *mueller,
                   double *mueller_1d, int32_t accumulate);

/* summation replacement, src/outputs_mod.f90:407-471: adds one orientation's
 * results (host arrays) to the context's device totals. */
int pbt_summation_c(pbt_ctx *ctx, const double *mueller, const double *mueller_1d,
                    const pbt_output_params *params, int64_t ntheta, int64_t nphi);

/* divide_by_num_orientations, src/outputs_mod.f90:13-43, applied to copies of
 * the device totals (the totals are left unchanged). */
int pbt_divide_by_num_orientations_c(pbt_ctx *ctx, int64_t num_orients, double *mueller_total,
                                     double *mueller_1d_total, pbt_output_params *params_total);

/* Zero the device totals (start of a new orientation average). */
int pbt_totals_reset_c(pbt_ctx *ctx);

/* -------------------------------------------------------- batched averaging */

/* Orientation averaging in one call: the per-orientation loop of
 * src/pbt_seq_mod.f90:146-269 from diff_main through summation, then
 * divide_by_num_orientations (src/pbt_seq_mod.f90:274).
 *   beam / ext        outbeams of all orientations, orientation-major; the
 *                     outbeams of orientation o are beam[beam_off[o] .. beam_off[o+1])
 *   verts             norient consecutive v(nverts,3) blocks (each orientation's
 *                     rotated geometry; topology shared)
 *   params_in         norient records (abs, geo_cross_sec, beam/ext energy)
 *   mueller_avg       (nphi,ntheta,16) orientation average
 *   mueller_1d_avg    (ntheta,16) orientation average
 *   params_avg        averaged parameters
 *   params_per_orient optional (NULL), norient records
 * PBT_PREC_FP32 runs the batched FP32 kernel over all orientations with an
 * FP64 epilogue; PBT_PREC_FP64 runs the reference-exact path per orientation. */
int pbt_diff_batch_c(pbt_ctx *ctx, int64_t norient, const pbt_outbeam *beam,
                     const int64_t *beam_off, const pbt_outbeam *ext, const int64_t *ext_off,
                     const double *verts, int64_t nverts, const int64_t *face_off,
                     const int64_t *face_vi, int64_t nfaces, const double *theta, int64_t ntheta,
                     const double *phi, int64_t nphi, double lambda, int32_t is_fast_diff,
                     int32_t scaling, int32_t precision, const pbt_output_params *params_in,
                     double *mueller_avg, double *mueller_1d_avg, pbt_output_params *params_avg,
                     pbt_output_params *params_per_orient);

/* Same as pbt_diff_batch_c with each orientation in its own host arrays (no
 * counterpart in the reference; its orientation loop keeps one outbeam tree
 * per orientation): beams[o] holds nbeam[o] records, exts[o] next[o] records
 * (a NULL pointer is allowed for a zero count), verts[o] the orientation's
 * v(nverts,3).  The arrays are copied to the device as they are, without a
 * host-side gather. */
int pbt_diff_batch_list_c(pbt_ctx *ctx, int64_t norient, const pbt_outbeam *const *beams,
                          const int64_t *nbeam, const pbt_outbeam *const *exts,
                          const int64_t *next, const double *const *verts, int64_t nverts,
                          const int64_t *face_off, const int64_t *face_vi, int64_t nfaces,
                          const double *theta, int64_t ntheta, const double *phi, int64_t nphi,
                          double lambda, int32_t is_fast_diff, int32_t scaling, int32_t precision,
                          const pbt_output_params *params_in, double *mueller_avg,
                          double *mueller_1d_avg, pbt_output_params *params_avg,
                          pbt_output_params *params_per_orient);

/* Same as pbt_diff_batch_c with the bulk arrays already in device memory of
 * the context's device: beam, ext, verts, face_vi, params_in and all outputs
 * are device pointers; beam_off, ext_off, face_off, theta and phi are host
 * arrays (the sizes and offsets that plan the launch).  Work is ordered on
 * `stream` (a cudaStream_t; NULL = the legacy default stream) and the call
 * returns without synchronising once the grid tables are cached.  FP32 only;
 * device-side input errors (a face index out of range) are not reported by
 * this entry point. */
int pbt_diff_batch_dev_c(pbt_ctx *ctx, void *stream, int64_t norient, const pbt_outbeam *beam,
                         const int64_t *beam_off, const pbt_outbeam *ext, const int64_t *ext_off,
                         const double *verts, int64_t nverts, const int64_t *face_off,
                         const int64_t *face_vi, int64_t nfaces, const double *theta,
                         int64_t ntheta, const double *phi, int64_t nphi, double lambda,
                         int32_t is_fast_diff, int32_t scaling, int32_t precision,
                         const pbt_output_params *params_in, double *mueller_avg,
                         double *mueller_1d_avg, pbt_output_params *params_avg,
                         pbt_output_params *params_per_orient);

/* CUDA graph of pbt_diff_batch_dev_c (no counterpart in the reference: the
 * orientation loop of src/pbt_seq_mod.f90:146-274 as one replayable graph).
 * Runs the batch once (the outputs hold its result), then captures the same
 * enqueue into a graph that owns private scratch, bin tables and staged
 * offsets.  The device arrays are baked in by address: refill them in place
 * and call pbt_graph_launch_c to recompute; the host arrays (offsets, face
 * offsets, theta, phi) are read only here.  One replay at a time per graph
 * (replays share its scratch); the arrays must outlive the graph. */
typedef struct pbt_graph pbt_graph;
int pbt_diff_batch_dev_graph_c(pbt_ctx *ctx, void *stream, int64_t norient,
                               const pbt_outbeam *beam, const int64_t *beam_off,
                               const pbt_outbeam *ext, const int64_t *ext_off,
                               const double *verts, int64_t nverts, const int64_t *face_off,
                               const int64_t *face_vi, int64_t nfaces, const double *theta,
                               int64_t ntheta, const double *phi, int64_t nphi, double lambda,
                               int32_t is_fast_diff, int32_t scaling,
                               const pbt_output_params *params_in, double *mueller_avg,
                               double *mueller_1d_avg, pbt_output_params *params_avg,
                               pbt_output_params *params_per_orient, pbt_graph **out);
/* Replay on `stream` (a cudaStream_t); returns without synchronising. */
int pbt_graph_launch_c(pbt_graph *graph, void *stream);
/* Kernels one replay launches. */
int64_t pbt_graph_kernel_count(const pbt_graph *graph);
int pbt_graph_destroy_c(pbt_graph *graph);

/* ---------------------------------------------------------- introspection */

/* Number of kernel launches made by the last completed compute call on this
 * context (for launch accounting in benchmarks). */
int64_t pbt_last_launch_count(pbt_ctx *ctx);

/* Enable (1) or disable (0) CUDA-event timing of the far-field kernels (the
 * FP64 and FP32 facet x bin sums).  While enabled, every such launch is
 * bracketed by events on its stream. */
int pbt_set_kernel_timing(pbt_ctx *ctx, int32_t enable);

/* Launch plan of the FP32 far-field kernel on this context: variant 1 = packed
 * two-facet kernel, 0 = one facet per step; bins_per_thread 1 or 2;
 * records_per_item = facet records per work item (32 .. 2^22).  variant < 0
 * restores the default: the packed kernel, one bin per thread, and work items
 * sized per call (about eight per resident CTA for the call's records and bin
 * tiles, 256 to 2,048 records).  Chosen by the tuner (abt_b200/tune.py). */
int pbt_set_plan(pbt_ctx *ctx, int32_t variant, int32_t bins_per_thread, int64_t records_per_item);

/* Sum of the device durations (ms) of the far-field kernel launches timed
 * since the previous call, and their number; waits for the last of them.
 * Resets the record. */
int pbt_kernel_time_ms(pbt_ctx *ctx, double *total_ms, int64_t *nlaunch);

/* ---------------------------------------------------------------------------
 * Beam-list files (no counterpart in the reference): the outbeam lists that
 * the tracer hands to diff_main (src/pbt_seq_mod.f90:212), one orientation
 * after another, saved for replay through pbt_diff_batch_c.  Host-only.
 * Writer: open with the far-field grid and the particle topology, add one
 * orientation per call (its outbeams, external-diffraction outbeams, rotated
 * vertices v(nverts,3) and params_in record), close.  Reader: the whole file
 * in host memory; pbt_beamlist_arrays gives pointers in pbt_diff_batch_c's
 * layout (orientation-major outbeams with offsets, norient vertex blocks,
 * norient params records), valid until pbt_beamlist_free.  A damaged,
 * truncated or foreign file fails with PBT_EINVAL (magic, version, counts
 * and a checksum are verified). */
typedef struct pbt_beamlist_writer pbt_beamlist_writer;
typedef struct pbt_beamlist pbt_beamlist;
int pbt_beamlist_writer_open(const char *path, const double *theta, int64_t ntheta,
                             const double *phi, int64_t nphi, int64_t nverts,
                             const int64_t *face_off, const int64_t *face_vi, int64_t nfaces,
                             double lambda, pbt_beamlist_writer **out);
int pbt_beamlist_writer_add(pbt_beamlist_writer *w, const pbt_outbeam *beam, int64_t nbeam,
                            const pbt_outbeam *ext, int64_t next, const double *verts,
                            const pbt_output_params *params_in);
int pbt_beamlist_writer_close(pbt_beamlist_writer *w);
int pbt_beamlist_read(const char *path, pbt_beamlist **out);
/* counts: norient, nverts, nfaces, nface_vi, ntheta, nphi, nbeam_total, next_total */
int pbt_beamlist_info(const pbt_beamlist *bl, int64_t counts[8], double *lambda);
int pbt_beamlist_arrays(const pbt_beamlist *bl, const double **theta, const double **phi,
                        const int64_t **face_off, const int64_t **face_vi, const double **verts,
                        const int64_t **beam_off, const pbt_outbeam **beam,
                        const int64_t **ext_off, const pbt_outbeam **ext,
                        const pbt_output_params **params_in);
int pbt_beamlist_free(pbt_beamlist *bl);

/* ---------------------------------------------------------------------------
 * Near-field tracer (host, FP64): the producer of the outbeam lists, for one
 * orientation at a time.  Replaces the reference's orientation step ahead of
 * diff_main (src/pbt_seq_mod.f90:165-201): PROT_MPI (src/input_mod.f90:
 * 1705-1908), make_incident_beam (:2112-2264) and beam_loop_for_speed
 * (src/beam_loop_mod.f90:1626-1806).  No device memory, no CUDA calls.
 *
 * pbt_particle_create prepares a particle as the reference does after reading
 * it (src/input_mod.f90:2663-2680): vertices v(nverts,3) column-major, faces
 * as a 0-based offset array plus 1-based vertex indices (triangles only: the
 * visibility test reads three vertices per face), face_ap the 1-based
 * aperture of each face (NULL: every face its own aperture, as without an
 * apertures file).  The centre of mass is moved to the origin.
 *
 * pbt_trace_orientation_c rotates the particle by the Euler angles euler[3]
 * (alpha, beta, gamma in radians; the reference's 'euler' method converts its
 * degrees and lifts |beta| < 1e-4 degree to 1e-4 first, 'multi' draws
 * alpha = 2 pi u1, beta = acos(1 - 2 u2), gamma = 2 pi u3), traces it and
 * keeps the result: the beam outbeams (beam_outbeam_tree), the external-
 * diffraction outbeams (ext_diff_outbeam_tree, fov = pi/2), the rotated
 * vertices (the geometry diff_main reads) and the energy record.  Outbeams
 * are listed in the order a single-threaded run of the reference appends
 * them, on any number of host threads.  A NaN outbeam amplitude (the
 * reference stops there, src/beam_loop_mod.f90:1570-1573) gives PBT_ESTATE. */
typedef struct pbt_particle pbt_particle;
typedef struct pbt_trace pbt_trace;
typedef struct pbt_trace_params {
    double lambda;        /* wavelength (job_params%la) */
    double rbi, ibi;      /* refractive index, real part > 1 and imaginary part >= 0 */
    int64_t rec;          /* max recursions (reference default 8) */
    int64_t refl;         /* max total internal reflections (default 10) */
    double thresh_area;   /* aperture area threshold for a new beam (default 0.1) */
    double thresh_energy; /* aperture energy threshold for a new beam (default 1e-4) */
} pbt_trace_params;
typedef struct pbt_trace_energy {
    double abs;             /* absorption cross section (output_parameters%abs) */
    double geo_cross_sec;   /* illuminated geometric cross section */
    double beam_energy_out; /* energy of the beam outbeams */
    double ext_energy_out;  /* energy of the external-diffraction outbeams */
    int64_t nbeams;         /* beams traced (beam-tree size) */
} pbt_trace_energy;
int pbt_particle_create(const double *verts, int64_t nverts, const int64_t *face_off,
                        const int64_t *face_vi, int64_t nfaces, const int64_t *face_ap,
                        pbt_particle **out);
/* counts of the prepared particle and the centre of mass it was moved by */
int pbt_particle_info(const pbt_particle *p, int64_t *nverts, int64_t *nfaces,
                      int64_t *napertures, double *com);
/* the centred vertices, (nverts,3) column-major */
int pbt_particle_verts(const pbt_particle *p, double *verts);
int pbt_particle_destroy(pbt_particle *p);
int pbt_trace_orientation_c(const pbt_particle *p, const double *euler,
                            const pbt_trace_params *params, pbt_trace **out);
/* n orientations (euler: n x 3, alpha beta gamma per orientation) traced in
 * parallel, one orientation per host thread; out receives n handles, each as
 * pbt_trace_orientation_c would give it.  On failure none is kept and the
 * message names the first failing orientation. */
int pbt_trace_batch_c(const pbt_particle *p, int64_t n, const double *euler,
                      const pbt_trace_params *params, pbt_trace **out);
int pbt_trace_sizes(const pbt_trace *t, int64_t *nbeam, int64_t *next);
/* copies the outbeams (nbeam, next records), the rotated vertices
 * ((nverts,3) column-major) and the energy record; NULL skips an output */
int pbt_trace_copy(const pbt_trace *t, pbt_outbeam *beam, pbt_outbeam *ext, double *verts,
                   pbt_trace_energy *energy);
int pbt_trace_destroy(pbt_trace *t);

/* Failure-detection self-test (no counterpart in the reference): launches a
 * device wait on an mbarrier that nothing completes, bounded like every wait of
 * the far-field kernels; it gives up after limit_ms (1..5000) and the call
 * returns PBT_ETIMEOUT, leaving the context usable. */
int pbt_selftest_bounded_wait_c(pbt_ctx *ctx, int32_t limit_ms);

/* Failure injection for tests (no counterpart in the reference, which stops
 * the program when an allocation fails, src/misc_submod.f90:2453-2459): the
 * next `count` device allocations the library makes, in any context of the
 * process, fail as a failing cudaMalloc would, so the calls that need them
 * return PBT_ENOMEM with a message and leave their context usable; a count of
 * 0 clears the injection.  Returns the count that was pending before. */
int pbt_test_fail_next_alloc(int32_t count);

#ifdef __cplusplus
}
#endif
#endif /* PBT_DIFF_H */
