/*
 * lps_cuda.h -- C ABI of the B200 LPS peridynamics time marcher.
 *
 * The reference (alhermann/peridynamic-lps-absorbing-boundary) has no plugin
 * or FFI surface: its solver is one monolithic main() with globals
 * (src/main.cpp:44-95, :145-1170) whose interface is the command line
 * `PD2_LPS_ABC <prefix> <jobname>`, the preprocessor's input files and the
 * .energy/.verify/VTK outputs.  The entry points below are the seams of that
 * main(): each one names the block of src/main.cpp it replaces.  The drop-in
 * executable lps_gpu (same command line, files and exit codes) is written on
 * top of them, and so are the Python bindings used by the tests and bench.
 *
 * Conventions
 *  - Every function returns an int status: 0 = LPS_OK, negative = error
 *    (LPS_ERR_*).  No C++ exception crosses this boundary.
 *  - Plain host pointers and sizes only.  The library copies every input to
 *    the device in lps_create; the caller keeps ownership of its arrays.
 *  - One handle = one CUDA stream + cached CUDA graphs.  A handle is not
 *    thread-safe; use one host thread per handle.
 *  - lps_step only enqueues work (asynchronous); lps_read_diag, lps_download
 *    and lps_synchronize synchronise the handle's stream.
 */
#ifndef LPS_CUDA_H
#define LPS_CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LPS_ABI_VERSION 2

/* status codes */
#define LPS_OK 0
#define LPS_ERR_INVALID_ARG -1     /* null pointer, bad size or option       */
#define LPS_ERR_HORIZON -2         /* a horizon exceeds max_horizon; the      */
                                   /* reference throws, kd_tree_interface.h:96 */
#define LPS_ERR_NONFINITE -3       /* NaN/Inf energy or displacement; the     */
                                   /* reference's FATAL, src/main.cpp:1126-1133 */
#define LPS_ERR_LAME -4            /* FATAL, src/main.cpp:317-321             */
#define LPS_ERR_LAMBDA_PD -5       /* FATAL, src/main.cpp:500-503             */
#define LPS_ERR_CUDA -6            /* a CUDA runtime call failed              */
#define LPS_ERR_NOMEM -7           /* device or host allocation failed        */
#define LPS_ERR_UNSUPPORTED -8     /* option combination not built            */
#define LPS_ERR_NO_DEVICE -9       /* no CUDA device / not an sm_100 device   */

/* precision forms */
#define LPS_FP64 0                 /* FP64 end to end (the plain form)        */
#define LPS_FP32_MIXED 1           /* FP32 bond arithmetic, FP64 state and ABC */

/* kernel paths */
#define LPS_PATH_AUTO 0            /* dense grid when every instance is a     */
                                   /* lattice, else CSR                       */
#define LPS_PATH_DENSE 1           /* masked dense-grid stencil               */
#define LPS_PATH_CSR 2             /* neighbour-list (ELL) kernel             */

/* One input set: what src/main.cpp:178-293 reads from the preprocessor's
 * files.  Array layouts are exactly the files' (row-major, x/y interleaved). */
typedef struct lps_problem {
  int32_t n_nodes;          /* .data1[0] NodeNo                               */
  int32_t n_abc;            /* .data1[4] constrainsNo                         */
  int32_t max_cloud;        /* .data1[5] maxCloudSize                         */
  int32_t n_prenotch;       /* .data1[2] PrenotchNo                           */
  double E, nu, rho, dt, delta, dx, dy;  /* .data2[0,1,2,6,7,8,9]             */
  const double *nodes;      /* [2N] .nodes                                    */
  const int32_t *bctypes;   /* [2N] .bctypes                                  */
  const double *u0;         /* [2N] .icvalues                                 */
  const double *v0;         /* [2N] .icdvalues                                */
  const double *prenotch;   /* [4P] .prenotch (may be NULL when P == 0)       */
  const int32_t *inf_nodes; /* [n_abc] .infNodesIndex                         */
  const int32_t *clouds;    /* [n_abc * max_cloud] .iClouds, -1 padded        */
  const double *gu;         /* [2 n_abc][2 abcs_step max_cloud] .ciNodesU     */
  const double *gv;         /* same shape, .ciNodesV                          */
  const double *gtheta;     /* [n_abc][abcs_step max_cloud] .ciNodesTheta;    */
                            /* NULL allowed when theta_method == 0            */
} lps_problem;

/* Run-time form of the reference's compile-time switches
 * (src/main.cpp:33-38) plus the device-side choices. */
typedef struct lps_options {
  int32_t abcs_step;        /* ABCS_STEP: 2 (default), 1, or -1 = ABCs off    */
  int32_t theta_method;     /* THETA_ABC_METHOD: 1 = G_theta (default),       */
                            /* 0 = inverse-distance weights                   */
  int32_t kinematic_v;      /* KINEMATIC_VELOCITY_ABC, default 0              */
  int32_t max_horizon;      /* MAX_HORIZON_LENGTH incl. self, default 128     */
  int32_t precision;        /* LPS_FP64 or LPS_FP32_MIXED                     */
  int32_t path;             /* LPS_PATH_*                                     */
  int32_t device;           /* CUDA device ordinal                            */
  int32_t use_graphs;       /* 1 (default): replay captured CUDA graphs       */
  void *stream;             /* cudaStream_t to run on, or NULL for an owned one */
  int32_t autotune;         /* 1: lps_create times the dense tile kernels'    */
                            /* step graph at each rows-per-thread choice and  */
                            /* resident-CTA count and keeps the fastest (no   */
                            /* effect on results); 0 (default): 4 dilatation */
                            /* and 2 force rows per thread, full occupancy    */
  int32_t theta_rows;       /* dense dilatation rows per thread: 0 (default:  */
                            /* 4, or the autotuner's choice), 2 or 4 (fixed)  */
  int32_t horizon_build;    /* horizon search (src/main.cpp:352-356): 0 auto  */
                            /* (on the GPU from 50,000 nodes), 1 host bucket  */
                            /* grid, 2 GPU; both give the same horizons       */
  int32_t force_rows;       /* dense FP32-mixed force rows per thread: 0      */
                            /* (default: 2, or the autotuner's choice), 2 or  */
                            /* 4 (fixed); the FP64 force pass always has 2    */
} lps_options;

/* One output record: the .energy columns (src/main.cpp:1108-1112), the
 * .verify columns (:1118-1122) and the console extras (:1065-1088). */
typedef struct lps_diag {
  double t, E, Ek, Ep, Px, Py, max_u, max_v, max_a;
  double theta_min, theta_max, uB_rms, vB_rms, dE_rel;
  int32_t step, max_u_node, max_v_node, n_active_abc;
} lps_diag;

/* Setup-time facts the reference prints (src/main.cpp:330-535). */
typedef struct lps_info {
  int32_t n_instances, path, precision, max_horizon_len;
  int64_t total_nodes, total_abc;
  double m_ref, m_min, lambda, mu, kappa, alpha, lambda_pd;  /* instance 0   */
  double output_exclude_r, domain_radius, dt_lps;             /* instance 0   */
  int64_t device_bytes;                                       /* allocated    */
  int64_t step;                                               /* steps taken  */
  int32_t n_abc_m_corrected, pad;                             /* instance 0   */
  int32_t tile_ctas_theta, tile_ctas_force;  /* dense path: CTAs per SM of the */
                                             /* dilatation / force tiles      */
  int32_t tile_rows_theta, tile_rows_force;  /* dense path: rows per thread of */
                                             /* the dilatation / force tiles  */
  double horizon_ms;                         /* instance: horizon search time */
  int32_t horizon_on_gpu, pad3;              /* 1: searched on the GPU        */
} lps_info;

typedef struct lps_handle lps_handle;

/* Fills *o with the reference defaults (ABCS_STEP 2, THETA_ABC_METHOD 1,
 * KINEMATIC_VELOCITY_ABC 0, MAX_HORIZON_LENGTH 128), FP64, auto path. */
void lps_default_options(lps_options *o);

/* Setup, replacing src/main.cpp:300-683: Lame constants and checks, horizon
 * search (:346-381), prenotch visibility (:386-402), weighted volumes and
 * m_ref with the ABC override (:408-480), LPS constants and checks
 * (:485-513), exclusion radius (:518-535), initial conditions (:624-634) and
 * the theta history (:664-683).  n_instances > 1 packs independent problems
 * into one batch that every call below advances together. */
int lps_create(const lps_problem *problems, int n_instances, const lps_options *opt,
               lps_handle **out);

/* Replaces the stored initial conditions of one instance (host arrays [2N],
 * x/y interleaved; either may be NULL to keep it).  Takes effect at the next
 * lps_reset.  This is the host->device copy of a run's inputs. */
int lps_set_initial(lps_handle *h, int instance, const double *u0, const double *v0);

/* Re-initialises every instance from its stored initial conditions, as
 * src/main.cpp:624-683 does (u^{-1} = v^{-1} = a^0 = 0, theta^0 from u^0,
 * theta^{-1} = 0), sets the step count to 0 and clears the diagnostics logs
 * and E0.  lps_create ends with an implicit reset.  After a device-side wait
 * timed out (a call returned LPS_ERR_CUDA saying so), the tile kernels do no
 * work until this call clears the device error flag and the tile-scheduler
 * counters; the handle then runs again. */
int lps_reset(lps_handle *h);

/* Enqueues n_steps time steps, src/main.cpp:718-1164 (predictor, dilatation,
 * ABC dilatation, force, ABC displacement, corrector, ABC velocity, history
 * rotation).  When diag_every > 0, a diagnostics record (:986-1062) is
 * computed on the device after every step s with s % diag_every == 0
 * (s counted from the last reset) and appended to the on-device log. */
int lps_step(lps_handle *h, int n_steps, int diag_every);

/* Copies the records logged since the last call (or reset) for instance;
 * dE_rel is relative to the first record after the reset, as :1046-1047.
 * Returns LPS_ERR_NONFINITE (after copying) if a record holds a NaN/Inf
 * energy or max|u|, the reference's FATAL at :1126-1133. */
int lps_read_diag(lps_handle *h, int instance, lps_diag *out, int max_records, int *n_records);

/* Copies the current state of one instance to host arrays (any may be NULL):
 * u, v, a [2N] interleaved, theta [N] (after the ABC override), m [N]
 * (weighted volumes after the ABC override). */
int lps_download(lps_handle *h, int instance, double *u, double *v, double *a, double *theta,
                 double *m);

int lps_synchronize(lps_handle *h);
int lps_get_info(lps_handle *h, int instance, lps_info *info);
/* Human-readable text of the last error on this handle (or of the last
 * failed lps_create when h is NULL). */
const char *lps_last_error(const lps_handle *h);
const char *lps_status_string(int status);
void lps_destroy(lps_handle *h);

/* Number of kernel launches this handle enqueued so far (graph replays count
 * every kernel node they contain). */
int64_t lps_kernel_launches(const lps_handle *h);

/* Per-kernel timing (no counterpart in the reference, whose only timer is
 * utils::timer around the whole loop, src/main.cpp:716,1166): runs n_steps
 * steps eagerly with CUDA events recorded on the handle's stream between the
 * launches, and reports per kernel kind its launch count and total device
 * time.  The state advances as with lps_step. */
typedef struct lps_kernel_time {
  char name[32];
  int32_t launches;
  int32_t pad;
  double total_ms;
} lps_kernel_time;
int lps_profile_kernels(lps_handle *h, int n_steps, int diag_every, lps_kernel_time *out,
                        int max_kinds, int *n_kinds);

/* State diagnostics without any allocation.  No counterpart in the
 * reference: it exists for callers that must not allocate device memory when
 * they call it (a time-critical loop that cannot afford cudaMalloc's implicit
 * synchronisation, a host whose GPU memory is owned by another allocator, code
 * running during a stream capture).  Given one instance's state already in
 * device memory -- xy, u, v, a as [2N] x/y interleaved doubles, theta [N] --
 * it enqueues on `stream` (NULL: the legacy default stream) the kinetic
 * energy, momentum and maxima of an output step, src/main.cpp:992-1016
 * (energy and momentum over r <= exclude_r when exclude_r > 0), and writes
 * LPS_NOALLOC_OUT doubles to the device buffer `out`:
 *   Ek, Px, Py, max|u|, max|v|, max|a|, theta_min, theta_max,
 *   node of max|u|, node of max|v|   (-1 when every magnitude is 0).
 * Its scratch is a file-scope device array sized for LPS_NOALLOC_MAX_NODES
 * nodes (about 0.46 MB on every GPU that loads the library, held until the
 * process exits); larger n_nodes is rejected with LPS_ERR_INVALID_ARG and a
 * message in lps_last_error(NULL).  xy, u, v and a are read as 16-byte x/y
 * pairs and must be 16-byte aligned, theta and out 8-byte aligned; a view
 * that starts on an odd double is rejected with LPS_ERR_INVALID_ARG before
 * any launch.  A CUDA error already pending on the calling thread is reported
 * as LPS_ERR_CUDA and left pending.  The first call on a device (and the
 * first after its context was destroyed and recreated, e.g. by
 * cudaDeviceReset) resolves the array's device address (cudaGetSymbolAddress)
 * -- make that first call before any stream capture on the device.  All calls
 * on a device share the array, so calls that overlap on the GPU (different
 * streams, no ordering) race and must be serialised by the caller; every call
 * rewrites the slots it reads, so nothing needs clearing.  The call returns
 * without synchronising. */
#define LPS_NOALLOC_MAX_NODES 1048576
#define LPS_NOALLOC_OUT 10
int lps_state_diag_noalloc(int n_nodes, const double *xy, const double *u, const double *v,
                           const double *a, const double *theta, double rho, double dx, double dy,
                           double exclude_r, double *out, void *stream);

#ifdef __cplusplus
}
#endif
#endif
