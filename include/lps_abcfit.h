/*
 * lps_abcfit.h -- host C ABI of the absorbing-boundary operator fit.
 *
 * The reference computes the absorbing-boundary updating vectors G_u, G_v and
 * G_theta in its preprocessor (preprocessor/main.cpp), a separate program
 * whose only interface is its command line `lps_abc_preprocessor <job> [nu]`
 * and the files it writes; its geometry (R = 125 mm, dx = 0.5 mm, delta = 4 dx)
 * is compiled in.  This entry point is that fit for any disc: the same plane-
 * wave basis, the same least-squares problems solved by LAPACK dgelsd, and the
 * same (dt, delta_kappa) stability sweep, on a node set, ring and clouds the
 * caller supplies (lps_b200/gen.py builds them as the preprocessor does).  It
 * runs on the host (OpenMP over ABC nodes and sweep points), as the north
 * star's preprocessor does; no GPU is involved.
 *
 * dgelsd is not linked: the caller passes a pointer to a Fortran-convention
 * dgelsd (for instance scipy's bundled OpenBLAS `scipy_dgelsd_`), which must
 * be safe to call from several threads at once with its own threading off.
 */
#ifndef LPS_ABCFIT_H
#define LPS_ABCFIT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* void dgelsd_(m, n, nrhs, a, lda, b, ldb, s, rcond, rank, work, lwork, iwork, info) */
typedef void (*lps_dgelsd_fn)(int *, int *, int *, double *, int *, double *, int *, double *, double *, int *,
                              double *, int *, int *, int *);

typedef struct lps_abcfit_params {
  double E, nu, rho;       /* material (preprocessor/main.cpp:58-61, nu from argv[2], :800-817) */
  double delta, dx, dy;    /* horizon and spacing (:64-67)                                        */
  int32_t abcs_step;       /* temporal stencil: 2 (the preprocessor's ABCS_STEP) or 1             */
  int32_t sweep;           /* 1: choose (dt, delta_kappa) by the stability sweep (:1047-1174);    */
                           /* 0: use dt and dk_factor below                                        */
  double dt;               /* sweep == 0: the time step                                           */
  double dk_factor;        /* sweep == 0: delta_kappa = dk_factor / sqrt(c_P)                     */
  int32_t n_threads;       /* OpenMP threads, 0 = all                                             */
  int32_t pad;
} lps_abcfit_params;

typedef struct lps_abcfit_result {
  double dt;               /* chosen time step                                                     */
  double delta_kappa;      /* chosen wavenumber range                                              */
  double dk_factor;        /* delta_kappa * sqrt(c_P)                                              */
  double sweep_max_g;      /* max ||G|| over the sweep's sample nodes at the chosen point          */
  double max_norm_gu, max_norm_gv, max_norm_gtheta;  /* Frobenius norms over all ABC nodes (:1217) */
  double m_ref;            /* template-grid weighted volume (:171-182)                             */
  int32_t n_steps;         /* ceil(210 us / dt), as :1177-1179                                     */
  int32_t n_modes;         /* wave modes after de-duplication (:350-366)                           */
  int32_t n_failed;        /* ABC nodes with ||G|| > 1 (:1197-1203)                                */
  int32_t stable_found;    /* 0 when no sweep point had max ||G|| <= 1 (:1150-1157)                */
  int32_t dgelsd_failures; /* nonzero LAPACK info codes                                            */
  int32_t pad;
} lps_abcfit_result;

/* Fits G_u, G_v (each [2 n_abc][2 abcs_step max_cloud], the .ciNodesU/V
 * layout) and G_theta ([n_abc][abcs_step max_cloud], .ciNodesTheta) for the
 * ABC nodes abc_nodes[n_abc] of the node set nodes[2 n_nodes] (x/y
 * interleaved) with clouds[n_abc * max_cloud] (node indices, -1 padded),
 * replacing preprocessor/main.cpp:809-1268.  Outputs are zero-filled past each
 * node's cloud.  Returns 0, or -1 on a bad argument. */
int lps_abcfit(const lps_abcfit_params *p, const double *nodes, int32_t n_nodes, const int32_t *abc_nodes,
               int32_t n_abc, const int32_t *clouds, int32_t max_cloud, lps_dgelsd_fn dgelsd, double *gu,
               double *gv, double *gtheta, lps_abcfit_result *out);

#ifdef __cplusplus
}
#endif
#endif
