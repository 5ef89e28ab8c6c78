/*
 * lps_oracle.h -- CPU restatement of the reference LPS time marcher.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the CUDA path is compared
 * against (tests/, __graft_entry__.smoke(), and bench.py's CPU-baseline leg).
 * No product code path links, loads or calls it.
 *
 * It restates src/main.cpp of alhermann/peridynamic-lps-absorbing-boundary
 * (setup :346-707, time loop :718-1164) in plain C with the same operation
 * order, so that against the compiled reference it differs only through the
 * order of equidistant neighbours (the reference sorts a k-d tree result with
 * std::sort, kd_tree_interface.h:107, which leaves ties unordered).
 * Parity is pinned against the compiled reference in tests/test_oracle_pin.py.
 */
#ifndef LPS_ORACLE_H
#define LPS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* One input set, as read from the preprocessor's files (src/main.cpp:178-293). */
typedef struct lpso_problem {
  int n_nodes;          /* .data1[0] NodeNo                                   */
  int n_abc;            /* .data1[4] constrainsNo                             */
  int max_cloud;        /* .data1[5] maxCloudSize                             */
  int n_prenotch;       /* .data1[2] PrenotchNo                               */
  double E, nu, rho, dt, delta, dx, dy; /* .data2 [0],[1],[2],[6],[7],[8],[9] */
  const double *nodes;  /* [2N] x,y                                           */
  const int *bctypes;   /* [2N]                                               */
  const double *u0;     /* [2N] .icvalues                                     */
  const double *v0;     /* [2N] .icdvalues                                    */
  const double *prenotch; /* [4P]                                             */
  const int *inf_nodes; /* [n_abc]                                            */
  const int *clouds;    /* [n_abc * max_cloud], -1 padded                     */
  const double *gu;     /* [2 n_abc][2 abcs_step C]                           */
  const double *gv;     /* same                                               */
  const double *gtheta; /* [n_abc][abcs_step C] (theta method 1 only)         */
} lpso_problem;

/* The reference's compile-time switches (src/main.cpp:33-38), at run time. */
typedef struct lpso_options {
  int abcs_step;        /* 2 (reference default), 1, or -1 (ABCs off)        */
  int theta_method;     /* 1 = G_theta (default), 0 = inverse-distance weights */
  int kinematic_v;      /* KINEMATIC_VELOCITY_ABC, default 0                 */
  int max_horizon;      /* MAX_HORIZON_LENGTH, default 128 (counts self)     */
  int substep;          /* SUBSTEP_NO, output cadence, default 30            */
  int n_threads;        /* OpenMP threads, 0 = runtime default               */
} lpso_options;

/* One output line: the .energy columns (src/main.cpp:1108-1112) and the
 * .verify columns (:1118-1122) plus the console extras.                      */
typedef struct lpso_diag {
  double t, E, Ek, Ep, Px, Py, max_u, max_v, max_a;
  double theta_min, theta_max, uB_rms, vB_rms, dE_rel;
  int step, max_u_node, max_v_node, n_active_abc;
} lpso_diag;

/* Status codes. */
#define LPSO_OK 0
#define LPSO_ERR_ARG -1
#define LPSO_ERR_HORIZON -2     /* horizon longer than max_horizon            */
#define LPSO_ERR_NONFINITE -3   /* the reference's FATAL at :1126-1133        */
#define LPSO_ERR_LAME -4        /* FATAL Lame identity check :310-322         */
#define LPSO_ERR_LAMBDAPD -5    /* FATAL lambda_PD identity check :496-504    */
#define LPSO_ERR_NOMEM -6

/* Neighbour search (kd_tree_interface.h:43-126 semantics, src/main.cpp:352):
 * every node within radius delta + dx/2 + 1e-5, sorted by distance, self
 * first, rows padded with -1 to max_len.  Ties are ordered by node index.
 * horizons is [N][max_len], lengths [N].  Returns the max length or <0.     */
int lpso_build_horizons(int n_nodes, const double *nodes, double radius,
                        int max_len, int *lengths, int *horizons);

/* Full run: setup, then n_steps velocity-Verlet steps with output every
 * substep steps into diag (up to max_diag records).  Final state (after the
 * last step's ABC updates) goes to the optional u/v/a/theta/m outputs.
 * elapsed_s receives the time-marching wall time (src/main.cpp:716,1166).   */
int lpso_run(const lpso_problem *p, const lpso_options *o, int n_steps,
             lpso_diag *diag, int max_diag, int *n_diag,
             double *u_out, double *v_out, double *a_out, double *theta_out,
             double *m_out, double *elapsed_s);

/* Single-kernel checkers for unit tests of individual GPU kernels: they take
 * the horizon table from lpso_build_horizons and run one phase on the
 * given arrays. */
void lpso_weighted_volume(int n, const double *nodes, const int *lengths,
                          const int *hz, int max_len, double delta, double dx,
                          double dy, double *m);
void lpso_dilatation(int n, const double *nodes, const int *lengths,
                     const int *hz, int max_len, double delta, double dx,
                     double dy, const double *m, const double *u, double *theta);
void lpso_force(int n, const double *nodes, const int *lengths, const int *hz,
                int max_len, double delta, double dx, double dy, double lam,
                double mu, double rho, const double *m, const double *theta,
                const double *u, double *acc);

#ifdef __cplusplus
}
#endif
#endif
