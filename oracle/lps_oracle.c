/*
 * lps_oracle.c -- CPU restatement of the reference LPS time marcher.
 *
 * TEST INFRASTRUCTURE ONLY (the checker; never the thing measured or
 * shipped).  Every function cites the lines of src/main.cpp of
 * alhermann/peridynamic-lps-absorbing-boundary that it follows.  Arithmetic
 * is written in the reference's evaluation order and compiled with the
 * reference's flags (-O3, no -march, hence no FMA contraction), so the only
 * difference from the compiled reference is the order of equidistant
 * neighbours inside each horizon.
 */
#include "lps_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* beta(xi), src/main.cpp:100-107 (R is the horizon delta). */
static inline double beta_fn(double xi, double R, double dx) {
  if (xi <= R - dx / 2.0) return 1.0;
  else if (xi <= R + dx / 2.0) return (R + dx / 2.0 - xi) / dx;
  else return 0.0;
}

/* ------------------------------------------------------------------------ */
/* Neighbour search.  The reference uses a k-d tree range query followed by a
 * Euclidean test dist <= r (kd_tree_interface.h:81-92) and a distance sort
 * (:107); self (distance 0) lands in column 0.  Restated with a uniform
 * bucket grid of cell size r.                                              */
typedef struct { double d; int idx; } nb_t;

static int nb_cmp(const void *a, const void *b) {
  const nb_t *x = (const nb_t *)a, *y = (const nb_t *)b;
  if (x->d < y->d) return -1;
  if (x->d > y->d) return 1;
  return (x->idx > y->idx) - (x->idx < y->idx);
}

int lpso_build_horizons(int n, const double *nodes, double r, int max_len,
                        int *lengths, int *hz) {
  if (n <= 0 || !nodes || !lengths || !hz || max_len <= 0) return LPSO_ERR_ARG;
  double xmin = nodes[0], xmax = nodes[0], ymin = nodes[1], ymax = nodes[1];
  for (int i = 1; i < n; i++) {
    double x = nodes[2 * i], y = nodes[2 * i + 1];
    if (x < xmin) xmin = x;
    if (x > xmax) xmax = x;
    if (y < ymin) ymin = y;
    if (y > ymax) ymax = y;
  }
  double cs = r > 0 ? r : 1.0;
  int gx = (int)floor((xmax - xmin) / cs) + 1, gy = (int)floor((ymax - ymin) / cs) + 1;
  int *head = (int *)malloc(sizeof(int) * (size_t)gx * gy);
  int *next = (int *)malloc(sizeof(int) * (size_t)n);
  if (!head || !next) { free(head); free(next); return LPSO_ERR_NOMEM; }
  for (long c = 0; c < (long)gx * gy; c++) head[c] = -1;
  /* insert in reverse so each bucket lists nodes in ascending index */
  for (int i = n - 1; i >= 0; i--) {
    int cx = (int)floor((nodes[2 * i] - xmin) / cs), cy = (int)floor((nodes[2 * i + 1] - ymin) / cs);
    long c = (long)cy * gx + cx;
    next[i] = head[c];
    head[c] = i;
  }
  int status = 0, maxfound = 0;
#pragma omp parallel
  {
    int cap = 4 * max_len + 64;
    nb_t *buf = (nb_t *)malloc(sizeof(nb_t) * cap);
#pragma omp for schedule(static) reduction(max : maxfound)
    for (int i = 0; i < n; i++) {
      double xi = nodes[2 * i], yi = nodes[2 * i + 1];
      int cx = (int)floor((xi - xmin) / cs), cy = (int)floor((yi - ymin) / cs);
      int cnt = 0;
      for (int by = cy - 1; by <= cy + 1; by++) {
        if (by < 0 || by >= gy) continue;
        for (int bx = cx - 1; bx <= cx + 1; bx++) {
          if (bx < 0 || bx >= gx) continue;
          for (int j = head[(long)by * gx + bx]; j >= 0; j = next[j]) {
            /* distance_euclidean, kd_tree_interface.h:29-34 */
            double x = nodes[2 * j] - xi, y = nodes[2 * j + 1] - yi;
            double d = sqrt(x * x + y * y);
            if (d <= r) {
              if (cnt == cap) {
                cap *= 2;
                buf = (nb_t *)realloc(buf, sizeof(nb_t) * cap);
              }
              buf[cnt].d = d;
              buf[cnt].idx = j;
              cnt++;
            }
          }
        }
      }
      if (cnt > max_len) {
#pragma omp atomic write
        status = LPSO_ERR_HORIZON;
        cnt = max_len;
      }
      qsort(buf, cnt, sizeof(nb_t), nb_cmp);
      for (int k = 0; k < cnt; k++) hz[(long)i * max_len + k] = buf[k].idx;
      for (int k = cnt; k < max_len; k++) hz[(long)i * max_len + k] = -1;
      lengths[i] = cnt;
      if (cnt > maxfound) maxfound = cnt;
    }
    free(buf);
  }
  free(head);
  free(next);
  return status ? status : maxfound;
}

/* ------------------------------------------------------------------------ */
/* Prenotch visibility, src/main.cpp:119-140 and :386-402. */
static int relative_ccw(double x1, double y1, double x2, double y2, double px, double py) {
  x2 -= x1; y2 -= y1; px -= x1; py -= y1;
  double ccw = px * y2 - py * x2;
  if (ccw == 0.0) {
    ccw = px * x2 + py * y2;
    if (ccw > 0.0) {
      px -= x2; py -= y2;
      ccw = px * x2 + py * y2;
      if (ccw < 0.0) ccw = 0.0;
    }
  }
  return (ccw < 0.0) ? -1 : ((ccw > 0.0) ? 1 : 0);
}

static int segments_intersect(double x1, double y1, double x2, double y2,
                              double x3, double y3, double x4, double y4) {
  return (relative_ccw(x1, y1, x2, y2, x3, y3) * relative_ccw(x1, y1, x2, y2, x4, y4) <= 0) &&
         (relative_ccw(x3, y3, x4, y4, x1, y1) * relative_ccw(x3, y3, x4, y4, x2, y2) <= 0);
}

/* ------------------------------------------------------------------------ */
/* m_i, src/main.cpp:412-426. */
void lpso_weighted_volume(int n, const double *nodes, const int *len, const int *hz,
                          int ml, double R, double dx, double dy, double *m) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++) {
    double m_i = 0.0;
    for (int j = 1; j < len[i]; j++) {
      int nb = hz[(long)i * ml + j];
      if (nb == -1) continue;
      const double xi_x = nodes[2 * nb] - nodes[2 * i];
      const double xi_y = nodes[2 * nb + 1] - nodes[2 * i + 1];
      const double xi_norm = sqrt(xi_x * xi_x + xi_y * xi_y);
      const double w = 1.0;
      const double b = beta_fn(xi_norm, R, dx);
      m_i += w * xi_norm * xi_norm * b * dx * dy;
    }
    m[i] = m_i;
  }
}

/* theta pass, src/main.cpp:736-761 (also the theta history init :664-682). */
void lpso_dilatation(int n, const double *nodes, const int *len, const int *hz, int ml,
                     double R, double dx, double dy, const double *m, const double *u,
                     double *theta) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++) {
    double theta_sum = 0.0;
    for (int j = 1; j < len[i]; j++) {
      int nb = hz[(long)i * ml + j];
      if (nb == -1) continue;
      const double xi_x = nodes[2 * nb] - nodes[2 * i];
      const double xi_y = nodes[2 * nb + 1] - nodes[2 * i + 1];
      const double xi_norm = sqrt(xi_x * xi_x + xi_y * xi_y);
      const double eta_x = u[2 * nb] - u[2 * i];
      const double eta_y = u[2 * nb + 1] - u[2 * i + 1];
      const double e = (eta_x * xi_x + eta_y * xi_y) / xi_norm;
      const double w = 1.0;
      const double b = beta_fn(xi_norm, R, dx);
      theta_sum += w * xi_norm * e * b * dx * dy;
    }
    theta[i] = (m[i] > 0.0) ? (2.0 / m[i]) * theta_sum : 0.0;
  }
}

/* force pass, src/main.cpp:821-874. */
void lpso_force(int n, const double *nodes, const int *len, const int *hz, int ml,
                double R, double dx, double dy, double Lambda, double Mu, double Rho,
                const double *m, const double *Theta, const double *u, double *acc) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++) {
    double F0 = 0.0, F1 = 0.0;
    const double m_i = m[i];
    if (m_i <= 0.0) {
      acc[2 * i] = 0.0;
      acc[2 * i + 1] = 0.0;
      continue;
    }
    for (int j = 1; j < len[i]; j++) {
      int nb = hz[(long)i * ml + j];
      if (nb == -1) continue;
      const double xi_x = nodes[2 * nb] - nodes[2 * i];
      const double xi_y = nodes[2 * nb + 1] - nodes[2 * i + 1];
      const double xi_norm = sqrt(xi_x * xi_x + xi_y * xi_y);
      const double eta_x = u[2 * nb] - u[2 * i];
      const double eta_y = u[2 * nb + 1] - u[2 * i + 1];
      const double e = (eta_x * xi_x + eta_y * xi_y) / xi_norm;
      const double w = 1.0;
      const double b = beta_fn(xi_norm, R, dx);
      const double m_j = m[nb];
      if (m_j <= 0.0) continue;
      const double t_i = (2.0 * (Lambda - Mu) / m_i) * Theta[i] * xi_norm * w + (8.0 * Mu / m_i) * w * e;
      const double t_j = (2.0 * (Lambda - Mu) / m_j) * Theta[nb] * xi_norm * w + (8.0 * Mu / m_j) * w * e;
      const double scale = (t_i + t_j) * b * dx * dy;
      F0 += scale * xi_x / xi_norm;
      F1 += scale * xi_y / xi_norm;
    }
    acc[2 * i] = F0 / Rho;
    acc[2 * i + 1] = F1 / Rho;
  }
}

/* G update of one ABC node's two components from a two-level history,
 * src/main.cpp:888-914 (displacement) and :945-971 (velocity). */
static void g_apply(int i, int C, int abcs_step, const int *clouds, const double *G,
                    const double *xn, const double *xnm1, double *out0, double *out1) {
  int cols = (abcs_step == 1 ? 2 : 4) * C;
  const double *g0 = G + (long)(2 * i) * cols, *g1 = G + (long)(2 * i + 1) * cols;
  double a0 = 0.0, a1 = 0.0;
  for (int j = 0; j < C; j++) {
    int k = clouds[(long)i * C + j];
    if (k == -1) continue;
    if (abcs_step == 1) {
      a0 += g0[2 * j] * xn[2 * k] + g0[2 * j + 1] * xn[2 * k + 1];
      a1 += g1[2 * j] * xn[2 * k] + g1[2 * j + 1] * xn[2 * k + 1];
    } else if (abcs_step == 2) {
      a0 += g0[4 * j] * xn[2 * k] + g0[4 * j + 1] * xn[2 * k + 1] +
            g0[4 * j + 2] * xnm1[2 * k] + g0[4 * j + 3] * xnm1[2 * k + 1];
      a1 += g1[4 * j] * xn[2 * k] + g1[4 * j + 1] * xn[2 * k + 1] +
            g1[4 * j + 2] * xnm1[2 * k] + g1[4 * j + 3] * xnm1[2 * k + 1];
    }
  }
  *out0 = a0;
  *out1 = a1;
}

static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* ------------------------------------------------------------------------ */
int lpso_run(const lpso_problem *p, const lpso_options *o, int n_steps, lpso_diag *diag,
             int max_diag, int *n_diag, double *u_out, double *v_out, double *a_out,
             double *theta_out, double *m_out, double *elapsed_s) {
  if (!p || !o || p->n_nodes <= 0 || !p->nodes || !p->bctypes || !p->u0 || !p->v0)
    return LPSO_ERR_ARG;
#ifdef _OPENMP
  if (o->n_threads > 0) omp_set_num_threads(o->n_threads);
#endif
  const int N = p->n_nodes, NA = p->n_abc, C = p->max_cloud;
  const int abcs = o->abcs_step, tm = o->theta_method, ML = o->max_horizon;
  const int substep = o->substep > 0 ? o->substep : 30;
  const double R = p->delta, dx = p->dx, dy = p->dy, dt = p->dt, Rho = p->rho;
  const int *bct = p->bctypes;
  if (n_diag) *n_diag = 0;
  if (abcs != -1 && NA > 0 && (!p->inf_nodes || !p->clouds || !p->gu || !p->gv)) return LPSO_ERR_ARG;
  if (abcs != -1 && NA > 0 && tm == 1 && !p->gtheta) return LPSO_ERR_ARG;

  /* Lame constants and identity check, :215-217, :310-322 */
  const double E_y = p->E, Nu = p->nu;
  const double Lambda = E_y * Nu / ((1.0 + Nu) * (1.0 - 2.0 * Nu));
  const double Mu = E_y / (2.0 * (1.0 + Nu));
  const double Kappa = Lambda + Mu;
  {
    double E_check = Mu * (3.0 * Lambda + 2.0 * Mu) / (Lambda + Mu);
    double Nu_check = Lambda / (2.0 * (Lambda + Mu));
    if (fabs(E_check - E_y) / E_y > 1e-10 || fabs(Nu_check - Nu) > 1e-10) return LPSO_ERR_LAME;
  }

  int status = LPSO_OK;
  int *len = (int *)malloc(sizeof(int) * N);
  int *hz = (int *)malloc(sizeof(int) * (size_t)N * ML);
  double *m = (double *)malloc(sizeof(double) * N);
  double *Theta = (double *)calloc(N, sizeof(double));
  double *ThetaN = (double *)calloc(N, sizeof(double));
  double *ThetaNm1 = (double *)calloc(N, sizeof(double));
  double *Unm1 = (double *)calloc(2 * N, sizeof(double)), *Un = (double *)malloc(sizeof(double) * 2 * N);
  double *Un1 = (double *)calloc(2 * N, sizeof(double));
  double *Udnm1 = (double *)calloc(2 * N, sizeof(double)), *Udn = (double *)malloc(sizeof(double) * 2 * N);
  double *Udn1 = (double *)calloc(2 * N, sizeof(double));
  double *Uddn = (double *)calloc(2 * N, sizeof(double)), *Uddn1 = (double *)calloc(2 * N, sizeof(double));
  if (!len || !hz || !m || !Theta || !ThetaN || !ThetaNm1 || !Unm1 || !Un || !Un1 || !Udnm1 ||
      !Udn || !Udn1 || !Uddn || !Uddn1) {
    status = LPSO_ERR_NOMEM;
    goto done;
  }

  /* horizons, :352-354 */
  {
    double horizon_search_r = R + dx / 2.0 + 1e-5;
    int r = lpso_build_horizons(N, p->nodes, horizon_search_r, ML, len, hz);
    if (r < 0) { status = r; goto done; }
  }
  /* prenotch visibility, :386-402 (note: scans every column, as the reference) */
  for (int q = 0; q < p->n_prenotch; q++) {
    const double n0x = p->prenotch[4 * q], n0y = p->prenotch[4 * q + 1];
    const double n1x = p->prenotch[4 * q + 2], n1y = p->prenotch[4 * q + 3];
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; i++)
      for (int j = 1; j < ML; j++) {
        int nb = hz[(long)i * ML + j];
        if (nb == -1) continue;
        if (segments_intersect(p->nodes[2 * i], p->nodes[2 * i + 1], p->nodes[2 * nb],
                               p->nodes[2 * nb + 1], n0x, n0y, n1x, n1y))
          hz[(long)i * ML + j] = -1;
      }
  }

  /* m_i, m_ref = max m_i, override at ABC nodes: :412-480 */
  lpso_weighted_volume(N, p->nodes, len, hz, ML, R, dx, dy, m);
  double m_ref = 0.0;
  for (int i = 0; i < N; i++)
    if (m[i] > 0.0 && m[i] > m_ref) m_ref = m[i];
  if (abcs != -1 && NA > 0)
    for (int i = 0; i < NA; i++) m[p->inf_nodes[i]] = m_ref;

  /* LPS constants and identity check, :485-504 */
  {
    const double AlphaLPS = 8.0 * Mu / m_ref;
    const double LambdaPD = 2.0 * (Lambda - Mu) / m_ref;
    double lpd_check = 2.0 * Kappa / m_ref - AlphaLPS / 2.0;
    if (fabs(lpd_check - LambdaPD) > 1e-15 * fabs(LambdaPD + 1e-30)) {
      status = LPSO_ERR_LAMBDAPD;
      goto done;
    }
  }

  /* output/energy exclusion radius, :518-530 */
  double domainRadius = 0.0;
  for (int i = 0; i < N; i++) {
    double r = sqrt(p->nodes[2 * i] * p->nodes[2 * i] + p->nodes[2 * i + 1] * p->nodes[2 * i + 1]);
    if (r > domainRadius) domainRadius = r;
  }
  const double output_exclude_r = (abcs != -1 && NA > 0) ? domainRadius - R - dx / 100.0 : -1.0;

  /* initial conditions, :624-634; theta history, :664-682 */
  for (int i = 0; i < 2 * N; i++) {
    Udn[i] = p->v0[i];
    Un[i] = p->u0[i];
  }
  if (tm == 1) {
    lpso_dilatation(N, p->nodes, len, hz, ML, R, dx, dy, m, Un, ThetaN);
    memset(ThetaNm1, 0, sizeof(double) * N);
  }

  double E0 = -1.0;
  int nd = 0;
  double t_start = now_s();
  for (int s = 1; s <= n_steps; s++) {
    const double t = s * dt;
    /* 1a predictor :725-728 */
#pragma omp parallel for schedule(static)
    for (int i = 0; i < 2 * N; i++) Un1[i] = Un[i] + dt * (Udn[i] + (dt / 2.0) * Uddn[i]);
    /* 1b dilatation :736-761 */
    lpso_dilatation(N, p->nodes, len, hz, ML, R, dx, dy, m, Un1, Theta);
    /* 1c override at ABC nodes :764-814 */
    if (abcs != -1) {
      if (tm == 0) {
        for (int i = 0; i < NA; i++) {
          int node = p->inf_nodes[i];
          if (bct[2 * node] != 1) continue;
          double theta_avg = 0.0, w_sum = 0.0;
          for (int j = 1; j < len[node]; j++) {
            int nb = hz[(long)node * ML + j];
            if (nb == -1) continue;
            if (bct[2 * nb] == 1) continue;
            double rx = p->nodes[2 * nb] - p->nodes[2 * node];
            double ry = p->nodes[2 * nb + 1] - p->nodes[2 * node + 1];
            double dist = sqrt(rx * rx + ry * ry);
            double wt = 1.0 / (dist + 1e-30);
            theta_avg += wt * Theta[nb];
            w_sum += wt;
          }
          if (w_sum > 0.0) Theta[node] = theta_avg / w_sum;
        }
      } else {
        for (int i = 0; i < NA; i++) {
          int node = p->inf_nodes[i];
          if (bct[2 * node] != 1) continue;
          double theta_abc = 0.0;
          for (int j = 0; j < C; j++) {
            int k = p->clouds[(long)i * C + j];
            if (k == -1) continue;
            if (abcs == 2)
              theta_abc += p->gtheta[(long)i * 2 * C + 2 * j] * ThetaN[k] +
                           p->gtheta[(long)i * 2 * C + 2 * j + 1] * ThetaNm1[k];
            else if (abcs == 1)
              theta_abc += p->gtheta[(long)i * C + j] * ThetaN[k];
          }
          Theta[node] = theta_abc;
        }
      }
    }
    /* 1d force :821-874 */
    lpso_force(N, p->nodes, len, hz, ML, R, dx, dy, Lambda, Mu, Rho, m, Theta, Un1, Uddn1);
    /* 1e displacement ABC :883-916 */
    if (abcs != -1)
      for (int i = 0; i < NA; i++) {
        int node = p->inf_nodes[i];
        if (bct[2 * node] != 1) continue;
        g_apply(i, C, abcs, p->clouds, p->gu, Un, Unm1, &Un1[2 * node], &Un1[2 * node + 1]);
      }
    /* 1f corrector :922-925 */
#pragma omp parallel for schedule(static)
    for (int i = 0; i < 2 * N; i++) Udn1[i] = Udn[i] + (dt / 2.0) * Uddn[i] + (dt / 2.0) * Uddn1[i];
    /* 1g velocity ABC :933-974 */
    if (abcs != -1)
      for (int i = 0; i < NA; i++) {
        int node = p->inf_nodes[i];
        if (bct[2 * node] != 1) continue;
        if (o->kinematic_v) {
          Udn1[2 * node] = (Un1[2 * node] - Un[2 * node]) / dt;
          Udn1[2 * node + 1] = (Un1[2 * node + 1] - Un[2 * node + 1]) / dt;
        } else {
          g_apply(i, C, abcs, p->clouds, p->gv, Udn, Udnm1, &Udn1[2 * node], &Udn1[2 * node + 1]);
        }
      }
    /* 1h output :981-1139 */
    if (s % substep == 0) {
      double energy = 0.0, energyK = 0.0, energyP = 0.0, Px = 0.0, Py = 0.0;
      double max_u = 0.0, max_v = 0.0, max_a = 0.0, theta_min = 1e30, theta_max = -1e30;
      int max_u_node = -1, max_v_node = -1;
      for (int i = 0; i < N; i++) {
        double x = p->nodes[2 * i], y = p->nodes[2 * i + 1];
        double r = sqrt(x * x + y * y);
        double u_mag = sqrt(Un1[2 * i] * Un1[2 * i] + Un1[2 * i + 1] * Un1[2 * i + 1]);
        double v_mag = sqrt(Udn1[2 * i] * Udn1[2 * i] + Udn1[2 * i + 1] * Udn1[2 * i + 1]);
        double a_mag = sqrt(Uddn1[2 * i] * Uddn1[2 * i] + Uddn1[2 * i + 1] * Uddn1[2 * i + 1]);
        if (u_mag > max_u) { max_u = u_mag; max_u_node = i; }
        if (v_mag > max_v) { max_v = v_mag; max_v_node = i; }
        max_a = (max_a < a_mag) ? a_mag : max_a;  /* std::max(max_a, a_mag) */
        theta_min = Theta[i] < theta_min ? Theta[i] : theta_min;
        theta_max = theta_max < Theta[i] ? Theta[i] : theta_max;
        if (output_exclude_r > 0.0 && r > output_exclude_r) continue;
        Px += Rho * Udn1[2 * i] * dx * dy;
        Py += Rho * Udn1[2 * i + 1] * dx * dy;
        double vx = Udn1[2 * i], vy = Udn1[2 * i + 1];
        double ek = 0.5 * Rho * (vx * vx + vy * vy) * dx * dy;
        energyK += ek;
        const double m_i = m[i];
        double W_i = 0.5 * Kappa * Theta[i] * Theta[i];
        for (int j = 1; j < len[i]; j++) {
          int nb = hz[(long)i * ML + j];
          if (nb == -1) continue;
          const double xi_x = p->nodes[2 * nb] - p->nodes[2 * i];
          const double xi_y = p->nodes[2 * nb + 1] - p->nodes[2 * i + 1];
          const double xi_norm = sqrt(xi_x * xi_x + xi_y * xi_y);
          const double eta_x = Un1[2 * nb] - Un1[2 * i];
          const double eta_y = Un1[2 * nb + 1] - Un1[2 * i + 1];
          const double e = (eta_x * xi_x + eta_y * xi_y) / xi_norm;
          const double ed = e - Theta[i] * xi_norm / 2.0;
          const double w = 1.0;
          const double b = beta_fn(xi_norm, R, dx);
          W_i += (4.0 * Mu / m_i) * w * ed * ed * b * dx * dy;
        }
        double ep = W_i * dx * dy;
        energyP += ep;
        energy += ek + ep;
      }
      if (E0 < 0.0) E0 = energy;
      double dE_rel = (E0 > 0.0) ? (energy - E0) / E0 : 0.0;
      double uB_sq = 0.0, vB_sq = 0.0;
      int nActive = 0;
      if (abcs != -1)
        for (int i = 0; i < NA; i++) {
          int node = p->inf_nodes[i];
          if (bct[2 * node] != 1) continue;
          nActive++;
          uB_sq += Un1[2 * node] * Un1[2 * node] + Un1[2 * node + 1] * Un1[2 * node + 1];
          vB_sq += Udn1[2 * node] * Udn1[2 * node] + Udn1[2 * node + 1] * Udn1[2 * node + 1];
        }
      if (diag && nd < max_diag) {
        lpso_diag *d = &diag[nd];
        d->t = t; d->E = energy; d->Ek = energyK; d->Ep = energyP; d->Px = Px; d->Py = Py;
        d->max_u = max_u; d->max_v = max_v; d->max_a = max_a;
        d->theta_min = theta_min; d->theta_max = theta_max;
        d->uB_rms = nActive > 0 ? sqrt(uB_sq / nActive) : 0.0;
        d->vB_rms = nActive > 0 ? sqrt(vB_sq / nActive) : 0.0;
        d->dE_rel = dE_rel; d->step = s; d->max_u_node = max_u_node; d->max_v_node = max_v_node;
        d->n_active_abc = nActive;
      }
      nd++;
      if (isnan(energy) || isinf(energy) || isnan(max_u) || isinf(max_u)) {
        status = LPSO_ERR_NONFINITE;
        if (n_diag) *n_diag = nd < max_diag ? nd : max_diag;
        goto finish;
      }
    }
    /* 1i rotation :1145-1163 */
    {
      double *tmp;
      tmp = Unm1; Unm1 = Un; Un = Un1; Un1 = tmp;
      tmp = Udnm1; Udnm1 = Udn; Udn = Udn1; Udn1 = tmp;
      tmp = Uddn; Uddn = Uddn1; Uddn1 = tmp;
      if (tm == 1) {
        tmp = ThetaNm1; ThetaNm1 = ThetaN; ThetaN = tmp;
        memcpy(ThetaN, Theta, sizeof(double) * N);
      }
    }
  }
  if (n_diag) *n_diag = nd < max_diag ? nd : max_diag;
finish:
  if (elapsed_s) *elapsed_s = now_s() - t_start;
  {
    /* After the loop the latest state sits in Un/Udn/Uddn (post-rotation);
     * after an early FATAL exit it is still in Un1/Udn1/Uddn1. */
    int rotated = (status == LPSO_OK);
    const double *uf = rotated ? Un : Un1, *vf = rotated ? Udn : Udn1, *af = rotated ? Uddn : Uddn1;
    if (u_out) memcpy(u_out, uf, sizeof(double) * 2 * N);
    if (v_out) memcpy(v_out, vf, sizeof(double) * 2 * N);
    if (a_out) memcpy(a_out, af, sizeof(double) * 2 * N);
    if (theta_out) memcpy(theta_out, Theta, sizeof(double) * N);
    if (m_out) memcpy(m_out, m, sizeof(double) * N);
  }
done:
  free(len); free(hz); free(m); free(Theta); free(ThetaN); free(ThetaNm1);
  free(Unm1); free(Un); free(Un1); free(Udnm1); free(Udn); free(Udn1); free(Uddn); free(Uddn1);
  return status;
}
