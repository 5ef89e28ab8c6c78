// lps_setup.cpp -- host-side setup of one instance.
//
// Follows src/main.cpp:300-535 of the reference: the formulas are kept in the
// reference's evaluation order so that m_i, m_ref and the constants come out
// bit-identical; the k-d tree of build_clouds (kd_tree_interface.h:43-126)
// is replaced by a uniform bucket grid with the same inclusion test.
#include "lps_setup.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <limits>

namespace lps {

namespace {

inline double beta_of(double xi, double R, double dx) {  // src/main.cpp:100-107
  if (xi <= R - dx / 2.0) return 1.0;
  if (xi <= R + dx / 2.0) return (R + dx / 2.0 - xi) / dx;
  return 0.0;
}

int relative_ccw(double x1, double y1, double x2, double y2, double px, double py) {
  // src/main.cpp:119-132
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

bool segments_cross(double x1, double y1, double x2, double y2, double x3, double y3, double x4,
                    double y4) {  // src/main.cpp:134-140
  return (relative_ccw(x1, y1, x2, y2, x3, y3) * relative_ccw(x1, y1, x2, y2, x4, y4) <= 0) &&
         (relative_ccw(x3, y3, x4, y4, x1, y1) * relative_ccw(x3, y3, x4, y4, x2, y2) <= 0);
}

}  // namespace

int build_horizons(int n, const double *xy, double r, int row_len, std::vector<int> &len,
                   std::vector<int> &hz) {
  double xmin = xy[0], xmax = xy[0], ymin = xy[1], ymax = xy[1];
  for (int i = 1; i < n; i++) {
    xmin = std::min(xmin, xy[2 * i]); xmax = std::max(xmax, xy[2 * i]);
    ymin = std::min(ymin, xy[2 * i + 1]); ymax = std::max(ymax, xy[2 * i + 1]);
  }
  const double cs = r > 0 ? r : 1.0;
  const long gx = (long)std::floor((xmax - xmin) / cs) + 1;
  const long gy = (long)std::floor((ymax - ymin) / cs) + 1;
  // counting sort of nodes into buckets (ascending node index inside a bucket)
  std::vector<int> start(gx * gy + 1, 0), order(n);
  std::vector<long> cell(n);
  for (int i = 0; i < n; i++) {
    long cx = (long)std::floor((xy[2 * i] - xmin) / cs), cy = (long)std::floor((xy[2 * i + 1] - ymin) / cs);
    cell[i] = cy * gx + cx;
    start[cell[i] + 1]++;
  }
  for (long c = 0; c < gx * gy; c++) start[c + 1] += start[c];
  {
    std::vector<int> fill(start.begin(), start.end() - 1);
    for (int i = 0; i < n; i++) order[fill[cell[i]]++] = i;
  }
  len.assign(n, 0);
  hz.assign((size_t)n * row_len, -1);
  int status = 0, longest = 0;
#pragma omp parallel
  {
    std::vector<std::pair<double, int>> buf;
    buf.reserve(4 * row_len + 64);
#pragma omp for schedule(dynamic, 1024) reduction(max : longest)
    for (int i = 0; i < n; i++) {
      const double xi = xy[2 * i], yi = xy[2 * i + 1];
      const long cx = cell[i] % gx, cy = cell[i] / gx;
      buf.clear();
      for (long by = std::max(0L, cy - 1); by <= std::min(gy - 1, cy + 1); by++)
        for (long bx = std::max(0L, cx - 1); bx <= std::min(gx - 1, cx + 1); bx++) {
          const long c = by * gx + bx;
          for (int q = start[c]; q < start[c + 1]; q++) {
            const int j = order[q];
            const double x = xy[2 * j] - xi, y = xy[2 * j + 1] - yi;
            const double d = std::sqrt(x * x + y * y);
            if (d <= r) buf.emplace_back(d, j);
          }
        }
      std::sort(buf.begin(), buf.end());
      int cnt = (int)buf.size();
      if (cnt > row_len) {
#pragma omp atomic write
        status = LPS_ERR_HORIZON;
        cnt = row_len;
      }
      for (int k = 0; k < cnt; k++) hz[(size_t)i * row_len + k] = buf[k].second;
      len[i] = cnt;
      longest = std::max(longest, (int)buf.size());
    }
  }
  return status ? status : longest;
}

int setup_instance(const lps_problem &p, const lps_options &o, InstanceSetup &s, std::string &err) {
  char msg[256];
  const int N = p.n_nodes;
  if (N <= 0 || !p.nodes || !p.bctypes || !p.u0 || !p.v0) {
    err = "lps_create: n_nodes <= 0 or a required array is NULL";
    return LPS_ERR_INVALID_ARG;
  }
  if (!(p.dt > 0) || !(p.rho > 0) || !(p.dx > 0) || !(p.dy > 0) || !(p.delta > 0) || !(p.E > 0)) {
    err = "lps_create: dt, rho, dx, dy, delta and E must be positive";
    return LPS_ERR_INVALID_ARG;
  }
  const bool abc_on = (o.abcs_step != -1) && p.n_abc > 0;
  if (o.abcs_step != -1 && o.abcs_step != 1 && o.abcs_step != 2) {
    err = "lps_create: abcs_step must be 2, 1 or -1";
    return LPS_ERR_INVALID_ARG;
  }
  if (abc_on && (!p.inf_nodes || !p.clouds || !p.gu || !p.gv || p.max_cloud <= 0 ||
                 (o.theta_method == 1 && !p.gtheta))) {
    err = "lps_create: absorbing-boundary arrays missing";
    return LPS_ERR_INVALID_ARG;
  }
  if (p.n_prenotch > 0 && !p.prenotch) {
    err = "lps_create: prenotch array missing";
    return LPS_ERR_INVALID_ARG;
  }
  if (abc_on) {
    for (int i = 0; i < p.n_abc; i++)
      if (p.inf_nodes[i] < 0 || p.inf_nodes[i] >= N) {
        snprintf(msg, sizeof msg, "lps_create: infNodesIndex[%d] = %d out of range", i, p.inf_nodes[i]);
        err = msg;
        return LPS_ERR_INVALID_ARG;
      }
    for (long i = 0; i < (long)p.n_abc * p.max_cloud; i++)
      if (p.clouds[i] < -1 || p.clouds[i] >= N) {
        snprintf(msg, sizeof msg, "lps_create: iClouds entry %ld = %d out of range", i, p.clouds[i]);
        err = msg;
        return LPS_ERR_INVALID_ARG;
      }
  }
  s.n = N;
  s.n_abc = p.n_abc;
  s.cloud = p.max_cloud;
  // Lame constants and the FATAL identity check, src/main.cpp:215-217, :310-322
  const double E = p.E, Nu = p.nu;
  s.lam = E * Nu / ((1.0 + Nu) * (1.0 - 2.0 * Nu));
  s.mu = E / (2.0 * (1.0 + Nu));
  s.kappa = s.lam + s.mu;
  {
    const double E_check = s.mu * (3.0 * s.lam + 2.0 * s.mu) / (s.lam + s.mu);
    const double Nu_check = s.lam / (2.0 * (s.lam + s.mu));
    if (!(std::abs(E_check - E) / E <= 1e-10) || !(std::abs(Nu_check - Nu) <= 1e-10)) {
      err = "FATAL: Lame parameter consistency check failed!";
      return LPS_ERR_LAME;
    }
  }
  // horizons, :352-356
  const double R = p.delta, dx = p.dx, dy = p.dy;
  s.row_len = o.max_horizon > 0 ? o.max_horizon : 128;
  {
    const double horizon_search_r = R + dx / 2.0 + 1e-5;
    s.horizon_on_gpu = o.horizon_build == 2 || (o.horizon_build == 0 && N >= 50000);
    const auto t0 = std::chrono::steady_clock::now();
    const int r = s.horizon_on_gpu ? build_horizons_gpu(N, p.nodes, horizon_search_r, s.row_len, s.hz_len, s.hz)
                                   : build_horizons(N, p.nodes, horizon_search_r, s.row_len, s.hz_len, s.hz);
    s.horizon_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (r == LPS_ERR_CUDA) {
      err = "lps_create: the horizon search on the GPU failed";
      return r;
    }
    if (r < 0) {
      err = "found_node_no > max_node_no; increase max_node_no.";
      return r;
    }
    s.max_len = r;
  }
  // coincident nodes would put a neighbour in column 0 and make |xi| = 0
  for (int i = 0; i < N; i++)
    if (s.hz[(size_t)i * s.row_len] != i) {
      snprintf(msg, sizeof msg, "lps_create: node %d coincides with another node", i);
      err = msg;
      return LPS_ERR_INVALID_ARG;
    }
  // prenotch visibility, :386-402
  for (int q = 0; q < p.n_prenotch; q++) {
    const double n0x = p.prenotch[4 * q], n0y = p.prenotch[4 * q + 1];
    const double n1x = p.prenotch[4 * q + 2], n1y = p.prenotch[4 * q + 3];
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; i++)
      for (int j = 1; j < s.row_len; j++) {
        int &nb = s.hz[(size_t)i * s.row_len + j];
        if (nb == -1) continue;
        if (segments_cross(p.nodes[2 * i], p.nodes[2 * i + 1], p.nodes[2 * nb], p.nodes[2 * nb + 1],
                           n0x, n0y, n1x, n1y))
          nb = -1;
      }
  }
  // weighted volume m_i, :412-426
  s.m.assign(N, 0.0);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < N; i++) {
    double m_i = 0.0;
    for (int j = 1; j < s.hz_len[i]; j++) {
      const int nb = s.hz[(size_t)i * s.row_len + j];
      if (nb == -1) continue;
      const double xi_x = p.nodes[2 * nb] - p.nodes[2 * i];
      const double xi_y = p.nodes[2 * nb + 1] - p.nodes[2 * i + 1];
      const double xi_norm = std::sqrt(xi_x * xi_x + xi_y * xi_y);
      const double w = 1.0;
      const double b = beta_of(xi_norm, R, dx);
      m_i += w * xi_norm * xi_norm * b * dx * dy;
    }
    s.m[i] = m_i;
  }
  // m_ref = max m_i, :429-442
  {
    double m_min = 1e30, m_max = 0.0;
    for (int i = 0; i < N; i++)
      if (s.m[i] > 0.0) {
        m_min = std::min(m_min, s.m[i]);
        m_max = std::max(m_max, s.m[i]);
      }
    s.m_ref = m_max;
    s.m_min = m_min;
  }
  // m_i <- m_ref at every ABC node, :469-480
  s.n_corrected = 0;
  if (abc_on)
    for (int i = 0; i < p.n_abc; i++) {
      const int node = p.inf_nodes[i];
      if (s.m[node] < s.m_ref * 0.99) s.n_corrected++;
      s.m[node] = s.m_ref;
    }
  // LPS constants and the FATAL check, :485-504
  s.alpha = 8.0 * s.mu / s.m_ref;
  s.lambda_pd = 2.0 * (s.lam - s.mu) / s.m_ref;
  {
    const double lpd_check = 2.0 * s.kappa / s.m_ref - s.alpha / 2.0;
    if (!(std::abs(lpd_check - s.lambda_pd) <= 1e-15 * std::abs(s.lambda_pd + 1e-30))) {
      err = "FATAL: lambda_PD consistency check failed!";
      return LPS_ERR_LAMBDA_PD;
    }
  }
  // exclusion radius, :518-530
  s.domain_radius = 0.0;
  for (int i = 0; i < N; i++) {
    const double r = std::sqrt(p.nodes[2 * i] * p.nodes[2 * i] + p.nodes[2 * i + 1] * p.nodes[2 * i + 1]);
    if (r > s.domain_radius) s.domain_radius = r;
  }
  s.out_r = abc_on ? s.domain_radius - R - dx / 100.0 : -1.0;
  // sampled LPS stable time step, :555-581 (reported, not enforced)
  {
    double max_denom = 0.0;
    for (int i = 0; i < std::min(N, 10000); i++) {
      double denom = 0.0;
      const double mi = s.m[i];
      if (mi <= 0.0) continue;
      for (int j = 1; j < s.hz_len[i]; j++) {
        const int nb = s.hz[(size_t)i * s.row_len + j];
        if (nb == -1) continue;
        const double xi_x = p.nodes[2 * nb] - p.nodes[2 * i];
        const double xi_y = p.nodes[2 * nb + 1] - p.nodes[2 * i + 1];
        const double xi2 = xi_x * xi_x + xi_y * xi_y;
        const double xi_norm = std::sqrt(xi2);
        const double b = beta_of(xi_norm, R, dx);
        denom += (2.0 * s.kappa * 2.0 * xi2 / (mi * mi) + 2.0 * s.alpha / xi2) * 1.0 * b * dx * dy;
      }
      max_denom = std::max(max_denom, denom);
    }
    s.dt_lps = max_denom > 0.0 ? std::sqrt(2.0 * p.rho / max_denom) : 0.0;
  }
  return LPS_OK;
}

}  // namespace lps
