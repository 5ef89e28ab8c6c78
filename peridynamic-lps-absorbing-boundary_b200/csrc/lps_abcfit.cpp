// lps_abcfit.cpp -- the absorbing-boundary operator fit of the reference
// preprocessor (preprocessor/main.cpp), for any disc, on the host.
//
// For each absorbing node the updating vectors are the least-squares solution
// (LAPACK dgelsd, SVD truncation 1e-14) that maps a set of plane waves sampled
// on the node's cloud at times 0 and -dt to the same waves at the node at +dt
// (:415-637 for G_u, G_v; :657-785 for G_theta); the plane waves are the LPS
// dispersion modes of a wave-vector fan (:189-342, :350-366).  The time step
// and the fan's wavenumber range come from a sweep that keeps the stable
// point (max ||G|| <= 1 over a sample of nodes) whose ||G|| is largest
// (:1047-1174).
//
// The arithmetic is restated in the reference's evaluation order (loop order,
// accumulated template-grid coordinates, std::complex sums, the same std::sort
// of the modes, the same dgelsd workspace query), so the operators come out
// bit for bit the same for the same LAPACK.  What differs is the organisation:
// the sweep's 140 (dt, delta_kappa) points and the final fits run in
// parallel (OpenMP) instead of in one loop, and the clouds come from the
// caller (a grid search) instead of an O(N_abc N) scan (:889-901).
#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>

#include <omp.h>

#include "lps_abcfit.h"

namespace {

constexpr double kModeDeltaPhi = 0.0392;   // :78
constexpr int kModeNSub = 5;               // :79
constexpr double kSvdRcond = 1e-14;        // :87
constexpr double kGNormTarget = 1.0;       // :1002
constexpr double kTFinal = 6000.0 * 35.0e-9;  // :1177

struct Material {
  double E, nu, rho, lambda, mu, kappa, c_P, m_ref, alpha_lps, lambda_pd;
};

struct Bond {
  double x, y;
};

struct Mode {
  double alpha1, alpha2, omega_P, omega_S;
  double gamma_P[2], gamma_S[2];
  double S_real[2], S_imag[2];
};

struct Geometry {
  double delta, dx, dy;
  int abcs_step;
};

double beta_of(double xi, double delta, double dx) {  // :134-141
  if (xi <= delta - dx / 2.0) return 1.0;
  if (xi <= delta + dx / 2.0) return (delta + dx / 2.0 - xi) / dx;
  return 0.0;
}

// Bonds of an interior node, in the order of the accumulated loops of :147-169.
std::vector<Bond> template_grid(const Geometry &g) {
  std::vector<Bond> grid;
  const double rmax = g.delta + g.dx / 2.0;
  const double loop_max = g.delta + g.dx;
  for (double xi_x = -loop_max; xi_x <= loop_max + 1e-10; xi_x += g.dx)
    for (double xi_y = -loop_max; xi_y <= loop_max + 1e-10; xi_y += g.dy) {
      const double r = std::sqrt(xi_x * xi_x + xi_y * xi_y);
      if (r > 1e-12 && r <= rmax + 1e-10) grid.push_back(Bond{xi_x, xi_y});
    }
  return grid;
}

double reference_volume(const std::vector<Bond> &tg, const Geometry &g) {  // :174-182
  double m = 0.0;
  for (const Bond &b : tg) {
    const double r = std::sqrt(b.x * b.x + b.y * b.y);
    m += r * r * beta_of(r, g.delta, g.dx) * g.dx * g.dy;
  }
  return m;
}

// LPS dispersion of the wave vector (a1, a2): the 2 x 2 matrix M^LPS from the
// discrete S_k and N_jk sums, its eigenvalues (P and S frequencies) and
// eigenvectors (polarisations), :199-342.
Mode dispersion(double a1, double a2, const Material &mc, const std::vector<Bond> &tg, const Geometry &g) {
  Mode mode;
  mode.alpha1 = a1;
  mode.alpha2 = a2;
  std::complex<double> S[2] = {{0, 0}, {0, 0}};
  std::complex<double> N[2][2] = {{{0, 0}, {0, 0}}, {{0, 0}, {0, 0}}};
  for (const Bond &bd : tg) {
    const double xi_x = bd.x, xi_y = bd.y;
    const double xi2 = xi_x * xi_x + xi_y * xi_y;
    const double b = beta_of(std::sqrt(xi2), g.delta, g.dx);
    const double dV = g.dx * g.dy;
    const double phase = a1 * xi_x + a2 * xi_y;
    const std::complex<double> ef(std::cos(phase) - 1.0, std::sin(phase));
    S[0] += xi_x * ef * b * dV;
    S[1] += xi_y * ef * b * dV;
    const double comp[2] = {xi_x, xi_y};
    for (int p = 0; p < 2; p++)
      for (int k = 0; k < 2; k++) N[p][k] += (comp[p] * comp[k] / xi2) * ef * b * dV;
  }
  mode.S_real[0] = S[0].real();
  mode.S_imag[0] = S[0].imag();
  mode.S_real[1] = S[1].real();
  mode.S_imag[1] = S[1].imag();
  const double coeff_S = 2.0 * mc.lambda_pd / mc.m_ref;
  const double coeff_N = 2.0 * mc.alpha_lps;
  double M[2][2];
  for (int p = 0; p < 2; p++)
    for (int k = 0; k < 2; k++) M[p][k] = (coeff_S * S[p] * S[k] + coeff_N * N[p][k]).real();
  const double tr = M[0][0] + M[1][1];
  const double det = M[0][0] * M[1][1] - M[0][1] * M[1][0];
  double disc = tr * tr - 4.0 * det;
  if (disc < 0.0) disc = 0.0;
  const double eig1 = (tr + std::sqrt(disc)) / 2.0;
  const double eig2 = (tr - std::sqrt(disc)) / 2.0;
  const double omP2 = -eig2 / mc.rho, omS2 = -eig1 / mc.rho;
  mode.omega_P = (omP2 > 0.0) ? std::sqrt(omP2) : 0.0;
  mode.omega_S = (omS2 > 0.0) ? std::sqrt(omS2) : 0.0;
  auto eigvec = [&](double eig, double *gamma) {
    const double a00 = M[0][0] - eig, a01 = M[0][1], a10 = M[1][0], a11 = M[1][1] - eig;
    const double r0 = std::abs(a00) + std::abs(a01), r1 = std::abs(a10) + std::abs(a11);
    if (r0 >= r1) {
      gamma[0] = -a01;
      gamma[1] = a00;
    } else {
      gamma[0] = a11;
      gamma[1] = -a10;
    }
    const double norm = std::sqrt(gamma[0] * gamma[0] + gamma[1] * gamma[1]);
    if (norm > 1e-30) {
      gamma[0] /= norm;
      gamma[1] /= norm;
    }
  };
  const double M_norm = std::abs(M[0][0]) + std::abs(M[0][1]) + std::abs(M[1][0]) + std::abs(M[1][1]);
  if (M_norm < 1e-30) {  // alpha = 0: any orthonormal pair
    mode.gamma_P[0] = 1.0;
    mode.gamma_P[1] = 0.0;
    mode.gamma_S[0] = 0.0;
    mode.gamma_S[1] = 1.0;
  } else {
    eigvec(eig2, mode.gamma_P);
    eigvec(eig1, mode.gamma_S);
  }
  return mode;
}

// The wave-vector fan: angles Delta_phi [-1, 1] in steps of 1/5, wavenumbers
// delta_kappa [0, 1] in steps of 1/5, duplicates dropped (:350-366), then
// ordered by |kappa| with the same std::sort call as :985-989.
std::vector<Mode> mode_fan(double delta_kappa, const Material &mc, const std::vector<Bond> &tg, const Geometry &g) {
  std::vector<Mode> modes;
  for (int i_theta = -kModeNSub; i_theta <= kModeNSub; i_theta++) {
    const double theta = kModeDeltaPhi * static_cast<double>(i_theta) / kModeNSub;
    for (int i_k = 0; i_k <= kModeNSub; i_k++) {
      const double kappa_val = delta_kappa * static_cast<double>(i_k) / kModeNSub;
      const double a1 = kappa_val * std::cos(theta);
      const double a2 = kappa_val * std::sin(theta);
      bool duplicate = false;
      for (const Mode &m : modes) {
        const double da1 = m.alpha1 - a1, da2 = m.alpha2 - a2;
        if (std::sqrt(da1 * da1 + da2 * da2) < 1e-12) {
          duplicate = true;
          break;
        }
      }
      if (!duplicate) modes.push_back(dispersion(a1, a2, mc, tg, g));
    }
  }
  std::sort(modes.begin(), modes.end(), [](const Mode &a, const Mode &b) {
    return (a.alpha1 * a.alpha1 + a.alpha2 * a.alpha2) < (b.alpha1 * b.alpha1 + b.alpha2 * b.alpha2);
  });
  return modes;
}

// dgelsd with the reference's workspace query and sizes (:381-402).
int least_squares(lps_dgelsd_fn dgelsd, int m, int n, int nrhs, std::vector<double> &A, std::vector<double> &B,
                  int ldb) {
  int lda = m, info = 0, rank = 0;
  double rcond = kSvdRcond;
  const int min_mn = std::min(m, n);
  std::vector<double> s(std::max(min_mn, 1));
  int lwork = -1, iwork_query = 0;
  double wkopt = 0.0;
  dgelsd(&m, &n, &nrhs, A.data(), &lda, B.data(), &ldb, s.data(), &rcond, &rank, &wkopt, &lwork, &iwork_query,
         &info);
  lwork = static_cast<int>(wkopt);
  std::vector<double> work(std::max(lwork, 1));
  const int nlvl = std::max(1, static_cast<int>(std::log2(min_mn / 26.0)) + 1);
  const int liwork = std::max(1, 3 * min_mn * nlvl + 11 * min_mn);
  std::vector<int> iwork(liwork);
  dgelsd(&m, &n, &nrhs, A.data(), &lda, B.data(), &ldb, s.data(), &rcond, &rank, work.data(), &lwork, iwork.data(),
         &info);
  return info;
}

struct NodeData {
  double x, y, tau;
  std::vector<int> cloud;
};

// G_u and G_v of one absorbing node (:415-637): rows [x-output, y-output] of
// 2 abcs_step max_cloud columns, per cloud entry (x, y) of each time level.
// Returns the number of failed dgelsd calls.
int fit_uv(const NodeData &nd, const double *X, const double *Y, const std::vector<Mode> &modes, int max_cloud,
           double dt_use, const Geometry &g, lps_dgelsd_fn dgelsd, double *gu0, double *gu1, double *gv0,
           double *gv1) {
  const int nCloud = static_cast<int>(nd.cloud.size());
  const int nModes = static_cast<int>(modes.size());
  const int nBasis = 4 * nModes, S = g.abcs_step;
  const double cosT = std::cos(nd.tau), sinT = std::sin(nd.tau);
  const int m_ls = nBasis, n_ls = 2 * nCloud * S, ldb = std::max(m_ls, n_ls);
  std::vector<double> AT_u((size_t)m_ls * n_ls, 0.0), AT_v((size_t)m_ls * n_ls, 0.0);
  auto at = [m_ls](int row, int col) { return (size_t)row + (size_t)col * m_ls; };
  for (int im = 0; im < nModes; im++) {
    const Mode &md = modes[im];
    const double a1 = md.alpha1, a2 = md.alpha2, omP = md.omega_P, omS = md.omega_S;
    const double *gP = md.gamma_P, *gS = md.gamma_S;
    for (int t_level = 0; t_level < S; t_level++) {
      const double t_val = -t_level * dt_use;
      for (int jc = 0; jc < nCloud; jc++) {
        const double dx_g = X[nd.cloud[jc]] - nd.x, dy_g = Y[nd.cloud[jc]] - nd.y;
        const double x_loc = cosT * dx_g + sinT * dy_g;
        const double y_loc = -sinT * dx_g + cosT * dy_g;
        const double phase = a1 * x_loc + a2 * y_loc;
        const double phase_P = phase - omP * t_val, phase_S = phase - omS * t_val;
        const double cos_P = std::cos(phase_P), sin_P = std::sin(phase_P);
        const double cos_S = std::cos(phase_S), sin_S = std::sin(phase_S);
        const int row_base = t_level * (2 * nCloud) + 2 * jc;
        const double disp[4][2] = {{gP[0] * cos_P, gP[1] * cos_P},
                                   {gS[0] * cos_S, gS[1] * cos_S},
                                   {gP[0] * sin_P, gP[1] * sin_P},
                                   {gS[0] * sin_S, gS[1] * sin_S}};
        const double vel[4][2] = {{gP[0] * omP * sin_P, gP[1] * omP * sin_P},
                                  {gS[0] * omS * sin_S, gS[1] * omS * sin_S},
                                  {-gP[0] * omP * cos_P, -gP[1] * omP * cos_P},
                                  {-gS[0] * omS * cos_S, -gS[1] * omS * cos_S}};
        for (int b = 0; b < 4; b++) {
          const int row = 4 * im + b;
          AT_u[at(row, row_base)] = cosT * disp[b][0] - sinT * disp[b][1];
          AT_u[at(row, row_base + 1)] = sinT * disp[b][0] + cosT * disp[b][1];
          AT_v[at(row, row_base)] = cosT * vel[b][0] - sinT * vel[b][1];
          AT_v[at(row, row_base + 1)] = sinT * vel[b][0] + cosT * vel[b][1];
        }
      }
    }
  }
  // targets: the modes at the node (x_loc = 0) at t = +dt (:572-615)
  std::vector<double> tu((size_t)ldb * 2, 0.0), tv((size_t)ldb * 2, 0.0);
  for (int im = 0; im < nModes; im++) {
    const Mode &md = modes[im];
    const double omP = md.omega_P, omS = md.omega_S;
    const double *gP = md.gamma_P, *gS = md.gamma_S;
    const double cos_Pdt = std::cos(-omP * dt_use), sin_Pdt = std::sin(-omP * dt_use);
    const double cos_Sdt = std::cos(-omS * dt_use), sin_Sdt = std::sin(-omS * dt_use);
    const double disp[4][2] = {{gP[0] * cos_Pdt, gP[1] * cos_Pdt},
                               {gS[0] * cos_Sdt, gS[1] * cos_Sdt},
                               {gP[0] * sin_Pdt, gP[1] * sin_Pdt},
                               {gS[0] * sin_Sdt, gS[1] * sin_Sdt}};
    const double vel[4][2] = {{gP[0] * omP * sin_Pdt, gP[1] * omP * sin_Pdt},
                              {gS[0] * omS * sin_Sdt, gS[1] * omS * sin_Sdt},
                              {-gP[0] * omP * cos_Pdt, -gP[1] * omP * cos_Pdt},
                              {-gS[0] * omS * cos_Sdt, -gS[1] * omS * cos_Sdt}};
    for (int b = 0; b < 4; b++) {
      const int row = 4 * im + b;
      tu[row] = cosT * disp[b][0] - sinT * disp[b][1];
      tu[row + ldb] = sinT * disp[b][0] + cosT * disp[b][1];
      tv[row] = cosT * vel[b][0] - sinT * vel[b][1];
      tv[row + ldb] = sinT * vel[b][0] + cosT * vel[b][1];
    }
  }
  int fails = 0;
  fails += least_squares(dgelsd, m_ls, n_ls, 2, AT_u, tu, ldb) != 0;
  fails += least_squares(dgelsd, m_ls, n_ls, 2, AT_v, tv, ldb) != 0;
  const int cols = 2 * S * max_cloud;
  std::fill(gu0, gu0 + cols, 0.0);
  std::fill(gu1, gu1 + cols, 0.0);
  std::fill(gv0, gv0 + cols, 0.0);
  std::fill(gv1, gv1 + cols, 0.0);
  for (int jc = 0; jc < nCloud; jc++)
    for (int tl = 0; tl < S; tl++) {
      const int d = tl * (2 * nCloud) + 2 * jc, c = 2 * S * jc + 2 * tl;
      gu0[c] = tu[d];
      gu0[c + 1] = tu[d + 1];
      gu1[c] = tu[d + ldb];
      gu1[c + 1] = tu[d + 1 + ldb];
      gv0[c] = tv[d];
      gv0[c + 1] = tv[d + 1];
      gv1[c] = tv[d + ldb];
      gv1[c + 1] = tv[d + 1 + ldb];
    }
  return fails;
}

// G_theta of one absorbing node (:657-785): the dilatation of each mode,
// theta_hat = (2 / m_ref) gamma . S, on the same fit.
int fit_theta(const NodeData &nd, const double *X, const double *Y, const std::vector<Mode> &modes, int max_cloud,
              double dt_use, const Geometry &g, const Material &mc, lps_dgelsd_fn dgelsd, double *gth) {
  const int nCloud = static_cast<int>(nd.cloud.size());
  const int nModes = static_cast<int>(modes.size());
  const int nBasis = 4 * nModes, S = g.abcs_step;
  const double cosT = std::cos(nd.tau), sinT = std::sin(nd.tau);
  const int m_ls = nBasis, n_ls = nCloud * S, ldb = std::max(m_ls, n_ls);
  std::vector<double> AT((size_t)m_ls * n_ls, 0.0), tgt((size_t)ldb, 0.0);
  auto at = [m_ls](int row, int col) { return (size_t)row + (size_t)col * m_ls; };
  for (int im = 0; im < nModes; im++) {
    const Mode &md = modes[im];
    const double a1 = md.alpha1, a2 = md.alpha2, omP = md.omega_P, omS = md.omega_S;
    const double *gP = md.gamma_P, *gS = md.gamma_S;
    const double coeff = 2.0 / mc.m_ref;
    const double thP_r = coeff * (gP[0] * md.S_real[0] + gP[1] * md.S_real[1]);
    const double thP_i = coeff * (gP[0] * md.S_imag[0] + gP[1] * md.S_imag[1]);
    const double thS_r = coeff * (gS[0] * md.S_real[0] + gS[1] * md.S_real[1]);
    const double thS_i = coeff * (gS[0] * md.S_imag[0] + gS[1] * md.S_imag[1]);
    for (int t_level = 0; t_level < S; t_level++) {
      const double t_val = -t_level * dt_use;
      for (int jc = 0; jc < nCloud; jc++) {
        const double dx_g = X[nd.cloud[jc]] - nd.x, dy_g = Y[nd.cloud[jc]] - nd.y;
        const double x_loc = cosT * dx_g + sinT * dy_g;
        const double y_loc = -sinT * dx_g + cosT * dy_g;
        const double phase = a1 * x_loc + a2 * y_loc;
        const double phase_P = phase - omP * t_val, phase_S = phase - omS * t_val;
        const double cos_P = std::cos(phase_P), sin_P = std::sin(phase_P);
        const double cos_S = std::cos(phase_S), sin_S = std::sin(phase_S);
        const int row = t_level * nCloud + jc;
        AT[at(4 * im + 0, row)] = thP_r * cos_P - thP_i * sin_P;
        AT[at(4 * im + 1, row)] = thS_r * cos_S - thS_i * sin_S;
        AT[at(4 * im + 2, row)] = thP_r * sin_P + thP_i * cos_P;
        AT[at(4 * im + 3, row)] = thS_r * sin_S + thS_i * cos_S;
      }
    }
    const double cos_Pdt = std::cos(-omP * dt_use), sin_Pdt = std::sin(-omP * dt_use);
    const double cos_Sdt = std::cos(-omS * dt_use), sin_Sdt = std::sin(-omS * dt_use);
    tgt[4 * im + 0] = thP_r * cos_Pdt - thP_i * sin_Pdt;
    tgt[4 * im + 1] = thS_r * cos_Sdt - thS_i * sin_Sdt;
    tgt[4 * im + 2] = thP_r * sin_Pdt + thP_i * cos_Pdt;
    tgt[4 * im + 3] = thS_r * sin_Sdt + thS_i * cos_Sdt;
  }
  const int fails = least_squares(dgelsd, m_ls, n_ls, 1, AT, tgt, ldb) != 0;
  const int cols = S * max_cloud;
  std::fill(gth, gth + cols, 0.0);
  for (int jc = 0; jc < nCloud; jc++)
    for (int tl = 0; tl < S; tl++) gth[S * jc + tl] = tgt[tl * nCloud + jc];
  return fails;
}

// max(||G_u||_F, ||G_v||_F) in the order of :1021-1031.
double g_norm(const double *gu0, const double *gu1, const double *gv0, const double *gv1, int cols) {
  double sq_u = 0.0, sq_v = 0.0;
  for (int c = 0; c < cols; c++) {
    sq_u += gu0[c] * gu0[c] + gu1[c] * gu1[c];
    sq_v += gv0[c] * gv0[c] + gv1[c] * gv1[c];
  }
  return std::max(std::sqrt(sq_u), std::sqrt(sq_v));
}

}  // namespace

extern "C" int lps_abcfit(const lps_abcfit_params *p, const double *nodes, int32_t n_nodes, const int32_t *abc_nodes,
                          int32_t n_abc, const int32_t *clouds, int32_t max_cloud, lps_dgelsd_fn dgelsd, double *gu,
                          double *gv, double *gtheta, lps_abcfit_result *out) {
  if (!p || !nodes || n_nodes <= 0 || n_abc < 0 || (n_abc > 0 && (!abc_nodes || !clouds || !gu || !gv || !gtheta)) ||
      max_cloud <= 0 || !dgelsd || !out || (p->abcs_step != 1 && p->abcs_step != 2) || !(p->rho > 0.0) ||
      !(p->dx > 0.0) || !(p->dy > 0.0) || !(p->delta > 0.0) || (!p->sweep && !(p->dt > 0.0)))
    return -1;
  const int nthreads = p->n_threads > 0 ? p->n_threads : omp_get_max_threads();
  const Geometry g{p->delta, p->dx, p->dy, p->abcs_step};
  // material constants, :95-125 and the nu override of :809-817
  Material mc{};
  mc.E = p->E;
  mc.nu = p->nu;
  mc.rho = p->rho;
  mc.lambda = mc.E * mc.nu / ((1.0 + mc.nu) * (1.0 - 2.0 * mc.nu));
  mc.mu = mc.E / (2.0 * (1.0 + mc.nu));
  mc.kappa = mc.lambda + mc.mu;
  mc.c_P = std::sqrt((mc.lambda + 2.0 * mc.mu) / mc.rho);
  const std::vector<Bond> tg = template_grid(g);
  mc.m_ref = reference_volume(tg, g);
  mc.alpha_lps = 8.0 * mc.mu / mc.m_ref;
  mc.lambda_pd = 2.0 * (mc.lambda - mc.mu) / mc.m_ref;
  // absorbing nodes: position, outward normal angle (:869-872) and cloud
  std::vector<NodeData> nd(n_abc);
  std::vector<double> X(n_nodes), Y(n_nodes);
  for (int i = 0; i < n_nodes; i++) {
    X[i] = nodes[2 * i];
    Y[i] = nodes[2 * i + 1];
  }
  for (int i = 0; i < n_abc; i++) {
    const int node = abc_nodes[i];
    if (node < 0 || node >= n_nodes) return -1;
    nd[i].x = X[node];
    nd[i].y = Y[node];
    nd[i].tau = std::atan2(Y[node], X[node]);
    for (int j = 0; j < max_cloud; j++) {
      const int k = clouds[(size_t)i * max_cloud + j];
      if (k == -1) continue;
      if (k < 0 || k >= n_nodes) return -1;
      nd[i].cloud.push_back(k);
    }
  }
  const double dk_base = 1.0 / std::sqrt(mc.c_P);  // :907
  const int cols = 2 * g.abcs_step * max_cloud;
  int dgelsd_failures = 0;
  double dt_opt = p->dt, dk_opt = dk_base * p->dk_factor, best_maxG = 0.0;
  int stable_found = 1;
  if (p->sweep) {
    // sample: every node with a cloud of at most 26 entries, the first 20 and
    // the last 20 (:1051-1057)
    std::vector<int> sample;
    for (int i = 0; i < n_abc; i++)
      if ((int)nd[i].cloud.size() <= 26) sample.push_back(i);
    for (int i = 0; i < std::min(20, (int)n_abc); i++) sample.push_back(i);
    for (int i = std::max(0, (int)n_abc - 20); i < n_abc; i++) sample.push_back(i);
    std::sort(sample.begin(), sample.end());
    sample.erase(std::unique(sample.begin(), sample.end()), sample.end());
    static const double dk_factors[] = {0.3, 0.5, 0.7, 0.8, 0.9, 1.0, 1.1, 1.2, 1.5, 2.0};
    static const double dt_values[] = {5.0e-9,  8.0e-9,  10.0e-9, 12.0e-9, 14.0e-9, 15.0e-9, 16.0e-9,
                                       17.0e-9, 17.5e-9, 18.0e-9, 20.0e-9, 25.0e-9, 30.0e-9, 35.0e-9};
    constexpr int n_dk = 10, n_dt = 14;
    std::vector<std::vector<Mode>> fans(n_dk);
    for (int idk = 0; idk < n_dk; idk++) fans[idk] = mode_fan(dk_base * dk_factors[idk], mc, tg, g);
    // every point walks the sample in order and stops once max ||G|| > 1.5,
    // as :1093-1108 does; the points run in parallel
    std::vector<double> maxG(n_dk * n_dt, 0.0);
    int fails = 0;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads) reduction(+ : fails)
    for (int pt = 0; pt < n_dk * n_dt; pt++) {
      const int idk = pt / n_dt, idt = pt % n_dt;
      std::vector<double> b0(cols), b1(cols), b2(cols), b3(cols);
      double mg = 0.0;
      for (int idx : sample) {
        fails += fit_uv(nd[idx], X.data(), Y.data(), fans[idk], max_cloud, dt_values[idt], g, dgelsd, b0.data(),
                        b1.data(), b2.data(), b3.data());
        mg = std::max(mg, g_norm(b0.data(), b1.data(), b2.data(), b3.data(), cols));
        if (mg > 1.5) break;
      }
      maxG[pt] = mg;
    }
    dgelsd_failures += fails;
    // the stable point with the largest max ||G|| (first in sweep order on a
    // tie); without one, the smallest max ||G|| (:1142-1158)
    double best_score = -1.0;
    int best = -1;
    for (int pt = 0; pt < n_dk * n_dt; pt++)
      if (maxG[pt] <= 1.0 && maxG[pt] > best_score) {
        best_score = maxG[pt];
        best = pt;
      }
    if (best < 0) {
      stable_found = 0;
      double min_G = 1e10;
      for (int pt = 0; pt < n_dk * n_dt; pt++)
        if (maxG[pt] < min_G) {
          min_G = maxG[pt];
          best = pt;
        }
    }
    dt_opt = dt_values[best % n_dt];
    dk_opt = dk_base * dk_factors[best / n_dt];
    best_maxG = maxG[best];
  }
  const std::vector<Mode> modes = mode_fan(dk_opt, mc, tg, g);
  // the operators of every absorbing node (:1183-1268)
  const int cth = g.abcs_step * max_cloud;
  int fails = 0;
  std::vector<double> norm_u(n_abc, 0.0), norm_v(n_abc, 0.0), norm_t(n_abc, 0.0);
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads) reduction(+ : fails)
  for (int i = 0; i < n_abc; i++) {
    double *u0 = gu + (size_t)(2 * i) * cols, *u1 = gu + (size_t)(2 * i + 1) * cols;
    double *v0 = gv + (size_t)(2 * i) * cols, *v1 = gv + (size_t)(2 * i + 1) * cols;
    fails += fit_uv(nd[i], X.data(), Y.data(), modes, max_cloud, dt_opt, g, dgelsd, u0, u1, v0, v1);
    fails += fit_theta(nd[i], X.data(), Y.data(), modes, max_cloud, dt_opt, g, mc, dgelsd,
                       gtheta + (size_t)i * cth);
    double su = 0.0, sv = 0.0, st = 0.0;
    for (int c = 0; c < cols; c++) {
      su += u0[c] * u0[c] + u1[c] * u1[c];
      sv += v0[c] * v0[c] + v1[c] * v1[c];
    }
    for (int c = 0; c < cth; c++) st += gtheta[(size_t)i * cth + c] * gtheta[(size_t)i * cth + c];
    norm_u[i] = std::sqrt(su);
    norm_v[i] = std::sqrt(sv);
    norm_t[i] = std::sqrt(st);
  }
  dgelsd_failures += fails;
  out->dt = dt_opt;
  out->delta_kappa = dk_opt;
  out->dk_factor = dk_opt / dk_base;
  out->sweep_max_g = best_maxG;
  out->max_norm_gu = out->max_norm_gv = out->max_norm_gtheta = 0.0;
  out->n_failed = 0;
  for (int i = 0; i < n_abc; i++) {
    out->max_norm_gu = std::max(out->max_norm_gu, norm_u[i]);
    out->max_norm_gv = std::max(out->max_norm_gv, norm_v[i]);
    out->max_norm_gtheta = std::max(out->max_norm_gtheta, norm_t[i]);
    out->n_failed += std::max(norm_u[i], norm_v[i]) > kGNormTarget;
  }
  out->m_ref = mc.m_ref;
  out->n_steps = static_cast<int>(std::ceil(kTFinal / dt_opt));
  out->n_modes = static_cast<int>(modes.size());
  out->stable_found = stable_found;
  out->dgelsd_failures = dgelsd_failures;
  out->pad = 0;
  return 0;
}
