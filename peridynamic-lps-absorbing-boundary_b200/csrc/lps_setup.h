// lps_setup.h -- host-side setup of one instance (runs once in lps_create).
#pragma once
#include <string>
#include <vector>

#include "lps_cuda.h"

namespace lps {

struct InstanceSetup {
  int n = 0, n_abc = 0, cloud = 0;
  double lam = 0, mu = 0, kappa = 0;       // src/main.cpp:215-217
  double m_ref = 0, m_min = 0;             // :442
  double alpha = 0, lambda_pd = 0;         // :485-486
  double domain_radius = 0, out_r = -1;    // :518-530
  double dt_lps = 0;                       // :555-581 (sampled, informational)
  int n_corrected = 0;                     // :473-475
  int max_len = 0;                         // longest horizon incl. self
  double horizon_ms = 0;                   // wall time of the horizon search
  int horizon_on_gpu = 0;                  // 1: lps_horizons.cu did it
  int row_len = 0;                         // columns of hz (the max_horizon option)
  std::vector<int> hz_len;                 // [n] horizon length incl. self
  std::vector<int> hz;                     // [n][row_len], col 0 = self, -1 padded
  std::vector<double> m;                   // weighted volume after the ABC override
};

// Builds horizons (src/main.cpp:352-354 semantics), applies prenotch
// visibility (:386-402), computes m_i, m_ref, the ABC override and the LPS
// constants with the reference's consistency checks.  Returns an LPS_* status
// and fills err on failure.
int setup_instance(const lps_problem &p, const lps_options &o, InstanceSetup &s,
                   std::string &err);

// Neighbour search: every node within radius r of node i (Euclidean, as
// kd_tree_interface.h:91), sorted by (distance, index) so self is column 0.
// Returns the longest row, or LPS_ERR_HORIZON if a row exceeds row_len.
int build_horizons(int n, const double *xy, double r, int row_len, std::vector<int> &len,
                   std::vector<int> &hz);
// The same search on the current CUDA device (lps_horizons.cu); the same
// result, or LPS_ERR_CUDA.
int build_horizons_gpu(int n, const double *xy, double r, int row_len, std::vector<int> &len,
                       std::vector<int> &hz);

}  // namespace lps
