// lps_api.cu -- the C ABI (include/lps_cuda.h): handle, batch packing, state
// rings, CUDA-graph replay and the diagnostics log.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "lps_cuda.h"
#include "lps_dense.cuh"
#include "lps_kernels.cuh"
#include "lps_setup.h"

using namespace lps;

namespace {

thread_local std::string g_create_error;

template <class T>
struct DevBuf {
  T *p = nullptr;
  size_t n = 0;
};

}  // namespace

namespace lps {
// Error text for entry points that have no handle (read by lps_last_error(NULL)).
void set_create_error(const char *msg) { g_create_error = msg; }
}  // namespace lps

struct lps_handle {
  lps_options opt{};
  int n_inst = 0;
  int path = LPS_PATH_CSR;
  std::string err;
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::vector<void *> allocs;
  int64_t device_bytes = 0;

  // per instance (host copies)
  std::vector<InstanceSetup> setup;
  std::vector<InstParams> params;
  std::vector<int> node_begin, node_count, abc_begin, abc_count;
  std::vector<double> E0;
  std::vector<std::vector<DiagRecord>> drained;  // records pulled off the device, not yet read

  // device layout
  LaunchGeo lg{};
  DenseGeo dg{};
  int n_total = 0, n_abc_total = 0;
  std::vector<int> local_of_global;  // for dense: cell -> local node index

  // state
  double2 *U[kUring] = {}, *V[3] = {}, *A[2] = {}, *VH = nullptr, *S = nullptr;
  int ring_u = 3;             // displacement ring depth: 3 (CSR path) or 4 (dense path)
  double *TH[3] = {};
  double2 *U0 = nullptr, *V0 = nullptr;
  bool fp32 = false;          // the FP32-mixed form
  float2 *U32[2] = {};        // FP32-mixed form: FP32 copies of the predicted level, by step parity
  float2 *coef32 = nullptr;   // FP32-mixed form: (q, q) with q = m_ref / m_i; (0, -1) where m_i <= 0
  float2 *AB32 = nullptr;     // FP32-mixed CSR form: force coefficients (A', B'), written with theta
  float *AP32 = nullptr;      // FP32-mixed dense form: force coefficient plane A', written with theta
  float *BP32 = nullptr;      // FP32-mixed dense form: static force coefficient plane B' = q
  // diagnostics
  DiagPartial *partials = nullptr;
  DiagRecord *log = nullptr;
  int *log_count = nullptr;
  int *d_step = nullptr;
  int log_capacity = 0;
  int pending_records = 0;  // records per instance on the device since the last drain

  int64_t step = 0;          // steps taken since reset
  int64_t launches = 0;
  std::map<int, cudaGraphExec_t> graphs;  // key: diag mask of the captured steps
  std::map<int, int> graph_kernels;
};

namespace {

const char *status_text(int s) {
  switch (s) {
    case LPS_OK: return "ok";
    case LPS_ERR_INVALID_ARG: return "invalid argument";
    case LPS_ERR_HORIZON: return "horizon longer than max_horizon";
    case LPS_ERR_NONFINITE: return "energy or displacement is NaN/Inf";
    case LPS_ERR_LAME: return "Lame parameter consistency check failed";
    case LPS_ERR_LAMBDA_PD: return "lambda_PD consistency check failed";
    case LPS_ERR_CUDA: return "CUDA error";
    case LPS_ERR_NOMEM: return "out of memory";
    case LPS_ERR_UNSUPPORTED: return "unsupported option combination";
    case LPS_ERR_NO_DEVICE: return "no usable CUDA device";
    default: return "unknown status";
  }
}

#define LPS_CUDA_TRY(h, expr)                                                          \
  do {                                                                                 \
    cudaError_t e_ = (expr);                                                           \
    if (e_ != cudaSuccess) {                                                           \
      (h)->err = std::string(#expr) + ": " + cudaGetErrorString(e_);                  \
      return LPS_ERR_CUDA;                                                             \
    }                                                                                  \
  } while (0)

template <class T>
int dev_alloc(lps_handle *h, T **p, size_t n) {
  *p = nullptr;
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void **)p, n * sizeof(T));
  if (e != cudaSuccess) {
    h->err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? LPS_ERR_NOMEM : LPS_ERR_CUDA;
  }
  h->allocs.push_back(*p);
  h->device_bytes += (int64_t)(n * sizeof(T));
  return LPS_OK;
}

template <class T>
int dev_upload(lps_handle *h, T **p, const std::vector<T> &v) {
  int s = dev_alloc(h, p, v.size());
  if (s) return s;
  if (!v.empty()) LPS_CUDA_TRY(h, cudaMemcpy(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return LPS_OK;
}

inline int round_up(int x, int m) { return (x + m - 1) / m * m; }

// ---------------------------------------------------------------------------
// Batch packing shared by both paths: per-instance ABC lists.
struct HostAbc {
  std::vector<int> node, inst, cl_off, cl_len, cl_idx, idw_off, idw_len, idw_idx;
  std::vector<uint8_t> writes, active;
  std::vector<double> gu, gv, idw_w;
  std::vector<double> gth;
};

// Appends instance k's absorbing-boundary data.  `gmap(local)` maps a local
// node index to the global node (or cell) index of the packed layout.
template <class Map>
void pack_abc(const lps_problem &p, const lps_options &o, const InstanceSetup &s, int k, Map gmap,
              int begin, HostAbc &H, std::vector<int> &abc_of_global, std::vector<uint8_t> &type) {
  const bool abc_on = o.abcs_step != -1 && p.n_abc > 0;
  const int na = abc_on ? p.n_abc : 0;
  const int C = p.max_cloud;
  const int cpc = (o.abcs_step == 1) ? 2 : 4;       // G columns per cloud entry
  const int cth = (o.abcs_step == 1) ? 1 : 2;       // G_theta columns per entry
  const size_t cols = (size_t)cpc * C;
  // the last active entry of a node is the one whose write survives
  std::vector<int> last(p.n_nodes, -1);
  for (int i = 0; i < na; i++)
    if (p.bctypes[2 * p.inf_nodes[i]] == 1) last[p.inf_nodes[i]] = i;
  for (int i = 0; i < na; i++) {
    const int node = p.inf_nodes[i];
    const int a = begin + i;
    const bool active = p.bctypes[2 * node] == 1;
    const bool writes = active && last[node] == i;
    H.node[a] = gmap(node);
    H.inst[a] = k;
    H.active[a] = active;
    H.writes[a] = writes;
    H.cl_off[a] = (int)H.cl_idx.size();
    // entries with k != -1, then the operators component-major (see lps_abc.cuh)
    std::vector<int> js;
    for (int j = 0; j < C; j++)
      if (p.clouds[(size_t)i * C + j] != -1) js.push_back(j);
    // segments have an even length (a zero-weight entry on the node itself
    // pads odd clouds) so that every operator row starts 16-byte aligned
    const int len = (int)js.size() + ((int)js.size() & 1);
    for (int j : js) H.cl_idx.push_back(gmap(p.clouds[(size_t)i * C + j]));
    if (writes)
      for (int j : js) type[gmap(p.clouds[(size_t)i * C + j])] |= kKeepState;
    if (len > (int)js.size()) H.cl_idx.push_back(gmap(node));
    const double *g0 = p.gu + (size_t)(2 * i) * cols, *g1 = p.gu + (size_t)(2 * i + 1) * cols;
    const double *h0 = p.gv + (size_t)(2 * i) * cols, *h1 = p.gv + (size_t)(2 * i + 1) * cols;
    for (int r = 0; r < 8; r++) {
      const int c = r & 3;  // column within the entry: x^n, y^n, x^{n-1}, y^{n-1}
      for (int j : js) {
        H.gu.push_back(c < cpc ? (r < 4 ? g0 : g1)[cpc * j + c] : 0.0);
        H.gv.push_back(c < cpc ? (r < 4 ? h0 : h1)[cpc * j + c] : 0.0);
      }
      if (len > (int)js.size()) {
        H.gu.push_back(0.0);
        H.gv.push_back(0.0);
      }
    }
    for (int r = 0; r < 2; r++) {
      for (int j : js) {
        double w = 0.0;
        if (o.theta_method == 1 && p.gtheta && r < cth) w = p.gtheta[(size_t)i * cth * C + cth * j + r];
        H.gth.push_back(w);
      }
      if (len > (int)js.size()) H.gth.push_back(0.0);
    }
    H.cl_len[a] = len;
    // inverse-distance lists, src/main.cpp:775-786
    H.idw_off[a] = (int)H.idw_idx.size();
    int il = 0;
    if (writes && o.theta_method == 0) {
      for (int j = 1; j < s.hz_len[node]; j++) {
        const int nb = s.hz[(size_t)node * s.row_len + j];
        if (nb == -1) continue;
        if (p.bctypes[2 * nb] == 1) continue;
        const double rx = p.nodes[2 * nb] - p.nodes[2 * node];
        const double ry = p.nodes[2 * nb + 1] - p.nodes[2 * node + 1];
        const double dist = std::sqrt(rx * rx + ry * ry);
        H.idw_idx.push_back(gmap(nb));
        type[gmap(nb)] |= kKeepState;
        H.idw_w.push_back(1.0 / (dist + 1e-30));
        il++;
      }
    }
    H.idw_len[a] = il;
    if (writes) {
      abc_of_global[gmap(node)] = a;
      type[gmap(node)] |= kActiveAbc;
    }
  }
}

void fill_params(InstParams &P, const lps_problem &p, const lps_options &o, const InstanceSetup &s) {
  memset(&P, 0, sizeof P);
  P.dt = p.dt;
  P.half_dt = p.dt / 2.0;
  P.rho = p.rho;
  P.lam = s.lam;
  P.mu = s.mu;
  P.kappa = s.kappa;
  P.c_lm = 2.0 * (s.lam - s.mu);
  P.c_mu8 = 8.0 * s.mu;
  P.c_mu4 = 4.0 * s.mu;
  P.dx = p.dx;
  P.dy = p.dy;
  P.delta = p.delta;
  P.beta_lo = p.delta - p.dx / 2.0;
  P.beta_hi = p.delta + p.dx / 2.0;
  P.out_r = s.out_r;
  P.f32_b0 = s.alpha;
  P.f32_ab = (s.lam - s.mu) / (4.0 * s.mu);
  P.mref = s.m_ref;
  P.kinematic = o.kinematic_v;
  P.theta_method = o.theta_method;
  P.abcs_step = o.abcs_step;
}

int upload_abc(lps_handle *h, const HostAbc &H, int total_abc, const std::vector<int> &abc_of) {
  Abc &B = h->lg.abc;
  int s;
  int *a_node, *a_inst, *a_cl_off, *a_cl_len, *a_cl_idx, *a_idw_off, *a_idw_len, *a_idw_idx;
  uint8_t *a_writes, *a_active;
  double *a_gu, *a_gv, *a_idw_w;
  double *a_gth;
  // which cloud entries are themselves G_u-written nodes (their u^n lives in
  // the previous step's G_u result until the next predictor merges it)
  if ((s = dev_upload(h, &a_node, H.node)) || (s = dev_upload(h, &a_inst, H.inst)) ||
      (s = dev_upload(h, &a_cl_off, H.cl_off)) || (s = dev_upload(h, &a_cl_len, H.cl_len)) ||
      (s = dev_upload(h, &a_cl_idx, H.cl_idx)) || (s = dev_upload(h, &a_idw_off, H.idw_off)) ||
      (s = dev_upload(h, &a_idw_len, H.idw_len)) || (s = dev_upload(h, &a_idw_idx, H.idw_idx)) ||
      (s = dev_upload(h, &a_writes, H.writes)) || (s = dev_upload(h, &a_active, H.active)) ||
      (s = dev_upload(h, &a_gu, H.gu)) || (s = dev_upload(h, &a_gv, H.gv)) ||
      (s = dev_upload(h, &a_idw_w, H.idw_w)) || (s = dev_upload(h, &a_gth, H.gth)))
    return s;
  B.n_abc = total_abc;
  B.node = a_node; B.inst = a_inst; B.cl_off = a_cl_off; B.cl_len = a_cl_len; B.cl_idx = a_cl_idx;
  B.idw_off = a_idw_off; B.idw_len = a_idw_len; B.idw_idx = a_idw_idx; B.writes = a_writes;
  B.active = a_active; B.gu = a_gu; B.gv = a_gv; B.idw_w = a_idw_w; B.gth = a_gth;
  return LPS_OK;
}

// Dense path: the sliced-ELL copy of the operators (see Abc::sell_g).
int upload_abc_sell(lps_handle *h, const HostAbc &H) {
  Abc &B = h->lg.abc;
  std::vector<int> ents;
  for (size_t a = 0; a < H.writes.size(); a++)
    if (H.writes[a]) ents.push_back((int)a);
  // longest clouds first; equal lengths keep their order (neighbouring
  // entries share cloud nodes)
  std::stable_sort(ents.begin(), ents.end(), [&](int x, int y) { return H.cl_len[x] > H.cl_len[y]; });
  const int n_sl = ((int)ents.size() + 31) / 32;
  std::vector<SellSlice> sl(n_sl);
  std::vector<double> g;
  std::vector<int> ix, sa((size_t)n_sl * 32, -1);
  for (int s = 0; s < n_sl; s++) {
    int len = 1;
    for (int l = 0; l < 32 && 32 * s + l < (int)ents.size(); l++) len = std::max(len, H.cl_len[ents[32 * s + l]]);
    sl[s].goff = (long long)g.size();
    sl[s].ioff = (long long)ix.size();
    sl[s].len = len;
    sl[s].pad = 0;
    g.resize(g.size() + (size_t)len * 18 * 32, 0.0);
    ix.resize(ix.size() + (size_t)len * 32, H.node[ents[32 * s]]);
    double *gs = g.data() + sl[s].goff;
    int *is = ix.data() + sl[s].ioff;
    for (int l = 0; l < 32 && 32 * s + l < (int)ents.size(); l++) {
      const int a = ents[32 * s + l];
      sa[(size_t)32 * s + l] = a;
      const size_t o = H.cl_off[a];
      const int la = H.cl_len[a];
      // past its own cloud a lane reads its own node with zero weights, so a
      // NaN in another instance of the slice cannot reach it
      for (int e = la; e < len; e++) is[(size_t)e * 32 + l] = H.node[a];
      for (int e = 0; e < la; e++) {
        is[(size_t)e * 32 + l] = H.cl_idx[o + e];
        for (int r = 0; r < 8; r++) {
          gs[((size_t)e * 18 + r) * 32 + l] = H.gu[8 * o + (size_t)r * la + e];
          gs[((size_t)e * 18 + 8 + r) * 32 + l] = H.gv[8 * o + (size_t)r * la + e];
        }
        for (int r = 0; r < 2; r++) gs[((size_t)e * 18 + 16 + r) * 32 + l] = H.gth[2 * o + (size_t)r * la + e];
      }
    }
  }
  SellSlice *d_sl;
  double *d_g;
  int *d_ix, *d_sa;
  int s;
  if ((s = dev_upload(h, &d_sl, sl)) || (s = dev_upload(h, &d_g, g)) || (s = dev_upload(h, &d_ix, ix)) ||
      (s = dev_upload(h, &d_sa, sa)))
    return s;
  B.n_slices = n_sl;
  B.slices = d_sl;
  B.sell_g = d_g;
  B.sell_idx = d_ix;
  B.sell_a = d_sa;
  return LPS_OK;
}

// ---------------------------------------------------------------------------
int build_csr(lps_handle *h, const lps_problem *probs) {
  const int K = h->n_inst;
  // node ranges
  int total = 0, total_abc = 0, width = 0;
  for (int k = 0; k < K; k++) {
    h->node_begin[k] = total;
    h->node_count[k] = probs[k].n_nodes;
    total += round_up(probs[k].n_nodes, kNodeBlock);
    const bool abc_on = h->opt.abcs_step != -1 && probs[k].n_abc > 0;
    h->abc_begin[k] = total_abc;
    h->abc_count[k] = abc_on ? probs[k].n_abc : 0;
    total_abc += round_up(h->abc_count[k], kNodeBlock);
    width = std::max(width, h->setup[k].max_len - 1);
  }
  width = std::max(width, 1);
  h->n_total = total;
  h->n_abc_total = total_abc;
  std::vector<double2> xy(total, make_double2(0, 0)), coef(total, make_double2(0, -1));
  std::vector<float2> coef32(total, make_float2(0.f, -1.f));
  std::vector<uint8_t> type(total, 0);
  std::vector<int> abc_of(total, -1), len(total, 0), nbr((size_t)width * total, -1);
  std::vector<double> m(total, 0.0);
  std::vector<int> blk_inst(total / kNodeBlock, 0);
  HostAbc H;
  H.node.assign(total_abc, 0); H.inst.assign(total_abc, 0);
  H.cl_off.assign(total_abc, 0); H.cl_len.assign(total_abc, 0);
  H.idw_off.assign(total_abc, 0); H.idw_len.assign(total_abc, 0);
  H.writes.assign(total_abc, 0); H.active.assign(total_abc, 0);
  for (int k = 0; k < K; k++) {
    const lps_problem &p = probs[k];
    const InstanceSetup &s = h->setup[k];
    const int nb0 = h->node_begin[k];
    for (int b = nb0 / kNodeBlock; b < (nb0 + round_up(p.n_nodes, kNodeBlock)) / kNodeBlock; b++) blk_inst[b] = k;
    for (int i = 0; i < p.n_nodes; i++) {
      const int g = nb0 + i;
      xy[g] = make_double2(p.nodes[2 * i], p.nodes[2 * i + 1]);
      type[g] = kExists | (p.bctypes[2 * i] == 1 ? kBcAbc : 0);
      m[g] = s.m[i];
      if (s.m[i] > 0.0) {  // src/main.cpp:857-863 coefficients, same division
        coef[g] = make_double2(2.0 * (s.lam - s.mu) / s.m[i], 8.0 * s.mu / s.m[i]);
        const float q = (float)(s.m_ref / s.m[i]);  // FP32-mixed form, as on the dense path
        coef32[g] = make_float2(q, q);
      }
      int l = 0;
      for (int j = 1; j < s.hz_len[i]; j++) {
        const int nb = s.hz[(size_t)i * s.row_len + j];
        nbr[(size_t)l * total + g] = nb < 0 ? -1 : nb0 + nb;
        l++;
      }
      len[g] = l;
    }
    for (int a = h->abc_begin[k]; a < h->abc_begin[k] + round_up(h->abc_count[k], kNodeBlock); a++) {
      H.inst[a] = k;
      H.node[a] = nb0;
    }
    // padding entries keep writes = active = 0
    pack_abc(p, h->opt, s, k, [nb0](int i) { return nb0 + i; }, h->abc_begin[k], H, abc_of, type);
    fill_params(h->params[k], p, h->opt, s);
    h->params[k].node_begin = nb0;
    h->params[k].node_count = p.n_nodes;
    h->params[k].abc_begin = h->abc_begin[k];
    h->params[k].abc_count = h->abc_count[k];
    int nact = 0;
    for (int i = 0; i < h->abc_count[k]; i++) nact += p.bctypes[2 * p.inf_nodes[i]] == 1;
    h->params[k].n_active_abc = nact;
  }
  // upload
  Geo &G = h->lg.geo;
  G.n_total = total;
  G.ell_width = width;
  double2 *d_xy, *d_coef;
  uint8_t *d_type;
  int *d_abc_of, *d_len, *d_nbr, *d_blk;
  double *d_m;
  int s;
  if ((s = dev_upload(h, &d_xy, xy)) || (s = dev_upload(h, &d_coef, coef)) ||
      (s = dev_upload(h, &d_type, type)) || (s = dev_upload(h, &d_abc_of, abc_of)) ||
      (s = dev_upload(h, &d_len, len)) || (s = dev_upload(h, &d_nbr, nbr)) ||
      (s = dev_upload(h, &d_blk, blk_inst)) || (s = dev_upload(h, &d_m, m)))
    return s;
  G.xy = d_xy; G.coef = d_coef; G.type = d_type; G.abc_of = d_abc_of; G.len = d_len;
  G.nbr = d_nbr; G.blk_inst = d_blk; G.m = d_m;
  if (h->fp32 && (s = dev_upload(h, &h->coef32, coef32))) return s;
  if ((s = upload_abc(h, H, total_abc, abc_of))) return s;
  h->lg.n_node_blocks = total / kNodeBlock;
  h->lg.n_abc_blocks = total_abc / kAbcWarpsPerBlock;
  h->lg.n_inst = K;
  h->lg.theta_method = h->opt.theta_method;
  h->lg.abcs_step = h->opt.abcs_step;
  return LPS_OK;
}

// ---------------------------------------------------------------------------
// Dense path: lattice detection and the padded-grid layout.
struct Lattice {
  int M = 0, NR = 0, NC = 0;
  std::vector<int> ix, iy;
};

// True when instance p sits exactly on a dx = dy lattice with delta = M dx,
// M in kDenseM, no prenotch, and the reference's horizon search
// (src/main.cpp:352) admits exactly the stencil offsets of M.
bool lattice_of(const lps_problem &p, const InstanceSetup &s, Lattice &L) {
  if (p.n_prenotch > 0 || p.dx != p.dy) return false;
  const double mr = p.delta / p.dx;
  const int M = (int)std::llround(mr);
  if (M <= 0 || std::abs(mr - M) > 1e-12 * mr || !dense_m_supported(M)) return false;
  std::vector<int> A, B;
  dense_offsets(M, A, B);
  const double r = p.delta + p.dx / 2.0 + 1e-5;
  int admitted = 0;
  for (int a = -M - 2; a <= M + 2; a++)
    for (int b = -M - 2; b <= M + 2; b++) {
      if (a == 0 && b == 0) continue;
      const double x = a * p.dx, y = b * p.dy;
      const bool in_ref = std::sqrt(x * x + y * y) <= r;
      const bool in_sten = a * a + b * b <= M * M + M;
      if (in_ref != in_sten) return false;
      admitted += in_ref;
    }
  if (admitted != (int)A.size()) return false;
  const int N = p.n_nodes;
  double x0 = p.nodes[0], y0 = p.nodes[1];
  for (int i = 1; i < N; i++) {
    x0 = std::min(x0, p.nodes[2 * i]);
    y0 = std::min(y0, p.nodes[2 * i + 1]);
  }
  L.M = M;
  L.ix.resize(N);
  L.iy.resize(N);
  long mx = 0, my = 0;
  for (int i = 0; i < N; i++) {
    const double x = p.nodes[2 * i], y = p.nodes[2 * i + 1];
    const long ix = std::lround((x - x0) / p.dx), iy = std::lround((y - y0) / p.dy);
    if (std::abs(x0 + ix * p.dx - x) > 1e-13 * (std::abs(x) + std::abs(x0) + p.dx)) return false;
    if (std::abs(y0 + iy * p.dy - y) > 1e-13 * (std::abs(y) + std::abs(y0) + p.dy)) return false;
    if (ix > (1 << 20) || iy > (1 << 20)) return false;
    L.ix[i] = (int)ix;
    L.iy[i] = (int)iy;
    mx = std::max(mx, ix);
    my = std::max(my, iy);
  }
  L.NR = (int)mx + 1;
  L.NC = (int)my + 1;
  if ((double)L.NR * L.NC > 2.0e9) return false;
  std::vector<int> seen((size_t)L.NR * L.NC, -1);
  for (int i = 0; i < N; i++) {
    int &c = seen[(size_t)L.ix[i] * L.NC + L.iy[i]];
    if (c >= 0) return false;  // two nodes in one cell
    c = i;
  }
  // the host horizons must be exactly the existing stencil neighbours
  for (int i = 0; i < N; i++) {
    int cnt = 1;
    for (size_t j = 0; j < A.size(); j++) {
      const long jx = L.ix[i] + A[j], jy = L.iy[i] + B[j];
      if (jx >= 0 && jx < L.NR && jy >= 0 && jy < L.NC && seen[(size_t)jx * L.NC + jy] >= 0) cnt++;
    }
    if (cnt != s.hz_len[i]) return false;
  }
  return true;
}

bool dense_possible(const lps_problem *probs, int K, const std::vector<InstanceSetup> &setup,
                    std::vector<Lattice> &lat) {
  lat.assign(K, Lattice());
  std::map<int, std::pair<double, double>> spacing;  // one constant set per M
  for (int k = 0; k < K; k++) {
    if (!lattice_of(probs[k], setup[k], lat[k])) return false;
    auto it = spacing.find(lat[k].M);
    if (it == spacing.end())
      spacing[lat[k].M] = {probs[k].dx, probs[k].delta};
    else if (it->second.first != probs[k].dx || it->second.second != probs[k].delta)
      return false;
  }
  return true;
}

int build_dense(lps_handle *h, const lps_problem *probs, const std::vector<Lattice> &lat) {
  const int K = h->n_inst;
  DenseGeo &D = h->dg;
  D.host_cell_of_node.assign(K, {});
  D.host_node_of_cell_v.assign(K, {});
  D.host_cells.assign(K, 0);
  D.host_cell_begin.assign(K, 0);
  // one pitch for the batch (multiple of 32 cells, at least one tile width of
  // slack past the padded lattice so the 48-byte type boxes stay in the row)
  int P = 0;
  for (int k = 0; k < K; k++)
    P = std::max(P, round_up(round_up(lat[k].NC, kTileCols) + 2 * lat[k].M, 32));
  std::vector<int> rows(K), cols(K), row_begin(K);
  long total_rows = 0;
  int total_abc = 0;
  for (int k = 0; k < K; k++) {
    const int M = lat[k].M;
    const int NRt = round_up(lat[k].NR, kTileRows);
    rows[k] = round_up(NRt + 2 * M, 8);  // 8 rows x 32k cells: bands start on 256-cell blocks
    cols[k] = round_up(lat[k].NC, kTileCols);
    row_begin[k] = (int)total_rows;
    total_rows += rows[k];
    D.host_cell_begin[k] = row_begin[k] * P;
    D.host_cells[k] = rows[k] * P;
    h->node_begin[k] = D.host_cell_begin[k];
    h->node_count[k] = probs[k].n_nodes;
    const bool abc_on = h->opt.abcs_step != -1 && probs[k].n_abc > 0;
    h->abc_begin[k] = total_abc;
    h->abc_count[k] = abc_on ? probs[k].n_abc : 0;
    total_abc += round_up(h->abc_count[k], kNodeBlock);
  }
  if (total_rows * (long)P > 2000000000L) {
    h->err = "lps_create: dense layout larger than 2^31 cells";
    return LPS_ERR_UNSUPPORTED;
  }
  const int n = (int)(total_rows * P);
  D.pitch = P;
  D.total_rows = (int)total_rows;
  h->n_total = n;
  h->n_abc_total = total_abc;
  std::vector<double2> xy(n, make_double2(0, 0)), coef(n, make_double2(0, -1));
  std::vector<float2> coef32(n, make_float2(0.f, -1.f));
  std::vector<uint8_t> type(n, 0);
  std::vector<int> abc_of(n, -1), blk_inst(n / kNodeBlock, 0);
  std::vector<double> m(n, 0.0);
  HostAbc H;
  H.node.assign(total_abc, 0); H.inst.assign(total_abc, 0);
  H.cl_off.assign(total_abc, 0); H.cl_len.assign(total_abc, 0);
  H.idw_off.assign(total_abc, 0); H.idw_len.assign(total_abc, 0);
  H.writes.assign(total_abc, 0); H.active.assign(total_abc, 0);
  for (int k = 0; k < K; k++) {
    const lps_problem &p = probs[k];
    const InstanceSetup &s = h->setup[k];
    const int M = lat[k].M, c0 = D.host_cell_begin[k];
    for (int b = c0 / kNodeBlock; b < (c0 + D.host_cells[k]) / kNodeBlock; b++) blk_inst[b] = k;
    auto &cell_of = D.host_cell_of_node[k];
    auto &node_of = D.host_node_of_cell_v[k];
    cell_of.resize(p.n_nodes);
    node_of.assign(D.host_cells[k], -1);
    for (int i = 0; i < p.n_nodes; i++) {
      const int c = c0 + (lat[k].ix[i] + M) * P + (lat[k].iy[i] + M);
      cell_of[i] = c;
      node_of[c - c0] = i;
      xy[c] = make_double2(p.nodes[2 * i], p.nodes[2 * i + 1]);
      type[c] = kExists | (p.bctypes[2 * i] == 1 ? kBcAbc : 0);
      m[c] = s.m[i];
      if (s.m[i] > 0.0) {
        coef[c] = make_double2(2.0 * (s.lam - s.mu) / s.m[i], 8.0 * s.mu / s.m[i]);
        // FP32-mixed form: both coefficients relative to their full-horizon
        // values, m_ref / m_i -- exactly 1 wherever m_i = m_ref, so the
        // material constants never round to FP32
        const float q = (float)(s.m_ref / s.m[i]);
        coef32[c] = make_float2(q, q);
      }
    }
    for (int a = h->abc_begin[k]; a < h->abc_begin[k] + round_up(h->abc_count[k], kNodeBlock); a++) {
      H.inst[a] = k;
      H.node[a] = c0;
    }
    pack_abc(p, h->opt, s, k, [&cell_of](int i) { return cell_of[i]; }, h->abc_begin[k], H, abc_of, type);
    fill_params(h->params[k], p, h->opt, s);
    InstParams &Pp = h->params[k];
    Pp.node_begin = c0;
    Pp.node_count = D.host_cells[k];
    Pp.abc_begin = h->abc_begin[k];
    Pp.abc_count = h->abc_count[k];
    int nact = 0;
    for (int i = 0; i < h->abc_count[k]; i++) nact += p.bctypes[2 * p.inf_nodes[i]] == 1;
    Pp.n_active_abc = nact;
    Pp.dense = 1;
    Pp.pitch = P;
    Pp.nrow = lat[k].NR;
    Pp.ncol = lat[k].NC;
    Pp.stencil = M;
  }
  // tiles: owned lattice rows [r0, r0+16) x columns [q0, q0+32); the staged
  // region starts m rows and m columns earlier
  std::vector<DenseTile> tiles;
  for (int k = 0; k < K; k++) {
    const int M = lat[k].M;
    std::vector<int> A, B;
    dense_offsets(M, A, B);
    const int NRt = round_up(lat[k].NR, kTileRows);
    for (int r0 = 0; r0 < NRt; r0 += kTileRows)
      for (int q0 = 0; q0 < cols[k]; q0 += kTileCols) {
        const int region_row = row_begin[k] + r0, region_col = q0;
        const long first = (long)(region_row + M) * P + region_col + M;
        bool any = false, full = true;
        for (int r = 0; r < kTileRows; r++)
          for (int q = 0; q < kTileCols; q++) {
            const long c = first + (long)r * P + q;
            if (!(type[c] & kExists)) continue;
            any = true;
            for (size_t j = 0; j < A.size() && full; j++)
              if (!(type[c + (long)A[j] * P + B[j]] & kExists)) full = false;
          }
        if (any) {
          int flags = full ? kTileFull : 0;
          if (full && h->fp32 && dense32_tile_deep(M, type, coef32, P, first)) flags |= kTileDeep32;
          tiles.push_back(DenseTile{region_row, region_col, k, flags});
        }
      }
  }
  std::stable_sort(tiles.begin(), tiles.end(), [&](const DenseTile &x, const DenseTile &y) {
    return lat[x.inst].M < lat[y.inst].M;
  });
  // each instance's tiles are contiguous (sorted by m, stable): its range
  for (int k = 0; k < K; k++) {
    h->params[k].tile_begin = 0;
    h->params[k].tile_count = 0;
  }
  for (int i = (int)tiles.size() - 1; i >= 0; i--) {
    InstParams &Pk = h->params[tiles[i].inst];
    Pk.tile_begin = i;
    Pk.tile_count++;
  }
  D.groups.clear();
  for (int i = 0; i < (int)tiles.size(); i++) {
    const int M = lat[tiles[i].inst].M;
    if (D.groups.empty() || D.groups.back().m != M) {
      D.groups.emplace_back();
      D.groups.back().m = M;
      D.groups.back().tile_begin = i;
      D.groups.back().n_tiles = 0;
    }
    D.groups.back().n_tiles++;
  }
  // upload
  Geo &G = h->lg.geo;
  G.n_total = n;
  G.ell_width = 0;
  double2 *d_xy, *d_coef;
  uint8_t *d_type;
  int *d_abc_of, *d_blk;
  double *d_m;
  DenseTile *d_tiles;
  int st;
  if ((st = dev_upload(h, &d_xy, xy)) || (st = dev_upload(h, &d_coef, coef)) ||
      (st = dev_upload(h, &d_type, type)) || (st = dev_upload(h, &d_abc_of, abc_of)) ||
      (st = dev_upload(h, &d_blk, blk_inst)) || (st = dev_upload(h, &d_m, m)) ||
      (st = dev_upload(h, &d_tiles, tiles)))
    return st;
  G.xy = d_xy; G.coef = d_coef; G.type = d_type; G.abc_of = d_abc_of; G.blk_inst = d_blk; G.m = d_m;
  G.len = nullptr; G.nbr = nullptr;
  D.tiles = d_tiles;
  D.fp32 = h->fp32;
  if (D.fp32) {
    // static per-cell corrections of the FP32-mixed tile kernels
    std::vector<float2> w32(n, make_float2(0.f, 0.f));
    std::vector<float4> ka32(n, make_float4(0.f, 0.f, 0.f, 0.f));
    for (int k = 0; k < K; k++)
      dense32_static(lat[k].M, type, P, D.host_cell_begin[k], D.host_cells[k], w32, ka32);
    // B' = q where the cell exists with m_i > 0, else 0
    std::vector<float> bp32(n, 0.f);
    for (int c = 0; c < n; c++) bp32[c] = coef32[c].y > 0.f ? coef32[c].y : 0.f;
    float2 *d_w32;
    float4 *d_ka32;
    if ((st = dev_upload(h, &h->BP32, bp32)) || (st = dev_upload(h, &d_w32, w32)) ||
        (st = dev_upload(h, &d_ka32, ka32)))
      return st;
    D.d32.bp32 = h->BP32;
    D.d32.w32 = d_w32;
    D.d32.ka32 = d_ka32;
  }
  if ((st = upload_abc(h, H, total_abc, abc_of))) return st;
  if ((st = upload_abc_sell(h, H))) return st;
  std::map<int, int> done;
  for (int k = 0; k < K; k++) {
    if (done.count(lat[k].M)) continue;
    done[lat[k].M] = 1;
    LPS_CUDA_TRY(h, upload_dense_constants(lat[k].M, probs[k].dx, probs[k].dy, probs[k].delta, h->stream));
  }
  LPS_CUDA_TRY(h, dense_prepare(D));
  h->lg.n_node_blocks = n / kNodeBlock;
  h->lg.n_abc_blocks = total_abc / kAbcWarpsPerBlock;
  h->lg.n_inst = K;
  h->lg.theta_method = h->opt.theta_method;
  h->lg.abcs_step = h->opt.abcs_step;
  return LPS_OK;
}

// Dense path, after the state buffers exist: TMA descriptors, the forked
// stream for the absorbing-boundary kernels and the device error flag.
int finish_dense(lps_handle *h) {
  DenseGeo &D = h->dg;
  const double2 *coef = h->lg.geo.coef;
  const uint8_t *type = h->lg.geo.type;
  for (auto &gr : D.groups) {
    const int s = dense_encode_maps(gr, D.pitch, D.total_rows, h->U, h->TH, coef, type, D.fp32 ? h->U32 : nullptr,
                                    h->AP32, h->BP32, h->err);
    if (s) return s;
  }
  LPS_CUDA_TRY(h, cudaStreamCreateWithFlags(&D.side, cudaStreamNonBlocking));
  for (int i = 0; i < 2; i++) {
    LPS_CUDA_TRY(h, cudaEventCreateWithFlags(&D.ev_fork[i], cudaEventDisableTiming));
    LPS_CUDA_TRY(h, cudaEventCreateWithFlags(&D.ev_join[i], cudaEventDisableTiming));
  }
  int s;
  if ((s = dev_alloc(h, &D.d_err, 1))) return s;
  LPS_CUDA_TRY(h, cudaMemset(D.d_err, 0, sizeof(int)));
  // tile-scheduler counters: per group (theta next, done, force next, done)
  int *sched = nullptr;
  const size_t n_sched = 4 * D.groups.size();
  if ((s = dev_alloc(h, &sched, n_sched))) return s;
  LPS_CUDA_TRY(h, cudaMemset(sched, 0, n_sched * sizeof(int)));
  for (size_t g = 0; g < D.groups.size(); g++) D.groups[g].sched = sched + 4 * g;
  D.sched = sched;
  D.n_sched = (int)n_sched;
  return LPS_OK;
}

// ---------------------------------------------------------------------------
// Ring indices of step s (1-based) whose current level is n = s - 1.
StepPtrs step_ptrs(lps_handle *h, int64_t n) {
  StepPtrs p;
  const int R = h->ring_u;
  const int u0 = (int)(n % 3), u1 = (int)((n + 1) % 3), um = (int)((n + 2) % 3);
  const int a0 = (int)(n % 2), a1 = (int)((n + 1) % 2);
  p.u_n = h->U[n % R];
  p.u_nm1 = h->U[(n + R - 1) % R];
  p.u_np1 = h->U[(n + 1) % R];
  p.u_np2 = h->U[(n + 2) % R];
  p.th_ring = u1;
  p.full = 1;
  p.v_n = h->V[u0];
  p.v_nm1 = h->V[um];
  p.v_np1 = h->V[u1];
  p.a_n = h->A[a0];
  p.a_np1 = h->A[a1];
  p.vh = h->VH;
  p.th_n = h->TH[u0];
  p.th_nm1 = h->TH[um];
  p.th_np1 = h->TH[u1];
  p.u32_np1 = h->U32[(n + 1) % 2];
  p.u32_np2 = h->U32[n % 2];
  p.s_abc = h->S;
  return p;
}

// Kernels of one step (and its diagnostics); returns the launch count.
// `mark`, when set, is called after each launch with the kernel's name.
int enqueue_step(lps_handle *h, int64_t n, bool diag, bool full, const Mark *mark = nullptr) {
  StepPtrs p = step_ptrs(h, n);
  p.full = (diag || full) ? 1 : 0;
  cudaStream_t st = h->stream;
  auto M = [&](const char *name) {
    if (mark) (*mark)(name);
  };
  int k = 0;
  if (h->path == LPS_PATH_DENSE) {
    k += enqueue_dense_step(h->dg, h->lg, p, h->d_step, st, mark, (int)((n + 1) % h->ring_u));
  } else {
    launch_predict_csr(h->lg, p, st);
    M("predict_csr");
    if (h->fp32) {
      launch_theta_csr32(h->lg, p.u32_np1, p.th_np1, h->AB32, h->coef32, p.th_n, p.th_nm1, st);
      M("theta_csr32");
    } else {
      launch_theta_csr(h->lg, p.u_np1, p.th_np1, p.th_n, p.th_nm1, true, st);
      M("theta_csr");
    }
    k += 2;
    if (h->opt.abcs_step != -1 && h->opt.theta_method == 0 && h->lg.abc.n_abc > 0) {
      launch_theta_idw(h->lg, p.th_np1, st, h->AB32, h->coef32);
      M("theta_idw");
      k++;
    }
    if (h->fp32) {
      launch_force_csr32(h->lg, p, h->AB32, h->d_step, st);
      M("force_csr32");
    } else {
      launch_force_csr(h->lg, p, h->d_step, st);
      M("force_csr");
    }
    k++;
  }
  if (diag) {
    // the dense step merges G_u results into the ring itself (k_abc_predict)
    const bool abc = h->opt.abcs_step != -1 && h->lg.abc.n_abc > 0 && h->path != LPS_PATH_DENSE;
    if (abc) {
      launch_merge_abc(h->lg, p.u_np1, p.s_abc, st);
      M("merge_abc");
      k++;
    }
    if (h->path == LPS_PATH_DENSE) {
      launch_diag_dense(h->dg, h->lg, (int)((n + 1) % h->ring_u), p.u_np1, p.v_np1, p.a_np1, p.th_np1,
                        h->partials, h->log, h->log_count, h->log_capacity, h->d_step, st);
      k += (int)h->dg.groups.size() + (h->lg.abc.n_abc > 0 ? 1 : 0) + 1;  // tiles per group, ABC, finish
    } else {
      launch_diag_csr(h->lg, p.u_np1, p.v_np1, p.a_np1, p.th_np1, h->partials, h->log, h->log_count,
                      h->log_capacity, h->d_step, st);
      k += 2;
    }
    M("diag");
  }
  return k;
}

int do_reset(lps_handle *h);
int check_device_error(lps_handle *h);
int get_graph(lps_handle *h, int mask, cudaGraphExec_t *out);

// The autotuner of the dense path: for each number of rows a dilatation
// thread owns (4 and 2; only the requested one when lps_options.theta_rows
// is set), each number of rows a FP32-mixed force thread owns (2 and 4; only
// the requested one when lps_options.force_rows is set) and every count of
// resident dilatation / force CTAs per SM (1 up to the occupancy limit) it
// captures the 12-step CUDA graph the run will replay and times two replays
// of it from the initial state (the faster of two tries); a choice replaces
// the default (4 / 2 rows, full occupancy) only if it is at least 2 % faster.  None of these changes a result: tiles come from
// a counter and each cell's arithmetic is the same whichever CTA and thread
// computes it.  The caller resets the state afterwards.
int autotune_dense(lps_handle *h, int rows_only, int force_rows_only) {
  int max_f[2] = {1, 0}, max_t[2] = {1, 1};  // [0]: two-row force / four-row dilatation, [1]: the other form
  for (const auto &gr : h->dg.groups) {
    max_t[0] = std::max(max_t[0], gr.max_theta_ctas);
    max_t[1] = std::max(max_t[1], gr.max_theta_ctas2);
    max_f[0] = std::max(max_f[0], gr.max_force_ctas);
    max_f[1] = std::max(max_f[1], gr.max_force_ctas4);
  }
  // the two timing events, destroyed on every return path
  struct EventPair {
    cudaEvent_t e[2] = {nullptr, nullptr};
    ~EventPair() {
      for (cudaEvent_t x : e)
        if (x) cudaEventDestroy(x);
    }
  } ev;
  LPS_CUDA_TRY(h, cudaEventCreate(&ev.e[0]));
  LPS_CUDA_TRY(h, cudaEventCreate(&ev.e[1]));
  cudaEvent_t e0 = ev.e[0], e1 = ev.e[1];
  auto drop_graphs = [h]() {
    for (auto &g : h->graphs) cudaGraphExecDestroy(g.second);
    h->graphs.clear();
    h->graph_kernels.clear();
  };
  auto time_choice = [&](int rows, int t, int fr, int f, float *ms_out) -> int {
    dense_set_ctas(h->dg, rows, t, f, fr);
    drop_graphs();
    cudaGraphExec_t ex;
    int st = get_graph(h, 0, &ex);
    if (st) return st;
    float best = 1e30f;
    for (int rep = 0; rep < 2; rep++) {
      if ((st = do_reset(h))) return st;
      LPS_CUDA_TRY(h, cudaGraphLaunch(ex, h->stream));  // warm
      LPS_CUDA_TRY(h, cudaEventRecord(e0, h->stream));
      LPS_CUDA_TRY(h, cudaGraphLaunch(ex, h->stream));
      LPS_CUDA_TRY(h, cudaGraphLaunch(ex, h->stream));
      LPS_CUDA_TRY(h, cudaEventRecord(e1, h->stream));
      LPS_CUDA_TRY(h, cudaEventSynchronize(e1));
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      best = std::min(best, ms);
    }
    *ms_out = best;
    return LPS_OK;
  };
  const int rows0 = rows_only == 2 ? 2 : 4, r0 = rows0 == 4 ? 0 : 1;
  const int fr0 = force_rows_only == 4 && max_f[1] > 0 ? 4 : 2, f0 = fr0 == 2 ? 0 : 1;
  float ref = 0.f;
  int st = time_choice(rows0, max_t[r0], fr0, max_f[f0], &ref);
  float best = ref;
  int best_r = rows0, best_t = max_t[r0], best_fr = fr0, best_f = max_f[f0];
  for (int rows : {4, 2}) {
    if (rows_only && rows != rows_only) continue;
    const int mt = max_t[rows == 4 ? 0 : 1];
    for (int fr : {2, 4}) {
      if ((force_rows_only && fr != force_rows_only) || max_f[fr == 2 ? 0 : 1] == 0) continue;
      const int mf = max_f[fr == 2 ? 0 : 1];
      for (int t = 1; t <= mt && st == LPS_OK; t++)
        for (int f = 1; f <= mf && st == LPS_OK; f++) {
          if (rows == rows0 && t == mt && fr == fr0 && f == mf) continue;
          float ms = 0.f;
          if ((st = time_choice(rows, t, fr, f, &ms))) break;
          if (ms < best && ms < 0.98f * ref) {
            best = ms;
            best_r = rows;
            best_t = t;
            best_fr = fr;
            best_f = f;
          }
        }
    }
  }
  drop_graphs();
  if (st == LPS_OK) st = check_device_error(h);
  if (st) return st;
  dense_set_ctas(h->dg, best_r, best_t, best_f, best_fr);
  return LPS_OK;
}

int drain_log(lps_handle *h) {
  if (h->pending_records == 0) return LPS_OK;
  LPS_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  std::vector<int> cnt(h->n_inst);
  LPS_CUDA_TRY(h, cudaMemcpy(cnt.data(), h->log_count, sizeof(int) * h->n_inst, cudaMemcpyDeviceToHost));
  std::vector<DiagRecord> buf((size_t)h->n_inst * h->log_capacity);
  LPS_CUDA_TRY(h, cudaMemcpy(buf.data(), h->log, sizeof(DiagRecord) * buf.size(), cudaMemcpyDeviceToHost));
  for (int k = 0; k < h->n_inst; k++) {
    const int c = std::min(cnt[k], h->log_capacity);
    h->drained[k].insert(h->drained[k].end(), buf.begin() + (size_t)k * h->log_capacity,
                         buf.begin() + (size_t)k * h->log_capacity + c);
  }
  LPS_CUDA_TRY(h, cudaMemsetAsync(h->log_count, 0, sizeof(int) * h->n_inst, h->stream));
  h->pending_records = 0;
  return LPS_OK;
}

// Steps per captured graph: the least common multiple of the ring depths, so
// a graph that starts on a multiple of it finds every buffer where it
// captured it.
int graph_period(const lps_handle *h) { return h->ring_u == 4 ? 12 : 6; }
constexpr int kFullBit = 16;  // graph masks: bits 0..11 diagnostics, 16..27 full steps

int check_device_error(lps_handle *h) {
  if (h->path != LPS_PATH_DENSE || !h->dg.d_err) return LPS_OK;
  int e = 0;
  LPS_CUDA_TRY(h, cudaMemcpy(&e, h->dg.d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) {
    h->err = "a device-side wait on a tile copy timed out";
    return LPS_ERR_CUDA;
  }
  return LPS_OK;
}

int get_graph(lps_handle *h, int mask, cudaGraphExec_t *out) {
  auto it = h->graphs.find(mask);
  if (it != h->graphs.end()) {
    *out = it->second;
    return LPS_OK;
  }
  cudaGraph_t g;
  LPS_CUDA_TRY(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  int kernels = 0;
  // mask bit r: diagnostics after step r; bit kFullBit + r: step r is full
  // (StepPtrs::full) without diagnostics
  for (int r = 0; r < graph_period(h); r++)
    kernels += enqueue_step(h, r, (mask >> r) & 1, (mask >> (kFullBit + r)) & 1);
  LPS_CUDA_TRY(h, cudaStreamEndCapture(h->stream, &g));
  cudaGraphExec_t ex;
  cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    h->err = std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e);
    return LPS_ERR_CUDA;
  }
  h->graphs[mask] = ex;
  h->graph_kernels[mask] = kernels;
  *out = ex;
  return LPS_OK;
}

__global__ void k_reset_state(int n, const double2 *u0, const double2 *v0, double2 *u_cur, double2 *u_prev,
                              double2 *v_cur, double2 *v_prev, double2 *a_cur, double *th_prev) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  u_cur[i] = u0[i];
  v_cur[i] = v0[i];
  u_prev[i] = make_double2(0.0, 0.0);   // Unm1 = 0, src/main.cpp:632
  v_prev[i] = make_double2(0.0, 0.0);   // Udnm1 = 0, :630
  a_cur[i] = make_double2(0.0, 0.0);    // Uddn = 0, :628
  th_prev[i] = 0.0;                     // ThetaNm1 = 0, :681
}

__global__ void k_reset_abc(Abc ab, const double2 *u0, double2 *s) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= ab.n_abc) return;
  s[a] = ab.writes[a] ? u0[ab.node[a]] : make_double2(0.0, 0.0);
}

int do_reset(lps_handle *h) {
  cudaStream_t st = h->stream;
  const int n = h->n_total;
  // a device-side wait that timed out left its flag set and the tile kernels
  // idle; clear it and the tile-scheduler counters so the handle runs again
  if (h->path == LPS_PATH_DENSE && h->dg.d_err) {
    LPS_CUDA_TRY(h, cudaStreamSynchronize(st));
    LPS_CUDA_TRY(h, cudaMemsetAsync(h->dg.d_err, 0, sizeof(int), st));
    if (h->dg.sched) LPS_CUDA_TRY(h, cudaMemsetAsync(h->dg.sched, 0, sizeof(int) * h->dg.n_sched, st));
  }
  k_reset_state<<<(n + 255) / 256, 256, 0, st>>>(n, h->U0, h->V0, h->U[0], h->U[h->ring_u - 1], h->V[0],
                                                  h->V[2], h->A[0], h->TH[2]);
  LPS_CUDA_TRY(h, cudaMemsetAsync(h->TH[0], 0, sizeof(double) * n, st));
  if (h->n_abc_total > 0)
    k_reset_abc<<<(h->n_abc_total + 255) / 256, 256, 0, st>>>(h->lg.abc, h->U0, h->S);
  // theta history from u^0 at every node (no override), src/main.cpp:664-682
  if (h->opt.theta_method == 1) {
    if (h->path == LPS_PATH_DENSE)
      launch_theta_dense_init(h->dg, h->lg, h->U[0], h->TH[0], st);
    else
      launch_theta_csr(h->lg, h->U[0], h->TH[0], nullptr, nullptr, false, st);
  }
  // dense path: G_theta runs a step ahead, so the first one runs here
  if (h->path == LPS_PATH_DENSE && h->opt.theta_method == 1 && h->opt.abcs_step != -1)
    launch_abc_theta_dense(h->dg, h->lg, h->TH[0], h->TH[2], h->TH[1], st);
  // dense path: the force pass predicts the next level, so level 1 is
  // predicted here (src/main.cpp:727 with a^0 = 0)
  if (h->path == LPS_PATH_DENSE) launch_dense_reset_predict(h->lg, h->U0, h->V0, h->U[1], h->U32[1], h->VH, st);
  LPS_CUDA_TRY(h, cudaMemsetAsync(h->d_step, 0, sizeof(int), st));
  LPS_CUDA_TRY(h, cudaMemsetAsync(h->log_count, 0, sizeof(int) * h->n_inst, st));
  LPS_CUDA_TRY(h, cudaGetLastError());
  h->pending_records = 0;
  h->step = 0;
  for (int k = 0; k < h->n_inst; k++) {
    h->E0[k] = -1.0;
    h->drained[k].clear();
  }
  return LPS_OK;
}

int alloc_state(lps_handle *h) {
  const int n = h->n_total;
  int s;
  for (int r = 0; r < h->ring_u; r++) {
    if ((s = dev_alloc(h, &h->U[r], n))) return s;
    LPS_CUDA_TRY(h, cudaMemset(h->U[r], 0, sizeof(double2) * n));
  }
  for (int r = 0; r < 3; r++) {
    if ((s = dev_alloc(h, &h->V[r], n)) || (s = dev_alloc(h, &h->TH[r], n))) return s;
    LPS_CUDA_TRY(h, cudaMemset(h->V[r], 0, sizeof(double2) * n));
    LPS_CUDA_TRY(h, cudaMemset(h->TH[r], 0, sizeof(double) * n));
  }
  for (int r = 0; r < 2; r++) {
    if ((s = dev_alloc(h, &h->A[r], n))) return s;
    LPS_CUDA_TRY(h, cudaMemset(h->A[r], 0, sizeof(double2) * n));
  }
  if ((s = dev_alloc(h, &h->VH, n)) || (s = dev_alloc(h, &h->S, std::max(h->n_abc_total, 1))) ||
      (s = dev_alloc(h, &h->U0, n)) || (s = dev_alloc(h, &h->V0, n)))
    return s;
  LPS_CUDA_TRY(h, cudaMemset(h->VH, 0, sizeof(double2) * n));
  if (h->fp32) {
    for (int r = 0; r < 2; r++) {
      if ((s = dev_alloc(h, &h->U32[r], n))) return s;
      LPS_CUDA_TRY(h, cudaMemset(h->U32[r], 0, sizeof(float2) * n));
    }
    // force coefficients, zero at absent cells (the dense kernels rely on it):
    // (A', B') pairs on the neighbour-list path, the A' plane on the dense path
    if (h->path == LPS_PATH_DENSE) {
      if ((s = dev_alloc(h, &h->AP32, n))) return s;
      LPS_CUDA_TRY(h, cudaMemset(h->AP32, 0, sizeof(float) * n));
      h->dg.d32.ap32 = h->AP32;
    } else {
      if ((s = dev_alloc(h, &h->AB32, n))) return s;
      LPS_CUDA_TRY(h, cudaMemset(h->AB32, 0, sizeof(float2) * n));
    }
  }
  // diagnostics partials: node blocks (CSR) or tiles (dense), then ABC blocks
  int n_tiles = 0;
  for (const auto &gr : h->dg.groups) n_tiles = std::max(n_tiles, gr.tile_begin + gr.n_tiles);
  const int n_part = std::max(h->lg.n_node_blocks, n_tiles) + (h->n_abc_total + kNodeBlock - 1) / kNodeBlock + 1;
  h->log_capacity = 1024;
  if ((s = dev_alloc(h, &h->partials, n_part)) ||
      (s = dev_alloc(h, &h->log, (size_t)h->n_inst * h->log_capacity)) ||
      (s = dev_alloc(h, &h->log_count, h->n_inst)) || (s = dev_alloc(h, &h->d_step, 1)))
    return s;
  return LPS_OK;
}

// Host-side interleaved (x,y) arrays -> node layout of the packed batch.
void scatter_ic(lps_handle *h, int k, const double *src, std::vector<double2> &dst) {
  const int n = h->node_count[k];
  if (h->path == LPS_PATH_DENSE) {
    const int *cell = h->dg.host_cell_of_node[k].data();
    for (int i = 0; i < n; i++) dst[cell[i]] = make_double2(src[2 * i], src[2 * i + 1]);
  } else {
    const int b = h->node_begin[k];
    for (int i = 0; i < n; i++) dst[b + i] = make_double2(src[2 * i], src[2 * i + 1]);
  }
}

int global_of(const lps_handle *h, int k, int i) {
  return h->path == LPS_PATH_DENSE ? h->dg.host_cell_of_node[k][i] : h->node_begin[k] + i;
}

void destroy_all(lps_handle *h) {
  if (!h) return;
  for (auto &g : h->graphs) cudaGraphExecDestroy(g.second);
  h->graphs.clear();
  for (void *p : h->allocs) cudaFree(p);
  h->allocs.clear();
  for (int i = 0; i < 2; i++) {
    if (h->dg.ev_fork[i]) cudaEventDestroy(h->dg.ev_fork[i]);
    if (h->dg.ev_join[i]) cudaEventDestroy(h->dg.ev_join[i]);
    h->dg.ev_fork[i] = h->dg.ev_join[i] = nullptr;
  }
  if (h->dg.side) cudaStreamDestroy(h->dg.side);
  h->dg.side = nullptr;
  if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
  h->stream = nullptr;
}

}  // namespace

// ===========================================================================
extern "C" {

void lps_default_options(lps_options *o) {
  if (!o) return;
  memset(o, 0, sizeof *o);
  o->abcs_step = 2;
  o->theta_method = 1;
  o->kinematic_v = 0;
  o->max_horizon = 128;
  o->precision = LPS_FP64;
  o->path = LPS_PATH_AUTO;
  o->device = 0;
  o->use_graphs = 1;
  o->stream = nullptr;
}

const char *lps_status_string(int s) { return status_text(s); }

const char *lps_last_error(const lps_handle *h) {
  return h ? h->err.c_str() : g_create_error.c_str();
}

int lps_create(const lps_problem *problems, int n_instances, const lps_options *opt, lps_handle **out) {
  g_create_error.clear();
  if (!out || !problems || n_instances <= 0) {
    g_create_error = "lps_create: bad arguments (need at least one instance and an output pointer)";
    return LPS_ERR_INVALID_ARG;
  }
  *out = nullptr;
  lps_options o;
  if (opt) o = *opt; else lps_default_options(&o);
  if (o.max_horizon <= 1) o.max_horizon = 128;
  if (o.horizon_build < 0 || o.horizon_build > 2) {
    g_create_error = "lps_create: horizon_build must be 0, 1 or 2";
    return LPS_ERR_INVALID_ARG;
  }
  if (o.theta_rows != 0 && o.theta_rows != 2 && o.theta_rows != 4) {
    g_create_error = "lps_create: theta_rows must be 0, 2 or 4";
    return LPS_ERR_INVALID_ARG;
  }
  if (o.force_rows != 0 && o.force_rows != 2 && o.force_rows != 4) {
    g_create_error = "lps_create: force_rows must be 0, 2 or 4";
    return LPS_ERR_INVALID_ARG;
  }
  if (o.precision != LPS_FP64 && o.precision != LPS_FP32_MIXED) {
    g_create_error = "lps_create: precision must be LPS_FP64 or LPS_FP32_MIXED";
    return LPS_ERR_INVALID_ARG;
  }
  if (o.theta_method != 0 && o.theta_method != 1) {
    g_create_error = "lps_create: theta_method must be 0 or 1";
    return LPS_ERR_INVALID_ARG;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0 || o.device < 0 || o.device >= ndev) {
    g_create_error = "lps_create: no CUDA device";
    return LPS_ERR_NO_DEVICE;
  }
  lps_handle *h = new lps_handle();
  h->opt = o;
  h->fp32 = o.precision == LPS_FP32_MIXED;
  h->n_inst = n_instances;
  h->device = o.device;
  auto fail = [&](int s) {
    g_create_error = h->err;
    destroy_all(h);
    delete h;
    return s;
  };
  if (cudaSetDevice(o.device) != cudaSuccess) {
    h->err = "cudaSetDevice failed";
    return fail(LPS_ERR_NO_DEVICE);
  }
  {
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, o.device);
    if (prop.major != 10) {
      h->err = std::string("lps_create: this library is built for sm_100a; device is ") + prop.name;
      return fail(LPS_ERR_NO_DEVICE);
    }
  }
  if (o.stream) {
    h->stream = (cudaStream_t)o.stream;
  } else {
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
      h->err = "cudaStreamCreate failed";
      return fail(LPS_ERR_CUDA);
    }
    h->own_stream = true;
  }
  const int K = n_instances;
  h->setup.resize(K);
  h->params.resize(K);
  h->node_begin.resize(K);
  h->node_count.resize(K);
  h->abc_begin.resize(K);
  h->abc_count.resize(K);
  h->E0.assign(K, -1.0);
  h->drained.resize(K);
  for (int k = 0; k < K; k++) {
    int s = setup_instance(problems[k], o, h->setup[k], h->err);
    if (s) {
      if (K > 1) h->err = "instance " + std::to_string(k) + ": " + h->err;
      return fail(s);
    }
  }
  // path choice: dense when every instance maps onto a lattice
  int s = LPS_OK;
  std::vector<Lattice> lat;
  const bool dense_ok = o.path != LPS_PATH_CSR && dense_possible(problems, K, h->setup, lat);
  if (o.path == LPS_PATH_DENSE && !dense_ok) {
    h->err = "lps_create: dense path requested but an instance is not an exact dx = dy lattice "
             "with delta/dx in {2,3,4,5,6,8} and no prenotch";
    return fail(LPS_ERR_UNSUPPORTED);
  }
  if (dense_ok) {
    h->path = LPS_PATH_DENSE;
    h->ring_u = kUring;
    s = build_dense(h, problems, lat);
  } else {
    h->path = LPS_PATH_CSR;
    s = build_csr(h, problems);
  }
  if (s) return fail(s);
  // per-instance constant table: device memory of this handle
  {
    InstParams *d_ip = nullptr;
    if ((s = dev_upload(h, &d_ip, h->params))) return fail(s);
    h->lg.geo.ip = d_ip;
    h->lg.abc.ip = d_ip;
  }
  if ((s = alloc_state(h))) return fail(s);
  if (h->path == LPS_PATH_DENSE && (s = finish_dense(h))) return fail(s);
  // initial conditions
  {
    std::vector<double2> u0(h->n_total, make_double2(0, 0)), v0(h->n_total, make_double2(0, 0));
    for (int k = 0; k < K; k++) {
      scatter_ic(h, k, problems[k].u0, u0);
      scatter_ic(h, k, problems[k].v0, v0);
    }
    if (cudaMemcpy(h->U0, u0.data(), sizeof(double2) * h->n_total, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(h->V0, v0.data(), sizeof(double2) * h->n_total, cudaMemcpyHostToDevice) != cudaSuccess) {
      h->err = "upload of initial conditions failed";
      return fail(LPS_ERR_CUDA);
    }
  }
  if ((s = do_reset(h))) return fail(s);
  if (h->path == LPS_PATH_DENSE && (o.theta_rows == 2 || o.force_rows == 4))
    dense_set_ctas(h->dg, o.theta_rows == 2 ? 2 : 4, 1 << 20, 1 << 20, o.force_rows == 4 ? 4 : 2);
  if (o.autotune && h->path == LPS_PATH_DENSE && (s = autotune_dense(h, o.theta_rows, o.force_rows)))
    return fail(s);
  if (o.autotune && h->path == LPS_PATH_DENSE && (s = do_reset(h))) return fail(s);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) {
    h->err = std::string("setup kernels failed: ") + cudaGetErrorString(cudaGetLastError());
    return fail(LPS_ERR_CUDA);
  }
  *out = h;
  return LPS_OK;
}

int lps_set_initial(lps_handle *h, int instance, const double *u0, const double *v0) {
  if (!h || instance < 0 || instance >= h->n_inst) return LPS_ERR_INVALID_ARG;
  const int n = h->node_count[instance];
  std::vector<double2> buf;
  for (int which = 0; which < 2; which++) {
    const double *src = which == 0 ? u0 : v0;
    if (!src) continue;
    double2 *dst = which == 0 ? h->U0 : h->V0;
    if (h->path == LPS_PATH_DENSE) {
      // scatter on the host into the instance's cell range, then one copy
      const int c0 = h->node_begin[instance], c1 = c0 + h->dg.host_cells[instance];
      buf.assign(c1 - c0, make_double2(0, 0));
      const int *cell = h->dg.host_cell_of_node[instance].data();
      for (int i = 0; i < n; i++) buf[cell[i] - c0] = make_double2(src[2 * i], src[2 * i + 1]);
      LPS_CUDA_TRY(h, cudaMemcpyAsync(dst + c0, buf.data(), sizeof(double2) * buf.size(),
                                      cudaMemcpyHostToDevice, h->stream));
      LPS_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    } else {
      // the interleaved host layout is the device layout: one copy
      LPS_CUDA_TRY(h, cudaMemcpyAsync(dst + h->node_begin[instance], src, sizeof(double2) * n,
                                      cudaMemcpyHostToDevice, h->stream));
    }
  }
  return LPS_OK;
}

int lps_reset(lps_handle *h) {
  if (!h) return LPS_ERR_INVALID_ARG;
  return do_reset(h);
}

int lps_step(lps_handle *h, int n_steps, int diag_every) {
  if (!h || n_steps < 0) return LPS_ERR_INVALID_ARG;
  int remaining = n_steps;
  while (remaining > 0) {
    // records this chunk adds per instance must fit in the device log
    const int G = graph_period(h);
    const int chunk = (h->step % G == 0 && remaining >= G && h->opt.use_graphs) ? G : 1;
    int new_rec = 0, mask = 0;
    for (int r = 0; r < chunk; r++) {
      const int64_t s = h->step + 1 + r;
      if (diag_every > 0 && s % diag_every == 0) {
        mask |= 1 << r;
        new_rec++;
      } else if (remaining - r == 1) {
        mask |= 1 << (kFullBit + r);  // the call's last step leaves every field current
      }
    }
    if (h->pending_records + new_rec > h->log_capacity) {
      int st = drain_log(h);
      if (st) return st;
    }
    if (chunk > 1) {
      cudaGraphExec_t ex;
      int st = get_graph(h, mask, &ex);
      if (st) return st;
      LPS_CUDA_TRY(h, cudaGraphLaunch(ex, h->stream));
      h->launches += h->graph_kernels[mask];
    } else {
      h->launches += enqueue_step(h, h->step, mask & 1, (mask >> kFullBit) & 1);
      LPS_CUDA_TRY(h, cudaGetLastError());
    }
    h->step += chunk;
    h->pending_records += new_rec;
    remaining -= chunk;
  }
  return LPS_OK;
}

int lps_read_diag(lps_handle *h, int instance, lps_diag *out, int max_records, int *n_records) {
  if (!h || instance < 0 || instance >= h->n_inst || (max_records > 0 && !out)) return LPS_ERR_INVALID_ARG;
  int st = drain_log(h);
  if (st) return st;
  LPS_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  if ((st = check_device_error(h))) return st;
  std::vector<DiagRecord> &v = h->drained[instance];
  const int n = std::min((int)v.size(), std::max(max_records, 0));
  int status = LPS_OK;
  for (int r = 0; r < n; r++) {
    const DiagRecord &d = v[r];
    lps_diag &o = out[r];
    o.t = d.t; o.E = d.E; o.Ek = d.Ek; o.Ep = d.Ep; o.Px = d.Px; o.Py = d.Py;
    o.max_u = d.max_u; o.max_v = d.max_v; o.max_a = d.max_a;
    o.theta_min = d.th_min; o.theta_max = d.th_max;
    o.uB_rms = d.nact > 0 ? std::sqrt(d.uB_sq / d.nact) : 0.0;   // src/main.cpp:1061-1062
    o.vB_rms = d.nact > 0 ? std::sqrt(d.vB_sq / d.nact) : 0.0;
    if (h->E0[instance] < 0.0) h->E0[instance] = d.E;                // :1046
    const double E0 = h->E0[instance];
    o.dE_rel = (E0 > 0.0) ? (d.E - E0) / E0 : 0.0;                  // :1047
    o.step = d.step; o.max_u_node = d.iu; o.max_v_node = d.iv; o.n_active_abc = d.nact;
    if (h->path == LPS_PATH_DENSE) {
      o.max_u_node = d.iu >= 0 ? h->dg.host_node_of_cell(instance, d.iu) : -1;
      o.max_v_node = d.iv >= 0 ? h->dg.host_node_of_cell(instance, d.iv) : -1;
    }
    if (std::isnan(d.E) || std::isinf(d.E) || std::isnan(d.max_u) || std::isinf(d.max_u)) {
      status = LPS_ERR_NONFINITE;  // :1126-1133
      h->err = "FATAL: Energy is NaN/Inf at step " + std::to_string(d.step) + "!";
    }
  }
  v.erase(v.begin(), v.begin() + n);
  if (n_records) *n_records = n;
  return status;
}

int lps_download(lps_handle *h, int instance, double *u, double *v, double *a, double *theta, double *m) {
  if (!h || instance < 0 || instance >= h->n_inst) return LPS_ERR_INVALID_ARG;
  const int64_t n = h->step;
  // the newest level: after step n the current level is n
  const int cur = (int)(n % h->ring_u), cur3 = (int)(n % 3), cura = (int)(n % 2);
  if (h->opt.abcs_step != -1 && h->lg.abc.n_abc > 0)
    launch_merge_abc(h->lg, h->U[cur], h->S, h->stream);
  LPS_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  if (int e = check_device_error(h)) return e;
  const int nn = h->node_count[instance];
  const int g0 = h->node_begin[instance];
  const int span = h->path == LPS_PATH_DENSE ? h->dg.host_cells[instance] : nn;
  std::vector<double2> b2(span);
  std::vector<double> b1(span);
  auto get2 = [&](const double2 *src, double *dst) -> int {
    if (!dst) return LPS_OK;
    LPS_CUDA_TRY(h, cudaMemcpy(b2.data(), src + g0, sizeof(double2) * span, cudaMemcpyDeviceToHost));
    for (int i = 0; i < nn; i++) {
      const int c = global_of(h, instance, i) - g0;
      dst[2 * i] = b2[c].x;
      dst[2 * i + 1] = b2[c].y;
    }
    return LPS_OK;
  };
  auto get1 = [&](const double *src, double *dst) -> int {
    if (!dst) return LPS_OK;
    LPS_CUDA_TRY(h, cudaMemcpy(b1.data(), src + g0, sizeof(double) * span, cudaMemcpyDeviceToHost));
    for (int i = 0; i < nn; i++) dst[i] = b1[global_of(h, instance, i) - g0];
    return LPS_OK;
  };
  int s;
  if ((s = get2(h->U[cur], u)) || (s = get2(h->V[cur3], v)) || (s = get2(h->A[cura], a)) ||
      (s = get1(h->TH[cur3], theta)))
    return s;
  if (m) {
    const InstanceSetup &su = h->setup[instance];
    std::copy(su.m.begin(), su.m.end(), m);
  }
  return LPS_OK;
}

int lps_synchronize(lps_handle *h) {
  if (!h) return LPS_ERR_INVALID_ARG;
  LPS_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  if (int e = check_device_error(h)) return e;
  return LPS_OK;
}

int lps_get_info(lps_handle *h, int instance, lps_info *info) {
  if (!h || !info || instance < 0 || instance >= h->n_inst) return LPS_ERR_INVALID_ARG;
  memset(info, 0, sizeof *info);
  const InstanceSetup &s = h->setup[instance];
  info->n_instances = h->n_inst;
  info->path = h->path;
  info->precision = h->opt.precision;
  info->max_horizon_len = s.max_len;
  int64_t tn = 0, ta = 0;
  for (int k = 0; k < h->n_inst; k++) {
    tn += h->node_count[k];
    ta += h->abc_count[k];
  }
  info->total_nodes = tn;
  info->total_abc = ta;
  info->m_ref = s.m_ref;
  info->m_min = s.m_min;
  info->lambda = s.lam;
  info->mu = s.mu;
  info->kappa = s.kappa;
  info->alpha = s.alpha;
  info->lambda_pd = s.lambda_pd;
  info->output_exclude_r = s.out_r;
  info->domain_radius = s.domain_radius;
  info->dt_lps = s.dt_lps;
  info->device_bytes = h->device_bytes;
  info->step = h->step;
  info->n_abc_m_corrected = s.n_corrected;
  if (h->path == LPS_PATH_DENSE && !h->dg.groups.empty()) {
    int dev = 0, n_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    const DenseGroup &g0 = h->dg.groups[0];
    info->tile_ctas_theta = (g0.grid_theta + n_sm - 1) / n_sm;
    info->tile_ctas_force = (g0.grid_force + n_sm - 1) / n_sm;
    info->tile_rows_theta = g0.theta_rows;
    info->tile_rows_force = g0.force_rows;
  }
  info->horizon_ms = s.horizon_ms;
  info->horizon_on_gpu = s.horizon_on_gpu;
  return LPS_OK;
}

int64_t lps_kernel_launches(const lps_handle *h) { return h ? h->launches : 0; }

int lps_profile_kernels(lps_handle *h, int n_steps, int diag_every, lps_kernel_time *out, int max_kinds,
                        int *n_kinds) {
  if (!h || n_steps < 0 || (max_kinds > 0 && !out)) return LPS_ERR_INVALID_ARG;
  std::vector<std::pair<std::string, cudaEvent_t>> ev;
  cudaEvent_t start;
  LPS_CUDA_TRY(h, cudaEventCreate(&start));
  LPS_CUDA_TRY(h, cudaEventRecord(start, h->stream));
  Mark mark = [&](const char *name) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    cudaEventRecord(e, h->stream);
    ev.emplace_back(name, e);
  };
  for (int r = 0; r < n_steps; r++) {
    const int64_t s = h->step + 1;
    const bool diag = diag_every > 0 && s % diag_every == 0;
    if (diag && h->pending_records + 1 > h->log_capacity) {
      int st = drain_log(h);
      if (st) return st;
    }
    h->launches += enqueue_step(h, h->step, diag, r == n_steps - 1, &mark);
    h->step += 1;
    h->pending_records += diag ? 1 : 0;
  }
  LPS_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  std::vector<std::string> names;
  std::vector<double> ms;
  std::vector<int> cnt;
  cudaEvent_t prev = start;
  for (auto &e : ev) {
    float t = 0.f;
    cudaEventElapsedTime(&t, prev, e.second);
    prev = e.second;
    auto it = std::find(names.begin(), names.end(), e.first);
    if (it == names.end()) {
      names.push_back(e.first);
      ms.push_back(t);
      cnt.push_back(1);
    } else {
      ms[it - names.begin()] += t;
      cnt[it - names.begin()] += 1;
    }
  }
  for (auto &e : ev) cudaEventDestroy(e.second);
  cudaEventDestroy(start);
  const int nk = std::min((int)names.size(), max_kinds);
  for (int i = 0; i < nk; i++) {
    memset(&out[i], 0, sizeof(lps_kernel_time));
    strncpy(out[i].name, names[i].c_str(), sizeof(out[i].name) - 1);
    out[i].launches = cnt[i];
    out[i].total_ms = ms[i];
  }
  if (n_kinds) *n_kinds = nk;
  return LPS_OK;
}

void lps_destroy(lps_handle *h) {
  if (!h) return;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  destroy_all(h);
  delete h;
}

}  // extern "C"
