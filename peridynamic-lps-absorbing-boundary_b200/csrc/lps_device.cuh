// lps_device.cuh -- data layout shared by the host setup and the sm_100a kernels.
//
// One handle holds a *batch* of independent instances packed into shared
// device arrays.  Two node layouts exist:
//
//  * CSR/ELL path: instance k owns the global node range
//    [node_begin_k, node_begin_k + n_k); node_begin_k is a multiple of
//    kNodeBlock so every thread block of a node kernel belongs to exactly one
//    instance.  Neighbours live in an ELL table nbr[slot * n_total + i]
//    (column-major, so a warp's loads of one slot are coalesced), sorted by
//    distance like the reference's horizons (kd_tree_interface.h:107).
//
//  * Dense path: instance k owns a padded 2-D cell grid; node index == cell
//    index (empty cells carry type 0).  See lps_dense.cuh.
//
// State is FP64 double2 per node (x, y), in rings so that no step copies
// data: v keeps three time levels (n-1, n, n+1: the ABC operators read two
// history levels, src/main.cpp:903-912), u three (CSR) or four (dense: the
// force pass already writes the next step's predicted level), a two, theta
// three (the G_theta history, :1157-1163).  The FP32-mixed form adds an FP32
// copy of the predicted displacement (two levels).
#pragma once
#include <cstdint>

namespace lps {

constexpr int kNodeBlock = 256;      // threads per node-kernel block
constexpr int kAbcWarpsPerBlock = 8; // warps per ABC block (one ABC node each)

// node type bits
constexpr uint8_t kExists = 1;       // a real node (not padding)
constexpr uint8_t kBcAbc = 2;        // BCTypes[2i] == 1 (IDW skips these, :778)
constexpr uint8_t kActiveAbc = 4;    // overwritten by the G operators this step
constexpr uint8_t kKeepState = 8;    // read every step by the absorbing-boundary kernels (a cloud entry of
                                     // a writing ABC node, or an IDW neighbour): its v and theta are
                                     // written on every step, not only on full steps (StepPtrs::full)

// Per-instance constants, one device table per handle (Geo::ip, Abc::ip),
// indexed by instance id.
struct InstParams {
  double dt, half_dt, rho, lam, mu, kappa;
  double c_lm;      // 2 (lambda - mu)      (src/main.cpp:857)
  double c_mu8;     // 8 mu                 (:858)
  double c_mu4;     // 4 mu                 (:1037)
  double dx, dy, delta;
  double beta_lo;   // delta - dx/2         (:101)
  double beta_hi;   // delta + dx/2         (:103)
  double out_r;     // energy exclusion radius, <= 0: none (:528-530)
  double f32_b0;    // FP32-mixed form: force scale alpha = 8 mu / m_ref (:485)
  double f32_ab;    // FP32-mixed form: lambda_PD / alpha = (lambda - mu) / (4 mu)
  double mref;      // m_ref = max m_i (:429-442): m_i of every full-horizon node
  int node_begin, node_count;   // global node (or cell) range
  int abc_begin, abc_count;     // packed ABC list range
  int n_active_abc;             // entries with BCTypes == 1 (uB/vB denominators)
  int kinematic;                // KINEMATIC_VELOCITY_ABC
  int theta_method;             // THETA_ABC_METHOD
  int abcs_step;                // ABCS_STEP
  int dense;                    // 1 = dense grid layout
  int pitch, nrow, ncol;        // dense grid geometry (pitch in cells)
  int stencil;                  // dense: stencil-class id
  int tile_begin, tile_count;   // dense: the instance's tiles in the tile list
};

// Buffer pointers of one time step, resolved on the host from the ring phase.
struct StepPtrs {
  double2 *u_n;            // u^n
  const double2 *u_nm1;    // u^{n-1}
  double2 *u_np1;          // predicted u^{n+1} (ABC nodes: see s_abc)
  const double2 *v_n, *v_nm1;
  double2 *v_np1;
  const double2 *a_n;
  double2 *a_np1;
  double2 *vh;             // v^n + dt/2 a^n (first half of the corrector)
  const double *th_n, *th_nm1;
  double *th_np1;
  double2 *s_abc;          // G_u result u^{n+1} at ABC nodes (merged into the ring
                           // by the dense step's end, by the CSR predictor)
  double2 *u_np2;          // dense path: predicted u^{n+2}, written by the force pass
  float2 *u32_np1;         // FP32-mixed form: FP32 copy of the predicted u^{n+1}
  float2 *u32_np2;         // FP32-mixed form: FP32 copy of u^{n+2}, written by the force pass
  int th_ring;             // ring index of th_np1
  int full;                // dense path: 1 = write v, a and theta at every node; 0 = only where a
                           // later step reads them (kKeepState and ABC nodes).  Diagnostic steps
                           // and the last step of every lps_step call are full, so whatever the
                           // diagnostics or lps_download read is current.
};

// Geometry + static per-node data.
struct Geo {
  const InstParams *ip;        // per-instance constants
  int n_total;                 // padded node count
  int ell_width;               // ELL slots
  const double2 *xy;           // coordinates
  const uint8_t *type;
  const int *abc_of;           // node -> ABC list index or -1
  const double *m;             // weighted volume after the ABC override
  const double2 *coef;         // (2(l-m)/m_i, 8mu/m_i); (0,-1) when m_i <= 0
  const int *len;              // ELL length (horizon minus self)
  const int *nbr;              // [ell_width][n_total]
  const int *blk_inst;         // node block -> instance id
};

// Packed absorbing-boundary data (all instances).
struct Abc {
  const InstParams *ip;        // per-instance constants (the same table as Geo::ip)
  int n_abc;
  const int *node;             // global node index
  const int *inst;             // instance id
  const uint8_t *writes;       // 1: this entry writes (active, last duplicate)
  const uint8_t *active;       // BCTypes[2 node] == 1
  const int *cl_off, *cl_len;  // compacted cloud list (k != -1 only)
  const int *cl_idx;           // global node index per cloud entry
  const double *gu;            // per entry 8 doubles: row x [4], row y [4]
  const double *gv;            // same
  const double *gth;           // per node: rows theta^n, theta^{n-1} of cl_len weights
  const int *idw_off, *idw_len;// IDW neighbour lists (THETA_ABC_METHOD 0)
  const int *idw_idx;
  const double *idw_w;
  // Dense path, sliced-ELL copy of the operators: the writing entries sorted
  // by cloud length and cut into slices of 32 (one entry per lane); slice s
  // holds for each cloud position e < len_s the 18 operator rows of its 32
  // entries ([e][row][lane], doubles) and their cloud indices ([e][lane]),
  // zero weights (and a valid index) past an entry's own length.
  int n_slices;
  const struct SellSlice *slices;
  const double *sell_g;
  const int *sell_idx;
  const int *sell_a;           // [slice][lane]: ABC entry, or -1
};

struct SellSlice {
  long long goff;              // first double of the slice in sell_g
  long long ioff;              // first int of the slice in sell_idx
  int len;                     // cloud positions in the slice
  int pad;
};

// Per-block partial sums of the diagnostics (src/main.cpp:986-1062).
struct DiagPartial {
  double E, Ek, Ep, Px, Py;
  double max_u, max_v, max_a, th_min, th_max;
  double uB_sq, vB_sq;
  int iu, iv, nact, pad;
};

// One raw record in the on-device log (host derives dE/E0 and the RMS).
struct DiagRecord {
  double t, E, Ek, Ep, Px, Py;
  double max_u, max_v, max_a, th_min, th_max, uB_sq, vB_sq;
  int step, iu, iv, nact;
};

}  // namespace lps
