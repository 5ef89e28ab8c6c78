// pd2_lps_abc_b200.cpp -- command-line drop-in for the reference solver
// (src/main.cpp), running the time loop on the GPU through the C ABI.
//
//   PD2_LPS_ABC_B200 <prefix> <jobname> [options]
//
// Reads the preprocessor's file set <jobname>.* unchanged (src/main.cpp:
// 176-293), runs StepNo velocity-Verlet steps, and writes what the reference
// writes, in its formats: <jobname><prefix>-0.vtk at start, then every
// SUBSTEP_NO steps the displacement / velocity / dilatation VTK files and one
// line each of <jobname><prefix>.energy and .verify (:686-707, :1090-1123).
// Exit status 1 on the reference's FATAL conditions (unreadable input,
// failed consistency checks, NaN/Inf energy or displacement, :1126-1133).
//
// The reference's compile-time switches (:32-38) are options here:
//   --substep N        SUBSTEP_NO, output every N steps (default 30)
//   --abcs-step S      ABCS_STEP: 2 (default), 1 or -1 (ABCs off)
//   --theta-method M   THETA_ABC_METHOD: 1 (default, G_theta) or 0 (IDW)
//   --kinematic        KINEMATIC_VELOCITY_ABC = 1
//   --max-horizon H    MAX_HORIZON_LENGTH (default 128)
// and the device-side choices:
//   --precision fp64|fp32_mixed   (default fp64)
//   --path auto|dense|csr         (default auto)
//   --device D                    CUDA device ordinal
//   --autotune                    time the dense tile kernels' rows per thread
//                                 and CTAs per SM at setup
//   --theta-rows 2|4              fix the rows per dilatation thread
//   --force-rows 2|4              fix the rows per FP32-mixed force thread
//   --no-vtk                      skip the VTK files (energy/verify only)
//   --sync-output                 write each output step's files before the
//                                 next steps are enqueued (the reference's order)
//   --output-threads T            threads that format VTK text (default: all)
// Input files are read strictly: a file with fewer values than .data1
// announces is an error (the reference reads short files silently,
// src/helpers/utils.h:25-80).
//
// Output path.  At the stock cadence the reference spends as long writing
// three ASCII VTK files per output step as it does computing (it formats them
// serially with iostreams while the solver waits, src/main.cpp:1095-1103).
// Here a writer thread takes each output step's state (downloaded once) from
// a queue of at most two snapshots and writes the files while the GPU runs
// the next steps; the text is the same (12 significant digits, %.12g, as the
// reference's precision(12) stream), formatted in parallel with std::to_chars,
// and the node list and vertex section that every VTK file repeats is
// formatted once.
#include <algorithm>
#include <charconv>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "lps_cuda.h"

namespace {

bool read_numbers(const std::string &path, size_t count, std::vector<double> &out) {
  std::ifstream f(path);
  if (!f) return false;
  out.resize(count);
  for (size_t i = 0; i < count; i++)
    if (!(f >> out[i])) return false;
  return true;
}

// Integer files are written as numbers and rounded on reading
// (src/helpers/utils.h:61,76); -1 (cloud padding) stays -1 here, which the
// kernels skip -- the reference's cast maps it to node 0, whose padded
// coefficients are zero in the preprocessor's output.
bool read_ints(const std::string &path, size_t count, std::vector<int32_t> &out) {
  std::vector<double> d;
  if (!read_numbers(path, count, d)) return false;
  out.resize(count);
  for (size_t i = 0; i < count; i++) out[i] = (int32_t)std::floor(d[i] + 0.5);
  return true;
}

size_t count_numbers(const std::string &path) {
  std::ifstream f(path);
  size_t n = 0;
  double x;
  while (f >> x) n++;
  return n;
}

// ---- fast VTK text ---------------------------------------------------------
// %.12g of v, appended to out (std::to_chars' general format with a precision
// prints as printf does).
inline void put_g12(std::string &out, double v) {
  char buf[40];
  const auto r = std::to_chars(buf, buf + sizeof buf, v, std::chars_format::general, 12);
  out.append(buf, r.ptr);
}

// Formats fmt(i, out) for i in [0, n) on `threads` threads in contiguous
// ranges and returns the pieces in order.
template <class F>
std::vector<std::string> format_parallel(size_t n, int threads, F fmt) {
  const int T = std::max(1, std::min<int>(threads, (int)(n / 4096) + 1));
  std::vector<std::string> parts(T);
  std::vector<std::thread> pool;
  for (int t = 0; t < T; t++)
    pool.emplace_back([&, t] {
      const size_t a = n * t / T, b = n * (t + 1) / T;
      std::string &o = parts[t];
      o.reserve((b - a) * 48);
      for (size_t i = a; i < b; i++) fmt(i, o);
    });
  for (auto &th : pool) th.join();
  return parts;
}

// The three VTK files of an output step, written from a queue by one thread.
class VtkWriter {
 public:
  VtkWriter(const std::vector<double> &xy, const std::vector<int> &keep, int threads)
      : keep_(keep), threads_(threads) {
    // header, points and vertices: the same in every file (utils.h:95-120)
    std::string h = "# vtk DataFile Version 3.0\nPD2_LPS_ABC output\nASCII\nDATASET POLYDATA\nPOINTS " +
                    std::to_string(keep.size()) + " double\n";
    for (auto &p : format_parallel(keep.size(), threads, [&](size_t i, std::string &o) {
           put_g12(o, xy[2 * keep[i]]);
           o += ' ';
           put_g12(o, xy[2 * keep[i] + 1]);
           o += " 0.0\n";
         }))
      h += p;
    h += "VERTICES " + std::to_string(keep.size()) + " " + std::to_string(2 * keep.size()) + "\n";
    for (auto &p : format_parallel(keep.size(), threads, [&](size_t i, std::string &o) {
           o += "1 ";
           o += std::to_string(i);
           o += '\n';
         }))
      h += p;
    h += "POINT_DATA " + std::to_string(keep.size()) + "\n";
    head_ = std::move(h);
  }

  bool vector_file(const std::string &path, const std::vector<double> &v, const char *name) const {
    const std::string sec1 = std::string("VECTORS ") + name + " double\n";
    const std::string sec2 = std::string("SCALARS ") + name + "_magnitude double 1\nLOOKUP_TABLE default\n";
    auto a = format_parallel(keep_.size(), threads_, [&](size_t i, std::string &o) {
      put_g12(o, v[2 * keep_[i]]);
      o += ' ';
      put_g12(o, v[2 * keep_[i] + 1]);
      o += " 0.0\n";
    });
    auto b = format_parallel(keep_.size(), threads_, [&](size_t i, std::string &o) {
      const double x = v[2 * keep_[i]], y = v[2 * keep_[i] + 1];
      put_g12(o, std::sqrt(x * x + y * y));
      o += '\n';
    });
    return write_parts(path, sec1, a, sec2, b);
  }

  bool scalar_file(const std::string &path, const std::vector<double> &v, const char *name) const {
    const std::string sec1 = std::string("SCALARS ") + name + " double 1\nLOOKUP_TABLE default\n";
    auto a = format_parallel(keep_.size(), threads_, [&](size_t i, std::string &o) {
      put_g12(o, v[keep_[i]]);
      o += '\n';
    });
    return write_parts(path, sec1, a, "", {});
  }

 private:
  bool write_parts(const std::string &path, const std::string &s1, const std::vector<std::string> &a,
                   const std::string &s2, const std::vector<std::string> &b) const {
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    bool ok = std::fwrite(head_.data(), 1, head_.size(), f) == head_.size();
    ok = ok && std::fwrite(s1.data(), 1, s1.size(), f) == s1.size();
    for (const auto &p : a) ok = ok && std::fwrite(p.data(), 1, p.size(), f) == p.size();
    ok = ok && std::fwrite(s2.data(), 1, s2.size(), f) == s2.size();
    for (const auto &p : b) ok = ok && std::fwrite(p.data(), 1, p.size(), f) == p.size();
    return std::fclose(f) == 0 && ok;
  }

  const std::vector<int> &keep_;
  int threads_;
  std::string head_;
};

// One output step's state on its way to the files.
struct Snapshot {
  std::string step;
  std::vector<double> u, v, th;
};

// Writes queued snapshots in order on a thread of its own; push() blocks while
// two snapshots are waiting, so at most three states are held on the host.
class OutputQueue {
 public:
  OutputQueue(const VtkWriter &w, std::string base) : w_(w), base_(std::move(base)), th_([this] { run(); }) {}
  ~OutputQueue() { finish(); }

  void push(Snapshot &&s) {
    std::unique_lock<std::mutex> l(mu_);
    cv_.wait(l, [&] { return q_.size() < 2; });
    q_.push_back(std::move(s));
    cv_.notify_all();
  }
  // Waits until every queued snapshot is written; false if a write failed.
  bool finish() {
    {
      std::lock_guard<std::mutex> l(mu_);
      done_ = true;
      cv_.notify_all();
    }
    if (th_.joinable()) th_.join();
    return ok_;
  }
  std::string error() const { return err_; }

 private:
  void run() {
    for (;;) {
      Snapshot s;
      {
        std::unique_lock<std::mutex> l(mu_);
        cv_.wait(l, [&] { return done_ || !q_.empty(); });
        if (q_.empty()) return;
        s = std::move(q_.front());
        q_.pop_front();
        cv_.notify_all();
      }
      if (!ok_) continue;
      if (!w_.vector_file(base_ + "-" + s.step + ".vtk", s.u, "displacement") ||
          !w_.vector_file(base_ + "-vel-" + s.step + ".vtk", s.v, "velocity") ||
          !w_.scalar_file(base_ + "-theta-" + s.step + ".vtk", s.th, "dilatation")) {
        ok_ = false;
        err_ = "cannot write the VTK files of step " + s.step;
      }
    }
  }

  const VtkWriter &w_;
  std::string base_;
  std::mutex mu_;
  std::condition_variable cv_;
  std::deque<Snapshot> q_;
  bool done_ = false;
  bool ok_ = true;
  std::string err_;
  std::thread th_;
};

int fatal(const std::string &msg) {
  std::cerr << msg << std::endl;
  return 1;
}

}  // namespace

int main(int argc, char **argv) {
  std::cout << "PD2_LPS_ABC (B200 time loop): LPS state-based PD with ABCs" << std::endl << std::endl;
  if (argc < 3) {
    std::cout << "Usage: " << argv[0] << " <prefix> <jobname> [options]" << std::endl;
    return 0;
  }
  const std::string prefix = argv[1], job = argv[2];
  lps_options opt;
  lps_default_options(&opt);
  int substep = 30;
  bool write_vtk = true, sync_output = false;
  int out_threads = (int)std::max(1u, std::thread::hardware_concurrency());
  for (int a = 3; a < argc; a++) {
    const std::string k = argv[a];
    auto next = [&](const char *what) -> const char * {
      if (a + 1 >= argc) {
        std::cerr << "missing value for " << what << std::endl;
        std::exit(2);
      }
      return argv[++a];
    };
    if (k == "--substep") substep = std::atoi(next("--substep"));
    else if (k == "--abcs-step") opt.abcs_step = std::atoi(next("--abcs-step"));
    else if (k == "--theta-method") opt.theta_method = std::atoi(next("--theta-method"));
    else if (k == "--kinematic") opt.kinematic_v = 1;
    else if (k == "--max-horizon") opt.max_horizon = std::atoi(next("--max-horizon"));
    else if (k == "--device") opt.device = std::atoi(next("--device"));
    else if (k == "--no-vtk") write_vtk = false;
    else if (k == "--sync-output") sync_output = true;
    else if (k == "--output-threads") out_threads = std::atoi(next("--output-threads"));
    else if (k == "--autotune") opt.autotune = 1;
    else if (k == "--theta-rows") opt.theta_rows = std::atoi(next("--theta-rows"));
    else if (k == "--force-rows") opt.force_rows = std::atoi(next("--force-rows"));
    else if (k == "--precision") {
      const std::string v = next("--precision");
      if (v == "fp64") opt.precision = LPS_FP64;
      else if (v == "fp32_mixed") opt.precision = LPS_FP32_MIXED;
      else return fatal("unknown precision " + v);
    } else if (k == "--path") {
      const std::string v = next("--path");
      if (v == "auto") opt.path = LPS_PATH_AUTO;
      else if (v == "dense") opt.path = LPS_PATH_DENSE;
      else if (v == "csr") opt.path = LPS_PATH_CSR;
      else return fatal("unknown path " + v);
    } else {
      return fatal("unknown option " + k);
    }
  }
  if (substep <= 0) return fatal("--substep must be positive");

  // ---- input file set (src/main.cpp:176-293) ----
  std::cout << "Reading data... " << std::flush;
  std::vector<double> d1, d2;
  if (!read_numbers(job + ".data1", 6, d1)) return fatal("FATAL: Cannot read " + job + ".data1");
  const size_t n_d2 = count_numbers(job + ".data2");
  if (n_d2 < 11 || !read_numbers(job + ".data2", n_d2 >= 15 ? 15 : 11, d2))
    return fatal("FATAL: Cannot read " + job + ".data2");
  const int N = (int)std::lround(d1[0]), n_steps = (int)std::lround(d1[1]), n_pre = (int)std::lround(d1[2]);
  const int n_abc = (int)std::lround(d1[4]), C = (int)std::lround(d1[5]);
  std::vector<double> nodes, icv, icd, bcv, pre, gu, gv, gth;
  std::vector<int32_t> bct, inf, clouds;
  if (!read_numbers(job + ".nodes", 2 * (size_t)N, nodes)) return fatal("FATAL: Cannot read " + job + ".nodes");
  if (!read_ints(job + ".bctypes", 2 * (size_t)N, bct)) return fatal("FATAL: Cannot read " + job + ".bctypes");
  if (!read_numbers(job + ".bcvalues", 2 * (size_t)N, bcv)) return fatal("FATAL: Cannot read " + job + ".bcvalues");
  if (!read_numbers(job + ".icdvalues", 2 * (size_t)N, icd)) return fatal("FATAL: Cannot read " + job + ".icdvalues");
  if (!read_numbers(job + ".icvalues", 2 * (size_t)N, icv)) return fatal("FATAL: Cannot read " + job + ".icvalues");
  if (n_pre > 0 && !read_numbers(job + ".prenotch", 4 * (size_t)n_pre, pre))
    return fatal("FATAL: Cannot read " + job + ".prenotch");
  const bool abc_files = opt.abcs_step != -1 && n_abc > 0;
  if (abc_files) {
    const size_t cols = (opt.abcs_step == 1 ? 2 : 4) * (size_t)C;
    if (!read_numbers(job + ".ciNodesU", 2 * (size_t)n_abc * cols, gu))
      return fatal("FATAL: Cannot read " + job + ".ciNodesU");
    if (!read_numbers(job + ".ciNodesV", 2 * (size_t)n_abc * cols, gv))
      return fatal("FATAL: Cannot read " + job + ".ciNodesV");
    if (!read_ints(job + ".iClouds", (size_t)n_abc * C, clouds))
      return fatal("FATAL: Cannot read " + job + ".iClouds");
    if (!read_ints(job + ".infNodesIndex", (size_t)n_abc, inf))
      return fatal("FATAL: Cannot read " + job + ".infNodesIndex");
    if (opt.theta_method == 1 &&
        !read_numbers(job + ".ciNodesTheta", (size_t)n_abc * opt.abcs_step * C, gth))
      return fatal("FATAL: Cannot read " + job + ".ciNodesTheta");
  }
  std::cout << "finished." << std::endl;

  lps_problem p;
  std::memset(&p, 0, sizeof p);
  p.n_nodes = N;
  p.n_abc = abc_files ? n_abc : 0;
  p.max_cloud = C;
  p.n_prenotch = n_pre;
  p.E = d2[0]; p.nu = d2[1]; p.rho = d2[2]; p.dt = d2[6]; p.delta = d2[7]; p.dx = d2[8]; p.dy = d2[9];
  p.nodes = nodes.data(); p.bctypes = bct.data(); p.u0 = icv.data(); p.v0 = icd.data();
  p.prenotch = n_pre > 0 ? pre.data() : nullptr;
  if (abc_files) {
    p.inf_nodes = inf.data(); p.clouds = clouds.data(); p.gu = gu.data(); p.gv = gv.data();
    p.gtheta = gth.empty() ? nullptr : gth.data();
  }

  std::cout << std::setprecision(10) << std::endl << "=== Discretization ===" << std::endl
            << "  NodeNo = " << N << std::endl << "  StepNo = " << n_steps << std::endl
            << "  delta (R) = " << p.delta << std::endl << "  dx = " << p.dx << ", dy = " << p.dy << std::endl
            << "  dt = " << p.dt << std::endl << "  ABC nodes = " << n_abc << std::endl
            << "  maxCloudSize = " << C << std::endl;

  lps_handle *h = nullptr;
  int st = lps_create(&p, 1, &opt, &h);
  if (st != LPS_OK) return fatal(lps_last_error(nullptr));
  lps_info info;
  lps_get_info(h, 0, &info);
  std::cout << "  m_ref = " << info.m_ref << ", alpha = " << info.alpha << ", lambda_PD = " << info.lambda_pd
            << std::endl << "  kernel path: " << (info.path == LPS_PATH_DENSE ? "dense" : "csr")
            << ", precision: " << (info.precision == LPS_FP32_MIXED ? "fp32_mixed" : "fp64") << std::endl;

  // nodes written to the VTK files (src/main.cpp:528-530 exclusion radius)
  const double rex = info.output_exclude_r;
  std::vector<int> keep;
  for (int i = 0; i < N; i++) {
    const double r = std::sqrt(nodes[2 * i] * nodes[2 * i] + nodes[2 * i + 1] * nodes[2 * i + 1]);
    if (rex > 0.0 && r > rex) continue;
    keep.push_back(i);
  }
  const std::string base = job + prefix;
  if (out_threads <= 0) out_threads = 1;
  VtkWriter writer(nodes, keep, out_threads);
  if (write_vtk && !writer.vector_file(base + "-0.vtk", icv, "displacement"))
    return fatal("cannot write " + base + "-0.vtk");
  {
    std::ofstream e(base + ".energy", std::ios::out | std::ios::trunc);
    e << "# t  E_total  E_kinetic  E_potential  P_x  P_y  max_u  max_theta" << std::endl;
    std::ofstream v(base + ".verify", std::ios::out | std::ios::trunc);
    v << "# t  E_total  dE/E0  P_x  P_y  max_theta  max_u  max_v  max_a" << std::endl;
    if (!e || !v) return fatal("cannot write the energy / verify logs");
  }

  std::cout << std::endl << "Time marching started (" << n_steps << " steps):" << std::endl;
  const auto t0 = std::chrono::steady_clock::now();
  OutputQueue queue(writer, base);
  int status = 0;
  int done = 0;
  while (done < n_steps && status == 0) {
    // one output record per chunk; without VTK files the whole run is one chunk
    const int chunk = write_vtk ? std::min(substep - done % substep, n_steps - done) : n_steps - done;
    if ((st = lps_step(h, chunk, substep)) != LPS_OK) return fatal(lps_last_error(h));
    done += chunk;
    std::vector<lps_diag> recs(chunk / substep + 1);
    int n_rec = 0;
    const int rs = lps_read_diag(h, 0, recs.data(), (int)recs.size(), &n_rec);
    if (rs != LPS_OK && rs != LPS_ERR_NONFINITE) return fatal(lps_last_error(h));
    if (n_rec > 0 && write_vtk) {
      // the reference writes VTK before it checks the energy; a non-finite
      // step ends the run below, after its log lines, as :1126-1133 do
      Snapshot snap;
      snap.step = std::to_string(done);
      snap.u.resize(2 * (size_t)N);
      snap.v.resize(2 * (size_t)N);
      snap.th.resize(N);
      if ((st = lps_download(h, 0, snap.u.data(), snap.v.data(), nullptr, snap.th.data(), nullptr)) != LPS_OK)
        return fatal(lps_last_error(h));
      if (sync_output) {
        if (!writer.vector_file(base + "-" + snap.step + ".vtk", snap.u, "displacement") ||
            !writer.vector_file(base + "-vel-" + snap.step + ".vtk", snap.v, "velocity") ||
            !writer.scalar_file(base + "-theta-" + snap.step + ".vtk", snap.th, "dilatation"))
          return fatal("cannot write the VTK files of step " + snap.step);
      } else {
        queue.push(std::move(snap));
      }
    }
    std::ofstream e(base + ".energy", std::ios::out | std::ios::app);
    std::ofstream v(base + ".verify", std::ios::out | std::ios::app);
    for (int r = 0; r < n_rec; r++) {
      const lps_diag &d = recs[r];
      std::cout << d.step / substep << "\tt=" << std::setprecision(6) << d.t << "\tE=" << std::setprecision(8)
                << d.E << "\tK=" << d.Ek << "\tP=" << d.Ep << "\tdE/E0=" << std::setprecision(4) << d.dE_rel
                << "\t|p|=" << std::sqrt(d.Px * d.Px + d.Py * d.Py) << "\tuB=" << d.uB_rms
                << "\tvB=" << d.vB_rms << std::setprecision(10) << std::endl;
      e << std::setprecision(16) << d.t << " " << d.E << " " << d.Ek << " " << d.Ep << " " << d.Px << " " << d.Py
        << " " << d.max_u << " " << d.theta_max << " " << d.uB_rms << " " << d.vB_rms << std::endl;
      v << std::setprecision(16) << d.t << " " << d.E << " " << d.dE_rel << " " << d.Px << " " << d.Py << " "
        << d.theta_max << " " << d.max_u << " " << d.max_v << " " << d.max_a << std::endl;
      if (std::isnan(d.E) || std::isinf(d.E)) {
        std::cerr << "FATAL: Energy is NaN/Inf at step " << d.step << "!" << std::endl;
        status = 1;
        break;
      }
      if (std::isnan(d.max_u) || std::isinf(d.max_u)) {
        std::cerr << "FATAL: Displacement is NaN/Inf at step " << d.step << "!" << std::endl;
        status = 1;
        break;
      }
      if (opt.abcs_step == -1 && d.dE_rel != 0.0 && std::abs(d.dE_rel) > 0.01)
        std::cerr << "WARNING: Energy drift > 1% at step " << d.step << " (dE/E0=" << d.dE_rel
                  << "). Check dt stability." << std::endl;
    }
  }
  if (!queue.finish()) return fatal(queue.error());
  const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  lps_destroy(h);
  if (status) return status;
  std::cout << std::endl << "Time marching took " << sec << " seconds." << std::endl;
  return 0;
}
