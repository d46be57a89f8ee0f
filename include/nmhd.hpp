// nmhd.hpp - header-only C++ mirror of the reference's class MHDSolver
// (src/library/mhd_solver.hrb:150-276) over the C ABI in nmhd.h.
//
// Same member names and meaning as the reference:
//   read/write        -> bool (false on open failure or size mismatch)
//   proceed           -> bool (true when goal_time was reached; false on the
//                        wallclock limit), wallclock_time_limit <= 0 ignored
//   current_time      -> PreciseReal (double), generation -> int
//   save_state/load_state(prefix) -> prefix.bin + prefix_setup.txt, the
//                        reference's checkpoint files (see nmhd::checkpoint)
// Problem hooks are not virtual here: the initial state is passed in with
// initialize_state(fields) and the source term is chosen by nmhd_config.
#ifndef NMHD_HPP
#define NMHD_HPP

#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <functional>
#include <fstream>
#include <iomanip>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "nmhd.h"

namespace nmhd {

// The reference's checkpoint text, prefix_setup.txt: MHDSolver::save_state /
// load_state (src/library/mhd_solver.inlrb:1023-1050) write GlobalSetup, a line
// of "################", then LocalSetup, each as a member count followed by
// "name value" lines with the default stream format (pod text of
// src/nushio_script/persistent_pod.hrb:129-176).  load_state keeps only
// generation and current_time (6 significant digits, so the reference's own
// restarts are lossy).  Files written here add one GlobalSetup member,
// current_time_exact (17 digits), which the reference's reader skips and this
// reader prefers; a file written by either code loads in the other.
namespace checkpoint {

// Spacings, computational and local extents by the reference's float chains
// (simulation_config_default.h:56-103) and the shear velocity -q Omega L_y.
struct Derived {
  float d[3], extent[3], local[3];
  double rel_vel;
};

inline Derived derive(const nmhd_config &c) {
  Derived r;
  const int py = c.parallel_size_y > 1 ? c.parallel_size_y : 1;
  const int s[3] = {c.size_x, c.size_y, c.size_z};
  const int li[3] = {c.size_x, c.size_y - 2 * c.margin_y, c.size_z - 2 * c.margin_z};
  const int gi[3] = {li[0], py * li[1], li[2]};
  const float L[3] = {c.extent_x, c.extent_y, c.extent_z};
  for (int i = 0; i < 3; ++i) {
    volatile float per = L[i] / (float)gi[i];
    volatile float comp = per * (float)s[i];
    volatile float local = per * (float)li[i];
    volatile float d = comp / (float)s[i];
    r.extent[i] = comp;
    r.local[i] = local;
    r.d[i] = d;
  }
  volatile float qo = -c.q * c.omega;
  volatile float rv = qo * r.local[1];
  r.rel_vel = c.problem == NMHD_PROBLEM_SHEARING_BOX ? (double)rv : 0.0;
  return r;
}

// relative_displacement()'s normalized displacement (mhd_solver.inlrb:244-259),
// as the reference's float; the same for every radial rank.
inline float shear_displacement(const nmhd_config &c, double t) {
  if (c.problem != NMHD_PROBLEM_SHEARING_BOX) return 0.0f;
  const Derived d = derive(c);
  const double d0 = 0.0 + t * d.rel_vel;
  const int fold = (int)std::floor(d0 / (double)d.extent[0]);
  const double d1 = d0 - (double)((float)fold * d.extent[0]);
  return (float)d1;
}

// encode_member(std::string): bytes outside 33..126 and '%' as %xx.
inline std::string encode(const std::string &s) {
  std::string out;
  char buf[4];
  for (unsigned char ch : s) {
    if (ch >= 33 && ch <= 126 && ch != '%') {
      out += (char)ch;
    } else {
      std::snprintf(buf, sizeof buf, "%%%02x", ch);
      out += buf;
    }
  }
  return out;
}

// `rank`: the radial slab's rank when c.parallel_size_y > 1, else 0.
inline std::string setup_text(const nmhd_config &c, int generation, double time, const std::string &dir,
                              int rank = 0) {
  const Derived d = derive(c);
  const int py = c.parallel_size_y > 1 ? c.parallel_size_y : 1;
  const int li[3] = {c.size_x, c.size_y - 2 * c.margin_y, c.size_z - 2 * c.margin_z};
  const int gs[3] = {li[0], py * li[1], li[2]};
  const int ps[3] = {1, py, 1}, r3[3] = {0, rank, 0};
  const int sz[3] = {c.size_x, c.size_y, c.size_z};
  const int mg[3] = {0, c.margin_y, c.margin_z};
  const float L[3] = {c.extent_x, c.extent_y, c.extent_z};
  const char *ax[3] = {"x", "y", "z"}, *AX[3] = {"X", "Y", "Z"};
  std::ostringstream o;
  o << 21 << std::endl;
  o << "generation " << generation << std::endl;
  o << "real_size " << 4 << std::endl;
  o << "real_precision float" << std::endl;
  o << "current_time " << time << std::endl;
  o << "parallel_size " << py << std::endl;
  for (int k = 0; k < 3; ++k) {
    o << "global_size_" << ax[k] << " " << gs[k] << std::endl;
    o << "parallel_size_" << ax[k] << " " << ps[k] << std::endl;
    o << "global_extent_" << ax[k] << " " << L[k] << std::endl;
    o << "global_corner_" << ax[k] << " " << 0.0f << std::endl;
    o << "d" << AX[k] << " " << d.d[k] << std::endl;
  }
  o << "current_time_exact " << std::setprecision(17) << time << std::setprecision(6) << std::endl;
  o << std::endl << "################" << std::endl;
  o << 21 << std::endl;
  char prefix[16];
  std::snprintf(prefix, sizeof prefix, "%04d", rank);
  o << "mpi_rank " << rank << std::endl;
  o << "output_directory " << encode(dir) << std::endl;
  o << "mpi_prefix " << encode(prefix) << std::endl;
  o << "relative_displacement " << (double)shear_displacement(c, time) << std::endl;
  o << "relative_velocity " << d.rel_vel << std::endl;
  o << "computational_size " << (size_t)c.size_x * c.size_y * c.size_z << std::endl;
  for (int k = 0; k < 3; ++k) {
    // kGlobalCorner + (kLocalSize * rank - kMarginSize) * kD (LocalSetup, mhd_solver.h:311-317)
    volatile float corner = (float)(li[k] * r3[k] - mg[k]) * d.d[k];
    o << "computational_size_" << ax[k] << " " << sz[k] << std::endl;
    o << "margin_" << ax[k] << " " << mg[k] << std::endl;
    o << "computational_corner_" << ax[k] << " " << (float)corner << std::endl;
    o << "computational_extent_" << ax[k] << " " << d.extent[k] << std::endl;
    o << "d" << AX[k] << " " << d.d[k] << std::endl;
  }
  o << std::endl;
  return o.str();
}

// The clock load_state restores: generation and current_time (the exact
// member when present).  False when the pod cannot be read.
inline bool clock_from_setup(std::istream &is, int &generation, double &time) {
  int n;
  if (!(is >> n) || n < 0) return false;
  std::map<std::string, std::string> m;
  for (int i = 0; i < n; ++i) {
    std::string k, v;
    if (!(is >> k >> v)) return false;
    m[k] = v;
  }
  if (!m.count("generation") || !m.count("current_time")) return false;
  try {
    generation = std::stoi(m["generation"]);
    time = std::stod(m.count("current_time_exact") ? m["current_time_exact"] : m["current_time"]);
  } catch (const std::exception &) {
    return false;
  }
  return true;
}

}  // namespace checkpoint

class Error : public std::runtime_error {
 public:
  Error(nmhd_status code, const std::string &msg) : std::runtime_error(msg), code_(code) {}
  nmhd_status code() const { return code_; }

 private:
  nmhd_status code_;
};

class MHDSolver {
 public:
  explicit MHDSolver(const nmhd_config &cfg) : cfg_(cfg) {
    nmhd_status st = nmhd_create(&cfg_, &s_);
    if (st != NMHD_OK) throw Error(st, nmhd_last_error(nullptr));
  }
  ~MHDSolver() { nmhd_destroy(s_); }
  MHDSolver(const MHDSolver &) = delete;
  MHDSolver &operator=(const MHDSolver &) = delete;

  const nmhd_config &config() const { return cfg_; }
  size_t cells() const { return (size_t)cfg_.size_x * cfg_.size_y * cfg_.size_z; }

  // initialize_state(): the hook's result, as 8 host arrays in .bin order.
  void initialize_state(const float *const fields[8]) { check(nmhd_set_state(s_, fields, 0)); }
  void initialize_state(const std::vector<float> &all) {
    const float *f[8];
    for (int v = 0; v < 8; ++v) f[v] = all.data() + v * cells();
    initialize_state(f);
  }
  std::vector<float> state() {
    std::vector<float> all(8 * cells());
    float *f[8];
    for (int v = 0; v < 8; ++v) f[v] = all.data() + v * cells();
    check(nmhd_get_state(s_, f, 0));
    return all;
  }

  bool read(const std::string &path) { return nmhd_read(s_, path.c_str()) == NMHD_OK; }
  bool write(const std::string &path) { return nmhd_write(s_, path.c_str()) == NMHD_OK; }

  // proceed(goal_time, wallclock_time_limit): true when the goal time was
  // reached.  Without a monitor the steps run in device-resident batches;
  // with one, as in the reference's loop (mhd_solver.inlrb:857-860), the
  // monitor is called before every step and a non-zero return stops the run
  // before that step (proceed then returns false).
  bool proceed(float goal_time, double wallclock_time_limit = -1, long long max_steps = 0) {
    if (!monitor_) {
      int64_t done = 0;
      nmhd_status st = nmhd_proceed(s_, goal_time, wallclock_time_limit, max_steps, &done);
      last_steps_ = done;
      if (st < 0) throw Error(st, nmhd_last_error(s_));
      return st == NMHD_GOAL_REACHED;
    }
    const auto t0 = std::chrono::steady_clock::now();
    last_steps_ = 0;
    for (;;) {
      if (max_steps > 0 && last_steps_ >= max_steps) return false;
      if (monitor_(*this)) return false;
      double left = -1;
      if (wallclock_time_limit > 0) {
        left = wallclock_time_limit - std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (left <= 0) return false;
      }
      int64_t done = 0;
      nmhd_status st = nmhd_proceed(s_, goal_time, left, 1, &done);
      last_steps_ += done;
      if (st < 0) throw Error(st, nmhd_last_error(s_));
      if (st == NMHD_GOAL_REACHED) return true;
      if (st == NMHD_TIMEOUT) return false;
    }
  }
  // Builds the CUDA graphs a later proceed(..., max_steps) launches, without
  // running them (nmhd_prepare).
  void prepare(long long max_steps = 0) { check(nmhd_prepare(s_, max_steps)); }
  // Kernel selection (nmhd_set_kernel / nmhd_get_kernel; every variant gives
  // bitwise the same results) and the autotuner, which times every variant on
  // this box from the current state and keeps the fastest (nmhd_autotune):
  // returns its rows (variant, tile_rows, z_chunk, ms per step).
  void set_kernel(int variant, int tile_rows = 8, int z_chunk = 0) {
    check(nmhd_set_kernel(s_, variant, tile_rows, z_chunk));
  }
  int kernel_variant() const {
    int v = 0;
    nmhd_get_kernel(s_, &v, nullptr, nullptr);
    return v;
  }
  std::vector<std::array<double, 4>> autotune(int steps = 5) {
    std::vector<double> rows(4 * 64);
    const int k = nmhd_autotune(s_, steps, rows.data(), 64);
    if (k < 0) throw Error((nmhd_status)k, nmhd_last_error(s_));
    std::vector<std::array<double, 4>> out(k);
    for (int i = 0; i < k; ++i) out[i] = {rows[4 * i], rows[4 * i + 1], rows[4 * i + 2], rows[4 * i + 3]};
    return out;
  }
  // The application's monitor() (e.g. src/application/kepler_disk_demo/
  // mhd_solver.curb:107-130); an empty function removes it.
  void set_monitor(std::function<int(MHDSolver &)> m) { monitor_ = std::move(m); }

  double current_time() const { return nmhd_current_time(s_); }
  int generation() const { return (int)nmhd_generation(s_); }
  long long last_steps() const { return last_steps_; }

  // save_state/load_state (mhd_solver.inlrb:1023-1050): the .bin dump plus
  // the reference's setup text (nmhd::checkpoint); `rank` of a radial slab.
  bool save_state(const std::string &prefix, int rank = 0) {
    if (!write(prefix + ".bin")) return false;
    std::ofstream ofs((prefix + "_setup.txt").c_str());
    if (!ofs) return false;
    const std::string::size_type slash = prefix.rfind('/');
    const std::string dir = slash == std::string::npos ? "." : prefix.substr(0, slash);
    ofs << checkpoint::setup_text(cfg_, generation(), current_time(), dir, rank);
    return (bool)ofs;
  }
  bool load_state(const std::string &prefix) {
    std::ifstream ifs((prefix + "_setup.txt").c_str());
    int gen = 0;
    double t = 0;
    if (!ifs || !checkpoint::clock_from_setup(ifs, gen, t)) return false;
    if (!read(prefix + ".bin")) return false;
    check(nmhd_set_time(s_, t, gen));
    return true;
  }

  nmhd_diag diagnostics() {
    nmhd_diag d;
    check(nmhd_diagnostics(s_, &d));
    return d;
  }

  nmhd_solver *handle() { return s_; }

 private:
  void check(nmhd_status st) {
    if (st < 0) throw Error(st, nmhd_last_error(s_));
  }
  nmhd_config cfg_;
  nmhd_solver *s_ = nullptr;
  long long last_steps_ = 0;
  std::function<int(MHDSolver &)> monitor_;
};

// Batched ensemble (nmhd_batch_*): many independent boxes advanced together,
// each bitwise as an MHDSolver would advance it alone.  No counterpart in the
// reference, which holds one compile-time box per process.
class Batch {
 public:
  explicit Batch(const std::vector<nmhd_config> &boxes) : cfg_(boxes) {
    nmhd_status st = nmhd_batch_create(cfg_.data(), (int)cfg_.size(), &b_);
    if (st != NMHD_OK) throw Error(st, nmhd_batch_last_error(nullptr));
  }
  ~Batch() { nmhd_batch_destroy(b_); }
  Batch(const Batch &) = delete;
  Batch &operator=(const Batch &) = delete;

  int size() const { return (int)cfg_.size(); }
  size_t cells(int box) const {
    const nmhd_config &c = cfg_.at(box);
    return (size_t)c.size_x * c.size_y * c.size_z;
  }
  // State of one box as 8 host arrays in .bin order, concatenated.
  void initialize_state(int box, const std::vector<float> &all) {
    const float *f[8];
    for (int v = 0; v < 8; ++v) f[v] = all.data() + v * cells(box);
    check(nmhd_batch_set_state(b_, box, f, 0));
  }
  std::vector<float> state(int box) {
    std::vector<float> all(8 * cells(box));
    float *f[8];
    for (int v = 0; v < 8; ++v) f[v] = all.data() + v * cells(box);
    check(nmhd_batch_get_state(b_, box, f, 0));
    return all;
  }
  // Every box's state at once (one host round trip to the control blocks).
  void initialize_states(const std::vector<std::vector<float>> &all) {
    if ((int)all.size() != size()) throw Error(NMHD_ERR_INVALID_ARGUMENT, "one state per box expected");
    std::vector<const float *> f(8 * all.size());
    for (size_t i = 0; i < all.size(); ++i)
      for (int v = 0; v < 8; ++v) f[8 * i + v] = all[i].data() + v * cells((int)i);
    check(nmhd_batch_set_states(b_, f.data(), 0));
  }
  std::vector<std::vector<float>> states() {
    std::vector<std::vector<float>> all(size());
    std::vector<float *> f(8 * all.size());
    for (size_t i = 0; i < all.size(); ++i) {
      all[i].resize(8 * cells((int)i));
      for (int v = 0; v < 8; ++v) f[8 * i + v] = all[i].data() + v * cells((int)i);
    }
    check(nmhd_batch_get_states(b_, f.data(), 0));
    return all;
  }
  // Every box until goal_time (or max_steps steps): true when all reached it.
  bool proceed(float goal_time, long long max_steps = 0) {
    int64_t done = 0;
    const nmhd_status st = nmhd_batch_proceed(b_, goal_time, max_steps, &done);
    check(st);
    last_steps_ = done;
    return st == NMHD_GOAL_REACHED;
  }
  double current_time(int box) {
    double t = 0;
    check(nmhd_batch_clock(b_, box, &t, nullptr));
    return t;
  }
  int generation(int box) {
    int64_t g = 0;
    check(nmhd_batch_clock(b_, box, nullptr, &g));
    return (int)g;
  }
  // Stage-kernel schedules timed on the current states (states unchanged).
  void autotune(int reps = 5) {
    const int k = nmhd_batch_autotune(b_, reps, nullptr, 0);
    if (k < 0) throw Error((nmhd_status)k, nmhd_batch_last_error(b_));
  }
  // One schedule pinned (nmhd_batch_set_schedule: kernel 0-2 the stage
  // kernels, 3 the fused update pass, 4 the staged flux pass).
  void set_schedule(int kernel, bool persistent, bool split) {
    check(nmhd_batch_set_schedule(b_, kernel, persistent ? 1 : 0, split ? 1 : 0));
  }
  // Builds the CUDA graphs a later proceed(..., max_steps) launches
  // (nmhd_batch_prepare).
  void prepare(long long max_steps = 0) { check(nmhd_batch_prepare(b_, max_steps)); }
  long long last_steps() const { return last_steps_; }
  nmhd_batch *handle() { return b_; }

 private:
  void check(nmhd_status st) {
    if (st < 0) throw Error(st, nmhd_batch_last_error(b_));
  }
  std::vector<nmhd_config> cfg_;
  nmhd_batch *b_ = nullptr;
  long long last_steps_ = 0;
};

}  // namespace nmhd

#endif  // NMHD_HPP
