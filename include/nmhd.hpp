// nmhd.hpp - header-only C++ mirror of the reference's class MHDSolver
// (src/library/mhd_solver.hrb:150-276) over the C ABI in nmhd.h.
//
// Same member names and meaning as the reference:
//   read/write        -> bool (false on open failure or size mismatch)
//   proceed           -> bool (true when goal_time was reached; false on the
//                        wallclock limit), wallclock_time_limit <= 0 ignored
//   current_time      -> PreciseReal (double), generation -> int
//   save_state/load_state(prefix) -> prefix.bin + prefix_setup.txt
// Problem hooks are not virtual here: the initial state is passed in with
// initialize_state(fields) and the source term is chosen by nmhd_config.
#ifndef NMHD_HPP
#define NMHD_HPP

#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "nmhd.h"

namespace nmhd {

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

  bool proceed(float goal_time, double wallclock_time_limit = -1, long long max_steps = 0) {
    int64_t done = 0;
    nmhd_status st = nmhd_proceed(s_, goal_time, wallclock_time_limit, max_steps, &done);
    last_steps_ = done;
    if (st < 0) throw Error(st, nmhd_last_error(s_));
    return st == NMHD_GOAL_REACHED;
  }

  double current_time() const { return nmhd_current_time(s_); }
  int generation() const { return (int)nmhd_generation(s_); }
  long long last_steps() const { return last_steps_; }

  // save_state/load_state (mhd_solver.inlrb:1023-1050): the .bin dump plus
  // the clock as text (generation and current_time, %.17g).
  bool save_state(const std::string &prefix) {
    if (!write(prefix + ".bin")) return false;
    FILE *fp = std::fopen((prefix + "_setup.txt").c_str(), "w");
    if (!fp) return false;
    std::fprintf(fp, "generation %d\ncurrent_time %.17g\n", generation(), current_time());
    return std::fclose(fp) == 0;
  }
  bool load_state(const std::string &prefix) {
    FILE *fp = std::fopen((prefix + "_setup.txt").c_str(), "r");
    if (!fp) return false;
    int gen = 0;
    double t = 0;
    const bool ok = std::fscanf(fp, "generation %d current_time %lf", &gen, &t) == 2;
    std::fclose(fp);
    if (!ok || !read(prefix + ".bin")) return false;
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
};

}  // namespace nmhd

#endif  // NMHD_HPP
