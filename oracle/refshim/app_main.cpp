// Driver for the host-compiled reference solver (test infrastructure only).
// Appended after the reference's src/library/mhd_solver.inl by oracle/Makefile.
//
//   <binary> IN.bin OUT.bin NSTEPS [GOAL_TIME] [TIMES.txt]
//
// Reads the initial primitive state with MHDSolver::read, advances until
// generation NSTEPS with MHDSolver::proceed (monitor() stops the loop, as in
// src/library/mhd_solver.inlrb:859-860), writes the state with
// MHDSolver::write, and prints one JSON line with the wallclock of the proceed()
// call.  TIMES.txt receives current_time() before every step and after the
// last, as %.17g.
//
// Checkpoints (MHDSolver::save_state/load_state, mhd_solver.inlrb:1023-1050):
// with NMHD_REF_DIR set, the solver's LocalSetup is that of this rank writing
// under NMHD_REF_DIR; NMHD_REF_LOAD=tag starts from load_state(tag) instead of
// IN.bin, NMHD_REF_SAVE=tag calls save_state(tag) after the run.
//
// Several ranks (a binary built with NMHD_REF_PY > 1): the caller starts one
// process per rank with NMHD_REF_RANK / NMHD_REF_NRANKS / NMHD_REF_MAILBOX
// (refshim/mpi.h) and NMHD_REF_DIR; "%d"-style conversions in IN.bin,
// OUT.bin and TIMES.txt are replaced by the rank, the way each rank of the
// reference's applications reads and writes its own files
// (src/application/kepler_disk_demo/main.curb:47-110).
#include <sys/time.h>
#include <omp.h>

static int g_max_steps = 0;
static std::vector<double> g_times;

void MHDSolver::dump(std::string) {}
int MHDSolver::monitor() {
  g_times.push_back(current_time());
  return generation() >= g_max_steps;
}
int MHDSolver::initial_event() { return 0; }
int MHDSolver::final_event() { return 0; }

static double nmhd_now() {
  timeval tv;
  gettimeofday(&tv, 0);
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}

int main(int argc, char **argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: %s IN.bin OUT.bin NSTEPS [GOAL_TIME] [TIMES.txt]\n", argv[0]);
    return 2;
  }
  g_max_steps = std::atoi(argv[3]);
  double goal = argc > 4 ? std::atof(argv[4]) : 1.0e30;
  const char *dir = std::getenv("NMHD_REF_DIR");
  const char *load_tag = std::getenv("NMHD_REF_LOAD");
  const char *save_tag = std::getenv("NMHD_REF_SAVE");
  int mpi_rank = 0, mpi_size = 1;
  MPI_Init(&argc, &argv);
  MPI_Comm_rank(MPI_COMM_WORLD, &mpi_rank);
  MPI_Comm_size(MPI_COMM_WORLD, &mpi_size);
  if (mpi_size != kParallelSize || (mpi_size > 1 && !dir)) {
    std::fprintf(stderr, "this binary runs %d rank(s) and needs NMHD_REF_DIR for more than one\n",
                 kParallelSize);
    return 2;
  }
  auto ranked = [mpi_rank](const char *path) {
    char b[4096];
    std::snprintf(b, sizeof b, path, mpi_rank);
    return std::string(b);
  };
  const std::string in_path = ranked(argv[1]), out_path = ranked(argv[2]);
  // LocalSetup(rank, dir) opens its log files under dir: only when asked
  LocalSetup *setup = dir ? new LocalSetup(mpi_rank, dir) : &blancLocalSetup;
  MHDSolver solver(*setup);
  if (dir && load_tag) {
    solver.load_state(load_tag);
  } else if (!solver.read(in_path)) {
    std::fprintf(stderr, "cannot read %s (missing or size mismatch)\n", in_path.c_str());
    return 1;
  }
  // The reference prints "t dt" to stderr every step; silence it for timing.
  std::cerr.setstate(std::ios_base::failbit);
  double t0 = nmhd_now();
  bool reached = solver.proceed(Real(goal));
  double t1 = nmhd_now();
  std::cerr.clear();
  if (!solver.write(out_path)) {
    std::fprintf(stderr, "cannot write %s\n", out_path.c_str());
    return 1;
  }
  if (dir && save_tag) solver.save_state(save_tag);
  if (argc > 5) {
    FILE *fp = std::fopen(ranked(argv[5]).c_str(), "w");
    for (size_t i = 0; i < g_times.size(); ++i) std::fprintf(fp, "%.17g\n", g_times[i]);
    std::fclose(fp);
  }
  std::printf(
      "{\"steps\": %d, \"cells\": %zu, \"seconds\": %.6f, \"threads\": %d, \"goal_reached\": %d, "
      "\"time\": %.17g, \"sizeof_real\": %d, \"rank\": %d}\n",
      solver.generation(), (size_t)kSize, t1 - t0, omp_get_max_threads(), reached ? 1 : 0,
      solver.current_time(), (int)sizeof(Real), mpi_rank);
  MPI_Finalize();
  return 0;
}
