/* Oracle: CPU restatement of the reference ideal-MHD time step.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load this library, and only as the
 * correctness reference or the timed CPU baseline; the product (libnmhd.so)
 * never calls it.
 *
 * It restates, in plain C, the reference's MHDSolver::proceed
 * (src/library/mhd_solver.inlrb:850-993, generated src/library/mhd_solver.inl)
 * with runtime sizes, including every float/double promotion the reference
 * source performs, so that the float build is bitwise equal to the reference
 * built on the host (oracle/_ref, pinned in tests/test_oracle_pin.py and by
 * the committed fixtures in tests/golden/).
 *
 * State layout: 8 arrays of Sx*Sy*Sz values, x fastest, in the order of the
 * reference's .bin dump: density, vx, vy, vz, pressure, Bx, By, Bz; B component
 * d at index i is the lower d-face of cell i.
 */
#ifndef NMHD_ORACLE_H
#define NMHD_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same field order as nmhd_config in include/nmhd.h. */
typedef struct oracle_config {
  int32_t size_x, size_y, size_z;
  int32_t margin_y, margin_z;
  float extent_x, extent_y, extent_z;
  float gamma, cfl;
  int32_t problem; /* 0 none, 1 shearing box */
  float q, omega;
  int32_t space_order; /* 2 minbee, 1 piecewise constant */
  int32_t time_order;  /* 2 midpoint, 1 Euler */
  int32_t flags;       /* 1: margins refilled before the second RK2 stage */
  /* kParallelSizeY: P > 1 makes the state one radial slab of a box split over
   * P ranks along Y (size_y: the slab's rows and margins; extent_y: the
   * box's), advanced with the split-phase functions below */
  int32_t parallel_size_y;
} oracle_config;

/* float build (the reference's FP32) */
/* Advances `state` by at most max_steps steps of MHDSolver::proceed(goal_time).
 * times_out (max_steps+1 entries) receives current_time before every step and
 * after the last; dt_out the dt of every step; *goal_reached is set when the
 * goal time was reached.  Returns the number of steps taken. */
int oracle_proceed_f32(const oracle_config *cfg, float *state, double *time, int64_t *generation,
                       double goal_time, int max_steps, double *times_out, float *dt_out,
                       int *goal_reached);
void oracle_hlld_f32(float gamma, float bx, const float lr[14], float out[7]);
float oracle_cfl_f32(const oracle_config *cfg, const float *state, float goal);
void oracle_shear_fill_f32(const oracle_config *cfg, float *state, double time);
/* Split-phase step of one rank of a P-rank run (MHDSolver::proceed with
 * communicate(), src/library/mhd_solver.inlrb:283-493, 850-993):
 *   halo_pack    the two outgoing Y messages of communicate_gather_kernel_y
 *                (:184-222) at time t: send_inc (to the rank above) and
 *                send_dec (to the rank below), each 8 x Sx*My*Sz values
 *   halo_unpack  communicate_scatter_kernel_y (:224-242) of the received
 *                messages into the Y margins, then the Z-margin copies
 *   stages       the RK stages of one step with the common dt (:904-978).
 * With P = 1 and each message delivered to itself this is oracle_proceed's
 * step. */
void oracle_halo_pack_f32(const oracle_config *cfg, const float *state, double time, float *send_inc,
                          float *send_dec);
void oracle_halo_unpack_f32(const oracle_config *cfg, float *state, const float *recv_inc,
                            const float *recv_dec);
void oracle_stages_f32(const oracle_config *cfg, float *state, float dt);

/* double build (the reference with Real = double) */
int oracle_proceed_f64(const oracle_config *cfg, double *state, double *time, int64_t *generation,
                       double goal_time, int max_steps, double *times_out, double *dt_out,
                       int *goal_reached);
void oracle_hlld_f64(double gamma, double bx, const double lr[14], double out[7]);
double oracle_cfl_f64(const oracle_config *cfg, const double *state, double goal);
void oracle_shear_fill_f64(const oracle_config *cfg, double *state, double time);
void oracle_halo_pack_f64(const oracle_config *cfg, const double *state, double time, double *send_inc,
                          double *send_dec);
void oracle_halo_unpack_f64(const oracle_config *cfg, double *state, const double *recv_inc,
                            const double *recv_dec);
void oracle_stages_f64(const oracle_config *cfg, double *state, double dt);

#ifdef __cplusplus
}
#endif
#endif
