// Host build of the single-box step's face arithmetic (nmhd_b200/csrc/
// mhd_math.cuh: minbee reconstruction and the HLLD flux), for the CPU tests
// only.  The library's kernels compile the same functions for sm_100a with
// -fmad=false and IEEE division and square root; here gcc rounds every float
// and double operation separately (-ffp-contract=off, SSE arithmetic), so the
// results are the device's and the tests can compare them bitwise with the
// oracle on a CPU.  Not part of the library; nothing in nmhd_b200 loads it.
#include "../../nmhd_b200/csrc/mhd_math.cuh"

extern "C" {

// lr: dl, dr, ul, ur, vl, vr, wl, wr, pl, pr, byl, byr, bzl, bzr (HlldIn order)
void cellh_hlld_f32(float gamma, float bx, const float *lr, float *out) {
  nmhd::HlldIn in;
  float *dst = &in.dl;
  for (int i = 0; i < 14; ++i) dst[i] = lr[i];
  nmhd::hlld_flux(gamma, bx, in, out);
}

void cellh_hlld_many_f32(float gamma, const float *bx, const float *lr, float *out, long n) {
  for (long i = 0; i < n; ++i) cellh_hlld_f32(gamma, bx[i], lr + 14 * i, out + 7 * i);
}

void cellh_reconstruct_f32(const float *x, float *lr, long n) {
  for (long i = 0; i < n; ++i) nmhd::reconstruct4(x[4 * i], x[4 * i + 1], x[4 * i + 2], x[4 * i + 3], lr[2 * i], lr[2 * i + 1]);
}

}  // extern "C"
