// Compile-time configuration for the host-compiled reference solver (test
// infrastructure only).
//
// The reference takes every size and physics constant from a generated
// simulation_config.h (defaults: src/library/simulation_config_default.h;
// per-application overrides: src/application/*/simulation_config.hrb).  This
// file provides the same names, filled from -D macros by oracle/Makefile, for
// NMHD_REF_PY ranks along Y (default 1; kParallelSize{X,Z} == 1), fully
// periodic addressing, and margins in Y (the shearing direction) and
// optionally Z.
//
//   NMHD_REF_DOUBLE   0: Real = float (USE_SINGLE_PRECISION), 1: Real = double
//   NMHD_REF_G{X,Y,Z} interior cell counts of the whole box (kGlobalSize*)
//   NMHD_REF_PY       ranks along Y (kParallelSizeY), each a radial slab
//   NMHD_REF_M{Y,Z}   margin widths (kMarginSize*)
//   NMHD_REF_L{X,Y,Z} global extents (kGlobalExtent*)
//   NMHD_REF_GAMMA    kGamma expression, e.g. (5.0f/3.0f)
//   NMHD_REF_CFL      kCflFactor
//   NMHD_REF_Q, NMHD_REF_OMEGA   shearing-box rotation parameters
#pragma once
#include "cuda_host_shim.h"
#include "library/direction.h"

#define USE_MPI

#if NMHD_REF_DOUBLE
#define USE_DOUBLE_PRECISION
#undef USE_SINGLE_PRECISION
typedef double Real;
#else
#define USE_SINGLE_PRECISION
#undef USE_DOUBLE_PRECISION
typedef float Real;
#endif
typedef double PreciseReal;

#include "library/math.h"

#define kGamma Real(NMHD_REF_GAMMA)
const Real kCflFactor = NMHD_REF_CFL;

typedef int addr_t;

#define CRYSTAL_PERIODIC_X
#define CRYSTAL_PERIODIC_Y
#define CRYSTAL_PERIODIC_Z

const int kGlobalSizeX = NMHD_REF_GX;
const int kGlobalSizeY = NMHD_REF_GY;
const int kGlobalSizeZ = NMHD_REF_GZ;

#ifndef NMHD_REF_PY
#define NMHD_REF_PY 1
#endif
const int kParallelSizeX = 1;
const int kParallelSizeY = NMHD_REF_PY;
const int kParallelSizeZ = 1;
const int kParallelSize = NMHD_REF_PY;

const int kMarginSizeX = 0;
const int kMarginSizeY = NMHD_REF_MY;
const int kMarginSizeZ = NMHD_REF_MZ;
const int gMarginSizeX = kMarginSizeX;
const int gMarginSizeY = kMarginSizeY;
const int gMarginSizeZ = kMarginSizeZ;

const int kLocalSizeX = kGlobalSizeX / kParallelSizeX;
const int kLocalSizeY = kGlobalSizeY / kParallelSizeY;
const int kLocalSizeZ = kGlobalSizeZ / kParallelSizeZ;

const int kSizeX = kLocalSizeX + 2 * kMarginSizeX;
const int kSizeY = kLocalSizeY + 2 * kMarginSizeY;
const int kSizeZ = kLocalSizeZ + 2 * kMarginSizeZ;
const size_t kSize = size_t(kSizeX) * size_t(kSizeY) * size_t(kSizeZ);
const int gSizeX = kSizeX;
const int gSizeY = kSizeY;
const int gSizeZ = kSizeZ;
const int gSize = kSize;

const Real kGlobalExtentX = NMHD_REF_LX;
const Real kGlobalExtentY = NMHD_REF_LY;
const Real kGlobalExtentZ = NMHD_REF_LZ;
const Real gGlobalExtentX = kGlobalExtentX;
const Real gGlobalExtentY = kGlobalExtentY;
const Real gGlobalExtentZ = kGlobalExtentZ;

const Real kExtentX = kGlobalExtentX / Real(kGlobalSizeX) * Real(kSizeX);
const Real kExtentY = kGlobalExtentY / Real(kGlobalSizeY) * Real(kSizeY);
const Real kExtentZ = kGlobalExtentZ / Real(kGlobalSizeZ) * Real(kSizeZ);
const Real gExtentX = kExtentX;
const Real gExtentY = kExtentY;
const Real gExtentZ = kExtentZ;

const Real kLocalExtentX = kGlobalExtentX / Real(kGlobalSizeX) * Real(kLocalSizeX);
const Real kLocalExtentY = kGlobalExtentY / Real(kGlobalSizeY) * Real(kLocalSizeY);
const Real kLocalExtentZ = kGlobalExtentZ / Real(kGlobalSizeZ) * Real(kLocalSizeZ);

const Real kGlobalCornerX = 0.0;
const Real kGlobalCornerY = 0.0;
const Real kGlobalCornerZ = 0.0;

const Real kDX = kExtentX / kSizeX;
const Real kDY = kExtentY / kSizeY;
const Real kDZ = kExtentZ / kSizeZ;

namespace {
namespace simulation_config {
int size(XAxis) { return kSizeX; }
int size(YAxis) { return kSizeY; }
int size(ZAxis) { return kSizeZ; }
Real extent(XAxis) { return kExtentX; }
Real extent(YAxis) { return kExtentY; }
Real extent(ZAxis) { return kExtentZ; }
}
Real dR(XAxis) { return kDX; }
Real dR(YAxis) { return kDY; }
Real dR(ZAxis) { return kDZ; }
}

const Real kDifferentialRotationIndex = NMHD_REF_Q;
const Real kOmega = NMHD_REF_OMEGA;
const Real gDifferentialRotationIndex = kDifferentialRotationIndex;
const Real gOmega = kOmega;
