// fixed_rotation.hpp — observability probe of translation-and-structure problems with fixed rotations
// (probe_fixed_rotation_observability, crates/openmvg-ba/src/kernel/fixed_rotation/observability.rs:
// 24-262) and its inputs in the library's own form.
#pragma once

#include <cstdint>
#include <vector>

#include "ba_cuda.h"
#include "ba_device.cuh"

namespace omvgba {

struct Context;

struct ProbeCamera {
  double R[9];           // world-to-camera rotation, row-major (held)
  double C[3];           // camera centre
  double intrinsics[9];  // fx, fy, cx, cy, k1, k2, k3, p1, p2 (a Brown-Conrady K1K2K3 / P1P2 camera)
  bool fixed;
};

struct ProbeProblem {
  std::vector<ProbeCamera> cameras;
  std::vector<double> points;     // 3 per point
  std::vector<uint64_t> track_off;  // points + 1
  std::vector<uint32_t> obs_cam;
  std::vector<double> obs_px;     // 2 per observation
  bool fixed_baseline = false;
  uint64_t anchor = 0, scale_camera = 1;
  double distance = 0.0;
  LossDev loss{kLossL2, 0.0};     // weights are taken relative to the loss at 0
};

// The probe's outcome; throws SolveFailure{OMVGBA_INVALID_ARGUMENT} for invalid options and
// SolveFailure{OMVGBA_INVALID_PROBLEM} for an inconsistent problem (FixedRotationError, api.rs).
omvgba_probe_report probe_fixed_rotation(Context* ctx, const ProbeProblem& problem,
                                         const omvgba_probe_options& options);

void probe_options_default(omvgba_probe_options* options);

// Positive definiteness of the symmetric n x n matrix whose lower triangle is given by the entries
// (row >= col), decided by the banded tiled Cholesky on the context's device. Throws SolveFailure.
bool device_certify_positive_definite(Context* ctx, int n, const std::vector<int>& rows, const std::vector<int>& cols,
                                      const std::vector<double>& values);

}  // namespace omvgba
