// diag.cuh -- device-side diagnostics of a scene (definitions in diag.cu):
// the collision validator's metrics over the current contact list and the
// energy tracker's moments of the velocities, reduced on the GPU so that a
// caller's per-frame check does not download the state.
#pragma once

#include "common.cuh"

namespace ando {

// Sums, extremes and counts of CollisionMetrics::compute_from_contacts
// (collision_validator.cpp:7-111) and of the relative normal velocities of
// CollisionValidator::compute_relative_velocities (:181-221). Gaps are
// compared in single precision, as the reference's Real does.
struct MetricSums {
  double min_gap, max_gap, sum_gap, max_pen, sum_pen, max_rv, sum_rv;
  int n, n_pt, n_ee, n_wall, n_pen, n_major, n_tunnel, n_ccd, n_rv;
};

// Kinetic energy, linear and angular momentum and the largest speed of a
// state (energy_tracker.cpp:7-42).
struct MomentSums {
  double ke, p[3], L[3], vmax2;
};

// Largest number of per-block partials (the grids are capped there).
constexpr int DIAG_MAX_BLOCKS = 4 * 148;

// Two launches each: per-block partials into `parts` (DIAG_MAX_BLOCKS
// entries), then one block folds them in block order into `out`. Results do
// not depend on timing.
void launch_contact_metrics(const ContactDev* contacts, int n, const double* v, double gap_max, int ccd, MetricSums* parts,
                            MetricSums* out, cudaStream_t s);
void launch_state_moments(int V, const double* x, const double* v, const double* mass, MomentSums* parts, MomentSums* out,
                          cudaStream_t s);

}  // namespace ando
