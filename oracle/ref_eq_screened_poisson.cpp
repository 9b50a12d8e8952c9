// oracle/_ref translation unit for the reference's `screened_poisson`
// equation.  TEST INFRASTRUCTURE ONLY.  The reference's equation source is
// compiled where it lies (src/equations/screened_poisson.cpp:20-167); the
// epsilon clamp is the reference's own screened_epsilon (:22-38), called with
// a non-zero rank so it does not print.
#include "equations/screened_poisson.cpp"
#include "ref_driver.hpp"

WOS_REF_ENTRY(screened_poisson,
              (ScreenedPoisson2D{pb->alpha, static_cast<SourceMode>(pb->source_mode)}),
              (ScreenedPoisson3D{pb->alpha, static_cast<SourceMode>(pb->source_mode)}),
              screened_epsilon(1, pb->epsilon, pb->alpha))
