// oracle/_ref translation unit for the reference's `poisson` equation.
// TEST INFRASTRUCTURE ONLY.  The reference's equation source is compiled where
// it lies (src/equations/poisson.cpp:15-142).
#include "equations/poisson.cpp"
#include "ref_driver.hpp"

WOS_REF_ENTRY(poisson, Poisson2D{static_cast<SourceMode>(pb->source_mode)},
              Poisson3D{static_cast<SourceMode>(pb->source_mode)}, pb->epsilon)
