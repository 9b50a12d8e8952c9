// oracle/_ref translation unit for the reference's `helmholtz` equation.
// TEST INFRASTRUCTURE ONLY.  The reference's equation source is compiled where
// it lies (src/equations/helmholtz.cpp:15-102).
#include "equations/helmholtz.cpp"
#include "ref_driver.hpp"

WOS_REF_ENTRY(helmholtz, Helmholtz2D{}, Helmholtz3D{}, pb->epsilon)
