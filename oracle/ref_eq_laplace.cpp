// oracle/_ref translation unit for the reference's `laplace` equation.
// TEST INFRASTRUCTURE ONLY.  The reference's equation source is compiled where
// it lies (src/equations/laplace.cpp:12-69); this file only adds the C entry
// points of oracle/ref_driver.hpp around its Laplace2D / Laplace3D values.
#include "equations/laplace.cpp"
#include "ref_driver.hpp"

WOS_REF_ENTRY(laplace, Laplace2D{}, Laplace3D{}, pb->epsilon)
