// Stand-in for hyteg/types/Matrix.hpp (Eigen wrapper) in the oracle's shell-map library.  Test
// infrastructure only.
#pragma once
#include "hyteg/types/PointMatrixForwardDeclare.hpp"
