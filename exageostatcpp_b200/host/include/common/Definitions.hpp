// Enumerations and constants of the ExaGeoStat C++ surface used by the MLE path
// (inst/include/common/Definitions.hpp: Computation, Dimension, Verbose,
// DescriptorName, UpperLower, Side, Trans, Diag, DistanceMetric, PI at :45).
#pragma once
#include <stdexcept>
#include <string>

namespace exageostat::common {

enum Computation { EXACT_DENSE = 0, DIAGONAL_APPROX = 1, TILE_LOW_RANK = 2 };
enum Dimension { Dimension2D = 0, Dimension3D = 1, DimensionST = 2 };
enum Verbose { QUIET_MODE = 0, STANDARD_MODE = 1, DETAILED_MODE = 2 };
enum Precision { SINGLE = 0, DOUBLE = 1, MIXED = 2 };
enum DistanceMetric { EUCLIDEAN_DISTANCE = 0, GREAT_CIRCLE_DISTANCE = 1 };
enum UpperLower { EXAGEOSTAT_UPPER = 121, EXAGEOSTAT_LOWER = 122, EXAGEOSTAT_UPPER_LOWER = 123 };
// Arguments of the triangular solve (Definitions.hpp:91-115).
enum Side { EXAGEOSTAT_LEFT = 141, EXAGEOSTAT_RIGHT = 142 };
enum Trans { EXAGEOSTAT_NO_TRANS = 111, EXAGEOSTAT_TRANS = 112, EXAGEOSTAT_CONJ_TRANS = 113 };
enum Diag { EXAGEOSTAT_NON_UNIT = 131, EXAGEOSTAT_UNIT = 132 };
// The device replaces the Chameleon descriptors; the enumerator is kept so that
// reference code selecting CHAMELEON_DESCRIPTOR still compiles and gets the device view.
enum DescriptorType { CHAMELEON_DESCRIPTOR = 0, HICMA_DESCRIPTOR = 1, CUDA_DESCRIPTOR = 2 };
enum DescriptorName {
  DESCRIPTOR_C = 0,
  DESCRIPTOR_Z,
  DESCRIPTOR_Z_COPY,
  DESCRIPTOR_DETERMINANT,
  DESCRIPTOR_PRODUCT,
  DESCRIPTOR_C12,
  DESCRIPTOR_C22,
  DESCRIPTOR_Z_MISS,
  DESCRIPTOR_Z_OBSERVATIONS,
  DESCRIPTOR_Z_Actual,
  DESCRIPTOR_MSPE
};

constexpr double PI = 3.141592653589793;

}  // namespace exageostat::common
