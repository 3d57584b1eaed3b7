// LinearAlgebraFactory<T>::CreateLinearAlgebraSolver
// (src/linear-algebra-solvers/LinearAlgebraFactory.cpp:31-54): EXACT_DENSE and
// DIAGONAL_APPROX map to the B200 backend (the latter with the configured band);
// TILE_LOW_RANK (HiCMA) is not part of this path.
#pragma once
#include <memory>
#include <stdexcept>
#include "linear-algebra-solvers/concrete/CudaDense.hpp"

namespace exageostat::linearAlgebra {

template <typename T>
class LinearAlgebraFactory {
 public:
  static std::unique_ptr<LinearAlgebraMethods<T>> CreateLinearAlgebraSolver(common::Computation aComputation) {
    if (aComputation == common::EXACT_DENSE || aComputation == common::DIAGONAL_APPROX)
      return std::make_unique<CudaDense<T>>();
    throw std::domain_error("TILE_LOW_RANK (HiCMA) is not part of the B200 path");
  }
};

}  // namespace exageostat::linearAlgebra
