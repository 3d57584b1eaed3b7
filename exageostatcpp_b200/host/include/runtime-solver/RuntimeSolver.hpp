// MLE driver (src/runtime-solver/concrete/StarpuRuntimeSolver.cpp:28-79): maximise
// the log-likelihood over the box [lb, ub] from the starting theta with
// ftol_abs = 10^-tolerance and maxeval = max MLE iterations, using the library's
// BOBYQA (egs_bobyqa_maximize, same first evaluations and stopping rules as
// NLopt's LN_BOBYQA).  Returns the best value found; the optimum is written back
// into the starting theta and the estimated theta (:48-49).  An exception thrown
// by an evaluation ends the fit and is re-thrown here, as NLopt propagates it.
#pragma once
#include <cmath>
#include <exception>
#include <limits>
#include <memory>
#include "configurations/Configurations.hpp"
#include "data-units/ExaGeoStatData.hpp"
#include "linear-algebra-solvers/LinearAlgebraFactory.hpp"

namespace exageostat::runtimesolver {

template <typename T>
class RuntimeSolver {
 public:
  T ModelingOperations(std::unique_ptr<dataunits::ExaGeoStatData<T>>& aData,
                       configurations::Configurations& aConfigurations, T* apMeasurementsMatrix,
                       const kernels::Kernel<T>& aKernel) {
    Context ctx{&aData, &aConfigurations, apMeasurementsMatrix, &aKernel, nullptr};
    const int np = aKernel.GetParametersNumbers();
    std::vector<double>& x = aConfigurations.GetStartingTheta();
    std::vector<double> lb = aConfigurations.GetLowerBounds(), ub = aConfigurations.GetUpperBounds();
    // Fixed parameters (lb == ub, from InitializeAllTheta) are not optimised.
    std::vector<int> free_idx;
    for (int i = 0; i < np; ++i)
      if (ub[i] > lb[i]) free_idx.push_back(i);
    ctx.full = x;
    ctx.free_idx = free_idx;
    double fbest = -std::numeric_limits<double>::infinity();
    if (free_idx.empty()) {
      fbest = Evaluate((int)x.size(), x.data(), &ctx);
    } else {
      std::vector<double> xf, lf, uf;
      for (int i : free_idx) {
        xf.push_back(x[i]);
        lf.push_back(lb[i]);
        uf.push_back(ub[i]);
      }
      int nevals = 0;
      const int rc = egs_bobyqa_maximize((int)xf.size(), xf.data(), lf.data(), uf.data(), 0.0,
                                         aConfigurations.GetTolerance(), aConfigurations.GetMaxMleIterations(),
                                         &RuntimeSolver::Trampoline, &ctx, &fbest, &nevals);
      if (ctx.error) std::rethrow_exception(ctx.error);
      dataunits::EgsCheck(rc, "egs_bobyqa_maximize");
      for (size_t k = 0; k < free_idx.size(); ++k) x[free_idx[k]] = xf[k];
    }
    aConfigurations.SetEstimatedTheta(x);
    return fbest;
  }

 private:
  struct Context {
    std::unique_ptr<dataunits::ExaGeoStatData<T>>* data;
    configurations::Configurations* config;
    T* measurements;
    const kernels::Kernel<T>* kernel;
    std::exception_ptr error;
    std::vector<double> full;
    std::vector<int> free_idx;
  };

  static double Evaluate(int, const double* theta, Context* ctx) {
    auto solver = linearAlgebra::LinearAlgebraFactory<T>::CreateLinearAlgebraSolver(ctx->config->GetComputation());
    return solver->ExaGeoStatMLETile(*ctx->data, *ctx->config, theta, ctx->measurements, *ctx->kernel);
  }

  // C callback of the optimiser: no exception may cross it.
  static double Trampoline(int n, const double* xf, void* p) {
    auto* ctx = static_cast<Context*>(p);
    if (ctx->error) return -std::numeric_limits<double>::infinity();
    try {
      std::vector<double> theta = ctx->full;
      for (int k = 0; k < n; ++k) theta[ctx->free_idx[k]] = xf[k];
      return Evaluate((int)theta.size(), theta.data(), ctx);
    } catch (...) {
      ctx->error = std::current_exception();
      return -std::numeric_limits<double>::infinity();
    }
  }
};

}  // namespace exageostat::runtimesolver
