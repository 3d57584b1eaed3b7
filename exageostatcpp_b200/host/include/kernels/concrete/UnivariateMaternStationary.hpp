// The univariate stationary Matern kernel plugin
// (src/kernels/concrete/UnivariateMaternStationary.cpp:25-67), theta = (sigma^2,
// beta, nu), registered by name.  GenerateCovarianceMatrix computes the block on
// the GPU (egs_matern_block) and returns it in the caller's host array; the MLE
// path never calls it -- CudaDense generates the covariance tiles in place on the
// device -- but reference code that calls the plugin directly gets the same values.
#pragma once
#include <cuda_runtime.h>
#include <stdexcept>
#include <vector>
#include "data-units/DescriptorData.hpp"
#include "kernels/Kernel.hpp"

namespace exageostat::kernels {

template <typename T>
class UnivariateMaternStationary : public Kernel<T> {
 public:
  UnivariateMaternStationary() {
    this->mP = 1;
    this->mParametersNumber = 3;
  }
  std::string GetKernelName() const override { return "UnivariateMaternStationary"; }
  static Kernel<T>* Create() {
    KernelsConfigurations::GetParametersNumberKernelMap()["UnivariateMaternStationary"] = 3;
    return new UnivariateMaternStationary<T>();
  }

  void GenerateCovarianceMatrix(T* apMatrixA, const int& aRowsNumber, const int& aColumnsNumber,
                                const int& aRowOffset, const int& aColumnOffset, dataunits::Locations<T>& aLocation1,
                                dataunits::Locations<T>& aLocation2, dataunits::Locations<T>&, T* aLocalTheta,
                                const int& aDistanceMetric) override {
    static_assert(sizeof(T) == sizeof(double), "the device path is FP64");
    const int r = aRowsNumber, c = aColumnsNumber;
    if (r <= 0 || c <= 0) return;
    double *d = nullptr, *x1 = nullptr, *y1 = nullptr, *x2 = nullptr, *y2 = nullptr;
    auto fail = [&](const char* what) {
      cudaFree(d); cudaFree(x1); cudaFree(y1); cudaFree(x2); cudaFree(y2);
      throw std::runtime_error(what);
    };
    if (cudaMalloc(&d, sizeof(double) * (size_t)r * c) || cudaMalloc(&x1, sizeof(double) * r) ||
        cudaMalloc(&y1, sizeof(double) * r) || cudaMalloc(&x2, sizeof(double) * c) ||
        cudaMalloc(&y2, sizeof(double) * c))
      fail("device allocation failed in GenerateCovarianceMatrix");
    cudaMemcpy(x1, aLocation1.GetLocationX() + aRowOffset, sizeof(double) * r, cudaMemcpyHostToDevice);
    cudaMemcpy(y1, aLocation1.GetLocationY() + aRowOffset, sizeof(double) * r, cudaMemcpyHostToDevice);
    cudaMemcpy(x2, aLocation2.GetLocationX() + aColumnOffset, sizeof(double) * c, cudaMemcpyHostToDevice);
    cudaMemcpy(y2, aLocation2.GetLocationY() + aColumnOffset, sizeof(double) * c, cudaMemcpyHostToDevice);
    const int rc = egs_matern_block(d, r, r, c, x1, y1, x2, y2, aLocalTheta, aDistanceMetric, nullptr);
    if (rc != EGS_OK) fail(egs_last_error());
    cudaMemcpy(apMatrixA, d, sizeof(double) * (size_t)r * c, cudaMemcpyDeviceToHost);
    cudaFree(d); cudaFree(x1); cudaFree(y1); cudaFree(x2); cudaFree(y2);
  }

 private:
  static inline bool plugin_name = plugins::PluginRegistry<Kernel<T>>::Add(
      "UnivariateMaternStationary", UnivariateMaternStationary<T>::Create);
};

template class UnivariateMaternStationary<double>;

}  // namespace exageostat::kernels
