// Singleton summary of an ExaGeoStat run (src/results/Results.cpp:26-259):
// log-likelihood, theta, MSPE, predicted values, Fisher matrix, MLOE/MMOM,
// iteration count and timings.
#pragma once
#include <vector>

namespace exageostat::results {

class Results {
 public:
  static Results* GetInstance() {
    static Results instance;
    return &instance;
  }
  void SetLogLikValue(double v) { mLogLik = v; }
  double GetLogLikValue() const { return mLogLik; }
  void SetMLEIterations(int v) { mMLEIterations = v; }
  int GetMLEIterations() const { return mMLEIterations; }
  void SetMaximumTheta(const std::vector<double>& v) { mMaximumTheta = v; }
  std::vector<double> GetMaximumTheta() const { return mMaximumTheta; }
  void SetMSPEError(double v) { mMSPE = v; }
  double GetMSPEError() const { return mMSPE; }
  void SetPredictedMissedValues(const std::vector<double>& v) { mZMiss = v; }
  std::vector<double> GetPredictedMissedValues() const { return mZMiss; }
  void SetZMiss(int v) { mZMissNumber = v; }
  int GetZMiss() const { return mZMissNumber; }
  void SetTotalModelingExecutionTime(double v) { mModelingTime = v; }
  double GetTotalModelingExecutionTime() const { return mModelingTime; }
  void SetTotalModelingFlops(double v) { mModelingFlops = v; }
  double GetTotalModelingFlops() const { return mModelingFlops; }
  void SetMSPEExecutionTime(double v) { mMSPETime = v; }
  double GetMSPEExecutionTime() const { return mMSPETime; }
  void SetGeneratedLocationsNumber(int v) { mGenerated = v; }
  int GetGeneratedLocationsNumber() const { return mGenerated; }
  // Results.cpp: Fisher matrix (inverse Fisher information, column-major), MLOE, MMOM
  void SetFisherMatrix(const std::vector<double>& v) { mFisher = v; }
  std::vector<double> GetFisherMatrix() const { return mFisher; }
  void SetMLOE(double v) { mMLOE = v; }
  double GetMLOE() const { return mMLOE; }
  void SetMMOM(double v) { mMMOM = v; }
  double GetMMOM() const { return mMMOM; }

 private:
  double mLogLik = 0, mMSPE = 0, mModelingTime = 0, mModelingFlops = 0, mMSPETime = 0, mMLOE = 0, mMMOM = 0;
  int mMLEIterations = 0, mZMissNumber = 0, mGenerated = 0;
  std::vector<double> mMaximumTheta, mZMiss, mFisher;
};

}  // namespace exageostat::results
