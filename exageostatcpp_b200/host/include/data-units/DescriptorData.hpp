// Descriptors of one data set (src/data-units/DescriptorData.cpp:101-191).
// The reference maps names to Chameleon tile descriptors; here the covariance,
// Z and Zcpy live together in one device-resident egs_problem (the C ABI of the
// B200 library), and GetDescriptor returns a view whose `mat` is a host mirror
// (Z, Zcpy) or nullptr (device-only tiles).  `chameleon_desc` and `cuda_desc`
// name the same view, so reference code reading
//   data->GetDescriptorData()->GetDescriptor(CHAMELEON_DESCRIPTOR, DESCRIPTOR_Z).chameleon_desc->mat
// keeps compiling.
#pragma once
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>
#include "common/Definitions.hpp"
#include "exageostat_b200.h"

namespace exageostat::dataunits {

// The descriptor handle that the solver's tile operations take as void*
// (the reference passes CHAM_desc_t*): the device problem it lives in and
// which of the problem's matrices it names.
template <typename T>
struct DescriptorView {
  T* mat = nullptr;
  int m = 0, n = 0, mb = 0, nb = 0, mt = 0, nt = 0, lm = 0, ln = 0;
  egs_problem* problem = nullptr;
  common::DescriptorName name = common::DESCRIPTOR_C;
};

template <typename T>
struct BaseDescriptor {
  DescriptorView<T>* chameleon_desc = nullptr;
  DescriptorView<T>* cuda_desc = nullptr;
  egs_problem* problem = nullptr;
};

inline void EgsCheck(int status, const char* where) {
  if (status == EGS_OK) return;
  if (status > 0) throw std::runtime_error("Matrix is not positive definite");
  throw std::runtime_error(std::string(where) + ": " + egs_status_string(status) + " " + egs_last_error());
}

template <typename T>
class DescriptorData {
 public:
  DescriptorData() = default;
  ~DescriptorData() {
    if (mProblem) egs_problem_destroy(mProblem);
  }
  DescriptorData(const DescriptorData&) = delete;
  DescriptorData& operator=(const DescriptorData&) = delete;

  // Creates the device problem of n points (dts: the dense tile size); replaces the
  // descriptors InitiateDescriptors makes (LinearAlgebraMethods.cpp:36-118).
  // precision: EGS_PRECISION_DOUBLE or EGS_PRECISION_MIXED (band_tiles FP64 tile
  // rows); a different shape or precision replaces the problem.
  // *created (optional) tells whether a new problem was made.
  egs_problem* EnsureProblem(int n, int dts, int precision = EGS_PRECISION_DOUBLE, int band_tiles = 0,
                             bool* created = nullptr) {
    if (created) *created = false;
    if (mProblem && mN == n && mDts == dts && mPrecision == precision && mBandTiles == band_tiles) return mProblem;
    if (created) *created = true;
    if (mProblem) egs_problem_destroy(mProblem);
    mProblem = nullptr;
    EgsCheck(egs_problem_create_ex(&mProblem, n, dts, precision, band_tiles), "egs_problem_create_ex");
    mN = n;
    mDts = dts;
    mPrecision = precision;
    mBandTiles = band_tiles;
    mIsDescriptorInitiated = true;
    return mProblem;
  }
  egs_problem* GetProblem() const { return mProblem; }

  // Host mirror of a vector descriptor (Z, Zcpy).
  std::vector<T>& HostVector(const common::DescriptorName& aName) { return mHost[aName]; }

  BaseDescriptor<T> GetDescriptor(const common::DescriptorType&, const common::DescriptorName& aName) {
    auto& v = mViews[aName];
    auto it = mHost.find(aName);
    v.mat = (it == mHost.end() || it->second.empty()) ? nullptr : it->second.data();
    const int ts = ((mDts < 64 ? 64 : mDts) + 63) / 64 * 64;
    v.m = mN;
    v.n = (aName == common::DESCRIPTOR_C) ? mN : 1;
    v.mb = mDts;
    v.nb = (aName == common::DESCRIPTOR_C) ? mDts : 1;
    v.mt = mDts > 0 ? (mN + mDts - 1) / mDts : 0;
    v.nt = (aName == common::DESCRIPTOR_C) ? v.mt : 1;
    v.lm = mN;
    v.ln = v.n;
    v.problem = mProblem;
    v.name = aName;
    (void)ts;
    BaseDescriptor<T> d;
    d.chameleon_desc = d.cuda_desc = &v;
    d.problem = mProblem;
    return d;
  }

  T* GetDescriptorMatrix(const common::DescriptorType& aType, const common::DescriptorName& aName) {
    return GetDescriptor(aType, aName).cuda_desc->mat;
  }

  bool GetIsDescriptorInitiated() const { return mIsDescriptorInitiated; }
  void SetIsDescriptorInitiated(bool v) { mIsDescriptorInitiated = v; }

 private:
  egs_problem* mProblem = nullptr;
  int mN = 0, mDts = 0;
  int mPrecision = EGS_PRECISION_DOUBLE, mBandTiles = 0;
  bool mIsDescriptorInitiated = false;
  std::map<int, std::vector<T>> mHost;
  std::map<int, DescriptorView<T>> mViews;
};

}  // namespace exageostat::dataunits
