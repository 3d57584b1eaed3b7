// Structure-of-arrays locations (src/data-units/Locations.cpp:94-118): x, y and,
// for 3-D / space-time data, z.  SetLocationX/Y copy `size` values from the
// first element referenced, as in the reference.
#pragma once
#include <cstring>
#include <stdexcept>
#include <vector>
#include "common/Definitions.hpp"

namespace exageostat::dataunits {

template <typename T>
class Locations {
 public:
  Locations(const int& aSize, const common::Dimension& aDimension) { Resize(aSize, aDimension); }
  Locations() = default;

  void SetSize(const int& aSize) { Resize(aSize, mDimension); }
  int GetSize() const { return mSize; }
  void SetDimension(const common::Dimension& aDimension) { Resize(mSize, aDimension); }
  common::Dimension GetDimension() const { return mDimension; }

  T* GetLocationX() { return mX.data(); }
  T* GetLocationY() { return mY.data(); }
  T* GetLocationZ() { return mZ.empty() ? nullptr : mZ.data(); }
  void SetLocationX(T& aData, const int& aSize) { Copy(mX, &aData, aSize); }
  void SetLocationY(T& aData, const int& aSize) { Copy(mY, &aData, aSize); }
  void SetLocationZ(T& aData, const int& aSize) { Copy(mZ, &aData, aSize); }

 private:
  void Resize(int n, common::Dimension d) {
    mSize = n;
    mDimension = d;
    mX.resize(n);
    mY.resize(n);
    if (d != common::Dimension2D) mZ.resize(n); else mZ.clear();
  }
  static void Copy(std::vector<T>& dst, const T* src, int n) {
    if (n < 0) throw std::runtime_error("negative location count");
    if ((int)dst.size() < n) dst.resize(n);
    std::memcpy(dst.data(), src, sizeof(T) * n);
  }
  int mSize = 0;
  common::Dimension mDimension = common::Dimension2D;
  std::vector<T> mX, mY, mZ;
};

}  // namespace exageostat::dataunits
