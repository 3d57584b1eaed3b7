// CSV data loader and writer (src/data-loader/concrete/CSVLoader.cpp:37-289) for
// univariate 2-D data: one line "x,y,z" per location.  A line with a fourth
// value does not match 2-D univariate data and is rejected, as the reference
// rejects data whose dimensions disagree with the configuration.
#pragma once
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>
#include "configurations/Configurations.hpp"
#include "data-units/ExaGeoStatData.hpp"

namespace exageostat::dataLoader::csv {

template <typename T>
class CSVLoader {
 public:
  // CSVLoader<T>::ReadData (CSVLoader.cpp:37-143): fills x, y and the
  // measurements; the problem size becomes the number of lines.
  static void ReadData(configurations::Configurations& aConfigurations, std::vector<T>& aMeasurements,
                       std::vector<T>& aX, std::vector<T>& aY) {
    const std::string path = aConfigurations.GetDataPath();
    if (path.empty()) throw std::runtime_error("Please enter the path to data file.");
    if (aConfigurations.GetDimension() != common::Dimension2D)
      throw std::domain_error("only 2D locations are on the B200 path");
    std::ifstream file(path);
    if (!file.is_open()) throw std::runtime_error("Cannot read locations file: " + path);
    std::string line;
    int lines = 0;
    while (std::getline(file, line)) {
      if (line.empty()) continue;
      std::istringstream iss(line);
      std::string tok;
      T v[3];
      for (int k = 0; k < 3; ++k) {
        if (!std::getline(iss, tok, ','))
          throw std::runtime_error("line " + std::to_string(lines + 1) + " of " + path + " has fewer than 3 values");
        v[k] = (T)std::stod(tok);
      }
      if (std::getline(iss, tok, ','))
        throw std::runtime_error("The data dimensions in the provided file isn't consistent with the dimensions input.");
      aX.push_back(v[0]);
      aY.push_back(v[1]);
      aMeasurements.push_back(v[2]);
      ++lines;
    }
    aConfigurations.SetProblemSize(lines);
  }

  // CSVLoader<T>::WriteData (CSVLoader.cpp:146-289), 2-D univariate: writes
  // <dir>/SYN_<n>_<i> with 15 significant digits, i the first index with no
  // <dir>/log_<n>_<i>; returns the file name.
  static std::string WriteData(const T* apZ, int aN, std::string aDirectory, dataunits::Locations<T>& aLocations) {
    if (aDirectory.empty()) aDirectory = "synthetic_ds";
    else aDirectory += (aDirectory.back() == '/') ? "synthetic_ds" : "/synthetic_ds";
    std::error_code ec;
    std::filesystem::create_directories(aDirectory, ec);
    if (!std::filesystem::exists(aDirectory)) throw std::runtime_error("Error creating directory: " + aDirectory);
    size_t i = 1;
    const std::string base_log = aDirectory + "/log_" + std::to_string(aN) + "_";
    while (std::filesystem::exists(base_log + std::to_string(i))) ++i;
    const std::string name = aDirectory + "/SYN_" + std::to_string(aN) + "_" + std::to_string(i);
    std::ofstream out(name);
    if (!out.is_open()) throw std::runtime_error("Cannot write " + name);
    for (int k = 0; k < aN; ++k)
      out << std::setprecision(15) << aLocations.GetLocationX()[k] << ',' << aLocations.GetLocationY()[k] << ','
          << std::setprecision(15) << apZ[k] << '\n';
    return name;
  }

  // Data object of the file's locations; the measurements go to the Z host vector.
  static std::unique_ptr<dataunits::ExaGeoStatData<T>> LoadData(configurations::Configurations& aConfigurations) {
    std::vector<T> z, x, y;
    ReadData(aConfigurations, z, x, y);
    const int n = aConfigurations.GetProblemSize();
    auto data = std::make_unique<dataunits::ExaGeoStatData<T>>(n, aConfigurations.GetDimension());
    data->GetLocations()->SetLocationX(*x.data(), n);
    data->GetLocations()->SetLocationY(*y.data(), n);
    data->GetDescriptorData()->HostVector(common::DESCRIPTOR_Z) = z;
    return data;
  }
};

}  // namespace exageostat::dataLoader::csv
