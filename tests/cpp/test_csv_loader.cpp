// Host-only checks of the CSV data loader and writer
// (exageostatcpp_b200/host/include/data-loader/CSVLoader.hpp, following
// src/data-loader/concrete/CSVLoader.cpp:37-289): no GPU call is made.
// Usage: test_csv_loader <scratch directory>; prints one "name: ok|FAIL ..."
// line per case and exits non-zero if any case failed.
#include <cmath>
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>
#include "data-loader/CSVLoader.hpp"

using exageostat::configurations::Configurations;
using exageostat::dataLoader::csv::CSVLoader;
using exageostat::dataunits::Locations;

namespace {

int failures = 0;

void report(const char* name, bool ok, const std::string& why = "") {
  std::printf("%s: %s%s%s\n", name, ok ? "ok" : "FAIL", why.empty() ? "" : " ", why.c_str());
  if (!ok) ++failures;
}

void write_file(const std::string& path, const std::string& text) {
  std::ofstream f(path);
  f << text;
}

// The error message of ReadData on a file holding `text`, or "" if it read.
std::string read_error(const std::string& path, const std::string& text) {
  write_file(path, text);
  Configurations c;
  c.SetDataPath(path);
  std::vector<double> z, x, y;
  try {
    CSVLoader<double>::ReadData(c, z, x, y);
  } catch (const std::exception& e) {
    return e.what();
  }
  return "";
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: %s <scratch directory>\n", argv[0]);
    return 2;
  }
  const std::string dir = argv[1];

  // Round trip: 15 significant digits written, read back within 1e-14.
  {
    const int n = 5;
    std::vector<double> x = {0.123456789012345, 0.5, 0.999999999999999, 1e-7, 0.25};
    std::vector<double> y = {0.3, 0.141592653589793, 0.0, 0.75, 2.0 / 3.0};
    std::vector<double> z = {-1.23456789012345, 0.0, 3.5e-3, 42.0, -7.0 / 3.0};
    Locations<double> loc(n, exageostat::common::Dimension2D);
    loc.SetLocationX(x[0], n);
    loc.SetLocationY(y[0], n);
    const std::string name = CSVLoader<double>::WriteData(z.data(), n, dir + "/rt", loc);
    report("write_name", name == dir + "/rt/synthetic_ds/SYN_5_1", name);
    Configurations c;
    c.SetDataPath(name);
    std::vector<double> rz, rx, ry;
    CSVLoader<double>::ReadData(c, rz, rx, ry);
    bool ok = c.GetProblemSize() == n && rz.size() == (size_t)n && rx.size() == (size_t)n && ry.size() == (size_t)n;
    for (int k = 0; ok && k < n; ++k) {
      auto close = [](double a, double b) { return std::fabs(a - b) <= 1e-14 * std::fmax(1.0, std::fabs(b)); };
      ok = close(rx[k], x[k]) && close(ry[k], y[k]) && close(rz[k], z[k]);
    }
    report("round_trip", ok);
  }

  // The file index is the first i without a log_<n>_<i> beside it.
  {
    const int n = 3;
    std::vector<double> v = {1.0, 2.0, 3.0};
    Locations<double> loc(n, exageostat::common::Dimension2D);
    loc.SetLocationX(v[0], n);
    loc.SetLocationY(v[0], n);
    const std::string sub = dir + "/idx";
    std::filesystem::create_directories(sub + "/synthetic_ds");
    write_file(sub + "/synthetic_ds/log_3_1", "");
    write_file(sub + "/synthetic_ds/log_3_2", "");
    const std::string name = CSVLoader<double>::WriteData(v.data(), n, sub, loc);
    report("write_index", name == sub + "/synthetic_ds/SYN_3_3", name);
  }

  // Blank lines are skipped; the problem size is the number of data lines.
  {
    write_file(dir + "/blank.csv", "0.1,0.2,0.3\n\n0.4,0.5,0.6\n");
    Configurations c;
    c.SetDataPath(dir + "/blank.csv");
    std::vector<double> z, x, y;
    CSVLoader<double>::ReadData(c, z, x, y);
    report("blank_lines", c.GetProblemSize() == 2 && z.size() == 2 && z[1] == 0.6);
  }

  // A fourth value does not match 2-D univariate data.
  {
    const std::string e = read_error(dir + "/four.csv", "0.1,0.2,0.3\n0.4,0.5,0.6,0.7\n");
    report("reject_four_values", e.find("dimensions") != std::string::npos, e);
  }
  // Fewer than three values.
  {
    const std::string e = read_error(dir + "/two.csv", "0.1,0.2\n");
    report("reject_two_values", e.find("fewer than 3 values") != std::string::npos, e);
  }
  // A missing path and an unreadable file.
  {
    Configurations c;
    std::vector<double> z, x, y;
    std::string e;
    try {
      CSVLoader<double>::ReadData(c, z, x, y);
    } catch (const std::exception& ex) {
      e = ex.what();
    }
    report("reject_empty_path", e.find("path") != std::string::npos, e);
    c.SetDataPath(dir + "/does_not_exist.csv");
    e.clear();
    try {
      CSVLoader<double>::ReadData(c, z, x, y);
    } catch (const std::exception& ex) {
      e = ex.what();
    }
    report("reject_missing_file", e.find("Cannot read") != std::string::npos, e);
  }
  return failures == 0 ? 0 : 1;
}
