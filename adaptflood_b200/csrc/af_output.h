// af_output.h -- the reference's file outputs, host side: ESRI ASCII grids
// with "%.4f " values (src/io.cpp:314-334 and src/async_output.cpp:158-176)
// and a background writer thread (src/async_output.cpp:84-106).
#pragma once

#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <functional>
#include <mutex>
#include <queue>
#include <string>
#include <thread>
#include <vector>

namespace af {

// The text printf("%.4f", x) produces, without printf: exact decimal rounding
// of the double (round half to even on exact ties, the sign kept on values
// that round to zero).  Returns the length written to out (>= 32 bytes).
int format_f4(double x, char* out);

// Header styles of the reference's two ASC writers.
enum AscStyle {
  kAscSync = 0,   // write_asc (src/io.cpp:314-334): xll/yll "%.1f", NODATA "-9999"
  kAscAsync = 1,  // the async writer (src/async_output.cpp:158-176): "%.6f", "%.0f"
};

// Writes one grid (row 0 = north, values[i + j*ncols]); the values are
// formatted by `threads` threads (0: one per hardware thread).  false on an
// I/O error.
bool write_asc(const char* path, const double* values, int ncols, int nrows, double xll,
               double yll, double cellsize, double nodata, int style, int threads);

// The reference's NetCDF output (src/async_output.cpp:20-51, 109-138): one
// file with dimensions time (unlimited), x = ncols, y = nrows; variables
// time(time) double "seconds", H(time, y, x) float with units, long_name and
// _FillValue = nodata, with velocity also Vx and Vy (their long_name cut to
// the 16 characters the reference passes); global attributes xllcorner,
// yllcorner and cellsize; one record per save, values rounded to float.
// Written in NetCDF's classic container with 64-bit offsets (the published
// classic format: big-endian header of dimension, attribute and variable
// lists, then the records), which every NetCDF reader reads with the same
// data model; the reference's NC_NETCDF4 flag selects the HDF5 container,
// whose library is not available here.  The record count in the header is
// rewritten after every record, so the file is complete after each one.
class NcFile {
 public:
  ~NcFile();
  // false on an I/O error or a grid whose one record of H exceeds 4 GiB - 4.
  bool open(const std::string& path, int nx, int ny, bool velocity, double xll, double yll,
            double cellsize, double nodata);
  bool append(double time, const double* H, const double* Vx, const double* Vy);

 private:
  FILE* fp_ = nullptr;
  long long ncells_ = 0, rec0_ = 0, recsize_ = 0;
  int nrec_ = 0;
  bool velocity_ = false;
  std::vector<unsigned char> buf_;
};

// A single background thread that runs file-writing jobs in order.
class Writer {
 public:
  Writer();
  ~Writer();  // finishes the queued jobs
  void post(std::function<void()> job);
  void drain();  // waits until every posted job has run
  int errors() const { return errors_; }
  void fail() { errors_++; }

 private:
  void loop();
  std::mutex mu_;
  std::condition_variable cv_, idle_;
  std::queue<std::function<void()>> q_;
  bool stop_ = false;
  int running_ = 0;
  std::atomic<int> errors_{0};
  std::thread th_;
};

}  // namespace af
