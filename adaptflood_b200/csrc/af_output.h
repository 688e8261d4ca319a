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
