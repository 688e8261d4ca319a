// af_output.cpp -- ASC output (see af_output.h) and the af_write_asc entry
// point.  Grids of 10^8 cells are written by formatting row blocks in
// parallel into memory and writing the blocks in order.
#include "af_output.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "adaptflood.h"

namespace af {

int format_f4(double x, char* out) {
  // Beyond 1e11, x*1e4 nears 2^53 and the exact-fraction argument below no
  // longer holds: leave those (and non-finite values) to printf.
  if (!std::isfinite(x) || std::fabs(x) >= 1e11) return snprintf(out, 32, "%.4f", x);
  char* o = out;
  if (std::signbit(x)) *o++ = '-';
  const double a = std::fabs(x);
  // a*1e4 = p + e exactly (e from one FMA); the fraction p - floor(p) is exact.
  const double p = a * 1e4;
  const double e = std::fma(a, 1e4, -p);
  const double k = std::floor(p);
  const double f = p - k;
  uint64_t n = (uint64_t)k;
  // f is a multiple of ulp(p) and |e| <= ulp(p)/2, so unless f is exactly
  // one half the comparison with 0.5 decides; at f == 0.5 the sign of e does,
  // and an exact tie rounds to even (printf's rounding of the exact value).
  if (f > 0.5 || (f == 0.5 && (e > 0.0 || (e == 0.0 && (n & 1u))))) n++;
  const uint64_t ip = n / 10000u, fp = n % 10000u;
  char buf[24];
  int m = 0;
  uint64_t v = ip;
  do {
    buf[m++] = (char)('0' + v % 10u);
    v /= 10u;
  } while (v);
  while (m) *o++ = buf[--m];
  *o++ = '.';
  o[0] = (char)('0' + fp / 1000u);
  o[1] = (char)('0' + fp / 100u % 10u);
  o[2] = (char)('0' + fp / 10u % 10u);
  o[3] = (char)('0' + fp % 10u);
  o += 4;
  return (int)(o - out);
}

static void format_rows(const double* values, int ncols, int j0, int j1, std::string& s) {
  s.clear();
  s.reserve((size_t)(j1 - j0) * ncols * 8);
  char cell[40];
  for (int j = j0; j < j1; j++) {
    const double* row = values + (size_t)j * ncols;
    for (int i = 0; i < ncols; i++) {
      const int n = format_f4(row[i], cell);
      cell[n] = ' ';
      s.append(cell, n + 1);
    }
    s.push_back('\n');
  }
}

bool write_asc(const char* path, const double* values, int ncols, int nrows, double xll,
               double yll, double cellsize, double nodata, int style, int threads) {
  FILE* fp = fopen(path, "wb");
  if (!fp) return false;
  if (style == kAscAsync) {
    fprintf(fp, "ncols         %d\n", ncols);
    fprintf(fp, "nrows         %d\n", nrows);
    fprintf(fp, "xllcorner     %.6f\n", xll);
    fprintf(fp, "yllcorner     %.6f\n", yll);
    fprintf(fp, "cellsize      %.1f\n", cellsize);
    fprintf(fp, "NODATA_value  %.0f\n", nodata);
  } else {
    fprintf(fp, "ncols         %d\n", ncols);
    fprintf(fp, "nrows         %d\n", nrows);
    fprintf(fp, "xllcorner     %.1f\n", xll);
    fprintf(fp, "yllcorner     %.1f\n", yll);
    fprintf(fp, "cellsize      %.1f\n", cellsize);
    fprintf(fp, "NODATA_value  -9999\n");
  }
  if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
  const long long cells = (long long)ncols * nrows;
  if (cells < 200000) threads = 1;
  // Blocks of rows, formatted `threads` at a time, written in order.
  const int rows_per = std::max(1, (int)std::min<long long>(nrows, (1 << 20) / std::max(1, ncols) + 1));
  std::vector<std::string> bufs(threads);
  bool ok = true;
  for (int j = 0; j < nrows && ok; j += rows_per * threads) {
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; t++) {
      const int a = j + t * rows_per, b = std::min(nrows, a + rows_per);
      if (a >= b) {
        bufs[t].clear();
        continue;
      }
      if (t == threads - 1 || threads == 1)
        format_rows(values, ncols, a, b, bufs[t]);
      else
        pool.emplace_back(format_rows, values, ncols, a, b, std::ref(bufs[t]));
    }
    for (auto& th : pool) th.join();
    for (auto& s : bufs)
      if (!s.empty() && fwrite(s.data(), 1, s.size(), fp) != s.size()) ok = false;
  }
  if (fclose(fp) != 0) ok = false;
  return ok;
}

Writer::Writer() : th_([this] { loop(); }) {}

Writer::~Writer() {
  {
    std::lock_guard<std::mutex> g(mu_);
    stop_ = true;
  }
  cv_.notify_all();
  th_.join();
}

void Writer::post(std::function<void()> job) {
  {
    std::lock_guard<std::mutex> g(mu_);
    q_.push(std::move(job));
  }
  cv_.notify_one();
}

void Writer::drain() {
  std::unique_lock<std::mutex> l(mu_);
  idle_.wait(l, [this] { return q_.empty() && running_ == 0; });
}

void Writer::loop() {
  for (;;) {
    std::function<void()> job;
    {
      std::unique_lock<std::mutex> l(mu_);
      cv_.wait(l, [this] { return stop_ || !q_.empty(); });
      if (q_.empty()) {
        if (stop_) return;
        continue;
      }
      job = std::move(q_.front());
      q_.pop();
      running_++;
    }
    job();
    {
      std::lock_guard<std::mutex> g(mu_);
      running_--;
    }
    idle_.notify_all();
  }
}

}  // namespace af

extern "C" int af_write_asc(const char* path, const double* values, int ncols, int nrows,
                            double xll, double yll, double cellsize, double nodata, int style) {
  if (!path || (!values && (long long)ncols * nrows > 0) || ncols < 0 || nrows < 0 ||
      (style != af::kAscSync && style != af::kAscAsync))
    return AF_EINVAL;
  return af::write_asc(path, values, ncols, nrows, xll, yll, cellsize, nodata, style, 0)
             ? AF_OK
             : AF_EIO;
}
