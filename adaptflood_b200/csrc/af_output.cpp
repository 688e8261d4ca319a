// af_output.cpp -- ASC and NetCDF output (see af_output.h) and the
// af_write_asc entry point.  ASC grids of 10^8 cells are written by
// formatting row blocks in parallel into memory and writing the blocks in
// order.
#include "af_output.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>

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

// ------------------------------------------------------------ NetCDF
namespace {

// Big-endian encoders of the classic format's header and data.
void put_u32(std::vector<unsigned char>& b, uint32_t v) {
  for (int k = 3; k >= 0; k--) b.push_back((unsigned char)(v >> (8 * k)));
}
void put_u64(std::vector<unsigned char>& b, uint64_t v) {
  for (int k = 7; k >= 0; k--) b.push_back((unsigned char)(v >> (8 * k)));
}
void put_f64(std::vector<unsigned char>& b, double x) {
  uint64_t v;
  std::memcpy(&v, &x, 8);
  put_u64(b, v);
}
void put_f32(std::vector<unsigned char>& b, float x) {
  uint32_t v;
  std::memcpy(&v, &x, 4);
  put_u32(b, v);
}
void pad4(std::vector<unsigned char>& b) {
  while (b.size() % 4) b.push_back(0);
}
// A name: its length, then its bytes padded to 4.
void put_name(std::vector<unsigned char>& b, const char* s) {
  const uint32_t n = (uint32_t)std::strlen(s);
  put_u32(b, n);
  b.insert(b.end(), s, s + n);
  pad4(b);
}
constexpr uint32_t kNcChar = 2, kNcFloat = 5, kNcDouble = 6;
constexpr uint32_t kTagDimension = 10, kTagVariable = 11, kTagAttribute = 12;

void put_text_att(std::vector<unsigned char>& b, const char* name, const char* text, int len) {
  put_name(b, name);
  put_u32(b, kNcChar);
  put_u32(b, (uint32_t)len);
  b.insert(b.end(), text, text + len);
  pad4(b);
}
void put_double_att(std::vector<unsigned char>& b, const char* name, double v) {
  put_name(b, name);
  put_u32(b, kNcDouble);
  put_u32(b, 1);
  put_f64(b, v);
}
void put_float_att(std::vector<unsigned char>& b, const char* name, float v) {
  put_name(b, name);
  put_u32(b, kNcFloat);
  put_u32(b, 1);
  put_f32(b, v);
}

}  // namespace

NcFile::~NcFile() {
  if (fp_) fclose(fp_);
}

bool NcFile::open(const std::string& path, int nx, int ny, bool velocity, double xll, double yll,
                  double cellsize, double nodata) {
  ncells_ = (long long)nx * ny;
  const long long vsize = ncells_ * 4;  // one record of H, Vx or Vy
  if (nx <= 0 || ny <= 0 || vsize > 0xFFFFFFFCLL) return false;
  velocity_ = velocity;
  // The header is built twice: the variables' offsets depend on its size.
  std::vector<unsigned char> h;
  for (int pass = 0; pass < 2; pass++) {
    const uint64_t hsize = h.size();
    h.clear();
    h.push_back('C'), h.push_back('D'), h.push_back('F'), h.push_back(2);
    put_u32(h, 0);  // records so far
    put_u32(h, kTagDimension);  // dimensions 0: time (the record dimension), 1: x, 2: y
    put_u32(h, 3);
    put_name(h, "time"), put_u32(h, 0);
    put_name(h, "x"), put_u32(h, (uint32_t)nx);
    put_name(h, "y"), put_u32(h, (uint32_t)ny);
    put_u32(h, kTagAttribute);  // global attributes (src/async_output.cpp:47-49)
    put_u32(h, 3);
    put_double_att(h, "xllcorner", xll);
    put_double_att(h, "yllcorner", yll);
    put_double_att(h, "cellsize", cellsize);
    put_u32(h, kTagVariable);
    put_u32(h, velocity ? 4 : 2);
    uint64_t begin = hsize;  // records start right after the header
    // time(time): double, "seconds" (src/async_output.cpp:27-28)
    put_name(h, "time");
    put_u32(h, 1), put_u32(h, 0);
    put_u32(h, kTagAttribute), put_u32(h, 1);
    put_text_att(h, "units", "seconds", 7);
    put_u32(h, kNcDouble), put_u32(h, 8), put_u64(h, begin);
    begin += 8;
    // H(time, y, x): float (src/async_output.cpp:30-35)
    put_name(h, "H");
    put_u32(h, 3), put_u32(h, 0), put_u32(h, 2), put_u32(h, 1);
    put_u32(h, kTagAttribute), put_u32(h, 3);
    put_text_att(h, "units", "m", 1);
    put_text_att(h, "long_name", "water_depth", 11);
    put_float_att(h, "_FillValue", (float)nodata);
    put_u32(h, kNcFloat), put_u32(h, (uint32_t)vsize), put_u64(h, begin);
    begin += vsize;
    if (velocity) {  // src/async_output.cpp:37-45 (long_name lengths 16 as passed there)
      const char* names[2] = {"Vx", "Vy"};
      const char* longs[2] = {"x_direction_velocity", "y_direction_velocity"};
      for (int v = 0; v < 2; v++) {
        put_name(h, names[v]);
        put_u32(h, 3), put_u32(h, 0), put_u32(h, 2), put_u32(h, 1);
        put_u32(h, kTagAttribute), put_u32(h, 2);
        put_text_att(h, "units", "m/s", 3);
        put_text_att(h, "long_name", longs[v], 16);
        put_u32(h, kNcFloat), put_u32(h, (uint32_t)vsize), put_u64(h, begin);
        begin += vsize;
      }
    }
  }
  rec0_ = (long long)h.size();
  recsize_ = 8 + vsize * (velocity ? 3 : 1);
  nrec_ = 0;
  fp_ = fopen(path.c_str(), "wb");
  if (!fp_) return false;
  return fwrite(h.data(), 1, h.size(), fp_) == h.size() && fflush(fp_) == 0;
}

bool NcFile::append(double time, const double* H, const double* Vx, const double* Vy) {
  if (!fp_) return false;
  const long long off = rec0_ + (long long)nrec_ * recsize_;
  if (fseeko(fp_, (off_t)off, SEEK_SET) != 0) return false;
  buf_.clear();
  put_f64(buf_, time);
  if (fwrite(buf_.data(), 1, buf_.size(), fp_) != buf_.size()) return false;
  // The fields in chunks of 1 Mi values, converted to big-endian float.
  constexpr long long kChunk = 1 << 20;
  const double* fields[3] = {H, Vx, Vy};
  for (int f = 0; f < (velocity_ ? 3 : 1); f++) {
    for (long long i0 = 0; i0 < ncells_; i0 += kChunk) {
      const long long i1 = std::min(ncells_, i0 + kChunk);
      buf_.resize((size_t)(i1 - i0) * 4);
      unsigned char* o = buf_.data();
      for (long long i = i0; i < i1; i++, o += 4) {
        const float x = fields[f] ? (float)fields[f][i] : 0.0f;
        uint32_t u;
        std::memcpy(&u, &x, 4);
#if __BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__
        u = __builtin_bswap32(u);
#endif
        std::memcpy(o, &u, 4);
      }
      if (fwrite(buf_.data(), 1, buf_.size(), fp_) != buf_.size()) return false;
    }
  }
  std::vector<unsigned char> n;
  put_u32(n, (uint32_t)(nrec_ + 1));
  // The record count last, so a reader never sees a record before its data.
  if (fflush(fp_) != 0 || fseeko(fp_, 4, SEEK_SET) != 0 || fwrite(n.data(), 1, 4, fp_) != 4 ||
      fflush(fp_) != 0)
    return false;
  nrec_++;
  return true;
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

struct af_netcdf {
  af::NcFile f;
  bool velocity = false;
};

extern "C" int af_netcdf_create(const char* path, int ncols, int nrows, int voutput, double xll,
                                double yll, double cellsize, double nodata, af_netcdf** out) {
  if (!path || !out || ncols <= 0 || nrows <= 0) return AF_EINVAL;
  if ((long long)ncols * nrows * 4 > 0xFFFFFFFCLL) return AF_ERANGE;
  af_netcdf* h = new (std::nothrow) af_netcdf();
  if (!h) return AF_ENOMEM;
  h->velocity = voutput != 0;
  if (!h->f.open(path, ncols, nrows, h->velocity, xll, yll, cellsize, nodata)) {
    delete h;
    return AF_EIO;
  }
  *out = h;
  return AF_OK;
}

extern "C" int af_netcdf_append(af_netcdf* f, double time, const double* H, const double* Vx,
                                const double* Vy) {
  if (!f || !H || (f->velocity && (!Vx || !Vy))) return AF_EINVAL;
  return f->f.append(time, H, f->velocity ? Vx : nullptr, f->velocity ? Vy : nullptr) ? AF_OK
                                                                                     : AF_EIO;
}

extern "C" int af_netcdf_close(af_netcdf* f) {
  delete f;
  return AF_OK;
}

extern "C" int af_write_asc(const char* path, const double* values, int ncols, int nrows,
                            double xll, double yll, double cellsize, double nodata, int style) {
  if (!path || (!values && (long long)ncols * nrows > 0) || ncols < 0 || nrows < 0 ||
      (style != af::kAscSync && style != af::kAscAsync))
    return AF_EINVAL;
  return af::write_asc(path, values, ncols, nrows, xll, yll, cellsize, nodata, style, 0)
             ? AF_OK
             : AF_EIO;
}
