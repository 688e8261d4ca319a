// af_io.cpp -- .par / DEM / .bci / .bdy / rain readers with the reference's
// parsing rules (src/io.cpp:9-296), producing an af_case_desc and the flat
// forcing tables of adaptflood.h.
//
// Rules kept from the reference, deliberately:
//   * .par: `key value` lines; '#' or empty lines skipped; unknown keys
//     ignored; the key spellings are the parser's (fpfric, depth_thresh,
//     initial_tstep, dirroot, ...) (src/io.cpp:27-43).
//   * DEM: six `key value` header pairs read in order without checking the
//     key names, then rows north to south (src/io.cpp:137-156).
//   * .bci `P X Y TYPE [v|name]`: world coordinates mapped with truncation
//     toward zero, y measured down from the top edge (src/io.cpp:185-187);
//     QFIX/HFIX values parsed with atof; a type without its required field,
//     or an unknown type, is skipped (src/io.cpp:183-217).
//   * .bci `N|S|E|W a b FREE` makes that whole side FREE; only the 4-field
//     form is recognised, so `N FREE` leaves the side CLOSED (src/io.cpp:221-249).
//   * .bdy: the first line is skipped; a line naming a QVAR/HVAR boundary
//     (name + end of line, space, CR or LF) starts its section -- the first
//     such boundary in .bci order gets it -- then a count line, then
//     `value time` lines (src/io.cpp:261-294).
//   * rain: a header line, then `rate time` lines; a missing rain file
//     disables rain (src/io.cpp:103-129).
// Differences, all on inputs the reference mishandles: a point outside the
// grid, a truncated DEM, or an unreadable .bdy count/value line is an error
// (AF_ERANGE / AF_EIO) instead of an out-of-bounds index or an uninitialised
// value; lines are not limited to 255 characters.
#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "adaptflood.h"

namespace {

struct PointBC {
  int x = 0, y = 0, idx = 0, type = AF_BC_CLOSED;
  double value = 0.0;
  std::string name;
  std::vector<double> times, values;
};

struct Par {
  std::string dem_file = "dem.ascii", bci_file = "bci.bci", bdy_file = "bdy.bdy";
  std::string rain_file, stage_file, output_dir = "results";
  double sim_time = 3600.0, save_int = 600.0, mass_int = 60.0, stage_int = 60.0;
  double init_tstep = 10.0, cfl = 0.7, fpn = 0.035, depth_thresh = 0.001;
  int output_format = 0;
  bool voutput = false, async_output = true;
};

bool parse_double(const std::string& s, double* out) {
  const char* b = s.c_str();
  char* e = nullptr;
  errno = 0;
  double v = strtod(b, &e);
  if (e == b) return false;
  *out = v;
  return true;
}

bool parse_int(const std::string& s, int* out) {
  const char* b = s.c_str();
  char* e = nullptr;
  long v = strtol(b, &e, 10);
  if (e == b) return false;
  *out = (int)v;
  return true;
}

// src/io.cpp:9-47
int read_par(const char* path, Par& p) {
  std::ifstream f(path);
  if (!f.is_open()) return AF_EIO;
  std::string line;
  while (std::getline(f, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::istringstream iss(line);
    std::string key, value;
    if (!(iss >> key)) continue;
    iss >> value;
    bool ok = true;
    if (key == "DEMfile") p.dem_file = value;
    else if (key == "bcifile") p.bci_file = value;
    else if (key == "bdyfile") p.bdy_file = value;
    else if (key == "dirroot") p.output_dir = value;
    else if (key == "sim_time") ok = parse_double(value, &p.sim_time);
    else if (key == "saveint") ok = parse_double(value, &p.save_int);
    else if (key == "massint") ok = parse_double(value, &p.mass_int);
    else if (key == "initial_tstep") ok = parse_double(value, &p.init_tstep);
    else if (key == "cfl") ok = parse_double(value, &p.cfl);
    else if (key == "fpfric") ok = parse_double(value, &p.fpn);
    else if (key == "depth_thresh") ok = parse_double(value, &p.depth_thresh);
    else if (key == "rainfile") p.rain_file = value;
    else if (key == "stagefile") p.stage_file = value;
    else if (key == "stageint") ok = parse_double(value, &p.stage_int);
    else if (key == "output_format") ok = parse_int(value, &p.output_format);
    else if (key == "voutput") p.voutput = true;
    else if (key == "async_output") {
      int v = 0;
      ok = parse_int(value, &v);
      p.async_output = v != 0;
    }
    if (!ok) return AF_EIO;  // the reference's std::stod/stoi would throw here
  }
  return AF_OK;
}

static inline bool is_ws(char c) {
  return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f';
}

// Parses the whitespace-separated values of [s, end) into out (at most cap
// values); each token is converted by strtod and must be consumed entirely.
// Returns the number of tokens, or -1 on a malformed token.
static long long parse_values(const char* s, const char* end, double* out, long long cap) {
  long long n = 0;
  while (s < end) {
    while (s < end && is_ws(*s)) s++;
    if (s >= end) break;
    const char* t = s;
    while (t < end && !is_ws(*t)) t++;
    if (n < cap) {
      char* e = nullptr;
      out[n] = strtod(s, &e);
      if (e != t) return -1;
    }
    n++;
    s = t;
  }
  return n;
}

static long long count_tokens(const char* s, const char* end) {
  long long n = 0;
  bool in = false;
  for (; s < end; s++) {
    const bool w = is_ws(*s);
    n += (!w && !in);
    in = !w;
  }
  return n;
}

// src/io.cpp:132-161: the six header pairs, then ncols*nrows values, row 0 =
// north.  The file is read in one piece and the values are converted in
// parallel: the text is cut at whitespace into one chunk per thread, the
// tokens of each chunk are counted, and each thread converts its chunk with
// strtod (the correctly rounded conversion fscanf("%lf") performs) at its
// offset, so the values are those of a sequential read.
int read_dem(const char* path, int& ncols, int& nrows, double& xll, double& yll, double& cs,
             double& nodata, std::vector<double>& data) {
  FILE* fp = fopen(path, "rb");
  if (!fp) return AF_EIO;
  std::string buf;
  if (fseek(fp, 0, SEEK_END) == 0) {
    const long sz = ftell(fp);
    if (sz > 0) {
      buf.resize((size_t)sz);
      rewind(fp);
      if (fread(&buf[0], 1, (size_t)sz, fp) != (size_t)sz) {
        fclose(fp);
        return AF_EIO;
      }
    }
  }
  fclose(fp);
  const char* s = buf.c_str();
  char* e = nullptr;
  auto skip_word = [&]() {
    while (is_ws(*s)) s++;
    while (*s && !is_ws(*s)) s++;
  };
  double hdr[6];
  for (int k = 0; k < 6; k++) {
    skip_word();
    if (k < 2) {
      long v = strtol(s, &e, 10);
      if (e == s) return AF_EIO;
      hdr[k] = (double)v;
    } else {
      double v = strtod(s, &e);
      if (e == s) return AF_EIO;
      hdr[k] = v;
    }
    s = e;
  }
  ncols = (int)hdr[0];
  nrows = (int)hdr[1];
  xll = hdr[2];
  yll = hdr[3];
  cs = hdr[4];
  nodata = hdr[5];
  if (ncols < 0 || nrows < 0) return AF_EIO;
  const long long n = (long long)ncols * (long long)nrows;
  data.assign((size_t)n, 0.0);
  const char* end = buf.c_str() + buf.size();
  int T = (int)std::min<unsigned>(32u, std::max(1u, std::thread::hardware_concurrency()));
  if (end - s < (1 << 20)) T = 1;
  // chunk boundaries at whitespace
  std::vector<const char*> cut(T + 1, end);
  cut[0] = s;
  for (int t = 1; t < T; t++) {
    const char* c = s + (end - s) * (long long)t / T;
    while (c < end && !is_ws(*c)) c++;
    cut[t] = std::max(c, cut[t - 1]);
  }
  std::vector<long long> cnt(T, 0), off(T + 1, 0);
  {
    std::vector<std::thread> th;
    for (int t = 0; t < T; t++)
      th.emplace_back([&, t] { cnt[t] = count_tokens(cut[t], cut[t + 1]); });
    for (auto& x : th) x.join();
  }
  for (int t = 0; t < T; t++) off[t + 1] = off[t] + cnt[t];
  if (off[T] < n) return AF_EIO;  // fewer values than the header announces
  std::vector<int> bad(T, 0);
  {
    std::vector<std::thread> th;
    for (int t = 0; t < T; t++)
      th.emplace_back([&, t] {
        if (off[t] >= n) return;
        const long long got =
            parse_values(cut[t], cut[t + 1], data.data() + off[t], n - off[t]);
        bad[t] = got < 0;
      });
    for (auto& x : th) x.join();
  }
  for (int t = 0; t < T; t++)
    if (bad[t]) return AF_EIO;
  return AF_OK;
}

// src/io.cpp:164-254
int read_bci(const char* path, double xll, double yll, int ncols, int nrows, double cs,
             std::vector<PointBC>& pts, bool free_side[4]) {
  std::ifstream f(path);
  if (!f.is_open()) return AF_EIO;
  const double tly = yll + nrows * cs;
  std::string ln;
  while (std::getline(f, ln)) {
    ln.push_back('\n');  // fgets keeps the newline
    const char* line = ln.c_str();
    if (line[0] == '#' || line[0] == '\n' || line[0] == '\r') continue;
    char type = line[0];
    if (type == 'P') {
      double x, y;
      char t = 0;
      std::vector<char> bctype(ln.size() + 1, 0), extra(ln.size() + 1, 0);
      int n = sscanf(line, "%c %lf %lf %s %s", &t, &x, &y, bctype.data(), extra.data());
      if (n < 4) continue;
      PointBC pb;
      pb.x = (int)((x - xll) / cs);
      pb.y = (int)((tly - y) / cs);
      if (pb.x < 0 || pb.x >= ncols || pb.y < 0 || pb.y >= nrows) return AF_ERANGE;
      pb.idx = pb.x + pb.y * ncols;
      pb.value = 0.0;
      const char* bt = bctype.data();
      if (strcmp(bt, "QVAR") == 0 && n >= 5) {
        pb.type = AF_BC_QVAR;
        pb.name = extra.data();
      } else if (strcmp(bt, "QFIX") == 0 && n >= 5) {
        pb.type = AF_BC_QFIX;
        pb.value = atof(extra.data());
      } else if (strcmp(bt, "FREE") == 0) {
        pb.type = AF_BC_FREE;
      } else if (strcmp(bt, "HFIX") == 0 && n >= 5) {
        pb.type = AF_BC_HFIX;
        pb.value = atof(extra.data());
      } else if (strcmp(bt, "HVAR") == 0 && n >= 5) {
        pb.type = AF_BC_HVAR;
        pb.name = extra.data();
      } else {
        continue;  // unknown point BC type: skipped
      }
      pts.push_back(pb);
    } else if (type == 'N' || type == 'S' || type == 'E' || type == 'W') {
      char t = 0;
      int a = 0, b = 0;
      std::vector<char> bctype(ln.size() + 1, 0);
      int n = sscanf(line, "%c %d %d %s", &t, &a, &b, bctype.data());
      bool is_free = (n >= 4 && strcmp(bctype.data(), "FREE") == 0);
      if (!is_free && n >= 2) {
        std::vector<char> bt2(ln.size() + 1, 0);
        is_free = sscanf(line, "%c %s", &t, bt2.data()) == 2 && strcmp(bt2.data(), "FREE") == 0;
      }
      if (is_free) {
        int side = type == 'W' ? 0 : type == 'E' ? 1 : type == 'N' ? 2 : 3;
        free_side[side] = true;
      }
    }
  }
  return AF_OK;
}

// src/io.cpp:257-296
int read_bdy(const char* path, std::vector<PointBC>& pts) {
  std::ifstream f(path);
  if (!f.is_open()) return AF_EIO;
  std::string line;
  std::getline(f, line);
  while (std::getline(f, line)) {
    if (line.empty() || line[0] == '#') continue;
    for (auto& pb : pts) {
      if (pb.type != AF_BC_QVAR && pb.type != AF_BC_HVAR) continue;
      const size_t L = pb.name.size();
      if (line.compare(0, L, pb.name) == 0 && line.size() >= L &&
          (line.size() == L || line[L] == ' ' || line[L] == '\n' || line[L] == '\r')) {
        if (!std::getline(f, line)) return AF_EIO;
        int n = 0;
        if (sscanf(line.c_str(), "%d", &n) != 1 || n < 0) return AF_EIO;
        for (int i = 0; i < n; i++) {
          if (!std::getline(f, line)) return AF_EIO;
          double val, time;
          if (sscanf(line.c_str(), "%lf %lf", &val, &time) != 2) return AF_EIO;
          pb.times.push_back(time);
          pb.values.push_back(val);
        }
        break;
      }
    }
  }
  return AF_OK;
}

// src/io.cpp:103-129; a missing file leaves rain disabled.
void read_rain(const char* path, std::vector<double>& times, std::vector<double>& rates) {
  std::ifstream f(path);
  if (!f.is_open()) return;
  std::string line;
  std::getline(f, line);
  while (std::getline(f, line)) {
    if (line.empty() || line[0] == '#') continue;
    double rate, time;
    if (sscanf(line.c_str(), "%lf %lf", &rate, &time) == 2) {
      times.push_back(time);
      rates.push_back(rate);
    }
  }
}

}  // namespace

struct af_scenario {
  af_case_desc c{};
  std::vector<double> dem;
  double par[3] = {0, 0, 0};
  double geo[3] = {0, 0, 0};
  std::vector<int> flow_idx, flow_type, flow_off, other_idx, other_type, other_off;
  std::vector<double> flow_value, flow_times, flow_vals, other_value, other_times, other_vals;
  std::vector<double> rain_times, rain_rates;
  // outputs (af_scenario_output)
  std::string out_dir;
  double save_int = 0.0, stage_int = 0.0;
  int voutput = 0, async_output = 1, output_format = 0;
  std::vector<int> stage_idx;
  std::vector<std::string> stage_names;
  std::vector<const char*> stage_name_ptrs;
};

namespace {

// src/io.cpp:50-85: stage points "x y [name]" in world coordinates, '#'
// comments; grid cell by the truncating mapping of the BCI points; a missing
// name is "Stage<n>".  The cell index the reference reads is gx + gy*ncols
// when that lies in the grid (src/main.cpp:312-313), else the point prints NaN
// (-1 here).  An unreadable file disables stage output, as there.
void read_stage_file(const char* path, double xll, double yll, int ncols, int nrows, double cs,
                     af_scenario& sc) {
  std::ifstream f(path);
  if (!f.is_open()) return;
  const double tly = yll + nrows * cs;
  std::string line;
  while (std::getline(f, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::istringstream iss(line);
    double x = 0.0, y = 0.0;
    if (!(iss >> x >> y)) continue;
    std::string name;
    iss >> name;
    if (name.empty()) name = "Stage" + std::to_string(sc.stage_names.size() + 1);
    const long long gx = (long long)(int)((x - xll) / cs);
    const long long gy = (long long)(int)((tly - y) / cs);
    const long long idx = gx + gy * ncols;
    sc.stage_idx.push_back(idx >= 0 && idx < (long long)ncols * nrows ? (int)idx : -1);
    sc.stage_names.push_back(name);
  }
}

}  // namespace

extern "C" {

int af_scenario_load(const char* parfile, af_scenario** out) {
  if (!parfile || !out) return AF_EINVAL;
  Par p;
  int rc = read_par(parfile, p);
  if (rc != AF_OK) return rc;
  int ncols = 0, nrows = 0;
  double xll = 0, yll = 0, cs = 0, nodata = 0;
  af_scenario* sc = new af_scenario();
  rc = read_dem(p.dem_file.c_str(), ncols, nrows, xll, yll, cs, nodata, sc->dem);
  if (rc != AF_OK) {
    delete sc;
    return rc;
  }
  std::vector<PointBC> pts;
  bool free_side[4] = {false, false, false, false};
  rc = read_bci(p.bci_file.c_str(), xll, yll, ncols, nrows, cs, pts, free_side);
  if (rc == AF_OK) rc = read_bdy(p.bdy_file.c_str(), pts);
  if (rc != AF_OK) {
    delete sc;
    return rc;
  }
  if (!p.rain_file.empty()) read_rain(p.rain_file.c_str(), sc->rain_times, sc->rain_rates);

  af_case_desc& c = sc->c;
  c.nx = ncols;
  c.ny = nrows;
  c.dx = cs;
  c.nodata = nodata;
  c.fpn = p.fpn;
  c.depth_thresh = p.depth_thresh;
  c.cfl = p.cfl;
  c.init_tstep = p.init_tstep;
  c.g = 9.81;         // src/main.cpp:123
  c.max_hflow = 10.0; // src/main.cpp:118
  c.theta = 1.0;      // src/main.cpp:124
  c.west_free = free_side[0];
  c.east_free = free_side[1];
  c.north_free = free_side[2];
  c.south_free = free_side[3];
  c.mass_int = p.mass_int;
  sc->par[0] = p.sim_time;
  sc->par[1] = p.save_int;
  sc->par[2] = p.mass_int;
  sc->geo[0] = xll;
  sc->geo[1] = yll;
  sc->geo[2] = cs;
  sc->out_dir = p.output_dir;
  sc->save_int = p.save_int;
  sc->stage_int = p.stage_int;
  sc->voutput = p.voutput;
  sc->async_output = p.async_output;
  sc->output_format = p.output_format;
  if (!p.stage_file.empty())
    read_stage_file(p.stage_file.c_str(), xll, yll, ncols, nrows, cs, *sc);
  for (const std::string& n : sc->stage_names) sc->stage_name_ptrs.push_back(n.c_str());

  sc->flow_off.push_back(0);
  sc->other_off.push_back(0);
  for (const auto& pb : pts) {  // src/main.cpp:77-85 and :185-190
    if (pb.type == AF_BC_QVAR || pb.type == AF_BC_QFIX) {
      sc->flow_idx.push_back(pb.idx);
      sc->flow_type.push_back(pb.type);
      sc->flow_value.push_back(pb.value);
      sc->flow_times.insert(sc->flow_times.end(), pb.times.begin(), pb.times.end());
      sc->flow_vals.insert(sc->flow_vals.end(), pb.values.begin(), pb.values.end());
      sc->flow_off.push_back(sc->flow_off.back() + (int)pb.times.size());
    } else {
      sc->other_idx.push_back(pb.idx);
      sc->other_type.push_back(pb.type == AF_BC_FREE ? 1 : pb.type == AF_BC_HFIX ? 2 : 3);
      sc->other_value.push_back(pb.value);
      sc->other_times.insert(sc->other_times.end(), pb.times.begin(), pb.times.end());
      sc->other_vals.insert(sc->other_vals.end(), pb.values.begin(), pb.values.end());
      sc->other_off.push_back(sc->other_off.back() + (int)pb.times.size());
    }
  }
  *out = sc;
  return AF_OK;
}

void af_scenario_free(af_scenario* sc) { delete sc; }

int af_scenario_output(const af_scenario* sc, af_output_desc* o) {
  if (!sc || !o) return AF_EINVAL;
  *o = af_output_desc{};
  o->out_dir = sc->out_dir.c_str();
  o->save_int = sc->save_int;
  o->voutput = sc->voutput;
  o->async_style = sc->async_output;
  o->xll = sc->geo[0];
  o->yll = sc->geo[1];
  o->n_stage = (int)sc->stage_idx.size();
  o->stage_idx = sc->stage_idx.empty() ? nullptr : sc->stage_idx.data();
  o->stage_names = sc->stage_name_ptrs.empty() ? nullptr : sc->stage_name_ptrs.data();
  o->stage_int = sc->stage_int;
  o->output_format = sc->output_format;
  return AF_OK;
}

int af_scenario_get(const af_scenario* sc, af_case_desc* c, af_forcing_desc* f,
                    const double** dem, double* par, double* geo) {
  if (!sc) return AF_EINVAL;
  if (c) *c = sc->c;
  if (f) {
    f->n_flow = (int)sc->flow_idx.size();
    f->flow_idx = sc->flow_idx.data();
    f->flow_type = sc->flow_type.data();
    f->flow_value = sc->flow_value.data();
    f->flow_off = sc->flow_off.data();
    f->flow_times = sc->flow_times.data();
    f->flow_vals = sc->flow_vals.data();
    f->n_other = (int)sc->other_idx.size();
    f->other_idx = sc->other_idx.data();
    f->other_type = sc->other_type.data();
    f->other_value = sc->other_value.data();
    f->other_off = sc->other_off.data();
    f->other_times = sc->other_times.data();
    f->other_vals = sc->other_vals.data();
    f->n_rain = (int)sc->rain_times.size();
    f->rain_times = sc->rain_times.data();
    f->rain_rates = sc->rain_rates.data();
  }
  if (dem) *dem = sc->dem.data();
  if (par)
    for (int k = 0; k < 3; k++) par[k] = sc->par[k];
  if (geo)
    for (int k = 0; k < 3; k++) geo[k] = sc->geo[k];
  return AF_OK;
}

}  // extern "C"
