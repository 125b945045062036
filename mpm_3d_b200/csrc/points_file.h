// Host-side reader of DefaultPoints .points files (the body point files the
// reference's configs name), parsed on several threads.
//
// The format and its parsing follow DefaultPoints::readFromFile
// (default_points.cpp:104-193): the first line holds the point count
// (std::stoi), then one line per point with the columns
// m, v, x[0..dim), x_t[0..dim), active, separated by single spaces. A line
// is split at every ' ' as Parser::splitString does (parser.hpp:24-35: empty
// pieces between or before spaces count, a trailing space adds none), each
// piece is converted like std::stod (strtod after optional leading
// whitespace, trailing characters ignored, no digits or an out-of-range
// value is an error) and active is the converted value truncated to an
// integer. Where the reference stops reading at a malformed line and keeps
// zeros for the rest, the reader reports the line instead.
#pragma once

#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace mpmb200 {

struct PointsFileResult {
  int ok = 0;
  int64_t bad_line = 0;  // 1-based line that failed (0: none, or the file itself)
  std::string error;
};

// Whole file into memory.
inline bool read_file(const char* path, std::vector<char>& buf) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  std::vector<char> out;
  char chunk[1 << 16];
  size_t got;
  while ((got = std::fread(chunk, 1, sizeof chunk, f)) > 0) out.insert(out.end(), chunk, chunk + got);
  std::fclose(f);
  out.push_back('\0');
  buf.swap(out);
  return true;
}

// std::stod on [b, e): leading whitespace skipped, trailing text ignored.
inline bool parse_double(const char* b, const char* e, double* out) {
  char tmp[128];
  const size_t len = (size_t)(e - b);
  std::string big;
  const char* s;
  if (len < sizeof tmp) {
    std::memcpy(tmp, b, len);
    tmp[len] = '\0';
    s = tmp;
  } else {
    big.assign(b, e);
    s = big.c_str();
  }
  char* end = nullptr;
  errno = 0;
  const double v = std::strtod(s, &end);
  if (end == s || errno == ERANGE) return false;
  *out = v;
  return true;
}

// std::stoi on the count line.
inline bool parse_count(const char* b, const char* e, int64_t* out) {
  std::string s(b, e);
  char* end = nullptr;
  errno = 0;
  const long long v = std::strtoll(s.c_str(), &end, 10);
  if (end == s.c_str() || errno == ERANGE || v < 0 || v > INT32_MAX) return false;
  *out = (int64_t)v;
  return true;
}

// Line starts of the first count + 1 lines (a line ends at '\n' or at the
// end of the text).
inline void line_starts(const std::vector<char>& buf, int64_t want, std::vector<size_t>& starts) {
  const size_t size = buf.size() - 1;  // without the terminating '\0'
  starts.clear();
  starts.push_back(0);
  for (size_t i = 0; i < size && (int64_t)starts.size() < want + 1; i++)
    if (buf[i] == '\n' && i + 1 <= size) starts.push_back(i + 1);
}

// Parses point lines [first, last) of the text; false at the first bad one.
inline bool parse_points(const std::vector<char>& buf, const std::vector<size_t>& starts, int dim, int64_t first,
                         int64_t last, double* m, double* v, double* x, double* x_t, int32_t* active,
                         int64_t* bad) {
  const size_t size = buf.size() - 1;
  // DefaultPoints::readFromFile (default_points.cpp:152-175) takes lines of
  // 2 + 2 job->DIM + 1 or of 2 + 2 GRID_DIM + 1 columns. For the job types
  // this path runs, JOB_2D and JOB_3D, job->DIM equals the grid's dimension
  // (Job::assignJobType, job.hpp:58-70), so both widths are 3 + 2 dim; the
  // 2D out-of-plane and axisymmetric types (job->DIM 3 over a 2D grid) are
  // refused by the solver plugin.
  const int cols = 3 + 2 * dim;
  const char* text = buf.data();
  std::vector<std::pair<const char*, const char*>> tok;
  for (int64_t i = first; i < last; i++) {
    const size_t li = (size_t)i + 1;  // line 0 is the count
    if (li >= starts.size()) {
      *bad = i + 2;
      return false;
    }
    const char* b = text + starts[li];
    const char* e = text + (li + 1 < starts.size() ? starts[li + 1] - 1 : size);
    const char* nl = static_cast<const char*>(std::memchr(b, '\n', (size_t)(e - b)));
    if (nl) e = nl;
    // Parser::splitString: pieces between ' '; the piece after a final ' ' is not one
    tok.clear();
    const char* p = b;
    while (p < e) {
      const char* q = static_cast<const char*>(std::memchr(p, ' ', (size_t)(e - p)));
      if (!q) {
        tok.emplace_back(p, e);
        break;
      }
      tok.emplace_back(p, q);
      p = q + 1;
    }
    double val[9];
    bool good = (int)tok.size() == cols;
    for (int c = 0; good && c < cols; c++) good = parse_double(tok[(size_t)c].first, tok[(size_t)c].second, &val[c]);
    if (!good) {
      *bad = i + 2;
      return false;
    }
    m[i] = val[0];
    v[i] = val[1];
    for (int d = 0; d < 3; d++) {
      x[3 * i + d] = d < dim ? val[2 + d] : 0.0;
      x_t[3 * i + d] = d < dim ? val[2 + dim + d] : 0.0;
    }
    active[i] = (int32_t)val[2 + 2 * dim];
  }
  return true;
}

inline PointsFileResult points_file_count(const char* path, int64_t* n) {
  PointsFileResult r;
  std::vector<char> buf;
  if (!read_file(path, buf)) {
    r.error = std::string("cannot open ") + path;
    return r;
  }
  const char* nl = static_cast<const char*>(std::memchr(buf.data(), '\n', buf.size() - 1));
  const char* e = nl ? nl : buf.data() + buf.size() - 1;
  if (!parse_count(buf.data(), e, n)) {
    r.bad_line = 1;
    r.error = "no point count on the first line";
    return r;
  }
  r.ok = 1;
  return r;
}

// Reads n points (the count the file's first line gives) on up to `threads`
// threads (0: the hardware's count).
inline PointsFileResult points_file_read(const char* path, int dim, int64_t n, double* m, double* v, double* x,
                                         double* x_t, int32_t* active, int threads) {
  PointsFileResult r;
  std::vector<char> buf;
  if (!read_file(path, buf)) {
    r.error = std::string("cannot open ") + path;
    return r;
  }
  std::vector<size_t> starts;
  line_starts(buf, n, starts);
  int64_t count = 0;
  const size_t first_end = starts.size() > 1 ? starts[1] - 1 : buf.size() - 1;
  if (!parse_count(buf.data(), buf.data() + first_end, &count)) {
    r.bad_line = 1;
    r.error = "no point count on the first line";
    return r;
  }
  if (count != n) {
    r.bad_line = 1;
    r.error = "the file's point count differs from n";
    return r;
  }
  int nt = threads > 0 ? threads : (int)std::thread::hardware_concurrency();
  if (nt < 1) nt = 1;
  if ((int64_t)nt > n / 4096 + 1) nt = (int)(n / 4096 + 1);
  std::vector<int64_t> bad((size_t)nt, 0);
  std::vector<char> good((size_t)nt, 1);
  std::vector<std::thread> pool;
  for (int t = 0; t < nt; t++) {
    const int64_t lo = n * t / nt, hi = n * (t + 1) / nt;
    auto work = [&, t, lo, hi] {
      good[(size_t)t] = parse_points(buf, starts, dim, lo, hi, m, v, x, x_t, active, &bad[(size_t)t]) ? 1 : 0;
    };
    if (t + 1 == nt)
      work();
    else
      pool.emplace_back(work);
  }
  for (auto& th : pool) th.join();
  for (int t = 0; t < nt; t++)
    if (!good[(size_t)t]) {
      r.bad_line = bad[(size_t)t];
      r.error = "unable to read line " + std::to_string(r.bad_line);
      return r;
    }
  r.ok = 1;
  return r;
}

}  // namespace mpmb200
