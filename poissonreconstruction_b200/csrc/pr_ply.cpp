// PLY input and output on the host: the on-disk formats on either side of the reconstruction.
//
// Reading mirrors ply::read_oriented_points (src/ply.rs:13-70): the header is scanned line by
// line until a line starting with "end_header"; "element vertex N" gives the count; a header
// line containing "nx" or "normal_x" marks normals (without one the file is rejected); every
// later line with at least six whitespace-separated tokens becomes a point from its first six
// tokens, each parsed as f64 with 0.0 in place of a token that does not parse, and shorter lines
// are skipped.  The data lines are parsed in parallel chunks and concatenated in file order.
// Extension: a "format binary_little_endian" file is read by property name (x y z nx ny nz,
// or normal_x normal_y normal_z), any scalar property types.
//
// Writing mirrors ply::write_mesh (src/ply.rs:73-107) byte for byte in ASCII mode: the same
// header, "x y z" per vertex with Rust's `{}` formatting of f64 (shortest round-trip digits,
// positional notation, never an exponent) and "3 a b c" per triangle.  Extension: a
// binary_little_endian writer (double vertices, uint32 or uint64 indices).
#include <errno.h>
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cctype>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/poisson_recon.h"

namespace pr {
void set_last_error(const std::string& msg);
}

namespace {

unsigned worker_count(size_t work_items, size_t per_worker) {
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t want = work_items / std::max<size_t>(per_worker, 1) + 1;
  return (unsigned)std::max<size_t>(1, std::min<size_t>({(size_t)hw, want, 32}));
}

// Rust's io::Error display: "<strerror> (os error N)"
std::string os_error(int e) { return std::string(std::strerror(e)) + " (os error " + std::to_string(e) + ")"; }

bool read_file(const char* path, std::string& data, std::string& err) {
  const int fd = ::open(path, O_RDONLY);
  if (fd < 0) {
    err = std::string("Cannot open ") + path + ": " + os_error(errno);
    return false;
  }
  struct stat st;
  if (::fstat(fd, &st) != 0) {
    err = std::string("Cannot open ") + path + ": " + os_error(errno);
    ::close(fd);
    return false;
  }
  data.resize((size_t)st.st_size);
  size_t got = 0;
  while (got < data.size()) {
    const ssize_t r = ::read(fd, &data[got], data.size() - got);
    if (r < 0) {
      if (errno == EINTR) continue;
      err = "Read error: " + os_error(errno);
      ::close(fd);
      return false;
    }
    if (r == 0) break;
    got += (size_t)r;
  }
  data.resize(got);
  ::close(fd);
  return true;
}

inline bool is_ws(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f'; }

// Rust `str::parse::<f64>()`: optional sign, then decimal digits with an optional fraction and
// exponent, or inf / infinity / nan (any case).  Anything else (hex, trailing text) is an
// error, which the reader turns into 0.0.
double parse_f64_or_zero(const char* b, const char* e) {
  const char* p = b;
  bool neg = false;
  if (p < e && (*p == '+' || *p == '-')) {
    neg = *p == '-';
    ++p;
  }
  if (p == e) return 0.0;
  if (*p == 'i' || *p == 'I' || *p == 'n' || *p == 'N') {
    std::string w(p, e);
    for (char& c : w) c = (char)std::tolower((unsigned char)c);
    if (w == "inf" || w == "infinity") return neg ? -HUGE_VAL : HUGE_VAL;
    if (w == "nan") return neg ? -NAN : NAN;
    return 0.0;
  }
  // decimal grammar check: digits* ['.' digits*] with at least one digit, then [eE [+-] digits+]
  const char* q = p;
  size_t nd = 0;
  while (q < e && *q >= '0' && *q <= '9') ++q, ++nd;
  if (q < e && *q == '.') {
    ++q;
    while (q < e && *q >= '0' && *q <= '9') ++q, ++nd;
  }
  if (nd == 0) return 0.0;
  if (q < e && (*q == 'e' || *q == 'E')) {
    ++q;
    if (q < e && (*q == '+' || *q == '-')) ++q;
    size_t ne = 0;
    while (q < e && *q >= '0' && *q <= '9') ++q, ++ne;
    if (ne == 0) return 0.0;
  }
  if (q != e) return 0.0;
  double v = 0.0;
  const auto r = std::from_chars(p, e, v, std::chars_format::general);
  if (r.ec == std::errc::result_out_of_range) {  // Rust rounds to inf / 0 instead of failing
    v = std::strtod(std::string(p, e).c_str(), nullptr);
  } else if (r.ec != std::errc() || r.ptr != e) {
    return 0.0;
  }
  return neg ? -v : v;
}

// Points of the data lines in [b, e) (whole lines), appended to out.
void parse_ascii_lines(const char* b, const char* e, std::vector<double>& out) {
  const char* p = b;
  while (p < e) {
    const char* eol = static_cast<const char*>(std::memchr(p, '\n', (size_t)(e - p)));
    const char* le = eol ? eol : e;
    const char* tb[6];
    const char* te[6];
    int nt = 0;
    const char* q = p;
    while (q < le && nt < 6) {
      while (q < le && is_ws(*q)) ++q;
      if (q >= le) break;
      const char* s = q;
      while (q < le && !is_ws(*q)) ++q;
      tb[nt] = s;
      te[nt] = q;
      ++nt;
    }
    if (nt == 6)
      for (int k = 0; k < 6; ++k) out.push_back(parse_f64_or_zero(tb[k], te[k]));
    p = eol ? eol + 1 : e;
  }
}

struct Prop {
  std::string name;
  int type = -1;  // size in bytes with sign/float flag, see read_scalar
  bool list = false;
};
struct Element {
  std::string name;
  uint64_t count = 0;
  std::vector<Prop> props;
};

int type_code(const std::string& t) {
  // 1 int8, 2 uint8, 3 int16, 4 uint16, 5 int32, 6 uint32, 7 float32, 8 float64
  if (t == "char" || t == "int8") return 1;
  if (t == "uchar" || t == "uint8") return 2;
  if (t == "short" || t == "int16") return 3;
  if (t == "ushort" || t == "uint16") return 4;
  if (t == "int" || t == "int32") return 5;
  if (t == "uint" || t == "uint32") return 6;
  if (t == "float" || t == "float32") return 7;
  if (t == "double" || t == "float64") return 8;
  return -1;
}
int type_size(int c) { return c <= 2 ? 1 : (c <= 4 ? 2 : (c <= 7 ? 4 : 8)); }
double read_scalar(const unsigned char* p, int c) {
  switch (c) {
    case 1: { int8_t v; std::memcpy(&v, p, 1); return v; }
    case 2: { uint8_t v; std::memcpy(&v, p, 1); return v; }
    case 3: { int16_t v; std::memcpy(&v, p, 2); return v; }
    case 4: { uint16_t v; std::memcpy(&v, p, 2); return v; }
    case 5: { int32_t v; std::memcpy(&v, p, 4); return v; }
    case 6: { uint32_t v; std::memcpy(&v, p, 4); return v; }
    case 7: { float v; std::memcpy(&v, p, 4); return v; }
    default: { double v; std::memcpy(&v, p, 8); return v; }
  }
}

std::vector<std::string> split_ws(const std::string& s) {
  std::vector<std::string> out;
  size_t i = 0;
  while (i < s.size()) {
    while (i < s.size() && is_ws(s[i])) ++i;
    size_t j = i;
    while (j < s.size() && !is_ws(s[j])) ++j;
    if (j > i) out.push_back(s.substr(i, j - i));
    i = j;
  }
  return out;
}

// Rust `usize::from_str`: optional '+', then decimal digits only
bool parse_usize(const std::string& s, uint64_t& v) {
  size_t i = (!s.empty() && s[0] == '+') ? 1 : 0;
  if (i >= s.size()) return false;
  uint64_t acc = 0;
  for (; i < s.size(); ++i) {
    if (s[i] < '0' || s[i] > '9') return false;
    const uint64_t d = (uint64_t)(s[i] - '0');
    if (acc > (UINT64_MAX - d) / 10) return false;
    acc = acc * 10 + d;
  }
  v = acc;
  return true;
}

int read_points(const char* path, std::vector<double>& pts, std::string& err) {
  std::string data;
  if (!read_file(path, data, err)) return PR_ERR_INVALID_ARGUMENT;
  size_t pos = 0;
  uint64_t num_vertices = 0;
  bool has_normals = false, binary = false, big_endian = false, end = false;
  std::vector<Element> elems;
  while (!end) {
    if (pos >= data.size()) {
      err = "Unexpected end of file";
      return PR_ERR_INVALID_ARGUMENT;
    }
    size_t eol = data.find('\n', pos);
    const size_t next = eol == std::string::npos ? data.size() : eol + 1;
    if (eol == std::string::npos) eol = data.size();
    std::string line = data.substr(pos, eol - pos);
    if (!line.empty() && line.back() == '\r') line.pop_back();
    pos = next;
    if (line.rfind("end_header", 0) == 0) {
      end = true;
    } else if (line.rfind("element vertex ", 0) == 0) {
      if (!parse_usize(line.substr(15), num_vertices)) {
        err = "Invalid vertex count";
        return PR_ERR_INVALID_ARGUMENT;
      }
    } else if (line.find("nx") != std::string::npos || line.find("normal_x") != std::string::npos) {
      has_normals = true;
    }
    // layout bookkeeping for the binary extension (the ASCII path ignores it)
    const std::vector<std::string> w = split_ws(line);
    if (w.size() >= 2 && w[0] == "format") {
      binary = w[1] == "binary_little_endian";
      big_endian = w[1] == "binary_big_endian";
    } else if (w.size() >= 3 && w[0] == "element") {
      Element el;
      el.name = w[1];
      parse_usize(w[2], el.count);
      elems.push_back(el);
    } else if (w.size() >= 3 && w[0] == "property" && !elems.empty()) {
      Prop pr;
      if (w[1] == "list" && w.size() >= 5) {
        pr.list = true;
        pr.name = w[4];
      } else {
        pr.type = type_code(w[1]);
        pr.name = w[2];
      }
      elems.back().props.push_back(pr);
    }
  }
  if (!has_normals) {
    err = "PLY file does not contain normal data (nx, ny, nz)";
    return PR_ERR_INVALID_ARGUMENT;
  }
  if (big_endian) {
    err = "binary_big_endian PLY is not supported";
    return PR_ERR_INVALID_ARGUMENT;
  }
  pts.clear();
  if (!binary) {
    // whole lines split into chunks, parsed in parallel, concatenated in order
    const char* b = data.data() + pos;
    const char* e = data.data() + data.size();
    const size_t bytes = (size_t)(e - b);
    const unsigned nt = worker_count(bytes, size_t(4) << 20);
    std::vector<const char*> cut(nt + 1, e);
    cut[0] = b;
    for (unsigned k = 1; k < nt; ++k) {
      const char* c = b + bytes * k / nt;
      if (c < cut[k - 1]) c = cut[k - 1];
      const char* nl = static_cast<const char*>(std::memchr(c, '\n', (size_t)(e - c)));
      cut[k] = nl ? nl + 1 : e;
    }
    std::vector<std::vector<double>> part(nt);
    std::vector<std::thread> th;
    for (unsigned k = 0; k < nt; ++k) {
      part[k].reserve(6 * (num_vertices / nt + 16));
      th.emplace_back([&, k] { parse_ascii_lines(cut[k], cut[k + 1], part[k]); });
    }
    for (auto& t : th) t.join();
    size_t total = 0;
    for (auto& v : part) total += v.size();
    pts.reserve(total);
    for (auto& v : part) pts.insert(pts.end(), v.begin(), v.end());
    return PR_OK;
  }
  // binary_little_endian: skip the elements before "vertex", then read its records by name
  size_t off = pos;
  const unsigned char* raw = reinterpret_cast<const unsigned char*>(data.data());
  for (const Element& el : elems) {
    size_t stride = 0;
    for (const Prop& p : el.props) {
      if (p.list || p.type < 0) {
        err = "binary PLY: element '" + el.name + "' has a list or unknown property before the vertices";
        return PR_ERR_INVALID_ARGUMENT;
      }
      stride += (size_t)type_size(p.type);
    }
    if (el.name != "vertex") {
      off += stride * el.count;
      continue;
    }
    int col[6] = {-1, -1, -1, -1, -1, -1};
    size_t at[6] = {0, 0, 0, 0, 0, 0};
    static const char* names[6][2] = {{"x", "x"}, {"y", "y"}, {"z", "z"},
                                      {"nx", "normal_x"}, {"ny", "normal_y"}, {"nz", "normal_z"}};
    size_t o = 0;
    for (const Prop& p : el.props) {
      for (int k = 0; k < 6; ++k)
        if (p.name == names[k][0] || p.name == names[k][1]) {
          col[k] = p.type;
          at[k] = o;
        }
      o += (size_t)type_size(p.type);
    }
    for (int k = 0; k < 6; ++k)
      if (col[k] < 0) {
        err = std::string("binary PLY: vertex property '") + names[k][0] + "' is missing";
        return PR_ERR_INVALID_ARGUMENT;
      }
    if (off + stride * el.count > data.size()) {
      err = "Unexpected end of file";
      return PR_ERR_INVALID_ARGUMENT;
    }
    pts.resize(6 * el.count);
    const uint64_t n = el.count;
    const unsigned nt = worker_count((size_t)n, 1 << 18);
    std::vector<std::thread> th;
    for (unsigned w = 0; w < nt; ++w)
      th.emplace_back([&, w] {
        for (uint64_t i = n * w / nt; i < n * (w + 1) / nt; ++i)
          for (int k = 0; k < 6; ++k) pts[6 * i + k] = read_scalar(raw + off + stride * i + at[k], col[k]);
      });
    for (auto& t : th) t.join();
    return PR_OK;
  }
  err = "binary PLY: no vertex element";
  return PR_ERR_INVALID_ARGUMENT;
}

// Rust's `{}` for f64: the shortest digits that round-trip, written in positional notation
// (zeros pad the integer part instead of an exponent); NaN as "NaN", infinities as "inf".
inline char* put_f64(char* p, double v) {
  if (v != v) {
    std::memcpy(p, "NaN", 3);
    return p + 3;
  }
  if (std::isinf(v)) {
    if (v < 0) *p++ = '-';
    std::memcpy(p, "inf", 3);
    return p + 3;
  }
  char sci[40];
  char* se = std::to_chars(sci, sci + sizeof(sci) - 1, v, std::chars_format::scientific).ptr;
  *se = '\0';
  const char* q = sci;
  if (*q == '-') *p++ = *q++;
  char dig[24];
  int nd = 0;
  while (q < se && *q != 'e') {
    if (*q != '.') dig[nd++] = *q;
    ++q;
  }
  int ex = std::atoi(q + 1);  // d.ddd x 10^ex
  const int pos = ex + 1;     // digits before the decimal point
  if (pos <= 0) {
    *p++ = '0';
    *p++ = '.';
    for (int i = 0; i < -pos; ++i) *p++ = '0';
    for (int i = 0; i < nd; ++i) *p++ = dig[i];
  } else if (pos >= nd) {
    for (int i = 0; i < nd; ++i) *p++ = dig[i];
    for (int i = nd; i < pos; ++i) *p++ = '0';
  } else {
    for (int i = 0; i < pos; ++i) *p++ = dig[i];
    *p++ = '.';
    for (int i = pos; i < nd; ++i) *p++ = dig[i];
  }
  return p;
}
inline char* put_u64(char* p, uint64_t v) { return std::to_chars(p, p + 24, v).ptr; }

// Items [0, count) formatted by `fmt(dst, i) -> end` into chunks of 4096 (max_item bytes each at
// most), several chunks at a time in parallel, written in order.
template <typename F>
bool write_formatted(FILE* f, uint64_t count, size_t max_item, F fmt, std::string& err) {
  const unsigned nt = worker_count((size_t)count, 1 << 12);
  const uint64_t chunk = 1 << 12;
  const uint64_t nchunks = (count + chunk - 1) / chunk;
  for (uint64_t c0 = 0; c0 < nchunks; c0 += nt) {  // nt chunks at a time, written in order
    const uint64_t c1 = std::min<uint64_t>(nchunks, c0 + nt);
    std::vector<std::string> buf(c1 - c0);
    std::vector<std::thread> th;
    for (uint64_t c = c0; c < c1; ++c)
      th.emplace_back([&, c] {
        const uint64_t lo = c * chunk, hi = std::min<uint64_t>(count, lo + chunk);
        std::string& s = buf[c - c0];
        s.resize((hi - lo) * max_item);
        char* p = &s[0];
        for (uint64_t i = lo; i < hi; ++i) p = fmt(p, i);
        s.resize((size_t)(p - s.data()));
      });
    for (auto& t : th) t.join();
    for (const std::string& s : buf)
      if (std::fwrite(s.data(), 1, s.size(), f) != s.size()) {
        err = os_error(errno);
        return false;
      }
  }
  return true;
}

int write_mesh(const char* path, const pr_mesh* m, int format, std::string& err) {
  FILE* f = std::fopen(path, "wb");
  if (!f) {
    err = std::string("Cannot create ") + path + ": " + os_error(errno);
    return PR_ERR_INVALID_ARGUMENT;
  }
  std::vector<char> iobuf(size_t(8) << 20);
  std::setvbuf(f, iobuf.data(), _IOFBF, iobuf.size());
  const uint64_t nv = m->n_vertices, nf = m->n_triangles;
  bool ok = true;
  if (format == 0) {
    std::string h = "ply\nformat ascii 1.0\nelement vertex " + std::to_string(nv) +
                    "\nproperty float x\nproperty float y\nproperty float z\nelement face " + std::to_string(nf) +
                    "\nproperty list uchar int vertex_indices\nend_header\n";
    ok = std::fwrite(h.data(), 1, h.size(), f) == h.size();
    if (ok)
      ok = write_formatted(f, nv, 3 * 400 + 3, [&](char* p, uint64_t i) {
        const double* v = m->vertices + 3 * i;
        p = put_f64(p, v[0]);
        *p++ = ' ';
        p = put_f64(p, v[1]);
        *p++ = ' ';
        p = put_f64(p, v[2]);
        *p++ = '\n';
        return p;
      }, err);
    if (ok)
      ok = write_formatted(f, nf, 3 * 24 + 6, [&](char* p, uint64_t i) {
        const uint64_t* t = m->triangles + 3 * i;
        *p++ = '3';
        *p++ = ' ';
        p = put_u64(p, t[0]);
        *p++ = ' ';
        p = put_u64(p, t[1]);
        *p++ = ' ';
        p = put_u64(p, t[2]);
        *p++ = '\n';
        return p;
      }, err);
  } else {
    const bool wide = nv > 0xffffffffull;
    std::string h = "ply\nformat binary_little_endian 1.0\nelement vertex " + std::to_string(nv) +
                    "\nproperty double x\nproperty double y\nproperty double z\nelement face " + std::to_string(nf) +
                    (wide ? "\nproperty list uchar uint64 vertex_indices\n" : "\nproperty list uchar uint vertex_indices\n") +
                    "end_header\n";
    ok = std::fwrite(h.data(), 1, h.size(), f) == h.size();
    if (ok && nv) ok = std::fwrite(m->vertices, sizeof(double), 3 * nv, f) == 3 * nv;
    const size_t rec = 1 + (wide ? 24 : 12);
    for (uint64_t lo = 0; ok && lo < nf; lo += (1 << 20)) {
      const uint64_t hi = std::min<uint64_t>(nf, lo + (1 << 20));
      std::vector<unsigned char> b((size_t)(hi - lo) * rec);
      for (uint64_t i = lo; i < hi; ++i) {
        unsigned char* p = b.data() + (size_t)(i - lo) * rec;
        p[0] = 3;
        for (int k = 0; k < 3; ++k) {
          const uint64_t v = m->triangles[3 * i + k];
          if (wide) std::memcpy(p + 1 + 8 * k, &v, 8);
          else {
            const uint32_t v32 = (uint32_t)v;
            std::memcpy(p + 1 + 4 * k, &v32, 4);
          }
        }
      }
      ok = std::fwrite(b.data(), 1, b.size(), f) == b.size();
    }
    if (!ok && err.empty()) err = os_error(errno);
  }
  if (std::fclose(f) != 0 && ok) {
    ok = false;
    err = os_error(errno);
  }
  return ok ? PR_OK : PR_ERR_INVALID_ARGUMENT;
}

}  // namespace

extern "C" {

int pr_ply_read_points(const char* path, double** out_points6, uint64_t* out_n) {
  if (!path || !out_points6 || !out_n) {
    pr::set_last_error("pr_ply_read_points: NULL argument");
    return PR_ERR_INVALID_ARGUMENT;
  }
  *out_points6 = nullptr;
  *out_n = 0;
  try {
    std::vector<double> pts;
    std::string err;
    const int rc = read_points(path, pts, err);
    if (rc != PR_OK) {
      pr::set_last_error(err);
      return rc;
    }
    if (!pts.empty()) {
      double* p = static_cast<double*>(std::malloc(pts.size() * sizeof(double)));
      if (!p) {
        pr::set_last_error("host allocation failed");
        return PR_ERR_OUT_OF_MEMORY;
      }
      std::memcpy(p, pts.data(), pts.size() * sizeof(double));
      *out_points6 = p;
    }
    *out_n = pts.size() / 6;
    return PR_OK;
  } catch (const std::bad_alloc&) {
    pr::set_last_error("host allocation failed");
    return PR_ERR_OUT_OF_MEMORY;
  }
}

int pr_ply_write_mesh(const char* path, const pr_mesh* mesh, int format) {
  if (!path || !mesh || (mesh->n_vertices && !mesh->vertices) || (mesh->n_triangles && !mesh->triangles)) {
    pr::set_last_error("pr_ply_write_mesh: NULL argument");
    return PR_ERR_INVALID_ARGUMENT;
  }
  if (format != PR_PLY_ASCII && format != PR_PLY_BINARY) {
    pr::set_last_error("pr_ply_write_mesh: format must be PR_PLY_ASCII or PR_PLY_BINARY");
    return PR_ERR_INVALID_ARGUMENT;
  }
  try {
    std::string err;
    const int rc = write_mesh(path, mesh, format, err);
    if (rc != PR_OK) pr::set_last_error(err);
    return rc;
  } catch (const std::bad_alloc&) {
    pr::set_last_error("host allocation failed");
    return PR_ERR_OUT_OF_MEMORY;
  }
}

}  // extern "C"
