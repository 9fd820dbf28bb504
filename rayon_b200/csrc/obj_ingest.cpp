// Wavefront OBJ ingest straight into a HostScene: the semantics of the
// reference's OBJLoader::loadOBJ (src/rayon/scenes/obj_loader.hpp:34-140),
// restated with a hand-written tokenizer over the whole file in memory
// instead of one istringstream per line.
//
// Rules kept from the reference:
//  * "v x y z": position = (x, y, z) * scale + position, component by
//    component in FP64; a "v" line that does not yield three numbers is
//    skipped. "vn x y z": normal, unscaled. Other records (vt, mtllib, usemtl,
//    s, g, o, comments) are skipped.
//  * Numbers are read as the reference's stream extraction reads them: an
//    optional sign, digits, at most one decimal point, an optional exponent
//    marker with optional sign and digits; the characters so accumulated
//    must form a whole number (so "1e" fails, and "1.2.3" reads 1.2 and then
//    .3 as the next number).
//  * "f" tokens "v", "v/vt", "v/vt/vn" or "v//vn"; each index is read like
//    std::stoi (sign and leading digits; no digits is an error). Index k > 0
//    means k - 1, k < 0 counts back from the current number of positions
//    (normals), and 0 stays 0. A face of n >= 3 corners becomes the fan
//    (0, i, i + 1); a triangle with an index outside the positions read so
//    far is skipped; it takes vertex normals only when there are normals and
//    all three of its normal indices are valid.
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "host_scene.hpp"

namespace rb {
namespace {

inline bool is_space(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r'; }
inline bool is_digit(char c) { return c >= '0' && c <= '9'; }

// Reads one floating-point number at p (after leading white space) as the
// stream extraction does; returns false when it fails.
bool read_double(const char *&p, const char *end, double &out) {
  while (p < end && is_space(*p)) ++p;
  const char *s = p;
  std::string acc;
  if (p < end && (*p == '+' || *p == '-')) acc.push_back(*p++);
  bool digits = false, point = false;
  while (p < end) {
    if (is_digit(*p)) {
      acc.push_back(*p++);
      digits = true;
    } else if (*p == '.' && !point) {
      acc.push_back(*p++);
      point = true;
    } else {
      break;
    }
  }
  if (digits && p < end && (*p == 'e' || *p == 'E')) {
    acc.push_back(*p++);
    if (p < end && (*p == '+' || *p == '-')) acc.push_back(*p++);
    while (p < end && is_digit(*p)) acc.push_back(*p++);
  }
  if (acc.empty() || !digits) {
    p = s;
    return false;
  }
  char *stop = nullptr;
  out = std::strtod(acc.c_str(), &stop);
  return stop == acc.c_str() + acc.size();
}

// std::stoi of a face-index part: sign and leading digits; false when there
// are none (the reference throws there).
bool read_index(const char *s, const char *e, long long &out) {
  const char *p = s;
  bool neg = false;
  if (p < e && (*p == '+' || *p == '-')) neg = *p++ == '-';
  if (p >= e || !is_digit(*p)) return false;
  long long v = 0;
  while (p < e && is_digit(*p)) {
    v = v * 10 + (*p++ - '0');
    if (v > 2147483647ll + (neg ? 1 : 0)) return false;  // out of int range
  }
  out = neg ? -v : v;
  return true;
}

}  // namespace

int64_t load_obj(HostScene &hs, const char *path, int mat, const V3 &pos, const V3 &scale, std::string &err) {
  std::FILE *f = std::fopen(path, "rb");
  if (!f) {
    err = std::string("cannot open ") + path;
    return -1;
  }
  std::vector<char> buf;
  if (std::fseek(f, 0, SEEK_END) == 0) {
    const long n = std::ftell(f);
    if (n > 0) {
      buf.resize((size_t)n);
      std::fseek(f, 0, SEEK_SET);
      if (std::fread(buf.data(), 1, buf.size(), f) != buf.size()) buf.clear();
    }
  }
  std::fclose(f);
  // room for the triangles of the face lines (one per "f" line at least)
  {
    size_t faces = 0;
    for (const char *c = buf.data(), *e = buf.data() + buf.size(); c < e; ++c)
      if ((c == buf.data() || c[-1] == '\n') && *c == 'f') ++faces;
    hs.geoms.reserve(hs.geoms.size() + faces);
  }
  std::vector<V3> vs, ns;
  struct Corner { long long v, n; };
  std::vector<Corner> face;
  int64_t tris = 0;
  const char *p = buf.data(), *end = buf.data() + buf.size();
  while (p < end) {
    const char *le = static_cast<const char *>(std::memchr(p, '\n', (size_t)(end - p)));
    if (!le) le = end;
    const char *q = p;
    p = le + 1;
    if (q == le || *q == '#') continue;  // empty line or comment in column 0
    while (q < le && is_space(*q)) ++q;
    const char *t = q;
    while (q < le && !is_space(*q)) ++q;
    const size_t tl = (size_t)(q - t);
    if (tl == 1 && t[0] == 'v') {
      double x, y, z;
      if (read_double(q, le, x) && read_double(q, le, y) && read_double(q, le, z))
        vs.emplace_back(x * scale.x + pos.x, y * scale.y + pos.y, z * scale.z + pos.z);
    } else if (tl == 2 && t[0] == 'v' && t[1] == 'n') {
      double x, y, z;
      if (read_double(q, le, x) && read_double(q, le, y) && read_double(q, le, z)) ns.emplace_back(x, y, z);
    } else if (tl == 1 && t[0] == 'f') {
      face.clear();
      while (true) {
        while (q < le && is_space(*q)) ++q;
        if (q >= le) break;
        const char *a = q;
        while (q < le && !is_space(*q)) ++q;
        // up to three '/'-separated parts: position, texture, normal
        const char *part[3] = {a, nullptr, nullptr}, *pend[3] = {q, nullptr, nullptr};
        int np = 1;
        for (const char *c = a; c < q && np < 3; ++c)
          if (*c == '/') {
            pend[np - 1] = c;
            part[np] = c + 1;
            pend[np] = q;
            ++np;
          }
        if (np == 3) {  // a fourth part, if any, is ignored
          const char *c = static_cast<const char *>(std::memchr(part[2], '/', (size_t)(pend[2] - part[2])));
          if (c) pend[2] = c;
        }
        long long vi = 0, ti = 0, ni = 0;
        if (pend[0] > part[0] && !read_index(part[0], pend[0], vi)) {
          err = "malformed face index";
          return -1;
        }
        if (np > 1 && pend[1] > part[1] && !read_index(part[1], pend[1], ti)) {
          err = "malformed face index";
          return -1;
        }
        if (np > 2 && pend[2] > part[2] && !read_index(part[2], pend[2], ni)) {
          err = "malformed face index";
          return -1;
        }
        if (vi > 0) vi -= 1;
        else if (vi < 0) vi = (long long)vs.size() + vi;
        if (ni > 0) ni -= 1;
        else if (ni < 0) ni = (long long)ns.size() + ni;
        face.push_back({vi, ni});
      }
      const long long nv = (long long)vs.size(), nn = (long long)ns.size();
      for (size_t i = 1; i + 1 < face.size(); ++i) {
        const Corner &c0 = face[0], &c1 = face[i], &c2 = face[i + 1];
        if (c0.v < 0 || c0.v >= nv || c1.v < 0 || c1.v >= nv || c2.v < 0 || c2.v >= nv) continue;
        const bool with_n = nn > 0 && c0.n >= 0 && c0.n < nn && c1.n >= 0 && c1.n < nn && c2.n >= 0 && c2.n < nn;
        if (with_n) hs.add_triangle_n(vs[c0.v], vs[c1.v], vs[c2.v], ns[c0.n], ns[c1.n], ns[c2.n], mat);
        else hs.add_triangle(vs[c0.v], vs[c1.v], vs[c2.v], mat);
        ++tris;
      }
    }
  }
  return tris;
}

}  // namespace rb
