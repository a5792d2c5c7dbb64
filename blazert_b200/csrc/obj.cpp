// Wavefront OBJ mesh ingestion with the mesh the reference's examples build from the same file
// (examples/scene_mesh/main.cc:15-43 over the vendored tiny_obj_loader 0.9.14,
// examples/common/tiny_obj_loader.cc:911-1081, the LoadObj overload without materials):
//
//  * numbers are read by that loader's own parser (tiny_obj_loader.cc:130-231: integer digits
//    accumulated as mantissa * 10 + d, fraction digits added as d * 10^-k, the value assembled
//    as ldexp(mantissa * 5^e, e); a token it cannot parse reads as 0) and rounded to float;
//  * statements: "v" (three numbers), "vn", "vt" (counted for index resolution), "f" (index
//    triples i, i/j, i//k, i/j/k; positive indices are 1-based, negative ones relative to the
//    elements read so far, 0 reads as the first), "g" and "o" end the current shape; every
//    other statement, including usemtl and mtllib, is ignored;
//  * each shape numbers its vertices in order of first use by its triangles, one vertex per
//    distinct (position, texcoord, normal) index triple, and splits polygons into the fan
//    (f0, f[k-1], f[k]) (tiny_obj_loader.cc:296-333, :358-408);
//  * the example concatenates the shapes: vertices in shape order, face indices offset by the
//    vertices of the shapes before.
//
// A face index outside the positions read when its shape ends is an error here (the reference
// asserts, tiny_obj_loader.cc:312, which release builds skip).
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "scene.h"

namespace bzr {
namespace {

bool is_space(char c) { return c == ' ' || c == '\t'; }
bool is_digit(char c) { return c >= '0' && c <= '9'; }
bool line_end(char c) { return c == '\r' || c == '\n' || c == '\0'; }

// The loader's number grammar: [sign] digits ["." digits] [("e"|"E") [sign] digits]; false
// when the text does not start a number or an exponent has no digits.
//
// This function restates tryParseDouble of tiny_obj_loader 0.9.14
// (examples/common/tiny_obj_loader.cc:130-231 in the reference), closely, because a mesh read
// here must have the bits the reference's examples read.  That loader's notice:
//
//   Copyright 2012-2015, Syoyo Fujita.
//   Licensed under 2-clause BSD license.
//
//   Redistribution and use in source and binary forms, with or without modification, are
//   permitted provided that the following conditions are met:
//   1. Redistributions of source code must retain the above copyright notice, this list of
//      conditions and the following disclaimer.
//   2. Redistributions in binary form must reproduce the above copyright notice, this list of
//      conditions and the following disclaimer in the documentation and/or other materials
//      provided with the distribution.
//   THIS SOFTWARE IS PROVIDED BY THE COPYRIGHT HOLDERS AND CONTRIBUTORS "AS IS" AND ANY EXPRESS
//   OR IMPLIED WARRANTIES, INCLUDING, BUT NOT LIMITED TO, THE IMPLIED WARRANTIES OF
//   MERCHANTABILITY AND FITNESS FOR A PARTICULAR PURPOSE ARE DISCLAIMED. IN NO EVENT SHALL THE
//   COPYRIGHT HOLDER OR CONTRIBUTORS BE LIABLE FOR ANY DIRECT, INDIRECT, INCIDENTAL, SPECIAL,
//   EXEMPLARY, OR CONSEQUENTIAL DAMAGES (INCLUDING, BUT NOT LIMITED TO, PROCUREMENT OF
//   SUBSTITUTE GOODS OR SERVICES; LOSS OF USE, DATA, OR PROFITS; OR BUSINESS INTERRUPTION)
//   HOWEVER CAUSED AND ON ANY THEORY OF LIABILITY, WHETHER IN CONTRACT, STRICT LIABILITY, OR
//   TORT (INCLUDING NEGLIGENCE OR OTHERWISE) ARISING IN ANY WAY OUT OF THE USE OF THIS
//   SOFTWARE, EVEN IF ADVISED OF THE POSSIBILITY OF SUCH DAMAGE.
bool parse_number(const char *s, const char *end, double *out) {
  if (s >= end) return false;
  double mantissa = 0.0;
  int exponent = 0;
  char sign = '+', exp_sign = '+';
  const char *c = s;
  if (*c == '+' || *c == '-') {
    sign = *c;
    ++c;
  } else if (!is_digit(*c)) {
    return false;
  }
  int digits = 0;
  bool more = false;
  while ((more = (c != end)) && is_digit(*c)) {
    mantissa *= 10;
    mantissa += static_cast<int>(*c - '0');
    ++c;
    ++digits;
  }
  if (digits == 0) return false;
  if (more) {
    bool exponent_part = false;
    if (*c == '.') {
      ++c;
      int k = 1;
      while ((more = (c != end)) && is_digit(*c)) {
        mantissa += static_cast<int>(*c - '0') * std::pow(10.0, -k);
        ++k;
        ++c;
      }
      exponent_part = more;
    } else if (*c == 'e' || *c == 'E') {
      exponent_part = true;
    }
    if (exponent_part && (*c == 'e' || *c == 'E')) {
      ++c;
      if ((more = (c != end)) && (*c == '+' || *c == '-')) {
        exp_sign = *c;
        ++c;
      } else if (!is_digit(*c)) {
        return false;
      }
      int n = 0;
      while ((more = (c != end)) && is_digit(*c)) {
        exponent *= 10;
        exponent += static_cast<int>(*c - '0');
        ++c;
        ++n;
      }
      exponent *= (exp_sign == '+' ? 1 : -1);
      if (n == 0) return false;
    }
  }
  *out = (sign == '+' ? 1 : -1) * std::ldexp(mantissa * std::pow(5.0, exponent), exponent);
  return true;
}

// One coordinate: skips blanks, reads to the next blank or '\r', as float.
float read_coordinate(const char *&t) {
  t += std::strspn(t, " \t");
  const char *end = t + std::strcspn(t, " \t\r");
  double v = 0.0;
  parse_number(t, end, &v);
  t = end;
  return static_cast<float>(v);
}

// 1-based, negative relative to n, 0 as the first element
int resolve(int idx, int n) { return idx > 0 ? idx - 1 : (idx == 0 ? 0 : n + idx); }

// atoi as the loader reads indices (leading blanks, sign, digits), with values outside int
// clamped instead of atoi's undefined result; the same value for every index that fits.
int read_int(const char *t) {
  const long v = std::strtol(t, nullptr, 10);
  return v > INT_MAX ? INT_MAX : (v < INT_MIN ? INT_MIN : static_cast<int>(v));
}

struct Corner {
  int v = -1, vt = -1, vn = -1;
  bool operator<(const Corner &o) const {
    return std::tie(v, vn, vt) < std::tie(o.v, o.vn, o.vt);
  }
};

Corner read_corner(const char *&t, int nv, int nvn, int nvt) {
  Corner c;
  c.v = resolve(read_int(t), nv);
  t += std::strcspn(t, "/ \t\r");
  if (t[0] != '/') return c;
  ++t;
  if (t[0] == '/') {  // i//k
    ++t;
    c.vn = resolve(read_int(t), nvn);
    t += std::strcspn(t, "/ \t\r");
    return c;
  }
  c.vt = resolve(read_int(t), nvt);  // i/j or i/j/k
  t += std::strcspn(t, "/ \t\r");
  if (t[0] != '/') return c;
  ++t;
  c.vn = resolve(read_int(t), nvn);
  t += std::strcspn(t, "/ \t\r");
  return c;
}

struct ObjBuilder {
  std::vector<float> pos;                 // every "v" so far
  std::vector<std::vector<Corner>> faces;  // faces of the current shape
  std::vector<double> out_v;
  std::vector<uint32_t> out_f;
  std::string error;

  // tiny_obj_loader.cc:358-408 for one shape, then the example's concatenation
  bool end_shape() {
    if (faces.empty()) return true;
    std::map<Corner, uint32_t> index;
    const uint64_t base = out_v.size() / 3;
    uint64_t next = 0;
    auto vertex = [&](const Corner &c, uint32_t *id) {
      const auto it = index.find(c);
      if (it != index.end()) {
        *id = it->second;
        return true;
      }
      if (c.v < 0 || static_cast<uint64_t>(c.v) >= pos.size() / 3) return false;
      for (int a = 0; a < 3; ++a) out_v.push_back(static_cast<double>(pos[3 * size_t(c.v) + a]));
      *id = static_cast<uint32_t>(next++);
      index.emplace(c, *id);
      return true;
    };
    for (const std::vector<Corner> &f : faces) {
      for (size_t k = 2; k < f.size(); ++k) {
        uint32_t t[3];
        if (!vertex(f[0], &t[0]) || !vertex(f[k - 1], &t[1]) || !vertex(f[k], &t[2])) {
          error = "face index outside the vertices";
          return false;
        }
        for (uint32_t x : t) {
          if (base + x > 0xFFFFFFFFull) {
            error = "too many vertices";
            return false;
          }
          out_f.push_back(static_cast<uint32_t>(base + x));
        }
      }
    }
    faces.clear();
    return true;
  }
};

}  // namespace

std::string load_obj(const std::string &path, std::vector<double> *vertices,
                     std::vector<uint32_t> *faces) {
  std::ifstream in(path, std::ios::binary);
  if (!in) return "cannot open " + path;
  ObjBuilder b;
  size_t nvn = 0, nvt = 0;
  std::string line;
  size_t lineno = 0;
  while (std::getline(in, line)) {
    ++lineno;
    if (!line.empty() && line.back() == '\r') line.pop_back();
    const char *t = line.c_str();
    t += std::strspn(t, " \t");
    if (t[0] == '\0' || t[0] == '#') continue;
    if (t[0] == 'v' && is_space(t[1])) {
      t += 2;
      for (int a = 0; a < 3; ++a) b.pos.push_back(read_coordinate(t));
    } else if (t[0] == 'v' && t[1] == 'n' && is_space(t[2])) {
      ++nvn;
    } else if (t[0] == 'v' && t[1] == 't' && is_space(t[2])) {
      ++nvt;
    } else if (t[0] == 'f' && is_space(t[1])) {
      t += 2;
      t += std::strspn(t, " \t");
      std::vector<Corner> f;
      while (!line_end(t[0])) {
        f.push_back(read_corner(t, static_cast<int>(b.pos.size() / 3), static_cast<int>(nvn),
                                static_cast<int>(nvt)));
        t += std::strspn(t, " \t\r");
      }
      b.faces.push_back(std::move(f));
    } else if ((t[0] == 'g' || t[0] == 'o') && is_space(t[1])) {
      if (!b.end_shape()) return b.error + " (shape ending at line " + std::to_string(lineno) + ")";
    }
  }
  if (!b.end_shape()) return b.error + " (last shape)";
  *vertices = std::move(b.out_v);
  *faces = std::move(b.out_f);
  return "";
}

}  // namespace bzr
