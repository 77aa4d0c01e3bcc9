// Mesh files: Mesh::loadFile (Src/mesh.cpp:612-617) with its Wavefront OBJ
// reader (Mesh::loadWavefrontObj, :235-456) and its PLY reader
// (Mesh::loadPly, :515-601) on top of tinyply 2.0's header and data parsing
// (3rdParty/tinyply/tinyply.cpp:186-603).  A file gives the mesh the
// reference's loader gives, array for array, whenever that mesh is valid
// (every face corner names an existing position); a file the reference
// rejects is rejected (FK_ERR_INVALID).
//
// OBJ.  Lines split at '\n'.  Statements: v x y z [w], vt u v [w],
// vn i j k, f with v, v/t, v//n or v/t/n corners (the first corner of the
// file fixes which indices every corner carries).  Numbers are read by
// strtod / strtol in the C locale, a range error rejects the file, and the
// rest of the line must be blank.  Every face corner becomes its own vertex,
// polygons become fans (first, previous, current), and faces with fewer than
// three corners add vertices but no triangles.  Indices are taken as written
// minus one (absent texcoord / normal indices become UINT32_MAX); relative
// (negative) and zero position indices therefore do not resolve, and such a
// file is rejected here where the reference returns a mesh that indexes past
// its positions.  A file that cannot be opened gives an empty mesh, as in the
// reference.
//
// PLY.  ASCII, binary little- and big-endian.  Header keywords as tinyply 2.0
// reads them (an unknown keyword ends the header).  Requested: vertex x y z,
// face vertex_indices, vertex s t, vertex nx ny nz or else face nx ny nz;
// a grouped request keeps the header's property order and the type of its
// last key, as tinyply's shared buffer does.  Faces are read as consecutive
// triples of the flattened index lists (the reference's loop; polygons with
// more corners are not split into fans); a face normal's index is 3 x the face
// (Src/mesh.cpp:582).  Where the reference's result is unusable this loader
// defines one:
//   * no s t or no normals: the reference dereferences a null buffer; here the
//     texcoords / normals stay empty and the vertices' indices are UINT32_MAX,
//     the values the reference's vertex loop assigns for that case;
//   * index lists of a type other than uint / ushort: the reference reads
//     every index as UINT32_MAX; here int, short, char and uchar lists are read
//     as their values;
//   * data shorter than the header announces, or an ASCII value that does not
//     parse: the reference goes on with zeros or uninitialised memory; here the
//     file is rejected.
#include <algorithm>
#include <clocale>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <locale.h>
#include <map>
#include <sstream>
#include <string>
#include <system_error>
#include <thread>
#include <vector>

#include "fk_internal.h"

namespace {

constexpr uint32_t kNone = 0xFFFFFFFFu;

bool read_file(const char* path, std::string& out) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  if (std::fseek(f, 0, SEEK_END) == 0) {  // one read of the whole file where its size is known
    const long size = std::ftell(f);
    std::rewind(f);
    if (size > 0) {
      out.resize((size_t)size);
      out.resize(std::fread(&out[0], 1, (size_t)size, f));  // then whatever a growing file added
    }
  }
  char chunk[1 << 16];
  size_t n;
  while ((n = std::fread(chunk, 1, sizeof(chunk), f)) > 0) out.append(chunk, n);
  std::fclose(f);
  return true;
}

bool ends_with(const char* s, const char* tail) {
  const size_t a = std::strlen(s), b = std::strlen(tail);
  return a >= b && std::memcmp(s + a - b, tail, b) == 0;
}

// isspace of the C locale (the reference's process never changes its locale).
inline bool blank(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r'; }

locale_t c_numeric() {
  static locale_t loc = newlocale(LC_ALL_MASK, "C", (locale_t)0);
  return loc;
}

// ------------------------------------------------------------------ OBJ
struct Corner {
  int p, t, n;
};

// strtod in the C locale narrowed to float; fails on a missing number (when
// required) and on a range error.
bool obj_float(const char*& s, float& v, bool required = true) {
  char* end;
  errno = 0;
  const locale_t c = c_numeric();
  v = (float)(c ? strtod_l(s, &end, c) : std::strtod(s, &end));  // without a C locale object: the process's
  if (required && end == s) return false;
  s = end;
  return errno == 0;
}

bool obj_int(const char*& s, int& v, bool required = true) {
  char* end;
  errno = 0;
  v = (int)std::strtol(s, &end, 10);
  if (required && end == s) return false;
  s = end;
  return errno == 0;
}

bool rest_blank(const char* s) {
  for (; *s; ++s)
    if (!blank(*s)) return false;
  return true;
}

// One range of whole lines: its statements in file order.  `first_t` /
// `first_n` are the index kinds of the range's first face corner, which every
// later corner of the range must repeat.
struct ObjRange {
  std::vector<float> pos, uv, nrm;
  std::vector<Corner> corners;
  std::vector<uint32_t> face_corners;  // corners per face
  bool any = false, first_t = false, first_n = false;
  int rc = FK_OK;
};

void parse_obj_lines(std::string& buf, size_t at, size_t stop, ObjRange& r) {
  while (at < stop) {
    size_t e = buf.find('\n', at);
    if (e == std::string::npos || e > stop) e = stop;
    char* line = &buf[at];
    const size_t len = e - at;
    if (e < buf.size() && buf[e] == '\n') buf[e] = '\0';  // C parsing stops at the line's end
    at = e + 1;
    size_t b = 0;
    while (b < len && blank(line[b])) ++b;
    if (b == len) continue;
    size_t te = b;
    while (te < len && !blank(line[te])) ++te;
    const char* tok = line + b;
    const size_t tl = te - b;
    const char* s = line + te;
    if (tok[0] == '#') continue;
    if (tok[0] == 'v' && tl == 1) {
      float x, y, z, w;
      if (!obj_float(s, x) || !obj_float(s, y) || !obj_float(s, z) || !obj_float(s, w, false) || !rest_blank(s)) {
        r.rc = FK_ERR_INVALID;
        return;
      }
      r.pos.insert(r.pos.end(), {x, y, z});
    } else if (tok[0] == 'v' && tl == 2 && tok[1] == 't') {
      float u, v, w;
      if (!obj_float(s, u) || !obj_float(s, v) || !obj_float(s, w, false) || !rest_blank(s)) {
        r.rc = FK_ERR_INVALID;
        return;
      }
      r.uv.insert(r.uv.end(), {u, v});
    } else if (tok[0] == 'v' && tl == 2 && tok[1] == 'n') {
      float i, j, k;
      if (!obj_float(s, i) || !obj_float(s, j) || !obj_float(s, k) || !rest_blank(s)) {
        r.rc = FK_ERR_INVALID;
        return;
      }
      r.nrm.insert(r.nrm.end(), {i, j, k});
    } else if (tok[0] == 'f' && tl == 1) {
      const size_t first = r.corners.size();
      while (!rest_blank(s)) {
        Corner c{0, 0, 0};
        bool ok = obj_int(s, c.p);
        if (ok && *s == '/') {
          ++s;
          ok = obj_int(s, c.t, false);
        }
        if (ok && *s == '/') {
          ++s;
          ok = obj_int(s, c.n);
        }
        if (ok && !r.any) {
          r.first_t = c.t != 0;
          r.first_n = c.n != 0;
          r.any = true;
        } else if (ok && ((c.t != 0) != r.first_t || (c.n != 0) != r.first_n)) {
          ok = false;
        }
        if (!ok) {
          r.rc = FK_ERR_INVALID;
          return;
        }
        r.corners.push_back(c);
        while (blank(*s)) ++s;
      }
      r.face_corners.push_back((uint32_t)(r.corners.size() - first));
    }
    // vp, p, l and unknown statements are skipped
  }
}

void parse_obj_range(std::string& buf, size_t at, size_t stop, ObjRange& r) {
  try {
    parse_obj_lines(buf, at, stop, r);
  } catch (const std::bad_alloc&) {
    r.rc = FK_ERR_NOMEM;
  }
}

int load_obj(const char* path, fk_mesh& m) {
  std::string buf;
  if (!read_file(path, buf)) return FK_OK;  // unreadable: empty mesh
  // Lines are independent but for the corner format the file's first corner
  // fixes, so large files are parsed in ranges of whole lines on threads of
  // their own and merged in file order; the format rule is then checked
  // across ranges (each range already checked its corners against its own
  // first one).  Any error anywhere rejects the file, as a sequential pass would.
  const size_t size = buf.size();
  const size_t min_range = (size_t)4 << 20;
  size_t parts = std::max<size_t>(1, std::min<size_t>(std::thread::hardware_concurrency(), 32));
  parts = std::max<size_t>(1, std::min(parts, size / min_range));
  std::vector<size_t> cut(1, 0);
  for (size_t k = 1; k < parts; ++k) {
    size_t c = std::max(cut.back(), size * k / parts);
    const size_t nl = buf.find('\n', c);
    if (nl == std::string::npos) break;
    cut.push_back(nl + 1);
  }
  cut.push_back(size);
  std::vector<ObjRange> ranges(cut.size() - 1);
  {
    std::vector<std::thread> pool;
    size_t started = 0;
    try {
      for (; ranges.size() > 1 && started < ranges.size(); ++started)
        pool.emplace_back(parse_obj_range, std::ref(buf), cut[started], cut[started + 1], std::ref(ranges[started]));
    } catch (const std::exception&) {  // no more threads: the rest on this one
    }
    for (size_t k = started; k < ranges.size(); ++k) parse_obj_range(buf, cut[k], cut[k + 1], ranges[k]);
    for (auto& t : pool) t.join();
  }
  const ObjRange* lead = nullptr;
  size_t np = 0, nt = 0, nn = 0, nc = 0, nf = 0;
  for (const auto& r : ranges) {
    if (r.rc != FK_OK) return r.rc;
    if (r.any) {
      if (!lead) lead = &r;
      else if (r.first_t != lead->first_t || r.first_n != lead->first_n) return FK_ERR_INVALID;
    }
    np += r.pos.size();
    nt += r.uv.size();
    nn += r.nrm.size();
    nc += r.corners.size();
    nf += r.face_corners.size();
  }
  if (nc >= 0xFFFFFFFFull || np / 3 >= 0xFFFFFFFFull) return FK_ERR_INVALID;  // beyond 32-bit vertex / position indices
  m.positions.reserve(np);
  m.texcoords.reserve(nt);
  m.normals.reserve(nn);
  for (const auto& r : ranges) {
    m.positions.insert(m.positions.end(), r.pos.begin(), r.pos.end());
    m.texcoords.insert(m.texcoords.end(), r.uv.begin(), r.uv.end());
    m.normals.insert(m.normals.end(), r.nrm.begin(), r.nrm.end());
  }
  m.vertices.resize(3 * nc);
  m.triangles.reserve(3 * (nc > 2 * nf ? nc - 2 * nf : 0));
  uint32_t v = 0;
  for (const auto& r : ranges) {
    size_t c0 = 0;
    for (const uint32_t count : r.face_corners) {
      uint32_t first = kNone, prev = kNone;
      for (uint32_t i = 0; i < count; ++i, ++v) {  // every corner its own vertex, polygons as fans
        const Corner& c = r.corners[c0 + i];
        uint32_t* x = &m.vertices[3 * (size_t)v];
        x[0] = (uint32_t)(c.p - 1);
        x[1] = c.t ? (uint32_t)(c.t - 1) : kNone;
        x[2] = c.n ? (uint32_t)(c.n - 1) : kNone;
        if (first == kNone) {
          first = v;
        } else if (prev == kNone) {
          prev = v;
        } else {
          m.triangles.insert(m.triangles.end(), {first, prev, v});
          prev = v;
        }
      }
      c0 += count;
    }
  }
  return FK_OK;
}

// ------------------------------------------------------------------ PLY
enum PlyType : uint8_t { kInvalid, kI8, kU8, kI16, kU16, kI32, kU32, kF32, kF64 };
const int kStride[] = {0, 1, 1, 2, 2, 4, 4, 4, 8};

PlyType ply_type(const std::string& s) {
  if (s == "int8" || s == "char") return kI8;
  if (s == "uint8" || s == "uchar") return kU8;
  if (s == "int16" || s == "short") return kI16;
  if (s == "uint16" || s == "ushort") return kU16;
  if (s == "int32" || s == "int") return kI32;
  if (s == "uint32" || s == "uint") return kU32;
  if (s == "float32" || s == "float") return kF32;
  if (s == "float64" || s == "double") return kF64;
  return kInvalid;
}

struct PlyProp {
  std::string name;
  PlyType type = kInvalid, count_type = kInvalid;
  bool list = false;
};
struct PlyElem {
  std::string name;
  size_t size = 0;
  std::vector<PlyProp> props;
};

// One grouped request: the values of its properties, in the order the data
// holds them, each stored as its own type; `type` is the last key's type.
struct Request {
  PlyType type = kInvalid;
  size_t count = 0;
  std::vector<uint8_t> bytes;
};

struct BadPly {};

class PlyReader {
 public:
  explicit PlyReader(const std::string& buf) : buf_(buf) {}

  // tinyply 2.0's header rules.  Returns false for a property line before
  // any element (the reference indexes an empty element list there).
  bool header() {
    while (at_ < buf_.size()) {
      size_t e = buf_.find('\n', at_);
      const std::string line = buf_.substr(at_, (e == std::string::npos ? buf_.size() : e) - at_);
      at_ = e == std::string::npos ? buf_.size() : e + 1;
      std::istringstream ls(line);
      ls.imbue(std::locale::classic());
      std::string tok;
      ls >> tok;
      if (tok == "ply" || tok == "PLY" || tok.empty() || tok == "comment" || tok == "obj_info") continue;
      if (tok == "format") {
        std::string f;
        ls >> f;
        if (f == "binary_little_endian") binary_ = true;
        else if (f == "binary_big_endian") binary_ = big_ = true;
      } else if (tok == "element") {
        PlyElem el;
        ls >> el.name >> el.size;
        elems_.push_back(el);
      } else if (tok == "property") {
        if (elems_.empty()) return false;
        PlyProp p;
        std::string t;
        ls >> t;
        if (t == "list") {
          std::string ct;
          ls >> ct >> t;
          p.count_type = ply_type(ct);
          p.list = true;
        }
        p.type = ply_type(t);
        ls >> p.name;
        elems_.back().props.push_back(p);
      } else {
        break;  // end_header, or a keyword tinyply stops at
      }
    }
    return true;
  }

  // request_properties_from_element: registers each key in turn and throws
  // (returns -1) at the first missing one, keeping the keys registered
  // before it, as tinyply does.
  int request(const std::string& elem, std::initializer_list<const char*> keys) {
    if (elems_.empty()) return -1;
    const PlyElem* el = nullptr;
    for (const auto& e : elems_)
      if (e.name == elem) {
        el = &e;
        break;
      }
    if (!el) return -1;
    const int id = (int)reqs_.size();
    reqs_.emplace_back();
    reqs_.back().count = el->size;
    for (const char* k : keys) {
      const PlyProp* p = nullptr;
      for (const auto& q : el->props)
        if (q.name == k) {
          p = &q;
          break;
        }
      if (!p) return -1;
      reqs_[id].type = p->type;
      if (!keys_.emplace(el->name + "-" + p->name, id).second) return -1;
    }
    return id;
  }

  // The data section, elements in header order; requested properties
  // append their values to their request, the others are skipped.
  void data() {
    if (!binary_) {
      ascii_.str(buf_.substr(at_));
      ascii_.imbue(std::locale::classic());
    }
    for (const auto& el : elems_) {
      // each property's request buffer, found once per element
      std::vector<std::vector<uint8_t>*> sink(el.props.size(), nullptr);
      for (size_t k = 0; k < el.props.size(); ++k) {
        auto it = keys_.find(el.name + "-" + el.props[k].name);
        if (it == keys_.end()) continue;
        sink[k] = &reqs_[it->second].bytes;
        if (binary_ && !el.props[k].list && el.props[k].type != kInvalid) {
          const size_t more = el.size * (size_t)kStride[el.props[k].type];
          if (more <= buf_.size() - at_) sink[k]->reserve(sink[k]->size() + more);  // never past the file's bytes
        }
      }
      if (binary_ && zero_width(el)) {  // unknown-type scalars only: no bytes to read, however many instances
        for (const auto* sk : sink)
          if (sk && el.size) throw BadPly();  // a requested unknown-type value (tinyply throws on the first)
        continue;
      }
      if (binary_ && fixed_layout(el)) {  // scalars only: fixed-size records, copied without per-value calls
        size_t rec = 0;
        for (const auto& p : el.props) rec += (size_t)kStride[p.type];
        if (rec && el.size > (buf_.size() - at_) / rec) throw BadPly();
        // per destination buffer, its properties' (record offset, size) in header order: one
        // instance's values land together, as the value-by-value path appends them
        std::vector<std::pair<std::vector<uint8_t>*, std::vector<std::pair<size_t, size_t>>>> groups;
        size_t off = 0;
        for (size_t k = 0; k < el.props.size(); ++k) {
          const size_t n = (size_t)kStride[el.props[k].type];
          if (sink[k]) {
            size_t g = 0;
            while (g < groups.size() && groups[g].first != sink[k]) ++g;
            if (g == groups.size()) groups.push_back({sink[k], {}});
            groups[g].second.push_back({off, n});
          }
          off += n;
        }
        const uint8_t* base = reinterpret_cast<const uint8_t*>(buf_.data()) + at_;
        for (auto& g : groups) {
          size_t per = 0;
          for (const auto& f : g.second) per += f.second;
          const size_t old = g.first->size();
          g.first->resize(old + el.size * per);
          uint8_t* dst = g.first->data() + old;
          // little-endian values of adjacent properties (x, y, z) are one span of each record
          bool span = !big_;
          for (size_t k = 1; k < g.second.size() && span; ++k)
            span = g.second[k].first == g.second[k - 1].first + g.second[k - 1].second;
          if (span) {
            strided_copy(dst, base + g.second[0].first, el.size, rec, per);
            continue;
          }
          for (size_t i = 0; i < el.size; ++i)
            for (const auto& f : g.second) {
              const uint8_t* src = base + i * rec + f.first;
              if (big_)
                for (size_t b = 0; b < f.second; ++b) dst[b] = src[f.second - 1 - b];
              else
                std::memcpy(dst, src, f.second);
              dst += f.second;
            }
        }
        at_ += el.size * rec;
        continue;
      }
      if (binary_ && el.props.size() == 1 && uniform_list(el, sink[0])) continue;
      for (size_t i = 0; i < el.size; ++i)
        for (size_t k = 0; k < el.props.size(); ++k) {
          const PlyProp& p = el.props[k];
          if (p.list) {
            const uint64_t n = count(p.count_type);
            if (binary_ && p.type != kInvalid) {  // the list's items in one copy, byte-swapped per item
              const size_t st = (size_t)kStride[p.type];
              if (n > (buf_.size() - at_) / st) throw BadPly();
              if (sink[k]) {
                const size_t old = sink[k]->size();
                sink[k]->resize(old + n * st);
                uint8_t* dst = sink[k]->data() + old;
                const uint8_t* src = reinterpret_cast<const uint8_t*>(buf_.data()) + at_;
                if (big_) {
                  for (size_t j = 0; j < n; ++j)
                    for (size_t b = 0; b < st; ++b) dst[j * st + b] = src[j * st + st - 1 - b];
                } else {
                  std::memcpy(dst, src, n * st);
                }
              }
              at_ += n * st;
            } else if (binary_) {  // unknown item type: no bytes per item
              if (sink[k] && n) throw BadPly();
            } else {
              for (uint64_t j = 0; j < n; ++j) value(p.type, sink[k]);
            }
          } else {
            value(p.type, sink[k]);
          }
        }
    }
  }

  const Request& req(int id) const { return reqs_[id]; }

 private:
  static bool zero_width(const PlyElem& el) {
    for (const auto& p : el.props)
      if (p.list || p.type != kInvalid) return false;
    return true;
  }
  // A binary element of one list property whose every instance has the
  // first one's length (a face element of triangles): its records have one
  // size, so the items are copied record by record without per-instance
  // count reads or buffer growth.  Leaves the data untouched and returns
  // false otherwise, for the value-by-value path (which also rejects what is
  // malformed).
  bool uniform_list(const PlyElem& el, std::vector<uint8_t>* sink) {
    if (el.props.size() != 1 || !el.props[0].list || el.props[0].type == kInvalid ||
        el.props[0].count_type == kInvalid || el.size == 0)
      return false;
    const PlyProp& p = el.props[0];
    const size_t cs = (size_t)kStride[p.count_type], st = (size_t)kStride[p.type];
    const size_t left = buf_.size() - at_;
    if (left < cs) return false;
    const uint8_t* base = reinterpret_cast<const uint8_t*>(buf_.data()) + at_;
    uint8_t v[8] = {0};
    for (size_t b = 0; b < cs; ++b) v[b] = base[big_ ? cs - 1 - b : b];
    uint64_t n;
    std::memcpy(&n, v, 8);
    if (n > (left - cs) / st) return false;
    const size_t rec = cs + (size_t)n * st;
    if (el.size > left / rec) return false;
    if (cs == 1) {
      for (size_t i = 1; i < el.size; ++i)
        if (base[i * rec] != base[0]) return false;
    } else {
      for (size_t i = 1; i < el.size; ++i)
        if (std::memcmp(base + i * rec, base, cs) != 0) return false;
    }
    if (sink) {
      const size_t old = sink->size(), item_bytes = (size_t)n * st;
      sink->resize(old + el.size * item_bytes);
      uint8_t* dst = sink->data() + old;
      if (!big_) {
        strided_copy(dst, base + cs, el.size, rec, item_bytes);
      } else {
        for (size_t i = 0; i < el.size; ++i, dst += item_bytes) {
          const uint8_t* src = base + i * rec + cs;
          for (size_t j = 0; j < n; ++j)
            for (size_t b = 0; b < st; ++b) dst[j * st + b] = src[j * st + st - 1 - b];
        }
      }
    }
    at_ += el.size * rec;
    return true;
  }
  // count pieces of `size` bytes, `stride` apart at src, packed at dst; the
  // usual piece sizes as fixed-size copies.
  static void strided_copy(uint8_t* dst, const uint8_t* src, size_t count, size_t stride, size_t size) {
    if (count == 0 || size == 0) return;  // dst may be an empty vector's null data
    switch (size) {
      case 4: for (size_t i = 0; i < count; ++i) std::memcpy(dst + 4 * i, src + i * stride, 4); break;
      case 6: for (size_t i = 0; i < count; ++i) std::memcpy(dst + 6 * i, src + i * stride, 6); break;
      case 8: for (size_t i = 0; i < count; ++i) std::memcpy(dst + 8 * i, src + i * stride, 8); break;
      case 12: for (size_t i = 0; i < count; ++i) std::memcpy(dst + 12 * i, src + i * stride, 12); break;
      case 16: for (size_t i = 0; i < count; ++i) std::memcpy(dst + 16 * i, src + i * stride, 16); break;
      default:
        if (size == stride) std::memcpy(dst, src, count * size);
        else for (size_t i = 0; i < count; ++i) std::memcpy(dst + size * i, src + i * stride, size);
    }
  }
  static bool fixed_layout(const PlyElem& el) {
    for (const auto& p : el.props)
      if (p.list || p.type == kInvalid) return false;
    return true;
  }

  // One value of type t; stored (native byte order) when out is given.
  void value(PlyType t, std::vector<uint8_t>* out) {
    uint8_t v[8] = {0};
    if (t == kInvalid) {
      if (out) throw BadPly();  // tinyply: "invalid ply property"
      if (!binary_) {           // skipped in ASCII: one token; in binary: no bytes
        std::string skip;
        if (!(ascii_ >> skip)) throw BadPly();
      }
      return;
    }
    const int n = kStride[t];
    if (binary_) {
      if (buf_.size() - at_ < (size_t)n) throw BadPly();
      for (int k = 0; k < n; ++k) v[k] = (uint8_t)buf_[at_ + (big_ ? n - 1 - k : k)];
      at_ += n;
    } else if (out) {
      parse(t, v);
    } else {
      std::string skip;
      if (!(ascii_ >> skip)) throw BadPly();
    }
    if (out) out->insert(out->end(), v, v + n);
  }

  // A list's length: the count type's value bits, zero-extended.
  uint64_t count(PlyType t) {
    if (t == kInvalid) throw BadPly();
    uint8_t v[8] = {0};
    const int n = kStride[t];
    if (binary_) {
      if (buf_.size() - at_ < (size_t)n) throw BadPly();
      for (int k = 0; k < n; ++k) v[k] = (uint8_t)buf_[at_ + (big_ ? n - 1 - k : k)];
      at_ += n;
    } else {
      parse(t, v);
    }
    uint64_t c;
    std::memcpy(&c, v, 8);
    return c;
  }

  // ASCII values through the stream extractors of the same types as
  // tinyply's read_property_ascii (chars through int32 / uint32).
  void parse(PlyType t, uint8_t* v) {
    bool ok = false;
    switch (t) {
      case kI8: { int32_t x; ok = (bool)(ascii_ >> x); int8_t y = (int8_t)x; std::memcpy(v, &y, 1); } break;
      case kU8: { uint32_t x; ok = (bool)(ascii_ >> x); uint8_t y = (uint8_t)x; std::memcpy(v, &y, 1); } break;
      case kI16: { int16_t x; ok = (bool)(ascii_ >> x); std::memcpy(v, &x, 2); } break;
      case kU16: { uint16_t x; ok = (bool)(ascii_ >> x); std::memcpy(v, &x, 2); } break;
      case kI32: { int32_t x; ok = (bool)(ascii_ >> x); std::memcpy(v, &x, 4); } break;
      case kU32: { uint32_t x; ok = (bool)(ascii_ >> x); std::memcpy(v, &x, 4); } break;
      case kF32: { float x; ok = (bool)(ascii_ >> x); std::memcpy(v, &x, 4); } break;
      case kF64: { double x; ok = (bool)(ascii_ >> x); std::memcpy(v, &x, 8); } break;
      default: break;
    }
    if (!ok) throw BadPly();
  }

  const std::string& buf_;
  size_t at_ = 0;
  bool binary_ = false, big_ = false;
  std::vector<PlyElem> elems_;
  std::vector<Request> reqs_;
  std::map<std::string, int> keys_;
  std::istringstream ascii_;
};

// copyPlyData (Src/mesh.cpp:460-513): float or double tuples of width w
// narrowed to float; other types give nothing.
bool tuples(const Request* r, int w, std::vector<float>& out) {
  out.clear();
  if (!r) return true;
  if (r->type == kF32) {
    if (r->bytes.size() < 4 * (size_t)w * r->count) return false;
    out.resize((size_t)w * r->count);
    if (!out.empty()) std::memcpy(out.data(), r->bytes.data(), 4 * out.size());
  } else if (r->type == kF64) {
    if (r->bytes.size() < 8 * (size_t)w * r->count) return false;
    out.resize((size_t)w * r->count);
    for (size_t i = 0; i < out.size(); ++i) {
      double d;
      std::memcpy(&d, r->bytes.data() + 8 * i, 8);
      out[i] = (float)d;
    }
  }
  return true;
}

int load_ply(const char* path, fk_mesh& m) {
  std::string buf;
  if (!read_file(path, buf)) return FK_ERR_INVALID;
  try {
    PlyReader r(buf);
    if (!r.header()) return FK_ERR_INVALID;
    const int verts = r.request("vertex", {"x", "y", "z"});
    if (verts < 0) return FK_ERR_INVALID;
    const int faces = r.request("face", {"vertex_indices"});
    if (faces < 0) return FK_ERR_INVALID;
    const int uvs = r.request("vertex", {"s", "t"});
    enum { kNowhere, kFace, kVertex } from = kNowhere;
    int norms = r.request("vertex", {"nx", "ny", "nz"});
    if (norms >= 0) {
      from = kVertex;
    } else {
      norms = r.request("face", {"nx", "ny", "nz"});
      if (norms >= 0) from = kFace;
    }
    r.data();
    if (!tuples(&r.req(verts), 3, m.positions) || !tuples(uvs >= 0 ? &r.req(uvs) : nullptr, 2, m.texcoords) ||
        !tuples(norms >= 0 ? &r.req(norms) : nullptr, 3, m.normals))
      return FK_ERR_INVALID;
    const Request& f = r.req(faces);
    if (f.count >= 0xFFFFFFFFull / 3) return FK_ERR_INVALID;  // corners beyond 32-bit vertex indices
    const int fs = kStride[f.type];
    if (f.type == kInvalid || f.type == kF32 || f.type == kF64) return FK_ERR_INVALID;
    if (f.bytes.size() < (size_t)fs * 3 * f.count) return FK_ERR_INVALID;
    m.vertices.resize(9 * f.count);
    m.triangles.resize(3 * f.count);
    // every face's three corners are vertices of their own: faces [a, b)
    // write their own slots, so large files split them over threads
    auto corners = [&](size_t a, size_t b) {
      uint32_t normal = kNone;
      for (size_t i = a; i < b; ++i) {
        const uint32_t v0 = (uint32_t)(3 * i);
        if (from == kFace) normal = (uint32_t)i * 3;
        for (size_t j = 0; j < 3; ++j) {
          const uint8_t* q = f.bytes.data() + (size_t)fs * (3 * i + j);
          uint32_t vi = 0;
          switch (f.type) {
            case kU32: std::memcpy(&vi, q, 4); break;
            case kU16: { uint16_t x; std::memcpy(&x, q, 2); vi = x; } break;
            case kI32: { int32_t x; std::memcpy(&x, q, 4); vi = (uint32_t)x; } break;
            case kI16: { int16_t x; std::memcpy(&x, q, 2); vi = (uint32_t)(int32_t)x; } break;
            case kI8: { int8_t x; std::memcpy(&x, q, 1); vi = (uint32_t)(int32_t)x; } break;
            default: vi = *q; break;  // kU8
          }
          if (from == kVertex) normal = vi;
          uint32_t* vx = &m.vertices[9 * i + 3 * j];
          vx[0] = vi;
          vx[1] = uvs >= 0 ? vi : kNone;
          vx[2] = normal;
        }
        m.triangles[3 * i] = v0;
        m.triangles[3 * i + 1] = v0 + 1;
        m.triangles[3 * i + 2] = v0 + 2;
      }
    };
    const size_t nf = (size_t)f.count;
    size_t parts = nf < ((size_t)1 << 16) ? 1 : std::max<size_t>(1, std::min<size_t>(std::thread::hardware_concurrency(), 16));
    std::vector<std::thread> pool;
    pool.reserve(parts);  // so that only starting a thread can throw below
    for (size_t k = 0; k < parts; ++k) {
      const size_t a = nf * k / parts, b = nf * (k + 1) / parts;
      if (k + 1 < parts) {
        try {
          pool.emplace_back(corners, a, b);
          continue;
        } catch (const std::system_error&) {  // no more threads: this range on this one
        }
      }
      corners(a, b);
    }
    for (auto& t : pool) t.join();
    return FK_OK;
  } catch (const BadPly&) {
    return FK_ERR_INVALID;
  } catch (const std::exception&) {
    return FK_ERR_INVALID;
  }
}

}  // namespace

extern "C" {

int fk_mesh_load(const char* path, fk_mesh** out) {
  if (!path || !out) return FK_ERR_INVALID;
  *out = nullptr;
  fk_mesh* m = new (std::nothrow) fk_mesh();
  if (!m) return FK_ERR_NOMEM;
  int rc = FK_ERR_INVALID;
  try {
    if (ends_with(path, ".obj")) rc = load_obj(path, *m);
    else if (ends_with(path, ".ply")) rc = load_ply(path, *m);
  } catch (const std::bad_alloc&) {
    rc = FK_ERR_NOMEM;
  }
  if (rc == FK_OK) {
    const uint32_t np = m->position_count();
    for (size_t v = 0; v < m->vertices.size(); v += 3)
      if (m->vertices[v] >= np) {
        rc = FK_ERR_INVALID;  // a corner names a position the file does not have
        break;
      }
  }
  if (rc != FK_OK) {
    delete m;
    return rc;
  }
  *out = m;
  return FK_OK;
}

}  // extern "C"
