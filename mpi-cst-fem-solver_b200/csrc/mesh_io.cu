// Gmsh .msh 4.1 ASCII reader (host code), so that the reference's meshes feed the GPU path
// directly. What it accepts and produces is the reference's read_gmsh (src/mesh_io.cpp): the
// sections $MeshFormat (4.1, ASCII), $PhysicalNames, $Entities, $Nodes and $Elements (others
// skipped), element types 1 (2-node line), 2 (3-node triangle) and 15 (point), triangles with a
// negative signed area turned counter-clockwise (and counted), line elements filed under the names
// of their entity's physical groups (the tag as text when unnamed), triangles with |area| below
// 1e-14 x (bounding-box diagonal)^2 rejected, errors as "path:line: message".
//
// The reader works in two passes over memory. The file is read whole and cut into tokens once
// (each token keeps its line number for the messages; a quoted physical name is one token); then
// every section is located in the token array and parsed from its token range. Nodes land in
// flat arrays (tags, coordinates) and their tag -> index lookup is a dense table when the tags are
// compact, a sorted (tag, index) array otherwise; element blocks are parsed into per-block corner
// arrays and turned into triangles and line groups afterwards.
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "../../include/cstfem_b200.h"

struct cstg_mesh {
  std::vector<double> xy;
  std::vector<long long> node_tags;
  std::vector<int32_t> tri;
  std::map<std::string, std::vector<int32_t>> groups;  // name -> 2 node indices per edge
  int flipped = 0;
};

namespace {

struct ReadError {
  std::string msg;
};

struct Token {
  size_t off, len;
  int line;
};

// The file cut into whitespace-separated tokens; "..." is one token (quotes included).
class TokenFile {
 public:
  TokenFile(std::string path, std::string text) : path_(std::move(path)), text_(std::move(text)) {
    int line = 1;
    size_t i = 0;
    const size_t n = text_.size();
    while (i < n) {
      const char ch = text_[i];
      if (ch == '\n') {
        ++line;
        ++i;
      } else if (ch == ' ' || ch == '\t' || ch == '\r') {
        ++i;
      } else if (ch == '"') {
        size_t j = i + 1;
        while (j < n && text_[j] != '"' && text_[j] != '\n') ++j;
        if (j < n && text_[j] == '"') ++j;
        tok_.push_back({i, j - i, line});
        i = j;
      } else {
        size_t j = i;
        while (j < n && text_[j] != ' ' && text_[j] != '\t' && text_[j] != '\r' && text_[j] != '\n') ++j;
        tok_.push_back({i, j - i, line});
        i = j;
      }
    }
    last_line_ = line;
  }
  size_t size() const { return tok_.size(); }
  std::string str(size_t k) const { return text_.substr(tok_[k].off, tok_[k].len); }
  bool is(size_t k, const char* s) const {
    return k < tok_.size() && tok_[k].len == std::strlen(s) && text_.compare(tok_[k].off, tok_[k].len, s) == 0;
  }
  bool is_header(size_t k) const { return k < tok_.size() && text_[tok_[k].off] == '$'; }
  int line_of(size_t k) const { return k < tok_.size() ? tok_[k].line : last_line_; }
  [[noreturn]] void fail_at(size_t k, const std::string& m) const {
    throw ReadError{path_ + ":" + std::to_string(line_of(k)) + ": " + m};
  }
  // numbers (strtoll / strtod over the token alone)
  bool as_int(size_t k, long long* v) const {
    const std::string s = str(k);
    char* e = nullptr;
    errno = 0;
    *v = std::strtoll(s.c_str(), &e, 10);
    return errno == 0 && e && *e == '\0' && !s.empty();
  }
  bool as_real(size_t k, double* v) const {
    const std::string s = str(k);
    char* e = nullptr;
    *v = std::strtod(s.c_str(), &e);
    return e && *e == '\0' && !s.empty();
  }

 private:
  std::string path_, text_;
  std::vector<Token> tok_;
  int last_line_ = 1;
};

// A cursor over one section's tokens [pos, end).
class Cursor {
 public:
  Cursor(const TokenFile& f, size_t pos, size_t end, const std::string& sec) : f_(f), k_(pos), end_(end), sec_(sec) {}
  size_t at() const { return k_; }
  bool done() const { return k_ >= end_; }
  size_t take(const char* what) {
    if (k_ >= end_) f_.fail_at(k_, std::string("unexpected end of $") + sec_ + " while reading " + what);
    return k_++;
  }
  long long integer(const char* what) {
    const size_t k = take(what);
    long long v;
    if (!f_.as_int(k, &v)) f_.fail_at(k, std::string("expected integer (") + what + ")");
    return v;
  }
  size_t count(const char* what) {
    const size_t k = k_;
    const long long v = integer(what);
    if (v < 0) f_.fail_at(k, std::string(what) + " must be non-negative");
    return (size_t)v;
  }
  int small(const char* what) {
    const size_t k = k_;
    const long long v = integer(what);
    if (v < std::numeric_limits<int>::min() || v > std::numeric_limits<int>::max())
      f_.fail_at(k, std::string(what) + " out of range");
    return (int)v;
  }
  double real(const char* what) {
    const size_t k = take(what);
    double v;
    if (!f_.as_real(k, &v)) f_.fail_at(k, std::string("expected number (") + what + ")");
    return v;
  }
  void skip(size_t n, const char* what) {
    for (size_t i = 0; i < n; ++i) take(what);
  }

 private:
  const TokenFile& f_;
  size_t k_, end_;
  std::string sec_;
};

struct Section {
  std::string name;
  size_t begin, end;  // body tokens (between the header and $End<name>)
  size_t header;
};

// Tag -> node index: a dense table over [min_tag, max_tag] when the tags fill at least a quarter
// of it, else binary search in (tag, index) pairs sorted by tag.
class NodeLookup {
 public:
  explicit NodeLookup(const std::vector<long long>& tags) {
    if (tags.empty()) return;
    lo_ = *std::min_element(tags.begin(), tags.end());
    const long long hi = *std::max_element(tags.begin(), tags.end());
    const unsigned long long span = (unsigned long long)(hi - lo_) + 1ull;
    if (span <= 4ull * tags.size() + 16ull) {
      dense_.assign((size_t)span, -1);
      for (size_t i = 0; i < tags.size(); ++i) {
        int& slot = dense_[(size_t)(tags[i] - lo_)];
        if (slot >= 0) dup_ = tags[i];
        slot = (int)i;
      }
    } else {
      sorted_.reserve(tags.size());
      for (size_t i = 0; i < tags.size(); ++i) sorted_.emplace_back(tags[i], (int)i);
      std::sort(sorted_.begin(), sorted_.end());
      for (size_t i = 1; i < sorted_.size(); ++i)
        if (sorted_[i].first == sorted_[i - 1].first) dup_ = sorted_[i].first;
    }
  }
  long long duplicate() const { return dup_; }
  int find(long long tag) const {
    if (!dense_.empty()) {
      if (tag < lo_ || tag - lo_ >= (long long)dense_.size()) return -1;
      return dense_[(size_t)(tag - lo_)];
    }
    const auto it = std::lower_bound(sorted_.begin(), sorted_.end(), std::make_pair(tag, -1));
    return it != sorted_.end() && it->first == tag ? it->second : -1;
  }

 private:
  long long lo_ = 0, dup_ = 0;
  std::vector<int> dense_;
  std::vector<std::pair<long long, int>> sorted_;
};

struct ElementBlock {
  int dim = 0, entity = 0, type = 0;
  std::vector<long long> corner_tags;  // `per` node tags per element
  std::vector<size_t> token;           // token of each element (its line for the messages)
};

// the reference's signed area (element.cpp:17-24), the same operations
double signed_area(const double* p0, const double* p1, const double* p2) {
  return 0.5 * ((p1[0] - p0[0]) * (p2[1] - p0[1]) - (p2[0] - p0[0]) * (p1[1] - p0[1]));
}

// The section table: every "$Name ... $EndName" span of the file, in file order.
std::vector<Section> sections(const TokenFile& f) {
  std::vector<Section> out;
  size_t k = 0;
  while (k < f.size()) {
    if (!f.is_header(k) || f.str(k).rfind("$End", 0) == 0)
      f.fail_at(k, "expected a section header, got '" + f.str(k) + "'");
    const std::string name = f.str(k).substr(1);
    if (out.empty() && name != "MeshFormat") f.fail_at(k, "file must start with $MeshFormat");
    const std::string end = "$End" + name;
    size_t j = k + 1;
    while (j < f.size() && !f.is(j, end.c_str())) ++j;
    if (j >= f.size()) f.fail_at(j, "unexpected end of file inside $" + name);
    out.push_back({name, k + 1, j, k});
    k = j + 1;
  }
  return out;
}

void parse_format(const TokenFile& f, const Section& s) {
  Cursor c(f, s.begin, s.end, s.name);
  const size_t v = c.take("version");
  if (!f.is(v, "4.1")) f.fail_at(v, "unsupported .msh version '" + f.str(v) + "' (need 4.1)");
  if (c.integer("file-type") != 0) f.fail_at(v, "binary .msh files are not supported (need ASCII, file-type 0)");
  c.integer("data-size");
  if (!c.done()) f.fail_at(c.at(), "expected $EndMeshFormat, got '" + f.str(c.at()) + "'");
}

// (dim, physical tag) -> name
std::map<std::pair<int, int>, std::string> parse_names(const TokenFile& f, const Section& s) {
  std::map<std::pair<int, int>, std::string> names;
  Cursor c(f, s.begin, s.end, s.name);
  const size_t n = c.count("numPhysicalNames");
  for (size_t i = 0; i < n; ++i) {
    const int dim = c.small("dimension"), tag = c.small("physical tag");
    const size_t k = c.take("physical name");
    const std::string q = f.str(k);
    if (q.size() < 2 || q.front() != '"' || q.back() != '"') f.fail_at(k, "physical name must be quoted");
    if (!names.emplace(std::make_pair(dim, tag), q.substr(1, q.size() - 2)).second)
      f.fail_at(k, "duplicate physical group (" + std::to_string(dim) + ", " + std::to_string(tag) + ")");
  }
  return names;
}

// (dim, entity tag) -> physical tags; every entity's bounding-entity list is consumed too
std::map<std::pair<int, int>, std::vector<int>> parse_entities(const TokenFile& f, const Section& s) {
  std::map<std::pair<int, int>, std::vector<int>> phys;
  Cursor c(f, s.begin, s.end, s.name);
  const char* what[4] = {"numPoints", "numCurves", "numSurfaces", "numVolumes"};
  size_t cnt[4];
  for (int d = 0; d < 4; ++d) cnt[d] = c.count(what[d]);
  for (int d = 0; d < 4; ++d)
    for (size_t i = 0; i < cnt[d]; ++i) {
      const int tag = c.small("entity tag");
      for (int q = 0; q < (d == 0 ? 3 : 6); ++q) c.real("entity coordinate");
      std::vector<int> tags(c.count("numPhysicalTags"));
      for (int& t : tags) t = c.small("physical tag");
      if (d > 0) c.skip(c.count("numBoundingEntities"), "bounding entity tag");
      phys[std::make_pair(d, tag)] = std::move(tags);
    }
  return phys;
}

void parse_nodes(const TokenFile& f, const Section& s, cstg_mesh& m) {
  Cursor c(f, s.begin, s.end, s.name);
  const size_t blocks = c.count("numEntityBlocks");
  const size_t total = c.count("numNodes");
  c.integer("minNodeTag");
  c.integer("maxNodeTag");
  m.node_tags.reserve(total);
  m.xy.reserve(2 * total);
  for (size_t b = 0; b < blocks; ++b) {
    const int dim = c.small("entityDim");
    c.small("entityTag");
    const bool parametric = c.integer("parametric") != 0;
    const size_t n = c.count("numNodesInBlock");
    for (size_t i = 0; i < n; ++i) {
      const size_t k = c.at();
      const long long tag = c.integer("node tag");
      if (tag <= 0) f.fail_at(k, "node tag must be positive");
      m.node_tags.push_back(tag);
    }
    for (size_t i = 0; i < n; ++i) {
      m.xy.push_back(c.real("x"));
      m.xy.push_back(c.real("y"));
      c.real("z");
      if (parametric) c.skip((size_t)std::max(dim, 0), "parametric coordinate");
    }
  }
  if (m.node_tags.size() != total)
    f.fail_at(s.header, "node count mismatch: header says " + std::to_string(total) + ", blocks contain " +
                            std::to_string(m.node_tags.size()));
}

std::vector<ElementBlock> parse_elements(const TokenFile& f, const Section& s) {
  Cursor c(f, s.begin, s.end, s.name);
  const size_t blocks = c.count("numEntityBlocks");
  const size_t total = c.count("numElements");
  c.integer("minElementTag");
  c.integer("maxElementTag");
  std::vector<ElementBlock> out(blocks);
  size_t seen = 0;
  for (ElementBlock& eb : out) {
    const size_t hk = c.at();
    eb.dim = c.small("entityDim");
    eb.entity = c.small("entityTag");
    eb.type = c.small("elementType");
    const size_t n = c.count("numElementsInBlock");
    const int per = eb.type == 1 ? 2 : eb.type == 2 ? 3 : eb.type == 15 ? 1 : 0;
    if (!per)
      f.fail_at(hk, "unsupported element type " + std::to_string(eb.type) +
                        " (supported: 1 = 2-node line, 2 = 3-node triangle, 15 = point)");
    eb.corner_tags.resize(n * (size_t)per);
    eb.token.resize(n);
    for (size_t i = 0; i < n; ++i) {
      eb.token[i] = c.at();
      c.integer("element tag");
      for (int q = 0; q < per; ++q) eb.corner_tags[i * per + q] = c.integer("element node tag");
    }
    seen += n;
  }
  if (seen != total)
    f.fail_at(s.header, "element count mismatch: header says " + std::to_string(total) + ", blocks contain " +
                            std::to_string(seen));
  return out;
}

// Triangles (oriented counter-clockwise, degenerate ones rejected) and line groups from the blocks.
void build_mesh(const TokenFile& f, const std::vector<ElementBlock>& blocks,
                const std::map<std::pair<int, int>, std::string>& names,
                const std::map<std::pair<int, int>, std::vector<int>>& phys, const NodeLookup& lookup, cstg_mesh& m) {
  double lo[2] = {std::numeric_limits<double>::max(), std::numeric_limits<double>::max()};
  double hi[2] = {std::numeric_limits<double>::lowest(), std::numeric_limits<double>::lowest()};
  for (size_t i = 0; i < m.xy.size(); ++i) {
    lo[i & 1] = std::min(lo[i & 1], m.xy[i]);
    hi[i & 1] = std::max(hi[i & 1], m.xy[i]);
  }
  const double diag2 = m.xy.empty() ? 0.0 : (hi[0] - lo[0]) * (hi[0] - lo[0]) + (hi[1] - lo[1]) * (hi[1] - lo[1]);
  const double min_area = 1e-14 * diag2;
  for (const ElementBlock& eb : blocks) {
    const int per = eb.type == 1 ? 2 : eb.type == 2 ? 3 : 1;
    std::vector<std::string> group_names;
    if (eb.type == 1) {
      const auto it = phys.find(std::make_pair(eb.dim, eb.entity));
      if (it != phys.end())
        for (int p : it->second) {
          const auto nm = names.find(std::make_pair(eb.dim, p));
          group_names.push_back(nm != names.end() ? nm->second : std::to_string(p));
        }
    }
    for (size_t i = 0; i < eb.token.size(); ++i) {
      int idx[3] = {0, 0, 0};
      for (int q = 0; q < per; ++q) {
        const long long tag = eb.corner_tags[i * per + q];
        const int v = tag > 0 ? lookup.find(tag) : -1;
        if (v < 0) f.fail_at(eb.token[i], "unknown node tag " + std::to_string(tag));
        idx[q] = v;
      }
      if (eb.type == 2) {
        const double a = signed_area(&m.xy[2 * (size_t)idx[0]], &m.xy[2 * (size_t)idx[1]], &m.xy[2 * (size_t)idx[2]]);
        if (a == 0.0 || std::fabs(a) < min_area) {
          char buf[160];
          std::snprintf(buf, sizeof buf, "degenerate triangle (area %g, threshold %g)", a, min_area);
          f.fail_at(eb.token[i], buf);
        }
        if (a < 0.0) {
          std::swap(idx[1], idx[2]);
          ++m.flipped;
        }
        m.tri.insert(m.tri.end(), idx, idx + 3);
      } else if (eb.type == 1) {
        for (const std::string& g : group_names) {
          std::vector<int32_t>& e = m.groups[g];
          e.push_back(idx[0]);
          e.push_back(idx[1]);
        }
      }
    }
  }
}

void read_msh(const std::string& path, const std::string& text, cstg_mesh& m) {
  const TokenFile f(path, text);
  const std::vector<Section> secs = sections(f);
  const Section* found[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  const char* required[5] = {"MeshFormat", "PhysicalNames", "Entities", "Nodes", "Elements"};
  for (const Section& s : secs)
    for (int r = 0; r < 5; ++r)
      if (s.name == required[r]) {
        if (found[r]) f.fail_at(s.header, "duplicate $" + s.name + " section");
        found[r] = &s;
      }
  for (int r = 0; r < 5; ++r)
    if (!found[r]) f.fail_at(f.size(), std::string("missing $") + required[r] + " section");
  if (found[4]->header < found[3]->header) f.fail_at(found[4]->header, "$Elements must come after $Nodes");
  if (found[4]->header < found[2]->header) f.fail_at(found[4]->header, "$Elements must come after $Entities");
  parse_format(f, *found[0]);
  const auto names = parse_names(f, *found[1]);
  const auto phys = parse_entities(f, *found[2]);
  parse_nodes(f, *found[3], m);
  const NodeLookup lookup(m.node_tags);
  if (lookup.duplicate()) f.fail_at(found[3]->header, "duplicate node tag " + std::to_string(lookup.duplicate()));
  const std::vector<ElementBlock> blocks = parse_elements(f, *found[4]);
  build_mesh(f, blocks, names, phys, lookup, m);
}

bool slurp(const char* path, std::string* text) {
  FILE* fp = std::fopen(path, "rb");
  if (!fp) return false;
  char buf[1 << 16];
  size_t got;
  while ((got = std::fread(buf, 1, sizeof buf, fp)) > 0) text->append(buf, got);
  const bool ok = !std::ferror(fp);
  std::fclose(fp);
  return ok;
}

void put_err(char* err, int len, const std::string& m) {
  if (err && len > 0) std::snprintf(err, (size_t)len, "%s", m.c_str());
}

}  // namespace

extern "C" {

int cstg_read_gmsh(const char* path, cstg_mesh** out, char* err, int err_len) {
  if (!path || !out) return CSTG_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  std::string text;
  if (!slurp(path, &text)) {
    put_err(err, err_len, std::string(path) + ": cannot open file");
    return CSTG_ERR_MESH;
  }
  cstg_mesh* m = new cstg_mesh();
  try {
    read_msh(path, text, *m);
  } catch (const ReadError& e) {
    delete m;
    put_err(err, err_len, e.msg);
    return CSTG_ERR_MESH;
  } catch (const std::exception& e) {
    delete m;
    put_err(err, err_len, std::string(path) + ": " + e.what());
    return CSTG_ERR_MESH;
  }
  *out = m;
  return CSTG_OK;
}

void cstg_mesh_destroy(cstg_mesh* m) { delete m; }

int cstg_mesh_info(const cstg_mesh* m, int* n_nodes, int* n_tri, int* n_groups, int* flipped) {
  if (!m) return CSTG_ERR_INVALID_ARGUMENT;
  if (n_nodes) *n_nodes = (int)m->node_tags.size();
  if (n_tri) *n_tri = (int)(m->tri.size() / 3);
  if (n_groups) *n_groups = (int)m->groups.size();
  if (flipped) *flipped = m->flipped;
  return CSTG_OK;
}

int cstg_mesh_arrays(const cstg_mesh* m, double* xy, int32_t* tri, long long* node_tags) {
  if (!m) return CSTG_ERR_INVALID_ARGUMENT;
  if (xy && !m->xy.empty()) std::memcpy(xy, m->xy.data(), sizeof(double) * m->xy.size());
  if (tri && !m->tri.empty()) std::memcpy(tri, m->tri.data(), sizeof(int32_t) * m->tri.size());
  if (node_tags && !m->node_tags.empty())
    std::memcpy(node_tags, m->node_tags.data(), sizeof(long long) * m->node_tags.size());
  return CSTG_OK;
}

int cstg_mesh_group(const cstg_mesh* m, int index, char* name, int name_len, int* n_edges, int32_t* edges) {
  if (!m || index < 0 || index >= (int)m->groups.size()) return CSTG_ERR_INVALID_ARGUMENT;
  auto it = m->groups.begin();
  std::advance(it, index);
  if (name && name_len > 0) std::snprintf(name, (size_t)name_len, "%s", it->first.c_str());
  if (n_edges) *n_edges = (int)(it->second.size() / 2);
  if (edges && !it->second.empty()) std::memcpy(edges, it->second.data(), sizeof(int32_t) * it->second.size());
  return CSTG_OK;
}

}  // extern "C"
