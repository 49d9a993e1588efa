// Gmsh .msh 4.1 ASCII reader (host code), so that the reference's meshes feed the GPU path
// directly. The accepted format and the resulting mesh are the reference's read_gmsh
// (src/mesh_io.cpp): sections $MeshFormat (4.1, ASCII), $PhysicalNames, $Entities, $Nodes,
// $Elements (others skipped); element types 1 (2-node line), 2 (3-node triangle), 15 (point);
// triangles with negative signed area are turned counter-clockwise (counted); line elements are
// filed under the names of their entity's physical groups (the tag as text when unnamed);
// triangles with |area| < 1e-14 x (bounding-box diagonal)^2 are rejected. Errors read
// "path:line: message".
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <map>
#include <sstream>
#include <string>
#include <unordered_map>
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

struct MshError {
  std::string msg;
};

class Lines {
 public:
  Lines(std::istream& in, std::string src) : in_(in), src_(std::move(src)) {}
  bool next(std::string& s) {
    std::string raw;
    while (std::getline(in_, raw)) {
      ++no_;
      const size_t a = raw.find_first_not_of(" \t\r");
      if (a == std::string::npos) continue;
      const size_t b = raw.find_last_not_of(" \t\r");
      s = raw.substr(a, b - a + 1);
      return true;
    }
    return false;
  }
  std::string need(const char* what) {
    std::string s;
    if (!next(s)) fail(std::string("unexpected end of file while reading ") + what);
    return s;
  }
  [[noreturn]] void fail(const std::string& m) const { throw MshError{src_ + ":" + std::to_string(no_) + ": " + m}; }

 private:
  std::istream& in_;
  std::string src_;
  int no_ = 0;
};

struct Fields {
  Fields(Lines& l, const std::string& s) : l(l), ss(s) {}
  long long i(const char* what) {
    long long v;
    if (!(ss >> v)) l.fail(std::string("expected integer (") + what + ")");
    return v;
  }
  double d(const char* what) {
    double v;
    if (!(ss >> v)) l.fail(std::string("expected number (") + what + ")");
    return v;
  }
  std::string rest() {
    std::string s;
    std::getline(ss, s);
    const size_t a = s.find_first_not_of(" \t");
    return a == std::string::npos ? std::string() : s.substr(a);
  }
  Lines& l;
  std::istringstream ss;
};

size_t count_of(Lines& l, long long v, const char* what) {
  if (v < 0) l.fail(std::string(what) + " must be non-negative");
  return (size_t)v;
}

int int_of(Lines& l, long long v, const char* what) {
  if (v < std::numeric_limits<int>::min() || v > std::numeric_limits<int>::max())
    l.fail(std::string(what) + " out of range");
  return (int)v;
}

void end_of(Lines& l, const char* sec) {
  const std::string s = l.need((std::string("$End") + sec).c_str());
  if (s != std::string("$End") + sec) l.fail(std::string("expected $End") + sec + ", got '" + s + "'");
}

// the reference's signed area (element.cpp:17-24), same operations
double signed_area(const double* p0, const double* p1, const double* p2) {
  return 0.5 * ((p1[0] - p0[0]) * (p2[1] - p0[1]) - (p2[0] - p0[0]) * (p1[1] - p0[1]));
}

void read_msh(std::istream& in, const std::string& src, cstg_mesh& m) {
  Lines L(in, src);
  bool fmt = false, names_ok = false, ents_ok = false, nodes_ok = false, elems_ok = false;
  std::map<std::pair<int, int>, std::string> names;           // (dim, physical tag) -> name
  std::map<std::pair<int, int>, std::vector<int>> ent_phys;   // (dim, entity tag) -> physical tags
  std::unordered_map<long long, int> index;                   // node tag -> index
  std::string s;
  while (L.next(s)) {
    if (s[0] != '$' || s.rfind("$End", 0) == 0) L.fail("expected a section header, got '" + s + "'");
    const std::string sec = s.substr(1);
    if (!fmt && sec != "MeshFormat") L.fail("file must start with $MeshFormat");
    if (sec == "MeshFormat") {
      if (fmt) L.fail("duplicate $MeshFormat section");
      const std::string h = L.need("$MeshFormat");
      if (h.substr(0, h.find_first_of(" \t")) != "4.1")
        L.fail("unsupported .msh version '" + h.substr(0, h.find_first_of(" \t")) + "' (need 4.1)");
      Fields f(L, h);
      f.d("version");
      if (f.i("file-type") != 0) L.fail("binary .msh files are not supported (need ASCII, file-type 0)");
      f.i("data-size");
      end_of(L, "MeshFormat");
      fmt = true;
    } else if (sec == "PhysicalNames") {
      Fields h(L, L.need("$PhysicalNames"));
      const size_t n = count_of(L, h.i("numPhysicalNames"), "numPhysicalNames");
      for (size_t k = 0; k < n; ++k) {
        Fields f(L, L.need("physical name"));
        const int dim = int_of(L, f.i("dimension"), "dimension"), tag = int_of(L, f.i("physical tag"), "physical tag");
        std::string nm = f.rest();
        if (nm.size() < 2 || nm.front() != '"' || nm.back() != '"') L.fail("physical name must be quoted");
        nm = nm.substr(1, nm.size() - 2);
        if (!names.emplace(std::make_pair(dim, tag), nm).second)
          L.fail("duplicate physical group (" + std::to_string(dim) + ", " + std::to_string(tag) + ")");
      }
      end_of(L, "PhysicalNames");
      names_ok = true;
    } else if (sec == "Entities") {
      Fields h(L, L.need("$Entities"));
      size_t cnt[4];
      const char* what[4] = {"numPoints", "numCurves", "numSurfaces", "numVolumes"};
      for (int d = 0; d < 4; ++d) cnt[d] = count_of(L, h.i(what[d]), what[d]);
      for (int d = 0; d < 4; ++d)
        for (size_t k = 0; k < cnt[d]; ++k) {
          Fields f(L, L.need("entity"));
          const int tag = int_of(L, f.i("entity tag"), "entity tag");
          for (int c = 0; c < (d == 0 ? 3 : 6); ++c) f.d("entity coordinate");
          std::vector<int> ph(count_of(L, f.i("numPhysicalTags"), "numPhysicalTags"));
          for (int& p : ph) p = int_of(L, f.i("physical tag"), "physical tag");
          ent_phys[std::make_pair(d, tag)] = ph;
        }
      end_of(L, "Entities");
      ents_ok = true;
    } else if (sec == "Nodes") {
      Fields h(L, L.need("$Nodes"));
      const size_t nb = count_of(L, h.i("numEntityBlocks"), "numEntityBlocks");
      const size_t nn = count_of(L, h.i("numNodes"), "numNodes");
      m.xy.reserve(2 * nn);
      m.node_tags.reserve(nn);
      for (size_t b = 0; b < nb; ++b) {
        Fields bh(L, L.need("node block header"));
        bh.i("entityDim");
        bh.i("entityTag");
        bh.i("parametric");
        const size_t n = count_of(L, bh.i("numNodesInBlock"), "numNodesInBlock");
        for (size_t k = 0; k < n; ++k) {
          Fields f(L, L.need("node tag"));
          const long long tag = f.i("node tag");
          if (tag <= 0) L.fail("node tag must be positive");
          if (!index.emplace(tag, (int)m.node_tags.size()).second) L.fail("duplicate node tag " + std::to_string(tag));
          m.node_tags.push_back(tag);
        }
        for (size_t k = 0; k < n; ++k) {
          Fields f(L, L.need("node coordinates"));
          const double x = f.d("x"), y = f.d("y");
          f.d("z");
          m.xy.push_back(x);
          m.xy.push_back(y);
        }
      }
      if (m.node_tags.size() != nn)
        L.fail("node count mismatch: header says " + std::to_string(nn) + ", blocks contain " +
               std::to_string(m.node_tags.size()));
      end_of(L, "Nodes");
      nodes_ok = true;
    } else if (sec == "Elements") {
      if (!nodes_ok) L.fail("$Elements must come after $Nodes");
      if (!ents_ok) L.fail("$Elements must come after $Entities");
      double x0 = std::numeric_limits<double>::max(), x1 = std::numeric_limits<double>::lowest();
      double y0 = x0, y1 = x1;
      for (size_t k = 0; k < m.node_tags.size(); ++k) {
        x0 = std::min(x0, m.xy[2 * k]);
        x1 = std::max(x1, m.xy[2 * k]);
        y0 = std::min(y0, m.xy[2 * k + 1]);
        y1 = std::max(y1, m.xy[2 * k + 1]);
      }
      const double diag2 = m.node_tags.empty() ? 0.0 : (x1 - x0) * (x1 - x0) + (y1 - y0) * (y1 - y0);
      const double min_area = 1e-14 * diag2;
      Fields h(L, L.need("$Elements"));
      const size_t nb = count_of(L, h.i("numEntityBlocks"), "numEntityBlocks");
      const size_t ne = count_of(L, h.i("numElements"), "numElements");
      size_t seen = 0;
      for (size_t b = 0; b < nb; ++b) {
        Fields bh(L, L.need("element block header"));
        const int edim = int_of(L, bh.i("entityDim"), "entityDim"), etag = int_of(L, bh.i("entityTag"), "entityTag");
        const int type = int_of(L, bh.i("elementType"), "elementType");
        const size_t n = count_of(L, bh.i("numElementsInBlock"), "numElementsInBlock");
        seen += n;
        const int per = type == 1 ? 2 : type == 2 ? 3 : type == 15 ? 1 : 0;
        if (!per)
          L.fail("unsupported element type " + std::to_string(type) +
                 " (supported: 1 = 2-node line, 2 = 3-node triangle, 15 = point)");
        std::vector<std::string> grp;
        if (type == 1) {
          const auto it = ent_phys.find(std::make_pair(edim, etag));
          if (it != ent_phys.end())
            for (int p : it->second) {
              const auto nt = names.find(std::make_pair(edim, p));
              grp.push_back(nt != names.end() ? nt->second : std::to_string(p));
            }
        }
        for (size_t k = 0; k < n; ++k) {
          Fields f(L, L.need("element"));
          f.i("element tag");
          int c[3] = {0, 0, 0};
          for (int q = 0; q < per; ++q) {
            const long long tag = f.i("element node tag");
            const auto it = index.find(tag);
            if (tag <= 0 || it == index.end()) L.fail("unknown node tag " + std::to_string(tag));
            c[q] = it->second;
          }
          if (type == 2) {
            const double a = signed_area(&m.xy[2 * (size_t)c[0]], &m.xy[2 * (size_t)c[1]], &m.xy[2 * (size_t)c[2]]);
            if (a == 0.0 || std::fabs(a) < min_area) {
              std::ostringstream o;
              o << "degenerate triangle (area " << a << ", threshold " << min_area << ")";
              L.fail(o.str());
            }
            if (a < 0.0) {
              std::swap(c[1], c[2]);
              ++m.flipped;
            }
            m.tri.insert(m.tri.end(), c, c + 3);
          } else if (type == 1) {
            for (const auto& g : grp) {
              auto& v = m.groups[g];
              v.push_back(c[0]);
              v.push_back(c[1]);
            }
          }
        }
      }
      if (seen != ne)
        L.fail("element count mismatch: header says " + std::to_string(ne) + ", blocks contain " +
               std::to_string(seen));
      end_of(L, "Elements");
      elems_ok = true;
    } else {
      bool closed = false;
      std::string t;
      while (L.next(t))
        if (t == "$End" + sec) {
          closed = true;
          break;
        }
      if (!closed) L.fail("unexpected end of file inside $" + sec);
    }
  }
  const std::pair<bool, const char*> req[] = {{fmt, "$MeshFormat"}, {names_ok, "$PhysicalNames"},
                                              {ents_ok, "$Entities"}, {nodes_ok, "$Nodes"},
                                              {elems_ok, "$Elements"}};
  for (const auto& r : req)
    if (!r.first) L.fail(std::string("missing ") + r.second + " section");
}

void put_err(char* err, int len, const std::string& m) {
  if (err && len > 0) {
    std::snprintf(err, (size_t)len, "%s", m.c_str());
  }
}

}  // namespace

extern "C" {

int cstg_read_gmsh(const char* path, cstg_mesh** out, char* err, int err_len) {
  if (!path || !out) return CSTG_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  std::ifstream in(path);
  if (!in) {
    put_err(err, err_len, std::string(path) + ": cannot open file");
    return CSTG_ERR_MESH;
  }
  cstg_mesh* m = new cstg_mesh();
  try {
    read_msh(in, path, *m);
  } catch (const MshError& e) {
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
