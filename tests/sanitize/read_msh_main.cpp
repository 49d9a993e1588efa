// Drives the .msh 4.1 reader (csrc/mesh_io.cu, host C++) through its C ABI for one file, so that
// tests/test_sanitize_reader.py can build it with AddressSanitizer and UndefinedBehaviorSanitizer
// and feed it valid and malformed files. Prints "ok <nodes> <triangles> <groups>" or
// "err <status> <message>"; exits 0 unless a mesh the reader accepted breaks its own contract
// (a triangle index outside the nodes, a boundary edge outside the nodes): exit 3.
#include <cstdio>
#include <vector>

#include "../../include/cstfem_b200.h"

int main(int argc, char** argv) {
  if (argc != 2) {
    std::fprintf(stderr, "usage: %s mesh.msh\n", argv[0]);
    return 2;
  }
  cstg_mesh* m = nullptr;
  char err[512] = {0};
  const int st = cstg_read_gmsh(argv[1], &m, err, (int)sizeof(err));
  if (st != CSTG_OK) {
    std::printf("err %d %s\n", st, err);
    return m == nullptr ? 0 : 3;  // a failed read hands back no mesh
  }
  int n_nodes = 0, n_tri = 0, n_groups = 0, flipped = 0;
  cstg_mesh_info(m, &n_nodes, &n_tri, &n_groups, &flipped);
  std::vector<double> xy((size_t)n_nodes * 2);
  std::vector<int32_t> tri((size_t)n_tri * 3);
  std::vector<long long> tags((size_t)n_nodes);
  cstg_mesh_arrays(m, xy.data(), tri.data(), tags.data());
  int bad = 0;
  for (int32_t v : tri) bad += v < 0 || v >= n_nodes;
  for (int g = 0; g < n_groups; ++g) {
    char name[256];
    int n_edges = 0;
    cstg_mesh_group(m, g, name, (int)sizeof(name), &n_edges, nullptr);
    std::vector<int32_t> edges((size_t)n_edges * 2);
    cstg_mesh_group(m, g, name, (int)sizeof(name), &n_edges, edges.data());
    for (int32_t v : edges) bad += v < 0 || v >= n_nodes;
  }
  cstg_mesh_destroy(m);
  std::printf("ok %d %d %d\n", n_nodes, n_tri, n_groups);
  return bad ? 3 : 0;
}
