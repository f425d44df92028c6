// fs_neutral.cu -- host-side face connectivity of Gambit neutral-file meshes.
//
// GlobalConnectivity (GlobalGridConnectivity.for:4-523) matches every new
// element face against all faces made so far and then against every face of
// every element: O(N^2).  The same face list comes out of one pass with a
// hash of the sorted face nodes: elements in order, local faces in order, a
// face on a boundary record is left for the boundary pass, a face already in
// the table is the second side of an interior face, anything else is the
// next interior face (its nodes in the creating element's local order, owner
// the creating, i.e. lower, element).  Boundary faces follow set by set,
// record by record, with the nodes of the element's local face.
#include <cstdint>
#include <unordered_map>
#include <vector>

#include "fsb200.h"

namespace {

struct FaceDef { int n; int v[4]; };

// LocalElementFaceNodes per NTypeGeometry, 0-based element-local node
// indices (GlobalGridConnectivity.for:21-120; Gambit's face conventions)
const FaceDef kBrick[6] = {{4, {0, 1, 5, 4}}, {4, {1, 3, 7, 5}}, {4, {3, 2, 6, 7}},
                           {4, {2, 0, 4, 6}}, {4, {1, 0, 2, 3}}, {4, {4, 5, 7, 6}}};
const FaceDef kWedge[5] = {{4, {0, 1, 4, 3}}, {4, {1, 2, 5, 4}}, {4, {2, 0, 3, 5}},
                           {3, {0, 2, 1, -1}}, {3, {3, 4, 5, -1}}};
const FaceDef kTet[4] = {{3, {1, 0, 2, -1}}, {3, {0, 1, 3, -1}}, {3, {1, 2, 3, -1}}, {3, {2, 0, 3, -1}}};
const FaceDef kPyramid[5] = {{4, {0, 2, 3, 1}}, {3, {0, 1, 4, -1}}, {3, {1, 3, 4, -1}},
                             {3, {3, 2, 4, -1}}, {3, {2, 0, 4, -1}}};

bool element_faces(int type, const FaceDef **defs, int *nf, int *nn) {
  switch (type) {
  case 4: *defs = kBrick; *nf = 6; *nn = 8; return true;
  case 5: *defs = kWedge; *nf = 5; *nn = 6; return true;
  case 6: *defs = kTet; *nf = 4; *nn = 4; return true;
  case 7: *defs = kPyramid; *nf = 5; *nn = 5; return true;
  }
  return false;
}

struct Key {
  int32_t v[4];
  bool operator==(const Key &o) const { return v[0] == o.v[0] && v[1] == o.v[1] && v[2] == o.v[2] && v[3] == o.v[3]; }
};
struct KeyHash {
  size_t operator()(const Key &k) const {
    uint64_t h = 0x9e3779b97f4a7c15ull;
    for (int q = 0; q < 4; q++) { h ^= (uint64_t)(uint32_t)k.v[q] + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2); }
    return (size_t)h;
  }
};

Key sorted_key(const int32_t *nodes, int n) {
  Key k{{-1, -1, -1, -1}};
  for (int q = 0; q < n; q++) k.v[q] = nodes[q];
  for (int a = 1; a < n; a++)   // insertion sort of at most 4 entries
    for (int b = a; b > 0 && k.v[b] < k.v[b - 1]; b--) std::swap(k.v[b], k.v[b - 1]);
  return k;
}

}  // namespace

extern "C" int fs_neu_connectivity(const fs_neu_in *in, int32_t *n_internal, int32_t *n_faces,
                                   int32_t *face_ptr, int32_t *face_nodes, int32_t *owner, int32_t *neighbour,
                                   int32_t *cell_face_ptr, int32_t *cell_faces) {
  if (!in || !n_internal || !n_faces || !face_ptr || !face_nodes || !owner || !neighbour || !cell_face_ptr || !cell_faces)
    return FS_E_ARG;
  const int NE = in->n_elements;
  // local faces per element and the slot base of each element
  std::vector<int32_t> nfe(NE);
  cell_face_ptr[0] = 0;
  for (int e = 0; e < NE; e++) {
    const FaceDef *d; int nf, nn;
    if (!element_faces(in->type[e], &d, &nf, &nn)) return FS_E_MESH;
    if (in->node_ptr[e + 1] - in->node_ptr[e] != nn) return FS_E_MESH;
    nfe[e] = nf;
    cell_face_ptr[e + 1] = cell_face_ptr[e] + nf;
  }
  const int64_t slots = cell_face_ptr[NE];
  for (int64_t q = 0; q < slots; q++) cell_faces[q] = -1;
  // boundary records: mark (element, local face); the boundary pass numbers them
  std::vector<int8_t> is_bc((size_t)slots, 0);
  int64_t nrec = 0;
  for (int s = 0; s < in->n_sets; s++) nrec += in->set_size[s];
  for (int64_t r = 0; r < nrec; r++) {
    int e = in->bc_element[r], j = in->bc_face[r];
    if (e < 0 || e >= NE || j < 0 || j >= nfe[e]) return FS_E_MESH;
    is_bc[(size_t)cell_face_ptr[e] + j] = 1;
  }
  std::unordered_map<Key, int32_t, KeyHash> table;
  table.reserve((size_t)slots);
  int32_t F = 0, q = 0;
  face_ptr[0] = 0;
  int32_t fn[4];
  for (int e = 0; e < NE; e++) {
    const FaceDef *d; int nf, nn;
    element_faces(in->type[e], &d, &nf, &nn);
    const int32_t *en = in->nodes + in->node_ptr[e];
    for (int j = 0; j < nf; j++) {
      const int64_t slot = cell_face_ptr[e] + j;
      if (is_bc[(size_t)slot]) continue;
      for (int t = 0; t < d[j].n; t++) fn[t] = en[d[j].v[t]];
      Key k = sorted_key(fn, d[j].n);
      auto it = table.find(k);
      if (it != table.end()) {   // the second side of an interior face
        int32_t f = it->second;
        if (neighbour[f] != -1) return FS_E_MESH;
        neighbour[f] = e;
        cell_faces[slot] = f;
        continue;
      }
      table.emplace(k, F);
      for (int t = 0; t < d[j].n; t++) face_nodes[q++] = fn[t];
      face_ptr[F + 1] = q;
      owner[F] = e;
      neighbour[F] = -1;
      cell_faces[slot] = F;
      F++;
    }
  }
  // interior faces all have a second side; GlobalConnectivity's owner is the
  // lower element, which made the face
  for (int32_t f = 0; f < F; f++) if (neighbour[f] < 0) return FS_E_MESH;
  int32_t nfaces = F;
  for (int64_t r = 0; r < nrec; r++) {
    int e = in->bc_element[r], j = in->bc_face[r];
    const FaceDef *d; int nf, nn;
    element_faces(in->type[e], &d, &nf, &nn);
    const int32_t *en = in->nodes + in->node_ptr[e];
    for (int t = 0; t < d[j].n; t++) face_nodes[q++] = en[d[j].v[t]];
    face_ptr[nfaces + 1] = q;
    owner[nfaces] = e;
    cell_faces[(size_t)cell_face_ptr[e] + j] = nfaces;
    nfaces++;
  }
  for (int64_t s = 0; s < slots; s++) if (cell_faces[s] < 0) return FS_E_MESH;   // a face with one side and no record
  *n_internal = F;
  *n_faces = nfaces;
  return FS_OK;
}
