// TEST INFRASTRUCTURE ONLY — never part of the product path.
//
// The reference's own multi-level glue on a static hierarchy: its
// TopologyManager and Tree build the tree (refining the nodes that hold finer
// leaves), its Averager fills every refined node with the conservative
// average of its children (Averager::AverageMaterial, multiresolution/
// averager.cpp:62), and its InternalHaloManager fills every node's halos level
// by level, coarse to fine: same-level neighbours copied, jump halos predicted
// from the parent (UpdateMaterialJumpNoMpi, communication/
// internal_halo_manager.cpp:230-290). It runs on one rank against the
// single-rank MPI stand-in oracle/mpi_shim/mpi.h; oracle/Makefile compiles it
// with the reference's sources, read in place. Tests compare the leaves' face
// halos with the restatement's (oracle_level_halos) bit for bit.
#include "communication/communication_manager.h"
#include "communication/internal_halo_manager.h"
#include "multiresolution/averager.h"
#include "topology/id_information.h"
#include "topology/topology_manager.h"
#include "topology/tree.h"

#include <algorithm>
#include <cstring>
#include <set>
#include <string>
#include <vector>

namespace {

constexpr unsigned NE = MF::ANOE();
constexpr std::size_t CELLS = std::size_t(CC::TCX()) * CC::TCY() * CC::TCZ();
constexpr MaterialName kMat = MaterialName::MaterialOne;
std::string g_error;

// The node of level l at position c (in units of level-l nodes): level-zero
// nodes follow each other through the neighbour functions from IdSeed, a
// child is its parent's id with its octant (bit d: high half along d) appended.
nid_t IdOf(int l, int const c[3]) {
  if (l == 0) {
    nid_t id = IdSeed();
    for (int i = 0; i < c[0]; ++i) id = EastNeighborOfNodeWithId(id);
    for (int j = 0; j < c[1]; ++j) id = NorthNeighborOfNodeWithId(id);
    for (int k = 0; k < c[2]; ++k) id = TopNeighborOfNodeWithId(id);
    return id;
  }
  int const p[3] = {c[0] >> 1, c[1] >> 1, c[2] >> 1};
  nid_t const octant = (nid_t)((c[0] & 1) | ((c[1] & 1) << 1) | ((c[2] & 1) << 2));
  return (IdOf(l - 1, p) << 3) | octant;
}

}  // namespace

extern "C" {

char const *glue_last_error() { return g_error.c_str(); }

// u [nleaf][NE][TCX][TCY][TCZ]: the leaves' states (interiors read); on return
// every leaf's buffer as the reference's glue leaves it, halos included.
// level / coord: each leaf's level and position in units of that level's
// nodes; n0: level-zero nodes per dimension. Returns 0, or -1 with
// glue_last_error() set.
int glue_level_halos(double *u, int nleaf, int const *level, int const *coord, int const *n0) {
  try {
    int maxlev = 0;
    for (int b = 0; b < nleaf; ++b) maxlev = std::max(maxlev, level[b]);
    TopologyManager topology({(unsigned)n0[0], (unsigned)n0[1], (unsigned)n0[2]},
                             (unsigned)maxlev, 0);
    // the ancestors of every leaf are refined, coarsest first
    std::vector<std::set<nid_t>> refined(maxlev + 1);
    for (int b = 0; b < nleaf; ++b)
      for (int l = 0; l < level[b]; ++l) {
        int const s = level[b] - l;
        int const c[3] = {coord[3 * b] >> s, coord[3 * b + 1] >> s, coord[3 * b + 2] >> s};
        refined[l].insert(IdOf(l, c));
      }
    for (int l = 0; l < maxlev; ++l) {
      for (nid_t const id : refined[l]) topology.RefineNodeWithId(id);
      topology.UpdateTopology();
    }
    for (nid_t const id : topology.LocalIds()) topology.AddMaterialToNode(id, kMat);
    topology.UpdateTopology();

    Tree tree(topology, (unsigned)maxlev, 1.0);
    for (nid_t const id : topology.IdsOnLevel(0)) tree.CreateNode(id, {kMat});
    for (int l = 0; l < maxlev; ++l)
      for (nid_t const id : refined[l]) tree.RefineNode(id);
    std::vector<nid_t> leaf_id(nleaf);
    for (int b = 0; b < nleaf; ++b) {
      leaf_id[b] = IdOf(level[b], &coord[3 * b]);
      if (!topology.NodeIsLeaf(leaf_id[b]))
        throw std::invalid_argument("leaf " + std::to_string(b) + " is not a leaf of the tree");
      Block &blk = tree.GetNodeWithId(leaf_id[b]).GetPhaseByMaterial(kMat);
      for (unsigned e = 0; e < NE; ++e)
        std::memcpy(&blk.GetRightHandSideBuffer(MF::ASOE()[e])[0][0][0],
                    u + (std::size_t(b) * NE + e) * CELLS, CELLS * sizeof(double));
    }

    CommunicationManager communication(topology, (unsigned)maxlev);
    for (int l = 0; l <= maxlev; ++l) communication.GenerateNeighborRelationForHaloUpdate(l);
    std::vector<unsigned> descending;
    for (int l = maxlev; l >= 0; --l) descending.push_back((unsigned)l);
    Averager(topology, communication, tree).AverageMaterial(descending);
    InternalHaloManager halos(tree, topology, communication, 1);
    for (int l = 0; l <= maxlev; ++l)
      halos.MaterialHaloUpdateOnLevel((unsigned)l, MaterialFieldType::Conservatives, false);

    for (int b = 0; b < nleaf; ++b) {
      Block const &blk = tree.GetNodeWithId(leaf_id[b]).GetPhaseByMaterial(kMat);
      for (unsigned e = 0; e < NE; ++e)
        std::memcpy(u + (std::size_t(b) * NE + e) * CELLS,
                    &blk.GetRightHandSideBuffer(MF::ASOE()[e])[0][0][0], CELLS * sizeof(double));
    }
  } catch (std::exception const &e) {
    g_error = e.what();
    return -1;
  }
  return 0;
}

}  // extern "C"
