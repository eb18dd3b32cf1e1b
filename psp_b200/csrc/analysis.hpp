// Host-side symbolic analysis of the moving-PML sweeping preconditioner.
//
// Geometry of the z-panels (PSP main.hpp:12-57, 728-821), the x-y nested
// dissection shared by every panel (main.hpp:1423-1477, 1709-1900) and the
// multifrontal fill structure that Clique's SymmetricAnalysis derives from it
// (called at main.hpp:432-435).
//
// Formulation: the dissection only cuts the x-y plane and every node owns
// whole columns of `vSize` planes, so the tree, the ND offsets and the fill
// structure are computed once in 2-D and expanded by the plane count of each
// panel class.  A node owning `c` x-y points holds the ND indices
// off + q + vLocal*c (q = point rank inside the node, leaf points x-fastest,
// separator points along the cut line), which reproduces ReorderedIndex.
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace psp_b200 {

enum BoundaryKind { kPML = 0, kDirichlet = 1 };

struct DiscParams {
    double omega;
    int nx, ny, nz;
    double wx, wy, wz;
    int frontBC, rightBC, backBC, leftBC, topBC;
    int bx, by, bz;
    double sigmax, sigmay, sigmaz;
};

// Panel split of the sweep direction (main.hpp:12-57).  "v" is the sweep
// coordinate, v = nz-1-z.
struct PanelGeometry {
    int nx = 0, ny = 0, nz = 0, bz = 0, planesPerPanel = 0;
    int bottomDepth = 0, topOrigDepth = 0, innerDepth = 0, leftoverDepth = 0;
    int numFullInner = 0, numPanels = 0;
    bool haveLeftover = false;

    void Init(const DiscParams& d, int planesPerPanel);
    int Padding(int p) const { return p == 0 ? 0 : bz; }           // main.hpp:728-738
    int Depth(int p) const;                                         // main.hpp:740-752
    int LowV(int p) const;                                          // main.hpp:779-793
    int Class(int p) const;                                         // main.hpp:705-726
    int ClassVSize(int c) const;
    int SubVOffset(int p) const { return LowV(p) - Padding(p); }    // first plane of the padded subproblem
};

// One node of the x-y dissection tree.
struct XYNode {
    int xOff = 0, yOff = 0, bnx = 0, bny = 0;
    bool leaf = false;
    bool cutX = false;        // separator is the column x = xOff + (bnx-1)/2
    int parent = -1;
    int child[2] = {-1, -1};
    int numChildren = 0;
    int depth = 0;            // root = 0
    int count = 0;            // x-y points owned by the node
    int prefix = 0;           // x-y points owned by the nodes before it in postorder
    std::vector<int> xyStruct; // 2-D fill structure: natural x-y indices in ancestors
};

struct XYTree {
    int nx = 0, ny = 0, cutoff = 0;
    std::vector<XYNode> nodes;   // postorder: left subtree, right subtree, node
    int maxDepth = 0;
    std::vector<int> pointNode;  // x-y natural index -> owning node
    std::vector<int> pointRank;  // x-y natural index -> rank q inside its node

    void Build(int nx, int ny, int cutoff);
    int PointXY(int node, int q) const;  // inverse of (pointNode, pointRank)
};

// The tree expanded to one panel class (vSize planes per column).
struct ClassStructure {
    int vSize = 0;
    int nSub = 0;                          // nx*ny*vSize
    std::vector<int> off, size, usize;     // per node
    std::vector<int64_t> lowerOff;         // per node offset into `lower` / `rel`
    std::vector<int> lower;                // concatenated sorted fill structures (ND indices)
    std::vector<int> rel;                  // each lower entry's row in the parent's front
    std::vector<int> ndToNat;              // ND index -> x + y*nx + vLocal*nx*ny
    std::vector<int> natToNd;
    // For each ND column index: front rows of its 6 lower-triangle stencil
    // neighbours in the order x-, x+, y-, y+, v-, v+ (-1 when absent or not in
    // the lower triangle).
    std::vector<int> nbrRows;

    void Build(const XYTree& tree, int vSize);
    int64_t FactorEntries() const;         // sum (s+u)*s
    int64_t UpdateEntries() const;         // sum u*u
};

struct Analysis {
    DiscParams disc{};
    PanelGeometry geom;
    XYTree tree;
    ClassStructure cls[3];
    bool classUsed[3] = {false, false, false};

    void Build(const DiscParams& d, int planesPerPanel, int cutoff);
};

}  // namespace psp_b200
