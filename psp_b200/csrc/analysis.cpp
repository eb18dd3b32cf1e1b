#include "analysis.hpp"

#include <algorithm>
#include <numeric>

namespace psp_b200 {

// ------------------------------------------------------------ panel geometry

void PanelGeometry::Init(const DiscParams& d, int P) {
    nx = d.nx; ny = d.ny; nz = d.nz; bz = d.bz; planesPerPanel = P;
    if (P <= 0) throw std::logic_error("numPlanesPerPanel must be positive");
    bottomDepth = bz + P;
    topOrigDepth = (d.topBC == kPML) ? bz + P : P;
    if (nz <= bottomDepth + topOrigDepth)
        throw std::logic_error(
            "The domain is very shallow. Please run a sparse-direct factorization instead.");
    innerDepth = nz - (bottomDepth + topOrigDepth);
    leftoverDepth = innerDepth % P;
    haveLeftover = leftoverDepth != 0;
    numFullInner = innerDepth / P;
    numPanels = 1 + numFullInner + (haveLeftover ? 1 : 0) + 1;
}

int PanelGeometry::Depth(int p) const {
    if (p == 0) return bottomDepth;
    if (p < 1 + numFullInner) return planesPerPanel;
    if (haveLeftover && p == 1 + numFullInner) return leftoverDepth;
    return topOrigDepth;
}

int PanelGeometry::LowV(int p) const {
    if (p == 0) return 0;
    if (p < 1 + numFullInner) return bottomDepth + planesPerPanel * (p - 1);
    if (haveLeftover && p == 1 + numFullInner) return bottomDepth + planesPerPanel * numFullInner;
    return bottomDepth + planesPerPanel * numFullInner + leftoverDepth;
}

int PanelGeometry::Class(int p) const {
    if (p < 1 + numFullInner) return 0;
    if (haveLeftover && p == 1 + numFullInner) return 1;
    return 2;
}

int PanelGeometry::ClassVSize(int c) const {
    if (c == 0) return bottomDepth;          // bottom (no padding) and full inner (bz + P)
    if (c == 1) return leftoverDepth + bz;
    return topOrigDepth + bz;
}

// ------------------------------------------------------------ x-y dissection

namespace {

struct TreeBuilder {
    XYTree& T;
    int Visit(int xOff, int yOff, int bnx, int bny, int depth) {
        XYNode node;
        node.xOff = xOff; node.yOff = yOff; node.bnx = bnx; node.bny = bny;
        node.depth = depth;
        T.maxDepth = std::max(T.maxDepth, depth);
        if (bnx * bny <= T.cutoff) {
            node.leaf = true;
            node.count = bnx * bny;
        } else if (bnx >= bny) {
            const int mid = (bnx - 1) / 2;
            node.cutX = true;
            node.child[0] = Visit(xOff, yOff, mid, bny, depth + 1);
            node.child[1] = Visit(xOff + mid + 1, yOff, bnx - mid - 1, bny, depth + 1);
            node.numChildren = 2;
            node.count = bny;
        } else {
            const int mid = (bny - 1) / 2;
            node.cutX = false;
            node.child[0] = Visit(xOff, yOff, bnx, mid, depth + 1);
            node.child[1] = Visit(xOff, yOff + mid + 1, bnx, bny - mid - 1, depth + 1);
            node.numChildren = 2;
            node.count = bnx;
        }
        T.nodes.push_back(node);
        const int me = (int)T.nodes.size() - 1;
        for (int c = 0; c < node.numChildren; ++c) T.nodes[node.child[c]].parent = me;
        return me;
    }
};

void SortedUnion(std::vector<int>& acc, const std::vector<int>& add) {
    std::vector<int> out;
    out.reserve(acc.size() + add.size());
    std::set_union(acc.begin(), acc.end(), add.begin(), add.end(), std::back_inserter(out));
    acc.swap(out);
}

}  // namespace

int XYTree::PointXY(int t, int q) const {
    const XYNode& n = nodes[t];
    int x, y;
    if (n.leaf) { x = n.xOff + q % n.bnx; y = n.yOff + q / n.bnx; }
    else if (n.cutX) { x = n.xOff + (n.bnx - 1) / 2; y = n.yOff + q; }
    else { x = n.xOff + q; y = n.yOff + (n.bny - 1) / 2; }
    return x + y * nx;
}

void XYTree::Build(int nx_, int ny_, int cutoff_) {
    nx = nx_; ny = ny_; cutoff = cutoff_;
    nodes.clear();
    maxDepth = 0;
    TreeBuilder b{*this};
    b.Visit(0, 0, nx, ny, 0);
    int prefix = 0;
    pointNode.assign((size_t)nx * ny, -1);
    pointRank.assign((size_t)nx * ny, -1);
    for (size_t t = 0; t < nodes.size(); ++t) {
        nodes[t].prefix = prefix;
        prefix += nodes[t].count;
        for (int q = 0; q < nodes[t].count; ++q) {
            const int xy = PointXY((int)t, q);
            pointNode[xy] = (int)t;
            pointRank[xy] = q;
        }
    }
    if (prefix != nx * ny) throw std::logic_error("x-y dissection does not cover the plane");
    // 2-D fill structure, children before parents (postorder).
    for (size_t t = 0; t < nodes.size(); ++t) {
        XYNode& n = nodes[t];
        std::vector<int> orig;
        if (n.leaf) {
            if (n.xOff > 0)
                for (int j = 0; j < n.bny; ++j) orig.push_back((n.xOff - 1) + (n.yOff + j) * nx);
            if (n.xOff + n.bnx < nx)
                for (int j = 0; j < n.bny; ++j) orig.push_back((n.xOff + n.bnx) + (n.yOff + j) * nx);
            if (n.yOff > 0)
                for (int i = 0; i < n.bnx; ++i) orig.push_back((n.xOff + i) + (n.yOff - 1) * nx);
            if (n.yOff + n.bny < ny)
                for (int i = 0; i < n.bnx; ++i) orig.push_back((n.xOff + i) + (n.yOff + n.bny) * nx);
        } else if (n.cutX) {
            const int x = n.xOff + (n.bnx - 1) / 2;
            if (n.yOff > 0) orig.push_back(x + (n.yOff - 1) * nx);
            if (n.yOff + n.bny < ny) orig.push_back(x + (n.yOff + n.bny) * nx);
        } else {
            const int y = n.yOff + (n.bny - 1) / 2;
            if (n.xOff > 0) orig.push_back((n.xOff - 1) + y * nx);
            if (n.xOff + n.bnx < nx) orig.push_back((n.xOff + n.bnx) + y * nx);
        }
        std::sort(orig.begin(), orig.end());
        std::vector<int> acc = orig;
        for (int c = 0; c < n.numChildren; ++c) SortedUnion(acc, nodes[n.child[c]].xyStruct);
        n.xyStruct.clear();
        for (int p : acc)
            if (pointNode[p] != (int)t) n.xyStruct.push_back(p);
    }
}

// ------------------------------------------------------------ panel classes

void ClassStructure::Build(const XYTree& T, int vs) {
    vSize = vs;
    const int nx = T.nx, ny = T.ny, nxy = nx * ny;
    const int numNodes = (int)T.nodes.size();
    nSub = nxy * vSize;
    off.resize(numNodes); size.resize(numNodes); usize.resize(numNodes);
    lowerOff.resize(numNodes + 1);
    for (int t = 0; t < numNodes; ++t) {
        off[t] = T.nodes[t].prefix * vSize;
        size[t] = T.nodes[t].count * vSize;
        usize[t] = (int)T.nodes[t].xyStruct.size() * vSize;
    }
    auto nd = [&](int xy, int v) {
        const int t = T.pointNode[xy];
        return off[t] + T.pointRank[xy] + v * T.nodes[t].count;
    };
    ndToNat.assign(nSub, 0);
    natToNd.assign(nSub, 0);
    for (int v = 0; v < vSize; ++v)
        for (int xy = 0; xy < nxy; ++xy) {
            const int i = nd(xy, v);
            ndToNat[i] = xy + v * nxy;
            natToNd[xy + v * nxy] = i;
        }
    lowerOff[0] = 0;
    for (int t = 0; t < numNodes; ++t) lowerOff[t + 1] = lowerOff[t] + usize[t];
    lower.assign(lowerOff[numNodes], 0);
    rel.assign(lowerOff[numNodes], 0);
    for (int t = 0; t < numNodes; ++t) {
        int* L = lower.data() + lowerOff[t];
        int k = 0;
        for (int xy : T.nodes[t].xyStruct)
            for (int v = 0; v < vSize; ++v) L[k++] = nd(xy, v);
        std::sort(L, L + k);
    }
    auto frontRow = [&](int t, int idx) -> int {
        if (idx < off[t] + size[t]) return idx - off[t];
        const int* L = lower.data() + lowerOff[t];
        const int* it = std::lower_bound(L, L + usize[t], idx);
        if (it == L + usize[t] || *it != idx) throw std::logic_error("index missing from front structure");
        return size[t] + int(it - L);
    };
    for (int t = 0; t < numNodes; ++t) {
        const int p = T.nodes[t].parent;
        if (p < 0) continue;
        for (int a = 0; a < usize[t]; ++a) rel[lowerOff[t] + a] = frontRow(p, lower[lowerOff[t] + a]);
    }
    nbrRows.assign((size_t)nSub * 6, -1);
    for (int t = 0; t < numNodes; ++t) {
        for (int j = 0; j < size[t]; ++j) {
            const int col = off[t] + j;
            const int pn = ndToNat[col];
            const int xy = pn % nxy, v = pn / nxy, x = xy % nx, y = xy / nx;
            int* rows = nbrRows.data() + (size_t)col * 6;
            auto put = [&](int slot, int nxy2, int v2) {
                const int idx = nd(nxy2, v2);
                if (idx > col) rows[slot] = frontRow(t, idx);
            };
            if (x > 0) put(0, xy - 1, v);
            if (x + 1 < nx) put(1, xy + 1, v);
            if (y > 0) put(2, xy - nx, v);
            if (y + 1 < ny) put(3, xy + nx, v);
            if (v > 0) put(4, xy, v - 1);
            if (v + 1 < vSize) put(5, xy, v + 1);
        }
    }
}

int64_t ClassStructure::FactorEntries() const {
    int64_t s = 0;
    for (size_t t = 0; t < off.size(); ++t) s += (int64_t)(size[t] + usize[t]) * size[t];
    return s;
}

int64_t ClassStructure::UpdateEntries() const {
    int64_t s = 0;
    for (size_t t = 0; t < off.size(); ++t) s += (int64_t)usize[t] * usize[t];
    return s;
}

void Analysis::Build(const DiscParams& d, int planesPerPanel, int cutoff) {
    disc = d;
    if (cutoff < 1) throw std::logic_error("cutoff must be positive");
    if (d.nx < 1 || d.ny < 1) throw std::logic_error("grid must be non-empty");
    geom.Init(d, planesPerPanel);
    tree.Build(d.nx, d.ny, cutoff);
    for (int c = 0; c < 3; ++c) classUsed[c] = false;
    for (int p = 0; p < geom.numPanels; ++p) classUsed[geom.Class(p)] = true;
    for (int c = 0; c < 3; ++c)
        if (classUsed[c]) cls[c].Build(tree, geom.ClassVSize(c));
}

}  // namespace psp_b200
