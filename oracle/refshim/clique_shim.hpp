// ORACLE — test infrastructure only (the checker, never the product).
//
// Declarations that let the reference's DistHelmholtz headers
// (include/psp/dist_helmholtz.hpp and dist_helmholtz/*.hpp) compile on one
// process without Clique and Elemental, so the reference's own constructor
// (panel geometry, nested-dissection ordering and elimination trees,
// main.hpp), PML stretches and global rows (initialize_finalize.hpp:415-587)
// can run as a checker.  Only those members are instantiated.  Clique's
// symbolic analysis, factorization and solves are absent from this tree;
// their names are declared as stubs that throw if called, and the
// Elemental matrix type is a plain column-major container.
#pragma once
#include <map>
#include <stack>

#include "elem_shim.hpp"

namespace psp {

namespace mpi {
enum Op { MAX, MIN, SUM };
inline double Time() { return 0.0; }
inline bool CongruentComms(Comm, Comm) { return true; }
inline void CommDup(Comm c, Comm& d) { d = c; }
inline void CommSplit(Comm c, int, int, Comm& d) { d = c; }
template <typename T>
inline void AllReduce(const T* s, T* r, int n, Op, Comm) {
    std::copy(s, s + n, r);
}
}  // namespace mpi

[[noreturn]] inline void Unavailable(const char* what) {
    throw std::logic_error(std::string(what) + " is part of Clique/Elemental, which this checker does not have");
}

// The box of an x-y subdomain in the nested-dissection recursion (the
// reference declares it in environment.hpp with these fields).
struct Box {
    int parentIndex, nx, ny, xOffset, yOffset;
    bool leftChild;
};

enum Distribution { MC, MR, VC, VR, STAR };
enum UpperOrLower { LOWER, UPPER };
enum Orientation { NORMAL, TRANSPOSE, ADJOINT };
enum UnitOrNonUnit { NON_UNIT, UNIT };

struct Grid {
    int Row() const { return 0; }
    int Col() const { return 0; }
    int Height() const { return 1; }
    int Width() const { return 1; }
    int Size() const { return 1; }
    int VCRank() const { return 0; }
    int VRRank() const { return 0; }
};

template <typename T>
class Matrix {
public:
    Matrix(int h = 0, int w = 0) : h_(h), w_(w), ld_(std::max(h, 1)), v_((size_t)std::max(h, 1) * w) {}
    int Height() const { return h_; }
    int Width() const { return w_; }
    int LDim() const { return ld_; }
    T* Buffer(int i = 0, int j = 0) { return v_.data() + i + (size_t)j * ld_; }
    const T* LockedBuffer(int i = 0, int j = 0) const { return v_.data() + i + (size_t)j * ld_; }
    T Get(int i, int j) const { return v_[i + (size_t)j * ld_]; }
    void Set(int i, int j, T x) { v_[i + (size_t)j * ld_] = x; }
    void Update(int i, int j, T x) { v_[i + (size_t)j * ld_] += x; }
    void Resize(int h, int w) { *this = Matrix(h, w); }
    void Empty() { *this = Matrix(); }

private:
    int h_, w_, ld_;
    std::vector<T> v_;
};
template <typename T, Distribution U = MC, Distribution V = MR>
class DistMatrix : public Matrix<T> {
public:
    void SetGrid(const Grid&) {}
    void Align(int, int) {}
    int ColShift() const { return 0; }
    int RowShift() const { return 0; }
    int ColStride() const { return 1; }
    int RowStride() const { return 1; }
    int LocalHeight() const { return this->Height(); }
    int LocalWidth() const { return this->Width(); }
};
template <typename T>
struct Base_ { typedef T type; };
template <typename T>
struct Base_<std::complex<T>> { typedef T type; };
template <typename T>
using Base = typename Base_<T>::type;
using std::conj;
using std::exp;
template <typename T>
inline T Conj(const T& x) { return conj(x); }
template <typename T>
inline T Exp(const T& x) { return exp(x); }

template <typename... A>
inline void View(A&&...) { Unavailable("View"); }
template <typename... A>
inline void LockedView(A&&...) { Unavailable("LockedView"); }

namespace elem {
template <typename T>
inline void MemZero(T* p, std::size_t n) { std::fill(p, p + n, T(0)); }
template <typename... A> inline void Axpy(A&&...) { Unavailable("elem::Axpy"); }
template <typename... A> inline void MakeZeros(A&&...) { Unavailable("elem::MakeZeros"); }
template <typename... A> inline void Scal(A&&...) { Unavailable("elem::Scal"); }
template <typename... A> inline void Trsv(A&&...) { Unavailable("elem::Trsv"); }
template <typename... A> inline void Zeros(A&&...) { Unavailable("elem::Zeros"); }
namespace lapack {
template <typename... A> inline void HessenbergEig(A&&...) { Unavailable("lapack::HessenbergEig"); }
}
}  // namespace elem
namespace blas {
template <typename... A> inline void Dot(A&&...) { Unavailable("blas::Dot"); }
template <typename... A> inline void Axpy(A&&...) { Unavailable("blas::Axpy"); }
template <typename... A> inline void Scal(A&&...) { Unavailable("blas::Scal"); }
template <typename... A> inline void Nrm2(A&&...) { Unavailable("blas::Nrm2"); }
}  // namespace blas
namespace lapack {
template <typename... A> inline void ComputeGivens(A&&...) { Unavailable("lapack::ComputeGivens"); }
}

namespace cliq {
enum SymmFrontType { SYMM_1D, SYMM_2D, LDL_1D, LDL_2D, LDL_SELINV_1D, LDL_SELINV_2D };
struct SymmNode {
    int size = 0, off = 0, parent = -1;
    std::vector<int> children, lowerStruct;
};
struct DistSymmNode {
    bool onLeft = false;
    int size = 0, off = 0;
    std::vector<int> lowerStruct;
    mpi::Comm comm = 0;
};
struct DistSymmElimTree {
    std::vector<DistSymmNode> distNodes;
    std::vector<SymmNode*> localNodes;
    ~DistSymmElimTree() {
        for (SymmNode* p : localNodes) delete p;
    }
};
struct MultiVecMeta {
    int localSize = 0;
};
struct SymmNodeInfo {
    int size = 0, off = 0;
    std::vector<int> lowerStruct, origLowerStruct, origLowerRelInds;
};
struct DistSymmNodeInfo {
    int size = 0, off = 0;
    std::vector<int> lowerStruct, origLowerStruct, origLowerRelInds;
    Grid* grid = nullptr;
    MultiVecMeta multiVecMeta;
};
struct DistSymmInfo {
    std::vector<SymmNodeInfo> localNodes;
    std::vector<DistSymmNodeInfo> distNodes;
};
template <typename F>
struct SymmFront {
    Matrix<F> frontL;
};
template <typename F>
struct DistSymmFront {
    Matrix<F> front;
};
template <typename F>
struct DistSymmFrontTree {
    bool isHermitian = false;
    SymmFrontType frontType = LDL_1D;
    std::vector<SymmFront<F>> localFronts;
    std::vector<DistSymmFront<F>> distFronts;
};
template <typename F>
struct DistNodalMultiVec {};
// The symbolic analysis is Clique's and is not reproduced; the stand-in
// records the elimination trees the reference built for it (one per call:
// bottom, leftover inner when there is one, top), so the checker can compare
// them.
inline std::vector<std::vector<SymmNode>>& RecordedTrees() {
    static std::vector<std::vector<SymmNode>> trees;
    return trees;
}
inline void SymmetricAnalysis(const DistSymmElimTree& eTree, DistSymmInfo&, bool) {
    std::vector<SymmNode> t;
    for (const SymmNode* n : eTree.localNodes) t.push_back(*n);
    RecordedTrees().push_back(t);
}
template <typename... A> inline void InitializeDistLeaf(A&&...) { Unavailable("cliq::InitializeDistLeaf"); }
template <typename... A> inline void LDL(A&&...) { Unavailable("cliq::LDL"); }
template <typename... A> inline void Solve(A&&...) { Unavailable("cliq::Solve"); }
template <typename... A> inline void SparseAllToAll(A&&...) { Unavailable("cliq::SparseAllToAll"); }
}  // namespace cliq

}  // namespace psp
