// ORACLE — test infrastructure only (the checker, never the product).
//
// A one-process stand-in for the parts of Clique and Elemental that the
// reference's headers use, found by the reference's own
// include/psp/environment.hpp through its `#include "clique.hpp"`, so that
// the reference's psp.hpp (environment, Discretization, DistUniformGrid,
// DistHelmholtz) compiles unchanged from the reference tree and runs as a
// checker on one process.
//
// * MPI on one rank: every collective copies rank 0's send buffer into its
//   receive buffer.
// * Elemental's dense types and kernels the PSP code calls: a column-major
//   Matrix with owning storage or views, Zeros / MakeZeros / Axpy / Scal,
//   the upper-triangular Trsv of the GMRES least-squares update, Nrm2, the
//   conjugated Dot, and ComputeGivens with LAPACK zlartg's convention
//   (c real, [c s; -conj(s) c] [f; g] = [r; 0]).
// * Clique: its tree and front types as plain structs.  Its symbolic
//   analysis records the elimination trees the reference hands it and
//   computes the node structures from them (restating Clique's published
//   symbolic factorization), which the reference's panel assembly and panel
//   solve read.  Clique's multifrontal factorization and solve are not in the
//   reference tree: LDL throws, and Solve calls a panel solver that the
//   harness installs (the oracle's, oracle/psp_oracle.cpp), so the
//   reference's sweep and GMRES run around it.
#pragma once
#include <sys/stat.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <fstream>
#include <functional>
#include <initializer_list>
#include <iostream>
#include <map>
#include <set>
#include <sstream>
#include <stack>
#include <stdexcept>
#include <string>
#include <vector>

#ifndef RELEASE
#define RELEASE
#endif
#define DEBUG_ONLY(cmd)
// psp/environment.hpp includes these two Elemental headers by macro.
#define ELEM_MAXNORM_INC "empty.hpp"
#define ELEM_SVD_INC "empty.hpp"

namespace elem {

template <typename R>
using Complex = std::complex<R>;

template <typename T>
struct BaseOf { typedef T type; };
template <typename T>
struct BaseOf<std::complex<T>> { typedef T type; };
template <typename T>
using Base = typename BaseOf<T>::type;

template <typename... Args>
inline std::string Message(const Args&... args) {
    std::ostringstream os;
    (void)std::initializer_list<int>{((os << args), 0)...};
    return os.str();
}
template <typename... Args>
[[noreturn]] inline void LogicError(const Args&... args) { throw std::logic_error(Message(args...)); }
template <typename... Args>
[[noreturn]] inline void RuntimeError(const Args&... args) { throw std::runtime_error(Message(args...)); }
struct ArgException : std::logic_error {
    ArgException() : std::logic_error("argument error") {}
};
template <typename T>
inline T Input(const std::string&, const std::string&, T dflt) { return dflt; }
inline void ProcessInput() {}

// Local length of an n-entry dimension dealt cyclically to `stride`
// processes, on the process with offset `shift` (or with rank `rank` when
// rank `firstRank` holds entry 0).
inline int Shift(int rank, int firstRank, int stride) { return (rank - firstRank + stride) % stride; }
inline int Length(int n, int shift, int stride) { return n > shift ? (n - shift - 1) / stride + 1 : 0; }
inline int Length(int n, int rank, int firstRank, int stride) { return Length(n, Shift(rank, firstRank, stride), stride); }

template <typename T>
inline void SwapClear(T& x) {
    T().swap(x);
}
template <typename T>
inline void MemCopy(T* dest, const T* src, std::size_t n) {
    std::copy(src, src + n, dest);
}
template <typename T>
inline void MemZero(T* p, std::size_t n) {
    std::fill(p, p + n, T(0));
}

template <typename T>
inline Base<T> Abs(const T& x) { return std::abs(x); }
inline double Abs(double x) { return std::fabs(x); }
template <typename T>
inline T Conj(const T& x) { return x; }
template <typename R>
inline std::complex<R> Conj(const std::complex<R>& x) { return std::conj(x); }
template <typename T>
inline T Exp(const T& x) { return std::exp(x); }

namespace unit_or_non_unit_wrapper { enum UnitOrNonUnit { NON_UNIT, UNIT }; }
namespace distribution_wrapper { enum Distribution { MC, MD, MR, VC, VR, STAR, CIRC }; }
namespace orientation_wrapper { enum Orientation { NORMAL, TRANSPOSE, ADJOINT }; }
namespace upper_or_lower_wrapper { enum UpperOrLower { LOWER, UPPER }; }
namespace left_or_right_wrapper { enum LeftOrRight { LEFT, RIGHT }; }
namespace vertical_or_horizontal_wrapper { enum VerticalOrHorizontal { VERTICAL, HORIZONTAL }; }
namespace forward_or_backward_wrapper { enum ForwardOrBackward { FORWARD, BACKWARD }; }
namespace conjugation_wrapper { enum Conjugation { UNCONJUGATED, CONJUGATED }; }
using namespace unit_or_non_unit_wrapper;
using namespace distribution_wrapper;
using namespace orientation_wrapper;
using namespace upper_or_lower_wrapper;

struct Grid {
    int Row() const { return 0; }
    int Col() const { return 0; }
    int Height() const { return 1; }
    int Width() const { return 1; }
    int Size() const { return 1; }
    int VCRank() const { return 0; }
    int VRRank() const { return 0; }
};

// Column-major matrix: owning storage, or a view into another matrix's.
template <typename T>
class Matrix {
public:
    Matrix() : h_(0), w_(0), ld_(1), p_(nullptr) {}
    Matrix(int h, int w) { Own(h, w, std::max(h, 1)); }
    Matrix(int h, int w, int ld) { Own(h, w, std::max(ld, std::max(h, 1))); }
    Matrix(const Matrix& o) : Matrix(o.h_, o.w_) { CopyFrom(o); }
    Matrix& operator=(const Matrix& o) {
        if (this != &o) {
            if (view_) {
                if (o.h_ != h_ || o.w_ != w_) LogicError("assignment to a view of another shape");
            } else if (o.h_ != h_ || o.w_ != w_ || !p_) {
                Own(o.h_, o.w_, std::max(o.h_, 1));
            }
            CopyFrom(o);
        }
        return *this;
    }
    int Height() const { return h_; }
    int Width() const { return w_; }
    int LDim() const { return ld_; }
    T* Buffer(int i = 0, int j = 0) { return p_ + i + (size_t)j * ld_; }
    const T* LockedBuffer(int i = 0, int j = 0) const { return p_ + i + (size_t)j * ld_; }
    T Get(int i, int j) const { return p_[i + (size_t)j * ld_]; }
    void Set(int i, int j, T x) { p_[i + (size_t)j * ld_] = x; }
    void Update(int i, int j, T x) { p_[i + (size_t)j * ld_] += x; }
    void Resize(int h, int w) { Resize(h, w, std::max(h, 1)); }
    void Resize(int h, int w, int ld) {
        if (view_) LogicError("resizing a view");
        Own(h, w, std::max(ld, std::max(h, 1)));
    }
    void Empty() { *this = Matrix(); }
    // The h x w block of `from` at (i, j), shared.
    void AttachView(const Matrix& from, int i, int j, int h, int w) {
        store_.clear();
        view_ = true;
        h_ = h;
        w_ = w;
        ld_ = from.ld_;
        p_ = const_cast<T*>(from.LockedBuffer(i, j));
    }

private:
    void Own(int h, int w, int ld) {
        view_ = false;
        h_ = h;
        w_ = w;
        ld_ = ld;
        store_.assign((size_t)ld * w, T(0));
        p_ = store_.data();
    }
    void CopyFrom(const Matrix& o) {
        for (int j = 0; j < w_; ++j) std::copy(o.LockedBuffer(0, j), o.LockedBuffer(0, j) + h_, Buffer(0, j));
    }
    int h_, w_, ld_;
    T* p_;
    bool view_ = false;
    std::vector<T> store_;
};

template <typename T, Distribution U = MC, Distribution V = MR>
class DistMatrix : public Matrix<T> {
public:
    void SetGrid(const Grid&) {}
    void Align(int, int) {}
    int LocalHeight() const { return this->Height(); }
    int LocalWidth() const { return this->Width(); }
    void SetLocal(int i, int j, T x) { this->Set(i, j, x); }
};

template <typename T>
inline void View(Matrix<T>& A, Matrix<T>& B, int i, int j, int h, int w) { A.AttachView(B, i, j, h, w); }
template <typename T>
inline void LockedView(Matrix<T>& A, const Matrix<T>& B, int i, int j, int h, int w) { A.AttachView(B, i, j, h, w); }
template <typename T>
inline void MakeZeros(Matrix<T>& A) {
    for (int j = 0; j < A.Width(); ++j) std::fill(A.Buffer(0, j), A.Buffer(0, j) + A.Height(), T(0));
}
template <typename T>
inline void Zeros(Matrix<T>& A, int h, int w) {
    A.Resize(h, w);
    MakeZeros(A);
}
// Y := alpha X + Y
template <typename T, typename S>
inline void Axpy(S alpha, const Matrix<T>& X, Matrix<T>& Y) {
    for (int j = 0; j < X.Width(); ++j)
        for (int i = 0; i < X.Height(); ++i) Y.Update(i, j, T(alpha) * X.Get(i, j));
}
template <typename T, typename S>
inline void Scal(S alpha, Matrix<T>& X) {
    for (int j = 0; j < X.Width(); ++j)
        for (int i = 0; i < X.Height(); ++i) X.Set(i, j, T(alpha) * X.Get(i, j));
}
// x := inv(A) x for upper-triangular A with its diagonal (back substitution).
template <typename T>
inline void Trsv(UpperOrLower uplo, Orientation orient, UnitOrNonUnit diag, const Matrix<T>& A, Matrix<T>& x) {
    if (uplo != UPPER || orient != NORMAL || diag != NON_UNIT) LogicError("only the upper, normal, non-unit Trsv");
    const int n = A.Height();
    for (int i = n - 1; i >= 0; --i) {
        T s = x.Get(i, 0);
        for (int q = i + 1; q < n; ++q) s -= A.Get(i, q) * x.Get(q, 0);
        x.Set(i, 0, s / A.Get(i, i));
    }
}

namespace blas {
template <typename T>
inline Base<T> Nrm2(int n, const T* x, int inc) {
    Base<T> s = 0;
    for (int i = 0; i < n; ++i) s += std::norm(x[(size_t)i * inc]);
    return std::sqrt(s);
}
inline double Nrm2(int n, const double* x, int inc) {
    double s = 0;
    for (int i = 0; i < n; ++i) s += x[(size_t)i * inc] * x[(size_t)i * inc];
    return std::sqrt(s);
}
// Conjugated dot product x^H y.
template <typename T>
inline T Dot(int n, const T* x, int incx, const T* y, int incy) {
    T s = 0;
    for (int i = 0; i < n; ++i) s += Conj(x[(size_t)i * incx]) * y[(size_t)i * incy];
    return s;
}
}  // namespace blas

namespace lapack {
// The rotation [c s; -conj(s) c] with c real that maps (f, g) to (r, 0).
template <typename R>
inline void ComputeGivens(const std::complex<R>& f, const std::complex<R>& g, R* c, std::complex<R>* s,
                          std::complex<R>* r) {
    const R af = std::abs(f), ag = std::abs(g);
    if (ag == 0) {
        *c = 1;
        *s = 0;
        *r = f;
    } else if (af == 0) {
        *c = 0;
        *s = std::conj(g) / ag;
        *r = ag;
    } else {
        const R nrm = std::hypot(af, ag);
        const std::complex<R> phase = f / af;
        *c = af / nrm;
        *s = phase * std::conj(g) / nrm;
        *r = phase * nrm;
    }
}
template <typename... A>
inline void HessenbergEig(A&&...) {
    LogicError("HessenbergEig is not part of this checker");
}
}  // namespace lapack

namespace mpi {
typedef int Comm;
enum Op { MAX, MIN, SUM };
inline int CommRank(Comm) { return 0; }
inline int CommSize(Comm) { return 1; }
inline void Barrier(Comm) {}
inline double Time() { return 0.0; }
inline bool CongruentComms(Comm, Comm) { return true; }
inline void CommDup(Comm c, Comm& d) { d = c; }
inline void CommSplit(Comm c, int, int, Comm& d) { d = c; }
inline void CommFree(Comm&) {}
template <typename T>
inline void AllToAll(const T* sbuf, int sc, T* rbuf, int rc, Comm) {
    if (sc != rc) LogicError("one-rank AllToAll with unequal counts");
    std::copy(sbuf, sbuf + sc, rbuf);
}
template <typename T>
inline void AllToAll(const T* sbuf, const int* scs, const int* sds, T* rbuf, const int* rcs, const int* rds, Comm) {
    if (scs[0] != rcs[0]) LogicError("one-rank AllToAll with unequal counts");
    std::copy(sbuf + sds[0], sbuf + sds[0] + scs[0], rbuf + rds[0]);
}
template <typename T>
inline void Gather(const T* sbuf, int sc, T* rbuf, const int* rcs, const int* rds, int root, Comm) {
    if (root != 0 || sc != rcs[0]) LogicError("one-rank Gather with unequal counts");
    std::copy(sbuf, sbuf + sc, rbuf + rds[0]);
}
template <typename T>
inline void Gather(const T* sbuf, int sc, T* rbuf, int rc, int root, Comm) {
    if (root != 0 || sc != rc) LogicError("one-rank Gather with unequal counts");
    std::copy(sbuf, sbuf + sc, rbuf);
}
template <typename T>
inline void AllGather(const T* sbuf, int sc, T* rbuf, int rc, Comm) {
    if (sc != rc) LogicError("one-rank AllGather with unequal counts");
    std::copy(sbuf, sbuf + sc, rbuf);
}
template <typename T>
inline void AllReduce(const T* sbuf, T* rbuf, int n, Op, Comm) {
    std::copy(sbuf, sbuf + n, rbuf);
}
}  // namespace mpi

}  // namespace elem

#define MPI_SUM elem::mpi::SUM

namespace cliq {

using elem::Matrix;
enum SymmFrontType { SYMM_1D, SYMM_2D, LDL_1D, LDL_2D, LDL_SELINV_1D, LDL_SELINV_2D };

struct SymmNode {
    int size = 0, off = 0, parent = -1;
    std::vector<int> children, lowerStruct;
};
struct DistSymmNode {
    bool onLeft = false;
    int size = 0, off = 0;
    std::vector<int> lowerStruct;
    elem::mpi::Comm comm = 0;
};
struct DistSymmElimTree {
    std::vector<DistSymmNode> distNodes;
    std::vector<SymmNode*> localNodes;
    DistSymmElimTree() = default;
    DistSymmElimTree(const DistSymmElimTree&) = delete;
    DistSymmElimTree& operator=(const DistSymmElimTree&) = delete;
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
    elem::Grid* grid = nullptr;
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
    elem::DistMatrix<F> front, front2dL;
};
template <typename F>
struct DistSymmFrontTree {
    bool isHermitian = false;
    SymmFrontType frontType = LDL_1D;
    std::vector<SymmFront<F>> localFronts;
    std::vector<DistSymmFront<F>> distFronts;
};
// Right-hand sides of one panel, node by node in the panel's elimination
// order (nodes of one rank only here).
template <typename F>
struct DistNodalMultiVec {
    std::vector<Matrix<F>> localNodes;
    std::vector<elem::DistMatrix<F, elem::VC, elem::STAR>> distNodes;
    void UpdateHeight() {}
    void UpdateWidth() {}
};

// The elimination trees the reference builds, in call order (bottom,
// leftover inner panel if any, top).
inline std::vector<std::vector<SymmNode>>& RecordedTrees() {
    static std::vector<std::vector<SymmNode>> trees;
    return trees;
}
// Clique's symbolic analysis (its published definition, restated): per
// node, in postorder, the original lower structure sorted; the structure
// after fill, the union of the original one and of the children's
// structures less this node's own indices, sorted; and the position of each
// original entry among the front's rows (own indices first, then the
// structure).  The reference's panel assembly (FillPanelFronts) reads these.
inline void SymmetricAnalysis(const DistSymmElimTree& eTree, DistSymmInfo& info, bool) {
    const size_t n = eTree.localNodes.size();
    std::vector<SymmNode> t;
    info.localNodes.assign(n, SymmNodeInfo());
    for (size_t i = 0; i < n; ++i) {
        const SymmNode& node = *eTree.localNodes[i];
        t.push_back(node);
        SymmNodeInfo& ni = info.localNodes[i];
        ni.size = node.size;
        ni.off = node.off;
        ni.origLowerStruct = node.lowerStruct;
        std::sort(ni.origLowerStruct.begin(), ni.origLowerStruct.end());
        ni.origLowerStruct.erase(std::unique(ni.origLowerStruct.begin(), ni.origLowerStruct.end()),
                                 ni.origLowerStruct.end());
        std::set<int> fill(ni.origLowerStruct.begin(), ni.origLowerStruct.end());
        for (int c : node.children)
            for (int x : info.localNodes[c].lowerStruct)
                if (x < node.off || x >= node.off + node.size) fill.insert(x);
        ni.lowerStruct.assign(fill.begin(), fill.end());
        ni.origLowerRelInds.resize(ni.origLowerStruct.size());
        for (size_t a = 0; a < ni.origLowerStruct.size(); ++a)
            ni.origLowerRelInds[a] = node.size + int(std::lower_bound(ni.lowerStruct.begin(), ni.lowerStruct.end(),
                                                                      ni.origLowerStruct[a]) -
                                                     ni.lowerStruct.begin());
    }
    info.distNodes.assign(std::max<size_t>(1, eTree.distNodes.size()), DistSymmNodeInfo());
    RecordedTrees().push_back(t);
}

// The panel solver behind Solve (installed by the harness): fact identifies
// the panel, X holds its right-hand sides.
typedef std::function<void(const void* fact, DistNodalMultiVec<std::complex<double>>& X)> PanelSolver;
inline PanelSolver& InstalledPanelSolver() {
    static PanelSolver s;
    return s;
}
template <typename F>
inline void Solve(const DistSymmInfo&, const DistSymmFrontTree<F>& fact, DistNodalMultiVec<F>& X) {
    if (!InstalledPanelSolver()) elem::LogicError("no panel solver installed");
    InstalledPanelSolver()(&fact, X);
}
template <typename... A>
inline void LDL(A&&...) {
    elem::LogicError("Clique's LDL is not part of this checker");
}
// On one rank no front is distributed: nothing to set up.
template <typename... A>
inline void InitializeDistLeaf(A&&...) {}
// One rank: the received vector is the sent one.
template <typename T>
inline void SparseAllToAll(const std::vector<T>& sendBuf, const std::vector<int>& sendCounts,
                           const std::vector<int>& sendDispls, std::vector<T>& recvBuf,
                           const std::vector<int>& recvCounts, const std::vector<int>& recvDispls, elem::mpi::Comm) {
    if (sendCounts[0] != recvCounts[0]) elem::LogicError("one-rank SparseAllToAll with unequal counts");
    std::copy(sendBuf.begin() + sendDispls[0], sendBuf.begin() + sendDispls[0] + sendCounts[0],
              recvBuf.begin() + recvDispls[0]);
}

}  // namespace cliq
