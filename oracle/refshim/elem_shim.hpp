// ORACLE — test infrastructure only (the checker, never the product).
//
// A one-process stand-in for the few Elemental / MPI names that
// include/psp/dist_uniform_grid.hpp of the reference uses (its
// environment.hpp pulls them in from Clique and Elemental, which are absent
// here).  With it that header compiles unchanged from the reference tree,
// so the reference's own grid code (SequentialLoad, InterpolateTo,
// WritePlane, WriteVolume) can be run on one process and checked against
// oracle/grid_io.py.  Every collective is the identity of a one-rank
// communicator; nothing here is part of the product.
#pragma once
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <fstream>
#include <initializer_list>
#include <iostream>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include <sys/stat.h>

#define DEBUG_ONLY(cmd)
#ifndef HAVE_MKDIR
#define HAVE_MKDIR
#endif
#ifndef RELEASE
#define RELEASE
#endif

namespace psp {

template <typename R>
using Complex = std::complex<R>;

// Messages are the arguments streamed one after another.
template <typename... Args>
inline std::string Message(const Args&... args) {
    std::ostringstream os;
    (void)std::initializer_list<int>{((os << args), 0)...};
    return os.str();
}
template <typename... Args>
inline void LogicError(const Args&... args) { throw std::logic_error(Message(args...)); }
template <typename... Args>
inline void RuntimeError(const Args&... args) { throw std::runtime_error(Message(args...)); }

// Local length of an n-entry dimension whose entries are dealt cyclically
// to `stride` processes, on the process with offset `shift`; the four-
// argument form takes the process rank and the rank holding entry 0.
inline int Length(int n, int shift, int stride) { return n > shift ? (n - shift - 1) / stride + 1 : 0; }
// Offset of process `rank` when the rank `firstRank` holds entry 0.
inline int Shift(int rank, int firstRank, int stride) { return (rank - firstRank + stride) % stride; }
inline int Length(int n, int rank, int firstRank, int stride) { return Length(n, Shift(rank, firstRank, stride), stride); }

template <typename T>
inline T Abs(T x) { return std::abs(x); }

template <typename T>
inline void SwapClear(T& x) {
    T().swap(x);
}

inline void EnsureDirExists(const char* path, mode_t mode = 0777) {
    struct stat st;
    if (stat(path, &st) != 0 && mkdir(path, mode) != 0) RuntimeError("Could not create directory ", path);
}

namespace elem {
template <typename T>
inline void MemCopy(T* dest, const T* src, std::size_t n) {
    std::copy(src, src + n, dest);
}
}  // namespace elem

namespace mpi {
typedef int Comm;
inline int CommRank(Comm) { return 0; }
inline int CommSize(Comm) { return 1; }
inline void Barrier(Comm) {}
// One rank: what rank 0 sends to itself is what it receives.
template <typename T>
inline void AllToAll(const T* sbuf, int sc, T* rbuf, int rc, Comm) {
    if (sc != rc) throw std::logic_error("one-rank AllToAll with unequal counts");
    std::copy(sbuf, sbuf + sc, rbuf);
}
template <typename T>
inline void AllToAll(const T* sbuf, const int* scs, const int* sds, T* rbuf, const int* rcs, const int* rds, Comm) {
    if (scs[0] != rcs[0]) throw std::logic_error("one-rank AllToAll with unequal counts");
    std::copy(sbuf + sds[0], sbuf + sds[0] + scs[0], rbuf + rds[0]);
}
template <typename T>
inline void Gather(const T* sbuf, int sc, T* rbuf, const int* rcs, const int* rds, int root, Comm) {
    if (root != 0 || sc != rcs[0]) throw std::logic_error("one-rank Gather with unequal counts");
    std::copy(sbuf, sbuf + sc, rbuf + rds[0]);
}
template <typename T>
inline void Gather(const T* sbuf, int sc, T* rbuf, int rc, int root, Comm) {
    if (root != 0 || sc != rc) throw std::logic_error("one-rank Gather with unequal counts");
    std::copy(sbuf, sbuf + sc, rbuf);
}
}  // namespace mpi

}  // namespace psp
