// Minimal stand-in for the Athena++ fork's athena.hpp, written for this
// harness (the fork is not vendored): just enough of its types and constants
// for the reference's exo3 and Riemann sources to compile unchanged.  Test
// infrastructure only.
#ifndef REF_STUB_ATHENA_HPP_
#define REF_STUB_ATHENA_HPP_

#include <cmath>
#include <cstdint>
#include <cstring>
#include <sstream>
#include <stdexcept>
#include <vector>

#ifdef MPI_PARALLEL
#include <mpi.h>
#endif

typedef double Real;

#define NGHOST 3

// hydro variable indices (dry ideal gas: NHYDRO = 5)
enum { IDN = 0, IM1 = 1, IM2 = 2, IM3 = 3, IEN = 4, NHYDRO = 5, NFIELD = 0 };
enum { IVX = 1, IVY = 2, IVZ = 3, IPR = 4, NWAVE = 5 };
enum { I11 = 0, I22, I33, I12, I13, I23, NMETRIC };
enum { X1DIR = 0, X2DIR = 1, X3DIR = 2 };

#define PI 3.1415926535897932
#define TINY_NUMBER 1.0e-20
#define SQR(x) ((x) * (x))
#define GENERAL_EOS 0
#define MAGNETIC_FIELDS_ENABLED 0

#define ATHENA_ERROR(x) throw std::runtime_error(x.str())

// A 1- to 4-D array with the (n,k,j,i) index order of Athena++'s AthenaArray,
// i fastest.  Owns its storage, or wraps caller storage (Wrap, harness only).
template <typename T>
class AthenaArray {
 public:
  AthenaArray() = default;
  AthenaArray(const AthenaArray&) = delete;
  AthenaArray& operator=(const AthenaArray&) = delete;

  void NewAthenaArray(int nx1) { alloc(1, 1, 1, nx1); }
  void NewAthenaArray(int nx2, int nx1) { alloc(1, 1, nx2, nx1); }
  void NewAthenaArray(int nx3, int nx2, int nx1) { alloc(1, nx3, nx2, nx1); }
  void NewAthenaArray(int nx4, int nx3, int nx2, int nx1) { alloc(nx4, nx3, nx2, nx1); }
  void Wrap(T* data, int nx4, int nx3, int nx2, int nx1) {
    own_.clear();
    p_ = data;
    nx4_ = nx4; nx3_ = nx3; nx2_ = nx2; nx1_ = nx1;
  }
  int GetDim1() const { return nx1_; }
  int GetDim2() const { return nx2_; }
  int GetDim3() const { return nx3_; }
  int GetDim4() const { return nx4_; }
  T* data() { return p_; }
  const T* data() const { return p_; }

  T& operator()(int i) { return p_[i]; }
  T operator()(int i) const { return p_[i]; }
  T& operator()(int j, int i) { return p_[(size_t)j * nx1_ + i]; }
  T operator()(int j, int i) const { return p_[(size_t)j * nx1_ + i]; }
  T& operator()(int k, int j, int i) { return p_[((size_t)k * nx2_ + j) * nx1_ + i]; }
  T operator()(int k, int j, int i) const { return p_[((size_t)k * nx2_ + j) * nx1_ + i]; }
  T& operator()(int n, int k, int j, int i) {
    return p_[(((size_t)n * nx3_ + k) * nx2_ + j) * nx1_ + i];
  }
  T operator()(int n, int k, int j, int i) const {
    return p_[(((size_t)n * nx3_ + k) * nx2_ + j) * nx1_ + i];
  }

 private:
  void alloc(int nx4, int nx3, int nx2, int nx1) {
    nx4_ = nx4; nx3_ = nx3; nx2_ = nx2; nx1_ = nx1;
    // one extra row of slack: a reference loop reads one (k, j) past its
    // 2-D tables at the last ghost column (gnomonic_equiangle.cpp:213-216)
    own_.assign((size_t)nx4 * nx3 * nx2 * nx1 + (size_t)nx1 * (nx2 + 1), T(0));
    p_ = own_.data();
  }
  std::vector<T> own_;
  T* p_ = nullptr;
  int nx4_ = 0, nx3_ = 0, nx2_ = 0, nx1_ = 0;
};

struct LogicalLocation {
  int64_t lx1 = 0, lx2 = 0, lx3 = 0;
  int level = 0;
};

class MeshBlock;
class ParameterInput;
class Coordinates;
class EquationOfState;
class Hydro;

#endif
