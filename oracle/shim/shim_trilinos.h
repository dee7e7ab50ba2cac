/*
 * shim_trilinos.h -- single-process stand-ins for the MPI / Epetra /
 * Trilinos_Util / Amesos declarations that the reference's headers include
 * (include/utils.h:8-46).  ORACLE TEST INFRASTRUCTURE ONLY: this lets the
 * reference's own hot-path translation units (src/*.cpp) compile unmodified
 * on a machine without MPI or Trilinos, so the CPU oracle IS the reference's
 * code.  Nothing here computes anything on the carrier path; it only moves
 * vectors around for one rank:
 *   - MPI: one rank, collectives copy send -> receive buffers;
 *   - Epetra_Map: a global-id list with a gid -> lid lookup;
 *   - Epetra_Vector / Epetra_IntVector: a contiguous array over a map;
 *   - Epetra_Import: with one rank, a gid-matched copy (Insert) or sum (Add);
 *   - Epetra_CrsMatrix: CSR rows keyed by global row id (the Poisson matrix
 *     built by src/mcmodel.cpp:4695-4869);
 *   - Trilinos_Util::InputFileReader: key = value lines, '#' starts a comment
 *     (the reference's own parser is third-party; this is our reading of the
 *     decks in finfet/input.txt).
 */
#ifndef ORACLE_SHIM_TRILINOS_H
#define ORACLE_SHIM_TRILINOS_H

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

/* ------------------------------------------------------------------ MPI -- */
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_INT 1
#define MPI_DOUBLE 2
#define MPI_LONG 3
#define MPI_DOUBLE_INT 4
#define MPI_SUM 1
#define MPI_MAXLOC 2
#define MPI_MAX 3
#define MPI_MIN 4

static inline size_t shim_mpi_type_size(MPI_Datatype t) {
  switch (t) {
    case MPI_INT: return sizeof(int);
    case MPI_DOUBLE: return sizeof(double);
    case MPI_LONG: return sizeof(long);
    case MPI_DOUBLE_INT: return sizeof(double) + sizeof(int) + 4;
    default: return 0;
  }
}
static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Finalize() { return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Allreduce(const void *in, void *out, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  if (in != out) std::memmove(out, in, (size_t)n * shim_mpi_type_size(t));
  return 0;
}
/* Point-to-point calls are only reached with a neighbouring rank, which a
 * single-rank run never has; reaching one is a harness error. */
static inline int shim_mpi_unreachable(const char *what) {
  std::cerr << "oracle shim: " << what << " called in a single-rank run" << std::endl;
  std::abort();
  return 1;
}
static inline int MPI_Send(const void *, int, MPI_Datatype, int, int, MPI_Comm) { return shim_mpi_unreachable("MPI_Send"); }
static inline int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { return shim_mpi_unreachable("MPI_Isend"); }
static inline int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) { return shim_mpi_unreachable("MPI_Recv"); }
static inline int MPI_Wait(MPI_Request *, MPI_Status *) { return shim_mpi_unreachable("MPI_Wait"); }

/* --------------------------------------------------------------- Epetra -- */
enum Epetra_CombineMode { Add, Zero, Insert, InsertAdd, Average, AbsMax };
enum Epetra_DataAccess { Copy, View };

class Epetra_Comm {
 public:
  virtual ~Epetra_Comm() {}
  int MyPID() const { return 0; }
  int NumProc() const { return 1; }
  void Barrier() const {}
};
class Epetra_MpiComm : public Epetra_Comm {
 public:
  explicit Epetra_MpiComm(MPI_Comm) {}
};
class Epetra_SerialComm : public Epetra_Comm {};

class Epetra_Map {
 public:
  /* Linear map of numGlobal elements, all owned by the single rank. */
  Epetra_Map(int numGlobal, int indexBase, const Epetra_Comm &) { init_linear(numGlobal, indexBase); }
  /* numGlobal (-1 = sum of local) and numMy elements numbered from indexBase. */
  Epetra_Map(int, int numMy, int indexBase, const Epetra_Comm &) { init_linear(numMy, indexBase); }
  /* Explicit global-id list. */
  Epetra_Map(int, int numMy, const int *gids, int, const Epetra_Comm &) {
    gid_.assign(gids, gids + numMy);
    index();
  }
  int NumMyElements() const { return (int)gid_.size(); }
  int NumGlobalElements() const { return (int)gid_.size(); }
  int *MyGlobalElements() const { return const_cast<int *>(gid_.data()); }
  int GID(int lid) const { return gid_[lid]; }
  int LID(int gid) const {
    auto it = lid_.find(gid);
    return it == lid_.end() ? -1 : it->second;
  }

 private:
  void init_linear(int n, int base) {
    gid_.resize(n);
    for (int i = 0; i < n; ++i) gid_[i] = base + i;
    index();
  }
  void index() {
    lid_.clear();
    for (int i = 0; i < (int)gid_.size(); ++i) lid_[gid_[i]] = i;
  }
  std::vector<int> gid_;
  std::unordered_map<int, int> lid_;
};

class Epetra_Import {
 public:
  Epetra_Import(const Epetra_Map &target, const Epetra_Map &source) : target_(&target), source_(&source) {
    perm_.resize(target.NumMyElements());
    for (int l = 0; l < target.NumMyElements(); ++l) perm_[l] = source.LID(target.GID(l));
  }
  const Epetra_Map *target_, *source_;
  std::vector<int> perm_; /* target lid -> source lid (-1: not present) */
};
class Epetra_Export {
 public:
  Epetra_Export(const Epetra_Map &, const Epetra_Map &) {}
};

template <typename T>
class ShimDistVector {
 public:
  explicit ShimDistVector(const Epetra_Map &m, bool zero = true) : map_(&m), v_(m.NumMyElements(), T(0)) { (void)zero; }
  ShimDistVector(const ShimDistVector &o) : map_(o.map_), v_(o.v_) {}
  T &operator[](int i) { return v_[i]; }
  const T &operator[](int i) const { return v_[i]; }
  int ExtractView(T **p) const { *p = const_cast<T *>(v_.data()); return 0; }
  int ExtractCopy(T *p) const { std::copy(v_.begin(), v_.end(), p); return 0; }
  int PutScalar(T s) { std::fill(v_.begin(), v_.end(), s); return 0; }
  int PutValue(T s) { return PutScalar(s); }
  int MyLength() const { return (int)v_.size(); }
  int GlobalLength() const { return (int)v_.size(); }
  const Epetra_Map &Map() const { return *map_; }
  T *Values() { return v_.data(); }
  int Import(const ShimDistVector &src, const Epetra_Import &imp, Epetra_CombineMode mode) {
    for (size_t l = 0; l < imp.perm_.size(); ++l) {
      int s = imp.perm_[l];
      if (s < 0) continue;
      if (mode == Add) v_[l] += src.v_[s];
      else v_[l] = src.v_[s];
    }
    return 0;
  }
  int Norm2(double *r) const {
    double s = 0;
    for (const T &x : v_) s += (double)x * (double)x;
    *r = std::sqrt(s);
    return 0;
  }

 protected:
  const Epetra_Map *map_;
  std::vector<T> v_;
};
class Epetra_MultiVector : public ShimDistVector<double> {
 public:
  using ShimDistVector<double>::ShimDistVector;
};
class Epetra_Vector : public Epetra_MultiVector {
 public:
  using Epetra_MultiVector::Epetra_MultiVector;
};
class Epetra_IntVector : public ShimDistVector<int> {
 public:
  using ShimDistVector<int>::ShimDistVector;
};

class Epetra_Time {
 public:
  explicit Epetra_Time(const Epetra_Comm &) { ResetStartTime(); }
  void ResetStartTime() { t0_ = std::chrono::steady_clock::now(); }
  double ElapsedTime() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
  }

 private:
  std::chrono::steady_clock::time_point t0_;
};

/* Row-compressed matrix over a row map with global column ids. */
class Epetra_CrsMatrix {
 public:
  Epetra_CrsMatrix(Epetra_DataAccess, const Epetra_Map &rows, const int *) : rows_(&rows), row_(rows.NumMyElements()) {}
  Epetra_CrsMatrix(Epetra_DataAccess, const Epetra_Map &rows, int) : rows_(&rows), row_(rows.NumMyElements()) {}
  int InsertGlobalValues(int grow, int n, const double *vals, const int *cols) {
    int l = rows_->LID(grow);
    if (l < 0) return -1;
    for (int i = 0; i < n; ++i) row_[l].push_back(std::make_pair(cols[i], vals[i]));
    return 0;
  }
  int FillComplete() { return 0; }
  const Epetra_Map &RowMap() const { return *rows_; }
  const std::vector<std::pair<int, double>> &Row(int lid) const { return row_[lid]; }
  int NumMyRows() const { return (int)row_.size(); }

 private:
  const Epetra_Map *rows_;
  std::vector<std::vector<std::pair<int, double>>> row_;
};

class Epetra_LinearProblem {
 public:
  void SetOperator(Epetra_CrsMatrix *a) { A = a; }
  void SetLHS(Epetra_Vector *x) { X = x; }
  void SetRHS(Epetra_Vector *b) { B = b; }
  Epetra_CrsMatrix *A = nullptr;
  Epetra_Vector *X = nullptr, *B = nullptr;
};

/* Amesos / AztecOO appear only as member types of the reference's
 * PoissonSolver classes (include/PoissonSolver.h); the oracle links its own
 * PoissonSolver implementation (oracle/harness/poisson_direct.cpp). */
class Amesos_BaseSolver {
 public:
  virtual ~Amesos_BaseSolver() {}
};
class Amesos {};
class AztecOO {};

/* ------------------------------------------------------- Trilinos_Util -- */
namespace Trilinos_Util {
class InputFileReader {
 public:
  explicit InputFileReader(const char *fname) : fname_(fname ? fname : "") {}
  int ReadFile() {
    std::ifstream in(fname_.c_str());
    std::string line;
    while (std::getline(in, line)) {
      size_t hash = line.find('#');
      if (hash != std::string::npos) line = line.substr(0, hash);
      size_t eq = line.find('=');
      if (eq == std::string::npos) continue;
      std::string k = trim(line.substr(0, eq)), v = trim(line.substr(eq + 1));
      if (!k.empty()) kv_[k] = v;
    }
    return 0;
  }
  int Get(const std::string &k, int d) const { auto it = kv_.find(k); return it == kv_.end() ? d : std::atoi(it->second.c_str()); }
  double Get(const std::string &k, double d) const { auto it = kv_.find(k); return it == kv_.end() ? d : std::atof(it->second.c_str()); }
  bool Get(const std::string &k, bool d) const { auto it = kv_.find(k); return it == kv_.end() ? d : (std::atoi(it->second.c_str()) != 0 || it->second == "true"); }
  std::string Get(const std::string &k, const std::string &d) const { auto it = kv_.find(k); return it == kv_.end() ? d : it->second; }
  std::string Get(const std::string &k, const char *d) const { return Get(k, std::string(d)); }

 private:
  static std::string trim(const std::string &s) {
    size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
    return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
  }
  std::string fname_;
  std::map<std::string, std::string> kv_;
};
}  // namespace Trilinos_Util

#endif
