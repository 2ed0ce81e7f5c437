// In-process stand-in for the few MPI calls of the reference's face-state
// exchange (src/exo3/cubed_sphere.cpp:289-688): every "rank" is a MeshBlock
// of this one process, MPI_Isend files a copy of the message under its tag
// and MPI_Recv takes it back (the harness runs every send before any
// receive).  Test infrastructure only.
#ifndef REF_STUB_MPI_H_
#define REF_STUB_MPI_H_
#include <cstring>
#include <map>
#include <stdexcept>
#include <vector>

typedef int MPI_Request;
typedef int MPI_Status;
typedef int MPI_Datatype;
typedef int MPI_Comm;
#define MPI_DOUBLE 1
#define MPI_COMM_WORLD 0
#define MPI_STATUS_IGNORE nullptr

inline std::map<int, std::vector<double>>& mpi_inproc_board() {
  static std::map<int, std::vector<double>> board;
  return board;
}
inline int MPI_Isend(const void* data, int n, MPI_Datatype, int, int tag, MPI_Comm,
                     MPI_Request* req) {
  auto& b = mpi_inproc_board();
  if (b.count(tag)) throw std::runtime_error("MPI stand-in: duplicate tag");
  const double* d = static_cast<const double*>(data);
  b[tag] = std::vector<double>(d, d + n);
  *req = tag;
  return 0;
}
inline int MPI_Recv(void* data, int n, MPI_Datatype, int, int tag, MPI_Comm, MPI_Status*) {
  auto& b = mpi_inproc_board();
  auto it = b.find(tag);
  if (it == b.end() || (int)it->second.size() != n)
    throw std::runtime_error("MPI stand-in: no message of that tag and size");
  std::memcpy(data, it->second.data(), n * sizeof(double));
  b.erase(it);
  return 0;
}
inline int MPI_Wait(MPI_Request*, MPI_Status*) { return 0; }
#endif
