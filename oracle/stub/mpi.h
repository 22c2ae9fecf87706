/*
 * Single-rank MPI stand-in used ONLY to compile the reference solvers as a
 * CPU oracle (test infrastructure; never linked into the product library).
 *
 * Every communicator has exactly one rank (rank 0 of 1).  Collectives that
 * move data (Gather, Gatherv, Scatterv) copy the caller's buffer to the
 * destination at displacement 0; broadcasts and barriers are no-ops; the
 * point-to-point calls are no-ops because a one-rank partition has no remote
 * neighbours (the reference's com_n is 0 at one rank).
 */
#ifndef ORACLE_STUB_MPI_H
#define ORACLE_STUB_MPI_H

#include <chrono>
#include <cstring>

typedef int MPI_Datatype;
typedef int MPI_Comm;
typedef int MPI_Request;
struct MPI_Status {
  int MPI_SOURCE;
  int MPI_TAG;
  int MPI_ERROR;
};

#define MPI_CHAR 1
#define MPI_INT 4
#define MPI_FLOAT 5
#define MPI_DOUBLE 8
#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)

static inline size_t oracle_mpi_type_size(MPI_Datatype t) {
  switch (t) {
    case MPI_CHAR: return 1;
    case MPI_INT: return sizeof(int);
    case MPI_FLOAT: return sizeof(float);
    case MPI_DOUBLE: return sizeof(double);
    default: return 1;
  }
}

namespace MPI {
struct OracleComm {
  int Get_rank() const { return 0; }
  int Get_size() const { return 1; }
};
static const OracleComm COMM_WORLD = OracleComm();
template <typename A, typename B>
inline void Init(A&, B&) {}
inline void Init() {}
inline void Finalize() {}
}  // namespace MPI

static inline int MPI_Init(int*, char***) { return 0; }
static inline int MPI_Finalize() { return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
static inline int MPI_Comm_dup(MPI_Comm c, MPI_Comm* out) { *out = c; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }

static inline int MPI_Gather(const void* sbuf, int scount, MPI_Datatype stype,
                             void* rbuf, int, MPI_Datatype, int, MPI_Comm) {
  if (rbuf && sbuf && rbuf != sbuf)
    std::memmove(rbuf, sbuf, (size_t)scount * oracle_mpi_type_size(stype));
  return 0;
}

static inline int MPI_Gatherv(const void* sbuf, int scount, MPI_Datatype stype,
                              void* rbuf, const int*, const int* displs,
                              MPI_Datatype rtype, int, MPI_Comm) {
  if (!rbuf || !sbuf) return 0;
  char* dst = (char*)rbuf + (size_t)(displs ? displs[0] : 0) * oracle_mpi_type_size(rtype);
  if (dst != sbuf) std::memmove(dst, sbuf, (size_t)scount * oracle_mpi_type_size(stype));
  return 0;
}

static inline int MPI_Scatterv(const void* sbuf, const int*, const int* displs,
                               MPI_Datatype stype, void* rbuf, int rcount,
                               MPI_Datatype rtype, int, MPI_Comm) {
  if (!rbuf || !sbuf) return 0;
  const char* src = (const char*)sbuf + (size_t)(displs ? displs[0] : 0) * oracle_mpi_type_size(stype);
  if (src != rbuf) std::memmove(rbuf, src, (size_t)rcount * oracle_mpi_type_size(rtype));
  return 0;
}

static inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* r) {
  if (r) *r = 0;
  return 0;
}
static inline int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* r) {
  if (r) *r = 0;
  return 0;
}
static inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) { return 0; }
static inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) { return 0; }
static inline int MPI_Wait(MPI_Request*, MPI_Status*) { return 0; }
static inline int MPI_Waitall(int, MPI_Request*, MPI_Status*) { return 0; }
static inline int MPI_Testall(int, MPI_Request*, int* flag, MPI_Status*) {
  if (flag) *flag = 1;
  return 0;
}

static inline double MPI_Wtime() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}
static inline double MPI_Wtick() { return 1e-9; }

#endif
