/*
 * Multi-process MPI stand-in used ONLY to run the reference's slab-decomposed
 * programs (two or more ranks) as a CPU oracle: test infrastructure, never
 * linked into the product library.
 *
 * Ranks are ordinary processes started by the test harness with
 *   MPISHIM_RANK=r  MPISHIM_SIZE=n  MPISHIM_DIR=<directory shared by all ranks>
 * (without them: rank 0 of 1).  A message is one file in MPISHIM_DIR named
 * after (source, destination, tag, sequence number), written under a
 * temporary name and renamed, so it appears whole; a receive waits for the
 * file of the next sequence number of its (source, tag), reads and deletes it.
 * Sends are buffered (they complete at once), so no exchange pattern can
 * deadlock on buffer space; receives match in posting order per (source, tag),
 * MPI's non-overtaking rule.  Collectives are built from point-to-point
 * messages on tags above every user tag.  A receive that waits more than
 * MPISHIM_TIMEOUT seconds (default 300) ends the process with an error
 * instead of hanging.
 *
 * Only the calls the reference programs use are provided.
 */
#ifndef ORACLE_MPISHIM_MPI_H
#define ORACLE_MPISHIM_MPI_H

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include <sys/stat.h>
#include <unistd.h>

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

namespace mpishim {

inline size_t type_size(MPI_Datatype t) {
  switch (t) {
    case MPI_CHAR: return 1;
    case MPI_INT: return sizeof(int);
    case MPI_FLOAT: return sizeof(float);
    case MPI_DOUBLE: return sizeof(double);
    default: return 1;
  }
}

struct State {
  int rank = 0, size = 1;
  std::string dir;
  double timeout = 300.0;
  std::map<std::pair<int, int>, long long> send_seq, recv_seq;  // (peer, tag) -> next number
  struct Pending {
    void* buf;
    size_t bytes;
    int src, tag;
    long long seq;
    bool done;
  };
  std::vector<Pending> reqs;  // request handle = index + 1
  bool inited = false;
};

inline State& S() {
  static State s;
  return s;
}

inline void init() {
  State& s = S();
  if (s.inited) return;
  s.inited = true;
  const char* r = std::getenv("MPISHIM_RANK");
  const char* n = std::getenv("MPISHIM_SIZE");
  const char* d = std::getenv("MPISHIM_DIR");
  const char* t = std::getenv("MPISHIM_TIMEOUT");
  if (r && n && d) {
    s.rank = std::atoi(r);
    s.size = std::atoi(n);
    s.dir = d;
  }
  if (t) s.timeout = std::atof(t);
}

inline std::string name(int src, int dst, int tag, long long seq, bool tmp) {
  char b[512];
  std::snprintf(b, sizeof(b), "%s/%s_%d_%d_%d_%lld", S().dir.c_str(), tmp ? "tmp" : "msg", src, dst, tag, seq);
  return b;
}

inline void fatal(const char* what) {
  std::fprintf(stderr, "mpishim rank %d: %s\n", S().rank, what);
  std::exit(97);
}

inline void send_bytes(const void* buf, size_t bytes, int dst, int tag) {
  init();
  State& s = S();
  if (dst == s.rank && s.size == 1) return;
  const long long seq = s.send_seq[{dst, tag}]++;
  const std::string tmp = name(s.rank, dst, tag, seq, true), fin = name(s.rank, dst, tag, seq, false);
  FILE* f = std::fopen(tmp.c_str(), "wb");
  if (!f) fatal("cannot create a message file");
  if (bytes && std::fwrite(buf, 1, bytes, f) != bytes) fatal("short message write");
  std::fclose(f);
  if (std::rename(tmp.c_str(), fin.c_str()) != 0) fatal("cannot publish a message file");
}

// Non-blocking attempt: true when the message was there and has been read.
inline bool try_recv(void* buf, size_t bytes, int src, int tag, long long seq) {
  const std::string fin = name(src, S().rank, tag, seq, false);
  FILE* f = std::fopen(fin.c_str(), "rb");
  if (!f) return false;
  std::fseek(f, 0, SEEK_END);
  const long len = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  if ((size_t)len > bytes) fatal("message longer than the receive buffer");
  if (len > 0 && std::fread(buf, 1, (size_t)len, f) != (size_t)len) fatal("short message read");
  std::fclose(f);
  std::remove(fin.c_str());
  return true;
}

inline void wait_recv(void* buf, size_t bytes, int src, int tag, long long seq) {
  using clk = std::chrono::steady_clock;
  const auto t0 = clk::now();
  while (!try_recv(buf, bytes, src, tag, seq)) {
    if (std::chrono::duration<double>(clk::now() - t0).count() > S().timeout) fatal("receive timed out");
    std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
}

inline void recv_bytes(void* buf, size_t bytes, int src, int tag) {
  init();
  State& s = S();
  const long long seq = s.recv_seq[{src, tag}]++;
  wait_recv(buf, bytes, src, tag, seq);
}

constexpr int kCollTag = 1 << 28;  // collectives: kCollTag + kind

}  // namespace mpishim

namespace MPI {
struct ShimComm {
  int Get_rank() const {
    mpishim::init();
    return mpishim::S().rank;
  }
  int Get_size() const {
    mpishim::init();
    return mpishim::S().size;
  }
};
static const ShimComm COMM_WORLD = ShimComm();
template <typename A, typename B>
inline void Init(A&, B&) {
  mpishim::init();
}
inline void Init() { mpishim::init(); }
inline void Finalize() {}
}  // namespace MPI

static inline int MPI_Init(int*, char***) {
  mpishim::init();
  return 0;
}
static inline int MPI_Finalize() { return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) {
  *r = MPI::COMM_WORLD.Get_rank();
  return 0;
}
static inline int MPI_Comm_size(MPI_Comm, int* s) {
  *s = MPI::COMM_WORLD.Get_size();
  return 0;
}
static inline int MPI_Comm_dup(MPI_Comm c, MPI_Comm* out) {
  *out = c;
  return 0;
}

static inline int MPI_Barrier(MPI_Comm) {
  mpishim::init();
  mpishim::State& s = mpishim::S();
  if (s.size == 1) return 0;
  char token = 0;
  if (s.rank == 0) {
    for (int r = 1; r < s.size; r++) mpishim::recv_bytes(&token, 1, r, mpishim::kCollTag + 1);
    for (int r = 1; r < s.size; r++) mpishim::send_bytes(&token, 1, r, mpishim::kCollTag + 2);
  } else {
    mpishim::send_bytes(&token, 1, 0, mpishim::kCollTag + 1);
    mpishim::recv_bytes(&token, 1, 0, mpishim::kCollTag + 2);
  }
  return 0;
}

static inline int MPI_Bcast(void* buf, int count, MPI_Datatype t, int root, MPI_Comm) {
  mpishim::init();
  mpishim::State& s = mpishim::S();
  if (s.size == 1) return 0;
  const size_t b = (size_t)count * mpishim::type_size(t);
  if (s.rank == root) {
    for (int r = 0; r < s.size; r++)
      if (r != root) mpishim::send_bytes(buf, b, r, mpishim::kCollTag + 3);
  } else {
    mpishim::recv_bytes(buf, b, root, mpishim::kCollTag + 3);
  }
  return 0;
}

static inline int MPI_Gather(const void* sbuf, int scount, MPI_Datatype stype, void* rbuf, int rcount,
                             MPI_Datatype rtype, int root, MPI_Comm) {
  mpishim::init();
  mpishim::State& s = mpishim::S();
  const size_t sb = (size_t)scount * mpishim::type_size(stype), rb = (size_t)rcount * mpishim::type_size(rtype);
  if (s.rank == root) {
    for (int r = 0; r < s.size; r++) {
      char* dst = (char*)rbuf + (size_t)r * rb;
      if (r == root) {
        if (dst != sbuf) std::memmove(dst, sbuf, sb);
      } else {
        mpishim::recv_bytes(dst, rb, r, mpishim::kCollTag + 4);
      }
    }
  } else {
    mpishim::send_bytes(sbuf, sb, root, mpishim::kCollTag + 4);
  }
  return 0;
}

static inline int MPI_Gatherv(const void* sbuf, int scount, MPI_Datatype stype, void* rbuf, const int* rcounts,
                              const int* displs, MPI_Datatype rtype, int root, MPI_Comm) {
  mpishim::init();
  mpishim::State& s = mpishim::S();
  const size_t sb = (size_t)scount * mpishim::type_size(stype), ts = mpishim::type_size(rtype);
  if (s.rank == root) {
    for (int r = 0; r < s.size; r++) {
      char* dst = (char*)rbuf + (size_t)displs[r] * ts;
      if (r == root) {
        if (dst != sbuf) std::memmove(dst, sbuf, sb);
      } else {
        mpishim::recv_bytes(dst, (size_t)rcounts[r] * ts, r, mpishim::kCollTag + 5);
      }
    }
  } else {
    mpishim::send_bytes(sbuf, sb, root, mpishim::kCollTag + 5);
  }
  return 0;
}

static inline int MPI_Scatterv(const void* sbuf, const int* scounts, const int* displs, MPI_Datatype stype,
                               void* rbuf, int rcount, MPI_Datatype rtype, int root, MPI_Comm) {
  mpishim::init();
  mpishim::State& s = mpishim::S();
  const size_t ts = mpishim::type_size(stype), rb = (size_t)rcount * mpishim::type_size(rtype);
  if (s.rank == root) {
    for (int r = 0; r < s.size; r++) {
      const char* src = (const char*)sbuf + (size_t)displs[r] * ts;
      if (r == root) {
        if (src != rbuf) std::memmove(rbuf, src, (size_t)scounts[r] * ts);
      } else {
        mpishim::send_bytes(src, (size_t)scounts[r] * ts, r, mpishim::kCollTag + 6);
      }
    }
  } else {
    mpishim::recv_bytes(rbuf, rb, root, mpishim::kCollTag + 6);
  }
  return 0;
}

static inline int MPI_Send(const void* buf, int count, MPI_Datatype t, int dst, int tag, MPI_Comm) {
  mpishim::send_bytes(buf, (size_t)count * mpishim::type_size(t), dst, tag);
  return 0;
}
static inline int MPI_Recv(void* buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm, MPI_Status* st) {
  mpishim::recv_bytes(buf, (size_t)count * mpishim::type_size(t), src, tag);
  if (st) {
    st->MPI_SOURCE = src;
    st->MPI_TAG = tag;
    st->MPI_ERROR = 0;
  }
  return 0;
}
static inline int MPI_Isend(const void* buf, int count, MPI_Datatype t, int dst, int tag, MPI_Comm,
                            MPI_Request* req) {
  mpishim::send_bytes(buf, (size_t)count * mpishim::type_size(t), dst, tag);
  if (req) *req = 0;  // buffered: complete
  return 0;
}
static inline int MPI_Irecv(void* buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm, MPI_Request* req) {
  mpishim::init();
  mpishim::State& s = mpishim::S();
  const long long seq = s.recv_seq[{src, tag}]++;
  s.reqs.push_back({buf, (size_t)count * mpishim::type_size(t), src, tag, seq, false});
  if (req) *req = (int)s.reqs.size();
  return 0;
}
static inline int MPI_Wait(MPI_Request* req, MPI_Status*) {
  if (!req || *req <= 0) return 0;
  mpishim::State::Pending& p = mpishim::S().reqs[*req - 1];
  if (!p.done) mpishim::wait_recv(p.buf, p.bytes, p.src, p.tag, p.seq);
  p.done = true;
  *req = 0;
  return 0;
}
static inline int MPI_Waitall(int n, MPI_Request* reqs, MPI_Status*) {
  for (int i = 0; i < n; i++) MPI_Wait(&reqs[i], nullptr);
  return 0;
}
static inline int MPI_Testall(int n, MPI_Request* reqs, int* flag, MPI_Status*) {
  bool all = true;
  for (int i = 0; i < n; i++) {
    if (reqs[i] <= 0) continue;
    mpishim::State::Pending& p = mpishim::S().reqs[reqs[i] - 1];
    if (!p.done && mpishim::try_recv(p.buf, p.bytes, p.src, p.tag, p.seq)) p.done = true;
    if (p.done)
      reqs[i] = 0;
    else
      all = false;
  }
  if (!all) std::this_thread::sleep_for(std::chrono::microseconds(20));
  if (flag) *flag = all ? 1 : 0;
  return 0;
}
static inline int MPI_Sendrecv(const void* sbuf, int scount, MPI_Datatype stype, int dst, int stag, void* rbuf,
                               int rcount, MPI_Datatype rtype, int src, int rtag, MPI_Comm c, MPI_Status* st) {
  MPI_Send(sbuf, scount, stype, dst, stag, c);
  return MPI_Recv(rbuf, rcount, rtype, src, rtag, c, st);
}

static inline double MPI_Wtime() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}
static inline double MPI_Wtick() { return 1e-9; }

#endif
