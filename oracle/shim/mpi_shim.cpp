// Single-rank MPI stand-in (oracle build only; see mpi.h).
#include "mpi.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <vector>

struct oracle_mpi_req {
  bool is_recv = false;
  bool done = false;
  void *buf = nullptr;
  long long cap_bytes = 0;
  int tag = 0;
  long long got_bytes = 0;
};

namespace {
struct Msg {
  int tag;
  std::vector<char> bytes;
};
std::deque<Msg> &queue() {
  static std::deque<Msg> q;
  return q;
}

size_t type_size(MPI_Datatype t) {
  switch (t) {
    case MPI_CHAR:
    case MPI_BYTE: return 1;
    case MPI_INT:
    case MPI_UNSIGNED:
    case MPI_FLOAT: return 4;
    case MPI_DOUBLE:
    case MPI_INT64_T:
    case MPI_LONG_LONG:
    case MPI_UNSIGNED_LONG_LONG:
    case MPI_UINT64_T:
    case MPI_LONG: return 8;
    case MPI_DOUBLE_INT: return 16;  // struct { double; int; } with padding
    default:
      std::fprintf(stderr, "oracle mpi shim: unknown datatype %d\n", t);
      std::abort();
  }
}

void copy_if_distinct(const void *s, void *r, size_t bytes) {
  if (s == MPI_IN_PLACE || s == r || bytes == 0) return;
  std::memmove(r, s, bytes);
}

bool try_match(oracle_mpi_req *rq) {
  auto &q = queue();
  for (auto it = q.begin(); it != q.end(); ++it) {
    if (rq->tag == MPI_ANY_TAG || it->tag == rq->tag) {
      long long n = (long long)it->bytes.size();
      if (n > rq->cap_bytes) {
        std::fprintf(stderr, "oracle mpi shim: message truncated (tag %d)\n", it->tag);
        std::abort();
      }
      if (n) std::memcpy(rq->buf, it->bytes.data(), (size_t)n);
      rq->got_bytes = n;
      rq->tag = it->tag;
      rq->done = true;
      q.erase(it);
      return true;
    }
  }
  return false;
}
}  // namespace

extern "C" {
int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
int MPI_Initialized(int *flag) { *flag = 1; return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm, int *size) { *size = 1; return MPI_SUCCESS; }
int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
double MPI_Wtime(void) {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}
int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  copy_if_distinct(s, r, (size_t)n * type_size(t));
  return MPI_SUCCESS;
}
int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  copy_if_distinct(s, r, (size_t)n * type_size(t));
  return MPI_SUCCESS;
}
int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
int MPI_Gather(const void *s, int sn, MPI_Datatype st, void *r, int, MPI_Datatype, int, MPI_Comm) {
  copy_if_distinct(s, r, (size_t)sn * type_size(st));
  return MPI_SUCCESS;
}
int MPI_Allgather(const void *s, int sn, MPI_Datatype st, void *r, int, MPI_Datatype, MPI_Comm) {
  copy_if_distinct(s, r, (size_t)sn * type_size(st));
  return MPI_SUCCESS;
}
int MPI_Allgatherv(const void *s, int sn, MPI_Datatype st, void *r, const int *, const int *displs,
                   MPI_Datatype rt, MPI_Comm) {
  if (s == MPI_IN_PLACE) return MPI_SUCCESS;
  copy_if_distinct(s, (char *)r + (size_t)displs[0] * type_size(rt), (size_t)sn * type_size(st));
  return MPI_SUCCESS;
}
int MPI_Alltoall(const void *s, int sn, MPI_Datatype st, void *r, int, MPI_Datatype, MPI_Comm) {
  copy_if_distinct(s, r, (size_t)sn * type_size(st));
  return MPI_SUCCESS;
}
int MPI_Alltoallv(const void *s, const int *sn, const int *sd, MPI_Datatype st, void *r, const int *,
                  const int *rd, MPI_Datatype rt, MPI_Comm) {
  copy_if_distinct((const char *)s + (size_t)sd[0] * type_size(st),
                   (char *)r + (size_t)rd[0] * type_size(rt), (size_t)sn[0] * type_size(st));
  return MPI_SUCCESS;
}
int MPI_Exscan(const void *, void *, int, MPI_Datatype, MPI_Op, MPI_Comm) {
  // Rank 0's receive buffer is undefined by the standard; leave it untouched.
  return MPI_SUCCESS;
}
int MPI_Isend(const void *b, int n, MPI_Datatype t, int dst, int tag, MPI_Comm, MPI_Request *req) {
  if (dst != 0) {
    std::fprintf(stderr, "oracle mpi shim: send to rank %d in a world of size 1\n", dst);
    std::abort();
  }
  Msg m;
  m.tag = tag;
  m.bytes.resize((size_t)n * type_size(t));
  if (n) std::memcpy(m.bytes.data(), b, m.bytes.size());
  queue().push_back(std::move(m));
  auto *rq = new oracle_mpi_req();
  rq->done = true;
  *req = rq;
  return MPI_SUCCESS;
}
int MPI_Irecv(void *b, int n, MPI_Datatype t, int src, int tag, MPI_Comm, MPI_Request *req) {
  if (src != 0 && src != MPI_ANY_SOURCE) {
    std::fprintf(stderr, "oracle mpi shim: recv from rank %d in a world of size 1\n", src);
    std::abort();
  }
  auto *rq = new oracle_mpi_req();
  rq->is_recv = true;
  rq->buf = b;
  rq->cap_bytes = (long long)n * (long long)type_size(t);
  rq->tag = tag;
  *req = rq;
  return MPI_SUCCESS;
}
int MPI_Wait(MPI_Request *req, MPI_Status *st) {
  oracle_mpi_req *rq = *req;
  if (!rq) return MPI_SUCCESS;
  if (rq->is_recv && !rq->done && !try_match(rq)) {
    std::fprintf(stderr, "oracle mpi shim: receive (tag %d) has no matching send\n", rq->tag);
    std::abort();
  }
  if (st) {
    st->MPI_SOURCE = 0;
    st->MPI_TAG = rq->tag;
    st->MPI_ERROR = MPI_SUCCESS;
    st->oracle_bytes = rq->got_bytes;
  }
  delete rq;
  *req = MPI_REQUEST_NULL;
  return MPI_SUCCESS;
}
int MPI_Waitall(int n, MPI_Request *reqs, MPI_Status *sts) {
  for (int i = 0; i < n; ++i) MPI_Wait(&reqs[i], sts ? &sts[i] : MPI_STATUS_IGNORE);
  return MPI_SUCCESS;
}
int MPI_Get_count(const MPI_Status *st, MPI_Datatype t, int *count) {
  *count = (int)(st->oracle_bytes / (long long)type_size(t));
  return MPI_SUCCESS;
}
int MPI_Abort(MPI_Comm, int code) { std::exit(code); }
}
