// Single-rank implementation of the MPI stand-in (shim/mpi.h): the result of
// every collective on one rank is the caller's own contribution, so each one
// copies its send buffer into its receive buffer; point-to-point messages can
// only go to self and are matched by tag in posting order.
#include "mpi.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <deque>
#include <vector>

namespace {
struct Msg {
  int tag;
  std::vector<char> data;
};
struct PendingRecv {
  int tag;
  char* buf;
  size_t cap;
  MPI_Request req;
};
std::deque<Msg> g_sent;
std::deque<PendingRecv> g_recv;
}  // namespace

struct MPI_Request_s {
  bool done = false;
};

static void copy_buf(const void* s, void* r, size_t n) {
  if (s != MPI_IN_PLACE && s != r && n) memmove(r, s, n);
}

static void deliver() {
  for (auto it = g_recv.begin(); it != g_recv.end();) {
    bool matched = false;
    for (auto m = g_sent.begin(); m != g_sent.end(); ++m) {
      if (m->tag != it->tag) continue;
      if (m->data.size() > it->cap) {
        fprintf(stderr, "mpi stub: message of %zu bytes into a %zu-byte receive\n", m->data.size(), it->cap);
        abort();
      }
      if (!m->data.empty()) memcpy(it->buf, m->data.data(), m->data.size());
      it->req->done = true;
      g_sent.erase(m);
      matched = true;
      break;
    }
    it = matched ? g_recv.erase(it) : it + 1;
  }
}

extern "C" {
int MPI_Init(int*, char***) { return MPI_SUCCESS; }
int MPI_Init_thread(int*, char***, int req, int* prov) {
  if (prov) *prov = req;
  return MPI_SUCCESS;
}
int MPI_Initialized(int* f) {
  *f = 1;
  return MPI_SUCCESS;
}
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm, int* s) {
  *s = 1;
  return MPI_SUCCESS;
}
int MPI_Comm_rank(MPI_Comm, int* r) {
  *r = 0;
  return MPI_SUCCESS;
}
int MPI_Comm_split(MPI_Comm c, int, int, MPI_Comm* n) {
  *n = c;
  return MPI_SUCCESS;
}
int MPI_Comm_free(MPI_Comm* c) {
  *c = MPI_COMM_NULL;
  return MPI_SUCCESS;
}
MPI_Comm MPI_Comm_f2c(MPI_Fint f) { return (MPI_Comm)f; }
int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  copy_buf(s, r, (size_t)n * t);
  return MPI_SUCCESS;
}
int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  copy_buf(s, r, (size_t)n * t);
  return MPI_SUCCESS;
}
int MPI_Scan(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  copy_buf(s, r, (size_t)n * t);
  return MPI_SUCCESS;
}
int MPI_Allgather(const void* s, int ns, MPI_Datatype ts, void* r, int, MPI_Datatype, MPI_Comm) {
  copy_buf(s, r, (size_t)ns * ts);
  return MPI_SUCCESS;
}
int MPI_Allgatherv(const void* s, int ns, MPI_Datatype ts, void* r, const int*, const int* displs, MPI_Datatype tr,
                   MPI_Comm) {
  copy_buf(s, (char*)r + (size_t)displs[0] * tr, (size_t)ns * ts);
  return MPI_SUCCESS;
}
int MPI_Alltoall(const void* s, int ns, MPI_Datatype ts, void* r, int, MPI_Datatype, MPI_Comm) {
  copy_buf(s, r, (size_t)ns * ts);
  return MPI_SUCCESS;
}
int MPI_Alltoallv(const void* s, const int* sc, const int* sd, MPI_Datatype ts, void* r, const int*, const int* rd,
                  MPI_Datatype tr, MPI_Comm) {
  copy_buf((const char*)s + (size_t)sd[0] * ts, (char*)r + (size_t)rd[0] * tr, (size_t)sc[0] * ts);
  return MPI_SUCCESS;
}
int MPI_Isend(const void* b, int n, MPI_Datatype t, int, int tag, MPI_Comm, MPI_Request* q) {
  Msg m;
  m.tag = tag;
  m.data.assign((const char*)b, (const char*)b + (size_t)n * t);
  g_sent.push_back(std::move(m));
  *q = new MPI_Request_s;
  (*q)->done = true;
  deliver();
  return MPI_SUCCESS;
}
int MPI_Issend(const void* b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c, MPI_Request* q) {
  return MPI_Isend(b, n, t, d, tag, c, q);
}
int MPI_Send(const void* b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c) {
  MPI_Request q;
  MPI_Isend(b, n, t, d, tag, c, &q);
  delete q;
  return MPI_SUCCESS;
}
int MPI_Irecv(void* b, int n, MPI_Datatype t, int, int tag, MPI_Comm, MPI_Request* q) {
  *q = new MPI_Request_s;
  g_recv.push_back({tag, (char*)b, (size_t)n * t, *q});
  deliver();
  return MPI_SUCCESS;
}
int MPI_Wait(MPI_Request* q, MPI_Status*) {
  if (!*q) return MPI_SUCCESS;
  deliver();
  if (!(*q)->done) {
    fprintf(stderr, "mpi stub: wait on a receive that no send to self matches\n");
    abort();
  }
  delete *q;
  *q = MPI_REQUEST_NULL;
  return MPI_SUCCESS;
}
int MPI_Waitall(int n, MPI_Request* q, MPI_Status*) {
  for (int i = 0; i < n; ++i) MPI_Wait(&q[i], nullptr);
  return MPI_SUCCESS;
}
int MPI_Recv(void* b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Status*) {
  MPI_Request q;
  MPI_Irecv(b, n, t, s, tag, c, &q);
  return MPI_Wait(&q, nullptr);
}
int MPI_Sendrecv(const void* sb, int sn, MPI_Datatype st, int d, int stag, void* rb, int rn, MPI_Datatype rt, int s,
                 int rtag, MPI_Comm c, MPI_Status*) {
  MPI_Request q;
  MPI_Irecv(rb, rn, rt, s, rtag, c, &q);
  MPI_Send(sb, sn, st, d, stag, c);
  return MPI_Wait(&q, nullptr);
}
int MPI_Type_contiguous(int n, MPI_Datatype t, MPI_Datatype* o) {
  *o = (MPI_Datatype)n * t;
  return MPI_SUCCESS;
}
int MPI_Type_commit(MPI_Datatype*) { return MPI_SUCCESS; }
int MPI_Type_free(MPI_Datatype*) { return MPI_SUCCESS; }
int MPI_Op_create(MPI_User_function* f, int, MPI_Op* o) {
  *o = f;
  return MPI_SUCCESS;
}
int MPI_Op_free(MPI_Op*) { return MPI_SUCCESS; }
int MPI_Get_count(const MPI_Status* s, MPI_Datatype t, int* c) {
  *c = s ? (int)(s->count / t) : 0;
  return MPI_SUCCESS;
}
double MPI_Wtime(void) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
}
