// mpi_shim.cpp -- the MPI subset the NUC3d reference needs, without an MPI library.
//
// TEST INFRASTRUCTURE ONLY: it exists so the reference CPU solver can be built
// and run as the correctness oracle and the timed CPU baseline.  Nothing in the
// GPU product links it.
//
// Model: MPI_Init forks NUC_SHIM_NP-1 child processes (default: 1 rank, no fork).
// All ranks share one anonymous MAP_SHARED region that holds
//   * a sense-counting barrier,
//   * per-rank slots for MPI_Allreduce (every rank reduces the slots in rank
//     order, so SUM gives the same bits on every rank),
//   * a message table plus fixed-size payload slots for Isend/Irecv.
// Isend copies the payload eagerly (the request completes at once); Wait on a
// receive polls the table for the oldest message with the wanted (src, tag),
// which gives MPI's non-overtaking order.  Every wait is bounded by
// NUC_SHIM_TIMEOUT seconds and by an abort flag that any rank may raise.
//
// The reference uses exactly these calls: src/MPICommunicator.cpp:55-115
// (Isend/Irecv/Wait, tags from src/MPICommunicator.h:33-47),
// src/PDEData3d.cpp:78,121 (Allreduce MIN/MAX), src/postproc.cpp:828-830
// (Allreduce SUM) and 19 Barriers.
#include "mpi.h"

#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <pthread.h>
#include <sched.h>
#include <signal.h>
#include <sys/mman.h>
#include <sys/wait.h>
#include <unistd.h>

namespace {

constexpr int kMaxRanks = 256;
constexpr int kRedMax = 16;
constexpr int kMaxMsgs = 4096;

struct MsgEntry {
  int state;  // 0 free, 1 being written, 2 ready, 3 being read
  int src, dst, tag;
  long long seq;
  int slot;
  long long bytes;
};

struct Shared {
  int np;
  std::atomic<int> bar_count;
  std::atomic<int> bar_gen;
  std::atomic<int> abort_code;
  std::atomic<int> abort_flag;
  pthread_mutex_t mtx;
  long long seq;
  int nslots;
  long long slot_bytes;
  double red[kMaxRanks][kRedMax];
  MsgEntry msgs[kMaxMsgs];
  unsigned char slot_used[1];  // nslots bytes follow, then the payload arena
};

Shared *g_sh = nullptr;
unsigned char *g_arena = nullptr;
int g_rank = 0;
int g_np = 1;
bool g_final = false;
pid_t g_children[kMaxRanks];
double g_timeout = 1800.0;

struct Req {
  int kind;  // 0 free, 1 completed send, 2 pending recv
  void *buf;
  long long bytes;
  int src, tag;
};
constexpr int kMaxReq = 4096;
Req g_req[kMaxReq];

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

[[noreturn]] void die(const char *msg, int code) {
  std::fprintf(stderr, "[mpi_shim rank %d] %s\n", g_rank, msg);
  std::fflush(stderr);
  if (g_sh) {
    g_sh->abort_code.store(code);
    g_sh->abort_flag.store(1);
  }
  std::fflush(stdout);
  _exit(code ? code : 1);
}

void check_wait(double t0, const char *what) {
  if (g_sh->abort_flag.load()) {
    std::fflush(stdout);
    _exit(g_sh->abort_code.load() ? g_sh->abort_code.load() : 1);
  }
  if (now_s() - t0 > g_timeout) die(what, 3);
  sched_yield();
}

long long type_size(MPI_Datatype t) { return t == MPI_INT ? (long long)sizeof(int) : (long long)sizeof(double); }

void barrier_impl() {
  if (g_np == 1) return;
  int gen = g_sh->bar_gen.load();
  if (g_sh->bar_count.fetch_add(1) + 1 == g_np) {
    g_sh->bar_count.store(0);
    g_sh->bar_gen.fetch_add(1);
    return;
  }
  double t0 = now_s();
  while (g_sh->bar_gen.load() == gen) check_wait(t0, "barrier timed out");
}

int alloc_req() {
  for (int i = 0; i < kMaxReq; ++i)
    if (g_req[i].kind == 0) return i;
  die("out of request handles", 4);
}

}  // namespace

extern "C" {

int MPI_Init(int *, char ***) {
  const char *e = std::getenv("NUC_SHIM_NP");
  g_np = e ? std::atoi(e) : 1;
  if (g_np < 1 || g_np > kMaxRanks) {
    std::fprintf(stderr, "[mpi_shim] NUC_SHIM_NP must be in 1..%d\n", kMaxRanks);
    std::exit(2);
  }
  if (const char *t = std::getenv("NUC_SHIM_TIMEOUT")) g_timeout = std::atof(t);
  int nslots = 8 * g_np + 8;
  long long slot_mb = 8;
  if (const char *s = std::getenv("NUC_SHIM_SLOT_MB")) slot_mb = std::atoll(s);
  long long slot_bytes = slot_mb << 20;
  size_t head = sizeof(Shared) + (size_t)nslots;
  head = (head + 4095) & ~(size_t)4095;
  size_t total = head + (size_t)nslots * (size_t)slot_bytes;
  void *p = mmap(nullptr, total, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS, -1, 0);
  if (p == MAP_FAILED) {
    std::perror("[mpi_shim] mmap");
    std::exit(2);
  }
  g_sh = static_cast<Shared *>(p);
  std::memset(g_sh, 0, sizeof(Shared) + (size_t)nslots);
  g_sh->np = g_np;
  g_sh->nslots = nslots;
  g_sh->slot_bytes = slot_bytes;
  pthread_mutexattr_t at;
  pthread_mutexattr_init(&at);
  pthread_mutexattr_setpshared(&at, PTHREAD_PROCESS_SHARED);
  pthread_mutex_init(&g_sh->mtx, &at);
  g_arena = static_cast<unsigned char *>(p) + head;
  std::fflush(stdout);
  std::cout.flush();
  for (int r = 1; r < g_np; ++r) {
    pid_t pid = fork();
    if (pid < 0) {
      std::perror("[mpi_shim] fork");
      std::exit(2);
    }
    if (pid == 0) {
      g_rank = r;
      return MPI_SUCCESS;
    }
    g_children[r] = pid;
  }
  g_rank = 0;
  return MPI_SUCCESS;
}

int MPI_Finalize(void) {
  if (g_final) return MPI_SUCCESS;
  g_final = true;
  barrier_impl();
  std::cout.flush();
  std::fflush(stdout);
  std::fflush(stderr);
  if (g_rank != 0) _exit(0);
  int bad = 0;
  for (int r = 1; r < g_np; ++r) {
    int st = 0;
    waitpid(g_children[r], &st, 0);
    if (!WIFEXITED(st) || WEXITSTATUS(st) != 0) bad = 1;
  }
  if (bad) {
    std::fprintf(stderr, "[mpi_shim] a child rank failed\n");
    std::exit(5);
  }
  return MPI_SUCCESS;
}

int MPI_Abort(MPI_Comm, int code) { die("MPI_Abort called", code ? code : 1); }

int MPI_Comm_rank(MPI_Comm, int *rank) {
  *rank = g_rank;
  return MPI_SUCCESS;
}

int MPI_Comm_size(MPI_Comm, int *size) {
  *size = g_np;
  return MPI_SUCCESS;
}

int MPI_Barrier(MPI_Comm) {
  barrier_impl();
  return MPI_SUCCESS;
}

double MPI_Wtime(void) { return now_s(); }

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op op,
                  MPI_Comm) {
  if (type != MPI_DOUBLE || count > kRedMax) die("Allreduce supports <=16 doubles", 6);
  const double *in = static_cast<const double *>(sendbuf);
  double *out = static_cast<double *>(recvbuf);
  if (g_np == 1) {
    for (int i = 0; i < count; ++i) out[i] = in[i];
    return MPI_SUCCESS;
  }
  for (int i = 0; i < count; ++i) g_sh->red[g_rank][i] = in[i];
  barrier_impl();
  for (int i = 0; i < count; ++i) {
    double acc = g_sh->red[0][i];
    for (int r = 1; r < g_np; ++r) {
      double v = g_sh->red[r][i];
      if (op == MPI_MIN)
        acc = v < acc ? v : acc;
      else if (op == MPI_MAX)
        acc = v > acc ? v : acc;
      else
        acc = acc + v;
    }
    out[i] = acc;
  }
  barrier_impl();
  return MPI_SUCCESS;
}

int MPI_Isend(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm,
              MPI_Request *req) {
  long long bytes = (long long)count * type_size(type);
  if (bytes > g_sh->slot_bytes) die("message larger than NUC_SHIM_SLOT_MB", 7);
  if (dest < 0 || dest >= g_np) die("Isend to an invalid rank", 7);
  double t0 = now_s();
  int e = -1, s = -1;
  for (;;) {
    pthread_mutex_lock(&g_sh->mtx);
    for (int i = 0; i < kMaxMsgs && e < 0; ++i)
      if (g_sh->msgs[i].state == 0) e = i;
    for (int i = 0; i < g_sh->nslots && s < 0; ++i)
      if (!g_sh->slot_used[i]) s = i;
    if (e >= 0 && s >= 0) {
      MsgEntry &m = g_sh->msgs[e];
      m.state = 1;
      m.src = g_rank;
      m.dst = dest;
      m.tag = tag;
      m.seq = g_sh->seq++;
      m.slot = s;
      m.bytes = bytes;
      g_sh->slot_used[s] = 1;
      pthread_mutex_unlock(&g_sh->mtx);
      break;
    }
    e = s = -1;
    pthread_mutex_unlock(&g_sh->mtx);
    check_wait(t0, "no free message slot");
  }
  std::memcpy(g_arena + (size_t)s * (size_t)g_sh->slot_bytes, buf, (size_t)bytes);
  pthread_mutex_lock(&g_sh->mtx);
  g_sh->msgs[e].state = 2;
  pthread_mutex_unlock(&g_sh->mtx);
  int r = alloc_req();
  g_req[r].kind = 1;
  *req = r;
  return MPI_SUCCESS;
}

int MPI_Irecv(void *buf, int count, MPI_Datatype type, int src, int tag, MPI_Comm,
              MPI_Request *req) {
  int r = alloc_req();
  g_req[r].kind = 2;
  g_req[r].buf = buf;
  g_req[r].bytes = (long long)count * type_size(type);
  g_req[r].src = src;
  g_req[r].tag = tag;
  *req = r;
  return MPI_SUCCESS;
}

int MPI_Wait(MPI_Request *req, MPI_Status *status) {
  int r = *req;
  if (r < 0 || r >= kMaxReq || g_req[r].kind == 0) return 1;
  if (g_req[r].kind == 1) {
    g_req[r].kind = 0;
    return MPI_SUCCESS;
  }
  Req &q = g_req[r];
  double t0 = now_s();
  for (;;) {
    pthread_mutex_lock(&g_sh->mtx);
    int best = -1;
    for (int i = 0; i < kMaxMsgs; ++i) {
      const MsgEntry &m = g_sh->msgs[i];
      if (m.state == 2 && m.dst == g_rank && m.src == q.src && m.tag == q.tag &&
          (best < 0 || m.seq < g_sh->msgs[best].seq))
        best = i;
    }
    if (best >= 0) {
      MsgEntry &m = g_sh->msgs[best];
      m.state = 3;
      pthread_mutex_unlock(&g_sh->mtx);
      if (m.bytes != q.bytes) die("message size mismatch", 8);
      std::memcpy(q.buf, g_arena + (size_t)m.slot * (size_t)g_sh->slot_bytes, (size_t)m.bytes);
      pthread_mutex_lock(&g_sh->mtx);
      g_sh->slot_used[m.slot] = 0;
      m.state = 0;
      pthread_mutex_unlock(&g_sh->mtx);
      if (status) {
        status->MPI_SOURCE = q.src;
        status->MPI_TAG = q.tag;
        status->MPI_ERROR = 0;
      }
      q.kind = 0;
      return MPI_SUCCESS;
    }
    pthread_mutex_unlock(&g_sh->mtx);
    check_wait(t0, "receive timed out");
  }
}

}  // extern "C"
