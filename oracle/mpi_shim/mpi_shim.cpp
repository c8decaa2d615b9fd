// Thread-based stand-in for the MPI subset the HPCG reference uses; see mpi.h.
// TEST INFRASTRUCTURE ONLY.
#include "mpi.h"

#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

namespace {

struct Message {
  int source, tag;
  std::vector<char> bytes;
};

struct PendingRecv {
  void* buf;
  size_t bytes;
  int source, tag;
};

struct World {
  int size = 1;
  std::mutex mu;
  std::condition_variable cv;
  std::vector<std::deque<Message> > inbox;  // per destination rank
  // barrier
  int arrived = 0;
  unsigned long generation = 0;
  // collectives: one contribution slot per rank
  std::vector<std::vector<char> > slot;
};

World g_world;
thread_local int t_rank = 0;
thread_local std::vector<PendingRecv> t_pending;

size_t type_size(MPI_Datatype t) {
  switch (t) {
    case MPI_CHAR: return 1;
    case MPI_INT: return sizeof(int);
    case MPI_LONG_LONG_INT: return sizeof(long long);
    case MPI_DOUBLE: return sizeof(double);
    default: std::abort();
  }
}

void barrier() {
  std::unique_lock<std::mutex> lk(g_world.mu);
  const unsigned long gen = g_world.generation;
  if (++g_world.arrived == g_world.size) {
    g_world.arrived = 0;
    ++g_world.generation;
    g_world.cv.notify_all();
  } else {
    g_world.cv.wait(lk, [&] { return g_world.generation != gen; });
  }
}

template <typename T>
void fold(const std::vector<std::vector<char> >& slots, int count, MPI_Op op, void* out) {
  T* o = static_cast<T*>(out);
  for (int i = 0; i < count; ++i) {
    T acc;
    std::memcpy(&acc, slots[0].data() + i * sizeof(T), sizeof(T));
    for (size_t r = 1; r < slots.size(); ++r) {
      T v;
      std::memcpy(&v, slots[r].data() + i * sizeof(T), sizeof(T));
      if (op == MPI_SUM) acc = acc + v;
      else if (op == MPI_MAX) acc = v > acc ? v : acc;
      else if (op == MPI_MIN) acc = v < acc ? v : acc;
      else std::abort();
    }
    o[i] = acc;
  }
}

}  // namespace

extern "C" {

void shim_run(int nranks, void (*fn)(int, void*), void* arg) {
  g_world.size = nranks;
  g_world.inbox.assign(nranks, std::deque<Message>());
  g_world.slot.assign(nranks, std::vector<char>());
  g_world.arrived = 0;
  std::vector<std::thread> th;
  for (int r = 0; r < nranks; ++r)
    th.emplace_back([=] {
      t_rank = r;
      t_pending.clear();
      fn(r, arg);
    });
  for (auto& t : th) t.join();
}

int MPI_Init(int*, char***) { return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm, int* size) {
  *size = g_world.size;
  return MPI_SUCCESS;
}
int MPI_Comm_rank(MPI_Comm, int* rank) {
  *rank = t_rank;
  return MPI_SUCCESS;
}

int MPI_Send(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm) {
  Message m;
  m.source = t_rank;
  m.tag = tag;
  m.bytes.resize(type_size(type) * (size_t)count);
  if (count > 0) std::memcpy(m.bytes.data(), buf, m.bytes.size());
  std::lock_guard<std::mutex> lk(g_world.mu);
  g_world.inbox[dest].push_back(std::move(m));
  g_world.cv.notify_all();
  return MPI_SUCCESS;
}

int MPI_Irecv(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm, MPI_Request* req) {
  t_pending.push_back(PendingRecv{buf, type_size(type) * (size_t)count, source, tag});
  *req = (int)t_pending.size() - 1;
  return MPI_SUCCESS;
}

int MPI_Wait(MPI_Request* req, MPI_Status* status) {
  PendingRecv p = t_pending[*req];
  std::unique_lock<std::mutex> lk(g_world.mu);
  std::deque<Message>& box = g_world.inbox[t_rank];
  for (;;) {
    for (auto it = box.begin(); it != box.end(); ++it) {
      if (it->source == p.source && it->tag == p.tag) {
        if (it->bytes.size() != p.bytes) std::abort();
        if (p.bytes) std::memcpy(p.buf, it->bytes.data(), p.bytes);
        if (status) {
          status->MPI_SOURCE = p.source;
          status->MPI_TAG = p.tag;
          status->MPI_ERROR = MPI_SUCCESS;
        }
        box.erase(it);
        // every request of one exchange is waited on before the next exchange posts its own
        if (*req == (int)t_pending.size() - 1) t_pending.clear();
        return MPI_SUCCESS;
      }
    }
    g_world.cv.wait(lk);
  }
}

int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm) {
  const size_t bytes = type_size(type) * (size_t)count;
  {
    std::lock_guard<std::mutex> lk(g_world.mu);
    g_world.slot[t_rank].assign(static_cast<const char*>(sendbuf), static_cast<const char*>(sendbuf) + bytes);
  }
  barrier();
  switch (type) {
    case MPI_INT: fold<int>(g_world.slot, count, op, recvbuf); break;
    case MPI_LONG_LONG_INT: fold<long long>(g_world.slot, count, op, recvbuf); break;
    case MPI_DOUBLE: fold<double>(g_world.slot, count, op, recvbuf); break;
    default: std::abort();
  }
  barrier();
  return MPI_SUCCESS;
}

int MPI_Bcast(void* buf, int count, MPI_Datatype type, int root, MPI_Comm) {
  const size_t bytes = type_size(type) * (size_t)count;
  if (t_rank == root) {
    std::lock_guard<std::mutex> lk(g_world.mu);
    g_world.slot[root].assign(static_cast<char*>(buf), static_cast<char*>(buf) + bytes);
  }
  barrier();
  if (t_rank != root) std::memcpy(buf, g_world.slot[root].data(), bytes);
  barrier();
  return MPI_SUCCESS;
}

int MPI_Barrier(MPI_Comm) {
  barrier();
  return MPI_SUCCESS;
}

int MPI_Abort(MPI_Comm, int code) { std::exit(code); }

double MPI_Wtime(void) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // extern "C"
