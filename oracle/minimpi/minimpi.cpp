// minimpi: MPI subset for building the camille reference as the oracle.
// Test infrastructure only; see mpi.h for the transports it provides.
#include "mpi.h"

#include <poll.h>
#include <unistd.h>
#include <errno.h>
#include <signal.h>

#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace {

struct Message {
  int src;     // world rank
  int comm;
  int tag;
  std::vector<char> data;
};

struct Header {
  int src, comm, tag, nbytes;
};

int g_rank = 0;
int g_size = 1;
std::vector<int> g_fds;  // socket to each world rank (-1 for self)
std::vector<std::vector<int>> g_groups;  // member world ranks per group handle
std::vector<std::vector<int>> g_comms;   // member world ranks per comm handle
std::vector<std::deque<Message>> g_queues;  // per source world rank
std::mutex g_mu;
std::condition_variable g_cv;
std::thread g_reader;
bool g_reader_stop = false;
bool g_reader_dead = false;
std::vector<int> g_coll_seq;  // per communicator: members call collectives in the same order
double g_timeout_s = 600.0;

[[noreturn]] void die(const char *what) {
  std::fprintf(stderr, "minimpi[rank %d]: %s\n", g_rank, what);
  std::fflush(stderr);
  _exit(97);
}

int type_size(MPI_Datatype t) {
  switch (t) {
    case MPI_INT: return (int)sizeof(int);
    case MPI_DOUBLE: return (int)sizeof(double);
    case MPI_CHAR: return 1;
  }
  die("unsupported MPI_Datatype");
}

void write_all(int fd, const void *p, size_t n) {
  const char *c = static_cast<const char *>(p);
  while (n > 0) {
    ssize_t w = ::write(fd, c, n);
    if (w < 0) {
      if (errno == EINTR) continue;
      die("socket write failed (peer gone)");
    }
    c += w;
    n -= (size_t)w;
  }
}

bool read_all(int fd, void *p, size_t n) {
  char *c = static_cast<char *>(p);
  while (n > 0) {
    ssize_t r = ::read(fd, c, n);
    if (r == 0) return false;
    if (r < 0) {
      if (errno == EINTR) continue;
      return false;
    }
    c += r;
    n -= (size_t)r;
  }
  return true;
}

void reader_loop() {
  std::vector<pollfd> pfds;
  std::vector<int> who;
  for (int r = 0; r < g_size; ++r)
    if (g_fds[r] >= 0) {
      pfds.push_back({g_fds[r], POLLIN, 0});
      who.push_back(r);
    }
  int open_peers = (int)pfds.size();
  while (open_peers > 0) {
    {
      std::lock_guard<std::mutex> lk(g_mu);
      if (g_reader_stop) return;
    }
    int n = ::poll(pfds.data(), pfds.size(), 200);
    if (n <= 0) continue;
    for (size_t i = 0; i < pfds.size(); ++i) {
      if (pfds[i].fd < 0 || !(pfds[i].revents & (POLLIN | POLLHUP | POLLERR))) continue;
      Header h;
      if (!read_all(pfds[i].fd, &h, sizeof h)) {
        pfds[i].fd = -1;
        --open_peers;
        continue;
      }
      Message m;
      m.src = h.src;
      m.comm = h.comm;
      m.tag = h.tag;
      m.data.resize((size_t)h.nbytes);
      if (h.nbytes > 0 && !read_all(pfds[i].fd, m.data.data(), (size_t)h.nbytes)) {
        pfds[i].fd = -1;
        --open_peers;
        continue;
      }
      {
        std::lock_guard<std::mutex> lk(g_mu);
        g_queues[who[i]].push_back(std::move(m));
      }
      g_cv.notify_all();
    }
  }
  std::lock_guard<std::mutex> lk(g_mu);
  g_reader_dead = true;
  g_cv.notify_all();
}

void post(int dest_world, int comm, int tag, const void *buf, int nbytes) {
  if (dest_world == g_rank) {
    Message m;
    m.src = g_rank;
    m.comm = comm;
    m.tag = tag;
    m.data.assign(static_cast<const char *>(buf), static_cast<const char *>(buf) + nbytes);
    {
      std::lock_guard<std::mutex> lk(g_mu);
      g_queues[g_rank].push_back(std::move(m));
    }
    g_cv.notify_all();
    return;
  }
  Header h{g_rank, comm, tag, nbytes};
  write_all(g_fds[dest_world], &h, sizeof h);
  if (nbytes > 0) write_all(g_fds[dest_world], buf, (size_t)nbytes);
}

void take(int src_world, int comm, int tag, void *buf, int max_bytes, MPI_Status *st) {
  std::unique_lock<std::mutex> lk(g_mu);
  auto deadline = std::chrono::steady_clock::now() +
                  std::chrono::milliseconds((long long)(g_timeout_s * 1000.0));
  for (;;) {
    auto &q = g_queues[src_world];
    for (auto it = q.begin(); it != q.end(); ++it) {
      if (it->comm == comm && it->tag == tag) {
        int n = (int)it->data.size();
        if (n > max_bytes) die("received message longer than the receive buffer");
        if (n > 0) std::memcpy(buf, it->data.data(), (size_t)n);
        if (st) {
          st->MPI_SOURCE = src_world;
          st->MPI_TAG = tag;
          st->MPI_ERROR = 0;
          st->count_bytes = n;
        }
        q.erase(it);
        return;
      }
    }
    if (g_reader_dead && src_world != g_rank) die("peer closed its connection before sending");
    if (g_cv.wait_until(lk, deadline) == std::cv_status::timeout) {
      char msg[160];
      std::snprintf(msg, sizeof msg, "receive from world rank %d (comm %d, tag %d) timed out",
                    src_world, comm, tag);
      die(msg);
    }
  }
}

int world_of(MPI_Comm comm, int rank_in_comm) {
  if (comm < 0 || comm >= (int)g_comms.size()) die("invalid communicator");
  const auto &m = g_comms[comm];
  if (rank_in_comm < 0 || rank_in_comm >= (int)m.size()) die("rank outside communicator");
  return m[rank_in_comm];
}

int my_index(const std::vector<int> &members) {
  for (size_t i = 0; i < members.size(); ++i)
    if (members[i] == g_rank) return (int)i;
  return MPI_UNDEFINED;
}

// Collectives use negative tags, distinct per call, counted per communicator.
int next_coll_tag(MPI_Comm comm) {
  if ((int)g_coll_seq.size() <= comm) g_coll_seq.resize((size_t)comm + 1, 0);
  return -1000 - (g_coll_seq[comm]++ & 0x3fffffff);
}

void reduce_into(void *acc, const void *in, int count, MPI_Datatype t, MPI_Op op) {
  if (t == MPI_DOUBLE) {
    double *a = static_cast<double *>(acc);
    const double *b = static_cast<const double *>(in);
    for (int i = 0; i < count; ++i) {
      if (op == MPI_SUM) a[i] += b[i];
      else if (op == MPI_MAX) a[i] = a[i] > b[i] ? a[i] : b[i];
      else if (op == MPI_MIN) a[i] = a[i] < b[i] ? a[i] : b[i];
      else die("unsupported MPI_Op");
    }
  } else if (t == MPI_INT) {
    int *a = static_cast<int *>(acc);
    const int *b = static_cast<const int *>(in);
    for (int i = 0; i < count; ++i) {
      if (op == MPI_SUM) a[i] += b[i];
      else if (op == MPI_MAX) a[i] = a[i] > b[i] ? a[i] : b[i];
      else if (op == MPI_MIN) a[i] = a[i] < b[i] ? a[i] : b[i];
      else die("unsupported MPI_Op");
    }
  } else {
    die("unsupported reduction type");
  }
}

}  // namespace

extern "C" {

int MPI_Init(int *, char ***) {
  const char *r = std::getenv("MINIMPI_RANK");
  const char *s = std::getenv("MINIMPI_SIZE");
  const char *t = std::getenv("MINIMPI_TIMEOUT_S");
  if (t) g_timeout_s = std::atof(t);
  g_rank = r ? std::atoi(r) : 0;
  g_size = s ? std::atoi(s) : 1;
  if (g_size < 1 || g_rank < 0 || g_rank >= g_size) die("bad MINIMPI_RANK/MINIMPI_SIZE");
  g_fds.assign((size_t)g_size, -1);
  if (g_size > 1) {
    const char *f = std::getenv("MINIMPI_FDS");
    if (!f) die("MINIMPI_FDS missing: start ranks with minimpi_run");
    std::string fs(f);
    size_t pos = 0;
    for (int i = 0; i < g_size; ++i) {
      size_t c = fs.find(',', pos);
      g_fds[i] = std::atoi(fs.substr(pos, c - pos).c_str());
      pos = (c == std::string::npos) ? fs.size() : c + 1;
    }
  }
  g_queues.assign((size_t)g_size, std::deque<Message>());
  std::vector<int> world;
  for (int i = 0; i < g_size; ++i) world.push_back(i);
  g_groups.push_back(world);
  g_comms.push_back(world);
  if (g_size > 1) g_reader = std::thread(reader_loop);
  return MPI_SUCCESS;
}

int MPI_Finalize(void) {
  if (g_size > 1) {
    MPI_Barrier(MPI_COMM_WORLD);
    {
      std::lock_guard<std::mutex> lk(g_mu);
      g_reader_stop = true;
    }
    if (g_reader.joinable()) g_reader.join();
  }
  return MPI_SUCCESS;
}

int MPI_Abort(MPI_Comm, int errorcode) {
  std::fprintf(stderr, "minimpi[rank %d]: MPI_Abort(%d)\n", g_rank, errorcode);
  std::fflush(stderr);
  _exit(errorcode ? errorcode : 98);
}

int MPI_Comm_rank(MPI_Comm comm, int *rank) {
  if (comm < 0 || comm >= (int)g_comms.size()) die("invalid communicator");
  *rank = my_index(g_comms[comm]);
  return MPI_SUCCESS;
}

int MPI_Comm_size(MPI_Comm comm, int *size) {
  if (comm < 0 || comm >= (int)g_comms.size()) die("invalid communicator");
  *size = (int)g_comms[comm].size();
  return MPI_SUCCESS;
}

int MPI_Comm_group(MPI_Comm comm, MPI_Group *group) {
  if (comm < 0 || comm >= (int)g_comms.size()) die("invalid communicator");
  g_groups.push_back(g_comms[comm]);
  *group = (int)g_groups.size() - 1;
  return MPI_SUCCESS;
}

int MPI_Comm_create(MPI_Comm comm, MPI_Group group, MPI_Comm *newcomm) {
  // Collective over comm: every member calls it in the same order, so the new
  // handle has the same value on every rank. Ranks outside the group get
  // MPI_COMM_NULL but still consume the handle.
  if (group < 0 || group >= (int)g_groups.size()) die("invalid group");
  MPI_Barrier(comm);
  g_comms.push_back(g_groups[group]);
  int id = (int)g_comms.size() - 1;
  *newcomm = my_index(g_groups[group]) == MPI_UNDEFINED ? MPI_COMM_NULL : id;
  return MPI_SUCCESS;
}

int MPI_Group_incl(MPI_Group group, int n, const int ranks[], MPI_Group *newgroup) {
  if (group < 0 || group >= (int)g_groups.size()) die("invalid group");
  std::vector<int> members;
  for (int i = 0; i < n; ++i) {
    if (ranks[i] < 0 || ranks[i] >= (int)g_groups[group].size()) die("rank outside group");
    members.push_back(g_groups[group][ranks[i]]);
  }
  g_groups.push_back(members);
  *newgroup = (int)g_groups.size() - 1;
  return MPI_SUCCESS;
}

int MPI_Group_rank(MPI_Group group, int *rank) {
  if (group < 0 || group >= (int)g_groups.size()) die("invalid group");
  *rank = my_index(g_groups[group]);
  return MPI_SUCCESS;
}

int MPI_Group_size(MPI_Group group, int *size) {
  if (group < 0 || group >= (int)g_groups.size()) die("invalid group");
  *size = (int)g_groups[group].size();
  return MPI_SUCCESS;
}

int MPI_Barrier(MPI_Comm comm) {
  int me, n;
  MPI_Comm_rank(comm, &me);
  MPI_Comm_size(comm, &n);
  if (n == 1) return MPI_SUCCESS;
  int tag = next_coll_tag(comm);
  char token = 0;
  if (me == 0) {
    for (int r = 1; r < n; ++r) take(world_of(comm, r), comm, tag, &token, 1, nullptr);
    for (int r = 1; r < n; ++r) post(world_of(comm, r), comm, tag, &token, 1);
  } else {
    post(world_of(comm, 0), comm, tag, &token, 1);
    take(world_of(comm, 0), comm, tag, &token, 1, nullptr);
  }
  return MPI_SUCCESS;
}

int MPI_Bcast(void *buffer, int count, MPI_Datatype datatype, int root, MPI_Comm comm) {
  int me, n;
  MPI_Comm_rank(comm, &me);
  MPI_Comm_size(comm, &n);
  int tag = next_coll_tag(comm);
  if (n == 1) return MPI_SUCCESS;
  int nbytes = count * type_size(datatype);
  if (me == root) {
    for (int r = 0; r < n; ++r)
      if (r != root) post(world_of(comm, r), comm, tag, buffer, nbytes);
  } else {
    take(world_of(comm, root), comm, tag, buffer, nbytes, nullptr);
  }
  return MPI_SUCCESS;
}

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype datatype,
                  MPI_Op op, MPI_Comm comm) {
  int me, n;
  MPI_Comm_rank(comm, &me);
  MPI_Comm_size(comm, &n);
  int nbytes = count * type_size(datatype);
  if (recvbuf != sendbuf) std::memmove(recvbuf, sendbuf, (size_t)nbytes);
  if (n == 1) return MPI_SUCCESS;
  int tag = next_coll_tag(comm);
  if (me == 0) {
    std::vector<char> tmp((size_t)nbytes);
    for (int r = 1; r < n; ++r) {
      take(world_of(comm, r), comm, tag, tmp.data(), nbytes, nullptr);
      reduce_into(recvbuf, tmp.data(), count, datatype, op);
    }
    for (int r = 1; r < n; ++r) post(world_of(comm, r), comm, tag, recvbuf, nbytes);
  } else {
    post(world_of(comm, 0), comm, tag, recvbuf, nbytes);
    take(world_of(comm, 0), comm, tag, recvbuf, nbytes, nullptr);
  }
  return MPI_SUCCESS;
}

int MPI_Send(const void *buf, int count, MPI_Datatype datatype, int dest, int tag, MPI_Comm comm) {
  post(world_of(comm, dest), comm, tag, buf, count * type_size(datatype));
  return MPI_SUCCESS;
}

int MPI_Recv(void *buf, int count, MPI_Datatype datatype, int source, int tag, MPI_Comm comm,
             MPI_Status *status) {
  take(world_of(comm, source), comm, tag, buf, count * type_size(datatype), status);
  return MPI_SUCCESS;
}

int MPI_Isend(const void *buf, int count, MPI_Datatype datatype, int dest, int tag, MPI_Comm comm,
              MPI_Request *request) {
  // Messages are copied into the transport at once, so the send is complete.
  post(world_of(comm, dest), comm, tag, buf, count * type_size(datatype));
  if (request) {
    std::memset(request, 0, sizeof *request);
    request->kind = 0;
  }
  return MPI_SUCCESS;
}

int MPI_Irecv(void *buf, int count, MPI_Datatype datatype, int source, int tag, MPI_Comm comm,
              MPI_Request *request) {
  request->kind = 1;
  request->buf = buf;
  request->count = count;
  request->type = datatype;
  request->source = source;
  request->tag = tag;
  request->comm = comm;
  return MPI_SUCCESS;
}

int MPI_Wait(MPI_Request *request, MPI_Status *status) {
  if (request && request->kind == 1) {
    take(world_of(request->comm, request->source), request->comm, request->tag, request->buf,
         request->count * type_size(request->type), status);
    request->kind = 0;
  }
  return MPI_SUCCESS;
}

}  // extern "C"
