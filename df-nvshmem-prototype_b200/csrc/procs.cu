// procs.cu -- process-per-PE mode: the prototype's own execution model, one
// OS process per PE (there: MPI ranks, nvshmem.cu:472-561), on one GPU
// without MPI.  Every process owns the physical memory of its slice and
// exports it as a POSIX file descriptor (a VMM shareable handle); the
// processes exchange the descriptors over Unix domain sockets in a
// rendezvous directory and map every slice at the same place of their own
// reserved arena, so the symmetric address translation is the same as in the
// one-process mode.  The host barrier (nvshmem_barrier_all) is a counter in a
// file-backed shared mapping in the same directory.
//
// The directory is made by the launcher (python -m nvshmem_b200.launch) and
// passed to every process in NVSHMEM_RENDEZVOUS with NVSHMEM_PROCESS_PE and
// NVSHMEM_NPES.  Kernels of different processes are separate launches with
// no co-residency guarantee, so in this mode PEs meet on the host only; a
// device-side wait on another process's flag is not supported.
#include <errno.h>
#include <fcntl.h>
#include <poll.h>
#include <stdio.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/socket.h>
#include <sys/stat.h>
#include <sys/un.h>
#include <time.h>
#include <unistd.h>

#include <atomic>
#include <string>
#include <thread>
#include <vector>

#include "procs.h"
#include "runtime.h"

namespace nvshm {

namespace {

struct SharedBarrier {
  std::atomic<unsigned> count;
  std::atomic<unsigned> gen;
  std::atomic<unsigned> left;  // processes that stopped; a barrier then fails
  unsigned pad[13];
};
static_assert(sizeof(SharedBarrier) == 64, "one cache line");

struct ProcState {
  int pe = -1;
  int npes = 0;
  std::string dir;
  int listen_fd = -1;
  SharedBarrier *bar = nullptr;
};
ProcState g_ps;

double now_s() {
  timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return t.tv_sec + 1e-9 * t.tv_nsec;
}

std::string sock_path(int pe) { return g_ps.dir + "/pe" + std::to_string(pe) + ".sock"; }

bool fill_addr(sockaddr_un &a, const std::string &path) {
  memset(&a, 0, sizeof a);
  a.sun_family = AF_UNIX;
  if (path.size() >= sizeof a.sun_path) return false;
  memcpy(a.sun_path, path.c_str(), path.size() + 1);
  return true;
}

// One message: the sender's PE and one descriptor (SCM_RIGHTS).
bool send_fd(int sock, int pe, int fd) {
  char cbuf[CMSG_SPACE(sizeof(int))];
  memset(cbuf, 0, sizeof cbuf);
  iovec iov{&pe, sizeof pe};
  msghdr m;
  memset(&m, 0, sizeof m);
  m.msg_iov = &iov;
  m.msg_iovlen = 1;
  m.msg_control = cbuf;
  m.msg_controllen = sizeof cbuf;
  cmsghdr *c = CMSG_FIRSTHDR(&m);
  c->cmsg_level = SOL_SOCKET;
  c->cmsg_type = SCM_RIGHTS;
  c->cmsg_len = CMSG_LEN(sizeof(int));
  memcpy(CMSG_DATA(c), &fd, sizeof fd);
  return sendmsg(sock, &m, 0) == (ssize_t)sizeof pe;
}

bool recv_fd(int sock, int *pe, int *fd) {
  char cbuf[CMSG_SPACE(sizeof(int))];
  iovec iov{pe, sizeof *pe};
  msghdr m;
  memset(&m, 0, sizeof m);
  m.msg_iov = &iov;
  m.msg_iovlen = 1;
  m.msg_control = cbuf;
  m.msg_controllen = sizeof cbuf;
  if (recvmsg(sock, &m, 0) != (ssize_t)sizeof *pe) return false;
  cmsghdr *c = CMSG_FIRSTHDR(&m);
  if (!c || c->cmsg_level != SOL_SOCKET || c->cmsg_type != SCM_RIGHTS) return false;
  memcpy(fd, CMSG_DATA(c), sizeof *fd);
  return true;
}

}  // namespace

bool proc_mode() { return g_ps.pe >= 0; }
int proc_pe() { return g_ps.pe; }

int proc_open(int pe, int npes, const char *dir) {
  if (pe < 0 || pe >= npes || !dir || !*dir)
    return fail(NVSHMEMX_ERR_INVALID, "process mode: PE %d of %d, rendezvous '%s'", pe, npes, dir ? dir : "");
  g_ps.pe = pe;
  g_ps.npes = npes;
  g_ps.dir = dir;
  // listening socket for the descriptors of the other PEs
  sockaddr_un a;
  const std::string path = sock_path(pe);
  if (!fill_addr(a, path)) return fail(NVSHMEMX_ERR_INVALID, "process mode: rendezvous path too long");
  unlink(path.c_str());
  g_ps.listen_fd = socket(AF_UNIX, SOCK_STREAM | SOCK_CLOEXEC, 0);
  if (g_ps.listen_fd < 0 || bind(g_ps.listen_fd, (sockaddr *)&a, sizeof a) != 0 ||
      listen(g_ps.listen_fd, npes) != 0) {
    proc_close();
    return fail(NVSHMEMX_ERR_STATE, "process mode: cannot listen on %s (%s)", path.c_str(), strerror(errno));
  }
  // shared barrier word (a new file reads as zeros)
  const std::string bpath = g_ps.dir + "/barrier";
  int bfd = open(bpath.c_str(), O_RDWR | O_CREAT | O_CLOEXEC, 0600);
  if (bfd < 0 || ftruncate(bfd, sizeof(SharedBarrier)) != 0) {
    if (bfd >= 0) close(bfd);
    proc_close();
    return fail(NVSHMEMX_ERR_STATE, "process mode: cannot open %s (%s)", bpath.c_str(), strerror(errno));
  }
  void *m = mmap(nullptr, sizeof(SharedBarrier), PROT_READ | PROT_WRITE, MAP_SHARED, bfd, 0);
  close(bfd);
  if (m == MAP_FAILED) {
    proc_close();
    return fail(NVSHMEMX_ERR_STATE, "process mode: cannot map the barrier (%s)", strerror(errno));
  }
  g_ps.bar = static_cast<SharedBarrier *>(m);
  return 0;
}

// Sends `my_fd` to every other PE and receives theirs into peer_fds[q]
// (peer_fds[pe] = my_fd).  Peers that are not listening yet are retried
// until the timeout.
int proc_exchange_fds(int my_fd, std::vector<int> &peer_fds, double timeout_s) {
  const int P = g_ps.npes, me = g_ps.pe;
  peer_fds.assign(P, -1);
  peer_fds[me] = my_fd;
  const double t_end = now_s() + timeout_s;
  int recv_rc = 0;
  std::thread receiver([&] {
    for (int got = 0; got < P - 1;) {
      pollfd pf{g_ps.listen_fd, POLLIN, 0};
      const int ms = (int)((t_end - now_s()) * 1000);
      if (ms <= 0 || poll(&pf, 1, ms) <= 0) {
        recv_rc = NVSHMEMX_ERR_TIMEOUT;
        return;
      }
      int s = accept4(g_ps.listen_fd, nullptr, nullptr, SOCK_CLOEXEC);
      if (s < 0) continue;
      int from = -1, fd = -1;
      const bool ok = recv_fd(s, &from, &fd);
      close(s);
      if (!ok || from < 0 || from >= P || from == me || peer_fds[from] >= 0) {
        recv_rc = NVSHMEMX_ERR_STATE;
        return;
      }
      peer_fds[from] = fd;
      ++got;
    }
  });
  int send_rc = 0;
  for (int q = 0; q < P && !send_rc; ++q) {
    if (q == me) continue;
    sockaddr_un a;
    fill_addr(a, sock_path(q));
    for (;;) {
      int s = socket(AF_UNIX, SOCK_STREAM | SOCK_CLOEXEC, 0);
      if (s >= 0 && connect(s, (sockaddr *)&a, sizeof a) == 0) {
        const bool ok = send_fd(s, me, my_fd);
        close(s);
        if (!ok) send_rc = NVSHMEMX_ERR_STATE;
        break;
      }
      if (s >= 0) close(s);
      if (now_s() > t_end) {
        send_rc = NVSHMEMX_ERR_TIMEOUT;
        break;
      }
      usleep(2000);
    }
  }
  receiver.join();
  if (send_rc || recv_rc)
    return fail(send_rc ? send_rc : recv_rc, "process mode: exchanging slice handles with the other PEs failed");
  return 0;
}

// Host barrier of all PE processes; fails (instead of hanging) when a PE has
// stopped or the timeout passes.
int proc_barrier(double timeout_s) {
  SharedBarrier *b = g_ps.bar;
  if (!b) return fail(NVSHMEMX_ERR_STATE, "process barrier before start");
  const unsigned g = b->gen.load(std::memory_order_acquire);
  if (b->count.fetch_add(1, std::memory_order_acq_rel) + 1 == (unsigned)g_ps.npes) {
    b->count.store(0, std::memory_order_relaxed);
    b->gen.fetch_add(1, std::memory_order_release);
    return 0;
  }
  const double t_end = now_s() + timeout_s;
  while (b->gen.load(std::memory_order_acquire) == g) {
    // a PE stops only after the barrier it last took part in completed, so
    // `left` counts only if the generation still has not moved
    if (b->left.load(std::memory_order_acquire) != 0 && b->gen.load(std::memory_order_acquire) == g)
      return fail(NVSHMEMX_ERR_STATE, "nvshmem_barrier_all: a PE process has stopped");
    if (now_s() > t_end) return fail(NVSHMEMX_ERR_TIMEOUT, "nvshmem_barrier_all: host barrier timed out");
    usleep(20);
  }
  return 0;
}

void proc_close() {
  if (g_ps.listen_fd >= 0) {
    close(g_ps.listen_fd);
    unlink(sock_path(g_ps.pe).c_str());
  }
  if (g_ps.bar) {
    g_ps.bar->left.fetch_add(1, std::memory_order_acq_rel);
    munmap(g_ps.bar, sizeof(SharedBarrier));
  }
  g_ps = ProcState();
}

}  // namespace nvshm
