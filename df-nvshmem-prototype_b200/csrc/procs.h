// procs.h -- process-per-PE mode (see procs.cu).
#pragma once

#include <vector>

namespace nvshm {

bool proc_mode();
int proc_pe();
// Listening socket and shared barrier in the rendezvous directory.
int proc_open(int pe, int npes, const char *dir);
// Every PE's slice descriptor, by PE (peer_fds[own PE] = my_fd).
int proc_exchange_fds(int my_fd, std::vector<int> &peer_fds, double timeout_s);
// Host barrier of all PE processes.
int proc_barrier(double timeout_s);
// Leaves the mode (a later barrier of the others then fails instead of
// waiting for this process).
void proc_close();

}  // namespace nvshm
