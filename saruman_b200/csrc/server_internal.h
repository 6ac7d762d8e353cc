// Hooks abi.cu gives the request server.
#pragma once
#include <stdint.h>

#include "../../include/saruman_b200.h"

namespace saru {
// kernel launches enqueued by the calling thread so far
uint64_t thread_launches();
// counts a kernel launch made outside abi.cu
void count_launch();
void set_last_error(const char *msg);
// aligns a host call as saru_align_host does, on the server's own lane
int redo_on_host_path(const saru_batch *b, saru_result *r);
}  // namespace saru
