// ORACLE -- test infrastructure.  Stand-in for the CPU-pinning helper the
// reference includes but does not ship (used at bespoke_tpch/query_impl.cpp:62-63).
#pragma once

#include <sched.h>
#include <unistd.h>

inline void pin_process_to_cpu(int cpu_id) {
  const long n = sysconf(_SC_NPROCESSORS_ONLN);
  if (cpu_id < 0 || n <= 0 || cpu_id >= n) return;
  cpu_set_t set;
  CPU_ZERO(&set);
  CPU_SET(cpu_id, &set);
  sched_setaffinity(0, sizeof(set), &set);
}

inline void unpin_process_from_cpus() {
  const long n = sysconf(_SC_NPROCESSORS_ONLN);
  cpu_set_t set;
  CPU_ZERO(&set);
  for (long i = 0; i < n && i < CPU_SETSIZE; ++i) CPU_SET(i, &set);
  sched_setaffinity(0, sizeof(set), &set);
}
