/* Single-node stand-in for libnuma, used only to compile the reference's own
 * CPU sources into the test oracle (oracle/_ref).  Every call behaves as on a
 * machine with one NUMA node; numa_alloc returns zeroed memory, as libnuma's
 * mmap-backed allocator does. */
#ifndef ORACLE_SHIM_NUMA_H
#define ORACLE_SHIM_NUMA_H
#include <stdlib.h>
struct bitmask { unsigned long size; unsigned long *maskp; };
static inline int numa_max_node(void) { return 0; }
static inline int numa_node_of_cpu(int cpu) { (void)cpu; return 0; }
static inline struct bitmask *numa_bitmask_alloc(unsigned int n) {
  struct bitmask *b = (struct bitmask *)calloc(1, sizeof(struct bitmask));
  b->size = n; b->maskp = (unsigned long *)calloc(1 + n / 64, sizeof(unsigned long));
  return b;
}
static inline struct bitmask *numa_bitmask_setbit(struct bitmask *b, unsigned int i) {
  b->maskp[i / 64] |= 1UL << (i % 64); return b;
}
static inline void numa_bind(struct bitmask *b) { (void)b; }
static inline void *numa_alloc(size_t n) { return calloc(1, n); }
#endif
