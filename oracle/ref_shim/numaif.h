/* Single-node stand-in for <numaif.h> (see numa.h in this folder). */
#ifndef ORACLE_SHIM_NUMAIF_H
#define ORACLE_SHIM_NUMAIF_H
#define MPOL_F_NODE (1 << 0)
#define MPOL_F_ADDR (1 << 1)
static inline long get_mempolicy(int *mode, unsigned long *nmask, unsigned long maxnode,
                                 void *addr, unsigned long flags) {
  (void)nmask; (void)maxnode; (void)addr; (void)flags;
  if (mode) *mode = 0;
  return 0;
}
#endif
