/* Minimal stand-in for libnuma's header so the reference compiles on a
 * machine without libnuma.  The reference only calls it for "-p 0"
 * (graphgrind/ligra-numa.h:1133-1134) and in NUMA=1 builds, which the
 * oracle recipe does not use. */
#ifndef GG_STUB_NUMA_H
#define GG_STUB_NUMA_H
struct bitmask;
static inline int numa_num_configured_nodes(void) { return 1; }
#endif
