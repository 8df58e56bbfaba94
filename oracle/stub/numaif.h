/* Empty stand-in for <numaif.h>; see stub/numa.h. */
#ifndef GG_STUB_NUMAIF_H
#define GG_STUB_NUMAIF_H
#endif
