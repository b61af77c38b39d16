/* Empty stand-in for <numa.h>: the reference includes it but calls nothing
 * from it. TEST INFRASTRUCTURE ONLY (reference build for the oracle). */
#ifndef DGQ_REF_SHIM_NUMA_H
#define DGQ_REF_SHIM_NUMA_H
#endif
