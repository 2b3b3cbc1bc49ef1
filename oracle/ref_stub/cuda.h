/* Empty stand-in: the reference's CPU sources include <cuda.h> through vars.h
 * but call nothing from it.  Test infrastructure only. */
#ifndef ISG_ORACLE_CUDA_STUB_H
#define ISG_ORACLE_CUDA_STUB_H
#endif
