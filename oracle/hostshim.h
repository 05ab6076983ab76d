/*
 * Host-side prototypes that let the reference's serial checkers
 * (testBFS.cu, testPageRank.cu, testCsrGraph.cu) compile with g++ from the
 * unmodified reference tree.  common.h defines a __device__ double atomicAdd
 * whose body names these three intrinsics; the host pass only needs them
 * declared.  They are never called.
 */
#ifndef OLIVE_ORACLE_HOSTSHIM_H
#define OLIVE_ORACLE_HOSTSHIM_H
unsigned long long atomicCAS(unsigned long long *, unsigned long long, unsigned long long);
long long __double_as_longlong(double);
double __longlong_as_double(long long);
#endif
