/* omp.h -- single-threaded stand-in for the OpenMP runtime calls made by the
 * reference's lib/contractions.cpp (contract_Mesons_omp), so that file builds
 * without libgomp.  TEST INFRASTRUCTURE ONLY: used by oracle/ref/Makefile. */
#ifndef QKX_REF_OMP_STUB_H
#define QKX_REF_OMP_STUB_H
static inline int omp_get_num_procs(void) { return 1; }
static inline int omp_get_max_threads(void) { return 1; }
#endif
