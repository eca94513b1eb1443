// ref_shim.cpp — exposes the reference's own host check (routines/dgemm/dgemm.cpp:122-133,
// dgemm::getReferenceResults) through a C symbol, for parity pinning and the timed reference arm.
// The reference translation unit is compiled where it lies (include path set by oracle/Makefile);
// nothing of it is copied. Test infrastructure only.
#include "routines/dgemm/dgemm.cpp"

extern "C" void ref_dgemm_host(const double* A, const double* B, double* C, int M, int N, int K,
                               double alpha, double beta) {
  // getReferenceResults reads the runner's static host buffers and scalars (dgemm.cpp:12-21).
  dgemm::cpuA = const_cast<double*>(A);
  dgemm::cpuB = const_cast<double*>(B);
  dgemm::cpuC = C;
  dgemm::cpuAlpha = alpha;
  dgemm::cpuBeta = beta;
  dgemm::getReferenceResults(M, N, K);
}
