/*
 * hml_sgemm.h -- drop-in replacement for the reference's public SGEMM
 * header (include/hml_sgemm.h:14-42 in the reference).  Same declarations,
 * same C++ linkage and therefore the same exported symbols:
 *   _Z20hmlSgemmKernelConfigPc, _Z13hmlSgemmBasicPfPKfS1_iiiff,
 *   _Z8hmlSgemmPfPKfS1_iiiff.
 *
 * Semantics kept from the reference: host pointers, row-major dense
 * matrices (no padding), A is M x K, B is K x N, C is M x N, synchronous
 * return after C has been written back.  C is read when beta != 0.
 * Differences: errors are reported on stderr and the call returns instead
 * of calling exit(1); a first call without configuration does not start a
 * multi-minute tuning run (it uses the B200 heuristic, or a table loaded by
 * hmlSgemmKernelConfig / hml_tune_load).
 */
#ifndef HML_SGEMM_H_INCLUDED_
#define HML_SGEMM_H_INCLUDED_

/* NULL: keep the current selection (measured table if loaded, else the
 * heuristic).  Otherwise read a tuning file: either this library's measured
 * table ("#HML-B200 tuning v2") or a reference v1 file
 * ("K colStops : kernelType rowStops"), every rule range-checked. */
void hmlSgemmKernelConfig(char *sgemmKernelConfigFileName);

/* C = alpha * A * B + beta * C with the default configuration. */
void hmlSgemmBasic(float *C, const float *A, const float *B, const int M, const int N,
                   const int K, const float alpha, const float beta);

/* C = alpha * A * B + beta * C with the tuned / predicted configuration. */
void hmlSgemm(float *C, const float *A, const float *B, const int M, const int N, const int K,
              const float alpha, const float beta);

#endif /* HML_SGEMM_H_INCLUDED_ */
