/*
 * hml_sgemv.h -- drop-in replacement for the reference's public SGEMV
 * header (include/hml_sgemv.h:12-38 in the reference).  Same declarations
 * and C++ linkage, hence the same symbols: _Z20hmlSgemvKernelConfigPc,
 * _Z13hmlSgemvBasicPfPKfS1_iiff, _Z8hmlSgemvPfPKfS1_iiff.
 *
 * y = alpha * A * x + beta * y with host pointers, A row-major M x N, x of
 * length N, y of length M, synchronous.  Errors go to stderr and the call
 * returns (the reference calls exit(1)).
 */
#ifndef HML_SGEMV_H_INCLUDED_
#define HML_SGEMV_H_INCLUDED_

/* NULL keeps the current selection; otherwise reads a reference v1 SGEMV
 * file ("N : kernelType blockStops rowStops"), every rule range-checked. */
void hmlSgemvKernelConfig(char *sgemvKernelConfigFileName);

void hmlSgemvBasic(float *y, const float *A, const float *x, const int M, const int N,
                   const float alpha, const float beta);

void hmlSgemv(float *y, const float *A, const float *x, const int M, const int N,
              const float alpha, const float beta);

#endif /* HML_SGEMV_H_INCLUDED_ */
