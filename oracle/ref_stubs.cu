/*
 * ref_stubs.cu -- link-time stand-ins for the reference GPU-side symbols that
 * the reference app translation units name but that the CPU oracle never
 * calls (the kernel repository, selector, autotuner and cfg I/O live in
 * translation units that oracle/_ref does not build).  TEST INFRASTRUCTURE
 * ONLY.  Each stand-in aborts if it is ever reached.
 */
#include <stdio.h>
#include <stdlib.h>
#include "hml_sgemm_kernel.h"
#include "hml_sgemv_kernel.h"

texture<float, 1> texFloatA;
texture<float, 1> texFloatB;
texture<float, 1> texFloatx;

static void hml_oracle_not_built(const char *what) {
  fprintf(stderr, "oracle/_ref: %s is not part of the CPU oracle build\n", what);
  abort();
}

void hmlSgemmKernelRepoInit(void) { hml_oracle_not_built(__func__); }
void hmlSgemmKernelConfigOnline(int, int, int) { hml_oracle_not_built(__func__); }
void hmlSgemmKernelConfigReadFile(const char *) { hml_oracle_not_built(__func__); }
void hmlSgemmKernelConfigPrint(FILE *) { hml_oracle_not_built(__func__); }
void hmlSgemmKernelSelect(HmlSgemmKernelVarK *, HmlSgemmKernelConstK *,
                          HmlKernelArg *, const int, const int, const int) {
  hml_oracle_not_built(__func__);
}
void hmlSgemmKernelSelectBasic(HmlSgemmKernelVarK *, HmlKernelArg *, const int,
                               const int, const int) {
  hml_oracle_not_built(__func__);
}
void hmlSgemvKernelInit(void) { hml_oracle_not_built(__func__); }
void hmlSgemvKernelConfigOnline(int, int, int) { hml_oracle_not_built(__func__); }
void hmlSgemvKernelConfigReadFile(const char *) { hml_oracle_not_built(__func__); }
void hmlSgemvKernelConfigPrint(FILE *) { hml_oracle_not_built(__func__); }
void hmlSgemvKernelSelect(HmlSgemvKernelVarN *, HmlSgemvKernelConstN *,
                          HmlKernelArg *, const int, const int) {
  hml_oracle_not_built(__func__);
}
void hmlSgemvKernelSelectBasic(HmlSgemvKernelVarN *, HmlKernelArg *, const int,
                               const int, const int) {
  hml_oracle_not_built(__func__);
}
