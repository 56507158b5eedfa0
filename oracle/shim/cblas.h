/* Stand-in for the CBLAS header (TEST INFRASTRUCTURE).  The reference's
 * Source/Arnoldi/Implicit_restart_Arnoldi.h includes <cblas.h> only for
 * OpenBLAS's thread-count calls, which it declares itself; the image has no
 * system CBLAS header, so this empty one lets that file compile unmodified.
 * oracle/arnoldi_harness.cu forwards openblas_set_num_threads to the OpenBLAS
 * that scipy ships. */
#pragma once
