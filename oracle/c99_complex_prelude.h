/* Build-recipe prelude for compiling the reference's Krylov sources
 * (Source/Arnoldi/*.cpp, *.cu) with g++ 13 / nvcc 12.9 (TEST INFRASTRUCTURE).
 *
 * Those files use C99 complex arithmetic ("real complex", creal, cimag,
 * cabs, conj, I from <complex.h>) inside C++ translation units, while their
 * Macros.h defines "real" as a macro, which breaks libstdc++'s <complex>.
 * oracle/Makefile force-includes this header ahead of every such source:
 * <complex> is parsed first (so the later "real" macro cannot break it) and
 * the C99 spellings are mapped onto the GNU "_Complex" extension, which has
 * the same layout as Fortran COMPLEX*16 (what zgeev_ expects).  The
 * reference sources themselves are compiled unmodified.
 */
#ifndef NS3D_ORACLE_C99_COMPLEX_PRELUDE_H
#define NS3D_ORACLE_C99_COMPLEX_PRELUDE_H

#include <complex>

#define complex _Complex

static inline double creal(double _Complex z) { return __real__ z; }
static inline double cimag(double _Complex z) { return __imag__ z; }
static inline double cabs(double _Complex z) { return __builtin_cabs(z); }
static inline double _Complex conj(double _Complex z) { return ~z; }
static inline double _Complex c99_imaginary_unit()
{
    double _Complex z;
    __real__ z = 0.0;
    __imag__ z = 1.0;
    return z;
}
#define I (c99_imaginary_unit())

#endif
