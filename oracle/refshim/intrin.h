/* Oracle test infrastructure: MSVC <intrin.h> maps to the GCC x86 intrinsics. */
#ifndef LENIA_REFSHIM_INTRIN_H
#define LENIA_REFSHIM_INTRIN_H
#include <x86intrin.h>
#endif
