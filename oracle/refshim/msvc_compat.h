/*
 * Oracle test infrastructure: forced-include header (gcc -include) that lets
 * the reference's MSVC sources (lenia.cpp, reintegration.cpp,
 * transposition.cpp, mesh.cpp) compile unmodified with g++ on Linux.
 *
 * Only the oracle reference build uses this file.  The product library never
 * includes it.
 */
#ifndef LENIA_REFSHIM_MSVC_COMPAT_H
#define LENIA_REFSHIM_MSVC_COMPAT_H

#include <stdio.h>
#include <string.h>
#include <stdlib.h>

/* Every __declspec in the reference is align(16) on an array or scalar. */
#define __declspec(x) __attribute__((aligned(16)))

/* MSVC bounded printf used for the reference's timing strings. */
#define sprintf_s(buf, n, ...) snprintf((buf), (n), __VA_ARGS__)

#endif
