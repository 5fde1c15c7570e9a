/*
 * Oracle test infrastructure: the subset of <windows.h> that the reference's
 * simulation and meshing sources name (types, events, timers, debug output).
 * Threads and events are never used by the oracle driver, which replays the
 * step order serially; the definitions exist so the sources compile.
 */
#ifndef LENIA_REFSHIM_WINDOWS_H
#define LENIA_REFSHIM_WINDOWS_H

#include <stdint.h>
#include <time.h>
#include <stdio.h>

typedef void *HANDLE;
typedef void *HWND;
typedef void *HINSTANCE;
typedef void *HFONT;
typedef void *LPVOID;
typedef int32_t LONG;
typedef uint32_t DWORD;
typedef unsigned int UINT;
typedef intptr_t WPARAM;
typedef intptr_t LPARAM;
typedef intptr_t LRESULT;
typedef int BOOL;
typedef long HRESULT;

#define WINAPI
#define CALLBACK

typedef union {
    struct { uint32_t LowPart; int32_t HighPart; } u;
    long long QuadPart;
} LARGE_INTEGER;

typedef struct { int dummy; } CRITICAL_SECTION;

static inline BOOL QueryPerformanceFrequency(LARGE_INTEGER *f)
{
    f->QuadPart = 1000000000LL;
    return 1;
}

static inline BOOL QueryPerformanceCounter(LARGE_INTEGER *c)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    c->QuadPart = (long long)ts.tv_sec * 1000000000LL + ts.tv_nsec;
    return 1;
}

/* The reference prints per-stage timings to the debugger; the oracle drops them. */
static inline void OutputDebugStringA(const char *s) { (void)s; }

#endif
