/* POSIX stand-in for azimuth's src/azimuth_platform_win32.h, used only by the
 * oracle build (test infrastructure).  It declares the handle, timer and
 * thread-procedure types that azimuth's platform API expects
 * (src/azimuth_platform.h:26-52) on top of pthreads and stdio streams. */
#pragma once
#include <pthread.h>
#include <stdio.h>
#include <string.h>

typedef struct az_posix_file_handle { FILE *F; } file_handle;
typedef struct thread_handle { pthread_t Thread; int Valid; } thread_handle;
typedef struct timer         { u64 Counter; } timer;
typedef struct timer_freq    { u64 Value; } timer_freq;

#define PlatformThreadProc(ProcName) unsigned int ProcName(void *Parameters)
typedef PlatformThreadProc(platform_thread_proc);

#ifndef ZeroMemory
#define ZeroMemory(Dest, Size) memset((Dest), 0, (Size))
#endif
