/* Test infrastructure: lets the reference program's sources compile on Linux
 * for the oracle's reference build.  Provides the one Win32 call the
 * reference makes (GlobalMemoryStatusEx, kde_cuda_kdtr_tiled.cu:41-47). */
#pragma once
#include <unistd.h>
typedef struct {
    unsigned long dwLength;
    unsigned long long ullTotalPhys;
} MEMORYSTATUSEX;
static inline int GlobalMemoryStatusEx(MEMORYSTATUSEX* s) {
    long pages = sysconf(_SC_PHYS_PAGES);
    long page = sysconf(_SC_PAGE_SIZE);
    s->ullTotalPhys = (unsigned long long)pages * (unsigned long long)page;
    return 1;
}
