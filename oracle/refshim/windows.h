/* Minimal POSIX stand-in for the three Win32 calls that the reference's
 * folder handling (CODE/C++/VS2010/simLB/simLB/fileHandling.cpp:12-126) makes.
 * Test infrastructure for building the reference as the parity oracle:
 * directories are not created (results are captured in memory instead). */
#ifndef REFSHIM_WINDOWS_H_
#define REFSHIM_WINDOWS_H_
#include <unistd.h>
#include <string.h>

#define MAX_PATH 4096

static inline int CreateDirectory(const char *path, void *attrs) { (void)path; (void)attrs; return 1; }
static inline int GetLastError(void) { return 0; }
static inline int GetCurrentDirectory(int n, char *buf)
{
    if (getcwd(buf, (size_t)n) == NULL) { buf[0] = '.'; buf[1] = 0; }
    return (int)strlen(buf);
}
#endif
