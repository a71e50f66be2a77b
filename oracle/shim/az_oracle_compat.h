/*
 * Force-included ahead of azimuth's sources in the oracle build (test
 * infrastructure).  It supplies the few MSVC/Win32 names azimuth uses outside
 * its platform layer, and the hooks that the build recipe splices into
 * azimuth's Random01 (src/azimuth_math.cpp:1-8), GetSampleCoord
 * (src/azimuth_main.cpp:1135-1153) and TraceRay (src/azimuth_main.cpp:966).
 */
#ifndef AZ_ORACLE_COMPAT_H
#define AZ_ORACLE_COMPAT_H
#include <stdio.h>
#include <stdarg.h>
#include <string.h>

#define __cdecl
#ifndef ZeroMemory
#define ZeroMemory(Dest, Size) memset((Dest), 0, (Size))
#endif

static inline int fopen_s(FILE **F, const char *Name, const char *Mode) {
    *F = fopen(Name, Mode);
    return *F ? 0 : 1;
}
#define sprintf_s(Buffer, ...) snprintf((Buffer), sizeof(Buffer), __VA_ARGS__)

/* --- counter-RNG hooks (defined in oracle/ref_harness.cpp) --- */
#ifdef __cplusplus
extern "C" {
#endif
float AzOracleRandom01(void);
void  AzOracleBeginSample(unsigned Row, unsigned Col, unsigned SampleX, unsigned SampleY);
void  AzOracleEnterNode(void);
void  AzOracleLeaveNode(void);
void  AzOracleSampleDone(float R, float G, float B);
#ifdef __cplusplus
}
#endif

#ifdef __cplusplus
/* One TraceRay activation = one node of the sample's path tree. */
struct AzOracleNodeScope {
    AzOracleNodeScope() { AzOracleEnterNode(); }
    ~AzOracleNodeScope() { AzOracleLeaveNode(); }
};
#define AZ_ORACLE_NODE_SCOPE() AzOracleNodeScope AzOracleNodeScope_ ## __LINE__
#endif

#endif
