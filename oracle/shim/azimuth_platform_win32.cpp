/* POSIX implementation of azimuth's platform API for the oracle build.
 *
 * It replaces src/azimuth_platform_win32.cpp (Win32 heap, files, threads,
 * QueryPerformanceCounter, InterlockedCompareExchange) with malloc, POSIX
 * file descriptors, pthreads, clock_gettime and a GCC compare-and-swap, and
 * keeps the Win32* function names and signatures that azimuth's
 * SetPlatformAPI(Win32) macro binds (src/azimuth_platform.h:7-23).          */
#include "azimuth_platform_win32.h"
#include <stdlib.h>
#include <time.h>
#include <unistd.h>

static b32
Win32MemoryAllocate(void **Ptr, size_t AllocSize){
    /* calloc instead of HeapAlloc: same contract, deterministic contents */
    if(!Ptr || AllocSize == 0){ return false; }
    *Ptr = calloc(1, AllocSize);
    return *Ptr != 0;
}

static b32
Win32MemoryFree(void **Ptr){
    if(!Ptr || !*Ptr){ return false; }
    free(*Ptr);
    *Ptr = 0;
    return true;
}

static b32
Win32MemoryCopy(void *Dest, size_t DestSize, void *Src, size_t SrcSize){
    if(!Dest || !Src){ return false; }
    size_t N = DestSize < SrcSize ? DestSize : SrcSize;
    memcpy(Dest, Src, N);
    return DestSize >= SrcSize;
}

static b32
Win32OpenFile(file_handle *Handle, char *Path, u32 FileAccessMode,
              u32 FileShareMode, file_creation_attrib FileCreationAttrib){
    (void)FileShareMode;
    if(!Handle || !Path){ return false; }
    b32 Read = (FileAccessMode & FileAccessMode_Read) != 0;
    b32 Write = (FileAccessMode & FileAccessMode_Write) != 0;
    const char *Mode = 0;
    switch(FileCreationAttrib){
        case FileCreationAttrib_CreateAlways:     Mode = Read ? "w+b" : "wb"; break;
        case FileCreationAttrib_CreateIfNotExist: Mode = Read ? "w+xb" : "wxb"; break;
        case FileCreationAttrib_OpenAlways:       Mode = "a+b"; break;
        case FileCreationAttrib_OpenIfExist:      Mode = Write ? "r+b" : "rb"; break;
        case FileCreationAttrib_OpenAndTruncate:  Mode = Read ? "w+b" : "wb"; break;
        default: return false;
    }
    Handle->F = fopen(Path, Mode);
    return Handle->F != 0;
}

static b32
Win32GetFileSize(file_handle FileHandle, u64 *FileSize){
    if(!FileSize || !FileHandle.F){ return false; }
    long Pos = ftell(FileHandle.F);
    if(fseek(FileHandle.F, 0, SEEK_END) != 0){ return false; }
    long End = ftell(FileHandle.F);
    fseek(FileHandle.F, Pos, SEEK_SET);
    if(End < 0){ return false; }
    *FileSize = (u64)End;
    return true;
}

static b32
Win32ReadFile32(file_handle File, void *MemoryPtr, u32 BytesToRead, u32 *BytesRead){
    if(!File.F || !MemoryPtr){ return false; }
    size_t N = fread(MemoryPtr, 1, BytesToRead, File.F);
    if(BytesRead){ *BytesRead = (u32)N; }
    return N == BytesToRead || feof(File.F);
}

static b32
Win32SetFilePointer(file_handle File, s64 SeekDistance, file_seek_pivot Pivot){
    int Whence = SEEK_SET;
    if(Pivot == FileSeekPivot_Current){ Whence = SEEK_CUR; }
    if(Pivot == FileSeekPivot_End){ Whence = SEEK_END; }
    return File.F && fseek(File.F, (long)SeekDistance, Whence) == 0;
}

static b32
Win32CloseFileHandle(file_handle Handle){
    return Handle.F && fclose(Handle.F) == 0;
}

static b32
Win32GetProcessorCoreCount(u32 *Result){
    if(!Result){ return false; }
    long N = sysconf(_SC_NPROCESSORS_ONLN);
    *Result = N > 0 ? (u32)N : 1;
    return true;
}

static b32
Win32GetAvailableMemory(u64 *Result){
    if(!Result){ return false; }
    long Pages = sysconf(_SC_AVPHYS_PAGES);
    long PageSize = sysconf(_SC_PAGESIZE);
    *Result = (Pages > 0 && PageSize > 0) ? (u64)Pages * (u64)PageSize : 0;
    return true;
}

static b32
Win32QueryTimer(timer *Timer){
    if(!Timer){ return false; }
    struct timespec Ts;
    clock_gettime(CLOCK_MONOTONIC, &Ts);
    Timer->Counter = (u64)Ts.tv_sec * 1000000000ull + (u64)Ts.tv_nsec;
    return true;
}

static b32
Win32QueryTimerFrequency(timer_freq *Freq){
    if(!Freq){ return false; }
    Freq->Value = 1000000000ull;
    return true;
}

typedef struct {
    platform_thread_proc *Proc;
    void *Params;
} az_posix_thread_start;

static void *
AzPosixThreadTrampoline(void *Arg){
    az_posix_thread_start Start = *(az_posix_thread_start *)Arg;
    free(Arg);
    Start.Proc(Start.Params);
    return 0;
}

static b32
Win32CreateThread(thread_handle *Handle, platform_thread_proc *ThreadProc,
                  void *Params, u32 *ThreadID, size_t StackSize){
    if(!Handle || !ThreadProc){ return false; }
    az_posix_thread_start *Start =
        (az_posix_thread_start *)malloc(sizeof(az_posix_thread_start));
    if(!Start){ return false; }
    Start->Proc = ThreadProc;
    Start->Params = Params;
    pthread_attr_t Attr;
    pthread_attr_init(&Attr);
    if(StackSize){ pthread_attr_setstacksize(&Attr, StackSize); }
    int Rc = pthread_create(&Handle->Thread, &Attr, AzPosixThreadTrampoline, Start);
    pthread_attr_destroy(&Attr);
    if(Rc != 0){ free(Start); Handle->Valid = 0; return false; }
    Handle->Valid = 1;
    if(ThreadID){ *ThreadID = 0; }
    return true;
}

static b32
Win32WaitForThreads(u32 ThreadCount, thread_handle *ThreadHandles,
                    b32 WaitAll, b32 WaitInfinitely, u32 WaitTimeLimit){
    (void)WaitAll; (void)WaitInfinitely; (void)WaitTimeLimit;
    b32 Success = true;
    for(u32 I = 0; I < ThreadCount; I++){
        if(ThreadHandles[I].Valid){
            if(pthread_join(ThreadHandles[I].Thread, 0) != 0){ Success = false; }
            ThreadHandles[I].Valid = 0;
        }
    }
    return Success;
}

static b32
Win32CloseThreadHandle(thread_handle Handle){
    (void)Handle;
    return true;
}

inline b32
Win32AtomicAddF32(f32 volatile *Dest, f32 Val){
    /* compare-and-swap loop on the float's bits, as the Win32 version does */
    u32 volatile *Bits = (u32 volatile *)Dest;
    for(;;){
        u32 Old = *Bits;
        f32 OldF;
        memcpy(&OldF, &Old, 4);
        f32 NewF = OldF + Val;
        u32 New;
        memcpy(&New, &NewF, 4);
        if(__sync_bool_compare_and_swap(Bits, Old, New)){ break; }
    }
    return true;
}
