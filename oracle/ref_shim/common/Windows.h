/* POSIX stand-in for the few Win32 calls CT_Recon/hf_cpp_functions.hpp
 * makes: console cursor positioning (cosmetic progress output, made a no-op
 * here) and directory probing / creation (stat / mkdir).  Checker shim: lets
 * the reference's own sources compile unmodified on Linux. */
#pragma once
#include <sys/stat.h>
#include <sys/types.h>

typedef void* HANDLE;
typedef unsigned long DWORD;
typedef const char* LPCSTR;
typedef int BOOL;
#ifndef FALSE
#define FALSE 0
#endif
#ifndef TRUE
#define TRUE 1
#endif
#define STD_OUTPUT_HANDLE ((DWORD)-11)
#define FILE_ATTRIBUTE_DIRECTORY 0x10UL
#define INVALID_FILE_ATTRIBUTES ((DWORD)-1)

typedef struct { short X; short Y; } COORD;
typedef struct { COORD dwSize; COORD dwCursorPosition; } CONSOLE_SCREEN_BUFFER_INFO;
typedef CONSOLE_SCREEN_BUFFER_INFO* PCONSOLE_SCREEN_BUFFER_INFO;
typedef struct { DWORD nLength; void* lpSecurityDescriptor; BOOL bInheritHandle; } SECURITY_ATTRIBUTES;

static inline HANDLE GetStdHandle(DWORD) { return (HANDLE)0; }
static inline BOOL SetConsoleCursorPosition(HANDLE, COORD) { return TRUE; }
static inline BOOL GetConsoleScreenBufferInfo(HANDLE, PCONSOLE_SCREEN_BUFFER_INFO p)
{
    p->dwCursorPosition.X = 0;
    p->dwCursorPosition.Y = 0;
    return TRUE;
}
static inline DWORD GetFileAttributes(const char* path)
{
    struct stat st;
    if (stat(path, &st) != 0) return INVALID_FILE_ATTRIBUTES;
    return S_ISDIR(st.st_mode) ? FILE_ATTRIBUTE_DIRECTORY : 0UL;
}
static inline BOOL CreateDirectory(LPCSTR path, SECURITY_ATTRIBUTES*)
{
    return mkdir(path, 0755) == 0 ? TRUE : FALSE;
}
