// Test infrastructure only (oracle). Force-included when compiling the
// reference's Geometry.cpp headless: its STL loader (Geometry.cpp:271) calls
// the Windows-only _wfopen. The TLM path never loads an STL, so the shim only
// has to compile; it converts the wide path to UTF-8 and calls fopen.
#pragma once
#include <cstdio>
#include <cwchar>
#include <string>

static inline FILE *_wfopen(const wchar_t *path, const wchar_t *mode)
{
    std::string p, m;
    for (const wchar_t *c = path; *c; ++c) p.push_back((char)*c);
    for (const wchar_t *c = mode; *c; ++c) m.push_back((char)*c);
    return std::fopen(p.c_str(), m.c_str());
}
