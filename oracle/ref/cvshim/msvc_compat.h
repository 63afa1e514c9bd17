// TEST INFRASTRUCTURE ONLY: the two MSVC C runtime names the reference's
// loader uses (rvs/src/image_loading.cpp), for building it with g++.
#pragma once
#include <cerrno>
#include <cstdio>
typedef int errno_t;
static inline errno_t fopen_s(FILE** f, const char* name, const char* mode) {
    *f = std::fopen(name, mode);
    return *f ? 0 : errno;
}
