// Stand-in for the reference's missing `ks/assertion.h`: ASSERT aborts with
// the message, as the reference's does.
#pragma once
#include <cstdio>
#include <cstdlib>

#define ASSERT(cond, ...)                                                                                             \
    do {                                                                                                              \
        if (!(cond)) {                                                                                                \
            std::fprintf(stderr, "ASSERT failed: %s: ", #cond);                                                      \
            std::fprintf(stderr, __VA_ARGS__);                                                                        \
            std::fprintf(stderr, "\n");                                                                               \
            std::abort();                                                                                             \
        }                                                                                                             \
    } while (0)
