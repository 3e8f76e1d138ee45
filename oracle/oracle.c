/*
 * CPU oracle: plain-C restatement of the reference's hot-path algorithms.
 * TEST INFRASTRUCTURE ONLY -- see oracle.h.  The scalar-generic body lives in
 * oracle_impl.h and is instantiated here for float and double.
 */
#define _GNU_SOURCE
#include "oracle.h"

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static __thread char orc_error_text[512];

const char* orc_last_error(void) { return orc_error_text; }

static int orc_fail(int status, const char* format, ...)
{
    va_list args;
    va_start(args, format);
    vsnprintf(orc_error_text, sizeof(orc_error_text), format, args);
    va_end(args);
    return status;
}

/* Stable bottom-up merge sort of a permutation by (key0, key1).  Equal keys keep
 * their input order, which is the std::stable_sort contract used by
 * sparse_ops_cpu.cpp:58-68 and the std::map ordering of the Schur slot set. */
static int orc_stable_sort_pairs(int64_t count, const int64_t* key0, const int64_t* key1,
                                 int64_t* permutation)
{
    int64_t* scratch = (int64_t*)malloc((size_t)(count > 0 ? count : 1) * sizeof(int64_t));
    if (!scratch)
    {
        return orc_fail(ORC_NO_MEMORY, "oracle: out of memory");
    }
    for (int64_t i = 0; i < count; ++i)
    {
        permutation[i] = i;
    }
    int64_t* source = permutation;
    int64_t* target = scratch;
    for (int64_t width = 1; width < count; width *= 2)
    {
        for (int64_t begin = 0; begin < count; begin += 2 * width)
        {
            int64_t middle = begin + width < count ? begin + width : count;
            int64_t end = begin + 2 * width < count ? begin + 2 * width : count;
            int64_t left = begin, right = middle, out = begin;
            while (left < middle && right < end)
            {
                const int64_t a = source[left];
                const int64_t b = source[right];
                /* take from the right run only when strictly smaller (stability) */
                const int right_smaller =
                    key0[b] < key0[a] || (key0[b] == key0[a] && key1[b] < key1[a]);
                target[out++] = right_smaller ? source[right++] : source[left++];
            }
            while (left < middle)
            {
                target[out++] = source[left++];
            }
            while (right < end)
            {
                target[out++] = source[right++];
            }
        }
        int64_t* swap = source;
        source = target;
        target = swap;
    }
    if (source != permutation)
    {
        memcpy(permutation, source, (size_t)count * sizeof(int64_t));
    }
    free(scratch);
    return ORC_OK;
}

#define ORC_SCALAR float
#define ORC_SFX f32
#define ORC_EPSILON 1.1920928955078125e-7
#include "oracle_impl.h"
#undef ORC_SCALAR
#undef ORC_SFX
#undef ORC_EPSILON

#define ORC_SCALAR double
#define ORC_SFX f64
#define ORC_EPSILON 2.2204460492503131e-16
#include "oracle_impl.h"
#undef ORC_SCALAR
#undef ORC_SFX
#undef ORC_EPSILON
