/*
 * Host-compilation shim for the reference's device predicate headers.
 *
 * Test infrastructure only: this header lets the recipe in oracle/Makefile
 * compile the reference's own GDelaunay/GDelaunay/GDelShewchukDevice.h and
 * GDelPredDevice.h (read in place, never copied) as plain host C++ with g++,
 * so that the oracle's predicates and Simulation-of-Simplicity table can be
 * pinned against the reference's code without a GPU.
 *
 * It provides the handful of CUDA qualifiers those headers use, plus the
 * type and enum declarations they expect from GDelKernels.h:59-108,
 * GDelCommon.h:719-735 and Common/Geometry.h:44-69 (same names and values,
 * since the headers index their scratch arrays with them).
 */
#pragma once

#include <cmath>
#include <cstdio>
#include <cstdlib>

#define __device__
#define __host__
#define __global__
#define __forceinline__ inline
#define __noinline__ __attribute__((noinline))
#define __dmul_rn(a, b) ((a) * (b))
#define __fmul_rn(a, b) ((a) * (b))

#ifndef REAL_TYPE_DOUBLE
#define REAL_TYPE_DOUBLE
#endif
typedef double RealType;

enum Orient { OrientNeg = -1, OrientZero = +0, OrientPos = +1 };

struct Point3 { RealType _p[3]; };

struct PredicateInfo { RealType* _consts; RealType* _data; };

struct KerPointData { Point3* _pointArr; int _num; };

/* GDelKernels.h:59-80 (order matters: values index the constants array). */
enum DPredicateBounds {
    Splitter, Epsilon, Resulterrbound,
    CcwerrboundA, CcwerrboundB, CcwerrboundC,
    O3derrboundA, O3derrboundB, O3derrboundC,
    IccerrboundA, IccerrboundB, IccerrboundC,
    IsperrboundA, IsperrboundB, IsperrboundC,
    DPredicateBoundNum
};

/* GDelKernels.h:82-108 (scratch-array sizes used by the exact insphere). */
enum DPredicateSizes {
    Temp96Size = 96, Temp192Size = 192,
    Det384xSize = 384, Det384ySize = 384, Det384zSize = 384,
    DetxySize = 768, AdetSize = 1152, AbdetSize = 2304,
    CdedetSize = 3456, DeterSize = 5760,
    PredicateTotalSize = 96 + 192 + 384 * 3 + 768 + 1152 + 2304 + 3456 + 5760
};

#define CudaAssert(X)

template <typename T>
inline void cuSwap(T& a, T& b) { T t = a; a = b; b = t; }
