// Host-build stand-in for the OptiX SDK header, used only to compile the
// reference renderer's shading headers (core/cuda/*.h) for the CPU.  It
// provides the two OptiX types those headers name and the std math overloads
// that device code finds through CUDA's headers.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
typedef int OptixResult;
enum { OPTIX_SUCCESS = 0 };
typedef unsigned long long OptixTraversableHandle;
using std::abs;
using std::exp;
using std::isnan;
using std::log;
using std::max;
using std::min;
using std::pow;
using std::sqrt;
