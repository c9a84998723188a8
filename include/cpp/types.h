// Scalar types of the class API.  Same names and meaning as the reference's types.h
// (include/types.h of rte-rrtmgp-cpp): Float is double unless RTE_USE_SP is defined, Bool is
// int unless RTE_USE_CBOOL is defined.  Callers compiled against the reference's headers keep
// their declarations; the Float choice selects the _f32 or _f64 entry points of the C ABI.
#ifndef RRTMGP_B200_CPP_TYPES_H
#define RRTMGP_B200_CPP_TYPES_H

#include <cfloat>

#ifdef RTE_USE_CBOOL
using Bool = signed char;
#else
using Bool = int;
#endif

#ifdef RTE_USE_SP
using Float = float;
const Float Float_epsilon = FLT_EPSILON;
#else
using Float = double;
const Float Float_epsilon = DBL_EPSILON;
#endif

#endif
