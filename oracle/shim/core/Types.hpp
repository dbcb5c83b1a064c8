/*
 * Stand-in for the reference's core/Types.hpp (include/core/Types.hpp:6), found
 * first on the include path by the oracle recipe so that the same reference
 * kernel sources build once with DATA_TYPE = double (as shipped) and once with
 * DATA_TYPE = float.  FM_REF_REAL is set on the compiler command line.
 */
#pragma once

#ifndef FM_REF_REAL
#define FM_REF_REAL double
#endif

using DATA_TYPE = FM_REF_REAL;
